"""The multi-GPU bench path is N independent replicas (the solve does not
shard): each rank solves its own system and the job's time is the slowest
rank's.  Its host logic runs here on two gloo ranks on the CPU, with the CPU
oracle solve standing in for the GPU solve."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    import oracle
    from agipc_learning_b200 import synth
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        w, r, lr = bench.dist_setup()
        assert (w, r, lr) == (world, rank, rank)
        s = synth.config_system(0, scale=8)
        x, res, _ = oracle.solve_system(s, gate=oracle.GATE_EUCLID)
        local_ms = 10.0 * (rank + 1)  # distinct per rank
        slowest = bench.max_over_ranks(local_ms, dist, "cpu")
        out[rank] = (slowest, res["iterations"], float(np.linalg.norm(x)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert sorted(out.keys()) == [0, 1]
    assert out[0][0] == out[1][0] == 20.0           # MAX over ranks, the same on every rank
    assert out[0][1] == out[1][1]                   # replicas: identical systems, identical solves
    assert out[0][2] == out[1][2]
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_ms_per_solve(20.0, world, 5) == 2.0
