#!/usr/bin/env python3
"""Newton-step linear solve benchmark (StiffGIPC's MAS-PCG) on B200.

One step = one Newton-step solve on a fixed assembled system: upload of the
assembled BCOO into the solver (set_matrix_bcoo), MAS32 preconditioner build
(hierarchy, Galerkin domain matrices, inverses) and PCG to an FP64-verified
relative residual ||b - A x|| / ||b|| <= 1e-4.

  value   ms per solve for the whole job, inputs resident in HBM
          (mixed precision: FP32 matrix/vectors, BF16 domain inverses, FP64
          dots and residual replacement), max over ranks / (ranks * steps)
  e2e     the same through the C ABI with host (pinned) buffers
  --impl reference   the reference's algorithm (FP64 PCG + FP32 MAS32 by
          Gauss-Jordan) on the host cores: the CPU oracle port, since the
          reference needs Eigen 3.4 in device code and does not build here.

Workload: 64^3-vertex tetrahedral cube (786,432 DOF), 50,000 point-triangle
barrier pairs (the 64^3 contact system); synthetic seeded inputs.
Multi-GPU: independent replicas (the solve does not shard); weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms per Newton-step solve to 1e-4 rel. residual: mixed-prec vs FP32 MAS-PCG, 1 B200"
WORKLOAD = "cube 64^3 (262,144 verts, 786,432 DOF), 50,000 point-triangle contacts, MAS32 + PCG to FP64 1e-4"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--scale", type=int, default=None, help="smaller cube edge (debug only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-widened", action="store_true", help="skip the rows in front of the solve")
    ap.add_argument("--other-configs", default="0,2,3,4",
                    help="comma-separated other workloads reported beside the headline (empty: none)")
    return ap.parse_args()


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.first = 0
        self.proc = None

    def __enter__(self):
        """Starts sampling and returns once the first sample has arrived (at
        most 5 s): nvidia-smi's own start-up (NVML initialisation) stalls the
        GPU's work for a while, and it must not fall inside the timed region."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.rows and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.first = len(self.rows)  # the samples from here on fall in the timed region
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = self.rows[self.first:] or self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[1]) for r in rows if len(r) > 2 and r[1].replace(".", "").isdigit())
        mx = max((float(r[2]) for r in rows if len(r) > 2 and r[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows if len(r) >= 9 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(ms: float, dist=None, device=None) -> float:
    """The slowest rank's time: every rank takes part in one MAX all-reduce."""
    if dist is None:
        return float(ms)
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_ms_per_solve(max_ms: float, world: int, steps: int) -> float:
    """Whole-job ms per solve of N replicas that each ran `steps` solves in
    `max_ms` (slowest rank): the job finishes world * steps solves."""
    return max_ms / (world * steps)


def oracle_solve_ms(s, max_iter=0):
    """Reference algorithm on the host cores: MAS32 build + FP64 PCG."""
    import oracle
    t0 = time.perf_counter()
    x, res, _ = oracle.solve_system(s, gate=oracle.GATE_EUCLID, max_iter=max_iter)
    return 1000.0 * (time.perf_counter() - t0), res


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    import oracle
    from agipc_learning_b200 import synth
    oracle.build()
    s = synth.config_system(args.config, args.scale)
    cores = oracle.num_threads()
    # A step is one full host solve while the run stays within ~4 minutes;
    # beyond that each step times the build plus a bounded number of PCG
    # iterations and scales the iteration part to the full count.
    full_ms, full = oracle_solve_ms(s)
    n_full = full["iterations"]
    if (args.warmup + args.steps) * full_ms <= 240e3:
        times = [oracle_solve_ms(s)[0] for _ in range(args.warmup + args.steps)][args.warmup:]
        value = sum(times) / len(times)
        sample = f"full host solves (MAS32 build + FP64 PCG, {n_full} iterations) of {WORKLOAD}"
    else:
        sample_its = min(n_full, 100)
        build_ms, _ = oracle_solve_ms(s, max_iter=2)
        times = [oracle_solve_ms(s, max_iter=sample_its + 1)[0] for _ in range(args.warmup + args.steps)][args.warmup:]
        per_it = (sum(times) / len(times) - build_ms) / max(sample_its - 1, 1)
        value = build_ms + per_it * n_full
        sample = (f"host oracle on {WORKLOAD}: per step the build + {sample_its} PCG iterations, scaled to the "
                  f"{n_full} iterations of one full solve ({full_ms:.0f} ms)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp64 (PCG), fp32 (MAS apply)", "data": "synthetic",
            "config": {"workload": WORKLOAD, "gate": "euclid 1e-4", "iterations": n_full},
            "cpu_baseline": {"value": value, "unit": "ms", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "full_solve_ms": full_ms, "rel_res_true": full["rel_res_true"]}
    print(json.dumps(line), flush=True)
    return 0


def widened_rows(stream, dev):
    """Device times of the rows in front of the solve, on the bench workload's
    64^3 mesh (1,500,282 tets): the SNK1 element kernel, the merge of its
    15 M triplets, and the Galerkin coarse matrix of the merged matrix for
    2x2x2 vertex cubes (affine coarse nodes).  CUDA events on the stream the
    library runs on; mean of 3 launches after one warm-up."""
    import ctypes
    import numpy as np
    import torch
    from agipc_learning_b200 import fem, galerkin, synth
    from agipc_learning_b200.solver import MasPcg

    n = 64
    X, tets = synth.box_mesh(n, n, n, 0.01)
    rng = np.random.default_rng(20261204)
    x = X + 0.001 * rng.uniform(-1, 1, X.shape)
    Di, vol, u, r = fem.rest_data(tets, X, 1e6, 0.45)
    nt, nv = len(tets), len(X)
    out = {"workload": f"{n}^3 box, {nt} tets, E=1e6, nu=0.45, positions perturbed by 0.1 h"}
    with torch.cuda.stream(stream):
        D = lambda a, t: torch.from_numpy(np.ascontiguousarray(a, t)).to(dev)  # noqa: E731
        tets_d, x_d, di_d = D(tets, np.int32), D(x, np.float64), D(Di, np.float64)
        vol_d, u_d, r_d = D(vol, np.float64), D(u, np.float64), D(r, np.float64)
        m_trip = 10 * nt
        rows_d = torch.empty(m_trip, dtype=torch.int32, device=dev)
        cols_d = torch.empty_like(rows_d)
        vals_d = torch.empty((m_trip, 9), dtype=torch.float64, device=dev)
        grad_d = torch.zeros(3 * nv, dtype=torch.float64, device=dev)
        orow_d, ocol_d = torch.empty_like(rows_d), torch.empty_like(rows_d)
        oval_d = torch.empty_like(vals_d)
        P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        with MasPcg() as m:
            m.set_stream(stream.cuda_stream)
            cnt = ctypes.c_int()

            def fem_call():
                grad_d.zero_()
                m._ck(m.lib.maspcg_fem_snk1_gradient_hessian(m.h, nt, P(tets_d), nv, P(x_d), P(di_d), P(vol_d),
                                                              P(u_d), P(r_d), 1 / 60, 0, P(grad_d), P(rows_d),
                                                              P(cols_d), P(vals_d)))

            def merge_call():
                m._ck(m.lib.maspcg_convert_bcoo(m.h, P(vals_d), P(rows_d), P(cols_d), m_trip, P(oval_d), P(orow_d),
                                                P(ocol_d), ctypes.byref(cnt)))

            def timed3(fn):
                fn()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(3):
                    fn()
                e1.record(stream)
                torch.cuda.synchronize()
                return e0.elapsed_time(e1) / 3

            ms_fem = timed3(fem_call)
            ms_merge = timed3(merge_call)
            # 12 gathered positions + Dm^-1 + volume + rates + tet in, 10 triplets + gradient atomics out
            fem_bytes = nt * (16 + 96 + 72 + 24 + 10 * (8 + 72) + 96)
            out["fem_snk1"] = {"ms": ms_fem, "tets_per_s": nt / (ms_fem * 1e-3), "algorithmic_bytes": fem_bytes,
                               "GBps": fem_bytes / (ms_fem * 1e-3) / 1e9}
            out["convert_bcoo"] = {"ms": ms_merge, "triplets": m_trip, "unique_blocks": cnt.value,
                                   "triplets_per_s": m_trip / (ms_merge * 1e-3)}
            # Galerkin coarse matrix of the merged fine matrix (host arrays, copies included)
            u_rows = orow_d[:cnt.value].cpu().numpy()
            u_cols = ocol_d[:cnt.value].cpu().numpy()
            u_vals = oval_d[:cnt.value].cpu().numpy()
            v = np.arange(nv)
            i, j, k = v % n, (v // n) % n, v // (n * n)
            h2 = n // 2
            groups = (((k // 2) * h2 + j // 2) * h2 + i // 2).astype(np.int32)
            nc = h2 ** 3
            mp = galerkin.GalerkinMapping(0, groups, (4 * np.arange(nc)).astype(np.int32),
                                          np.full(nc, 15, np.int32), X, 4 * nc)
            r_d2, c_d2, v_d2 = (torch.from_numpy(u_rows).to(dev), torch.from_numpy(u_cols).to(dev),
                                torch.from_numpy(u_vals).to(dev))
            g, keep = mp._struct()
            cap = 16 * cnt.value
            crow_d = torch.empty(cap, dtype=torch.int32, device=dev)
            ccol_d = torch.empty_like(crow_d)
            cval_d = torch.empty((cap, 9), dtype=torch.float64, device=dev)
            ncoarse = ctypes.c_int()

            def gal_call():
                m._ck(m.lib.maspcg_galerkin_coarse_matrix(m.h, ctypes.byref(g), P(v_d2), P(r_d2), P(c_d2), cnt.value,
                                                          P(cval_d), P(crow_d), P(ccol_d), cap,
                                                          ctypes.byref(ncoarse)))

            ms_gal = timed3(gal_call)
            out["galerkin_coarse_matrix"] = {"ms": ms_gal, "fine_blocks": cnt.value, "coarse_blocks": ncoarse.value,
                                             "coarse_rows": 4 * nc, "mapping": "2x2x2 vertex cubes, affine"}
    return out


def cemas16_row(s, stream, dev, steps):
    """The same Newton system under CEMAS16 (16-vertex banks, 48x48 domains)
    with the vertex-sorted partition the app's METIS-sorted meshes give:
    build + solve device time in the reference precision with the reference's
    rz gate, and with FP32 vectors / FP64 refinement to the bench's FP64
    gate; the apply and factor stages alone.  CUDA events on the library's
    stream; one warm-up, then the mean of `steps`."""
    import torch
    from agipc_learning_b200 import synth
    from agipc_learning_b200.solver import MasPcg

    t = synth.partition_for_bank(s, 16)
    D = lambda a: torch.from_numpy(a).to(dev)  # noqa: E731
    vals_d, rows_d, cols_d, b_d = D(t.vals), D(t.rows), D(t.cols), D(t.b)
    x_d = torch.zeros_like(b_d)
    out = {"partition": "16-slot banks, vertices renumbered in Morton order (slot = vertex)"}
    for key, precision, gate in (("reference_rz_gate", "reference", "rz"), ("mixed_fp32_inverse", "mixed", "euclid")):
        with MasPcg(preconditioner="cemas16", precision=precision, gate=gate, tolerance=1e-4) as m:
            m.set_stream(stream.cuda_stream)
            m.set_graph(t.fem_count, t.node_offset, t.neighbor_start, t.neighbor_num, t.neighbor_list,
                        t.part_map_real, t.real_map_part)
            m.set_contacts(t.pairs)

            def step():
                m.set_matrix(vals_d, rows_d, cols_d, t.nb, t.fem_offset, t.abd_bodies)
                m.build()
                return m.solve(b_d, x_d)[1]

            step()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                res = step()
            e1.record(stream)
            torch.cuda.synchronize()
            row = {"ms_per_solve": e0.elapsed_time(e1) / steps, "iterations": res["iterations"],
                   "rel_res_true": res["rel_res_true"], "status": res["status_name"]}
            if precision == "mixed":
                info = m.info()
                ms_prec, ms_fac = m.time_stage(1, 20), m.time_stage(3, 3)
                c0 = len(t.part_map_real)
                # FP32 records (9 diagonals x 9 x 16 floats) of every domain; r read
                # twice, z written, read and written again (FP32), 24 B of coarse table
                apply_bytes = info["domains"] * 5184 + (5 * 12 + 24) * c0
                row.update({"domains": info["domains"], "levels": info["levelnum"], "precondition_ms": ms_prec,
                            "domain_factor_ms": ms_fac, "precondition_algorithmic_bytes": apply_bytes,
                            "precondition_GBps": apply_bytes / (ms_prec * 1e-3) / 1e9})
            out[key] = row
    return out


def fp32_comparison(make, step, timed, t_mixed, res_mixed, t_plain, res_plain, steps):
    """Plain FP32 beside the mixed form.  A speed-up is reported only between
    solves that both meet the FP64-verified tolerance.  When plain FP32 stops
    on its recursive residual with its FP64 residual above 1e-4 (it stalls on
    stiff contact systems), the line says so and compares the two forms at
    the tightest FP64 tolerance both reach: 2x, 5x, 20x the level plain FP32
    stalls at, the first where both solves meet it."""
    out = {"ms_per_solve": t_plain / steps, "iterations": res_plain["iterations"],
           "rel_res_true": res_plain["rel_res_true"], "status": res_plain["status_name"],
           "fp64_gate_met": bool(res_plain["fp64_gate_met"])}
    if res_plain["fp64_gate_met"] and res_mixed["fp64_gate_met"]:
        out["speedup_mixed_vs_fp32"] = t_plain / t_mixed if t_mixed > 0 else None
        return out
    stall = res_plain["rel_res_true"]
    out["speedup_mixed_vs_fp32"] = None
    out["note"] = (f"plain FP32 does not reach the FP64-verified 1e-4: its recursive residual meets the gate while "
                   f"||b - Ax||/||b|| in FP64 stalls at {stall:.2e}")
    for f in (2.0, 5.0, 20.0):
        tol = min(0.5, f * stall)
        ms, res = {}, {}
        for name, prec, inv in (("mixed", "mixed", "bf16"), ("fp32", "fp32", "fp32")):
            mm = make(prec, inv, tol=tol)
            step(mm)
            t, r = timed(mm, step, max(1, min(steps, 3)))
            ms[name], res[name] = t / max(1, min(steps, 3)), r
            mm.close()
        if res["mixed"]["fp64_gate_met"] and res["fp32"]["fp64_gate_met"]:
            out["at_common_fp64_tolerance"] = {
                "tolerance": tol, "mixed_ms": ms["mixed"], "fp32_ms": ms["fp32"],
                "mixed_iterations": res["mixed"]["iterations"], "fp32_iterations": res["fp32"]["iterations"],
                "speedup_mixed_vs_fp32": ms["fp32"] / ms["mixed"] if ms["mixed"] > 0 else None}
            break
    return out


def block_jacobi_cpu(s, stream):
    """The CPU baseline of the survey's measurement plan: FP64 CG with the
    3x3 block-Jacobi preconditioner (DiagPreconditioner) on every host core,
    Euclidean 1e-4 gate, reported only.  Its full iteration count comes from
    the same algorithm on the GPU (reference precision, block-Jacobi); the
    host times the build and a bounded number of iterations (about 20 s of
    work at most) and scales the iteration time to that count."""
    import oracle
    from agipc_learning_b200.solver import MasPcg
    with MasPcg.from_system(s, preconditioner="block_jacobi", precision="reference", gate="euclid",
                            max_iterations=200000) as m:
        _, rg = m.solve(s.b)
    n_full = rg["iterations"]
    t0 = time.perf_counter()
    oracle.solve_system(s, precond=oracle.PRECOND_DIAG3, gate=oracle.GATE_EUCLID, max_iter=2)
    t_build = time.perf_counter() - t0
    k = 50
    t0 = time.perf_counter()
    oracle.solve_system(s, precond=oracle.PRECOND_DIAG3, gate=oracle.GATE_EUCLID, max_iter=k + 1)
    per_it = max(0.0, (time.perf_counter() - t0 - t_build) / (k - 1))
    return {"value": 1000.0 * (t_build + per_it * n_full), "unit": "ms", "cores": oracle.num_threads(),
            "kind": "port", "iterations": n_full, "gpu_rel_res_true": rg["rel_res_true"],
            "sample": f"host FP64 block-Jacobi CG: the set-up plus {k} iterations timed, the per-iteration time "
                      f"scaled to the {n_full} iterations the same algorithm takes to 1e-4 (run on the GPU in FP64)"}


def other_configs(args, stream, dev, peak):
    """The other workloads, one entry each: build + solve device time (CUDA
    events, mean after a warm-up), iterations and FP64 residual in mixed
    precision (BF16 inverses) and in the reference precision, and the SpMV's
    HBM rate (the L2-resident small systems are latency-bound: their rate is
    reported, not compared with the HBM peak)."""
    import torch
    from agipc_learning_b200 import synth
    from agipc_learning_b200.solver import MasPcg
    out = {}
    for cid in [int(c) for c in args.other_configs.split(",") if c.strip()]:
        if cid == args.config:
            continue
        try:
            t0 = time.perf_counter()
            s = synth.config_system(cid)
            gen_s = time.perf_counter() - t0
            D = lambda a: torch.from_numpy(a).to(dev)  # noqa: E731
            vals_d, rows_d, cols_d, b_d = D(s.vals), D(s.rows), D(s.cols), D(s.b)
            x_d = torch.zeros_like(b_d)
            row = {"name": s.name, "block_rows": s.nb, "blocks": len(s.rows), "generate_s": gen_s}
            for key, prec, inv in (("mixed_bf16", "mixed", "bf16"), ("reference_precision", "reference", "fp32")):
                with MasPcg(gate="euclid", precision=prec, inverse=inv, tolerance=1e-4) as m:
                    m.set_stream(stream.cuda_stream)
                    if s.fem_count > 0:
                        m.set_graph(s.fem_count, s.node_offset, s.neighbor_start, s.neighbor_num, s.neighbor_list,
                                    s.part_map_real, s.real_map_part)
                        m.set_contacts(s.pairs)

                    def one():
                        m.set_matrix(vals_d, rows_d, cols_d, s.nb, s.fem_offset, s.abd_bodies)
                        m.build()
                        return m.solve(b_d, x_d)[1]

                    one()
                    reps = 3 if s.nb < 1_000_000 else 1
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    for _ in range(reps):
                        res = one()
                    e1.record(stream)
                    torch.cuda.synchronize()
                    entry = {"ms_per_solve": e0.elapsed_time(e1) / reps, "iterations": res["iterations"],
                             "rel_res_true": res["rel_res_true"], "fp64_gate_met": bool(res["fp64_gate_met"]),
                             "solve_device_ms": res["solve_ms"]}
                    if prec == "mixed":
                        info = m.info()
                        ms_spmv = m.time_stage(0, 10)
                        nbi, bf = info["internal_block_rows"], info["bcsr_blocks"]
                        by = 40 * bf + 4 * (nbi + 1) + 24 * nbi
                        entry["spmv"] = {"ms": ms_spmv, "algorithmic_bytes": by,
                                         "GBps": by / (ms_spmv * 1e-3) / 1e9 if ms_spmv else None,
                                         "frac_of_measured_hbm": by / (ms_spmv * 1e-3) / 1e9 / peak if ms_spmv else None,
                                         "us_per_iteration": 1000.0 * res["solve_ms"] / max(1, res["iterations"])}
                    row[key] = entry
            out[f"config{cid}"] = row
            del vals_d, rows_d, cols_d, b_d, x_d
            torch.cuda.empty_cache()
        except Exception as exc:  # reported, not fatal for the headline
            out[f"config{cid}"] = {"error": str(exc)}
    return out


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    from agipc_learning_b200 import synth
    from agipc_learning_b200.solver import MasPcg

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    s = synth.config_system(args.config, args.scale)
    dev = torch.device("cuda", local)
    vals_d = torch.from_numpy(s.vals).to(dev)
    rows_d = torch.from_numpy(s.rows).to(dev)
    cols_d = torch.from_numpy(s.cols).to(dev)
    b_d = torch.from_numpy(s.b).to(dev)
    x_d = torch.zeros_like(b_d)
    stream = torch.cuda.Stream(device=dev)

    def make(precision, inverse, gate="euclid", tol=1e-4, **opts):
        m = MasPcg(gate=gate, precision=precision, inverse=inverse, tolerance=tol, **opts)
        m.set_stream(stream.cuda_stream)
        m.set_graph(s.fem_count, s.node_offset, s.neighbor_start, s.neighbor_num, s.neighbor_list,
                    s.part_map_real, s.real_map_part)
        m.set_contacts(s.pairs)
        return m

    def step(m):
        m.set_matrix(vals_d, rows_d, cols_d, s.nb, s.fem_offset, s.abd_bodies)
        m.build()
        _, res = m.solve(b_d, x_d)
        return res

    def timed(m, fn, k, steps_ms=None):
        """k steps between two events on the library's stream; with a list,
        also each step's own time (an event after every step)."""
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(k + 1)]
        ev[0].record(stream)
        res = None
        for i in range(k):
            res = fn(m)
            ev[i + 1].record(stream)
        torch.cuda.synchronize()
        if steps_ms is not None:
            steps_ms.extend(round(ev[i].elapsed_time(ev[i + 1]), 3) for i in range(k))
        return max_over_ranks(ev[0].elapsed_time(ev[k]), dist, dev), res

    mixed = make("mixed", "bf16")
    plain = make("fp32", "fp32")
    for _ in range(args.warmup):
        step(mixed)
        step(plain)
    launches0 = mixed.info()["kernel_launches"]
    step_ms = []
    with ClockSampler(local) as clk:
        t_mixed, res_mixed = timed(mixed, step, args.steps, step_ms)
    launches = mixed.info()["kernel_launches"] - launches0
    t_plain, res_plain = timed(plain, step, args.steps)
    fp32_report = fp32_comparison(make, step, timed, t_mixed, res_mixed, t_plain, res_plain, args.steps)
    # the step when only the values change (same triplets, graph and contacts):
    # refresh_fixed_graph_bcoo + solve
    def step_refresh(m):
        m.refresh_values(vals_d)
        _, res = m.solve(b_d, x_d)
        return res

    step_refresh(mixed)
    t_refresh, res_refresh = timed(mixed, step_refresh, args.steps)
    # the opt-in forms of the mixed solve on the same step: exact FP64 sums in
    # the SpMV, the BF16 remainder of the matrix, reliable-update replacement
    variants = {}
    for key, opts in (("reliable_replacement", {"replacement": "reliable"}),
                      ("matrix_f32_accurate", {"matrix": "f32_accurate", "replacement": "reliable"}),
                      ("matrix_f32_compensated", {"matrix": "f32_compensated"}),
                      ("matrix_f32_split", {"matrix": "f32_split"})):
        mv = make("mixed", "bf16", **opts)
        step(mv)
        t_v, res_v = timed(mv, step, max(1, min(args.steps, 3)))
        variants[key] = {"ms_per_solve": t_v / max(1, min(args.steps, 3)), "iterations": res_v["iterations"],
                         "refinements": res_v["refinements"], "rel_res_true": res_v["rel_res_true"],
                         "fp64_gate_met": bool(res_v["fp64_gate_met"]), "options": opts}
        mv.close()
    # the reference's own stopping rule (rz gate) in the reference precision
    refp = make("reference", "fp32", gate="rz")
    step(refp)
    k_ref = max(1, min(args.steps, 3))
    t_ref, res_ref = timed(refp, step, k_ref)
    refp.close()

    # end to end through the C ABI with host (pinned) buffers
    vals_h = torch.from_numpy(s.vals).pin_memory().numpy()
    rows_h = torch.from_numpy(s.rows).pin_memory().numpy()
    cols_h = torch.from_numpy(s.cols).pin_memory().numpy()
    b_h = torch.from_numpy(s.b).pin_memory().numpy()
    x_h = torch.zeros(len(s.b), dtype=torch.float64).pin_memory().numpy()

    def step_host(m):
        m.set_matrix(vals_h, rows_h, cols_h, s.nb, s.fem_offset, s.abd_bodies)
        m.build()
        _, res = m.solve(b_h, x_h)
        return res

    step_host(mixed)
    t_e2e, res_e2e = timed(mixed, step_host, args.steps)

    # roofline of the dominant kernel (SpMV + p.Ap) and the other stages
    info = mixed.info()
    stage_errors = {}

    def stage(k, reps):
        try:
            return mixed.time_stage(k, reps)
        except Exception as exc:  # reported in the line, not fatal
            stage_errors[k] = str(exc)
            return None

    ms_spmv = stage(0, 20)
    ms_prec = stage(1, 20)
    ms_l0 = stage(2, 20)
    ms_factor = stage(3, 3)
    ms_replace = stage(7, 10)
    ms_l0_variants = {"tma_staged_x2": stage(4, 20), "tma_staged_x1": stage(5, 20), "direct_loads": stage(6, 20)}
    nbi, bf = info["internal_block_rows"], info["bcsr_blocks"]
    d0 = s.fem_count // 32 if s.fem_count % 32 == 0 else (s.fem_count + 31) // 32
    spmv_bytes = 40 * bf + 4 * (nbi + 1) + 8 * (3 * nbi)
    # per domain: the 16-bit record (21 tiles of 16x16, 10,752 B), 96 column scales, r and z (FP32) and the slot map
    l0_bytes = d0 * (10752 + 96 * 4) + 3 * 4 * 32 * d0 * 3
    peak, peak_kind = peaks()
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "k_spmv_cube64_contacts_traffic.json")
    if os.path.exists(tfile):
        try:
            traffic = json.load(open(tfile)).get("dram_bytes_per_launch_full_workload")
        except Exception:
            traffic = None
    ach = spmv_bytes / (ms_spmv * 1e-3) / 1e9 if ms_spmv else None

    value = job_ms_per_solve(t_mixed, world, args.steps)
    line = {
        "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_mixed / args.steps, "step_ms": step_ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32 (matrix, vectors) + bf16 (MAS inverses) + fp64 (dots, residual)", "data": "synthetic",
        "config": {"workload": WORKLOAD, "replicas": world, "gate": "FP64-verified ||b-Ax||/||b|| <= 1e-4",
                   "l2": "inputs larger than L2: FP64 BCOO %.0f MB uploaded per step" % (72 * len(s.rows) / 1e6),
                   "precision": "mixed", "inverse": "bf16", "refinement_period": 16, "matrix_form": "f32",
                   "residual_replacement": "periodic"},
        "iterations": res_mixed["iterations"], "rel_res_true": res_mixed["rel_res_true"],
        "refinements": res_mixed["refinements"],
        "fp32_plain": fp32_report,
        "mixed_variants": variants,
        "refresh_step": {"ms_per_solve": t_refresh / args.steps, "iterations": res_refresh["iterations"],
                         "rel_res_true": res_refresh["rel_res_true"],
                         "what": "maspcg_refresh_matrix_values (values only: merge values, domain factors) + solve"},
        "solves_per_s": 1000.0 * world * args.steps / t_mixed if t_mixed > 0 else None,
        "rz_gate_reference_precision": {"ms_per_solve": t_ref / k_ref, "iterations": res_ref["iterations"],
                                        "rel_res_true": res_ref["rel_res_true"], "status": res_ref["status_name"],
                                        "gate": "reference rz gate |r.z| <= 1e-4 r0.z0, FP64 PCG + FP32 MAS"},
        "stages_ms": {"spmv": ms_spmv, "precondition": ms_prec, "mas_level0": ms_l0,
                      "mas_level0_variants": ms_l0_variants, "domain_factor": ms_factor,
                      "residual_replacement": ms_replace,
                      "solve_device_ms": res_mixed["solve_ms"]},
        "stage_errors": stage_errors or None,
        "roofline": {"kernel": "k_spmv (BCSR SpMV + p.Ap, FP32 32-block tiles)", "bound": "hbm", "achieved": ach,
                     "peak": peak,
                     "unit": "GB/s", "frac": ach / peak if ach else None, "traffic": traffic, "peak_kind": peak_kind,
                     "algorithmic_bytes": spmv_bytes,
                     "mas_level0_GBps": l0_bytes / (ms_l0 * 1e-3) / 1e9 if ms_l0 else None},
        "e2e": {"value": job_ms_per_solve(t_e2e, world, args.steps), "unit": "ms",
                "h2d_bytes_per_step": int(80 * len(s.rows) + 24 * s.nb), "d2h_bytes_per_step": int(24 * s.nb)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if not args.no_widened:
        try:
            line["widened_rows"] = widened_rows(stream, dev)
        except Exception as exc:  # reported, not fatal for the headline
            line["widened_rows"] = {"error": str(exc)}
        try:
            line["cemas16"] = cemas16_row(s, stream, dev, max(1, min(args.steps, 3)))
        except Exception as exc:
            line["cemas16"] = {"error": str(exc)}
    if args.other_configs and rank == 0:
        line["other_configs"] = other_configs(args, stream, dev, peak)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        oracle.build()
        ms_cpu, rc = oracle_solve_ms(s)
        line["cpu_baseline"] = {"value": ms_cpu, "unit": "ms", "cores": oracle.num_threads(), "kind": "port",
                                "sample": f"one full host solve (MAS32 build + FP64 PCG, {rc['iterations']} "
                                          f"iterations) of the same workload"}
        line["cpu_block_jacobi_cg"] = block_jacobi_cpu(s, stream)
    if rank == 0:
        print(json.dumps(line), flush=True)
    mixed.close()
    plain.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    return run_ours(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
