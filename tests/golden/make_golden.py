#!/usr/bin/env python3
"""Regenerate the golden fixtures under tests/golden/ from the reference.

Usage: make_golden.py REFERENCE_ROOT, the path of a read-only checkout of the
reference project.  The GPU box never runs this: the outputs are committed.

kat257/  -- the reference's own coarse-replay known-answer system
            (reports/agipc_reproduction/make_coarse_replay_fixture.py, default
            257 blocks) and the reference's own CPU replay of it
            (reports/agipc_reproduction/replay_frozen_coarse.py --direct-reference),
            plus the published GPU MAS32 / Jacobi results of that system
            (reports/agipc_reproduction/AGIPC_COARSE_MAS32_REPLAY.md:35-52).
cfg0_replay/ -- the 20^3 cube (config 0) written as a coarse snapshot
            (agipc_learning_b200.frozen_io.write_coarse_snapshot) and replayed by
            the reference's own CPU block-Jacobi PCG at the 1e-4 Euclidean gate
            (replay_frozen_coarse.py --direct-reference).  Only the replay's
            report and the SHA-256 of the exported arrays are kept: the tests
            regenerate the system from its seed and check it against them.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main() -> int:
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        print("usage: make_golden.py REFERENCE_ROOT (a checkout of the reference project)", file=sys.stderr)
        return 2
    REF = sys.argv[1]
    tools = os.path.join(REF, "reports", "agipc_reproduction")
    out = os.path.join(HERE, "kat257")
    subprocess.run([sys.executable, os.path.join(tools, "make_coarse_replay_fixture.py"), out], check=True)
    subprocess.run([sys.executable, os.path.join(tools, "replay_frozen_coarse.py"), out, "--direct-reference",
                    "--quiet", "--output", os.path.join(out, "reference_cpu_replay.json")], check=True)
    published = {
        "source": "reports/agipc_reproduction/AGIPC_COARSE_MAS32_REPLAY.md:35-52",
        "padded_block_nodes": 288,
        "block_jacobi": {"iterations": 47, "true_relative_residual": 9.431245e-4,
                         "relative_direction_difference": 0.003456},
        "mas32": {"iterations": 14, "true_relative_residual": 9.428987e-4,
                  "relative_direction_difference": 0.001798, "spd_domains": 12, "domains": 12,
                  "max_local_inverse_residual": 7.06e-7},
        "stopping": "Euclidean ||r||/||b|| <= 1e-3 on the recursive residual (agipc_coarse_replay.cu:135-147)",
    }
    with open(os.path.join(out, "published.json"), "w") as f:
        json.dump(published, f, indent=2)
        f.write("\n")
    make_cfg0_replay(tools)
    return 0


def cfg0_snapshot(directory: str) -> dict:
    """Config 0 as a coarse snapshot; returns the SHA-256 of each array file."""
    import hashlib

    import numpy as np

    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from agipc_learning_b200 import frozen_io, synth

    from scipy.sparse.linalg import spsolve

    from oracle.mixed_emulation import full_matrix

    s = synth.config_system(0)
    x_direct = spsolve(full_matrix(s).tocsc(), s.b)  # the saved solution the replay compares against
    meta = {"format": "agipc_coarse_system_v1", "sample_name": "cfg0", "category": "config 0, 20^3 cube",
            "coarse_block_nodes": int(s.nb), "coarse_matrix_half_storage": True,
            "coarse_solve": {"max_iterations": 5000, "relative_tolerance": 1e-4}}
    snap = frozen_io.CoarseSnapshot(meta, s.rows.astype(np.int32), s.cols.astype(np.int32),
                                    s.vals.reshape(-1, 9), s.b, np.asarray(x_direct, np.float64))
    frozen_io.write_coarse_snapshot(directory, snap)
    meta["coarse_unique_blocks"] = int(len(snap.rows))
    with open(os.path.join(directory, "manifest.json"), "w") as f:  # a sample root holding this one sample
        json.dump({"format": "agipc_coarse_samples_v1", "samples": [dict(meta, sample_name=".")]}, f, indent=2)
    sums = {}
    for f in ("coarse_A_values.f64x9.bin", "coarse_A_rows.i32.bin", "coarse_A_cols.i32.bin", "coarse_rhs.f64.bin"):
        with open(os.path.join(directory, f), "rb") as fh:
            sums[f] = hashlib.sha256(fh.read()).hexdigest()
    return sums


def make_cfg0_replay(tools: str) -> None:
    import tempfile

    out = os.path.join(HERE, "cfg0_replay")
    os.makedirs(out, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        snap_dir = os.path.join(tmp, "cfg0")
        sums = cfg0_snapshot(snap_dir)
        subprocess.run([sys.executable, os.path.join(tools, "replay_frozen_coarse.py"), snap_dir,
                        "--direct-reference", "--quiet", "--output", os.path.join(out, "reference_cpu_replay.json")],
                       check=True)
    with open(os.path.join(out, "manifest.json"), "w") as f:
        json.dump({"system": "synth.config_system(0) as a coarse snapshot (make_golden.cfg0_snapshot)",
                   "sha256": sums}, f, indent=2)
        f.write("\n")


if __name__ == "__main__":
    raise SystemExit(main())
