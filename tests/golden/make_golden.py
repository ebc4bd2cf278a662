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
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
