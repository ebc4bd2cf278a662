"""The two largest workloads at full size (needs a B200): the 64^3 cube with
50,000 point-triangle contacts (the bench workload) and the 128^3 cube with
400,000 point-triangle and edge-edge contacts.

The oracle's full solve would take hours on the host at these sizes, so the
checks are the ones that do not depend on size:
  * the integer hierarchy is bit-exact against the oracle's (whose integer
    part runs in about a second), for MAS32 and, on the 64^3 system, CEMAS16;
  * the solution meets the FP64 gate when its residual b - A x is recomputed
    by the separate FP64 SpMV entry point, and that residual agrees with the
    one the solve reports.
"""
import numpy as np
import pytest

import oracle
from agipc_learning_b200 import synth
from agipc_learning_b200.solver import MasPcg
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def systems():
    return {"cfg1": synth.config_system(1), "cfg4": synth.config_system(4)}


def _independent_residual(m, s, x):
    y = m.spmv(x, -1.0, 1.0, s.b.copy())  # b - A x in FP64
    return np.linalg.norm(y) / np.linalg.norm(s.b)


@pytest.mark.parametrize("which", ["cfg1", "cfg4"])
def test_hierarchy_bit_exact_full_size(systems, which):
    s = systems[which]
    o = oracle.Mas32.from_system(s)
    o.reorder(s.pairs)
    with MasPcg.from_system(s, precision="mixed", inverse="bf16") as m:
        H.compare_hierarchy(m.hierarchy(), o.hierarchy())


@pytest.mark.parametrize("which", ["cfg1", "cfg4"])
def test_mixed_solve_meets_the_fp64_gate_full_size(systems, which):
    s = systems[which]
    with MasPcg.from_system(s, precision="mixed", inverse="bf16", gate="euclid", tolerance=1e-4) as m:
        x, res = m.solve(s.b)
        rel = _independent_residual(m, s, x)
    assert res["status_name"] == "converged"
    assert rel <= 1e-4 * 1.01
    assert abs(rel - res["rel_res_true"]) <= 1e-3 * rel


def test_cemas16_full_size(systems):
    t = synth.partition_for_bank(systems["cfg1"], 16)
    o = oracle.Mas16.from_system(t)
    o.reorder(t.pairs)
    with MasPcg.from_system(t, preconditioner="cemas16", precision="mixed", gate="euclid", tolerance=1e-4) as m:
        H.compare_hierarchy(m.hierarchy(), o.hierarchy())
        x, res = m.solve(t.b)
        rel = _independent_residual(m, t, x)
    assert res["status_name"] == "converged"
    assert rel <= 1e-4 * 1.01
