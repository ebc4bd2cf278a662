"""The GPU solve against an FP64 sparse direct solve (SciPy SuperLU, and on
the 20^3 system also the oracle's envelope Cholesky) of the
20^3 system (both precisions, to 1e-12 and 1e-10) and of the hybrid ABD + FEM
system scaled down (reference precision, 1e-8).  The solution error is
bounded by the condition number times the residual; the hybrid system's
affine bodies make it far worse conditioned, so its bounds are looser.  Mixed
precision on the hybrid system is not run to a tight tolerance here: it did
not reach a 1e-6 true residual within 20,000 iterations (measured), as the
FP32 iteration between FP64 residual replacements loses too much on a
system this ill-conditioned."""
import numpy as np
import pytest

import oracle
from agipc_learning_b200 import synth
from agipc_learning_b200.solver import MasPcg
from tests.test_direct_cpu import sparse_from_upper

pytestmark = pytest.mark.gpu
spla = pytest.importorskip("scipy.sparse.linalg")

CASES = [  # system, precision, tolerance, allowed true residual / tolerance, bound on ||x - x_direct|| / ||x_direct||
    ("cfg0", "reference", 1e-12, 1.05, 1e-9),
    ("cfg0", "mixed", 1e-10, 1.05, 1e-8),
    # reference precision stops on the recursive residual, as the reference
    # does; on the hybrid system (affine bodies, condition ~1e11) the true
    # residual drifts above it (measured 1.7x at 1e-8)
    ("cfg2_small", "reference", 1e-8, 5.0, 1e-5),
]


@pytest.mark.parametrize("which,precision,tol,drift,bound", CASES)
def test_solution_matches_direct_solve(which, precision, tol, drift, bound):
    s = synth.config_system(0) if which == "cfg0" else synth.config_system(2, scale=16)
    A = sparse_from_upper(s)
    xd = spla.spsolve(A, s.b)
    with MasPcg.from_system(s, gate="euclid", precision=precision, inverse="bf16", tolerance=tol,
                            max_iterations=20000) as m:
        x, res = m.solve(s.b)
    assert res["status_name"] == "converged", res
    assert np.linalg.norm(A @ x - s.b) <= drift * tol * np.linalg.norm(s.b)
    assert np.linalg.norm(x - xd) <= bound * np.linalg.norm(xd)
    if which == "cfg0":
        # also against the oracle's own FP64 Cholesky (RCM + envelope)
        xc = oracle.direct_solve(s.nb, s.rows, s.cols, s.vals, s.b)
        assert np.linalg.norm(x - xc) <= bound * np.linalg.norm(xc)
