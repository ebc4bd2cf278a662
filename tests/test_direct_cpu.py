"""FP64 reference solutions by a sparse direct solve (SciPy SuperLU, as the
reference's own replay tool uses at reports/agipc_reproduction/
replay_frozen_coarse.py:141): the oracle's FP64 PCG at 1e-12 reproduces it
on the 20^3 system."""
import numpy as np
import pytest

import oracle
from agipc_learning_b200 import synth

sp = pytest.importorskip("scipy.sparse")
spla = pytest.importorskip("scipy.sparse.linalg")


def sparse_from_upper(s):
    """The full symmetric matrix of an upper BCOO system (Eigen column-major blocks)."""
    r, c, v = s.rows.astype(np.int64), s.cols.astype(np.int64), s.vals.reshape(-1, 3, 3).transpose(0, 2, 1)
    ii, jj = np.meshgrid(np.arange(3), np.arange(3), indexing="ij")
    R = (3 * r[:, None, None] + ii).ravel()
    C = (3 * c[:, None, None] + jj).ravel()
    V = v.ravel()
    off = np.repeat(r != c, 9)
    A = sp.coo_matrix((np.concatenate([V, V[off]]), (np.concatenate([R, C[off]]), np.concatenate([C, R[off]]))),
                      shape=(3 * s.nb, 3 * s.nb)).tocsc()
    return A


def test_oracle_pcg_matches_direct_solve():
    s = synth.config_system(0)
    A = sparse_from_upper(s)
    xd = spla.spsolve(A, s.b)
    assert np.linalg.norm(A @ xd - s.b) <= 1e-12 * np.linalg.norm(s.b)
    xo, ro, _ = oracle.solve_system(s, gate=oracle.GATE_EUCLID, tol=1e-12)
    assert np.linalg.norm(xo - xd) <= 1e-9 * np.linalg.norm(xd)
