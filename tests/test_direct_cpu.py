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


def test_envelope_cholesky_matches_sparse_lu_on_config0():
    """The oracle's own FP64 direct solve (reverse Cuthill-McKee + envelope
    Cholesky, orc_direct_solve) on the 20^3 system: the same solution as
    SciPy's sparse LU to 1e-10, residual at FP64 rounding level."""
    s = synth.config_system(0)
    A = sparse_from_upper(s)
    xd = spla.spsolve(A, s.b)
    stats = {}
    xc = oracle.direct_solve(s.nb, s.rows, s.cols, s.vals, s.b, stats)
    assert np.linalg.norm(A @ xc - s.b) <= 1e-12 * np.linalg.norm(s.b)
    assert np.linalg.norm(xc - xd) <= 1e-10 * np.linalg.norm(xd)
    assert 0 < stats["envelope"] < 3 * s.nb * 3 * s.nb // 2  # the ordering keeps L far from dense


def test_envelope_cholesky_matches_dense_solve_on_the_6cube():
    """The 6^3 sub-cube of the differentiation workload (648 DOF) with a
    contact pair set: the direct solve against numpy's dense FP64 solve of
    the assembled matrix.  The contact stiffness makes the system ill
    conditioned, so two backward-stable FP64 solves agree to about the
    condition number times the rounding unit (measured 3.7e-10 relative)."""
    s = synth.cube_system(6, E=1e6, nu=0.45, seed=synth.SEED_BASE + 3, pt_pairs=20, name="cube6")
    A = sparse_from_upper(s).toarray()
    xd = np.linalg.solve(A, s.b)
    xc = oracle.direct_solve(s.nb, s.rows, s.cols, s.vals, s.b)
    assert np.linalg.norm(A @ xc - s.b) <= 1e-10 * np.linalg.norm(s.b)
    assert np.linalg.norm(xc - xd) <= 1e-8 * np.linalg.norm(xd)


def test_envelope_cholesky_rejects_an_indefinite_matrix():
    s = synth.cube_system(4, E=1e6, nu=0.45, seed=synth.SEED_BASE, pt_pairs=0, name="cube4")
    vals = s.vals.copy()
    diag = np.nonzero(s.rows == s.cols)[0][0]
    vals[diag, 0] = -1e12  # one diagonal entry made hugely negative
    with pytest.raises(ValueError):
        oracle.direct_solve(s.nb, s.rows, s.cols, vals, s.b)
