"""The allocation-free residual entry point (maspcg_residual_norms_noalloc)
against the existing maspcg_spmv entry point, through the C ABI.

Collected last on purpose: the scratch is per device and per process, so the
test must pass both alone and after every other GPU test has used the device.
"""
import numpy as np
import pytest

from agipc_learning_b200 import _native as N
from agipc_learning_b200 import synth
from agipc_learning_b200.solver import MasPcg

pytestmark = pytest.mark.gpu

# FP64 with a different summation order than maspcg_spmv: random vectors
# have no cancellation in b - A x; a converged solve's residual is 1e-4 of b,
# which amplifies the rounding of A x by about 1e4.
RTOL_RANDOM = 1e-12
RTOL_SOLVED = 1e-9


def _spmv_residual(m, x, b):
    return float(np.linalg.norm(m.spmv(x, -1.0, 1.0, b.copy())))


def test_residual_norms_noalloc_matches_spmv():
    import torch
    s = synth.config_system(1, scale=24)
    n = 3 * s.nb
    rng = np.random.default_rng(20261203)
    with MasPcg.from_system(s, gate="euclid") as m:
        x_sol, res = m.solve(s.b)
        assert res["status_name"] == "converged"
        X = rng.standard_normal((3, n))
        B = rng.standard_normal((3, n))
        # call 1: three random pairs; call 2 (right after): the solve's own
        # solution against the right-hand side, plus one random pair
        calls = [(X, B, RTOL_RANDOM), (np.stack([x_sol, X[0]]), np.stack([s.b, B[1]]), None)]
        for xs, bs, rtol in calls:
            xd = torch.tensor(xs, dtype=torch.float64, device="cuda")
            bd = torch.tensor(bs, dtype=torch.float64, device="cuda")
            got_r, got_b = m.residual_norms_noalloc(xd, bd)
            assert got_r.shape == (len(xs),)
            for j in range(len(xs)):
                want = _spmv_residual(m, xs[j], bs[j])
                tol = rtol if rtol is not None else (RTOL_SOLVED if j == 0 else RTOL_RANDOM)
                assert got_r[j] == pytest.approx(want, rel=tol), (j, got_r[j], want)
                assert got_b[j] == pytest.approx(float(np.linalg.norm(bs[j])), rel=1e-13)
        # the solve's reported FP64 residual is the same quantity
        assert got_r[0] / got_b[0] == pytest.approx(res["rel_res_true"], rel=RTOL_SOLVED)


def test_residual_norms_noalloc_rejects_sizes_beyond_scratch():
    import torch
    s = synth.config_system(0)
    n = 3 * s.nb
    with MasPcg.from_system(s) as m:
        too_many = torch.zeros((N.RESIDUAL_MAX_VECTORS + 1, n), dtype=torch.float64, device="cuda")
        with pytest.raises(N.MaspcgError) as e:
            m.residual_norms_noalloc(too_many, too_many)
        assert e.value.status == N.ERR_CAPACITY
        hx, hb, out = np.zeros(n), np.zeros(n), np.zeros(1)
        st = m.lib.maspcg_residual_norms_noalloc(m.h, 1, hx.ctypes.data, hb.ctypes.data, out.ctypes.data, None)
        assert st == N.ERR_INVALID_ARGUMENT  # host vectors: nothing is staged
        # still usable after the rejections
        ok = torch.ones((N.RESIDUAL_MAX_VECTORS, n), dtype=torch.float64, device="cuda")
        got_r, got_b = m.residual_norms_noalloc(torch.zeros_like(ok), ok)
        assert np.allclose(got_r, np.sqrt(n), rtol=1e-13) and np.allclose(got_b, np.sqrt(n), rtol=1e-13)
