"""The SNK1 element kernel (maspcg_fem_snk1_gradient_hessian; femEnergy.cu:
1720-1856) on the GPU against the numpy restatement: triplet structure
bit-exact, projected Hessian values within 1e-9 of each tet's largest entry
(closed-form eigensystem on the GPU, LAPACK eigendecomposition on the host),
vertex gradient within 1e-10 of its largest entry (FP64 atomics in another
order)."""
import numpy as np
import pytest

import oracle
from agipc_learning_b200 import synth
from agipc_learning_b200.solver import MasPcg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    with MasPcg() as m:
        yield m


def _case(n, noise, seed, E):
    X, tets = synth.box_mesh(n, n, n, 0.01)
    rng = np.random.default_rng(seed)
    x = X + noise * 0.01 * rng.uniform(-1, 1, X.shape)
    Di, vol, u, r = oracle.fem_rest_data(tets, X, E(len(tets), rng), 0.45)
    return tets, x, Di, vol, u, r


@pytest.mark.parametrize("n,noise,offset", [(20, 0.1, 0), (12, 0.7, 16)])
def test_fem_snk1_matches_restatement(handle, n, noise, offset):
    """20^3 box (41,154 tets, per-tet modulus log-uniform in [1e4, 1e6]) and a
    12^3 box perturbed by 0.7 h, where many elements invert and need the
    projection."""
    tets, x, Di, vol, u, r = _case(n, noise, n, lambda m, rng: 10 ** rng.uniform(4, 6, m))
    dt = 1 / 60
    g0, R0, C0, V0 = oracle.fem_snk1(tets, x, Di, vol, u, r, dt, offset)
    g1, R1, C1, V1 = handle.fem_snk1(tets, x, Di, vol, u, r, dt, offset)
    assert np.array_equal(R1, R0) and np.array_equal(C1, C0)
    nt = len(tets)
    d = np.abs(V1 - V0).reshape(nt, 90).max(axis=1)
    sc = np.abs(V0).reshape(nt, 90).max(axis=1)
    assert np.all(d <= 1e-9 * sc), (d / sc).max()
    assert np.abs(g1 - g0).max() <= 1e-10 * np.abs(g0).max()
    assert np.all(np.isfinite(V1))


def test_fem_snk1_accumulates_into_gradient(handle):
    tets, x, Di, vol, u, r = _case(4, 0.2, 1, lambda m, rng: np.full(m, 1e5))
    g0 = handle.fem_snk1(tets, x, Di, vol, u, r, 0.01)[0]
    base = np.arange(x.size, dtype=np.float64)
    g1 = handle.fem_snk1(tets, x, Di, vol, u, r, 0.01, gradient=base)[0]
    assert np.abs(g1 - (base + g0)).max() <= 1e-12 * np.abs(base + g0).max()


def test_fem_snk1_rejects_bad_vertex_id(handle):
    tets, x, Di, vol, u, r = _case(3, 0.1, 2, lambda m, rng: np.full(m, 1e5))
    bad = tets.copy()
    bad[0, 0] = len(x) + 5
    with pytest.raises(RuntimeError):
        handle.fem_snk1(bad, x, Di, vol, u, r, 0.01)
