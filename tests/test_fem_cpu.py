"""The SNK1 element restatement (oracle.fem_snk1; StiffGIPC/femEnergy.cu:
1720-1856) pinned by finite differences: gradient against the energy, the
exact Hessian against the gradient, the projected Hessian PSD and equal to
the exact one where the 9x9 Hessian in F is already positive, and equal to
the synthetic generator's element Hessian there."""
import numpy as np
import pytest

import oracle
from agipc_learning_b200 import synth


def _mesh(n=4, h=0.01, noise=0.1, seed=3):
    X, tets = synth.box_mesh(n, n, n, h)
    rng = np.random.default_rng(seed)
    x = X + noise * h * rng.uniform(-1, 1, X.shape)
    return X, tets, x


def _blocks_to_dense(rows, cols, vals, nv):
    A = np.zeros((3 * nv, 3 * nv))
    for r, c, v in zip(rows, cols, vals):
        B = np.asarray(v).reshape(3, 3).T
        A[3 * r:3 * r + 3, 3 * c:3 * c + 3] += B
        if r != c:
            A[3 * c:3 * c + 3, 3 * r:3 * r + 3] += B.T
    return A


def test_gradient_matches_energy_differences():
    X, tets, x = _mesh()
    Di, vol, u, r = oracle.fem_rest_data(tets, X, 1e5, 0.45)
    g, _, _, _ = oracle.fem_snk1(tets, x, Di, vol, u, r, 1 / 60)
    rng = np.random.default_rng(0)
    eps = 1e-7
    for k in rng.choice(x.size, 12, replace=False):
        xp, xm = x.copy().reshape(-1), x.copy().reshape(-1)
        xp[k] += eps
        xm[k] -= eps
        fd = (oracle.fem_snk1_energy(tets, xp, Di, vol, u, r, 1 / 60) -
              oracle.fem_snk1_energy(tets, xm, Di, vol, u, r, 1 / 60)) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-5 * np.abs(g).max(), (k, fd, g[k])


@pytest.mark.parametrize("noise", [0.1, 0.8])
def test_exact_hessian_matches_gradient_differences(noise):
    X, tets, x = _mesh(n=2, noise=noise, seed=7)  # 6 tets on 8 vertices; 0.8 h inverts some
    nv = len(X)
    Di, vol, u, r = oracle.fem_rest_data(tets, X, 1e5, 0.45)
    _, R, C, V = oracle.fem_snk1(tets, x, Di, vol, u, r, 1 / 60, project=False)
    H = _blocks_to_dense(R, C, V, nv)
    rng = np.random.default_rng(1)
    d = rng.standard_normal(3 * nv)
    eps = 1e-7
    gp = oracle.fem_snk1(tets, x.reshape(-1) + eps * d, Di, vol, u, r, 1 / 60)[0]
    gm = oracle.fem_snk1(tets, x.reshape(-1) - eps * d, Di, vol, u, r, 1 / 60)[0]
    fd = (gp - gm) / (2 * eps)
    assert np.abs(H @ d - fd).max() <= 1e-5 * np.abs(fd).max()


def test_projection_is_psd_and_exact_where_positive():
    X, tets, x = _mesh(n=3, noise=0.5, seed=11)
    nv = len(X)
    Di, vol, u, r = oracle.fem_rest_data(tets, X, 1e5, 0.45)
    _, R, C, Vp = oracle.fem_snk1(tets, x, Di, vol, u, r, 1 / 60)
    _, _, _, Ve = oracle.fem_snk1(tets, x, Di, vol, u, r, 1 / 60, project=False)
    nt = len(tets)
    npos = 0
    for t in range(nt):
        sl = slice(10 * t, 10 * t + 10)
        loc = {v: i for i, v in enumerate(sorted(set(tets[t])))}
        Hp = _blocks_to_dense([loc[a] for a in R[sl]], [loc[b] for b in C[sl]], Vp[sl], 4)
        He = _blocks_to_dense([loc[a] for a in R[sl]], [loc[b] for b in C[sl]], Ve[sl], 4)
        wp = np.linalg.eigvalsh(Hp)
        assert wp.min() >= -1e-10 * np.abs(wp).max()
        we = np.linalg.eigvalsh(He)
        if we.min() >= -1e-12 * np.abs(we).max():  # already PSD (rigid modes give zeros)
            npos += 1
            assert np.abs(Hp - He).max() <= 1e-9 * np.abs(He).max()
    assert 0 < npos < nt  # both kinds occur at this deformation


def test_matches_the_generator_on_positive_elements():
    """syn_fem_triplets (the synthetic systems' element Hessian) keeps the exact
    Hessian where its 9x9 is positive definite: the same values there."""
    X, tets, x = _mesh(n=4, noise=0.1, seed=5)
    Di, vol, u, r = oracle.fem_rest_data(tets, X, 1e5, 0.45)
    _, R, C, Ve = oracle.fem_snk1(tets, x, Di, vol, u, r, 1 / 60, project=False)
    (gr, _), (gc, _), (gv, _), projected = synth._fem_block(X, tets, x, 1e5, 0.45, 1 / 60, 1000.0, 0)
    assert np.array_equal(R, gr) and np.array_equal(C, gc)
    # every tet the generator did not project agrees with the exact Hessian
    diff = np.abs(Ve - gv).reshape(len(tets), 90).max(axis=1)
    scale = np.abs(Ve).reshape(len(tets), 90).max(axis=1)
    agree = diff <= 1e-10 * scale
    assert agree.sum() >= len(tets) - projected
