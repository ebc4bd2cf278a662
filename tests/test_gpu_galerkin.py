"""The AGIPC Galerkin coarse space on the GPU through the C ABI: the coarse
matrix bit-exact against the restatement (expansion + merge) and equal to
P^T A P on the reference's known-answer test (galerkin_self_test,
agipc_galerkin.cu:1417-1470) and on an 8^3 box; restriction and
prolongation against the dense P; the coarse direction P A_c^-1 P^T b of a
MAS32 + PCG coarse solve against a dense solve."""
import numpy as np
import pytest

import oracle
from agipc_learning_b200 import galerkin, synth
from agipc_learning_b200.solver import MasPcg
from tests.test_galerkin_cpu import dense_from_upper, kat

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    with MasPcg() as m:
        yield m


def _mapping(mp):
    return galerkin.GalerkinMapping(mp["prefix"], mp["fine_to_coarse"], mp["bases"], mp["masks"], mp["rest"],
                                    mp["coarse_block_nodes"])


def _box_case():
    s = synth.config_system(0, scale=8)  # 8^3 box, 512 blocks
    X, _ = synth.box_mesh(8, 8, 8, 0.01)
    v = np.arange(512)
    i, j, k = v % 8, (v // 8) % 8, v // 64
    groups = (((k // 2) * 4 + j // 2) * 4 + i // 2).astype(np.int32)  # 64 coarse nodes: 2x2x2 vertex cubes
    masks = np.where(np.arange(64) % 2 == 0, 15, 1).astype(np.int32)
    widths = np.array([bin(m).count("1") for m in masks])
    bases = np.concatenate([[0], np.cumsum(widths)[:-1]]).astype(np.int32)
    mp = dict(prefix=0, fine_to_coarse=groups, bases=bases, masks=masks, rest=X, coarse_block_nodes=int(widths.sum()))
    return s, mp


@pytest.mark.parametrize("case", ["kat", "box"])
def test_coarse_matrix_restrict_prolong(handle, case):
    if case == "kat":
        dense, (r, c, v), mp, b = kat()
        nf = 7
    else:
        s, mp = _box_case()
        r, c, v, b, nf = s.rows, s.cols, s.vals, s.b, s.nb
        dense = dense_from_upper(r, c, v, nf)
    mapping = _mapping(mp)
    gr, gc, gv = galerkin.coarse_matrix(handle, mapping, r, c, v)
    er, ec, ev = oracle.galerkin_expand(r, c, v, mp["prefix"], mp["fine_to_coarse"], mp["bases"], mp["masks"],
                                        mp["rest"])
    orow, ocol, oval = oracle.convert_triplets(er, ec, ev)
    assert np.array_equal(gr, orow) and np.array_equal(gc, ocol) and np.array_equal(gv, oval)
    nc = mapping.coarse_blocks
    P = oracle.galerkin_prolongation(nf, nc, mp["prefix"], mp["fine_to_coarse"], mp["bases"], mp["masks"],
                                     mp["rest"])
    expected = P.T @ dense @ P
    assert np.linalg.norm(dense_from_upper(gr, gc, gv, nc) - expected) <= 1e-12 * max(1.0, np.linalg.norm(expected))
    bc = galerkin.restrict(handle, mapping, b)
    assert np.abs(bc - P.T @ b).max() <= 1e-13 * np.abs(P.T @ b).max()
    xc = np.random.default_rng(3).standard_normal(3 * nc)
    assert np.abs(galerkin.prolong(handle, mapping, xc) - P @ xc).max() <= 1e-14 * np.abs(P @ xc).max()


@pytest.mark.parametrize("case", ["kat", "box"])
def test_coarse_direction_matches_dense_solve(case):
    if case == "kat":
        dense, (r, c, v), mp, b = kat()
        nf = 7
    else:
        s, mp = _box_case()
        r, c, v, b, nf = s.rows, s.cols, s.vals, s.b, s.nb
        dense = dense_from_upper(r, c, v, nf)
    mapping = _mapping(mp)
    nc = mapping.coarse_blocks
    P = oracle.galerkin_prolongation(nf, nc, mp["prefix"], mp["fine_to_coarse"], mp["bases"], mp["masks"],
                                     mp["rest"])
    want = P @ np.linalg.solve(P.T @ dense @ P, P.T @ b)
    x, xc, res = galerkin.coarse_solve(mapping, r, c, v, b, tolerance=1e-11, max_iterations=2000)
    assert res["status_name"] == "converged", res
    assert np.linalg.norm(x - want) <= 1e-8 * np.linalg.norm(want)


def test_invalid_mapping_is_rejected(handle):
    dense, (r, c, v), mp, b = kat()
    bad = dict(mp, masks=np.array([16, 1], np.int32))
    with pytest.raises(RuntimeError):
        galerkin.coarse_matrix(handle, _mapping(bad), r, c, v)
    bad = dict(mp, fine_to_coarse=np.array([0, 0, 0, 0, 1, 2], np.int32))
    with pytest.raises(RuntimeError):
        galerkin.restrict(handle, _mapping(bad), b)
