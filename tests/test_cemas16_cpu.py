"""CEMAS16 (MASPreconditioner, 16-vertex banks, 48x48 domains) in the CPU
oracle, no GPU.

The 16-vertex oracle (liboracle16.so) is the MAS32 restatement, pinned by the
MAS32 known-answer tests, compiled with a 16-vertex bank plus CEMAS16's three
differences.  Here it is checked against the hierarchy and the domain
matrices by their meaning (tests/helpers.py: connected components per bank,
Galerkin sums with CEMAS16's rules), on three partitions of one contact
system: vertex-sorted (slots follow the vertex order, as the app's
METIS-sorted meshes), Morton-packed (slot order runs against vertex order
inside banks) and gapped (slot 2 of every bank empty).
"""
import numpy as np
import pytest

import oracle
from agipc_learning_b200 import synth
from tests import helpers as H


@pytest.fixture(scope="module")
def systems():
    base = synth.config_system(1, scale=10)
    srt = synth.partition_for_bank(base, 16)
    return {"base": base, "sorted": srt, "packed": synth.partition_for_bank(base, 16, sorted_ids=False),
            "gapped": H.gapped_partition(srt)}


def _oracle(s, cls):
    m = cls.from_system(s)
    m.reorder(s.pairs)
    sel = np.nonzero((s.rows >= s.fem_offset) & (s.rows < s.fem_offset + s.fem_count) &
                     (s.cols >= s.fem_offset) & (s.cols < s.fem_offset + s.fem_count))[0].astype(np.uint32)
    m.prepare_hessian(s.vals, s.rows, s.cols, sel, s.fem_offset)
    return m


def test_compute_num_levels_bank16():
    # MASPreconditioner::computeNumLevels (:1727-1746) by hand: 256 slots ->
    # 16 -> stop (3 levels); 257 -> 272 -> 17 -> 32 -> 2 -> 16 (4 levels)
    assert oracle.compute_num_levels(16, 16) == 2
    assert oracle.compute_num_levels(256, 16) == 3
    assert oracle.compute_num_levels(257, 16) == 4
    assert oracle.compute_num_levels(4096, 16) == 4
    assert oracle.compute_num_levels(4097, 16) == 5
    assert oracle.compute_num_levels(1 << 24, 16) == 6


@pytest.mark.parametrize("which", ["sorted", "packed", "gapped"])
def test_hierarchy_is_components_per_bank(systems, which):
    s = systems[which]
    hi = _oracle(s, oracle.Mas16).hierarchy()
    lev = H.mas_levels(s, 16)
    L = lev["levelnum"]
    assert hi["levelnum"] == L
    assert np.array_equal(hi["fine_mask"], lev["fine_mask"])
    assert np.array_equal(hi["coarse_space_tables"], lev["ids"])
    assert np.array_equal(hi["level_size"][1:], lev["level_size"][1:])
    assert np.array_equal(hi["prefix_original"], lev["prefix"])


def test_components_restatement_matches_the_pinned_mas32_oracle(systems):
    s = systems["base"]
    hi = _oracle(s, oracle.Mas32).hierarchy()
    lev = H.mas_levels(s, 32)
    assert np.array_equal(hi["fine_mask"], lev["fine_mask"])
    assert np.array_equal(hi["coarse_space_tables"], lev["ids"])
    assert np.array_equal(hi["level_size"][1:], lev["level_size"][1:])


@pytest.mark.parametrize("which", ["sorted", "packed", "gapped"])
def test_domain_matrices_are_galerkin_sums_with_cemas16_rules(systems, which):
    s = systems[which]
    p64, _ = _oracle(s, oracle.Mas16).domains()
    lev = H.mas_levels(s, 16)
    ref = H.galerkin_domains(s, lev, 16, cemas16=True)
    plain = H.galerkin_domains(s, lev, 16, cemas16=False)
    assert p64.shape == ref.shape
    assert np.max(np.abs(p64 - ref)) <= 1e-12 * np.max(np.abs(ref))
    changed = np.max(np.abs(plain - ref)) > 1e-9 * np.max(np.abs(ref))
    # the sorted partition loses nothing; the packed one drops reversed
    # in-bank pairs; the gapped one drops rows 3, 19, ... above level 0
    assert changed == (which != "sorted")


def test_mas32_keeps_reversed_pairs(systems):
    s = systems["base"]  # Morton-packed 32-slot banks
    p64, _ = _oracle(s, oracle.Mas32).domains()
    lev = H.mas_levels(s, 32)
    ref = H.galerkin_domains(s, lev, 32, cemas16=False)
    assert np.max(np.abs(p64 - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_inverses(systems):
    # (the gapped partition's coarse matrices lose rows to CEMAS16's pair
    # rule and need not stay positive definite)
    s = systems["sorted"]
    p64, i32 = _oracle(s, oracle.Mas16).domains()
    # CEMAS16 stores the diagonal 3x3 blocks exactly symmetric
    diag = [16 * a - a * (a + 1) // 2 + a for a in range(16)]
    d = i32[:, diag, :].reshape(-1, 3, 3)
    assert np.array_equal(d, d.transpose(0, 2, 1))
    checks = oracle.local_checks(p64, i32, bank=16)
    assert all(c["local_spd"] and c["inverse_spd"] for c in checks)
    # FP32 inverse quality on the level-0 domains (the coarsest, contact-
    # stiffened ones reach ~1e-1 in FP32, as with the 32-vertex bank)
    d0 = len(s.part_map_real) // 16
    assert max(c["inverse_residual"] for c in checks[:d0]) <= 1e-4


def test_pcg_with_cemas16_converges():
    s = synth.partition_for_bank(synth.config_system(0, 12), 16)
    x, r, _ = oracle.solve_system(s, precond=oracle.PRECOND_MAS16, gate=oracle.GATE_EUCLID, tol=1e-6)
    xj, rj, _ = oracle.solve_system(s, precond=oracle.PRECOND_DIAG3, gate=oracle.GATE_EUCLID, tol=1e-6)
    assert r["status"] == "converged" and r["rel_res_true"] <= 1e-6 * (1 + 1e-6)
    assert r["iterations"] < rj["iterations"]
