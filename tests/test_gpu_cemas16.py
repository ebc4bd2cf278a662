"""CEMAS16 (16-vertex banks, 48x48 domains) on the GPU vs the 16-vertex CPU
oracle, through the C ABI (needs a B200).

Same bars as the MAS32 parity tests: the hierarchy bit-exact, FP64 domain
matrices to 1e-13 of the same sums over |A|, FP32 inverses and the apply to
2e-4 relative, PCG in the reference precision to the oracle's iteration count
(within 10%) and solution (1e-4 relative).  Partitions: vertex-sorted (slots
follow vertex order, as the app's METIS-sorted meshes), Morton-packed
(CEMAS16 drops reversed in-bank pairs) and gapped (slot 2 of every bank
empty: CEMAS16's row-pair rule drops rows above level 0).
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
    base = synth.config_system(1, scale=20)
    srt = synth.partition_for_bank(base, 16)
    return {"sorted": srt, "packed": synth.partition_for_bank(base, 16, sorted_ids=False),
            "gapped": H.gapped_partition(srt), "cube0": synth.partition_for_bank(synth.config_system(0), 16)}


def _oracle(s, vals=None):
    m = oracle.Mas16.from_system(s)
    m.reorder(s.pairs)
    sel = np.nonzero((s.rows >= s.fem_offset) & (s.rows < s.fem_offset + s.fem_count) &
                     (s.cols >= s.fem_offset) & (s.cols < s.fem_offset + s.fem_count))[0].astype(np.uint32)
    m.prepare_hessian(s.vals if vals is None else vals, s.rows, s.cols, sel, s.fem_offset)
    return m


@pytest.mark.parametrize("which", ["sorted", "packed", "gapped", "cube0"])
def test_hierarchy_bit_exact(systems, which):
    s = systems[which]
    o = _oracle(s).hierarchy()
    with MasPcg.from_system(s, preconditioner="cemas16") as m:
        g = m.hierarchy()
    L = o["levelnum"]
    assert g["levelnum"] == L
    assert np.array_equal(g["fine_mask"], o["fine_mask"])
    assert np.array_equal(g["coarse_space_tables"], o["coarse_space_tables"])
    assert np.array_equal(g["going_next"], o["going_next"])
    assert np.array_equal(g["level_size"][1:], o["level_size"][1:])
    assert np.array_equal(g["coarse_table"][:, :L - 1], o["coarse_table"][:, :L - 1])
    assert np.array_equal(g["prefix_original"], o["prefix_original"])
    assert g["total_clusters"] == o["total_clusters"]


@pytest.mark.parametrize("which", ["sorted", "packed", "gapped"])
def test_domain_matrices(systems, which):
    s = systems[which]
    p64, _ = _oracle(s).domains()
    bound, _ = _oracle(s, np.abs(s.vals)).domains()
    with MasPcg.from_system(s, preconditioner="cemas16") as m:
        g64 = m.domain_matrices()
    assert g64.shape == p64.shape
    assert np.all(np.abs(g64 - p64) <= 1e-13 * bound + 1e-300)


# (dropping reversed pairs or rows leaves some packed and gapped domain
# matrices indefinite, so their inverses are not compared)
@pytest.mark.parametrize("which", ["sorted", "cube0"])
def test_inverses_and_apply(systems, which):
    s = systems[which]
    o = _oracle(s)
    p64, i32 = o.domains()
    with MasPcg.from_system(s, preconditioner="cemas16") as m:
        assert m.info()["failed_domains"] == 0
        gi = m.domain_inverses()
        z = m.apply_preconditioner(s.b)
    d0 = len(s.part_map_real) // 16
    iscale = np.abs(i32[:d0]).reshape(d0, -1).max(axis=1)[:, None, None]
    assert np.max(np.abs(gi[:d0] - i32[:d0]) / iscale) <= 2e-4
    diag = [16 * a - a * (a + 1) // 2 + a for a in range(16)]
    d = gi[:, diag, :].reshape(-1, 3, 3)
    assert np.array_equal(d, d.transpose(0, 2, 1))
    z_ref = o.precondition(s.b)
    assert np.linalg.norm(z - z_ref) / np.linalg.norm(z_ref) <= 2e-4


@pytest.mark.parametrize("gate", ["rz", "euclid"])
def test_pcg_reference_precision_matches_oracle(systems, gate):
    s = systems["cube0"]
    og = oracle.GATE_RZ if gate == "rz" else oracle.GATE_EUCLID
    xo, ro, _ = oracle.solve_system(s, precond=oracle.PRECOND_MAS16, gate=og)
    with MasPcg.from_system(s, preconditioner="cemas16", gate=gate, precision="reference") as m:
        x, res = m.solve(s.b)
    assert res["status_name"] == "converged"
    assert abs(res["iterations"] - ro["iterations"]) <= max(1, int(0.1 * ro["iterations"]))
    if res["iterations"] != ro["iterations"]:
        with MasPcg.from_system(s, preconditioner="cemas16", gate=gate, precision="reference", tolerance=1e-30,
                                max_iterations=ro["iterations"] + 1) as m:
            x, _ = m.solve(s.b)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-4


@pytest.mark.parametrize("precision,sequential", [("fp32", False), ("mixed", False), ("mixed", True)])
def test_lower_precision_forms_reach_tolerance(systems, precision, sequential):
    # sequential: the coarse levels before the level-0 apply, which then adds
    # the coarse correction itself (else they run beside it on the side stream)
    from agipc_learning_b200 import _native as N
    s = systems["cube0"]
    flags = N.FLAG_SEQUENTIAL_COARSE if sequential else 0
    with MasPcg.from_system(s, preconditioner="cemas16", gate="euclid", tolerance=1e-6, precision=precision,
                            flags=flags) as m:
        x, res = m.solve(s.b)
    assert res["status_name"] == "converged"
    tol = 1e-6 if precision == "mixed" else 1e-4
    assert res["rel_res_true"] <= tol * 1.01


def test_hybrid_abd_fem_matches_oracle():
    s = synth.partition_for_bank(synth.config_system(2, scale=16), 16)
    xo, ro, _ = oracle.solve_system(s, precond=oracle.PRECOND_MAS16, gate=oracle.GATE_EUCLID, tol=1e-5)
    with MasPcg.from_system(s, preconditioner="cemas16", gate="euclid", tolerance=1e-5) as m:
        x, res = m.solve(s.b)
    assert res["status_name"] == ro["status"] == "converged"
    assert abs(res["iterations"] - ro["iterations"]) <= max(2, int(0.1 * ro["iterations"]))
    assert res["rel_res_true"] <= 1e-5 * 1.01


@pytest.mark.parametrize("bank", [32, 16])
def test_reference_call_sequence(bank):
    """The reference's caller sequence (gl_main.cu:1502-1536) on the mirror
    classes: TraditionalMAS32Preconditioner and MASPreconditioner (CEMAS16)."""
    from agipc_learning_b200.solver import MASPreconditioner, TraditionalMAS32Preconditioner
    base = synth.config_system(0)
    s = synth.partition_for_bank(base, 16) if bank == 16 else base
    p = (MASPreconditioner if bank == 16 else TraditionalMAS32Preconditioner)()
    p.initPreconditioner_Neighbor(s.fem_count, s.node_offset, len(s.neighbor_list), s.pairs, len(s.part_map_real))
    p.neighborListSize = len(s.neighbor_list)
    p.d_neighborListInit, p.d_neighborStart, p.d_neighborNumInit = s.neighbor_list, s.neighbor_start, s.neighbor_num
    p.d_partId_map_real, p.d_real_map_partId = s.part_map_real, s.real_map_part
    p.initPreconditioner_Matrix()
    p.setPreconditioner_bcoo(s.vals, s.rows, s.cols, np.arange(len(s.rows)), 0, len(s.rows), len(s.pairs))
    z = p.preconditioning(s.b)
    p.FreeMAS()
    o = _oracle(s) if bank == 16 else oracle.Mas32.from_system(s)
    if bank == 32:
        o.reorder(s.pairs)
        o.prepare_hessian(s.vals, s.rows, s.cols, None, 0)
    z_ref = o.precondition(s.b)
    assert np.linalg.norm(z - z_ref) / np.linalg.norm(z_ref) <= 2e-4


def test_apply_with_fp32_vectors(systems):
    """The apply of the FP32-vector forms (r rounded to FP32 on entry, z
    widened on exit) against the oracle's FP64-edged apply."""
    s = systems["sorted"]
    z_ref = _oracle(s).precondition(s.b)
    with MasPcg.from_system(s, preconditioner="cemas16", precision="mixed") as m:
        z = m.apply_preconditioner(s.b)
    assert np.linalg.norm(z - z_ref) / np.linalg.norm(z_ref) <= 2e-4
