"""The CPU oracle against the reference's own known-answer tests (no GPU).

Pins: spmv self-test (spmv.cu:301-459), MAS32 hierarchy self-test
(TraditionalMAS32Preconditioner.cu:257-427), local-diagnostics cases
(:182-215), hierarchy_capacity asserts (tests/runtime_options_tests.cpp:33-36)
and the 257-block coarse replay fixture with its published results
(reports/agipc_reproduction/AGIPC_COARSE_MAS32_REPLAY.md:35-52); config 0
replayed by the reference's own CPU block-Jacobi PCG
(reports/agipc_reproduction/replay_frozen_coarse.py:70-111).
"""
import numpy as np
import pytest

import oracle
from tests import helpers as H


def test_spmv_kat():
    vals, rows, cols, x, y0, a, b = H.spmv_kat_system()
    assert len(rows) == 210
    ref = H.spmv_kat_expected(vals, rows, cols, x, y0, a, b)
    y = oracle.sym_spmv(a, vals, rows, cols, x, b, y0)
    assert np.max(np.abs(y - ref)) <= 1e-10


def test_hierarchy_capacity_asserts():
    assert oracle.hierarchy_capacity(38386, 38386, 4, 32) == 153600
    assert oracle.hierarchy_capacity(1001, 1024, 6, 32) == 6144
    assert oracle.hierarchy_capacity(0, 0, 4, 32) == 0


def test_compute_num_levels():
    # computeNumLevels (TraditionalMAS32Preconditioner.cu:2142-2161)
    assert oracle.compute_num_levels(64) == 3
    assert oracle.compute_num_levels(288) == 3
    assert oracle.compute_num_levels(8000) == 4
    assert oracle.compute_num_levels(32768) == 4
    assert oracle.compute_num_levels(262144) == 5
    assert oracle.compute_num_levels(2097152) == 6


def test_hierarchy_kat():
    valid, start, num, lst, pmr, rmp = H.hierarchy_kat_inputs()
    exp = H.hierarchy_kat_expected()
    m = oracle.Mas32(valid, 0, start, num, lst, pmr, rmp)
    m.reorder(None)
    hi = m.hierarchy()
    assert np.array_equal(hi["fine_mask"], exp["fine_mask"])
    assert np.array_equal(hi["coarse_space_tables"][0], exp["coarse"])
    assert np.array_equal(hi["going_next"][:valid], exp["going_next"])
    assert list(hi["prefix_original"]) == exp["prefix"]
    assert tuple(hi["level_size"][1]) == exp["level_size1"]


def test_local_diagnostics_cases():
    """run_local_diagnostics_gpu_self_test (:182-215): identity passes; a negative
    local pivot, a negative inverse pivot, a NaN inverse, a doubled inverse and a
    NaN local each fail the documented check."""
    eye9 = np.eye(3).T.reshape(9)
    diag_idx = [32 * r - r * (r + 1) // 2 + r for r in range(32)]
    local = np.zeros((6, 528, 9))
    inv = np.zeros((6, 528, 9), np.float32)
    local[:, diag_idx] = eye9
    inv[:, diag_idx] = eye9
    local[1, 0, 0] = -1
    inv[2, 0, 0] = -1
    inv[3, 0, 0] = np.nan
    inv[4, diag_idx] *= 2.0
    local[5, 0, 0] = np.nan
    res = oracle.local_checks(local, inv)

    def passed(r):
        return r["local_spd"] and r["inverse_spd"] and r["local_finite"] and r["inverse_finite"] and \
            r["inverse_residual"] <= 1e-3

    assert passed(res[0])
    assert not passed(res[1]) and res[1]["local_spd"] == 0
    assert not passed(res[2]) and res[2]["inverse_spd"] == 0
    assert not passed(res[3]) and res[3]["inverse_finite"] == 0
    assert not passed(res[4]) and res[4]["inverse_residual"] > 1e-3
    assert not passed(res[5]) and res[5]["local_finite"] == 0


def test_kat257_replay():
    k = H.kat257_padded()
    pub = k["published"]
    assert k["padded"] == pub["padded_block_nodes"]
    mas = oracle.Mas32(k["padded"], 0, k["start"], k["num"], k["lst"], k["ident"], k["ident"])
    mas.reorder(None)
    mas.prepare_hessian(k["vals"], k["rows"], k["cols"], np.arange(len(k["rows"]), dtype=np.uint32), 0)
    p64, i32 = mas.domains()
    chk = oracle.local_checks(p64, i32)
    assert len(chk) == pub["mas32"]["domains"]
    assert sum(int(c["local_spd"] and c["inverse_spd"]) for c in chk) == pub["mas32"]["spd_domains"]
    assert max(c["inverse_residual"] for c in chk) == pytest.approx(pub["mas32"]["max_local_inverse_residual"],
                                                                     rel=0.01)
    x, res = oracle.pcg(k["vals"], k["rows"], k["cols"], k["padded"], k["rhs"], precond=oracle.PRECOND_MAS32,
                        gate=oracle.GATE_EUCLID, tol=1e-3, max_iter=k["limit"], fem_count=k["padded"], mas=mas,
                        replay_checks=True)
    assert res["iterations"] == pub["mas32"]["iterations"]
    assert res["rel_res_true"] == pytest.approx(pub["mas32"]["true_relative_residual"], abs=2e-8)
    direction = np.linalg.norm(x - k["ref"]) / np.linalg.norm(k["ref"])
    assert direction == pytest.approx(pub["mas32"]["relative_direction_difference"], abs=5e-6)
    # block-Jacobi arm, also against the reference's own CPU replay output
    x, res = oracle.pcg(k["vals"], k["rows"], k["cols"], k["padded"], k["rhs"], precond=oracle.PRECOND_DIAG3,
                        gate=oracle.GATE_EUCLID, tol=1e-3, max_iter=k["limit"], replay_checks=True)
    cpu = k["cpu"]["samples"][0]["cpu_block_jacobi"]
    assert res["iterations"] == pub["block_jacobi"]["iterations"] == cpu["iterations"]
    assert res["rel_res_true"] == pytest.approx(cpu["relative_residual"], rel=1e-9)


def test_converter_semantics():
    rng = np.random.default_rng(1)
    n = 500
    rows = rng.integers(0, 20, n).astype(np.int32)
    cols = rng.integers(0, 20, n).astype(np.int32)
    vals = rng.standard_normal((n, 9))
    r, c, v = oracle.convert_triplets(rows, cols, vals)
    keys = (r.astype(np.int64) << 32) + c
    assert np.all(np.diff(keys) > 0)
    for k in range(0, len(r), 17):
        sel = (rows == r[k]) & (cols == c[k])
        acc = np.zeros(9)
        for q in np.nonzero(sel)[0]:  # input order
            acc += vals[q]
        assert np.array_equal(acc, v[k])


def test_full_bcsr_matches_symmetric_spmv():
    vals, rows, cols, x, y0, a, b = H.spmv_kat_system()
    rp, ci, fv = oracle.upper_to_full_bcsr(20, rows, cols, vals)
    y = oracle.bcsr_spmv(rp, ci, fv, x)
    ref = oracle.sym_spmv(1.0, vals, rows, cols, x)
    assert np.max(np.abs(y - ref)) <= 1e-12


def test_block_jacobi_on_config0_against_the_reference_replay():
    """Config 0 written as a coarse snapshot and solved by the reference's own
    CPU block-Jacobi PCG at the 1e-4 Euclidean gate (replay_frozen_coarse.py:
    70-111; report committed by tests/golden/make_golden.py).  The regenerated
    system hashes to the one the reference read, and the oracle's block-Jacobi
    PCG takes the replay's iteration count, with its true residual and its
    direction error against the sparse direct solution."""
    from agipc_learning_b200 import synth

    report, sums = H.load_cfg0_replay()
    assert H.cfg0_snapshot_sums() == sums
    s = synth.config_system(0)
    x, res, _ = oracle.solve_system(s, precond=oracle.PRECOND_DIAG3, gate=oracle.GATE_EUCLID, tol=1e-4)
    cpu = report["cpu_block_jacobi"]
    assert cpu["converged"] and res["iterations"] == cpu["iterations"] == 300
    # 300 iterations in another summation order: the residuals agree to 1e-3
    assert res["rel_res_true"] == pytest.approx(cpu["relative_residual"], rel=1e-3)
    xd = H.direct_solution(s)
    direction = np.linalg.norm(x - xd) / np.linalg.norm(xd)
    assert direction == pytest.approx(report["direct_reference"]["cpu_relative_direction_error"], rel=1e-3)
