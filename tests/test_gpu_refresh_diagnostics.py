"""The rest of the MAS object API through the C ABI (needs a B200):

* refresh_fixed_graph_bcoo: new values on a kept structure give the same
  preconditioner and solve, bit for bit, as a full set_matrix + build;
* setPreconditioner_bcoo's (indices, offset) sub-range, gathered on the
  device from device arrays;
* local_diagnostics_gpu / gpu_local_checks: the reference's six self-test
  cases (TraditionalMAS32Preconditioner.cu:185-215) and the oracle's
  restatement of check_local_matrices on real domains.
"""
import numpy as np
import pytest

import oracle
from agipc_learning_b200 import synth
from agipc_learning_b200.solver import MasPcg, TraditionalMAS32Preconditioner

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cfg1_small():
    return synth.config_system(1, scale=24)


def _scaled_values(s, seed):
    """The same structure with new values that keep A SPD: the whole matrix
    scaled by a seeded factor near 1, and a seeded positive multiple of the
    identity added to every diagonal block."""
    rng = np.random.default_rng(seed)
    v = s.vals * (1.0 + 0.1 * rng.random())
    diag = s.rows == s.cols
    shift = 0.05 * np.abs(v[diag][:, [0, 4, 8]]).mean() * rng.random()
    v[diag] += shift * np.eye(3).reshape(9)
    return v


@pytest.mark.parametrize("precision,inverse", [("reference", "fp32"), ("mixed", "bf16")])
def test_refresh_matches_full_rebuild_bit_for_bit(cfg1_small, precision, inverse):
    s = cfg1_small
    v2 = _scaled_values(s, 3)
    cfg = dict(precision=precision, inverse=inverse, gate="euclid")
    with MasPcg.from_system(s, **cfg) as m:
        m.solve(s.b)
        m.refresh_values(v2)
        inv_r = m.domain_inverses()
        _, _, val_r, _ = m.bcsr()
        x_r, res_r = m.solve(s.b)
    with MasPcg(**cfg) as m:
        m.set_graph(s.fem_count, s.node_offset, s.neighbor_start, s.neighbor_num, s.neighbor_list, s.part_map_real,
                    s.real_map_part)
        m.set_contacts(s.pairs)
        m.set_matrix(v2, s.rows, s.cols, s.nb, s.fem_offset, s.abd_bodies)
        m.build()
        inv_f = m.domain_inverses()
        _, _, val_f, _ = m.bcsr()
        x_f, res_f = m.solve(s.b)
    assert np.array_equal(val_r, val_f)
    assert np.array_equal(inv_r, inv_f)
    assert res_r["iterations"] == res_f["iterations"]
    assert np.array_equal(x_r, x_f)


def test_refresh_keeps_hybrid_bodies_in_step():
    s = synth.config_system(2, scale=16)
    v2 = _scaled_values(s, 4)
    with MasPcg.from_system(s, gate="euclid") as m:
        m.refresh_values(v2)
        x_r, r_r = m.solve(s.b)
    with MasPcg.from_system(s, gate="euclid") as m:
        m.set_matrix(v2, s.rows, s.cols, s.nb, s.fem_offset, s.abd_bodies)
        m.build()
        x_f, r_f = m.solve(s.b)
    assert r_r["iterations"] == r_f["iterations"] and np.array_equal(x_r, x_f)


def test_mirror_device_arrays_and_refresh(cfg1_small):
    """The reference caller sequence with device arrays: the subsystem's
    triplets sit inside a larger list (other triplets before and after),
    picked by indices with an offset, as LocalPreconditioner hands them."""
    import torch
    s = cfg1_small
    rng = np.random.default_rng(8)
    off = 5
    junk = 1000
    n = len(s.rows)
    perm = rng.permutation(n + junk)
    big_vals = np.zeros((n + junk, 9))
    big_rows = np.full(n + junk, -7, np.int32)
    big_cols = np.full(n + junk, -7, np.int32)
    where = perm[:n]
    big_vals[where] = s.vals
    big_rows[where] = s.rows + off
    big_cols[where] = s.cols + off
    idx = where.astype(np.uint32)
    r = rng.standard_normal(3 * s.nb)
    with MasPcg.from_system(s) as ref:
        z_ref = ref.apply_preconditioner(r)
    P = TraditionalMAS32Preconditioner()
    P.initPreconditioner_Neighbor(s.fem_count, s.node_offset, len(s.neighbor_list), s.pairs, len(s.part_map_real))
    P.neighborListSize = len(s.neighbor_list)
    P.d_neighborListInit, P.d_neighborStart, P.d_neighborNumInit = s.neighbor_list, s.neighbor_start, s.neighbor_num
    P.d_partId_map_real, P.d_real_map_partId = s.part_map_real, s.real_map_part
    P.initPreconditioner_Matrix()
    dv = torch.from_numpy(big_vals).cuda()
    dr, dc = torch.from_numpy(big_rows).cuda(), torch.from_numpy(big_cols).cuda()
    di = torch.from_numpy(idx.astype(np.int32)).cuda()
    P.setPreconditioner_bcoo(dv, dr, dc, di, off, n, len(s.pairs))
    rt = torch.from_numpy(r).cuda()
    z = torch.zeros_like(rt)
    P.preconditioning(rt, z)
    torch.cuda.synchronize()
    assert np.array_equal(z.cpu().numpy(), z_ref)
    # new values through the same indices
    v2 = _scaled_values(s, 9)
    big_vals[where] = v2
    P.refresh_fixed_graph_bcoo(torch.from_numpy(big_vals).cuda(), dr, dc, di, off, n)
    z2 = torch.zeros_like(rt)
    P.preconditioning(rt, z2)
    torch.cuda.synchronize()
    with MasPcg.from_system(s) as ref:
        ref.set_matrix(v2, s.rows, s.cols, s.nb, s.fem_offset, s.abd_bodies)
        ref.build()
        z2_ref = ref.apply_preconditioner(r)
    assert np.array_equal(z2.cpu().numpy(), z2_ref)
    P.FreeMAS()


def _identity_domains(count, bank=32):
    P = bank * (bank + 1) // 2
    a = np.zeros((count, P, 9))
    b = np.zeros((count, P, 9), np.float32)
    for row in range(bank):
        k = bank * row - row * (row + 1) // 2 + row
        a[:, k] = np.eye(3).T.reshape(9)
        b[:, k] = np.eye(3).T.reshape(9)
    return a, b


def test_local_checks_reference_self_test_cases():
    """run_local_diagnostics_gpu_self_test (TraditionalMAS32Preconditioner.cu:
    185-215): identity passes; a negative local diagonal fails local SPD; a
    negative inverse diagonal fails inverse SPD; a NaN inverse is counted
    non-finite; an inverse doubled on the diagonal has residual > 1e-3; a NaN
    local matrix is counted non-finite."""
    a, b = _identity_domains(6)
    a[1, 0, 0] = -1.0
    b[2, 0, 0] = -1.0
    b[3, 0, 0] = np.nan
    for row in range(32):
        b[4, 32 * row - row * (row + 1) // 2 + row] *= 2.0
    a[5, 0, 0] = np.nan
    with MasPcg(preconditioner="none") as m:
        for case in range(6):
            summ, per = m.check_local_matrices(a[case:case + 1], b[case:case + 1])
            assert summ["passed"] == (case == 0), (case, summ)
            if case == 1:
                assert summ["local_spd_count"] == 0
            if case == 2:
                assert summ["inverse_spd_count"] == 0
            if case == 3:
                assert summ["nonfinite_inverse_count"] == 1
            if case == 4:
                assert summ["maximum_inverse_residual"] > 1e-3
            if case == 5:
                assert summ["nonfinite_local_count"] == 1
        summ, per = m.check_local_matrices(a, b)
    assert summ["matrix_count"] == 6 and summ["first_local_spd_failure"] == 1
    assert summ["first_inverse_spd_failure"] in (2, 3)


@pytest.mark.parametrize("precision,inverse", [("reference", "fp32"), ("mixed", "bf16")])
def test_local_diagnostics_match_oracle(cfg1_small, precision, inverse):
    """The checks on the handle's own domains against the oracle's
    restatement of check_local_matrices on the same matrices: the matrices
    the stored inverses were built from (level 0 gathered again, the coarse
    levels from the build's own Galerkin sums), which neither the checks nor
    the matrix read-back rebuild, so the preconditioner is unchanged."""
    s = cfg1_small
    rng = np.random.default_rng(2)
    r = rng.standard_normal(3 * s.nb)
    with MasPcg.from_system(s, precision=precision, inverse=inverse) as m:
        inv0 = m.domain_inverses()
        z0 = m.apply_preconditioner(r)
        d = m.local_diagnostics(per_domain=True)
        p64 = m.domain_matrices()
        inv = m.domain_inverses()
        z1 = m.apply_preconditioner(r)
    assert np.array_equal(inv0, inv) and np.array_equal(z0, z1)
    o = oracle.local_checks(p64, inv)
    assert d["matrix_count"] == len(o)
    for g, c in zip(d["domains"], o):
        assert bool(g["local_spd"]) == bool(c["local_spd"])
        assert bool(g["inverse_spd"]) == bool(c["inverse_spd"])
        assert g["minimum_local_diagonal"] == pytest.approx(c["minimum_local_diagonal"], rel=1e-12)
        assert g["inverse_residual"] == pytest.approx(c["inverse_residual"], rel=1e-6, abs=1e-12)
    assert d["passed"] == all(c["local_spd"] and c["inverse_spd"] and c["inverse_residual"] <= 1e-3 for c in o)


def test_solve_graph_is_reused_across_newton_steps(cfg1_small):
    """A Newton step on the same structure (set_matrix + build, or a values
    refresh) reuses the captured solve graph: maspcg_info.graph_captures stays
    at one, and every solve gives the first one's answer.  A new stream is
    captured anew."""
    s = cfg1_small
    with MasPcg.from_system(s, gate="euclid", precision="mixed", inverse="bf16") as m:
        x0, r0 = m.solve(s.b)
        assert m.info()["graph_captures"] == 1
        for _ in range(2):
            m.set_matrix(s.vals, s.rows, s.cols, s.nb, s.fem_offset, s.abd_bodies)
            m.build()
            x1, r1 = m.solve(s.b)
            # the rebuild re-sums the coarse domain matrices (FP64 atomics):
            # the same solve up to rounding
            assert r1["status_name"] == "converged" and abs(r1["iterations"] - r0["iterations"]) <= 1
            assert np.linalg.norm(x1 - x0) <= 1e-6 * np.linalg.norm(x0)
        m.refresh_values(s.vals)
        x2, r2 = m.solve(s.b)
        assert r2["status_name"] == "converged" and np.linalg.norm(x2 - x0) <= 1e-6 * np.linalg.norm(x0)
        assert m.info()["graph_captures"] == 1
        import torch
        st = torch.cuda.Stream()
        m.set_stream(st.cuda_stream)
        x3, r3 = m.solve(s.b)
        assert m.info()["graph_captures"] == 2
        assert np.linalg.norm(x3 - x0) <= 1e-6 * np.linalg.norm(x0)
        m.set_stream(None)
