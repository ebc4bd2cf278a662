"""The differentiable solve (agipc_learning_b200.autograd) against FP64 dense
references and central finite differences (needs a B200).

Workload: the per-tet-modulus cube (Young's modulus log-uniform in
[1e4, 1e6] Pa), loss ||x - x*||^2 with x* ~ N(0, 1).
"""
import numpy as np
import pytest

from agipc_learning_b200 import synth
from agipc_learning_b200.solver import MasPcg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dense(rows, cols, vals, nb):
    A = np.zeros((3 * nb, 3 * nb))
    for r, c, v in zip(rows, cols, vals):
        B = np.asarray(v).reshape(3, 3).T  # Eigen column-major -> (row, col)
        A[3 * r:3 * r + 3, 3 * c:3 * c + 3] += B
        if r != c:
            A[3 * c:3 * c + 3, 3 * r:3 * r + 3] += B.T
    return A


def _system(n, seed):
    ntet = 6 * (n - 1) ** 3
    E = synth.log_uniform_E(ntet, 1e4, 1e6, seed + 5)
    return synth.cube_system(n, E=1e5, nu=0.45, seed=seed, E_tet=E, keep_raw=True, name=f"adj{n}"), E


def _solver(s, tol):
    m = MasPcg(gate="euclid", precision="reference", tolerance=tol, max_iterations=20000)
    m.set_graph(s.fem_count, s.node_offset, s.neighbor_start, s.neighbor_num, s.neighbor_list, s.part_map_real,
                s.real_map_part)
    m.set_contacts(s.pairs)
    return m


def _library_gradient(s, E, x_star, tol):
    from agipc_learning_b200.autograd import modulus_gradient, newton_solve
    R, C, V = s.meta["raw"]
    dev = torch.device("cuda")
    vals = torch.tensor(V, dtype=torch.float64, device=dev, requires_grad=True)
    b = torch.tensor(s.b, dtype=torch.float64, device=dev, requires_grad=True)
    rows = torch.tensor(R, dtype=torch.int32, device=dev)
    cols = torch.tensor(C, dtype=torch.int32, device=dev)
    with _solver(s, tol) as m:
        x = newton_solve(vals, b, m, rows, cols, s.nb)
        loss = ((x - torch.tensor(x_star, device=dev)) ** 2).sum()
        loss.backward()
        gE = modulus_gradient(vals.grad, vals.detach(), torch.tensor(E, device=dev))
    return x.detach().cpu().numpy(), b.grad.cpu().numpy(), gE.cpu().numpy(), float(loss.detach())


def test_adjoint_matches_dense_reference_and_fd_on_6cube():
    s, E = _system(6, synth.SEED_BASE + 3)
    rng = np.random.default_rng(11)
    x_star = rng.standard_normal(3 * s.nb)
    x, gb, gE, loss = _library_gradient(s, E, x_star, 1e-13)
    # dense FP64 reference: x, lambda, and the per-tet gradient -(1/E_t) lam_t^T H_t x_t
    R, C, V = s.meta["raw"]
    A = _dense(R, C, V, s.nb)
    xd = np.linalg.solve(A, s.b)
    lam = np.linalg.solve(A, 2 * (xd - x_star))
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) <= 1e-10
    assert np.linalg.norm(gb - lam) / np.linalg.norm(lam) <= 1e-9
    ne = s.meta["elem_blocks"]
    gref = np.zeros(len(E))
    for k in range(ne):
        r, c = R[k], C[k]
        B = V[k].reshape(3, 3).T
        q = lam[3 * r:3 * r + 3] @ B @ xd[3 * c:3 * c + 3]
        if r != c:
            q += lam[3 * c:3 * c + 3] @ B.T @ xd[3 * r:3 * r + 3]
        gref[k // 10] -= q / E[k // 10]
    assert np.max(np.abs(gE - gref)) <= 1e-8 * np.max(np.abs(gref))
    # central differences of the dense FP64 solve along seeded directions.
    # Step 1e-3, relative in E per unit-variance direction component: the
    # loss is ~1e7 against a derivative ~1e4, so at a 1e-6 step FP64 roundoff
    # of the two losses alone is ~2e-5 of the difference (measured on this
    # system: 2.4e-5 at 1e-6, 6e-7 at 1e-3).
    h = 1e-3
    for j in range(8):
        d = np.random.default_rng(100 + j).standard_normal(len(E))
        def L(eps):
            Vp = V.copy()
            Vp[:ne] *= np.repeat(1 + eps * d, 10)[:, None]
            xp = np.linalg.solve(_dense(R, C, Vp, s.nb), s.b)
            return float(np.sum((xp - x_star) ** 2))
        fd = (L(h) - L(-h)) / (2 * h)
        an = float(np.dot(gE, d * E))
        assert abs(fd - an) <= 1e-5 * max(abs(fd), 1e-12), (j, fd, an)


def test_adjoint_matches_central_differences_of_the_gpu_solve():
    """Per-tet modulus gradient of the loss through PCG solves (reference
    precision, tolerance 1e-14) against central finite differences of the
    same GPU solve, step 1e-3 relative in E (see the dense test for why not
    1e-6), on seeded random directions."""
    from agipc_learning_b200.autograd import scale_element_blocks
    s, E = _system(12, synth.SEED_BASE + 3)
    rng = np.random.default_rng(12)
    x_star = rng.standard_normal(3 * s.nb)
    _, _, gE, _ = _library_gradient(s, E, x_star, 1e-14)
    R, C, V = s.meta["raw"]
    dev = torch.device("cuda")
    vals = torch.tensor(V, dtype=torch.float64, device=dev)
    rows = torch.tensor(R, dtype=torch.int32, device=dev)
    cols = torch.tensor(C, dtype=torch.int32, device=dev)
    b = torch.tensor(s.b, dtype=torch.float64, device=dev)
    xs = torch.tensor(x_star, device=dev)
    h = 1e-3
    with _solver(s, 1e-14) as m:
        def L(eps, d):
            m.set_matrix(scale_element_blocks(vals, torch.tensor(1 + eps * d, device=dev)), rows, cols, s.nb)
            m.build()
            x = torch.empty_like(b)
            _, res = m.solve(b, x)
            assert res["status_name"] == "converged"
            return float(((x - xs) ** 2).sum())
        for j in range(5):
            d = np.random.default_rng(200 + j).standard_normal(len(E))
            fd = (L(h, d) - L(-h, d)) / (2 * h)
            an = float(np.dot(gE, d * E))
            assert abs(fd - an) <= 1e-5 * abs(fd), (j, fd, an)


def _modulus_gradient_fused(s, E, x_star, precision, tol):
    """dL/dE and dL/db through newton_solve_modulus (the adjoint solve and the
    fused outer-product kernel maspcg_element_modulus_gradient)."""
    from agipc_learning_b200.autograd import newton_solve_modulus
    R, C, V = s.meta["raw"]
    dev = torch.device("cuda")
    Et = torch.tensor(E, dtype=torch.float64, device=dev, requires_grad=True)
    b = torch.tensor(s.b, dtype=torch.float64, device=dev, requires_grad=True)
    vals = torch.tensor(V, dtype=torch.float64, device=dev)
    rows = torch.tensor(R, dtype=torch.int32, device=dev)
    cols = torch.tensor(C, dtype=torch.int32, device=dev)
    m = MasPcg(gate="euclid", precision=precision, inverse="bf16" if precision == "mixed" else "fp32",
               tolerance=tol, max_iterations=20000)
    m.set_graph(s.fem_count, s.node_offset, s.neighbor_start, s.neighbor_num, s.neighbor_list, s.part_map_real,
                s.real_map_part)
    m.set_contacts(s.pairs)
    x = newton_solve_modulus(Et, b, vals, m, rows, cols, s.nb)
    loss = ((x - torch.tensor(x_star, device=dev)) ** 2).sum()
    loss.backward()
    return m, Et.grad.cpu().numpy(), b.grad.cpu().numpy(), (vals, rows, cols)


def test_fused_modulus_kernel_matches_the_two_step_chain():
    """maspcg_element_modulus_gradient equals maspcg_bcoo_gradient followed by
    the per-tet sum <dL/dval, val> / E (12^3 cube)."""
    s, E = _system(12, synth.SEED_BASE + 3)
    x_star = np.random.default_rng(4).standard_normal(3 * s.nb)
    _, gb_ref, gE_ref, _ = _library_gradient(s, E, x_star, 1e-13)
    m, gE, gb, _ = _modulus_gradient_fused(s, E, x_star, "reference", 1e-13)
    m.close()
    assert np.max(np.abs(gE - gE_ref)) <= 1e-10 * np.max(np.abs(gE_ref))
    assert np.max(np.abs(gb - gb_ref)) <= 1e-10 * np.max(np.abs(gb_ref))


@pytest.mark.parametrize("precision,tol", [("reference", 1e-12), ("mixed", 1e-10)])
def test_config3_gradient_on_200_fd_directions(precision, tol):
    """The differentiation workload as stated: the 32^3 cube (98,304 DOF) with
    per-tet Young's modulus log-uniform in [1e4, 1e6], loss ||x - x*||^2,
    x* ~ N(0, 1); the gradient in (E, b) from the autograd backward against
    FP64 central finite differences of the solve on 200 seeded random
    directions, each within 1e-5 relative.  A direction scales E by
    (1 + eps d_E) and moves b by eps d_b; the FD step is 1e-3 (relative in E),
    for the roundoff reason given in the 6^3 test.  Forward and adjoint in the
    reference precision, and in mixed precision (FP32 vectors, BF16 domain
    inverses, FP64 residual replacement) solved to 1e-10.  The finite
    differences re-solve with values refreshed on the kept structure."""
    from agipc_learning_b200.autograd import scale_element_blocks
    s, E = _system(32, synth.SEED_BASE + 3)
    x_star = np.random.default_rng(33).standard_normal(3 * s.nb)
    m, gE, gb, (vals, rows, cols) = _modulus_gradient_fused(s, E, x_star, precision, tol)
    dev = torch.device("cuda")
    b0 = torch.tensor(s.b, dtype=torch.float64, device=dev)
    xs = torch.tensor(x_star, device=dev)
    # the handle now holds the system at E (the backward reused it)
    h = 1e-3
    worst = 0.0
    try:
        def L(eps, dE, db):
            m.refresh_values(scale_element_blocks(vals, torch.tensor(1 + eps * dE, device=dev)))
            x = torch.empty_like(b0)
            _, res = m.solve(b0 + eps * torch.tensor(db, device=dev), x)
            assert res["status_name"] == "converged", res
            return float(((x - xs) ** 2).sum())
        for j in range(200):
            rng = np.random.default_rng(1000 + j)
            dE, db = rng.standard_normal(len(E)), rng.standard_normal(3 * s.nb)
            fd = (L(h, dE, db) - L(-h, dE, db)) / (2 * h)
            an = float(np.dot(gE, dE * E) + np.dot(gb, db))
            rel = abs(fd - an) / abs(fd)
            worst = max(worst, rel)
            assert rel <= 1e-5, (j, fd, an, rel)
    finally:
        m.close()
    print(f"config 3 ({precision}): worst relative FD mismatch over 200 directions {worst:.2e}")
