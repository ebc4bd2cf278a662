"""The Newton-step solve as a differentiable PyTorch operation.

`newton_solve(vals, b, solver, rows, cols, nb)` returns x = A^-1 b for the
block-sparse A given by upper BCOO blocks (`vals`: [n, 9] FP64, Eigen
column-major; repeated (row, col) entries add), through the C ABI of
libmaspcg.  Its backward:

  lam     = A^-1 dL/dx           (adjoint solve: A is symmetric, so the same
                                  operator and preconditioner are reused)
  dL/db   = lam
  dL/dval = maspcg_bcoo_gradient(lam, x): -(lam_r x_c^T + x_r lam_c^T) per
            off-diagonal block, -lam_r x_r^T per diagonal block

x is kept from the forward pass (no Krylov history is stored).

`newton_solve_modulus(E_tet, vals, b, solver, rows, cols, nb)` is the same
solve differentiable in the per-tet Young's modulus: a tet's Hessian blocks
scale with its modulus (stable Neo-Hookean with the Lame pair linear in E,
and the PSD projection commutes with a positive scale), so dL/dE_t = sum
over the tet's element blocks k of <dL/dval_k, val_k> / E_t.  Its backward
runs the adjoint solve and maspcg_element_modulus_gradient, one kernel that
forms the outer products and chains them to E without storing dL/dval.

The solves, the adjoint outer products and the chain to E run in the
library's kernels; torch holds the device memory and the autograd graph.
`scale_element_blocks` and `modulus_gradient` are torch helpers for tests and
callers that build perturbed systems or already hold dL/dval.
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import MasPcg


class NewtonSolveFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vals, b, solver: MasPcg, rows, cols, nb: int, fem_offset: int = 0, abd_bodies: int = 0):
        for t, dt in ((vals, torch.float64), (b, torch.float64), (rows, torch.int32), (cols, torch.int32)):
            if not (t.is_cuda and t.dtype == dt and t.is_contiguous()):
                raise ValueError("vals/b must be contiguous CUDA float64, rows/cols contiguous CUDA int32")
        solver.set_matrix(vals, rows, cols, nb, fem_offset, abd_bodies)
        solver.build()
        x = torch.empty_like(b)
        _, res = solver.solve(b, x)
        if res["status_name"] != "converged":
            raise RuntimeError(f"forward solve did not converge: {res}")
        ctx.solver = solver
        ctx.version = solver.matrix_version
        ctx.dims = (nb, fem_offset, abd_bodies)
        ctx.save_for_backward(vals, rows, cols, x)
        return x

    @staticmethod
    def backward(ctx, gx):
        vals, rows, cols, x = ctx.saved_tensors
        solver = ctx.solver
        if solver.matrix_version != ctx.version:  # the handle was reused: restore this system
            solver.set_matrix(vals, rows, cols, *ctx.dims)
            solver.build()
        gx = gx.contiguous().to(torch.float64)
        lam = torch.empty_like(gx)
        _, res = solver.solve(gx, lam)
        if res["status_name"] != "converged":
            raise RuntimeError(f"adjoint solve did not converge: {res}")
        gvals = torch.empty_like(vals)
        solver.bcoo_gradient(rows, cols, lam, x, gvals)
        return gvals, lam, None, None, None, None, None, None


class NewtonSolveModulusFunction(torch.autograd.Function):
    """x(E, b) = A(E)^-1 b with the first blocks_per_tet * ntet blocks of
    `vals` the element blocks at the moduli E (tet order)."""

    @staticmethod
    def forward(ctx, E_tet, b, vals, solver: MasPcg, rows, cols, nb: int, blocks_per_tet: int = 10,
                fem_offset: int = 0, abd_bodies: int = 0):
        x = NewtonSolveFunction.forward(ctx, vals, b, solver, rows, cols, nb, fem_offset, abd_bodies)
        ctx.bpt = blocks_per_tet
        ctx.E = E_tet
        return x

    @staticmethod
    def backward(ctx, gx):
        vals, rows, cols, x = ctx.saved_tensors
        solver = ctx.solver
        if solver.matrix_version != ctx.version:
            solver.set_matrix(vals, rows, cols, *ctx.dims)
            solver.build()
        gx = gx.contiguous().to(torch.float64)
        lam = torch.empty_like(gx)
        _, res = solver.solve(gx, lam)
        if res["status_name"] != "converged":
            raise RuntimeError(f"adjoint solve did not converge: {res}")
        E = ctx.E.contiguous().to(torch.float64)
        gE = torch.empty_like(E)
        a = [solver._arg(rows, np.int32), solver._arg(cols, np.int32), solver._arg(vals, np.float64),
             solver._arg(lam, np.float64), solver._arg(x, np.float64), solver._arg(E, np.float64),
             solver._arg(gE, np.float64, writable=True)]
        solver._ck(solver.lib.maspcg_element_modulus_gradient(solver.h, int(E.shape[0]), int(ctx.bpt),
                                                               *[q.ptr for q in a]))
        return gE, lam, None, None, None, None, None, None, None, None


def newton_solve_modulus(E_tet: torch.Tensor, b: torch.Tensor, vals: torch.Tensor, solver: MasPcg,
                         rows: torch.Tensor, cols: torch.Tensor, nb: int, blocks_per_tet: int = 10,
                         fem_offset: int = 0, abd_bodies: int = 0) -> torch.Tensor:
    """x = A(E)^-1 b, differentiable in the per-tet moduli E_tet and in b;
    `vals` are the triplet values at E_tet (see the module docstring)."""
    return NewtonSolveModulusFunction.apply(E_tet, b, vals, solver, rows, cols, nb, blocks_per_tet, fem_offset,
                                            abd_bodies)


def newton_solve(vals: torch.Tensor, b: torch.Tensor, solver: MasPcg, rows: torch.Tensor, cols: torch.Tensor,
                 nb: int, fem_offset: int = 0, abd_bodies: int = 0) -> torch.Tensor:
    """x = A^-1 b, differentiable in `vals` and `b` (see the module docstring)."""
    return NewtonSolveFunction.apply(vals, b, solver, rows, cols, nb, fem_offset, abd_bodies)


def modulus_gradient(grad_vals: torch.Tensor, vals: torch.Tensor, E_tet: torch.Tensor,
                     blocks_per_tet: int = 10) -> torch.Tensor:
    """dL/dE per tet from dL/d(vals) of the raw triplets whose first
    blocks_per_tet * ntet entries are the element blocks in tet order."""
    ntet = E_tet.shape[0]
    k = blocks_per_tet * ntet
    s = (grad_vals[:k] * vals[:k]).sum(dim=1).view(ntet, blocks_per_tet).sum(dim=1)
    return s / E_tet


def scale_element_blocks(vals: torch.Tensor, factor: torch.Tensor, blocks_per_tet: int = 10) -> torch.Tensor:
    """Triplet values after scaling each tet's modulus by `factor` (per tet)."""
    out = vals.clone()
    ntet = factor.shape[0]
    k = blocks_per_tet * ntet
    out[:k] *= factor.repeat_interleave(blocks_per_tet).unsqueeze(1)
    return out


__all__ = ["NewtonSolveFunction", "NewtonSolveModulusFunction", "newton_solve", "newton_solve_modulus",
           "modulus_gradient", "scale_element_blocks", "np"]
