"""CPU emulation of the mixed-precision PCG iteration, for the precision study
(test infrastructure: nothing in the product path imports it).

It runs the iteration of the library's MIXED precision on a synth.System with
numpy and scipy, using the oracle's MAS32 apply (FP32 domain inverses) and
12x12 body inverses as the preconditioner, and lets each source of rounding be
switched on or off:

* `matrix`: "f64" (the FP64 values), "f32" (the values of the FEM rows
  rounded to FP32; the affine-body rows keep FP64, as the library's
  iteration does), or "split" (FP32 values plus the BF16 rounding of the
  remainder A - A32);
* `round32`: which vectors are rounded to FP32 after each update, any of
  "r", "p", "z", "Ap", "x";
* `replacement`: "periodic" (the recursive residual replaced by the FP64
  true residual every `period` iterations), "reliable" (once ||r|| fell to
  `drop` of its largest value since the last replacement, checked every
  `period` iterations), or "none";
* `beta`: "fr" (r.z ratio, the reference's) or "flexible" (Polak-Ribiere);
* `sums` (with matrix="f32"): "f64" (exact products summed in FP64, the
  library's MASPCG_MATRIX_F32_ACCURATE), "block32" (each 3x3 block's three row
  sums in FP32, products rounded, then FP64 across blocks) or "f32"
  (the same, and the blocks of a row added in FP32 in column order).  The
  FP32 forms round every product, where the GPU's fused multiply-adds round
  only the sums, so they overstate the GPU's FP32 error; they show where the
  error comes from, not its GPU size.

Every run meets the recursive gate ||r|| <= tol ||b|| first and then stops
only on the FP64 true residual, as the library's mixed solve does.  With
matrix="f64", round32=(), replacement="none" it is the reference's FP64 PCG
under the Euclidean gate (tests/test_precision_emulation_cpu.py pins it to
the oracle).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import Mas32, abd_inverse


def _r32(v):
    return np.asarray(v, np.float64).astype(np.float32).astype(np.float64)


def _bf16(v):
    u = np.asarray(v, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16  # round to nearest even
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def full_matrix(s) -> sp.csr_matrix:
    """The symmetric matrix of the system's upper BCOO triplets (Eigen
    column-major 3x3 values; repeated entries add)."""
    rows, cols = s.rows.astype(np.int64), s.cols.astype(np.int64)
    blk = s.vals.reshape(-1, 3, 3).transpose(0, 2, 1)
    i3 = np.arange(3)
    ri = (3 * rows[:, None, None] + i3[None, :, None]).repeat(3, 2)
    ci = (3 * cols[:, None, None] + i3[None, None, :]).repeat(3, 1)
    n = 3 * s.nb
    A = sp.coo_matrix((blk.ravel(), (ri.ravel(), ci.ravel())), shape=(n, n))
    off = rows != cols
    At = sp.coo_matrix((blk[off].ravel(), (ci[off].ravel(), ri[off].ravel())), shape=(n, n))
    return (A + At).tocsr()


class Emulation:
    def __init__(self, s):
        self.s = s
        self.A = full_matrix(s)
        self.nbody = 12 * s.abd_bodies
        self.mas = None
        if s.fem_count > 0:
            self.mas = Mas32.from_system(s)
            self.mas.reorder(s.pairs)
            sel = np.nonzero((s.rows >= s.fem_offset) & (s.rows < s.fem_offset + s.fem_count) &
                             (s.cols >= s.fem_offset) & (s.cols < s.fem_offset + s.fem_count))[0].astype(np.uint32)
            self.mas.prepare_hessian(s.vals, s.rows, s.cols, sel, s.fem_offset)
        self.abd = abd_inverse(s.abd_bodies, s.rows, s.cols, s.vals)[0] if s.abd_bodies else None

    def precondition(self, r):
        s = self.s
        z = r.copy()
        if self.abd is not None:
            nb = self.nbody
            z[:nb] = np.einsum("bij,bj->bi", self.abd, r[:nb].reshape(-1, 12)).reshape(-1)
        if self.mas is not None:
            fo = 3 * s.fem_offset
            z[fo:fo + 3 * s.fem_count] = self.mas.precondition(r[fo:fo + 3 * s.fem_count])
        return z

    def operator(self, matrix: str) -> sp.csr_matrix:
        if matrix == "f64":
            return self.A
        C = self.A.tocoo()
        fem = C.row >= self.nbody
        hi = C.data.copy()
        hi[fem] = _r32(hi[fem])
        if matrix == "split":
            hi[fem] += _bf16(C.data[fem] - hi[fem])
        elif matrix != "f32":
            raise ValueError(matrix)
        return sp.csr_matrix((hi, (C.row, C.col)), shape=C.shape)

    def _blocked(self, sums):
        """y = A32 p with FP32 block sums (see the module docstring)."""
        s = self.s
        rows, cols = s.rows.astype(np.int64), s.cols.astype(np.int64)
        blk = s.vals.reshape(-1, 3, 3).transpose(0, 2, 1)
        off = rows != cols
        R = np.concatenate([rows, cols[off]])
        C = np.concatenate([cols, rows[off]])
        B = np.concatenate([blk, blk[off].transpose(0, 2, 1)])
        key = R * s.nb + C
        order = np.argsort(key, kind="stable")
        uk, start = np.unique(key[order], return_index=True)
        B = np.add.reduceat(B[order], start, axis=0)
        R, C = uk // s.nb, uk % s.nb
        rowptr = np.searchsorted(R, np.arange(s.nb + 1))
        body = R < 4 * s.abd_bodies
        B32 = B.astype(np.float32)
        nbody = self.nbody

        def f(p):
            pc = p.astype(np.float32).reshape(-1, 3)[C]
            y = B32[:, :, 2] * pc[:, 2:3]
            y = (B32[:, :, 1] * pc[:, 1:2]).astype(np.float32) + y
            y = ((B32[:, :, 0] * pc[:, 0:1]).astype(np.float32) + y).astype(np.float32)
            if sums == "block32":
                out = np.add.reduceat(y.astype(np.float64), rowptr[:-1], axis=0)
            else:
                out = np.add.reduceat(y, rowptr[:-1], axis=0, dtype=np.float32).astype(np.float64)
            out = out.reshape(-1)
            if nbody:
                yb = np.einsum("tij,tj->ti", B[body], p.reshape(-1, 3)[C[body]])
                out[:nbody] = np.add.reduceat(yb, rowptr[:4 * s.abd_bodies], axis=0).reshape(-1)
            return out

        return f

    def run(self, matrix="f32", round32=("r", "p", "z", "Ap", "x"), replacement="periodic", period=16, drop=0.1,
            beta="fr", tol=1e-4, max_iter=5000, sums="f64"):
        """Returns (iterations, status, replacements)."""
        A64 = self.A
        if sums == "f64":
            Wop = self.operator(matrix)
            Aw_mul = Wop.__matmul__
        else:
            if matrix != "f32":
                raise ValueError("FP32 sums model the FP32 matrix form")
            Aw_mul = self._blocked(sums)
        R = {k: (_r32 if k in round32 else (lambda v: v)) for k in ("r", "p", "z", "Ap", "x")}
        b = self.s.b
        n, bn = len(b), np.linalg.norm(b)
        xhi, xlo = np.zeros(n), np.zeros(n)
        r = R["r"](b.copy())
        z = R["z"](self.precondition(r))
        p = R["p"](z.copy())
        rz = float(r @ z)
        peak, reps = float(np.linalg.norm(r)), 0
        for k in range(1, max_iter + 1):
            Ap = R["Ap"](Aw_mul(p))
            pap = float(p @ Ap)
            if not pap > 0:
                return k, "nonpositive_curvature", reps
            a = rz / pap
            r_old = r
            xlo = R["x"](xlo + a * p)
            r = R["r"](r - a * Ap)
            rn = float(np.linalg.norm(r))
            peak = max(peak, rn)
            gate = rn <= tol * bn
            check = k % period == 0
            if check or gate:
                xhi, xlo = xhi + xlo, np.zeros(n)
            due = gate or (check and (replacement == "periodic" or (replacement == "reliable" and rn <= drop * peak)))
            if due:
                rt = b - A64 @ xhi
                if np.linalg.norm(rt) <= tol * bn:
                    return k, "converged", reps
                if replacement != "none" or gate:
                    r = R["r"](rt)
                    reps += 1
                    peak = float(np.linalg.norm(r))
            z = R["z"](self.precondition(r))
            rzn = float(r @ z)
            bt = (rzn - float(z @ r_old)) / rz if beta == "flexible" else rzn / rz
            rz = rzn
            p = R["p"](z + bt * p)
        return max_iter, "iteration_cap", reps
