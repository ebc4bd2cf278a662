"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle restates the reference's Newton-step linear solve in plain C
(``maspcg_oracle.c``), built for the 32-vertex MAS bank (``liboracle.so``,
TraditionalMAS32Preconditioner) and the 16-vertex bank (``liboracle16.so``,
CEMAS16 / MASPreconditioner).  It is the parity checker for the CUDA path and the
timed CPU baseline; nothing in ``agipc_learning_b200`` imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}

PRECOND_DIAG3 = 0
PRECOND_MAS16 = 1
PRECOND_MAS32 = 2
PRECOND_NONE = -1
GATE_RZ = 0
GATE_EUCLID = 1
STATUS_NAMES = {1: "converged", 2: "iteration_cap", 3: "nonpositive_curvature", 4: "nonfinite", 5: "invalid_rz"}


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


class _PcgOpts(ctypes.Structure):
    _fields_ = [("precond", ctypes.c_int), ("gate", ctypes.c_int), ("tol", ctypes.c_double),
                ("max_iter", ctypes.c_int), ("nb", ctypes.c_int), ("fem_offset", ctypes.c_int),
                ("fem_count", ctypes.c_int), ("abd_bodies", ctypes.c_int), ("replay_checks", ctypes.c_int)]


class _PcgResult(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("status", ctypes.c_int), ("rz0", ctypes.c_double),
                ("rz_last", ctypes.c_double), ("rel_res_recursive", ctypes.c_double),
                ("rel_res_true", ctypes.c_double)]


def lib(bank=32):
    if bank not in _LIBS:
        path = os.path.join(_HERE, "liboracle.so" if bank == 32 else "liboracle16.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P, I, D, LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
        sig = {
            "orc_convert_triplets": (I, [I, P, P, P, P, P, P]),
            "orc_partition_contacts": (I, [I, P, P, P, P, P, P, P, P]),
            "orc_sym_spmv": (None, [D, P, P, P, I, I, P, D, P]),
            "orc_upper_to_full_bcsr": (I, [I, I, P, P, P, P, P, P]),
            "orc_bcsr_spmv": (None, [I, P, P, P, P, P]),
            "orc_mas_create": (P, [I, I, P, P, P, I, P, I, P]),
            "orc_mas_free": (None, [P]),
            "orc_compute_num_levels": (I, [I]),
            "orc_mas_levelnum": (I, [P]),
            "orc_hierarchy_capacity": (LL, [LL, LL, LL, LL]),
            "orc_mas_going_next_capacity": (LL, [P]),
            "orc_mas_reorder": (I, [P, P, I]),
            "orc_mas_get_hierarchy": (None, [P, P, P, P, P, P, P]),
            "orc_mas_total_clusters": (I, [P]),
            "orc_mas_prepare_hessian": (None, [P, P, P, P, P, I, I]),
            "orc_mas_get_domains": (None, [P, P, P]),
            "orc_mas_precondition": (None, [P, P, P]),
            "orc_local_checks": (None, [I, P, P, P]),
            "orc_diag3_inverse": (None, [I, I, P, P, P, P]),
            "orc_abd_inverse": (I, [I, I, P, P, P, P]),
            "orc_pcg": (I, [ctypes.POINTER(_PcgOpts), P, P, P, I, P, P, P, ctypes.POINTER(_PcgResult)]),
            "orc_num_threads": (I, []),
            "orc_adjust_contacts": (I, [I, P, P, P, P, I, I]),
            "orc_zero_boundary": (I, [I, P, P, P, P, I, I]),
            "orc_mas_set_inverses": (None, [P, P]),
            "orc_direct_solve": (I, [I, I, P, P, P, P, P, ctypes.POINTER(LL)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIBS[bank] = L
    return _LIBS[bank]


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def convert_triplets(rows, cols, vals):
    n = len(rows)
    r, c, v = _c(rows, np.int32), _c(cols, np.int32), _c(vals, np.float64).reshape(n, 9)
    orow, ocol, oval = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros((n, 9))
    u = lib().orc_convert_triplets(n, _p(r), _p(c), _p(v), _p(orow), _p(ocol), _p(oval))
    return orow[:u].copy(), ocol[:u].copy(), oval[:u].copy()


def partition_contacts(rows, cols, vals, types):
    """Contact triplets ordered by type hash 0..3, stable; and the count of each type."""
    n = len(rows)
    r, c, v = _c(rows, np.int32), _c(cols, np.int32), _c(vals, np.float64).reshape(n, 9)
    t = _c(types, np.uint64)
    orow, ocol, oval = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros((n, 9))
    counts = np.zeros(4, np.int32)
    rc = lib().orc_partition_contacts(n, _p(r), _p(c), _p(v), _p(t), _p(orow), _p(ocol), _p(oval), _p(counts))
    if rc != 0:
        raise ValueError("contact type hash outside 0..3")
    return orow, ocol, oval, counts


def adjust_contacts(rows, cols, vals, bd_type, offset):
    """adjust_fem_fem_contact_indices_kernel restated: returns adjusted copies
    (rows, cols, vals) and the first out-of-range triplet (-1 if none)."""
    n = len(rows)
    r, c = _c(rows, np.int32).copy(), _c(cols, np.int32).copy()
    v = _c(vals, np.float64).reshape(n, 9).copy()
    bd = _c(bd_type, np.int32)
    bad = lib().orc_adjust_contacts(n, _p(r), _p(c), _p(v), _p(bd), len(bd), int(offset))
    return r, c, v, bad


def zero_boundary(rows, cols, vals, bd_type, offset):
    """zero_fem_boundary_hessian_kernel restated: returns the cleared copy of
    vals and the first out-of-range triplet (-1 if none)."""
    n = len(rows)
    v = _c(vals, np.float64).reshape(n, 9).copy()
    bd = _c(bd_type, np.int32)
    bad = lib().orc_zero_boundary(n, _p(_c(rows, np.int32)), _p(_c(cols, np.int32)), _p(v), _p(bd), len(bd),
                                  int(offset))
    return v, bad


def _skew(w):
    z = np.zeros(w.shape[:-1] + (3, 3))
    z[..., 0, 1], z[..., 0, 2] = -w[..., 2], w[..., 1]
    z[..., 1, 0], z[..., 1, 2] = w[..., 2], -w[..., 0]
    z[..., 2, 0], z[..., 2, 1] = -w[..., 1], w[..., 0]
    return z


def fem_snk1(tets, x, dm_inverse, volume, len_rate, vol_rate, dt, offset=0, project=True):
    """Per-tet SNK1 gradient and Hessian, StiffGIPC/femEnergy.cu:1720-1856.

    Energy u/2 (I2 - 3) + r/2 (I3 - 1 - u/r)^2 of F = Ds Dm^-1 (u, r: the
    Lame rates, gl_main.cu:586-630), times dt^2 V.  The gradient
    (__computePEPF_StableNHK3D1_double, :432-455) is summed per vertex.  The
    exact 9x9 Hessian in F (vec column-major, index i + 3j) is projected onto
    the PSD cone by a full eigendecomposition (numpy.linalg.eigh), which is
    what the reference's closed-form eigensystem (:1641-1717) computes; then
    H = dF/dx^T H_F dF/dx (:1389, :1814) and the 10 upper 3x3 blocks per tet,
    row <= col, values column-major (:1821-1852).  Returns (gradient,
    rows, cols, values9).  project=False keeps the exact Hessian (for finite
    difference checks)."""
    T = np.asarray(tets, np.int64).reshape(-1, 4)
    nt = len(T)
    X = np.asarray(x, np.float64).reshape(-1, 3)
    Di = np.asarray(dm_inverse, np.float64).reshape(nt, 3, 3)
    vol = np.asarray(volume, np.float64)
    u = np.asarray(len_rate, np.float64)
    r = np.asarray(vol_rate, np.float64)
    Ds = np.stack([X[T[:, c + 1]] - X[T[:, 0]] for c in range(3)], axis=2)
    F = Ds @ Di
    f = [F[:, :, c] for c in range(3)]
    cof = np.stack([np.cross(f[1], f[2]), np.cross(f[2], f[0]), np.cross(f[0], f[1])], axis=2)  # dJ/dF
    J = np.einsum("ti,ti->t", f[0], cof[:, :, 0])
    s = r * (J - 1.0) - u
    P = u[:, None, None] * F + s[:, None, None] * cof
    cf = np.zeros((nt, 4, 3))
    cf[:, 1:, :] = Di
    cf[:, 0, :] = -Di.sum(axis=1)
    scale = dt * dt * vol
    g12 = scale[:, None, None] * np.einsum("taj,tij->tai", cf, P)  # (nt, 4, 3)
    grad = np.zeros_like(X)
    np.add.at(grad, T.reshape(-1), g12.reshape(-1, 3))
    vg = cof.transpose(0, 2, 1).reshape(nt, 9)  # index i + 3j
    H9 = u[:, None, None] * np.eye(9) + r[:, None, None] * np.einsum("ta,tb->tab", vg, vg)
    for c in range(3):
        c1, c2 = (c + 1) % 3, (c + 2) % 3
        H9[:, 3 * c:3 * c + 3, 3 * c1:3 * c1 + 3] += -s[:, None, None] * _skew(f[c2])
        H9[:, 3 * c:3 * c + 3, 3 * c2:3 * c2 + 3] += s[:, None, None] * _skew(f[c1])
    if project:
        w, Q = np.linalg.eigh(H9)
        H9 = np.einsum("tak,tk,tbk->tab", Q, np.maximum(w, 0.0), Q)
    PF = np.zeros((nt, 9, 12))
    for a in range(4):
        for i in range(3):
            for j in range(3):
                PF[:, i + 3 * j, 3 * a + i] = cf[:, a, j]
    H12 = scale[:, None, None] * np.einsum("tpa,tpq,tqb->tab", PF, H9, PF)
    rows, cols, vals = np.zeros((nt, 10), np.int32), np.zeros((nt, 10), np.int32), np.zeros((nt, 10, 9))
    k = 0
    for a in range(4):
        for b in range(a, 4):
            ra, rb = T[:, a] + offset, T[:, b] + offset
            sw = ra > rb
            rows[:, k] = np.where(sw, rb, ra)
            cols[:, k] = np.where(sw, ra, rb)
            B = H12[:, 3 * a:3 * a + 3, 3 * b:3 * b + 3]
            B = np.where(sw[:, None, None], B.transpose(0, 2, 1), B)
            vals[:, k, :] = B.transpose(0, 2, 1).reshape(nt, 9)  # column-major: index i + 3j
            k += 1
    return grad.reshape(-1), rows.reshape(-1), cols.reshape(-1), vals.reshape(-1, 9)


def fem_snk1_energy(tets, x, dm_inverse, volume, len_rate, vol_rate, dt):
    """Total dt^2 V Psi of the SNK1 energy above (for finite differences)."""
    T = np.asarray(tets, np.int64).reshape(-1, 4)
    X = np.asarray(x, np.float64).reshape(-1, 3)
    Di = np.asarray(dm_inverse, np.float64).reshape(len(T), 3, 3)
    F = np.stack([X[T[:, c + 1]] - X[T[:, 0]] for c in range(3)], axis=2) @ Di
    u, r = np.asarray(len_rate, np.float64), np.asarray(vol_rate, np.float64)
    I2 = np.einsum("tij,tij->t", F, F)
    J = np.linalg.det(F)
    psi = 0.5 * u * (I2 - 3.0) + 0.5 * r * (J - 1.0 - u / r) ** 2
    return float(np.sum(dt * dt * np.asarray(volume) * psi))


def fem_rest_data(tets, X, E, nu):
    """Dm^-1 (row-major), rest volume |det Dm| / 6 and the Lame rates per tet
    (gl_main.cu:586-630): u = 4/3 mu, r = lambda + 5/6 mu."""
    T = np.asarray(tets, np.int64).reshape(-1, 4)
    Xr = np.asarray(X, np.float64).reshape(-1, 3)
    Dm = np.stack([Xr[T[:, c + 1]] - Xr[T[:, 0]] for c in range(3)], axis=2)
    E = np.broadcast_to(np.asarray(E, np.float64), (len(T),))
    mu, la = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    return np.linalg.inv(Dm).reshape(-1, 9), np.abs(np.linalg.det(Dm)) / 6.0, 4 * mu / 3, la + 5 * mu / 6


def galerkin_transform(block, prefix, fine_to_coarse, bases, masks, rest):
    """transform_for_block (StiffGIPC/agipc/agipc_galerkin.cu:200-219): the
    first coarse block, the width and the basis values of a fine block."""
    if block < prefix:
        return block, 1, [1.0, 0.0, 0.0, 0.0]
    k = block - prefix
    c = int(fine_to_coarse[k])
    mask = int(masks[c])
    raw = [1.0, float(rest[3 * k]), float(rest[3 * k + 1]), float(rest[3 * k + 2])]
    phi = [raw[q] for q in range(4) if mask & (1 << q)] + [0.0] * 4
    return prefix + int(bases[c]), bin(mask & 15).count("1"), phi[:4]


def galerkin_expand(rows, cols, vals, prefix, fine_to_coarse, bases, masks, rest):
    """count_expanded_blocks + emit_expanded_blocks (agipc_galerkin.cu:221-283):
    every fine upper triplet as its coarse triplets, in fine order."""
    rest = np.asarray(rest, np.float64).reshape(-1)
    V = np.asarray(vals, np.float64).reshape(-1, 9)
    orow, ocol, oval = [], [], []
    for i in range(len(rows)):
        r, c = int(rows[i]), int(cols[i])
        rb, rw, rp = galerkin_transform(r, prefix, fine_to_coarse, bases, masks, rest)
        cb, cw, cp = galerkin_transform(c, prefix, fine_to_coarse, bases, masks, rest)
        M = V[i].reshape(3, 3).T  # Eigen column-major -> (row, col)
        for a in range(rw):
            for b in range(cw):
                if r == c and a > b:
                    continue
                mr, mc = rb + a, cb + b
                w = rp[a] * cp[b]
                B = w * M
                if r != c and mr == mc:
                    B = B + B.T
                elif mr > mc:
                    mr, mc, B = mc, mr, B.T
                orow.append(mr)
                ocol.append(mc)
                oval.append(B.T.reshape(9))
    return (np.array(orow, np.int32), np.array(ocol, np.int32), np.array(oval, np.float64).reshape(-1, 9))


def galerkin_prolongation(fine_blocks, coarse_blocks, prefix, fine_to_coarse, bases, masks, rest):
    """The dense prolongation P (3 fine_blocks x 3 coarse_blocks) of the map."""
    rest = np.asarray(rest, np.float64).reshape(-1)
    P = np.zeros((3 * fine_blocks, 3 * coarse_blocks))
    for blk in range(fine_blocks):
        base, width, phi = galerkin_transform(blk, prefix, fine_to_coarse, bases, masks, rest)
        for a in range(width):
            P[3 * blk:3 * blk + 3, 3 * (base + a):3 * (base + a) + 3] = phi[a] * np.eye(3)
    return P


def sym_spmv(a, vals, rows, cols, x, b=0.0, y=None):
    x = _c(x, np.float64)
    y = np.zeros_like(x) if y is None else _c(y, np.float64).copy()
    v = _c(vals, np.float64)
    lib().orc_sym_spmv(float(a), _p(v), _p(_c(rows, np.int32)), _p(_c(cols, np.int32)), len(rows), len(x), _p(x),
                       float(b), _p(y))
    return y


def upper_to_full_bcsr(nb, rows, cols, vals):
    n = len(rows)
    rowptr = np.zeros(nb + 1, np.int32)
    col = np.zeros(2 * n + 1, np.int32)
    fv = np.zeros((2 * n + 1, 9))
    t = lib().orc_upper_to_full_bcsr(nb, n, _p(_c(rows, np.int32)), _p(_c(cols, np.int32)),
                                     _p(_c(vals, np.float64)), _p(rowptr), _p(col), _p(fv))
    return rowptr, col[:t].copy(), fv[:t].copy()


def bcsr_spmv(rowptr, col, vals, x):
    x = _c(x, np.float64)
    y = np.zeros_like(x)
    lib().orc_bcsr_spmv(len(rowptr) - 1, _p(_c(rowptr, np.int32)), _p(_c(col, np.int32)), _p(_c(vals, np.float64)),
                        _p(x), _p(y))
    return y


def direct_solve(nb, rows, cols, vals, b, stats=None):
    """x = A^-1 b in FP64 for the upper BCOO system: reverse Cuthill-McKee
    ordering and an envelope Cholesky (orc_direct_solve).  Raises ValueError
    on a non-positive pivot.  `stats` (a dict) receives the envelope size."""
    x = np.zeros(3 * int(nb))
    env = ctypes.c_longlong()
    rc = lib().orc_direct_solve(int(nb), len(rows), _p(_c(rows, np.int32)), _p(_c(cols, np.int32)),
                                _p(_c(vals, np.float64)), _p(_c(b, np.float64)), _p(x), ctypes.byref(env))
    if rc == -1:
        raise ValueError("orc_direct_solve: the matrix is not positive definite")
    if rc != 0:
        raise MemoryError("orc_direct_solve: out of memory")
    if stats is not None:
        stats["envelope"] = env.value
    return x


def compute_num_levels(n, bank=32):
    return lib(bank).orc_compute_num_levels(int(n))


def hierarchy_capacity(vertices, mapped, levels, bank):
    return lib().orc_hierarchy_capacity(vertices, mapped, levels, bank)


class Mas32:
    """TraditionalMAS32Preconditioner restated on the CPU."""

    BANK = 32

    def __init__(self, vert_num, node_offset, neighbor_start, neighbor_num, neighbor_list, part_map_real,
                 real_map_part):
        self._lib = lib(self.BANK)
        self._keep = [_c(neighbor_start, np.uint32), _c(neighbor_num, np.uint32),
                      _c(neighbor_list if len(neighbor_list) else np.zeros(1), np.uint32),
                      _c(part_map_real, np.int32), _c(real_map_part, np.int32)]
        s, n, l, pm, rm = self._keep
        self.h = self._lib.orc_mas_create(int(vert_num), int(node_offset), _p(s), _p(n), _p(l),
                                          int(len(neighbor_list)), _p(pm), int(len(pm)), _p(rm))
        if not self.h:
            raise ValueError("invalid MAS inputs")
        self.nv = int(vert_num)
        self.c0 = len(pm)
        self.levelnum = self._lib.orc_mas_levelnum(self.h)
        self.total_clusters = 0

    @classmethod
    def from_system(cls, s):
        return cls(s.fem_count, s.node_offset, s.neighbor_start, s.neighbor_num, s.neighbor_list, s.part_map_real,
                   s.real_map_part)

    def __del__(self):
        if getattr(self, "h", None):
            self._lib.orc_mas_free(self.h)
            self.h = None

    def reorder(self, pairs=None):
        p = None if pairs is None or len(pairs) == 0 else _c(pairs, np.int32).reshape(-1, 4)
        self.total_clusters = self._lib.orc_mas_reorder(self.h, _p(p), 0 if p is None else len(p))
        return self.total_clusters

    def hierarchy(self):
        L = self.levelnum
        cap = self._lib.orc_mas_going_next_capacity(self.h)
        fm = np.zeros(self.nv, np.uint32)
        cst = np.zeros(self.nv * L, np.int32)
        gn = np.zeros(cap, np.int32)
        ls = np.zeros(2 * (L + 1), np.int32)
        ct = np.zeros(self.nv * 6, np.int32)
        po = np.zeros(self.c0 // self.BANK, np.int32)
        self._lib.orc_mas_get_hierarchy(self.h, _p(fm), _p(cst), _p(gn), _p(ls), _p(ct), _p(po))
        return {"fine_mask": fm, "coarse_space_tables": cst.reshape(L, self.nv), "going_next": gn,
                "level_size": ls.reshape(L + 1, 2), "coarse_table": ct.reshape(self.nv, 6),
                "prefix_original": po, "total_clusters": self.total_clusters, "levelnum": L}

    def prepare_hessian(self, vals, rows, cols, indices=None, offset=0):
        n = len(rows) if indices is None else len(indices)
        self._mat = (_c(vals, np.float64), _c(rows, np.int32), _c(cols, np.int32))
        ind = None if indices is None else _c(indices, np.uint32)
        self._lib.orc_mas_prepare_hessian(self.h, _p(self._mat[0]), _p(self._mat[1]), _p(self._mat[2]), _p(ind),
                                          int(offset), int(n))

    def domains(self):
        B = self.BANK
        nd = self.total_clusters // B
        p64 = np.zeros((nd, B * (B + 1) // 2, 9))
        i32 = np.zeros((nd, B * (B + 1) // 2, 9), np.float32)
        self._lib.orc_mas_get_domains(self.h, _p(p64), _p(i32))
        return p64, i32

    def set_inverses(self, inverse32):
        """Replace the domain inverses (packed upper FP32 blocks, the layout of
        domains()) with the given ones, e.g. the decoded inverses of the GPU
        build, so precondition() applies exactly those operators."""
        B = self.BANK
        inv = _c(inverse32, np.float32).reshape(self.total_clusters // B, B * (B + 1) // 2, 9)
        self._lib.orc_mas_set_inverses(self.h, _p(inv))

    def precondition(self, R):
        R = _c(R, np.float64)
        Z = np.zeros_like(R)
        self._lib.orc_mas_precondition(self.h, _p(R), _p(Z))
        return Z


class Mas16(Mas32):
    """CEMAS16 (MASPreconditioner, 16-vertex banks, 48x48 domains) restated on
    the CPU: the MAS32 restatement built with a 16-vertex bank, plus the three
    places where CEMAS16's kernels differ (maspcg_oracle.c, ORC_BANK == 16)."""

    BANK = 16


def local_checks(packed64, inverse32, bank=32):
    packed64 = _c(packed64, np.float64)
    inverse32 = _c(inverse32, np.float32)
    n = packed64.shape[0]
    out = np.zeros((n, 7))
    lib(bank).orc_local_checks(n, _p(packed64), _p(inverse32), _p(out))
    keys = ["local_finite", "inverse_finite", "local_spd", "inverse_spd", "minimum_local_diagonal",
            "minimum_inverse_diagonal", "inverse_residual"]
    return [dict(zip(keys, row)) for row in out]


def diag3_inverse(nb, rows, cols, vals):
    out = np.zeros((nb, 9))
    lib().orc_diag3_inverse(nb, len(rows), _p(_c(rows, np.int32)), _p(_c(cols, np.int32)), _p(_c(vals, np.float64)),
                            _p(out))
    return out


def abd_inverse(bodies, rows, cols, vals):
    out = np.zeros((bodies, 12, 12))
    ok = lib().orc_abd_inverse(bodies, len(rows), _p(_c(rows, np.int32)), _p(_c(cols, np.int32)),
                               _p(_c(vals, np.float64)), _p(out))
    return out, bool(ok)


def pcg(vals, rows, cols, nb, b, *, precond=PRECOND_MAS32, gate=GATE_RZ, tol=1e-4, max_iter=0, fem_offset=0,
        fem_count=0, abd_bodies=0, mas: Mas32 | None = None, replay_checks=False):
    """PCGSolver::pcg restated; returns (x, result dict)."""
    o = _PcgOpts(precond, gate, tol, max_iter, nb, fem_offset, fem_count, abd_bodies, 1 if replay_checks else 0)
    res = _PcgResult()
    b = _c(b, np.float64)
    x = np.zeros_like(b)
    L = lib() if mas is None else mas._lib
    L.orc_pcg(ctypes.byref(o), _p(_c(vals, np.float64)), _p(_c(rows, np.int32)), _p(_c(cols, np.int32)),
              len(rows), None if mas is None else mas.h, _p(b), _p(x), ctypes.byref(res))
    return x, {"iterations": res.iterations, "status": STATUS_NAMES.get(res.status, res.status), "rz0": res.rz0,
               "rz_last": res.rz_last, "rel_res_recursive": res.rel_res_recursive, "rel_res_true": res.rel_res_true}


def solve_system(s, *, precond=PRECOND_MAS32, gate=GATE_RZ, tol=1e-4, max_iter=0, replay_checks=False):
    """Full reference pipeline on a synth.System: MAS build then PCG."""
    mas = None
    if precond in (PRECOND_MAS32, PRECOND_MAS16) and s.fem_count > 0:
        mas = (Mas32 if precond == PRECOND_MAS32 else Mas16).from_system(s)
        mas.reorder(s.pairs)
        sel = np.nonzero((s.rows >= s.fem_offset) & (s.rows < s.fem_offset + s.fem_count) &
                         (s.cols >= s.fem_offset) & (s.cols < s.fem_offset + s.fem_count))[0].astype(np.uint32)
        mas.prepare_hessian(s.vals, s.rows, s.cols, sel, s.fem_offset)
    x, r = pcg(s.vals, s.rows, s.cols, s.nb, s.b, precond=precond, gate=gate, tol=tol, max_iter=max_iter,
               fem_offset=s.fem_offset, fem_count=s.fem_count, abd_bodies=s.abd_bodies, mas=mas,
               replay_checks=replay_checks)
    return x, r, mas


def num_threads():
    return lib().orc_num_threads()
