"""Seeded synthetic IPC Newton systems for the MAS-PCG solve.

The reference (StiffGIPC) builds its Newton Hessian from a scene.  The five
workloads below rebuild systems of the same structure from the same formulas
(see ``csrc/synth.c``): Freudenthal tetrahedral boxes with stable Neo-Hookean
element Hessians (``femEnergy.cu:432-459``), lumped mass (``gl_main.cu:611-614``),
IPC barrier Hessians for point-triangle / edge-edge pairs, and affine bodies
with ``J^T H`` coupling blocks (``setup_abd_system_gradient_and_hessian.cu:348-405``).
Scaling: ``A = M + dt^2 (K + kappa * barrier)``, the incremental potential
of IPC.  The reference enters mass unscaled and elasticity with dt^2
(``GIPC.cu:10183-10199``, ``femEnergy.cu:1719-1856``) and passes an adaptive
kappa that absorbs dt^2 to the barrier (``GIPC.cu:9935-9943``); the workloads
fix kappa, so dt^2 is applied explicitly.  Unscaled, kappa=1e7 makes contact
blocks ~1e7 times the elastic ones and FP32 products of A lose positivity.

Every system is returned as the unique upper BCOO that
``GlobalLinearSystem::convert_new`` hands to the solver
(``global_linear_system.cu:310-319``) plus the caller-side MAS32 inputs:
the vertex neighbour CSR (``load_mesh.cpp:934-1040``), the Morton partition
maps (``gl_main.cu:1178-1242``) and the int4 contact pairs.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

SEED_BASE = 20261203


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libmassynth.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run agipc_learning_b200.build.build_all() first")
        lib = ctypes.CDLL(path)
        P = ctypes.c_void_p
        LL = ctypes.c_longlong
        I = ctypes.c_int
        D = ctypes.c_double
        U64 = ctypes.c_uint64
        sig = {
            "syn_normal": (None, [LL, U64, I, P]),
            "syn_box_sizes": (None, [I, I, I, P, P]),
            "syn_box_mesh": (None, [I, I, I, D, P, P]),
            "syn_perturb": (None, [LL, P, D, U64, P]),
            "syn_fem_triplets": (LL, [LL, P, P, P, P, D, D, D, I, P, P, P]),
            "syn_lumped_mass": (None, [LL, LL, P, P, D, P]),
            "syn_mass_triplets": (None, [LL, P, I, P, P, P]),
            "syn_boundary_triangles": (LL, [LL, LL, P, P]),
            "syn_boundary_edges": (LL, [LL, P, P]),
            "syn_contacts_pt": (LL, [I, I, I, D, P, LL, P, LL, D, D, U64, I, I, P, P, P, P]),
            "syn_contacts_ee": (LL, [I, I, I, D, P, LL, P, LL, D, D, U64, I, I, P, P, P, P]),
            "syn_abd_bodies": (None, [I, D, D, D, D, D, U64, P, P, P]),
            "syn_abd_contacts": (LL, [I, D, LL, P, P, LL, D, D, D, U64, I, P, P, P, P]),
            "syn_assemble": (LL, [LL, P, P, P, P, P, P]),
            "syn_vertex_neighbors": (LL, [LL, LL, P, P, P, P]),
            "syn_morton_partition": (None, [LL, P, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class System:
    """An assembled Newton system plus the caller-side MAS32 inputs."""

    name: str
    nb: int                       # block rows
    rows: np.ndarray              # int32 [B_u], row <= col
    cols: np.ndarray              # int32 [B_u]
    vals: np.ndarray              # float64 [B_u, 9], Eigen column-major 3x3
    b: np.ndarray                 # float64 [3*nb]
    fem_offset: int               # first FEM block row
    fem_count: int                # FEM vertices (MAS range)
    abd_bodies: int = 0
    neighbor_start: np.ndarray | None = None
    neighbor_num: np.ndarray | None = None
    neighbor_list: np.ndarray | None = None
    part_map_real: np.ndarray | None = None
    real_map_part: np.ndarray | None = None
    pairs: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int32))
    node_offset: int = 0          # vertex-number offset of the FEM range in `pairs`
    X: np.ndarray | None = None   # rest positions of the FEM vertices
    tets: np.ndarray | None = None
    E_tet: np.ndarray | None = None
    meta: dict = field(default_factory=dict)

    @property
    def dof(self) -> int:
        return 3 * self.nb


def box_mesh(nx: int, ny: int, nz: int, h: float):
    lib = _lib()
    nv = ctypes.c_longlong()
    nt = ctypes.c_longlong()
    lib.syn_box_sizes(nx, ny, nz, ctypes.byref(nv), ctypes.byref(nt))
    X = np.zeros((nv.value, 3), np.float64)
    tets = np.zeros((nt.value, 4), np.int32)
    lib.syn_box_mesh(nx, ny, nz, h, _p(X), _p(tets))
    return X, tets


def vertex_neighbors(nv: int, tets: np.ndarray):
    """Neighbour CSR with the ordering of tetrahedra_obj::getVertNeighbors."""
    lib = _lib()
    start = np.zeros(nv, np.uint32)
    num = np.zeros(nv, np.uint32)
    lst = np.zeros(12 * len(tets) + 1, np.uint32)
    n = lib.syn_vertex_neighbors(nv, len(tets), _p(np.ascontiguousarray(tets, np.int32)), _p(start), _p(num), _p(lst))
    return start, num, lst[:n].copy()


def morton_partition(X: np.ndarray):
    """part_map_real (ceil32(nv), -1 padded) and real_map_part (nv)."""
    lib = _lib()
    nv = len(X)
    pmr = np.full((nv + 31) // 32 * 32, -1, np.int32)
    rmp = np.zeros(nv, np.int32)
    lib.syn_morton_partition(nv, _p(np.ascontiguousarray(X, np.float64)), _p(pmr), _p(rmp))
    return pmr, rmp


def assemble(rows, cols, vals):
    """Sum duplicate triplets; returns the sorted unique BCOO."""
    lib = _lib()
    n = len(rows)
    r = np.ascontiguousarray(rows, np.int32)
    c = np.ascontiguousarray(cols, np.int32)
    v = np.ascontiguousarray(vals, np.float64).reshape(n, 9)
    orow = np.zeros(n, np.int32)
    ocol = np.zeros(n, np.int32)
    oval = np.zeros((n, 9), np.float64)
    u = lib.syn_assemble(n, _p(r), _p(c), _p(v), _p(orow), _p(ocol), _p(oval))
    return orow[:u].copy(), ocol[:u].copy(), oval[:u].copy()


def normal_rhs(n: int, seed: int, fp32: bool = True) -> np.ndarray:
    out = np.zeros(n, np.float64)
    _lib().syn_normal(n, seed, 1 if fp32 else 0, _p(out))
    return out


def _fem_block(X, tets, x, E, nu, dt, rho, row_offset, E_tet=None):
    lib = _lib()
    nt = len(tets)
    rows = np.zeros(10 * nt, np.int32)
    cols = np.zeros(10 * nt, np.int32)
    vals = np.zeros((10 * nt, 9), np.float64)
    Et = None if E_tet is None else np.ascontiguousarray(E_tet, np.float64)
    projected = lib.syn_fem_triplets(nt, _p(tets), _p(X), _p(x), None if Et is None else _p(Et),
                                     float(E), float(nu), float(dt), int(row_offset), _p(rows), _p(cols), _p(vals))
    mass = np.zeros(len(X), np.float64)
    lib.syn_lumped_mass(len(X), nt, _p(tets), _p(X), float(rho), _p(mass))
    mr = np.zeros(len(X), np.int32)
    mc = np.zeros(len(X), np.int32)
    mv = np.zeros((len(X), 9), np.float64)
    lib.syn_mass_triplets(len(X), _p(mass), int(row_offset), _p(mr), _p(mc), _p(mv))
    return [rows, mr], [cols, mc], [vals, mv], int(projected)


def cube_system(n: int, *, E: float = 1e5, nu: float = 0.45, rho: float = 1000.0, dt: float = 1 / 60,
                h: float = 0.01, noise: float = 0.1, seed: int = SEED_BASE, pt_pairs: int = 0, ee_pairs: int = 0,
                dhat: float = 1e-3, kappa: float = 1e7, E_tet=None, name: str | None = None,
                nxyz: tuple[int, int, int] | None = None, keep_raw: bool = False) -> System:
    """FEM box (n^3 vertices unless nxyz is given) with optional IPC contacts.

    keep_raw: also keep the unmerged triplets in meta["raw"] = (rows, cols,
    vals), element blocks first (10 per tet, in tet order, each proportional
    to the tet's Young's modulus), then the mass and contact blocks;
    meta["elem_blocks"] is the element-block count."""
    lib = _lib()
    nx, ny, nz = nxyz if nxyz else (n, n, n)
    X, tets = box_mesh(nx, ny, nz, h)
    nv = len(X)
    x = np.zeros_like(X)
    lib.syn_perturb(nv, _p(X), noise * h, seed, _p(x))
    R, C, V, projected = _fem_block(X, tets, x, E, nu, dt, rho, 0, E_tet)
    pairs = []
    if pt_pairs or ee_pairs:
        tris = np.zeros((4 * len(tets), 3), np.int32)
        ntri = lib.syn_boundary_triangles(nv, len(tets), _p(tets), _p(tris))
        tris = tris[:ntri].copy()
        if pt_pairs:
            p4 = np.zeros((pt_pairs, 4), np.int32)
            r = np.zeros(10 * pt_pairs, np.int32)
            c = np.zeros(10 * pt_pairs, np.int32)
            v = np.zeros((10 * pt_pairs, 9), np.float64)
            k = lib.syn_contacts_pt(nx, ny, nz, h, _p(X), ntri, _p(tris), pt_pairs, dhat, kappa * dt * dt, seed + 101, 0, 0,
                                    _p(p4), _p(r), _p(c), _p(v))
            pairs.append(p4[:k]); R.append(r[:10 * k]); C.append(c[:10 * k]); V.append(v[:10 * k])
        if ee_pairs:
            edges = np.zeros((3 * ntri, 2), np.int32)
            ne = lib.syn_boundary_edges(ntri, _p(tris), _p(edges))
            edges = edges[:ne].copy()
            p4 = np.zeros((ee_pairs, 4), np.int32)
            r = np.zeros(10 * ee_pairs, np.int32)
            c = np.zeros(10 * ee_pairs, np.int32)
            v = np.zeros((10 * ee_pairs, 9), np.float64)
            k = lib.syn_contacts_ee(nx, ny, nz, h, _p(X), ne, _p(edges), ee_pairs, dhat, kappa * dt * dt, seed + 202, 0, 0,
                                    _p(p4), _p(r), _p(c), _p(v))
            pairs.append(p4[:k]); R.append(r[:10 * k]); C.append(c[:10 * k]); V.append(v[:10 * k])
    raw = (np.concatenate(R), np.concatenate(C), np.concatenate(V))
    rows, cols, vals = assemble(*raw)
    start, num, lst = vertex_neighbors(nv, tets)
    pmr, rmp = morton_partition(X)
    b = normal_rhs(3 * nv, seed + 7, fp32=True)
    meta = {"projected_tets": projected, "E": E, "nu": nu, "dt": dt, "rho": rho, "h": h}
    if keep_raw:
        meta["raw"] = raw
        meta["elem_blocks"] = 10 * len(tets)
    return System(name=name or f"cube{n}", nb=nv, rows=rows, cols=cols, vals=vals, b=b, fem_offset=0,
                  fem_count=nv, neighbor_start=start, neighbor_num=num, neighbor_list=lst, part_map_real=pmr,
                  real_map_part=rmp, pairs=np.concatenate(pairs) if pairs else np.zeros((0, 4), np.int32),
                  node_offset=0, X=X, tets=tets, E_tet=None if E_tet is None else np.asarray(E_tet), meta=meta)


def hybrid_system(bodies: int = 2000, slab=(100, 100, 10), *, E: float = 1e8, nu: float = 0.3, rho: float = 1000.0,
                  dt: float = 1 / 60, h: float = 0.01, noise: float = 0.1, body_mass: float = 1.0,
                  body_size: float = 0.05, orth_stiffness: float = 1e8, body_noise: float = 1e-3,
                  pairs: int = 30000, dhat: float = 1e-3, kappa: float = 1e8, seed: int = SEED_BASE + 2,
                  name: str = "hybrid") -> System:
    """ABD bodies (block rows [0, 4*bodies)) coupled to a FEM slab."""
    lib = _lib()
    X, tets = box_mesh(*slab, h)
    nv = len(X)
    x = np.zeros_like(X)
    lib.syn_perturb(nv, _p(X), noise * h, seed, _p(x))
    off = 4 * bodies
    R, C, V, projected = _fem_block(X, tets, x, E, nu, dt, rho, off)
    br = np.zeros(10 * bodies, np.int32)
    bc = np.zeros(10 * bodies, np.int32)
    bv = np.zeros((10 * bodies, 9), np.float64)
    lib.syn_abd_bodies(bodies, body_mass, body_size, orth_stiffness, body_noise, dt, seed + 11, _p(br), _p(bc), _p(bv))
    R.append(br); C.append(bc); V.append(bv)
    tris = np.zeros((4 * len(tets), 3), np.int32)
    ntri = lib.syn_boundary_triangles(nv, len(tets), _p(tets), _p(tris))
    tris = tris[:ntri]
    ztop = (slab[2] - 1) * h
    top = np.ascontiguousarray(tris[np.all(np.abs(X[tris][:, :, 2] - ztop) < 1e-9, axis=1)], np.int32)
    p4 = np.zeros((pairs, 4), np.int32)
    cr = np.zeros(28 * pairs, np.int32)
    cc = np.zeros(28 * pairs, np.int32)
    cv = np.zeros((28 * pairs, 9), np.float64)
    w = lib.syn_abd_contacts(bodies, body_size, len(top), _p(top), _p(X), pairs, dhat, kappa * dt * dt, h, seed + 303, off,
                             _p(p4), _p(cr), _p(cc), _p(cv))
    R.append(cr[:w]); C.append(cc[:w]); V.append(cv[:w])
    rows, cols, vals = assemble(np.concatenate(R), np.concatenate(C), np.concatenate(V))
    start, num, lst = vertex_neighbors(nv, tets)
    pmr, rmp = morton_partition(X)
    nb = off + nv
    b = normal_rhs(3 * nb, seed + 7, fp32=True)
    return System(name=name, nb=nb, rows=rows, cols=cols, vals=vals, b=b, fem_offset=off, fem_count=nv,
                  abd_bodies=bodies, neighbor_start=start, neighbor_num=num, neighbor_list=lst, part_map_real=pmr,
                  real_map_part=rmp, pairs=p4, node_offset=8 * bodies, X=X, tets=tets,
                  meta={"projected_tets": projected, "E": E, "nu": nu, "dt": dt, "rho": rho, "h": h})


def partition_for_bank(s: System, bank: int, *, sorted_ids: bool = True) -> System:
    """The system with a MAS partition of `bank`-slot banks (16: CEMAS16).

    sorted_ids=True renumbers the FEM vertices in Morton order, as the app's
    METIS-sorted meshes number a part's vertices consecutively for CEMAS16
    (gl_main.cu:1118-1145), so vertex v sits in slot v and the slots of every
    bank follow the vertex order.  sorted_ids=False keeps the numbering and
    packs the Morton order into banks, so inside a bank the slot order runs
    against the vertex order."""
    import dataclasses
    nv, fo = s.fem_count, s.fem_offset
    order = np.asarray(s.part_map_real)[np.asarray(s.part_map_real) >= 0].astype(np.int64)  # Morton order
    padded = (nv + bank - 1) // bank * bank
    pmr = np.full(padded, -1, np.int32)
    if not sorted_ids:
        pmr[:nv] = order
        rmp = np.zeros(nv, np.int32)
        rmp[order] = np.arange(nv, dtype=np.int32)
        return dataclasses.replace(s, part_map_real=pmr, real_map_part=rmp)
    new = np.empty(nv, np.int64)
    new[order] = np.arange(nv)
    gmap = np.arange(s.nb, dtype=np.int64)
    gmap[fo:fo + nv] = fo + new
    r, c = gmap[s.rows], gmap[s.cols]
    v = np.asarray(s.vals, np.float64).reshape(-1, 3, 3).copy()
    swap = r > c
    r2, c2 = np.where(swap, c, r), np.where(swap, r, c)
    v[swap] = v[swap].transpose(0, 2, 1)
    rows, cols, vals = assemble(r2, c2, v.reshape(-1, 9))
    b = np.asarray(s.b, np.float64).reshape(-1, 3).copy()
    b[fo + new] = np.asarray(s.b).reshape(-1, 3)[fo:fo + nv]
    st, nn, nl = (np.asarray(a) for a in (s.neighbor_start, s.neighbor_num, s.neighbor_list))
    lists = [new[nl[st[o]:st[o] + nn[o]]] for o in order]
    num = np.array([len(x) for x in lists], np.uint32)
    start = np.zeros(nv, np.uint32)
    start[1:] = np.cumsum(num)[:-1]
    lst = np.concatenate(lists).astype(np.uint32) if nv else np.zeros(0, np.uint32)
    pairs = np.asarray(s.pairs, np.int64).copy()
    if pairs.size:
        vtx = np.where(pairs >= 0, pairs, -pairs - 1)
        loc = vtx - s.node_offset
        inr = (loc >= 0) & (loc < nv)
        mapped = np.where(inr, s.node_offset + new[np.clip(loc, 0, nv - 1)], vtx)
        pairs = np.where(pairs >= 0, mapped, -mapped - 1)
    pmr[:nv] = np.arange(nv, dtype=np.int32)
    meta = {k: v_ for k, v_ in s.meta.items() if k not in ("raw", "elem_blocks")}
    X = None if s.X is None else np.asarray(s.X)[order]
    tets = None if s.tets is None else new[np.asarray(s.tets)].astype(np.int32)
    return dataclasses.replace(s, rows=rows, cols=cols, vals=vals, b=b.reshape(-1), neighbor_start=start,
                               neighbor_num=num, neighbor_list=lst, part_map_real=pmr,
                               real_map_part=np.arange(nv, dtype=np.int32), pairs=pairs.astype(np.int32), X=X,
                               tets=tets, meta=meta, name=f"{s.name}_b{bank}")


def log_uniform_E(ntet: int, lo: float, hi: float, seed: int) -> np.ndarray:
    """Per-tet Young's modulus, log-uniform in [lo, hi] (numpy PCG64 stream)."""
    u = np.random.default_rng(seed).random(ntet)
    return np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))


CONFIGS = {
    0: "cube 20^3, E=1e5, nu=0.45, no contact",
    1: "cube 64^3, E=1e6, 50,000 point-triangle pairs, kappa=1e7",
    2: "2,000 ABD bodies + 100x100x10 slab (E=1e8, nu=0.3), 30,000 ABD-FEM pairs, kappa=1e8",
    3: "cube 32^3, per-tet E log-uniform [1e4, 1e6]",
    4: "cube 128^3, E=1e8, 400,000 point-triangle + edge-edge pairs, kappa=1e8",
}


def config_system(cid: int, scale: int | None = None) -> System:
    """The five workloads.  `scale` overrides the cube edge (tests use small ones)."""
    seed = SEED_BASE + cid
    if cid == 0:
        return cube_system(scale or 20, E=1e5, nu=0.45, seed=seed, name="cfg0")
    if cid == 1:
        n = scale or 64
        npairs = 50000 if n == 64 else max(1, int(50000 * (n / 64) ** 2))
        return cube_system(n, E=1e6, nu=0.45, seed=seed, pt_pairs=npairs, dhat=1e-3, kappa=1e7, name="cfg1")
    if cid == 2:
        if scale:
            return hybrid_system(bodies=max(4, scale * 2), slab=(scale, scale, max(3, scale // 4)),
                                 pairs=max(8, scale * 30), seed=seed, name="cfg2")
        return hybrid_system(seed=seed, name="cfg2")
    if cid == 3:
        n = scale or 32
        ntet = 6 * (n - 1) ** 3
        E_tet = log_uniform_E(ntet, 1e4, 1e6, seed + 5)
        return cube_system(n, E=1e5, nu=0.45, seed=seed, E_tet=E_tet, name="cfg3", keep_raw=True)
    if cid == 4:
        n = scale or 128
        npairs = 400000 if n == 128 else max(2, int(400000 * (n / 128) ** 2))
        return cube_system(n, E=1e8, nu=0.45, seed=seed, pt_pairs=npairs // 2, ee_pairs=npairs - npairs // 2,
                           dhat=1e-3, kappa=1e8, name="cfg4")
    raise ValueError(cid)


def blocks_to_vals9(blocks: np.ndarray) -> np.ndarray:
    """[n,3,3] (row, col) -> [n,9] Eigen column-major."""
    return np.ascontiguousarray(np.asarray(blocks).transpose(0, 2, 1).reshape(-1, 9))


def vals9_to_blocks(vals: np.ndarray) -> np.ndarray:
    return np.asarray(vals).reshape(-1, 3, 3).transpose(0, 2, 1)
