"""Host-side mirror of StiffGIPC's linear-solve interface over the C ABI.

``MasPcg`` owns one ``maspcg_handle``.  ``PCGSolverConfig``, ``PCGSolver`` and
``TraditionalMAS32Preconditioner`` keep the reference's names, argument
meaning and call order (``linear_system/solver/pcg_solver.h:7-50``,
``TraditionalMAS32Preconditioner.cuh:35-129``, caller ``gl_main.cu:1502-1536``)
so code written against the reference maps one to one.  Arrays may be numpy
arrays (host) or CUDA torch tensors (device); every call goes through
``libmaspcg.so``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native as N

_PREC = {"reference": N.PREC_REFERENCE, "fp32": N.PREC_FP32, "mixed": N.PREC_MIXED}
_GATE = {"rz": N.GATE_RZ, "euclid": N.GATE_EUCLID}
_INV = {"fp32": N.INV_FP32, "bf16": N.INV_BF16, "fp16": N.INV_FP16}
_MATRIX = {"f32": N.MATRIX_F32, "f32_accurate": N.MATRIX_F32_ACCURATE, "f32_split": N.MATRIX_F32_SPLIT,
           "f32_compensated": N.MATRIX_F32_COMPENSATED}
_REPLACE = {"reliable": N.REPLACE_RELIABLE, "periodic": N.REPLACE_PERIODIC}
_PC = {"mas32": N.PRECOND_MAS32, "cemas16": N.PRECOND_MAS16, "block_jacobi": N.PRECOND_BLOCK_JACOBI,
       "none": N.PRECOND_NONE}


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


class _Arg:
    """Pointer to a contiguous numpy array or CUDA tensor of a given dtype."""

    def __init__(self, a, np_dtype, writable=False):
        self.keep = None
        self.device = None  # CUDA tensors: the device of the torch stream that produces / consumes them
        if a is None:
            self.ptr = None
            return
        if _is_torch(a):
            import torch
            want = {np.float64: torch.float64, np.int32: torch.int32, np.uint32: torch.int32,
                    np.uint64: torch.int64}[np_dtype]
            if a.dtype != want or not a.is_contiguous():
                if writable:
                    raise ValueError("output tensor must be contiguous with the right dtype")
                a = a.to(want).contiguous()
            self.keep = a
            self.ptr = ctypes.c_void_p(a.data_ptr())
            self.device = a.device if a.is_cuda else None
        else:
            arr = np.asarray(a)
            if arr.dtype != np_dtype or not arr.flags["C_CONTIGUOUS"]:
                if writable:
                    raise ValueError("output array must be C-contiguous with the right dtype")
                arr = np.ascontiguousarray(arr, dtype=np_dtype)
            self.keep = arr
            self.ptr = arr.ctypes.data_as(ctypes.c_void_p)


class MasPcg:
    """One linear system on one GPU: graph -> contacts -> matrix -> build -> solve."""

    def __init__(self, *, tolerance=1e-4, max_iter_ratio=0.3, max_iterations=0, gate="rz", precision="reference",
                 inverse="fp32", preconditioner="mas32", refinement_period=16, iterations_per_launch=8, flags=0,
                 matrix="f32", replacement="periodic"):
        self._torch_args = []
        lib = N.load()
        cfg = N.Config()
        lib.maspcg_config_default(ctypes.byref(cfg))
        cfg.tolerance = tolerance
        cfg.max_iter_ratio = max_iter_ratio
        cfg.max_iterations = max_iterations
        cfg.gate = _GATE[gate]
        cfg.precision = _PREC[precision]
        cfg.inverse_storage = _INV[inverse]
        cfg.preconditioner = _PC[preconditioner]
        cfg.bank_size = 16 if preconditioner == "cemas16" else 32
        cfg.refinement_period = refinement_period
        cfg.iterations_per_launch = iterations_per_launch
        cfg.flags = flags
        cfg.matrix_form = _MATRIX[matrix]
        cfg.residual_replacement = _REPLACE[replacement]
        self.cfg = cfg
        h = ctypes.c_void_p()
        N.check(lib.maspcg_create(ctypes.byref(cfg), ctypes.byref(h)), None)
        self.h = h
        self.lib = lib
        self.nb = 0
        self.nv = 0

    # -- lifecycle
    def close(self):
        if getattr(self, "h", None):
            self.lib.maspcg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ck(self, status):
        """Checks a call's status.  If the call took CUDA tensors, torch's
        current stream first waits for the handle's stream (an event, no host
        sync): torch work after the call sees the outputs, and tensors the call
        read are not recycled by torch's allocator before the reads are done."""
        pending, self._torch_args = self._torch_args, []
        if pending:
            import torch
            ev = torch.cuda.Event()
            ev.record(torch.cuda.ExternalStream(self._stream_ptr(), device=pending[0]))
            torch.cuda.current_stream(pending[0]).wait_event(ev)
        N.check(status, self.h)

    def _stream_ptr(self) -> int:
        s = ctypes.c_void_p()
        N.check(self.lib.maspcg_get_stream(self.h, ctypes.byref(s)), self.h)
        return s.value or 0

    def _arg(self, a, np_dtype, writable=False) -> "_Arg":
        """An argument for the next call.  A CUDA tensor may still be being
        written by torch's current stream, and the library runs on its own
        stream (non-blocking unless set_stream chose another): the handle's
        stream waits for torch's first (an event, no host sync)."""
        arg = _Arg(a, np_dtype, writable)
        if arg.device is not None:
            import torch
            ev = torch.cuda.Event()
            ev.record(torch.cuda.current_stream(arg.device))
            torch.cuda.ExternalStream(self._stream_ptr(), device=arg.device).wait_event(ev)
            self._torch_args.append(arg.device)
        return arg

    # -- inputs
    def set_stream(self, stream_ptr: int | None):
        self._ck(self.lib.maspcg_set_stream(self.h, ctypes.c_void_p(stream_ptr or 0)))

    def set_graph(self, vert_num, node_offset, neighbor_start, neighbor_num, neighbor_list, part_map_real,
                  real_map_part):
        a = [self._arg(neighbor_start, np.uint32), self._arg(neighbor_num, np.uint32),
             self._arg(neighbor_list if len(neighbor_list) else np.zeros(1, np.uint32), np.uint32),
             self._arg(part_map_real, np.int32), self._arg(real_map_part, np.int32)]
        self._ck(self.lib.maspcg_set_graph(self.h, int(vert_num), int(node_offset), a[0].ptr, a[1].ptr, a[2].ptr,
                                           int(len(neighbor_list)), a[3].ptr, int(len(part_map_real)), a[4].ptr))
        self.nv = int(vert_num)

    def set_contacts(self, pairs):
        p = np.zeros((0, 4), np.int32) if pairs is None else pairs
        n = len(p)
        arg = self._arg(p if n else np.zeros(4, np.int32), np.int32)
        self._ck(self.lib.maspcg_set_contacts(self.h, arg.ptr, int(n)))

    def set_matrix(self, vals, rows, cols, block_rows, fem_offset=0, abd_bodies=0):
        v, r, c = self._arg(vals, np.float64), self._arg(rows, np.int32), self._arg(cols, np.int32)
        self._ck(self.lib.maspcg_set_matrix_bcoo(self.h, v.ptr, r.ptr, c.ptr, int(len(rows)), int(block_rows),
                                                 int(fem_offset), int(abd_bodies)))
        self.nb = int(block_rows)
        self.matrix_version = getattr(self, "matrix_version", 0) + 1

    def set_matrix_indexed(self, vals, rows, cols, indices, offset, block_rows, fem_offset=0, abd_bodies=0):
        """The subsystem triplets indices[t] of a larger list, indices minus
        `offset` (maspcg_set_matrix_bcoo_indexed); the gather runs on the
        device, so CUDA tensors stay on the device."""
        v, r, c = self._arg(vals, np.float64), self._arg(rows, np.int32), self._arg(cols, np.int32)
        ix = self._arg(indices, np.uint32)
        n = len(rows) if indices is None else len(indices)
        self._ck(self.lib.maspcg_set_matrix_bcoo_indexed(self.h, v.ptr, r.ptr, c.ptr, int(len(rows)), ix.ptr, int(n),
                                                         int(offset), int(block_rows), int(fem_offset),
                                                         int(abd_bodies)))
        self.nb = int(block_rows)
        self.matrix_version = getattr(self, "matrix_version", 0) + 1

    def build(self):
        self._ck(self.lib.maspcg_build_preconditioner(self.h))

    def refresh_values(self, vals):
        """New values for the blocks of the last set_matrix (same triplets, same
        order): merged values, domain matrices and inverses recomputed on the
        kept structure and hierarchy (maspcg_refresh_matrix_values)."""
        self._ck(self.lib.maspcg_refresh_matrix_values(self.h, self._arg(vals, np.float64).ptr))

    def refresh_values_indexed(self, vals, indices):
        """refresh_values with the values picked by index on the device
        (maspcg_refresh_matrix_values_indexed)."""
        v, ix = self._arg(vals, np.float64), self._arg(indices, np.uint32)
        self._ck(self.lib.maspcg_refresh_matrix_values_indexed(self.h, v.ptr, int(len(vals)), ix.ptr))

    def local_diagnostics(self, per_domain=False):
        """Per-domain SPD and inverse-residual checks of the last build
        (maspcg_local_diagnostics): the summary dict, and with per_domain the
        list of per-domain checks."""
        d = self.info()["domains"]
        arr = (N.DomainCheck * max(d, 1))() if per_domain else None
        summ = N.Diagnostics()
        self._ck(self.lib.maspcg_local_diagnostics(self.h, ctypes.cast(arr, ctypes.c_void_p) if arr else None,
                                                   ctypes.byref(summ)))
        out = summ.as_dict()
        if per_domain:
            out["domains"] = [{k: getattr(c, k) for k, _ in c._fields_} for c in arr[:d]]
        return out

    def check_local_matrices(self, packed64, inverse32, bank=32):
        """gpu_local_checks on caller matrices (maspcg_check_local_matrices):
        returns (summary, per-domain list)."""
        p = np.ascontiguousarray(packed64, np.float64)
        q = np.ascontiguousarray(inverse32, np.float32)
        count = p.shape[0]
        arr = (N.DomainCheck * max(count, 1))()
        summ = N.Diagnostics()
        self._ck(self.lib.maspcg_check_local_matrices(self.h, int(count), int(bank), p.ctypes.data_as(ctypes.c_void_p),
                                                      q.ctypes.data_as(ctypes.c_void_p),
                                                      ctypes.cast(arr, ctypes.c_void_p), ctypes.byref(summ)))
        return summ.as_dict(), [{k: getattr(c, k) for k, _ in c._fields_} for c in arr[:count]]

    @classmethod
    def from_system(cls, s, **cfg):
        """Set up graph, contacts and matrix of a synth.System and build."""
        m = cls(**cfg)
        if m.cfg.preconditioner in (N.PRECOND_MAS32, N.PRECOND_MAS16) and s.fem_count > 0:
            m.set_graph(s.fem_count, s.node_offset, s.neighbor_start, s.neighbor_num, s.neighbor_list,
                        s.part_map_real, s.real_map_part)
            m.set_contacts(s.pairs)
        m.set_matrix(s.vals, s.rows, s.cols, s.nb, s.fem_offset, s.abd_bodies)
        m.build()
        return m

    # -- operations
    def _out(self, out, n):
        if out is None:
            out = np.zeros(n, np.float64)
        return out, self._arg(out, np.float64, writable=True)

    def solve(self, b, x=None):
        bx = self._arg(b, np.float64)
        x, xa = self._out(x, 3 * self.nb)
        res = N.Result()
        self._ck(self.lib.maspcg_solve(self.h, bx.ptr, xa.ptr, ctypes.byref(res)))
        return x, res.as_dict()

    def apply_preconditioner(self, r, z=None):
        ra = self._arg(r, np.float64)
        z, za = self._out(z, 3 * self.nb)
        self._ck(self.lib.maspcg_apply_preconditioner(self.h, ra.ptr, za.ptr))
        return z

    def spmv(self, x, a=1.0, b=0.0, y=None):
        xa = self._arg(x, np.float64)
        if y is None:
            y = np.zeros(3 * self.nb, np.float64)
        ya = self._arg(y, np.float64, writable=True)
        self._ck(self.lib.maspcg_spmv(self.h, float(a), xa.ptr, float(b), ya.ptr))
        return y

    def spmv_working(self, x, y=None):
        """y = A x as the PCG iteration's own SpMV kernel forms it, in the
        working precision (maspcg_spmv_working)."""
        xa = self._arg(x, np.float64)
        y, ya = self._out(y, 3 * self.nb)
        self._ck(self.lib.maspcg_spmv_working(self.h, xa.ptr, ya.ptr))
        return y

    def adjust_contact_triplets(self, rows, cols, values9, bd_type, fem_offset):
        """Contact-pair dedup in place (maspcg_adjust_contact_triplets;
        adjust_fem_fem_contact_indices_kernel).  numpy arrays are adjusted in
        place and returned; CUDA tensors likewise."""
        r, c, v = self._arg(rows, np.int32, True), self._arg(cols, np.int32, True), self._arg(values9, np.float64, True)
        bd = self._arg(bd_type, np.int32)
        self._ck(self.lib.maspcg_adjust_contact_triplets(self.h, int(len(rows)), r.ptr, c.ptr, v.ptr, bd.ptr,
                                                         int(len(bd_type)), int(fem_offset)))
        return rows, cols, values9

    def zero_boundary_triplets(self, rows, cols, values9, bd_type, index_offset):
        """Boundary blocks cleared in place (maspcg_zero_boundary_triplets;
        zero_fem_boundary_hessian_kernel)."""
        r, c, v = self._arg(rows, np.int32), self._arg(cols, np.int32), self._arg(values9, np.float64, True)
        bd = self._arg(bd_type, np.int32)
        self._ck(self.lib.maspcg_zero_boundary_triplets(self.h, int(len(rows)), r.ptr, c.ptr, v.ptr, bd.ptr,
                                                        int(len(bd_type)), int(index_offset)))
        return values9

    def _outs(self, like, n):
        """rows, cols (int32) and values (n x 9 float64) outputs on the device of `like`."""
        if _is_torch(like) and like.is_cuda:
            import torch
            return (torch.empty(n, dtype=torch.int32, device=like.device),
                    torch.empty(n, dtype=torch.int32, device=like.device),
                    torch.empty((n, 9), dtype=torch.float64, device=like.device))
        return np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros((n, 9), np.float64)

    def convert_bcoo(self, rows, cols, values9):
        """The triplet merge (maspcg_convert_bcoo; Converter::convert): unique
        (row, col) keys in ascending order with their blocks summed in input
        order.  Returns (rows, cols, values9) trimmed to the unique count."""
        n = int(len(rows))
        ro, co, vo = self._outs(rows, n)
        r, c, v = self._arg(rows, np.int32), self._arg(cols, np.int32), self._arg(values9, np.float64)
        ra, ca, va = self._arg(ro, np.int32, True), self._arg(co, np.int32, True), self._arg(vo, np.float64, True)
        cnt = ctypes.c_int()
        self._ck(self.lib.maspcg_convert_bcoo(self.h, v.ptr, r.ptr, c.ptr, n, va.ptr, ra.ptr, ca.ptr, ctypes.byref(cnt)))
        u = cnt.value
        return ro[:u], co[:u], vo[:u]

    def partition_contact_triplets(self, rows, cols, values9, type_hash):
        """Contact triplets grouped by type hash 0..3 (maspcg_partition_contact_triplets;
        GIPC::partitionContactHessian).  Returns (rows, cols, values9, counts[4])."""
        n = int(len(rows))
        ro, co, vo = self._outs(rows, n)
        r, c, v = self._arg(rows, np.int32), self._arg(cols, np.int32), self._arg(values9, np.float64)
        t = self._arg(type_hash, np.uint64)
        ra, ca, va = self._arg(ro, np.int32, True), self._arg(co, np.int32, True), self._arg(vo, np.float64, True)
        counts = (ctypes.c_int * 4)()
        self._ck(self.lib.maspcg_partition_contact_triplets(self.h, v.ptr, r.ptr, c.ptr, t.ptr, n, va.ptr, ra.ptr,
                                                            ca.ptr, counts))
        return ro, co, vo, np.array(list(counts), np.int32)

    def fem_snk1(self, tets, x, dm_inverse, volume, len_rate, vol_rate, dt, hessian_offset=0, gradient=None):
        """Per-tet SNK1 gradient (accumulated into `gradient`, zeros if None)
        and projected Hessian triplets (maspcg_fem_snk1_gradient_hessian).
        numpy in, numpy out.  Returns (gradient, rows, cols, values9)."""
        tets = np.ascontiguousarray(tets, np.uint32).reshape(-1, 4)
        x = np.ascontiguousarray(x, np.float64).reshape(-1)
        nt, nv = len(tets), len(x) // 3
        grad = np.zeros(3 * nv) if gradient is None else np.ascontiguousarray(gradient, np.float64).copy()
        rows, cols, vals = np.zeros(10 * nt, np.int32), np.zeros(10 * nt, np.int32), np.zeros((10 * nt, 9))
        a = [self._arg(tets, np.uint32), self._arg(x, np.float64), self._arg(dm_inverse, np.float64), self._arg(volume, np.float64),
             self._arg(len_rate, np.float64), self._arg(vol_rate, np.float64)]
        o = [self._arg(grad, np.float64, True), self._arg(rows, np.int32, True), self._arg(cols, np.int32, True),
             self._arg(vals, np.float64, True)]
        self._ck(self.lib.maspcg_fem_snk1_gradient_hessian(self.h, nt, a[0].ptr, nv, a[1].ptr, a[2].ptr, a[3].ptr,
                                                           a[4].ptr, a[5].ptr, float(dt), int(hessian_offset),
                                                           o[0].ptr, o[1].ptr, o[2].ptr, o[3].ptr))
        return grad, rows, cols, vals

    def bcoo_gradient(self, rows, cols, lam, x, out=None):
        """dL/d(values) of upper BCOO blocks for lam = A^-1 dL/dx (maspcg_bcoo_gradient)."""
        n = int(len(rows))
        r, c = self._arg(rows, np.int32), self._arg(cols, np.int32)
        la, xa = self._arg(lam, np.float64), self._arg(x, np.float64)
        if out is None:
            out = np.zeros((n, 9), np.float64)
        oa = self._arg(out, np.float64, writable=True)
        self._ck(self.lib.maspcg_bcoo_gradient(self.h, r.ptr, c.ptr, n, la.ptr, xa.ptr, oa.ptr))
        return out

    def residual_norms_noalloc(self, x, b):
        """FP64 ||b_j - A x_j|| and ||b_j|| for the rows of two CUDA float64
        tensors of shape (count, 3*nb) (or (3*nb,)), through the
        allocation-free entry point: nothing is staged or allocated."""
        if not (_is_torch(x) and _is_torch(b) and x.is_cuda and b.is_cuda):
            raise ValueError("x and b must be CUDA tensors")
        import torch
        for t in (x, b):
            if t.dtype != torch.float64 or not t.is_contiguous():
                raise ValueError("x and b must be contiguous float64")
        x2, b2 = x.reshape(-1, 3 * self.nb), b.reshape(-1, 3 * self.nb)
        if x2.shape != b2.shape:
            raise ValueError("x and b differ in shape")
        count = x2.shape[0]
        res = np.zeros(max(count, 1), np.float64)
        rhs = np.zeros(max(count, 1), np.float64)
        xa, ba = self._arg(x2, np.float64), self._arg(b2, np.float64)
        self._ck(self.lib.maspcg_residual_norms_noalloc(self.h, int(count), xa.ptr, ba.ptr,
                                                        res.ctypes.data_as(ctypes.c_void_p),
                                                        rhs.ctypes.data_as(ctypes.c_void_p)))
        return res[:count], rhs[:count]

    # -- introspection
    def info(self):
        i = N.Info()
        self._ck(self.lib.maspcg_get_info(self.h, ctypes.byref(i)))
        return {k: getattr(i, k) for k, _ in i._fields_}

    def hierarchy(self):
        i = self.info()
        L, nv = i["levelnum"], i["vert_num"]
        fm = np.zeros(nv, np.uint32)
        cst = np.zeros(L * nv, np.int32)
        gn = np.zeros(i["going_next_capacity"], np.int32)
        ls = np.zeros(2 * (L + 1), np.int32)
        ct = np.zeros(6 * nv, np.int32)
        po = np.zeros(i["part_map_size"] // self.cfg.bank_size, np.int32)
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        self._ck(self.lib.maspcg_get_hierarchy(self.h, p(fm), p(cst), p(gn), p(ls), p(ct), p(po)))
        return {"fine_mask": fm, "coarse_space_tables": cst.reshape(L, nv), "going_next": gn,
                "level_size": ls.reshape(L + 1, 2), "coarse_table": ct.reshape(nv, 6), "prefix_original": po,
                "total_clusters": i["total_clusters"], "levelnum": L}

    def bcsr(self):
        i = self.info()
        rp = np.zeros(i["internal_block_rows"] + 1, np.int32)
        ci = np.zeros(i["bcsr_blocks"], np.int32)
        vals = np.zeros((i["bcsr_blocks"], 9), np.float64)
        iof = np.zeros(self.nb, np.int32)
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        self._ck(self.lib.maspcg_get_bcsr(self.h, p(rp), p(ci), p(vals), p(iof)))
        return rp, ci, vals, iof

    def domain_inverses(self):
        d = self.info()["domains"]
        B = self.cfg.bank_size
        out = np.zeros((d, B * (B + 1) // 2, 9), np.float32)
        self._ck(self.lib.maspcg_get_domain_inverses(self.h, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def time_stage(self, stage: int, repeats: int = 20) -> float:
        """Mean device ms of one stage (0 SpMV, 1 preconditioner, 2 MAS level-0
        apply, 3 domain assembly + inversion, 4-6 level-0 apply variants, 7 the
        mixed solve's FP64 residual replacement) over `repeats` runs, each
        after an L2 eviction."""
        ms = ctypes.c_double()
        self._ck(self.lib.maspcg_time_stage(self.h, int(stage), int(repeats), ctypes.byref(ms)))
        return ms.value

    def domain_matrices(self):
        d = self.info()["domains"]
        B = self.cfg.bank_size
        out = np.zeros((d, B * (B + 1) // 2, 9), np.float64)
        self._ck(self.lib.maspcg_get_domain_matrices(self.h, out.ctypes.data_as(ctypes.c_void_p)))
        return out


# ------------------------------------------------------------ reference names


@dataclass
class PCGSolverConfig:
    """gipc::PCGSolverConfig (linear_system/solver/pcg_solver.h:7-17)."""

    max_iter_ratio: float = 0.3
    global_tol_rate: float = 1e-4
    use_bsr: bool = True


class PCGSolver:
    """gipc::PCGSolver over an assembled system: solve(x, b) -> iterations.

    ``system`` is anything with ``vals, rows, cols, nb, fem_offset, fem_count,
    abd_bodies`` and the MAS32 graph fields (``synth.System``)."""

    def __init__(self, cfg: PCGSolverConfig | None = None, *, preconditioner="mas32", **engine_cfg):
        self.cfg = cfg or PCGSolverConfig()
        self.preconditioner = preconditioner
        self.engine_cfg = engine_cfg
        self.engine: MasPcg | None = None
        self.last_result = None

    def bind(self, system):
        self.engine = MasPcg.from_system(system, tolerance=self.cfg.global_tol_rate,
                                         max_iter_ratio=self.cfg.max_iter_ratio, preconditioner=self.preconditioner,
                                         **self.engine_cfg)
        return self

    def solve(self, x, b) -> int:
        if self.engine is None:
            raise RuntimeError("bind(system) first")
        _, res = self.engine.solve(b, x)
        self.last_result = res
        return res["iterations"]


class TraditionalMAS32Preconditioner:
    """gpu_mas32::TraditionalMAS32Preconditioner (TraditionalMAS32Preconditioner.cuh:35-129).

    The caller sequence of gl_main.cu:1502-1536 works unchanged:
    initPreconditioner_Neighbor, fill the public arrays, initPreconditioner_Matrix,
    then per Newton step setPreconditioner_bcoo and preconditioning."""

    _PRECONDITIONER = "mas32"

    def __init__(self, **engine_cfg):
        self.engine_cfg = engine_cfg
        self.neighborListSize = 0
        self.d_neighborListInit = None
        self.d_neighborStart = None
        self.d_neighborNumInit = None
        self.d_partId_map_real = None
        self.d_real_map_partId = None
        self._engine: MasPcg | None = None

    def initPreconditioner_Neighbor(self, vertNum, mCollision_node_offset, totalNeighborNum, m_collisonPairs,
                                    partMapSize):
        self.totalNodes = int(vertNum)
        self.collision_node_Offset = int(mCollision_node_offset)
        self.totalNeighborNum = int(totalNeighborNum)
        self._collisonPairs = m_collisonPairs
        self.totalMapNodes = int(partMapSize)

    def initPreconditioner_Matrix(self):
        e = MasPcg(preconditioner=self._PRECONDITIONER, **self.engine_cfg)
        lst = np.asarray(self.d_neighborListInit)[: self.neighborListSize]
        e.set_graph(self.totalNodes, self.collision_node_Offset, self.d_neighborStart, self.d_neighborNumInit, lst,
                    np.asarray(self.d_partId_map_real)[: self.totalMapNodes], self.d_real_map_partId)
        self._engine = e

    def setPreconditioner_bcoo(self, triplet_values, row_ids, col_ids, indices, offset, triplet_num, cpNum):
        """The subsystem's triplets are gathered on the device by index
        (maspcg_set_matrix_bcoo_indexed), so the reference's device arrays
        (CUDA tensors here) are used where they are."""
        pairs = None if self._collisonPairs is None else np.asarray(self._collisonPairs).reshape(-1, 4)[:cpNum]
        self._engine.set_contacts(pairs)
        idx = indices[:triplet_num] if indices is not None else None
        vals = triplet_values.reshape(-1, 9) if hasattr(triplet_values, "reshape") else triplet_values
        self._engine.set_matrix_indexed(vals, row_ids, col_ids, idx, offset, self.totalNodes, 0, 0)
        self._engine.build()

    def refresh_fixed_graph_bcoo(self, values, rows, cols, indices, offset, count):
        """refresh_fixed_graph_bcoo (TraditionalMAS32Preconditioner.cu:229-234):
        new values on the unchanged graph, BCOO structure and contacts; the
        caller guarantees they are unchanged, as in the reference.  The values
        are gathered by the same indices as setPreconditioner_bcoo's."""
        vals = values.reshape(-1, 9) if hasattr(values, "reshape") else values
        if indices is None:
            self._engine.refresh_values(vals[:count])
        else:
            self._engine.refresh_values_indexed(vals, indices[:count])

    def local_diagnostics_gpu(self):
        """local_diagnostics_gpu (TraditionalMAS32Preconditioner.cu:182-183)."""
        return self._engine.local_diagnostics()

    def numerical_diagnostics(self, R=None):
        """The local part of numerical_diagnostics (:2727-2887): the per-domain
        SPD and inverse-residual summary (the per-level r.z sums of the last
        apply are not restated)."""
        return self._engine.local_diagnostics()

    def preconditioning(self, R, Z=None):
        return self._engine.apply_preconditioner(R, Z)

    def FreeMAS(self):
        if self._engine is not None:
            self._engine.close()
            self._engine = None


class MASPreconditioner(TraditionalMAS32Preconditioner):
    """MASPreconditioner, CEMAS16 (MASPreconditioner.cuh; MASPreconditioner.cu:
    2209-2364): the same caller sequence (initPreconditioner_Neighbor,
    initPreconditioner_Matrix, setPreconditioner_bcoo, preconditioning,
    FreeMAS) with d_partId_map_real in 16-slot banks."""

    _PRECONDITIONER = "cemas16"
