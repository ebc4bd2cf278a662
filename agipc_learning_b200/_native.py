"""ctypes binding of ``libmaspcg.so`` (the C ABI in ``include/maspcg.h``).

The library is built in-tree by ``agipc_learning_b200.build``.  There is no
fallback: if the library is missing every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmaspcg.so")

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_NULL_HANDLE = 2
ERR_CUDA = 3
ERR_OUT_OF_MEMORY = 4
ERR_NOT_READY = 5
ERR_CAPACITY = 6
ERR_NO_DEVICE = 7
ERR_UNSUPPORTED = 8

PRECOND_BLOCK_JACOBI = 0
PRECOND_MAS16 = 1
PRECOND_MAS32 = 2
PRECOND_NONE = 3

PREC_REFERENCE = 0
PREC_FP32 = 1
PREC_MIXED = 2

GATE_RZ = 0
GATE_EUCLID = 1

FLAG_PDL = 1
FLAG_APPLY_STAGED2 = 2
FLAG_APPLY_DIRECT = 4
FLAG_SEQUENTIAL_COARSE = 8
FLAG_FUSED_HEAD = 16
FLAG_FUSED_UPDATE = 32
FLAG_HOST_LOOP = 64

INV_FP32 = 0
INV_BF16 = 1
INV_FP16 = 2
MATRIX_F32 = 0
MATRIX_F32_ACCURATE = 1
MATRIX_F32_SPLIT = 2
MATRIX_F32_COMPENSATED = 3
REPLACE_PERIODIC = 0
REPLACE_RELIABLE = 1

SOLVE_STATUS = {0: "running", 1: "converged", 2: "iteration_cap", 3: "nonpositive_curvature", 4: "nonfinite",
                5: "invalid_rz"}

# every function declared in include/maspcg.h
EXPORTS = (
    "maspcg_config_default", "maspcg_status_string", "maspcg_last_error", "maspcg_create", "maspcg_destroy",
    "maspcg_set_stream", "maspcg_get_stream", "maspcg_set_graph", "maspcg_set_contacts", "maspcg_set_matrix_bcoo",
    "maspcg_build_preconditioner", "maspcg_solve", "maspcg_apply_preconditioner", "maspcg_spmv", "maspcg_get_info",
    "maspcg_get_hierarchy", "maspcg_get_bcsr", "maspcg_get_domain_inverses", "maspcg_get_domain_matrices",
    "maspcg_time_stage", "maspcg_residual_norms_noalloc", "maspcg_bcoo_gradient", "maspcg_convert_bcoo",
    "maspcg_partition_contact_triplets", "maspcg_fem_snk1_gradient_hessian", "maspcg_galerkin_coarse_matrix",
    "maspcg_galerkin_restrict", "maspcg_galerkin_prolong", "maspcg_adjust_contact_triplets",
    "maspcg_zero_boundary_triplets", "maspcg_spmv_working", "maspcg_refresh_matrix_values",
    "maspcg_set_matrix_bcoo_indexed", "maspcg_local_diagnostics", "maspcg_check_local_matrices",
    "maspcg_refresh_matrix_values_indexed", "maspcg_set_wait_test_hooks", "maspcg_element_modulus_gradient",
)

RESIDUAL_MAX_VECTORS = 8


class GalerkinMap(ctypes.Structure):
    """maspcg_galerkin_map: the AGIPC coarse mapping."""
    _fields_ = [("fine_to_coarse", ctypes.c_void_p), ("coarse_block_bases", ctypes.c_void_p),
                ("basis_masks", ctypes.c_void_p), ("rest_positions", ctypes.c_void_p),
                ("prefix_blocks", ctypes.c_int), ("fem_nodes", ctypes.c_int), ("coarse_nodes", ctypes.c_int),
                ("coarse_block_nodes", ctypes.c_int)]


class Config(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("max_iter_ratio", ctypes.c_double), ("max_iterations", ctypes.c_int),
                ("gate", ctypes.c_int), ("precision", ctypes.c_int), ("inverse_storage", ctypes.c_int),
                ("preconditioner", ctypes.c_int), ("refinement_period", ctypes.c_int), ("bank_size", ctypes.c_int),
                ("iterations_per_launch", ctypes.c_int), ("flags", ctypes.c_int), ("matrix_form", ctypes.c_int),
                ("residual_replacement", ctypes.c_int)]


class Result(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("status", ctypes.c_int), ("refinements", ctypes.c_int),
                ("launches", ctypes.c_int), ("rz0", ctypes.c_double), ("rz_final", ctypes.c_double),
                ("rel_res_recursive", ctypes.c_double), ("rel_res_true", ctypes.c_double),
                ("solve_ms", ctypes.c_double), ("fp64_gate_met", ctypes.c_int)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["status_name"] = SOLVE_STATUS.get(self.status, str(self.status))
        return d


class DomainCheck(ctypes.Structure):
    """maspcg_domain_check (LocalGpuCheck)."""
    _fields_ = [("local_finite", ctypes.c_int), ("inverse_finite", ctypes.c_int), ("local_spd", ctypes.c_int),
                ("inverse_spd", ctypes.c_int), ("minimum_local_diagonal", ctypes.c_double),
                ("minimum_inverse_diagonal", ctypes.c_double), ("inverse_residual", ctypes.c_double)]


class Diagnostics(ctypes.Structure):
    """maspcg_diagnostics (the summary of gpu_local_checks)."""
    _fields_ = [("matrix_count", ctypes.c_int), ("local_spd_count", ctypes.c_int),
                ("inverse_spd_count", ctypes.c_int), ("first_local_spd_failure", ctypes.c_int),
                ("first_inverse_spd_failure", ctypes.c_int), ("nonfinite_local_count", ctypes.c_int),
                ("nonfinite_inverse_count", ctypes.c_int), ("passed", ctypes.c_int),
                ("minimum_local_diagonal", ctypes.c_double), ("minimum_inverse_diagonal", ctypes.c_double),
                ("maximum_inverse_residual", ctypes.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["passed"] = bool(d["passed"])
        return d


class Info(ctypes.Structure):
    _fields_ = [("levelnum", ctypes.c_int), ("total_clusters", ctypes.c_int), ("domains", ctypes.c_int),
                ("vert_num", ctypes.c_int), ("part_map_size", ctypes.c_int),
                ("going_next_capacity", ctypes.c_longlong), ("internal_block_rows", ctypes.c_int),
                ("bcsr_blocks", ctypes.c_int), ("failed_domains", ctypes.c_int),
                ("kernel_launches", ctypes.c_longlong), ("graph_captures", ctypes.c_longlong)]


_LIB = None


def load():
    """Load libmaspcg.so; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: the CUDA extension must be built "
                           "(agipc_learning_b200.build.build_all()); there is no CPU fallback")
    lib = ctypes.CDLL(LIB_PATH)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    H = ctypes.c_void_p
    sig = {
        "maspcg_config_default": (None, [ctypes.POINTER(Config)]),
        "maspcg_status_string": (ctypes.c_char_p, [I]),
        "maspcg_last_error": (ctypes.c_char_p, [H]),
        "maspcg_create": (I, [ctypes.POINTER(Config), ctypes.POINTER(H)]),
        "maspcg_destroy": (I, [H]),
        "maspcg_set_stream": (I, [H, P]),
        "maspcg_get_stream": (I, [H, ctypes.POINTER(ctypes.c_void_p)]),
        "maspcg_set_graph": (I, [H, I, I, P, P, P, I, P, I, P]),
        "maspcg_set_contacts": (I, [H, P, I]),
        "maspcg_set_matrix_bcoo": (I, [H, P, P, P, I, I, I, I]),
        "maspcg_build_preconditioner": (I, [H]),
        "maspcg_solve": (I, [H, P, P, ctypes.POINTER(Result)]),
        "maspcg_apply_preconditioner": (I, [H, P, P]),
        "maspcg_spmv": (I, [H, D, P, D, P]),
        "maspcg_get_info": (I, [H, ctypes.POINTER(Info)]),
        "maspcg_get_hierarchy": (I, [H, P, P, P, P, P, P]),
        "maspcg_get_bcsr": (I, [H, P, P, P, P]),
        "maspcg_get_domain_inverses": (I, [H, P]),
        "maspcg_get_domain_matrices": (I, [H, P]),
        "maspcg_time_stage": (I, [H, I, I, ctypes.POINTER(ctypes.c_double)]),
        "maspcg_residual_norms_noalloc": (I, [H, I, P, P, P, P]),
        "maspcg_bcoo_gradient": (I, [H, P, P, I, P, P, P]),
        "maspcg_convert_bcoo": (I, [H, P, P, P, I, P, P, P, P]),
        "maspcg_partition_contact_triplets": (I, [H, P, P, P, P, I, P, P, P, P]),
        "maspcg_fem_snk1_gradient_hessian": (I, [H, I, P, I, P, P, P, P, P, D, I, P, P, P, P]),
        "maspcg_galerkin_coarse_matrix": (I, [H, ctypes.POINTER(GalerkinMap), P, P, P, I, P, P, P, I, P]),
        "maspcg_galerkin_restrict": (I, [H, ctypes.POINTER(GalerkinMap), P, P]),
        "maspcg_galerkin_prolong": (I, [H, ctypes.POINTER(GalerkinMap), P, P]),
        "maspcg_adjust_contact_triplets": (I, [H, I, P, P, P, P, I, I]),
        "maspcg_zero_boundary_triplets": (I, [H, I, P, P, P, P, I, I]),
        "maspcg_spmv_working": (I, [H, P, P]),
        "maspcg_refresh_matrix_values": (I, [H, P]),
        "maspcg_refresh_matrix_values_indexed": (I, [H, P, ctypes.c_longlong, P]),
        "maspcg_set_wait_test_hooks": (I, [H, ctypes.c_longlong, I]),
        "maspcg_element_modulus_gradient": (I, [H, I, I, P, P, P, P, P, P, P]),
        "maspcg_set_matrix_bcoo_indexed": (I, [H, P, P, P, ctypes.c_longlong, P, I, I, I, I, I]),
        "maspcg_local_diagnostics": (I, [H, P, ctypes.POINTER(Diagnostics)]),
        "maspcg_check_local_matrices": (I, [H, I, I, P, P, P, ctypes.POINTER(Diagnostics)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


class MaspcgError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"maspcg status {status}: {message}")
        self.status = status


def check(status: int, handle=None):
    if status != OK:
        lib = load()
        msg = lib.maspcg_last_error(handle)
        raise MaspcgError(status, (msg or b"").decode() or lib.maspcg_status_string(status).decode())
