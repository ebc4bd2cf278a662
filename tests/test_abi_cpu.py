"""C-ABI checks that need no GPU: the library loads, exports every function
include/maspcg.h declares, and fails cleanly without a device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "maspcg.h")).read()
    return sorted(set(re.findall(r"MASPCG_API\s+[\w\s\*]+?\b(maspcg_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from agipc_learning_b200 import build, _native
    build.build_cuda()
    return _native.load()


def test_every_declared_symbol_is_exported(lib):
    from agipc_learning_b200 import _native
    declared = _declared()
    assert len(declared) >= 30
    assert sorted(_native.EXPORTS) == declared
    for name in declared:
        assert hasattr(lib, name), name


def test_config_defaults_match_pcg_solver_config(lib):
    from agipc_learning_b200 import _native as N
    cfg = N.Config()
    lib.maspcg_config_default(ctypes.byref(cfg))
    assert cfg.tolerance == 1e-4 and cfg.max_iter_ratio == 0.3      # pcg_solver.h:7-17
    assert cfg.preconditioner == N.PRECOND_MAS32 and cfg.bank_size == 32
    assert cfg.gate == N.GATE_RZ and cfg.precision == N.PREC_REFERENCE


def test_null_handle_and_status_strings(lib):
    from agipc_learning_b200 import _native as N
    assert lib.maspcg_destroy(None) == N.ERR_NULL_HANDLE
    assert lib.maspcg_build_preconditioner(None) == N.ERR_NULL_HANDLE
    assert lib.maspcg_solve(None, None, None, None) == N.ERR_NULL_HANDLE
    assert lib.maspcg_status_string(N.ERR_CAPACITY) == b"capacity exceeded"


def test_create_rejects_bad_config(lib):
    from agipc_learning_b200 import _native as N
    cfg = N.Config()
    lib.maspcg_config_default(ctypes.byref(cfg))
    cfg.bank_size = 16  # MAS32 with a 16-vertex bank
    h = ctypes.c_void_p()
    assert lib.maspcg_create(ctypes.byref(cfg), ctypes.byref(h)) == N.ERR_UNSUPPORTED
    assert b"32-vertex" in lib.maspcg_last_error(None)
    cfg.bank_size = 24
    assert lib.maspcg_create(ctypes.byref(cfg), ctypes.byref(h)) == N.ERR_UNSUPPORTED
    cfg.preconditioner, cfg.bank_size = N.PRECOND_MAS16, 32  # CEMAS16 with a 32-vertex bank
    assert lib.maspcg_create(ctypes.byref(cfg), ctypes.byref(h)) == N.ERR_UNSUPPORTED
    assert b"16-vertex" in lib.maspcg_last_error(None)
    cfg.bank_size, cfg.inverse_storage = 16, N.INV_BF16  # CEMAS16 stores FP32 inverses
    assert lib.maspcg_create(ctypes.byref(cfg), ctypes.byref(h)) == N.ERR_UNSUPPORTED
    assert b"FP32" in lib.maspcg_last_error(None)


def test_create_without_device_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from agipc_learning_b200 import _native as N
    h = ctypes.c_void_p()
    assert lib.maspcg_create(None, ctypes.byref(h)) == N.ERR_NO_DEVICE
    assert not h.value
