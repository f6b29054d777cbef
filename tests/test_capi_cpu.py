"""C-ABI library checks that need no GPU: it loads, exports every symbol the
public header declares, and reports a clean error (not a crash) when no CUDA
device is present."""
import ctypes as C
import os

import pytest

from polystokes_brownian_b200 import _capi


def test_library_built_and_loads():
    assert os.path.exists(_capi.LIB_PATH), "run python -m polystokes_brownian_b200.build"
    C.CDLL(_capi.LIB_PATH)


def test_exports_every_declared_symbol():
    names = _capi.declared_symbols()
    assert len(names) >= 20
    L = C.CDLL(_capi.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_layouts_match_header():
    # ps_desc must match the C layout field by field (sizes checked against the header)
    assert C.sizeof(_capi.PsDesc) % 8 == 0
    assert C.sizeof(_capi.PsKspResult) == 24
    assert C.sizeof(_capi.PsStepResult) == 24


def test_bad_arguments_rejected_without_gpu():
    L = _capi.lib()
    out = C.c_void_p()
    assert L.ps_ctx_create(None, 0, 0, C.byref(out)) < 0
    assert L.ps_matmult(None, None, None, None) < 0
    assert L.ps_ksp_solve(None, None, None, None, None, None) < 0
    assert L.ps_last_error() is not None
