"""C-ABI library checks that need no GPU: it loads, exports every symbol the
public header declares, and reports a clean error (not a crash) when no CUDA
device is present."""
import ctypes as C
import os
import subprocess

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


def test_struct_layouts_match_header(tmp_path):
    """Every ctypes struct has the size and field offsets that a C compiler gives
    the header's struct."""
    structs = {"ps_desc": _capi.PsDesc, "ps_ksp_opts": _capi.PsKspOpts, "ps_ksp_result": _capi.PsKspResult,
               "ps_sqrt_opts": _capi.PsSqrtOpts, "ps_sqrt_result": _capi.PsSqrtResult,
               "ps_step_inputs": _capi.PsStepInputs, "ps_step_result": _capi.PsStepResult,
               "ps_obs_out": _capi.PsObsOut}
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{os.path.abspath(_capi.HEADER)}"',
             "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln.strip():
            parts = ln.split()
            got[(parts[0], parts[1])] = int(parts[2])
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_bad_arguments_rejected_without_gpu():
    L = _capi.lib()
    out = C.c_void_p()
    assert L.ps_ctx_create(None, 0, 0, C.byref(out)) < 0
    assert L.ps_matmult(None, None, None, None) < 0
    assert L.ps_ksp_solve(None, None, None, None, None, None) < 0
    assert L.ps_last_error() is not None
