"""ctypes binding of the C-ABI in include/polystokes_b200.h.

The shared library is built in-tree (polystokes_brownian_b200/_lib/libpsb200.so,
``python -m polystokes_brownian_b200.build``).  There is no CPU fallback: if
the library is missing or cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libpsb200.so")
HEADER = os.path.join(HERE, "..", "include", "polystokes_b200.h")

PS_OK = 0
PS_AB_REFERENCE = 0
PS_AB_RPY = 1
PS_AA_REFERENCE = 0
PS_AA_RPY = 1
PS_PREC_FP64 = 0
PS_PREC_MIXED = 1
PS_SOLVE_MINRES = 0
PS_SOLVE_STRUCTURED = 1


class PsDesc(C.Structure):
    _fields_ = [
        ("Nm", C.c_int32), ("Nc", C.c_int32), ("Npoly", C.c_int32), ("Nmono_per_chain", C.c_int32),
        ("beta", C.c_double), ("kT", C.c_double), ("epsilon", C.c_double), ("kbond", C.c_double),
        ("r0", C.c_double), ("Lmax", C.c_double), ("tau", C.c_double),
        ("dt", C.c_double),
        ("mm_HI", C.c_int32), ("chain_HI", C.c_int32), ("fene", C.c_int32), ("tether", C.c_int32),
        ("mono_ev", C.c_int32), ("record_forces", C.c_int32),
        ("box_on", C.c_int32), ("box", C.c_double * 3),
        ("ktrap", C.c_double), ("tstart", C.c_double), ("trun", C.c_double), ("weaken_trap", C.c_double),
        ("t0", C.c_double), ("restart", C.c_int32), ("ab_mode", C.c_int32),
        ("hs_kpref", C.c_double), ("hs_kmode", C.c_int32), ("lanczos_nc", C.c_int32),
        ("lub_on", C.c_int32), ("lub_gap", C.c_double), ("aa_mode", C.c_int32), ("lub_bonded", C.c_int32),
    ]


class PsKspOpts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("maxit", C.c_int32), ("warm", C.c_int32), ("check_every", C.c_int32),
                ("method", C.c_int32)]


class PsKspResult(C.Structure):
    _fields_ = [("reason", C.c_int32), ("iters_max", C.c_int32), ("iters_sum", C.c_int64),
                ("rnorm_max", C.c_double)]


class PsSqrtOpts(C.Structure):
    _fields_ = [("kmax", C.c_int32), ("tol", C.c_double)]


class PsSqrtResult(C.Structure):
    _fields_ = [("iters_max", C.c_int32), ("nneg", C.c_int32)]


class PsStepInputs(C.Structure):
    _fields_ = [("fb", C.c_void_p), ("wrfd", C.c_void_p), ("zlub", C.c_void_p),
                ("rtol", C.c_double), ("maxit", C.c_int32), ("sqrt_kmax", C.c_int32), ("sqrt_tol", C.c_double),
                ("solver", C.c_int32), ("refine", C.c_int32)]


class PsStepResult(C.Structure):
    _fields_ = [("iters", C.c_int32 * 5), ("reason", C.c_int32), ("lanczos_iters", C.c_int32),
                ("lanczos_nneg", C.c_int32)]


class PsObsOut(C.Structure):
    _fields_ = [("bond", C.c_void_p), ("bond_hist", C.c_void_p), ("trap", C.c_void_p), ("trap_hist", C.c_void_p),
                ("msd", C.c_void_p), ("msd_count", C.c_void_p)]


def declared_symbols(header: str = HEADER) -> list[str]:
    """Names of every function the public header declares."""
    txt = open(header).read()
    return sorted(set(re.findall(r"^\s*(?:int|uint64_t|const char \*|void)\s*\*?\s*(ps_\w+)\s*\(", txt, re.M)))


_lib = None


def lib():
    """Load the engine library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"B200 engine library not built: {LIB_PATH} "
                           "(run `python -m polystokes_brownian_b200.build`)")
    L = C.CDLL(LIB_PATH)
    vp, P = C.c_void_p, C.c_void_p
    I64P = C.POINTER(C.c_int64)
    L.ps_last_error.restype = C.c_char_p
    L.ps_ctx_create.argtypes = [C.POINTER(PsDesc), C.c_int32, C.c_int32, C.POINTER(vp)]
    L.ps_ctx_destroy.argtypes = [vp]
    L.ps_ctx_sizes.argtypes = [vp, I64P]
    L.ps_ctx_offsets.argtypes = [vp, C.c_int32, I64P]
    L.ps_set_lub_table.argtypes = [vp, P, C.c_int32, C.c_int32]
    L.ps_set_seed.argtypes = [vp, C.c_uint64]
    L.ps_set_replica_seeds.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.ps_get_replica_steps.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.ps_get_aux.argtypes = [vp, P, P, P, vp]
    L.ps_autotune.argtypes = [vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double), vp]
    L.ps_obs_reset.argtypes = [vp, C.c_int32, C.c_double, C.c_double, C.c_int32]
    L.ps_observe.argtypes = [vp, vp]
    L.ps_obs_read.argtypes = [vp, C.POINTER(PsObsOut), vp]
    L.ps_set_aux.argtypes = [vp, P, P, P, vp]
    L.ps_set_state.argtypes = [vp, P, P, vp]
    L.ps_get_state.argtypes = [vp, P, P, vp]
    L.ps_set_time.argtypes = [vp, C.c_double]
    L.ps_build_pairs.argtypes = [vp, vp]
    L.ps_pair_list.argtypes = [vp, C.c_int32, P, P, C.c_int64, I64P, vp]
    L.ps_rhs.argtypes = [vp, C.c_int32, P, P, vp]
    L.ps_assemble.argtypes = [vp, vp]
    L.ps_matmult.argtypes = [vp, P, P, vp]
    L.ps_mobility_apply.argtypes = [vp, P, P, vp]
    L.ps_get_diagonal.argtypes = [vp, P, vp]
    L.ps_ksp_solve.argtypes = [vp, P, P, C.POINTER(PsKspOpts), C.POINTER(PsKspResult), vp]
    L.ps_sqrtm_apply.argtypes = [vp, P, P, C.POINTER(PsSqrtOpts), C.POINTER(PsSqrtResult), vp]
    L.ps_step.argtypes = [vp, C.POINTER(PsStepInputs), C.POINTER(PsStepResult), vp]
    L.ps_step_outputs.argtypes = [vp, P, P, P, P, vp]
    L.ps_time_kernel.argtypes = [vp, C.c_int32, C.c_int32, P, C.POINTER(C.c_double), vp]
    L.ps_fma_peak.argtypes = [C.c_int32, C.POINTER(C.c_double), vp]
    L.ps_kernel_launches.restype = C.c_uint64
    L.ps_mobility_apply_noalloc.argtypes = [P, P, P, C.c_int32, C.c_double, C.c_int32, C.c_int32, vp]
    _lib = L
    return L


def check(rc: int, what: str = "") -> int:
    if rc < 0:
        msg = lib().ps_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed ({rc}): {msg}")
    return rc
