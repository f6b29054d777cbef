"""ctypes front end of the CPU oracle (oracle/psoracle.c).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()``
and by the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``, where it
is the checker or the timed CPU restatement.  The product path
(``polystokes_brownian_b200``) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libpsoracle.so")
_lib = None

AB_REFERENCE = 0
AB_RPY = 1
AB_RPY_REG = 2


class OrParams(C.Structure):
    _fields_ = [
        ("Nm", C.c_int), ("Nc", C.c_int), ("Npoly", C.c_int), ("Nmono_per_chain", C.c_int),
        ("beta", C.c_double), ("kT", C.c_double), ("epsilon", C.c_double), ("kbond", C.c_double),
        ("r0", C.c_double), ("Lmax", C.c_double), ("tau", C.c_double),
        ("dt", C.c_double),
        ("mm_HI", C.c_int), ("chain_HI", C.c_int), ("fene", C.c_int), ("tether", C.c_int),
        ("mono_ev", C.c_int), ("record_forces", C.c_int),
        ("box_on", C.c_int), ("box", C.c_double * 3),
        ("ktrap", C.c_double), ("tstart", C.c_double), ("trun", C.c_double), ("weaken_trap", C.c_double),
        ("t0", C.c_double), ("restart", C.c_int), ("ab_mode", C.c_int),
        ("hs_kpref", C.c_double), ("hs_kmode", C.c_int), ("lanczos_nc", C.c_int),
        ("lub_on", C.c_int), ("lub_gap", C.c_double), ("noise_lanczos", C.c_int), ("aa_mode", C.c_int),
        ("lub_bonded", C.c_int),
    ]


class OrStepOut(C.Structure):
    _fields_ = [(k, C.POINTER(C.c_double)) for k in
                ("v_det_n", "v_det_c", "v_brown", "up", "udiff", "sb", "fext")] + \
               [("iters", C.c_int * 5)]


def build() -> str:
    """Compile the oracle shared library (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.POINTER(C.c_double)
        I = C.POINTER(C.c_int)
        L.or_create.restype = C.c_void_p
        L.or_create.argtypes = [C.POINTER(OrParams)]
        L.or_destroy.argtypes = [C.c_void_p]
        L.or_set_state.argtypes = [C.c_void_p, P, P]
        L.or_get_state.argtypes = [C.c_void_p, P, P]
        L.or_set_time.argtypes = [C.c_void_p, C.c_double]
        L.or_get_time.restype = C.c_double
        L.or_get_time.argtypes = [C.c_void_p]
        L.or_sizes.argtypes = [C.c_void_p, I]
        L.or_set_lub_tables.argtypes = [C.c_void_p, P, C.c_int, C.c_int]
        L.or_tensor_aa.argtypes = [C.c_double, C.c_double, P, C.c_double, C.c_int, P]
        L.or_tensor_ab_rpy.argtypes = [C.c_double, C.c_double, P, C.c_double, C.c_int, P]
        L.or_tensor_ab.argtypes = [C.c_double, C.c_double, P, C.c_double, C.c_int, P, P]
        L.or_ab_reg_scalars.argtypes = [C.c_double, C.c_double, P, P, P]
        L.or_tensor_bb.argtypes = [C.c_double, C.c_double, P, P, P, P, P, P, P]
        for f in ("or_check_dist", "or_mob", "or_schur_sync"):
            getattr(L, f).argtypes = [C.c_void_p]
        L.or_verlet_pairs.argtypes = [C.c_void_p, I, I, C.c_int]
        L.or_cell_pairs.argtypes = [C.c_void_p, I, I, C.c_int]
        L.or_lub_pairs.argtypes = [C.c_void_p, I, I, C.c_int]
        L.or_rhs.argtypes = [C.c_void_p, C.c_int, P, P]
        L.or_stale_a.argtypes = [C.c_void_p, P]
        for f in ("or_dense_mobility", "or_saddle_diag", "or_mcm", "or_mcc"):
            getattr(L, f).argtypes = [C.c_void_p, P]
        for f in ("or_mobility_apply", "or_saddle_apply", "or_slip_noise", "or_lub_apply"):
            getattr(L, f).argtypes = [C.c_void_p, P, P]
        L.or_minres.argtypes = [C.c_void_p, P, P, C.c_int, C.c_double, C.c_int, I, P]
        L.or_sqrtm_eig.argtypes = [P, C.c_int, P, P]
        L.or_lanczos_sqrt.argtypes = [C.c_void_p, P, P, C.c_int, C.c_double]
        L.or_jacobi_eig.argtypes = [P, C.c_int, P, P]
        L.or_step.argtypes = [C.c_void_p, P, P, P, C.c_double, C.POINTER(OrStepOut)]
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_int))


def default_params(**kw) -> OrParams:
    p = OrParams()
    d = dict(Nm=0, Nc=0, Npoly=0, Nmono_per_chain=1, beta=1.0, kT=0.0, epsilon=1.0, kbond=1.0,
             r0=1.0, Lmax=10.0, tau=1000.0, dt=1e-3, mm_HI=1, chain_HI=0, fene=0, tether=0,
             mono_ev=0, record_forces=1, box_on=0, ktrap=0.0, tstart=0.0, trun=0.0,
             weaken_trap=-1.0, t0=0.0, restart=0, ab_mode=AB_REFERENCE, hs_kpref=1.0,
             hs_kmode=0, lanczos_nc=64, lub_on=0, lub_gap=0.5, noise_lanczos=0, aa_mode=0,
             lub_bonded=0)
    box = kw.pop("box", None)
    d.update({k: v for k, v in kw.items() if k in d})
    for k, v in d.items():
        setattr(p, k, v)
    if box is not None:
        p.box_on = 1
        for i in range(3):
            p.box[i] = float(box[i])
    return p


class OracleSim:
    """One PolyStokes system held by the oracle."""

    def __init__(self, params: OrParams, x: np.ndarray, q: np.ndarray | None = None,
                 lub_table: np.ndarray | None = None):
        self.L = lib()
        self.p = params
        self.h = self.L.or_create(C.byref(params))
        sz = (C.c_int * 8)()
        self.L.or_sizes(self.h, sz)
        (self.nm3, self.nc11, self.nm3nc6, self.nm3nc11, self.n, self.Np, self.nc5, self.n3) = list(sz)
        if lub_table is not None:
            t = np.ascontiguousarray(lub_table, dtype=np.float64)
            self.L.or_set_lub_tables(self.h, _p(t), t.shape[0], t.shape[1])
        self.set_state(x, q)

    def __del__(self):
        try:
            if self.h:
                self.L.or_destroy(self.h)
                self.h = None
        except Exception:
            pass

    # state ---------------------------------------------------------------
    def set_state(self, x, q=None):
        x = np.ascontiguousarray(x, dtype=np.float64).ravel()
        qq = None if q is None else np.ascontiguousarray(q, dtype=np.float64).ravel()
        self.L.or_set_state(self.h, _p(x), _p(qq))

    def state(self):
        x = np.zeros(self.n3)
        q = np.zeros(max(4 * self.p.Nc, 1))
        self.L.or_get_state(self.h, _p(x), _p(q))
        return x, q[: 4 * self.p.Nc]

    @property
    def t(self):
        return self.L.or_get_time(self.h)

    @t.setter
    def t(self, v):
        self.L.or_set_time(self.h, float(v))

    # stage ---------------------------------------------------------------
    def stage(self):
        """check_dist + RHS + mob + Schur sync; returns the rhs vector."""
        self.L.or_check_dist(self.h)
        rhs = np.zeros(self.n)
        self.L.or_rhs(self.h, 0, None, _p(rhs))
        self.L.or_mob(self.h)
        self.L.or_schur_sync(self.h)
        return rhs

    def check_dist(self):
        self.L.or_check_dist(self.h)

    def mob(self):
        self.L.or_mob(self.h)

    def rhs(self, drift=False, fext=None):
        r = np.zeros(self.n)
        f = None if fext is None else np.ascontiguousarray(fext, dtype=np.float64)
        self.L.or_rhs(self.h, int(drift), _p(f), _p(r))
        return r

    def verlet_pairs(self):
        n = self.L.or_verlet_pairs(self.h, None, None, 0)
        a = np.zeros(max(n, 1), np.int32)
        b = np.zeros(max(n, 1), np.int32)
        self.L.or_verlet_pairs(self.h, _ip(a), _ip(b), n)
        return a[:n], b[:n]

    def cell_pairs(self):
        n = self.L.or_cell_pairs(self.h, None, None, 0)
        a = np.zeros(max(n, 1), np.int32)
        b = np.zeros(max(n, 1), np.int32)
        self.L.or_cell_pairs(self.h, _ip(a), _ip(b), n)
        return a[:n], b[:n]

    def lub_pairs(self):
        n = self.L.or_lub_pairs(self.h, None, None, 0)
        a = np.zeros(max(n, 1), np.int32)
        b = np.zeros(max(n, 1), np.int32)
        self.L.or_lub_pairs(self.h, _ip(a), _ip(b), n)
        return a[:n], b[:n]

    def stale_a(self):
        t = np.zeros(9)
        self.L.or_stale_a(self.h, _p(t))
        return t.reshape(3, 3)

    # operators -----------------------------------------------------------
    def dense_mobility(self):
        M = np.zeros((self.nm3nc11, self.nm3nc11))
        self.L.or_dense_mobility(self.h, _p(M))
        return M

    def mobility_apply(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        y = np.zeros(self.nm3nc11)
        self.L.or_mobility_apply(self.h, _p(u), _p(y))
        return y

    def saddle_apply(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.n)
        self.L.or_saddle_apply(self.h, _p(x), _p(y))
        return y

    def saddle_diag(self):
        d = np.zeros(self.n)
        self.L.or_saddle_diag(self.h, _p(d))
        return d

    def lub_apply(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        y = np.zeros(self.nm3nc6)
        self.L.or_lub_apply(self.h, _p(u), _p(y))
        return y

    def mcm(self):
        M = np.zeros((self.nc11, self.nm3))
        self.L.or_mcm(self.h, _p(M))
        return M

    def mcc(self):
        M = np.zeros((self.nc11, self.nc11))
        self.L.or_mcc(self.h, _p(M))
        return M

    def minres(self, b, x0=None, rtol=1e-8, maxit=100000):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        it = C.c_int(0)
        rn = C.c_double(0)
        reason = self.L.or_minres(self.h, _p(b), _p(x), int(x0 is not None), rtol, maxit,
                                  C.byref(it), C.byref(rn))
        return x, reason, it.value, rn.value

    def slip_noise(self, fb):
        fb = np.ascontiguousarray(fb, dtype=np.float64)
        W = np.zeros(self.nm3nc11)
        self.L.or_slip_noise(self.h, _p(fb), _p(W))
        return W

    def lanczos_sqrt(self, z, kmax=60, tol=1e-12):
        z = np.ascontiguousarray(z, dtype=np.float64)
        w = np.zeros(self.nm3nc11)
        m = self.L.or_lanczos_sqrt(self.h, _p(z), _p(w), kmax, tol)
        return w, m

    def step(self, fb=None, wrfd=None, zlub=None, rtol=1e-8):
        n6 = self.nm3nc6
        fb = np.zeros(self.nm3nc11) if fb is None else np.ascontiguousarray(fb, dtype=np.float64)
        wr = np.zeros(n6) if wrfd is None else np.ascontiguousarray(wrfd, dtype=np.float64)
        zl = None if zlub is None else np.ascontiguousarray(zlub, dtype=np.float64)
        out = {k: np.zeros(n6) for k in ("v_det_n", "v_det_c", "v_brown", "up", "udiff", "fext")}
        out["sb"] = np.zeros(max(self.nc5, 1))
        so = OrStepOut()
        for k, v in out.items():
            setattr(so, k, _p(v))
        self.L.or_step(self.h, _p(fb), _p(wr), _p(zl), rtol, C.byref(so))
        out["iters"] = list(so.iters)
        out["sb"] = out["sb"][: self.nc5]
        return out


def sqrtm_eig(M, z):
    M = np.ascontiguousarray(M, dtype=np.float64)
    z = np.ascontiguousarray(z, dtype=np.float64)
    w = np.zeros_like(z)
    lib().or_sqrtm_eig(_p(M), M.shape[0], _p(z), _p(w))
    return w


def tensor_bb(e, r):
    e = np.ascontiguousarray(e, dtype=np.float64)
    outs = [np.zeros(k) for k in (9, 9, 9, 15, 15, 25)]
    lib().or_tensor_bb(r, 1.0 / r, _p(e), *[_p(o) for o in outs])
    return outs


def tensor_ab(e, r, beta, reg=0):
    e = np.ascontiguousarray(e, dtype=np.float64)
    b = np.zeros(9)
    g = np.zeros(15)
    lib().or_tensor_ab(r, 1.0 / r, _p(e), beta, reg, _p(b), _p(g))
    return b, g


def tensor_aa(e, r, beta, mode=0):
    e = np.ascontiguousarray(e, dtype=np.float64)
    a = np.zeros(9)
    lib().or_tensor_aa(r, 1.0 / r, _p(e), beta, mode, _p(a))
    return a


def tensor_ab_rpy(e, r, beta, reg=0):
    e = np.ascontiguousarray(e, dtype=np.float64)
    a = np.zeros(9)
    lib().or_tensor_ab_rpy(r, 1.0 / r, _p(e), beta, reg, _p(a))
    return a


def ab_reg_scalars(r, beta):
    out = [np.zeros(1) for _ in range(3)]
    lib().or_ab_reg_scalars(r, beta, *[_p(o) for o in out])
    return tuple(float(o[0]) for o in out)
