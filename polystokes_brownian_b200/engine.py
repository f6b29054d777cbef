"""Python front end of the C-ABI: one context over a batch of systems, with
device buffers held in torch tensors (plumbing only -- every operation below
is a call into the CUDA library)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi
from ._capi import check, lib
from .configs import System


def _ptr(t: torch.Tensor | None):
    if t is None:
        return None
    assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
    return C.c_void_p(t.data_ptr())


def make_desc(params: dict) -> _capi.PsDesc:
    d = _capi.PsDesc()
    for k, v in params.items():
        if k == "box":
            continue
        setattr(d, k, v)
    if params.get("box") is not None:
        d.box_on = 1
        for i in range(3):
            d.box[i] = float(params["box"][i])
    return d


class Batch:
    """A batch of independent systems advanced by the B200 engine."""

    def __init__(self, systems: list[System], precision: int = _capi.PS_PREC_FP64, device: str = "cuda:0",
                 lub_table: np.ndarray | None = None):
        self.systems = systems
        self.R = len(systems)
        self.device = torch.device(device)
        torch.cuda.set_device(self.device)
        arr = (_capi.PsDesc * self.R)()
        for i, s in enumerate(systems):
            arr[i] = make_desc(s.params)
        self.h = C.c_void_p()
        check(lib().ps_ctx_create(arr, self.R, precision, C.byref(self.h)), "ps_ctx_create")
        sz = (C.c_int64 * 8)()
        lib().ps_ctx_sizes(self.h, sz)
        self.ntot, self.nvec, self.ntop, self.nvel, self.ncoll = [int(v) for v in sz[:5]]
        self.off = []
        coll = 0
        for r in range(self.R):
            o = (C.c_int64 * 4)()
            lib().ps_ctx_offsets(self.h, r, o)
            self.off.append(dict(bead=int(o[0]), vec=int(o[1]), top=int(o[2]), vel=int(o[3]), coll=coll))
            coll += systems[r].params["Nc"]
        if any(s.params.get("lub_on") for s in systems):
            from .lubdat import load_table
            tab = np.ascontiguousarray(load_table() if lub_table is None else lub_table, dtype=np.float64)
            check(lib().ps_set_lub_table(self.h, tab.ctypes.data_as(C.c_void_p), tab.shape[0], tab.shape[1]),
                  "ps_set_lub_table")
        x = np.concatenate([np.ascontiguousarray(s.x, dtype=np.float64).ravel() for s in systems])
        self.set_state(torch.from_numpy(x).to(self.device))

    def close(self):
        if self.h:
            torch.cuda.synchronize()
            lib().ps_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def zeros(self, n):
        return torch.zeros(n, dtype=torch.float64, device=self.device)

    # state -----------------------------------------------------------------
    def set_state(self, x: torch.Tensor, q: torch.Tensor | None = None):
        check(lib().ps_set_state(self.h, _ptr(x.contiguous()), _ptr(q), self.stream), "ps_set_state")

    def state(self):
        x = self.zeros(3 * self.ntot)
        q = self.zeros(max(4 * self.ncoll, 1))
        check(lib().ps_get_state(self.h, _ptr(x), _ptr(q), self.stream), "ps_get_state")
        return x, q[: 4 * self.ncoll]

    def set_time(self, t: float):
        check(lib().ps_set_time(self.h, float(t)), "ps_set_time")

    def set_seed(self, seed: int):
        check(lib().ps_set_seed(self.h, int(seed)), "ps_set_seed")

    def set_replica_seeds(self, seeds, steps=None):
        sd = (C.c_uint64 * self.R)(*[int(v) for v in seeds])
        stp = None if steps is None else (C.c_uint64 * self.R)(*[int(v) for v in steps])
        check(lib().ps_set_replica_seeds(self.h, sd, stp), "ps_set_replica_seeds")

    def replica_steps(self) -> list[int]:
        out = (C.c_uint64 * self.R)()
        check(lib().ps_get_replica_steps(self.h, out), "ps_get_replica_steps")
        return list(out)

    def aux(self):
        """(time[R], ktrap[R], xpos0[3 ncoll]) as device tensors."""
        t, k, xp = self.zeros(self.R), self.zeros(self.R), self.zeros(max(3 * self.ncoll, 1))
        check(lib().ps_get_aux(self.h, _ptr(t), _ptr(k), _ptr(xp), self.stream), "ps_get_aux")
        return t, k, xp[: 3 * self.ncoll]

    def autotune(self, reps: int = 5):
        """Pick the monomer far-field column-chunk width for this process (ps_autotune);
        returns (width, {width: ms per mobility apply, combine included})."""
        best = C.c_int32(0)
        ms = (C.c_double * 4)()
        check(lib().ps_autotune(self.h, reps, C.byref(best), ms, self.stream), "ps_autotune")
        return int(best.value), dict(zip((128, 256, 512, 1024), list(ms)))

    # observables -----------------------------------------------------------
    def obs_reset(self, nbins: int = 64, bond_max: float = 4.0, trap_max: float = 2.0, lags: int = 64):
        self._obs = (nbins, lags)
        check(lib().ps_obs_reset(self.h, nbins, bond_max, trap_max, lags), "ps_obs_reset")

    def observe(self):
        check(lib().ps_observe(self.h, self.stream), "ps_observe")

    def observables(self) -> dict:
        """Per-replica accumulators (see ps_obs_out in the C header)."""
        nbins, lags = self._obs
        R = self.R
        out = {"bond": np.zeros((R, 10)), "bond_hist": np.zeros((R, nbins), np.uint64),
               "trap": np.zeros((R, 9)), "trap_hist": np.zeros((R, nbins), np.uint64),
               "msd": np.zeros((R, lags, 6)), "msd_count": np.zeros((R, lags), np.uint64)}
        o = _capi.PsObsOut(*[C.c_void_p(out[k].ctypes.data) for k in
                             ("bond", "bond_hist", "trap", "trap_hist", "msd", "msd_count")])
        check(lib().ps_obs_read(self.h, C.byref(o), self.stream), "ps_obs_read")
        return out

    def set_aux(self, time=None, ktrap=None, xpos0=None):
        check(lib().ps_set_aux(self.h, _ptr(time), _ptr(ktrap), _ptr(xpos0), self.stream), "ps_set_aux")

    # stage -----------------------------------------------------------------
    def stage(self) -> torch.Tensor:
        """check_dist + RHS + mob (+ Schur floor); returns the rhs vector."""
        rhs = self.zeros(self.nvec)
        check(lib().ps_build_pairs(self.h, self.stream), "ps_build_pairs")
        check(lib().ps_rhs(self.h, 0, None, _ptr(rhs), self.stream), "ps_rhs")
        check(lib().ps_assemble(self.h, self.stream), "ps_assemble")
        return rhs

    def pair_list(self, which: int):
        cnt = C.c_int64(0)
        check(lib().ps_pair_list(self.h, which, None, None, 0, C.byref(cnt), self.stream), "ps_pair_list")
        n = cnt.value
        pi = torch.zeros(max(n, 1), dtype=torch.int32, device=self.device)
        pj = torch.zeros(max(n, 1), dtype=torch.int32, device=self.device)
        check(lib().ps_pair_list(self.h, which, C.c_void_p(pi.data_ptr()), C.c_void_p(pj.data_ptr()), n,
                                 C.byref(cnt), self.stream), "ps_pair_list")
        return pi[:n], pj[:n]

    # operators -------------------------------------------------------------
    def matmult(self, x: torch.Tensor) -> torch.Tensor:
        y = self.zeros(self.nvec)
        check(lib().ps_matmult(self.h, _ptr(x), _ptr(y), self.stream), "ps_matmult")
        return y

    def mobility_apply(self, u: torch.Tensor) -> torch.Tensor:
        y = self.zeros(self.ntop)
        check(lib().ps_mobility_apply(self.h, _ptr(u), _ptr(y), self.stream), "ps_mobility_apply")
        return y

    def diagonal(self) -> torch.Tensor:
        d = self.zeros(self.nvec)
        check(lib().ps_get_diagonal(self.h, _ptr(d), self.stream), "ps_get_diagonal")
        return d

    def solve(self, b: torch.Tensor, x0: torch.Tensor | None = None, rtol: float = 1e-8, maxit: int = 10000,
              method: int = _capi.PS_SOLVE_MINRES):
        x = self.zeros(self.nvec) if x0 is None else x0.clone()
        o = _capi.PsKspOpts(rtol, maxit, int(x0 is not None), 8, method)
        r = _capi.PsKspResult()
        rc = lib().ps_ksp_solve(self.h, _ptr(b), _ptr(x), C.byref(o), C.byref(r), self.stream)
        if rc == _capi.PS_OK - 2:
            check(rc, "ps_ksp_solve")
        return x, r

    def sqrtm(self, z: torch.Tensor, kmax: int = 60, tol: float = 1e-12):
        w = self.zeros(self.ntop)
        o = _capi.PsSqrtOpts(kmax, tol)
        r = _capi.PsSqrtResult()
        check(lib().ps_sqrtm_apply(self.h, _ptr(z), _ptr(w), C.byref(o), C.byref(r), self.stream), "ps_sqrtm_apply")
        return w, r

    def step(self, fb: torch.Tensor | None = None, wrfd: torch.Tensor | None = None, rtol: float = 1e-8,
             maxit: int = 10000, sqrt_kmax: int = 0, sqrt_tol: float = 0.0, solver: int = 0,
             zlub: torch.Tensor | None = None, refine: int = 0):
        inp = _capi.PsStepInputs(None if fb is None else fb.data_ptr(), None if wrfd is None else wrfd.data_ptr(),
                                 None if zlub is None else zlub.data_ptr(), rtol, maxit, sqrt_kmax, sqrt_tol, solver,
                                 refine)
        res = _capi.PsStepResult()
        check(lib().ps_step(self.h, C.byref(inp), C.byref(res), self.stream), "ps_step")
        return res

    def step_outputs(self):
        bufs = [self.zeros(self.nvel) for _ in range(4)]
        check(lib().ps_step_outputs(self.h, *[_ptr(b) for b in bufs], self.stream), "ps_step_outputs")
        return dict(zip(("up", "udiff", "sb", "fext"), bufs))

    # per-replica views -----------------------------------------------------
    def seg(self, t: torch.Tensor, r: int, kind: str):
        s = self.systems[r].params
        Nm, Nc = s["Nm"], s["Nc"]
        n = {"vec": 6 * Nm + 17 * Nc, "top": 3 * Nm + 11 * Nc, "vel": 3 * Nm + 6 * Nc, "bead": 3 * (Nm + Nc)}[kind]
        o = self.off[r][kind] * (3 if kind == "bead" else 1)
        return t[o:o + n]
