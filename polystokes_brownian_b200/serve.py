"""Continuous-batching request loop for trajectory requests.

Requests (a system, a step count, a noise seed) arrive open-loop; the loop keeps
every admitted trajectory resident on the device and advances all of them one
Heun step per launch sequence (one engine context over the active set).  New
arrivals are admitted, and finished trajectories retired, between steps:

  * admission is first-come-first-served against an HBM budget (the engine's
    per-replica footprint, ``footprint_bytes``) and a slot limit; a request whose
    footprint alone exceeds the budget is refused with an error result;
  * thermal (kT > 0) and athermal (kT = 0) trajectories advance in separate
    contexts (an engine context takes one kind: the step either draws noise and
    runs the RFD probes for every replica or for none), stepped back to back;
  * when the active set changes the context is rebuilt over the new set and the
    continuing trajectories carry their state across: positions, quaternions,
    time, trap constant and centres, and their own noise stream (seed and step
    counter) -- the kernels are per-replica deterministic (column chunking,
    reductions and Philox streams depend on the replica alone), so a trajectory
    ends bit-identical whether it ran alone or in any mix;
  * to amortise rebuilds a finished trajectory's result is taken at its last
    step and the replica may keep stepping (discarded work) until the next
    rebuild, at most ``rebuild_every`` steps later.

Per-step latency is the device time of one batch step (CUDA events); request
latency is wall time from arrival to the step that finishes it.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import time
from collections import deque

import numpy as np
import torch

from . import _capi, configs
from .configs import System
from .engine import Batch


@dataclasses.dataclass
class Request:
    rid: int
    system: System
    steps: int
    seed: int
    arrival: float = 0.0          # seconds after the start of the trace


@dataclasses.dataclass
class Result:
    rid: int
    x: np.ndarray
    q: np.ndarray
    steps: int
    arrival: float
    admitted: float
    finished: float
    error: str | None = None      # set when the request was refused (no trajectory)


@dataclasses.dataclass
class _Slot:
    req: Request
    x: np.ndarray
    q: np.ndarray
    time: float
    ktrap: float
    xpos0: np.ndarray
    done_steps: int = 0
    rng_steps: int = 0
    admitted: float = 0.0
    result: Result | None = None


def footprint_bytes(sysm: System, precision: int = _capi.PS_PREC_MIXED, lanczos_kmax: int = 64) -> int:
    """Device bytes one replica holds in a context: saddle vectors (13), mobility
    vectors incl. the Lanczos basis (kmax + 6) and far-field chunk partials,
    velocity vectors (27), positions, lists."""
    p = sysm.params
    Nm, Nc = p["Nm"], p["Nc"]
    n, top, vel, Np = 6 * Nm + 17 * Nc, 3 * Nm + 11 * Nc, 3 * Nm + 6 * Nc, Nm + Nc
    nch = max(1, math.ceil(Nm / 256))
    b = 8 * (13 * n + (lanczos_kmax + 6 + nch) * top + 27 * vel) + 160 * Np + 4 * 16 * Np
    if Nc and 5 * Nc <= 64:
        b += 8 * (5 * Nc) ** 2
    return int(b)


def make_trace(n_req: int, rate: float, seed: int = 0, nmin: int = 64, nmax: int = 16384,
               smin: int = 10, smax: int = 500, **kw) -> list[Request]:
    """Open-loop Poisson arrivals at `rate` requests/s; bead counts log-uniform in
    [nmin, nmax], step counts uniform in [smin, smax], structure as in the
    batched ensemble."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_req):
        t += rng.exponential(1.0 / rate) if rate > 0 else 0.0
        N = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        sysm = configs.ensemble_member(np.random.default_rng([seed, i]), N, **kw)
        out.append(Request(i, sysm, int(rng.integers(smin, smax + 1)), int(rng.integers(1, 2 ** 62)), t))
    return out


class Server:
    _tuned = False

    def __init__(self, precision: int = _capi.PS_PREC_MIXED, budget_bytes: float = 150e9, max_slots: int = 256,
                 rtol: float = 1e-6, solver: int = _capi.PS_SOLVE_STRUCTURED, rebuild_every: int = 1,
                 device: str = "cuda:0", lub_table: np.ndarray | None = None):
        self.precision = precision
        self.budget = budget_bytes
        self.max_slots = max_slots
        self.rtol = rtol
        self.solver = solver
        self.rebuild_every = max(1, rebuild_every)
        self.device = device
        self.lub_table = lub_table
        self.step_ms: list[float] = []
        self.batch_sizes: list[int] = []
        self.rebuilds = 0
        self.bead_steps = 0          # useful bead-steps (requested steps only)

    # -- state transfer ------------------------------------------------------
    def _admit(self, req: Request, now: float) -> _Slot:
        p = req.system.params
        x = np.ascontiguousarray(req.system.x, dtype=np.float64).ravel()
        Nc, Nm = p["Nc"], p["Nm"]
        q = np.tile(np.array([1.0, 0.0, 0.0, 0.0]), Nc)
        xpos0 = x[3 * Nm:].copy()          # fresh start: trap centres at the colloids
        return _Slot(req, x, q, float(p.get("t0", 0.0)), float(p.get("ktrap", 0.0)), xpos0, admitted=now)

    def _build(self, slots: list[_Slot]) -> list[tuple[list[_Slot], Batch]]:
        """One context per kT class present in the active set, in (thermal, athermal) order."""
        groups = []
        for thermal in (True, False):
            grp = [s for s in slots if (s.req.system.params["kT"] > 0) == thermal]
            if grp:
                groups.append((grp, self._build_one(grp)))
        return groups

    def _build_one(self, slots: list[_Slot]) -> Batch:
        systems = [s.req.system for s in slots]
        b = Batch(systems, precision=self.precision, device=self.device, lub_table=self.lub_table)
        dev = b.device
        x = torch.from_numpy(np.concatenate([s.x for s in slots])).to(dev)
        qs = [s.q for s in slots if s.q.size]
        q = torch.from_numpy(np.concatenate(qs)).to(dev) if qs else None
        b.set_state(x, q)
        t = torch.tensor([s.time for s in slots], dtype=torch.float64, device=dev)
        k = torch.tensor([s.ktrap for s in slots], dtype=torch.float64, device=dev)
        xp = [s.xpos0 for s in slots if s.xpos0.size]
        xp = torch.from_numpy(np.concatenate(xp)).to(dev) if xp else None
        b.set_aux(t, k, xp)
        b.set_replica_seeds([s.req.seed for s in slots], [s.rng_steps for s in slots])
        if not Server._tuned:
            # one process-wide choice, so every later context chunks replicas the same way
            b.stage()
            self.aa_chunk_cols, _ = b.autotune(3)
            Server._tuned = True
        self.rebuilds += 1
        return b

    def _export(self, b: Batch, slots: list[_Slot]):
        x, q = b.state()
        t, k, xp = b.aux()
        x, q, t, k, xp = (v.cpu().numpy() for v in (x, q, t, k, xp))
        steps = b.replica_steps()
        for r, s in enumerate(slots):
            s.x = b.seg(torch.from_numpy(x), r, "bead").numpy().copy()
            Nc = s.req.system.params["Nc"]
            co = b.off[r]["coll"]
            if Nc:
                s.q = q[4 * co:4 * co + 4 * Nc].copy()
                s.xpos0 = xp[3 * co:3 * co + 3 * Nc].copy()
            s.time, s.ktrap, s.rng_steps = float(t[r]), float(k[r]), int(steps[r])

    # -- main loop -------------------------------------------------------------
    def run(self, trace: list[Request], clock: str = "wall") -> list[Result]:
        pending = deque(sorted(trace, key=lambda r: r.arrival))
        active: list[_Slot] = []
        results: list[Result] = []
        used = 0.0
        groups: list[tuple[list[_Slot], Batch]] = []
        since_rebuild = 0
        t0 = time.perf_counter()
        vnow = 0.0

        def now():
            return time.perf_counter() - t0 if clock == "wall" else vnow

        while pending or active:
            live = [s for s in active if s.result is None]
            finished = [s for s in active if s.result is not None]
            arrivals = bool(pending) and pending[0].arrival <= now()
            must = not groups or not live
            if must or (since_rebuild >= self.rebuild_every and (finished or arrivals)):
                for grp, b in groups:
                    self._export(b, grp)
                    b.close()
                groups = []
                for s in finished:
                    used -= footprint_bytes(s.req.system, self.precision)
                active = live
                while pending and pending[0].arrival <= now() and len(active) < self.max_slots:
                    fb = footprint_bytes(pending[0].system, self.precision)
                    if fb > self.budget:
                        req = pending.popleft()
                        results.append(Result(req.rid, np.zeros(0), np.zeros(0), 0, req.arrival, now(), now(),
                                              error=f"footprint {fb:.3e} B exceeds the HBM budget {self.budget:.3e} B"))
                        continue
                    if used + fb > self.budget:
                        break
                    req = pending.popleft()
                    used += fb
                    active.append(self._admit(req, now()))
                if not active:
                    if pending:
                        wait = pending[0].arrival - now()
                        if clock == "wall":
                            time.sleep(max(0.0, wait))
                        else:
                            vnow = pending[0].arrival
                    continue
                groups = self._build(active)
                since_rebuild = 0
            # one step of the whole active set (one context per kT class, back to back)
            st = torch.cuda.current_stream()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _, b in groups:
                b.step(rtol=self.rtol, solver=self.solver)
            e1.record(st)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            self.step_ms.append(ms)
            self.batch_sizes.append(len(active))
            vnow += ms * 1e-3
            since_rebuild += 1
            for grp, b in groups:
                done_now = []
                for s in grp:
                    if s.result is None:
                        s.done_steps += 1
                        self.bead_steps += s.req.system.Np
                        if s.done_steps == s.req.steps:
                            done_now.append(s)
                if not done_now:
                    continue
                x, q = b.state()
                x, q = x.cpu(), q.cpu()
                for s in done_now:
                    r = grp.index(s)
                    Nc = s.req.system.params["Nc"]
                    co = b.off[r]["coll"]
                    s.result = Result(s.req.rid, b.seg(x, r, "bead").numpy().copy(),
                                      q[4 * co:4 * co + 4 * Nc].numpy().copy(), s.done_steps, s.req.arrival,
                                      s.admitted, now())
                    results.append(s.result)
        for _, b in groups:
            b.close()
        return sorted(results, key=lambda r: r.rid)

    def stats(self, results: list[Result], wall_s: float) -> dict:
        lat = sorted(self.step_ms)
        req = sorted(r.finished - r.arrival for r in results if r.error is None)

        def pct(v, p):
            return v[min(len(v) - 1, int(p * len(v)))] if v else None
        return {"bead_steps_per_s": self.bead_steps / wall_s if wall_s > 0 else None,
                "device_bead_steps_per_s": self.bead_steps / (sum(lat) * 1e-3) if lat else None,
                "step_ms": {"p50": pct(lat, 0.5), "p99": pct(lat, 0.99), "n": len(lat)},
                "request_s": {"p50": pct(req, 0.5), "p99": pct(req, 0.99), "n": len(req)},
                "mean_batch": float(np.mean(self.batch_sizes)) if self.batch_sizes else 0.0,
                "rebuilds": self.rebuilds, "refused": sum(r.error is not None for r in results)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=32)
    ap.add_argument("--rate", type=float, default=4.0, help="Poisson arrival rate, requests/s")
    ap.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"])
    ap.add_argument("--nmax", type=int, default=16384)
    ap.add_argument("--smax", type=int, default=500)
    ap.add_argument("--no-lub", action="store_true")
    ap.add_argument("--rtol", type=float, default=1e-8)
    ap.add_argument("--rebuild-every", type=int, default=4)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args()
    trace = make_trace(a.requests, a.rate, seed=a.seed, nmax=a.nmax, smax=a.smax, lub=not a.no_lub)
    precs = ["mixed", "fp64"] if a.precision == "both" else [a.precision]
    out = {"requests": len(trace), "rate": a.rate, "lub": not a.no_lub, "rtol": a.rtol,
           "bead_steps_requested": int(sum(r.system.Np * r.steps for r in trace))}
    for name in precs:
        prec = _capi.PS_PREC_MIXED if name == "mixed" else _capi.PS_PREC_FP64
        srv = Server(precision=prec, rebuild_every=a.rebuild_every, rtol=a.rtol)
        t = time.perf_counter()
        res = srv.run(trace)
        wall = time.perf_counter() - t
        out[name] = {"wall_s": wall, **srv.stats(res, wall)}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
