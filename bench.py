"""Benchmark: bead-steps/s of the per-timestep Stokesian-dynamics path on B200.

One step = one full predictor-corrector step of every replica (5 saddle solves,
Brownian noise M^{1/2} z, the RFD drift and lubrication; src/run.cpp:70-162 of
the reference).  bead-steps = sum over replicas of N_r x steps.

Default: the batched ensemble (256 replicas, N log-uniform in [64, 4096], full
HI with lubrication), FP32-mixed far field, structured saddle solve, rtol 1e-8
(the tolerance at which the mixed form stays within 1e-6 of FP64).  Beside the
headline value the line carries the same ensemble in FP64 (batched), the plain
FP64 GPU drop-in (one replica at a time, Jacobi MINRES) projected from a sample,
and the mixed form's velocity error against FP64.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload ensemble|brush|suspension|polymer_probe]
                  [--precision fp64|mixed] [--replicas R] [--no-lub] [--rtol T]

For N > 1 it is launched under torchrun; every rank advances its own seeded
ensemble (weak scaling, no collective in the step) and rank 0 prints the line.
The reference arm (--impl reference) times the reference's own code
(oracle/_ref: its sources built against the PETSc/SLEPc stand-in; the CPU
restatement in oracle/ where that build is absent) on all host cores, on a
bounded, stratified sample of the same workload's replicas.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from polystokes_brownian_b200 import configs  # noqa: E402

METRIC = "bead-steps/s"
FLOP_AA = 40      # algorithmic FLOP per directed monomer-monomer pair (F-F RPY)
FLOP_BB = 250     # per directed colloid-colloid FTS pair (contracted block action, mul and add each counted)
# DRAM bytes (read + write) of one launch of the roofline kernel, from one ncu
# capture on the bench workload (profiles/k_rpy_aa_f2_ensemble256_lub.md:
# dram__bytes_read.sum 16.47 MB + dram__bytes_write.sum 12.61 MB, chunk width 256)
NCU_TRAFFIC = {("ensemble256_lub", "k_rpy_aa_f2"): {"bytes": 29.08e6, "chunk_cols": 256}}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="ensemble", choices=["ensemble", "brush", "suspension", "polymer_probe"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--replicas", type=int, default=256)
    ap.add_argument("--no-lub", action="store_true", help="ensemble/suspension without near-field lubrication")
    ap.add_argument("--rtol", type=float, default=1e-8)
    ap.add_argument("--solver", default="structured", choices=["minres", "structured"])
    ap.add_argument("--plain-sample", type=int, default=12,
                    help="replicas timed one by one in the plain FP64 drop-in form (0: skip)")
    ap.add_argument("--err-sample", type=int, default=16, help="replicas of the mixed-vs-FP64 error check (0: skip)")
    ap.add_argument("--no-fp64-batched", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the bounded runs of the other configurations")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="N > 1: weak = one seeded ensemble per rank; strong = one ensemble split across ranks (LPT)")
    ap.add_argument("--profile-steps", type=int, default=0, metavar="S",
                    help="profiler driver: build the workload and run S steps (no autotuning, no bench line)")
    ap.add_argument("--profile-kernel", type=int, default=0, metavar="K",
                    help="profiler driver: build the workload, stage it once, launch only the monomer pair kernel "
                         "K times (default chunk width, no autotuning, no steps) and exit; prints no bench line")
    return ap.parse_args()


def profile_kernel(args):
    """A short, fixed launch sequence for profiler captures of the dominant kernel:
    the packing and pair-list kernels of one staging, then K launches of the
    monomer pair kernel through ps_time_kernel (one untimed warm launch + K)."""
    import ctypes as C

    import torch
    from polystokes_brownian_b200 import _capi
    from polystokes_brownian_b200.engine import Batch, _ptr

    torch.cuda.set_device(0)
    systems, name = workload(args)
    prec = _capi.PS_PREC_MIXED if args.precision == "mixed" else _capi.PS_PREC_FP64
    b = Batch(systems, precision=prec)
    b.stage()
    u = torch.randn(b.ntop, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    ms = C.c_double(0)
    _capi.check(_capi.lib().ps_time_kernel(b.h, 0, args.profile_kernel, _ptr(u), C.byref(ms), b.stream),
                "ps_time_kernel")
    free, total = torch.cuda.mem_get_info()
    print(json.dumps({"profile_kernel": "k_rpy_aa_f2" if prec == _capi.PS_PREC_MIXED else "k_rpy_aa",
                      "workload": name, "launches": args.profile_kernel + 1, "ms_per_launch": ms.value,
                      "device_gb_in_use": (total - free) / 1e9}))
    b.close()


def profile_steps(args):
    """A short, fixed step sequence for profiler captures of the step's kernels (launch
    lists, the HBM-bound solver kernels): the workload at the default chunk width, S steps."""
    import torch
    from polystokes_brownian_b200 import _capi
    from polystokes_brownian_b200.engine import Batch

    torch.cuda.set_device(0)
    systems, name = workload(args)
    prec = _capi.PS_PREC_MIXED if args.precision == "mixed" else _capi.PS_PREC_FP64
    solver = _capi.PS_SOLVE_STRUCTURED if args.solver == "structured" else _capi.PS_SOLVE_MINRES
    b = Batch(systems, precision=prec)
    st = torch.cuda.current_stream()
    ms = []
    for _ in range(args.profile_steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        b.step(rtol=args.rtol, maxit=50000, solver=solver)
        e1.record(st)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    print(json.dumps({"profile_steps": args.profile_steps, "workload": name, "precision": args.precision,
                      "solver": args.solver, "ms_per_step": ms}))
    b.close()


def workload(args, rank=0, world=1):
    if args.scaling == "strong" and world > 1:
        from polystokes_brownian_b200 import shard
        systems, name = workload(args, 0, 1)
        return shard.rank_systems(systems, rank, world), name
    seed = args.seed + 1000 * rank
    lub = not args.no_lub
    if args.workload == "ensemble":
        return configs.ensemble(args.replicas, seed=seed, lub=lub), f"ensemble{args.replicas}" + ("_lub" if lub else "")
    if args.workload == "brush":
        return [configs.brush(seed=seed)], "brush4097"
    if args.workload == "suspension":
        s = configs.suspension(seed=seed)
        if lub:
            s = configs.System(s.name, dict(s.params, lub_on=1, lub_gap=0.5), s.x)
        return [s], "suspension1024" + ("_lub" if lub else "")
    return [configs.polymer_probe(seed=seed)], "polymer_probe222"


def pair_flops(systems):
    f = 0.0
    for s in systems:
        p = s.params
        if p["mm_HI"]:
            f += FLOP_AA * p["Nm"] * (p["Nm"] - 1)
    return f


def colloid_pair_flops(systems):
    return float(sum(FLOP_BB * s.params["Nc"] * (s.params["Nc"] - 1) for s in systems))


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index=0):
        self.f = tempfile.NamedTemporaryFile(prefix="clk", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def scaled_instances(args):
    """Smaller instances of a single-system workload (same kind, density and
    parameters) for the CPU sample: the oracle cannot step the full system in a
    bounded time."""
    lub = not args.no_lub
    if args.workload == "suspension":
        out = []
        for n in (24, 48, 72):
            s = configs.suspension(n=n, seed=args.seed)
            if lub:
                s = configs.System(s.name, dict(s.params, lub_on=1, lub_gap=0.5), s.x)
            out.append(s)
        return out, "suspensions of 24, 48 and 72 colloids at volume fraction 0.2"
    if args.workload == "brush":
        return [configs.brush(nchain=k, nper=32, seed=args.seed) for k in (2, 4, 6)], \
            "brushes of 2, 4 and 6 chains of 32 beads on the same colloid"
    return None, None


def cpu_baseline(systems, steps_budget_s=20.0, rtol=1e-6, threads=1, sample_systems=None, sample_desc=None):
    """Oracle (CPU restatement, 1 thread) on a stratified sample of replicas (or
    on smaller instances of a single-system workload); the per-replica step time
    is fitted as a N^2 + b N and projected onto the whole workload."""
    from oracle import psoracle as po
    Ns = np.array([s.Np for s in systems])
    if sample_systems is not None:
        pool = sample_systems
    else:
        pool = [systems[int(i)] for i in np.argsort(Ns)[:: max(1, len(systems) // 12)]]
    # smallest-to-larger sample until the budget is used
    sample, times = [], []
    t_start = time.perf_counter()
    for s in pool:
        if s.Np > 700 and sample:
            break
        tab = None
        if s.params.get("lub_on"):
            from polystokes_brownian_b200.lubdat import load_table
            tab = load_table()
        o = po.OracleSim(po.default_params(**dict(s.params, noise_lanczos=1)), s.x.ravel(), lub_table=tab)
        rng = np.random.default_rng(0)
        zl = rng.normal(size=12 * len(o.lub_pairs()[0])) if tab is not None else None
        t0 = time.perf_counter()
        o.step(fb=rng.normal(size=o.nm3nc11), wrfd=rng.normal(size=o.nm3nc6), zlub=zl, rtol=rtol)
        times.append(time.perf_counter() - t0)
        sample.append(s.Np)
        if time.perf_counter() - t_start > steps_budget_s:
            break
    n = np.array(sample, float)
    A = np.stack([n * n, n], 1)
    coef, *_ = np.linalg.lstsq(A, np.array(times), rcond=None)
    coef = np.maximum(coef, 0)
    proj = float(sum(coef[0] * N * N + coef[1] * N for N in Ns))
    if len(systems) == 1 and sample_systems is None:
        proj = float(np.mean(times))
    value = float(Ns.sum()) / proj
    what = sample_desc or f"{len(sample)} replicas"
    desc = (f"oracle (C restatement) 1 thread, one step of each of {what}, N in "
            f"[{int(n.min())},{int(n.max())}], step time fitted a*N^2+b*N and projected onto the workload")
    return {"value": value, "unit": METRIC, "cores": threads, "kind": "port", "sample": desc,
            "sample_seconds": float(sum(times))}


def _oracle_step_seconds(s, rtol):
    """One oracle step of system s (worker-process entry point); returns (Np, seconds)."""
    from oracle import psoracle as po
    tab = None
    if s.params.get("lub_on"):
        from polystokes_brownian_b200.lubdat import load_table
        tab = load_table()
    o = po.OracleSim(po.default_params(**dict(s.params, noise_lanczos=1)), s.x.ravel(), lub_table=tab)
    rng = np.random.default_rng(0)
    zl = rng.normal(size=12 * len(o.lub_pairs()[0])) if tab is not None else None
    t0 = time.perf_counter()
    o.step(fb=rng.normal(size=o.nm3nc11), wrfd=rng.normal(size=o.nm3nc6), zlub=zl, rtol=rtol)
    return s.Np, time.perf_counter() - t0


def _ref_step_seconds(params, x, rtol):
    """One step of the reference's own module on one system (fresh worker process)."""
    from oracle import refrun
    return refrun.step_seconds(params, np.ascontiguousarray(x, dtype=np.float64).ravel(), rtol)


def ref_pool(cores):
    """Fresh spawned process per task (the reference keeps global state); a worker that dies
    raises BrokenProcessPool instead of stalling the arm."""
    import concurrent.futures as cf
    import multiprocessing as mp
    return cf.ProcessPoolExecutor(cores, mp_context=mp.get_context("spawn"), max_tasks_per_child=1)


def power_fit(n, t):
    """t = a N^p by least squares in log-log; returns (a, p, relative rms residual)."""
    n, t = np.asarray(n, float), np.asarray(t, float)
    p, la = np.polyfit(np.log(n), np.log(t), 1)
    pred = np.exp(la) * n ** p
    return float(np.exp(la)), float(p), float(np.sqrt(np.mean(((pred - t) / t) ** 2)))


def ref_sample(systems, nmax, k, offset=0):
    """k replicas of the workload with N <= nmax and at least one colloid, spread evenly over
    that range (rotated by offset).  The reference cannot run a system without a colloid
    (initial_configuration reads the trap centre of colloid 0)."""
    Ns = np.array([s.Np for s in systems])
    small = [systems[int(i)] for i in np.argsort(Ns) if systems[int(i)].Np <= nmax and systems[int(i)].params["Nc"] > 0]
    if not small:
        small = [systems[int(np.argmin(Ns))]]
    m = len(small)
    return [small[(int(round(i * (m - 1) / max(1, k - 1))) + offset) % m] for i in range(k)]


def reference_cpu(systems, rtol, cores, steps, nmax=300, pool=None):
    """The reference's own code (oracle/_ref) stepping replicas of the workload on `cores`
    host cores: per bench step, `cores` replicas (N <= nmax, rotated through the range)
    run one reference step each, concurrently in fresh processes, so every time carries a
    loaded host's contention.  The per-replica step time is fitted as a N^p over all
    samples and the whole batch is scheduled longest-first on the cores.  The reference
    runs its own model on the same positions: its own pair scalars, no lubrication (it
    has none), MINRES + Jacobi at the workload's rtol."""
    own = pool is None
    if own:
        pool = ref_pool(cores)
    n, t = [], []
    try:
        for k in range(steps):
            pick = ref_sample(systems, nmax, cores, offset=k)
            res = list(pool.map(_ref_step_seconds, [s.params for s in pick], [s.x for s in pick],
                                [rtol] * len(pick)))
            n += [r[0] for r in res]
            t += [r[1] for r in res]
    finally:
        if own:
            pool.shutdown()
    a, pw, resid = power_fit(n, t)
    Ns = np.array([s.Np for s in systems])
    makespan = lpt_makespan([a * N ** pw for N in Ns], cores)
    desc = (f"the reference's own code (sources built against the PETSc/SLEPc stand-in) on {cores} cores: "
            f"{len(n)} one-step runs of workload replicas with N in [{min(n)},{max(n)}], {cores} at a time; "
            f"step time fitted as a*N^p (p = {pw:.2f}, rms residual {resid:.2f}), the batch scheduled "
            f"longest-first on the {cores} cores; its own model (reference pair scalars, no lubrication)")
    return {"value": float(Ns.sum()) / makespan, "unit": METRIC, "cores": cores, "kind": "reference",
            "sample": desc, "sample_seconds": float(sum(t)), "fit": {"a_s": a, "p": pw, "rms_rel_residual": resid,
                                                                      "N": n, "s": t}}


def cpu_baseline_ref(systems, rtol, k=6, nmax=250):
    """The reference's own code (oracle/_ref) on one core: one step each of k workload
    replicas with N <= nmax, one after another; step time fitted as a N^p and summed over
    the workload."""
    pool = ref_pool(1)
    try:
        pick = ref_sample(systems, nmax, k)
        res = list(pool.map(_ref_step_seconds, [s.params for s in pick], [s.x for s in pick], [rtol] * len(pick)))
    finally:
        pool.shutdown()
    n, t = [r[0] for r in res], [r[1] for r in res]
    a, pw, resid = power_fit(n, t)
    Ns = np.array([s.Np for s in systems])
    total = float(sum(a * N ** pw for N in Ns))
    desc = (f"the reference's own code (sources built against the PETSc/SLEPc stand-in), 1 core, one step each "
            f"of {len(n)} workload replicas with N in [{min(n)},{max(n)}]; step time fitted as a*N^p "
            f"(p = {pw:.2f}, rms residual {resid:.2f}) and summed over the workload; its own model (reference "
            f"pair scalars, no lubrication)")
    return {"value": float(Ns.sum()) / total, "unit": METRIC, "cores": 1, "kind": "reference", "sample": desc,
            "sample_seconds": float(sum(t)), "fit": {"a_s": a, "p": pw, "rms_rel_residual": resid, "N": n, "s": t}}


def lpt_makespan(times, cores):
    """Longest-processing-time-first schedule of independent jobs on `cores` workers."""
    loads = [0.0] * max(1, cores)
    for t in sorted(times, reverse=True):
        k = loads.index(min(loads))
        loads[k] += t
    return max(loads)


def cpu_baseline_parallel(systems, rtol, cores, pool, nmax=322):
    """The oracle on all host cores for a batch of independent replicas: `cores`
    spawned worker processes step a stratified sample of the smaller replicas
    (N <= nmax) at the same time, so each step time carries the contention of a
    fully loaded host; the per-replica step time is fitted as a N^2 + b N and the
    whole batch is scheduled on the cores (longest job first).  The oracle's step
    time grows faster than N^2 (its Jacobi MINRES needs more iterations as N
    grows: about N^2.6 over N = 50..700), so the quadratic projection overstates
    the CPU throughput on the large replicas; the same N range as the one-thread
    baseline keeps the two comparable."""
    Ns = np.array([s.Np for s in systems])
    small = [systems[int(i)] for i in np.argsort(Ns) if systems[int(i)].Np <= nmax]
    if not small:
        small = [systems[int(np.argmin(Ns))]]
    pick = [small[int(round(i * (len(small) - 1) / max(1, cores - 1)))] for i in range(cores)]
    res = pool.starmap(_oracle_step_seconds, [(s, rtol) for s in pick])
    n = np.array([r[0] for r in res], float)
    t = np.array([r[1] for r in res], float)
    coef, *_ = np.linalg.lstsq(np.stack([n * n, n], 1), t, rcond=None)
    coef = np.maximum(coef, 0)
    makespan = lpt_makespan([coef[0] * N * N + coef[1] * N for N in Ns], cores)
    desc = (f"oracle (C restatement) on {cores} worker processes, one step each of {len(pick)} replicas with N in "
            f"[{int(n.min())},{int(n.max())}] run concurrently, step time fitted a*N^2+b*N, the batch scheduled "
            f"longest-first on the {cores} cores")
    return {"value": float(Ns.sum()) / makespan, "unit": METRIC, "cores": cores, "kind": "port", "sample": desc,
            "sample_seconds": float(t.sum())}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import refrun
    systems, name = workload(args, 0)
    vals = []
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    single = len(systems) == 1
    use_ref = refrun.available() and not single
    pool = None
    if use_ref:
        pool = ref_pool(cores)
    elif not single:
        import multiprocessing as mp
        pool = mp.get_context("spawn").Pool(cores)     # spawned once; no GPU in this arm
    try:
        if use_ref:
            # the fit uses every timed sample; the warm-up steps prime the page cache and processes
            reference_cpu(systems, args.rtol, cores, args.warmup, pool=pool)
            cb = reference_cpu(systems, args.rtol, cores, args.steps, pool=pool)
            vals = [cb["value"]]
        else:
            for k in range(args.warmup + args.steps):
                if single:
                    # one system: the port has no parallelism inside a system
                    ss, sd = scaled_instances(args) if systems[0].Np > 700 else (None, None)
                    cb = cpu_baseline(systems, steps_budget_s=6.0, rtol=args.rtol, sample_systems=ss, sample_desc=sd)
                else:
                    cb = cpu_baseline_parallel(systems, args.rtol, cores, pool)
                if k >= args.warmup:
                    vals.append(cb["value"])
    finally:
        if use_ref:
            pool.shutdown()
        elif pool is not None:
            pool.close()
            pool.join()
    v = float(np.median(vals))
    out = {"metric": METRIC, "value": v, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": name, "replicas_per_rank": len(systems),
                      "beads_job": int(sum(s.Np for s in systems)), "rtol": args.rtol},
           "cpu_baseline": {"value": v, "unit": METRIC, "cores": cb["cores"], "kind": cb["kind"],
                            "sample": cb["sample"]},
           "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if "fit" in cb:
        out["cpu_baseline"]["fit"] = cb["fit"]
    print(json.dumps(out), flush=True)


def _fit_project(n, ms, Ns):
    """Per-replica step time interpolated linearly in log N - log t between the
    sampled replicas (the sample holds the smallest and the largest N, so no
    replica is extrapolated; equal N are averaged), summed over Ns.  Returns
    (total ms, rms relative deviation of a quadratic a + b N + c N^2 fit from the
    sample, which shows how far the step time is from a smooth law in N: MINRES
    iteration counts vary from replica to replica)."""
    n = np.asarray(n, float)
    ms = np.asarray(ms, float)
    un = np.unique(n)
    ut = np.array([np.exp(np.mean(np.log(ms[n == v]))) for v in un])
    lt = np.interp(np.log(np.clip(np.asarray(Ns, float), un[0], un[-1])), np.log(un), np.log(ut))
    A = np.stack([np.ones_like(n), n, n * n], 1)
    coef, *_ = np.linalg.lstsq(A, ms, rcond=None)
    resid = float(np.sqrt(np.mean(((A @ coef - ms) / ms) ** 2))) if len(n) >= 3 else float("nan")
    return float(np.sum(np.exp(lt))), resid


def plain_fp64(systems, args, budget_s=90.0):
    """The plain FP64 GPU drop-in: each replica in its own context, one at a time,
    FP64 operator and Jacobi-preconditioned MINRES -- the reference's MatShell +
    KSPSolve path moved to the GPU.  The same replicas are also stepped one at a time
    with the structured solve, which splits the headline ratio into algorithm
    (MINRES -> structured, one replica at a time), batching (one at a time -> batched,
    FP64) and precision (FP64 -> mixed, batched).  A stratified sample that includes
    the three largest replicas is stepped (one timed step each, CUDA events); the
    per-replica step time is interpolated log-log in N between the sampled replicas
    and summed over the workload."""
    import torch
    from polystokes_brownian_b200 import _capi
    from polystokes_brownian_b200.engine import Batch
    Ns = np.array([s.Np for s in systems])
    order = np.argsort(Ns)
    k = min(args.plain_sample, len(systems))
    pick = [int(order[int(round(i * (len(order) - 1) / max(1, k - 1)))]) for i in range(k)]
    pick += [int(i) for i in order[-3:]]
    pick = sorted(set(pick), key=lambda i: Ns[i])
    st = torch.cuda.current_stream()

    def timed_step(b, solver):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        r = b.step(rtol=args.rtol, maxit=50000, solver=solver)
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1), r

    n, ms, ms_struct, iters = [], [], [], []
    t_start = time.perf_counter()
    for idx in pick:
        for solver in (_capi.PS_SOLVE_STRUCTURED, _capi.PS_SOLVE_MINRES):
            b = Batch([systems[idx]], precision=_capi.PS_PREC_FP64)
            if solver == _capi.PS_SOLVE_STRUCTURED or Ns[idx] < 1000:
                b.step(rtol=args.rtol, maxit=50000, solver=solver)     # warm-up (skipped for the long MINRES runs)
            t, r = timed_step(b, solver)
            b.close()
            if solver == _capi.PS_SOLVE_MINRES:
                ms.append(t)
                iters.append(max(r.iters))
            else:
                ms_struct.append(t)
        n.append(systems[idx].Np)
        if time.perf_counter() - t_start > budget_s:
            break
    total_ms, resid = _fit_project(n, ms, Ns)
    total_struct, resid_s = _fit_project(n, ms_struct, Ns)
    return {"value": float(Ns.sum()) / (total_ms * 1e-3), "unit": METRIC, "ms_per_step_projected": total_ms,
            "sample_N": [int(v) for v in n], "sample_ms": ms, "sample_max_minres_iters": iters,
            "quadratic_fit_rms_rel_deviation": resid,
            "form": "FP64, one replica per context, Jacobi-preconditioned MINRES (the reference's KSPSolve), "
                    "rtol as the batched run",
            "projection": "per-replica step time interpolated linearly in log N - log t between the sampled replicas "
                          "(smallest and largest N included), summed over all replicas",
            "structured_single": {"value": float(Ns.sum()) / (total_struct * 1e-3), "unit": METRIC,
                                  "ms_per_step_projected": total_struct, "sample_ms": ms_struct,
                                  "quadratic_fit_rms_rel_deviation": resid_s,
                                  "form": "FP64, one replica per context, structured solve"}}


def velocity_error(systems, args, precision=None):
    """Relative velocity error of one step of the benchmarked form against FP64
    at rtol 1e-10 on the same state and the same injected noise (first
    err_sample replicas)."""
    import torch
    from polystokes_brownian_b200 import _capi
    from polystokes_brownian_b200.engine import Batch
    sub = systems[: max(1, args.err_sample)]
    precision = precision or args.precision
    prec = _capi.PS_PREC_MIXED if precision == "mixed" else _capi.PS_PREC_FP64
    solver = _capi.PS_SOLVE_STRUCTURED if args.solver == "structured" else _capi.PS_SOLVE_MINRES
    out = []
    runs = [(prec, args.rtol, 0), (_capi.PS_PREC_FP64, 1e-10, 0)]
    if prec == _capi.PS_PREC_MIXED:
        runs.append((prec, args.rtol, 1))      # one FP64 iterative-refinement sweep per solve
    for pr, rt, rf in runs:
        b = Batch(sub, precision=pr)
        fb = torch.from_numpy(np.random.default_rng(1).normal(size=b.ntop)).cuda()
        wr = torch.from_numpy(np.random.default_rng(2).normal(size=b.nvel)).cuda()
        b.step(fb=fb, wrfd=wr, rtol=rt, maxit=50000, solver=solver, refine=rf)
        out.append(b.step_outputs()["up"].cpu().numpy())
        b.close()
    err = float(np.linalg.norm(out[0] - out[1]) / np.linalg.norm(out[1]))
    res = {"rel_err_up": err, "replicas": len(sub), "against": "FP64 at rtol 1e-10, same state and injected noise",
           "bound": 1e-6, "ok": err <= 1e-6}
    if len(out) > 2:
        res["rel_err_up_refined"] = float(np.linalg.norm(out[2] - out[1]) / np.linalg.norm(out[1]))
    return res


def time_steps(systems, precision, solver, rtol, steps, warmup=1, refine=0):
    """Device time of `steps` steps of one context (CUDA events, after `warmup` steps);
    refine = FP64 iterative-refinement sweeps per solve."""
    import torch
    from polystokes_brownian_b200.engine import Batch
    b = Batch(systems, precision=precision)
    st = torch.cuda.current_stream()
    its = []
    for _ in range(warmup):
        b.step(rtol=rtol, maxit=50000, solver=solver, refine=refine)
    torch.cuda.synchronize()
    lat = []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        r = b.step(rtol=rtol, maxit=50000, solver=solver, refine=refine)
        e1.record(st)
        e1.synchronize()
        lat.append(e0.elapsed_time(e1))
        its.append(max(r.iters))
    x, _ = b.state()
    finite = bool(torch.isfinite(x).all().item())
    b.close()
    beads = sum(s.Np for s in systems)
    lat_s = sorted(lat)
    return {"value": beads * steps / (sum(lat) * 1e-3), "unit": METRIC, "ms_per_step": sum(lat) / steps,
            "p50_ms": lat_s[len(lat) // 2], "p99_ms": lat_s[min(len(lat) - 1, int(0.99 * len(lat)))],
            "steps": steps, "warmup": warmup, "max_solver_iters": max(its), "state_finite": finite}


def config_entries(args):
    """Bounded runs of the other benchmark configurations, each on its own context:
    C1 polymer + probes (plain FP64 drop-in: Jacobi MINRES), C2 1024-colloid suspension
    with lubrication and C3 4097-bead brush (mixed and FP64, with the mixed form's
    velocity error), C5 a short serving trace (p50/p99 step and request latency)."""
    from polystokes_brownian_b200 import _capi, serve
    F64, MIX = _capi.PS_PREC_FP64, _capi.PS_PREC_MIXED
    ST, MR = _capi.PS_SOLVE_STRUCTURED, _capi.PS_SOLVE_MINRES
    out = {}
    c1 = configs.polymer_probe(seed=args.seed)
    out["C1_polymer_probe222"] = {
        "plain_fp64_minres": time_steps([c1], F64, MR, args.rtol, steps=20, warmup=2),
        "fp64_structured": time_steps([c1], F64, ST, args.rtol, steps=20, warmup=2),
        "config": "2 probes (a_c = 3) + 11 harmonic chains x 20 beads, shell path, dt 1e-3, rtol as the headline"}
    s2 = configs.suspension(seed=args.seed)
    s2 = configs.System(s2.name, dict(s2.params, lub_on=1, lub_gap=0.5), s2.x)
    e2 = argparse.Namespace(**vars(args))
    e2.err_sample = 1
    out["C2_suspension1024_lub"] = {
        "mixed": time_steps([s2], MIX, ST, args.rtol, steps=5, warmup=2),
        "fp64": time_steps([s2], F64, ST, args.rtol, steps=5, warmup=2),
        "velocity_error": velocity_error([s2], e2, "mixed"),
        "config": "1024 colloids, volume fraction 0.2, lubrication for gaps < 0.5 a, dt 1e-4; colloid blocks are "
                  "FP64 in both forms"}
    s3 = configs.brush(seed=args.seed)
    out["C3_brush4097"] = {
        "mixed": time_steps([s3], MIX, ST, args.rtol, steps=5, warmup=2),
        # the brush's forces cancel strongly in M F (|M|F|| / |M F| about 170 on the staged
        # state), which lifts the FP32 far field's relative error above 1e-6; one FP64
        # refinement sweep per solve brings it back (velocity_error.rel_err_up_refined)
        "mixed_refined": time_steps([s3], MIX, ST, args.rtol, steps=5, warmup=2, refine=1),
        "fp64": time_steps([s3], F64, ST, args.rtol, steps=5, warmup=2),
        "velocity_error": velocity_error([s3], e2, "mixed"),
        "config": "1 colloid (a_c = 5) + 128 FENE chains x 32 beads, full monomer HI, dt 1e-4"}
    trace = serve.make_trace(12, rate=4.0, seed=args.seed, nmax=4096, smax=40, lub=True)
    c5 = {"requests": len(trace), "rate_per_s": 4.0, "N": "log-uniform in [64, 4096]", "steps": "uniform in [10, 40]"}
    for name, prec in (("mixed", MIX), ("fp64", F64)):
        srv = serve.Server(precision=prec, rebuild_every=4, rtol=args.rtol)
        t0 = time.perf_counter()
        res = srv.run(trace)
        c5[name] = srv.stats(res, time.perf_counter() - t0)
    out["C5_serving"] = c5
    return out


def run_b200(args):
    import ctypes as C

    import torch
    import torch.distributed as dist
    from polystokes_brownian_b200 import _capi
    from polystokes_brownian_b200.engine import Batch, _ptr

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from polystokes_brownian_b200 import shard
    systems, name = workload(args, rank, world)
    prec = _capi.PS_PREC_MIXED if args.precision == "mixed" else _capi.PS_PREC_FP64
    solver = _capi.PS_SOLVE_STRUCTURED if args.solver == "structured" else _capi.PS_SOLVE_MINRES
    b = Batch(systems, precision=prec)
    beads = int(sum(s.Np for s in systems))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > L2
    st = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    b.stage()
    aa_cols, aa_tune_ms = b.autotune(5)      # far-field chunk width for this GPU and workload
    for _ in range(args.warmup):
        b.step(rtol=args.rtol, solver=solver)
    barrier()
    L = _capi.lib()
    launches0 = L.ps_kernel_launches()
    clk = Clocks(local)
    lat, iters, reasons = [], [], []
    t_total = 0.0
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        r = b.step(rtol=args.rtol, solver=solver)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        lat.append(ms)
        t_total += ms
        iters.append(list(r.iters) + [r.lanczos_iters])
        reasons.append(r.reason)
    barrier()
    clocks = clk.stop()
    launches = int(L.ps_kernel_launches() - launches0)
    xs, _ = b.state()
    finite = bool(torch.isfinite(xs).all().item())
    t_total = shard.max_over_ranks(t_total, device="cuda")
    job_beads = int(shard.sum_over_ranks(beads, device="cuda"))
    value = job_beads * args.steps / (t_total * 1e-3)

    # end to end through the C-ABI with host buffers: H2D positions, step, D2H positions
    xh = torch.empty(3 * b.ntot, dtype=torch.float64, pin_memory=True)
    xh.copy_(xs.cpu())
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        _capi.check(L.ps_set_state(b.h, C.c_void_p(xh.data_ptr()), None, b.stream), "ps_set_state")
        b.step(rtol=args.rtol, solver=solver)
        _capi.check(L.ps_get_state(b.h, C.c_void_p(xh.data_ptr()), None, b.stream), "ps_get_state")
    e1.record(st)
    e1.synchronize()
    te = shard.max_over_ranks(e0.elapsed_time(e1), device="cuda")
    e2e = job_beads * args.steps / (te * 1e-3)

    # roofline of the dominant kernel, timed live: the monomer-monomer pair kernel,
    # or the colloid-colloid FTS kernel (FP64 in both forms) for colloid-only workloads
    u = torch.randn(b.ntop, dtype=torch.float64, device="cuda")
    ms_k, ms_all, peak = C.c_double(0), C.c_double(0), C.c_double(0)
    flops = pair_flops(systems)
    if flops > 0:
        which, fp64_peak = 0, prec == _capi.PS_PREC_FP64
        kname = "k_rpy_aa_f2" if prec == _capi.PS_PREC_MIXED else "k_rpy_aa"
        funit = f"{FLOP_AA} per directed monomer pair"
    else:
        flops = colloid_pair_flops(systems)
        which, fp64_peak, kname = 2, True, "k_rpy_bb"
        funit = f"{FLOP_BB} per directed colloid pair (FTS block action, contracted)"
    _capi.check(L.ps_time_kernel(b.h, which, 10, _ptr(u), C.byref(ms_k), b.stream), "ps_time_kernel")
    _capi.check(L.ps_time_kernel(b.h, 3, 10, _ptr(u), C.byref(ms_all), b.stream), "ps_time_kernel")
    _capi.check(L.ps_fma_peak(1 if fp64_peak else 0, C.byref(peak), b.stream), "ps_fma_peak")
    achieved = flops / (ms_k.value * 1e-3) / 1e12 if ms_k.value > 0 else 0.0
    roof = {"bound": "fp64" if fp64_peak else "fp32", "kernel": kname,
            "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
            "frac": achieved / peak.value if peak.value else None,
            "traffic": NCU_TRAFFIC.get((name, kname), {}).get("bytes"),
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch at chunk width "
                               f"{NCU_TRAFFIC[(name, kname)]['chunk_cols']} (compute-bound: the FLOP roofline "
                               "applies)") if (name, kname) in NCU_TRAFFIC else None,
            "peak_source": "measured FMA throughput of this GPU in bench.py (ps_fma_peak); CUDA-core work, "
                           "no tensor-core or HBM denominator applies",
            "flop_per_launch": flops, "flop_unit": funit,
            "ms_per_launch": ms_k.value, "ms_mobility_apply": ms_all.value}
    ntot = b.ntot
    b.close()
    del flush

    extra = {}
    if rank == 0 and world == 1:
        if not args.no_fp64_batched and prec == _capi.PS_PREC_MIXED:
            bf = Batch(systems, precision=_capi.PS_PREC_FP64)
            bf.step(rtol=args.rtol, solver=solver)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(2):
                bf.step(rtol=args.rtol, solver=solver)
            e1.record(st)
            e1.synchronize()
            extra["fp64_batched"] = {"value": beads * 2 / (e0.elapsed_time(e1) * 1e-3), "unit": METRIC,
                                     "ms_per_step": e0.elapsed_time(e1) / 2, "form": "FP64, batched, same solver"}
            # the FP64 monomer pair kernel of this form against the measured FP64 FMA peak
            ms64, pk64 = C.c_double(0), C.c_double(0)
            u64 = torch.randn(bf.ntop, dtype=torch.float64, device="cuda")
            _capi.check(L.ps_time_kernel(bf.h, 0, 10, _ptr(u64), C.byref(ms64), bf.stream), "ps_time_kernel")
            _capi.check(L.ps_fma_peak(1, C.byref(pk64), bf.stream), "ps_fma_peak")
            f64 = pair_flops(systems)
            if f64 > 0 and ms64.value > 0:
                ach = f64 / (ms64.value * 1e-3) / 1e12
                extra["roofline_fp64"] = {"bound": "fp64", "kernel": "k_rpy_aa_d2", "achieved": ach, "peak": pk64.value,
                                          "unit": "TFLOP/s", "frac": ach / pk64.value, "ms_per_launch": ms64.value,
                                          "flop_per_launch": f64, "flop_unit": f"{FLOP_AA} per directed monomer pair",
                                          "peak_source": "measured FP64 FMA throughput of this GPU (ps_fma_peak)"}
            bf.close()
        if args.plain_sample > 0:
            pf = plain_fp64(systems, args)
            pf["ratio"] = value / pf["value"]
            extra["plain_fp64_drop_in"] = pf
        if args.err_sample > 0:
            extra["velocity_error"] = velocity_error(systems, args)
        if "fp64_batched" in extra and "plain_fp64_drop_in" in extra:
            pf, fb = extra["plain_fp64_drop_in"], extra["fp64_batched"]["value"]
            ss = pf["structured_single"]["value"]
            extra["decomposition"] = {
                "algorithm": ss / pf["value"], "batching": fb / ss, "precision": value / fb,
                "total": value / pf["value"],
                "note": "algorithm: FP64 one replica at a time, Jacobi MINRES -> structured solve; batching: FP64 "
                        "structured, one at a time -> all replicas in one context; precision: FP64 batched -> mixed "
                        "batched (one-at-a-time forms projected from the same sample)"}
        if args.workload == "ensemble" and not args.no_configs:
            extra["configs"] = config_entries(args)

    if rank == 0:
        from oracle import refrun
        cb = None
        if world == 1:
            if len(systems) > 1 and refrun.available():
                cb = cpu_baseline_ref(systems, args.rtol)
            else:
                ss, sd = scaled_instances(args) if len(systems) == 1 and systems[0].Np > 700 else (None, None)
                cb = cpu_baseline(systems, rtol=args.rtol, sample_systems=ss, sample_desc=sd)
        lat_sorted = sorted(lat)
        out = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": t_total / args.steps, "higher_is_better": True,
               "scaling": args.scaling, "vs_baseline": None, "dtype": "f32+f64" if prec == _capi.PS_PREC_MIXED else "f64",
               "data": "synthetic",
               "config": {"workload": name, "replicas_per_rank": len(systems), "beads_job": job_beads,
                          "rtol": args.rtol,
                          "precision": args.precision, "solver": args.solver,
                          "aa_chunk_cols": aa_cols, "autotune_ms_per_apply": aa_tune_ms,
                          "l2": "flushed (256 MB write) before every timed step",
                          "parallelism": f"independent replicas on {world} GPU(s) ({args.scaling} scaling), "
                                         "no collective in the step"},
               "latency_ms": {"p50": lat_sorted[len(lat) // 2],
                              "p99": lat_sorted[min(len(lat) - 1, int(0.99 * len(lat)))]},
               "iters": iters, "iters_note": "per step: max Krylov iterations of the 5 solves, then the Lanczos "
                                             "subspace size", "reason": reasons,
               "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": 8 * 3 * ntot,
                       "d2h_bytes_per_step": 8 * 3 * ntot},
               "gpu_launches": launches, "roofline": roof, "clocks": clocks, "state_finite": finite}
        out.update(extra)
        if cb:
            out["cpu_baseline"] = cb
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    a = parse()
    if a.profile_kernel:
        profile_kernel(a)
    elif a.profile_steps:
        profile_steps(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_b200(a)
