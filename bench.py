"""Benchmark: bead-steps/s of the per-timestep Stokesian-dynamics path on B200.

One step = one full predictor-corrector step of every replica (5 saddle solves,
Brownian noise M^{1/2} z and the RFD drift; src/run.cpp:70-162 of the
reference).  bead-steps = sum over replicas of N_r x steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload ensemble|brush|suspension|polymer_probe]
                  [--precision fp64|mixed] [--replicas R]

For N > 1 it is launched under torchrun; every rank advances its own seeded
ensemble (weak scaling, no collective in the step) and rank 0 prints the line.
The reference arm (--impl reference) times the CPU restatement of the
reference (oracle/, the reference itself needs PETSc/SLEPc and cannot be built
here) on a bounded, stratified sample of the same workload.
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
FLOP_BB = 600     # per directed colloid-colloid FTS pair


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="ensemble", choices=["ensemble", "brush", "suspension", "polymer_probe"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--replicas", type=int, default=256)
    ap.add_argument("--rtol", type=float, default=1e-6)
    ap.add_argument("--solver", default="structured", choices=["minres", "structured"])
    ap.add_argument("--seed", type=int, default=0)
    return ap.parse_args()


def workload(args, rank=0):
    seed = args.seed + 1000 * rank
    if args.workload == "ensemble":
        return configs.ensemble(args.replicas, seed=seed), f"ensemble{args.replicas}"
    if args.workload == "brush":
        return [configs.brush(seed=seed)], "brush4097"
    if args.workload == "suspension":
        return [configs.suspension(seed=seed)], "suspension1024"
    return [configs.polymer_probe(seed=seed)], "polymer_probe222"


def pair_flops(systems):
    f = 0.0
    for s in systems:
        p = s.params
        if p["mm_HI"]:
            f += FLOP_AA * p["Nm"] * (p["Nm"] - 1)
    return f


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


def cpu_baseline(systems, steps_budget_s=20.0, rtol=1e-6, threads=1):
    """Oracle (CPU restatement, 1 thread) on a stratified sample of replicas; the
    per-replica step time is fitted as a N^2 + b N and projected onto the whole
    workload."""
    from oracle import psoracle as po
    Ns = np.array([s.Np for s in systems])
    order = np.argsort(Ns)
    # smallest-to-larger sample until the budget is used
    sample, times = [], []
    t_start = time.perf_counter()
    for idx in order[:: max(1, len(order) // 12)]:
        s = systems[int(idx)]
        if s.Np > 700 and sample:
            break
        o = po.OracleSim(po.default_params(**dict(s.params, noise_lanczos=1)), s.x.ravel())
        rng = np.random.default_rng(0)
        t0 = time.perf_counter()
        o.step(fb=rng.normal(size=o.nm3nc11), wrfd=rng.normal(size=o.nm3nc6), rtol=rtol)
        times.append(time.perf_counter() - t0)
        sample.append(s.Np)
        if time.perf_counter() - t_start > steps_budget_s:
            break
    n = np.array(sample, float)
    A = np.stack([n * n, n], 1)
    coef, *_ = np.linalg.lstsq(A, np.array(times), rcond=None)
    coef = np.maximum(coef, 0)
    proj = float(sum(coef[0] * N * N + coef[1] * N for N in Ns))
    if len(systems) == 1:
        proj = float(np.mean(times))
    value = float(Ns.sum()) / proj
    desc = (f"oracle (C restatement) 1 thread, one step of each of {len(sample)} replicas with N in "
            f"[{int(n.min())},{int(n.max())}], step time fitted a*N^2+b*N and projected onto the workload")
    return {"value": value, "unit": METRIC, "cores": threads, "kind": "port", "sample": desc,
            "sample_seconds": float(sum(times))}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    systems, name = workload(args, 0)
    vals = []
    for k in range(args.warmup + args.steps):
        cb = cpu_baseline(systems, steps_budget_s=8.0, rtol=args.rtol)
        if k >= args.warmup:
            vals.append(cb["value"])
    v = float(np.median(vals))
    out = {"metric": METRIC, "value": v, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": name, "replicas": len(systems), "beads": int(sum(s.Np for s in systems)),
                      "rtol": args.rtol},
           "cpu_baseline": {"value": v, "unit": METRIC, "cores": 1, "kind": "port", "sample": cb["sample"]},
           "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_b200(args):
    import torch
    import torch.distributed as dist
    from polystokes_brownian_b200 import _capi
    from polystokes_brownian_b200.engine import Batch, _ptr
    import ctypes as C

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    systems, name = workload(args, rank)
    prec = _capi.PS_PREC_MIXED if args.precision == "mixed" else _capi.PS_PREC_FP64
    b = Batch(systems, precision=prec)
    beads = int(sum(s.Np for s in systems))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > L2
    st = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    solver = _capi.PS_SOLVE_STRUCTURED if args.solver == "structured" else _capi.PS_SOLVE_MINRES
    for _ in range(args.warmup):
        b.step(rtol=args.rtol, solver=solver)
    barrier()
    L = _capi.lib()
    launches0 = L.ps_kernel_launches()
    clk = Clocks(local)
    lat = []
    t_total = 0.0
    iters = []
    reasons = []
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
    xs, _ = b.state()
    finite = bool(torch.isfinite(xs).all().item())
    clocks = clk.stop()
    launches = int(L.ps_kernel_launches() - launches0)
    tmax = torch.tensor([t_total], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    t_total = float(tmax.item())
    value = beads * args.steps * world / (t_total * 1e-3)

    # end to end through the C-ABI with host buffers: H2D positions, step, D2H positions
    xh = torch.empty(3 * b.ntot, dtype=torch.float64, pin_memory=True)
    xd_state, _ = b.state()
    xh.copy_(xd_state.cpu())
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    e2e_iters = []
    for _ in range(args.steps):
        _capi.check(L.ps_set_state(b.h, C.c_void_p(xh.data_ptr()), None, b.stream), "ps_set_state")
        r = b.step(rtol=args.rtol, solver=solver)
        e2e_iters.append(list(r.iters))
        _capi.check(L.ps_get_state(b.h, C.c_void_p(xh.data_ptr()), None, b.stream), "ps_get_state")
    e1.record(st)
    e1.synchronize()
    te = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e = beads * args.steps * world / (float(te.item()) * 1e-3)

    # roofline of the dominant kernel (monomer-monomer pair kernel), timed live
    u = torch.randn(b.ntop, dtype=torch.float64, device="cuda")
    ms_aa = C.c_double(0)
    _capi.check(L.ps_time_kernel(b.h, 0, 10, _ptr(u), C.byref(ms_aa), b.stream), "ps_time_kernel")
    ms_all = C.c_double(0)
    _capi.check(L.ps_time_kernel(b.h, 3, 10, _ptr(u), C.byref(ms_all), b.stream), "ps_time_kernel")
    peak = C.c_double(0)
    _capi.check(L.ps_fma_peak(1 if prec == _capi.PS_PREC_FP64 else 0, C.byref(peak), b.stream), "ps_fma_peak")
    flops = pair_flops(systems)
    achieved = flops / (ms_aa.value * 1e-3) / 1e12 if ms_aa.value > 0 else 0.0
    roof = {"bound": "fp64" if prec == _capi.PS_PREC_FP64 else "fp32", "kernel": "k_rpy_aa",
            "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
            "frac": achieved / peak.value if peak.value else None, "traffic": None,
            "peak_source": "measured in bench.py (FMA microkernel, ps_fma_peak)",
            "flop_per_launch": flops, "ms_per_launch": ms_aa.value, "ms_mobility_apply": ms_all.value}

    if rank == 0:
        cb = cpu_baseline(systems, rtol=args.rtol) if world == 1 else None
        lat_sorted = sorted(lat)
        out = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": t_total / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == _capi.PS_PREC_FP64 else "f32+f64",
               "data": "synthetic",
               "config": {"workload": name, "replicas": len(systems), "beads": beads, "rtol": args.rtol,
                          "precision": args.precision, "solver": args.solver,
                          "l2": "flushed (256 MB write) before every timed step",
                          "parallelism": f"replicas x{world}"},
               "latency_ms": {"p50": lat_sorted[len(lat) // 2], "p99": lat_sorted[min(len(lat) - 1, int(0.99 * len(lat)))]},
               "minres_iters": iters, "minres_iters_note": "per step: max MINRES iterations of the 5 solves, then the Lanczos subspace size", "minres_reason": reasons, "e2e_minres_iters": e2e_iters,
               "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": 8 * 3 * b.ntot,
                       "d2h_bytes_per_step": 8 * 3 * b.ntot},
               "gpu_launches": launches, "roofline": roof, "clocks": clocks, "state_finite": finite}
        if cb:
            out["cpu_baseline"] = cb
        print(json.dumps(out), flush=True)
    b.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_b200(a)
