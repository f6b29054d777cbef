"""Run the reference's own module (oracle/_ref/PolyStokes, built from its sources by
``make -C oracle ref``) on one system and time its step.

TEST INFRASTRUCTURE ONLY: the timed CPU leg of bench.py (``--impl reference`` and
the ``cpu_baseline`` entry).  The reference keeps its state in globals (one
simulation per process), so every call runs in a fresh worker process.
"""
from __future__ import annotations

import ctypes
import glob
import io
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REFDIR = os.path.join(HERE, "_ref")


def available() -> bool:
    return bool(glob.glob(os.path.join(REFDIR, "PolyStokes*.so")))


def step_seconds(params: dict, x, rtol: float, seed: int = 0, nsteps: int = 1):
    """(N, seconds per step, saddle iterations unknown) of the reference's run() loop for one
    system: the module's own init() and fill_self() are excluded (the clock starts at
    the first check_dist() of step 1).  MINRES runs at `rtol` (the reference hard-codes
    1e-6, init.cpp:64; the stand-in's ORACLE_KSP_RTOL sets it)."""
    os.environ["ORACLE_KSP_RTOL"] = repr(float(rtol))
    if REFDIR not in sys.path:
        sys.path.insert(0, REFDIR)
    import PolyStokes as R   # noqa: N814  the reference's module

    so = glob.glob(os.path.join(REFDIR, "PolyStokes*.so"))[0]
    first = ctypes.CDLL(so).refshim_first_event_time
    first.restype = ctypes.c_double
    p = params
    Np = p["Nm"] + p["Nc"]
    out = io.StringIO()
    with tempfile.TemporaryDirectory() as td:
        sim = R.PolyStokes(p["dt"], 10 ** 9, (nsteps + 0.5) * p["dt"], td, mm_HI=bool(p["mm_HI"]),
                           chain_HI=bool(p["chain_HI"]), fene=bool(p["fene"]), record_forces=False, seed=seed)
        old = sys.stdout
        sys.stdout = out
        try:
            sim.particle_info(p["kT"], p["epsilon"], Np, p["Nc"], p["Nm"], p["Npoly"], p["Nmono_per_chain"],
                              p["beta"], p["kbond"], p["r0"], p["Lmax"], p["tau"])
            sim.trap_info(p["ktrap"], p["tstart"], p["trun"])
            sim.initial_configuration(x)
            sim.set_warn_neg_eig(False)
            sim.run()
            t_end = time.monotonic()
        finally:
            sys.stdout = old
    return Np, (t_end - first()) / nsteps
