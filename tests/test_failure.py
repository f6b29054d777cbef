"""Failure paths, all made on the host: a solver capped below convergence, non-finite
input, and the module's strict mode.  No test faults or stalls a GPU: a capped solve
is an ordinary bounded loop that reports its reason.

The reference only prints when KSPSolve fails (vel.cpp:45-51) and aborts on PETSc
errors (init.cpp:367); this build returns the KSP reason from ps_ksp_solve / ps_step,
negative PS_ERR_* codes from the C-ABI, and RuntimeError from the module."""
import ctypes as C
import os
import sys

import numpy as np
import pytest
import torch

from polystokes_brownian_b200 import _capi, configs
from polystokes_brownian_b200._capi import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_null_context_rejected_without_gpu():
    L = lib()
    x = np.zeros(3)
    assert L.ps_set_state(None, x.ctypes.data_as(C.c_void_p), None, None) == -1   # PS_ERR_ARG
    assert L.ps_step(None, None, None, None) < 0


@pytest.mark.gpu
def test_capped_minres_reports_negative_reason():
    from polystokes_brownian_b200.engine import Batch
    sysm = configs.small_mixed(seed=1, mm_HI=1)
    b = Batch([sysm])
    rhs = b.stage()
    x, r = b.solve(rhs, rtol=1e-12, maxit=1, method=_capi.PS_SOLVE_MINRES)
    assert r.reason == -3                     # KSP_DIVERGED_ITS
    assert r.iters_max == 1
    assert torch.isfinite(x).all()
    x, r = b.solve(rhs, rtol=1e-12, maxit=100000, method=_capi.PS_SOLVE_MINRES)
    assert r.reason > 0                       # the context is intact afterwards
    b.close()


@pytest.mark.gpu
def test_non_finite_positions_rejected_before_launch():
    from polystokes_brownian_b200.engine import Batch
    sysm = configs.small_mixed(seed=2, mm_HI=1)
    b = Batch([sysm])
    x0, _ = b.state()
    bad = np.ascontiguousarray(sysm.x.ravel().copy())
    bad[7] = np.nan
    rc = lib().ps_set_state(b.h, bad.ctypes.data_as(C.c_void_p), None, b.stream)
    assert rc == -1
    assert b"non-finite position at index 7" in lib().ps_last_error()
    bad[7] = np.inf
    assert lib().ps_set_state(b.h, bad.ctypes.data_as(C.c_void_p), None, b.stream) == -1
    x1, _ = b.state()
    assert torch.equal(x0, x1)                # state untouched
    b.close()


@pytest.mark.gpu
def test_module_strict_raises_on_unconverged_solve(tmp_path):
    sys.path.insert(0, os.path.join(ROOT, "polystokes_brownian_b200", "_lib"))
    import PolyStokes

    sysm = configs.small_mixed(seed=3, mm_HI=1)
    p = sysm.params

    def make(strict, out):
        os.makedirs(out, exist_ok=True)
        sim = PolyStokes.PolyStokes(p["dt"], 1, 3.5 * p["dt"], str(out), mm_HI=True)
        sim.particle_info(p["kT"], p["epsilon"], sysm.Np, p["Nc"], p["Nm"], p["Npoly"], p["Nmono_per_chain"],
                          p["beta"], p["kbond"], p["r0"], p["Lmax"], p["tau"])
        sim.trap_info(p["ktrap"], p["tstart"], p["trun"])
        sim.set_options(solver="minres", rtol=1e-12, maxit=1, strict=strict, aa_mode=1, ab_mode=1)
        sim.initial_configuration(sysm.x.ravel())
        return sim

    with pytest.raises(RuntimeError, match="did not converge"):
        make(True, tmp_path / "strict").run()
    sim = make(False, tmp_path / "lenient")   # the reference's behaviour: report and carry on
    sim.run()
    assert np.all(np.isfinite(np.asarray(sim.positions())))
    with pytest.raises(ValueError):
        sim.set_options(maxit=0)
