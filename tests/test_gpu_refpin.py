"""The CUDA path (through the C-ABI) pinned to the reference's own code.

Fixtures: tests/golden/ref_*.npz, made by the reference's sources compiled
unmodified against the PETSc/SLEPc stand-in (tests/golden/make_ref_fixtures.py).

Tolerances: the saddle operator against the reference's assembled dense matrix
<= 1e-12 relative; MINRES at rtol 1e-13 on the reference's own right-hand sides
<= 1e-10 relative; full steps driven by the reference's noise stream: velocities
<= 1e-10 relative to the reference's solves (RFD difference <= 1e-9), positions
and quaternions <= 2e-10 absolute against its %.10f output files."""
import numpy as np
import pytest
import torch

from polystokes_brownian_b200.engine import Batch
from refpin import ALL, SMALL, RefCase, rel

pytestmark = pytest.mark.gpu


def dense_cases():
    return [n for n in SMALL if RefCase(n).has("A")]


@pytest.mark.parametrize("name", dense_cases())
def test_operator_vs_reference_matrix(name):
    c = RefCase(name)
    b = Batch([c.system])
    rhs = b.stage().cpu().numpy()
    assert rel(rhs, c.d["ksp_rhs"][0]) <= 1e-13
    A = c.d["A"][0]
    rng = np.random.default_rng(3)
    for _ in range(2):
        x = rng.normal(size=c.n)
        y = b.matmult(torch.from_numpy(x).cuda()).cpu().numpy()
        assert rel(y, A @ x) <= 1e-12
    b.close()


@pytest.mark.parametrize("name", ALL)
def test_minres_on_reference_rhs(name):
    """The first step's deterministic solve: the reference's right-hand side, the GPU's
    Jacobi MINRES (the reference's KSPSolve) at rtol 1e-13."""
    c = RefCase(name)
    b = Batch([c.system])
    rhs = b.stage()
    assert rel(rhs.cpu().numpy(), c.d["ksp_rhs"][0]) <= 1e-13
    x, r = b.solve(torch.from_numpy(c.d["ksp_rhs"][0]).cuda(), rtol=1e-13, maxit=100000)
    assert r.reason > 0
    # the replica's saddle system has condition number ~7e3 and takes ~3300 MINRES iterations
    assert rel(x.cpu().numpy(), c.d["ksp_x"][0]) <= (1e-8 if name == "replica1000" else 1e-10)
    b.close()


@pytest.mark.parametrize("name", SMALL)
def test_steps_vs_reference(name):
    c = RefCase(name)
    b = Batch([c.system])
    for k in range(c.steps):
        fb, W = c.noise(k)
        res = b.step(fb=None if fb is None else torch.from_numpy(fb).cuda(),
                     wrfd=None if W is None else torch.from_numpy(W).cuda(),
                     rtol=1e-13, maxit=100000, sqrt_kmax=c.nm3nc11, sqrt_tol=1e-15)
        assert res.reason > 0
        out = {k2: v.cpu().numpy() for k2, v in b.step_outputs().items()}
        v = c.velocities(k)
        assert rel(out["up"], v["up"]) <= 1e-10
        if c.kT > 0:
            assert rel(out["udiff"], v["udiff"]) <= 1e-9
        x, q = b.state()
        assert np.abs(x.cpu().numpy() - c.d["config"][k].ravel()).max() <= 2e-10
        if c.Nc:
            assert np.abs(q.cpu().numpy() - c.d["quats"][k].ravel()).max() <= 2e-10
    b.close()


def test_replica_step_vs_reference():
    """One step of the ~1000-bead replica in the reference's scalars: its MFN root failed
    (indefinite M), so the reference added no slip noise; the GPU gets a zero slip draw
    and the reference's RFD direction."""
    c = RefCase("replica1000")
    b = Batch([c.system])
    fb, W = c.noise(0)
    assert not fb.any()
    res = b.step(fb=torch.from_numpy(fb).cuda(), wrfd=torch.from_numpy(W).cuda(), rtol=1e-13, maxit=100000)
    assert res.reason > 0
    out = {k2: v.cpu().numpy() for k2, v in b.step_outputs().items()}
    v = c.velocities(0)
    assert rel(out["up"], v["up"]) <= 1e-9
    assert rel(out["udiff"], v["udiff"]) <= 1e-8
    x, _ = b.state()
    assert np.abs(x.cpu().numpy() - c.d["config"][0].ravel()).max() <= 2e-10
    b.close()


@pytest.mark.parametrize("name", SMALL)
def test_module_run_vs_reference_files(name, tmp_path, monkeypatch):
    """The drop-in module (PolyStokes over the C-ABI) against the reference module on the same
    inputs and seed: same output file names, and the same contents to the printed 10 decimals
    (the module draws the reference's mt19937_64 noise stream itself)."""
    import os
    import sys

    lib = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "polystokes_brownian_b200", "_lib")
    sys.path.insert(0, lib)
    import PolyStokes

    c = RefCase(name)
    p = c.params
    monkeypatch.setenv("POLYSTOKES_LANCZOS_NC", str(p["lanczos_nc"]))
    sim = PolyStokes.PolyStokes(p["dt"], 1, (c.steps + 0.5) * p["dt"], str(tmp_path), mm_HI=bool(p["mm_HI"]),
                                chain_HI=bool(p["chain_HI"]), fene=bool(p["fene"]), record_forces=True,
                                seed=int(c.d["seed"]))
    sim.particle_info(c.kT, p["epsilon"], c.Nm + c.Nc, c.Nc, c.Nm, p["Npoly"], p["Nmono_per_chain"], p["beta"],
                      p["kbond"], p["r0"], p["Lmax"], p["tau"])
    sim.trap_info(p["ktrap"], p["tstart"], p["trun"])
    sim.set_options(rtol=1e-13, sqrt_kmax=c.nm3nc11, sqrt_tol=1e-15)
    sim.initial_configuration(np.ascontiguousarray(c.x0.ravel()))
    sim.set_warn_neg_eig(False)
    sim.run()
    for pre in ("config", "quats", "force", "brownian_stresslet"):
        names = list(c.d[pre + "_names"])
        for k, nm in enumerate(names):
            got = np.loadtxt(os.path.join(str(tmp_path), nm), ndmin=2)
            assert got.shape == c.d[pre][k].shape, (pre, nm)
            assert np.abs(got - c.d[pre][k]).max() <= 3e-10, (pre, nm)
