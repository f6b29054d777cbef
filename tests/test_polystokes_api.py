"""The reference's Python API (pybind11 module `PolyStokes`, src/bindings.cpp:41-119)
over the B200 engine: class and argument names, defaults, the Box utility, the
output files of write_configuration.cpp:10-166 and restart (Stokes.cpp:19-34,
init.cpp initial_configuration).

GPU runs compare a deterministic (kT = 0) trajectory against the oracle step
for step (<= 1e-9 relative to the displacement, solves at rtol 1e-12)."""
import glob
import os
import sys

import numpy as np
import pytest

from oracle import psoracle as po
from polystokes_brownian_b200 import configs

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "polystokes_brownian_b200", "_lib")
sys.path.insert(0, LIB)
PolyStokes = pytest.importorskip("PolyStokes")


def make_sim(sysm, out, samplerate=2, nsteps=5, seed=12345, restart=0.0, **kw):
    p = sysm.params
    tmax = restart + nsteps * p["dt"] + 0.5 * p["dt"]
    sim = PolyStokes.PolyStokes(p["dt"], samplerate, tmax, str(out), mm_HI=bool(p["mm_HI"]),
                                chain_HI=bool(p["chain_HI"]), fene=bool(p["fene"]), record_forces=True,
                                seed=seed, restart=restart, **kw)
    sim.particle_info(p["kT"], p["epsilon"], sysm.Np, p["Nc"], p["Nm"], p["Npoly"], p["Nmono_per_chain"], p["beta"],
                      p["kbond"], p["r0"], p["Lmax"], p["tau"])
    sim.trap_info(p["ktrap"], p["tstart"], p["trun"])
    return sim


def test_box_utility():
    b = PolyStokes.Box()
    assert not b.active()
    assert b.minimum_image(7.0, -8.0, 1.0) == (7.0, -8.0, 1.0)
    b.configure([10.0, 10.0, 4.0])
    assert b.active()
    dx, dy, dz = b.minimum_image(7.0, -8.0, 3.0)
    assert (dx, dy, dz) == (-3.0, 2.0, -1.0)
    assert b.wrap(12.0, 0.5, -2.5) == (2.0, 0.5, 1.5)
    b.configure([])
    assert not b.active()
    with pytest.raises(ValueError):
        b.configure([1.0, 2.0])
    with pytest.raises(ValueError):
        b.configure([1.0, -2.0, 3.0])


def test_signature_defaults_and_checks(tmp_path, capfd):
    sysm = configs.small_mixed(seed=1, mm_HI=1)
    sim = PolyStokes.PolyStokes(1e-3, 10, 0.01, str(tmp_path))
    with pytest.raises(RuntimeError):
        sim.initial_configuration(sysm.x.ravel())          # particle_info first
    p = sysm.params
    with pytest.raises(RuntimeError):
        sim.particle_info(1.0, 1.0, sysm.Np + 1, p["Nc"], p["Nm"], p["Npoly"], p["Nmono_per_chain"], p["beta"],
                          1.0, 1.0, 10.0, 1000.0)
    sim = make_sim(sysm, tmp_path)
    with pytest.raises(RuntimeError):
        sim.initial_configuration(np.zeros(5))
    sim.initial_configuration(sysm.x.ravel())
    sim.set_warn_neg_eig(False)
    with pytest.raises(ValueError):
        sim.set_options(precision="fp16")
    out = capfd.readouterr().out
    assert "kT: 1" in out and "Nmono_per_chain: 4" in out


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-GPU error path")
def test_run_without_gpu_raises(tmp_path):
    sysm = configs.small_mixed(seed=1, mm_HI=1)
    sim = make_sim(sysm, tmp_path)
    sim.initial_configuration(sysm.x.ravel())
    with pytest.raises(RuntimeError):
        sim.run()


def _read(path):
    rows = [ln.rstrip("\n").split("\t") for ln in open(path)]
    for r in rows:
        for v in r:
            assert len(v.split(".")[1]) == 10, v         # %.10f
    return np.array(rows, dtype=float)


@pytest.mark.gpu
def test_run_kT0_matches_oracle_and_writes_files(tmp_path):
    base = configs.small_mixed(seed=2, mm_HI=1, aa_mode=1, ab_mode=1)
    sysm = configs.System(base.name, dict(base.params, kT=0.0), base.x)
    sim = make_sim(sysm, tmp_path, samplerate=2, nsteps=5)
    sim.set_options(rtol=1e-12, ab_mode=1, aa_mode=1)
    sim.initial_configuration(sysm.x.ravel())
    sim.run()
    o = po.OracleSim(po.default_params(**sysm.params), sysm.x.ravel())
    x0 = sysm.x.ravel().copy()
    for _ in range(5):
        o.step(rtol=1e-12)
    xo, qo = o.state()
    xg = np.asarray(sim.positions())
    assert np.linalg.norm(xg - xo) <= 1e-9 * np.linalg.norm(xo - x0)
    names = sorted(os.path.basename(f) for f in glob.glob(str(tmp_path / "*.txt")))
    # samples after steps 1, 3, 5 (i == 0 or i % samplerate == 0), time as std::ostream prints it
    want = []
    for t in ("0.001", "0.003", "0.005"):
        want += [f"config_{t}_.txt", f"quats_{t}_.txt", f"force_{t}_.txt", f"brownian_stresslet_{t}_.txt"]
    assert names == sorted(want)
    c = _read(tmp_path / "config_0.005_.txt")
    assert c.shape == (sysm.Np, 3)
    assert np.abs(c.ravel() - xo).max() < 1e-9
    assert _read(tmp_path / "quats_0.005_.txt").shape == (sysm.params["Nc"], 4)
    assert _read(tmp_path / "force_0.005_.txt").shape == (sysm.Np + sysm.params["Nc"], 3)
    assert _read(tmp_path / "brownian_stresslet_0.005_.txt").shape == (sysm.params["Nc"], 5)


@pytest.mark.gpu
def test_seeded_noise_reproducible(tmp_path):
    sysm = configs.small_mixed(seed=3, mm_HI=1, aa_mode=1, ab_mode=1)
    xs = []
    for k, seed in enumerate((7, 7, 8)):
        d = tmp_path / str(k)
        d.mkdir()
        sim = make_sim(sysm, d, samplerate=100, nsteps=3, seed=seed)
        sim.set_options(ab_mode=1, aa_mode=1)
        sim.initial_configuration(sysm.x.ravel())
        sim.run()
        xs.append(np.asarray(sim.positions()))
    assert np.array_equal(xs[0], xs[1])
    assert not np.allclose(xs[0], xs[2])


@pytest.mark.gpu
def test_restart_continues_trajectory(tmp_path):
    # chains only (no trap centre to carry), kT = 0: 6 steps == 3 steps + restart for 3 steps,
    # up to the 10 decimals of the configuration file
    base = configs.small_mixed(seed=4, Nc=0, mm_HI=1, aa_mode=1, ab_mode=1)
    sysm = configs.System(base.name, dict(base.params, kT=0.0), base.x)
    full = make_sim(sysm, tmp_path / "full", nsteps=6)
    os.makedirs(tmp_path / "full")
    full.set_options(rtol=1e-12, ab_mode=1, aa_mode=1)
    full.initial_configuration(sysm.x.ravel())
    full.run()
    os.makedirs(tmp_path / "a")
    a = make_sim(sysm, tmp_path / "a", samplerate=1, nsteps=3)
    a.set_options(rtol=1e-12, ab_mode=1, aa_mode=1)
    a.initial_configuration(sysm.x.ravel())
    a.run()
    x3 = _read(tmp_path / "a" / "config_0.003_.txt").ravel()
    os.makedirs(tmp_path / "b")
    b = make_sim(sysm, tmp_path / "b", samplerate=1, nsteps=3, restart=0.003)
    b.set_options(rtol=1e-12, ab_mode=1, aa_mode=1)
    b.initial_configuration(x3)
    b.run()
    assert os.path.exists(tmp_path / "b" / "config_0.006_.txt")
    xf, xb = np.asarray(full.positions()), np.asarray(b.positions())
    assert np.abs(xf - xb).max() < 1e-8
