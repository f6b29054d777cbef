"""Lubrication (absent from the reference, whose lubdat/*.dat tables are never
read): CPU checks of the oracle's restatement and GPU parity of the device path.

The oracle follows Fiore & Swan, J. Fluid Mech. 878 (2019) 544: the saddle's
lower-right block is -R_lub, the sum over near equal-radius pairs of the table
r2babc.dat (two-body resistance minus the inverted far-field two-body mobility).
GPU tolerances: pair lists bit-exact; operator and diagonal <= 1e-12 relative;
solves at rtol 1e-13 <= 1e-10 relative; one step with injected noise <= 5e-10
relative to the step displacement.
"""
import numpy as np
import pytest

from oracle import psoracle as po
from polystokes_brownian_b200 import configs
from polystokes_brownian_b200.lubdat import load_table


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def with_lub(sysm, gap, bonded=0):
    return configs.System(sysm.name, dict(sysm.params, lub_on=1, lub_gap=gap, lub_bonded=bonded), sysm.x)


CASES = {
    # 64 colloids at volume fraction 0.3 (gaps from 0.01): colloid pairs with rotation coupling
    "colloids": lambda: with_lub(configs.suspension(n=64, phi=0.3, seed=1), 0.5),
    # chains (bond 2.5 beta) and 3 colloids, dense HI: monomer pairs, bonded neighbours included
    "mixed": lambda: with_lub(configs.small_mixed(seed=7, Nm_chain=(3, 6), Nc=3, mm_HI=1, spread=4.0), 1.2, bonded=1),
    # shell path (no monomer HI) with lubricated chain neighbours
    "shell": lambda: with_lub(configs.small_mixed(seed=8, Nm_chain=(4, 5), Nc=2, mm_HI=0, spread=4.0), 1.2, bonded=1),
    # one batched-ensemble replica (chains at contact, 1-2 probes), bonded neighbours skipped
    "ensemble": lambda: with_lub(configs.ensemble_member(np.random.default_rng([0, 160]), 160), 0.5),
}


def oracle_for(sysm, tab=None):
    return po.OracleSim(po.default_params(**sysm.params), sysm.x.ravel(), lub_table=load_table() if tab is None else tab)


# ---------------------------------------------------------------------------
# oracle (CPU)
def test_table_shape_and_packaged_copy(golden_dir):
    import os
    t = load_table()
    g = np.load(os.path.join(golden_dir, "lubdat.npz"))["r2babc"]
    assert np.array_equal(t, g)
    assert t.shape[1] == 11 and np.all(np.diff(t[:, 0]) > 0)
    assert t[0, 0] == pytest.approx(2.1) and t[-1, 0] == pytest.approx(4.0)


@pytest.mark.parametrize("case", list(CASES))
def test_oracle_lub_symmetric_and_pairs(case):
    sysm = CASES[case]()
    o = oracle_for(sysm)
    o.stage()
    pi, pj = o.lub_pairs()
    assert len(pi) > 0
    n6 = o.nm3nc6
    Rl = np.column_stack([o.lub_apply(e) for e in np.eye(n6)])
    assert np.abs(Rl - Rl.T).max() <= 1e-12 * np.abs(Rl).max()
    # the saddle's lower-right block is -R_lub
    n11 = o.nm3nc11
    A = np.column_stack([o.saddle_apply(e) for e in np.eye(o.n)[n11:]]).T
    assert np.allclose(A[:, n11:], -Rl, atol=1e-13 * np.abs(Rl).max())
    d = o.saddle_diag()
    want = np.abs(np.diag(Rl))
    want[want == 0] = 1.0
    assert np.allclose(d[n11:], want, rtol=1e-14)


def test_oracle_lub_bonded_option():
    sysm = CASES["mixed"]()
    o1 = oracle_for(sysm)
    o0 = oracle_for(configs.System(sysm.name, dict(sysm.params, lub_bonded=0), sysm.x))
    a1 = set(zip(*[v.tolist() for v in o1.lub_pairs()]))
    a0 = set(zip(*[v.tolist() for v in o0.lub_pairs()]))
    L = sysm.params["Nmono_per_chain"]
    bonded = {(i, j) for (i, j) in a1 if j < sysm.params["Nm"] and j == i + 1 and i // L == j // L}
    assert bonded and a0 == a1 - bonded


def test_oracle_lub_extrapolation_continuous():
    # below the first table row the singular terms are added to the row's value: continuous at r = 2.1
    t = load_table()
    a = 1.0
    x = np.array([[0.0, 0.0, 0.0], [2.1 + 1e-12, 0.0, 0.0]])
    vals = []
    for r in (2.1 - 1e-9, 2.1 + 1e-9):
        x[1, 0] = r
        p = po.default_params(Nm=0, Nc=2, Npoly=0, Nmono_per_chain=1, beta=a, mm_HI=1, lub_on=1, lub_gap=0.5)
        o = po.OracleSim(p, x.ravel(), lub_table=t)
        o.stage()
        vals.append(np.column_stack([o.lub_apply(e) for e in np.eye(o.nm3nc6)]))
    assert np.abs(vals[0] - vals[1]).max() < 1e-6 * np.abs(vals[1]).max()


def test_oracle_lub_step_noise_changes_only_with_pairs():
    sysm = CASES["mixed"]()
    o1, o2 = oracle_for(sysm), oracle_for(sysm)
    o1.stage()
    np_ = len(o1.lub_pairs()[0])
    rng = np.random.default_rng(0)
    fb = rng.normal(size=o1.nm3nc11)
    wr = rng.normal(size=o1.nm3nc6)
    zl = rng.normal(size=12 * np_)
    a = o1.step(fb=fb, wrfd=wr, zlub=zl, rtol=1e-12)
    b = o2.step(fb=fb, wrfd=wr, zlub=np.zeros_like(zl), rtol=1e-12)
    assert rel(a["up"], b["up"]) > 1e-6          # the lubrication noise enters the velocities
    assert np.all(np.isfinite(a["up"]))


# ---------------------------------------------------------------------------
# device parity
@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
def test_gpu_lub_pairs_and_operator(case):
    import torch
    from polystokes_brownian_b200.engine import Batch
    sysm = CASES[case]()
    o = oracle_for(sysm)
    rhs_o = o.stage()
    b = Batch([sysm])
    rhs_g = b.stage()
    assert rel(rhs_g.cpu().numpy(), rhs_o) < 1e-13
    pi, pj = o.lub_pairs()
    gi, gj = b.pair_list(2)
    assert list(zip(pi.tolist(), pj.tolist())) == list(zip(gi.cpu().tolist(), gj.cpu().tolist()))
    x = np.random.default_rng(9).normal(size=o.n)
    yo = o.saddle_apply(x)
    yg = b.matmult(torch.from_numpy(x).cuda()).cpu().numpy()
    assert rel(yg, yo) < 1e-12, rel(yg, yo)
    n11 = o.nm3nc11
    assert rel(yg[n11:], yo[n11:]) < 1e-12
    assert rel(b.diagonal().cpu().numpy(), o.saddle_diag()) < 1e-13
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("method", [0, 1])
@pytest.mark.parametrize("case", list(CASES))
def test_gpu_lub_solve(case, method):
    import torch
    from polystokes_brownian_b200.engine import Batch
    sysm = CASES[case]()
    o = oracle_for(sysm)
    rhs = o.stage()
    rhs[: o.nm3nc11] += np.random.default_rng(4).normal(size=o.nm3nc11)
    xo, reason_o, _, _ = o.minres(rhs, rtol=1e-13)
    assert reason_o > 0
    b = Batch([sysm])
    b.stage()
    xg, r = b.solve(torch.from_numpy(rhs).cuda(), rtol=1e-13, method=method)
    assert r.reason > 0
    assert rel(xg.cpu().numpy(), xo) < 1e-10, rel(xg.cpu().numpy(), xo)
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("solver", [0, 1])
@pytest.mark.parametrize("case", ["mixed", "shell", "ensemble"])
def test_gpu_lub_step(case, solver):
    import torch
    from polystokes_brownian_b200.engine import Batch
    sysm = CASES[case]()
    o = oracle_for(sysm)
    o.stage()
    npairs = len(o.lub_pairs()[0])
    o = oracle_for(sysm)
    rng = np.random.default_rng(12)
    fb = rng.normal(size=o.nm3nc11)
    wr = rng.normal(size=o.nm3nc6)
    zl = rng.normal(size=12 * npairs)
    x0 = sysm.x.ravel().copy()
    oo = o.step(fb=fb, wrfd=wr, zlub=zl, rtol=1e-13)
    xo, _ = o.state()
    b = Batch([sysm])
    b.step(fb=torch.from_numpy(fb).cuda(), wrfd=torch.from_numpy(wr).cuda(), zlub=torch.from_numpy(zl).cuda(),
           rtol=1e-13, sqrt_kmax=64, sqrt_tol=1e-15, solver=solver)
    xg = b.state()[0].cpu().numpy()
    disp = np.linalg.norm(xo - x0)
    # five solves of a saddle whose condition grows like 1/gap, each stopped at
    # rtol 1e-13 by a different Krylov method: 5e-10 of the step displacement
    assert np.linalg.norm(xg - xo) <= 5e-10 * disp, (np.linalg.norm(xg - xo), disp)
    assert rel(b.step_outputs()["up"].cpu().numpy(), oo["up"]) < 1e-9
    b.close()


@pytest.mark.gpu
def test_gpu_lub_device_noise_runs():
    import torch
    from polystokes_brownian_b200.engine import Batch
    sysm = CASES["colloids"]()
    b = Batch([sysm])
    b.step(rtol=1e-8, solver=1)
    x = b.state()[0].cpu().numpy()
    assert np.all(np.isfinite(x))
    assert np.linalg.norm(x - sysm.x.ravel()) > 0
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("solver", [0, 1])
def test_gpu_lub_step_ragged_batch(solver):
    """Three lubricated replicas in one context with 17, 0 and 27 near pairs (and
    different gap and bonded options): one step with injected noise, each replica
    against its own oracle run, at the single-replica bound."""
    import torch
    from polystokes_brownian_b200.engine import Batch
    systems = [CASES["mixed"](),
               with_lub(configs.small_mixed(seed=5, Nm_chain=(3, 4), Nc=2, mm_HI=1, spread=12.0), 0.5),
               CASES["ensemble"]()]
    fbs, wrs, zls, want = [], [], [], []
    for i, s in enumerate(systems):
        o = oracle_for(s)
        o.stage()
        npairs = len(o.lub_pairs()[0])
        o = oracle_for(s)
        rng = np.random.default_rng(40 + i)
        fb = rng.normal(size=o.nm3nc11)
        wr = rng.normal(size=o.nm3nc6)
        zl = rng.normal(size=12 * npairs)
        o.step(fb=fb, wrfd=wr, zlub=zl, rtol=1e-13)
        fbs.append(fb)
        wrs.append(wr)
        zls.append(zl)
        want.append((s.x.ravel().copy(), o.state()[0]))
    assert [len(z) // 12 for z in zls] == [17, 0, 27]
    b = Batch(systems)
    b.step(fb=torch.from_numpy(np.concatenate(fbs)).cuda(), wrfd=torch.from_numpy(np.concatenate(wrs)).cuda(),
           zlub=torch.from_numpy(np.concatenate(zls)).cuda(), rtol=1e-13, sqrt_kmax=64, sqrt_tol=1e-15,
           solver=solver)
    xg = b.state()[0]
    for i, s in enumerate(systems):
        x0, xo = want[i]
        xr = b.seg(xg, i, "bead").cpu().numpy()
        disp = np.linalg.norm(xo - x0)
        assert np.linalg.norm(xr - xo) <= 5e-10 * disp, (i, np.linalg.norm(xr - xo), disp)
    b.close()
