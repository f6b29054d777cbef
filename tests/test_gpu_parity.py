"""Parity of the CUDA path (through the C-ABI) against the CPU oracle.

Tolerances: FP64 operator applies <= 1e-12 relative; solves at rtol 1e-13 in both
<= 1e-10 relative; pair sets bit-exact; one full step with injected noise
<= 1e-10 relative to the step displacement.
"""
import numpy as np
import pytest
import torch

from oracle import psoracle as po
from polystokes_brownian_b200 import configs
from polystokes_brownian_b200.engine import Batch

pytestmark = pytest.mark.gpu


def oracle_for(sysm):
    return po.OracleSim(po.default_params(**sysm.params), sysm.x.ravel())


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


CASES = {
    "shell_C1": lambda: configs.polymer_probe(seed=0),
    "mmhi_mixed": lambda: configs.small_mixed(seed=1, mm_HI=1),
    "mmhi_chain": lambda: configs.small_mixed(seed=2, mm_HI=1, chain_HI=1),
    "mmhi_rpy": lambda: configs.small_mixed(seed=3, mm_HI=1, ab_mode=1),
    "shell_rpy": lambda: configs.small_mixed(seed=4, mm_HI=0, ab_mode=1),
    "colloids": lambda: configs.suspension(n=96, phi=0.1, seed=0),
    "brush_small": lambda: configs.brush(nchain=8, nper=8, seed=0),
    # regularised unequal-radii monomer-colloid coupling, one monomer overlapping, one inside the colloid
    "rpy_reg_overlap": lambda: __import__("test_oracle").overlapping_system(2),
}


@pytest.mark.parametrize("case", list(CASES))
def test_operator_parity(case):
    sysm = CASES[case]()
    o = oracle_for(sysm)
    rhs_o = o.stage()
    b = Batch([sysm])
    rhs_g = b.stage()
    assert rel(rhs_g.cpu().numpy(), rhs_o) < 1e-13
    x = np.random.default_rng(7).normal(size=o.n)
    yo = o.saddle_apply(x)
    yg = b.matmult(torch.from_numpy(x).cuda()).cpu().numpy()
    assert rel(yg, yo) < 1e-12, rel(yg, yo)
    u = x[: o.nm3nc11].copy()
    assert rel(b.mobility_apply(torch.from_numpy(u).cuda()).cpu().numpy(), o.mobility_apply(u)) < 1e-12
    assert rel(b.diagonal().cpu().numpy(), o.saddle_diag()) < 1e-13
    b.close()


@pytest.mark.parametrize("case", ["shell_C1", "mmhi_mixed", "colloids", "brush_small"])
def test_minres_parity(case):
    sysm = CASES[case]()
    o = oracle_for(sysm)
    rhs = o.stage()
    rhs[: o.nm3nc11] += np.random.default_rng(3).normal(size=o.nm3nc11)
    xo, reason_o, it_o, _ = o.minres(rhs, rtol=1e-13)
    b = Batch([sysm])
    b.stage()
    xg, r = b.solve(torch.from_numpy(rhs).cuda(), rtol=1e-13)
    assert r.reason > 0
    assert rel(xg.cpu().numpy(), xo) < 1e-10, rel(xg.cpu().numpy(), xo)
    assert abs(r.iters_max - it_o) <= max(2, it_o // 10)
    # warm start from the solution converges immediately
    xw, r2 = b.solve(torch.from_numpy(rhs).cuda(), x0=xg, rtol=1e-8)
    assert r2.iters_max <= 2
    b.close()


@pytest.mark.parametrize("case", ["shell_C1", "mmhi_mixed", "colloids", "brush_small", "mmhi_rpy", "rpy_reg_overlap"])
def test_structured_solve_parity(case):
    """Exact block elimination of the constraint (PS_SOLVE_STRUCTURED) against the
    oracle's MINRES at rtol 1e-13; the colloid case (96 colloids) exercises the
    warm-started MINRES polish beyond the dense stresslet limit."""
    sysm = CASES[case]()
    o = oracle_for(sysm)
    rhs = o.stage()
    rhs[: o.nm3nc11] += np.random.default_rng(5).normal(size=o.nm3nc11)
    xo, _, _, _ = o.minres(rhs, rtol=1e-13)
    b = Batch([sysm])
    b.stage()
    xg, r = b.solve(torch.from_numpy(rhs).cuda(), rtol=1e-13, method=1)
    assert r.reason > 0
    assert rel(xg.cpu().numpy(), xo) < 1e-10, rel(xg.cpu().numpy(), xo)
    b.close()


@pytest.mark.parametrize("case", ["shell_C1", "mmhi_mixed", "brush_small"])
def test_pair_lists_bitexact(case):
    sysm = CASES[case]()
    o = po.OracleSim(po.default_params(**dict(sysm.params, mono_ev=1)), sysm.x.ravel())
    o.stage()
    b = Batch([configs.System(sysm.name, dict(sysm.params, mono_ev=1), sysm.x)])
    b.stage()
    vi, vj = o.verlet_pairs()
    gi, gj = b.pair_list(0)
    assert sorted(zip(vi.tolist(), vj.tolist())) == list(zip(gi.cpu().tolist(), gj.cpu().tolist()))
    if not sysm.params["mm_HI"]:
        ci, cj = o.cell_pairs()
        want = sorted((min(a, c), max(a, c)) for a, c in zip(ci.tolist(), cj.tolist()))
        wi, wj = b.pair_list(1)
        assert want == list(zip(wi.cpu().tolist(), wj.cpu().tolist()))
    b.close()


def test_sqrt_parity_dense_and_shell():
    # dense (mm_HI) path: Lanczos vs the exact eigen square root with negative
    # eigenvalues floored at 0.  With 58 DOFs the Krylov space is exhausted at
    # kmax = 64, so the projected floor equals the floor on M itself.
    sysm = configs.small_mixed(seed=5, Nm_chain=(3, 4), Nc=2, mm_HI=1)
    o = oracle_for(sysm)
    o.stage()
    M = o.dense_mobility()
    assert M.shape[0] <= 64
    z = np.random.default_rng(2).normal(size=M.shape[0])
    b = Batch([sysm])
    b.stage()
    w, r = b.sqrtm(torch.from_numpy(z).cuda(), kmax=64, tol=1e-14)
    assert rel(w.cpu().numpy(), po.sqrtm_eig(M, z)) < 1e-10
    b.close()
    # shell path: block-Cholesky with the Schur floor
    sysm = configs.polymer_probe(seed=0)
    o = oracle_for(sysm)
    o.stage()
    z = np.random.default_rng(4).normal(size=o.nm3nc11)
    b = Batch([sysm])
    b.stage()
    w, _ = b.sqrtm(torch.from_numpy(z).cuda())
    assert rel(w.cpu().numpy(), o.slip_noise(z)) < 1e-12
    b.close()


STEP_CASES = {
    # shell path: block-Cholesky noise, Schur floor, two colloids
    "shell_C1": lambda: configs.polymer_probe(seed=0),
    # dense path with noise: 58 mobility DOFs, so the Lanczos square root is exact
    "mmhi_noise": lambda: configs.small_mixed(seed=5, Nm_chain=(3, 4), Nc=2, mm_HI=1),
    # dense path, deterministic (kT = 0), FENE chains around a colloid
    "brush_kT0": lambda: configs.System("brush", dict(configs.brush(nchain=8, nper=8, seed=0).params, kT=0.0),
                                        configs.brush(nchain=8, nper=8, seed=0).x),
    # shell path above the dense Schur limit: 8 colloids (nc11 = 88 > 64), Schur Lanczos noise
    "shell_lanczos8": lambda: configs.small_mixed(seed=6, Nm_chain=(4, 6), Nc=8, mm_HI=0, spread=12.0),
}


@pytest.mark.parametrize("solver", [0, 1])
@pytest.mark.parametrize("case", list(STEP_CASES))
def test_step_parity(case, solver):
    sysm = STEP_CASES[case]()
    o = oracle_for(sysm)
    rng = np.random.default_rng(11)
    fb = rng.normal(size=o.nm3nc11)
    wr = rng.normal(size=o.nm3nc6)
    x0 = sysm.x.ravel().copy()
    oo = o.step(fb=fb, wrfd=wr, rtol=1e-13)
    xo, qo = o.state()
    b = Batch([sysm])
    b.step(fb=torch.from_numpy(fb).cuda(), wrfd=torch.from_numpy(wr).cuda(), rtol=1e-13, sqrt_kmax=64,
           sqrt_tol=1e-15, solver=solver)
    xg, qg = b.state()
    xg = xg.cpu().numpy()
    disp = np.linalg.norm(xo - x0)
    assert np.linalg.norm(xg - xo) <= 1e-10 * max(disp, 1e-30), (np.linalg.norm(xg - xo), disp)
    if sysm.params["Nc"]:
        assert np.abs(qg.cpu().numpy() - qo).max() < 1e-12
    outs = b.step_outputs()
    if sysm.params["kT"] > 0:
        assert rel(outs["udiff"].cpu().numpy(), oo["udiff"]) < 1e-8
    b.close()


@pytest.mark.parametrize("lnc", [64, 0])
def test_schur_lanczos_noise(lnc):
    """Shell-path slip noise through the Schur Lanczos branch (slip_vel.cpp:351-477): 8
    colloids (nc11 = 88 above the crossover of 64), or the crossover set to 0, which sends
    every shell replica there (the reference's POLYSTOKES_LANCZOS_NC=0)."""
    sysm = configs.small_mixed(seed=6, Nm_chain=(4, 6), Nc=8 if lnc else 2, mm_HI=0, spread=12.0, lanczos_nc=lnc)
    o = oracle_for(sysm)
    o.stage()
    z = np.random.default_rng(8).normal(size=o.nm3nc11)
    b = Batch([sysm])
    b.stage()
    w, r = b.sqrtm(torch.from_numpy(z).cuda())
    assert rel(w.cpu().numpy(), o.slip_noise(z)) < 1e-10
    b.close()


def test_batch_matches_single():
    systems = [CASES["mmhi_mixed"](), CASES["colloids"](), CASES["shell_C1"]()]
    xs = [np.random.default_rng(i).normal(size=6 * s.params["Nm"] + 17 * s.params["Nc"]) for i, s in enumerate(systems)]
    b = Batch(systems)
    b.stage()
    yb = b.matmult(torch.from_numpy(np.concatenate(xs)).cuda()).cpu().numpy()
    for i, s in enumerate(systems):
        one = Batch([s])
        one.stage()
        y1 = one.matmult(torch.from_numpy(xs[i]).cuda()).cpu().numpy()
        o = b.off[i]["vec"]
        assert rel(yb[o:o + len(xs[i])], y1) < 1e-13
        one.close()
    b.close()


def test_hs_partner_overflow():
    """Monomers piled inside one Verlet radius (about 99 hard-sphere partners each, beyond
    the 64 gathered in registers): the forces still take every partner, in ascending order,
    as the oracle's Verlet sweep does."""
    rng = np.random.default_rng(5)
    Nm = 100
    x = rng.uniform(-0.15, 0.15, size=(Nm, 3))
    p = configs.make_params(Nm=Nm, Nc=0, Npoly=20, Nmono_per_chain=5, beta=0.3, kT=0.0, kbond=10.0, r0=0.1,
                            Lmax=1.0, mm_HI=1, mono_ev=1)
    sysm = configs.System("pile", p, x)
    o = oracle_for(sysm)
    rhs_o = o.stage()
    pi, pj = o.verlet_pairs()
    assert np.bincount(np.concatenate([pi, pj]), minlength=Nm).min() > 64
    b = Batch([sysm])
    rhs_g = b.stage().cpu().numpy()
    assert rel(rhs_g, rhs_o) < 1e-13
    b.close()


def test_fp64_pair_rsqrt_within_two_ulp():
    """The FP64 pair kernel's reciprocal square root (single-precision seed, second-order
    binomial correction) against CUDA's rsqrt: at most 2 units in the last place over
    squared separations from 1e-8 to 1e12."""
    import ctypes as C
    from polystokes_brownian_b200 import _capi
    rng = np.random.default_rng(0)
    a = np.concatenate([10.0 ** rng.uniform(-8, 12, size=1 << 20), [1.0, 4.0, 0.25, 2.0, 3.0, 1e-8, 1e12]])
    d = torch.from_numpy(a).cuda()
    worst = C.c_uint64(0)
    rc = _capi.lib().ps_rsqrt_check(C.c_void_p(d.data_ptr()), C.c_int64(a.size), C.byref(worst), None)
    assert rc == 0
    assert worst.value <= 2, worst.value
