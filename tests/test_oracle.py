"""CPU checks of the oracle (oracle/psoracle.c) itself: pinned against the
reference's own mob.csv dump, plus algebraic properties the reference relies on
(symmetric grand mobility, saddle solve, square-root consistency, pair sets)."""
import os

import numpy as np
import pytest

from oracle import psoracle as po
from polystokes_brownian_b200 import configs


def oracle_for(sysm, **over):
    p = dict(sysm.params)
    p.update(over)
    return po.OracleSim(po.default_params(**p), sysm.x.ravel())


# ---------------------------------------------------------------------------
# mob.csv pin
def test_mobcsv_pin(golden_dir):
    g = np.load(os.path.join(golden_dir, "mobcsv.npz"))
    M, x = g["M"], g["x"]
    Nm, Nc, beta = int(g["Nm"]), int(g["Nc"]), float(g["beta"])
    p = po.default_params(Nm=Nm, Nc=Nc, Npoly=11, Nmono_per_chain=3, beta=beta, mm_HI=0)
    s = po.OracleSim(p, x.ravel())
    s.check_dist()
    s.mob()                      # no Schur floor: mob.csv holds the raw M
    Mo = s.dense_mobility()
    nm3, nc3 = 3 * Nm, 3 * Nc
    mask = np.ones_like(M, dtype=bool)
    mask[nm3:nm3 + nc3, :nm3] = False     # AB translation block: older formula in mob.csv
    mask[:nm3, nm3:nm3 + nc3] = False
    err = np.abs(Mo - M)[mask].max()
    assert err < 1e-13, err
    # the AB translation block of mob.csv follows X = 1/r - b^2/(2r^3), Y = 1/(2r) - b^2/(4r^3)
    for m in range(Nm):
        for c in range(Nc):
            d = x[m] - x[Nm + c]
            r = np.linalg.norm(d)
            e = d / r
            X = 1 / r - beta ** 2 / (2 * r ** 3)
            Y = 0.5 / r - beta ** 2 / (4 * r ** 3)
            T = X * np.outer(e, e) + Y * (np.eye(3) - np.outer(e, e))
            assert np.abs(M[nm3 + 3 * c:nm3 + 3 * c + 3, 3 * m:3 * m + 3] - T).max() < 1e-12


def test_reference_ab_translation_is_zero_in_shell_path(golden_dir):
    g = np.load(os.path.join(golden_dir, "mobcsv.npz"))
    p = po.default_params(Nm=33, Nc=2, Npoly=11, Nmono_per_chain=3, beta=0.1, mm_HI=0)
    s = po.OracleSim(p, g["x"].ravel())
    s.stage()
    assert np.all(s.mcm()[:6] == 0.0)


# ---------------------------------------------------------------------------
@pytest.mark.parametrize("mm_HI,ab_mode,chain_HI", [(1, 0, 0), (1, 0, 1), (1, 1, 0), (0, 0, 0), (0, 1, 0)])
def test_dense_symmetric_and_matfree(mm_HI, ab_mode, chain_HI):
    sysm = configs.small_mixed(seed=1, mm_HI=mm_HI, chain_HI=chain_HI, ab_mode=ab_mode)
    s = oracle_for(sysm)
    s.stage()
    M = s.dense_mobility()
    assert np.abs(M - M.T).max() < 1e-13 * np.abs(M).max()
    u = np.random.default_rng(0).normal(size=M.shape[0])
    assert np.allclose(s.mobility_apply(u), M @ u, rtol=1e-13, atol=1e-13)


def test_stale_ab_block_is_last_aa_pair():
    sysm = configs.small_mixed(seed=2, mm_HI=1)
    s = oracle_for(sysm)
    s.stage()
    Nm = sysm.params["Nm"]
    d = sysm.x[Nm - 2] - sysm.x[Nm - 1]
    r = np.linalg.norm(d)
    T = po.tensor_aa(d / r, r, sysm.params["beta"], 0).reshape(3, 3)
    assert np.allclose(s.stale_a(), T, rtol=0, atol=1e-15)


def test_bb_rotation_block_quirk():
    # the reference places +mob_b(e12) in both [r1,t2] and [r2,t1] (mob.cpp:1051-1078)
    sysm = configs.small_mixed(seed=3, Nm_chain=(0, 0), Nc=2, mm_HI=1)
    s = oracle_for(sysm)
    s.stage()
    M = s.dense_mobility()
    t1, t2, r1, r2 = 0, 3, 6, 9
    assert np.allclose(M[r1:r1 + 3, t2:t2 + 3], M[r2:r2 + 3, t1:t1 + 3], atol=1e-15)


def test_saddle_solve_and_jacobi():
    sysm = configs.small_mixed(seed=4, mm_HI=1)
    s = oracle_for(sysm)
    b = s.stage()
    b[: s.nm3nc11] += np.random.default_rng(1).normal(size=s.nm3nc11)
    x, reason, it, rn = s.minres(b, rtol=1e-12)
    assert reason > 0
    A = np.column_stack([s.saddle_apply(e) for e in np.eye(s.n)])
    assert np.abs(A - A.T).max() < 1e-12
    assert np.linalg.norm(A @ x - b) <= 1e-9 * np.linalg.norm(b)
    d = s.saddle_diag()
    assert np.all(d[s.nm3nc11:] == 1.0)


def test_sqrt_paths_agree():
    sysm = configs.small_mixed(seed=5, mm_HI=1, spread=9.0)
    s = oracle_for(sysm)
    s.stage()
    M = s.dense_mobility()
    lam = np.linalg.eigvalsh(M)
    z = np.random.default_rng(2).normal(size=M.shape[0])
    w_eig = po.sqrtm_eig(M, z)
    if lam.min() > 0:
        w_np = np.linalg.cholesky(M)  # SPD: the symmetric root squares back to M
        W = np.column_stack([po.sqrtm_eig(M, e) for e in np.eye(M.shape[0])])
        assert np.allclose(W @ W, M, atol=1e-10)
        del w_np
    w_lz, m = s.lanczos_sqrt(z, kmax=M.shape[0], tol=1e-13)
    assert np.linalg.norm(w_lz - w_eig) <= 1e-8 * np.linalg.norm(w_eig)


def test_shell_noise_covariance():
    sysm = configs.polymer_probe(seed=0)
    s = oracle_for(sysm)
    s.stage()
    n11 = s.nm3nc11
    W = np.column_stack([s.slip_noise(e) for e in np.eye(n11)])   # W = L, cov = L L^T
    M = s.dense_mobility()
    C = W @ W.T
    # block-Cholesky with the Schur floor reproduces M with Mcc_block (floored) exactly
    assert np.allclose(C, M, atol=1e-10)


def test_cell_pairs_match_reference_grid():
    sysm = configs.polymer_probe(seed=1)
    s = oracle_for(sysm, mono_ev=1)
    s.stage()
    a, b = s.cell_pairs()
    # every pair within the WCA cutoff whose reference cells are adjacent
    x = sysm.x[:220]
    d = np.linalg.norm(x[:, None] - x[None], axis=2)
    rc = np.float32(2 ** (1 / 6) * np.float64(np.float32(2 / 3)))
    brute = {(i, j) for i in range(220) for j in range(i + 1, 220) if d[i, j] ** 2 < float(rc) ** 2}
    got = {(min(i, j), max(i, j)) for i, j in zip(a, b)}
    assert got <= brute
    assert len(got) == len(a)


def test_step_kT0_deterministic_and_finite():
    sysm = configs.small_mixed(seed=6, mm_HI=1, kT=0.0)
    s1, s2 = oracle_for(sysm), oracle_for(sysm)
    o1 = s1.step(rtol=1e-10)
    o2 = s2.step(rtol=1e-10)
    x1, _ = s1.state()
    x2, _ = s2.state()
    assert np.array_equal(x1, x2)
    assert np.all(np.isfinite(x1))
    assert np.allclose(o1["v_brown"], 0.0)


def test_step_with_noise_runs():
    sysm = configs.polymer_probe(seed=2)
    s = oracle_for(sysm)
    rng = np.random.default_rng(3)
    o = s.step(fb=rng.normal(size=s.nm3nc11), wrfd=rng.normal(size=s.nm3nc6), rtol=1e-10)
    x, q = s.state()
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(o["udiff"]))
    assert np.allclose(np.linalg.norm(q.reshape(-1, 4), axis=1), 1.0)
    assert all(i > 0 for i in o["iters"])


# ---------------------------------------------------------------------------
# regularised unequal-radii monomer-colloid coupling (ab_mode 2)
def overlapping_system(ab_mode):
    """One colloid, chains around it; monomer 0 overlaps the colloid (r = 1.1),
    monomer 5 sits inside it (r = 0.5); beta = 0.3."""
    sysm = configs.small_mixed(seed=12, Nm_chain=(3, 4), Nc=1, mm_HI=1, aa_mode=1, ab_mode=ab_mode)
    x = sysm.x.copy()
    c = x[-1]
    x[0] = c + np.array([1.1, 0.0, 0.0])
    x[5] = c + np.array([0.0, 0.5, 0.0])
    return configs.System(sysm.name, sysm.params, x)


def test_ab_regularised_scalars_continuous():
    for beta in (0.2, 1.0 / 3.0, 0.5):
        for rb, eps in ((1 + beta, 1e-9), (1 - beta, 1e-9)):
            lo = np.array(po.ab_reg_scalars(rb - eps, beta))
            hi = np.array(po.ab_reg_scalars(rb + eps, beta))
            assert np.abs(lo - hi).max() < 1e-7
        # far field: the PS_AB_RPY scalars
        r = 3.0
        x, y, yb = po.ab_reg_scalars(r, beta)
        assert x == pytest.approx(1.5 / r - 0.5 * (1 + beta ** 2) / r ** 3)
        assert y == pytest.approx(0.75 / r + 0.25 * (1 + beta ** 2) / r ** 3)
        assert yb == pytest.approx(-0.75 / r ** 2)
        # engulfed: the colloid's self mobility
        assert po.ab_reg_scalars(0.3 * (1 - beta), beta)[:2] == (1.0, 1.0)


def test_ab_regularised_keeps_force_torque_mobility_definite():
    # the translation / rotation block (forces and torques -> velocities): the far-field
    # 1/r^k terms make it indefinite once a monomer penetrates the colloid; the
    # regularised branches keep it positive definite.  The stresslet coupling stays
    # far-field, as in the reference (mob.cpp:455-470), so the full FTS matrix is not.
    lam = {}
    for mode in (1, 2):
        s = oracle_for(overlapping_system(mode))
        s.stage()
        M = s.dense_mobility()
        assert np.abs(M - M.T).max() < 1e-13 * np.abs(M).max()
        n6 = s.nm3nc6
        lam[mode] = np.linalg.eigvalsh(M[:n6, :n6]).min()
    assert lam[1] < 0 < lam[2]
