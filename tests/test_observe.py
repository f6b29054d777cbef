"""Trajectory observables on the device (observe.cu): exact agreement of every
accumulator with numpy on the recorded states, and thermal equilibrium of a
trapped colloid with dumbbells against the theory the reference's thermal test
uses (test_sim_dumbbells_thermal.py:178-248): the bond-length moments and the
trap variance kT/ktrap."""
import numpy as np
import pytest

from polystokes_brownian_b200 import analysis, configs


def test_theory_limits():
    # a stiff bond at r0 -> 0 is the trap: the same radial law
    sigma, rmean, rmode, rstd = analysis.trap_stats(1e4, 1.0)
    m, mo, sd = analysis.bond_length_stats(1e4, 0.0, 1.0)
    assert m == pytest.approx(rmean, rel=1e-4) and sd == pytest.approx(rstd, rel=1e-3)
    # a stiff bond at r0 > 0 sits at r0
    m, mo, sd = analysis.bond_length_stats(1e6, 1.0, 1.0)
    assert m == pytest.approx(1.0, abs=1e-5)


def _expected(systems, frames, nbins, bmax, tmax, lags):
    R = len(systems)
    out = {"bond": np.zeros((R, 10)), "bond_hist": np.zeros((R, nbins), np.uint64), "trap": np.zeros((R, 9)),
           "trap_hist": np.zeros((R, nbins), np.uint64), "msd": np.zeros((R, lags, 6)),
           "msd_count": np.zeros((R, lags), np.uint64)}
    for r, s in enumerate(systems):
        p = s.params
        Nm, Nc, L = p["Nm"], p["Nc"], p["Nmono_per_chain"]
        bonds = [(c * L + j, c * L + j + 1) for c in range(p["Npoly"]) for j in range(L - 1)]
        xs = [f[r] for f in frames]
        prev = None
        for n, x in enumerate(xs):
            v = np.array([x[j] - x[i] for i, j in bonds]).reshape(-1, 3)
            ln = np.linalg.norm(v, axis=1)
            out["bond"][r, 0] += len(bonds)
            out["bond"][r, 1:4] += v.sum(0)
            out["bond"][r, 4] += ln.sum()
            out["bond"][r, 5] += (ln ** 2).sum()
            if prev is not None:
                out["bond"][r, 6] += len(bonds)
                out["bond"][r, 7:10] += (v - prev).sum(0)
            prev = v
            for l in ln:
                bn = int(l / bmax * nbins)
                if 0 <= bn < nbins:
                    out["bond_hist"][r, bn] += 1
            d = x[Nm:] - s.x[Nm:]
            dn = np.linalg.norm(d, axis=1)
            out["trap"][r, 0] += Nc
            out["trap"][r, 1:4] += d.sum(0)
            out["trap"][r, 4] += dn.sum()
            out["trap"][r, 5] += (dn ** 2).sum()
            out["trap"][r, 6:9] += (d ** 2).sum(0)
            for l in dn:
                bn = int(l / tmax * nbins)
                if 0 <= bn < nbins:
                    out["trap_hist"][r, bn] += 1
            for lag in range(min(n, lags - 1) + 1):
                dd = x[Nm:] - xs[n - lag][Nm:]
                out["msd"][r, lag] += np.stack([dd[:, 0] ** 2, dd[:, 1] ** 2, dd[:, 2] ** 2, dd[:, 0] * dd[:, 1],
                                                dd[:, 0] * dd[:, 2], dd[:, 1] * dd[:, 2]], 1).sum(0)
                out["msd_count"][r, lag] += Nc
    return out


@pytest.mark.gpu
def test_observables_match_numpy():
    from polystokes_brownian_b200.engine import Batch
    systems = [configs.dumbbells(seed=1, n_db=3), configs.small_mixed(seed=2, mm_HI=1, aa_mode=1, ab_mode=1),
               configs.polymer_probe(seed=0)]
    b = Batch(systems)
    nbins, bmax, tmax, lags = 32, 3.0, 1.0, 4
    b.obs_reset(nbins, bmax, tmax, lags)
    frames = []
    for _ in range(6):
        b.step(rtol=1e-8, solver=1)
        b.observe()
        x = b.state()[0].cpu().numpy()
        frames.append([x[3 * b.off[r]["bead"]:3 * (b.off[r]["bead"] + s.Np)].reshape(-1, 3)
                       for r, s in enumerate(systems)])
    got = b.observables()
    want = _expected(systems, frames, nbins, bmax, tmax, lags)
    for k in ("bond", "trap", "msd"):
        assert np.allclose(got[k], want[k], rtol=1e-12, atol=1e-12), k
    for k in ("bond_hist", "trap_hist", "msd_count"):
        assert np.array_equal(got[k], want[k]), k
    b.close()


@pytest.mark.gpu
def test_thermal_equilibrium_dumbbells_and_trap():
    from polystokes_brownian_b200.engine import Batch
    systems = [configs.dumbbells(seed=100 + i, n_db=4) for i in range(64)]
    p = systems[0].params
    b = Batch(systems)
    b.set_seed(7)
    for _ in range(200):
        b.step(rtol=1e-8, solver=1)
    b.obs_reset(64, 3.0, 1.0, 8)
    for k in range(1000):
        b.step(rtol=1e-8, solver=1)
        if k % 5 == 4:
            b.observe()
    s = analysis.summarize(b.observables())
    b.close()
    mean, _, std = analysis.bond_length_stats(p["kbond"], p["r0"], p["kT"])
    nb = 64 * 4 * 200
    assert abs(s["bond_mean_length"] - mean) < 5 * std / np.sqrt(nb / 2), (s["bond_mean_length"], mean)
    assert s["bond_length_std"] == pytest.approx(std, rel=0.05)
    # isotropy: bond-vector components fluctuate with |b|/sqrt(3) and decorrelate on
    # the dumbbell's rotational time (about 100 steps here): ~10 orientations per dumbbell
    assert np.all(np.abs(s["bond_mean_vector"]) < 5 * (p["r0"] / np.sqrt(3)) / np.sqrt(64 * 4 * 10))
    sigma2 = p["kT"] / p["ktrap"]
    assert np.allclose(s["trap_component_variance"], sigma2, rtol=0.15), (s["trap_component_variance"], sigma2)
