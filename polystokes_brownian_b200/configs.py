"""Seeded synthetic systems in the reference's units.

The reference fixes the colloid radius to 1 and the monomer radius to beta
(src/mob.cpp:400-401): positions, r0, Lmax and box lengths are divided by the
colloid radius a_c, and spring constants are multiplied by a_c**2 (energies
stay in kT).  Initial configurations follow the style of the reference's own
scenario builders (seeded numpy RNG, rejection sampling, test_sim.py /
test_sim_dumbbells_thermal.py): chains are self-avoiding random walks whose
beads keep at least the contact distance from every bead already placed.

Workloads (sizes as stated in the benchmark definition):
  polymer_probe   2 probes (a_c = 3) + 11 chains x 20 beads, shell path
  suspension      1024 colloids, volume fraction 0.2, spherical cluster
  brush           1 colloid (a_c = 5) + 128 chains x 32 beads, full HI
  ensemble        256 replicas, N log-uniform in [64, 4096], full HI
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class System:
    name: str
    params: dict          # ps_desc / or_params fields
    x: np.ndarray         # (Np, 3) float64, monomers first then colloids

    @property
    def Np(self):
        return self.params["Nm"] + self.params["Nc"]


DEFAULTS = dict(Nm=0, Nc=0, Npoly=0, Nmono_per_chain=1, beta=1.0, kT=1.0, epsilon=1.0, kbond=1.0,
                r0=1.0, Lmax=10.0, tau=1000.0, dt=1e-3, mm_HI=1, chain_HI=0, fene=0, tether=0,
                mono_ev=0, record_forces=1, box_on=0, ktrap=0.0, tstart=0.0, trun=0.0, weaken_trap=-1.0,
                t0=0.0, restart=0, ab_mode=0, hs_kpref=1.0, hs_kmode=0, lanczos_nc=64, lub_on=0, lub_gap=0.5,
                aa_mode=0, lub_bonded=0)


def make_params(**kw) -> dict:
    p = dict(DEFAULTS)
    p.update(kw)
    return p


class _Grid:
    """Spatial hash for overlap rejection: small beads in a grid of edge h,
    the few large ones (radius > h/2) in a plain list."""

    def __init__(self, h):
        self.h = h
        self.cells: dict = {}
        self.big: list = []

    def key(self, p):
        return (int(math.floor(p[0] / self.h)), int(math.floor(p[1] / self.h)), int(math.floor(p[2] / self.h)))

    def add(self, p, rad):
        p = np.asarray(p, dtype=float)
        if 2 * rad > self.h:
            self.big.append((p, rad))
        else:
            self.cells.setdefault(self.key(p), []).append((float(p[0]), float(p[1]), float(p[2]), rad))

    def clear(self, p, rad, reach=None):
        for q, rq in self.big:
            d = p - q
            if d @ d < (rad + rq) ** 2:
                return False
        kx, ky, kz = self.key(p)
        n = int(math.ceil(2 * rad / self.h))
        px, py, pz = float(p[0]), float(p[1]), float(p[2])
        for dx in range(-n, n + 1):
            for dy in range(-n, n + 1):
                for dz in range(-n, n + 1):
                    for qx, qy, qz, rq in self.cells.get((kx + dx, ky + dy, kz + dz), ()):
                        ex, ey, ez = px - qx, py - qy, pz - qz
                        if ex * ex + ey * ey + ez * ez < (rad + rq) ** 2:
                            return False
        return True


def _unit(rng):
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


def _chains(rng, npoly, nper, beta, step, colloids, start_fn, grid, bound=None, max_try=50):
    """Self-avoiding random walks; start_fn(rng, chain) gives the first bead."""
    beads = []
    reach = 2.0 + 2 * beta
    for c in range(npoly):
        prev = None
        for k in range(nper):
            for attempt in range(max_try):
                if k == 0:
                    p, direction = start_fn(rng, c)
                else:
                    direction = _unit(rng)
                    if k >= 2 and attempt < max_try // 2:
                        # bias away from the previous bond reversal
                        direction = direction + 0.5 * (prev - beads[-2])
                        direction /= np.linalg.norm(direction)
                    p = prev + step * direction
                if bound is not None and np.linalg.norm(p) > bound:
                    continue
                if grid.clear(p, beta, reach) or attempt == max_try - 1:
                    break
            grid.add(p, beta)
            beads.append(p)
            prev = p
    return np.array(beads).reshape(-1, 3)


def polymer_probe(seed: int = 0) -> System:
    """2 probes of radius 3 + 11 harmonic chains x 20 beads of radius 1 (a_c = 3)."""
    rng = np.random.default_rng(seed)
    ac = 3.0
    beta = 1.0 / ac
    colloids = np.array([[10.0, 0, 0], [-10.0, 0, 0]]) / ac
    grid = _Grid(2 * beta)
    for c in colloids:
        grid.add(c, 1.0)
    step = 2.0 / ac

    def start(rng, c):
        while True:
            p = rng.uniform(-30, 30, size=3) / ac
            if grid.clear(p, beta, 2.0 + 2 * beta):
                return p, None

    xm = _chains(rng, 11, 20, beta, step, colloids, start, grid)
    params = make_params(Nm=220, Nc=2, Npoly=11, Nmono_per_chain=20, beta=beta, kT=1.0, kbond=100 * ac * ac,
                         r0=step, Lmax=10 * step, dt=1e-3, mm_HI=0, chain_HI=1, fene=0, ktrap=500 * ac * ac,
                         tstart=0.0, trun=0.5)
    return System("polymer_probe", params, np.vstack([xm, colloids]))


def suspension(n: int = 1024, phi: float = 0.2, seed: int = 0, gap: float = 0.01) -> System:
    """n equal colloids of radius 1 uniformly in a sphere at volume fraction phi."""
    rng = np.random.default_rng(seed)
    R = (n / phi) ** (1.0 / 3.0)
    grid = _Grid(2.0)
    pts = []
    while len(pts) < n:
        p = rng.uniform(-R, R, size=3)
        if p @ p > (R - 1.0) ** 2:
            continue
        if grid.clear(p, 1.0 + gap / 2, 2.0 + gap):
            grid.add(p, 1.0 + gap / 2)
            pts.append(p)
    params = make_params(Nm=0, Nc=n, Npoly=0, Nmono_per_chain=1, beta=1.0, kT=1.0, dt=1e-4, mm_HI=1)
    return System("suspension", params, np.array(pts))


def brush(nchain: int = 128, nper: int = 32, seed: int = 0, dt: float = 1e-4, pair_mode: int = 1) -> System:
    """1 colloid (a_c = 5) with nchain chains of nper beads grown outward from its surface.

    Each chain starts just outside the colloid on a uniformly random direction (the first
    beads of this dense brush cannot all touch the surface: up to 0.4 further out), and the
    chains grow together, one layer of beads at a time, by steps of 2.2 beta whose direction
    mixes the outward radial direction with a random one: every bead stays farther from the
    centre than the previous one of its chain and is placed where it overlaps no bead
    placed before (the outward weight grows on each rejected try).  At 128 chains the grafting is dense
    (about 0.15 of surface per chain), so the chains are stretched, as in a brush.

    The chains are free (tether=0): the reference tethers with the chain's own
    FENE r0/Lmax (init.cpp:308-317, rhs.cpp:110-121), which is singular for a
    graft distance (1 + beta) larger than Lmax = 0.6."""
    rng = np.random.default_rng(seed)
    ac = 5.0
    beta = 1.0 / ac
    grid = _Grid(2 * beta)
    grid.add(np.zeros(3), 1.0)
    step = 2.2 * beta
    # layer by layer: every chain's first bead, then every chain's second bead, ...
    chains = np.zeros((nchain, nper, 3))
    for c in range(nchain):
        # graft direction uniform on the sphere; the first bead sits just off the surface, pushed
        # out by up to 0.4 where the dense first layer has no room at contact
        for attempt in range(4000):
            p = _unit(rng) * (1.0 + beta + 0.05 + 0.4 * min(1.0, attempt / 2000.0) * rng.random())
            if grid.clear(p, beta, 2.0 + 2 * beta):
                break
        grid.add(p, beta)
        chains[c, 0] = p
    for k in range(1, nper):
        for c in range(nchain):
            prev = chains[c, k - 1]
            rad = prev / np.linalg.norm(prev)
            for attempt in range(2000):
                w = min(1.0, 0.35 + attempt / 400.0)
                d = w * rad + (1.0 - w) * _unit(rng)
                d /= np.linalg.norm(d)
                q = prev + step * d
                if np.linalg.norm(q) > np.linalg.norm(prev) and grid.clear(q, beta, 2.0 + 2 * beta):
                    break
            grid.add(q, beta)
            chains[c, k] = q
    beads = list(chains.reshape(-1, 3))
    xm = np.array(beads).reshape(-1, 3)
    params = make_params(Nm=nchain * nper, Nc=1, Npoly=nchain, Nmono_per_chain=nper, beta=beta, kT=1.0,
                         kbond=30 * ac * ac, r0=step, Lmax=3.0 / ac, fene=1, dt=dt, mm_HI=1, chain_HI=0,
                         aa_mode=pair_mode, ab_mode=pair_mode)
    return System("brush", params, np.vstack([xm, np.zeros((1, 3))]))


def ensemble_member(rng, N: int, beta: float = 1.0 / 3.0, dt: float = 1e-4, pair_mode: int = 1,
                    lub: bool = False, lub_gap: float = 0.5) -> System:
    """One batched-ensemble replica: harmonic chains + 0..2 trapped probes.

    lub: near-field lubrication for equal-radius pairs with gap < lub_gap * a;
    bonded chain neighbours (held at contact by their springs) are not lubricated.

    pair_mode 1 (default) uses the RPY monomer-monomer and monomer-colloid
    scalars; with the reference's own scalars (pair_mode 0) the grand mobility is
    indefinite and the explicit predictor-corrector diverges within a few steps.
    dt defaults to 1e-4: at 1e-3 the stated spring constants (kbond = 900,
    mobility up to ~40) exceed the explicit integrator's stability limit."""
    nprobe = int(rng.integers(0, 3))
    L = int(rng.integers(16, 65))
    npoly = max(1, int(round((N - nprobe) / L)))
    Nm = npoly * L
    phi = float(rng.uniform(0.05, 0.2))
    vol = 4.0 / 3.0 * math.pi * (Nm * beta ** 3 + nprobe)
    R = (vol / phi) ** (1.0 / 3.0)
    grid = _Grid(2 * beta)
    colloids = []
    for c in range(nprobe):
        while True:
            p = rng.uniform(-R, R, size=3) * 0.6
            if grid.clear(p, 1.0, 2.0):
                grid.add(p, 1.0)
                colloids.append(p)
                break
    step = 2.0 * beta

    def start(rng, c):
        while True:
            p = rng.uniform(-R, R, size=3)
            if p @ p < R * R and grid.clear(p, beta, 2.0 + 2 * beta):
                return p, None

    xm = _chains(rng, npoly, L, beta, step, None, start, grid, bound=R * 1.5)
    x = np.vstack([xm] + ([np.array(colloids)] if colloids else []))
    params = make_params(Nm=Nm, Nc=nprobe, Npoly=npoly, Nmono_per_chain=L, beta=beta, kT=1.0,
                         kbond=900.0, r0=step, Lmax=10 * step, dt=dt, mm_HI=1, chain_HI=0, fene=0,
                         ktrap=4500.0 if nprobe else 0.0, tstart=0.0, trun=1e9, aa_mode=pair_mode,
                         ab_mode=pair_mode, lub_on=int(lub), lub_gap=lub_gap)
    return System(f"ensemble_{N}", params, x)


def dumbbells(seed: int = 0, n_db: int = 4, beta: float = 0.3, r0: float = 1.2, kbond: float = 25.0,
              ktrap: float = 50.0, dt: float = 1e-3, mm_HI: int = 1) -> System:
    """One trapped colloid at the origin and n_db harmonic dumbbells (two monomers
    of radius beta at their rest length r0) around it, the setting of the
    reference's thermal test (test_sim_dumbbells_thermal.py).  RPY pair scalars,
    so the grand mobility is positive definite and the noise exact."""
    rng = np.random.default_rng(seed)
    grid = _Grid(2 * beta)
    grid.add(np.zeros(3), 1.0)
    xs = []
    while len(xs) < 2 * n_db:
        c = rng.uniform(-6.0, 6.0, size=3)
        if c @ c < 9.0:
            continue
        u = _unit(rng)
        p0, p1 = c - 0.5 * r0 * u, c + 0.5 * r0 * u
        if grid.clear(p0, beta, 2.5 * beta) and grid.clear(p1, beta, 2.5 * beta):
            grid.add(p0, beta)
            grid.add(p1, beta)
            xs += [p0, p1]
    x = np.vstack([np.array(xs), np.zeros((1, 3))])
    params = make_params(Nm=2 * n_db, Nc=1, Npoly=n_db, Nmono_per_chain=2, beta=beta, kT=1.0, kbond=kbond, r0=r0,
                         Lmax=10 * r0, dt=dt, mm_HI=mm_HI, chain_HI=0, fene=0, ktrap=ktrap, tstart=0.0, trun=1e9,
                         aa_mode=1, ab_mode=1)
    return System("dumbbells", params, x)


def ensemble(n_rep: int = 256, seed: int = 0, nmin: int = 64, nmax: int = 4096, **kw) -> list[System]:
    rng = np.random.default_rng(seed)
    Ns = np.rint(np.exp(rng.uniform(math.log(nmin), math.log(nmax), size=n_rep))).astype(int)
    return [ensemble_member(np.random.default_rng([seed, i]), int(N), **kw) for i, N in enumerate(Ns)]


def small_mixed(seed: int = 0, Nm_chain=(3, 4), Nc: int = 3, mm_HI: int = 1, beta: float = 0.3,
                spread: float = 6.0, **kw) -> System:
    """A small system with every pair type (AA, AB, BB), well separated, for parity tests."""
    rng = np.random.default_rng(seed)
    npoly, nper = Nm_chain
    grid = _Grid(2 * beta)
    colloids = []
    while len(colloids) < Nc:
        p = rng.uniform(-spread, spread, size=3)
        if grid.clear(p, 1.0, 2.5):
            grid.add(p, 1.25)
            colloids.append(p)
    step = 2.5 * beta

    def start(rng, c):
        while True:
            p = rng.uniform(-spread, spread, size=3)
            if grid.clear(p, beta, 3.0):
                return p, None

    xm = _chains(rng, npoly, nper, beta, step, None, start, grid) if npoly * nper else np.zeros((0, 3))
    x = np.vstack([xm] + ([np.array(colloids)] if Nc else []))
    p = dict(Nm=npoly * nper, Nc=Nc, Npoly=npoly, Nmono_per_chain=nper if npoly else 1, beta=beta,
             kT=1.0, kbond=50.0, r0=step, Lmax=3 * step, dt=1e-3, mm_HI=mm_HI, chain_HI=0,
             ktrap=20.0 if Nc else 0.0, tstart=0.0, trun=10.0)
    p.update(kw)
    return System("small_mixed", make_params(**p), x)
