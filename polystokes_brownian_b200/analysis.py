"""Equilibrium references for the trajectory observables (observe.cu / Batch.observables).

The same theory the reference's thermal test compares its runs against
(test_sim_dumbbells_thermal.py:178-248), restated:

* a harmonic bond V = kbond (r - r0)^2 / 2 has the length density
  P(r) ~ r^2 exp(-V/kT) (the r^2 is the spherical-shell Jacobian);
* a colloid in a 3D harmonic trap V = ktrap |d|^2 / 2 has Gaussian components of
  variance kT/ktrap and the Maxwell radial moments <d> = 2 sqrt(2/pi) sigma,
  std = sqrt(3 - 8/pi) sigma.
"""
from __future__ import annotations

import numpy as np


def bond_length_stats(kbond: float, r0: float, kT: float, n: int = 40000):
    """(mean, mode, std) of the equilibrium bond length."""
    hi = r0 + 8.0 * np.sqrt(kT / kbond) + 3.0
    r = np.linspace(0.0, hi, n)
    w = r ** 2 * np.exp(-0.5 * kbond * (r - r0) ** 2 / kT)
    w /= np.trapezoid(w, r)
    mean = np.trapezoid(r * w, r)
    std = np.sqrt(np.trapezoid((r - mean) ** 2 * w, r))
    return float(mean), float(r[np.argmax(w)]), float(std)


def trap_stats(ktrap: float, kT: float):
    """(sigma, radial mean, radial mode, radial std) in a 3D harmonic trap."""
    sigma = np.sqrt(kT / ktrap)
    return (float(sigma), float(2.0 * np.sqrt(2.0 / np.pi) * sigma), float(np.sqrt(2.0) * sigma),
            float(np.sqrt(3.0 - 8.0 / np.pi) * sigma))


def summarize(obs: dict) -> dict:
    """Pool the per-replica accumulators of Batch.observables() into means."""
    b, t = obs["bond"].sum(0), obs["trap"].sum(0)
    out = {}
    if b[0] > 0:
        out["bond_mean_vector"] = b[1:4] / b[0]
        out["bond_mean_length"] = b[4] / b[0]
        out["bond_length_std"] = float(np.sqrt(max(b[5] / b[0] - (b[4] / b[0]) ** 2, 0.0)))
    if b[6] > 0:
        out["bond_mean_increment"] = b[7:10] / b[6]
    if t[0] > 0:
        out["trap_mean_displacement"] = t[1:4] / t[0]
        out["trap_mean_radius"] = t[4] / t[0]
        out["trap_component_variance"] = t[6:9] / t[0] - (t[1:4] / t[0]) ** 2
    m, n = obs["msd"].sum(0), obs["msd_count"].sum(0).astype(float)
    ok = n > 0
    out["msd"] = np.where(ok[:, None], m / np.maximum(n, 1)[:, None], np.nan)
    return out
