"""CPU model of the FP32 monomer far-field kernel's separation scheme: hi-only
separations (positions rounded to float) outside a per-replica exact radius
max(2.1 beta, X / 16), hi + lo separations inside it.  Against an FP64 apply of
the same RPY-form far field the scheme stays within 1.5x of the full hi + lo
difference's error, while hi-only separations everywhere lose more than that
and degrade further as the replica moves away from the origin."""
import numpy as np

from polystokes_brownian_b200 import configs

f32 = np.float32


def _apply(d, u, beta):
    """y_i = sum_j [y(r) u_j + h(r) (d.u_j) d] with the kernel's factored scalars."""
    dt = d.dtype
    c0, c1, c2, c3 = (dt.type(v) for v in (0.75 * beta, 0.5 * beta ** 3, 0.75 * beta, -1.5 * beta ** 3))
    r2 = (d * d).sum(-1, dtype=dt)
    np.fill_diagonal(r2, dt.type(1))
    ri = (dt.type(1) / np.sqrt(r2)).astype(dt)
    np.fill_diagonal(ri, dt.type(0))
    ri2 = ri * ri
    y = ri * (c2 + c3 * ri2)
    h = ri2 * ri * ((c0 - c2) + (c1 - c3) * ri2)
    du = (d * u[None].astype(dt)).sum(-1, dtype=dt)
    return (y[:, :, None] * u[None].astype(dt) + (h * du)[:, :, None] * d).sum(1, dtype=np.float64)


def _errors(shift):
    s = configs.ensemble_member(np.random.default_rng([0, 3]), 512)
    x = s.x[: s.params["Nm"]] + np.asarray(shift)
    beta = s.params["beta"]
    u = np.random.default_rng(1).standard_normal(x.shape)
    truth = _apply(x[:, None, :] - x[None], u, beta)
    hi = x.astype(f32)
    lo = (x - hi.astype(np.float64)).astype(f32)
    d_hi = hi[:, None, :] - hi[None]
    d_ex = d_hi + (lo[:, None, :] - lo[None])
    X = np.abs(x).max()
    te = max(2.1 * beta, X / 16.0)
    inner = ((d_hi * d_hi).sum(-1, dtype=f32) <= f32(te * te))[:, :, None]
    nrm = np.linalg.norm(truth)
    err = {k: np.linalg.norm(_apply(d, u, beta) - truth) / nrm
           for k, d in (("exact", d_ex), ("hi_only", d_hi), ("scheme", np.where(inner, d_ex, d_hi)))}
    return err


def test_exact_radius_keeps_full_difference_accuracy():
    e = _errors([0.0, 0.0, 0.0])
    assert e["exact"] < 2e-7
    assert e["scheme"] < 1.6 * e["exact"]
    assert e["hi_only"] > 1.4 * e["scheme"]


def test_exact_radius_grows_with_distance_from_origin():
    e = _errors([500.0, -250.0, 125.0])
    assert e["scheme"] < 1.6 * e["exact"]
    assert e["hi_only"] > 10 * e["scheme"]
