"""Degenerate replicas in one ragged batch: a two-monomer chain, a lone colloid,
one monomer beside one colloid, and a 14-bead replica with every pair type.
One thermal step with injected noise (dense mobility path, Lanczos square root
exact at these sizes) against the oracle, replica by replica."""
import numpy as np
import pytest
import torch

from oracle import psoracle as po
from polystokes_brownian_b200 import configs
from polystokes_brownian_b200.engine import Batch

pytestmark = pytest.mark.gpu


def _systems():
    out = []
    p = configs.make_params(Nm=2, Nc=0, Npoly=1, Nmono_per_chain=2, beta=0.3, kT=1.0, mm_HI=1, chain_HI=1)
    out.append(configs.System("dimer", p, np.array([[0.0, 0.0, 0.0], [0.5, 0.1, -0.2]])))
    p = configs.make_params(Nm=0, Nc=1, Npoly=0, Nmono_per_chain=1, beta=1.0, kT=1.0, mm_HI=1)
    out.append(configs.System("lone_colloid", p, np.array([[1.0, -2.0, 0.5]])))
    p = configs.make_params(Nm=1, Nc=1, Npoly=1, Nmono_per_chain=1, beta=0.3, kT=1.0, mm_HI=1, chain_HI=1)
    out.append(configs.System("mono_colloid", p, np.array([[3.0, 0.0, 0.0], [0.0, 0.0, 0.0]])))
    out.append(configs.small_mixed(seed=5, Nm_chain=(3, 4), Nc=2, mm_HI=1))
    return out


@pytest.mark.parametrize("solver", [0, 1])
def test_degenerate_replicas_in_a_ragged_batch(solver):
    systems = _systems()
    fbs, wrs, want = [], [], []
    for i, s in enumerate(systems):
        o = po.OracleSim(po.default_params(**s.params), s.x.ravel())
        rng = np.random.default_rng(100 + i)
        fb = rng.normal(size=o.nm3nc11)
        wr = rng.normal(size=o.nm3nc6)
        o.step(fb=fb, wrfd=wr, rtol=1e-13)
        xo, _ = o.state()
        fbs.append(fb)
        wrs.append(wr)
        want.append((s.x.ravel().copy(), xo))
    b = Batch(systems)
    b.step(fb=torch.from_numpy(np.concatenate(fbs)).cuda(), wrfd=torch.from_numpy(np.concatenate(wrs)).cuda(),
           rtol=1e-13, sqrt_kmax=64, sqrt_tol=1e-15, solver=solver)
    xg, _ = b.state()
    for i, s in enumerate(systems):
        x0, xo = want[i]
        xr = b.seg(xg, i, "bead").cpu().numpy()
        assert np.all(np.isfinite(xr)), s.name
        disp = np.linalg.norm(xo - x0)
        assert np.linalg.norm(xr - xo) <= 1e-10 * disp, (s.name, np.linalg.norm(xr - xo), disp)
    b.close()
