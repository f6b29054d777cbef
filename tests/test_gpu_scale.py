"""Parity of the CUDA path against the CPU oracle at the benchmark sizes:
the 1024-colloid lubricated suspension, the 4097-bead brush and the largest
replica of the 256-replica lubricated ensemble (N about 4000).

At these sizes the oracle's own Jacobi MINRES would need hours, so a solve is
checked by a size-independent property instead: the FP64 structured solve at
rtol 1e-13 is put through the oracle's saddle operator, and its residual must
be at the solve's tolerance.

Tolerances: FP64 operator applies <= 1e-12 relative (as at the small sizes);
structured solve residual through the oracle's operator <= 1e-9 relative (the
near-contact suspension's saddle operator is ill-conditioned, so a preconditioned
rtol of 1e-13 leaves a larger true residual).
"""
import numpy as np
import pytest
import torch

from oracle import psoracle as po
from polystokes_brownian_b200 import configs
from polystokes_brownian_b200.engine import Batch
from polystokes_brownian_b200.lubdat import load_table

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def suspension_lub():
    s = configs.suspension(seed=0)
    return configs.System(s.name, dict(s.params, lub_on=1, lub_gap=0.5), s.x)


def largest_ensemble_replica():
    systems = configs.ensemble(256, seed=0, lub=True)
    return max(systems, key=lambda s: s.Np)


CASES = {
    "C2_suspension1024_lub": suspension_lub,
    "C3_brush4097": lambda: configs.brush(seed=0),
    "C4_largest_replica": largest_ensemble_replica,
}


def oracle_for(sysm):
    tab = load_table() if sysm.params.get("lub_on") else None
    return po.OracleSim(po.default_params(**sysm.params), sysm.x.ravel(), lub_table=tab)


@pytest.mark.parametrize("case", list(CASES))
def test_operator_parity_full_size(case):
    sysm = CASES[case]()
    o = oracle_for(sysm)
    rhs_o = o.stage()
    b = Batch([sysm])
    rhs_g = b.stage()
    assert rel(rhs_g.cpu().numpy(), rhs_o) < 1e-13
    x = np.random.default_rng(11).normal(size=o.n)
    assert rel(b.matmult(torch.from_numpy(x).cuda()).cpu().numpy(), o.saddle_apply(x)) < 1e-12
    u = x[: o.nm3nc11].copy()
    assert rel(b.mobility_apply(torch.from_numpy(u).cuda()).cpu().numpy(), o.mobility_apply(u)) < 1e-12
    b.close()


@pytest.mark.parametrize("case", list(CASES))
def test_structured_solve_residual_full_size(case):
    sysm = CASES[case]()
    o = oracle_for(sysm)
    rhs = o.stage()
    rhs[: o.nm3nc11] += np.random.default_rng(5).normal(size=o.nm3nc11)
    b = Batch([sysm])
    b.stage()
    x, res = b.solve(torch.from_numpy(rhs).cuda(), rtol=1e-13, maxit=20000, method=1)
    assert res.reason > 0
    r = np.linalg.norm(rhs - o.saddle_apply(x.cpu().numpy())) / np.linalg.norm(rhs)
    assert r < 1e-9, r
    b.close()
