"""The allocation-free mobility apply (ps_mobility_apply_noalloc) against the
regular context-based entry point (ps_mobility_apply) and the CPU oracle's FP64
mobility apply.

ps_mobility_apply_noalloc serves callers that must not allocate device memory
(for example an operator callback run inside a host solver that owns the
device memory pool); it keeps its scratch in a fixed __device__ array.  This
file is named so that pytest collects it last; it must pass both alone in a
fresh process and after every other test.

Tolerance: 1e-12 relative, as for every FP64 operator apply.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import psoracle as po
from polystokes_brownian_b200 import _capi, configs
from polystokes_brownian_b200.engine import Batch

pytestmark = pytest.mark.gpu

MAX_BEADS = 8192


def monomers(npoly, nper, seed, beta=1.0 / 3.0, chain_HI=0):
    """npoly chains of nper monomers (random walks of step 2 beta from random starts);
    overlaps are allowed, both sides evaluate the overlap branch of the pair scalars."""
    rng = np.random.default_rng(seed)
    N = npoly * nper
    box = 2.0 * (N * beta ** 3 / 0.05) ** (1.0 / 3.0)
    x = np.empty((N, 3))
    for c in range(npoly):
        steps = rng.normal(size=(nper, 3))
        steps *= 2 * beta / np.linalg.norm(steps, axis=1, keepdims=True)
        steps[0] = rng.uniform(-box, box, size=3)
        x[c * nper:(c + 1) * nper] = np.cumsum(steps, axis=0)
    p = configs.make_params(Nm=N, Nc=0, Npoly=npoly, Nmono_per_chain=nper, beta=beta, kT=0.0, mm_HI=1,
                            chain_HI=chain_HI, aa_mode=0)   # the allocation-free apply uses the reference's scalars
    return configs.System("monomers", p, x)


def noalloc_apply(sysm, u, stream=None):
    L = _capi.lib()
    p = sysm.params
    N = p["Nm"]
    x = torch.from_numpy(np.ascontiguousarray(sysm.x.ravel())).cuda()
    y = torch.zeros(3 * N, dtype=torch.float64, device="cuda")
    rc = L.ps_mobility_apply_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(u.data_ptr()), C.c_void_p(y.data_ptr()),
                                    N, p["beta"], p["chain_HI"], p["Nmono_per_chain"], stream)
    assert rc == 0, L.ps_last_error()
    torch.cuda.synchronize()
    return y


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("chain_HI", [0, 1])
def test_noalloc_matches_context_apply_and_oracle_twice(chain_HI):
    sysm = monomers(12, 40, seed=3, chain_HI=chain_HI)
    N = sysm.params["Nm"]
    b = Batch([sysm])
    b.stage()
    o = po.OracleSim(po.default_params(**sysm.params), sysm.x.ravel())
    o.stage()
    for call in range(2):   # two calls in a row share (and reuse) the scratch array
        u = torch.randn(3 * N, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(call))
        y = noalloc_apply(sysm, u, b.stream).cpu().numpy()
        assert rel(y, b.mobility_apply(u).cpu().numpy()) < 1e-12, call
        assert rel(y, o.mobility_apply(u.cpu().numpy())) < 1e-12, call
    b.close()


def test_noalloc_near_the_size_limit():
    """N = 8190 (195 chains of 42; not a multiple of the 128-row tile), near the 8192 limit,
    against the oracle's FP64 apply."""
    sysm = monomers(195, 42, seed=5, chain_HI=1)
    N = sysm.params["Nm"]
    assert MAX_BEADS - 128 < N <= MAX_BEADS and N % 128
    o = po.OracleSim(po.default_params(**sysm.params), sysm.x.ravel())
    o.stage()
    u = np.random.default_rng(9).normal(size=3 * N)
    y = noalloc_apply(sysm, torch.from_numpy(u).cuda()).cpu().numpy()
    assert rel(y, o.mobility_apply(u)) < 1e-12


def test_noalloc_rejects_oversize():
    L = _capi.lib()
    d = torch.zeros(3, dtype=torch.float64, device="cuda")
    p = C.c_void_p(d.data_ptr())
    rc = L.ps_mobility_apply_noalloc(p, p, p, MAX_BEADS + 1, 1.0, 0, 1, None)
    assert rc == -6
    assert b"exceeds" in L.ps_last_error()
