"""The allocation-free mobility apply (ps_mobility_apply_noalloc) against the
regular context-based entry point (ps_mobility_apply).

ps_mobility_apply_noalloc serves callers that must not allocate device memory
(for example an operator callback run inside a host solver that owns the
device memory pool); it keeps its scratch in a fixed __device__ array.  This
file is named so that pytest collects it last; it must pass both alone in a
fresh process and after every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from polystokes_brownian_b200 import _capi, configs
from polystokes_brownian_b200.engine import Batch

pytestmark = pytest.mark.gpu


def _chains(npoly, nper, seed):
    s = configs.ensemble_member(np.random.default_rng([seed, 7]), npoly * nper)
    p = dict(s.params)
    Nm, nper = p["Nm"], p["Nmono_per_chain"]
    x = s.x[:Nm]
    p.update(Nc=0, ktrap=0.0, aa_mode=0)   # the allocation-free apply uses the reference's scalars
    return configs.System("monomers", p, x)


@pytest.mark.parametrize("chain_HI", [0, 1])
def test_noalloc_matches_context_apply_twice(chain_HI):
    sysm = _chains(12, 40, seed=3)
    sysm.params["chain_HI"] = chain_HI
    N, beta, nper = sysm.params["Nm"], sysm.params["beta"], sysm.params["Nmono_per_chain"]
    L = _capi.lib()
    b = Batch([sysm])
    b.stage()
    x = torch.from_numpy(np.ascontiguousarray(sysm.x.ravel())).cuda()
    st = b.stream
    for call in range(2):   # two calls in a row share (and reuse) the scratch array
        u = torch.randn(3 * N, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(call))
        y_ref = b.mobility_apply(u)
        y = torch.zeros(3 * N, dtype=torch.float64, device="cuda")
        rc = L.ps_mobility_apply_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(u.data_ptr()),
                                        C.c_void_p(y.data_ptr()), N, beta, chain_HI, nper, st)
        assert rc == 0, L.ps_last_error()
        torch.cuda.synchronize()
        err = (torch.linalg.norm(y - y_ref) / torch.linalg.norm(y_ref)).item()
        assert err < 1e-12, (call, err)
    b.close()


def test_noalloc_rejects_oversize():
    L = _capi.lib()
    d = torch.zeros(3, dtype=torch.float64, device="cuda")
    p = C.c_void_p(d.data_ptr())
    rc = L.ps_mobility_apply_noalloc(p, p, p, 8193, 1.0, 0, 1, None)
    assert rc == -6
    assert b"exceeds" in L.ps_last_error()
