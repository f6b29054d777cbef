"""Continuous-batching request loop (polystokes_brownian_b200/serve.py).

CPU: trace generation, footprint-based admission bookkeeping.
GPU: every trajectory's result is the same alone and in the mix -- the kernels
are per-replica deterministic (column chunking, segmented reductions, Philox
streams keyed by the replica's own seed and step), so the bar is bit-identity.
"""
import numpy as np
import pytest

from polystokes_brownian_b200 import _capi, serve


def small_trace(seed=0, lub=False):
    tr = serve.make_trace(6, rate=50.0, seed=seed, nmin=64, nmax=400, smin=3, smax=9, lub=lub)
    return tr


def test_trace_is_seeded_and_sorted():
    a, b = small_trace(1), small_trace(1)
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert all(np.array_equal(x.system.x, y.system.x) for x, y in zip(a, b))
    assert all(a[i].arrival <= a[i + 1].arrival for i in range(len(a) - 1))
    assert len({r.seed for r in a}) == len(a)
    for r in a:
        assert 3 <= r.steps <= 9 and 64 <= r.system.Np <= 460


def test_footprint_grows_with_beads():
    from polystokes_brownian_b200 import configs
    fp = [serve.footprint_bytes(configs.small_mixed(seed=0, Nm_chain=(k, 8), Nc=2, spread=20.0)) for k in (2, 4, 8)]
    assert fp[0] < fp[1] < fp[2]
    # the Lanczos basis dominates: at least (kmax + 1) mobility vectors per replica
    s = configs.small_mixed(seed=0, Nm_chain=(8, 8), Nc=2, spread=20.0)
    assert fp[2] >= 8 * 65 * (3 * 64 + 22)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,lub,rebuild", [(_capi.PS_PREC_FP64, False, 1), (_capi.PS_PREC_MIXED, False, 3),
                                                   (_capi.PS_PREC_MIXED, True, 2)])
def test_alone_equals_mixed(precision, lub, rebuild):
    trace = small_trace(3, lub=lub)
    mixed = serve.Server(precision=precision, rebuild_every=rebuild).run(trace, clock="virtual")
    assert [r.rid for r in mixed] == [r.rid for r in trace]
    for req in (trace[0], trace[3], trace[5]):
        alone_req = serve.Request(req.rid, req.system, req.steps, req.seed, 0.0)
        alone = serve.Server(precision=precision).run([alone_req], clock="virtual")[0]
        got = mixed[req.rid]
        assert got.steps == req.steps
        assert np.all(np.isfinite(alone.x))
        assert np.array_equal(alone.x, got.x), np.abs(alone.x - got.x).max()
        assert np.array_equal(alone.q, got.q)


@pytest.mark.gpu
def test_admission_respects_budget():
    trace = small_trace(4)
    one = max(serve.footprint_bytes(r.system) for r in trace)
    srv = serve.Server(budget_bytes=1.5 * one, rebuild_every=1)
    res = srv.run(trace, clock="virtual")
    assert len(res) == len(trace)
    assert max(srv.batch_sizes) <= 2


def test_oversize_request_refused():
    """A request whose footprint alone is beyond the HBM budget gets an error result; the
    loop never builds a context for it (host only, runs without a GPU)."""
    trace = small_trace(5)[:1]
    fp = serve.footprint_bytes(trace[0].system)
    srv = serve.Server(budget_bytes=0.5 * fp)
    res = srv.run(trace, clock="virtual")
    assert len(res) == 1 and res[0].error is not None and "budget" in res[0].error
    assert res[0].x.size == 0 and srv.rebuilds == 0


@pytest.mark.gpu
def test_mixed_kT_trace():
    """kT = 0 and kT > 0 requests in one trace run in two contexts side by side; each
    trajectory equals its run alone."""
    from polystokes_brownian_b200 import configs
    trace = small_trace(6)
    r1 = trace[1]
    cold = configs.System(r1.system.name, dict(r1.system.params, kT=0.0), r1.system.x)
    trace[1] = serve.Request(r1.rid, cold, r1.steps, r1.seed, r1.arrival)
    mixed = serve.Server(precision=_capi.PS_PREC_FP64, rebuild_every=1).run(trace, clock="virtual")
    assert [r.rid for r in mixed] == [r.rid for r in trace] and all(r.error is None for r in mixed)
    for req in (trace[0], trace[1]):
        alone = serve.Server(precision=_capi.PS_PREC_FP64).run(
            [serve.Request(req.rid, req.system, req.steps, req.seed, 0.0)], clock="virtual")[0]
        assert np.array_equal(alone.x, mixed[req.rid].x)
