"""Mixed precision (FP32 far-field pair kernels with compensated cross-tile sums,
FP64 combine and Krylov) against the FP64 path: relative error <= 1e-6 on the
operator and on the structured solve's velocities."""
import numpy as np
import pytest
import torch

from polystokes_brownian_b200 import configs
from polystokes_brownian_b200.engine import Batch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()


@pytest.mark.parametrize("n_rep", [1, 6])
def test_mixed_operator_and_solve_error(n_rep):
    systems = configs.ensemble(n_rep, seed=3, nmin=200, nmax=2500)
    b64 = Batch(systems, precision=0)
    b32 = Batch(systems, precision=1)
    rhs = b64.stage()
    b32.stage()
    g = torch.Generator("cuda").manual_seed(0)
    x = torch.randn(b64.nvec, dtype=torch.float64, device="cuda", generator=g)
    assert _rel(b32.matmult(x), b64.matmult(x)) < 1e-6
    rhs[: 0] += 0
    X64, r64 = b64.solve(rhs, rtol=1e-10, method=1)
    X32, r32 = b32.solve(rhs, rtol=1e-10, method=1)
    assert r64.reason > 0 and r32.reason > 0
    assert _rel(X32, X64) < 1e-6
    b64.close()
    b32.close()


@pytest.mark.parametrize("shift", [0.0, 1000.0])
def test_mixed_far_from_origin(shift):
    """The FP32 monomer kernel adds the low parts of positions within an exact
    radius that grows with the replica's largest coordinate: a replica moved
    1000 units from the origin, where hi-only separations would be off by
    ~1e-4, keeps the 1e-6 bound on the mobility apply."""
    s = configs.ensemble(1, seed=5, nmin=1500, nmax=1500)[0]
    s.x = s.x + np.array([shift, -0.5 * shift, 0.25 * shift])
    b64 = Batch([s], precision=0)
    b32 = Batch([s], precision=1)
    b64.stage()
    b32.stage()
    g = torch.Generator("cuda").manual_seed(2)
    u = torch.randn(b64.ntop, dtype=torch.float64, device="cuda", generator=g)
    assert _rel(b32.mobility_apply(u), b64.mobility_apply(u)) < 1e-6
    b64.close()
    b32.close()


@pytest.mark.parametrize("lub", [False, True])
def test_iterative_refinement_recovers_fp64(lub):
    """One FP64 iterative-refinement sweep per solve (ps_step_inputs.refine): the residual is
    formed with the FP64 operator and a mixed-precision correction is added.  At kT = 0 (the
    step's velocities come from its saddle solves alone; with noise the FP32 Lanczos square
    root adds its own ~1e-7) a step of the replicas lands several times closer to the FP64
    step at the same rtol 1e-8."""
    systems = configs.ensemble(4, seed=7, nmin=300, nmax=1500, lub=lub)
    for s in systems:
        s.params["kT"] = 0.0
    ups = []
    for prec, rtol, refine in ((0, 1e-11, 0), (1, 1e-8, 0), (1, 1e-8, 1)):
        b = Batch(systems, precision=prec)
        res = b.step(rtol=rtol, maxit=50000, solver=1, refine=refine)
        assert res.reason > 0
        ups.append(b.step_outputs()["up"])
        b.close()
    e_plain, e_ref = _rel(ups[1], ups[0]), _rel(ups[2], ups[0])
    assert e_plain < 1e-6
    assert e_ref < 5e-8 and e_ref < 0.25 * e_plain, (e_plain, e_ref)


@pytest.mark.parametrize("precision", [0, 1])
def test_lanczos_paths_bit_identical(precision):
    """The Lanczos square root orthogonalises a batch of up to 16 replicas with one
    thread-block-cluster launch per basis vector and larger batches with the
    reduction-table launch sequence; both sum in the same order, so a replica's
    M^{1/2} z is bit-identical whether it runs alone or in a 20-replica batch."""
    systems = configs.ensemble(20, seed=4, nmin=64, nmax=600)
    big = Batch(systems, precision=precision)
    big.stage()
    z = torch.randn(big.ntop, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    w_big, _ = big.sqrtm(z, kmax=40, tol=1e-6)
    for r in (0, 7, 19):
        one = Batch([systems[r]], precision=precision)
        one.stage()
        w_one, _ = one.sqrtm(big.seg(z, r, "top").contiguous(), kmax=40, tol=1e-6)
        assert torch.equal(w_one, big.seg(w_big, r, "top")), r
        one.close()
    big.close()
