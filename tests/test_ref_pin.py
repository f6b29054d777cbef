"""The oracle (oracle/psoracle.c) pinned to the reference's own code.

The fixtures come from the reference's sources compiled unmodified against the
PETSc/SLEPc stand-in (tests/golden/make_ref_fixtures.py, oracle/Makefile `ref`):
its assembled dense saddle matrix, every saddle solve of its run loop at rtol
1e-13, its MFN square roots and its output files.

Tolerances: the dense mobility block <= 1e-13 relative (it is assembled from the
same long-double tensors); solve outputs <= 1e-10 relative (both sides solved at
rtol 1e-13 with independently written MINRES); positions against the reference's
config_ files <= 2e-10 absolute (they are printed with %.10f, write_configuration.cpp);
square roots <= 1e-10 relative."""
import numpy as np
import pytest

from oracle import psoracle as po
from refpin import SMALL, RefCase, rel


def oracle(case: RefCase):
    return po.OracleSim(po.default_params(**case.params), case.x0.ravel())


@pytest.mark.parametrize("name", [n for n in SMALL if RefCase(n).has("A")])
def test_dense_saddle_matrix(name):
    c = RefCase(name)
    o = oracle(c)
    o.stage()
    M = o.dense_mobility()
    A = c.d["A"][0]
    n11, n6 = c.nm3nc11, c.nm3nc6
    assert np.abs(A[:n11, :n11] - M).max() <= 1e-13 * np.abs(M).max()
    # B = [-I; 0] and its transpose (arrays.cpp:349-408); zero lower-right block
    B = np.zeros((n11, n6))
    B[:n6, :n6] = -np.eye(n6)
    assert np.array_equal(A[:n11, n11:], B) and np.array_equal(A[n11:, :n11], B.T)
    assert not A[n11:, n11:].any()
    if c.kT > 0:
        # solve 3 runs at the RFD probe x_n + eps W (drift.cpp:27-30, eps = 1e-3)
        _, W = c.noise(0)
        n3 = 3 * (c.Nm + c.Nc)
        o2 = po.OracleSim(po.default_params(**c.params), c.x0.ravel() + 1e-3 * W[:n3])
        o2.check_dist()
        o2.mob()
        M2 = o2.dense_mobility()
        assert np.abs(c.d["A"][1][:n11, :n11] - M2).max() <= 1e-13 * np.abs(M2).max()


@pytest.mark.parametrize("name", SMALL)
def test_first_solve(name):
    """The oracle's RHS and MINRES on the reference's first saddle system."""
    c = RefCase(name)
    o = oracle(c)
    rhs = o.stage()
    assert rel(rhs, c.d["ksp_rhs"][0]) <= 1e-13
    x, reason, its, _ = o.minres(c.d["ksp_rhs"][0], rtol=1e-13)
    assert reason > 0
    assert rel(x, c.d["ksp_x"][0]) <= 1e-10


@pytest.mark.parametrize("name", SMALL)
def test_trajectory(name):
    """Steps of the oracle with the reference's own noise stream against the reference's
    solves and output files."""
    c = RefCase(name)
    o = oracle(c)
    for k in range(c.steps):
        fb, W = c.noise(k)
        out = o.step(fb=fb, wrfd=W, rtol=1e-13)
        v = c.velocities(k)
        assert rel(out["v_det_n"], v["v_det_n"]) <= 1e-10
        assert rel(out["v_det_c"], v["v_det_c"]) <= 1e-10
        assert rel(out["up"], v["up"]) <= 1e-10
        if c.kT > 0:
            assert rel(out["v_det_n"] + out["v_brown"], v["v_pred"]) <= 1e-10
            assert rel(out["udiff"], v["udiff"]) <= 1e-9
        x, q = o.state()
        assert np.abs(x - c.d["config"][k].ravel()).max() <= 2e-10
        if c.Nc:
            assert np.abs(q - c.d["quats"][k].ravel()).max() <= 2e-10


@pytest.mark.parametrize("name", [n for n in SMALL if RefCase(n).has("mfn_out")])
def test_mfn_square_root(name):
    """The stand-in's MFN output (the reference's slip noise before scaling) is sqrt(M) z
    for the oracle's M at the same positions."""
    c = RefCase(name)
    o = oracle(c)
    o.stage()
    M = o.dense_mobility()
    z = c.d["mfn_in"][0]
    assert c.d["mfn_reason"][0] > 0
    assert rel(po.sqrtm_eig(M, z), c.d["mfn_out"][0]) <= 1e-10


def test_replica_first_solves():
    """A ~1000-bead ensemble replica in the reference's scalars: the first step's RHS and
    deterministic solve (the operator is indefinite, so the MFN root failed and the
    reference added no slip noise)."""
    c = RefCase("replica1000")
    o = oracle(c)
    rhs = o.stage()
    assert rel(rhs, c.d["ksp_rhs"][0]) <= 1e-13
    assert c.d["mfn_reason"][0] < 0
    # the reference's solution satisfies the oracle's operator to its own tolerance
    r = o.saddle_apply(c.d["ksp_x"][0]) - c.d["ksp_rhs"][0]
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(c.d["ksp_rhs"][0])


