"""Fluctuation-dissipation of the Brownian noise on the device: the slip
velocities W = M^{1/2} z (slip_vel.cpp:19-79 of the reference: SLEPc FNSQRT on the
dense mobility, or the block-Cholesky of the arrowhead path) must have
covariance M.

* exact: a batch of n copies of one system, copy k fed z = e_k, gives the
  columns of W; W W^T = M (dense path: the symmetric root; shell path: the
  block-Cholesky factor with the Schur floor) to 1e-10 relative;
* statistical: 4096 copies fed independent Gaussian z; the sample covariance
  matches M within 4 standard errors of the Frobenius norm,
  sqrt((||M||_F^2 + tr(M)^2) / n) / ||M||_F.
"""
import numpy as np
import pytest
import torch

from oracle import psoracle as po
from polystokes_brownian_b200 import configs
from polystokes_brownian_b200.engine import Batch

pytestmark = pytest.mark.gpu


def dense_m(sysm):
    o = po.OracleSim(po.default_params(**sysm.params), sysm.x.ravel())
    o.stage()
    return o.dense_mobility()


def columns(sysm, Z, kmax=64, tol=1e-14):
    n = Z.shape[1]
    b = Batch([sysm] * n)
    b.stage()
    w, _ = b.sqrtm(torch.from_numpy(np.ascontiguousarray(Z.T).ravel()).cuda(), kmax=kmax, tol=tol)
    W = w.cpu().numpy().reshape(n, -1).T
    b.close()
    return W


@pytest.mark.parametrize("case", ["dense", "shell"])
def test_noise_covariance_exact(case):
    if case == "dense":
        sysm = configs.small_mixed(seed=5, Nm_chain=(3, 4), Nc=2, mm_HI=1, aa_mode=1, ab_mode=1)
    else:
        sysm = configs.small_mixed(seed=6, Nm_chain=(4, 5), Nc=2, mm_HI=0, spread=8.0)
    M = dense_m(sysm)
    n = M.shape[0]
    if case == "dense":
        assert n <= 64          # the Lanczos subspace (kmax 64) spans the whole space: the root is exact
    assert np.linalg.eigvalsh(M).min() > 0
    W = columns(sysm, np.eye(n))
    assert np.linalg.norm(W @ W.T - M) <= 1e-10 * np.linalg.norm(M)


def test_noise_covariance_sampled():
    sysm = configs.small_mixed(seed=5, Nm_chain=(3, 4), Nc=2, mm_HI=1, aa_mode=1, ab_mode=1)
    M = dense_m(sysm)
    n = M.shape[0]
    ns = 4096
    Z = np.random.default_rng(11).normal(size=(n, ns))
    W = columns(sysm, Z)
    C = W @ W.T / ns
    se = np.sqrt((np.linalg.norm(M) ** 2 + np.trace(M) ** 2) / ns) / np.linalg.norm(M)
    err = np.linalg.norm(C - M) / np.linalg.norm(M)
    assert err < 4 * se, (err, se)
    # and the samples are the symmetric root of the SPD M applied to z
    lam, Q = np.linalg.eigh(M)
    R = (Q * np.sqrt(lam)) @ Q.T
    assert np.linalg.norm(W - R @ Z) <= 1e-9 * np.linalg.norm(R @ Z)
