"""The far-field autotuner (ps_autotune): it picks one of the candidate column
chunk widths, the apply is unchanged up to summation order (FP64, 1e-13), and
the choice is process-wide (a context created afterwards uses it)."""
import numpy as np
import pytest

from polystokes_brownian_b200 import configs

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_width_and_keeps_the_operator():
    import torch
    from polystokes_brownian_b200.engine import Batch
    systems = configs.ensemble(8, seed=5, nmin=100, nmax=1500)
    b = Batch(systems)
    b.stage()
    n = b.nvec
    x = torch.from_numpy(np.random.default_rng(0).normal(size=n)).cuda()
    y0 = b.matmult(x).cpu().numpy()
    best, ms = b.autotune(3)
    assert best in (128, 256, 512, 1024) and all(v > 0 for v in ms.values())
    assert ms[best] == min(ms.values())
    y1 = b.matmult(x).cpu().numpy()
    assert np.linalg.norm(y1 - y0) <= 1e-13 * np.linalg.norm(y0)
    # a later context chunks the same way: its apply equals the tuned context's bit for bit
    b2 = Batch(systems)
    b2.stage()
    assert np.array_equal(b2.matmult(x).cpu().numpy(), y1)
    b.close()
    b2.close()
