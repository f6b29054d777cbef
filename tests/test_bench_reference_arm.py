"""The reference arm's CPU machinery (no GPU): the longest-first schedule and
the oracle stepped concurrently in spawned worker processes."""
import multiprocessing as mp
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402
from polystokes_brownian_b200 import configs  # noqa: E402


def test_lpt_makespan():
    assert bench.lpt_makespan([3.0, 3.0, 2.0, 2.0, 2.0], 2) == 7.0     # longest first: 3+2+2 | 3+2
    assert bench.lpt_makespan([5.0, 1.0, 1.0], 4) == 5.0
    assert abs(bench.lpt_makespan([1.0] * 10, 1) - 10.0) < 1e-12


def test_parallel_oracle_baseline_small_batch():
    systems = configs.ensemble(6, seed=2, nmin=40, nmax=90)
    with mp.get_context("spawn").Pool(2) as pool:
        cb = bench.cpu_baseline_parallel(systems, 1e-6, 2, pool)
    assert cb["cores"] == 2 and cb["kind"] == "port"
    assert np.isfinite(cb["value"]) and cb["value"] > 0
    assert cb["sample_seconds"] > 0
