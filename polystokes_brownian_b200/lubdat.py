"""Two-body lubrication table of the reference (lubdat/r2babc.dat).

Rows: r/a, then X11A X12A Y11A Y12A Y11B Y12B X11C X12C Y11C Y12C -- the two-body
resistance functions minus the inverted far-field two-body mobility, for
r/a in [2.1, 4.0].  The package ships the table as data/lubdat_r2babc.npy
(generated from the reference's file by tests/golden/make_golden.py); a user
may also pass the reference's own .dat file.
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_table(path: str | None = None) -> np.ndarray:
    if path is None:
        return np.load(os.path.join(HERE, "data", "lubdat_r2babc.npy"))
    if os.path.isdir(path):
        path = os.path.join(path, "r2babc.dat")
    if path.endswith(".npy"):
        return np.load(path)
    return np.loadtxt(path)
