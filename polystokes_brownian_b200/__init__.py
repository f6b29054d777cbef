"""B200-native engine for the PolyStokes per-timestep Stokesian-dynamics path.

The compute path is the CUDA library behind include/polystokes_b200.h
(polystokes_brownian_b200/_lib/libpsb200.so); this package holds its ctypes
binding, the batch front end and the seeded synthetic workloads.
"""
from . import configs  # noqa: F401

__all__ = ["configs", "engine", "build"]
