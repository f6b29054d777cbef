"""Programmatic dependent launch decides only when a grid is scheduled, never
what it computes: two steps of a lubricated 24-replica ensemble (the reduction
table's Lanczos sweeps, pair-space CG) and of a lubricated 96-colloid
suspension (the cluster Lanczos kernel, pair-space MINRES) leave bit-identical
states with the attribute on (twice) and off (PS_PDL=0).  The attribute is read
once per process, so each run is a child process."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.join(os.path.dirname(__file__), "..")

CHILD = r"""
import sys
import numpy as np
from polystokes_brownian_b200 import _capi, configs
from polystokes_brownian_b200.engine import Batch

out = {}
ens = configs.ensemble(24, seed=5, nmin=64, nmax=800, lub=True)
s = configs.suspension(n=96, seed=2)
susp = [configs.System(s.name, dict(s.params, lub_on=1, lub_gap=0.5), s.x)]
for name, systems in (("ens", ens), ("susp", susp)):
    b = Batch(systems, precision=_capi.PS_PREC_MIXED)
    b.set_replica_seeds(list(range(11, 11 + len(systems))))
    for _ in range(2):
        b.step(rtol=1e-8, maxit=50000, solver=_capi.PS_SOLVE_STRUCTURED)
    x, q = b.state()
    o = b.step_outputs()
    out[name + "_x"] = x.cpu().numpy()
    out[name + "_q"] = q.cpu().numpy()
    out[name + "_up"] = o["up"].cpu().numpy()
    b.close()
np.savez(sys.argv[1], **out)
"""


def _run(tmp_path, tag, pdl):
    path = str(tmp_path / f"{tag}.npz")
    env = dict(os.environ, PS_PDL=pdl)
    subprocess.run([sys.executable, "-c", CHILD, path], cwd=ROOT, env=env, check=True, timeout=600)
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def test_dependent_launch_bit_identical(tmp_path):
    on1 = _run(tmp_path, "on1", "1")
    on2 = _run(tmp_path, "on2", "1")
    off = _run(tmp_path, "off", "0")
    for k in on1:
        assert np.all(np.isfinite(on1[k])), k
        assert np.array_equal(on1[k], on2[k]), k
        assert np.array_equal(on1[k], off[k]), k
