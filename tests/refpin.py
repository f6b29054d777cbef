"""Loader for the golden fixtures made by the reference's own code
(tests/golden/make_ref_fixtures.py): inputs, per-step noise, the reference's
saddle solves in run order and the output files it wrote."""
from __future__ import annotations

import json
import os

import numpy as np

from polystokes_brownian_b200 import configs

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SMALL = ["dense_spd", "dense_spd_nc2", "dense_kt0", "shell_probe", "shell_lanczos", "probe_c1"]
ALL = SMALL + ["replica1000"]


class RefCase:
    def __init__(self, name: str):
        self.name = name
        self.d = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
        p = json.loads(str(self.d["params"]))
        p["kT"] = float(self.d["kT"])
        self.params = p
        self.x0 = self.d["x0"]
        self.system = configs.System(name, configs.make_params(**p), self.x0.copy())
        self.Nm, self.Nc = p["Nm"], p["Nc"]
        self.nm3nc11 = 3 * self.Nm + 11 * self.Nc
        self.nm3nc6 = 3 * self.Nm + 6 * self.Nc
        self.n = self.nm3nc11 + self.nm3nc6
        self.steps = int(self.d["steps"])
        self.kT = p["kT"]
        self.nsolve = 5 if self.kT > 0 else 3

    def has(self, key):
        return key in self.d.files

    def noise(self, k: int):
        """(fb, W) the reference drew at step k; fb is zero where its MFN square root failed
        (the reference then adds no slip noise, slip_vel.cpp:40-48)."""
        if self.kT <= 0:
            return None, None
        per = self.nm3nc11 + self.nm3nc6
        z = self.d["normals"][k * per:(k + 1) * per]
        fb = z[: self.nm3nc11].copy()
        if self.has("mfn_reason") and self.d["mfn_reason"][k] < 0:
            fb[:] = 0.0
        return fb, z[self.nm3nc11:].copy()

    def solves(self, k: int):
        """The saddle solutions of step k, in run order."""
        return self.d["ksp_x"][self.nsolve * k:self.nsolve * (k + 1)]

    def velocities(self, k: int) -> dict:
        """Velocity-part quantities of step k assembled from the reference's solves
        (run.cpp:70-162): v_det_n, the predictor velocity, udiff, v_det_c, the corrector up."""
        X = self.solves(k)[:, self.nm3nc11:]
        out = {"v_det_n": X[0], "v_det_c": X[-1]}
        if self.kT > 0:
            out["v_pred"] = X[1]
            out["udiff"] = X[3] - X[2]
            out["up"] = 0.5 * (X[0] + X[-1]) + (X[1] - X[0])
        else:
            out["up"] = 0.5 * (X[0] + X[-1])
        return out


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
