"""Generate golden fixtures from the reference's own code (tests/golden/ref_*.npz).

The reference's sources are compiled unmodified into its pybind11 module
oracle/_ref/PolyStokes<ext> (``make -C oracle ref REF=<reference project>``,
against the PETSc/SLEPc stand-in in oracle/refshim/).  Each case below builds a
seeded system, runs the reference's own ``PolyStokes.run()`` for a few steps in a
child process (the reference keeps its state in globals: one simulation per
process) with the stand-in's hooks on:

  ORACLE_KSP_RTOL=1e-13   every saddle solve converged tightly,
  ORACLE_REF_DUMP=<file>  every KSPSolve's right-hand side and solution, every
                          MFNSolve's input and output, and (small dense cases)
                          the assembled saddle matrix A,

and stores in one .npz per case: the inputs (parameters, positions, seed), the
reference's Gaussian stream for those steps, the dumped solves, and the output
files the reference wrote (config_, quats_, force_, brownian_stresslet_).

Per step the reference solves, in order (run.cpp:70-162, drift.cpp:17-62): the
deterministic predictor velocity at x_n; with kT > 0 the full predictor velocity
(slip noise added) and the two RFD probes at x_n +/- eps W (the second warm-started);
the deterministic corrector velocity at x_pred.  So 5 solves per step with kT > 0,
3 with kT = 0.

Usage (in a container with the reference tree; the GPU box only reads the .npz):
    python tests/golden/make_ref_fixtures.py <reference project path> [case ...]
"""
from __future__ import annotations

import ctypes
import glob
import json
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REFDIR = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, ROOT)


def cases():
    """name -> (system builder, run options).  Sizes keep each fixture small."""
    from polystokes_brownian_b200 import configs as cf

    def dense_spd():
        # inter-chain monomer HI only (chain_HI): the last monomer pair the dense assembly
        # evaluates is then far apart, so the stale monomer-colloid translation block it leaves
        # (mob.cpp:845-904) is weak and M stays positive definite; the reference's MFN square root
        # converges and the slip noise is added
        s = cf.small_mixed(seed=4, Nm_chain=(4, 5), Nc=1, mm_HI=1, beta=0.5, spread=7.0, chain_HI=1)
        return s, dict(steps=3, kT=1.0, seed=11, dump_mat=True)

    def dense_spd_nc2():
        s = cf.small_mixed(seed=1, Nm_chain=(4, 5), Nc=2, mm_HI=1, beta=0.4, spread=8.0, chain_HI=1)
        return s, dict(steps=3, kT=1.0, seed=5, dump_mat=True)

    def dense_kt0():
        # full monomer HI in the reference's scalars; at bond length 2.5 beta they give an
        # indefinite M, so kT = 0 (no square root) and the bonds start stretched (r0 = 2 beta)
        s = cf.small_mixed(seed=1, Nm_chain=(3, 4), Nc=2, mm_HI=1, r0=0.6)
        return s, dict(steps=4, kT=0.0, seed=1, dump_mat=True)

    def shell_probe():
        # the arrowhead (matrix-free) path with one probe: Nc = 1 is the regime the reference's
        # shell operator supports (matfree_A.cpp:15-17, 127-131)
        s = cf.small_mixed(seed=2, Nm_chain=(4, 10), Nc=1, mm_HI=0, beta=1.0 / 3.0, spread=8.0)
        return s, dict(steps=3, kT=1.0, seed=3, dump_mat=False)

    def shell_lanczos():
        # the same path with the crossover at 0 (POLYSTOKES_LANCZOS_NC=0, slip_vel.cpp:283-288):
        # the colloid noise comes from schur_sqrt_lanczos (slip_vel.cpp:351-477) and Mcc carries
        # no eigenvalue-floor correction (sync_mcc_schur_correction returns early)
        s = cf.small_mixed(seed=2, Nm_chain=(4, 10), Nc=1, mm_HI=0, beta=1.0 / 3.0, spread=8.0, lanczos_nc=0)
        return s, dict(steps=3, kT=1.0, seed=4, dump_mat=False, env={"POLYSTOKES_LANCZOS_NC": "0"})

    def probe_c1():
        # the polymer-plus-probe workload (11 chains x 20 beads, a_c = 3) with one probe: the
        # reference's shell path cannot take two (its colloid-colloid blocks are written into
        # the shell matrix, mob.cpp:1026-1144, which has no MATOP_SET_VALUES)
        s = cf.polymer_probe(seed=0)
        p = dict(s.params)
        p["Nc"] = 1
        s = cf.System("probe_c1", cf.make_params(**p), s.x[:221].copy())
        return s, dict(steps=3, kT=1.0, seed=0, dump_mat=False)

    def replica1000():
        # one batched-ensemble replica of about 1000 beads in the reference's own pair scalars
        s = cf.ensemble_member(np.random.default_rng([0, 7]), 1000, pair_mode=0, dt=1e-4)
        return s, dict(steps=1, kT=1.0, seed=2, dump_mat=False)

    return {"dense_spd": dense_spd, "dense_spd_nc2": dense_spd_nc2, "dense_kt0": dense_kt0,
            "shell_probe": shell_probe, "shell_lanczos": shell_lanczos, "probe_c1": probe_c1,
            "replica1000": replica1000}


def run_case(name: str, out: str) -> None:
    """Child process: run the reference module on one case."""
    sys.path.insert(0, REFDIR)
    import PolyStokes as R  # the reference's module built from its own sources

    s, o = cases()[name]()
    p = s.params
    dt = p["dt"]
    sim = R.PolyStokes(dt, 1, (o["steps"] + 0.5) * dt, out, mm_HI=bool(p["mm_HI"]), chain_HI=bool(p["chain_HI"]),
                       fene=bool(p["fene"]), record_forces=True, seed=o["seed"])
    sim.particle_info(o["kT"], p["epsilon"], s.Np, p["Nc"], p["Nm"], p["Npoly"], p["Nmono_per_chain"], p["beta"],
                      p["kbond"], p["r0"], p["Lmax"], p["tau"])
    sim.trap_info(p["ktrap"], p["tstart"], p["trun"])
    sim.initial_configuration(np.ascontiguousarray(s.x.ravel()))
    sim.set_warn_neg_eig(False)
    sim.run()


def parse_dump(path):
    """Records of the stand-in's dump file, in order."""
    recs = []
    with open(path, "rb") as f:
        buf = f.read()
    off = 0
    while off < len(buf):
        tag, n, a, b = struct.unpack_from("<4i", buf, off)
        off += 16
        if tag == ord("A"):
            A = np.frombuffer(buf, "<f8", n * n, off).reshape(n, n).T.copy()   # stored column-major
            off += 8 * n * n
            recs.append(("A", A))
        elif tag == ord("K"):
            (its,) = struct.unpack_from("<i", buf, off)
            off += 4
            rhs = np.frombuffer(buf, "<f8", n, off).copy()
            off += 8 * n
            x = np.frombuffer(buf, "<f8", n, off).copy()
            off += 8 * n
            recs.append(("K", dict(warm=a, reason=b, its=its, rhs=rhs, x=x)))
        elif tag == ord("F"):
            zin = np.frombuffer(buf, "<f8", n, off).copy()
            off += 8 * n
            zout = np.frombuffer(buf, "<f8", n, off).copy()
            off += 8 * n
            recs.append(("F", dict(reason=a, zin=zin, zout=zout)))
        else:
            raise ValueError(f"bad dump tag {tag} at {off - 16}")
    return recs


def read_outputs(out):
    """The reference's text outputs, keyed by file prefix, each stacked over the steps."""
    res = {}
    for pre in ("config", "quats", "force", "brownian_stresslet"):
        files = glob.glob(os.path.join(out, pre + "_*_.txt"))
        files.sort(key=lambda f: float(os.path.basename(f)[len(pre) + 1:-5]))
        arrs = [np.loadtxt(f, ndmin=2) for f in files]
        if arrs:
            res[pre] = np.stack(arrs)
            res[pre + "_names"] = np.array([os.path.basename(f) for f in files])
    return res


def ref_normals(seed, n):
    L = ctypes.CDLL(os.path.join(REFDIR, "librefnoise.so"))
    L.ref_normals.argtypes = [ctypes.c_ulong, ctypes.c_long, ctypes.POINTER(ctypes.c_double)]
    out = np.zeros(n)
    L.ref_normals(seed, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


def make(name: str) -> str:
    s, o = cases()[name]()
    p = s.params
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "out")
        os.makedirs(out)
        dump = os.path.join(td, "dump.bin")
        env = dict(os.environ, ORACLE_KSP_RTOL="1e-13", ORACLE_REF_DUMP=dump, **o.get("env", {}))
        if o["dump_mat"]:
            env["ORACLE_REF_DUMP_MAT"] = "1"
        log = subprocess.run([sys.executable, os.path.abspath(__file__), "--run-case", name, out], env=env,
                             capture_output=True, text=True)
        if log.returncode != 0:
            raise RuntimeError(f"reference run failed for {name}:\n{log.stdout[-3000:]}\n{log.stderr[-3000:]}")
        recs = parse_dump(dump)
        outs = read_outputs(out)
    Nm, Nc = p["Nm"], p["Nc"]
    nm3nc11, nm3nc6 = 3 * Nm + 11 * Nc, 3 * Nm + 6 * Nc
    kT = o["kT"]
    per_step = (nm3nc11 + nm3nc6) if kT > 0 else 0
    data = dict(x0=s.x, seed=o["seed"], steps=o["steps"], kT=kT,
                params=json.dumps({k: (float(v) if isinstance(v, float) else v) for k, v in p.items()}),
                normals=ref_normals(o["seed"], per_step * o["steps"]) if per_step else np.zeros(0))
    ks = [r[1] for r in recs if r[0] == "K"]
    data["ksp_rhs"] = np.stack([k["rhs"] for k in ks])
    data["ksp_x"] = np.stack([k["x"] for k in ks])
    data["ksp_warm"] = np.array([k["warm"] for k in ks], np.int32)
    data["ksp_reason"] = np.array([k["reason"] for k in ks], np.int32)
    data["ksp_its"] = np.array([k["its"] for k in ks], np.int32)
    fs = [r[1] for r in recs if r[0] == "F"]
    if fs:
        data["mfn_reason"] = np.array([f["reason"] for f in fs], np.int32)
        data["mfn_in"] = np.stack([f["zin"] for f in fs])
        data["mfn_out"] = np.stack([f["zout"] for f in fs])
    mats = [r[1] for r in recs if r[0] == "A"]
    if mats:
        # the operators of the first step's distinct stages: x_n (solve 1) and x_n + eps W
        # (solve 3) with kT > 0; x_n and x_pred (solves 1 and 3) with kT = 0
        keep = [0, 2]
        data["A"] = np.stack([mats[i] for i in keep if i < len(mats)])
        data["A_solve"] = np.array([i for i in keep if i < len(mats)], np.int32)
    data.update(outs)
    path = os.path.join(HERE, f"ref_{name}.npz")
    np.savez_compressed(path, **data)
    return path


def main():
    if len(sys.argv) >= 2 and sys.argv[1] == "--run-case":
        run_case(sys.argv[2], sys.argv[3])
        return
    if len(sys.argv) < 2:
        sys.exit(__doc__)
    ref = sys.argv[1]
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={ref}"], check=True)
    names = sys.argv[2:] or list(cases())
    for nm in names:
        print(make(nm), os.path.getsize(os.path.join(HERE, f"ref_{nm}.npz")), "bytes")


if __name__ == "__main__":
    main()
