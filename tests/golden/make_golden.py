"""Generate the golden fixtures under tests/golden/ from files that ship with the
reference (run in a container where the reference tree is mounted; the GPU box
only reads the committed .npz files).

mobcsv.npz: the dense grand mobility written by the reference (mob.csv; Nm=33,
Nc=2, beta=0.1, shell path) together with bead positions reconstructed from its
rotation-force blocks (mob_b = y12b eps.e with y12b = -3/(4 r^2), so each
monomer-colloid and colloid-colloid block gives the separation vector exactly).

lubdat.npz: the five two-body resistance tables of lubdat/*.dat.
"""
import os
import sys

import numpy as np

if len(sys.argv) < 2:
    sys.exit("usage: python tests/golden/make_golden.py <reference project path>")
REF = sys.argv[1]
OUT = os.path.dirname(os.path.abspath(__file__))


def read_mobcsv(path):
    lines = open(path).read().split("\n")[2:]
    return np.array([list(map(float, l.split())) for l in lines if l.strip()])


def rot_to_sep(B):
    v = np.array([B[1, 2], B[2, 0], B[0, 1]])
    nv = np.linalg.norm(v)
    return -v / nv, np.sqrt(0.75 / nv)


def mobcsv():
    M = read_mobcsv(os.path.join(REF, "mob.csv"))
    Nm, Nc, beta = 33, 2, 0.1
    nm3, nc3 = 3 * Nm, 3 * Nc
    x = np.zeros((Nm + Nc, 3))
    rc0 = nm3 + nc3
    e, r = rot_to_sep(M[rc0:rc0 + 3, nm3 + 3:nm3 + 6])
    x[Nm + 1] = x[Nm] - r * e
    for m in range(Nm):
        e, r = rot_to_sep(M[rc0:rc0 + 3, 3 * m:3 * m + 3])
        x[m] = x[Nm] + r * e
    # consistency against the second colloid's blocks
    err = 0.0
    for m in range(Nm):
        e, r = rot_to_sep(M[rc0 + 3:rc0 + 6, 3 * m:3 * m + 3])
        err = max(err, np.abs(x[Nm + 1] + r * e - x[m]).max())
    assert err < 1e-12, err
    np.savez_compressed(os.path.join(OUT, "mobcsv.npz"), M=M, x=x, Nm=Nm, Nc=Nc, beta=beta)


def lubdat():
    tabs = {}
    for name in ("r2babc", "r2babcd", "r2bgh", "r2bghd", "r2bm"):
        tabs[name] = np.loadtxt(os.path.join(REF, "lubdat", name + ".dat"))
    np.savez_compressed(os.path.join(OUT, "lubdat.npz"), **tabs)
    # the table the lubrication path consumes, shipped with the package
    pkg = os.path.join(OUT, "..", "..", "polystokes_brownian_b200", "data")
    os.makedirs(pkg, exist_ok=True)
    np.save(os.path.join(pkg, "lubdat_r2babc.npy"), tabs["r2babc"])


if __name__ == "__main__":
    mobcsv()
    lubdat()
    print("wrote", OUT)
