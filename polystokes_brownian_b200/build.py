"""Build the B200 engine: every .cu under csrc/ -> one shared library
polystokes_brownian_b200/_lib/libpsb200.so, compiled for sm_100a only; then the
host module csrc/host/polystokes_module.cpp (the reference's pybind11 module
`PolyStokes`) -> polystokes_brownian_b200/_lib/PolyStokes<ext>, linked to it.

Usage: python -m polystokes_brownian_b200.build [--force] [-j N]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libpsb200.so")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-Xptxas", "-v", "-I" + os.path.join(HERE, "..", "include")]
# translation units whose arithmetic must round like the reference's C++
NO_FMA = {"stage.cu", "step.cu", "pairs.cu", "lub.cu"}
# FP32 subnormals flushed to zero: the far-field kernels' FP32 operands (pair
# separations and their squares, reciprocal square roots, inputs of order one)
# stay many decades above the subnormal range (1e-38), and without the flag every
# rsqrtf carries a subnormal guard (4 of 25 instructions per pair in the FP32x2
# monomer kernel, measured with ncu's per-pipe instruction counts)
FTZ = {"rpy.cu"}


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _needs(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src):
    obj = os.path.join(BUILD, src[:-3] + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(HERE, "..", "include", "polystokes_b200.h"))
    if not _needs(obj, deps):
        return obj, ""
    cmd = [NVCC] + ARCH + COMMON + (["--fmad=false"] if src in NO_FMA else []) + \
          (["-ftz=true"] if src in FTZ else []) + ["-c", os.path.join(CSRC, src), "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{p.stdout}\n{p.stderr}")
    with open(os.path.join(BUILD, src[:-3] + ".ptxas.txt"), "w") as f:
        f.write(p.stderr)
    return obj, p.stderr


def build(force: bool = False, jobs: int = 8) -> str:
    os.makedirs(OUT, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = [o for o, _ in ex.map(_compile, srcs)]
    if force or _needs(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"link failed:\n{p.stdout}\n{p.stderr}")
    return LIB


def build_host(force: bool = False) -> str:
    import sysconfig

    import pybind11
    src = os.path.join(CSRC, "host", "polystokes_module.cpp")
    out = os.path.join(OUT, "PolyStokes" + sysconfig.get_config_var("EXT_SUFFIX"))
    hdr = os.path.join(HERE, "..", "include", "polystokes_b200.h")
    if not force and not _needs(out, [src, hdr, LIB]):
        return out
    cxx = shutil.which("g++") or "c++"
    cmd = [cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
           "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"],
           "-I" + os.path.join(HERE, "..", "include"), src, "-o", out,
           "-L" + OUT, "-lpsb200", "-Wl,-rpath,$ORIGIN"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"host module build failed:\n{p.stdout}\n{p.stderr}")
    return out


if __name__ == "__main__":
    j = 8
    if "-j" in sys.argv:
        j = int(sys.argv[sys.argv.index("-j") + 1])
    print(build(force="--force" in sys.argv, jobs=j))
    print(build_host(force="--force" in sys.argv))
