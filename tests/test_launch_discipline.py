"""Source checks of the kernels' launch discipline (no GPU needed).

The library launches its kernels with programmatic dependent launch
(`ps_launch`, csrc/ps_internal.h): a grid may be scheduled while the previous
grid of the stream is still running, so every kernel launched that way must
open with `pdl_enter()` (griddepcontrol.wait before anything else, early-exit
blocks included).  A kernel that skipped it could read its inputs before their
producer finished.  These tests read the CUDA sources and check that rule, and
that no launch site bypasses the launcher with a bare triple-chevron launch
except the ones that stay plain (a cluster launch, the FMA peak probes and
the allocation-free apply, whose kernels do not open with pdl_enter())."""
import os
import re

CSRC = os.path.join(os.path.dirname(__file__), "..", "polystokes_brownian_b200", "csrc")
SOURCES = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
# launches that stay plain on purpose
PLAIN_OK = {"k_lz_orth_cluster", "k_fma", "k_fma2", "k_na_pack", "k_na_pairs", "k_na_combine"}


def _read(f):
    with open(os.path.join(CSRC, f)) as fh:
        return fh.read()


def _kernels(src):
    """name -> first statement of the body, for every __global__ function."""
    out = {}
    for m in re.finditer(r"__global__", src):
        brace = src.index("{", m.end())
        head = src[m.end():brace]
        name = re.findall(r"(\w+)\s*\(", head)
        assert name, head[:80]
        nm = [n for n in name if n not in ("__launch_bounds__", "__cluster_dims__")][0]
        body = src[brace + 1:brace + 200].lstrip()
        out[nm] = body.split(";")[0].strip()
    return out


def test_every_kernel_launched_by_ps_launch_opens_with_pdl_enter():
    kernels, launched = {}, set()
    for f in SOURCES:
        src = _read(f)
        kernels.update(_kernels(src))
        for m in re.finditer(r"ps_launch\(\s*([A-Za-z_]\w*)", src):
            launched.add(m.group(1))
    assert len(launched) > 60
    missing = sorted(k for k in launched if k not in kernels)
    assert not missing, f"launched but not defined in csrc: {missing}"
    bad = sorted(k for k in launched if kernels[k] != "pdl_enter()")
    assert not bad, f"kernels launched with dependent launch that do not open with pdl_enter(): {bad}"


def test_no_bare_launch_outside_the_allowed_ones():
    bare = []
    for f in SOURCES:
        for m in re.finditer(r"([A-Za-z_]\w*)(?:<[^<>]*>)?\s*<<<", _read(f)):
            if m.group(1) not in PLAIN_OK:
                bare.append((f, m.group(1)))
    assert not bare, bare


def test_launcher_sets_the_programmatic_serialisation_attribute():
    h = open(os.path.join(CSRC, "ps_internal.h")).read()
    assert "cudaLaunchAttributeProgrammaticStreamSerialization" in h
    assert re.search(r"griddepcontrol\.wait;\\n\\tgriddepcontrol\.launch_dependents;", h)
