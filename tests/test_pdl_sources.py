"""Programmatic dependent launch, checked in the sources (CPU): a kernel
launched with launch_pdl may start before the kernel ahead of it in the
stream has finished, so its first statement must be pdl_wait(), which
returns once that kernel has completed and its writes are visible.  Every
kernel that any .cu file of the library passes to launch_pdl is looked up
and its body must open with that call."""
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "blade_b200", "csrc")


def _sources():
    return {os.path.basename(p): open(p).read() for p in glob.glob(os.path.join(CSRC, "*.cu"))}


def _launched(src):
    """Kernel names passed to launch_pdl (template arguments stripped), local
    aliases (`auto k = k_pair<...>;`) resolved to the kernel they name."""
    alias = {m.group(1): m.group(2) for m in re.finditer(r"auto\s+(\w+)\s*=\s*([A-Za-z_]\w*)\s*<", src)}
    names = set()
    for m in re.finditer(r"launch_pdl\(\s*([A-Za-z_]\w*)", src):
        names.add(alias.get(m.group(1), m.group(1)))
    return names


def _bodies(src, name):
    """Opening statements of every __global__ definition of `name`."""
    pat = re.compile(r"__global__\s+void\s+(?:__launch_bounds__\([^)]*\)\s+)?" + re.escape(name) + r"\s*\(")
    out = []
    for m in pat.finditer(src):
        depth, i = 0, m.end() - 1
        while True:                      # skip the parameter list
            c = src[i]
            depth += c == "("
            depth -= c == ")"
            i += 1
            if depth == 0:
                break
        brace = src.index("{", i)
        body = src[brace + 1:brace + 400]
        body = re.sub(r"//[^\n]*", "", body)
        out.append(body.strip())
    return out


def test_every_pdl_kernel_waits_first():
    srcs = _sources()
    launched = set()
    for src in srcs.values():
        launched |= _launched(src)
    assert {"k_pair", "k_finalize", "k_order", "k_pack", "k_cull", "k_spread", "k_gather"} <= launched
    allsrc = "\n".join(srcs.values())
    for name in sorted(launched):
        bodies = _bodies(allsrc, name)
        assert bodies, f"no definition of {name}"
        for b in bodies:
            assert b.startswith("pdl_wait();"), (name, b[:80])


def test_pdl_wait_is_the_grid_dependency_wait():
    hdr = open(os.path.join(CSRC, "bnb_internal.h")).read()
    assert "cudaGridDependencySynchronize()" in hdr
    assert "cudaLaunchAttributeProgrammaticStreamSerialization" in hdr
