"""libbnb called from plain C (tests/c_abi/abi_calls.c), the way BLaDE's C++
step loop links it: the program compiles against include/bnb.h with gcc and
links libbnb.so and the CUDA runtime, with no Python in the call path.  On the
CPU it checks arguments and call order; on the GPU it evaluates the 216-water
box and must give the bits of the Python host mirror."""
import os
import subprocess

import numpy as np
import pytest

from blade_b200 import _lib, systems

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(tmp_path):
    exe = tmp_path / "abi_calls"
    libdir = os.path.dirname(_lib.LIB_PATH)
    cmd = ["gcc", "-std=c11", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "c_abi", "abi_calls.c"), "-o", str(exe), "-L", libdir, "-l:libbnb.so",
           "-Wl,-rpath," + libdir, "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_caller_argument_checks(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "abi checks ok" in r.stdout


@pytest.mark.gpu
def test_c_caller_evaluates_like_python(cuda, tmp_path):
    from blade_b200.nbdirect import NbDirect, params_for
    s = systems.water_box()
    p = params_for(s)
    excl = np.ascontiguousarray(s.excl, np.int32)
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        f.write(np.array([s.N, s.nTypes, len(excl)], np.int32).tobytes())
        f.write(np.ascontiguousarray(s.box, np.float32).tobytes())
        f.write(bytes(p))
        f.write(np.ascontiguousarray(s.xyz, np.float32).tobytes())
        f.write(np.ascontiguousarray(s.nbonds).tobytes())
        f.write(np.ascontiguousarray(s.vdw, np.float32).tobytes())
        f.write(excl.tobytes())
    out = tmp_path / "out.bin"
    exe = _build(tmp_path)
    r = subprocess.run([str(exe), str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    res = np.fromfile(out, np.float64)
    f_c, e_c = res[:-1].reshape(-1, 3), res[-1]
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    f_py, _, e_py = nb.evaluate(pos)
    assert np.array_equal(f_c, f_py.cpu().numpy())
    assert e_c == float(e_py[0].cpu())
    nb.close()
