"""C ABI checks that need no GPU: the library loads, exports every entry point
declared in include/bnb.h, validates arguments, and its host-side heuristics
agree with the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
from blade_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?[a-z_]+\s*\**\s*(bnb_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_version_string():
    assert b"sm_100a" in _lib.lib().bnb_version()


def test_default_params():
    p = _lib.Params()
    _lib.lib().bnb_default_params(C.byref(p))
    assert (p.rCut, p.rSwitch, p.elecMethod, p.vdwMethod) == (12.0, 10.0, 1, 0)
    assert p.kElectric == pytest.approx(332.0716)
    assert p.softCoreRadius == 4.0


@pytest.mark.parametrize("n,box", [(648, 18.856), (23558, 62.23), (3000, 31.4), (30000, 67.74), (1, 30.0)])
def test_domain_div_matches_oracle(n, box):
    b = np.full(3, box, np.float32)
    x, y = C.c_int(), C.c_int()
    assert _lib.lib().bnb_domain_div(n, b.ctypes.data_as(C.c_void_p), C.byref(x), C.byref(y)) == 0
    assert (x.value, y.value) == oracle.domain_div(n, b)


def test_create_rejects_bad_arguments():
    lib = _lib.lib()
    p = _lib.Params()
    lib.bnb_default_params(C.byref(p))
    h = C.c_void_p()
    counts = np.array([10], np.int32)
    cp = counts.ctypes.data_as(C.c_void_p)
    bad = [("elecMethod", 3), ("vdwMethod", -1), ("rCut", 0.0), ("rSwitch", 20.0), ("cullPad", -1.0)]
    for field, val in bad:
        q = _lib.Params.from_buffer_copy(p)
        setattr(q, field, val)
        assert lib.bnb_create(C.byref(q), 1, cp, C.byref(h)) == _lib.BNB_ERR_ARG
    assert lib.bnb_create(C.byref(p), 0, cp, C.byref(h)) == _lib.BNB_ERR_ARG
    assert lib.bnb_create(None, 1, cp, C.byref(h)) == _lib.BNB_ERR_ARG
    # a valid handle can be created and destroyed without touching the GPU
    assert lib.bnb_create(C.byref(p), 1, cp, C.byref(h)) == 0
    assert lib.bnb_rebuild(h, None, np.zeros(3, np.float32).ctypes.data_as(C.c_void_p), None, 0) == _lib.BNB_ERR_ARG
    assert lib.bnb_destroy(h) == 0


def test_call_order_is_checked():
    lib = _lib.lib()
    p = _lib.Params()
    lib.bnb_default_params(C.byref(p))
    h = C.c_void_p()
    counts = np.array([0], np.int32)
    assert lib.bnb_create(C.byref(p), 1, counts.ctypes.data_as(C.c_void_p), C.byref(h)) == 0
    box = np.full(3, 40.0, np.float32)
    # rebuild before topology
    assert lib.bnb_rebuild(h, None, box.ctypes.data_as(C.c_void_p), None, 0) == _lib.BNB_ERR_STATE
    out = _lib.Outputs()
    assert lib.bnb_compute(h, None, None, box.ctypes.data_as(C.c_void_p), 1, C.byref(out), None) == _lib.BNB_ERR_STATE
    lib.bnb_destroy(h)


def test_no_fallback_when_library_missing(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError):
        _lib.lib()


def test_pme_call_order_and_arguments():
    lib = _lib.lib()
    p = _lib.Params()
    lib.bnb_default_params(C.byref(p))
    h = C.c_void_p()
    counts = np.array([0], np.int32)
    assert lib.bnb_create(C.byref(p), 1, counts.ctypes.data_as(C.c_void_p), C.byref(h)) == 0
    box = np.full(3, 40.0, np.float32)
    bp = box.ctypes.data_as(C.c_void_p)
    out = _lib.Outputs()
    K = np.zeros(3, np.int32)
    for order in (0, 3, 5, 10):                      # orders 4, 6, 8 only (nbrecip.cu:537-545)
        assert lib.bnb_set_pme(h, order, C.c_float(1.0), None, bp) == _lib.BNB_ERR_ARG
    assert lib.bnb_set_pme(h, 6, C.c_float(0.0), None, bp) == _lib.BNB_ERR_ARG   # no spacing, no grid
    assert lib.bnb_set_pme(h, 6, C.c_float(1.0), None, None) == _lib.BNB_ERR_ARG
    assert lib.bnb_set_pme(h, 6, C.c_float(1.0), None, bp) == _lib.BNB_ERR_STATE  # before the topology
    assert lib.bnb_pme_grid(h, 0, K.ctypes.data_as(C.c_void_p)) == _lib.BNB_ERR_STATE
    assert lib.bnb_compute_pme(h, None, None, bp, 1, C.byref(out), None) == _lib.BNB_ERR_STATE
    assert lib.bnb_compute_ewald_self(h, None, 1, C.byref(out), None) == _lib.BNB_ERR_STATE
    assert lib.bnb_compute_pme(h, None, None, None, 1, C.byref(out), None) == _lib.BNB_ERR_ARG
    lib.bnb_destroy(h)


def test_constraint_and_split_step_arguments():
    lib = _lib.lib()
    x = np.zeros(9)
    xp = x.ctypes.data_as(C.c_void_p)
    empty = _lib.ConstraintSet(0, 0, 0, 0, None, None, None, None)
    assert lib.bnb_holonomic_position(None, xp, xp, None, xp, 0.02, 1e-10, 10, None, None, None) == _lib.BNB_ERR_ARG
    bad = _lib.ConstraintSet(-1, 0, 0, 0, None, None, None, None)
    assert lib.bnb_holonomic_position(C.byref(bad), xp, xp, None, xp, 0.02, 1e-10, 10, None, None,
                                      None) == _lib.BNB_ERR_ARG
    missing = _lib.ConstraintSet(2, 0, 0, 0, None, None, None, None)   # a count without its array
    assert lib.bnb_holonomic_velocity(C.byref(missing), xp, xp, xp, None) == _lib.BNB_ERR_ARG
    for halfdt, tol, it in ((0.0, 1e-10, 10), (0.02, 0.0, 10), (0.02, 1e-10, 0)):
        assert lib.bnb_holonomic_position(C.byref(empty), xp, xp, None, xp, halfdt, tol, it, None, None,
                                          None) == _lib.BNB_ERR_ARG
    # nothing to constrain: success without a launch
    assert lib.bnb_holonomic_position(C.byref(empty), xp, xp, None, xp, 0.02, 1e-10, 10, None, None, None) == 0
    assert lib.bnb_holonomic_velocity(C.byref(empty), xp, xp, xp, None) == 0
    args = (xp, xp, xp, xp, xp, xp, xp, xp, xp, 0.04, 0.9, 0.3, 0.9, 0.3, C.c_ulonglong(1), C.c_ulonglong(0),
            None, None, None, None)
    assert lib.bnb_langevin_half(2, 3, 0, *args) == _lib.BNB_ERR_ARG
    assert lib.bnb_langevin_half(0, 0, 0, *args) == 0
    assert lib.bnb_langevin_half(0, 3, 0, xp, xp, None, None, xp, None, None, None, None, 0.04, 0.9, 0.3, 0.9,
                                 0.3, C.c_ulonglong(1), C.c_ulonglong(0), None, None, None, None) == _lib.BNB_ERR_ARG
