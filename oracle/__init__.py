"""ctypes front end of the CPU oracle (test infrastructure only).

Imported by tests/, by ``__graft_entry__.smoke()`` as the checker and by
``bench.py`` for the CPU baseline.  The product never imports this package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class _Params(C.Structure):
    _fields_ = [("rCut", C.c_double), ("rSwitch", C.c_double), ("betaEwald", C.c_double),
                ("elecMethod", C.c_int), ("vdwMethod", C.c_int), ("calcAlch", C.c_int),
                ("useSoftCore", C.c_int), ("kElectric", C.c_double), ("softCoreRadius", C.c_double)]


class _List(C.Structure):
    _fields_ = [("N", C.c_int), ("divX", C.c_int), ("divY", C.c_int), ("nCols", C.c_int),
                ("blockCount", C.c_int),
                ("wrap", C.POINTER(C.c_int)), ("colCount", C.POINTER(C.c_int)),
                ("blockBounds", C.POINTER(C.c_int)), ("sortedAtom", C.POINTER(C.c_int)),
                ("slotAtom", C.POINTER(C.c_int)), ("bmin", C.POINTER(C.c_float)),
                ("bmax", C.POINTER(C.c_float)), ("candCount", C.c_int),
                ("candStart", C.POINTER(C.c_int)), ("cand", C.POINTER(C.c_int)),
                ("candExcl", C.POINTER(C.c_int)), ("maskCount", C.c_int),
                ("masks", C.POINTER(C.c_uint32))]


class _VarBias(C.Structure):
    _fields_ = [("i", C.c_int), ("j", C.c_int), ("type", C.c_int), ("l0", C.c_float),
                ("k", C.c_float), ("n", C.c_int)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", _HERE], check=True)
        _LIB = C.CDLL(path)
        d, i, f, p = C.c_double, C.c_int, C.c_float, C.c_void_p
        _LIB.orc_nbdirect.argtypes = [i, p, p, p, i, p, i, p, C.POINTER(_Params), p, i, p, p, p, p, i]
        _LIB.orc_nbdirect_brute.argtypes = [i, p, p, p, i, p, i, p, C.POINTER(_Params), p, i, p, p, p, p]
        _LIB.orc_nbdirect64.argtypes = _LIB.orc_nbdirect.argtypes
        _LIB.orc_nbdirect_window64.argtypes = _LIB.orc_nbdirect.argtypes + [i, i]
        _LIB.orc_nbdirect_brute64.argtypes = _LIB.orc_nbdirect_brute.argtypes
        _LIB.orc_nbdirect_tric64.argtypes = _LIB.orc_nbdirect_brute.argtypes
        _LIB.orc_shift_table.argtypes = [p, p]
        _LIB.orc_pair.argtypes = [d, d, d, d, d, i, i, d, d, C.POINTER(_Params), p, p, p, p]
        _LIB.orc_lambda_from_theta.argtypes = [i, p, d, p, p, p]
        _LIB.orc_thetaForce_from_lambdaForce.argtypes = [i, p, p, d, p, p, p, p, p]
        _LIB.orc_bias.argtypes = [i, p, p, i, p, p, p]
        _LIB.orc_domain_div.argtypes = [i, p, p, p]
        _LIB.orc_build_list.argtypes = [i, p, p, f, p, p, C.POINTER(_List)]
        _LIB.orc_free_list.argtypes = [C.POINTER(_List)]
        _LIB.orc_pack.argtypes = [C.POINTER(_List), p, p, p, p, p]
        _LIB.orc_shift_vector.argtypes = [i, p, p, p]
        _LIB.orc_aabb_hit.argtypes = [p, p, p, p, p, f]
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def params(sys, alch=None):
    m = sys.msld
    calc = (m is not None and m.blockCount > 1) if alch is None else alch
    return _Params(sys.rCut, sys.rSwitch, sys.betaEwald, sys.elecMethod, sys.vdwMethod,
                   int(calc), int(bool(m and m.useSoftCore)), 332.0716, 4.0)


def nbdirect(sys, lam=None, xyz=None, brute=False, nthreads=0, calc_alch=None):
    """FP64 direct-space energy, gradient dU/dx [N,3], dU/dlambda, pair count.

    ``xyz`` defaults to the system's FP32 coordinates; a float64 array is used
    as is (finite-difference tests)."""
    f64 = xyz is not None and np.asarray(xyz).dtype == np.float64
    xyz = np.ascontiguousarray(sys.xyz if xyz is None else xyz, np.float64 if f64 else np.float32)
    N = xyz.shape[0]
    box = np.ascontiguousarray(sys.box, np.float64)
    nb = np.ascontiguousarray(sys.nbonds)
    vdw = np.ascontiguousarray(sys.vdw, np.float32)
    excl = np.ascontiguousarray(sys.excl, np.int32)
    if lam is None:
        lam = sys.lambdas()
    lam = np.ascontiguousarray(lam, np.float64)
    g = np.zeros((N, 3))
    lf = np.zeros(len(lam))
    e = np.zeros(1)
    cnt = np.zeros(1, np.int64)
    p = params(sys, calc_alch)
    if sys.tric is not None:           # triclinic cell: all-pairs over lattice images
        x64 = np.ascontiguousarray(xyz, np.float64)
        b6 = np.ascontiguousarray(sys.box6(), np.float64)
        rc = lib().orc_nbdirect_tric64(N, _ptr(x64), _ptr(b6), _ptr(nb), sys.nTypes, _ptr(vdw), len(excl),
                                       _ptr(excl), C.byref(p), _ptr(lam), len(lam), _ptr(g), _ptr(lf), _ptr(e),
                                       _ptr(cnt))
    elif brute:
        fn = lib().orc_nbdirect_brute64 if f64 else lib().orc_nbdirect_brute
        rc = fn(N, _ptr(xyz), _ptr(box), _ptr(nb), sys.nTypes, _ptr(vdw), len(excl), _ptr(excl),
                C.byref(p), _ptr(lam), len(lam), _ptr(g), _ptr(lf), _ptr(e), _ptr(cnt))
    else:
        fn = lib().orc_nbdirect64 if f64 else lib().orc_nbdirect
        rc = fn(N, _ptr(xyz), _ptr(box), _ptr(nb), sys.nTypes, _ptr(vdw), len(excl), _ptr(excl),
                C.byref(p), _ptr(lam), len(lam), _ptr(g), _ptr(lf), _ptr(e), _ptr(cnt), int(nthreads))
    if rc != 0:
        raise ValueError("oracle: box smaller than twice the cutoff")
    return {"grad": g, "lambdaForce": lf, "energy": float(e[0]), "pairs": int(cnt[0])}


class Sampler:
    """Repeated oracle evaluations of a bounded sample (pairs whose lower atom
    index falls in a window) -- the timed CPU baseline."""

    def __init__(self, sys, nthreads=0):
        self.sys = sys
        self.N = sys.N
        self.box = np.ascontiguousarray(sys.box, np.float64)
        self.nb = np.ascontiguousarray(sys.nbonds)
        self.vdw = np.ascontiguousarray(sys.vdw, np.float32)
        self.excl = np.ascontiguousarray(sys.excl, np.int32)
        self.lam = np.ascontiguousarray(sys.lambdas(), np.float64)
        self.p = params(sys)
        self.nthreads = nthreads
        self.g = np.zeros((self.N, 3))
        self.lf = np.zeros(len(self.lam))
        self.e = np.zeros(1)
        self.cnt = np.zeros(1, np.int64)

    def run(self, xyz64, i0, i1):
        x = np.ascontiguousarray(xyz64, np.float64)
        rc = lib().orc_nbdirect_window64(self.N, _ptr(x), _ptr(self.box), _ptr(self.nb), self.sys.nTypes,
                                         _ptr(self.vdw), len(self.excl), _ptr(self.excl), C.byref(self.p),
                                         _ptr(self.lam), len(self.lam), _ptr(self.g), _ptr(self.lf),
                                         _ptr(self.e), _ptr(self.cnt), int(self.nthreads), int(i0), int(i1))
        if rc != 0:
            raise ValueError("oracle: box smaller than twice the cutoff")
        return int(self.cnt[0])


def pair(r, qi, qj, c12, c6, bi, bj, li, lj, sys_or_params):
    p = sys_or_params if isinstance(sys_or_params, _Params) else params(sys_or_params)
    out = np.zeros(4)
    lib().orc_pair(r, qi, qj, c12, c6, bi, bj, li, lj, C.byref(p),
                   _ptr(out[0:1]), _ptr(out[1:2]), _ptr(out[2:3]), _ptr(out[3:4]))
    return out


def lambda_from_theta(site_bound, fnex, theta, fixed=None):
    sb = np.ascontiguousarray(site_bound, np.int32)
    th = np.ascontiguousarray(theta, np.float64)
    fx = None if fixed is None else np.ascontiguousarray(fixed, np.int32)
    lam = np.zeros_like(th)
    lib().orc_lambda_from_theta(len(sb) - 1, _ptr(sb), fnex, _ptr(th), _ptr(fx), _ptr(lam))
    return lam


def theta_force(lambda_site, site_bound, fnex, lam, theta, lforce, fixed=None):
    ls = np.ascontiguousarray(lambda_site, np.int32)
    sb = np.ascontiguousarray(site_bound, np.int32)
    lam = np.ascontiguousarray(lam, np.float64)
    th = np.ascontiguousarray(theta, np.float64)
    lf = np.ascontiguousarray(lforce, np.float64)
    fx = None if fixed is None else np.ascontiguousarray(fixed, np.int32)
    out = np.zeros(len(ls))
    lib().orc_thetaForce_from_lambdaForce(len(ls), _ptr(ls), _ptr(sb), fnex, _ptr(lam), _ptr(th),
                                          _ptr(lf), _ptr(fx), _ptr(out))
    return out


VARBIAS_DTYPE = np.dtype([("i", "<i4"), ("j", "<i4"), ("type", "<i4"), ("l0", "<f4"),
                          ("k", "<f4"), ("n", "<i4")])


def bias(lam, fixed_bias, varbias):
    lam = np.ascontiguousarray(lam, np.float64)
    fb = None if fixed_bias is None else np.ascontiguousarray(fixed_bias, np.float64)
    vb = np.ascontiguousarray(varbias, VARBIAS_DTYPE)
    lf = np.zeros(len(lam))
    e = np.zeros(1)
    lib().orc_bias(len(lam), _ptr(lam), _ptr(fb), len(vb), _ptr(vb), _ptr(lf), _ptr(e))
    return lf, float(e[0])


def domain_div(N, box):
    b = np.ascontiguousarray(box, np.float32)
    x = np.zeros(1, np.int32)
    y = np.zeros(1, np.int32)
    lib().orc_domain_div(N, _ptr(b), _ptr(x), _ptr(y))
    return int(x[0]), int(y[0])


def build_list(sys, xyz=None, rcull=None):
    """FP32/integer block list: same structures as the CUDA builder exports."""
    from blade_b200.systems import excl_csr
    xyz = np.ascontiguousarray(sys.xyz if xyz is None else xyz, np.float32)
    box = np.ascontiguousarray(sys.box6(), np.float32)
    N = xyz.shape[0]
    es, ea = excl_csr(N, sys.excl)
    rc = np.float32(sys.rCut) + np.float32(sys.cullPad) if rcull is None else np.float32(rcull)
    L = _List()
    lib().orc_build_list(N, _ptr(xyz), _ptr(box), C.c_float(rc), _ptr(es), _ptr(ea), C.byref(L))
    B = L.blockCount

    def arr(ptr, n, dt):
        return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt).copy() if n > 0 else np.zeros(0, dt)
    out = {
        "divX": L.divX, "divY": L.divY, "blockCount": B,
        "wrap": arr(L.wrap, N, np.int32), "colCount": arr(L.colCount, L.nCols, np.int32),
        "blockBounds": arr(L.blockBounds, B + 1, np.int32), "sortedAtom": arr(L.sortedAtom, N, np.int32),
        "slotAtom": arr(L.slotAtom, 32 * B, np.int32),
        "bmin": arr(L.bmin, 3 * B, np.float32).reshape(B, 3), "bmax": arr(L.bmax, 3 * B, np.float32).reshape(B, 3),
        "candStart": arr(L.candStart, B + 1, np.int32),
        "cand": arr(L.cand, 2 * L.candCount, np.int32).reshape(-1, 2),
        "candExcl": arr(L.candExcl, L.candCount, np.int32),
        "masks": arr(L.masks, 32 * L.maskCount, np.uint32).reshape(-1, 32),
    }
    lib().orc_free_list(C.byref(L))
    return out


def shift_vector(code):
    x = np.zeros(1, np.int32); y = np.zeros(1, np.int32); z = np.zeros(1, np.int32)
    lib().orc_shift_vector(code, _ptr(x), _ptr(y), _ptr(z))
    return int(x[0]), int(y[0]), int(z[0])


def box6_of(box):
    """A box argument as the 6-float cell (A_x, B_y, C_z, B_x, C_x, C_y):
    3 edges (orthorhombic) are padded with zeros."""
    b = np.asarray(box, np.float32).reshape(-1)
    return np.ascontiguousarray(np.concatenate([b, np.zeros(6 - len(b), np.float32)]) if len(b) < 6 else b[:6])


def shift_table(box):
    """[14,3] image shift vectors of the half-shell codes for a box (3 or 6 floats)."""
    t = np.zeros((14, 3), np.float32)
    lib().orc_shift_table(_ptr(box6_of(box)), _ptr(t))
    return t


def pack(lst, xyz, box):
    """Pack with stored wrap shifts; returns packed [32B,3] and AABBs.
    box: 3 edges or the 6-float cell."""
    B = lst["blockCount"]
    L = _List()
    L.N = len(xyz)
    L.blockCount = B
    wrap = np.ascontiguousarray(lst["wrap"], np.int32)
    slot = np.ascontiguousarray(lst["slotAtom"], np.int32)
    L.wrap = wrap.ctypes.data_as(C.POINTER(C.c_int))
    L.slotAtom = slot.ctypes.data_as(C.POINTER(C.c_int))
    x = np.ascontiguousarray(xyz, np.float32)
    b = box6_of(box)
    packed = np.zeros((32 * B, 3), np.float32)
    mn = np.zeros((B, 3), np.float32)
    mx = np.zeros((B, 3), np.float32)
    lib().orc_pack(C.byref(L), _ptr(x), _ptr(b), _ptr(packed), _ptr(mn), _ptr(mx))
    return packed, mn, mx


def active_tiles(lst, bmin, bmax, box, rcut):
    """Per-step recull at rCut: boolean per candidate (recull.cu:41-122)."""
    c2 = np.float32(np.float32(rcut) * np.float32(rcut))
    out = np.zeros(len(lst["cand"]), bool)
    table = shift_table(box)
    for i in range(lst["blockCount"]):
        for c in range(lst["candStart"][i], lst["candStart"][i + 1]):
            j, code = lst["cand"][c]
            s = table[int(code)]
            out[c] = bool(lib().orc_aabb_hit(_ptr(np.ascontiguousarray(bmin[i])),
                                             _ptr(np.ascontiguousarray(bmax[i])),
                                             _ptr(np.ascontiguousarray(bmin[j])),
                                             _ptr(np.ascontiguousarray(bmax[j])),
                                             _ptr(np.ascontiguousarray(s, np.float32)), C.c_float(c2)))
    return out


NB14_DTYPE = np.dtype([("idx", "<i4", 2), ("siteBlock", "<i4", 2), ("qxq", "<f4"), ("c12", "<f4"), ("c6", "<f4"),
                       ("e14fac", "<f4")])
NBEX_DTYPE = np.dtype([("idx", "<i4", 2), ("siteBlock", "<i4", 2), ("qxq", "<f4")])


def pair_lists(sys, xyz=None, lam=None, which="nb14", soft14=False):
    """FP64 nb14 or nbex energy, gradient dU/dx [N,3] and dU/dlambda
    (src/bonded/pair.cu) for the system's pair lists."""
    xyz = np.ascontiguousarray(sys.xyz if xyz is None else xyz, np.float64)
    box = np.ascontiguousarray(sys.box6(), np.float64)
    lam = np.ascontiguousarray(sys.lambdas() if lam is None else lam, np.float64)
    g = np.zeros((xyz.shape[0], 3))
    lf = np.zeros(len(lam))
    e = np.zeros(1)
    p = params(sys, True)
    if which == "nb14":
        pp = np.ascontiguousarray(sys.nb14, NB14_DTYPE)
        lib().orc_nb14_pairs(len(pp), _ptr(pp), _ptr(xyz), _ptr(box), _ptr(lam), C.byref(p), int(soft14),
                             _ptr(g), _ptr(lf), _ptr(e))
    else:
        pp = np.ascontiguousarray(sys.nbex, NBEX_DTYPE)
        lib().orc_nbex_pairs(len(pp), _ptr(pp), _ptr(xyz), _ptr(box), _ptr(lam), C.byref(p), _ptr(g), _ptr(lf),
                             _ptr(e))
    return {"grad": g, "lambdaForce": lf, "energy": float(e[0])}

