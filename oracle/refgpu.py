"""ctypes front end of oracle/_ref/libbladeref.so: the reference's own CUDA
direct-space path (src/nbdirect + src/domdec, unmodified), its pair lists,
PME, constraints, MSLD maps and biases and its integrator step, driven by
oracle/ref/ref_harness.cu.  Comparison and golden-vector infrastructure only.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libbladeref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        p, i, f, d = C.c_void_p, C.c_int, C.c_float, C.c_double
        L.ref_create.argtypes = [i, p, p, p, i, p, i, p, i, i, f, f, f, i, i, f, p, p]
        L.ref_set_state.argtypes = [p, p, p]
        L.ref_evaluate.argtypes = [p, i, i, p, p, p]
        L.ref_time.argtypes = [p, p, i, i, i, p, C.c_size_t, p]
        L.ref_list_info.argtypes = [p, p, p]
        L.ref_set_pairs.argtypes = [p, i, p, i, p, i]
        L.ref_evaluate_pairs.argtypes = [p, i, i, p, p, p]
        L.ref_set_pme.argtypes = [p, i, p, p, p]
        L.ref_evaluate_pme.argtypes = [p, i, i, p, p, p]
        L.ref_time_pme.argtypes = [p, i, i, p]
        L.ref_holonomic.argtypes = [p, i, i, p, i, p, i, p, i, p, p, p, p, p, f, f]
        L.ref_set_msld.argtypes = [p, i, p, p, p, p, i, p, f]
        L.ref_set_tric.argtypes = [p, p]
        L.ref_msld_lambda.argtypes = [p, p, p]
        L.ref_msld_theta_force.argtypes = [p, p, p, p, p]
        L.ref_msld_bias.argtypes = [p, p, i, p, p]
        L.ref_update_step.argtypes = [p, p, p, p, p, p, p, i, p, i, p, i, p, i, p, f]
        _lib = L
    return _lib


class RefGPU:
    """The reference path for one synthetic System (AKMA units)."""

    def __init__(self, sys):
        self.sys = sys
        nb = sys.nbonds
        self.N = sys.N
        self.nL = sys.msld.blockCount if sys.msld else 1
        sb = np.ascontiguousarray(nb["siteBlock"], np.int32)
        q = np.ascontiguousarray(nb["q"], np.float32)
        t = np.ascontiguousarray(nb["typeIdx"], np.int32)
        vdw = np.ascontiguousarray(sys.vdw, np.float32)
        ex = np.ascontiguousarray(sys.excl, np.int32)
        box = np.ascontiguousarray(sys.box, np.float64)
        soft = int(bool(sys.msld and sys.msld.useSoftCore))
        h = C.c_void_p()
        P = lambda a: a.ctypes.data_as(C.c_void_p)
        rc = lib().ref_create(self.N, P(sb), P(q), P(t), sys.nTypes, P(vdw), len(ex), P(ex), self.nL, soft,
                              sys.rCut, sys.rSwitch, sys.betaEwald, sys.elecMethod, sys.vdwMethod,
                              sys.cullPad, P(box), C.byref(h))
        if rc != 0:
            raise RuntimeError("reference harness: create failed")
        self.h = h
        if getattr(sys, "tric", None) is not None:   # State::typeBox = true, tricBox from the cell
            self._tric = np.ascontiguousarray(sys.tric_box(), np.float64)
            lib().ref_set_tric(self.h, self._tric.ctypes.data_as(C.c_void_p))

    def set_state(self, xyz=None, lam=None):
        P = lambda a: None if a is None else np.ascontiguousarray(a, np.float64).ctypes.data_as(C.c_void_p)
        x = None if xyz is None else np.ascontiguousarray(xyz, np.float64)
        l = None if lam is None else np.ascontiguousarray(lam, np.float64)
        lib().ref_set_state(self.h, P(x), P(l))

    def evaluate(self, xyz=None, lam=None, reset=True, energy=True):
        self.set_state(self.sys.xyz if xyz is None else xyz, self.sys.lambdas() if lam is None else lam)
        g = np.zeros(3 * self.N)
        e = np.zeros(1)
        lf = np.zeros(self.nL)
        rc = lib().ref_evaluate(self.h, int(reset), int(energy), g.ctypes.data_as(C.c_void_p),
                                e.ctypes.data_as(C.c_void_p), lf.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise RuntimeError("reference harness: evaluate failed")
        return {"grad": g.reshape(-1, 3), "energy": float(e[0]), "lambdaForce": lf}

    def set_pairs(self, soft14=False):
        """The system's nb14 / nbex lists (NB14_DTYPE / NBEX_DTYPE, the reference's layouts)."""
        from blade_b200.systems import NB14_DTYPE, NBEX_DTYPE
        self._p14 = np.ascontiguousarray(self.sys.nb14 if self.sys.nb14 is not None else np.zeros(0, NB14_DTYPE))
        self._pex = np.ascontiguousarray(self.sys.nbex if self.sys.nbex is not None else np.zeros(0, NBEX_DTYPE))
        rc = lib().ref_set_pairs(self.h, len(self._p14), self._p14.ctypes.data_as(C.c_void_p), len(self._pex),
                                 self._pex.ctypes.data_as(C.c_void_p), int(bool(soft14)))
        if rc != 0:
            raise RuntimeError("reference harness: set_pairs failed")

    def evaluate_pairs(self, which="nb14", xyz=None, lam=None, energy=True):
        """getforce_nb14 / getforce_nbex of the reference on the given state."""
        self.set_state(self.sys.xyz if xyz is None else xyz, self.sys.lambdas() if lam is None else lam)
        g = np.zeros(3 * self.N)
        e = np.zeros(1)
        lf = np.zeros(self.nL)
        rc = lib().ref_evaluate_pairs(self.h, 0 if which == "nb14" else 1, int(energy), g.ctypes.data_as(C.c_void_p),
                                      e.ctypes.data_as(C.c_void_p), lf.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise RuntimeError("reference harness: evaluate_pairs failed")
        return {"grad": g.reshape(-1, 3), "energy": float(e[0]), "lambdaForce": lf}

    def set_pme(self, order, K):
        """PME grids and plans for grid K (3 sizes) and B-spline order."""
        self._K = np.ascontiguousarray(K, np.int32)
        self._q = np.ascontiguousarray(self.sys.nbonds["q"], np.float32)
        self._blk = np.ascontiguousarray(self.sys.nbonds["siteBlock"] & 0xFFFF, np.int32)
        P = lambda a: a.ctypes.data_as(C.c_void_p)
        if lib().ref_set_pme(self.h, int(order), P(self._K), P(self._q), P(self._blk)) != 0:
            raise RuntimeError("reference harness: set_pme failed")

    def evaluate_pme(self, which="recip", xyz=None, lam=None, energy=True):
        """getforce_ewald (which="recip") or getforce_ewaldself (which="self") of the reference."""
        self.set_state(self.sys.xyz if xyz is None else xyz, self.sys.lambdas() if lam is None else lam)
        g = np.zeros(3 * self.N)
        e = np.zeros(1)
        lf = np.zeros(self.nL)
        rc = lib().ref_evaluate_pme(self.h, 0 if which == "recip" else 1, int(energy), g.ctypes.data_as(C.c_void_p),
                                    e.ctypes.data_as(C.c_void_p), lf.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise RuntimeError("reference harness: evaluate_pme failed")
        return {"grad": g.reshape(-1, 3), "energy": float(e[0]), "lambdaForce": lf}

    def time_pme(self, reps, energy_every=10):
        """Device time (ms) of `reps` getforce_ewald calls on the current state."""
        ms = C.c_double()
        if lib().ref_time_pme(self.h, int(reps), int(energy_every), C.byref(ms)) != 0:
            raise RuntimeError("reference harness: time_pme failed")
        return ms.value

    def time(self, frames_d, steps, rebuild_every=10, energy_every=10, flush=None):
        """Device time (ms) of `steps` steps over a torch float64 CUDA tensor [steps, 3N]."""
        ms = C.c_double()
        fptr = C.c_void_p(flush.data_ptr()) if flush is not None else None
        fbytes = flush.numel() * flush.element_size() if flush is not None else 0
        rc = lib().ref_time(self.h, C.c_void_p(frames_d.data_ptr()), int(steps), int(rebuild_every), int(energy_every),
                            fptr, C.c_size_t(fbytes), C.byref(ms))
        if rc != 0:
            raise RuntimeError("reference harness: timing failed")
        return ms.value


def holonomic(which, tri, b1, b2, b3, x_prev, x, v, ism, halfdt, tolerance):
    """The reference's holonomic_position (which="position") or
    holonomic_velocity (which="velocity") on the given clusters
    (TriangleCons / Branch*Cons layouts) and state; returns (x, v) with the
    reference's precisions (x double, v and ism float)."""
    N = len(x_prev)
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    z = np.zeros(N, np.int32)
    zf = np.zeros(N, np.float32)
    vdw = np.zeros(2, np.float32)
    box = np.full(3, 100.0)
    h = C.c_void_p()
    if lib().ref_create(N, P(z), P(zf), P(z), 1, P(vdw), 0, None, 1, 0, 9.0, 8.0, 0.34, 1, 0, 2.0, P(box),
                        C.byref(h)) != 0:
        raise RuntimeError("reference harness: create failed")
    xp = np.ascontiguousarray(x_prev, np.float64).reshape(-1)
    xo = np.ascontiguousarray(x, np.float64).reshape(-1).copy()
    vo = np.ascontiguousarray(v, np.float32).reshape(-1).copy()
    im = np.ascontiguousarray(ism, np.float32).reshape(-1)
    arrs = [np.ascontiguousarray(a) for a in (tri, b1, b2, b3)]
    ptr = lambda a: P(a) if len(a) else None
    rc = lib().ref_holonomic(h, 0 if which == "position" else 1, len(arrs[0]), ptr(arrs[0]), len(arrs[1]),
                             ptr(arrs[1]), len(arrs[2]), ptr(arrs[2]), len(arrs[3]), ptr(arrs[3]), P(xp), P(xo),
                             P(vo), P(im), float(halfdt), float(tolerance))
    if rc != 0:
        raise RuntimeError("reference harness: holonomic failed")
    return xo.reshape(-1, 3), vo.reshape(-1, 3)


class RefMsld:
    """The reference's Msld lambda maps, biases and State::update step on a
    given MSLD layout (ref_set_msld, ref_msld_*, ref_update_step)."""

    def __init__(self, site_bound, lambda_site, fnex=5.5, fixed=None, fixed_bias=None, var_bias=None,
                 n_atoms=1, box=(100.0, 100.0, 100.0)):
        from blade_b200.msld import VARBIAS_DTYPE
        self.nL = len(lambda_site)
        self.N = n_atoms
        P = lambda a: a.ctypes.data_as(C.c_void_p)
        z = np.zeros(n_atoms, np.int32)
        zf = np.zeros(n_atoms, np.float32)
        vdw = np.zeros(2, np.float32)
        b = np.ascontiguousarray(box, np.float64)
        h = C.c_void_p()
        if lib().ref_create(n_atoms, P(z), P(zf), P(z), 1, P(vdw), 0, None, self.nL, 0, 9.0, 8.0, 0.34, 1, 0, 2.0,
                            P(b), C.byref(h)) != 0:
            raise RuntimeError("reference harness: create failed")
        self.h = h
        self._sb = np.ascontiguousarray(site_bound, np.int32)
        self._ls = np.ascontiguousarray(lambda_site, np.int32)
        self._fx = np.ascontiguousarray(np.zeros(self.nL) if fixed is None else fixed, np.uint8)
        self._fb = np.ascontiguousarray(np.zeros(self.nL) if fixed_bias is None else fixed_bias, np.float32)
        self._vb = np.ascontiguousarray(np.zeros(0, VARBIAS_DTYPE) if var_bias is None else var_bias, VARBIAS_DTYPE)
        rc = lib().ref_set_msld(self.h, len(self._sb) - 1, P(self._sb), P(self._ls), P(self._fx), P(self._fb),
                                len(self._vb), P(self._vb) if len(self._vb) else None, float(fnex))
        if rc != 0:
            raise RuntimeError("reference harness: set_msld failed")

    def lambda_from_theta(self, theta):
        th = np.ascontiguousarray(theta, np.float64)
        lam = np.zeros(self.nL)
        if lib().ref_msld_lambda(self.h, th.ctypes.data_as(C.c_void_p), lam.ctypes.data_as(C.c_void_p)) != 0:
            raise RuntimeError("reference harness: msld_lambda failed")
        return lam

    def theta_force(self, lam_f, theta_f, lforce_f):
        a = [np.ascontiguousarray(x, np.float32) for x in (lam_f, theta_f, lforce_f)]
        out = np.zeros(self.nL, np.float32)
        P = lambda x: x.ctypes.data_as(C.c_void_p)
        if lib().ref_msld_theta_force(self.h, P(a[0]), P(a[1]), P(a[2]), P(out)) != 0:
            raise RuntimeError("reference harness: msld_theta_force failed")
        return out

    def bias(self, lam_f, energy=True):
        lf = np.ascontiguousarray(lam_f, np.float32)
        out = np.zeros(self.nL, np.float32)
        e = np.zeros(1)
        P = lambda x: x.ctypes.data_as(C.c_void_p)
        if lib().ref_msld_bias(self.h, P(lf), int(energy), P(out), P(e)) != 0:
            raise RuntimeError("reference harness: msld_bias failed")
        return out, float(e[0])

    def update_step(self, pos, vel, frc, ism, random, lp, tri=None, b1=None, b2=None, b3=None, tolerance=2e-7):
        """One State::update (non-energy step): returns (pos, vel, frc) after
        the step, in the layouts documented at ref_update_step."""
        from blade_b200.holonomic import TRI_DTYPE, B1_DTYPE, B2_DTYPE, B3_DTYPE
        pos = np.ascontiguousarray(pos, np.float64).copy()
        vel = np.ascontiguousarray(vel, np.float32).copy()
        frc = np.ascontiguousarray(frc, np.float32).copy()
        ism = np.ascontiguousarray(ism, np.float32)
        rnd = np.ascontiguousarray(random, np.float32)
        lp = np.ascontiguousarray(lp, np.float32)
        arrs = [np.ascontiguousarray(np.zeros(0, dt) if a is None else a, dt)
                for a, dt in ((tri, TRI_DTYPE), (b1, B1_DTYPE), (b2, B2_DTYPE), (b3, B3_DTYPE))]
        P = lambda x: x.ctypes.data_as(C.c_void_p)
        ptr = lambda x: P(x) if len(x) else None
        rc = lib().ref_update_step(self.h, P(pos), P(vel), P(frc), P(ism), P(rnd), P(lp), len(arrs[0]), ptr(arrs[0]),
                                   len(arrs[1]), ptr(arrs[1]), len(arrs[2]), ptr(arrs[2]), len(arrs[3]),
                                   ptr(arrs[3]), float(tolerance))
        if rc != 0:
            raise RuntimeError("reference harness: update_step failed")
        return pos, vel, frc
