"""ctypes binding of libbnb.so, the C ABI declared in include/bnb.h.

The library is built in-tree (``__graft_entry__.build()`` or
``make -C blade_b200/csrc``).  There is no fallback: if the shared library is
missing, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbnb.so")

BNB_OK, BNB_ERR_ARG, BNB_ERR_CUDA, BNB_ERR_CAPACITY, BNB_ERR_UNSUPPORTED, BNB_ERR_STATE, BNB_ERR_DEVICE = range(7)
BNB_ASYNC = 1
BNB_OUT_SET, BNB_OUT_ADD64 = 2, 4   # output modes ORed into calcEnergy (include/bnb.h)
STATUS_BLOCK_OVERFLOW, STATUS_TILE_OVERFLOW, STATUS_MASK_OVERFLOW, STATUS_WORK_OVERFLOW, STATUS_NONFINITE = 1, 2, 4, 8, 16
_ERRORS = {1: "bad argument", 2: "CUDA error", 3: "list capacity exceeded", 4: "unsupported",
           5: "call order", 6: "device status", 7: "size above the fixed limit"}


class BnbError(RuntimeError):
    def __init__(self, fn, code):
        super().__init__(f"{fn} failed: {_ERRORS.get(code, code)} ({code})")
        self.code = code


class Params(C.Structure):
    _fields_ = [("rCut", C.c_float), ("rSwitch", C.c_float), ("betaEwald", C.c_float),
                ("elecMethod", C.c_int), ("vdwMethod", C.c_int), ("useSoftCore", C.c_int),
                ("cullPad", C.c_float), ("kElectric", C.c_float), ("softCoreRadius", C.c_float)]


class Outputs(C.Structure):
    _fields_ = [("force", C.c_void_p), ("lambdaForce", C.c_void_p), ("energy", C.c_void_p),
                ("force64", C.c_void_p), ("lambdaForce64", C.c_void_p), ("energy64", C.c_void_p)]


class ConstraintSet(C.Structure):
    _fields_ = [("nTriangle", C.c_int), ("nBranch1", C.c_int), ("nBranch2", C.c_int), ("nBranch3", C.c_int),
                ("triangle", C.c_void_p), ("branch1", C.c_void_p), ("branch2", C.c_void_p), ("branch3", C.c_void_p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libbnb.so not built ({LIB_PATH}); run __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        p, i, f, d = C.c_void_p, C.c_int, C.c_float, C.c_double
        sig = {
            "bnb_default_params": (None, [p]),
            "bnb_create": (i, [p, i, p, p]),
            "bnb_destroy": (i, [p]),
            "bnb_set_topology": (i, [p, p, p, p, p, i, p, p]),
            "bnb_rebuild": (i, [p, p, p, p, i]),
            "bnb_compute": (i, [p, p, p, p, i, p, p]),
            "bnb_status": (i, [p, p, i, p]),
            "bnb_list_sizes": (i, [p, p, p, p, p, p]),
            "bnb_get_list": (i, [p, p, p, p, p, p, p, p, p, p, p, p]),
            "bnb_set_counting": (i, [p, i]),
            "bnb_reserve": (i, [p, i, i, i]),
            "bnb_profile": (i, [p, i]),
            "bnb_fp32_peak": (i, [p, p]),
            "bnb_profile_read": (i, [p, p, p, p, p, p, i]),
            "bnb_pair_count": (i, [p, p, p]),
            "bnb_domain_div": (i, [i, p, p, p]),
            "bnb_lambda_from_theta": (i, [i, p, d, p, p, p, p, p]),
            "bnb_theta_force": (i, [i, p, p, d, p, p, p, p, p, p]),
            "bnb_bias": (i, [i, p, p, i, p, p, p, p]),
            "bnb_theta_force_f32": (i, [i, p, p, d, p, p, p, p, p, p]),
            "bnb_bias_f32": (i, [i, p, p, i, p, p, p, p]),
            "bnb_set_tuning": (i, [p, i, i, i]),
            "bnb_get_tuning": (i, [p, p, p, p]),
            "bnb_autotune": (i, [p, p, p, p, i, p, p]),
            "bnb_set_pairs": (i, [p, i, p, i, p, i]),
            "bnb_compute_nb14": (i, [p, p, p, p, i, p, p]),
            "bnb_compute_nbex": (i, [p, p, p, p, i, p, p]),
            "bnb_nbdirect_noalloc": (i, [p, i, p, p, p, i, p, p, p, i, p, p]),
            "bnb_holonomic_position": (i, [p, p, p, p, p, d, d, i, p, p, p]),
            "bnb_holonomic_velocity": (i, [p, p, p, p, p]),
            "bnb_langevin_half": (i, [i, i, i, p, p, p, p, p, p, p, p, p, d, d, d, d, d, C.c_ulonglong,
                                      C.c_ulonglong, p, p, p, p]),
            "bnb_set_pme": (i, [p, i, f, p, p]),
            "bnb_pme_grid": (i, [p, i, p]),
            "bnb_compute_pme": (i, [p, p, p, p, i, p, p]),
            "bnb_compute_ewald_self": (i, [p, p, i, p, p]),
            "bnb_mlp_linear_forward": (i, [i, i, i, p, p, p, i, p, p, p, p]),
            "bnb_mlp_linear_backward": (i, [i, i, i, p, p, i, p, p, p, p, p, p, p, p]),
            "bnb_mlp_mse": (i, [i, i, p, p, p, p, p, p, p]),
            "bnb_mlp_adam": (i, [i, p, p, p, p, p, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, i, p]),
            "bnb_to_bf16": (i, [i, p, p, p]),
            "bnb_lambda_histogram": (i, [i, p, p, i, p, p, p, p, p]),
            "bnb_bond_gradient": (i, [i, p, p, p, p, p, p]),
            "bnb_langevin_vrorv": (i, [i, i, p, p, p, p, p, p, p, p, d, d, d, d, d, C.c_ulonglong, C.c_ulonglong,
                                       p, p, p, p]),
            "bnb_set_box_type": (i, [p, i]),
            "bnb_version": (C.c_char_p, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(fn: str, code: int):
    if code != BNB_OK:
        raise BnbError(fn, code)


def call(name: str, *args):
    check(name, getattr(lib(), name)(*args))
