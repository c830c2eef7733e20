"""MSLD lambda maps and biases on the device (wrappers over libbnb).

Counterparts of Msld::calc_lambda_from_theta, calc_thetaForce_from_lambdaForce
and getforce_fixedBias/getforce_variableBias (src/msld/msld.cu:863-1153).
Arguments are torch CUDA tensors (int32 indices, float64 values, uint8
block-fixed flags in the layout of the reference's bool array).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

VARBIAS_DTYPE = np.dtype([("i", "<i4"), ("j", "<i4"), ("type", "<i4"), ("l0", "<f4"), ("k", "<f4"), ("n", "<i4")])


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _s(stream):
    import torch
    return C.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)


def lambda_from_theta(site_bound, fnex, theta, lam, lam_f=None, fixed=None, stream=None):
    _lib.call("bnb_lambda_from_theta", site_bound.numel() - 1, _p(site_bound), float(fnex), _p(theta),
              _p(fixed), _p(lam), _p(lam_f), _s(stream))


def theta_force(lambda_site, site_bound, fnex, lam, theta, lambda_force, theta_force_out, fixed=None,
                stream=None):
    _lib.call("bnb_theta_force", lambda_site.numel(), _p(lambda_site), _p(site_bound), float(fnex), _p(lam),
              _p(theta), _p(lambda_force), _p(fixed), _p(theta_force_out), _s(stream))


def theta_force_f32(lambda_site, site_bound, fnex, lam_f, theta_f, lambda_force_f, theta_force_f, fixed=None,
                    stream=None):
    """Same on the reference's FP32 State buffers (computed in FP64)."""
    _lib.call("bnb_theta_force_f32", lambda_site.numel(), _p(lambda_site), _p(site_bound), float(fnex),
              _p(lam_f), _p(theta_f), _p(lambda_force_f), _p(fixed), _p(theta_force_f), _s(stream))


def bias(lam, fixed_bias, var_bias, lambda_force, energy=None, stream=None):
    """var_bias: torch uint8 tensor holding VARBIAS_DTYPE records (or None)."""
    nvar = 0 if var_bias is None else var_bias.numel() // VARBIAS_DTYPE.itemsize
    _lib.call("bnb_bias", lam.numel(), _p(lam), _p(fixed_bias), nvar, _p(var_bias), _p(lambda_force),
              _p(energy), _s(stream))
