"""Holonomic bond constraints on the GPU (bnb_holonomic_position /
bnb_holonomic_velocity), the counterpart of holonomic_position /
holonomic_velocity (src/holonomic/holonomic.cu:238-758).

Clusters use the reference's layouts (TriangleCons, Branch1Cons, Branch2Cons,
Branch3Cons, src/system/potential.h:120-138): a rigid triangle (water) or a
heavy atom with 1-3 hydrogens.  torch holds the device arrays; the solver is
libbnb's kernel.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

TRI_DTYPE = np.dtype([("idx", "<i4", 3), ("b0", "<f4", 3)])
B1_DTYPE = np.dtype([("idx", "<i4", 2), ("b0", "<f4", 1)])
B2_DTYPE = np.dtype([("idx", "<i4", 3), ("b0", "<f4", 2)])
B3_DTYPE = np.dtype([("idx", "<i4", 4), ("b0", "<f4", 3)])


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class Constraints:
    def __init__(self, tri=None, b1=None, b2=None, b3=None, device="cuda"):
        import torch
        self.torch = torch
        arrays = []
        for a, dt in ((tri, TRI_DTYPE), (b1, B1_DTYPE), (b2, B2_DTYPE), (b3, B3_DTYPE)):
            a = np.zeros(0, dt) if a is None else np.ascontiguousarray(np.asarray(a, dt))
            t = torch.from_numpy(a.view(np.uint8).copy()).to(device) if len(a) else None
            arrays.append((len(a), t))
        self._keep = arrays
        self.set = _lib.ConstraintSet(arrays[0][0], arrays[1][0], arrays[2][0], arrays[3][0],
                                      *[None if t is None else t.data_ptr() for _, t in arrays])
        self.count = sum(n for n, _ in arrays)

    def _s(self, stream):
        return C.c_void_p((stream or self.torch.cuda.current_stream()).cuda_stream)

    def position(self, x_prev, x, v, ism, halfdt, tolerance=1e-10, max_iter=10, x_f=None, status=None,
                 stream=None):
        """x, v updated in place (device double [3N]); v may be None."""
        _lib.call("bnb_holonomic_position", C.byref(self.set), _p(x_prev), _p(x), _p(v), _p(ism), float(halfdt),
                  float(tolerance), int(max_iter), _p(x_f), _p(status), self._s(stream))

    def velocity(self, x, v, ism, stream=None):
        _lib.call("bnb_holonomic_velocity", C.byref(self.set), _p(x), _p(v), _p(ism), self._s(stream))


def water_triangles(first_atom: int, n_water: int, r_oh: float = 0.9572, r_hh: float = 1.5139) -> np.ndarray:
    """Rigid TIP3P triangles for waters stored O, H, H from first_atom."""
    t = np.zeros(n_water, TRI_DTYPE)
    base = first_atom + 3 * np.arange(n_water)
    t["idx"] = np.stack([base, base + 1, base + 2], 1)
    t["b0"] = (r_oh, r_oh, r_hh)
    return t
