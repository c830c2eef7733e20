"""Host side of the direct-space path: the Domdec / getforce_nbdirect mirror.

``NbDirect`` owns one libbnb handle for one system or a batch of replicas and
exposes the reference's calling surface for this path:

* ``update_domdec(positions, reset)``  -- Domdec::update_domdec
  (src/domdec/domdec.cu:213-222): ``reset=True`` rebuilds the block list
  (reset_domdec), otherwise nothing happens until the next force call.
* ``getforce_nbdirect(positions, lambdas, calc_energy, ...)`` -- the entry
  point of src/nbdirect/nbdirect.cu:574: pack, recull, pair kernel, unpack.
  Like the reference, outputs are accumulated into caller buffers (dU/dx in
  ``force``, dU/dlambda in ``lambda_force``, energy in ``energy``); the exact
  fixed-point totals are also available as FP64 (``force64`` etc.).

Device memory and streams come from torch (plumbing only); every kernel is
in libbnb.so.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from .systems import NBOND_DTYPE, System


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def params_for(sys: System) -> _lib.Params:
    p = _lib.Params()
    _lib.lib().bnb_default_params(C.byref(p))
    p.rCut, p.rSwitch, p.betaEwald = sys.rCut, sys.rSwitch, sys.betaEwald
    p.elecMethod, p.vdwMethod = sys.elecMethod, sys.vdwMethod
    p.useSoftCore = int(bool(sys.msld and sys.msld.useSoftCore))
    p.cullPad = sys.cullPad
    return p


class NbDirect:
    """One handle over ``systems`` (a System or a list of replicas)."""

    def __init__(self, systems: System | Sequence[System], device=None):
        import torch
        self.systems = [systems] if isinstance(systems, System) else list(systems)
        s0 = self.systems[0]
        for s in self.systems[1:]:
            if (s.rCut, s.rSwitch, s.betaEwald, s.elecMethod, s.vdwMethod, s.cullPad) != \
               (s0.rCut, s0.rSwitch, s0.betaEwald, s0.elecMethod, s0.vdwMethod, s0.cullPad):
                raise ValueError("replicas of one handle share cutoffs and methods")
        self.device = torch.device(device if device is not None else "cuda")
        self.R = len(self.systems)
        self.counts = np.array([s.N for s in self.systems], np.int32)
        self.starts = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        self.N = int(self.starts[-1])
        self.lam_counts = np.array([s.msld.blockCount if s.msld else 1 for s in self.systems], np.int32)
        self.lam_starts = np.concatenate([[0], np.cumsum(self.lam_counts)]).astype(np.int64)
        self.L = int(self.lam_starts[-1])
        self.params = params_for(s0)
        self.params.useSoftCore = int(any(bool(s.msld and s.msld.useSoftCore) for s in self.systems))
        h = C.c_void_p()
        _lib.call("bnb_create", C.byref(self.params), self.R, self.counts.ctypes.data_as(C.c_void_p), C.byref(h))
        self.h = h
        self._set_topology()
        # triclinic cells (any replica): every boxes argument is State::tricBox_f
        # per replica (A_x, B_x, B_y, C_x, C_y, C_z); bnb_set_box_type
        self.triclinic = any(s.tric is not None for s in self.systems)
        if self.triclinic:
            _lib.call("bnb_set_box_type", self.h, 1)
            self.boxes = np.concatenate([s.tric_box() for s in self.systems]).astype(np.float32)
        else:
            self.boxes = np.concatenate([np.asarray(s.box, np.float32) for s in self.systems]).astype(np.float32)

    # -- topology --------------------------------------------------------------
    def _set_topology(self):
        nb = np.ascontiguousarray(np.concatenate([s.nbonds for s in self.systems]).astype(NBOND_DTYPE))
        types = np.array([s.nTypes for s in self.systems], np.int32)
        vdw = np.ascontiguousarray(np.concatenate([s.vdw.reshape(-1, 2) for s in self.systems]), np.float32)
        excl = [s.excl.astype(np.int32) for s in self.systems]
        exr = np.ascontiguousarray(np.concatenate([np.full(len(e), r, np.int32) for r, e in enumerate(excl)]))
        ex = np.ascontiguousarray(np.concatenate(excl) if excl else np.zeros((0, 2), np.int32))
        _lib.call("bnb_set_topology", self.h, nb.ctypes.data_as(C.c_void_p), types.ctypes.data_as(C.c_void_p),
                  vdw.ctypes.data_as(C.c_void_p), self.lam_counts.ctypes.data_as(C.c_void_p), len(ex),
                  ex.ctypes.data_as(C.c_void_p), exr.ctypes.data_as(C.c_void_p))

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().bnb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference calling surface ---------------------------------------------
    def update_domdec(self, positions, reset: bool, stream=None, asynchronous: bool = False,
                      boxes=None):
        """Domdec::update_domdec: rebuild the list when ``reset`` is true."""
        if not reset:
            return
        b = np.ascontiguousarray(self.boxes if boxes is None else boxes, np.float32)
        _lib.call("bnb_rebuild", self.h, _ptr(positions), b.ctypes.data_as(C.c_void_p), _stream(stream),
                  _lib.BNB_ASYNC if asynchronous else 0)

    reset_domdec = lambda self, positions, stream=None: self.update_domdec(positions, True, stream)

    def getforce_nbdirect(self, positions, lambdas=None, calc_energy=True, force=None,
                          lambda_force=None, energy=None, force64=None, lambda_force64=None,
                          energy64=None, stream=None, boxes=None, mode=0):
        """bnb_compute; ``mode`` ORs in BNB_OUT_SET / BNB_OUT_ADD64 (output modes)."""
        out = _lib.Outputs(force=_ptr(force), lambdaForce=_ptr(lambda_force), energy=_ptr(energy),
                           force64=_ptr(force64), lambdaForce64=_ptr(lambda_force64), energy64=_ptr(energy64))
        b = np.ascontiguousarray(self.boxes if boxes is None else boxes, np.float32)
        _lib.call("bnb_compute", self.h, _ptr(positions), _ptr(lambdas), b.ctypes.data_as(C.c_void_p),
                  int(bool(calc_energy)) | int(mode), C.byref(out), _stream(stream))

    # -- nb14 / nbex pair lists (getforce_nb14 / getforce_nbex) ---------------------
    def set_pairs(self, soft14: bool = False):
        """Uploads every replica's ``nb14`` / ``nbex`` lists (bnb_set_pairs),
        with atom and block indices shifted to the concatenated layout."""
        from .systems import NB14_DTYPE, NBEX_DTYPE
        n14, nex = [], []
        for r, s in enumerate(self.systems):
            for src, dst, dt in ((s.nb14, n14, NB14_DTYPE), (s.nbex, nex, NBEX_DTYPE)):
                if src is None or len(src) == 0:
                    continue
                a = np.array(src, dt)
                a["idx"] += int(self.starts[r])
                blk = a["siteBlock"] & 0xFFFF
                a["siteBlock"] = np.where(blk != 0, (a["siteBlock"] & ~0xFFFF) | (blk + int(self.lam_starts[r])), 0)
                dst.append(a)
        a14 = np.ascontiguousarray(np.concatenate(n14) if n14 else np.zeros(0, NB14_DTYPE))
        aex = np.ascontiguousarray(np.concatenate(nex) if nex else np.zeros(0, NBEX_DTYPE))
        _lib.call("bnb_set_pairs", self.h, len(a14), a14.ctypes.data_as(C.c_void_p) if len(a14) else None,
                  len(aex), aex.ctypes.data_as(C.c_void_p) if len(aex) else None, int(bool(soft14)))

    def getforce_pairs(self, which: str, positions, lambdas=None, calc_energy=True, force=None,
                       lambda_force=None, energy=None, force64=None, lambda_force64=None, energy64=None,
                       stream=None, boxes=None, mode=0):
        """bnb_compute_nb14 (which="nb14") or bnb_compute_nbex (which="nbex")."""
        out = _lib.Outputs(force=_ptr(force), lambdaForce=_ptr(lambda_force), energy=_ptr(energy),
                           force64=_ptr(force64), lambdaForce64=_ptr(lambda_force64), energy64=_ptr(energy64))
        b = np.ascontiguousarray(self.boxes if boxes is None else boxes, np.float32)
        _lib.call("bnb_compute_" + which, self.h, _ptr(positions), _ptr(lambdas), b.ctypes.data_as(C.c_void_p),
                  int(bool(calc_energy)) | int(mode), C.byref(out), _stream(stream))

    def evaluate_pairs(self, which: str, positions=None, lambdas=None, calc_energy=True):
        import torch
        pos = self.positions_tensor() if positions is None else positions
        lam = self.lambdas_tensor() if lambdas is None else lambdas
        f64 = torch.zeros(3 * self.N, dtype=torch.float64, device=self.device)
        l64 = torch.zeros(self.L, dtype=torch.float64, device=self.device)
        e64 = torch.zeros(self.R, dtype=torch.float64, device=self.device)
        self.getforce_pairs(which, pos, lam, calc_energy, force64=f64, lambda_force64=l64, energy64=e64)
        return f64.reshape(-1, 3), l64, e64

    # -- PME reciprocal space and Ewald self term (getforce_ewald / getforce_ewaldself)
    def set_pme(self, order: int = 6, grid_space: float = 1.0, grid=None):
        """bnb_set_pme: one grid per replica, from ``grid`` ([R,3] sizes) or
        the reference's rule for ``grid_space`` (Run::gridSpace, 1 A)."""
        b = np.ascontiguousarray(self.boxes, np.float32)
        g = None if grid is None else np.ascontiguousarray(np.broadcast_to(np.asarray(grid, np.int32),
                                                                           (self.R, 3)))
        _lib.call("bnb_set_pme", self.h, int(order), float(grid_space),
                  None if g is None else g.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p))

    def pme_grid(self, replica: int = 0):
        K = np.zeros(3, np.int32)
        _lib.call("bnb_pme_grid", self.h, int(replica), K.ctypes.data_as(C.c_void_p))
        return tuple(int(k) for k in K)

    def getforce_ewald(self, positions, lambdas=None, calc_energy=True, force=None, lambda_force=None,
                       energy=None, force64=None, lambda_force64=None, energy64=None, stream=None, boxes=None,
                       mode=0):
        """bnb_compute_pme (getforce_ewald)."""
        out = _lib.Outputs(force=_ptr(force), lambdaForce=_ptr(lambda_force), energy=_ptr(energy),
                           force64=_ptr(force64), lambdaForce64=_ptr(lambda_force64), energy64=_ptr(energy64))
        b = np.ascontiguousarray(self.boxes if boxes is None else boxes, np.float32)
        _lib.call("bnb_compute_pme", self.h, _ptr(positions), _ptr(lambdas), b.ctypes.data_as(C.c_void_p),
                  int(bool(calc_energy)) | int(mode), C.byref(out), _stream(stream))

    def getforce_ewaldself(self, lambdas=None, calc_energy=True, lambda_force=None, energy=None,
                           lambda_force64=None, energy64=None, stream=None, mode=0):
        """bnb_compute_ewald_self (getforce_ewaldself)."""
        out = _lib.Outputs(lambdaForce=_ptr(lambda_force), energy=_ptr(energy), lambdaForce64=_ptr(lambda_force64),
                           energy64=_ptr(energy64))
        _lib.call("bnb_compute_ewald_self", self.h, _ptr(lambdas), int(bool(calc_energy)) | int(mode), C.byref(out),
                  _stream(stream))

    def evaluate_pme(self, positions=None, lambdas=None, calc_energy=True):
        """Reciprocal term with fresh FP64 outputs: (dU/dx [N,3], dU/dlambda [L], energy [R])."""
        import torch
        pos = self.positions_tensor() if positions is None else positions
        lam = self.lambdas_tensor() if lambdas is None else lambdas
        f64 = torch.zeros(3 * self.N, dtype=torch.float64, device=self.device)
        l64 = torch.zeros(self.L, dtype=torch.float64, device=self.device)
        e64 = torch.zeros(self.R, dtype=torch.float64, device=self.device)
        self.getforce_ewald(pos, lam, calc_energy, force64=f64, lambda_force64=l64, energy64=e64)
        return f64.reshape(-1, 3), l64, e64

    def evaluate_ewald_self(self, lambdas=None):
        import torch
        lam = self.lambdas_tensor() if lambdas is None else lambdas
        l64 = torch.zeros(self.L, dtype=torch.float64, device=self.device)
        e64 = torch.zeros(self.R, dtype=torch.float64, device=self.device)
        self.getforce_ewaldself(lam, True, lambda_force64=l64, energy64=e64)
        return l64, e64

    # -- tuning -------------------------------------------------------------------
    def set_tuning(self, tiles_per_work: int, ctas_per_sm: int = 0, tail_items: int = 2):
        """bnb_set_tuning: candidate tiles per work item (1..32), resident CTAs
        per SM of the persistent pair kernel (0 = occupancy) and the work-list
        tail (0..8 full items' worth of each block's tiles in quarter-size
        items at the end); the next rebuild applies it."""
        _lib.call("bnb_set_tuning", self.h, int(tiles_per_work), int(ctas_per_sm), int(tail_items))

    def tuning(self) -> dict:
        """bnb_get_tuning."""
        t, c, l = C.c_int(), C.c_int(), C.c_int()
        _lib.call("bnb_get_tuning", self.h, C.byref(t), C.byref(c), C.byref(l))
        return {"tiles_per_work": t.value, "ctas_per_sm": c.value, "tail_items": l.value}

    def autotune(self, positions, lambdas=None, reps: int = 5, stream=None) -> dict:
        """bnb_autotune: tries tiles per work item x CTAs per SM x tail on this
        system, keeps the fastest (median of ``reps``), rebuilds the list;
        returns the choice."""
        best = C.c_float()
        b = np.ascontiguousarray(self.boxes, np.float32)
        _lib.call("bnb_autotune", self.h, _ptr(positions), _ptr(lambdas), b.ctypes.data_as(C.c_void_p), int(reps),
                  _stream(stream), C.byref(best))
        return dict(self.tuning(), best_ms=best.value)

    # -- conveniences ------------------------------------------------------------
    def positions_tensor(self, xyz_list=None):
        import torch
        xs = xyz_list if xyz_list is not None else [s.xyz for s in self.systems]
        return torch.from_numpy(np.ascontiguousarray(np.concatenate(xs), np.float32)).to(self.device).reshape(-1)

    def lambdas_tensor(self, lam_list=None):
        import torch
        ls = lam_list if lam_list is not None else [s.lambdas() for s in self.systems]
        return torch.from_numpy(np.concatenate(ls).astype(np.float32)).to(self.device)

    def evaluate(self, positions=None, lambdas=None, calc_energy=True, stream=None):
        """One evaluation with fresh FP64 outputs: (force64 [N,3], dU/dlambda [L], energy [R])."""
        import torch
        pos = self.positions_tensor() if positions is None else positions
        lam = self.lambdas_tensor() if lambdas is None else lambdas
        f64 = torch.zeros(3 * self.N, dtype=torch.float64, device=self.device)
        l64 = torch.zeros(self.L, dtype=torch.float64, device=self.device)
        e64 = torch.zeros(self.R, dtype=torch.float64, device=self.device)
        self.getforce_nbdirect(pos, lam, calc_energy, force64=f64, lambda_force64=l64, energy64=e64,
                               stream=stream)
        return f64.reshape(-1, 3), l64, e64

    def status(self, clear=False, stream=None) -> int:
        v = C.c_int()
        _lib.call("bnb_status", self.h, _stream(stream), int(clear), C.byref(v))
        return v.value

    def reserve(self, tiles=0, masks=0, work=0):
        """Preset list capacities before the next rebuild (bnb_reserve)."""
        _lib.call("bnb_reserve", self.h, int(tiles), int(masks), int(work))

    def profile(self, on: bool):
        """Record CUDA events around the pair kernel and list rebuilds."""
        _lib.call("bnb_profile", self.h, int(on))

    def profile_read(self, reset=True):
        pm, rm = C.c_double(), C.c_double()
        pn, rn = C.c_int(), C.c_int()
        kl = C.c_ulonglong()
        _lib.call("bnb_profile_read", self.h, C.byref(pm), C.byref(pn), C.byref(rm), C.byref(rn),
                  C.byref(kl), int(reset))
        return {"pair_ms": pm.value, "pair_launches": pn.value, "rebuild_ms": rm.value,
                "rebuilds": rn.value, "kernel_launches": kl.value}

    def set_counting(self, on: bool):
        _lib.call("bnb_set_counting", self.h, int(on))

    def pair_count(self, stream=None) -> int:
        v = C.c_ulonglong()
        _lib.call("bnb_pair_count", self.h, _stream(stream), C.byref(v))
        return v.value

    def list_sizes(self, stream=None):
        v = [C.c_int() for _ in range(4)]
        _lib.call("bnb_list_sizes", self.h, _stream(stream), *[C.byref(x) for x in v])
        return {"blocks": v[0].value, "tiles": v[1].value, "masks": v[2].value, "work": v[3].value}

    def get_list(self, stream=None):
        sz = self.list_sizes(stream)
        B, T, M = sz["blocks"], sz["tiles"], sz["masks"]
        wrap = np.zeros(self.N, np.int32)
        bb = np.zeros(B + 1, np.int32)
        sa = np.zeros(self.N, np.int32)
        slot = np.zeros(32 * B, np.int32)
        bmin = np.zeros((B, 3), np.float32)
        bmax = np.zeros((B, 3), np.float32)
        cs = np.zeros(B + 1, np.int32)
        cand = np.zeros((T, 2), np.int32)
        cm = np.zeros(T, np.int32)
        masks = np.zeros((M, 32), np.uint32)
        P = lambda a: a.ctypes.data_as(C.c_void_p)
        _lib.call("bnb_get_list", self.h, _stream(stream), P(wrap), P(bb), P(sa), P(slot), P(bmin), P(bmax),
                  P(cs), P(cand), P(cm), P(masks))
        return {"blockCount": B, "wrap": wrap, "blockBounds": bb, "sortedAtom": sa, "slotAtom": slot,
                "bmin": bmin, "bmax": bmax, "candStart": cs, "cand": cand, "candExcl": cm, "masks": masks}


def domain_div(n: int, box) -> tuple[int, int]:
    b = np.ascontiguousarray(box, np.float32)
    x, y = C.c_int(), C.c_int()
    _lib.call("bnb_domain_div", n, b.ctypes.data_as(C.c_void_p), C.byref(x), C.byref(y))
    return x.value, y.value
