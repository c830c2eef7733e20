"""Batched MSLD stepping: many replicas in one launch sequence under a CUDA graph.

A step (the same for the batched and the one-at-a-time runs) is
  list maintenance (rebuild every ``rebuild_every`` steps, asynchronous),
  direct-space forces with MSLD scaling and soft core (bnb_compute),
  harmonic bonds of the systems' covalent topology (bnb_bond_gradient),
  dU/dlambda -> dU/dtheta (bnb_theta_force),
  Langevin VRORV update of coordinates and theta (bnb_langevin_vrorv),
  theta -> lambda (bnb_lambda_from_theta),
mirroring Run::dynamics (src/run/run.cu:554-564) and State::update
(src/update/update.cu:233-305) without PME reciprocal and angles/dihedrals;
the bonds (TIP3P O-H and H-H included) stand in for the reference's bonded
terms and keep molecules whole.  With ``constraints=True`` the waters are
rigid instead (holonomic triangles, src/holonomic/holonomic.cu): the update
is split at its middle (bnb_langevin_half) and bnb_holonomic_position follows
each half drift, as update_VVhbpR / holonomic_position / update_OOhbpR /
holonomic_position do (update.cu:276-303), with true hydrogen masses and
the water bonds dropped.  With ``pme=True`` the electrostatics are complete:
the 1-4 pairs and exclusion corrections (bnb_compute_nb14 / bnb_compute_nbex,
lists from systems.with_pair_lists), PME reciprocal space and the Ewald self
term (bnb_compute_pme / bnb_compute_ewald_self), as Potential::calc_force
sums them (src/system/potential.cxx:1851-1941); each adds into the step's FP64
force and dU/dlambda (BNB_OUT_ADD64), so no per-term buffers or additions.  All replicas share one libbnb handle, so every kernel of a step
covers all of them; ``capture`` records ``rebuild_every`` steps in one CUDA
graph that is replayed.  Units are AKMA; dt is 2 fs.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib, holonomic
from .nbdirect import NbDirect
from . import systems
from .systems import System

KB = 0.001987191                 # kcal/mol/K (src/main/defines.h:53)
PICOSECOND = 20.454828284385908  # AKMA time units per ps (defines.h:51)
# Hydrogen mass repartitioning (3.024 amu per H, taken from its oxygen): the
# step has no bonded terms or constraints, so heavier hydrogens keep the
# coordinates' drift per list period within the pad.
MASS_H, MASS_O, MASS_HEAVY = 3.024, 15.9994 - 2 * (3.024 - 1.008), 12.011
THETA_MASS = 12.0                # amu A^2, the usual MSLD theta mass
SHAKE_TOL, SHAKE_ITERS = 1e-10, 10  # FP64 state; the reference's FP32-era default is 2e-7 (run.cu:64)


def atom_masses(s: System, repartition: bool = True) -> np.ndarray:
    """Water H/O by type index (0 = HT, 1 = OT in the generators), heavy atoms
    otherwise; hydrogen mass repartitioning unless ``repartition`` is false."""
    t = s.nbonds["typeIdx"]
    m = np.full(s.N, MASS_HEAVY)
    m[t == 0] = MASS_H if repartition else 1.008
    m[t == 1] = MASS_O if repartition else 15.9994
    return m


def water_oxygens(s: System) -> np.ndarray:
    """First atom of every O, H, H water (types 1, 0, 0 in the generators)."""
    t = s.nbonds["typeIdx"]
    i = np.nonzero(t[:-2] == 1)[0]
    return i[(t[i + 1] == 0) & (t[i + 2] == 0)]


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class MsldBatch:
    """State and step of R MSLD replicas on one GPU."""

    def __init__(self, reps: list[System], dt_fs: float = 2.0, T: float = 300.0, gamma_ps: float = 1.0,
                 seed: int = 1, rebuild_every: int = 10, energy_every: int = 10, device="cuda", tune=False,
                 theta_mass: float = THETA_MASS, gamma_theta_ps: float | None = None, constraints: bool = False,
                 pme: bool = False, pme_order: int = 6):
        import torch
        self.torch = torch
        if pme:                                            # 1-4 pairs join the exclusions; nbex lists
            reps = [systems.with_pair_lists(s) for s in reps]
        self.reps = reps
        self.dev = torch.device(device)
        self.nb = NbDirect(reps, device=self.dev)
        self.rebuild_every = rebuild_every
        self.energy_every = energy_every
        self.seed = seed
        self.step_index = 0
        N = self.nb.N
        f64, f32, i32 = torch.float64, torch.float32, torch.int32
        x = np.concatenate([s.xyz.astype(np.float64) for s in reps]).reshape(-1)
        self.x = torch.from_numpy(x).to(self.dev)
        self.xf = self.x.float()
        masses = np.concatenate([atom_masses(s, repartition=not constraints) for s in reps])
        rng = np.random.default_rng(seed)
        kT = KB * T
        vx = rng.normal(size=(N, 3)) * np.sqrt(kT / masses)[:, None]
        self.v = torch.from_numpy(vx.reshape(-1)).to(self.dev)
        self.ismx = torch.from_numpy(np.repeat(1 / np.sqrt(masses), 3)).to(self.dev)
        self.force = torch.zeros(3 * N, dtype=f64, device=self.dev)
        bonds, prm, tri = [], [], []
        for r, s in enumerate(reps):
            keep = np.ones(0 if s.bonds is None else len(s.bonds), bool)
            if constraints:
                ox = water_oxygens(s)
                tri.append(holonomic.water_triangles(0, len(ox)))
                tri[-1]["idx"] = (ox[:, None] + np.arange(3)[None, :] + int(self.nb.starts[r])).astype(np.int32)
                wat = np.zeros(s.N, bool)
                wat[(ox[:, None] + np.arange(3)).reshape(-1)] = True
                if s.bonds is not None and len(s.bonds):
                    keep = ~(wat[s.bonds[:, 0]] & wat[s.bonds[:, 1]])
            if s.bonds is not None and keep.any():
                bonds.append(s.bonds[keep].astype(np.int64) + self.nb.starts[r])
                prm.append(s.bond_param[keep])
        self.cons = holonomic.Constraints(tri=np.concatenate(tri), device=self.dev) if constraints else None
        self.x_prev = torch.zeros(3 * N, dtype=f64, device=self.dev) if constraints else None
        self.cons_status = torch.zeros(1, dtype=i32, device=self.dev)
        self.cons_tol, self.cons_iters = SHAKE_TOL, SHAKE_ITERS
        self.bond_start = None
        if bonds:
            st, pa, pr = systems.bond_csr(N, np.concatenate(bonds), np.concatenate(prm))
            self.bond_start = torch.from_numpy(st).to(self.dev)
            self.bond_partner = torch.from_numpy(pa).to(self.dev)
            self.bond_param = torch.from_numpy(pr.reshape(-1)).to(self.dev)
        # MSLD: global blocks = concatenation of each replica's blocks; block 0
        # of every replica is its environment (site 0, lambda fixed at 1)
        theta, bound, site, fixed = [], [0], [], []
        site_base = 0
        for s in reps:
            m = s.msld
            if m is None:
                theta.append([0.0]); site.append([site_base]); bound.append(bound[-1] + 1)
                fixed.append([1]); site_base += 1
                continue
            th = m.theta.copy()
            th[0] = 1.0                                    # environment: fixed block, lambda = theta = 1
            theta.append(th)
            fx = np.zeros(m.blockCount, np.uint8)
            fx[0] = 1
            fixed.append(fx)
            site.append(m.lambdaSite + site_base)
            for k in range(1, m.siteCount + 1):
                bound.append(bound[-1] + int(m.siteBound[k] - m.siteBound[k - 1]))
            site_base += m.siteCount
        self.theta = torch.from_numpy(np.concatenate(theta).astype(np.float64)).to(self.dev)
        L = self.theta.numel()
        assert L == self.nb.L
        self.site_bound = torch.from_numpy(np.array(bound, np.int32)).to(self.dev)
        self.lambda_site = torch.from_numpy(np.concatenate(site).astype(np.int32)).to(self.dev)
        self.fixed = torch.from_numpy(np.concatenate(fixed).astype(np.uint8)).to(self.dev)
        self.fnex = reps[0].msld.fnex if reps[0].msld else 5.5
        ism_t = np.full(L, 1 / math.sqrt(theta_mass))
        ism_t[np.concatenate(fixed).astype(bool)] = np.inf  # frozen, as fixed blocks in the reference
        self.ismt = torch.from_numpy(ism_t).to(self.dev)
        self.vt = torch.from_numpy(rng.normal(size=L) * math.sqrt(kT / theta_mass)).to(self.dev)
        self.vt[self.fixed.bool()] = 0
        self.lam = torch.zeros(L, dtype=f64, device=self.dev)
        self.lamf = torch.zeros(L, dtype=f32, device=self.dev)
        self.lforce = torch.zeros(L, dtype=f64, device=self.dev)
        self.tforce = torch.zeros(L, dtype=f64, device=self.dev)
        self.energy = torch.zeros(self.nb.R, dtype=f64, device=self.dev)
        self.nan = torch.zeros(1, dtype=i32, device=self.dev)
        self.step_counter = torch.zeros(2, dtype=torch.int64, device=self.dev)  # RNG step, blocks done
        # integrator constants (State::alloc_leapparms2)
        self.dt = dt_fs * 1e-3 * PICOSECOND
        a = math.exp(-gamma_ps / PICOSECOND * self.dt)
        self.fric = a
        self.noise = math.sqrt((1 - a * a) * kT)
        at = a if gamma_theta_ps is None else math.exp(-gamma_theta_ps / PICOSECOND * self.dt)
        self.fric_t = at                                  # theta friction (Msld gamma, msld.cu:46, 232-235)
        self.noise_t = math.sqrt((1 - at * at) * kT)
        self._lambda_from_theta()
        if self.cons is not None:                          # start on the constraint surface
            self.cons.velocity(self.x, self.v, self.ismx)
        self.fixed_bias = None                             # lambda biases (set_bias)
        self.var_bias = None
        self.hist1 = None                                  # lambda histograms (enable_histograms)
        self.pme = pme
        if pme:
            self.nb.set_pairs()
            self.nb.set_pme(order=pme_order)
        self.nb.update_domdec(self.xf, True)               # synchronous first build sizes the list
        if tune:
            self.tuned_ms = self.autotune()
        self.graph = None

    # -- kernels of one step ------------------------------------------------------
    def _lambda_from_theta(self, stream=None):
        _lib.call("bnb_lambda_from_theta", self.site_bound.numel() - 1, _p(self.site_bound), float(self.fnex),
                  _p(self.theta), _p(self.fixed), _p(self.lam), _p(self.lamf), self._s(stream))

    def _s(self, stream):
        return C.c_void_p((stream or self.torch.cuda.current_stream()).cuda_stream)

    def enqueue_step(self, k: int, stream=None):
        s = self._s(stream)
        nb = self.nb
        if k % self.rebuild_every == 0:
            nb.update_domdec(self.xf, True, asynchronous=True, stream=stream)
        calc_e = self.energy_every > 0 and k % self.energy_every == 0
        nb.getforce_nbdirect(self.xf, self.lamf, calc_e, force64=self.force, lambda_force64=self.lforce,
                             energy64=self.energy if calc_e else None, stream=stream)
        if self.bond_start is not None:
            _lib.call("bnb_bond_gradient", self.nb.N, _p(self.bond_start), _p(self.bond_partner),
                      _p(self.bond_param), _p(self.x), _p(self.force), s)
        if self.pme:                                       # the other electrostatic terms of calc_force,
            add = _lib.BNB_OUT_ADD64                       # each added into the step's FP64 outputs
            e = self.energy if calc_e else None
            for term in ("nb14", "nbex"):
                nb.getforce_pairs(term, self.xf, self.lamf, calc_e, force64=self.force, lambda_force64=self.lforce,
                                  energy64=e, stream=stream, mode=add)
            nb.getforce_ewald(self.xf, self.lamf, calc_e, force64=self.force, lambda_force64=self.lforce,
                              energy64=e, stream=stream, mode=add)
            nb.getforce_ewaldself(self.lamf, calc_e, lambda_force64=self.lforce, energy64=e, stream=stream, mode=add)
        if self.fixed_bias is not None:
            _lib.call("bnb_bias", self.theta.numel(), _p(self.lam), _p(self.fixed_bias), self.n_var,
                      _p(self.var_bias), _p(self.lforce), None, s)
        self.tforce.zero_()
        _lib.call("bnb_theta_force", self.lambda_site.numel(), _p(self.lambda_site), _p(self.site_bound),
                  float(self.fnex), _p(self.lam), _p(self.theta), _p(self.lforce), _p(self.fixed), _p(self.tforce), s)
        if self.cons is None:
            _lib.call("bnb_langevin_vrorv", self.x.numel(), self.theta.numel(), _p(self.x), _p(self.v),
                      _p(self.force), _p(self.ismx), _p(self.theta), _p(self.vt), _p(self.tforce), _p(self.ismt),
                      self.dt, self.fric, self.noise, self.fric_t, self.noise_t, C.c_ulonglong(self.seed),
                      C.c_ulonglong(0), _p(self.step_counter), _p(self.xf), _p(self.nan), s)
        else:
            for phase in (0, 1):                           # VV+R, constrain, OO+R, constrain (update.cu:276-303)
                _lib.call("bnb_langevin_half", phase, self.x.numel(), self.theta.numel(), _p(self.x), _p(self.v),
                          _p(self.x_prev), _p(self.force), _p(self.ismx), _p(self.theta), _p(self.vt),
                          _p(self.tforce), _p(self.ismt), self.dt, self.fric, self.noise, self.fric_t, self.noise_t,
                          C.c_ulonglong(self.seed), C.c_ulonglong(0), _p(self.step_counter), _p(self.xf),
                          _p(self.nan), s)
                self.cons.position(self.x_prev, self.x, self.v, self.ismx, 0.5 * self.dt, self.cons_tol,
                                   self.cons_iters, x_f=self.xf, status=self.cons_status,
                                   stream=stream)
        _lib.call("bnb_lambda_from_theta", self.site_bound.numel() - 1, _p(self.site_bound), float(self.fnex),
                  _p(self.theta), _p(self.fixed), _p(self.lam), _p(self.lamf), s)
        if self.hist1 is not None:
            _lib.call("bnb_lambda_histogram", self.theta.numel(), _p(self.lam), _p(self.fixed), self.n_pairs,
                      _p(self.hist_pairs), _p(self.hist1), _p(self.hist2), _p(self.hist_end), s)

    # -- lambda biases and histograms (adaptive landscape flattening) -------------
    def set_bias(self, fixed: np.ndarray, var: np.ndarray):
        """Fixed bias per global block (FP64 [L]) and variable biases
        (``msld.VARBIAS_DTYPE``, global block indices).  Updating biases of
        the same count rewrites the captured buffers in place, so a recorded
        graph picks them up."""
        torch = self.torch
        fixed_t = torch.from_numpy(np.ascontiguousarray(fixed, np.float64))
        var_t = torch.from_numpy(np.ascontiguousarray(var).view(np.uint8).copy())
        if self.fixed_bias is not None and self.var_bias.numel() == var_t.numel():
            self.fixed_bias.copy_(fixed_t)
            self.var_bias.copy_(var_t)
            return
        self.graph = None
        self.fixed_bias = fixed_t.to(self.dev)
        self.var_bias = var_t.to(self.dev)
        self.n_var = len(var)

    def enable_histograms(self, pairs: np.ndarray):
        """Sample lambda into histograms after every step (bnb_lambda_histogram);
        ``pairs`` [P,2] global block pairs for the 8x8 histograms."""
        torch = self.torch
        L = self.theta.numel()
        self.n_pairs = len(pairs)
        self.hist_pairs = torch.from_numpy(np.ascontiguousarray(pairs, np.int32).reshape(-1)).to(self.dev)
        self.hist1 = torch.zeros(L * 32, dtype=torch.int32, device=self.dev)
        self.hist2 = torch.zeros(max(1, self.n_pairs) * 64, dtype=torch.int32, device=self.dev)
        self.hist_end = torch.zeros(L, dtype=torch.int32, device=self.dev)
        self.graph = None

    def take_histograms(self):
        """(hist1 [L,32], hist2 [P,8,8], endCount [L]) as numpy, then cleared.
        The samples taken are the row sums of hist1 (one count per step)."""
        L = self.theta.numel()
        h1 = self.hist1.cpu().numpy().reshape(L, 32).astype(np.int64)
        h2 = self.hist2.cpu().numpy()[:64 * self.n_pairs].reshape(self.n_pairs, 8, 8).astype(np.int64)
        he = self.hist_end.cpu().numpy().astype(np.int64)
        self.hist1.zero_()
        self.hist2.zero_()
        self.hist_end.zero_()
        return h1, h2, he

    def run_eager(self, nsteps: int):
        for k in range(nsteps):
            self.enqueue_step(k)
        self.step_index += nsteps

    def capture(self):
        """Record ``rebuild_every`` steps (one rebuild, one energy step) as a CUDA graph."""
        torch = self.torch
        side = torch.cuda.Stream(device=self.dev)
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):          # warm-up outside capture
            for k in range(self.rebuild_every):
                self.enqueue_step(k, stream=side)
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for k in range(self.rebuild_every):
                self.enqueue_step(k)
        self.graph = g
        return g

    def run_graph(self, nsteps: int):
        assert self.graph is not None and nsteps % self.rebuild_every == 0
        for _ in range(nsteps // self.rebuild_every):
            self.graph.replay()

    def autotune(self, reps: int = 5) -> float:
        best = C.c_float()
        b = np.ascontiguousarray(self.nb.boxes, np.float32)
        _lib.call("bnb_autotune", self.nb.h, _p(self.xf), _p(self.lamf), b.ctypes.data_as(C.c_void_p), reps,
                  self._s(None), C.byref(best))
        return best.value

    def tuning(self):
        return self.nb.tuning()

    def check(self):
        st = self.nb.status()
        nan = int(self.nan.item())
        return st, nan

    def close(self):
        self.graph = None
        self.nb.close()


def ns_per_day(steps: int, seconds: float, dt_fs: float = 2.0, replicas: int = 1) -> float:
    return replicas * steps * dt_fs * 1e-6 * 86400.0 / seconds
