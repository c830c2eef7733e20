"""Adaptive landscape flattening (ALF) of MSLD lambda biases: plain and learned.

The reference consumes ALF's result but does not contain ALF: the fixed bias
b (Msld lambdaBias, src/msld/msld.cu:1000-1018) and the variable biases of
type 6 (c, l0 = 0), 10 (x, l0 = -5.56) and 8 (s, l0 = 0.017)
(msld.cu:1055-1066), set from ALF's variable files in
test/T4L/prep/T4L149F.inp:81,105-109.  ALF itself (Hayes, Armacost, Vilseck &
Brooks, J. Phys. Chem. B 121:3626, 2017) is an external package absent from
the reference tree, so the plain update here is written from the published
method and its parity against ALF is unpinned:

  run a short MSLD simulation with the current biases, histogram lambda
  (32-bin 1-D histograms per substituent, 8x8 2-D histograms per substituent
  pair of a site, counts of end states lambda > 0.99), and change the bias
  terms so that the sampled free energies G = -kT ln(count) become equal
  across the end states of a site (b) and the free energy along every
  two-substituent edge (lambda_i + lambda_j = 1, the anti-diagonal of the
  pair's 2-D histogram) approaches a low target barrier (c, x, s by weighted
  least squares with a ridge; c also keeps at least END_FRAC_TARGET of the
  samples at end states), each change capped per iteration.

Bias terms of a site with n substituents (global block indices i, j):
  b_i lambda_i                                      (fixed bias)
  c_ij lambda_i lambda_j                            (type 6, i < j)
  x_ij lambda_j (1 - exp(-5.56 lambda_i))           (type 10, ordered)
  s_ij lambda_i lambda_j / (lambda_i + 0.017)       (type 8, ordered)
Parameter vector of a site: [b (n), c (P), x (2P), s (2P)], P = n(n-1)/2,
pairs (i,j) i<j in lexicographic order, ordered terms as (i,j) then (j,i).

Flatness (the criterion both methods are measured by): per site the end-state
populations p_i = count(lambda_i > 0.99) / sum over the site; its deviation
is max_i |p_i - 1/n|.  A replica is flat when every site deviates by at most
FLAT_TOL and spends at least END_FRAC_MIN of its samples at an end state.

Learned flattening: a BF16 MLP (``blade_b200.mlp``) maps the normalised
histograms and the current parameters of a replica (3 sites x 4
substituents) to the remaining correction, trained on pairs from plain runs
(target: the plain run's converged parameters minus the current ones).  The
plain update stays as fallback (non-finite prediction, or flatness worse by
more than FALLBACK_MARGIN after a learned step).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .msld import VARBIAS_DTYPE

X_L0, S_L0 = -5.56, 0.017
FLAT_TOL = 0.2
END_FRAC_MIN = 0.1
B_STEP = 0.5                        # fraction of the end-state free-energy gap closed per iteration
FALLBACK_MARGIN = 0.15
CAP_B, CAP_PAIR = 3.0, 1.0          # kcal/mol per plain iteration
RIDGE_B, RIDGE_PAIR = 0.01, 0.2
END_FRAC_TARGET = 0.2               # least fraction of samples at an end state that c keeps
EDGE_BARRIER_KT = 1.5               # target profile along an edge: 1.5 kT bump at lambda = 1/2
KB = 0.001987191
CHARGE_SIGMA, VARIANT_SIGMA = 0.1, 0.15   # e: fragment charges, variant perturbation
THETA_MASS = 5.0                    # test/T4L/prep/T4L149F.inp:69,81 (msld initialize ... mass 5)


def flattening_system(seed: int):
    """An MSLD water-box replica for flattening: the 216-water box with 3 sites x
    4 substituents of 8-15 atoms (charges ~N(0, 0.35) e, per-atom LJ with eps
    ~U(0.02, 0.2) kcal/mol and Rmin/2 ~U(1.2, 2.1) A), sites kept apart.  The 4 substituents of a site are
    variants of one fragment, as R-groups that differ at a few atoms: one
    shape, charges perturbed by N(0, VARIANT_SIGMA) e, one atom's LJ changed;
    they are rigid (no pairs inside a substituent) and tied atom by atom with
    zero-length bonds, so that variants out of play stay in place.
    Measured without these choices (independent walks and parameters per
    substituent, floppy and untied): unoccupied variants drift through the
    water and see dU/dlambda of +100 to +1000 kcal/mol, and lambda stays in one
    end state for tens of flattening iterations of either method."""
    from .systems import msld_water
    return msld_water(seed, avoid_sites=True, rigid_substituents=True, shared_geometry=True,
                      charge_sigma=CHARGE_SIGMA, variant_sigma=VARIANT_SIGMA, variant_lj_atoms=1,
                      tie_variants=True)


@dataclasses.dataclass
class SiteMap:
    """Sites of a batch of replicas, in global (concatenated) block indices."""
    sites: list                # [S] arrays of global block indices
    site_replica: np.ndarray   # [S]
    pairs: np.ndarray          # [P,2] global (i<j), all sites
    pair_offset: np.ndarray    # [S+1] first pair of each site
    param_offset: np.ndarray   # [S+1] first parameter of each site
    n_replicas: int
    n_blocks: int

    @property
    def n_params(self):
        return int(self.param_offset[-1])


def n_site_params(n: int) -> int:
    P = n * (n - 1) // 2
    return n + 5 * P


def site_map(reps, lam_starts) -> SiteMap:
    sites, srep, pairs, poff, qoff = [], [], [], [0], [0]
    for r, s in enumerate(reps):
        m = s.msld
        for k in range(1, m.siteCount):
            g = np.arange(m.siteBound[k], m.siteBound[k + 1]) + int(lam_starts[r])
            sites.append(g)
            srep.append(r)
            pp = [(g[a], g[b]) for a in range(len(g)) for b in range(a + 1, len(g))]
            pairs += pp
            poff.append(poff[-1] + len(pp))
            qoff.append(qoff[-1] + n_site_params(len(g)))
    return SiteMap(sites, np.array(srep), np.array(pairs, np.int32).reshape(-1, 2), np.array(poff),
                   np.array(qoff), len(reps), int(lam_starts[-1]))


def bias_arrays(sm: SiteMap, params: np.ndarray):
    """(fixed bias [L] FP64, variable biases VARBIAS_DTYPE) from the parameter vector."""
    fixed = np.zeros(sm.n_blocks)
    var = []
    for k, g in enumerate(sm.sites):
        n = len(g)
        q = params[sm.param_offset[k]:sm.param_offset[k + 1]]
        P = n * (n - 1) // 2
        fixed[g] = q[:n]
        c, x, s = q[n:n + P], q[n + P:n + 3 * P], q[n + 3 * P:n + 5 * P]
        p = 0
        for a in range(n):
            for b in range(a + 1, n):
                i, j = int(g[a]), int(g[b])
                var.append((i, j, 6, 0.0, c[p], 0))
                var.append((i, j, 10, X_L0, x[2 * p], 0))
                var.append((j, i, 10, X_L0, x[2 * p + 1], 0))
                var.append((i, j, 8, S_L0, s[2 * p], 0))
                var.append((j, i, 8, S_L0, s[2 * p + 1], 0))
                p += 1
    return fixed, np.array(var, VARBIAS_DTYPE)


def edge_basis(t: np.ndarray) -> np.ndarray:
    """Bias terms of one pair along its edge lambda_i = t, lambda_j = 1-t:
    columns b_i, b_j, c_ij, x_ij, x_ji, s_ij, s_ji."""
    u = 1.0 - t
    return np.stack([t, u, t * u, u * (1 - np.exp(X_L0 * t)), t * (1 - np.exp(X_L0 * u)),
                     t * u / (t + S_L0), t * u / (u + S_L0)], 1)


def flatness(sm: SiteMap, hist1, end_count):
    """Per replica: (max deviation of end-state populations from uniform,
    minimum fraction of samples at an end state), over its sites."""
    dev = np.zeros(sm.n_replicas)
    frac = np.ones(sm.n_replicas)
    for k, g in enumerate(sm.sites):
        r = sm.site_replica[k]
        c = end_count[g].astype(np.float64)
        samples = max(1, int(hist1[g[0]].sum()))
        tot = c.sum()
        p = c / tot if tot > 0 else np.zeros(len(g))
        dev[r] = max(dev[r], float(np.abs(p - 1.0 / len(g)).max()) if tot > 0 else 1.0 - 1.0 / len(g))
        frac[r] = min(frac[r], tot / samples)
    return dev, frac


def is_flat(dev, frac):
    return (dev <= FLAT_TOL) & (frac >= END_FRAC_MIN)


def site_flatness(sm: SiteMap, hist1, end_count):
    """Per site: (deviation of end-state populations from uniform, fraction of
    samples at an end state)."""
    dev = np.zeros(len(sm.sites))
    frac = np.zeros(len(sm.sites))
    for k, g in enumerate(sm.sites):
        c = end_count[g].astype(np.float64)
        samples = max(1, int(hist1[g[0]].sum()))
        tot = c.sum()
        dev[k] = float(np.abs(c / tot - 1.0 / len(g)).max()) if tot > 0 else 1.0 - 1.0 / len(g)
        frac[k] = tot / samples
    return dev, frac


def site_flatness_pooled(sm: SiteMap, recs, window: int, T: float = 300.0):
    """Per site: (deviation of the end-state populations from uniform, fraction
    of samples at an end state) from the last ``window`` iterations of
    ``recs`` pooled, each iteration's end-state counts reweighted to the
    parameters of the last one.  At an end state of a site (lambda_i = 1, the
    others 0) only the fixed bias b_i of that substituent acts -- the c, x and
    s terms vanish there -- so counts gathered under b' reweight to b by
    exp(-(b_i - b'_i) / kT) exactly; pooling several short runs lowers the
    sampling noise of the judgement."""
    kT = KB * T
    recs = recs[-window:]
    last = recs[-1]["params"]
    dev = np.zeros(len(sm.sites))
    frac = np.zeros(len(sm.sites))
    for k, g in enumerate(sm.sites):
        n = len(g)
        o = sm.param_offset[k]
        c = np.zeros(n)
        ends = samples = 0.0
        for r in recs:
            cnt = r["he"][g].astype(np.float64)
            shift = last[o:o + n] - r["params"][o:o + n]
            num = cnt * np.exp(-(shift - shift.min()) / kT)   # the common factor cancels
            if num.sum() > 0:                                 # this run's populations under the last
                c += cnt.sum() * num / num.sum()              # biases, weighted by its end samples
            ends += cnt.sum()
            samples += max(1, int(r["h1"][g[0]].sum()))
        tot = c.sum()
        dev[k] = float(np.abs(c / tot - 1.0 / n).max()) if tot > 0 else 1.0 - 1.0 / n
        frac[k] = ends / samples
    return dev, frac


def plain_update(sm: SiteMap, hist1, hist2, end_count, T: float = 300.0) -> np.ndarray:
    """The plain flattening update (change of every parameter) from one
    iteration's histograms, site by site:
      b    end-state balance: db_i = B_STEP (mean_j G_j - G_i) with
           G_i = -kT ln(n_i + 1/2), so that the end states of the site move
           toward equal free energy (B_STEP < 1 damps the noise of short runs);
      c, x, s  edge shape: weighted least squares that brings the free energy
           along each edge (anti-diagonal of the pair's 8x8 histogram) to
           the target barrier, given the new b: c sets the symmetric height
           of mixed states, antisymmetric x and s changes (x_ij = -x_ji,
           s_ij = -s_ji) the skew, with a ridge; when fewer than
           END_FRAC_TARGET of the samples sit at end states, c is raised by
           kT ln(END_FRAC_TARGET / f_end) on top (c lambda_i lambda_j raises
           every mixed state, also those inside the simplex);
    each change capped per iteration."""
    kT = KB * T
    delta = np.zeros(sm.n_params)
    t = (np.arange(8) + 0.5) / 8
    basis = edge_basis(t)                       # [8, 7]: b_i, b_j, c, x_ij, x_ji, s_ij, s_ji
    target = EDGE_BARRIER_KT * kT * 4 * t * (1 - t)
    for k, g in enumerate(sm.sites):
        n = len(g)
        P = n * (n - 1) // 2
        samples = max(1, int(hist1[g[0]].sum()))
        c = end_count[g].astype(np.float64)
        G_end = -kT * np.log(c + 0.5)
        db = np.clip(B_STEP * (G_end.mean() - G_end), -CAP_B, CAP_B)
        db -= db.mean()
        f_end = max(c.sum() / samples, 1e-3)
        dc_frac = max(0.0, kT * np.log(END_FRAC_TARGET / f_end))   # only raises mixed states
        dc = np.full(P, dc_frac)
        dx = np.zeros(2 * P)
        ds = np.zeros(2 * P)
        p = 0
        for a in range(n):
            for b in range(a + 1, n):
                h = hist2[sm.pair_offset[k] + p]
                cnt = np.array([h[m, 7 - m] for m in range(8)], np.float64)
                if cnt.sum() > 0:
                    G = -kT * np.log(cnt + 0.5)
                    w = np.sqrt(cnt / (cnt + 10.0))
                    known = basis[:, 0] * db[a] + basis[:, 1] * db[b]
                    cols = np.stack([basis[:, 2], basis[:, 3] - basis[:, 4], basis[:, 5] - basis[:, 6],
                                     -np.ones(8)], 1)
                    A = np.concatenate([cols * w[:, None], np.sqrt(RIDGE_PAIR) * np.eye(4)[:3]], 0)
                    y = np.concatenate([(target - G - known) * w, np.zeros(3)])
                    c_fit, u, v, _ = np.linalg.lstsq(A, y, rcond=None)[0]
                    dc[p] += c_fit
                    dx[2 * p:2 * p + 2] = (u, -u)
                    ds[2 * p:2 * p + 2] = (v, -v)
                p += 1
        o = sm.param_offset[k]
        delta[o:o + n] = db
        delta[o + n:o + n + P] = np.clip(dc, -CAP_PAIR, CAP_PAIR)
        delta[o + n + P:o + n + 3 * P] = np.clip(dx, -CAP_PAIR, CAP_PAIR)
        delta[o + n + 3 * P:o + n + 5 * P] = np.clip(ds, -CAP_PAIR, CAP_PAIR)
    return delta


def gauge(sm: SiteMap, params: np.ndarray) -> np.ndarray:
    """Parameters with the fixed biases of every site shifted to zero mean."""
    q = params.copy()
    for k, g in enumerate(sm.sites):
        o = sm.param_offset[k]
        q[o:o + len(g)] -= q[o:o + len(g)].mean()
    return q


# ---------------------------------------------------------------------------
# learned flattening: features and model
# ---------------------------------------------------------------------------
SITES, SUBS = 3, 4
N_PAIRS_SITE = SUBS * (SUBS - 1) // 2
N_PARAMS_REP = SITES * n_site_params(SUBS)                       # 102
N_FEAT = SITES * SUBS * 32 + SITES * N_PAIRS_SITE * 64 + N_PARAMS_REP  # 1638
FEAT_PAD, OUT_PAD = 1664, 128
PARAM_SCALE, TARGET_SCALE = 10.0, 5.0
HIDDEN = (256, 256, 256)


def replica_features(sm: SiteMap, hist1, hist2, params) -> np.ndarray:
    """[R, FEAT_PAD] features (replicas must all have 3 sites x 4 substituents)."""
    R = sm.n_replicas
    X = np.zeros((R, FEAT_PAD), np.float32)
    per = SITES * SUBS * 32 + SITES * N_PAIRS_SITE * 64
    for k, g in enumerate(sm.sites):
        r = sm.site_replica[k]
        ks = k - int(np.searchsorted(sm.site_replica, r))         # site index within the replica
        samples = max(1, int(hist1[g[0]].sum()))
        X[r, ks * SUBS * 32:(ks + 1) * SUBS * 32] = (hist1[g] / samples).reshape(-1)
        h2 = hist2[sm.pair_offset[k]:sm.pair_offset[k + 1]] / samples
        o = SITES * SUBS * 32 + ks * N_PAIRS_SITE * 64
        X[r, o:o + N_PAIRS_SITE * 64] = h2.reshape(-1)
    q = gauge(sm, params) / PARAM_SCALE
    for r in range(R):
        X[r, per:per + N_PARAMS_REP] = q[r * N_PARAMS_REP:(r + 1) * N_PARAMS_REP]
    return X


def check_layout(sm: SiteMap):
    ok = all(len(g) == SUBS for g in sm.sites) and len(sm.sites) == SITES * sm.n_replicas
    if not ok:
        raise ValueError("learned flattening expects replicas of 3 sites x 4 substituents")


def permutation_tables(rng, n_aug: int):
    """Random relabelings (site order, substituent order within each site)
    of one replica, as index maps over features and parameters."""
    out = []
    pairs = [(a, b) for a in range(SUBS) for b in range(a + 1, SUBS)]
    pidx = {pq: i for i, pq in enumerate(pairs)}
    for _ in range(n_aug):
        sp = rng.permutation(SITES)
        fmap = np.arange(FEAT_PAD)
        qmap = np.arange(N_PARAMS_REP)
        nps = n_site_params(SUBS)
        P = N_PAIRS_SITE
        for new_s in range(SITES):
            old_s = sp[new_s]
            perm = rng.permutation(SUBS)              # new substituent a <- old perm[a]
            for a in range(SUBS):
                fmap[new_s * SUBS * 32 + a * 32:new_s * SUBS * 32 + (a + 1) * 32] = \
                    np.arange(32) + old_s * SUBS * 32 + perm[a] * 32
                qmap[new_s * nps + a] = old_s * nps + perm[a]
            base2 = SITES * SUBS * 32
            for (a, b), p_new in pidx.items():
                oa, ob = perm[a], perm[b]
                swap = oa > ob
                p_old = pidx[(min(oa, ob), max(oa, ob))]
                src = base2 + old_s * P * 64 + p_old * 64 + np.arange(64)
                if swap:                               # transpose the 8x8 histogram
                    src = src.reshape(8, 8).T.reshape(-1)
                fmap[base2 + new_s * P * 64 + p_new * 64:base2 + new_s * P * 64 + (p_new + 1) * 64] = src
                o_new, o_old = new_s * nps, old_s * nps
                qmap[o_new + SUBS + p_new] = o_old + SUBS + p_old
                for t0 in (SUBS + P, SUBS + 3 * P):    # ordered terms: (i,j) then (j,i)
                    qmap[o_new + t0 + 2 * p_new] = o_old + t0 + 2 * p_old + (1 if swap else 0)
                    qmap[o_new + t0 + 2 * p_new + 1] = o_old + t0 + 2 * p_old + (0 if swap else 1)
        per = SITES * SUBS * 32 + SITES * N_PAIRS_SITE * 64
        fmap[per:per + N_PARAMS_REP] = per + qmap
        out.append((fmap, qmap))
    return out


# ---------------------------------------------------------------------------
# iteration driver (GPU)
# ---------------------------------------------------------------------------
class AlfBatch:
    """R replicas stepped together; each iteration runs ``steps`` MSLD steps
    (CUDA graph) with the current biases and returns the lambda histograms."""

    def __init__(self, reps, steps: int = 2000, seed: int = 1, gamma_ps: float = 5.0, equil_steps: int = 2000,
                 T: float = 300.0, theta_mass: float = THETA_MASS, gamma_theta_ps: float = 1.0):
        from .batch import MsldBatch
        self.reps = reps
        self.steps = steps
        self.T = T
        self.B = MsldBatch(reps, gamma_ps=gamma_ps, seed=seed, T=T, theta_mass=theta_mass,
                           gamma_theta_ps=gamma_theta_ps)
        self.sm = site_map(reps, self.B.nb.lam_starts)
        self.params = np.zeros(self.sm.n_params)
        self.B.set_bias(*bias_arrays(self.sm, self.params))
        self.B.enable_histograms(self.sm.pairs)
        if equil_steps:
            self.B.run_eager(equil_steps)
        self.B.capture()
        self.B.take_histograms()

    def set_params(self, params):
        self.params = np.asarray(params, np.float64)
        self.B.set_bias(*bias_arrays(self.sm, self.params))

    def iterate(self):
        self.B.run_graph(self.steps)
        return self.B.take_histograms()

    def status(self):
        return self.B.check()

    def close(self):
        self.B.close()


def run_plain(drv: AlfBatch, n_iter: int, log=None):
    """Plain flattening for n_iter iterations.  Returns per-iteration records
    (params before the iteration, histograms, flatness)."""
    recs = []
    for it in range(n_iter):
        h1, h2, he = drv.iterate()
        dev, frac = flatness(drv.sm, h1, he)
        recs.append({"params": drv.params.copy(), "h1": h1, "h2": h2, "he": he, "dev": dev, "frac": frac})
        if log:
            log(it, dev, frac)
        drv.set_params(drv.params + plain_update(drv.sm, h1, h2, he, drv.T))
    return recs


def run_learned(drv: AlfBatch, model, n_iter: int, log=None):
    """Learned flattening with the plain update as fallback (non-finite output,
    or flatness worse by more than FALLBACK_MARGIN after a learned step)."""
    import torch
    check_layout(drv.sm)
    R = drv.sm.n_replicas
    prev_dev = np.full(R, np.inf)
    used_learned = np.zeros(R, bool)
    recs = []
    for it in range(n_iter):
        h1, h2, he = drv.iterate()
        dev, frac = flatness(drv.sm, h1, he)
        X = torch.from_numpy(replica_features(drv.sm, h1, h2, drv.params)).to(drv.B.dev)
        pred = model.forward(X).cpu().numpy()[:, :N_PARAMS_REP].astype(np.float64) * TARGET_SCALE
        plain = plain_update(drv.sm, h1, h2, he, drv.T)
        learned = pred.reshape(-1)
        bad = ~np.isfinite(pred).all(1) | (used_learned & (dev > prev_dev + FALLBACK_MARGIN))
        use_plain = np.repeat(bad, N_PARAMS_REP)
        delta = np.where(use_plain, plain, learned)
        recs.append({"params": drv.params.copy(), "dev": dev, "frac": frac, "fallback": bad.copy()})
        if log:
            log(it, dev, frac)
        used_learned = ~bad
        prev_dev = dev
        drv.set_params(drv.params + delta)
    return recs


def iterations_to_flat(recs) -> np.ndarray:
    """1-based index of the first iteration whose histograms were flat (0 = never)."""
    R = len(recs[0]["dev"])
    out = np.zeros(R, np.int64)
    for it, r in enumerate(recs):
        f = is_flat(r["dev"], r["frac"]) & (out == 0)
        out[f] = it + 1
    return out


# ---------------------------------------------------------------------------
# learned flattening: data, training, per-site evaluation
# ---------------------------------------------------------------------------
LOOKAHEAD = 10          # the learned step predicts the plain loop's change over this many iterations


def training_pairs(sm: SiteMap, recs, lookahead: int = LOOKAHEAD):
    """(X [n, FEAT_PAD], Y [n, OUT_PAD]) from one plain run: the features of
    iteration t and, as target, gauge(params[t + lookahead]) - gauge(params[t])
    (scaled by 1/TARGET_SCALE): where the plain loop stands ``lookahead``
    iterations later, seen from the histograms it has now."""
    check_layout(sm)
    X, Y = [], []
    for t in range(len(recs) - lookahead):
        X.append(replica_features(sm, recs[t]["h1"], recs[t]["h2"], recs[t]["params"]))
        d = gauge(sm, recs[t + lookahead]["params"]) - gauge(sm, recs[t]["params"])
        y = np.zeros((sm.n_replicas, OUT_PAD), np.float32)
        y[:, :N_PARAMS_REP] = d.reshape(sm.n_replicas, N_PARAMS_REP) / TARGET_SCALE
        Y.append(y)
    return np.concatenate(X), np.concatenate(Y)


def flat_targets(Xseq: np.ndarray):
    """Targets that point at flatness: for features Xseq [T, R, FEAT_PAD] of
    consecutive plain iterations of R replicas, each site's target is the
    change from its current parameters to those it had at the first iteration
    its histograms were flat (zero from then on); sites that never became
    flat get weight 0.  Flatness is measured on the top histogram bin
    (lambda > 31/32) standing in for the end-state count.  Returns
    (Y, W) [T, R, OUT_PAD] with Y scaled by 1/TARGET_SCALE."""
    T, R, _ = Xseq.shape
    per = SITES * SUBS * 32 + SITES * N_PAIRS_SITE * 64
    nps = n_site_params(SUBS)
    Y = np.zeros((T, R, OUT_PAD), np.float32)
    W = np.zeros((T, R, OUT_PAD), np.float32)
    for s in range(SITES):
        h = Xseq[:, :, s * SUBS * 32:(s + 1) * SUBS * 32].reshape(T, R, SUBS, 32).astype(np.float64)
        end = h[..., 31]
        tot = end.sum(-1)
        p = end / np.maximum(tot, 1e-12)[..., None]
        flat = (np.abs(p - 1.0 / SUBS).max(-1) <= FLAT_TOL) & (tot >= END_FRAC_MIN)
        q = Xseq[:, :, per + s * nps:per + (s + 1) * nps].astype(np.float64) * PARAM_SCALE
        for r in range(R):
            hit = np.nonzero(flat[:, r])[0]
            if len(hit) == 0:
                continue
            t0 = hit[0]
            Y[:t0, r, s * nps:(s + 1) * nps] = (q[t0, r] - q[:t0, r]) / TARGET_SCALE
            W[:, r, s * nps:(s + 1) * nps] = 1.0
    return Y, W


def new_model(seed: int = 0, max_batch: int = 256):
    from .mlp import BF16MLP
    return BF16MLP([FEAT_PAD, *HIDDEN, OUT_PAD], max_batch=max_batch, seed=seed)


def train(model, X, Y, steps: int = 3000, batch: int = 256, lr: float = 1e-3, seed: int = 0, n_aug: int = 64,
          X_val=None, Y_val=None, log=None, W=None, W_val=None):
    """Adam on the MSE, every step on a batch relabeled by a random site /
    substituent permutation (the task is symmetric under relabeling).
    Returns (first loss, last loss, validation loss or None)."""
    import torch
    rng = np.random.default_rng(seed)
    tables = permutation_tables(rng, n_aug)
    dev = model.dev
    first = last = None
    n = len(X)
    for step in range(steps):
        idx = rng.integers(0, n, batch)
        fmap, qmap = tables[rng.integers(len(tables))]
        xb = X[idx][:, fmap]
        yb = Y[idx].copy()
        yb[:, :N_PARAMS_REP] = yb[:, :N_PARAMS_REP][:, qmap]
        wb = None
        if W is not None:
            wb = W[idx].copy()
            wb[:, :N_PARAMS_REP] = wb[:, :N_PARAMS_REP][:, qmap]
            wb = torch.from_numpy(np.ascontiguousarray(wb)).to(dev)
        lr_t = lr * 0.5 * (1 + math.cos(math.pi * step / steps))
        loss = model.train_step(torch.from_numpy(np.ascontiguousarray(xb)).to(dev),
                                torch.from_numpy(np.ascontiguousarray(yb)).to(dev), lr=lr_t, elem_weight=wb)
        if step == 0:
            first = float(loss.cpu()[0])
        if log and step % 500 == 0:
            log(step, float(loss.cpu()[0]))
    last = float(loss.cpu()[0]) if steps else None
    val = None
    if X_val is not None and len(X_val):
        tot, cnt = 0.0, 0
        for k in range(0, len(X_val), model.max_batch):
            xb = torch.from_numpy(np.ascontiguousarray(X_val[k:k + model.max_batch])).to(dev)
            yb = torch.from_numpy(np.ascontiguousarray(Y_val[k:k + model.max_batch])).to(dev)
            wb = None if W_val is None else torch.from_numpy(np.ascontiguousarray(W_val[k:k + model.max_batch])).to(dev)
            tot += float(model.loss_grad(xb, yb, elem_weight=wb).cpu()[0]) * len(xb)
            cnt += len(xb)
        val = tot / cnt
    return first, last, val


def site_iterations_to_flat(recs_dev_frac) -> np.ndarray:
    """Per site, the 1-based first iteration whose histograms were flat (0 = never)."""
    first = None
    for it, (dev, frac) in enumerate(recs_dev_frac):
        flat = (dev <= FLAT_TOL) & (frac >= END_FRAC_MIN)
        if first is None:
            first = np.zeros(len(dev), np.int64)
        first[(first == 0) & flat] = it + 1
    return first


def run_sites(drv: AlfBatch, n_iter: int, model=None, scale: float = 1.0, with_plain: bool = False,
              learned_iters: int | None = None, pool: int = 0):
    """n_iter iterations of plain (model None) or learned flattening; returns
    per-iteration records with per-site flatness and whether the plain
    fallback was used.  The learned step is ``scale`` times the predicted
    lookahead change, added to the plain update when ``with_plain``; with
    ``learned_iters`` only the first that many iterations use the network.
    With ``pool`` > 1 the records also hold the flatness of the last ``pool``
    iterations pooled (site_flatness_pooled)."""
    import torch
    R = drv.sm.n_replicas
    prev = np.full(R, np.inf)
    used_learned = np.zeros(R, bool)
    recs = []
    for it in range(n_iter):
        h1, h2, he = drv.iterate()
        sdev, sfrac = site_flatness(drv.sm, h1, he)
        rdev, rfrac = flatness(drv.sm, h1, he)
        plain = plain_update(drv.sm, h1, h2, he, drv.T)
        rec = {"params": drv.params.copy(), "h1": h1, "h2": h2, "he": he, "site_dev": sdev, "site_frac": sfrac,
               "fallback": None}
        if model is None or (learned_iters is not None and it >= learned_iters):
            delta = plain
        else:
            X = torch.from_numpy(replica_features(drv.sm, h1, h2, drv.params)).to(drv.B.dev)
            pred = model.forward(X).cpu().numpy()[:, :N_PARAMS_REP].astype(np.float64) * TARGET_SCALE
            bad = ~np.isfinite(pred).all(1) | (used_learned & (rdev > prev + FALLBACK_MARGIN))
            step = scale * pred.reshape(-1) + (plain if with_plain else 0.0)
            delta = np.where(np.repeat(bad, N_PARAMS_REP), plain, step)
            used_learned = ~bad
            rec["fallback"] = bad
        prev = rdev
        recs.append(rec)
        if pool > 1:
            rec["site_dev_pool"], rec["site_frac_pool"] = site_flatness_pooled(drv.sm, recs, pool, drv.T)
        drv.set_params(drv.params + delta)
    return recs


def _replica_map() -> SiteMap:
    """Site map of one replica of 3 sites x 4 substituents (blocks 1..12)."""
    sites = [np.arange(1 + SUBS * k, 1 + SUBS * (k + 1)) for k in range(SITES)]
    pairs = np.array([(g[a], g[b]) for g in sites for a in range(SUBS) for b in range(a + 1, SUBS)], np.int32)
    return SiteMap(sites, np.zeros(SITES, np.int64), pairs, np.arange(SITES + 1) * N_PAIRS_SITE,
                   np.arange(SITES + 1) * n_site_params(SUBS), 1, 1 + SITES * SUBS)


def plain_update_from_features(x: np.ndarray, samples: int) -> np.ndarray:
    """The plain update recomputed from one replica's features (histograms
    times ``samples``; the top 1-D bin stands in for the end-state count)."""
    sm = _replica_map()
    h1 = np.zeros((sm.n_blocks, 32), np.int64)
    h2 = np.zeros((len(sm.pairs), 8, 8), np.int64)
    o2 = SITES * SUBS * 32
    for k in range(SITES):
        h1[1 + SUBS * k:1 + SUBS * (k + 1)] = np.round(x[k * SUBS * 32:(k + 1) * SUBS * 32].reshape(SUBS, 32)
                                                       * samples)
        h2[N_PAIRS_SITE * k:N_PAIRS_SITE * (k + 1)] = np.round(
            x[o2 + k * N_PAIRS_SITE * 64:o2 + (k + 1) * N_PAIRS_SITE * 64].reshape(N_PAIRS_SITE, 8, 8) * samples)
    return plain_update(sm, h1, h2, h1[:, 31].copy())


def distance_to_flat(X: np.ndarray, Y: np.ndarray, W: np.ndarray, pred: np.ndarray, samples: int):
    """RMS distance (kcal/mol, weighted entries only) from the flat parameters
    of (a) the network's step, (b) the plain update, (c) no change."""
    em, ep, e0 = [], [], []
    for n in range(len(X)):
        sel = W[n, :N_PARAMS_REP] > 0
        if not sel.any():
            continue
        tgt = Y[n, :N_PARAMS_REP].astype(np.float64) * TARGET_SCALE
        pu = plain_update_from_features(X[n].astype(np.float64), samples)
        em.append(((pred[n, :N_PARAMS_REP] * TARGET_SCALE - tgt)[sel] ** 2).mean())
        ep.append(((pu - tgt)[sel] ** 2).mean())
        e0.append((tgt[sel] ** 2).mean())
    return {"samples": len(em), "network": float(np.sqrt(np.mean(em))), "plain_update": float(np.sqrt(np.mean(ep))),
            "no_change": float(np.sqrt(np.mean(e0)))}
