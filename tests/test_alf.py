"""Plain landscape flattening (blade_b200.alf) on the CPU: the parameter
layout against the reference's bias forms (through the oracle's FP64 bias
routine), the update's fixed point on a synthetic landscape, and the
relabeling tables used to augment the learned model's training data."""

import numpy as np
import pytest

import oracle
from blade_b200 import alf, systems


@pytest.fixture(scope="module")
def sm():
    reps = [systems.msld_water(100 + k, avoid_sites=True) for k in range(2)]
    ls = np.concatenate([[0], np.cumsum([r.msld.blockCount for r in reps])])
    return alf.site_map(reps, ls)


def test_layout(sm):
    assert sm.n_params == 2 * 3 * alf.n_site_params(4) == 204
    assert len(sm.pairs) == 2 * 3 * 6
    assert all(len(g) == 4 for g in sm.sites)


def test_edge_basis_matches_reference_bias_forms(sm):
    rng = np.random.default_rng(0)
    params = rng.normal(0, 2, sm.n_params)
    fixed, var = alf.bias_arrays(sm, params)
    g = sm.sites[1]
    q = params[sm.param_offset[1]:sm.param_offset[2]]
    n, P = 4, 6
    for a, b, p in ((0, 1, 0), (1, 3, 4), (2, 3, 5)):
        for t in (0.1, 0.5, 0.93):
            lam = np.zeros(sm.n_blocks)
            lam[g[a]], lam[g[b]] = t, 1 - t
            _, e = oracle.bias(lam, fixed, var)
            phi = alf.edge_basis(np.array([t]))[0]
            cols = [a, b, n + p, n + P + 2 * p, n + P + 2 * p + 1, n + 3 * P + 2 * p, n + 3 * P + 2 * p + 1]
            assert e == pytest.approx(float(phi @ q[cols]), rel=1e-6, abs=1e-6)


def test_stuck_site_raises_its_state(sm):
    L = sm.n_blocks
    h2 = np.zeros((len(sm.pairs), 8, 8), np.int64)
    he = np.zeros(L, np.int64)
    h1 = np.zeros((L, 32), np.int64)
    for g in sm.sites:
        he[g[0]] = 2000
        h1[g[0], 31] = 2000
        h1[g[1:], 0] = 2000
    d = alf.plain_update(sm, h1, h2, he)
    for k, g in enumerate(sm.sites):
        db = d[sm.param_offset[k]:sm.param_offset[k] + 4]
        assert db[0] > 0 and (db[1:] < 0).all()
        assert abs(db.sum()) < 1e-9 and np.abs(db).max() <= alf.CAP_B
        # all samples at end states and no edge samples: the pair terms stay
        assert np.all(d[sm.param_offset[k] + 4:sm.param_offset[k + 1]] == 0)


def test_plain_update_flattens_synthetic_landscape(sm):
    """End-state free energies F_i; sampled populations follow exp(-(F+b)/kT)
    and transitions along every edge are flat: the update converges to
    b = -F (up to a constant) and the flatness criterion is met."""
    rng = np.random.default_rng(3)
    kT = alf.KB * 300
    F = rng.uniform(-6, 6, sm.n_blocks)
    params = np.zeros(sm.n_params)
    for it in range(40):
        fixed, _ = alf.bias_arrays(sm, params)
        he = np.zeros(sm.n_blocks, np.int64)
        h1 = np.zeros((sm.n_blocks, 32), np.int64)
        h2 = np.zeros((len(sm.pairs), 8, 8), np.int64)
        for k, g in enumerate(sm.sites):
            w = np.exp(-(F[g] + fixed[g]) / kT)
            pop = np.floor(4000 * w / w.sum()).astype(np.int64)
            he[g] = pop
            h1[g, 31] = pop
            h1[g, 0] = 4000 - pop
            for p in range(sm.pair_offset[k], sm.pair_offset[k + 1]):
                for m in range(8):
                    h2[p, m, 7 - m] = 50
        dev, frac = alf.flatness(sm, h1, he)
        if (dev <= 0.01).all():
            break
        params = params + alf.plain_update(sm, h1, h2, he)
    assert alf.is_flat(dev, frac).all() and (dev <= 0.01).all()
    fixed, _ = alf.bias_arrays(sm, params)
    for g in sm.sites:
        v = F[g] + fixed[g]
        assert np.ptp(v) < 0.2


def test_permutation_tables_relabel_consistently(sm):
    """Relabeling the substituents of a replica and permuting its features and
    parameters with the same table gives the same features as the relabeled
    replica's own histograms."""
    rng = np.random.default_rng(1)
    L = sm.n_blocks
    h1 = rng.integers(0, 100, (L, 32))
    h2 = rng.integers(0, 100, (len(sm.pairs), 8, 8))
    params = rng.normal(size=sm.n_params)
    X = alf.replica_features(sm, h1, h2, params)
    fmap, qmap = alf.permutation_tables(np.random.default_rng(7), 1)[0]
    # build the relabeled replica explicitly from the table's parameter map (replica 0)
    per = alf.SITES * alf.SUBS * 32 + alf.SITES * alf.N_PAIRS_SITE * 64
    Xp = X[0][fmap]
    q0 = alf.gauge(sm, params)[:alf.N_PARAMS_REP] / alf.PARAM_SCALE
    np.testing.assert_array_equal(Xp[per:per + alf.N_PARAMS_REP], q0[qmap].astype(np.float32))
    # histogram rows of the new labeling are rows of the old one
    for s_new in range(alf.SITES):
        for a in range(alf.SUBS):
            src = fmap[s_new * alf.SUBS * 32 + a * 32]
            assert src % 32 == 0
    # a pair's 8x8 block maps to an old pair's block, possibly transposed
    base2 = alf.SITES * alf.SUBS * 32
    blk = fmap[base2:base2 + 64] - base2
    old_p = blk.min() // 64
    rel = (blk - 64 * old_p).reshape(8, 8)
    assert (rel == np.arange(64).reshape(8, 8)).all() or (rel == np.arange(64).reshape(8, 8).T).all()


def test_committed_network_step_beats_plain_update():
    """The committed flattening network, evaluated by the FP64 oracle: one
    step lands closer to the flat parameters than the plain update."""
    import os
    from oracle import mlp_oracle as mo
    gold = os.path.join(os.path.dirname(__file__), "golden")
    w = np.load(os.path.join(gold, "flat_mlp.npz"))
    d = np.load(os.path.join(gold, "flat_val.npz"))
    L = len(w["sizes"]) - 1
    Ws = [mo.from_bf16_bits(w[f"W{l}_bf16"]) for l in range(L)]
    bs = [w[f"b{l}"].astype(np.float64) for l in range(L)]
    X = d["X"].astype(np.float64)
    _, outs = mo.mlp_forward(X, Ws, bs)
    dist = alf.distance_to_flat(X, d["Y"], d["W"], outs[-1][1], int(d["samples"]))
    assert dist["network"] < 0.85 * dist["plain_update"], dist


def test_pooled_flatness_reweights_end_states_exactly():
    """Runs under different fixed biases pool to the populations of the last
    biases: counts drawn as exact expectations from known end-state free
    energies reweight to the same flatness as a run under the last biases."""
    sm = alf._replica_map()
    kT = alf.KB * 300.0
    rng = np.random.default_rng(4)
    G = rng.normal(0.0, 1.0, 13)                       # end-state free energies per block
    recs = []
    params = np.zeros(sm.n_params)
    for t in range(4):
        params = params.copy()
        for k, g in enumerate(sm.sites):
            params[sm.param_offset[k]:sm.param_offset[k] + len(g)] = rng.normal(0.0, 0.8, len(g))
        he = np.zeros(13)
        h1 = np.zeros((13, 32))
        for k, g in enumerate(sm.sites):
            b = params[sm.param_offset[k]:sm.param_offset[k] + len(g)]
            p = np.exp(-(G[g] + b) / kT)
            he[g] = 1e6 * p / p.sum()                      # all samples at end states
            h1[g[0], 0] = 1e6
        recs.append({"params": params, "he": he, "h1": h1})
    dev_pool, frac_pool = alf.site_flatness_pooled(sm, recs, 4)
    dev_last, frac_last = alf.site_flatness(sm, recs[-1]["h1"], recs[-1]["he"])
    assert np.allclose(dev_pool, dev_last, atol=1e-9)
    assert np.allclose(frac_pool, 1.0) and np.allclose(frac_last, 1.0)
    same = [dict(r, params=recs[-1]["params"]) for r in recs]   # equal biases: plain sums
    dev_same, _ = alf.site_flatness_pooled(sm, same, 4)
    tot = sum(r["he"] for r in recs)
    for k, g in enumerate(sm.sites):
        c = tot[g]
        assert dev_same[k] == pytest.approx(np.abs(c / c.sum() - 0.25).max(), abs=1e-12)
