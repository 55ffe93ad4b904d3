"""Learned warm start on the GPU against its CPU restatement (oracle/mpnn.cpp).

Features are compared element by element (the walk counts bit-exactly), the
forward pass, stress loss and every gradient block within the tolerances that
bf16 storage and tensor-core accumulation order allow (stated per test), the
evaluator against the oracle's metric restatements, and training for
determinism, checkpoint round trips and what it gains over a random start.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 0x5EED


def star_ring(jc, leaves=1500):
    """A hub of degree > 1024 (rows summed in segments by a whole block) plus a ring."""
    pairs = [(0, i) for i in range(1, leaves + 1)] + [(i, i % leaves + 1) for i in range(1, leaves + 1)]
    return jc.csr_from_pairs(leaves + 1, pairs)


def mixed_graphs(jc, hub=True):
    gs = [jc.gen_scale_free(300, 3, 11), jc.gen_watts_strogatz(257, 6, 0.1, 12),
          jc.gen_rgg(400, float(np.sqrt(6.0 / (np.pi * 400))), 13), jc.csr_from_pairs(1, []),
          jc.gen_path(9)]
    if hub:
        gs.append(star_ring(jc))
    return gs


def rand_targets(graphs, seed, dim=2):
    rng = np.random.default_rng(seed)
    out = []
    for g in graphs:
        t = np.zeros((g.n_nodes, 3), np.float32)
        t[:, :dim] = rng.uniform(-1, 1, (g.n_nodes, dim))
        out.append(t.reshape(-1))
    return out


def t4(targets):
    t = np.concatenate([x.reshape(-1, 3) for x in targets])
    return np.concatenate([t, np.zeros((len(t), 1), np.float32)], axis=1)


def fa2_layouts(jc, graphs, seeds, iters=200):
    eng = jc.LayoutEngine("fa2-bh")
    eng.set_params({"theta": 0.8})
    eng.init_batch(graphs, seeds)
    eng.step_many(iters, readback=False)
    xyz = eng.positions()
    eng.close()
    out, b = [], 0
    for g in graphs:
        out.append(xyz[3 * b: 3 * (b + g.n_nodes)].copy())
        b += g.n_nodes
    return out


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


BLOCKS = {"W0": (0, 8192), "b0": (8192, 8320), "W1": (8320, 41088), "b1": (41088, 41216),
          "W2": (41216, 73984), "b2": (73984, 74112), "Wh": (74112, 74624), "bh": (74624, 74628)}


def test_features_match_oracle(jc, orc):
    graphs = mixed_graphs(jc)
    net = jc.Mpnn(2, SEED)
    net.bind(graphs, rand_targets(graphs, 1))
    xg = net.features()
    xo = orc.mpnn_features(orc.GraphSet(graphs), SEED)
    # walk return probabilities: integer counts, bit-exact
    assert np.array_equal(xg[:, 1:17], xo[:, 1:17])
    assert np.array_equal(xg[:, 25:], xo[:, 25:])
    # log(1 + deg): device log1pf vs host log1p in f32, then bf16: at most one bf16 step apart
    assert np.all(np.abs(xg[:, 0] - xo[:, 0]) <= 2.0 ** -7 * np.abs(xo[:, 0]) + 1e-30)
    # projections: same f32 smoothing in the same order; the per-graph mean and
    # deviation are f64 sums in different orders, so a bf16 rounding may flip
    p_g, p_o = xg[:, 17:25], xo[:, 17:25]
    diff = np.abs(p_g - p_o)
    assert np.all(diff <= 2.0 ** -7 * np.abs(p_o) + 1e-6)
    assert np.mean(diff > 0) < 0.01


def test_chebyshev_features_match_oracle(jc, orc):
    """The Chebyshev filter (three-term recurrence with paired re-centring)
    followed by plain lazy steps, against the oracle's restatement."""
    graphs = mixed_graphs(jc)
    net = jc.Mpnn(2, SEED)
    net.set_params({"cheb_steps": 40, "cheb_b": 0.99, "smooth_steps": 16})
    net.bind(graphs, rand_targets(graphs, 1))
    xg = net.features()
    xo = orc.mpnn_features(orc.GraphSet(graphs), SEED, smooth_steps=16, cheb_steps=40, cheb_b=0.99)
    assert np.array_equal(xg[:, 1:17], xo[:, 1:17])
    assert np.all(np.abs(xg[:, 0] - xo[:, 0]) <= 2.0 ** -7 * np.abs(xo[:, 0]) + 1e-30)
    p_g, p_o = xg[:, 17:25], xo[:, 17:25]
    diff = np.abs(p_g - p_o)
    assert np.all(diff <= 2.0 ** -6 * np.abs(p_o) + 1e-5)
    assert np.mean(diff > 0) < 0.02


@pytest.mark.parametrize("dim,partners", [(2, 8), (3, 4)])
def test_gradients_match_oracle(jc, orc, dim, partners):
    """Loss within 1e-3 relative, prediction within 1e-2 and every parameter
    block's gradient within 3e-2 relative L2 of the f64 restatement that rounds
    to bf16 where the device stores bf16."""
    graphs = mixed_graphs(jc)
    targets = rand_targets(graphs, 2, dim)
    net = jc.Mpnn(dim, SEED)
    net.set_params({"partners": partners})
    net.bind(graphs, targets)
    X = net.features()
    theta = net.weights()
    gs = orc.GraphSet(graphs)
    G = len(graphs)
    loss_g, y_g, grad_g = net.grad(0, G, pair_step=3)
    loss_o, y_o, grad_o = orc.mpnn_grad(gs, X, t4(targets), dim, theta, partners, SEED, 3, 0, G, emulate=True)
    assert loss_g == pytest.approx(loss_o, rel=1e-3)
    assert rel_l2(y_g[:, :dim], y_o[:, :dim]) < 1e-2
    for name, (b, e) in BLOCKS.items():
        if name in ("Wh", "bh"):
            cols = [k for k in range(b, e) if (k - b) % 4 < dim]
            assert rel_l2(grad_g[cols], grad_o[cols]) < 3e-2, name
        else:
            assert rel_l2(grad_g[b:e], grad_o[b:e]) < 3e-2, name


def test_gradient_of_a_graph_subrange(jc, orc):
    """A batch that starts mid-set (node and graph offsets non-zero)."""
    graphs = mixed_graphs(jc, hub=False)
    targets = rand_targets(graphs, 3)
    net = jc.Mpnn(2, SEED)
    net.bind(graphs, targets)
    loss_g, y_g, grad_g = net.grad(1, 3, pair_step=0)
    loss_o, y_o, grad_o = orc.mpnn_grad(orc.GraphSet(graphs), net.features(), t4(targets), 2, net.weights(), 8,
                                        SEED, 0, 1, 3, emulate=True)
    assert loss_g == pytest.approx(loss_o, rel=1e-3)
    assert rel_l2(grad_g, grad_o) < 3e-2


def test_training_is_deterministic(jc):
    graphs, seeds = jc.gen_batch_graphs(12, seed=77, lo=50, hi=600)
    targets = fa2_layouts(jc, graphs, seeds, 100)
    runs = []
    for _ in range(2):
        net = jc.Mpnn(2, SEED)
        net.set_params({"batch_nodes": 1500})
        net.bind(graphs, targets)
        losses = net.train(10)
        runs.append((losses, net.weights()))
        net.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])


def test_checkpoint_round_trip(jc):
    graphs, seeds = jc.gen_batch_graphs(8, seed=78, lo=50, hi=500)
    targets = fa2_layouts(jc, graphs, seeds, 60)
    net = jc.Mpnn(2, SEED)
    net.set_params({"batch_nodes": 1000})
    net.bind(graphs, targets)
    net.train(3)
    state = net.save_state()
    net.train(4)
    w_ref = net.weights()
    other = jc.Mpnn(2, SEED)
    other.set_params({"batch_nodes": 1000})
    other.bind(graphs, targets)
    other.load_state(state)
    other.train(4)
    assert np.array_equal(other.weights(), w_ref)
    with pytest.raises(jc.JcError):
        jc.Mpnn(3, SEED).load_state(state)


def test_training_lowers_held_out_loss(jc):
    train, tseeds = jc.gen_batch_graphs(60, seed=91, lo=50, hi=1500)
    held, hseeds = jc.gen_batch_graphs(15, seed=92, lo=50, hi=1500)
    t_train = fa2_layouts(jc, train, tseeds, 200)
    t_held = fa2_layouts(jc, held, hseeds, 200)
    net = jc.Mpnn(2, SEED)
    net.set_params({"batch_nodes": 8192, "lr": 2e-3})
    net.bind(held, t_held)
    before = net.eval_loss()
    net.bind(train, t_train)
    losses = net.train(300)
    net.bind(held, t_held)
    after = net.eval_loss()
    assert np.all(np.isfinite(losses))
    assert after < 0.8 * before, (before, after)


def first_below(curve, target):
    for t, s in curve:
        if s <= target:
            return t
    return None


def test_warm_start_reaches_plain_stress_sooner(jc):
    """What the trained network gains: ForceAtlas2 continued from its
    prediction reaches 1.01 x the plain run's pivot stress after 300
    iterations at least 3x sooner than the plain run from a random start
    (measured on B200: 60 against 280 iterations; training is deterministic).
    The converged-stress target of the bench is a harder bar (1.27x there)."""
    train, tseeds = jc.gen_batch_graphs(90, seed=93, lo=100, hi=2000)
    held, hseeds = jc.gen_batch_graphs(24, seed=94, lo=100, hi=2000)
    net = jc.Mpnn(2, SEED)
    net.set_params({"batch_nodes": 16384, "lr": 2e-3, "smooth_steps": 64})
    net.bind(train, fa2_layouts(jc, train, tseeds, 300))
    net.train(400)
    ev = jc.Evaluator(held, n_pivots=16, seed=5)
    curves = []
    for start in (hseeds, net.predict(held)[0]):
        eng = jc.LayoutEngine("fa2-bh")
        eng.set_params({"theta": 0.8})
        eng.init_batch(held, start)
        curve = [(0, ev(eng.positions())[0])]
        for t in range(10, 301, 10):
            eng.step_many(10, readback=False)
            curve.append((t, ev(eng.positions())[0]))
        curves.append(curve)
        eng.close()
    plain, learned = curves
    target = 1.01 * plain[-1][1]
    it_plain, it_learned = first_below(plain, target), first_below(learned, target)
    assert learned[0][1] < 0.85 * plain[0][1], (learned[0], plain[0])
    assert it_learned is not None and 3 * it_learned <= it_plain, (it_learned, it_plain)


def test_evaluator_matches_oracle_metrics(jc, orc):
    graphs = [jc.gen_scale_free(200, 2, 5), jc.gen_grid(9, 7), jc.gen_path(2), jc.csr_from_pairs(1, [])]
    ev = jc.Evaluator(graphs, n_pivots=6, seed=3)
    rng = np.random.default_rng(4)
    xyz = [rng.uniform(-1, 1, 3 * g.n_nodes).astype(np.float32) for g in graphs]
    mean_s, mean_cv, st, cv = ev(np.concatenate(xyz))
    piv = ev.pivots()
    base = 0
    want_s, want_cv = [], []
    for gi, g in enumerate(graphs):
        ps = [int(p) - base for p in piv[gi] if p != 0xFFFFFFFF]
        dist = np.stack([orc.bfs(g, p) for p in ps]) if ps else np.zeros((0, g.n_nodes), np.uint32)
        terms = orc.pivot_terms(np.array(ps, np.uint32), dist)
        s = orc.scale_normalized_stress(xyz[gi], terms)
        ei = [(i, j) for i in range(g.n_nodes) for j in g.neighbors[g.offsets[i]:g.offsets[i + 1]] if j > i]
        c = orc.edge_length_cv(xyz[gi], np.array(ei, np.uint32).reshape(-1, 2))
        assert st[gi] == pytest.approx(s, rel=1e-5, abs=1e-7)
        assert cv[gi] == pytest.approx(c, rel=1e-5, abs=1e-7)
        base += g.n_nodes
        if len(terms):
            want_s.append(s)
        if len(ei) >= 2:
            want_cv.append(c)
    assert mean_s == pytest.approx(np.mean(want_s), rel=1e-5)
    assert mean_cv == pytest.approx(np.mean(want_cv), rel=1e-5)


def test_guarded_warm_start_keeps_the_better_start(jc):
    """The guarded hand-off keeps, per graph, the prediction only where its
    pivot stress is below the seed's; every other graph starts from its seed."""
    graphs, seeds = jc.gen_batch_graphs(12, seed=95, lo=50, hi=800)
    net = jc.Mpnn(2, SEED)
    net.bind(graphs[:6], rand_targets(graphs[:6], 3))
    net.train(40)  # barely trained: some predictions lose to the seed
    ev = jc.Evaluator(graphs, n_pivots=8, seed=7)
    pred = net.predict(graphs)[0]
    _, _, s_pred, _ = ev(np.concatenate(pred))
    _, _, s_seed, _ = ev(np.concatenate(seeds))
    out, keep, ms, dev_ms = net.warm_start(graphs, seeds, ev)
    assert np.array_equal(keep, s_pred < s_seed)
    assert 0 < keep.sum() < len(graphs)
    assert ms >= dev_ms > 0.0
    for k, o, p, s in zip(keep, out, pred, seeds):
        assert np.array_equal(o, p if k else np.asarray(s, np.float32).reshape(-1))
    with pytest.raises(jc.JcError) as ei:
        net.warm_start(graphs[:-1], seeds[:-1], ev)  # evaluator built on other graphs
    assert ei.value.code == jc.JC_ERR_ARG
