"""The learned warm start's CPU restatement checked on its own (CPU only).

The device network has no reference counterpart, so its oracle (oracle/mpnn.cpp)
is pinned by mathematics instead: central finite differences of the f64 forward
pass against the f64 backward pass, the closed-form scale of the stress loss
against a direct minimisation over the scale, and the features' defining
properties (walk return counts, standardised projections).
"""
import numpy as np
import pytest


def small_set(jc, orc):
    graphs = [jc.gen_scale_free(14, 2, 3), jc.gen_watts_strogatz(12, 4, 0.2, 5), jc.csr_from_pairs(1, [])]
    return graphs, orc.GraphSet(graphs)


def rand_theta(orc, seed, scale=0.2):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(orc.mpnn_num_params()) * scale).astype(np.float32)


def targets(n, seed, dim=3):
    rng = np.random.default_rng(seed)
    t = np.zeros((n, 4), np.float32)
    t[:, :dim] = rng.uniform(-1, 1, (n, dim))
    return t


def fd_check(f, theta, grad, idx, rel=2e-4):
    """Central differences; a step that crosses a ReLU kink (the one-sided
    differences disagree) is retried 10x and 100x smaller. Returns the indices
    that disagree and those left on a kink at every step."""
    bad, kinked = [], []
    f0 = f(theta)
    for k in idx:
        for scale in (1e-3, 1e-4, 1e-5):
            h = np.float32(scale * max(abs(float(theta[k])), 0.05))
            tp, tm = theta.copy(), theta.copy()
            tp[k] = theta[k] + h
            tm[k] = theta[k] - h
            fp, fm = f(tp), f(tm)
            up = (fp - f0) / (float(tp[k]) - float(theta[k]))
            dn = (f0 - fm) / (float(theta[k]) - float(tm[k]))
            fd = (fp - fm) / (float(tp[k]) - float(tm[k]))
            tol = rel * max(abs(fd), abs(grad[k])) + 1e-9
            if abs(up - dn) <= 20 * tol + 1e-6 * max(abs(up), abs(dn)):
                break
        else:
            kinked.append(int(k))
            continue
        if abs(fd - grad[k]) > tol:
            bad.append((int(k), fd, grad[k]))
    assert len(kinked) <= len(idx) // 10, kinked
    return bad


def test_features_properties(jc, orc):
    graphs, gs = small_set(jc, orc)
    X = orc.mpnn_features(gs, 0x5EED)
    deg = np.diff(gs.off.astype(np.int64))
    # column 0: log(1 + deg) in bf16
    assert np.allclose(X[:, 0], np.log1p(deg), rtol=1e-2)
    # walks never return after one step (no self-loops); isolated nodes always "return"
    assert np.all(X[deg > 0, 1] == 0.0)
    iso = np.where(deg == 0)[0]
    assert len(iso) == 1 and np.all(X[iso[0], 1:17] == 1.0)
    # return probabilities are multiples of 1/32
    assert np.all(np.abs(X[:, 1:17] * 32 - np.round(X[:, 1:17] * 32)) == 0)
    # projections: zero degree-weighted mean and unit mean square per graph
    # (bf16 rounding aside)
    for g in range(gs.G - 1):
        b, e = gs.go[g], gs.go[g + 1]
        p = X[b:e, 17:25].astype(np.float64)
        d = deg[b:e].astype(np.float64)
        assert np.all(np.abs((d[:, None] * p).sum(0) / d.sum()) < 2e-2)
        assert np.all(np.abs((p * p).mean(0) - 1.0) < 2e-2)
    assert np.all(X[:, 25:] == 0.0)


def test_chebyshev_features_properties(jc, orc):
    """With the Chebyshev phase the projections end centred and unit-scaled
    too, and differ from the plain filter's."""
    graphs, gs = small_set(jc, orc)
    X = orc.mpnn_features(gs, 0x5EED, smooth_steps=8, cheb_steps=24, cheb_b=0.99)
    deg = np.diff(gs.off.astype(np.int64))
    for g in range(gs.G - 1):
        b, e = gs.go[g], gs.go[g + 1]
        p = X[b:e, 17:25].astype(np.float64)
        d = deg[b:e].astype(np.float64)
        assert np.all(np.abs((d[:, None] * p).sum(0) / d.sum()) < 2e-2)
        assert np.all(np.abs((p * p).mean(0) - 1.0) < 2e-2)
    assert not np.array_equal(X[:, 17:25], orc.mpnn_features(gs, 0x5EED, smooth_steps=32)[:, 17:25])
    assert np.array_equal(X[:, :17], orc.mpnn_features(gs, 0x5EED, smooth_steps=32)[:, :17])


def test_features_deterministic_and_seeded(jc, orc):
    _, gs = small_set(jc, orc)
    a = orc.mpnn_features(gs, 7)
    assert np.array_equal(a, orc.mpnn_features(gs, 7))
    assert not np.array_equal(a[:, 17:25], orc.mpnn_features(gs, 8)[:, 17:25])


def test_backward_matches_finite_differences(jc, orc):
    """Network backward (all parameter blocks) under a linear upstream loss."""
    _, gs = small_set(jc, orc)
    X = orc.mpnn_features(gs, 1)
    T = targets(gs.n, 2)
    theta = rand_theta(orc, 3)
    up = np.random.default_rng(4).standard_normal((int(gs.go[2]), 4))
    f = lambda th: orc.mpnn_grad(gs, X, T, 3, th, 0, 1, 0, 0, 2, emulate=False, upstream=up)[0]
    _, _, grad = orc.mpnn_grad(gs, X, T, 3, theta, 0, 1, 0, 0, 2, emulate=False, upstream=up)
    # spot-check every parameter block: W0, b0, W1, b1, W2, b2, Wh, bh
    blocks = [(0, 8192), (8192, 8320), (8320, 41088), (41088, 41216), (41216, 73984), (73984, 74112),
              (74112, 74624), (74624, 74627)]
    rng = np.random.default_rng(5)
    idx = []
    for b, e in blocks:
        live = [k for k in range(b, e) if grad[k] != 0.0]
        idx += list(rng.choice(live, size=min(6, len(live)), replace=False)) if live else []
    assert len(idx) >= 40
    bad = fd_check(f, theta, grad, idx)
    assert not bad, bad[:5]


def test_stress_loss_gradient_is_half_the_symmetric_gradient(jc, orc):
    """With edge pairs only, each undirected edge appears from both ends, so the
    per-node (first-endpoint) gradient is exactly half the full gradient."""
    _, gs = small_set(jc, orc)
    X = orc.mpnn_features(gs, 1)
    T = targets(gs.n, 6)
    theta = rand_theta(orc, 7)
    f = lambda th: orc.mpnn_grad(gs, X, T, 3, th, 0, 1, 0, 0, 2, emulate=False)[0]
    loss, _, grad = orc.mpnn_grad(gs, X, T, 3, theta, 0, 1, 0, 0, 2, emulate=False)
    assert 0.0 < loss < 1.0
    rng = np.random.default_rng(8)
    live = np.where(grad != 0.0)[0]
    idx = rng.choice(live, size=40, replace=False)
    bad = fd_check(f, theta, 2.0 * grad, idx)
    assert not bad, bad[:5]


def test_loss_closed_form_matches_scale_search(jc, orc):
    """L_g = min over alpha of mean (alpha q - 1)^2 (metrics.rs:31-59 with w = 1/d^2)."""
    graphs, gs = small_set(jc, orc)
    X = orc.mpnn_features(gs, 1)
    T = targets(gs.n, 9)
    theta = rand_theta(orc, 10)
    loss, Y, _ = orc.mpnn_grad(gs, X, T, 3, theta, 0, 1, 0, 0, 1, emulate=False)
    g = graphs[0]
    q = []
    for i in range(g.n_nodes):
        for j in g.neighbors[g.offsets[i]:g.offsets[i + 1]]:
            d = np.linalg.norm(T[i, :3].astype(np.float64) - T[j, :3])
            q.append(np.linalg.norm(Y[i, :3] - Y[j, :3]) / d)
    q = np.array(q)
    alphas = np.linspace(0.0, 4.0 / q.mean(), 20001)
    brute = min(np.mean((a * q - 1.0) ** 2) for a in alphas[::20])
    a0 = q.sum() / (q * q).sum()
    assert loss == pytest.approx(np.mean((a0 * q - 1.0) ** 2), rel=1e-9)
    assert loss <= brute + 1e-12


def test_emulated_and_exact_modes_agree_roughly(jc, orc):
    """bf16 rounding at the device's storage points moves the gradient by ~1e-2."""
    _, gs = small_set(jc, orc)
    X = orc.mpnn_features(gs, 1)
    T = targets(gs.n, 11)
    theta = rand_theta(orc, 12)
    l0, y0, g0 = orc.mpnn_grad(gs, X, T, 3, theta, 8, 1, 3, 0, 3, emulate=False)
    l1, y1, g1 = orc.mpnn_grad(gs, X, T, 3, theta, 8, 1, 3, 0, 3, emulate=True)
    assert abs(l0 - l1) < 2e-2 * abs(l0)
    assert np.linalg.norm(y0 - y1) < 3e-2 * np.linalg.norm(y0)
    assert np.linalg.norm(g0 - g1) < 1e-1 * np.linalg.norm(g0)
