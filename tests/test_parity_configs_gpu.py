"""Parity on the configurations the measured numbers are quoted on.

  * The headline graph: R-MAT scale 20 (1,048,576 nodes, 16,777,216 unique
    undirected edges, a,b,c,d = .57/.19/.19/.05, seed 20; uniform [-1,1]^3
    seed from seed 21, theta 0.8) -- the exact workload bench.py times. One
    step against the oracle from the seed, and one step from the state the
    device reached after 50 steps (positions, previous forces, speed and
    speed efficiency handed to the oracle), where the tree is no longer the
    uniform seed's. Forces and swing/traction are bit-identical for every
    node whose list is shorter than the hub threshold (2048 entries; the
    engine sums longer lists with a reassociated block reduction), the whole
    force vector is within 1e-6 relative L2 from the seed and within the
    per-iteration bar of 1e-4 after 50 steps,
    and the tree size and the walk counts are equal.
  * The reference's CPU-path run: Barabasi-Albert n=10,000, m=3, uniform
    [-1,1]^3 seed, theta 0.8, scaling 2, gravity 1, 500 iterations, device
    against oracle: final scale-normalized stress (metrics.rs:31-59, over
    the terms of 32 BFS pivots) within 0.5 %, final positions close.
  * Barnes-Hut against the exact O(n^2) FP64 force oracle at n = 20,000:
    theta 0 within 1e-5 relative L2, theta 0.8 within 5 % and equal to the
    oracle's own Barnes-Hut error (the device forces are the oracle's).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HUB = 2048


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def rmat20(jc):
    g = jc.gen_rmat(20, 16_777_216, 0.57, 0.19, 0.19, 20)
    pos = jc.seed_uniform(g.n_nodes, 3, 21)
    return g, pos


def check_step(e, o, deg, hub_bar=1e-6, speed_rel=1e-6):
    f, st = e.forces()
    ref = o.get()
    light3 = np.repeat(deg < HUB, 3)
    light2 = np.repeat(deg < HUB, 2)
    assert np.array_equal(bits(f)[light3], bits(ref["force"])[light3])
    assert np.array_equal(bits(st)[light2], bits(ref["stats"])[light2])
    assert rel_l2(f, ref["force"]) < hub_bar
    assert e.tree_info()["nodes"] == ref["n_octree"]
    assert e.walk_counts() == (ref["n_inter"], ref["n_open"])
    sp, eff = e.speed()
    assert sp == pytest.approx(ref["speed"], rel=speed_rel) and eff == pytest.approx(ref["speed_eff"], rel=speed_rel)
    assert rel_l2(e.positions(), ref["pos"]) < hub_bar


def test_rmat20_headline_step_against_oracle(jc, orc, rmat20):
    g, pos = rmat20
    assert g.n_nodes == 1 << 20 and len(g.neighbors) == 2 * 16_777_216
    deg = np.diff(g.offsets.astype(np.int64))
    assert deg.max() >= HUB  # the hub path is exercised
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": 0.8})
    e.init(g, pos)
    e.step_many(1, readback=False)
    o = orc.Fa2(g, pos, bh=True, theta=0.8)
    o.step()
    check_step(e, o, deg)


def test_rmat20_step_after_50_steps_against_oracle(jc, orc, rmat20):
    g, pos = rmat20
    deg = np.diff(g.offsets.astype(np.int64))
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": 0.8})
    e.init(g, pos)
    e.step_many(50, readback=False)
    p50 = e.positions()
    f50, _ = e.forces()
    sp, eff = e.speed()
    o = orc.Fa2(g, p50, bh=True, theta=0.8)
    o.set_state(pos=p50, old_force=f50, speed=sp, speed_eff=eff)
    e.step_many(1, readback=False)
    o.step()
    # after 50 steps the hubs' 3e4-7e4-entry sums cancel to forces of ~4e9:
    # their reassociated block sums differ from the list-order sums by
    # ~1e-5 relative (measured 8.8e-6), inside the 1e-4 per-iteration bar;
    # the hubs' swing and traction enter the f64 speed sums, so the adaptive
    # speed moves by as much (measured 7.8e-5 relative)
    check_step(e, o, deg, hub_bar=1e-4, speed_rel=1e-3)


def pivot_terms(orc, g, k, seed):
    rng = np.random.default_rng(seed)
    piv = rng.choice(g.n_nodes, size=k, replace=False)
    ti, tj, td = [], [], []
    for j in piv:
        d = orc.bfs(g, int(j)).astype(np.int64)
        ok = (d != 0xFFFFFFFF) & (d > 0)
        idx = np.nonzero(ok)[0]
        ti.append(idx)
        tj.append(np.full(len(idx), j))
        td.append(d[idx])
    ti, tj, td = np.concatenate(ti), np.concatenate(tj), np.concatenate(td)
    return list(zip(ti.tolist(), tj.tolist(), td.astype(float).tolist()))


def test_ba10k_500_iterations_final_stress_within_half_percent(jc, orc):
    g = jc.gen_scale_free(10000, 3, 0xBA)
    pos = jc.seed_uniform(g.n_nodes, 3, 0xBA + 1)
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": 0.8, "scaling_ratio": 2.0, "gravity": 1.0})
    e.init(g, pos)
    dev = e.step_many(500)
    o = orc.Fa2(g, pos, bh=True, theta=0.8, scaling_ratio=2.0, gravity=1.0)
    for _ in range(500):
        o.step()
    ref = o.get()["pos"]
    assert np.all(np.isfinite(dev))
    terms = pivot_terms(orc, g, 32, 7)
    s_dev = orc.scale_normalized_stress(dev, terms)
    s_ref = orc.scale_normalized_stress(ref, terms)
    assert abs(s_dev - s_ref) <= 0.005 * s_ref, (s_dev, s_ref)
    assert rel_l2(dev, ref) < 1e-3


@pytest.mark.parametrize("theta", [0.0, 0.8])
def test_barnes_hut_against_exact_fp64_at_20k(jc, orc, theta):
    n = 20_000
    g = jc.gen_scale_free(n, 3, 2020)
    pos = jc.seed_uniform(n, 3, 2021)
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": theta})
    e.init(g, pos)
    e.step_many(1, readback=False)
    f, _ = e.forces()
    o = orc.Fa2(g, pos, bh=True, theta=theta)
    exact = o.exact_forces_f64()
    o.force_pass()
    err = rel_l2(f, exact)
    if theta == 0.0:
        assert err < 1e-5, err
    else:
        assert err < 0.05, err
        assert err == pytest.approx(rel_l2(o.get()["force"], exact), rel=1e-6)
