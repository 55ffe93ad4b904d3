"""The CTA-per-graph schedule of the batched fa2-bh engine
(batch_schedule = 1): every graph of a batch owned by one CTA of a
persistent launch that runs all requested iterations. Each graph must evolve
bit for bit as on the forest schedule and as in an engine of its own
(same octree, walk, forces, adaptive speed), through the tie re-sort, tree
capacity growth, non-finite bodies and the autotuner's probes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TILE = {"theta": 0.8, "batch_schedule": 1}
FOREST = {"theta": 0.8, "batch_schedule": 0}


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def small_batch(jc):
    graphs = [jc.gen_scale_free(700, 3, 1), jc.gen_watts_strogatz(500, 6, 0.1, 2), jc.gen_path(1),
              jc.gen_grid(9), jc.gen_rgg(900, float(np.sqrt(6 / (np.pi * 900))), 3), jc.gen_path(2),
              jc.gen_scale_free(1500, 2, 4), jc.gen_scale_free(9000, 3, 7)]
    pos = [jc.seed_uniform(g.n_nodes, 2 if k % 2 else 3, 10 + k) for k, g in enumerate(graphs)]
    return graphs, pos


def engine(jc, params, graphs, pos):
    e = jc.LayoutEngine("fa2-bh")
    e.set_params(params)
    e.init_batch(graphs, pos)
    return e


def test_tile_schedule_is_taken(jc):
    graphs, pos = small_batch(jc)
    assert engine(jc, TILE, graphs, pos).batch_schedule()[0]
    assert not engine(jc, FOREST, graphs, pos).batch_schedule()[0]


def test_tile_matches_forest_and_independent_engines(jc):
    graphs, pos = small_batch(jc)
    t = engine(jc, TILE, graphs, pos)
    f = engine(jc, FOREST, graphs, pos)
    off = np.concatenate([[0], np.cumsum([g.n_nodes for g in graphs])])
    singles = []
    for g, p in zip(graphs, pos):
        e = jc.LayoutEngine("fa2-bh")
        e.set_params({"theta": 0.8})
        e.init(g, p)
        singles.append(e)
    for step in range(4):
        ot = t.step()
        of = f.step()
        ft, st = t.forces()
        ff, sf = f.forces()
        assert np.array_equal(bits(ft), bits(ff)), step
        assert np.array_equal(bits(st), bits(sf)), step
        assert np.array_equal(bits(ot), bits(of)), step
        assert t.walk_counts() == f.walk_counts()
        assert t.tree_info()["nodes"] == f.tree_info()["nodes"]
        for k, e in enumerate(singles):
            o = e.step()
            fe, _ = e.forces()
            sl = slice(3 * off[k], 3 * off[k + 1])
            assert np.array_equal(bits(ft[sl]), bits(fe)), (step, k)
            assert np.array_equal(bits(ot[sl]), bits(o)), (step, k)
            assert t.graph_speed(k) == f.graph_speed(k)


def test_tile_against_oracle(jc, orc):
    graphs, pos = small_batch(jc)
    t = engine(jc, TILE, graphs, pos)
    t.step_many(3, readback=False)
    out = t.positions()
    off = np.concatenate([[0], np.cumsum([g.n_nodes for g in graphs])])
    for k, (g, p) in enumerate(zip(graphs, pos)):
        o = orc.Fa2(g, p, bh=True, theta=0.8)
        for _ in range(3):
            o.step()
        assert np.array_equal(bits(out[3 * off[k]:3 * off[k + 1]]), bits(o.get()["pos"])), k


def test_tile_step_many_equals_single_steps(jc):
    graphs, pos = small_batch(jc)
    a = engine(jc, TILE, graphs, pos)
    for _ in range(9):
        ra = a.step()
    b = engine(jc, TILE, graphs, pos)
    rb = b.step_many(9)
    c = engine(jc, FOREST, graphs, pos)
    rc = c.step_many(9)
    assert np.array_equal(bits(ra), bits(rb)) and np.array_equal(bits(rb), bits(rc))


def test_tile_ties_capacity_and_non_finite(jc):
    """A graph whose bodies tie in 21+ levels (full re-sort), one whose tree
    needs more than 3n+64 nodes (regions grow, the same target is re-run),
    and one with a non-finite body, among ordinary graphs."""
    n = 400
    x_tie = jc.seed_uniform(n, 3, 41).reshape(n, 3)
    for k in range(0, 120, 2):
        x_tie[k + 1] = x_tie[k] + np.array([2e-7, -1.2e-7, 0.0], np.float32)
    rng = np.random.default_rng(44)
    x_tie[200:300] = x_tie[300] + rng.uniform(-3e-4, 3e-4, (100, 3)).astype(np.float32)
    m = 64
    x_cap = np.zeros((m, 3), np.float32)
    x_cap[:, 0] = np.arange(m, dtype=np.float32) * 100.0
    for k in range(0, m, 2):
        x_cap[k + 1] = x_cap[k] + np.array([0.01, 0.0, 0.0], np.float32)
    x_nan = jc.seed_uniform(300, 3, 5)
    x_nan[3 * 17] = np.nan
    graphs = [jc.gen_scale_free(n, 3, 2), jc.gen_path(m), jc.gen_scale_free(300, 2, 3), jc.gen_grid(20)]
    pos = [x_tie.reshape(-1), x_cap.reshape(-1), x_nan, jc.seed_uniform(400, 2, 9)]
    t = engine(jc, TILE, graphs, pos)
    f = engine(jc, FOREST, graphs, pos)
    for step in range(3):
        t.step_many(1, readback=False)
        f.step_many(1, readback=False)
        ft, _ = t.forces()
        ff, _ = f.forces()
        nan = np.isnan(ff)
        assert np.array_equal(np.isnan(ft), nan)
        assert np.array_equal(bits(ft)[~nan], bits(ff)[~nan]), step
    assert t.tree_info()["nodes"] == f.tree_info()["nodes"]
    bits_t = t.status_bits()  # reading clears the warning bits
    assert bits_t & jc.JC_WARN_NONFINITE and bits_t & jc.JC_WARN_REF_CAPACITY
    pt, pf = t.positions(), f.positions()
    nan = np.isnan(pf)
    assert np.array_equal(bits(pt)[~nan], bits(pf)[~nan])


def test_tile_not_taken_with_a_hub_list(jc):
    graphs = [jc.gen_rmat(15, 1 << 19, seed=5), jc.gen_path(50)]
    assert np.diff(graphs[0].offsets.astype(np.int64)).max() >= 2048
    pos = [jc.seed_uniform(g.n_nodes, 3, 3 + k) for k, g in enumerate(graphs)]
    e = engine(jc, TILE, graphs, pos)
    assert not e.batch_schedule()[0]


def test_autotune_times_the_tile_schedule_and_keeps_the_state(jc):
    graphs, pos = small_batch(jc)
    a = engine(jc, {"theta": 0.8}, graphs, pos)
    a.step_many(3, readback=False)
    group, ms = a.autotune(2)
    tile, tile_ms = a.batch_schedule()
    assert tile_ms > 0.0 and np.all(ms > 0)
    assert tile == (tile_ms < ms.min())
    ra = a.step_many(5)
    b = engine(jc, FOREST, graphs, pos)
    b.step_many(3, readback=False)
    rb = b.step_many(5)
    assert np.array_equal(bits(ra), bits(rb))


def test_tile_frames_and_checkpoint(jc):
    graphs, pos = small_batch(jc)
    t = engine(jc, TILE, graphs, pos)
    t.step_many(2, readback=False)
    blob = t.save_state()
    t.stream_open("f32", depth=2)
    t.stream_step()
    fr = t.stream_next()
    assert np.array_equal(bits(fr.payload), bits(t.positions()))
    t.stream_close()
    after = t.step_many(4)
    t.load_state(blob)
    again = t.step_many(5)  # 2 + 5 from the checkpoint == 2 + 1 (frame) + 4
    assert np.array_equal(bits(after), bits(again))
