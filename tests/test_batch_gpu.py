"""Batched layout of many independent graphs in one engine (fa2-bh,
jc_engine_init_batch): every graph must evolve exactly as it would in its own
engine (same octree, same forces, its own adaptive speed), and the autotuner
must leave the layout state untouched."""
import numpy as np
import pytest

from conftest import spiral_seed

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def small_batch(jc):
    graphs = [jc.gen_scale_free(700, 3, 1), jc.gen_watts_strogatz(500, 6, 0.1, 2), jc.gen_path(1),
              jc.gen_grid(9), jc.gen_rgg(900, float(np.sqrt(6 / (np.pi * 900))), 3), jc.gen_path(2),
              jc.gen_scale_free(1500, 2, 4)]
    pos = [jc.seed_uniform(g.n_nodes, 2 if k % 2 else 3, 10 + k) for k, g in enumerate(graphs)]
    return graphs, pos


def test_batch_matches_independent_engines(jc):
    graphs, pos = small_batch(jc)
    b = jc.LayoutEngine("fa2-bh")
    b.set_params({"theta": 0.8})
    b.init_batch(graphs, pos)
    off = np.concatenate([[0], np.cumsum([g.n_nodes for g in graphs])])
    singles = []
    for g, p in zip(graphs, pos):
        e = jc.LayoutEngine("fa2-bh")
        e.set_params({"theta": 0.8})
        e.init(g, p)
        singles.append(e)
    for step in range(4):
        out = b.step()
        fb, _ = b.forces()
        for k, e in enumerate(singles):
            o = e.step()
            f, _ = e.forces()
            sl = slice(3 * off[k], 3 * off[k + 1])
            assert np.array_equal(bits(fb[sl]), bits(f)), (step, k)
            assert np.allclose(out[sl], o, rtol=1e-6, atol=1e-6), (step, k)
            assert b.graph_speed(k)[0] == pytest.approx(e.speed()[0], rel=1e-6)


def test_batch_against_oracle(jc, orc):
    graphs, pos = small_batch(jc)
    b = jc.LayoutEngine("fa2-bh")
    b.init_batch(graphs, pos)
    b.step()
    fb, _ = b.forces()
    off = np.concatenate([[0], np.cumsum([g.n_nodes for g in graphs])])
    for k, (g, p) in enumerate(zip(graphs, pos)):
        o = orc.Fa2(g, p, bh=True)
        o.step()
        assert np.array_equal(bits(fb[3 * off[k]:3 * off[k + 1]]), bits(o.get()["force"])), k


def test_autotune_keeps_the_state(jc):
    graphs, pos = small_batch(jc)
    a = jc.LayoutEngine("fa2-bh")
    a.init_batch(graphs, pos)
    a.step_many(3)
    group, ms = a.autotune(2)
    assert group in (1, 2, 4, 8, 16, 32) and np.all(ms > 0)
    ra = a.step_many(5)
    b = jc.LayoutEngine("fa2-bh")
    b.init_batch(graphs, pos)
    b.step_many(3)
    rb = b.step_many(5)
    assert np.array_equal(bits(ra), bits(rb))


def test_batch_walk_groups_agree(jc):
    graphs, pos = small_batch(jc)
    outs = []
    for group in (1, 8, 32):
        e = jc.LayoutEngine("fa2-bh")
        e.set_params({"walk_group": group})
        e.init_batch(graphs, pos)
        outs.append(e.step_many(3))
    assert np.array_equal(bits(outs[0]), bits(outs[1])) and np.array_equal(bits(outs[0]), bits(outs[2]))


def test_high_word_ties_in_a_large_batch(jc):
    """3,000 graphs put a 12-bit graph id in the high key word, which then
    holds 17 octant levels. Two bodies 1e-6 apart in graph 0 share all 64
    high bits and differ only in the low word: the run fix-up must order them
    by the full key, giving graph 0 exactly the tree (and forces) of its own
    engine, where the high word holds 21 levels and they do not tie."""
    g0 = jc.gen_scale_free(300, 2, 5)
    x0 = jc.seed_uniform(g0.n_nodes, 3, 6)
    x0[3 * 7:3 * 7 + 3] = x0[3 * 3:3 * 3 + 3] + np.array([1e-6, -1e-6, 5e-7], np.float32)
    x0[3 * 8:3 * 8 + 3] = x0[3 * 3:3 * 3 + 3] + np.array([-1e-6, 2e-6, 0.0], np.float32)
    graphs = [g0] + [jc.gen_path(2) for _ in range(2999)]
    pos = [x0] + [jc.seed_uniform(2, 3, 100 + k) for k in range(2999)]
    b = jc.LayoutEngine("fa2-bh")
    b.set_params({"theta": 0.8})
    b.init_batch(graphs, pos)
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": 0.8})
    e.init(g0, x0)
    for _ in range(3):
        b.step_many(1, readback=False)
        e.step_many(1, readback=False)
        fb, _ = b.forces()
        fe, _ = e.forces()
        assert np.array_equal(bits(fb[:3 * g0.n_nodes]), bits(fe))
    assert np.array_equal(bits(b.positions()[:3 * g0.n_nodes]), bits(e.positions()))
    b.close()
    e.close()


def test_batch_builder_matches_init_batch(jc):
    """jc_batch_* (graphs added one at a time) lays out exactly what
    jc_engine_init_batch does, and reads each graph's slice from the device."""
    graphs, pos = small_batch(jc)
    ref = jc.LayoutEngine("fa2-bh")
    ref.set_params({"theta": 0.8})
    ref.init_batch(graphs, pos)
    ref.step_many(7, readback=False)
    want = ref.positions()
    off = np.concatenate([[0], np.cumsum([g.n_nodes for g in graphs])])
    with jc.Batch({"theta": 0.8}) as b:
        for k, (g, p) in enumerate(zip(graphs, pos)):
            assert b.add_graph(g, p) == k
        b.bind()
        with pytest.raises(jc.JcError) as ei:
            b.add_graph(graphs[0], pos[0])
        assert ei.value.code == jc.JC_ERR_STATE
        assert np.array_equal(bits(b.positions(3)), bits(pos[3]))  # bound, not yet stepped
        b.run(3)
        b.run(4)
        for k in range(len(graphs)):
            assert np.array_equal(bits(b.positions(k)), bits(want[3 * off[k]: 3 * off[k + 1]])), k
        eng = b.engine()
        assert np.array_equal(bits(eng.positions()), bits(want))
        eng.step_many(2, readback=False)
        ref.step_many(2, readback=False)
        assert np.array_equal(bits(b.positions(6)), bits(ref.positions()[3 * off[6]:]))
        with pytest.raises(jc.JcError):
            b.positions(len(graphs))
    ref.close()
