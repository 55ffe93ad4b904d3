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
