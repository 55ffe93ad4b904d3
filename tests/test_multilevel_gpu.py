"""The "multilevel" wrapper on the GPU against an emulation of the reference's
wrapper (crates/graph-compute/src/engines/multilevel.rs:359-468) built from
the oracle: the oracle's cascade, fold-up, prolongation and level CSRs
(oracle/multilevel.cpp) driving the oracle's FA2 engine level by level. The
device folds the seed up, draws the prolongation jitter (a jump-ahead of the
reference's xorshift stream) and rebinds the inner engine from device
positions; every step's positions must equal the emulation's bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def emulate(jc, orc, g, x, steps, bh, theta, max_levels, target, spl, schedule, spring_len, seed):
    cas = orc.Cascade(g.n_nodes, orc.csr_edges(g), max_levels, target)
    lv = cas.levels
    level = len(lv) - 1
    pos = cas.fold_up(x)

    def bind(level, pos):
        off, nb = orc.level_csr(lv[level][0], lv[level][1])
        return orc.Fa2(jc.Csr(lv[level][0], off, nb), pos, bh=bh, theta=theta)

    eng, sweeps, outs, levels = bind(level, pos), 0, [], []
    for _ in range(steps):
        eng.step(1)
        p = eng.get()["pos"].reshape(-1)
        sweeps += 1
        if level > 0 and sweeps >= orc.sweeps_for_level(schedule, level, spl):
            child = level - 1
            p = orc.prolong(p, lv[level][2], lv[child][0], np.float32(spring_len) * np.float32(0.5),
                            (seed + child + 1) & 0xFFFFFFFF)
            level, sweeps = child, 0
            eng = bind(level, p)
        outs.append(p.copy())
        levels.append(level)
    return outs, levels, cas


@pytest.mark.parametrize("inner,graph,target,spl,schedule", [("fa2-bh", "grid30x27", 40, 2, "linear"),
                                                             ("fa2-brute", "ws800", 60, 2, "geometric"),
                                                             ("fa2-bh", "grid80x75", 500, 1, "uniform")])
def test_descent_matches_the_oracle_emulation(jc, orc, inner, graph, target, spl, schedule):
    g = {"grid30x27": lambda: jc.gen_grid(30, 27), "ws800": lambda: jc.gen_watts_strogatz(800, 4, 0.05, 3),
         "grid80x75": lambda: jc.gen_grid(80, 75)}[graph]()
    x = jc.seed_uniform(g.n_nodes, 3, 72)
    params = {"inner": inner, "inner_params": {"theta": 0.8}, "max_levels": 6, "target_size": target,
              "sweeps_per_level": spl, "sweep_schedule": schedule, "spring_len": 12.0, "seed": 0x5EED}
    n_levels = len(orc.Cascade(g.n_nodes, orc.csr_edges(g), 6, target).levels)
    assert n_levels >= 5
    steps = sum(orc.sweeps_for_level(schedule, l, spl) for l in range(1, n_levels)) + 5
    want, want_levels, cas = emulate(jc, orc, g, x, steps, inner == "fa2-bh", 0.8, 6, target, spl, schedule, 12.0,
                                     0x5EED)
    assert want_levels[-1] == 0
    e = jc.LayoutEngine("multilevel")
    e.set_params(params)
    e.init(g, x)
    got_cascade = e.cascade()
    assert len(got_cascade) == len(cas.levels)
    for (na, ea, pa), (nb, eb, pb) in zip(got_cascade, cas.levels):
        assert na == nb and np.array_equal(ea, eb) and np.array_equal(pa, pb)
    # the coarsest level starts from the folded seed
    assert np.array_equal(e.positions(), cas.fold_up(x))
    for t in range(steps):
        out = e.step()
        level, n_levels, _ = e.level_info()
        assert level == want_levels[t]
        assert np.array_equal(out, want[t]), (t, level)
    e.close()


def test_step_many_crosses_levels_like_single_steps(jc):
    g = jc.gen_watts_strogatz(3000, 6, 0.1, 5)
    x = jc.seed_uniform(3000, 3, 6)
    params = {"inner": "fa2-bh", "inner_params": {"theta": 0.8}, "target_size": 100, "sweeps_per_level": 4}
    a = jc.LayoutEngine("multilevel")
    a.set_params(params)
    a.init(g, x)
    for _ in range(75):
        a.step()
    b = jc.LayoutEngine("multilevel")
    b.set_params(params)
    b.init(g, x)
    b.step_many(30, readback=False)
    b.step_many(45, readback=False)
    assert a.level_info() == b.level_info()
    assert np.array_equal(a.positions(), b.positions())
    a.close()
    b.close()


def test_full_descent_with_sgd_inner(jc):
    """full_descent_reaches_finest_level_with_real_inner (multilevel.rs:826-857)."""
    g = jc.gen_path(8)
    x = np.zeros(24, np.float32)
    x[0::3] = np.arange(8, dtype=np.float32)
    for inner in ("sgd-stress", "sgd-stress-gpu"):
        e = jc.LayoutEngine("multilevel")
        e.set_params({"inner": inner, "max_levels": 6, "target_size": 2, "sweeps_per_level": 2})
        e.init(g, x)
        for _ in range(500):
            out = e.step()
        assert e.level_info()[0] == 0
        assert out.shape == (24,) and np.all(np.isfinite(out))
        e.close()


def test_runs_are_reproducible_and_state_round_trips(jc):
    """reinit_reuse_is_deterministic_and_matches (multilevel.rs:800-806), plus
    save / load of the cascade position and the inner state."""
    g = jc.gen_grid(50, 40)
    x = jc.seed_uniform(2000, 2, 8)
    params = {"inner": "fa2-bh", "target_size": 100, "sweeps_per_level": 5}
    runs = []
    for _ in range(2):
        e = jc.LayoutEngine("multilevel")
        e.set_params(params)
        e.init(g, x)
        e.step_many(20, readback=False)
        runs.append((e.level_info(), e.positions()))
        if len(runs) == 1:
            state = e.save_state()
            e.step_many(25, readback=False)
            after = (e.level_info(), e.positions())
        e.close()
    assert runs[0][0] == runs[1][0] and np.array_equal(runs[0][1], runs[1][1])
    e = jc.LayoutEngine("multilevel")
    e.set_params(params)
    e.init(g, x)
    e.load_state(state)
    e.step_many(25, readback=False)
    assert e.level_info() == after[0] and np.array_equal(e.positions(), after[1])
    e.close()


def test_inner_params_errors_surface_at_init(jc):
    g = jc.gen_path(100)
    e = jc.LayoutEngine("multilevel")
    e.set_params({"inner": "fa2-bh", "inner_params": {"theta": "wide"}})
    with pytest.raises(jc.JcError) as ei:
        e.init(g, jc.seed_uniform(100, 3, 1))
    assert ei.value.code == jc.JC_ERR_PARAMS
    e.close()
