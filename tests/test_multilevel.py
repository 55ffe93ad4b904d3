"""The multilevel wrapper's host side on the CPU
(crates/graph-compute/src/engines/multilevel.rs,
crates/graph-layouts/src/layout/coarsen.rs): the library's matching cascade
(jc_coarsen) against the oracle restatement (oracle/multilevel.cpp), both
against the reference's own tests (coarsen.rs:325-358, multilevel.rs:520-858),
and the settings contract."""
import numpy as np
import pytest


def cascades_equal(a, b):
    assert len(a) == len(b)
    for (na, ea, pa), (nb, eb, pb) in zip(a, b):
        assert na == nb
        assert np.array_equal(ea, eb)
        assert np.array_equal(pa, pb)


def graphs(jc):
    rng = np.random.default_rng(9)
    return [jc.gen_path(6), jc.gen_path(1000), jc.gen_grid(40, 30), jc.gen_scale_free(3000, 3, 2),
            jc.gen_watts_strogatz(2000, 6, 0.1, 3), jc.gen_rgg(3000, 0.03, 4),
            jc.csr_from_pairs(500, rng.integers(0, 500, (300, 2)).tolist()),  # isolated nodes, sparse
            jc.gen_rmat(12, 20000, 0.57, 0.19, 0.19, 5)]


@pytest.mark.parametrize("max_levels,target", [(6, 500), (4, 2), (10, 50), (1, 10), (0, 10)])
def test_cascade_matches_oracle(jc, orc, max_levels, target):
    for g in graphs(jc):
        e = orc.csr_edges(g)
        got = jc.coarsen(g.n_nodes, e, max_levels, target)
        want = orc.Cascade(g.n_nodes, e, max_levels, target).levels
        cascades_equal(got, want)


def test_cascade_edge_cases(jc, orc):
    # out-of-range ids and self-loops in the flat list are skipped, as the reference does
    e = np.array([0, 1, 1, 1, 2, 9, 3, 4, 4, 2, 0, 1], np.uint32)
    cascades_equal(jc.coarsen(5, e, 6, 1), orc.Cascade(5, e, 6, 1).levels)
    # an edge-free graph stops at once: the matching makes no progress
    lv = jc.coarsen(100, np.zeros(0, np.uint32), 6, 10)
    assert len(lv) == 1 and lv[0][0] == 100
    assert len(jc.coarsen(0, np.zeros(0, np.uint32), 6, 10)) == 1


def test_coarsen_collapses_a_path(jc):
    """coarsen_collapses_a_path (coarsen.rs:325-336): pairs (0,1),(2,3),(4,5)."""
    lv = jc.coarsen(6, [0, 1, 1, 2, 2, 3, 3, 4, 4, 5], 4, 2)
    assert lv[0][0] == 6 and len(lv) >= 2
    assert lv[1][0] == 3 and lv[1][2].tolist() == [0, 0, 1, 1, 2, 2]
    assert lv[1][1].tolist() == [0, 1, 1, 2]


def test_single_edge_folds_to_its_midpoint(orc):
    """fold_up_averages_children (multilevel.rs:568-583)."""
    c = orc.Cascade(2, [0, 1], 4, 1)
    assert len(c.levels) == 2
    assert np.array_equal(c.fold_up([0, 0, 0, 2, 0, 0]), np.array([1, 0, 0], np.float32))


def test_level_csr_and_schedules(orc):
    """level_csr_is_symmetric, schedule_concrete_values, schedule_anneals_coarse_ge_fine
    (multilevel.rs:520-530, :655-668, :620-653)."""
    off, nb = orc.level_csr(3, [0, 1, 1, 2])
    assert off.tolist() == [0, 1, 3, 4] and nb.tolist() == [1, 0, 2, 1]
    assert orc.sweeps_for_level("linear", 0, 4) == 4 and orc.sweeps_for_level("linear", 2, 4) == 12
    assert orc.sweeps_for_level("geometric", 0, 4) == 4 and orc.sweeps_for_level("geometric", 3, 4) == 32
    assert orc.sweeps_for_level("linear", 0, 0) == 1
    for sched in ("uniform", "linear", "geometric"):
        v = [orc.sweeps_for_level(sched, l, 30) for l in range(20)]
        assert all(b >= a for a, b in zip(v, v[1:]))


def test_prolong_without_jitter_inherits(orc):
    """prolong_inherits_parent_position (coarsen.rs:349-357)."""
    out = orc.prolong([10, 20, 30], [0, 0], 2, 0.0, 7)
    assert out.tolist() == [10, 20, 30, 10, 20, 30]


def test_settings_contract(jc):
    """rejects_self_wrap / rejects_unknown_inner / accepts_known_inner /
    settings_backcompat_without_sweep_schedule (multilevel.rs:532-566, :587-600)."""
    with jc.LayoutEngine("multilevel") as e:
        d = e.descriptor()
        assert d["id"] == "multilevel" and d["kind"] == "Physics"
        e.set_params("null")
        e.set_params({"inner": "sgd-stress", "max_levels": 5, "target_size": 100, "sweeps_per_level": 20})
        e.set_params({"inner": "fa2-bh", "inner_params": {"theta": 0.8, "gravity": 2.0},
                      "sweep_schedule": "geometric", "spring_len": 10.0, "seed": 7})
        e.set_params({"inner_params": None})
        for bad in [{"inner": "multilevel"}, {"inner": "no-such-engine"}, {"sweep_schedule": "cubic"},
                    {"max_levels": -1}, {"seed": 1.5}, {"inner": 3}]:
            with pytest.raises(jc.JcError) as ei:
                e.set_params(bad)
            assert ei.value.code == jc.JC_ERR_PARAMS, bad
        assert e.level_info() == (0, 0, 0)  # no cascade before init
    with jc.LayoutEngine("fa2-bh") as e:
        with pytest.raises(jc.JcError):
            e.level_info()  # not a multilevel engine
