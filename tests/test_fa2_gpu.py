"""FA2 engines on the GPU against the CPU oracle (through the C ABI).

Parity bar: forces, swing/traction stats, tree size and walk counts are
bit-identical to the oracle for every node whose edge list is shorter than
the hub threshold; hub attraction sums are reassociated and held to a 1e-6
relative L2 bound (1e-4 relative L2 per iteration).
The reference's engine-level tests are restated at the end
(crates/graph-compute/tests/gpu_engines.rs, layout_stability.rs).
"""
import numpy as np
import pytest

from conftest import spiral_seed

pytestmark = pytest.mark.gpu

BIG_HUB = {"hub_threshold": 1 << 30}  # every node summed in the reference's order


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def oracle_settings(s):
    return {k: v for k, v in s.items() if k != "hub_threshold"}


def one_step(jc, orc, g, pos, settings, bh=True, cap=None):
    e = jc.LayoutEngine("fa2-bh" if bh else "fa2-brute")
    e.set_params(settings)
    e.init(g, pos)
    out = e.step()
    f, st = e.forces()
    o = orc.Fa2(g, pos, bh=bh, **oracle_settings(settings))
    if cap:
        o.set_tree_capacity(cap)
    o.step()
    return e, out, f, st, o.get()


CASES = {
    "path24-theta0": (lambda jc: (jc.gen_path(24), spiral_seed(24)), {"theta": 0.0}),
    "path24-theta08": (lambda jc: (jc.gen_path(24), spiral_seed(24)), {"theta": 0.8}),
    "grid6-theta07": (lambda jc: (jc.gen_grid(6), spiral_seed(36)), {"theta": 0.7}),
    "ba2000-cube": (lambda jc: (jc.gen_scale_free(2000, 3, 9), jc.seed_uniform(2000, 3, 1)), {"theta": 0.8}),
    "ba9724-ball": (lambda jc: (jc.gen_scale_free(9724, 5, 0xC0FFEE), jc.seed_ball(9724, 0x5EED)), {}),
    "rmat13-cube": (lambda jc: (jc.gen_rmat(13, 65536, seed=2), jc.seed_uniform(8192, 3, 3)),
                    {"theta": 0.8, **BIG_HUB}),
    "ba3000-2d": (lambda jc: (jc.gen_scale_free(3000, 3, 4), jc.seed_uniform(3000, 2, 6)), {"theta": 0.8}),
    "ws2000-strong": (lambda jc: (jc.gen_watts_strogatz(2000, 6, 0.1, 3), jc.seed_uniform(2000, 3, 8)),
                      {"theta": 0.6, "strong_gravity": True, "scaling_ratio": 5.0, "gravity": 0.5}),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_one_step_bit_exact_against_oracle(jc, orc, case):
    make, settings = CASES[case]
    g, pos = make(jc)
    e, out, f, st, ref = one_step(jc, orc, g, pos, settings)
    assert np.array_equal(bits(f), bits(ref["force"])), rel_l2(f, ref["force"])
    assert np.array_equal(bits(st), bits(ref["stats"]))
    sp, eff = e.speed()
    assert sp == pytest.approx(ref["speed"], rel=1e-6) and eff == pytest.approx(ref["speed_eff"], rel=1e-6)
    assert rel_l2(out, ref["pos"]) < 1e-6
    if sp == ref["speed"]:
        assert np.array_equal(bits(out), bits(ref["pos"]))
    info = e.tree_info()
    assert info["nodes"] == ref["n_octree"]
    assert e.walk_counts() == (ref["n_inter"], ref["n_open"])


@pytest.mark.parametrize("group", [1, 2, 4, 8, 16, 32])
def test_walk_group_does_not_change_results(jc, orc, group):
    g = jc.gen_scale_free(3000, 3, 31)
    pos = jc.seed_uniform(3000, 3, 32)
    e, out, f, st, ref = one_step(jc, orc, g, pos, {"theta": 0.8, "walk_group": group})
    assert np.array_equal(bits(f), bits(ref["force"]))
    assert e.walk_counts() == (ref["n_inter"], ref["n_open"])


STAGE_CASES = {
    "one-body": (lambda jc: (jc.gen_path(1), np.array([0.5, -0.25, 1.0], np.float32))),
    "two-bodies": (lambda jc: (jc.gen_path(2), spiral_seed(2))),
    "path24": (lambda jc: (jc.gen_path(24), spiral_seed(24))),
    "ba3000-cube": (lambda jc: (jc.gen_scale_free(3000, 3, 31), jc.seed_uniform(3000, 3, 32))),
    "ba3000-2d": (lambda jc: (jc.gen_scale_free(3000, 3, 4), jc.seed_uniform(3000, 2, 6))),
    "rmat13-cube": (lambda jc: (jc.gen_rmat(13, 65536, seed=2), jc.seed_uniform(8192, 3, 3))),
}


@pytest.mark.parametrize("case", sorted(STAGE_CASES))
def test_staged_top_walk_matches_rope_walk(jc, orc, case):
    """The walk with the tree's top (depth <= 3) in shared memory visits the
    same nodes in the same order as the plain rope walk: forces and walk
    counts bit-identical to the unstaged engine and to the oracle, over 20
    steps."""
    g, pos = STAGE_CASES[case](jc)
    engines = []
    for stage in (True, False):
        e = jc.LayoutEngine("fa2-bh")
        e.set_params({"theta": 0.8, "walk_stage_top": stage, **BIG_HUB})
        e.init(g, pos)
        engines.append(e)
    o = orc.Fa2(g, pos, bh=True, theta=0.8)
    o.step()
    ref = o.get()
    for k in range(20):
        outs = [e.step() for e in engines]
        fs = [e.forces()[0] for e in engines]
        assert np.array_equal(bits(fs[0]), bits(fs[1])), k
        assert np.array_equal(bits(outs[0]), bits(outs[1])), k
        assert engines[0].walk_counts() == engines[1].walk_counts()
        if k == 0:
            assert np.array_equal(bits(fs[0]), bits(ref["force"]))
            assert engines[0].walk_counts() == (ref["n_inter"], ref["n_open"])


def test_tie_resort_for_bodies_sharing_21_levels(jc, orc):
    """Bodies 2e-7 apart in a root cell of ~2 share more than 21 octant digits:
    the 63-bit key ties and the conditional 96-bit re-sort must run."""
    n = 400
    pos = jc.seed_uniform(n, 3, 41).reshape(n, 3)
    for k in range(0, 120, 2):
        pos[k + 1] = pos[k] + np.array([2e-7, -1.2e-7, 0.0], np.float32)
    pos[200] = pos[2] + np.array([0.0, 0.0, 3e-7], np.float32)
    g = jc.gen_scale_free(n, 3, 2)
    e, out, f, st, ref = one_step(jc, orc, g, pos.reshape(-1), {"theta": 0.8}, cap=1 << 20)
    assert e.tree_info()["nodes"] == ref["n_octree"]
    assert e.tree_info()["max_depth"] > 21
    assert np.array_equal(bits(f), bits(ref["force"]))


@pytest.mark.parametrize("cluster", [24, 100])
def test_runs_sharing_the_top_key_half(jc, orc, cluster):
    """The single-graph sort orders by the top 32 key bits (ten octant levels)
    and then sorts each run of equal top halves; a cluster of 24 bodies in one
    level-10 cell is fixed in place, one of 100 takes the full re-sort."""
    n = 600
    pos = jc.seed_uniform(n, 3, 43).reshape(n, 3)
    rng = np.random.default_rng(44)
    pos[:cluster] = pos[300] + rng.uniform(-3e-4, 3e-4, (cluster, 3)).astype(np.float32)
    g = jc.gen_scale_free(n, 3, 5)
    e, out, f, st, ref = one_step(jc, orc, g, pos.reshape(-1), {"theta": 0.8}, cap=1 << 20)
    assert e.tree_info()["nodes"] == ref["n_octree"]
    assert np.array_equal(bits(f), bits(ref["force"]))
    assert e.walk_counts() == (ref["n_inter"], ref["n_open"])


def test_trajectory_parity_50_steps(jc, orc):
    g = jc.gen_scale_free(3000, 3, 21)
    pos = jc.seed_uniform(3000, 3, 22)
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": 0.8})
    e.init(g, pos)
    o = orc.Fa2(g, pos, bh=True, theta=0.8)
    for k in range(50):
        out = e.step()
        o.step()
        r = o.get()
        assert rel_l2(out, r["pos"]) < 1e-5, k
    f, _ = e.forces()
    assert rel_l2(f, r["force"]) < 1e-4


def test_hub_nodes_within_tolerance(jc, orc):
    """Nodes with >= hub_threshold edges are summed by a whole block."""
    g = jc.gen_rmat(15, 1 << 19, seed=5)
    pos = jc.seed_uniform(g.n_nodes, 3, 7)
    deg = np.diff(g.offsets.astype(np.int64))
    assert deg.max() >= 2048
    e, out, f, st, ref = one_step(jc, orc, g, pos, {"theta": 0.8})
    assert rel_l2(f, ref["force"]) < 1e-6
    light = np.repeat(deg < 2048, 3)
    assert np.array_equal(bits(f)[light], bits(ref["force"])[light])


def test_brute_engine_bit_exact(jc, orc):
    g = jc.gen_scale_free(1500, 4, 3)
    pos = jc.seed_uniform(1500, 3, 2)
    e, out, f, st, ref = one_step(jc, orc, g, pos, {}, bh=False)
    assert np.array_equal(bits(f), bits(ref["force"]))


def test_unsorted_asymmetric_csr_matches_oracle(jc, orc):
    rng = np.random.default_rng(11)
    n = 500
    rows = [list(rng.integers(0, n, rng.integers(0, 9))) + ([v] if v % 9 == 0 else []) for v in range(n)]
    off = np.zeros(n + 1, np.uint32)
    off[1:] = np.cumsum([len(r) for r in rows])
    g = jc.Csr(n, off, np.array([u for r in rows for u in r], np.uint32))
    pos = rng.uniform(-5, 5, 3 * n).astype(np.float32)
    e, out, f, st, ref = one_step(jc, orc, g, pos, {"theta": 0.8})
    assert np.array_equal(bits(f), bits(ref["force"]))


def _with_entry(jc, g, v, u):
    """The CSR g with u inserted into row v (rows stay strictly increasing)."""
    rows = [list(g.neighbors[g.offsets[i]:g.offsets[i + 1]]) for i in range(g.n_nodes)]
    rows[v] = sorted(rows[v] + [u])
    off = np.zeros(g.n_nodes + 1, np.uint32)
    off[1:] = np.cumsum([len(r) for r in rows])
    return jc.Csr(g.n_nodes, off, np.array([x for r in rows for x in r], np.uint32))


def test_csr_check_verdict_on_sorted_one_sided_entries(jc, orc, capfd, monkeypatch):
    """The device check's symmetry verdict (a search in the shorter row and a
    balance of the entries that did not search): a canonical CSR keeps the
    device lists, and a sorted, loop-free CSR with one one-sided entry, in a
    hub's row or pointing at the hub, is caught and takes the host rebuild.
    Forces equal the oracle's in all three cases."""
    monkeypatch.setenv("JC_TRACE", "1")
    g = jc.gen_scale_free(600, 3, 5)
    deg = np.diff(g.offsets.astype(np.int64))
    hub = int(np.argmax(deg))
    hub_row = set(g.neighbors[g.offsets[hub]:g.offsets[hub + 1]].tolist())
    x = next(i for i in range(g.n_nodes) if i != hub and i not in hub_row and deg[i] > 0)
    pos = jc.seed_uniform(600, 3, 9)
    for csr, general in ((g, False), (_with_entry(jc, g, hub, x), True), (_with_entry(jc, g, x, hub), True)):
        capfd.readouterr()
        e, out, f, st, ref = one_step(jc, orc, csr, pos, {"theta": 0.8})
        err = capfd.readouterr().err
        assert ("general_csr" in err) == general, err[-400:]
        assert np.array_equal(bits(f), bits(ref["force"]))
        e.close()


def test_coincident_bodies_depth_cap(jc, orc):
    """Duplicates are dropped from the tree as the reference's depth cap does."""
    g = jc.gen_scale_free(400, 2, 1)
    pos = jc.seed_uniform(400, 3, 1).reshape(-1, 3)
    pos[10] = pos[3]
    pos[11] = pos[3]
    pos[200] = pos[199]
    pos = pos.reshape(-1)
    e, out, f, st, ref = one_step(jc, orc, g, pos, {"theta": 0.8})
    assert np.array_equal(bits(f), bits(ref["force"]))
    assert e.tree_info()["dropped"] == 3
    assert e.status_bits() & jc.JC_WARN_DEPTH_CAP


def test_non_finite_body(jc, orc):
    g = jc.gen_path(50)
    pos = spiral_seed(50)
    pos[3 * 7 + 1] = np.nan
    e, out, f, st, ref = one_step(jc, orc, g, pos, {"theta": 0.5})
    nan = np.isnan(f)
    assert np.array_equal(nan, np.isnan(ref["force"]))
    assert nan[3 * 7 + 1] and nan.sum() >= 1
    assert np.array_equal(bits(f)[~nan], bits(ref["force"])[~nan])
    assert e.status_bits() & jc.JC_WARN_NONFINITE


def test_tree_capacity_grows(jc, orc):
    """Tight clusters need long single-child chains: more nodes than 3n+64.
    The engine grows its tree (the reference would truncate at 2n+8)."""
    n = 64
    pos = np.zeros((n, 3), np.float32)
    pos[:, 0] = np.arange(n, dtype=np.float32) * 100.0
    for k in range(0, n, 2):
        # partners 0.01 apart share ~19 octant digits below a 6.5e3 root cell
        pos[k + 1] = pos[k] + np.array([0.01, 0.0, 0.0], np.float32)
    g = jc.gen_path(n)
    e, out, f, st, ref = one_step(jc, orc, g, pos.reshape(-1), {"theta": 0.8}, cap=1 << 20)
    assert e.tree_info()["nodes"] == ref["n_octree"] > 3 * n + 64
    assert np.array_equal(bits(f), bits(ref["force"]))
    assert e.status_bits() & jc.JC_WARN_REF_CAPACITY


def test_empty_and_tiny_graphs(jc, orc):
    for n in (0, 1, 2, 3):
        g = jc.gen_path(n)
        pos = spiral_seed(n)
        for eid in ("fa2-bh", "fa2-brute"):
            e = jc.LayoutEngine(eid)
            e.init(g, pos)
            out = e.step()
            assert len(out) == 3 * n
            if n:
                o = orc.Fa2(g, pos, bh=eid == "fa2-bh")
                o.step()
                assert np.array_equal(bits(out), bits(o.get()["pos"]))


def test_step_many_equals_repeated_steps(jc):
    g = jc.gen_scale_free(2000, 3, 5)
    pos = jc.seed_uniform(2000, 3, 5)
    a = jc.LayoutEngine("fa2-bh")
    a.init(g, pos)
    for _ in range(7):
        ra = a.step()
    b = jc.LayoutEngine("fa2-bh")
    b.init(g, pos)
    rb = b.step_many(7)
    assert np.array_equal(bits(ra), bits(rb))


def test_eager_launches_match_graph_replays(jc):
    g = jc.gen_scale_free(3000, 3, 8)
    pos = jc.seed_uniform(3000, 3, 8)
    runs = []
    for use_graph in (True, False):
        e = jc.LayoutEngine("fa2-bh")
        e.set_params({"theta": 0.8, "use_graph": use_graph})
        e.init(g, pos)
        runs.append(e.step_many(12))
    assert np.array_equal(bits(runs[0]), bits(runs[1]))


def test_save_load_state_resumes_exactly(jc):
    g = jc.gen_scale_free(1000, 3, 2)
    pos = jc.seed_uniform(1000, 3, 2)
    e = jc.LayoutEngine("fa2-bh")
    e.init(g, pos)
    e.step_many(10)
    blob = e.save_state()
    a = e.step_many(10)
    e.load_state(blob)
    b = e.step_many(10)
    assert np.array_equal(bits(a), bits(b))
    fresh = jc.LayoutEngine("fa2-bh")
    fresh.init(g, pos)
    fresh.load_state(blob)
    assert np.array_equal(bits(fresh.step_many(10)), bits(a))


def test_reinit_to_another_graph(jc, orc):
    e = jc.LayoutEngine("fa2-bh")
    e.init(jc.gen_path(100), spiral_seed(100))
    e.step_many(3)
    g = jc.gen_grid(12)
    pos = spiral_seed(144)
    e.reinit(g, pos)
    out = e.step()
    o = orc.Fa2(g, pos, bh=True)
    o.step()
    assert np.array_equal(bits(out), bits(o.get()["pos"]))


# ---- the reference's engine tests (gpu_engines.rs, layout_stability.rs) ----
def test_gpu_engines_run_and_move(jc):
    """gpu_engines.rs:75-106."""
    g = jc.gen_path(32)
    s = spiral_seed(32)
    for eid in ("fa2-brute", "fa2-bh"):
        e = jc.LayoutEngine(eid)
        e.init(g, s)
        out = e.step_many(30)
        assert len(out) == len(s) and np.all(np.isfinite(out))
        assert np.abs(out - s).sum() > 1e-3


def test_barnes_hut_matches_brute_force_single_step(jc):
    """gpu_engines.rs:114-143 (documented as failing in the reference)."""
    g = jc.gen_path(24)
    s = spiral_seed(24)
    b = jc.LayoutEngine("fa2-brute")
    b.init(g, s)
    bo = b.step()
    h = jc.LayoutEngine("fa2-bh")
    h.set_params({"theta": 0.0})
    h.init(g, s)
    ho = h.step()
    assert np.max(np.abs(bo - ho)) < 5e-2


def test_fa2_single_edge_stays_finite(jc):
    """gpu_engines.rs:176-195."""
    e = jc.LayoutEngine("fa2-brute")
    e.init(jc.gen_path(2), np.array([0, 0, 0, 5, 0, 0], np.float32))
    for _ in range(400):
        assert np.all(np.isfinite(e.step()))


def test_fa2_triangle_relaxes_to_equilateral(jc):
    """gpu_engines.rs:200-224."""
    tri = jc.csr_from_pairs(3, [(0, 1), (1, 2), (2, 0)])
    e = jc.LayoutEngine("fa2-brute")
    e.init(tri, np.array([0, 0, 0, 10, 0, 0, 3, 4, 0], np.float32))
    out = e.step_many(600).reshape(3, 3)
    d = [np.linalg.norm(out[a] - out[b]) for a, b in ((0, 1), (1, 2), (2, 0))]
    mean = np.mean(d)
    assert mean > 1e-3 and max(abs(x - mean) for x in d) / mean < 0.15


def test_fa2_bh_is_run_to_run_bit_exact(jc):
    """gpu_engines.rs:405-430."""
    g = jc.gen_grid(6)
    s = spiral_seed(36)
    runs = []
    for _ in range(2):
        e = jc.LayoutEngine("fa2-bh")
        e.set_params({"theta": 0.7})
        e.init(g, s)
        for _ in range(60):
            out = e.step()
        runs.append(out)
    assert np.all(np.isfinite(runs[0]))
    assert np.array_equal(bits(runs[0]), bits(runs[1]))


def test_fa2_bh_stable_at_vault_scale_synthetic(jc):
    """layout_stability.rs:133-149 with assert_stable (:91-129)."""
    n = 9724
    g = jc.gen_scale_free(n, 5, 0xC0FFEE)
    s = jc.seed_ball(n, 0x5EED)
    e = jc.LayoutEngine("fa2-bh")
    e.init(g, s)
    steps = 1000
    prev = s.copy()
    disp, mx, med_r = [], 0.0, 0.0
    for _ in range(steps):
        cur = e.step()
        disp.append(float(np.median(np.linalg.norm((cur - prev).reshape(-1, 3), axis=1))))
        prev = cur
    ceiling = np.sqrt(n) * 5.0 + steps * 10.0
    assert np.all(np.isfinite(cur))
    assert np.max(np.abs(cur)) <= 1.01 * ceiling
    r = np.linalg.norm(cur.reshape(-1, 3), axis=1)
    assert 1.0 < np.median(r) < 0.25 * ceiling
    early = np.median(disp[steps // 10:steps // 3])
    mid = np.median(disp[steps // 3:2 * steps // 3])
    late = np.median(disp[8 * steps // 10:])
    assert late <= mid * 1.15 and mid <= early * 1.15
    assert late < 0.5 * early or late < 0.05


# ---- tolerance mode of the walk (fast_repulsion) ----
@pytest.mark.parametrize("case", ["ba2000-cube", "rmat13-cube", "ba3000-2d", "ws2000-strong"])
def test_fast_repulsion_within_tolerance(jc, orc, case):
    """Approximate reciprocal + fused accumulation in the repulsion terms
    only: the same nodes are visited (walk counts and tree equal the
    oracle's) and the force vector stays within 1e-5 relative L2 of the
    oracle's (the per-iteration bar is 1e-4)."""
    make, settings = CASES[case]
    g, pos = make(jc)
    e, out, f, st, ref = one_step(jc, orc, g, pos, {**settings, "fast_repulsion": True})
    assert rel_l2(f, ref["force"]) < 1e-5
    assert e.walk_counts() == (ref["n_inter"], ref["n_open"])
    assert e.tree_info()["nodes"] == ref["n_octree"]


def test_fast_repulsion_trajectory(jc, orc):
    g = jc.gen_scale_free(3000, 3, 21)
    pos = jc.seed_uniform(3000, 3, 22)
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": 0.8, "fast_repulsion": True})
    e.init(g, pos)
    o = orc.Fa2(g, pos, bh=True, theta=0.8)
    for k in range(50):
        out = e.step()
        o.step()
        f, _ = e.forces()
        r = o.get()
        # per iteration: the force vector within the 1e-4 bar of the oracle
        # step taken from the same state
        assert rel_l2(f, r["force"]) < 1e-4, k
        o.set_state(pos=out, old_force=f, speed=e.speed()[0], speed_eff=e.speed()[1])


def test_init_rejects_out_of_range_ids(jc, orc):
    """fa2-bh checks the neighbour ids while it stages them to the device;
    a bad id is JC_ERR_ARG and the engine can be initialised again."""
    g = jc.gen_scale_free(3000, 3, 8)
    pos = jc.seed_uniform(3000, 3, 8)
    bad = jc.Csr(g.n_nodes, g.offsets.copy(), g.neighbors.copy())
    bad.neighbors[len(bad.neighbors) - 3] = 3000
    e = jc.LayoutEngine("fa2-bh")
    with pytest.raises(jc.JcError) as ei:
        e.init(bad, pos)
    assert ei.value.code == jc.JC_ERR_ARG and "out of range" in str(ei.value)
    e.set_params({"theta": 0.8})
    e.init(g, pos)
    e.step()
    f, _ = e.forces()
    o = orc.Fa2(g, pos, bh=True, theta=0.8)
    o.step()
    assert np.array_equal(bits(f), bits(o.get()["force"]))
