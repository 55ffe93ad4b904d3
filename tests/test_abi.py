"""C-ABI contract of libjc_layout.so without a GPU: exports, registry,
descriptors, set_params decoding, argument validation and the seeded graph
generators (crates/graph-compute/src/engines/mod.rs:383-488,
crates/graph-compute/src/stability.rs)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def header_functions():
    text = (ROOT / "include" / "jc_layout.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol(jc):
    L = jc.lib()
    names = header_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_registry_lists_layout_engines(jc):
    ids = jc.engine_ids()
    assert set(ids) == {"fa2-bh", "fa2-brute", "sgd-stress", "sgd-stress-gpu", "multilevel"}
    h = ctypes.c_void_p()
    assert jc.lib().jc_engine_create(b"cpu-spring", ctypes.byref(h)) == jc.JC_ERR_UNKNOWN_ENGINE
    assert jc.lib().jc_engine_create(b"nope", ctypes.byref(h)) == jc.JC_ERR_UNKNOWN_ENGINE


@pytest.mark.parametrize("eid", ["fa2-bh", "fa2-brute", "sgd-stress", "sgd-stress-gpu"])
def test_descriptor(jc, eid):
    with jc.LayoutEngine(eid) as e:
        d = e.descriptor()
        assert d["id"] == eid
        assert d["kind"] == "Physics"
        assert d["requirements"] == {"needs_edges": True, "needs_cpu_positions": True,
                                     "needs_gpu_positions_buffer": False}
        assert not e.is_halted()


def test_set_params_serde_semantics(jc):
    """fa2_bh.rs:212-220: null keeps, objects replace (defaults for missing
    fields), unknown keys ignored, wrong types rejected."""
    with jc.LayoutEngine("fa2-bh") as e:
        e.set_params(None if False else "null")
        e.set_params({"theta": 0.8, "gravity": 2})
        e.set_params({"theta": 0.5, "not_a_field": [1, {"x": 2}], "dim": 2})
        e.set_params("{}")
        for bad in ['{"theta": "x"}', '{"strong_gravity": 1}', '{"theta": 0.1, "theta": 0.2}', "[1,2]",
                    '{"theta": 0.8', '{"hub_threshold": -1}', '{"hub_threshold": 1.5}', "3"]:
            with pytest.raises(jc.JcError) as ei:
                e.set_params(bad)
            assert ei.value.code == jc.JC_ERR_PARAMS, bad
    with jc.LayoutEngine("sgd-stress") as e:
        e.set_params({"n_pivots": 200, "seed": 18446744073709551615, "eta_max": 1e3})
        with pytest.raises(jc.JcError):
            e.set_params({"n_pivots": 4294967296})
        with pytest.raises(jc.JcError):
            e.set_params({"seed": -5})


def test_step_before_init_is_a_state_error(jc):
    for eid in jc.engine_ids():
        with jc.LayoutEngine(eid) as e:
            with pytest.raises(jc.JcError) as ei:
                e.step()
            assert ei.value.code == jc.JC_ERR_STATE


def test_init_validates_the_csr(jc):
    with jc.LayoutEngine("fa2-bh") as e:
        good = jc.gen_path(4)
        with pytest.raises(jc.JcError) as ei:
            e.init(good, np.zeros(11, np.float32))
        assert ei.value.code == jc.JC_ERR_ARG
        bad = jc.Csr(4, np.array([0, 1, 3, 2, 6], np.uint32), good.neighbors)
        with pytest.raises(jc.JcError) as ei:
            e.init(bad, np.zeros(12, np.float32))
        assert ei.value.code == jc.JC_ERR_ARG and "non-decreasing" in str(ei.value)
        # neighbour ids are range-checked by the staged upload on the way to
        # the device (tests/test_fa2_gpu.py::test_init_rejects_out_of_range_ids);
        # the other engines check them on the host
    with jc.LayoutEngine("sgd-stress") as e:
        oob = jc.Csr(4, good.offsets, np.array([1, 0, 9, 1, 3, 2], np.uint32))
        with pytest.raises(jc.JcError) as ei:
            e.init(oob, np.zeros(12, np.float32))
        assert "out of range" in str(ei.value)


# ---- generators (product code; stability.rs fixtures restated) -----------
def test_splitmix_uniform_seed_matches_reference_generator(jc):
    """stability.rs:11-26 next_f32 = (next_u64 >> 40) / 2^24, from SplitMix64
    whose first outputs for seed 0 are Vigna's published test vectors."""
    mask = (1 << 64) - 1

    def splitmix(seed, k):
        out, s = [], seed
        for _ in range(k):
            s = (s + 0x9E3779B97F4A7C15) & mask
            z = s
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
            out.append(z ^ (z >> 31))
        return out

    assert splitmix(0, 3) == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]
    u = jc.seed_uniform(5, 3, 1234)
    ref = [np.float32(2.0) * np.float32((x >> 40) / (1 << 24)) - np.float32(1.0) for x in splitmix(1234, 15)]
    assert np.array_equal(u, np.array(ref, np.float32))
    u2 = jc.seed_uniform(5, 2, 1234)
    assert np.all(u2[2::3] == 0)


def test_ball_seed_shape(jc):
    n = 1000
    p = jc.seed_ball(n, 0x5EED).reshape(n, 3)
    r = np.linalg.norm(p, axis=1)
    assert np.all(r <= np.sqrt(n) * 5.0 * (1 + 1e-6))
    assert np.all(np.isfinite(p))


def test_scale_free_profile(jc):
    """stability.rs:51-55: n=9724, m=5 gives ~48k edges, symmetric sorted CSR."""
    g = jc.gen_scale_free(9724, 5, 0xC0FFEE)
    m = len(g.neighbors) // 2
    assert 40000 < m < 50000
    for v in range(0, g.n_nodes, 97):
        row = g.neighbors[g.offsets[v]:g.offsets[v + 1]]
        assert np.all(np.diff(row.astype(np.int64)) > 0) and v not in row


def test_csr_from_pairs_dedups_and_drops_self_loops(jc):
    g = jc.csr_from_pairs(4, [(0, 1), (1, 0), (2, 2), (1, 3), (3, 1), (0, 9)])
    assert g.offsets.tolist() == [0, 1, 3, 3, 4]
    assert g.neighbors.tolist() == [1, 0, 3, 1]


def test_grid_neighbour_order(jc):
    """gpu_engines.rs:267-292 grid2d: left, right, up, down."""
    g = jc.gen_grid(3)
    assert g.neighbors[g.offsets[4]:g.offsets[5]].tolist() == [3, 5, 1, 7]
    assert g.n_nodes == 9 and len(g.neighbors) == 24


def test_rmat_unique_edges(jc):
    g = jc.gen_rmat(10, 5000, seed=3)
    assert g.n_nodes == 1024 and len(g.neighbors) == 10000
    pairs = g.pairs()
    assert len(np.unique(pairs[:, 0].astype(np.int64) * 2048 + pairs[:, 1])) == 5000


def test_ws_and_rgg(jc):
    ws = jc.gen_watts_strogatz(1000, 6, 0.1, 9)
    assert abs(len(ws.neighbors) / 1000 - 6.0) < 0.2
    n = 20000
    r = float(np.sqrt(6.0 / (np.pi * n)))
    g, pts = jc.gen_rgg(n, r, 4, return_points=True)
    assert 5.0 < len(g.neighbors) / n < 6.5
    e = g.pairs()
    d = np.linalg.norm(pts[e[:, 0]].astype(np.float64) - pts[e[:, 1]], axis=1)
    assert np.all(d <= r * (1 + 1e-6))


def test_csr_binary_round_trip(jc):
    """sim.rs:53-129 wire format."""
    g = jc.gen_scale_free(300, 3, 1)
    h = jc.Csr.from_bin(g.to_bin())
    assert h.n_nodes == g.n_nodes and np.array_equal(h.offsets, g.offsets)
    assert np.array_equal(h.neighbors, g.neighbors)
    with pytest.raises(ValueError):
        jc.Csr.from_bin(g.to_bin()[:-1])
