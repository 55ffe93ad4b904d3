"""jc_fa2_bh_forces_noalloc: the Barnes-Hut force pass for callers that
cannot allocate device memory (for example a host framework that hands the
library a fixed device-memory budget). Its scratch lives in a static device
array inside the library; inputs and outputs are the caller's device buffers.

The checks:
  * two calls in a row (different graphs, so stale scratch from the first
    call would show) give forces bit-identical to the existing fa2-bh engine
    entry points (jc_engine_init + jc_engine_step + jc_engine_forces), the
    same exactness bar as the other force-parity tests;
  * against the oracle directly, on a graph with a node of degree >= 2048
    (the engine sums such rows with a block reduction; this pass sums every
    row in order, so it is bit-identical to the oracle), with the default
    force law and with lin_log_mode + strong gravity (logf on the device vs
    the host's logf: within 1e-6 relative L2);
  * a malformed CSR (a neighbour id >= n, decreasing offsets, a missing
    neighbour array) is rejected with JC_ERR_ARG by the device check before
    anything is gathered through it, and the next call works again.
Collected last (file name) so that a run stopping at the first failure has
run every other test first; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def engine_forces(jc, g, pos, theta):
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": theta})
    e.init(g, pos)
    e.step()
    f, _ = e.forces()
    e.close()
    return f


def to_dev(torch, g, pos):
    dev = torch.device("cuda", 0)
    off = torch.from_numpy(g.offsets.astype(np.int32)).to(dev)
    nb = torch.from_numpy(g.neighbors.astype(np.int32)).to(dev)
    p = torch.from_numpy(pos.astype(np.float32)).to(dev)
    out = torch.full((3 * g.n_nodes,), float("nan"), dtype=torch.float32, device=dev)
    return off, nb, p, out


def noalloc_forces(jc, torch, g, pos, theta, **law):
    off, nb, p, out = to_dev(torch, g, pos)
    torch.cuda.synchronize()
    jc.fa2_bh_forces_noalloc(g.n_nodes, off.data_ptr(), nb.data_ptr(), p.data_ptr(), out.data_ptr(), theta=theta,
                             **law)
    return out.cpu().numpy()


def test_noalloc_force_pass_matches_engine_twice(jc):
    torch = pytest.importorskip("torch")
    jc.set_device(0)
    grid = jc.gen_grid(40, 25)
    grid = jc.csr_from_pairs(grid.n_nodes, grid.pairs())  # rows ascending: row order = the engine's edge order
    cases = [(jc.gen_scale_free(3000, 3, 17), 3, 0.8), (grid, 2, 0.6)]
    for g, dim, theta in cases:
        pos = jc.seed_uniform(g.n_nodes, dim, 99)
        ref = engine_forces(jc, g, pos, theta)
        got = noalloc_forces(jc, torch, g, pos, theta)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_noalloc_matches_oracle_with_a_hub_and_lin_log(jc, orc):
    torch = pytest.importorskip("torch")
    jc.set_device(0)
    g = jc.gen_rmat(14, 1 << 17, seed=12)
    deg = np.diff(g.offsets.astype(np.int64))
    assert deg.max() >= 2048 and g.n_nodes <= 32768
    pos = jc.seed_uniform(g.n_nodes, 3, 13)
    laws = [({"theta": 0.8}, True),
            ({"theta": 0.7, "lin_log_mode": True, "strong_gravity": True, "gravity": 0.5, "scaling_ratio": 3.0},
             False)]
    for law, exact in laws:
        o = orc.Fa2(g, pos, bh=True, **law)
        o.force_pass()
        ref = o.get()["force"]
        kw = {k: v for k, v in law.items() if k != "theta"}
        got = noalloc_forces(jc, torch, g, pos, law["theta"], **kw)
        assert np.all(np.isfinite(got))
        if exact:
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), rel_l2(got, ref)
        else:
            assert rel_l2(got, ref) < 1e-6


def test_noalloc_rejects_a_malformed_csr(jc):
    torch = pytest.importorskip("torch")
    jc.set_device(0)
    g = jc.gen_scale_free(2000, 3, 5)
    pos = jc.seed_uniform(g.n_nodes, 3, 6)
    good = noalloc_forces(jc, torch, g, pos, 0.8)

    bad_id = jc.Csr(g.n_nodes, g.offsets.copy(), g.neighbors.copy())
    bad_id.neighbors[len(bad_id.neighbors) // 2] = g.n_nodes + 5
    bad_off = jc.Csr(g.n_nodes, g.offsets.copy(), g.neighbors.copy())
    i = 700
    bad_off.offsets[i], bad_off.offsets[i + 1] = g.offsets[i + 1], g.offsets[i]  # row i decreases, all in range
    assert bad_off.offsets[i] > bad_off.offsets[i + 1]
    for bad in (bad_id, bad_off):
        with pytest.raises(jc.JcError) as ei:
            noalloc_forces(jc, torch, bad, pos, 0.8)
        assert ei.value.code == jc.JC_ERR_ARG

    off, nb, p, out = to_dev(torch, g, pos)
    torch.cuda.synchronize()
    with pytest.raises(jc.JcError) as ei:
        jc.fa2_bh_forces_noalloc(g.n_nodes, off.data_ptr(), 0, p.data_ptr(), out.data_ptr(), theta=0.8)
    assert ei.value.code == jc.JC_ERR_ARG

    # the scratch keeps nothing of the failed calls
    again = noalloc_forces(jc, torch, g, pos, 0.8)
    assert np.array_equal(again.view(np.uint32), good.view(np.uint32))


def test_noalloc_rejects_oversized_graphs(jc):
    torch = pytest.importorskip("torch")
    with pytest.raises(jc.JcError) as ei:
        jc.fa2_bh_forces_noalloc(32769, 1, 1, 1, 1)
    assert ei.value.code == jc.JC_ERR_CAPACITY
