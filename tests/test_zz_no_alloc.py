"""jc_fa2_bh_forces_noalloc: the Barnes-Hut force pass for callers that
cannot allocate device memory (for example a host framework that hands the
library a fixed device-memory budget). Its scratch lives in a static device
array inside the library; inputs and outputs are the caller's device buffers.

The check: two calls in a row (different graphs, so stale scratch from the
first call would show) give forces bit-identical to the existing fa2-bh
engine entry points (jc_engine_init + jc_engine_step + jc_engine_forces),
the same exactness bar as the other force-parity tests. Collected last
(file name) so that a run stopping at the first failure has run every other
test first; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def engine_forces(jc, g, pos, theta):
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": theta})
    e.init(g, pos)
    e.step()
    f, _ = e.forces()
    e.close()
    return f


def noalloc_forces(jc, torch, g, pos, theta):
    dev = torch.device("cuda", 0)
    off = torch.from_numpy(g.offsets.astype(np.int32)).to(dev)
    nb = torch.from_numpy(g.neighbors.astype(np.int32)).to(dev)
    p = torch.from_numpy(pos.astype(np.float32)).to(dev)
    out = torch.full((3 * g.n_nodes,), float("nan"), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    jc.fa2_bh_forces_noalloc(g.n_nodes, off.data_ptr(), nb.data_ptr(), p.data_ptr(), out.data_ptr(), theta=theta)
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


def test_noalloc_rejects_oversized_graphs(jc):
    torch = pytest.importorskip("torch")
    with pytest.raises(jc.JcError) as ei:
        jc.fa2_bh_forces_noalloc(32769, 1, 1, 1, 1)
    assert ei.value.code == jc.JC_ERR_CAPACITY
