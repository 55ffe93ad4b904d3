"""Partition-driven batching on the GPU: one fa2-bh engine lays out every
partition of partition_csr (crates/graph-compute/src/partition.rs:191) as one
batch, and must give each partition exactly the trajectory of its own engine
on that partition's local graph (what the reference's BSP workers run,
run_superstep_local, partition.rs:1099-1136; FA2 keeps the default no-op
apply_halo). The coordinator's view (owned positions at their global ids)
and the boundary HaloDelta payloads (boundary_delta, partition.rs:116-158)
are read from the batch on the device."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def per_partition_engines(jc, P, x, steps):
    """Each partition in its own engine, seeded from the global positions."""
    out = []
    for part in P:
        if part.local.n_nodes == 0:
            out.append(np.zeros(0, np.float32))
            continue
        e = jc.LayoutEngine("fa2-bh")
        e.set_params({"theta": 0.8})
        xs = x.reshape(-1, 3)[part.global_ids].reshape(-1)
        e.init(part.local, xs)
        e.step_many(steps, readback=False)
        out.append(e.positions())
        e.close()
    return out


@pytest.mark.parametrize("refine", [False, True])
def test_batch_of_partitions_equals_one_engine_per_partition(jc, refine):
    g = jc.gen_scale_free(6000, 3, 61)
    x = jc.seed_uniform(g.n_nodes, 3, 62)
    P = jc.partition_csr(g, 6, refine=refine)
    want = per_partition_engines(jc, P, x, 25)
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": 0.8})
    e.init_partitions(P, x)
    e.step_many(25, readback=False)
    assert np.array_equal(e.positions(), np.concatenate(want))
    glob = e.partition_positions()
    expect = np.zeros((g.n_nodes, 3), np.float32)
    for part, w in zip(P, want):
        expect[part.owned_global_ids] = w.reshape(-1, 3)[:part.n_owned]
    assert np.array_equal(glob, expect.reshape(-1))
    for i, part in enumerate(P):
        h = e.halo_delta(i)
        assert np.array_equal(h.reshape(-1, 3), expect[part.boundary])
    e.close()


def test_partitions_with_empty_ones_and_frames(jc):
    g = jc.gen_path(3)
    x = jc.seed_uniform(3, 3, 7)
    P = jc.partition_csr(g, 5)
    e = jc.LayoutEngine("fa2-bh")
    e.init_partitions(P, x)
    e.step_many(4, readback=False)
    want = per_partition_engines(jc, P, x, 4)
    assert np.array_equal(e.positions(), np.concatenate(want))
    assert [len(e.halo_delta(i)) for i in range(5)] == [3, 3, 3, 0, 0]
    # the frame stream carries the batch positions (owned + ghosts)
    e.stream_open("f32", depth=1)
    e.stream_step(2)
    f = e.stream_next()
    assert np.array_equal(f.payload, e.positions())
    e.close()


def test_partition_layout_needs_a_partition_binding(jc):
    g = jc.gen_path(50)
    e = jc.LayoutEngine("fa2-bh")
    e.init(g, jc.seed_uniform(50, 3, 1))
    assert jc.lib().jc_engine_partition_positions(e._h, None) == jc.JC_ERR_STATE
    P = jc.partition_csr(g, 3)
    e.init_partitions(P, jc.seed_uniform(50, 3, 1))
    assert e.partition_positions().shape == (150,)
    e.init(g, jc.seed_uniform(50, 3, 1))  # re-binding drops the partition layout
    rc = jc.lib().jc_engine_partition_positions(e._h, None)
    assert rc == jc.JC_ERR_STATE
    e.close()
