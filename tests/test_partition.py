"""Edge-cut partitioning on the CPU (crates/graph-compute/src/partition.rs):
the library's partitioner (jc_partition_csr) against the oracle restatement
(oracle/partition.py), and both against the reference's own partition tests
(partition.rs:1140-1801), restated here with their pinned values."""
import numpy as np
import pytest

from oracle import partition as opart


def ring(jc, n):
    """ring(n) of the reference tests (partition.rs:1521-1535): row i = [i-1, i+1] mod n."""
    off = np.arange(0, 2 * n + 1, 2, dtype=np.uint32)
    nb = np.array([[(i + n - 1) % n, (i + 1) % n] for i in range(n)], np.uint32).reshape(-1)
    return jc.Csr(n, off, nb)


def undirected(jc, n, edges):
    """undirected(n, edges) of the reference tests (partition.rs:1538-1557)."""
    adj = [[] for _ in range(n)]
    for u, v in edges:
        adj[u].append(v)
        adj[v].append(u)
    off, nb = [0], []
    for a in adj:
        nb += sorted(a)
        off.append(len(nb))
    return jc.Csr(n, np.array(off, np.uint32), np.array(nb, np.uint32))


def oracle_parts(g, p, refine):
    off, nb = [int(x) for x in g.offsets], [int(x) for x in g.neighbors]
    f = opart.partition_csr_refined if refine else opart.partition_csr
    return f(g.n_nodes, off, nb, p)


def same_as_oracle(g, P, want):
    assert len(P) == len(want)
    for got, w in zip(P.parts, want):
        assert got.partition_id == w.partition_id and got.n_partitions == w.n_partitions
        assert got.n_owned == w.n_owned
        assert got.global_ids.tolist() == w.global_ids
        assert got.boundary.tolist() == w.boundary
        assert got.local.offsets.tolist() == w.offsets
        assert got.local.neighbors.tolist() == w.neighbors


def invariants(g, P):
    """assert_partition_invariants (partition.rs:1589-1638)."""
    owned = np.sort(np.concatenate([p.owned_global_ids for p in P.parts] + [np.zeros(0, np.uint32)]))
    assert owned.tolist() == list(range(g.n_nodes))
    ghosts = set()
    for p in P.parts:
        assert np.all(p.local.neighbors < p.local.n_nodes)
        assert p.n_owned + len(p.ghost_global_ids) == p.local.n_nodes
        ghosts |= set(p.ghost_global_ids.tolist())
    for p in P.parts:
        want = {int(v) for v in p.owned_global_ids if int(v) in ghosts}
        assert set(p.boundary.tolist()) == want
        assert np.all(np.diff(p.boundary.astype(np.int64)) > 0)


def cut_of(g, owner):
    src = np.repeat(np.arange(g.n_nodes), np.diff(g.offsets.astype(np.int64)))
    m = src < g.neighbors
    return int(np.sum(owner[src[m]] != owner[g.neighbors[m]]))


def graphs(jc):
    rng = np.random.default_rng(3)
    pairs = rng.integers(0, 300, (500, 2))
    gs = [jc.gen_path(6), jc.gen_path(11), ring(jc, 8), ring(jc, 16), jc.gen_grid(9, 7),
          jc.gen_scale_free(400, 3, 5), jc.gen_watts_strogatz(300, 6, 0.2, 6),
          jc.gen_rgg(500, 0.05, 7), jc.csr_from_pairs(300, pairs.tolist()),  # isolated nodes
          jc.gen_rmat(9, 2000, 0.57, 0.19, 0.19, 8)]
    # a CSR with self-loops and a repeated neighbour (not canonical)
    gs.append(jc.Csr(4, np.array([0, 3, 5, 7, 8], np.uint32), np.array([0, 1, 1, 0, 2, 1, 3, 2], np.uint32)))
    return gs


@pytest.mark.parametrize("refine", [False, True])
def test_library_matches_oracle(jc, refine):
    for g in graphs(jc):
        for p in (1, 2, 3, 4, 7, 16):
            P = jc.partition_csr(g, p, refine=refine)
            same_as_oracle(g, P, oracle_parts(g, p, refine))
            invariants(g, P)
            assert P.edge_cut == cut_of(g, P.owner)


def test_path_split_in_two(jc):
    """partition_path_two_ways / superstep_ships_fewer_than_owned (partition.rs:1140-1172, :1378-1419)."""
    P = jc.partition_csr(jc.gen_path(6), 2)
    assert [p.owned_global_ids.tolist() for p in P] == [[0, 1, 2], [3, 4, 5]]
    assert [p.ghost_global_ids.tolist() for p in P] == [[3], [2]]
    assert [p.boundary.tolist() for p in P] == [[2], [3]]
    assert P.edge_cut == 1


def test_bfs_suboptimal_cut_refines_to_one(jc):
    """refine_strictly_reduces_when_bfs_suboptimal (partition.rs:1692-1730): BFS
    owners [0,0,1,0,0,1,1,1], cut 3; FM moves node 7, cut 1, sizes in [3, 5]."""
    g = undirected(jc, 8, [(0, 3), (0, 4), (1, 3), (2, 4), (2, 5), (3, 4), (3, 7), (4, 7), (5, 6)])
    raw = jc.partition_csr(g, 2)
    assert raw.owner.tolist() == [0, 0, 1, 0, 0, 1, 1, 1]
    assert raw.edge_cut == 3
    ref = jc.partition_csr(g, 2, refine=True)
    assert ref.edge_cut == 1
    assert all(3 <= p.n_owned <= 5 for p in ref)
    invariants(g, ref)


def test_refinement_never_raises_the_cut_and_stays_balanced(jc):
    """refine_does_not_increase_cut / refine_stays_balanced (partition.rs:1660-1690, :1732-1756)."""
    for g in (jc.gen_path(6), jc.gen_path(12), ring(jc, 8), ring(jc, 12), ring(jc, 16)):
        for p in (2, 3, 4):
            raw = jc.partition_csr(g, p)
            ref = jc.partition_csr(g, p, refine=True)
            assert ref.edge_cut <= raw.edge_cut
            ideal = g.n_nodes / p
            lo, hi = int(np.floor(0.9 * ideal)), int(np.ceil(1.1 * ideal))
            if g.n_nodes >= 12:
                assert all(lo <= q.n_owned <= hi for q in ref), [q.n_owned for q in ref]


def test_degenerate_inputs(jc):
    """empty_graph_partitions_cleanly / refine_handles_degenerate_inputs (partition.rs:1188-1201, :1793-1813)."""
    empty = jc.Csr(0, np.zeros(1, np.uint32), np.zeros(0, np.uint32))
    for refine in (False, True):
        P = jc.partition_csr(empty, 3, refine=refine)
        assert len(P) == 3 and all(p.n_owned == 0 and p.local.n_nodes == 0 for p in P)
    one = jc.partition_csr(jc.gen_path(5), 1, refine=True)
    assert len(one) == 1 and one[0].n_owned == 5 and len(one[0].boundary) == 0
    # more partitions than nodes: the rest stay empty
    P = jc.partition_csr(jc.gen_path(3), 5)
    assert [p.n_owned for p in P] == [1, 1, 1, 0, 0]
    # zero partitions is taken as one
    assert len(jc.partition_csr(jc.gen_path(4), 0)) == 1


def test_rejects_malformed_csr(jc):
    bad = jc.Csr(3, np.array([0, 1, 2, 3], np.uint32), np.array([1, 2, 9], np.uint32))
    with pytest.raises(jc.JcError):
        jc.partition_csr(bad, 2)
