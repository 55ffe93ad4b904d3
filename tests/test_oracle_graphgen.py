"""The oracle's own workload generator (oracle/graphgen.cpp) builds the same
R-MAT graph and uniform seed as the product library, so the benchmark's
reference arm and CPU-baseline leg can build their inputs without loading
the product library."""
import numpy as np
import pytest


@pytest.mark.parametrize("scale,edges,seed", [(10, 4000, 3), (14, 1 << 17, 12), (16, 1 << 19, 20)])
def test_oracle_rmat_equals_library_rmat(jc, orc, scale, edges, seed):
    a = jc.gen_rmat(scale, edges, 0.57, 0.19, 0.19, seed)
    b = orc.gen_rmat(scale, edges, 0.57, 0.19, 0.19, seed)
    assert a.n_nodes == b.n_nodes == 1 << scale
    assert np.array_equal(a.offsets, b.offsets)
    assert np.array_equal(a.neighbors, b.neighbors)
    assert len(b.neighbors) == 2 * edges


def test_oracle_rmat_equals_library_rmat_at_the_headline_size(jc, orc):
    a = jc.gen_rmat(20, 16_777_216, 0.57, 0.19, 0.19, 20)
    b = orc.gen_rmat(20, 16_777_216, 0.57, 0.19, 0.19, 20)
    assert np.array_equal(a.offsets, b.offsets)
    assert np.array_equal(a.neighbors, b.neighbors)


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_seed_equals_library_seed(jc, orc, dim):
    assert np.array_equal(jc.seed_uniform(5000, dim, 21).view(np.uint32),
                          orc.seed_uniform(5000, dim, 21).view(np.uint32))


def test_oracle_csr_from_pairs(jc, orc):
    pairs = [(0, 1), (1, 0), (2, 2), (3, 1), (1, 3), (4, 0), (9, 1)]
    a = jc.csr_from_pairs(5, pairs)
    b = orc.csr_from_pairs(5, pairs)
    assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.neighbors, b.neighbors)
