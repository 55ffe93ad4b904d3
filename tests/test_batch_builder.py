"""The batch builder (jc_batch_*) on the host: handle lifecycle, argument
checks and state errors, none of which touch the device. The device side
(bind, run, per-graph positions) is in test_batch_gpu.py."""
import numpy as np
import pytest


def test_builder_validates_graphs(jc):
    with jc.Batch({"theta": 0.8}) as b:
        assert len(b) == 0
        g = jc.gen_path(5)
        assert b.add_graph(g, jc.seed_uniform(5, 3, 1)) == 0
        assert b.add_graph(jc.gen_grid(3, 3), jc.seed_uniform(9, 3, 2)) == 1
        assert len(b) == 2
        L = jc.lib()
        pos = np.zeros(15, np.float32)
        bad_off = np.array([0, 1, 2, 3, 4, 3], np.uint32)  # decreasing
        nb = np.array([1, 0, 2], np.uint32)
        for off, nbr, nnz, want in [(bad_off, nb, 3, jc.JC_ERR_ARG),
                                    (np.array([1, 1, 1, 1, 1, 1], np.uint32), nb, 0, jc.JC_ERR_ARG),
                                    (np.array([0, 1, 2, 3, 3, 3], np.uint32), np.array([1, 0, 9], np.uint32), 3,
                                     jc.JC_ERR_ARG),
                                    (np.array([0, 1, 2, 3, 3, 3], np.uint32), nb, 4, jc.JC_ERR_ARG)]:
            rc = L.jc_batch_add_graph(b._h, 5, jc._p(off, jc._u32p), jc._p(nbr, jc._u32p), nnz,
                                      jc._p(pos, jc._f32p), None)
            assert rc == want
            assert L.jc_batch_last_error(b._h)
        assert L.jc_batch_add_graph(b._h, 0, None, None, 0, None, None) == jc.JC_ERR_ARG
        assert L.jc_batch_add_graph(b._h, 5, jc._p(np.array([0, 1, 2, 3, 3, 3], np.uint32), jc._u32p),
                                    jc._p(nb, jc._u32p), 3, None, None) == jc.JC_ERR_ARG  # no positions
        assert len(b) == 2  # rejected graphs are not added
        with pytest.raises(jc.JcError) as ei:
            b.positions(0)  # not bound
        assert ei.value.code == jc.JC_ERR_STATE


def test_builder_creation_errors(jc):
    L = jc.lib()
    h = jc._vp()
    assert L.jc_batch_create(b"sgd-stress", None, jc.ctypes.byref(h)) == jc.JC_ERR_UNKNOWN_ENGINE
    assert L.jc_batch_create(b"fa2-bh", b'{"theta": "wide"}', jc.ctypes.byref(h)) == jc.JC_ERR_PARAMS
    assert L.jc_batch_create(None, None, jc.ctypes.byref(h)) == jc.JC_ERR_ARG
    assert L.jc_batch_create(b"fa2-bh", None, None) == jc.JC_ERR_ARG
    assert L.jc_batch_graph_count(None) == 0
    assert L.jc_batch_engine(None) is None
    assert L.jc_batch_bind(None) == jc.JC_ERR_ARG
    L.jc_batch_destroy(None)
    with jc.Batch() as b:
        with pytest.raises(jc.JcError) as ei:
            b.bind()  # no graphs
        assert ei.value.code == jc.JC_ERR_STATE
        with pytest.raises(jc.JcError):
            b.run(1)
