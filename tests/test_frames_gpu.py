"""Position frames streamed from the engines on the GPU (jc_engine_stream_*).

An f32 frame must carry exactly the positions that jc_engine_step returns
for the same steps (the reference's PositionDelta payload, raw LE f32 x,y,z,
crates/graph-compute/proto/compute.proto:84-91); a binary16 delta frame must
be exactly what the oracle encoder makes of those positions, and the host
decoder must reproduce the encoder's reconstruction bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def fa2(jc, g, x, **params):
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": 0.8, **params})
    e.init(g, x)
    return e


def twin_positions(jc, g, x, iters_per_frame, frames, engine="fa2-bh", **params):
    e = jc.LayoutEngine(engine)
    e.set_params({"theta": 0.8, **params} if engine.startswith("fa2") else params)
    e.init(g, x)
    out = []
    for _ in range(frames):
        e.step_many(iters_per_frame, readback=False)
        out.append(e.positions())
    e.close()
    return out


@pytest.mark.parametrize("depth,iters", [(1, 1), (2, 1), (3, 4)])
def test_f32_frames_are_the_step_positions(jc, depth, iters):
    g = jc.gen_scale_free(3000, 3, 21)
    x = jc.seed_uniform(g.n_nodes, 3, 22)
    want = twin_positions(jc, g, x, iters, 12)
    e = fa2(jc, g, x)
    e.stream_open("f32", depth=depth)
    got = []
    for t in range(12):
        if t >= depth:
            got.append(e.stream_next())
        e.stream_step(iters)
    while len(got) < 12:
        got.append(e.stream_next())
    for t, f in enumerate(got):
        assert f.frame == t and f.encoding == "f32" and f.n_nodes == g.n_nodes
        assert len(f.data) == 64 + 12 * g.n_nodes
        assert np.array_equal(f.payload, want[t])
    # the engine's own read-out agrees with the last frame
    assert np.array_equal(e.positions(), want[-1])
    e.close()


def test_f16_frames_match_the_oracle_encoder(jc, orc):
    g = jc.gen_watts_strogatz(5000, 6, 0.1, 31)
    x = jc.seed_uniform(g.n_nodes, 3, 32)
    want = twin_positions(jc, g, x, 1, 40)
    e = fa2(jc, g, x)
    e.stream_open("f16", depth=2, keyframe_interval=16)
    enc = orc.FrameEncoder(g.n_nodes)
    dec = jc.FrameDecoder(g.n_nodes)
    e.stream_step()
    for t in range(40):
        if t + 1 < 40:
            e.stream_step()
        f = e.stream_next()
        if t % 16 == 0:
            enc.started = False  # keyframe: the oracle restarts from f32
        kind, payload = enc.encode(want[t])
        assert f.frame == t and f.encoding == kind
        assert np.array_equal(f.payload, payload)
        assert len(f.data) == 64 + (12 if kind == "f32" else 6) * g.n_nodes
        got = dec.decode(f)
        assert np.array_equal(got, enc.rec)
        assert np.max(np.abs(got - want[t])) <= 1e-2
    e.close()


def test_f16_frame_turns_f32_when_a_difference_overflows(jc, orc):
    """Positions 1e10 apart with no displacement cap move by more than
    65504 in one step; that frame goes out as f32 and decoding stays exact."""
    g = jc.gen_path(64)
    x = (jc.seed_uniform(g.n_nodes, 3, 41) * np.float32(1e10)).astype(np.float32)
    want = twin_positions(jc, g, x, 1, 6, max_displacement=0.0)
    e = fa2(jc, g, x, max_displacement=0.0)
    e.stream_open("f16", depth=1)
    enc = orc.FrameEncoder(g.n_nodes)
    dec = jc.FrameDecoder(g.n_nodes)
    kinds = []
    for t in range(6):
        e.stream_step()
        f = e.stream_next()
        kind, payload = enc.encode(want[t])
        kinds.append(f.encoding)
        assert f.encoding == kind and np.array_equal(f.payload, payload)
        assert np.array_equal(dec.decode(f), enc.rec)
    assert "f32" in kinds[1:]
    e.close()


def test_stream_from_the_sgd_and_batch_engines(jc):
    g = jc.gen_grid(40, 30)
    x = jc.seed_uniform(g.n_nodes, 2, 51)
    for eid in ("sgd-stress-gpu", "sgd-stress"):
        params = {"n_pivots": 20}
        want = twin_positions(jc, g, x, 2, 5, engine=eid, **params)
        e = jc.LayoutEngine(eid)
        e.set_params(params)
        e.init(g, x)
        e.stream_open("f32", depth=2)
        got = []
        for t in range(5):
            e.stream_step(2)
            if t >= 1:
                got.append(e.stream_next())
        got.append(e.stream_next())
        for t, f in enumerate(got):
            assert np.array_equal(f.payload, want[t]), (eid, t)
        e.close()
    graphs, seeds = jc.gen_batch_graphs(20, seed=5, lo=50, hi=400)
    a = jc.LayoutEngine("fa2-bh")
    a.init_batch(graphs, seeds)
    a.step_many(3, readback=False)
    want = a.positions()
    b = jc.LayoutEngine("fa2-bh")
    b.init_batch(graphs, seeds)
    b.stream_open("f32", depth=1)
    b.stream_step(3)
    assert np.array_equal(b.stream_next().payload, want)
    a.close()
    b.close()


def test_stream_misuse_is_reported(jc):
    g = jc.gen_path(100)
    e = fa2(jc, g, jc.seed_uniform(100, 3, 1))
    with pytest.raises(jc.JcError):
        e.stream_open("f32", depth=0)
    e.stream_open("f32", depth=2)
    with pytest.raises(jc.JcError) as err:
        e.stream_next()
    assert err.value.code == jc.JC_ERR_STATE
    e.stream_step()
    e.stream_step()
    with pytest.raises(jc.JcError) as err:
        e.stream_step()  # both slots pending
    assert err.value.code == jc.JC_ERR_STATE
    assert e.stream_next().frame == 0
    # a plain step between frames is allowed and shows in the next frame
    e.step_many(1, readback=False)
    assert e.stream_next().frame == 1
    e.stream_step()
    f = e.stream_next()
    assert np.array_equal(f.payload, e.positions())
    # re-initializing closes the stream
    e.init(g, jc.seed_uniform(100, 3, 2))
    with pytest.raises(jc.JcError):
        e.stream_step()
    e.close()
