"""Position frames on the CPU: the oracle's binary16 conversion against
numpy's, the delta encoder's properties, and the library's host decoder
(jc_frame_decode) against the oracle encoder. f32 frames carry the
reference's PositionDelta payload, raw LE f32 x,y,z
(crates/graph-compute/proto/compute.proto:84-91)."""
import numpy as np
import pytest


def test_f16_conversion_matches_numpy(orc):
    rng = np.random.default_rng(1)
    # random bit patterns over every exponent, plus the edges of the binary16 range
    bits = rng.integers(0, 2 ** 32, 400_000, dtype=np.uint64).astype(np.uint32)
    x = bits.view(np.float32)
    x = x[np.isfinite(x)]
    edges = np.array([0.0, -0.0, 65504.0, 65519.996, 65520.0, 65536.0, 6.1035156e-05, 6.0975552e-05,
                      5.9604645e-08, 2.9802322e-08, 2.9802326e-08, 4.4703484e-08, 1e-10, -1e-10, 1.0, -1.0,
                      1.00048828125, 1.0009765625, 2049.0, 2051.0, np.inf, -np.inf], np.float32)
    fine = (rng.standard_normal(200_000) * rng.choice([1e-6, 1e-3, 1.0, 1e3], 200_000)).astype(np.float32)
    for v in (x, edges, fine):
        with np.errstate(over="ignore"):
            want = v.astype(np.float16).view(np.uint16)
        assert np.array_equal(orc.f32_to_f16_bits(v), want)


def test_f16_to_f32_is_exact(orc):
    h = np.arange(0, 2 ** 16, dtype=np.uint32)
    h = h[(h & 0x7C00) != 0x7C00]  # finite values
    want = h.astype(np.uint16).view(np.float16).astype(np.float32)
    got = np.array([orc.lib().orc_f16_to_f32(int(b)) for b in h[::7]], np.float32)
    assert np.array_equal(got, want[::7])


def walk(n, frames, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    x = (rng.uniform(-100, 100, 3 * n)).astype(np.float32)
    out = [x.copy()]
    for _ in range(frames - 1):
        x = (x + rng.standard_normal(3 * n).astype(np.float32) * np.float32(scale)).astype(np.float32)
        out.append(x.copy())
    return out


def test_decoder_tracks_the_encoder_bit_for_bit(jc, orc):
    n = 500
    enc = orc.FrameEncoder(n)
    dec = jc.FrameDecoder(n)
    worst = 0.0
    for t, x in enumerate(walk(n, 300, 2, 0.5)):
        kind, payload = enc.encode(x)
        assert kind == ("f32" if t == 0 else "f16")
        got = dec.decode(jc.frame_message(t, n, kind, payload))
        assert np.array_equal(got, enc.rec)
        worst = max(worst, float(np.max(np.abs(got - x))))
    # error = rounding of one difference (|d| ~ 0.5..4): half a binary16 ulp of it
    assert worst <= 2.0 ** -11 * 8


def test_reconstruction_error_does_not_accumulate(orc):
    """Per frame the error is the latest difference's binary16 rounding plus
    the f32 rounding of r + h, whatever the number of frames before it."""
    n = 200
    enc = orc.FrameEncoder(n)
    for x in walk(n, 2000, 3, 0.01):
        prev = enc.rec.copy()
        kind, payload = enc.encode(x)
        if kind == "f16":
            d = np.abs(x.astype(np.float64) - prev)
            bound = d * 2.0 ** -11 + 2.0 ** -25 + np.abs(x.astype(np.float64)) * 2.0 ** -24
            assert np.all(np.abs(enc.rec.astype(np.float64) - x) <= bound * 1.01)


def test_out_of_range_difference_makes_an_f32_frame(jc, orc):
    n = 10
    enc = orc.FrameEncoder(n)
    dec = jc.FrameDecoder(n)
    x0 = np.zeros(3 * n, np.float32)
    x1 = x0.copy()
    x1[7] = 70000.0
    x2 = x1 + np.float32(0.25)
    kinds = []
    for t, x in enumerate((x0, x1, x2)):
        kind, payload = enc.encode(x)
        kinds.append(kind)
        assert np.array_equal(dec.decode(jc.frame_message(t, n, kind, payload)), x)
    assert kinds == ["f32", "f32", "f16"]


def test_decoder_rejects_bad_streams(jc):
    n = 4
    dec = jc.FrameDecoder(n)
    delta = jc.frame_message(1, n, "f16", np.zeros(3 * n, np.uint16))
    with pytest.raises(jc.JcError) as e:
        dec.decode(delta)
    assert e.value.code == jc.JC_ERR_STATE
    dec.decode(jc.frame_message(0, n, "f32", np.ones(3 * n, np.float32)))
    with pytest.raises(jc.JcError) as e:  # frame 2 after frame 0
        dec.decode(jc.frame_message(2, n, "f16", np.zeros(3 * n, np.uint16)))
    assert e.value.code == jc.JC_ERR_STATE
    with pytest.raises(jc.JcError):  # wrong node count
        dec.decode(jc.frame_message(1, n + 1, "f16", np.zeros(3 * (n + 1), np.uint16)))
    bad = bytearray(delta)
    bad[0] ^= 0xFF
    with pytest.raises(jc.JcError):
        dec.decode(bytes(bad))
    with pytest.raises(jc.JcError):
        dec.decode(delta[:-2])
    with pytest.raises(jc.JcError):
        dec.decode(b"short")
    # the failed calls left the reconstruction alone
    assert np.array_equal(dec.decode(delta), np.ones(3 * n, np.float32))


def test_f32_frame_payload_is_the_position_delta_bytes(jc):
    x = np.arange(12, dtype=np.float32) * np.float32(0.5)
    msg = jc.frame_message(9, 4, "f32", x)
    assert len(msg) == 64 + 48
    assert msg[64:] == x.astype("<f4").tobytes()
    f = jc.Frame(9, 4, "f32", msg)
    assert np.array_equal(f.payload, x)


def test_stream_calls_need_an_initialized_engine(jc):
    with jc.LayoutEngine("fa2-bh") as e:
        with pytest.raises(jc.JcError) as err:
            e.stream_step()
        assert err.value.code == jc.JC_ERR_STATE
        with pytest.raises(jc.JcError):
            e.stream_open("f16")
