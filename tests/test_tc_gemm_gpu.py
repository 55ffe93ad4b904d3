"""The tcgen05 BF16 GEMM (jc_tc_gemm.cuh) against an FP32 reference of the
same op on bf16-rounded inputs: K-major and MN-major operands, ragged M, N
and K, 128- and 256-wide tiles, split-K. Tolerance: FP32 accumulation order
differs, so 1e-3 relative to the row scale."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run_case(jc, M, N, K, a_kmajor, b_kmajor, bn, splits, seed, staging="auto"):
    rng = np.random.default_rng(seed)
    a = jc.from_bf16_bits(jc.to_bf16_bits(rng.standard_normal((M, K)).astype(np.float32)))
    b = jc.from_bf16_bits(jc.to_bf16_bits(rng.standard_normal((K, N)).astype(np.float32)))
    a_src = a if a_kmajor else a.T                # K-major: M x K rows; MN-major: K x M rows
    b_src = b.T if b_kmajor else b                # K-major: N x K rows; MN-major: K x N rows
    c = jc.tc_gemm_bf16(jc.to_bf16_bits(a_src), jc.to_bf16_bits(b_src), M, N, K, a_kmajor, b_kmajor, bn, splits,
                        staging)
    ref = a.astype(np.float64) @ b.astype(np.float64)
    scale = np.sqrt(K) + 1.0
    err = np.max(np.abs(c - ref)) / scale
    assert err < 1e-3, err


@pytest.mark.parametrize("M,N,K,ak,bk,bn,splits", [
    (128, 128, 64, True, True, 128, 1),
    (128, 128, 256, True, True, 128, 1),
    (300, 128, 256, True, True, 128, 1),
    (256, 256, 192, True, True, 256, 1),
    (200, 100, 100, True, True, 128, 1),
    (256, 128, 512, False, True, 128, 1),
    (128, 128, 128, True, False, 128, 1),
    (256, 128, 1000, False, False, 128, 4),
])
def test_tc_gemm_matches_fp32_reference(jc, M, N, K, ak, bk, bn, splits):
    run_case(jc, M, N, K, ak, bk, bn, splits, seed=M * 7 + N * 3 + K, staging="cp.async")
    run_case(jc, M, N, K, ak, bk, bn, splits, seed=M * 7 + N * 3 + K)


# The TMA-staged kernel (128-byte swizzled tiles, persistent CTAs), every
# operand major-ness: one and several 64-wide chunks, a ragged last chunk
# (zero fill past K), ragged M and N, rings that wrap (16 chunks through 2 or
# 3 stages), split-K, and CTAs that run several tiles (the next tile's loads
# in flight during the epilogue). MN-major operands arrive as 64 x 64 boxes.
TMA_SHAPES = [
    (128, 128, 64, 128, 1),
    (128, 128, 256, 128, 1),
    (296, 128, 256, 128, 1),
    (256, 256, 192, 256, 1),
    (200, 200, 96, 256, 1),
    (136, 72, 40, 128, 1),
    (384, 128, 1024, 128, 1),
    (256, 256, 1024, 256, 1),
    (256, 128, 1000, 128, 4),
    (1000, 256, 128, 256, 1),
    (40000, 128, 320, 128, 1),   # more tiles than resident CTAs: each CTA loops over tiles
    (40000, 256, 192, 256, 1),
    (40000, 200, 136, 128, 2),
]


@pytest.mark.parametrize("M,N,K,bn,splits", TMA_SHAPES)
@pytest.mark.parametrize("ak,bk", [(True, True), (False, True), (True, False), (False, False)])
def test_tc_gemm_tma_matches_fp32_reference(jc, M, N, K, bn, splits, ak, bk):
    run_case(jc, M, N, K, ak, bk, bn, splits, seed=M * 5 + N * 11 + K, staging="tma")


def test_tc_gemm_weight_gradient_shape_through_tma(jc):
    """The weight-gradient shape of the warm-start network: A = activations
    read transposed (MN-major, M = 64 or 256 layer inputs), B = dZ (MN-major,
    N = 128), K = node rows split across CTAs."""
    for M in (64, 256):
        run_case(jc, M, 128, 30000, False, False, 128, 12, seed=M, staging="tma")


def test_tc_gemm_tma_refuses_unaligned_rows(jc):
    a = jc.to_bf16_bits(np.ones((128, 100), np.float32))   # K-major A with a 200-byte row stride
    b = jc.to_bf16_bits(np.ones((128, 100), np.float32))
    with pytest.raises(jc.JcError):
        jc.tc_gemm_bf16(a, b, 128, 128, 100, True, True, 128, 1, "tma")
