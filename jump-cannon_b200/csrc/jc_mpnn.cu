// Learned warm start: the message-passing network and its tensor-core GEMMs.
// This file currently holds the GEMM launcher and its test entry point; the
// network (features, forward, backward, Adam, training) builds on them.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "jc_common.h"
#include "jc_tc_gemm.cuh"

namespace jc {
namespace mpnn {

inline uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// Launch C (op)= A * B on the tensor cores; `splits` > 1 splits K across CTAs
// (each writes its own f32 partial at C + z * c_split_stride).
inline void gemm(const tc::GemmArgs& g, int splits, int bn, cudaStream_t s) {
  dim3 grid(cdiv(g.M, tc::BM), cdiv(g.N, bn), std::max(splits, 1));
  if (bn == 256) {
    const int smem = tc::gemm_smem_bytes<256>();
    JC_CUDA_CHECK(cudaFuncSetAttribute(tc::k_tc_gemm<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    tc::k_tc_gemm<256><<<grid, 128, smem, s>>>(g);
  } else {
    const int smem = tc::gemm_smem_bytes<128>();
    JC_CUDA_CHECK(cudaFuncSetAttribute(tc::k_tc_gemm<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    tc::k_tc_gemm<128><<<grid, 128, smem, s>>>(g);
  }
  JC_CUDA_CHECK(cudaGetLastError());
}

}  // namespace mpnn
}  // namespace jc

// Test entry point: C = A * B from host bf16 bit patterns (A: M x K row-major
// if a_kmajor else K x M row-major; B: N x K row-major if b_kmajor else K x N
// row-major), f32 result in C (M x N row-major, summed over split-K parts).
extern "C" jc_status jc_tc_gemm_bf16(int32_t M, int32_t N, int32_t K, const uint16_t* a_bits, int32_t a_kmajor,
                                     const uint16_t* b_bits, int32_t b_kmajor, int32_t bn, int32_t splits,
                                     float* c_out) {
  using namespace jc;
  if (M <= 0 || N <= 0 || K <= 0 || !a_bits || !b_bits || !c_out || (bn != 128 && bn != 256) || splits < 1)
    return JC_ERR_ARG;
  try {
    __nv_bfloat16 *dA = nullptr, *dB = nullptr;
    float* dC = nullptr;
    uint32_t* dErr = nullptr;
    const size_t na = (size_t)M * K, nb = (size_t)N * K, nc = (size_t)M * N * splits;
    JC_CUDA_CHECK(cudaMalloc(&dA, na * 2));
    JC_CUDA_CHECK(cudaMalloc(&dB, nb * 2));
    JC_CUDA_CHECK(cudaMalloc(&dC, nc * 4));
    JC_CUDA_CHECK(cudaMalloc(&dErr, 4));
    JC_CUDA_CHECK(cudaMemcpy(dA, a_bits, na * 2, cudaMemcpyHostToDevice));
    JC_CUDA_CHECK(cudaMemcpy(dB, b_bits, nb * 2, cudaMemcpyHostToDevice));
    JC_CUDA_CHECK(cudaMemset(dErr, 0, 4));
    tc::GemmArgs g{};
    g.A0 = dA;
    g.A1 = dA;
    g.lda0 = g.lda1 = a_kmajor ? K : M;
    g.k_split = 1 << 30;
    g.a_kmajor = a_kmajor != 0;
    g.B = dB;
    g.ldb = b_kmajor ? K : N;
    g.b_kmajor = b_kmajor != 0;
    g.M = M;
    g.N = N;
    g.K = K;
    g.k_per_split = (int)(((K + splits - 1) / splits + tc::BK - 1) / tc::BK * tc::BK);
    g.C = dC;
    g.ldc = N;
    g.c_split_stride = (long long)M * N;
    g.epilogue = tc::EPI_STORE_F32;
    g.err = dErr;
    mpnn::gemm(g, splits, bn, 0);
    JC_CUDA_CHECK(cudaDeviceSynchronize());
    std::vector<float> parts(nc);
    uint32_t err = 0;
    JC_CUDA_CHECK(cudaMemcpy(parts.data(), dC, nc * 4, cudaMemcpyDeviceToHost));
    JC_CUDA_CHECK(cudaMemcpy(&err, dErr, 4, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < (size_t)M * N; ++i) {
      float acc = 0.0f;
      for (int z = 0; z < splits; ++z) acc += parts[(size_t)z * M * N + i];
      c_out[i] = acc;
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    cudaFree(dErr);
    return err ? (jc_status)err : JC_OK;
  } catch (const Error& e) {
    return e.code;
  }
}
