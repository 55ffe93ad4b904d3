// BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (tcgen05) for
// the message-passing network of the learned warm start.
//
//   C[M x N] (op)= sum_k A(m, k) * B(k, n)
//
// A is row-major M x K ("K-major") or its transpose (K x M row-major,
// "MN-major"); likewise B is N x K row-major (K-major) or K x N row-major
// (MN-major). Two kernels, one epilogue:
//
// * k_tc_gemm_tma (every GEMM of the network): operands staged by the tensor
//   memory accelerator into 128-byte-swizzled tiles, persistent CTAs of 8
//   warps, the next tile's loads in flight during the epilogue (the section
//   "TMA-staged variant" below).
// * k_tc_gemm (operands the TMA kernel does not take: row strides that are not
//   whole 16-byte units, A split over two bases): tiles staged by the threads
//   with 16-byte cp.async copies (all of a chunk's copies in flight at once)
//   into the canonical no-swizzle UMMA core-matrix layout that matches the
//   global layout:
//     K-major : element (r, k) at (r%8)*16 + (k%8)*2 + (r/8)*SBO + (k/8)*LBO
//     MN-major: element (r, k) at (k%8)*16 + (r%8)*2 + (r/8)*SBO + (k/8)*LBO
//   (LBO: byte stride of core matrices along K, SBO: along M/N; 128-byte core
//   matrices; descriptor fields as the PTX ISA's tcgen05 shared memory
//   descriptor, version 1). One CTA (4 warps) per 128 x BN tile, K in chunks
//   of 64 through two stages: while the tensor core works on one stage the
//   threads fill the other.
//
// In both, one elected thread issues the tcgen05.mma instructions (f32
// accumulator in tensor memory, BN = 128 or 256 columns allocated per CTA)
// and commits them to mbarriers. Every mbarrier wait is bounded: past the
// bound the kernel records an error, drains, frees its tensor memory and
// returns.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdint>

namespace jc {
namespace tc {

constexpr int BM = 128;
constexpr int BK = 64;
constexpr uint32_t WAIT_LIMIT = 1u << 24;

enum Epilogue : int {
  EPI_STORE_F32 = 0,       // C (+ z * c_split_stride) = acc (f32)
  EPI_BIAS_RELU_BF16 = 1,  // C = bf16(max(acc + bias[n], 0))
  EPI_STORE_BF16 = 3,      // C = bf16(acc)
};

struct GemmArgs {
  const __nv_bfloat16* A0;  // A columns k < k_split (or rows, for MN-major) come from A0 ...
  const __nv_bfloat16* A1;  // ... and k >= k_split from A1 (concatenation without a copy); may equal A0
  int lda0, lda1, k_split;
  bool a_kmajor;
  const __nv_bfloat16* B;
  int ldb;
  bool b_kmajor;
  int M, N, K;
  int k_per_split;          // split-K: CTA z covers [z * k_per_split, (z+1) * k_per_split)
  void* C;
  int ldc;
  long long c_split_stride; // elements between split-K partial outputs
  int epilogue;
  const float* bias;
  uint32_t* err;            // error word (bounded waits)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: f32 accumulate, bf16 A and B.
__host__ __device__ constexpr uint32_t make_idesc(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait; false when the bound was hit. One try_wait may itself block
// for a hardware-chosen time before it reports an incomplete phase, so the
// bound is kept in time as well as in polls: at most WAIT_NS of the global
// timer (checked every 64 polls) or WAIT_LIMIT polls, whichever comes first.
constexpr uint64_t WAIT_NS = 1000000000ull;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  uint64_t t0 = 0;
  for (uint32_t i = 0; i < WAIT_LIMIT; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i == 64) t0 = global_ns();
    if (i > 64) {
      __nanosleep(64);
      if ((i & 63u) == 0u && global_ns() - t0 > WAIT_NS) return false;
    }
  }
  return false;
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accum) {
  const uint32_t mask0 = 0u, mask1 = 0u, mask2 = 0u, mask3 = 0u;  // no output lanes disabled
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accum), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_ld8(uint32_t taddr, float* v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 16-byte asynchronous copy global -> shared (cp.async, L2 only): the copies
// of a whole chunk are in flight together instead of one load after another.
__device__ __forceinline__ void cp_async16(uint8_t* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Wait until at most 1 (0) of this thread's committed copy groups are in flight.
__device__ __forceinline__ void cp_async_wait_pending1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_pending0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Stage one (R x BK) operand chunk (R = rows of the tile: M or N side) into
// shared memory in the canonical layout. `kmajor`: the global source is
// contiguous along K. Rows >= rows_valid and k >= k_valid are zero. Whole
// aligned vectors go by cp.async (the caller commits them as one group and
// waits for it); zeros and ragged vectors are stored directly.
template <int R>
__device__ __forceinline__ void stage(uint8_t* sm, const __nv_bfloat16* src0, const __nv_bfloat16* src1, int ld0,
                                      int ld1, int k_split, bool kmajor, int row0, int rows_valid, int k0,
                                      int k_end) {
  // 16-byte vectors: R*BK/8 of them.
  constexpr int VECS = R * BK / 8;
  for (int v = threadIdx.x; v < VECS; v += blockDim.x) {
    int r, kk;
    uint32_t off;
    if (kmajor) {
      r = v / (BK / 8);                 // row of the tile
      kk = (v % (BK / 8)) * 8;          // first k of the vector
      // core (r/8, kk/8): LBO = 128 B along K, SBO = (BK/8)*128 B along rows
      off = (uint32_t)((r / 8) * (BK / 8) * 128 + (kk / 8) * 128 + (r % 8) * 16);
    } else {
      kk = v / (R / 8);                 // k row of the source
      r = (v % (R / 8)) * 8;            // first tile row of the vector
      // MN-major core (r/8, kk/8): SBO = 128 B along rows, LBO = (R/8)*128 B along K
      off = (uint32_t)((kk / 8) * (R / 8) * 128 + (r / 8) * 128 + (kk % 8) * 16);
    }
    uint4 val = make_uint4(0u, 0u, 0u, 0u);
    const int gk = k0 + kk;
    const int gr = row0 + r;
    if (kmajor) {
      if (gr < rows_valid && gk < k_end) {
        const __nv_bfloat16* src = gk < k_split ? src0 + (size_t)gr * ld0 + gk : src1 + (size_t)gr * ld1 + (gk - k_split);
        if (gk + 8 <= k_end && ((gk < k_split) == (gk + 7 < k_split)) && (((uintptr_t)src & 15u) == 0)) {
          cp_async16(sm + off, src);
          continue;
        } else {
          __align__(16) __nv_bfloat16 tmp[8];
          for (int e = 0; e < 8; ++e) {
            int kq = gk + e;
            tmp[e] = kq < k_end ? (kq < k_split ? src0[(size_t)gr * ld0 + kq] : src1[(size_t)gr * ld1 + (kq - k_split)])
                                : __float2bfloat16(0.0f);
          }
          val = *reinterpret_cast<uint4*>(tmp);
        }
      }
    } else {
      if (gk < k_end && gr < rows_valid) {
        const __nv_bfloat16* base = gk < k_split ? src0 + (size_t)gk * ld0 : src1 + (size_t)(gk - k_split) * ld1;
        if (gr + 8 <= rows_valid && (((uintptr_t)(base + gr) & 15u) == 0)) {
          cp_async16(sm + off, base + gr);
          continue;
        } else {
          __align__(16) __nv_bfloat16 tmp[8];
          for (int e = 0; e < 8; ++e) tmp[e] = gr + e < rows_valid ? base[gr + e] : __float2bfloat16(0.0f);
          val = *reinterpret_cast<uint4*>(tmp);
        }
      }
    }
    *reinterpret_cast<uint4*>(sm + off) = val;
  }
}

// 32 consecutive f32 columns of one TMEM lane per thread (warp-collective).
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Epilogue shared by both GEMM kernels. Warp w reads TMEM lanes
// 32 (w % 4) .. + 31 (= tile rows); with 8 warps, warps 4-7 take the second
// half of the tile's columns. Each thread loads 32 columns of its row per
// tcgen05.ld and writes them as whole 16-byte vectors when the tile lies
// inside C (per-element checks only on ragged tiles). The bias of a column
// group is read once per group as four 16-byte vectors when aligned.
template <int BN, int NWARPS>
__device__ __forceinline__ void tc_epilogue(const GemmArgs& g, uint32_t tmem, bool ok, int nk, int m0, int n0) {
  static_assert(NWARPS == 4 || NWARPS == 8, "4 or 8 warps");
  constexpr int COLS = BN / (NWARPS / 4);
  const int warp = threadIdx.x >> 5, quad = warp & 3;
  const int cbeg = (warp >> 2) * COLS;
  const int row = m0 + quad * 32 + (threadIdx.x & 31);
  const bool zero = !ok || nk == 0;
  const int epi = g.epilogue;
  const bool f32 = epi == EPI_STORE_F32;
  const int esize = f32 ? 4 : 2;
  const bool vec_ok = ((reinterpret_cast<uintptr_t>(g.C) & 15u) == 0) && (g.ldc % (16 / esize)) == 0 &&
                      (!f32 || (g.c_split_stride % 4) == 0);
  const bool bias_vec = epi != EPI_BIAS_RELU_BF16 || (reinterpret_cast<uintptr_t>(g.bias) & 15u) == 0;
#pragma unroll 1
  for (int c0 = cbeg; c0 < cbeg + COLS; c0 += 32) {
    float v[32];
    tc_ld32(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)c0, v);
    tc_wait_ld();
    if (zero) {
#pragma unroll
      for (int i = 0; i < 32; ++i) v[i] = 0.0f;
    }
    const int col = n0 + c0;
    if (row >= g.M || col >= g.N) continue;
    const bool full = col + 32 <= g.N && vec_ok;
    if (epi == EPI_BIAS_RELU_BF16) {
      if (full && bias_vec) {
        const float4* b4 = reinterpret_cast<const float4*>(g.bias + col);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float4 b = __ldg(b4 + q);
          v[4 * q] += b.x;
          v[4 * q + 1] += b.y;
          v[4 * q + 2] += b.z;
          v[4 * q + 3] += b.w;
        }
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = fmaxf(v[i], 0.0f);
      } else {
        for (int i = 0; i < 32; ++i) v[i] = col + i < g.N ? fmaxf(v[i] + g.bias[col + i], 0.0f) : 0.0f;
      }
    }
    if (f32) {
      float* C = reinterpret_cast<float*>(g.C) + (size_t)blockIdx.z * g.c_split_stride + (size_t)row * g.ldc + col;
      if (full) {
#pragma unroll
        for (int q = 0; q < 8; ++q)
          reinterpret_cast<float4*>(C)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      } else {
        for (int i = 0; i < 32; ++i)
          if (col + i < g.N) C[i] = v[i];
      }
    } else {
      __nv_bfloat16* C = reinterpret_cast<__nv_bfloat16*>(g.C) + (size_t)row * g.ldc + col;
      if (full) {
        uint32_t h[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const __nv_bfloat162 pr = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
          h[i] = *reinterpret_cast<const uint32_t*>(&pr);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
          reinterpret_cast<uint4*>(C)[q] = make_uint4(h[4 * q], h[4 * q + 1], h[4 * q + 2], h[4 * q + 3]);
      } else {
        for (int i = 0; i < 32; ++i)
          if (col + i < g.N) C[i] = __float2bfloat16_rn(v[i]);
      }
    }
  }
}

template <int BN>
__global__ void __launch_bounds__(128) k_tc_gemm(GemmArgs g) {
  constexpr int A_BYTES = BM * BK * 2;
  constexpr int B_BYTES = BN * BK * 2;
  constexpr int STAGE = A_BYTES + B_BYTES;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ uint32_t tmem_base_sh;
  const int warp = threadIdx.x >> 5;
  const int m0 = blockIdx.x * BM;
  const int n0 = blockIdx.y * BN;
  const int kz0 = blockIdx.z * g.k_per_split;
  const int kz1 = min(g.K, kz0 + g.k_per_split);
  const int nk = (kz1 - kz0 + BK - 1) / BK;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"((uint32_t)BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  const bool a_mn = !g.a_kmajor, b_mn = !g.b_kmajor;
  const uint32_t idesc = make_idesc(BM, BN, a_mn, b_mn);
  // descriptor strides (bytes) for the two layouts (see the file comment)
  const uint32_t a_lbo = g.a_kmajor ? 128u : (uint32_t)(BM / 8) * 128u;
  const uint32_t a_sbo = g.a_kmajor ? (uint32_t)(BK / 8) * 128u : 128u;
  const uint32_t b_lbo = g.b_kmajor ? 128u : (uint32_t)(BN / 8) * 128u;
  const uint32_t b_sbo = g.b_kmajor ? (uint32_t)(BK / 8) * 128u : 128u;
  // advance of one MMA (K = 16 = two core matrices along K)
  const uint32_t a_kstep = 2u * a_lbo;
  const uint32_t b_kstep = 2u * b_lbo;

  bool ok = true;
  uint32_t phase[2] = {0u, 0u};
  bool pending[2] = {false, false};
  // chunk c goes to stage c & 1; the copies of chunk c + 1 are issued before
  // the CTA waits for those of chunk c, so two chunks' copies are in flight
  auto issue = [&](int c) {
    uint8_t* sa = smem + (c & 1) * STAGE;
    const int k0 = kz0 + c * BK;
    stage<BM>(sa, g.A0, g.A1, g.lda0, g.lda1, g.k_split, g.a_kmajor, m0, g.M, k0, kz1);
    stage<BN>(sa + A_BYTES, g.B, g.B, g.ldb, g.ldb, 1 << 30, g.b_kmajor, n0, g.N, k0, kz1);
    cp_async_commit();
  };
  if (nk > 0) issue(0);
  for (int c = 0; c < nk; ++c) {
    const int s = c & 1;
    uint8_t* sa = smem + s * STAGE;
    uint8_t* sb = sa + A_BYTES;
    if (c + 1 < nk) {
      if (pending[s ^ 1]) {  // the MMAs of chunk c - 1 read the stage chunk c + 1 goes to
        if (!mbar_wait(&bars[s ^ 1], phase[s ^ 1])) ok = false;
        phase[s ^ 1] ^= 1u;
        pending[s ^ 1] = false;
      }
      issue(c + 1);
      cp_async_wait_pending1();  // chunk c's copies are done; chunk c + 1's may still be in flight
    } else {
      cp_async_wait_pending0();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0) {
      const uint32_t a_addr = smem_u32(sa), b_addr = smem_u32(sb);
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        const uint64_t da = make_desc(a_addr + kk * a_kstep, a_lbo, a_sbo);
        const uint64_t db = make_desc(b_addr + kk * b_kstep, b_lbo, b_sbo);
        tc_mma(tmem, da, db, idesc, (c > 0 || kk > 0) ? 1u : 0u);
      }
      tc_commit(&bars[s]);
    }
    pending[s] = true;
    __syncwarp();
  }
  for (int s = 0; s < 2; ++s) {
    if (pending[s]) {
      if (!mbar_wait(&bars[s], phase[s])) ok = false;
      phase[s] ^= 1u;
    }
  }
  tc_fence_after();
  if (!ok && threadIdx.x == 0) atomicCAS(g.err, 0u, 4u);

  tc_epilogue<BN, 4>(g, tmem, ok, nk, m0, n0);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN) : "memory");
  }
}

template <int BN>
constexpr int gemm_smem_bytes() {
  return 2 * (BM * BK * 2 + BN * BK * 2);
}

// ------------------------------------------------- TMA-staged variant --
// Each operand K-major (A: M x K rows, B: N x K rows) or MN-major (A: K x M
// rows, B: K x N rows); one base per operand (no A0/A1 split). Every K chunk
// of 64 is brought into shared memory by the tensor-memory accelerator
// (cp.async.bulk.tensor, no multicast, no cluster), the tensor maps built on
// the host with 128-byte swizzling, so each operand tile is a canonical
// SWIZZLE_128B UMMA layout of 1024-byte atoms (8 rows of 128 bytes):
//  K-major : one box of 64 K x rows; row r at 128 r; atoms of 8 rows 1024
//            bytes apart (stride offset); a k-step of 16 moves the start by
//            32 bytes.
//  MN-major: one box of 64 MN x 64 K per 64 rows of the tile; K row k at
//            128 k inside a box, so the 8-row K groups are 1024 bytes apart
//            (stride offset) and the 64-wide MN blocks 8192 bytes apart
//            (leading offset); a k-step of 16 moves the start by 2048 bytes.
// Rows past M or N and K past the operand read as zero. One
// thread issues the loads and the MMAs over a ring of S stages (2 for
// 256-wide tiles, 3 for 128-wide ones: two CTAs per SM either way, so one
// CTA's epilogue overlaps the other's loads; eight warps share the epilogue).
// The CTAs are persistent (two per SM, each looping over output tiles) and
// load the next tile's first stages while the current tile's epilogue runs:
// a full barrier per stage (the loads' transaction bytes) and an empty
// barrier per stage (the tcgen05.commit of the MMAs that read it). Every
// wait is bounded; after a failed wait the thread waits (bounded) for the
// loads it issued and for its last commit before the CTA frees its tensor
// memory and returns.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int c0, int c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}

// SWIZZLE_128B K-major descriptor: LBO unused (16 B), SBO 1024 B.
__device__ __forceinline__ uint64_t make_desc_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) | (1ull << 46) |
         (2ull << 61);
}

// SWIZZLE_128B MN-major descriptor: LBO 8192 B (64-wide MN blocks), SBO 1024 B
// (8-row K groups).
__device__ __forceinline__ uint64_t make_desc_sw128_mn(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(8192u >> 4) << 16) | ((uint64_t)(1024u >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}

// One operand's chunk: K-major, one box {64 K, R rows}; MN-major, R / 64
// boxes {64 MN, 64 K}, 8192 bytes apart.
template <int R, bool MN>
__device__ __forceinline__ void tma_operand(uint8_t* dst, const void* tmap, int k0, int row0, uint64_t* bar) {
  if (MN) {
#pragma unroll
    for (int h = 0; h < R / 64; ++h) tma_load_2d(dst + h * 8192, tmap, row0 + 64 * h, k0, bar);
  } else {
    tma_load_2d(dst, tmap, k0, row0, bar);
  }
}

template <bool MN>
__device__ __forceinline__ uint64_t operand_desc(uint32_t base, int kk) {
  return MN ? make_desc_sw128_mn(base + 2048u * (uint32_t)kk) : make_desc_sw128(base + 32u * (uint32_t)kk);
}

template <int BN>
__host__ __device__ constexpr int tma_stages() {
  return BN == 256 ? 2 : 3;
}

template <int BN>
__host__ __device__ constexpr int gemm_tma_smem_bytes() {
  return tma_stages<BN>() * (BM * BK * 2 + BN * BK * 2) + 1024;  // + alignment slack
}

constexpr int TMA_THREADS = 256;

template <int BN, bool A_MN, bool B_MN>
__global__ void __launch_bounds__(TMA_THREADS) k_tc_gemm_tma(const __grid_constant__ GemmArgs g,
                                                     const __grid_constant__ CUtensorMap tmap_a,
                                                     const __grid_constant__ CUtensorMap tmap_b) {
  constexpr int A_BYTES = BM * BK * 2;
  constexpr int B_BYTES = BN * BK * 2;
  constexpr int STAGE = A_BYTES + B_BYTES;
  constexpr int TMA_STAGES = tma_stages<BN>();
  extern __shared__ uint8_t smem_raw[];
  // SWIZZLE_128B tiles start on 1024-byte boundaries
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  __shared__ __align__(8) uint64_t full[TMA_STAGES], empty[TMA_STAGES];
  __shared__ uint32_t tmem_base_sh, ok_sh;
  const int warp = threadIdx.x >> 5;
  const int tiles_m = (g.M + BM - 1) / BM;
  const int n_tiles = tiles_m * ((g.N + BN - 1) / BN);
  const int kz0 = blockIdx.z * g.k_per_split;
  const int kz1 = min(g.K, kz0 + g.k_per_split);
  const int nk = (kz1 - kz0 + BK - 1) / BK;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"((uint32_t)BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    for (int q = 0; q < TMA_STAGES; ++q) {
      mbar_init(&full[q], 1);
      mbar_init(&empty[q], 1);
    }
    ok_sh = 1u;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  // Persistent: this CTA takes tiles blockIdx.x, + gridDim.x, ... (M fastest).
  // Chunks are numbered across the CTA's tiles (chunk G of the CTA sits in
  // stage G % S, its barriers in phase G / S), so the first stages of the
  // next tile are loaded while the epilogue of this one runs.
  // Thread 0's bookkeeping: loads issued, loads waited for, MMAs committed.
  uint32_t issued = 0, consumed = 0, committed = 0;
  const uint32_t idesc = make_idesc(BM, BN, A_MN, B_MN);
  auto load = [&](uint32_t G, int t, int c) {
    const int q = (int)(G % TMA_STAGES);
    uint8_t* sa = smem + q * STAGE;
    mbar_expect_tx(&full[q], (uint32_t)STAGE);
    tma_operand<BM, A_MN>(sa, &tmap_a, kz0 + c * BK, (t % tiles_m) * BM, &full[q]);
    tma_operand<BN, B_MN>(sa + A_BYTES, &tmap_b, kz0 + c * BK, (t / tiles_m) * BN, &full[q]);
    issued = G + 1;
  };
  if (threadIdx.x == 0 && nk > 0 && (int)blockIdx.x < n_tiles)
    for (int c = 0; c < min(nk, TMA_STAGES); ++c) load((uint32_t)c, (int)blockIdx.x, c);

  for (int t = blockIdx.x, done = 0; t < n_tiles; t += gridDim.x, ++done) {
    if (threadIdx.x == 0 && nk > 0) {
      const uint32_t G0 = (uint32_t)done * (uint32_t)nk;
      bool ok = true;
      for (int c = 0; c < nk; ++c) {
        const uint32_t G = G0 + (uint32_t)c;
        const int q = (int)(G % TMA_STAGES);
        if (!mbar_wait(&full[q], (G / TMA_STAGES) & 1u)) { ok = false; break; }
        consumed = G + 1;
        tc_fence_after();
        const uint32_t a_addr = smem_u32(smem + q * STAGE), b_addr = a_addr + (uint32_t)A_BYTES;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk)
          tc_mma(tmem, operand_desc<A_MN>(a_addr, kk), operand_desc<B_MN>(b_addr, kk), idesc,
                 (c > 0 || kk > 0) ? 1u : 0u);
        tc_commit(&empty[q]);
        committed = G + 1;
        if (c + TMA_STAGES < nk) {
          // the stage is refilled once the MMAs that read it are done
          if (!mbar_wait(&empty[q], (G / TMA_STAGES) & 1u)) { ok = false; break; }
          load(G + TMA_STAGES, t, c + TMA_STAGES);
        }
      }
      if (ok) {
        // commits complete in order: the last one covers every MMA of the tile
        const uint32_t G = G0 + (uint32_t)nk - 1u;
        if (!mbar_wait(&empty[G % TMA_STAGES], (G / TMA_STAGES) & 1u)) ok = false;
      }
      if (ok) {
        // every stage is free: the next tile's first chunks go in now
        const int tn = t + (int)gridDim.x;
        if (tn < n_tiles)
          for (int c = 0; c < min(nk, TMA_STAGES); ++c) load(G0 + (uint32_t)nk + (uint32_t)c, tn, c);
      } else {
        // drain: the loads still in flight and the MMAs already committed
        for (uint32_t G = consumed; G < issued; ++G) (void)mbar_wait(&full[G % TMA_STAGES], (G / TMA_STAGES) & 1u);
        if (committed > 0) {
          const uint32_t G = committed - 1u;
          (void)mbar_wait(&empty[G % TMA_STAGES], (G / TMA_STAGES) & 1u);
        }
        ok_sh = 0u;
        atomicCAS(g.err, 0u, 4u);
      }
    }
    __syncthreads();
    tc_fence_after();
    const bool ok = ok_sh != 0u;
    tc_epilogue<BN, TMA_THREADS / 32>(g, tmem, ok, nk, (t % tiles_m) * BM, (t / tiles_m) * BN);
    tc_fence_before();
    __syncthreads();  // the accumulator is read out: the next tile's MMAs may overwrite it
    if (!ok) break;
  }
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN) : "memory");
  }
}

}  // namespace tc
}  // namespace jc
