// Learned warm start: a message-passing network that maps cheap node features
// to initial coordinates, trained on the GPU with a stress loss against
// layouts that plain ForceAtlas2 produced, plus the pivot-stress /
// edge-length evaluator that judges warm-started and plain layouts alike.
//
// The reference has no learned component. The quality measures restate
// crates/graph-layouts/src/metrics.rs:31-76 (scale-normalized stress with the
// closed-form scale, w = 1/d^2) and :150-164 (edge-length coefficient of
// variation); the hand-off goes to the plain engines unchanged.
//
// Network (node rows are local to a batch of whole graphs):
//   X     25 features per node in 32 bf16 columns (7 zero): log(1 + deg); the
//         return probabilities p_t(i -> i), t = 1..16, of 32 seeded random
//         walks per node (one per lane of a warp, counted by ballot); 8
//         Irwin-Hall random projections low-pass filtered by the lazy walk
//         P x = (x + D^-1 A x) / 2 (`cheb_steps` steps of a Chebyshev
//         recurrence, then `smooth_steps` plain steps; see compute_features),
//         each column kept at zero degree-weighted mean and unit mean square
//         per graph: what survives the filter are the graph's slowest
//         diffusion modes, a spectral-like global frame the network can place
//         nodes in.
//   A_0 = [X | mean_nbr X]                                  n x 64
//   H_1 = ReLU(A_0 W_0 + b_0)                               n x 128
//   A_l = [H_l | mean_nbr H_l], H_l+1 = ReLU(A_l W_l + b_l), l = 1, 2
//   Y   = H_3 W_h + b_h                                     n x dim (2 or 3)
// The layer GEMMs, their weight gradients (split-K over nodes) and the
// activation gradients run on the tcgen05 tensor cores (bf16 operands, f32
// accumulation). Activations and activation gradients are stored bf16;
// biases, the head's accumulation and the optimiser state are f32.
//
// Loss, per graph g of a batch: the scale-normalized stress between the
// prediction and the target layout over the pairs P_g = every CSR entry plus
// `partners` random same-graph nodes per node:
//   q = |Y_i - Y_j| / |T_i - T_j|,  alpha_g = sum q / sum q^2,
//   L_g = (1/|P_g|) sum (alpha_g q - 1)^2 = 1 - (sum q)^2 / (|P_g| sum q^2),
// averaged over the batch's graphs. alpha_g is the minimiser, so its
// derivative drops out. A pair's gradient goes to its first node only: edges
// appear from both ends, so every node gathers its own gradient and no float
// atomics are needed (for the partner pairs this is a semi-gradient).
//
// Every sum has a fixed order, so training is bitwise reproducible. Mean
// aggregations sum a row in CSR order, or, for rows longer than HUB_DEG, in
// eight contiguous segments added in order; the CPU oracle restates that order.
//
// Hand-off scale: ForceAtlas2 is not scale-free, so each predicted graph is
// centred and scaled by the s that balances the virial of its forces,
//   s^2 sum_edges r^2 + s * gravity * sum deg_i |y_i| = k_r/2 (sum deg sum m - sum deg m),
// (attraction, gravity and repulsion of fa2_barnes_hut.wgsl:114-197 with
// mass m = deg + 1), the equilibrium the plain iteration would settle into.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "jc_common.h"
#include "jc_engine.h"
#include "jc_params.h"
#include "jc_tc_gemm.cuh"

namespace jc {
namespace mpnn {

typedef __nv_bfloat16 bf16;

constexpr int FEAT = 32;        // input columns (25 features + zero padding)
constexpr int NFEAT = 25;
constexpr int HID = 128;
constexpr int WALKS = 32;       // random walks per node: one per lane
constexpr int WALK_LEN = 16;
constexpr int NPROJ = 8;
constexpr uint32_t RECENTER = 8;  // smoothing steps between re-centrings
constexpr uint32_t HUB_DEG = 1024;  // longer rows are summed in HUB_SEGS segments by a block
constexpr int HUB_SEGS = 8;
constexpr uint32_t ITEM_NODES = 4096;  // nodes per reduction item
constexpr int HEAD_W = HID * 4 + 4;    // head weight (128 x 4) + bias (4) gradient row
constexpr uint32_t NO_PIVOT = 0xFFFFFFFFu;
constexpr uint16_t NO_DIST = 0xFFFFu;

constexpr uint64_t SALT_WALK = 0x57A1C0FFEE000001ull;
constexpr uint64_t SALT_PROJ = 0x9B0C5EED00000002ull;
constexpr uint64_t SALT_PAIR = 0x7A1B2C3D00000003ull;
constexpr uint64_t SALT_INIT = 0x1D1E2F3000000004ull;
constexpr uint64_t SALT_ORDER = 0x0DDBA11000000005ull;

inline uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// Flat parameter vector: f32 master copy and a bf16 shadow at the same offsets.
struct ParamLayout {
  size_t w[3], b[3], wh, bh, total;
  int kin[3];
};

inline ParamLayout param_layout() {
  ParamLayout L{};
  const int kin[3] = {2 * FEAT, 2 * HID, 2 * HID};
  size_t o = 0;
  for (int l = 0; l < 3; ++l) {
    L.kin[l] = kin[l];
    L.w[l] = o;
    o += (size_t)kin[l] * HID;
    L.b[l] = o;
    o += HID;
  }
  L.wh = o;
  o += (size_t)HID * 4;
  L.bh = o;
  o += 4;
  L.total = (o + 7) & ~(size_t)7;
  return L;
}

// ------------------------------------------------------------ hashing --
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t hash4(uint64_t s, uint64_t a, uint64_t b, uint64_t c) {
  return mix64(mix64(mix64(s ^ a) ^ b) ^ c);
}

// Uniform integer in [0, n) from the high 32 bits (multiply-shift).
__host__ __device__ __forceinline__ uint32_t pick(uint64_t h, uint32_t n) {
  return (uint32_t)(((h >> 32) * (uint64_t)n) >> 32);
}

// Approximately standard normal: four uniforms on the midpoints of 4096 bins
// (Irwin-Hall, mean 2, variance 1/3), centred and scaled. The sum and the
// power-of-two scaling are exact in f32; only the final product rounds.
__device__ __forceinline__ float irwin4(uint64_t h) {
  const uint32_t s = (uint32_t)((h >> 52) & 0xFFF) + (uint32_t)((h >> 40) & 0xFFF) +
                     (uint32_t)((h >> 28) & 0xFFF) + (uint32_t)((h >> 16) & 0xFFF);
  const float u = (float)(2u * s + 4u) * (1.0f / 8192.0f);
  return __fmul_rn(__fsub_rn(u, 2.0f), 1.7320508075688772f);
}

// ------------------------------------------------------------- bf16 --
__device__ __forceinline__ float bf2f(bf16 x) { return __bfloat162float(x); }

__device__ __forceinline__ void unpack4(uint2 q, float* f) {
  f[0] = __uint_as_float(q.x << 16);
  f[1] = __uint_as_float(q.x & 0xFFFF0000u);
  f[2] = __uint_as_float(q.y << 16);
  f[3] = __uint_as_float(q.y & 0xFFFF0000u);
}

__device__ __forceinline__ uint2 pack4(const float* f) {
  const uint32_t a = __bfloat16_as_ushort(__float2bfloat16_rn(f[0]));
  const uint32_t b = __bfloat16_as_ushort(__float2bfloat16_rn(f[1]));
  const uint32_t c = __bfloat16_as_ushort(__float2bfloat16_rn(f[2]));
  const uint32_t d = __bfloat16_as_ushort(__float2bfloat16_rn(f[3]));
  return make_uint2(a | (b << 16), c | (d << 16));
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

__device__ __forceinline__ float warp_sumf(float x) {
#pragma unroll
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// A batch of whole graphs inside a graph set (global CSR, global node ids).
struct GView {
  const uint32_t* off;
  const uint32_t* nbr;
  const uint32_t* deg;
  const uint32_t* gid;  // node -> graph
  const uint32_t* go;   // graph -> first node (G + 1 entries)
  uint32_t n0, nb;      // nodes [n0, n0 + nb)
  uint32_t g0;          // first graph
};

// ========================================================== features ==
// One warp per node. Lane w walks WALK_LEN steps from i; a ballot counts the
// walks that are back at i after each step. Isolated nodes stay put.
__global__ void __launch_bounds__(256) k_features(GView v, uint64_t seed, bf16* __restrict__ X,
                                                  float* __restrict__ P) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= v.nb) return;
  const uint32_t i = v.n0 + w, deg = v.deg[i];
  bf16* x = X + (size_t)i * FEAT;
  uint32_t cur = i;
  for (int t = 1; t <= WALK_LEN; ++t) {
    const uint32_t d = v.deg[cur];
    if (d) cur = v.nbr[v.off[cur] + pick(hash4(seed ^ SALT_WALK, i, lane, (uint64_t)t), d)];
    const uint32_t back = __popc(__ballot_sync(0xffffffffu, cur == i));
    if (lane == 0) x[t] = __float2bfloat16_rn((float)back * (1.0f / WALKS));
  }
  if (lane == 0) x[0] = __float2bfloat16_rn(log1pf((float)deg));
  if (lane >= NFEAT) x[lane] = __float2bfloat16_rn(0.0f);
  if (lane < NPROJ) P[(size_t)i * NPROJ + lane] = irwin4(hash4(seed ^ SALT_PROJ, i, lane, 0));
}

// A neighbour's 8 projection columns: one 32-byte row, fetched as one
// 256-bit load (one L1 request instead of two; the rows are 32-byte aligned).
__device__ __forceinline__ void load_row8(const float* p, float4& q0, float4& q1) {
  uint32_t r0, r1, r2, r3, r4, r5, r6, r7;
  asm("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5), "=r"(r6), "=r"(r7)
      : "l"(p));
  q0 = make_float4(__uint_as_float(r0), __uint_as_float(r1), __uint_as_float(r2), __uint_as_float(r3));
  q1 = make_float4(__uint_as_float(r4), __uint_as_float(r5), __uint_as_float(r6), __uint_as_float(r7));
}

// One lazy random-walk step x <- (x + D^-1 A x) / 2 over the projection
// columns: one thread per node, each neighbour's 8 columns fetched as one
// 32-byte row, sums in CSR order. (The lazy step has no
// eigenvalue -1, so bipartite graphs such as grids do not oscillate.)
// The output of one filter step from P x (px) and the node's own columns:
// MODE 0, a lazy step: px; MODE 1, the first Chebyshev step: c1 px - x;
// MODE 2, a Chebyshev step: (c1 px - 2 x) - x_prev (see compute_features).
template <int MODE>
__device__ __forceinline__ float filter_out(float px, float x, float xp, float c1) {
  if (MODE == 0) return px;
  if (MODE == 1) return __fsub_rn(__fmul_rn(c1, px), x);
  return __fsub_rn(__fsub_rn(__fmul_rn(c1, px), __fmul_rn(2.0f, x)), xp);
}

// Bounded to 40 registers (six blocks per SM, no spills): the gathers are
// latency-bound, so more resident warps keep more rows in flight (128 filter
// steps over 13.4 M nodes 131.8 -> 127.8 ms, with the node's own row read
// after the sum).
template <int MODE>
__global__ void __launch_bounds__(256, 6) k_smooth(GView v, const float* __restrict__ pin, float* __restrict__ pout,
                                                const float* __restrict__ pprev, float c1) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= v.nb) return;
  const uint32_t i = v.n0 + w, d = v.deg[i];
  if (d > HUB_DEG) return;
  const float4* src = reinterpret_cast<const float4*>(pin);
  float4* dst = reinterpret_cast<float4*>(pout);
  // the node's own row and the previous iterate are read after the neighbour
  // sum (they only enter the output), so they hold no registers in its loop
  auto own = [&](float* xs, float* xp) {
    const float4 x0 = src[2 * (size_t)i], x1 = src[2 * (size_t)i + 1];
    xs[0] = x0.x; xs[1] = x0.y; xs[2] = x0.z; xs[3] = x0.w;
    xs[4] = x1.x; xs[5] = x1.y; xs[6] = x1.z; xs[7] = x1.w;
#pragma unroll
    for (int c = 0; c < 8; ++c) xp[c] = 0.0f;
    if (MODE == 2) {
      const float4 p0 = reinterpret_cast<const float4*>(pprev)[2 * (size_t)i];
      const float4 p1 = reinterpret_cast<const float4*>(pprev)[2 * (size_t)i + 1];
      xp[0] = p0.x; xp[1] = p0.y; xp[2] = p0.z; xp[3] = p0.w;
      xp[4] = p1.x; xp[5] = p1.y; xp[6] = p1.z; xp[7] = p1.w;
    }
  };
  float xs[8], xp[8];
  if (d == 0) {  // P x = x
    own(xs, xp);
    float o[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) o[c] = filter_out<MODE>(xs[c], xs[c], xp[c], c1);
    dst[2 * (size_t)i] = make_float4(o[0], o[1], o[2], o[3]);
    dst[2 * (size_t)i + 1] = make_float4(o[4], o[5], o[6], o[7]);
    return;
  }
  const uint32_t* row = v.nbr + v.off[i];
  float a[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  uint32_t e = 0;
  // ids up to a 16-byte boundary one row at a time, then four ids per vector
  // load and four rows in flight, summed in CSR order
  for (; e < d && (reinterpret_cast<uintptr_t>(row + e) & 15u); ++e) {
    float4 q0, q1;
    load_row8(pin + 8 * (size_t)row[e], q0, q1);
    a[0] = __fadd_rn(a[0], q0.x);
    a[1] = __fadd_rn(a[1], q0.y);
    a[2] = __fadd_rn(a[2], q0.z);
    a[3] = __fadd_rn(a[3], q0.w);
    a[4] = __fadd_rn(a[4], q1.x);
    a[5] = __fadd_rn(a[5], q1.y);
    a[6] = __fadd_rn(a[6], q1.z);
    a[7] = __fadd_rn(a[7], q1.w);
  }
  for (; e + 4 <= d; e += 4) {
    const uint4 ids = __ldg(reinterpret_cast<const uint4*>(row + e));
    const uint32_t id[4] = {ids.x, ids.y, ids.z, ids.w};
    float4 q[8];
#pragma unroll
    for (int u = 0; u < 4; ++u) load_row8(pin + 8 * (size_t)id[u], q[2 * u], q[2 * u + 1]);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a[0] = __fadd_rn(a[0], q[2 * u].x);
      a[1] = __fadd_rn(a[1], q[2 * u].y);
      a[2] = __fadd_rn(a[2], q[2 * u].z);
      a[3] = __fadd_rn(a[3], q[2 * u].w);
      a[4] = __fadd_rn(a[4], q[2 * u + 1].x);
      a[5] = __fadd_rn(a[5], q[2 * u + 1].y);
      a[6] = __fadd_rn(a[6], q[2 * u + 1].z);
      a[7] = __fadd_rn(a[7], q[2 * u + 1].w);
    }
  }
  for (; e < d; ++e) {
    float4 q0, q1;
    load_row8(pin + 8 * (size_t)row[e], q0, q1);
    a[0] = __fadd_rn(a[0], q0.x);
    a[1] = __fadd_rn(a[1], q0.y);
    a[2] = __fadd_rn(a[2], q0.z);
    a[3] = __fadd_rn(a[3], q0.w);
    a[4] = __fadd_rn(a[4], q1.x);
    a[5] = __fadd_rn(a[5], q1.y);
    a[6] = __fadd_rn(a[6], q1.z);
    a[7] = __fadd_rn(a[7], q1.w);
  }
  own(xs, xp);
  const float fd = (float)d;
  float o[8];
#pragma unroll
  for (int c = 0; c < 8; ++c)
    o[c] = filter_out<MODE>(__fmul_rn(__fadd_rn(xs[c], __fdiv_rn(a[c], fd)), 0.5f), xs[c], xp[c], c1);
  dst[2 * (size_t)i] = make_float4(o[0], o[1], o[2], o[3]);
  dst[2 * (size_t)i + 1] = make_float4(o[4], o[5], o[6], o[7]);
}

template <int MODE>
__global__ void __launch_bounds__(256) k_smooth_hub(GView v, const uint32_t* __restrict__ hubs,
                                                    const float* __restrict__ pin, float* __restrict__ pout,
                                                    const float* __restrict__ pprev, float c1) {
  __shared__ float part[HUB_SEGS][NPROJ];
  const uint32_t i = hubs[blockIdx.x], d = v.deg[i];
  const uint32_t* row = v.nbr + v.off[i];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t seg = (d + HUB_SEGS - 1) / HUB_SEGS;
  const uint32_t b = min(d, (uint32_t)w * seg), e = min(d, b + seg);
  if (lane < NPROJ) {
    float acc = 0.0f;
    for (uint32_t q = b; q < e; ++q) acc = __fadd_rn(acc, pin[(size_t)row[q] * NPROJ + lane]);
    part[w][lane] = acc;
  }
  __syncthreads();
  if (threadIdx.x < NPROJ) {
    float s = part[0][threadIdx.x];
    for (int q = 1; q < HUB_SEGS; ++q) s = __fadd_rn(s, part[q][threadIdx.x]);
    const float x = pin[(size_t)i * NPROJ + threadIdx.x];
    const float xp = MODE == 2 ? pprev[(size_t)i * NPROJ + threadIdx.x] : 0.0f;
    pout[(size_t)i * NPROJ + threadIdx.x] =
        filter_out<MODE>(__fmul_rn(__fadd_rn(x, __fdiv_rn(s, (float)d)), 0.5f), x, xp, c1);
  }
}

// Per item (one warp): sum deg_i x_c (8), sum deg_i, and sum x_c^2 (8). The
// walk's stationary distribution is proportional to the degree, so a
// projection with zero degree-weighted mean keeps it under smoothing: the
// constant mode is removed before smoothing and every RECENTER steps (rounding
// leaks into it while every other mode decays), and each column is rescaled
// to unit mean square at the same time so the decaying modes never underflow.
constexpr int CEN = 2 * NPROJ + 1;
__global__ void __launch_bounds__(256) k_proj_center_sums(const float* __restrict__ P, const uint32_t* __restrict__ deg,
                                                          const int4* __restrict__ items, uint32_t n_items,
                                                          double* __restrict__ part) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_items) return;
  const int4 it = items[w];
  double acc[CEN];
#pragma unroll
  for (int k = 0; k < CEN; ++k) acc[k] = 0.0;
  for (uint32_t i = (uint32_t)it.y + lane; i < (uint32_t)it.z; i += 32) {
    const double d = (double)deg[i];
#pragma unroll
    for (int c = 0; c < NPROJ; ++c) {
      const double x = P[(size_t)i * NPROJ + c];
      acc[c] += d * x;
      acc[NPROJ + 1 + c] += x * x;
    }
    acc[NPROJ] += d;
  }
#pragma unroll
  for (int k = 0; k < CEN; ++k) acc[k] = warp_sum(acc[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < CEN; ++k) part[(size_t)w * CEN + k] = acc[k];
  }
}

// x <- (x - m) * sc with m the degree-weighted mean (graphs with edges) and
// sc = 1 / sqrt(mean of x^2) (columns that are not all zero).
__global__ void k_proj_center(GView v, const double* __restrict__ gsum, float* __restrict__ P) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t w = t >> 3, c = t & 7;
  if (w >= v.nb) return;
  const uint32_t i = v.n0 + w, g = v.gid[i];
  const double* s = gsum + (size_t)(g - v.g0) * CEN;
  const double ms = s[NPROJ + 1 + c] / (double)(v.go[g + 1] - v.go[g]);
  const float m = s[NPROJ] > 0.0 ? (float)(s[c] / s[NPROJ]) : 0.0f;
  const float sc = ms > 0.0 ? (float)(1.0 / sqrt(ms)) : 1.0f;
  P[(size_t)i * NPROJ + c] = __fmul_rn(__fsub_rn(P[(size_t)i * NPROJ + c], m), sc);
}

// The Chebyshev pair (x, x_prev): each loses its own degree-weighted mean and
// both are scaled by x's factor, which keeps the three-term recurrence intact
// (the constant vector is an eigenvector of the walk and the projection that
// removes it commutes with the walk).
__global__ void k_proj_center_pair(GView v, const double* __restrict__ gsum, const double* __restrict__ gsum_prev,
                                   float* __restrict__ P, float* __restrict__ Pprev) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t w = t >> 3, c = t & 7;
  if (w >= v.nb) return;
  const uint32_t i = v.n0 + w, g = v.gid[i];
  const double* s = gsum + (size_t)(g - v.g0) * CEN;
  const double* sp = gsum_prev + (size_t)(g - v.g0) * CEN;
  const double ms = s[NPROJ + 1 + c] / (double)(v.go[g + 1] - v.go[g]);
  const float m = s[NPROJ] > 0.0 ? (float)(s[c] / s[NPROJ]) : 0.0f;
  const float mp = sp[NPROJ] > 0.0 ? (float)(sp[c] / sp[NPROJ]) : 0.0f;
  const float sc = ms > 0.0 ? (float)(1.0 / sqrt(ms)) : 1.0f;
  P[(size_t)i * NPROJ + c] = __fmul_rn(__fsub_rn(P[(size_t)i * NPROJ + c], m), sc);
  Pprev[(size_t)i * NPROJ + c] = __fmul_rn(__fsub_rn(Pprev[(size_t)i * NPROJ + c], mp), sc);
}

// Feature columns 17..24: the smoothed, centred and scaled projections in bf16.
__global__ void k_proj_write(GView v, const float* __restrict__ P, bf16* __restrict__ X) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t w = t >> 3, c = t & 7;
  if (w >= v.nb) return;
  const uint32_t i = v.n0 + w;
  X[(size_t)i * FEAT + 1 + WALK_LEN + c] = __float2bfloat16_rn(P[(size_t)i * NPROJ + c]);
}

// ========================================================= reductions ==
// Item = (graph, first node, end node): one warp sums V per-node doubles
// (rows local to n0) over the item's nodes; then one thread per graph adds
// its items in order. Fixed order throughout.
template <int V>
__global__ void __launch_bounds__(256) k_item_reduce(const double* __restrict__ vals, uint32_t n0,
                                                     const int4* __restrict__ items, uint32_t n_items,
                                                     double* __restrict__ part) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_items) return;
  const int4 it = items[w];
  double acc[V];
#pragma unroll
  for (int c = 0; c < V; ++c) acc[c] = 0.0;
  for (uint32_t i = (uint32_t)it.y + lane; i < (uint32_t)it.z; i += 32) {
#pragma unroll
    for (int c = 0; c < V; ++c) acc[c] += vals[(size_t)(i - n0) * V + c];
  }
#pragma unroll
  for (int c = 0; c < V; ++c) acc[c] = warp_sum(acc[c]);
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < V; ++c) part[(size_t)w * V + c] = acc[c];
  }
}

template <int V>
__global__ void k_graph_sum(const double* __restrict__ part, const uint32_t* __restrict__ item_off, uint32_t g0,
                            uint32_t ng, uint32_t i0, double* __restrict__ gsum) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng) return;
  const uint32_t a = item_off[g0 + g] - i0, b = item_off[g0 + g + 1] - i0;
  for (int c = 0; c < V; ++c) {
    double s = 0.0;
    for (uint32_t it = a; it < b; ++it) s += part[(size_t)it * V + c];
    gsum[(size_t)g * V + c] = s;
  }
}

// out[col] = sum over z of part[z][col] in f64, one warp per column: lane l
// adds z = l, l + 32, ... in order, then a fixed butterfly over the lanes
// (the same association on every run).
__global__ void k_reduce_parts(const double* __restrict__ part, uint32_t chunks, uint32_t width,
                               float* __restrict__ out) {
  const uint32_t col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
  if (col >= width) return;  // whole warps
  double s = 0.0;
  for (uint32_t z = lane; z < chunks; z += 32u) s += part[(size_t)z * width + col];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
  if (lane == 0) out[col] = (float)s;
}
inline uint32_t reduce_parts_blocks(uint32_t width) { return cdiv(width * 32u, 256u); }

__global__ void k_reduce_splits(const float* __restrict__ part, uint32_t splits, uint32_t width,
                                float* __restrict__ out) {
  const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= width) return;
  double s = 0.0;
  for (uint32_t z = 0; z < splits; ++z) s += (double)part[(size_t)z * width + col];
  out[col] = (float)s;
}

// ============================================================ forward ==
// Mean of the neighbours' rows (bf16, D columns of src) into dst[:, D:2D];
// copy_self also copies the node's own row into dst[:, 0:D]. D/4 lanes per
// node, 4 columns each, f32 sums in CSR order. src and dst may be the same
// buffer (the halves are disjoint). Rows are local to the batch.
template <int D>
__global__ void __launch_bounds__(256) k_agg(GView v, const bf16* src, int src_ld, bf16* dst, int dst_ld,
                                             int copy_self) {
  constexpr int LPN = D / 4;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t w = t / LPN, c = (t % LPN) * 4;
  if (w >= v.nb) return;
  const uint32_t i = v.n0 + w, d = v.deg[i];
  if (copy_self)
    *reinterpret_cast<uint2*>(dst + (size_t)w * dst_ld + c) =
        *reinterpret_cast<const uint2*>(src + (size_t)w * src_ld + c);
  if (d > HUB_DEG) return;
  const uint32_t* row = v.nbr + v.off[i];
  float a[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  uint32_t e = 0;
  for (; e + 4 <= d; e += 4) {
    uint2 q[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      q[u] = *reinterpret_cast<const uint2*>(src + (size_t)(row[e + u] - v.n0) * src_ld + c);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      float f[4];
      unpack4(q[u], f);
#pragma unroll
      for (int k = 0; k < 4; ++k) a[k] = __fadd_rn(a[k], f[k]);
    }
  }
  for (; e < d; ++e) {
    float f[4];
    unpack4(*reinterpret_cast<const uint2*>(src + (size_t)(row[e] - v.n0) * src_ld + c), f);
#pragma unroll
    for (int k = 0; k < 4; ++k) a[k] = __fadd_rn(a[k], f[k]);
  }
  float m[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) m[k] = d ? __fdiv_rn(a[k], (float)d) : 0.0f;
  *reinterpret_cast<uint2*>(dst + (size_t)w * dst_ld + D + c) = pack4(m);
}

// Hub rows (deg > HUB_DEG): one block, warp s sums segment s, segments added in order.
template <int D>
__global__ void __launch_bounds__(256) k_agg_hub(GView v, const uint32_t* __restrict__ hubs, const bf16* src,
                                                 int src_ld, bf16* dst, int dst_ld) {
  __shared__ float part[HUB_SEGS][D];
  const uint32_t i = hubs[blockIdx.x], d = v.deg[i];
  const uint32_t* row = v.nbr + v.off[i];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t seg = (d + HUB_SEGS - 1) / HUB_SEGS;
  const uint32_t b = min(d, (uint32_t)w * seg), e = min(d, b + seg);
  if (lane < D / 4) {
    const int c = lane * 4;
    float a[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (uint32_t q = b; q < e; ++q) {
      float f[4];
      unpack4(*reinterpret_cast<const uint2*>(src + (size_t)(row[q] - v.n0) * src_ld + c), f);
#pragma unroll
      for (int k = 0; k < 4; ++k) a[k] = __fadd_rn(a[k], f[k]);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) part[w][c + k] = a[k];
  }
  __syncthreads();
  for (int c = threadIdx.x; c < D; c += blockDim.x) {
    float s = part[0][c];
    for (int q = 1; q < HUB_SEGS; ++q) s = __fadd_rn(s, part[q][c]);
    dst[(size_t)(i - v.n0) * dst_ld + D + c] = __float2bfloat16_rn(__fdiv_rn(s, (float)d));
  }
}

// Y = H3 W_h + b_h: one warp per node, lane k holds hidden columns 4k..4k+3.
// Y = H3 Wh + bh, one thread per node: the node's 128-wide bf16 row in 16
// 16-byte loads (all independent, so they are in flight together), the head
// weights (128 x 4) broadcast from shared memory; terms added in k order.
__global__ void __launch_bounds__(256) k_head(uint32_t nb, const bf16* __restrict__ H3, const bf16* __restrict__ Wh,
                                              const float* __restrict__ bh, int dim, float4* __restrict__ Y) {
  __shared__ float w[HID * 4];
  for (uint32_t t = threadIdx.x; t < HID * 4; t += blockDim.x) w[t] = bf2f(Wh[t]);
  __syncthreads();
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nb) return;
  const uint4* row = reinterpret_cast<const uint4*>(H3 + (size_t)r * HID);
  uint4 u[HID / 8];
#pragma unroll
  for (int q = 0; q < HID / 8; ++q) u[q] = row[q];
  float y0 = 0.0f, y1 = 0.0f, y2 = 0.0f;
#pragma unroll
  for (int q = 0; q < HID / 8; ++q) {
    float h[8];
    unpack4(make_uint2(u[q].x, u[q].y), h);
    unpack4(make_uint2(u[q].z, u[q].w), h + 4);
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const float* wr = w + (q * 8 + e) * 4;
      y0 += h[e] * wr[0];
      y1 += h[e] * wr[1];
      y2 += h[e] * wr[2];
    }
  }
  Y[r] = make_float4(y0 + bh[0], y1 + bh[1], dim == 3 ? y2 + bh[2] : 0.0f, 0.0f);
}

// =============================================================== loss ==
struct PairCtx {
  GView v;
  const float4* T;  // target layout (global rows)
  const float4* Y;  // prediction (batch rows)
  uint32_t partners;
  uint64_t seed, step;
};

// Pair q of node i: its CSR entries first, then `partners` uniform
// same-graph nodes other than i (none when the graph has one node).
__device__ __forceinline__ bool pair_at(const PairCtx& p, uint32_t i, uint32_t d, uint32_t rowb, uint32_t q,
                                        uint32_t gb, uint32_t ng, uint32_t* j) {
  if (q < d) {
    *j = p.v.nbr[rowb + q];
    return true;
  }
  if (ng < 2) return false;
  const uint32_t r = gb + pick(hash4(p.seed ^ SALT_PAIR, i, q - d, p.step), ng - 1);
  *j = r + (r >= i ? 1u : 0u);
  return true;
}

__device__ __forceinline__ float len3(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

// Per node: sum q, sum q^2 and the pair count (target distances < 1e-6 skipped).
__global__ void __launch_bounds__(256) k_loss_stats(PairCtx p, double* __restrict__ vals) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= p.v.nb) return;
  const uint32_t i = p.v.n0 + w, d = p.v.deg[i], rowb = p.v.off[i], g = p.v.gid[i];
  const uint32_t gb = p.v.go[g], ng = p.v.go[g + 1] - gb;
  const float4 ti = p.T[i], yi = p.Y[w];
  double s1 = 0.0, s2 = 0.0, c = 0.0;
  for (uint32_t q = lane; q < d + p.partners; q += 32) {
    uint32_t j;
    if (!pair_at(p, i, d, rowb, q, gb, ng, &j)) continue;
    const float4 tj = p.T[j], yj = p.Y[j - p.v.n0];
    const float dt = len3(ti.x - tj.x, ti.y - tj.y, ti.z - tj.z);
    if (!(dt >= 1e-6f)) continue;
    const float r = len3(yi.x - yj.x, yi.y - yj.y, yi.z - yj.z);
    const double qq = (double)r / (double)dt;
    s1 += qq;
    s2 += qq * qq;
    c += 1.0;
  }
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  c = warp_sum(c);
  if (lane == 0) {
    vals[(size_t)w * 3] = s1;
    vals[(size_t)w * 3 + 1] = s2;
    vals[(size_t)w * 3 + 2] = c;
  }
}

// Per graph: alpha, the gradient coefficient 2 / (|P_g| G) and the batch's
// mean loss over graphs with at least one pair. One block, fixed tree order.
__global__ void __launch_bounds__(256) k_loss_finish(const double* __restrict__ gsum, uint32_t ng,
                                                     double* __restrict__ galpha, double* __restrict__ gcoef,
                                                     float* __restrict__ loss_out) {
  __shared__ double sl[256], sc[256];
  double l = 0.0, c = 0.0;
  for (uint32_t g = threadIdx.x; g < ng; g += 256) {
    const double s1 = gsum[(size_t)g * 3], s2 = gsum[(size_t)g * 3 + 1], P = gsum[(size_t)g * 3 + 2];
    galpha[g] = s2 > 0.0 ? s1 / s2 : 0.0;
    if (P > 0.0) {
      l += s2 > 0.0 ? 1.0 - s1 * s1 / (s2 * P) : 1.0;
      c += 1.0;
    }
  }
  sl[threadIdx.x] = l;
  sc[threadIdx.x] = c;
  __syncthreads();
  for (int s = 128; s; s >>= 1) {
    if ((int)threadIdx.x < s) {
      sl[threadIdx.x] += sl[threadIdx.x + s];
      sc[threadIdx.x] += sc[threadIdx.x + s];
    }
    __syncthreads();
  }
  const double G = sc[0];
  for (uint32_t g = threadIdx.x; g < ng; g += 256) {
    const double P = gsum[(size_t)g * 3 + 2];
    gcoef[g] = (P > 0.0 && G > 0.0) ? 2.0 / (P * G) : 0.0;
  }
  if (threadIdx.x == 0 && loss_out) *loss_out = G > 0.0 ? (float)(sl[0] / G) : 0.0f;
}

// dL/dY_i = sum over i's pairs of coef_g (alpha q - 1) alpha / d * (Y_i - Y_j) / r.
__global__ void __launch_bounds__(256) k_loss_grad(PairCtx p, const double* __restrict__ galpha,
                                                   const double* __restrict__ gcoef, float4* __restrict__ dY) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= p.v.nb) return;
  const uint32_t i = p.v.n0 + w, d = p.v.deg[i], rowb = p.v.off[i], g = p.v.gid[i];
  const uint32_t gb = p.v.go[g], ng = p.v.go[g + 1] - gb;
  const double a = galpha[g - p.v.g0], cf = gcoef[g - p.v.g0];
  const float4 ti = p.T[i], yi = p.Y[w];
  double gx = 0.0, gy = 0.0, gz = 0.0;
  for (uint32_t q = lane; q < d + p.partners; q += 32) {
    uint32_t j;
    if (!pair_at(p, i, d, rowb, q, gb, ng, &j)) continue;
    const float4 tj = p.T[j], yj = p.Y[j - p.v.n0];
    const float dt = len3(ti.x - tj.x, ti.y - tj.y, ti.z - tj.z);
    if (!(dt >= 1e-6f)) continue;
    const float dx = yi.x - yj.x, dy = yi.y - yj.y, dz = yi.z - yj.z;
    const float r = len3(dx, dy, dz);
    if (!(r > 1e-12f)) continue;
    const double qq = (double)r / (double)dt;
    const double wgt = cf * (a * qq - 1.0) * a / ((double)dt * (double)r);
    gx += wgt * dx;
    gy += wgt * dy;
    gz += wgt * dz;
  }
  gx = warp_sum(gx);
  gy = warp_sum(gy);
  gz = warp_sum(gz);
  if (lane == 0) dY[w] = make_float4((float)gx, (float)gy, (float)gz, 0.0f);
}

// =========================================================== backward ==
// dZ_2 = (dY W_h^T) * (H3 > 0), bf16.
// dZ = (dY Wh^T) masked by H3 > 0, one thread per node (16-byte loads and
// stores of its 128-wide bf16 rows, head weights in shared memory).
__global__ void __launch_bounds__(256) k_head_bwd(uint32_t nb, const bf16* __restrict__ H3,
                                                  const bf16* __restrict__ Wh, const float4* __restrict__ dY,
                                                  bf16* __restrict__ dZ) {
  __shared__ float w[HID * 4];
  for (uint32_t t = threadIdx.x; t < HID * 4; t += blockDim.x) w[t] = bf2f(Wh[t]);
  __syncthreads();
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nb) return;
  const float4 g = dY[r];
  const uint4* row = reinterpret_cast<const uint4*>(H3 + (size_t)r * HID);
  uint4* out = reinterpret_cast<uint4*>(dZ + (size_t)r * HID);
  uint4 u[HID / 8];
#pragma unroll
  for (int q = 0; q < HID / 8; ++q) u[q] = row[q];
#pragma unroll
  for (int q = 0; q < HID / 8; ++q) {
    float h[8], o[8];
    unpack4(make_uint2(u[q].x, u[q].y), h);
    unpack4(make_uint2(u[q].z, u[q].w), h + 4);
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const float* wr = w + (q * 8 + e) * 4;
      const float v = g.x * wr[0] + g.y * wr[1] + g.z * wr[2];
      o[e] = h[e] > 0.0f ? v : 0.0f;
    }
    const uint2 a = pack4(o), b = pack4(o + 4);
    out[q] = make_uint4(a.x, a.y, b.x, b.y);
  }
}

// Head gradient partials per chunk of rows: [k*4 + c] = sum H3[r][k] dY[r][c],
// [512 + c] = sum dY[r][c].
__global__ void __launch_bounds__(HID) k_head_wgrad(uint32_t nb, uint32_t chunk, const bf16* __restrict__ H3,
                                                    const float4* __restrict__ dY, double* __restrict__ part) {
  const uint32_t k = threadIdx.x;
  const uint32_t r0 = blockIdx.x * chunk, r1 = min(nb, r0 + chunk);
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, bsum = 0.0;
  for (uint32_t r = r0; r < r1; ++r) {
    const double h = bf2f(H3[(size_t)r * HID + k]);
    const float4 g = dY[r];
    a0 += h * g.x;
    a1 += h * g.y;
    a2 += h * g.z;
    if (k < 4) bsum += k == 0 ? g.x : k == 1 ? g.y : k == 2 ? g.z : 0.0f;
  }
  double* o = part + (size_t)blockIdx.x * HEAD_W;
  o[k * 4] = a0;
  o[k * 4 + 1] = a1;
  o[k * 4 + 2] = a2;
  o[k * 4 + 3] = 0.0;
  if (k < 4) o[HID * 4 + k] = bsum;
}

// Bias gradient partials: column sums of dZ (bf16, 128 wide) per chunk of rows.
__global__ void __launch_bounds__(HID) k_colsum(uint32_t nb, uint32_t chunk, const bf16* __restrict__ dZ,
                                                double* __restrict__ part) {
  const uint32_t c = threadIdx.x;
  const uint32_t r0 = blockIdx.x * chunk, r1 = min(nb, r0 + chunk);
  double a = 0.0;
  for (uint32_t r = r0; r < r1; ++r) a += bf2f(dZ[(size_t)r * HID + c]);
  part[(size_t)blockIdx.x * HID + c] = a;
}

// dZ_{l-1}[j] = bf16((dA[j][0:128] + sum_{i in N(j)} dA[i][128:256] * (1 / deg_i)) * (H_l[j] > 0)):
// the transpose of the mean aggregation (the CSR is symmetric), CSR order.
// dA is the bf16 output of the activation-gradient GEMM (8 bytes per lane
// and neighbour gathered).
__global__ void __launch_bounds__(256) k_agg_bwd(GView v, const bf16* __restrict__ dA, const bf16* __restrict__ A,
                                                 bf16* __restrict__ dZ) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= v.nb) return;
  const uint32_t i = v.n0 + w, d = v.deg[i];
  if (d > HUB_DEG) return;
  const uint32_t c = lane * 4;
  const uint32_t* row = v.nbr + v.off[i];
  float a[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  // 32 neighbours at a time: lane k reads the k-th id and its neighbour's
  // 1/degree (one round trip for all 32), then the warp gathers the rows
  // four at a time, added in CSR order.
  for (uint32_t base = 0; base < d; base += 32) {
    const uint32_t cnt = min(32u, d - base);
    uint32_t jl = 0;
    float il = 0.0f;
    if (lane < cnt) {
      jl = row[base + lane];
      il = __frcp_rn((float)v.deg[jl]);
    }
    for (uint32_t t = 0; t < cnt; t += 4) {
      float q[4][4], inv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t j = __shfl_sync(0xFFFFFFFFu, jl, (int)(t + u) & 31);
        inv[u] = __shfl_sync(0xFFFFFFFFu, il, (int)(t + u) & 31);
        if (t + u < cnt) unpack4(*reinterpret_cast<const uint2*>(dA + (size_t)(j - v.n0) * 2 * HID + HID + c), q[u]);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (t + u < cnt)
#pragma unroll
          for (int k = 0; k < 4; ++k) a[k] = __fadd_rn(a[k], __fmul_rn(q[u][k], inv[u]));
    }
  }
  float h[4], o[4], sv[4];
  unpack4(*reinterpret_cast<const uint2*>(dA + (size_t)w * 2 * HID + c), sv);
  unpack4(*reinterpret_cast<const uint2*>(A + (size_t)w * 2 * HID + c), h);
#pragma unroll
  for (int k = 0; k < 4; ++k) o[k] = h[k] > 0.0f ? __fadd_rn(sv[k], a[k]) : 0.0f;
  *reinterpret_cast<uint2*>(dZ + (size_t)w * HID + c) = pack4(o);
}

__global__ void __launch_bounds__(256) k_agg_bwd_hub(GView v, const uint32_t* __restrict__ hubs,
                                                     const bf16* __restrict__ dA, const bf16* __restrict__ A,
                                                     bf16* __restrict__ dZ) {
  __shared__ float part[HUB_SEGS][HID];
  const uint32_t i = hubs[blockIdx.x], d = v.deg[i];
  const uint32_t* row = v.nbr + v.off[i];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t seg = (d + HUB_SEGS - 1) / HUB_SEGS;
  const uint32_t b = min(d, (uint32_t)w * seg), e = min(d, b + seg);
  const int c = lane * 4;
  float a[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (uint32_t q = b; q < e; ++q) {
    const uint32_t j = row[q];
    const float ij = __frcp_rn((float)v.deg[j]);
    float x[4];
    unpack4(*reinterpret_cast<const uint2*>(dA + (size_t)(j - v.n0) * 2 * HID + HID + c), x);
#pragma unroll
    for (int k = 0; k < 4; ++k) a[k] = __fadd_rn(a[k], __fmul_rn(x[k], ij));
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) part[w][c + k] = a[k];
  __syncthreads();
  if (threadIdx.x < HID) {
    const int col = threadIdx.x;
    float s = part[0][col];
    for (int q = 1; q < HUB_SEGS; ++q) s = __fadd_rn(s, part[q][col]);
    const size_t r = (size_t)(i - v.n0);
    const float h = bf2f(A[r * 2 * HID + col]);
    dZ[r * HID + col] = __float2bfloat16_rn(h > 0.0f ? __fadd_rn(bf2f(dA[r * 2 * HID + col]), s) : 0.0f);
  }
}

// ========================================================== optimiser ==
__global__ void __launch_bounds__(1024) k_grad_norm(const float* __restrict__ g, uint32_t n, double* __restrict__ out) {
  __shared__ double s[1024];
  double a = 0.0;
  for (uint32_t i = threadIdx.x; i < n; i += 1024) a += (double)g[i] * (double)g[i];
  s[threadIdx.x] = a;
  __syncthreads();
  for (int k = 512; k; k >>= 1) {
    if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = s[0];
}

// Adam with bias correction folded into lr_t; the gradient is clipped to the
// global norm `clip` first. Writes the bf16 shadow the GEMMs read.
__global__ void k_adam(float* __restrict__ th, bf16* __restrict__ thb, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, uint32_t n, const double* __restrict__ norm2,
                       float clip, float lr_t, float b1, float b2, float eps) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double nr = sqrt(*norm2);
  const float sc = (clip > 0.0f && nr > (double)clip) ? (float)((double)clip / nr) : 1.0f;
  const float gi = g[i] * sc;
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float t = th[i] - lr_t * mi / (sqrtf(vi) + eps);
  th[i] = t;
  thb[i] = __float2bfloat16_rn(t);
}

__global__ void k_to_bf16(const float* __restrict__ x, uint32_t n, bf16* __restrict__ y) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

// The three layer weights (kin x HID row-major at L.w[l]) transposed to
// HID x kin row-major at the same offsets: the K-major B operand of the
// TMA-staged forward GEMMs. One thread per element; consecutive threads
// write consecutive elements of a transposed row.
__global__ void k_transpose_w(const bf16* __restrict__ w, ParamLayout L, bf16* __restrict__ wt) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  for (int l = 0; l < 3; ++l) {
    const uint32_t n = (uint32_t)L.kin[l] * HID;
    if (i < n) {
      const uint32_t c = i / (uint32_t)L.kin[l], k = i % (uint32_t)L.kin[l];
      wt[L.w[l] + i] = w[L.w[l] + (size_t)k * HID + c];
      return;
    }
    i -= n;
  }
}

// ============================================================ hand-off ==
// Per node (one warp): Y.xyz, sum over row entries j > i of |Y_i - Y_j|^2, deg, deg^2.
__global__ void __launch_bounds__(256) k_scale_vals(GView v, const float4* __restrict__ Y, double* __restrict__ vals) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= v.nb) return;
  const uint32_t i = v.n0 + w, d = v.deg[i], rowb = v.off[i];
  const float4 yi = Y[w];
  double a = 0.0;
  for (uint32_t q = lane; q < d; q += 32) {
    const uint32_t j = v.nbr[rowb + q];
    if (j <= i) continue;
    const float4 yj = Y[j - v.n0];
    const double dx = (double)yi.x - yj.x, dy = (double)yi.y - yj.y, dz = (double)yi.z - yj.z;
    a += dx * dx + dy * dy + dz * dz;
  }
  a = warp_sum(a);
  if (lane == 0) {
    double* o = vals + (size_t)w * 6;
    o[0] = yi.x;
    o[1] = yi.y;
    o[2] = yi.z;
    o[3] = a;
    o[4] = (double)d;
    o[5] = (double)d * (double)d;
  }
}

__global__ void k_scale_grav(GView v, const float4* __restrict__ Y, const double* __restrict__ gsum6,
                             double* __restrict__ vals1) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= v.nb) return;
  const uint32_t i = v.n0 + w, g = v.gid[i];
  const double ng = (double)(v.go[g + 1] - v.go[g]);
  const double* s = gsum6 + (size_t)(g - v.g0) * 6;
  const float4 y = Y[w];
  const double dx = y.x - s[0] / ng, dy = y.y - s[1] / ng, dz = y.z - s[2] / ng;
  vals1[w] = (double)v.deg[i] * sqrt(dx * dx + dy * dy + dz * dz);
}

// Per graph: centre mu and the virial scale s (1 when undetermined).
__global__ void k_scale_finish(const double* __restrict__ gsum6, const double* __restrict__ gsum1,
                               const uint32_t* __restrict__ go, uint32_t g0, uint32_t ng, float kr, float grav,
                               float4* __restrict__ gs) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng) return;
  const double n = (double)(go[g0 + g + 1] - go[g0 + g]);
  if (n <= 0.0) {
    gs[g] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    return;
  }
  const double* s = gsum6 + (size_t)g * 6;
  const double A = s[3], sd = s[4], sd2 = s[5];
  const double R = 0.5 * (double)kr * (sd * (sd + n) - (sd2 + sd));
  const double G = (double)grav * gsum1[g];
  double sc = 1.0;
  if (A > 0.0 && R > 0.0) sc = (-G + sqrt(G * G + 4.0 * A * R)) / (2.0 * A);
  gs[g] = make_float4((float)(s[0] / n), (float)(s[1] / n), (float)(s[2] / n), (float)sc);
}

__global__ void k_scale_apply(GView v, const float4* __restrict__ Y, const float4* __restrict__ gs, int dim,
                              float* __restrict__ out) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= v.nb) return;
  const float4 s = gs[v.gid[v.n0 + w] - v.g0], y = Y[w];
  out[(size_t)w * 3] = s.w * (y.x - s.x);
  out[(size_t)w * 3 + 1] = s.w * (y.y - s.y);
  out[(size_t)w * 3 + 2] = dim == 3 ? s.w * (y.z - s.z) : 0.0f;
}

// ========================================================= evaluation ==
__global__ void k_xyz_to_f4(const float* __restrict__ xyz, uint32_t n, float4* __restrict__ P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) P[i] = make_float4(xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2], 0.0f);
}

// Per node (one warp): pivot terms q = |x_i - x_p| / d(i, p) (sum q, sum q^2,
// count) and edge lengths over row entries j > i (sum l, sum l^2, count).
__global__ void __launch_bounds__(256) k_eval_vals(GView v, const float4* __restrict__ P,
                                                   const uint32_t* __restrict__ piv, const uint16_t* __restrict__ dist,
                                                   uint32_t k, double* __restrict__ vals) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= v.nb) return;
  const uint32_t i = v.n0 + w, d = v.deg[i], rowb = v.off[i], g = v.gid[i];
  const float4 pi = P[i];
  double s1 = 0.0, s2 = 0.0, c = 0.0, l1 = 0.0, l2 = 0.0, lc = 0.0;
  for (uint32_t q = lane; q < k; q += 32) {
    const uint32_t j = piv[(size_t)g * k + q];
    if (j == NO_PIVOT || j == i) continue;
    const uint16_t du = dist[(size_t)i * k + q];
    if (du == 0 || du == NO_DIST) continue;
    const float4 pj = P[j];
    const double dx = (double)pi.x - pj.x, dy = (double)pi.y - pj.y, dz = (double)pi.z - pj.z;
    const double qq = sqrt(dx * dx + dy * dy + dz * dz) / (double)du;
    s1 += qq;
    s2 += qq * qq;
    c += 1.0;
  }
  for (uint32_t q = lane; q < d; q += 32) {
    const uint32_t j = v.nbr[rowb + q];
    if (j <= i) continue;
    const float4 pj = P[j];
    const double dx = (double)pi.x - pj.x, dy = (double)pi.y - pj.y, dz = (double)pi.z - pj.z;
    const double l = sqrt(dx * dx + dy * dy + dz * dz);
    l1 += l;
    l2 += l * l;
    lc += 1.0;
  }
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  c = warp_sum(c);
  l1 = warp_sum(l1);
  l2 = warp_sum(l2);
  lc = warp_sum(lc);
  if (lane == 0) {
    double* o = vals + (size_t)w * 6;
    o[0] = s1;
    o[1] = s2;
    o[2] = c;
    o[3] = l1;
    o[4] = l2;
    o[5] = lc;
  }
}

// Per graph: scale-normalized stress 1 - (sum q)^2 / (count sum q^2) (0 with
// no terms or a collapsed layout, as metrics.rs:31-59) and the edge-length
// coefficient of variation (0 below two edges or a zero mean, :150-164).
__global__ void k_eval_finish(const double* __restrict__ gsum, uint32_t G, double* __restrict__ out) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  const double* s = gsum + (size_t)g * 6;
  double st = 0.0, cv = 0.0;
  if (s[2] > 0.0 && s[1] > 0.0) st = 1.0 - s[0] * s[0] / (s[1] * s[2]);
  if (s[5] >= 2.0) {
    const double mean = s[3] / s[5];
    if (mean > 1e-12) cv = sqrt(fmax(s[4] / s[5] - mean * mean, 0.0)) / mean;
  }
  out[(size_t)g * 4] = st;
  out[(size_t)g * 4 + 1] = cv;
  out[(size_t)g * 4 + 2] = s[2];
  out[(size_t)g * 4 + 3] = s[5];
}

// =============================================================== host ==
template <typename T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    if (count <= n && p) return;
    free();
    const size_t c = std::max<size_t>(count, 1);
    JC_CUDA_CHECK(cudaMalloc(&p, c * sizeof(T)));
    n = c;
  }
  void zero(cudaStream_t s) { JC_CUDA_CHECK(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
  void upload(const T* src, size_t count, cudaStream_t s) {
    alloc(count);
    if (count) JC_CUDA_CHECK(cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  Buf() = default;
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  ~Buf() { free(); }
};

// Graphs given as concatenated per-graph CSRs (local ids), joined into one
// global CSR plus the per-graph and per-item bookkeeping the kernels use.
struct HostSet {
  uint32_t n = 0, G = 0;
  std::vector<uint32_t> go, off, nbr, deg, gid, item_off, hubs;
  std::vector<int4> items;
};

HostSet assemble(uint32_t G, const uint32_t* graph_nodes, const uint32_t* offsets, const uint32_t* neighbors,
                 bool undirected) {
  if (G == 0) fail(JC_ERR_ARG, "at least one graph is required");
  if (!graph_nodes || !offsets) fail(JC_ERR_ARG, "graph_nodes and offsets must be non-null");
  HostSet h;
  h.G = G;
  h.go.resize(G + 1);
  uint64_t n = 0, nnz = 0;
  for (uint32_t g = 0; g < G; ++g) {
    h.go[g] = (uint32_t)n;
    const uint32_t* o = offsets + n + g;
    n += graph_nodes[g];
    if (n > 0x7FFFFFFFull) fail(JC_ERR_ARG, "too many nodes");
    nnz += o[graph_nodes[g]];
  }
  h.go[G] = (uint32_t)n;
  if (nnz > 0xFFFFFFFFull) fail(JC_ERR_ARG, "too many CSR entries");
  if (nnz && !neighbors) fail(JC_ERR_ARG, "neighbors must be non-null");
  h.n = (uint32_t)n;
  h.off.resize(n + 1);
  h.nbr.resize(nnz);
  h.deg.resize(n);
  h.gid.resize(n);
  uint64_t e0 = 0;
  for (uint32_t g = 0; g < G; ++g) {
    const uint32_t ng = graph_nodes[g], b = h.go[g];
    const uint32_t* o = offsets + b + g;
    if (o[0] != 0) fail(JC_ERR_ARG, "graph " + std::to_string(g) + ": offsets[0] must be 0");
    for (uint32_t v = 0; v < ng; ++v) {
      if (o[v + 1] < o[v]) fail(JC_ERR_ARG, "graph " + std::to_string(g) + ": offsets must be non-decreasing");
      h.off[b + v] = (uint32_t)(e0 + o[v]);
      h.deg[b + v] = o[v + 1] - o[v];
      h.gid[b + v] = g;
    }
    const uint32_t* nb = neighbors + e0;
    for (uint32_t e = 0; e < o[ng]; ++e) {
      if (nb[e] >= ng)
        fail(JC_ERR_ARG, "graph " + std::to_string(g) + ": neighbor id " + std::to_string(nb[e]) + " out of range");
      h.nbr[e0 + e] = b + nb[e];
    }
    e0 += o[ng];
  }
  h.off[n] = (uint32_t)e0;
  if (undirected) {
    // The mean aggregation's backward pass gathers over the node's own row, which
    // is its transpose only when every entry (v, u) has its (u, v); self-loops
    // would pair a node with itself in the loss.
    std::vector<uint32_t> sorted(h.nbr);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t vv = 0; vv < (int64_t)n; ++vv)
      std::sort(sorted.begin() + h.off[vv], sorted.begin() + h.off[vv + 1]);
    bool bad = false;
#pragma omp parallel for schedule(dynamic, 4096) reduction(|| : bad)
    for (int64_t vv = 0; vv < (int64_t)n; ++vv) {
      const uint32_t v = (uint32_t)vv;
      for (uint32_t e = h.off[v]; e < h.off[v + 1] && !bad; ++e) {
        const uint32_t u = sorted[e];
        const uint32_t* ru = sorted.data() + h.off[u];
        if (u == v || !std::binary_search(ru, ru + h.deg[u], v)) bad = true;
      }
    }
    if (bad) fail(JC_ERR_ARG, "graphs must be undirected (every entry (v, u) has (u, v)) without self-loops");
  }
  h.item_off.resize(G + 1);
  for (uint32_t g = 0; g < G; ++g) {
    h.item_off[g] = (uint32_t)h.items.size();
    for (uint32_t b = h.go[g]; b < h.go[g + 1]; b += ITEM_NODES)
      h.items.push_back(make_int4((int)g, (int)b, (int)std::min(h.go[g + 1], b + ITEM_NODES), 0));
  }
  h.item_off[G] = (uint32_t)h.items.size();
  for (uint32_t v = 0; v < n; ++v)
    if (h.deg[v] > HUB_DEG) h.hubs.push_back(v);
  return h;
}

struct Batch {
  uint32_t g0, g1, n0, nb, i0, i1, h0, h1;
};

struct DevSet {
  HostSet h;
  Buf<uint32_t> go, off, nbr, deg, gid, item_off, hubs;
  Buf<int4> items;
  void upload(HostSet&& hs, cudaStream_t s) {
    h = std::move(hs);
    go.upload(h.go.data(), h.go.size(), s);
    off.upload(h.off.data(), h.off.size(), s);
    nbr.upload(h.nbr.data(), h.nbr.size(), s);
    deg.upload(h.deg.data(), h.deg.size(), s);
    gid.upload(h.gid.data(), h.gid.size(), s);
    item_off.upload(h.item_off.data(), h.item_off.size(), s);
    hubs.upload(h.hubs.data(), h.hubs.size(), s);
    items.upload(h.items.data(), h.items.size(), s);
    JC_CUDA_CHECK(cudaStreamSynchronize(s));  // host vectors stay owned by h
  }
  Batch batch(uint32_t g0, uint32_t g1) const {
    Batch b{};
    b.g0 = g0;
    b.g1 = g1;
    b.n0 = h.go[g0];
    b.nb = h.go[g1] - h.go[g0];
    b.i0 = h.item_off[g0];
    b.i1 = h.item_off[g1];
    b.h0 = (uint32_t)(std::lower_bound(h.hubs.begin(), h.hubs.end(), b.n0) - h.hubs.begin());
    b.h1 = (uint32_t)(std::lower_bound(h.hubs.begin(), h.hubs.end(), b.n0 + b.nb) - h.hubs.begin());
    return b;
  }
  GView view(const Batch& b) const {
    return GView{off.p, nbr.p, deg.p, gid.p, go.p, b.n0, b.nb, b.g0};
  }
};

// cuTensorMapEncodeTiled, taken from the driver through the runtime's
// entry-point query (the library does not link against libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      (void)cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// Tensor map of a bf16 operand with `rows` tile rows (M or N) and K
// columns, row stride `ld` elements, 128-byte swizzle, zero fill outside the
// operand. K-major (rows x K in memory): boxes of 64 K x box_rows rows.
// MN-major (K x rows in memory): boxes of 64 rows x 64 K.
inline bool tmap_operand(CUtensorMap* m, const void* base, int rows, int K, int ld, int box_rows, bool kmajor) {
  const EncodeTiledFn f = encode_tiled();
  if (!f) return false;
  const cuuint64_t dims[2] = {kmajor ? (cuuint64_t)K : (cuuint64_t)rows, kmajor ? (cuuint64_t)rows : (cuuint64_t)K};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2u};
  const cuuint32_t box[2] = {64u, kmajor ? (cuuint32_t)box_rows : 64u};
  const cuuint32_t elem[2] = {1u, 1u};
  return f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, elem,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Operand staging of a GEMM launch.
enum GemmStaging : int { STAGE_AUTO = 0, STAGE_CP_ASYNC = 1, STAGE_TMA = 2 };

// The TMA-staged kernel takes each operand from one base (no A0/A1
// concatenation), 16-byte aligned, with a row stride of whole 16-byte units
// that covers the row (K for a K-major operand, M or N for an MN-major one),
// and split-K parts that start on 64-wide chunks.
inline bool tma_eligible(const tc::GemmArgs& g, int splits) {
  auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  return (g.A0 == g.A1 || g.k_split >= g.K) && g.lda0 % 8 == 0 && g.ldb % 8 == 0 &&
         g.lda0 >= (g.a_kmajor ? g.K : g.M) && g.ldb >= (g.b_kmajor ? g.K : g.N) && al16(g.A0) && al16(g.B) &&
         (splits <= 1 || g.k_per_split % tc::BK == 0) && encode_tiled() != nullptr;
}

// Persistent launch: two CTAs per SM (the shared memory of both fits), each
// looping over output tiles (per split-K part).
template <int BN, bool A_MN, bool B_MN>
inline void launch_tma(const tc::GemmArgs& g, const CUtensorMap& ta, const CUtensorMap& tb, dim3 grid,
                       cudaStream_t s) {
  const int smem = tc::gemm_tma_smem_bytes<BN>();
  auto k = tc::k_tc_gemm_tma<BN, A_MN, B_MN>;
  JC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k<<<grid, tc::TMA_THREADS, smem, s>>>(g, ta, tb);
}

template <int BN>
inline void gemm_tma(const tc::GemmArgs& g, int splits, cudaStream_t s) {
  CUtensorMap ta, tb;
  if (!tmap_operand(&ta, g.A0, g.M, g.K, g.lda0, tc::BM, g.a_kmajor) ||
      !tmap_operand(&tb, g.B, g.N, g.K, g.ldb, BN, g.b_kmajor))
    throw Error(JC_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  int dev = 0, sms = 0;
  JC_CUDA_CHECK(cudaGetDevice(&dev));
  JC_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const uint32_t tiles = cdiv(g.M, tc::BM) * cdiv(g.N, BN);
  const dim3 grid(std::min<uint32_t>(tiles, 2u * (uint32_t)sms), 1, (uint32_t)std::max(splits, 1));
  if (g.a_kmajor && g.b_kmajor) launch_tma<BN, false, false>(g, ta, tb, grid, s);
  else if (g.a_kmajor) launch_tma<BN, false, true>(g, ta, tb, grid, s);
  else if (g.b_kmajor) launch_tma<BN, true, false>(g, ta, tb, grid, s);
  else launch_tma<BN, true, true>(g, ta, tb, grid, s);
}

// Launch C (op)= A * B on the tensor cores; `splits` > 1 splits K across CTAs
// (each writes its own f32 partial at C + z * c_split_stride). Operands that
// the TMA-staged kernel takes go through it unless `staging` asks for the
// cp.async kernel; STAGE_TMA on operands it does not take is an argument error.
inline void gemm(const tc::GemmArgs& g, int splits, int bn, cudaStream_t s, int staging = STAGE_AUTO) {
  dim3 grid(cdiv(g.M, tc::BM), cdiv(g.N, bn), std::max(splits, 1));
  const bool tma = staging != STAGE_CP_ASYNC && tma_eligible(g, splits);
  if (staging == STAGE_TMA && !tma) throw Error(JC_ERR_ARG, "operands not eligible for the TMA-staged GEMM");
  if (tma) {
    if (bn == 256)
      gemm_tma<256>(g, splits, s);
    else
      gemm_tma<128>(g, splits, s);
  } else if (bn == 256) {
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

inline uint32_t warps_grid(uint64_t warps) { return cdiv(warps * 32, 256); }

// Reduction scratch shared by features, loss, hand-off and evaluation.
struct Reduce {
  Buf<double> vals, part, gsum, gsum2;
  void ensure(uint32_t nodes, uint32_t items, uint32_t graphs) {
    vals.alloc((size_t)nodes * 8);
    part.alloc((size_t)items * CEN);
    gsum.alloc((size_t)graphs * CEN);
    gsum2.alloc((size_t)graphs * 8);
  }
  // vals (V per local node) -> gsum (V per graph of the batch).
  template <int V>
  void run(const DevSet& s, const Batch& b, double* out, cudaStream_t st) {
    const uint32_t ni = b.i1 - b.i0, ng = b.g1 - b.g0;
    if (ni) k_item_reduce<V><<<warps_grid(ni), 256, 0, st>>>(vals.p, b.n0, s.items.p + b.i0, ni, part.p);
    if (ng) k_graph_sum<V><<<cdiv(ng, 128), 128, 0, st>>>(part.p, s.item_off.p, b.g0, ng, b.i0, out);
  }
};

// Features of every node of a set into X (n x 32 bf16). The projections are
// low-pass filtered by the lazy walk P x = (x + D^-1 A x) / 2: first
// cheb_steps steps of the Chebyshev recurrence for the interval [0, cheb_b]
// of P's spectrum (y1 = (2/b) P y0 - y0, y_{k+1} = (4/b) P y_k - 2 y_k -
// y_{k-1}: modes below b stay bounded while the slow modes above it grow like
// cosh(k acosh(2 lambda / b - 1)), the filtering of hundreds of plain steps
// in tens), then smooth_steps plain lazy steps (which separate the slowest
// modes of small graphs, whose whole spectrum may lie below b). Centring and
// rescaling before, every RECENTER steps of each phase, and at the end.
void compute_features(const DevSet& s, uint64_t seed, uint32_t smooth_steps, uint32_t cheb_steps, float cheb_b,
                      Buf<bf16>& X, Buf<float>& P, Buf<float>& P2, Buf<float>& P3, Reduce& red, Reduce& red2,
                      cudaStream_t st) {
  const uint32_t n = s.h.n;
  X.alloc((size_t)n * FEAT);
  P.alloc((size_t)n * NPROJ);
  P2.alloc((size_t)n * NPROJ);
  if (cheb_steps) P3.alloc((size_t)n * NPROJ);
  const Batch all = s.batch(0, s.h.G);
  const GView v = s.view(all);
  red.ensure(n, (uint32_t)s.h.items.size(), s.h.G);
  if (cheb_steps) red2.ensure(n, (uint32_t)s.h.items.size(), s.h.G);
  if (n == 0) return;
  k_features<<<warps_grid(n), 256, 0, st>>>(v, seed, X.p, P.p);
  const uint32_t ni = (uint32_t)s.h.items.size(), G = s.h.G;
  auto sums = [&](const float* x, Reduce& r) {
    k_proj_center_sums<<<warps_grid(ni), 256, 0, st>>>(x, s.deg.p, s.items.p, ni, r.part.p);
    k_graph_sum<CEN><<<cdiv(G, 128), 128, 0, st>>>(r.part.p, s.item_off.p, 0, G, 0, r.gsum.p);
  };
  auto center = [&](float* x) {
    sums(x, red);
    k_proj_center<<<cdiv((uint64_t)n * 8, 256), 256, 0, st>>>(v, red.gsum.p, x);
  };
  const uint32_t n_hubs = (uint32_t)s.h.hubs.size();
  float* a = P.p;
  float* b = P2.p;
  center(a);
  if (cheb_steps) {
    // a = y_{k-1}, b = y_k, c = y_{k+1}
    float* c = P3.p;
    const float c1_first = 2.0f / cheb_b, c1 = 4.0f / cheb_b;
    k_smooth<1><<<cdiv(n, 256), 256, 0, st>>>(v, a, b, nullptr, c1_first);
    if (n_hubs) k_smooth_hub<1><<<n_hubs, 256, 0, st>>>(v, s.hubs.p, a, b, nullptr, c1_first);
    for (uint32_t r = 1; r < cheb_steps; ++r) {
      if (r % RECENTER == 0) {
        sums(b, red);
        sums(a, red2);
        k_proj_center_pair<<<cdiv((uint64_t)n * 8, 256), 256, 0, st>>>(v, red.gsum.p, red2.gsum.p, b, a);
      }
      k_smooth<2><<<cdiv(n, 256), 256, 0, st>>>(v, b, c, a, c1);
      if (n_hubs) k_smooth_hub<2><<<n_hubs, 256, 0, st>>>(v, s.hubs.p, b, c, a, c1);
      float* t = a;
      a = b;
      b = c;
      c = t;
    }
    std::swap(a, b);  // the last y_k is the input of the plain phase
    center(a);
  }
  for (uint32_t r = 0; r < smooth_steps; ++r) {
    k_smooth<0><<<cdiv(n, 256), 256, 0, st>>>(v, a, b, nullptr, 1.0f);
    if (n_hubs) k_smooth_hub<0><<<n_hubs, 256, 0, st>>>(v, s.hubs.p, a, b, nullptr, 1.0f);
    std::swap(a, b);
    if (r % RECENTER == RECENTER - 1) center(a);
  }
  center(a);
  k_proj_write<<<cdiv((uint64_t)n * 8, 256), 256, 0, st>>>(v, a, X.p);
  JC_CUDA_CHECK(cudaGetLastError());
}

struct Hyper {
  float lr = 1e-3f, beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f, clip = 1.0f;
  uint32_t partners = 8, batch_nodes = 1u << 19, smooth_steps = 64, cheb_steps = 64;
  float cheb_b = 0.993f;
  float scaling_ratio = 2.0f, gravity = 1.0f;
};

class Net {
 public:
  Net(int dim, uint64_t seed) : dim_(dim), seed_(seed), L_(param_layout()) {
    if (dim != 2 && dim != 3) fail(JC_ERR_ARG, "dim must be 2 or 3");
    JC_CUDA_CHECK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    JC_CUDA_CHECK(cudaEventCreate(&ev0_));
    JC_CUDA_CHECK(cudaEventCreate(&ev1_));
    JC_CUDA_CHECK(cudaEventCreate(&evf_));
    JC_CUDA_CHECK(cudaEventCreate(&evn_));
    theta_.alloc(L_.total);
    theta_bf_.alloc(L_.total);
    wt_.alloc(L_.total);
    grad_.alloc(L_.total);
    m_.alloc(L_.total);
    v_.alloc(L_.total);
    err_.alloc(1);
    norm2_.alloc(1);
    grad_.zero(st_);
    err_.zero(st_);
    init_weights();
  }
  ~Net() {
    if (st_) cudaStreamSynchronize(st_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (evf_) cudaEventDestroy(evf_);
    if (evn_) cudaEventDestroy(evn_);
    if (st_) cudaStreamDestroy(st_);
  }

  static size_t num_params() { return param_layout().total; }

  void set_params(const char* json) {
    std::map<std::string, JsonValue> m;
    if (parse_object(json, &m, "mpnn")) return;
    Hyper t;
    FieldReader r{m, "decode mpnn settings"};
    r.f32("lr", &t.lr);
    r.f32("beta1", &t.beta1);
    r.f32("beta2", &t.beta2);
    r.f32("eps", &t.eps);
    r.f32("clip", &t.clip);
    r.u32("partners", &t.partners);
    r.u32("batch_nodes", &t.batch_nodes);
    r.u32("smooth_steps", &t.smooth_steps);
    r.u32("cheb_steps", &t.cheb_steps);
    r.f32("cheb_b", &t.cheb_b);
    r.f32("scaling_ratio", &t.scaling_ratio);
    r.f32("gravity", &t.gravity);
    if (!(t.lr > 0.0f) || t.batch_nodes == 0 || t.partners > 256 || t.smooth_steps > 4096 || t.cheb_steps > 4096 ||
        !(t.cheb_b > 0.0f && t.cheb_b <= 1.0f))
      fail(JC_ERR_PARAMS,
           "decode mpnn settings: lr > 0, batch_nodes > 0, partners <= 256, smooth_steps <= 4096, cheb_steps <= 4096 "
           "and 0 < cheb_b <= 1 are required");
    hp_ = t;
    if (data_.h.G) make_batches();
  }

  void get_weights(float* out) {
    JC_CUDA_CHECK(cudaMemcpyAsync(out, theta_.p, L_.total * 4, cudaMemcpyDeviceToHost, st_));
    JC_CUDA_CHECK(cudaStreamSynchronize(st_));
  }
  void set_weights(const float* w) {
    JC_CUDA_CHECK(cudaMemcpyAsync(theta_.p, w, L_.total * 4, cudaMemcpyHostToDevice, st_));
    k_to_bf16<<<cdiv(L_.total, 256), 256, 0, st_>>>(theta_.p, (uint32_t)L_.total, theta_bf_.p);
    JC_CUDA_CHECK(cudaStreamSynchronize(st_));
  }

  void bind(uint32_t G, const uint32_t* graph_nodes, const uint32_t* offsets, const uint32_t* neighbors,
            const float* target_xyz) {
    HostSet hs = assemble(G, graph_nodes, offsets, neighbors, true);
    if (!target_xyz && hs.n) fail(JC_ERR_ARG, "target positions must be non-null");
    std::vector<float4> t(hs.n);
    for (uint32_t i = 0; i < hs.n; ++i)
      t[i] = make_float4(target_xyz[3 * (size_t)i], target_xyz[3 * (size_t)i + 1],
                         dim_ == 3 ? target_xyz[3 * (size_t)i + 2] : 0.0f, 0.0f);
    data_.upload(std::move(hs), st_);
    T_.upload(t.data(), t.size(), st_);
    compute_features(data_, seed_, hp_.smooth_steps, hp_.cheb_steps, hp_.cheb_b, X_, P_, P2_, P3_, red_, red2_, st_);
    make_batches();
    JC_CUDA_CHECK(cudaStreamSynchronize(st_));
  }

  uint32_t n_batches() const { return (uint32_t)batches_.size(); }

  void features(float* out) {
    require_bound();
    std::vector<uint16_t> raw((size_t)data_.h.n * FEAT);
    JC_CUDA_CHECK(cudaMemcpyAsync(raw.data(), X_.p, raw.size() * 2, cudaMemcpyDeviceToHost, st_));
    JC_CUDA_CHECK(cudaStreamSynchronize(st_));
    for (size_t k = 0; k < raw.size(); ++k) {
      const uint32_t u = (uint32_t)raw[k] << 16;
      std::memcpy(&out[k], &u, 4);
    }
  }

  void train(uint32_t steps, float* losses) {
    require_bound();
    if (steps == 0) return;
    loss_dev_.alloc(steps);
    for (uint32_t s = 0; s < steps; ++s) {
      if (epoch_pos_ == 0) shuffle_order();
      const Batch& b = batches_[order_[epoch_pos_]];
      step_on(data_, b, X_.p, opt_step_, loss_dev_.p + s, true);
      ++opt_step_;
      if (++epoch_pos_ == batches_.size()) {
        epoch_pos_ = 0;
        ++epoch_;
      }
    }
    std::vector<float> l(steps);
    JC_CUDA_CHECK(cudaMemcpyAsync(l.data(), loss_dev_.p, steps * 4, cudaMemcpyDeviceToHost, st_));
    JC_CUDA_CHECK(cudaStreamSynchronize(st_));
    check_err();
    if (losses) std::memcpy(losses, l.data(), steps * 4);
  }

  // Mean batch loss over all batches of the bound set (no update; partners
  // drawn for optimiser step 0).
  double eval_loss() {
    require_bound();
    loss_dev_.alloc(batches_.size());
    for (size_t k = 0; k < batches_.size(); ++k)
      step_on(data_, batches_[k], X_.p, 0, loss_dev_.p + k, false, false);
    std::vector<float> l(batches_.size());
    JC_CUDA_CHECK(cudaMemcpyAsync(l.data(), loss_dev_.p, l.size() * 4, cudaMemcpyDeviceToHost, st_));
    JC_CUDA_CHECK(cudaStreamSynchronize(st_));
    check_err();
    double s = 0.0;
    for (float x : l) s += x;
    return l.empty() ? 0.0 : s / (double)l.size();
  }

  // Forward + loss + backward on graphs [g0, g1) of the bound set, partners
  // drawn for optimiser step `pair_step`; no update. Outputs the loss, the
  // prediction (nb x 4) and the unclipped gradient (num_params).
  void grad(uint32_t g0, uint32_t g1, uint64_t pair_step, float* loss, float* y, float* g) {
    require_bound();
    if (g0 >= g1 || g1 > data_.h.G) fail(JC_ERR_ARG, "graph range out of bounds");
    const Batch b = data_.batch(g0, g1);
    loss_dev_.alloc(1);
    step_on(data_, b, X_.p, pair_step, loss_dev_.p, false, true);
    if (loss) JC_CUDA_CHECK(cudaMemcpyAsync(loss, loss_dev_.p, 4, cudaMemcpyDeviceToHost, st_));
    if (y) JC_CUDA_CHECK(cudaMemcpyAsync(y, Y_.p, (size_t)b.nb * 16, cudaMemcpyDeviceToHost, st_));
    if (g) JC_CUDA_CHECK(cudaMemcpyAsync(g, grad_.p, L_.total * 4, cudaMemcpyDeviceToHost, st_));
    JC_CUDA_CHECK(cudaStreamSynchronize(st_));
    check_err();
  }

  // Features, forward and hand-off scale for new graphs; device time of those
  // three stages in *ms (the CSR upload is outside it).
  void predict(uint32_t G, const uint32_t* graph_nodes, const uint32_t* offsets, const uint32_t* neighbors,
               float* out_xyz, float* ms) {
    HostSet hs = assemble(G, graph_nodes, offsets, neighbors, true);
    if (hs.n && !out_xyz) fail(JC_ERR_ARG, "out_xyz must be non-null");
    predict_device(std::move(hs), ms);
    if (pred_.h.n) {
      JC_CUDA_CHECK(cudaMemcpyAsync(out_xyz, out_.p, (size_t)pred_.h.n * 12, cudaMemcpyDeviceToHost, st_));
      JC_CUDA_CHECK(cudaStreamSynchronize(st_));
    }
  }

  // Features, forward and hand-off of a graph set into out_ (3 floats per
  // node, device); returns with the stream drained.
  void predict_device(HostSet&& hs, float* ms) {
    pred_.upload(std::move(hs), st_);
    const uint32_t n = pred_.h.n, G = pred_.h.G;
    const Batch b = pred_.batch(0, G);
    ensure_work(b, false);
    red_.ensure(n, (uint32_t)pred_.h.items.size(), G);
    out_.alloc((size_t)n * 3);
    gscale_.alloc(G);
    JC_CUDA_CHECK(cudaEventRecord(ev0_, st_));
    compute_features(pred_, seed_, hp_.smooth_steps, hp_.cheb_steps, hp_.cheb_b, PX_, P_, P2_, P3_, red_, red2_,
                     st_);
    JC_CUDA_CHECK(cudaEventRecord(evf_, st_));
    if (n) forward(pred_, b, PX_.p);
    JC_CUDA_CHECK(cudaEventRecord(evn_, st_));
    if (n) hand_off(pred_, b);
    JC_CUDA_CHECK(cudaEventRecord(ev1_, st_));
    JC_CUDA_CHECK(cudaStreamSynchronize(st_));
    check_err();
    float t = 0.0f;
    JC_CUDA_CHECK(cudaEventElapsedTime(&t, ev0_, ev1_));
    JC_CUDA_CHECK(cudaEventElapsedTime(&stage_ms_[0], ev0_, evf_));
    JC_CUDA_CHECK(cudaEventElapsedTime(&stage_ms_[1], evf_, evn_));
    JC_CUDA_CHECK(cudaEventElapsedTime(&stage_ms_[2], evn_, ev1_));
    if (ms) *ms = t;
  }

  const float* predicted() const { return out_.p; }
  uint32_t predicted_nodes() const { return pred_.h.n; }

  // Device ms of the last predict's stages: features, network, hand-off scale.
  void predict_stages(float* ms3) const { std::memcpy(ms3, stage_ms_, sizeof stage_ms_); }

  // Checkpoint: header, weights, Adam moments.
  struct Header {
    uint64_t magic, version, dim, total, opt_step, epoch, epoch_pos, seed;
  };
  static constexpr uint64_t kMagic = 0x4A434D504E4E0001ull;
  uint64_t state_size() const { return sizeof(Header) + 3 * L_.total * 4; }
  void save_state(void* buf) {
    Header h{kMagic, 1, (uint64_t)dim_, L_.total, opt_step_, epoch_, epoch_pos_, seed_};
    uint8_t* p = static_cast<uint8_t*>(buf);
    std::memcpy(p, &h, sizeof h);
    p += sizeof h;
    JC_CUDA_CHECK(cudaMemcpyAsync(p, theta_.p, L_.total * 4, cudaMemcpyDeviceToHost, st_));
    JC_CUDA_CHECK(cudaMemcpyAsync(p + L_.total * 4, m_.p, L_.total * 4, cudaMemcpyDeviceToHost, st_));
    JC_CUDA_CHECK(cudaMemcpyAsync(p + 2 * L_.total * 4, v_.p, L_.total * 4, cudaMemcpyDeviceToHost, st_));
    JC_CUDA_CHECK(cudaStreamSynchronize(st_));
  }
  void load_state(const void* buf, uint64_t len) {
    if (len != state_size()) fail(JC_ERR_ARG, "state size mismatch");
    Header h;
    std::memcpy(&h, buf, sizeof h);
    if (h.magic != kMagic || h.version != 1 || h.dim != (uint64_t)dim_ || h.total != L_.total)
      fail(JC_ERR_ARG, "state does not belong to a network of this shape");
    const uint8_t* p = static_cast<const uint8_t*>(buf) + sizeof h;
    JC_CUDA_CHECK(cudaMemcpyAsync(theta_.p, p, L_.total * 4, cudaMemcpyHostToDevice, st_));
    JC_CUDA_CHECK(cudaMemcpyAsync(m_.p, p + L_.total * 4, L_.total * 4, cudaMemcpyHostToDevice, st_));
    JC_CUDA_CHECK(cudaMemcpyAsync(v_.p, p + 2 * L_.total * 4, L_.total * 4, cudaMemcpyHostToDevice, st_));
    k_to_bf16<<<cdiv(L_.total, 256), 256, 0, st_>>>(theta_.p, (uint32_t)L_.total, theta_bf_.p);
    JC_CUDA_CHECK(cudaStreamSynchronize(st_));
    opt_step_ = h.opt_step;
    epoch_ = h.epoch;
    epoch_pos_ = h.epoch_pos < batches_.size() ? h.epoch_pos : 0;
    seed_ = h.seed;
    if (data_.h.G && epoch_pos_) shuffle_order_for(epoch_);
  }

  std::string last_error;

 private:
  void require_bound() const {
    if (data_.h.G == 0) fail(JC_ERR_STATE, "no graphs bound (call jc_mpnn_bind first)");
  }

  void check_err() {
    uint32_t e = 0;
    JC_CUDA_CHECK(cudaMemcpy(&e, err_.p, 4, cudaMemcpyDeviceToHost));
    if (e) {
      JC_CUDA_CHECK(cudaMemset(err_.p, 0, 4));
      fail(JC_ERR_DEVICE_TIMEOUT, "a tensor-core GEMM gave up waiting on its pipeline");
    }
  }

  void init_weights() {
    std::vector<float> w(L_.total, 0.0f);
    SplitMix64 r(seed_ ^ SALT_INIT);
    for (int l = 0; l < 3; ++l) {
      const float a = std::sqrt(6.0f / (float)L_.kin[l]);
      for (size_t k = 0; k < (size_t)L_.kin[l] * HID; ++k) w[L_.w[l] + k] = (2.0f * r.next_f32() - 1.0f) * a;
    }
    const float ah = std::sqrt(3.0f / (float)HID);
    for (int k = 0; k < HID; ++k)
      for (int c = 0; c < 4; ++c) w[L_.wh + k * 4 + c] = c < dim_ ? (2.0f * r.next_f32() - 1.0f) * ah : 0.0f;
    m_.zero(st_);
    v_.zero(st_);
    set_weights(w.data());
  }

  void make_batches() {
    batches_.clear();
    uint32_t g0 = 0;
    const uint32_t G = data_.h.G;
    while (g0 < G) {
      uint32_t g1 = g0 + 1;
      while (g1 < G && data_.h.go[g1 + 1] - data_.h.go[g0] <= hp_.batch_nodes) ++g1;
      batches_.push_back(data_.batch(g0, g1));
      g0 = g1;
    }
    epoch_pos_ = 0;
  }

  void shuffle_order_for(uint64_t epoch) {
    order_.resize(batches_.size());
    for (size_t k = 0; k < order_.size(); ++k) order_[k] = (uint32_t)k;
    SplitMix64 r(seed_ ^ SALT_ORDER ^ (epoch * kSplitMixGamma));
    for (size_t k = order_.size(); k > 1; --k) std::swap(order_[k - 1], order_[r.below(k)]);
  }
  void shuffle_order() { shuffle_order_for(epoch_); }

  void ensure_work(const Batch& b, bool train) {
    const size_t nb = std::max<uint32_t>(b.nb, 1);
    A0_.alloc(nb * 2 * FEAT);
    A1_.alloc(nb * 2 * HID);
    A2_.alloc(nb * 2 * HID);
    H3_.alloc(nb * HID);
    Y_.alloc(nb);
    const uint32_t ng = b.g1 - b.g0;
    galpha_.alloc(ng);
    gcoef_.alloc(ng);
    if (train) {
      dY_.alloc(nb);
      dZ_.alloc(nb * HID);
      dA_.alloc(nb * 2 * HID);
      wpart_.alloc((size_t)kMaxSplits * 2 * HID * HID);
      cpart_.alloc((size_t)cdiv(nb, kChunk) * HEAD_W);
    }
  }

  // rows per block of the chunked column sums (head weights, biases): small
  // enough that the blocks fill the GPU, each thread's row loop is serial
  static constexpr uint32_t kChunk = 256;
  // split-K CTAs of a weight-gradient GEMM: three 64 KB CTAs per SM
  static constexpr int kMaxSplits = 3 * 148;

  tc::GemmArgs gemm_args() const {
    tc::GemmArgs g{};
    g.k_split = 1 << 30;
    g.err = err_.p;
    return g;
  }

  void forward(const DevSet& s, const Batch& b, const bf16* X) {
    const GView v = s.view(b);
    const uint32_t nb = b.nb, nh = b.h1 - b.h0;
    const uint32_t* hubs = s.hubs.p + b.h0;
    const bf16* Xb = X + (size_t)b.n0 * FEAT;
    const size_t n_w = (size_t)(L_.kin[0] + L_.kin[1] + L_.kin[2]) * HID;
    k_transpose_w<<<cdiv(n_w, 256), 256, 0, st_>>>(theta_bf_.p, L_, wt_.p);
    k_agg<FEAT><<<cdiv((uint64_t)nb * (FEAT / 4), 256), 256, 0, st_>>>(v, Xb, FEAT, A0_.p, 2 * FEAT, 1);
    if (nh) k_agg_hub<FEAT><<<nh, 256, 0, st_>>>(v, hubs, Xb, FEAT, A0_.p, 2 * FEAT);
    bf16* A[3] = {A0_.p, A1_.p, A2_.p};
    for (int l = 0; l < 3; ++l) {
      tc::GemmArgs g = gemm_args();
      g.A0 = g.A1 = A[l];
      g.lda0 = g.lda1 = L_.kin[l];
      g.a_kmajor = true;
      g.B = wt_.p + L_.w[l];
      g.ldb = L_.kin[l];
      g.b_kmajor = true;
      g.M = (int)nb;
      g.N = HID;
      g.K = L_.kin[l];
      g.k_per_split = L_.kin[l];
      g.C = l < 2 ? (void*)A[l + 1] : (void*)H3_.p;
      g.ldc = l < 2 ? 2 * HID : HID;
      g.epilogue = tc::EPI_BIAS_RELU_BF16;
      g.bias = theta_.p + L_.b[l];
      gemm(g, 1, HID, st_);
      if (l < 2) {
        k_agg<HID><<<cdiv((uint64_t)nb * (HID / 4), 256), 256, 0, st_>>>(v, A[l + 1], 2 * HID, A[l + 1], 2 * HID, 0);
        if (nh) k_agg_hub<HID><<<nh, 256, 0, st_>>>(v, hubs, A[l + 1], 2 * HID, A[l + 1], 2 * HID);
      }
    }
    k_head<<<cdiv(nb, 256), 256, 0, st_>>>(nb, H3_.p, theta_bf_.p + L_.wh, theta_.p + L_.bh, dim_, Y_.p);
    JC_CUDA_CHECK(cudaGetLastError());
  }

  // One batch: forward, loss; with `backward`, gradients; with `update`, Adam.
  void step_on(const DevSet& s, const Batch& b, const bf16* X, uint64_t pair_step, float* loss_slot, bool update,
               bool backward = true) {
    if (b.nb == 0) {  // a batch of empty graphs: no pairs, zero loss and gradient
      JC_CUDA_CHECK(cudaMemsetAsync(loss_slot, 0, 4, st_));
      if (backward) grad_.zero(st_);
      return;
    }
    ensure_work(b, backward);
    red_.ensure(b.nb, b.i1 - b.i0, b.g1 - b.g0);
    const GView v = s.view(b);
    const uint32_t nb = b.nb, ng = b.g1 - b.g0, nh = b.h1 - b.h0;
    const uint32_t* hubs = s.hubs.p + b.h0;
    forward(s, b, X);
    PairCtx pc{v, T_.p, Y_.p, hp_.partners, seed_, pair_step};
    k_loss_stats<<<warps_grid(nb), 256, 0, st_>>>(pc, red_.vals.p);
    red_.run<3>(s, b, red_.gsum.p, st_);
    k_loss_finish<<<1, 256, 0, st_>>>(red_.gsum.p, ng, galpha_.p, gcoef_.p, loss_slot);
    if (!backward) return;
    k_loss_grad<<<warps_grid(nb), 256, 0, st_>>>(pc, galpha_.p, gcoef_.p, dY_.p);
    // head
    k_head_bwd<<<cdiv(nb, 256), 256, 0, st_>>>(nb, H3_.p, theta_bf_.p + L_.wh, dY_.p, dZ_.p);
    const uint32_t chunks = cdiv(nb, kChunk);
    k_head_wgrad<<<chunks, HID, 0, st_>>>(nb, kChunk, H3_.p, dY_.p, cpart_.p);
    k_reduce_parts<<<reduce_parts_blocks(HEAD_W), 256, 0, st_>>>(cpart_.p, chunks, HEAD_W, grad_.p + L_.wh);
    bf16* A[3] = {A0_.p, A1_.p, A2_.p};
    for (int l = 2; l >= 0; --l) {
      const int kin = L_.kin[l];
      const int mt = cdiv(kin, tc::BM);
      int splits = (int)std::min<uint32_t>(cdiv(nb, 256), (uint32_t)(kMaxSplits / mt));
      splits = std::max(splits, 1);
      tc::GemmArgs g = gemm_args();
      g.A0 = g.A1 = A[l];
      g.lda0 = g.lda1 = kin;
      g.a_kmajor = false;
      g.B = dZ_.p;
      g.ldb = HID;
      g.b_kmajor = false;
      g.M = kin;
      g.N = HID;
      g.K = (int)nb;
      g.k_per_split = (int)(cdiv(cdiv(nb, splits), tc::BK) * tc::BK);
      splits = (int)cdiv(nb, g.k_per_split);
      g.C = wpart_.p;
      g.ldc = HID;
      g.c_split_stride = (long long)kin * HID;
      g.epilogue = tc::EPI_STORE_F32;
      gemm(g, splits, HID, st_);
      k_reduce_splits<<<cdiv((uint64_t)kin * HID, 256), 256, 0, st_>>>(wpart_.p, (uint32_t)splits, kin * HID,
                                                                       grad_.p + L_.w[l]);
      k_colsum<<<chunks, HID, 0, st_>>>(nb, kChunk, dZ_.p, cpart_.p);
      k_reduce_parts<<<reduce_parts_blocks(HID), 256, 0, st_>>>(cpart_.p, chunks, HID, grad_.p + L_.b[l]);
      if (l == 0) break;
      tc::GemmArgs h = gemm_args();
      h.A0 = h.A1 = dZ_.p;
      h.lda0 = h.lda1 = HID;
      h.a_kmajor = true;
      h.B = theta_bf_.p + L_.w[l];
      h.ldb = HID;
      h.b_kmajor = true;
      h.M = (int)nb;
      h.N = kin;
      h.K = HID;
      h.k_per_split = HID;
      h.C = dA_.p;
      h.ldc = 2 * HID;
      h.c_split_stride = 0;
      h.epilogue = tc::EPI_STORE_BF16;
      gemm(h, 1, 256, st_);
      k_agg_bwd<<<warps_grid(nb), 256, 0, st_>>>(v, dA_.p, A[l], dZ_.p);
      if (nh) k_agg_bwd_hub<<<nh, 256, 0, st_>>>(v, hubs, dA_.p, A[l], dZ_.p);
    }
    JC_CUDA_CHECK(cudaGetLastError());
    if (!update) return;
    k_grad_norm<<<1, 1024, 0, st_>>>(grad_.p, (uint32_t)L_.total, norm2_.p);
    const double t = (double)(opt_step_ + 1);
    const double lr_t = hp_.lr * std::sqrt(1.0 - std::pow((double)hp_.beta2, t)) / (1.0 - std::pow((double)hp_.beta1, t));
    k_adam<<<cdiv(L_.total, 256), 256, 0, st_>>>(theta_.p, theta_bf_.p, grad_.p, m_.p, v_.p, (uint32_t)L_.total,
                                                 norm2_.p, hp_.clip, (float)lr_t, hp_.beta1, hp_.beta2, hp_.eps);
    JC_CUDA_CHECK(cudaGetLastError());
  }

  void hand_off(const DevSet& s, const Batch& b) {
    const GView v = s.view(b);
    const uint32_t nb = b.nb, ng = b.g1 - b.g0;
    k_scale_vals<<<warps_grid(nb), 256, 0, st_>>>(v, Y_.p, red_.vals.p);
    red_.run<6>(s, b, red_.gsum.p, st_);
    k_scale_grav<<<cdiv(nb, 256), 256, 0, st_>>>(v, Y_.p, red_.gsum.p, red_.vals.p);
    red_.run<1>(s, b, red_.gsum2.p, st_);
    k_scale_finish<<<cdiv(ng, 128), 128, 0, st_>>>(red_.gsum.p, red_.gsum2.p, s.go.p, b.g0, ng, hp_.scaling_ratio,
                                                   hp_.gravity, gscale_.p);
    k_scale_apply<<<cdiv(nb, 256), 256, 0, st_>>>(v, Y_.p, gscale_.p, dim_, out_.p);
    JC_CUDA_CHECK(cudaGetLastError());
  }

  int dim_;
  uint64_t seed_;
  ParamLayout L_;
  Hyper hp_;
  cudaStream_t st_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr, evf_ = nullptr, evn_ = nullptr;
  float stage_ms_[3] = {0.0f, 0.0f, 0.0f};
  Buf<float> theta_, grad_, m_, v_;
  Buf<bf16> theta_bf_, wt_;
  Buf<uint32_t> err_;
  Buf<double> norm2_;
  DevSet data_, pred_;
  Buf<bf16> X_, PX_;
  Buf<float> P_, P2_, P3_;
  Buf<float4> T_;
  std::vector<Batch> batches_;
  std::vector<uint32_t> order_;
  uint64_t opt_step_ = 0, epoch_ = 0, epoch_pos_ = 0;
  Buf<bf16> A0_, A1_, A2_, H3_, dZ_;
  Buf<float4> Y_, dY_;
  Buf<bf16> dA_;
  Buf<float> wpart_, loss_dev_, out_;
  Buf<double> cpart_, galpha_, gcoef_;
  Buf<float4> gscale_;
  Reduce red_, red2_;
};

// Pivot stress and edge-length spread of layouts of a fixed set of graphs.
class Evaluator {
 public:
  Evaluator(uint32_t G, const uint32_t* graph_nodes, const uint32_t* offsets, const uint32_t* neighbors, uint32_t k,
            uint64_t seed)
      : k_(k) {
    if (k == 0 || k > 1024) fail(JC_ERR_ARG, "n_pivots must be in 1..1024");
    JC_CUDA_CHECK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    HostSet hs = assemble(G, graph_nodes, offsets, neighbors, false);
    const uint32_t n = hs.n;
    // k distinct pivots per graph (all nodes when the graph is smaller).
    piv_h_.assign((size_t)G * k, NO_PIVOT);
    for (uint32_t g = 0; g < G; ++g) {
      const uint32_t b = hs.go[g], ng = hs.go[g + 1] - b, kg = std::min(k, ng);
      SplitMix64 r(seed ^ ((uint64_t)(g + 1) * kSplitMixGamma));
      uint32_t got = 0;
      while (got < kg) {
        const uint32_t c = b + (uint32_t)r.below(ng);
        bool dup = false;
        for (uint32_t q = 0; q < got; ++q) dup |= piv_h_[(size_t)g * k + q] == c;
        if (!dup) piv_h_[(size_t)g * k + got++] = c;
      }
    }
    // Breadth-first hop distances from every pivot inside its graph.
    std::vector<uint16_t> dist((size_t)n * k, NO_DIST);
    const int64_t tasks = (int64_t)G * k;
#pragma omp parallel
    {
      std::vector<uint32_t> queue;
#pragma omp for schedule(dynamic, 8)
      for (int64_t t = 0; t < tasks; ++t) {
        const uint32_t g = (uint32_t)(t / k), q = (uint32_t)(t % k);
        const uint32_t src = piv_h_[(size_t)g * k + q];
        if (src == NO_PIVOT) continue;
        queue.clear();
        queue.push_back(src);
        dist[(size_t)src * k + q] = 0;
        for (size_t head = 0; head < queue.size(); ++head) {
          const uint32_t u = queue[head];
          const uint16_t du = dist[(size_t)u * k + q];
          const uint16_t nd = du >= NO_DIST - 1 ? (uint16_t)(NO_DIST - 1) : (uint16_t)(du + 1);
          for (uint32_t e = hs.off[u]; e < hs.off[u + 1]; ++e) {
            const uint32_t x = hs.nbr[e];
            if (dist[(size_t)x * k + q] == NO_DIST) {
              dist[(size_t)x * k + q] = nd;
              queue.push_back(x);
            }
          }
        }
      }
    }
    set_.upload(std::move(hs), st_);
    piv_.upload(piv_h_.data(), piv_h_.size(), st_);
    dist_.upload(dist.data(), dist.size(), st_);
    JC_CUDA_CHECK(cudaStreamSynchronize(st_));
  }
  ~Evaluator() {
    if (st_) {
      cudaStreamSynchronize(st_);
      cudaStreamDestroy(st_);
    }
  }

  uint32_t n_graphs() const { return set_.h.G; }
  const std::vector<uint32_t>& pivots() const { return piv_h_; }

  void eval(const float* xyz, double* stress_g, double* cv_g, double* means) {
    const uint32_t n = set_.h.n;
    if (n && !xyz) fail(JC_ERR_ARG, "positions must be non-null");
    xyz_.upload(xyz, (size_t)n * 3, st_);
    eval_device(xyz_.p, stress_g, cv_g, means);
  }

  uint32_t n_nodes() const { return set_.h.n; }
  cudaStream_t stream() const { return st_; }
  // Same graph set as the arrays of a predict call (node counts and edges).
  bool same_graphs(const HostSet& hs) const {
    return hs.G == set_.h.G && hs.n == set_.h.n && hs.go == set_.h.go && hs.off == set_.h.off &&
           hs.nbr == set_.h.nbr;
  }

  // Evaluation of device positions (3 floats per node) on this stream.
  void eval_device(const float* d_xyz, double* stress_g, double* cv_g, double* means) {
    const uint32_t n = set_.h.n, G = set_.h.G;
    pos_.alloc(n);
    red_.ensure(n, (uint32_t)set_.h.items.size(), G);
    res_.alloc((size_t)G * 4);
    const Batch b = set_.batch(0, G);
    const GView v = set_.view(b);
    if (n) {
      k_xyz_to_f4<<<cdiv(n, 256), 256, 0, st_>>>(d_xyz, n, pos_.p);
      k_eval_vals<<<warps_grid(n), 256, 0, st_>>>(v, pos_.p, piv_.p, dist_.p, k_, red_.vals.p);
      red_.run<6>(set_, b, red_.gsum.p, st_);
    } else {
      red_.gsum.zero(st_);
    }
    k_eval_finish<<<cdiv(G, 128), 128, 0, st_>>>(red_.gsum.p, G, res_.p);
    JC_CUDA_CHECK(cudaGetLastError());
    std::vector<double> r((size_t)G * 4);
    JC_CUDA_CHECK(cudaMemcpyAsync(r.data(), res_.p, r.size() * 8, cudaMemcpyDeviceToHost, st_));
    JC_CUDA_CHECK(cudaStreamSynchronize(st_));
    double ms = 0.0, mc = 0.0;
    uint32_t ns = 0, nc = 0;
    for (uint32_t g = 0; g < G; ++g) {
      if (stress_g) stress_g[g] = r[(size_t)g * 4];
      if (cv_g) cv_g[g] = r[(size_t)g * 4 + 1];
      if (r[(size_t)g * 4 + 2] > 0.0) {
        ms += r[(size_t)g * 4];
        ++ns;
      }
      if (r[(size_t)g * 4 + 3] >= 2.0) {
        mc += r[(size_t)g * 4 + 1];
        ++nc;
      }
    }
    if (means) {
      means[0] = ns ? ms / ns : 0.0;
      means[1] = nc ? mc / nc : 0.0;
    }
  }

  std::string last_error;

 private:
  uint32_t k_;
  cudaStream_t st_ = nullptr;
  DevSet set_;
  std::vector<uint32_t> piv_h_;
  Buf<uint32_t> piv_;
  Buf<uint16_t> dist_;
  Buf<float> xyz_;
  Buf<float4> pos_;
  Buf<double> res_;
  Reduce red_;
};

// Guarded warm start: the prediction per graph only where its pivot stress
// is below the seed's, else the seed. Positions meet on the host once.
inline void warm_start(Net& net, Evaluator& ev, uint32_t G, const uint32_t* graph_nodes, const uint32_t* offsets,
                       const uint32_t* neighbors, const float* seed_xyz, float* out_xyz, uint8_t* kept,
                       float* device_ms) {
  HostSet hs = assemble(G, graph_nodes, offsets, neighbors, true);
  if (!ev.same_graphs(hs)) fail(JC_ERR_ARG, "the evaluator was built for other graphs");
  const uint32_t n = hs.n;
  if (n && (!seed_xyz || !out_xyz)) fail(JC_ERR_ARG, "seed_xyz and out_xyz must be non-null");
  const std::vector<uint32_t> go = hs.go;
  float pred_ms = 0.0f;
  net.predict_device(std::move(hs), &pred_ms);
  cudaEvent_t e0, e1;
  JC_CUDA_CHECK(cudaEventCreate(&e0));
  JC_CUDA_CHECK(cudaEventCreate(&e1));
  std::vector<double> s_pred(G), s_seed(G);
  float eval_ms = 0.0f;
  try {
    Buf<float> seed;
    seed.upload(seed_xyz, (size_t)n * 3, ev.stream());
    JC_CUDA_CHECK(cudaEventRecord(e0, ev.stream()));
    ev.eval_device(net.predicted(), s_pred.data(), nullptr, nullptr);
    ev.eval_device(seed.p, s_seed.data(), nullptr, nullptr);
    JC_CUDA_CHECK(cudaEventRecord(e1, ev.stream()));
    if (n) JC_CUDA_CHECK(cudaMemcpyAsync(out_xyz, net.predicted(), (size_t)n * 12, cudaMemcpyDeviceToHost,
                                         ev.stream()));
    JC_CUDA_CHECK(cudaStreamSynchronize(ev.stream()));
    JC_CUDA_CHECK(cudaEventElapsedTime(&eval_ms, e0, e1));
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (uint32_t g = 0; g < G; ++g) {
    const bool keep = s_pred[g] < s_seed[g];
    if (kept) kept[g] = keep ? 1 : 0;
    if (!keep)
      std::memcpy(out_xyz + 3 * (size_t)go[g], seed_xyz + 3 * (size_t)go[g],
                  3 * (size_t)(go[g + 1] - go[g]) * sizeof(float));
  }
  if (device_ms) *device_ms = pred_ms + eval_ms;
}

}  // namespace mpnn
}  // namespace jc

// ================================================================ C ABI ==
struct jc_mpnn {
  jc::mpnn::Net* net = nullptr;
  std::string last_error;
};

struct jc_eval {
  jc::mpnn::Evaluator* ev = nullptr;
  std::string last_error;
};

namespace {

template <typename H, typename F>
jc_status guarded_h(H* h, F&& f) {
  if (h == nullptr) return JC_ERR_ARG;
  try {
    f();
    h->last_error.clear();
    return JC_OK;
  } catch (const jc::Error& e) {
    h->last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    h->last_error = "host allocation failed";
    return JC_ERR_ARG;
  } catch (const std::exception& e) {
    h->last_error = e.what();
    return JC_ERR_ARG;
  }
}

}  // namespace

extern "C" {

jc_status jc_mpnn_create(int32_t dim, uint64_t seed, jc_mpnn** out) {
  if (!out) return JC_ERR_ARG;
  *out = nullptr;
  try {
    auto* h = new jc_mpnn;
    try {
      h->net = new jc::mpnn::Net(dim, seed);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return JC_OK;
  } catch (const jc::Error& e) {
    return e.code;
  } catch (...) {
    return JC_ERR_ARG;
  }
}

void jc_mpnn_destroy(jc_mpnn* m) {
  if (!m) return;
  delete m->net;
  delete m;
}

const char* jc_mpnn_last_error(const jc_mpnn* m) { return m ? m->last_error.c_str() : "null handle"; }

uint32_t jc_mpnn_num_params(void) { return (uint32_t)jc::mpnn::Net::num_params(); }

jc_status jc_mpnn_set_params(jc_mpnn* m, const char* json) {
  return guarded_h(m, [&] { m->net->set_params(json); });
}

jc_status jc_mpnn_get_weights(jc_mpnn* m, float* out) {
  return guarded_h(m, [&] {
    if (!out) jc::fail(JC_ERR_ARG, "out must be non-null");
    m->net->get_weights(out);
  });
}

jc_status jc_mpnn_set_weights(jc_mpnn* m, const float* w) {
  return guarded_h(m, [&] {
    if (!w) jc::fail(JC_ERR_ARG, "weights must be non-null");
    m->net->set_weights(w);
  });
}

jc_status jc_mpnn_bind(jc_mpnn* m, uint32_t n_graphs, const uint32_t* graph_nodes, const uint32_t* offsets,
                       const uint32_t* neighbors, const float* target_xyz) {
  return guarded_h(m, [&] { m->net->bind(n_graphs, graph_nodes, offsets, neighbors, target_xyz); });
}

jc_status jc_mpnn_batches(jc_mpnn* m, uint32_t* count) {
  return guarded_h(m, [&] {
    if (count) *count = m->net->n_batches();
  });
}

jc_status jc_mpnn_features(jc_mpnn* m, float* out) {
  return guarded_h(m, [&] {
    if (!out) jc::fail(JC_ERR_ARG, "out must be non-null");
    m->net->features(out);
  });
}

jc_status jc_mpnn_train(jc_mpnn* m, uint32_t steps, float* losses) {
  return guarded_h(m, [&] { m->net->train(steps, losses); });
}

jc_status jc_mpnn_eval_loss(jc_mpnn* m, double* loss) {
  return guarded_h(m, [&] {
    const double l = m->net->eval_loss();
    if (loss) *loss = l;
  });
}

jc_status jc_mpnn_grad(jc_mpnn* m, uint32_t g0, uint32_t g1, uint64_t pair_step, float* loss, float* y,
                       float* grad) {
  return guarded_h(m, [&] { m->net->grad(g0, g1, pair_step, loss, y, grad); });
}

jc_status jc_mpnn_predict(jc_mpnn* m, uint32_t n_graphs, const uint32_t* graph_nodes, const uint32_t* offsets,
                          const uint32_t* neighbors, float* out_xyz, float* device_ms) {
  return guarded_h(m, [&] { m->net->predict(n_graphs, graph_nodes, offsets, neighbors, out_xyz, device_ms); });
}

jc_status jc_mpnn_warm_start(jc_mpnn* m, jc_eval* ev, uint32_t n_graphs, const uint32_t* graph_nodes,
                             const uint32_t* offsets, const uint32_t* neighbors, const float* seed_xyz,
                             float* out_xyz, uint8_t* kept, float* device_ms) {
  return guarded_h(m, [&] {
    if (!ev) jc::fail(JC_ERR_ARG, "null evaluator");
    jc::mpnn::warm_start(*m->net, *ev->ev, n_graphs, graph_nodes, offsets, neighbors, seed_xyz, out_xyz, kept,
                         device_ms);
  });
}

jc_status jc_mpnn_predict_stages(jc_mpnn* m, float* ms3) {
  return guarded_h(m, [&] {
    if (!ms3) jc::fail(JC_ERR_ARG, "ms3 must be non-null");
    m->net->predict_stages(ms3);
  });
}

uint64_t jc_mpnn_state_size(const jc_mpnn* m) { return m ? m->net->state_size() : 0; }

jc_status jc_mpnn_save_state(jc_mpnn* m, void* buf) {
  return guarded_h(m, [&] {
    if (!buf) jc::fail(JC_ERR_ARG, "buf must be non-null");
    m->net->save_state(buf);
  });
}

jc_status jc_mpnn_load_state(jc_mpnn* m, const void* buf, uint64_t len) {
  return guarded_h(m, [&] {
    if (!buf) jc::fail(JC_ERR_ARG, "buf must be non-null");
    m->net->load_state(buf, len);
  });
}

jc_status jc_eval_create(uint32_t n_graphs, const uint32_t* graph_nodes, const uint32_t* offsets,
                         const uint32_t* neighbors, uint32_t n_pivots, uint64_t seed, jc_eval** out) {
  if (!out) return JC_ERR_ARG;
  *out = nullptr;
  try {
    auto* h = new jc_eval;
    try {
      h->ev = new jc::mpnn::Evaluator(n_graphs, graph_nodes, offsets, neighbors, n_pivots, seed);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return JC_OK;
  } catch (const jc::Error& e) {
    return e.code;
  } catch (...) {
    return JC_ERR_ARG;
  }
}

void jc_eval_destroy(jc_eval* e) {
  if (!e) return;
  delete e->ev;
  delete e;
}

const char* jc_eval_last_error(const jc_eval* e) { return e ? e->last_error.c_str() : "null handle"; }

jc_status jc_eval_pivots(jc_eval* e, uint32_t* out) {
  return guarded_h(e, [&] {
    if (!out) jc::fail(JC_ERR_ARG, "out must be non-null");
    const auto& p = e->ev->pivots();
    std::memcpy(out, p.data(), p.size() * 4);
  });
}

jc_status jc_eval_layout(jc_eval* e, const float* xyz, double* stress_per_graph, double* cv_per_graph,
                         double* means) {
  return guarded_h(e, [&] { e->ev->eval(xyz, stress_per_graph, cv_per_graph, means); });
}

}  // extern "C"

// Test entry point: C = A * B from host bf16 bit patterns (A: M x K row-major
// if a_kmajor else K x M row-major; B: N x K row-major if b_kmajor else K x N
// row-major), f32 result in C (M x N row-major, summed over split-K parts).
// staging: 0 automatic, 1 cp.async kernel, 2 TMA kernel (JC_ERR_ARG when the
// operands do not suit it).
extern "C" jc_status jc_tc_gemm_bf16(int32_t M, int32_t N, int32_t K, const uint16_t* a_bits, int32_t a_kmajor,
                                     const uint16_t* b_bits, int32_t b_kmajor, int32_t bn, int32_t splits,
                                     int32_t staging, float* c_out) {
  using namespace jc;
  if (M <= 0 || N <= 0 || K <= 0 || !a_bits || !b_bits || !c_out || (bn != 128 && bn != 256) || splits < 1 ||
      staging < 0 || staging > 2)
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
    try {
      mpnn::gemm(g, splits, bn, 0, staging);
    } catch (...) {
      cudaFree(dA);
      cudaFree(dB);
      cudaFree(dC);
      cudaFree(dErr);
      throw;
    }
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

namespace jc {
namespace tc {

// Failure-detection self-test of the GEMM's bounded mbarrier waits: one CTA
// set up exactly as k_tc_gemm sets itself up (tensor memory allocated by
// warp 0, one mbarrier initialised by thread 0) whose threads then wait on
// that barrier's first phase with mbar_wait. No tcgen05.commit is ever
// issued, so nothing arrives: every wait must give up after its bound (about
// a second of the global timer),
// the kernel records JC_ERR_DEVICE_TIMEOUT in the error word as k_tc_gemm
// does, frees its tensor memory and returns.
__global__ void __launch_bounds__(128) k_selftest_mbar_wait(uint32_t* err) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base_sh;
  const int warp = threadIdx.x >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(32u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  const bool ok = mbar_wait(&bar, 0u);
  if (!ok && threadIdx.x == 0) atomicCAS(err, 0u, (uint32_t)JC_ERR_DEVICE_TIMEOUT);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32u) : "memory");
  }
}

}  // namespace tc
}  // namespace jc

extern "C" jc_status jc_selftest_gemm_wait(uint32_t* device_status, float* wait_ms) {
  using namespace jc;
  if (!device_status) return JC_ERR_ARG;
  uint32_t* err = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  jc_status rc = JC_OK;
  try {
    JC_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    JC_CUDA_CHECK(cudaMalloc(&err, 4));
    JC_CUDA_CHECK(cudaMemsetAsync(err, 0, 4, s));
    JC_CUDA_CHECK(cudaEventCreate(&e0));
    JC_CUDA_CHECK(cudaEventCreate(&e1));
    JC_CUDA_CHECK(cudaEventRecord(e0, s));
    tc::k_selftest_mbar_wait<<<1, 128, 0, s>>>(err);
    JC_CUDA_CHECK(cudaGetLastError());
    JC_CUDA_CHECK(cudaEventRecord(e1, s));
    JC_CUDA_CHECK(cudaMemcpyAsync(device_status, err, 4, cudaMemcpyDeviceToHost, s));
    JC_CUDA_CHECK(cudaStreamSynchronize(s));
    float ms = 0.0f;
    JC_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    if (wait_ms) *wait_ms = ms;
  } catch (const Error& ex) {
    rc = ex.code;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (err) cudaFree(err);
  if (s) cudaStreamDestroy(s);
  return rc;
}
