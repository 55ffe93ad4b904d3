// SGD pivot-stress layout on B200: "sgd-stress-gpu" (Jacobi move-self) and
// "sgd-stress" (per-pair scatter that moves both endpoints).
//
// Reference behaviour (paths in the jump-cannon repo):
//   crates/graph-compute/src/engines/sgd_stress.rs       settings, SplitMix64,
//       select_pivots :143-175, step :275-318, anneal_eta :324-334,
//       sgd_pair_update :340-366, bfs_distances :372-394
//   crates/graph-compute/src/engines/sgd_stress_gpu.rs   init :165-366, step :368-449
//   crates/graph-compute/src/shaders/sgd_stress.wgsl     sgd_step :34-62
//
// Pivot selection and the per-pivot BFS stay on the host at init, as in the
// reference (a device BFS is future work). Distances are stored pivot-major
// (dist[t * n + i]) so that the threads of a warp, one node each, read one
// contiguous row per pivot; u16 when every finite distance fits, else u32,
// with the all-ones value as "unreachable".
//
// Jacobi sweep (sgd_stress.wgsl): node i walks its k pivots in order against
// the start-of-sweep positions; pivot positions are staged in shared memory.
// Bit-identical to the shader's arithmetic (IEEE ops in source order).
//
// Per-pair scatter (sgd_stress.rs semantics on a GPU): the CPU engine draws
// n (node, pivot) samples per sweep from one SplitMix64 stream and moves both
// endpoints sequentially. SplitMix64 is counter based, so sample q of the run
// is computed directly from the stream position; the GPU draws exactly the
// reference's samples. A sweep is split into batches; inside a batch every
// pair update is evaluated against the batch-start positions and the two
// endpoint moves are accumulated in 64-bit fixed point with integer atomics
// (order-independent, so the result is deterministic). Each node then moves
// by the mean of its accumulated moves: a pivot takes part in ~n/(k*batches)
// pairs per batch and summing them would overshoot, averaging keeps each
// pivot's move the size of one pair update. Like the CPU engine it is a
// stochastic method: from the same seed it does not follow the sequential
// trajectory, and it is judged by the stress it converges to.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "jc_common.h"
#include "jc_engine.h"
#include "jc_params.h"

namespace jc {
namespace sgd {

constexpr uint32_t UNREACH = 0xFFFFFFFFu;
constexpr double FIX_SCALE = 4294967296.0;  // 2^32: fixed-point scale of pair moves

__device__ __forceinline__ float len3(float x, float y, float z) {
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
}

__device__ __forceinline__ uint64_t smix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <typename D>
__device__ __forceinline__ float dist_value(D du) {
  // sgd_stress_gpu.rs:203-207: unreachable or self -> 0.0 (skipped)
  const D sent = (D)~(D)0;
  return (du == sent || du == 0) ? 0.0f : (float)du;
}

// One Jacobi sweep (sgd_stress.wgsl:34-62). eta_idx points at the step's
// sweep counter; eta comes from the host-computed schedule table.
template <typename D>
__global__ void __launch_bounds__(256)
k_jacobi(const float4* __restrict__ pin, float4* __restrict__ pout, const uint32_t* __restrict__ pivots,
         const D* __restrict__ dist, uint32_t n, uint32_t k, const float* __restrict__ eta_table, uint32_t n_eta,
         const uint32_t* __restrict__ sweep_ctr, uint32_t mu_len) {
  extern __shared__ float4 piv[];
  // mu = min(1, eta / d^2) depends only on the hop distance d and this sweep's
  // eta: with mu_len > 0 it is tabulated for d < mu_len (the same operations
  // as below, once per block), which takes one IEEE division per term out of
  // the serial chain
  float* mu_tab = reinterpret_cast<float*>(piv + k);
  const uint32_t sw = *sweep_ctr;
  const float eta = eta_table[sw < n_eta ? sw : n_eta - 1];
  for (uint32_t t = threadIdx.x; t < k; t += blockDim.x) {
    float4 q = pin[pivots[t]];
    piv[t] = make_float4(q.x, q.y, q.z, __uint_as_float(pivots[t]));
  }
  for (uint32_t du = threadIdx.x; du < mu_len; du += blockDim.x) {
    const float d = (float)du;
    mu_tab[du] = fminf(1.0f, __fmul_rn(__fdiv_rn(1.0f, __fmul_rn(d, d)), eta));
  }
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p4 = pin[i];
  float px = p4.x, py = p4.y, pz = p4.z;
  // The position update is a serial chain over the pivots; the distances do
  // not depend on it, so JACOBI_PF of them are loaded ahead (in flight
  // together) instead of one exposed load per pivot. Same operations, same
  // order.
  constexpr uint32_t JACOBI_PF = 8;
  for (uint32_t t0 = 0; t0 < k; t0 += JACOBI_PF) {
    D dv[JACOBI_PF];
#pragma unroll
    for (uint32_t u = 0; u < JACOBI_PF; ++u) dv[u] = t0 + u < k ? dist[(size_t)(t0 + u) * n + i] : (D)0;
#pragma unroll
    for (uint32_t u = 0; u < JACOBI_PF; ++u) {
      const uint32_t t = t0 + u;
      if (t >= k) break;
      const float4 q = piv[t];
      if (__float_as_uint(q.w) == i) continue;
      const float d = dist_value<D>(dv[u]);
      if (d <= 0.0f) continue;
      const float ex = __fsub_rn(px, q.x), ey = __fsub_rn(py, q.y), ez = __fsub_rn(pz, q.z);
      const float mag = fmaxf(len3(ex, ey, ez), 1e-6f);
      const float mu = (uint32_t)dv[u] < mu_len ? mu_tab[(uint32_t)dv[u]]
                                                 : fminf(1.0f, __fmul_rn(__fdiv_rn(1.0f, __fmul_rn(d, d)), eta));
      const float r = __fdiv_rn(__fmul_rn(mu, __fsub_rn(mag, d)), mag);
      px = __fsub_rn(px, __fmul_rn(r, ex));
      py = __fsub_rn(py, __fmul_rn(r, ey));
      pz = __fsub_rn(pz, __fmul_rn(r, ez));
    }
  }
  pout[i] = make_float4(px, py, pz, 0.0f);
}

// One batch of the per-pair scatter. Sample q = sweep * n + q0 + t.
template <typename D>
__global__ void __launch_bounds__(256)
k_pairs(const float4* __restrict__ pos, long long* __restrict__ acc, uint32_t* __restrict__ cnt,
        const uint32_t* __restrict__ pivots, const D* __restrict__ dist, uint32_t n, uint32_t k, uint64_t s0,
        uint32_t q0, uint32_t count, const float* __restrict__ eta_table, uint32_t n_eta,
        const uint32_t* __restrict__ sweep_ctr) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const uint32_t sw = *sweep_ctr;
  const float eta = eta_table[sw < n_eta ? sw : n_eta - 1];
  const uint64_t q = (uint64_t)sw * n + q0 + t;
  const uint64_t G = 0x9E3779B97F4A7C15ull;
  const uint32_t i = (uint32_t)(smix(s0 + (2 * q + 1) * G) % n);
  const uint32_t pidx = (uint32_t)(smix(s0 + (2 * q + 2) * G) % k);
  const uint32_t j = pivots[pidx];
  if (i == j) return;
  const D du = dist[(size_t)pidx * n + i];
  const D sent = (D)~(D)0;
  if (du == sent || du == 0) return;
  const float d = (float)du;
  const float4 a = pos[i], b = pos[j];
  const float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y), dz = __fsub_rn(a.z, b.z);
  const float mag = fmaxf(len3(dx, dy, dz), 1e-6f);
  const float w = __fdiv_rn(1.0f, __fmul_rn(d, d));
  const float mu = fminf(__fmul_rn(w, eta), 1.0f);
  const float r = __fdiv_rn(__fmul_rn(__fmul_rn(0.5f, mu), __fsub_rn(mag, d)), mag);
  const float rx = __fmul_rn(r, dx), ry = __fmul_rn(r, dy), rz = __fmul_rn(r, dz);
  const long long fx = __double2ll_rn((double)rx * FIX_SCALE);
  const long long fy = __double2ll_rn((double)ry * FIX_SCALE);
  const long long fz = __double2ll_rn((double)rz * FIX_SCALE);
  atomicAdd((unsigned long long*)&acc[3 * (size_t)i], (unsigned long long)(-fx));
  atomicAdd((unsigned long long*)&acc[3 * (size_t)i + 1], (unsigned long long)(-fy));
  atomicAdd((unsigned long long*)&acc[3 * (size_t)i + 2], (unsigned long long)(-fz));
  atomicAdd((unsigned long long*)&acc[3 * (size_t)j], (unsigned long long)fx);
  atomicAdd((unsigned long long*)&acc[3 * (size_t)j + 1], (unsigned long long)fy);
  atomicAdd((unsigned long long*)&acc[3 * (size_t)j + 2], (unsigned long long)fz);
  atomicAdd(&cnt[i], 1u);
  atomicAdd(&cnt[j], 1u);
}

__global__ void __launch_bounds__(256)
k_pairs_apply(float4* __restrict__ pos, long long* __restrict__ acc, uint32_t* __restrict__ cnt, uint32_t n) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const uint32_t c = cnt[v];
  if (c == 0) return;
  const double inv = 1.0 / (FIX_SCALE * (double)c);
  float4 p = pos[v];
  p.x = __fadd_rn(p.x, (float)((double)acc[3 * (size_t)v] * inv));
  p.y = __fadd_rn(p.y, (float)((double)acc[3 * (size_t)v + 1] * inv));
  p.z = __fadd_rn(p.z, (float)((double)acc[3 * (size_t)v + 2] * inv));
  pos[v] = p;
  acc[3 * (size_t)v] = 0;
  acc[3 * (size_t)v + 1] = 0;
  acc[3 * (size_t)v + 2] = 0;
  cnt[v] = 0;
}

__global__ void k_add_counter(uint32_t* ctr, uint32_t by) { *ctr += by; }

__global__ void k_pack(const float4* __restrict__ v, uint32_t n, float* __restrict__ xyz) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = v[i];
  xyz[3 * (size_t)i] = p.x;
  xyz[3 * (size_t)i + 1] = p.y;
  xyz[3 * (size_t)i + 2] = p.z;
}

// ------------------------------------------------- multi-source BFS --
// Hop distances from all k pivots at once: every node keeps one bit per pivot
// (the pivots that have reached it) and one per pivot that reached it in the
// previous level (the frontier). A level is one pull pass: node i ORs its
// neighbours' frontier words, keeps the bits it has not seen, and records the
// level as its distance to those pivots. Exact BFS distances, independent of
// thread order. Words of 64 pivots, up to MS_WORDS per pass over a row.
constexpr uint32_t MS_WORDS = 4;

__global__ void k_msbfs_seed(uint32_t n, uint32_t k, uint32_t W, const uint32_t* __restrict__ piv,
                             unsigned long long* __restrict__ visited, unsigned long long* __restrict__ front,
                             uint32_t* __restrict__ dist) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= k) return;
  const uint32_t v = piv[p];
  const unsigned long long bit = 1ull << (p & 63u);
  atomicOr(&visited[(size_t)v * W + (p >> 6)], bit);
  atomicOr(&front[(size_t)v * W + (p >> 6)], bit);
  dist[(size_t)p * n + v] = 0u;
}

__global__ void __launch_bounds__(256)
k_msbfs_level(uint32_t n, uint32_t W, const uint32_t* __restrict__ off, const uint32_t* __restrict__ nbr,
              const unsigned long long* __restrict__ front, unsigned long long* __restrict__ next,
              unsigned long long* __restrict__ visited, uint32_t* __restrict__ dist, uint32_t level,
              uint32_t* __restrict__ progress) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bool grew = false;
  for (uint32_t w0 = 0; w0 < W; w0 += MS_WORDS) {
    const uint32_t ww = min(MS_WORDS, W - w0);
    unsigned long long acc[MS_WORDS] = {0ull, 0ull, 0ull, 0ull};
    for (uint32_t e = off[i]; e < off[i + 1]; ++e) {
      const unsigned long long* f = front + (size_t)nbr[e] * W + w0;
      for (uint32_t w = 0; w < ww; ++w) acc[w] |= f[w];
    }
    for (uint32_t w = 0; w < ww; ++w) {
      unsigned long long* vis = visited + (size_t)i * W + w0 + w;
      unsigned long long nb = acc[w] & ~*vis;
      next[(size_t)i * W + w0 + w] = nb;
      if (!nb) continue;
      *vis |= nb;
      grew = true;
      while (nb) {
        const uint32_t b = (uint32_t)__ffsll((long long)nb) - 1u;
        nb &= nb - 1ull;
        dist[(size_t)((w0 + w) * 64u + b) * n + i] = level;
      }
    }
  }
  if (grew) {
    atomicAdd(&progress[0], 1u);
    atomicMax(&progress[1], level);
  }
}

__global__ void k_dist_to_u16(const uint32_t* __restrict__ d32, size_t count, uint16_t* __restrict__ d16) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const uint32_t d = d32[t];
  d16[t] = d == UNREACH ? (uint16_t)0xFFFFu : (uint16_t)d;
}

// ============================================================== host ==
// sgd_stress.rs:372-394
static void bfs(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint32_t src, uint32_t* dist,
                std::vector<uint32_t>& q) {
  std::fill(dist, dist + n, UNREACH);
  q.clear();
  dist[src] = 0;
  q.push_back(src);
  for (size_t h = 0; h < q.size(); ++h) {
    uint32_t v = q[h], dv = dist[v];
    for (uint32_t e = off[v]; e < off[v + 1]; ++e) {
      uint32_t u = nbr[e];
      if (dist[u] == UNREACH) {
        dist[u] = dv + 1;
        q.push_back(u);
      }
    }
  }
}

// sgd_stress.rs:324-334
static float anneal_eta(uint64_t sweep, float eta_max, float eta_min, uint32_t n_anneal) {
  if (n_anneal == 0) return eta_min;
  float t = (float)sweep / (float)n_anneal;
  if (t >= 1.0f) return eta_min;
  float ratio = std::fmax(eta_min / eta_max, 1e-9f);
  return eta_max * std::pow(ratio, t);
}

template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t c) {
    if (p && c <= n) return;
    free();
    c = std::max<size_t>(c, 1);
    JC_CUDA_CHECK(cudaMalloc(&p, c * sizeof(T)));
    n = c;
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { free(); }
};

inline uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

class SgdEngine : public Engine {
 public:
  explicit SgdEngine(bool jacobi) : jacobi_(jacobi) {
    desc_.id = jacobi ? "sgd-stress-gpu" : "sgd-stress";
    desc_.kind = 1;
    desc_.display_name = jacobi ? "SGD stress (B200, Jacobi pivot)" : "SGD stress (B200, per-pair scatter)";
    desc_.description =
        jacobi ? "Pivot stress by SGD (s_gd2 step, Ortmann sparse pivots): one thread per node slides itself "
                 "along its k pivot terms against start-of-sweep positions (Jacobi), pivot positions "
                 "staged in shared memory, distances pivot-major."
               : "Pivot stress by SGD with the s_gd2 pair update moving both endpoints: the reference "
                 "engine's own random (node, pivot) samples, evaluated in parallel batches with "
                 "deterministic fixed-point accumulation.";
    desc_.needs_edges = 1;
    desc_.needs_cpu_positions = 1;
    desc_.needs_gpu_positions_buffer = 0;
  }
  ~SgdEngine() override { release(); }

  const jc_descriptor& descriptor() const override { return desc_; }

  void set_params(const char* json) override {
    decode_sgd(json, &s_, desc_.id);
    drop_graph();
  }

  void init(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint64_t nnz, const float* xyz) override {
    validate_csr(n, off, nbr, nnz, xyz);
    ensure_stream();
    initialized_ = false;
    drop_graph();
    n_ = n;
    // select_pivots (sgd_stress.rs:143-175) with the engine's SplitMix64.
    SplitMix64 rng(s_.seed);
    k_ = n == 0 ? 0 : std::min(std::max(s_.n_pivots, 1u), n);
    pivots_.clear();
    host_dist_valid_ = true;
    if (s_.random_pivots && n && k_) {
      init_random_pivots(n, off, nbr, nnz, xyz, rng);
      return;
    }
    std::vector<uint32_t> dist32((size_t)k_ * n);
    if (n && k_) {
      std::vector<uint32_t> min_d(n, UNREACH), q;
      q.reserve(n);
      uint32_t next = (uint32_t)rng.below(n);
      for (uint32_t t = 0; t < k_; ++t) {
        uint32_t* d = &dist32[(size_t)t * n];
        bfs(n, off, nbr, next, d, q);
        uint32_t best = next, best_d = 0;
        for (uint32_t v = 0; v < n; ++v) {
          uint32_t dv = d[v];
          if (dv != UNREACH && dv < min_d[v]) min_d[v] = dv;
          uint32_t cover = min_d[v];
          if (cover != UNREACH && cover > best_d) { best_d = cover; best = v; }
        }
        pivots_.push_back(next);
        next = best;
      }
    }
    stream_state_ = rng.state;  // position of the pair-sampling stream
    host_dist_ = dist32;
    uint32_t maxd = 0;
    for (uint32_t d : dist32)
      if (d != UNREACH) maxd = std::max(maxd, d);
    finish_init(n, xyz, maxd, &dist32);
  }

  // k distinct uniformly random pivots (a partial Fisher-Yates shuffle on the
  // engine's SplitMix64) and their hop distances by the device multi-source BFS.
  void init_random_pivots(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint64_t nnz, const float* xyz,
                          SplitMix64& rng) {
    std::vector<uint32_t> idx(n);
    for (uint32_t i = 0; i < n; ++i) idx[i] = i;
    for (uint32_t t = 0; t < k_; ++t) std::swap(idx[t], idx[t + (uint32_t)rng.below(n - t)]);
    pivots_.assign(idx.begin(), idx.begin() + k_);
    stream_state_ = rng.state;
    const uint32_t W = (k_ + 63u) / 64u;
    DBuf<uint32_t> doff, dnbr, dpiv, prog;
    DBuf<unsigned long long> vis, fa, fb;
    doff.alloc((size_t)n + 1);
    dnbr.alloc(std::max<uint64_t>(nnz, 1));
    dpiv.alloc(k_);
    prog.alloc(2);
    vis.alloc((size_t)n * W);
    fa.alloc((size_t)n * W);
    fb.alloc((size_t)n * W);
    dist32_.alloc((size_t)k_ * n);
    JC_CUDA_CHECK(cudaMemcpyAsync(doff.p, off, sizeof(uint32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, stream_));
    if (nnz) JC_CUDA_CHECK(cudaMemcpyAsync(dnbr.p, nbr, sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice, stream_));
    JC_CUDA_CHECK(cudaMemcpyAsync(dpiv.p, pivots_.data(), sizeof(uint32_t) * k_, cudaMemcpyHostToDevice, stream_));
    JC_CUDA_CHECK(cudaMemsetAsync(vis.p, 0, sizeof(unsigned long long) * n * W, stream_));
    JC_CUDA_CHECK(cudaMemsetAsync(fa.p, 0, sizeof(unsigned long long) * n * W, stream_));
    JC_CUDA_CHECK(cudaMemsetAsync(dist32_.p, 0xFF, sizeof(uint32_t) * k_ * n, stream_));
    JC_CUDA_CHECK(cudaMemsetAsync(prog.p, 0, 8, stream_));
    k_msbfs_seed<<<cdiv(k_, 256), 256, 0, stream_>>>(n, k_, W, dpiv.p, vis.p, fa.p, dist32_.p);
    // levels in chunks of 16; stop after a chunk in which no node grew (every
    // level after the last growing one changes nothing)
    uint32_t level = 1, maxd = 0;
    for (;;) {
      uint32_t h[2] = {0, 0};
      JC_CUDA_CHECK(cudaMemsetAsync(prog.p, 0, 4, stream_));
      for (int c = 0; c < 16; ++c, ++level) {
        k_msbfs_level<<<cdiv(n, 256), 256, 0, stream_>>>(n, W, doff.p, dnbr.p, fa.p, fb.p, vis.p, dist32_.p, level,
                                                         prog.p);
        std::swap(fa.p, fb.p);
      }
      JC_CUDA_CHECK(cudaGetLastError());
      JC_CUDA_CHECK(cudaMemcpyAsync(h, prog.p, 8, cudaMemcpyDeviceToHost, stream_));
      JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
      maxd = h[1];
      if (h[0] == 0 || level > n + 16u) break;
    }
    host_dist_.clear();
    host_dist_valid_ = false;  // copied back on demand (stress and pivot read-outs)
    finish_init(n, xyz, maxd, nullptr);
  }

  // The rest of init, from the pivot distances: host rows (dist32 != null)
  // or dist32_ already on the device.
  void finish_init(uint32_t n, const float* xyz, uint32_t maxd, const std::vector<uint32_t>* dist32) {
    wide_ = maxd >= 0xFFFFu;
    // eta schedule, one entry per sweep up to the end of annealing
    float eta_max = s_.eta_max, eta_min = s_.eta_min;
    if (s_.auto_eta && maxd > 0) {
      eta_max = (float)maxd * (float)maxd;
      eta_min = 0.01f;
    }
    n_eta_ = s_.n_anneal_steps + 1;
    std::vector<float> eta(n_eta_);
    for (uint32_t w = 0; w < n_eta_; ++w) eta[w] = anneal_eta(w, eta_max, eta_min, s_.n_anneal_steps);
    max_dist_ = maxd;
    // device buffers
    pos_a_.alloc(n); pos_b_.alloc(n); xyz_.alloc((size_t)3 * n); piv_.alloc(k_); eta_.alloc(n_eta_);
    ctr_.alloc(1);
    if (!dist32) {  // distances on the device already (multi-source BFS)
      if (!wide_ && k_ && n) {
        dist16_.alloc((size_t)k_ * n);
        const size_t cnt = (size_t)k_ * n;
        k_dist_to_u16<<<(unsigned)((cnt + 255) / 256), 256, 0, stream_>>>(dist32_.p, cnt, dist16_.p);
        JC_CUDA_CHECK(cudaGetLastError());
      }
    } else if (wide_) {
      dist32_.alloc((size_t)k_ * n);
      if (k_ && n)
        JC_CUDA_CHECK(cudaMemcpyAsync(dist32_.p, dist32->data(), sizeof(uint32_t) * k_ * n, cudaMemcpyHostToDevice,
                                      stream_));
    } else {
      std::vector<uint16_t> d16(dist32->size());
      for (size_t t = 0; t < d16.size(); ++t) d16[t] = (*dist32)[t] == UNREACH ? 0xFFFFu : (uint16_t)(*dist32)[t];
      dist16_.alloc((size_t)k_ * n);
      if (k_ && n)
        JC_CUDA_CHECK(cudaMemcpyAsync(dist16_.p, d16.data(), sizeof(uint16_t) * k_ * n, cudaMemcpyHostToDevice, stream_));
    }
    if (!jacobi_) {
      acc_.alloc((size_t)3 * std::max<uint32_t>(n, 1));
      cnt_.alloc(std::max<uint32_t>(n, 1));
      JC_CUDA_CHECK(cudaMemsetAsync(acc_.p, 0, sizeof(long long) * 3 * std::max<uint32_t>(n, 1), stream_));
      JC_CUDA_CHECK(cudaMemsetAsync(cnt_.p, 0, sizeof(uint32_t) * std::max<uint32_t>(n, 1), stream_));
    }
    std::vector<float> pos4((size_t)4 * n, 0.0f);
    for (uint32_t i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) pos4[4 * (size_t)i + c] = xyz[3 * (size_t)i + c];
    if (n) {
      JC_CUDA_CHECK(cudaMemcpyAsync(pos_a_.p, pos4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, stream_));
      JC_CUDA_CHECK(cudaMemcpyAsync(xyz_.p, xyz, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, stream_));
    }
    if (k_) JC_CUDA_CHECK(cudaMemcpyAsync(piv_.p, pivots_.data(), sizeof(uint32_t) * k_, cudaMemcpyHostToDevice, stream_));
    JC_CUDA_CHECK(cudaMemcpyAsync(eta_.p, eta.data(), sizeof(float) * n_eta_, cudaMemcpyHostToDevice, stream_));
    JC_CUDA_CHECK(cudaMemsetAsync(ctr_.p, 0, sizeof(uint32_t), stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    if (!wide_) dist32_.free();  // the sweeps read the 16-bit copy
    initialized_ = true;
  }

  void step(float* out) override { step_many(1, out); }

  void step_many(uint32_t iters, float* out) override {
    require_init();
    if (n_ == 0 || k_ == 0 || iters == 0) return;
    ensure_graph();
    for (uint32_t s = 0; s < iters; ++s) JC_CUDA_CHECK(cudaGraphLaunch(gexec_, stream_));
    if (out) JC_CUDA_CHECK(cudaMemcpyAsync(out, xyz_.p, sizeof(float) * 3 * n_, cudaMemcpyDeviceToHost, stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
  }

  void positions(float* out) override {
    require_init();
    if (n_ == 0) return;
    JC_CUDA_CHECK(cudaMemcpyAsync(out, xyz_.p, sizeof(float) * 3 * n_, cudaMemcpyDeviceToHost, stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
  }

  void time_steps(uint32_t iters, float* total_ms, float* phase_ms4) override {
    require_init();
    if (phase_ms4)
      for (int k = 0; k < 4; ++k) phase_ms4[k] = 0.0f;
    if (n_ == 0 || k_ == 0 || iters == 0) {
      if (total_ms) *total_ms = 0.0f;
      return;
    }
    ensure_graph();
    cudaEvent_t e0, e1;
    JC_CUDA_CHECK(cudaEventCreate(&e0));
    JC_CUDA_CHECK(cudaEventCreate(&e1));
    JC_CUDA_CHECK(cudaEventRecord(e0, stream_));
    for (uint32_t s = 0; s < iters; ++s) JC_CUDA_CHECK(cudaGraphLaunch(gexec_, stream_));
    JC_CUDA_CHECK(cudaEventRecord(e1, stream_));
    JC_CUDA_CHECK(cudaEventSynchronize(e1));
    float ms = 0.0f;
    JC_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    if (total_ms) *total_ms = ms;
    if (phase_ms4) phase_ms4[1] = ms / (float)iters;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }

  uint32_t launches_per_step() const override { return launches_; }

  uint32_t node_count() const override { return n_; }
  void enqueue_steps(uint32_t iters) override {
    require_init();
    if (n_ == 0 || k_ == 0) return;
    ensure_graph();
    for (uint32_t s = 0; s < iters; ++s) JC_CUDA_CHECK(cudaGraphLaunch(gexec_, stream_));
  }
  const float* device_xyz() const override { return xyz_.p; }
  cudaStream_t cuda_stream() const override { return stream_; }

  // Stress of the current layout over the engine's (node, pivot) terms:
  // raw Σ w (|x_i - x_j| - d)^2 and the scale-normalized value, w = 1/d^2, in
  // f64 as crates/graph-layouts/src/metrics.rs:31-76 defines them.
  void stress(double* raw, double* normalized) override {
    require_init();
    fetch_host_dist();
    std::vector<float> xyz((size_t)3 * n_);
    positions(xyz.data());
    auto dist_ij = [&](uint32_t i, uint32_t j) {
      double dx = (double)(xyz[3 * (size_t)i] - xyz[3 * (size_t)j]);
      double dy = (double)(xyz[3 * (size_t)i + 1] - xyz[3 * (size_t)j + 1]);
      double dz = (double)(xyz[3 * (size_t)i + 2] - xyz[3 * (size_t)j + 2]);
      return std::sqrt(dx * dx + dy * dy + dz * dz);
    };
    // Fixed-order sums (independent of the thread count): every pivot row is
    // cut into the same CHUNKS ranges, each summed in node order, and the
    // chunk partials are added in chunk order, pivot after pivot.
    constexpr int64_t CHUNKS = 64;
    const int64_t span = ((int64_t)n_ + CHUNKS - 1) / CHUNKS;
    std::vector<double> part(4 * CHUNKS);
    double num = 0, den = 0, wd2 = 0, rs = 0;
    for (uint32_t t = 0; t < k_; ++t) {
      const uint32_t j = pivots_[t];
      const uint32_t* row = &host_dist_[(size_t)t * n_];
#pragma omp parallel for schedule(static)
      for (int64_t c = 0; c < CHUNKS; ++c) {
        double a = 0, b = 0, w2 = 0, r2 = 0;
        const int64_t lo = c * span, hi = std::min<int64_t>((int64_t)n_, lo + span);
        for (int64_t ii = lo; ii < hi; ++ii) {
          const uint32_t i = (uint32_t)ii, du = row[i];
          if (i == j || du == UNREACH || du == 0) continue;
          const double d = (double)du, w = 1.0 / (d * d), big = dist_ij(i, j);
          a += w * d * big;
          b += w * big * big;
          w2 += w * d * d;
          r2 += w * (big - d) * (big - d);
        }
        part[4 * c] = a; part[4 * c + 1] = b; part[4 * c + 2] = w2; part[4 * c + 3] = r2;
      }
      for (int64_t c = 0; c < CHUNKS; ++c) {
        num += part[4 * c]; den += part[4 * c + 1]; wd2 += part[4 * c + 2]; rs += part[4 * c + 3];
      }
    }
    if (raw) *raw = rs;
    if (!normalized) return;
    if (den <= 0.0 || wd2 <= 0.0) {
      *normalized = 0.0;
      return;
    }
    const double alpha = num / den;
    double acc = 0;
    for (uint32_t t = 0; t < k_; ++t) {
      const uint32_t j = pivots_[t];
      const uint32_t* row = &host_dist_[(size_t)t * n_];
#pragma omp parallel for schedule(static)
      for (int64_t c = 0; c < CHUNKS; ++c) {
        double a = 0;
        const int64_t lo = c * span, hi = std::min<int64_t>((int64_t)n_, lo + span);
        for (int64_t ii = lo; ii < hi; ++ii) {
          const uint32_t i = (uint32_t)ii, du = row[i];
          if (i == j || du == UNREACH || du == 0) continue;
          const double d = (double)du, w = 1.0 / (d * d), r = alpha * dist_ij(i, j) - d;
          a += w * r * r;
        }
        part[c] = a;
      }
      for (int64_t c = 0; c < CHUNKS; ++c) acc += part[c];
    }
    *normalized = acc / wd2;
  }

  // Pivot ids (k) and hop distances (k x n, pivot-major, 0xFFFFFFFF =
  // unreachable); either pointer may be null. Returns k.
  uint32_t pivots(uint32_t* piv, uint32_t* dist) override {
    require_init();
    if (piv && k_) std::memcpy(piv, pivots_.data(), sizeof(uint32_t) * k_);
    if (dist && k_ && n_) {
      fetch_host_dist();
      std::memcpy(dist, host_dist_.data(), sizeof(uint32_t) * k_ * n_);
    }
    return k_;
  }

  uint64_t state_size() override { return 8 + (uint64_t)16 * n_; }
  void save_state(void* buf) override {
    require_init();
    uint8_t* b = (uint8_t*)buf;
    uint32_t sw = 0;
    JC_CUDA_CHECK(cudaMemcpyAsync(&sw, ctr_.p, 4, cudaMemcpyDeviceToHost, stream_));
    if (n_) JC_CUDA_CHECK(cudaMemcpyAsync(b + 8, pos_a_.p, sizeof(float4) * n_, cudaMemcpyDeviceToHost, stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    std::memcpy(b, &n_, 4);
    std::memcpy(b + 4, &sw, 4);
  }
  void load_state(const void* buf, uint64_t len) override {
    require_init();
    if (len != state_size()) fail(JC_ERR_ARG, "state size mismatch");
    const uint8_t* b = (const uint8_t*)buf;
    uint32_t n, sw;
    std::memcpy(&n, b, 4);
    std::memcpy(&sw, b + 4, 4);
    if (n != n_) fail(JC_ERR_ARG, "state is for a graph with a different node count");
    JC_CUDA_CHECK(cudaMemcpyAsync(ctr_.p, &sw, 4, cudaMemcpyHostToDevice, stream_));
    if (n_) {
      JC_CUDA_CHECK(cudaMemcpyAsync(pos_a_.p, b + 8, sizeof(float4) * n_, cudaMemcpyHostToDevice, stream_));
      k_pack<<<cdiv(n_, 256), 256, 0, stream_>>>(pos_a_.p, n_, xyz_.p);
      JC_CUDA_CHECK(cudaGetLastError());
    }
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
  }

 private:
  bool jacobi_;
  jc_descriptor desc_{};
  SgdSettings s_;
  uint32_t n_ = 0, k_ = 0, n_eta_ = 1, launches_ = 0, max_dist_ = 0;
  bool wide_ = false, initialized_ = false;
  uint64_t stream_state_ = 0;
  std::vector<uint32_t> pivots_;
  std::vector<uint32_t> host_dist_;  // k x n pivot distances (for the stress read-out)
  bool host_dist_valid_ = true;

  void fetch_host_dist() {
    if (host_dist_valid_) return;
    host_dist_.resize((size_t)k_ * n_);
    if (k_ && n_) {
      if (wide_) {
        JC_CUDA_CHECK(cudaMemcpyAsync(host_dist_.data(), dist32_.p, sizeof(uint32_t) * k_ * n_,
                                      cudaMemcpyDeviceToHost, stream_));
        JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
      } else {
        std::vector<uint16_t> d16((size_t)k_ * n_);
        JC_CUDA_CHECK(cudaMemcpyAsync(d16.data(), dist16_.p, sizeof(uint16_t) * k_ * n_, cudaMemcpyDeviceToHost,
                                      stream_));
        JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
        for (size_t t = 0; t < d16.size(); ++t) host_dist_[t] = d16[t] == 0xFFFFu ? UNREACH : d16[t];
      }
    }
    host_dist_valid_ = true;
  }
  cudaStream_t stream_ = nullptr;
  cudaGraphExec_t gexec_ = nullptr;
  DBuf<float4> pos_a_, pos_b_;
  DBuf<float> xyz_, eta_;
  DBuf<uint32_t> piv_, ctr_, dist32_, cnt_;
  DBuf<uint16_t> dist16_;
  DBuf<long long> acc_;

  void ensure_stream() {
    if (!stream_) {
      int dev_count = 0;
      if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
        fail(JC_ERR_CUDA, "no CUDA device is available");
      JC_CUDA_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    }
  }
  void release() {
    drop_graph();
    if (stream_) {
      cudaStreamSynchronize(stream_);
      cudaStreamDestroy(stream_);
      stream_ = nullptr;
    }
  }
  void drop_graph() {
    if (gexec_) {
      cudaGraphExecDestroy(gexec_);
      gexec_ = nullptr;
    }
  }
  void require_init() const {
    if (!initialized_) fail(JC_ERR_STATE, std::string(desc_.id) + " step called before successful init");
  }

  template <typename D>
  int enqueue_sweeps(const D* dist) {
    const uint32_t n = n_, k = k_;
    const uint32_t sweeps = std::max(s_.sweeps_per_step, 1u);
    int L = 0;
    if (jacobi_) {
      // sgd_stress_gpu.rs:377-428: one eta per step, `sweeps` ping-pong sweeps.
      // the mu table covers distances up to the largest one when it fits in 16 KB
      const uint32_t mu_len = max_dist_ + 1 <= 4096u ? max_dist_ + 1 : 0u;
      const size_t smem = sizeof(float4) * k + sizeof(float) * mu_len;
      if (smem > 200 * 1024) fail(JC_ERR_ARG, "too many pivots for the shared-memory pivot stage");
      if (smem > 48 * 1024)
        JC_CUDA_CHECK(cudaFuncSetAttribute(k_jacobi<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      float4* in = pos_a_.p;
      float4* out = pos_b_.p;
      for (uint32_t s = 0; s < sweeps; ++s) {
        k_jacobi<D><<<cdiv(n, 256), 256, smem, stream_>>>(in, out, piv_.p, dist, n, k, eta_.p, n_eta_, ctr_.p,
                                                           mu_len);
        std::swap(in, out);
        ++L;
      }
      if (in != pos_a_.p) {
        JC_CUDA_CHECK(cudaMemcpyAsync(pos_a_.p, in, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream_));
        ++L;
      }
      k_add_counter<<<1, 1, 0, stream_>>>(ctr_.p, sweeps);
      ++L;
    } else {
      // sgd_stress.rs:287-315: per sweep, eta(sweep), n samples, sweep += 1.
      // Default: batches of max(256, n/64) samples (at most 64 per sweep).
      uint32_t batches = s_.scatter_batches ? s_.scatter_batches : cdiv(n, std::max(256u, cdiv(n, 64)));
      batches = std::max(1u, std::min(batches, n));
      const uint32_t per = cdiv(n, batches);
      for (uint32_t s = 0; s < sweeps; ++s) {
        for (uint32_t q0 = 0; q0 < n; q0 += per) {
          const uint32_t cnt = std::min(per, n - q0);
          k_pairs<D><<<cdiv(cnt, 256), 256, 0, stream_>>>(pos_a_.p, acc_.p, cnt_.p, piv_.p, dist, n, k,
                                                          stream_state_, q0, cnt, eta_.p, n_eta_, ctr_.p);
          k_pairs_apply<<<cdiv(n, 256), 256, 0, stream_>>>(pos_a_.p, acc_.p, cnt_.p, n);
          L += 2;
        }
        k_add_counter<<<1, 1, 0, stream_>>>(ctr_.p, 1u);
        ++L;
      }
    }
    k_pack<<<cdiv(n, 256), 256, 0, stream_>>>(pos_a_.p, n, xyz_.p);
    ++L;
    JC_CUDA_CHECK(cudaGetLastError());
    return L;
  }

  void ensure_graph() {
    if (gexec_) return;
    cudaGraph_t g;
    JC_CUDA_CHECK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    int L = 0;
    try {
      L = wide_ ? enqueue_sweeps<uint32_t>(dist32_.p) : enqueue_sweeps<uint16_t>(dist16_.p);
    } catch (...) {
      cudaStreamEndCapture(stream_, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    JC_CUDA_CHECK(cudaStreamEndCapture(stream_, &g));
    cudaError_t e = cudaGraphInstantiate(&gexec_, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) fail(JC_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    launches_ = (uint32_t)L;
  }
};

}  // namespace sgd

Engine* make_sgd_engine(bool jacobi) { return new sgd::SgdEngine(jacobi); }

}  // namespace jc
