// ForceAtlas2 layout step on B200: Barnes-Hut ("fa2-bh") and all-pairs
// ("fa2-brute") engines.
//
// Reference behaviour being reproduced (paths in the jump-cannon repo):
//   crates/graph-compute/src/engines/fa2_bh.rs      engine, host octree build
//   crates/graph-compute/src/shaders/fa2_barnes_hut.wgsl  fa2_force / fa2_apply
//   crates/graph-compute/src/shaders/force_atlas2.wgsl    brute-force fa2_force
//   crates/graph-compute/src/engines/fa2_speed.rs   AdaptiveSpeed::update
//
// One step is a fixed sequence of kernels on the engine's stream, captured
// once into a CUDA graph and replayed (no host round trip inside a step):
//
//   k_bbox      finite-coordinate bounding box -> root centre / half extent
//               (fa2_bh.rs:768-799), last block finalises.
//   k_keys      per body, the octant digits of levels 0..31 computed with the
//               reference's own float tests `p >= centre` and child centres
//               `c +/- half*0.5` (fa2_bh.rs:841-861). Packed as a 96-bit key
//               (levels 0..20 in 63 bits, 21..31 in 33 bits). Bodies with a
//               non-finite coordinate get bit 63 and sort last.
//   radix sort  stable LSD over the 64-bit high key (8 passes). If two valid
//               keys tie in those 21 levels, a device-gated re-sort by the
//               low 33 bits then the high 64 bits restores full order.
//   k_count     per sorted body: the number of octree nodes whose pre-order
//               run starts at it. The reference's pointer octree (split a cell
//               while it holds >= 2 bodies, one node per level, depth cap 32)
//               is exactly determined by the longest common digit prefixes of
//               sorted neighbours; bodies whose 32 digits equal their
//               predecessor's are the ones the reference drops at the depth
//               cap (fa2_bh.rs:874-922) and get zero nodes.
//   scan        node index of each body's first node (pre-order == DFS order
//               with children in octant order 0..7, as assign_ropes walks).
//   k_fill      writes every node: pre-order makes `next` = index + 1 and
//               `skip` = first node after the subtree (found by a binary
//               search over the sorted keys); parent links; child counts.
//   k_com       bottom-up centre of mass with arrival counters; the last child
//               to arrive sums the children in octant order in f32, as
//               aggregate_com_postorder does (fa2_bh.rs:927-967).
//   k_walk      theta-criterion walk. A warp takes 32 consecutive bodies in
//               key order and walks the union of their paths node by node in
//               pre-order; every lane keeps its own accept/open decision via
//               per-depth ballot masks, so each body sees exactly the node
//               sequence of the reference's rope walk (wgsl:114-156).
//   k_att       attraction over the per-node edge list in the shader's edge
//               order, gravity, swing/traction, per-block f64 partial sums;
//               the last block finishes the reduction and runs the adaptive
//               speed state machine on the device (fa2_speed.rs:48-100).
//   k_apply     displacement (wgsl:203-226), F_old <- F, xyz for readback.
//
// Arithmetic: every f32 operation that the reference writes is issued as one
// IEEE round-to-nearest operation in the same order (__fadd_rn, __fmul_rn,
// __fdiv_rn, __fsqrt_rn: no contraction into FMA), so forces are bit-identical
// to the CPU restatement of the reference for nodes whose edge list is
// shorter than the hub threshold.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "jc_check.cuh"
#include "jc_common.h"
#include "jc_engine.h"
#include "jc_params.h"
#include "jc_sort.cuh"
#include "jc_pool.h"
#include "jc_upload.h"

namespace jc {
namespace fa2 {

constexpr uint32_t END = 0xFFFFFFFFu;
constexpr int WALK_THREADS = 256;
constexpr int ATT_THREADS = 256;

constexpr int APPLY_THREADS = 256;
constexpr int BBOX_THREADS = 256;
constexpr int BBOX_BLOCKS = 296;  // 2 x 148 SMs
constexpr uint32_t DEFAULT_HUB_THRESHOLD = 2048;
// Lists at least this long (and below the hub threshold) are gathered by a
// whole warp, 32 neighbours at a time, and summed in list order by lane 0: a
// thread alone would wait on hundreds of dependent gather rounds.
constexpr uint32_t DEFAULT_WARP_THRESHOLD = 512;
constexpr uint32_t DEFAULT_WALK_GROUP = 1;  // fastest in the B200 sweep (1, 2, 4, ..., 32)
// The top of a single graph's tree (depth <= TOP_DEPTH, at most
// 1 + 8 + 64 + 512 nodes) is staged in shared memory for the walk.
constexpr int TOP_DEPTH = 3;
constexpr uint32_t TOP_MAX = 585;

// Fixed per captured graph; passed by value.
struct KParams {
  uint32_t n;
  float gravity;
  float scaling_ratio;
  float att_w;  // pow(max(edge weight 1.0, 1e-6), edge_weight_influence)
  float ewi;
  float jitter_tolerance;
  float time_step;
  float theta2;
  float max_disp;
  int strong_gravity;
  int lin_log;
  uint32_t tree_cap;
  uint32_t ref_cap;
  uint32_t n_hubs;
  uint32_t n_med;  // nodes after the hubs whose lists a whole warp gathers
};

// One octree node in pre-order (32 bytes): centre of mass and mass, then
// {skip (first node after the subtree, END at the end), body (-1 for an
// internal node), s^2 = (2 * half extent)^2 as float bits, depth}.
struct __align__(32) TNode {
  float4 cm;
  int4 meta;
};
static_assert(sizeof(TNode) == 32, "a node is one 32-byte sector");

// One node in a single 256-bit load (read-only path): the walk is bound by
// L1 request throughput, and one 32-byte request per visit replaces two.
__device__ __forceinline__ void load_node(const TNode* p, float4& cm, int4& meta) {
  uint32_t r0, r1, r2, r3, r4, r5, r6, r7;
  asm("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5), "=r"(r6), "=r"(r7)
               : "l"(p));
  cm = make_float4(__uint_as_float(r0), __uint_as_float(r1), __uint_as_float(r2), __uint_as_float(r3));
  meta = make_int4((int)r4, (int)r5, (int)r6, (int)r7);
}

// Device-resident scalars (one per engine).
struct DevState {
  float speed;
  float speed_eff;
  float root[4];
  uint32_t n_invalid;
  uint32_t n_valid;
  uint32_t tie;
  uint32_t n_tree;
  uint32_t max_depth;
  uint32_t dropped;
  uint32_t warn;
  uint32_t error;
  uint32_t bbox_done;
  uint32_t att_done;
  uint32_t steps_done;
  uint32_t n_top;  // nodes of depth <= TOP_DEPTH listed this step (single graph)
  unsigned long long n_inter;
  unsigned long long n_open;
};

// Graph (segment) layout of a batch. A single graph has n_graphs = 1,
// gbits = 0, lh = 21 and null arrays, and every formula below reduces to the
// one-graph form. A batch prefixes each key with its graph id (gbits bits
// under the invalid bit) so the sort groups bodies by graph; each graph gets
// its own octree in the shared pre-order node array.
struct Forest {
  uint32_t n_graphs;
  uint32_t gbits;               // graph-id bits in the high key
  int lh;                       // octant levels held in the high key
  const uint32_t* node_graph;   // graph of each body (batch only)
  const uint32_t* graph_off;    // bodies of graph g: [graph_off[g], graph_off[g+1])
  float4* roots;                // per-graph root cell (centre xyz, half)
  uint32_t* tree_root;          // per-graph node index of its root (END: no body)
  uint32_t* tree_end;           // per-graph one past its last node
  float2* gspeed;               // per-graph (speed, speed efficiency)
  // Per-graph reductions run over slices of at most GRAPH_SLICE bodies, so a
  // batch of a few large graphs (partitions) still fills the GPU.
  uint32_t n_slices;
  const uint32_t* slice_graph;  // graph of slice s
  const uint32_t* graph_slice;  // slices of graph g: [graph_slice[g], graph_slice[g+1])
  float* slice_box;             // 6 per slice: min x,y,z, max x,y,z of finite coordinates
  double2* slice_sums;          // per slice: (swing, traction) sums
  // per graph: 0, or (1 << 32) | its 32 z octant bits when every finite body
  // of the graph has the same z (a 2D layout): all its bodies then share the
  // z half of every octant digit, computed once per graph
  uint64_t* zflat;
};

constexpr uint32_t GRAPH_SLICE = 8192;

// ------------------------------------------------------------ helpers --
__device__ __forceinline__ float len3(float x, float y, float z) {
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
}

// Longest common octant-digit prefix of two valid keys, in levels; -1 when
// the bodies belong to different graphs of a batch.
__device__ __forceinline__ int lcp_levels(uint64_t ha, uint64_t la, uint64_t hb, uint64_t lb, uint32_t gbits = 0,
                                          int lh = 21) {
  uint64_t x = ha ^ hb;
  if (gbits) {
    if (x >> (63 - gbits)) return -1;
    x &= (1ull << (63 - gbits)) - 1ull;
  }
  if (x) return (__clzll((long long)x) - 1 - (int)gbits) / 3;
  uint64_t y = la ^ lb;
  if (y) return lh + (__clzll((long long)y) - (64 - 3 * (32 - lh))) / 3;
  return 32;
}

__device__ __forceinline__ uint32_t key_graph(uint64_t h, uint32_t gbits) {
  return gbits ? (uint32_t)((h >> (63 - gbits)) & ((1u << gbits) - 1u)) : 0u;
}

__device__ __forceinline__ void set_error(DevState* st, uint32_t code) { atomicCAS(&st->error, 0u, code); }

// --------------------------------------------------------------- bbox --
__global__ void __launch_bounds__(BBOX_THREADS)
k_bbox(const float4* __restrict__ pos, uint32_t n, float* __restrict__ part, DevState* st) {
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 p = pos[i];
    float v[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (isfinite(v[k])) {
        mn[k] = fminf(mn[k], v[k]);
        mx[k] = fmaxf(mx[k], v[k]);
      }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn[k] = fminf(mn[k], __shfl_xor_sync(0xFFFFFFFFu, mn[k], o));
      mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xFFFFFFFFu, mx[k], o));
    }
  __shared__ float sh[BBOX_THREADS / 32][6];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 3; ++k) { sh[w][k] = mn[k]; sh[w][3 + k] = mx[k]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    float r[6];
    for (int k = 0; k < 6; ++k) r[k] = sh[0][k];
    for (int ww = 1; ww < BBOX_THREADS / 32; ++ww)
      for (int k = 0; k < 3; ++k) { r[k] = fminf(r[k], sh[ww][k]); r[3 + k] = fmaxf(r[3 + k], sh[ww][3 + k]); }
    for (int k = 0; k < 6; ++k) part[blockIdx.x * 6 + k] = r[k];
    __threadfence();
    last = atomicAdd(&st->bbox_done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x >= 32) return;
  __threadfence();
  // warp 0 of the last block: lane-strided partials, then a butterfly
  float r[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  for (uint32_t b = threadIdx.x; b < gridDim.x; b += 32)
    for (int k = 0; k < 3; ++k) {
      r[k] = fminf(r[k], __ldcg(&part[b * 6 + k]));
      r[3 + k] = fmaxf(r[3 + k], __ldcg(&part[b * 6 + 3 + k]));
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      r[k] = fminf(r[k], __shfl_xor_sync(0xFFFFFFFFu, r[k], o));
      r[3 + k] = fmaxf(r[3 + k], __shfl_xor_sync(0xFFFFFFFFu, r[3 + k], o));
    }
  if (threadIdx.x != 0) return;
  // fa2_bh.rs:785-799
  if (!isfinite(r[0]))
    for (int k = 0; k < 3; ++k) { r[k] = -1.0f; r[3 + k] = 1.0f; }
  float c0 = __fmul_rn(0.5f, __fadd_rn(r[0], r[3]));
  float c1 = __fmul_rn(0.5f, __fadd_rn(r[1], r[4]));
  float c2 = __fmul_rn(0.5f, __fadd_rn(r[2], r[5]));
  float half = __fmul_rn(fmaxf(fmaxf(__fsub_rn(r[3], r[0]), __fsub_rn(r[4], r[1])), __fsub_rn(r[5], r[2])), 0.5f);
  if (!isfinite(half) || half <= 0.0f) half = 1.0f;
  half = __fmul_rn(half, 1.05f);
  st->root[0] = c0;
  st->root[1] = c1;
  st->root[2] = c2;
  st->root[3] = half;
  st->bbox_done = 0;
  st->n_top = 0;
  st->n_invalid = 0;
  st->tie = 0;
  st->max_depth = 0;
  st->dropped = 0;
  st->n_inter = 0;
  st->n_open = 0;
}

// --------------------------------------------------------------- keys --
__global__ void __launch_bounds__(256)
k_keys(const float4* __restrict__ pos, uint32_t n, DevState* st, uint64_t* __restrict__ hi_orig,
       uint64_t* __restrict__ lo_orig, uint64_t* __restrict__ hi_sort, uint32_t* __restrict__ val, Forest F) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  bool invalid = false;
  if (i < n) {
    float4 p = pos[i];
    uint64_t hi = 0, lo = 0;
    if (isfinite(p.x) && isfinite(p.y) && isfinite(p.z)) {
      const uint32_t g = F.node_graph ? F.node_graph[i] : 0u;
      float cx, cy, cz, h;
      uint64_t zf = 0;
      if (F.n_graphs > 1) {
        const float4 r = F.roots[g];
        cx = r.x; cy = r.y; cz = r.z; h = r.w;
        zf = F.zflat[g];
      } else {
        cx = st->root[0]; cy = st->root[1]; cz = st->root[2]; h = st->root[3];
      }
      const int lh = F.lh < 32 ? F.lh : 32;
      if (zf >> 32) {
        // every body of this graph has the same z: its z bits are the graph's
        auto level = [&](uint64_t& w, int l) {
          const uint32_t o = (p.x >= cx ? 1u : 0u) | (p.y >= cy ? 2u : 0u) | ((uint32_t)(zf >> l) & 1u) << 2;
          w = (w << 3) | o;
          const float hh = __fmul_rn(h, 0.5f);
          cx = __fadd_rn(cx, (o & 1u) ? hh : -hh);
          cy = __fadd_rn(cy, (o & 2u) ? hh : -hh);
          h = hh;
        };
        int l = 0;
#pragma unroll 4
        for (; l < lh; ++l) level(hi, l);
#pragma unroll 4
        for (; l < 32; ++l) level(lo, l);
      } else {
        // levels [0, lh) into the high word, the rest into the low word: two
        // loops instead of a per-level choice of the destination word
        auto level = [&](uint64_t& w) {
          const uint32_t o = (p.x >= cx ? 1u : 0u) | (p.y >= cy ? 2u : 0u) | (p.z >= cz ? 4u : 0u);
          w = (w << 3) | o;
          const float hh = __fmul_rn(h, 0.5f);
          cx = __fadd_rn(cx, (o & 1u) ? hh : -hh);
          cy = __fadd_rn(cy, (o & 2u) ? hh : -hh);
          cz = __fadd_rn(cz, (o & 4u) ? hh : -hh);
          h = hh;
        };
        int l = 0;
#pragma unroll 4
        for (; l < lh; ++l) level(hi);
#pragma unroll 4
        for (; l < 32; ++l) level(lo);
      }
      hi <<= (63 - (int)F.gbits - 3 * F.lh);  // digits right under the graph id (no shift for one graph)
      if (F.gbits) hi |= (uint64_t)g << (63 - F.gbits);
    } else {
      hi = 1ull << 63;
      invalid = true;
    }
    hi_orig[i] = hi;
    lo_orig[i] = lo;
    hi_sort[i] = hi;
    val[i] = i;
  }
  uint32_t bal = __ballot_sync(0xFFFFFFFFu, invalid);
  if (bal && (threadIdx.x & 31) == 0) {
    atomicAdd(&st->n_invalid, (uint32_t)__popc(bal));
    atomicOr(&st->warn, JC_WARN_NONFINITE);
  }
}

// The tree sort orders the keys by their top bits only (a single graph: the
// top 32, four radix passes instead of eight, the first ten octant levels,
// which separate almost all bodies; a batch: the top 48, six passes, the graph
// id and about eleven levels); this kernel then sorts every run of equal top
// parts by the full 96-bit key (high word, then the low word read through the
// body index) and body index, one thread per run, which is the order of the
// full sort. Keys equal in all 64 high bits (bodies closer than one cell of
// the last level the high word holds: in a batch of 4,096 2D graphs that is
// level 17, and among 13.8 M bodies such pairs occur every step) are thereby
// ordered without the full re-sort. A run longer than SEG_MAX sets the tie
// flag instead, which sends the step through the full 96-bit re-sort.
// Non-finite bodies (bit 63) sort last in any order.
constexpr uint32_t SEG_MAX = 32;
__global__ void __launch_bounds__(256)
k_seg_fix(uint64_t* __restrict__ hi, uint32_t* __restrict__ val, const uint64_t* __restrict__ lo_orig, uint32_t n,
          DevState* st, int shift) {
  const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a == 0) st->n_valid = n - st->n_invalid;  // valid bodies (the non-finite sort last)
  if (a >= n || st->error) return;
  const uint64_t h = hi[a];
  if (h >> 63) return;
  const uint64_t top = h >> shift;
  // (runs only permute keys with equal top parts, so these reads are stable)
  if (a > 0 && (hi[a - 1] >> shift) == top) return;  // not the first of its run
  uint32_t len = 1;
  while (a + len < n && len <= SEG_MAX && (hi[a + len] >> shift) == top) ++len;
  if (len == 1) return;
  if (len > SEG_MAX) {
    st->tie = 1u;
    return;
  }
  uint64_t k[SEG_MAX], l[SEG_MAX];
  uint32_t v[SEG_MAX];
  for (uint32_t i = 0; i < len; ++i) {
    k[i] = hi[a + i];
    v[i] = val[a + i];
    l[i] = JC_IN_BOUNDS(v[i], n, &st->error) ? lo_orig[v[i]] : 0ull;
  }
  for (uint32_t i = 1; i < len; ++i) {
    const uint64_t kk = k[i], ll = l[i];
    const uint32_t vv = v[i];
    uint32_t j = i;
    while (j > 0 && (k[j - 1] > kk || (k[j - 1] == kk && (l[j - 1] > ll || (l[j - 1] == ll && v[j - 1] > vv))))) {
      k[j] = k[j - 1];
      l[j] = l[j - 1];
      v[j] = v[j - 1];
      --j;
    }
    k[j] = kk;
    l[j] = ll;
    v[j] = vv;
  }
  for (uint32_t i = 0; i < len; ++i) {
    hi[a + i] = k[i];
    val[a + i] = v[i];
  }
}

__global__ void __launch_bounds__(256)
k_gather_u64(const uint64_t* __restrict__ src, const uint32_t* __restrict__ val, uint64_t* __restrict__ dst,
             DevState* st, const uint32_t* gate, uint32_t n) {
  if (gate && *gate == 0) return;
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a < st->n_valid) {
    const uint32_t v = val[a];
    if (JC_IN_BOUNDS(v, n, &st->error)) dst[a] = src[v];
  }
  (void)n;
}

// ---------------------------------------------------- prefix lengths --
// L[j] = lcp(j, j+1) of the sorted bodies in levels (-1 across graphs of a
// batch, at the last valid body and beyond), with two levels of block minima
// (m1 over 32 entries, m2 over 1024), so the end or start of the run of
// bodies sharing d digits is found by scanning at most 32 bytes per level
// instead of binary-searching the 16-byte keys.
struct LcpIndex {
  int8_t* L;
  int8_t* m1;
  int8_t* m2;
  uint32_t n1, n2;  // entries in m1, m2 (L holds 32 * n1 = 1024 * n2 bytes)
};

__host__ __device__ inline uint32_t lcp_index_bytes(uint32_t n) { return ((max(n, 1u) + 1023u) / 1024u) * 1024u; }
// m2 is padded to whole 32-byte blocks with 127 ("no run ends here").
inline uint32_t lcp_m2_bytes(uint32_t nl) { return ((nl / 1024u + 31u) / 32u) * 32u; }

// Bit k set where byte k of the 32-byte block p (32-byte aligned) is < d
// (signed bytes; d in [0, 33]): two 16-byte loads and per-byte SIMD compares.
__device__ __forceinline__ uint32_t block_below(const int8_t* p, int d) {
  const uint4 u0 = *reinterpret_cast<const uint4*>(p);
  const uint4 u1 = *reinterpret_cast<const uint4*>(p + 16);
  const uint32_t dd = (uint32_t)(uint8_t)d * 0x01010101u;
  const uint32_t w[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
  uint32_t mask = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t lt = __vcmplts4(w[k], dd);  // 0xFF in each byte where w < d
    mask |= (((lt >> 7) & 1u) | ((lt >> 14) & 2u) | ((lt >> 21) & 4u) | ((lt >> 28) & 8u)) << (4 * k);
  }
  return mask;
}

// First j >= a with L[j] < d; the run of bodies sharing d levels with a is
// [a, j]. END if there is none (cannot happen: L ends in -1 and d >= 0).
__device__ __forceinline__ uint32_t lcp_next_below(const LcpIndex& X, uint32_t a, int d) {
  // most runs are short (deep cells): the next few entries one by one first
#pragma unroll
  for (uint32_t k = 0; k < 3; ++k)
    if (a + k < 32u * X.n1 && (int)X.L[a + k] < d) return a + k;
  const uint32_t base0 = a & ~31u;
  uint32_t m = block_below(X.L + base0, d) & (~0u << (a & 31u));
  if (m) return base0 + (uint32_t)__ffs(m) - 1u;
  const uint32_t b1 = (base0 >> 5) + 1u;  // next 32-body block
  uint32_t blk = END;
  if (b1 < X.n1) {
    const uint32_t base1 = b1 & ~31u;
    m = block_below(X.m1 + base1, d) & (~0u << (b1 & 31u));
    if (m) blk = base1 + (uint32_t)__ffs(m) - 1u;
  }
  if (blk == END) {
    for (uint32_t b2 = (b1 >> 5) + 1u; b2 < X.n2; b2 = (b2 & ~31u) + 32u) {
      const uint32_t base2 = b2 & ~31u;
      m = block_below(X.m2 + base2, d) & (~0u << (b2 & 31u));
      if (m) {
        const uint32_t c = base2 + (uint32_t)__ffs(m) - 1u;  // m2 padding is 127: c < n2
        m = block_below(X.m1 + 32u * c, d);
        if (!m) return END;
        blk = 32u * c + (uint32_t)__ffs(m) - 1u;
        break;
      }
    }
    if (blk == END) return END;
  }
  m = block_below(X.L + 32u * blk, d);
  return m ? 32u * blk + (uint32_t)__ffs(m) - 1u : END;
}

// Last j < a with L[j] < p, or -1: the run of bodies sharing p levels with a
// starts at that j + 1.
__device__ __forceinline__ int64_t lcp_prev_below(const LcpIndex& X, uint32_t a, int p) {
  if (a == 0) return -1;
#pragma unroll
  for (uint32_t k = 1; k <= 3; ++k) {
    if (k > a) return -1;
    if ((int)X.L[a - k] < p) return (int64_t)(a - k);
  }
  const uint32_t j0 = a - 1u, base0 = j0 & ~31u;
  uint32_t m = block_below(X.L + base0, p) & (0xFFFFFFFFu >> (31u - (j0 & 31u)));
  if (m) return (int64_t)(base0 + 31u - (uint32_t)__clz(m));
  if (base0 == 0) return -1;
  const uint32_t b1 = (base0 >> 5) - 1u;  // previous 32-body block
  const uint32_t base1 = b1 & ~31u;
  int64_t blk = -1;
  m = block_below(X.m1 + base1, p) & (0xFFFFFFFFu >> (31u - (b1 & 31u)));
  if (m) blk = (int64_t)(base1 + 31u - (uint32_t)__clz(m));
  if (blk < 0) {
    for (int64_t b2 = (int64_t)(base1 >> 5) - 1; b2 >= 0; b2 = (int64_t)((uint32_t)b2 & ~31u) - 1) {
      const uint32_t base2 = (uint32_t)b2 & ~31u;
      m = block_below(X.m2 + base2, p) & (0xFFFFFFFFu >> (31u - ((uint32_t)b2 & 31u)));
      if (m) {
        const uint32_t c = base2 + 31u - (uint32_t)__clz(m);
        m = block_below(X.m1 + 32u * c, p);
        if (!m) return -1;
        blk = (int64_t)(32u * c + 31u - (uint32_t)__clz(m));
        break;
      }
    }
    if (blk < 0) return -1;
  }
  m = block_below(X.L + 32u * (uint32_t)blk, p);
  return m ? (int64_t)(32u * (uint32_t)blk + 31u - (uint32_t)__clz(m)) : -1;
}

// ------------------------------------------------------------- count --
// One block of 1024 threads per 1024 entries of L: its 32 warps write 32
// first-level minima (m1) and the block their minimum (m2), so the whole
// index is built in this pass.
constexpr int COUNT_THREADS = 1024;
__global__ void __launch_bounds__(COUNT_THREADS)
k_count(const uint64_t* __restrict__ hi, const uint64_t* __restrict__ lo, uint32_t n, DevState* st,
        uint32_t* __restrict__ count, Forest F, LcpIndex X) {
  const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t N = st->n_valid;
  uint32_t c = 0;
  bool dup = false;
  int next = -1;  // lcp(a, a + 1), -1 at the last valid body and beyond
  if (a < N) {
    uint64_t ha = hi[a], la = lo[a];
    int prev = -1;
    if (a > 0) {
      prev = lcp_levels(hi[a - 1], lo[a - 1], ha, la, F.gbits, F.lh);
      dup = prev == 32;
    }
    if (a + 1 < N) next = lcp_levels(ha, la, hi[a + 1], lo[a + 1], F.gbits, F.lh);
    if (!dup) c = 1u + (uint32_t)max(0, max(0, next) - prev);
  }
  if (a < n) count[a] = c;
  // the grid covers the index exactly: 32 * X.n1 = 1024 * X.n2 entries
  __shared__ int wmin[COUNT_THREADS / 32];
  X.L[a] = (int8_t)next;
  int m = next;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  if ((threadIdx.x & 31) == 0) {
    X.m1[a >> 5] = (int8_t)m;
    wmin[threadIdx.x >> 5] = m;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    int v = wmin[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    if (threadIdx.x == 0) X.m2[blockIdx.x] = (int8_t)v;
  }
  const uint32_t bal = __ballot_sync(0xFFFFFFFFu, dup);
  if (bal && (threadIdx.x & 31) == 0) {
    atomicAdd(&st->dropped, (uint32_t)__popc(bal));
    atomicOr(&st->warn, JC_WARN_DEPTH_CAP);
  }
}

// Capacity check + clearing of the per-node counters for this step.
__global__ void __launch_bounds__(256)
k_clear(const uint32_t* __restrict__ first, uint32_t n, KParams P, DevState* st,
        uint32_t* __restrict__ nchild, uint32_t* __restrict__ arrive) {
  uint32_t T = first[n];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (T > P.tree_cap) {
      set_error(st, JC_ERR_CAPACITY);
      st->n_tree = 0;
    } else {
      st->n_tree = T;
    }
    if (T > P.ref_cap) atomicOr(&st->warn, JC_WARN_REF_CAPACITY);
  }
  uint32_t lim = min(T, P.tree_cap);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < lim; i += gridDim.x * blockDim.x) {
    nchild[i] = 0;
    arrive[i] = 0;
  }
}

// ---------------------------------------------------------------- fill --
// Bounded to 32 registers (eight blocks per SM, no spills): the fill waits on
// its prefix-length searches and position gathers (tree build 0.443 -> 0.440 ms
// on the 1M-node R-MAT against 40 registers).
__global__ void __launch_bounds__(256, 8)
k_fill(const uint64_t* __restrict__ hi, const LcpIndex X, const uint32_t* __restrict__ val,
       const uint32_t* __restrict__ first, const float4* __restrict__ pos, const float* __restrict__ degf,
       uint32_t n, KParams P, DevState* st, TNode* __restrict__ nodes,
       uint32_t* __restrict__ parent, uint32_t* __restrict__ nchild, Forest F,
       uint32_t* __restrict__ top_list = nullptr) {
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t N = st->n_valid;
  if (st->error) return;
  uint32_t leaf_depth = 0;
  if (a < N) {
    const uint32_t T = first[n];
    uint32_t base = first[a], stop = first[a + 1];
    if (stop > base) {  // not a dropped duplicate
      const int prev = a > 0 ? (int)X.L[a - 1] : -1;
      const int top = max(0, (int)X.L[a]);
      const int n_int = max(0, top - prev);
      const uint32_t g = key_graph(hi[a], F.gbits);
      const uint32_t tend = F.n_graphs > 1 ? F.tree_end[g] : T;
      // root half extent halved once per level, as child_center does.
      float half = F.n_graphs > 1 ? F.roots[g].w : st->root[3];
      {
        // prev + 1 exact halvings: an exponent decrement while the result
        // stays a normal number, the multiplications themselves otherwise
        const int e = (__float_as_int(half) >> 23) & 0xFF;
        if (half > 0.0f && e != 0xFF && e - (prev + 1) >= 1)
          half = __int_as_float(__float_as_int(half) - ((prev + 1) << 23));
        else
          for (int k = 0; k <= prev; ++k) half = __fmul_rn(half, 0.5f);
      }
      uint32_t first_parent = END;
      if (prev >= 0) {
        // the parent is the node of depth prev on the run that contains a - 1
        const uint32_t ap = (uint32_t)(lcp_prev_below(X, a, prev) + 1);
        const int pp = ap == 0 ? -1 : (int)X.L[ap - 1];
        first_parent = first[ap] + (uint32_t)(prev - pp - 1);
      }
      for (int j = 0; j < n_int; ++j) {
        int d = prev + 1 + j;
        uint32_t idx = base + (uint32_t)j;
        uint32_t b = (d == 0 && F.n_graphs == 1) ? N - 1 : lcp_next_below(X, a, d);
        if (b >= N) {
          set_error(st, JC_ERR_DEVICE_TIMEOUT);
          return;
        }
        uint32_t sk = first[b + 1];
        if (sk >= tend) sk = END;
        float s = __fmul_rn(half, 2.0f);
        if (!JC_IN_BOUNDS(idx, P.tree_cap, &st->error)) return;
        nodes[idx].meta = make_int4((int)sk, -1, __float_as_int(__fmul_rn(s, s)), d);
        nodes[idx].cm = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t par = j == 0 ? first_parent : idx - 1;
        parent[idx] = par;
        if (par != END && JC_IN_BOUNDS(par, P.tree_cap, &st->error)) atomicAdd(&nchild[par], 1u);
        if (top_list && d <= TOP_DEPTH) {
          const uint32_t slot = atomicAdd(&st->n_top, 1u);
          if (slot < TOP_MAX) top_list[slot] = idx;
        }
        half = __fmul_rn(half, 0.5f);
      }
      uint32_t leaf = base + (uint32_t)n_int;
      leaf_depth = (uint32_t)(max(prev, top) + 1);
      uint32_t body = val[a];
      if (!JC_IN_BOUNDS(leaf, P.tree_cap, &st->error) || !JC_IN_BOUNDS(body, n, &st->error)) return;
      float4 p = pos[body];
      uint32_t sk = first[a + 1];
      if (sk >= tend) sk = END;
      nodes[leaf].meta = make_int4((int)sk, (int)body, 0, (int)leaf_depth);
      nodes[leaf].cm = make_float4(p.x, p.y, p.z, fmaxf(degf[body], 1e-3f));
      uint32_t par = n_int > 0 ? leaf - 1 : first_parent;
      parent[leaf] = par;
      if (par != END && JC_IN_BOUNDS(par, P.tree_cap, &st->error)) atomicAdd(&nchild[par], 1u + (1u << 16));  // leaves also count in the high half
      if (top_list && (int)leaf_depth <= TOP_DEPTH) {
        const uint32_t slot = atomicAdd(&st->n_top, 1u);
        if (slot < TOP_MAX) top_list[slot] = leaf;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) leaf_depth = max(leaf_depth, __shfl_xor_sync(0xFFFFFFFFu, leaf_depth, o));
  if ((threadIdx.x & 31) == 0 && leaf_depth) atomicMax(&st->max_depth, leaf_depth);
}

// ----------------------------------------------------------------- COM --
__global__ void __launch_bounds__(256)
k_com(const uint32_t* __restrict__ first, TNode* nodes, const uint32_t* __restrict__ parent,
      const uint32_t* __restrict__ nchild, uint32_t* __restrict__ arrive, uint32_t n, DevState* st) {
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (st->error) return;
  const uint32_t N = st->n_valid;
  if (a >= N) return;
  uint32_t base = first[a], stop = first[a + 1];
  if (stop == base) return;
  const uint32_t T = first[n];
  // nchild[v] holds v's children in its low half and its leaf children in the
  // high half. Leaves never arrive: a cell whose children are all leaves is
  // finished by the thread of its first child (index v + 1), without an
  // arrival; a cell with cell children counts arrivals from those only.
  const uint32_t leaf = stop - 1;
  if (!JC_IN_BOUNDS(leaf, T, &st->error)) return;
  uint32_t node = parent[leaf];
  if (node == END || !JC_IN_BOUNDS(node, T, &st->error)) return;
  {
    const uint32_t nc = nchild[node];
    if ((nc >> 16) != (nc & 0xFFFFu) || leaf != node + 1u) return;
  }
  bool first_cell = true;
  uint32_t guard = 0;
  while (node != END) {
    if (++guard > 64u) { set_error(st, JC_ERR_DEVICE_TIMEOUT); return; }
    // acq_rel: publishes this thread's child sums and, for the last arrival,
    // makes every other child's sums visible before they are read. A cell with
    // one cell child needs no arrival: that child's sums are this thread's own.
    if (!first_cell) {
      const uint32_t nc = nchild[node];
      const uint32_t cells = (nc & 0xFFFFu) - (nc >> 16);
      if (cells != 1u) {
        uint32_t old;
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(arrive + node) : "memory");
        if (old + 1u != cells) return;
      }
    }
    first_cell = false;
    float tot = 0.0f, sx = 0.0f, sy = 0.0f, sz = 0.0f;
    const uint32_t end = (uint32_t)nodes[node].meta.x;
    uint32_t c = node + 1;
    uint32_t kids = 0;
    while (c != end) {
      if (c >= T || ++kids > 8u) { set_error(st, JC_ERR_DEVICE_TIMEOUT); return; }
      float4 v = __ldcg(&nodes[c].cm);
      tot = __fadd_rn(tot, v.w);
      sx = __fadd_rn(sx, __fmul_rn(v.x, v.w));
      sy = __fadd_rn(sy, __fmul_rn(v.y, v.w));
      sz = __fadd_rn(sz, __fmul_rn(v.z, v.w));
      uint32_t nx = (uint32_t)nodes[c].meta.x;
      if (nx != END && nx <= c) { set_error(st, JC_ERR_DEVICE_TIMEOUT); return; }
      c = nx;
    }
    if (tot > 0.0f) {
      sx = __fdiv_rn(sx, tot);
      sy = __fdiv_rn(sy, tot);
      sz = __fdiv_rn(sz, tot);
    }
    __stcg(&nodes[node].cm, make_float4(sx, sy, sz, tot));
    if (node == 0) return;
    uint32_t up = parent[node];
    if (up != END && up >= node) { set_error(st, JC_ERR_DEVICE_TIMEOUT); return; }
    node = up;
  }
}

// ---------------------------------------------------------------- walk --
// One repulsion term k = srd * m / max(r2, 1e-4), f += d * k. Exact: the
// reference's roundings, one IEEE operation each in source order (bit-exact
// with the oracle). FAST (the `fast_repulsion` setting): the same term with
// the division replaced by a multiply with the approximate reciprocal
// (__fdividef, within 2 ulp) and the three accumulations fused into FMAs.
// Only the force sum changes; every tree decision (r2 and the theta test)
// is computed exactly in both modes, so the walk is the same node sequence.
template <bool FAST>
__device__ __forceinline__ void rep_term(float dx, float dy, float dz, float r2, float srd, float m, float& fx,
                                         float& fy, float& fz) {
  if (FAST) {
    const float k = __fdividef(srd * m, fmaxf(r2, 1.0e-4f));
    fx = fmaf(dx, k, fx);
    fy = fmaf(dy, k, fy);
    fz = fmaf(dz, k, fz);
  } else {
    const float k = __fdiv_rn(__fmul_rn(srd, m), fmaxf(r2, 1.0e-4f));
    fx = __fadd_rn(fx, __fmul_rn(dx, k));
    fy = __fadd_rn(fy, __fmul_rn(dy, k));
    fz = __fadd_rn(fz, __fmul_rn(dz, k));
  }
}

// Bodies are taken in key order (spatially coherent). A walk group of G
// consecutive lanes shares one stream of nodes in pre-order: it visits a
// node when at least one of its lanes opened the node's parent, and each lane
// keeps its own decision through a path bitmask (bit d set = this lane
// opened the node at depth d on the current path), so a lane is active at a
// node of depth d exactly when bits 0..d-1 are set. Every lane therefore
// meets the nodes of its own rope walk (wgsl:114-156) in the same order and
// accumulates the same sequence of terms, whatever G is. G = 1 is one
// independent rope walk per lane; G = 32 shares every node load across the
// warp at the cost of walking the union of 32 paths.
template <int G, bool FAST>
__global__ void __launch_bounds__(WALK_THREADS)
k_walk(const TNode* __restrict__ nodes, const uint32_t* __restrict__ order, const float4* __restrict__ pos,
       const float* __restrict__ degf, uint32_t n, KParams P, DevState* st, float4* __restrict__ frep, Forest F) {
  const int lane = threadIdx.x & 31;
  const uint32_t a = blockIdx.x * WALK_THREADS + threadIdx.x;
  const uint32_t body0 = a < n ? order[a] : 0u;
  const bool have = a < n && JC_IN_BOUNDS(body0, n, &st->error);
  const uint32_t body = have ? body0 : 0u;
  // In a batch a walk group shares a node stream only among lanes of the
  // same graph (each graph has its own root).
  uint32_t root = 0u;
  if (F.n_graphs > 1) root = have ? F.tree_root[F.node_graph[body]] : END;
  uint32_t gmask = G == 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << (lane & ~(G - 1)));
  if (F.n_graphs > 1) gmask &= __match_any_sync(0xFFFFFFFFu, root);
  const float4 p = have ? pos[body] : make_float4(0.f, 0.f, 0.f, 0.f);
  const float srd = have ? __fmul_rn(P.scaling_ratio, degf[body]) : 0.0f;
  float fx = 0.0f, fy = 0.0f, fz = 0.0f;
  uint32_t n_inter = 0, n_open = 0;
  const uint32_t T = st->error ? 0u : st->n_tree;
  const bool group_has = (__ballot_sync(0xFFFFFFFFu, have) & gmask) != 0u;
  uint32_t idx = (T > 0u && group_has) ? root : END;
  uint64_t path = 0;
  while (__any_sync(0xFFFFFFFFu, idx != END)) {
    const bool alive = idx != END;
    float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
    int4 m = make_int4(-1, -1, 0, 0);
    if (alive) {
      c = nodes[idx].cm;
      m = nodes[idx].meta;
    }
    const uint32_t depth = (uint32_t)m.w;
    const uint64_t below = (1ull << depth) - 1ull;
    const bool me = have && alive && ((path & below) == below);
    const float dx = __fsub_rn(p.x, c.x), dy = __fsub_rn(p.y, c.y), dz = __fsub_rn(p.z, c.z);
    const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    const bool leaf = m.y >= 0;
    bool contrib, open = false;
    if (leaf) {
      contrib = me && (uint32_t)m.y != body && c.w > 0.0f;
    } else {
      const bool acc = c.w > 0.0f && r2 > 0.0f && __int_as_float(m.z) < __fmul_rn(P.theta2, r2);
      contrib = me && acc;
      open = me && !acc;
      if (me) path = open ? (path | (1ull << depth)) : (path & ~(1ull << depth));
    }
    if (contrib) {
      rep_term<FAST>(dx, dy, dz, r2, srd, c.w, fx, fy, fz);
      ++n_inter;
    }
    n_open += open ? 1u : 0u;
    const uint32_t om = __ballot_sync(0xFFFFFFFFu, open) & gmask;
    if (alive) {
      uint32_t next = (!leaf && om) ? idx + 1u : (uint32_t)m.x;
      if (next != END && (next <= idx || next >= T)) {
        set_error(st, JC_ERR_DEVICE_TIMEOUT);
        next = END;
      }
      idx = next;
    }
  }
  if (have) frep[body] = make_float4(fx, fy, fz, 0.0f);
  unsigned long long ci = n_inter, co = n_open;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ci += __shfl_xor_sync(0xFFFFFFFFu, ci, o);
    co += __shfl_xor_sync(0xFFFFFFFFu, co, o);
  }
  if (lane == 0 && (ci | co)) {
    atomicAdd(&st->n_inter, ci);
    atomicAdd(&st->n_open, co);
  }
}

// One independent rope walk per lane (walk group 1): the reference's walk
// (wgsl:114-156) with nothing shared between lanes, so no masks or votes.
// Adds this body's repulsion terms in the reference's visit order and writes
// frep[body]; returns false (error set) on a malformed rope.
template <bool FAST>
__device__ __forceinline__ void walk_one(const TNode* __restrict__ nodes, uint32_t body, const float4 p, float srd,
                                         uint32_t root, uint32_t T, float theta2, DevState* st,
                                         float4* __restrict__ frep, uint32_t& n_inter, uint32_t& n_open) {
  float fx = 0.0f, fy = 0.0f, fz = 0.0f;
  uint32_t idx = root;
  // Ropes strictly increase, so the walk ends; it leaves the loop at END or at
  // a rope past the tree (a malformed tree, reported below), never reading
  // outside [0, T).
  while (idx < T) {
    float4 c;
    int4 m;
    load_node(nodes + idx, c, m);
    const float dx = __fsub_rn(p.x, c.x), dy = __fsub_rn(p.y, c.y), dz = __fsub_rn(p.z, c.z);
    const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    const bool leaf = m.y >= 0;
    // (the reference also requires m > 0; every node's mass is >= 1e-3 here:
    // leaves hold max(deg + 1, 1e-3), cells sums of their leaves, so that test
    // is always true and is left out of the hot loop. Its r2 > 0 test is
    // implied: size^2 >= 0 is never below theta^2 * 0, nor below a NaN.)
    const bool use = leaf ? (uint32_t)m.y != body : __int_as_float(m.z) < __fmul_rn(theta2, r2);
    if (use) {
      rep_term<FAST>(dx, dy, dz, r2, srd, c.w, fx, fy, fz);
      ++n_inter;
    }
    const bool descend = !leaf && !use;
    n_open += descend ? 1u : 0u;
    const uint32_t next = descend ? idx + 1u : (uint32_t)m.x;
    if (next <= idx) break;
    idx = next;
  }
  if (idx != END) set_error(st, JC_ERR_DEVICE_TIMEOUT);
  frep[body] = make_float4(fx, fy, fz, 0.0f);
}

__device__ __forceinline__ void walk_counts_flush(uint32_t n_inter, uint32_t n_open, DevState* st) {
  unsigned long long ci = n_inter, co = n_open;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ci += __shfl_xor_sync(0xFFFFFFFFu, ci, o);
    co += __shfl_xor_sync(0xFFFFFFFFu, co, o);
  }
  if ((threadIdx.x & 31) == 0 && (ci | co)) {
    atomicAdd(&st->n_inter, ci);
    atomicAdd(&st->n_open, co);
  }
}

// One thread per body, bodies in key order. Bounded to 32 registers, so
// eight blocks (every warp slot of the SM) are resident: the walk waits on
// its node loads, and full occupancy hides more of that (1M-node R-MAT walk
// 0.538 -> 0.516 ms against 37 registers and six blocks, no spills).
template <bool FAST>
__global__ void __launch_bounds__(WALK_THREADS, 2048 / WALK_THREADS)
k_walk_rope(const TNode* __restrict__ nodes, const uint32_t* __restrict__ order, const float4* __restrict__ pos,
            const float* __restrict__ degf, uint32_t n, KParams P, DevState* st, float4* __restrict__ frep, Forest F) {
  const uint32_t a = blockIdx.x * WALK_THREADS + threadIdx.x;
  const uint32_t T = st->error ? 0u : st->n_tree;
  uint32_t n_inter = 0, n_open = 0;
  if (a < n && T > 0u) {
    const uint32_t body = order[a];
    if (!JC_IN_BOUNDS(body, n, &st->error)) return;
    const uint32_t root = F.n_graphs > 1 ? F.tree_root[F.node_graph[body]] : 0u;
    walk_one<FAST>(nodes, body, pos[body], __fmul_rn(P.scaling_ratio, degf[body]), root, T, P.theta2, st, frep,
                   n_inter, n_open);
  } else if (a < n) {
    const uint32_t body = order[a];
    if (JC_IN_BOUNDS(body, n, &st->error)) frep[body] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  walk_counts_flush(n_inter, n_open, st);
}

// ------------------------------------------------------ staged top --
// The nodes of depth <= TOP_DEPTH of a single graph's tree in pre-order, 32
// bytes each: {cm.xyzw, s^2 bits, kind, top skip, global skip}. kind: the
// body of a leaf; -1 for a cell of depth < TOP_DEPTH (its children are the
// next top entries); -2 - g for a cell g of depth TOP_DEPTH, whose subtree
// [g + 1, global skip) the walk runs in global memory. top skip: the entry
// of the node that follows the subtree in pre-order (always a node of depth
// <= TOP_DEPTH, or the end), so the staged walk visits exactly the nodes of
// the rope walk, in the same order.
__global__ void __launch_bounds__(1024)
k_top_build(const TNode* __restrict__ nodes, const uint32_t* __restrict__ top_list, DevState* st,
            uint4* __restrict__ top) {
  __shared__ uint32_t key[1024];
  const uint32_t t = threadIdx.x;
  const uint32_t listed = st->n_top;
  const uint32_t nt = (st->error || listed > TOP_MAX) ? 0u : listed;
  if (listed > TOP_MAX && t == 0) set_error(st, JC_ERR_DEVICE_TIMEOUT);
  key[t] = t < nt ? top_list[t] : END;
  __syncthreads();
  // bitonic sort of the listed node indices
  for (uint32_t k = 2; k <= 1024; k <<= 1)
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      const uint32_t o = t ^ j;
      if (o > t) {
        const uint32_t x = key[t], y = key[o];
        if (((t & k) == 0) == (x > y)) {
          key[t] = y;
          key[o] = x;
        }
      }
      __syncthreads();
    }
  if (t < nt) {
    const uint32_t g = key[t];
    const TNode nd = nodes[g];
    const uint32_t skip = (uint32_t)nd.meta.x;
    uint32_t tskip = nt;
    if (skip != END) {
      uint32_t lo = 0, hi = nt;  // first entry >= skip
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (key[mid] < skip) lo = mid + 1; else hi = mid;
      }
      if (lo >= nt || key[lo] != skip) set_error(st, JC_ERR_DEVICE_TIMEOUT);
      tskip = lo;
    }
    const int kind = nd.meta.y >= 0 ? nd.meta.y : (nd.meta.w < TOP_DEPTH ? -1 : -2 - (int)g);
    top[2 * t] = make_uint4(__float_as_uint(nd.cm.x), __float_as_uint(nd.cm.y), __float_as_uint(nd.cm.z),
                            __float_as_uint(nd.cm.w));
    top[2 * t + 1] = make_uint4((uint32_t)nd.meta.z, (uint32_t)kind, tskip, skip);
  }
  if (t == 0) st->n_top = nt;
}

// The rope walk with the top of the tree in shared memory: each lane walks
// the staged entries and, at a cell of depth TOP_DEPTH it opens, that cell's
// subtree in global memory, then continues at the cell's top skip. Single
// graph only (root = node 0).
template <bool FAST>
__global__ void __launch_bounds__(WALK_THREADS)
k_walk_top(const TNode* __restrict__ nodes, const uint4* __restrict__ top, const uint32_t* __restrict__ order,
           const float4* __restrict__ pos, const float* __restrict__ degf, uint32_t n, KParams P, DevState* st,
           float4* __restrict__ frep) {
  __shared__ uint4 tsm[2 * TOP_MAX];
  const uint32_t T = st->error ? 0u : st->n_tree;
  const uint32_t nt = min(st->n_top, TOP_MAX);
  for (uint32_t k = threadIdx.x; k < 2 * nt; k += WALK_THREADS) tsm[k] = __ldcg(top + k);
  __syncthreads();
  const uint32_t a = blockIdx.x * WALK_THREADS + threadIdx.x;
  uint32_t n_inter = 0, n_open = 0;
  if (a < n) {
    const uint32_t body = order[a];
    if (!JC_IN_BOUNDS(body, n, &st->error)) return;
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    if (T > 0u && nt > 0u) {
      const float4 p = pos[body];
      const float srd = __fmul_rn(P.scaling_ratio, degf[body]);
      uint32_t ti = 0;         // top entry (top mode)
      uint32_t idx = END;      // global node (subtree mode)
      uint32_t gend = 0, tnext = 0;
      bool ok = true;
      while (true) {
        float4 c;
        uint32_t s2b;
        int kind;
        uint32_t skip_next;
        const bool in_top = idx == END;
        if (in_top) {
          if (ti >= nt) break;
          const uint4 u0 = tsm[2 * ti], u1 = tsm[2 * ti + 1];
          c = make_float4(__uint_as_float(u0.x), __uint_as_float(u0.y), __uint_as_float(u0.z), __uint_as_float(u0.w));
          s2b = u1.x;
          kind = (int)u1.y;
          skip_next = u1.z;
        } else {
          float4 cc;
          int4 m;
          load_node(nodes + idx, cc, m);
          c = cc;
          s2b = (uint32_t)m.z;
          kind = m.y;  // body of a leaf, -1 for a cell
          skip_next = (uint32_t)m.x;
        }
        const float dx = __fsub_rn(p.x, c.x), dy = __fsub_rn(p.y, c.y), dz = __fsub_rn(p.z, c.z);
        const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
        const bool leaf = kind >= 0;
        const bool use = leaf ? (uint32_t)kind != body : __uint_as_float(s2b) < __fmul_rn(P.theta2, r2);
        if (use) {
          rep_term<FAST>(dx, dy, dz, r2, srd, c.w, fx, fy, fz);
          ++n_inter;
        }
        const bool descend = !leaf && !use;
        n_open += descend ? 1u : 0u;
        if (in_top) {
          if (descend && kind < -1) {
            // a cell of depth TOP_DEPTH: its subtree in global memory
            idx = (uint32_t)(-2 - kind) + 1u;
            gend = tsm[2 * ti + 1].w;
            tnext = skip_next;
            if (idx >= T || idx >= gend) { ok = false; break; }
          } else {
            const uint32_t nx = descend ? ti + 1u : skip_next;
            if (nx <= ti) { ok = false; break; }
            ti = nx;
          }
        } else {
          const uint32_t next = descend ? idx + 1u : skip_next;
          if (next <= idx) { ok = false; break; }
          if (next >= gend) {
            if (next != gend) { ok = false; break; }
            idx = END;
            ti = tnext;
          } else {
            if (next >= T) { ok = false; break; }
            idx = next;
          }
        }
      }
      if (!ok) set_error(st, JC_ERR_DEVICE_TIMEOUT);
    }
    frep[body] = make_float4(fx, fy, fz, 0.0f);
  }
  walk_counts_flush(n_inter, n_open, st);
}

// Sets the graph condition that runs the full 96-bit re-sort.
__global__ void k_set_tie_condition(cudaGraphConditionalHandle h, const DevState* st) {
  cudaGraphSetConditional(h, st->tie ? 1u : 0u);
}

__device__ void speed_update(DevState* st, uint32_t n, float jitter_tolerance, double ts, double tt);

// ------------------------------------------------------ batch kernels --
// Bounding box of each slice of a batch's graphs (finite coordinates only).
__global__ void __launch_bounds__(256)
k_bbox_slices(const float4* __restrict__ pos, Forest F) {
  const uint32_t sl = blockIdx.x, g = F.slice_graph[sl];
  const uint32_t b = F.graph_off[g] + (sl - F.graph_slice[g]) * GRAPH_SLICE;
  const uint32_t e = min(F.graph_off[g + 1], b + GRAPH_SLICE);
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = b + threadIdx.x; i < e; i += blockDim.x) {
    const float4 p = pos[i];
    const float v[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (isfinite(v[k])) {
        mn[k] = fminf(mn[k], v[k]);
        mx[k] = fmaxf(mx[k], v[k]);
      }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn[k] = fminf(mn[k], __shfl_xor_sync(0xFFFFFFFFu, mn[k], o));
      mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xFFFFFFFFu, mx[k], o));
    }
  __shared__ float sh[8][6];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 3; ++k) { sh[w][k] = mn[k]; sh[w][3 + k] = mx[k]; }
  __syncthreads();
  if (threadIdx.x < 6) {
    const bool lo = threadIdx.x < 3;
    float r = lo ? INFINITY : -INFINITY;
    for (int ww = 0; ww < (int)(blockDim.x / 32); ++ww)
      r = lo ? fminf(r, sh[ww][threadIdx.x]) : fmaxf(r, sh[ww][threadIdx.x]);
    F.slice_box[6 * (size_t)sl + threadIdx.x] = r;
  }
}

// Root cell of each graph (one warp per graph) from its slices' boxes,
// exactly as k_bbox finalises it (min/max are exact in any order); graph 0
// also clears the per-step counters.
__global__ void __launch_bounds__(256)
k_bbox_roots(Forest F, DevState* st) {
  const uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= F.n_graphs) return;
  float r[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  for (uint32_t sl = F.graph_slice[g] + lane; sl < F.graph_slice[g + 1]; sl += 32)
    for (int k = 0; k < 3; ++k) {
      r[k] = fminf(r[k], F.slice_box[6 * (size_t)sl + k]);
      r[3 + k] = fmaxf(r[3 + k], F.slice_box[6 * (size_t)sl + 3 + k]);
    }
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      r[k] = fminf(r[k], __shfl_xor_sync(0xFFFFFFFFu, r[k], o));
      r[3 + k] = fmaxf(r[3 + k], __shfl_xor_sync(0xFFFFFFFFu, r[3 + k], o));
    }
  if (lane != 0) return;
  if (!isfinite(r[0]))
    for (int k = 0; k < 3; ++k) { r[k] = -1.0f; r[3 + k] = 1.0f; }
  float half = __fmul_rn(fmaxf(fmaxf(__fsub_rn(r[3], r[0]), __fsub_rn(r[4], r[1])), __fsub_rn(r[5], r[2])), 0.5f);
  if (!isfinite(half) || half <= 0.0f) half = 1.0f;
  const float4 root = make_float4(__fmul_rn(0.5f, __fadd_rn(r[0], r[3])), __fmul_rn(0.5f, __fadd_rn(r[1], r[4])),
                                  __fmul_rn(0.5f, __fadd_rn(r[2], r[5])), __fmul_rn(half, 1.05f));
  F.roots[g] = root;
  F.tree_root[g] = END;
  uint64_t zf = 0;
  if (r[2] == r[5] && isfinite(r[2])) {  // one z for every finite body: k_keys' z tests, once
    float cz = root.z, h = root.w;
    uint32_t bits = 0;
    for (int l = 0; l < 32; ++l) {
      const bool up = r[2] >= cz;
      bits |= (up ? 1u : 0u) << l;
      const float hh = __fmul_rn(h, 0.5f);
      cz = __fadd_rn(cz, up ? hh : -hh);
      h = hh;
    }
    zf = (1ull << 32) | bits;
  }
  F.zflat[g] = zf;
  if (g == 0) {
    st->n_invalid = 0;
    st->tie = 0;
    st->max_depth = 0;
    st->dropped = 0;
    st->n_inter = 0;
    st->n_open = 0;
  }
}

// Root and end of each graph's tree from the sorted keys and node offsets.
__global__ void __launch_bounds__(256)
k_graph_trees(const uint64_t* __restrict__ hi, const uint32_t* __restrict__ first, const DevState* st, Forest F) {
  const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t N = st->n_valid;
  if (a >= N) return;
  const uint32_t g = key_graph(hi[a], F.gbits);
  if (a == 0 || key_graph(hi[a - 1], F.gbits) != g) F.tree_root[g] = first[a];
  if (a + 1 == N || key_graph(hi[a + 1], F.gbits) != g) F.tree_end[g] = first[a + 1];
}

// Adaptive speed of each graph: f64 sums of the finite swing/traction pairs
// over each slice in a fixed-shape reduction (k_speed_slices), then per graph
// the slices' sums in slice order and AdaptiveSpeed::update with the graph's
// own node count (k_speed_graphs). Deterministic: every shape is fixed.
__global__ void __launch_bounds__(256)
k_speed_slices(const float2* __restrict__ stats, Forest F, const DevState* st) {
  if (st->error) return;
  const uint32_t sl = blockIdx.x, g = F.slice_graph[sl];
  const uint32_t b = F.graph_off[g] + (sl - F.graph_slice[g]) * GRAPH_SLICE;
  const uint32_t e = min(F.graph_off[g + 1], b + GRAPH_SLICE);
  double sw = 0.0, tr = 0.0;
  for (uint32_t i = b + threadIdx.x; i < e; i += blockDim.x) {
    const float2 v = stats[i];
    if (isfinite(v.x) && isfinite(v.y)) {
      sw += (double)v.x;
      tr += (double)v.y;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sw += __shfl_xor_sync(0xFFFFFFFFu, sw, o);
    tr += __shfl_xor_sync(0xFFFFFFFFu, tr, o);
  }
  __shared__ double rs[8], rt[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { rs[w] = sw; rt[w] = tr; }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double a = 0.0, c = 0.0;
  for (int ww = 0; ww < (int)(blockDim.x / 32); ++ww) { a += rs[ww]; c += rt[ww]; }
  F.slice_sums[sl] = make_double2(a, c);
}

__global__ void __launch_bounds__(256)
k_speed_graphs(Forest F, float jitter_tolerance, const DevState* st) {
  if (st->error) return;
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= F.n_graphs) return;
  double a = 0.0, c = 0.0;
  for (uint32_t sl = F.graph_slice[g]; sl < F.graph_slice[g + 1]; ++sl) {
    const double2 v = F.slice_sums[sl];
    a += v.x;
    c += v.y;
  }
  DevState tmp;
  tmp.speed = F.gspeed[g].x;
  tmp.speed_eff = F.gspeed[g].y;
  speed_update(&tmp, F.graph_off[g + 1] - F.graph_off[g], jitter_tolerance, a, c);
  F.gspeed[g] = make_float2(tmp.speed, tmp.speed_eff);
}

// ------------------------------------------------------- brute force --
__global__ void __launch_bounds__(256)
k_brute(const float4* __restrict__ pos, const float* __restrict__ degf, uint32_t n, KParams P,
        float4* __restrict__ frep) {
  __shared__ float4 tile[256];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  float4 p = i < n ? pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  const float srd = i < n ? __fmul_rn(P.scaling_ratio, degf[i]) : 0.0f;
  float fx = 0.0f, fy = 0.0f, fz = 0.0f;
  for (uint32_t base = 0; base < n; base += 256) {
    uint32_t j = base + threadIdx.x;
    if (j < n) {
      float4 q = pos[j];
      tile[threadIdx.x] = make_float4(q.x, q.y, q.z, degf[j]);
    }
    __syncthreads();
    uint32_t lim = min(256u, n - base);
    for (uint32_t t = 0; t < lim; ++t) {
      if (base + t == i) continue;
      float4 q = tile[t];
      float dx = __fsub_rn(p.x, q.x), dy = __fsub_rn(p.y, q.y), dz = __fsub_rn(p.z, q.z);
      float r2 = fmaxf(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)), 1.0e-4f);
      float k = __fdiv_rn(__fmul_rn(srd, q.w), r2);
      fx = __fadd_rn(fx, __fmul_rn(dx, k));
      fy = __fadd_rn(fy, __fmul_rn(dy, k));
      fz = __fadd_rn(fz, __fmul_rn(dz, k));
    }
    __syncthreads();
  }
  if (i < n) frep[i] = make_float4(fx, fy, fz, 0.0f);
}

// ----------------------------------------------- attraction + speed --
struct NodeOut {
  double sw, tr;
};

// Gravity, force store and swing/traction for node i given its summed force.
__device__ __forceinline__ NodeOut finish_node(uint32_t i, float fx, float fy, float fz, float4 pi, float deg,
                                               const KParams& P, const float4* old_force, float4* force,
                                               float2* stats) {
  const float r0 = fmaxf(len3(pi.x, pi.y, pi.z), 1.0e-3f);
  const float gd = __fmul_rn(P.gravity, deg);
  if (P.strong_gravity) {
    fx = __fsub_rn(fx, __fmul_rn(pi.x, gd));
    fy = __fsub_rn(fy, __fmul_rn(pi.y, gd));
    fz = __fsub_rn(fz, __fmul_rn(pi.z, gd));
  } else {
    fx = __fsub_rn(fx, __fmul_rn(__fdiv_rn(pi.x, r0), gd));
    fy = __fsub_rn(fy, __fmul_rn(__fdiv_rn(pi.y, r0), gd));
    fz = __fsub_rn(fz, __fmul_rn(__fdiv_rn(pi.z, r0), gd));
  }
  const float4 o = old_force[i];
  force[i] = make_float4(fx, fy, fz, 0.0f);
  const float swing = __fmul_rn(deg, len3(__fsub_rn(o.x, fx), __fsub_rn(o.y, fy), __fsub_rn(o.z, fz)));
  const float trac = __fmul_rn(__fmul_rn(deg, 0.5f), len3(__fadd_rn(o.x, fx), __fadd_rn(o.y, fy), __fadd_rn(o.z, fz)));
  stats[i] = make_float2(swing, trac);
  NodeOut r{0.0, 0.0};
  if (isfinite(swing) && isfinite(trac)) {
    r.sw = (double)swing;
    r.tr = (double)trac;
  }
  return r;
}

__device__ __forceinline__ void att_term(const float4 q, const float4 pi, const KParams& P, float& fx, float& fy,
                                         float& fz) {
  const float dx = __fsub_rn(q.x, pi.x), dy = __fsub_rn(q.y, pi.y), dz = __fsub_rn(q.z, pi.z);
  if (!P.lin_log && P.att_w == 1.0f) {  // d * 1.0 == d exactly: skip the multiply
    fx = __fadd_rn(fx, dx);
    fy = __fadd_rn(fy, dy);
    fz = __fadd_rn(fz, dz);
    return;
  }
  float att = P.att_w;
  if (P.lin_log) {
    const float r = fmaxf(len3(dx, dy, dz), 1.0e-3f);
    att = __fdiv_rn(__fmul_rn(P.att_w, logf(__fadd_rn(1.0f, r))), r);
  }
  fx = __fadd_rn(fx, __fmul_rn(dx, att));
  fy = __fadd_rn(fy, __fmul_rn(dy, att));
  fz = __fadd_rn(fz, __fmul_rn(dz, att));
}

// fa2_speed.rs:48-100 on the device, f64, single thread.
__device__ void speed_update(DevState* st, uint32_t n, float jitter_tolerance, double ts, double tt) {
  if (!(ts > 0.0) || !(tt > 0.0) || n == 0) return;
  const double nn = (double)n;
  const double jtol = (double)jitter_tolerance;
  const double est = 0.05 * sqrt(nn);
  const double min_jt = sqrt(est);
  const double max_jt = 10.0;
  double jt = jtol * fmax(min_jt, fmin(max_jt, est * tt / (nn * nn)));
  const float min_eff = 0.05f;
  float eff = st->speed_eff;
  float speed = st->speed;
  if (ts / tt > 2.0) {
    if (eff > min_eff) eff = __fmul_rn(eff, 0.5f);
    jt = fmax(jt, jtol);
  }
  const double target = jt * (double)eff * tt / ts;
  if (ts > jt * tt) {
    if (eff > min_eff) eff = __fmul_rn(eff, 0.7f);
  } else if (speed < 1000.0f) {
    eff = __fmul_rn(eff, 1.3f);
  }
  const double sp = (double)speed;
  st->speed = (float)(sp + fmin(target - sp, 0.5 * sp));
  st->speed_eff = eff;
}

__global__ void __launch_bounds__(ATT_THREADS)
k_att(const uint32_t* __restrict__ order, const uint32_t* __restrict__ off, const uint32_t* __restrict__ nbr,
      const float4* __restrict__ pos, const float4* __restrict__ frep, const float4* __restrict__ old_force,
      const float* __restrict__ degf, KParams P, DevState* st, float4* __restrict__ force,
      float2* __restrict__ stats, double2* __restrict__ partials, uint32_t n_graphs) {
  __shared__ double red_sw[ATT_THREADS / 32], red_tr[ATT_THREADS / 32];
  __shared__ float hub_sum[3][ATT_THREADS / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const bool skip_all = st->error != 0u;
  double sw = 0.0, tr = 0.0;
  if (!skip_all) {
    if (blockIdx.x < P.n_hubs) {
      // One block per hub: strided partial sums, fixed-shape tree reduction.
      const uint32_t i0 = order[blockIdx.x];
      const uint32_t i = JC_IN_BOUNDS(i0, P.n, &st->error) ? i0 : 0u;
      const float4 pi = pos[i];
      float fx = 0.0f, fy = 0.0f, fz = 0.0f;
      for (uint32_t k = off[i] + threadIdx.x; k < off[i + 1]; k += ATT_THREADS) {
        const uint32_t u = nbr[k];
        if (JC_IN_BOUNDS(u, P.n, &st->error)) att_term(pos[u], pi, P, fx, fy, fz);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        fx = __fadd_rn(fx, __shfl_xor_sync(0xFFFFFFFFu, fx, o));
        fy = __fadd_rn(fy, __shfl_xor_sync(0xFFFFFFFFu, fy, o));
        fz = __fadd_rn(fz, __shfl_xor_sync(0xFFFFFFFFu, fz, o));
      }
      if (lane == 0) { hub_sum[0][w] = fx; hub_sum[1][w] = fy; hub_sum[2][w] = fz; }
      __syncthreads();
      if (threadIdx.x == 0) {
        float sx = 0.0f, sy = 0.0f, sz = 0.0f;
        for (int ww = 0; ww < ATT_THREADS / 32; ++ww) {
          sx = __fadd_rn(sx, hub_sum[0][ww]);
          sy = __fadd_rn(sy, hub_sum[1][ww]);
          sz = __fadd_rn(sz, hub_sum[2][ww]);
        }
        const float4 fr = frep[i];
        NodeOut r = finish_node(i, __fadd_rn(fr.x, sx), __fadd_rn(fr.y, sy), __fadd_rn(fr.z, sz), pi, degf[i], P,
                                old_force, force, stats);
        sw = r.sw;
        tr = r.tr;
      }
    } else if (blockIdx.x < P.n_hubs + (P.n_med + ATT_THREADS / 32 - 1) / (ATT_THREADS / 32)) {
      // One warp per long list: the lanes gather 32 neighbours at a time (the
      // next 32 are in flight while lane 0 adds the current ones in list
      // order), so the sum is the same sequence of roundings as one thread's.
      const uint32_t mi = (blockIdx.x - P.n_hubs) * (ATT_THREADS / 32) + w;
      if (mi < P.n_med) {
        const uint32_t i0 = order[P.n_hubs + mi];
        const uint32_t i = JC_IN_BOUNDS(i0, P.n, &st->error) ? i0 : 0u;
        const float4 pi = pos[i];
        const float4 fr = frep[i];
        float fx = fr.x, fy = fr.y, fz = fr.z;
        const uint32_t e0 = off[i], e1 = off[i + 1];
        auto gather = [&](uint32_t k) {
          const uint32_t u = __ldg(nbr + k);
          return JC_IN_BOUNDS(u, P.n, &st->error) ? __ldg(pos + u) : pi;
        };
        float4 q = e0 + lane < e1 ? gather(e0 + lane) : pi;
        for (uint32_t base = e0; base < e1; base += 32) {
          const float4 cur = q;
          const uint32_t nk = base + 32 + lane;
          if (base + 32 < e1) q = nk < e1 ? gather(nk) : pi;
          float tx = -0.0f, ty = -0.0f, tz = -0.0f;  // -0 + term = term, signed zeros included
          att_term(cur, pi, P, tx, ty, tz);
          const uint32_t cnt = min(32u, e1 - base);
          for (uint32_t l = 0; l < cnt; ++l) {
            const float ax = __shfl_sync(0xFFFFFFFFu, tx, l);
            const float ay = __shfl_sync(0xFFFFFFFFu, ty, l);
            const float az = __shfl_sync(0xFFFFFFFFu, tz, l);
            fx = __fadd_rn(fx, ax);
            fy = __fadd_rn(fy, ay);
            fz = __fadd_rn(fz, az);
          }
        }
        if (lane == 0) {
          NodeOut r = finish_node(i, fx, fy, fz, pi, degf[i], P, old_force, force, stats);
          sw = r.sw;
          tr = r.tr;
        }
      }
    } else {
      const uint32_t med_blocks = (P.n_med + ATT_THREADS / 32 - 1) / (ATT_THREADS / 32);
      const uint32_t t = P.n_hubs + P.n_med + (blockIdx.x - P.n_hubs - med_blocks) * ATT_THREADS + threadIdx.x;
      const uint32_t i0 = t < P.n ? order[t] : 0u;
      const bool have = t < P.n && JC_IN_BOUNDS(i0, P.n, &st->error);
      const uint32_t i = have ? i0 : 0u;
      const float4 pi = have ? pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 fr = have ? frep[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      float fx = fr.x, fy = fr.y, fz = fr.z;
      const uint32_t e0 = have ? off[i] : 0u, e1 = have ? off[i + 1] : 0u;
      if (have) {
        uint32_t k = e0;
        // ids up to a 16-byte boundary one by one, then eight ids in two
        // vector loads and eight gathers in flight, terms always in list order
        auto gather = [&](uint32_t u) { return JC_IN_BOUNDS(u, P.n, &st->error) ? __ldg(pos + u) : pi; };
        for (; k < e1 && (reinterpret_cast<uintptr_t>(nbr + k) & 15u); ++k)
          att_term(gather(__ldg(nbr + k)), pi, P, fx, fy, fz);
        for (; k + 8 <= e1; k += 8) {
          const uint4 a = __ldg(reinterpret_cast<const uint4*>(nbr + k));
          const uint4 b = __ldg(reinterpret_cast<const uint4*>(nbr + k + 4));
          const uint32_t o[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
          float4 q[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) q[u] = gather(o[u]);
#pragma unroll
          for (int u = 0; u < 8; ++u) att_term(q[u], pi, P, fx, fy, fz);
        }
        for (; k < e1; ++k) att_term(gather(__ldg(nbr + k)), pi, P, fx, fy, fz);
      }
      if (have) {
        NodeOut r = finish_node(i, fx, fy, fz, pi, degf[i], P, old_force, force, stats);
        sw = r.sw;
        tr = r.tr;
      }
    }
  }
  // deterministic block reduction (fixed shape)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sw += __shfl_xor_sync(0xFFFFFFFFu, sw, o);
    tr += __shfl_xor_sync(0xFFFFFFFFu, tr, o);
  }
  if (lane == 0) { red_sw[w] = sw; red_tr[w] = tr; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int ww = 0; ww < ATT_THREADS / 32; ++ww) { a += red_sw[ww]; b += red_tr[ww]; }
    partials[blockIdx.x] = make_double2(a, b);
    __threadfence();
    last = atomicAdd(&st->att_done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (w == 0) {
    double a = 0.0, b = 0.0;
    for (uint32_t k = lane; k < gridDim.x; k += 32) {
      double2 v = __ldcg(&partials[k]);
      a += v.x;
      b += v.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
      b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
    }
    if (lane == 0) {
      if (!skip_all) {
        if (n_graphs == 1) speed_update(st, P.n, P.jitter_tolerance, a, b);  // batches: k_speed_graphs
        st->steps_done += 1u;
      }
      st->att_done = 0;
    }
  }
}

// --------------------------------------------------------------- apply --
__global__ void __launch_bounds__(APPLY_THREADS)
k_apply(float4* __restrict__ pos, float4* __restrict__ old_force, const float4* __restrict__ force,
        const float* __restrict__ degf, KParams P, const DevState* st, float* __restrict__ xyz, Forest F) {
  if (st->error) return;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const float speed = F.n_graphs > 1 ? F.gspeed[F.node_graph[i]].x : st->speed;
  const float4 f = force[i];
  const float4 o = old_force[i];
  const float deg = degf[i];
  const float swinging = __fmul_rn(deg, len3(__fsub_rn(o.x, f.x), __fsub_rn(o.y, f.y), __fsub_rn(o.z, f.z)));
  float factor = __fdiv_rn(speed, __fadd_rn(1.0f, __fsqrt_rn(__fmul_rn(speed, swinging))));
  const float df = len3(f.x, f.y, f.z);
  if (P.max_disp > 0.0f && df > 1.0e-9f) factor = fminf(factor, __fdiv_rn(P.max_disp, df));
  const float k = __fmul_rn(factor, P.time_step);
  float4 p = pos[i];
  p.x = __fadd_rn(p.x, __fmul_rn(f.x, k));
  p.y = __fadd_rn(p.y, __fmul_rn(f.y, k));
  p.z = __fadd_rn(p.z, __fmul_rn(f.z, k));
  p.w = 0.0f;
  pos[i] = p;
  old_force[i] = make_float4(f.x, f.y, f.z, 0.0f);
  xyz[3 * (size_t)i] = p.x;
  xyz[3 * (size_t)i + 1] = p.y;
  xyz[3 * (size_t)i + 2] = p.z;
}

__global__ void k_pack_xyz(const float4* __restrict__ v, uint32_t n, float* __restrict__ xyz) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = v[i];
  xyz[3 * (size_t)i] = p.x;
  xyz[3 * (size_t)i + 1] = p.y;
  xyz[3 * (size_t)i + 2] = p.z;
}

__global__ void k_unpack_xyz(const float* __restrict__ xyz, uint32_t n, float4* __restrict__ v) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  v[i] = make_float4(xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2], 0.0f);
}

#include "jc_fa2_tile.cuh"

// ============================================================== host ==
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    if (count <= n && p) return;
    free();
    size_t c = std::max<size_t>(count, 1);
    p = static_cast<T*>(DevicePool::instance().alloc(c * sizeof(T)));
    n = c;
  }
  void free() {
    DevicePool::instance().free(p);
    p = nullptr;
    n = 0;
  }
  ~DevBuf() { free(); }
};

inline uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// Mass of every body of a canonical CSR: 1 + its row length (the
// non-self CSR entries, fa2_bh.rs:264-294), as the host computes it.
__global__ void k_degf_from_offsets(const uint32_t* __restrict__ off, uint32_t n, float* __restrict__ degf) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) degf[i] = __fadd_rn((float)(off[i + 1] - off[i]), 1.0f);
}

// Attraction schedule: nodes by list length, longest first, stable (ties in
// node order), lengths capped at 2^20. Lists of at least 1,024 entries (few)
// are sorted directly; the others by a counting sort over their 1,024 lengths
// with per-thread histograms and a stable parallel scatter.
inline void schedule_by_length(const uint32_t* lo, uint32_t n, uint32_t* order) {
  constexpr uint32_t CUT = 1024;
  auto len = [&](uint32_t i) { return std::min<uint32_t>(lo[i + 1] - lo[i], 1u << 20); };
  // bucket 0: lengths >= CUT; bucket 1 + (CUT - 1 - l): length l < CUT
  auto bucket = [&](uint32_t i) { const uint32_t l = len(i); return l >= CUT ? 0u : 1u + (CUT - 1u - l); };
  constexpr uint32_t NB = CUT + 1;
  int T = 1;
#ifdef _OPENMP
  T = std::max(1, std::min(omp_get_max_threads(), (int)std::max<uint32_t>(1, n / 65536)));
#endif
  std::vector<uint32_t> hist((size_t)T * NB, 0);
#pragma omp parallel num_threads(T)
  {
#ifdef _OPENMP
    const int t = omp_get_thread_num();
#else
    const int t = 0;
#endif
    const uint64_t a = (uint64_t)n * t / T, b = (uint64_t)n * (t + 1) / T;
    uint32_t* h = &hist[(size_t)t * NB];
    for (uint64_t i = a; i < b; ++i) ++h[bucket((uint32_t)i)];
#pragma omp barrier
#pragma omp single
    {
      uint32_t run = 0;
      for (uint32_t k = 0; k < NB; ++k)
        for (int q = 0; q < T; ++q) {
          const uint32_t c = hist[(size_t)q * NB + k];
          hist[(size_t)q * NB + k] = run;
          run += c;
        }
    }
    for (uint64_t i = a; i < b; ++i) order[h[bucket((uint32_t)i)]++] = (uint32_t)i;
  }
  // the long lists (bucket 0, in node order) by length, descending, stable
  uint32_t m = 0;
  while (m < n && len(order[m]) >= CUT) ++m;
  std::stable_sort(order, order + m, [&](uint32_t x, uint32_t y) { return len(x) > len(y); });
}

// Clears *ok when some row is not strictly increasing, holds a self-loop, or
// has an entry (v, u) without its (u, v). One thread per CSR entry (a hub
// row's entries spread over many blocks): the row of entry e is the last v
// with off[v] <= e, searched inside the rows that the block's first and last
// entries fall in. The host has already checked that off is non-decreasing
// from 0 to m and every id is below n.
// Symmetry: nodes are ordered by (row length, id); an entry (v, u) whose row v
// comes later in that order looks for its (u, v) with a binary search in the
// shorter row u and counts +1, every other entry counts -1 without a search.
// With strictly increasing rows (no duplicate entries), if every search
// succeeds the mirror map takes the +1 entries one-to-one into the -1 entries,
// so the CSR is symmetric exactly when the counts also balance (the counts
// go to CSR_BAL_SLOTS spread words; k_csr_balance sums them). No entry has
// to search a hub's long row, which on scale-free graphs most entries did.
constexpr uint32_t CSR_BAL_SLOTS = 64;
__device__ __forceinline__ uint32_t csr_row_of(const uint32_t* __restrict__ off, uint32_t lo, uint32_t hi,
                                               uint32_t e) {
  // off[lo] <= e < off[hi]
  while (hi - lo > 1) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (off[mid] <= e) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(256) k_csr_canonical(uint32_t n, uint32_t m, const uint32_t* __restrict__ off,
                                                       const uint32_t* __restrict__ nbr, uint32_t* ok,
                                                       int* __restrict__ balance) {
  __shared__ uint32_t s_rows[2];
  __shared__ int s_bal[8];
  const uint32_t base = blockIdx.x * blockDim.x;
  if (threadIdx.x < 2) {
    const uint32_t e = threadIdx.x == 0 ? base : min(base + blockDim.x, m) - 1;
    s_rows[threadIdx.x] = csr_row_of(off, 0, n, e);
  }
  __syncthreads();
  const uint32_t e = base + threadIdx.x;
  int bal = 0;
  if (e < m) {
    const uint32_t v = csr_row_of(off, s_rows[0], s_rows[1] + 1, e);
    const uint32_t u = nbr[e];
    if (u == v || (e > off[v] && nbr[e - 1] >= u)) {
      *ok = 0u;
    } else {
      const uint32_t ub = off[u], ue = off[u + 1];
      const uint32_t dv = off[v + 1] - off[v], du = ue - ub;
      if (dv > du || (dv == du && v > u)) {
        uint32_t lo = ub, hi = ue;
        while (lo < hi) {
          const uint32_t mid = lo + (hi - lo) / 2;
          if (nbr[mid] < v) lo = mid + 1; else hi = mid;
        }
        if (lo >= ue || nbr[lo] != v) *ok = 0u;
        bal = 1;
      } else {
        bal = -1;
      }
    }
  }
  bal = __reduce_add_sync(0xFFFFFFFFu, bal);
  if ((threadIdx.x & 31) == 0) s_bal[threadIdx.x >> 5] = bal;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < 8; ++w) t += s_bal[w];
    if (t) atomicAdd(balance + (blockIdx.x % CSR_BAL_SLOTS), t);
  }
}

// Clears *ok unless the +1 and -1 counts of k_csr_canonical balance.
__global__ void k_csr_balance(const int* __restrict__ balance, uint32_t* ok) {
  int t = balance[threadIdx.x];
  t = __reduce_add_sync(0xFFFFFFFFu, t);
  __shared__ int s[CSR_BAL_SLOTS / 32];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    int sum = 0;
    for (uint32_t w = 0; w < CSR_BAL_SLOTS / 32; ++w) sum += s[w];
    if (sum != 0) *ok = 0u;
  }
}

class Fa2Engine : public Engine {
 public:
  explicit Fa2Engine(bool bh) : bh_(bh) {
    desc_.id = bh ? "fa2-bh" : "fa2-brute";
    desc_.kind = 1;
    desc_.display_name = bh ? "ForceAtlas2 (Barnes-Hut, B200)" : "ForceAtlas2 (brute force, B200)";
    desc_.description =
        bh ? "O(n log n) ForceAtlas2 on B200: the reference octree rebuilt on the device every step "
             "(Morton-digit radix sort, exact pre-order octree, bottom-up centre of mass), a "
             "warp-cooperative theta walk, CSR attraction with the adaptive-speed reduction fused, "
             "all replayed from a CUDA graph."
           : "O(n^2) ForceAtlas2 on B200: all-pairs repulsion tiled through shared memory, same "
             "attraction, gravity and adaptive speed as fa2-bh.";
    desc_.needs_edges = 1;
    desc_.needs_cpu_positions = 1;
    desc_.needs_gpu_positions_buffer = 0;
  }
  ~Fa2Engine() override { release(); }

  const jc_descriptor& descriptor() const override { return desc_; }

  void set_params(const char* json) override {
    decode_fa2(json, &s_, bh_, bh_ ? "fa2-bh" : "fa2-brute");
    drop_graph();
  }

  void init(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint64_t nnz, const float* xyz) override {
    Trace tr("fa2.init");
    // offsets and pointers here; the neighbour ids are range-checked by the
    // staged upload in init_common, in the same pass that copies them
    if (n > 0 && xyz == nullptr) fail(JC_ERR_ARG, "positions must be non-null for a non-empty graph");
    validate_csr_offsets(n, off, nbr, nnz);
    tr.mark("validate_offsets");
    graph_off_host_.assign({0u, n});
    ids_checked_ = false;
    try {
      init_common(n, off, nbr, nnz, xyz);
    } catch (...) {
      ids_checked_ = true;
      throw;
    }
    ids_checked_ = true;
  }

  // Positions already in device memory (3n floats, complete before the
  // call): packed on the device instead of staged through the host.
  void reinit_device(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint64_t nnz,
                     const float* d_xyz) override {
    validate_csr_arrays(n, off, nbr, nnz);
    if (n && !d_xyz) fail(JC_ERR_ARG, "positions must be non-null for a non-empty graph");
    graph_off_host_.assign({0u, n});
    dev_xyz_ = d_xyz;
    try {
      init_common(n, off, nbr, nnz, nullptr);
    } catch (...) {
      dev_xyz_ = nullptr;
      throw;
    }
    dev_xyz_ = nullptr;
  }

  // A batch of independent graphs laid out together: graph g has graph_nodes[g]
  // nodes, its CSR (local ids, offsets starting at 0) follows the previous
  // graph's in offsets/neighbors, and its 3*n_g positions follow in xyz.
  void init_batch(uint32_t n_graphs, const uint32_t* graph_nodes, const uint32_t* offsets,
                  const uint32_t* neighbors, const float* xyz) override {
    if (!bh_) fail(JC_ERR_ARG, "batches are laid out by fa2-bh");
    if (n_graphs == 0 || graph_nodes == nullptr || offsets == nullptr)
      fail(JC_ERR_ARG, "a batch needs at least one graph");
    if (n_graphs > 65536) fail(JC_ERR_ARG, "at most 65536 graphs per batch");
    uint64_t total_n = 0, total_e = 0;
    {
      const uint32_t* o = offsets;
      for (uint32_t g = 0; g < n_graphs; ++g) {
        total_n += graph_nodes[g];
        total_e += o[graph_nodes[g]];
        o += graph_nodes[g] + 1;
      }
    }
    if (total_n > 0xFFFFFFF0ull || total_e > 0xFFFFFFF0ull) fail(JC_ERR_ARG, "batch too large");
    std::vector<uint32_t> goff(n_graphs + 1, 0), off((size_t)total_n + 1, 0), nb(total_e);
    const uint32_t* o = offsets;
    const uint32_t* nbp = neighbors;
    uint32_t node_base = 0, edge_base = 0;
    for (uint32_t g = 0; g < n_graphs; ++g) {
      const uint32_t ng = graph_nodes[g];
      const uint32_t eg = o[ng];
      validate_csr(ng, o, nbp, eg, ng ? xyz + 3 * (size_t)node_base : xyz);
      for (uint32_t v = 0; v < ng; ++v) off[node_base + v + 1] = edge_base + o[v + 1];
      for (uint32_t e = 0; e < eg; ++e) nb[edge_base + e] = node_base + nbp[e];
      node_base += ng;
      edge_base += eg;
      goff[g + 1] = node_base;
      o += ng + 1;
      nbp += eg;
    }
    graph_off_host_ = goff;
    init_common((uint32_t)total_n, off.data(), nb.data(), total_e, xyz);
  }

  void init_common(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint64_t nnz, const float* xyz) {
    Trace tr("fa2.init_common");
    ensure_stream();
    tr.mark("stream");
    n_ = n;
    initialized_ = false;
    drop_graph();
    // ---- the CSR to the device, checked there (fa2_bh.rs:246-294) -------
    // A host check of symmetry costs one cache-missing binary search per
    // entry, so the device checks. Its verdict is read at the end of init:
    // everything in between assumes the common canonical CSR (the CSR on the
    // device is then already the attraction list) and overlaps the tail of
    // the copy and the check; a CSR that is not canonical is then rebuilt on
    // the host and every buffer that depends on it is written again.
    aoff_.alloc((size_t)n + 1);
    anbr_.alloc(std::max<uint64_t>(nnz, 1));
    if (n) {
      okb_.alloc(1 + CSR_BAL_SLOTS);  // the verdict word, then the balance slots
      HostStager& up = HostStager::instance();
      up.upload(aoff_.p, off, sizeof(uint32_t) * ((size_t)n + 1), stream_);
      if (nnz) {
        const uint32_t mx = up.upload_u32_max(anbr_.p, nbr, nnz, stream_);
        if (!ids_checked_ && mx >= n)
          fail(JC_ERR_ARG, "neighbor id " + std::to_string(mx) + " out of range for " + std::to_string(n) + " nodes");
      }
      JC_CUDA_CHECK(cudaMemsetAsync(okb_.p, 1, 4, stream_));  // nonzero: canonical until the check clears it
      if (nnz) {
        int* bal = reinterpret_cast<int*>(okb_.p + 1);
        JC_CUDA_CHECK(cudaMemsetAsync(bal, 0, sizeof(int) * CSR_BAL_SLOTS, stream_));
        k_csr_canonical<<<(uint32_t)cdiv(nnz, 256), 256, 0, stream_>>>(n, (uint32_t)nnz, aoff_.p, anbr_.p, okb_.p,
                                                                       bal);
        k_csr_balance<<<1, CSR_BAL_SLOTS, 0, stream_>>>(bal, okb_.p);
      }
      JC_CUDA_CHECK(cudaGetLastError());
      JC_CUDA_CHECK(cudaMemcpyAsync(ok_host_, okb_.p, 4, cudaMemcpyDeviceToHost, stream_));
    }
    tr.mark("csr_upload");
    hub_threshold_ = s_.hub_threshold ? s_.hub_threshold : DEFAULT_HUB_THRESHOLD;
    walk_group_ = DEFAULT_WALK_GROUP;
    if (s_.walk_group) {
      uint32_t g = s_.walk_group;
      if (g != 1 && g != 2 && g != 4 && g != 8 && g != 16 && g != 32)
        fail(JC_ERR_ARG, "walk_group must be 1, 2, 4, 8, 16 or 32");
      walk_group_ = g;
    }
    std::unique_ptr<uint32_t[]> order(new uint32_t[std::max<uint32_t>(n, 1)]);
    // Attraction schedule: nodes by edge-list length, longest first (stable);
    // lo = the attraction-list offsets.
    auto schedule = [&](const uint32_t* lo) {
      schedule_by_length(lo, n, order.get());
      n_hubs_ = 0;
      while (n_hubs_ < n && lo[order[n_hubs_] + 1] - lo[order[n_hubs_]] >= hub_threshold_) ++n_hubs_;
      n_med_ = 0;
      const uint32_t warp_thr = s_.warp_threshold ? s_.warp_threshold : DEFAULT_WARP_THRESHOLD;
      while (n_hubs_ + n_med_ < n && lo[order[n_hubs_ + n_med_] + 1] - lo[order[n_hubs_ + n_med_]] >= warp_thr)
        ++n_med_;
      n_att_ = lo[n];
      att_blocks_ = n_hubs_ + cdiv(n_med_, ATT_THREADS / 32) + cdiv(n - n_hubs_ - n_med_, ATT_THREADS);
    };
    // A canonical CSR (rows sorted and duplicate-free, no self-loops,
    // symmetric: what csr_from_pairs produces) is its own attraction list:
    // node i's edges in edge-index order are the v < u edges of lower rows
    // that end at i (row i's entries below i, in increasing v) followed by its
    // own (row i's entries above i), i.e. row i; a node's degree is its row
    // length.
    schedule(off);
    tr.mark("host_prep");
    // ---- device buffers -------------------------------------------------
    pos_.alloc(n); old_.alloc(n); force_.alloc(n); frep_.alloc(n); degf_.alloc(n); stats_.alloc(n);
    aorder_.alloc(n); xyz_.alloc((size_t)3 * n);
    state_.alloc(1); bbox_part_.alloc(6 * BBOX_BLOCKS);
    partials_.alloc(std::max<uint32_t>(att_blocks_, 1));
    if (bh_) alloc_tree(n);
    setup_forest(n);
    auto setup_schedule_modes = [&]() {
      const uint32_t G = (uint32_t)graph_off_host_.size() - 1;
      uint32_t biggest = 0;
      for (uint32_t g = 0; g < G; ++g) biggest = std::max(biggest, graph_off_host_[g + 1] - graph_off_host_[g]);
      tile_ok_ = bh_ && G > 1 && n_hubs_ == 0 && biggest <= TILE_MAX_NODES;
      tile_mode_ = tile_ok_ && s_.batch_schedule == 1;
      tile_synced_ = false;
      tile_probe_ms_ = 0.0f;
      tile_mult_ = 3;
      if (tile_mode_) setup_tile();
    };
    setup_schedule_modes();
    tr.mark("alloc");
    if (n) {
      // positions: the caller's xyz to xyz_ (host arrays) or read in place
      // (device arrays), then widened to float4 on the device
      if (!dev_xyz_) HostStager::instance().upload(xyz_.p, xyz, sizeof(float) * 3 * (size_t)n, stream_);
      k_unpack_xyz<<<cdiv(n, 256), 256, 0, stream_>>>(dev_xyz_ ? dev_xyz_ : xyz_.p, n, pos_.p);
      JC_CUDA_CHECK(cudaGetLastError());
      // masses from the row lengths (a canonical CSR's degrees)
      k_degf_from_offsets<<<cdiv(n, 256), 256, 0, stream_>>>(aoff_.p, n, degf_.p);
      JC_CUDA_CHECK(cudaGetLastError());
    }
    JC_CUDA_CHECK(cudaMemsetAsync(old_.p, 0, sizeof(float4) * std::max<uint32_t>(n, 1), stream_));
    JC_CUDA_CHECK(cudaMemsetAsync(force_.p, 0, sizeof(float4) * std::max<uint32_t>(n, 1), stream_));
    JC_CUDA_CHECK(cudaMemsetAsync(stats_.p, 0, sizeof(float2) * std::max<uint32_t>(n, 1), stream_));
    HostStager::instance().upload(aorder_.p, order.get(), sizeof(uint32_t) * n, stream_);
    DevState st0;
    std::memset(&st0, 0, sizeof(st0));
    st0.speed = 1.0f;  // fa2_speed.rs:32-39
    st0.speed_eff = 1.0f;
    JC_CUDA_CHECK(cudaMemcpyAsync(state_.p, &st0, sizeof(st0), cudaMemcpyHostToDevice, stream_));
    if (n && dev_xyz_) {  // (host positions are in xyz_ already)
      k_pack_xyz<<<cdiv(n, 256), 256, 0, stream_>>>(pos_.p, n, xyz_.p);
      JC_CUDA_CHECK(cudaGetLastError());
    }
    // A single graph's step graph is captured now, while the device still
    // works through the uploads and the CSR check (capture only records).
    if (n && bh_ && forest_.n_graphs == 1) ensure_graph();
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    const bool canonical = n == 0 || *ok_host_ != 0u;
    tr.mark("upload_sync");
    if (!canonical) {
      drop_graph();  // captured for the canonical schedule
      // Per-node edge lists in the shader's edge-scan order (wgsl:160-181):
      // node i meets its edges in edge-index order; self-loops skipped.
      std::vector<uint32_t> deg(n, 0), aoff, anbr;
      std::vector<uint32_t> ev, eu;  // (v,u) edges, v < u, edge-index order
      for (uint32_t v = 0; v < n; ++v)
        for (uint32_t e = off[v]; e < off[v + 1]; ++e) {
          uint32_t u = nbr[e];
          if (u == v) continue;
          deg[v] += 1;
          if (v < u) { ev.push_back(v); eu.push_back(u); }
        }
      aoff.assign((size_t)n + 1, 0);
      for (size_t e = 0; e < ev.size(); ++e) { aoff[ev[e] + 1]++; aoff[eu[e] + 1]++; }
      for (uint32_t i = 0; i < n; ++i) aoff[i + 1] += aoff[i];
      anbr.resize(aoff[n]);
      std::vector<uint32_t> cur(aoff.begin(), aoff.end() - 1);
      for (size_t e = 0; e < ev.size(); ++e) {
        anbr[cur[ev[e]]++] = eu[e];
        anbr[cur[eu[e]]++] = ev[e];
      }
      schedule(aoff.data());
      std::vector<float> degf(n);
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < (int64_t)n; ++i) degf[i] = (float)deg[i] + 1.0f;
      partials_.alloc(std::max<uint32_t>(att_blocks_, 1));
      setup_schedule_modes();
      HostStager::instance().upload(degf_.p, degf.data(), sizeof(float) * n, stream_);
      anbr_.alloc(std::max<uint32_t>(n_att_, 1));
      JC_CUDA_CHECK(cudaMemcpyAsync(aoff_.p, aoff.data(), sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice, stream_));
      if (n_att_)
        JC_CUDA_CHECK(cudaMemcpyAsync(anbr_.p, anbr.data(), sizeof(uint32_t) * n_att_, cudaMemcpyHostToDevice, stream_));
      HostStager::instance().upload(aorder_.p, order.get(), sizeof(uint32_t) * n, stream_);
      JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
      tr.mark("general_csr");
    }
    warn_accum_ = 0;
    host_steps_ = 0;
    initialized_ = true;
    (void)nnz;
  }

  void step(float* out_xyz) override {
    require_init();
    if (n_ == 0) return;
    run_steps(1, out_xyz);
  }

  void step_many(uint32_t iters, float* out_xyz) override {
    require_init();
    if (n_ == 0 || iters == 0) return;
    run_steps(iters, out_xyz);
  }

  void graph_speed(uint32_t g, float* sp, float* eff) override {
    require_init();
    const uint32_t G = (uint32_t)graph_off_host_.size() - 1;
    if (g >= G) fail(JC_ERR_ARG, "graph index out of range");
    if (G == 1) {
      speed(sp, eff);
      return;
    }
    float2 v;
    JC_CUDA_CHECK(cudaMemcpyAsync(&v, gspeed_.p + g, sizeof(v), cudaMemcpyDeviceToHost, stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    if (sp) *sp = v.x;
    if (eff) *eff = v.y;
  }

  // Autotuner: times `probe` steps of every walk-group schedule from the same
  // device snapshot of the state, restores the snapshot after each, and keeps
  // the fastest. ms_out (6 entries: groups 1, 2, 4, 8, 16, 32) may be NULL.
  uint32_t autotune(uint32_t probe, float* ms_out) override {
    require_init();
    if (!bh_ || n_ == 0) return walk_group_;
    const uint32_t groups[6] = {1, 2, 4, 8, 16, 32};
    const uint32_t G = (uint32_t)graph_off_host_.size() - 1;
    DevBuf<float4> spos, sold;
    DevBuf<float2> sgs;
    DevBuf<DevState> sst;
    spos.alloc(n_); sold.alloc(n_); sst.alloc(1);
    if (G > 1) sgs.alloc(G);
    auto snap = [&](bool save) {
      auto cp = [&](void* dst, const void* src, size_t bytes) {
        JC_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream_));
      };
      if (save) {
        cp(spos.p, pos_.p, sizeof(float4) * n_); cp(sold.p, old_.p, sizeof(float4) * n_);
        cp(sst.p, state_.p, sizeof(DevState));
        if (G > 1) cp(sgs.p, gspeed_.p, sizeof(float2) * G);
      } else {
        cp(pos_.p, spos.p, sizeof(float4) * n_); cp(old_.p, sold.p, sizeof(float4) * n_);
        cp(state_.p, sst.p, sizeof(DevState));
        if (G > 1) cp(gspeed_.p, sgs.p, sizeof(float2) * G);
      }
    };
    snap(true);
    const uint32_t keep_steps = host_steps_;
    float best = 0.0f;
    uint32_t best_g = walk_group_;
    const bool was_tile = tile_mode_;
    tile_mode_ = false;
    for (int c = 0; c < 6; ++c) {
      walk_group_ = groups[c];
      drop_graph();
      float ms = 0.0f;
      time_steps(probe, &ms, nullptr);
      if (ms_out) ms_out[c] = ms / (float)std::max(probe, 1u);
      if (c == 0 || ms < best) { best = ms; best_g = groups[c]; }
      snap(false);
      host_steps_ = keep_steps;
    }
    // the tile schedule (one CTA per graph), when every graph qualifies
    bool tile_best = false;
    tile_probe_ms_ = 0.0f;
    if (tile_ok_) {
      tile_mode_ = true;
      tile_synced_ = false;
      if (!t_gsteps_.p) setup_tile();
      float ms = 0.0f;
      time_steps(probe, &ms, nullptr);
      tile_probe_ms_ = ms / (float)std::max(probe, 1u);
      tile_best = ms < best;
      snap(false);
      host_steps_ = keep_steps;
      tile_synced_ = false;
    }
    (void)was_tile;
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    walk_group_ = best_g;
    tile_mode_ = tile_best;
    drop_graph();
    return best_g;
  }

  void positions(float* out) override {
    require_init();
    if (n_ == 0) return;
    JC_CUDA_CHECK(cudaMemcpyAsync(out, xyz_.p, sizeof(float) * 3 * n_, cudaMemcpyDeviceToHost, stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
  }

  void positions_range(uint64_t first, uint64_t count, float* out) override {
    require_init();
    if (first > n_ || count > n_ - first) fail(JC_ERR_ARG, "node range out of bounds");
    if (count == 0) return;
    JC_CUDA_CHECK(cudaMemcpyAsync(out, xyz_.p + 3 * first, sizeof(float) * 3 * count, cudaMemcpyDeviceToHost,
                                  stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
  }

  void forces(float* out_xyz, float* out_stats) override {
    require_init();
    if (n_ == 0) return;
    std::vector<float> f4((size_t)4 * n_);
    JC_CUDA_CHECK(cudaMemcpyAsync(f4.data(), force_.p, sizeof(float4) * n_, cudaMemcpyDeviceToHost, stream_));
    if (out_stats)
      JC_CUDA_CHECK(cudaMemcpyAsync(out_stats, stats_.p, sizeof(float2) * n_, cudaMemcpyDeviceToHost, stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    for (uint32_t i = 0; i < n_; ++i)
      for (int k = 0; k < 3; ++k) out_xyz[3 * (size_t)i + k] = f4[4 * (size_t)i + k];
  }

  void speed(float* sp, float* eff) override {
    require_init();
    DevState st = read_state();
    if (sp) *sp = st.speed;
    if (eff) *eff = st.speed_eff;
  }

  uint32_t status_bits() override {
    if (!initialized_) return 0;
    DevState st = read_state();
    uint32_t w = st.warn | warn_accum_;
    warn_accum_ = 0;
    uint32_t zero = 0;
    JC_CUDA_CHECK(cudaMemcpyAsync(&state_.p->warn, &zero, sizeof(zero), cudaMemcpyHostToDevice, stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    return w;
  }

  void tree_info(uint32_t* out4) override {
    require_init();
    if (!bh_) fail(JC_ERR_ARG, "fa2-brute builds no tree");
    DevState st = read_state();
    out4[0] = st.n_tree;
    out4[1] = st.n_valid - st.dropped;
    out4[2] = st.max_depth;
    out4[3] = st.dropped;
  }

  void walk_counts(uint64_t* out2) override {
    require_init();
    if (!bh_) fail(JC_ERR_ARG, "fa2-brute walks no tree");
    DevState st = read_state();
    out2[0] = st.n_inter;
    out2[1] = st.n_open;
  }

  void time_steps(uint32_t iters, float* total_ms, float* phase_ms4) override {
    require_init();
    if (n_ == 0 || iters == 0) {
      if (total_ms) *total_ms = 0.0f;
      return;
    }
    if (tile_mode_) {
      // one launch covers all `iters` iterations; no per-phase split
      cudaEvent_t e0, e1;
      JC_CUDA_CHECK(cudaEventCreate(&e0));
      JC_CUDA_CHECK(cudaEventCreate(&e1));
      sync_tile_steps();
      JC_CUDA_CHECK(cudaEventRecord(e0, stream_));
      launch_tile(host_steps_ + iters);
      JC_CUDA_CHECK(cudaEventRecord(e1, stream_));
      JC_CUDA_CHECK(cudaEventSynchronize(e1));
      float ms = 0.0f;
      JC_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
      if (total_ms) *total_ms = ms;
      if (phase_ms4)
        for (int k = 0; k < 4; ++k) phase_ms4[k] = 0.0f;
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      host_steps_ += iters;
      check_state();
      return;
    }
    tile_synced_ = false;
    ensure_graph();
    cudaEvent_t e0, e1;
    JC_CUDA_CHECK(cudaEventCreate(&e0));
    JC_CUDA_CHECK(cudaEventCreate(&e1));
    JC_CUDA_CHECK(cudaEventRecord(e0, stream_));
    for (uint32_t k = 0; k < iters; ++k) launch_step();
    JC_CUDA_CHECK(cudaEventRecord(e1, stream_));
    JC_CUDA_CHECK(cudaEventSynchronize(e1));
    float ms = 0.0f;
    JC_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    if (total_ms) *total_ms = ms;
    if (phase_ms4) {
      // Per-phase device times, averaged over further replays that each end
      // in a synchronisation (replays of the phase graph: the same kernels
      // with event nodes between the phases).
      const uint32_t reps = std::min<uint32_t>(iters, 10);
      for (int k = 0; k < 4; ++k) phase_ms4[k] = 0.0f;
      if (s_.use_graph) ensure_phase_graph();
      for (uint32_t r = 0; r < reps; ++r) {
        if (s_.use_graph) JC_CUDA_CHECK(cudaGraphLaunch(gexec_phase_, stream_));
        else launch_step();
        JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
        for (int k = 0; k < 4; ++k) {
          float t = 0.0f;
          JC_CUDA_CHECK(cudaEventElapsedTime(&t, ev_[k], ev_[k + 1]));
          phase_ms4[k] += t / (float)reps;
        }
      }
      host_steps_ += reps;
    }
    host_steps_ += iters;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_state();
  }

  uint32_t launches_per_step() const override { return tile_mode_ ? 3u : launches_; }

  void schedule_info(uint32_t* tile, float* tile_ms) override {
    if (tile) *tile = tile_mode_ ? 1u : 0u;
    if (tile_ms) *tile_ms = tile_probe_ms_;
  }

  uint32_t node_count() const override { return n_; }
  void enqueue_steps(uint32_t iters) override {
    require_init();
    if (n_ == 0) return;
    if (tile_mode_) {
      sync_tile_steps();
      launch_tile(host_steps_ + iters);
      host_steps_ += iters;
      return;
    }
    tile_synced_ = false;
    ensure_graph();
    for (uint32_t k = 0; k < iters; ++k) launch_step();
    host_steps_ += iters;
  }
  const float* device_xyz() const override { return xyz_.p; }
  cudaStream_t cuda_stream() const override { return stream_; }
  cudaStream_t copy_stream() const override { return copy_; }
  const uint32_t* device_error_word() const override { return state_.p ? &state_.p->error : nullptr; }
  void after_stream_error() override {
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    JC_CUDA_CHECK(cudaMemcpy(hst_, state_.p, sizeof(DevState), cudaMemcpyDeviceToHost));
    host_steps_ = hst_->steps_done;
    if (hst_->error == JC_ERR_CAPACITY) {
      grow_tree();
      fail(JC_ERR_CAPACITY, "the octree outgrew its buffers during a streamed step; the buffers were grown and "
                            "the steps after step " + std::to_string(host_steps_) + " were not run");
    }
    check_state();
  }

  // state: n, speed, speed_eff, steps, pos[4n], old_force[4n], and for a
  // batch of G graphs each graph's (speed, speed_eff)
  uint32_t batch_graphs() const { return graph_off_host_.size() > 2 ? (uint32_t)graph_off_host_.size() - 1 : 0u; }
  uint64_t state_size() override { return 16 + (uint64_t)32 * n_ + (uint64_t)8 * batch_graphs(); }
  void save_state(void* buf) override {
    require_init();
    DevState st = read_state();
    uint8_t* b = (uint8_t*)buf;
    std::memcpy(b, &n_, 4);
    std::memcpy(b + 4, &st.speed, 4);
    std::memcpy(b + 8, &st.speed_eff, 4);
    std::memcpy(b + 12, &st.steps_done, 4);
    if (n_) {
      JC_CUDA_CHECK(cudaMemcpyAsync(b + 16, pos_.p, sizeof(float4) * n_, cudaMemcpyDeviceToHost, stream_));
      JC_CUDA_CHECK(cudaMemcpyAsync(b + 16 + 16 * (size_t)n_, old_.p, sizeof(float4) * n_, cudaMemcpyDeviceToHost, stream_));
    }
    if (batch_graphs())
      JC_CUDA_CHECK(cudaMemcpyAsync(b + 16 + 32 * (size_t)n_, gspeed_.p, sizeof(float2) * batch_graphs(),
                                    cudaMemcpyDeviceToHost, stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
  }
  void load_state(const void* buf, uint64_t len) override {
    require_init();
    if (len != state_size()) fail(JC_ERR_ARG, "state size mismatch");
    const uint8_t* b = (const uint8_t*)buf;
    uint32_t n;
    std::memcpy(&n, b, 4);
    if (n != n_) fail(JC_ERR_ARG, "state is for a graph with a different node count");
    DevState st = read_state();
    std::memcpy(&st.speed, b + 4, 4);
    std::memcpy(&st.speed_eff, b + 8, 4);
    std::memcpy(&st.steps_done, b + 12, 4);
    st.error = 0;
    host_steps_ = st.steps_done;
    JC_CUDA_CHECK(cudaMemcpyAsync(state_.p, &st, sizeof(st), cudaMemcpyHostToDevice, stream_));
    if (n_) {
      JC_CUDA_CHECK(cudaMemcpyAsync(pos_.p, b + 16, sizeof(float4) * n_, cudaMemcpyHostToDevice, stream_));
      JC_CUDA_CHECK(cudaMemcpyAsync(old_.p, b + 16 + 16 * (size_t)n_, sizeof(float4) * n_, cudaMemcpyHostToDevice, stream_));
      k_pack_xyz<<<cdiv(n_, 256), 256, 0, stream_>>>(pos_.p, n_, xyz_.p);
      JC_CUDA_CHECK(cudaGetLastError());
    }
    if (batch_graphs())
      JC_CUDA_CHECK(cudaMemcpyAsync(gspeed_.p, b + 16 + 32 * (size_t)n_, sizeof(float2) * batch_graphs(),
                                    cudaMemcpyHostToDevice, stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    tile_synced_ = false;
  }

 private:
  bool bh_;
  jc_descriptor desc_{};
  Fa2Settings s_;
  uint32_t n_ = 0, n_att_ = 0, n_hubs_ = 0, n_med_ = 0, hub_threshold_ = DEFAULT_HUB_THRESHOLD, att_blocks_ = 0;
  uint32_t tree_cap_ = 0, sort_tiles_ = 0, scan_tiles_ = 0;
  uint32_t walk_group_ = DEFAULT_WALK_GROUP;
  uint32_t launches_ = 0;
  uint32_t warn_accum_ = 0;
  uint32_t host_steps_ = 0;
  const float* dev_xyz_ = nullptr;  // set while reinit_device runs
  DevState* hst_ = nullptr;  // page-locked mirror of the device state
  bool initialized_ = false;
  // Tile schedule of a batch (jc_fa2_tile.cuh): eligible when every graph
  // fits (no hub list, at most TILE_MAX_NODES nodes); chosen by the
  // batch_schedule setting or the autotuner. gsteps (iterations per graph)
  // follows host_steps_ while tile_synced_.
  bool tile_ok_ = false;
  bool tile_mode_ = false;
  bool tile_synced_ = false;
  uint32_t tile_mult_ = 3;
  uint32_t tile_ctas_ = 0;
  float tile_probe_ms_ = 0.0f;
  DevBuf<uint32_t> t_work_, t_cap_, t_first_base_, t_gsteps_, t_next_, t_cells_, t_first_;
  DevBuf<uint64_t> t_node_base_, t_lcp_base_;
  DevBuf<TNode> t_nodes_;
  DevBuf<int8_t> t_lcp_;
  // false while init() runs: the neighbour ids have not been range-checked
  // yet (the staged upload checks them); the other entry points validate first
  bool ids_checked_ = true;
  cudaStream_t stream_ = nullptr;
  cudaStream_t side_ = nullptr;  // captures the conditional re-sort body
  cudaStream_t copy_ = nullptr;  // frame-stream copies (overlapping the steps)
  uint32_t* ok_host_ = nullptr;  // page-locked word: the device CSR check's verdict
  DevBuf<uint32_t> okb_;
  cudaGraphExec_t gexec_ = nullptr;        // the step, no event nodes (every replayed step)
  cudaGraphExec_t gexec_phase_ = nullptr;  // the same step with phase events (phase split only)
  bool capture_phases_ = false;            // set while gexec_phase_ is captured
  cudaEvent_t ev_[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};

  DevBuf<float4> pos_, old_, force_, frep_;
  DevBuf<float> degf_, bbox_part_, xyz_;
  DevBuf<float2> stats_;
  DevBuf<uint32_t> aoff_, anbr_, aorder_;
  DevBuf<DevState> state_;
  DevBuf<double2> partials_;
  // tree
  DevBuf<uint64_t> hi_orig_, lo_orig_, hi_, hi_alt_, lo_, lo_alt_;
  DevBuf<uint32_t> val_, val_alt_, sort_work_, sort_work2_, count_, first_, scan_sums_;
  DevBuf<int8_t> lcp_;  // prefix-length index: L, m1, m2 back to back
  LcpIndex lcpx_{};
  DevBuf<TNode> nodes_;
  DevBuf<uint32_t> parent_, nchild_, arrive_, top_list_;
  DevBuf<uint4> top_;
  // batch (forest) layout
  std::vector<uint32_t> graph_off_host_{0u, 0u};
  Forest forest_{1, 0, 21, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0, nullptr, nullptr, nullptr, nullptr,
                 nullptr};
  DevBuf<uint32_t> node_graph_, graph_off_, tree_root_, tree_end_;
  DevBuf<float4> roots_;
  DevBuf<float2> gspeed_;
  DevBuf<uint64_t> zflat_;
  DevBuf<uint32_t> slice_graph_, graph_slice_;
  DevBuf<float> slice_box_;
  DevBuf<double2> slice_sums_;

  void ensure_stream() {
    if (!stream_) {
      int dev_count = 0;
      if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
        fail(JC_ERR_CUDA, "no CUDA device is available");
      stream_ = StreamCache::instance().take();
      side_ = StreamCache::instance().take();
      copy_ = StreamCache::instance().take();
      for (auto& e : ev_) JC_CUDA_CHECK(cudaEventCreate(&e));
      static_assert(sizeof(DevState) <= SmallPinned::kSlot, "state mirror fits a small page-locked block");
      hst_ = static_cast<DevState*>(SmallPinned::instance().take(sizeof(DevState)));
      ok_host_ = static_cast<uint32_t*>(SmallPinned::instance().take(sizeof(uint32_t)));
    }
  }

  void setup_forest(uint32_t n) {
    const uint32_t G = (uint32_t)graph_off_host_.size() - 1;
    forest_ = Forest{};
    forest_.n_graphs = G;
    forest_.gbits = 0;
    forest_.lh = 21;
    if (G <= 1) return;
    uint32_t gb = 1;
    while ((1u << gb) < G) ++gb;
    forest_.gbits = gb;
    forest_.lh = (63 - (int)gb) / 3;
    if (32 - forest_.lh > 21) fail(JC_ERR_ARG, "too many graphs for the key layout");
    std::vector<uint32_t> ng(n);
    for (uint32_t g = 0; g < G; ++g)
      for (uint32_t i = graph_off_host_[g]; i < graph_off_host_[g + 1]; ++i) ng[i] = g;
    node_graph_.alloc(n); graph_off_.alloc(G + 1); roots_.alloc(G); tree_root_.alloc(G); tree_end_.alloc(G);
    gspeed_.alloc(G);
    zflat_.alloc(G);
    if (n) JC_CUDA_CHECK(cudaMemcpyAsync(node_graph_.p, ng.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, stream_));
    JC_CUDA_CHECK(cudaMemcpyAsync(graph_off_.p, graph_off_host_.data(), sizeof(uint32_t) * (G + 1),
                                  cudaMemcpyHostToDevice, stream_));
    std::vector<float2> sp(G, make_float2(1.0f, 1.0f));  // fa2_speed.rs:32-39, per graph
    JC_CUDA_CHECK(cudaMemcpyAsync(gspeed_.p, sp.data(), sizeof(float2) * G, cudaMemcpyHostToDevice, stream_));
    std::vector<uint32_t> slice_graph, graph_slice(G + 1, 0);
    for (uint32_t g = 0; g < G; ++g) {
      const uint32_t k = std::max<uint32_t>(1, cdiv(graph_off_host_[g + 1] - graph_off_host_[g], GRAPH_SLICE));
      graph_slice[g + 1] = graph_slice[g] + k;
      slice_graph.insert(slice_graph.end(), k, g);
    }
    const uint32_t S = graph_slice[G];
    slice_graph_.alloc(S); graph_slice_.alloc(G + 1); slice_box_.alloc(6 * (size_t)S); slice_sums_.alloc(S);
    JC_CUDA_CHECK(cudaMemcpyAsync(slice_graph_.p, slice_graph.data(), sizeof(uint32_t) * S, cudaMemcpyHostToDevice,
                                  stream_));
    JC_CUDA_CHECK(cudaMemcpyAsync(graph_slice_.p, graph_slice.data(), sizeof(uint32_t) * (G + 1),
                                  cudaMemcpyHostToDevice, stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    forest_.n_slices = S;
    forest_.slice_graph = slice_graph_.p;
    forest_.graph_slice = graph_slice_.p;
    forest_.slice_box = slice_box_.p;
    forest_.slice_sums = slice_sums_.p;
    forest_.node_graph = node_graph_.p;
    forest_.graph_off = graph_off_.p;
    forest_.roots = roots_.p;
    forest_.tree_root = tree_root_.p;
    forest_.tree_end = tree_end_.p;
    forest_.gspeed = gspeed_.p;
    forest_.zflat = zflat_.p;
  }

  void alloc_tree(uint32_t n) {
    // Exact tree: <= n leaves + internal nodes; 3n + 64 covers every layout
    // short of deep coincident clusters, which report JC_ERR_CAPACITY and
    // grow the buffers before the step is retried.
    tree_cap_ = std::max<uint32_t>(tree_cap_, 3 * n + 64);
    hi_orig_.alloc(n); lo_orig_.alloc(n); hi_.alloc(n); hi_alt_.alloc(n); lo_.alloc(n); lo_alt_.alloc(n);
    val_.alloc(n); val_alt_.alloc(n);
    sort_tiles_ = dev::rs_tiles(std::max<uint32_t>(n, 1));
    sort_work_.alloc(dev::sort_work_words(std::max<uint32_t>(n, 1), 8));
    sort_work2_.alloc(dev::sort_work_words(std::max<uint32_t>(n, 1), 8));
    count_.alloc((size_t)n + 1);
    first_.alloc((size_t)n + 2);
    scan_tiles_ = std::max<uint32_t>(1, cdiv(n, dev::SC_TILE));
    scan_sums_.alloc(scan_tiles_ + 1);
    nodes_.alloc(tree_cap_); parent_.alloc(tree_cap_); nchild_.alloc(tree_cap_);
    top_list_.alloc(TOP_MAX); top_.alloc(2 * TOP_MAX);
    arrive_.alloc(tree_cap_);
    const uint32_t nl = lcp_index_bytes(n), n2p = lcp_m2_bytes(nl);
    if (lcp_.n < (size_t)nl + nl / 32 + n2p || !lcp_.p) {
      lcp_.alloc((size_t)nl + nl / 32 + n2p);
      // entries past the bodies stay -1 ("run ends here") and the m2 padding
      // 127 ("never") for good; k_count rewrites the rest
      JC_CUDA_CHECK(cudaMemset(lcp_.p, 0xFF, (size_t)nl + nl / 32));
      JC_CUDA_CHECK(cudaMemset(lcp_.p + nl + nl / 32, 0x7F, n2p));
    }
    lcpx_ = LcpIndex{lcp_.p, lcp_.p + nl, lcp_.p + nl + nl / 32, nl / 32, nl / 1024};
  }

  void release() {
    drop_graph();
    if (stream_) {
      cudaStreamSynchronize(stream_);
      for (auto& e : ev_)
        if (e) cudaEventDestroy(e);
      StreamCache::instance().give(stream_);
      StreamCache::instance().give(side_);
      StreamCache::instance().give(copy_);
      stream_ = nullptr;
      side_ = nullptr;
      copy_ = nullptr;
    }
    SmallPinned::instance().give(hst_);
    hst_ = nullptr;
    SmallPinned::instance().give(ok_host_);
    ok_host_ = nullptr;
  }

  void drop_graph() {
    if (gexec_) {
      cudaGraphExecDestroy(gexec_);
      gexec_ = nullptr;
    }
    if (gexec_phase_) {
      cudaGraphExecDestroy(gexec_phase_);
      gexec_phase_ = nullptr;
    }
  }

  void require_init() const {
    if (!initialized_) fail(JC_ERR_STATE, std::string(desc_.id) + " step called before successful init");
  }

  KParams kparams() const {
    KParams P;
    P.n = n_;
    P.gravity = s_.gravity;
    P.scaling_ratio = s_.scaling_ratio;
    P.att_w = std::pow(std::fmax(1.0f, 1.0e-6f), s_.edge_weight_influence);
    P.ewi = s_.edge_weight_influence;
    P.jitter_tolerance = s_.jitter_tolerance;
    P.time_step = s_.time_step;
    float th = std::fmax(s_.theta, 0.0f);  // fa2_bh.rs:716
    P.theta2 = th * th;
    P.max_disp = s_.max_displacement;
    P.strong_gravity = s_.strong_gravity ? 1 : 0;
    P.lin_log = s_.lin_log_mode ? 1 : 0;
    P.tree_cap = tree_cap_;
    P.ref_cap = 2 * n_ + 8;
    P.n_hubs = n_hubs_;
    P.n_med = n_med_;
    return P;
  }

  // Issue one step's kernels on stream_ (eagerly or under capture).
  int enqueue_step() {
    const KParams P = kparams();
    const uint32_t n = n_;
    DevState* st = state_.p;
    int L = 0;
    record_phase(0);
    if (bh_) {
      const Forest F = forest_;
      if (F.n_graphs > 1) {
        k_bbox_slices<<<F.n_slices, 256, 0, stream_>>>(pos_.p, F);
        k_bbox_roots<<<cdiv(F.n_graphs, 8), 256, 0, stream_>>>(F, st);
        ++L;
      } else {
        k_bbox<<<BBOX_BLOCKS, BBOX_THREADS, 0, stream_>>>(pos_.p, n, bbox_part_.p, st);
      }
      k_keys<<<cdiv(n, 256), 256, 0, stream_>>>(pos_.p, n, st, hi_orig_.p, lo_orig_.p, hi_.p, val_.p, F);
      L += 2;
      {
        // a single graph: the top 32 bits (ten levels); a batch: the top 48
        // (the graph id takes up to 16 of them), then the runs are fixed up
        const int split = F.n_graphs > 1 ? 16 : 32;
        L += dev::radix_sort_pairs<uint64_t>(hi_.p, val_.p, hi_alt_.p, val_alt_.p, n, nullptr, split, 64,
                                             sort_work_.p, &st->error, nullptr, stream_);
        k_seg_fix<<<cdiv(n, 256), 256, 0, stream_>>>(hi_.p, val_.p, lo_orig_.p, n, st, split);
        ++L;
      }
      L += enqueue_tie_resort(st);
      k_gather_u64<<<cdiv(n, 256), 256, 0, stream_>>>(lo_orig_.p, val_.p, lo_.p, st, nullptr, n);
      k_count<<<lcpx_.n2, COUNT_THREADS, 0, stream_>>>(hi_.p, lo_.p, n, st, count_.p, F, lcpx_);
      L += 2;
      L += dev::exclusive_scan(count_.p, first_.p, n, scan_sums_.p, stream_);
      k_clear<<<std::min<uint32_t>(cdiv(tree_cap_, 256), 1184), 256, 0, stream_>>>(first_.p, n, P, st, nchild_.p,
                                                                                     arrive_.p);
      if (F.n_graphs > 1) {
        k_graph_trees<<<cdiv(n, 256), 256, 0, stream_>>>(hi_.p, first_.p, st, F);
        ++L;
      }
      const bool stage = stage_top();
      k_fill<<<cdiv(n, 256), 256, 0, stream_>>>(hi_.p, lcpx_, val_.p, first_.p, pos_.p, degf_.p, n, P, st,
                                                 nodes_.p, parent_.p, nchild_.p, F, stage ? top_list_.p : nullptr);
      k_com<<<cdiv(n, 256), 256, 0, stream_>>>(first_.p, nodes_.p, parent_.p, nchild_.p, arrive_.p, n, st);
      L += 3;
      if (stage) {
        k_top_build<<<1, 1024, 0, stream_>>>(nodes_.p, top_list_.p, st, top_.p);
        ++L;
      }
      record_phase(1);
      launch_walk(P, st);
      L += 1;
    } else {
      record_phase(1);
      k_brute<<<cdiv(n, 256), 256, 0, stream_>>>(pos_.p, degf_.p, n, P, frep_.p);
      L += 1;
    }
    record_phase(2);
    k_att<<<att_blocks_, ATT_THREADS, 0, stream_>>>(aorder_.p, aoff_.p, anbr_.p, pos_.p, frep_.p, old_.p, degf_.p, P,
                                                    st, force_.p, stats_.p, partials_.p, forest_.n_graphs);
    if (forest_.n_graphs > 1) {
      k_speed_slices<<<forest_.n_slices, 256, 0, stream_>>>(stats_.p, forest_, st);
      k_speed_graphs<<<cdiv(forest_.n_graphs, 256), 256, 0, stream_>>>(forest_, s_.jitter_tolerance, st);
      ++L;
      ++L;
    }
    record_phase(3);
    k_apply<<<cdiv(n, APPLY_THREADS), APPLY_THREADS, 0, stream_>>>(pos_.p, old_.p, force_.p, degf_.p, P, st, xyz_.p,
                                                                   forest_);
    record_phase(4);
    L += 2;
    JC_CUDA_CHECK(cudaGetLastError());
    return L;
  }

  // The staged-top walk: a single graph, walk group 1.
  bool stage_top() const { return s_.walk_stage_top && forest_.n_graphs == 1 && walk_group_ == 1; }

  template <bool FAST>
  void launch_walk_mode(const KParams& P, DevState* st) {
    const uint32_t n = n_;
    const dim3 grid(cdiv(n, WALK_THREADS));
    if (stage_top()) {
      k_walk_top<FAST><<<grid, WALK_THREADS, 0, stream_>>>(nodes_.p, top_.p, val_.p, pos_.p, degf_.p, n, P, st,
                                                          frep_.p);
      return;
    }
    switch (walk_group_) {
      case 1: k_walk_rope<FAST><<<grid, WALK_THREADS, 0, stream_>>>(nodes_.p, val_.p, pos_.p, degf_.p, n, P, st, frep_.p, forest_); break;
      case 2: k_walk<2, FAST><<<grid, WALK_THREADS, 0, stream_>>>(nodes_.p, val_.p, pos_.p, degf_.p, n, P, st, frep_.p, forest_); break;
      case 4: k_walk<4, FAST><<<grid, WALK_THREADS, 0, stream_>>>(nodes_.p, val_.p, pos_.p, degf_.p, n, P, st, frep_.p, forest_); break;
      case 8: k_walk<8, FAST><<<grid, WALK_THREADS, 0, stream_>>>(nodes_.p, val_.p, pos_.p, degf_.p, n, P, st, frep_.p, forest_); break;
      case 16: k_walk<16, FAST><<<grid, WALK_THREADS, 0, stream_>>>(nodes_.p, val_.p, pos_.p, degf_.p, n, P, st, frep_.p, forest_); break;
      default: k_walk<32, FAST><<<grid, WALK_THREADS, 0, stream_>>>(nodes_.p, val_.p, pos_.p, degf_.p, n, P, st, frep_.p, forest_); break;
    }
  }

  void launch_walk(const KParams& P, DevState* st) {
    if (s_.fast_repulsion) launch_walk_mode<true>(P, st);
    else launch_walk_mode<false>(P, st);
  }

  // Rare path (two valid keys tie in their first 21 levels): a conditional
  // IF node whose body re-sorts by the low 33 bits and then the high 64 bits,
  // giving the full 96-bit order. A one-thread kernel sets the condition
  // from the device tie flag, so the body costs nothing when it is not taken.
  int enqueue_tie_resort(DevState* st) {
    const uint32_t n = n_;
    if (!s_.use_graph) {
      // Eager launches: the same kernels, each returning at once unless the
      // device tie flag is set.
      const uint32_t* gate = &st->tie;
      const uint32_t* nvalid = &st->n_valid;
      k_gather_u64<<<cdiv(n, 256), 256, 0, stream_>>>(lo_orig_.p, val_.p, lo_.p, st, gate, n);
      int L = 1 + dev::radix_sort_pairs<uint64_t>(lo_.p, val_.p, lo_alt_.p, val_alt_.p, n, nvalid, 0, 33,
                                                  sort_work2_.p, &st->error, gate, stream_);
      k_gather_u64<<<cdiv(n, 256), 256, 0, stream_>>>(hi_orig_.p, val_.p, hi_.p, st, gate, n);
      L += 1 + dev::radix_sort_pairs<uint64_t>(hi_.p, val_.p, hi_alt_.p, val_alt_.p, n, nvalid, 0, 64,
                                               sort_work2_.p, &st->error, gate, stream_);
      return L;
    }
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    JC_CUDA_CHECK(cudaStreamGetCaptureInfo(stream_, &cs, nullptr, &cg, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) fail(JC_ERR_CUDA, "the step must be enqueued under stream capture");
    cudaGraphConditionalHandle h;
    JC_CUDA_CHECK(cudaGraphConditionalHandleCreate(&h, cg, 0, cudaGraphCondAssignDefault));
    k_set_tie_condition<<<1, 1, 0, stream_>>>(h, st);
    JC_CUDA_CHECK(cudaGetLastError());
    JC_CUDA_CHECK(cudaStreamGetCaptureInfo(stream_, &cs, nullptr, &cg, &deps, &nd));
    alignas(cudaGraphNodeParams) unsigned char cp_storage[sizeof(cudaGraphNodeParams)] = {};
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_storage);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    JC_CUDA_CHECK(cudaGraphAddNode(&cnode, cg, deps, nd, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    JC_CUDA_CHECK(cudaStreamUpdateCaptureDependencies(stream_, &cnode, 1, cudaStreamSetCaptureDependencies));
    JC_CUDA_CHECK(cudaStreamBeginCaptureToGraph(side_, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    const uint32_t* nvalid = &st->n_valid;
    k_gather_u64<<<cdiv(n, 256), 256, 0, side_>>>(lo_orig_.p, val_.p, lo_.p, st, nullptr, n);
    dev::radix_sort_pairs<uint64_t>(lo_.p, val_.p, lo_alt_.p, val_alt_.p, n, nvalid, 0, 33, sort_work2_.p,
                                    &st->error, nullptr, side_);
    k_gather_u64<<<cdiv(n, 256), 256, 0, side_>>>(hi_orig_.p, val_.p, hi_.p, st, nullptr, n);
    dev::radix_sort_pairs<uint64_t>(hi_.p, val_.p, hi_alt_.p, val_alt_.p, n, nvalid, 0, 64, sort_work2_.p,
                                    &st->error, nullptr, side_);
    JC_CUDA_CHECK(cudaGetLastError());
    cudaGraph_t captured;
    JC_CUDA_CHECK(cudaStreamEndCapture(side_, &captured));
    return 2;  // the condition kernel and the conditional node
  }

  // Phase boundary events: plain records when the kernels are launched one
  // by one; under capture, event nodes only in the phase graph (the five
  // event nodes cost 8 us of a replayed step on the 1M-node graph, measured).
  void record_phase(int k) {
    if (!s_.use_graph) JC_CUDA_CHECK(cudaEventRecord(ev_[k], stream_));
    else if (capture_phases_) JC_CUDA_CHECK(cudaEventRecordWithFlags(ev_[k], stream_, cudaEventRecordExternal));
  }

  // One step: a graph replay, or the kernels launched one by one.
  void launch_step() {
    if (s_.use_graph) {
      JC_CUDA_CHECK(cudaGraphLaunch(gexec_, stream_));
    } else {
      launches_ = (uint32_t)enqueue_step();
    }
  }

  void ensure_graph() {
    if (!s_.use_graph) return;
    if (gexec_) return;
    Trace tr("fa2.graph");
    launches_ = (uint32_t)capture_step(&gexec_, false);
    tr.mark("capture_instantiate");
  }

  // The step with its phase events, captured on first use.
  void ensure_phase_graph() {
    if (gexec_phase_) return;
    capture_step(&gexec_phase_, true);
  }

  int capture_step(cudaGraphExec_t* out, bool phases) {
    cudaGraph_t g;
    JC_CUDA_CHECK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    int L = 0;
    capture_phases_ = phases;
    try {
      L = enqueue_step();
    } catch (...) {
      capture_phases_ = false;
      cudaStreamEndCapture(stream_, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    capture_phases_ = false;
    JC_CUDA_CHECK(cudaStreamEndCapture(stream_, &g));
    cudaError_t e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) fail(JC_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return L;
  }

  // Per-graph tree, prefix-index and offset regions of the tile schedule,
  // graphs in work order (largest first), and the persistent grid size.
  void setup_tile() {
    const uint32_t G = (uint32_t)graph_off_host_.size() - 1;
    std::vector<uint32_t> work(G), cap(G), fbase(G);
    std::vector<uint64_t> nbase(G), lbase(G);
    for (uint32_t g = 0; g < G; ++g) work[g] = g;
    auto size = [&](uint32_t g) { return graph_off_host_[g + 1] - graph_off_host_[g]; };
    std::stable_sort(work.begin(), work.end(), [&](uint32_t a, uint32_t b) { return size(a) > size(b); });
    uint64_t nodes = 0, lbytes = 0;
    for (uint32_t g = 0; g < G; ++g) {
      const uint32_t ng = size(g);
      cap[g] = tile_mult_ * ng + 64;
      nbase[g] = nodes;
      nodes += cap[g];
      const uint32_t nl = lcp_index_bytes(ng);
      lbase[g] = lbytes;
      lbytes += (uint64_t)nl + nl / 32 + lcp_m2_bytes(nl);
      fbase[g] = graph_off_host_[g] + 2 * g;
    }
    t_work_.alloc(G); t_cap_.alloc(G); t_first_base_.alloc(G); t_gsteps_.alloc(G); t_next_.alloc(1);
    t_node_base_.alloc(G); t_lcp_base_.alloc(G);
    t_nodes_.alloc(nodes); t_cells_.alloc(nodes);
    t_first_.alloc((size_t)n_ + 2 * (size_t)G + 2);
    t_lcp_.alloc(lbytes);
    // prefix index: -1 (a run ends here) in L and m1, 127 (never) in m2's padding
    std::vector<int8_t> lcp_init(lbytes, (int8_t)-1);
    for (uint32_t g = 0; g < G; ++g) {
      const uint32_t nl = lcp_index_bytes(size(g));
      std::memset(&lcp_init[lbase[g] + nl + nl / 32], 0x7F, lcp_m2_bytes(nl));
    }
    HostStager& up = HostStager::instance();
    up.upload(t_work_.p, work.data(), 4 * (size_t)G, stream_);
    up.upload(t_cap_.p, cap.data(), 4 * (size_t)G, stream_);
    up.upload(t_first_base_.p, fbase.data(), 4 * (size_t)G, stream_);
    up.upload(t_node_base_.p, nbase.data(), 8 * (size_t)G, stream_);
    up.upload(t_lcp_base_.p, lbase.data(), 8 * (size_t)G, stream_);
    up.upload(t_lcp_.p, lcp_init.data(), lbytes, stream_);
    int per_sm = 0, sms = 0, dev = 0;
    JC_CUDA_CHECK(cudaGetDevice(&dev));
    JC_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    JC_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile_steps<false>, TILE_THREADS, 0));
    tile_ctas_ = std::max<uint32_t>(1, std::min<uint32_t>(G, (uint32_t)std::max(per_sm, 1) * (uint32_t)sms));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    tile_synced_ = false;
  }

  // Every graph's iteration count := the engine's (after forest steps, a
  // restored snapshot or a fresh bind).
  void sync_tile_steps() {
    if (tile_synced_) return;
    const uint32_t G = (uint32_t)graph_off_host_.size() - 1;
    std::vector<uint32_t> v(G, host_steps_);
    JC_CUDA_CHECK(cudaMemcpyAsync(t_gsteps_.p, v.data(), 4 * (size_t)G, cudaMemcpyHostToDevice, stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    tile_synced_ = true;
  }

  // One persistent launch: every graph from its own count up to `target`.
  void launch_tile(uint32_t target) {
    const uint32_t G = (uint32_t)graph_off_host_.size() - 1;
    TileBatch tb{G, graph_off_.p, t_work_.p, t_node_base_.p, t_cap_.p, t_lcp_base_.p, t_first_base_.p, t_gsteps_.p,
                 t_next_.p, gspeed_.p, t_nodes_.p, t_cells_.p, t_lcp_.p, t_first_.p};
    TileBufs tbufs{pos_.p, old_.p, force_.p, frep_.p, degf_.p, stats_.p, xyz_.p, aoff_.p, anbr_.p,
                   hi_orig_.p, lo_orig_.p, hi_.p, lo_.p, val_.p, val_alt_.p, count_.p};
    const KParams P = kparams();
    k_tile_begin<<<1, 1, 0, stream_>>>(state_.p, t_next_.p);
    if (s_.fast_repulsion)
      k_tile_steps<true><<<tile_ctas_, TILE_THREADS, 0, stream_>>>(tb, tbufs, P, state_.p, target,
                                                                   s_.jitter_tolerance);
    else
      k_tile_steps<false><<<tile_ctas_, TILE_THREADS, 0, stream_>>>(tb, tbufs, P, state_.p, target,
                                                                    s_.jitter_tolerance);
    k_tile_end<<<1, TILE_THREADS, 0, stream_>>>(t_gsteps_.p, G, n_, state_.p);
    JC_CUDA_CHECK(cudaGetLastError());
  }

  // Tile-schedule counterpart of run_steps: a graph whose tree outgrew its
  // region stops at that iteration; the regions grow and the same target is
  // launched again (graphs already there do nothing).
  void run_tile(uint32_t iters, float* out_xyz) {
    sync_tile_steps();
    const uint32_t target = host_steps_ + iters;
    for (int attempt = 0; attempt < 6; ++attempt) {
      launch_tile(target);
      if (out_xyz)
        JC_CUDA_CHECK(cudaMemcpyAsync(out_xyz, xyz_.p, sizeof(float) * 3 * n_, cudaMemcpyDeviceToHost, stream_));
      JC_CUDA_CHECK(cudaMemcpyAsync(hst_, state_.p, sizeof(DevState), cudaMemcpyDeviceToHost, stream_));
      JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
      host_steps_ = hst_->steps_done;
      if (hst_->error == 0) return;
      if (hst_->error != JC_ERR_CAPACITY) break;
      warn_accum_ |= hst_->warn;
      tile_mult_ *= 2;
      t_nodes_.free(); t_cells_.free();
      // keep every graph's count: the regions move, the per-graph state stays
      std::vector<uint32_t> gs((size_t)graph_off_host_.size() - 1);
      JC_CUDA_CHECK(cudaMemcpy(gs.data(), t_gsteps_.p, 4 * gs.size(), cudaMemcpyDeviceToHost));
      setup_tile();
      JC_CUDA_CHECK(cudaMemcpy(t_gsteps_.p, gs.data(), 4 * gs.size(), cudaMemcpyHostToDevice));
      tile_synced_ = true;
      uint32_t zero = 0;
      JC_CUDA_CHECK(cudaMemcpy(&state_.p->error, &zero, sizeof(uint32_t), cudaMemcpyHostToDevice));
    }
    check_state();
  }

  DevState read_state() {
    DevState st;
    JC_CUDA_CHECK(cudaMemcpyAsync(&st, state_.p, sizeof(st), cudaMemcpyDeviceToHost, stream_));
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    return st;
  }

  // Replays the step graph `iters` times, optionally reads the positions
  // back, and reads the device state once (one synchronisation). A tree
  // that outgrew its buffers makes the remaining replays no-ops; the buffers
  // are grown and the missing steps re-run.
  void run_steps(uint32_t iters, float* out_xyz) {
    if (tile_mode_) {
      run_tile(iters, out_xyz);
      return;
    }
    tile_synced_ = false;
    ensure_graph();
    const uint32_t target = host_steps_ + iters;
    for (int attempt = 0; attempt < 6; ++attempt) {
      for (uint32_t k = host_steps_; k < target; ++k) launch_step();
      if (out_xyz)
        JC_CUDA_CHECK(cudaMemcpyAsync(out_xyz, xyz_.p, sizeof(float) * 3 * n_, cudaMemcpyDeviceToHost, stream_));
      JC_CUDA_CHECK(cudaMemcpyAsync(hst_, state_.p, sizeof(DevState), cudaMemcpyDeviceToHost, stream_));
      JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
      host_steps_ = hst_->steps_done;
      if (hst_->error == 0) return;
      if (hst_->error != JC_ERR_CAPACITY) break;
      grow_tree();
      ensure_graph();
    }
    check_state();
  }

  // After a capacity error: size the tree buffers for the failed step's
  // node count (first_[n]) with headroom, clear the error, drop the graph.
  void grow_tree() {
    uint32_t need = 0;
    JC_CUDA_CHECK(cudaMemcpy(&need, first_.p + n_, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    tree_cap_ = std::max<uint32_t>(need + need / 4 + 64, tree_cap_ * 2);
    nodes_.free(); parent_.free(); nchild_.free(); arrive_.free();
    alloc_tree(n_);
    warn_accum_ |= hst_->warn;
    uint32_t zero = 0;
    JC_CUDA_CHECK(cudaMemcpy(&state_.p->error, &zero, sizeof(uint32_t), cudaMemcpyHostToDevice));
    drop_graph();
  }

  void check_state() {
    DevState st = read_state();
    if (st.error) {
      uint32_t code = st.error;
      uint32_t zero = 0;
      JC_CUDA_CHECK(cudaMemcpy(&state_.p->error, &zero, sizeof(zero), cudaMemcpyHostToDevice));
      fail((jc_status)code, code == JC_ERR_CAPACITY ? "octree exceeded its device capacity"
                                                    : "a bounded device loop found a malformed octree");
    }
  }
};

// ===================================================== no-allocation entry ==
// jc_fa2_bh_forces_noalloc: one Barnes-Hut force pass over caller-owned device
// buffers with every piece of scratch memory (keys, sort workspace, octree,
// partial sums, device state) carved from one file-scope device array. It is
// for callers that must not call cudaMalloc: code that runs under a fixed
// device-memory budget handed out by a host framework, or inside a region
// where an allocation would synchronise the device or be refused. The array
// is sized for NOALLOC_MAX_NODES bodies and is held by every GPU that loads
// the library until the process exits.
constexpr uint32_t NOALLOC_MAX_NODES = 32768;
constexpr uint32_t NOALLOC_TREE_CAP = 3 * NOALLOC_MAX_NODES + 64;
constexpr uint32_t NOALLOC_LCP = NOALLOC_MAX_NODES;  // prefix-length index bytes (multiple of 1024)

__host__ __device__ constexpr size_t na_round(size_t b) { return (b + 255) & ~(size_t)255; }

struct NoAllocLayout {
  size_t st, bbox, pos4, frep, force4, old4, degf, stats, order, hi_orig, lo_orig, hi, hi_alt, lo, lo_alt, val,
      val_alt, count, first, sums, work, work2, partials, nodes, parent, nchild, arrive, lcp, total;
};

constexpr NoAllocLayout noalloc_layout() {
  NoAllocLayout L{};
  const size_t N = NOALLOC_MAX_NODES, C = NOALLOC_TREE_CAP;
  size_t o = 0;
  L.st = o; o += na_round(sizeof(DevState));
  L.bbox = o; o += na_round(sizeof(float) * 6 * BBOX_BLOCKS);
  L.pos4 = o; o += na_round(16 * N);
  L.frep = o; o += na_round(16 * N);
  L.force4 = o; o += na_round(16 * N);
  L.old4 = o; o += na_round(16 * N);
  L.degf = o; o += na_round(4 * N);
  L.stats = o; o += na_round(8 * N);
  L.order = o; o += na_round(4 * N);
  L.hi_orig = o; o += na_round(8 * N);
  L.lo_orig = o; o += na_round(8 * N);
  L.hi = o; o += na_round(8 * N);
  L.hi_alt = o; o += na_round(8 * N);
  L.lo = o; o += na_round(8 * N);
  L.lo_alt = o; o += na_round(8 * N);
  L.val = o; o += na_round(4 * N);
  L.val_alt = o; o += na_round(4 * N);
  L.count = o; o += na_round(4 * (N + 1));
  L.first = o; o += na_round(4 * (N + 2));
  L.sums = o; o += na_round(4 * (N / dev::SC_TILE + 2));
  L.work = o; o += na_round(4 * dev::sort_work_words((uint32_t)N, 8));
  L.work2 = o; o += na_round(4 * dev::sort_work_words((uint32_t)N, 8));
  L.partials = o; o += na_round(sizeof(double2) * (N / ATT_THREADS + 1));
  L.nodes = o; o += na_round(sizeof(TNode) * C);
  L.parent = o; o += na_round(4 * C);
  L.nchild = o; o += na_round(4 * C);
  L.arrive = o; o += na_round(4 * C);
  L.lcp = o; o += na_round(NOALLOC_LCP + NOALLOC_LCP / 32 + 32);
  L.total = o;
  return L;
}

constexpr NoAllocLayout kNoAlloc = noalloc_layout();

// The scratch. Host code never uses this name as an address (on the host it
// is only a stand-in for the symbol); the device address comes from
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAlloc.total];

// Degrees, identity order and the CSR check of the no-allocation pass. The
// caller's CSR never went through the host validation of jc_engine_init, so
// every row is checked here before anything gathers through it: decreasing
// offsets, a non-empty row with no neighbour array, or a neighbour id >= n
// records JC_ERR_ARG in the error word and skips the row's reads; every later
// kernel of the pass (k_walk_rope, k_att, ...) then does no work.
__global__ void k_noalloc_prepare(const uint32_t* __restrict__ off, const uint32_t* __restrict__ nbr, uint32_t n,
                                  float* __restrict__ degf, uint32_t* __restrict__ order, DevState* st) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    st->speed = 1.0f;
    st->speed_eff = 1.0f;
  }
  if (i >= n) return;
  order[i] = i;
  const uint32_t e0 = off[i], e1 = off[i + 1];
  uint32_t d = 0;
  if (e1 < e0 || (e1 > e0 && nbr == nullptr)) {
    set_error(st, JC_ERR_ARG);
  } else {
    bool bad = false;
    for (uint32_t e = e0; e < e1; ++e) {
      const uint32_t u = nbr[e];
      bad |= u >= n;
      d += u != i ? 1u : 0u;
    }
    if (bad) set_error(st, JC_ERR_ARG);
  }
  degf[i] = (float)d + 1.0f;  // fa2_bh.rs:264-294: non-self CSR entries, mass = deg + 1
}

}  // namespace fa2

Engine* make_fa2_engine(bool barnes_hut) { return new fa2::Fa2Engine(barnes_hut); }

}  // namespace jc

namespace {

// Device address of the scratch array for each device, looked up once per
// device with that device current (first call of the entry point there).
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {};

}  // namespace

extern "C" jc_status jc_fa2_bh_forces_noalloc(uint32_t n_nodes, const uint32_t* d_offsets,
                                              const uint32_t* d_neighbors, const float* d_positions_xyz,
                                              const jc_fa2_params* params, float* d_forces_xyz,
                                              void* cuda_stream) {
  using namespace jc;
  using namespace jc::fa2;
  if (params == nullptr || (n_nodes > 0 && (d_offsets == nullptr || d_positions_xyz == nullptr ||
                                            d_forces_xyz == nullptr)))
    return JC_ERR_ARG;
  if (n_nodes > NOALLOC_MAX_NODES) return JC_ERR_CAPACITY;
  if (n_nodes == 0) return JC_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return JC_ERR_CUDA;
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_ptr[dev] == nullptr) {
      void* ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || ptr == nullptr) {
        (void)cudaGetLastError();
        return JC_ERR_CUDA;
      }
      g_noalloc_ptr[dev] = ptr;
    }
    base = (unsigned char*)g_noalloc_ptr[dev];
  }
  const NoAllocLayout& L = kNoAlloc;
  cudaStream_t s = (cudaStream_t)cuda_stream;
  DevState* st = (DevState*)(base + L.st);
  float4* pos4 = (float4*)(base + L.pos4);
  float4* frep = (float4*)(base + L.frep);
  float4* force4 = (float4*)(base + L.force4);
  float4* old4 = (float4*)(base + L.old4);
  float* degf = (float*)(base + L.degf);
  float2* stats = (float2*)(base + L.stats);
  uint32_t* order = (uint32_t*)(base + L.order);
  uint64_t* hi_orig = (uint64_t*)(base + L.hi_orig);
  uint64_t* lo_orig = (uint64_t*)(base + L.lo_orig);
  uint64_t* hi = (uint64_t*)(base + L.hi);
  uint64_t* hi_alt = (uint64_t*)(base + L.hi_alt);
  uint64_t* lo = (uint64_t*)(base + L.lo);
  uint64_t* lo_alt = (uint64_t*)(base + L.lo_alt);
  uint32_t* val = (uint32_t*)(base + L.val);
  uint32_t* val_alt = (uint32_t*)(base + L.val_alt);
  uint32_t* count = (uint32_t*)(base + L.count);
  uint32_t* first = (uint32_t*)(base + L.first);
  uint32_t* sums = (uint32_t*)(base + L.sums);
  uint32_t* work = (uint32_t*)(base + L.work);
  uint32_t* work2 = (uint32_t*)(base + L.work2);
  double2* partials = (double2*)(base + L.partials);
  TNode* nodes = (TNode*)(base + L.nodes);
  uint32_t* parent = (uint32_t*)(base + L.parent);
  uint32_t* nchild = (uint32_t*)(base + L.nchild);
  uint32_t* arrive = (uint32_t*)(base + L.arrive);
  int8_t* lcp = (int8_t*)(base + L.lcp);
  const LcpIndex X{lcp, lcp + NOALLOC_LCP, lcp + NOALLOC_LCP + NOALLOC_LCP / 32, NOALLOC_LCP / 32,
                   NOALLOC_LCP / 1024};

  KParams P;
  P.n = n_nodes;
  P.gravity = params->gravity;
  P.scaling_ratio = params->scaling_ratio;
  P.att_w = std::pow(std::fmax(1.0f, 1.0e-6f), params->edge_weight_influence);
  P.ewi = params->edge_weight_influence;
  P.jitter_tolerance = 1.0f;
  P.time_step = 1.0f;
  const float th = std::fmax(params->theta, 0.0f);
  P.theta2 = th * th;
  P.max_disp = 0.0f;
  P.strong_gravity = params->strong_gravity ? 1 : 0;
  P.lin_log = params->lin_log_mode ? 1 : 0;
  P.tree_cap = NOALLOC_TREE_CAP;
  P.ref_cap = 2 * n_nodes + 8;
  P.n_hubs = 0;
  P.n_med = 0;

  const uint32_t n = n_nodes;
  const Forest F1{1, 0, 21, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  // The array keeps the previous call's contents: zero what must start at 0.
  if (cudaMemsetAsync(st, 0, sizeof(DevState), s) != cudaSuccess ||
      cudaMemsetAsync(old4, 0, sizeof(float4) * n, s) != cudaSuccess ||
      cudaMemsetAsync(lcp, 0xFF, NOALLOC_LCP + NOALLOC_LCP / 32, s) != cudaSuccess ||  // -1: run ends
      cudaMemsetAsync(lcp + NOALLOC_LCP + NOALLOC_LCP / 32, 0x7F, 32, s) != cudaSuccess) {  // m2 padding: never
    (void)cudaGetLastError();
    return JC_ERR_CUDA;
  }
  k_noalloc_prepare<<<cdiv(n, 256), 256, 0, s>>>(d_offsets, d_neighbors, n, degf, order, st);
  k_unpack_xyz<<<cdiv(n, 256), 256, 0, s>>>(d_positions_xyz, n, pos4);
  k_bbox<<<BBOX_BLOCKS, BBOX_THREADS, 0, s>>>(pos4, n, (float*)(base + L.bbox), st);
  k_keys<<<cdiv(n, 256), 256, 0, s>>>(pos4, n, st, hi_orig, lo_orig, hi, val, F1);
  dev::radix_sort_pairs<uint64_t>(hi, val, hi_alt, val_alt, n, nullptr, 32, 64, work, &st->error, nullptr, s);
  k_seg_fix<<<cdiv(n, 256), 256, 0, s>>>(hi, val, lo_orig, n, st, 32);
  // ties in the first 21 levels: full 96-bit order, gated on the device flag
  const uint32_t* gate = &st->tie;
  k_gather_u64<<<cdiv(n, 256), 256, 0, s>>>(lo_orig, val, lo, st, gate, n);
  dev::radix_sort_pairs<uint64_t>(lo, val, lo_alt, val_alt, n, &st->n_valid, 0, 33, work2, &st->error, gate, s);
  k_gather_u64<<<cdiv(n, 256), 256, 0, s>>>(hi_orig, val, hi, st, gate, n);
  dev::radix_sort_pairs<uint64_t>(hi, val, hi_alt, val_alt, n, &st->n_valid, 0, 64, work2, &st->error, gate, s);
  k_gather_u64<<<cdiv(n, 256), 256, 0, s>>>(lo_orig, val, lo, st, nullptr, n);
  k_count<<<X.n2, COUNT_THREADS, 0, s>>>(hi, lo, n, st, count, F1, X);
  dev::exclusive_scan(count, first, n, sums, s);
  k_clear<<<std::min<uint32_t>(cdiv(NOALLOC_TREE_CAP, 256), 1184), 256, 0, s>>>(first, n, P, st, nchild, arrive);
  k_fill<<<cdiv(n, 256), 256, 0, s>>>(hi, X, val, first, pos4, degf, n, P, st, nodes, parent, nchild, F1);
  k_com<<<cdiv(n, 256), 256, 0, s>>>(first, nodes, parent, nchild, arrive, n, st);
  k_walk_rope<false><<<cdiv(n, WALK_THREADS), WALK_THREADS, 0, s>>>(nodes, val, pos4, degf, n, P, st, frep, F1);
  k_att<<<cdiv(n, ATT_THREADS), ATT_THREADS, 0, s>>>(order, d_offsets, d_neighbors, pos4, frep, old4, degf, P, st,
                                                    force4, stats, partials, 1u);
  k_pack_xyz<<<cdiv(n, 256), 256, 0, s>>>(force4, n, d_forces_xyz);
  if (cudaGetLastError() != cudaSuccess) return JC_ERR_CUDA;
  uint32_t err = 0;
  if (cudaMemcpyAsync(&err, &st->error, sizeof(err), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    (void)cudaGetLastError();
    return JC_ERR_CUDA;
  }
  return err ? (jc_status)err : JC_OK;
}

// Failure-detection self-test of the bounded waits: one radix pass over two
// tiles of keys in which only tile 1 runs (the tile counter starts at 1), so
// its look-back waits on tile 0's status word, which nothing ever writes. The
// wait must give up after OS_SPIN_LIMIT rounds, record JC_ERR_DEVICE_TIMEOUT
// in the error word and let the kernel finish (its writes stay in bounds: the
// output offsets come from the full histogram); the context stays usable.
extern "C" jc_status jc_selftest_sort_wait(uint32_t* device_status, float* wait_ms) {
  using namespace jc;
  using namespace jc::fa2;
  if (!device_status) return JC_ERR_ARG;
  const uint32_t n = 2 * dev::RS_TILE;
  uint64_t *keys = nullptr, *keys_out = nullptr;
  uint32_t *vals = nullptr, *vals_out = nullptr, *work = nullptr, *err = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  jc_status rc = JC_OK;
  try {
    JC_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    JC_CUDA_CHECK(cudaMalloc(&keys, 8 * (size_t)n));
    JC_CUDA_CHECK(cudaMalloc(&keys_out, 8 * (size_t)n));
    JC_CUDA_CHECK(cudaMalloc(&vals, 4 * (size_t)n));
    JC_CUDA_CHECK(cudaMalloc(&vals_out, 4 * (size_t)n));
    const size_t words = (size_t)dev::RS_RADIX + 1 + 2 * (size_t)dev::RS_RADIX;
    JC_CUDA_CHECK(cudaMalloc(&work, 4 * words));
    JC_CUDA_CHECK(cudaMalloc(&err, 4));
    std::vector<uint64_t> hk(n);
    std::vector<uint32_t> hv(n);
    SplitMix64 rng(0x5E1F7E57ull);
    for (uint32_t i = 0; i < n; ++i) {
      hk[i] = rng.next_u64();
      hv[i] = i;
    }
    JC_CUDA_CHECK(cudaMemcpyAsync(keys, hk.data(), 8 * (size_t)n, cudaMemcpyHostToDevice, s));
    JC_CUDA_CHECK(cudaMemcpyAsync(vals, hv.data(), 4 * (size_t)n, cudaMemcpyHostToDevice, s));
    JC_CUDA_CHECK(cudaMemsetAsync(work, 0, 4 * words, s));
    JC_CUDA_CHECK(cudaMemsetAsync(err, 0, 4, s));
    uint32_t* counts = work;
    uint32_t* tile_ctr = work + dev::RS_RADIX;
    uint32_t* status = tile_ctr + 1;
    dev::os_hist<uint64_t><<<2, dev::RS_THREADS, 0, s>>>(keys, n, nullptr, 0, 1, counts, nullptr);
    const uint32_t one = 1u;
    JC_CUDA_CHECK(cudaMemcpyAsync(tile_ctr, &one, 4, cudaMemcpyHostToDevice, s));
    JC_CUDA_CHECK(cudaEventCreate(&e0));
    JC_CUDA_CHECK(cudaEventCreate(&e1));
    JC_CUDA_CHECK(cudaEventRecord(e0, s));
    dev::os_pass<uint64_t, dev::RS_ROUNDS><<<1, dev::RS_THREADS, 0, s>>>(keys, vals, keys_out, vals_out, n, nullptr, 0,
                                                                        counts, status,
                                                        tile_ctr, nullptr, err);
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
  for (void* p : {(void*)keys, (void*)keys_out, (void*)vals, (void*)vals_out, (void*)work, (void*)err})
    if (p) cudaFree(p);
  if (s) cudaStreamDestroy(s);
  return rc;
}
