// Tile schedule of the batched fa2-bh engine: one CTA per graph.
//
// Included by jc_fa2.cu after the device helpers it reuses (TNode, DevState,
// KParams, the prefix-length index, att_term, finish_node, speed_update,
// rep_term). A batch of independent graphs (jc_engine_init_batch) can be
// laid out either as one forest per launch (every kernel of the step covers
// all graphs; the sort key carries the graph id) or, here, with every graph
// owned by one CTA of a persistent launch: the CTA takes the next graph from
// a counter (graphs largest first), runs all the step's phases for that graph
// with __syncthreads between them, and repeats them for as many iterations as
// the launch asks before taking the next graph. Nothing crosses CTAs, so a
// whole step_many(K) is one launch with no device-wide pass, and a graph's
// keys, sort, tree and prefix index stay in the SM's L1 and the L2.
//
// Every phase computes what the forest path computes for that graph, with the
// same roundings in the same order: the root cell (fa2_bh.rs:768-799), the
// octant-digit keys (fa2_bh.rs:841-861), the full 96-bit order (top 32 bits by
// a stable radix sort, runs of equal tops sorted by (high word, low word, body);
// a run longer than SEG_MAX takes the stable full re-sort), the pre-order
// octree from the prefix lengths, the centre of mass summed child by child
// (fa2_bh.rs:927-967), the rope walk (wgsl:114-156), attraction in list order
// (wgsl:158-197), the f64 speed sums in the forest path's slice order and
// AdaptiveSpeed::update (fa2_speed.rs:48-100), and the apply (wgsl:203-226).
// A graph therefore evolves bit for bit as it does on the forest path and in
// an engine of its own. Lists of hub_threshold entries or more (summed by a
// block reduction on the forest path) are not taken here: a batch with such a
// list keeps the forest schedule.
#pragma once

// (included inside namespace jc::fa2)

constexpr int TILE_THREADS = 256;  // == the forest's speed-slice block shape
constexpr int TILE_ROUNDS = 4;     // radix-pass entries per thread per tile
constexpr uint32_t TILE_MAX_NODES = 1u << 20;

struct TileBatch {
  uint32_t n_graphs;
  const uint32_t* graph_off;   // bodies of graph g: [graph_off[g], graph_off[g + 1])
  const uint32_t* work;        // graph ids, largest first
  const uint64_t* node_base;   // first tree node of graph g
  const uint32_t* node_cap;    // tree capacity of graph g
  const uint64_t* lcp_base;    // first byte of graph g's prefix-length index
  const uint32_t* first_base;  // first entry of graph g's node offsets (n_g + 2 entries)
  uint32_t* gsteps;            // iterations done, per graph
  uint32_t* next;              // work counter, zeroed before each launch
  float2* gspeed;              // per-graph (speed, speed efficiency)
  TNode* nodes;
  uint32_t* cells;             // a graph's cell indices grouped by depth
  int8_t* lcp;
  uint32_t* first;
};

struct TileBufs {
  float4* pos;
  float4* old_force;
  float4* force;
  float4* frep;
  const float* degf;
  float2* stats;
  float* xyz;
  const uint32_t* aoff;
  const uint32_t* anbr;
  uint64_t* hi_orig;  // keys by body
  uint64_t* lo_orig;
  uint64_t* hs;       // keys in sorted order
  uint64_t* ls;
  uint32_t* val;      // sorted permutation (local body indices)
  uint32_t* val_alt;
  uint32_t* count;
};

// Coherent 256-bit node load: the tile kernel reads nodes written earlier in
// the same launch, so the non-coherent read-only path cannot be used.
__device__ __forceinline__ void load_node_c(const TNode* p, float4& cm, int4& meta) {
  uint32_t r0, r1, r2, r3, r4, r5, r6, r7;
  asm volatile("ld.global.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5), "=r"(r6), "=r"(r7)
               : "l"(p));
  cm = make_float4(__uint_as_float(r0), __uint_as_float(r1), __uint_as_float(r2), __uint_as_float(r3));
  meta = make_int4((int)r4, (int)r5, (int)r6, (int)r7);
}

// The rope walk of one body over its graph's tree (local node indices,
// root 0, T nodes); the same visit sequence and terms as walk_one.
template <bool FAST>
__device__ __forceinline__ float4 tile_walk(const TNode* __restrict__ nodes, uint32_t body, const float4 p, float srd,
                                            uint32_t T, float theta2, bool& bad, uint32_t& n_inter,
                                            uint32_t& n_open) {
  float fx = 0.0f, fy = 0.0f, fz = 0.0f;
  uint32_t idx = 0;
  while (idx < T) {
    float4 c;
    int4 m;
    load_node_c(nodes + idx, c, m);
    const float dx = __fsub_rn(p.x, c.x), dy = __fsub_rn(p.y, c.y), dz = __fsub_rn(p.z, c.z);
    const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    const bool leaf = m.y >= 0;
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
  if (idx != END) bad = true;
  return make_float4(fx, fy, fz, 0.0f);
}

// Block-wide exclusive scan of one value per thread (TILE_THREADS threads).
__device__ __forceinline__ uint32_t tile_scan(uint32_t x, uint32_t* total, uint32_t* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t v = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, v, o);
    if (lane >= o) v += y;
  }
  if (lane == 31) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    uint32_t t = lane < TILE_THREADS / 32 ? sh[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < TILE_THREADS / 32) sh[lane] = t;
  }
  __syncthreads();
  const uint32_t ex = v - x + (w > 0 ? sh[w - 1] : 0u);
  *total = sh[TILE_THREADS / 32 - 1];
  __syncthreads();
  return ex;
}

constexpr int TILE_DEPTHS = 34;  // cell depths 0..32 (chains to the depth cap), one spare

struct TileShared {
  uint32_t hist[256];
  uint32_t dcnt[TILE_DEPTHS];
  uint32_t dstart[TILE_DEPTHS];
  uint32_t wcnt[TILE_THREADS / 32][256];
  uint32_t scan[32];
  float box[TILE_THREADS / 32][6];
  double red[2][TILE_THREADS / 32];
  float4 root;
  unsigned long long zf;
  uint32_t graph;
  uint32_t n_invalid;
  uint32_t tie;
  uint32_t T;
  uint32_t wnext;  // next body for the walk phase
  uint32_t stop;   // this graph stops (error)
  uint32_t max_depth;
  uint32_t dropped;
  uint32_t warn;
  float speed;
};

// One stable LSD pass of the permutation `vin` -> `vout` (n entries) by the
// byte at `shift` of key[vin[i]] (keys indexed by local body).
__device__ __forceinline__ void tile_radix_pass(const uint64_t* __restrict__ key, const uint32_t* __restrict__ vin,
                                                uint32_t* __restrict__ vout, uint32_t n, int shift, TileShared& S,
                                                uint32_t* err) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < 256; d += TILE_THREADS) S.hist[d] = 0;
  for (int k = threadIdx.x; k < (TILE_THREADS / 32) * 256; k += TILE_THREADS) (&S.wcnt[0][0])[k] = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += TILE_THREADS) {
    const uint32_t v = vin[i];
    if (JC_IN_BOUNDS(v, n, err)) atomicAdd(&S.hist[(uint32_t)(key[v] >> shift) & 0xFFu], 1u);
  }
  __syncthreads();
  {
    uint32_t tot;
    const uint32_t h = threadIdx.x < 256 ? S.hist[threadIdx.x] : 0u;
    const uint32_t ex = tile_scan(h, &tot, S.scan);
    if (threadIdx.x < 256) S.hist[threadIdx.x] = ex;  // running base of each digit
  }
  __syncthreads();
  // Tiles of TILE_ROUNDS * 256 entries: warp w ranks its 32 * TILE_ROUNDS
  // consecutive entries round by round (match_any + its own digit counts),
  // then thread d turns every warp's count of digit d into that warp's first
  // position, so the scatter keeps entry order (stable) with four barriers
  // per tile.
  static_assert(TILE_THREADS == 256, "one thread per digit");
  const uint32_t lt = (1u << lane) - 1u;
  constexpr uint32_t ITEMS = TILE_THREADS * TILE_ROUNDS;
  for (uint32_t t0 = 0; t0 < n; t0 += ITEMS) {
    uint32_t v[TILE_ROUNDS], d[TILE_ROUNDS], rank[TILE_ROUNDS];
    const uint32_t base = t0 + (uint32_t)w * 32u * TILE_ROUNDS;
#pragma unroll
    for (int r = 0; r < TILE_ROUNDS; ++r) {
      const uint32_t i = base + (uint32_t)r * 32u + (uint32_t)lane;
      const uint32_t v0 = i < n ? vin[i] : 0u;
      const bool ok = i < n && JC_IN_BOUNDS(v0, n, err);
      v[r] = ok ? v0 : 0u;
      d[r] = ok ? ((uint32_t)(key[v[r]] >> shift) & 0xFFu) : 256u;
    }
#pragma unroll
    for (int r = 0; r < TILE_ROUNDS; ++r) {
      const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d[r]);
      const bool ok = d[r] < 256u;
      const uint32_t before = ok ? S.wcnt[w][d[r]] : 0u;
      __syncwarp();
      if (ok && lane == __ffs(peers) - 1) S.wcnt[w][d[r]] = before + (uint32_t)__popc(peers);
      __syncwarp();
      rank[r] = before + (uint32_t)__popc(peers & lt);
    }
    __syncthreads();
    {
      const uint32_t dd = threadIdx.x;
      uint32_t run = S.hist[dd];
#pragma unroll
      for (int ww = 0; ww < TILE_THREADS / 32; ++ww) {
        const uint32_t c = S.wcnt[ww][dd];
        S.wcnt[ww][dd] = run;
        run += c;
      }
      S.hist[dd] = run;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < TILE_ROUNDS; ++r) {
      if (d[r] < 256u) {
        const uint32_t dst = S.wcnt[w][d[r]] + rank[r];
        if (JC_IN_BOUNDS(dst, n, err)) vout[dst] = v[r];
      }
    }
    __syncthreads();
#pragma unroll
    for (int ww = 0; ww < TILE_THREADS / 32; ++ww) S.wcnt[ww][threadIdx.x] = 0;
    __syncthreads();
  }
}

// The tile schedule: CTA c takes graphs from tb.next (graphs largest first)
// and runs each from tb.gsteps[g] up to `target` iterations.
// (at most 64 registers: four CTAs per SM; the 80-register build fitted
// three and was 12 % slower on the 4,096-graph batch)
template <bool FAST>
__global__ void __launch_bounds__(TILE_THREADS, 4)
k_tile_steps(TileBatch tb, TileBufs b, KParams P, DevState* st, uint32_t target, float jitter_tolerance) {
  __shared__ TileShared S;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) {
      const uint32_t k = atomicAdd(tb.next, 1u);
      S.graph = k < tb.n_graphs ? tb.work[k] : END;
      S.stop = 0;
    }
    __syncthreads();
    const uint32_t g = S.graph;
    __syncthreads();
    if (g == END) return;
    const uint32_t B = tb.graph_off[g];
    const uint32_t n = tb.graph_off[g + 1] - B;
    TNode* nodes = tb.nodes + tb.node_base[g];
    uint32_t* cells = tb.cells + tb.node_base[g];
    uint32_t* first = tb.first + tb.first_base[g];
    const uint32_t cap = tb.node_cap[g];
    const uint32_t nl = lcp_index_bytes(n);
    const LcpIndex X{tb.lcp + tb.lcp_base[g], tb.lcp + tb.lcp_base[g] + nl, tb.lcp + tb.lcp_base[g] + nl + nl / 32,
                     nl / 32, nl / 1024};
    uint64_t* hi_orig = b.hi_orig + B;
    uint64_t* lo_orig = b.lo_orig + B;
    uint64_t* hs = b.hs + B;
    uint64_t* ls = b.ls + B;
    uint32_t* val = b.val + B;
    uint32_t* val_alt = b.val_alt + B;
    uint32_t* count = b.count + B;
    uint32_t it = tb.gsteps[g];
    for (; it < target; ++it) {
      const bool last = it + 1 == target;
      // ---- bounding box -> root cell (k_bbox_roots' arithmetic) -----------
      float r[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
      for (uint32_t i = threadIdx.x; i < n; i += TILE_THREADS) {
        const float4 p = b.pos[B + i];
        const float v[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int k = 0; k < 3; ++k)
          if (isfinite(v[k])) {
            r[k] = fminf(r[k], v[k]);
            r[3 + k] = fmaxf(r[3 + k], v[k]);
          }
      }
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          r[k] = fminf(r[k], __shfl_xor_sync(0xFFFFFFFFu, r[k], o));
          r[3 + k] = fmaxf(r[3 + k], __shfl_xor_sync(0xFFFFFFFFu, r[3 + k], o));
        }
      if (lane == 0)
        for (int k = 0; k < 6; ++k) S.box[w][k] = r[k];
      if (threadIdx.x == 0) {
        S.n_invalid = 0;
        S.tie = 0;
        S.wnext = 0;
        S.stop = 0;
        S.max_depth = 0;
        S.dropped = 0;
        S.warn = 0;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        for (int k = 0; k < 3; ++k) {
          r[k] = INFINITY;
          r[3 + k] = -INFINITY;
          for (int ww = 0; ww < TILE_THREADS / 32; ++ww) {
            r[k] = fminf(r[k], S.box[ww][k]);
            r[3 + k] = fmaxf(r[3 + k], S.box[ww][3 + k]);
          }
        }
        if (!isfinite(r[0]))
          for (int k = 0; k < 3; ++k) { r[k] = -1.0f; r[3 + k] = 1.0f; }
        float half =
            __fmul_rn(fmaxf(fmaxf(__fsub_rn(r[3], r[0]), __fsub_rn(r[4], r[1])), __fsub_rn(r[5], r[2])), 0.5f);
        if (!isfinite(half) || half <= 0.0f) half = 1.0f;
        const float4 root = make_float4(__fmul_rn(0.5f, __fadd_rn(r[0], r[3])), __fmul_rn(0.5f, __fadd_rn(r[1], r[4])),
                                        __fmul_rn(0.5f, __fadd_rn(r[2], r[5])), __fmul_rn(half, 1.05f));
        uint64_t zf = 0;
        if (r[2] == r[5] && isfinite(r[2])) {
          float cz = root.z, h = root.w;
          uint32_t zb = 0;
          for (int l = 0; l < 32; ++l) {
            const bool up = r[2] >= cz;
            zb |= (up ? 1u : 0u) << l;
            const float hh = __fmul_rn(h, 0.5f);
            cz = __fadd_rn(cz, up ? hh : -hh);
            h = hh;
          }
          zf = (1ull << 32) | zb;
        }
        S.root = root;
        S.zf = zf;
      }
      __syncthreads();
      // ---- keys (k_keys, one graph: 21 levels in the high word) ----------
      {
        const float4 root = S.root;
        const uint64_t zf = S.zf;
        uint32_t inval = 0;
        for (uint32_t i = threadIdx.x; i < n; i += TILE_THREADS) {
          const float4 p = b.pos[B + i];
          uint64_t hi = 0, lo = 0;
          if (isfinite(p.x) && isfinite(p.y) && isfinite(p.z)) {
            float cx = root.x, cy = root.y, cz = root.z, h = root.w;
            // levels 0..20 into the high word, 21..31 into the low word
            if (zf >> 32) {
              auto level = [&](uint64_t& w, int l) {
                const uint32_t o = (p.x >= cx ? 1u : 0u) | (p.y >= cy ? 2u : 0u) | ((uint32_t)(zf >> l) & 1u) << 2;
                w = (w << 3) | o;
                const float hh = __fmul_rn(h, 0.5f);
                cx = __fadd_rn(cx, (o & 1u) ? hh : -hh);
                cy = __fadd_rn(cy, (o & 2u) ? hh : -hh);
                h = hh;
              };
#pragma unroll 3
              for (int l = 0; l < 21; ++l) level(hi, l);
#pragma unroll 3
              for (int l = 21; l < 32; ++l) level(lo, l);
            } else {
              auto level = [&](uint64_t& w) {
                const uint32_t o = (p.x >= cx ? 1u : 0u) | (p.y >= cy ? 2u : 0u) | (p.z >= cz ? 4u : 0u);
                w = (w << 3) | o;
                const float hh = __fmul_rn(h, 0.5f);
                cx = __fadd_rn(cx, (o & 1u) ? hh : -hh);
                cy = __fadd_rn(cy, (o & 2u) ? hh : -hh);
                cz = __fadd_rn(cz, (o & 4u) ? hh : -hh);
                h = hh;
              };
#pragma unroll 3
              for (int l = 0; l < 21; ++l) level(hi);
#pragma unroll 3
              for (int l = 21; l < 32; ++l) level(lo);
            }
          } else {
            hi = 1ull << 63;
            ++inval;
          }
          hi_orig[i] = hi;
          lo_orig[i] = lo;
          val[i] = i;
        }
        if (inval) atomicAdd(&S.n_invalid, inval);
      }
      __syncthreads();
      const uint32_t N = n - S.n_invalid;
      // ---- sort: top 32 bits, then runs of equal tops (k_seg_fix) ---------
      for (int pass = 0; pass < 4; ++pass) {
        uint32_t* vin = (pass & 1) ? val_alt : val;
        uint32_t* vout = (pass & 1) ? val : val_alt;
        tile_radix_pass(hi_orig, vin, vout, n, 32 + 8 * pass, S, &st->error);
      }
      // sorted keys, then the runs of equal top halves
      for (uint32_t a = threadIdx.x; a < n; a += TILE_THREADS) {
        const uint32_t v = val[a];
        hs[a] = JC_IN_BOUNDS(v, n, &st->error) ? hi_orig[v] : 0ull;
      }
      __syncthreads();
      for (uint32_t a = threadIdx.x; a < N; a += TILE_THREADS) {
        const uint64_t top = hs[a] >> 32;
        if (a > 0 && (hs[a - 1] >> 32) == top) continue;
        uint32_t len = 1;
        while (a + len < N && len <= SEG_MAX && (hs[a + len] >> 32) == top) ++len;
        if (len == 1) continue;
        if (len > SEG_MAX) {
          S.tie = 1u;
          continue;
        }
        uint64_t k[SEG_MAX], l[SEG_MAX];
        uint32_t v[SEG_MAX];
        for (uint32_t q = 0; q < len; ++q) {
          k[q] = hs[a + q];
          v[q] = val[a + q];
          l[q] = JC_IN_BOUNDS(v[q], n, &st->error) ? lo_orig[v[q]] : 0ull;
        }
        for (uint32_t q = 1; q < len; ++q) {
          const uint64_t kk = k[q], ll = l[q];
          const uint32_t vv = v[q];
          uint32_t j = q;
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
        for (uint32_t q = 0; q < len; ++q) {
          hs[a + q] = k[q];
          val[a + q] = v[q];
        }
      }
      __syncthreads();
      if (S.tie) {
        // a long run: the full order, stably by the low word and then the
        // high word from body order (the forest's tie re-sort)
        for (uint32_t i = threadIdx.x; i < n; i += TILE_THREADS) val[i] = i;
        __syncthreads();
        for (int pass = 0; pass < 6; ++pass) {
          uint32_t* vin = (pass & 1) ? val_alt : val;
          uint32_t* vout = (pass & 1) ? val : val_alt;
          tile_radix_pass(lo_orig, vin, vout, n, 8 * pass, S, &st->error);
        }
        for (int pass = 0; pass < 8; ++pass) {
          uint32_t* vin = (pass & 1) ? val_alt : val;
          uint32_t* vout = (pass & 1) ? val : val_alt;
          tile_radix_pass(hi_orig, vin, vout, n, 8 * pass, S, &st->error);
        }
        for (uint32_t a = threadIdx.x; a < n; a += TILE_THREADS) {
        const uint32_t v = val[a];
        hs[a] = JC_IN_BOUNDS(v, n, &st->error) ? hi_orig[v] : 0ull;
      }
        __syncthreads();
      }
      for (uint32_t a = threadIdx.x; a < n; a += TILE_THREADS) {
        const uint32_t v = val[a];
        ls[a] = JC_IN_BOUNDS(v, n, &st->error) ? lo_orig[v] : 0ull;
      }
      __syncthreads();
      // ---- node counts and the prefix-length index (k_count) --------------
      {
        uint32_t drop = 0;
        for (uint32_t a0 = 0; a0 < nl; a0 += TILE_THREADS) {
          const uint32_t a = a0 + threadIdx.x;
          uint32_t c = 0;
          bool dup = false;
          int nxt = -1;
          if (a < N) {
            const uint64_t ha = hs[a], la = ls[a];
            int prev = -1;
            if (a > 0) {
              prev = lcp_levels(hs[a - 1], ls[a - 1], ha, la);
              dup = prev == 32;
            }
            if (a + 1 < N) nxt = lcp_levels(ha, la, hs[a + 1], ls[a + 1]);
            if (!dup) c = 1u + (uint32_t)max(0, max(0, nxt) - prev);
          }
          if (a < n) count[a] = c;
          X.L[a] = (int8_t)nxt;
          int mn = nxt;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
          if (lane == 0) X.m1[a >> 5] = (int8_t)mn;
          drop += dup ? 1u : 0u;
        }
        if (drop) atomicAdd(&S.dropped, drop);
      }
      __syncthreads();
      for (uint32_t bb = threadIdx.x; bb < X.n2; bb += TILE_THREADS) {
        int mn = 127;
        for (int k = 0; k < 32; ++k) mn = min(mn, (int)X.m1[32 * bb + k]);
        X.m2[bb] = (int8_t)mn;
      }
      // ---- exclusive scan of the counts -> first node of each body --------
      {
        const uint32_t per = (n + TILE_THREADS - 1) / TILE_THREADS;
        const uint32_t a0 = min(n, threadIdx.x * per), a1 = min(n, a0 + per);
        uint32_t sum = 0;
        for (uint32_t a = a0; a < a1; ++a) sum += count[a];
        uint32_t tot;
        uint32_t run = tile_scan(sum, &tot, S.scan);
        for (uint32_t a = a0; a < a1; ++a) {
          const uint32_t c = count[a];
          first[a] = run;
          run += c;
        }
        if (threadIdx.x == 0) {
          first[n] = tot;
          first[n + 1] = tot;
          S.T = tot;
          if (tot > cap) S.stop = JC_ERR_CAPACITY;
        }
      }
      __syncthreads();
      const uint32_t T = S.T;
      if (S.stop) break;
      // ---- pre-order nodes (k_fill, one graph; no parent links: the centre
      // of mass below works level by level) -----------------------------------
      {
        uint32_t leaf_depth = 0;
        bool bad = false;
        for (uint32_t a = threadIdx.x; a < N; a += TILE_THREADS) {
          const uint32_t base = first[a], stop = first[a + 1];
          if (stop <= base) continue;  // a dropped duplicate
          const int prev = a > 0 ? (int)X.L[a - 1] : -1;
          const int top = max(0, (int)X.L[a]);
          const int n_int = max(0, top - prev);
          float half = S.root.w;
          for (int k = 0; k <= prev; ++k) half = __fmul_rn(half, 0.5f);
          for (int j = 0; j < n_int; ++j) {
            const int d = prev + 1 + j;
            const uint32_t idx = base + (uint32_t)j;
            const uint32_t e = d == 0 ? N - 1 : lcp_next_below(X, a, d);
            if (e >= N || idx >= cap) {
              bad = true;
              break;
            }
            uint32_t sk = first[e + 1];
            if (sk >= T) sk = END;
            const float s = __fmul_rn(half, 2.0f);
            nodes[idx].meta = make_int4((int)sk, -1, __float_as_int(__fmul_rn(s, s)), d);
            nodes[idx].cm = make_float4(0.f, 0.f, 0.f, 0.f);
            half = __fmul_rn(half, 0.5f);
          }
          if (bad) break;
          const uint32_t leaf = base + (uint32_t)n_int;
          if (leaf >= cap) {
            bad = true;
            break;
          }
          const uint32_t ld = (uint32_t)(max(prev, top) + 1);
          leaf_depth = max(leaf_depth, ld);
          const uint32_t body = val[a];
          if (!JC_IN_BOUNDS(body, n, &st->error)) {
            bad = true;
            break;
          }
          const float4 p = b.pos[B + body];
          uint32_t sk = first[a + 1];
          if (sk >= T) sk = END;
          nodes[leaf].meta = make_int4((int)sk, (int)(B + body), 0, (int)ld);
          nodes[leaf].cm = make_float4(p.x, p.y, p.z, fmaxf(b.degf[B + body], 1e-3f));
        }
        if (bad) atomicCAS(&S.stop, 0u, (uint32_t)JC_ERR_DEVICE_TIMEOUT);
        if (leaf_depth) atomicMax(&S.max_depth, leaf_depth);
      }
      __syncthreads();
      if (S.stop) break;
      // ---- centre of mass, deepest cells first ----------------------------
      // The CTA owns the whole tree, so the cells are summed level by level
      // (a barrier between levels) instead of by climbing threads with
      // arrival counters: each cell adds its children in pre-order (octant
      // order), exactly the sums of aggregate_com_postorder (fa2_bh.rs:927-967).
      {
        uint32_t* list = cells;
        for (int d = threadIdx.x; d < TILE_DEPTHS; d += TILE_THREADS) S.dcnt[d] = 0;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < T; i += TILE_THREADS) {
          const int4 m = nodes[i].meta;
          if (m.y < 0) atomicAdd(&S.dcnt[min(max(m.w, 0), TILE_DEPTHS - 1)], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          uint32_t run = 0;
          for (int d = 0; d < TILE_DEPTHS; ++d) {
            S.dstart[d] = run;
            run += S.dcnt[d];
            S.dcnt[d] = S.dstart[d];  // scatter cursor; the level's end afterwards
          }
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < T; i += TILE_THREADS) {
          const int4 m = nodes[i].meta;
          if (m.y < 0) {
            const uint32_t q = atomicAdd(&S.dcnt[min(max(m.w, 0), TILE_DEPTHS - 1)], 1u);
            if (JC_IN_BOUNDS(q, T, &st->error)) list[q] = i;
          }
        }
        __syncthreads();
        bool bad = false;
        for (int d = TILE_DEPTHS - 1; d >= 0; --d) {
          const uint32_t b0 = S.dstart[d], b1 = S.dcnt[d];
          if (b0 == b1) continue;  // (uniform: every thread reads the same counts)
          for (uint32_t k = b0 + threadIdx.x; k < b1; k += TILE_THREADS) {
            const uint32_t v = list[k];
            if (!JC_IN_BOUNDS(v, T, &st->error)) continue;
            float tot = 0.0f, sx = 0.0f, sy = 0.0f, sz = 0.0f;
            const uint32_t end = (uint32_t)nodes[v].meta.x;
            uint32_t c = v + 1;
            uint32_t kids = 0;
            while (c != end) {
              if (c >= T || ++kids > 8u) { bad = true; break; }
              const float4 q = nodes[c].cm;
              tot = __fadd_rn(tot, q.w);
              sx = __fadd_rn(sx, __fmul_rn(q.x, q.w));
              sy = __fadd_rn(sy, __fmul_rn(q.y, q.w));
              sz = __fadd_rn(sz, __fmul_rn(q.z, q.w));
              const uint32_t nx = (uint32_t)nodes[c].meta.x;
              if (nx != END && nx <= c) { bad = true; break; }
              c = nx;
            }
            if (tot > 0.0f) {
              sx = __fdiv_rn(sx, tot);
              sy = __fdiv_rn(sy, tot);
              sz = __fdiv_rn(sz, tot);
            }
            nodes[v].cm = make_float4(sx, sy, sz, tot);
          }
          __syncthreads();
        }
        if (bad) atomicCAS(&S.stop, 0u, (uint32_t)JC_ERR_DEVICE_TIMEOUT);
      }
      __syncthreads();
      if (S.stop) break;
      // ---- theta walk (bodies in key order) -------------------------------
      // Each warp takes the next 32 consecutive bodies from a counter until
      // none are left, so warps whose bodies walk long paths do not hold the
      // CTA at the barrier while the others idle.
      {
        uint32_t n_inter = 0, n_open = 0;
        bool bad = false;
        for (;;) {
          uint32_t a0 = 0;
          if (lane == 0) a0 = atomicAdd(&S.wnext, 32u);
          a0 = __shfl_sync(0xFFFFFFFFu, a0, 0);
          if (a0 >= n) break;
          const uint32_t a = a0 + (uint32_t)lane;
          if (a >= n) continue;
          const uint32_t lb = val[a];
          if (!JC_IN_BOUNDS(lb, n, &st->error)) continue;
          const uint32_t body = B + lb;
          float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
          if (T > 0u)
            f = tile_walk<FAST>(nodes, body, b.pos[body], __fmul_rn(P.scaling_ratio, b.degf[body]), T, P.theta2, bad,
                                n_inter, n_open);
          b.frep[body] = f;
        }
        if (bad) atomicCAS(&S.stop, 0u, (uint32_t)JC_ERR_DEVICE_TIMEOUT);
        if (last) walk_counts_flush(n_inter, n_open, st);
      }
      __syncthreads();
      if (S.stop) break;
      // ---- attraction, gravity, swing / traction (k_att, list order) ------
      for (uint32_t i = B + threadIdx.x; i < B + n; i += TILE_THREADS) {
        const float4 pi = b.pos[i];
        const float4 fr = b.frep[i];
        float fx = fr.x, fy = fr.y, fz = fr.z;
        const uint32_t e0 = b.aoff[i], e1 = b.aoff[i + 1];
        for (uint32_t k = e0; k < e1; ++k) {
          const uint32_t u = b.anbr[k];
          if (JC_IN_BOUNDS(u, P.n, &st->error)) att_term(b.pos[u], pi, P, fx, fy, fz);
        }
        finish_node(i, fx, fy, fz, pi, b.degf[i], P, b.old_force, b.force, b.stats);
      }
      __syncthreads();
      // ---- f64 speed sums in the forest's slice order, then the update ----
      {
        double a_sum = 0.0, c_sum = 0.0;
        for (uint32_t s0 = 0; s0 < n; s0 += GRAPH_SLICE) {
          const uint32_t e = min(n, s0 + GRAPH_SLICE);
          double sw = 0.0, tr = 0.0;
          for (uint32_t i = s0 + threadIdx.x; i < e; i += TILE_THREADS) {
            const float2 v = b.stats[B + i];
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
          if (lane == 0) {
            S.red[0][w] = sw;
            S.red[1][w] = tr;
          }
          __syncthreads();
          if (threadIdx.x == 0) {
            double x = 0.0, y = 0.0;
            for (int ww = 0; ww < TILE_THREADS / 32; ++ww) {
              x += S.red[0][ww];
              y += S.red[1][ww];
            }
            a_sum += x;
            c_sum += y;
          }
          __syncthreads();
        }
        if (threadIdx.x == 0) {
          DevState tmp;
          tmp.speed = tb.gspeed[g].x;
          tmp.speed_eff = tb.gspeed[g].y;
          speed_update(&tmp, n, jitter_tolerance, a_sum, c_sum);
          tb.gspeed[g] = make_float2(tmp.speed, tmp.speed_eff);
          S.speed = tmp.speed;
        }
      }
      __syncthreads();
      // ---- apply (k_apply) ------------------------------------------------
      {
        const float speed = S.speed;
        for (uint32_t i = B + threadIdx.x; i < B + n; i += TILE_THREADS) {
          const float4 f = b.force[i];
          const float4 o = b.old_force[i];
          const float deg = b.degf[i];
          const float swinging = __fmul_rn(deg, len3(__fsub_rn(o.x, f.x), __fsub_rn(o.y, f.y), __fsub_rn(o.z, f.z)));
          float factor = __fdiv_rn(speed, __fadd_rn(1.0f, __fsqrt_rn(__fmul_rn(speed, swinging))));
          const float df = len3(f.x, f.y, f.z);
          if (P.max_disp > 0.0f && df > 1.0e-9f) factor = fminf(factor, __fdiv_rn(P.max_disp, df));
          const float k = __fmul_rn(factor, P.time_step);
          float4 p = b.pos[i];
          p.x = __fadd_rn(p.x, __fmul_rn(f.x, k));
          p.y = __fadd_rn(p.y, __fmul_rn(f.y, k));
          p.z = __fadd_rn(p.z, __fmul_rn(f.z, k));
          p.w = 0.0f;
          b.pos[i] = p;
          b.old_force[i] = make_float4(f.x, f.y, f.z, 0.0f);
          if (last) {
            b.xyz[3 * (size_t)i] = p.x;
            b.xyz[3 * (size_t)i + 1] = p.y;
            b.xyz[3 * (size_t)i + 2] = p.z;
          }
        }
      }
      if (last && threadIdx.x == 0) {
        atomicAdd(&st->n_invalid, S.n_invalid);
        atomicAdd(&st->n_tree, T);
        atomicAdd(&st->dropped, S.dropped);
        atomicMax(&st->max_depth, S.max_depth);
        uint32_t warn = 0;
        if (S.n_invalid) warn |= JC_WARN_NONFINITE;
        if (S.dropped) warn |= JC_WARN_DEPTH_CAP;
        if (T > 2 * n + 8) warn |= JC_WARN_REF_CAPACITY;
        if (warn) atomicOr(&st->warn, warn);
        if (S.tie) st->tie = 1u;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      tb.gsteps[g] = it;
      if (S.stop) set_error(st, S.stop);
    }
    __syncthreads();
  }
}

// Before a tile launch: the per-step read-outs start from zero and the work
// counter is reset (one thread).
__global__ void k_tile_begin(DevState* st, uint32_t* next) {
  st->n_invalid = 0;
  st->n_tree = 0;
  st->dropped = 0;
  st->max_depth = 0;
  st->tie = 0;
  st->n_inter = 0;
  st->n_open = 0;
  *next = 0;
}

// After a tile launch: the engine's step counter is the smallest per-graph
// count (a graph stopped by a capacity error is re-run from there).
__global__ void k_tile_end(const uint32_t* gsteps, uint32_t n_graphs, uint32_t n_bodies, DevState* st) {
  __shared__ uint32_t red[TILE_THREADS / 32];
  uint32_t m = 0xFFFFFFFFu;
  for (uint32_t g = threadIdx.x; g < n_graphs; g += blockDim.x) m = min(m, gsteps[g]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    m = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = min(m, red[w]);
    st->steps_done = m;
    st->n_valid = n_bodies - st->n_invalid;
  }
}

