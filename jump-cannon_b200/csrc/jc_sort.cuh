// Device-wide primitives for the octree build: a stable LSD radix sort of
// (key, u32 value) pairs with 8-bit digits, and an exclusive scan of u32.
//
// Both read their item count from device memory (so they can sit inside a
// captured CUDA graph while the count changes from step to step) and accept
// an optional device "gate" word: when the gate is 0 every kernel returns at
// once, which is how the rare tie-breaking re-sort is made conditional
// without a host round trip.
//
// Radix sort: one histogram kernel for all passes, then one kernel per
// 8-bit pass (os_pass): per-tile stable ranking with warp ballots and
// per-warp digit counters (item order in a tile = warp, round, lane = input
// order) and decoupled look-back across tiles for the output offsets.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "jc_check.cuh"

namespace jc {
namespace dev {

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ROUNDS = 16;                        // items per lane
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;      // 4096 items per block
constexpr int RS_RADIX = 256;
// Below RS_SMALL_N items a tile holds 8 items per lane (2048 per block): a
// tile's ranking is a serial chain of rounds, so where the tiles would not
// fill the GPU shorter tiles finish sooner (B200: a 10,000-body step 0.274 ->
// 0.261 ms); above it 16 per lane keep the look-back chains short (1M bodies:
// tree build 0.446 ms against 0.471 with 8).
constexpr int RS_ROUNDS_SMALL = 8;
constexpr uint32_t RS_SMALL_N = 296u * 2048u;
__host__ __device__ constexpr int rs_rounds(uint32_t n_max) {
  return n_max <= RS_SMALL_N ? RS_ROUNDS_SMALL : RS_ROUNDS;
}
__host__ __device__ constexpr uint32_t rs_tiles(uint32_t n_max) {
  return (n_max + (uint32_t)(RS_THREADS * rs_rounds(n_max)) - 1) / (uint32_t)(RS_THREADS * rs_rounds(n_max));
}

__device__ __forceinline__ uint32_t rs_count(uint32_t n_max, const uint32_t* d_count) {
  if (d_count == nullptr) return n_max;
  uint32_t c = *d_count;
  return c < n_max ? c : n_max;
}

// Exclusive scan across a 256-thread block (one value per thread).
__device__ __forceinline__ uint32_t block_excl_scan_256(uint32_t x, uint32_t* total, uint32_t* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t v = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, v, o);
    if (lane >= o) v += y;
  }
  if (lane == 31) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    uint32_t t = lane < 8 ? sh[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < 8) sh[lane] = t;
  }
  __syncthreads();
  uint32_t ex = v - x + (w > 0 ? sh[w - 1] : 0u);
  *total = sh[7];
  return ex;
}

// ------------------------------------------------------------ onesweep --
// One global histogram of every pass's digits (counts do not depend on the
// order of the keys), then one kernel per pass that ranks a tile locally and
// finds its output offsets by decoupled look-back over the status words of
// the tiles before it (Merrill & Garland's single-pass scan, applied per
// digit). Tiles take their ids from an atomic counter in launch order, so a
// tile only ever waits on tiles that are already running; every wait is
// bounded and, if the bound is hit, sets the error word and proceeds (the
// sort is then wrong but nothing hangs; the host reports the error).
constexpr uint32_t OS_AGG = 1u << 30;      // status: aggregate of this tile only
constexpr uint32_t OS_INC = 2u << 30;      // status: inclusive prefix through this tile
constexpr uint32_t OS_VAL = (1u << 30) - 1;
constexpr uint32_t OS_SPIN_LIMIT = 1u << 20;  // about a second of waiting
constexpr uint32_t OS_ERR_TIMEOUT = 4u;    // JC_ERR_DEVICE_TIMEOUT

__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// A status word carries everything it publishes (flag + count in one 32-bit
// word), so the look-back reads need no acquire ordering: relaxed loads, of
// which a window can be in flight at once (acquire loads would complete one
// after another).
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
constexpr int OS_WINDOW = 8;  // predecessors' status words read per round trip

// counts[p * 256 + digit] for passes p = 0..passes-1 (digit = bits
// bit_begin + 8p .. +8). counts must be zeroed first.
template <typename K>
__global__ void __launch_bounds__(RS_THREADS)
os_hist(const K* __restrict__ keys, uint32_t n_max, const uint32_t* d_count, int bit_begin, int passes,
        uint32_t* __restrict__ counts, const uint32_t* gate) {
  if (gate && *gate == 0) return;
  __shared__ uint32_t h[8][RS_RADIX];
  for (int i = threadIdx.x; i < 8 * RS_RADIX; i += RS_THREADS) (&h[0][0])[i] = 0;
  __syncthreads();
  const uint32_t n = rs_count(n_max, d_count);
  for (uint32_t i = blockIdx.x * RS_THREADS + threadIdx.x; i < n; i += gridDim.x * RS_THREADS) {
    const K k = keys[i];
    for (int p = 0; p < passes; ++p) {
      int sh = bit_begin + 8 * p;
      if (sh >= (int)(8 * sizeof(K))) sh = 8 * (int)sizeof(K) - 8;
      atomicAdd(&h[p][(uint32_t)(k >> sh) & 0xFFu], 1u);
    }
  }
  __syncthreads();
  for (int p = 0; p < passes; ++p) {
    uint32_t v = h[p][threadIdx.x];
    if (v) atomicAdd(&counts[p * RS_RADIX + threadIdx.x], v);
  }
}

template <typename K, int ROUNDS = RS_ROUNDS>
__global__ void __launch_bounds__(RS_THREADS)
os_pass(const K* __restrict__ kin, const uint32_t* __restrict__ vin, K* __restrict__ kout,
        uint32_t* __restrict__ vout, uint32_t n_max, const uint32_t* d_count, int shift,
        const uint32_t* __restrict__ gcount, uint32_t* status, uint32_t* tile_ctr, const uint32_t* gate,
        uint32_t* err) {
  if (gate && *gate == 0) return;
  __shared__ uint32_t wcnt[RS_WARPS][RS_RADIX];
  __shared__ uint32_t base[RS_RADIX];
  __shared__ uint32_t sh_scan[32];
  __shared__ uint32_t s_tile;
  const uint32_t n = rs_count(n_max, d_count);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
  for (int i = threadIdx.x; i < RS_WARPS * RS_RADIX; i += RS_THREADS) (&wcnt[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t chunk = tile * (RS_THREADS * ROUNDS) + w * (ROUNDS * 32);
  const uint32_t lt_mask = (1u << lane) - 1u;
  K key[ROUNDS];
  uint32_t val[ROUNDS];
  uint32_t rank[ROUNDS];
  // all of the tile's loads first (ROUNDS in flight per lane), then the ranking
#pragma unroll
  for (int r = 0; r < ROUNDS; ++r) {
    const uint32_t idx = chunk + r * 32 + lane;
    const bool ok = idx < n;
    key[r] = ok ? kin[idx] : (K)0;
    val[r] = ok ? vin[idx] : 0u;
  }
#pragma unroll
  for (int r = 0; r < ROUNDS; ++r) {
    uint32_t idx = chunk + r * 32 + lane;
    bool ok = idx < n;
    uint32_t d = ok ? ((uint32_t)(key[r] >> shift) & 0xFFu) : 256u;
    // lanes with the same digit: one ballot per digit bit (plus one for the
    // in-range flag), cheaper than match.any on the MIO pipe
    uint32_t peers = ok ? __ballot_sync(0xFFFFFFFFu, ok) : ~__ballot_sync(0xFFFFFFFFu, ok);
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const bool bit = (d >> b) & 1u;
      const uint32_t bb = __ballot_sync(0xFFFFFFFFu, bit);
      peers &= bit ? bb : ~bb;
    }
    uint32_t before = ok ? wcnt[w][d] : 0u;
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) wcnt[w][d] = before + __popc(peers);
    __syncwarp();
    rank[r] = before + __popc(peers & lt_mask);
  }
  __syncthreads();
  const uint32_t d = threadIdx.x;  // RS_THREADS == RS_RADIX: one digit per thread
  uint32_t tot = 0;
#pragma unroll
  for (int ww = 0; ww < RS_WARPS; ++ww) {
    uint32_t c = wcnt[ww][d];
    wcnt[ww][d] = tot;
    tot += c;
  }
  uint32_t* my = status + (size_t)tile * RS_RADIX + d;
  uint32_t excl = 0;
  if (tile == 0) {
    st_release_u32(my, OS_INC | tot);
  } else {
    st_release_u32(my, OS_AGG | tot);
    // All tiles run at once and publish their aggregates early, so the chain
    // back to the nearest inclusive prefix can be long: read OS_WINDOW
    // predecessors per round trip, add them in order, stop at the first
    // inclusive one, and wait (bounded) where a predecessor has not published.
    int64_t t = (int64_t)tile - 1;
    uint32_t spins = 0;
    bool done = false;
    while (!done && t >= 0) {
      uint32_t v[OS_WINDOW];
#pragma unroll
      for (int k = 0; k < OS_WINDOW; ++k)
        v[k] = t - k >= 0 ? ld_relaxed_u32(status + (size_t)(t - k) * RS_RADIX + d) : 0u;
      int k = 0;
#pragma unroll
      for (int q = 0; q < OS_WINDOW; ++q) {
        if (k != q || t - q < 0 || v[q] == 0u || done) continue;
        excl += v[q] & OS_VAL;
        if ((v[q] & ~OS_VAL) == OS_INC) done = true;
        k = q + 1;
      }
      if (done) break;
      t -= k;
      if (k < OS_WINDOW && t >= 0) {  // tile t has not published yet
        if (++spins > OS_SPIN_LIMIT) {
          atomicCAS(err, 0u, OS_ERR_TIMEOUT);
          break;
        }
        __nanosleep(32);
      }
    }
    st_release_u32(my, OS_INC | (excl + tot));
  }
  uint32_t total_dummy;
  const uint32_t start = block_excl_scan_256(gcount[d], &total_dummy, sh_scan);
  base[d] = start + excl;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < ROUNDS; ++r) {
    uint32_t idx = chunk + r * 32 + lane;
    if (idx < n) {
      uint32_t dg = (uint32_t)(key[r] >> shift) & 0xFFu;
      uint32_t dst = base[dg] + wcnt[w][dg] + rank[r];
      if (JC_IN_BOUNDS(dst, n, err)) {
        kout[dst] = key[r];
        vout[dst] = val[r];
      }
    }
  }
}

// Words of workspace one sort needs: digit counts (passes x 256), tile
// counters (passes) and look-back status words (passes x tiles x 256).
__host__ __device__ constexpr size_t sort_work_words(uint32_t n_max, int passes) {
  return (size_t)passes * RS_RADIX + passes + (size_t)passes * rs_tiles(n_max) * RS_RADIX;
}

// Sorts (keys, vals) by bits [bit_begin, bit_end) with an even number of
// passes (the result ends in keys/vals). `work` holds sort_work_words words.
// Returns the number of nodes (kernels + memsets) issued.
template <typename K>
inline int radix_sort_pairs(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt, uint32_t n_max,
                            const uint32_t* d_count, int bit_begin, int bit_end, uint32_t* work,
                            uint32_t* err, const uint32_t* gate, cudaStream_t s) {
  if (n_max == 0) return 0;
  const uint32_t tiles = rs_tiles(n_max);
  const bool small = rs_rounds(n_max) == RS_ROUNDS_SMALL;
  int passes = (bit_end - bit_begin + 7) / 8;
  if (passes & 1) ++passes;
  uint32_t* counts = work;
  uint32_t* tile_ctr = counts + passes * RS_RADIX;
  uint32_t* status = tile_ctr + passes;
  cudaMemsetAsync(work, 0, sizeof(uint32_t) * sort_work_words(n_max, passes), s);
  const uint32_t hist_blocks = tiles < 592u ? tiles : 592u;
  os_hist<K><<<hist_blocks, RS_THREADS, 0, s>>>(keys, n_max, d_count, bit_begin, passes, counts, gate);
  K* kin = keys;
  uint32_t* vin = vals;
  K* kout = keys_alt;
  uint32_t* vout = vals_alt;
  for (int p = 0; p < passes; ++p) {
    int shift = bit_begin + 8 * p;
    if (shift >= (int)(8 * sizeof(K))) shift = 8 * (int)sizeof(K) - 8;
    if (small)
      os_pass<K, RS_ROUNDS_SMALL><<<tiles, RS_THREADS, 0, s>>>(kin, vin, kout, vout, n_max, d_count, shift,
                                                               counts + p * RS_RADIX,
                                                               status + (size_t)p * tiles * RS_RADIX, tile_ctr + p,
                                                               gate, err);
    else
      os_pass<K, RS_ROUNDS><<<tiles, RS_THREADS, 0, s>>>(kin, vin, kout, vout, n_max, d_count, shift,
                                                         counts + p * RS_RADIX, status + (size_t)p * tiles * RS_RADIX,
                                                         tile_ctr + p, gate, err);
    K* tk = kin; kin = kout; kout = tk;
    uint32_t* tv = vin; vin = vout; vout = tv;
  }
  return 2 + passes;
}

// ---------------------------------------------------------------- scan --
// Exclusive scan of u32 over [0, len) in three kernels (tile sums, scan of
// tile sums in one block, tile scans + offsets). out may alias in. The total
// is written to out[len] (so out needs len + 1 entries).
constexpr int SC_THREADS = 512;
constexpr int SC_PER = 8;
constexpr int SC_TILE = SC_THREADS * SC_PER;  // 4096

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t x, uint32_t* total, uint32_t* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  uint32_t v = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, v, o);
    if (lane >= o) v += y;
  }
  if (lane == 31) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    uint32_t t = lane < nw ? sh[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
      if (lane >= o) t += y;
    }
    sh[lane] = t;
  }
  __syncthreads();
  uint32_t ex = v - x + (w > 0 ? sh[w - 1] : 0u);
  *total = sh[nw - 1];
  __syncthreads();
  return ex;
}

__global__ void __launch_bounds__(SC_THREADS)
sc_tile_sums(const uint32_t* __restrict__ in, uint32_t len, uint32_t* __restrict__ sums) {
  __shared__ uint32_t sh[32];
  uint32_t base = blockIdx.x * SC_TILE + threadIdx.x * SC_PER;
  uint32_t acc = 0;
#pragma unroll
  for (int k = 0; k < SC_PER; ++k)
    if (base + k < len) acc += in[base + k];
  uint32_t tot;
  block_excl_scan(acc, &tot, sh);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) sc_scan_sums(uint32_t* sums, uint32_t n_tiles) {
  __shared__ uint32_t sh[32];
  // sequential chunks per thread (n_tiles is small: len / 4096)
  const uint32_t per = (n_tiles + 1023) / 1024;
  const uint32_t b = threadIdx.x * per, e = min(n_tiles, b + per);
  uint32_t local = 0;
  for (uint32_t i = b; i < e; ++i) local += sums[i];
  uint32_t tot;
  uint32_t run = block_excl_scan(local, &tot, sh);
  for (uint32_t i = b; i < e; ++i) {
    uint32_t v = sums[i];
    sums[i] = run;
    run += v;
  }
  if (threadIdx.x == 0) sums[n_tiles] = tot;
}

__global__ void __launch_bounds__(SC_THREADS)
sc_tile_scan(const uint32_t* in, uint32_t len, const uint32_t* __restrict__ sums, uint32_t* out) {
  __shared__ uint32_t sh[32];
  uint32_t base = blockIdx.x * SC_TILE + threadIdx.x * SC_PER;
  uint32_t v[SC_PER];
  uint32_t acc = 0;
#pragma unroll
  for (int k = 0; k < SC_PER; ++k) {
    v[k] = (base + k < len) ? in[base + k] : 0u;
    acc += v[k];
  }
  uint32_t tot;
  uint32_t run = block_excl_scan(acc, &tot, sh) + sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SC_PER; ++k) {
    if (base + k < len) out[base + k] = run;
    run += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[len] = sums[gridDim.x];
}

// Short inputs (up to SC_SMALL): one block walks the input in chunks of
// 8,192, carrying the running total, instead of three launches.
constexpr uint32_t SC_SMALL = 65536;
__global__ void __launch_bounds__(1024) sc_small(const uint32_t* in, uint32_t len, uint32_t* out) {
  __shared__ uint32_t sh[32];
  uint32_t carry = 0;
  for (uint32_t c0 = 0; c0 < len; c0 += 1024 * SC_PER) {
    const uint32_t base = c0 + threadIdx.x * SC_PER;
    uint32_t v[SC_PER];
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < SC_PER; ++k) {
      v[k] = (base + k < len) ? in[base + k] : 0u;
      acc += v[k];
    }
    uint32_t tot;
    uint32_t run = block_excl_scan(acc, &tot, sh) + carry;
#pragma unroll
    for (int k = 0; k < SC_PER; ++k) {
      if (base + k < len) out[base + k] = run;
      run += v[k];
    }
    carry += tot;
  }
  if (threadIdx.x == 0) out[len] = carry;
}

// sums must hold n_tiles + 1 entries, n_tiles = ceil(len / SC_TILE).
inline int exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t len, uint32_t* sums,
                          cudaStream_t s) {
  if (len <= SC_SMALL) {
    sc_small<<<1, 1024, 0, s>>>(in, len, out);
    return 1;
  }
  uint32_t n_tiles = (len + SC_TILE - 1) / SC_TILE;
  if (n_tiles == 0) n_tiles = 1;
  sc_tile_sums<<<n_tiles, SC_THREADS, 0, s>>>(in, len, sums);
  sc_scan_sums<<<1, 1024, 0, s>>>(sums, n_tiles);
  sc_tile_scan<<<n_tiles, SC_THREADS, 0, s>>>(in, len, sums, out);
  return 3;
}

}  // namespace dev
}  // namespace jc
