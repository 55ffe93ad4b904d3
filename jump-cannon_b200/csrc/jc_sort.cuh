// Device-wide primitives for the octree build: a stable LSD radix sort of
// (key, u32 value) pairs with 8-bit digits, and an exclusive scan of u32.
//
// Both read their item count from device memory (so they can sit inside a
// captured CUDA graph while the count changes from step to step) and accept
// an optional device "gate" word: when the gate is 0 every kernel returns at
// once, which is how the rare tie-breaking re-sort is made conditional
// without a host round trip.
//
// Radix pass = three kernels:
//   rs_hist    per-tile digit histogram        -> counts[digit * tiles + tile]
//   rs_scan    exclusive scan of counts (digit-major, so equal digits keep
//              tile order = stability across tiles)
//   rs_scatter per-tile stable ranking (warp match_any + per-warp counters,
//              item order inside a tile = warp, round, lane = input order)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace jc {
namespace dev {

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ROUNDS = 16;                        // items per lane
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;      // 4096 items per block
constexpr int RS_RADIX = 256;

__device__ __forceinline__ uint32_t rs_count(uint32_t n_max, const uint32_t* d_count) {
  if (d_count == nullptr) return n_max;
  uint32_t c = *d_count;
  return c < n_max ? c : n_max;
}

template <typename K>
__global__ void __launch_bounds__(RS_THREADS)
rs_hist(const K* __restrict__ keys, uint32_t n_max, const uint32_t* d_count, int shift,
        uint32_t* __restrict__ counts, uint32_t tiles, const uint32_t* gate) {
  if (gate && *gate == 0) return;
  __shared__ uint32_t h[RS_RADIX];
  const uint32_t n = rs_count(n_max, d_count);
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t base = blockIdx.x * RS_TILE;
#pragma unroll 4
  for (int r = 0; r < RS_ROUNDS; ++r) {
    uint32_t idx = base + r * RS_THREADS + threadIdx.x;
    if (idx < n) atomicAdd(&h[(uint32_t)(keys[idx] >> shift) & 0xFFu], 1u);
  }
  __syncthreads();
  counts[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of `len` u32 in place by one block of 1024 threads, each
// owning a contiguous chunk. Used for the (256 x tiles) digit counts.
__global__ void __launch_bounds__(1024) rs_scan(uint32_t* data, uint32_t len, const uint32_t* gate) {
  if (gate && *gate == 0) return;
  __shared__ uint32_t warp_tot[32];
  const uint32_t per = (len + 1023) / 1024;
  const uint32_t b = threadIdx.x * per;
  const uint32_t e = min(len, b + per);
  uint32_t local = 0;
  for (uint32_t i = b; i < e; ++i) local += data[i];
  // block-wide exclusive scan of `local`
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t t = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;  // inclusive
  }
  __syncthreads();
  uint32_t run = x - local + (w > 0 ? warp_tot[w - 1] : 0u);
  for (uint32_t i = b; i < e; ++i) {
    uint32_t v = data[i];
    data[i] = run;
    run += v;
  }
}

template <typename K>
__global__ void __launch_bounds__(RS_THREADS)
rs_scatter(const K* __restrict__ kin, const uint32_t* __restrict__ vin, K* __restrict__ kout,
           uint32_t* __restrict__ vout, uint32_t n_max, const uint32_t* d_count, int shift,
           const uint32_t* __restrict__ offsets, uint32_t tiles, const uint32_t* gate) {
  if (gate && *gate == 0) return;
  __shared__ uint32_t wcnt[RS_WARPS][RS_RADIX];
  __shared__ uint32_t boff[RS_RADIX];
  const uint32_t n = rs_count(n_max, d_count);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < RS_WARPS * RS_RADIX; i += RS_THREADS) (&wcnt[0][0])[i] = 0;
  __syncthreads();
  const uint32_t chunk = blockIdx.x * RS_TILE + w * (RS_ROUNDS * 32);
  const uint32_t lt_mask = (1u << lane) - 1u;
  K key[RS_ROUNDS];
  uint32_t val[RS_ROUNDS];
  uint32_t rank[RS_ROUNDS];
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    uint32_t idx = chunk + r * 32 + lane;
    bool ok = idx < n;
    key[r] = ok ? kin[idx] : (K)0;
    val[r] = ok ? vin[idx] : 0u;
    uint32_t d = ok ? ((uint32_t)(key[r] >> shift) & 0xFFu) : 256u;
    uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
    uint32_t before = ok ? wcnt[w][d] : 0u;
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) wcnt[w][d] = before + __popc(peers);
    __syncwarp();
    rank[r] = before + __popc(peers & lt_mask);
  }
  __syncthreads();
  {
    uint32_t t = threadIdx.x;  // RS_THREADS == RS_RADIX
    uint32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < RS_WARPS; ++ww) {
      uint32_t c = wcnt[ww][t];
      wcnt[ww][t] = run;
      run += c;
    }
    boff[t] = offsets[t * tiles + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    uint32_t idx = chunk + r * 32 + lane;
    if (idx < n) {
      uint32_t d = (uint32_t)(key[r] >> shift) & 0xFFu;
      uint32_t dst = boff[d] + wcnt[w][d] + rank[r];
      kout[dst] = key[r];
      vout[dst] = val[r];
    }
  }
}

// Host launcher: sorts (keys, vals) by bits [bit_begin, bit_end) with an even
// number of passes, so the sorted result ends in keys/vals again.
// counts must hold 256 * tiles u32, tiles = ceil(n_max / RS_TILE).
// Returns the number of kernel launches issued.
template <typename K>
inline int radix_sort_pairs(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt,
                            uint32_t n_max, const uint32_t* d_count, int bit_begin, int bit_end,
                            uint32_t* counts, const uint32_t* gate, cudaStream_t s) {
  if (n_max == 0) return 0;
  const uint32_t tiles = (n_max + RS_TILE - 1) / RS_TILE;
  int passes = (bit_end - bit_begin + 7) / 8;
  if (passes & 1) ++passes;
  K* kin = keys;
  uint32_t* vin = vals;
  K* kout = keys_alt;
  uint32_t* vout = vals_alt;
  int launches = 0;
  for (int p = 0; p < passes; ++p) {
    int shift = bit_begin + 8 * p;
    if (shift >= (int)(8 * sizeof(K))) shift = 8 * (int)sizeof(K) - 8;  // padding pass: stable no-op order
    rs_hist<K><<<tiles, RS_THREADS, 0, s>>>(kin, n_max, d_count, shift, counts, tiles, gate);
    rs_scan<<<1, 1024, 0, s>>>(counts, RS_RADIX * tiles, gate);
    rs_scatter<K><<<tiles, RS_THREADS, 0, s>>>(kin, vin, kout, vout, n_max, d_count, shift, counts,
                                              tiles, gate);
    launches += 3;
    K* tk = kin; kin = kout; kout = tk;
    uint32_t* tv = vin; vin = vout; vout = tv;
  }
  return launches;
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

// sums must hold n_tiles + 1 entries, n_tiles = ceil(len / SC_TILE).
inline int exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t len, uint32_t* sums,
                          cudaStream_t s) {
  uint32_t n_tiles = (len + SC_TILE - 1) / SC_TILE;
  if (n_tiles == 0) n_tiles = 1;
  sc_tile_sums<<<n_tiles, SC_THREADS, 0, s>>>(in, len, sums);
  sc_scan_sums<<<1, 1024, 0, s>>>(sums, n_tiles);
  sc_tile_scan<<<n_tiles, SC_THREADS, 0, s>>>(in, len, sums, out);
  return 3;
}

}  // namespace dev
}  // namespace jc
