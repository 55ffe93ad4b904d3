// Seeded workload generators for the oracle side — TEST INFRASTRUCTURE ONLY.
//
// The reference arm of the benchmark and the CPU-baseline leg must build
// their input graph without loading the product library, so the oracle
// carries its own generator for the one graph family that arm times:
//
//   * SplitMix64 exactly as crates/graph-compute/src/stability.rs:11-26
//     (next_u64, next_f32 = top 24 bits / 2^24), plus next_f64 = top 53 bits
//     / 2^53;
//   * R-MAT (Chakrabarti, Zhan & Faloutsos 2004): every candidate edge
//     descends `scale` levels of the adjacency matrix, one uniform f64 draw
//     per level picking quadrant (0,0) / (0,1) / (1,0) / (1,1) with
//     probabilities a, b, c, 1-a-b-c (row bit to u, column bit to v, most
//     significant first); self pairs are dropped and sampling stops at the
//     first `n_edges` distinct unordered pairs in draw order; labels are not
//     permuted;
//   * the symmetric CSR of those pairs, each row sorted ascending and
//     deduplicated (csr_from_pairs, stability.rs:86-110);
//   * the uniform seed 2*next_f32()-1 per coordinate, node by node (z = 0
//     for dim 2).
//
// tests/test_oracle_graphgen.py checks that the product library's generator
// gives the same CSR and seed.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct Mix64 {  // stability.rs:11-26
  uint64_t s;
  uint64_t next_u64() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  float next_f32() { return (float)(next_u64() >> 40) / (float)(1u << 24); }
  double next_f64() { return (double)(next_u64() >> 11) / 9007199254740992.0; }
};

// Linear-probing set of non-zero 64-bit keys (Fibonacci hashing).
class KeySet {
 public:
  explicit KeySet(uint64_t expect) {
    int bits = 4;
    while ((1ull << bits) < 2 * expect + 16) ++bits;
    shift_ = 64 - bits;
    mask_ = (1ull << bits) - 1;
    slot_.assign(1ull << bits, 0);
  }
  bool add(uint64_t k) {
    uint64_t h = (k * 0x9E3779B97F4A7C15ull) >> shift_;
    while (slot_[h] != 0) {
      if (slot_[h] == k) return false;
      h = (h + 1) & mask_;
    }
    slot_[h] = k;
    return true;
  }

 private:
  std::vector<uint64_t> slot_;
  uint64_t mask_ = 0;
  int shift_ = 0;
};

}  // namespace

extern "C" {

// R-MAT pairs: writes up to `n_edges` distinct unordered pairs as (lo, hi)
// into pairs_out[2 * n_edges]; returns the number written (0 on bad args).
uint64_t orc_gen_rmat_pairs(uint32_t scale, uint64_t n_edges, double a, double b, double c, uint64_t seed,
                            uint32_t* pairs_out) {
  if (scale == 0 || scale > 31) return 0;
  const uint64_t n = 1ull << scale;
  if (n_edges > n * (n - 1) / 4) return 0;  // rejection sampling stays bounded
  Mix64 rng{seed};
  KeySet seen(n_edges);
  uint64_t have = 0;
  while (have < n_edges) {
    uint32_t u = 0, v = 0;
    for (uint32_t l = 0; l < scale; ++l) {
      const double r = rng.next_f64();
      const uint32_t q = r < a ? 0u : r < a + b ? 1u : r < a + b + c ? 2u : 3u;
      u = (u << 1) | (q >> 1);
      v = (v << 1) | (q & 1u);
    }
    if (u == v) continue;
    const uint32_t lo = u < v ? u : v, hi = u < v ? v : u;
    if (seen.add(((uint64_t)lo << 32) | (uint64_t)hi)) {
      pairs_out[2 * have] = lo;
      pairs_out[2 * have + 1] = hi;
      ++have;
    }
  }
  return have;
}

// Symmetric CSR of unordered pairs (self pairs and out-of-range ids
// skipped), rows sorted and deduplicated. offsets_out[n + 1]; neighbors_out
// must hold 2 * count entries; returns offsets_out[n].
uint64_t orc_csr_from_pairs(uint32_t n, const uint32_t* pairs, uint64_t count, uint32_t* offsets_out,
                            uint32_t* neighbors_out) {
  std::vector<uint64_t> start((size_t)n + 1, 0);
  for (uint64_t t = 0; t < count; ++t) {
    const uint32_t x = pairs[2 * t], y = pairs[2 * t + 1];
    if (x == y || x >= n || y >= n) continue;
    ++start[x + 1];
    ++start[y + 1];
  }
  for (uint32_t i = 0; i < n; ++i) start[i + 1] += start[i];
  std::vector<uint32_t> all(start[n]);
  std::vector<uint64_t> fill(start.begin(), start.end() - 1);
  for (uint64_t t = 0; t < count; ++t) {
    const uint32_t x = pairs[2 * t], y = pairs[2 * t + 1];
    if (x == y || x >= n || y >= n) continue;
    all[fill[x]++] = y;
    all[fill[y]++] = x;
  }
  uint64_t w = 0;
  offsets_out[0] = 0;
  for (uint32_t i = 0; i < n; ++i) {
    auto b = all.begin() + (int64_t)start[i], e = all.begin() + (int64_t)start[i + 1];
    std::sort(b, e);
    e = std::unique(b, e);
    for (auto it = b; it != e; ++it) neighbors_out[w++] = *it;
    offsets_out[i + 1] = (uint32_t)w;
  }
  return w;
}

// Uniform seed in [-1, 1]^dim, 3 floats per node (z = 0 when dim < 3).
void orc_seed_uniform(uint32_t n, uint32_t dim, uint64_t seed, float* xyz_out) {
  Mix64 rng{seed};
  for (uint64_t i = 0; i < n; ++i) {
    xyz_out[3 * i] = 2.0f * rng.next_f32() - 1.0f;
    xyz_out[3 * i + 1] = 2.0f * rng.next_f32() - 1.0f;
    xyz_out[3 * i + 2] = dim >= 3 ? 2.0f * rng.next_f32() - 1.0f : 0.0f;
  }
}

}  // extern "C"
