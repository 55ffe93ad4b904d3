// Synthetic graphs and seed layouts for the layout engines.
//
// The reference's own fixtures are restated bit-compatibly so seeds reproduce
// its graphs: synthetic_scale_free, csr_from_pairs and ball_seed
// (crates/graph-compute/src/stability.rs:30-110), CsrGraph::path
// (crates/graph-compute/src/sim.rs:31-49) and the tests' grid2d
// (crates/graph-compute/tests/gpu_engines.rs:267-292). The reference has no
// R-MAT, Watts–Strogatz or random-geometric generator; those are written
// here from their published definitions, seeded with the same SplitMix64.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <unordered_set>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "jc_common.h"

struct jc_csr {
  uint32_t n = 0;
  std::vector<uint32_t> offsets;
  std::vector<uint32_t> neighbors;
};

namespace {

// stability.rs:86-110: symmetric CSR, both directions, each row sorted and
// deduplicated; self-loops and out-of-range endpoints skipped.
jc_csr* csr_from_pairs_impl(uint32_t n, const uint32_t* pairs, uint64_t count) {
  jc_csr* g = new jc_csr();
  g->n = n;
  std::vector<uint64_t> cnt((size_t)n + 1, 0);
  for (uint64_t t = 0; t < count; ++t) {
    uint32_t a = pairs[2 * t], b = pairs[2 * t + 1];
    if (a == b || a >= n || b >= n) continue;
    cnt[a + 1]++;
    cnt[b + 1]++;
  }
  for (uint32_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
  std::vector<uint32_t> raw(cnt[n]);
  std::vector<uint64_t> cur(cnt.begin(), cnt.end() - 1);
  for (uint64_t t = 0; t < count; ++t) {
    uint32_t a = pairs[2 * t], b = pairs[2 * t + 1];
    if (a == b || a >= n || b >= n) continue;
    raw[cur[a]++] = b;
    raw[cur[b]++] = a;
  }
  std::vector<uint32_t> keep((size_t)n, 0);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1024)
#endif
  for (int64_t v = 0; v < (int64_t)n; ++v) {
    auto b = raw.begin() + (int64_t)cnt[v], e = raw.begin() + (int64_t)cnt[v + 1];
    std::sort(b, e);
    keep[v] = (uint32_t)(std::unique(b, e) - b);
  }
  g->offsets.assign((size_t)n + 1, 0);
  for (uint32_t v = 0; v < n; ++v) g->offsets[v + 1] = g->offsets[v] + keep[v];
  g->neighbors.resize(g->offsets[n]);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1024)
#endif
  for (int64_t v = 0; v < (int64_t)n; ++v)
    std::memcpy(&g->neighbors[g->offsets[v]], &raw[cnt[v]], sizeof(uint32_t) * keep[v]);
  return g;
}

// Open-addressing set of non-zero u64 keys (0 = empty slot).
struct PairSet {
  std::vector<uint64_t> slots;
  uint64_t mask;
  explicit PairSet(uint64_t expect) {
    uint64_t cap = 16;
    while (cap < expect * 2) cap <<= 1;
    slots.assign(cap, 0);
    mask = cap - 1;
  }
  bool insert(uint64_t key) {
    uint64_t h = jc::SplitMix64::mix(key) & mask;
    for (;;) {
      uint64_t s = slots[h];
      if (s == key) return false;
      if (s == 0) { slots[h] = key; return true; }
      h = (h + 1) & mask;
    }
  }
};

}  // namespace

extern "C" {

jc_csr* jc_csr_from_pairs(uint32_t n, const uint32_t* pairs, uint64_t count) {
  try {
    return csr_from_pairs_impl(n, pairs, count);
  } catch (...) {
    return nullptr;
  }
}

// stability.rs:56-81
jc_csr* jc_gen_scale_free(uint32_t n_in, uint32_t m_in, uint64_t seed) {
  try {
    jc::SplitMix64 rng(seed);
    uint32_t n = std::max(n_in, 2u);
    size_t m = std::max<size_t>(m_in, 1);
    std::vector<uint32_t> targets = {0, 1, 1, 0};
    std::vector<uint32_t> pairs = {0, 1};
    std::vector<uint32_t> picked;
    for (uint32_t v = 2; v < n; ++v) {
      picked.clear();
      int guard = 0;
      while (picked.size() < std::min<size_t>(m, v) && guard < 64) {
        ++guard;
        uint32_t t = targets[(size_t)(rng.next_u64() % (uint64_t)targets.size())];
        if (t != v && std::find(picked.begin(), picked.end(), t) == picked.end()) picked.push_back(t);
      }
      for (uint32_t t : picked) {
        pairs.push_back(v);
        pairs.push_back(t);
        targets.push_back(v);
        targets.push_back(t);
      }
    }
    return csr_from_pairs_impl(n, pairs.data(), pairs.size() / 2);
  } catch (...) {
    return nullptr;
  }
}

// sim.rs:31-49
jc_csr* jc_gen_path(uint32_t n) {
  jc_csr* g = new (std::nothrow) jc_csr();
  if (!g) return nullptr;
  g->n = n;
  g->offsets.reserve((size_t)n + 1);
  for (uint32_t i = 0; i < n; ++i) {
    g->offsets.push_back((uint32_t)g->neighbors.size());
    if (i > 0) g->neighbors.push_back(i - 1);
    if (i + 1 < n) g->neighbors.push_back(i + 1);
  }
  g->offsets.push_back((uint32_t)g->neighbors.size());
  return g;
}

// gpu_engines.rs:267-292 (square dim x dim there; width x height here, same
// neighbour order: left, right, up, down).
jc_csr* jc_gen_grid(uint32_t w, uint32_t h) {
  jc_csr* g = new (std::nothrow) jc_csr();
  if (!g) return nullptr;
  g->n = w * h;
  g->offsets.push_back(0);
  for (uint32_t y = 0; y < h; ++y)
    for (uint32_t x = 0; x < w; ++x) {
      if (x > 0) g->neighbors.push_back(y * w + (x - 1));
      if (x + 1 < w) g->neighbors.push_back(y * w + (x + 1));
      if (y > 0) g->neighbors.push_back((y - 1) * w + x);
      if (y + 1 < h) g->neighbors.push_back((y + 1) * w + x);
      g->offsets.push_back((uint32_t)g->neighbors.size());
    }
  return g;
}

// R-MAT (Chakrabarti, Zhan, Faloutsos 2004): each edge descends `scale`
// levels of the adjacency matrix, choosing quadrant (0,0),(0,1),(1,0),(1,1)
// with probabilities a, b, c, 1-a-b-c. Vertex labels are not permuted.
// Sampling stops at `n_edges` unique undirected non-self pairs.
jc_csr* jc_gen_rmat(uint32_t scale, uint64_t n_edges, double a, double b, double c, uint64_t seed) {
  try {
    if (scale == 0 || scale > 31) return nullptr;
    uint32_t n = 1u << scale;
    uint64_t max_pairs = (uint64_t)n * (n - 1) / 2;
    if (n_edges > max_pairs / 2) return nullptr;  // keep rejection sampling bounded
    jc::SplitMix64 rng(seed);
    PairSet set(n_edges);
    std::vector<uint32_t> pairs;
    pairs.reserve(2 * n_edges);
    double ab = a + b, abc = a + b + c;
    uint64_t have = 0;
    while (have < n_edges) {
      uint32_t u = 0, v = 0;
      for (uint32_t l = 0; l < scale; ++l) {
        double r = rng.next_f64();
        uint32_t bu = 0, bv = 0;
        if (r < a) {
        } else if (r < ab) {
          bv = 1;
        } else if (r < abc) {
          bu = 1;
        } else {
          bu = 1;
          bv = 1;
        }
        u = (u << 1) | bu;
        v = (v << 1) | bv;
      }
      if (u == v) continue;
      uint32_t lo = std::min(u, v), hi = std::max(u, v);
      if (set.insert(((uint64_t)lo << 32) | hi)) {
        pairs.push_back(u);
        pairs.push_back(v);
        ++have;
      }
    }
    return csr_from_pairs_impl(n, pairs.data(), have);
  } catch (...) {
    return nullptr;
  }
}

// Watts & Strogatz 1998: ring lattice, node i joined to i+1..i+k/2; each
// lattice edge (u, u+j) is rewired with probability p to (u, w), w uniform,
// avoiding self-loops and existing edges.
jc_csr* jc_gen_watts_strogatz(uint32_t n, uint32_t k, double p, uint64_t seed) {
  try {
    if (n < 3) return jc_gen_path(n);
    jc::SplitMix64 rng(seed);
    uint32_t half = std::max(1u, k / 2);
    std::unordered_set<uint64_t> edges;
    auto key = [](uint32_t x, uint32_t y) {
      uint32_t lo = std::min(x, y), hi = std::max(x, y);
      return ((uint64_t)lo << 32) | hi;
    };
    std::vector<std::pair<uint32_t, uint32_t>> list;
    for (uint32_t j = 1; j <= half; ++j)
      for (uint32_t u = 0; u < n; ++u) {
        uint32_t v = (u + j) % n;
        if (u != v && edges.insert(key(u, v)).second) list.push_back({u, v});
      }
    for (auto& e : list) {
      if (rng.next_f64() >= p) continue;
      uint32_t u = e.first;
      for (int tries = 0; tries < 64; ++tries) {
        uint32_t w = (uint32_t)rng.below(n);
        if (w == u || edges.count(key(u, w))) continue;
        edges.erase(key(e.first, e.second));
        edges.insert(key(u, w));
        e.second = w;
        break;
      }
    }
    std::vector<uint32_t> pairs;
    pairs.reserve(list.size() * 2);
    for (auto& e : list) {
      pairs.push_back(e.first);
      pairs.push_back(e.second);
    }
    return csr_from_pairs_impl(n, pairs.data(), list.size());
  } catch (...) {
    return nullptr;
  }
}

// Random geometric graph (Penrose 2003): n points uniform in the unit square,
// an edge between every pair closer than `radius` (cell-list search).
jc_csr* jc_gen_rgg(uint32_t n, double radius, uint64_t seed, float* points_xy) {
  try {
    jc::SplitMix64 rng(seed);
    std::vector<float> xy((size_t)2 * n);
    for (size_t i = 0; i < (size_t)2 * n; ++i) xy[i] = rng.next_f32();
    if (points_xy) std::memcpy(points_xy, xy.data(), sizeof(float) * 2 * n);
    uint32_t cells = (uint32_t)std::max(1.0, std::floor(1.0 / std::max(radius, 1e-9)));
    cells = std::min(cells, 4096u);
    std::vector<uint32_t> cnt((size_t)cells * cells + 1, 0), idx(n);
    auto cell_of = [&](uint32_t i) {
      uint32_t cx = std::min(cells - 1, (uint32_t)(xy[2 * i] * cells));
      uint32_t cy = std::min(cells - 1, (uint32_t)(xy[2 * i + 1] * cells));
      return cy * cells + cx;
    };
    for (uint32_t i = 0; i < n; ++i) cnt[cell_of(i) + 1]++;
    for (size_t c = 0; c < (size_t)cells * cells; ++c) cnt[c + 1] += cnt[c];
    std::vector<uint32_t> cur(cnt.begin(), cnt.end() - 1);
    for (uint32_t i = 0; i < n; ++i) idx[cur[cell_of(i)]++] = i;
    double r2 = radius * radius;
    std::vector<uint32_t> pairs;
    for (uint32_t i = 0; i < n; ++i) {
      uint32_t c = cell_of(i), cx = c % cells, cy = c / cells;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int64_t nx = (int64_t)cx + dx, ny = (int64_t)cy + dy;
          if (nx < 0 || ny < 0 || nx >= cells || ny >= cells) continue;
          size_t cc = (size_t)ny * cells + (size_t)nx;
          for (uint32_t t = cnt[cc]; t < cnt[cc + 1]; ++t) {
            uint32_t j = idx[t];
            if (j <= i) continue;
            double ddx = (double)xy[2 * i] - xy[2 * j], ddy = (double)xy[2 * i + 1] - xy[2 * j + 1];
            if (ddx * ddx + ddy * ddy <= r2) {
              pairs.push_back(i);
              pairs.push_back(j);
            }
          }
        }
    }
    return csr_from_pairs_impl(n, pairs.data(), pairs.size() / 2);
  } catch (...) {
    return nullptr;
  }
}

uint32_t jc_csr_n_nodes(const jc_csr* g) { return g ? g->n : 0; }
uint64_t jc_csr_n_neighbors(const jc_csr* g) { return g ? g->neighbors.size() : 0; }
const uint32_t* jc_csr_offsets(const jc_csr* g) { return g ? g->offsets.data() : nullptr; }
const uint32_t* jc_csr_neighbors(const jc_csr* g) { return g ? g->neighbors.data() : nullptr; }
void jc_csr_free(jc_csr* g) { delete g; }

// stability.rs:30-49: rejection-sampled ball of radius sqrt(n)*5.
void jc_seed_ball(uint32_t n, uint64_t seed, float* out) {
  jc::SplitMix64 rng(seed);
  float radius = std::sqrt((float)n) * 5.0f;
  for (uint32_t i = 0; i < n; ++i) {
    for (;;) {
      float x = 2.0f * rng.next_f32() - 1.0f;
      float y = 2.0f * rng.next_f32() - 1.0f;
      float z = 2.0f * rng.next_f32() - 1.0f;
      if (x * x + y * y + z * z <= 1.0f) {
        out[3 * (size_t)i] = x * radius;
        out[3 * (size_t)i + 1] = y * radius;
        out[3 * (size_t)i + 2] = z * radius;
        break;
      }
    }
  }
}

// Uniform seed in [-1,1]^dim: 2*next_f32()-1 per coordinate, node by node.
void jc_seed_uniform(uint32_t n, uint32_t dim, uint64_t seed, float* out) {
  jc::SplitMix64 rng(seed);
  for (uint32_t i = 0; i < n; ++i) {
    out[3 * (size_t)i] = 2.0f * rng.next_f32() - 1.0f;
    out[3 * (size_t)i + 1] = 2.0f * rng.next_f32() - 1.0f;
    out[3 * (size_t)i + 2] = dim >= 3 ? 2.0f * rng.next_f32() - 1.0f : 0.0f;
  }
}

}  // extern "C"
