// CPU oracle for the multilevel wrapper — TEST INFRASTRUCTURE ONLY (loaded by
// tests/ through liboracle.so; never linked into the product library).
//
// A line-by-line restatement of
//   crates/graph-layouts/src/layout/coarsen.rs
//     coarsen :52-90, contract_one_level :96-150, prolong :157-183
//   crates/graph-compute/src/engines/multilevel.rs
//     SweepSchedule::sweeps_for_level :104-120, level_csr :259-294,
//     edge flattening in init :372-386, fold_up :480-510
// in the reference's own sequential order, so that the device cascade,
// fold-up and prolongation (jump-cannon_b200/csrc/jc_multilevel.cu) can be
// compared with it bit for bit. Pinned by the reference's coarsen tests
// (coarsen.rs:325-358), restated in tests/test_multilevel.py.
#include <cstdint>
#include <cstring>
#include <unordered_set>
#include <vector>

namespace {

struct Level {
  uint32_t n;
  std::vector<uint32_t> edges;       // flat [s,t, s,t, ...]
  std::vector<uint32_t> parent_map;  // length = previous level's n (empty at level 0)
};

struct Cascade {
  std::vector<Level> levels;
};

void contract_one_level(uint32_t n, const std::vector<uint32_t>& edges, uint32_t* n_super_out,
                        std::vector<uint32_t>* parent_out, std::vector<uint32_t>* edges_out) {
  std::vector<uint32_t> parent(n, 0xFFFFFFFFu);
  uint32_t next_super = 0;
  for (size_t i = 0; i + 1 < edges.size(); i += 2) {
    const uint32_t s = edges[i], t = edges[i + 1];
    if (s == t || s >= n || t >= n) continue;
    if (parent[s] == 0xFFFFFFFFu && parent[t] == 0xFFFFFFFFu) {
      parent[s] = next_super;
      parent[t] = next_super;
      next_super += 1;
    }
  }
  for (uint32_t& p : parent)
    if (p == 0xFFFFFFFFu) p = next_super++;
  std::unordered_set<uint64_t> seen;
  std::vector<uint32_t> out;
  for (size_t j = 0; j + 1 < edges.size(); j += 2) {
    const uint32_t es = edges[j], et = edges[j + 1];
    if (es >= n || et >= n) continue;
    const uint32_t s = parent[es], t = parent[et];
    if (s == t) continue;
    const uint32_t a = s < t ? s : t, b = s < t ? t : s;
    if (seen.insert(((uint64_t)a << 32) | b).second) {
      out.push_back(s);
      out.push_back(t);
    }
  }
  *n_super_out = next_super;
  *parent_out = std::move(parent);
  *edges_out = std::move(out);
}

}  // namespace

extern "C" {

void* orc_coarsen(uint32_t n, const uint32_t* edges, uint64_t n_words, uint64_t max_levels, uint64_t target_size) {
  Cascade* c = new Cascade();
  c->levels.push_back(Level{n, std::vector<uint32_t>(edges, edges + n_words), {}});
  for (uint64_t it = 1; it < max_levels; ++it) {
    const Level& cur = c->levels.back();
    if (cur.n <= target_size) break;
    Level next;
    contract_one_level(cur.n, cur.edges, &next.n, &next.parent_map, &next.edges);
    const float ratio = (float)cur.n / (float)(next.n > 1 ? next.n : 1);
    if (ratio < 1.6f && next.n == cur.n) break;
    const uint32_t nn = next.n;
    c->levels.push_back(std::move(next));
    if (nn <= target_size || ratio < 1.6f) break;
  }
  return c;
}

uint32_t orc_cascade_levels(void* h) { return (uint32_t)((Cascade*)h)->levels.size(); }

uint32_t orc_cascade_level(void* h, uint32_t l, uint64_t* n_words) {
  const Level& L = ((Cascade*)h)->levels[l];
  *n_words = L.edges.size();
  return L.n;
}

void orc_cascade_get(void* h, uint32_t l, uint32_t* edges, uint32_t* parent_map) {
  const Level& L = ((Cascade*)h)->levels[l];
  if (edges && !L.edges.empty()) std::memcpy(edges, L.edges.data(), 4 * L.edges.size());
  if (parent_map && !L.parent_map.empty()) std::memcpy(parent_map, L.parent_map.data(), 4 * L.parent_map.size());
}

void orc_cascade_free(void* h) { delete (Cascade*)h; }

// prolong (coarsen.rs:157-183) with its xorshift jitter stream.
void orc_prolong(const float* parent_positions, const uint32_t* parent_map, uint32_t n_child, float jitter,
                 uint32_t seed, float* out) {
  uint64_t s = (uint64_t)seed + 0x9E3779B97F4A7C15ull;
  auto next = [&]() -> float {
    s ^= s >> 12;
    s ^= s << 25;
    s ^= s >> 27;
    const uint64_t v = s * 0x2545F4914F6CDD1Dull;
    return (float)((double)(v >> 11) / (double)(1ull << 53)) * 2.0f - 1.0f;
  };
  for (uint32_t i = 0; i < n_child; ++i) {
    const size_t base = 3 * (size_t)parent_map[i];
    out[3 * (size_t)i] = parent_positions[base] + next() * jitter;
    out[3 * (size_t)i + 1] = parent_positions[base + 1] + next() * jitter;
    out[3 * (size_t)i + 2] = parent_positions[base + 2] + next() * jitter;
  }
}

// fold_up (multilevel.rs:480-510): the coarsest level's positions as the
// mean of each super-node's children, level by level.
void orc_fold_up(void* h, const float* fine, float* out_coarsest) {
  const Cascade& c = *(Cascade*)h;
  std::vector<float> cur(fine, fine + 3 * (size_t)c.levels[0].n);
  for (size_t l = 1; l < c.levels.size(); ++l) {
    const std::vector<uint32_t>& pm = c.levels[l].parent_map;
    const uint32_t cn = c.levels[l].n;
    std::vector<float> sums(3 * (size_t)cn, 0.0f);
    std::vector<uint32_t> counts(cn, 0);
    for (size_t child = 0; child < pm.size(); ++child) {
      const uint32_t p = pm[child];
      if (p >= cn || child * 3 + 2 >= cur.size()) continue;
      sums[3 * (size_t)p] += cur[child * 3];
      sums[3 * (size_t)p + 1] += cur[child * 3 + 1];
      sums[3 * (size_t)p + 2] += cur[child * 3 + 2];
      counts[p] += 1;
    }
    for (uint32_t p = 0; p < cn; ++p) {
      const float cc = (float)(counts[p] > 1 ? counts[p] : 1);
      sums[3 * (size_t)p] /= cc;
      sums[3 * (size_t)p + 1] /= cc;
      sums[3 * (size_t)p + 2] /= cc;
    }
    cur.swap(sums);
  }
  std::memcpy(out_coarsest, cur.data(), 4 * cur.size());
}

// level_csr (multilevel.rs:259-294): symmetric CSR from a flat edge list,
// rows filled in edge order. offsets: n+1; neighbors: capacity 2 * edges.
uint64_t orc_level_csr(uint32_t n, const uint32_t* edges, uint64_t n_words, uint32_t* offsets, uint32_t* neighbors) {
  std::vector<uint32_t> degree(n, 0);
  for (uint64_t i = 0; i + 1 < n_words; i += 2) {
    const uint32_t s = edges[i], t = edges[i + 1];
    if (s < n && t < n && s != t) {
      degree[s] += 1;
      degree[t] += 1;
    }
  }
  uint32_t acc = 0;
  for (uint32_t v = 0; v < n; ++v) {
    offsets[v] = acc;
    acc += degree[v];
  }
  offsets[n] = acc;
  std::vector<uint32_t> cursor(offsets, offsets + n + 1);
  for (uint64_t j = 0; j + 1 < n_words; j += 2) {
    const uint32_t s = edges[j], t = edges[j + 1];
    if (s < n && t < n && s != t) {
      neighbors[cursor[s]++] = t;
      neighbors[cursor[t]++] = s;
    }
  }
  return acc;
}

// SweepSchedule::sweeps_for_level (multilevel.rs:104-120); schedule 0
// uniform, 1 linear, 2 geometric.
uint32_t orc_sweeps_for_level(uint32_t schedule, uint64_t level, uint32_t base) {
  if (base < 1) base = 1;
  uint64_t s;
  if (schedule == 0) {
    s = base;
  } else if (schedule == 1) {
    s = (uint64_t)base * (1 + level);
  } else {
    const uint64_t shift = level < 16 ? level : 16;
    s = (uint64_t)base << shift;
  }
  if (s > 0xFFFFFFFFull) s = 0xFFFFFFFFull;
  return (uint32_t)(s < 1 ? 1 : s);
}

}  // extern "C"
