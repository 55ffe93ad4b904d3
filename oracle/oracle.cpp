// CPU oracle for the jump-cannon layout step — TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++, the arithmetic of the reference's own
// layout-step code so the CUDA engine can be checked against it. It is never
// linked into the product library; only tests/, the smoke check and the CPU
// baseline leg of bench.py load it (as liboracle.so through ctypes).
//
// What it restates (paths relative to the jump-cannon repository):
//   * crates/graph-compute/src/engines/fa2_bh.rs
//       - init data prep (CSR -> v<u edge list, degrees, mass = deg+1)  :246-294
//       - OctreeBuild::rebuild / insert_body / aggregate_com_postorder /
//         assign_ropes                                                   :761-1045
//       - walk_repulsion (the reference's own CPU replica of the walk)  :1096-1147
//   * crates/graph-compute/src/shaders/fa2_barnes_hut.wgsl
//       - fa2_force (walk, attraction, gravity, swing/traction)          :96-198
//       - fa2_apply                                                      :203-226
//   * crates/graph-compute/src/shaders/force_atlas2.wgsl (brute force)   :69-165
//   * crates/graph-compute/src/engines/fa2_speed.rs AdaptiveSpeed::update :48-100
//   * crates/graph-compute/src/engines/sgd_stress.rs
//       - SplitMix64 :104-125, select_pivots :143-175, step :275-318,
//         anneal_eta :324-334, sgd_pair_update :340-366, bfs_distances :372-394
//   * crates/graph-compute/src/shaders/sgd_stress.wgsl sgd_step :34-62 and
//     crates/graph-compute/src/engines/sgd_stress_gpu.rs init/step :188-218, :368-428
//   * crates/graph-layouts/src/metrics.rs :17-164
//
// Floating-point conventions (they are what the parity tests pin):
//   * every f32 expression is evaluated left to right exactly as written in
//     the WGSL / Rust source, one IEEE-rounded operation at a time (this file
//     is compiled with -ffp-contract=off, so no fused multiply-add);
//   * length(v) and dot(v, v) are ((x*x + y*y) + z*z), the order the
//     reference's CPU walk replica uses (fa2_bh.rs:1123);
//   * WGSL max/min on f32 are fmaxf/fminf (the non-NaN operand wins), which is
//     also Rust's f32::max/min.
//
// Parity status: the reference is Rust + WGSL and cannot be compiled or run in
// this environment (no Rust toolchain, no graphics stack), so this restatement
// is pinned against the reference's own known-answer tests, restated in
// tests/test_oracle.py (theta=0 walk == brute force at n=16, leaf mass sum,
// the adaptive-speed state-machine tests, BFS on a path, SGD stress decrease,
// metric identities) and against the literal O(n*m) edge scan of the shader.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr uint32_t OCT_END = 0xFFFFFFFFu;
constexpr uint32_t OCT_BODY_INTERNAL = 0xFFFFFFFFu;

struct Fa2Settings {  // fa2_bh.rs:84-119 (Fa2BhSettings); brute ignores theta
  float gravity;
  int32_t strong_gravity;
  float scaling_ratio;
  float edge_weight_influence;
  float jitter_tolerance;
  int32_t lin_log_mode;
  int32_t prevent_overlap;
  float time_step;
  float theta;
  float max_displacement;
};

inline float len3(float x, float y, float z) { return std::sqrt(x * x + y * y + z * z); }

// ---------------------------------------------------------------- octree --
// fa2_bh.rs:739-745 OctNodeRaw: pos_size, com_mass, meta (u32 x4).
struct OctNode {
  float pos_size[4];
  float com_mass[4];
  uint32_t meta[4];
};

struct Children { uint32_t c[8]; };

// OctreeBuild, fa2_bh.rs:747-1045.
struct Octree {
  std::vector<OctNode> nodes;
  std::vector<Children> children;

  uint32_t push_internal(const float c[3], float h) {  // fa2_bh.rs:829-838
    uint32_t idx = (uint32_t)nodes.size();
    OctNode nd;
    nd.pos_size[0] = c[0]; nd.pos_size[1] = c[1]; nd.pos_size[2] = c[2]; nd.pos_size[3] = h;
    nd.com_mass[0] = nd.com_mass[1] = nd.com_mass[2] = nd.com_mass[3] = 0.0f;
    nd.meta[0] = OCT_BODY_INTERNAL; nd.meta[1] = OCT_END; nd.meta[2] = OCT_END; nd.meta[3] = 0;
    nodes.push_back(nd);
    Children ch; for (int k = 0; k < 8; ++k) ch.c[k] = OCT_END;
    children.push_back(ch);
    return idx;
  }

  static uint32_t octant_for(const float center[4], const float p[3]) {  // :841-853
    uint32_t o = 0;
    if (p[0] >= center[0]) o |= 1;
    if (p[1] >= center[1]) o |= 2;
    if (p[2] >= center[2]) o |= 4;
    return o;
  }

  static void child_center(const float pc[4], uint32_t oct, float cc[3], float* hh) {  // :855-861
    float h = pc[3] * 0.5f;
    cc[0] = pc[0] + ((oct & 1) ? h : -h);
    cc[1] = pc[1] + ((oct & 2) ? h : -h);
    cc[2] = pc[2] + ((oct & 4) ? h : -h);
    *hh = h;
  }

  // :863-923. Returns false on capacity overflow (Err(())).
  bool insert_body(uint32_t root, const float p[3], uint32_t body_idx, float body_mass,
                   uint32_t max_nodes) {
    uint32_t node_idx = root;
    for (int depth = 0; depth < 32; ++depth) {
      float center[4];
      std::memcpy(center, nodes[node_idx].pos_size, sizeof(center));
      uint32_t oct = octant_for(center, p);
      uint32_t child_idx = children[node_idx].c[oct];
      if (child_idx == OCT_END) {
        if ((uint32_t)nodes.size() >= max_nodes) return false;
        float cc[3], hh;
        child_center(center, oct, cc, &hh);
        uint32_t new_idx = (uint32_t)nodes.size();
        OctNode nd;
        nd.pos_size[0] = cc[0]; nd.pos_size[1] = cc[1]; nd.pos_size[2] = cc[2]; nd.pos_size[3] = hh;
        nd.com_mass[0] = p[0]; nd.com_mass[1] = p[1]; nd.com_mass[2] = p[2]; nd.com_mass[3] = body_mass;
        nd.meta[0] = body_idx; nd.meta[1] = OCT_END; nd.meta[2] = OCT_END; nd.meta[3] = 0;
        nodes.push_back(nd);
        Children ch; for (int k = 0; k < 8; ++k) ch.c[k] = OCT_END;
        children.push_back(ch);
        children[node_idx].c[oct] = new_idx;
        nodes[node_idx].meta[3] += 1;
        return true;
      }
      if (nodes[child_idx].meta[0] == OCT_BODY_INTERNAL) {
        node_idx = child_idx;
        continue;
      }
      float prev_com[4];
      std::memcpy(prev_com, nodes[child_idx].com_mass, sizeof(prev_com));
      uint32_t prev_body = nodes[child_idx].meta[0];
      nodes[child_idx].com_mass[0] = nodes[child_idx].com_mass[1] = 0.0f;
      nodes[child_idx].com_mass[2] = nodes[child_idx].com_mass[3] = 0.0f;
      nodes[child_idx].meta[0] = OCT_BODY_INTERNAL;
      nodes[child_idx].meta[3] = 0;
      float pp[3] = {prev_com[0], prev_com[1], prev_com[2]};
      if (!insert_body(child_idx, pp, prev_body, std::fmax(prev_com[3], 1e-3f), max_nodes))
        return false;
      node_idx = child_idx;
    }
    return true;
  }

  void aggregate_com_postorder() {  // :927-967
    if (nodes.empty()) return;
    std::vector<std::pair<uint32_t, uint32_t>> stack;
    stack.reserve(64);
    stack.push_back({0, 0});
    while (!stack.empty()) {
      uint32_t idx = stack.back().first, cursor = stack.back().second;
      if (nodes[idx].meta[0] != OCT_BODY_INTERNAL) { stack.pop_back(); continue; }
      if (cursor < 8) {
        stack.back().second = cursor + 1;
        uint32_t ch = children[idx].c[cursor];
        if (ch != OCT_END) stack.push_back({ch, 0});
        continue;
      }
      float total = 0.0f, com[3] = {0.0f, 0.0f, 0.0f};
      for (int k = 0; k < 8; ++k) {
        uint32_t ch = children[idx].c[k];
        if (ch == OCT_END) continue;
        const float* cm = nodes[ch].com_mass;
        total += cm[3];
        com[0] += cm[0] * cm[3];
        com[1] += cm[1] * cm[3];
        com[2] += cm[2] * cm[3];
      }
      if (total > 0.0f) { com[0] /= total; com[1] /= total; com[2] /= total; }
      nodes[idx].com_mass[0] = com[0]; nodes[idx].com_mass[1] = com[1];
      nodes[idx].com_mass[2] = com[2]; nodes[idx].com_mass[3] = total;
      stack.pop_back();
    }
  }

  void assign_ropes() {  // :971-1045
    if (nodes.empty()) return;
    struct Frame { uint32_t left[8]; uint32_t outer_skip; };
    size_t n = nodes.size();
    std::vector<uint32_t> skip(n, OCT_END), next(n, OCT_END);
    std::vector<Frame> stack;
    stack.reserve(64);
    Frame f0;
    for (int k = 0; k < 8; ++k)
      f0.left[k] = nodes[0].meta[0] == OCT_BODY_INTERNAL ? children[0].c[k] : OCT_END;
    f0.outer_skip = OCT_END;
    stack.push_back(f0);
    bool have_prev = true;
    uint32_t prev_visited = 0;
    while (!stack.empty()) {
      Frame& top = stack.back();
      uint32_t next_child = OCT_END;
      for (int k = 0; k < 8; ++k) {
        if (top.left[k] != OCT_END) { next_child = top.left[k]; top.left[k] = OCT_END; break; }
      }
      if (next_child != OCT_END) {
        if (have_prev && next[prev_visited] == OCT_END) next[prev_visited] = next_child;
        uint32_t child_outer = top.outer_skip;
        for (int k = 0; k < 8; ++k) {
          if (top.left[k] != OCT_END) { child_outer = top.left[k]; break; }
        }
        skip[next_child] = child_outer;
        bool internal = nodes[next_child].meta[0] == OCT_BODY_INTERNAL;
        Frame fr;
        for (int k = 0; k < 8; ++k) fr.left[k] = internal ? children[next_child].c[k] : OCT_END;
        fr.outer_skip = child_outer;
        stack.push_back(fr);  // may invalidate `top`; not used afterwards
        have_prev = true;
        prev_visited = next_child;
        continue;
      }
      stack.pop_back();
    }
    skip[0] = OCT_END;
    for (size_t i = 0; i < n; ++i) { nodes[i].meta[1] = next[i]; nodes[i].meta[2] = skip[i]; }
  }

  // :761-827. positions in vec4 stride. Returns the populated node count.
  uint32_t rebuild(const float* positions, const float* mass, uint32_t n_bodies,
                   uint32_t max_nodes, uint32_t* inserted_out = nullptr) {
    nodes.clear();
    children.clear();
    if (inserted_out) *inserted_out = 0;
    if (n_bodies == 0 || max_nodes == 0) return 0;
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = 0; i < n_bodies; ++i) {
      for (int k = 0; k < 3; ++k) {
        float v = positions[(size_t)i * 4 + k];
        if (!std::isfinite(v)) continue;
        if (v < mn[k]) mn[k] = v;
        if (v > mx[k]) mx[k] = v;
      }
    }
    if (!std::isfinite(mn[0])) {
      for (int k = 0; k < 3; ++k) { mn[k] = -1.0f; mx[k] = 1.0f; }
    }
    float center[3] = {0.5f * (mn[0] + mx[0]), 0.5f * (mn[1] + mx[1]), 0.5f * (mn[2] + mx[2])};
    float half = std::fmax(std::fmax(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]) * 0.5f;
    if (!std::isfinite(half) || half <= 0.0f) half = 1.0f;
    half *= 1.05f;
    push_internal(center, half);
    uint32_t inserted = 0;
    for (uint32_t b = 0; b < n_bodies; ++b) {
      float p[3] = {positions[(size_t)b * 4], positions[(size_t)b * 4 + 1], positions[(size_t)b * 4 + 2]};
      float bm = std::fmax(mass ? mass[b] : 1.0f, 1e-3f);
      if (!(std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]))) continue;
      if (!insert_body(0, p, b, bm, max_nodes)) break;  // overflow: stop (partial tree)
      ++inserted;
    }
    if (inserted_out) *inserted_out = inserted;
    aggregate_com_postorder();
    assign_ropes();
    return (uint32_t)nodes.size();
  }
};

// fa2_bh.rs:1096-1147 (walk_repulsion) == fa2_barnes_hut.wgsl:114-156.
// Accumulates into f (the shader's running `f`).
inline void walk_repulsion(const OctNode* nodes, uint32_t n_oct, const float pos_i[3], uint32_t i,
                           float deg_i, float scaling, float theta, float f[3],
                           uint64_t* n_inter, uint64_t* n_open) {
  if (n_oct == 0) return;
  float theta2 = theta * theta;
  uint32_t idx = 0;
  uint32_t cap = std::max(n_oct * 4u, 16u);
  uint32_t walk = 0;
  for (;;) {
    if (idx == OCT_END || walk >= cap) break;
    ++walk;
    const OctNode& nd = nodes[idx];
    uint32_t body = nd.meta[0];
    float mass_n = nd.com_mass[3];
    float s = nd.pos_size[3] * 2.0f;
    float d0 = pos_i[0] - nd.com_mass[0], d1 = pos_i[1] - nd.com_mass[1], d2 = pos_i[2] - nd.com_mass[2];
    float r2 = d0 * d0 + d1 * d1 + d2 * d2;
    if (body != OCT_BODY_INTERNAL) {
      if (body != i && mass_n > 0.0f) {
        float r2c = std::fmax(r2, 1.0e-4f);
        float c = scaling * deg_i * mass_n / r2c;
        f[0] += d0 * c; f[1] += d1 * c; f[2] += d2 * c;
        if (n_inter) ++*n_inter;
      }
      idx = nd.meta[2];
      continue;
    }
    if (mass_n > 0.0f && r2 > 0.0f && (s * s) < (theta2 * r2)) {
      float r2c = std::fmax(r2, 1.0e-4f);
      float c = scaling * deg_i * mass_n / r2c;
      f[0] += d0 * c; f[1] += d1 * c; f[2] += d2 * c;
      if (n_inter) ++*n_inter;
      idx = nd.meta[2];
    } else {
      if (n_open) ++*n_open;
      idx = nd.meta[1];
    }
  }
}

// ------------------------------------------------------- FA2 engine state --
// Attraction order: fa2_barnes_hut.wgsl:160-181 scans the (v<u) edge list in
// edge-index order. For node i the touched edges come in edge-index order,
// which is reproduced by the per-node lists built in build_attraction().
struct Fa2 {
  uint32_t n = 0;
  int bh = 1;
  Fa2Settings s{};
  std::vector<float> pos;       // vec4 stride
  std::vector<float> old_force; // vec4 stride
  std::vector<float> force;     // vec4 stride
  std::vector<float> stats;     // 2 per node
  std::vector<uint32_t> degrees;
  std::vector<float> mass;
  std::vector<uint32_t> edges;  // (v,u) pairs, v<u, edge-index order (fa2_bh.rs:264-287)
  std::vector<uint32_t> att_off, att_nbr;
  float speed = 1.0f, speed_eff = 1.0f;  // fa2_speed.rs:32-39
  Octree tree;
  uint32_t n_octree = 0, n_inserted = 0;
  uint32_t tree_capacity = 0;  // 0: the reference's 2n+8 (fa2_bh.rs:344)
  uint64_t n_inter = 0, n_open = 0;

  void build_attraction() {
    uint32_t m = (uint32_t)(edges.size() / 2);
    att_off.assign((size_t)n + 1, 0);
    for (uint32_t e = 0; e < m; ++e) { att_off[edges[2 * e] + 1]++; att_off[edges[2 * e + 1] + 1]++; }
    for (uint32_t i = 0; i < n; ++i) att_off[i + 1] += att_off[i];
    att_nbr.assign(att_off[n], 0);
    std::vector<uint32_t> cur(att_off.begin(), att_off.end() - 1);
    for (uint32_t e = 0; e < m; ++e) {
      uint32_t v = edges[2 * e], u = edges[2 * e + 1];
      att_nbr[cur[v]++] = u;
      att_nbr[cur[u]++] = v;
    }
  }
};

// fa2_speed.rs:48-100
float adaptive_update(float* speed, float* speed_eff, uint32_t n_nodes, float jitter_tolerance,
                      const float* stats, size_t n_pairs) {
  double ts = 0.0, tt = 0.0;
  for (size_t k = 0; k < n_pairs; ++k) {
    float swg = stats[2 * k], tra = stats[2 * k + 1];
    if (std::isfinite(swg) && std::isfinite(tra)) { ts += (double)swg; tt += (double)tra; }
  }
  if (!(ts > 0.0) || !(tt > 0.0) || n_nodes == 0) return *speed;
  double n = (double)n_nodes;
  double jt_tol = (double)jitter_tolerance;
  double est = 0.05 * std::sqrt(n);
  double min_jt = std::sqrt(est);
  double max_jt = 10.0;
  double jt = jt_tol * std::fmax(min_jt, std::fmin(max_jt, est * tt / (n * n)));
  const float min_eff = 0.05f;
  if (ts / tt > 2.0) {
    if (*speed_eff > min_eff) *speed_eff *= 0.5f;
    jt = std::fmax(jt, jt_tol);
  }
  double target = jt * (double)*speed_eff * tt / ts;
  if (ts > jt * tt) {
    if (*speed_eff > min_eff) *speed_eff *= 0.7f;
  } else if (*speed < 1000.0f) {
    *speed_eff *= 1.3f;
  }
  double sp = (double)*speed;
  *speed = (float)(sp + std::fmin(target - sp, 0.5 * sp));
  return *speed;
}

// fa2_barnes_hut.wgsl:96-198 (bh=1) / force_atlas2.wgsl:69-136 (bh=0) for one node.
void force_node(const Fa2& st, uint32_t i, uint64_t* n_inter, uint64_t* n_open) {
  const float* p4 = &st.pos[(size_t)i * 4];
  float pos_i[3] = {p4[0], p4[1], p4[2]};
  float deg_i = (float)st.degrees[i] + 1.0f;
  float f[3] = {0.0f, 0.0f, 0.0f};
  if (st.bh) {
    if (st.n_octree > 0)
      walk_repulsion(st.tree.nodes.data(), st.n_octree, pos_i, i, deg_i, st.s.scaling_ratio,
                     st.s.theta, f, n_inter, n_open);
  } else {
    for (uint32_t j = 0; j < st.n; ++j) {
      if (j == i) continue;
      const float* q = &st.pos[(size_t)j * 4];
      float d0 = pos_i[0] - q[0], d1 = pos_i[1] - q[1], d2 = pos_i[2] - q[2];
      float r2 = std::fmax(d0 * d0 + d1 * d1 + d2 * d2, 1.0e-4f);
      float deg_j = (float)st.degrees[j] + 1.0f;
      float coeff = st.s.scaling_ratio * deg_i * deg_j / r2;
      f[0] += d0 * coeff; f[1] += d1 * coeff; f[2] += d2 * coeff;
    }
  }
  float ewi = st.s.edge_weight_influence;
  for (uint32_t k = st.att_off[i]; k < st.att_off[i + 1]; ++k) {
    const float* q = &st.pos[(size_t)st.att_nbr[k] * 4];
    float d0 = q[0] - pos_i[0], d1 = q[1] - pos_i[1], d2 = q[2] - pos_i[2];
    float r = std::fmax(len3(d0, d1, d2), 1.0e-3f);
    float w = std::pow(std::fmax(1.0f, 1.0e-6f), ewi);  // every edge weight is 1.0 (fa2_bh.rs:279)
    float att = w;
    if (st.s.lin_log_mode) att = w * std::log(1.0f + r) / r;
    f[0] += d0 * att; f[1] += d1 * att; f[2] += d2 * att;
  }
  float r0 = std::fmax(len3(pos_i[0], pos_i[1], pos_i[2]), 1.0e-3f);
  float gd = st.s.gravity * deg_i;
  if (st.s.strong_gravity) {
    f[0] -= pos_i[0] * gd; f[1] -= pos_i[1] * gd; f[2] -= pos_i[2] * gd;
  } else {
    f[0] -= (pos_i[0] / r0) * gd; f[1] -= (pos_i[1] / r0) * gd; f[2] -= (pos_i[2] / r0) * gd;
  }
  const float* o = &st.old_force[(size_t)i * 4];
  float* fo = const_cast<float*>(&st.force[(size_t)i * 4]);
  fo[0] = f[0]; fo[1] = f[1]; fo[2] = f[2]; fo[3] = 0.0f;
  float* so = const_cast<float*>(&st.stats[(size_t)i * 2]);
  so[0] = deg_i * len3(o[0] - f[0], o[1] - f[1], o[2] - f[2]);
  so[1] = deg_i * 0.5f * len3(o[0] + f[0], o[1] + f[1], o[2] + f[2]);
}

void force_pass(Fa2& st, int threads) {
  if (st.bh) {
    uint32_t cap = st.tree_capacity ? st.tree_capacity : 2 * st.n + 8;
    st.n_octree = st.tree.rebuild(st.pos.data(), st.mass.data(), st.n, cap, &st.n_inserted);
  }
  uint64_t ni = 0, no = 0;
#ifdef _OPENMP
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads) reduction(+ : ni, no)
#endif
  for (int64_t i = 0; i < (int64_t)st.n; ++i) force_node(st, (uint32_t)i, &ni, &no);
  (void)threads;
  st.n_inter = ni;
  st.n_open = no;
}

// fa2_barnes_hut.wgsl:203-226
void apply_pass(Fa2& st, int threads) {
  (void)threads;
#ifdef _OPENMP
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(threads)
#endif
  for (int64_t ii = 0; ii < (int64_t)st.n; ++ii) {
    size_t i = (size_t)ii;
    float* p = &st.pos[i * 4];
    const float* f = &st.force[i * 4];
    float* o = &st.old_force[i * 4];
    float deg_i = (float)st.degrees[i] + 1.0f;
    float swinging = deg_i * len3(o[0] - f[0], o[1] - f[1], o[2] - f[2]);
    float factor = st.speed / (1.0f + std::sqrt(st.speed * swinging));
    float df = len3(f[0], f[1], f[2]);
    if (st.s.max_displacement > 0.0f && df > 1.0e-9f) factor = std::fmin(factor, st.s.max_displacement / df);
    float k = factor * st.s.time_step;
    p[0] = p[0] + f[0] * k; p[1] = p[1] + f[1] * k; p[2] = p[2] + f[2] * k; p[3] = 0.0f;
    o[0] = f[0]; o[1] = f[1]; o[2] = f[2]; o[3] = 0.0f;
  }
}

// ------------------------------------------------------------------ SGD --
struct SplitMix64 {  // sgd_stress.rs:104-125
  uint64_t state;
  uint64_t next_u64() {
    state += 0x9E3779B97F4A7C15ull;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  uint64_t below(uint64_t n) { return next_u64() % n; }
};

// sgd_stress.rs:372-394
void bfs(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint32_t src, uint32_t* dist) {
  for (uint32_t v = 0; v < n; ++v) dist[v] = 0xFFFFFFFFu;
  if (n == 0) return;
  std::vector<uint32_t> q;
  q.reserve(n);
  dist[src] = 0;
  q.push_back(src);
  for (size_t h = 0; h < q.size(); ++h) {
    uint32_t v = q[h];
    uint32_t dv = dist[v];
    for (uint32_t e = off[v]; e < off[v + 1]; ++e) {
      uint32_t u = nbr[e];
      if (dist[u] == 0xFFFFFFFFu) { dist[u] = dv + 1; q.push_back(u); }
    }
  }
}

struct Sgd {
  uint32_t n = 0, k = 0;
  // 0 = CPU s_gd2 (sgd_stress.rs), 1 = GPU Jacobi (sgd_stress.wgsl),
  // 2 = the batched fixed-point scatter of this repository's "sgd-stress"
  // device engine (its own algorithm, restated to check the device code)
  int mode = 0;
  uint32_t scatter_batches = 0;  // mode 2: 0 = the engine's default
  uint32_t n_pivots = 50, sweeps_per_step = 1, n_anneal = 30;
  float eta_max = 1.0f, eta_min = 0.01f;
  uint64_t seed = 0x5EEDC0DE12345678ull;
  std::vector<float> pos;               // modes 0 and 2: 3n (xyz), mode 1: 4n (vec4)
  std::vector<uint32_t> pivots;         // k
  std::vector<uint32_t> dist;           // k x n, row = pivot (u32, MAX = unreachable)
  SplitMix64 rng{0};
  uint64_t sweep = 0;
};

// sgd_stress.rs:143-175
void select_pivots(Sgd& sg, const uint32_t* off, const uint32_t* nbr, SplitMix64& rng) {
  uint32_t n = sg.n;
  uint32_t k = n == 0 ? 0 : std::min(std::max(sg.n_pivots, 1u), n);
  sg.pivots.clear();
  sg.dist.clear();
  sg.k = 0;
  if (n == 0 || k == 0) return;
  std::vector<uint32_t> min_d(n, 0xFFFFFFFFu), d(n);
  uint32_t next = (uint32_t)rng.below(n);
  sg.dist.resize((size_t)k * n);
  for (uint32_t t = 0; t < k; ++t) {
    bfs(n, off, nbr, next, d.data());
    uint32_t best = next, best_d = 0;
    for (uint32_t v = 0; v < n; ++v) {
      uint32_t dv = d[v];
      if (dv != 0xFFFFFFFFu && dv < min_d[v]) min_d[v] = dv;
      uint32_t cover = min_d[v];
      if (cover != 0xFFFFFFFFu && cover > best_d) { best_d = cover; best = v; }
    }
    sg.pivots.push_back(next);
    std::memcpy(&sg.dist[(size_t)t * n], d.data(), sizeof(uint32_t) * n);
    next = best;
  }
  sg.k = k;
}

// sgd_stress.rs:324-334
float anneal_eta(uint64_t sweep, float eta_max, float eta_min, uint32_t n_anneal) {
  if (n_anneal == 0) return eta_min;
  float t = (float)sweep / (float)n_anneal;
  if (t >= 1.0f) return eta_min;
  float ratio = std::fmax(eta_min / eta_max, 1e-9f);
  return eta_max * std::pow(ratio, t);
}

// sgd_stress.rs:340-366
void sgd_pair_update(float* P, size_t i, size_t j, float d_ij, float eta) {
  float xi = P[3 * i], yi = P[3 * i + 1], zi = P[3 * i + 2];
  float xj = P[3 * j], yj = P[3 * j + 1], zj = P[3 * j + 2];
  float dx = xi - xj, dy = yi - yj, dz = zi - zj;
  float mag = std::fmax(std::sqrt(dx * dx + dy * dy + dz * dz), 1e-6f);
  float w = 1.0f / (d_ij * d_ij);
  float mu = std::fmin(w * eta, 1.0f);
  float r = 0.5f * mu * (mag - d_ij) / mag;
  float rx = r * dx, ry = r * dy, rz = r * dz;
  P[3 * i] = xi - rx; P[3 * i + 1] = yi - ry; P[3 * i + 2] = zi - rz;
  P[3 * j] = xj + rx; P[3 * j + 1] = yj + ry; P[3 * j + 2] = zj + rz;
}

// sgd_stress.wgsl:34-62, one Jacobi sweep from pos_in to pos_out (vec4 stride).
void sgd_jacobi_sweep(const Sgd& sg, const float* pin, float* pout, float eta, int threads) {
  (void)threads;
  uint32_t n = sg.n, k = sg.k;
#ifdef _OPENMP
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(threads)
#endif
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    uint32_t i = (uint32_t)ii;
    float p0 = pin[(size_t)i * 4], p1 = pin[(size_t)i * 4 + 1], p2 = pin[(size_t)i * 4 + 2];
    for (uint32_t t = 0; t < k; ++t) {
      uint32_t j = sg.pivots[t];
      if (j == i) continue;
      uint32_t du = sg.dist[(size_t)t * n + i];
      float d = (du == 0xFFFFFFFFu || du == 0) ? 0.0f : (float)du;  // sgd_stress_gpu.rs:203-207
      if (d <= 0.0f) continue;
      const float* q = &pin[(size_t)j * 4];
      float e0 = p0 - q[0], e1 = p1 - q[1], e2 = p2 - q[2];
      float mag = std::fmax(std::sqrt(e0 * e0 + e1 * e1 + e2 * e2), 1e-6f);
      float w = 1.0f / (d * d);
      float mu = std::fmin(1.0f, w * eta);
      float r = mu * (mag - d) / mag;
      p0 = p0 - r * e0; p1 = p1 - r * e1; p2 = p2 - r * e2;
    }
    pout[(size_t)i * 4] = p0; pout[(size_t)i * 4 + 1] = p1; pout[(size_t)i * 4 + 2] = p2;
    pout[(size_t)i * 4 + 3] = 0.0f;
  }
}

double euclid(const float* P, size_t i, size_t j) {  // metrics.rs:19-24
  double dx = (double)(P[3 * i] - P[3 * j]);
  double dy = (double)(P[3 * i + 1] - P[3 * j + 1]);
  double dz = (double)(P[3 * i + 2] - P[3 * j + 2]);
  return std::sqrt(dx * dx + dy * dy + dz * dz);
}

}  // namespace

// =================================================================== C ABI ==
extern "C" {

// --- octree (reference layout: 12 x 32-bit words per node) ---------------
// Returns the populated node count; writes up to cap_nodes nodes and the
// number of bodies inserted before any overflow.
uint32_t orc_octree_build(uint32_t n, const float* pos4, const float* mass, uint32_t max_nodes,
                          void* nodes_out, uint32_t cap_nodes, uint32_t* inserted) {
  Octree t;
  uint32_t used = t.rebuild(pos4, mass, n, max_nodes, inserted);
  if (nodes_out) std::memcpy(nodes_out, t.nodes.data(), sizeof(OctNode) * std::min(used, cap_nodes));
  return used;
}

// Walk every body against a tree in the reference layout (theta criterion).
void orc_octree_walk_all(const void* nodes, uint32_t n_oct, uint32_t n, const float* pos4,
                         const float* deg_plus1, float scaling, float theta, float* f_out3) {
  const OctNode* nd = (const OctNode*)nodes;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    uint32_t i = (uint32_t)ii;
    float p[3] = {pos4[(size_t)i * 4], pos4[(size_t)i * 4 + 1], pos4[(size_t)i * 4 + 2]};
    float f[3] = {0.0f, 0.0f, 0.0f};
    walk_repulsion(nd, n_oct, p, i, deg_plus1[i], scaling, theta, f, nullptr, nullptr);
    f_out3[(size_t)i * 3] = f[0]; f_out3[(size_t)i * 3 + 1] = f[1]; f_out3[(size_t)i * 3 + 2] = f[2];
  }
}

// --- FA2 engine (bh = 1: fa2-bh, bh = 0: fa2-brute) -----------------------
void* orc_fa2_create(uint32_t n, const uint32_t* offsets, const uint32_t* nbrs,
                     const float* pos_xyz, const void* settings, int bh) {
  Fa2* st = new Fa2();
  st->n = n;
  st->bh = bh;
  std::memcpy(&st->s, settings, sizeof(Fa2Settings));
  if (st->s.theta < 0.0f) st->s.theta = 0.0f;  // fa2_bh.rs:716 theta.max(0)
  st->pos.assign((size_t)n * 4, 0.0f);
  for (uint32_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) st->pos[(size_t)i * 4 + k] = pos_xyz[(size_t)i * 3 + k];
  st->old_force.assign((size_t)n * 4, 0.0f);
  st->force.assign((size_t)n * 4, 0.0f);
  st->stats.assign((size_t)n * 2, 0.0f);
  st->degrees.assign(n, 0);
  for (uint32_t v = 0; v < n; ++v) {
    for (uint32_t e = offsets[v]; e < offsets[v + 1]; ++e) {
      uint32_t u = nbrs[e];
      if (u == v) continue;
      st->degrees[v] += 1;
      if (v < u) { st->edges.push_back(v); st->edges.push_back(u); }
    }
  }
  st->mass.resize(n);
  for (uint32_t i = 0; i < n; ++i) st->mass[i] = (float)st->degrees[i] + 1.0f;
  st->build_attraction();
  return st;
}

void orc_fa2_destroy(void* h) { delete (Fa2*)h; }

// Test hook: build the octree with a larger capacity than the reference's
// 2n+8, to compare against an engine that grows its tree instead of
// truncating it. 0 restores 2n+8.
void orc_fa2_set_tree_capacity(void* h, uint32_t cap) { ((Fa2*)h)->tree_capacity = cap; }

// One full engine step: (tree build), force pass, host speed reduction, apply.
void orc_fa2_step(void* h, int threads) {
  Fa2& st = *(Fa2*)h;
  if (st.n == 0) return;
  force_pass(st, threads);
  adaptive_update(&st.speed, &st.speed_eff, st.n, st.s.jitter_tolerance, st.stats.data(), st.n);
  apply_pass(st, threads);
}

// Force pass only (tree build + fa2_force) at the current state.
void orc_fa2_force_pass(void* h, int threads) { force_pass(*(Fa2*)h, threads); }

void orc_fa2_get(void* h, float* pos_xyz, float* force_xyz, float* old_force_xyz, float* stats2,
                 float* speed2, uint32_t* info4) {
  Fa2& st = *(Fa2*)h;
  for (uint32_t i = 0; i < st.n; ++i)
    for (int k = 0; k < 3; ++k) {
      if (pos_xyz) pos_xyz[(size_t)i * 3 + k] = st.pos[(size_t)i * 4 + k];
      if (force_xyz) force_xyz[(size_t)i * 3 + k] = st.force[(size_t)i * 4 + k];
      if (old_force_xyz) old_force_xyz[(size_t)i * 3 + k] = st.old_force[(size_t)i * 4 + k];
    }
  if (stats2) std::memcpy(stats2, st.stats.data(), sizeof(float) * 2 * st.n);
  if (speed2) { speed2[0] = st.speed; speed2[1] = st.speed_eff; }
  if (info4) {
    info4[0] = st.n_octree; info4[1] = st.n_inserted;
    info4[2] = (uint32_t)std::min<uint64_t>(st.n_inter, 0xFFFFFFFFull);
    info4[3] = (uint32_t)std::min<uint64_t>(st.n_open, 0xFFFFFFFFull);
  }
}

void orc_fa2_counts(void* h, uint64_t* inter_open2) {
  Fa2& st = *(Fa2*)h;
  inter_open2[0] = st.n_inter;
  inter_open2[1] = st.n_open;
}

void orc_fa2_set_state(void* h, const float* pos_xyz, const float* old_force_xyz, float speed,
                       float speed_eff) {
  Fa2& st = *(Fa2*)h;
  for (uint32_t i = 0; i < st.n; ++i)
    for (int k = 0; k < 3; ++k) {
      if (pos_xyz) st.pos[(size_t)i * 4 + k] = pos_xyz[(size_t)i * 3 + k];
      if (old_force_xyz) st.old_force[(size_t)i * 4 + k] = old_force_xyz[(size_t)i * 3 + k];
    }
  st.speed = speed;
  st.speed_eff = speed_eff;
}

// The per-node attraction lists the oracle derived (for checks of ordering).
uint64_t orc_fa2_attraction(void* h, uint32_t* off_out, uint32_t* nbr_out) {
  Fa2& st = *(Fa2*)h;
  if (off_out) std::memcpy(off_out, st.att_off.data(), sizeof(uint32_t) * (st.n + 1));
  if (nbr_out) std::memcpy(nbr_out, st.att_nbr.data(), sizeof(uint32_t) * st.att_nbr.size());
  return st.att_nbr.size();
}

// Literal restatement of the shader's O(n*m) edge scan (fa2_barnes_hut.wgsl:160-181)
// for node i, accumulated onto f3 — small-graph cross-check of the list order.
void orc_fa2_attraction_scan(void* h, uint32_t i, float* f3) {
  Fa2& st = *(Fa2*)h;
  const float* pi = &st.pos[(size_t)i * 4];
  uint32_t m = (uint32_t)(st.edges.size() / 2);
  for (uint32_t e = 0; e < m; ++e) {
    uint32_t x = st.edges[2 * e], y = st.edges[2 * e + 1], other;
    if (x == i) other = y; else if (y == i) other = x; else continue;
    const float* q = &st.pos[(size_t)other * 4];
    float d0 = q[0] - pi[0], d1 = q[1] - pi[1], d2 = q[2] - pi[2];
    float r = std::fmax(len3(d0, d1, d2), 1.0e-3f);
    float w = std::pow(std::fmax(1.0f, 1.0e-6f), st.s.edge_weight_influence);
    float att = w;
    if (st.s.lin_log_mode) att = w * std::log(1.0f + r) / r;
    f3[0] += d0 * att; f3[1] += d1 * att; f3[2] += d2 * att;
  }
}

// Exact FA2 force in FP64: all-pairs repulsion, the same attraction list and
// gravity, evaluated in double. Quantifies the Barnes-Hut error of both sides.
void orc_fa2_exact_forces_f64(void* h, double* f_out3) {
  Fa2& st = *(Fa2*)h;
  uint32_t n = st.n;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    uint32_t i = (uint32_t)ii;
    const float* pf = &st.pos[(size_t)i * 4];
    double p[3] = {pf[0], pf[1], pf[2]};
    double deg_i = (double)st.degrees[i] + 1.0;
    double f[3] = {0, 0, 0};
    for (uint32_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const float* q = &st.pos[(size_t)j * 4];
      double d[3] = {p[0] - q[0], p[1] - q[1], p[2] - q[2]};
      double r2 = std::fmax(d[0] * d[0] + d[1] * d[1] + d[2] * d[2], 1.0e-4);
      double c = (double)st.s.scaling_ratio * deg_i * ((double)st.degrees[j] + 1.0) / r2;
      for (int k = 0; k < 3; ++k) f[k] += d[k] * c;
    }
    for (uint32_t e = st.att_off[i]; e < st.att_off[i + 1]; ++e) {
      const float* q = &st.pos[(size_t)st.att_nbr[e] * 4];
      double d[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
      double att = 1.0;
      if (st.s.lin_log_mode) {
        double r = std::fmax(std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), 1.0e-3);
        att = std::log(1.0 + r) / r;
      }
      for (int k = 0; k < 3; ++k) f[k] += d[k] * att;
    }
    double r0 = std::fmax(std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]), 1.0e-3);
    double gd = (double)st.s.gravity * deg_i;
    for (int k = 0; k < 3; ++k) f[k] -= st.s.strong_gravity ? p[k] * gd : (p[k] / r0) * gd;
    for (int k = 0; k < 3; ++k) f_out3[(size_t)i * 3 + k] = f[k];
  }
}

float orc_adaptive_speed_update(float* speed, float* speed_eff, uint32_t n_nodes,
                                float jitter_tolerance, const float* stats, uint64_t n_pairs) {
  return adaptive_update(speed, speed_eff, n_nodes, jitter_tolerance, stats, (size_t)n_pairs);
}

// --- SGD ---------------------------------------------------------------
// The batched scatter of the device "sgd-stress" engine (csrc/jc_sgd.cu,
// k_pairs / k_pairs_apply; no counterpart in the reference, whose CPU engine
// moves the pairs one after another). Sample q of the run is the reference's
// q-th (node, pivot) draw of the SplitMix64 stream that follows the pivot
// choice (outputs 2q and 2q + 1). A sweep's n samples are cut into batches of
// ceil(n / batches); inside a batch every pair update is computed from the
// batch-start positions with the reference's f32 operations, and its two
// endpoint moves are added as 64-bit fixed point (x 2^32, rounded to nearest
// even); then every node moves by the mean of its moves.
void sgd_scatter_sweeps(Sgd& sg, uint32_t sweeps) {
  const uint32_t n = sg.n, k = sg.k;
  uint32_t batches = sg.scatter_batches ? sg.scatter_batches : (n + std::max(256u, (n + 63) / 64) - 1) /
                                                                      std::max(256u, (n + 63) / 64);
  batches = std::max(1u, std::min(batches, n));
  const uint32_t per = (n + batches - 1) / batches;
  const uint64_t s0 = sg.rng.state, G = 0x9E3779B97F4A7C15ull;
  const double FIX = 4294967296.0;
  auto mix = [](uint64_t z) {  // SplitMix64 output for a given stream position
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  std::vector<int64_t> acc((size_t)3 * n);
  std::vector<uint32_t> cnt(n);
  float* P = sg.pos.data();
  for (uint32_t s = 0; s < sweeps; ++s) {
    const float eta = anneal_eta(sg.sweep, sg.eta_max, sg.eta_min, sg.n_anneal);
    for (uint32_t q0 = 0; q0 < n; q0 += per) {
      const uint32_t c = std::min(per, n - q0);
      std::fill(acc.begin(), acc.end(), 0);
      std::fill(cnt.begin(), cnt.end(), 0u);
      for (uint32_t t = 0; t < c; ++t) {
        const uint64_t q = sg.sweep * n + q0 + t;
        const size_t i = (size_t)(mix(s0 + (2 * q + 1) * G) % n);
        const size_t pidx = (size_t)(mix(s0 + (2 * q + 2) * G) % k);
        const size_t j = sg.pivots[pidx];
        if (i == j) continue;
        const uint32_t du = sg.dist[pidx * n + i];
        if (du == 0xFFFFFFFFu || du == 0) continue;
        const float d = (float)du;
        const float dx = P[3 * i] - P[3 * j], dy = P[3 * i + 1] - P[3 * j + 1], dz = P[3 * i + 2] - P[3 * j + 2];
        const float mag = std::fmax(std::sqrt(dx * dx + dy * dy + dz * dz), 1e-6f);
        const float w = 1.0f / (d * d);
        const float mu = std::fmin(w * eta, 1.0f);
        const float r = 0.5f * mu * (mag - d) / mag;
        const int64_t f[3] = {std::llrint((double)(r * dx) * FIX), std::llrint((double)(r * dy) * FIX),
                              std::llrint((double)(r * dz) * FIX)};
        for (int a = 0; a < 3; ++a) {
          acc[3 * i + a] -= f[a];
          acc[3 * j + a] += f[a];
        }
        cnt[i] += 1;
        cnt[j] += 1;
      }
      for (uint32_t v = 0; v < n; ++v) {
        if (cnt[v] == 0) continue;
        const double inv = 1.0 / (FIX * (double)cnt[v]);
        for (int a = 0; a < 3; ++a) P[3 * (size_t)v + a] = P[3 * (size_t)v + a] + (float)((double)acc[3 * (size_t)v + a] * inv);
      }
    }
    sg.sweep += 1;
  }
}

void orc_bfs(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint32_t src, uint32_t* dist) {
  bfs(n, off, nbr, src, dist);
}

// mode 0: CPU s_gd2 engine, mode 1: GPU Jacobi engine. settings: n_pivots,
// sweeps_per_step, n_anneal_steps (u32) then eta_max, eta_min (f32), seed (u64).
void* orc_sgd_create(uint32_t n, const uint32_t* off, const uint32_t* nbr, const float* pos_xyz,
                     uint32_t n_pivots, uint32_t sweeps_per_step, float eta_max, float eta_min,
                     uint32_t n_anneal, uint64_t seed, int mode) {
  Sgd* sg = new Sgd();
  sg->n = n; sg->mode = mode; sg->n_pivots = n_pivots; sg->sweeps_per_step = sweeps_per_step;
  sg->eta_max = eta_max; sg->eta_min = eta_min; sg->n_anneal = n_anneal; sg->seed = seed;
  SplitMix64 rng{seed};
  select_pivots(*sg, off, nbr, rng);
  sg->rng = rng;  // the CPU engine keeps using the same stream (sgd_stress.rs:262-271)
  if (mode != 1) {
    sg->pos.assign(pos_xyz, pos_xyz + (size_t)3 * n);
  } else {
    sg->pos.assign((size_t)4 * std::max(n, 1u), 0.0f);
    for (uint32_t i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) sg->pos[(size_t)4 * i + c] = pos_xyz[(size_t)3 * i + c];
  }
  return sg;
}

void orc_sgd_destroy(void* h) { delete (Sgd*)h; }

uint32_t orc_sgd_pivots(void* h, uint32_t* pivots_out, uint32_t* dist_out) {
  Sgd& sg = *(Sgd*)h;
  if (pivots_out) std::memcpy(pivots_out, sg.pivots.data(), sizeof(uint32_t) * sg.k);
  if (dist_out) std::memcpy(dist_out, sg.dist.data(), sizeof(uint32_t) * sg.dist.size());
  return sg.k;
}

void orc_sgd_step(void* h, int threads) {
  Sgd& sg = *(Sgd*)h;
  uint32_t n = sg.n;
  if (n == 0 || sg.k == 0) return;
  uint32_t sweeps = std::max(sg.sweeps_per_step, 1u);
  if (sg.mode == 0) {  // sgd_stress.rs:275-318
    for (uint32_t s = 0; s < sweeps; ++s) {
      float eta = anneal_eta(sg.sweep, sg.eta_max, sg.eta_min, sg.n_anneal);
      for (uint32_t q = 0; q < n; ++q) {
        size_t i = (size_t)sg.rng.below(n);
        size_t pidx = (size_t)sg.rng.below(sg.k);
        size_t j = sg.pivots[pidx];
        if (i == j) continue;
        uint32_t d = sg.dist[pidx * n + i];
        if (d == 0xFFFFFFFFu || d == 0) continue;
        sgd_pair_update(sg.pos.data(), i, j, (float)d, eta);
      }
      sg.sweep += 1;
    }
  } else if (sg.mode == 2) {
    sgd_scatter_sweeps(sg, sweeps);
  } else {  // sgd_stress_gpu.rs:368-428: one eta per step, `sweeps` Jacobi sweeps
    float eta = anneal_eta(sg.sweep, sg.eta_max, sg.eta_min, sg.n_anneal);
    std::vector<float> tmp(sg.pos.size());
    for (uint32_t s = 0; s < sweeps; ++s) {
      sgd_jacobi_sweep(sg, sg.pos.data(), tmp.data(), eta, threads);
      sg.pos.swap(tmp);
    }
    sg.sweep += sweeps;
  }
}

void orc_sgd_set_scatter_batches(void* h, uint32_t batches) { ((Sgd*)h)->scatter_batches = batches; }

void orc_sgd_positions(void* h, float* xyz_out) {
  Sgd& sg = *(Sgd*)h;
  if (sg.mode != 1) {
    std::memcpy(xyz_out, sg.pos.data(), sizeof(float) * 3 * sg.n);
  } else {
    for (uint32_t i = 0; i < sg.n; ++i)
      for (int c = 0; c < 3; ++c) xyz_out[(size_t)3 * i + c] = sg.pos[(size_t)4 * i + c];
  }
}

void orc_sgd_set_positions(void* h, const float* xyz) {
  Sgd& sg = *(Sgd*)h;
  for (uint32_t i = 0; i < sg.n; ++i)
    for (int c = 0; c < 3; ++c) {
      if (sg.mode != 1) sg.pos[(size_t)3 * i + c] = xyz[(size_t)3 * i + c];
      else sg.pos[(size_t)4 * i + c] = xyz[(size_t)3 * i + c];
    }
}

float orc_anneal_eta(uint64_t sweep, float eta_max, float eta_min, uint32_t n_anneal) {
  return anneal_eta(sweep, eta_max, eta_min, n_anneal);
}

// --- metrics (metrics.rs) ------------------------------------------------
float orc_scale_normalized_stress(const float* P, const uint32_t* ti, const uint32_t* tj,
                                  const float* td, uint64_t count) {  // :31-59
  double num = 0, den = 0, wd2 = 0;
  for (uint64_t t = 0; t < count; ++t) {
    if (td[t] <= 0.0f) continue;
    double d = td[t], w = 1.0 / (d * d), big = euclid(P, ti[t], tj[t]);
    num += w * d * big; den += w * big * big; wd2 += w * d * d;
  }
  if (den <= 0.0 || wd2 <= 0.0) return 0.0f;
  double alpha = num / den, s = 0;
  for (uint64_t t = 0; t < count; ++t) {
    if (td[t] <= 0.0f) continue;
    double d = td[t], w = 1.0 / (d * d), r = alpha * euclid(P, ti[t], tj[t]) - d;
    s += w * r * r;
  }
  return (float)(s / wd2);
}

float orc_stress(const float* P, const uint32_t* ti, const uint32_t* tj, const float* td,
                 uint64_t count) {  // :64-76
  double s = 0;
  for (uint64_t t = 0; t < count; ++t) {
    if (td[t] <= 0.0f) continue;
    double d = td[t], w = 1.0 / (d * d), r = euclid(P, ti[t], tj[t]) - d;
    s += w * r * r;
  }
  return (float)s;
}

float orc_edge_length_cv(const float* P, const uint32_t* ei, const uint32_t* ej, uint64_t count) {
  if (count < 2) return 0.0f;  // :150-164
  std::vector<double> lens(count);
  double sum = 0;
  for (uint64_t t = 0; t < count; ++t) { lens[t] = euclid(P, ei[t], ej[t]); sum += lens[t]; }
  double mean = sum / (double)count;
  if (mean <= 1e-12) return 0.0f;
  double var = 0;
  for (uint64_t t = 0; t < count; ++t) var += (lens[t] - mean) * (lens[t] - mean);
  var /= (double)count;
  return (float)(std::sqrt(var) / mean);
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
