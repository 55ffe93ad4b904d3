// The "multilevel" wrapper engine (crates/graph-compute/src/engines/multilevel.rs):
// coarsen the graph into a cascade G_0 ... G_L by greedy matching
// (crates/graph-layouts/src/layout/coarsen.rs), lay out the coarsest level with
// the wrapped engine, prolong the positions one level finer, refine there with
// the same engine instance, and so on down to G_0, where it keeps refining.
//
// Division of work. The matching is first-touch greedy over the edge list, a
// sequential rule whose result depends on the order of the edges; it runs on
// the host once per init, exactly as the reference orders it, together with
// the contraction of each level's edges. Everything that touches positions
// runs on the device: folding the seed up the cascade (the mean of each
// super-node's one or two children), and prolongation (each child takes its
// parent's position plus the reference's xorshift jitter). The jitter stream
// is sequential by definition; it is split into chunks whose starting states
// are reached with a GF(2) jump-ahead of the xorshift map, so every device
// thread produces its own chunk of the exact sequence. The wrapped engine is
// rebound to each finer level from those device positions (reinit_device),
// and its device buffers grow once per level and are reused after that.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "jc_common.h"
#include "jc_engine.h"
#include "jc_params.h"

namespace jc {

void Engine::reinit_device(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint64_t nnz, const float* d_xyz) {
  std::vector<float> h(3ull * n);
  if (n) JC_CUDA_CHECK(cudaMemcpy(h.data(), d_xyz, 12ull * n, cudaMemcpyDeviceToHost));
  reinit(n, off, nbr, nnz, h.data());
}

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;
constexpr uint32_t JITTER_CHUNK = 256;  // jitter values per device thread

// ------------------------------------------------------------- cascade --
struct Level {
  uint32_t n = 0;
  std::vector<uint32_t> edges;       // flat [s,t, ...] after contraction
  std::vector<uint32_t> parent_map;  // previous (finer) level's node -> node here
  std::vector<uint32_t> children;    // 2 per node here: its finer-level children (NONE pads)
};

// Open-addressing set of undirected super-node pairs, first insertion wins.
class PairSet {
 public:
  explicit PairSet(size_t expect) {
    size_t cap = 16;
    while (cap < 2 * expect + 16) cap <<= 1;
    slots_.assign(cap, EMPTY);
    mask_ = cap - 1;
  }
  bool insert(uint64_t key) {
    size_t h = (size_t)((key * 0x9E3779B97F4A7C15ull) >> 17) & mask_;
    for (;;) {
      if (slots_[h] == EMPTY) {
        slots_[h] = key;
        return true;
      }
      if (slots_[h] == key) return false;
      h = (h + 1) & mask_;
    }
  }

 private:
  static constexpr uint64_t EMPTY = ~0ull;  // never a key: a < b < 2^32 - 1
  std::vector<uint64_t> slots_;
  size_t mask_;
};

// contract_one_level (coarsen.rs:96-150): first-touch greedy matching over
// the edges in order, singletons promoted after, then the contracted edges
// without self-loops and without repeats of an unordered pair, each kept at
// its first occurrence with its orientation.
Level contract(uint32_t n, const std::vector<uint32_t>& edges) {
  Level next;
  next.parent_map.assign(n, NONE);
  std::vector<uint32_t>& parent = next.parent_map;
  uint32_t next_super = 0;
  for (size_t i = 0; i + 1 < edges.size(); i += 2) {
    const uint32_t s = edges[i], t = edges[i + 1];
    if (s == t || s >= n || t >= n) continue;
    if (parent[s] == NONE && parent[t] == NONE) {
      parent[s] = parent[t] = next_super++;
    }
  }
  for (uint32_t& p : parent)
    if (p == NONE) p = next_super++;
  next.n = next_super;
  PairSet seen(edges.size() / 2);
  next.edges.reserve(edges.size() / 2);
  for (size_t j = 0; j + 1 < edges.size(); j += 2) {
    const uint32_t es = edges[j], et = edges[j + 1];
    if (es >= n || et >= n) continue;
    const uint32_t s = parent[es], t = parent[et];
    if (s == t) continue;
    const uint64_t key = s < t ? ((uint64_t)s << 32) | t : ((uint64_t)t << 32) | s;
    if (seen.insert(key)) {
      next.edges.push_back(s);
      next.edges.push_back(t);
    }
  }
  // children in increasing finer-level index (the order fold_up sums them)
  next.children.assign(2 * (size_t)next.n, NONE);
  for (uint32_t c = 0; c < n; ++c) {
    uint32_t* slot = &next.children[2 * (size_t)parent[c]];
    slot[slot[0] == NONE ? 0 : 1] = c;
  }
  return next;
}

// coarsen (coarsen.rs:52-90): stop at target_size, at max_levels, or when the
// matching stops shrinking the graph (ratio < 1.6 in f32).
std::vector<Level> coarsen(uint32_t n, std::vector<uint32_t> edges, uint64_t max_levels, uint64_t target_size) {
  std::vector<Level> levels(1);
  levels[0].n = n;
  levels[0].edges = std::move(edges);
  for (uint64_t it = 1; it < max_levels; ++it) {
    const Level& cur = levels.back();
    if (cur.n <= target_size) break;
    Level next = contract(cur.n, cur.edges);
    const float ratio = (float)cur.n / (float)std::max(next.n, 1u);
    if (ratio < 1.6f && next.n == cur.n) break;
    const uint32_t nn = next.n;
    levels.push_back(std::move(next));
    if (nn <= target_size || ratio < 1.6f) break;
  }
  return levels;
}

// level_csr (multilevel.rs:259-294): rows filled in edge order, both
// directions, self-loops and out-of-range ids skipped.
void level_csr(const Level& L, std::vector<uint32_t>* off, std::vector<uint32_t>* nbr) {
  const uint32_t n = L.n;
  off->assign((size_t)n + 1, 0);
  for (size_t i = 0; i + 1 < L.edges.size(); i += 2) {
    const uint32_t s = L.edges[i], t = L.edges[i + 1];
    if (s < n && t < n && s != t) {
      (*off)[s + 1] += 1;
      (*off)[t + 1] += 1;
    }
  }
  for (uint32_t v = 0; v < n; ++v) (*off)[v + 1] += (*off)[v];
  nbr->assign((*off)[n], 0);
  std::vector<uint32_t> cur(off->begin(), off->end() - 1);
  for (size_t j = 0; j + 1 < L.edges.size(); j += 2) {
    const uint32_t s = L.edges[j], t = L.edges[j + 1];
    if (s < n && t < n && s != t) {
      (*nbr)[cur[s]++] = t;
      (*nbr)[cur[t]++] = s;
    }
  }
}

// SweepSchedule::sweeps_for_level (multilevel.rs:104-120).
uint32_t sweeps_for_level(uint32_t schedule, uint64_t level, uint32_t base) {
  const uint64_t b = std::max(base, 1u);
  uint64_t s = schedule == 0 ? b : schedule == 1 ? b * (1 + level) : b << std::min<uint64_t>(level, 16);
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(s, 0xFFFFFFFFull));
}

// ------------------------------------------------------ xorshift jump --
// The jitter generator's state update s ^= s>>12; s ^= s<<25; s ^= s>>27 is
// linear over GF(2)^64; a map is kept as its 64 columns (images of the unit
// vectors), applied as the XOR of the columns of the set bits.
struct Gf2Map {
  uint64_t col[64];
  uint64_t apply(uint64_t s) const {
    uint64_t r = 0;
    while (s) {
      const int j = __builtin_ctzll(s);
      r ^= col[j];
      s &= s - 1;
    }
    return r;
  }
  Gf2Map then(const Gf2Map& after) const {  // after(this(x))
    Gf2Map m;
    for (int j = 0; j < 64; ++j) m.col[j] = after.apply(col[j]);
    return m;
  }
};

inline uint64_t xorshift_step(uint64_t s) {
  s ^= s >> 12;
  s ^= s << 25;
  s ^= s >> 27;
  return s;
}

// Starting state of every JITTER_CHUNK-value chunk of the stream that
// prolong (coarsen.rs:157-183) draws for `count` values from `seed`.
std::vector<unsigned long long> chunk_states(uint32_t seed, uint64_t count) {
  Gf2Map step;
  for (int j = 0; j < 64; ++j) step.col[j] = xorshift_step(1ull << j);
  Gf2Map jump = step;  // step^(2^k) by squaring up to JITTER_CHUNK
  for (uint32_t k = 1; k < JITTER_CHUNK; k <<= 1) jump = jump.then(jump);
  const uint64_t chunks = (count + JITTER_CHUNK - 1) / JITTER_CHUNK;
  std::vector<unsigned long long> out(chunks);
  uint64_t s = (uint64_t)seed + 0x9E3779B97F4A7C15ull;
  for (uint64_t c = 0; c < chunks; ++c) {
    out[c] = s;
    s = jump.apply(s);
  }
  return out;
}

// ------------------------------------------------------------- kernels --
// fold_up (multilevel.rs:480-510) for one level: the mean of each coarse
// node's children, summed from 0 in increasing child index, f32.
__global__ void k_fold_up(const float* __restrict__ fine, const uint32_t* __restrict__ children, uint32_t n_coarse,
                          float* __restrict__ coarse) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_coarse) return;
  const uint32_t c0 = children[2 * (size_t)p], c1 = children[2 * (size_t)p + 1];
  float sx = 0.0f, sy = 0.0f, sz = 0.0f, cnt = 0.0f;
  if (c0 != NONE) {
    sx = __fadd_rn(sx, fine[3 * (size_t)c0]);
    sy = __fadd_rn(sy, fine[3 * (size_t)c0 + 1]);
    sz = __fadd_rn(sz, fine[3 * (size_t)c0 + 2]);
    cnt = 1.0f;
  }
  if (c1 != NONE) {
    sx = __fadd_rn(sx, fine[3 * (size_t)c1]);
    sy = __fadd_rn(sy, fine[3 * (size_t)c1 + 1]);
    sz = __fadd_rn(sz, fine[3 * (size_t)c1 + 2]);
    cnt = 2.0f;
  }
  cnt = fmaxf(cnt, 1.0f);
  coarse[3 * (size_t)p] = __fdiv_rn(sx, cnt);
  coarse[3 * (size_t)p + 1] = __fdiv_rn(sy, cnt);
  coarse[3 * (size_t)p + 2] = __fdiv_rn(sz, cnt);
}

// prolong (coarsen.rs:157-183): value k of the child positions (child k/3,
// axis k%3) is parent[parent_map[k/3]][k%3] + jitter * r_k, where r_k is the
// k-th xorshift draw mapped to [-1, 1). One thread per chunk of draws.
__global__ void k_prolong(const float* __restrict__ parent_xyz, const uint32_t* __restrict__ parent_map,
                          uint64_t count, const unsigned long long* __restrict__ states, float jitter,
                          float* __restrict__ out) {
  const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t k0 = c * JITTER_CHUNK;
  if (k0 >= count) return;
  const uint64_t k1 = min(count, k0 + JITTER_CHUNK);
  unsigned long long s = states[c];
  for (uint64_t k = k0; k < k1; ++k) {
    s ^= s >> 12;
    s ^= s << 25;
    s ^= s >> 27;
    const unsigned long long v = s * 0x2545F4914F6CDD1Dull;
    const double u = __dmul_rn(__ull2double_rn(v >> 11), 1.0 / 9007199254740992.0);
    const float r = __fsub_rn(__fmul_rn(__double2float_rn(u), 2.0f), 1.0f);
    const uint64_t child = k / 3;
    const uint32_t axis = (uint32_t)(k - 3 * child);
    const float base = parent_xyz[3 * (size_t)parent_map[child] + axis];
    out[k] = __fadd_rn(base, __fmul_rn(r, jitter));
  }
}

template <typename T>
struct DArr {
  T* p = nullptr;
  size_t n = 0;
  void upload(const std::vector<T>& v, cudaStream_t s) {
    reserve(v.size());
    if (!v.empty()) JC_CUDA_CHECK(cudaMemcpyAsync(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
  }
  void reserve(size_t count) {
    if (count <= n && p) return;
    release();
    JC_CUDA_CHECK(cudaMalloc((void**)&p, sizeof(T) * std::max<size_t>(count, 1)));
    n = std::max<size_t>(count, 1);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void swap(DArr& o) {
    std::swap(p, o.p);
    std::swap(n, o.n);
  }
  DArr() = default;
  DArr(const DArr&) = delete;
  DArr& operator=(const DArr&) = delete;
  ~DArr() { release(); }
};

inline uint32_t blocks_for(uint64_t work, uint32_t threads) { return (uint32_t)((work + threads - 1) / threads); }

bool is_leaf_id(const std::string& id) {
  return id == "fa2-bh" || id == "fa2-brute" || id == "sgd-stress" || id == "sgd-stress-gpu";
}

Engine* make_leaf(const std::string& id) {
  if (id == "fa2-bh") return make_fa2_engine(true);
  if (id == "fa2-brute") return make_fa2_engine(false);
  if (id == "sgd-stress") return make_sgd_engine(false);
  if (id == "sgd-stress-gpu") return make_sgd_engine(true);
  return nullptr;
}

// ------------------------------------------------------------- engine --
class MultilevelEngine : public Engine {
 public:
  MultilevelEngine() {
    desc_.id = "multilevel";
    desc_.kind = 1;
    desc_.display_name = "Multilevel (multiscale wrapper, B200)";
    desc_.description =
        "Coarsen -> solve coarsest -> prolong -> refine, wrapping any inner engine (Walshaw/FM3/sfdp): the "
        "matching cascade is built once on the host, fold-up and prolongation with the exact xorshift jitter "
        "run on the device, and the inner engine is rebound level by level from device positions.";
    desc_.needs_edges = 1;
    desc_.needs_cpu_positions = 1;
    desc_.needs_gpu_positions_buffer = 0;
  }
  ~MultilevelEngine() override {
    inner_.reset();
    if (stream_) {
      cudaStreamSynchronize(stream_);
      cudaStreamDestroy(stream_);
    }
  }

  const jc_descriptor& descriptor() const override { return desc_; }

  // MultilevelEngine::set_params (multilevel.rs:336-357): null keeps the
  // settings; the inner id must be a leaf engine (not "multilevel").
  void set_params(const char* json) override {
    MultilevelSettings t = s_;
    decode_multilevel(json, &t);
    if (t.inner == "multilevel") fail(JC_ERR_PARAMS, "multilevel cannot wrap itself");
    if (!is_leaf_id(t.inner)) fail(JC_ERR_PARAMS, "unknown inner engine \"" + t.inner + "\" for multilevel wrapper");
    s_ = t;
  }

  // MultilevelEngine::init (multilevel.rs:359-410).
  void init(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint64_t nnz, const float* xyz) override {
    validate_csr(n, off, nbr, nnz, xyz);
    initialized_ = false;
    if (!stream_) JC_CUDA_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    std::vector<uint32_t> edges;
    edges.reserve(nnz);
    for (uint32_t v = 0; v < n; ++v)
      for (uint32_t e = off[v]; e < off[v + 1]; ++e)
        if (v < nbr[e]) {
          edges.push_back(v);
          edges.push_back(nbr[e]);
        }
    levels_ = coarsen(n, std::move(edges), s_.max_levels, s_.target_size);
    // device copies of the maps, and the seed folded up to the coarsest level
    const size_t L = levels_.size();
    parent_d_.clear();
    children_d_.clear();
    parent_d_.resize(L);
    children_d_.resize(L);
    for (size_t l = 1; l < L; ++l) {
      parent_d_[l] = std::make_unique<DArr<uint32_t>>();
      children_d_[l] = std::make_unique<DArr<uint32_t>>();
      parent_d_[l]->upload(levels_[l].parent_map, stream_);
      children_d_[l]->upload(levels_[l].children, stream_);
    }
    pos_a_.reserve(3ull * n);
    pos_b_.reserve(3ull * n);
    if (n) JC_CUDA_CHECK(cudaMemcpyAsync(pos_a_.p, xyz, 12ull * n, cudaMemcpyHostToDevice, stream_));
    for (size_t l = 1; l < L; ++l) {
      const uint32_t cn = levels_[l].n;
      k_fold_up<<<blocks_for(cn, 256), 256, 0, stream_>>>(pos_a_.p, children_d_[l]->p, cn, pos_b_.p);
      JC_CUDA_CHECK(cudaGetLastError());
      pos_a_.swap(pos_b_);
    }
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    // the inner engine, built once and rebound per level (multilevel.rs:299-322)
    inner_.reset(make_leaf(s_.inner));
    if (!inner_) fail(JC_ERR_PARAMS, "unknown inner engine \"" + s_.inner + "\"");
    inner_->set_params(s_.inner_params.c_str());
    level_ = (uint32_t)(L - 1);
    sweeps_done_ = 0;
    bind_level(pos_a_.p);
    initialized_ = true;
  }

  // One inner step; when the level's sweep budget is spent, prolong to the
  // next finer level and rebind (multilevel.rs:412-468).
  void step(float* out) override {
    require_init();
    inner_->step_many(1, nullptr);
    ++sweeps_done_;
    maybe_descend();
    if (out) inner_->positions(out);
  }

  void step_many(uint32_t iters, float* out) override {
    require_init();
    uint32_t left = iters;
    while (left > 0) {
      uint32_t k = left;
      if (level_ > 0) {
        const uint32_t budget = sweeps_for_level(s_.sweep_schedule, level_, s_.sweeps_per_level);
        k = std::min(k, budget > sweeps_done_ ? budget - sweeps_done_ : 1u);
      }
      inner_->step_many(k, nullptr);
      sweeps_done_ += k;
      left -= k;
      maybe_descend();
    }
    if (out) inner_->positions(out);
  }

  bool is_halted() const override { return initialized_ && level_ == 0 && inner_->is_halted(); }
  void positions(float* out) override {
    require_init();
    inner_->positions(out);
  }
  void forces(float* f, float* s) override {
    require_init();
    inner_->forces(f, s);
  }
  void speed(float* a, float* b) override {
    require_init();
    inner_->speed(a, b);
  }
  uint32_t status_bits() override { return inner_ ? inner_->status_bits() : 0u; }
  void tree_info(uint32_t* o) override {
    require_init();
    inner_->tree_info(o);
  }
  void walk_counts(uint64_t* o) override {
    require_init();
    inner_->walk_counts(o);
  }
  void stress(double* a, double* b) override {
    require_init();
    inner_->stress(a, b);
  }
  void time_steps(uint32_t iters, float* total_ms, float* phase_ms4) override {
    require_init();
    inner_->time_steps(iters, total_ms, phase_ms4);
  }
  uint32_t launches_per_step() const override { return inner_ ? inner_->launches_per_step() : 0u; }
  uint32_t node_count() const override { return levels_.empty() ? 0u : levels_[0].n; }
  uint32_t output_nodes() const override { return inner_ ? inner_->node_count() : 0u; }

  // Cascade read-out: the current level, the level count and each level's nodes.
  void level_info(uint32_t* level, uint32_t* n_levels, uint32_t* sweeps_done) const {
    *level = level_;
    *n_levels = (uint32_t)levels_.size();
    *sweeps_done = sweeps_done_;
  }
  const std::vector<Level>& levels() const { return levels_; }

  // State: the cascade position, then the inner engine's state.
  uint64_t state_size() override {
    require_init();
    return 8 + inner_->state_size();
  }
  void save_state(void* buf) override {
    require_init();
    uint8_t* b = (uint8_t*)buf;
    std::memcpy(b, &level_, 4);
    std::memcpy(b + 4, &sweeps_done_, 4);
    inner_->save_state(b + 8);
  }
  void load_state(const void* buf, uint64_t len) override {
    require_init();
    if (len < 8) fail(JC_ERR_ARG, "state size mismatch");
    const uint8_t* b = (const uint8_t*)buf;
    uint32_t level, sweeps;
    std::memcpy(&level, b, 4);
    std::memcpy(&sweeps, b + 4, 4);
    if (level >= levels_.size()) fail(JC_ERR_ARG, "state is for another cascade");
    if (level != level_) {
      // bind the saved level (positions are replaced by the inner state)
      pos_a_.reserve(3ull * std::max(levels_[level].n, 1u));
      JC_CUDA_CHECK(cudaMemsetAsync(pos_a_.p, 0, 12ull * levels_[level].n, stream_));
      JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
      level_ = level;
      bind_level(pos_a_.p);
    }
    inner_->load_state(b + 8, len - 8);
    sweeps_done_ = sweeps;
  }

 private:
  void require_init() const {
    if (!initialized_) fail(JC_ERR_STATE, "multilevel step called before successful init");
  }

  void bind_level(const float* d_xyz) {
    std::vector<uint32_t> off, nbr;
    level_csr(levels_[level_], &off, &nbr);
    inner_->reinit_device(levels_[level_].n, off.data(), nbr.empty() ? nullptr : nbr.data(), nbr.size(), d_xyz);
  }

  void maybe_descend() {
    if (level_ == 0) return;
    const uint32_t budget = sweeps_for_level(s_.sweep_schedule, level_, s_.sweeps_per_level);
    if (sweeps_done_ < budget) return;
    const uint32_t child = level_ - 1;
    const uint32_t child_n = levels_[child].n;
    const uint64_t count = 3ull * child_n;
    const float jitter = s_.spring_len * 0.5f;
    const uint32_t seed = s_.seed + child + 1u;  // wrapping add
    // the coarse positions come from the inner engine's device buffer
    const float* coarse = inner_->device_xyz();
    std::vector<unsigned long long> states = chunk_states(seed, count);
    states_.upload(states, stream_);
    pos_b_.reserve(std::max<uint64_t>(count, 1));
    cudaStream_t is = inner_->cuda_stream();
    if (is) JC_CUDA_CHECK(cudaStreamSynchronize(is));  // the inner steps have written `coarse`
    if (count) {
      k_prolong<<<blocks_for(states.size(), 128), 128, 0, stream_>>>(coarse, parent_d_[level_]->p, count,
                                                                      states_.p, jitter, pos_b_.p);
      JC_CUDA_CHECK(cudaGetLastError());
    }
    JC_CUDA_CHECK(cudaStreamSynchronize(stream_));
    level_ = child;
    sweeps_done_ = 0;
    bind_level(pos_b_.p);
  }

  jc_descriptor desc_{};
  MultilevelSettings s_;
  std::unique_ptr<Engine> inner_;
  std::vector<Level> levels_;
  std::vector<std::unique_ptr<DArr<uint32_t>>> parent_d_, children_d_;
  DArr<float> pos_a_, pos_b_;
  DArr<unsigned long long> states_;
  cudaStream_t stream_ = nullptr;
  uint32_t level_ = 0, sweeps_done_ = 0;
  bool initialized_ = false;
};

}  // namespace

Engine* make_multilevel_engine() { return new MultilevelEngine(); }

namespace {
struct CascadeHandle {
  std::vector<Level> levels;
};
bool level_out(const Level& L, uint32_t* n_nodes, uint64_t* n_edge_words, uint32_t* edges, uint32_t* parent_map) {
  *n_nodes = L.n;
  *n_edge_words = L.edges.size();
  if (edges && !L.edges.empty()) std::memcpy(edges, L.edges.data(), 4 * L.edges.size());
  if (parent_map && !L.parent_map.empty()) std::memcpy(parent_map, L.parent_map.data(), 4 * L.parent_map.size());
  return true;
}
}  // namespace

// The cascade alone (graph_layouts::coarsen is public in the reference).
void* cascade_build(uint32_t n, const uint32_t* edges, uint64_t n_words, uint64_t max_levels, uint64_t target_size) {
  CascadeHandle* h = new CascadeHandle();
  try {
    h->levels = coarsen(n, std::vector<uint32_t>(edges, edges + n_words), max_levels, target_size);
  } catch (...) {
    delete h;
    throw;
  }
  return h;
}
uint32_t cascade_count(const void* h) { return (uint32_t)((const CascadeHandle*)h)->levels.size(); }
bool cascade_get(const void* h, uint32_t l, uint32_t* n_nodes, uint64_t* n_edge_words, uint32_t* edges,
                 uint32_t* parent_map) {
  const CascadeHandle* c = (const CascadeHandle*)h;
  if (l >= c->levels.size()) return false;
  return level_out(c->levels[l], n_nodes, n_edge_words, edges, parent_map);
}
void cascade_free(void* h) { delete (CascadeHandle*)h; }

// Cascade read-outs for the C ABI.
bool multilevel_level_info(Engine* e, uint32_t* level, uint32_t* n_levels, uint32_t* sweeps_done) {
  MultilevelEngine* m = dynamic_cast<MultilevelEngine*>(e);
  if (!m) return false;
  m->level_info(level, n_levels, sweeps_done);
  return true;
}

bool multilevel_level_get(Engine* e, uint32_t l, uint32_t* n_nodes, uint64_t* n_edge_words, uint32_t* edges,
                          uint32_t* parent_map) {
  MultilevelEngine* m = dynamic_cast<MultilevelEngine*>(e);
  if (!m || l >= m->levels().size()) return false;
  return level_out(m->levels()[l], n_nodes, n_edge_words, edges, parent_map);
}

}  // namespace jc
