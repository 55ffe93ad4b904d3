// C ABI of libjc_layout: engine registry and the LayoutEngine trait methods
// (crates/graph-compute/src/engines/mod.rs:383-488), with every C++
// exception turned into a jc_status plus a per-handle message.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "jc_check.cuh"
#include "jc_common.h"
#include "jc_engine.h"
#include "jc_frames.h"
#include "jc_partition.h"

struct jc_engine {
  jc::Engine* impl = nullptr;
  jc::FrameStream* frames = nullptr;        // open frame stream, if any
  jc::PartitionLayout* partition = nullptr;  // set by jc_engine_init_partitions
  std::string last_error;
  void close_frames() {
    delete frames;
    frames = nullptr;
  }
  void unbind() {  // before the engine is bound to another graph
    close_frames();
    delete partition;
    partition = nullptr;
  }
};

struct jc_partitions {
  jc::PartitionSet set;
};

struct jc_frame_decoder {
  jc::FrameDecoder d;
  std::string last_error;
};

namespace jc {

void validate_csr(uint32_t n, const uint32_t* offsets, const uint32_t* neighbors, uint64_t nnz,
                  const float* xyz) {
  if (n > 0 && xyz == nullptr) fail(JC_ERR_ARG, "positions must be non-null for a non-empty graph");
  validate_csr_arrays(n, offsets, neighbors, nnz);
}

void validate_csr_offsets(uint32_t n, const uint32_t* offsets, const uint32_t* neighbors, uint64_t nnz) {
  if (n > 0 && offsets == nullptr) fail(JC_ERR_ARG, "offsets must be non-null for a non-empty graph");
  if (n == 0) return;
  if (offsets[0] != 0) fail(JC_ERR_ARG, "offsets[0] must be 0");
  bool decreasing = false;
#pragma omp parallel for schedule(static) reduction(|| : decreasing)
  for (int64_t v = 0; v < (int64_t)n; ++v)
    if (offsets[v + 1] < offsets[v]) decreasing = true;
  if (decreasing) fail(JC_ERR_ARG, "offsets must be non-decreasing");
  if ((uint64_t)offsets[n] != nnz)
    fail(JC_ERR_ARG, "offsets[n_nodes] (" + std::to_string(offsets[n]) + ") != n_neighbors (" +
                         std::to_string(nnz) + ")");
  if (nnz && neighbors == nullptr) fail(JC_ERR_ARG, "neighbors must be non-null");
}

void validate_csr_arrays(uint32_t n, const uint32_t* offsets, const uint32_t* neighbors, uint64_t nnz) {
  validate_csr_offsets(n, offsets, neighbors, nnz);
  if (n == 0) return;
  int64_t bad = -1;
#pragma omp parallel for schedule(static) reduction(max : bad)
  for (int64_t e = 0; e < (int64_t)nnz; ++e)
    if (neighbors[e] >= n) bad = std::max<int64_t>(bad, e);
  if (bad >= 0)
    fail(JC_ERR_ARG, "neighbor id " + std::to_string(neighbors[bad]) + " out of range for " + std::to_string(n) +
                         " nodes");
}

}  // namespace jc

namespace {

// LEAF_ENGINE_IDS (mod.rs:455-463) restricted to the layout-step engines,
// then the multilevel wrapper (engines/multilevel.rs, MultilevelEngine::ID).
const char* kIds[] = {"fa2-brute", "fa2-bh", "sgd-stress", "sgd-stress-gpu", "multilevel"};

template <typename F>
jc_status guarded(jc_engine* e, F&& f) {
  if (e == nullptr) return JC_ERR_ARG;
  try {
    f();
    e->last_error.clear();
    return JC_OK;
  } catch (const jc::Error& err) {
    e->last_error = err.what();
    return err.code;
  } catch (const std::bad_alloc&) {
    e->last_error = "host allocation failed";
    return JC_ERR_ARG;
  } catch (const std::exception& err) {
    e->last_error = err.what();
    return JC_ERR_ARG;
  }
}

}  // namespace

extern "C" {

uint32_t jc_engine_count(void) { return (uint32_t)(sizeof(kIds) / sizeof(kIds[0])); }

const char* jc_engine_id_at(uint32_t index) { return index < jc_engine_count() ? kIds[index] : nullptr; }

jc_status jc_engine_create(const char* engine_id, jc_engine** out) {
  if (out == nullptr || engine_id == nullptr) return JC_ERR_ARG;
  *out = nullptr;
  jc::Engine* impl = nullptr;
  try {
    if (std::strcmp(engine_id, "fa2-bh") == 0) impl = jc::make_fa2_engine(true);
    else if (std::strcmp(engine_id, "fa2-brute") == 0) impl = jc::make_fa2_engine(false);
    else if (std::strcmp(engine_id, "sgd-stress-gpu") == 0) impl = jc::make_sgd_engine(true);
    else if (std::strcmp(engine_id, "sgd-stress") == 0) impl = jc::make_sgd_engine(false);
    else if (std::strcmp(engine_id, "multilevel") == 0) impl = jc::make_multilevel_engine();
    else return JC_ERR_UNKNOWN_ENGINE;
  } catch (...) {
    return JC_ERR_ARG;
  }
  jc_engine* e = new (std::nothrow) jc_engine();
  if (!e) {
    delete impl;
    return JC_ERR_ARG;
  }
  e->impl = impl;
  *out = e;
  return JC_OK;
}

void jc_engine_destroy(jc_engine* e) {
  if (!e) return;
  e->unbind();
  delete e->impl;
  delete e;
}

jc_status jc_engine_descriptor(const jc_engine* e, jc_descriptor* out) {
  if (!e || !out) return JC_ERR_ARG;
  *out = e->impl->descriptor();
  return JC_OK;
}

jc_status jc_engine_set_params(jc_engine* e, const char* json) {
  return guarded(e, [&] { e->impl->set_params(json); });
}

jc_status jc_engine_init(jc_engine* e, uint32_t n, const uint32_t* off, const uint32_t* nbr, uint64_t nnz,
                         const float* xyz) {
  return guarded(e, [&] {
    e->unbind();
    e->impl->init(n, off, nbr, nnz, xyz);
  });
}

jc_status jc_engine_reinit(jc_engine* e, uint32_t n, const uint32_t* off, const uint32_t* nbr, uint64_t nnz,
                           const float* xyz) {
  return guarded(e, [&] {
    e->unbind();
    e->impl->reinit(n, off, nbr, nnz, xyz);
  });
}

jc_status jc_engine_step(jc_engine* e, float* out_xyz) {
  return guarded(e, [&] { e->impl->step(out_xyz); });
}

jc_status jc_engine_step_many(jc_engine* e, uint32_t iters, float* out_xyz) {
  return guarded(e, [&] { e->impl->step_many(iters, out_xyz); });
}

jc_status jc_engine_apply_halo(jc_engine* e, uint64_t frame, uint32_t owner, const uint32_t* ids,
                               const float* xyz, uint32_t count) {
  return guarded(e, [&] { e->impl->apply_halo(frame, owner, ids, xyz, count); });
}

int32_t jc_engine_is_halted(const jc_engine* e) { return (e && e->impl->is_halted()) ? 1 : 0; }

const char* jc_engine_last_error(const jc_engine* e) { return e ? e->last_error.c_str() : "null engine handle"; }

jc_status jc_engine_save_state(jc_engine* e, void* buf, uint64_t capacity, uint64_t* needed) {
  return guarded(e, [&] {
    uint64_t need = e->impl->state_size();
    if (needed) *needed = need;
    if (buf == nullptr) return;
    if (capacity < need) jc::fail(JC_ERR_ARG, "state buffer too small");
    e->impl->save_state(buf);
  });
}

jc_status jc_engine_load_state(jc_engine* e, const void* buf, uint64_t len) {
  return guarded(e, [&] {
    if (!buf) jc::fail(JC_ERR_ARG, "null state buffer");
    e->close_frames();
    e->impl->load_state(buf, len);
  });
}

jc_status jc_engine_positions(jc_engine* e, float* out) {
  return guarded(e, [&] {
    if (!out) jc::fail(JC_ERR_ARG, "null output buffer");
    e->impl->positions(out);
  });
}

jc_status jc_engine_forces(jc_engine* e, float* out, float* stats) {
  return guarded(e, [&] {
    if (!out) jc::fail(JC_ERR_ARG, "null output buffer");
    e->impl->forces(out, stats);
  });
}

jc_status jc_engine_speed(jc_engine* e, float* speed, float* eff) {
  return guarded(e, [&] { e->impl->speed(speed, eff); });
}

uint32_t jc_engine_status_bits(jc_engine* e) {
  if (!e) return 0;
  try {
    return e->impl->status_bits();
  } catch (...) {
    return 0;
  }
}

jc_status jc_engine_tree_info(jc_engine* e, uint32_t* out4) {
  return guarded(e, [&] {
    if (!out4) jc::fail(JC_ERR_ARG, "null output");
    e->impl->tree_info(out4);
  });
}

jc_status jc_engine_walk_counts(jc_engine* e, uint64_t* out2) {
  return guarded(e, [&] {
    if (!out2) jc::fail(JC_ERR_ARG, "null output");
    e->impl->walk_counts(out2);
  });
}

jc_status jc_engine_init_batch(jc_engine* e, uint32_t n_graphs, const uint32_t* graph_nodes,
                               const uint32_t* offsets, const uint32_t* neighbors, const float* xyz) {
  return guarded(e, [&] {
    e->unbind();
    e->impl->init_batch(n_graphs, graph_nodes, offsets, neighbors, xyz);
  });
}

jc_status jc_partition_csr(uint32_t n_nodes, const uint32_t* offsets, const uint32_t* neighbors,
                           uint64_t n_neighbors, uint32_t n_partitions, int32_t refine, jc_partitions** out) {
  if (!out) return JC_ERR_ARG;
  *out = nullptr;
  try {
    jc::validate_csr_arrays(n_nodes, offsets, neighbors, n_neighbors);
    jc_partitions* p = new jc_partitions();
    try {
      p->set = jc::partition_csr(n_nodes, offsets, neighbors, n_partitions, refine != 0);
    } catch (...) {
      delete p;
      throw;
    }
    *out = p;
    return JC_OK;
  } catch (const jc::Error& err) {
    return err.code;
  } catch (...) {
    return JC_ERR_ARG;
  }
}

void jc_partitions_free(jc_partitions* p) { delete p; }

uint32_t jc_partitions_count(const jc_partitions* p) { return p ? (uint32_t)p->set.parts.size() : 0u; }

uint64_t jc_partitions_edge_cut(const jc_partitions* p) { return p ? p->set.edge_cut : 0u; }

const uint32_t* jc_partitions_owner(const jc_partitions* p) {
  return p && !p->set.owner.empty() ? p->set.owner.data() : nullptr;
}

jc_status jc_partition_get(const jc_partitions* p, uint32_t index, jc_partition_view* out) {
  if (!p || !out || index >= p->set.parts.size()) return JC_ERR_ARG;
  const jc::PartitionPart& part = p->set.parts[index];
  out->partition_id = part.id;
  out->n_partitions = p->set.n_partitions;
  out->n_local = part.n_local();
  out->n_owned = part.n_owned;
  out->n_neighbors = part.neighbors.size();
  out->n_boundary = (uint32_t)part.boundary.size();
  out->offsets = part.offsets.data();
  out->neighbors = part.neighbors.empty() ? nullptr : part.neighbors.data();
  out->global_ids = part.global_ids.empty() ? nullptr : part.global_ids.data();
  out->boundary = part.boundary.empty() ? nullptr : part.boundary.data();
  return JC_OK;
}

jc_status jc_engine_init_partitions(jc_engine* e, const jc_partitions* p, const float* global_xyz) {
  return guarded(e, [&] {
    if (!p) jc::fail(JC_ERR_ARG, "null partition set");
    const jc::PartitionSet& ps = p->set;
    if (ps.n_nodes && !global_xyz) jc::fail(JC_ERR_ARG, "null positions");
    // Empty partitions hold no nodes and are left out of the batch (the
    // slots of the others do not move).
    std::vector<uint32_t> nodes, off, nbr;
    std::vector<float> xyz;
    for (const jc::PartitionPart& part : ps.parts) {
      if (part.n_local() == 0) continue;
      nodes.push_back(part.n_local());
      off.insert(off.end(), part.offsets.begin(), part.offsets.end());
      nbr.insert(nbr.end(), part.neighbors.begin(), part.neighbors.end());
      for (uint32_t g : part.global_ids)
        xyz.insert(xyz.end(), global_xyz + 3 * (size_t)g, global_xyz + 3 * (size_t)g + 3);
    }
    e->unbind();
    if (nodes.empty()) {
      const uint32_t zero = 0;
      e->impl->init(0, &zero, nullptr, 0, nullptr);
    } else {
      e->impl->init_batch((uint32_t)nodes.size(), nodes.data(), off.data(), nbr.data(), xyz.data());
    }
    e->partition = new jc::PartitionLayout(e->impl, ps);
  });
}

jc_status jc_engine_partition_positions(jc_engine* e, float* global_xyz) {
  return guarded(e, [&] {
    if (!e->partition) jc::fail(JC_ERR_STATE, "engine is not bound to a partition set");
    e->partition->owned_positions(global_xyz);
  });
}

jc_status jc_engine_halo_delta(jc_engine* e, uint32_t p, float* out_xyz, uint32_t* count) {
  return guarded(e, [&] {
    if (!e->partition) jc::fail(JC_ERR_STATE, "engine is not bound to a partition set");
    if (p >= e->partition->n_partitions()) jc::fail(JC_ERR_ARG, "partition index out of range");
    if (count) *count = e->partition->boundary_count(p);
    if (out_xyz) e->partition->halo_delta(p, out_xyz);
  });
}

jc_status jc_engine_level_info(jc_engine* e, uint32_t* level, uint32_t* n_levels, uint32_t* sweeps_done) {
  return guarded(e, [&] {
    uint32_t a = 0, b = 0, c = 0;
    if (!jc::multilevel_level_info(e->impl, &a, &b, &c)) jc::fail(JC_ERR_ARG, "not a multilevel engine");
    if (level) *level = a;
    if (n_levels) *n_levels = b;
    if (sweeps_done) *sweeps_done = c;
  });
}

jc_status jc_engine_cascade_level(jc_engine* e, uint32_t l, uint32_t* n_nodes, uint64_t* n_edge_words,
                                  uint32_t* edges, uint32_t* parent_map) {
  return guarded(e, [&] {
    uint32_t n = 0;
    uint64_t w = 0;
    if (!jc::multilevel_level_get(e->impl, l, &n, &w, edges, parent_map))
      jc::fail(JC_ERR_ARG, "not a multilevel engine, or no such level");
    if (n_nodes) *n_nodes = n;
    if (n_edge_words) *n_edge_words = w;
  });
}

jc_status jc_coarsen(uint32_t n_nodes, const uint32_t* edges, uint64_t n_edge_words, uint64_t max_levels,
                     uint64_t target_size, jc_cascade** out) {
  if (!out || (n_edge_words && !edges)) return JC_ERR_ARG;
  *out = nullptr;
  try {
    *out = (jc_cascade*)jc::cascade_build(n_nodes, edges, n_edge_words, max_levels, target_size);
    return JC_OK;
  } catch (const jc::Error& err) {
    return err.code;
  } catch (...) {
    return JC_ERR_ARG;
  }
}

uint32_t jc_cascade_levels(const jc_cascade* c) { return c ? jc::cascade_count(c) : 0u; }

jc_status jc_cascade_get(const jc_cascade* c, uint32_t l, uint32_t* n_nodes, uint64_t* n_edge_words,
                         uint32_t* edges, uint32_t* parent_map) {
  if (!c || !n_nodes || !n_edge_words) return JC_ERR_ARG;
  return jc::cascade_get(c, l, n_nodes, n_edge_words, edges, parent_map) ? JC_OK : JC_ERR_ARG;
}

void jc_cascade_free(jc_cascade* c) {
  if (c) jc::cascade_free(c);
}

uint32_t jc_engine_output_nodes(const jc_engine* e) {
  if (!e) return 0;
  try {
    return e->impl->output_nodes();
  } catch (...) {
    return 0;
  }
}

jc_status jc_engine_stream_open(jc_engine* e, uint32_t encoding, uint32_t depth, uint32_t keyframe_interval) {
  return guarded(e, [&] {
    e->close_frames();
    e->frames = new jc::FrameStream(e->impl, encoding, depth, keyframe_interval);
  });
}

jc_status jc_engine_stream_step(jc_engine* e, uint32_t iters) {
  return guarded(e, [&] {
    if (!e->frames) jc::fail(JC_ERR_STATE, "no frame stream open");
    e->frames->step(iters);
  });
}

jc_status jc_engine_stream_next(jc_engine* e, jc_frame* out) {
  return guarded(e, [&] {
    if (!e->frames) jc::fail(JC_ERR_STATE, "no frame stream open");
    if (!out) jc::fail(JC_ERR_ARG, "null frame");
    e->frames->next(out);
  });
}

jc_status jc_engine_stream_close(jc_engine* e) {
  return guarded(e, [&] { e->close_frames(); });
}

jc_frame_decoder* jc_frame_decoder_create(uint32_t n_nodes) {
  jc_frame_decoder* d = new (std::nothrow) jc_frame_decoder();
  if (!d) return nullptr;
  try {
    d->d.n = n_nodes;
    d->d.rec.assign(3ull * n_nodes, 0.0f);
  } catch (...) {
    delete d;
    return nullptr;
  }
  return d;
}

void jc_frame_decoder_destroy(jc_frame_decoder* d) { delete d; }

jc_status jc_frame_decode(jc_frame_decoder* d, const uint8_t* data, uint64_t bytes, float* out_xyz) {
  if (!d) return JC_ERR_ARG;
  try {
    jc::decode_frame(d->d, data, bytes, out_xyz);
    d->last_error.clear();
    return JC_OK;
  } catch (const jc::Error& err) {
    d->last_error = err.what();
    return err.code;
  }
}

const char* jc_frame_decoder_last_error(const jc_frame_decoder* d) { return d ? d->last_error.c_str() : ""; }

jc_status jc_engine_graph_speed(jc_engine* e, uint32_t graph, float* speed, float* eff) {
  return guarded(e, [&] { e->impl->graph_speed(graph, speed, eff); });
}

jc_status jc_engine_autotune(jc_engine* e, uint32_t probe_steps, uint32_t* walk_group, float* ms6) {
  return guarded(e, [&] {
    uint32_t g = e->impl->autotune(probe_steps, ms6);
    if (walk_group) *walk_group = g;
  });
}

jc_status jc_engine_batch_schedule(jc_engine* e, uint32_t* tile_schedule, float* tile_ms_per_step) {
  return guarded(e, [&] { e->impl->schedule_info(tile_schedule, tile_ms_per_step); });
}

jc_status jc_engine_pivots(jc_engine* e, uint32_t* k, uint32_t* pivots, uint32_t* dist) {
  return guarded(e, [&] {
    const uint32_t kk = e->impl->pivots(pivots, dist);
    if (k) *k = kk;
  });
}

jc_status jc_engine_stress(jc_engine* e, double* raw, double* normalized) {
  return guarded(e, [&] { e->impl->stress(raw, normalized); });
}

jc_status jc_engine_time_steps(jc_engine* e, uint32_t iters, float* total_ms, float* phase_ms4) {
  return guarded(e, [&] { e->impl->time_steps(iters, total_ms, phase_ms4); });
}

uint32_t jc_engine_launches_per_step(const jc_engine* e) { return e ? e->impl->launches_per_step() : 0; }

jc_status jc_set_device(int32_t device) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return JC_ERR_CUDA;
  return cudaSetDevice(device) == cudaSuccess ? JC_OK : JC_ERR_CUDA;
}

const char* jc_build_info(void) {
  return JC_BOUNDS_BUILD ? "libjc_layout: CUDA kernels built for sm_100a (B200); host C++17; bounds-check build "
                           "(device index checks record JC_ERR_BOUNDS)"
                         : "libjc_layout: CUDA kernels built for sm_100a (B200); host C++17";
}

}  // extern "C"

// Batch builder: graphs added one at a time, bound together by
// jc_engine_init_batch on the first bind, then stepped as one batch.
struct jc_batch {
  jc_engine* engine = nullptr;
  bool bound = false;
  std::vector<uint32_t> nodes, offsets, neighbors;  // concatenated per-graph CSR
  std::vector<float> xyz;                            // concatenated seeds
  std::vector<uint64_t> node_base;                   // first node of each graph
  std::string last_error;
};

namespace {

template <typename F>
jc_status batch_guarded(jc_batch* b, F&& f) {
  if (b == nullptr) return JC_ERR_ARG;
  try {
    f();
    b->last_error.clear();
    return JC_OK;
  } catch (const jc::Error& err) {
    b->last_error = err.what();
    return err.code;
  } catch (const std::bad_alloc&) {
    b->last_error = "host allocation failed";
    return JC_ERR_ARG;
  } catch (const std::exception& err) {
    b->last_error = err.what();
    return JC_ERR_ARG;
  }
}

void batch_bind(jc_batch* b) {
  if (b->bound) return;
  if (b->nodes.empty()) jc::fail(JC_ERR_STATE, "no graphs were added to the batch");
  const jc_status rc = jc_engine_init_batch(b->engine, (uint32_t)b->nodes.size(), b->nodes.data(),
                                            b->offsets.data(), b->neighbors.data(), b->xyz.data());
  if (rc != JC_OK) jc::fail(rc, b->engine->last_error);
  b->bound = true;
  // the bound engine holds its own copies
  std::vector<uint32_t>().swap(b->offsets);
  std::vector<uint32_t>().swap(b->neighbors);
  std::vector<float>().swap(b->xyz);
}

}  // namespace

extern "C" {

jc_status jc_batch_create(const char* engine_id, const char* params_json, jc_batch** out) {
  if (out == nullptr || engine_id == nullptr) return JC_ERR_ARG;
  *out = nullptr;
  if (std::strcmp(engine_id, "fa2-bh") != 0) return JC_ERR_UNKNOWN_ENGINE;
  jc_engine* e = nullptr;
  jc_status rc = jc_engine_create(engine_id, &e);
  if (rc != JC_OK) return rc;
  if (params_json != nullptr && (rc = jc_engine_set_params(e, params_json)) != JC_OK) {
    jc_engine_destroy(e);
    return rc;
  }
  jc_batch* b = new (std::nothrow) jc_batch();
  if (!b) {
    jc_engine_destroy(e);
    return JC_ERR_ARG;
  }
  b->engine = e;
  *out = b;
  return JC_OK;
}

void jc_batch_destroy(jc_batch* b) {
  if (!b) return;
  jc_engine_destroy(b->engine);
  delete b;
}

const char* jc_batch_last_error(const jc_batch* b) { return b ? b->last_error.c_str() : "null batch handle"; }

jc_status jc_batch_add_graph(jc_batch* b, uint32_t n_nodes, const uint32_t* offsets, const uint32_t* neighbors,
                             uint64_t n_neighbors, const float* positions_xyz, uint32_t* index) {
  return batch_guarded(b, [&] {
    if (b->bound) jc::fail(JC_ERR_STATE, "graphs cannot be added after the batch was bound");
    if (b->nodes.size() >= 65536) jc::fail(JC_ERR_ARG, "at most 65536 graphs per batch");
    if (n_nodes == 0) jc::fail(JC_ERR_ARG, "a graph of a batch needs at least one node");
    jc::validate_csr(n_nodes, offsets, neighbors, n_neighbors, positions_xyz);
    const uint64_t total_n = (b->node_base.empty() ? 0 : b->node_base.back() + b->nodes.back()) + n_nodes;
    if (total_n > 0xFFFFFFF0ull || b->neighbors.size() + n_neighbors > 0xFFFFFFF0ull)
      jc::fail(JC_ERR_ARG, "batch too large");
    b->node_base.push_back(total_n - n_nodes);
    b->nodes.push_back(n_nodes);
    b->offsets.insert(b->offsets.end(), offsets, offsets + n_nodes + 1);
    b->neighbors.insert(b->neighbors.end(), neighbors, neighbors + n_neighbors);
    b->xyz.insert(b->xyz.end(), positions_xyz, positions_xyz + 3 * (size_t)n_nodes);
    if (index) *index = (uint32_t)(b->nodes.size() - 1);
  });
}

jc_status jc_batch_bind(jc_batch* b) {
  return batch_guarded(b, [&] { batch_bind(b); });
}

jc_status jc_batch_run(jc_batch* b, uint32_t iters) {
  return batch_guarded(b, [&] {
    batch_bind(b);
    const jc_status rc = jc_engine_step_many(b->engine, iters, nullptr);
    if (rc != JC_OK) jc::fail(rc, b->engine->last_error);
  });
}

uint32_t jc_batch_graph_count(const jc_batch* b) { return b ? (uint32_t)b->nodes.size() : 0u; }

jc_status jc_batch_positions(jc_batch* b, uint32_t graph, float* out_xyz) {
  return batch_guarded(b, [&] {
    if (!out_xyz) jc::fail(JC_ERR_ARG, "null output buffer");
    if (graph >= b->nodes.size()) jc::fail(JC_ERR_ARG, "graph index out of range");
    if (!b->bound) jc::fail(JC_ERR_STATE, "the batch is not bound yet");
    b->engine->impl->positions_range(b->node_base[graph], b->nodes[graph], out_xyz);
  });
}

jc_engine* jc_batch_engine(jc_batch* b) { return b ? b->engine : nullptr; }

}  // extern "C"
