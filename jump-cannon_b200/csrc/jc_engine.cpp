// C ABI of libjc_layout: engine registry and the LayoutEngine trait methods
// (crates/graph-compute/src/engines/mod.rs:383-488), with every C++
// exception turned into a jc_status plus a per-handle message.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>

#include "jc_common.h"
#include "jc_engine.h"

struct jc_engine {
  jc::Engine* impl = nullptr;
  std::string last_error;
};

namespace jc {

void validate_csr(uint32_t n, const uint32_t* offsets, const uint32_t* neighbors, uint64_t nnz,
                  const float* xyz) {
  if (n > 0 && (offsets == nullptr || xyz == nullptr))
    fail(JC_ERR_ARG, "offsets and positions must be non-null for a non-empty graph");
  if (n == 0) return;
  if (offsets[0] != 0) fail(JC_ERR_ARG, "offsets[0] must be 0");
  for (uint32_t v = 0; v < n; ++v)
    if (offsets[v + 1] < offsets[v]) fail(JC_ERR_ARG, "offsets must be non-decreasing");
  if ((uint64_t)offsets[n] != nnz)
    fail(JC_ERR_ARG, "offsets[n_nodes] (" + std::to_string(offsets[n]) + ") != n_neighbors (" +
                         std::to_string(nnz) + ")");
  if (nnz && neighbors == nullptr) fail(JC_ERR_ARG, "neighbors must be non-null");
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

// LEAF_ENGINE_IDS (mod.rs:455-463) restricted to the layout-step engines.
const char* kIds[] = {"fa2-brute", "fa2-bh", "sgd-stress", "sgd-stress-gpu"};

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
  return guarded(e, [&] { e->impl->init(n, off, nbr, nnz, xyz); });
}

jc_status jc_engine_reinit(jc_engine* e, uint32_t n, const uint32_t* off, const uint32_t* nbr, uint64_t nnz,
                           const float* xyz) {
  return guarded(e, [&] { e->impl->reinit(n, off, nbr, nnz, xyz); });
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
  return guarded(e, [&] { e->impl->init_batch(n_graphs, graph_nodes, offsets, neighbors, xyz); });
}

jc_status jc_engine_graph_speed(jc_engine* e, uint32_t graph, float* speed, float* eff) {
  return guarded(e, [&] { e->impl->graph_speed(graph, speed, eff); });
}

jc_status jc_engine_autotune(jc_engine* e, uint32_t probe_steps, uint32_t* walk_group, float* ms6) {
  return guarded(e, [&] {
    uint32_t g = e->impl->autotune(probe_steps, ms6);
    if (walk_group) *walk_group = g;
  });
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
  return "libjc_layout: CUDA kernels built for sm_100a (B200); host C++17";
}

}  // extern "C"
