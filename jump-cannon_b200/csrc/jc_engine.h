// The engine interface behind the C ABI. It mirrors the reference's Rust
// trait `LayoutEngine` (crates/graph-compute/src/engines/mod.rs:383-444):
// descriptor / set_params / init / reinit / step / apply_halo / is_halted,
// plus the read-outs the tests and the benchmark use.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "jc_common.h"

namespace jc {

class Engine {
 public:
  virtual ~Engine() = default;

  virtual const jc_descriptor& descriptor() const = 0;
  virtual void set_params(const char* json) = 0;
  virtual void init(uint32_t n, const uint32_t* offsets, const uint32_t* neighbors, uint64_t nnz,
                    const float* xyz) = 0;
  virtual void reinit(uint32_t n, const uint32_t* offsets, const uint32_t* neighbors, uint64_t nnz,
                      const float* xyz) {
    init(n, offsets, neighbors, nnz, xyz);
  }
  // reinit with positions already in device memory (3n floats, complete
  // before the call). The default stages them through the host.
  virtual void reinit_device(uint32_t n, const uint32_t* offsets, const uint32_t* neighbors, uint64_t nnz,
                             const float* d_xyz);
  // Nodes of the positions the last step / positions() wrote: n_nodes for a
  // leaf engine, the current cascade level's count for the multilevel one.
  virtual uint32_t output_nodes() const { return node_count(); }
  virtual void step(float* out_xyz) = 0;
  virtual void step_many(uint32_t iters, float* out_xyz) = 0;
  virtual void apply_halo(uint64_t, uint32_t, const uint32_t*, const float*, uint32_t) {}
  virtual bool is_halted() const { return false; }

  virtual void positions(float* out_xyz) = 0;
  // Positions of nodes [first, first + count) (3 floats each).
  virtual void positions_range(uint64_t, uint64_t, float*) { fail(JC_ERR_ARG, "this engine reads all positions"); }
  virtual void forces(float*, float*) { fail(JC_ERR_ARG, "this engine has no force vector"); }
  virtual void speed(float*, float*) { fail(JC_ERR_ARG, "this engine has no adaptive speed"); }
  virtual uint32_t status_bits() { return 0; }
  virtual void tree_info(uint32_t*) { fail(JC_ERR_ARG, "this engine builds no tree"); }
  virtual void walk_counts(uint64_t*) { fail(JC_ERR_ARG, "this engine walks no tree"); }
  virtual void init_batch(uint32_t, const uint32_t*, const uint32_t*, const uint32_t*, const float*) {
    fail(JC_ERR_ARG, "this engine lays out one graph at a time");
  }
  virtual void graph_speed(uint32_t, float*, float*) { fail(JC_ERR_ARG, "this engine has no adaptive speed"); }
  virtual uint32_t autotune(uint32_t, float*) { fail(JC_ERR_ARG, "this engine has no schedules to tune"); }
  // Batch schedule in use (1 = one CTA per graph) and the autotuner's timing
  // of that schedule (ms per step, 0 when it was not probed).
  virtual void schedule_info(uint32_t* tile, float* tile_ms) {
    if (tile) *tile = 0;
    if (tile_ms) *tile_ms = 0.0f;
  }
  virtual void stress(double*, double*) { fail(JC_ERR_ARG, "this engine has no pivot distances"); }
  virtual uint32_t pivots(uint32_t*, uint32_t*) { fail(JC_ERR_ARG, "this engine has no pivot distances"); }
  virtual void time_steps(uint32_t iters, float* total_ms, float* phase_ms4) = 0;
  virtual uint32_t launches_per_step() const = 0;
  // Frame streaming (jc_engine_stream_*): steps enqueued on the engine's
  // stream without a host wait, the positions left in device memory (3n
  // floats written by the last enqueued step) for the frame encoder, and the
  // device word that a failed step sets.
  virtual uint32_t node_count() const = 0;
  virtual void enqueue_steps(uint32_t) { fail(JC_ERR_ARG, "this engine does not stream frames"); }
  virtual const float* device_xyz() const { return nullptr; }
  virtual cudaStream_t cuda_stream() const { return nullptr; }
  // A second stream of the engine for copies that overlap its steps (the
  // frame stream's device-to-host copies); null: the caller finds its own.
  virtual cudaStream_t copy_stream() const { return nullptr; }
  virtual const uint32_t* device_error_word() const { return nullptr; }
  // After a streamed step failed on the device: wait, clear the device
  // error (growing buffers where that is the remedy) and throw it.
  virtual void after_stream_error() {}
  virtual uint64_t state_size() = 0;
  virtual void save_state(void* buf) = 0;
  virtual void load_state(const void* buf, uint64_t len) = 0;

  std::string last_error;
};

// Validates a CSR handed across the ABI (offsets monotone, offsets[n] ==
// nnz, neighbour ids in range). The reference indexes these arrays
// unchecked; out-of-range ids would be device out-of-bounds reads here.
void validate_csr(uint32_t n, const uint32_t* offsets, const uint32_t* neighbors, uint64_t nnz,
                  const float* xyz);
void validate_csr_arrays(uint32_t n, const uint32_t* offsets, const uint32_t* neighbors, uint64_t nnz);
// The offset checks of validate_csr_arrays alone (no pass over the ids).
void validate_csr_offsets(uint32_t n, const uint32_t* offsets, const uint32_t* neighbors, uint64_t nnz);

Engine* make_fa2_engine(bool barnes_hut);
Engine* make_multilevel_engine();
// Multilevel read-outs; false when `e` is not the multilevel engine (or l is
// not a level of its cascade). edges / parent_map may be null (sizes only).
bool multilevel_level_info(Engine* e, uint32_t* level, uint32_t* n_levels, uint32_t* sweeps_done);
bool multilevel_level_get(Engine* e, uint32_t l, uint32_t* n_nodes, uint64_t* n_edge_words, uint32_t* edges,
                          uint32_t* parent_map);
// The matching cascade on its own (host only).
void* cascade_build(uint32_t n, const uint32_t* edges, uint64_t n_words, uint64_t max_levels, uint64_t target_size);
uint32_t cascade_count(const void* h);
bool cascade_get(const void* h, uint32_t l, uint32_t* n_nodes, uint64_t* n_edge_words, uint32_t* edges,
                 uint32_t* parent_map);
void cascade_free(void* h);
Engine* make_sgd_engine(bool jacobi);

}  // namespace jc
