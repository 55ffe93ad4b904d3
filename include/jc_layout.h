/*
 * jc_layout.h — C ABI of the B200 layout-step engine (libjc_layout.so).
 *
 * The reference's drop-in boundary is the Rust trait `LayoutEngine`
 * (crates/graph-compute/src/engines/mod.rs:383-444) with the engine ids
 * registered in `construct_leaf` (mod.rs:477-488). Every entry point below
 * replaces one trait method or registry call for the engines on the layout
 * hot path: "fa2-bh" (engines/fa2_bh.rs), "fa2-brute" (engines/fa2_brute.rs),
 * "sgd-stress" (engines/sgd_stress.rs) and "sgd-stress-gpu"
 * (engines/sgd_stress_gpu.rs). Plain pointers and sizes only; no C++
 * exceptions cross this boundary.
 *
 * Conventions
 *  - Every call returns a jc_status (0 = ok). On error the engine keeps a
 *    message readable through jc_engine_last_error().
 *  - A handle is not re-entrant: one thread at a time per handle (the
 *    reference's sim loop moves the engine out of its mutex for each step,
 *    crates/graph-compute/src/service.rs:655-693). Different handles may run
 *    concurrently; each owns its CUDA stream, device buffers and graphs.
 *  - Positions are interleaved x,y,z f32, length 3*n_nodes, as on the trait.
 *  - Graphs are CSR: offsets[n_nodes+1], neighbors[offsets[n_nodes]]
 *    (crates/graph-compute/src/sim.rs:20-27 CsrGraph).
 */
#ifndef JC_LAYOUT_H
#define JC_LAYOUT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t jc_status;

#define JC_OK 0
#define JC_ERR_ARG 1             /* bad argument (lengths, null pointers, ranges) */
#define JC_ERR_CUDA 2            /* a CUDA runtime call failed / no device */
#define JC_ERR_CAPACITY 3        /* the octree did not fit its device capacity */
#define JC_ERR_DEVICE_TIMEOUT 4  /* a bounded device loop gave up (malformed tree) */
#define JC_ERR_NONFINITE 5       /* non-finite positions were produced */
#define JC_ERR_STATE 6           /* step before init, or similar lifecycle misuse */
#define JC_ERR_UNKNOWN_ENGINE 7  /* jc_engine_create with an unregistered id */
#define JC_ERR_PARAMS 8          /* set_params: malformed JSON or wrong field type */
#define JC_ERR_BOUNDS 9          /* a device index check failed (bounds-check build only) */

/* Status-word warning bits reported by jc_engine_status_bits(). */
#define JC_WARN_REF_CAPACITY 1u  /* tree exceeded 2n+8 nodes: the reference would
                                    have stopped inserting bodies (fa2_bh.rs:813-819) */
#define JC_WARN_DEPTH_CAP 2u     /* coincident bodies dropped at the depth cap of 32
                                    (fa2_bh.rs:874-922), as the reference does */
#define JC_WARN_NONFINITE 4u     /* some body had a non-finite coordinate */

typedef struct jc_engine jc_engine;

/* Mirrors graph_layouts::LayoutDescriptor (graph-layouts/src/layout/layout_trait.rs:20-42). */
typedef struct jc_descriptor {
  const char* id;
  int32_t kind; /* 0 = Static, 1 = Physics (LayoutKind) */
  const char* display_name;
  const char* description;
  int32_t needs_edges;
  int32_t needs_cpu_positions;
  int32_t needs_gpu_positions_buffer;
} jc_descriptor;

/* ---- registry (engines/mod.rs:455-488 LEAF_ENGINE_IDS / construct_leaf) ---- */

/* Number of engine ids this library provides, and the id at an index. */
uint32_t jc_engine_count(void);
const char* jc_engine_id_at(uint32_t index);

/* construct_leaf(id): a fresh, uninitialized engine. */
jc_status jc_engine_create(const char* engine_id, jc_engine** out);
void jc_engine_destroy(jc_engine* engine);

/* ---- trait methods ---- */

/* LayoutEngine::descriptor (mod.rs:387). Strings stay owned by the library. */
jc_status jc_engine_descriptor(const jc_engine* engine, jc_descriptor* out);

/* LayoutEngine::set_params (mod.rs:394). json_utf8 is a JSON object (or
 * "null" / NULL = keep the current settings). Like serde with
 * #[serde(default)], every field not named is reset to its default and
 * unknown keys are ignored (fa2_bh.rs:212-220); a wrong type is JC_ERR_PARAMS. */
jc_status jc_engine_set_params(jc_engine* engine, const char* json_utf8);

/* LayoutEngine::init (mod.rs:401): bind to a graph and seed positions
 * (3*n_nodes floats). Copies everything; the caller keeps ownership.
 * n_neighbors must equal offsets[n_nodes]. */
jc_status jc_engine_init(jc_engine* engine, uint32_t n_nodes, const uint32_t* offsets,
                         const uint32_t* neighbors, uint64_t n_neighbors,
                         const float* positions_xyz);

/* LayoutEngine::reinit (mod.rs:422-429): re-bind a live engine to another
 * graph, reusing device buffers when they are large enough. */
jc_status jc_engine_reinit(jc_engine* engine, uint32_t n_nodes, const uint32_t* offsets,
                           const uint32_t* neighbors, uint64_t n_neighbors,
                           const float* positions_xyz);

/* Batched layout (fa2-bh): bind many independent graphs at once (the
 * partition subgraphs of crates/graph-compute/src/partition.rs, or any set of
 * small graphs). Graph g has graph_nodes[g] nodes; its CSR (offsets starting
 * at 0, local neighbour ids, graph_nodes[g]+1 offsets) follows the previous
 * graph's in `offsets` / `neighbors`, and its 3*n_g positions follow in
 * positions_xyz. Each graph keeps its own octree and adaptive speed, exactly
 * as if it had its own engine; every launch covers all graphs. step / step_many /
 * positions then work on all graphs' positions concatenated. No counterpart
 * in the reference (which lays out one graph per engine). */
jc_status jc_engine_init_batch(jc_engine* engine, uint32_t n_graphs, const uint32_t* graph_nodes,
                               const uint32_t* offsets, const uint32_t* neighbors,
                               const float* positions_xyz);

/* Batch builder over jc_engine_init_batch, for callers that produce graphs
 * one at a time (a partitioner's subgraphs): create, add graphs, run. No
 * counterpart in the reference. engine_id must be "fa2-bh"; params_json
 * (optional) is passed to jc_engine_set_params. */
typedef struct jc_batch jc_batch;
jc_status jc_batch_create(const char* engine_id, const char* params_json, jc_batch** out);
void jc_batch_destroy(jc_batch* batch);
const char* jc_batch_last_error(const jc_batch* batch);
/* Copies one graph (CSR with local ids, offsets[0] = 0, offsets[n_nodes] =
 * n_neighbors, n_nodes >= 1) and its 3*n_nodes seed positions; *index
 * (optional) receives its index in the batch. JC_ERR_STATE once the batch is
 * bound. */
jc_status jc_batch_add_graph(jc_batch* batch, uint32_t n_nodes, const uint32_t* offsets,
                             const uint32_t* neighbors, uint64_t n_neighbors, const float* positions_xyz,
                             uint32_t* index);
/* Binds the added graphs (jc_engine_init_batch); jc_batch_run binds on its
 * first call when this was not called. JC_ERR_STATE with no graphs. */
jc_status jc_batch_bind(jc_batch* batch);
/* `iters` steps of every graph, no readback. */
jc_status jc_batch_run(jc_batch* batch, uint32_t iters);
uint32_t jc_batch_graph_count(const jc_batch* batch);
/* Current positions of one graph (3 * n_nodes floats), read from the device. */
jc_status jc_batch_positions(jc_batch* batch, uint32_t graph, float* out_xyz);
/* The engine the batch is bound to, owned by the batch (NULL for a NULL
 * batch): jc_engine_autotune, checkpoints and frame streams work on it once
 * the batch is bound. */
jc_engine* jc_batch_engine(jc_batch* batch);

/* ---- partition-driven batching (crates/graph-compute/src/partition.rs) ---- */

typedef struct jc_partitions jc_partitions;

/* One partition (partition.rs:54-91 Partition): a local CSR over
 * [0, n_local) with the owned nodes first (ascending global id) and the
 * ghosts after them (first-seen order; their rows are empty), the global id
 * of every local node, and the boundary: owned nodes that are some other
 * partition's ghost, ascending. Pointers stay owned by the partition set. */
typedef struct jc_partition_view {
  uint32_t partition_id;
  uint32_t n_partitions;
  uint32_t n_local;
  uint32_t n_owned;
  uint64_t n_neighbors;
  uint32_t n_boundary;
  const uint32_t* offsets;    /* n_local + 1 */
  const uint32_t* neighbors;  /* n_neighbors, local ids */
  const uint32_t* global_ids; /* n_local */
  const uint32_t* boundary;   /* n_boundary global ids */
} jc_partition_view;

/* partition_csr (partition.rs:191-221): n_partitions balanced BFS regions
 * (:244-293) with their ghost tables (:298-431); with refine != 0,
 * partition_csr_refined (:510-516), which adds the Fiduccia-Mattheyses
 * boundary refinement of refine_partitions (:550-643). Sequential host work,
 * as in the reference. n_partitions 0 is taken as 1. */
jc_status jc_partition_csr(uint32_t n_nodes, const uint32_t* offsets, const uint32_t* neighbors,
                           uint64_t n_neighbors, uint32_t n_partitions, int32_t refine, jc_partitions** out);
void jc_partitions_free(jc_partitions* parts);
uint32_t jc_partitions_count(const jc_partitions* parts);
/* edge_cut (partition.rs:456-477): undirected edges between partitions. */
uint64_t jc_partitions_edge_cut(const jc_partitions* parts);
/* owner[global id] -> partition id (n_nodes entries; NULL for an empty graph). */
const uint32_t* jc_partitions_owner(const jc_partitions* parts);
jc_status jc_partition_get(const jc_partitions* parts, uint32_t index, jc_partition_view* out);

/* Binds an fa2-bh engine to every partition's local graph at once, as the
 * graphs of one batch in partition order (jc_engine_init_batch), seeded from
 * the global positions (3*n_nodes floats) by global id. Each partition then
 * evolves exactly as the reference's worker engine on that partition
 * (run_superstep_local, partition.rs:1099-1136: FA2 engines keep the default
 * no-op apply_halo, so ghosts move with their partition's layout). */
jc_status jc_engine_init_partitions(jc_engine* engine, const jc_partitions* parts, const float* global_xyz);

/* The coordinator's view after a superstep: every partition's owned
 * positions written at their global ids (3*n_nodes floats), gathered on the
 * device and copied once. */
jc_status jc_engine_partition_positions(jc_engine* engine, float* global_xyz);

/* Partition p's outgoing HaloDelta payload (boundary_delta,
 * partition.rs:116-158): the positions of its boundary nodes (3*count
 * floats, parallel to jc_partition_view.boundary). *count receives the
 * boundary size; out_xyz may be NULL to query it. */
jc_status jc_engine_halo_delta(jc_engine* engine, uint32_t p, float* out_xyz, uint32_t* count);

/* Adaptive speed state of one graph of a batch (graph 0 of a single graph). */
jc_status jc_engine_graph_speed(jc_engine* engine, uint32_t graph, float* speed,
                                float* speed_efficiency);

/* Autotuner: times probe_steps steps of each walk schedule (lanes sharing a
 * node stream: 1, 2, 4, 8, 16, 32) from one device snapshot of the state,
 * restores the state after each, and keeps the fastest. Writes the chosen
 * group size and, if ms6 is not NULL, the measured ms per step of each. */
jc_status jc_engine_autotune(jc_engine* engine, uint32_t probe_steps, uint32_t* walk_group,
                             float* ms6);

/* Batch schedule (no reference counterpart). A batch runs either as one
 * forest per launch (every kernel covers all graphs) or with one CTA per
 * graph in a persistent launch that runs all requested iterations; the
 * second is eligible when no attraction list reaches hub_threshold. The
 * setting "batch_schedule" (0 forest, 1 CTA per graph) chooses it, and
 * jc_engine_autotune also times it and keeps it when it is faster. Writes
 * whether the CTA-per-graph schedule is in use and the autotuner's ms per
 * step for it (0 when it was not probed). Results are identical either way. */
jc_status jc_engine_batch_schedule(jc_engine* engine, uint32_t* tile_schedule, float* tile_ms_per_step);

/* LayoutEngine::step (mod.rs:433): advance one tick and write the owned
 * positions (3*n_nodes floats) into out_xyz. For the fastest transfer pass
 * page-locked host memory. */
jc_status jc_engine_step(jc_engine* engine, float* out_xyz);

/* Advance `iters` ticks back to back (replayed from a captured CUDA graph)
 * and, if out_xyz is not NULL, read the final positions once. Equivalent to
 * `iters` calls of jc_engine_step without the intermediate readbacks. */
jc_status jc_engine_step_many(jc_engine* engine, uint32_t iters, float* out_xyz_or_null);

/* LayoutEngine::apply_halo (mod.rs:437): no-op for single-worker engines,
 * kept for interface completeness. */
jc_status jc_engine_apply_halo(jc_engine* engine, uint64_t frame, uint32_t owner_id,
                               const uint32_t* node_ids, const float* positions_xyz,
                               uint32_t count);

/* ---- position frames (the sim loop's per-tick PositionDelta,
 *      crates/graph-compute/proto/compute.proto:84-91, produced without a
 *      host wait per step) ---- */

#define JC_FRAME_F32 0u       /* payload: raw LE f32 x,y,z = PositionDelta.positions */
#define JC_FRAME_F16_DELTA 1u /* payload: LE binary16 differences from the receiver's
                                 reconstruction (see jc_frame_decode) */

/* One frame message: a 64-byte little-endian header (u32 magic "JCF1",
 * u32 encoding, u64 frame, u32 n_nodes, u32 0, u64 payload_bytes, 32 zero
 * bytes) followed by the payload. `data`/`bytes` cover the whole message. */
typedef struct jc_frame {
  uint64_t frame;          /* 0, 1, 2, ... since jc_engine_stream_open */
  uint32_t n_nodes;
  uint32_t encoding;       /* JC_FRAME_F32 or JC_FRAME_F16_DELTA */
  const uint8_t* data;     /* header + payload, in library-owned page-locked memory */
  uint64_t bytes;
  const uint8_t* payload;  /* data + 64 */
  uint64_t payload_bytes;  /* 12*n_nodes (f32) or 6*n_nodes (f16) */
} jc_frame;

/* Opens a frame stream on an initialized engine (replacing any open one):
 * a ring of `depth` (1..8) slots of page-locked host memory. With
 * JC_FRAME_F16_DELTA, frame 0, every keyframe_interval-th frame (0 = none)
 * and any frame whose differences do not fit binary16 are sent as f32.
 * init / reinit / init_batch / load_state close the stream. */
jc_status jc_engine_stream_open(jc_engine* engine, uint32_t encoding, uint32_t depth,
                                uint32_t keyframe_interval);

/* Enqueues `iters` steps and the frame of the positions after them, and
 * returns without waiting for the GPU: the copy of this frame to the host
 * overlaps the steps of the next call. Fails with JC_ERR_STATE when `depth`
 * frames are pending (take one with jc_engine_stream_next first). */
jc_status jc_engine_stream_step(jc_engine* engine, uint32_t iters);

/* Waits for the oldest pending frame and describes it. The memory stays
 * valid until the stream_step call that reuses its slot: frame k lives
 * until call number k + depth of jc_engine_stream_step (counting from 0).
 * A device error in the frame's steps stops the stream and is returned
 * here (the engine's buffers are grown on JC_ERR_CAPACITY; reopen). */
jc_status jc_engine_stream_next(jc_engine* engine, jc_frame* out);

jc_status jc_engine_stream_close(jc_engine* engine);

/* Host decoder: keeps the f32 reconstruction r of one receiver. An f32 frame
 * sets r to its payload; a delta frame (the next frame number after the
 * previous one decoded) adds each binary16 value, converted exactly, to r in
 * f32. The encoder computes the same r, so the decoded positions differ from
 * the engine's by the rounding of the latest difference only (at most half a
 * binary16 unit of that difference). out_xyz (3*n_nodes floats) may be NULL. */
typedef struct jc_frame_decoder jc_frame_decoder;
jc_frame_decoder* jc_frame_decoder_create(uint32_t n_nodes);
void jc_frame_decoder_destroy(jc_frame_decoder* decoder);
jc_status jc_frame_decode(jc_frame_decoder* decoder, const uint8_t* data, uint64_t bytes, float* out_xyz);
const char* jc_frame_decoder_last_error(const jc_frame_decoder* decoder);

/* LayoutEngine::is_halted (mod.rs:441): always 0 for these engines. */
int32_t jc_engine_is_halted(const jc_engine* engine);

/* Message for the last failed call on this handle ("" if none). */
const char* jc_engine_last_error(const jc_engine* engine);

/* ---- state save / resume (the reference has none: positions are its only
 *      resumable state, compute.proto:42-46) ---- */

/* Serialize the full engine state (positions, previous forces, adaptive
 * speed -- every graph's for a batch --, sweep counter, RNG). Call with
 * buf == NULL to get the size. */
jc_status jc_engine_save_state(jc_engine* engine, void* buf, uint64_t capacity,
                               uint64_t* needed);
jc_status jc_engine_load_state(jc_engine* engine, const void* buf, uint64_t len);

/* ---- read-outs used by tests and the benchmark ---- */

/* Positions as of the last completed step (3*n floats). */
jc_status jc_engine_positions(jc_engine* engine, float* out_xyz);

/* FA2 engines: the force vector F_t of the last step (3*n floats) and the
 * per-node (deg*swing, deg*traction) pairs (2*n floats; may be NULL). */
jc_status jc_engine_forces(jc_engine* engine, float* out_xyz, float* out_stats2);

/* FA2 engines: adaptive speed state (speed, speed_efficiency). */
jc_status jc_engine_speed(jc_engine* engine, float* speed, float* speed_efficiency);

/* Accumulated warning bits (JC_WARN_*) since init; reading clears them. */
uint32_t jc_engine_status_bits(jc_engine* engine);

/* FA2-BH: facts about the last tree: [0] nodes, [1] bodies in the tree,
 * [2] max depth, [3] bodies dropped at the depth cap. */
jc_status jc_engine_tree_info(jc_engine* engine, uint32_t* out4);

/* FA2-BH: per-step interaction counters of the last step: [0] accepted
 * cells + leaf interactions, [1] opened cells (summed over all bodies). */
jc_status jc_engine_walk_counts(jc_engine* engine, uint64_t* out2);

/* SGD engines: stress of the current layout over the engine's (node, pivot)
 * terms, raw and scale-normalized (crates/graph-layouts/src/metrics.rs:31-76). */
/* SGD engines: the pivots (k ids) and their hop distances (k x n, pivot-major,
 * 0xFFFFFFFF = unreachable); *k receives k. pivots / dist may be NULL (read k
 * first). With "random_pivots" the distances come from the device BFS. */
jc_status jc_engine_pivots(jc_engine* engine, uint32_t* k, uint32_t* pivots, uint32_t* dist);

jc_status jc_engine_stress(jc_engine* engine, double* raw, double* normalized);

/* Device-side timing of `iters` steps replayed from the captured graph:
 * total milliseconds (CUDA events on the engine's stream) and, per kernel
 * phase, the mean milliseconds over up to 10 further synchronised replays of
 * a second capture of the step that holds event nodes between the phases
 * (the timed graph holds none): [0] tree build, [1] walk,
 * [2] attraction+speed, [3] apply. phase_ms may be NULL (no further replays). */
jc_status jc_engine_time_steps(jc_engine* engine, uint32_t iters, float* total_ms,
                               float* phase_ms4);

/* ---- the "multilevel" wrapper (crates/graph-compute/src/engines/multilevel.rs) ----
 * jc_engine_create("multilevel") wraps one of the engines above. Its settings
 * are MultilevelSettings (multilevel.rs:126-203): "inner" (engine id, default
 * "fa2-brute"), "inner_params" (object forwarded to the inner engine),
 * "max_levels" (6), "target_size" (500), "sweeps_per_level" (30),
 * "sweep_schedule" ("uniform" | "linear" (default) | "geometric"),
 * "spring_len" (30.0), "seed" (0x5EED). init coarsens the graph
 * (crates/graph-layouts/src/layout/coarsen.rs) and binds the inner engine to
 * the coarsest level; every step is one inner step, and when a level's sweep
 * budget is spent the positions are prolonged to the next finer level. While
 * descending, step / positions write the current level's positions
 * (jc_engine_output_nodes of them), as the reference's StepOutput does. */

/* The current cascade level (0 = the input graph), the number of levels and
 * the inner steps taken at the current level. */
jc_status jc_engine_level_info(jc_engine* engine, uint32_t* level, uint32_t* n_levels, uint32_t* sweeps_done);

/* Level l of the cascade: its node count, its flat edge list [s,t, s,t, ...]
 * (n_edge_words u32) and its parent map (the previous level's node count of
 * entries; none at level 0). edges / parent_map may be NULL to read sizes. */
jc_status jc_engine_cascade_level(jc_engine* engine, uint32_t l, uint32_t* n_nodes, uint64_t* n_edge_words,
                                  uint32_t* edges, uint32_t* parent_map);

/* The matching cascade alone: graph_layouts::coarsen (coarsen.rs:52-90) of a
 * flat undirected edge list [s,t, s,t, ...] (host only; what the multilevel
 * engine builds at init). */
typedef struct jc_cascade jc_cascade;
jc_status jc_coarsen(uint32_t n_nodes, const uint32_t* edges, uint64_t n_edge_words, uint64_t max_levels,
                     uint64_t target_size, jc_cascade** out);
uint32_t jc_cascade_levels(const jc_cascade* cascade);
jc_status jc_cascade_get(const jc_cascade* cascade, uint32_t l, uint32_t* n_nodes, uint64_t* n_edge_words,
                         uint32_t* edges, uint32_t* parent_map);
void jc_cascade_free(jc_cascade* cascade);

/* Nodes of the positions that step / step_many / positions write (3 floats
 * each): n_nodes of the bound graph (the sum over a batch or partition set);
 * for "multilevel", the current cascade level's node count, which changes
 * when a step moves to a finer level (buffers for the full graph's 3*n_nodes
 * floats always suffice). 0 before init. */
uint32_t jc_engine_output_nodes(const jc_engine* engine);

/* Number of kernel launches one step issues (for launch accounting). */
uint32_t jc_engine_launches_per_step(const jc_engine* engine);

/* ---- synthetic graphs and seeds (crates/graph-compute/src/stability.rs) ---- */

typedef struct jc_csr jc_csr;

/* stability.rs:56-81 synthetic_scale_free(n, m, seed). */
jc_csr* jc_gen_scale_free(uint32_t n, uint32_t m, uint64_t seed);
/* stability.rs:86-110 csr_from_pairs (pairs as 2*count u32). */
jc_csr* jc_csr_from_pairs(uint32_t n, const uint32_t* pairs, uint64_t count);
/* sim.rs:31-49 CsrGraph::path(n). */
jc_csr* jc_gen_path(uint32_t n);
/* 4-neighbour grid in the reference tests' neighbour order
 * (crates/graph-compute/tests/gpu_engines.rs:267-292 grid2d). */
jc_csr* jc_gen_grid(uint32_t width, uint32_t height);
/* R-MAT: 2^scale nodes, sampled until `n_edges` unique undirected non-self
 * edges exist (first-seen order), then csr_from_pairs. */
jc_csr* jc_gen_rmat(uint32_t scale, uint64_t n_edges, double a, double b, double c,
                    uint64_t seed);
/* Watts–Strogatz ring lattice (k neighbours) with rewiring probability p. */
jc_csr* jc_gen_watts_strogatz(uint32_t n, uint32_t k, double p, uint64_t seed);
/* Random geometric graph: n points uniform in [0,1]^2 (written to
 * points_xy if not NULL, 2n floats), edges between points closer than radius. */
jc_csr* jc_gen_rgg(uint32_t n, double radius, uint64_t seed, float* points_xy);

uint32_t jc_csr_n_nodes(const jc_csr* g);
uint64_t jc_csr_n_neighbors(const jc_csr* g);
const uint32_t* jc_csr_offsets(const jc_csr* g);
const uint32_t* jc_csr_neighbors(const jc_csr* g);
void jc_csr_free(jc_csr* g);

/* Seeds: stability.rs:30-49 ball_seed, and the uniform cube/square seed
 * 2*next_f32()-1 per coordinate (dim 2 leaves z = 0). */
void jc_seed_ball(uint32_t n, uint64_t seed, float* out_xyz);
void jc_seed_uniform(uint32_t n, uint32_t dim, uint64_t seed, float* out_xyz);

/* Failure-detection self-test (no reference counterpart): runs one radix-sort
 * pass in which a tile waits on a predecessor tile that never publishes its
 * status. The bounded wait must give up and record JC_ERR_DEVICE_TIMEOUT in
 * the device error word, which is returned in *device_status, and the kernel
 * finishes normally (no fault, no hang; *wait_ms: the pass's duration). */
jc_status jc_selftest_sort_wait(uint32_t* device_status, float* wait_ms);

/* Failure-detection self-test of the tensor-core GEMM's bounded mbarrier
 * waits (no reference counterpart): one CTA sets up tensor memory and an
 * mbarrier as the GEMM kernel does and waits on a phase that no commit ever
 * completes. Every wait must give up after its poll limit, record
 * JC_ERR_DEVICE_TIMEOUT in the device error word (returned in
 * *device_status), free the tensor memory and return (no fault, no hang;
 * *wait_ms: the kernel's duration). */
jc_status jc_selftest_gemm_wait(uint32_t* device_status, float* wait_ms);

/* Library build facts: compute capability the kernels were built for. */
const char* jc_build_info(void);

/* ---- Barnes-Hut force pass without device allocation ---- */

/* Force-law settings of jc_fa2_bh_forces_noalloc (the subset of the
 * fa2-bh settings that shapes F; see jc_engine_set_params for the meaning). */
typedef struct jc_fa2_params {
  float gravity;
  int32_t strong_gravity;
  float scaling_ratio;
  float edge_weight_influence;
  int32_t lin_log_mode;
  float theta;
} jc_fa2_params;

/* No counterpart in the reference: an entry point for callers that cannot
 * call cudaMalloc (a host framework that hands out a fixed device-memory
 * budget, or code where an allocation would synchronise or be refused).
 * Computes the fa2-bh force vector F (3*n floats, repulsion + attraction +
 * gravity with F_old = 0) for positions already on the device, from a CSR
 * already on the device, writing d_forces_xyz.
 * The CSR is used as given: a node's mass is 1 + its non-self entries and
 * its attraction is summed over its row in row order. That equals the
 * fa2-bh engine (and the reference's edge scan, fa2_barnes_hut.wgsl:158-181)
 * only for a canonical CSR: symmetric, no duplicate entries, every row in
 * ascending order (csr_from_pairs form); self-loop entries add no force.
 * The CSR is checked on the device before any gather: decreasing offsets, a
 * neighbour id >= n_nodes, or d_neighbors == NULL with a non-empty row give
 * JC_ERR_ARG and nothing is read through the bad entry (d_neighbors may be
 * NULL when every row is empty). offsets[n_nodes] must not exceed the
 * length of the caller's neighbour array, which cannot be checked here.
 * All scratch memory (keys, sort workspace, octree, partial sums) lives in
 * one static device array sized for n_nodes <= 32768 (about 9 MB, held by
 * every GPU that loads the library until the process exits); larger n is
 * JC_ERR_CAPACITY. The octree has room for 3*32768+64 nodes and does not
 * grow (the engine's does): a layout with deep chains of nearly coincident
 * bodies can need more and then also returns JC_ERR_CAPACITY, even with
 * n_nodes <= 32768. It allocates nothing and calls no cudaMalloc/cudaFree.
 * The first call on a device looks the array up on that device (make that
 * call before any stream capture). Every call reuses the same array, so calls
 * that overlap on the GPU (other streams, other host threads) race; the call
 * is synchronous: it returns after `cuda_stream` has finished the pass.
 * cuda_stream is a cudaStream_t (NULL = the default stream). */
jc_status jc_fa2_bh_forces_noalloc(uint32_t n_nodes, const uint32_t* d_offsets,
                                   const uint32_t* d_neighbors, const float* d_positions_xyz,
                                   const jc_fa2_params* params, float* d_forces_xyz,
                                   void* cuda_stream);

/* Select the CUDA device used by engines created afterwards on this thread
 * (one process per GPU: rank r calls jc_set_device(local_rank)). */
jc_status jc_set_device(int32_t device);

/* ---------------------------------------------------------------------------
 * Learned warm start (no reference counterpart: the reference has no learned
 * layout initialiser). A 3-layer message-passing network, hidden width 128,
 * bf16 weights and activations with f32 accumulation on the tensor cores,
 * maps per-node features (log-degree, 16 random-walk return probabilities,
 * 8 smoothed random projections) to `dim`-D coordinates. It is trained on the
 * GPU with a scale-normalized stress loss against layouts the plain engines
 * produced, and its predictions are centred and scaled per graph to the
 * ForceAtlas2 force balance so that a plain engine can continue from them.
 *
 * Graph sets use the jc_engine_init_batch convention: graph_nodes[g] nodes per
 * graph, `offsets` = the per-graph CSR offset arrays (n_g + 1 entries each)
 * concatenated, `neighbors` = the per-graph neighbour arrays (local ids)
 * concatenated. Graphs must be undirected (every entry (v, u) has its (u, v))
 * without self-loops, as jc_csr_from_pairs produces; otherwise JC_ERR_ARG.
 * ------------------------------------------------------------------------ */
typedef struct jc_mpnn jc_mpnn;
typedef struct jc_eval jc_eval; /* layout quality, below */

/* dim = 2 or 3; seed fixes the initial weights, the feature walks and
 * projections, the partner pairs of the loss and the batch order. */
jc_status jc_mpnn_create(int32_t dim, uint64_t seed, jc_mpnn** out);
void jc_mpnn_destroy(jc_mpnn* m);
const char* jc_mpnn_last_error(const jc_mpnn* m);

/* JSON object, keys optional: lr (1e-3), beta1 (0.9), beta2 (0.999), eps
 * (1e-8), clip (global gradient-norm clip, 1.0; 0 = off), partners (random
 * same-graph pairs per node in the loss, 8), batch_nodes (nodes per
 * training batch of whole graphs, 524288), scaling_ratio (2.0) and gravity
 * (1.0) of the ForceAtlas2 run that continues from a prediction,
 * and the filter of the random projections: cheb_steps (64) steps of the
 * Chebyshev recurrence for the lazy walk's spectrum interval [0, cheb_b]
 * (cheb_b 0.993), then smooth_steps (64) plain lazy random-walk steps. */
jc_status jc_mpnn_set_params(jc_mpnn* m, const char* json_utf8);

/* Size of the flat parameter vector (f32): W0 64x128, b0, W1 256x128, b1,
 * W2 256x128, b2, Wh 128x4, bh 4, padded to a multiple of 8. */
uint32_t jc_mpnn_num_params(void);
jc_status jc_mpnn_get_weights(jc_mpnn* m, float* out);
jc_status jc_mpnn_set_weights(jc_mpnn* m, const float* weights);

/* Bind a training set: graphs plus their target layouts (3 floats per node,
 * z ignored when dim = 2). Computes the features on the device and splits the
 * graphs, in the given order, into batches of at most batch_nodes nodes. */
jc_status jc_mpnn_bind(jc_mpnn* m, uint32_t n_graphs, const uint32_t* graph_nodes, const uint32_t* offsets,
                       const uint32_t* neighbors, const float* target_xyz);
jc_status jc_mpnn_batches(jc_mpnn* m, uint32_t* count);
/* Features of the bound set: n x 32 floats (the bf16 values; columns 25..31 are 0). */
jc_status jc_mpnn_features(jc_mpnn* m, float* out);
/* `steps` Adam steps, one batch each, batches in a seeded order per epoch;
 * losses (optional, `steps` floats) receives each step's batch loss. */
jc_status jc_mpnn_train(jc_mpnn* m, uint32_t steps, float* losses);
/* Mean batch loss over the bound set, no update. */
jc_status jc_mpnn_eval_loss(jc_mpnn* m, double* loss);
/* Forward + loss + backward on graphs [g0, g1) of the bound set with the
 * partner pairs of optimiser step `pair_step`, no update: loss, prediction
 * (4 floats per node, optional) and the unclipped gradient (num_params
 * floats, optional). For gradient checks against a CPU restatement. */
jc_status jc_mpnn_grad(jc_mpnn* m, uint32_t g0, uint32_t g1, uint64_t pair_step, float* loss, float* y,
                       float* grad);
/* Warm start for new graphs: features, forward and the per-graph hand-off
 * scale, written as 3 floats per node (z = 0 when dim = 2). device_ms
 * (optional) receives the device time of those stages. */
jc_status jc_mpnn_predict(jc_mpnn* m, uint32_t n_graphs, const uint32_t* graph_nodes, const uint32_t* offsets,
                          const uint32_t* neighbors, float* out_xyz, float* device_ms);
/* Guarded warm start: jc_mpnn_predict for the graphs `ev` was created on
 * (the same arrays), then per graph the prediction only where its pivot
 * stress (jc_eval, on the device) is below that of the graph's seed in
 * seed_xyz; every other graph gets its seed, so plain ForceAtlas2 from the
 * seed stays the fallback. kept (optional, n_graphs bytes): 1 where the
 * prediction was kept. device_ms (optional): device time of the prediction
 * and both evaluations. JC_ERR_ARG when `ev` was built on other graphs. */
jc_status jc_mpnn_warm_start(jc_mpnn* m, jc_eval* ev, uint32_t n_graphs, const uint32_t* graph_nodes,
                             const uint32_t* offsets, const uint32_t* neighbors, const float* seed_xyz,
                             float* out_xyz, uint8_t* kept, float* device_ms);
/* Device ms of the last jc_mpnn_predict's stages: ms3[0] features, ms3[1]
 * network forward, ms3[2] hand-off scale. */
jc_status jc_mpnn_predict_stages(jc_mpnn* m, float* ms3);
/* Checkpoint: weights, Adam moments, step and batch-order position. */
uint64_t jc_mpnn_state_size(const jc_mpnn* m);
jc_status jc_mpnn_save_state(jc_mpnn* m, void* buf);
jc_status jc_mpnn_load_state(jc_mpnn* m, const void* buf, uint64_t len);

/* Layout quality of a fixed set of graphs on the device: per graph the
 * scale-normalized stress over (node, pivot) pairs with hop distances from
 * n_pivots seeded pivots (crates/graph-layouts/src/metrics.rs:31-59, w =
 * 1/d^2) and the edge-length coefficient of variation (metrics.rs:150-164).
 * No reference counterpart as a device routine: the reference computes these
 * metrics on the host in its tests. */
jc_status jc_eval_create(uint32_t n_graphs, const uint32_t* graph_nodes, const uint32_t* offsets,
                         const uint32_t* neighbors, uint32_t n_pivots, uint64_t seed, jc_eval** out);
void jc_eval_destroy(jc_eval* e);
const char* jc_eval_last_error(const jc_eval* e);
/* Global node ids of each graph's pivots, n_graphs x n_pivots (0xFFFFFFFF = none). */
jc_status jc_eval_pivots(jc_eval* e, uint32_t* out);
/* xyz: 3 floats per node. stress / cv per graph (optional, n_graphs doubles
 * each); means[0] = mean stress over graphs with a pivot pair, means[1] =
 * mean cv over graphs with at least two edges (optional). */
jc_status jc_eval_layout(jc_eval* e, const float* xyz, double* stress_per_graph, double* cv_per_graph,
                         double* means);

/* Test entry point for the tcgen05 bf16 GEMM that the learned warm start
 * runs on: C = A * B with f32 accumulation, from host bf16 bit patterns.
 * A is M x K row-major when a_kmajor, else K x M row-major; B is N x K
 * row-major when b_kmajor, else K x N row-major; C (host, M x N row-major)
 * receives the sum over `splits` split-K partial products. bn is the tile
 * width (128 or 256). staging picks the kernel: 0 automatic (TMA-staged
 * when both operands are K-major with row strides of whole 16-byte units and
 * split-K parts of whole 64-column chunks, else cp.async-staged), 1 the
 * cp.async-staged kernel, 2 the TMA-staged kernel (JC_ERR_ARG when the
 * operands do not suit it). No reference counterpart: the reference has no
 * learned layout initialiser. */
jc_status jc_tc_gemm_bf16(int32_t M, int32_t N, int32_t K, const uint16_t* a_bits, int32_t a_kmajor,
                          const uint16_t* b_bits, int32_t b_kmajor, int32_t bn, int32_t splits,
                          int32_t staging, float* c_out);

#ifdef __cplusplus
}
#endif

#endif /* JC_LAYOUT_H */
