// Edge-cut partitions of a CSR graph with ghost tables
// (crates/graph-compute/src/partition.rs), the units that the batched engine
// lays out together: every partition's local graph (owned nodes, then
// read-only ghosts) becomes one graph of a batch.
#pragma once

#include <cstdint>
#include <vector>

namespace jc {

struct PartitionPart {
  uint32_t id = 0;
  uint32_t n_owned = 0;
  std::vector<uint32_t> offsets{0};   // local CSR over [0, n_local)
  std::vector<uint32_t> neighbors;
  std::vector<uint32_t> global_ids;   // local index -> global id (owned first)
  std::vector<uint32_t> boundary;     // owned global ids that are some peer's ghost, ascending
  uint32_t n_local() const { return (uint32_t)global_ids.size(); }
};

struct PartitionSet {
  uint32_t n_nodes = 0;
  uint32_t n_partitions = 1;
  std::vector<uint32_t> owner;  // owner[global id] -> partition id
  std::vector<PartitionPart> parts;
  uint64_t edge_cut = 0;
};

// partition_csr (partition.rs:191-221); with refine, partition_csr_refined
// (partition.rs:510-516: the BFS cut, then refine_partitions :550-643).
PartitionSet partition_csr(uint32_t n, const uint32_t* offsets, const uint32_t* neighbors, uint32_t n_partitions,
                           bool refine);

}  // namespace jc

#include "jc_engine.h"

namespace jc {

// Device maps of an engine that was bound to a PartitionSet as a batch (one
// graph per partition, in partition order): where each global node's owned
// copy sits among the batch's nodes, and each partition's boundary slots.
class PartitionLayout {
 public:
  PartitionLayout(Engine* engine, const PartitionSet& ps);
  ~PartitionLayout();
  PartitionLayout(const PartitionLayout&) = delete;
  PartitionLayout& operator=(const PartitionLayout&) = delete;

  // Owned positions of every partition at their global ids (3*n floats).
  void owned_positions(float* global_xyz);
  // Partition p's boundary positions, parallel to its boundary ids
  // (boundary_delta, partition.rs:116-158).
  void halo_delta(uint32_t p, float* out_xyz);
  uint32_t n_partitions() const { return (uint32_t)bnd_off_.size() - 1; }
  uint32_t boundary_count(uint32_t p) const { return bnd_off_[p + 1] - bnd_off_[p]; }

 private:
  void release();
  Engine* eng_;
  uint32_t n_ = 0;
  std::vector<uint32_t> bnd_off_;
  uint32_t* d_owned_slot_ = nullptr;     // [n]: batch slot of global g's owned copy
  uint32_t* d_boundary_slot_ = nullptr;  // [sum of boundary sizes]
  float* d_out_ = nullptr;               // [3 * max(n, largest boundary)]
};

}  // namespace jc
