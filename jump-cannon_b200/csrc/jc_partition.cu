// Edge-cut partitions (crates/graph-compute/src/partition.rs) and the device
// maps that turn a batched layout of the partitions back into the
// coordinator's view. The partitioner is sequential host work at bind time,
// as in the reference: BFS region growth is order dependent, and the
// partitions must be the reference's own so that a partition-driven batch
// lays out exactly the graphs that the reference's workers would.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <deque>

#include "jc_common.h"
#include "jc_partition.h"

namespace jc {
namespace {

constexpr uint32_t UNSET = 0xFFFFFFFFu;

// assign_owners_bfs (partition.rs:244-293): P balanced BFS regions of
// ceil(n/P) nodes, each reseeded from the lowest unassigned node whenever its
// frontier drains; the last region takes what remains.
std::vector<uint32_t> assign_owners_bfs(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint32_t p) {
  const uint64_t target = std::max<uint64_t>(((uint64_t)n + p - 1) / p, 1);
  std::vector<uint32_t> owner(n, UNSET);
  uint64_t assigned = 0;
  uint32_t next_seed = 0;
  std::deque<uint32_t> queue;
  for (uint32_t pid = 0; pid < p; ++pid) {
    const uint64_t cap = pid + 1 == p ? UINT64_MAX : target;
    uint64_t count = 0;
    queue.clear();
    while (count < cap && assigned < n) {
      if (queue.empty()) {
        while (next_seed < n && owner[next_seed] != UNSET) ++next_seed;
        if (next_seed >= n) break;
        queue.push_back(next_seed);
        owner[next_seed] = pid;
        ++assigned;
        ++count;
      }
      const uint32_t v = queue.front();
      queue.pop_front();
      for (uint32_t e = off[v]; e < off[v + 1]; ++e) {
        const uint32_t u = nbr[e];
        if (owner[u] == UNSET && count < cap) {
          owner[u] = pid;
          ++assigned;
          ++count;
          queue.push_back(u);
        }
      }
    }
  }
  for (uint32_t& o : owner)
    if (o == UNSET) o = p - 1;
  return owner;
}

// refine_partitions (partition.rs:550-643): single-node Fiduccia-Mattheyses
// moves of nodes in ascending id to the neighbouring partition holding most of
// their neighbours (smallest id on ties) when that strictly lowers the cut
// and keeps every size within 10 % of n/P; at most 8 passes.
void refine_owners(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint32_t p, std::vector<uint32_t>& owner) {
  std::vector<uint64_t> sizes(p, 0);
  for (uint32_t o : owner) sizes[o] += 1;
  const double ideal = (double)n / (double)p;
  const uint64_t max_size = (uint64_t)std::ceil((1.0 + 0.10) * ideal);
  const uint64_t min_size = (uint64_t)std::floor((1.0 - 0.10) * ideal);
  std::vector<uint64_t> ext(p, 0);
  std::vector<uint32_t> touched;
  for (int pass = 0; pass < 8; ++pass) {
    bool moved = false;
    for (uint32_t v = 0; v < n; ++v) {
      const uint32_t a = owner[v];
      uint64_t internal = 0;
      touched.clear();
      for (uint32_t e = off[v]; e < off[v + 1]; ++e) {
        const uint32_t u = nbr[e];
        if (u == v) continue;
        const uint32_t o = owner[u];
        if (o == a) {
          ++internal;
        } else {
          if (ext[o] == 0) touched.push_back(o);
          ext[o] += 1;
        }
      }
      // best destination: the largest external count, smallest id on ties
      uint32_t best = UNSET;
      uint64_t best_ext = 0;
      for (uint32_t b : touched)
        if (ext[b] > best_ext || (ext[b] == best_ext && b < best)) {
          best_ext = ext[b];
          best = b;
        }
      for (uint32_t b : touched) ext[b] = 0;
      if (best == UNSET) continue;
      if ((int64_t)best_ext - (int64_t)internal <= 0) continue;
      if (sizes[best] + 1 > max_size) continue;
      if ((sizes[a] == 0 ? 0 : sizes[a] - 1) < min_size) continue;
      owner[v] = best;
      sizes[a] -= 1;
      sizes[best] += 1;
      moved = true;
    }
    if (!moved) break;
  }
}

// edge_cut_owner (partition.rs:461-477): undirected edges (u < v) whose
// endpoints have different owners.
uint64_t edge_cut_owner(uint32_t n, const uint32_t* off, const uint32_t* nbr, const std::vector<uint32_t>& owner) {
  uint64_t cut = 0;
  for (uint32_t u = 0; u < n; ++u)
    for (uint32_t e = off[u]; e < off[u + 1]; ++e) {
      const uint32_t v = nbr[e];
      if (u < v && owner[u] != owner[v]) ++cut;
    }
  return cut;
}

// build_partitions_from_owner / build_partition (partition.rs:227-236,
// :298-431): owned nodes in ascending id, then ghosts (neighbours owned
// elsewhere) in first-seen order; owned rows keep their whole adjacency
// remapped to local ids, ghost rows are empty; boundary = owned nodes with a
// neighbour owned elsewhere. `local_of` is an all-UNSET scratch map of size n
// and is left all-UNSET.
PartitionPart build_partition(const uint32_t* off, const uint32_t* nbr, const std::vector<uint32_t>& owner,
                              uint32_t pid, std::vector<uint32_t> owned, std::vector<uint32_t>& local_of) {
  PartitionPart part;
  part.id = pid;
  part.n_owned = (uint32_t)owned.size();
  part.global_ids = std::move(owned);
  for (uint32_t li = 0; li < part.n_owned; ++li) local_of[part.global_ids[li]] = li;
  for (uint32_t li = 0; li < part.n_owned; ++li) {
    const uint32_t g = part.global_ids[li];
    bool is_boundary = false;
    for (uint32_t e = off[g]; e < off[g + 1]; ++e) {
      const uint32_t u = nbr[e];
      if (owner[u] != pid) {
        is_boundary = true;
        if (local_of[u] == UNSET) {
          local_of[u] = (uint32_t)part.global_ids.size();
          part.global_ids.push_back(u);
        }
      }
    }
    if (is_boundary) part.boundary.push_back(g);
  }
  const uint32_t n_local = (uint32_t)part.global_ids.size();
  part.offsets.assign(1, 0);
  part.offsets.reserve((size_t)n_local + 1);
  for (uint32_t li = 0; li < n_local; ++li) {
    if (li < part.n_owned) {
      const uint32_t g = part.global_ids[li];
      for (uint32_t e = off[g]; e < off[g + 1]; ++e) part.neighbors.push_back(local_of[nbr[e]]);
    }
    part.offsets.push_back((uint32_t)part.neighbors.size());
  }
  for (uint32_t g : part.global_ids) local_of[g] = UNSET;
  return part;
}

}  // namespace

PartitionSet partition_csr(uint32_t n, const uint32_t* off, const uint32_t* nbr, uint32_t n_partitions, bool refine) {
  PartitionSet ps;
  ps.n_nodes = n;
  ps.n_partitions = std::max(n_partitions, 1u);
  const uint32_t p = ps.n_partitions;
  if (n == 0) {
    ps.parts.resize(p);
    for (uint32_t pid = 0; pid < p; ++pid) ps.parts[pid].id = pid;
    return ps;
  }
  ps.owner = assign_owners_bfs(n, off, nbr, p);
  if (refine && p > 1) refine_owners(n, off, nbr, p, ps.owner);
  std::vector<std::vector<uint32_t>> owned(p);
  for (uint32_t g = 0; g < n; ++g) owned[ps.owner[g]].push_back(g);
  std::vector<uint32_t> local_of(n, UNSET);
  ps.parts.reserve(p);
  for (uint32_t pid = 0; pid < p; ++pid)
    ps.parts.push_back(build_partition(off, nbr, ps.owner, pid, std::move(owned[pid]), local_of));
  ps.edge_cut = edge_cut_owner(n, off, nbr, ps.owner);
  return ps;
}

// ------------------------------------------------------------ device maps --
namespace {

__global__ void k_gather_xyz(const float* __restrict__ xyz, const uint32_t* __restrict__ slot, uint32_t count,
                             float* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint32_t s = slot[i];
  out[3 * (size_t)i] = xyz[3 * (size_t)s];
  out[3 * (size_t)i + 1] = xyz[3 * (size_t)s + 1];
  out[3 * (size_t)i + 2] = xyz[3 * (size_t)s + 2];
}

}  // namespace

PartitionLayout::PartitionLayout(Engine* engine, const PartitionSet& ps) : eng_(engine), n_(ps.n_nodes) {
  const uint32_t p = (uint32_t)ps.parts.size();
  std::vector<uint32_t> owned_slot(n_, 0), bslots;
  bnd_off_.assign(1, 0);
  uint64_t base = 0, max_b = 0;
  for (uint32_t pid = 0; pid < p; ++pid) {
    const PartitionPart& part = ps.parts[pid];
    for (uint32_t li = 0; li < part.n_owned; ++li) owned_slot[part.global_ids[li]] = (uint32_t)(base + li);
    // boundary ids are ascending owned ids; owned ids are ascending too
    uint32_t li = 0;
    for (uint32_t g : part.boundary) {
      while (li < part.n_owned && part.global_ids[li] < g) ++li;
      if (li >= part.n_owned || part.global_ids[li] != g) fail(JC_ERR_ARG, "boundary id not owned");
      bslots.push_back((uint32_t)(base + li));
    }
    bnd_off_.push_back((uint32_t)bslots.size());
    max_b = std::max<uint64_t>(max_b, part.boundary.size());
    base += part.n_local();
  }
  if (base != eng_->node_count()) fail(JC_ERR_STATE, "engine is not bound to this partition set");
  try {
    if (n_) {
      JC_CUDA_CHECK(cudaMalloc((void**)&d_owned_slot_, sizeof(uint32_t) * n_));
      JC_CUDA_CHECK(cudaMemcpy(d_owned_slot_, owned_slot.data(), sizeof(uint32_t) * n_, cudaMemcpyHostToDevice));
      JC_CUDA_CHECK(cudaMalloc((void**)&d_out_, sizeof(float) * 3 * std::max<uint64_t>(n_, max_b)));
    }
    if (!bslots.empty()) {
      JC_CUDA_CHECK(cudaMalloc((void**)&d_boundary_slot_, sizeof(uint32_t) * bslots.size()));
      JC_CUDA_CHECK(cudaMemcpy(d_boundary_slot_, bslots.data(), sizeof(uint32_t) * bslots.size(),
                               cudaMemcpyHostToDevice));
    }
  } catch (...) {
    release();
    throw;
  }
}

PartitionLayout::~PartitionLayout() { release(); }

void PartitionLayout::release() {
  if (d_owned_slot_) cudaFree(d_owned_slot_);
  if (d_boundary_slot_) cudaFree(d_boundary_slot_);
  if (d_out_) cudaFree(d_out_);
  d_owned_slot_ = d_boundary_slot_ = nullptr;
  d_out_ = nullptr;
}

void PartitionLayout::owned_positions(float* global_xyz) {
  if (n_ == 0) return;
  if (!global_xyz) fail(JC_ERR_ARG, "null output");
  cudaStream_t s = eng_->cuda_stream();
  k_gather_xyz<<<(n_ + 255) / 256, 256, 0, s>>>(eng_->device_xyz(), d_owned_slot_, n_, d_out_);
  JC_CUDA_CHECK(cudaGetLastError());
  JC_CUDA_CHECK(cudaMemcpyAsync(global_xyz, d_out_, sizeof(float) * 3 * n_, cudaMemcpyDeviceToHost, s));
  JC_CUDA_CHECK(cudaStreamSynchronize(s));
}

void PartitionLayout::halo_delta(uint32_t p, float* out_xyz) {
  if (p >= n_partitions()) fail(JC_ERR_ARG, "partition index out of range");
  const uint32_t cnt = boundary_count(p);
  if (cnt == 0) return;
  if (!out_xyz) fail(JC_ERR_ARG, "null output");
  cudaStream_t s = eng_->cuda_stream();
  k_gather_xyz<<<(cnt + 255) / 256, 256, 0, s>>>(eng_->device_xyz(), d_boundary_slot_ + bnd_off_[p], cnt, d_out_);
  JC_CUDA_CHECK(cudaGetLastError());
  JC_CUDA_CHECK(cudaMemcpyAsync(out_xyz, d_out_, sizeof(float) * 3 * cnt, cudaMemcpyDeviceToHost, s));
  JC_CUDA_CHECK(cudaStreamSynchronize(s));
}

}  // namespace jc
