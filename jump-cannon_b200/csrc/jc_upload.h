// Host -> device uploads of large pageable arrays (engine init).
//
// A copy from pageable memory goes through the driver's own staging on one
// host thread. Here every host thread copies its share of a chunk into a
// small page-locked ring while the copy engine moves the previous chunk, so
// the host side runs at memory bandwidth and overlaps the DMA; the id upload
// also checks, in the same pass over the data, that every neighbour id is
// below the node count (the host validation this replaces read the array
// once more). One ring per process, held until exit, shared by all engines
// under a mutex (init is not a hot path; steps never use it).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "jc_common.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace jc {

class HostStager {
 public:
  static constexpr size_t kChunk = (size_t)8 << 20;  // bytes per ring slot

  // Created on first use and never destroyed: the page-locked ring lives
  // until the process exits (no CUDA call from a static destructor).
  static HostStager& instance() {
    static HostStager* s = new HostStager();
    return *s;
  }

  // bytes from host `src` to device `dst` on stream `s`; returns after the
  // last chunk is staged (its DMA may still be in flight on `s`).
  void upload(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    std::lock_guard<std::mutex> lock(mu_);
    run(dst, src, bytes, s, nullptr, 0);
  }

  // n u32 values from `src` to `dst`; returns the largest value (0 if n == 0).
  uint32_t upload_u32_max(uint32_t* dst, const uint32_t* src, uint64_t n, cudaStream_t s) {
    std::lock_guard<std::mutex> lock(mu_);
    uint32_t mx = 0;
    run(dst, src, n * sizeof(uint32_t), s, &mx, 1);
    return mx;
  }

 private:
  HostStager() = default;

  void ensure() {
    for (int k = 0; k < 2; ++k) {
      if (!buf_[k]) JC_CUDA_CHECK(cudaHostAlloc((void**)&buf_[k], kChunk, cudaHostAllocDefault));
      if (!ev_[k]) JC_CUDA_CHECK(cudaEventCreateWithFlags(&ev_[k], cudaEventDisableTiming));
    }
  }

  // Copies chunk by chunk; with `mx`, also reduces the max of the u32 words.
  void run(void* dst, const void* src, size_t bytes, cudaStream_t s, uint32_t* mx, int words) {
    if (bytes == 0) return;
    ensure();
    // Every slot's previous copy (an earlier upload, maybe on another
    // stream) must have left the slot before it is refilled.
    for (int k = 0; k < 2; ++k)
      if (used_[k]) JC_CUDA_CHECK(cudaEventSynchronize(ev_[k]));
    const uint8_t* in = static_cast<const uint8_t*>(src);
    uint8_t* out = static_cast<uint8_t*>(dst);
    uint32_t best = 0;
    size_t done = 0;
    int slot = 0;
    while (done < bytes) {
      const size_t len = std::min(kChunk, bytes - done);
      if (used_[slot]) JC_CUDA_CHECK(cudaEventSynchronize(ev_[slot]));
      uint8_t* stage = buf_[slot];
      const uint8_t* from = in + done;
      // equal shares per thread, cut at 4-byte boundaries
      const int64_t units = (int64_t)(len / 4), tail = (int64_t)(len % 4);
      uint32_t cmax = 0;
#pragma omp parallel reduction(max : cmax)
      {
#ifdef _OPENMP
        const int64_t T = omp_get_num_threads(), t = omp_get_thread_num();
#else
        const int64_t T = 1, t = 0;
#endif
        const int64_t a = units * t / T, b = units * (t + 1) / T;
        std::memcpy(stage + 4 * a, from + 4 * a, (size_t)(4 * (b - a)));
        if (words) {
          const uint32_t* w = reinterpret_cast<const uint32_t*>(stage) + a;
          uint32_t m = 0;
          for (int64_t k = 0; k < b - a; ++k) m = std::max(m, w[k]);
          cmax = std::max(cmax, m);
        }
      }
      if (tail) std::memcpy(stage + 4 * units, from + 4 * units, (size_t)tail);
      best = std::max(best, cmax);
      JC_CUDA_CHECK(cudaMemcpyAsync(out + done, stage, len, cudaMemcpyHostToDevice, s));
      JC_CUDA_CHECK(cudaEventRecord(ev_[slot], s));
      used_[slot] = true;
      done += len;
      slot ^= 1;
    }
    if (mx) *mx = best;
  }

  std::mutex mu_;
  uint8_t* buf_[2] = {nullptr, nullptr};
  cudaEvent_t ev_[2] = {nullptr, nullptr};
  bool used_[2] = {false, false};
};

}  // namespace jc
