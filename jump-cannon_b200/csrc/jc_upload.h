// Host -> device uploads of large pageable arrays (engine init).
//
// A copy from pageable memory goes through the driver's own staging on one
// host thread. Here every host thread copies its share of a chunk into a
// small page-locked ring while the copy engine moves the previous chunk, so
// the host side runs at memory bandwidth and overlaps the DMA; the id upload
// also checks, in the same pass over the data, that every neighbour id is
// below the node count (the host validation this replaces read the array
// once more). One stager per process, shared by all engines under a mutex
// (init is not a hot path; steps never use it); its two slots are borrowed
// from the process's pinned-block cache for each upload.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "jc_common.h"

#ifdef _OPENMP
#include <omp.h>
#endif
#if defined(__x86_64__)
#include <immintrin.h>
#endif

namespace jc {

#if defined(__x86_64__)
// Copies n u32 words into page-locked memory (dst 32-byte aligned) with
// streaming stores, so the staged lines are written without first being read
// into this core's caches (the copy engine reads them next, not this core);
// returns the largest word when want_max is set.
__attribute__((target("avx2"))) inline uint32_t stage_u32_stream(uint32_t* dst, const uint32_t* src, int64_t n,
                                                                  bool want_max) {
  __m256i m = _mm256_setzero_si256();
  int64_t k = 0;
  for (; k + 16 <= n; k += 16) {
    const __m256i v0 = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(src + k));
    const __m256i v1 = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(src + k + 8));
    if (want_max) m = _mm256_max_epu32(m, _mm256_max_epu32(v0, v1));
    _mm256_stream_si256(reinterpret_cast<__m256i*>(dst + k), v0);
    _mm256_stream_si256(reinterpret_cast<__m256i*>(dst + k + 8), v1);
  }
  _mm_sfence();
  alignas(32) uint32_t r[8];
  _mm256_store_si256(reinterpret_cast<__m256i*>(r), m);
  uint32_t best = 0;
  for (int j = 0; j < 8; ++j) best = std::max(best, r[j]);
  for (; k < n; ++k) {
    dst[k] = src[k];
    best = std::max(best, src[k]);
  }
  return want_max ? best : 0u;
}
inline bool cpu_has_avx2() {
  static const bool has = __builtin_cpu_supports("avx2");
  return has;
}
#endif

// Page-locked host blocks, kept for reuse once given back: pinning takes
// milliseconds per 10 MB, so the init stager's ring and the frame streams'
// slots come from here and return here. take() hands out the smallest kept
// block of at least `bytes` (or pins a new one); at most kKeep blocks are
// kept, the rest are unpinned. Portable, so a block serves any device. A
// block is given back only when no copy in flight touches it.
class PinnedCache {
 public:
  static PinnedCache& instance() {
    static PinnedCache* c = new PinnedCache();
    return *c;
  }
  uint8_t* take(uint64_t bytes, uint64_t* got) {
    {
      std::lock_guard<std::mutex> lock(mu_);
      size_t best = kept_.size();
      for (size_t k = 0; k < kept_.size(); ++k)
        if (kept_[k].second >= bytes && (best == kept_.size() || kept_[k].second < kept_[best].second)) best = k;
      if (best < kept_.size()) {
        uint8_t* p = kept_[best].first;
        *got = kept_[best].second;
        kept_.erase(kept_.begin() + (std::ptrdiff_t)best);
        return p;
      }
    }
    uint8_t* p = nullptr;
    JC_CUDA_CHECK(cudaHostAlloc((void**)&p, bytes, cudaHostAllocPortable));
    *got = bytes;
    return p;
  }
  void give(uint8_t* p, uint64_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(mu_);
    if (kept_.size() < kKeep) {
      kept_.emplace_back(p, bytes);
      return;
    }
    cudaFreeHost(p);
  }

 private:
  static constexpr size_t kKeep = 8;
  std::mutex mu_;
  std::vector<std::pair<uint8_t*, uint64_t>> kept_;
};

// Small page-locked blocks (up to 256 bytes: state mirrors, flags) carved
// from 64 KB page-locked arenas that are kept for the life of the process:
// cudaMallocHost of even a few bytes pins pages and took 1-4 ms per call on
// B200 hosts, which every engine init paid.
class SmallPinned {
 public:
  static constexpr size_t kSlot = 256, kArena = 64 * 1024;
  static SmallPinned& instance() {
    static SmallPinned* s = new SmallPinned();
    return *s;
  }
  void* take(size_t bytes) {
    if (bytes > kSlot) fail(JC_ERR_ARG, "small page-locked block larger than 256 bytes");
    std::lock_guard<std::mutex> lock(mu_);
    if (free_.empty()) {
      uint8_t* a = nullptr;
      JC_CUDA_CHECK(cudaHostAlloc((void**)&a, kArena, cudaHostAllocPortable));
      for (size_t o = 0; o < kArena; o += kSlot) free_.push_back(a + o);
    }
    void* p = free_.back();
    free_.pop_back();
    return p;
  }
  void give(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(mu_);
    free_.push_back(static_cast<uint8_t*>(p));
  }

 private:
  std::mutex mu_;
  std::vector<uint8_t*> free_;
};

// Non-blocking streams of each device, kept for reuse once an engine is done
// with them (creating one took up to a few milliseconds). A stream is given
// back only after its work has completed.
class StreamCache {
 public:
  static StreamCache& instance() {
    static StreamCache* c = new StreamCache();
    return *c;
  }
  cudaStream_t take() {
    int dev = 0;
    JC_CUDA_CHECK(cudaGetDevice(&dev));
    {
      std::lock_guard<std::mutex> lock(mu_);
      for (size_t k = 0; k < kept_.size(); ++k)
        if (kept_[k].second == dev) {
          cudaStream_t s = kept_[k].first;
          kept_.erase(kept_.begin() + (std::ptrdiff_t)k);
          return s;
        }
    }
    cudaStream_t s = nullptr;
    JC_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return s;
  }
  // No exception leaves this call (it runs in destructors).
  void give(cudaStream_t s) {
    if (!s) return;
    int dev = 0;
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess) {
      (void)cudaGetLastError();
      cudaStreamDestroy(s);
      return;
    }
    std::lock_guard<std::mutex> lock(mu_);
    kept_.emplace_back(s, dev);
  }

 private:
  std::mutex mu_;
  std::vector<std::pair<cudaStream_t, int>> kept_;
};

class HostStager {
 public:
  static constexpr size_t kChunk = (size_t)16 << 20;  // bytes per ring slot

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
    Release r{this};
    run(dst, src, bytes, s, nullptr, 0);
  }

  // n u32 values from `src` to `dst`; returns the largest value (0 if n == 0).
  uint32_t upload_u32_max(uint32_t* dst, const uint32_t* src, uint64_t n, cudaStream_t s) {
    std::lock_guard<std::mutex> lock(mu_);
    Release r{this};
    uint32_t mx = 0;
    run(dst, src, n * sizeof(uint32_t), s, &mx, 1);
    return mx;
  }

 private:
  HostStager() = default;

  // The ring's two slots come from the pinned cache for the length of one
  // upload and go back to it (after their copies completed) when it ends, so
  // that a frame stream opened afterwards can take them.
  void ensure() {
    for (int k = 0; k < 2; ++k) {
      if (!buf_[k]) {
        uint64_t got = 0;
        buf_[k] = PinnedCache::instance().take(kChunk, &got);
      }
      if (!ev_[k]) JC_CUDA_CHECK(cudaEventCreateWithFlags(&ev_[k], cudaEventDisableTiming));
    }
  }
  void hand_back() {
    for (int k = 0; k < 2; ++k) {
      if (used_[k]) cudaEventSynchronize(ev_[k]);
      used_[k] = false;
      PinnedCache::instance().give(buf_[k], kChunk);
      buf_[k] = nullptr;
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
      // equal shares per thread, cut at 64-byte boundaries of the slot
      const int64_t units = (int64_t)(len / 4), tail = (int64_t)(len % 4);
      uint32_t cmax = 0;
#pragma omp parallel reduction(max : cmax)
      {
#ifdef _OPENMP
        const int64_t T = omp_get_num_threads(), t = omp_get_thread_num();
#else
        const int64_t T = 1, t = 0;
#endif
        const int64_t a = t == 0 ? 0 : (units * t / T) & ~(int64_t)15;
        const int64_t b = t == T - 1 ? units : (units * (t + 1) / T) & ~(int64_t)15;
        bool done_here = false;
#if defined(__x86_64__)
        if (cpu_has_avx2() && b > a && (reinterpret_cast<uintptr_t>(stage) & 31u) == 0) {
          const uint32_t m = stage_u32_stream(reinterpret_cast<uint32_t*>(stage) + a,
                                              reinterpret_cast<const uint32_t*>(from) + a, b - a, words != 0);
          cmax = std::max(cmax, m);
          done_here = true;
        }
#endif
        if (!done_here && b > a) {
          std::memcpy(stage + 4 * a, from + 4 * a, (size_t)(4 * (b - a)));
          if (words) {
            const uint32_t* w = reinterpret_cast<const uint32_t*>(stage) + a;
            uint32_t m = 0;
            for (int64_t k = 0; k < b - a; ++k) m = std::max(m, w[k]);
            cmax = std::max(cmax, m);
          }
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

  struct Release {  // the slots go back to the cache however run() ends
    HostStager* h;
    ~Release() { h->hand_back(); }
  };
  std::mutex mu_;
  uint8_t* buf_[2] = {nullptr, nullptr};
  cudaEvent_t ev_[2] = {nullptr, nullptr};
  bool used_[2] = {false, false};
};

}  // namespace jc
