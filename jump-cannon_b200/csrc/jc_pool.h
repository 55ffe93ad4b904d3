// Device memory of the layout engines: blocks from cudaMalloc that go back
// to a per-device cache when an engine frees them, and are handed to the
// next engine that asks for a block of about the same size.
//
// An engine's buffers are large (about 0.45 GB for the 1M-node R-MAT graph)
// and a process often builds engines one after another (a graph swap, a
// level of the multilevel wrapper, a batch per superstep). Measured on B200:
// the buffers of a fresh engine took 10-94 ms of cudaMalloc once other
// engines had come and gone (most of jc_engine_init), a CUDA memory pool
// with an unlimited release threshold 0.13 ms when it held the blocks but
// 460 ms when it had to grow. Here a miss is a plain cudaMalloc (the cold
// path stays as fast as before) and a freed block is kept: a request takes
// the smallest cached block of the same device that is at least as large and
// at most twice as large. The cache keeps what the process freed, up to the
// peak it used, until the process exits.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "jc_common.h"

namespace jc {

class DevicePool {
 public:
  static DevicePool& instance() {
    static DevicePool* p = new DevicePool();
    return *p;
  }

  void* alloc(size_t bytes) {
    int dev = 0;
    JC_CUDA_CHECK(cudaGetDevice(&dev));
    {
      std::lock_guard<std::mutex> lock(mu_);
      size_t best = free_.size();
      for (size_t k = 0; k < free_.size(); ++k) {
        const Block& b = free_[k];
        if (b.device == dev && b.bytes >= bytes && b.bytes <= 2 * bytes &&
            (best == free_.size() || b.bytes < free_[best].bytes))
          best = k;
      }
      if (best < free_.size()) {
        const Block b = free_[best];
        free_.erase(free_.begin() + (std::ptrdiff_t)best);
        used_.push_back(b);
        return b.p;
      }
    }
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      // out of memory: give the cached blocks of this device back, retry once
      (void)cudaGetLastError();
      release_cached(dev);
      JC_CUDA_CHECK(cudaMalloc(&p, bytes));
    }
    std::lock_guard<std::mutex> lock(mu_);
    used_.push_back(Block{p, bytes, dev});
    return p;
  }

  // Back to the cache once the device has finished with it (the
  // synchronisation cudaFree would have made). No exception leaves this call
  // (it runs in destructors).
  void free(void* p) {
    if (!p) return;
    Block b{};
    {
      std::lock_guard<std::mutex> lock(mu_);
      size_t k = 0;
      while (k < used_.size() && used_[k].p != p) ++k;
      if (k == used_.size()) return;
      b = used_[k];
      used_.erase(used_.begin() + (std::ptrdiff_t)k);
    }
    int cur = 0;
    const bool other = cudaGetDevice(&cur) == cudaSuccess && cur != b.device;
    if (other) cudaSetDevice(b.device);
    cudaDeviceSynchronize();
    if (other) cudaSetDevice(cur);
    (void)cudaGetLastError();
    std::lock_guard<std::mutex> lock(mu_);
    free_.push_back(b);
  }

 private:
  void release_cached(int dev) {
    std::vector<void*> drop;
    {
      std::lock_guard<std::mutex> lock(mu_);
      for (size_t k = 0; k < free_.size();) {
        if (free_[k].device == dev) {
          drop.push_back(free_[k].p);
          free_.erase(free_.begin() + (std::ptrdiff_t)k);
        } else {
          ++k;
        }
      }
    }
    for (void* q : drop) cudaFree(q);
  }

  struct Block {
    void* p;
    size_t bytes;
    int device;
  };
  std::mutex mu_;
  std::vector<Block> free_, used_;
};

}  // namespace jc
