// Device memory of the layout engines: one stream-ordered pool per device
// that keeps the blocks it gets back.
//
// An engine's buffers are large (about 0.45 GB for the 1M-node R-MAT graph)
// and a process often builds engines one after another (a graph swap, a
// level of the multilevel wrapper, a batch per superstep). cudaMalloc of a
// fresh engine's buffers took 10-94 ms on B200 when other engines had come
// and gone, most of jc_engine_init. Blocks from a pool whose release
// threshold is unlimited stay mapped after they are freed, so the next
// engine reuses them. The pool grows to the process's peak use and is kept
// until the process exits.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "jc_common.h"

namespace jc {

class DevicePool {
 public:
  static DevicePool& instance() {
    static DevicePool* p = new DevicePool();
    return *p;
  }

  // `bytes` of device memory, usable from any stream when this returns.
  void* alloc(size_t bytes) {
    Slot& s = slot();
    void* p = nullptr;
    JC_CUDA_CHECK(cudaMallocFromPoolAsync(&p, bytes, s.pool, s.stream));
    JC_CUDA_CHECK(cudaStreamSynchronize(s.stream));
    return p;
  }

  // Back to the pool once every stream of the device is done with it (the
  // device-wide synchronisation cudaFree would have made).
  // No exception leaves this call (it runs in destructors).
  void free(void* p) {
    if (!p) return;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess || at.device < 0 || at.device >= kMaxDevices) {
      (void)cudaGetLastError();
      return;
    }
    cudaStream_t st = nullptr;
    {
      std::lock_guard<std::mutex> lock(mu_);
      st = slots_[at.device].stream;
    }
    if (!st) return;
    int cur = 0;
    const bool other = cudaGetDevice(&cur) == cudaSuccess && cur != at.device;
    if (other) cudaSetDevice(at.device);
    cudaDeviceSynchronize();
    cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    if (other) cudaSetDevice(cur);
    (void)cudaGetLastError();
  }

 private:
  struct Slot {
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
  };

  Slot& slot() {
    int dev = 0;
    JC_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) fail(JC_ERR_CUDA, "device index out of range");
    std::lock_guard<std::mutex> lock(mu_);
    Slot& s = slots_[dev];
    if (!s.pool) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      JC_CUDA_CHECK(cudaMemPoolCreate(&s.pool, &props));
      uint64_t keep = UINT64_MAX;
      JC_CUDA_CHECK(cudaMemPoolSetAttribute(s.pool, cudaMemPoolAttrReleaseThreshold, &keep));
      JC_CUDA_CHECK(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
    }
    return s;
  }

  static constexpr int kMaxDevices = 64;
  std::mutex mu_;
  Slot slots_[kMaxDevices];
};

}  // namespace jc
