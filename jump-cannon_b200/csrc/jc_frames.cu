// Position frames without a host wait per step (see jc_frames.h).
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "jc_frames.h"
#include "jc_pool.h"
#include "jc_upload.h"

namespace jc {
namespace {

constexpr uint32_t FRAME_THREADS = 256;
constexpr uint32_t FRAME_BLOCKS = 148 * 4;

__global__ void k_frame_head(FrameHeader* h, uint32_t encoding, uint64_t frame, uint32_t n,
                             const uint32_t* error_word) {
  h->magic = kFrameMagic;
  h->encoding = encoding;
  h->frame = frame;
  h->n_nodes = n;
  h->status = error_word ? *error_word : 0u;
  h->payload_bytes = (encoding == JC_FRAME_F32 ? 12ull : 6ull) * n;
#pragma unroll
  for (int i = 0; i < 8; ++i) h->reserved[i] = 0u;
}

// A difference that is not a finite f16 of magnitude <= 65504 (or a NaN)
// turns the frame into an f32 frame.
__global__ void __launch_bounds__(FRAME_THREADS)
k_frame_check(const float* __restrict__ xyz, const float* __restrict__ rec, uint64_t m, FrameHeader* h) {
  bool bad = false;
  for (uint64_t i = (uint64_t)blockIdx.x * FRAME_THREADS + threadIdx.x; i < m; i += (uint64_t)gridDim.x * FRAME_THREADS)
    bad |= !(fabsf(__fsub_rn(xyz[i], rec[i])) <= 65504.0f);
  if (__any_sync(0xFFFFFFFFu, bad) && (threadIdx.x & 31) == 0) atomicExch(&h->encoding, JC_FRAME_F32);
}

// Writes the payload in the encoding the header holds after k_frame_check,
// and keeps the receiver's reconstruction `rec` (when tracked).
__global__ void __launch_bounds__(FRAME_THREADS)
k_frame_encode(const float* __restrict__ xyz, float* __restrict__ rec, uint64_t m, FrameHeader* h,
               uint8_t* __restrict__ payload, int track) {
  const uint32_t enc = *(volatile uint32_t*)&h->encoding;
  if (blockIdx.x == 0 && threadIdx.x == 0) h->payload_bytes = (enc == JC_FRAME_F32 ? 4ull : 2ull) * m;
  const uint64_t stride = (uint64_t)gridDim.x * FRAME_THREADS;
  const uint64_t t0 = (uint64_t)blockIdx.x * FRAME_THREADS + threadIdx.x;
  const uint64_t m4 = m / 4;
  if (enc == JC_FRAME_F32) {
    const float4* x4 = reinterpret_cast<const float4*>(xyz);
    float4* o4 = reinterpret_cast<float4*>(payload);
    float4* r4 = reinterpret_cast<float4*>(rec);
    for (uint64_t i = t0; i < m4; i += stride) {
      const float4 v = x4[i];
      o4[i] = v;
      if (track) r4[i] = v;
    }
    float* o = reinterpret_cast<float*>(payload);
    for (uint64_t i = 4 * m4 + t0; i < m; i += stride) {
      o[i] = xyz[i];
      if (track) rec[i] = xyz[i];
    }
  } else {
    const float4* x4 = reinterpret_cast<const float4*>(xyz);
    float4* r4 = reinterpret_cast<float4*>(rec);
    uint2* o4 = reinterpret_cast<uint2*>(payload);
    for (uint64_t i = t0; i < m4; i += stride) {
      const float4 x = x4[i];
      float4 r = r4[i];
      const __half h0 = __float2half_rn(__fsub_rn(x.x, r.x));
      const __half h1 = __float2half_rn(__fsub_rn(x.y, r.y));
      const __half h2 = __float2half_rn(__fsub_rn(x.z, r.z));
      const __half h3 = __float2half_rn(__fsub_rn(x.w, r.w));
      r.x = __fadd_rn(r.x, __half2float(h0));
      r.y = __fadd_rn(r.y, __half2float(h1));
      r.z = __fadd_rn(r.z, __half2float(h2));
      r.w = __fadd_rn(r.w, __half2float(h3));
      r4[i] = r;
      o4[i] = make_uint2((uint32_t)__half_as_ushort(h0) | ((uint32_t)__half_as_ushort(h1) << 16),
                         (uint32_t)__half_as_ushort(h2) | ((uint32_t)__half_as_ushort(h3) << 16));
    }
    __half* o = reinterpret_cast<__half*>(payload);
    for (uint64_t i = 4 * m4 + t0; i < m; i += stride) {
      const __half q = __float2half_rn(__fsub_rn(xyz[i], rec[i]));
      rec[i] = __fadd_rn(rec[i], __half2float(q));
      o[i] = q;
    }
  }
}

uint32_t frame_blocks(uint64_t m) {
  const uint64_t want = (m / 4 + FRAME_THREADS - 1) / FRAME_THREADS;
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, FRAME_BLOCKS));
}

// binary16 -> f32, exact (IEEE 754 layout: 1 sign, 5 exponent, 10 fraction bits).
inline float half_bits_to_float(uint16_t b) {
  const uint32_t sign = (uint32_t)(b >> 15) << 31;
  const uint32_t e = (b >> 10) & 0x1Fu, f = b & 0x3FFu;
  uint32_t bits;
  if (e == 0x1Fu) {
    bits = sign | 0x7F800000u | (f << 13);
  } else if (e == 0) {
    const float v = (float)f * 5.9604644775390625e-8f;  // f * 2^-24, exact
    std::memcpy(&bits, &v, 4);
    bits |= sign;
  } else {
    bits = sign | ((e + 112u) << 23) | (f << 13);
  }
  float v;
  std::memcpy(&v, &bits, 4);
  return v;
}

}  // namespace

FrameStream::FrameStream(Engine* engine, uint32_t encoding, uint32_t depth, uint32_t keyframe_interval)
    : eng_(engine), n_(engine->node_count()), mode_(encoding), depth_(depth), keyframe_interval_(keyframe_interval) {
  if (encoding != JC_FRAME_F32 && encoding != JC_FRAME_F16_DELTA) fail(JC_ERR_ARG, "unknown frame encoding");
  if (depth < 1 || depth > 8) fail(JC_ERR_ARG, "frame ring depth must be 1..8");
  if (!eng_->cuda_stream()) fail(JC_ERR_STATE, "engine has no stream yet (init first)");
  Trace tr("frames.open");
  try {
    const uint64_t bytes = kFrameHeaderBytes + 12ull * n_;
    slots_.resize(depth_);
    for (Slot& s : slots_) {
      s.host = PinnedCache::instance().take(bytes, &s.host_bytes);
      s.dev = static_cast<uint8_t*>(DevicePool::instance().alloc(bytes));
      JC_CUDA_CHECK(cudaEventCreateWithFlags(&s.encoded, cudaEventDisableTiming));
      JC_CUDA_CHECK(cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming));
    }
    if (mode_ == JC_FRAME_F16_DELTA && n_) rec_ = static_cast<float*>(DevicePool::instance().alloc(12ull * n_));
    // the engine's copy stream, else a kept one (creating one costs ~1 ms)
    copy_ = eng_->copy_stream();
    if (!copy_) {
      copy_ = StreamCache::instance().take();
      owns_copy_ = true;
    }
    tr.mark("ring_alloc");
  } catch (...) {
    release();
    throw;
  }
}

FrameStream::~FrameStream() { release(); }

void FrameStream::release() {
  for (Slot& s : slots_)
    if (s.used && s.copied) cudaEventSynchronize(s.copied);
  if (eng_ && eng_->cuda_stream()) cudaStreamSynchronize(eng_->cuda_stream());
  for (Slot& s : slots_) {
    PinnedCache::instance().give(s.host, s.host_bytes);
    DevicePool::instance().free(s.dev);
    if (s.encoded) cudaEventDestroy(s.encoded);
    if (s.copied) cudaEventDestroy(s.copied);
    s = Slot{};
  }
  slots_.clear();
  DevicePool::instance().free(rec_);
  rec_ = nullptr;
  if (owns_copy_) StreamCache::instance().give(copy_);
  owns_copy_ = false;
  copy_ = nullptr;
}

void FrameStream::step(uint32_t iters) {
  if (broken_) fail(JC_ERR_STATE, "the frame stream stopped after a device error; close and reopen it");
  if (produced_ - consumed_ >= depth_)
    fail(JC_ERR_STATE, "every frame slot holds a pending frame: call jc_engine_stream_next first");
  Slot& s = slots_[produced_ % depth_];
  cudaStream_t es = eng_->cuda_stream();
  eng_->enqueue_steps(iters);
  // The slot's previous copy must have left the device staging buffer.
  if (s.used) JC_CUDA_CHECK(cudaStreamWaitEvent(es, s.copied, 0));
  const bool key = mode_ == JC_FRAME_F32 || produced_ == 0 ||
                   (keyframe_interval_ && produced_ % keyframe_interval_ == 0);
  FrameHeader* h = reinterpret_cast<FrameHeader*>(s.dev);
  const uint64_t m = 3ull * n_;
  k_frame_head<<<1, 1, 0, es>>>(h, key ? JC_FRAME_F32 : JC_FRAME_F16_DELTA, produced_, n_, eng_->device_error_word());
  JC_CUDA_CHECK(cudaGetLastError());
  if (m) {
    const float* xyz = eng_->device_xyz();
    if (!key) k_frame_check<<<frame_blocks(m), FRAME_THREADS, 0, es>>>(xyz, rec_, m, h);
    k_frame_encode<<<frame_blocks(m), FRAME_THREADS, 0, es>>>(xyz, rec_, m, h, s.dev + kFrameHeaderBytes,
                                                               mode_ == JC_FRAME_F16_DELTA ? 1 : 0);
    JC_CUDA_CHECK(cudaGetLastError());
  }
  JC_CUDA_CHECK(cudaEventRecord(s.encoded, es));
  JC_CUDA_CHECK(cudaStreamWaitEvent(copy_, s.encoded, 0));
  // A delta frame copies 6n payload bytes; if the device turned it into an
  // f32 frame, stream_next fetches the rest.
  s.copied_bytes = kFrameHeaderBytes + (key ? 12ull : 6ull) * n_;
  JC_CUDA_CHECK(cudaMemcpyAsync(s.host, s.dev, s.copied_bytes, cudaMemcpyDeviceToHost, copy_));
  JC_CUDA_CHECK(cudaEventRecord(s.copied, copy_));
  s.used = true;
  ++produced_;
}

void FrameStream::next(jc_frame* out) {
  if (broken_) fail(JC_ERR_STATE, "the frame stream stopped after a device error; close and reopen it");
  if (consumed_ == produced_) fail(JC_ERR_STATE, "no frame pending: call jc_engine_stream_step first");
  Slot& s = slots_[consumed_ % depth_];
  JC_CUDA_CHECK(cudaEventSynchronize(s.copied));
  FrameHeader h;
  std::memcpy(&h, s.host, sizeof(h));
  if (h.status != 0) {
    broken_ = true;
    JC_CUDA_CHECK(cudaStreamSynchronize(copy_));
    eng_->after_stream_error();  // throws the engine's error
    fail(JC_ERR_STATE, "device error during a streamed step");
  }
  const uint64_t need = kFrameHeaderBytes + h.payload_bytes;
  if (need > s.copied_bytes) {
    JC_CUDA_CHECK(cudaMemcpyAsync(s.host + s.copied_bytes, s.dev + s.copied_bytes, need - s.copied_bytes,
                                  cudaMemcpyDeviceToHost, copy_));
    JC_CUDA_CHECK(cudaEventRecord(s.copied, copy_));
    JC_CUDA_CHECK(cudaEventSynchronize(s.copied));
    s.copied_bytes = need;
  }
  out->frame = h.frame;
  out->n_nodes = h.n_nodes;
  out->encoding = h.encoding;
  out->data = s.host;
  out->bytes = need;
  out->payload = s.host + kFrameHeaderBytes;
  out->payload_bytes = h.payload_bytes;
  ++consumed_;
}

void decode_frame(FrameDecoder& d, const uint8_t* data, uint64_t bytes, float* out_xyz) {
  if (data == nullptr || bytes < kFrameHeaderBytes) fail(JC_ERR_ARG, "frame shorter than its 64-byte header");
  FrameHeader h;
  std::memcpy(&h, data, sizeof(h));
  if (h.magic != kFrameMagic) fail(JC_ERR_ARG, "not a position frame (bad magic)");
  if (h.n_nodes != d.n) fail(JC_ERR_ARG, "frame is for " + std::to_string(h.n_nodes) + " nodes, decoder for " +
                                             std::to_string(d.n));
  const uint64_t m = 3ull * d.n;
  if (h.encoding == JC_FRAME_F32) {
    if (h.payload_bytes != 4 * m || bytes != kFrameHeaderBytes + 4 * m) fail(JC_ERR_ARG, "f32 frame size mismatch");
    std::memcpy(d.rec.data(), data + kFrameHeaderBytes, 4 * m);
    d.have_key = true;
  } else if (h.encoding == JC_FRAME_F16_DELTA) {
    if (h.payload_bytes != 2 * m || bytes != kFrameHeaderBytes + 2 * m) fail(JC_ERR_ARG, "f16 frame size mismatch");
    if (!d.have_key) fail(JC_ERR_STATE, "delta frame before any f32 frame");
    if (h.frame != d.last_frame + 1) fail(JC_ERR_STATE, "delta frame out of sequence");
    const uint8_t* p = data + kFrameHeaderBytes;
    for (uint64_t i = 0; i < m; ++i) {
      uint16_t b;
      std::memcpy(&b, p + 2 * i, 2);
      d.rec[i] = d.rec[i] + half_bits_to_float(b);
    }
  } else {
    fail(JC_ERR_ARG, "unknown frame encoding");
  }
  d.last_frame = h.frame;
  if (out_xyz && m) std::memcpy(out_xyz, d.rec.data(), 4 * m);
}

}  // namespace jc
