// Position frames: the per-tick position message the reference's sim loop
// broadcasts (PositionDelta, crates/graph-compute/proto/compute.proto:84-91:
// frame number, n_nodes, raw little-endian f32 x,y,z) produced without a
// host wait per step, plus a half-size encoding of the same message.
//
// A FrameStream owns a ring of `depth` slots, each a device staging buffer
// and a page-locked host buffer. stream_step enqueues the engine's steps on
// the engine's stream, encodes the positions into the next slot's device
// buffer and copies that slot to the host on a second stream, so the copy of
// frame t overlaps the steps of frame t+1; stream_next waits for the oldest
// pending slot only.
//
// Encodings of the payload:
//  JC_FRAME_F32        raw LE f32 x,y,z (exactly PositionDelta.positions).
//  JC_FRAME_F16_DELTA  LE binary16 differences from the receiver's
//                      reconstruction. Encoder and decoder keep the same
//                      f32 reconstruction r (r += f32(h) after each delta
//                      frame, r = x after each f32 frame), and the encoder
//                      takes h = f16_rn(x - r), so a receiver's error is the
//                      rounding of the latest difference alone and never
//                      accumulates. A frame in which some difference is not
//                      a finite f16 of magnitude <= 65504 is sent as f32.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "jc_engine.h"

namespace jc {

constexpr uint32_t kFrameMagic = 0x3146434Au;  // "JCF1" as LE bytes
constexpr uint32_t kFrameHeaderBytes = 64;

// Little-endian wire header in front of every payload (64 bytes).
struct FrameHeader {
  uint32_t magic;
  uint32_t encoding;       // JC_FRAME_F32 or JC_FRAME_F16_DELTA
  uint64_t frame;          // 0, 1, 2, ... since the stream was opened
  uint32_t n_nodes;
  uint32_t status;         // device error word after the steps (0 on the wire)
  uint64_t payload_bytes;  // 12 n (f32) or 6 n (f16)
  uint32_t reserved[8];
};
static_assert(sizeof(FrameHeader) == kFrameHeaderBytes, "frame header is 64 bytes");

class FrameStream {
 public:
  FrameStream(Engine* engine, uint32_t encoding, uint32_t depth, uint32_t keyframe_interval);
  ~FrameStream();
  FrameStream(const FrameStream&) = delete;
  FrameStream& operator=(const FrameStream&) = delete;

  void step(uint32_t iters);
  void next(jc_frame* out);

 private:
  struct Slot {
    uint8_t* host = nullptr;
    uint8_t* dev = nullptr;
    cudaEvent_t encoded = nullptr;
    cudaEvent_t copied = nullptr;
    uint64_t copied_bytes = 0;
    uint64_t host_bytes = 0;  // size of `host` (it returns to the pinned cache)
    bool used = false;
  };
  void release();

  Engine* eng_;
  uint32_t n_, mode_, depth_, keyframe_interval_;
  std::vector<Slot> slots_;
  float* rec_ = nullptr;
  cudaStream_t copy_ = nullptr;
  bool owns_copy_ = false;  // copy_ borrowed from the stream cache (else the engine's)
  uint64_t produced_ = 0, consumed_ = 0;
  bool broken_ = false;
};

// Host decoder state (the receiver's reconstruction).
struct FrameDecoder {
  uint32_t n = 0;
  bool have_key = false;
  uint64_t last_frame = 0;
  std::vector<float> rec;
};

void decode_frame(FrameDecoder& d, const uint8_t* data, uint64_t bytes, float* out_xyz);

}  // namespace jc
