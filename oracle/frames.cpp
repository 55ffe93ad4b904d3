// CPU oracle for position frames — TEST INFRASTRUCTURE ONLY (loaded by tests/
// through liboracle.so; never linked into the product library).
//
// f32 frames are the reference's PositionDelta payload, raw little-endian
// f32 x,y,z (crates/graph-compute/proto/compute.proto:84-91, filled from the
// engine's StepOutput positions, crates/graph-compute/src/sim.rs tick loop);
// they need no restatement beyond a byte copy. The binary16 delta frames have
// no reference counterpart; this file restates their encoder from its
// definition so the device encoder can be checked bit for bit:
//   r: the receiver's f32 reconstruction (r = x after an f32 frame);
//   a frame is sent as f32 when some |x_i - r_i| (f32 subtraction) is not
//   <= 65504 (this includes NaN); otherwise h_i = f16_rn(x_i - r_i) and
//   r_i = r_i + f32(h_i) in f32.
// The binary16 conversion below is written from the IEEE 754 bit layouts
// (binary32: 1/8/23 bits, bias 127; binary16: 1/5/10 bits, bias 15) with
// round-to-nearest, ties to even; tests pin it against numpy's float16 cast.
#include <cstdint>
#include <cstring>

namespace {

uint16_t f32_to_f16_rn(float x) {
  uint32_t b;
  std::memcpy(&b, &x, 4);
  const uint32_t sign = (b >> 16) & 0x8000u;
  const uint32_t e = (b >> 23) & 0xFFu;
  const uint32_t f = b & 0x7FFFFFu;
  if (e == 0xFFu) return (uint16_t)(sign | 0x7C00u | (f ? 0x200u | (f >> 13) : 0u));  // inf, quiet NaN
  const int E = (int)e - 127;
  if (E > 15) return (uint16_t)(sign | 0x7C00u);  // >= 2^16: infinity
  if (E >= -14) {
    // normal binary16 range: keep 10 of the 23 fraction bits, round the 13 dropped
    uint32_t h = ((uint32_t)(E + 15) << 10) | (f >> 13);
    const uint32_t rem = f & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1u;  // a carry moves into the exponent (up to inf)
    return (uint16_t)(sign | h);
  }
  if (E < -25) return (uint16_t)sign;  // below half the smallest subnormal (2^-25): zero
  // subnormal result in units of 2^-24: significand (24 bits) * 2^(E + 1)
  const uint32_t sig = f | 0x800000u;
  const int s = -E - 1;  // 14..24
  uint32_t m = sig >> s;
  const uint32_t rem = sig & ((1u << s) - 1u), half = 1u << (s - 1);
  if (rem > half || (rem == half && (m & 1u))) m += 1u;  // 0x400 is the smallest normal, encoded alike
  return (uint16_t)(sign | m);
}

float f16_to_f32(uint16_t h) {
  const uint32_t sign = (uint32_t)(h >> 15) << 31;
  const uint32_t e = (h >> 10) & 0x1Fu, f = h & 0x3FFu;
  uint32_t bits;
  if (e == 0x1Fu) {
    bits = sign | 0x7F800000u | (f << 13);
  } else if (e == 0) {
    // f * 2^-24 is exact in binary32
    const float v = (float)f * (1.0f / 16777216.0f);
    std::memcpy(&bits, &v, 4);
    bits |= sign;
  } else {
    bits = sign | ((e - 15u + 127u) << 23) | (f << 13);
  }
  float v;
  std::memcpy(&v, &bits, 4);
  return v;
}

}  // namespace

extern "C" {

uint16_t orc_f32_to_f16(float x) { return f32_to_f16_rn(x); }
float orc_f16_to_f32(uint16_t h) { return f16_to_f32(h); }

void orc_f32_to_f16_array(uint64_t m, const float* x, uint16_t* out) {
  for (uint64_t i = 0; i < m; ++i) out[i] = f32_to_f16_rn(x[i]);
}

// One frame of the delta encoder over m = 3n coordinates. Returns 1 when the
// frame goes out as f32 (rec := xyz, out untouched), 0 for a delta frame
// (out := halves, rec advanced as the receiver advances it).
int orc_frame_encode_f16(uint64_t m, const float* xyz, float* rec, uint16_t* out) {
  bool key = false;
  for (uint64_t i = 0; i < m && !key; ++i) {
    const float d = xyz[i] - rec[i];
    key = !(d <= 65504.0f && d >= -65504.0f);
  }
  if (key) {
    std::memcpy(rec, xyz, sizeof(float) * m);
    return 1;
  }
  for (uint64_t i = 0; i < m; ++i) {
    const uint16_t h = f32_to_f16_rn(xyz[i] - rec[i]);
    out[i] = h;
    rec[i] = rec[i] + f16_to_f32(h);
  }
  return 0;
}

}  // extern "C"
