// Shared host-side definitions for libjc_layout: status plumbing, CUDA error
// checks and the SplitMix64 generator used by every seeded fixture.
#pragma once

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "../../include/jc_layout.h"

namespace jc {

// An error that carries a jc_status across the C++ layer; converted to a
// status code + message at the C-ABI boundary (no exception crosses it).
struct Error : std::runtime_error {
  jc_status code;
  Error(jc_status c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

[[noreturn]] inline void fail(jc_status code, const std::string& msg) { throw Error(code, msg); }

// SplitMix64 (crates/graph-compute/src/stability.rs:11-26 and
// engines/sgd_stress.rs:104-125): a counter-based generator, so the k-th
// output is mix(seed + k * gamma) and can also be computed out of order.
struct SplitMix64 {
  uint64_t state;
  explicit SplitMix64(uint64_t s) : state(s) {}
  static inline uint64_t mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  inline uint64_t next_u64() {
    state += 0x9E3779B97F4A7C15ull;
    return mix(state);
  }
  // Uniform f32 in [0, 1) (stability.rs:22-25).
  inline float next_f32() { return (float)(next_u64() >> 40) / (float)(1u << 24); }
  // Uniform f64 in [0, 1).
  inline double next_f64() { return (double)(next_u64() >> 11) * (1.0 / 9007199254740992.0); }
  // Uniform integer in [0, n), n > 0 (sgd_stress.rs:121-124).
  inline uint64_t below(uint64_t n) { return next_u64() % n; }
};

constexpr uint64_t kSplitMixGamma = 0x9E3779B97F4A7C15ull;

// Host wall-clock phase timings of one call, printed to stderr as
// "jc-trace <call> <phase> <ms>" when the JC_TRACE environment variable is
// set (a no-op otherwise).
class Trace {
 public:
  explicit Trace(const char* call) : call_(call), on_(std::getenv("JC_TRACE") != nullptr) {
    if (on_) last_ = std::chrono::steady_clock::now();
  }
  void mark(const char* phase) {
    if (!on_) return;
    const auto t = std::chrono::steady_clock::now();
    std::fprintf(stderr, "jc-trace %s %s %.3f\n", call_, phase,
                 std::chrono::duration<double, std::milli>(t - last_).count());
    last_ = t;
  }

 private:
  const char* call_;
  bool on_;
  std::chrono::steady_clock::time_point last_{};
};

}  // namespace jc

#define JC_CUDA_CHECK(expr)                                                              \
  do {                                                                                   \
    cudaError_t jc_err_ = (expr);                                                        \
    if (jc_err_ != cudaSuccess) {                                                        \
      (void)cudaGetLastError(); /* clear the non-sticky last-error state */              \
      ::jc::fail(JC_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(jc_err_)); \
    }                                                                                    \
  } while (0)
