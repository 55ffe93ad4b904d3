// Engine settings and their JSON decoding.
//
// The reference decodes `set_params` with serde_json into a struct marked
// #[serde(default)] (engines/fa2_bh.rs:82-119 + :212-220,
// engines/fa2_brute.rs:63-94, engines/sgd_stress.rs:59-98): a JSON `null`
// keeps the current settings; otherwise the settings are REPLACED by the
// defaults overlaid with the named fields; unknown keys are ignored; a field
// of the wrong type (or an integer field given a fraction / negative value)
// is an error. This header reproduces exactly that contract.
#pragma once

#include <cctype>
#include <cmath>
#include <cstring>
#include <cstdint>
#include <cstdlib>
#include <map>
#include <string>

#include "jc_common.h"

namespace jc {

struct JsonValue {
  enum Kind { Null, Bool, Number, String, Other } kind = Null;
  bool b = false;
  double num = 0.0;
  bool is_integer = false;  // number token had no '.', 'e' or 'E'
  bool negative = false;
  uint64_t u = 0;           // magnitude when is_integer (saturating)
  std::string s;
  std::string raw;          // the value's JSON text (objects and arrays)
};

class JsonParser {
 public:
  explicit JsonParser(const char* text) : p_(text) {}

  // Parses a top-level value; returns false on syntax error. Only a flat
  // object's members are recorded; nested values are validated and skipped.
  bool parse_top(bool* is_null, std::map<std::string, JsonValue>* out, std::string* err) {
    ws();
    if (lit("null")) {
      ws();
      *is_null = true;
      return at_end(err);
    }
    *is_null = false;
    if (*p_ != '{') {
      *err = "expected a JSON object";
      return false;
    }
    ++p_;
    ws();
    if (*p_ == '}') {
      ++p_;
      return at_end(err);
    }
    for (;;) {
      ws();
      std::string key;
      if (!str(&key)) { *err = "expected a string key"; return false; }
      ws();
      if (*p_ != ':') { *err = "expected ':'"; return false; }
      ++p_;
      ws();
      JsonValue v;
      if (!value(&v, 0)) { *err = "malformed value for key '" + key + "'"; return false; }
      if (out->count(key)) { *err = "duplicate field `" + key + "`"; return false; }
      (*out)[key] = v;
      ws();
      if (*p_ == ',') { ++p_; continue; }
      if (*p_ == '}') { ++p_; break; }
      *err = "expected ',' or '}'";
      return false;
    }
    return at_end(err);
  }

 private:
  const char* p_;
  void ws() { while (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r') ++p_; }
  bool lit(const char* w) {
    size_t n = std::strlen(w);
    if (std::strncmp(p_, w, n) == 0) { p_ += n; return true; }
    return false;
  }
  bool at_end(std::string* err) {
    ws();
    if (*p_ != '\0') { *err = "trailing characters after JSON value"; return false; }
    return true;
  }
  bool str(std::string* out) {
    if (*p_ != '"') return false;
    ++p_;
    while (*p_ && *p_ != '"') {
      if (*p_ == '\\') {
        ++p_;
        if (!*p_) return false;
        if (*p_ == 'u') {
          for (int k = 0; k < 4; ++k) { ++p_; if (!std::isxdigit((unsigned char)*p_)) return false; }
          out->push_back('?');
          ++p_;
          continue;
        }
        char c = *p_;
        out->push_back(c == 'n' ? '\n' : c == 't' ? '\t' : c == 'r' ? '\r' : c == 'b' ? '\b' : c == 'f' ? '\f' : c);
        ++p_;
        continue;
      }
      out->push_back(*p_++);
    }
    if (*p_ != '"') return false;
    ++p_;
    return true;
  }
  bool number(JsonValue* v) {
    const char* start = p_;
    if (*p_ == '-') { v->negative = true; ++p_; }
    if (!std::isdigit((unsigned char)*p_)) return false;
    bool integer = true;
    while (std::isdigit((unsigned char)*p_)) ++p_;
    if (*p_ == '.') {
      integer = false;
      ++p_;
      if (!std::isdigit((unsigned char)*p_)) return false;
      while (std::isdigit((unsigned char)*p_)) ++p_;
    }
    if (*p_ == 'e' || *p_ == 'E') {
      integer = false;
      ++p_;
      if (*p_ == '+' || *p_ == '-') ++p_;
      if (!std::isdigit((unsigned char)*p_)) return false;
      while (std::isdigit((unsigned char)*p_)) ++p_;
    }
    std::string tok(start, p_);
    v->kind = JsonValue::Number;
    v->num = std::strtod(tok.c_str(), nullptr);
    v->is_integer = integer;
    if (integer) {
      uint64_t acc = 0;
      bool sat = false;
      for (const char* q = tok.c_str() + (v->negative ? 1 : 0); *q; ++q) {
        uint64_t d = (uint64_t)(*q - '0');
        if (acc > (UINT64_MAX - d) / 10) { sat = true; acc = UINT64_MAX; break; }
        acc = acc * 10 + d;
      }
      v->u = sat ? UINT64_MAX : acc;
      if (sat) v->is_integer = false;  // out of u64 range: not representable
    }
    return true;
  }
  bool value(JsonValue* v, int depth) {
    if (depth > 64) return false;
    ws();
    if (lit("null")) { v->kind = JsonValue::Null; return true; }
    if (lit("true")) { v->kind = JsonValue::Bool; v->b = true; return true; }
    if (lit("false")) { v->kind = JsonValue::Bool; v->b = false; return true; }
    if (*p_ == '"') { v->kind = JsonValue::String; return str(&v->s); }
    if (*p_ == '-' || std::isdigit((unsigned char)*p_)) return number(v);
    if (*p_ == '{' || *p_ == '[') {
      const char* start = p_;
      char close = *p_ == '{' ? '}' : ']';
      bool obj = *p_ == '{';
      ++p_;
      v->kind = JsonValue::Other;
      v->b = obj;  // an object (true) or an array
      ws();
      if (*p_ == close) { ++p_; v->raw.assign(start, p_); return true; }
      for (;;) {
        ws();
        if (obj) {
          std::string k;
          if (!str(&k)) return false;
          ws();
          if (*p_ != ':') return false;
          ++p_;
        }
        JsonValue inner;
        if (!value(&inner, depth + 1)) return false;
        ws();
        if (*p_ == ',') { ++p_; continue; }
        if (*p_ == close) { ++p_; v->raw.assign(start, p_); return true; }
        return false;
      }
    }
    return false;
  }
};

// Field readers with serde's type rules.
struct FieldReader {
  const std::map<std::string, JsonValue>& m;
  std::string prefix;
  void f32(const char* name, float* dst) const {
    auto it = m.find(name);
    if (it == m.end()) return;
    if (it->second.kind != JsonValue::Number)
      fail(JC_ERR_PARAMS, prefix + ": invalid type for `" + name + "`, expected f32");
    *dst = (float)it->second.num;
  }
  void boolean(const char* name, bool* dst) const {
    auto it = m.find(name);
    if (it == m.end()) return;
    if (it->second.kind != JsonValue::Bool)
      fail(JC_ERR_PARAMS, prefix + ": invalid type for `" + name + "`, expected a boolean");
    *dst = it->second.b;
  }
  void u32(const char* name, uint32_t* dst) const {
    auto it = m.find(name);
    if (it == m.end()) return;
    const JsonValue& v = it->second;
    if (v.kind != JsonValue::Number || !v.is_integer || (v.negative && v.u != 0) || v.u > 0xFFFFFFFFull)
      fail(JC_ERR_PARAMS, prefix + ": invalid value for `" + name + "`, expected u32");
    *dst = (uint32_t)v.u;
  }
  void u64(const char* name, uint64_t* dst) const {
    auto it = m.find(name);
    if (it == m.end()) return;
    const JsonValue& v = it->second;
    if (v.kind != JsonValue::Number || !v.is_integer || (v.negative && v.u != 0))
      fail(JC_ERR_PARAMS, prefix + ": invalid value for `" + name + "`, expected u64");
    *dst = v.u;
  }
};

// Fa2BhSettings (fa2_bh.rs:84-119) / Fa2Settings (fa2_brute.rs:63-94).
// Fields after `max_displacement` are this engine's own knobs; the reference
// ignores unknown keys, so they are backward compatible on the wire.
struct Fa2Settings {
  float gravity = 1.0f;
  bool strong_gravity = false;
  float scaling_ratio = 2.0f;
  float edge_weight_influence = 1.0f;
  float jitter_tolerance = 1.0f;
  bool lin_log_mode = false;
  bool prevent_overlap = false;  // plumbed but unused by the reference shader
  float time_step = 1.0f;
  float theta = 0.7f;
  float max_displacement = 10.0f;
  // Nodes whose attraction list is at least this long are summed by a whole
  // block (reassociated, deterministic); shorter lists are summed by one
  // thread in the reference's edge order. 0 = use the engine default.
  uint32_t hub_threshold = 0;
  // Nodes whose attraction list is at least this long (and below the hub
  // threshold) are gathered by a whole warp and summed in list order by one
  // lane (same roundings as one thread). 0 = the engine default.
  uint32_t warp_threshold = 0;
  // Lanes that share one node stream in the theta walk (1, 2, 4, 8, 16 or
  // 32; 0 = the engine default). Results do not depend on it.
  uint32_t walk_group = 0;
  // Stage the top of a single graph's tree (depth <= 3) in shared memory for
  // the walk (walk group 1). Results do not depend on it. Off by default: on
  // B200 the walk of the 1M-node R-MAT graph took 0.75 ms staged against
  // 0.53 ms from global memory (lanes in the staged top and lanes in the
  // global subtrees diverge, so every iteration issues both load paths).
  bool walk_stage_top = false;
  // Replay each step from a captured CUDA graph (default). false launches the
  // same kernels one by one (for profilers that cannot see into graphs with
  // conditional nodes); results are identical.
  bool use_graph = true;
  // Tolerance mode of the Barnes-Hut walk (off by default): each repulsion
  // term srd*m/r2 uses the approximate reciprocal and the sums fuse into
  // FMAs. The tree decisions stay exact (same nodes visited, same walk
  // counts); forces differ from the exact mode by ~1e-7 relative L2, well
  // inside the 1e-4 per-iteration bar. fa2-brute ignores it.
  bool fast_repulsion = false;
  // Schedule of a batch (jc_engine_init_batch): 0 = one forest per launch
  // (every kernel covers all graphs), 1 = one CTA per graph in a persistent
  // launch that runs all requested iterations (taken when every graph
  // qualifies: no list of hub_threshold entries or more). jc_engine_autotune
  // times both and keeps the faster. Results are identical.
  uint32_t batch_schedule = 0;
};

// SgdStressSettings (sgd_stress.rs:59-98).
struct SgdSettings {
  uint32_t n_pivots = 50;
  uint32_t sweeps_per_step = 1;
  float eta_max = 1.0f;
  float eta_min = 0.01f;
  uint32_t n_anneal_steps = 30;
  uint64_t seed = 0x5EEDC0DE12345678ull;
  // Pair updates per scatter batch = n / batches (per-pair engine only).
  uint32_t scatter_batches = 0;
  // s_gd2 schedule from the data: eta_max = 1/w_min = (max pivot distance)^2,
  // eta_min = 0.01/w_max = 0.01 (hop distances are >= 1).
  bool auto_eta = false;
  // k distinct uniformly random pivots with hop distances from one device
  // multi-source BFS, instead of the reference's sequential max-min choice
  // with one host BFS per pivot.
  bool random_pivots = false;
};

// MultilevelSettings (engines/multilevel.rs:126-203): the wrapped engine's
// id, its settings forwarded verbatim, and the cascade / sweep knobs.
struct MultilevelSettings {
  std::string inner = "fa2-brute";
  std::string inner_params = "null";  // JSON text given to the inner engine's set_params
  uint64_t max_levels = 6;
  uint64_t target_size = 500;
  uint32_t sweeps_per_level = 30;
  uint32_t sweep_schedule = 1;  // 0 uniform, 1 linear (default), 2 geometric
  float spring_len = 30.0f;
  uint32_t seed = 0x5EED;
};

// Returns true when the JSON was `null` (keep current settings).
inline bool parse_object(const char* json, std::map<std::string, JsonValue>* fields,
                         const std::string& what) {
  if (json == nullptr) return true;
  JsonParser p(json);
  bool is_null = false;
  std::string err;
  if (!p.parse_top(&is_null, fields, &err)) fail(JC_ERR_PARAMS, "decode " + what + " settings: " + err);
  return is_null;
}

inline void decode_fa2(const char* json, Fa2Settings* s, bool with_theta, const std::string& what) {
  std::map<std::string, JsonValue> m;
  if (parse_object(json, &m, what)) return;
  Fa2Settings t;  // defaults
  FieldReader r{m, "decode " + what + " settings"};
  r.f32("gravity", &t.gravity);
  r.boolean("strong_gravity", &t.strong_gravity);
  r.f32("scaling_ratio", &t.scaling_ratio);
  r.f32("edge_weight_influence", &t.edge_weight_influence);
  r.f32("jitter_tolerance", &t.jitter_tolerance);
  r.boolean("lin_log_mode", &t.lin_log_mode);
  r.boolean("prevent_overlap", &t.prevent_overlap);
  r.f32("time_step", &t.time_step);
  if (with_theta) r.f32("theta", &t.theta);
  r.f32("max_displacement", &t.max_displacement);
  r.u32("hub_threshold", &t.hub_threshold);
  r.u32("warp_threshold", &t.warp_threshold);
  r.u32("walk_group", &t.walk_group);
  r.boolean("walk_stage_top", &t.walk_stage_top);
  r.boolean("use_graph", &t.use_graph);
  r.boolean("fast_repulsion", &t.fast_repulsion);
  r.u32("batch_schedule", &t.batch_schedule);
  *s = t;
}

inline void decode_sgd(const char* json, SgdSettings* s, const std::string& what) {
  std::map<std::string, JsonValue> m;
  if (parse_object(json, &m, what)) return;
  SgdSettings t;
  FieldReader r{m, "decode " + what + " settings"};
  r.u32("n_pivots", &t.n_pivots);
  r.u32("sweeps_per_step", &t.sweeps_per_step);
  r.f32("eta_max", &t.eta_max);
  r.f32("eta_min", &t.eta_min);
  r.u32("n_anneal_steps", &t.n_anneal_steps);
  r.u64("seed", &t.seed);
  r.u32("scatter_batches", &t.scatter_batches);
  r.boolean("auto_eta", &t.auto_eta);
  r.boolean("random_pivots", &t.random_pivots);
  *s = t;
}

inline void decode_multilevel(const char* json, MultilevelSettings* s) {
  std::map<std::string, JsonValue> m;
  if (parse_object(json, &m, "multilevel")) return;
  MultilevelSettings t;
  FieldReader r{m, "decode multilevel settings"};
  auto it = m.find("inner");
  if (it != m.end()) {
    if (it->second.kind != JsonValue::String)
      fail(JC_ERR_PARAMS, "decode multilevel settings: invalid type for `inner`, expected a string");
    t.inner = it->second.s;
  }
  it = m.find("inner_params");
  if (it != m.end()) {
    const JsonValue& v = it->second;
    if (v.kind == JsonValue::Null) t.inner_params = "null";
    else if (v.kind == JsonValue::Other && v.b) t.inner_params = v.raw;
    else t.inner_params = "[]";  // not an object: the inner engine's decode rejects it at init
  }
  r.u64("max_levels", &t.max_levels);
  r.u64("target_size", &t.target_size);
  r.u32("sweeps_per_level", &t.sweeps_per_level);
  it = m.find("sweep_schedule");
  if (it != m.end()) {
    const JsonValue& v = it->second;
    if (v.kind != JsonValue::String || (v.s != "uniform" && v.s != "linear" && v.s != "geometric"))
      fail(JC_ERR_PARAMS, "decode multilevel settings: unknown variant for `sweep_schedule`, expected one of "
                          "`uniform`, `linear`, `geometric`");
    t.sweep_schedule = v.s == "uniform" ? 0u : v.s == "linear" ? 1u : 2u;
  }
  r.f32("spring_len", &t.spring_len);
  r.u32("seed", &t.seed);
  *s = t;
}

}  // namespace jc
