// CPU restatement of the learned warm start - TEST INFRASTRUCTURE ONLY.
//
// The reference has no learned component; this file restates, in plain C++
// with f64 arithmetic, the features, forward pass, stress loss and backward
// pass of the device network so the tests can check the device gradients.
// Its loss restates the scale-normalized stress of
// crates/graph-layouts/src/metrics.rs:31-59 (closed-form scale, w = 1/d^2).
//
// Graphs arrive as one global CSR (node ids global, sorted symmetric rows)
// with graph g owning nodes [go[g], go[g+1]).
//
// Two modes:
//   emulate = 1: values are rounded to bf16 (round to nearest even) where the
//                device stores them: input features, weights read by the
//                GEMMs, the mean aggregations, hidden activations, the
//                activation-gradient GEMM outputs and the activation
//                gradients; mean aggregations and the random
//                projections use the device's f32 operations in its order.
//   emulate = 0: everything in f64, no rounding: the function the device
//                approximates, for finite-difference checks of this file.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr int FEAT = 32, HID = 128, WALKS = 32, WALK_LEN = 16, NPROJ = 8;
constexpr uint32_t HUB_DEG = 1024;
constexpr int HUB_SEGS = 8;
constexpr uint64_t SALT_WALK = 0x57A1C0FFEE000001ull;
constexpr uint64_t SALT_PROJ = 0x9B0C5EED00000002ull;
constexpr uint64_t SALT_PAIR = 0x7A1B2C3D00000003ull;

uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
uint64_t hash4(uint64_t s, uint64_t a, uint64_t b, uint64_t c) { return mix64(mix64(mix64(s ^ a) ^ b) ^ c); }
uint32_t pick(uint64_t h, uint32_t n) { return (uint32_t)(((h >> 32) * (uint64_t)n) >> 32); }

float irwin4(uint64_t h) {
  const uint32_t s = (uint32_t)((h >> 52) & 0xFFF) + (uint32_t)((h >> 40) & 0xFFF) +
                     (uint32_t)((h >> 28) & 0xFFF) + (uint32_t)((h >> 16) & 0xFFF);
  const float u = (float)(2u * s + 4u) * (1.0f / 8192.0f);
  return (u - 2.0f) * 1.7320508075688772f;
}

float bf16r(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) {  // inf / nan: truncate, keep nan quiet
    if (u & 0x007FFFFFu) u |= 0x00400000u;
    u &= 0xFFFF0000u;
  } else {
    u += 0x7FFFu + ((u >> 16) & 1u);
    u &= 0xFFFF0000u;
  }
  std::memcpy(&f, &u, 4);
  return f;
}

struct Csr {
  uint32_t n, G;
  const uint32_t *go, *off, *nbr;
  uint32_t deg(uint32_t v) const { return off[v + 1] - off[v]; }
};

// Row sum in the device order: CSR order, or 8 contiguous segments added in
// order for rows longer than HUB_DEG. term(j) returns the f32 addend.
template <class F>
float row_sum_f32(const Csr& g, uint32_t v, F term) {
  const uint32_t d = g.deg(v);
  const uint32_t* row = g.nbr + g.off[v];
  if (d <= HUB_DEG) {
    float a = 0.0f;
    for (uint32_t e = 0; e < d; ++e) a += term(row[e]);
    return a;
  }
  const uint32_t seg = (d + HUB_SEGS - 1) / HUB_SEGS;
  float total = 0.0f;
  for (int q = 0; q < HUB_SEGS; ++q) {
    const uint32_t b = std::min(d, (uint32_t)q * seg), e = std::min(d, b + seg);
    float a = 0.0f;
    for (uint32_t k = b; k < e; ++k) a += term(row[k]);
    total = q == 0 ? a : total + a;
  }
  return total;
}

struct Layout {
  size_t w[3], b[3], wh, bh, total;
  int kin[3];
};
Layout layout() {
  Layout L{};
  const int kin[3] = {2 * FEAT, 2 * HID, 2 * HID};
  size_t o = 0;
  for (int l = 0; l < 3; ++l) {
    L.kin[l] = kin[l];
    L.w[l] = o;
    o += (size_t)kin[l] * HID;
    L.b[l] = o;
    o += HID;
  }
  L.wh = o;
  o += (size_t)HID * 4;
  L.bh = o;
  o += 4;
  L.total = (o + 7) & ~(size_t)7;
  return L;
}

}  // namespace

extern "C" {

uint32_t orc_mpnn_num_params(void) { return (uint32_t)layout().total; }

// Features of every node: n x 32 floats (bf16 values).
void orc_mpnn_features(uint32_t n, uint32_t G, const uint32_t* go, const uint32_t* off, const uint32_t* nbr,
                       uint64_t seed, uint32_t smooth_steps, uint32_t cheb_steps, float cheb_b, float* X) {
  const Csr g{n, G, go, off, nbr};
  std::vector<float> P((size_t)n * NPROJ), P2((size_t)n * NPROJ);
  for (uint32_t i = 0; i < n; ++i) {
    float* x = X + (size_t)i * FEAT;
    for (int c = 0; c < FEAT; ++c) x[c] = 0.0f;
    x[0] = bf16r(std::log1p((float)g.deg(i)));
    uint32_t cur[WALKS];
    for (int w = 0; w < WALKS; ++w) cur[w] = i;
    for (int t = 1; t <= WALK_LEN; ++t) {
      uint32_t back = 0;
      for (int w = 0; w < WALKS; ++w) {
        const uint32_t d = g.deg(cur[w]);
        if (d) cur[w] = nbr[off[cur[w]] + pick(hash4(seed ^ SALT_WALK, i, (uint64_t)w, (uint64_t)t), d)];
        back += cur[w] == i;
      }
      x[t] = bf16r((float)back * (1.0f / WALKS));
    }
    for (int c = 0; c < NPROJ; ++c) P[(size_t)i * NPROJ + c] = irwin4(hash4(seed ^ SALT_PROJ, i, (uint64_t)c, 0));
  }
  // remove each graph's degree-weighted mean from every column of x and
  // rescale to unit mean square; `pair` (if given) loses its own mean and
  // takes x's scale (the Chebyshev pair)
  auto center = [&](std::vector<float>& x, std::vector<float>* pair) {
    for (uint32_t gr = 0; gr < G; ++gr) {
      double sx[NPROJ] = {0}, sq[NPROJ] = {0}, sd = 0.0, spx[NPROJ] = {0};
      for (uint32_t i = go[gr]; i < go[gr + 1]; ++i) {
        for (int c = 0; c < NPROJ; ++c) {
          const double v = x[(size_t)i * NPROJ + c];
          sx[c] += (double)g.deg(i) * v;
          sq[c] += v * v;
          if (pair) spx[c] += (double)g.deg(i) * (double)(*pair)[(size_t)i * NPROJ + c];
        }
        sd += (double)g.deg(i);
      }
      const double ng = (double)(go[gr + 1] - go[gr]);
      for (int c = 0; c < NPROJ; ++c) {
        const float m = sd > 0.0 ? (float)(sx[c] / sd) : 0.0f;
        const float mp = sd > 0.0 ? (float)(spx[c] / sd) : 0.0f;
        const double ms = sq[c] / ng;
        const float sc = ms > 0.0 ? (float)(1.0 / std::sqrt(ms)) : 1.0f;
        for (uint32_t i = go[gr]; i < go[gr + 1]; ++i) {
          x[(size_t)i * NPROJ + c] = (x[(size_t)i * NPROJ + c] - m) * sc;
          if (pair) (*pair)[(size_t)i * NPROJ + c] = ((*pair)[(size_t)i * NPROJ + c] - mp) * sc;
        }
      }
    }
  };
  // one filter step out = f(P x) with P x = (x + D^-1 A x) / 2: mode 0 the
  // lazy step P x; mode 1 c1 P x - x; mode 2 (c1 P x - 2 x) - x_prev
  auto step = [&](const std::vector<float>& x, std::vector<float>& out, const std::vector<float>* prev, int mode,
                  float c1) {
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t d = g.deg(i);
      for (int c = 0; c < NPROJ; ++c) {
        const float xi = x[(size_t)i * NPROJ + c];
        float px = xi;
        if (d != 0) {
          const float s = row_sum_f32(g, i, [&](uint32_t j) { return x[(size_t)j * NPROJ + c]; });
          px = (xi + s / (float)d) * 0.5f;
        }
        float o = px;
        if (mode == 1) o = c1 * px - xi;
        if (mode == 2) o = (c1 * px - 2.0f * xi) - (*prev)[(size_t)i * NPROJ + c];
        out[(size_t)i * NPROJ + c] = o;
      }
    }
  };
  center(P, nullptr);
  if (cheb_steps) {
    // Chebyshev recurrence on [0, cheb_b]: y1 = (2/b) P y0 - y0,
    // y_{k+1} = (4/b) P y_k - 2 y_k - y_{k-1}; the pair re-centred every 8 steps
    std::vector<float> P3((size_t)n * NPROJ);
    std::vector<float>* a = &P;   // y_{k-1}
    std::vector<float>* b = &P2;  // y_k
    std::vector<float>* c = &P3;  // y_{k+1}
    step(*a, *b, nullptr, 1, 2.0f / cheb_b);
    for (uint32_t r = 1; r < cheb_steps; ++r) {
      if (r % 8 == 0) center(*b, a);
      step(*b, *c, a, 2, 4.0f / cheb_b);
      std::vector<float>* t = a;
      a = b;
      b = c;
      c = t;
    }
    if (b != &P) P.swap(*b);
    center(P, nullptr);
  }
  for (uint32_t r = 0; r < smooth_steps; ++r) {  // lazy walk steps (x + D^-1 A x) / 2
    step(P, P2, nullptr, 0, 1.0f);
    P.swap(P2);
    if (r % 8 == 7) center(P, nullptr);
  }
  center(P, nullptr);
  for (uint32_t i = 0; i < n; ++i)
    for (int c = 0; c < NPROJ; ++c) X[(size_t)i * FEAT + 1 + WALK_LEN + c] = bf16r(P[(size_t)i * NPROJ + c]);
}

// Forward, loss and backward on graphs [g0, g1). X: n x 32 features, T: n x 4
// targets, theta: flat parameters. If `upstream` is non-null the loss is
// sum_i <upstream_i, Y_i> (nb x 4 doubles) instead of the stress loss.
// Outputs: *loss, Y (nb x 4, optional), grad (num_params doubles).
void orc_mpnn_grad(uint32_t n, uint32_t G, const uint32_t* go, const uint32_t* off, const uint32_t* nbr,
                   const float* X, const float* T, int dim, const float* theta, uint32_t partners, uint64_t seed,
                   uint64_t pair_step, uint32_t g0, uint32_t g1, int emulate, const double* upstream, double* loss,
                   double* Yout, double* grad) {
  const Csr g{n, G, go, off, nbr};
  const Layout L = layout();
  const uint32_t n0 = go[g0], nb = go[g1] - n0;
  auto rd = [&](double x) { return emulate ? (double)bf16r((float)x) : x; };
  std::vector<double> W(L.total);
  for (size_t k = 0; k < L.total; ++k) W[k] = theta[k];
  std::vector<double> Wq(W);  // weights as the GEMMs and the head read them
  if (emulate)
    for (size_t k = 0; k < L.total; ++k) Wq[k] = bf16r(theta[k]);

  // ---- forward
  std::vector<std::vector<double>> A(3);  // A_l: nb x kin_l
  std::vector<double> H3((size_t)nb * HID), Y((size_t)nb * 4, 0.0);
  A[0].assign((size_t)nb * 2 * FEAT, 0.0);
  for (uint32_t w = 0; w < nb; ++w)
    for (int c = 0; c < FEAT; ++c) A[0][(size_t)w * 2 * FEAT + c] = X[(size_t)(n0 + w) * FEAT + c];
  auto aggregate = [&](std::vector<double>& Al, int D, int ld) {
    for (uint32_t w = 0; w < nb; ++w) {
      const uint32_t i = n0 + w, d = g.deg(i);
      for (int c = 0; c < D; ++c) {
        double m = 0.0;
        if (d) {
          if (emulate) {
            const float s = row_sum_f32(g, i, [&](uint32_t j) { return (float)Al[(size_t)(j - n0) * ld + c]; });
            m = bf16r(s / (float)d);
          } else {
            double s = 0.0;
            for (uint32_t e = off[i]; e < off[i + 1]; ++e) s += Al[(size_t)(nbr[e] - n0) * ld + c];
            m = s / d;
          }
        }
        Al[(size_t)w * ld + D + c] = m;
      }
    }
  };
  aggregate(A[0], FEAT, 2 * FEAT);
  for (int l = 0; l < 3; ++l) {
    const int kin = L.kin[l];
    std::vector<double>* next = nullptr;
    if (l < 2) {
      A[l + 1].assign((size_t)nb * 2 * HID, 0.0);
      next = &A[l + 1];
    }
    for (uint32_t w = 0; w < nb; ++w) {
      const double* a = &A[l][(size_t)w * kin];
      for (int c = 0; c < HID; ++c) {
        double z = 0.0;
        for (int k = 0; k < kin; ++k) z += a[k] * Wq[L.w[l] + (size_t)k * HID + c];
        z = emulate ? (double)((float)z + theta[L.b[l] + c]) : z + W[L.b[l] + c];
        const double h = rd(z > 0.0 ? z : 0.0);
        if (next) (*next)[(size_t)w * 2 * HID + c] = h;
        else H3[(size_t)w * HID + c] = h;
      }
    }
    if (next) aggregate(*next, HID, 2 * HID);
  }
  for (uint32_t w = 0; w < nb; ++w)
    for (int c = 0; c < 3; ++c) {
      if (c >= dim) continue;
      double y = 0.0;
      for (int k = 0; k < HID; ++k) y += H3[(size_t)w * HID + k] * Wq[L.wh + (size_t)k * 4 + c];
      Y[(size_t)w * 4 + c] = y + W[L.bh + c];
    }
  if (Yout) std::memcpy(Yout, Y.data(), Y.size() * 8);

  // ---- loss and dL/dY
  std::vector<double> dY((size_t)nb * 4, 0.0);
  double total = 0.0;
  if (upstream) {
    for (size_t k = 0; k < dY.size(); ++k) {
      dY[k] = (k % 4) < (size_t)dim ? upstream[k] : 0.0;
      total += dY[k] * Y[k];
    }
  } else {
    auto pair_node = [&](uint32_t i, uint32_t q, uint32_t* j) {
      const uint32_t d = g.deg(i);
      if (q < d) {
        *j = nbr[off[i] + q];
        return true;
      }
      uint32_t gi = g0;
      while (go[gi + 1] <= i) ++gi;
      const uint32_t gb = go[gi], ng = go[gi + 1] - gb;
      if (ng < 2) return false;
      const uint32_t r = gb + pick(hash4(seed ^ SALT_PAIR, i, q - d, pair_step), ng - 1);
      *j = r + (r >= i ? 1u : 0u);
      return true;
    };
    auto tdist = [&](uint32_t i, uint32_t j) {
      double s = 0.0;
      for (int c = 0; c < 3; ++c) {
        const double x = (double)T[(size_t)i * 4 + c] - (double)T[(size_t)j * 4 + c];
        s += x * x;
      }
      return std::sqrt(s);
    };
    auto ydiff = [&](uint32_t i, uint32_t j, double* dv) {
      double s = 0.0;
      for (int c = 0; c < 3; ++c) {
        dv[c] = Y[(size_t)(i - n0) * 4 + c] - Y[(size_t)(j - n0) * 4 + c];
        s += dv[c] * dv[c];
      }
      return std::sqrt(s);
    };
    const uint32_t ngr = g1 - g0;
    std::vector<double> S1(ngr, 0.0), S2(ngr, 0.0), P(ngr, 0.0), alpha(ngr, 0.0), coef(ngr, 0.0);
    for (uint32_t gi = g0; gi < g1; ++gi)
      for (uint32_t i = go[gi]; i < go[gi + 1]; ++i)
        for (uint32_t q = 0; q < g.deg(i) + partners; ++q) {
          uint32_t j;
          if (!pair_node(i, q, &j)) continue;
          const double dt = tdist(i, j);
          if (!(dt >= 1e-6)) continue;
          double dv[3];
          const double qq = ydiff(i, j, dv) / dt;
          S1[gi - g0] += qq;
          S2[gi - g0] += qq * qq;
          P[gi - g0] += 1.0;
        }
    double cnt = 0.0;
    for (uint32_t k = 0; k < ngr; ++k) {
      alpha[k] = S2[k] > 0.0 ? S1[k] / S2[k] : 0.0;
      if (P[k] > 0.0) {
        total += S2[k] > 0.0 ? 1.0 - S1[k] * S1[k] / (S2[k] * P[k]) : 1.0;
        cnt += 1.0;
      }
    }
    if (cnt > 0.0) total /= cnt;
    for (uint32_t k = 0; k < ngr; ++k) coef[k] = (P[k] > 0.0 && cnt > 0.0) ? 2.0 / (P[k] * cnt) : 0.0;
    for (uint32_t gi = g0; gi < g1; ++gi)
      for (uint32_t i = go[gi]; i < go[gi + 1]; ++i) {
        double acc[3] = {0.0, 0.0, 0.0};
        for (uint32_t q = 0; q < g.deg(i) + partners; ++q) {
          uint32_t j;
          if (!pair_node(i, q, &j)) continue;
          const double dt = tdist(i, j);
          if (!(dt >= 1e-6)) continue;
          double dv[3];
          const double r = ydiff(i, j, dv);
          if (!(r > 1e-12)) continue;
          const double a = alpha[gi - g0];
          const double wgt = coef[gi - g0] * (a * r / dt - 1.0) * a / (dt * r);
          for (int c = 0; c < 3; ++c) acc[c] += wgt * dv[c];
        }
        for (int c = 0; c < 3; ++c) dY[(size_t)(i - n0) * 4 + c] = acc[c];
      }
  }
  *loss = total;

  // ---- backward
  std::vector<double> gr(L.total, 0.0);
  for (int k = 0; k < HID; ++k)
    for (int c = 0; c < 3; ++c) {
      double s = 0.0;
      for (uint32_t w = 0; w < nb; ++w) s += H3[(size_t)w * HID + k] * dY[(size_t)w * 4 + c];
      gr[L.wh + (size_t)k * 4 + c] = s;
    }
  for (int c = 0; c < 3; ++c) {
    double s = 0.0;
    for (uint32_t w = 0; w < nb; ++w) s += dY[(size_t)w * 4 + c];
    gr[L.bh + c] = s;
  }
  std::vector<double> dZ((size_t)nb * HID);
  for (uint32_t w = 0; w < nb; ++w)
    for (int k = 0; k < HID; ++k) {
      double v = 0.0;
      for (int c = 0; c < 3; ++c) v += dY[(size_t)w * 4 + c] * Wq[L.wh + (size_t)k * 4 + c];
      dZ[(size_t)w * HID + k] = H3[(size_t)w * HID + k] > 0.0 ? rd(v) : 0.0;
    }
  for (int l = 2; l >= 0; --l) {
    const int kin = L.kin[l];
    const std::vector<double>& Al = A[l];
    for (int k = 0; k < kin; ++k)
      for (int c = 0; c < HID; ++c) {
        double s = 0.0;
        for (uint32_t w = 0; w < nb; ++w) s += Al[(size_t)w * kin + k] * dZ[(size_t)w * HID + c];
        gr[L.w[l] + (size_t)k * HID + c] = s;
      }
    for (int c = 0; c < HID; ++c) {
      double s = 0.0;
      for (uint32_t w = 0; w < nb; ++w) s += dZ[(size_t)w * HID + c];
      gr[L.b[l] + c] = s;
    }
    if (l == 0) break;
    std::vector<double> dA((size_t)nb * kin);
    for (uint32_t w = 0; w < nb; ++w)
      for (int k = 0; k < kin; ++k) {
        double s = 0.0;
        for (int c = 0; c < HID; ++c) s += dZ[(size_t)w * HID + c] * Wq[L.w[l] + (size_t)k * HID + c];
        dA[(size_t)w * kin + k] = rd(s);
      }
    std::vector<double> nz((size_t)nb * HID);
    for (uint32_t w = 0; w < nb; ++w) {
      const uint32_t i = n0 + w;
      for (int c = 0; c < HID; ++c) {
        double s = 0.0;
        for (uint32_t e = off[i]; e < off[i + 1]; ++e) {
          const uint32_t j = nbr[e];
          s += dA[(size_t)(j - n0) * kin + HID + c] / (double)g.deg(j);
        }
        const double v = dA[(size_t)w * kin + c] + s;
        nz[(size_t)w * HID + c] = Al[(size_t)w * kin + c] > 0.0 ? rd(v) : 0.0;
      }
    }
    dZ.swap(nz);
  }
  std::memcpy(grad, gr.data(), gr.size() * 8);
}

}  // extern "C"
