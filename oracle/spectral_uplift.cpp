// spectral_uplift.cpp — RGB -> spectrum uplift, restated in double (test infrastructure only: the
// CPU checker for the CUDA uplift in metal_vibe_tracer_b200/csrc/spectral.cu).
//
// A bounded linear-sRGB colour becomes a reflectance spectrum through three trigonometric moments
// of Peters' bounded MESE on an even phase warp (Peters, Merzbach, Hanika, Dachsbacher 2019, "Using
// Moments to Represent Bounded Signals for Spectral Rendering"):
//   * moments of a colour: trilinear interpolation of an 86^3 grid of exactly solved nodes (codes
//     0, 3, ..., 255), with cells the interpolation reproduces worse than 0.35 8-bit steps replaced
//     by exact 4x4x4 blocks (main.swift:842-897, 8187-8260);
//   * Lagrange multipliers from moments: Eqs. 6, 7, 10 with Levinson's recursion and the Appendix A
//     biasing (scripts/generate_spectral_tables.py:621-656, main.swift:8635-8668);
//   * the reflectance, Eq. 11: atan(L0 + 2 L1 cos phi + 2 L2 cos 2 phi) / pi + 1/2 (main.swift:900-907);
//   * the exact solve: Levenberg-Marquardt in Lagrange space to 1e-10 in linear sRGB, then the moments
//     by a 1024-node midpoint rule (scripts/generate_spectral_tables.py:227-340);
//   * emission: Smits' decomposition over the six saturated corners' spectra (main.swift:913-931).
// Grid nodes are solved on demand and remembered, so a check touches only the cells it needs.
#include "spectral_uplift.h"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <unordered_map>

namespace vto_uplift_impl {
namespace {
constexpr double kPi = 3.14159265358979323846;
constexpr double kEps = 1e-4;       // moment clamp of c0 and the solver's target clamp
constexpr int kNodes = 1024;        // midpoint rule of the moments
constexpr double kTolerance = 1e-10;
}  // namespace

double srgb_eotf(double v) { return v <= 0.04045 ? v / 12.92 : std::pow((v + 0.055) / 1.055, 2.4); }
double srgb_oetf(double v) {
  v = std::min(std::max(v, 0.0), 1.0);
  return v <= 0.0031308 ? 12.92 * v : 1.055 * std::pow(v, 1.0 / 2.4) - 0.055;
}

// Complex helpers on (re, im) pairs.
namespace {
struct Cx {
  double x, y;
};
Cx cmul(Cx a, Cx b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
Cx cconj(Cx a) { return {a.x, -a.y}; }
Cx cadd(Cx a, Cx b) { return {a.x + b.x, a.y + b.y}; }
Cx csub(Cx a, Cx b) { return {a.x - b.x, a.y - b.y}; }
Cx cscale(Cx a, double s) { return {a.x * s, a.y * s}; }
double cdot(Cx a, Cx b) { return a.x * b.x + a.y * b.y; }
}  // namespace

void fourier_lagrange(const double c[3], double L[3]) {
  const double c0 = std::min(std::max(c[0], kEps), 1.0 - kEps);
  const Cx g0p = cscale(Cx{std::sin(kPi * c0), -std::cos(kPi * c0)}, 1.0 / (4.0 * kPi));  // Eq. 6
  const double g0 = 2.0 * g0p.x;
  Cx g1 = cscale(Cx{-g0p.y, g0p.x}, 2.0 * kPi * c[1]);                                    // Eq. 7
  Cx g2 = cscale(Cx{-(2.0 * c[2] * g0p.y + c[1] * g1.y), 2.0 * c[2] * g0p.x + c[1] * g1.x}, kPi);
  const double q0 = 1.0 / g0;
  Cx u1 = cscale(g1, q0);
  double n1 = cdot(u1, u1), keep = 0.9999;
  if (n1 >= 1.0) {  // biasing (FOURIERSRGB2019 Alg. 2)
    u1 = cscale(u1, keep / std::sqrt(n1));
    g1 = cscale(u1, 1.0 / q0);
    n1 = keep * keep;
    keep = 0.0;
  }
  const double d1 = 1.0 / (1.0 - n1);
  const double a0 = q0 * d1;
  const Cx a1 = cscale(u1, -q0 * d1);
  Cx u2 = cadd(cscale(g2, a0), cmul(a1, g1));
  double n2 = cdot(u2, u2);
  if (n2 >= 1.0) {
    u2 = cscale(u2, keep / std::sqrt(n2));
    g2 = cscale(csub(u2, cmul(a1, g1)), 1.0 / a0);
    n2 = keep * keep;
  }
  const double d2 = 1.0 / (1.0 - n2);
  const double b0 = a0 * d2;
  const Cx b1 = cscale(csub(a1, cmul(u2, cconj(a1))), d2);
  const Cx b2 = cscale(u2, -a0 * d2);
  // Eq. 10: lambda_l = 2 Im(sum_k gamma'_k sum_j conj(b_{j+k+l}) b_j) / b0.
  const Cx r0 = {b0 * b0 + cdot(b1, b1) + cdot(b2, b2), 0.0};
  const Cx r1 = cadd(cmul(cconj(b1), Cx{b0, 0.0}), cmul(cconj(b2), b1));
  const Cx r2 = cmul(cconj(b2), Cx{b0, 0.0});
  const Cx s0 = cadd(cadd(cmul(g0p, r0), cmul(g1, r1)), cmul(g2, r2));
  const Cx s1 = cadd(cmul(g0p, r1), cmul(g1, r2));
  const Cx s2 = cmul(g0p, r2);
  L[0] = s0.y * (2.0 / b0);
  L[1] = s1.y * (2.0 / b0);
  L[2] = s2.y * (2.0 / b0);
}

double reflectance(const double L[3], double cos_phi) {
  return std::atan(L[0] + 2.0 * L[1] * cos_phi + 2.0 * L[2] * (2.0 * cos_phi * cos_phi - 1.0)) / kPi + 0.5;
}

Model::Model(const double *weights, const double *cos_phi, uint32_t n) : n_(n), w_(3 * n), cos1_(n), cos2_(n) {
  for (uint32_t i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) w_[3 * i + k] = weights[3 * i + k];
    const double c = cos_phi[i];
    cos1_[i] = 2.0 * c;
    cos2_[i] = 2.0 * (2.0 * c * c - 1.0);
  }
}

// rgb_of_lagrange / rgb_and_jacobian (generate_spectral_tables.py:263-297); J row-major (rgb x L).
void Model::rgb_of(const double L[3], double rgb[3], double *J) const {
  rgb[0] = rgb[1] = rgb[2] = 0.0;
  if (J) std::fill(J, J + 9, 0.0);
  for (uint32_t i = 0; i < n_; ++i) {
    const double a1 = cos1_[i], a2 = cos2_[i];
    const double s = L[0] + L[1] * a1 + L[2] * a2;
    const double v = std::atan(s) / kPi + 0.5;
    for (int k = 0; k < 3; ++k) rgb[k] += w_[3 * i + k] * v;
    if (J) {
      const double dv = 1.0 / (kPi * (1.0 + s * s));
      for (int k = 0; k < 3; ++k) {
        const double x = w_[3 * i + k] * dv;
        J[3 * k] += x;
        J[3 * k + 1] += x * a1;
        J[3 * k + 2] += x * a2;
      }
    }
  }
}

namespace {
bool solve3(const double m[9], const double f[3], double x[3]) {
  const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], g_ = m[5], g = m[6], h = m[7], i = m[8];
  const double det = a * (e * i - g_ * h) - b * (d * i - g_ * g) + c * (d * h - e * g);
  if (det == 0.0 || !std::isfinite(det)) return false;
  x[0] = (f[0] * (e * i - g_ * h) - b * (f[1] * i - g_ * f[2]) + c * (f[1] * h - e * f[2])) / det;
  x[1] = (a * (f[1] * i - g_ * f[2]) - f[0] * (d * i - g_ * g) + c * (d * f[2] - f[1] * g)) / det;
  x[2] = (a * (e * f[2] - f[1] * h) - b * (d * f[2] - f[1] * g) + f[0] * (d * h - e * g)) / det;
  return true;
}
double max_abs3(const double f[3]) { return std::max(std::fabs(f[0]), std::max(std::fabs(f[1]), std::fabs(f[2]))); }
}  // namespace

// solve_lagrange (generate_spectral_tables.py:308-340): Levenberg-Marquardt, damping on the normal
// matrix's diagonal, accepted steps must lower the largest residual.
double Model::solve(const double target[3], const double start[3], double L[3]) const {
  double lam[3] = {start[0], start[1], start[2]}, rgb[3], J[9];
  rgb_of(lam, rgb, J);
  double f[3] = {target[0] - rgb[0], target[1] - rgb[1], target[2] - rgb[2]};
  double err = max_abs3(f), mu = 0.0;
  for (int n = 0; err > kTolerance && n < 80; ++n) {
    double normal[9], grad[3];
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c) normal[3 * r + c] = J[r] * J[c] + J[3 + r] * J[3 + c] + J[6 + r] * J[6 + c];
      grad[r] = J[r] * f[0] + J[3 + r] * f[1] + J[6 + r] * f[2];
    }
    bool moved = false;
    while (true) {
      double damped[9];
      std::copy(normal, normal + 9, damped);
      damped[0] *= 1.0 + mu;
      damped[4] *= 1.0 + mu;
      damped[8] *= 1.0 + mu;
      double step[3];
      if (!solve3(damped, grad, step)) break;
      double trial[3] = {lam[0] + step[0], lam[1] + step[1], lam[2] + step[2]}, rt[3], Jt[9];
      rgb_of(trial, rt, Jt);
      double ft[3] = {target[0] - rt[0], target[1] - rt[1], target[2] - rt[2]};
      const double et = max_abs3(ft);
      if (et < err) {
        mu = mu > 1e-12 ? mu * 0.1 : 0.0;
        std::copy(trial, trial + 3, lam);
        std::copy(Jt, Jt + 9, J);
        std::copy(ft, ft + 3, f);
        err = et;
        moved = true;
        break;
      }
      mu = std::max(mu * 10.0, 1e-6);
      if (mu > 1e8) break;
    }
    if (!moved) break;
  }
  std::copy(lam, lam + 3, L);
  return err;
}

// moments_of_lagrange (generate_spectral_tables.py:227-239).
void moments_of(const double L[3], double c[3]) {
  const double h = kPi / kNodes;
  double c0 = 0.0, c1 = 0.0, c2 = 0.0;
  for (int i = 0; i < kNodes; ++i) {
    const double cp = std::cos(-kPi + (i + 0.5) * h), c2p = 2.0 * cp * cp - 1.0;
    const double v = std::atan(L[0] + 2.0 * L[1] * cp + 2.0 * L[2] * c2p) / kPi + 0.5;
    c0 += v;
    c1 += v * cp;
    c2 += v * c2p;
  }
  c[0] = c0 * h / kPi;
  c[1] = c1 * h / kPi;
  c[2] = c2 * h / kPi;
}

// solve_code (generate_spectral_tables.py:381-386) from a zero start: target = the code's linear
// value clamped to [eps, 1 - eps].
double Model::solve_code(const uint32_t code[3], double c[3], double L[3]) const {
  double target[3];
  for (int k = 0; k < 3; ++k) target[k] = std::min(std::max(srgb_eotf(code[k] / 255.0), kEps), 1.0 - kEps);
  const double zero[3] = {0.0, 0.0, 0.0};
  const double err = solve(target, zero, L);
  moments_of(L, c);
  return err;
}

void Model::node(uint32_t i, uint32_t j, uint32_t k, double c[3]) const {
  const uint32_t key = (i * 86u + j) * 86u + k;
  {
    std::lock_guard<std::mutex> g(mu_);
    auto it = nodes_.find(key);
    if (it != nodes_.end()) {
      std::copy(it->second.begin(), it->second.end(), c);
      return;
    }
  }
  const uint32_t code[3] = {std::min(3u * i, 255u), std::min(3u * j, 255u), std::min(3u * k, 255u)};
  double L[3];
  solve_code(code, c, L);
  std::lock_guard<std::mutex> g(mu_);
  nodes_[key] = {c[0], c[1], c[2]};
}

void Model::block_entry(uint32_t ci, uint32_t cj, uint32_t ck, uint32_t a, uint32_t b, uint32_t d, double c[3]) const {
  const uint32_t key = 0x80000000u | (((ci * 85u + cj) * 85u + ck) << 6) | (a << 4) | (b << 2) | d;
  {
    std::lock_guard<std::mutex> g(mu_);
    auto it = nodes_.find(key);
    if (it != nodes_.end()) {
      std::copy(it->second.begin(), it->second.end(), c);
      return;
    }
  }
  const uint32_t code[3] = {std::min(3u * ci + a, 255u), std::min(3u * cj + b, 255u), std::min(3u * ck + d, 255u)};
  double L[3];
  solve_code(code, c, L);
  std::lock_guard<std::mutex> g(mu_);
  nodes_[key] = {c[0], c[1], c[2]};
}

namespace {
double code85_of(double v) { return srgb_oetf(v) * 85.0; }
uint32_t cell_of(double code85) { return (uint32_t)std::min(std::max(code85, 0.0), 84.0); }
double sat(double v) { return std::min(std::max(v, 0.0), 1.0); }
}  // namespace

// spectral_moments_coarse (main.swift:856-869): trilinear in linear light between the cell's nodes.
void Model::moments_coarse(const double rgb[3], const uint32_t cell[3], double m[3]) const {
  double t[3];
  for (int k = 0; k < 3; ++k) {
    const double lo = srgb_eotf(3.0 * cell[k] / 255.0), hi = srgb_eotf(3.0 * (cell[k] + 1) / 255.0);
    t[k] = sat((rgb[k] - lo) / (hi - lo));
  }
  m[0] = m[1] = m[2] = 0.0;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int d = 0; d < 2; ++d) {
        const double w = (a ? t[0] : 1.0 - t[0]) * (b ? t[1] : 1.0 - t[1]) * (d ? t[2] : 1.0 - t[2]);
        double c[3];
        node(cell[0] + a, cell[1] + b, cell[2] + d, c);
        for (int k = 0; k < 3; ++k) m[k] += w * c[k];
      }
}

// spectral_code_error (main.swift:8207-8217): one 8-bit code through the unrefined conversion.
double Model::code_error(const uint32_t code[3]) const {
  double c[3];
  for (int k = 0; k < 3; ++k) c[k] = srgb_eotf(code[k] / 255.0);
  if (c[0] == c[1] && c[1] == c[2]) return 0.0;
  uint32_t cell[3];
  for (int k = 0; k < 3; ++k) cell[k] = cell_of(code85_of(c[k]));
  double m[3], L[3], rgb[3];
  moments_coarse(c, cell, m);
  fourier_lagrange(m, L);
  rgb_of(L, rgb, nullptr);
  double worst = 0.0;
  for (int k = 0; k < 3; ++k) worst = std::max(worst, std::fabs(srgb_oetf(sat(rgb[k])) * 255.0 - code[k]));
  return worst;
}

// A cell is refined when one of its codes (3i .. 3i + 2, and 255 in the last cell) round-trips worse
// than 0.35 steps (spectral_refine_flags_kernel, main.swift:8218-8226).
bool Model::refined(const uint32_t cell[3]) const {
  const uint32_t key = 0x40000000u | ((cell[0] * 85u + cell[1]) * 85u + cell[2]);
  {
    std::lock_guard<std::mutex> g(mu_);
    auto it = flags_.find(key);
    if (it != flags_.end()) return it->second;
  }
  bool r = false;
  const uint32_t na = cell[0] == 84u ? 4u : 3u, nb = cell[1] == 84u ? 4u : 3u, nd = cell[2] == 84u ? 4u : 3u;
  for (uint32_t a = 0; a < na && !r; ++a)
    for (uint32_t b = 0; b < nb && !r; ++b)
      for (uint32_t d = 0; d < nd && !r; ++d) {
        const uint32_t code[3] = {3u * cell[0] + a, 3u * cell[1] + b, 3u * cell[2] + d};
        r = code_error(code) > 0.35;
      }
  std::lock_guard<std::mutex> g(mu_);
  flags_[key] = r;
  return r;
}

// spectral_moments (main.swift:870-887).
void Model::moments(const double rgb[3], double m[3]) const {
  double code85[3];
  uint32_t cell[3];
  for (int k = 0; k < 3; ++k) {
    code85[k] = code85_of(rgb[k]);
    cell[k] = cell_of(code85[k]);
  }
  if (!refined(cell)) return moments_coarse(rgb, cell, m);
  uint32_t s[3];
  double t[3];
  for (int k = 0; k < 3; ++k) {
    s[k] = (uint32_t)std::min(std::max(code85[k] * 3.0 - 3.0 * cell[k], 0.0), 2.0);
    const double n0 = 3.0 * cell[k] + s[k];
    const double lo = srgb_eotf(n0 / 255.0), hi = srgb_eotf((n0 + 1.0) / 255.0);
    t[k] = sat((rgb[k] - lo) / (hi - lo));
  }
  m[0] = m[1] = m[2] = 0.0;
  for (uint32_t a = 0; a < 2; ++a)
    for (uint32_t b = 0; b < 2; ++b)
      for (uint32_t d = 0; d < 2; ++d) {
        const double w = (a ? t[0] : 1.0 - t[0]) * (b ? t[1] : 1.0 - t[1]) * (d ? t[2] : 1.0 - t[2]);
        double c[3];
        block_entry(cell[0], cell[1], cell[2], s[0] + a, s[1] + b, s[2] + d, c);
        for (int k = 0; k < 3; ++k) m[k] += w * c[k];
      }
}

// spectral_lagrange (main.swift:889-897): greys (within 1e-4) are flat, flag 2.
void Model::lagrange(const double rgb_in[3], double out[4]) const {
  double c[3];
  for (int k = 0; k < 3; ++k) c[k] = sat(rgb_in[k]);
  const double lo = std::min(c[0], std::min(c[1], c[2])), hi = std::max(c[0], std::max(c[1], c[2]));
  if (hi - lo <= 1e-4) {
    out[0] = (c[0] + c[1] + c[2]) / 3.0;
    out[1] = out[2] = 0.0;
    out[3] = 2.0;
    return;
  }
  double m[3];
  moments(c, m);
  fourier_lagrange(m, out);
  out[3] = 1.0;
}

double spectral_value(const double L[4], double cos_phi) { return L[3] == 2.0 ? L[0] : reflectance(L, cos_phi); }

// spectral_emission_weights (main.swift:917-927).
EmissionWeights emission_weights(const double e_in[3]) {
  double e[3];
  for (int k = 0; k < 3; ++k) e[k] = std::max(e_in[k], 0.0);
  const double hi = std::max(e[0], std::max(e[1], e[2])), lo = std::min(e[0], std::min(e[1], e[2]));
  const double mid = e[0] + e[1] + e[2] - hi - lo;
  EmissionWeights w;
  w.primary_index = e[0] == hi ? 0u : e[1] == hi ? 1u : 2u;
  w.secondary_index = w.primary_index != 2u && e[2] == lo ? 2u : w.primary_index != 1u && e[1] == lo ? 1u : 0u;
  w.lo = lo;
  w.secondary = std::max(mid - lo, 0.0);
  w.primary = std::max(hi - mid, 0.0);
  return w;
}

}  // namespace vto_uplift_impl

using namespace vto_uplift_impl;

struct vto_uplift {
  Model model;
  vto_uplift(const double *w, const double *c, uint32_t n) : model(w, c, n) {}
};

extern "C" {

vto_uplift *vto_uplift_create(const double *weights, const double *cos_phi, uint32_t n) {
  return new vto_uplift(weights, cos_phi, n);
}
void vto_uplift_destroy(vto_uplift *u) { delete u; }

void vto_fourier_lagrange(const double *c, double *L) { fourier_lagrange(c, L); }

double vto_uplift_solve_code(const vto_uplift *u, const uint32_t *code, double *moments, double *lagrange) {
  return u->model.solve_code(code, moments, lagrange);
}

void vto_uplift_rgb_of_lagrange(const vto_uplift *u, const double *L, double *rgb) { u->model.rgb_of(L, rgb, nullptr); }

void vto_uplift_moments_of_lagrange(const double *L, double *c) { moments_of(L, c); }

void vto_uplift_node(const vto_uplift *u, uint32_t i, uint32_t j, uint32_t k, double *c) { u->model.node(i, j, k, c); }

double vto_uplift_code_error(const vto_uplift *u, const uint32_t *code) { return u->model.code_error(code); }

int32_t vto_uplift_cell_refined(const vto_uplift *u, const uint32_t *cell) { return u->model.refined(cell) ? 1 : 0; }

void vto_spectral_lagrange(const vto_uplift *u, const double *rgb, uint32_t n, double *out4) {
  for (uint32_t i = 0; i < n; ++i) u->model.lagrange(rgb + 3 * i, out4 + 4 * i);
}

}  // extern "C"
