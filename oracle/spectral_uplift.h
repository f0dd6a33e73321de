/* spectral_uplift.h — the oracle's RGB -> spectrum uplift (test infrastructure only; see
 * spectral_uplift.cpp for the reference functions each part restates). */
#ifndef VTO_SPECTRAL_UPLIFT_H
#define VTO_SPECTRAL_UPLIFT_H

#include <stdint.h>

#ifdef __cplusplus
#include <array>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace vto_uplift_impl {

double srgb_eotf(double v);
double srgb_oetf(double v);
/* Bounded-MESE Lagrange multipliers of moments c (with biasing); Eq. 11 reflectance. */
void fourier_lagrange(const double c[3], double L[3]);
double reflectance(const double L[3], double cos_phi);
/* A (L0, L1, L2, flag) quadruple: flag 2 = flat spectrum of value L0. */
double spectral_value(const double L[4], double cos_phi);
void moments_of(const double L[3], double c[3]);

struct EmissionWeights {
  double lo, secondary, primary;
  uint32_t secondary_index, primary_index;
};
EmissionWeights emission_weights(const double e[3]);

/* The colour model (per nm weights and cos phase over 360-830 nm) and the lazily solved grid. */
class Model {
 public:
  Model(const double *weights, const double *cos_phi, uint32_t n);
  void rgb_of(const double L[3], double rgb[3], double *J) const;
  double solve(const double target[3], const double start[3], double L[3]) const;
  double solve_code(const uint32_t code[3], double c[3], double L[3]) const;
  void node(uint32_t i, uint32_t j, uint32_t k, double c[3]) const;
  void block_entry(uint32_t ci, uint32_t cj, uint32_t ck, uint32_t a, uint32_t b, uint32_t d, double c[3]) const;
  void moments_coarse(const double rgb[3], const uint32_t cell[3], double m[3]) const;
  double code_error(const uint32_t code[3]) const;
  bool refined(const uint32_t cell[3]) const;
  void moments(const double rgb[3], double m[3]) const;
  void lagrange(const double rgb[3], double out[4]) const;

 private:
  uint32_t n_;
  std::vector<double> w_, cos1_, cos2_;
  mutable std::mutex mu_;
  mutable std::unordered_map<uint32_t, std::array<double, 3>> nodes_;
  mutable std::unordered_map<uint32_t, bool> flags_;
};

}  // namespace vto_uplift_impl

extern "C" {
#endif

typedef struct vto_uplift vto_uplift;

/* weights: n x 3 (linear-sRGB CMFs x D65, Y = 1, per nm over 360-830); cos_phi: n. */
vto_uplift *vto_uplift_create(const double *weights, const double *cos_phi, uint32_t n);
void vto_uplift_destroy(vto_uplift *u);
void vto_fourier_lagrange(const double *c, double *L);
/* Exact solve of an 8-bit code: moments and multipliers; returns the residual (max |rgb - target|). */
double vto_uplift_solve_code(const vto_uplift *u, const uint32_t *code, double *moments, double *lagrange);
void vto_uplift_rgb_of_lagrange(const vto_uplift *u, const double *L, double *rgb);
void vto_uplift_moments_of_lagrange(const double *L, double *c);
/* Moments of coarse node (i, j, k), codes (3i, 3j, 3k) clamped to 255. */
void vto_uplift_node(const vto_uplift *u, uint32_t i, uint32_t j, uint32_t k, double *c);
/* Round trip of a code through the unrefined conversion, in 8-bit steps. */
double vto_uplift_code_error(const vto_uplift *u, const uint32_t *code);
int32_t vto_uplift_cell_refined(const vto_uplift *u, const uint32_t *cell);
/* spectral_lagrange of n linear colours (rgb n x 3) -> n x 4. */
void vto_spectral_lagrange(const vto_uplift *u, const double *rgb, uint32_t n, double *out4);

#ifdef __cplusplus
}
#endif
#endif
