// spectral.cu — the RGB -> spectrum uplift's moment grid, solved and refined on the device.
//
// The reference solves the 86^3 grid offline (scripts/generate_spectral_tables.py: `solve_code` /
// `solve_lagrange` :308-340, `moments_of_lagrange` :227-239; codes 0, 3, ..., 255 per channel) and
// ships it as FourierSRGB86.bin; the renderer then flags, on the GPU, the cells whose trilinear
// interpolation misses an 8-bit code by more than 0.35 steps and solves their 4 x 4 x 4 codes
// exactly (spectral_refine_flags_kernel / spectral_refine_solve_kernel, main.swift:8187-8260;
// refineSpectralGrid, main.swift:10658-10705). Here all of it runs as kernels when a context first
// needs the uplift:
//   k_grid_solve      one thread per node: Levenberg-Marquardt in Lagrange space in double (to a
//                     1e-10 linear-sRGB residual, from a zero start), then the moments by the
//                     1024-node midpoint rule, stored as float;
//   k_refine_flags    one thread per 8-bit code (2^24): the round trip through the coarse grid;
//   k_refine_solve    64 threads per flagged cell (the first 8192 in index order): the block's
//                     exact moments, in float, from the interpolated start.
// The colour model (per nm weights and cos phase over 360-830 nm) sits in shared memory.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "spectral.cuh"
#include "vt_internal.cuh"

namespace {
using namespace vtd;

constexpr uint32_t kMaxModel = 512;  // model samples (471 for 360-830 nm)
constexpr double kPiD = 3.14159265358979323846;

__device__ __forceinline__ double srgb_eotf_d(double v) { return v <= 0.04045 ? v / 12.92 : pow((v + 0.055) / 1.055, 2.4); }

struct ModelD {
  const double *w, *c1, *c2;  // weights (3 per sample), 2 cos phi, 2 cos 2 phi
  uint32_t n;
};

// rgb_and_jacobian (generate_spectral_tables.py:276-297); J[3 * channel + multiplier].
__device__ void rgb_jac_d(const ModelD &M, const double L[3], double rgb[3], double J[9]) {
  for (int k = 0; k < 3; ++k) rgb[k] = 0.0;
  for (int k = 0; k < 9; ++k) J[k] = 0.0;
  for (uint32_t i = 0; i < M.n; ++i) {
    const double a1 = M.c1[i], a2 = M.c2[i];
    const double s = L[0] + L[1] * a1 + L[2] * a2;
    const double v = atan(s) / kPiD + 0.5, dv = 1.0 / (kPiD * (1.0 + s * s));
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double w = M.w[3 * i + k];
      rgb[k] += w * v;
      const double x = w * dv;
      J[3 * k] += x;
      J[3 * k + 1] += x * a1;
      J[3 * k + 2] += x * a2;
    }
  }
}

__device__ __forceinline__ bool solve3_d(const double m[9], const double f[3], double x[3]) {
  const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], g_ = m[5], g = m[6], h = m[7], i = m[8];
  const double det = a * (e * i - g_ * h) - b * (d * i - g_ * g) + c * (d * h - e * g);
  if (det == 0.0 || !isfinite(det)) return false;
  x[0] = (f[0] * (e * i - g_ * h) - b * (f[1] * i - g_ * f[2]) + c * (f[1] * h - e * f[2])) / det;
  x[1] = (a * (f[1] * i - g_ * f[2]) - f[0] * (d * i - g_ * g) + c * (d * f[2] - f[1] * g)) / det;
  x[2] = (a * (e * f[2] - f[1] * h) - b * (d * f[2] - f[1] * g) + f[0] * (d * h - e * g)) / det;
  return true;
}

__device__ __forceinline__ double max_abs3_d(const double f[3]) { return fmax(fabs(f[0]), fmax(fabs(f[1]), fabs(f[2]))); }

// One coarse node per thread. Shared memory: the model (3n + 2n doubles) and the 1024 midpoint
// cosines of the moment integral.
__global__ void __launch_bounds__(128) k_grid_solve(const double *__restrict__ weights, const double *__restrict__ cosPhi,
                                                    uint32_t n, float4 *__restrict__ grid,
                                                    unsigned long long *__restrict__ residual) {
  extern __shared__ double sm[];
  double *w = sm, *c1 = sm + 3 * n, *c2 = c1 + n, *xs = c2 + n;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    w[3 * i] = weights[3 * i];
    w[3 * i + 1] = weights[3 * i + 1];
    w[3 * i + 2] = weights[3 * i + 2];
    const double c = cosPhi[i];
    c1[i] = 2.0 * c;
    c2[i] = 2.0 * (2.0 * c * c - 1.0);
  }
  const double h = kPiD / 1024.0;
  for (uint32_t i = threadIdx.x; i < 1024u; i += blockDim.x) xs[i] = cos(-kPiD + (i + 0.5) * h);
  __syncthreads();
  const uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= kGridNodes) return;
  const ModelD M{w, c1, c2, n};
  const uint32_t code[3] = {min(3u * (node / (kGridN * kGridN)), 255u), min(3u * ((node / kGridN) % kGridN), 255u),
                            min(3u * (node % kGridN), 255u)};
  double target[3];
  for (int k = 0; k < 3; ++k) target[k] = fmin(fmax(srgb_eotf_d(code[k] / 255.0), 1e-4), 1.0 - 1e-4);
  double lam[3] = {0.0, 0.0, 0.0}, rgb[3], J[9];
  rgb_jac_d(M, lam, rgb, J);
  double f[3] = {target[0] - rgb[0], target[1] - rgb[1], target[2] - rgb[2]};
  double err = max_abs3_d(f), mu = 0.0;
  for (int it = 0; err > 1e-10 && it < 80; ++it) {
    double normal[9], grad[3];
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c) normal[3 * r + c] = J[r] * J[c] + J[3 + r] * J[3 + c] + J[6 + r] * J[6 + c];
      grad[r] = J[r] * f[0] + J[3 + r] * f[1] + J[6 + r] * f[2];
    }
    bool moved = false;
    for (int tries = 0; tries < 32; ++tries) {  // mu runs from 1e-6 past 1e8 within 16 tries
      double damped[9];
      for (int k = 0; k < 9; ++k) damped[k] = normal[k];
      damped[0] *= 1.0 + mu;
      damped[4] *= 1.0 + mu;
      damped[8] *= 1.0 + mu;
      double step[3];
      if (!solve3_d(damped, grad, step)) break;
      double trial[3] = {lam[0] + step[0], lam[1] + step[1], lam[2] + step[2]}, rt[3], Jt[9];
      rgb_jac_d(M, trial, rt, Jt);
      double ft[3] = {target[0] - rt[0], target[1] - rt[1], target[2] - rt[2]};
      const double et = max_abs3_d(ft);
      if (et < err) {
        mu = mu > 1e-12 ? mu * 0.1 : 0.0;
        for (int k = 0; k < 3; ++k) { lam[k] = trial[k]; f[k] = ft[k]; }
        for (int k = 0; k < 9; ++k) J[k] = Jt[k];
        err = et;
        moved = true;
        break;
      }
      mu = fmax(mu * 10.0, 1e-6);
      if (mu > 1e8) break;
    }
    if (!moved) break;
  }
  double m0 = 0.0, m1 = 0.0, m2 = 0.0;
  for (uint32_t i = 0; i < 1024u; ++i) {
    const double cp = xs[i], c2p = 2.0 * cp * cp - 1.0;
    const double v = atan(lam[0] + 2.0 * lam[1] * cp + 2.0 * lam[2] * c2p) / kPiD + 0.5;
    m0 += v;
    m1 += v * cp;
    m2 += v * c2p;
  }
  const double s = h / kPiD;
  grid[node] = make_float4((float)(m0 * s), (float)(m1 * s), (float)(m2 * s), 0.0f);
  atomicMax(residual, (unsigned long long)__double_as_longlong(err));  // residuals are >= 0
}

struct ModelF {
  const float *w, *c1, *c2;
  uint32_t n;
};

// spectral_rgb_of_lagrange (main.swift:8190-8205), float, with the Jacobian's columns when asked.
__device__ float3 rgb_of_f(const ModelF &M, float3 L, float J[9]) {
  float3 rgb = make_float3(0.0f, 0.0f, 0.0f);
  if (J)
    for (int k = 0; k < 9; ++k) J[k] = 0.0f;
  for (uint32_t i = 0; i < M.n; ++i) {
    const float c1 = M.c1[i], c2 = M.c2[i];
    const float s = L.x + L.y * c1 + L.z * c2;
    const float v = atanf(s) * kInvPiF + 0.5f;
    const float wx = M.w[3 * i], wy = M.w[3 * i + 1], wz = M.w[3 * i + 2];
    rgb.x += wx * v;
    rgb.y += wy * v;
    rgb.z += wz * v;
    if (J) {
      const float d = kInvPiF / (1.0f + s * s);
      const float dx = wx * d, dy = wy * d, dz = wz * d;
      J[0] += dx; J[1] += dx * c1; J[2] += dx * c2;
      J[3] += dy; J[4] += dy * c1; J[5] += dy * c2;
      J[6] += dz; J[7] += dz * c1; J[8] += dz * c2;
    }
  }
  return rgb;
}

__device__ __forceinline__ void load_model_f(const double *weights, const double *cosPhi, uint32_t n, float *sm) {
  float *w = sm, *c1 = sm + 3 * n, *c2 = c1 + n;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    w[3 * i] = (float)weights[3 * i];
    w[3 * i + 1] = (float)weights[3 * i + 1];
    w[3 * i + 2] = (float)weights[3 * i + 2];
    const float x = (float)cosPhi[i];
    c1[i] = 2.0f * x;
    c2[i] = 2.0f * (2.0f * x * x - 1.0f);
  }
}

__device__ __forceinline__ float code_back(float v) {
  v = saturate_f(v);
  return (v <= 0.0031308f ? 12.92f * v : 1.055f * powf(v, 1.0f / 2.4f) - 0.055f) * 255.0f;
}

// spectral_code_error over every code; flags the cell of each code that misses by > 0.35 steps.
__global__ void __launch_bounds__(256) k_refine_flags(UpliftView U, const double *__restrict__ weights,
                                                      const double *__restrict__ cosPhi, uint32_t n,
                                                      uint8_t *__restrict__ flags) {
  extern __shared__ float smf[];
  load_model_f(weights, cosPhi, n, smf);
  __syncthreads();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (1u << 24)) return;
  const float3 code = make_float3(float(tid >> 16), float((tid >> 8) & 255u), float(tid & 255u));
  const float3 c = make_float3(srgb_eotf_f(code.x / 255.0f), srgb_eotf_f(code.y / 255.0f), srgb_eotf_f(code.z / 255.0f));
  if (c.x == c.y && c.y == c.z) return;
  const uint3 i = make_uint3(spectral_cell_f(srgb_code85_f(c.x)), spectral_cell_f(srgb_code85_f(c.y)),
                             spectral_cell_f(srgb_code85_f(c.z)));
  const ModelF M{smf, smf + 3 * n, smf + 4 * n, n};
  const float3 rgb = rgb_of_f(M, fourier_lagrange(spectral_moments_coarse(U, c, i)), nullptr);
  const float d = fmaxf(fabsf(code_back(rgb.x) - code.x), fmaxf(fabsf(code_back(rgb.y) - code.y), fabsf(code_back(rgb.z) - code.z)));
  if (d > 0.35f) flags[(i.x * 85u + i.y) * 85u + i.z] = 1u;
}

__global__ void k_mark_cells(const uint32_t *__restrict__ cells, uint32_t count, float4 *__restrict__ grid) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  const uint32_t cell = cells[s], i = cell / (85u * 85u), j = (cell / 85u) % 85u, k = cell % 85u;
  grid[(i * kGridN + j) * kGridN + k].w = float(s + 1u);
}

__device__ __forceinline__ bool inverse3_f(const float m[9], float inv[9]) {
  // m row-major; inverse by cofactors.
  const float c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
  const float det = m[0] * c00 + m[1] * c01 + m[2] * c02;
  if (!(fabsf(det) > 0.0f)) return false;
  const float r = 1.0f / det;
  inv[0] = c00 * r; inv[1] = (m[2] * m[7] - m[1] * m[8]) * r; inv[2] = (m[1] * m[5] - m[2] * m[4]) * r;
  inv[3] = c01 * r; inv[4] = (m[0] * m[8] - m[2] * m[6]) * r; inv[5] = (m[2] * m[3] - m[0] * m[5]) * r;
  inv[6] = c02 * r; inv[7] = (m[1] * m[6] - m[0] * m[7]) * r; inv[8] = (m[0] * m[4] - m[1] * m[3]) * r;
  return true;
}

// A refined cell's 64 codes (spectral_refine_solve_kernel): float Levenberg-Marquardt from the
// interpolated start (40 iterations, 2e-7), then the 1024-node midpoint moments.
__global__ void __launch_bounds__(64) k_refine_solve(UpliftView U, const double *__restrict__ weights,
                                                     const double *__restrict__ cosPhi, uint32_t n,
                                                     const uint32_t *__restrict__ cells, uint32_t count,
                                                     float4 *__restrict__ blocks) {
  extern __shared__ float smf[];
  load_model_f(weights, cosPhi, n, smf);
  __syncthreads();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 64u * count) return;
  const ModelF M{smf, smf + 3 * n, smf + 4 * n, n};
  const uint32_t slot = tid / 64u, entry = tid % 64u, cell = cells[slot];
  const uint3 i = make_uint3(cell / (85u * 85u), (cell / 85u) % 85u, cell % 85u);
  const uint3 code = make_uint3(min(3u * i.x + entry / 16u, 255u), min(3u * i.y + (entry / 4u) % 4u, 255u),
                                min(3u * i.z + entry % 4u, 255u));
  const float3 c = make_float3(srgb_eotf_f(float(code.x) / 255.0f), srgb_eotf_f(float(code.y) / 255.0f),
                               srgb_eotf_f(float(code.z) / 255.0f));
  const float3 target = make_float3(fminf(fmaxf(c.x, kMomentEps), 1.0f - kMomentEps), fminf(fmaxf(c.y, kMomentEps), 1.0f - kMomentEps),
                                    fminf(fmaxf(c.z, kMomentEps), 1.0f - kMomentEps));
  float3 L = fourier_lagrange(spectral_moments_coarse(U, c, i));
  float J[9];
  float3 rgb = rgb_of_f(M, L, J);
  float3 f = make_float3(target.x - rgb.x, target.y - rgb.y, target.z - rgb.z);
  float error = fmaxf(fabsf(f.x), fmaxf(fabsf(f.y), fabsf(f.z))), mu = 0.0f;
  for (uint32_t it = 0; it < 40u && error > 2e-7f; ++it) {
    float normal[9], grad[3];
    for (int r = 0; r < 3; ++r) {
      for (int q = 0; q < 3; ++q) normal[3 * r + q] = J[r] * J[q] + J[3 + r] * J[3 + q] + J[6 + r] * J[6 + q];
      grad[r] = J[r] * f.x + J[3 + r] * f.y + J[6 + r] * f.z;
    }
    bool improved = false;
    for (uint32_t k = 0; k < 24u && !improved; ++k) {
      float damped[9], inv[9];
      for (int q = 0; q < 9; ++q) damped[q] = normal[q];
      damped[0] *= 1.0f + mu;
      damped[4] *= 1.0f + mu;
      damped[8] *= 1.0f + mu;
      if (!inverse3_f(damped, inv)) break;
      const float3 trial = make_float3(L.x + inv[0] * grad[0] + inv[1] * grad[1] + inv[2] * grad[2],
                                       L.y + inv[3] * grad[0] + inv[4] * grad[1] + inv[5] * grad[2],
                                       L.z + inv[6] * grad[0] + inv[7] * grad[1] + inv[8] * grad[2]);
      float Jt[9];
      const float3 rt = rgb_of_f(M, trial, Jt);
      const float3 ft = make_float3(target.x - rt.x, target.y - rt.y, target.z - rt.z);
      const float et = fmaxf(fabsf(ft.x), fmaxf(fabsf(ft.y), fabsf(ft.z)));
      if (et < error) {
        L = trial;
        for (int q = 0; q < 9; ++q) J[q] = Jt[q];
        f = ft;
        error = et;
        mu = mu > 1e-12f ? mu * 0.1f : 0.0f;
        improved = true;
      } else {
        mu = fmaxf(mu * 10.0f, 1e-6f);
      }
    }
    if (!improved) break;
  }
  float3 m = make_float3(0.0f, 0.0f, 0.0f);
  for (uint32_t k = 0; k < 1024u; ++k) {
    const float x = cosf(-3.14159265358979f + (float(k) + 0.5f) * (3.14159265358979f / 1024.0f));
    const float c2 = 2.0f * x * x - 1.0f;
    const float g = atanf(L.x + 2.0f * L.y * x + 2.0f * L.z * c2) * kInvPiF + 0.5f;
    m.x += g;
    m.y += g * x;
    m.z += g * c2;
  }
  blocks[64u * slot + entry] = make_float4(m.x / 1024.0f, m.y / 1024.0f, m.z / 1024.0f, 0.0f);
}

__global__ void k_lagrange(UpliftView U, const float *__restrict__ rgb, uint32_t n, float4 *__restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = spectral_lagrange(U, make_float3(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]));
}

__global__ void k_emission_basis(const float4 *__restrict__ corners, const float *__restrict__ cosPhase, uint32_t nbins,
                                 float4 *__restrict__ basis) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbins) return;
  const float x = cosPhase[b];
  basis[2u * b] = make_float4(fourier_reflectance(corners[0], x), fourier_reflectance(corners[1], x),
                              fourier_reflectance(corners[2], x), 0.0f);
  basis[2u * b + 1u] = make_float4(fourier_reflectance(corners[3], x), fourier_reflectance(corners[4], x),
                                   fourier_reflectance(corners[5], x), 0.0f);
}

// The round-trip check over every code (tests/Fix_spectral.swift's spectral_round_trip kernel).
__global__ void __launch_bounds__(256) k_round_trip(UpliftView U, const double *__restrict__ weights,
                                                    const double *__restrict__ cosPhi, uint32_t n,
                                                    unsigned int *__restrict__ worstBits, unsigned int *__restrict__ over) {
  extern __shared__ float smf[];
  load_model_f(weights, cosPhi, n, smf);
  __syncthreads();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  float d = 0.0f;
  if (tid < (1u << 24)) {
    const float3 code = make_float3(float(tid >> 16), float((tid >> 8) & 255u), float(tid & 255u));
    const float3 c = make_float3(srgb_eotf_f(code.x / 255.0f), srgb_eotf_f(code.y / 255.0f), srgb_eotf_f(code.z / 255.0f));
    const float4 L = spectral_lagrange(U, c);
    const ModelF M{smf, smf + 3 * n, smf + 4 * n, n};
    float3 rgb;
    if (L.w == 2.0f) {
      float3 sw = make_float3(0.0f, 0.0f, 0.0f);
      for (uint32_t i = 0; i < n; ++i) {
        sw.x += M.w[3 * i];
        sw.y += M.w[3 * i + 1];
        sw.z += M.w[3 * i + 2];
      }
      rgb = make_float3(L.x * sw.x, L.x * sw.y, L.x * sw.z);
    } else {
      rgb = rgb_of_f(M, make_float3(L.x, L.y, L.z), nullptr);
    }
    d = fmaxf(fabsf(code_back(rgb.x) - code.x), fmaxf(fabsf(code_back(rgb.y) - code.y), fabsf(code_back(rgb.z) - code.z)));
  }
  const unsigned bad = __ballot_sync(0xffffffffu, d > 0.5f);
  float m = d;
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31u) == 0u) {
    atomicMax(worstBits, __float_as_uint(m));  // nonnegative floats order as their bits
    if (bad) atomicAdd(over, (unsigned)__popc(bad));
  }
}

vt_status check_tables(vt_ctx *ctx, const vt_spectral_tables *t) {
  if (!t || !t->uplift_weights || !t->uplift_cos || t->uplift_n < 2 || t->uplift_n > kMaxModel)
    return vt_fail(ctx, VT_ERR_INVALID, "spectral tables need the uplift's colour model (uplift_weights, uplift_cos, "
                                        "2 <= uplift_n <= 512)");
  return VT_OK;
}

struct DeviceModel {
  double *d = nullptr;
  ~DeviceModel() { cudaFree(d); }
};

}  // namespace

vt_status vt_uplift_ensure(vt_ctx *ctx, const vt_spectral_tables *t) {
  {
    const vt_status st = check_tables(ctx, t);
    if (st != VT_OK) return st;
  }
  const uint32_t n = t->uplift_n;
  std::vector<double> model(4 * (size_t)n);
  std::memcpy(model.data(), t->uplift_weights, 3 * (size_t)n * sizeof(double));
  std::memcpy(model.data() + 3 * (size_t)n, t->uplift_cos, (size_t)n * sizeof(double));
  if (ctx->d_fgrid) {
    if (model != ctx->fgrid_model)
      return vt_fail(ctx, VT_ERR_INVALID, "the context's uplift grid was solved for another colour model");
    return VT_OK;
  }
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  DeviceModel dm;
  unsigned long long *d_res = nullptr;
  uint8_t *d_flags = nullptr;
  uint32_t *d_cells = nullptr;
  float4 *grid = nullptr;
  float *gnodes = nullptr;
  auto cleanup = [&]() {
    cudaFree(d_res);
    cudaFree(d_flags);
    cudaFree(d_cells);
    cudaFree(grid);
    cudaFree(gnodes);
  };
#define VT_UPLIFT_CUDA(call)                                  \
  do {                                                        \
    const cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) { cleanup(); return vt_cuda_fail(ctx, _e, #call); } \
  } while (0)
  VT_UPLIFT_CUDA(cudaMalloc(&dm.d, model.size() * sizeof(double)));
  VT_UPLIFT_CUDA(cudaMemcpy(dm.d, model.data(), model.size() * sizeof(double), cudaMemcpyHostToDevice));
  const double *dW = dm.d, *dC = dm.d + 3 * (size_t)n;
  VT_UPLIFT_CUDA(cudaMalloc(&grid, ((size_t)kGridNodes + 64u * (size_t)kRefinedCapacity) * sizeof(float4)));
  VT_UPLIFT_CUDA(cudaMalloc(&gnodes, kGridN * sizeof(float)));
  VT_UPLIFT_CUDA(cudaMalloc(&d_res, sizeof(unsigned long long)));
  VT_UPLIFT_CUDA(cudaMalloc(&d_flags, kGridCells));
  VT_UPLIFT_CUDA(cudaMemsetAsync(d_res, 0, sizeof(unsigned long long), s));
  VT_UPLIFT_CUDA(cudaMemsetAsync(d_flags, 0, kGridCells, s));
  float hnodes[kGridN];
  for (uint32_t i = 0; i < kGridN; ++i) {
    const double v = 3.0 * i / 255.0;
    hnodes[i] = (float)(v <= 0.04045 ? v / 12.92 : std::pow((v + 0.055) / 1.055, 2.4));
  }
  VT_UPLIFT_CUDA(cudaMemcpyAsync(gnodes, hnodes, sizeof hnodes, cudaMemcpyHostToDevice, s));
  // 1. Coarse nodes.
  const size_t smemD = (5 * (size_t)n + 1024) * sizeof(double);
  VT_UPLIFT_CUDA(cudaFuncSetAttribute(k_grid_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemD));
  k_grid_solve<<<(kGridNodes + 127) / 128, 128, smemD, s>>>(dW, dC, n, grid, d_res);
  VT_UPLIFT_CUDA(cudaGetLastError());
  // 2. Flag the cells that interpolate a code worse than 0.35 steps.
  const UpliftView U{grid, gnodes};
  const size_t smemF = 5 * (size_t)n * sizeof(float);
  k_refine_flags<<<(1u << 24) / 256, 256, smemF, s>>>(U, dW, dC, n, d_flags);
  VT_UPLIFT_CUDA(cudaGetLastError());
  std::vector<uint8_t> flags(kGridCells);
  unsigned long long resBits = 0;
  VT_UPLIFT_CUDA(cudaMemcpyAsync(flags.data(), d_flags, kGridCells, cudaMemcpyDeviceToHost, s));
  VT_UPLIFT_CUDA(cudaMemcpyAsync(&resBits, d_res, sizeof resBits, cudaMemcpyDeviceToHost, s));
  VT_UPLIFT_CUDA(cudaStreamSynchronize(s));
  std::vector<uint32_t> cells;
  uint32_t flagged = 0;
  for (uint32_t i = 0; i < kGridCells; ++i)
    if (flags[i]) {
      ++flagged;
      if (cells.size() < kRefinedCapacity) cells.push_back(i);
    }
  // 3. Exact blocks for the flagged cells.
  if (!cells.empty()) {
    const uint32_t count = (uint32_t)cells.size();
    VT_UPLIFT_CUDA(cudaMalloc(&d_cells, count * sizeof(uint32_t)));
    VT_UPLIFT_CUDA(cudaMemcpyAsync(d_cells, cells.data(), count * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    k_refine_solve<<<count, 64, smemF, s>>>(U, dW, dC, n, d_cells, count, grid + kGridNodes);
    VT_UPLIFT_CUDA(cudaGetLastError());
    k_mark_cells<<<(count + 255) / 256, 256, 0, s>>>(d_cells, count, grid);
    VT_UPLIFT_CUDA(cudaGetLastError());
    VT_UPLIFT_CUDA(cudaStreamSynchronize(s));
  }
#undef VT_UPLIFT_CUDA
  cudaFree(d_res);
  cudaFree(d_flags);
  cudaFree(d_cells);
  ctx->d_fgrid = grid;
  ctx->d_gnodes = gnodes;
  ctx->fgrid_cells = (uint32_t)cells.size();
  ctx->fgrid_flagged = flagged;
  double res;
  std::memcpy(&res, &resBits, sizeof res);
  ctx->fgrid_residual = res;
  ctx->fgrid_model = std::move(model);
  return VT_OK;
}

// Lagrange quadruples of n host colours into a device array (scene materials, emission corners).
vt_status vt_uplift_colours(vt_ctx *ctx, const float *rgb, uint32_t n, float4 *out_dev) {
  if (n == 0) return VT_OK;
  if (!ctx->d_fgrid) return vt_fail(ctx, VT_ERR_INVALID, "the uplift grid is not built");
  float *d_rgb = nullptr;
  VT_CUDA(ctx, cudaMalloc(&d_rgb, 3 * (size_t)n * sizeof(float)));
  cudaError_t e = cudaMemcpyAsync(d_rgb, rgb, 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    k_lagrange<<<(n + 127) / 128, 128, 0, ctx->stream>>>(UpliftView{ctx->d_fgrid, ctx->d_gnodes}, d_rgb, n, out_dev);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_rgb);
  if (e != cudaSuccess) return vt_cuda_fail(ctx, e, "uplifting colours");
  return VT_OK;
}

// The emission basis at the render bins: the six saturated corners' spectra (R, G, B, C, M, Y).
vt_status vt_uplift_basis(vt_ctx *ctx, const float *cosPhase_dev, uint32_t nbins, float4 *basis_dev) {
  const float corners[18] = {1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 1, 1, 1, 0, 1, 1, 1, 0};
  float4 *d_corners = nullptr;
  VT_CUDA(ctx, cudaMalloc(&d_corners, 6 * sizeof(float4)));
  vt_status st = vt_uplift_colours(ctx, corners, 6, d_corners);
  if (st == VT_OK) {
    k_emission_basis<<<(nbins + 127) / 128, 128, 0, ctx->stream>>>(d_corners, cosPhase_dev, nbins, basis_dev);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) st = vt_cuda_fail(ctx, e, "k_emission_basis");
  }
  cudaFree(d_corners);
  return st;
}

extern "C" {

vt_status vt_spectral_grid_build(vt_ctx *ctx, const vt_spectral_tables *tables) {
  if (!ctx) return VT_ERR_INVALID;
  return vt_uplift_ensure(ctx, tables);
}

vt_status vt_spectral_grid_get_info(vt_ctx *ctx, vt_spectral_grid_info *out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!out) return vt_fail(ctx, VT_ERR_INVALID, "out is null");
  std::memset(out, 0, sizeof *out);
  out->built = ctx->d_fgrid ? 1u : 0u;
  out->refined_cells = ctx->fgrid_cells;
  out->flagged_cells = ctx->fgrid_flagged;
  out->max_residual = ctx->fgrid_residual;
  return VT_OK;
}

vt_status vt_spectral_grid_read(vt_ctx *ctx, float *out, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!out) return vt_fail(ctx, VT_ERR_INVALID, "out is null");
  if (!ctx->d_fgrid) return vt_fail(ctx, VT_ERR_INVALID, "the uplift grid is not built");
  const size_t want = 4 * ((size_t)kGridNodes + 64u * (size_t)ctx->fgrid_cells);
  if (n != want) return vt_fail(ctx, VT_ERR_INVALID, "n must be 4 * (86^3 + 64 * refined_cells)");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  VT_CUDA(ctx, cudaMemcpy(out, ctx->d_fgrid, want * sizeof(float), cudaMemcpyDeviceToHost));
  return VT_OK;
}

vt_status vt_spectral_lagrange(vt_ctx *ctx, const float *rgb, uint32_t n, float *out) {
  if (!ctx) return VT_ERR_INVALID;
  if ((!rgb || !out) && n) return vt_fail(ctx, VT_ERR_INVALID, "rgb or out is null");
  if (!ctx->d_fgrid) return vt_fail(ctx, VT_ERR_INVALID, "the uplift grid is not built (vt_spectral_grid_build)");
  if (n == 0) return VT_OK;
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  float4 *d_out = nullptr;
  VT_CUDA(ctx, cudaMalloc(&d_out, (size_t)n * sizeof(float4)));
  vt_status st = vt_uplift_colours(ctx, rgb, n, d_out);
  if (st == VT_OK) {
    const cudaError_t e = cudaMemcpy(out, d_out, (size_t)n * sizeof(float4), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = vt_cuda_fail(ctx, e, "cudaMemcpy(lagrange)");
  }
  cudaFree(d_out);
  return st;
}

vt_status vt_spectral_round_trip(vt_ctx *ctx, float *worst, uint32_t *over_half) {
  if (!ctx) return VT_ERR_INVALID;
  if (!worst || !over_half) return vt_fail(ctx, VT_ERR_INVALID, "worst or over_half is null");
  if (!ctx->d_fgrid) return vt_fail(ctx, VT_ERR_INVALID, "the uplift grid is not built (vt_spectral_grid_build)");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  const uint32_t n = (uint32_t)(ctx->fgrid_model.size() / 4);
  double *d_model = nullptr;
  unsigned int *d_acc = nullptr;
  VT_CUDA(ctx, cudaMalloc(&d_model, ctx->fgrid_model.size() * sizeof(double)));
  cudaError_t e = cudaMalloc(&d_acc, 2 * sizeof(unsigned int));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_model, ctx->fgrid_model.data(), ctx->fgrid_model.size() * sizeof(double), cudaMemcpyHostToDevice,
                        ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_acc, 0, 2 * sizeof(unsigned int), ctx->stream);
  if (e == cudaSuccess) {
    k_round_trip<<<(1u << 24) / 256, 256, 5 * (size_t)n * sizeof(float), ctx->stream>>>(
        UpliftView{ctx->d_fgrid, ctx->d_gnodes}, d_model, d_model + 3 * (size_t)n, n, d_acc, d_acc + 1);
    e = cudaGetLastError();
  }
  unsigned int h[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d_acc, sizeof h, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_model);
  cudaFree(d_acc);
  if (e != cudaSuccess) return vt_cuda_fail(ctx, e, "k_round_trip");
  std::memcpy(worst, &h[0], sizeof(float));
  *over_half = h[1];
  return VT_OK;
}

}  // extern "C"
