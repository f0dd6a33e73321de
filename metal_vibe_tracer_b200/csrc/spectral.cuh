// spectral.cuh — the RGB -> spectrum uplift on the device (bounded MESE of three trigonometric
// moments; Peters, Merzbach, Hanika, Dachsbacher 2019).
//
// Reference: spectral_eotf / spectral_code85 / spectral_cell / spectral_moments_coarse /
// spectral_moments / spectral_lagrange / spectral_from_lagrange (main.swift:849-907), the runtime
// multipliers vibe_fourier_lagrange and reflectance (scripts/generate_spectral_tables.py:621-664),
// and spectral_emission_weights / spectral_emission_basis (main.swift:917-931). Float arithmetic in
// the reference's operation order; the grid (86^3 float4 nodes (c0, c1, c2, refined slot + 1) then
// 64-entry refined blocks) is built by spectral.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace vtd {

constexpr uint32_t kGridN = 86u;
constexpr uint32_t kGridNodes = kGridN * kGridN * kGridN;  // refined blocks start here (float4 units)
constexpr uint32_t kGridCells = 85u * 85u * 85u;
constexpr uint32_t kRefinedCapacity = 8192u;
constexpr float kMomentEps = 1e-4f;
constexpr float kInvPiF = 0.318309886f;

struct UpliftView {
  const float4 *grid;  // kGridNodes + 64 * refined blocks
  const float *nodes;  // 86 linear values of codes 0, 3, ..., 255
};

__device__ __forceinline__ float srgb_eotf_f(float v) {
  return v <= 0.04045f ? v / 12.92f : powf((v + 0.055f) / 1.055f, 2.4f);
}
__device__ __forceinline__ float srgb_code85_f(float c) {
  return (c <= 0.0031308f ? 12.92f * c : 1.055f * powf(c, 1.0f / 2.4f) - 0.055f) * 85.0f;
}
__device__ __forceinline__ uint32_t spectral_cell_f(float code85) {
  return min((uint32_t)fmaxf(code85, 0.0f), kGridN - 2u);
}
__device__ __forceinline__ float saturate_f(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// Trilinear interpolation of the coarse nodes around cell i (in linear light).
__device__ __forceinline__ float3 spectral_moments_coarse(const UpliftView &U, float3 c, uint3 i) {
  const float tx = saturate_f((c.x - U.nodes[i.x]) / (U.nodes[i.x + 1u] - U.nodes[i.x]));
  const float ty = saturate_f((c.y - U.nodes[i.y]) / (U.nodes[i.y + 1u] - U.nodes[i.y]));
  const float tz = saturate_f((c.z - U.nodes[i.z]) / (U.nodes[i.z + 1u] - U.nodes[i.z]));
  float3 m = make_float3(0.0f, 0.0f, 0.0f);
#pragma unroll
  for (uint32_t a = 0; a < 2u; ++a)
#pragma unroll
    for (uint32_t b = 0; b < 2u; ++b) {
      const uint32_t row = ((i.x + a) * kGridN + (i.y + b)) * kGridN + i.z;
      const float w = (a == 0u ? 1.0f - tx : tx) * (b == 0u ? 1.0f - ty : ty);
      const float4 g0 = __ldg(U.grid + row), g1 = __ldg(U.grid + row + 1u);
      m.x += w * ((1.0f - tz) * g0.x + tz * g1.x);
      m.y += w * ((1.0f - tz) * g0.y + tz * g1.y);
      m.z += w * ((1.0f - tz) * g0.z + tz * g1.z);
    }
  return m;
}

// Moments of a linear colour in [0, 1]: the coarse cell, or its refined block at one-code spacing.
__device__ __forceinline__ float3 spectral_moments(const UpliftView &U, float3 c) {
  const float3 code85 = make_float3(srgb_code85_f(c.x), srgb_code85_f(c.y), srgb_code85_f(c.z));
  const uint3 i = make_uint3(spectral_cell_f(code85.x), spectral_cell_f(code85.y), spectral_cell_f(code85.z));
  const float slot = __ldg(U.grid + (i.x * kGridN + i.y) * kGridN + i.z).w;
  if (!(slot > 0.0f)) return spectral_moments_coarse(U, c, i);
  const uint3 s = make_uint3(min((uint32_t)fmaxf(code85.x * 3.0f - float(3u * i.x), 0.0f), 2u),
                             min((uint32_t)fmaxf(code85.y * 3.0f - float(3u * i.y), 0.0f), 2u),
                             min((uint32_t)fmaxf(code85.z * 3.0f - float(3u * i.z), 0.0f), 2u));
  const float n0x = float(3u * i.x + s.x), n0y = float(3u * i.y + s.y), n0z = float(3u * i.z + s.z);
  const float tx = saturate_f((c.x - srgb_eotf_f(n0x / 255.0f)) / (srgb_eotf_f((n0x + 1.0f) / 255.0f) - srgb_eotf_f(n0x / 255.0f)));
  const float ty = saturate_f((c.y - srgb_eotf_f(n0y / 255.0f)) / (srgb_eotf_f((n0y + 1.0f) / 255.0f) - srgb_eotf_f(n0y / 255.0f)));
  const float tz = saturate_f((c.z - srgb_eotf_f(n0z / 255.0f)) / (srgb_eotf_f((n0z + 1.0f) / 255.0f) - srgb_eotf_f(n0z / 255.0f)));
  const float4 *block = U.grid + kGridNodes + 64u * ((uint32_t)slot - 1u);
  float3 m = make_float3(0.0f, 0.0f, 0.0f);
#pragma unroll
  for (uint32_t a = 0; a < 2u; ++a)
#pragma unroll
    for (uint32_t b = 0; b < 2u; ++b) {
      const uint32_t row = ((s.x + a) * 4u + (s.y + b)) * 4u + s.z;
      const float w = (a == 0u ? 1.0f - tx : tx) * (b == 0u ? 1.0f - ty : ty);
      const float4 g0 = __ldg(block + row), g1 = __ldg(block + row + 1u);
      m.x += w * ((1.0f - tz) * g0.x + tz * g1.x);
      m.y += w * ((1.0f - tz) * g0.y + tz * g1.y);
      m.z += w * ((1.0f - tz) * g0.z + tz * g1.z);
    }
  return m;
}

// Complex float pairs.
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 sc2(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float dot2f(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }

// Bounded-MESE Lagrange multipliers of moments c (Eqs. 6, 7, 10; Levinson's recursion with the
// Appendix A biasing of invalid moments, so every input yields a reflectance).
__device__ __forceinline__ float3 fourier_lagrange(float3 c) {
  const float pi = 3.14159265358979f;
  const float c0 = fminf(fmaxf(c.x, kMomentEps), 1.0f - kMomentEps);
  const float2 g0p = sc2(make_float2(sinpif(c0), -cospif(c0)), 1.0f / (4.0f * pi));
  const float g0 = 2.0f * g0p.x;
  float2 g1 = sc2(make_float2(-g0p.y, g0p.x), 2.0f * pi * c.y);
  float2 g2 = sc2(make_float2(-(2.0f * c.z * g0p.y + c.y * g1.y), 2.0f * c.z * g0p.x + c.y * g1.x), pi);
  const float q0 = 1.0f / g0;
  float2 u1 = sc2(g1, q0);
  float n1 = dot2f(u1, u1), keep = 0.9999f;
  if (n1 >= 1.0f) {
    u1 = sc2(u1, keep * rsqrtf(n1));
    g1 = sc2(u1, 1.0f / q0);
    n1 = keep * keep;
    keep = 0.0f;
  }
  const float d1 = 1.0f / (1.0f - n1);
  const float a0 = q0 * d1;
  const float2 a1 = sc2(u1, -(q0 * d1));
  float2 u2 = add2(sc2(g2, a0), cmulf(a1, g1));
  float n2 = dot2f(u2, u2);
  if (n2 >= 1.0f) {
    u2 = sc2(u2, keep * rsqrtf(n2));
    g2 = sc2(sub2(u2, cmulf(a1, g1)), 1.0f / a0);
    n2 = keep * keep;
  }
  const float d2 = 1.0f / (1.0f - n2);
  const float b0 = a0 * d2;
  const float2 b1 = sc2(sub2(a1, cmulf(u2, conjf2(a1))), d2);
  const float2 b2 = sc2(u2, -(a0 * d2));
  const float2 r0 = make_float2(b0 * b0 + dot2f(b1, b1) + dot2f(b2, b2), 0.0f);
  const float2 r1 = add2(cmulf(conjf2(b1), make_float2(b0, 0.0f)), cmulf(conjf2(b2), b1));
  const float2 r2 = cmulf(conjf2(b2), make_float2(b0, 0.0f));
  const float2 s0 = add2(add2(cmulf(g0p, r0), cmulf(g1, r1)), cmulf(g2, r2));
  const float2 s1 = add2(cmulf(g0p, r1), cmulf(g1, r2));
  const float2 s2 = cmulf(g0p, r2);
  const float scale = 2.0f / b0;
  return make_float3(s0.y * scale, s1.y * scale, s2.y * scale);
}

// (L0, L1, L2, 1), or (value, 0, 0, 2) for a grey (within 1e-4: flat spectra).
__device__ __forceinline__ float4 spectral_lagrange(const UpliftView &U, float3 rgb) {
  const float3 c = make_float3(saturate_f(rgb.x), saturate_f(rgb.y), saturate_f(rgb.z));
  const float lo = fminf(c.x, fminf(c.y, c.z)), hi = fmaxf(c.x, fmaxf(c.y, c.z));
  if (hi - lo <= 1e-4f) return make_float4((c.x + c.y + c.z) / 3.0f, 0.0f, 0.0f, 2.0f);
  const float3 L = fourier_lagrange(spectral_moments(U, c));
  return make_float4(L.x, L.y, L.z, 1.0f);
}

// Eq. 11 at cos(phi) = x.
__device__ __forceinline__ float fourier_reflectance(float4 L, float x) {
  if (L.w == 2.0f) return L.x;
  const float series = L.x + 2.0f * L.y * x + 2.0f * L.z * (2.0f * x * x - 1.0f);
  return atanf(series) * kInvPiF + 0.5f;
}

// Smits' decomposition of an RGB emission: e = lo + secondary * (C, M or Y) + primary * (R, G or B).
struct EmissionWeights {
  float lo, secondary, primary;
  uint32_t secondaryIndex, primaryIndex;
};
__device__ __forceinline__ EmissionWeights emission_weights(float3 e) {
  e = make_float3(fmaxf(e.x, 0.0f), fmaxf(e.y, 0.0f), fmaxf(e.z, 0.0f));
  const float hi = fmaxf(e.x, fmaxf(e.y, e.z)), lo = fminf(e.x, fminf(e.y, e.z)), mid = e.x + e.y + e.z - hi - lo;
  EmissionWeights w;
  w.primaryIndex = e.x == hi ? 0u : e.y == hi ? 1u : 2u;
  w.secondaryIndex = w.primaryIndex != 2u && e.z == lo ? 2u : w.primaryIndex != 1u && e.y == lo ? 1u : 0u;
  w.lo = lo;
  w.secondary = fmaxf(mid - lo, 0.0f);
  w.primary = fmaxf(hi - mid, 0.0f);
  return w;
}
__device__ __forceinline__ float pick3(float4 v, uint32_t k) { return k == 0u ? v.x : k == 1u ? v.y : v.z; }
// basis: 2 float4 per bin, (R, G, B, 0) and (C, M, Y, 0).
__device__ __forceinline__ float emission_basis(const EmissionWeights &w, const float4 *basis, uint32_t bin) {
  return w.lo + w.secondary * pick3(__ldg(basis + 2u * bin + 1u), w.secondaryIndex) +
         w.primary * pick3(__ldg(basis + 2u * bin), w.primaryIndex);
}

}  // namespace vtd
