// nrc.cuh — the neural radiance cache's device definitions: the query record, the input encoding
// (a multiresolution hash grid of the position plus one-blob encodings of the directions and the
// roughness) and the tensor-core helpers of the fused MLP.
//
// The reference has no radiance cache; this follows Mueller et al. 2021, "Real-time Neural Radiance
// Caching for Path Tracing", with the multiresolution hash encoding of Mueller et al. 2022 ("Instant
// Neural Graphics Primitives", its spatial hash and trilinear interpolation) and the one-blob
// encoding of Mueller et al. 2019 ("Neural Importance Sampling").
//
// Input vector (64 halves): [0, 32) the grid's 16 levels x 2 features; [32, 36) one-blob(4) of the
// outgoing direction's theta / pi, [36, 40) of its phi / 2 pi + 1/2; [40, 48) the same for the
// shading normal; [48, 52) one-blob(4) of 1 - exp(-roughness); [52, 55) diffuse reflectance;
// [55] specular reflectance; [56, 60) one-blob(4) of the path's wavelength number u (spectral
// transport: the four hero wavelengths are F^-1((u + k) / 4); 0 in RGB transport); [60, 63) the
// frequency encoding sin(2 pi q) of the normalised position q (a collision-free coarse term beside
// the hash grid); [63] one (the first layer's bias).
// Network: 64 -> 64 (ReLU) x 5 hidden layers -> 4 (linear), fp16 operands, fp32 accumulation,
// no biases besides input 63. Outputs: per hero wavelength of the path its radiance over the
// illuminant at that wavelength (spectral caches), or rgb and 0 (RGB caches). Weights are stored
// [out][in], fp32 masters, the output layer padded to 16 rows (rows 4-15 stay zero).
#pragma once

#include <cuda_fp16.h>
#include <stdint.h>

#include "vt_internal.cuh"

namespace vtd {

constexpr int kNrcIn = 64;
constexpr int kNrcWidth = 64;
constexpr int kNrcHidden = 5;                 // hidden layers (64 x 64 matrices)
constexpr int kNrcOutRows = 16;               // output layer rows (kNrcOut used)
constexpr int kNrcMlpParams = kNrcHidden * kNrcWidth * kNrcIn + kNrcOutRows * kNrcWidth;  // 21,504
constexpr int kNrcMaxLevels = 16;
constexpr int kNrcLd = 72;                    // padded smem row stride in halves (144 B)
constexpr int kNrcTile = 128;                 // rows per CTA tile (4 warps x 32 rows)
constexpr int kNrcOut = 4;                    // outputs used (rows of the output layer)
// The backward pass multiplies the loss gradient by this before it meets fp16 (so that small
// per-record gradients keep their precision instead of flushing to fp16 subnormals or zero); the
// fp32 gradient sums are divided by it in the optimiser step.
constexpr float kNrcLossScale = 64.0f;

// A cache query at a path vertex (vt_nrc_input, 64 B).
struct NrcInput {
  float4 a;  // position xyz, roughness
  float4 b;  // outgoing direction (theta / pi, phi / 2 pi + 1/2), shading normal (same)
  float4 c;  // diffuse reflectance rgb, specular reflectance
  float4 d;  // wavelength number u, 0, 0, 0
};
static_assert(sizeof(NrcInput) == 64, "NrcInput layout");

// The hash grid: levels x 2^logT entries x 2 fp32 features; positions normalised by the scene box.
struct NrcGrid {
  float2 *table;
  uint32_t levels, logT;
  float lo[3], inv[3];          // position -> [0, 1]^3: (p - lo) * inv
  uint32_t res[kNrcMaxLevels];  // cells per axis per level
  uint32_t dense;               // bit l: level l indexes its (res + 1)^3 points directly
  uint32_t *status;             // index checks: an entry out of range is clamped and sets a bit
};

// Status bits of the cache's index checks (the context's status word 3).
constexpr uint32_t kNrcBadEntry = 1u, kNrcBadGradient = 2u;
__device__ __forceinline__ void nrc_fault(const NrcGrid &G, uint32_t bit) {
  if (G.status) atomicOr(G.status, bit);
}

__device__ __forceinline__ float nrc_sat(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }  // NaN -> 0

// The 8 corners of level l around normalised position q: entry indices (within the level) and
// trilinear weights. Corner c is (cx + (c & 1), cy + (c >> 1 & 1), cz + (c >> 2)); the hash terms of
// y and z and the dense strides are formed once per level.
__device__ __forceinline__ void nrc_corners(const NrcGrid &G, uint32_t l, float3 q, uint32_t (&idx)[8], float (&w)[8]) {
  const uint32_t res = G.res[l];
  const float fr = float(res);
  const float x = q.x * fr, y = q.y * fr, z = q.z * fr;
  const uint32_t cx = min((uint32_t)x, res - 1u), cy = min((uint32_t)y, res - 1u), cz = min((uint32_t)z, res - 1u);
  const float fx = x - float(cx), fy = y - float(cy), fz = z - float(cz);
  const float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {1.0f - fz, fz};
  if ((G.dense >> l) & 1u) {
    const uint32_t side = res + 1u, plane = side * side, base = cx + side * cy + plane * cz;
#pragma unroll
    for (int c = 0; c < 8; ++c) idx[c] = base + (c & 1) + ((c >> 1) & 1) * side + (c >> 2) * plane;
  } else {
    const uint32_t mask = (1u << G.logT) - 1u;
    const uint32_t hy[2] = {cy * 2654435761u, (cy + 1u) * 2654435761u};
    const uint32_t hz[2] = {cz * 805459861u, (cz + 1u) * 805459861u};
#pragma unroll
    for (int c = 0; c < 8; ++c) idx[c] = ((cx + (c & 1)) ^ hy[(c >> 1) & 1] ^ hz[c >> 2]) & mask;
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) w[c] = (wx[c & 1] * wy[(c >> 1) & 1]) * wz[c >> 2];
}

__device__ __forceinline__ float3 nrc_position(const NrcGrid &G, const NrcInput &in) {
  return make_float3(nrc_sat((in.a.x - G.lo[0]) * G.inv[0]), nrc_sat((in.a.y - G.lo[1]) * G.inv[1]),
                     nrc_sat((in.a.z - G.lo[2]) * G.inv[2]));
}

// One-blob encoding of s in [0, 1] over 4 bins: Gaussian kernels of sigma 1/4 at the bin centres.
__device__ __forceinline__ void nrc_blob4(float s, __half *out) {
  s = nrc_sat(s);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float d = (s - (float(i) + 0.5f) * 0.25f) * 4.0f;
    out[i] = __float2half_rn(__expf(-0.5f * d * d));
  }
}

// The 64-half input row of one query. Levels go in groups of four whose 32 corner loads are all
// issued before any is summed (the gathers are latency-bound L2 reads); an entry index out of range
// (none by construction) is clamped and flagged.
__device__ __forceinline__ void nrc_encode(const NrcGrid &G, const NrcInput &in, __half *row) {
  const float3 q = nrc_position(G, in);
  const uint32_t mask = (1u << G.logT) - 1u;
  bool bad = false;
#pragma unroll
  for (int grp = 0; grp < kNrcMaxLevels / 4; ++grp) {
    float2 v[4][8];
    float w[4][8];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t l = 4u * grp + j;
      if (l < G.levels) {
        uint32_t idx[8];
        nrc_corners(G, l, q, idx, w[j]);
        const float2 *lev = G.table + ((size_t)l << G.logT);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          bad |= idx[c] > mask;
          v[j][c] = __ldg(lev + min(idx[c], mask));
        }
      } else {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          v[j][c] = make_float2(0.0f, 0.0f);
          w[j][c] = 0.0f;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        f0 += w[j][c] * v[j][c].x;
        f1 += w[j][c] * v[j][c].y;
      }
      row[2 * (4 * grp + j)] = __float2half_rn(f0);
      row[2 * (4 * grp + j) + 1] = __float2half_rn(f1);
    }
  }
  if (bad) nrc_fault(G, kNrcBadEntry);
  nrc_blob4(in.b.x, row + 32);
  nrc_blob4(in.b.y, row + 36);
  nrc_blob4(in.b.z, row + 40);
  nrc_blob4(in.b.w, row + 44);
  nrc_blob4(1.0f - __expf(-fmaxf(in.a.w, 0.0f)), row + 48);
  row[52] = __float2half_rn(nrc_sat(in.c.x));
  row[53] = __float2half_rn(nrc_sat(in.c.y));
  row[54] = __float2half_rn(nrc_sat(in.c.z));
  row[55] = __float2half_rn(nrc_sat(in.c.w));
  nrc_blob4(in.d.x, row + 56);
  row[60] = __float2half_rn(sinpif(2.0f * q.x));
  row[61] = __float2half_rn(sinpif(2.0f * q.y));
  row[62] = __float2half_rn(sinpif(2.0f * q.z));
  row[63] = __float2half_rn(1.0f);
}

// (theta / pi, phi / 2 pi + 1/2) of a unit vector.
__device__ __forceinline__ float2 nrc_sphere(float3 d) {
  const float z = fminf(fmaxf(d.z, -1.0f), 1.0f);
  return make_float2(acosf(z) * 0.318309886f, atan2f(d.y, d.x) * 0.159154943f + 0.5f);
}

// ---- tensor-core helpers (mma.sync m16n8k16, fp16 x fp16 -> fp32) ---------------------------
__device__ __forceinline__ void nrc_mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ void nrc_ldsm4(uint32_t (&r)[4], const __half *p) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(s));
}
__device__ __forceinline__ void nrc_ldsm4t(uint32_t (&r)[4], const __half *p) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(s));
}
// max(0, x) of two floats as a half2 register (lo in the low 16 bits), one conversion instruction.
__device__ __forceinline__ uint32_t nrc_pack_relu(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.relu.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
// Two floats as a half2 register (lo in the low 16 bits), clamped to the finite fp16 range.
__device__ __forceinline__ uint32_t nrc_pack(float lo, float hi) {
  lo = fminf(fmaxf(lo, -65504.0f), 65504.0f);
  hi = fminf(fmaxf(hi, -65504.0f), 65504.0f);
  const __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&h);
}

}  // namespace vtd

// ---- host side: the cache object (nrc.cu) and what the integrator (render.cu) calls -----------
struct vt_nrc {
  vt_nrc_config cfg;
  vtd::NrcGrid grid;
  float *d_p = nullptr, *d_m = nullptr, *d_v = nullptr, *d_g = nullptr;  // [MLP | grid], Adam moments, gradient sums
  uint64_t nparams = 0;
  uint32_t steps = 0;
  uint32_t frames = 0;  // frames trained (training-path pixel patterns)
  // Training records of the current step: inputs, targets (rgb, 0) and their count.
  vtd::NrcInput *d_tin = nullptr;
  float4 *d_ttarget = nullptr;
  uint32_t tcap = 0;
  uint32_t *d_count = nullptr;  // [0] records written, [1] records wanted
  float4 *d_scratch = nullptr;  // training paths' records before their targets are known
  size_t scratch_cap = 0;       // float4s
  float *d_loss = nullptr;      // loss sum of the last step
  // Render queries: inputs, the resolve's per-lane throughput and lane bins, the predictions.
  vtd::NrcInput *d_q = nullptr;
  float4 *d_qT = nullptr;
  uint2 *d_qbins = nullptr;
  float4 *d_qout = nullptr;
  size_t qcap = 0;
  // A frame that trains and renders traces its training paths on `side`, beside the rendering.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_start = nullptr, ev_paths = nullptr;
};

// One optimiser step on the records in d_tin / d_ttarget (d_count[0] of them, at most cap).
vt_status vt_nrc_step(vt_ctx *ctx, vt_nrc *nrc, uint32_t cap, cudaStream_t s);
// Predictions for n device queries into out (n float4).
vt_status vt_nrc_predict(vt_ctx *ctx, vt_nrc *nrc, const vtd::NrcInput *in, uint32_t n, float4 *out, cudaStream_t s);
// The inference kernel on the tcgen05 tensor cores (nrc_tc.cu), which vt_nrc_predict launches.
vt_status vt_nrc_infer_tc(vt_ctx *ctx, vt_nrc *nrc, const vtd::NrcInput *in, uint32_t n, float4 *out, cudaStream_t s);
vt_status vt_nrc_reserve_queries(vt_ctx *ctx, vt_nrc *nrc, size_t n);
vt_status vt_nrc_reserve_records(vt_ctx *ctx, vt_nrc *nrc, uint32_t n);
