// SPDX-License-Identifier: Apache-2.0
// Derivative work of the Adobe OpenPBR BSDF (https://github.com/adobe/openpbr-bsdf, c91aad1d),
// Copyright 2026 Adobe, licensed under the Apache License, Version 2.0 (LICENSES/Apache-2.0.txt,
// http://www.apache.org/licenses/LICENSE-2.0); modified as described below and in NOTICE.
// openpbr.cu — the OpenPBR energy tables on the device, and the BSDF's diagnostic entry point.
//
// The dense isotropic GGX energy complement (the reference's Shaders/MetalEnergy.metal, generated
// by scripts/generate_metal_energy.py on a Metal device) is solved here by one kernel: 129 roughness
// x 129 sqrt-cosine nodes, each the mean of 1 - G1(l) over 16,384 Hammersley samples of the
// spherical-cap VNDF (l the reflection of the view about the sampled normal; 0 energy when l is
// below the horizon), roughness r = i / 128, cos = max(1e-5, (j / 128)^2). The per-roughness
// average integrates the piecewise-linear table exactly (in double, on the host):
// sum over segments of offset (hi^4 - lo^4) + 0.8 slope (hi^5 - lo^5). The opaque-dielectric
// tables (32^3 and 32^2 unorm16) come from the caller (the upstream library's data).
#include <cmath>
#include <cstring>
#include <vector>

#include "openpbr.cuh"
#include "vt_internal.cuh"

namespace {
using namespace vtd;

__global__ void k_metal_energy(float *__restrict__ table) {
  const uint32_t i = blockIdx.x, j = threadIdx.x;  // roughness node, cosine node
  if (i >= kMetalEnergyN || j >= kMetalEnergyN) return;
  if (i == 0) {
    table[j] = 0.0f;
    return;
  }
  const float roughness = float(i) / 128.0f;
  const float cosine = fmaxf(1e-5f, powf(float(j) / 128.0f, 2.0f));
  const float3 v = make_float3(sqrtf(fmaxf(0.0f, 1.0f - cosine * cosine)), 0.0f, cosine);
  const float alpha = roughness * roughness;
  float sum = 0.0f;
  for (uint32_t s = 0; s < 16384u; ++s) {
    const float2 r = make_float2((float(s) + 0.5f) / 16384.0f, float(__brev(s)) * 2.3283064365386963e-10f);
    const float3 h = ggx_sample_vndf(alpha, alpha, v, r);
    const float d = 2.0f * pdot(v, h);
    const float3 l = pf3(h.x * d - v.x, h.y * d - v.y, h.z * d - v.z);  // reflect(-v, h)
    const float energy = l.z > 0.0f ? smith_g1(l, alpha, alpha) : 0.0f;
    sum += 1.0f - energy;
  }
  table[i * kMetalEnergyN + j] = sum / 16384.0f;
}

struct CaseDev {
  float base[3], metal, rough, ior, sw, diffRough;
  float n[3], wo[3], wi[3], rand[3];
  float tfWeight, tfThickness, tfIor, lambda[3];
  float coat, fuzz;
  float aniso, tangent[3];
};
struct ResultDev {
  float fcos[3], pdf, dir[3], weight[3], spdf, ok;
};
static_assert(sizeof(CaseDev) == sizeof(vt_openpbr_case), "vt_openpbr_case layout");
static_assert(sizeof(ResultDev) == sizeof(vt_openpbr_result), "vt_openpbr_result layout");

__device__ __forceinline__ PbrParams case_params(const CaseDev &c) {
  PbrParams P;
  P.base = pf3(psat(c.base[0]), psat(c.base[1]), psat(c.base[2]));
  P.metal = c.metal;
  P.rough = fmaxf(0.03f, c.rough);
  P.ior = fmaxf(1.01f, c.ior);
  P.sw = c.sw;
  P.diffRough = c.diffRough;
  P.tfWeight = c.tfWeight;
  P.tfThickness = c.tfThickness;
  P.tfIor = c.tfIor;
  // The upstream RGB wavelengths unless the case gives its own (openpbr_bsdf.h: OpenPBR_BaseRgbWavelengths_nm).
  P.lambda = c.lambda[0] > 0.0f ? pf3(c.lambda[0], c.lambda[1], c.lambda[2]) : pf3(kPbrRgbNm[0], kPbrRgbNm[1], kPbrRgbNm[2]);
  P.coat = c.coat;
  P.fuzz = c.fuzz;
  P.aniso = c.aniso;
  return P;
}

__global__ void k_openpbr_cases(PbrTables T, const CaseDev *__restrict__ cases, uint32_t n, ResultDev *__restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const CaseDev c = cases[i];
  const PbrPrepared p = pbr_prepare(case_params(c), T, pf3(c.n[0], c.n[1], c.n[2]), pf3(c.wo[0], c.wo[1], c.wo[2]), true,
                                    pf3(c.tangent[0], c.tangent[1], c.tangent[2]));
  const float3 wi = pf3(c.wi[0], c.wi[1], c.wi[2]);
  const float3 f = pbr_eval(p, T, wi);
  ResultDev r;
  r.fcos[0] = f.x; r.fcos[1] = f.y; r.fcos[2] = f.z;
  r.pdf = pbr_pdf(p, T, wi);
  float3 d = pf3(0.0f, 0.0f, 0.0f), w = pf3(0.0f, 0.0f, 0.0f);
  float q = 0.0f;
  const bool ok = pbr_sample(p, T, pf3(c.rand[0], c.rand[1], c.rand[2]), d, w, q);
  r.dir[0] = d.x; r.dir[1] = d.y; r.dir[2] = d.z;
  r.weight[0] = w.x; r.weight[1] = w.y; r.weight[2] = w.z;
  r.spdf = ok ? q : 0.0f;
  r.ok = ok ? 1.0f : 0.0f;
  out[i] = r;
}

}  // namespace

// The context's tables: the metal table (solved once) and the opaque-dielectric tables.
vt_status vt_openpbr_ensure(vt_ctx *ctx, const vt_openpbr_tables *tables) {
  if (ctx->d_pbr && (!tables || ctx->pbr_opaque)) return VT_OK;
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t nMetal = kMetalEnergyN * kMetalEnergyN, nAvg = kMetalEnergyN, nOpq = 32 * 32 * 32, nOpqAvg = 32 * 32,
               nLtc = 3 * kPbrLtc * kPbrLtc;
  if (!ctx->d_pbr) {
    float *d = nullptr;
    VT_CUDA(ctx, cudaMalloc(&d, (nMetal + nAvg + nOpq + nOpqAvg + nLtc) * sizeof(float)));
    cudaError_t e = cudaMemsetAsync(d, 0, (nMetal + nAvg + nOpq + nOpqAvg + nLtc) * sizeof(float), ctx->stream);
    if (e == cudaSuccess) {
      k_metal_energy<<<kMetalEnergyN, kMetalEnergyN, 0, ctx->stream>>>(d);
      e = cudaGetLastError();
    }
    std::vector<float> table(nMetal);
    if (e == cudaSuccess) e = cudaMemcpyAsync(table.data(), d, nMetal * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      cudaFree(d);
      return vt_cuda_fail(ctx, e, "solving the metal energy table");
    }
    std::vector<float> avg(nAvg);
    for (uint32_t r = 0; r < kMetalEnergyN; ++r) {
      double integral = 0.0;
      for (uint32_t c = 0; c < kMetalEnergyN - 1; ++c) {
        const double lo = c / 128.0, hi = (c + 1) / 128.0;
        const double a = table[r * kMetalEnergyN + c], b = table[r * kMetalEnergyN + c + 1];
        const double slope = (b - a) * 128.0, offset = a - slope * lo;
        integral += offset * (std::pow(hi, 4) - std::pow(lo, 4)) + 0.8 * slope * (std::pow(hi, 5) - std::pow(lo, 5));
      }
      avg[r] = (float)integral;
    }
    e = cudaMemcpy(d + nMetal, avg.data(), nAvg * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(d);
      return vt_cuda_fail(ctx, e, "uploading the metal average energy");
    }
    ctx->d_pbr = d;
  }
  if (tables && !ctx->pbr_opaque) {
    if (!tables->opaque_energy || !tables->opaque_average || !tables->ltc)
      return vt_fail(ctx, VT_ERR_INVALID, "OpenPBR tables need the opaque-dielectric energy tables and the fuzz LTC table");
    std::vector<float> f(nOpq + nOpqAvg);
    for (size_t i = 0; i < nOpq; ++i) f[i] = float(tables->opaque_energy[i]) * (1.0f / 65535.0f);
    for (size_t i = 0; i < nOpqAvg; ++i) f[nOpq + i] = float(tables->opaque_average[i]) * (1.0f / 65535.0f);
    VT_CUDA(ctx, cudaMemcpy(ctx->d_pbr + nMetal + nAvg, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
    VT_CUDA(ctx, cudaMemcpy(ctx->d_pbr + nMetal + nAvg + nOpq + nOpqAvg, tables->ltc, nLtc * sizeof(float), cudaMemcpyHostToDevice));
    ctx->pbr_opaque = true;
  }
  return VT_OK;
}

extern "C" {

vt_status vt_openpbr_tables_set(vt_ctx *ctx, const vt_openpbr_tables *tables) {
  if (!ctx) return VT_ERR_INVALID;
  if (!tables) return vt_fail(ctx, VT_ERR_INVALID, "tables is null");
  return vt_openpbr_ensure(ctx, tables);
}

vt_status vt_openpbr_energy_table(vt_ctx *ctx, float *table, float *average) {
  if (!ctx) return VT_ERR_INVALID;
  if (!table || !average) return vt_fail(ctx, VT_ERR_INVALID, "table or average is null");
  {
    const vt_status st = vt_openpbr_ensure(ctx, nullptr);
    if (st != VT_OK) return st;
  }
  VT_CUDA(ctx, cudaMemcpy(table, ctx->d_pbr, kMetalEnergyN * kMetalEnergyN * sizeof(float), cudaMemcpyDeviceToHost));
  VT_CUDA(ctx, cudaMemcpy(average, ctx->d_pbr + kMetalEnergyN * kMetalEnergyN, kMetalEnergyN * sizeof(float),
                          cudaMemcpyDeviceToHost));
  return VT_OK;
}

vt_status vt_openpbr_evaluate(vt_ctx *ctx, const vt_openpbr_case *cases, uint32_t n, vt_openpbr_result *out) {
  if (!ctx) return VT_ERR_INVALID;
  if ((!cases || !out) && n) return vt_fail(ctx, VT_ERR_INVALID, "cases or out is null");
  if (!ctx->pbr_opaque) return vt_fail(ctx, VT_ERR_INVALID, "OpenPBR tables are not set (vt_openpbr_tables_set)");
  if (n == 0) return VT_OK;
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  CaseDev *dc = nullptr;
  ResultDev *dr = nullptr;
  VT_CUDA(ctx, cudaMalloc(&dc, (size_t)n * sizeof(CaseDev)));
  cudaError_t e = cudaMalloc(&dr, (size_t)n * sizeof(ResultDev));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dc, cases, (size_t)n * sizeof(CaseDev), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    k_openpbr_cases<<<(n + 127) / 128, 128, 0, ctx->stream>>>(pbr_tables_at(ctx->d_pbr), dc, n, dr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, dr, (size_t)n * sizeof(ResultDev), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(dc);
  cudaFree(dr);
  if (e != cudaSuccess) return vt_cuda_fail(ctx, e, "k_openpbr_cases");
  return VT_OK;
}

}  // extern "C"
