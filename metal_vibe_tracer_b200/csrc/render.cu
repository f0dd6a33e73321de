// render.cu — the path-tracing integrator (MIS mode) and its C ABI (vt_scene_*, vt_render,
// vt_accum_*).
//
// Reference: shading_kernel (main.swift:7370-7914) with the primary hit of restir_temporal_kernel
// (main.swift:4842-4893), in the reference's MIS mode (Uniforms.samplingMode = 1) with the PCG
// sampler: per pixel and sample the stream starts at (y w + x) ^ (sampleIndex * 1999999973)
// (pixel_sampler, main.swift:508-515); the wavelength numbers hash a copy of it
// (wavelength_numbers, main.swift:2222-2231); pass 2 rehashes it (decorrelate_shading_seed,
// main.swift:109-111) before NEE (2 draws, sample_direct_light's quad branch, main.swift:2957-2978),
// BSDF sampling (3 draws, sample_bsdf's Lambert branch, main.swift:3354-3360) and Russian roulette
// after bounce 3 (1 draw, main.swift:7819-7827). Direct light uses the power heuristic against the
// BSDF pdf, BSDF hits on the emitter the complementary weight (emission_weight, main.swift:
// 3462-3466); the scattering budget is max(0, depth - 1) non-delta continuations
// (scattering_limit, main.swift:3471-3473).
//
// Spectral transport (VIBE_SPECTRAL): four hero wavelengths lambda_k = F^-1((u + k) / 4) from the
// inverse CDF, each weighted by 1 / (4 p(lambda_k)) (spectral_lambda, main.swift:810-816), tabulated
// at their 1 nm bin (spectral_bin, main.swift:828-830), converted with the sRGB CMFs where added
// (spectrum_rgb, main.swift:839-848). Supported here: grey reflectances (flat spectra, as
// spectral_lagrange treats greys, main.swift:905-910) and grey emitters under the illuminant
// (spectral_emission's white term, main.swift:945-959).
//
// Layout: a grid-stride loop over (sample group, pixel) items; an item runs its group's samples of
// one pixel in order and adds their FP64 sum to the pixel's accumulator (FP64 atomics when a call's
// samples are split into several groups to fill the GPU). Traversal is the 4-wide watertight
// traversal of traverse.cu with a per-thread local stack.
#include <algorithm>
#include <cstring>
#include <vector>

#include "sampler.cuh"
#include "trace_common.cuh"
#include "vt_internal.cuh"

namespace {
using namespace vtd;

constexpr float kInvPi = 0.318309886183790671538f;
constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kEps = 0.001f;            // ray_epsilon / ray_t_min of the procedural scenes
constexpr int kRenderStack = 96;
constexpr int kRenderBlock = 128;

struct RenderArgs {
  const float4 *nodes, *tris;
  float rootMax;
  const vt_material *mats;
  uint32_t nmat;
  float3 lc, lsu, lsv, ln, le;
  float larea;
  const float4 *spec;
  const float *icdf;
  uint32_t nbins, segments;
  float lambdaMin;
  int spectral;
  float3 cam, fwd, right, up;
  float aspect, fovScale;
  uint32_t W, H, maxDepth, first, spp;
  uint32_t mode;  // Uniforms.samplingMode: 1 MIS, 2 light sampling, 3 BSDF sampling
  uint32_t zSampler, zModel, firstFrame;  // Z++ sampler on/off, its temporal model, frame of `first`
  const float2 *jitter;
  double *accum;
};

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 mul(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 normalize3(float3 a) { return mul(a, rsqrtf(dot3(a, a))); }

// ---- traversal (the 4-wide watertight traversal with a local stack) ---------------------------
struct Hit {
  float t;
  int pos;  // BVH position of the triangle
};

__device__ bool rt_closest(const RenderArgs &A, float3 o, float3 d, float tMin, float tMax, Hit &h, int *stack) {
  const WRay wr = make_wray(o.x, o.y, o.z, d.x, d.y, d.z);
  const SlabRay sr = make_slab(o.x, o.y, o.z, d.x, d.y, d.z, A.rootMax);
  float closest = tMax;
  int best = -1;
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    Node4 nd;
    load_node(A.nodes, stack[--top], nd);
    float nearT[4];
    const int mask = node_hits(nd, sr, tMin, closest, nearT);
    const Sorted4 s = sort_children(nd, mask, nearT);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (j >= s.m || s.child[j] > 0 || beyond(s.key[j], closest)) continue;
      const int first = -s.child[j] - 1;
      for (int q = 0; q < s.count[j]; ++q) {
        const float4 *tp = A.tris + 3 * (size_t)(first + q);
        float t, b1, b2;
        if (!intersect_tri(wr, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), tMin, closest, t, b1, b2)) continue;
        closest = t;
        best = first + q;
      }
    }
#pragma unroll
    for (int j = 3; j >= 0; --j)
      if (j < s.m && s.child[j] > 0 && !beyond(s.key[j], closest) && top < kRenderStack) stack[top++] = s.child[j];
  }
  h.t = closest;
  h.pos = best;
  return best >= 0;
}

__device__ bool rt_any(const RenderArgs &A, float3 o, float3 d, float tMin, float tMax, int *stack) {
  const WRay wr = make_wray(o.x, o.y, o.z, d.x, d.y, d.z);
  const SlabRay sr = make_slab(o.x, o.y, o.z, d.x, d.y, d.z, A.rootMax);
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    Node4 nd;
    load_node(A.nodes, stack[--top], nd);
    float nearT[4];
    const int mask = node_hits(nd, sr, tMin, tMax, nearT);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!(mask >> k & 1)) continue;
      const int c = i4(nd.child, k);
      if (c > 0) { if (top < kRenderStack) stack[top++] = c; continue; }
      const int first = -c - 1, cnt = i4(nd.count, k);
      for (int q = 0; q < cnt; ++q) {
        const float4 *tp = A.tris + 3 * (size_t)(first + q);
        float t, b1, b2;
        if (intersect_tri(wr, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), tMin, tMax, t, b1, b2)) return true;
      }
    }
  }
  return false;
}

// ---- surfaces, lights, spectra -----------------------------------------------------------------
struct Surface {
  float3 pos, gn;  // position, geometric normal facing the incoming ray (the shading normal)
  uint32_t slot;
};

__device__ __forceinline__ Surface surface_at(const RenderArgs &A, const Hit &h, float3 o, float3 d) {
  Surface s;
  const float4 a = __ldg(A.tris + 3 * (size_t)h.pos), b = __ldg(A.tris + 3 * (size_t)h.pos + 1),
               c = __ldg(A.tris + 3 * (size_t)h.pos + 2);
  s.pos = add(o, mul(d, h.t));
  float3 ng = normalize3(cross3(f3(b.x - a.x, b.y - a.y, b.z - a.z), f3(c.x - a.x, c.y - a.y, c.z - a.z)));
  s.gn = dot3(ng, d) < 0.0f ? ng : mul(ng, -1.0f);
  s.slot = __float_as_uint(b.w);
  return s;
}

__device__ __forceinline__ vt_material material(const RenderArgs &A, uint32_t slot) {
  vt_material m;
  if (slot < A.nmat) return A.mats[slot];
  m.type = VT_MAT_DIFFUSE;
  m.albedo[0] = m.albedo[1] = m.albedo[2] = 0.0f;
  m.emission[0] = m.emission[1] = m.emission[2] = 0.0f;
  return m;
}

// The path's wavelengths: per lane its 1 nm bin and its share 1 / (4 p(lambda)).
struct Lanes {
  int bin[4];
  float w[4];
};

__device__ __forceinline__ Lanes make_lanes(const RenderArgs &A, float u) {
  Lanes L;
  const float seg = float(A.segments);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float x = (u + float(k)) * 0.25f * seg;
    const uint32_t i = min((uint32_t)x, A.segments - 1u);
    const float low = __ldg(A.icdf + i), width = __ldg(A.icdf + i + 1) - low;
    L.w[k] = 0.25f * seg * width;
    const float lambda = low + (x - float(i)) * width;
    L.bin[k] = (int)min((uint32_t)fminf(fmaxf(lambda - A.lambdaMin + 0.5f, 0.0f), float(A.nbins - 1u)), A.nbins - 1u);
  }
  return L;
}

// Linear sRGB of a four-lane spectrum (spectrum_rgb).
__device__ __forceinline__ float3 lanes_rgb(const RenderArgs &A, const Lanes &L, float4 s) {
  float3 rgb = f3(0.0f, 0.0f, 0.0f);
  const float v[4] = {s.x, s.y, s.z, s.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float4 c = __ldg(A.spec + L.bin[k]);
    const float a = v[k] * L.w[k];
    rgb = add(rgb, f3(a * c.x, a * c.y, a * c.z));
  }
  return rgb;
}

// Grey emission e under the illuminant, per lane.
__device__ __forceinline__ float4 lanes_emission(const RenderArgs &A, const Lanes &L, float e) {
  return make_float4(e * __ldg(A.spec + L.bin[0]).w, e * __ldg(A.spec + L.bin[1]).w, e * __ldg(A.spec + L.bin[2]).w,
                     e * __ldg(A.spec + L.bin[3]).w);
}

struct LightSample {
  float3 pos, wi;
  float dist, pdf;
};

// Quad light sample (2 draws).
__device__ __forceinline__ LightSample sample_light(const RenderArgs &A, float3 p, Sampler &seed) {
  LightSample ls;
  ls.pdf = 0.0f;
  const float2 uv = rand_f2(seed);
  const float u = uv.x, v = uv.y;
  const float3 lp = add(A.lc, add(mul(A.lsu, u), mul(A.lsv, v)));
  float3 dir = sub(lp, p);
  const float dist = sqrtf(dot3(dir, dir));
  dir = mul(dir, 1.0f / dist);
  const float cos_l = fmaxf(0.0f, -dot3(dir, A.ln));
  if (cos_l > 1e-4f) {
    ls.pos = lp;
    ls.wi = dir;
    ls.dist = dist;
    ls.pdf = dist * dist / (A.larea * cos_l);
  }
  return ls;
}

__device__ __forceinline__ float light_pdf(const RenderArgs &A, float3 p, float3 hitPos) {
  float3 dir = sub(hitPos, p);
  const float dist = sqrtf(dot3(dir, dir));
  dir = mul(dir, 1.0f / dist);
  const float cos_l = fmaxf(0.0f, -dot3(dir, A.ln));
  return cos_l <= 0.0f ? 0.0f : dist * dist / (A.larea * cos_l);
}

// ray_origin (main.swift:1366-1369) with the procedural scenes' epsilon.
__device__ __forceinline__ float3 ray_origin(float3 p, float3 gn, float3 dir) {
  return add(p, mul(gn, dot3(dir, gn) >= 0.0f ? kEps : -kEps));
}

// light_visible (main.swift:3254-3264): shadow ray from the offset origin to the sample, shortened
// by the endpoint tolerance 2 epsilon.
__device__ __forceinline__ bool light_visible(const RenderArgs &A, float3 p, float3 gn, const LightSample &ls,
                                              int *stack) {
  if (ls.pdf <= 0.0f) return false;
  const float3 o = ray_origin(p, gn, ls.wi);
  float3 delta = sub(ls.pos, o);
  const float d = sqrtf(dot3(delta, delta));
  const float tol = 2.0f * kEps;
  if (d <= tol) return false;
  delta = mul(delta, 1.0f / d);
  return !rt_any(A, o, delta, kEps, d - tol, stack);
}

__device__ __forceinline__ float power_heuristic(float pf, float pg) {
  const float scale = fmaxf(pf, pg);
  if (scale <= 0.0f) return 0.0f;
  const float f = pf / scale, g = pg / scale;
  return f * f / (f * f + g * g);
}

__device__ __forceinline__ void make_basis(float3 n, float3 &u, float3 &v) {
  const float3 up = fabsf(n.z) < 0.999f ? f3(0.0f, 0.0f, 1.0f) : f3(1.0f, 0.0f, 0.0f);
  u = normalize3(cross3(up, n));
  v = cross3(n, u);
}

// sample_cosine_hemisphere (main.swift:2462-2472).
__device__ __forceinline__ float3 cosine_hemisphere(float3 n, float r0, float r1) {
  const float phi = kTwoPi * r0;
  const float cos_th = sqrtf(r1 + (0.5f / 16777216.0f));
  const float sin_th = sqrtf(fmaxf(0.0f, 1.0f - cos_th * cos_th));
  float3 u, v;
  make_basis(n, u, v);
  float s, c;
  sincosf(phi, &s, &c);
  return normalize3(add(add(mul(u, c * sin_th), mul(v, s * sin_th)), mul(n, cos_th)));
}

__device__ __forceinline__ float grey(const float c[3]) { return (c[0] + c[1] + c[2]) * (1.0f / 3.0f); }

// Reflectance / emission as a 4-lane spectrum (spectral) or rgb in xyz (RGB transport).
__device__ __forceinline__ float4 reflectance(const RenderArgs &A, const vt_material &m) {
  if (A.spectral) { const float g = grey(m.albedo); return make_float4(g, g, g, g); }
  return make_float4(m.albedo[0], m.albedo[1], m.albedo[2], 0.0f);
}
__device__ __forceinline__ float4 emission(const RenderArgs &A, const Lanes &L, const float e[3]) {
  if (A.spectral) return lanes_emission(A, L, e[0]);
  return make_float4(e[0], e[1], e[2], 0.0f);
}
__device__ __forceinline__ float3 to_rgb(const RenderArgs &A, const Lanes &L, float4 s) {
  return A.spectral ? lanes_rgb(A, L, s) : f3(s.x, s.y, s.z);
}
__device__ __forceinline__ float4 scale4(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ float4 mul4(float4 a, float4 b) { return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
__device__ __forceinline__ float max4(const RenderArgs &A, float4 a) {
  return A.spectral ? fmaxf(fmaxf(a.x, a.y), fmaxf(a.z, a.w)) : fmaxf(fmaxf(a.x, a.y), a.z);
}

// NEE at a Lambert vertex: the contribution's rgb (2 draws).
__device__ __forceinline__ float3 direct_light(const RenderArgs &A, const Lanes &L, float3 p, float3 n, float3 wo,
                                               float4 T, float4 albedo, bool useMIS, Sampler &seed, int *stack,
                                               bool requirePdf) {
  const LightSample ls = sample_light(A, p, seed);
  if (requirePdf && !(ls.pdf > 0.0f)) return f3(0.0f, 0.0f, 0.0f);
  if (!light_visible(A, p, n, ls, stack)) return f3(0.0f, 0.0f, 0.0f);
  const float cosine = fabsf(dot3(n, ls.wi));
  // eval_bsdf / eval_bsdf_pdf for DIFFUSE (main.swift:2665-2686), shading normal = geometric.
  float f = 0.0f, bpdf = 0.0f;
  const float ni = dot3(n, ls.wi), no = dot3(n, wo);
  if (no > 0.0f) {
    bpdf = fmaxf(0.0f, ni) * kInvPi;
    if (ni > 0.0f && cosine >= 1e-7f) f = kInvPi;
  }
  const float weight = useMIS ? power_heuristic(ls.pdf, bpdf) : 1.0f;
  const float le[3] = {A.le.x, A.le.y, A.le.z};
  const float4 Le = emission(A, L, le);
  const float4 s = scale4(mul4(mul4(T, albedo), Le), f * cosine * weight / ls.pdf);
  return to_rgb(A, L, s);
}

__device__ float3 path_sample(const RenderArgs &A, uint32_t x, uint32_t y, uint32_t si, uint32_t frame, float2 jit,
                              int *stack) {
  Sampler seed = pixel_sampler(x, y, A.W, si, A.zSampler != 0u, A.zModel, frame);
  Lanes L;
  if (A.spectral) L = make_lanes(A, wavelength_numbers(seed).x);
  // Camera ray (restir_temporal_kernel, main.swift:4874-4893).
  const float jx = jit.x + 0.5f, jy = jit.y + 0.5f;
  float u = ((float(x) + jx) / float(A.W)) * 2.0f - 1.0f;
  float v = ((float(y) + jy) / float(A.H)) * 2.0f - 1.0f;
  v = -v;
  u *= A.aspect * A.fovScale;
  v *= A.fovScale;
  const float3 dir0 = normalize3(add(A.fwd, add(mul(A.right, u), mul(A.up, v))));
  Hit h;
  const bool hit0 = rt_closest(A, A.cam, dir0, kEps, __int_as_float(0x7f800000), h, stack);
  seed.state = pcg_hash(seed.state ^ 0x27d4eb2fu);  // decorrelate_shading_seed
  if (!hit0) return f3(0.0f, 0.0f, 0.0f);
  Surface S = surface_at(A, h, A.cam, dir0);
  vt_material m = material(A, S.slot);
  if (m.type == VT_MAT_EMISSIVE) return f3(m.emission[0], m.emission[1], m.emission[2]);
  const int limit = max(0, (int)A.maxDepth - 1);
  const bool nee = A.mode != 3u, mis = A.mode == 1u;
  float4 T = A.spectral ? make_float4(1.0f, 1.0f, 1.0f, 1.0f) : make_float4(1.0f, 1.0f, 1.0f, 0.0f);
  float3 R = f3(0.0f, 0.0f, 0.0f);
  if (nee) {
    sampler_event(seed, 1u, kZNee);
    R = direct_light(A, L, S.pos, S.gn, mul(dir0, -1.0f), T, reflectance(A, m), mis && limit > 0, seed, stack, true);
  }
  float3 dir = dir0;
  int scattering = 0;
  bool emissionOnly = false;
  for (int bounce = 1;; ++bounce) {
    if (scattering >= limit) {
      // BSDF-only paths take one final continuation that may only reach emission.
      if (nee || emissionOnly) break;
      emissionOnly = true;
    }
    ++scattering;
    // sample_bsdf, Lambert: one 3D draw (three PCG draws), the direction from the last two.
    sampler_event(seed, (uint32_t)bounce, kZBsdf);
    const float3 r = rand_f3(seed);
    const float3 nd = cosine_hemisphere(S.gn, r.y, r.z);
    const float bpdf = fmaxf(0.0f, dot3(S.gn, nd)) * kInvPi;
    if (!(bpdf > 0.0f) || !(dot3(nd, S.gn) > 0.0f)) break;
    T = mul4(T, reflectance(A, m));
    if (!isfinite(T.x) || !isfinite(T.y) || !isfinite(T.z) || !isfinite(T.w) || max4(A, T) <= 0.0f) break;
    const float3 prev = S.pos;
    const float3 o = ray_origin(S.pos, S.gn, nd);
    dir = nd;
    if (!rt_closest(A, o, dir, kEps, __int_as_float(0x7f800000), h, stack)) break;
    S = surface_at(A, h, o, dir);
    m = material(A, S.slot);
    if (m.type == VT_MAT_EMISSIVE) {
      // emission_weight (main.swift:3462-3466): 1 without NEE or without a light pdf, else the
      // power heuristic (MIS) or 0 (light sampling).
      const float lpdf = light_pdf(A, prev, S.pos);
      const float w = !nee || lpdf <= 0.0f ? 1.0f : (mis ? power_heuristic(bpdf, lpdf) : 0.0f);
      R = add(R, to_rgb(A, L, scale4(mul4(T, emission(A, L, m.emission)), w)));
      break;
    }
    if (emissionOnly) break;
    if (nee) {
      sampler_event(seed, (uint32_t)bounce + 1u, kZNee);
      R = add(R, direct_light(A, L, S.pos, S.gn, mul(dir, -1.0f), T, reflectance(A, m), mis && scattering < limit, seed,
                              stack, false));
    }
    if (bounce > 3) {
      const float survival = fminf(fmaxf(max4(A, T), 0.05f), 0.95f);
      sampler_event(seed, (uint32_t)bounce + 1u, kZRoulette);
      if (rand_f(seed) >= survival) break;
      T = scale4(T, 1.0f / survival);
    }
  }
  if (!isfinite(R.x) || !isfinite(R.y) || !isfinite(R.z)) R = f3(0.0f, 0.0f, 0.0f);
  return R;
}

// Work item i = (sample group g, pixel p), pixel-major within a group so that a warp traces
// neighbouring pixels; a group covers `per` consecutive samples of the call. Each item adds its
// FP64 sum to the pixel with one atomic per channel (groups > 1) or a plain add (groups = 1).
__global__ void __launch_bounds__(kRenderBlock) k_render(RenderArgs A, uint32_t groups, uint32_t per) {
  int stack[kRenderStack];
  const uint32_t npix = A.W * A.H;
  const uint64_t items = (uint64_t)npix * groups;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < items; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t p = (uint32_t)(i % npix), g = (uint32_t)(i / npix);
    const uint32_t x = p % A.W, y = p / A.W;
    const uint32_t k0 = g * per, k1 = min(A.spp, k0 + per);
    double sr = 0.0, sg = 0.0, sb = 0.0;
    for (uint32_t k = k0; k < k1; ++k) {
      const float3 c = path_sample(A, x, y, A.first + k, A.firstFrame + k, A.jitter[k], stack);
      sr += c.x;
      sg += c.y;
      sb += c.z;
    }
    double *acc = A.accum + 3 * (size_t)p;
    if (groups == 1) {
      acc[0] += sr; acc[1] += sg; acc[2] += sb;
    } else {
      atomicAdd(acc, sr); atomicAdd(acc + 1, sg); atomicAdd(acc + 2, sb);
    }
  }
}

// frameJitter (main.swift:8773-8785): base-2/base-3 Halton, 1024-frame period, minus 0.5.
float halton(uint32_t index, uint32_t base) {
  uint32_t n = index;
  float fraction = 1.0f, result = 0.0f;
  while (n > 0) {
    fraction /= float(base);
    result += fraction * float(n % base);
    n /= base;
  }
  return result;
}

void host_normalize(float v[3]) {
  const float l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  v[0] /= l; v[1] /= l; v[2] /= l;
}

}  // namespace

extern "C" {

vt_status vt_scene_create(vt_ctx *ctx, const vt_mesh *mesh, const vt_material *materials, uint32_t nmat,
                          const vt_quad_light *light, const vt_spectral_tables *tables, vt_scene **out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!out || !mesh || !light || (nmat && !materials)) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  *out = nullptr;
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  if (tables) {
    if (!tables->cmf_rgb || !tables->illuminant || !tables->icdf || tables->nbins < 2 || tables->segments < 1)
      return vt_fail(ctx, VT_ERR_INVALID, "incomplete spectral tables");
    // Spectral transport here supports grey reflectances and grey emitters (flat spectra).
    for (uint32_t i = 0; i < nmat; ++i) {
      const float *c = materials[i].type == VT_MAT_EMISSIVE ? materials[i].emission : materials[i].albedo;
      if (std::fabs(c[0] - c[1]) > 1e-4f || std::fabs(c[1] - c[2]) > 1e-4f)
        return vt_fail(ctx, VT_ERR_INVALID, "spectral transport supports grey materials only (slot " + std::to_string(i) + ")");
    }
    const float *e = light->emission;
    if (std::fabs(e[0] - e[1]) > 1e-4f || std::fabs(e[1] - e[2]) > 1e-4f)
      return vt_fail(ctx, VT_ERR_INVALID, "spectral transport supports a grey light emission only");
  }
  vt_scene *sc = new vt_scene();
  sc->mesh = mesh;
  sc->nmat = nmat;
  sc->light = *light;
  auto fail = [&](cudaError_t err, const char *what) {
    cudaFree(sc->d_mats); cudaFree(sc->d_spec); cudaFree(sc->d_icdf);
    delete sc;
    return vt_cuda_fail(ctx, err, what);
  };
  cudaError_t e;
  if (nmat) {
    if ((e = cudaMalloc(&sc->d_mats, nmat * sizeof(vt_material))) != cudaSuccess) return fail(e, "cudaMalloc(materials)");
    if ((e = cudaMemcpy(sc->d_mats, materials, nmat * sizeof(vt_material), cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail(e, "cudaMemcpy(materials)");
  }
  if (tables) {
    std::vector<float4> spec(tables->nbins);
    for (uint32_t i = 0; i < tables->nbins; ++i)
      spec[i] = make_float4(tables->cmf_rgb[3 * i], tables->cmf_rgb[3 * i + 1], tables->cmf_rgb[3 * i + 2], tables->illuminant[i]);
    sc->nbins = tables->nbins;
    sc->segments = tables->segments;
    sc->lambda_min = tables->lambda_min;
    if ((e = cudaMalloc(&sc->d_spec, spec.size() * sizeof(float4))) != cudaSuccess) return fail(e, "cudaMalloc(spectral)");
    if ((e = cudaMemcpy(sc->d_spec, spec.data(), spec.size() * sizeof(float4), cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail(e, "cudaMemcpy(spectral)");
    if ((e = cudaMalloc(&sc->d_icdf, (tables->segments + 1) * sizeof(float))) != cudaSuccess) return fail(e, "cudaMalloc(icdf)");
    if ((e = cudaMemcpy(sc->d_icdf, tables->icdf, (tables->segments + 1) * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail(e, "cudaMemcpy(icdf)");
  }
  *out = sc;
  return VT_OK;
}

vt_status vt_scene_destroy(vt_ctx *ctx, vt_scene *scene) {
  if (!scene) return VT_OK;
  if (ctx) cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  cudaFree(scene->d_mats);
  cudaFree(scene->d_spec);
  cudaFree(scene->d_icdf);
  cudaFree(scene->d_accum);
  cudaFree(scene->d_jitter);
  delete scene;
  return VT_OK;
}

vt_status vt_accum_reset(vt_ctx *ctx, vt_scene *scene) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene) return vt_fail(ctx, VT_ERR_INVALID, "scene is null");
  if (scene->d_accum)
    VT_CUDA(ctx, cudaMemset(scene->d_accum, 0, 3 * (size_t)scene->width * scene->height * sizeof(double)));
  scene->samples = 0;
  return VT_OK;
}

vt_status vt_render(vt_ctx *ctx, vt_scene *scene, const vt_frame_params *p, uint32_t spp, void *stream) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene || !p) return vt_fail(ctx, VT_ERR_INVALID, "scene or params is null");
  if (p->width == 0 || p->height == 0 || (uint64_t)p->width * p->height > (1u << 28))
    return vt_fail(ctx, VT_ERR_INVALID, "bad image size");
  if (p->sampling_mode < 1 || p->sampling_mode > 3)
    return vt_fail(ctx, VT_ERR_INVALID, "sampling_mode must be 1 (MIS), 2 (light) or 3 (BSDF)");
  if (p->spectral && !scene->d_spec) return vt_fail(ctx, VT_ERR_INVALID, "spectral transport needs spectral tables");
  if (p->first_sample == 0) return vt_fail(ctx, VT_ERR_INVALID, "first_sample starts at 1");
  if (p->sampler > 1 || p->z_temporal > 3) return vt_fail(ctx, VT_ERR_INVALID, "sampler must be 0 (PCG) or 1 (Z++), z_temporal 0-3");
  const vt_mesh *mesh = scene->mesh;
  if (mesh->nfaces > 0 && mesh->depth > 32) return vt_fail(ctx, VT_ERR_LIMIT, "BVH deeper than the render stack");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  if (p->width != scene->width || p->height != scene->height || !scene->d_accum) {
    cudaFree(scene->d_accum);
    scene->d_accum = nullptr;
    const size_t bytes = 3 * (size_t)p->width * p->height * sizeof(double);
    VT_CUDA(ctx, cudaMalloc(&scene->d_accum, bytes));
    VT_CUDA(ctx, cudaMemset(scene->d_accum, 0, bytes));
    scene->width = p->width;
    scene->height = p->height;
    scene->samples = 0;
  }
  if (spp == 0) return VT_OK;
  if (spp > scene->jitter_cap) {
    cudaFree(scene->d_jitter);
    scene->d_jitter = nullptr;
    VT_CUDA(ctx, cudaMalloc(&scene->d_jitter, spp * sizeof(float2)));
    scene->jitter_cap = spp;
  }
  std::vector<float2> jit(spp);
  for (uint32_t k = 0; k < spp; ++k) {
    const uint32_t n = (std::max(1u, p->first_sample + k) - 1u) % 1024u + 1u;
    jit[k] = make_float2(halton(n, 2) - 0.5f, halton(n, 3) - 0.5f);
  }
  VT_CUDA(ctx, cudaMemcpyAsync(scene->d_jitter, jit.data(), spp * sizeof(float2), cudaMemcpyHostToDevice, s));
  if (mesh->nfaces == 0) { scene->samples += spp; return VT_OK; }

  RenderArgs A;
  std::memset(&A, 0, sizeof A);
  A.nodes = reinterpret_cast<const float4 *>(mesh->d_nodes);
  A.tris = mesh->d_tris;
  A.rootMax = mesh->root_max;
  A.mats = scene->d_mats;
  A.nmat = scene->nmat;
  const vt_quad_light &l = scene->light;
  A.lc = make_float3(l.corner[0], l.corner[1], l.corner[2]);
  A.lsu = make_float3(l.su[0], l.su[1], l.su[2]);
  A.lsv = make_float3(l.sv[0], l.sv[1], l.sv[2]);
  A.ln = make_float3(l.normal[0], l.normal[1], l.normal[2]);
  A.le = make_float3(l.emission[0], l.emission[1], l.emission[2]);
  {
    const float cx = l.su[1] * l.sv[2] - l.su[2] * l.sv[1], cy = l.su[2] * l.sv[0] - l.su[0] * l.sv[2],
                cz = l.su[0] * l.sv[1] - l.su[1] * l.sv[0];
    A.larea = std::sqrt(cx * cx + cy * cy + cz * cz);
  }
  A.spec = scene->d_spec;
  A.icdf = scene->d_icdf;
  A.nbins = scene->nbins;
  A.segments = scene->segments;
  A.lambdaMin = scene->lambda_min;
  A.spectral = p->spectral ? 1 : 0;
  // Camera basis (main.swift:4884-4887).
  float fwd[3] = {p->camera_target[0] - p->camera_pos[0], p->camera_target[1] - p->camera_pos[1],
                  p->camera_target[2] - p->camera_pos[2]};
  host_normalize(fwd);
  float right[3] = {fwd[1] * p->camera_up[2] - fwd[2] * p->camera_up[1], fwd[2] * p->camera_up[0] - fwd[0] * p->camera_up[2],
                    fwd[0] * p->camera_up[1] - fwd[1] * p->camera_up[0]};
  host_normalize(right);
  const float up[3] = {right[1] * fwd[2] - right[2] * fwd[1], right[2] * fwd[0] - right[0] * fwd[2],
                       right[0] * fwd[1] - right[1] * fwd[0]};
  A.cam = make_float3(p->camera_pos[0], p->camera_pos[1], p->camera_pos[2]);
  A.fwd = make_float3(fwd[0], fwd[1], fwd[2]);
  A.right = make_float3(right[0], right[1], right[2]);
  A.up = make_float3(up[0], up[1], up[2]);
  A.aspect = float(p->width) / float(p->height);
  A.fovScale = std::tan((p->fov_deg * 0.5f) * 3.14159265358979323846f / 180.0f);
  A.W = p->width;
  A.H = p->height;
  A.maxDepth = p->max_depth;
  A.first = p->first_sample;
  A.spp = spp;
  A.mode = p->sampling_mode;
  A.zSampler = p->sampler;
  A.zModel = p->z_temporal;
  A.firstFrame = p->first_frame ? p->first_frame : scene->samples + 1u;
  A.jitter = scene->d_jitter;
  A.accum = scene->d_accum;
  // Enough (pixel, sample group) items to fill the GPU about four times over.
  const uint32_t npix = p->width * p->height;
  const uint64_t target = (uint64_t)ctx->sm_count * 2048u * 4u;
  uint32_t groups = (uint32_t)std::min<uint64_t>(spp, std::max<uint64_t>(1, (target + npix - 1) / npix));
  const uint32_t per = (spp + groups - 1) / groups;
  groups = (spp + per - 1) / per;
  const uint64_t items = (uint64_t)npix * groups;
  const uint32_t grid = (uint32_t)std::min<uint64_t>((items + kRenderBlock - 1) / kRenderBlock, (uint64_t)ctx->sm_count * 32u);
  k_render<<<grid, kRenderBlock, 0, s>>>(A, groups, per);
  VT_CUDA(ctx, cudaGetLastError());
  scene->samples += spp;
  return VT_OK;
}

vt_status vt_accum_readback(vt_ctx *ctx, vt_scene *scene, double *rgb, uint32_t n, uint32_t *samples) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene || !rgb) return vt_fail(ctx, VT_ERR_INVALID, "scene or rgb is null");
  const size_t want = 3 * (size_t)scene->width * scene->height;
  if (n != want) return vt_fail(ctx, VT_ERR_INVALID, "n must equal width * height * 3");
  VT_CUDA(ctx, cudaDeviceSynchronize());
  if (want) VT_CUDA(ctx, cudaMemcpy(rgb, scene->d_accum, want * sizeof(double), cudaMemcpyDeviceToHost));
  const double inv = scene->samples ? 1.0 / scene->samples : 0.0;
  for (size_t i = 0; i < want; ++i) rgb[i] *= inv;
  if (samples) *samples = scene->samples;
  return VT_OK;
}

}  // extern "C"

// ---- sampler draws (diagnostic entry point) -----------------------------------------------------
namespace {
__global__ void k_sampler_frame(uint32_t width, uint32_t height, uint32_t z, uint32_t model, uint32_t sampleIndex,
                                uint32_t frameIndex, uint32_t vertex, uint32_t stream, float *out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= width * height) return;
  const uint32_t x = i % width, y = i / width;
  Sampler s = pixel_sampler(x, y, width, sampleIndex, z != 0u, model, frameIndex);
  sampler_event(s, vertex, stream);
  const float a = rand_f(s);
  const float2 b = rand_f2(s);
  const float3 c = rand_f3(s);
  float *o = out + 6 * (size_t)i;
  o[0] = a; o[1] = b.x; o[2] = b.y; o[3] = c.x; o[4] = c.y; o[5] = c.z;
}
}  // namespace

extern "C" vt_status vt_sampler_frame(vt_ctx *ctx, uint32_t width, uint32_t height, uint32_t sampler,
                                      uint32_t z_temporal, uint32_t sample_index, uint32_t frame_index,
                                      uint32_t vertex, uint32_t stream, float *out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!out || width == 0 || height == 0 || (uint64_t)width * height > (1u << 24) || sampler > 1 || z_temporal > 3)
    return vt_fail(ctx, VT_ERR_INVALID, "bad sampler_frame arguments");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t n = (size_t)width * height;
  float *d = nullptr;
  VT_CUDA(ctx, cudaMalloc(&d, 6 * n * sizeof(float)));
  k_sampler_frame<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(width, height, sampler, z_temporal, sample_index,
                                                                          frame_index, vertex, stream, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, 6 * n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  if (e != cudaSuccess) return vt_cuda_fail(ctx, e, "vt_sampler_frame");
  return VT_OK;
}
