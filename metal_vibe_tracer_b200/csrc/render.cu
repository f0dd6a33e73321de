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
#include <cmath>
#include <cstring>
#include <vector>

#include "sampler.cuh"
#include "spectral.cuh"
#include "openpbr.cuh"
#include "nrc.cuh"
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
  const float4 *nrm;  // vertex normals per BVH position (3 per triangle)
  float rootMax;
  const vt_material *mats;
  uint32_t nmat;
  float3 lc, lsu, lsv, ln, le;
  float larea;
  const float4 *spec;
  const float *icdf;
  const float4 *slotL;     // per slot: the albedo's uplift multipliers (L0, L1, L2, flag)
  const float *cosPhase;   // per bin: cos of the warped phase
  const float4 *ebasis;    // per bin: the emission basis (R, G, B, 0), (C, M, Y, 0)
  const float4 *pbr;       // per slot: roughness, metalness, IOR, diffuse roughness; thin film
  PbrTables pbrT;          // OpenPBR energy tables
  uint32_t layered;        // some slot is OPENPBR, GLOSSY or DIELECTRIC (the kPbr kernel variants)
  uint32_t nbins, segments;
  float lambdaMin;
  int spectral;
  float3 cam, fwd, right, up;
  float aspect, fovScale;
  uint32_t W, H, maxDepth, first, spp;
  uint32_t stride, OW, OH;  // pixel stride; the accumulation's width and height (ceil(W / stride), ...)
  uint32_t mode;  // Uniforms.samplingMode: 1 MIS, 2 light sampling, 3 BSDF sampling
  uint32_t zSampler, zModel, firstFrame;  // Z++ sampler on/off, its temporal model, frame of `first`
  const float2 *jitter;
  double *accum;
  // Imported scenes (sceneIndex 6): emitter triangles instead of the quad light.
  uint32_t imported;
  const uint32_t *emitters;  // packed list (vt_emitter_list_pack layout)
  const float4 *emissions;   // per slot: emission rgb, selection weight
  const int32_t *facePos;    // input face -> BVH position
  uint32_t ecount, treeNodes;
  // Procedural sky and sun of imported scenes (Uniforms.environment.x, sunParams, skyMode); env = 1
  // when the sky's intensity is positive.
  int env;
  float envIntensity, sunIntensity;
  float3 sunDir;
  uint32_t skyMode;
  // Environment image (vt_scene_set_environment_map): linear-sRGB lat-long pixels, the marginal row
  // CDFs (2 per row: compensated, original) and the conditional column CDFs (the compensated table's
  // rows first), its size and rotation about +y; envMap = 1 when the image replaces the sky.
  const float4 *envImg;
  const float *envRows, *envCols;
  uint32_t envW, envH, envMap;
  float envRot;
  float etotal;
  const uint4 *ltNodes;
  const uint32_t *ltLeaves;
  float3 ltLo, ltScale;
  // ReSTIR DI (sampling mode 0): the primary-surface cache and reservoirs of this frame (written by
  // pass 1, read by pass 2) and of the previous frame (temporal reuse), and the previous camera.
  float aperture, focus;  // thin lens (aperture 0: pinhole)
  uint32_t diCandidates, diBits, history;
  float4 *gPos, *gNrm;           // (position, distance or -1), (normal, material type)
  uint4 *gInfo;                  // (face, slot | front << 31, error bits, 0)
  float4 *gGeo;                  // geometric normal (the shading normal is in gNrm)
  float4 *rPos, *rEmit, *rW;     // (position, light id bits), (emission, pdf), (weight sum, M, W, u)
  const float4 *hPos, *hNrm, *hrPos, *hrEmit, *hrW;
  // ReSTIR GI (sampling mode 0, diffuse primaries): per pixel the secondary point and its source pdf,
  // its normal and a validity flag, its outgoing direct radiance per lane, (weight sum, M, W, u); this
  // frame's and the previous frame's.
  float4 *giPos, *giNrm, *giRad, *giW;
  const float4 *hgiPos, *hgiNrm, *hgiRad, *hgiW;
  float3 pcam, pfwd, pright, pup;
  float paspect, pfovScale;
  // Radiance cache (vt_render_nrc): per (sample, pixel) slot the query at vertex nrcVertex, the
  // path's per-lane throughput there (times the lane's share) and its lanes' bins.
  NrcInput *nrcIn;
  float4 *nrcT;
  uint2 *nrcBins;
  uint32_t nrcVertex;  // 0: the spread-angle heuristic with constant nrcSpread
  float nrcSpread;
  // Index checks: a hit's triangle index is clamped into the triangle array, a training record's
  // slot into its buffers; one out of range sets a bit of *status (read back with the accumulation).
  uint32_t faceCount;
  uint32_t *status;
  uint32_t kernelId;  // which kernel a failed check was in (render_fault)
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

// Status bits of the integrator's index checks (the context's status word 2): a hit's triangle
// index, a training record's slot.
constexpr uint32_t kBadHit = 4u, kBadRecord = 8u, kBadEmitter = 16u;
// The first failure also records its value and the kernel it happened in: status words 8-10 of
// the context (status[6..8] here).
__device__ __forceinline__ void render_fault(const RenderArgs &A, uint32_t bit, uint32_t value = 0u) {
  if (!A.status) return;
  atomicOr(A.status, bit);
  if (atomicCAS(A.status + 6, 0u, 1u) == 0u) {
    A.status[7] = value;
    A.status[8] = A.kernelId | (bit << 24);
  }
}

// ---- traversal (the 4-wide watertight traversal with a local stack) ---------------------------
struct Hit {
  float t, b1, b2;
  int pos;  // BVH position of the triangle
};

__device__ bool rt_closest(const RenderArgs &A, float3 o, float3 d, float tMin, float tMax, Hit &h, int *stack) {
  const WRay wr = make_wray(o.x, o.y, o.z, d.x, d.y, d.z);
  const SlabRay sr = make_slab(o.x, o.y, o.z, d.x, d.y, d.z, A.rootMax);
  float closest = tMax, bb1 = 0.0f, bb2 = 0.0f;
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
        bb1 = b1;
        bb2 = b2;
        best = first + q;
      }
    }
#pragma unroll
    for (int j = 3; j >= 0; --j)
      if (j < s.m && s.child[j] > 0 && !beyond(s.key[j], closest) && top < kRenderStack) stack[top++] = s.child[j];
  }
  h.t = closest;
  h.b1 = bb1;
  h.b2 = bb2;
  h.pos = best;
  return best >= 0;
}

__device__ __forceinline__ float max_abs3(float x, float y, float z) { return fmaxf(fabsf(x), fmaxf(fabsf(y), fabsf(z))); }
__device__ __forceinline__ float max_abs(float3 p) { return max_abs3(p.x, p.y, p.z); }

// mesh_hit_error (main.swift:1353-1355) of an imported triangle: its vertices' rounding bound.
__device__ __forceinline__ float mesh_hit_error(float4 a, float4 b, float4 c) { return tri_error_bound(a, b, c); }

// Any hit in [tMin, tMax); with `slack` (imported scenes) each triangle's own rounding bound is
// taken off tMax, so the endpoint surface does not occlude itself (scene_occluded, main.swift:
// 2066-2069).
__device__ bool rt_any(const RenderArgs &A, float3 o, float3 d, float tMin, float tMax, int *stack, bool slack) {
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
        const float4 ta = __ldg(tp), tb = __ldg(tp + 1), tc = __ldg(tp + 2);
        float t, b1, b2;
        if (intersect_tri(wr, ta, tb, tc, tMin, slack ? tMax - mesh_hit_error(ta, tb, tc) : tMax, t, b1, b2)) return true;
      }
    }
  }
  return false;
}

// ---- surfaces, lights, spectra -----------------------------------------------------------------
struct Surface {
  float3 pos, gn;  // position, geometric normal facing the incoming ray
  float3 n;        // shading normal: the interpolated vertex normals on gn's side, else gn
  float err;       // HitRecord.error: the position's rounding bound
  uint32_t slot, face;
  uint32_t tri;    // the triangle's position in BVH order (its vertex records)
  bool front;      // the ray meets the side cross(b - a, c - a) points to
};

// ray_epsilon (main.swift:1343-1345): the procedural scenes' 0.001, or for imported scenes a bound
// that scales with the coordinates' magnitude.
__device__ __forceinline__ float ray_eps(const RenderArgs &A, float3 p) {
  return A.imported ? fmaxf(1e-7f, 9.536743e-7f * max_abs(p)) : kEps;
}
// ray_t_min (main.swift:1362-1364).
__device__ __forceinline__ float ray_tmin(const RenderArgs &A, float3 o) {
  return A.imported ? ray_eps(A, o) * 0.25f : kEps;
}

// The hit record (trace_scene and mesh_hit_attributes, main.swift:1587-1592, 2025-2032): imported
// scenes rebuild the point from barycentrics and take the triangle's rounding bound as its error.
__device__ __forceinline__ Surface surface_at(const RenderArgs &A, const Hit &h, float3 o, float3 d) {
  Surface s;
  const size_t hp = min((uint32_t)h.pos, A.faceCount - 1u);
  if ((uint32_t)h.pos >= A.faceCount) render_fault(A, kBadHit, (uint32_t)h.pos);
  const float4 a = __ldg(A.tris + 3 * hp), b = __ldg(A.tris + 3 * hp + 1), c = __ldg(A.tris + 3 * hp + 2);
  const float3 e1 = f3(b.x - a.x, b.y - a.y, b.z - a.z), e2 = f3(c.x - a.x, c.y - a.y, c.z - a.z);
  const float3 ng = normalize3(cross3(e1, e2));
  s.front = dot3(ng, d) < 0.0f;
  s.gn = s.front ? ng : mul(ng, -1.0f);
  s.slot = __float_as_uint(b.w);
  s.face = __float_as_uint(a.w);
  s.tri = (uint32_t)hp;
  const float b0 = 1.0f - h.b1 - h.b2;
  if (A.imported) {
    s.pos = add(add(mul(f3(a.x, a.y, a.z), b0), mul(f3(b.x, b.y, b.z), h.b1)), mul(f3(c.x, c.y, c.z), h.b2));
    s.err = mesh_hit_error(a, b, c);
  } else {
    s.pos = add(o, mul(d, h.t));
    s.err = kEps;
  }
  // mesh_hit_attributes (main.swift:1590-1593): smooth normal when the vertex normals give one.
  s.n = s.gn;
  if (A.nrm) {
    const float4 na = __ldg(A.nrm + 3 * hp), nb = __ldg(A.nrm + 3 * hp + 1), nc = __ldg(A.nrm + 3 * hp + 2);
    const float3 sm = add(add(mul(f3(na.x, na.y, na.z), b0), mul(f3(nb.x, nb.y, nb.z), h.b1)),
                          mul(f3(nc.x, nc.y, nc.z), h.b2));
    if (dot3(sm, sm) > 1e-12f) {
      s.n = normalize3(sm);
      if (dot3(s.n, s.gn) < 0.0f) s.n = mul(s.n, -1.0f);
    }
  }
  return s;
}

__device__ __forceinline__ vt_material material(const RenderArgs &A, uint32_t slot) {
  vt_material m;
  if (slot < A.nmat) return A.mats[slot];
  m.type = VT_MAT_DIFFUSE;
  m.albedo[0] = m.albedo[1] = m.albedo[2] = 0.0f;
  m.emission[0] = m.emission[1] = m.emission[2] = 0.0f;
  m.pad = __uint_as_float(0xffffffffu);  // no slot: black in spectral transport too
  return m;
}

// The path's wavelengths: per lane its 1 nm bin and its share 1 / (4 p(lambda)).
struct Lanes {
  int bin[4];
  float w[4];
  float u;  // the wavelength number the lanes come from
};

__device__ __forceinline__ Lanes make_lanes(const RenderArgs &A, float u) {
  Lanes L;
  L.u = u;
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

// An RGB emission e under the illuminant S, per lane (spectral_emission, main.swift:933-944): the
// emission basis at the lane's bin times S there; white is S exactly.
__device__ __forceinline__ float4 lanes_emission(const RenderArgs &A, const Lanes &L, float3 e) {
  if (!(fmaxf(e.x, fmaxf(e.y, e.z)) > 0.0f)) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (e.x == e.y && e.y == e.z)  // white: e S exactly (the basis terms have zero weight)
    return make_float4(e.x * __ldg(A.spec + L.bin[0]).w, e.x * __ldg(A.spec + L.bin[1]).w, e.x * __ldg(A.spec + L.bin[2]).w,
                       e.x * __ldg(A.spec + L.bin[3]).w);
  const EmissionWeights w = emission_weights(e);
  float v[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) v[k] = emission_basis(w, A.ebasis, (uint32_t)L.bin[k]) * __ldg(A.spec + L.bin[k]).w;
  return make_float4(v[0], v[1], v[2], v[3]);
}
// A slot's albedo as a reflectance at the lanes' bins (spectral_reflectance, main.swift:905-907).
__device__ __forceinline__ float4 lanes_reflectance(const RenderArgs &A, const Lanes &L, uint32_t slot) {
  const float4 q = __ldg(A.slotL + slot);
  if (q.w == 2.0f) return make_float4(q.x, q.x, q.x, q.x);  // a grey: flat
  return make_float4(fourier_reflectance(q, __ldg(A.cosPhase + L.bin[0])), fourier_reflectance(q, __ldg(A.cosPhase + L.bin[1])),
                     fourier_reflectance(q, __ldg(A.cosPhase + L.bin[2])), fourier_reflectance(q, __ldg(A.cosPhase + L.bin[3])));
}

struct LightSample {
  float3 pos, wi, emission;
  float dist, pdf;
  uint32_t face;  // sampled emitter triangle (imported scenes), else 0xffffffff
};

// Quad light sample (2 draws).
__device__ __forceinline__ LightSample sample_light(const RenderArgs &A, float3 p, Sampler &seed) {
  LightSample ls;
  ls.pdf = 0.0f;
  ls.face = 0xffffffffu;
  ls.emission = A.le;
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

// ---- emitter triangles: power sampling and the light tree (imported scenes) -------------------
struct Tri {
  float3 a, b, c;
  uint32_t slot;
};

__device__ __forceinline__ Tri scene_triangle(const RenderArgs &A, uint32_t face) {
  if (face >= A.faceCount) {
    render_fault(A, kBadEmitter, face);
    face = 0;
  }
  uint32_t pos = __ldg(A.facePos + face);
  if (pos >= A.faceCount) {
    render_fault(A, kBadEmitter, pos);
    pos = 0;
  }
  const float4 *t = A.tris + 3 * (size_t)pos;
  const float4 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + 2);
  return Tri{f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), f3(c.x, c.y, c.z), __float_as_uint(b.w)};
}

// imported_geometry (main.swift:2721-2725): cos at the emitter (front side) over d^2.
__device__ __forceinline__ float imported_geometry(float3 p, float3 position, const Tri &t) {
  const float3 d = sub(position, p);
  const float d2 = dot3(d, d);
  const float3 n = cross3(sub(t.b, t.a), sub(t.c, t.a));
  return d2 > 1e-12f && dot3(n, n) > 1e-20f ? fmaxf(0.0f, dot3(normalize3(n), mul(d, -rsqrtf(d2)))) / d2 : 0.0f;
}

__device__ __forceinline__ float triangle_area(const Tri &t) {
  const float3 n = cross3(sub(t.b, t.a), sub(t.c, t.a));
  return 0.5f * sqrtf(dot3(n, n));
}

struct LtNode {
  float3 lo, hi, w;
  float phi, cosO, cosE;
  uint32_t child, parent, count;
};

// light_tree_axis (main.swift:2751-2756): the octahedral cone axis.
__device__ __forceinline__ float3 lt_axis(uint32_t q) {
  const float fx = float(q & 0xffffu) / 65535.0f * 2.0f - 1.0f, fy = float(q >> 16) / 65535.0f * 2.0f - 1.0f;
  float3 v = f3(fx, fy, 1.0f - fabsf(fx) - fabsf(fy));
  if (v.z < 0.0f) {
    const float vx = (1.0f - fabsf(v.y)) * (v.x >= 0.0f ? 1.0f : -1.0f);
    const float vy = (1.0f - fabsf(v.x)) * (v.y >= 0.0f ? 1.0f : -1.0f);
    v.x = vx;
    v.y = vy;
  }
  return normalize3(v);
}

// light_tree_node (main.swift:2768-2778).
__device__ __forceinline__ LtNode lt_node(const RenderArgs &A, uint32_t i) {
  const uint4 a = __ldg(A.ltNodes + 2 * (size_t)i), b = __ldg(A.ltNodes + 2 * (size_t)i + 1);
  LtNode n;
  n.w = lt_axis(a.x);
  n.phi = __uint_as_float(a.y);
  n.cosO = float(a.z & 0xffffu) / 65535.0f * 2.0f - 1.0f;
  n.cosE = float(a.z >> 16) / 65535.0f * 2.0f - 1.0f;
  n.lo = add(A.ltLo, f3(float(a.w & 0xffffu) * A.ltScale.x, float(a.w >> 16) * A.ltScale.y, float(b.x & 0xffffu) * A.ltScale.z));
  n.hi = add(A.ltLo, f3(float(b.x >> 16) * A.ltScale.x, float(b.y & 0xffffu) * A.ltScale.y, float(b.y >> 16) * A.ltScale.z));
  n.child = b.z;
  n.parent = b.w & 0x7ffffffu;
  n.count = b.w >> 27;
  return n;
}

__device__ __forceinline__ uint32_t lt_leaf_word(const RenderArgs &A, uint32_t position, uint32_t k) {
  return __ldg(A.ltLeaves + 3 * (size_t)position + k);
}
__device__ __forceinline__ float lt_leaf_sum(const RenderArgs &A, const LtNode &n) {
  float sum = 0.0f;
  for (uint32_t i = 0; i < n.count; ++i) sum += __uint_as_float(lt_leaf_word(A, n.child + i, 1u));
  return sum;
}

__device__ __forceinline__ float cos_sub_clamped(float sinA, float cosA, float sinB, float cosB) {
  return cosA > cosB ? 1.0f : cosA * cosB + sinA * sinB;
}
__device__ __forceinline__ float sin_sub_clamped(float sinA, float cosA, float sinB, float cosB) {
  return cosA > cosB ? 0.0f : sinA * cosB - cosA * sinB;
}

// light_tree_importance (main.swift:2788-2805): pbrt-v4's bound without the receiver normal.
__device__ float lt_importance(const LtNode &n, float3 p) {
  if (!(n.phi > 0.0f)) return 0.0f;
  const float3 pc = mul(add(n.lo, n.hi), 0.5f);
  const float3 dp = sub(p, pc), ext = sub(n.hi, n.lo);
  const float dist2 = dot3(dp, dp);
  const float d2 = fmaxf(dist2, fmaxf(0.5f * sqrtf(dot3(ext, ext)), 1e-20f));
  if (p.x >= n.lo.x && p.y >= n.lo.y && p.z >= n.lo.z && p.x <= n.hi.x && p.y <= n.hi.y && p.z <= n.hi.z)
    return n.phi / d2;
  const float3 wi = mul(dp, rsqrtf(dist2));
  const float cosW = dot3(n.w, wi), sinW = sqrtf(fmaxf(0.0f, 1.0f - cosW * cosW));
  const float3 dh = sub(pc, n.hi);
  const float s2 = dot3(dh, dh) / dist2;
  const float cosB = s2 >= 1.0f ? -1.0f : sqrtf(fmaxf(0.0f, 1.0f - s2)), sinB = sqrtf(fmaxf(0.0f, 1.0f - cosB * cosB));
  const float sinO = sqrtf(fmaxf(0.0f, 1.0f - n.cosO * n.cosO));
  const float cosX = cos_sub_clamped(sinW, cosW, sinO, n.cosO), sinX = sin_sub_clamped(sinW, cosW, sinO, n.cosO);
  const float cosP = cos_sub_clamped(sinX, cosX, sinB, cosB);
  return cosP <= n.cosE ? 0.0f : n.phi * cosP / d2;
}

// light_tree_sample (main.swift:2809-2833): walk from the root with one number, rescaled at each
// choice, then choose within the leaf by power. Returns the leaf position, or 0xffffffff.
__device__ uint32_t lt_sample(const RenderArgs &A, float3 p, float u, float &pmf) {
  pmf = 1.0f;
  uint32_t index = 0;
  for (uint32_t depth = 0; depth <= 64u; ++depth) {
    const LtNode n = lt_node(A, index);
    if (n.count != 0u) {
      const float sum = lt_leaf_sum(A, n), target = u * sum;
      float cumulative = 0.0f, chosen = 0.0f;
      uint32_t position = 0xffffffffu;
      for (uint32_t i = 0; i < n.count && sum > 0.0f; ++i) {
        const float power = __uint_as_float(lt_leaf_word(A, n.child + i, 1u));
        if (!(power > 0.0f)) continue;
        position = n.child + i;
        chosen = power;
        cumulative += power;
        if (target < cumulative) break;
      }
      if (position == 0xffffffffu) break;
      pmf *= chosen / sum;
      return position;
    }
    const float l = lt_importance(lt_node(A, index + 1u), p), r = lt_importance(lt_node(A, n.child), p);
    if (!(l + r > 0.0f)) break;
    const float pl = l / (l + r);
    if (u < pl) {
      u = fminf(u / pl, 0x1.fffffep-1f);
      index = index + 1u;
      pmf *= pl;
    } else {
      u = fminf((u - pl) / (1.0f - pl), 0x1.fffffep-1f);
      index = n.child;
      pmf *= r / (l + r);
    }
  }
  pmf = 0.0f;
  return 0xffffffffu;
}

// light_tree_pmf (main.swift:2835-2850): the same choices from the leaf up to the root.
__device__ float lt_pmf(const RenderArgs &A, float3 p, uint32_t position) {
  uint32_t index = lt_leaf_word(A, position, 2u);
  LtNode node = lt_node(A, index);
  const float sum = lt_leaf_sum(A, node);
  float pmf = sum > 0.0f ? __uint_as_float(lt_leaf_word(A, position, 1u)) / sum : 0.0f;
  for (uint32_t depth = 0; depth <= 64u && pmf > 0.0f; ++depth) {
    const uint32_t parent = node.parent;
    if (parent == 0x7ffffffu) return pmf;
    const LtNode up = lt_node(A, parent);
    const float l = lt_importance(lt_node(A, parent + 1u), p), r = lt_importance(lt_node(A, up.child), p);
    const float mine = index == parent + 1u ? l : r;
    if (!(l + r > 0.0f) || !(mine > 0.0f)) return 0.0f;
    pmf *= mine / (l + r);
    index = parent;
    node = up;
  }
  return 0.0f;
}

// imported_emitter_position (main.swift:2852-2856): a face's leaf position, by binary search of
// the sorted ids.
__device__ __forceinline__ uint32_t emitter_position(const RenderArgs &A, uint32_t face) {
  uint32_t low = 0, high = A.ecount;
  while (low < high) {
    const uint32_t middle = (low + high) / 2;
    if (__ldg(A.emitters + 1 + middle) < face) low = middle + 1; else high = middle;
  }
  return low < A.ecount && __ldg(A.emitters + 1 + low) == face ? __ldg(A.emitters + 1 + A.ecount + low) : 0xffffffffu;
}

// imported_emitter_area_pdf (main.swift:2859-2869): density per unit area of choosing the face.
__device__ __forceinline__ float emitter_area_pdf(const RenderArgs &A, uint32_t face, float3 p, const Tri &t) {
  if (A.ecount == 0u) return 0.0f;
  if (A.treeNodes > 0u) {
    const uint32_t position = emitter_position(A, face);
    const float area = triangle_area(t);
    return position != 0xffffffffu && area > 0.0f ? lt_pmf(A, p, position) / area : 0.0f;
  }
  return A.etotal > 0.0f ? __ldg(A.emissions + t.slot).w / A.etotal : 0.0f;
}

// sample_direct_light's emitter branch (main.swift:2892-2920), with the emitter probability 1 (no
// environment): the choice draw, then one 3D draw (emitter, point on it).
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

// ---- procedural sky and sun (imported scenes) ----------------------------------------------------
constexpr uint32_t kEnvFace = 0xfffffffeu;  // LightSample.face of an environment sample
constexpr float kPiF = 3.14159265358979323846f;

// in_sun_cone (main.swift:522-525): sin^2 through a cross product, for sub-degree cones.
__device__ __forceinline__ bool in_sun_cone(float3 d, float3 sunDir, float oneMinusCos) {
  const float3 c = cross3(d, sunDir);
  return dot3(d, sunDir) > 0.0f && dot3(c, c) <= oneMinusCos * (2.0f - oneMinusCos);
}
// procedural_sun_one_minus_cos (main.swift:527-529).
__device__ __forceinline__ float sun_one_minus_cos(uint32_t skyMode) {
  return skyMode == 0u ? 8e-4f : (skyMode == 1u ? 7e-4f : 9e-4f);
}
__device__ __forceinline__ float3 mix3(float3 a, float3 b, float t) { return add(a, mul(sub(b, a), t)); }

// eval_procedural_sky (main.swift:541-597): three presets of horizon-to-zenith gradients with a Mie
// lobe and a sun disc of brightness sunIntensity above the horizon, a darkened ground below.
__device__ float3 procedural_sky(const RenderArgs &A, float3 d) {
  const float sunCos = dot3(d, A.sunDir), y = d.y;
  float3 zenith, horizon, ground, lobe, disc;
  float gradient, lobePower, lobeGain, discGain, groundPower, groundScale, gain;
  if (A.skyMode == 0u) {
    zenith = f3(0.08f, 0.18f, 0.46f); horizon = f3(0.96f, 0.52f, 0.22f); ground = f3(0.12f, 0.10f, 0.08f);
    lobe = f3(1.0f, 0.70f, 0.30f); disc = f3(1.0f, 0.78f, 0.45f);
    gradient = 0.40f; lobePower = 6.0f; lobeGain = 3.0f; discGain = 0.45f; groundPower = 5.0f; groundScale = 0.35f;
    gain = 1.5f;
  } else if (A.skyMode == 1u) {
    zenith = f3(0.16f, 0.42f, 0.92f); horizon = f3(0.74f, 0.85f, 0.96f); ground = f3(0.14f, 0.15f, 0.12f);
    lobe = f3(1.0f, 0.98f, 0.92f); disc = f3(1.0f, 0.98f, 0.94f);
    gradient = 0.48f; lobePower = 12.0f; lobeGain = 2.2f; discGain = 0.40f; groundPower = 4.0f; groundScale = 0.40f;
    gain = 1.8f;
  } else {
    zenith = f3(0.04f, 0.06f, 0.14f); horizon = f3(0.46f, 0.26f, 0.42f); ground = f3(0.04f, 0.04f, 0.05f);
    lobe = f3(0.95f, 0.65f, 0.75f); disc = f3(1.0f, 0.85f, 0.78f);
    gradient = 0.55f; lobePower = 10.0f; lobeGain = 1.8f; discGain = 0.35f; groundPower = 3.0f; groundScale = 0.25f;
    gain = 1.6f;
  }
  float3 col;
  if (y >= 0.0f) {
    col = mix3(horizon, zenith, powf(y, gradient));
    col = add(col, mul(lobe, powf(fmaxf(0.0f, sunCos), lobePower) * lobeGain));
    if (in_sun_cone(d, A.sunDir, sun_one_minus_cos(A.skyMode))) col = add(col, mul(disc, A.sunIntensity * discGain));
  } else {
    col = mix3(ground, mul(horizon, groundScale), powf(1.0f + y, groundPower));
  }
  return mul(col, gain);
}
// The image's texel lookup as the reference's sampler does it (main.swift:2127-2134: lat-long
// coordinates u = atan2(z, x) / 2pi + 1/2 + rotation / 2pi, v = acos(y) / pi clamped half a texel in from
// the poles, bilinear filtering, repeat in u).
__device__ float3 env_image(const RenderArgs &A, float3 d) {
  const float W = float(A.envW), H = float(A.envH);
  const float u = atan2f(d.z, d.x) * (0.5f * kInvPi) + 0.5f + A.envRot * (0.5f * kInvPi);
  float v = acosf(fminf(fmaxf(d.y, -1.0f), 1.0f)) * kInvPi;
  v = fminf(fmaxf(v, 0.5f / H), 1.0f - 0.5f / H);
  const float x = u * W - 0.5f, y = v * H - 0.5f;
  const float fx = floorf(x), fy = floorf(y), tx = x - fx, ty = y - fy;
  int x0 = (int)fmodf(fx, W);
  if (x0 < 0) x0 += (int)A.envW;
  x0 = min(x0, (int)A.envW - 1);
  const int x1 = x0 + 1 == (int)A.envW ? 0 : x0 + 1;
  const int y0 = min(max((int)fy, 0), (int)A.envH - 1), y1 = min(y0 + 1, (int)A.envH - 1);
  const float4 a = __ldg(A.envImg + (size_t)y0 * A.envW + x0), b = __ldg(A.envImg + (size_t)y0 * A.envW + x1);
  const float4 c = __ldg(A.envImg + (size_t)y1 * A.envW + x0), e = __ldg(A.envImg + (size_t)y1 * A.envW + x1);
  const float w00 = (1.0f - tx) * (1.0f - ty), w10 = tx * (1.0f - ty), w01 = (1.0f - tx) * ty, w11 = tx * ty;
  return f3(w00 * a.x + w10 * b.x + w01 * c.x + w11 * e.x, w00 * a.y + w10 * b.y + w01 * c.y + w11 * e.y,
            w00 * a.z + w10 * b.z + w01 * c.z + w11 * e.z);
}
// eval_environment (main.swift:2127-2134) without an imported sun: the image or the procedural sky,
// times the intensity.
__device__ __forceinline__ float3 environment(const RenderArgs &A, float3 d) {
  return mul(A.envMap ? env_image(A, d) : procedural_sky(A, d), A.envIntensity);
}
// The environment tables (main.swift:2084-2085): ENV_COMPENSATED samples max(0, L - mean L) and is
// used where the vertex's BSDF continuation is traced; ENV_ORIGINAL samples L.
constexpr uint32_t kEnvCompensated = 0u, kEnvOriginal = 1u;
// environment_cdf_index (main.swift:2089-2097): the first index whose CDF reaches `value`.
__device__ __forceinline__ uint32_t env_cdf_index(const float *cdf, uint32_t count, uint32_t stride, uint32_t base,
                                                  float value) {
  uint32_t low = 0, high = max(1u, count) - 1u;
  for (uint32_t it = 0; it < 16u && low < high; ++it) {
    const uint32_t middle = (low + high) / 2u;
    if (__ldg(cdf + base + (size_t)middle * stride) >= value) high = middle; else low = middle + 1u;
  }
  return low;
}
// environment_cell_pdf (main.swift:2104-2113): the solid-angle density of texel (x, y) in `table`.
__device__ __forceinline__ float env_cell_pdf(const RenderArgs &A, uint32_t x, uint32_t y, float sinTheta, uint32_t table) {
  const float row = __ldg(A.envRows + 2u * y + table);
  const float prevRow = y == 0u ? 0.0f : __ldg(A.envRows + 2u * (y - 1u) + table);
  const float *cols = A.envCols + (size_t)(y + table * A.envH) * A.envW;
  const float col = __ldg(cols + x), prevCol = x == 0u ? 0.0f : __ldg(cols + x - 1u);
  const float cell = fmaxf(0.0f, row - prevRow) * fmaxf(0.0f, col - prevCol);
  return cell * float(A.envW * A.envH) / (2.0f * kPiF * kPiF * fmaxf(1e-5f, sinTheta));
}
// environment_image_pdf (main.swift:2115-2122).
__device__ __forceinline__ float env_image_pdf(const RenderArgs &A, float3 wi, uint32_t table) {
  const float theta = acosf(fminf(fmaxf(wi.y, -1.0f), 1.0f));
  float u = atan2f(wi.z, wi.x) * (0.5f * kInvPi) + 0.5f + A.envRot * (0.5f * kInvPi);
  u = u - floorf(u);
  const float v = fminf(fmaxf(theta * kInvPi, 0.0f), 1.0f - 1e-7f);
  const uint32_t x = min(A.envW - 1u, (uint32_t)(u * float(A.envW))), y = min(A.envH - 1u, (uint32_t)(v * float(A.envH)));
  return env_cell_pdf(A, x, y, sinf(theta), table);
}
// imported_light_probability (main.swift:2716-2719): emitters and the environment share NEE.
__device__ __forceinline__ float imported_probability(const RenderArgs &A) {
  if (A.ecount == 0u) return 0.0f;
  return A.env ? 0.5f : 1.0f;
}
// environment_sun_probability (main.swift:2700-2706) for the procedural sun: 0.6 while the disc is above
// the horizon.
__device__ __forceinline__ float sun_probability(const RenderArgs &A) {
  if (!(A.sunIntensity > 0.0f) || !A.env || A.envMap) return 0.0f;
  const float w = sun_one_minus_cos(A.skyMode);
  return A.sunDir.y >= -sqrtf(w * (2.0f - w)) ? 0.60f : 0.0f;
}
// eval_environment_pdf (main.swift:2880-2883, environment_mixture_pdf :2707-2712): the sun cone and a
// cosine lobe about the receiver's normal n, or the image's density in `table`, times the
// environment's share of NEE. BSDF continuations that escape weigh against the compensated table.
__device__ __forceinline__ float environment_pdf(const RenderArgs &A, float3 wi, float3 n, uint32_t table = kEnvCompensated) {
  const float sp = sun_probability(A), w = sun_one_minus_cos(A.skyMode);
  const float sunPdf = in_sun_cone(wi, A.sunDir, w) ? 1.0f / (kTwoPi * w) : 0.0f;
  const float rest = A.envMap ? env_image_pdf(A, wi, table) : fmaxf(0.0f, dot3(n, wi)) * kInvPi;
  return (1.0f - imported_probability(A)) * (sp * sunPdf + (1.0f - sp) * rest);
}

// sample_direct_light's imported branch (main.swift:2889-2955): an emitter triangle with probability
// imported_probability, else the environment (the sun cone with probability sun_probability, else the
// image's cell from `table` and a uniform point in it, else a cosine lobe about n). `compensated`:
// the vertex's BSDF continuation is traced (ENV_COMPENSATED), else ENV_ORIGINAL.
__device__ LightSample sample_emitters(const RenderArgs &A, float3 p, float3 n, Sampler &seed, bool compensated) {
  LightSample ls;
  ls.pdf = 0.0f;
  ls.face = 0xffffffffu;
  ls.emission = f3(0.0f, 0.0f, 0.0f);
  const float ip = imported_probability(A);
  if (!(ip > 0.0f) && !A.env) return ls;
  if (!(ip > 0.0f && rand_f(seed) < ip)) {
    const float sp = sun_probability(A);
    const float3 q = sp > 0.0f ? rand_f3(seed) : f3(1.0f, 1.0f, 1.0f);
    if (sp > 0.0f && q.x < sp) {
      const float oneMinusCos = q.y * sun_one_minus_cos(A.skyMode);
      const float cosTh = 1.0f - oneMinusCos, sinTh = sqrtf(fmaxf(0.0f, oneMinusCos * (2.0f - oneMinusCos)));
      float3 su, sv;
      make_basis(A.sunDir, su, sv);
      float sn, cs;
      sincosf(kTwoPi * q.z, &sn, &cs);
      ls.wi = normalize3(add(add(mul(su, cs * sinTh), mul(sv, sn * sinTh)), mul(A.sunDir, cosTh)));
    } else if (A.envMap) {
      const uint32_t table = compensated ? kEnvCompensated : kEnvOriginal;
      const float2 c = sp > 0.0f ? make_float2(q.y, q.z) : rand_f2(seed);
      const uint32_t y = env_cdf_index(A.envRows, A.envH, 2u, table, c.x);
      const uint32_t x = env_cdf_index(A.envCols, A.envW, 1u, (y + table * A.envH) * A.envW, c.y);
      // The in-texel offset stays inside the chosen cell, and that cell's probability is used.
      const float W = float(A.envW), H = float(A.envH);
      const float2 r = rand_f2(seed);
      const float u = fminf(float(x) / W + r.x / W, nextafterf(float(x + 1u) / W, 0.0f));
      const float v = fminf(float(y) / H + r.y / H, nextafterf(float(y + 1u) / H, 0.0f));
      const float theta = v * kPiF, phi = (u - 0.5f - A.envRot * (0.5f * kInvPi)) * kTwoPi;
      const float sinTheta = sinf(theta);
      ls.wi = normalize3(f3(sinTheta * cosf(phi), cosf(theta), sinTheta * sinf(phi)));
      ls.pos = add(p, mul(ls.wi, 1e6f));
      ls.dist = 1e6f;
      ls.face = kEnvFace;
      ls.pdf = (1.0f - ip) * (1.0f - sp) * env_cell_pdf(A, x, y, sinTheta, table);
      ls.emission = environment(A, ls.wi);
      return ls;
    } else {
      const float2 r = sp > 0.0f ? make_float2(q.y, q.z) : rand_f2(seed);
      ls.wi = cosine_hemisphere(n, r.x, r.y);
    }
    ls.pos = add(p, mul(ls.wi, 1e6f));
    ls.dist = 1e6f;
    ls.face = kEnvFace;
    ls.pdf = environment_pdf(A, ls.wi, n, compensated ? kEnvCompensated : kEnvOriginal);
    ls.emission = environment(A, ls.wi);
    return ls;
  }
  const float3 q = rand_f3(seed);
  const bool tree = A.treeNodes > 0u;
  float pmf = 0.0f;
  uint32_t face;
  if (tree) {
    const uint32_t position = lt_sample(A, p, q.x, pmf);
    if (position == 0xffffffffu) return ls;
    face = lt_leaf_word(A, position, 0u);
  } else {
    uint32_t low = 0, high = A.ecount - 1u;
    while (low < high) {
      const uint32_t middle = (low + high) / 2;
      if (__uint_as_float(__ldg(A.emitters + 1 + A.ecount + middle)) >= q.x) high = middle; else low = middle + 1;
    }
    face = __ldg(A.emitters + 1 + low);
  }
  const Tri t = scene_triangle(A, face);
  const float root = sqrtf(q.y);
  ls.pos = add(add(mul(t.a, 1.0f - root), mul(t.b, root * (1.0f - q.z))), mul(t.c, root * q.z));
  const float3 delta = sub(ls.pos, p);
  ls.dist = sqrtf(dot3(delta, delta));
  ls.wi = mul(delta, 1.0f / fmaxf(ls.dist, 1e-8f));
  const float geometry = imported_geometry(p, ls.pos, t);
  const float4 e = __ldg(A.emissions + t.slot);
  ls.emission = f3(e.x, e.y, e.z);
  ls.face = face;
  const float area = tree ? triangle_area(t) : 0.0f;
  const float areaPdf = !tree ? emitter_area_pdf(A, face, p, t) : (area > 0.0f ? pmf / area : 0.0f);
  ls.pdf = geometry > 1e-12f ? ip * areaPdf / geometry : 0.0f;
  return ls;
}

// eval_light_pdf for imported emitters (main.swift:3066-3071): the BSDF hit's own triangle.
__device__ __forceinline__ float emitter_pdf(const RenderArgs &A, float3 p, float3 hitPos, uint32_t face) {
  if (A.ecount == 0u) return 0.0f;
  const Tri t = scene_triangle(A, face);
  const float g = imported_geometry(p, hitPos, t);
  return g > 1e-12f ? imported_probability(A) * emitter_area_pdf(A, face, p, t) / g : 0.0f;
}

__device__ __forceinline__ LightSample sample_direct(const RenderArgs &A, float3 p, float3 n, Sampler &seed,
                                                     bool compensated) {
  return A.imported ? sample_emitters(A, p, n, seed, compensated) : sample_light(A, p, seed);
}

// ray_origin (main.swift:1366-1369): offset along the geometric normal by max(error, epsilon).
__device__ __forceinline__ float3 ray_origin(const RenderArgs &A, float3 p, float3 gn, float3 dir, float err) {
  const float offset = fmaxf(err, ray_eps(A, p));
  return add(p, mul(gn, dot3(dir, gn) >= 0.0f ? offset : -offset));
}

// light_visible (main.swift:3254-3264): shadow ray from the offset origin to the sample, shortened
// by the endpoint tolerance (endpoint_tolerance, main.swift:1358-1361).
// Its shadow ray: origin, unit direction and end; false when there is none to trace (no sample, or
// the sample within the endpoint tolerance).
__device__ __forceinline__ bool shadow_ray(const RenderArgs &A, float3 p, float3 gn, float err, const LightSample &ls,
                                           float3 &o, float3 &dir, float &tmax) {
  if (ls.pdf <= 0.0f) return false;
  o = ray_origin(A, p, gn, ls.wi, err);
  float3 delta = sub(ls.pos, o);
  const float d = sqrtf(dot3(delta, delta));
  const float legacy = 2.0f * ray_eps(A, ls.pos);
  const float tol = A.imported ? fmaxf(legacy, 1.907349e-6f * (max_abs(o) + max_abs(ls.pos) + d)) : legacy;
  if (d <= tol) return false;
  dir = mul(delta, 1.0f / d);
  tmax = d - tol;
  return true;
}
__device__ __forceinline__ bool light_visible(const RenderArgs &A, float3 p, float3 gn, float err,
                                              const LightSample &ls, int *stack) {
  float3 o, dir;
  float tmax;
  if (!shadow_ray(A, p, gn, err, ls, o, dir, tmax)) return false;
  return !rt_any(A, o, dir, ray_tmin(A, o), tmax, stack, A.imported != 0u);
}

// power_heuristic (main.swift:2454-2460): beta = 2, scaled by the larger density.
__device__ __forceinline__ float power_heuristic(float pf, float pg) {
  const float scale = fmaxf(pf, pg);
  if (scale <= 0.0f) return 0.0f;
  const float f = pf / scale, g = pg / scale;
  return f * f / (f * f + g * g);
}
// emission_weight (main.swift:3462-3466): the weight of an emitter reached by a BSDF continuation.
__device__ __forceinline__ float emission_weight(bool previousDelta, bool previousNEE, bool previousMIS, float bsdfPdf,
                                                 float lightPdf) {
  if (previousDelta || !previousNEE || lightPdf <= 0.0f) return 1.0f;
  return previousMIS ? power_heuristic(bsdfPdf, lightPdf) : 0.0f;
}

// Reflectance / emission as a 4-lane spectrum (spectral) or rgb in xyz (RGB transport). A slot's
// material carries its index in `pad`; a slot out of range (material()'s black default) has none.
__device__ __forceinline__ float4 reflectance(const RenderArgs &A, const Lanes &L, const vt_material &m) {
  if (A.spectral) {
    const uint32_t slot = __float_as_uint(m.pad);
    return slot < A.nmat ? lanes_reflectance(A, L, slot) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
  return make_float4(m.albedo[0], m.albedo[1], m.albedo[2], 0.0f);
}
__device__ __forceinline__ float4 emission(const RenderArgs &A, const Lanes &L, const float e[3]) {
  if (A.spectral) return lanes_emission(A, L, make_float3(e[0], e[1], e[2]));
  return make_float4(e[0], e[1], e[2], 0.0f);
}
__device__ __forceinline__ float4 emission3(const RenderArgs &A, const Lanes &L, float3 e) {
  if (A.spectral) return lanes_emission(A, L, e);
  return make_float4(e.x, e.y, e.z, 0.0f);
}
__device__ __forceinline__ float3 to_rgb(const RenderArgs &A, const Lanes &L, float4 s) {
  return A.spectral ? lanes_rgb(A, L, s) : f3(s.x, s.y, s.z);
}
__device__ __forceinline__ float4 scale4(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ float4 mul4(float4 a, float4 b) { return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
__device__ __forceinline__ float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float max4(const RenderArgs &A, float4 a) {
  return A.spectral ? fmaxf(fmaxf(a.x, a.y), fmaxf(a.z, a.w)) : fmaxf(fmaxf(a.x, a.y), a.z);
}

// ---- per-slot lobe parameters, OpenPBR vertices (openpbr.cuh) and delta vertices ----------------
// Per slot kSlotF4 float4 (vt_scene_set_openpbr): (roughness, metalness, IOR, diffuse roughness), the
// thin film (weight, thickness in micrometres, IOR) with the coat weight, and (fuzz weight, anisotropy,
// 0, 0).
// Without a table (or for a slot past it) a slot is ideal: roughness 0, IOR 1.5, no film, coat or fuzz.
constexpr uint32_t kSlotF4 = 3;
__device__ __forceinline__ float4 slot_lobe(const RenderArgs &A, const vt_material &m) {
  const uint32_t slot = __float_as_uint(m.pad);
  return A.pbr && slot < A.nmat ? __ldg(A.pbr + kSlotF4 * slot) : make_float4(0.0f, 0.0f, 1.5f, 0.0f);
}
// The slot's second float4: the thin film (weight, thickness in micrometres, IOR) and the coat weight.
__device__ __forceinline__ float4 slot_extra(const RenderArgs &A, const vt_material &m) {
  const uint32_t slot = __float_as_uint(m.pad);
  return A.pbr && slot < A.nmat ? __ldg(A.pbr + kSlotF4 * slot + 1u) : make_float4(0.0f, 0.0f, 1.4f, 0.0f);
}
// The thin film is a spectral-transport input (prepare_openpbr_lanes, main.swift:2527-2568, and
// spectral_thin_film_mirror; the RGB adapter leaves it at zero).
__device__ __forceinline__ float4 slot_film(const RenderArgs &A, const vt_material &m) {
  return A.spectral ? slot_extra(A, m) : make_float4(0.0f, 0.0f, 1.4f, 0.0f);
}
// prepare_bsdf (main.swift:2547-2568): RGB transport evaluates the base colour's three channels; in
// spectral transport `a` takes the reflectance at lanes 0-2 and `b` lane 3, skipped for a flat
// (grey) base where lane 3 equals lane 0. Sampling, lobe choice and pdfs are those of `a`. A GLOSSY
// slot is the BSDF with metalness 1 (prepare_openpbr, main.swift:2489). The film is evaluated at the
// preparation's wavelengths `lambda`.
__device__ __forceinline__ PbrParams pbr_params(const RenderArgs &A, const vt_material &m, float3 base, float3 lambda) {
  const float4 q = slot_lobe(A, m);
  PbrParams P;
  P.base = make_float3(psat(base.x), psat(base.y), psat(base.z));
  P.rough = fmaxf(0.03f, q.x);
  P.metal = m.type == VT_MAT_GLOSSY ? 1.0f : q.y;
  P.ior = fmaxf(1.01f, q.z);
  P.sw = 1.0f;
  P.diffRough = q.w;
  const float4 x = slot_extra(A, m);
  P.tfWeight = A.spectral ? x.x : 0.0f;
  P.tfThickness = A.spectral ? x.y : 0.0f;
  P.tfIor = A.spectral ? x.z : 1.4f;
  P.coat = x.w;  // in both transports (prepare_openpbr and prepare_openpbr_lanes, main.swift:2494, 2537)
  const uint32_t slot = __float_as_uint(m.pad);
  const float4 x3 = A.pbr && slot < A.nmat ? __ldg(A.pbr + kSlotF4 * slot + 2u) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  P.fuzz = x3.x;   // main.swift:2497, 2540
  P.aniso = x3.y;  // main.swift:2496, 2539
  P.lambda = lambda;
  return P;
}
// The adapter's mat.tangent at an anisotropic slot (zero elsewhere): mesh_hit_attributes' tangent
// for a mesh without UVs (main.swift:1594-1599), the triangle's first edge b - a made perpendicular
// to the shading normal n, or n x y (n x x near the poles) when the edge runs along n; unit length.
__device__ __forceinline__ float3 surface_tangent(const RenderArgs &A, const vt_material &m, uint32_t tri, float3 n) {
  const uint32_t slot = __float_as_uint(m.pad);
  if (!A.pbr || slot >= A.nmat || tri >= A.faceCount || !(__ldg(A.pbr + kSlotF4 * slot + 2u).y > 0.0f))
    return f3(0.0f, 0.0f, 0.0f);
  const float4 a = __ldg(A.tris + 3 * (size_t)tri), b = __ldg(A.tris + 3 * (size_t)tri + 1);
  const float3 e1 = f3(b.x - a.x, b.y - a.y, b.z - a.z);
  float3 t = sub(e1, mul(n, dot3(e1, n)));
  if (dot3(t, t) < 1e-12f) t = cross3(n, fabsf(n.y) < 0.9f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f));
  return normalize3(t);
}
// The thin film's weight at slot m (spectral transport only).
__device__ __forceinline__ bool pbr_thin_film_slot(const RenderArgs &A, const vt_material &m) {
  return slot_film(A, m).x > 0.0f;
}
// Lane k's wavelength lambda_k = F^-1((u + k) / 4) (spectral_lambda, main.swift:795-801).
__device__ __forceinline__ float lane_lambda(const RenderArgs &A, const Lanes &L, int k) {
  const float seg = float(A.segments);
  const float x = (L.u + float(k)) * 0.25f * seg;
  const uint32_t i = min((uint32_t)x, A.segments - 1u);
  const float low = __ldg(A.icdf + i), width = __ldg(A.icdf + i + 1) - low;
  return low + (x - float(i)) * width;
}
// kPbr: the kernel variant for scenes with OPENPBR, GLOSSY or DIELECTRIC slots; scenes of Lambert and
// emissive slots run a variant compiled without that code, which keeps its register count (and
// occupancy) down.
// is_delta (main.swift:3285-3287): glass, and GLOSSY mirrors smoother than 0.02.
template <bool kPbr>
__device__ __forceinline__ bool is_delta(const RenderArgs &A, const vt_material &m) {
  return kPbr && (m.type == VT_MAT_DIELECTRIC || (m.type == VT_MAT_GLOSSY && slot_lobe(A, m).x < 0.02f));
}
// The OpenPBR BSDF: OPENPBR slots and rough GLOSSY ones, given the slot table.
template <bool kPbr>
__device__ __forceinline__ bool is_pbr(const RenderArgs &A, const vt_material &m) {
  return kPbr && A.pbr && __float_as_uint(m.pad) < A.nmat &&
         (m.type == VT_MAT_OPENPBR || (m.type == VT_MAT_GLOSSY && __ldg(A.pbr + kSlotF4 * __float_as_uint(m.pad)).x >= 0.02f));
}
// eval_bsdf_with_pdf (main.swift:2695-2706) at an OPENPBR vertex: f (without the cosine) per lane
// and the pdf of `a`.
__device__ float4 pbr_eval_lanes(const RenderArgs &A, const Lanes &L, const vt_material &m, float3 n, float3 gn, uint32_t tri,
                                 float3 wo, float3 wi, float &pdf) {
  pdf = 0.0f;
  const float cosine = fabsf(dot3(n, wi));
  if (cosine < 1e-7f || dot3(n, wo) <= 0.0f) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float4 rho = reflectance(A, L, m);
  // prepare_bsdf (main.swift:2573-2593): the lanes' wavelengths only with a thin film (else the
  // upstream RGB ones), and `b` whenever lane 3 can differ from lane 0.
  const bool film = pbr_thin_film_slot(A, m);
  const float3 lam = film ? make_float3(lane_lambda(A, L, 0), lane_lambda(A, L, 1), lane_lambda(A, L, 2))
                          : make_float3(kPbrRgbNm[0], kPbrRgbNm[1], kPbrRgbNm[2]);
  const float3 tan = surface_tangent(A, m, tri, n);
  const PbrPrepared a = pbr_prepare(pbr_params(A, m, make_float3(rho.x, rho.y, rho.z), lam), A.pbrT, n, wo, true, tan);
  pdf = pbr_pdf(a, A.pbrT, wi);
  if (dot3(wi, gn) <= 0.0f) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float3 fa = pbr_eval(a, A.pbrT, wi);
  float f3w = fa.x;
  if (A.spectral && (rho.w != rho.x || film)) {
    const float l3 = film ? lane_lambda(A, L, 3) : kPbrRgbNm[0];
    const PbrPrepared b = pbr_prepare(pbr_params(A, m, make_float3(rho.w, rho.w, rho.w), make_float3(l3, l3, l3)), A.pbrT, n, wo,
                                      false, tan);
    f3w = pbr_eval(b, A.pbrT, wi).x;
  }
  return make_float4(fa.x / cosine, fa.y / cosine, fa.z / cosine, A.spectral ? f3w / cosine : 0.0f);
}
// sample_bsdf (main.swift:3359-3366) at an OPENPBR vertex: direction, weight f |cos| / pdf per lane.
__device__ bool pbr_sample_lanes(const RenderArgs &A, const Lanes &L, const vt_material &m, float3 n, float3 gn, uint32_t tri,
                                 float3 wo, float3 r, float3 &dir, float4 &weight, float &pdf) {
  const float4 rho = reflectance(A, L, m);
  const bool film = pbr_thin_film_slot(A, m);
  const float3 lam = film ? make_float3(lane_lambda(A, L, 0), lane_lambda(A, L, 1), lane_lambda(A, L, 2))
                          : make_float3(kPbrRgbNm[0], kPbrRgbNm[1], kPbrRgbNm[2]);
  const float3 tan = surface_tangent(A, m, tri, n);
  const PbrPrepared a = pbr_prepare(pbr_params(A, m, make_float3(rho.x, rho.y, rho.z), lam), A.pbrT, n, wo, true, tan);
  float3 w;
  if (!pbr_sample(a, A.pbrT, r, dir, w, pdf) || !(pdf > 0.0f)) return false;
  if (dot3(dir, gn) <= 0.0f) return false;
  float w3 = w.x;
  if (A.spectral && (rho.w != rho.x || film)) {
    const float l3 = film ? lane_lambda(A, L, 3) : kPbrRgbNm[0];
    const PbrPrepared b = pbr_prepare(pbr_params(A, m, make_float3(rho.w, rho.w, rho.w), make_float3(l3, l3, l3)), A.pbrT, n, wo,
                                      false, tan);
    w3 = pbr_eval(b, A.pbrT, dir).x / pdf;
  }
  weight = make_float4(w.x, w.y, w.z, A.spectral ? w3 : 0.0f);
  return isfinite(weight.x) && isfinite(weight.y) && isfinite(weight.z) && isfinite(weight.w) && weight.x >= 0.0f &&
         weight.y >= 0.0f && weight.z >= 0.0f && weight.w >= 0.0f;
}

// sample_bsdf's delta branches (main.swift:3318-3352): weight = f |cos| / pdf per lane, pdf 0.
// DIELECTRIC refracts or reflects by Schlick's Fresnel at the slot's IOR (cosine on the less dense
// side; one draw, none under total internal reflection), tinted by the albedo, eta^2 on refraction;
// an event that the shading normal sends to the wrong side of the surface is retried once about the
// geometric normal. A GLOSSY mirror reflects about the shading normal (the geometric one when that
// reflection would go below the surface) with Schlick's conductor Fresnel of F0 = albedo per lane;
// in spectral transport a thin film over it mixes in the film-over-metal reflectance by its presence
// (spectral_thin_film_mirror, main.swift:3272-3283). `front`: the ray meets the outer side.
__device__ __forceinline__ float3 reflect3(float3 i, float3 n) { return sub(i, mul(n, 2.0f * dot3(n, i))); }
__device__ __forceinline__ float schlick5(float x) {
  const float x2 = x * x;
  return x2 * x2 * x;
}
__device__ __forceinline__ bool sample_delta(const RenderArgs &A, const Lanes &L, const vt_material &m, float3 n, float3 gn, float3 in,
                             bool front, Sampler &seed, float3 &dir, float4 &weight) {
  const float4 tint = reflectance(A, L, m);
  if (m.type == VT_MAT_DIELECTRIC) {
    const float ior = slot_lobe(A, m).z;
    const float eta = front ? 1.0f / ior : ior;
    const float r0 = (1.0f - ior) / (1.0f + ior), f0 = r0 * r0;
    for (int attempt = 0; attempt < 2; ++attempt) {
      const float3 mm = attempt == 0 ? n : gn;
      const float cosI = fminf(fmaxf(-dot3(in, mm), 0.0f), 1.0f);
      const float sin2T = eta * eta * (1.0f - cosI * cosI);
      const float cosine = eta > 1.0f && sin2T < 1.0f ? sqrtf(1.0f - sin2T) : cosI;
      const float fresnel = f0 + (1.0f - f0) * schlick5(1.0f - cosine);
      const bool reflected = sin2T >= 1.0f || rand_f(seed) < fresnel;
      if (reflected) {
        dir = normalize3(reflect3(in, mm));
        weight = tint;
      } else {
        dir = normalize3(add(mul(in, eta), mul(mm, eta * cosI - sqrtf(1.0f - sin2T))));
        weight = scale4(tint, eta * eta);
      }
      if ((dot3(dir, gn) > 0.0f) == reflected) return true;
    }
    return false;
  }
  const float3 mm = dot3(reflect3(in, n), gn) > 0.0f ? n : gn;
  dir = normalize3(reflect3(in, mm));
  const float cosI = fminf(fmaxf(-dot3(in, mm), 0.0f), 1.0f);
  const float s = schlick5(1.0f - cosI);
  weight = make_float4(tint.x + (1.0f - tint.x) * s, tint.y + (1.0f - tint.y) * s, tint.z + (1.0f - tint.z) * s,
                       A.spectral ? tint.w + (1.0f - tint.w) * s : 0.0f);
  if (A.spectral) {
    const float4 film = slot_film(A, m);
    const float nm = film.y * 1000.0f;
    const float presence = pbr_thin_film_presence(film.x, nm);
    if (presence > 0.0f) {
      float3 rd, rm, rm3;
      pbr_thin_film(cosI, 1.0f, film.z, 1.5f, make_float3(tint.x, tint.y, tint.z), false, true, nm,
                    make_float3(lane_lambda(A, L, 0), lane_lambda(A, L, 1), lane_lambda(A, L, 2)), rd, rm);
      const float l3 = lane_lambda(A, L, 3);
      pbr_thin_film(cosI, 1.0f, film.z, 1.5f, make_float3(tint.w, tint.w, tint.w), false, true, nm, make_float3(l3, l3, l3),
                    rd, rm3);
      weight = make_float4(weight.x + (rm.x - weight.x) * presence, weight.y + (rm.y - weight.y) * presence,
                           weight.z + (rm.z - weight.z) * presence, weight.w + (rm3.x - weight.w) * presence);
    }
  }
  return dot3(dir, gn) > 0.0f;
}

// NEE at a vertex: the contribution per lane (quad: 2 draws; emitters: 4).
// n is the shading normal, gn the geometric one (both facing the incoming ray).
// The contribution of a visible light sample ls per lane (throughput T, BSDF, emission, cosine,
// MIS weight against the BSDF pdf when useMIS, over the light pdf).
template <bool kPbr>
__device__ __forceinline__ float4 nee_lanes(const RenderArgs &A, const Lanes &L, float3 n, float3 gn, uint32_t tri, float3 wo, float4 T,
                                            const vt_material &m, bool useMIS, const LightSample &ls) {
  const float cosine = fabsf(dot3(n, ls.wi));
  if (is_pbr<kPbr>(A, m)) {
    float bpdf;
    const float4 f = pbr_eval_lanes(A, L, m, n, gn, tri, wo, ls.wi, bpdf);
    const float weight = useMIS ? power_heuristic(ls.pdf, bpdf) : 1.0f;
    const float le[3] = {ls.emission.x, ls.emission.y, ls.emission.z};
    return scale4(mul4(mul4(T, f), emission(A, L, le)), cosine * weight / ls.pdf);
  }
  const float4 albedo = reflectance(A, L, m);
  // eval_bsdf / eval_bsdf_pdf for DIFFUSE (main.swift:2659-2676): no light below the geometric
  // surface; cosine, f and pdf from the shading normal.
  float f = 0.0f, bpdf = 0.0f;
  const float ni = dot3(n, ls.wi), no = dot3(n, wo);
  if (no > 0.0f) {
    bpdf = fmaxf(0.0f, ni) * kInvPi;
    if (ni > 0.0f && cosine >= 1e-7f && dot3(ls.wi, gn) > 0.0f) f = kInvPi;
  }
  const float weight = useMIS ? power_heuristic(ls.pdf, bpdf) : 1.0f;
  const float le[3] = {ls.emission.x, ls.emission.y, ls.emission.z};
  const float4 Le = emission(A, L, le);
  return scale4(mul4(mul4(T, albedo), Le), f * cosine * weight / ls.pdf);
}
template <bool kPbr>
__device__ __forceinline__ float4 direct_light_lanes(const RenderArgs &A, const Lanes &L, float3 p, float3 n, float3 gn,
                                                     uint32_t tri, float err, float3 wo, float4 T, const vt_material &m, bool useMIS,
                                                     bool compensated, Sampler &seed, int *stack, bool requirePdf) {
  const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const LightSample ls = sample_direct(A, p, n, seed, compensated);
  if (requirePdf && !(ls.pdf > 0.0f)) return zero;
  if (!light_visible(A, p, gn, err, ls, stack)) return zero;
  return nee_lanes<kPbr>(A, L, n, gn, tri, wo, T, m, useMIS, ls);
}
// The same as rgb.
template <bool kPbr>
__device__ __forceinline__ float3 direct_light(const RenderArgs &A, const Lanes &L, float3 p, float3 n, float3 gn,
                                               uint32_t tri, float err, float3 wo, float4 T, const vt_material &m, bool useMIS,
                                               bool compensated, Sampler &seed, int *stack, bool requirePdf) {
  return to_rgb(A, L, direct_light_lanes<kPbr>(A, L, p, n, gn, tri, err, wo, T, m, useMIS, compensated, seed, stack, requirePdf));
}

// ---- ReSTIR DI (sampling mode 0): reservoirs at the primary vertex --------------------------------
// Light ids of stored samples (LightSample.isDirectional): 0 the quad light, face + 2 an emitter.
struct DISample {
  float3 pos, emission;
  float pdf, u;
  uint32_t id;
};
struct DIReservoir {
  DISample s;
  float wsum, M;
};

// light_geometry (main.swift:3165-3183): cos at the light over d^2 seen from p.
__device__ __forceinline__ float light_geometry(const RenderArgs &A, float3 p, const DISample &c) {
  if (A.imported && c.id >= 2u) return imported_geometry(p, c.pos, scene_triangle(A, c.id - 2u));
  const float3 delta = sub(c.pos, p);
  const float d2 = dot3(delta, delta);
  if (d2 < 1e-10f) return 0.0f;
  return fmaxf(0.0f, dot3(A.ln, mul(delta, -rsqrtf(d2)))) / d2;
}

// Lambert f (eval_bsdf for DIFFUSE, main.swift:2665-2686) as direct_light evaluates it.
__device__ __forceinline__ float lambert_f(float3 n, float3 gn, float3 wo, float3 wi) {
  const float ni = dot3(n, wi), no = dot3(n, wo);
  return no > 0.0f && ni > 0.0f && fabsf(ni) >= 1e-7f && dot3(wi, gn) > 0.0f ? kInvPi : 0.0f;
}

// The sample's contribution at the shading point before its weight: bsdf * Le * cos * G, in the
// sample's own wavelengths (u), as linear sRGB.
template <bool kPbr>
__device__ __forceinline__ float3 di_contribution(const RenderArgs &A, float3 p, float3 n, float3 gn, uint32_t tri, float3 view,
                                                  const vt_material &m, const DISample &c) {
  const float3 dir = normalize3(sub(c.pos, p));
  const float cos_th = fmaxf(0.0f, dot3(n, dir));
  if (cos_th <= 0.0f) return f3(0.0f, 0.0f, 0.0f);
  Lanes L;
  if (A.spectral) L = make_lanes(A, c.u);
  const float e[3] = {c.emission.x, c.emission.y, c.emission.z};
  if (is_pbr<kPbr>(A, m)) {
    float pdf;
    const float4 f = pbr_eval_lanes(A, L, m, n, gn, tri, mul(view, -1.0f), dir, pdf);
    return mul(to_rgb(A, L, scale4(mul4(f, emission(A, L, e)), cos_th)), light_geometry(A, p, c));
  }
  const float f = lambert_f(n, gn, mul(view, -1.0f), dir);
  const float4 s = scale4(mul4(reflectance(A, L, m), emission(A, L, e)), f * cos_th);
  return mul(to_rgb(A, L, s), light_geometry(A, p, c));
}

// eval_restir_target_pdf (main.swift:3187-3197): the length of that contribution.
template <bool kPbr>
__device__ __forceinline__ float di_target(const RenderArgs &A, float3 p, float3 n, float3 gn, uint32_t tri, float3 view,
                                           const vt_material &m, const DISample &c) {
  if (c.pdf <= 0.0f) return 0.0f;
  const float3 v = di_contribution<kPbr>(A, p, n, gn, tri, view, m, c);
  return sqrtf(dot3(v, v));
}

__device__ __forceinline__ LightSample di_light_sample(const DISample &c, float3 p) {
  LightSample ls;
  ls.pos = c.pos;
  const float3 d = sub(c.pos, p);
  ls.dist = sqrtf(dot3(d, d));
  ls.wi = normalize3(d);
  ls.emission = c.emission;
  ls.pdf = c.pdf;
  ls.face = c.id >= 2u ? c.id - 2u : 0xffffffffu;
  return ls;
}

__device__ __forceinline__ DISample load_di(const float4 *pos, const float4 *emit, const float4 *w, uint32_t i) {
  const float4 a = pos[i], b = emit[i], c = w[i];
  DISample s;
  s.pos = f3(a.x, a.y, a.z);
  s.id = __float_as_uint(a.w);
  s.emission = f3(b.x, b.y, b.z);
  s.pdf = b.w;
  s.u = c.w;
  return s;
}

// restir_same_surface (main.swift:4816-4820) and restir2020_compatible (main.swift:5030-5033).
__device__ __forceinline__ bool same_surface(float4 pos, float4 nrm, float4 oldPos, float4 oldNrm) {
  const float3 d = f3(oldPos.x - pos.x, oldPos.y - pos.y, oldPos.z - pos.z);
  return oldPos.w > 0.0f && oldNrm.w == nrm.w && oldNrm.x * nrm.x + oldNrm.y * nrm.y + oldNrm.z * nrm.z > 0.95f &&
         sqrtf(dot3(d, d)) < fmaxf(0.01f, pos.w * 0.01f);
}
__device__ __forceinline__ bool compatible(float4 pos, float4 nrm, float4 nPos, float4 nNrm) {
  return nPos.w > 0.0f && nNrm.w == nrm.w && nrm.x * nNrm.x + nrm.y * nNrm.y + nrm.z * nNrm.z > 0.95f &&
         fabsf(pos.w - nPos.w) < 0.05f * pos.w;
}

// restir_backproject (main.swift:4828-4836): the pixel of the previous frame's camera that sees p.
__device__ __forceinline__ bool backproject(const RenderArgs &A, float3 p, int &px, int &py) {
  if (!A.history) return false;
  const float3 d = sub(p, A.pcam);
  const float z = dot3(d, A.pfwd);
  if (!(z > 0.0f)) return false;
  const float nx = dot3(d, A.pright) / (z * A.paspect * A.pfovScale), ny = dot3(d, A.pup) / (z * A.pfovScale);
  const float ux = nx * 0.5f + 0.5f, uy = -ny * 0.5f + 0.5f;
  if (!(ux >= 0.0f && uy >= 0.0f && ux < 1.0f && uy < 1.0f)) return false;
  px = (int)(ux * float(A.W));
  py = (int)(uy * float(A.H));
  return px >= 0 && px < (int)A.W && py >= 0 && py < (int)A.H;
}

// Camera ray (restir_temporal_kernel, main.swift:4874-4893).
__device__ __forceinline__ float3 camera_dir(const RenderArgs &A, uint32_t x, uint32_t y, float2 jit) {
  const float jx = jit.x + 0.5f, jy = jit.y + 0.5f;
  float u = ((float(x) + jx) / float(A.W)) * 2.0f - 1.0f;
  float v = ((float(y) + jy) / float(A.H)) * 2.0f - 1.0f;
  v = -v;
  u *= A.aspect * A.fovScale;
  v *= A.fovScale;
  return normalize3(add(A.fwd, add(mul(A.right, u), mul(A.up, v))));
}

// lens_ray (main.swift:2210-2216): a thin lens moves the origin on the aperture disk (one 2D draw of
// the vertex-0 lens event) and aims through the point in focus.
__device__ __forceinline__ void lens_ray(const RenderArgs &A, float3 &o, float3 &d, Sampler &seed) {
  if (A.aperture <= 0.0f) return;
  sampler_event(seed, 0u, kZLens);
  const float2 r = rand_f2(seed);
  const float radius = sqrtf(r.x) * A.aperture, angle = kTwoPi * r.y;
  const float3 focus = add(o, mul(d, A.focus / fmaxf(1e-5f, dot3(d, A.fwd))));
  float sn, cs;
  sincosf(angle, &sn, &cs);
  o = add(o, add(mul(A.right, radius * cs), mul(A.up, radius * sn)));
  d = normalize3(sub(focus, o));
}

// What the camera sees on an emitter: its radiance, in spectral transport its four-wavelength
// estimate (emitter_rgb, main.swift:7467-7468); imported emitters emit from their front face only
// (trace_scene, main.swift:2031).
__device__ __forceinline__ float3 primary_emission(const RenderArgs &A, const Lanes &L, const Surface &S,
                                                   const vt_material &m) {
  if (A.imported && !S.front) return f3(0.0f, 0.0f, 0.0f);
  return to_rgb(A, L, emission(A, L, m.emission));
}

// The path after its primary vertex S (the bounce loop of shading_kernel, main.swift:7709-7833):
// BSDF continuations, NEE with MIS at later vertices, emitter hits weighed by emission_weight and
// Russian roulette. With diPrimary (sampling mode 0) the primary vertex's direct light came from its
// ReSTIR DI reservoir, so a BSDF hit on an emitter from it gets no weight (previousMIS false,
// main.swift:7717-7718).
// The cache's query record of a vertex (nrc.cuh's input layout): OpenPBR slots give their
// roughness and split the base colour by metalness; Lambert slots are rough and diffuse.
template <bool kPbr>
__device__ __forceinline__ NrcInput nrc_query(const RenderArgs &A, const Lanes &L, const Surface &S, const vt_material &m,
                                              float3 dir) {
  NrcInput q;
  float rough = 1.0f, metal = 0.0f;
  if (is_pbr<kPbr>(A, m)) {
    const float4 pq = slot_lobe(A, m);
    rough = pq.x;
    metal = m.type == VT_MAT_GLOSSY ? 1.0f : nrc_sat(pq.y);
  }
  const float2 w = nrc_sphere(mul(dir, -1.0f)), n = nrc_sphere(S.n);
  q.a = make_float4(S.pos.x, S.pos.y, S.pos.z, rough);
  q.b = make_float4(w.x, w.y, n.x, n.y);
  q.c = make_float4(m.albedo[0] * (1.0f - metal), m.albedo[1] * (1.0f - metal), m.albedo[2] * (1.0f - metal), metal);
  q.d = make_float4(A.spectral ? L.u : 0.0f, 0.0f, 0.0f, 0.0f);
  return q;
}
// The primary spread a0 = |x0 - x1|^2 / (4 pi cos theta_1) of a path's first hit at distance t, times
// the cache's constant c: the spread-angle heuristic (Mueller et al. 2021) stops the path at the
// first vertex n whose spread (sum_i sqrt(|x_i-1 - x_i|^2 / (p(w_i) |cos theta_i|)))^2 exceeds it.
__device__ __forceinline__ float nrc_spread_limit(const RenderArgs &A, float t, float3 gn, float3 dir) {
  const float c = fmaxf(fabsf(dot3(gn, dir)), 1e-6f);
  return A.nrcSpread * t * t / (4.0f * 3.14159265f * c);
}
// The illuminant at a lane's bin: a spectral cache learns each lane's radiance over it.
__device__ __forceinline__ float lane_illuminant(const RenderArgs &A, const Lanes &L, int k) {
  return __ldg(A.spec + L.bin[k]).w;
}
// Stores the query of slot `slot`, with the lanes' bins and the throughput T times, per lane, its
// share and the illuminant there (a spectral cache predicts each lane's radiance over the
// illuminant, so the resolve multiplies both back).
__device__ __forceinline__ void nrc_store(const RenderArgs &A, size_t slot, const NrcInput &q, const Lanes &L, float4 T) {
  A.nrcIn[slot] = q;
  if (A.spectral) {
    A.nrcT[slot] = make_float4(T.x * L.w[0] * lane_illuminant(A, L, 0), T.y * L.w[1] * lane_illuminant(A, L, 1),
                               T.z * L.w[2] * lane_illuminant(A, L, 2), T.w * L.w[3] * lane_illuminant(A, L, 3));
    A.nrcBins[slot] = make_uint2((uint32_t)L.bin[0] | ((uint32_t)L.bin[1] << 16), (uint32_t)L.bin[2] | ((uint32_t)L.bin[3] << 16));
  } else {
    A.nrcT[slot] = make_float4(T.x, T.y, T.z, 0.0f);
    A.nrcBins[slot] = make_uint2(0u, 0u);
  }
}
__device__ __forceinline__ void nrc_store_none(const RenderArgs &A, size_t slot) {
  A.nrcT[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// kNrc (vt_render_nrc): the path ends, after the vertex's emission, at vertex A.nrcVertex, or with
// A.nrcVertex 0 at the first vertex where its spread exceeds spreadLimit (nrc_spread_limit), with
// its cache query stored in `slot`; `queried` tells whether it got there.
template <bool kPbr, bool kNrc = false>
__device__ float3 continue_path(const RenderArgs &A, const Lanes &L, Surface S, vt_material m, float3 dir,
                                Sampler &seed, int *stack, bool diPrimary, float spreadLimit = 0.0f, size_t slot = 0,
                                bool *queried = nullptr) {
  const int limit = max(0, (int)A.maxDepth - 1);
  const bool nee = A.mode != 3u, mis = A.mode <= 1u;
  float4 T = A.spectral ? make_float4(1.0f, 1.0f, 1.0f, 1.0f) : make_float4(1.0f, 1.0f, 1.0f, 0.0f);
  float3 R = f3(0.0f, 0.0f, 0.0f);
  int scattering = 0;
  bool emissionOnly = false;
  float spread = 0.0f;  // sum of the vertices' sqrt(d^2 / (p |cos|)) (kNrc)
  // ReSTIR GI's reservoir estimates the direct light of the secondary diffuse vertex of a path whose
  // diffuse primary took ReSTIR DI, so that vertex skips NEE (restirGISecondary, main.swift:7801-7803).
  const bool giPrimary = diPrimary && !kNrc && m.type == VT_MAT_DIFFUSE;
  // Ideal reflections and refractions spend no scattering event (main.swift:7716-7723); `delta`
  // follows the path's current vertex. The cache-terminated form (kNrc: vt_render_nrc's ReSTIR DI
  // frames) is compiled without glass and mirrors, and the host refuses scenes that have them there.
  bool delta = !kNrc && is_delta<kPbr>(A, m);
  for (int bounce = 1;; ++bounce) {
    if (!delta && scattering >= limit) {
      // BSDF-only paths take one final continuation that may only reach emission.
      if (nee || emissionOnly) break;
      emissionOnly = true;
    }
    if (!delta) ++scattering;
    const bool previousMIS = mis && !(diPrimary && bounce == 1);
    sampler_event(seed, (uint32_t)bounce, kZBsdf);
    float3 nd;
    float bpdf;
    if (delta) {  // glass or mirror: its own draws (sample_delta)
      float4 w;
      if (!sample_delta(A, L, m, S.n, S.gn, dir, S.front, seed, nd, w)) break;
      T = mul4(T, w);
      bpdf = 0.0f;
    } else {
      // One 3D draw (three PCG draws): the prepared OpenPBR sample takes all three, sample_bsdf's
      // Lambert branch the direction from the last two.
      const float3 r = rand_f3(seed);
      if (is_pbr<kPbr>(A, m)) {
        float4 w;
        if (!pbr_sample_lanes(A, L, m, S.n, S.gn, S.tri, mul(dir, -1.0f), r, nd, w, bpdf)) break;
        T = mul4(T, w);
      } else {
        nd = cosine_hemisphere(S.n, r.y, r.z);
        bpdf = fmaxf(0.0f, dot3(S.n, nd)) * kInvPi;
        if (!(bpdf > 0.0f) || !(dot3(nd, S.gn) > 0.0f)) break;
        T = mul4(T, reflectance(A, L, m));
      }
    }
    if (!isfinite(T.x) || !isfinite(T.y) || !isfinite(T.z) || !isfinite(T.w) || max4(A, T) <= 0.0f) break;
    const float3 prev = S.pos;
    const float3 o = ray_origin(A, S.pos, S.gn, nd, S.err);
    dir = nd;
    Hit h;
    if (!rt_closest(A, o, dir, ray_tmin(A, o), __int_as_float(0x7f800000), h, stack)) {
      // An escape sees the environment, weighed like an emitter hit against its NEE density at the
      // previous vertex (main.swift:7751-7756).
      if (A.env) {
        const float lpdf = nee ? environment_pdf(A, dir, S.n) : 0.0f;
        const float w = emission_weight(delta, nee, previousMIS, bpdf, lpdf);
        R = add(R, to_rgb(A, L, scale4(mul4(T, emission3(A, L, environment(A, dir))), w)));
      }
      break;
    }
    S = surface_at(A, h, o, dir);
    m = material(A, S.slot);
    if (kNrc && !delta) spread += h.t * rsqrtf(fmaxf(bpdf * fabsf(dot3(S.gn, dir)), 1e-30f));
    if (m.type == VT_MAT_EMISSIVE) {
      // emission_weight (main.swift:3462-3466): 1 after an ideal bounce, without NEE or without a
      // light pdf, else the power heuristic (MIS) or 0 (light sampling, or a ReSTIR DI vertex).
      const float lpdf = A.imported ? emitter_pdf(A, prev, S.pos, S.face) : light_pdf(A, prev, S.pos);
      const float w = emission_weight(delta, nee, previousMIS, bpdf, lpdf);
      if (!A.imported || S.front) R = add(R, to_rgb(A, L, scale4(mul4(T, emission(A, L, m.emission)), w)));
      break;
    }
    if (emissionOnly) break;
    // Glass and mirrors take no NEE, and the cache is queried at rough vertices only.
    const bool nextDelta = !kNrc && is_delta<kPbr>(A, m);
    delta = nextDelta;
    if (kNrc && !nextDelta && (A.nrcVertex ? (uint32_t)bounce >= A.nrcVertex : spread * spread > spreadLimit)) {
      nrc_store(A, slot, nrc_query<kPbr>(A, L, S, m, dir), L, T);
      *queried = true;
      break;
    }
    if (nee && !nextDelta && !(giPrimary && bounce == 1 && m.type == VT_MAT_DIFFUSE)) {
      sampler_event(seed, (uint32_t)bounce + 1u, kZNee);
      R = add(R, direct_light<kPbr>(A, L, S.pos, S.n, S.gn, S.tri, S.err, mul(dir, -1.0f), T, m, mis && scattering < limit, scattering < limit,
                              seed, stack, false));
    }
    if (bounce > 3) {
      // A higher ceiling at ideal vertices keeps long mirror chains alive (main.swift:7820-7823).
      const float survival = fminf(fmaxf(max4(A, T), 0.05f), nextDelta ? 0.99f : 0.95f);
      sampler_event(seed, (uint32_t)bounce + 1u, kZRoulette);
      if (rand_f(seed) >= survival) break;
      T = scale4(T, 1.0f / survival);
    }
  }
  return R;
}

// One path of sampling modes 1-3: camera ray, primary hit, NEE there, then the continuation.
template <bool kPbr, bool kNrc>
__device__ __forceinline__ float3 path_sample_body(const RenderArgs &A, uint32_t x, uint32_t y, uint32_t si, uint32_t frame,
                                                   float2 jit, int *stack, size_t slot, bool &queried) {
  Sampler seed = pixel_sampler(x, y, A.W, si, A.zSampler != 0u, A.zModel, frame);
  Lanes L;
  if (A.spectral) L = make_lanes(A, wavelength_numbers(seed).x);
  float3 dir0 = camera_dir(A, x, y, jit), o0 = A.cam;
  lens_ray(A, o0, dir0, seed);
  Hit h;
  const bool hit0 = rt_closest(A, o0, dir0, ray_tmin(A, o0), __int_as_float(0x7f800000), h, stack);
  seed.state = pcg_hash(seed.state ^ 0x27d4eb2fu);  // decorrelate_shading_seed
  if (!hit0) return A.env ? environment(A, dir0) : f3(0.0f, 0.0f, 0.0f);  // environment_rgb (main.swift:7453-7455)
  const Surface S = surface_at(A, h, o0, dir0);
  const vt_material m = material(A, S.slot);
  if (m.type == VT_MAT_EMISSIVE) return primary_emission(A, L, S, m);
  float3 R = f3(0.0f, 0.0f, 0.0f);
  if (A.mode != 3u && (kNrc || !is_delta<kPbr>(A, m))) {  // no NEE at glass or a mirror (main.swift:7657)
    const int limit = max(0, (int)A.maxDepth - 1);
    const float4 T = A.spectral ? make_float4(1.0f, 1.0f, 1.0f, 1.0f) : make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    sampler_event(seed, 1u, kZNee);
    R = direct_light<kPbr>(A, L, S.pos, S.n, S.gn, S.tri, S.err, mul(dir0, -1.0f), T, m, A.mode == 1u && limit > 0, limit > 0, seed,
                     stack, true);
  }
  const float spreadLimit = kNrc ? nrc_spread_limit(A, h.t, S.gn, dir0) : 0.0f;
  R = add(R, continue_path<kPbr, kNrc>(A, L, S, m, dir0, seed, stack, false, spreadLimit, slot, &queried));
  if (!isfinite(R.x) || !isfinite(R.y) || !isfinite(R.z)) R = f3(0.0f, 0.0f, 0.0f);
  return R;
}
template <bool kPbr, bool kNrc = false>
__device__ float3 path_sample(const RenderArgs &A, uint32_t x, uint32_t y, uint32_t si, uint32_t frame, float2 jit,
                              int *stack, size_t slot = 0) {
  bool queried = false;
  const float3 c = path_sample_body<kPbr, kNrc>(A, x, y, si, frame, jit, stack, slot, queried);
  if (kNrc && !queried) nrc_store_none(A, slot);
  return c;
}

// ---- ReSTIR GI (sampling mode 0): the first indirect diffuse vertex ------------------------------
// The reference's ReSTIR GI (RESTIRGI2021 in its REFERENCES.md): at a diffuse primary vertex x1, one
// BSDF sample to a diffuse secondary vertex x2 and one NEE sample there give a reservoir holding x2,
// its normal and its outgoing direct radiance (restir_gi_initial, main.swift:4718-4770), merged with
// the previous frame's reservoir of the backprojected pixel (restir_gi_merge, :4775-4795) and, in
// pass 2, with four compatible neighbours (:7582-7649); the reconnection x1 -> x2 is shaded with the
// reservoir's weight when visible (:7650-7656). The path's own continuation then skips NEE at its
// secondary diffuse vertex (main.swift:7801-7803), whose direct light the reservoir estimates.
struct GISample {
  float3 pos, nrm;  // x2 and its shading normal
  float4 rad;       // x2's outgoing direct radiance toward x1 per lane (rgb in RGB transport)
  float pdf, u;     // source pdf of x2 in area measure; the wavelength number the radiance was traced at
};

// gi_geometry (main.swift:3201-3207).
__device__ __forceinline__ float gi_geometry(float3 x1, float3 n1, float3 x2, float3 n2) {
  const float3 delta = sub(x2, x1);
  const float d2 = dot3(delta, delta);
  if (d2 < 1e-10f) return 0.0f;
  const float3 dir = mul(delta, rsqrtf(d2));
  return fmaxf(0.0f, dot3(n1, dir)) * fmaxf(0.0f, -dot3(n2, dir)) / d2;
}
// restir_gi_jacobian / restir_gi_accepts_shift (main.swift:3213-3226): the reconnection's solid-angle
// Jacobian must lie in [0.1, 10].
__device__ __forceinline__ bool gi_accepts_shift(float3 x1r, float3 x1q, float3 x2, float3 n2) {
  const float3 cur = sub(x1r, x2), src = sub(x1q, x2);
  const float cd2 = dot3(cur, cur), sd2 = dot3(src, src);
  if (cd2 < 1e-10f || sd2 < 1e-10f) return false;
  const float cc = fmaxf(0.0f, dot3(n2, mul(cur, rsqrtf(cd2)))), sc = fmaxf(0.0f, dot3(n2, mul(src, rsqrtf(sd2))));
  float j = cc * sd2 / (sc * cd2);
  if (!isfinite(j)) j = 0.0f;
  return j >= 0.1f && j <= 10.0f;
}
// eval_bsdf_with_pdf for DIFFUSE (main.swift:2659-2676) as direct_light evaluates it: f = 1 / pi and
// the cosine pdf from the shading normal, no light below the geometric surface.
__device__ __forceinline__ float lambert_eval(float3 n, float3 gn, float3 wo, float3 wi, float &pdf) {
  const float ni = dot3(n, wi), no = dot3(n, wo);
  pdf = 0.0f;
  if (!(no > 0.0f)) return 0.0f;
  pdf = fmaxf(0.0f, ni) * kInvPi;
  return ni > 0.0f && fabsf(ni) >= 1e-7f && dot3(wi, gn) > 0.0f ? kInvPi : 0.0f;
}
// eval_restir_gi_target (main.swift:3230-3236) at a diffuse x1: |rgb(f(x1 -> x2) L2 G)| in the
// sample's own wavelengths.
__device__ __forceinline__ float gi_target(const RenderArgs &A, float3 x1, float3 n1, float3 gn1, float3 rayDir,
                                           const vt_material &m, const GISample &c) {
  const float geometry = gi_geometry(x1, n1, c.pos, c.nrm);
  if (geometry <= 0.0f || !isfinite(c.rad.x) || !isfinite(c.rad.y) || !isfinite(c.rad.z) || !isfinite(c.rad.w))
    return 0.0f;
  const float3 dir = normalize3(sub(c.pos, x1));
  Lanes L;
  if (A.spectral) L = make_lanes(A, c.u);
  float pdf;
  const float f = lambert_eval(n1, gn1, mul(rayDir, -1.0f), dir, pdf);
  const float3 v = to_rgb(A, L, scale4(mul4(reflectance(A, L, m), c.rad), f * geometry));
  return sqrtf(dot3(v, v));
}
// gi_connection_visible (main.swift:3238-3252): x1 sees x2 (the endpoint tolerance at x2).
__device__ __forceinline__ bool gi_visible(const RenderArgs &A, float3 x1, float3 n1, float3 x2, float err, int *stack) {
  float3 delta = sub(x2, x1);
  const float dist = sqrtf(dot3(delta, delta));
  if (dist <= 2.0f * ray_eps(A, x1)) return false;
  const float3 o = ray_origin(A, x1, n1, mul(delta, 1.0f / dist), err);
  const float3 e = sub(x2, o);
  const float d = sqrtf(dot3(e, e));
  const float legacy = 2.0f * ray_eps(A, x2);
  const float tol = A.imported ? fmaxf(legacy, 1.907349e-6f * (max_abs(o) + max_abs(x2) + d)) : legacy;
  return !rt_any(A, o, mul(e, 1.0f / d), ray_tmin(A, o), d - tol, stack, A.imported != 0u);
}
__device__ __forceinline__ GISample gi_load(const float4 *pos, const float4 *nrm, const float4 *rad, const float4 *w,
                                            uint32_t j) {
  GISample s;
  const float4 p = pos[j], n = nrm[j];
  s.pos = f3(p.x, p.y, p.z);
  s.pdf = p.w;
  s.nrm = f3(n.x, n.y, n.z);
  s.rad = rad[j];
  s.u = w[j].w;
  return s;
}

// restir_gi_initial (main.swift:4718-4770) at the diffuse primary vertex S (material m), seen along
// view: (reservoir sample, weight sum); M is 1.
__device__ GISample gi_initial(const RenderArgs &A, const Surface &S, const vt_material &m, float3 view, float u,
                               Sampler &seed, int *stack, float &wsum) {
  GISample r;
  r.pos = r.nrm = f3(0.0f, 0.0f, 0.0f);
  r.rad = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  r.pdf = 0.0f;
  r.u = u;
  wsum = 0.0f;
  const int limit = max(0, (int)A.maxDepth - 1);
  sampler_event(seed, 1u, kZGiBsdf);
  const float3 rr = rand_f3(seed);  // sample_bsdf's Lambert branch: the direction from the last two
  const float3 gd = cosine_hemisphere(S.n, rr.y, rr.z);
  const float bpdf = fmaxf(0.0f, dot3(S.n, gd)) * kInvPi;
  if (!(bpdf > 0.0f) || !(dot3(gd, S.gn) > 0.0f)) return r;
  const float3 o = ray_origin(A, S.pos, S.gn, gd, S.err);
  Hit h;
  if (!rt_closest(A, o, gd, ray_tmin(A, o), __int_as_float(0x7f800000), h, stack)) return r;
  const Surface S2 = surface_at(A, h, o, gd);
  const vt_material m2 = material(A, S2.slot);
  if (m2.type != VT_MAT_DIFFUSE) return r;
  Lanes L;
  if (A.spectral) L = make_lanes(A, u);
  float4 rad = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  sampler_event(seed, 2u, kZGiNee);
  const LightSample ls = sample_direct(A, S2.pos, S2.n, seed, limit >= 2);
  if (ls.pdf > 0.0f && light_visible(A, S2.pos, S2.gn, S2.err, ls, stack)) {
    const float c2 = fmaxf(0.0f, dot3(S2.n, ls.wi));
    float pdf2;
    const float f2 = lambert_eval(S2.n, S2.gn, mul(gd, -1.0f), ls.wi, pdf2);
    // The power heuristic only when a second continuation can sample x2's BSDF
    // (restir_gi_has_complementary_bsdf, main.swift:3482-3484).
    const float mis = limit >= 2 ? power_heuristic(ls.pdf, pdf2) : 1.0f;
    const float le[3] = {ls.emission.x, ls.emission.y, ls.emission.z};
    rad = scale4(mul4(reflectance(A, L, m2), emission(A, L, le)), f2 * c2 * mis / ls.pdf);
  }
  const float3 delta = sub(S2.pos, S.pos);
  const float d2 = dot3(delta, delta);
  const float cos2 = fmaxf(0.0f, -dot3(S2.n, gd));
  const float srcPdf = d2 > 1e-10f ? bpdf * cos2 / d2 : 0.0f;
  GISample c;
  c.pos = S2.pos;
  c.nrm = S2.n;
  c.rad = rad;
  c.pdf = srcPdf;
  c.u = u;
  const float pHat = gi_target(A, S.pos, S.n, S.gn, view, m, c);
  if (srcPdf > 0.0f && pHat > 0.0f) {
    r = c;
    wsum = pHat / srcPdf;
  }
  return r;
}

// ReSTIR DI pass 1 for frame k (restir_temporal_kernel, main.swift:4842-5005): the primary hit into
// the primary-surface cache, then at a diffuse (Lambert) hit the initial reservoir (RIS over the
// frame's candidates, restir_di_initial, main.swift:4638-4668), merged with the previous frame's
// reservoir of the backprojected pixel when it saw the same surface (restir_di_merge, main.swift:
// 4686-4699, confidence capped at 20), stored with W = wsum / (M p_hat) (restir_di_encode); then,
// with a scattering budget, the ReSTIR GI reservoir the same way (restir_gi_initial / _merge /
// _encode). Other primaries get empty reservoirs and shade with NEE in pass 2 (main.swift:4931-4943).
template <bool kPbr>
__global__ void __launch_bounds__(kRenderBlock, kPbr ? 3 : 4) k_di_primary(RenderArgs A, uint32_t k) {
  int stack[kRenderStack];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.W * A.H) return;
  const uint32_t x = i % A.W, y = i / A.W;
  Sampler seed = pixel_sampler(x, y, A.W, A.first + k, A.zSampler != 0u, A.zModel, A.firstFrame + k);
  const float u = A.spectral ? wavelength_numbers(seed).x : 0.0f;
  float3 dir0 = camera_dir(A, x, y, A.jitter[k]), o0 = A.cam;
  lens_ray(A, o0, dir0, seed);
  const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  Hit h;
  if (!rt_closest(A, o0, dir0, ray_tmin(A, o0), __int_as_float(0x7f800000), h, stack)) {
    A.gPos[i] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    A.gNrm[i] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    A.rPos[i] = zero; A.rEmit[i] = zero; A.rW[i] = zero;
    A.giPos[i] = zero; A.giNrm[i] = zero; A.giRad[i] = zero; A.giW[i] = zero;
    return;
  }
  const Surface S = surface_at(A, h, o0, dir0);
  const vt_material m = material(A, S.slot);
  const float4 gp = make_float4(S.pos.x, S.pos.y, S.pos.z, h.t), gn = make_float4(S.n.x, S.n.y, S.n.z, float(m.type));
  A.gPos[i] = gp;
  A.gNrm[i] = gn;
  A.gGeo[i] = make_float4(S.gn.x, S.gn.y, S.gn.z, 0.0f);
  A.gInfo[i] = make_uint4(S.face, S.slot | (S.front ? 0x80000000u : 0u), __float_as_uint(S.err), S.tri);
  if (m.type != VT_MAT_DIFFUSE) {
    A.rPos[i] = zero; A.rEmit[i] = zero; A.rW[i] = zero;
    A.giPos[i] = zero; A.giNrm[i] = zero; A.giRad[i] = zero; A.giW[i] = zero;
    return;
  }
  DIReservoir r;
  r.s.pos = f3(0.0f, 0.0f, 0.0f); r.s.emission = f3(0.0f, 0.0f, 0.0f);
  r.s.pdf = 0.0f; r.s.u = u; r.s.id = 0u;
  r.wsum = 0.0f;
  r.M = 0.0f;
  for (uint32_t c = 0; c < A.diCandidates; ++c) {
    sampler_candidate(seed, 1u, kZDi, c, A.diBits);
    const LightSample ls = sample_direct(A, S.pos, S.n, seed, (int)A.maxDepth - 1 > 0);
    r.M += 1.0f;  // zero-weight candidates still count
    if (!(ls.pdf > 0.0f)) continue;
    DISample cand;
    cand.pos = ls.pos; cand.emission = ls.emission; cand.pdf = ls.pdf; cand.u = u;
    cand.id = ls.face == 0xffffffffu ? 0u : ls.face + 2u;
    const float pHat = di_target<kPbr>(A, S.pos, S.n, S.gn, S.tri, dir0, m, cand);
    const float proposal = cand.pdf * light_geometry(A, S.pos, cand);
    const float w = proposal > 0.0f ? pHat / proposal : 0.0f;
    r.wsum += w;
    if (rand_decision(seed) * r.wsum < w) r.s = cand;
  }
  int px, py;
  const bool temporal = backproject(A, S.pos, px, py);
  const uint32_t j = temporal ? (uint32_t)py * A.W + (uint32_t)px : 0u;
  if (temporal) {
    const float4 hw = A.hrW[j];
    if (same_surface(gp, gn, A.hPos[j], A.hNrm[j]) && hw.y > 0.0f && hw.z > 0.0f) {
      const DISample hs = load_di(A.hrPos, A.hrEmit, A.hrW, j);
      const float cM = fminf(hw.y, 20.0f);
      const float w = di_target<kPbr>(A, S.pos, S.n, S.gn, S.tri, dir0, m, hs) * hw.z * cM;
      r.M += cM;
      r.wsum += w;
      if (rand_decision(seed) * r.wsum < w) r.s = hs;
    }
  }
  const float pHat = di_target<kPbr>(A, S.pos, S.n, S.gn, S.tri, dir0, m, r.s);
  const float W = r.M > 0.0f && pHat > 0.0f ? r.wsum / (r.M * pHat) : 0.0f;
  A.rPos[i] = make_float4(r.s.pos.x, r.s.pos.y, r.s.pos.z, __uint_as_float(r.s.id));
  A.rEmit[i] = make_float4(r.s.emission.x, r.s.emission.y, r.s.emission.z, r.s.pdf);
  A.rW[i] = make_float4(r.wsum, r.M, W, r.s.u);
  // ReSTIR GI: depth 1 has no indirect bounce for it (restir_gi_enabled, main.swift:3476-3478).
  if ((int)A.maxDepth - 1 < 1) {
    A.giPos[i] = zero; A.giNrm[i] = zero; A.giRad[i] = zero; A.giW[i] = zero;
    return;
  }
  float gwsum, gM = 1.0f;
  GISample g = gi_initial(A, S, m, dir0, u, seed, stack, gwsum);
  if (temporal) {
    const float4 ow = A.hgiW[j], op = A.hgiPos[j], on = A.hgiNrm[j], hp = A.hPos[j];
    if (same_surface(gp, gn, hp, A.hNrm[j]) && ow.y > 0.0f && ow.z > 0.0f && op.w > 0.0f && on.w > 0.0f) {
      const GISample hs = gi_load(A.hgiPos, A.hgiNrm, A.hgiRad, A.hgiW, j);
      if (gi_accepts_shift(S.pos, f3(hp.x, hp.y, hp.z), hs.pos, hs.nrm)) {
        const float cM = fminf(ow.y, 20.0f);
        const float w = gi_target(A, S.pos, S.n, S.gn, dir0, m, hs) * ow.z * cM;
        gM += cM;
        gwsum += w;
        if (pcg_rand(seed.state) * gwsum < w) g = hs;
      }
    }
  }
  const float gHat = gi_target(A, S.pos, S.n, S.gn, dir0, m, g);
  const float gW = gM > 0.0f && gHat > 0.0f ? gwsum / (gM * gHat) : 0.0f;
  A.giPos[i] = make_float4(g.pos.x, g.pos.y, g.pos.z, g.pdf);
  A.giNrm[i] = make_float4(g.nrm.x, g.nrm.y, g.nrm.z, g.pdf > 0.0f ? 1.0f : 0.0f);
  A.giRad[i] = g.rad;
  A.giW[i] = make_float4(gwsum, gM, gW, g.u);
}

// ReSTIR DI pass 2 for frame k (shading_kernel, main.swift:7484-7656): at a diffuse primary, spatial
// reuse of 4 uniform taps in a 32-pixel box that pass RESTIR2020's compatibility test
// (uniform_neighbor, main.swift:5025-5027), the selected sample's contribution W * bsdf * Le * cos *
// G when visible; then the same for the GI reservoirs (the reconnection x1 -> x2 shaded with the
// secondary radiance, W and the area-measure geometry term); other primaries take NEE with MIS
// (main.swift:7767-7780). Then the path's continuation (MIS at later vertices). The sample is added
// to the FP64 accumulation.
template <bool kPbr, bool kNrc = false>
__global__ void __launch_bounds__(kRenderBlock, kPbr ? 3 : 4) k_di_shade(RenderArgs A, uint32_t k) {
  int stack[kRenderStack];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.W * A.H) return;
  const size_t slot = (size_t)k * A.W * A.H + i;
  bool queried = false;
  const uint32_t x = i % A.W, y = i / A.W;
  Sampler seed = pixel_sampler(x, y, A.W, A.first + k, A.zSampler != 0u, A.zModel, A.firstFrame + k);
  Lanes L;
  if (A.spectral) L = make_lanes(A, wavelength_numbers(seed).x);
  float3 dir0 = camera_dir(A, x, y, A.jitter[k]), o0 = A.cam;
  lens_ray(A, o0, dir0, seed);  // the same draws as pass 1
  seed.state = pcg_hash(seed.state ^ 0x27d4eb2fu);  // decorrelate_shading_seed
  const float4 gp = A.gPos[i];
  if (gp.w <= 0.0f) {
    if (kNrc) nrc_store_none(A, slot);
    return;
  }
  const float4 gn = A.gNrm[i];
  const uint4 gi = A.gInfo[i];
  Surface S;
  S.pos = f3(gp.x, gp.y, gp.z);
  S.n = f3(gn.x, gn.y, gn.z);
  const float4 gg = A.gGeo[i];
  S.gn = f3(gg.x, gg.y, gg.z);
  S.face = gi.x;
  S.slot = gi.y & 0x7fffffffu;
  S.front = (gi.y >> 31) != 0u;
  S.err = __uint_as_float(gi.z);
  S.tri = gi.w;
  const vt_material m = material(A, S.slot);
  float3 R;
  if (m.type == VT_MAT_EMISSIVE) {
    R = primary_emission(A, L, S, m);
  } else if (m.type != VT_MAT_DIFFUSE) {
    const int limit = max(0, (int)A.maxDepth - 1);
    const float4 T = A.spectral ? make_float4(1.0f, 1.0f, 1.0f, 1.0f) : make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    R = f3(0.0f, 0.0f, 0.0f);
    if (kNrc || !is_delta<kPbr>(A, m)) {  // no NEE at glass or a mirror (main.swift:7657)
      sampler_event(seed, 1u, kZNee);
      R = direct_light<kPbr>(A, L, S.pos, S.n, S.gn, S.tri, S.err, mul(dir0, -1.0f), T, m, limit > 0, limit > 0, seed, stack, true);
    }
    const float spreadLimit = kNrc ? nrc_spread_limit(A, gp.w, S.gn, dir0) : 0.0f;
    R = add(R, continue_path<kPbr, kNrc>(A, L, S, m, dir0, seed, stack, false, spreadLimit, slot, &queried));
  } else {
    const float4 cw = A.rW[i];
    DISample sel = load_di(A.rPos, A.rEmit, A.rW, i);
    float wsum = di_target<kPbr>(A, S.pos, S.n, S.gn, S.tri, dir0, m, sel) * cw.z * cw.y, M = cw.y;
    for (int t = 0; t < 4; ++t) {
      const float ox = pcg_rand(seed.state), oy = pcg_rand(seed.state);
      const int nx = (int)x + (int)((ox * 2.0f - 1.0f) * 16.0f), ny = (int)y + (int)((oy * 2.0f - 1.0f) * 16.0f);
      if (nx < 0 || nx >= (int)A.W || ny < 0 || ny >= (int)A.H) continue;
      const uint32_t j = (uint32_t)ny * A.W + (uint32_t)nx;
      if (!compatible(gp, gn, A.gPos[j], A.gNrm[j])) continue;
      const float4 nw = A.rW[j];
      if (!(nw.y > 0.0f && nw.z > 0.0f)) continue;
      const DISample ns = load_di(A.rPos, A.rEmit, A.rW, j);
      const float w = di_target<kPbr>(A, S.pos, S.n, S.gn, S.tri, dir0, m, ns) * nw.z * nw.y;
      wsum += w;
      M += nw.y;
      if (rand_decision(seed) * wsum < w) sel = ns;
    }
    const float pHat = di_target<kPbr>(A, S.pos, S.n, S.gn, S.tri, dir0, m, sel);
    const float W = M > 0.0f && pHat > 0.0f ? wsum / (M * pHat) : 0.0f;
    R = f3(0.0f, 0.0f, 0.0f);
    if (W > 0.0f && light_visible(A, S.pos, S.gn, S.err, di_light_sample(sel, S.pos), stack))
      R = mul(di_contribution<kPbr>(A, S.pos, S.n, S.gn, S.tri, dir0, m, sel), W);
    // ReSTIR GI (a cache-terminated path's cache covers this light, so the cache's kernel leaves it out).
    if (!kNrc && (int)A.maxDepth - 1 >= 1) {
      const float4 cgw = A.giW[i];
      GISample gsel = gi_load(A.giPos, A.giNrm, A.giRad, A.giW, i);
      bool gvalid = A.giNrm[i].w > 0.0f;
      float gwsum = gvalid ? gi_target(A, S.pos, S.n, S.gn, dir0, m, gsel) * cgw.z * cgw.y : 0.0f, gM = cgw.y;
      for (int t = 0; t < 4; ++t) {
        const float ox = pcg_rand(seed.state), oy = pcg_rand(seed.state);
        const int nx = (int)x + (int)((ox * 2.0f - 1.0f) * 16.0f), ny = (int)y + (int)((oy * 2.0f - 1.0f) * 16.0f);
        if (nx < 0 || nx >= (int)A.W || ny < 0 || ny >= (int)A.H) continue;
        const uint32_t j = (uint32_t)ny * A.W + (uint32_t)nx;
        const float4 q = A.gPos[j];
        if (!compatible(gp, gn, q, A.gNrm[j])) continue;
        const float4 nw = A.giW[j], np = A.giPos[j], nn = A.giNrm[j];
        if (nw.y <= 0.0f || nw.z <= 0.0f || np.w <= 0.0f || nn.w <= 0.0f) continue;
        if (!gi_accepts_shift(S.pos, f3(q.x, q.y, q.z), f3(np.x, np.y, np.z), f3(nn.x, nn.y, nn.z))) continue;
        const GISample ns = gi_load(A.giPos, A.giNrm, A.giRad, A.giW, j);
        const float w = gi_target(A, S.pos, S.n, S.gn, dir0, m, ns) * nw.z * nw.y;
        gwsum += w;
        gM += nw.y;
        if (rand_decision(seed) * gwsum < w) {
          gsel = ns;
          gvalid = true;
        }
      }
      const float gHat = gvalid ? gi_target(A, S.pos, S.n, S.gn, dir0, m, gsel) : 0.0f;
      const float gW = gM > 0.0f && gHat > 0.0f ? gwsum / (gM * gHat) : 0.0f;
      if (gW > 0.0f && gi_visible(A, S.pos, S.gn, gsel.pos, S.err, stack)) {
        const float3 dir = normalize3(sub(gsel.pos, S.pos));
        Lanes Ls;
        if (A.spectral) Ls = make_lanes(A, gsel.u);
        float pdf;
        const float f = lambert_eval(S.n, S.gn, mul(dir0, -1.0f), dir, pdf);
        const float geometry = gi_geometry(S.pos, S.n, gsel.pos, gsel.nrm);
        R = add(R, to_rgb(A, Ls, scale4(mul4(reflectance(A, Ls, m), gsel.rad), f * geometry * gW)));
      }
    }
    const float spreadLimit = kNrc ? nrc_spread_limit(A, gp.w, S.gn, dir0) : 0.0f;
    R = add(R, continue_path<kPbr, kNrc>(A, L, S, m, dir0, seed, stack, true, spreadLimit, slot, &queried));
  }
  if (kNrc && !queried) nrc_store_none(A, slot);
  if (!isfinite(R.x) || !isfinite(R.y) || !isfinite(R.z)) return;
  double *acc = A.accum + 3 * (size_t)i;
  acc[0] += R.x; acc[1] += R.y; acc[2] += R.z;
}

// Work item i = (sample group g, pixel p), pixel-major within a group so that a warp traces
// neighbouring pixels; a group covers `per` consecutive samples of the call. Each item adds its
// FP64 sum to the pixel with one atomic per channel (groups > 1) or a plain add (groups = 1).
template <bool kPbr, bool kNrc = false>
__global__ void __launch_bounds__(kRenderBlock, kPbr ? 3 : 4) k_render(RenderArgs A, uint32_t groups, uint32_t per) {
  int stack[kRenderStack];
  const uint32_t npix = A.OW * A.OH;  // accumulation pixels: the frame's pixels (s i, s j)
  const uint64_t items = (uint64_t)npix * groups;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < items; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t p = (uint32_t)(i % npix), g = (uint32_t)(i / npix);
    const uint32_t x = (p % A.OW) * A.stride, y = (p / A.OW) * A.stride;
    const uint32_t k0 = g * per, k1 = min(A.spp, k0 + per);
    double sr = 0.0, sg = 0.0, sb = 0.0;
    for (uint32_t k = k0; k < k1; ++k) {
      const float3 c = path_sample<kPbr, kNrc>(A, x, y, A.first + k, A.firstFrame + k, A.jitter[k], stack,
                                               (size_t)k * npix + p);
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

// frameJitter on the device, with the host's float operations (no contraction).
__device__ __forceinline__ float halton_d(uint32_t index, uint32_t base) {
  uint32_t n = index;
  float fraction = 1.0f, result = 0.0f;
  while (n > 0) {
    fraction = __fdiv_rn(fraction, float(base));
    result = __fadd_rn(result, __fmul_rn(fraction, float(n % base)));
    n /= base;
  }
  return result;
}
__device__ __forceinline__ float2 frame_jitter(uint32_t sampleIndex) {
  const uint32_t n = (max(1u, sampleIndex) - 1u) % 1024u + 1u;
  return make_float2(__fsub_rn(halton_d(n, 2u), 0.5f), __fsub_rn(halton_d(n, 3u), 0.5f));
}

// ---- wavefront integrator (vt_render_wavefront; sampling modes 1-3) ------------------------------
// The paths of k_render / path_sample taken apart into stage kernels over queues of path indices,
// with the path's state in HBM between them (WfArgs, structure of arrays). Per bounce b:
//   extend  the persistent closest-hit traversal of traverse.cu (quantised nodes, shared-memory
//           stacks) over the queue of live paths, hits reporting BVH positions;
//   shade   k_wf_shade: first the previous vertex's shadow result, then one vertex of the path in
//           continue_path's order (emission with its MIS weight, NEE, Russian roulette, the BSDF
//           continuation), drawing the same numbers from the same sampler; the NEE sample's shadow
//           ray and contribution go to the shadow queue, a continuing path to the next live queue;
//   shadow  the persistent any-hit traversal over the shadow queue (with imported scenes' endpoint
//           slack).
// Queues are compacted per block: a warp ballot gives each surviving lane its rank, one shared-
// memory atomic per warp and one global atomic per block reserve the slots, and the block's
// entries land contiguously. k_wf_finish adds each path's radiance (primary NEE + continuation,
// summed in k_render's order) to its pixel's FP64 accumulation.
constexpr int kWfBlock = 256;
constexpr uint32_t kWfShadow = 1u, kWfShadowPrimary = 2u, kWfEmissionOnly = 4u, kWfPrevMIS = 8u, kWfQueried = 16u,
                   kWfDead = 32u, kWfPrevDelta = 64u;

struct WfArgs {
  float4 *T;      // throughput per lane
  float4 *Rc;     // radiance of the continuation (rgb)
  float4 *Rp;     // radiance at the primary vertex: its NEE, or its emission / the sky it sees (rgb)
  float4 *prev;   // previous vertex: position, BSDF pdf of the continuation from it
  float4 *prevN;  // previous vertex's shading normal, the path's wavelength number
  uint4 *seedA;   // sampler: state, key, dimension, sub
  uint2 *seedB;   // sampler: subBits, z
  uint4 *meta;    // pixel, bounce, scattering, flags
  float2 *spread; // the cache's termination: the path's spread so far, its limit (nrc_spread_limit)
  float4 *ray;    // the path's next ray (vt_ray: origin, tmin; direction, tmax)
  const int4 *hit;  // its closest hit (t, b1, b2 bits; BVH position or -1)
  float4 *sray;   // the NEE sample's shadow ray (vt_ray)
  float4 *scon;   // its contribution (rgb)
  const uint8_t *occ;  // its occlusion
  const uint32_t *inQ, *inCount;  // live paths of this bounce (null: paths 0 .. paths - 1)
  uint32_t *outQ, *outCount;      // live paths of the next bounce
  uint32_t *shQ, *shCount;        // shadow rays of this bounce
  uint32_t *grpQ;                 // the live queue regrouped by material (k_wf_group)
  uint32_t npix, paths, k0;       // accumulation pixels; paths of the pass; its first sample (of the call)
  uint32_t compact;               // 1: this bounce compacts the live queue; 0: it keeps every entry in
                                  // place (ended paths flagged kWfDead, their next ray empty)
  uint32_t deadFlags;             // 1: some bounce of the pass keeps ended paths queued
};
// The cache's query slot of path i: sample k0 + i / npix of pixel i % npix (k_render's slots).
__device__ __forceinline__ size_t wf_slot(const WfArgs &W, uint32_t i) { return (size_t)W.k0 * W.npix + i; }

__device__ __forceinline__ void wf_store_seed(const WfArgs &W, uint32_t i, const Sampler &s) {
  W.seedA[i] = make_uint4(s.state, s.key, s.dimension, s.sub);
  W.seedB[i] = make_uint2(s.subBits, s.z ? 1u : 0u);
}
__device__ __forceinline__ Sampler wf_load_seed(const WfArgs &W, uint32_t i) {
  const uint4 a = W.seedA[i];
  const uint2 b = W.seedB[i];
  Sampler s;
  s.state = a.x; s.key = a.y; s.dimension = a.z; s.sub = a.w; s.subBits = b.x; s.z = b.y != 0u;
  return s;
}
__device__ __forceinline__ void wf_set_ray(float4 *r, uint32_t i, float3 o, float tmin, float3 d, float tmax) {
  r[2 * (size_t)i] = make_float4(o.x, o.y, o.z, tmin);
  r[2 * (size_t)i + 1] = make_float4(d.x, d.y, d.z, tmax);
}

// Appends v to queue q when `push`; every thread of the block calls it (uniform control flow).
__device__ __forceinline__ void wf_push(bool push, uint32_t v, uint32_t *q, uint32_t *count, uint32_t &sTotal,
                                        uint32_t &sBase) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned m = __ballot_sync(0xffffffffu, push);
  if (threadIdx.x == 0) sTotal = 0;
  __syncthreads();
  uint32_t w = 0;
  if (lane == 0 && m) w = atomicAdd(&sTotal, (uint32_t)__popc(m));
  w = __shfl_sync(0xffffffffu, w, 0);
  __syncthreads();
  if (threadIdx.x == 0) sBase = sTotal ? atomicAdd(count, sTotal) : 0u;
  __syncthreads();
  if (push) q[sBase + w + (uint32_t)__popc(m & ((1u << lane) - 1u))] = v;
  __syncthreads();  // sTotal and sBase are reused by the next push
}

// wf_push from the back: the block's entries go to n - 1 - (reserved rank) of queue q.
__device__ __forceinline__ void wf_push_back(bool push, uint32_t v, uint32_t *q, uint32_t *count, uint32_t n, uint32_t &sTotal,
                                             uint32_t &sBase) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned m = __ballot_sync(0xffffffffu, push);
  if (threadIdx.x == 0) sTotal = 0;
  __syncthreads();
  uint32_t w = 0;
  if (lane == 0 && m) w = atomicAdd(&sTotal, (uint32_t)__popc(m));
  w = __shfl_sync(0xffffffffu, w, 0);
  __syncthreads();
  if (threadIdx.x == 0) sBase = sTotal ? atomicAdd(count, sTotal) : 0u;
  __syncthreads();
  if (push) q[n - 1u - (sBase + w + (uint32_t)__popc(m & ((1u << lane) - 1u)))] = v;
  __syncthreads();
}

// Shading grouped by material: the live queue of a bounce regrouped so that paths whose hit has a
// thin film (the costly iridescence evaluations of spectral transport) come after all others. With
// a tenth of the slots filmed nearly every 32-path warp holds a film vertex; grouped, the shade
// kernel's warps run one kind of vertex. Others fill W.grpQ from the front, film paths from the
// back; counts[0] and counts[1] must be zero on entry.
__global__ void __launch_bounds__(kWfBlock) k_wf_group(RenderArgs A, WfArgs W, uint32_t *counts) {
  __shared__ uint32_t sTotal, sBase;
  const uint32_t n = W.inCount ? min(*W.inCount, W.paths) : W.paths;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t q = base + threadIdx.x;
    uint32_t i = 0;
    bool film = false;
    if (q < n) {
      i = W.inQ ? W.inQ[q] : q;
      const int pos = W.hit[i].w;
      if (pos >= 0 && (uint32_t)pos < A.faceCount && !(W.deadFlags && (W.meta[i].w & kWfDead))) {
        const uint32_t slot = __float_as_uint(__ldg(A.tris + 3 * (size_t)pos + 1).w);
        film = slot < A.nmat && pbr_thin_film_slot(A, material(A, slot));
      }
    }
    wf_push(q < n && !film, i, W.grpQ, counts, sTotal, sBase);
    wf_push_back(q < n && film, i, W.grpQ, counts + 1, n, sTotal, sBase);
  }
}

// The NEE of one vertex up to its visibility: the sample (the draws of direct_light_lanes), its
// shadow ray into sray[i] and its contribution as rgb into scon[i]; false when there is nothing
// to trace.
template <bool kPbr>
__device__ __forceinline__ bool wf_nee(const RenderArgs &A, const WfArgs &W, uint32_t i, const Lanes &L, const Surface &S,
                                       float3 wo, float4 T, const vt_material &m, bool useMIS, bool compensated,
                                       Sampler &seed, bool requirePdf) {
  const LightSample ls = sample_direct(A, S.pos, S.n, seed, compensated);
  if (requirePdf && !(ls.pdf > 0.0f)) return false;
  float3 o, dir;
  float tmax;
  if (!shadow_ray(A, S.pos, S.gn, S.err, ls, o, dir, tmax)) return false;
  const float3 c = to_rgb(A, L, nee_lanes<kPbr>(A, L, S.n, S.gn, S.tri, wo, T, m, useMIS, ls));
  W.scon[i] = make_float4(c.x, c.y, c.z, 0.0f);
  wf_set_ray(W.sray, i, o, ray_tmin(A, o), dir, tmax);
  return true;
}

// One vertex of path i at bounce b (0: the primary hit). Sets `next` when the path continues and
// `shadow` when it queued a shadow ray. kNrc: the path ends with a cache query where continue_path's
// query rule stops it (vt_render_nrc).
template <bool kPbr, bool kNrc>
__device__ __forceinline__ void wf_vertex(const RenderArgs &A, const WfArgs &W, uint32_t i, uint32_t b, bool &next,
                                          bool &shadow) {
  uint4 meta = W.meta[i];
  uint32_t flags = meta.w;
  float4 Rc = W.Rc[i], Rp = W.Rp[i];
  if (flags & kWfShadow) {  // the previous vertex's NEE, traced since
    if (!W.occ[i]) {
      const float4 c = W.scon[i];
      if (flags & kWfShadowPrimary) Rp = make_float4(Rp.x + c.x, Rp.y + c.y, Rp.z + c.z, 0.0f);
      else Rc = make_float4(Rc.x + c.x, Rc.y + c.y, Rc.z + c.z, 0.0f);
    }
    flags &= ~(kWfShadow | kWfShadowPrimary);
  }
  Sampler seed = wf_load_seed(W, i);
  const float4 pn = W.prevN[i];
  Lanes L;
  if (A.spectral) L = make_lanes(A, pn.w);
  const float4 r0 = W.ray[2 * (size_t)i], r1 = W.ray[2 * (size_t)i + 1];
  const float3 o = f3(r0.x, r0.y, r0.z), dir = f3(r1.x, r1.y, r1.z);
  const int4 h4 = W.hit[i];
  Hit h;
  h.t = __int_as_float(h4.x); h.b1 = __int_as_float(h4.y); h.b2 = __int_as_float(h4.z); h.pos = h4.w;
  const int limit = max(0, (int)A.maxDepth - 1);
  const bool nee = A.mode != 3u, mis = A.mode <= 1u;
  float4 T = W.T[i];
  int scattering = (int)meta.z;
  bool emissionOnly = (flags & kWfEmissionOnly) != 0u;
  Surface S;
  vt_material m;
  bool alive = true;
  if (b == 0u) {  // path_sample_body after the camera ray's trace
    if (h.pos < 0) {
      if (A.env) {
        const float3 e = environment(A, dir);
        Rp = make_float4(e.x, e.y, e.z, 0.0f);
      }
      alive = false;
    } else {
      S = surface_at(A, h, o, dir);
      m = material(A, S.slot);
      if (m.type == VT_MAT_EMISSIVE) {
        const float3 e = primary_emission(A, L, S, m);
        Rp = make_float4(e.x, e.y, e.z, 0.0f);
        alive = false;
      } else {
        T = A.spectral ? make_float4(1.0f, 1.0f, 1.0f, 1.0f) : make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        if (kNrc) W.spread[i] = make_float2(0.0f, nrc_spread_limit(A, h.t, S.gn, dir));
        if (A.mode != 3u && !is_delta<kPbr>(A, m)) {
          sampler_event(seed, 1u, kZNee);
          if (wf_nee<kPbr>(A, W, i, L, S, mul(dir, -1.0f), T, m, A.mode == 1u && limit > 0, limit > 0, seed, true)) {
            shadow = true;
            flags |= kWfShadow | kWfShadowPrimary;
          }
        }
        scattering = 0;
        emissionOnly = false;
      }
    }
  } else {  // continue_path after its trace at bounce b
    const float4 pv = W.prev[i];
    const float bpdf = pv.w;
    const bool previousMIS = (flags & kWfPrevMIS) != 0u, previousDelta = (flags & kWfPrevDelta) != 0u;
    if (h.pos < 0) {
      if (A.env) {
        const float lpdf = nee ? environment_pdf(A, dir, f3(pn.x, pn.y, pn.z)) : 0.0f;
        const float w = emission_weight(previousDelta, nee, previousMIS, bpdf, lpdf);
        const float3 c = to_rgb(A, L, scale4(mul4(T, emission3(A, L, environment(A, dir))), w));
        Rc = make_float4(Rc.x + c.x, Rc.y + c.y, Rc.z + c.z, 0.0f);
      }
      alive = false;
    } else {
      const float3 prevPos = f3(pv.x, pv.y, pv.z);
      S = surface_at(A, h, o, dir);
      m = material(A, S.slot);
      float2 sp = make_float2(0.0f, 0.0f);
      if (kNrc) {
        sp = W.spread[i];
        if (!previousDelta) sp.x += h.t * rsqrtf(fmaxf(bpdf * fabsf(dot3(S.gn, dir)), 1e-30f));
        W.spread[i] = sp;
      }
      const bool delta = is_delta<kPbr>(A, m);
      if (m.type == VT_MAT_EMISSIVE) {
        const float lpdf = A.imported ? emitter_pdf(A, prevPos, S.pos, S.face) : light_pdf(A, prevPos, S.pos);
        const float w = emission_weight(previousDelta, nee, previousMIS, bpdf, lpdf);
        if (!A.imported || S.front) {
          const float3 c = to_rgb(A, L, scale4(mul4(T, emission(A, L, m.emission)), w));
          Rc = make_float4(Rc.x + c.x, Rc.y + c.y, Rc.z + c.z, 0.0f);
        }
        alive = false;
      } else if (emissionOnly) {
        alive = false;
      } else if (kNrc && !delta && (A.nrcVertex ? b >= A.nrcVertex : sp.x * sp.x > sp.y)) {
        nrc_store(A, wf_slot(W, i), nrc_query<kPbr>(A, L, S, m, dir), L, T);
        flags |= kWfQueried;
        alive = false;
      } else {
        if (nee && !delta) {
          sampler_event(seed, b + 1u, kZNee);
          if (wf_nee<kPbr>(A, W, i, L, S, mul(dir, -1.0f), T, m, mis && scattering < limit, scattering < limit, seed, false)) {
            shadow = true;
            flags |= kWfShadow;
          }
        }
        if (b > 3u) {
          const float survival = fminf(fmaxf(max4(A, T), 0.05f), delta ? 0.99f : 0.95f);
          sampler_event(seed, b + 1u, kZRoulette);
          if (rand_f(seed) >= survival) alive = false;
          else T = scale4(T, 1.0f / survival);
        }
      }
    }
  }
  if (alive) {  // continue_path's loop head at bounce b + 1: the BSDF continuation
    const uint32_t nb = b + 1u;
    const bool delta = is_delta<kPbr>(A, m);
    if (!delta && scattering >= limit) {
      if (nee || emissionOnly) alive = false;
      emissionOnly = true;
    }
    if (alive) {
      if (!delta) ++scattering;
      sampler_event(seed, nb, kZBsdf);
      float3 nd;
      float bpdf;
      if (delta) {
        float4 w;
        bpdf = 0.0f;
        if (!sample_delta(A, L, m, S.n, S.gn, dir, S.front, seed, nd, w)) alive = false;
        else T = mul4(T, w);
      } else {
        const float3 r = rand_f3(seed);
        if (is_pbr<kPbr>(A, m)) {
          float4 w;
          if (!pbr_sample_lanes(A, L, m, S.n, S.gn, S.tri, mul(dir, -1.0f), r, nd, w, bpdf)) alive = false;
          else T = mul4(T, w);
        } else {
          nd = cosine_hemisphere(S.n, r.y, r.z);
          bpdf = fmaxf(0.0f, dot3(S.n, nd)) * kInvPi;
          if (!(bpdf > 0.0f) || !(dot3(nd, S.gn) > 0.0f)) alive = false;
          else T = mul4(T, reflectance(A, L, m));
        }
      }
      if (alive && (!isfinite(T.x) || !isfinite(T.y) || !isfinite(T.z) || !isfinite(T.w) || max4(A, T) <= 0.0f))
        alive = false;
      if (alive) {
        const float3 no = ray_origin(A, S.pos, S.gn, nd, S.err);
        wf_set_ray(W.ray, i, no, ray_tmin(A, no), nd, __int_as_float(0x7f800000));
        W.prev[i] = make_float4(S.pos.x, S.pos.y, S.pos.z, bpdf);
        W.prevN[i] = make_float4(S.n.x, S.n.y, S.n.z, pn.w);
        W.T[i] = T;
        flags = mis ? (flags | kWfPrevMIS) : (flags & ~kWfPrevMIS);
        flags = delta ? (flags | kWfPrevDelta) : (flags & ~kWfPrevDelta);
        next = true;
      }
    }
  }
  flags = emissionOnly ? (flags | kWfEmissionOnly) : (flags & ~kWfEmissionOnly);
  W.meta[i] = make_uint4(meta.x, next ? b + 1u : b, (uint32_t)scattering, flags);
  W.Rc[i] = Rc;
  W.Rp[i] = Rp;
  if (next) wf_store_seed(W, i, seed);
}

// The pass's paths: sampler, wavelengths and camera ray (path_sample_body's draws before the trace;
// the shading seed's rehash needs no hit, so it happens here too); path i is sample k0 + i / npix
// of accumulation pixel i % npix.
__global__ void __launch_bounds__(kWfBlock) k_wf_generate(RenderArgs A, WfArgs W) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < W.paths; i += gridDim.x * blockDim.x) {
    const uint32_t p = i % W.npix, k = W.k0 + i / W.npix;
    const uint32_t x = (p % A.OW) * A.stride, y = (p / A.OW) * A.stride;
    Sampler seed = pixel_sampler(x, y, A.W, A.first + k, A.zSampler != 0u, A.zModel, A.firstFrame + k);
    const float u = A.spectral ? wavelength_numbers(seed).x : 0.0f;
    float3 dir0 = camera_dir(A, x, y, A.jitter ? A.jitter[k] : frame_jitter(A.first + k)), o0 = A.cam;
    lens_ray(A, o0, dir0, seed);
    seed.state = pcg_hash(seed.state ^ 0x27d4eb2fu);  // decorrelate_shading_seed
    wf_set_ray(W.ray, i, o0, ray_tmin(A, o0), dir0, __int_as_float(0x7f800000));
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    W.T[i] = zero;
    W.Rc[i] = zero;
    W.Rp[i] = zero;
    W.prevN[i] = make_float4(0.0f, 0.0f, 0.0f, u);
    W.meta[i] = make_uint4(p, 0u, 0u, 0u);
    wf_store_seed(W, i, seed);
  }
}

// Two blocks of kWfBlock per SM (at most 128 registers): the OpenPBR variant's register demand
// (with thin films) would otherwise leave one block, and the stage is latency-bound on its loads.
template <bool kPbr, bool kNrc>
__global__ void __launch_bounds__(kWfBlock, 2) k_wf_shade(RenderArgs A, WfArgs W, uint32_t bounce) {
  __shared__ uint32_t sTotal, sBase;
  const uint32_t n = W.inCount ? min(*W.inCount, W.paths) : W.paths;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t q = base + threadIdx.x;
    bool next = false, shadow = false;
    uint32_t i = 0;
    if (q < n) {
      i = W.inQ ? W.inQ[q] : q;
      const bool dead = W.deadFlags && (W.meta[i].w & kWfDead);
      if (!dead) {
        wf_vertex<kPbr, kNrc>(A, W, i, bounce, next, shadow);
        // A path that ends on a bounce without compaction stays queued: flagged, with an empty ray.
        if (!next && !W.compact) {
          W.meta[i].w |= kWfDead;
          reinterpret_cast<float *>(W.ray + 2 * (size_t)i + 1)[3] = -1.0f;
        }
      }
    }
    if (W.compact) {
      wf_push(next, i, W.outQ, W.outCount, sTotal, sBase);
    } else {
      if (q < n) W.outQ[q] = i;
      if (q == 0) *W.outCount = n;
    }
    wf_push(shadow, i, W.shQ, W.shCount, sTotal, sBase);
  }
}

// Each path's radiance (its last shadow result first) into its pixel's FP64 sum: primary NEE plus
// continuation, in k_render's order, non-finite sums dropped. kNrc: a path without a query clears its
// slot's throughput (the resolve skips it).
template <bool kNrc>
__global__ void __launch_bounds__(kWfBlock) k_wf_finish(RenderArgs A, WfArgs W) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < W.paths; i += gridDim.x * blockDim.x) {
    const uint4 meta = W.meta[i];
    if (kNrc && !(meta.w & kWfQueried)) nrc_store_none(A, wf_slot(W, i));
    float4 Rc = W.Rc[i], Rp = W.Rp[i];
    if ((meta.w & kWfShadow) && !W.occ[i]) {
      const float4 c = W.scon[i];
      if (meta.w & kWfShadowPrimary) Rp = make_float4(Rp.x + c.x, Rp.y + c.y, Rp.z + c.z, 0.0f);
      else Rc = make_float4(Rc.x + c.x, Rc.y + c.y, Rc.z + c.z, 0.0f);
    }
    const float3 R = add(f3(Rp.x, Rp.y, Rp.z), f3(Rc.x, Rc.y, Rc.z));
    if (!isfinite(R.x) || !isfinite(R.y) || !isfinite(R.z)) continue;
    double *acc = A.accum + 3 * (size_t)meta.x;
    atomicAdd(acc, (double)R.x);
    atomicAdd(acc + 1, (double)R.y);
    atomicAdd(acc + 2, (double)R.z);
  }
}

// ---- radiance cache: training paths and the resolve (vt_render_nrc) -----------------------------
constexpr int kNrcRecords = 8;  // records per training path: its first 8 vertices

// Training path j of a frame (sampling mode 1 semantics: NEE with MIS at every vertex, Russian
// roulette after bounce 3, full depth): pixel (offset + j stride) mod npix, its own PCG stream
// (sample index si), a random sub-pixel position. Each non-emissive vertex i of the path gives a
// record: its cache query and, as target, the radiance the rest of the path brought to it, rgb of
// the lanes' (R_end - R_i) / T_i, R_i the path's radiance when it reached vertex i (after that
// vertex's emission) and T_i its throughput there. Records go to consecutive slots claimed with
// one atomic per path; those past `cap` are dropped.
template <bool kPbr>
__global__ void __launch_bounds__(kRenderBlock, kPbr ? 3 : 4)
    k_nrc_paths(RenderArgs A, uint32_t npaths, uint32_t offset, uint32_t stride, uint32_t si0, uint32_t cap,
                float4 *__restrict__ scratch, size_t scratchCap, NrcInput *__restrict__ outIn,
                float4 *__restrict__ outTarget, uint32_t outCap, uint32_t *__restrict__ count) {
  int stack[kRenderStack];
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j == 0) count[1] = cap;
  if (j >= npaths) return;
  const uint32_t npix = A.W * A.H;
  const uint64_t lin = (uint64_t)offset + (uint64_t)j * stride;
  const uint32_t p = (uint32_t)(lin % npix), wrap = (uint32_t)(lin / npix);
  const uint32_t x = p % A.W, y = p / A.W;
  Sampler seed = pixel_sampler(x, y, A.W, si0 + wrap, false, 0u, 0u);
  Lanes L;
  if (A.spectral) L = make_lanes(A, wavelength_numbers(seed).x);
  const float2 jit = make_float2(rand_f(seed) - 0.5f, rand_f(seed) - 0.5f);
  float3 dir = camera_dir(A, x, y, jit), o = A.cam;
  lens_ray(A, o, dir, seed);
  Hit h;
  if (!rt_closest(A, o, dir, ray_tmin(A, o), __int_as_float(0x7f800000), h, stack)) return;
  seed.state = pcg_hash(seed.state ^ 0x27d4eb2fu);  // decorrelate_shading_seed
  Surface S = surface_at(A, h, o, dir);
  vt_material m = material(A, S.slot);
  if (m.type == VT_MAT_EMISSIVE) return;
  const int limit = max(0, (int)A.maxDepth - 1);
  float4 T = A.spectral ? make_float4(1.0f, 1.0f, 1.0f, 1.0f) : make_float4(1.0f, 1.0f, 1.0f, 0.0f);
  float4 R = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  // The path's records as they are met: query, T_i, R_i (5 float4 each) in its scratch slots.
  if ((size_t)(j + 1) * kNrcRecords * 5 > scratchCap) {
    render_fault(A, kBadRecord);
    return;
  }
  float4 *rec = scratch + (size_t)j * kNrcRecords * 5;
  int nrec = 0;
  // Records and NEE at rough vertices only; glass and mirrors spend no scattering event.
  if (!is_delta<kPbr>(A, m)) {
    const NrcInput q = nrc_query<kPbr>(A, L, S, m, dir);
    rec[0] = q.a; rec[1] = q.b; rec[2] = q.c; rec[3] = T; rec[4] = R;
    nrec = 1;
    R = add4(R, direct_light_lanes<kPbr>(A, L, S.pos, S.n, S.gn, S.tri, S.err, mul(dir, -1.0f), T, m, limit > 0, limit > 0, seed, stack,
                                         true));
  }
  int scattering = 0;
  for (int bounce = 1;; ++bounce) {
    const bool delta = is_delta<kPbr>(A, m);
    if (!delta && scattering >= limit) break;
    if (!delta) ++scattering;
    float3 nd;
    float bpdf;
    if (delta) {
      float4 w;
      if (!sample_delta(A, L, m, S.n, S.gn, dir, S.front, seed, nd, w)) break;
      T = mul4(T, w);
      bpdf = 0.0f;
    } else {
      const float3 r = rand_f3(seed);
      if (is_pbr<kPbr>(A, m)) {
        float4 w;
        if (!pbr_sample_lanes(A, L, m, S.n, S.gn, S.tri, mul(dir, -1.0f), r, nd, w, bpdf)) break;
        T = mul4(T, w);
      } else {
        nd = cosine_hemisphere(S.n, r.y, r.z);
        bpdf = fmaxf(0.0f, dot3(S.n, nd)) * kInvPi;
        if (!(bpdf > 0.0f) || !(dot3(nd, S.gn) > 0.0f)) break;
        T = mul4(T, reflectance(A, L, m));
      }
    }
    if (!isfinite(T.x) || !isfinite(T.y) || !isfinite(T.z) || !isfinite(T.w) || max4(A, T) <= 0.0f) break;
    const float3 prev = S.pos;
    o = ray_origin(A, S.pos, S.gn, nd, S.err);
    dir = nd;
    if (!rt_closest(A, o, dir, ray_tmin(A, o), __int_as_float(0x7f800000), h, stack)) {
      // An escape sees the environment, weighed against its NEE density at the last vertex.
      if (A.env) {
        const float lpdf = environment_pdf(A, dir, S.n);
        const float w = emission_weight(delta, true, true, bpdf, lpdf);
        R = add4(R, scale4(mul4(T, emission3(A, L, environment(A, dir))), w));
      }
      break;
    }
    S = surface_at(A, h, o, dir);
    m = material(A, S.slot);
    if (m.type == VT_MAT_EMISSIVE) {
      const float lpdf = A.imported ? emitter_pdf(A, prev, S.pos, S.face) : light_pdf(A, prev, S.pos);
      const float w = emission_weight(delta, true, true, bpdf, lpdf);
      if (!A.imported || S.front) R = add4(R, scale4(mul4(T, emission(A, L, m.emission)), w));
      break;
    }
    const bool nextDelta = is_delta<kPbr>(A, m);
    if (!nextDelta) {
      if (nrec < kNrcRecords) {
        const NrcInput q = nrc_query<kPbr>(A, L, S, m, dir);
        float4 *r = rec + 5 * nrec;
        r[0] = q.a; r[1] = q.b; r[2] = q.c; r[3] = T; r[4] = R;
        ++nrec;
      }
      R = add4(R, direct_light_lanes<kPbr>(A, L, S.pos, S.n, S.gn, S.tri, S.err, mul(dir, -1.0f), T, m, scattering < limit,
                                           scattering < limit, seed, stack, false));
    }
    if (bounce > 3) {
      const float survival = fminf(fmaxf(max4(A, T), 0.05f), nextDelta ? 0.99f : 0.95f);
      if (rand_f(seed) >= survival) break;
      T = scale4(T, 1.0f / survival);
    }
  }
  const uint32_t first = atomicAdd(count, (uint32_t)nrec);
  for (int i = 0; i < nrec; ++i) {
    if (first + (uint32_t)i >= cap) break;
    if (first + (uint32_t)i >= outCap) {
      render_fault(A, kBadRecord);
      break;
    }
    const float4 *r = rec + 5 * i;
    const float4 t = r[3], r0 = r[4];
    float4 d = make_float4(t.x > 1e-20f ? (R.x - r0.x) / t.x : 0.0f, t.y > 1e-20f ? (R.y - r0.y) / t.y : 0.0f,
                           t.z > 1e-20f ? (R.z - r0.z) / t.z : 0.0f, t.w > 1e-20f ? (R.w - r0.w) / t.w : 0.0f);
    // Spectral targets: each lane's radiance over the illuminant at its wavelength (a smooth quantity
    // of the size of rgb radiance; the bare lane radiance of a D65-relative emitter is ~1/100 of it,
    // where the relative loss's epsilon would swamp it).
    if (A.spectral)
      d = make_float4(d.x / lane_illuminant(A, L, 0), d.y / lane_illuminant(A, L, 1), d.z / lane_illuminant(A, L, 2),
                      d.w / lane_illuminant(A, L, 3));
    if (!isfinite(d.x) || !isfinite(d.y) || !isfinite(d.z) || !isfinite(d.w)) d = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    NrcInput q;
    q.a = r[0]; q.b = r[1]; q.c = r[2];
    q.d = make_float4(A.spectral ? L.u : 0.0f, 0.0f, 0.0f, 0.0f);
    outIn[first + i] = q;
    outTarget[first + i] = d;
  }
}

// Adds each pixel's cache contributions: per sample slot with a query, the throughput times the
// prediction (clamped at zero) lane by lane, to rgb (spectral transport: the lanes' colour-matching
// functions at the slot's bins; the stored throughput carries each lane's share and illuminant).
__global__ void k_nrc_resolve(RenderArgs A, const float4 *__restrict__ pred, uint32_t spp) {
  const uint32_t npix = A.W * A.H;
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npix) return;
  double sr = 0.0, sg = 0.0, sb = 0.0;
  for (uint32_t k = 0; k < spp; ++k) {
    const size_t slot = (size_t)k * npix + p;
    const float4 t = A.nrcT[slot];
    if (t.x == 0.0f && t.y == 0.0f && t.z == 0.0f && t.w == 0.0f) continue;
    const float4 c = pred[slot];
    const float4 e = make_float4(fmaxf(c.x, 0.0f), fmaxf(c.y, 0.0f), fmaxf(c.z, 0.0f), fmaxf(c.w, 0.0f));
    float3 v;
    if (A.spectral) {
      const uint2 b = A.nrcBins[slot];
      Lanes L;
      L.bin[0] = (int)(b.x & 0xffffu); L.bin[1] = (int)(b.x >> 16);
      L.bin[2] = (int)(b.y & 0xffffu); L.bin[3] = (int)(b.y >> 16);
      L.w[0] = L.w[1] = L.w[2] = L.w[3] = 1.0f;
      L.u = 0.0f;
      v = lanes_rgb(A, L, mul4(t, e));
    } else {
      v = f3(t.x * e.x, t.y * e.y, t.z * e.z);
    }
    if (!isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z)) continue;
    sr += v.x;
    sg += v.y;
    sb += v.z;
  }
  double *acc = A.accum + 3 * (size_t)p;
  acc[0] += sr;
  acc[1] += sg;
  acc[2] += sb;
}

// ---- batched scenes: one persistent launch over many scenes (config C4) ---------------------------
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Items are (scene, pixel), each running all of the pass's samples of its pixel. Warps take 32 x chunk
// consecutive items with one atomic; a scene's last finished item stamps its completion time.
template <bool kPbr>
__global__ void __launch_bounds__(256) k_render_batch(const RenderArgs *__restrict__ scenes,
                                                      const unsigned long long *__restrict__ begin, uint32_t nscenes,
                                                      unsigned long long total, uint32_t chunk,
                                                      const uint32_t *__restrict__ firstSample,
                                                      const uint32_t *__restrict__ firstFrame,
                                                      unsigned long long *counter, unsigned long long *start,
                                                      uint32_t *done, unsigned long long *doneNs) {
  int stack[kRenderStack];
  if (threadIdx.x == 0) atomicMin(start, global_ns());
  const uint32_t lane = threadIdx.x & 31u;
  while (true) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(counter, 32ull * chunk);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    for (uint32_t j = 0; j < chunk; ++j) {
      const unsigned long long item = base + lane + 32ull * j;
      if (item >= total) break;
      uint32_t lo = 0, hi = nscenes - 1u;
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) / 2u;
        if (begin[mid] <= item) lo = mid; else hi = mid - 1u;
      }
      const RenderArgs &A = scenes[lo];
      const uint32_t p = (uint32_t)(item - begin[lo]);
      const uint32_t x = p % A.W, y = p / A.W, f0 = firstSample[lo], fr0 = firstFrame[lo];
      double sr = 0.0, sg = 0.0, sb = 0.0;
      for (uint32_t k = 0; k < A.spp; ++k) {
        const float3 c = path_sample<kPbr, false>(A, x, y, f0 + k, fr0 + k, frame_jitter(f0 + k), stack);
        sr += c.x; sg += c.y; sb += c.z;
      }
      double *acc = A.accum + 3 * (size_t)p;
      acc[0] += sr; acc[1] += sg; acc[2] += sb;
      const uint32_t items = (uint32_t)(begin[lo + 1] - begin[lo]);
      if (atomicAdd(done + lo, 1u) == items - 1u) doneNs[lo] = global_ns();
    }
  }
}

// After a pass: each scene's sample and frame indices move on by its spp; counters reset.
__global__ void k_batch_advance(const RenderArgs *__restrict__ scenes, uint32_t nscenes, uint32_t *firstSample,
                                uint32_t *firstFrame, uint32_t *done) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nscenes) return;
  firstSample[s] += scenes[s].spp;
  firstFrame[s] += scenes[s].spp;
  done[s] = 0u;
}

// ---- imported scenes: emitter collection and the light-selection check --------------------------
__global__ void k_face_positions(const int32_t *__restrict__ order, uint32_t n, int32_t *__restrict__ facePos) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) facePos[order[i]] = (int32_t)i;
}

// Emitter faces: those whose slot has a positive selection weight. Pass 1 counts, pass 2 writes
// (face, a, b, c) records in arbitrary order (the host sorts them by face).
__global__ void k_collect_emitters(const float4 *__restrict__ tris, uint32_t n, const float4 *__restrict__ emissions,
                                   uint32_t nslots, uint32_t *counter, float4 *out, uint32_t capacity) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 b = tris[3 * (size_t)i + 1];
  const uint32_t slot = __float_as_uint(b.w);
  if (slot >= nslots || !(emissions[slot].w > 0.0f)) return;
  const uint32_t k = atomicAdd(counter, 1u);
  if (!out || k >= capacity) return;
  out[3 * (size_t)k] = tris[3 * (size_t)i];
  out[3 * (size_t)k + 1] = b;
  out[3 * (size_t)k + 2] = tris[3 * (size_t)i + 2];
}

// lt_estimate (tests/Fix_light-tree.swift:66-93) on the scene's emitter list.
__global__ void k_light_estimate(RenderArgs A, const float4 *__restrict__ points, uint32_t npoints, uint32_t perPoint,
                                 uint32_t samples, float *out) {
  int stack[kRenderStack];
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= npoints * perPoint) return;
  const float4 pp = points[tid / perPoint];
  const float3 p = f3(pp.x, pp.y, pp.z);
  Sampler seed;
  seed.state = pcg_hash(tid * 7919u + 3u);
  seed.z = false;
  seed.key = seed.dimension = seed.sub = seed.subBits = 0u;
  float sum = 0.0f, squares = 0.0f, hits = 0.0f, zero = 0.0f, error = 0.0f, backFacing = 0.0f;
  for (uint32_t i = 0; i < samples; ++i) {
    const LightSample ls = sample_emitters(A, p, f3(0.0f, 0.0f, 1.0f), seed, true);
    if (ls.face == 0xffffffffu) continue;
    const Tri t = scene_triangle(A, ls.face);
    if (dot3(cross3(sub(t.b, t.a), sub(t.c, t.a)), sub(p, ls.pos)) <= 0.0f) backFacing += 1.0f;
    if (!(ls.pdf > 0.0f)) continue;
    const float c = (0.2126f * ls.emission.x + 0.7152f * ls.emission.y + 0.0722f * ls.emission.z) / ls.pdf;
    sum += c;
    squares += c * c;
    Hit h;
    if (!rt_closest(A, p, ls.wi, ray_tmin(A, p), __int_as_float(0x7f800000), h, stack)) continue;
    const Surface S = surface_at(A, h, p, ls.wi);
    if (material(A, S.slot).type != VT_MAT_EMISSIVE || S.face != ls.face) continue;
    hits += 1.0f;
    const float pdf = emitter_pdf(A, p, S.pos, S.face);
    if (!(pdf > 0.0f)) zero += 1.0f; else error = fmaxf(error, fabsf(pdf - ls.pdf) / ls.pdf);
  }
  float *o = out + 8 * (size_t)tid;
  o[0] = sum; o[1] = squares; o[2] = hits; o[3] = zero;
  o[4] = error; o[5] = backFacing; o[6] = 0.0f; o[7] = 0.0f;
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

namespace {

// Shared by both scene kinds: validation, material slots, spectral tables.
// Some slot is ideal glass, or a GLOSSY mirror smoother than 0.02 (is_delta on the host).
static bool scene_has_delta(const vt_scene *sc) {
  for (size_t i = 0; i < sc->slot_types.size(); ++i)
    if (sc->slot_types[i] == VT_MAT_DIELECTRIC || (sc->slot_types[i] == VT_MAT_GLOSSY && sc->slot_rough[i] < 0.02f)) return true;
  return false;
}

vt_status scene_common(vt_ctx *ctx, const vt_mesh *mesh, const vt_material *materials, uint32_t nmat,
                       const float *lightEmission, const vt_spectral_tables *tables, vt_scene *sc) {
  (void)lightEmission;
  if (tables) {
    if (!tables->cmf_rgb || !tables->illuminant || !tables->icdf || tables->nbins < 2 || tables->segments < 1)
      return vt_fail(ctx, VT_ERR_INVALID, "incomplete spectral tables");
    if (!tables->cos_phase) return vt_fail(ctx, VT_ERR_INVALID, "spectral tables need cos_phase (the render bins' phase)");
    const vt_status st = vt_uplift_ensure(ctx, tables);
    if (st != VT_OK) return st;
  }
  for (uint32_t i = 0; i < nmat; ++i)
    if (materials[i].type < VT_MAT_DIFFUSE || materials[i].type > VT_MAT_OPENPBR)
      return vt_fail(ctx, VT_ERR_INVALID, "material slot " + std::to_string(i) + " has an unknown type");
  sc->mesh = mesh;
  sc->nmat = nmat;
  sc->layered = false;
  sc->slot_types.resize(nmat);
  sc->slot_rough.assign(nmat, 0.0f);
  for (uint32_t i = 0; i < nmat; ++i) {
    sc->slot_types[i] = materials[i].type;
    if (materials[i].type == VT_MAT_GLOSSY || materials[i].type == VT_MAT_DIELECTRIC || materials[i].type == VT_MAT_OPENPBR)
      sc->layered = true;
  }
  if (nmat) {
    // The device copy carries each slot's index in `pad` (the key of its uplifted reflectance).
    std::vector<vt_material> mats(materials, materials + nmat);
    for (uint32_t i = 0; i < nmat; ++i) std::memcpy(&mats[i].pad, &i, sizeof i);
    VT_CUDA(ctx, cudaMalloc(&sc->d_mats, nmat * sizeof(vt_material)));
    VT_CUDA(ctx, cudaMemcpy(sc->d_mats, mats.data(), nmat * sizeof(vt_material), cudaMemcpyHostToDevice));
  }
  if (tables) {
    std::vector<float4> spec(tables->nbins);
    for (uint32_t i = 0; i < tables->nbins; ++i)
      spec[i] = make_float4(tables->cmf_rgb[3 * i], tables->cmf_rgb[3 * i + 1], tables->cmf_rgb[3 * i + 2], tables->illuminant[i]);
    sc->nbins = tables->nbins;
    sc->segments = tables->segments;
    sc->lambda_min = tables->lambda_min;
    VT_CUDA(ctx, cudaMalloc(&sc->d_spec, spec.size() * sizeof(float4)));
    VT_CUDA(ctx, cudaMemcpy(sc->d_spec, spec.data(), spec.size() * sizeof(float4), cudaMemcpyHostToDevice));
    VT_CUDA(ctx, cudaMalloc(&sc->d_icdf, (tables->segments + 1) * sizeof(float)));
    VT_CUDA(ctx, cudaMemcpy(sc->d_icdf, tables->icdf, (tables->segments + 1) * sizeof(float), cudaMemcpyHostToDevice));
    // Uplift: the bins' phase, the emission basis there, and each slot's albedo multipliers.
    VT_CUDA(ctx, cudaMalloc(&sc->d_cosphase, tables->nbins * sizeof(float)));
    VT_CUDA(ctx, cudaMemcpy(sc->d_cosphase, tables->cos_phase, tables->nbins * sizeof(float), cudaMemcpyHostToDevice));
    VT_CUDA(ctx, cudaMalloc(&sc->d_ebasis, 2 * (size_t)tables->nbins * sizeof(float4)));
    vt_status st = vt_uplift_basis(ctx, sc->d_cosphase, tables->nbins, sc->d_ebasis);
    if (st != VT_OK) return st;
    if (nmat) {
      std::vector<float> albedo(3 * (size_t)nmat);
      for (uint32_t i = 0; i < nmat; ++i)
        for (int k = 0; k < 3; ++k) albedo[3 * i + k] = materials[i].albedo[k];
      VT_CUDA(ctx, cudaMalloc(&sc->d_slotL, nmat * sizeof(float4)));
      st = vt_uplift_colours(ctx, albedo.data(), nmat, sc->d_slotL);
      if (st != VT_OK) return st;
    }
  }
  return VT_OK;
}

// MaterialLibrary.environmentImportance (Sources/StudioModel.swift:1300-1392), restated: the pixels'
// luminance (at least 1e-6), dilated by a separable 3 x 3 maximum (wrapping in longitude, clamped in
// latitude) so that a bright texel's bilinear spill into its neighbours is sampled too; the compensated
// table weighs max(0, L - mean L) (the mean over solid angle), the original one L, both times sin(theta);
// a map with nothing above its mean samples L in both. Rows: rows[2 y + table] is the marginal CDF;
// columns: cols[(table H + y) W + x] the conditional CDF of row y. Float arithmetic as the reference's.
void environment_tables(const float *px, uint32_t w, uint32_t h, float *rows, float *cols) {
  const size_t n = (size_t)w * h;
  const float kPiHost = 3.14159265f;
  std::vector<float> lum(n), horizontal(n);
  for (size_t i = 0; i < n; ++i)
    lum[i] = std::max(1e-6f, 0.2126f * px[4 * i] + 0.7152f * px[4 * i + 1] + 0.0722f * px[4 * i + 2]);
  for (uint32_t y = 0; y < h; ++y) {
    const size_t base = (size_t)y * w;
    for (uint32_t x = 0; x < w; ++x)
      horizontal[base + x] = std::max(lum[base + x], std::max(lum[base + (x + w - 1) % w], lum[base + (x + 1) % w]));
  }
  double meanSum = 0.0, angleSum = 0.0;
  for (uint32_t y = 0; y < h; ++y) {
    const double sinTheta = (double)std::max(1e-4f, std::sin((kPiHost * ((float)y + 0.5f)) / (float)h));
    double row = 0.0;
    for (uint32_t x = 0; x < w; ++x) row += (double)lum[(size_t)y * w + x];
    meanSum += row * sinTheta;
    angleSum += sinTheta * (double)w;
  }
  const float mean = (float)(meanSum / angleSum);
  std::fill(rows, rows + 2 * (size_t)h, 0.0f);
  float compensatedTotal = 0.0f;
  for (uint32_t y = 0; y < h; ++y) {
    const float theta = (kPiHost * ((float)y + 0.5f)) / (float)h;
    const float sinTheta = std::max(1e-4f, std::sin(theta));
    const size_t above = (size_t)(y > 0 ? y - 1 : 0) * w, here = (size_t)y * w, below = (size_t)std::min(h - 1, y + 1) * w;
    for (uint32_t x = 0; x < w; ++x) {
      const float dilated = std::max(horizontal[above + x], std::max(horizontal[here + x], horizontal[below + x]));
      const float compensated = std::max(0.0f, dilated - mean) * sinTheta, original = dilated * sinTheta;
      rows[2 * (size_t)y] += compensated;
      rows[2 * (size_t)y + 1] += original;
      cols[here + x] = compensated;
      cols[n + here + x] = original;
      compensatedTotal += compensated;
    }
  }
  if (!(compensatedTotal > 0.0f)) {
    for (uint32_t y = 0; y < h; ++y) rows[2 * (size_t)y] = rows[2 * (size_t)y + 1];
    for (size_t i = 0; i < n; ++i) cols[i] = cols[n + i];
  }
  auto cdf = [](float *weights, size_t count, size_t nrows, size_t stride, size_t step) {
    for (size_t r = 0; r < nrows; ++r) {
      const size_t start = r * stride;
      float total = 0.0f;
      for (size_t k = 0; k < count; ++k) total += weights[start + k * step];
      total = std::max(1e-12f, total);
      float sum = 0.0f;
      for (size_t k = 0; k < count; ++k) {
        sum += weights[start + k * step] / total;
        weights[start + k * step] = k == count - 1 ? 1.0f : sum;
      }
    }
  };
  cdf(rows, h, 2, 1, 2);
  cdf(cols, w, 2 * (size_t)h, w, 1);
}

void scene_free(vt_scene *scene) {
  cudaFree(scene->d_pbr);
  cudaFree(scene->d_slotL);
  cudaFree(scene->d_cosphase);
  cudaFree(scene->d_ebasis);
  cudaFree(scene->d_mats);
  cudaFree(scene->d_spec);
  cudaFree(scene->d_icdf);
  cudaFree(scene->d_accum);
  cudaFree(scene->d_jitter);
  cudaFree(scene->d_emitters);
  cudaFree(scene->d_emissions);
  cudaFree(scene->d_face_pos);
  cudaFree(scene->d_di);
  cudaFree(scene->d_wf);
  cudaFree(scene->d_env_img);
  cudaFree(scene->d_env_rows);
  cudaFree(scene->d_env_cols);
  delete scene;
}

// Selection weight of an emission slot (main.swift:9303-9306): the float luminance, at least 1e-8.
float selection_weight(const float e[3]) {
  const float lum = 0.2126f * e[0] + 0.7152f * e[1] + 0.0722f * e[2];
  return std::max(1e-8f, lum);
}

// Emitter list of an imported scene: collect emitter faces on the device, compute their power on
// the host (area in double from float edges, times the float weight, main.swift:9318-9323), sort
// by face id and pack.
vt_status build_emitters(vt_ctx *ctx, vt_scene *sc, const vt_material *materials, uint32_t nmat, bool lightTree) {
  const vt_mesh *mesh = sc->mesh;
  std::vector<float4> emis(std::max(1u, nmat), make_float4(0, 0, 0, 0));
  for (uint32_t i = 0; i < nmat; ++i) {
    const vt_material &m = materials[i];
    if (m.type != VT_MAT_EMISSIVE) continue;
    const double l2 = double(m.emission[0]) * m.emission[0] + double(m.emission[1]) * m.emission[1] +
                      double(m.emission[2]) * m.emission[2];
    emis[i] = make_float4(m.emission[0], m.emission[1], m.emission[2], l2 > 0 ? selection_weight(m.emission) : 0.0f);
  }
  VT_CUDA(ctx, cudaMalloc(&sc->d_emissions, emis.size() * sizeof(float4)));
  VT_CUDA(ctx, cudaMemcpy(sc->d_emissions, emis.data(), emis.size() * sizeof(float4), cudaMemcpyHostToDevice));
  const uint32_t n = mesh->nfaces;
  VT_CUDA(ctx, cudaMalloc(&sc->d_face_pos, std::max(1u, n) * sizeof(int32_t)));
  std::vector<float4> recs;
  if (n) {
    const unsigned blocks = (n + 255) / 256;
    k_face_positions<<<blocks, 256, 0, ctx->stream>>>(mesh->d_order, n, sc->d_face_pos);
    uint32_t *counter = vt_scratch_word(ctx);
    VT_CUDA(ctx, cudaMemsetAsync(counter, 0, sizeof(uint32_t), ctx->stream));
    k_collect_emitters<<<blocks, 256, 0, ctx->stream>>>(mesh->d_tris, n, sc->d_emissions, nmat, counter, nullptr, 0);
    uint32_t count = 0;
    VT_CUDA(ctx, cudaMemcpyAsync(&count, counter, sizeof count, cudaMemcpyDeviceToHost, ctx->stream));
    VT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (count) {
      float4 *d_recs = nullptr;
      VT_CUDA(ctx, cudaMalloc(&d_recs, 3 * (size_t)count * sizeof(float4)));
      cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(uint32_t), ctx->stream);
      if (e == cudaSuccess) {
        k_collect_emitters<<<blocks, 256, 0, ctx->stream>>>(mesh->d_tris, n, sc->d_emissions, nmat, counter, d_recs, count);
        e = cudaGetLastError();
      }
      recs.resize(3 * (size_t)count);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(recs.data(), d_recs, recs.size() * sizeof(float4), cudaMemcpyDeviceToHost, ctx->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
      cudaFree(d_recs);
      if (e != cudaSuccess) return vt_cuda_fail(ctx, e, "collecting emitters");
    }
  }
  const uint32_t count = (uint32_t)(recs.size() / 3);
  std::vector<uint32_t> idx(count), ids(count);
  for (uint32_t i = 0; i < count; ++i) idx[i] = i;
  auto face_of = [&](uint32_t i) { uint32_t f; std::memcpy(&f, &recs[3 * (size_t)i].w, 4); return f; };
  std::sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) { return face_of(x) < face_of(y); });
  std::vector<vt_emitter> em(count);
  for (uint32_t j = 0; j < count; ++j) {
    const float4 a = recs[3 * (size_t)idx[j]], b = recs[3 * (size_t)idx[j] + 1], c = recs[3 * (size_t)idx[j] + 2];
    ids[j] = face_of(idx[j]);
    vt_emitter &e = em[j];
    std::memset(&e, 0, sizeof e);
    const float av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z}, cv[3] = {c.x, c.y, c.z};
    for (int k = 0; k < 3; ++k) { e.a[k] = av[k]; e.b[k] = bv[k]; e.c[k] = cv[k]; }
    const double e1[3] = {double(bv[0] - av[0]), double(bv[1] - av[1]), double(bv[2] - av[2])};
    const double e2[3] = {double(cv[0] - av[0]), double(cv[1] - av[1]), double(cv[2] - av[2])};
    const double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2], cz = e1[0] * e2[1] - e1[1] * e2[0];
    uint32_t slot;
    std::memcpy(&slot, &b.w, 4);
    e.power = 0.5 * std::sqrt((cx * cx + cy * cy) + cz * cz) * double(emis[slot].w);
    e.cos_emission = 0.0;
  }
  const vt_status st = vt_emitter_list_compute(ids.data(), em.data(), count, lightTree, sc->emitter_words, nullptr);
  if (st != VT_OK) return vt_fail(ctx, st, "light tree exceeds 2^27 - 1 nodes");
  VT_CUDA(ctx, cudaMalloc(&sc->d_emitters, sc->emitter_words.size() * sizeof(uint32_t)));
  VT_CUDA(ctx, cudaMemcpy(sc->d_emitters, sc->emitter_words.data(), sc->emitter_words.size() * sizeof(uint32_t),
                          cudaMemcpyHostToDevice));
  return VT_OK;
}

// The emitter fields of the kernel arguments, from the packed list.
void emitter_args(const vt_scene *sc, RenderArgs &A) {
  A.imported = sc->imported ? 1u : 0u;
  if (!sc->imported) return;
  const std::vector<uint32_t> &w = sc->emitter_words;
  A.emitters = sc->d_emitters;
  A.emissions = sc->d_emissions;
  A.facePos = sc->d_face_pos;
  A.ecount = w[0];
  if (A.ecount == 0) return;
  const uint32_t c = A.ecount;
  float total;
  std::memcpy(&total, &w[2 * c + 1], 4);
  A.etotal = total;
  A.treeNodes = w[2 * c + 2];
  if (A.treeNodes) {
    A.ltNodes = reinterpret_cast<const uint4 *>(sc->d_emitters + w[2 * c + 3]);
    A.ltLeaves = sc->d_emitters + w[2 * c + 4];
    float g[6];
    std::memcpy(g, &w[2 * c + 5], sizeof g);
    A.ltLo = make_float3(g[0], g[1], g[2]);
    A.ltScale = make_float3((g[3] - g[0]) / 65535.0f, (g[4] - g[1]) / 65535.0f, (g[5] - g[2]) / 65535.0f);
  }
}

}  // namespace

extern "C" {

vt_status vt_scene_create(vt_ctx *ctx, const vt_mesh *mesh, const vt_material *materials, uint32_t nmat,
                          const vt_quad_light *light, const vt_spectral_tables *tables, vt_scene **out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!out || !mesh || !light || (nmat && !materials)) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  *out = nullptr;
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  vt_scene *sc = new vt_scene();
  sc->light = *light;
  const vt_status st = scene_common(ctx, mesh, materials, nmat, light->emission, tables, sc);
  if (st != VT_OK) { scene_free(sc); return st; }
  *out = sc;
  return VT_OK;
}

vt_status vt_scene_create_imported(vt_ctx *ctx, const vt_mesh *mesh, const vt_material *materials, uint32_t nmat,
                                   const vt_spectral_tables *tables, uint32_t light_tree, vt_scene **out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!out || !mesh || (nmat && !materials)) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  *out = nullptr;
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  vt_scene *sc = new vt_scene();
  std::memset(&sc->light, 0, sizeof sc->light);
  sc->imported = true;
  vt_status st = scene_common(ctx, mesh, materials, nmat, nullptr, tables, sc);
  if (st == VT_OK) st = build_emitters(ctx, sc, materials, nmat, light_tree != 0);
  if (st != VT_OK) { scene_free(sc); return st; }
  *out = sc;
  return VT_OK;
}

vt_status vt_scene_emitter_words(vt_ctx *ctx, const vt_scene *scene, uint32_t *words, uint32_t capacity,
                                 uint32_t *count) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene || !count) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  if (!scene->imported) return vt_fail(ctx, VT_ERR_INVALID, "the scene has a quad light, not an emitter list");
  *count = (uint32_t)scene->emitter_words.size();
  if (words) {
    if (capacity < scene->emitter_words.size()) return vt_fail(ctx, VT_ERR_INVALID, "capacity below the word count");
    std::copy(scene->emitter_words.begin(), scene->emitter_words.end(), words);
  }
  return VT_OK;
}

vt_status vt_light_estimate(vt_ctx *ctx, const vt_scene *scene, const float *points, uint32_t npoints,
                            uint32_t per_point, uint32_t samples, float *out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene || !points || !out) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  if (!scene->imported) return vt_fail(ctx, VT_ERR_INVALID, "vt_light_estimate needs an imported scene");
  const uint64_t threads = (uint64_t)npoints * per_point;
  if (threads == 0 || threads > (1u << 24)) return vt_fail(ctx, VT_ERR_INVALID, "npoints * per_point must be 1 .. 2^24");
  const vt_mesh *mesh = scene->mesh;
  if (mesh->nfaces == 0) return vt_fail(ctx, VT_ERR_INVALID, "empty mesh");
  if (mesh->depth > 32) return vt_fail(ctx, VT_ERR_LIMIT, "BVH deeper than the render stack");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  RenderArgs A;
  std::memset(&A, 0, sizeof A);
  A.nodes = reinterpret_cast<const float4 *>(mesh->d_nodes);
  A.tris = mesh->d_tris;
  A.nrm = mesh->d_nrm;
  A.rootMax = mesh->root_max;
  A.mats = scene->d_mats;
  A.nmat = scene->nmat;
  A.faceCount = mesh->nfaces;
  A.status = ctx->d_status + 2;
  A.kernelId = 8;
  emitter_args(scene, A);
  float4 *d_points = nullptr;
  float *d_out = nullptr;
  VT_CUDA(ctx, cudaMalloc(&d_points, npoints * sizeof(float4)));
  cudaError_t e = cudaMalloc(&d_out, 8 * threads * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_points, points, npoints * sizeof(float4), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    k_light_estimate<<<(unsigned)((threads + 63) / 64), 64, 0, ctx->stream>>>(A, d_points, npoints, per_point, samples, d_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, 8 * threads * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_points);
  cudaFree(d_out);
  if (e != cudaSuccess) return vt_cuda_fail(ctx, e, "vt_light_estimate");
  return VT_OK;
}

vt_status vt_scene_destroy(vt_ctx *ctx, vt_scene *scene) {
  if (!scene) return VT_OK;
  if (ctx) cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  scene_free(scene);
  return VT_OK;
}

vt_status vt_accum_reset(vt_ctx *ctx, vt_scene *scene) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene) return vt_fail(ctx, VT_ERR_INVALID, "scene is null");
  if (scene->d_accum)
    VT_CUDA(ctx, cudaMemset(scene->d_accum, 0, 3 * (size_t)scene->width * scene->height * sizeof(double)));
  scene->samples = 0;
  scene->di_frames = 0;  // a cut clears the ReSTIR history; camera motion alone keeps it
  return VT_OK;
}

}  // extern "C"

namespace {

// Checks one scene's frame parameters (vt_render's contract).
vt_status check_params(vt_ctx *ctx, const vt_scene *scene, const vt_frame_params *p) {
  if (p->width == 0 || p->height == 0 || (uint64_t)p->width * p->height > (1u << 28))
    return vt_fail(ctx, VT_ERR_INVALID, "bad image size");
  if (p->sampling_mode > 3)
    return vt_fail(ctx, VT_ERR_INVALID, "sampling_mode must be 0 (ReSTIR DI), 1 (MIS), 2 (light) or 3 (BSDF)");
  if (p->di_candidates > 1024) return vt_fail(ctx, VT_ERR_INVALID, "di_candidates must be at most 1024");
  if (p->spectral && !scene->d_spec) return vt_fail(ctx, VT_ERR_INVALID, "spectral transport needs spectral tables");
  if (p->first_sample == 0) return vt_fail(ctx, VT_ERR_INVALID, "first_sample starts at 1");
  if (p->sampler > 1 || p->z_temporal > 3) return vt_fail(ctx, VT_ERR_INVALID, "sampler must be 0 (PCG) or 1 (Z++), z_temporal 0-3");
  if (p->sampling_mode == 0 && scene->environment.intensity > 0.0f)
    return vt_fail(ctx, VT_ERR_INVALID, "ReSTIR DI (sampling mode 0) does not sample the environment; use modes 1-3");
  if (p->pixel_stride > 64) return vt_fail(ctx, VT_ERR_INVALID, "pixel_stride must be at most 64");
  if (p->pixel_stride > 1 && p->sampling_mode == 0)
    return vt_fail(ctx, VT_ERR_INVALID, "a pixel stride needs sampling modes 1-3 (ReSTIR DI reuses neighbouring pixels)");
  const vt_mesh *mesh = scene->mesh;
  if (mesh->nfaces > 0 && mesh->depth > 32) return vt_fail(ctx, VT_ERR_LIMIT, "BVH deeper than the render stack");
  return VT_OK;
}

// Sizes the scene's accumulation to the frame (a new size starts a new accumulation).
// The accumulation's size for a frame: width x height, or ceil(width / s) x ceil(height / s) at a
// pixel stride s.
void accum_dims(const vt_frame_params *p, uint32_t &w, uint32_t &h) {
  const uint32_t st = p->pixel_stride > 1 ? p->pixel_stride : 1u;
  w = (p->width + st - 1) / st;
  h = (p->height + st - 1) / st;
}

vt_status ensure_accum(vt_ctx *ctx, vt_scene *scene, const vt_frame_params *p) {
  uint32_t w, h;
  accum_dims(p, w, h);
  if (w == scene->width && h == scene->height && scene->d_accum) return VT_OK;
  cudaFree(scene->d_accum);
  scene->d_accum = nullptr;
  const size_t bytes = 3 * (size_t)w * h * sizeof(double);
  VT_CUDA(ctx, cudaMalloc(&scene->d_accum, bytes));
  VT_CUDA(ctx, cudaMemset(scene->d_accum, 0, bytes));
  scene->width = w;
  scene->height = h;
  scene->samples = 0;
  return VT_OK;
}

// The kernel arguments of one scene and frame (everything but the jitter and ReSTIR buffers).
void fill_args(const vt_scene *scene, const vt_frame_params *p, uint32_t spp, RenderArgs &A) {
  const vt_mesh *mesh = scene->mesh;
  std::memset(&A, 0, sizeof A);
  A.nodes = reinterpret_cast<const float4 *>(mesh->d_nodes);
  A.tris = mesh->d_tris;
  A.nrm = mesh->d_nrm;
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
  A.slotL = scene->d_slotL;
  A.pbr = scene->d_pbr;
  A.layered = scene->layered ? 1u : 0u;
  if (scene->pbr_tables) A.pbrT = pbr_tables_at(scene->pbr_tables);
  A.cosPhase = scene->d_cosphase;
  A.ebasis = scene->d_ebasis;
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
  A.aperture = p->aperture;
  A.focus = p->focus_distance;
  A.W = p->width;
  A.stride = p->pixel_stride > 1 ? p->pixel_stride : 1u;
  A.OW = (p->width + A.stride - 1) / A.stride;
  A.OH = (p->height + A.stride - 1) / A.stride;
  A.H = p->height;
  A.maxDepth = p->max_depth;
  A.first = p->first_sample;
  A.spp = spp;
  A.mode = p->sampling_mode;
  A.zSampler = p->sampler;
  A.zModel = p->z_temporal;
  A.firstFrame = p->first_frame ? p->first_frame : scene->samples + 1u;
  A.accum = scene->d_accum;
  A.faceCount = mesh->nfaces;
  emitter_args(scene, A);
  const vt_environment &env = scene->environment;
  if (scene->imported && env.intensity > 0.0f) {
    A.env = 1;
    A.envIntensity = env.intensity;
    A.sunIntensity = env.sun_intensity;
    A.sunDir = make_float3(env.sun_dir[0], env.sun_dir[1], env.sun_dir[2]);
    A.skyMode = env.sky_mode;
    if (scene->env_map) {
      A.envMap = 1u;
      A.envImg = scene->d_env_img;
      A.envRows = scene->d_env_rows;
      A.envCols = scene->d_env_cols;
      A.envW = scene->env_w;
      A.envH = scene->env_h;
      A.envRot = scene->env_rot;
      A.sunIntensity = 0.0f;
    }
  }
}

}  // namespace

namespace {

// The cache's part of a frame rendered with queries: predictions for every slot, then the resolve.
vt_status nrc_finish(vt_ctx *ctx, vt_nrc *nrc, const RenderArgs &A, uint32_t spp, cudaStream_t s) {
  const size_t n = (size_t)A.W * A.H * spp;
  if (n > 0xffffffffull) return vt_fail(ctx, VT_ERR_LIMIT, "too many cache queries in one frame");
  {
    const vt_status st = vt_nrc_predict(ctx, nrc, nrc->d_q, (uint32_t)n, nrc->d_qout, s);
    if (st != VT_OK) return st;
  }
  k_nrc_resolve<<<(A.W * A.H + 255) / 256, 256, 0, s>>>(A, nrc->d_qout, spp);
  VT_CUDA(ctx, cudaGetLastError());
  return VT_OK;
}

// vt_render, and with a cache (nrc not null) vt_render_nrc's rendering: the same frames, paths
// ending at the cache's query vertex, then the predictions and the resolve.
vt_status render_impl(vt_ctx *ctx, vt_scene *scene, const vt_frame_params *p, uint32_t spp, void *stream,
                      vt_nrc *nrc) {
  {
    const vt_status st = check_params(ctx, scene, p);
    if (st != VT_OK) return st;
  }
  const vt_mesh *mesh = scene->mesh;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  {
    const vt_status st = ensure_accum(ctx, scene, p);
    if (st != VT_OK) return st;
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
  fill_args(scene, p, spp, A);
  A.jitter = scene->d_jitter;
  A.status = ctx->d_status + 2;
  const uint32_t npix = A.OW * A.OH;  // the frame's pixels, or its strided subset
  if (nrc) {
    const vt_status st = vt_nrc_reserve_queries(ctx, nrc, (size_t)npix * spp);
    if (st != VT_OK) return st;
    A.nrcIn = nrc->d_q;
    A.nrcT = nrc->d_qT;
    A.nrcBins = nrc->d_qbins;
    A.nrcVertex = nrc->cfg.query_vertex;
    A.nrcSpread = nrc->cfg.spread;
  }
  if (p->sampling_mode == 0u) {
    // ReSTIR DI: frames in order, two launches each (the primary pass, then reuse and shading).
    if (!scene->d_di || scene->di_width != p->width || scene->di_height != p->height) {
      cudaFree(scene->d_di);
      scene->d_di = nullptr;
      VT_CUDA(ctx, cudaMalloc(&scene->d_di, 20 * (size_t)npix * sizeof(float4)));
      scene->di_width = p->width;
      scene->di_height = p->height;
      scene->di_frames = 0;
    }
    const uint32_t m = p->di_candidates ? p->di_candidates : 4u;
    uint32_t bits = 0;
    while ((1u << bits) < m) ++bits;
    A.diCandidates = m;
    A.diBits = bits;
    float4 *base = scene->d_di;
    // Per frame parity 9 arrays (surface cache 2, DI reservoir 3, GI reservoir 4), then the primary
    // hit's info and geometric normal.
    A.gInfo = reinterpret_cast<uint4 *>(base + 18 * (size_t)npix);
    A.gGeo = base + 19 * (size_t)npix;
    const float cam[14] = {A.cam.x, A.cam.y, A.cam.z, A.fwd.x, A.fwd.y, A.fwd.z, A.right.x, A.right.y, A.right.z,
                           A.up.x, A.up.y, A.up.z, A.aspect, A.fovScale};
    const unsigned blocks = (npix + kRenderBlock - 1) / kRenderBlock;
    for (uint32_t k = 0; k < spp; ++k) {
      float4 *cur = base + 9 * (size_t)npix * scene->di_parity, *prev = base + 9 * (size_t)npix * (scene->di_parity ^ 1u);
      A.gPos = cur; A.gNrm = cur + npix; A.rPos = cur + 2 * (size_t)npix; A.rEmit = cur + 3 * (size_t)npix;
      A.rW = cur + 4 * (size_t)npix;
      A.giPos = cur + 5 * (size_t)npix; A.giNrm = cur + 6 * (size_t)npix; A.giRad = cur + 7 * (size_t)npix;
      A.giW = cur + 8 * (size_t)npix;
      A.hPos = prev; A.hNrm = prev + npix; A.hrPos = prev + 2 * (size_t)npix; A.hrEmit = prev + 3 * (size_t)npix;
      A.hrW = prev + 4 * (size_t)npix;
      A.hgiPos = prev + 5 * (size_t)npix; A.hgiNrm = prev + 6 * (size_t)npix; A.hgiRad = prev + 7 * (size_t)npix;
      A.hgiW = prev + 8 * (size_t)npix;
      A.history = scene->di_frames > 0 ? 1u : 0u;
      const float *pc = scene->di_cam;
      A.pcam = make_float3(pc[0], pc[1], pc[2]);
      A.pfwd = make_float3(pc[3], pc[4], pc[5]);
      A.pright = make_float3(pc[6], pc[7], pc[8]);
      A.pup = make_float3(pc[9], pc[10], pc[11]);
      A.paspect = pc[12];
      A.pfovScale = pc[13];
      if (A.layered) {
        A.kernelId = 3;
        k_di_primary<true><<<blocks, kRenderBlock, 0, s>>>(A, k);
        A.kernelId = nrc ? 5 : 4;
        if (nrc) k_di_shade<true, true><<<blocks, kRenderBlock, 0, s>>>(A, k);
        else k_di_shade<true><<<blocks, kRenderBlock, 0, s>>>(A, k);
      } else {
        A.kernelId = 3;
        k_di_primary<false><<<blocks, kRenderBlock, 0, s>>>(A, k);
        A.kernelId = nrc ? 5 : 4;
        if (nrc) k_di_shade<false, true><<<blocks, kRenderBlock, 0, s>>>(A, k);
        else k_di_shade<false><<<blocks, kRenderBlock, 0, s>>>(A, k);
      }
      VT_CUDA(ctx, cudaGetLastError());
      scene->di_parity ^= 1u;
      ++scene->di_frames;
      std::memcpy(scene->di_cam, cam, sizeof cam);
    }
    if (nrc) {
      const vt_status st = nrc_finish(ctx, nrc, A, spp, s);
      if (st != VT_OK) return st;
    }
    scene->samples += spp;
    return VT_OK;
  }
  // Enough (pixel, sample group) items to fill the GPU about four times over.
  const uint64_t target = (uint64_t)ctx->sm_count * 2048u * 4u;
  uint32_t groups = (uint32_t)std::min<uint64_t>(spp, std::max<uint64_t>(1, (target + npix - 1) / npix));
  const uint32_t per = (spp + groups - 1) / groups;
  groups = (spp + per - 1) / per;
  const uint64_t items = (uint64_t)npix * groups;
  const uint32_t grid = (uint32_t)std::min<uint64_t>((items + kRenderBlock - 1) / kRenderBlock, (uint64_t)ctx->sm_count * 32u);
  if (nrc) {
    A.kernelId = 2;
    if (A.layered) k_render<true, true><<<grid, kRenderBlock, 0, s>>>(A, groups, per);
    else k_render<false, true><<<grid, kRenderBlock, 0, s>>>(A, groups, per);
    VT_CUDA(ctx, cudaGetLastError());
    const vt_status st = nrc_finish(ctx, nrc, A, spp, s);
    if (st != VT_OK) return st;
  } else {
    A.kernelId = 1;
    if (A.layered) k_render<true><<<grid, kRenderBlock, 0, s>>>(A, groups, per);
    else k_render<false><<<grid, kRenderBlock, 0, s>>>(A, groups, per);
    VT_CUDA(ctx, cudaGetLastError());
  }
  scene->samples += spp;
  return VT_OK;
}


// ---- wavefront integrator: host side ------------------------------------------------------------
// Paths per pass: as many whole samples of the frame as fit 4M paths (about 1 GB of state).
constexpr uint32_t kWfMaxPaths = 1u << 22;

// Bytes of wavefront state per path (each array 256-byte aligned in wf_carve).
size_t wf_carve(unsigned char *base, uint32_t cap, WfArgs &W, uint32_t **q0, uint32_t **q1, uint32_t **counts,
                uint8_t **occ, int4 **hit) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    unsigned char *p = base ? base + off : nullptr;
    off += (bytes + 255) & ~size_t(255);
    return p;
  };
  const size_t n = cap;
  W.T = reinterpret_cast<float4 *>(take(16 * n));
  W.Rc = reinterpret_cast<float4 *>(take(16 * n));
  W.Rp = reinterpret_cast<float4 *>(take(16 * n));
  W.prev = reinterpret_cast<float4 *>(take(16 * n));
  W.prevN = reinterpret_cast<float4 *>(take(16 * n));
  W.seedA = reinterpret_cast<uint4 *>(take(16 * n));
  W.seedB = reinterpret_cast<uint2 *>(take(8 * n));
  W.meta = reinterpret_cast<uint4 *>(take(16 * n));
  W.spread = reinterpret_cast<float2 *>(take(8 * n));
  W.ray = reinterpret_cast<float4 *>(take(32 * n));
  *hit = reinterpret_cast<int4 *>(take(16 * n));
  W.sray = reinterpret_cast<float4 *>(take(32 * n));
  W.scon = reinterpret_cast<float4 *>(take(16 * n));
  *occ = reinterpret_cast<uint8_t *>(take(n));
  *q0 = reinterpret_cast<uint32_t *>(take(4 * n));
  *q1 = reinterpret_cast<uint32_t *>(take(4 * n));
  W.shQ = reinterpret_cast<uint32_t *>(take(4 * n));
  W.grpQ = reinterpret_cast<uint32_t *>(take(4 * n));
  *counts = reinterpret_cast<uint32_t *>(take(64));
  return off;
}

vt_status nrc_finish(vt_ctx *ctx, vt_nrc *nrc, const RenderArgs &A, uint32_t spp, cudaStream_t s);

// Launch settings of a wavefront render and where its state lives. The defaults are vt_render_wavefront's:
// the scene's own state, up to 4M paths per pass, 256-thread stage blocks, compaction every bounce and the
// frame jitter uploaded from the host. Batches give each stream its own state and tune the rest.
struct WfRun {
  unsigned char **state = nullptr;  // state buffer (null: the scene's own)
  uint32_t *stateCap = nullptr;     // its capacity in paths
  uint32_t maxPaths = kWfMaxPaths;  // queue size: paths per pass
  int block = kWfBlock;             // stage kernels' block size (at most kWfBlock)
  uint32_t compactEvery = 1;        // compact the live queue on every n-th bounce
  bool deviceJitter = false;        // the camera jitter computed in k_wf_generate (no host upload)
};

// vt_render_wavefront, and with a cache (nrc not null, sampling mode 1) vt_render_nrc's rendering:
// paths ending where the cache's query rule stops them, then the predictions and the resolve.
vt_status wavefront_impl(vt_ctx *ctx, vt_scene *scene, const vt_frame_params *p, uint32_t spp, void *stream,
                         vt_nrc *nrc = nullptr, const WfRun &run = WfRun()) {
  if (p->sampling_mode == 0)
    return vt_fail(ctx, VT_ERR_INVALID, "the wavefront integrator renders sampling modes 1-3 (ReSTIR DI frames use vt_render)");
  {
    const vt_status st = check_params(ctx, scene, p);
    if (st != VT_OK) return st;
  }
  const vt_mesh *mesh = scene->mesh;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  {
    const vt_status st = ensure_accum(ctx, scene, p);
    if (st != VT_OK) return st;
  }
  if (spp == 0) return VT_OK;
  if (!run.deviceJitter) {
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
  }
  if (mesh->nfaces == 0) { scene->samples += spp; return VT_OK; }

  RenderArgs A;
  fill_args(scene, p, spp, A);
  A.jitter = run.deviceJitter ? nullptr : scene->d_jitter;
  A.status = ctx->d_status + 2;
  A.kernelId = 7;
  const uint32_t npix = A.OW * A.OH;
  const uint32_t maxPaths = std::min(run.maxPaths, kWfMaxPaths);
  if (npix > maxPaths)
    return vt_fail(ctx, VT_ERR_LIMIT, "the frame has more pixels than the wavefront queue holds (" + std::to_string(maxPaths) + ")");
  if (nrc) {
    const vt_status st = vt_nrc_reserve_queries(ctx, nrc, (size_t)npix * spp);
    if (st != VT_OK) return st;
    A.nrcIn = nrc->d_q;
    A.nrcT = nrc->d_qT;
    A.nrcBins = nrc->d_qbins;
    A.nrcVertex = nrc->cfg.query_vertex;
    A.nrcSpread = nrc->cfg.spread;
  }
  const uint32_t chunk = std::max(1u, std::min(spp, maxPaths / npix));
  const uint32_t cap = npix * chunk;
  unsigned char **state = run.state ? run.state : &scene->d_wf;
  uint32_t *stateCap = run.state ? run.stateCap : &scene->wf_cap;
  if (cap > *stateCap) {
    cudaFree(*state);
    *state = nullptr;
    *stateCap = 0;
    WfArgs probe;
    uint32_t *a, *b, *c;
    uint8_t *o;
    int4 *h;
    const size_t bytes = wf_carve(nullptr, cap, probe, &a, &b, &c, &o, &h);
    VT_CUDA(ctx, cudaMalloc(state, bytes));
    *stateCap = cap;
  }
  WfArgs W;
  uint32_t *q[2], *counts;
  uint8_t *occ;
  int4 *hit;
  wf_carve(*state, *stateCap, W, &q[0], &q[1], &counts, &occ, &hit);
  W.hit = hit;
  W.occ = occ;
  W.npix = npix;
  const uint32_t every = std::max(1u, run.compactEvery);
  W.deadFlags = every > 1u ? 1u : 0u;
  const int block = std::max(32, std::min(run.block, kWfBlock));
  const bool pbr = A.layered != 0u, unbounded = scene_has_delta(scene);
  const bool group = pbr && A.spectral && scene->has_film;
  const uint32_t gridMax = (uint32_t)ctx->sm_count * (8u * kWfBlock / (uint32_t)block);
  uint32_t *slot = vt_queue_slot(ctx);
  for (uint32_t k0 = 0; k0 < spp; k0 += chunk) {
    const uint32_t P = npix * std::min(chunk, spp - k0);
    W.paths = P;
    W.k0 = k0;
    const uint32_t grid = std::min<uint32_t>((P + block - 1) / block, gridMax);
    k_wf_generate<<<grid, block, 0, s>>>(A, W);
    VT_CUDA(ctx, cudaGetLastError());
    for (uint32_t b = 0;; ++b) {
      if (b > A.maxDepth) {
        // Ideal reflections and refractions spend no scattering event, so paths through glass and
        // mirrors can outlive the depth (Russian roulette ends them): bounce on while a path lives,
        // its count read back every 8 bounces (compacted queues from the depth on).
        if (!unbounded) break;
        if ((b - A.maxDepth - 1u) % 8u == 0u) {
          uint32_t live = 0;
          VT_CUDA(ctx, cudaMemcpyAsync(&live, counts + (b & 1u), sizeof live, cudaMemcpyDeviceToHost, s));
          VT_CUDA(ctx, cudaStreamSynchronize(s));
          if (live == 0u) break;
        }
      }
      W.compact = ((b + 1u) % every == 0u || b >= A.maxDepth) ? 1u : 0u;
      // Live queue of bounce b (all paths at b = 0), the next bounce's queue and the shadow queue.
      const uint32_t *inQ = b == 0 ? nullptr : q[b & 1u];
      const uint32_t *inCount = b == 0 ? nullptr : counts + (b & 1u);
      W.inQ = inQ;
      W.inCount = inCount;
      W.outQ = q[(b + 1) & 1u];
      W.outCount = counts + ((b + 1) & 1u);
      W.shCount = counts + 2;
      VT_CUDA(ctx, cudaMemsetAsync(W.outCount, 0, sizeof(uint32_t), s));
      VT_CUDA(ctx, cudaMemsetAsync(W.shCount, 0, sizeof(uint32_t), s));
      vt_launch_closest(mesh, reinterpret_cast<const vt_ray *>(W.ray), P, reinterpret_cast<vt_hit *>(hit), ctx->sm_count,
                        slot, inQ, ctx->d_status + 1, s, inCount, true);
      if (group) {
        VT_CUDA(ctx, cudaMemsetAsync(counts + 3, 0, 2 * sizeof(uint32_t), s));
        k_wf_group<<<grid, block, 0, s>>>(A, W, counts + 3);
        W.inQ = W.grpQ;  // the same entries, regrouped (the count stays)
      }
      if (nrc) {
        if (pbr) k_wf_shade<true, true><<<grid, block, 0, s>>>(A, W, b);
        else k_wf_shade<false, true><<<grid, block, 0, s>>>(A, W, b);
      } else {
        if (pbr) k_wf_shade<true, false><<<grid, block, 0, s>>>(A, W, b);
        else k_wf_shade<false, false><<<grid, block, 0, s>>>(A, W, b);
      }
      vt_launch_any(mesh, reinterpret_cast<const vt_ray *>(W.sray), P, occ, ctx->sm_count, slot, W.shQ, ctx->d_status + 1, s,
                    W.shCount, A.imported != 0u);
      VT_CUDA(ctx, cudaGetLastError());
    }
    if (nrc) k_wf_finish<true><<<grid, block, 0, s>>>(A, W);
    else k_wf_finish<false><<<grid, block, 0, s>>>(A, W);
    VT_CUDA(ctx, cudaGetLastError());
  }
  if (nrc) {
    const vt_status st = nrc_finish(ctx, nrc, A, spp, s);
    if (st != VT_OK) return st;
  }
  scene->samples += spp;
  return VT_OK;
}
}  // namespace

extern "C" {

vt_status vt_render(vt_ctx *ctx, vt_scene *scene, const vt_frame_params *p, uint32_t spp, void *stream) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene || !p) return vt_fail(ctx, VT_ERR_INVALID, "scene or params is null");
  return render_impl(ctx, scene, p, spp, stream, nullptr);
}

vt_status vt_render_wavefront(vt_ctx *ctx, vt_scene *scene, const vt_frame_params *p, uint32_t spp, void *stream) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene || !p) return vt_fail(ctx, VT_ERR_INVALID, "scene or params is null");
  return wavefront_impl(ctx, scene, p, spp, stream);
}

vt_status vt_render_nrc(vt_ctx *ctx, vt_scene *scene, vt_nrc *nrc, const vt_frame_params *p, uint32_t spp,
                        uint32_t flags, void *stream) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene || !p || !nrc) return vt_fail(ctx, VT_ERR_INVALID, "scene, nrc or params is null");
  if (flags & ~(uint32_t)(VT_NRC_TRAIN | VT_NRC_RENDER)) return vt_fail(ctx, VT_ERR_INVALID, "unknown flags");
  if ((flags & VT_NRC_RENDER) && p->sampling_mode > 1)
    return vt_fail(ctx, VT_ERR_INVALID, "the cache renders sampling modes 0 (ReSTIR DI) and 1 (MIS)");
  if ((p->spectral != 0) != (nrc->cfg.spectral != 0))
    return vt_fail(ctx, VT_ERR_INVALID, "the frame's transport (spectral or rgb) differs from the cache's `spectral` setting");
  if (p->pixel_stride > 1) return vt_fail(ctx, VT_ERR_INVALID, "the cache renders whole frames (pixel_stride 0 or 1)");
  if ((flags & VT_NRC_RENDER) && p->sampling_mode == 0u && scene_has_delta(scene))
    return vt_fail(ctx, VT_ERR_INVALID, "the cache's ReSTIR DI frames (sampling mode 0) do not take glass or mirror slots; "
                                        "render them in sampling mode 1");
  {
    const vt_status st = check_params(ctx, scene, p);
    if (st != VT_OK) return st;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  // Training and rendering: the training paths run on the cache's side stream beside the frame's
  // rendering (which reads the parameters of the previous step); the step follows both.
  const bool both = (flags & VT_NRC_TRAIN) && (flags & VT_NRC_RENDER) && scene->mesh->nfaces > 0;
  cudaStream_t ps = s;
  if (both) {
    VT_CUDA(ctx, cudaEventRecord(nrc->ev_start, s));
    VT_CUDA(ctx, cudaStreamWaitEvent(nrc->side, nrc->ev_start, 0));
    ps = nrc->side;
  }
  if ((flags & VT_NRC_TRAIN) && scene->mesh->nfaces > 0) {
    const uint32_t cap = nrc->cfg.train_records;
    const uint32_t npaths = nrc->cfg.train_paths ? nrc->cfg.train_paths : std::max(1u, cap / 4u);
    {
      const vt_status st = vt_nrc_reserve_records(ctx, nrc, cap);
      if (st != VT_OK) return st;
    }
    RenderArgs A;
    fill_args(scene, p, 1, A);
    A.status = ctx->d_status + 2;
    A.kernelId = 6;
    const uint32_t npix = p->width * p->height;
    // A fresh pixel pattern each frame: an offset from the frame's index, pixels `stride` apart.
    const uint32_t frame = nrc->frames++;
    uint32_t h = nrc->cfg.seed ^ (frame * 0x9e3779b9u);
    h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
    const uint32_t stride = std::max(1u, npix / npaths);
    VT_CUDA(ctx, cudaMemsetAsync(nrc->d_count, 0, sizeof(uint32_t), ps));
    const uint32_t si0 = 0x40000000u + (frame << 8);
    const size_t scratch = (size_t)npaths * kNrcRecords * 5;
    if (scratch > nrc->scratch_cap) {
      cudaFree(nrc->d_scratch);
      nrc->d_scratch = nullptr;
      nrc->scratch_cap = 0;
      VT_CUDA(ctx, cudaMalloc(&nrc->d_scratch, scratch * sizeof(float4)));
      nrc->scratch_cap = scratch;
    }
    const unsigned blocks = (npaths + kRenderBlock - 1) / kRenderBlock;
    if (A.layered)
      k_nrc_paths<true><<<blocks, kRenderBlock, 0, ps>>>(A, npaths, h % npix, stride, si0, cap, nrc->d_scratch,
                                                        nrc->scratch_cap, nrc->d_tin, nrc->d_ttarget, nrc->tcap,
                                                        nrc->d_count);
    else
      k_nrc_paths<false><<<blocks, kRenderBlock, 0, ps>>>(A, npaths, h % npix, stride, si0, cap, nrc->d_scratch,
                                                         nrc->scratch_cap, nrc->d_tin, nrc->d_ttarget, nrc->tcap,
                                                         nrc->d_count);
    VT_CUDA(ctx, cudaGetLastError());
    if (!both) {
      const vt_status st = vt_nrc_step(ctx, nrc, cap, s);
      if (st != VT_OK) return st;
    }
  }
  if (flags & VT_NRC_RENDER) {
    // MIS primaries through the wavefront integrator; ReSTIR DI's frames through its two passes
    // (compiled without glass and mirrors, see continue_path).
    const vt_status st = p->sampling_mode == 1u ? wavefront_impl(ctx, scene, p, spp, stream, nrc)
                                                : render_impl(ctx, scene, p, spp, stream, nrc);
    if (both) {
      VT_CUDA(ctx, cudaEventRecord(nrc->ev_paths, nrc->side));
      VT_CUDA(ctx, cudaStreamWaitEvent(s, nrc->ev_paths, 0));
      if (st != VT_OK) return st;
      return vt_nrc_step(ctx, nrc, nrc->cfg.train_records, s);
    }
    return st;
  }
  return VT_OK;
}

}  // extern "C"

// A batch of scenes rendered by one persistent launch per pass (vt_batch_*).
struct vt_batch {
  struct Config {
    int block;
    uint32_t chunk;
    float ms;
  };
  std::vector<vt_scene *> scenes;
  std::vector<uint32_t> spp;
  unsigned long long total = 0;
  RenderArgs *d_args = nullptr;
  unsigned long long *d_begin = nullptr, *d_counter = nullptr, *d_start = nullptr, *d_doneNs = nullptr;
  uint32_t *d_first = nullptr, *d_frame = nullptr, *d_done = nullptr;
  std::vector<Config> configs;
  size_t tried = 0;
  int best = -1;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float last_ms = 0.0f;
  uint32_t passes = 0;
  bool pbr = false;  // some scene has OPENPBR slots: the kernel variant with the OpenPBR code
  int mode = 0;      // the integrator of the batch's passes: 0 none yet, 1 megakernel, 2 wavefront
  // Wavefront passes (vt_batch_render_wavefront): per-scene queues on kStreams streams, each stream
  // with its own path state; the scenes' frame parameters kept on the host and advanced per pass.
  static constexpr int kStreams = 4;
  struct WfConfig {
    uint32_t queue;  // paths per wavefront pass
    int block;       // stage kernels' block size
    uint32_t every;  // compaction frequency (bounces)
    float ms;
  };
  std::vector<vt_frame_params> params;
  std::vector<WfConfig> wfConfigs;
  size_t wfTried = 0, wfLast = 0;  // configs tried; the config of the last pass
  int wfBest = -1;
  cudaStream_t streams[kStreams] = {};
  cudaEvent_t fork = nullptr, join[kStreams] = {};
  unsigned char *state[kStreams] = {};
  uint32_t stateCap[kStreams] = {};
  std::vector<cudaEvent_t> sceneEv;
  std::vector<int> streamOf;     // stream of each scene (longest-processing-time assignment)
  std::vector<uint32_t> orderBy; // scenes by decreasing work
  std::vector<double> sceneMs;   // completion of each scene from the pass's start (wavefront)
};

namespace {

void batch_free(vt_batch *b) {
  for (int k = 0; k < vt_batch::kStreams; ++k) {
    if (b->streams[k]) cudaStreamDestroy(b->streams[k]);
    if (b->join[k]) cudaEventDestroy(b->join[k]);
    cudaFree(b->state[k]);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  for (cudaEvent_t e : b->sceneEv) cudaEventDestroy(e);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->e0) cudaEventDestroy(b->e0);
  if (b->e1) cudaEventDestroy(b->e1);
  cudaFree(b->d_args);
  cudaFree(b->d_begin);
  cudaFree(b->d_counter);
  cudaFree(b->d_start);
  cudaFree(b->d_doneNs);
  cudaFree(b->d_first);
  cudaFree(b->d_frame);
  cudaFree(b->d_done);
  delete b;
}

// One pass: reset the work counter and start stamp, run every scene's items, advance the indices.
cudaError_t batch_enqueue(vt_ctx *ctx, vt_batch *b, const vt_batch::Config &c, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->d_start, 0xff, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  int perSm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, b->pbr ? k_render_batch<true> : k_render_batch<false>, c.block, 0) !=
          cudaSuccess || perSm < 1)
    perSm = 1;
  const unsigned long long warps = (b->total + 32ull * c.chunk - 1) / (32ull * c.chunk);
  const unsigned long long want = (warps * 32ull + c.block - 1) / c.block;
  const unsigned grid = (unsigned)std::min<unsigned long long>(want, (unsigned long long)perSm * ctx->sm_count);
  const uint32_t n = (uint32_t)b->scenes.size();
  (b->pbr ? k_render_batch<true> : k_render_batch<false>)<<<grid, c.block, 0, s>>>(b->d_args, b->d_begin, n, b->total, c.chunk, b->d_first, b->d_frame,
                                           b->d_counter, b->d_start, b->d_done, b->d_doneNs);
  k_batch_advance<<<(n + 127) / 128, 128, 0, s>>>(b->d_args, n, b->d_first, b->d_frame, b->d_done);
  return cudaGetLastError();
}

}  // namespace

extern "C" {

vt_status vt_environment_tables(const float *rgba, uint32_t width, uint32_t height, float *rows, float *cols) {
  if (!rgba || !rows || !cols || width == 0 || height == 0) return VT_ERR_INVALID;
  environment_tables(rgba, width, height, rows, cols);
  return VT_OK;
}

vt_status vt_scene_set_environment_map(vt_ctx *ctx, vt_scene *scene, const float *rgba, uint32_t width, uint32_t height,
                                       float intensity, float rotation) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene) return vt_fail(ctx, VT_ERR_INVALID, "scene is null");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!rgba || !(intensity > 0.0f)) {
    scene->env_map = false;
    scene->environment = vt_environment{};
    return vt_accum_reset(ctx, scene);
  }
  if (!scene->imported) return vt_fail(ctx, VT_ERR_INVALID, "an environment needs an imported scene");
  if (!std::isfinite(intensity) || !std::isfinite(rotation)) return vt_fail(ctx, VT_ERR_INVALID, "intensity and rotation must be finite");
  if (width == 0 || height == 0 || width > 16384 || height > 8192 || (uint64_t)width * height > 33554432ull)
    return vt_fail(ctx, VT_ERR_INVALID, "Could not decode the environment image (maximum 16384x8192).");
  const size_t n = (size_t)width * height;
  std::vector<float> px(4 * n);
  for (size_t i = 0; i < 4 * n; ++i) {
    if (!std::isfinite(rgba[i])) return vt_fail(ctx, VT_ERR_INVALID, "Environment pixels must be finite.");
    px[i] = rgba[i] < 0.0f ? 0.0f : rgba[i];  // radiance is non-negative
  }
  std::vector<float> rows(2 * (size_t)height), cols(2 * n);
  environment_tables(px.data(), width, height, rows.data(), cols.data());
  cudaFree(scene->d_env_img);
  cudaFree(scene->d_env_rows);
  cudaFree(scene->d_env_cols);
  scene->d_env_img = nullptr;
  scene->d_env_rows = scene->d_env_cols = nullptr;
  scene->env_map = false;
  VT_CUDA(ctx, cudaMalloc(&scene->d_env_img, n * sizeof(float4)));
  VT_CUDA(ctx, cudaMalloc(&scene->d_env_rows, rows.size() * sizeof(float)));
  VT_CUDA(ctx, cudaMalloc(&scene->d_env_cols, cols.size() * sizeof(float)));
  VT_CUDA(ctx, cudaMemcpy(scene->d_env_img, px.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
  VT_CUDA(ctx, cudaMemcpy(scene->d_env_rows, rows.data(), rows.size() * sizeof(float), cudaMemcpyHostToDevice));
  VT_CUDA(ctx, cudaMemcpy(scene->d_env_cols, cols.data(), cols.size() * sizeof(float), cudaMemcpyHostToDevice));
  scene->env_w = width;
  scene->env_h = height;
  scene->env_rot = rotation;
  scene->env_map = true;
  vt_environment e{};
  e.intensity = intensity;
  e.sun_dir[1] = 1.0f;
  scene->environment = e;
  return vt_accum_reset(ctx, scene);
}

vt_status vt_batch_create(vt_ctx *ctx, vt_scene *const *scenes, const vt_frame_params *params, const uint32_t *spp,
                          uint32_t n, vt_batch **out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scenes || !params || !spp || !out || n == 0) return vt_fail(ctx, VT_ERR_INVALID, "null argument or empty batch");
  *out = nullptr;
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  for (uint32_t i = 0; i < n; ++i) {
    if (!scenes[i]) return vt_fail(ctx, VT_ERR_INVALID, "scene " + std::to_string(i) + " is null");
    for (uint32_t j = 0; j < i; ++j)
      if (scenes[j] == scenes[i]) return vt_fail(ctx, VT_ERR_INVALID, "a scene appears twice in the batch");
    const vt_status st = check_params(ctx, scenes[i], params + i);
    if (st != VT_OK) return st;
    if (params[i].sampling_mode == 0)
      return vt_fail(ctx, VT_ERR_INVALID, "batched scenes use sampling modes 1-3 (ReSTIR DI frames run in order per scene)");
    if (params[i].pixel_stride > 1) return vt_fail(ctx, VT_ERR_INVALID, "batched scenes render whole frames (pixel_stride 0 or 1)");
    if (spp[i] == 0 || spp[i] > 65536) return vt_fail(ctx, VT_ERR_INVALID, "spp must be 1 .. 65536 per scene");
    if (scenes[i]->mesh->nfaces == 0) return vt_fail(ctx, VT_ERR_INVALID, "scene " + std::to_string(i) + " has no faces");
  }
  vt_batch *b = new vt_batch();
  std::vector<RenderArgs> args(n);
  std::vector<unsigned long long> begin(n + 1, 0);
  std::vector<uint32_t> first(n), frame(n);
  for (uint32_t i = 0; i < n; ++i) {
    vt_status st = ensure_accum(ctx, scenes[i], params + i);
    if (st != VT_OK) { batch_free(b); return st; }
    fill_args(scenes[i], params + i, spp[i], args[i]);
    args[i].status = ctx->d_status + 2;
    args[i].kernelId = 7;
    args[i].jitter = nullptr;
    first[i] = args[i].first;
    if (args[i].layered) b->pbr = true;
    frame[i] = args[i].firstFrame;
    begin[i + 1] = begin[i] + (unsigned long long)params[i].width * params[i].height;
    b->scenes.push_back(scenes[i]);
    b->spp.push_back(spp[i]);
    b->params.push_back(params[i]);
  }
  b->total = begin[n];
  auto fail = [&](cudaError_t e, const char *what) { batch_free(b); return vt_cuda_fail(ctx, e, what); };
  cudaError_t e;
  if ((e = cudaMalloc(&b->d_args, n * sizeof(RenderArgs))) != cudaSuccess) return fail(e, "cudaMalloc(batch args)");
  if ((e = cudaMalloc(&b->d_begin, (n + 1) * sizeof(unsigned long long))) != cudaSuccess) return fail(e, "cudaMalloc(batch)");
  if ((e = cudaMalloc(&b->d_counter, sizeof(unsigned long long))) != cudaSuccess) return fail(e, "cudaMalloc(batch)");
  if ((e = cudaMalloc(&b->d_start, sizeof(unsigned long long))) != cudaSuccess) return fail(e, "cudaMalloc(batch)");
  if ((e = cudaMalloc(&b->d_doneNs, n * sizeof(unsigned long long))) != cudaSuccess) return fail(e, "cudaMalloc(batch)");
  if ((e = cudaMalloc(&b->d_first, n * sizeof(uint32_t))) != cudaSuccess) return fail(e, "cudaMalloc(batch)");
  if ((e = cudaMalloc(&b->d_frame, n * sizeof(uint32_t))) != cudaSuccess) return fail(e, "cudaMalloc(batch)");
  if ((e = cudaMalloc(&b->d_done, n * sizeof(uint32_t))) != cudaSuccess) return fail(e, "cudaMalloc(batch)");
  if ((e = cudaMemcpy(b->d_args, args.data(), n * sizeof(RenderArgs), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(b->d_begin, begin.data(), (n + 1) * sizeof(unsigned long long), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(b->d_first, first.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(b->d_frame, frame.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemset(b->d_done, 0, n * sizeof(uint32_t))) != cudaSuccess ||
      (e = cudaMemset(b->d_doneNs, 0, n * sizeof(unsigned long long))) != cudaSuccess)
    return fail(e, "uploading the batch");
  if ((e = cudaEventCreate(&b->e0)) != cudaSuccess || (e = cudaEventCreate(&b->e1)) != cudaSuccess)
    return fail(e, "cudaEventCreate");
  // Launch shapes the first passes try, one each; the fastest is then captured in a graph.
  for (int block : {64, 128, 256})
    for (uint32_t chunk : {1u, 4u}) b->configs.push_back({block, chunk, 0.0f});
  // Wavefront settings the first wavefront passes try, one each: queue size x block size x
  // compaction frequency. Queues must hold the largest frame.
  uint32_t maxPix = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t s = std::max(1u, params[i].pixel_stride);
    maxPix = std::max(maxPix, ((params[i].width + s - 1) / s) * ((params[i].height + s - 1) / s));
  }
  for (uint32_t queue : {1u << 20, 1u << 22})
    for (int block : {128, 256})
      for (uint32_t every : {1u, 2u})
        if (queue >= maxPix) b->wfConfigs.push_back({queue, block, every, 0.0f});
  if (b->wfConfigs.empty()) b->wfConfigs.push_back({kWfMaxPaths, kWfBlock, 1u, 0.0f});
  *out = b;
  return VT_OK;
}

vt_status vt_batch_render(vt_ctx *ctx, vt_batch *b, void *stream) {
  if (!ctx) return VT_ERR_INVALID;
  if (!b) return vt_fail(ctx, VT_ERR_INVALID, "batch is null");
  if (b->mode == 2) return vt_fail(ctx, VT_ERR_INVALID, "this batch renders through the wavefront integrator");
  b->mode = 1;
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  VT_CUDA(ctx, cudaEventRecord(b->e0, s));
  if (b->best < 0) {
    const cudaError_t be = batch_enqueue(ctx, b, b->configs[b->tried], s);
    if (be != cudaSuccess) return vt_cuda_fail(ctx, be, "batched render");
  } else {
    VT_CUDA(ctx, cudaGraphLaunch(b->exec, s));
  }
  VT_CUDA(ctx, cudaEventRecord(b->e1, s));
  VT_CUDA(ctx, cudaEventSynchronize(b->e1));
  VT_CUDA(ctx, cudaEventElapsedTime(&b->last_ms, b->e0, b->e1));
  for (size_t i = 0; i < b->scenes.size(); ++i) b->scenes[i]->samples += b->spp[i];
  ++b->passes;
  if (b->best < 0) {
    b->configs[b->tried].ms = b->last_ms;
    if (++b->tried == b->configs.size()) {
      b->best = 0;
      for (size_t c = 1; c < b->configs.size(); ++c)
        if (b->configs[c].ms < b->configs[b->best].ms) b->best = (int)c;
      // Capture the fastest shape: later passes replay one graph.
      VT_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      const cudaError_t ce = batch_enqueue(ctx, b, b->configs[b->best], ctx->stream);
      cudaGraph_t g = nullptr;
      const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &g);
      if (ce != cudaSuccess) { if (g) cudaGraphDestroy(g); return vt_cuda_fail(ctx, ce, "capturing the batch"); }
      VT_CUDA(ctx, ee);
      b->graph = g;
      VT_CUDA(ctx, cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
  }
  return VT_OK;
}

vt_status vt_batch_render_wavefront(vt_ctx *ctx, vt_batch *b, void *stream) {
  if (!ctx) return VT_ERR_INVALID;
  if (!b) return vt_fail(ctx, VT_ERR_INVALID, "batch is null");
  if (b->mode == 1) return vt_fail(ctx, VT_ERR_INVALID, "this batch renders through the persistent megakernel");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  const uint32_t n = (uint32_t)b->scenes.size();
  if (b->mode == 0) {
    b->mode = 2;
    for (int k = 0; k < vt_batch::kStreams; ++k) {
      VT_CUDA(ctx, cudaStreamCreateWithFlags(&b->streams[k], cudaStreamNonBlocking));
      VT_CUDA(ctx, cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming));
    }
    VT_CUDA(ctx, cudaEventCreate(&b->fork));
    b->sceneEv.assign(n, nullptr);
    for (uint32_t i = 0; i < n; ++i) VT_CUDA(ctx, cudaEventCreate(&b->sceneEv[i]));
    b->sceneMs.assign(n, 0.0);
    // Longest processing time first: scenes by decreasing paths, each to the least loaded stream.
    b->orderBy.resize(n);
    for (uint32_t i = 0; i < n; ++i) b->orderBy[i] = i;
    auto work = [&](uint32_t i) { return (double)b->params[i].width * b->params[i].height * b->spp[i]; };
    std::stable_sort(b->orderBy.begin(), b->orderBy.end(), [&](uint32_t x, uint32_t y) { return work(x) > work(y); });
    b->streamOf.assign(n, 0);
    double load[vt_batch::kStreams] = {};
    for (uint32_t i : b->orderBy) {
      int k = 0;
      for (int j = 1; j < vt_batch::kStreams; ++j)
        if (load[j] < load[k]) k = j;
      b->streamOf[i] = k;
      load[k] += work(i);
    }
  }
  b->wfLast = b->wfBest >= 0 ? (size_t)b->wfBest : b->wfTried;
  const vt_batch::WfConfig &c = b->wfConfigs[b->wfLast];
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  VT_CUDA(ctx, cudaEventRecord(b->fork, s));
  for (int k = 0; k < vt_batch::kStreams; ++k) VT_CUDA(ctx, cudaStreamWaitEvent(b->streams[k], b->fork, 0));
  for (uint32_t i : b->orderBy) {
    const int k = b->streamOf[i];
    WfRun run;
    run.state = &b->state[k];
    run.stateCap = &b->stateCap[k];
    run.maxPaths = c.queue;
    run.block = c.block;
    run.compactEvery = c.every;
    run.deviceJitter = true;
    const vt_status st = wavefront_impl(ctx, b->scenes[i], &b->params[i], b->spp[i], b->streams[k], nullptr, run);
    if (st != VT_OK) return st;
    VT_CUDA(ctx, cudaEventRecord(b->sceneEv[i], b->streams[k]));
    vt_frame_params &p = b->params[i];
    p.first_sample += b->spp[i];
    if (p.first_frame) p.first_frame += b->spp[i];
  }
  for (int k = 0; k < vt_batch::kStreams; ++k) {
    VT_CUDA(ctx, cudaEventRecord(b->join[k], b->streams[k]));
    VT_CUDA(ctx, cudaStreamWaitEvent(s, b->join[k], 0));
  }
  VT_CUDA(ctx, cudaEventRecord(b->e1, s));
  VT_CUDA(ctx, cudaEventSynchronize(b->e1));
  VT_CUDA(ctx, cudaEventElapsedTime(&b->last_ms, b->fork, b->e1));
  for (uint32_t i = 0; i < n; ++i) {
    float ms = 0.0f;
    VT_CUDA(ctx, cudaEventElapsedTime(&ms, b->fork, b->sceneEv[i]));
    b->sceneMs[i] = ms;
  }
  ++b->passes;
  if (b->wfBest < 0) {
    b->wfConfigs[b->wfTried].ms = b->last_ms;
    if (++b->wfTried == b->wfConfigs.size()) {
      b->wfBest = 0;
      for (size_t k = 1; k < b->wfConfigs.size(); ++k)
        if (b->wfConfigs[k].ms < b->wfConfigs[b->wfBest].ms) b->wfBest = (int)k;
    }
  }
  return VT_OK;
}

vt_status vt_batch_stats(vt_ctx *ctx, const vt_batch *b, vt_batch_info *out, double *scene_ms, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!b || !out) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  if (scene_ms && n != b->scenes.size()) return vt_fail(ctx, VT_ERR_INVALID, "n must equal the batch's scene count");
  std::memset(out, 0, sizeof *out);
  out->scenes = (uint32_t)b->scenes.size();
  out->passes = b->passes;
  out->items = b->total;
  out->last_ms = b->last_ms;
  if (b->mode == 2) {
    out->wavefront = 1;
    out->tuned = b->wfBest >= 0 ? 1u : 0u;
    const vt_batch::WfConfig &c = b->wfConfigs[b->wfLast];
    out->block = (uint32_t)c.block;
    out->queue_paths = c.queue;
    out->compact_every = c.every;
    out->streams = vt_batch::kStreams;
    if (scene_ms && b->passes)
      for (size_t i = 0; i < b->scenes.size(); ++i) scene_ms[i] = b->sceneMs[i];
    return VT_OK;
  }
  out->tuned = b->best >= 0 ? 1u : 0u;
  const vt_batch::Config &c = b->configs[b->best >= 0 ? (size_t)b->best : (b->tried ? b->tried - 1 : 0)];
  out->block = (uint32_t)c.block;
  out->chunk = c.chunk;
  if (scene_ms && b->passes) {
    std::vector<unsigned long long> done(b->scenes.size());
    unsigned long long start = 0;
    VT_CUDA(ctx, cudaDeviceSynchronize());
    VT_CUDA(ctx, cudaMemcpy(done.data(), b->d_doneNs, done.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    VT_CUDA(ctx, cudaMemcpy(&start, b->d_start, sizeof start, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < done.size(); ++i) scene_ms[i] = done[i] >= start ? double(done[i] - start) * 1e-6 : 0.0;
  }
  return VT_OK;
}

vt_status vt_batch_destroy(vt_ctx *ctx, vt_batch *b) {
  if (!b) return VT_OK;
  if (ctx) cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  batch_free(b);
  return VT_OK;
}

vt_status vt_scene_set_environment(vt_ctx *ctx, vt_scene *scene, const vt_environment *env) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene) return vt_fail(ctx, VT_ERR_INVALID, "scene is null");
  scene->env_map = false;  // the procedural sky replaces an image
  vt_environment e{};
  if (env && env->intensity > 0.0f) {
    if (!scene->imported) return vt_fail(ctx, VT_ERR_INVALID, "an environment needs an imported scene");
    e = *env;
    if (!std::isfinite(e.intensity) || !std::isfinite(e.sun_intensity) || e.sun_intensity < 0.0f)
      return vt_fail(ctx, VT_ERR_INVALID, "intensities must be finite, the sun's non-negative");
    if (e.sky_mode > 2) return vt_fail(ctx, VT_ERR_INVALID, "sky_mode must be 0, 1 or 2");
    const double l = std::sqrt((double)e.sun_dir[0] * e.sun_dir[0] + (double)e.sun_dir[1] * e.sun_dir[1] +
                               (double)e.sun_dir[2] * e.sun_dir[2]);
    if (!(l > 0.0) || !std::isfinite(l)) return vt_fail(ctx, VT_ERR_INVALID, "sun_dir must be a non-zero vector");
    for (int k = 0; k < 3; ++k) e.sun_dir[k] = (float)(e.sun_dir[k] / l);
  }
  scene->environment = e;
  return vt_accum_reset(ctx, scene);
}

vt_status vt_scene_set_openpbr(vt_ctx *ctx, vt_scene *scene, const vt_openpbr_params *params, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene || (!params && n)) return vt_fail(ctx, VT_ERR_INVALID, "scene or params is null");
  if (n != scene->nmat) return vt_fail(ctx, VT_ERR_INVALID, "n must equal the scene's material slot count");
  if (!ctx->pbr_opaque) return vt_fail(ctx, VT_ERR_INVALID, "OpenPBR tables are not set (vt_openpbr_tables_set)");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  std::vector<float4> q(kSlotF4 * (size_t)n);
  bool film = false;
  for (uint32_t i = 0; i < n; ++i) {
    const vt_openpbr_params &p = params[i];
    if (!(p.roughness >= 0.0f && p.roughness <= 1.0f) || !(p.metalness >= 0.0f && p.metalness <= 1.0f) || !(p.ior > 0.0f) ||
        !(p.diffuse_roughness >= 0.0f && p.diffuse_roughness <= 1.0f))
      return vt_fail(ctx, VT_ERR_INVALID, "OpenPBR slot " + std::to_string(i) + ": roughness, metalness and diffuse roughness "
                                          "must lie in [0, 1] and the IOR be positive");
    if (!(p.coat >= 0.0f && p.coat <= 1.0f) || !(p.fuzz >= 0.0f && p.fuzz <= 1.0f) || !(p.anisotropy >= 0.0f && p.anisotropy <= 1.0f))
      return vt_fail(ctx, VT_ERR_INVALID, "OpenPBR slot " + std::to_string(i) + ": coat and fuzz weights and the anisotropy must lie "
                                          "in [0, 1]");
    q[kSlotF4 * (size_t)i + 2] = make_float4(p.fuzz, p.anisotropy, 0.0f, 0.0f);
    if (!(p.thin_film_weight >= 0.0f && p.thin_film_weight <= 1.0f) || !(p.thin_film_thickness >= 0.0f) ||
        !std::isfinite(p.thin_film_thickness) || (p.thin_film_weight > 0.0f && !(p.thin_film_ior > 0.0f)))
      return vt_fail(ctx, VT_ERR_INVALID, "OpenPBR slot " + std::to_string(i) + ": thin-film weight must lie in [0, 1], its "
                                          "thickness be finite and non-negative and its IOR positive");
    q[kSlotF4 * (size_t)i] = make_float4(p.roughness, p.metalness, p.ior, p.diffuse_roughness);
    scene->slot_rough[i] = p.roughness;
    if (p.thin_film_weight > 0.0f) film = true;
    q[kSlotF4 * (size_t)i + 1] = make_float4(p.thin_film_weight, p.thin_film_thickness, p.thin_film_weight > 0.0f ? p.thin_film_ior : 1.4f,
                                       p.coat);
  }
  if (!scene->d_pbr && n) VT_CUDA(ctx, cudaMalloc(&scene->d_pbr, q.size() * sizeof(float4)));
  if (n) VT_CUDA(ctx, cudaMemcpy(scene->d_pbr, q.data(), q.size() * sizeof(float4), cudaMemcpyHostToDevice));
  scene->pbr_tables = ctx->d_pbr;
  scene->has_film = film;
  return VT_OK;
}

vt_status vt_scene_di_weights(vt_ctx *ctx, const vt_scene *scene, float *out, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene || !out) return vt_fail(ctx, VT_ERR_INVALID, "scene or out is null");
  if (!scene->d_di || scene->di_frames == 0) return vt_fail(ctx, VT_ERR_INVALID, "no ReSTIR DI frame rendered");
  const size_t npix = (size_t)scene->di_width * scene->di_height;
  if (n != 4 * npix) return vt_fail(ctx, VT_ERR_INVALID, "n must equal width * height * 4");
  const float4 *last = scene->d_di + 9 * npix * (scene->di_parity ^ 1u) + 4 * npix;
  VT_CUDA(ctx, cudaDeviceSynchronize());
  VT_CUDA(ctx, cudaMemcpy(out, last, npix * sizeof(float4), cudaMemcpyDeviceToHost));
  return VT_OK;
}

vt_status vt_scene_gi_weights(vt_ctx *ctx, const vt_scene *scene, float *out, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene || !out) return vt_fail(ctx, VT_ERR_INVALID, "scene or out is null");
  if (!scene->d_di || scene->di_frames == 0) return vt_fail(ctx, VT_ERR_INVALID, "no ReSTIR DI frame rendered");
  const size_t npix = (size_t)scene->di_width * scene->di_height;
  if (n != 4 * npix) return vt_fail(ctx, VT_ERR_INVALID, "n must equal width * height * 4");
  const float4 *last = scene->d_di + 9 * npix * (scene->di_parity ^ 1u) + 8 * npix;
  VT_CUDA(ctx, cudaDeviceSynchronize());
  VT_CUDA(ctx, cudaMemcpy(out, last, npix * sizeof(float4), cudaMemcpyDeviceToHost));
  return VT_OK;
}

vt_status vt_accum_readback(vt_ctx *ctx, vt_scene *scene, double *rgb, uint32_t n, uint32_t *samples) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene || !rgb) return vt_fail(ctx, VT_ERR_INVALID, "scene or rgb is null");
  const size_t want = 3 * (size_t)scene->width * scene->height;
  if (n != want) return vt_fail(ctx, VT_ERR_INVALID, "n must equal width * height * 3");
  VT_CUDA(ctx, cudaDeviceSynchronize());
  {
    uint32_t w[16];
    VT_CUDA(ctx, cudaMemcpy(w, ctx->d_status, sizeof w, cudaMemcpyDeviceToHost));
    if (w[1] & VT_DEV_STACK) {
      VT_CUDA(ctx, cudaMemset(ctx->d_status + 1, 0, sizeof(uint32_t)));
      return vt_fail(ctx, VT_ERR_DEVICE, "a traversal stack would have overflowed; the entries were dropped");
    }
    if (w[2]) {
      VT_CUDA(ctx, cudaMemset(ctx->d_status + 2, 0, sizeof(uint32_t)));
      VT_CUDA(ctx, cudaMemset(ctx->d_status + 8, 0, 3 * sizeof(uint32_t)));
      return vt_fail(ctx, VT_ERR_DEVICE,
                     "the integrator met an out-of-range index (status " + std::to_string(w[2]) +
                         ": 4 hit, 8 cache record, 16 emitter face; first: value " + std::to_string(w[9]) +
                         ", kernel " + std::to_string(w[10] & 0xffu) + "); those accesses were clamped or skipped");
    }
  }
  if (want) VT_CUDA(ctx, cudaMemcpy(rgb, scene->d_accum, want * sizeof(double), cudaMemcpyDeviceToHost));
  const double inv = scene->samples ? 1.0 / scene->samples : 0.0;
  for (size_t i = 0; i < want; ++i) rgb[i] *= inv;
  if (samples) *samples = scene->samples;
  return VT_OK;
}

vt_status vt_accum_restore(vt_ctx *ctx, vt_scene *scene, uint32_t width, uint32_t height, uint32_t pixel_stride,
                           const double *rgb, uint32_t n, uint32_t samples) {
  if (!ctx) return VT_ERR_INVALID;
  if (!scene || !rgb) return vt_fail(ctx, VT_ERR_INVALID, "scene or rgb is null");
  if (width == 0 || height == 0 || (uint64_t)width * height > (1u << 28) || pixel_stride > 64)
    return vt_fail(ctx, VT_ERR_INVALID, "bad image size or pixel stride");
  vt_frame_params p;
  std::memset(&p, 0, sizeof p);
  p.width = width;
  p.height = height;
  p.pixel_stride = pixel_stride;
  uint32_t w, h;
  accum_dims(&p, w, h);
  const size_t want = 3 * (size_t)w * h;
  if (n != want) return vt_fail(ctx, VT_ERR_INVALID, "n must equal the accumulation's pixels * 3");
  for (size_t i = 0; i < want; ++i)
    if (!std::isfinite(rgb[i])) return vt_fail(ctx, VT_ERR_INVALID, "the saved accumulation holds a non-finite value");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  VT_CUDA(ctx, cudaDeviceSynchronize());
  {
    const vt_status st = ensure_accum(ctx, scene, &p);
    if (st != VT_OK) return st;
  }
  std::vector<double> sums(rgb, rgb + want);
  for (double &v : sums) v *= (double)samples;
  VT_CUDA(ctx, cudaMemcpy(scene->d_accum, sums.data(), want * sizeof(double), cudaMemcpyHostToDevice));
  scene->samples = samples;
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

// ---- the reference's device known answers (regression_checks, tests/GPUChecks.swift:14-37) ------
// One thread evaluates the device functions on the reference's own inputs; the host compares.
//   out[0]     power_heuristic(1e-10, 1e-10) (expected 0.5)
//   out[1..3]  emission_weight(false, true, false, 0.2, 1), (true, true, true, 0, 1),
//              (false, false, false, 0.2, 1) (expected 0, 1, 1)
//   out[4]     the second PCG draw from seed 890625759 (expected exactly 0)
//   out[5]     dot(n, sample_cosine_hemisphere(n, seed 890625759)) for the grazing normal
//              normalize(0.31456656, 0, -0.9492354) (expected > 1e-4: above the tangent plane)
//   out[6..7]  min and max of rand_f over 100,000 draws from seed 17 (expected in [0, 1))
//   out[8..10] scattering_limit of depths 0, 1 and 8 (main.swift:3471-3473; expected 0, 0, 7)
namespace {
__global__ void k_known_answers(float *out, const float4 *glassParams) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  out[0] = power_heuristic(1e-10f, 1e-10f);
  out[1] = emission_weight(false, true, false, 0.2f, 1.0f);
  out[2] = emission_weight(true, true, true, 0.0f, 1.0f);
  out[3] = emission_weight(false, false, false, 0.2f, 1.0f);
  uint32_t g = 890625759u;
  const float r0 = pcg_rand(g), r1 = pcg_rand(g);
  out[4] = r1;
  const float3 n = normalize3(f3(0.31456656f, 0.0f, -0.9492354f));
  out[5] = dot3(n, cosine_hemisphere(n, r0, r1));
  uint32_t s = 17u;
  float lo = 1.0f, hi = 0.0f;
  for (int i = 0; i < 100000; ++i) {
    const float v = pcg_rand(s);
    lo = fminf(lo, v);
    hi = fmaxf(hi, v);
  }
  out[6] = lo;
  out[7] = hi;
  const uint32_t depths[3] = {0u, 1u, 8u};
  for (int k = 0; k < 3; ++k) out[8 + k] = float(max(0, (int)depths[k] - 1));
  // Glass (IOR 1.52, white) met from inside at normal (0, 0, -1) by normalize(0.9, 0, 0.435): total
  // internal reflection, so the sample exists, goes to z < 0 and weighs exactly 1 (the shading normal
  // is the geometric one, as the reference's Material without a geometric normal gives).
  RenderArgs A = {};
  A.pbr = glassParams;
  A.nmat = 1u;
  vt_material glass;
  glass.type = VT_MAT_DIELECTRIC;
  glass.albedo[0] = glass.albedo[1] = glass.albedo[2] = 1.0f;
  glass.emission[0] = glass.emission[1] = glass.emission[2] = 0.0f;
  glass.pad = __uint_as_float(0u);
  Sampler seed = {};
  seed.state = s;
  Lanes L = {};
  const float3 nn = f3(0.0f, 0.0f, -1.0f);
  float3 dir = f3(0.0f, 0.0f, 0.0f);
  float4 w = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const bool ok = sample_delta(A, L, glass, nn, nn, normalize3(f3(0.9f, 0.0f, 0.435f)), false, seed, dir, w);
  out[11] = ok ? 1.0f : 0.0f;
  out[12] = dir.z;
  out[13] = w.x;
  out[14] = w.y;
  out[15] = w.z;
}
}  // namespace

extern "C" vt_status vt_known_answers(vt_ctx *ctx, float *out, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!out || n < VT_KNOWN_ANSWERS) return vt_fail(ctx, VT_ERR_INVALID, "out must hold VT_KNOWN_ANSWERS floats");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  // The answers, then the glass slot's parameters (roughness, metalness, IOR 1.52, 0; no film).
  float *d = nullptr;
  VT_CUDA(ctx, cudaMalloc(&d, (VT_KNOWN_ANSWERS + 8) * sizeof(float)));
  const float glass[8] = {0.0f, 0.0f, 1.52f, 0.0f, 0.0f, 0.0f, 1.4f, 0.0f};
  float4 *dGlass = reinterpret_cast<float4 *>(d + ((VT_KNOWN_ANSWERS + 3u) & ~3u));
  cudaError_t e = cudaMemsetAsync(d, 0xff, VT_KNOWN_ANSWERS * sizeof(float), ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dGlass, glass, sizeof glass, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    k_known_answers<<<1, 32, 0, ctx->stream>>>(d, dGlass);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, VT_KNOWN_ANSWERS * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  if (e != cudaSuccess) return vt_cuda_fail(ctx, e, "vt_known_answers");
  return VT_OK;
}
