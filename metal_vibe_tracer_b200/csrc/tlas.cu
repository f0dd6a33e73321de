// tlas.cu — the two-level hierarchy: a 4-wide TLAS over instances of meshes, each instance tracing
// its mesh's own hierarchy (the BLAS) in object space.
//
// Reference: MeshLayout.addInstance and MeshSceneLayout.sceneBlob (Sources/Acceleration.swift:474-573)
// build the instance records, the world boxes and the TLAS (a WideBVH of leaf size 1 whose leaves name
// instances); mesh_closest / mesh_occluded (main.swift:1840-1984) traverse it, growing the TLAS boxes per
// ray by lo.w (max|origin| + hi.w) and tracing each instance with instance_ray (main.swift:1634-1637).
//
// B200 layout: the TLAS is built by the same GPU LBVH as a mesh, over one degenerate triangle per
// instance whose box is the instance's world box (vertices lo, hi and (lo.x, hi.y, lo.z)); its leaf
// children are then rewritten to name the instance, as the reference does. Instance records (128 B) and
// a table of the meshes' node and triangle arrays sit in HBM; a 1024-instance TLAS is ~45 KB and stays
// in L1/L2. The traversal is one thread per ray: the TLAS with the reference's 128-byte nodes and a
// 32-entry stack, and per instance the quantised single-ray BLAS traversal of traverse.cu, so an
// instance's object-space hits equal vt_trace_closest's on the same object-space ray.
//
// The ray transform is written with explicitly rounded operations in one fixed order (the oracle
// repeats it): o'_r = ((l_r.x o.x + l_r.y o.y) + l_r.z o.z) + l_r.w with the products and sums fused as
// fma(l.z, o.z, fma(l.y, o.y, l.x * o.x)) + l.w, d'_r = fma(l.z, d.z, fma(l.y, d.y, l.x * d.x)).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "trace_common.cuh"
#include "vt_internal.cuh"

namespace {
using namespace vtd;

constexpr int kTlasStack = 32;  // mesh_closest's TLAS stack (main.swift:1887)
constexpr int kTlasBlock = 128;

struct TlasInst {  // vt_instance_record on the device
  float4 world[3];
  float4 local[3];
  uint4 range;  // mesh, slot base, rendered base, mirrored
  float4 bound;
};
static_assert(sizeof(TlasInst) == sizeof(vt_instance_record), "instance record layout");

struct TlasMesh {
  const float4 *qnodes;
  const float4 *tris;
  const float4 *nrm;
  const int32_t *order;
  uint32_t faces;
  float rootMax;
  uint32_t pad[2];
};

__device__ __forceinline__ float xform_point(float4 l, float x, float y, float z) {
  return __fadd_rn(__fmaf_rn(l.z, z, __fmaf_rn(l.y, y, __fmul_rn(l.x, x))), l.w);
}
__device__ __forceinline__ float xform_dir(float4 l, float x, float y, float z) {
  return __fmaf_rn(l.z, z, __fmaf_rn(l.y, y, __fmul_rn(l.x, x)));
}

// mesh_closest (kAny = false) / mesh_occluded (kAny = true), one thread per ray.
template <bool kAny>
__global__ void __launch_bounds__(kTlasBlock) k_tlas_trace(const float4 *__restrict__ nodes, const TlasInst *__restrict__ inst,
                                                          const TlasMesh *__restrict__ meshes, float grow, float reach,
                                                          const float4 *__restrict__ rays, uint32_t n, int4 *__restrict__ hits,
                                                          uint32_t *__restrict__ instOut, uint8_t *__restrict__ occ) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 r0 = __ldcs(rays + 2 * (size_t)i), r1 = __ldcs(rays + 2 * (size_t)i + 1);
  const float e = __fmul_rn(grow, __fadd_rn(max_abs_origin(r0.x, r0.y, r0.z), reach));
  const SlabRay sr = make_slab_e(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z, e);
  const float tMin = r0.w;
  float closest = r1.w, hb1 = 0.0f, hb2 = 0.0f;
  int prim = -1;
  uint32_t hitInst = 0xffffffffu;
  uint32_t nv = 0, nt = 0;
  int stack[kTlasStack];
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    Node4 nd;
    load_node(nodes, stack[--top], nd);
    float nearT[4];
    const int mask = node_hits(nd, sr, tMin, closest, nearT);
    if (kAny) {
      // mesh_occluded: children in slot order, inner nodes pushed as met, instances traced as met.
      for (int k = 0; k < 4; ++k) {
        if (!(mask >> k & 1)) continue;
        const int c = i4(nd.child, k);
        if (c > 0) {
          if (top < kTlasStack) stack[top++] = c;
          continue;
        }
        const TlasInst I = inst[-c - 1];
        const TlasMesh M = meshes[I.range.x];
        const float4 o = make_float4(xform_point(I.local[0], r0.x, r0.y, r0.z), xform_point(I.local[1], r0.x, r0.y, r0.z),
                                     xform_point(I.local[2], r0.x, r0.y, r0.z), tMin);
        const float4 d = make_float4(xform_dir(I.local[0], r1.x, r1.y, r1.z), xform_dir(I.local[1], r1.x, r1.y, r1.z),
                                     xform_dir(I.local[2], r1.x, r1.y, r1.z), r1.w);
        if (trace_any<false>(M.qnodes, M.tris, I.bound.z, o, d, nv, nt)) {
          occ[i] = 1;
          return;
        }
      }
      continue;
    }
    // mesh_closest: instances near to far, then inner children pushed far to near.
    const Sorted4 s = sort_children(nd, mask, nearT);
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
      if (j >= s.m || s.child[j] > 0 || beyond(s.key[j], closest)) continue;
      const uint32_t k = (uint32_t)(-s.child[j] - 1);
      const TlasInst I = inst[k];
      const TlasMesh M = meshes[I.range.x];
      const float4 o = make_float4(xform_point(I.local[0], r0.x, r0.y, r0.z), xform_point(I.local[1], r0.x, r0.y, r0.z),
                                   xform_point(I.local[2], r0.x, r0.y, r0.z), tMin);
      const float4 d = make_float4(xform_dir(I.local[0], r1.x, r1.y, r1.z), xform_dir(I.local[1], r1.x, r1.y, r1.z),
                                   xform_dir(I.local[2], r1.x, r1.y, r1.z), closest);
      float t, b1, b2;
      int p = -1;
      if (trace_closest<false>(M.qnodes, M.tris, I.bound.z, o, d, t, b1, b2, p, nv, nt)) {
        closest = t;
        hb1 = b1;
        hb2 = b2;
        prim = p;
        hitInst = k;
      }
    }
#pragma unroll
    for (int j = 3; j >= 0; --j)
      if (j < s.m && s.child[j] > 0 && !beyond(s.key[j], closest) && top < kTlasStack) stack[top++] = s.child[j];
  }
  if (kAny) {
    occ[i] = 0;
    return;
  }
  hits[i] = prim >= 0 ? make_int4(__float_as_int(closest), __float_as_int(hb1), __float_as_int(hb2), prim)
                      : make_int4(0, 0, 0, -1);
  if (instOut) instOut[i] = prim >= 0 ? hitInst : 0xffffffffu;
}

// The TLAS leaves name instances: child -(first + 1) at BVH position `first` becomes -(order[first] + 1)
// (sceneBlob, Sources/Acceleration.swift:530-535).
__global__ void k_tlas_leaves(vt_wide_node *nodes, uint32_t count, const int32_t *order) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  for (int k = 0; k < 4; ++k) {
    const int c = nodes[i].child[k];
    if (c < 0) nodes[i].child[k] = -(order[-c - 1] + 1);
  }
}

// One instance's triangles in world space (instance_triangle, main.swift:1645-1668): per BVH position
// of its mesh, the input face f becomes rendered face base + f with its three vertices transformed,
// the normals by the inverse transpose (normalised; a zero normal stays zero: the mesh then shades
// with geometric normals), the tag offset by the slot base and b, c swapped when mirrored.
__global__ void k_tlas_flatten(const TlasInst *__restrict__ inst, uint32_t instance, TlasMesh M, vt_face *__restrict__ faces,
                               vt_vertex *__restrict__ verts) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= M.faces) return;
  const TlasInst I = inst[instance];
  const uint32_t f = (uint32_t)__ldg(M.order + p);
  const size_t out = (size_t)I.range.z + f;
  const float4 *tp = M.tris + 3 * (size_t)p;
  const float4 *np = M.nrm ? M.nrm + 3 * (size_t)p : nullptr;
  const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const uint32_t tag = __float_as_uint(__ldg(tp + 1).w) + I.range.y;
  const bool mirrored = I.range.w != 0u;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int src = k == 0 ? 0 : (mirrored ? 3 - k : k);  // b and c swap places when mirrored
    const float4 a = __ldg(tp + src), nk = np ? __ldg(np + src) : zero;
    vt_vertex w;
    w.px = xform_point(I.world[0], a.x, a.y, a.z);
    w.py = xform_point(I.world[1], a.x, a.y, a.z);
    w.pz = xform_point(I.world[2], a.x, a.y, a.z);
    // Inverse transpose: sum over rows r of local[r].xyz * n[r].
    float nx = __fmaf_rn(I.local[2].x, nk.z, __fmaf_rn(I.local[1].x, nk.y, __fmul_rn(I.local[0].x, nk.x)));
    float ny = __fmaf_rn(I.local[2].y, nk.z, __fmaf_rn(I.local[1].y, nk.y, __fmul_rn(I.local[0].y, nk.x)));
    float nz = __fmaf_rn(I.local[2].z, nk.z, __fmaf_rn(I.local[1].z, nk.y, __fmul_rn(I.local[0].z, nk.x)));
    const float l2 = nx * nx + ny * ny + nz * nz;
    if (l2 > 1e-12f) {
      const float sc = rsqrtf(l2);
      nx *= sc; ny *= sc; nz *= sc;
    } else {
      nx = ny = nz = 0.0f;
    }
    w.nx = nx; w.ny = ny; w.nz = nz;
    w.u = 0.0f; w.v = 0.0f;
    verts[3 * out + k] = w;
  }
  faces[out] = vt_face{(uint32_t)(3 * out), (uint32_t)(3 * out + 1), (uint32_t)(3 * out + 2), tag};
}

double norm_inf(const double m[3][3]) {
  double r = 0.0;
  for (int i = 0; i < 3; ++i) r = std::max(r, std::fabs(m[i][0]) + std::fabs(m[i][1]) + std::fabs(m[i][2]));
  return r;
}

}  // namespace

struct vt_tlas {
  std::vector<const vt_mesh *> meshes;
  std::vector<vt_instance_record> records;
  vt_mesh *boxes = nullptr;  // the LBVH over the instance boxes (leaves rewritten to name instances)
  TlasInst *d_inst = nullptr;
  TlasMesh *d_meshes = nullptr;
  uint64_t rendered = 0;
  float grow = 0.0f, reach = 0.0f;
  float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  float build_ms = 0.0f;
};

static void free_tlas(vt_tlas *t) {
  if (!t) return;
  if (t->boxes) vt_mesh_destroy(nullptr, t->boxes);
  cudaFree(t->d_inst);
  cudaFree(t->d_meshes);
  delete t;
}

vt_status vt_tlas_build(vt_ctx *ctx, const vt_mesh *const *meshes, uint32_t nmeshes, const vt_instance *instances,
                        uint32_t ninstances, vt_tlas **out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!out) return vt_fail(ctx, VT_ERR_INVALID, "out is null");
  *out = nullptr;
  if (ninstances == 0) return vt_fail(ctx, VT_ERR_INVALID, "a TLAS needs at least one instance");
  if (!instances || !meshes || nmeshes == 0) return vt_fail(ctx, VT_ERR_INVALID, "meshes or instances is null");
  if (ninstances > (1u << 24)) return vt_fail(ctx, VT_ERR_LIMIT, "more than 2^24 instances");
  for (uint32_t k = 0; k < nmeshes; ++k)
    if (!meshes[k] || meshes[k]->nfaces == 0) return vt_fail(ctx, VT_ERR_INVALID, "mesh " + std::to_string(k) + " is null or empty");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  vt_tlas *t = new vt_tlas();
  t->meshes.assign(meshes, meshes + nmeshes);
  t->records.resize(ninstances);
  std::vector<vt_face> bf(ninstances);
  std::vector<vt_vertex> bv(3 * (size_t)ninstances);
  double condition = 0.0, reach = 0.0;
  float glo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, ghi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  uint64_t rendered = 0;
  // First pass: validation, inverses, reach and condition (the TLAS box margin needs the reach of
  // the instance itself; the per-ray growth the largest values over all instances).
  std::vector<double> reachOf(ninstances);
  for (uint32_t i = 0; i < ninstances; ++i) {
    const vt_instance &in = instances[i];
    if (in.mesh >= nmeshes) {
      free_tlas(t);
      return vt_fail(ctx, VT_ERR_INVALID, "instance " + std::to_string(i) + " names mesh " + std::to_string(in.mesh) + " of " + std::to_string(nmeshes));
    }
    double m[3][3], tr[3];
    bool finite = true;
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c) {
        m[r][c] = in.world[4 * r + c];
        finite = finite && std::isfinite(m[r][c]);
      }
      tr[r] = in.world[4 * r + 3];
      finite = finite && std::isfinite(tr[r]);
    }
    const double scale = std::sqrt(m[0][0] * m[0][0] + m[1][0] * m[1][0] + m[2][0] * m[2][0]);
    if (!finite || !(scale >= 1e-6 && scale <= 1e6)) {
      free_tlas(t);
      return vt_fail(ctx, VT_ERR_INVALID, "Combined hierarchy scale exceeds the supported range. (instance " + std::to_string(i) + ")");
    }
    const double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                       m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    if (!std::isfinite(det) || !(std::fabs(det) > 1e-18)) {
      free_tlas(t);
      return vt_fail(ctx, VT_ERR_INVALID, "Singular USD transform. (instance " + std::to_string(i) + ")");
    }
    double inv[3][3];
    inv[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) / det;
    inv[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) / det;
    inv[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) / det;
    inv[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) / det;
    inv[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) / det;
    inv[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) / det;
    inv[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) / det;
    inv[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) / det;
    inv[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) / det;
    const vt_mesh *mesh = meshes[in.mesh];
    const double n = norm_inf(m);
    const double tmax = std::max(std::fabs(tr[0]), std::max(std::fabs(tr[1]), std::fabs(tr[2])));
    reachOf[i] = tmax + n * (double)mesh->root_max;
    if (!(reachOf[i] < 1e8)) {
      free_tlas(t);
      return vt_fail(ctx, VT_ERR_INVALID, "Hierarchy transform exceeds the supported scene extent. (instance " + std::to_string(i) + ")");
    }
    condition = std::max(condition, n * norm_inf(inv));
    reach = std::max(reach, reachOf[i]);
    vt_instance_record &R = t->records[i];
    std::memset(&R, 0, sizeof R);
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 4; ++c) R.world[4 * r + c] = in.world[4 * r + c];
      // local = [inv | -inv t]
      for (int c = 0; c < 3; ++c) R.local[4 * r + c] = (float)inv[r][c];
      R.local[4 * r + 3] = (float)-(inv[r][0] * tr[0] + inv[r][1] * tr[1] + inv[r][2] * tr[2]);
    }
    R.mesh = in.mesh;
    R.slot_base = in.slot_base;
    R.rendered_base = (uint32_t)rendered;
    R.mirrored = det < 0.0 ? 1u : 0u;
    R.bound[0] = (float)tmax;
    R.bound[1] = (float)n;
    R.bound[2] = mesh->root_max;
    rendered += mesh->nfaces;
    if (rendered > (1ull << 32) - 1) {
      free_tlas(t);
      return vt_fail(ctx, VT_ERR_LIMIT, "more than 2^32 - 1 rendered triangles");
    }
    // World box: the mesh box's eight corners transformed (in double, rounded outward), enlarged by
    // 2^-20 of the instance's reach (addInstance, Sources/Acceleration.swift:501-508).
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int k = 0; k < 8; ++k) {
      const double p[3] = {(k & 1) ? mesh->hi[0] : mesh->lo[0], (k & 2) ? mesh->hi[1] : mesh->lo[1], (k & 4) ? mesh->hi[2] : mesh->lo[2]};
      for (int r = 0; r < 3; ++r) {
        const double v = m[r][0] * p[0] + m[r][1] * p[1] + m[r][2] * p[2] + tr[r];
        lo[r] = std::min(lo[r], std::nextafter((float)v, -FLT_MAX));
        hi[r] = std::max(hi[r], std::nextafter((float)v, FLT_MAX));
      }
    }
    const float margin = (float)(std::ldexp(1.0, -20) * reachOf[i]);
    for (int r = 0; r < 3; ++r) {
      lo[r] -= margin;
      hi[r] += margin;
      glo[r] = std::min(glo[r], lo[r]);
      ghi[r] = std::max(ghi[r], hi[r]);
    }
    bv[3 * (size_t)i] = vt_vertex{lo[0], lo[1], lo[2], 0, 0, 0, 0, 0};
    bv[3 * (size_t)i + 1] = vt_vertex{hi[0], hi[1], hi[2], 0, 0, 0, 0, 0};
    bv[3 * (size_t)i + 2] = vt_vertex{lo[0], hi[1], lo[2], 0, 0, 0, 0, 0};
    bf[i] = vt_face{3 * i, 3 * i + 1, 3 * i + 2, 0};
  }
  t->rendered = rendered;
  t->grow = (float)(std::ldexp(1.0, -18) * (1.0 + condition));
  t->reach = (float)reach;
  for (int r = 0; r < 3; ++r) { t->lo[r] = glo[r]; t->hi[r] = ghi[r]; }

  vt_build_options o{};
  o.leaf_size = 1;
  vt_status st = vt_mesh_build(ctx, bf.data(), ninstances, bv.data(), 3 * ninstances, &o, &t->boxes);
  if (st != VT_OK) {
    free_tlas(t);
    return st;
  }
  t->build_ms = t->boxes->build_ms;
  cudaStream_t s = ctx->stream;
  std::vector<TlasMesh> hm(nmeshes);
  for (uint32_t k = 0; k < nmeshes; ++k) {
    const vt_mesh *mk = meshes[k];
    hm[k] = TlasMesh{reinterpret_cast<const float4 *>(mk->d_qnodes), mk->d_tris, mk->d_nrm, mk->d_order, mk->nfaces, mk->root_max, {0, 0}};
  }
  cudaError_t e = cudaMalloc(&t->d_inst, ninstances * sizeof(TlasInst));
  if (e == cudaSuccess) e = cudaMalloc(&t->d_meshes, nmeshes * sizeof(TlasMesh));
  if (e == cudaSuccess) e = cudaMemcpyAsync(t->d_inst, t->records.data(), ninstances * sizeof(TlasInst), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(t->d_meshes, hm.data(), nmeshes * sizeof(TlasMesh), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    k_tlas_leaves<<<(t->boxes->nnodes + 127) / 128, 128, 0, s>>>(t->boxes->d_nodes, t->boxes->nnodes, t->boxes->d_order);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    free_tlas(t);
    return vt_cuda_fail(ctx, e, "vt_tlas_build");
  }
  *out = t;
  return VT_OK;
}

vt_status vt_tlas_destroy(vt_ctx *ctx, vt_tlas *tlas) {
  if (ctx) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
  }
  free_tlas(tlas);
  return VT_OK;
}

vt_status vt_tlas_get_info(vt_ctx *ctx, const vt_tlas *tlas, vt_tlas_info *out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!tlas || !out) return vt_fail(ctx, VT_ERR_INVALID, "tlas or out is null");
  std::memset(out, 0, sizeof *out);
  out->instances = (uint32_t)tlas->records.size();
  out->meshes = (uint32_t)tlas->meshes.size();
  out->nodes = tlas->boxes->nnodes;
  out->depth = tlas->boxes->depth;
  out->rendered_triangles = tlas->rendered;
  for (int r = 0; r < 3; ++r) { out->lo[r] = tlas->lo[r]; out->hi[r] = tlas->hi[r]; }
  out->grow = tlas->grow;
  out->reach = tlas->reach;
  out->build_ms = tlas->build_ms;
  return VT_OK;
}

vt_status vt_tlas_get_nodes(vt_ctx *ctx, const vt_tlas *tlas, vt_wide_node *nodes, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!tlas || (n && !nodes)) return vt_fail(ctx, VT_ERR_INVALID, "tlas or nodes is null");
  if (n != tlas->boxes->nnodes) return vt_fail(ctx, VT_ERR_INVALID, "n must equal the TLAS node count");
  VT_CUDA(ctx, cudaMemcpy(nodes, tlas->boxes->d_nodes, n * sizeof(vt_wide_node), cudaMemcpyDeviceToHost));
  return VT_OK;
}

vt_status vt_tlas_get_instances(vt_ctx *ctx, const vt_tlas *tlas, vt_instance_record *records, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!tlas || (n && !records)) return vt_fail(ctx, VT_ERR_INVALID, "tlas or records is null");
  if (n != tlas->records.size()) return vt_fail(ctx, VT_ERR_INVALID, "n must equal the instance count");
  std::memcpy(records, tlas->records.data(), n * sizeof(vt_instance_record));
  return VT_OK;
}

static vt_status tlas_trace(vt_ctx *ctx, const vt_tlas *tlas, const vt_ray *rays, uint32_t n, void *out, uint32_t *instOut,
                            bool closest, cudaStream_t s) {
  if (!ctx) return VT_ERR_INVALID;
  if (!tlas || (n && (!rays || !out))) return vt_fail(ctx, VT_ERR_INVALID, "tlas, rays or output is null");
  if ((reinterpret_cast<uintptr_t>(rays) & 15u) || (closest && (reinterpret_cast<uintptr_t>(out) & 15u)))
    return vt_fail(ctx, VT_ERR_INVALID, "rays and hits must be 16-byte aligned");
  if (n == 0) return VT_OK;
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  const uint32_t grid = (n + kTlasBlock - 1) / kTlasBlock;
  const float4 *nodes = reinterpret_cast<const float4 *>(tlas->boxes->d_nodes);
  if (closest)
    k_tlas_trace<false><<<grid, kTlasBlock, 0, s>>>(nodes, tlas->d_inst, tlas->d_meshes, tlas->grow, tlas->reach,
                                                   reinterpret_cast<const float4 *>(rays), n, static_cast<int4 *>(out), instOut,
                                                   nullptr);
  else
    k_tlas_trace<true><<<grid, kTlasBlock, 0, s>>>(nodes, tlas->d_inst, tlas->d_meshes, tlas->grow, tlas->reach,
                                                  reinterpret_cast<const float4 *>(rays), n, nullptr, nullptr,
                                                  static_cast<uint8_t *>(out));
  VT_CUDA(ctx, cudaGetLastError());
  return VT_OK;
}

vt_status vt_tlas_trace_closest(vt_ctx *ctx, const vt_tlas *tlas, const vt_ray *rays_dev, uint32_t n, vt_hit *hits_dev,
                                uint32_t *instances_dev, void *stream) {
  return tlas_trace(ctx, tlas, rays_dev, n, hits_dev, instances_dev, true, static_cast<cudaStream_t>(stream));
}

vt_status vt_tlas_trace_any(vt_ctx *ctx, const vt_tlas *tlas, const vt_ray *rays_dev, uint32_t n, uint8_t *occluded_dev,
                            void *stream) {
  return tlas_trace(ctx, tlas, rays_dev, n, occluded_dev, nullptr, false, static_cast<cudaStream_t>(stream));
}

vt_status vt_tlas_flatten(vt_ctx *ctx, const vt_tlas *tlas, const vt_build_options *opts, vt_mesh **out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!tlas || !out) return vt_fail(ctx, VT_ERR_INVALID, "tlas or out is null");
  *out = nullptr;
  if (tlas->rendered > (1u << 30)) return vt_fail(ctx, VT_ERR_LIMIT, "more than 2^30 rendered triangles");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  const uint32_t nf = (uint32_t)tlas->rendered;
  vt_face *df = nullptr;
  vt_vertex *dv = nullptr;
  VT_CUDA(ctx, cudaMalloc(&df, (size_t)nf * sizeof(vt_face)));
  cudaError_t e = cudaMalloc(&dv, 3 * (size_t)nf * sizeof(vt_vertex));
  if (e != cudaSuccess) {
    cudaFree(df);
    return vt_cuda_fail(ctx, e, "cudaMalloc(flattened vertices)");
  }
  cudaStream_t s = ctx->stream;
  for (uint32_t i = 0; i < tlas->records.size(); ++i) {
    const vt_mesh *mk = tlas->meshes[tlas->records[i].mesh];
    const TlasMesh M{reinterpret_cast<const float4 *>(mk->d_qnodes), mk->d_tris, mk->d_nrm, mk->d_order, mk->nfaces, mk->root_max, {0, 0}};
    k_tlas_flatten<<<(mk->nfaces + 255) / 256, 256, 0, s>>>(tlas->d_inst, i, M, df, dv);
  }
  e = cudaGetLastError();
  vt_status st = e == cudaSuccess ? vt_mesh_build_device(ctx, df, nf, dv, 3 * nf, opts, out) : vt_cuda_fail(ctx, e, "k_tlas_flatten");
  cudaStreamSynchronize(s);
  cudaFree(df);
  cudaFree(dv);
  return st;
}
