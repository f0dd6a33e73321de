// traverse.cu — closest-hit and any-hit traversal of the 4-wide BVH with the watertight
// triangle test.
//
// Reference: blas_closest / blas_any (main.swift:1788-1838), wide_ray / wide_node_hit /
// wide_order (main.swift:1758-1785), watertight_ray / watertight_edge / intersect_mesh_triangle
// (main.swift:1536-1582).
//
// Layout: a node is the reference's 128-byte MeshWideNode, fetched as eight 16-byte vector loads
// through the read-only path; a triangle is three float4 in BVH order (vertex a carries the input
// face index in .w), 48 bytes fetched as three 16-byte loads. The whole structure of a 1M-triangle
// mesh (~40 MB nodes + 48 MB triangles) sits in the 126 MB L2.
//
// The watertight arithmetic is written with explicitly rounded intrinsics in one fixed order
// (each product and sum rounded on its own; the exact FMA fallback on edge ties), which the CPU
// oracle reproduces, so hits compare bit for bit.
#include "vt_internal.cuh"

namespace {

constexpr int kStack = 96;  // 1 + 3 (depth - 1) entries for depth <= 32

struct Node4 {
  float4 lox, loy, loz, hix, hiy, hiz;
  int4 child, count;
};

__device__ __forceinline__ void load_node(const float4 *__restrict__ nodes, int i, Node4 &n) {
  const float4 *p = nodes + 8 * (size_t)i;
  n.lox = __ldg(p + 0); n.loy = __ldg(p + 1); n.loz = __ldg(p + 2);
  n.hix = __ldg(p + 3); n.hiy = __ldg(p + 4); n.hiz = __ldg(p + 5);
  n.child = __ldg(reinterpret_cast<const int4 *>(p + 6));
  n.count = __ldg(reinterpret_cast<const int4 *>(p + 7));
}

__device__ __forceinline__ float f4(const float4 &v, int k) {
  return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}
__device__ __forceinline__ int i4(const int4 &v, int k) {
  return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}
__device__ __forceinline__ float comp3(float x, float y, float z, int k) {
  return k == 0 ? x : (k == 1 ? y : z);
}

// Watertight ray (main.swift:1536-1551): permutation (kx, ky, kz), shear Sx, Sy and scale Sz.
struct WRay {
  float ox, oy, oz;
  int kx, ky, kz;
  float Sx, Sy, Sz;
};

__device__ __forceinline__ WRay make_wray(float ox, float oy, float oz, float dx, float dy, float dz) {
  WRay w;
  float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
  int kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  int kx = kz == 2 ? 0 : kz + 1, ky = kx == 2 ? 0 : kx + 1;
  float dkz = comp3(dx, dy, dz, kz);
  if (dkz < 0.0f) { int s = kx; kx = ky; ky = s; }
  w.kx = kx; w.ky = ky; w.kz = kz;
  w.Sx = __fdiv_rn(comp3(dx, dy, dz, kx), dkz);
  w.Sy = __fdiv_rn(comp3(dx, dy, dz, ky), dkz);
  w.Sz = __fdiv_rn(1.0f, dkz);
  w.ox = ox; w.oy = oy; w.oz = oz;
  return w;
}

// p.x q.y - p.y q.x with each product rounded on its own; on a tie the exact rounding errors
// decide (main.swift:1557-1562).
__device__ __forceinline__ float edge_fn(float px, float py, float qx, float qy) {
  float x = __fmul_rn(px, qy), y = __fmul_rn(py, qx), e = __fsub_rn(x, y);
  if (e == 0.0f) e = __fsub_rn(__fmaf_rn(px, qy, -x), __fmaf_rn(py, qx, -y));
  return e;
}

// Two-sided hit in [tMin, tMax) (main.swift:1564-1579).
__device__ __forceinline__ bool intersect_tri(const WRay &r, float4 a, float4 b, float4 c, float tMin,
                                              float tMax, float &t, float &b1, float &b2) {
  float A[3] = {__fsub_rn(a.x, r.ox), __fsub_rn(a.y, r.oy), __fsub_rn(a.z, r.oz)};
  float B[3] = {__fsub_rn(b.x, r.ox), __fsub_rn(b.y, r.oy), __fsub_rn(b.z, r.oz)};
  float C[3] = {__fsub_rn(c.x, r.ox), __fsub_rn(c.y, r.oy), __fsub_rn(c.z, r.oz)};
  const float Akz = A[r.kz], Bkz = B[r.kz], Ckz = C[r.kz];
  const float ax = __fsub_rn(A[r.kx], __fmul_rn(r.Sx, Akz)), ay = __fsub_rn(A[r.ky], __fmul_rn(r.Sy, Akz));
  const float bx = __fsub_rn(B[r.kx], __fmul_rn(r.Sx, Bkz)), by = __fsub_rn(B[r.ky], __fmul_rn(r.Sy, Bkz));
  const float cx = __fsub_rn(C[r.kx], __fmul_rn(r.Sx, Ckz)), cy = __fsub_rn(C[r.ky], __fmul_rn(r.Sy, Ckz));
  const float U = edge_fn(cx, cy, bx, by), V = edge_fn(ax, ay, cx, cy);
  if ((U < 0.0f && V > 0.0f) || (U > 0.0f && V < 0.0f)) return false;
  const float W = edge_fn(bx, by, ax, ay);
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  const float det = __fadd_rn(__fadd_rn(U, V), W);
  if (det == 0.0f) return false;
  const float az = __fmul_rn(r.Sz, Akz), bz = __fmul_rn(r.Sz, Bkz), cz = __fmul_rn(r.Sz, Ckz);
  const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, az), __fmul_rn(V, bz)), __fmul_rn(W, cz));
  const float inv = __fdiv_rn(1.0f, det);
  t = __fmul_rn(T, inv);
  b1 = __fmul_rn(V, inv);
  b2 = __fmul_rn(W, inv);
  return t >= tMin && t < tMax;
}

// Conservative slab ray (wide_ray, main.swift:1758-1763): origins shifted by the per-ray bound
// e = 2^-23 (max|o| + rootMax) so traversal never culls a triangle the edge test would hit.
struct SlabRay {
  float lowx, lowy, lowz, highx, highy, highz, invx, invy, invz;
  bool px, py, pz;
};

__device__ __forceinline__ SlabRay make_slab(float ox, float oy, float oz, float dx, float dy, float dz,
                                             float rootMax) {
  SlabRay s;
  float om = fmaxf(fmaxf(fabsf(ox), fabsf(oy)), fabsf(oz));
  // Explicitly rounded (no contraction into an FMA) so the oracle reproduces the culling.
  float e = __fmul_rn(1.1920929e-6f, __fadd_rn(om, rootMax));
  s.lowx = __fadd_rn(ox, e); s.lowy = __fadd_rn(oy, e); s.lowz = __fadd_rn(oz, e);
  s.highx = __fsub_rn(ox, e); s.highy = __fsub_rn(oy, e); s.highz = __fsub_rn(oz, e);
  s.px = fabsf(dx) < 1e-8f; s.py = fabsf(dy) < 1e-8f; s.pz = fabsf(dz) < 1e-8f;
  s.invx = __fdiv_rn(1.0f, s.px ? 1.0f : dx);
  s.invy = __fdiv_rn(1.0f, s.py ? 1.0f : dy);
  s.invz = __fdiv_rn(1.0f, s.pz ? 1.0f : dz);
  return s;
}

// wide_node_hit (main.swift:1764-1779): child hit mask and entry distances.
__device__ __forceinline__ int node_hits(const Node4 &n, const SlabRay &w, float tMin, float tMax,
                                         float nearT[4]) {
  int mask = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float ax = __fmul_rn(__fsub_rn(f4(n.lox, k), w.lowx), w.invx), bx = __fmul_rn(__fsub_rn(f4(n.hix, k), w.highx), w.invx);
    float ay = __fmul_rn(__fsub_rn(f4(n.loy, k), w.lowy), w.invy), by = __fmul_rn(__fsub_rn(f4(n.hiy, k), w.highy), w.invy);
    float az = __fmul_rn(__fsub_rn(f4(n.loz, k), w.lowz), w.invz), bz = __fmul_rn(__fsub_rn(f4(n.hiz, k), w.highz), w.invz);
    float lx = w.px ? -1e30f : fminf(ax, bx), hx = w.px ? 1e30f : fmaxf(ax, bx);
    float ly = w.py ? -1e30f : fminf(ay, by), hy = w.py ? 1e30f : fmaxf(ay, by);
    float lz = w.pz ? -1e30f : fminf(az, bz), hz = w.pz ? 1e30f : fmaxf(az, bz);
    float nt = fmaxf(fmaxf(lx, ly), fmaxf(lz, tMin));
    float ft = fminf(fminf(hx, hy), fminf(hz, tMax));
    bool hit = nt <= ft && i4(n.child, k) != 0;
    if (w.px) hit = hit && !(w.lowx < f4(n.lox, k) || w.highx > f4(n.hix, k));
    if (w.py) hit = hit && !(w.lowy < f4(n.loy, k) || w.highy > f4(n.hiy, k));
    if (w.pz) hit = hit && !(w.lowz < f4(n.loz, k) || w.highz > f4(n.hiz, k));
    nearT[k] = nt;
    mask |= hit ? (1 << k) : 0;
  }
  return mask;
}

template <bool kCount>
__device__ __forceinline__ bool trace_closest(const float4 *__restrict__ nodes,
                                              const float4 *__restrict__ tris, float rootMax,
                                              float4 r0, float4 r1, float &best, float &hb1,
                                              float &hb2, int &prim, uint32_t &nv, uint32_t &nt) {
  const WRay wr = make_wray(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z);
  const SlabRay sr = make_slab(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z, rootMax);
  const float tMin = r0.w;
  float closest = r1.w;
  bool found = false;
  int stack[kStack];
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    Node4 nd;
    load_node(nodes, stack[--top], nd);
    if (kCount) ++nv;
    float nearT[4];
    const int mask = node_hits(nd, sr, tMin, closest, nearT);
    // Near-to-far insertion sort of the hit children (wide_order, main.swift:1780-1785).
    int order[4];
    float key[4];
    int m = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!(mask >> k & 1)) continue;
      int j = m++;
      while (j > 0 && key[j - 1] > nearT[k]) { key[j] = key[j - 1]; order[j] = order[j - 1]; --j; }
      key[j] = nearT[k];
      order[j] = k;
    }
    for (int j = 0; j < m; ++j) {
      const int k = order[j];
      const int c = i4(nd.child, k);
      if (c > 0 || key[j] > closest) continue;
      const int first = -c - 1, cnt = i4(nd.count, k);
      for (int q = 0; q < cnt; ++q) {
        const float4 *tp = tris + 3 * (size_t)(first + q);
        const float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
        float t, b1, b2;
        if (kCount) ++nt;
        if (!intersect_tri(wr, a, b, cc, tMin, closest, t, b1, b2)) continue;
        closest = t; hb1 = b1; hb2 = b2; prim = __float_as_int(a.w); found = true;
      }
    }
    for (int j = m - 1; j >= 0; --j) {
      const int k = order[j];
      const int c = i4(nd.child, k);
      if (c > 0 && key[j] <= closest && top < kStack) stack[top++] = c;
    }
  }
  best = closest;
  return found;
}

template <bool kCount>
__device__ __forceinline__ bool trace_any(const float4 *__restrict__ nodes,
                                          const float4 *__restrict__ tris, float rootMax, float4 r0,
                                          float4 r1, uint32_t &nv, uint32_t &nt) {
  const WRay wr = make_wray(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z);
  const SlabRay sr = make_slab(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z, rootMax);
  const float tMin = r0.w, tMax = r1.w;
  int stack[kStack];
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    Node4 nd;
    load_node(nodes, stack[--top], nd);
    if (kCount) ++nv;
    float nearT[4];
    const int mask = node_hits(nd, sr, tMin, tMax, nearT);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!(mask >> k & 1)) continue;
      const int c = i4(nd.child, k);
      if (c > 0) { if (top < kStack) stack[top++] = c; continue; }
      const int first = -c - 1, cnt = i4(nd.count, k);
      for (int q = 0; q < cnt; ++q) {
        const float4 *tp = tris + 3 * (size_t)(first + q);
        const float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
        float t, b1, b2;
        if (kCount) ++nt;
        if (intersect_tri(wr, a, b, cc, tMin, tMax, t, b1, b2)) return true;
      }
    }
  }
  return false;
}

__global__ void __launch_bounds__(128) k_closest(const float4 *__restrict__ nodes,
                                                  const float4 *__restrict__ tris, float rootMax,
                                                  const float4 *__restrict__ rays, uint32_t n,
                                                  int4 *__restrict__ hits) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 r0 = __ldg(rays + 2 * (size_t)i), r1 = __ldg(rays + 2 * (size_t)i + 1);
  float t = 0.0f, b1 = 0.0f, b2 = 0.0f;
  int prim = -1;
  uint32_t nv = 0, nt = 0;
  int4 out = make_int4(0, 0, 0, -1);
  if (trace_closest<false>(nodes, tris, rootMax, r0, r1, t, b1, b2, prim, nv, nt))
    out = make_int4(__float_as_int(t), __float_as_int(b1), __float_as_int(b2), prim);
  hits[i] = out;
}

__global__ void __launch_bounds__(128) k_any(const float4 *__restrict__ nodes,
                                              const float4 *__restrict__ tris, float rootMax,
                                              const float4 *__restrict__ rays, uint32_t n,
                                              uint8_t *__restrict__ occ) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 r0 = __ldg(rays + 2 * (size_t)i), r1 = __ldg(rays + 2 * (size_t)i + 1);
  uint32_t nv = 0, nt = 0;
  occ[i] = trace_any<false>(nodes, tris, rootMax, r0, r1, nv, nt) ? 1 : 0;
}

__global__ void __launch_bounds__(128) k_count(const float4 *__restrict__ nodes,
                                                const float4 *__restrict__ tris, float rootMax,
                                                const float4 *__restrict__ rays, uint32_t n,
                                                int closest, unsigned long long *acc) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t nv = 0, nt = 0;
  if (i < n) {
    const float4 r0 = __ldg(rays + 2 * (size_t)i), r1 = __ldg(rays + 2 * (size_t)i + 1);
    if (closest) {
      float t, b1, b2;
      int prim;
      trace_closest<true>(nodes, tris, rootMax, r0, r1, t, b1, b2, prim, nv, nt);
    } else {
      trace_any<true>(nodes, tris, rootMax, r0, r1, nv, nt);
    }
  }
  unsigned long long a = nv, b = nt;
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(acc, a);
    atomicAdd(acc + 1, b);
  }
}

}  // namespace

void vt_launch_closest(const vt_mesh *mesh, const vt_ray *rays, uint32_t n, vt_hit *hits,
                       int sm_count, cudaStream_t s) {
  (void)sm_count;
  if (n == 0) return;
  k_closest<<<(n + 127) / 128, 128, 0, s>>>(reinterpret_cast<const float4 *>(mesh->d_nodes), mesh->d_tris,
                                           mesh->root_max, reinterpret_cast<const float4 *>(rays), n,
                                           reinterpret_cast<int4 *>(hits));
}

void vt_launch_any(const vt_mesh *mesh, const vt_ray *rays, uint32_t n, uint8_t *occ, int sm_count,
                   cudaStream_t s) {
  (void)sm_count;
  if (n == 0) return;
  k_any<<<(n + 127) / 128, 128, 0, s>>>(reinterpret_cast<const float4 *>(mesh->d_nodes), mesh->d_tris,
                                       mesh->root_max, reinterpret_cast<const float4 *>(rays), n, occ);
}

void vt_launch_count(const vt_mesh *mesh, const vt_ray *rays, uint32_t n, int closest,
                     unsigned long long *acc, cudaStream_t s) {
  if (n == 0) return;
  k_count<<<(n + 127) / 128, 128, 0, s>>>(reinterpret_cast<const float4 *>(mesh->d_nodes), mesh->d_tris,
                                         mesh->root_max, reinterpret_cast<const float4 *>(rays), n,
                                         closest, acc);
}
