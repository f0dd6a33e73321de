// trace_common.cuh — device building blocks shared by the traversal kernels and the integrator:
// the 4-wide node fetch, the watertight ray/triangle test (main.swift:1536-1582), the conservative
// slab test (main.swift:1758-1779) and the near-to-far child order (main.swift:1780-1785).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace vtd {

constexpr int kStack = 100;  // 1 + 3 depth entries for depth <= 33 (leaf children are stack entries)

struct Node4 {
  float4 lox, loy, loz, hix, hiy, hiz;
  int4 child, count;
};

#ifndef VT_NODE_LD256
#define VT_NODE_LD256 1
#endif
// A node is fetched through the read-only path as four 32-byte vector loads (sm_100 ld.global.v8;
// nodes are 128-byte records in a 256-byte aligned buffer): half the load instructions, and so half
// the L1 wavefronts, of eight 16-byte loads when the lanes of a warp fetch different nodes.
// The asm is volatile so that the compiler cannot speculate the load above the branch that guards
// it: a traversal pops leaf entries (negative) and node indices from one stack, and a load hoisted
// above the entry's sign test would read before the start of the node array.
__device__ __forceinline__ void ld256(const float4 *p, float4 &a, float4 &b) {
#if VT_NODE_LD256
  asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
               : "l"(p));
#else
  a = __ldg(p);
  b = __ldg(p + 1);
#endif
}
__device__ __forceinline__ void load_node(const float4 *__restrict__ nodes, int i, Node4 &n) {
  const float4 *p = nodes + 8 * (size_t)i;
  float4 c, d;
  ld256(p + 0, n.lox, n.loy);
  ld256(p + 2, n.loz, n.hix);
  ld256(p + 4, n.hiy, n.hiz);
  ld256(p + 6, c, d);
  n.child = make_int4(__float_as_int(c.x), __float_as_int(c.y), __float_as_int(c.z), __float_as_int(c.w));
  n.count = make_int4(__float_as_int(d.x), __float_as_int(d.y), __float_as_int(d.z), __float_as_int(d.w));
}

// Three-operand max / min (sm_100's max.f32 / min.f32 with three sources): one instruction where two
// fmaxf / fminf would take two. Exact (the result is one of the inputs), NaN-free inputs here.
__device__ __forceinline__ float fmax3(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float fmin3(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
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

// Two-sided hit in [tMin, tMax) (main.swift:1564-1579). The ray's permuted coordinates are picked
// with selects (comp3), so the test keeps every value in registers. The shear of each vertex,
// A[kx] - Sx A[kz], is one fused multiply-add (a single rounding), and so is each step of the
// numerator T; the edge functions keep the reference's separately rounded products with the exact
// fallback on ties (main.swift:1557-1562). The CPU oracle uses the same operations (std::fma), so
// hits compare bit for bit. Each vertex is transformed on its own, from the vertex and the ray only,
// so an edge shared by two triangles gets the same edge-function value in both: the test stays
// watertight.
__device__ __forceinline__ bool intersect_tri(const WRay &r, float4 a, float4 b, float4 c, float tMin,
                                              float tMax, float &t, float &b1, float &b2) {
  const float A0 = __fsub_rn(a.x, r.ox), A1 = __fsub_rn(a.y, r.oy), A2 = __fsub_rn(a.z, r.oz);
  const float B0 = __fsub_rn(b.x, r.ox), B1 = __fsub_rn(b.y, r.oy), B2 = __fsub_rn(b.z, r.oz);
  const float C0 = __fsub_rn(c.x, r.ox), C1 = __fsub_rn(c.y, r.oy), C2 = __fsub_rn(c.z, r.oz);
  const float Akz = comp3(A0, A1, A2, r.kz), Bkz = comp3(B0, B1, B2, r.kz), Ckz = comp3(C0, C1, C2, r.kz);
  const float nSx = -r.Sx, nSy = -r.Sy;
  const float ax = __fmaf_rn(nSx, Akz, comp3(A0, A1, A2, r.kx)), ay = __fmaf_rn(nSy, Akz, comp3(A0, A1, A2, r.ky));
  const float bx = __fmaf_rn(nSx, Bkz, comp3(B0, B1, B2, r.kx)), by = __fmaf_rn(nSy, Bkz, comp3(B0, B1, B2, r.ky));
  const float cx = __fmaf_rn(nSx, Ckz, comp3(C0, C1, C2, r.kx)), cy = __fmaf_rn(nSy, Ckz, comp3(C0, C1, C2, r.ky));
  const float U = edge_fn(cx, cy, bx, by), V = edge_fn(ax, ay, cx, cy);
  if ((U < 0.0f && V > 0.0f) || (U > 0.0f && V < 0.0f)) return false;
  const float W = edge_fn(bx, by, ax, ay);
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  const float det = __fadd_rn(__fadd_rn(U, V), W);
  if (det == 0.0f) return false;
  const float az = __fmul_rn(r.Sz, Akz), bz = __fmul_rn(r.Sz, Bkz), cz = __fmul_rn(r.Sz, Ckz);
  const float T = __fmaf_rn(W, cz, __fmaf_rn(V, bz, __fmul_rn(U, az)));
  const float inv = __fdiv_rn(1.0f, det);
  t = __fmul_rn(T, inv);
  b1 = __fmul_rn(V, inv);
  b2 = __fmul_rn(W, inv);
  return t >= tMin && t < tMax;
}

// mesh_hit_error (main.swift:1353-1355) of a triangle: its vertices' rounding bound. Shadow rays of
// imported scenes end this far before each triangle's own endpoint (scene_occluded's slack,
// main.swift:2066-2069), so the surface a light sample lies on does not occlude itself.
__device__ __forceinline__ float tri_error_bound(float4 a, float4 b, float4 c) {
  const float ma = fmaxf(fabsf(a.x), fmaxf(fabsf(a.y), fabsf(a.z)));
  const float mb = fmaxf(fabsf(b.x), fmaxf(fabsf(b.y), fabsf(b.z)));
  const float mc = fmaxf(fabsf(c.x), fmaxf(fabsf(c.y), fabsf(c.z)));
  return fmaxf(1e-7f, 1.907349e-6f * fmaxf(ma, fmaxf(mb, mc)));
}

// Conservative slab ray (wide_ray, main.swift:1758-1763): origins shifted by the per-ray bound
// e = 2^-23 (max|o| + rootMax) so traversal never culls a triangle the edge test would hit. An axis
// the ray runs parallel to (|d| < 1e-8) gets the inverse +-1e30 instead of the reference's separate
// inside-slab test: the slab distances are then -huge/+huge inside the shifted slab and cull outside
// it (the same decisions except where the origin lies exactly on a shifted face, where this form
// keeps the child), so the per-child test needs no parallel-axis branches.
struct SlabRay {
  float lowx, lowy, lowz, highx, highy, highz, invx, invy, invz;
};

__device__ __forceinline__ float slab_inverse(float d) {
  return fabsf(d) < 1e-8f ? copysignf(1e30f, d) : __fdiv_rn(1.0f, d);
}

// The slab ray with a given origin shift e.
__device__ __forceinline__ SlabRay make_slab_e(float ox, float oy, float oz, float dx, float dy, float dz, float e) {
  SlabRay s;
  s.lowx = __fadd_rn(ox, e); s.lowy = __fadd_rn(oy, e); s.lowz = __fadd_rn(oz, e);
  s.highx = __fsub_rn(ox, e); s.highy = __fsub_rn(oy, e); s.highz = __fsub_rn(oz, e);
  s.invx = slab_inverse(dx);
  s.invy = slab_inverse(dy);
  s.invz = slab_inverse(dz);
  return s;
}

__device__ __forceinline__ float max_abs_origin(float ox, float oy, float oz) {
  return fmaxf(fmaxf(fabsf(ox), fabsf(oy)), fabsf(oz));
}

__device__ __forceinline__ SlabRay make_slab(float ox, float oy, float oz, float dx, float dy, float dz,
                                             float rootMax) {
  // Explicitly rounded (no contraction into an FMA) so the oracle reproduces the culling.
  const float e = __fmul_rn(1.1920929e-6f, __fadd_rn(max_abs_origin(ox, oy, oz), rootMax));
  return make_slab_e(ox, oy, oz, dx, dy, dz, e);
}

// wide_node_hit (main.swift:1764-1779): child hit mask and entry distances.
__device__ __forceinline__ int node_hits(const Node4 &n, const SlabRay &w, float tMin, float tMax,
                                         float nearT[4]) {
  int mask = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float ax = __fmul_rn(__fsub_rn(f4(n.lox, k), w.lowx), w.invx), bx = __fmul_rn(__fsub_rn(f4(n.hix, k), w.highx), w.invx);
    const float ay = __fmul_rn(__fsub_rn(f4(n.loy, k), w.lowy), w.invy), by = __fmul_rn(__fsub_rn(f4(n.hiy, k), w.highy), w.invy);
    const float az = __fmul_rn(__fsub_rn(f4(n.loz, k), w.lowz), w.invz), bz = __fmul_rn(__fsub_rn(f4(n.hiz, k), w.highz), w.invz);
    const float nt = fmax3(fminf(ax, bx), fminf(ay, by), fmaxf(fminf(az, bz), tMin));
    const float ft = fmin3(fmaxf(ax, bx), fmaxf(ay, by), fminf(fmaxf(az, bz), tMax));
    nearT[k] = nt;
    mask |= (nt <= ft && i4(n.child, k) != 0) ? (1 << k) : 0;
  }
  return mask;
}

// Order-preserving map of a float to an unsigned integer.
__device__ __forceinline__ uint32_t ord32(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Hit children near to far, in registers. Each hit child gets the key (ord32(entry + 0), so -0 and +0
// agree, with its two low bits replaced by the slot): a 5-comparator network of unsigned min/max sorts them by entry distance
// with slots breaking ties (the reference's stable insertion sort, wide_order, main.swift:1780-1785,
// up to entry distances equal in all but their two lowest bits); missed children sort last. A child
// is culled against the closest hit when (key & ~3) > ord32(closest), i.e. only when its entry
// distance is certainly beyond it.
struct Sorted4 {
  uint32_t key[4];
  int child[4], count[4];
  int m;  // number of hit children (the first m entries)
};
__device__ __forceinline__ void ucswap(uint32_t &a, uint32_t &b) {
  const uint32_t lo = min(a, b), hi = max(a, b);
  a = lo; b = hi;
}
__device__ __forceinline__ int pick4(const int4 &v, uint32_t slot) {
  const int lo = (slot & 1u) ? v.y : v.x, hi = (slot & 1u) ? v.w : v.z;
  return (slot & 2u) ? hi : lo;
}
__device__ __forceinline__ Sorted4 sort_children(const Node4 &nd, int mask, const float nearT[4]) {
  uint32_t k[4];
#pragma unroll
  for (int c = 0; c < 4; ++c)
    k[c] = (mask >> c & 1) ? ((ord32(__fadd_rn(nearT[c], 0.0f)) & ~3u) | (uint32_t)c) : 0xffffffffu;
  ucswap(k[0], k[1]);
  ucswap(k[2], k[3]);
  ucswap(k[0], k[2]);
  ucswap(k[1], k[3]);
  ucswap(k[1], k[2]);
  Sorted4 o;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    o.key[j] = k[j];
    o.child[j] = pick4(nd.child, k[j] & 3u);
    o.count[j] = pick4(nd.count, k[j] & 3u);
  }
  o.m = __popc(mask);
  return o;
}
// Whether sorted entry j lies certainly beyond the closest hit.
__device__ __forceinline__ bool beyond(uint32_t key, float closest) {
  return (key & ~3u) > ord32(__fadd_rn(closest, 0.0f));
}

// ---- quantised nodes (qnode.cu): conservative decoding ---------------------------------------
// A child's near distance on an axis is a lower bound, and its far distance an upper bound, of the
// exact distances to the decoded planes p + q 2^e, which enclose the child's box: every product
// and sum is rounded toward the safe side (FFMA.RM / FFMA.RP), so the test never culls a child the
// reference's slab test (on the exact box, origin shifted by e) keeps. Per ray: the inverse
// direction, and per axis the slab origins of the near and far planes times the inverse, rounded
// up and down respectively.
struct QRay {
  float invx, invy, invz;
  float nx, ny, nz;  // round-up (near-plane origin) * inv
  float fx, fy, fz;  // round-down (far-plane origin) * inv
  uint32_t neg;      // bit a: the ray runs toward decreasing coordinates on axis a
};

__device__ __forceinline__ QRay make_qray(float ox, float oy, float oz, float dx, float dy, float dz, float rootMax) {
  const SlabRay sr = make_slab(ox, oy, oz, dx, dy, dz, rootMax);
  QRay q;
  q.invx = sr.invx; q.invy = sr.invy; q.invz = sr.invz;
  const bool nx = sr.invx < 0.0f, ny = sr.invy < 0.0f, nz = sr.invz < 0.0f;
  q.neg = (nx ? 1u : 0u) | (ny ? 2u : 0u) | (nz ? 4u : 0u);
  // The lo plane pairs with the origin shifted by +e (low), the hi plane with -e (high).
  q.nx = __fmul_ru(nx ? sr.highx : sr.lowx, sr.invx);
  q.ny = __fmul_ru(ny ? sr.highy : sr.lowy, sr.invy);
  q.nz = __fmul_ru(nz ? sr.highz : sr.lowz, sr.invz);
  q.fx = __fmul_rd(nx ? sr.lowx : sr.highx, sr.invx);
  q.fy = __fmul_rd(ny ? sr.lowy : sr.highy, sr.invy);
  q.fz = __fmul_rd(nz ? sr.lowz : sr.highz, sr.invz);
  return q;
}

struct QNode {
  float px, py, pz;
  uint32_t e;
  uint32_t qlo[3], qhi[3];
  int4 child;
  uint32_t counts;
};

__device__ __forceinline__ void load_qnode(const float4 *__restrict__ qnodes, int i, QNode &n) {
  const float4 *p = qnodes + 4 * (size_t)i;
  float4 a, b, c, d;
  ld256(p, a, b);
  ld256(p + 2, c, d);
  n.px = a.x; n.py = a.y; n.pz = a.z; n.e = __float_as_uint(a.w);
  n.qlo[0] = __float_as_uint(b.x); n.qlo[1] = __float_as_uint(b.y); n.qlo[2] = __float_as_uint(b.z);
  n.qhi[0] = __float_as_uint(b.w); n.qhi[1] = __float_as_uint(c.x); n.qhi[2] = __float_as_uint(c.y);
  n.child = make_int4(__float_as_int(c.z), __float_as_int(c.w), __float_as_int(d.x), __float_as_int(d.y));
  n.counts = __float_as_uint(d.z);
}

// A leaf child goes on a traversal stack as the entry ~(node << 2 | slot) (node indices are below
// 2^29); popping it reads the slot's first triangle and count from the node, in L1 since the node's
// visit.
__device__ __forceinline__ int leaf_entry_of(int node, int slot) { return ~((node << 2) | slot); }
__device__ __forceinline__ void leaf_range(const float4 *__restrict__ qnodes, int entry, int &first, int &cnt) {
  const int code = ~entry, slot = code & 3;
  const int *nd = reinterpret_cast<const int *>(qnodes + 4 * (size_t)(code >> 2));
  first = -__ldg(nd + 10 + slot) - 1;
  cnt = (__ldg(nd + 14) >> (4 * slot)) & 15;
}

// Byte k of w as the float 1 + byte 2^-15 (the byte in mantissa bits 8-15), exact.
__device__ __forceinline__ float qbyte(uint32_t w, int k) {
  return __uint_as_float(__byte_perm(w, 0x3F800000u, 0x7604u | ((uint32_t)k << 4)));
}

struct QAxis {
  float d, cn, cf;   // 2^15 step * inv; near and far offsets minus that (the byte's bias)
  uint32_t nw, fw;   // near-plane and far-plane bytes
};

// A plane at p + q 2^e lies at (1 + q 2^-15) d + (p * inv - origin * inv - d) with d = 2^(e+15) inv;
// the bias removal rounds to the safe side too, so the bound loosens by at most 2^-9 of a step.
__device__ __forceinline__ QAxis q_axis(float p, uint32_t eb, uint32_t qlo, uint32_t qhi, float inv, float nO, float fO,
                                        bool neg) {
  QAxis a;
  a.d = __uint_as_float((eb + 15u) << 23) * inv;  // 2^(e+15) * inv, exact
  a.cn = __fadd_rd(__fmaf_rd(p, inv, -nO), -a.d);
  a.cf = __fadd_ru(__fmaf_ru(p, inv, -fO), -a.d);
  a.nw = neg ? qhi : qlo;
  a.fw = neg ? qlo : qhi;
  return a;
}

// Child hit mask and entry distances of a quantised node.
__device__ __forceinline__ int qnode_hits(const QNode &n, const QRay &r, float tMin, float tMax, float nearT[4]) {
  const QAxis x = q_axis(n.px, n.e & 0xffu, n.qlo[0], n.qhi[0], r.invx, r.nx, r.fx, (r.neg & 1u) != 0u);
  const QAxis y = q_axis(n.py, (n.e >> 8) & 0xffu, n.qlo[1], n.qhi[1], r.invy, r.ny, r.fy, (r.neg & 2u) != 0u);
  const QAxis z = q_axis(n.pz, (n.e >> 16) & 0xffu, n.qlo[2], n.qhi[2], r.invz, r.nz, r.fz, (r.neg & 4u) != 0u);
  int mask = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float nxk = __fmaf_rd(qbyte(x.nw, k), x.d, x.cn), fxk = __fmaf_ru(qbyte(x.fw, k), x.d, x.cf);
    const float nyk = __fmaf_rd(qbyte(y.nw, k), y.d, y.cn), fyk = __fmaf_ru(qbyte(y.fw, k), y.d, y.cf);
    const float nzk = __fmaf_rd(qbyte(z.nw, k), z.d, z.cn), fzk = __fmaf_ru(qbyte(z.fw, k), z.d, z.cf);
    const float nt = fmaxf(fmax3(nxk, nyk, nzk), tMin);
    const float ft = fminf(fmin3(fxk, fyk, fzk), tMax);
    nearT[k] = nt;
    mask |= (nt <= ft && i4(n.child, k) != 0) ? (1 << k) : 0;
  }
  return mask;
}

// Hit children of a quantised node near to far (the packed-key network of sort_children).
__device__ __forceinline__ Sorted4 sort_qchildren(const QNode &nd, int mask, const float nearT[4]) {
  uint32_t k[4];
#pragma unroll
  for (int c = 0; c < 4; ++c)
    k[c] = (mask >> c & 1) ? ((ord32(__fadd_rn(nearT[c], 0.0f)) & ~3u) | (uint32_t)c) : 0xffffffffu;
  ucswap(k[0], k[1]);
  ucswap(k[2], k[3]);
  ucswap(k[0], k[2]);
  ucswap(k[1], k[3]);
  ucswap(k[1], k[2]);
  Sorted4 o;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    o.key[j] = k[j];
    o.child[j] = pick4(nd.child, k[j] & 3u);
    o.count[j] = (int)((nd.counts >> (4u * (k[j] & 3u))) & 15u);
  }
  o.m = __popc(mask);
  return o;
}

// ---- single-ray traversals ------------------------------------------------------------------------
// In the persistent kernels' order (leaf children pushed as stack entries, near entries popped first),
// counting node visits and triangle tests when kCount. `r0` is (origin, tmin), `r1` (direction, tmax);
// the closest hit reports the input face index (vertex a's .w).

template <bool kCount>
__device__ __forceinline__ bool trace_closest(const float4 *__restrict__ nodes,
                                              const float4 *__restrict__ tris, float rootMax,
                                              float4 r0, float4 r1, float &best, float &hb1,
                                              float &hb2, int &prim, uint32_t &nv, uint32_t &nt) {
  const WRay wr = make_wray(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z);
  const QRay qr = make_qray(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z, rootMax);
  const float tMin = r0.w;
  float closest = r1.w;
  bool found = false;
  int stack[kStack];
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    const int entry = stack[--top];
    if (entry < 0) {
      int first, cnt;
      leaf_range(nodes, entry, first, cnt);
      for (int q = 0; q < cnt; ++q) {
        const float4 *tp = tris + 3 * (size_t)(first + q);
        const float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
        float t, b1, b2;
        if (kCount) ++nt;
        if (!intersect_tri(wr, a, b, cc, tMin, closest, t, b1, b2)) continue;
        closest = t; hb1 = b1; hb2 = b2; prim = __float_as_int(a.w); found = true;
      }
      continue;
    }
    QNode nd;
    load_qnode(nodes, entry, nd);
    if (kCount) ++nv;
    float nearT[4];
    const int mask = qnode_hits(nd, qr, tMin, closest, nearT);
    const Sorted4 o = sort_qchildren(nd, mask, nearT);
#pragma unroll
    for (int j = 3; j >= 0; --j) {
      if (j >= o.m || beyond(o.key[j], closest) || top >= kStack) continue;
      stack[top++] = o.child[j] > 0 ? o.child[j] : leaf_entry_of(entry, (int)(o.key[j] & 3u));
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
  const QRay qr = make_qray(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z, rootMax);
  const float tMin = r0.w, tMax = r1.w;
  int stack[kStack];
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    const int entry = stack[--top];
    if (entry < 0) {
      int first, cnt;
      leaf_range(nodes, entry, first, cnt);
      for (int q = 0; q < cnt; ++q) {
        const float4 *tp = tris + 3 * (size_t)(first + q);
        const float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
        float t, b1, b2;
        if (kCount) ++nt;
        if (intersect_tri(wr, a, b, cc, tMin, tMax, t, b1, b2)) return true;
      }
      continue;
    }
    QNode nd;
    load_qnode(nodes, entry, nd);
    if (kCount) ++nv;
    float nearT[4];
    const int mask = qnode_hits(nd, qr, tMin, tMax, nearT);
#pragma unroll
    for (int k = 3; k >= 0; --k) {
      if (!(mask >> k & 1) || top >= kStack) continue;
      const int c = i4(nd.child, k);
      stack[top++] = c > 0 ? c : leaf_entry_of(entry, k);
    }
  }
  return false;
}

}  // namespace vtd
