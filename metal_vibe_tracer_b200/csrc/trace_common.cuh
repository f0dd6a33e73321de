// trace_common.cuh — device building blocks shared by the traversal kernels and the integrator:
// the 4-wide node fetch, the watertight ray/triangle test (main.swift:1536-1582), the conservative
// slab test (main.swift:1758-1779) and the near-to-far child order (main.swift:1780-1785).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace vtd {

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

// Children of a node in near-to-far order, in registers. A 4-element sorting network on
// (entry distance, slot) gives exactly the order of the reference's stable insertion sort
// (wide_order, main.swift:1780-1785), since slots break distance ties; missed children sort last.
struct Sorted4 {
  float key[4];
  int child[4], count[4];
  int m;  // number of hit children (the first m entries)
};
__device__ __forceinline__ void cswap(float &ka, int &sa, int &ca, int &na, float &kb, int &sb, int &cb, int &nb) {
  const bool sw = ka > kb || (ka == kb && sa > sb);
  const float k = sw ? kb : ka; kb = sw ? ka : kb; ka = k;
  const int sl = sw ? sb : sa; sb = sw ? sa : sb; sa = sl;
  const int c = sw ? cb : ca; cb = sw ? ca : cb; ca = c;
  const int n = sw ? nb : na; nb = sw ? na : nb; na = n;
}
__device__ __forceinline__ Sorted4 sort_children(const Node4 &nd, int mask, const float nearT[4]) {
  Sorted4 o;
  float k0 = (mask & 1) ? nearT[0] : __int_as_float(0x7f800000), k1 = (mask & 2) ? nearT[1] : __int_as_float(0x7f800000);
  float k2 = (mask & 4) ? nearT[2] : __int_as_float(0x7f800000), k3 = (mask & 8) ? nearT[3] : __int_as_float(0x7f800000);
  int s0 = (mask & 1) ? 0 : 4, s1 = (mask & 2) ? 1 : 5, s2 = (mask & 4) ? 2 : 6, s3 = (mask & 8) ? 3 : 7;
  int c0 = nd.child.x, c1 = nd.child.y, c2 = nd.child.z, c3 = nd.child.w;
  int n0 = nd.count.x, n1 = nd.count.y, n2 = nd.count.z, n3 = nd.count.w;
  cswap(k0, s0, c0, n0, k1, s1, c1, n1);
  cswap(k2, s2, c2, n2, k3, s3, c3, n3);
  cswap(k0, s0, c0, n0, k2, s2, c2, n2);
  cswap(k1, s1, c1, n1, k3, s3, c3, n3);
  cswap(k1, s1, c1, n1, k2, s2, c2, n2);
  o.key[0] = k0; o.key[1] = k1; o.key[2] = k2; o.key[3] = k3;
  o.child[0] = c0; o.child[1] = c1; o.child[2] = c2; o.child[3] = c3;
  o.count[0] = n0; o.count[1] = n1; o.count[2] = n2; o.count[3] = n3;
  o.m = __popc(mask);
  return o;
}

}  // namespace vtd
