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
#include <algorithm>

#include "trace_common.cuh"
#include "vt_internal.cuh"

namespace {
using namespace vtd;

// ---- persistent traversal -----------------------------------------------------------------------
// Rays vary a lot in length (65 node visits on average for the incoherent set, with a long tail), so
// a thread-per-ray grid leaves most lanes of a warp idle while its longest ray finishes.
// Persistent traversal (k_closest, k_any): each warp stays resident and refills idle lanes from a
// global ray counter: one warp-aggregated atomicAdd hands out as many rays as there are idle lanes,
// whenever at least kRefill lanes are idle. Each loop iteration handles one stack entry per active
// lane (a node visit or a leaf's triangles) with the per-ray order of trace_closest / trace_any, so
// the hits equal those of the single-ray form bit for bit. Rays are read and hits written with
// streaming cache hints so that the ray stream does not evict the BVH from L2.
#ifndef VT_TRACE_REFILL
#define VT_TRACE_REFILL 8
#endif
#ifndef VT_TRACE_MIN_BLOCKS
#define VT_TRACE_MIN_BLOCKS 6
#endif
constexpr unsigned kFull = 0xffffffffu;
constexpr int kRefill = VT_TRACE_REFILL;      // refill once this many lanes are idle
constexpr int kBlock = 128;
constexpr int kMinBlocks = VT_TRACE_MIN_BLOCKS;  // register budget: 65536 / (kBlock * kMinBlocks)

struct RayState {
  WRay wr;
  QRay qr;
  float tMin, tMax;
};

__device__ __forceinline__ void load_ray(const float4 *__restrict__ rays, uint32_t r, RayState &s,
                                         float rootMax) {
  const float4 r0 = __ldcs(rays + 2 * (size_t)r), r1 = __ldcs(rays + 2 * (size_t)r + 1);
  s.wr = make_wray(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z);
  s.qr = make_qray(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z, rootMax);
  s.tMin = r0.w;
  s.tMax = r1.w;
}

// Hands rays [base, base + idle lanes) to the idle lanes of the warp. Returns the lane's ray
// index, or n if it got none; *exhausted is set (warp-uniformly) once the pool is empty.
__device__ __forceinline__ uint32_t refill(unsigned idle, uint32_t *counter, uint32_t n, bool &exhausted) {
  const unsigned lane = threadIdx.x & 31u;
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(counter, (uint32_t)__popc(idle));
  base = __shfl_sync(kFull, base, 0);
  if (base + (uint32_t)__popc(idle) >= n) exhausted = true;
  const uint32_t r = base + (uint32_t)__popc(idle & ((1u << lane) - 1u));
  return (idle >> lane & 1u) && r < n ? r : n;
}

// The traversal stack lives in shared memory, one column per thread: entry d of thread t is
// word d * kBlock + t, so every lane of a warp hits its own bank whatever its stack depth.
__device__ __forceinline__ int *stack_slot(int *sstack, int d) { return sstack + d * kBlock + threadIdx.x; }

// Stack entries: an inner node is its index (>= 0); a leaf child is ~(node << 2 | slot).

// Per lane, one iteration handles the top stack entry: a node visit (its hit children, leaves
// included, pushed far to near, so they pop near first) or one leaf's triangle tests. The warp runs
// only the kind more of its lanes need this iteration; the others wait one iteration. A ray's own
// order (LIFO over its stack) does not depend on the warp.
// kPos: a hit reports the triangle's BVH position instead of its input face (the integrator's
// hit record). count: when not null, the queue length on the device (at most n).
template <bool kPos>
__global__ void __launch_bounds__(kBlock, kMinBlocks) k_closest(const float4 *__restrict__ nodes,
                                                        const float4 *__restrict__ tris, float rootMax,
                                                        const float4 *__restrict__ rays, uint32_t n,
                                                        int4 *__restrict__ hits, uint32_t *counter,
                                                        const uint32_t *__restrict__ perm, int stackSize,
                                                        uint32_t *status, const uint32_t *__restrict__ count) {
  extern __shared__ int sstack[];
  if (count) n = min(n, *count);
  int top = 0;  // 0: the lane holds no ray
  uint32_t rid = 0;
  RayState s;
  float closest = 0.0f, hb1 = 0.0f, hb2 = 0.0f;
  int prim = -1;
  bool exhausted = false;  // warp-uniform
  while (true) {
    const unsigned idle = __ballot_sync(kFull, top == 0);
    if (!exhausted && __popc(idle) >= kRefill) {
      const uint32_t r = refill(idle, counter, n, exhausted);
      if (r < n) {
        rid = perm ? __ldcs(perm + r) : r;
        load_ray(rays, rid, s, rootMax);
        closest = s.tMax;
        prim = -1;
        *stack_slot(sstack, 0) = 0;
        top = 1;
      }
    }
    if (exhausted && !__any_sync(kFull, top > 0)) break;
    const int entry = top > 0 ? *stack_slot(sstack, top - 1) : 0;
    const bool leaf = top > 0 && entry < 0;
    const unsigned leaves = __ballot_sync(kFull, leaf), inner = __ballot_sync(kFull, top > 0 && !leaf);
    const bool leafPhase = __popc(leaves) >= __popc(inner);
    if (top == 0 || leaf != leafPhase) continue;
    --top;
    if (leaf) {
      int first, cnt;
      leaf_range(nodes, entry, first, cnt);
      for (int q = 0; q < cnt; ++q) {
        const float4 *tp = tris + 3 * (size_t)(first + q);
        const float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
        float t, b1, b2;
        if (!intersect_tri(s.wr, a, b, cc, s.tMin, closest, t, b1, b2)) continue;
        closest = t; hb1 = b1; hb2 = b2; prim = kPos ? first + q : __float_as_int(a.w);
      }
    } else {
      QNode nd;
      load_qnode(nodes, entry, nd);
      float nearT[4];
      const int mask = qnode_hits(nd, s.qr, s.tMin, closest, nearT);
      const Sorted4 o = sort_qchildren(nd, mask, nearT);
#pragma unroll
      for (int j = 3; j >= 0; --j) {
        if (j >= o.m || beyond(o.key[j], closest)) continue;
        const int e = o.child[j] > 0 ? o.child[j] : leaf_entry_of(entry, (int)(o.key[j] & 3u));
        if (top < stackSize) *stack_slot(sstack, top++) = e;
        else atomicOr(status, (uint32_t)VT_DEV_STACK);
      }
    }
    if (top == 0) {
      const int4 out = prim >= 0 ? make_int4(__float_as_int(closest), __float_as_int(hb1), __float_as_int(hb2), prim)
                                 : make_int4(0, 0, 0, -1);
      __stcs(hits + rid, out);
    }
  }
}

// kSlack: each triangle's own rounding bound comes off tmax (the integrator's shadow rays in
// imported scenes, scene_occluded main.swift:2066-2069). count: as k_closest's.
template <bool kSlack>
__global__ void __launch_bounds__(kBlock, kMinBlocks) k_any(const float4 *__restrict__ nodes,
                                                    const float4 *__restrict__ tris, float rootMax,
                                                    const float4 *__restrict__ rays, uint32_t n,
                                                    uint8_t *__restrict__ occ, uint32_t *counter,
                                                    const uint32_t *__restrict__ perm, int stackSize,
                                                    uint32_t *status, const uint32_t *__restrict__ count) {
  extern __shared__ int sstack[];
  if (count) n = min(n, *count);
  int top = 0;
  uint32_t rid = 0;
  RayState s;
  bool exhausted = false;
  while (true) {
    const unsigned idle = __ballot_sync(kFull, top == 0);
    if (!exhausted && __popc(idle) >= kRefill) {
      const uint32_t r = refill(idle, counter, n, exhausted);
      if (r < n) {
        rid = perm ? __ldcs(perm + r) : r;
        load_ray(rays, rid, s, rootMax);
        *stack_slot(sstack, 0) = 0;
        top = 1;
      }
    }
    if (exhausted && !__any_sync(kFull, top > 0)) break;
    const int entry = top > 0 ? *stack_slot(sstack, top - 1) : 0;
    const bool leaf = top > 0 && entry < 0;
    const unsigned leaves = __ballot_sync(kFull, leaf), inner = __ballot_sync(kFull, top > 0 && !leaf);
    const bool leafPhase = __popc(leaves) >= __popc(inner);
    if (top == 0 || leaf != leafPhase) continue;
    --top;
    bool hit = false;
    if (leaf) {
      int first, cnt;
      leaf_range(nodes, entry, first, cnt);
      for (int q = 0; q < cnt; ++q) {
        const float4 *tp = tris + 3 * (size_t)(first + q);
        const float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
        float t, b1, b2;
        const float tMax = kSlack ? s.tMax - tri_error_bound(a, b, cc) : s.tMax;
        if (intersect_tri(s.wr, a, b, cc, s.tMin, tMax, t, b1, b2)) { hit = true; break; }
      }
    } else {
      QNode nd;
      load_qnode(nodes, entry, nd);
      float nearT[4];
      const int mask = qnode_hits(nd, s.qr, s.tMin, s.tMax, nearT);
#pragma unroll
      for (int k = 3; k >= 0; --k) {
        if (!(mask >> k & 1)) continue;
        const int c = i4(nd.child, k);
        const int e = c > 0 ? c : leaf_entry_of(entry, k);
        if (top < stackSize) *stack_slot(sstack, top++) = e;
        else atomicOr(status, (uint32_t)VT_DEV_STACK);
      }
    }
    if (hit) top = 0;
    if (top == 0) occ[rid] = hit ? 1 : 0;
  }
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

// ---- ray ordering ----------------------------------------------------------------------------------
// Large ray batches are traced in the order of a 30-bit key of origin and direction, so that the
// rays of a warp follow similar paths (fewer idle lanes at divergent branches, shared cache lines).
// The key is computed per ray, sorted with the LBVH's radix sort, and the persistent kernels read
// ray perm[q] at queue position q; results still go to each ray's own slot.
#ifndef VT_TRACE_SORT
#define VT_TRACE_SORT 0
#endif
constexpr uint32_t kSortMinRays = 1u << 20;

__device__ __forceinline__ uint32_t quant(float x, float lo, float inv, uint32_t bits) {
  float f = (x - lo) * inv;
  const float top = (float)((1u << bits) - 1u);
  f = fminf(fmaxf(f, 0.0f), top);
  return (uint32_t)f;
}
// Octahedral map of a unit direction to [0, 1]^2.
__device__ __forceinline__ float2 octahedral(float dx, float dy, float dz) {
  const float sum = fabsf(dx) + fabsf(dy) + fabsf(dz);
  float u = dx / sum, v = dy / sum;
  if (dz < 0.0f) {
    const float uu = (1.0f - fabsf(v)) * (u >= 0.0f ? 1.0f : -1.0f);
    const float vv = (1.0f - fabsf(u)) * (v >= 0.0f ? 1.0f : -1.0f);
    u = uu; v = vv;
  }
  return make_float2(u * 0.5f + 0.5f, v * 0.5f + 0.5f);
}

__global__ void k_ray_keys(const float4 *__restrict__ rays, uint32_t n, float3 lo, float3 inv,
                           uint32_t *__restrict__ keys, uint32_t *__restrict__ vals, int mode) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 r0 = __ldcs(rays + 2 * (size_t)i), r1 = __ldcs(rays + 2 * (size_t)i + 1);
  uint32_t key = 0;
  if (mode == 1 || mode == 2) {
    // Origin Morton code (10 bits per axis), or octant + 9 bits per axis.
    const uint32_t b = mode == 1 ? 10u : 9u;
    const float sc = (float)(1u << b);
    uint32_t q[3] = {quant(r0.x, lo.x, inv.x * sc, b), quant(r0.y, lo.y, inv.y * sc, b), quant(r0.z, lo.z, inv.z * sc, b)};
    for (uint32_t bit = 0; bit < b; ++bit)
      for (int a = 0; a < 3; ++a) key |= ((q[a] >> bit) & 1u) << (3 * bit + (2 - a));
    if (mode == 2) key |= ((r1.x < 0.0f ? 4u : 0u) | (r1.y < 0.0f ? 2u : 0u) | (r1.z < 0.0f ? 1u : 0u)) << 27;
  } else if (mode == 3) {
    // 5-D Morton code: 6 bits each of origin x, y, z and octahedral direction u, v.
    const float2 o = octahedral(r1.x, r1.y, r1.z);
    uint32_t q[5] = {quant(r0.x, lo.x, inv.x * 64.0f, 6), quant(r0.y, lo.y, inv.y * 64.0f, 6),
                     quant(r0.z, lo.z, inv.z * 64.0f, 6), quant(o.x, 0.0f, 64.0f, 6), quant(o.y, 0.0f, 64.0f, 6)};
    for (uint32_t bit = 0; bit < 6; ++bit)
      for (int a = 0; a < 5; ++a) key |= ((q[a] >> bit) & 1u) << (5 * bit + (4 - a));
  } else {
    // Direction major (5 + 5 octahedral bits), origin Morton minor (20 bits).
    const float2 o = octahedral(r1.x, r1.y, r1.z);
    const uint32_t du = quant(o.x, 0.0f, 32.0f, 5), dv = quant(o.y, 0.0f, 32.0f, 5);
    uint32_t q[3] = {quant(r0.x, lo.x, inv.x * 128.0f, 7), quant(r0.y, lo.y, inv.y * 128.0f, 7), quant(r0.z, lo.z, inv.z * 64.0f, 6)};
    uint32_t m = 0, pos = 0;
    for (uint32_t bit = 0; bit < 7; ++bit)
      for (int a = 0; a < 3; ++a)
        if (bit < (a == 2 ? 6u : 7u)) m |= ((q[a] >> bit) & 1u) << pos++;
    key = (du << 25) | (dv << 20) | m;
  }
  keys[i] = key;
  vals[i] = i;
}

namespace {
// Stack entries a traversal of a tree of `depth` levels needs: the root, then at most 3 net pushes
// per level below it (a visit pops one node and pushes up to four).
inline int stack_entries(uint32_t depth) { return 3 * (int)depth + 1; }

// Resident blocks per SM for a persistent kernel with `smem` bytes of dynamic shared memory.
template <typename K> int resident_blocks(K kernel, size_t smem) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kBlock, smem) != cudaSuccess || b < 1) b = 1;
  return b;
}

template <typename K> void prepare(K kernel, size_t smem) {
  if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}
}  // namespace

void vt_launch_closest(const vt_mesh *mesh, const vt_ray *rays, uint32_t n, vt_hit *hits, int sm_count,
                       uint32_t *counter, const uint32_t *perm, uint32_t *status, cudaStream_t s,
                       const uint32_t *count, bool bvhPos) {
  if (n == 0) return;
  const int S = stack_entries(mesh->depth);
  const size_t smem = (size_t)S * kBlock * sizeof(int);
  auto kernel = bvhPos ? k_closest<true> : k_closest<false>;
  prepare(kernel, smem);
  const uint32_t want = (n + kBlock - 1) / kBlock;
  const uint32_t grid = std::min<uint32_t>(want, (uint32_t)(resident_blocks(kernel, smem) * sm_count));
  cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
  kernel<<<grid, kBlock, smem, s>>>(reinterpret_cast<const float4 *>(mesh->d_qnodes), mesh->d_tris, mesh->root_max,
                                    reinterpret_cast<const float4 *>(rays), n, reinterpret_cast<int4 *>(hits), counter,
                                    perm, S, status, count);
}

void vt_launch_any(const vt_mesh *mesh, const vt_ray *rays, uint32_t n, uint8_t *occ, int sm_count,
                   uint32_t *counter, const uint32_t *perm, uint32_t *status, cudaStream_t s,
                   const uint32_t *count, bool slack) {
  if (n == 0) return;
  const int S = stack_entries(mesh->depth);
  const size_t smem = (size_t)S * kBlock * sizeof(int);
  auto kernel = slack ? k_any<true> : k_any<false>;
  prepare(kernel, smem);
  const uint32_t want = (n + kBlock - 1) / kBlock;
  const uint32_t grid = std::min<uint32_t>(want, (uint32_t)(resident_blocks(kernel, smem) * sm_count));
  cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
  kernel<<<grid, kBlock, smem, s>>>(reinterpret_cast<const float4 *>(mesh->d_qnodes), mesh->d_tris, mesh->root_max,
                                    reinterpret_cast<const float4 *>(rays), n, occ, counter, perm, S, status, count);
}

void vt_launch_count(const vt_mesh *mesh, const vt_ray *rays, uint32_t n, int closest,
                     unsigned long long *acc, cudaStream_t s) {
  if (n == 0) return;
  k_count<<<(n + 127) / 128, 128, 0, s>>>(reinterpret_cast<const float4 *>(mesh->d_qnodes), mesh->d_tris,
                                         mesh->root_max, reinterpret_cast<const float4 *>(rays), n,
                                         closest, acc);
}

size_t vt_ray_order_words(uint32_t n) { return 4 * (((size_t)n + 63) & ~size_t(63)) + vt_radix_temp_words(n) + 64; }

const uint32_t *vt_ray_order(const vt_mesh *mesh, const vt_ray *rays, uint32_t n, uint32_t *scratch,
                             cudaStream_t s) {
  if (VT_TRACE_SORT == 0 || n < kSortMinRays) return nullptr;
  // Each array starts on a 256-byte boundary: the sort reads them with 16-byte vector loads.
  const size_t stride = ((size_t)n + 63) & ~size_t(63);
  uint32_t *keys = scratch, *vals = keys + stride, *keysAlt = vals + stride, *valsAlt = keysAlt + stride;
  uint32_t *temp = valsAlt + stride;
  float3 lo = make_float3(mesh->lo[0], mesh->lo[1], mesh->lo[2]);
  float ex = mesh->hi[0] - mesh->lo[0], ey = mesh->hi[1] - mesh->lo[1], ez = mesh->hi[2] - mesh->lo[2];
  float3 inv = make_float3(ex > 0 ? 1.0f / ex : 0.0f, ey > 0 ? 1.0f / ey : 0.0f, ez > 0 ? 1.0f / ez : 0.0f);
  k_ray_keys<<<(n + 255) / 256, 256, 0, s>>>(reinterpret_cast<const float4 *>(rays), n, lo, inv, keys, vals, VT_TRACE_SORT);
  vt_radix_sort_pairs(keys, vals, keysAlt, valsAlt, n, 30, temp, s);
  return vals;
}
