// lbvh.cu — GPU acceleration-structure build: LBVH (30-bit Morton codes, stable radix sort,
// Karras hierarchy), bottom-up refit, SAH treelet restructuring and the collapse to the
// reference's 4-wide node layout (MeshWideNode, main.swift:617; Sources/Acceleration.swift:23-30).
//
// Replaces the reference's CPU binned-SAH WideBVH.build (Sources/Acceleration.swift:106-352).
// Every arithmetic step that decides topology is written with explicitly rounded intrinsics
// (__fadd_rn, __fmul_rn, __fdiv_rn) so the CPU oracle (oracle/vt_oracle.cpp, built with
// -ffp-contract=off) reproduces Morton codes, sorted order and topology bit for bit.
#include <cfloat>
#include <vector>

#include "vt_internal.cuh"

namespace {

constexpr float kCi = 1.2f, kCt = 1.0f;  // treelet costs: internal node, triangle
constexpr int kMaxTreelet = 8;

struct Box { float3 lo, hi; };

__device__ __forceinline__ float box_area(float3 lo, float3 hi) {
  float ex = fmaxf(__fsub_rn(hi.x, lo.x), 0.0f), ey = fmaxf(__fsub_rn(hi.y, lo.y), 0.0f),
        ez = fmaxf(__fsub_rn(hi.z, lo.z), 0.0f);
  return __fadd_rn(__fadd_rn(__fmul_rn(ex, ey), __fmul_rn(ey, ez)), __fmul_rn(ez, ex));
}
__device__ __forceinline__ Box box_union(const Box &a, const Box &b) {
  return {make_float3(fminf(a.lo.x, b.lo.x), fminf(a.lo.y, b.lo.y), fminf(a.lo.z, b.lo.z)),
          make_float3(fmaxf(a.hi.x, b.hi.x), fmaxf(a.hi.y, b.hi.y), fmaxf(a.hi.z, b.hi.z))};
}
// Boxes live as two float4 (lo.xyz, hi.xyz). L2 loads (.cg) because other threads of the same
// launch write them in the bottom-up passes.
__device__ __forceinline__ Box load_box_cg(const float4 *b, int i) {
  float4 l = __ldcg(b + 2 * i), h = __ldcg(b + 2 * i + 1);
  return {make_float3(l.x, l.y, l.z), make_float3(h.x, h.y, h.z)};
}
__device__ __forceinline__ void store_box(float4 *b, int i, const Box &x) {
  __stcg(b + 2 * i, make_float4(x.lo.x, x.lo.y, x.lo.z, 0.0f));
  __stcg(b + 2 * i + 1, make_float4(x.hi.x, x.hi.y, x.hi.z, 0.0f));
}

// Order-preserving float <-> uint map for atomic min/max of the scene bounds.
__device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ inline float ord2f(uint32_t u) {
  uint32_t b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float f;
  memcpy(&f, &b, 4);
  return f;
#endif
}

// ---- stage 1: face boxes, centroid bounds, scene bounds, validation ---------------------------
// bounds[0..5] = centroid lo xyz, hi xyz; bounds[6..11] = scene lo xyz, hi xyz (ordered uints).
__global__ void k_init_bounds(uint32_t *bounds) {
  int i = threadIdx.x;
  if (i < 12) bounds[i] = (i % 6) < 3 ? 0xffffffffu : 0u;
}

__global__ void __launch_bounds__(256) k_face_boxes(const vt_face *faces, uint32_t nfaces,
                                                      const vt_vertex *verts, uint32_t nverts,
                                                      float4 *boxes, uint32_t *bounds,
                                                      uint32_t *status) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  float3 clo = make_float3(FLT_MAX, FLT_MAX, FLT_MAX), chi = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
  float3 slo = clo, shi = chi;
  if (i < nfaces) {
    vt_face f = faces[i];
    Box b{make_float3(0, 0, 0), make_float3(0, 0, 0)};
    if (f.a >= nverts || f.b >= nverts || f.c >= nverts) {
      atomicOr(status, (uint32_t)VT_DEV_BAD_INDEX);
    } else {
      const vt_vertex &va = verts[f.a], &vb = verts[f.b], &vc = verts[f.c];
      float3 a = make_float3(va.px, va.py, va.pz), p = make_float3(vb.px, vb.py, vb.pz),
             q = make_float3(vc.px, vc.py, vc.pz);
      bool finite = isfinite(a.x) && isfinite(a.y) && isfinite(a.z) && isfinite(p.x) &&
                    isfinite(p.y) && isfinite(p.z) && isfinite(q.x) && isfinite(q.y) && isfinite(q.z);
      if (!finite) {
        atomicOr(status, (uint32_t)VT_DEV_NONFINITE);
      } else {
        b.lo = make_float3(fminf(fminf(a.x, p.x), q.x), fminf(fminf(a.y, p.y), q.y), fminf(fminf(a.z, p.z), q.z));
        b.hi = make_float3(fmaxf(fmaxf(a.x, p.x), q.x), fmaxf(fmaxf(a.y, p.y), q.y), fmaxf(fmaxf(a.z, p.z), q.z));
      }
    }
    boxes[2 * i] = make_float4(b.lo.x, b.lo.y, b.lo.z, 0.0f);
    boxes[2 * i + 1] = make_float4(b.hi.x, b.hi.y, b.hi.z, 0.0f);
    float3 c = make_float3(__fmul_rn(__fadd_rn(b.lo.x, b.hi.x), 0.5f), __fmul_rn(__fadd_rn(b.lo.y, b.hi.y), 0.5f),
                           __fmul_rn(__fadd_rn(b.lo.z, b.hi.z), 0.5f));
    clo = chi = c;
    slo = b.lo;
    shi = b.hi;
  }
  // Warp then block reduction of the 12 bounds, one atomic per block per bound.
  float v[12] = {clo.x, clo.y, clo.z, chi.x, chi.y, chi.z, slo.x, slo.y, slo.z, shi.x, shi.y, shi.z};
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const bool isMin = (k % 6) < 3;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      float u = __shfl_xor_sync(0xffffffffu, v[k], o);
      v[k] = isMin ? fminf(v[k], u) : fmaxf(v[k], u);
    }
  }
  __shared__ float red[8][12];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 12; ++k) red[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x < 12) {
    const int k = threadIdx.x;
    const bool isMin = (k % 6) < 3;
    float x = red[0][k];
    for (int w = 1; w < (int)(blockDim.x / 32); ++w) x = isMin ? fminf(x, red[w][k]) : fmaxf(x, red[w][k]);
    if (isMin) atomicMin(&bounds[k], f2ord(x));
    else atomicMax(&bounds[k], f2ord(x));
  }
}

// ---- stage 2: Morton codes --------------------------------------------------------------------
__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}
// q = min(uint((c - clo) * (1024 / (chi - clo))), 1023), 0 on a flat axis.
__device__ __forceinline__ uint32_t quantize(float c, float clo, float chi) {
  float ext = __fsub_rn(chi, clo);
  if (!(ext > 0.0f)) return 0u;
  float scale = __fdiv_rn(1024.0f, ext);
  float f = __fmul_rn(__fsub_rn(c, clo), scale);
  return f >= 1023.0f ? 1023u : (uint32_t)f;
}

__global__ void k_morton(const float4 *boxes, uint32_t n, const uint32_t *bounds, uint32_t *codes,
                         uint32_t *vals) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 l = boxes[2 * i], h = boxes[2 * i + 1];
  float cx = __fmul_rn(__fadd_rn(l.x, h.x), 0.5f), cy = __fmul_rn(__fadd_rn(l.y, h.y), 0.5f),
        cz = __fmul_rn(__fadd_rn(l.z, h.z), 0.5f);
  uint32_t qx = quantize(cx, ord2f(bounds[0]), ord2f(bounds[3]));
  uint32_t qy = quantize(cy, ord2f(bounds[1]), ord2f(bounds[4]));
  uint32_t qz = quantize(cz, ord2f(bounds[2]), ord2f(bounds[5]));
  codes[i] = (expand_bits(qx) << 2) | (expand_bits(qy) << 1) | expand_bits(qz);
  vals[i] = i;
}

// ---- stage 3: Karras hierarchy (HPG 2012) -----------------------------------------------------
// Children: internal index >= 0, leaf = -(sorted position + 1). parent[] holds internal nodes at
// [0, n-1) and leaves at n - 1 + position; the root's parent is -1.
__device__ __forceinline__ int delta(const uint32_t *codes, int n, int i, int j) {
  if (j < 0 || j > n - 1) return -1;
  uint32_t a = codes[i], b = codes[j];
  if (a != b) return __clz(a ^ b);
  return 32 + __clz((uint32_t)i ^ (uint32_t)j);
}

__global__ void k_karras(const uint32_t *codes, int n, int2 *child, int32_t *parent) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) parent[0] = -1;
  if (i >= n - 1) return;
  const int d = delta(codes, n, i, i + 1) - delta(codes, n, i, i - 1) > 0 ? 1 : -1;
  const int dmin = delta(codes, n, i, i - d);
  int lmax = 2;
  while (delta(codes, n, i, i + lmax * d) > dmin) lmax *= 2;
  int l = 0;
  for (int s = lmax / 2; s >= 1; s /= 2)
    if (delta(codes, n, i, i + (l + s) * d) > dmin) l += s;
  const int j = i + l * d;
  const int dnode = delta(codes, n, i, j);
  int s = 0;
  for (int div = 2;; div *= 2) {
    const int step = (l + div - 1) / div;
    if (delta(codes, n, i, i + (s + step) * d) > dnode) s += step;
    if (step == 1) break;
  }
  const int gamma = i + s * d + min(d, 0);
  const int lo = min(i, j), hi = max(i, j);
  const int left = lo == gamma ? -(gamma + 1) : gamma;
  const int right = hi == gamma + 1 ? -(gamma + 2) : gamma + 1;
  child[i] = make_int2(left, right);
  parent[left >= 0 ? left : (n - 1 + gamma)] = i;
  parent[right >= 0 ? right : (n - 1 + gamma + 1)] = i;
}

__global__ void k_leaf_boxes(const float4 *boxes, const uint32_t *sorted, uint32_t n, float4 *leaf) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t f = sorted[i];
  leaf[2 * i] = boxes[2 * f];
  leaf[2 * i + 1] = boxes[2 * f + 1];
}

// ---- bottom-up passes ---------------------------------------------------------------------------
struct TreeView {
  int n;
  int2 *child;
  int32_t *parent;
  const float4 *leafBox;
  float4 *nodeBox;
  uint32_t *count;
  float *cost;
};

__device__ __forceinline__ int2 load_child(const TreeView &t, int i) {
  return __ldcg(t.child + i);
}
__device__ __forceinline__ Box child_box(const TreeView &t, int c) {
  return c >= 0 ? load_box_cg(t.nodeBox, c) : load_box_cg(t.leafBox, -c - 1);
}
__device__ __forceinline__ float child_cost(const TreeView &t, int c) {
  if (c >= 0) return __ldcg(t.cost + c);
  Box b = load_box_cg(t.leafBox, -c - 1);
  return __fmul_rn(kCt, box_area(b.lo, b.hi));
}
__device__ __forceinline__ uint32_t child_count(const TreeView &t, int c) {
  return c >= 0 ? __ldcg(t.count + c) : 1u;
}
__device__ __forceinline__ void refit_node(const TreeView &t, int i) {
  int2 ch = load_child(t, i);
  Box b = box_union(child_box(t, ch.x), child_box(t, ch.y));
  store_box(t.nodeBox, i, b);
  __stcg(t.count + i, child_count(t, ch.x) + child_count(t, ch.y));
  __stcg(t.cost + i, __fadd_rn(__fmul_rn(kCi, box_area(b.lo, b.hi)),
                               __fadd_rn(child_cost(t, ch.x), child_cost(t, ch.y))));
}

// Treelet restructuring at internal node `root` (Karras and Aila, HPG 2013), in the
// deterministic form the oracle restates: grow the treelet by opening its largest-area internal
// leaf (first in list order on ties; opened node replaced in place by its left child, right child
// appended), DP over subsets (partitions p = (p - 1) & s downwards, strict improvement), rebuild
// only on a strict cost improvement, internal nodes reassigned depth first, left = the side with
// the lowest leaf bit.
//
// Two executions of that one algorithm give the same tree. restructure_node is one thread's
// serial loop. restructure_warp spreads one treelet over a warp (Karras and Aila's warp-wide DP):
// lane q holds treelet leaf q while the treelet grows (its box, children, cost and leaf count
// loaded in one round trip, the largest area chosen by a shuffle reduction that keeps the first
// slot on ties); the subsets are listed by size with ballots (increasing s within a size); per
// size either each lane takes whole subsets (fewer than 32 partitions) or all lanes split one
// subset's partitions and reduce (cost, then serial order), so the chosen partition is the
// serial loop's; the rebuilt nodes' boxes, counts and costs are formed in shared memory in
// refit_node's order (union of left then right, costs added left + right) and stored by one lane
// per node. Scratch lives in shared memory, one slice per warp.
__device__ void restructure_node(const TreeView &t, int root, int size, uint32_t *status) {
  int leaves[kMaxTreelet], internals[kMaxTreelet];
  int nl = 0, ni = 0;
  internals[ni++] = root;
  int2 rc = load_child(t, root);
  leaves[nl++] = rc.x;
  leaves[nl++] = rc.y;
  while (nl < size) {
    int best = -1;
    float bestA = -1.0f;
    for (int k = 0; k < nl; ++k) {
      int c = leaves[k];
      if (c < 0) continue;
      Box b = load_box_cg(t.nodeBox, c);
      float a = box_area(b.lo, b.hi);
      if (a > bestA) { bestA = a; best = k; }
    }
    if (best < 0) break;
    int c = leaves[best];
    internals[ni++] = c;
    int2 cc = load_child(t, c);
    leaves[best] = cc.x;
    leaves[nl++] = cc.y;
  }
  const int k = nl;
  if (k < 3) return;
  const int full = (1 << k) - 1;
  float area[1 << kMaxTreelet], copt[1 << kMaxTreelet];
  uint8_t part[1 << kMaxTreelet];
  Box lb[kMaxTreelet];
  for (int q = 0; q < k; ++q) {
    lb[q] = child_box(t, leaves[q]);
    copt[1 << q] = child_cost(t, leaves[q]);
  }
  for (int s = 1; s <= full; ++s) {
    int low = __ffs(s) - 1;
    Box b = lb[low];
    for (int r = s & (s - 1); r; r &= r - 1) b = box_union(b, lb[__ffs(r) - 1]);
    area[s] = box_area(b.lo, b.hi);
  }
  for (int sz = 2; sz <= k; ++sz) {
    for (int s = 1; s <= full; ++s) {
      if (__popc(s) != sz) continue;
      float best = FLT_MAX;
      int bp = 0;
      for (int p = (s - 1) & s; p > 0; p = (p - 1) & s) {
        float c = __fadd_rn(copt[p], copt[s ^ p]);
        if (c < best) { best = c; bp = p; }
      }
      copt[s] = __fadd_rn(__fmul_rn(kCi, area[s]), best);
      part[s] = (uint8_t)bp;
    }
  }
  if (!(copt[full] < __ldcg(t.cost + root))) return;
  int next = 0;
  int st_s[kMaxTreelet * 2], st_n[kMaxTreelet * 2];
  int top = 0;
  st_s[top] = full; st_n[top] = internals[next++]; ++top;
  while (top) {
    --top;
    const int s = st_s[top], node = st_n[top];
    const int p = part[s], q = s ^ p;
    const int lowbit = s & -s;
    const int subs[2] = {(p & lowbit) ? p : q, (p & lowbit) ? q : p};
    int kids[2];
    for (int c = 0; c < 2; ++c) {
      const int x = subs[c];
      if ((x & (x - 1)) == 0) kids[c] = leaves[__ffs(x) - 1];
      else {
        if (next >= ni) { atomicOr(status, (uint32_t)VT_DEV_TREELET); return; }
        kids[c] = internals[next++];
      }
    }
    __stcg(t.child + node, make_int2(kids[0], kids[1]));
    for (int c = 1; c >= 0; --c)
      if ((subs[c] & (subs[c] - 1)) != 0) { st_s[top] = subs[c]; st_n[top] = kids[c]; ++top; }
  }
  for (int i = ni - 1; i >= 0; --i) {
    const int nd = internals[i];
    refit_node(t, nd);
    int2 ch = load_child(t, nd);
    __stcg(t.parent + (ch.x >= 0 ? ch.x : (t.n - 1 + (-ch.x - 1))), nd);
    __stcg(t.parent + (ch.y >= 0 ? ch.y : (t.n - 1 + (-ch.y - 1))), nd);
  }
}

struct TreeletScratch {
  float area[1 << kMaxTreelet];
  float copt[1 << kMaxTreelet];
  uint8_t part[1 << kMaxTreelet];
  uint8_t list[1 << kMaxTreelet];  // subsets grouped by size, increasing within a size
  Box lb[kMaxTreelet];             // treelet leaves' boxes
  Box nb[kMaxTreelet];             // rebuilt internal nodes' boxes (assignment order)
  float nc[kMaxTreelet];           // and costs
  uint32_t ncount[kMaxTreelet], lcount[kMaxTreelet];
  int leaves[kMaxTreelet], internals[kMaxTreelet];
  int2 kid[kMaxTreelet];           // rebuilt node j's children: >= 0 internal index, else -(leaf slot + 1)
  int start[kMaxTreelet + 2];      // list offset of each subset size
  int ok;
};

// The bits of m deposited into the set bits of s, lowest first (pdep).
__device__ __forceinline__ int deposit_bits(int m, int s) {
  int out = 0;
  for (int r = s; r; r &= r - 1) {
    if (m & 1) out |= r & -r;
    m >>= 1;
  }
  return out;
}

__device__ void restructure_warp(const TreeView &t, int root, int size, uint32_t *status, TreeletScratch &w) {
  const unsigned kAll = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const float rootCost = __ldcg(t.cost + root);
  const int2 rc = load_child(t, root);
  // Lane q < nl holds treelet leaf q: its node, box, children, cost and leaf count.
  int myLeaf = lane == 0 ? rc.x : rc.y;
  bool dirty = lane < 2;
  Box myBox{};
  int2 myKids = make_int2(0, 0);
  float myArea = -INFINITY, myCost = 0.0f;
  uint32_t myCount = 1u;
  int myInternal = lane == 0 ? root : -1;
  int nl = 2, ni = 1;
  while (true) {
    if (dirty) {
      if (myLeaf >= 0) {
        myBox = load_box_cg(t.nodeBox, myLeaf);
        myKids = load_child(t, myLeaf);
        myCost = __ldcg(t.cost + myLeaf);
        myCount = __ldcg(t.count + myLeaf);
        myArea = box_area(myBox.lo, myBox.hi);
      } else {
        myBox = load_box_cg(t.leafBox, -myLeaf - 1);
        myCost = __fmul_rn(kCt, box_area(myBox.lo, myBox.hi));
        myCount = 1u;
        myArea = -INFINITY;  // a primitive is never opened
      }
      dirty = false;
    }
    if (nl >= size) break;
    float a = lane < nl ? myArea : -INFINITY;
    int q = lane;
    for (int off = 16; off > 0; off >>= 1) {
      const float oa = __shfl_xor_sync(kAll, a, off);
      const int oq = __shfl_xor_sync(kAll, q, off);
      if (oa > a || (oa == a && oq < q)) { a = oa; q = oq; }
    }
    if (a == -INFINITY) break;  // no internal node left to open
    const int c = __shfl_sync(kAll, myLeaf, q);
    const int cx = __shfl_sync(kAll, myKids.x, q), cy = __shfl_sync(kAll, myKids.y, q);
    if (lane == ni) myInternal = c;
    if (lane == q) { myLeaf = cx; dirty = true; }
    if (lane == nl) { myLeaf = cy; dirty = true; }
    ++ni;
    ++nl;
  }
  const int k = nl;
  if (k < 3) return;
  const int full = (1 << k) - 1;
  if (lane < k) {
    w.leaves[lane] = myLeaf;
    w.lb[lane] = myBox;
    w.copt[1 << lane] = myCost;
    w.lcount[lane] = myCount;
  }
  if (lane < ni) w.internals[lane] = myInternal;
  if (lane == 0) {
    // Subsets of size j start after those of sizes 2..j-1: C(k, 2) + ... + C(k, j-1).
    int off = 0, c = k;  // c = C(k, j) for j = 1
    for (int j = 2; j <= k; ++j) {
      c = c * (k - j + 1) / j;
      w.start[j] = off;
      off += c;
    }
    w.start[k + 1] = off;
  }
  __syncwarp();
  // Subset areas and the by-size lists, 32 subsets per step.
  int fill[kMaxTreelet + 1];
#pragma unroll
  for (int j = 0; j <= kMaxTreelet; ++j) fill[j] = 0;
  for (int base = 0; base < full; base += 32) {
    const int s = base + lane + 1;
    const bool valid = s <= full;
    if (valid) {
      Box b = w.lb[__ffs(s) - 1];
      for (int r = s & (s - 1); r; r &= r - 1) b = box_union(b, w.lb[__ffs(r) - 1]);
      w.area[s] = box_area(b.lo, b.hi);
    }
    const int pc = valid ? __popc(s) : 0;
#pragma unroll
    for (int j = 2; j <= kMaxTreelet; ++j) {
      if (j > k) break;
      const unsigned m = __ballot_sync(kAll, pc == j);
      if (pc == j) w.list[w.start[j] + fill[j] + __popc(m & ((1u << lane) - 1u))] = (uint8_t)s;
      fill[j] += __popc(m);
    }
  }
  __syncwarp();
  for (int sz = 2; sz <= k; ++sz) {
    const int np = (1 << sz) - 2;  // partitions of a subset of size sz
    const int b0 = w.start[sz], nsub = w.start[sz + 1] - b0;
    if (np < 32) {
      for (int j = lane; j < nsub; j += 32) {
        const int s = w.list[b0 + j];
        float best = FLT_MAX;
        int bp = 0;
        for (int p = (s - 1) & s; p > 0; p = (p - 1) & s) {
          const float c = __fadd_rn(w.copt[p], w.copt[s ^ p]);
          if (c < best) { best = c; bp = p; }
        }
        w.copt[s] = __fadd_rn(__fmul_rn(kCi, w.area[s]), best);
        w.part[s] = (uint8_t)bp;
      }
    } else {
      // All lanes on one subset: partition i (serial order, p descending) is deposit(np - i, s).
      for (int j = 0; j < nsub; ++j) {
        const int s = w.list[b0 + j];
        float best = FLT_MAX;
        int bi = 0x7fffffff;
        for (int i = lane; i < np; i += 32) {
          const int p = deposit_bits(np - i, s);
          const float c = __fadd_rn(w.copt[p], w.copt[s ^ p]);
          if (c < best) { best = c; bi = i; }
        }
        for (int off = 16; off > 0; off >>= 1) {
          const float ob = __shfl_xor_sync(kAll, best, off);
          const int oi = __shfl_xor_sync(kAll, bi, off);
          if (ob < best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        if (lane == 0) {
          w.copt[s] = __fadd_rn(__fmul_rn(kCi, w.area[s]), best);
          w.part[s] = (uint8_t)deposit_bits(np - bi, s);
        }
      }
    }
    __syncwarp();
  }
  if (!(w.copt[full] < rootCost)) return;
  if (lane == 0) {
    // Depth-first assignment of the internal nodes (index j in assignment order), then their
    // boxes, counts and costs bottom up (children are assigned after their parent).
    int next = 1;
    int st_s[kMaxTreelet * 2], st_j[kMaxTreelet * 2];
    int top = 0;
    st_s[top] = full; st_j[top] = 0; ++top;
    w.ok = 1;
    while (top) {
      --top;
      const int s = st_s[top], j = st_j[top];
      const int p = w.part[s], q = s ^ p;
      const int lowbit = s & -s;
      const int subs[2] = {(p & lowbit) ? p : q, (p & lowbit) ? q : p};
      int ref[2];
      for (int c = 0; c < 2; ++c) {
        const int x = subs[c];
        if ((x & (x - 1)) == 0) ref[c] = -__ffs(x);  // -(leaf slot + 1)
        else {
          if (next >= ni) { w.ok = 0; top = 0; break; }
          ref[c] = next++;
        }
      }
      if (!w.ok) break;
      w.kid[j] = make_int2(ref[0], ref[1]);
      for (int c = 1; c >= 0; --c)
        if (ref[c] >= 0) { st_s[top] = subs[c]; st_j[top] = ref[c]; ++top; }
    }
    if (w.ok) {
      for (int j = ni - 1; j >= 0; --j) {
        const int2 r = w.kid[j];
        const Box bx = r.x >= 0 ? w.nb[r.x] : w.lb[-r.x - 1];
        const Box by = r.y >= 0 ? w.nb[r.y] : w.lb[-r.y - 1];
        const Box b = box_union(bx, by);
        const float cx = r.x >= 0 ? w.nc[r.x] : w.copt[1 << (-r.x - 1)];
        const float cy = r.y >= 0 ? w.nc[r.y] : w.copt[1 << (-r.y - 1)];
        w.nb[j] = b;
        w.nc[j] = __fadd_rn(__fmul_rn(kCi, box_area(b.lo, b.hi)), __fadd_rn(cx, cy));
        w.ncount[j] = (r.x >= 0 ? w.ncount[r.x] : w.lcount[-r.x - 1]) + (r.y >= 0 ? w.ncount[r.y] : w.lcount[-r.y - 1]);
      }
    } else {
      atomicOr(status, (uint32_t)VT_DEV_TREELET);
    }
  }
  __syncwarp();
  if (!w.ok || lane >= ni) return;
  const int node = w.internals[lane];
  const int2 r = w.kid[lane];
  const int kx = r.x >= 0 ? w.internals[r.x] : w.leaves[-r.x - 1];
  const int ky = r.y >= 0 ? w.internals[r.y] : w.leaves[-r.y - 1];
  __stcg(t.child + node, make_int2(kx, ky));
  store_box(t.nodeBox, node, w.nb[lane]);
  __stcg(t.count + node, w.ncount[lane]);
  __stcg(t.cost + node, w.nc[lane]);
  __stcg(t.parent + (kx >= 0 ? kx : (t.n - 1 + (-kx - 1))), node);
  __stcg(t.parent + (ky >= 0 ? ky : (t.n - 1 + (-ky - 1))), node);
}

// One thread per leaf walks to the root; the second thread to reach a node owns it (its two
// subtrees are final) and refits it. flags[] must be zero on entry.
__global__ void __launch_bounds__(128) k_bottom_up(TreeView t, uint32_t *flags, uint32_t *status) {
  const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= t.n) return;
  int node = __ldcg(t.parent + (t.n - 1 + leaf));
  // A walk longer than the node count means a corrupted parent chain: stop and report.
  for (int guard = 0; node >= 0; ++guard) {
    if (guard >= t.n) { atomicOr(status, (uint32_t)VT_DEV_TREELET); return; }
    __threadfence();
    if (atomicAdd(&flags[node], 1u) == 0u) return;
    __threadfence();
    refit_node(t, node);
    __threadfence();
    node = __ldcg(t.parent + node);
  }
}

// The same walk for restructuring. Nodes owned by lanes of one warp in the same step are disjoint
// subtrees (an owner's subtrees are final), so they may be restructured in any order: when more
// than kWarpTreelets lanes own a node with >= size leaves, each runs restructure_node on its own;
// otherwise the whole warp takes them one after another (restructure_warp).
constexpr int kWarpTreelets = 4;
__global__ void __launch_bounds__(128) k_restructure(TreeView t, uint32_t *flags, int size, uint32_t *status) {
  __shared__ TreeletScratch scratch[4];
  TreeletScratch &w = scratch[threadIdx.x >> 5];
  const unsigned kAll = 0xffffffffu;
  const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
  int node = leaf < t.n ? __ldcg(t.parent + (t.n - 1 + leaf)) : -1;
  int guard = 0;
  while (true) {
    bool own = false;
    if (node >= 0) {
      if (guard++ >= t.n) {
        atomicOr(status, (uint32_t)VT_DEV_TREELET);
        node = -1;
      } else {
        __threadfence();
        if (atomicAdd(&flags[node], 1u) == 0u) node = -1;
        else own = true;
        __threadfence();
      }
    }
    const bool mine = own && __ldcg(t.count + node) >= (uint32_t)size;
    unsigned work = __ballot_sync(kAll, mine);
    if (__popc(work) > kWarpTreelets) {
      if (mine) restructure_node(t, node, size, status);
    } else {
      while (work) {
        const int src = __ffs(work) - 1;
        work &= work - 1;
        const int root = __shfl_sync(kAll, node, src);
        restructure_warp(t, root, size, status, w);
        __syncwarp();
      }
    }
    __syncwarp();
    __threadfence();
    if (own) node = __ldcg(t.parent + node);
    if (!__any_sync(kAll, node >= 0)) break;
  }
}

// ---- collapse to 4-wide -------------------------------------------------------------------------
// A wide node rooted at binary node b starts with children [b] and splits the child of largest
// area among those with more than leafSize leaves (the reference's rule,
// Sources/Acceleration.swift:255-263) until four children.
__global__ void k_collapse_count(TreeView t, const int32_t *level, uint32_t L, int leafSize,
                                 int4 *chOut, uint32_t *nInner, uint32_t *nPrims) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= L) return;
  int ch[4] = {level[w], 0, 0, 0};
  int m = 1;
  while (m < 4) {
    int best = -1;
    float bestA = 0.0f;
    for (int k = 0; k < m; ++k) {
      if (child_count(t, ch[k]) <= (uint32_t)leafSize) continue;
      Box b = child_box(t, ch[k]);
      float a = box_area(b.lo, b.hi);
      if (best < 0 || a > bestA) { best = k; bestA = a; }
    }
    if (best < 0) break;
    const int c = ch[best];
    for (int k = m; k > best + 1; --k) ch[k] = ch[k - 1];
    int2 cc = load_child(t, c);
    ch[best] = cc.x;
    ch[best + 1] = cc.y;
    ++m;
  }
  uint32_t inner = 0, prims = 0;
  for (int k = 0; k < m; ++k) {
    uint32_t cnt = child_count(t, ch[k]);
    if (cnt <= (uint32_t)leafSize) prims += cnt;
    else ++inner;
  }
  // Unused slots marked INT_MIN (a valid leaf encoding never reaches it).
  int4 out = make_int4(ch[0], m > 1 ? ch[1] : INT_MIN, m > 2 ? ch[2] : INT_MIN, m > 3 ? ch[3] : INT_MIN);
  chOut[w] = out;
  nInner[w] = inner;
  nPrims[w] = prims;
}

__global__ void k_collapse_emit(TreeView t, uint32_t L, int leafSize, const int4 *chIn,
                                const uint32_t *offInner, const uint32_t *offPrims, uint32_t base,
                                uint32_t nextBase, uint32_t primBase, vt_wide_node *nodes,
                                int32_t *nextLevel, const uint32_t *sorted, const vt_face *faces,
                                const vt_vertex *verts, uint32_t nverts, int32_t *order, float4 *tris,
                                uint32_t *status, float4 *nrm = nullptr) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= L) return;
  int4 c4 = chIn[w];
  int ch[4] = {c4.x, c4.y, c4.z, c4.w};
  vt_wide_node nd;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    nd.lox[k] = nd.loy[k] = nd.loz[k] = nd.hix[k] = nd.hiy[k] = nd.hiz[k] = 0.0f;
    nd.child[k] = 0;
    nd.count[k] = 0;
  }
  uint32_t inner = offInner[w], prim = primBase + offPrims[w];
  for (int k = 0; k < 4; ++k) {
    if (ch[k] == INT_MIN) break;
    Box b = child_box(t, ch[k]);
    nd.lox[k] = b.lo.x; nd.loy[k] = b.lo.y; nd.loz[k] = b.lo.z;
    nd.hix[k] = b.hi.x; nd.hiy[k] = b.hi.y; nd.hiz[k] = b.hi.z;
    uint32_t cnt = child_count(t, ch[k]);
    if (cnt <= (uint32_t)leafSize) {
      nd.child[k] = -(int32_t)(prim + 1);
      nd.count[k] = (int32_t)cnt;
      // Leaves of the binary subtree, depth first, left first.
      int st[2 * 8 + 2];
      int top = 0;
      st[top++] = ch[k];
      while (top) {
        int c = st[--top];
        if (c < 0) {
          if (prim >= (uint32_t)t.n) { atomicOr(status, (uint32_t)VT_DEV_TREELET); return; }
          uint32_t f = sorted[-c - 1];
          order[prim] = (int32_t)f;
          vt_face fc = faces[f];
          if (fc.a >= nverts || fc.b >= nverts || fc.c >= nverts) {
            // k_face_boxes flagged this face already; its vertices are not read (the build then
            // returns VT_ERR_INVALID), the slot gets a degenerate triangle at the origin.
            atomicOr(status, (uint32_t)VT_DEV_BAD_INDEX);
            const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            tris[3 * prim] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float((int)f));
            tris[3 * prim + 1] = z;
            tris[3 * prim + 2] = z;
            if (nrm) nrm[3 * prim] = nrm[3 * prim + 1] = nrm[3 * prim + 2] = z;
            ++prim;
            continue;
          }
          const vt_vertex &va = verts[fc.a], &vb = verts[fc.b], &vc = verts[fc.c];
          tris[3 * prim] = make_float4(va.px, va.py, va.pz, __int_as_float((int)f));
          tris[3 * prim + 1] = make_float4(vb.px, vb.py, vb.pz, __uint_as_float(fc.tag));
          tris[3 * prim + 2] = make_float4(vc.px, vc.py, vc.pz, 0.0f);
          if (nrm) {  // vertex normals for smooth shading (mesh_hit_attributes)
            nrm[3 * prim] = make_float4(va.nx, va.ny, va.nz, 0.0f);
            nrm[3 * prim + 1] = make_float4(vb.nx, vb.ny, vb.nz, 0.0f);
            nrm[3 * prim + 2] = make_float4(vc.nx, vc.ny, vc.nz, 0.0f);
            const bool some = va.nx != 0.0f || va.ny != 0.0f || va.nz != 0.0f || vb.nx != 0.0f || vb.ny != 0.0f ||
                              vb.nz != 0.0f || vc.nx != 0.0f || vc.ny != 0.0f || vc.nz != 0.0f;
            if (some) atomicOr(status, (uint32_t)VT_DEV_NORMALS);
          }
          ++prim;
          continue;
        }
        if (top + 2 > 2 * 8 + 2) { atomicOr(status, (uint32_t)VT_DEV_TREELET); return; }
        int2 cc = load_child(t, c);
        st[top++] = cc.y;
        st[top++] = cc.x;
      }
    } else {
      nd.child[k] = (int32_t)(nextBase + inner);
      nextLevel[inner] = ch[k];
      ++inner;
    }
  }
  nodes[base + w] = nd;
}

// SAH cost of the wide tree (node cost 1, triangle cost 1, areas over the root box's area).
__global__ void k_sah(const vt_wide_node *nodes, uint32_t nn, double *acc) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const vt_wide_node &r = nodes[0];
  float3 lo = make_float3(FLT_MAX, FLT_MAX, FLT_MAX), hi = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
  for (int k = 0; k < 4; ++k) {
    if (r.child[k] == 0) continue;
    lo = make_float3(fminf(lo.x, r.lox[k]), fminf(lo.y, r.loy[k]), fminf(lo.z, r.loz[k]));
    hi = make_float3(fmaxf(hi.x, r.hix[k]), fmaxf(hi.y, r.hiy[k]), fmaxf(hi.z, r.hiz[k]));
  }
  auto dA = [](double lx, double ly, double lz, double hx, double hy, double hz) {
    double ex = fmax(0.0, hx - lx), ey = fmax(0.0, hy - ly), ez = fmax(0.0, hz - lz);
    return ex * ey + ey * ez + ez * ex;
  };
  double A0 = dA(lo.x, lo.y, lo.z, hi.x, hi.y, hi.z);
  if (!(A0 > 0.0)) A0 = 1.0;
  double v = 0.0;
  if (i < nn) {
    if (i == 0) v += 1.0;
    const vt_wide_node &nd = nodes[i];
    for (int k = 0; k < 4; ++k) {
      if (nd.child[k] == 0) continue;
      double a = dA(nd.lox[k], nd.loy[k], nd.loz[k], nd.hix[k], nd.hiy[k], nd.hiz[k]) / A0;
      v += nd.child[k] > 0 ? a : a * nd.count[k];
    }
  }
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(acc, v);
}

struct DeviceArena {
  std::vector<void *> ptrs;
  ~DeviceArena() {
    for (void *p : ptrs) cudaFree(p);
  }
  template <typename T> cudaError_t alloc(T **p, size_t count) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 16);
    if (e == cudaSuccess) {
      ptrs.push_back(q);
      *p = static_cast<T *>(q);
    }
    return e;
  }
};

inline uint32_t blocks(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

}  // namespace

vt_status vt_lbvh_build(vt_ctx *ctx, const vt_face *faces, uint32_t nfaces, const vt_vertex *verts,
                        uint32_t nverts, const vt_build_options &opt, vt_mesh *mesh) {
  cudaStream_t s = ctx->stream;
  const uint32_t n = nfaces;
  mesh->nfaces = n;
  if (n == 0) { mesh->nnodes = 0; mesh->depth = 0; return VT_OK; }
  int leafSize = opt.leaf_size > 0 ? opt.leaf_size : 2;
  int treelet = opt.treelet_size == 0 ? 7 : opt.treelet_size;
  int rounds = opt.refine_rounds > 0 ? opt.refine_rounds : 2;
  int maxDepth = opt.max_depth > 0 ? opt.max_depth : 31;
  if (leafSize > 8) return vt_fail(ctx, VT_ERR_INVALID, "leaf_size must be in 1..8");
  if (treelet > kMaxTreelet) treelet = kMaxTreelet;
  if (treelet > 0 && treelet < 3) treelet = 3;

  DeviceArena tmp;
  float4 *boxes, *leafBox, *nodeBox;
  uint32_t *bounds, *codes, *vals, *codesAlt, *valsAlt, *sortTemp, *flags, *count;
  int2 *child;
  int32_t *parent;
  float *cost;
  const uint32_t ni = n > 1 ? n - 1 : 1;
  VT_CUDA(ctx, tmp.alloc(&boxes, 2 * (size_t)n));
  VT_CUDA(ctx, tmp.alloc(&leafBox, 2 * (size_t)n));
  VT_CUDA(ctx, tmp.alloc(&nodeBox, 2 * (size_t)ni));
  VT_CUDA(ctx, tmp.alloc(&bounds, 16));
  VT_CUDA(ctx, tmp.alloc(&codesAlt, n));
  VT_CUDA(ctx, tmp.alloc(&valsAlt, n));
  VT_CUDA(ctx, tmp.alloc(&sortTemp, vt_radix_temp_words(n)));
  VT_CUDA(ctx, tmp.alloc(&flags, ni));
  VT_CUDA(ctx, tmp.alloc(&count, ni));
  VT_CUDA(ctx, tmp.alloc(&child, ni));
  VT_CUDA(ctx, tmp.alloc(&parent, 2 * (size_t)n));
  VT_CUDA(ctx, tmp.alloc(&cost, ni));
  // Outputs kept by the mesh.
  VT_CUDA(ctx, cudaMalloc(&mesh->d_codes, n * sizeof(uint32_t)));
  VT_CUDA(ctx, cudaMalloc(&mesh->d_sorted, n * sizeof(int32_t)));
  VT_CUDA(ctx, cudaMalloc(&mesh->d_order, n * sizeof(int32_t)));
  VT_CUDA(ctx, cudaMalloc(&mesh->d_tris, 3 * (size_t)n * sizeof(float4)));
  VT_CUDA(ctx, cudaMalloc(&mesh->d_nrm, 3 * (size_t)n * sizeof(float4)));
  codes = mesh->d_codes;
  vals = reinterpret_cast<uint32_t *>(mesh->d_sorted);

  VT_CUDA(ctx, cudaEventRecord(ctx->ev0, s));
  VT_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), s));
  k_init_bounds<<<1, 32, 0, s>>>(bounds);
  k_face_boxes<<<blocks(n, 256), 256, 0, s>>>(faces, n, verts, nverts, boxes, bounds, ctx->d_status);
  k_morton<<<blocks(n, 256), 256, 0, s>>>(boxes, n, bounds, codes, vals);
  vt_radix_sort_pairs(codes, vals, codesAlt, valsAlt, n, 30, sortTemp, s);
  k_leaf_boxes<<<blocks(n, 256), 256, 0, s>>>(boxes, vals, n, leafBox);
  TreeView t{(int)n, child, parent, leafBox, nodeBox, count, cost};
  if (n >= 2) {
    k_karras<<<blocks(n - 1, 256), 256, 0, s>>>(codes, (int)n, child, parent);
    VT_CUDA(ctx, cudaMemsetAsync(flags, 0, ni * sizeof(uint32_t), s));
    k_bottom_up<<<blocks(n, 128), 128, 0, s>>>(t, flags, ctx->d_status);
    if (treelet > 0 && n >= 3) {
      for (int r = 0; r < rounds; ++r) {
        VT_CUDA(ctx, cudaMemsetAsync(flags, 0, ni * sizeof(uint32_t), s));
        k_restructure<<<blocks(n, 128), 128, 0, s>>>(t, flags, treelet, ctx->d_status);
      }
    }
  }
  VT_CUDA(ctx, cudaGetLastError());

  // Collapse, level by level. Per-level arrays are sized by the level (at most n wide nodes per
  // level, fewer in practice); totals come back to the host to size the next level.
  int32_t *levelA, *levelB;
  int4 *chBuf;
  uint32_t *nInner, *nPrims, *scanTemp, *totals;
  VT_CUDA(ctx, tmp.alloc(&levelA, n));
  VT_CUDA(ctx, tmp.alloc(&levelB, n));
  VT_CUDA(ctx, tmp.alloc(&chBuf, n));
  VT_CUDA(ctx, tmp.alloc(&nInner, n));
  VT_CUDA(ctx, tmp.alloc(&nPrims, n));
  VT_CUDA(ctx, tmp.alloc(&scanTemp, vt_scan_temp_words(n)));
  VT_CUDA(ctx, tmp.alloc(&totals, 4));
  // Wide node count is bounded by the binary internal count (each wide inner node consumes at
  // least one binary internal node) plus the root.
  const uint32_t maxNodes = ni + 1;
  vt_wide_node *nodes;
  VT_CUDA(ctx, cudaMalloc(&nodes, maxNodes * sizeof(vt_wide_node)));
  mesh->d_nodes = nodes;
  const int32_t rootRef = n >= 2 ? 0 : -1;
  VT_CUDA(ctx, cudaMemcpyAsync(levelA, &rootRef, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  uint32_t L = 1, base = 0, primBase = 0, depth = 0;
  uint32_t host_tot[2];
  while (L > 0) {
    ++depth;
    if ((int)depth > maxDepth) {
      return vt_fail(ctx, VT_ERR_LIMIT, "BVH depth exceeds max_depth (" + std::to_string(maxDepth) + ")");
    }
    k_collapse_count<<<blocks(L, 128), 128, 0, s>>>(t, levelA, L, leafSize, chBuf, nInner, nPrims);
    vt_scan_exclusive(nInner, nInner, L, scanTemp, totals, s);
    vt_scan_exclusive(nPrims, nPrims, L, scanTemp, totals + 1, s);
    const uint32_t nextBase = base + L;
    k_collapse_emit<<<blocks(L, 128), 128, 0, s>>>(t, L, leafSize, chBuf, nInner, nPrims, base,
                                                   nextBase, primBase, nodes, levelB, vals, faces,
                                                   verts, nverts, mesh->d_order, mesh->d_tris, ctx->d_status,
                                                   mesh->d_nrm);
    uint32_t st_level = 0;
    VT_CUDA(ctx, cudaMemcpyAsync(host_tot, totals, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    VT_CUDA(ctx, cudaMemcpyAsync(&st_level, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    VT_CUDA(ctx, cudaStreamSynchronize(s));
    if (st_level & VT_DEV_TREELET) return vt_fail(ctx, VT_ERR_DEVICE, "hierarchy inconsistency during the collapse");
    if (st_level & (VT_DEV_BAD_INDEX | VT_DEV_NONFINITE)) break;
    primBase += host_tot[1];
    base = nextBase;
    L = host_tot[0];
    if (base + L > maxNodes) return vt_fail(ctx, VT_ERR_LIMIT, "wide node count exceeds its bound");
    int32_t *x = levelA; levelA = levelB; levelB = x;
  }
  mesh->nnodes = base;
  mesh->depth = depth;
  {
    uint32_t st0 = 0;
    VT_CUDA(ctx, cudaMemcpy(&st0, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (st0 & VT_DEV_BAD_INDEX) return vt_fail(ctx, VT_ERR_INVALID, "a face indexes past the vertex array");
    if (st0 & VT_DEV_NONFINITE) return vt_fail(ctx, VT_ERR_INVALID, "a vertex position is not finite");
    // A mesh without vertex normals shades with geometric normals: no normal buffer to read.
    if (!(st0 & VT_DEV_NORMALS)) {
      VT_CUDA(ctx, cudaFree(mesh->d_nrm));
      mesh->d_nrm = nullptr;
    }
  }
  if (primBase != n) return vt_fail(ctx, VT_ERR_DEVICE, "collapse emitted " + std::to_string(primBase) + " of " + std::to_string(n) + " triangles");

  {
    const vt_status qs = vt_quantize_nodes(ctx, mesh, s);
    if (qs != VT_OK) return qs;
  }
  // Keep the refined binary tree for parity checks.
  if (n >= 2) {
    VT_CUDA(ctx, cudaMalloc(&mesh->d_bin_child, 2 * (size_t)(n - 1) * sizeof(int32_t)));
    VT_CUDA(ctx, cudaMalloc(&mesh->d_bin_box, 8 * (size_t)(n - 1) * sizeof(float)));
    VT_CUDA(ctx, cudaMemcpyAsync(mesh->d_bin_child, child, 2 * (size_t)(n - 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    VT_CUDA(ctx, cudaMemcpyAsync(mesh->d_bin_box, nodeBox, 8 * (size_t)(n - 1) * sizeof(float), cudaMemcpyDeviceToDevice, s));
  }
  double *sah;
  VT_CUDA(ctx, tmp.alloc(&sah, 1));
  VT_CUDA(ctx, cudaMemsetAsync(sah, 0, sizeof(double), s));
  k_sah<<<blocks(mesh->nnodes, 256), 256, 0, s>>>(nodes, mesh->nnodes, sah);
  VT_CUDA(ctx, cudaEventRecord(ctx->ev1, s));
  uint32_t hb[12], status = 0;
  double hsah = 0.0;
  VT_CUDA(ctx, cudaMemcpyAsync(hb, bounds + 0, 12 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  VT_CUDA(ctx, cudaMemcpyAsync(&status, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  VT_CUDA(ctx, cudaMemcpyAsync(&hsah, sah, sizeof(double), cudaMemcpyDeviceToHost, s));
  VT_CUDA(ctx, cudaStreamSynchronize(s));
  if (status & VT_DEV_BAD_INDEX) return vt_fail(ctx, VT_ERR_INVALID, "a face indexes past the vertex array");
  if (status & VT_DEV_NONFINITE) return vt_fail(ctx, VT_ERR_INVALID, "a vertex position is not finite");
  if (status & VT_DEV_TREELET) return vt_fail(ctx, VT_ERR_DEVICE, "treelet restructuring inconsistency");
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  mesh->build_ms = ms;
  mesh->sah = (float)hsah;
  float m = 0.0f;
  for (int k = 0; k < 3; ++k) {
    mesh->lo[k] = ord2f(hb[6 + k]);
    mesh->hi[k] = ord2f(hb[9 + k]);
    m = fmaxf(m, fmaxf(fabsf(mesh->lo[k]), fabsf(mesh->hi[k])));
  }
  mesh->root_max = m;
  return VT_OK;
}

// =============================================================================================
// Allocation-free build (vt_mesh_build_noalloc). No counterpart in the reference.
//
// For callers that cannot call cudaMalloc: hosts that run under a fixed device-memory budget
// owned elsewhere (their own arena, or a framework's caching allocator holding the GPU memory),
// and loops that must not pay cudaMalloc/cudaFree's implicit device synchronisation. The caller
// passes the faces, vertices and the output buffers; every temporary of the build comes from
// g_build_scratch, a file-scope device array of kNoAllocScratchBytes that every GPU loading this
// library holds until the process exits. It fits VT_NOALLOC_MAX_FACES faces; larger meshes are
// rejected. The first call on a device looks the array's address up (cudaGetSymbolAddress, with
// that device current) and caches it, so that first call should come before any stream capture.
// Every call blocks the host until its build has finished: it synchronises its stream once per
// collapse level (the level's node count sizes the next launch) and at the end, and on an error
// after its first launch it still waits for the work it queued before returning.
// All calls share the one array and find the previous call's contents in it: every region the
// build needs zeroed is cleared on the call's stream, and two calls overlapping on the GPU (other
// streams or other host threads) race on it.
#include <chrono>
#include <cstring>
#include <mutex>

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(6) << 20;  // 6 MiB per GPU
static __device__ __align__(256) unsigned char g_build_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_scratch_mutex;
unsigned char *g_scratch_addr[kNoAllocMaxDevices] = {};

// Bump allocator over the scratch array (256-byte aligned regions). With base == nullptr it only
// measures.
struct ScratchCarve {
  unsigned char *base;
  size_t off = 0;
  template <typename T> T *take(size_t count) {
    size_t bytes = (count * sizeof(T) + 16 + 255) & ~size_t(255);
    T *p = base ? reinterpret_cast<T *>(base + off) : nullptr;
    off += bytes;
    return p;
  }
};

struct NoAllocBuffers {
  float4 *boxes, *leafBox, *nodeBox;
  uint32_t *bounds, *codes, *vals, *codesAlt, *valsAlt, *sortTemp, *flags, *count, *status;
  int2 *child;
  int32_t *parent, *levelA, *levelB;
  float *cost;
  int4 *chBuf;
  uint32_t *nInner, *nPrims, *scanTemp, *totals;
  double *sah;
};

size_t carve_noalloc(unsigned char *base, uint32_t n, NoAllocBuffers &b) {
  ScratchCarve c{base};
  const uint32_t ni = n > 1 ? n - 1 : 1;
  b.boxes = c.take<float4>(2 * (size_t)n);
  b.leafBox = c.take<float4>(2 * (size_t)n);
  b.nodeBox = c.take<float4>(2 * (size_t)ni);
  b.bounds = c.take<uint32_t>(16);
  b.codes = c.take<uint32_t>(n);
  b.vals = c.take<uint32_t>(n);
  b.codesAlt = c.take<uint32_t>(n);
  b.valsAlt = c.take<uint32_t>(n);
  b.sortTemp = c.take<uint32_t>(vt_radix_temp_words(n));
  b.flags = c.take<uint32_t>(ni);
  b.count = c.take<uint32_t>(ni);
  b.child = c.take<int2>(ni);
  b.parent = c.take<int32_t>(2 * (size_t)n);
  b.cost = c.take<float>(ni);
  b.levelA = c.take<int32_t>(n);
  b.levelB = c.take<int32_t>(n);
  b.chBuf = c.take<int4>(n);
  b.nInner = c.take<uint32_t>(n);
  b.nPrims = c.take<uint32_t>(n);
  b.scanTemp = c.take<uint32_t>(vt_scan_temp_words(n));
  b.totals = c.take<uint32_t>(4);
  b.status = c.take<uint32_t>(4);
  b.sah = c.take<double>(1);
  return c.off;
}

vt_status noalloc_fail(char *error, uint32_t capacity, vt_status code, const std::string &msg) {
  if (error && capacity) {
    std::strncpy(error, msg.c_str(), capacity - 1);
    error[capacity - 1] = '\0';
  }
  return code;
}

}  // namespace

extern "C" vt_status vt_mesh_build_noalloc(const vt_face *faces, uint32_t nfaces, const vt_vertex *verts,
                                           uint32_t nverts, const vt_build_options *opts,
                                           vt_wide_node *nodes, uint32_t nodes_capacity, float *tris,
                                           int32_t *order, vt_mesh_info *info, void *stream,
                                           char *error, uint32_t error_capacity) {
  auto t_start = std::chrono::steady_clock::now();
  if (error && error_capacity) error[0] = '\0';
  // Once work is queued on the stream, a failing call first waits for it (ignoring the result), so
  // that no kernel of this call still writes the shared scratch array after the call returns.
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  bool queued = false;
  auto fail = [&](vt_status code, const std::string &msg) {
    if (queued) (void)cudaStreamSynchronize(s);
    return noalloc_fail(error, error_capacity, code, msg);
  };
  if (nfaces > VT_NOALLOC_MAX_FACES)
    return fail(VT_ERR_LIMIT, "vt_mesh_build_noalloc: " + std::to_string(nfaces) + " faces exceed the limit of " +
                                  std::to_string(VT_NOALLOC_MAX_FACES) + " (the library's static build scratch)");
  if (!info) return fail(VT_ERR_INVALID, "vt_mesh_build_noalloc: info is null");
  std::memset(info, 0, sizeof *info);
  if (nfaces == 0) return VT_OK;
  if (!faces || !verts || !nodes || !tris || !order)
    return fail(VT_ERR_INVALID, "vt_mesh_build_noalloc: null input or output pointer");
  if (nodes_capacity < nfaces)
    return fail(VT_ERR_INVALID, "vt_mesh_build_noalloc: nodes_capacity must be at least nfaces");
  if ((reinterpret_cast<uintptr_t>(nodes) | reinterpret_cast<uintptr_t>(tris)) & 15u)
    return fail(VT_ERR_INVALID, "vt_mesh_build_noalloc: nodes and tris must be 16-byte aligned");
  vt_build_options o;
  std::memset(&o, 0, sizeof o);
  if (opts) o = *opts;
  const int leafSize = o.leaf_size > 0 ? o.leaf_size : 2;
  int treelet = o.treelet_size == 0 ? 7 : o.treelet_size;
  const int rounds = o.refine_rounds > 0 ? o.refine_rounds : 2;
  const int maxDepth = o.max_depth > 0 ? o.max_depth : 31;
  if (leafSize > 8) return fail(VT_ERR_INVALID, "vt_mesh_build_noalloc: leaf_size must be in 1..8");
  if (treelet > kMaxTreelet) treelet = kMaxTreelet;
  if (treelet > 0 && treelet < 3) treelet = 3;

  // Per-device set-up: the scratch array's device address, looked up once with the device current.
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(VT_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(VT_ERR_LIMIT, "vt_mesh_build_noalloc: device index too large");
  unsigned char *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_build_scratch);
      if (e != cudaSuccess) return fail(VT_ERR_CUDA, std::string("cudaGetSymbolAddress(build scratch): ") + cudaGetErrorString(e));
      NoAllocBuffers probe;
      if (carve_noalloc(nullptr, VT_NOALLOC_MAX_FACES, probe) > kNoAllocScratchBytes)
        return fail(VT_ERR_LIMIT, "vt_mesh_build_noalloc: static scratch smaller than the face limit needs");
      g_scratch_addr[dev] = static_cast<unsigned char *>(p);
    }
    scratch = g_scratch_addr[dev];
  }
  NoAllocBuffers b;
  carve_noalloc(scratch, nfaces, b);

  const uint32_t n = nfaces, ni = n > 1 ? n - 1 : 1;
#define VT_NA(call)                                                                  \
  do {                                                                               \
    cudaError_t _e = (call);                                                         \
    if (_e != cudaSuccess) return fail(VT_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(_e)); \
  } while (0)
  queued = true;
  VT_NA(cudaMemsetAsync(b.status, 0, 4 * sizeof(uint32_t), s));
  k_init_bounds<<<1, 32, 0, s>>>(b.bounds);
  k_face_boxes<<<blocks(n, 256), 256, 0, s>>>(faces, n, verts, nverts, b.boxes, b.bounds, b.status);
  k_morton<<<blocks(n, 256), 256, 0, s>>>(b.boxes, n, b.bounds, b.codes, b.vals);
  vt_radix_sort_pairs(b.codes, b.vals, b.codesAlt, b.valsAlt, n, 30, b.sortTemp, s);
  k_leaf_boxes<<<blocks(n, 256), 256, 0, s>>>(b.boxes, b.vals, n, b.leafBox);
  TreeView t{(int)n, b.child, b.parent, b.leafBox, b.nodeBox, b.count, b.cost};
  if (n >= 2) {
    k_karras<<<blocks(n - 1, 256), 256, 0, s>>>(b.codes, (int)n, b.child, b.parent);
    VT_NA(cudaMemsetAsync(b.flags, 0, ni * sizeof(uint32_t), s));
    k_bottom_up<<<blocks(n, 128), 128, 0, s>>>(t, b.flags, b.status);
    if (treelet > 0 && n >= 3) {
      for (int r = 0; r < rounds; ++r) {
        VT_NA(cudaMemsetAsync(b.flags, 0, ni * sizeof(uint32_t), s));
        k_restructure<<<blocks(n, 128), 128, 0, s>>>(t, b.flags, treelet, b.status);
      }
    }
  }
  VT_NA(cudaGetLastError());
  // Root reference of the first level: binary node 0, or leaf 0 (-1, all bits set) for one face.
  VT_NA(cudaMemsetAsync(b.levelA, n >= 2 ? 0 : 0xff, sizeof(int32_t), s));
  uint32_t L = 1, base = 0, primBase = 0, depth = 0;
  int32_t *levelA = b.levelA, *levelB = b.levelB;
  while (L > 0) {
    ++depth;
    if ((int)depth > maxDepth) return fail(VT_ERR_LIMIT, "vt_mesh_build_noalloc: BVH depth exceeds max_depth");
    k_collapse_count<<<blocks(L, 128), 128, 0, s>>>(t, levelA, L, leafSize, b.chBuf, b.nInner, b.nPrims);
    vt_scan_exclusive(b.nInner, b.nInner, L, b.scanTemp, b.totals, s);
    vt_scan_exclusive(b.nPrims, b.nPrims, L, b.scanTemp, b.totals + 1, s);
    const uint32_t nextBase = base + L;
    k_collapse_emit<<<blocks(L, 128), 128, 0, s>>>(t, L, leafSize, b.chBuf, b.nInner, b.nPrims, base, nextBase,
                                                   primBase, nodes, levelB, b.vals, faces, verts, nverts, order,
                                                   reinterpret_cast<float4 *>(tris), b.status);
    uint32_t tot[2] = {0, 0}, st = 0;
    VT_NA(cudaMemcpyAsync(tot, b.totals, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    VT_NA(cudaMemcpyAsync(&st, b.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    VT_NA(cudaStreamSynchronize(s));
    if (st & VT_DEV_BAD_INDEX) return fail(VT_ERR_INVALID, "vt_mesh_build_noalloc: a face indexes past the vertex array");
    if (st & VT_DEV_NONFINITE) return fail(VT_ERR_INVALID, "vt_mesh_build_noalloc: a vertex position is not finite");
    if (st & VT_DEV_TREELET) return fail(VT_ERR_DEVICE, "vt_mesh_build_noalloc: hierarchy inconsistency");
    primBase += tot[1];
    base = nextBase;
    L = tot[0];
    if (base + L > nodes_capacity) return fail(VT_ERR_LIMIT, "vt_mesh_build_noalloc: wide nodes exceed nodes_capacity");
    int32_t *x = levelA; levelA = levelB; levelB = x;
  }
  if (primBase != n) return fail(VT_ERR_DEVICE, "vt_mesh_build_noalloc: collapse emitted too few triangles");
  VT_NA(cudaMemsetAsync(b.sah, 0, sizeof(double), s));
  k_sah<<<blocks(base, 256), 256, 0, s>>>(nodes, base, b.sah);
  VT_NA(cudaGetLastError());
  uint32_t hb[12];
  double hsah = 0.0;
  VT_NA(cudaMemcpyAsync(hb, b.bounds, 12 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  VT_NA(cudaMemcpyAsync(&hsah, b.sah, sizeof(double), cudaMemcpyDeviceToHost, s));
  VT_NA(cudaStreamSynchronize(s));
#undef VT_NA
  info->faces = n;
  info->wide_nodes = base;
  info->binary_nodes = n - 1;
  info->depth = depth;
  info->sah_cost = (float)hsah;
  for (int k = 0; k < 3; ++k) {
    info->lo[k] = ord2f(hb[6 + k]);
    info->hi[k] = ord2f(hb[9 + k]);
  }
  info->build_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  return VT_OK;
}
