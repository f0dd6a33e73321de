// vt_oracle.cpp — CPU restatement of the reference's traversal and BVH-build arithmetic.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (tests, smoke check, bench CPU
// baseline). Built by oracle/Makefile with -ffp-contract=off so every float product and sum
// rounds on its own, exactly as the CUDA kernels' __fmul_rn/__fadd_rn sequence does.
// See vt_oracle.h for the list of reference functions restated here.
#include "vt_oracle.h"
#include "spectral_uplift.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>
#include <type_traits>
#include <vector>

namespace {

// ------------------------------------------------------------------------------------------
// PCG hash stream (main.swift:91-101): pcg_hash and the 24-bit float draw of rand_f.
uint32_t pcg_hash(uint32_t input) {
  uint32_t state = input * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}

// ------------------------------------------------------------------------------------------
// Small vector helpers.
struct F3 { float x, y, z; };
inline float comp(const F3 &v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
inline F3 fmin3(F3 a, F3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
inline F3 fmax3(F3 a, F3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }

// Surface-area measure of the reference's WideBVH.area (Sources/Acceleration.swift:125-128):
// e = max(hi - lo, 0); e.x e.y + e.y e.z + e.z e.x, each product and sum rounded on its own.
inline float box_area(F3 lo, F3 hi) {
  float ex = std::fmax(hi.x - lo.x, 0.0f), ey = std::fmax(hi.y - lo.y, 0.0f),
        ez = std::fmax(hi.z - lo.z, 0.0f);
  return (ex * ey + ey * ez) + ez * ex;
}

struct Box { F3 lo, hi; };
inline Box box_union(const Box &a, const Box &b) { return {fmin3(a.lo, b.lo), fmax3(a.hi, b.hi)}; }
const float kBig = 3.4028234663852886e38f;
inline Box empty_box() { return {{kBig, kBig, kBig}, {-kBig, -kBig, -kBig}}; }

inline F3 vpos(const vt_vertex &v) { return {v.px, v.py, v.pz}; }

// Triangle bounds of face i (Sources/Acceleration.swift:466-473, MeshSceneLayout.bounds).
inline Box face_box(const vt_face &f, const vt_vertex *v) {
  F3 a = vpos(v[f.a]), b = vpos(v[f.b]), c = vpos(v[f.c]);
  return {fmin3(fmin3(a, b), c), fmax3(fmax3(a, b), c)};
}

// ------------------------------------------------------------------------------------------
// Watertight ray/triangle test (main.swift:1536-1582). The ray is translated to the origin and
// sheared/scaled onto +z once; each vertex maps to (fma(-Sx, A[kz], A[kx]), fma(-Sy, A[kz], A[ky]),
// Sz A[kz]); edge functions are fl(fl(p.x q.y) - fl(p.y q.x)) with the exact FMA tie fallback
// (main.swift:1557-1562); a hit needs all edge signs to agree (0 counts for both), det != 0 and t in
// [tMin, tMax); the numerator is fma(W, cz, fma(V, bz, U az)).
template <typename T> struct WRay {
  T o[3];
  int kx, ky, kz;
  T Sx, Sy, Sz;
};
template <typename T> WRay<T> make_wray(const T o[3], const T d[3]) {
  WRay<T> w;
  T ax = std::fabs(d[0]), ay = std::fabs(d[1]), az = std::fabs(d[2]);
  int kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  int kx = kz == 2 ? 0 : kz + 1, ky = kx == 2 ? 0 : kx + 1;
  // Swapping x and y for a negative z direction preserves the winding.
  if (d[kz] < T(0)) std::swap(kx, ky);
  w.kx = kx; w.ky = ky; w.kz = kz;
  w.Sx = d[kx] / d[kz];
  w.Sy = d[ky] / d[kz];
  w.Sz = T(1) / d[kz];
  for (int k = 0; k < 3; ++k) w.o[k] = o[k];
  return w;
}
template <typename T> inline T edge_fn(T px, T py, T qx, T qy) {
  T x = px * qy, y = py * qx, e = x - y;
  if (e == T(0)) e = std::fma(px, qy, -x) - std::fma(py, qx, -y);
  return e;
}
template <typename T>
bool intersect_tri(const WRay<T> &r, const T a[3], const T b[3], const T c[3], T tMin, T tMax, T &t,
                   T &b1, T &b2) {
  T A[3], B[3], C[3];
  for (int k = 0; k < 3; ++k) { A[k] = a[k] - r.o[k]; B[k] = b[k] - r.o[k]; C[k] = c[k] - r.o[k]; }
  // The shear is one fused multiply-add per coordinate, as the CUDA test computes it.
  T ax = std::fma(-r.Sx, A[r.kz], A[r.kx]), ay = std::fma(-r.Sy, A[r.kz], A[r.ky]);
  T bx = std::fma(-r.Sx, B[r.kz], B[r.kx]), by = std::fma(-r.Sy, B[r.kz], B[r.ky]);
  T cx = std::fma(-r.Sx, C[r.kz], C[r.kx]), cy = std::fma(-r.Sy, C[r.kz], C[r.ky]);
  T U = edge_fn(cx, cy, bx, by), V = edge_fn(ax, ay, cx, cy);
  if ((U < 0 && V > 0) || (U > 0 && V < 0)) return false;
  T W = edge_fn(bx, by, ax, ay);
  if ((U < 0 || V < 0 || W < 0) && (U > 0 || V > 0 || W > 0)) return false;
  T det = (U + V) + W;
  if (det == T(0)) return false;
  T az = r.Sz * A[r.kz], bz = r.Sz * B[r.kz], cz = r.Sz * C[r.kz];
  T Tn = std::fma(W, cz, std::fma(V, bz, U * az));
  T inv = T(1) / det;
  t = Tn * inv;
  b1 = V * inv;
  b2 = W * inv;
  return t >= tMin && t < tMax;
}

// ------------------------------------------------------------------------------------------
// A built 4-wide BVH: nodes in the reference layout plus the triangles in BVH order.
struct BinNode { int32_t child[2]; Box box; };

}  // namespace

struct vto_bvh {
  std::vector<vt_wide_node> nodes;
  std::vector<int32_t> order;       // order[i] = input face at BVH position i
  std::vector<float> tris;          // 9 floats per BVH position
  uint32_t faces = 0, depth = 0;
  float root_max = 0.0f;            // max |coordinate| over the scene bounds
  Box bounds = empty_box();
  // LBVH-only stages
  std::vector<uint32_t> codes;      // sorted Morton codes
  std::vector<int32_t> sorted;      // face index per sorted position
  std::vector<BinNode> binary;      // refined binary tree (n - 1 internal nodes)
  double sah = 0.0;
  // The CUDA traversal's copy of the nodes with 8-bit child boxes (16 words each).
  std::vector<std::array<uint32_t, 16>> qnodes;
};

namespace {
void quantize_nodes(vto_bvh &h);
}  // namespace

namespace {

void finish_bvh(vto_bvh *h, const vt_face *faces, const vt_vertex *verts) {
  size_t n = h->order.size();
  h->tris.resize(9 * n);
  for (size_t i = 0; i < n; ++i) {
    const vt_face &f = faces[h->order[i]];
    const vt_vertex *p[3] = {&verts[f.a], &verts[f.b], &verts[f.c]};
    for (int k = 0; k < 3; ++k) {
      h->tris[9 * i + 3 * k + 0] = p[k]->px;
      h->tris[9 * i + 3 * k + 1] = p[k]->py;
      h->tris[9 * i + 3 * k + 2] = p[k]->pz;
    }
  }
  Box b = empty_box();
  for (uint32_t i = 0; i < h->faces; ++i) b = box_union(b, face_box(faces[i], verts));
  h->bounds = b;
  float m = 0.0f;
  if (h->faces) {
    m = std::fmax(std::fmax(std::fabs(b.lo.x), std::fabs(b.lo.y)), std::fabs(b.lo.z));
    m = std::fmax(m, std::fmax(std::fmax(std::fabs(b.hi.x), std::fabs(b.hi.y)), std::fabs(b.hi.z)));
  }
  h->root_max = m;
  // SAH cost: wide node cost 1, triangle cost 1, areas relative to the root box.
  double sah = 0.0;
  if (!h->nodes.empty()) {
    std::vector<double> area(h->nodes.size(), 0.0);
    Box root = empty_box();
    const vt_wide_node &r = h->nodes[0];
    for (int k = 0; k < 4; ++k)
      if (r.child[k] != 0) root = box_union(root, Box{{r.lox[k], r.loy[k], r.loz[k]}, {r.hix[k], r.hiy[k], r.hiz[k]}});
    auto dA = [](Box x) {
      double ex = std::max(0.0, double(x.hi.x) - x.lo.x), ey = std::max(0.0, double(x.hi.y) - x.lo.y),
             ez = std::max(0.0, double(x.hi.z) - x.lo.z);
      return ex * ey + ey * ez + ez * ex;
    };
    double A0 = dA(root);
    if (A0 <= 0) A0 = 1.0;
    area[0] = A0;
    for (size_t i = 0; i < h->nodes.size(); ++i) {
      const vt_wide_node &nd = h->nodes[i];
      sah += area[i] / A0;
      for (int k = 0; k < 4; ++k) {
        Box cb{{nd.lox[k], nd.loy[k], nd.loz[k]}, {nd.hix[k], nd.hiy[k], nd.hiz[k]}};
        if (nd.child[k] > 0) area[nd.child[k]] = dA(cb);
        else if (nd.child[k] < 0) sah += dA(cb) / A0 * nd.count[k];
      }
    }
  }
  h->sah = sah;
}

// ------------------------------------------------------------------------------------------
// LBVH (the GPU build's definition; no reference counterpart).
//
// Morton code of a centroid c = (lo + hi) * 0.5 inside the centroid bounds [clo, chi]: per axis
// q = min(uint((c - clo) * (1024 / (chi - clo))), 1023) (0 on a flat axis), bits interleaved
// x2 y1 z0. Faces sort by (code, face index). The binary hierarchy is Karras' (HPG 2012) over
// the sorted keys with the face index breaking code ties.
inline uint32_t expand_bits(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}
inline uint32_t quantize(float c, float clo, float chi) {
  float ext = chi - clo;
  if (!(ext > 0.0f)) return 0u;
  float scale = 1024.0f / ext;
  float f = (c - clo) * scale;
  uint32_t q = f >= 1023.0f ? 1023u : (uint32_t)f;
  return q;
}

inline int clz32(uint32_t v) { return v ? __builtin_clz(v) : 32; }

struct Karras {
  const uint32_t *codes;
  int n;
  int delta(int i, int j) const {
    if (j < 0 || j > n - 1) return -1;
    uint32_t a = codes[i], b = codes[j];
    if (a != b) return clz32(a ^ b);
    return 32 + clz32((uint32_t)i ^ (uint32_t)j);
  }
};

// Leaf encoding in the binary tree: internal node index >= 0, leaf = -(sorted position + 1).
struct LbvhTree {
  int n;
  std::vector<BinNode> nodes;      // n - 1 internal nodes
  std::vector<Box> leafBox;        // per sorted position
  std::vector<int32_t> parent;     // internal nodes then leaves (index n - 1 + pos)
  std::vector<uint32_t> count;     // leaves under each internal node
  std::vector<float> cost;         // SAH cost of each internal node's subtree
};

const float kCi = 1.2f, kCt = 1.0f;  // treelet restructuring costs (internal node, triangle)

inline Box child_box(const LbvhTree &t, int c) { return c >= 0 ? t.nodes[c].box : t.leafBox[-c - 1]; }
inline float child_cost(const LbvhTree &t, int c) {
  return c >= 0 ? t.cost[c] : kCt * box_area(t.leafBox[-c - 1].lo, t.leafBox[-c - 1].hi);
}
inline uint32_t child_count(const LbvhTree &t, int c) { return c >= 0 ? t.count[c] : 1u; }

// Bottom-up boxes, leaf counts and SAH costs (post-order, so children are final first).
void lbvh_refit(LbvhTree &t) {
  if (t.n < 2) return;
  std::vector<int> stack{0}, post;
  while (!stack.empty()) {
    int i = stack.back(); stack.pop_back();
    post.push_back(i);
    for (int k = 0; k < 2; ++k) if (t.nodes[i].child[k] >= 0) stack.push_back(t.nodes[i].child[k]);
  }
  for (auto it = post.rbegin(); it != post.rend(); ++it) {
    int i = *it;
    int l = t.nodes[i].child[0], r = t.nodes[i].child[1];
    Box b = box_union(child_box(t, l), child_box(t, r));
    t.nodes[i].box = b;
    t.count[i] = child_count(t, l) + child_count(t, r);
    t.cost[i] = kCi * box_area(b.lo, b.hi) + (child_cost(t, l) + child_cost(t, r));
  }
}

// Treelet restructuring (Karras and Aila, HPG 2013), deterministic form shared with the GPU:
// at an internal node whose subtree holds >= gamma leaves, grow a treelet by repeatedly opening
// the treelet leaf (an internal node) of largest area (first in list order on ties; the opened
// node is replaced in place by its left child and its right child is appended) until `size`
// leaves; find the SAH-optimal topology over those leaves by dynamic programming over subsets
// (partitions enumerated p = (p - 1) & s downwards, strict improvement keeps the first); if its
// cost is strictly below the current subtree cost, rebuild the treelet with the same internal
// nodes (root first, then in the order they were opened), assigning them depth-first, left
// partition (the one holding the lowest set leaf bit) first.
struct Treelet {
  int size;
  int leaves[8];
  int internals[8];
  int nl = 0, ni = 0;
};

void restructure_node(LbvhTree &t, int root, int size) {
  Treelet tl;
  tl.size = size;
  tl.internals[tl.ni++] = root;
  tl.leaves[tl.nl++] = t.nodes[root].child[0];
  tl.leaves[tl.nl++] = t.nodes[root].child[1];
  while (tl.nl < size) {
    int best = -1;
    float bestA = -1.0f;
    for (int k = 0; k < tl.nl; ++k) {
      int c = tl.leaves[k];
      if (c < 0) continue;
      float a = box_area(t.nodes[c].box.lo, t.nodes[c].box.hi);
      if (a > bestA) { bestA = a; best = k; }
    }
    if (best < 0) break;
    int c = tl.leaves[best];
    tl.internals[tl.ni++] = c;
    tl.leaves[best] = t.nodes[c].child[0];
    tl.leaves[tl.nl++] = t.nodes[c].child[1];
  }
  int k = tl.nl;
  if (k < 3) return;
  int full = (1 << k) - 1;
  float area[256], copt[256];
  uint8_t part[256];
  Box sb[256];
  for (int s = 1; s <= full; ++s) {
    int low = __builtin_ctz(s);
    Box b = child_box(t, tl.leaves[low]);
    if (s != (1 << low)) b = box_union(sb[s & (s - 1)], b);
    sb[s] = b;
    area[s] = box_area(b.lo, b.hi);
  }
  for (int i = 0; i < k; ++i) copt[1 << i] = child_cost(t, tl.leaves[i]);
  // Subsets by increasing size so every proper subset is final first.
  for (int sz = 2; sz <= k; ++sz) {
    for (int s = 1; s <= full; ++s) {
      if (__builtin_popcount(s) != sz) continue;
      float best = kBig;
      int bp = 0;
      for (int p = (s - 1) & s; p > 0; p = (p - 1) & s) {
        float c = copt[p] + copt[s ^ p];
        if (c < best) { best = c; bp = p; }
      }
      copt[s] = kCi * area[s] + best;
      part[s] = (uint8_t)bp;
    }
  }
  if (!(copt[full] < t.cost[root])) return;
  // Rebuild: assign internal nodes depth-first from the root.
  int next = 0;
  struct Item { int s, node; };
  Item stack[16];
  int top = 0;
  stack[top++] = {full, tl.internals[next++]};
  while (top) {
    Item it = stack[--top];
    int p = part[it.s], q = it.s ^ p;
    // Left = the side holding the lowest leaf bit of the subset.
    int lowbit = it.s & -it.s;
    int L = (p & lowbit) ? p : q, R = (p & lowbit) ? q : p;
    int kids[2];
    int subs[2] = {L, R};
    for (int c = 0; c < 2; ++c) {
      int s = subs[c];
      if ((s & (s - 1)) == 0) kids[c] = tl.leaves[__builtin_ctz(s)];
      else kids[c] = tl.internals[next++];
    }
    t.nodes[it.node].child[0] = kids[0];
    t.nodes[it.node].child[1] = kids[1];
    // Push right then left so the left subtree is assigned first.
    for (int c = 1; c >= 0; --c) if ((subs[c] & (subs[c] - 1)) != 0) stack[top++] = {subs[c], kids[c]};
  }
  // Refit the treelet's internal nodes bottom-up (reverse assignment order is a valid order:
  // every node was assigned after its parent).
  for (int i = tl.ni - 1; i >= 0; --i) {
    int nd = tl.internals[i];
    int l = t.nodes[nd].child[0], r = t.nodes[nd].child[1];
    Box b = box_union(child_box(t, l), child_box(t, r));
    t.nodes[nd].box = b;
    t.count[nd] = child_count(t, l) + child_count(t, r);
    t.cost[nd] = kCi * box_area(b.lo, b.hi) + (child_cost(t, l) + child_cost(t, r));
    for (int c = 0; c < 2; ++c) {
      int ch = t.nodes[nd].child[c];
      t.parent[ch >= 0 ? ch : (t.n - 1 + (-ch - 1))] = nd;
    }
  }
}

// One restructuring round: nodes in post-order (children before parents), as the GPU's
// bottom-up pass finalises them.
void restructure_round(LbvhTree &t, int size) {
  if (t.n < 2) return;
  std::vector<int> stack{0}, post;
  while (!stack.empty()) {
    int i = stack.back(); stack.pop_back();
    post.push_back(i);
    for (int k = 0; k < 2; ++k) if (t.nodes[i].child[k] >= 0) stack.push_back(t.nodes[i].child[k]);
  }
  for (auto it = post.rbegin(); it != post.rend(); ++it)
    if (t.count[*it] >= (uint32_t)size) restructure_node(t, *it, size);
}

// Collapse to the 4-wide layout, numbered level by level (breadth first): a wide node rooted at
// binary node b starts with children [b] and repeatedly splits the child of largest area among
// those with more than leafSize leaves (the reference's rule, Sources/Acceleration.swift:255-263);
// children with <= leafSize leaves become leaves whose triangles (depth-first, left first) are
// numbered in (node, slot) order; the others become the next level's nodes in (node, slot) order.
void lbvh_collapse(const LbvhTree &t, const std::vector<int32_t> &sorted, int leafSize, vto_bvh *h) {
  int n = t.n;
  h->nodes.clear();
  h->order.clear();
  if (n == 0) { h->depth = 0; return; }
  int rootRef = n >= 2 ? 0 : -1;
  std::vector<int> level{rootRef};
  uint32_t depth = 0;
  while (!level.empty()) {
    ++depth;
    size_t base = h->nodes.size();
    size_t nextBase = base + level.size();
    std::vector<int> next;
    for (size_t w = 0; w < level.size(); ++w) {
      int ch[4];
      int m = 0;
      ch[m++] = level[w];
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
        int c = ch[best];
        for (int k = m; k > best + 1; --k) ch[k] = ch[k - 1];
        ch[best] = t.nodes[c].child[0];
        ch[best + 1] = t.nodes[c].child[1];
        ++m;
      }
      vt_wide_node nd;
      std::memset(&nd, 0, sizeof nd);
      for (int k = 0; k < m; ++k) {
        Box b = child_box(t, ch[k]);
        nd.lox[k] = b.lo.x; nd.loy[k] = b.lo.y; nd.loz[k] = b.lo.z;
        nd.hix[k] = b.hi.x; nd.hiy[k] = b.hi.y; nd.hiz[k] = b.hi.z;
        uint32_t cnt = child_count(t, ch[k]);
        if (cnt <= (uint32_t)leafSize) {
          nd.child[k] = -(int32_t)(h->order.size() + 1);
          nd.count[k] = (int32_t)cnt;
          // Leaves of the binary subtree, depth first, left first.
          int st[64];
          int top = 0;
          st[top++] = ch[k];
          while (top) {
            int c = st[--top];
            if (c < 0) { h->order.push_back(sorted[-c - 1]); continue; }
            st[top++] = t.nodes[c].child[1];
            st[top++] = t.nodes[c].child[0];
          }
        } else {
          nd.child[k] = (int32_t)(nextBase + next.size());
          nd.count[k] = 0;
          next.push_back(ch[k]);
        }
      }
      h->nodes.push_back(nd);
    }
    level.swap(next);
  }
  h->depth = depth;
}

}  // namespace

extern "C" {

uint32_t vto_pcg_hash(uint32_t v) { return pcg_hash(v); }
float vto_rand_f(uint32_t *seed) {
  *seed = pcg_hash(*seed);
  return float(*seed >> 8u) * (1.0f / 16777216.0f);
}

int32_t vto_intersect_f32(const vt_ray *ray, const float *tri, float *t, float *b1, float *b2) {
  float o[3] = {ray->ox, ray->oy, ray->oz}, d[3] = {ray->dx, ray->dy, ray->dz};
  WRay<float> w = make_wray(o, d);
  return intersect_tri<float>(w, tri, tri + 3, tri + 6, ray->tmin, ray->tmax, *t, *b1, *b2) ? 1 : 0;
}
int32_t vto_intersect_f64(const double *ray, const double *tri, double tmin, double tmax, double *t,
                          double *b1, double *b2) {
  WRay<double> w = make_wray(ray, ray + 3);
  return intersect_tri<double>(w, tri, tri + 3, tri + 6, tmin, tmax, *t, *b1, *b2) ? 1 : 0;
}

// A hierarchy built elsewhere (the device's: its 4-wide nodes, leaf order and depth) over the same
// faces and vertices, for traversal and rendering without rebuilding it here.
vto_bvh *vto_bvh_import(const vt_wide_node *nodes, uint32_t nnodes, const int32_t *order, uint32_t nfaces,
                        const vt_face *faces, const vt_vertex *verts, uint32_t depth) {
  vto_bvh *h = new vto_bvh();
  h->faces = nfaces;
  h->depth = depth;
  h->nodes.assign(nodes, nodes + nnodes);
  h->order.assign(order, order + nfaces);
  finish_bvh(h, faces, verts);
  quantize_nodes(*h);
  return h;
}

vto_bvh *vto_lbvh_build(const vt_face *faces, uint32_t nfaces, const vt_vertex *verts,
                        uint32_t nverts, int32_t leaf_size, int32_t treelet_size, int32_t rounds) {
  (void)nverts;
  vto_bvh *h = new vto_bvh();
  h->faces = nfaces;
  int n = (int)nfaces;
  if (leaf_size < 1) leaf_size = 2;
  std::vector<Box> boxes(n);
  std::vector<F3> cent(n);
  Box cb = empty_box();
  for (int i = 0; i < n; ++i) {
    boxes[i] = face_box(faces[i], verts);
    F3 c = {(boxes[i].lo.x + boxes[i].hi.x) * 0.5f, (boxes[i].lo.y + boxes[i].hi.y) * 0.5f,
            (boxes[i].lo.z + boxes[i].hi.z) * 0.5f};
    cent[i] = c;
    cb.lo = fmin3(cb.lo, c);
    cb.hi = fmax3(cb.hi, c);
  }
  std::vector<uint64_t> keys(n);
  for (int i = 0; i < n; ++i) {
    uint32_t qx = quantize(cent[i].x, cb.lo.x, cb.hi.x), qy = quantize(cent[i].y, cb.lo.y, cb.hi.y),
             qz = quantize(cent[i].z, cb.lo.z, cb.hi.z);
    uint32_t code = (expand_bits(qx) << 2) | (expand_bits(qy) << 1) | expand_bits(qz);
    keys[i] = (uint64_t(code) << 32) | uint32_t(i);
  }
  std::sort(keys.begin(), keys.end());
  h->codes.resize(n);
  h->sorted.resize(n);
  for (int i = 0; i < n; ++i) {
    h->codes[i] = uint32_t(keys[i] >> 32);
    h->sorted[i] = int32_t(keys[i] & 0xffffffffu);
  }
  LbvhTree t;
  t.n = n;
  t.nodes.resize(n > 1 ? n - 1 : 0);
  t.count.assign(t.nodes.size(), 0);
  t.cost.assign(t.nodes.size(), 0.0f);
  t.parent.assign(n > 0 ? 2 * n - 1 : 0, -1);
  t.leafBox.resize(n);
  for (int i = 0; i < n; ++i) t.leafBox[i] = boxes[h->sorted[i]];
  Karras K{h->codes.data(), n};
  for (int i = 0; i < n - 1; ++i) {
    int d = K.delta(i, i + 1) - K.delta(i, i - 1) > 0 ? 1 : -1;
    int dmin = K.delta(i, i - d);
    int lmax = 2;
    while (K.delta(i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int s = lmax / 2; s >= 1; s /= 2)
      if (K.delta(i, i + (l + s) * d) > dmin) l += s;
    int j = i + l * d;
    int dnode = K.delta(i, j);
    int s = 0;
    for (int div = 2;; div *= 2) {
      int step = (l + div - 1) / div;
      if (K.delta(i, i + (s + step) * d) > dnode) s += step;
      if (step == 1) break;
    }
    int gamma = i + s * d + std::min(d, 0);
    int lo = std::min(i, j), hi = std::max(i, j);
    int left = lo == gamma ? -(gamma + 1) : gamma;
    int right = hi == gamma + 1 ? -(gamma + 2) : gamma + 1;
    t.nodes[i].child[0] = left;
    t.nodes[i].child[1] = right;
    t.parent[left >= 0 ? left : (n - 1 + gamma)] = i;
    t.parent[right >= 0 ? right : (n - 1 + gamma + 1)] = i;
  }
  lbvh_refit(t);
  if (treelet_size == 0) treelet_size = 7;
  if (rounds <= 0) rounds = 2;
  if (treelet_size > 0 && n >= 3) {
    if (treelet_size < 3) treelet_size = 3;
    if (treelet_size > 8) treelet_size = 8;
    for (int r = 0; r < rounds; ++r) restructure_round(t, treelet_size);
  }
  h->binary = t.nodes;
  lbvh_collapse(t, h->sorted, leaf_size, h);
  finish_bvh(h, faces, verts);
  quantize_nodes(*h);
  return h;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Reference binned-SAH 4-wide build (WideBVH, Sources/Acceleration.swift:106-352), restated:
// 16 bins on each axis with a non-zero finite scale, SAH cost area x count of both sides, the
// in-place two-pointer partition, coincident-centroid / balanced fallback to an object median on
// the widest centroid axis, each node splitting its largest-area child (most populous in median
// mode) until four children, depth-first numbering with subtrees below n/16 deferred and appended
// in order (n >= 65536), and a median rebuild past the depth limit.
namespace {

struct Range {
  int start, end;
  F3 lo, hi, clo, chi;
  int count() const { return end - start; }
  float area() const { return box_area(lo, hi); }
};

struct WideBuilder {
  const float *bounds;  // 6 per item
  int32_t *order;
  int leafSize;
  bool median;
  static const int kBins = 16;
  F3 binLo[3 * kBins], binHi[3 * kBins], binCLo[3 * kBins], binCHi[3 * kBins];
  int binCount[3 * kBins];
  float suffix[kBins];

  F3 lo(int i) const { return {bounds[6 * i], bounds[6 * i + 1], bounds[6 * i + 2]}; }
  F3 hi(int i) const { return {bounds[6 * i + 3], bounds[6 * i + 4], bounds[6 * i + 5]}; }
  Range measure(int start, int end) const {
    Range r{start, end, {kBig, kBig, kBig}, {-kBig, -kBig, -kBig}, {kBig, kBig, kBig}, {-kBig, -kBig, -kBig}};
    for (int k = start; k < end; ++k) {
      int i = order[k];
      F3 l = lo(i), h = hi(i), c = {(l.x + h.x) * 0.5f, (l.y + h.y) * 0.5f, (l.z + h.z) * 0.5f};
      r.lo = fmin3(r.lo, l); r.hi = fmax3(r.hi, h); r.clo = fmin3(r.clo, c); r.chi = fmax3(r.chi, c);
    }
    return r;
  }
  static float bin_scale(float e) {
    float s = float(kBins) / e;
    return e > 0 && std::isfinite(s) ? s : 0.0f;
  }
  static int to_bin(float f) {
    // Swift Int(Float) truncates toward zero; clamp to [0, bins - 1].
    long v = (long)f;
    return (int)std::min<long>(kBins - 1, std::max<long>(0, v));
  }
  void split(const Range &r, Range &left, Range &right) {
    F3 ext = {r.chi.x - r.clo.x, r.chi.y - r.clo.y, r.chi.z - r.clo.z};
    float emax = std::fmax(ext.x, std::fmax(ext.y, ext.z));
    F3 big = {kBig, kBig, kBig}, nbig = {-kBig, -kBig, -kBig};
    if (!median && emax > 0) {
      float scale[3] = {bin_scale(ext.x), bin_scale(ext.y), bin_scale(ext.z)};
      for (int k = 0; k < 3 * kBins; ++k) { binLo[k] = big; binHi[k] = nbig; binCLo[k] = big; binCHi[k] = nbig; binCount[k] = 0; }
      for (int k = r.start; k < r.end; ++k) {
        int i = order[k];
        F3 l = lo(i), h = hi(i), c = {(l.x + h.x) * 0.5f, (l.y + h.y) * 0.5f, (l.z + h.z) * 0.5f};
        float f[3] = {(c.x - r.clo.x) * scale[0], (c.y - r.clo.y) * scale[1], (c.z - r.clo.z) * scale[2]};
        for (int a = 0; a < 3; ++a) {
          int s = a * kBins + to_bin(f[a]);
          binCount[s] += 1;
          binLo[s] = fmin3(binLo[s], l); binHi[s] = fmax3(binHi[s], h);
          binCLo[s] = fmin3(binCLo[s], c); binCHi[s] = fmax3(binCHi[s], c);
        }
      }
      float bestCost = kBig;
      int best = -1, bin = 0;
      for (int a = 0; a < 3; ++a) {
        if (!(scale[a] > 0)) continue;
        F3 l = big, h = nbig;
        int count = 0;
        for (int b = kBins - 1; b > 0; --b) {
          int k = a * kBins + b;
          if (binCount[k] > 0) { l = fmin3(l, binLo[k]); h = fmax3(h, binHi[k]); }
          count += binCount[k];
          suffix[b] = count > 0 ? box_area(l, h) * float(count) : 0.0f;
        }
        l = big; h = nbig; count = 0;
        for (int b = 0; b < kBins - 1; ++b) {
          int k = a * kBins + b;
          if (binCount[k] > 0) { l = fmin3(l, binLo[k]); h = fmax3(h, binHi[k]); }
          count += binCount[k];
          if (count == 0 || count == r.count()) continue;
          float cost = box_area(l, h) * float(count) + suffix[b + 1];
          if (cost < bestCost) { bestCost = cost; best = a; bin = b; }
        }
      }
      if (best >= 0) {
        float s = scale[best], origin = comp(r.clo, best);
        int i = r.start, j = r.end - 1;
        while (i <= j) {
          int tt = order[i];
          float c = (bounds[6 * tt + best] + bounds[6 * tt + 3 + best]) * 0.5f;
          if (to_bin((c - origin) * s) <= bin) ++i;
          else { std::swap(order[i], order[j]); --j; }
        }
        if (i > r.start && i < r.end) {
          left = Range{r.start, i, big, nbig, big, nbig};
          right = Range{i, r.end, big, nbig, big, nbig};
          for (int b = 0; b < kBins; ++b) {
            int k = best * kBins + b;
            if (binCount[k] <= 0) continue;
            Range &x = b <= bin ? left : right;
            x.lo = fmin3(x.lo, binLo[k]); x.hi = fmax3(x.hi, binHi[k]);
            x.clo = fmin3(x.clo, binCLo[k]); x.chi = fmax3(x.chi, binCHi[k]);
          }
          return;
        }
      }
    }
    int middle = (r.start + r.end) / 2;
    if (emax > 0) {
      int a = ext.x > ext.y ? (ext.x > ext.z ? 0 : 2) : (ext.y > ext.z ? 1 : 2);
      const float *b = bounds;
      std::sort(order + r.start, order + r.end, [b, a](int32_t x, int32_t y) {
        float cx = b[6 * x + a] + b[6 * x + 3 + a], cy = b[6 * y + a] + b[6 * y + 3 + a];
        return cx == cy ? x < y : cx < cy;
      });
    }
    left = measure(r.start, middle);
    right = measure(middle, r.end);
  }
  struct Work { Range r; int parent, slot, level; };
  int run(const Range &root, int depth, std::vector<vt_wide_node> &nodes, int deferThreshold,
          std::vector<Work> &deferred) {
    int reached = depth;
    std::vector<Work> work{{root, -1, 0, depth}};
    while (!work.empty()) {
      Work wk = work.back(); work.pop_back();
      reached = std::max(reached, wk.level);
      std::vector<Range> children{wk.r};
      while (children.size() < 4) {
        int best = -1;
        for (size_t k = 0; k < children.size(); ++k) {
          const Range &c = children[k];
          if (c.count() <= leafSize) continue;
          if (best < 0 || (median ? c.count() > children[best].count() : c.area() > children[best].area())) best = (int)k;
        }
        if (best < 0) break;
        Range a, b;
        split(children[best], a, b);
        children[best] = a;
        children.insert(children.begin() + best + 1, b);
      }
      vt_wide_node nd;
      std::memset(&nd, 0, sizeof nd);
      int index = (int)nodes.size();
      if (wk.parent >= 0) nodes[wk.parent].child[wk.slot] = index;
      for (size_t k = 0; k < children.size(); ++k) {
        const Range &c = children[k];
        nd.lox[k] = c.lo.x; nd.loy[k] = c.lo.y; nd.loz[k] = c.lo.z;
        nd.hix[k] = c.hi.x; nd.hiy[k] = c.hi.y; nd.hiz[k] = c.hi.z;
        if (c.count() <= leafSize) { nd.child[k] = -(c.start + 1); nd.count[k] = c.count(); }
      }
      nodes.push_back(nd);
      for (int k = (int)children.size() - 1; k >= 0; --k) {
        if (children[k].count() <= leafSize) continue;
        if (children[k].count() < deferThreshold) deferred.push_back({children[k], index, k, wk.level + 1});
        else work.push_back({children[k], index, k, wk.level + 1});
      }
    }
    return reached;
  }
};

int wide_build(const float *bounds, int n, int leafSize, bool median, int threads,
               std::vector<int32_t> &order, std::vector<vt_wide_node> &nodes) {
  order.resize(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  nodes.clear();
  if (n <= 0) return 0;
  WideBuilder *b = new WideBuilder{bounds, order.data(), leafSize, median};
  std::vector<WideBuilder::Work> deferred;
  int threshold = n >= 65536 ? n / 16 : 0;
  int depth = b->run(b->measure(0, n), 1, nodes, threshold, deferred);
  delete b;
  if (!deferred.empty()) {
    size_t T = deferred.size();
    std::vector<std::vector<vt_wide_node>> parts(T);
    std::vector<int> depths(T, 0);
    std::atomic<size_t> next{0};
    auto worker = [&]() {
      WideBuilder *local = new WideBuilder{bounds, order.data(), leafSize, median};
      for (size_t t; (t = next.fetch_add(1)) < T;) {
        std::vector<WideBuilder::Work> none;
        depths[t] = local->run(deferred[t].r, deferred[t].level, parts[t], 0, none);
      }
      delete local;
    };
    int nt = std::max(1, std::min<int>(threads, (int)T));
    std::vector<std::thread> pool;
    for (int i = 0; i < nt; ++i) pool.emplace_back(worker);
    for (auto &th : pool) th.join();
    for (size_t t = 0; t < T; ++t) {
      int32_t offset = (int32_t)nodes.size();
      nodes[deferred[t].parent].child[deferred[t].slot] = offset;
      for (vt_wide_node nd : parts[t]) {
        for (int k = 0; k < 4; ++k) if (nd.child[k] > 0) nd.child[k] += offset;
        nodes.push_back(nd);
      }
      depth = std::max(depth, depths[t]);
    }
  }
  return depth;
}

}  // namespace

extern "C" {

vto_bvh *vto_widebvh_build(const vt_face *faces, uint32_t nfaces, const vt_vertex *verts,
                           uint32_t nverts, int32_t leaf_size, int32_t max_depth, int32_t threads) {
  (void)nverts;
  vto_bvh *h = new vto_bvh();
  h->faces = nfaces;
  int n = (int)nfaces;
  if (leaf_size < 1) leaf_size = 2;
  if (max_depth <= 0) max_depth = 20;
  if (threads <= 0) threads = 1;
  std::vector<float> bounds(6 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    Box b = face_box(faces[i], verts);
    bounds[6 * i] = b.lo.x; bounds[6 * i + 1] = b.lo.y; bounds[6 * i + 2] = b.lo.z;
    bounds[6 * i + 3] = b.hi.x; bounds[6 * i + 4] = b.hi.y; bounds[6 * i + 5] = b.hi.z;
  }
  int depth = wide_build(bounds.data(), n, leaf_size, false, threads, h->order, h->nodes);
  if (depth > max_depth) depth = wide_build(bounds.data(), n, leaf_size, true, threads, h->order, h->nodes);
  h->depth = (uint32_t)depth;
  finish_bvh(h, faces, verts);
  quantize_nodes(*h);
  return h;
}

void vto_bvh_free(vto_bvh *h) { delete h; }

void vto_bvh_get_info(const vto_bvh *h, vto_bvh_info *out) {
  out->faces = h->faces;
  out->wide_nodes = (uint32_t)h->nodes.size();
  out->binary_nodes = (uint32_t)h->binary.size();
  out->depth = h->depth;
  out->sah_cost = (float)h->sah;
  out->lo[0] = h->bounds.lo.x; out->lo[1] = h->bounds.lo.y; out->lo[2] = h->bounds.lo.z;
  out->hi[0] = h->bounds.hi.x; out->hi[1] = h->bounds.hi.y; out->hi[2] = h->bounds.hi.z;
}
void vto_bvh_get_nodes(const vto_bvh *h, vt_wide_node *out) {
  if (!h->nodes.empty()) std::memcpy(out, h->nodes.data(), h->nodes.size() * sizeof(vt_wide_node));
}
void vto_bvh_get_order(const vto_bvh *h, int32_t *out) {
  if (!h->order.empty()) std::memcpy(out, h->order.data(), h->order.size() * sizeof(int32_t));
}
void vto_bvh_get_morton(const vto_bvh *h, uint32_t *codes, int32_t *sorted) {
  if (!h->codes.empty()) std::memcpy(codes, h->codes.data(), h->codes.size() * sizeof(uint32_t));
  if (!h->sorted.empty()) std::memcpy(sorted, h->sorted.data(), h->sorted.size() * sizeof(int32_t));
}
void vto_bvh_get_binary(const vto_bvh *h, int32_t *children, float *boxes) {
  for (size_t i = 0; i < h->binary.size(); ++i) {
    const BinNode &b = h->binary[i];
    children[2 * i] = b.child[0];
    children[2 * i + 1] = b.child[1];
    float v[6] = {b.box.lo.x, b.box.lo.y, b.box.lo.z, b.box.hi.x, b.box.hi.y, b.box.hi.z};
    std::memcpy(boxes + 6 * i, v, sizeof v);
  }
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Traversal (main.swift:1758-1838): conservative slab test with origins shifted by
// e = 2^-23 (|o|max + rootMax) (wide_ray, main.swift:1758-1763), near-to-far insertion order
// (wide_order, :1780-1785), closest hit popping the nearest inner child first (blas_closest),
// any hit in child-slot order (blas_any, without endpoint slack).
namespace {

template <typename T> struct TraceRay {
  T o[3], d[3], tmin, tmax;
};

template <typename T> struct SlabRay {
  T low[3], high[3], inv[3];
  bool parallel[3];
};

template <typename T> T max_abs_origin(const TraceRay<T> &r) {
  return std::fmax(std::fmax(std::fabs(r.o[0]), std::fabs(r.o[1])), std::fabs(r.o[2]));
}

// The slab ray with origin shift e.
template <typename T> SlabRay<T> make_slab_e(const TraceRay<T> &r, T e) {
  SlabRay<T> s;
  for (int k = 0; k < 3; ++k) {
    s.low[k] = r.o[k] + e;
    s.high[k] = r.o[k] - e;
    if (std::is_same<T, float>::value) {
      // The CUDA kernels' form: a parallel axis gets the inverse +-1e30 (no separate inside test).
      s.parallel[k] = false;
      s.inv[k] = std::fabs(r.d[k]) < T(1e-8) ? std::copysign(T(1e30f), r.d[k]) : T(1) / r.d[k];
    } else {
      // The reference's form (wide_ray / wide_node_hit, main.swift:1758-1779).
      s.parallel[k] = std::fabs(r.d[k]) < T(1e-8);
      s.inv[k] = T(1) / (s.parallel[k] ? T(1) : r.d[k]);
    }
  }
  return s;
}

template <typename T> SlabRay<T> make_slab(const TraceRay<T> &r, T rootMax) {
  // fp64 needs no enlargement for its own rounding but keeps the fp32 one (it is conservative).
  return make_slab_e(r, T(1.1920929e-6) * (max_abs_origin(r) + rootMax));
}

inline uint32_t ord32(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Near-to-far order of the hit children. fp32 (the CUDA kernels' order): keys ord32(entry + 0)
// with the two low bits replaced by the slot, sorted ascending; a child is skipped when
// (key & ~3) > ord32(closest + 0). fp64: the reference's stable insertion sort on the entry
// distance (wide_order, main.swift:1780-1785), skipped when the entry exceeds the closest hit.
template <typename T> struct ChildOrder {
  int order[4];
  uint32_t key[4];
  T dist[4];
  int m = 0;
  ChildOrder(int mask, const T nearT[4]) {
    if (std::is_same<T, float>::value) {
      for (int k = 0; k < 4; ++k) {
        if (!(mask >> k & 1)) continue;
        const float z = float(nearT[k]) + 0.0f;
        key[m] = (ord32(z) & ~3u) | (uint32_t)k;
        ++m;
      }
      std::sort(key, key + m);
      for (int j = 0; j < m; ++j) order[j] = key[j] & 3u;
    } else {
      for (int k = 0; k < 4; ++k) {
        if (!(mask >> k & 1)) continue;
        int j = m++;
        while (j > 0 && dist[j - 1] > nearT[k]) { dist[j] = dist[j - 1]; order[j] = order[j - 1]; --j; }
        dist[j] = nearT[k];
        order[j] = k;
      }
    }
  }
  bool beyond(int j, T closest) const {
    if (std::is_same<T, float>::value) return (key[j] & ~3u) > ord32(float(closest) + 0.0f);
    return dist[j] > closest;
  }
};

template <typename T>
int node_hits(const vt_wide_node &n, const SlabRay<T> &w, T tMin, T tMax, T nearT[4]) {
  int mask = 0;
  const float *lo[3] = {n.lox, n.loy, n.loz}, *hi[3] = {n.hix, n.hiy, n.hiz};
  for (int k = 0; k < 4; ++k) {
    if (n.child[k] == 0) continue;
    T nt = tMin, ft = tMax;
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
      if (w.parallel[a]) {
        if (w.low[a] < T(lo[a][k]) || w.high[a] > T(hi[a][k])) ok = false;
        continue;
      }
      T x = (T(lo[a][k]) - w.low[a]) * w.inv[a], y = (T(hi[a][k]) - w.high[a]) * w.inv[a];
      // Plain comparisons (no NaN can arise: every operand is finite).
      T mn = x < y ? x : y, mx = x < y ? y : x;
      nt = nt < mn ? mn : nt;
      ft = ft < mx ? ft : mx;
    }
    nearT[k] = nt;
    if (ok && nt <= ft) mask |= 1 << k;
  }
  return mask;
}

// ---- quantised nodes: the CUDA traversal's node copy and its conservative box test ------------------
// Spec (restated from the CUDA build): per node, p = the children's union lower corner; per axis the
// smallest e in [-126, 127] with 255 2^e >= (hi - p); per child qlo = floor((lo - p) / 2^e) and
// qhi = ceil((hi - p) / 2^e), clamped to [0, 255], all in double, e in [-126, 112]. Words: p.xyz,
// biased exponents, qlo.xyz, qhi.xyz (byte k = child k), child[4], 4-bit leaf counts, 0.
int quant_exponent(double extent) {
  if (!(extent > 0.0)) return -126;
  int e;
  std::frexp(extent, &e);
  e = std::min(112, std::max(-126, e - 8));
  while (e < 112 && std::ldexp(255.0, e) < extent) ++e;
  while (e > -126 && std::ldexp(255.0, e - 1) >= extent) --e;
  return e;
}

uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

void quantize_nodes(vto_bvh &h) {
  h.qnodes.assign(h.nodes.size(), {});
  for (size_t i = 0; i < h.nodes.size(); ++i) {
    const vt_wide_node &nd = h.nodes[i];
    std::array<uint32_t, 16> &q = h.qnodes[i];
    const float *clo[3] = {nd.lox, nd.loy, nd.loz}, *chi[3] = {nd.hix, nd.hiy, nd.hiz};
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    bool any = false;
    for (int k = 0; k < 4; ++k) {
      if (nd.child[k] == 0) continue;
      any = true;
      for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], clo[a][k]); hi[a] = std::max(hi[a], chi[a][k]); }
    }
    if (any) {
      for (int a = 0; a < 3; ++a) {
        const float p = lo[a];
        const int e = quant_exponent(double(hi[a]) - double(p));
        q[a] = fbits(p);
        q[3] |= uint32_t(e + 127) << (8 * a);
        for (int k = 0; k < 4; ++k) {
          if (nd.child[k] == 0) continue;
          const double l = std::floor(std::ldexp(double(clo[a][k]) - double(p), -e));
          const double u = std::ceil(std::ldexp(double(chi[a][k]) - double(p), -e));
          q[4 + a] |= uint32_t(std::min(std::max(l, 0.0), 255.0)) << (8 * k);
          q[7 + a] |= uint32_t(std::min(std::max(u, 0.0), 255.0)) << (8 * k);
        }
      }
    }
    for (int k = 0; k < 4; ++k) {
      q[10 + k] = uint32_t(nd.child[k]);
      q[14] |= (uint32_t(nd.count[k]) & 15u) << (4 * k);
    }
  }
}

// Directed rounding of a float FMA / product, from the round-to-nearest result and an exact
// double-double of the real value (no floating-point environment changes).
inline void two_sum(double a, double b, double &s, double &e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
// An overflowed result rounds to the largest finite value on the side it is rounded toward.
inline float overflowed(float s, bool up) {
  if (s == INFINITY && !up) return FLT_MAX;
  if (s == -INFINITY && up) return -FLT_MAX;
  return s;
}
inline float fma_dir(float a, float b, float c, bool up) {
  const float s = std::fmaf(a, b, c);
  if (!std::isfinite(s)) return std::isfinite(a) && std::isfinite(b) && std::isfinite(c) ? overflowed(s, up) : s;
  double hi, lo;
  two_sum(double(a) * double(b), double(c), hi, lo);
  const double d = double(s) - hi;  // exact: s and hi agree to within a float ulp
  if (up) return d < lo ? std::nextafter(s, INFINITY) : s;
  return d > lo ? std::nextafter(s, -INFINITY) : s;
}
inline float mul_dir(float a, float b, bool up) {
  const float s = a * b;
  if (!std::isfinite(s)) return std::isfinite(a) && std::isfinite(b) ? overflowed(s, up) : s;
  const double v = double(a) * double(b);
  if (up) return double(s) < v ? std::nextafter(s, INFINITY) : s;
  return double(s) > v ? std::nextafter(s, -INFINITY) : s;
}

struct QRayO {
  float inv[3], n[3], f[3];
  bool neg[3];
};
QRayO make_qray_o(const SlabRay<float> &s) {
  QRayO q;
  for (int a = 0; a < 3; ++a) {
    q.inv[a] = s.inv[a];
    q.neg[a] = s.inv[a] < 0.0f;
    q.n[a] = mul_dir(q.neg[a] ? s.high[a] : s.low[a], s.inv[a], true);
    q.f[a] = mul_dir(q.neg[a] ? s.low[a] : s.high[a], s.inv[a], false);
  }
  return q;
}

// The CUDA kernels' quantised child test (qnode_hits): lower bounds of near and upper bounds of
// far plane distances.
int qnode_hits_o(const std::array<uint32_t, 16> &q, const QRayO &r, float tMin, float tMax, float nearT[4]) {
  float d[3], cn[3], cf[3];
  uint32_t nw[3], fw[3];
  for (int a = 0; a < 3; ++a) {
    const float p = bitsf(q[a]);
    d[a] = bitsf((((q[3] >> (8 * a)) & 0xffu) + 15u) << 23) * r.inv[a];
    cn[a] = fma_dir(1.0f, fma_dir(p, r.inv[a], -r.n[a], false), -d[a], false);
    cf[a] = fma_dir(1.0f, fma_dir(p, r.inv[a], -r.f[a], true), -d[a], true);
    nw[a] = r.neg[a] ? q[7 + a] : q[4 + a];
    fw[a] = r.neg[a] ? q[4 + a] : q[7 + a];
  }
  int mask = 0;
  for (int k = 0; k < 4; ++k) {
    float nt[3], ft[3];
    for (int a = 0; a < 3; ++a) {
      nt[a] = fma_dir(bitsf(0x3F800000u | (((nw[a] >> (8 * k)) & 0xffu) << 8)), d[a], cn[a], false);
      ft[a] = fma_dir(bitsf(0x3F800000u | (((fw[a] >> (8 * k)) & 0xffu) << 8)), d[a], cf[a], true);
    }
    const float n0 = std::fmax(std::fmax(nt[0], nt[1]), std::fmax(nt[2], tMin));
    const float f0 = std::fmin(std::fmin(ft[0], ft[1]), std::fmin(ft[2], tMax));
    nearT[k] = n0;
    if (n0 <= f0 && q[10 + k] != 0u) mask |= 1 << k;
  }
  return mask;
}

template <typename T>
bool closest_hit(const vto_bvh &h, const TraceRay<T> &r, T &best, int &prim, T &hb1, T &hb2,
                 uint64_t *nodes = nullptr, uint64_t *tests = nullptr) {
  if (h.nodes.empty()) return false;
  WRay<T> w = make_wray(r.o, r.d);
  SlabRay<T> s = make_slab(r, T(h.root_max));
  T closest = r.tmax;
  bool found = false;
  int stack[160];
  int top = 0;
  stack[top++] = 0;
  if constexpr (std::is_same<T, float>::value) {
    // The CUDA kernels' order and node test: quantised nodes; leaf children are stack entries
    // ~(node << 2 | slot), pushed with the inner children far to near, so a ray pops its entries
    // near first.
    const QRayO qr = make_qray_o(s);
    while (top > 0) {
      const int entry = stack[--top];
      if (entry < 0) {
        const int code = ~entry;
        const vt_wide_node &ln = h.nodes[code >> 2];
        const int first = -ln.child[code & 3] - 1, cnt = ln.count[code & 3];
        for (int q = 0; q < cnt; ++q) {
          const float *tf = &h.tris[9 * (size_t)(first + q)];
          T a[3] = {T(tf[0]), T(tf[1]), T(tf[2])}, b[3] = {T(tf[3]), T(tf[4]), T(tf[5])},
            c[3] = {T(tf[6]), T(tf[7]), T(tf[8])};
          T t, b1, b2;
          if (tests) ++*tests;
          if (!intersect_tri<T>(w, a, b, c, r.tmin, closest, t, b1, b2)) continue;
          closest = t; prim = h.order[first + q]; hb1 = b1; hb2 = b2; found = true;
        }
        continue;
      }
      const vt_wide_node &nd = h.nodes[entry];
      if (nodes) ++*nodes;
      T nearT[4];
      const int mask = qnode_hits_o(h.qnodes[entry], qr, r.tmin, closest, nearT);
      const ChildOrder<T> co(mask, nearT);
      for (int j = co.m - 1; j >= 0; --j) {
        const int k = co.order[j];
        if (co.beyond(j, closest) || top >= 160) continue;
        stack[top++] = nd.child[k] > 0 ? nd.child[k] : ~((entry << 2) | k);
      }
    }
    best = closest;
    return found;
  }
  while (top > 0) {
    const vt_wide_node &nd = h.nodes[stack[--top]];
    if (nodes) ++*nodes;
    T nearT[4];
    int mask = node_hits(nd, s, r.tmin, closest, nearT);
    const ChildOrder<T> co(mask, nearT);
    const int m = co.m;
    for (int j = 0; j < m; ++j) {
      int k = co.order[j];
      if (nd.child[k] > 0 || co.beyond(j, closest)) continue;
      int first = -nd.child[k] - 1;
      for (int q = 0; q < nd.count[k]; ++q) {
        const float *tf = &h.tris[9 * (size_t)(first + q)];
        T a[3] = {T(tf[0]), T(tf[1]), T(tf[2])}, b[3] = {T(tf[3]), T(tf[4]), T(tf[5])},
          c[3] = {T(tf[6]), T(tf[7]), T(tf[8])};
        T t, b1, b2;
        if (tests) ++*tests;
        if (!intersect_tri<T>(w, a, b, c, r.tmin, closest, t, b1, b2)) continue;
        closest = t; prim = h.order[first + q]; hb1 = b1; hb2 = b2; found = true;
      }
    }
    for (int j = m - 1; j >= 0; --j) {
      int k = co.order[j];
      if (nd.child[k] > 0 && !co.beyond(j, closest) && top < 160) stack[top++] = nd.child[k];
    }
  }
  best = closest;
  return found;
}

template <typename T>
bool any_hit(const vto_bvh &h, const TraceRay<T> &r, uint64_t *nodes = nullptr, uint64_t *tests = nullptr,
             bool slack = false) {
  if (h.nodes.empty()) return false;
  WRay<T> w = make_wray(r.o, r.d);
  SlabRay<T> s = make_slab(r, T(h.root_max));
  int stack[160];
  int top = 0;
  stack[top++] = 0;
  if constexpr (std::is_same<T, float>::value) {
   if (!slack) {
    // The CUDA kernels' order and node test: quantised nodes; leaf children are stack entries,
    // pushed with the inner children from slot 3 down to slot 0.
    const QRayO qr = make_qray_o(s);
    while (top > 0) {
      const int entry = stack[--top];
      if (entry < 0) {
        const int code = ~entry;
        const vt_wide_node &ln = h.nodes[code >> 2];
        const int first = -ln.child[code & 3] - 1, cnt = ln.count[code & 3];
        for (int q = 0; q < cnt; ++q) {
          const float *tf = &h.tris[9 * (size_t)(first + q)];
          T a[3] = {T(tf[0]), T(tf[1]), T(tf[2])}, b[3] = {T(tf[3]), T(tf[4]), T(tf[5])},
            c[3] = {T(tf[6]), T(tf[7]), T(tf[8])};
          T t, b1, b2;
          if (tests) ++*tests;
          if (intersect_tri<T>(w, a, b, c, r.tmin, r.tmax, t, b1, b2)) return true;
        }
        continue;
      }
      const vt_wide_node &nd = h.nodes[entry];
      if (nodes) ++*nodes;
      T nearT[4];
      const int mask = qnode_hits_o(h.qnodes[entry], qr, r.tmin, r.tmax, nearT);
      for (int k = 3; k >= 0; --k) {
        if (!(mask >> k & 1) || top >= 160) continue;
        stack[top++] = nd.child[k] > 0 ? nd.child[k] : ~((entry << 2) | k);
      }
    }
    return false;
   }
  }
  while (top > 0) {
    const vt_wide_node &nd = h.nodes[stack[--top]];
    if (nodes) ++*nodes;
    T nearT[4];
    int mask = node_hits(nd, s, r.tmin, r.tmax, nearT);
    for (int k = 0; k < 4; ++k) {
      if (!(mask >> k & 1)) continue;
      if (nd.child[k] > 0) { if (top < 160) stack[top++] = nd.child[k]; continue; }
      int first = -nd.child[k] - 1;
      for (int q = 0; q < nd.count[k]; ++q) {
        const float *tf = &h.tris[9 * (size_t)(first + q)];
        T a[3] = {T(tf[0]), T(tf[1]), T(tf[2])}, b[3] = {T(tf[3]), T(tf[4]), T(tf[5])},
          c[3] = {T(tf[6]), T(tf[7]), T(tf[8])};
        T t, b1, b2;
        if (tests) ++*tests;
        // Imported scenes take each triangle's rounding bound off tMax (scene_occluded,
        // main.swift:2066-2069; mesh_hit_error, :1353-1355).
        T tmax = r.tmax;
        if (slack) {
          T m = 0;
          for (int k = 0; k < 3; ++k) m = std::max(m, std::max(std::fabs(a[k]), std::max(std::fabs(b[k]), std::fabs(c[k]))));
          tmax = r.tmax - std::max(T(1e-7), T(1.907349e-6) * m);
        }
        if (intersect_tri<T>(w, a, b, c, r.tmin, tmax, t, b1, b2)) return true;
      }
    }
  }
  return false;
}

// ---- two-level traversal (mesh_closest / mesh_occluded, main.swift:1840-1984) ----------------------
// The TLAS (128-byte nodes whose leaves name instances: -(instance + 1)) with boxes grown per ray by
// grow (max|origin| + reach); each instance traced in object space with instance_ray
// (main.swift:1634-1637), the direction not renormalised. fp32: the CUDA kernel's order and
// arithmetic (o'_r = fma(l.z, o.z, fma(l.y, o.y, l.x o.x)) + l.w; quantised BLAS nodes); fp64: the
// reference's form in double on the same float records.
template <typename T> TraceRay<T> instance_ray(const vt_instance_record &I, const TraceRay<T> &r) {
  TraceRay<T> o;
  for (int a = 0; a < 3; ++a) {
    const float *l = I.local + 4 * a;
    if constexpr (std::is_same<T, float>::value) {
      o.o[a] = std::fma(l[2], r.o[2], std::fma(l[1], r.o[1], l[0] * r.o[0])) + l[3];
      o.d[a] = std::fma(l[2], r.d[2], std::fma(l[1], r.d[1], l[0] * r.d[0]));
    } else {
      o.o[a] = T(l[0]) * r.o[0] + T(l[1]) * r.o[1] + T(l[2]) * r.o[2] + T(l[3]);
      o.d[a] = T(l[0]) * r.d[0] + T(l[1]) * r.d[1] + T(l[2]) * r.d[2];
    }
  }
  o.tmin = r.tmin;
  o.tmax = r.tmax;
  return o;
}

struct TlasView {
  const vt_wide_node *nodes;
  const vt_instance_record *inst;
  const vto_bvh *const *meshes;
  float grow, reach;
};

template <typename T>
bool tlas_closest(const TlasView &V, const TraceRay<T> &r, T &best, int &prim, uint32_t &inst, T &hb1, T &hb2) {
  const SlabRay<T> s = make_slab_e(r, T(V.grow) * (max_abs_origin(r) + T(V.reach)));
  T closest = r.tmax;
  bool found = false;
  int stack[32];
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    const vt_wide_node &nd = V.nodes[stack[--top]];
    T nearT[4];
    const int mask = node_hits(nd, s, r.tmin, closest, nearT);
    const ChildOrder<T> co(mask, nearT);
    for (int j = 0; j < co.m; ++j) {
      const int k = co.order[j];
      if (nd.child[k] > 0 || co.beyond(j, closest)) continue;
      const uint32_t i = (uint32_t)(-nd.child[k] - 1);
      const vt_instance_record &I = V.inst[i];
      TraceRay<T> lr = instance_ray(I, r);
      lr.tmax = closest;
      T t, b1 = 0, b2 = 0;
      int p = -1;
      if (closest_hit<T>(*V.meshes[I.mesh], lr, t, p, b1, b2)) {
        closest = t; prim = p; inst = i; hb1 = b1; hb2 = b2; found = true;
      }
    }
    for (int j = co.m - 1; j >= 0; --j) {
      const int k = co.order[j];
      if (nd.child[k] > 0 && !co.beyond(j, closest) && top < 32) stack[top++] = nd.child[k];
    }
  }
  best = closest;
  return found;
}

template <typename T> bool tlas_any(const TlasView &V, const TraceRay<T> &r) {
  const SlabRay<T> s = make_slab_e(r, T(V.grow) * (max_abs_origin(r) + T(V.reach)));
  int stack[32];
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    const vt_wide_node &nd = V.nodes[stack[--top]];
    T nearT[4];
    const int mask = node_hits(nd, s, r.tmin, r.tmax, nearT);
    for (int k = 0; k < 4; ++k) {
      if (!(mask >> k & 1)) continue;
      if (nd.child[k] > 0) {
        if (top < 32) stack[top++] = nd.child[k];
        continue;
      }
      const vt_instance_record &I = V.inst[-nd.child[k] - 1];
      if (any_hit<T>(*V.meshes[I.mesh], instance_ray(I, r))) return true;
    }
  }
  return false;
}

template <typename T> TraceRay<T> load_ray(const vt_ray &r) {
  TraceRay<T> x;
  x.o[0] = r.ox; x.o[1] = r.oy; x.o[2] = r.oz;
  x.d[0] = r.dx; x.d[1] = r.dy; x.d[2] = r.dz;
  x.tmin = r.tmin; x.tmax = r.tmax;
  return x;
}

template <typename F> void parallel_for(uint32_t n, int threads, F f) {
  if (threads <= 1 || n < 2048) { for (uint32_t i = 0; i < n; ++i) f(i); return; }
  std::atomic<uint32_t> next{0};
  const uint32_t chunk = 512;
  auto worker = [&]() {
    for (uint32_t s; (s = next.fetch_add(chunk)) < n;) {
      uint32_t e = std::min(n, s + chunk);
      for (uint32_t i = s; i < e; ++i) f(i);
    }
  };
  std::vector<std::thread> pool;
  for (int i = 0; i < threads; ++i) pool.emplace_back(worker);
  for (auto &t : pool) t.join();
}

}  // namespace

extern "C" {

void vto_trace_closest(const vto_bvh *h, const vt_ray *rays, uint32_t n, vt_hit *hits,
                       int32_t precision, int32_t threads) {
  parallel_for(n, threads, [&](uint32_t i) {
    vt_hit out{0.0f, 0.0f, 0.0f, -1};
    int prim = -1;
    if (precision == 64) {
      TraceRay<double> r = load_ray<double>(rays[i]);
      double t, b1 = 0, b2 = 0;
      if (closest_hit<double>(*h, r, t, prim, b1, b2)) out = {float(t), float(b1), float(b2), prim};
    } else {
      TraceRay<float> r = load_ray<float>(rays[i]);
      float t, b1 = 0, b2 = 0;
      if (closest_hit<float>(*h, r, t, prim, b1, b2)) out = {t, b1, b2, prim};
    }
    hits[i] = out;
  });
}

void vto_trace_any(const vto_bvh *h, const vt_ray *rays, uint32_t n, uint8_t *occluded,
                   int32_t precision, int32_t threads) {
  parallel_for(n, threads, [&](uint32_t i) {
    bool hit = precision == 64 ? any_hit<double>(*h, load_ray<double>(rays[i]))
                               : any_hit<float>(*h, load_ray<float>(rays[i]));
    occluded[i] = hit ? 1 : 0;
  });
}

void vto_brute_closest(const vt_face *faces, uint32_t nfaces, const vt_vertex *verts,
                       const vt_ray *rays, uint32_t n, vt_hit *hits, int32_t precision,
                       int32_t threads) {
  parallel_for(n, threads, [&](uint32_t i) {
    vt_hit out{0.0f, 0.0f, 0.0f, -1};
    if (precision == 64) {
      TraceRay<double> r = load_ray<double>(rays[i]);
      WRay<double> w = make_wray(r.o, r.d);
      double best = r.tmax;
      for (uint32_t f = 0; f < nfaces; ++f) {
        const vt_vertex *p[3] = {&verts[faces[f].a], &verts[faces[f].b], &verts[faces[f].c]};
        double a[3] = {p[0]->px, p[0]->py, p[0]->pz}, b[3] = {p[1]->px, p[1]->py, p[1]->pz},
               c[3] = {p[2]->px, p[2]->py, p[2]->pz};
        double t, b1, b2;
        if (intersect_tri<double>(w, a, b, c, r.tmin, best, t, b1, b2)) { best = t; out = {float(t), float(b1), float(b2), int32_t(f)}; }
      }
    } else {
      TraceRay<float> r = load_ray<float>(rays[i]);
      WRay<float> w = make_wray(r.o, r.d);
      float best = r.tmax;
      for (uint32_t f = 0; f < nfaces; ++f) {
        const vt_vertex *p[3] = {&verts[faces[f].a], &verts[faces[f].b], &verts[faces[f].c]};
        float a[3] = {p[0]->px, p[0]->py, p[0]->pz}, b[3] = {p[1]->px, p[1]->py, p[1]->pz},
              c[3] = {p[2]->px, p[2]->py, p[2]->pz};
        float t, b1, b2;
        if (intersect_tri<float>(w, a, b, c, r.tmin, best, t, b1, b2)) { best = t; out = {t, b1, b2, int32_t(f)}; }
      }
    }
    hits[i] = out;
  });
}

void vto_tlas_trace(const vt_wide_node *nodes, const vt_instance_record *inst, const vto_bvh *const *meshes,
                    float grow, float reach, const vt_ray *rays, uint32_t n, vt_hit *hits, uint32_t *instances,
                    uint8_t *occluded, int32_t closest, int32_t precision, int32_t threads) {
  const TlasView V{nodes, inst, meshes, grow, reach};
  parallel_for(n, threads, [&](uint32_t i) {
    if (!closest) {
      const bool hit = precision == 64 ? tlas_any<double>(V, load_ray<double>(rays[i])) : tlas_any<float>(V, load_ray<float>(rays[i]));
      occluded[i] = hit ? 1 : 0;
      return;
    }
    vt_hit out{0.0f, 0.0f, 0.0f, -1};
    int prim = -1;
    uint32_t k = 0xffffffffu;
    if (precision == 64) {
      double t, b1 = 0, b2 = 0;
      if (tlas_closest<double>(V, load_ray<double>(rays[i]), t, prim, k, b1, b2)) out = {float(t), float(b1), float(b2), prim};
    } else {
      float t, b1 = 0, b2 = 0;
      if (tlas_closest<float>(V, load_ray<float>(rays[i]), t, prim, k, b1, b2)) out = {t, b1, b2, prim};
    }
    hits[i] = out;
    if (instances) instances[i] = out.prim >= 0 ? k : 0xffffffffu;
  });
}

void vto_trace_count(const vto_bvh *h, const vt_ray *rays, uint32_t n, int32_t closest,
                     uint64_t *nodes_visited, uint64_t *tris_tested, int32_t threads) {
  std::atomic<uint64_t> nv{0}, tt{0};
  parallel_for(n, threads, [&](uint32_t i) {
    uint64_t a = 0, b = 0;
    TraceRay<float> r = load_ray<float>(rays[i]);
    if (closest) { float t, b1 = 0, b2 = 0; int p = -1; closest_hit<float>(*h, r, t, p, b1, b2, &a, &b); }
    else any_hit<float>(*h, r, &a, &b);
    nv += a; tt += b;
  });
  *nodes_visited = nv;
  *tris_tested = tt;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Z++ sampler (main.swift:122-305, 497-515), restated: per-pixel keys from a shuffled Morton code
// and a temporal index, sampling events of 32 dimensions, van der Corput / Sobol' / O2m3
// constituents under Owen scrambling, frame offsets from the pixel's own sequence. Integer
// arithmetic throughout: every draw equals the GPU's bit for bit.
namespace {

inline uint32_t rev32(uint32_t v) {
  v = ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
  v = ((v >> 2) & 0x33333333u) | ((v & 0x33333333u) << 2);
  v = ((v >> 4) & 0x0F0F0F0Fu) | ((v & 0x0F0F0F0Fu) << 4);
  v = ((v >> 8) & 0x00FF00FFu) | ((v & 0x00FF00FFu) << 8);
  return (v >> 16) | (v << 16);
}
inline uint32_t zmix(uint32_t v) {
  v ^= v >> 16; v *= 0x7feb352du; v ^= v >> 15; v *= 0x846ca68bu; v ^= v >> 16;
  return v;
}
const uint64_t kZPerm = 0x6c9c78d8b4e4ull;
uint32_t zshuffle(uint32_t index, uint32_t dimension) {
  const uint32_t seed = zmix(dimension * 0x9e3779b9u + 0x632be5abu);
  uint32_t result = index & ~((1u << 24) - 1u);
  for (int d = 11; d >= 0; --d) {
    const uint32_t shift = 2u * d, digit = (index >> shift) & 3u;
    const uint32_t h = zmix((index >> (shift + 2u)) ^ seed);
    const uint32_t sigma = ((h >> 16) * 6u) >> 16;
    const uint32_t image = (uint32_t)(kZPerm >> (8u * sigma + 2u * digit)) & 3u;
    result |= (image ^ (h & 3u)) << shift;
  }
  return result;
}
uint32_t zowen(uint32_t v, uint32_t seed) {
  v = rev32(v);
  v ^= v * 0x3d20adeau;
  v += seed;
  v *= (seed >> 16) | 1u;
  v ^= v * 0x05526c56u;
  v ^= v * 0x53a22864u;
  return rev32(v);
}
uint32_t zowen_seed(uint32_t dimension, uint32_t axis) {
  const uint32_t h = (dimension ^ (axis << 24)) * 0x9e3779b9u;
  return (h ^ (h >> 16)) * 0x85ebca6bu;
}
uint32_t zsobol1(uint32_t i) {
  i ^= (i & 0xAAAAAAAAu) >> 1; i ^= (i & 0xCCCCCCCCu) >> 2; i ^= (i & 0xF0F0F0F0u) >> 4;
  i ^= (i & 0xFF00FF00u) >> 8; i ^= (i & 0xFFFF0000u) >> 16;
  return rev32(i);
}
uint32_t zo2m3x(uint32_t V) {
  V ^= ((V << 2) & 0xF3CF3CF3u) ^ ((V << 3) & 0x41041041u);
  V ^= (V << 4) & 0x3F03F03Fu;
  V ^= (V << 8) & 0x0FFF000Fu;
  V ^= (V << 16) & 0x00FFFFFFu;
  return V;
}
uint32_t zo2m3y(uint32_t V) { return zo2m3x(((V >> 1) & 0x45145145u) ^ (V & 0xB5EB5EB5u) ^ ((V << 1) & 0x8A28A28Au)); }
uint32_t zo2m3z(uint32_t V) { return zo2m3x(((V >> 1) & 0x45145145u) ^ (V & 0x7AD7AD7Au) ^ ((V << 1) & 0x8A28A28Au)); }
inline double zfloat(uint32_t v) { return double(v >> 8) * (1.0 / 16777216.0); }
uint32_t zmorton(uint32_t x, uint32_t y) {
  auto spread = [](uint32_t v) {
    v &= 0xFFFFu;
    v = (v | (v << 8)) & 0x00FF00FFu; v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u; v = (v | (v << 1)) & 0x55555555u;
    return v;
  };
  return spread(x) | (spread(y) << 1);
}

struct ZSampler {
  uint32_t state = 0, key = 0, dimension = 0, sub = 0, subBits = 0;
  bool z = false;

  static ZSampler pixel(uint32_t x, uint32_t y, uint32_t width, uint32_t sampleIndex, bool z, uint32_t model,
                        uint32_t frameIndex) {
    ZSampler s;
    s.state = (y * width + x) ^ (sampleIndex * 1999999973u);
    s.z = z;
    if (z) {
      const uint32_t j = std::max(frameIndex, 1u) - 1u, s0 = sampleIndex - j;
      uint32_t t = model == 1u || model == 2u ? s0 ^ ((s0 & 0xAAAAAAAAu) << 1) : model == 3u ? zmix(s0 ^ 0x2c1b3c6du) : s0;
      uint32_t k = zshuffle(zmorton(x, y), 0xffffffffu);
      if (model == 2u) k ^= k << 2;
      if ((j >> 14) != 0u) t ^= zmix(j >> 14);
      s.key = ((k ^ t) << 14) | (j & 0x3FFFu);
    }
    return s;
  }
  uint32_t code() const { return key >> 14; }
  uint32_t frame() const { return ((key & 0x3FFFu) << subBits) | sub; }
  uint32_t index(uint32_t d) const { return zowen(code(), zowen_seed(d, 3u)); }
  uint32_t next_dimension() { return dimension++ | ((code() >> 12) << 17); }
  static uint32_t frame_index(uint32_t J, uint32_t d) {
    const uint32_t seed = zowen_seed(d, 4u);
    return zowen(J, seed) ^ zowen(0u, seed);
  }
  uint32_t frame_offset(uint32_t v, uint32_t d, uint32_t axis) const {
    const uint32_t seed = zowen_seed(d, axis) ^ zmix(code() ^ 0x68e31da4u);
    return ((zowen(v, seed) ^ zowen(0u, seed)) & 0x3FFFFFFFu) | (v & 0xC0000000u);
  }
  double pcg() { state = pcg_hash(state); return double(state >> 8u) * (1.0 / 16777216.0); }
  double f1() {
    if (!z) return pcg();
    const uint32_t d = next_dimension(), J = frame();
    uint32_t x = zowen(rev32(index(d)), zowen_seed(d, 0u));
    if (J) x ^= frame_offset(rev32(frame_index(J, d)), d, 0u);
    return zfloat(x);
  }
  void f2(double &a, double &b) {
    if (!z) { a = pcg(); b = pcg(); return; }
    const uint32_t d = next_dimension(), i = index(d), J = frame();
    uint32_t x = zowen(rev32(i), zowen_seed(d, 0u)), y = zowen(zsobol1(i), zowen_seed(d, 1u));
    if (J) {
      const uint32_t k = frame_index(J, d);
      x ^= frame_offset(rev32(k), d, 0u);
      y ^= frame_offset(zsobol1(k), d, 1u);
    }
    a = zfloat(x); b = zfloat(y);
  }
  void f3(double &a, double &b, double &c) {
    if (!z) { a = pcg(); b = pcg(); c = pcg(); return; }
    const uint32_t d = next_dimension(), V = rev32(index(d)), J = frame();
    uint32_t x = zowen(zo2m3x(V), zowen_seed(d, 0u)), y = zowen(zo2m3y(V), zowen_seed(d, 1u)), w = zowen(zo2m3z(V), zowen_seed(d, 2u));
    if (J) {
      const uint32_t W = rev32(frame_index(J, d));
      x ^= frame_offset(zo2m3x(W), d, 0u);
      y ^= frame_offset(zo2m3y(W), d, 1u);
      w ^= frame_offset(zo2m3z(W), d, 2u);
    }
    a = zfloat(x); b = zfloat(y); c = zfloat(w);
  }
  void event(uint32_t vertex, uint32_t stream) { dimension = (vertex * 16u + stream) * 32u; sub = 0u; subBits = 0u; }
  // sampler_candidate (main.swift:296-298) and rand_decision (main.swift:117, 280).
  void candidate(uint32_t vertex, uint32_t stream, uint32_t index, uint32_t bits) {
    event(vertex, stream);
    if (z) { sub = index; subBits = bits; }
  }
  double decision() { return pcg(); }
  // wavelength_numbers: from a copy.
  double wavelength_u() const {
    if (z) { ZSampler c = *this; c.event(0u, 12u); return c.f1(); }
    const uint32_t h = pcg_hash(state ^ 0x5bd1e995u);
    return double(h >> 8u) * (1.0 / 16777216.0);
  }
};

}  // namespace

extern "C" {
void vto_z_sequences(uint32_t seed, uint32_t n, uint32_t *o2m3, uint32_t *sobol) {
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t V = rev32(i);
    uint32_t p[3] = {zo2m3x(V), zo2m3y(V), zo2m3z(V)}, q[2] = {V, zsobol1(i)};
    if (seed) {
      for (int a = 0; a < 3; ++a) p[a] = zowen(p[a], zowen_seed(seed, a));
      for (int a = 0; a < 2; ++a) q[a] = zowen(q[a], zowen_seed(seed, a));
    }
    for (int a = 0; a < 3; ++a) o2m3[3 * i + a] = p[a];
    for (int a = 0; a < 2; ++a) sobol[2 * i + a] = q[a];
  }
}
void vto_z_shuffles(uint32_t base, uint32_t dimension, uint32_t n, uint32_t *out) {
  for (uint32_t i = 0; i < n; ++i) out[i] = zshuffle(base + i, dimension);
}
// Per pixel: rand_f, rand_f2 and rand_f3 of one sampling event (vertex, stream).
void vto_sampler_frame(uint32_t width, uint32_t height, int32_t z, uint32_t model, uint32_t sampleIndex,
                       uint32_t frameIndex, uint32_t vertex, uint32_t stream, float *out) {
  for (uint32_t y = 0; y < height; ++y)
    for (uint32_t x = 0; x < width; ++x) {
      ZSampler s = ZSampler::pixel(x, y, width, sampleIndex, z != 0, model, frameIndex);
      s.event(vertex, stream);
      double v[6];
      v[0] = s.f1();
      s.f2(v[1], v[2]);
      s.f3(v[3], v[4], v[5]);
      for (int k = 0; k < 6; ++k) out[6 * ((size_t)y * width + x) + k] = (float)v[k];
    }
}
}  // extern "C"

// ------------------------------------------------------------------------------------------
// Path tracer: FP64 restatement of the MIS integrator (shading_kernel, main.swift:7370-7914, with
// the primary hit of restir_temporal_kernel, main.swift:4842-4893), PCG sampler. The stream
// consumption order is the reference's: wavelength numbers from a hashed copy
// (wavelength_numbers, main.swift:2222-2231), decorrelate_shading_seed (main.swift:109-111)
// after the camera ray, then per vertex NEE (2 draws, main.swift:2957-2978), Lambert sampling
// (3 draws, the last two used, main.swift:3354-3360) and, after bounce 3, Russian roulette
// (1 draw, main.swift:7819-7827).
namespace {

struct D3 { double x, y, z; };
inline D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline D3 normalize(D3 a) { return a * (1.0 / std::sqrt(dot(a, a))); }
inline D3 d3(const float *v) { return {v[0], v[1], v[2]}; }

const double kPi = 3.14159265358979323846;
const double kEpsPt = 0.001;  // ray_epsilon / ray_t_min of the procedural scenes


// frameJitter (main.swift:8773-8785) in float, as the host computes it.
float halton_f(uint32_t index, uint32_t base) {
  uint32_t n = index;
  float fraction = 1.0f, result = 0.0f;
  while (n > 0) {
    fraction /= float(base);
    result += fraction * float(n % base);
    n /= base;
  }
  return result;
}

struct Spec4 { double v[4]; };

struct PtContext {
  const vto_pt_inputs *in;
  const vt_frame_params *p;
  vto_bvh *bvh;
  D3 cam, fwd, right, up;
  double aspect, fovScale, larea;
  bool spectral;
  // Imported scenes: per slot (emission rgb, selection weight), the packed emitter list.
  bool imported = false;
  std::vector<std::array<double, 4>> emis;
  const uint32_t *E = nullptr;
  uint32_t ecount = 0, treeNodes = 0;
  double etotal = 0;
  const uint32_t *ltNodes = nullptr, *ltLeaves = nullptr;
  double ltLo[3] = {0, 0, 0}, ltScale[3] = {0, 0, 0};
  // Spectral uplift: materials carrying their slot in `pad`, per slot the albedo's multipliers,
  // per bin the emission basis (R, G, B, C, M, Y).
  std::vector<vt_material> mats;
  std::vector<std::array<double, 4>> slotL;
  std::vector<std::array<double, 6>> basis;
  // Imported scenes: the procedural sky and sun (vt_environment; the sun direction normalised as the
  // library does, in double and then stored as float).
  bool env = false;
  double envIntensity = 0, sunIntensity = 0;
  D3 sunDir{0, 1, 0};
  uint32_t skyMode = 0;
  // Environment image: pixels (4 floats each), size, rotation, and its sampling tables built here
  // (rows[2 y + table], cols[(table H + y) W + x]).
  bool envMap = false;
  const float *envImg = nullptr;
  uint32_t envW = 0, envH = 0;
  double envRot = 0;
  std::vector<double> envRows, envCols;
};

inline double fword(uint32_t w) { float f; std::memcpy(&f, &w, 4); return f; }
inline double max_abs_d(D3 p) { return std::max(std::fabs(p.x), std::max(std::fabs(p.y), std::fabs(p.z))); }
// ray_epsilon / ray_t_min (main.swift:1343-1345, 1362-1364).
inline double ray_eps_d(const PtContext &C, D3 p) { return C.imported ? std::max(1e-7, 9.536743e-7 * max_abs_d(p)) : kEpsPt; }
inline double ray_tmin_d(const PtContext &C, D3 o) { return C.imported ? ray_eps_d(C, o) * 0.25 : kEpsPt; }

struct PtLanes { int bin[4]; double w[4]; double lambda[4]; };

PtLanes make_lanes(const PtContext &C, double u) {
  PtLanes L;
  const uint32_t seg = C.in->segments;
  for (int k = 0; k < 4; ++k) {
    const double x = (u + k) * 0.25 * seg;
    const uint32_t i = std::min((uint32_t)x, seg - 1u);
    const double low = C.in->icdf[i], width = double(C.in->icdf[i + 1]) - low;
    L.w[k] = 0.25 * seg * width;
    const double lambda = low + (x - i) * width;
    L.lambda[k] = lambda;
    const double b = std::min(std::max(lambda - C.in->lambda_min + 0.5, 0.0), double(C.in->nbins - 1u));
    L.bin[k] = (int)std::min((uint32_t)b, C.in->nbins - 1u);
  }
  return L;
}

D3 to_rgb(const PtContext &C, const PtLanes &L, const Spec4 &s) {
  if (!C.spectral) return {s.v[0], s.v[1], s.v[2]};
  D3 rgb{0, 0, 0};
  for (int k = 0; k < 4; ++k) {
    const float *c = C.in->cmf_rgb + 3 * L.bin[k];
    const double a = s.v[k] * L.w[k];
    rgb = rgb + D3{a * c[0], a * c[1], a * c[2]};
  }
  return rgb;
}

// spectral_reflectance (main.swift:905-907) of the slot's albedo at the lanes' bins.
Spec4 reflectance(const PtContext &C, const PtLanes &L, const vt_material &m) {
  if (C.spectral) {
    uint32_t slot;
    std::memcpy(&slot, &m.pad, sizeof slot);
    if (slot >= C.slotL.size()) return {{0, 0, 0, 0}};
    Spec4 s;
    for (int k = 0; k < 4; ++k) s.v[k] = vto_uplift_impl::spectral_value(C.slotL[slot].data(), C.in->cos_phase[L.bin[k]]);
    return s;
  }
  return {{m.albedo[0], m.albedo[1], m.albedo[2], 0.0}};
}
// spectral_emission (main.swift:913-944): Smits' decomposition on the corners' spectra, times S.
Spec4 emission(const PtContext &C, const PtLanes &L, const float e[3]) {
  if (C.spectral) {
    Spec4 s{{0, 0, 0, 0}};
    if (!(std::max(e[0], std::max(e[1], e[2])) > 0.0f)) return s;
    const double ed[3] = {e[0], e[1], e[2]};
    const vto_uplift_impl::EmissionWeights w = vto_uplift_impl::emission_weights(ed);
    for (int k = 0; k < 4; ++k) {
      const std::array<double, 6> &b = C.basis[L.bin[k]];
      s.v[k] = (w.lo + w.secondary * b[3 + w.secondary_index] + w.primary * b[w.primary_index]) * C.in->illum[L.bin[k]];
    }
    return s;
  }
  return {{e[0], e[1], e[2], 0.0}};
}
inline Spec4 mul(const Spec4 &a, const Spec4 &b) { return {{a.v[0] * b.v[0], a.v[1] * b.v[1], a.v[2] * b.v[2], a.v[3] * b.v[3]}}; }
inline Spec4 scale(const Spec4 &a, double s) { return {{a.v[0] * s, a.v[1] * s, a.v[2] * s, a.v[3] * s}}; }
inline double smax(const PtContext &C, const Spec4 &a) {
  double m = std::max(std::max(a.v[0], a.v[1]), a.v[2]);
  return C.spectral ? std::max(m, a.v[3]) : m;
}

struct PtHit { D3 pos, gn, n, e1; double err, t; uint32_t slot, face; bool front; };  // e1: the edge b - a

struct PtTri { D3 a, b, c; uint32_t slot; };
PtTri pt_triangle(const PtContext &C, uint32_t face) {
  const vt_face &f = C.in->faces[face];
  return {d3(&C.in->verts[f.a].px), d3(&C.in->verts[f.b].px), d3(&C.in->verts[f.c].px), f.tag};
}
// mesh_hit_error (main.swift:1353-1355).
double mesh_hit_error_d(const PtTri &t) {
  return std::max(1e-7, 1.907349e-6 * std::max(max_abs_d(t.a), std::max(max_abs_d(t.b), max_abs_d(t.c))));
}

// The hit record: imported scenes rebuild the point from barycentrics (main.swift:2025-2028).
bool pt_closest(const PtContext &C, D3 o, D3 d, PtHit &h) {
  TraceRay<double> r;
  r.o[0] = o.x; r.o[1] = o.y; r.o[2] = o.z;
  r.d[0] = d.x; r.d[1] = d.y; r.d[2] = d.z;
  r.tmin = ray_tmin_d(C, o); r.tmax = INFINITY;
  double t = 0, b1 = 0, b2 = 0;
  int prim = -1;
  if (!closest_hit<double>(*C.bvh, r, t, prim, b1, b2)) return false;
  const PtTri tri = pt_triangle(C, (uint32_t)prim);
  const D3 ng = normalize(cross(tri.b - tri.a, tri.c - tri.a));
  h.front = dot(ng, d) < 0.0;
  h.gn = h.front ? ng : ng * -1.0;
  h.e1 = tri.b - tri.a;
  h.slot = tri.slot;
  h.face = (uint32_t)prim;
  h.t = t;
  // mesh_hit_attributes (main.swift:1590-1593): the interpolated vertex normals on gn's side.
  const vt_face &fc = C.in->faces[prim];
  const vt_vertex &va = C.in->verts[fc.a], &vb = C.in->verts[fc.b], &vc = C.in->verts[fc.c];
  const D3 sm = D3{va.nx, va.ny, va.nz} * (1.0 - b1 - b2) + D3{vb.nx, vb.ny, vb.nz} * b1 + D3{vc.nx, vc.ny, vc.nz} * b2;
  h.n = h.gn;
  if (dot(sm, sm) > 1e-12) {
    h.n = normalize(sm);
    if (dot(h.n, h.gn) < 0.0) h.n = h.n * -1.0;
  }
  if (C.imported) {
    h.pos = tri.a * (1.0 - b1 - b2) + tri.b * b1 + tri.c * b2;
    h.err = mesh_hit_error_d(tri);
  } else {
    h.pos = o + d * t;
    h.err = kEpsPt;
  }
  return true;
}

bool pt_occluded(const PtContext &C, D3 o, D3 d, double tmax) {
  TraceRay<double> r;
  r.o[0] = o.x; r.o[1] = o.y; r.o[2] = o.z;
  r.d[0] = d.x; r.d[1] = d.y; r.d[2] = d.z;
  r.tmin = ray_tmin_d(C, o); r.tmax = tmax;
  return any_hit<double>(*C.bvh, r, nullptr, nullptr, C.imported);
}

vt_material pt_material(const PtContext &C, uint32_t slot) {
  if (slot < C.in->nmat) return C.mats[slot];
  vt_material m;
  std::memset(&m, 0, sizeof m);
  const uint32_t none = 0xffffffffu;
  std::memcpy(&m.pad, &none, sizeof none);
  return m;
}

// ray_origin (main.swift:1366-1369).
inline D3 ray_origin_d(const PtContext &C, D3 p, D3 gn, D3 dir, double err) {
  const double offset = std::max(err, ray_eps_d(C, p));
  return p + gn * (dot(dir, gn) >= 0.0 ? offset : -offset);
}

double power_heuristic_d(double pf, double pg) {
  const double s = std::max(pf, pg);
  if (s <= 0.0) return 0.0;
  const double f = pf / s, g = pg / s;
  return f * f / (f * f + g * g);
}

struct PtLight { D3 pos, wi, emission; double dist, pdf; uint32_t face; };

PtLight sample_light_d(const PtContext &C, D3 p, ZSampler &seed) {
  PtLight ls{};
  ls.face = 0xffffffffu;
  ls.emission = d3(C.in->light.emission);
  const vt_quad_light &l = C.in->light;
  double u, v;
  seed.f2(u, v);
  const D3 lp = d3(l.corner) + d3(l.su) * u + d3(l.sv) * v;
  D3 dir = lp - p;
  const double dist = std::sqrt(dot(dir, dir));
  dir = dir * (1.0 / dist);
  const double cos_l = std::max(0.0, -dot(dir, d3(l.normal)));
  if (cos_l > 1e-4) { ls.pos = lp; ls.wi = dir; ls.dist = dist; ls.pdf = dist * dist / (C.larea * cos_l); }
  return ls;
}

double light_pdf_d(const PtContext &C, D3 p, D3 hit) {
  D3 dir = hit - p;
  const double dist = std::sqrt(dot(dir, dir));
  dir = dir * (1.0 / dist);
  const double cos_l = std::max(0.0, -dot(dir, d3(C.in->light.normal)));
  return cos_l <= 0.0 ? 0.0 : dist * dist / (C.larea * cos_l);
}

// ---- emitter triangles (imported scenes): power sampling and the light tree -------------------
// imported_geometry (main.swift:2721-2725).
double imported_geometry_d(D3 p, D3 position, const PtTri &t) {
  const D3 d = position - p;
  const double d2 = dot(d, d);
  const D3 n = cross(t.b - t.a, t.c - t.a);
  return d2 > 1e-12 && dot(n, n) > 1e-20 ? std::max(0.0, dot(normalize(n), d * (-1.0 / std::sqrt(d2)))) / d2 : 0.0;
}
double triangle_area_d(const PtTri &t) { const D3 n = cross(t.b - t.a, t.c - t.a); return 0.5 * std::sqrt(dot(n, n)); }

struct PtLtNode { D3 lo, hi, w; double phi, cosO, cosE; uint32_t child, parent, count; };

// light_tree_axis / light_tree_node (main.swift:2751-2778), decoded in double.
D3 lt_axis_d(uint32_t q) {
  const double fx = double(q & 0xffffu) / 65535.0 * 2.0 - 1.0, fy = double(q >> 16) / 65535.0 * 2.0 - 1.0;
  D3 v{fx, fy, 1.0 - std::fabs(fx) - std::fabs(fy)};
  if (v.z < 0.0) {
    const double vx = (1.0 - std::fabs(v.y)) * (v.x >= 0.0 ? 1.0 : -1.0), vy = (1.0 - std::fabs(v.x)) * (v.y >= 0.0 ? 1.0 : -1.0);
    v.x = vx;
    v.y = vy;
  }
  return normalize(v);
}
PtLtNode lt_node_d(const PtContext &C, uint32_t i) {
  const uint32_t *a = C.ltNodes + 8 * (size_t)i, *b = a + 4;
  PtLtNode n;
  n.w = lt_axis_d(a[0]);
  n.phi = fword(a[1]);
  n.cosO = double(a[2] & 0xffffu) / 65535.0 * 2.0 - 1.0;
  n.cosE = double(a[2] >> 16) / 65535.0 * 2.0 - 1.0;
  n.lo = {C.ltLo[0] + double(a[3] & 0xffffu) * C.ltScale[0], C.ltLo[1] + double(a[3] >> 16) * C.ltScale[1],
          C.ltLo[2] + double(b[0] & 0xffffu) * C.ltScale[2]};
  n.hi = {C.ltLo[0] + double(b[0] >> 16) * C.ltScale[0], C.ltLo[1] + double(b[1] & 0xffffu) * C.ltScale[1],
          C.ltLo[2] + double(b[1] >> 16) * C.ltScale[2]};
  n.child = b[2];
  n.parent = b[3] & 0x7ffffffu;
  n.count = b[3] >> 27;
  return n;
}
uint32_t lt_leaf_word_d(const PtContext &C, uint32_t position, uint32_t k) { return C.ltLeaves[3 * (size_t)position + k]; }
double lt_leaf_sum_d(const PtContext &C, const PtLtNode &n) {
  double sum = 0.0;
  for (uint32_t i = 0; i < n.count; ++i) sum += fword(lt_leaf_word_d(C, n.child + i, 1u));
  return sum;
}
double cos_sub_clamped_d(double sinA, double cosA, double sinB, double cosB) { return cosA > cosB ? 1.0 : cosA * cosB + sinA * sinB; }
double sin_sub_clamped_d(double sinA, double cosA, double sinB, double cosB) { return cosA > cosB ? 0.0 : sinA * cosB - cosA * sinB; }

// light_tree_importance (main.swift:2788-2805).
double lt_importance_d(const PtLtNode &n, D3 p) {
  if (!(n.phi > 0.0)) return 0.0;
  const D3 pc = (n.lo + n.hi) * 0.5, dp = p - pc, ext = n.hi - n.lo;
  const double dist2 = dot(dp, dp);
  const double d2 = std::max(dist2, std::max(0.5 * std::sqrt(dot(ext, ext)), 1e-20));
  if (p.x >= n.lo.x && p.y >= n.lo.y && p.z >= n.lo.z && p.x <= n.hi.x && p.y <= n.hi.y && p.z <= n.hi.z) return n.phi / d2;
  const D3 wi = dp * (1.0 / std::sqrt(dist2));
  const double cosW = dot(n.w, wi), sinW = std::sqrt(std::max(0.0, 1.0 - cosW * cosW));
  const D3 dh = pc - n.hi;
  const double s2 = dot(dh, dh) / dist2;
  const double cosB = s2 >= 1.0 ? -1.0 : std::sqrt(std::max(0.0, 1.0 - s2)), sinB = std::sqrt(std::max(0.0, 1.0 - cosB * cosB));
  const double sinO = std::sqrt(std::max(0.0, 1.0 - n.cosO * n.cosO));
  const double cosX = cos_sub_clamped_d(sinW, cosW, sinO, n.cosO), sinX = sin_sub_clamped_d(sinW, cosW, sinO, n.cosO);
  const double cosP = cos_sub_clamped_d(sinX, cosX, sinB, cosB);
  return cosP <= n.cosE ? 0.0 : n.phi * cosP / d2;
}

// light_tree_sample (main.swift:2809-2833).
uint32_t lt_sample_d(const PtContext &C, D3 p, double u, double &pmf) {
  const double below1 = 1.0 - 1.0 / 16777216.0;
  pmf = 1.0;
  uint32_t index = 0;
  for (uint32_t depth = 0; depth <= 64u; ++depth) {
    const PtLtNode n = lt_node_d(C, index);
    if (n.count != 0u) {
      const double sum = lt_leaf_sum_d(C, n), target = u * sum;
      double cumulative = 0.0, chosen = 0.0;
      uint32_t position = 0xffffffffu;
      for (uint32_t i = 0; i < n.count && sum > 0.0; ++i) {
        const double power = fword(lt_leaf_word_d(C, n.child + i, 1u));
        if (!(power > 0.0)) continue;
        position = n.child + i;
        chosen = power;
        cumulative += power;
        if (target < cumulative) break;
      }
      if (position == 0xffffffffu) break;
      pmf *= chosen / sum;
      return position;
    }
    const double l = lt_importance_d(lt_node_d(C, index + 1u), p), r = lt_importance_d(lt_node_d(C, n.child), p);
    if (!(l + r > 0.0)) break;
    const double pl = l / (l + r);
    if (u < pl) { u = std::min(u / pl, below1); index = index + 1u; pmf *= pl; }
    else { u = std::min((u - pl) / (1.0 - pl), below1); index = n.child; pmf *= r / (l + r); }
  }
  pmf = 0.0;
  return 0xffffffffu;
}

// light_tree_pmf (main.swift:2835-2850).
double lt_pmf_d(const PtContext &C, D3 p, uint32_t position) {
  uint32_t index = lt_leaf_word_d(C, position, 2u);
  PtLtNode node = lt_node_d(C, index);
  const double sum = lt_leaf_sum_d(C, node);
  double pmf = sum > 0.0 ? fword(lt_leaf_word_d(C, position, 1u)) / sum : 0.0;
  for (uint32_t depth = 0; depth <= 64u && pmf > 0.0; ++depth) {
    const uint32_t parent = node.parent;
    if (parent == 0x7ffffffu) return pmf;
    const PtLtNode up = lt_node_d(C, parent);
    const double l = lt_importance_d(lt_node_d(C, parent + 1u), p), r = lt_importance_d(lt_node_d(C, up.child), p);
    const double mine = index == parent + 1u ? l : r;
    if (!(l + r > 0.0) || !(mine > 0.0)) return 0.0;
    pmf *= mine / (l + r);
    index = parent;
    node = up;
  }
  return 0.0;
}

uint32_t emitter_position_d(const PtContext &C, uint32_t face) {
  const uint32_t *ids = C.E + 1;
  const uint32_t *it = std::lower_bound(ids, ids + C.ecount, face);
  return it != ids + C.ecount && *it == face ? C.E[1 + C.ecount + (it - ids)] : 0xffffffffu;
}

// imported_emitter_area_pdf (main.swift:2859-2869).
double emitter_area_pdf_d(const PtContext &C, uint32_t face, D3 p, const PtTri &t) {
  if (C.ecount == 0) return 0.0;
  if (C.treeNodes > 0) {
    const uint32_t position = emitter_position_d(C, face);
    const double area = triangle_area_d(t);
    return position != 0xffffffffu && area > 0.0 ? lt_pmf_d(C, p, position) / area : 0.0;
  }
  return C.etotal > 0.0 && t.slot < C.emis.size() ? C.emis[t.slot][3] / C.etotal : 0.0;
}

void make_basis_d(D3 n, D3 &u, D3 &v);

// ---- procedural sky and sun (imported scenes; main.swift:522-597, 2127-2134, 2700-2719) ----------
constexpr uint32_t kEnvFaceD = 0xfffffffeu;
bool in_sun_cone_d(D3 d, D3 s, double omc) {
  const D3 c = cross(d, s);
  return dot(d, s) > 0.0 && dot(c, c) <= omc * (2.0 - omc);
}
double sun_omc_d(uint32_t mode) { return mode == 0u ? (double)8e-4f : (mode == 1u ? (double)7e-4f : (double)9e-4f); }
D3 mix_d(D3 a, D3 b, double t) { return a + (b - a) * t; }
D3 f3d(float x, float y, float z) { return D3{x, y, z}; }
D3 procedural_sky_d(const PtContext &C, D3 d) {
  const double sunCos = dot(d, C.sunDir), y = d.y;
  D3 zenith, horizon, ground, lobe, disc;
  double gradient, lobePower, lobeGain, discGain, groundPower, groundScale, gain;
  if (C.skyMode == 0u) {
    zenith = f3d(0.08f, 0.18f, 0.46f); horizon = f3d(0.96f, 0.52f, 0.22f); ground = f3d(0.12f, 0.10f, 0.08f);
    lobe = f3d(1.0f, 0.70f, 0.30f); disc = f3d(1.0f, 0.78f, 0.45f);
    gradient = 0.40f; lobePower = 6.0; lobeGain = 3.0; discGain = 0.45f; groundPower = 5.0; groundScale = 0.35f; gain = 1.5;
  } else if (C.skyMode == 1u) {
    zenith = f3d(0.16f, 0.42f, 0.92f); horizon = f3d(0.74f, 0.85f, 0.96f); ground = f3d(0.14f, 0.15f, 0.12f);
    lobe = f3d(1.0f, 0.98f, 0.92f); disc = f3d(1.0f, 0.98f, 0.94f);
    gradient = 0.48f; lobePower = 12.0; lobeGain = 2.2f; discGain = 0.40f; groundPower = 4.0; groundScale = 0.40f; gain = 1.8f;
  } else {
    zenith = f3d(0.04f, 0.06f, 0.14f); horizon = f3d(0.46f, 0.26f, 0.42f); ground = f3d(0.04f, 0.04f, 0.05f);
    lobe = f3d(0.95f, 0.65f, 0.75f); disc = f3d(1.0f, 0.85f, 0.78f);
    gradient = 0.55f; lobePower = 10.0; lobeGain = 1.8f; discGain = 0.35f; groundPower = 3.0; groundScale = 0.25f; gain = 1.6f;
  }
  D3 col;
  if (y >= 0.0) {
    col = mix_d(horizon, zenith, std::pow(y, gradient));
    col = col + lobe * (std::pow(std::max(0.0, sunCos), lobePower) * lobeGain);
    if (in_sun_cone_d(d, C.sunDir, sun_omc_d(C.skyMode))) col = col + disc * (C.sunIntensity * discGain);
  } else {
    col = mix_d(ground, horizon * groundScale, std::pow(1.0 + y, groundPower));
  }
  return col * gain;
}
// The image lookup (main.swift:2127-2134): lat-long coordinates with the rotation, v clamped half a
// texel in from the poles, bilinear with repeat in u; in double.
D3 env_image_d(const PtContext &C, D3 d) {
  const double W = C.envW, H = C.envH;
  const double u = std::atan2(d.z, d.x) / (2.0 * kPi) + 0.5 + C.envRot / (2.0 * kPi);
  double v = std::acos(std::min(1.0, std::max(-1.0, d.y))) / kPi;
  v = std::min(std::max(v, 0.5 / H), 1.0 - 0.5 / H);
  const double x = u * W - 0.5, y = v * H - 0.5, fx = std::floor(x), fy = std::floor(y), tx = x - fx, ty = y - fy;
  long x0 = (long)fx % (long)C.envW;
  if (x0 < 0) x0 += C.envW;
  const long x1 = (x0 + 1) % (long)C.envW;
  const long y0 = std::min<long>(std::max<long>((long)fy, 0), C.envH - 1), y1 = std::min<long>(y0 + 1, C.envH - 1);
  auto px = [&](long xx, long yy) {
    const float *q = C.envImg + 4 * ((size_t)yy * C.envW + xx);
    return D3{q[0], q[1], q[2]};
  };
  return px(x0, y0) * ((1 - tx) * (1 - ty)) + px(x1, y0) * (tx * (1 - ty)) + px(x0, y1) * ((1 - tx) * ty) +
         px(x1, y1) * (tx * ty);
}
D3 environment_d(const PtContext &C, D3 d) {
  return (C.envMap ? env_image_d(C, d) : procedural_sky_d(C, d)) * C.envIntensity;
}
// MaterialLibrary.environmentImportance (Sources/StudioModel.swift:1300-1392): dilated luminance, the
// compensated table max(0, L - mean) sin(theta) and the original L sin(theta), normalised to CDFs.
void env_tables_d(PtContext &C) {
  const uint32_t w = C.envW, h = C.envH;
  const size_t n = (size_t)w * h;
  std::vector<double> lum(n), hor(n);
  for (size_t i = 0; i < n; ++i)
    lum[i] = std::max(1e-6, 0.2126 * C.envImg[4 * i] + 0.7152 * C.envImg[4 * i + 1] + 0.0722 * C.envImg[4 * i + 2]);
  for (uint32_t y = 0; y < h; ++y)
    for (uint32_t x = 0; x < w; ++x) {
      const size_t b = (size_t)y * w;
      hor[b + x] = std::max(lum[b + x], std::max(lum[b + (x + w - 1) % w], lum[b + (x + 1) % w]));
    }
  double meanSum = 0, angleSum = 0;
  for (uint32_t y = 0; y < h; ++y) {
    const double st = std::max(1e-4, std::sin(kPi * (y + 0.5) / h));
    double row = 0;
    for (uint32_t x = 0; x < w; ++x) row += lum[(size_t)y * w + x];
    meanSum += row * st;
    angleSum += st * w;
  }
  const double mean = meanSum / angleSum;
  C.envRows.assign(2 * (size_t)h, 0.0);
  C.envCols.assign(2 * n, 0.0);
  double comp = 0;
  for (uint32_t y = 0; y < h; ++y) {
    const double st = std::max(1e-4, std::sin(kPi * (y + 0.5) / h));
    const size_t above = (size_t)(y ? y - 1 : 0) * w, here = (size_t)y * w, below = (size_t)std::min(h - 1, y + 1) * w;
    for (uint32_t x = 0; x < w; ++x) {
      const double dil = std::max(hor[above + x], std::max(hor[here + x], hor[below + x]));
      const double c = std::max(0.0, dil - mean) * st, o = dil * st;
      C.envRows[2 * (size_t)y] += c;
      C.envRows[2 * (size_t)y + 1] += o;
      C.envCols[here + x] = c;
      C.envCols[n + here + x] = o;
      comp += c;
    }
  }
  if (!(comp > 0)) {
    for (uint32_t y = 0; y < h; ++y) C.envRows[2 * (size_t)y] = C.envRows[2 * (size_t)y + 1];
    for (size_t i = 0; i < n; ++i) C.envCols[i] = C.envCols[n + i];
  }
  auto cdf = [](std::vector<double> &wt, size_t count, size_t rows, size_t stride, size_t step) {
    for (size_t r = 0; r < rows; ++r) {
      double total = 0;
      for (size_t k = 0; k < count; ++k) total += wt[r * stride + k * step];
      total = std::max(1e-12, total);
      double sum = 0;
      for (size_t k = 0; k < count; ++k) {
        sum += wt[r * stride + k * step] / total;
        wt[r * stride + k * step] = k == count - 1 ? 1.0 : sum;
      }
    }
  };
  cdf(C.envRows, h, 2, 1, 2);
  cdf(C.envCols, w, 2 * (size_t)h, w, 1);
}
uint32_t env_cdf_index_d(const std::vector<double> &cdf, uint32_t count, size_t stride, size_t base, double value) {
  uint32_t low = 0, high = std::max(1u, count) - 1;
  for (int it = 0; it < 16 && low < high; ++it) {
    const uint32_t mid = (low + high) / 2;
    if (cdf[base + mid * stride] >= value) high = mid; else low = mid + 1;
  }
  return low;
}
double env_cell_pdf_d(const PtContext &C, uint32_t x, uint32_t y, double sinTheta, uint32_t table) {
  const double row = C.envRows[2 * (size_t)y + table], prevRow = y ? C.envRows[2 * (size_t)(y - 1) + table] : 0.0;
  const size_t b = (size_t)(y + table * C.envH) * C.envW;
  const double col = C.envCols[b + x], prevCol = x ? C.envCols[b + x - 1] : 0.0;
  return std::max(0.0, row - prevRow) * std::max(0.0, col - prevCol) * ((double)C.envW * C.envH) /
         (2.0 * kPi * kPi * std::max(1e-5, sinTheta));
}
double env_image_pdf_d(const PtContext &C, D3 wi, uint32_t table) {
  const double theta = std::acos(std::min(1.0, std::max(-1.0, wi.y)));
  double u = std::atan2(wi.z, wi.x) / (2.0 * kPi) + 0.5 + C.envRot / (2.0 * kPi);
  u -= std::floor(u);
  const double v = std::min(std::max(theta / kPi, 0.0), 1.0 - 1e-7);
  const uint32_t x = std::min(C.envW - 1, (uint32_t)(u * C.envW)), y = std::min(C.envH - 1, (uint32_t)(v * C.envH));
  return env_cell_pdf_d(C, x, y, std::sin(theta), table);
}
double imported_probability_d(const PtContext &C) { return C.ecount == 0 ? 0.0 : (C.env ? 0.5 : 1.0); }
double sun_probability_d(const PtContext &C) {
  if (!(C.sunIntensity > 0.0) || !C.env || C.envMap) return 0.0;
  const double w = sun_omc_d(C.skyMode);
  return C.sunDir.y >= -std::sqrt(w * (2.0 - w)) ? 0.60 : 0.0;
}
double environment_pdf_d(const PtContext &C, D3 wi, D3 n, uint32_t table = 0) {
  const double sp = sun_probability_d(C), w = sun_omc_d(C.skyMode);
  const double sunPdf = in_sun_cone_d(wi, C.sunDir, w) ? 1.0 / (2.0 * kPi * w) : 0.0;
  const double rest = C.envMap ? env_image_pdf_d(C, wi, table) : std::max(0.0, dot(n, wi)) / kPi;
  return (1.0 - imported_probability_d(C)) * (sp * sunPdf + (1.0 - sp) * rest);
}
D3 cosine_hemisphere_d(D3 n, double r0, double r1) {
  const double phi = 2.0 * kPi * r0, cos_th = std::sqrt(r1 + 0.5 / 16777216.0);
  const double sin_th = std::sqrt(std::max(0.0, 1.0 - cos_th * cos_th));
  D3 u, v;
  make_basis_d(n, u, v);
  return normalize(u * (std::cos(phi) * sin_th) + v * (std::sin(phi) * sin_th) + n * cos_th);
}

// sample_direct_light's imported branch (main.swift:2889-2955): an emitter triangle with probability
// imported_probability_d, else the environment (sun cone or cosine lobe about n).
// `compensated`: the vertex's BSDF continuation is traced, so the image is sampled from the compensated
// table (main.swift:2077-2085), else from the original one.
PtLight sample_emitters_d(const PtContext &C, D3 p, D3 n, ZSampler &seed, bool compensated) {
  PtLight ls{};
  ls.face = 0xffffffffu;
  const double ip = imported_probability_d(C);
  if (!(ip > 0.0) && !C.env) return ls;
  if (!(ip > 0.0 && seed.f1() < ip)) {
    const double sp = sun_probability_d(C);
    double qx = 1.0, qy = 1.0, qz = 1.0;
    if (sp > 0.0) seed.f3(qx, qy, qz);
    if (sp > 0.0 && qx < sp) {
      const double omc = qy * sun_omc_d(C.skyMode);
      const double cos_th = 1.0 - omc, sin_th = std::sqrt(std::max(0.0, omc * (2.0 - omc)));
      D3 su, sv;
      make_basis_d(C.sunDir, su, sv);
      const double phi = 2.0 * kPi * qz;
      ls.wi = normalize(su * (std::cos(phi) * sin_th) + sv * (std::sin(phi) * sin_th) + C.sunDir * cos_th);
    } else if (C.envMap) {
      const uint32_t table = compensated ? 0u : 1u;
      double c0 = qy, c1 = qz;
      if (!(sp > 0.0)) seed.f2(c0, c1);
      const uint32_t y = env_cdf_index_d(C.envRows, C.envH, 2, table, c0);
      const uint32_t x = env_cdf_index_d(C.envCols, C.envW, 1, (size_t)(y + table * C.envH) * C.envW, c1);
      double r0, r1;
      seed.f2(r0, r1);
      const double u = (x + r0) / C.envW, v = (y + r1) / C.envH;
      const double theta = v * kPi, phi = (u - 0.5 - C.envRot / (2.0 * kPi)) * 2.0 * kPi, st = std::sin(theta);
      ls.wi = normalize(D3{st * std::cos(phi), std::cos(theta), st * std::sin(phi)});
      ls.pos = p + ls.wi * 1e6;
      ls.dist = 1e6;
      ls.face = kEnvFaceD;
      ls.pdf = (1.0 - ip) * (1.0 - sp) * env_cell_pdf_d(C, x, y, st, table);
      ls.emission = environment_d(C, ls.wi);
      return ls;
    } else {
      double r0 = qy, r1 = qz;
      if (!(sp > 0.0)) seed.f2(r0, r1);
      ls.wi = cosine_hemisphere_d(n, r0, r1);
    }
    ls.pos = p + ls.wi * 1e6;
    ls.dist = 1e6;
    ls.face = kEnvFaceD;
    ls.pdf = environment_pdf_d(C, ls.wi, n, compensated ? 0u : 1u);
    ls.emission = environment_d(C, ls.wi);
    return ls;
  }
  double qx, qy, qz;
  seed.f3(qx, qy, qz);
  const bool tree = C.treeNodes > 0;
  double pmf = 0.0;
  uint32_t face;
  if (tree) {
    const uint32_t position = lt_sample_d(C, p, qx, pmf);
    if (position == 0xffffffffu) return ls;
    face = lt_leaf_word_d(C, position, 0u);
  } else {
    uint32_t low = 0, high = C.ecount - 1;
    while (low < high) {
      const uint32_t middle = (low + high) / 2;
      if (fword(C.E[1 + C.ecount + middle]) >= qx) high = middle; else low = middle + 1;
    }
    face = C.E[1 + low];
  }
  const PtTri t = pt_triangle(C, face);
  const double root = std::sqrt(qy);
  ls.pos = t.a * (1.0 - root) + t.b * (root * (1.0 - qz)) + t.c * (root * qz);
  const D3 delta = ls.pos - p;
  ls.dist = std::sqrt(dot(delta, delta));
  ls.wi = delta * (1.0 / std::max(ls.dist, 1e-8));
  const double geometry = imported_geometry_d(p, ls.pos, t);
  ls.emission = t.slot < C.emis.size() ? D3{C.emis[t.slot][0], C.emis[t.slot][1], C.emis[t.slot][2]} : D3{0, 0, 0};
  ls.face = face;
  const double area = tree ? triangle_area_d(t) : 0.0;
  const double areaPdf = !tree ? emitter_area_pdf_d(C, face, p, t) : (area > 0.0 ? pmf / area : 0.0);
  ls.pdf = geometry > 1e-12 ? ip * areaPdf / geometry : 0.0;
  return ls;
}

// eval_light_pdf for imported emitters (main.swift:3066-3071).
double emitter_pdf_d(const PtContext &C, D3 p, D3 hitPos, uint32_t face) {
  if (C.ecount == 0) return 0.0;
  const PtTri t = pt_triangle(C, face);
  const double g = imported_geometry_d(p, hitPos, t);
  return g > 1e-12 ? imported_probability_d(C) * emitter_area_pdf_d(C, face, p, t) / g : 0.0;
}

// light_visible (main.swift:3254-3264) with endpoint_tolerance (main.swift:1358-1361).
bool visible_d(const PtContext &C, D3 p, D3 gn, double err, const PtLight &ls) {
  if (!(ls.pdf > 0.0)) return false;
  const D3 o = ray_origin_d(C, p, gn, ls.wi, err);
  D3 delta = ls.pos - o;
  const double d = std::sqrt(dot(delta, delta));
  const double legacy = 2.0 * ray_eps_d(C, ls.pos);
  const double tol = C.imported ? std::max(legacy, 1.907349e-6 * (max_abs_d(o) + max_abs_d(ls.pos) + d)) : legacy;
  if (d <= tol) return false;
  return !pt_occluded(C, o, delta * (1.0 / d), d - tol);
}

// n: shading normal; gn: geometric normal (eval_bsdf for DIFFUSE, main.swift:2659-2676).
// ---- OPENPBR vertices: the reference BSDF (float) through vto_pt_inputs ---------------------------
// A slot's lobe parameters (8 floats; null without a table or past it).
const float *slot_params(const PtContext &C, const vt_material &m) {
  uint32_t slot;
  std::memcpy(&slot, &m.pad, sizeof slot);
  return C.in->pbr_params && slot < C.in->nmat ? C.in->pbr_params + 12 * (size_t)slot : nullptr;
}
// is_delta (main.swift:3285-3287): glass, and GLOSSY mirrors smoother than 0.02.
bool is_delta_d(const PtContext &C, const vt_material &m) {
  const float *pp = slot_params(C, m);
  return m.type == VT_MAT_DIELECTRIC || (m.type == VT_MAT_GLOSSY && (pp ? pp[0] : 0.0f) < 0.02f);
}
// The OpenPBR BSDF: OPENPBR slots and rough GLOSSY ones (metalness 1 in the adapter).
bool pbr_slot(const PtContext &C, const vt_material &m) {
  const float *pp = slot_params(C, m);
  return pp && C.in->pbr_eval && (m.type == VT_MAT_OPENPBR || (m.type == VT_MAT_GLOSSY && pp[0] >= 0.02f));
}
// The adapter's mat.tangent for an anisotropic slot: mesh_hit_attributes' tangent of a mesh without UVs
// (main.swift:1594-1599), the edge e1 = b - a made perpendicular to the shading normal n (n x y, or
// n x x near the poles, when e1 runs along n), unit length. Isotropic slots keep the basis from the
// normal alone, as the device does: their lobes are symmetric about it.
vto_pbr_material pbr_material_d(const PtContext &C, const vt_material &m, double b0, double b1, double b2, D3 n, D3 e1) {
  uint32_t slot;
  std::memcpy(&slot, &m.pad, sizeof slot);
  vto_pbr_material q;
  std::memset(&q, 0, sizeof q);
  q.type = m.type;
  q.albedo[0] = (float)b0;
  q.albedo[1] = (float)b1;
  q.albedo[2] = (float)b2;
  const float *pp = C.in->pbr_params + 12 * (size_t)slot;
  q.roughness = pp[0];
  q.metalness = pp[1];
  q.ior = pp[2];
  q.coat = pp[7];  // both transports (prepare_openpbr, main.swift:2494)
  q.fuzz = pp[8];  // main.swift:2497
  q.anisotropy = pp[9];  // main.swift:2496
  if (q.anisotropy > 0.0f) {
    D3 t = e1 - n * dot(e1, n);
    if (dot(t, t) < 1e-12) t = cross(n, std::fabs(n.y) < 0.9 ? D3{0, 1, 0} : D3{1, 0, 0});
    t = normalize(t);
    q.tangent[0] = (float)t.x;
    q.tangent[1] = (float)t.y;
    q.tangent[2] = (float)t.z;
  }
  // The thin film is a spectral-transport input (prepare_openpbr_lanes, main.swift:2527-2568).
  if (C.spectral) {
    q.thin_film_weight = pp[4];
    q.thin_film_thickness = pp[5];
    q.thin_film_ior = pp[6];
  }
  return q;
}
// prepare_bsdf (main.swift:2573-2593): with a thin film the lanes' wavelengths (a: lanes 0-2, b: lane
// 3), else the library's default RGB wavelengths (null).
bool pbr_film_d(const PtContext &C, const vt_material &m) {
  uint32_t slot;
  std::memcpy(&slot, &m.pad, sizeof slot);
  return C.spectral && C.in->pbr_params[12 * (size_t)slot + 4] > 0.0f;
}
// eval_bsdf_with_pdf (main.swift:2695-2706): f (no cosine) per lane, pdf of lanes 0-2.
Spec4 pbr_eval_lanes_d(const PtContext &C, const PtLanes &L, const vt_material &m, D3 n, D3 gn, D3 e1, D3 wo, D3 wi, double &pdf) {
  pdf = 0.0;
  const double cosine = std::fabs(dot(n, wi));
  if (cosine < 1e-7 || dot(n, wo) <= 0.0) return {{0, 0, 0, 0}};
  const Spec4 rho = reflectance(C, L, m);
  const float fn[3] = {(float)n.x, (float)n.y, (float)n.z}, fo[3] = {(float)wo.x, (float)wo.y, (float)wo.z},
              fi[3] = {(float)wi.x, (float)wi.y, (float)wi.z};
  const vto_pbr_material a = pbr_material_d(C, m, rho.v[0], rho.v[1], rho.v[2], n, e1);
  const bool film = pbr_film_d(C, m);
  const float la[3] = {(float)L.lambda[0], (float)L.lambda[1], (float)L.lambda[2]};
  const float lb[3] = {(float)L.lambda[3], (float)L.lambda[3], (float)L.lambda[3]};
  float f[3], q;
  C.in->pbr_eval(&a, fn, fo, fi, film ? la : nullptr, f, &q);
  pdf = q;
  if (dot(wi, gn) <= 0.0) return {{0, 0, 0, 0}};
  double f3 = f[0];
  if (C.spectral && (rho.v[3] != rho.v[0] || film)) {
    const vto_pbr_material b = pbr_material_d(C, m, rho.v[3], rho.v[3], rho.v[3], n, e1);
    float g[3], qb;
    C.in->pbr_eval(&b, fn, fo, fi, film ? lb : nullptr, g, &qb);
    f3 = g[0];
  }
  return {{f[0] / cosine, f[1] / cosine, f[2] / cosine, C.spectral ? f3 / cosine : 0.0}};
}
// sample_bsdf (main.swift:3359-3366): direction, f |cos| / pdf per lane, pdf.
bool pbr_sample_lanes_d(const PtContext &C, const PtLanes &L, const vt_material &m, D3 n, D3 gn, D3 e1, D3 wo, const double r[3],
                        D3 &dir, Spec4 &w, double &pdf) {
  const Spec4 rho = reflectance(C, L, m);
  const float fn[3] = {(float)n.x, (float)n.y, (float)n.z}, fo[3] = {(float)wo.x, (float)wo.y, (float)wo.z},
              fr[3] = {(float)r[0], (float)r[1], (float)r[2]};
  const vto_pbr_material a = pbr_material_d(C, m, rho.v[0], rho.v[1], rho.v[2], n, e1);
  const bool film = pbr_film_d(C, m);
  const float la[3] = {(float)L.lambda[0], (float)L.lambda[1], (float)L.lambda[2]};
  const float lb[3] = {(float)L.lambda[3], (float)L.lambda[3], (float)L.lambda[3]};
  float d[3], ww[3], q;
  int32_t lobe;
  C.in->pbr_sample(&a, fn, fo, fr, film ? la : nullptr, d, ww, &q, &lobe);
  if (!(q > 0.0f)) return false;
  dir = D3{d[0], d[1], d[2]};
  if (dot(dir, gn) <= 0.0) return false;
  pdf = q;
  double w3 = ww[0];
  if (C.spectral && (rho.v[3] != rho.v[0] || film)) {
    const vto_pbr_material b = pbr_material_d(C, m, rho.v[3], rho.v[3], rho.v[3], n, e1);
    float g[3], qb;
    C.in->pbr_eval(&b, fn, fo, d, film ? lb : nullptr, g, &qb);
    w3 = g[0] / q;
  }
  w = {{ww[0], ww[1], ww[2], C.spectral ? w3 : 0.0}};
  for (double x : w.v)
    if (!std::isfinite(x) || x < 0.0) return false;
  return true;
}

// sample_bsdf's delta branches (main.swift:3318-3352), in double: DIELECTRIC refracts or reflects by
// Schlick's Fresnel at the slot's IOR (the cosine on the less dense side; one draw, none under total
// internal reflection; tint = albedo, times eta^2 on refraction), retried once about the geometric
// normal when the event lands on the wrong side; a GLOSSY mirror reflects about the shading normal
// (the geometric one when that reflection goes below the surface) with Schlick's conductor Fresnel,
// F0 = albedo, and in spectral transport the reference's film over it (ref_thin_film_mirror) mixed in
// by its presence. Weight = f |cos| / pdf per lane.
D3 reflect_d(D3 i, D3 n) { return i - n * (2.0 * dot(n, i)); }
bool sample_delta_d(const PtContext &C, const PtLanes &L, const vt_material &m, D3 n, D3 gn, D3 in, bool front,
                    ZSampler &seed, D3 &dir, Spec4 &w) {
  const Spec4 tint = reflectance(C, L, m);
  const float *pp = slot_params(C, m);
  if (m.type == VT_MAT_DIELECTRIC) {
    const double ior = pp ? pp[2] : 1.5;
    const double eta = front ? 1.0 / ior : ior;
    const double r0 = (1.0 - ior) / (1.0 + ior), f0 = r0 * r0;
    for (int attempt = 0; attempt < 2; ++attempt) {
      const D3 mm = attempt == 0 ? n : gn;
      const double cosI = std::min(std::max(-dot(in, mm), 0.0), 1.0);
      const double sin2T = eta * eta * (1.0 - cosI * cosI);
      const double cosine = eta > 1.0 && sin2T < 1.0 ? std::sqrt(1.0 - sin2T) : cosI;
      const double fresnel = f0 + (1.0 - f0) * std::pow(1.0 - cosine, 5.0);
      const bool reflected = sin2T >= 1.0 || seed.f1() < fresnel;
      if (reflected) {
        dir = normalize(reflect_d(in, mm));
        w = tint;
      } else {
        dir = normalize(in * eta + mm * (eta * cosI - std::sqrt(1.0 - sin2T)));
        w = scale(tint, eta * eta);
      }
      if ((dot(dir, gn) > 0.0) == reflected) return true;
    }
    return false;
  }
  const D3 mm = dot(reflect_d(in, n), gn) > 0.0 ? n : gn;
  dir = normalize(reflect_d(in, mm));
  const double cosI = std::min(std::max(-dot(in, mm), 0.0), 1.0);
  const double s5 = std::pow(1.0 - cosI, 5.0);
  for (int k = 0; k < 4; ++k) w.v[k] = tint.v[k] + (1.0 - tint.v[k]) * s5;
  if (!C.spectral) w.v[3] = 0.0;
  if (C.spectral && pp && C.in->pbr_film_mirror && pp[4] > 0.0f) {
    const float f0a[3] = {(float)tint.v[0], (float)tint.v[1], (float)tint.v[2]}, f0b[3] = {(float)tint.v[3], (float)tint.v[3], (float)tint.v[3]};
    const float la[3] = {(float)L.lambda[0], (float)L.lambda[1], (float)L.lambda[2]};
    const float lb[3] = {(float)L.lambda[3], (float)L.lambda[3], (float)L.lambda[3]};
    float ra[3], rb[3];
    const double presence = C.in->pbr_film_mirror((float)cosI, pp[4], pp[5], pp[6], f0a, la, ra);
    if (presence > 0.0) {
      C.in->pbr_film_mirror((float)cosI, pp[4], pp[5], pp[6], f0b, lb, rb);
      const double film[4] = {ra[0], ra[1], ra[2], rb[0]};
      for (int k = 0; k < 4; ++k) w.v[k] = w.v[k] + (film[k] - w.v[k]) * presence;
    }
  }
  return dot(dir, gn) > 0.0;
}

D3 direct_d(const PtContext &C, const PtLanes &L, D3 p, D3 n, D3 gn, D3 e1, double err, D3 wo, const Spec4 &T,
            const vt_material &m, bool useMIS, bool compensated, ZSampler &seed, bool requirePdf) {
  const PtLight ls = C.imported ? sample_emitters_d(C, p, n, seed, compensated) : sample_light_d(C, p, seed);
  if (requirePdf && !(ls.pdf > 0.0)) return {0, 0, 0};
  if (!visible_d(C, p, gn, err, ls)) return {0, 0, 0};
  const double cosine = std::fabs(dot(n, ls.wi)), ni = dot(n, ls.wi), no = dot(n, wo);
  if (pbr_slot(C, m)) {
    double bpdf;
    const Spec4 f = pbr_eval_lanes_d(C, L, m, n, gn, e1, wo, ls.wi, bpdf);
    const double w = useMIS ? power_heuristic_d(ls.pdf, bpdf) : 1.0;
    const float le[3] = {(float)ls.emission.x, (float)ls.emission.y, (float)ls.emission.z};
    return to_rgb(C, L, scale(mul(mul(T, f), emission(C, L, le)), cosine * w / ls.pdf));
  }
  const Spec4 albedo = reflectance(C, L, m);
  double f = 0.0, bpdf = 0.0;
  if (no > 0.0) {
    bpdf = std::max(0.0, ni) / kPi;
    if (ni > 0.0 && cosine >= 1e-7 && dot(ls.wi, gn) > 0.0) f = 1.0 / kPi;
  }
  const double w = useMIS ? power_heuristic_d(ls.pdf, bpdf) : 1.0;
  const float le[3] = {(float)ls.emission.x, (float)ls.emission.y, (float)ls.emission.z};
  return to_rgb(C, L, scale(mul(mul(T, albedo), emission(C, L, le)), f * cosine * w / ls.pdf));
}

void make_basis_d(D3 n, D3 &u, D3 &v) {
  const D3 up = std::fabs(n.z) < 0.999 ? D3{0, 0, 1} : D3{1, 0, 0};
  u = normalize(cross(up, n));
  v = cross(n, u);
}

D3 camera_dir_d(const PtContext &C, uint32_t x, uint32_t y, float jx_f, float jy_f) {
  const double jx = double(jx_f) + 0.5, jy = double(jy_f) + 0.5;
  double u = ((x + jx) / C.p->width) * 2.0 - 1.0, v = ((y + jy) / C.p->height) * 2.0 - 1.0;
  v = -v;
  u *= C.aspect * C.fovScale;
  v *= C.fovScale;
  return normalize(C.fwd + C.right * u + C.up * v);
}

// lens_ray (main.swift:2210-2216).
void lens_d(const PtContext &C, D3 &o, D3 &d, ZSampler &seed) {
  if (!(C.p->aperture > 0.0f)) return;
  seed.event(0u, 3u);
  double r0, r1;
  seed.f2(r0, r1);
  const double radius = std::sqrt(r0) * C.p->aperture, angle = 2.0 * kPi * r1;
  const D3 focus = o + d * (double(C.p->focus_distance) / std::max(1e-5, dot(d, C.fwd)));
  o = o + C.right * (radius * std::cos(angle)) + C.up * (radius * std::sin(angle));
  d = normalize(focus - o);
}

// emitter_rgb at the primary hit (main.swift:7467-7468); imported emitters emit from the front.
D3 primary_emission_d(const PtContext &C, const PtLanes &L, const PtHit &h, const vt_material &m) {
  if (C.imported && !h.front) return {0, 0, 0};
  return to_rgb(C, L, emission(C, L, m.emission));
}

// The path after its primary vertex (shading_kernel's bounce loop, main.swift:7709-7833). With
// diPrimary (sampling mode 0) a BSDF hit on an emitter from the primary vertex gets no weight.
D3 continue_path_d(const PtContext &C, const PtLanes &L, PtHit h, vt_material m, D3 dir, ZSampler &seed, bool diPrimary) {
  const int limit = std::max(0, (int)C.p->max_depth - 1);
  const bool nee = C.p->sampling_mode != 3u, mis = C.p->sampling_mode <= 1u;
  // ReSTIR GI estimates the secondary diffuse vertex's direct light (restirGISecondary,
  // main.swift:7801-7803).
  const bool giPrimary = diPrimary && m.type == VT_MAT_DIFFUSE;
  Spec4 T = C.spectral ? Spec4{{1, 1, 1, 1}} : Spec4{{1, 1, 1, 0}};
  D3 R{0, 0, 0};
  int scattering = 0;
  bool emissionOnly = false;
  for (int bounce = 1;; ++bounce) {
    // Ideal reflections and refractions spend no scattering event (main.swift:7716-7723).
    const bool delta = is_delta_d(C, m);
    if (!delta && scattering >= limit) {
      if (nee || emissionOnly) break;
      emissionOnly = true;
    }
    if (!delta) ++scattering;
    const bool previousMIS = mis && !(diPrimary && bounce == 1);
    seed.event((uint32_t)bounce, 0u);
    D3 nd;
    double bpdf = 0.0;
    double r0 = 0.0, r1 = 0.0, r2 = 0.0;
    if (!delta) seed.f3(r0, r1, r2);
    if (delta) {
      Spec4 w;
      if (!sample_delta_d(C, L, m, h.n, h.gn, dir, h.front, seed, nd, w)) break;
      T = mul(T, w);
    } else if (pbr_slot(C, m)) {
      const double r[3] = {r0, r1, r2};
      Spec4 w;
      if (!pbr_sample_lanes_d(C, L, m, h.n, h.gn, h.e1, dir * -1.0, r, nd, w, bpdf)) break;
      T = mul(T, w);
    } else {
      const double phi = 2.0 * kPi * r1, cos_th = std::sqrt(r2 + 0.5 / 16777216.0);
      const double sin_th = std::sqrt(std::max(0.0, 1.0 - cos_th * cos_th));
      D3 bu, bv;
      make_basis_d(h.n, bu, bv);
      nd = normalize(bu * (std::cos(phi) * sin_th) + bv * (std::sin(phi) * sin_th) + h.n * cos_th);
      bpdf = std::max(0.0, dot(h.n, nd)) / kPi;
      if (!(bpdf > 0.0) || !(dot(nd, h.gn) > 0.0)) break;
      T = mul(T, reflectance(C, L, m));
    }
    dir = nd;
    bool finite = true;
    for (double t : T.v) finite = finite && std::isfinite(t);
    if (!finite || smax(C, T) <= 0.0) break;
    const D3 prev = h.pos, prevN = h.n;
    const D3 o = ray_origin_d(C, h.pos, h.gn, nd, h.err);
    if (!pt_closest(C, o, nd, h)) {
      // An escape sees the environment, weighed against its NEE density (main.swift:7751-7756).
      if (C.env) {
        const double lpdf = nee ? environment_pdf_d(C, nd, prevN) : 0.0;
        const double w = delta || !nee || lpdf <= 0.0 ? 1.0 : (previousMIS ? power_heuristic_d(bpdf, lpdf) : 0.0);
        const D3 e = environment_d(C, nd);
        const float ef[3] = {(float)e.x, (float)e.y, (float)e.z};
        R = R + to_rgb(C, L, scale(mul(T, emission(C, L, ef)), w));
      }
      break;
    }
    m = pt_material(C, h.slot);
    if (m.type == VT_MAT_EMISSIVE) {
      const double lpdf = C.imported ? emitter_pdf_d(C, prev, h.pos, h.face) : light_pdf_d(C, prev, h.pos);
      const double w = delta || !nee || lpdf <= 0.0 ? 1.0 : (previousMIS ? power_heuristic_d(bpdf, lpdf) : 0.0);
      if (!C.imported || h.front) R = R + to_rgb(C, L, scale(mul(T, emission(C, L, m.emission)), w));
      break;
    }
    if (emissionOnly) break;
    // No NEE at glass or mirrors (main.swift:7803); the roulette ceiling is 0.99 there (:7820-7823).
    const bool nextDelta = is_delta_d(C, m);
    if (nee && !nextDelta && !(giPrimary && bounce == 1 && m.type == VT_MAT_DIFFUSE)) {
      seed.event((uint32_t)bounce + 1u, 1u);
      R = R + direct_d(C, L, h.pos, h.n, h.gn, h.e1, h.err, nd * -1.0, T, m, mis && scattering < limit, scattering < limit, seed,
                       false);
    }
    if (bounce > 3) {
      const double survival = std::min(std::max(smax(C, T), 0.05), nextDelta ? 0.99 : 0.95);
      seed.event((uint32_t)bounce + 1u, 2u);
      if (seed.f1() >= survival) break;
      T = scale(T, 1.0 / survival);
    }
  }
  return R;
}

// ---- ReSTIR DI (sampling mode 0), FP64 ---------------------------------------------------------
// restir_temporal_kernel (main.swift:4842-4960) and the spatial reuse of shading_kernel
// (main.swift:7484-7561): per frame, pass 1 over every pixel, then pass 2 over every pixel.
struct DiS { D3 pos{0, 0, 0}, emission{0, 0, 0}; double pdf = 0, u = 0; uint32_t id = 0; };
// A ReSTIR GI sample: x2, its normal, its outgoing direct radiance per lane, its source pdf (area
// measure), the wavelength number, validity (restir_gi_encode's normal flag).
struct GiS { D3 pos{0, 0, 0}, nrm{0, 0, 0}; Spec4 rad{{0, 0, 0, 0}}; double pdf = 0, u = 0; bool valid = false; };
struct DiPix {
  double pos[4] = {0, 0, 0, -1}, nrm[4] = {0, 0, 0, -1};
  PtHit hit{};
  DiS s;
  double wsum = 0, M = 0, W = 0;
  GiS g;
  double gwsum = 0, gM = 0, gW = 0;
};

// light_geometry (main.swift:3165-3183).
double light_geometry_d(const PtContext &C, D3 p, const DiS &c) {
  if (C.imported && c.id >= 2u) return imported_geometry_d(p, c.pos, pt_triangle(C, c.id - 2u));
  const D3 delta = c.pos - p;
  const double d2 = dot(delta, delta);
  if (d2 < 1e-10) return 0.0;
  return std::max(0.0, dot(d3(C.in->light.normal), delta * (-1.0 / std::sqrt(d2)))) / d2;
}

D3 di_contribution_d(const PtContext &C, D3 p, D3 n, D3 gn, D3 e1, D3 view, const vt_material &m, const DiS &c) {
  const D3 dir = normalize(c.pos - p);
  const double cos_th = std::max(0.0, dot(n, dir));
  if (cos_th <= 0.0) return {0, 0, 0};
  PtLanes L{};
  if (C.spectral) L = make_lanes(C, c.u);
  const float e[3] = {(float)c.emission.x, (float)c.emission.y, (float)c.emission.z};
  if (pbr_slot(C, m)) {
    double pdf;
    const Spec4 f = pbr_eval_lanes_d(C, L, m, n, gn, e1, view * -1.0, dir, pdf);
    return to_rgb(C, L, scale(mul(f, emission(C, L, e)), cos_th)) * light_geometry_d(C, p, c);
  }
  const double ni = dot(n, dir), no = -dot(n, view);
  const double f = no > 0.0 && ni > 0.0 && std::fabs(ni) >= 1e-7 && dot(dir, gn) > 0.0 ? 1.0 / kPi : 0.0;
  return to_rgb(C, L, scale(mul(reflectance(C, L, m), emission(C, L, e)), f * cos_th)) * light_geometry_d(C, p, c);
}

// eval_restir_target_pdf (main.swift:3187-3197).
double di_target_d(const PtContext &C, D3 p, D3 n, D3 gn, D3 e1, D3 view, const vt_material &m, const DiS &c) {
  if (c.pdf <= 0.0) return 0.0;
  const D3 v = di_contribution_d(C, p, n, gn, e1, view, m, c);
  return std::sqrt(dot(v, v));
}

bool same_surface_d(const double *pos, const double *nrm, const double *op, const double *on) {
  const double dx = op[0] - pos[0], dy = op[1] - pos[1], dz = op[2] - pos[2];
  return op[3] > 0.0 && on[3] == nrm[3] && on[0] * nrm[0] + on[1] * nrm[1] + on[2] * nrm[2] > 0.95 &&
         std::sqrt(dx * dx + dy * dy + dz * dz) < std::max(0.01, pos[3] * 0.01);
}
bool compatible_d(const double *pos, const double *nrm, const double *np, const double *nn) {
  return np[3] > 0.0 && nn[3] == nrm[3] && nrm[0] * nn[0] + nrm[1] * nn[1] + nrm[2] * nn[2] > 0.95 &&
         std::fabs(pos[3] - np[3]) < 0.05 * pos[3];
}

// restir_backproject (main.swift:4828-4836) with an unmoved camera between frames.
bool backproject_d(const PtContext &C, D3 p, int &px, int &py) {
  const D3 d = p - C.cam;
  const double z = dot(d, C.fwd);
  if (!(z > 0.0)) return false;
  const double nx = dot(d, C.right) / (z * C.aspect * C.fovScale), ny = dot(d, C.up) / (z * C.fovScale);
  const double ux = nx * 0.5 + 0.5, uy = -ny * 0.5 + 0.5;
  if (!(ux >= 0.0 && uy >= 0.0 && ux < 1.0 && uy < 1.0)) return false;
  px = (int)(ux * C.p->width);
  py = (int)(uy * C.p->height);
  return px >= 0 && px < (int)C.p->width && py >= 0 && py < (int)C.p->height;
}

DiS di_from_light(const PtLight &ls, double u) {
  DiS c;
  c.pos = ls.pos; c.emission = ls.emission; c.pdf = ls.pdf; c.u = u;
  c.id = ls.face == 0xffffffffu ? 0u : ls.face + 2u;
  return c;
}

PtLight light_from_di(const DiS &c, D3 p) {
  PtLight ls{};
  ls.pos = c.pos;
  const D3 d = c.pos - p;
  ls.dist = std::sqrt(dot(d, d));
  ls.wi = normalize(d);
  ls.emission = c.emission;
  ls.pdf = c.pdf;
  ls.face = c.id >= 2u ? c.id - 2u : 0xffffffffu;
  return ls;
}


// ---- ReSTIR GI (main.swift:3201-3252, 4718-4806, 7582-7656), FP64 ---------------------------------
double gi_geometry_d(D3 x1, D3 n1, D3 x2, D3 n2) {
  const D3 delta = x2 - x1;
  const double d2 = dot(delta, delta);
  if (d2 < 1e-10) return 0.0;
  const D3 dir = delta * (1.0 / std::sqrt(d2));
  return std::max(0.0, dot(n1, dir)) * std::max(0.0, -dot(n2, dir)) / d2;
}
bool gi_accepts_shift_d(D3 x1r, D3 x1q, D3 x2, D3 n2) {
  const D3 cur = x1r - x2, src = x1q - x2;
  const double cd2 = dot(cur, cur), sd2 = dot(src, src);
  if (cd2 < 1e-10 || sd2 < 1e-10) return false;
  const double cc = std::max(0.0, dot(n2, cur * (1.0 / std::sqrt(cd2)))), sc = std::max(0.0, dot(n2, src * (1.0 / std::sqrt(sd2))));
  double j = cc * sd2 / (sc * cd2);
  if (!std::isfinite(j)) j = 0.0;
  return j >= 0.1 && j <= 10.0;
}
double lambert_eval_d(D3 n, D3 gn, D3 wo, D3 wi, double &pdf) {
  const double ni = dot(n, wi), no = dot(n, wo);
  pdf = 0.0;
  if (!(no > 0.0)) return 0.0;
  pdf = std::max(0.0, ni) / kPi;
  return ni > 0.0 && std::fabs(ni) >= 1e-7 && dot(wi, gn) > 0.0 ? 1.0 / kPi : 0.0;
}
double gi_target_d(const PtContext &C, const PtHit &h, D3 rayDir, const vt_material &m, const GiS &c) {
  const double geometry = gi_geometry_d(h.pos, h.n, c.pos, c.nrm);
  bool finite = true;
  for (double x : c.rad.v) finite = finite && std::isfinite(x);
  if (geometry <= 0.0 || !finite) return 0.0;
  const D3 dir = normalize(c.pos - h.pos);
  PtLanes L{};
  if (C.spectral) L = make_lanes(C, c.u);
  double pdf;
  const double f = lambert_eval_d(h.n, h.gn, rayDir * -1.0, dir, pdf);
  const D3 v = to_rgb(C, L, scale(mul(reflectance(C, L, m), c.rad), f * geometry));
  return std::sqrt(dot(v, v));
}
bool gi_visible_d(const PtContext &C, D3 x1, D3 n1, D3 x2, double err) {
  const D3 delta = x2 - x1;
  const double dist = std::sqrt(dot(delta, delta));
  if (dist <= 2.0 * ray_eps_d(C, x1)) return false;
  const D3 o = ray_origin_d(C, x1, n1, delta * (1.0 / dist), err);
  const D3 e = x2 - o;
  const double d = std::sqrt(dot(e, e));
  const double legacy = 2.0 * ray_eps_d(C, x2);
  const double tol = C.imported ? std::max(legacy, 1.907349e-6 * (max_abs_d(o) + max_abs_d(x2) + d)) : legacy;
  return !pt_occluded(C, o, e * (1.0 / d), d - tol);
}
// restir_gi_initial (main.swift:4718-4770) at a diffuse primary hit h (material m) seen along view.
GiS gi_initial_d(const PtContext &C, const PtHit &h, const vt_material &m, D3 view, double u, ZSampler &seed,
                 double &wsum) {
  GiS r;
  r.u = u;
  wsum = 0.0;
  const int limit = std::max(0, (int)C.p->max_depth - 1);
  seed.event(1u, 5u);
  double r0, r1, r2;
  seed.f3(r0, r1, r2);
  const D3 gd = cosine_hemisphere_d(h.n, r1, r2);
  const double bpdf = std::max(0.0, dot(h.n, gd)) / kPi;
  if (!(bpdf > 0.0) || !(dot(gd, h.gn) > 0.0)) return r;
  PtHit h2;
  if (!pt_closest(C, ray_origin_d(C, h.pos, h.gn, gd, h.err), gd, h2)) return r;
  const vt_material m2 = pt_material(C, h2.slot);
  if (m2.type != VT_MAT_DIFFUSE) return r;
  PtLanes L{};
  if (C.spectral) L = make_lanes(C, u);
  Spec4 rad{{0, 0, 0, 0}};
  seed.event(2u, 6u);
  const PtLight ls = C.imported ? sample_emitters_d(C, h2.pos, h2.n, seed, limit >= 2) : sample_light_d(C, h2.pos, seed);
  if (ls.pdf > 0.0 && visible_d(C, h2.pos, h2.gn, h2.err, ls)) {
    const double c2 = std::max(0.0, dot(h2.n, ls.wi));
    double pdf2;
    const double f2 = lambert_eval_d(h2.n, h2.gn, gd * -1.0, ls.wi, pdf2);
    const double mis = limit >= 2 ? power_heuristic_d(ls.pdf, pdf2) : 1.0;
    const float le[3] = {(float)ls.emission.x, (float)ls.emission.y, (float)ls.emission.z};
    rad = scale(mul(reflectance(C, L, m2), emission(C, L, le)), f2 * c2 * mis / ls.pdf);
  }
  const D3 delta = h2.pos - h.pos;
  const double d2 = dot(delta, delta);
  const double cos2 = std::max(0.0, -dot(h2.n, gd));
  const double src = d2 > 1e-10 ? bpdf * cos2 / d2 : 0.0;
  GiS c;
  c.pos = h2.pos;
  c.nrm = h2.n;
  c.rad = rad;
  c.pdf = src;
  c.u = u;
  c.valid = src > 0.0;
  const double pHat = gi_target_d(C, h, view, m, c);
  if (src > 0.0 && pHat > 0.0) {
    r = c;
    wsum = pHat / src;
  }
  return r;
}

void di_primary_d(const PtContext &C, uint32_t x, uint32_t y, uint32_t si, uint32_t frame, float jx, float jy,
                  uint32_t M, uint32_t bits, bool history, const std::vector<DiPix> &prev, DiPix &out) {
  out = DiPix{};
  ZSampler seed = ZSampler::pixel(x, y, C.p->width, si, C.p->sampler != 0u, C.p->z_temporal, frame);
  const double u = C.spectral ? seed.wavelength_u() : 0.0;
  D3 dir0 = camera_dir_d(C, x, y, jx, jy), o0 = C.cam;
  lens_d(C, o0, dir0, seed);
  PtHit h;
  if (!pt_closest(C, o0, dir0, h)) return;
  const vt_material m = pt_material(C, h.slot);
  out.hit = h;
  const double pos[4] = {h.pos.x, h.pos.y, h.pos.z, h.t}, nrm[4] = {h.n.x, h.n.y, h.n.z, double(m.type)};
  std::memcpy(out.pos, pos, sizeof pos);
  std::memcpy(out.nrm, nrm, sizeof nrm);
  if (m.type != VT_MAT_DIFFUSE) return;
  out.s.u = u;
  for (uint32_t c = 0; c < M; ++c) {
    seed.candidate(1u, 4u, c, bits);
    const PtLight ls = C.imported ? sample_emitters_d(C, h.pos, h.n, seed, (int)C.p->max_depth - 1 > 0)
                                  : sample_light_d(C, h.pos, seed);
    out.M += 1.0;
    if (!(ls.pdf > 0.0)) continue;
    const DiS cand = di_from_light(ls, u);
    const double pHat = di_target_d(C, h.pos, h.n, h.gn, h.e1, dir0, m, cand);
    const double proposal = cand.pdf * light_geometry_d(C, h.pos, cand);
    const double w = proposal > 0.0 ? pHat / proposal : 0.0;
    out.wsum += w;
    if (seed.decision() * out.wsum < w) out.s = cand;
  }
  int px, py;
  const bool temporal = history && backproject_d(C, h.pos, px, py);
  if (temporal) {
    const DiPix &o = prev[(size_t)py * C.p->width + px];
    if (same_surface_d(pos, nrm, o.pos, o.nrm) && o.M > 0.0 && o.W > 0.0) {
      const double cM = std::min(o.M, 20.0);
      const double w = di_target_d(C, h.pos, h.n, h.gn, h.e1, dir0, m, o.s) * o.W * cM;
      out.M += cM;
      out.wsum += w;
      if (seed.decision() * out.wsum < w) out.s = o.s;
    }
  }
  const double pHat = di_target_d(C, h.pos, h.n, h.gn, h.e1, dir0, m, out.s);
  out.W = out.M > 0.0 && pHat > 0.0 ? out.wsum / (out.M * pHat) : 0.0;
  if ((int)C.p->max_depth - 1 < 1) return;
  double gwsum, gM = 1.0;
  GiS g = gi_initial_d(C, h, m, dir0, u, seed, gwsum);
  if (temporal) {
    const DiPix &o = prev[(size_t)py * C.p->width + px];
    if (same_surface_d(pos, nrm, o.pos, o.nrm) && o.gM > 0.0 && o.gW > 0.0 && o.g.pdf > 0.0 && o.g.valid &&
        gi_accepts_shift_d(h.pos, D3{o.pos[0], o.pos[1], o.pos[2]}, o.g.pos, o.g.nrm)) {
      const double cM = std::min(o.gM, 20.0);
      const double w = gi_target_d(C, h, dir0, m, o.g) * o.gW * cM;
      gM += cM;
      gwsum += w;
      if (seed.pcg() * gwsum < w) g = o.g;
    }
  }
  const double gHat = gi_target_d(C, h, dir0, m, g);
  out.g = g;
  out.gwsum = gwsum;
  out.gM = gM;
  out.gW = gM > 0.0 && gHat > 0.0 ? gwsum / (gM * gHat) : 0.0;
}

D3 di_shade_d(const PtContext &C, uint32_t x, uint32_t y, uint32_t si, uint32_t frame, float jx, float jy,
              const std::vector<DiPix> &cur) {
  ZSampler seed = ZSampler::pixel(x, y, C.p->width, si, C.p->sampler != 0u, C.p->z_temporal, frame);
  PtLanes L{};
  if (C.spectral) L = make_lanes(C, seed.wavelength_u());
  D3 dir0 = camera_dir_d(C, x, y, jx, jy), o0 = C.cam;
  lens_d(C, o0, dir0, seed);
  seed.state = pcg_hash(seed.state ^ 0x27d4eb2fu);
  const DiPix &me = cur[(size_t)y * C.p->width + x];
  if (me.pos[3] <= 0.0) return {0, 0, 0};
  const PtHit &h = me.hit;
  const vt_material m = pt_material(C, h.slot);
  if (m.type == VT_MAT_EMISSIVE) return primary_emission_d(C, L, h, m);
  if (m.type != VT_MAT_DIFFUSE) {
    // Other primaries: NEE with MIS (main.swift:7657-7672), none at glass or mirrors.
    const int limit = std::max(0, (int)C.p->max_depth - 1);
    const Spec4 T = C.spectral ? Spec4{{1, 1, 1, 1}} : Spec4{{1, 1, 1, 0}};
    D3 R{0, 0, 0};
    if (!is_delta_d(C, m)) {
      seed.event(1u, 1u);
      R = direct_d(C, L, h.pos, h.n, h.gn, h.e1, h.err, dir0 * -1.0, T, m, limit > 0, limit > 0, seed, true);
    }
    R = R + continue_path_d(C, L, h, m, dir0, seed, false);
    if (!std::isfinite(R.x) || !std::isfinite(R.y) || !std::isfinite(R.z)) R = {0, 0, 0};
    return R;
  }
  DiS sel = me.s;
  double wsum = di_target_d(C, h.pos, h.n, h.gn, h.e1, dir0, m, sel) * me.W * me.M, M = me.M;
  for (int t = 0; t < 4; ++t) {
    const double ox = seed.pcg(), oy = seed.pcg();
    const int nx = (int)x + (int)((ox * 2.0 - 1.0) * 16.0), ny = (int)y + (int)((oy * 2.0 - 1.0) * 16.0);
    if (nx < 0 || nx >= (int)C.p->width || ny < 0 || ny >= (int)C.p->height) continue;
    const DiPix &n = cur[(size_t)ny * C.p->width + nx];
    if (!compatible_d(me.pos, me.nrm, n.pos, n.nrm)) continue;
    if (!(n.M > 0.0 && n.W > 0.0)) continue;
    const double w = di_target_d(C, h.pos, h.n, h.gn, h.e1, dir0, m, n.s) * n.W * n.M;
    wsum += w;
    M += n.M;
    if (seed.decision() * wsum < w) sel = n.s;
  }
  const double pHat = di_target_d(C, h.pos, h.n, h.gn, h.e1, dir0, m, sel);
  const double W = M > 0.0 && pHat > 0.0 ? wsum / (M * pHat) : 0.0;
  D3 R{0, 0, 0};
  if (W > 0.0 && visible_d(C, h.pos, h.gn, h.err, light_from_di(sel, h.pos)))
    R = di_contribution_d(C, h.pos, h.n, h.gn, h.e1, dir0, m, sel) * W;
  if ((int)C.p->max_depth - 1 >= 1) {
    GiS gs = me.g;
    bool gvalid = me.g.valid;
    double gwsum = gvalid ? gi_target_d(C, h, dir0, m, gs) * me.gW * me.gM : 0.0, gM = me.gM;
    for (int t = 0; t < 4; ++t) {
      const double ox = seed.pcg(), oy = seed.pcg();
      const int nx = (int)x + (int)((ox * 2.0 - 1.0) * 16.0), ny = (int)y + (int)((oy * 2.0 - 1.0) * 16.0);
      if (nx < 0 || nx >= (int)C.p->width || ny < 0 || ny >= (int)C.p->height) continue;
      const DiPix &n = cur[(size_t)ny * C.p->width + nx];
      if (!compatible_d(me.pos, me.nrm, n.pos, n.nrm)) continue;
      if (n.gM <= 0.0 || n.gW <= 0.0 || n.g.pdf <= 0.0 || !n.g.valid) continue;
      if (!gi_accepts_shift_d(h.pos, D3{n.pos[0], n.pos[1], n.pos[2]}, n.g.pos, n.g.nrm)) continue;
      const double w = gi_target_d(C, h, dir0, m, n.g) * n.gW * n.gM;
      gwsum += w;
      gM += n.gM;
      if (seed.decision() * gwsum < w) {
        gs = n.g;
        gvalid = true;
      }
    }
    const double gHat = gvalid ? gi_target_d(C, h, dir0, m, gs) : 0.0;
    const double gW = gM > 0.0 && gHat > 0.0 ? gwsum / (gM * gHat) : 0.0;
    if (gW > 0.0 && gi_visible_d(C, h.pos, h.gn, gs.pos, h.err)) {
      const D3 dir = normalize(gs.pos - h.pos);
      PtLanes Ls{};
      if (C.spectral) Ls = make_lanes(C, gs.u);
      double pdf;
      const double f = lambert_eval_d(h.n, h.gn, dir0 * -1.0, dir, pdf);
      const double geometry = gi_geometry_d(h.pos, h.n, gs.pos, gs.nrm);
      R = R + to_rgb(C, Ls, scale(mul(reflectance(C, Ls, m), gs.rad), f * geometry * gW));
    }
  }
  R = R + continue_path_d(C, L, h, m, dir0, seed, true);
  if (!std::isfinite(R.x) || !std::isfinite(R.y) || !std::isfinite(R.z)) R = {0, 0, 0};
  return R;
}

D3 path_sample_d(const PtContext &C, uint32_t x, uint32_t y, uint32_t si, uint32_t frame, float jx_f, float jy_f) {
  ZSampler seed = ZSampler::pixel(x, y, C.p->width, si, C.p->sampler != 0u, C.p->z_temporal, frame);
  PtLanes L{};
  if (C.spectral) L = make_lanes(C, seed.wavelength_u());
  D3 dir0 = camera_dir_d(C, x, y, jx_f, jy_f), o0 = C.cam;
  lens_d(C, o0, dir0, seed);
  PtHit h;
  const bool hit0 = pt_closest(C, o0, dir0, h);
  seed.state = pcg_hash(seed.state ^ 0x27d4eb2fu);
  if (!hit0) return C.env ? environment_d(C, dir0) : D3{0, 0, 0};
  const vt_material m = pt_material(C, h.slot);
  if (m.type == VT_MAT_EMISSIVE) return primary_emission_d(C, L, h, m);
  const int limit = std::max(0, (int)C.p->max_depth - 1);
  D3 R{0, 0, 0};
  if (C.p->sampling_mode != 3u && !is_delta_d(C, m)) {  // no NEE at glass or mirrors (main.swift:7657)
    const Spec4 T = C.spectral ? Spec4{{1, 1, 1, 1}} : Spec4{{1, 1, 1, 0}};
    seed.event(1u, 1u);
    R = direct_d(C, L, h.pos, h.n, h.gn, h.e1, h.err, dir0 * -1.0, T, m, C.p->sampling_mode == 1u && limit > 0, limit > 0,
                 seed, true);
  }
  R = R + continue_path_d(C, L, h, m, dir0, seed, false);
  if (!std::isfinite(R.x) || !std::isfinite(R.y) || !std::isfinite(R.z)) R = {0, 0, 0};
  return R;
}

}  // namespace

extern "C" void vto_render(const vto_pt_inputs *in, const vt_frame_params *p, uint32_t spp, double *out_rgb,
                           int32_t threads) {
  PtContext C;
  C.in = in;
  C.p = p;
  // A prebuilt hierarchy (vto_bvh_import of the device's) skips the build; it stays the caller's.
  const bool ownBvh = in->bvh == nullptr;
  C.bvh = ownBvh ? vto_lbvh_build(in->faces, in->nfaces, in->verts, in->nverts, 2, 7, 2) : const_cast<vto_bvh *>(in->bvh);
  C.spectral = p->spectral != 0 && in->cmf_rgb != nullptr;
  C.mats.assign(in->materials, in->materials + in->nmat);
  for (uint32_t i = 0; i < in->nmat; ++i) std::memcpy(&C.mats[i].pad, &i, sizeof i);
  if (C.spectral) {
    // The uplift: each slot's albedo and the six saturated corners (main.swift:10730-10733).
    C.slotL.resize(in->nmat);
    for (uint32_t i = 0; i < in->nmat; ++i) {
      const double rgb[3] = {in->materials[i].albedo[0], in->materials[i].albedo[1], in->materials[i].albedo[2]};
      vto_spectral_lagrange(in->uplift, rgb, 1, C.slotL[i].data());
    }
    const double corners[18] = {1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 1, 1, 1, 0, 1, 1, 1, 0};
    double cl[24];
    vto_spectral_lagrange(in->uplift, corners, 6, cl);
    C.basis.resize(in->nbins);
    for (uint32_t b = 0; b < in->nbins; ++b)
      for (int k = 0; k < 6; ++k) C.basis[b][k] = vto_uplift_impl::spectral_value(cl + 4 * k, in->cos_phase[b]);
  }
  const D3 pos = d3(p->camera_pos), target = d3(p->camera_target), upv = d3(p->camera_up);
  C.cam = pos;
  C.fwd = normalize(target - pos);
  C.right = normalize(cross(C.fwd, upv));
  C.up = cross(C.right, C.fwd);
  C.aspect = double(p->width) / p->height;
  C.fovScale = std::tan(p->fov_deg * 0.5 * kPi / 180.0);
  C.larea = std::sqrt(dot(cross(d3(in->light.su), d3(in->light.sv)), cross(d3(in->light.su), d3(in->light.sv))));
  C.imported = in->imported != 0;
  if (C.imported && in->environment.intensity > 0.0f) {
    const vt_environment &e = in->environment;
    const double l = std::sqrt((double)e.sun_dir[0] * e.sun_dir[0] + (double)e.sun_dir[1] * e.sun_dir[1] +
                               (double)e.sun_dir[2] * e.sun_dir[2]);
    C.env = true;
    C.envIntensity = e.intensity;
    C.sunIntensity = e.sun_intensity;
    C.sunDir = D3{(float)(e.sun_dir[0] / l), (float)(e.sun_dir[1] / l), (float)(e.sun_dir[2] / l)};
    C.skyMode = e.sky_mode;
    if (in->env_rgba && in->env_w > 0 && in->env_h > 0) {
      C.envMap = true;
      C.envImg = in->env_rgba;
      C.envW = in->env_w;
      C.envH = in->env_h;
      C.envRot = in->env_rot;
      C.sunIntensity = 0.0;
      env_tables_d(C);
    }
  }
  if (C.imported) {
    // Per slot (rgb, selection weight max(1e-8, luminance) in float, main.swift:9303-9306).
    C.emis.assign(in->nmat, {0, 0, 0, 0});
    for (uint32_t i = 0; i < in->nmat; ++i) {
      const vt_material &mm = in->materials[i];
      if (mm.type != VT_MAT_EMISSIVE) continue;
      const float *e = mm.emission;
      const bool lit = double(e[0]) * e[0] + double(e[1]) * e[1] + double(e[2]) * e[2] > 0;
      const float lum = 0.2126f * e[0] + 0.7152f * e[1] + 0.0722f * e[2];
      C.emis[i] = {e[0], e[1], e[2], lit ? double(std::max(1e-8f, lum)) : 0.0};
    }
    C.E = in->emitters;
    C.ecount = in->nemitter_words ? in->emitters[0] : 0;
    if (C.ecount) {
      const uint32_t c = C.ecount;
      C.etotal = fword(C.E[2 * c + 1]);
      C.treeNodes = C.E[2 * c + 2];
      if (C.treeNodes) {
        C.ltNodes = C.E + C.E[2 * c + 3];
        C.ltLeaves = C.E + C.E[2 * c + 4];
        for (int k = 0; k < 3; ++k) {
          C.ltLo[k] = fword(C.E[2 * c + 5 + k]);
          C.ltScale[k] = (fword(C.E[2 * c + 8 + k]) - C.ltLo[k]) / 65535.0;
        }
      }
    }
  }
  std::vector<float> jx(spp), jy(spp);
  for (uint32_t k = 0; k < spp; ++k) {
    const uint32_t n = (std::max(1u, p->first_sample + k) - 1u) % 1024u + 1u;
    jx[k] = halton_f(n, 2) - 0.5f;
    jy[k] = halton_f(n, 3) - 0.5f;
  }
  const uint32_t npix = p->width * p->height;
  if (p->sampling_mode == 0u) {
    // ReSTIR DI: frames in order, each a primary pass over every pixel, then reuse and shading.
    const uint32_t M = p->di_candidates ? p->di_candidates : 4u;
    uint32_t bits = 0;
    while ((1u << bits) < M) ++bits;
    std::vector<DiPix> buf[2] = {std::vector<DiPix>(npix), std::vector<DiPix>(npix)};
    std::vector<double> sum(3 * (size_t)npix, 0.0);
    for (uint32_t k = 0; k < spp; ++k) {
      std::vector<DiPix> &cur = buf[k & 1u], &prev = buf[(k & 1u) ^ 1u];
      const uint32_t si = p->first_sample + k, frame = std::max(1u, p->first_frame) + k;
      parallel_for(npix, threads, [&](uint32_t i) {
        di_primary_d(C, i % p->width, i / p->width, si, frame, jx[k], jy[k], M, bits, k > 0, prev, cur[i]);
      });
      parallel_for(npix, threads, [&](uint32_t i) {
        const D3 c = di_shade_d(C, i % p->width, i / p->width, si, frame, jx[k], jy[k], cur);
        sum[3 * (size_t)i] += c.x; sum[3 * (size_t)i + 1] += c.y; sum[3 * (size_t)i + 2] += c.z;
      });
    }
    for (size_t i = 0; i < sum.size(); ++i) out_rgb[i] = spp ? sum[i] / spp : 0.0;
    if (ownBvh) vto_bvh_free(C.bvh);
    return;
  }
  // Pixel stride s (vt_frame_params.pixel_stride, sampling modes 1-3): every s-th pixel in x and y,
  // each with the full frame's camera ray and its own sample stream; ceil(w / s) x ceil(h / s) out.
  const uint32_t st = std::max(1u, p->pixel_stride), OW = (p->width + st - 1) / st, OH = (p->height + st - 1) / st;
  parallel_for(OW * OH, threads, [&](uint32_t i) {
    const uint32_t x = (i % OW) * st, y = (i / OW) * st;
    double s[3] = {0, 0, 0};
    for (uint32_t k = 0; k < spp; ++k) {
      const D3 c = path_sample_d(C, x, y, p->first_sample + k, std::max(1u, p->first_frame) + k, jx[k], jy[k]);
      s[0] += c.x; s[1] += c.y; s[2] += c.z;
    }
    for (int c = 0; c < 3; ++c) out_rgb[3 * (size_t)i + c] = spp ? s[c] / spp : 0.0;
  });
  if (ownBvh) vto_bvh_free(C.bvh);
}
