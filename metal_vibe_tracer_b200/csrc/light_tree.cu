// light_tree.cu — host side of the emitter lights: the light BVH build (LightTree.build,
// Sources/LightTree.swift:112-160) and the packed emitter list the integrator reads
// (MaterialLibrary's power-sampling list and lightTreeList, main.swift:9313-9345, 9374-9401).
//
// Host C++ in double precision, as the reference's builder: per node the union of its emitters'
// LightBounds (spatial box, power, normal cone, emission half-angle; pbrt-v4 LightBounds), a
// 12-bucket SAOH split per axis (pbrt-v4 BVHLightSampler::EvaluateCost), leaves of at most
// `max_leaf` emitters kept whole when the best split saves less than `leaf_ratio`, and 8-word
// nodes (octahedral cone axis, power, quantised cone cosines and bounds, child links) in
// depth-first order. Numbering, partition order and quantisation follow the reference exactly,
// so the words are comparable bit for bit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "vt_internal.cuh"

namespace {

constexpr int kBuckets = 12;
constexpr uint32_t kMaxNodes = (1u << 27) - 1u;
constexpr uint32_t kNoParent = kMaxNodes;
constexpr uint32_t kMaxDepth = 64;
const double kPi = 3.14159265358979323846;

struct V3 { double x, y, z; };
inline V3 v3(double x, double y, double z) { return {x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double at(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
inline double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(V3 a) { const double l = length(a); return {a.x / l, a.y / l, a.z / l}; }
inline V3 vmin(V3 a, V3 b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }
inline double clamp1(double c) { return std::min(1.0, std::max(-1.0, c)); }

const double kInf = std::numeric_limits<double>::infinity();

// pbrt-v4 AngleBetween (LightTree.angleBetween).
double angle_between(V3 a, V3 b) {
  if (dot(a, b) < 0) return kPi - 2 * std::asin(std::min(1.0, length(a + b) / 2));
  return 2 * std::asin(std::min(1.0, length(b - a) / 2));
}

// Rotation of v about the unit axis k by `angle`, through the unit quaternion (k sin(angle/2),
// cos(angle/2)): t = 2 (q.xyz x v), v' = v + q.w t + q.xyz x t.
V3 rotate(V3 v, V3 k, double angle) {
  const double s = std::sin(angle / 2), w = std::cos(angle / 2);
  const V3 q = k * s;
  const V3 t = cross(q, v) * 2.0;
  return v + t * w + cross(q, t);
}

// pbrt-v4 Union(DirectionCone, DirectionCone) (LightTree.coneUnion).
void cone_union(V3 wa, double ca, V3 wb, double cb, V3 &w, double &c) {
  const double thetaA = std::acos(clamp1(ca)), thetaB = std::acos(clamp1(cb));
  const double thetaD = angle_between(wa, wb);
  if (std::min(thetaD + thetaB, kPi) <= thetaA) { w = wa; c = ca; return; }
  if (std::min(thetaD + thetaA, kPi) <= thetaB) { w = wb; c = cb; return; }
  const double thetaO = (thetaA + thetaD + thetaB) / 2;
  if (thetaO >= kPi) { w = wa; c = -1; return; }
  const V3 axis = cross(wa, wb);
  if (dot(axis, axis) == 0) { w = wa; c = -1; return; }
  w = normalize(rotate(wa, normalize(axis), thetaO - thetaA));
  c = std::cos(thetaO);
}

// LightTree.Bounds (pbrt-v4 LightBounds).
struct Bounds {
  V3 lo{kInf, kInf, kInf}, hi{-kInf, -kInf, -kInf};
  double phi = 0;
  V3 w{0, 0, 1};
  double cosO = 1, cosE = 1;
  V3 centroid() const { return (lo + hi) * 0.5; }
};

Bounds emitter_bounds(const vt_emitter &e) {
  Bounds b;
  const V3 a = v3(e.a[0], e.a[1], e.a[2]), bb = v3(e.b[0], e.b[1], e.b[2]), c = v3(e.c[0], e.c[1], e.c[2]);
  b.lo = vmin(a, vmin(bb, c));
  b.hi = vmax(a, vmax(bb, c));
  const V3 n = cross(bb - a, c - a);
  const double len = length(n);
  b.phi = len > 0 && std::isfinite(e.power) ? std::max(0.0, e.power) : 0.0;
  b.w = len > 0 ? V3{n.x / len, n.y / len, n.z / len} : V3{0, 0, 1};
  b.cosO = 1;
  b.cosE = std::min(1.0, std::max(0.0, e.cos_emission));
  return b;
}

// pbrt-v4 Union(LightBounds, LightBounds): a powerless side contributes nothing.
Bounds unite(const Bounds &a, const Bounds &o) {
  if (a.phi == 0) return o;
  if (o.phi == 0) return a;
  Bounds r;
  r.lo = vmin(a.lo, o.lo);
  r.hi = vmax(a.hi, o.hi);
  r.phi = a.phi + o.phi;
  cone_union(a.w, a.cosO, o.w, o.cosO, r.w, r.cosO);
  r.cosE = std::min(a.cosE, o.cosE);
  return r;
}

// SAOH of a set of lights (LightTree.cost; axis < 0: no thin-split penalty).
double cost(const Bounds &b, V3 diag, int axis) {
  if (!(b.phi > 0)) return 0;
  const double thetaO = std::acos(clamp1(b.cosO)), thetaE = std::acos(clamp1(b.cosE));
  const double thetaW = std::min(thetaO + thetaE, kPi);
  const double sinO = std::sqrt(std::max(0.0, 1 - b.cosO * b.cosO));
  const double mOmega = 2 * kPi * (1 - b.cosO) +
                        kPi / 2 * (2 * thetaW * sinO - std::cos(thetaO - 2 * thetaW) - 2 * thetaO * sinO + b.cosO);
  const double kr = axis >= 0 ? std::max(std::max(diag.x, diag.y), diag.z) / std::max(at(diag, axis), 1e-300) : 1.0;
  const V3 d = b.hi - b.lo;
  const double area = 2 * (d.x * d.y + d.x * d.z + d.y * d.z);
  return b.phi * mOmega * kr * area;
}

struct Centroids { V3 lo{kInf, kInf, kInf}, hi{-kInf, -kInf, -kInf}; };
struct Split { double cost; int axis, bucket; };

int bucket_of(const Bounds &b, int axis, const Centroids &c) {
  const double lo = at(c.lo, axis), extent = at(c.hi, axis) - lo;
  return std::min(kBuckets - 1, (int)(double(kBuckets) * (at(b.centroid(), axis) - lo) / extent));
}

bool best_split(uint32_t begin, uint32_t end, const std::vector<Bounds> &bounds, const std::vector<int32_t> &order,
                const Bounds &node, const Centroids &cent, Split &best) {
  const V3 diag = node.hi - node.lo;
  bool found = false;
  for (int axis = 0; axis < 3; ++axis) {
    if (!(at(cent.hi, axis) > at(cent.lo, axis))) continue;
    Bounds bucket[kBuckets], below[kBuckets], above[kBuckets];
    for (uint32_t i = begin; i < end; ++i) {
      const Bounds &b = bounds[order[i]];
      const int k = bucket_of(b, axis, cent);
      bucket[k] = unite(bucket[k], b);
    }
    for (int k = 0; k < kBuckets; ++k) below[k] = k == 0 ? bucket[0] : unite(below[k - 1], bucket[k]);
    for (int k = kBuckets - 1; k >= 0; --k) above[k] = k == kBuckets - 1 ? bucket[k] : unite(above[k + 1], bucket[k]);
    for (int k = 0; k < kBuckets - 1; ++k) {
      if (!(below[k].phi > 0 || above[k + 1].phi > 0)) continue;
      const double c = cost(below[k], diag, axis) + cost(above[k + 1], diag, axis);
      if (c < (found ? best.cost : kInf)) { best = {c, axis, k}; found = true; }
    }
  }
  return found;
}

// The split's partition (two pointers from both ends, as the reference's partition(by:)), or the
// middle of the range when every centroid coincides or a side is empty.
uint32_t partition(std::vector<int32_t> &order, uint32_t begin, uint32_t end, const std::vector<Bounds> &bounds,
                   const Centroids &cent, const Split *split) {
  const uint32_t middle = begin + (end - begin) / 2;
  if (!split) return middle;
  auto second = [&](int32_t e) { return bucket_of(bounds[e], split->axis, cent) > split->bucket; };
  uint32_t lo = begin, hi = end;
  for (;;) {
    for (;;) {
      if (lo >= hi) goto done;
      if (second(order[lo])) break;
      ++lo;
    }
    for (;;) {
      --hi;
      if (lo >= hi) goto done;
      if (!second(order[hi])) break;
    }
    std::swap(order[lo], order[hi]);
    ++lo;
  }
done:
  return lo == begin || lo == end ? middle : lo;
}

// pbrt-v4 CompactLightBounds as 8 words (LightTree.node): bounds rounded outward in the grid,
// cosines rounded down.
uint32_t octahedral(V3 v) {
  const double s = std::fabs(v.x) + std::fabs(v.y) + std::fabs(v.z);
  double px = v.x / s, py = v.y / s;
  if (v.z < 0) {
    const double qx = (1 - std::fabs(py)) * (px >= 0 ? 1 : -1), qy = (1 - std::fabs(px)) * (py >= 0 ? 1 : -1);
    px = qx;
    py = qy;
  }
  auto e = [](double x) { return (uint32_t)std::min(65535.0, std::max(0.0, std::round((x * 0.5 + 0.5) * 65535))); };
  return e(px) | e(py) << 16;
}

void emit_node(std::vector<uint32_t> &words, const Bounds &b, const float glo[3], const float ghi[3], uint32_t child,
               uint32_t parent, uint32_t leafCount) {
  auto q = [&](double v, int axis, bool up) -> uint32_t {
    const double g = glo[axis], extent = double(ghi[axis]) - g;
    if (!(extent > 0) || !std::isfinite(v)) return up ? 65535u : 0u;
    const double x = (v - g) / extent * 65535;
    return (uint32_t)std::min(65535.0, std::max(0.0, up ? std::ceil(x) : std::floor(x)));
  };
  auto qcos = [](double c) { return (uint32_t)std::min(65535.0, std::max(0.0, std::floor((c + 1) / 2 * 65535))); };
  const uint32_t lo0 = q(b.lo.x, 0, false), lo1 = q(b.lo.y, 1, false), lo2 = q(b.lo.z, 2, false);
  const uint32_t hi0 = q(b.hi.x, 0, true), hi1 = q(b.hi.y, 1, true), hi2 = q(b.hi.z, 2, true);
  const float phi = (float)b.phi;
  uint32_t phiBits;
  std::memcpy(&phiBits, &phi, 4);
  const uint32_t w[8] = {octahedral(b.w), phiBits, qcos(b.cosO) | qcos(b.cosE) << 16, lo0 | lo1 << 16, lo2 | hi0 << 16,
                         hi1 | hi2 << 16, child, parent | leafCount << 27};
  words.insert(words.end(), w, w + 8);
}

}  // namespace

// LightTree.build (Sources/LightTree.swift:112-160).
vt_status vt_light_tree_compute(const vt_emitter *emitters, uint32_t count, uint32_t maxLeaf, double leafRatio,
                                vt_light_tree &out) {
  out.words.clear();
  out.order.resize(count);
  out.leaf_node.assign(count, 0);
  out.node_count = 0;
  out.depth = 0;
  std::vector<Bounds> bounds(count);
  V3 glo{kInf, kInf, kInf}, ghi{-kInf, -kInf, -kInf};
  for (uint32_t i = 0; i < count; ++i) {
    bounds[i] = emitter_bounds(emitters[i]);
    glo = vmin(glo, bounds[i].lo);
    ghi = vmax(ghi, bounds[i].hi);
  }
  for (int k = 0; k < 3; ++k) {
    out.grid_lo[k] = count ? std::nextafter((float)at(glo, k), -INFINITY) : 0.0f;
    out.grid_hi[k] = count ? std::nextafter((float)at(ghi, k), INFINITY) : 0.0f;
  }
  for (uint32_t i = 0; i < count; ++i) out.order[i] = (int32_t)i;
  struct Work { uint32_t begin, end, parent; bool second; uint32_t level; };
  std::vector<Work> work;
  if (count) work.push_back({0, count, kNoParent, false, 0});
  out.words.reserve(8 * std::max<size_t>(1, 2 * (size_t)count));
  while (!work.empty()) {
    const Work it = work.back();
    work.pop_back();
    const uint32_t index = out.node_count++;
    if (out.node_count > kMaxNodes) return VT_ERR_LIMIT;
    out.depth = std::max(out.depth, it.level);
    if (it.second) out.words[8 * (size_t)it.parent + 6] = index;
    Bounds total;
    Centroids cent;
    for (uint32_t i = it.begin; i < it.end; ++i) {
      const Bounds &b = bounds[out.order[i]];
      total = unite(total, b);
      cent.lo = vmin(cent.lo, b.centroid());
      cent.hi = vmax(cent.hi, b.centroid());
    }
    if (total.phi == 0) {
      for (uint32_t i = it.begin; i < it.end; ++i) {
        total.lo = vmin(total.lo, bounds[out.order[i]].lo);
        total.hi = vmax(total.hi, bounds[out.order[i]].hi);
      }
    }
    const uint32_t n = it.end - it.begin;
    Split split{};
    const bool has = n > 1 && best_split(it.begin, it.end, bounds, out.order, total, cent, split);
    const bool leaf = n == 1 || (n <= maxLeaf && (total.phi == 0 ||
                                                  (has ? split.cost : kInf) >= leafRatio * cost(total, total.hi - total.lo, -1)));
    if (leaf) {
      for (uint32_t i = it.begin; i < it.end; ++i) out.leaf_node[i] = index;
      emit_node(out.words, total, out.grid_lo, out.grid_hi, it.begin, it.parent, n);
      continue;
    }
    const uint32_t mid = partition(out.order, it.begin, it.end, bounds, cent, has ? &split : nullptr);
    emit_node(out.words, total, out.grid_lo, out.grid_hi, 0, it.parent, 0);
    work.push_back({mid, it.end, index, true, it.level + 1});
    work.push_back({it.begin, mid, index, false, it.level + 1});
  }
  return VT_OK;
}

namespace {
uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
}  // namespace

// The packed emitter list (main.swift:9313-9345, 9374-9401). Entries are (id, power) sorted by id.
// Power sampling: [count, ids, cdf (last 1), total, 0]. Light tree (when asked for, more than one
// emitter, the build splits them and the GPU can walk it): [count, ids, leaf positions, total,
// node count, node offset, leaf offset, grid lo, grid hi, padding to 16 bytes, nodes (8 words),
// per leaf position (id, power, leaf node)]. No power: [0, 0].
vt_status vt_emitter_list_compute(const uint32_t *ids, const vt_emitter *emitters, uint32_t count, bool lightTree,
                                  std::vector<uint32_t> &words, vt_light_tree *treeOut) {
  words.clear();
  double total = 0.0;
  std::vector<double> cumulative(count);
  for (uint32_t i = 0; i < count; ++i) {
    total += emitters[i].power;
    cumulative[i] = total;
  }
  if (!(total > 0) || !std::isfinite(total)) {
    words = {0u, 0u};
    return VT_OK;
  }
  if (lightTree && count > 1) {
    vt_light_tree tree;
    const vt_status st = vt_light_tree_compute(emitters, count, 8, 0.75, tree);
    if (st != VT_OK) return st;
    if (tree.node_count > 1 && tree.depth <= kMaxDepth && tree.node_count < kMaxNodes) {
      std::vector<uint32_t> position(count);
      for (uint32_t leaf = 0; leaf < count; ++leaf) position[tree.order[leaf]] = leaf;
      words.push_back(count);
      words.insert(words.end(), ids, ids + count);
      words.insert(words.end(), position.begin(), position.end());
      words.push_back(fbits((float)total));
      uint32_t nodeOffset = (uint32_t)words.size() + 9;
      while (nodeOffset % 4) ++nodeOffset;
      const uint32_t leafOffset = nodeOffset + (uint32_t)tree.words.size();
      words.push_back(tree.node_count);
      words.push_back(nodeOffset);
      words.push_back(leafOffset);
      for (int k = 0; k < 3; ++k) words.push_back(fbits(tree.grid_lo[k]));
      for (int k = 0; k < 3; ++k) words.push_back(fbits(tree.grid_hi[k]));
      words.resize(nodeOffset, 0u);
      words.insert(words.end(), tree.words.begin(), tree.words.end());
      for (uint32_t leaf = 0; leaf < count; ++leaf) {
        const uint32_t input = (uint32_t)tree.order[leaf];
        words.push_back(ids[input]);
        words.push_back(fbits((float)emitters[input].power));
        words.push_back(tree.leaf_node[leaf]);
      }
      if (treeOut) *treeOut = std::move(tree);
      return VT_OK;
    }
  }
  words.push_back(count);
  words.insert(words.end(), ids, ids + count);
  for (uint32_t i = 0; i < count; ++i) words.push_back(fbits(i == count - 1 ? 1.0f : (float)(cumulative[i] / total)));
  words.push_back(fbits((float)total));
  words.push_back(0u);
  return VT_OK;
}

extern "C" {

vt_status vt_light_tree_build(vt_ctx *ctx, const vt_emitter *emitters, uint32_t n, uint32_t max_leaf,
                              double leaf_ratio, vt_light_tree **out) {
  if (!out || (n && !emitters)) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  *out = nullptr;
  if (max_leaf < 1 || max_leaf > 31) return vt_fail(ctx, VT_ERR_INVALID, "max_leaf must be 1-31 (5-bit leaf count)");
  if (!(leaf_ratio >= 0.0)) return vt_fail(ctx, VT_ERR_INVALID, "leaf_ratio must be >= 0");
  vt_light_tree *t = new vt_light_tree();
  const vt_status st = vt_light_tree_compute(emitters, n, max_leaf, leaf_ratio, *t);
  if (st != VT_OK) {
    delete t;
    return vt_fail(ctx, st, "light tree exceeds 2^27 - 1 nodes");
  }
  *out = t;
  return VT_OK;
}

vt_status vt_light_tree_destroy(vt_ctx *ctx, vt_light_tree *tree) {
  (void)ctx;
  delete tree;
  return VT_OK;
}

vt_status vt_light_tree_get_info(vt_ctx *ctx, const vt_light_tree *tree, vt_light_tree_info *info) {
  if (!tree || !info) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  std::memset(info, 0, sizeof *info);
  info->node_count = tree->node_count;
  info->depth = tree->depth;
  info->count = (uint32_t)tree->order.size();
  for (int k = 0; k < 3; ++k) {
    info->grid_lo[k] = tree->grid_lo[k];
    info->grid_hi[k] = tree->grid_hi[k];
  }
  return VT_OK;
}

vt_status vt_light_tree_get_words(vt_ctx *ctx, const vt_light_tree *tree, uint32_t *words, uint32_t n) {
  if (!tree || (n && !words)) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  if (n != tree->words.size()) return vt_fail(ctx, VT_ERR_INVALID, "n must be 8 * node_count");
  std::copy(tree->words.begin(), tree->words.end(), words);
  return VT_OK;
}

vt_status vt_light_tree_get_order(vt_ctx *ctx, const vt_light_tree *tree, int32_t *order, uint32_t *leaf_nodes,
                                  uint32_t n) {
  if (!tree || (n && (!order || !leaf_nodes))) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  if (n != tree->order.size()) return vt_fail(ctx, VT_ERR_INVALID, "n must equal the emitter count");
  std::copy(tree->order.begin(), tree->order.end(), order);
  std::copy(tree->leaf_node.begin(), tree->leaf_node.end(), leaf_nodes);
  return VT_OK;
}

vt_status vt_emitter_list_pack(vt_ctx *ctx, const uint32_t *ids, const vt_emitter *emitters, uint32_t n,
                               uint32_t light_tree, uint32_t *words, uint32_t capacity, uint32_t *count) {
  if (!count || (n && (!ids || !emitters))) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  for (uint32_t i = 1; i < n; ++i)
    if (ids[i] <= ids[i - 1]) return vt_fail(ctx, VT_ERR_INVALID, "emitter ids must be strictly increasing");
  std::vector<uint32_t> w;
  const vt_status st = vt_emitter_list_compute(ids, emitters, n, light_tree != 0, w, nullptr);
  if (st != VT_OK) return vt_fail(ctx, st, "light tree exceeds 2^27 - 1 nodes");
  *count = (uint32_t)w.size();
  if (words) {
    if (capacity < w.size()) return vt_fail(ctx, VT_ERR_INVALID, "capacity below the list's word count");
    std::copy(w.begin(), w.end(), words);
  }
  return VT_OK;
}

}  // extern "C"
