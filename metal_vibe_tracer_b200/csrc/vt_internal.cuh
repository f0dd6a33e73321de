// vt_internal.cuh — shared device/host definitions of libvt_b200 (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/vt.h"

// ---------------------------------------------------------------------------------------------
// Context and mesh objects behind the opaque C handles.

struct vt_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;        // the context's own stream
  cudaStream_t pipe[2] = {nullptr, nullptr};  // host-buffer pipelining (copy in, trace, copy out)
  std::string error;
  uint32_t *d_status = nullptr;         // device-side error word (build validation, kernels)
  uint32_t *d_counters = nullptr;       // scratch: ray-queue heads (kQueueSlots words, one per
                                        // launch in rotation) then the count accumulators
  uint32_t next_slot = 0;               // next ray-queue slot
  // Host-pipeline device buffers (allocated on first use, grown as needed).
  void *d_chunk_in[2] = {nullptr, nullptr};
  void *d_chunk_out[2] = {nullptr, nullptr};
  size_t chunk_in_bytes = 0, chunk_out_bytes = 0;
  // Pinned host staging for callers' pageable buffers (allocated on first use, grown as needed), and
  // per staging slot the event recorded after its chunk's copy back.
  void *h_stage_in[2] = {nullptr, nullptr};
  void *h_stage_out[2] = {nullptr, nullptr};
  size_t stage_in_bytes = 0, stage_out_bytes = 0;
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  // Ray-ordering scratch (keys, permutation, sort buffers), grown on demand. One per pipeline
  // stream plus one for caller streams, so concurrent launches do not share it.
  uint32_t *d_order[3] = {nullptr, nullptr, nullptr};
  size_t order_words[3] = {0, 0, 0};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // RGB -> spectrum uplift (spectral.cu), built once per context: the moment grid (86^3 float4
  // nodes, then refined 64-entry blocks) and the 86 node values; the colour model it was solved for.
  float4 *d_fgrid = nullptr;
  float *d_gnodes = nullptr;
  uint32_t fgrid_cells = 0;        // refined cells
  uint32_t fgrid_flagged = 0;      // cells flagged (before the capacity cap)
  double fgrid_residual = 0.0;     // largest linear-sRGB residual of the coarse solves
  std::vector<double> fgrid_model; // weights and cos phase it was solved with
  // OpenPBR energy tables (openpbr.cu): the dense metal table (129 x 129) and its averages (129),
  // then the opaque-dielectric energy complement (32^3) and its average (32^2), as floats.
  float *d_pbr = nullptr;
  bool pbr_opaque = false;         // the opaque-dielectric tables are set
};

// Traversal copy of a 4-wide node with 8-bit child boxes (qnode.cu): 64 bytes, two 32-byte loads.
struct __align__(64) vt_qnode {
  uint32_t w[16];
};

struct vt_mesh {
  uint32_t nfaces = 0;
  uint32_t nnodes = 0;       // 4-wide nodes
  uint32_t depth = 0;        // 4-wide depth (root = 1)
  float root_max = 0.0f;     // max |coordinate| over the scene bounds (slab enlargement)
  float sah = 0.0f;
  float build_ms = 0.0f;
  float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  vt_wide_node *d_nodes = nullptr;   // nnodes, reference layout (128 B, 16-B vector loads)
  float4 *d_tris = nullptr;          // 3 per BVH position: (a, face id bits), (b, face tag bits), (c, 0)
  int32_t *d_order = nullptr;        // BVH position -> input face
  uint32_t *d_codes = nullptr;       // sorted Morton codes
  int32_t *d_sorted = nullptr;       // sorted position -> input face
  int32_t *d_bin_child = nullptr;    // 2 per binary internal node (refined)
  float *d_bin_box = nullptr;        // 8 per binary internal node (lo xyz, -, hi xyz, -)
  vt_qnode *d_qnodes = nullptr;      // nnodes, quantised copy read by the traversal kernels
  float4 *d_nrm = nullptr;           // 3 per BVH position: the vertex normals (smooth shading)
};

// Light BVH (host words, LightTree.Built).
struct vt_light_tree {
  std::vector<uint32_t> words;
  std::vector<int32_t> order;
  std::vector<uint32_t> leaf_node;
  uint32_t node_count = 0, depth = 0;
  float grid_lo[3] = {0, 0, 0}, grid_hi[3] = {0, 0, 0};
};
vt_status vt_light_tree_compute(const vt_emitter *emitters, uint32_t count, uint32_t maxLeaf, double leafRatio,
                                vt_light_tree &out);
vt_status vt_emitter_list_compute(const uint32_t *ids, const vt_emitter *emitters, uint32_t count, bool lightTree,
                                  std::vector<uint32_t> &words, vt_light_tree *treeOut);

struct vt_scene {
  const vt_mesh *mesh = nullptr;
  // Imported scenes (emissive triangles, no quad light): the packed emitter list, per slot
  // (emission rgb, selection weight), and face -> BVH position.
  bool imported = false;
  vt_environment environment{};  // procedural sky and sun of an imported scene (intensity 0: none)
  // Environment image (vt_scene_set_environment_map): pixels, marginal row CDFs (2 x height) and
  // conditional column CDFs (width x 2 height), its size and rotation; env_map when it is set.
  float4 *d_env_img = nullptr;
  float *d_env_rows = nullptr, *d_env_cols = nullptr;
  uint32_t env_w = 0, env_h = 0;
  float env_rot = 0.0f;
  bool env_map = false;
  uint32_t *d_emitters = nullptr;
  std::vector<uint32_t> emitter_words;
  float4 *d_emissions = nullptr;
  int32_t *d_face_pos = nullptr;
  vt_material *d_mats = nullptr;
  uint32_t nmat = 0;
  bool layered = false;  // some slot is OPENPBR, GLOSSY or DIELECTRIC
  std::vector<int32_t> slot_types;  // host copies: each slot's type and roughness (vt_scene_set_openpbr)
  std::vector<float> slot_rough;
  bool has_film = false;  // some slot has a thin film (vt_scene_set_openpbr)
  vt_quad_light light;
  // Spectral tables: per 1 nm bin (cmf r, g, b, illuminant), the inverse CDF.
  float4 *d_spec = nullptr;
  float *d_icdf = nullptr;
  uint32_t nbins = 0, segments = 0;
  float lambda_min = 0.0f;
  // FP64 accumulation (3 doubles per pixel) and its sample count.
  double *d_accum = nullptr;
  uint32_t width = 0, height = 0, samples = 0;
  float2 *d_jitter = nullptr;
  uint32_t jitter_cap = 0;
  // ReSTIR DI (sampling mode 0): per pixel the primary-surface cache (position, normal) and the
  // reservoir (sample position, emission and pdf, weights) for this frame and the previous one,
  // plus the primary hit's face/slot/error and geometric normal: 12 float4 per pixel in one
  // allocation.
  // OpenPBR slots (vt_scene_set_openpbr): per slot (roughness, metalness, IOR, diffuse roughness),
  // and the context's energy tables.
  float4 *d_pbr = nullptr;
  const float *pbr_tables = nullptr;
  // Spectral uplift: per slot the albedo's multipliers, per bin the phase and the emission basis.
  float4 *d_slotL = nullptr;
  float *d_cosphase = nullptr;
  float4 *d_ebasis = nullptr;
  float4 *d_di = nullptr;
  uint32_t di_width = 0, di_height = 0, di_frames = 0, di_parity = 0;
  // Wavefront integrator (vt_render_wavefront): the paths' state, rays and queues, one allocation
  // sized for wf_cap paths.
  unsigned char *d_wf = nullptr;
  uint32_t wf_cap = 0;
  float di_cam[14] = {};  // previous frame's camera: position, forward, right, up, aspect, fov scale
};

// ---------------------------------------------------------------------------------------------
// Error plumbing.

vt_status vt_fail(vt_ctx *ctx, vt_status code, const std::string &msg);
// RGB -> spectrum uplift (spectral.cu): build the context's moment grid for the tables' colour model
// (once), uplift host colours into device (L0, L1, L2, flag) quadruples, and tabulate the emission
// basis at device bins of the given phase.
vt_status vt_uplift_ensure(vt_ctx *ctx, const vt_spectral_tables *tables);
vt_status vt_uplift_colours(vt_ctx *ctx, const float *rgb, uint32_t n, float4 *out_dev);
vt_status vt_uplift_basis(vt_ctx *ctx, const float *cosPhase_dev, uint32_t nbins, float4 *basis_dev);
// OpenPBR (openpbr.cu): solve the metal energy table once per context and, with `tables`, set the
// opaque-dielectric tables.
vt_status vt_openpbr_ensure(vt_ctx *ctx, const vt_openpbr_tables *tables);
vt_status vt_cuda_fail(vt_ctx *ctx, cudaError_t err, const char *what);

#define VT_CUDA(ctx, call)                                   \
  do {                                                       \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return vt_cuda_fail(ctx, _e, #call); \
  } while (0)

// Ray-queue slots: consecutive traversal launches take slots in rotation (32 bytes apart), so up
// to kQueueSlots launches of one context may run concurrently on different streams.
constexpr uint32_t kQueueSlots = 16;
constexpr uint32_t kCounterWords = kQueueSlots * 8 + 8;  // + two uint64 count accumulators
inline uint32_t *vt_queue_slot(vt_ctx *ctx) {
  uint32_t *p = ctx->d_counters + 8 * (ctx->next_slot % kQueueSlots);
  ++ctx->next_slot;
  return p;
}
inline unsigned long long *vt_count_words(vt_ctx *ctx) {
  return reinterpret_cast<unsigned long long *>(ctx->d_counters + kQueueSlots * 8);
}
// A spare counter word after the accumulators (host-synchronised uses on the context stream).
inline uint32_t *vt_scratch_word(vt_ctx *ctx) { return ctx->d_counters + kQueueSlots * 8 + 4; }

// Device error word bits (ctx->d_status).
enum : uint32_t {
  VT_DEV_BAD_INDEX = 1u,       // a face indexes past the vertex array
  VT_DEV_NONFINITE = 2u,       // a vertex position is NaN or infinite
  VT_DEV_STACK = 4u,           // traversal stack overflow
  VT_DEV_TREELET = 8u,         // treelet restructuring hit an internal inconsistency
  VT_DEV_NORMALS = 16u         // information, not an error: some vertex normal is nonzero
};

// ---------------------------------------------------------------------------------------------
// Build helpers implemented in scan_sort.cu / lbvh.cu.

// Exclusive prefix sum of n uint32 values (in place allowed). `temp` must hold
// vt_scan_temp_words(n) words. Returns the total through *total_dev if non-null (device word).
size_t vt_scan_temp_words(uint32_t n);
void vt_scan_exclusive(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *temp,
                       uint32_t *total_dev, cudaStream_t s);

// Stable LSD radix sort of (key, value) pairs on the low `bits` bits of the keys.
// keys/vals are sorted in place using the alternate buffers; temp is vt_radix_temp_words(n).
size_t vt_radix_temp_words(uint32_t n);
void vt_radix_sort_pairs(uint32_t *keys, uint32_t *vals, uint32_t *keys_alt, uint32_t *vals_alt,
                         uint32_t n, int bits, uint32_t *temp, cudaStream_t s);

vt_status vt_quantize_nodes(vt_ctx *ctx, vt_mesh *mesh, cudaStream_t s);
vt_status vt_lbvh_build(vt_ctx *ctx, const vt_face *faces, uint32_t nfaces, const vt_vertex *verts,
                        uint32_t nverts, const vt_build_options &opt, vt_mesh *mesh);

// Traversal launches (traverse.cu).
// Persistent kernels; `counter` is one device word of scratch (the ray queue head), reset by the
// launch on stream s.
// `status` receives VT_DEV_STACK if a traversal stack would overflow (it cannot for a tree within
// the mesh's recorded depth; the check keeps a corrupted tree from writing out of bounds).
// `count` (optional): the queue length on the device, at most n (the wavefront integrator's queues);
// `bvhPos`: hits report BVH positions instead of input faces; `slack`: shadow rays end each
// triangle's rounding bound early (imported scenes).
void vt_launch_closest(const vt_mesh *mesh, const vt_ray *rays, uint32_t n, vt_hit *hits,
                       int sm_count, uint32_t *counter, const uint32_t *perm, uint32_t *status,
                       cudaStream_t s, const uint32_t *count = nullptr, bool bvhPos = false);
void vt_launch_any(const vt_mesh *mesh, const vt_ray *rays, uint32_t n, uint8_t *occ,
                   int sm_count, uint32_t *counter, const uint32_t *perm, uint32_t *status,
                   cudaStream_t s, const uint32_t *count = nullptr, bool slack = false);
// Ray ordering for large batches: returns the device permutation (inside `scratch`, which must
// hold vt_ray_order_words(n) words) or nullptr when the batch is traced in input order.
size_t vt_ray_order_words(uint32_t n);
const uint32_t *vt_ray_order(const vt_mesh *mesh, const vt_ray *rays, uint32_t n, uint32_t *scratch,
                             cudaStream_t s);
void vt_launch_count(const vt_mesh *mesh, const vt_ray *rays, uint32_t n, int closest,
                     unsigned long long *acc /* 2 device words */, cudaStream_t s);
