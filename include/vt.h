/*
 * vt.h — C ABI of the B200 rendering hot path (libvt_b200.so).
 *
 * The reference renderer is a Swift host that builds its acceleration structures on the CPU
 * and dispatches Metal kernels. Each entry point below replaces one reference interface; the
 * comment above it names the reference file:line it stands in for. Signatures carry plain
 * pointers, sizes and POD structs only: no CUDA, torch or C++ types. A stream argument is a
 * cudaStream_t passed as `void *` (NULL = the CUDA default stream, as in the CUDA runtime).
 * Builds run on the context's own stream and return only when the structure is complete.
 *
 * Errors: every call returns a vt_status. A non-zero status leaves a human-readable message in
 * vt_last_error(ctx) (the role of MaterialLibrary.error(String), Sources/Acceleration.swift:733,
 * and of renderFrame's onError callback, main.swift:11199-11202). A context is single-threaded,
 * like the reference's @MainActor renderer.
 */
#ifndef VT_H
#define VT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VT_ABI_VERSION 1u

typedef int32_t vt_status;
enum {
  VT_OK = 0,
  VT_ERR_INVALID = 1,   /* bad argument (null pointer, out-of-range index, bad size) */
  VT_ERR_CUDA = 2,      /* a CUDA runtime call failed; the message holds cudaGetErrorString */
  VT_ERR_MEMORY = 3,    /* device allocation failed or the scene exceeds the memory budget */
  VT_ERR_LIMIT = 4,     /* a structural limit was exceeded (BVH depth vs traversal stack, sizes) */
  VT_ERR_DEVICE = 5     /* a kernel reported an error status (bounded wait expired, stack overflow) */
};

typedef struct vt_ctx vt_ctx;
typedef struct vt_mesh vt_mesh;

/* MSL MeshFace (main.swift:616, Sources/Acceleration.swift:62): three absolute vertex indices
 * and the stored tag (material slot / subset). 16 bytes. */
typedef struct vt_face { uint32_t a, b, c, tag; } vt_face;

/* MSL MeshVertex (main.swift:615, Sources/Acceleration.swift:61): position, normal, uv. 32 B. */
typedef struct vt_vertex { float px, py, pz, nx, ny, nz, u, v; } vt_vertex;

/* MSL MeshWideNode (main.swift:617, Sources/Acceleration.swift:23-30): 4-wide node, 128 bytes.
 * Child k is an inner node (> 0, index of the node), a leaf (< 0: -(first + 1) with count[k]
 * triangles starting at `first` in BVH order) or empty (0). Node 0 is the root. */
typedef struct vt_wide_node {
  float lox[4], loy[4], loz[4], hix[4], hiy[4], hiz[4];
  int32_t child[4];
  int32_t count[4];
} vt_wide_node;

/* A ray with its parametric interval [tmin, tmax). 32 bytes, two 16-byte vectors. */
typedef struct vt_ray { float ox, oy, oz, tmin, dx, dy, dz, tmax; } vt_ray;

/* Closest-hit record (the MSL MeshHit, main.swift:1843): t, barycentrics b1/b2 weighting
 * vertices b and c, and the hit face's index in the caller's input order (-1 = miss). 16 B. */
typedef struct vt_hit { float t, b1, b2; int32_t prim; } vt_hit;

/* Build options. Zero-initialised fields take the defaults noted. */
typedef struct vt_build_options {
  int32_t leaf_size;          /* triangles per wide-BVH leaf, 1..8 (default 2, the reference BLAS
                                 leaf size, Sources/Acceleration.swift:692) */
  int32_t treelet_size;       /* SAH treelet restructuring: leaves per treelet, 0 = default 7,
                                 -1 = plain LBVH (no refinement) */
  int32_t refine_rounds;      /* restructuring rounds (default 2) */
  int32_t max_depth;          /* reject trees deeper than this (default 31; stack bound) */
} vt_build_options;

typedef struct vt_mesh_info {
  uint32_t faces;             /* triangles in the mesh */
  uint32_t wide_nodes;        /* 4-wide nodes (vt_mesh_get_nodes count) */
  uint32_t binary_nodes;      /* internal nodes of the binary LBVH (faces - 1) */
  uint32_t depth;             /* 4-wide depth, root = 1 */
  float sah_cost;             /* SAH cost of the 4-wide tree (node cost 1, triangle cost 1) */
  float build_ms;             /* device time of the last build, ms */
  float lo[3], hi[3];         /* scene bounds */
} vt_mesh_info;

/* ---- context ---------------------------------------------------------------------------- */

/* Creates a context on CUDA device `device` with its own stream. Replaces PathTracerRenderer's
 * init(device:) (main.swift:9513) for the traversal and build paths. */
vt_status vt_ctx_create(int32_t device, vt_ctx **out);
vt_status vt_ctx_destroy(vt_ctx *ctx);
/* Message of the last failing call on `ctx` ("" if none). Valid until the next call. */
const char *vt_last_error(const vt_ctx *ctx);
uint32_t vt_abi_version(void);
/* Blocks until the context's stream has drained. */
vt_status vt_sync(vt_ctx *ctx);

/* ---- mesh publish / BVH build ------------------------------------------------------------- */

/* Builds a mesh's acceleration structure on the device from caller-owned HOST arrays (copied).
 * Replaces MaterialLibrary.setMesh -> publishTwoLevel (Sources/Acceleration.swift:652-782) and
 * WideBVH.build(bounds:count:leafSize:depth:) (Sources/Acceleration.swift:296) for one asset:
 * a GPU LBVH (30-bit Morton codes, radix sort, Karras hierarchy), SAH treelet restructuring and
 * a collapse to the reference's 4-wide node layout. Face indices must be < nverts. */
vt_status vt_mesh_build(vt_ctx *ctx, const vt_face *faces, uint32_t nfaces, const vt_vertex *verts,
                        uint32_t nverts, const vt_build_options *opts, vt_mesh **out);
/* The same from DEVICE arrays (no host copy). */
vt_status vt_mesh_build_device(vt_ctx *ctx, const vt_face *faces_dev, uint32_t nfaces,
                               const vt_vertex *verts_dev, uint32_t nverts,
                               const vt_build_options *opts, vt_mesh **out);
vt_status vt_mesh_destroy(vt_ctx *ctx, vt_mesh *mesh);
vt_status vt_mesh_get_info(vt_ctx *ctx, const vt_mesh *mesh, vt_mesh_info *out);
/* BVH leaf order (WideBVH.Result.order, Sources/Acceleration.swift:107-110): order[i] is the input
 * face stored at BVH position i. `n` must equal the face count. Host output. */
vt_status vt_mesh_get_order(vt_ctx *ctx, const vt_mesh *mesh, int32_t *order, uint32_t n);
/* The 4-wide nodes (WideBVH.Result.nodes). `n` must equal info.wide_nodes. Host output. */
vt_status vt_mesh_get_nodes(vt_ctx *ctx, const vt_mesh *mesh, vt_wide_node *nodes, uint32_t n);
/* Sorted 30-bit Morton codes of the face centroids (parity of the LBVH's first stage), and the
 * sorted face indices they belong to (before restructuring). Host outputs of `n` = face count. */
vt_status vt_mesh_get_morton(vt_ctx *ctx, const vt_mesh *mesh, uint32_t *codes, int32_t *sorted,
                             uint32_t n);
/* Binary LBVH after refinement: per internal node its two children (>= 0 internal index,
 * < 0 leaf -(sorted position + 1)) and its box (lo xyz, hi xyz). `n` = faces - 1. Host outputs. */
vt_status vt_mesh_get_binary(vt_ctx *ctx, const vt_mesh *mesh, int32_t *children /* 2n */,
                             float *boxes /* 6n */, uint32_t n);

/* ---- traversal ----------------------------------------------------------------------------- */

/* Closest hit of `n` DEVICE rays; writes `n` DEVICE hits. Replaces mesh_closest/blas_closest
 * (main.swift:1788-1812, 1843-1901): watertight triangle test (main.swift:1536-1582), conservative
 * 4-wide slab test (main.swift:1758-1785), nearest child first. Stream-ordered, asynchronous. */
vt_status vt_trace_closest(vt_ctx *ctx, const vt_mesh *mesh, const vt_ray *rays_dev, uint32_t n,
                           vt_hit *hits_dev, void *stream);
/* Any hit in [tmin, tmax) of `n` DEVICE rays; writes one byte per ray (1 = occluded). Replaces
 * mesh_occluded/blas_any (main.swift:1815-1838, 1902-1984) without endpoint slack. */
vt_status vt_trace_any(vt_ctx *ctx, const vt_mesh *mesh, const vt_ray *rays_dev, uint32_t n,
                       uint8_t *occluded_dev, void *stream);
/* The same from HOST arrays: copies in, traces and copies out in pipelined chunks of 2^22 rays on
 * the context's two streams, then synchronises. Pinned (or registered) buffers are copied directly;
 * ordinary pageable buffers go through the context's pinned staging buffers (allocated on first
 * use), filled and drained by up to 8 host threads while the GPU works on the neighbouring chunk. */
vt_status vt_trace_closest_host(vt_ctx *ctx, const vt_mesh *mesh, const vt_ray *rays, uint32_t n,
                                vt_hit *hits);
vt_status vt_trace_any_host(vt_ctx *ctx, const vt_mesh *mesh, const vt_ray *rays, uint32_t n,
                            uint8_t *occluded);

/* Per-ray traversal counters for the roofline: wide nodes fetched and triangles tested, summed
 * over `n` DEVICE rays into two host uint64 values. A separate instrumented kernel; it does not
 * slow the traversal entry points. closest = 1 counts closest-hit traversal, 0 any-hit. */
vt_status vt_trace_count(vt_ctx *ctx, const vt_mesh *mesh, const vt_ray *rays_dev, uint32_t n,
                         int32_t closest, uint64_t *nodes_visited, uint64_t *tris_tested);

/* ---- two-level hierarchy (instances of meshes) ----------------------------------------------- */

typedef struct vt_tlas vt_tlas;

/* One placed copy of a mesh (MeshLayout.addInstance, Sources/Acceleration.swift:474-516). 64 B. */
typedef struct vt_instance {
  float world[12];      /* object -> world transform, row-major 3 x 4 (the rows of MeshInstance.world,
                           main.swift:1609) */
  uint32_t mesh;        /* index into vt_tlas_build's mesh array */
  uint32_t slot_base;   /* added to the mesh's face tags (material slots) by vt_tlas_flatten */
  uint32_t reserved[2]; /* 0 */
} vt_instance;

/* An instance as the device holds it (MeshInstance, main.swift:1609; MeshInstanceRecord,
 * Sources/Acceleration.swift:545-557). 128 B (the reference record without its binding word, which serves scene-graph slots). */
typedef struct vt_instance_record {
  float world[12];      /* object -> world, row-major 3 x 4 */
  float local[12];      /* world -> object: the inverse, computed in double and rounded once */
  uint32_t mesh;        /* the instance's mesh */
  uint32_t slot_base;
  uint32_t rendered_base; /* first rendered triangle: sum of the faces of the instances before it */
  uint32_t mirrored;    /* 1 when det(world) < 0 (flattening swaps vertices b and c) */
  float bound[4];       /* max |translation|, infinity norm of the linear part, the mesh's max
                           |coordinate|, 0 */
} vt_instance_record;

typedef struct vt_tlas_info {
  uint32_t instances;   /* instances in the hierarchy */
  uint32_t meshes;      /* meshes it references */
  uint32_t nodes;       /* 4-wide TLAS nodes */
  uint32_t depth;       /* TLAS depth, root = 1 */
  uint64_t rendered_triangles; /* sum over instances of their mesh's faces */
  float lo[3], hi[3];   /* world bounds (the union of the instance boxes) */
  float grow;           /* per-ray TLAS box growth factor 2^-18 (1 + largest condition number of an
                           instance's linear part) (MeshSceneHeader.lo.w) */
  float reach;          /* max over instances of |translation| + norm(linear) * mesh max |coordinate|
                           (MeshSceneHeader.hi.w) */
  float build_ms;       /* device time of the TLAS build */
  float pad;
} vt_tlas_info;

/* Builds the two-level hierarchy: a 4-wide TLAS (leaf size 1) over the instances' world boxes
 * (the mesh's box corners transformed, enlarged by 2^-20 reach), whose leaves name instances, over
 * the meshes' own hierarchies (the BLAS). Replaces MeshSceneLayout.sceneBlob (Sources/
 * Acceleration.swift:519-573). The meshes must outlive the TLAS. Rejects (VT_ERR_INVALID) a mesh
 * index out of range, a transform with a non-finite entry, a first-column scale outside
 * [1e-6, 1e6], |det| <= 1e-18 or a reach of 1e8 or more (the reference's "Combined hierarchy scale
 * exceeds the supported range.", "Singular USD transform.", "Hierarchy transform exceeds the
 * supported scene extent."). */
vt_status vt_tlas_build(vt_ctx *ctx, const vt_mesh *const *meshes, uint32_t nmeshes, const vt_instance *instances,
                        uint32_t ninstances, vt_tlas **out);
vt_status vt_tlas_destroy(vt_ctx *ctx, vt_tlas *tlas);
vt_status vt_tlas_get_info(vt_ctx *ctx, const vt_tlas *tlas, vt_tlas_info *out);
/* The TLAS nodes (leaf children name instances: -(instance + 1), count 1). `n` = info.nodes. */
vt_status vt_tlas_get_nodes(vt_ctx *ctx, const vt_tlas *tlas, vt_wide_node *nodes, uint32_t n);
/* The instance records. `n` = info.instances. */
vt_status vt_tlas_get_instances(vt_ctx *ctx, const vt_tlas *tlas, vt_instance_record *records, uint32_t n);
/* Closest hit of `n` DEVICE world rays through the two levels (mesh_closest, main.swift:1840-1901):
 * the TLAS boxes grown per ray by grow * (max|origin| + reach), instances in near-to-far order,
 * each traced in object space (the ray transformed by `local`, its direction not renormalised, so t
 * is the world ray's). Hits carry the instance's mesh face (input order); `instances_dev` (may be
 * NULL) receives the hit instance (0xFFFFFFFF on a miss). */
vt_status vt_tlas_trace_closest(vt_ctx *ctx, const vt_tlas *tlas, const vt_ray *rays_dev, uint32_t n,
                                vt_hit *hits_dev, uint32_t *instances_dev, void *stream);
/* Any hit in [tmin, tmax) through the two levels (mesh_occluded, main.swift:1957-1984), without
 * endpoint slack. */
vt_status vt_tlas_trace_any(vt_ctx *ctx, const vt_tlas *tlas, const vt_ray *rays_dev, uint32_t n,
                            uint8_t *occluded_dev, void *stream);
/* One world-space mesh of every instance's triangles (SceneGraph.forEachRenderTriangle, as
 * instance_triangle renders them, main.swift:1645-1668): rendered face rendered_base + f is the
 * instance's face f with vertices transformed by `world`, normals by the inverse transpose, tag +
 * slot_base, b and c swapped when mirrored; then built like vt_mesh_build_device. */
vt_status vt_tlas_flatten(vt_ctx *ctx, const vt_tlas *tlas, const vt_build_options *opts, vt_mesh **out);

/* ---- path tracing (integrator) ------------------------------------------------------------- */

typedef struct vt_scene vt_scene;

/* Material types: the reference's MaterialType values (main.swift:316-322). GLOSSY is a metal: an
 * ideal mirror below roughness 0.02 (Schlick's conductor Fresnel with F0 = albedo), else the OpenPBR
 * BSDF with metalness 1. DIELECTRIC is ideal glass (Schlick's Fresnel at the slot's IOR, albedo as
 * the tint). Their roughness and IOR come from the slot's vt_openpbr_params; without them a GLOSSY
 * slot is a mirror and a DIELECTRIC slot has IOR 1.5. */
enum { VT_MAT_DIFFUSE = 0, VT_MAT_GLOSSY = 1, VT_MAT_DIELECTRIC = 2, VT_MAT_EMISSIVE = 3, VT_MAT_OPENPBR = 4 };

/* A constant material slot (the role of SurfaceSettings / MaterialResources, main.swift:2253-2263,
 * 628-654, for constant Lambert and emissive surfaces). A face's tag selects its slot. 32 bytes. */
typedef struct vt_material {
  int32_t type;        /* VT_MAT_*; albedo is the base colour (OPENPBR), F0 (GLOSSY) or the tint (DIELECTRIC) */
  float albedo[3];     /* linear sRGB reflectance (Lambert) */
  float emission[3];   /* linear sRGB radiance (emissive) */
  float pad;
} vt_material;

/* The procedural area light of the reference's scenes 1/3/4 (sample_direct_light, main.swift:
 * 2957-2978; eval_light_pdf, main.swift:3046-3050): a parallelogram corner + u su + v sv emitting
 * towards `normal`. The scene's emissive faces should cover the same quad. 64 bytes. */
typedef struct vt_quad_light {
  float corner[3], su[3], sv[3], normal[3];
  float emission[3];   /* radiance, linear sRGB (the light tint applied) */
  float pad;
} vt_quad_light;

/* Spectral transport tables (1 nm bins from lambda_min): linear-sRGB colour-matching functions,
 * the emitters' illuminant (luminance 1) and the wavelength inverse CDF (segments + 1 nodes); the
 * roles of the spectral sampling buffer written by spectral_icdf_kernel (main.swift:8117-8185).
 * The uplift part is the colour model of the RGB -> spectrum conversion (bounded MESE of three
 * trigonometric moments, main.swift:842-944): per nm over the model's range (360-830 nm, uplift_n
 * = 471) the linear-sRGB CMFs times D65 (Y = 1) and the cosine of Peters' warped phase, in double,
 * plus the cosine at each of the render bins. The moment grid is solved from it on the device
 * (vt_spectral_grid_build) and reflectances and emitters use it at the path's wavelengths. */
typedef struct vt_spectral_tables {
  const float *cmf_rgb;     /* nbins x 3 */
  const float *illuminant;  /* nbins */
  const float *icdf;        /* segments + 1 */
  uint32_t nbins, segments;
  float lambda_min;
  uint32_t pad;
  const float *cos_phase;        /* nbins: cos(phi(lambda)) at the render bins */
  const double *uplift_weights;  /* uplift_n x 3 */
  const double *uplift_cos;      /* uplift_n */
  uint32_t uplift_n, pad2;
} vt_spectral_tables;

/* Per-frame parameters: the subset of Uniforms (main.swift:393-420) the integrator reads. */
typedef struct vt_frame_params {
  float camera_pos[3];
  float fov_deg;            /* vertical field of view (Uniforms.cameraPos.w) */
  float camera_target[3];
  uint32_t max_depth;       /* path depth, 1 = direct light only (Uniforms.cameraTarget.w) */
  float camera_up[3];
  uint32_t sampling_mode;   /* 0 = ReSTIR DI at the primary vertex, MIS elsewhere; 1 = NEE + BSDF
                               with power-heuristic MIS; 2 = light sampling (NEE); 3 = BSDF sampling
                               (Uniforms.samplingMode 0-3) */
  uint32_t width, height;
  uint32_t first_sample;    /* sample index of the first frame (>= 1, Uniforms.sampleIndex) */
  uint32_t spectral;        /* 1 = four hero wavelengths, 0 = RGB transport */
  uint32_t sampler;         /* 0 = PCG streams, 1 = Z++ sampler (Uniforms.indirectReuse bit 6) */
  uint32_t z_temporal;      /* Z++ temporal model 0-3 (bits 7-8; the reference's default is 3) */
  uint32_t first_frame;     /* accumulation frame of the first sample (Uniforms.frameIndex, >= 1);
                               0 = continue the scene's accumulation */
  uint32_t di_candidates;   /* ReSTIR DI initial candidates per pixel (sampling_mode 0); 0 = the
                               reference's 4 (restir_di_initial, main.swift:4646) */
  float aperture;           /* thin-lens radius, 0 = pinhole (Uniforms.lens.x, lens_ray,
                               main.swift:2210-2216) */
  float focus_distance;     /* distance to the plane in focus along the view axis (Uniforms.lens.y) */
  uint32_t pixel_stride;    /* 0 or 1: every pixel; s > 1: only pixels (s i, s j) of the width x
                               height frame, with the full frame's camera rays and sample streams,
                               into a ceil(width / s) x ceil(height / s) accumulation (sampling
                               modes 1-3; a subsampled render of the same image, for long reference
                               renders and sampled error measurements) */
} vt_frame_params;

/* A renderable scene: the mesh, its material slots, the area light and (optionally) the spectral
 * tables, plus the FP64 accumulation. Replaces MaterialLibrary.bind + the renderer's resources
 * (main.swift:9432-9449, 11016-11154). Host arrays are copied. */
vt_status vt_scene_create(vt_ctx *ctx, const vt_mesh *mesh, const vt_material *materials, uint32_t nmat,
                          const vt_quad_light *light, const vt_spectral_tables *tables, vt_scene **out);
vt_status vt_scene_destroy(vt_ctx *ctx, vt_scene *scene);
/* Renders `spp` frames (sample indices first_sample .. first_sample + spp - 1, one sample per pixel
 * each, jittered by the reference's frameJitter) and adds them to the scene's FP64 accumulation.
 * Replaces renderFrame(output:samples:) / encodeSample (main.swift:10978, 11214-11708) for the
 * MIS integrator: camera ray, closest hit, NEE with MIS, BSDF continuation, Russian roulette
 * (shading_kernel, main.swift:7370-7914). Resizing (a new width/height) resets the accumulation.
 * Stream-ordered; NULL = the CUDA default stream. */
vt_status vt_render(vt_ctx *ctx, vt_scene *scene, const vt_frame_params *params, uint32_t spp, void *stream);
/* The same frames and samples (sampling modes 1-3) through the wavefront integrator: the paths'
 * state lives in device memory between stage kernels over queues of live paths (camera rays;
 * per bounce the closest-hit traversal of the queue, shading with NEE and the BSDF continuation,
 * the shadow rays' any-hit traversal; then the accumulation), with the megakernel's sampler draws
 * and arithmetic per path; a path's primary and continuation radiance are summed apart, so the image
 * equals vt_render's to float rounding (1e-6 relative per pixel). The
 * reference has no wavefront path; its design note proposes the split (docs/KERNEL_SPLIT_DESIGN.md:
 * 72-74). Paths per pass are capped at 4M (whole samples of the frame); the state takes ~250 bytes
 * per path, allocated with the scene on first use. */
vt_status vt_render_wavefront(vt_ctx *ctx, vt_scene *scene, const vt_frame_params *params, uint32_t spp, void *stream);
vt_status vt_accum_reset(vt_ctx *ctx, vt_scene *scene);
/* Mean radiance per pixel (linear sRGB, row-major, 3 doubles per pixel; n = width * height * 3
 * of the accumulation, ceil(width / s) * ceil(height / s) * 3 for a pixel stride s) and the number
 * of samples accumulated. Synchronises. */
vt_status vt_accum_readback(vt_ctx *ctx, vt_scene *scene, double *rgb, uint32_t n, uint32_t *samples);
/* Resumes an accumulation saved from vt_accum_readback: sets the scene's FP64 accumulation to
 * rgb x samples (the FP64 sums) and its sample count to `samples`, for a width x height frame at
 * pixel stride s (n as vt_accum_readback's). The next vt_render continues it (first_sample =
 * samples + 1 continues the same sample streams). A long render (the 64k-spp FP64 reference) is
 * taken in pieces this way. No counterpart in the reference, whose accumulation restarts on any
 * change (main.swift:10993-11009). */
vt_status vt_accum_restore(vt_ctx *ctx, vt_scene *scene, uint32_t width, uint32_t height, uint32_t pixel_stride,
                           const double *rgb, uint32_t n, uint32_t samples);

/* The ReSTIR DI reservoirs of the last frame rendered in sampling mode 0, for checking reuse: per
 * pixel (weight sum, M, W, wavelength number), 4 floats into the HOST array out (n = width *
 * height * 4). M counts the frame's candidates plus the confidence merged from the previous frame
 * (capped at 20, restir_di_merge, main.swift:4686-4699). vt_accum_reset clears the history. */
vt_status vt_scene_di_weights(vt_ctx *ctx, const vt_scene *scene, float *out, uint32_t n);
/* The same for the ReSTIR GI reservoirs of the last mode-0 frame (restir_gi_encode, main.swift:
 * 4797-4806): per pixel (weight sum, M, W, wavelength number); M 0 where no GI reservoir was built
 * (non-diffuse primaries, depth 1). */
vt_status vt_scene_gi_weights(vt_ctx *ctx, const vt_scene *scene, float *out, uint32_t n);

/* Per pixel the first draws of one sampling event (vertex, stream) of the pixel's sampler: rand_f,
 * rand_f2 and rand_f3, 6 floats per pixel into the HOST array `out` (width * height * 6). The
 * role of the reference's z_frame test kernel (tests/Fix_zsampling.swift:58-66), for checking the
 * sampler against a CPU restatement. sampler 0 = PCG, 1 = Z++ with temporal model z_temporal. */
vt_status vt_sampler_frame(vt_ctx *ctx, uint32_t width, uint32_t height, uint32_t sampler, uint32_t z_temporal,
                           uint32_t sample_index, uint32_t frame_index, uint32_t vertex, uint32_t stream,
                           float *out);

/* The reference's device known answers (regression_checks, tests/GPUChecks.swift:14-37), evaluated
 * by the integrator's own device functions on the reference's inputs, VT_KNOWN_ANSWERS floats into
 * the HOST array `out`: [0] power_heuristic(1e-10, 1e-10); [1..3] emission_weight(false, true,
 * false, 0.2, 1), (true, true, true, 0, 1), (false, false, false, 0.2, 1); [4] the second PCG draw
 * from seed 890625759; [5] the cosine of the grazing cosine-hemisphere sample drawn from that seed
 * against its normal; [6..7] min and max of 100,000 rand_f draws from seed 17; [8..10]
 * scattering_limit of depths 0, 1, 8; [11..15] the glass total-internal-reflection sample
 * (GPUChecks.swift:32-34): 1 when it exists, its direction's z, its weight rgb. */
#define VT_KNOWN_ANSWERS 16u
vt_status vt_known_answers(vt_ctx *ctx, float *out, uint32_t n);

/* ---- batched scenes ---------------------------------------------------------------------- */

/* Many scenes of uneven size rendered by one persistent launch per pass (config C4; no counterpart
 * in the reference, which renders one scene per encodeSample). Each pass renders spp[i] frames of
 * scene i (sampling modes 1-3) into its accumulation, items being (scene, pixel) pairs handed out
 * to warps by an atomic work counter. The first passes try six launch shapes (64/128/256 threads,
 * 1 or 4 items per lane per fetch), one per pass, and keep the fastest, which later passes replay
 * as one captured CUDA graph. Sample and frame indices advance on the device. A scene belongs to
 * at most one live batch, and must not be rendered otherwise while its batch lives. */
typedef struct vt_batch vt_batch;
typedef struct vt_batch_info {
  uint32_t scenes, passes;
  unsigned long long items;   /* pixels per pass */
  float last_ms;              /* the last pass, device time */
  uint32_t tuned;             /* 1 once the launch shape is chosen (and, for the megakernel, captured) */
  uint32_t block, chunk;      /* the launch shape (chunk: megakernel items per grab): for the megakernel
                                 the chosen one once tuned, for the wavefront the last pass's */
  uint32_t wavefront;         /* 1: the batch renders through vt_batch_render_wavefront */
  uint32_t queue_paths;       /* wavefront: paths per pass of a scene's queues (the last pass's) */
  uint32_t compact_every;     /* wavefront: the live queue is compacted on every n-th bounce */
  uint32_t streams;           /* wavefront: streams the scenes are spread over */
} vt_batch_info;
vt_status vt_batch_create(vt_ctx *ctx, vt_scene *const *scenes, const vt_frame_params *params, const uint32_t *spp,
                          uint32_t n, vt_batch **out);
/* One pass; synchronises (it times the pass). */
vt_status vt_batch_render(vt_ctx *ctx, vt_batch *batch, void *stream);
/* One pass through the wavefront integrator instead (config C4's per-scene ray queues): each scene's
 * spp[i] frames run as vt_render_wavefront's stages over its own queues, the scenes spread over four
 * streams (longest first, each to the least loaded stream, one path-state buffer per stream) and the
 * camera jitter computed on the device. The first passes try, one each, the queue size (1M or 4M
 * paths per wavefront pass; only sizes that hold the largest frame), the stage kernels' block size
 * (128 or 256) and the compaction frequency (every bounce, or every second bounce with ended paths
 * kept in place); later passes use the fastest. Images equal vt_render_wavefront's of the same
 * frames (FP64 summation order aside). A batch renders through one integrator: after a wavefront pass
 * vt_batch_render refuses it, and the other way round. Synchronises (it times the pass). */
vt_status vt_batch_render_wavefront(vt_ctx *ctx, vt_batch *batch, void *stream);
/* Statistics of the last pass; scene_ms (n = scene count, may be NULL) receives each scene's
 * completion time from the pass's start, in ms. */
vt_status vt_batch_stats(vt_ctx *ctx, const vt_batch *batch, vt_batch_info *out, double *scene_ms, uint32_t n);
vt_status vt_batch_destroy(vt_ctx *ctx, vt_batch *batch);

/* ---- RGB -> spectrum uplift (spectral.cu) ------------------------------------------------------ */
/* Solves the uplift's moment grid on the device for the tables' colour model, once per context
 * (a second call with the same model returns at once; another model is an error). The reference
 * ships the 86^3 grid solved offline (scripts/generate_spectral_tables.py: solve_lagrange,
 * moments_of_lagrange; FourierSRGB86.bin) and refines it on the GPU (refineSpectralGrid,
 * main.swift:10658-10705): here both steps run as kernels. Scene creation with spectral tables
 * calls this itself. */
vt_status vt_spectral_grid_build(vt_ctx *ctx, const vt_spectral_tables *tables);

typedef struct vt_spectral_grid_info {
  uint32_t built;          /* 1 once the grid is solved */
  uint32_t refined_cells;  /* cells given exact 4x4x4 blocks (at most 8192) */
  uint32_t flagged_cells;  /* cells whose interpolation missed a code by more than 0.35 steps */
  uint32_t pad;
  double max_residual;     /* largest linear-sRGB residual of the coarse solves */
} vt_spectral_grid_info;
vt_status vt_spectral_grid_get_info(vt_ctx *ctx, vt_spectral_grid_info *out);
/* The grid as float4 (c0, c1, c2, refined slot + 1 or 0): 86^3 nodes then 64 per refined cell;
 * n = 4 * (86^3 + 64 * refined_cells) floats. */
vt_status vt_spectral_grid_read(vt_ctx *ctx, float *out, uint32_t n);
/* spectral_lagrange (main.swift:889-897) of n linear colours (rgb n x 3) on the device: per colour
 * (L0, L1, L2, 1), or (value, 0, 0, 2) for a grey. */
vt_status vt_spectral_lagrange(vt_ctx *ctx, const float *rgb, uint32_t n, float *out);
/* Every 8-bit sRGB code through the runtime conversion (grid, multipliers, reflectance at 1 nm,
 * back to sRGB under D65), on the device: the largest error in 8-bit steps and how many codes
 * miss by more than half a step (the reference's round-trip check, tests/Fix_spectral.swift). */
vt_status vt_spectral_round_trip(vt_ctx *ctx, float *worst, uint32_t *over_half);

/* ---- OpenPBR materials (openpbr.cu) ------------------------------------------------------------ */
/* The layered BSDF of the reference's OPENPBR material type (prepare_openpbr, main.swift:2485-2512,
 * around the vendored Adobe openpbr-bsdf) for opaque materials: specular_weight, base colour,
 * metalness, specular roughness and IOR, diffuse roughness, thin film (spectral transport), coat and
 * fuzz as the adapter sets them; transmission and anisotropy are not supported. Its data: the dense
 * metal table is solved on the device (the reference's Shaders/MetalEnergy.metal); the
 * opaque-dielectric energy complement tables (32^3 and 32^2 unorm16) and the fuzz lobe's LTC table
 * (32 x 32 x 3 floats), the upstream library's data, come from the caller, once per context. */
typedef struct vt_openpbr_tables {
  const uint16_t *opaque_energy;   /* 32 x 32 x 32: IOR, sqrt(alpha), cos */
  const uint16_t *opaque_average;  /* 32 x 32: IOR, sqrt(alpha) */
  const float *ltc;                /* 32 x 32 x 3: the fuzz lobe's LTC fit (a_inv, b_inv, R); rows roughness, columns cos */
} vt_openpbr_tables;
vt_status vt_openpbr_tables_set(vt_ctx *ctx, const vt_openpbr_tables *tables);
/* The dense isotropic GGX energy complement (129 x 129: roughness i/128, sqrt(cos) j/128) and its
 * per-roughness average (129), as solved on the device. */
vt_status vt_openpbr_energy_table(vt_ctx *ctx, float *table, float *average);

/* One BSDF query: an OPENPBR material's parameters as the adapter reads them (roughness and IOR are
 * clamped to >= 0.03 and >= 1.01 inside), a unit shading normal, the view (outward) and light
 * directions, and three random numbers for a sample. 128 bytes. */
typedef struct vt_openpbr_case {
  float base_color[3], metalness, roughness, ior, specular_weight, diffuse_roughness;
  float normal[3], view[3], light[3], rand[3];
  float thin_film_weight, thin_film_thickness /* micrometres */, thin_film_ior;
  float lambda[3];      /* the preparation's wavelengths in nm; 0: the upstream RGB wavelengths */
  float coat, fuzz;     /* coat and fuzz weights */
  /* specular_roughness_anisotropy in [0, 1] and the unit surface tangent it is oriented by (the
   * adapter's mat.tangent: used when anisotropy > 0, |tangent|^2 > 0.5 and |tangent . normal| < 0.99) */
  float anisotropy, tangent[3];
} vt_openpbr_case;
/* f |cos| at the light direction and its pdf; the sample: direction, weight f |cos| / pdf, its pdf,
 * and 1 when a sample was produced. 48 bytes. */
typedef struct vt_openpbr_result {
  float f_cos[3], pdf;
  float dir[3], weight[3], sample_pdf, ok;
} vt_openpbr_result;
/* openpbr_prepare + openpbr_eval / openpbr_pdf / openpbr_sample for n queries on the device. */
vt_status vt_openpbr_evaluate(vt_ctx *ctx, const vt_openpbr_case *cases, uint32_t n, vt_openpbr_result *out);

/* A scene's per-slot lobe parameters (SurfaceSettings surface/detail, main.swift:2253-2263, as
 * resolve_material sets them; base colour is the slot's albedo): one per material slot, read for
 * OPENPBR slots, for GLOSSY slots (roughness, IOR, thin film) and for DIELECTRIC slots (IOR). Needs
 * vt_openpbr_tables_set on the context first. */
typedef struct vt_openpbr_params {
  float roughness, metalness, ior, diffuse_roughness;
  /* Thin-film iridescence (SpectralMaterial, main.swift:730-735; spectral transport only, as the
   * reference's adapter): weight in [0, 1], thickness in micrometres, IOR. */
  float thin_film_weight, thin_film_thickness, thin_film_ior;
  /* Coat weight in [0, 1] (main.swift:2494; the adapter's coat: roughness 0.12, IOR 1.6, white). */
  float coat;
  /* Fuzz weight in [0, 1] (main.swift:2497; the upstream default fuzz: roughness 0.5, white). */
  float fuzz;
  /* specular_roughness_anisotropy in [0, 1] (main.swift:2496), oriented by the surface tangent: a mesh
   * without UVs takes the triangle's first edge b - a made perpendicular to the shading normal
   * (mesh_hit_attributes, main.swift:1594-1599). */
  float anisotropy;
  float pad[2];
} vt_openpbr_params;
vt_status vt_scene_set_openpbr(vt_ctx *ctx, vt_scene *scene, const vt_openpbr_params *params, uint32_t n);

/* ---- emitter lights: light tree and emitter list ----------------------------------------- */

/* One emitter triangle (LightTree.Emitter, Sources/LightTree.swift:11-16): world corners, power
 * (area x selection weight) and the cosine of the emission half-angle (0 = one-sided Lambertian).
 * 56 bytes. */
typedef struct vt_emitter {
  float a[3], b[3], c[3];
  float pad;
  double power;
  double cos_emission;
} vt_emitter;

/* A light BVH built on the host (LightTree.Built, Sources/LightTree.swift:100-108). */
typedef struct vt_light_tree vt_light_tree;
typedef struct vt_light_tree_info {
  uint32_t node_count, depth, count, pad;
  float grid_lo[3], grid_hi[3];   /* the box node bounds are quantised in */
} vt_light_tree_info;

/* LightTree.build(_:maxLeaf:leafRatio:) (Sources/LightTree.swift:112): 8 words per node in
 * depth-first order (LightTree.node, :190-203), `order` mapping leaf positions to input emitters
 * and each leaf position's node. The reference's defaults are max_leaf 8, leaf_ratio 0.75.
 * Host only, no device work: ctx may be NULL (errors then go to vt_last_error(NULL)), as for the
 * getters and vt_emitter_list_pack. */
vt_status vt_light_tree_build(vt_ctx *ctx, const vt_emitter *emitters, uint32_t n, uint32_t max_leaf,
                              double leaf_ratio, vt_light_tree **out);
vt_status vt_light_tree_destroy(vt_ctx *ctx, vt_light_tree *tree);
vt_status vt_light_tree_get_info(vt_ctx *ctx, const vt_light_tree *tree, vt_light_tree_info *info);
/* n = 8 * node_count */
vt_status vt_light_tree_get_words(vt_ctx *ctx, const vt_light_tree *tree, uint32_t *words, uint32_t n);
/* n = emitter count: order[leaf position] = input emitter, leaf_nodes[leaf position] = its node */
vt_status vt_light_tree_get_order(vt_ctx *ctx, const vt_light_tree *tree, int32_t *order, uint32_t *leaf_nodes,
                                  uint32_t n);

/* The packed emitter list the integrator reads (MaterialLibrary's list, main.swift:9313-9345, and
 * lightTreeList, :9374-9401) for emitters with strictly increasing ids. Power sampling:
 * [count, ids, cdf, total, 0]; with light_tree = 1 (more than one emitter, and a tree the build
 * splits and the GPU can walk): [count, ids, leaf positions, total, node count, node offset,
 * leaf offset, grid lo/hi, padding to 16 bytes, nodes, per leaf position (id, power, leaf node)].
 * `count` receives the word count; words may be NULL to query it. Host only. */
vt_status vt_emitter_list_pack(vt_ctx *ctx, const uint32_t *ids, const vt_emitter *emitters, uint32_t n,
                               uint32_t light_tree, uint32_t *words, uint32_t capacity, uint32_t *count);

/* A scene lit by its emissive triangles: the reference's imported scenes (sceneIndex 6 with a scene
 * graph), replacing vt_scene_create's quad light. Every face whose slot is VT_MAT_EMISSIVE with
 * non-zero emission is an emitter with the selection weight max(1e-8, luminance) (main.swift:
 * 9300-9309); the emitter ids are input face indices. NEE chooses an emitter by power or, with
 * light_tree = 1, by walking the light tree (sample_direct_light / light_tree_sample, main.swift:
 * 2892-2912, 2807-2833); BSDF hits on emitters weigh with the matching density (light_tree_pmf,
 * imported_emitter_area_pdf, :2835-2850, 2871-2881). Emitters emit from their front face
 * (cross(b - a, c - a)). Offsets and tolerances are the reference's imported-scene rounding bounds
 * (ray_epsilon, mesh_hit_error, endpoint_tolerance, ray_t_min, main.swift:1343-1364). */
vt_status vt_scene_create_imported(vt_ctx *ctx, const vt_mesh *mesh, const vt_material *materials, uint32_t nmat,
                                   const vt_spectral_tables *tables, uint32_t light_tree, vt_scene **out);
/* The scene's packed emitter list (see vt_emitter_list_pack); words may be NULL to query the
 * count. */
vt_status vt_scene_emitter_words(vt_ctx *ctx, const vt_scene *scene, uint32_t *words, uint32_t capacity,
                                 uint32_t *count);
/* The reference's light-selection check (lt_estimate, tests/Fix_light-tree.swift:66-93) on an
 * imported scene: thread i takes the receiver points[i / per_point] (4 floats, xyz used), seeds
 * pcg_hash(i * 7919 + 3) and draws `samples` light samples. It writes 8 floats per thread to the
 * HOST array out: the sum and sum of squares of luminance / pdf, the samples whose traced ray hit
 * the sampled triangle, those with a zero BSDF-hit pdf, the largest relative pdf difference, the
 * samples that chose a back-facing emitter, 0, 0. */
vt_status vt_light_estimate(vt_ctx *ctx, const vt_scene *scene, const float *points, uint32_t npoints,
                            uint32_t per_point, uint32_t samples, float *out);

/* ---- environment of imported scenes ------------------------------------------------------------
 * The reference's procedural sky and sun for sceneIndex 6 (eval_procedural_sky, main.swift:541-597;
 * eval_environment, :2127-2134): three presets of sky gradient with a sun lobe and a sun disc.
 * Next-event estimation splits its samples between the emitter triangles (half of them when both
 * exist, imported_light_probability, :2716-2719) and the environment (the sun cone with probability
 * 0.6 while the sun is above the horizon, else a cosine lobe about the receiver's normal,
 * :2922-2955); rays that escape pick up the environment with the power-heuristic weight against that
 * density (:7751-7756) and camera rays that miss see it directly (:7453-7455). Spectral transport
 * upsamples it as a D65-relative colour. Not built: image maps (environment.z), their rotation, the
 * compensated sampling tables, imported DistantLight suns and other sun illuminants. */
typedef struct vt_environment {
  float intensity;      /* Uniforms.environment.x: the sky's scale; 0 = no environment */
  float sun_dir[3];     /* Uniforms.sunParams.xyz, toward the sun (normalised by the library) */
  float sun_intensity;  /* Uniforms.sunParams.w: the disc's brightness; 0 = no sun disc or sun sampling */
  uint32_t sky_mode;    /* Uniforms.skyMode: 0 golden hour, 1 high noon, 2 twilight */
  uint32_t pad[2];
} vt_environment;
/* Sets (or with NULL / intensity 0 clears) an imported scene's environment; restarts its
 * accumulation. Sampling modes 1-3 only: ReSTIR DI (mode 0) rejects a scene with an environment, so
 * vt_render_nrc renders one with MIS primaries (mode 1); its training paths see the environment. */
vt_status vt_scene_set_environment(vt_ctx *ctx, vt_scene *scene, const vt_environment *env);
/* An equirectangular (lat-long) environment image instead of the procedural sky (MaterialLibrary's
 * makeEnvironment / environmentImportance, Sources/StudioModel.swift:1300-1436; eval_environment and
 * its sampling, main.swift:2077-2134, 2918-2950): `rgba` holds width x height linear-sRGB pixels, 4
 * floats each (alpha ignored, negatives clamped to 0), row 0 at +y; `rotation` (radians) turns it
 * about +y (Uniforms.environment.y), `intensity` scales it. NEE samples the image's texels from a
 * compensated table (luminance above the map's mean; used where the vertex's BSDF continuation is
 * traced) or the original one. Sampling modes 1-3. Restarts the accumulation; NULL or intensity 0
 * clears the environment. Limits as the reference's: width <= 16384, height <= 8192, at most 2^25
 * pixels, finite pixels. */
vt_status vt_scene_set_environment_map(vt_ctx *ctx, vt_scene *scene, const float *rgba, uint32_t width,
                                       uint32_t height, float intensity, float rotation);
/* The image's sampling tables as the scene holds them, computed on the host from HOST pixels:
 * rows[2 y + table] (2 x height marginal CDFs; table 0 compensated, 1 original) and
 * cols[(table height + y) width + x] (2 x width x height conditional CDFs). For checks. */
vt_status vt_environment_tables(const float *rgba, uint32_t width, uint32_t height, float *rows, float *cols);

/* ---- neural radiance cache (nrc.cu) -------------------------------------------------------------
 * No counterpart in the reference (it has no radiance cache). A radiance cache after Mueller et al.
 * 2021: a multiresolution hash grid of the position (Mueller et al. 2022) plus one-blob encodings of
 * the outgoing direction, the shading normal and the roughness, and the reflectances, into an MLP
 * of 5 hidden layers 64 wide (fp16 operands, fp32 accumulation, ReLU) with 3 linear outputs: the
 * radiance leaving the vertex toward the previous one, without the vertex's own emission, in linear
 * sRGB. Trained online by Adam (lazy for the hash grid: an entry without gradient in a step keeps
 * its moments) under the relative L2 loss on the suffix radiance of training paths
 * that the integrator traces to full depth. */
typedef struct vt_nrc vt_nrc;
typedef struct vt_nrc_config {
  uint32_t levels;           /* hash-grid levels, 1-16 (16) */
  uint32_t log2_table;       /* log2 of the entries per level, 12-24 (19) */
  uint32_t base_resolution;  /* cells per axis of the coarsest level, >= 2 (16) */
  uint32_t max_resolution;   /* cells per axis of the finest level (2048) */
  uint32_t train_records;    /* training records per optimiser step (65536) */
  uint32_t train_paths;      /* training paths per frame; 0: train_records / 4 */
  uint32_t query_vertex;     /* 0: rendered paths query the cache where their spread exceeds
                                `spread` times the primary spread (the spread-angle heuristic of
                                Mueller et al. 2021) (0); k >= 1: at vertex k, 1 = the first
                                bounce's hit; vertices before it are traced as usual */
  uint32_t seed;             /* parameter initialisation and training-path pixels */
  float learning_rate;       /* Adam step size (0.01) */
  float beta1, beta2, epsilon;  /* Adam (0.9, 0.99, 1e-15) */
  float spread;              /* the heuristic's constant c: a path stops at vertex n once
                                (sum_i sqrt(|x_i-1 - x_i|^2 / (p(w_i) |cos theta_i|)))^2 > c a0,
                                a0 = |x0 - x1|^2 / (4 pi cos theta_1) (0.01) */
  uint32_t spectral;         /* 1: the outputs are, per hero wavelength of a path, its radiance
                                over the illuminant at that wavelength, and scenes render with
                                spectral transport; 0: rgb (0) */
} vt_nrc_config;
/* A cache query (64 bytes). Directions are (theta / pi, phi / (2 pi) + 1/2), theta from +z and phi
 * = atan2(y, x). */
typedef struct vt_nrc_input {
  float position[3];
  float roughness;       /* 1 for Lambert slots */
  float direction[2];    /* outgoing direction (toward the previous vertex) */
  float normal[2];       /* shading normal */
  float diffuse[3];      /* diffuse reflectance: albedo x (1 - metalness) */
  float specular;        /* specular reflectance: metalness */
  float wavelength;      /* the path's wavelength number u in [0, 1): its hero wavelengths are
                            F^-1((u + k) / 4), k = 0..3 (spectral caches; 0 for rgb) */
  float pad[3];
} vt_nrc_input;
typedef struct vt_nrc_info {
  unsigned long long mlp_params, grid_params;  /* 21,504; levels x 2^log2_table x 2 */
  uint32_t steps;          /* optimiser steps taken */
  uint32_t last_records;   /* records of the last step */
  float last_loss;         /* mean relative L2 loss of the last step's records */
  uint32_t pad;
} vt_nrc_info;
enum { VT_NRC_TRAIN = 1, VT_NRC_RENDER = 2 };

vt_status vt_nrc_config_default(vt_nrc_config *cfg);
/* A cache over the box [lo, hi] (the scene's bounds), parameters initialised from cfg->seed. */
vt_status vt_nrc_create(vt_ctx *ctx, const vt_nrc_config *cfg, const float lo[3], const float hi[3], vt_nrc **out);
vt_status vt_nrc_destroy(vt_ctx *ctx, vt_nrc *nrc);
/* Synchronises the context's stream and the cache's last step. */
vt_status vt_nrc_get_info(vt_ctx *ctx, vt_nrc *nrc, vt_nrc_info *out);
/* Parameters as fp32: mlp = 21,504 floats (5 hidden 64 x 64 matrices [out][in], then the output
 * layer 16 x 64 with rows 4-15 zero), grid = levels x 2^log2_table x 2 floats (may be NULL).
 * Setting them also clears Adam's moments and step count. */
vt_status vt_nrc_get_params(vt_ctx *ctx, const vt_nrc *nrc, float *mlp, float *grid);
vt_status vt_nrc_set_params(vt_ctx *ctx, vt_nrc *nrc, const float *mlp, const float *grid);
/* Predictions for n host queries: out = n x 4 floats (the four lanes' terms, or rgb and 0). The
 * network runs on the tcgen05 tensor cores (M = 128 tiles, fp16 operands, fp32 accumulators in
 * tensor memory). */
vt_status vt_nrc_infer(vt_ctx *ctx, vt_nrc *nrc, const vt_nrc_input *in, uint32_t n, float *out);
/* The loss and its gradient sums over n host records (targets n x 4, as vt_nrc_infer's outputs),
 * without an update: mlp_grad 21,504 floats, grid_grad as vt_nrc_get_params' grid (may be NULL),
 * loss the loss sum. The backward pass runs with the loss scaled by 64 in fp16; the sums returned
 * are the loss's own. */
vt_status vt_nrc_gradients(vt_ctx *ctx, vt_nrc *nrc, const vt_nrc_input *in, const float *target, uint32_t n,
                           float *mlp_grad, float *grid_grad, double *loss);
/* One Adam step on n host records; loss (may be NULL) receives their mean loss before the step. */
vt_status vt_nrc_train(vt_ctx *ctx, vt_nrc *nrc, const vt_nrc_input *in, const float *target, uint32_t n, float *loss);
/* One frame of spp samples with the cache, stream-ordered like vt_render. flags VT_NRC_TRAIN:
 * trace the frame's training paths (MIS, full depth) and take one optimiser step on their records
 * first; VT_NRC_RENDER: render spp samples per pixel whose paths end where the cache's query rule
 * (query_vertex, spread) stops them, with the cache's prediction (sampling modes 0 and 1), added to
 * the scene's accumulation; sampling mode 1 renders through the wavefront integrator
 * (vt_render_wavefront's stages), mode 0 through ReSTIR DI's two passes. The frame's transport must
 * match the cache's `spectral` setting. */
vt_status vt_render_nrc(vt_ctx *ctx, vt_scene *scene, vt_nrc *nrc, const vt_frame_params *p, uint32_t spp,
                        uint32_t flags, void *stream);

/* ---- allocation-free build --------------------------------------------------------------- */

/* No counterpart in the reference. The same GPU build as vt_mesh_build_device, for callers that
 * cannot call cudaMalloc: hosts running under a fixed device-memory budget owned elsewhere (their
 * own arena, or a framework's caching allocator holding the GPU memory), and loops that must not
 * pay cudaMalloc/cudaFree's implicit device synchronisation. It needs no vt_ctx and allocates
 * nothing: the caller passes DEVICE faces and vertices and DEVICE outputs, and every temporary
 * comes from a 6 MiB static device array that each GPU loading the library holds until exit.
 *   nodes: nodes_capacity >= nfaces 4-wide nodes (16-byte aligned); info->wide_nodes are written.
 *   tris:  12 floats per face (three float4 per BVH position: a with the input face index's bits
 *          in .w, b with the face's tag bits in .w, c; 16-byte aligned).
 *   order: nfaces int32 (BVH position -> input face).
 *   info:  host output (build_ms is host wall time).  stream: NULL = the CUDA default stream.
 *          The call blocks the host: it synchronises that stream once per collapse level (the
 *          level's node count sizes the next launch) and at the end, so it returns when the build
 *          is complete; a call that fails after queueing work also waits for that work first.
 *   error: optional host buffer of error_capacity bytes for the failure message.
 * Meshes over VT_NOALLOC_MAX_FACES faces are rejected with VT_ERR_LIMIT. The first call on each
 * device looks up the static array's address (with that device current), so make that first call
 * before any stream capture. Every call shares the one array: calls that overlap on the GPU (on
 * other streams or from other host threads) race on it. */
#define VT_NOALLOC_MAX_FACES 32768u
vt_status vt_mesh_build_noalloc(const vt_face *faces_dev, uint32_t nfaces, const vt_vertex *verts_dev,
                                uint32_t nverts, const vt_build_options *opts, vt_wide_node *nodes_dev,
                                uint32_t nodes_capacity, float *tris_dev, int32_t *order_dev,
                                vt_mesh_info *info, void *stream, char *error, uint32_t error_capacity);

#ifdef __cplusplus
}
#endif
#endif /* VT_H */
