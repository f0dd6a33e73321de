/*
 * vt_oracle.h — CPU restatement of the reference's traversal and BVH-build arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA path: the tests, the smoke
 * check and bench.py's CPU-baseline leg load it; the product library never links or calls it.
 *
 * What it restates (reference file:line):
 *   - PCG hash stream: main.swift:91-101 (pcg_hash, rand_f).
 *   - Watertight ray/triangle test: main.swift:1536-1582 (watertight_ray, watertight_edge,
 *     intersect_mesh_triangle), in two precisions:
 *       fp32: the op order fixed for the CUDA kernels (every product and sum rounded on its own,
 *             the exact-tie FMA fallback of watertight_edge), so GPU hits compare bit for bit;
 *       fp64: the same algorithm in double precision, the accuracy judge (hit IDs, t error).
 *   - Conservative 4-wide slab test and near-to-far order: main.swift:1758-1785.
 *   - Closest-hit / any-hit 4-wide traversal: main.swift:1788-1838.
 *   - Binned-SAH 4-wide build (WideBVH): Sources/Acceleration.swift:106-352, with its deferred
 *     subtree numbering (:302-350) and the median rebuild past the depth limit (:296-300).
 *   - The LBVH that replaces it on the GPU (no reference counterpart; restated from the CUDA
 *     build's own definition so Morton codes, order and topology compare bit for bit).
 */
#ifndef VT_ORACLE_H
#define VT_ORACLE_H
#include <stdint.h>
#include "../include/vt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vto_bvh vto_bvh;

typedef struct vto_bvh_info {
  uint32_t faces, wide_nodes, binary_nodes, depth;
  float sah_cost;
  float lo[3], hi[3];
} vto_bvh_info;

uint32_t vto_pcg_hash(uint32_t v);
float vto_rand_f(uint32_t *seed);

/* One watertight test (fp32 op order of the CUDA kernels). tri = 9 floats (a, b, c). Returns
 * 1 on a hit in [tmin, tmax) and writes t, b1, b2. */
int32_t vto_intersect_f32(const vt_ray *ray, const float *tri, float *t, float *b1, float *b2);
int32_t vto_intersect_f64(const double *ray /* o xyz, d xyz */, const double *tri, double tmin,
                          double tmax, double *t, double *b1, double *b2);

/* LBVH restatement. treelet_size < 0 disables the SAH restructuring. */
vto_bvh *vto_lbvh_build(const vt_face *faces, uint32_t nfaces, const vt_vertex *verts,
                        uint32_t nverts, int32_t leaf_size, int32_t treelet_size,
                        int32_t rounds);
/* Reference binned-SAH 4-wide build (WideBVH.build with leafSize and depth limit). */
vto_bvh *vto_widebvh_build(const vt_face *faces, uint32_t nfaces, const vt_vertex *verts,
                           uint32_t nverts, int32_t leaf_size, int32_t max_depth, int32_t threads);
void vto_bvh_free(vto_bvh *h);
/* A hierarchy built elsewhere (4-wide nodes, leaf order, depth) over `faces` / `verts`. */
vto_bvh *vto_bvh_import(const vt_wide_node *nodes, uint32_t nnodes, const int32_t *order, uint32_t nfaces,
                        const vt_face *faces, const vt_vertex *verts, uint32_t depth);
void vto_bvh_get_info(const vto_bvh *h, vto_bvh_info *out);
void vto_bvh_get_nodes(const vto_bvh *h, vt_wide_node *out);
void vto_bvh_get_order(const vto_bvh *h, int32_t *out);
/* LBVH only: sorted codes/faces and the refined binary tree (children 2n, boxes 6n). */
void vto_bvh_get_morton(const vto_bvh *h, uint32_t *codes, int32_t *sorted);
void vto_bvh_get_binary(const vto_bvh *h, int32_t *children, float *boxes);

/* Traversal over an oracle BVH. precision = 32 (bit-exact CUDA op order) or 64. */
void vto_trace_closest(const vto_bvh *h, const vt_ray *rays, uint32_t n, vt_hit *hits,
                       int32_t precision, int32_t threads);
void vto_trace_any(const vto_bvh *h, const vt_ray *rays, uint32_t n, uint8_t *occluded,
                   int32_t precision, int32_t threads);
/* Brute force over all faces (input order ids). */
void vto_brute_closest(const vt_face *faces, uint32_t nfaces, const vt_vertex *verts,
                       const vt_ray *rays, uint32_t n, vt_hit *hits, int32_t precision,
                       int32_t threads);
/* Two-level traversal (mesh_closest / mesh_occluded, main.swift:1840-1984): TLAS nodes whose leaves
 * name instances, the instance records and each record's mesh (meshes[record.mesh]); closest = 1
 * writes hits and (if non-null) instances, 0 writes occluded. precision 32 or 64 as above. */
void vto_tlas_trace(const vt_wide_node *nodes, const vt_instance_record *inst, const vto_bvh *const *meshes,
                    float grow, float reach, const vt_ray *rays, uint32_t n, vt_hit *hits, uint32_t *instances,
                    uint8_t *occluded, int32_t closest, int32_t precision, int32_t threads);
/* Traversal statistics of closest (1) or any-hit (0) traversal, fp32 order. */
void vto_trace_count(const vto_bvh *h, const vt_ray *rays, uint32_t n, int32_t closest,
                     uint64_t *nodes_visited, uint64_t *tris_tested, int32_t threads);

/* ---- path tracer (FP64 restatement of the MIS integrator) ------------------------------------ */
/* shading_kernel (main.swift:7370-7914) in MIS mode with the PCG sampler, on a triangle scene whose
 * faces' tags select material slots, the procedural quad light (main.swift:2957-2978, 3046-3050)
 * and, when `spectral`, four hero wavelengths from the tables (main.swift:755-848, 945-959). All
 * arithmetic in double; random numbers are the reference's exact 24-bit PCG draws. */
/* OpenPBR materials: the reference BSDF (oracle/openpbr_ref, compiled from the reference's vendored
 * headers) called through these entry points; the material record mirrors its adapter's fields. */
typedef struct vto_pbr_material {
  int32_t type;
  float albedo[3];
  float roughness, metalness, ior, coat, anisotropy, fuzz, transmission;
  float thin_film_weight, thin_film_thickness, thin_film_ior;
  int32_t inside;
  float tangent[3];
  float pad;
} vto_pbr_material;
typedef void (*vto_pbr_eval_fn)(const vto_pbr_material *m, const float *n, const float *wo, const float *wi,
                                const float *lambda, float *f_cos, float *pdf);
typedef void (*vto_pbr_sample_fn)(const vto_pbr_material *m, const float *n, const float *wo, const float *rand,
                                  const float *lambda, float *dir, float *weight, float *pdf, int32_t *lobe);
/* A thin film over an ideal mirror (spectral_thin_film_mirror): returns the film's presence and,
 * where it is positive, the film-over-metal reflectance at three wavelengths. */
typedef float (*vto_pbr_film_mirror_fn)(float cos_i, float weight, float thickness_um, float film_ior, const float *f0,
                                        const float *lambda, float *reflectance);

typedef struct vto_pt_inputs {
  const vt_face *faces;
  uint32_t nfaces;
  const vt_vertex *verts;
  uint32_t nverts;
  const vt_material *materials;
  uint32_t nmat;
  vt_quad_light light;
  const float *cmf_rgb;   /* nbins x 3 (may be null for RGB transport) */
  const float *illum;     /* nbins */
  const float *icdf;      /* segments + 1 */
  uint32_t nbins, segments;
  float lambda_min;
  /* Imported scenes (emitter triangles instead of the quad light): the packed emitter list
   * (vt_emitter_list_pack layout, ids = face indices); imported = 0 selects the quad light. */
  const uint32_t *emitters;
  uint32_t nemitter_words;
  uint32_t imported;
  /* Spectral uplift (spectral_uplift.h): the colour model with its lazily solved grid, and cos of
   * the warped phase at each of the nbins bins. Needed when spectral. */
  const struct vto_uplift *uplift;
  const float *cos_phase;
  /* Per-slot lobe parameters, read for OPENPBR, GLOSSY and DIELECTRIC slots (types 4, 1, 2): 12 floats
   * (roughness, metalness, IOR, diffuse roughness, thin-film weight, thickness in micrometres and IOR,
   * coat weight, fuzz weight, 3 unused), and the BSDF (null parameters: GLOSSY slots are mirrors, DIELECTRIC slots have IOR 1.5). */
  const float *pbr_params;
  vto_pbr_eval_fn pbr_eval;
  vto_pbr_sample_fn pbr_sample;
  /* Imported scenes: the procedural sky and sun (intensity 0: none). */
  vt_environment environment;
  /* An environment image instead of the sky (env_rgba null: none): width x height pixels, 4 floats
   * each, its rotation about +y in radians; the intensity is environment.intensity. */
  const float *env_rgba;
  uint32_t env_w, env_h;
  float env_rot;
  /* A prebuilt hierarchy over these faces (vto_bvh_import); null: the renderer builds its LBVH. */
  const vto_bvh *bvh;
  /* The thin film over GLOSSY mirrors in spectral transport (null: none). */
  vto_pbr_film_mirror_fn pbr_film_mirror;
} vto_pt_inputs;

/* Z++ sampler primitives (main.swift:122-305): `n` points of the O2m3 and 2D Sobol' sequences
 * (Owen-scrambled under `seed` unless 0), `n` quadrant shuffles of base + i, and per pixel the
 * rand_f, rand_f2, rand_f3 draws (6 floats) of one sampling event. */
void vto_z_sequences(uint32_t seed, uint32_t n, uint32_t *o2m3, uint32_t *sobol);
void vto_z_shuffles(uint32_t base, uint32_t dimension, uint32_t n, uint32_t *out);
void vto_sampler_frame(uint32_t width, uint32_t height, int32_t z, uint32_t model, uint32_t sampleIndex,
                       uint32_t frameIndex, uint32_t vertex, uint32_t stream, float *out);

/* Mean linear-sRGB radiance per pixel over `spp` frames starting at params->first_sample
 * (accumulation frames from max(1, params->first_frame)). */
void vto_render(const vto_pt_inputs *in, const vt_frame_params *params, uint32_t spp, double *out_rgb,
                int32_t threads);

#ifdef __cplusplus
}
#endif
#endif
