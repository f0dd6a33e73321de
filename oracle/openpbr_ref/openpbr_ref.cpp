// openpbr_ref.cpp — the reference's OpenPBR BSDF compiled for the CPU (test infrastructure only:
// the checker of the CUDA restatement in metal_vibe_tracer_b200/csrc/openpbr.cuh).
//
// Built by oracle/openpbr_ref/Makefile from the reference's vendored Adobe OpenPBR headers
// (Vendor/OpenPBR, openpbr-bsdf c91aad1d, Apache-2.0) where they lie, into oracle/_ref/; nothing of
// them is copied here. As the reference's shader preparation does (scripts/prepare_shaders.py:
// 28-39), the two ideal-metal energy lookups call the dense table of Shaders/MetalEnergy.metal
// (compiled from there as C++). That script's third adaptation (the thin-wall subsurface share of
// the dielectric multiple-scattering lobe) is not applied: it only touches thin-walled materials,
// which these checks do not use.
//
// The entry points mirror the reference's adapter prepare_openpbr (main.swift:2485-2512) for a
// non-MaterialX material: the inputs it sets, the basis from the shading normal (and tangent), and
// openpbr_prepare / openpbr_eval / openpbr_pdf / openpbr_sample.
#include "glmlite.h"

#define OPENPBR_LANGUAGE_TARGET_CPP 1
#define OPENPBR_USE_CUSTOM_VEC_TYPES 1
#define OPENPBR_ASSERT(expr, message) ((void)0)
#define OPENPBR_ASSERT_UNREACHABLE(message) ((void)0)
#include "openpbr_settings.h"
#include "openpbr_data_constants.h"
#include "interop/openpbr_interop.h"

// Shaders/MetalEnergy.metal as C++.
typedef unsigned int uint;
#define constant static const
#include "MetalEnergy.metal"
#undef constant

// The upstream lookups get other names; the substitutes below take theirs.
#define openpbr_look_up_ideal_metal_energy_complement openpbr_upstream_ideal_metal_energy_complement
#define openpbr_look_up_ideal_metal_average_energy_complement openpbr_upstream_ideal_metal_average_energy_complement
#include "impl/openpbr_microfacet_multiple_scattering_data.h"
#undef openpbr_look_up_ideal_metal_energy_complement
#undef openpbr_look_up_ideal_metal_average_energy_complement
float openpbr_look_up_ideal_metal_energy_complement(const float alpha, const float cos_theta) {
  return vibe_metal_energy(alpha, cos_theta);
}
float openpbr_look_up_ideal_metal_average_energy_complement(const float alpha) { return vibe_metal_average_energy(alpha); }

#include "openpbr.h"

extern "C" {

// The adapter's material fields (Material, main.swift:321-346) that prepare_openpbr reads.
typedef struct ref_openpbr_material {
  int32_t type;            // 0 DIFFUSE, 1 GLOSSY (metal), 2 DIELECTRIC, 4 OPENPBR
  float albedo[3];
  float roughness, metalness, ior, coat, anisotropy, fuzz, transmission;
  float thin_film_weight, thin_film_thickness, thin_film_ior;  // spectral transport only
  int32_t inside;
  float tangent[3];
  float pad;
} ref_openpbr_material;

static OpenPBR_PreparedBsdf ref_prepare(const ref_openpbr_material *m, const float *n3, const float *wo3, const float *lambda3) {
  OpenPBR_ResolvedInputs inputs = openpbr_make_default_resolved_inputs();
  inputs.base_color = clamp(vec3(m->albedo[0], m->albedo[1], m->albedo[2]), 0.0f, 1.0f);
  inputs.specular_roughness = max(0.03f, m->roughness);
  inputs.base_metalness = m->type == 1 ? 1.0f : m->metalness;
  inputs.specular_weight = m->type == 0 ? 0.0f : 1.0f;
  inputs.specular_ior = max(1.01f, m->ior);
  inputs.specular_color = vec3(1.0f);
  inputs.coat_weight = m->coat;
  inputs.coat_roughness = 0.12f;
  inputs.specular_roughness_anisotropy = m->anisotropy;
  inputs.fuzz_weight = m->fuzz;
  inputs.transmission_weight = m->transmission;
  inputs.transmission_color = vec3(1.0f);
  inputs.thin_film_weight = m->thin_film_weight;
  inputs.thin_film_thickness = m->thin_film_thickness;
  inputs.thin_film_ior = m->thin_film_ior;
  inputs.geometry_thin_walled = false;
  const vec3 n(n3[0], n3[1], n3[2]), t(m->tangent[0], m->tangent[1], m->tangent[2]);
  const vec3 outward = m->transmission > 0.0f && m->inside ? -n : n;
  inputs.geometry_basis = dot(t, t) > 0.5f && abs(dot(t, outward)) < 0.99f ? openpbr_make_basis(outward, t, 1.0f) : openpbr_make_basis(outward);
  inputs.geometry_coat_basis = inputs.geometry_basis;
  const vec3 lambda = lambda3 ? vec3(lambda3[0], lambda3[1], lambda3[2]) : OpenPBR_BaseRgbWavelengths_nm;
  return openpbr_prepare(inputs, vec3(1.0f), lambda, 1.0f, vec3(wo3[0], wo3[1], wo3[2]));
}

// f |cos| at wi (diffuse + specular, per colour channel) and the pdf of wi.
void ref_openpbr_eval(const ref_openpbr_material *m, const float *n, const float *wo, const float *wi, const float *lambda,
                      float *f_cos, float *pdf) {
  const OpenPBR_PreparedBsdf p = ref_prepare(m, n, wo, lambda);
  const vec3 l(wi[0], wi[1], wi[2]);
  const vec3 f = openpbr_get_sum_of_diffuse_specular(openpbr_eval(p, l));
  f_cos[0] = f.x;
  f_cos[1] = f.y;
  f_cos[2] = f.z;
  *pdf = openpbr_pdf(p, l);
}

// One sample from three random numbers: direction, weight f |cos| / pdf, pdf and the lobe type bits.
void ref_openpbr_sample(const ref_openpbr_material *m, const float *n, const float *wo, const float *rand, const float *lambda,
                        float *dir, float *weight, float *pdf, int32_t *lobe) {
  const OpenPBR_PreparedBsdf p = ref_prepare(m, n, wo, lambda);
  vec3 d;
  OpenPBR_DiffuseSpecular w;
  float q = 0.0f;
  OpenPBR_BsdfLobeType type;
  openpbr_sample(p, vec3(rand[0], rand[1], rand[2]), d, w, q, type);
  const vec3 s = openpbr_get_sum_of_diffuse_specular(w);
  dir[0] = d.x;
  dir[1] = d.y;
  dir[2] = d.z;
  weight[0] = s.x;
  weight[1] = s.y;
  weight[2] = s.z;
  *pdf = q;
  *lobe = (int32_t)type;
}

// A thin film over an ideal mirror (spectral_thin_film_mirror, main.swift:3272-3283): the film's
// presence (weight times the upstream presence ramp at thickness_um * 1000 nm) and, where it is
// positive, the upstream Airy reflectance of the film over metal at cos_i per wavelength, with the
// mirror's F0, a white F82 tint, exterior IOR 1 and the unused dielectric base IOR 1.5.
float ref_thin_film_mirror(float cos_i, float weight, float thickness_um, float film_ior, const float *f0,
                           const float *lambda, float *reflectance) {
  const float nm = thickness_um * 1000.0f;
  const float presence = weight * openpbr_thin_film_presence_multiplier(nm);
  if (!(presence > 0.0f)) return presence;
  const OpenPBR_ThinFilmResults r = openpbr_thin_film_and_base_reflectance(
      cos_i, 1.0f, film_ior, vec3(1.5f), false, vec3(f0[0], f0[1], f0[2]), vec3(1.0f), false, true, nm,
      vec3(lambda[0], lambda[1], lambda[2]));
  reflectance[0] = r.reflectance_metal.x;
  reflectance[1] = r.reflectance_metal.y;
  reflectance[2] = r.reflectance_metal.z;
  return presence;
}

// The dense isotropic GGX energy complement (Shaders/MetalEnergy.metal) and its average.
float ref_metal_energy(float alpha, float cos_theta) { return vibe_metal_energy(alpha, cos_theta); }
float ref_metal_average_energy(float alpha) { return vibe_metal_average_energy(alpha); }
void ref_metal_energy_table(float *table, float *average) {
  for (int i = 0; i < 129 * 129; ++i) table[i] = vibeMetalEnergy[i];
  for (int i = 0; i < 129; ++i) average[i] = vibeMetalAverageEnergy[i];
}

}  // extern "C"
