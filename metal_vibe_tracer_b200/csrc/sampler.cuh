// sampler.cuh — the per-pixel sampler: the PCG stream and the Z++ sampler (main.swift:89-305,
// 497-515).
//
// PCG mode: every draw continues one 32-bit state (pcg_hash, rand_f; main.swift:91-101).
// Z++ mode (ZPP2026 in the reference's REFERENCES.md): a pixel's key (z_pixel_key, main.swift:
// 497-506) holds its shuffled Morton code XOR a temporal index in bits 14-31 and the frame j of the
// accumulation in bits 0-13. A sampling event (path vertex, stream) owns 32 consecutive
// dimensions; each rand_f / rand_f2 / rand_f3 takes the event's next dimension and returns a 1D
// van der Corput, 2D Sobol' or 3D O2m3 constituent, Owen-scrambled per dimension, its frame-0 index
// a nested scramble of the pixel code and, for frames j > 0, XOR-shifted by point j of the pixel's
// own sequence. All integer arithmetic: the CPU oracle reproduces every draw bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace vtd {

__device__ __forceinline__ uint32_t pcg_hash(uint32_t input) {
  uint32_t state = input * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}
__device__ __forceinline__ float pcg_rand(uint32_t &seed) {
  seed = pcg_hash(seed);
  return float(seed >> 8u) * (1.0f / 16777216.0f);
}

// Wellons' lowbias32 finaliser.
__device__ __forceinline__ uint32_t z_mix(uint32_t v) {
  v ^= v >> 16; v *= 0x7feb352du; v ^= v >> 15; v *= 0x846ca68bu; v ^= v >> 16;
  return v;
}
// The six permutations of four quadrants that fix quadrant 0 (2 bits per digit, 8 per entry).
constexpr unsigned long long kZPermutations = 0x6c9c78d8b4e4ull;
constexpr uint32_t kZShuffleDigits = 12u;
constexpr uint32_t kZFrameBits = 14u;

// Recursive quadrant shuffle of the low 12 base-4 digits (maps aligned 4^m blocks onto aligned
// blocks); digit permutations chosen by a hash of the digits above and of `dimension`.
__device__ __forceinline__ uint32_t z_shuffle(uint32_t index, uint32_t dimension) {
  const uint32_t seed = z_mix(dimension * 0x9e3779b9u + 0x632be5abu);
  uint32_t result = index & ~((1u << (2u * kZShuffleDigits)) - 1u);
  for (uint32_t d = kZShuffleDigits; d-- > 0u;) {
    const uint32_t shift = 2u * d, digit = (index >> shift) & 3u;
    const uint32_t h = z_mix((index >> (shift + 2u)) ^ seed);
    const uint32_t sigma = ((h >> 16) * 6u) >> 16;
    const uint32_t image = (uint32_t)(kZPermutations >> (8u * sigma + 2u * digit)) & 3u;
    result |= (image ^ (h & 3u)) << shift;
  }
  return result;
}
// Nested uniform (Owen) scramble of a 0.32 fixed-point value (Laine-Karras hash form).
__device__ __forceinline__ uint32_t z_owen(uint32_t v, uint32_t seed) {
  v = __brev(v);
  v ^= v * 0x3d20adeau;
  v += seed;
  v *= (seed >> 16) | 1u;
  v ^= v * 0x05526c56u;
  v ^= v * 0x53a22864u;
  return __brev(v);
}
__device__ __forceinline__ uint32_t z_owen_seed(uint32_t dimension, uint32_t axis) {
  const uint32_t h = (dimension ^ (axis << 24)) * 0x9e3779b9u;
  return (h ^ (h >> 16)) * 0x85ebca6bu;
}
// Second Sobol' dimension of index i (binary Pascal matrix), as a 0.32 fraction.
__device__ __forceinline__ uint32_t z_sobol1(uint32_t i) {
  i ^= (i & 0xAAAAAAAAu) >> 1;
  i ^= (i & 0xCCCCCCCCu) >> 2;
  i ^= (i & 0xF0F0F0F0u) >> 4;
  i ^= (i & 0xFF00FF00u) >> 8;
  i ^= (i & 0xFFFF0000u) >> 16;
  return __brev(i);
}
// O2m3: the three coordinates of the point with bit-reversed index V.
__device__ __forceinline__ uint32_t z_o2m3_x(uint32_t V) {
  V ^= ((V << 2) & 0xF3CF3CF3u) ^ ((V << 3) & 0x41041041u);
  V ^= (V << 4) & 0x3F03F03Fu;
  V ^= (V << 8) & 0x0FFF000Fu;
  V ^= (V << 16) & 0x00FFFFFFu;
  return V;
}
__device__ __forceinline__ uint32_t z_o2m3_y(uint32_t V) {
  return z_o2m3_x(((V >> 1) & 0x45145145u) ^ (V & 0xB5EB5EB5u) ^ ((V << 1) & 0x8A28A28Au));
}
__device__ __forceinline__ uint32_t z_o2m3_z(uint32_t V) {
  return z_o2m3_x(((V >> 1) & 0x45145145u) ^ (V & 0x7AD7AD7Au) ^ ((V << 1) & 0x8A28A28Au));
}
__device__ __forceinline__ float z_float(uint32_t v) { return float(v >> 8) * (1.0f / 16777216.0f); }
// Morton index of a pixel, x in the even bits.
__device__ __forceinline__ uint32_t z_morton(uint32_t x, uint32_t y) {
  x &= 0xFFFFu; y &= 0xFFFFu;
  x = (x | (x << 8)) & 0x00FF00FFu; x = (x | (x << 4)) & 0x0F0F0F0Fu; x = (x | (x << 2)) & 0x33333333u; x = (x | (x << 1)) & 0x55555555u;
  y = (y | (y << 8)) & 0x00FF00FFu; y = (y | (y << 4)) & 0x0F0F0F0Fu; y = (y | (y << 2)) & 0x33333333u; y = (y | (y << 1)) & 0x55555555u;
  return x | (y << 1);
}

// Sampling-event streams (main.swift:291-292): 32 dimensions each, 16 per path vertex.
constexpr uint32_t kZBsdf = 0u, kZNee = 1u, kZRoulette = 2u, kZLens = 3u, kZDi = 4u, kZGiBsdf = 5u, kZGiNee = 6u,
                   kZWavelength = 12u;

struct Sampler {
  uint32_t state, key, dimension, sub, subBits;
  bool z;
};

// z_pixel_key: model 0 per-pixel, 1 TZ, 2 STZ, 3 reshuffled; frameIndex is the accumulation frame
// (1-based), sampleIndex the global sample counter.
__device__ __forceinline__ uint32_t z_pixel_key(uint32_t x, uint32_t y, uint32_t model, uint32_t frameIndex,
                                                uint32_t sampleIndex) {
  const uint32_t j = max(frameIndex, 1u) - 1u, s0 = sampleIndex - j;
  uint32_t t = model == 1u || model == 2u ? s0 ^ ((s0 & 0xAAAAAAAAu) << 1) : model == 3u ? z_mix(s0 ^ 0x2c1b3c6du) : s0;
  uint32_t k = z_shuffle(z_morton(x, y), 0xffffffffu);
  if (model == 2u) k ^= k << 2;
  if ((j >> kZFrameBits) != 0u) t ^= z_mix(j >> kZFrameBits);
  return ((k ^ t) << kZFrameBits) | (j & ((1u << kZFrameBits) - 1u));
}

// pixel_sampler (main.swift:508-515).
__device__ __forceinline__ Sampler pixel_sampler(uint32_t x, uint32_t y, uint32_t width, uint32_t sampleIndex,
                                                 bool z, uint32_t model, uint32_t frameIndex) {
  Sampler s;
  s.state = (y * width + x) ^ (sampleIndex * 1999999973u);
  s.z = z;
  s.key = z ? z_pixel_key(x, y, model, frameIndex, sampleIndex) : 0u;
  s.dimension = 0u; s.sub = 0u; s.subBits = 0u;
  return s;
}

__device__ __forceinline__ uint32_t z_pixel_code(uint32_t key) { return key >> kZFrameBits; }
__device__ __forceinline__ uint32_t z_frame(const Sampler &s) {
  return ((s.key & ((1u << kZFrameBits) - 1u)) << s.subBits) | s.sub;
}
__device__ __forceinline__ uint32_t z_index(const Sampler &s, uint32_t d) {
  return z_owen(z_pixel_code(s.key), z_owen_seed(d, 3u));
}
__device__ __forceinline__ uint32_t z_dimension(Sampler &s) {
  return s.dimension++ | ((z_pixel_code(s.key) >> 12) << 17);
}
__device__ __forceinline__ uint32_t z_frame_index(uint32_t J, uint32_t d) {
  const uint32_t seed = z_owen_seed(d, 4u);
  return z_owen(J, seed) ^ z_owen(0u, seed);
}
__device__ __forceinline__ uint32_t z_frame_offset(const Sampler &s, uint32_t v, uint32_t d, uint32_t axis) {
  const uint32_t seed = z_owen_seed(d, axis) ^ z_mix(z_pixel_code(s.key) ^ 0x68e31da4u);
  return ((z_owen(v, seed) ^ z_owen(0u, seed)) & 0x3FFFFFFFu) | (v & 0xC0000000u);
}

__device__ __forceinline__ float rand_f(Sampler &s) {
  if (!s.z) return pcg_rand(s.state);
  const uint32_t d = z_dimension(s), J = z_frame(s);
  uint32_t x = z_owen(__brev(z_index(s, d)), z_owen_seed(d, 0u));
  if (J != 0u) x ^= z_frame_offset(s, __brev(z_frame_index(J, d)), d, 0u);
  return z_float(x);
}
__device__ __forceinline__ float2 rand_f2(Sampler &s) {
  if (!s.z) { const float a = pcg_rand(s.state); return make_float2(a, pcg_rand(s.state)); }
  const uint32_t d = z_dimension(s), i = z_index(s, d), J = z_frame(s);
  uint32_t x = z_owen(__brev(i), z_owen_seed(d, 0u)), y = z_owen(z_sobol1(i), z_owen_seed(d, 1u));
  if (J != 0u) {
    const uint32_t k = z_frame_index(J, d);
    x ^= z_frame_offset(s, __brev(k), d, 0u);
    y ^= z_frame_offset(s, z_sobol1(k), d, 1u);
  }
  return make_float2(z_float(x), z_float(y));
}
__device__ __forceinline__ float3 rand_f3(Sampler &s) {
  if (!s.z) {
    const float a = pcg_rand(s.state), b = pcg_rand(s.state);
    return make_float3(a, b, pcg_rand(s.state));
  }
  const uint32_t d = z_dimension(s), V = __brev(z_index(s, d)), J = z_frame(s);
  uint32_t x = z_owen(z_o2m3_x(V), z_owen_seed(d, 0u)), y = z_owen(z_o2m3_y(V), z_owen_seed(d, 1u)),
           z = z_owen(z_o2m3_z(V), z_owen_seed(d, 2u));
  if (J != 0u) {
    const uint32_t W = __brev(z_frame_index(J, d));
    x ^= z_frame_offset(s, z_o2m3_x(W), d, 0u);
    y ^= z_frame_offset(s, z_o2m3_y(W), d, 1u);
    z ^= z_frame_offset(s, z_o2m3_z(W), d, 2u);
  }
  return make_float3(z_float(x), z_float(y), z_float(z));
}
// sampler_event (main.swift:293-295): vertex v's stream owns dimensions (16 v + stream) 32 ...
__device__ __forceinline__ void sampler_event(Sampler &s, uint32_t vertex, uint32_t stream) {
  s.dimension = (vertex * 16u + stream) * 32u;
  s.sub = 0u;
  s.subBits = 0u;
}
// sampler_candidate (main.swift:296-298): candidate `index` of an event draws from the event's
// dimensions with `bits` extra frame bits, so a block of 2^bits candidates is stratified.
__device__ __forceinline__ void sampler_candidate(Sampler &s, uint32_t vertex, uint32_t stream, uint32_t index,
                                                  uint32_t bits) {
  sampler_event(s, vertex, stream);
  if (s.z) { s.sub = index; s.subBits = bits; }
}
// rand_decision (main.swift:117, 280): resampling decisions draw from the PCG state in either mode.
__device__ __forceinline__ float rand_decision(Sampler &s) { return pcg_rand(s.state); }
// wavelength_numbers (main.swift:2222-2231): from a copy, so the sampler's streams are unchanged.
__device__ __forceinline__ float2 wavelength_numbers(Sampler s) {
  if (s.z) {
    sampler_event(s, 0u, kZWavelength);
    const float u = rand_f(s);
    return make_float2(u, rand_f(s));
  }
  const uint32_t h = pcg_hash(s.state ^ 0x5bd1e995u);
  return make_float2(float(h >> 8u) * (1.0f / 16777216.0f), float(pcg_hash(h) >> 8u) * (1.0f / 16777216.0f));
}

}  // namespace vtd
