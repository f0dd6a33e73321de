// glmlite.h — the small GLM-style vector library the vendored OpenPBR headers need for a CPU build
// (test infrastructure only: it lets oracle/openpbr_ref compile the reference's own BSDF as the
// checker of the CUDA restatement). The headers' C++ interop expects GLM, absent here; with
// OPENPBR_USE_CUSTOM_VEC_TYPES these types and functions stand in. `mix` is x + (y - x) t, the
// Metal Shading Language's form (the reference runs the headers as MSL).
#pragma once

#include <cmath>
#include <cstdint>

#define GLM_VERSION 999
#define GLM_CONSTEXPR constexpr

namespace glmlite {

struct bvec2 { bool x, y; };
struct bvec3 { bool x, y, z; };
struct bvec4 { bool x, y, z, w; };

struct vec2 {
  union { float x; float r; };
  union { float y; float g; };
  constexpr vec2() : x(0), y(0) {}
  constexpr explicit vec2(float s) : x(s), y(s) {}
  constexpr vec2(float a, float b) : x(a), y(b) {}
  float &operator[](int i) { return i == 0 ? x : y; }
  float operator[](int i) const { return i == 0 ? x : y; }
};
struct vec3 {
  union { float x; float r; };
  union { float y; float g; };
  union { float z; float b; };
  constexpr vec3() : x(0), y(0), z(0) {}
  constexpr explicit vec3(float s) : x(s), y(s), z(s) {}
  constexpr vec3(float a, float b, float c) : x(a), y(b), z(c) {}
  constexpr vec3(vec2 a, float c) : x(a.x), y(a.y), z(c) {}
  constexpr explicit vec3(bvec3 b) : x(b.x ? 1.0f : 0.0f), y(b.y ? 1.0f : 0.0f), z(b.z ? 1.0f : 0.0f) {}
  float &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
struct vec4 {
  union { float x; float r; };
  union { float y; float g; };
  union { float z; float b; };
  union { float w; float a; };
  constexpr vec4() : x(0), y(0), z(0), w(0) {}
  constexpr explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
  constexpr vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
  constexpr vec4(vec3 a, float d) : x(a.x), y(a.y), z(a.z), w(d) {}
  float &operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};

#define GLMLITE_OPS(V, N)                                                                          \
  inline V operator+(V a, V b) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] + b[i]; return r; } \
  inline V operator-(V a, V b) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] - b[i]; return r; } \
  inline V operator*(V a, V b) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] * b[i]; return r; } \
  inline V operator/(V a, V b) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] / b[i]; return r; } \
  inline V operator+(V a, float s) { return a + V(s); }                                         \
  inline V operator-(V a, float s) { return a - V(s); }                                         \
  inline V operator*(V a, float s) { return a * V(s); }                                         \
  inline V operator/(V a, float s) { return a / V(s); }                                         \
  inline V operator+(float s, V a) { return V(s) + a; }                                         \
  inline V operator-(float s, V a) { return V(s) - a; }                                         \
  inline V operator*(float s, V a) { return V(s) * a; }                                         \
  inline V operator/(float s, V a) { return V(s) / a; }                                         \
  inline V operator-(V a) { V r; for (int i = 0; i < N; ++i) r[i] = -a[i]; return r; }         \
  inline V &operator+=(V &a, V b) { a = a + b; return a; }                                      \
  inline V &operator-=(V &a, V b) { a = a - b; return a; }                                      \
  inline V &operator*=(V &a, V b) { a = a * b; return a; }                                      \
  inline V &operator/=(V &a, V b) { a = a / b; return a; }                                      \
  inline V &operator+=(V &a, float s) { a = a + s; return a; }                                  \
  inline V &operator-=(V &a, float s) { a = a - s; return a; }                                  \
  inline V &operator*=(V &a, float s) { a = a * s; return a; }                                  \
  inline V &operator/=(V &a, float s) { a = a / s; return a; }                                  \
  inline float dot(V a, V b) { float s = 0.0f; for (int i = 0; i < N; ++i) s += a[i] * b[i]; return s; } \
  inline float length(V a) { return std::sqrt(dot(a, a)); }                                     \
  inline V normalize(V a) { return a / length(a); }

GLMLITE_OPS(vec2, 2)
GLMLITE_OPS(vec3, 3)
GLMLITE_OPS(vec4, 4)
#undef GLMLITE_OPS

#define GLMLITE_UNARY(name, f)                                                         \
  inline float name(float a) { return f(a); }                                         \
  inline vec2 name(vec2 a) { return vec2(f(a.x), f(a.y)); }                           \
  inline vec3 name(vec3 a) { return vec3(f(a.x), f(a.y), f(a.z)); }                   \
  inline vec4 name(vec4 a) { return vec4(f(a.x), f(a.y), f(a.z), f(a.w)); }
GLMLITE_UNARY(abs, std::fabs)
GLMLITE_UNARY(acos, std::acos)
GLMLITE_UNARY(cos, std::cos)
GLMLITE_UNARY(sin, std::sin)
GLMLITE_UNARY(exp, std::exp)
GLMLITE_UNARY(log, std::log)
GLMLITE_UNARY(floor, std::floor)
GLMLITE_UNARY(sqrt, std::sqrt)
GLMLITE_UNARY(atan, std::atan)
#undef GLMLITE_UNARY

inline float min(float a, float b) { return b < a ? b : a; }
inline float max(float a, float b) { return a < b ? b : a; }
inline float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
inline float mix(float a, float b, float t) { return a + (b - a) * t; }
inline float pow(float a, float b) { return std::pow(a, b); }
inline float fma(float a, float b, float c) { return std::fma(a, b, c); }
inline float smoothstep(float e0, float e1, float x) {
  const float t = clamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

#define GLMLITE_VFUNCS(V, N, B)                                                                                   \
  inline V min(V a, V b) { V r; for (int i = 0; i < N; ++i) r[i] = min(a[i], b[i]); return r; }                  \
  inline V max(V a, V b) { V r; for (int i = 0; i < N; ++i) r[i] = max(a[i], b[i]); return r; }                  \
  inline V min(V a, float b) { return min(a, V(b)); }                                                            \
  inline V max(V a, float b) { return max(a, V(b)); }                                                            \
  inline V clamp(V x, V lo, V hi) { return min(max(x, lo), hi); }                                                \
  inline V clamp(V x, float lo, float hi) { return clamp(x, V(lo), V(hi)); }                                     \
  inline V mix(V a, V b, V t) { return a + (b - a) * t; }                                                        \
  inline V mix(V a, V b, float t) { return a + (b - a) * t; }                                                    \
  inline V pow(V a, V b) { V r; for (int i = 0; i < N; ++i) r[i] = std::pow(a[i], b[i]); return r; }            \
  inline V smoothstep(V e0, V e1, V x) { V r; for (int i = 0; i < N; ++i) r[i] = smoothstep(e0[i], e1[i], x[i]); return r; } \
  inline B equal(V a, V b) { B r; bool *p = &r.x; for (int i = 0; i < N; ++i) p[i] = a[i] == b[i]; return r; }     \
  inline B notEqual(V a, V b) { B r; bool *p = &r.x; for (int i = 0; i < N; ++i) p[i] = a[i] != b[i]; return r; }  \
  inline B greaterThan(V a, V b) { B r; bool *p = &r.x; for (int i = 0; i < N; ++i) p[i] = a[i] > b[i]; return r; } \
  inline B greaterThanEqual(V a, V b) { B r; bool *p = &r.x; for (int i = 0; i < N; ++i) p[i] = a[i] >= b[i]; return r; } \
  inline B lessThan(V a, V b) { B r; bool *p = &r.x; for (int i = 0; i < N; ++i) p[i] = a[i] < b[i]; return r; }  \
  inline bool all(B b) { const bool *p = &b.x; for (int i = 0; i < N; ++i) if (!p[i]) return false; return true; } \
  inline bool any(B b) { const bool *p = &b.x; for (int i = 0; i < N; ++i) if (p[i]) return true; return false; }
GLMLITE_VFUNCS(vec2, 2, bvec2)
GLMLITE_VFUNCS(vec3, 3, bvec3)
GLMLITE_VFUNCS(vec4, 4, bvec4)
#undef GLMLITE_VFUNCS

inline vec3 cross(vec3 a, vec3 b) { return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline vec3 reflect(vec3 i, vec3 n) { return i - 2.0f * dot(n, i) * n; }

}  // namespace glmlite

using glmlite::bvec2;
using glmlite::bvec3;
using glmlite::bvec4;
using glmlite::vec2;
using glmlite::vec3;
using glmlite::vec4;
using namespace glmlite;
