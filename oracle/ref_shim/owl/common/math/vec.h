// TEST INFRASTRUCTURE ONLY.  A minimal stand-in for the vector types of OWL's math
// library (owl-project/owl, owl/common/math/vec.h), which the reference's sources include
// but whose submodule is empty and whose commit is unpinned.  It declares what the
// reference's dda.h, rawFile.h, camera.h and deviceCode.cu use, so that oracle/Makefile
// can compile those reference files where they lie (into oracle/_ref/) and the oracle can
// be checked against them.
//
// Element-wise semantics are those of the reference's CUDA device code, where OWL's
// helpers resolve to CUDA's float overloads: scalar min/max are fminf/fmaxf, abs is
// fabsf, rcp is the correctly rounded 1/x, and sqrt is the correctly rounded square root.
// length(v) = sqrt(dot(v, v)) and normalize(v) = v * (1 / sqrt(dot(v, v))), the
// arithmetic this project fixes for OWL's helpers (the oracle and the kernels use it).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <type_traits>

#include <vector_types.h>   // CUDA's float3 / float4 / uint3 (host-usable plain structs)

#ifndef __CUDACC__
#ifndef __device__
#define __device__
#endif
#ifndef __host__
#define __host__
#endif
#endif
#ifndef __both__
#ifdef __CUDACC__
#define __both__ __host__ __device__
#else
#define __both__
#endif
#endif
// Every function of the stand-in is usable from host and device code under nvcc (the
// reference's renderer.cu, compiled for the GPU pins) and plain under a host compiler.
#ifdef __CUDACC__
#define SHIM_HD __host__ __device__
#else
#define SHIM_HD
#endif
#ifndef CUDART_INF
#define CUDART_INF __builtin_inf()   // a double, like CUDA's math_constants.h
#endif

namespace owl {
namespace common {

#ifdef __CUDACC__
// under nvcc the scalar overloads are CUDA's own (fminf / fmaxf for float)
using ::min;
using ::max;
using ::abs;
#else
inline float min(float a, float b) { return fminf(a, b); }
inline float max(float a, float b) { return fmaxf(a, b); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline float abs(float a) { return fabsf(a); }
#endif
SHIM_HD inline float rcp(float a) { return 1.0f / a; }

// ---------------------------------------------------------------- 2-D
struct vec2i;
struct vec2f {
  union { float x; float u; };
  union { float y; float v; };
  SHIM_HD vec2f() : x(0.f), y(0.f) {}
  SHIM_HD explicit vec2f(float s) : x(s), y(s) {}
  SHIM_HD vec2f(float a, float b) : x(a), y(b) {}
  SHIM_HD explicit vec2f(const vec2i &o);
  SHIM_HD vec2f(const float2 &o) : x(o.x), y(o.y) {}
};
struct vec2i {
  int x = 0, y = 0;
  vec2i() = default;
  SHIM_HD vec2i(int a, int b) : x(a), y(b) {}
};
SHIM_HD inline vec2f::vec2f(const vec2i &o) : x((float)o.x), y((float)o.y) {}
SHIM_HD inline vec2f operator+(const vec2f &a, float s) { return vec2f(a.x + s, a.y + s); }
SHIM_HD inline vec2f operator+(const vec2f &a, const vec2f &b) { return vec2f(a.x + b.x, a.y + b.y); }
SHIM_HD inline vec2f operator/(const vec2f &a, const vec2f &b) { return vec2f(a.x / b.x, a.y / b.y); }

// ---------------------------------------------------------------- 3-D
struct vec3ui {
  uint32_t x = 0, y = 0, z = 0;
  vec3ui() = default;
  SHIM_HD vec3ui(uint32_t a, uint32_t b, uint32_t c) : x(a), y(b), z(c) {}
  SHIM_HD const uint32_t &operator[](unsigned i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

struct vec3i;
struct vec4f;

struct vec3f {
  float x = 0.f, y = 0.f, z = 0.f;
  vec3f() = default;
  SHIM_HD vec3f(float s) : x(s), y(s), z(s) {}
  SHIM_HD vec3f(float a, float b, float c) : x(a), y(b), z(c) {}
  SHIM_HD explicit vec3f(const vec3ui &v) : x((float)v.x), y((float)v.y), z((float)v.z) {}
  SHIM_HD explicit vec3f(const vec3i &v);
  SHIM_HD explicit vec3f(const vec4f &v);
  SHIM_HD vec3f(const float3 &v) : x(v.x), y(v.y), z(v.z) {}
  SHIM_HD explicit vec3f(const float4 &v) : x(v.x), y(v.y), z(v.z) {}
  SHIM_HD operator float3() const { return make_float3_(x, y, z); }
  SHIM_HD float &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  SHIM_HD const float &operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }

 private:
  SHIM_HD static float3 make_float3_(float a, float b, float c) { float3 r; r.x = a; r.y = b; r.z = c; return r; }
};

struct vec3i {
  int x = 0, y = 0, z = 0;
  vec3i() = default;
  SHIM_HD explicit vec3i(int s) : x(s), y(s), z(s) {}
  SHIM_HD vec3i(int a, int b, int c) : x(a), y(b), z(c) {}
  SHIM_HD explicit vec3i(const uint3 &v) : x((int)v.x), y((int)v.y), z((int)v.z) {}
  SHIM_HD explicit vec3i(const vec3f &v) : x((int)v.x), y((int)v.y), z((int)v.z) {}
  SHIM_HD int &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  SHIM_HD const int &operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
SHIM_HD inline vec3f::vec3f(const vec3i &v) : x((float)v.x), y((float)v.y), z((float)v.z) {}

struct vec3l {
  int64_t x = 0, y = 0, z = 0;
  vec3l() = default;
  SHIM_HD vec3l(int64_t a, int64_t b, int64_t c) : x(a), y(b), z(c) {}
};

template <typename V>
SHIM_HD inline typename std::enable_if<std::is_same<V, vec3f>::value, V>::type operator+(const V &a,
                                                                                   const V &b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename V>
SHIM_HD inline typename std::enable_if<std::is_same<V, vec3f>::value, V>::type operator-(const V &a,
                                                                                   const V &b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename V>
SHIM_HD inline typename std::enable_if<std::is_same<V, vec3f>::value, V>::type operator*(const V &a,
                                                                                   const V &b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
template <typename V>
SHIM_HD inline typename std::enable_if<std::is_same<V, vec3f>::value, V>::type operator/(const V &a,
                                                                                   const V &b) { return V(a.x / b.x, a.y / b.y, a.z / b.z); }
// The vec3f-by-vec3f operators are templates, as OWL's are, so that a float3 operand
// (with the reference's own float3 operators in scope) selects those instead.
SHIM_HD inline vec3f operator*(float s, const vec3f &b) { return vec3f(s * b.x, s * b.y, s * b.z); }
SHIM_HD inline vec3f operator*(const vec3f &a, float s) { return vec3f(a.x * s, a.y * s, a.z * s); }
SHIM_HD inline vec3f operator/(const vec3f &a, float s) { return vec3f(a.x / s, a.y / s, a.z / s); }
SHIM_HD inline vec3f operator/(float s, const vec3f &b) { return vec3f(s / b.x, s / b.y, s / b.z); }
SHIM_HD inline vec3f operator+(const vec3f &a, float s) { return vec3f(a.x + s, a.y + s, a.z + s); }
SHIM_HD inline vec3f operator-(const vec3f &a, float s) { return vec3f(a.x - s, a.y - s, a.z - s); }
SHIM_HD inline vec3f operator-(const vec3f &a) { return vec3f(-a.x, -a.y, -a.z); }
SHIM_HD inline vec3f &operator+=(vec3f &a, const vec3f &b) { a = a + b; return a; }
SHIM_HD inline vec3f &operator-=(vec3f &a, const vec3f &b) { a = a - b; return a; }
SHIM_HD inline vec3f &operator*=(vec3f &a, float s) { a = a * s; return a; }
SHIM_HD inline vec3f &operator/=(vec3f &a, float s) { a = a / s; return a; }
SHIM_HD inline bool operator==(const vec3f &a, const vec3f &b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
SHIM_HD inline vec3i operator+(const vec3i &a, const vec3i &b) { return vec3i(a.x + b.x, a.y + b.y, a.z + b.z); }
SHIM_HD inline vec3i operator-(const vec3i &a, const vec3i &b) { return vec3i(a.x - b.x, a.y - b.y, a.z - b.z); }
SHIM_HD inline vec3i operator*(const vec3i &a, const vec3i &b) { return vec3i(a.x * b.x, a.y * b.y, a.z * b.z); }
SHIM_HD inline vec3i operator/(const vec3i &a, const vec3i &b) { return vec3i(a.x / b.x, a.y / b.y, a.z / b.z); }
SHIM_HD inline vec3i operator+(const vec3i &a, int s) { return vec3i(a.x + s, a.y + s, a.z + s); }
SHIM_HD inline vec3i operator-(const vec3i &a, int s) { return vec3i(a.x - s, a.y - s, a.z - s); }
// (a + b - 1) / b, per component, and for integers
SHIM_HD inline vec3i divRoundUp(const vec3i &a, const vec3i &b) { return (a + b - 1) / b; }
template <typename I, typename = typename std::enable_if<std::is_integral<I>::value>::type>
SHIM_HD inline I divRoundUp(I a, I b) { return (a + b - 1) / b; }

SHIM_HD inline vec3f min(const vec3f &a, const vec3f &b) { return vec3f(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
SHIM_HD inline vec3f max(const vec3f &a, const vec3f &b) { return vec3f(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
SHIM_HD inline vec3f abs(const vec3f &a) { return vec3f(abs(a.x), abs(a.y), abs(a.z)); }
SHIM_HD inline vec3f rcp(const vec3f &a) { return vec3f(rcp(a.x), rcp(a.y), rcp(a.z)); }
SHIM_HD inline float reduce_min(const vec3f &a) { return min(min(a.x, a.y), a.z); }
SHIM_HD inline float reduce_max(const vec3f &a) { return max(max(a.x, a.y), a.z); }
SHIM_HD inline float dot(const vec3f &a, const vec3f &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SHIM_HD inline vec3f cross(const vec3f &a, const vec3f &b) {
  return vec3f(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
SHIM_HD inline float length(const vec3f &a) { return sqrtf(dot(a, a)); }
SHIM_HD inline vec3f normalize(const vec3f &a) { return a * (1.0f / sqrtf(dot(a, a))); }

// ---------------------------------------------------------------- 4-D
struct vec4f {
  float x = 0.f, y = 0.f, z = 0.f, w = 0.f;
  vec4f() = default;
  SHIM_HD explicit vec4f(float s) : x(s), y(s), z(s), w(s) {}
  SHIM_HD vec4f(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
  SHIM_HD vec4f(const vec3f &v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
  SHIM_HD vec4f(const float4 &v) : x(v.x), y(v.y), z(v.z), w(v.w) {}
  SHIM_HD operator float4() const { float4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r; }
};
SHIM_HD inline vec3f::vec3f(const vec4f &v) : x(v.x), y(v.y), z(v.z) {}
template <typename V>
SHIM_HD inline typename std::enable_if<std::is_same<V, vec4f>::value, V>::type operator+(const V &a,
                                                                                   const V &b) { return V(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
SHIM_HD inline vec4f operator*(const vec4f &a, float s) { return vec4f(a.x * s, a.y * s, a.z * s, a.w * s); }
SHIM_HD inline vec4f operator*(float s, const vec4f &a) { return vec4f(s * a.x, s * a.y, s * a.z, s * a.w); }
SHIM_HD inline vec4f operator/(const vec4f &a, float s) { return vec4f(a.x / s, a.y / s, a.z / s, a.w / s); }
SHIM_HD inline vec4f &operator+=(vec4f &a, const vec4f &b) { a = a + b; return a; }
SHIM_HD inline vec4f &operator/=(vec4f &a, float s) { a = a / s; return a; }

}  // namespace common
using namespace common;
}  // namespace owl
