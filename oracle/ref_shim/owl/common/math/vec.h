// TEST INFRASTRUCTURE ONLY.  A minimal stand-in for the vector types of OWL's math
// library (owl-project/owl, owl/common/math/vec.h), which the reference's sources include
// but whose submodule is empty and whose commit is unpinned.  It declares only what the
// reference's dda.h and rawFile.h use, so that oracle/Makefile can compile those reference
// files where they lie (into oracle/_ref/) and the oracle can be checked against them.
//
// Element-wise semantics are those of the reference's CUDA device code, where OWL's
// helpers resolve to CUDA's float overloads: scalar min/max are fminf/fmaxf, abs is
// fabsf, and rcp is the correctly rounded 1/x.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>

#ifndef __CUDACC__
#define __device__
#define __host__
#endif
#ifndef CUDART_INF
#define CUDART_INF __builtin_inf()   // a double, like CUDA's math_constants.h
#endif

namespace owl {
namespace common {

inline float min(float a, float b) { return fminf(a, b); }
inline float max(float a, float b) { return fmaxf(a, b); }
inline float abs(float a) { return fabsf(a); }
inline float rcp(float a) { return 1.0f / a; }

struct vec3ui {
  uint32_t x = 0, y = 0, z = 0;
  vec3ui() = default;
  vec3ui(uint32_t a, uint32_t b, uint32_t c) : x(a), y(b), z(c) {}
};

struct vec3i;

struct vec3f {
  float x = 0.f, y = 0.f, z = 0.f;
  vec3f() = default;
  explicit vec3f(float s) : x(s), y(s), z(s) {}
  vec3f(float a, float b, float c) : x(a), y(b), z(c) {}
  explicit vec3f(const vec3ui &v) : x((float)v.x), y((float)v.y), z((float)v.z) {}
  explicit vec3f(const vec3i &v);
};

struct vec3i {
  int x = 0, y = 0, z = 0;
  vec3i() = default;
  vec3i(int a, int b, int c) : x(a), y(b), z(c) {}
  explicit vec3i(const vec3f &v) : x((int)v.x), y((int)v.y), z((int)v.z) {}
};
inline vec3f::vec3f(const vec3i &v) : x((float)v.x), y((float)v.y), z((float)v.z) {}

struct vec3l {
  int64_t x = 0, y = 0, z = 0;
  vec3l() = default;
  vec3l(int64_t a, int64_t b, int64_t c) : x(a), y(b), z(c) {}
};

struct vec4f {
  float x = 0.f, y = 0.f, z = 0.f, w = 0.f;
  vec4f() = default;
  vec4f(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
};

inline vec3f operator+(const vec3f &a, const vec3f &b) { return vec3f(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3f operator-(const vec3f &a, const vec3f &b) { return vec3f(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3f operator*(const vec3f &a, const vec3f &b) { return vec3f(a.x * b.x, a.y * b.y, a.z * b.z); }
inline vec3f operator*(float s, const vec3f &b) { return vec3f(s * b.x, s * b.y, s * b.z); }
inline vec3f operator*(const vec3f &a, float s) { return vec3f(a.x * s, a.y * s, a.z * s); }
inline vec3f operator+(const vec3f &a, float s) { return vec3f(a.x + s, a.y + s, a.z + s); }
inline vec3f operator-(const vec3f &a, float s) { return vec3f(a.x - s, a.y - s, a.z - s); }
inline bool operator==(const vec3f &a, const vec3f &b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

inline vec3f min(const vec3f &a, const vec3f &b) { return vec3f(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline vec3f max(const vec3f &a, const vec3f &b) { return vec3f(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline vec3f abs(const vec3f &a) { return vec3f(abs(a.x), abs(a.y), abs(a.z)); }
inline vec3f rcp(const vec3f &a) { return vec3f(rcp(a.x), rcp(a.y), rcp(a.z)); }
inline float reduce_min(const vec3f &a) { return min(min(a.x, a.y), a.z); }
inline float reduce_max(const vec3f &a) { return max(max(a.x, a.y), a.z); }

}  // namespace common
using namespace common;
}  // namespace owl
