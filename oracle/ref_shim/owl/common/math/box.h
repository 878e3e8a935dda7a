// TEST INFRASTRUCTURE ONLY.  Stand-in for OWL's box types (owl/common/math/box.h):
// the lower/upper pairs the reference's dda.h, rawFile.h and deviceCode.cu construct and
// read, and box3f::including (the bounds programs of deviceCode.cu); extend and size for
// the range raster of renderer.cu (component-wise min / max, upper - lower).
#pragma once

#include "vec.h"

namespace owl {
namespace common {

struct box3f {
  vec3f lower, upper;
  box3f() = default;
  SHIM_HD box3f(const vec3f &lo, const vec3f &hi) : lower(lo), upper(hi) {}
  SHIM_HD box3f including(const vec3f &p) const { return box3f(min(lower, p), max(upper, p)); }
  SHIM_HD box3f &extend(const vec3f &p) { lower = min(lower, p); upper = max(upper, p); return *this; }
  SHIM_HD vec3f size() const { return upper - lower; }
  SHIM_HD vec3f center() const { return (lower + upper) * 0.5f; }
};

struct box4f {
  vec4f lower, upper;
  box4f() = default;
  SHIM_HD box4f &extend(const vec4f &p) {
    lower = vec4f(min(lower.x, p.x), min(lower.y, p.y), min(lower.z, p.z), min(lower.w, p.w));
    upper = vec4f(max(upper.x, p.x), max(upper.y, p.y), max(upper.z, p.z), max(upper.w, p.w));
    return *this;
  }
  SHIM_HD vec4f size() const { return vec4f(upper.x - lower.x, upper.y - lower.y, upper.z - lower.z, upper.w - lower.w); }
  SHIM_HD vec4f center() const {
    return vec4f((lower.x + upper.x) * 0.5f, (lower.y + upper.y) * 0.5f, (lower.z + upper.z) * 0.5f,
                 (lower.w + upper.w) * 0.5f);
  }
  SHIM_HD box4f(const vec4f &lo, const vec4f &hi) : lower(lo), upper(hi) {}
};

}  // namespace common
}  // namespace owl
