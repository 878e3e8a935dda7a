// TEST INFRASTRUCTURE ONLY.  Stand-in for OWL's box types (owl/common/math/box.h):
// the lower/upper pairs the reference's dda.h, rawFile.h and deviceCode.cu construct and
// read, and box3f::including (the bounds programs of deviceCode.cu).
#pragma once

#include "vec.h"

namespace owl {
namespace common {

struct box3f {
  vec3f lower, upper;
  box3f() = default;
  box3f(const vec3f &lo, const vec3f &hi) : lower(lo), upper(hi) {}
  box3f including(const vec3f &p) const { return box3f(min(lower, p), max(upper, p)); }
  box3f &extend(const vec3f &p) { lower = min(lower, p); upper = max(upper, p); return *this; }
};

struct box4f {
  vec4f lower, upper;
  box4f() = default;
  box4f(const vec4f &lo, const vec4f &hi) : lower(lo), upper(hi) {}
};

}  // namespace common
}  // namespace owl
