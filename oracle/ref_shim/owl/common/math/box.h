// TEST INFRASTRUCTURE ONLY.  Stand-in for OWL's box types (owl/common/math/box.h):
// the lower/upper pairs the reference's dda.h and rawFile.h construct and read.
#pragma once

#include "vec.h"

namespace owl {
namespace common {

struct box3f {
  vec3f lower, upper;
  box3f() = default;
  box3f(const vec3f &lo, const vec3f &hi) : lower(lo), upper(hi) {}
};

struct box4f {
  vec4f lower, upper;
  box4f() = default;
  box4f(const vec4f &lo, const vec4f &hi) : lower(lo), upper(hi) {}
};

}  // namespace common
}  // namespace owl
