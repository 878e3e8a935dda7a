// TEST INFRASTRUCTURE ONLY.  Stand-in for OWL's 3x3 linear frame (owl/common/math/
// LinearSpace.h): the camera frame of the reference's camera.h (columns vx, vy, vz,
// identity from `one`; LinearSpace3f and det() for unstructuredElementHelper.h).  Rotation and products are declared for camera.h's manipulator,
// which the pins never call.
#pragma once

#include "box.h"

namespace owl {
namespace common {

struct OneTy {};
static const OneTy one = OneTy();

struct linear3f {
  vec3f vx, vy, vz;
  linear3f() = default;
  SHIM_HD linear3f(OneTy) : vx(1.f, 0.f, 0.f), vy(0.f, 1.f, 0.f), vz(0.f, 0.f, 1.f) {}
  SHIM_HD linear3f(const vec3f &a, const vec3f &b, const vec3f &c) : vx(a), vy(b), vz(c) {}
  SHIM_HD static linear3f rotate(const vec3f &axis, float radians);
  SHIM_HD float det() const { return dot(vx, cross(vy, vz)); }
};
typedef linear3f LinearSpace3f;
linear3f operator*(const linear3f &a, const linear3f &b);

}  // namespace common
}  // namespace owl
