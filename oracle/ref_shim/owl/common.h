// TEST INFRASTRUCTURE ONLY.  Stand-in for OWL's owl/common.h: the __both__ qualifier
// and the interval<T> pair the reference's headers name.
#pragma once

#include "common/math/vec.h"

namespace owl {
namespace common {

// the reference names the bounds both lo / hi (deviceCode.cu) and lower / upper (renderer.cu)
template <typename T>
struct interval {
  union { T lo; T lower; };
  union { T hi; T upper; };
  SHIM_HD interval() : lo(), hi() {}
  SHIM_HD interval(T a, T b) : lo(a), hi(b) {}
};

}  // namespace common
}  // namespace owl
