// TEST INFRASTRUCTURE ONLY.  Stand-in for OWL's owl/common.h: the __both__ qualifier
// and the interval<T> pair the reference's headers name.
#pragma once

#include "common/math/vec.h"

namespace owl {
namespace common {

template <typename T>
struct interval {
  T lo{}, hi{};
  interval() = default;
  interval(T a, T b) : lo(a), hi(b) {}
};

}  // namespace common
}  // namespace owl
