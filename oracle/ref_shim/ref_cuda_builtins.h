// TEST INFRASTRUCTURE ONLY.  What CUDA device code finds without an include and a host
// compile of deviceCode.cu does not: the threadIdx built-in (per host thread, set by the
// pipeline of oracle/ref_track_pins.cpp for each launch index) and the unqualified
// float isnan of CUDA's math overloads.
#pragma once

#include <cmath>
#include <vector_types.h>

extern thread_local uint3 threadIdx;
using std::isnan;
