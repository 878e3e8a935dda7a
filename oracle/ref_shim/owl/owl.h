// TEST INFRASTRUCTURE ONLY.  Stand-in for OWL's owl/owl.h (submodule empty): the host
// handle types the reference's renderer.h declares members of, and the device-side
// helpers deviceCode.cu calls (launch index and size, per-ray payload, program data,
// Ray, traceRay).  The device helpers read the per-thread state that the host-side
// pipeline of oracle/ref_track_pins.cpp sets up; traceRay hands the ray to that pipeline.
#pragma once

#include <cstdint>

#include "common.h"
#include "common/math/box.h"
#include "common/math/random.h"
#include "../optix_device.h"

typedef struct _OWLContext *OWLContext;
typedef struct _OWLBuffer *OWLBuffer;
typedef struct _OWLGeom *OWLGeom;
typedef struct _OWLGeomType *OWLGeomType;
typedef struct _OWLGroup *OWLGroup;
typedef struct _OWLModule *OWLModule;
typedef struct _OWLParams *OWLParams;
typedef struct _OWLRayGen *OWLRayGen;
typedef struct _OWLMissProg *OWLMissProg;

namespace owl {

struct Ray {
  vec3f origin, direction;
  float tmin = 0.f, tmax = 1e30f, time = 0.f;
};

namespace shim {
// per-thread state of the host-side pipeline (defined in oracle/ref_track_pins.cpp)
vec2i launch_index();
vec2i launch_dims();
void *payload();
const void *program_data();
void trace(OptixTraversableHandle handle, const Ray &ray, void *prd, unsigned flags);
}  // namespace shim

inline vec2i getLaunchIndex() { return shim::launch_index(); }
inline vec2i getLaunchDims() { return shim::launch_dims(); }
template <typename T>
inline T &getPRD() { return *static_cast<T *>(shim::payload()); }
template <typename T>
inline const T &getProgramData() { return *static_cast<const T *>(shim::program_data()); }
template <typename PRD>
inline void traceRay(OptixTraversableHandle handle, const Ray &ray, PRD &prd, unsigned flags = 0u) {
  shim::trace(handle, ray, &prd, flags);
}

// OWL's RGBA8 packing, as this project specifies it (the submodule is not vendored):
// each channel clamped to [0, 1], times 255, plus 0.5, truncated; r in the low byte.
uint32_t make_rgba(const vec4f &c);

}  // namespace owl
