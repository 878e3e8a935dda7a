// TEST INFRASTRUCTURE ONLY.  Stand-in for the OptiX 7 device API (optix_device.h; the
// OptiX SDK is not installed here) for compiling the reference's deviceCode.cu as host
// code.  The program macros name plain functions (__raygen__mainRG, __closesthit__...,
// ...), and the ray-state queries read the state of the trace that the host-side
// pipeline of oracle/ref_track_pins.cpp is running on the calling thread.
#pragma once

#include <cstdint>
#include <vector_types.h>

typedef unsigned long long OptixTraversableHandle;

enum OptixRayFlags {
  OPTIX_RAY_FLAG_NONE = 0u,
  OPTIX_RAY_FLAG_DISABLE_ANYHIT = 1u << 0,
};

#define OPTIX_RAYGEN_PROGRAM(name) extern "C" void __raygen__##name
#define OPTIX_CLOSEST_HIT_PROGRAM(name) extern "C" void __closesthit__##name
#define OPTIX_ANY_HIT_PROGRAM(name) extern "C" void __anyhit__##name
#define OPTIX_INTERSECT_PROGRAM(name) extern "C" void __intersection__##name
#define OPTIX_MISS_PROGRAM(name) extern "C" void __miss__##name
#define OPTIX_BOUNDS_PROGRAM(name) extern "C" void __boundsFunc__##name

float3 optixGetWorldRayOrigin();
float3 optixGetWorldRayDirection();
float3 optixGetObjectRayOrigin();
float3 optixGetObjectRayDirection();
float optixGetRayTmin();
float optixGetRayTmax();
unsigned int optixGetPrimitiveIndex();
float2 optixGetTriangleBarycentrics();
bool optixReportIntersection(float hitT, unsigned int hitKind);
