// TEST INFRASTRUCTURE ONLY.  Stand-ins for CUDA's texture fetches tex3D<float> and
// tex2D<float4>, which deviceCode.cu calls on the volume and transfer-function textures
// (normalized coordinates, linear filtering, clamp addressing).  The fetch follows the
// CUDA C Programming Guide's description of linear filtering, in the arithmetic this
// project fixes for it: x = fmaf(u, N, -0.5), i = floor(x), weight = rint((x - i) * 256)
// / 256 (8 fractional bits), texel indices clamped to [0, N-1], lerp(a, p, q) =
// fmaf(a, q, (1 - a) * p), along x, then y, then z.  Texture objects are handles that
// oracle/ref_track_pins.cpp registers.
#pragma once

#include <cuda_runtime.h>

template <typename T>
T tex3D(cudaTextureObject_t tex, float x, float y, float z);
template <typename T>
T tex2D(cudaTextureObject_t tex, float x, float y);
template <>
float tex3D<float>(cudaTextureObject_t tex, float x, float y, float z);
template <>
float4 tex2D<float4>(cudaTextureObject_t tex, float x, float y);
