// TEST INFRASTRUCTURE ONLY: the stand-ins of oracle/ref_shim whose arithmetic must not
// be contracted into FMA (compiled with -ffp-contract=off, linked into
// oracle/_ref/libref_track.so): CUDA's texture fetches and OWL's RGBA8 packing, in the
// arithmetic this project fixes for them (ref_shim/ref_texture.h, ref_shim/owl/owl.h).
#include <cmath>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "owl/owl.h"
#include "ref_texture.h"

namespace {

struct Texture {
  const float *data;   // volume: float voxels; transfer function: RGBA texels
  int X, Y, Z;         // a transfer function is X texels by 1
  bool rgba;
};
std::vector<Texture> g_textures;   // handle h is g_textures[h - 1]

int f2i(float x) {
  if (!(x == x)) return 0;
  if (x >= 2147483648.0f) return 2147483647;
  if (x <= -2147483648.0f) return (-2147483647 - 1);
  return (int)x;
}
int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// linear filtering along one axis of n texels: the two texels and the 8-bit weight
struct Tap {
  int i0, i1;
  float a;
};
Tap tap(float u, int n) {
  const float x = std::fma(u, (float)n, -0.5f);
  const float fl = std::floor(x);
  Tap t;
  t.a = std::rint((x - fl) * 256.0f) * (1.0f / 256.0f);
  const int i = f2i(fl);
  t.i0 = clampi(i, 0, n - 1);
  t.i1 = clampi(i + 1, 0, n - 1);
  return t;
}
float lerp(float a, float p, float q) { return std::fma(a, q, (1.0f - a) * p); }

}  // namespace

extern "C" {

cudaTextureObject_t ref_texture_volume(const float *data, int X, int Y, int Z) {
  g_textures.push_back(Texture{data, X, Y, Z, false});
  return (cudaTextureObject_t)g_textures.size();
}
cudaTextureObject_t ref_texture_tf(const float *rgba, int n) {
  g_textures.push_back(Texture{rgba, n, 1, 1, true});
  return (cudaTextureObject_t)g_textures.size();
}
void ref_textures_clear() { g_textures.clear(); }

}  // extern "C"

template <>
float tex3D<float>(cudaTextureObject_t tex, float x, float y, float z) {
  const Texture &t = g_textures[(size_t)tex - 1];
  const Tap ax = tap(x, t.X), ay = tap(y, t.Y), az = tap(z, t.Z);
  auto at = [&](int i, int j, int k) { return t.data[((size_t)k * t.Y + j) * t.X + i]; };
  const float c00 = lerp(ax.a, at(ax.i0, ay.i0, az.i0), at(ax.i1, ay.i0, az.i0));
  const float c10 = lerp(ax.a, at(ax.i0, ay.i1, az.i0), at(ax.i1, ay.i1, az.i0));
  const float c01 = lerp(ax.a, at(ax.i0, ay.i0, az.i1), at(ax.i1, ay.i0, az.i1));
  const float c11 = lerp(ax.a, at(ax.i0, ay.i1, az.i1), at(ax.i1, ay.i1, az.i1));
  return lerp(az.a, lerp(ay.a, c00, c10), lerp(ay.a, c01, c11));
}

template <>
float4 tex2D<float4>(cudaTextureObject_t tex, float x, float y) {
  const Texture &t = g_textures[(size_t)tex - 1];
  const Tap ax = tap(x, t.X), ay = tap(y, t.Y);
  float out[4];
  for (int k = 0; k < 4; k++) {
    auto at = [&](int i, int j) { return t.data[4 * ((size_t)j * t.X + i) + k]; };
    out[k] = lerp(ay.a, lerp(ax.a, at(ax.i0, ay.i0), at(ax.i1, ay.i0)), lerp(ax.a, at(ax.i0, ay.i1), at(ax.i1, ay.i1)));
  }
  return float4{out[0], out[1], out[2], out[3]};
}

namespace owl {
uint32_t make_rgba(const vec4f &c) {
  auto q = [](float v) {
    v = std::fmin(std::fmax(v, 0.f), 1.f);
    return (uint32_t)f2i(v * 255.0f + 0.5f);
  };
  return q(c.x) | (q(c.y) << 8) | (q(c.z) << 16) | (q(c.w) << 24);
}
}  // namespace owl
