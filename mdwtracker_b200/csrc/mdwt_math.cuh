// mdwt_math.cuh -- device side of the arithmetic specification shared with the CPU
// oracle: float->int conversion, the TEA-seeded LCG, the project log, and the
// software texture filter (8-bit fractional weights, clamp addressing).  Every
// translation unit that includes it is compiled with --fmad=false; fused
// multiply-adds appear only as explicit fmaf().
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "mdwt_internal.h"

namespace mdwt {
namespace {

// ------------------------------------------------------------------ arithmetic spec
__device__ __forceinline__ int f2i(float x) {
  if (!(x == x)) return 0;
  if (x >= 2147483648.0f) return 2147483647;
  if (x <= -2147483648.0f) return (-2147483647 - 1);
  return (int)x;
}
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// 4-round TEA of the seed words (Wheeler & Needham 1994), key = SHA-256 IV words 0..3.
__device__ __forceinline__ uint32_t tea4(uint32_t v0, uint32_t v1) {
  uint32_t sum = 0;
#pragma unroll
  for (int n = 0; n < 4; n++) {
    sum += 0x9E3779B9u;
    v0 += ((v1 << 4) + 0x6a09e667u) ^ (v1 + sum) ^ ((v1 >> 5) + 0xbb67ae85u);
    v1 += ((v0 << 4) + 0x3c6ef372u) ^ (v0 + sum) ^ ((v0 >> 5) + 0xa54ff53au);
  }
  return v0;
}
// LCG with the Numerical Recipes constants; a draw is the top 24 bits times 2^-24.
__device__ __forceinline__ float rng_next(uint32_t &s) {
  s = 1664525u * s + 1013904223u;
  return (float)(s >> 8) * (1.0f / 16777216.0f);
}

// log(x) for positive normal x: e*ln2 + 2*atanh(s), s = (m-1)/(m+1), m in (sqrt(1/2), sqrt(2)].
__device__ __forceinline__ float mlog(float x) {
  uint32_t b = __float_as_uint(x);
  int e = (int)((b >> 23) & 0xffu) - 127;
  float m = __uint_as_float((b & 0x007fffffu) | 0x3f800000u);
  if (m > 1.41421353816986083984375f) { m = m * 0.5f; e = e + 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float z = s * s;
  float p = fmaf(z, 1.0f / 9.0f, 1.0f / 7.0f);
  p = fmaf(z, p, 1.0f / 5.0f);
  p = fmaf(z, p, 1.0f / 3.0f);
  float s2 = s + s;
  float r = fmaf(s2 * z, p, s2);
  float fe = (float)e;
  return fmaf(fe, 0.693145751953125f, fmaf(fe, 1.428606765330187e-06f, r));
}

// exp(z): z = k*ln2 + r (Cody-Waite reduction with ln2 split hi/lo), |r| <= ln2/2, the
// degree-7 Taylor polynomial of e^r, times 2^k built in the exponent field; 0 below 2^-126.
__device__ __forceinline__ float mexp(float z) {
  if (!(z == z)) return z;
  if (z > 88.0f) return __int_as_float(0x7f800000);
  if (z < -87.0f) return 0.0f;
  const float kf = rintf(z * 1.44269502162933349609375f);
  float r = fmaf(-kf, 0.693145751953125f, z);
  r = fmaf(-kf, 1.428606765330187e-06f, r);
  float p = fmaf(r, 1.0f / 5040.0f, 1.0f / 720.0f);
  p = fmaf(r, p, 1.0f / 120.0f);
  p = fmaf(r, p, 1.0f / 24.0f);
  p = fmaf(r, p, 1.0f / 6.0f);
  p = fmaf(r, p, 0.5f);
  p = fmaf(r, p, 1.0f);
  p = fmaf(r, p, 1.0f);
  const int k = (int)kf;
  if (k < -126) return 0.0f;
  return p * __uint_as_float((uint32_t)(k + 127) << 23);
}
// pow(x, y) for x >= 0: exp(y * log(x)), pow(0, y) = 0.
__device__ __forceinline__ float mpow(float x, float y) {
  if (x == 0.0f) return 0.0f;
  return mexp(y * mlog(x));
}

// a / b correctly rounded, from y = RN(1/b): q = RN(a*y), then one correction with the
// exact residual a - q*b (Markstein 1990: with y the correctly rounded reciprocal and no
// underflow or overflow, RN(q + y*(a - q*b)) is the correctly rounded quotient).  The
// correction runs where |a| >= 2^-80 and 2^-80 <= |q| <= 2^80, so the residual stays a
// normal number; elsewhere (y = 0 included, and NaN) the IEEE division itself.
__device__ __forceinline__ float div_by(float a, float b, float y) {
  const float q = a * y;
  const float aq = fabsf(q);
  if (fabsf(a) >= 8.271806125530277e-25f && aq >= 8.271806125530277e-25f && aq <= 1.2089258196146292e24f)
    return fmaf(fmaf(-q, b, a), y, q);
  return a / b;
}
// RN(1/b) for 2^-80 <= |b| <= 2^80, else 0 (div_by then divides).
__device__ __forceinline__ float recip_for_div(float b) {
  const float ab = fabsf(b);
  return (ab >= 8.271806125530277e-25f && ab <= 1.2089258196146292e24f) ? 1.0f / b : 0.0f;
}

// One Woodcock free flight t - (log(1 - u) / majorant) * dt * w2g (deviceCode.cu:805),
// the quotient from the majorant's reciprocal rmaj = recip_for_div(maj).
__device__ __forceinline__ float flight(float t, float u, float maj, float rmaj, float dt, float w2g) {
  return fmaf(-(div_by(mlog(1.0f - u), maj, rmaj) * dt), w2g, t);
}

// Exit filter of a free flight: true only when flight(t, u, maj, rmaj, dt, w2g) >= lim is
// certain, decided from the hardware log2 (lg2.approx) instead of the exact chain; a
// false answer means "run the exact flight".  k = rmaj * dt * w2g * ln 2.
//   The estimate xf = -log2(1 - u) * k of the flight length differs from the exact chain's
// length by at most |xf| * kFlightRel + |k| * kFlightAbs (negative majorants included), where
//   - mlog's relative error over every 1 - u of the 24-bit draw grid is <= 1.6e-7
//     (checked exhaustively against a double-precision log on the host),
//   - lg2.approx's error over the same 2^24 inputs is below 2^-20 * (1 + |log2 x|)
//     (checked exhaustively on the GPU by the tests),
//   - the roundings of the exact chain (quotient, product by dt) and of k add a few 2^-24,
// and the constants kFlightRel = kFlightAbs = 2^-18 (mdwt_internal.h) take four times
// those bounds and more.  The term |tf| * kFlightTf (2^-22) covers the roundings of tf and
// of the final comparison.  Since the exact t' = RN(t + length) and RN is monotone,
// t + length >= lim implies t' >= lim.
//   Under the fast arithmetic (TrackParams::fast) the flight is fast_flight(t, u, k) = tf
// itself, and a true answer (tf - m >= lim with m >= 0) implies tf >= lim there too.
constexpr float kLn2 = 0.693147182464599609375f;     // RN(ln 2)
__device__ __forceinline__ bool flight_surely_exits(float t, float u, float k, float lim) {
  const float xf = -__log2f(1.0f - u) * k;
  const float tf = t + xf;
  const float m = fmaf(fabsf(xf), kFlightRel, fmaf(fabsf(k), kFlightAbs, fabsf(tf) * kFlightTf));
  return tf - m >= lim;
}
// The fast arithmetic's free flight (TrackParams::fast): the exit filter's estimate
// t + xf itself, k = rmaj * dt * w2g * ln 2 with rmaj = 1 / majorant.  The reference
// computes log(1 - u) / majorant (deviceCode.cu:564, 805, 913, 1023); this is the same
// length from the hardware log2, within lg2.approx's error.
__device__ __forceinline__ float fast_flight(float t, float u, float k) {
  const float xf = -__log2f(1.0f - u) * k;
  return t + xf;
}

__device__ __forceinline__ float quant(float a) { return rintf(a * 256.0f) * (1.0f / 256.0f); }
__device__ __forceinline__ float lerpf(float a, float p, float q) { return fmaf(a, q, (1.0f - a) * p); }

struct Axis { int i0, i1; float a; };
__device__ __forceinline__ Axis axis(float u, int n) {
  const float x = fmaf(u, (float)n, -0.5f);
  const float fl = floorf(x);
  Axis r;
  r.a = quant(x - fl);
  const int i = f2i(fl);
  r.i0 = clampi(i, 0, n - 1);
  r.i1 = clampi(i, -1, n - 2) + 1;
  return r;
}

template <int SK>
__device__ __forceinline__ float vox(const void *base, size_t idx) {
  if (SK == kStoreU8) return (float)__ldg(reinterpret_cast<const uint8_t *>(base) + idx) * 255.0f;
  return __ldg(reinterpret_cast<const float *>(base) + idx);
}
// The element index of voxel (x, y, z) in the storage layout SK (StoreKind).
template <int SK, typename IDX>
__device__ __forceinline__ IDX vidx(int x, int y, int z, int X, int Y) {
  if (SK == kStoreF32) {
    const IDX Xb = (IDX)((X + 1) >> 1), Yb = (IDX)((Y + 1) >> 1);
    return (((IDX)(z >> 1) * Yb + (IDX)(y >> 1)) * Xb + (IDX)(x >> 1)) * 8u + (IDX)(((z & 1) << 2) | ((y & 1) << 1) | (x & 1));
  }
  return ((IDX)z * (IDX)Y + (IDX)y) * (IDX)X + (IDX)x;
}

}  // namespace
}  // namespace mdwt
