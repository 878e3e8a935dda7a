// mdwt_expected.cu -- FP64 ground truth for convergence measurements.
//
// expected_kernel: per pixel, the expected value of the trackers' per-sample estimate
// (unshaded), in double precision.  All trackers (-m 0..3) sample the first collision of
// the superposed channels: a channel-c collision at world distance t has density
// T(t) mu_c(t), mu_c = alpha_c / dt (dt scales every free flight, deviceCode.cu:800-806)
// and shows channel c's shaded TF colour (deviceCode.cu:408-433); no collision before the
// root-box exit shows the background.  The integral over t is a midpoint rule with the
// extinction held constant over each step (exact exponential attenuation per step); the
// pixel footprint is the diagonal jitter (one draw for x and y, deviceCode.cu:298),
// averaged by a J-point midpoint rule.  Opacity and colour follow the trackers' filtering
// semantics (8-bit fractional weights, clamp) evaluated in double.
//
// rmse_kernel: sum of squared differences between the accumulation buffer's RGB and the
// expected image, in double.
#include <cuda_runtime.h>
#include <stdint.h>

#include "mdwt_internal.h"
#include "mdwt_math.cuh"

namespace mdwt {
namespace {

struct AxisD {
  int i0, i1;
  double a;
};
__device__ __forceinline__ AxisD axis_d(double u, int n) {
  const double x = u * (double)n - 0.5;
  const double fl = floor(x);
  AxisD r;
  r.a = rint((x - fl) * 256.0) / 256.0;
  const long long i = (long long)fl;
  r.i0 = (int)(i < 0 ? 0 : (i > n - 1 ? n - 1 : i));
  r.i1 = (int)(i < -1 ? -1 : (i > n - 2 ? n - 2 : i)) + 1;
  return r;
}
__device__ __forceinline__ double lerp_d(double a, double p, double q) { return (1.0 - a) * p + a * q; }

template <int SK>
__device__ double volume_d(const TrackParams &P, int c, const double p[3]) {
  for (int a = 0; a < 3; a++)
    if (!(p[a] >= 0.0 && p[a] <= 1.0)) return __longlong_as_double(0x7ff8000000000000ll);
  const int X = P.dims[c][0], Y = P.dims[c][1], Z = P.dims[c][2];
  const AxisD ax = axis_d(p[0], X), ay = axis_d(p[1], Y), az = axis_d(p[2], Z);
  const void *v = P.vol[c];
  auto at = [&](int x, int y, int z) { return (double)vox<SK>(v, vidx<SK, size_t>(x, y, z, X, Y)); };
  const double c00 = lerp_d(ax.a, at(ax.i0, ay.i0, az.i0), at(ax.i1, ay.i0, az.i0));
  const double c10 = lerp_d(ax.a, at(ax.i0, ay.i1, az.i0), at(ax.i1, ay.i1, az.i0));
  const double c01 = lerp_d(ax.a, at(ax.i0, ay.i0, az.i1), at(ax.i1, ay.i0, az.i1));
  const double c11 = lerp_d(ax.a, at(ax.i0, ay.i1, az.i1), at(ax.i1, ay.i1, az.i1));
  return lerp_d(az.a, lerp_d(ay.a, c00, c10), lerp_d(ay.a, c01, c11));
}

__device__ double tf_d(const TrackParams &P, int c, double f, double rgb[3]) {
  rgb[0] = rgb[1] = rgb[2] = 0.0;
  const int n = P.tfN[c];
  const double vd0 = P.vd[c][0], vd1 = P.vd[c][1];
  if (n <= 0 || !(f >= vd0 && f <= vd1)) return 0.0;
  const double r1 = (f - vd0) / (vd1 - vd0);
  const double r2 = (r1 - (double)P.xd[c][0]) / ((double)P.xd[c][1] - (double)P.xd[c][0]);
  const AxisD a = axis_d(r2, n);
  const float *R = P.tfRgba[c];
  for (int k = 0; k < 3; k++) rgb[k] = lerp_d(a.a, R[4 * a.i0 + k], R[4 * a.i1 + k]);
  return lerp_d(a.a, R[4 * a.i0 + 3], R[4 * a.i1 + 3]) * (double)P.os[c];
}

template <int SK>
__global__ void __launch_bounds__(128) expected_kernel(const __grid_constant__ TrackParams P, int J, double h0,
                                                       double *out) {
  const unsigned npix = (unsigned)P.W * (unsigned)P.H;
  const int C = P.C;
  const double org[3] = {P.camOrg.x, P.camOrg.y, P.camOrg.z};
  const double llc[3] = {P.camLlc.x, P.camLlc.y, P.camLlc.z}, hor[3] = {P.camHor.x, P.camHor.y, P.camHor.z};
  const double ver[3] = {P.camVer.x, P.camVer.y, P.camVer.z};
  const double rlo[3] = {P.rootLo.x, P.rootLo.y, P.rootLo.z}, rhi[3] = {P.rootHi.x, P.rootHi.y, P.rootHi.z};
  const double glo[3] = {P.gLo.x, P.gLo.y, P.gLo.z};
  const double ghi[3] = {P.gHi.x, P.gHi.y, P.gHi.z};
  const double w2u[3] = {1.0 / (ghi[0] - glo[0]), 1.0 / (ghi[1] - glo[1]), 1.0 / (ghi[2] - glo[2])};
  const double bg[3] = {P.bg.x, P.bg.y, P.bg.z};
  const double dt = P.dt, amb = P.ambient, li = P.lightIntensity;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
    const int px = (int)(i % (unsigned)P.W), py = (int)(i / (unsigned)P.W);
    double acc[3] = {0, 0, 0};
    for (int m = 0; m < J; m++) {
      const double j = (m + 0.5) / J;
      const double sx = (px + j) / P.W, sy = (py + j) / P.H;
      double d[3];
      for (int a = 0; a < 3; a++) {
        d[a] = llc[a] + sx * hor[a] + sy * ver[a];
        if (fabs(d[a]) < 1e-5) d[a] = 1e-5;   // generateRay clamps the point (deviceCode.cu:70-72)
        d[a] -= org[a];
      }
      const double inv = 1.0 / sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      for (int a = 0; a < 3; a++) d[a] *= inv;
      double ta = 0.0, tb = 1e300;
      for (int a = 0; a < 3; a++) {
        const double lo[2] = {rlo[a], glo[a]}, hi[2] = {rhi[a], ghi[a]};
        for (int b = 0; b < 2; b++) {
          const double t1 = (lo[b] - org[a]) / d[a], t2 = (hi[b] - org[a]) / d[a];
          ta = fmax(ta, fmin(t1, t2));
          tb = fmin(tb, fmax(t1, t2));
        }
      }
      double L[3] = {0, 0, 0}, T = 1.0;
      if (tb > ta) {
        const long long n = (long long)ceil((tb - ta) / h0);
        const double h = (tb - ta) / (double)n;
        for (long long s = 0; s < n && T > 1e-300; s++) {
          const double t = ta + (s + 0.5) * h;
          double p[3];
          for (int a = 0; a < 3; a++) p[a] = (org[a] + t * d[a]) * w2u[a];
          double mu = 0.0, cw[3] = {0, 0, 0};
          for (int c = 0; c < C; c++) {
            const double v = volume_d<SK>(P, c, p);
            if (v != v) continue;
            double alb[3];
            const double al = tf_d(P, c, v, alb);
            if (!(al > 0.0)) continue;
            const double mc = al / dt;
            mu += mc;
            const double sc[3] = {P.matSpec[c].x, P.matSpec[c].y, P.matSpec[c].z};
            for (int k = 0; k < 3; k++) cw[k] += mc * (amb * (0.75 * alb[k] + 0.25 * sc[k]) + li * alb[k]);
          }
          if (mu > 0.0) {
            const double att = exp(-mu * h);
            for (int k = 0; k < 3; k++) L[k] += T * (1.0 - att) * (cw[k] / mu);
            T *= att;
          }
        }
      }
      for (int k = 0; k < 3; k++) acc[k] += L[k] + T * bg[k];
    }
    for (int k = 0; k < 3; k++) out[3 * (size_t)i + k] = acc[k] / J;
  }
}

__global__ void __launch_bounds__(256) rmse_kernel(const float *accum, const double *ref, unsigned npix, double *sum) {
  double s = 0.0;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
    const float4 a = reinterpret_cast<const float4 *>(accum)[i];
    const double d0 = (double)a.x - ref[3 * (size_t)i], d1 = (double)a.y - ref[3 * (size_t)i + 1];
    const double d2 = (double)a.z - ref[3 * (size_t)i + 2];
    s += d0 * d0 + d1 * d1 + d2 * d2;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double ws[8];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += ws[w];
    atomicAdd(sum, t);
  }
}

}  // namespace

int launch_expected(const TrackParams &p, int storeKind, int J, double h0, double *out, void *stream, int numSMs,
                    int *launches) {
  cudaStream_t st = (cudaStream_t)stream;
  const size_t npix = (size_t)p.W * (size_t)p.H;
  size_t g = (npix + 127) / 128;
  if (g > (size_t)numSMs * 16) g = (size_t)numSMs * 16;
  if (storeKind == kStoreU8) expected_kernel<kStoreU8><<<(unsigned)g, 128, 0, st>>>(p, J, h0, out);
  else expected_kernel<kStoreF32><<<(unsigned)g, 128, 0, st>>>(p, J, h0, out);
  if (launches) *launches += 1;
  return (int)cudaGetLastError();
}

int launch_rmse(const float *accum, const double *ref, size_t npix, double *sum, void *stream, int numSMs,
                int *launches) {
  cudaStream_t st = (cudaStream_t)stream;
  size_t g = (npix + 255) / 256;
  if (g > (size_t)numSMs * 8) g = (size_t)numSMs * 8;
  if (g == 0) g = 1;
  rmse_kernel<<<(unsigned)g, 256, 0, st>>>(accum, ref, (unsigned)npix, sum);
  if (launches) *launches += 1;
  return (int)cudaGetLastError();
}

}  // namespace mdwt
