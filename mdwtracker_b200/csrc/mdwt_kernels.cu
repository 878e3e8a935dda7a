// mdwt_kernels.cu -- sm_100a kernels of the multi-density Woodcock tracker.
//
// Compiled with --fmad=false: every fused multiply-add below is an explicit fmaf(),
// placed where the reference's expression has the a*b+c form that nvcc contracts
// by default.  Divisions and square roots are IEEE (no fast-math), so the kernels
// reproduce the CPU oracle bit for bit.
//
// Kernels
//   range_xy_kernel / range_z_kernel : per-(cell, channel) value range, the result of
//       rasterElements + rasterBox (renderer.cu:487-519, 835-893) computed as a
//       separable box min/max over voxel intervals (no atomics, volume read once).
//   majorant_kernel : _recalculateDensityRangesMM / _recalculateDensityRanges(float2*)
//       (renderer.cu:111-203): TF-mapped maximum per (cell, channel) or per cell.
//   track_kernel<MODE, STORE> : mainRG + baseLineDTCH (-m 0) / altMultiMajDTCH (-m 2)
//       (deviceCode.cu:283-471, 747-970) + dda3 (dda.h:81-202), one persistent thread
//       per pixel at a time, the spp loop and the DDA/Woodcock loops flattened into one
//       state machine so that a lane that finishes a path starts its next path at once.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <mutex>

#include "../../include/mdwt.h"
#include "mdwt_internal.h"

namespace mdwt {
namespace {

constexpr int kTrackTPB = 128;

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

// sampleVolumeTexture (deviceCode.cu:122-132): NaN outside [0,1]^3, else trilinear.
template <int SK>
__device__ __forceinline__ float sample_volume(const TrackParams &P, int ch, float px, float py, float pz) {
  if (px < 0.0f || px > 1.0f || py < 0.0f || py > 1.0f || pz < 0.0f || pz > 1.0f) return __int_as_float(0x7fc00000);
  const int X = P.dims[ch][0], Y = P.dims[ch][1], Z = P.dims[ch][2];
  const Axis ax = axis(px, X), ay = axis(py, Y), az = axis(pz, Z);
  const void *base = P.vol[ch];
  const size_t sXY = (size_t)X * (size_t)Y;
  const size_t z0 = (size_t)az.i0 * sXY, z1 = (size_t)az.i1 * sXY;
  const size_t y0 = (size_t)ay.i0 * X, y1 = (size_t)ay.i1 * X;
  const float v000 = vox<SK>(base, z0 + y0 + ax.i0), v100 = vox<SK>(base, z0 + y0 + ax.i1);
  const float v010 = vox<SK>(base, z0 + y1 + ax.i0), v110 = vox<SK>(base, z0 + y1 + ax.i1);
  const float v001 = vox<SK>(base, z1 + y0 + ax.i0), v101 = vox<SK>(base, z1 + y0 + ax.i1);
  const float v011 = vox<SK>(base, z1 + y1 + ax.i0), v111 = vox<SK>(base, z1 + y1 + ax.i1);
  const float c00 = lerpf(ax.a, v000, v100);
  const float c10 = lerpf(ax.a, v010, v110);
  const float c01 = lerpf(ax.a, v001, v101);
  const float c11 = lerpf(ax.a, v011, v111);
  const float c0 = lerpf(ay.a, c00, c10);
  const float c1 = lerpf(ay.a, c01, c11);
  return lerpf(az.a, c0, c1);
}

// transferFunction (deviceCode.cu:27-42), alpha part; the lookup axis is returned for
// the colour fetch at a hit.
__device__ __forceinline__ float tf_alpha(const TrackParams &P, int ch, float f, Axis &ax) {
  const int n = P.tfN[ch];
  if (n <= 0) return 0.f;
  const float v0 = P.vd[ch][0], v1 = P.vd[ch][1];
  if (f < v0 || f > v1) return 0.f;
  const float r1 = (f - v0) / (v1 - v0);
  const float r2 = (r1 - P.xd[ch][0]) / (P.xd[ch][1] - P.xd[ch][0]);
  ax = axis(r2, n);
  const float *A = P.tfAlpha[ch];
  return lerpf(ax.a, __ldg(A + ax.i0), __ldg(A + ax.i1)) * P.os[ch];
}

__device__ __forceinline__ uint32_t q8(float c) {
  const float v = fminf(fmaxf(c, 0.f), 1.f);
  return (uint32_t)f2i(v * 255.0f + 0.5f);
}

// ------------------------------------------------------------------ 3D-DDA (dda.h:81-202)
struct DDA {
  float tnx, tny, tnz;   // t_next
  float tsx, tsy, tsz;   // t_step
  int cx, cy, cz;        // cell
  int sx, sy, sz;        // stop (gridSize or -1; delta = +1 / -1 follows from it)
  float rt0, ncb;        // ray_t0, next_cell_begin
  uint32_t visits;
};

__device__ __forceinline__ bool dda_init(const TrackParams &P, float ox, float oy, float oz,
                                         float dx, float dy, float dz, DDA &d) {
  const float fsx = (float)P.mc[0], fsy = (float)P.mc[1], fsz = (float)P.mc[2];
  const float rx = 1.0f / dx, ry = 1.0f / dy, rz = 1.0f / dz;
  const float tlx = (0.0f - ox) * rx, thx = (fsx - ox) * rx;
  const float tly = (0.0f - oy) * ry, thy = (fsy - oy) * ry;
  const float tlz = (0.0f - oz) * rz, thz = (fsz - oz) * rz;
  float nrx = fminf(tlx, thx), nry = fminf(tly, thy), nrz = fminf(tlz, thz);
  const float frx = fmaxf(tlx, thx), fry = fmaxf(tly, thy), frz = fmaxf(tlz, thz);
  if (dx == 0.f) { if (ox < 0.f || ox > fsx) return false; nrx = __int_as_float(0x7f800000); }
  if (dy == 0.f) { if (oy < 0.f || oy > fsy) return false; nry = __int_as_float(0x7f800000); }
  if (dz == 0.f) { if (oz < 0.f || oz > fsz) return false; nrz = __int_as_float(0x7f800000); }
  const float rt0 = fmaxf(0.f, fmaxf(fmaxf(nrx, nry), nrz));
  const float rt1 = fminf(1e20f, fminf(fminf(frx, fry), frz));
  if (rt0 > rt1) return false;
  const float ivx = fmaf(rt0, dx, ox), ivy = fmaf(rt0, dy, oy), ivz = fmaf(rt0, dz, oz);
  const float fcx = fmaxf(0.f, fminf(fsx - 1.f, floorf(ivx)));
  const float fcy = fmaxf(0.f, fminf(fsy - 1.f, floorf(ivy)));
  const float fcz = fmaxf(0.f, fminf(fsz - 1.f, floorf(ivz)));
  const float ex = dx > 0.f ? fcx + 1.f : fcx;
  const float ey = dy > 0.f ? fcy + 1.f : fcy;
  const float ez = dz > 0.f ? fcz + 1.f : fcz;
  d.tsx = fabsf(rx); d.tsy = fabsf(ry); d.tsz = fabsf(rz);
  const float inf = __int_as_float(0x7f800000);
  d.tnx = (dx == 0.f) ? inf : fabsf(ex - ivx) * d.tsx;
  d.tny = (dy == 0.f) ? inf : fabsf(ey - ivy) * d.tsy;
  d.tnz = (dz == 0.f) ? inf : fabsf(ez - ivz) * d.tsz;
  d.sx = dx > 0.f ? (int)P.mc[0] : -1;
  d.sy = dy > 0.f ? (int)P.mc[1] : -1;
  d.sz = dz > 0.f ? (int)P.mc[2] : -1;
  d.cx = (int)fcx; d.cy = (int)fcy; d.cz = (int)fcz;
  d.rt0 = rt0;
  d.ncb = 0.f;
  d.visits = 0;
  return true;
}

// Advance past the current cell; false when the walk leaves the grid.
__device__ __forceinline__ bool dda_advance(DDA &d, uint32_t maxCells) {
  const float tc = fminf(fminf(d.tnx, d.tny), d.tnz);
  d.ncb = tc;
  if (d.tnx == tc) { d.tnx += d.tsx; d.cx += d.sx < 0 ? -1 : 1; if (d.cx == d.sx) return false; }
  if (d.tny == tc) { d.tny += d.tsy; d.cy += d.sy < 0 ? -1 : 1; if (d.cy == d.sy) return false; }
  if (d.tnz == tc) { d.tnz += d.tsz; d.cz += d.sz < 0 ? -1 : 1; if (d.cz == d.sz) return false; }
  return d.visits < maxCells;
}

// Grid-space ray of the trackers (deviceCode.cu:759-778).
__device__ __forceinline__ void grid_ray(const TrackParams &P, float wdx, float wdy, float wdz,
                                         float &ox, float &oy, float &oz, float &dx, float &dy, float &dz,
                                         float &w2g, float &g2w) {
  ox = P.gScale.x * (P.camOrg.x - P.gLo.x);
  oy = P.gScale.y * (P.camOrg.y - P.gLo.y);
  oz = P.gScale.z * (P.camOrg.z - P.gLo.z);
  dx = P.gScale.x * wdx; dy = P.gScale.y * wdy; dz = P.gScale.z * wdz;
  const float n2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
  w2g = sqrtf(n2);
  g2w = 1.f / w2g;
  const float inv = 1.0f / sqrtf(n2);
  dx = dx * inv; dy = dy * inv; dz = dz * inv;
}

enum : int { ST_PIXEL = 0, ST_SAMPLE, ST_DDAINIT, ST_CELL, ST_CHAN, ST_ADVANCE, ST_FINISH, ST_STEP, ST_DONE };

template <int MODE, int SK>
__global__ void __launch_bounds__(kTrackTPB) track_kernel(const __grid_constant__ TrackParams P) {
  const int C = P.C;
  const uint32_t maxCells = P.mc[0] + P.mc[1] + P.mc[2] + 3u;
  const unsigned int nthreads = gridDim.x * blockDim.x;
  unsigned int item = blockIdx.x * blockDim.x + threadIdx.x;
  bool first = true;

  int state = ST_PIXEL;
  int px = 0, py = 0, s = 0;
  float fr = 0.f, fg = 0.f, fbb = 0.f, fa = 1.f;
  uint32_t nsamp = 0, nrej = 0, ncell = 0, nhits = 0, chx = 0;
  unsigned long long totSamp = 0, totRej = 0, totCell = 0, totPaths = 0, totCap = 0;
  uint32_t rng = 0, steps = 0;
  float wdx = 0.f, wdy = 0.f, wdz = 0.f, t1w = 0.f, w2g = 0.f, g2w = 0.f;
  DDA d;
  d.visits = 0;
  int ch = 0;
  float maj = 0.f, t = 0.f, lim = 0.f, ct0 = 0.f, ct1 = 0.f;
  bool hit = false, capped = false;
  int hitCh = 0;
  float ar = 0.f, ag = 0.f, ab = 0.f;
  int cellID = 0;

  while (true) {
    // ---------------- bookkeeping transitions until the lane is ready to step
    while (state != ST_STEP && state != ST_DONE) {
      switch (state) {
        case ST_PIXEL: {
          unsigned int idx;
          if (first) { idx = item; first = false; }
          else idx = nthreads + atomicAdd(P.workCounter, 1u);
          if (idx >= (unsigned int)P.numTiles * 32u) { state = ST_DONE; break; }
          const int tile = (int)(idx >> 5), w = (int)(idx & 31u);
          px = (tile % P.tilesX) * 8 + (w & 7);
          py = (tile / P.tilesX) * 4 + (w >> 3);
          if (px >= P.W || py >= P.H) break;  // stay in ST_PIXEL: fetch the next one
          s = 0;
          fr = 0.f; fg = 0.f; fbb = 0.f; fa = 1.f;
          nsamp = nrej = ncell = nhits = chx = 0;
          state = ST_SAMPLE;
        } break;

        case ST_SAMPLE: {
          if (s == P.spp) {
            // end of pixel: /spp, running mean, RGBA8 (deviceCode.cu:435, 463-471)
            const float fs = (float)P.spp;
            float o0 = fr / fs, o1 = fg / fs, o2 = fbb / fs, o3 = fa / fs;
            const size_t pix = (size_t)px + (size_t)P.W * (size_t)py;
            if (P.accumulate) {
              float4 *ap = reinterpret_cast<float4 *>(P.accum) + pix;
              const float4 prev = *ap;
              const float k = (float)P.accumParam, k1 = (float)(P.accumParam + 1u);
              o0 = fmaf(k, prev.x, o0) / k1;
              o1 = fmaf(k, prev.y, o1) / k1;
              o2 = fmaf(k, prev.z, o2) / k1;
              o3 = fmaf(k, prev.w, o3) / k1;
              *ap = make_float4(o0, o1, o2, o3);
            }
            const int fx = P.mirror ? (P.W - 1 - px) : px;
            P.fb[(size_t)fx + (size_t)P.W * (size_t)py] = q8(o0) | (q8(o1) << 8) | (q8(o2) << 16) | (q8(o3) << 24);
            if (P.stats) {
              uint4 *sp = reinterpret_cast<uint4 *>(P.stats) + pix;
              *sp = make_uint4(nsamp, nrej, nhits, chx);
            }
            totSamp += nsamp; totRej += nrej; totCell += ncell;
            state = ST_PIXEL;
            break;
          }
          // seeding, jitter, generateRay (deviceCode.cu:293-298, 61-76)
          const uint32_t seed = (uint32_t)P.W * (uint32_t)P.H * (P.frameParam + 1u) * (uint32_t)(s + 1);
          rng = tea4((uint32_t)px + seed, (uint32_t)py + seed);
          const float jit = rng_next(rng);
          const float sxf = ((float)px + jit) / (float)P.W;
          const float syf = ((float)py + jit) / (float)P.H;
          float dx = fmaf(syf, P.camVer.x, fmaf(sxf, P.camHor.x, P.camLlc.x));
          float dy = fmaf(syf, P.camVer.y, fmaf(sxf, P.camHor.y, P.camLlc.y));
          float dz = fmaf(syf, P.camVer.z, fmaf(sxf, P.camHor.z, P.camLlc.z));
          if (fabsf(dx) < 1e-5f) dx = 1e-5f;
          if (fabsf(dy) < 1e-5f) dy = 1e-5f;
          if (fabsf(dz) < 1e-5f) dz = 1e-5f;
          dx = dx - P.camOrg.x; dy = dy - P.camOrg.y; dz = dz - P.camOrg.z;
          const float inv = 1.0f / sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
          wdx = dx * inv; wdy = dy * inv; wdz = dz * inv;
          hit = false; capped = false; steps = 0;
          // volumeIntersection against the union box (deviceCode.cu:1676-1726)
          const float frx = 1.0f / wdx, fry = 1.0f / wdy, frz = 1.0f / wdz;
          const float t1 = (P.rootLo.x - P.camOrg.x) * frx, t2 = (P.rootHi.x - P.camOrg.x) * frx;
          const float t3 = (P.rootLo.y - P.camOrg.y) * fry, t4 = (P.rootHi.y - P.camOrg.y) * fry;
          const float t5 = (P.rootLo.z - P.camOrg.z) * frz, t6 = (P.rootHi.z - P.camOrg.z) * frz;
          const float th0 = fmaxf(fmaxf(fminf(t1, t2), fminf(t3, t4)), fminf(t5, t6));
          const float th1 = fminf(fminf(fmaxf(t1, t2), fmaxf(t3, t4)), fmaxf(t5, t6));
          if (th1 < 0 || th0 >= th1) { state = ST_FINISH; break; }
          t1w = fminf(1e20f, th1);
          if (MODE == 2) {
            float ox, oy, oz, gx, gy, gz;
            grid_ray(P, wdx, wdy, wdz, ox, oy, oz, gx, gy, gz, w2g, g2w);
            state = dda_init(P, ox, oy, oz, gx, gy, gz, d) ? ST_CELL : ST_FINISH;
          } else {
            ch = 0;
            lim = 1e20f;
            state = ST_DDAINIT;
          }
        } break;

        case ST_DDAINIT: {  // N-DDA: one full traversal per channel (deviceCode.cu:965-969)
          if (ch == C) { state = ST_FINISH; break; }
          float ox, oy, oz, gx, gy, gz;
          grid_ray(P, wdx, wdy, wdz, ox, oy, oz, gx, gy, gz, w2g, g2w);
          if (dda_init(P, ox, oy, oz, gx, gy, gz, d)) state = ST_CELL;
          else ch++;
        } break;

        case ST_CELL: {
          const float tc = fminf(fminf(d.tnx, d.tny), d.tnz);
          ct0 = d.rt0 + d.ncb;
          ct1 = d.rt0 + fminf(tc, 1e20f);
          d.visits++;
          ncell++;
          cellID = d.cx + d.cy * (int)P.mc[0] + d.cz * (int)P.mc[0] * (int)P.mc[1];
          if (MODE == 2) {
            lim = ct1;   // minT
            ch = 0;
            state = ST_CHAN;
          } else {
            maj = __ldg(P.majorants + (size_t)cellID * C + ch);
            if (maj == 0.0f) state = ST_ADVANCE;
            else { t = ct0; state = ST_STEP; }
          }
        } break;

        case ST_CHAN: {  // syncDDA: next channel of this cell
          if (ch == C) { state = hit ? ST_FINISH : ST_ADVANCE; break; }
          maj = __ldg(P.majorants + (size_t)cellID * C + ch);
          t = ct0;
          if (maj == 0.0f) { ch++; break; }
          state = ST_STEP;
        } break;

        case ST_ADVANCE: {
          if (dda_advance(d, maxCells)) state = ST_CELL;
          else if (MODE == 2) state = ST_FINISH;
          else { ch++; state = ST_DDAINIT; }
        } break;

        case ST_FINISH: {
          // shading with the default flags (deviceCode.cu:323-433) and over(color, bg)
          float cr = 0.f, cg = 0.f, cb = 0.f, ca = 0.f;
          if (hit) {
            nhits++;
            chx ^= (uint32_t)(hitCh + 1) << (s & 15);
            const float kd = (1.0f * 1.0f) * P.lightIntensity;
            const float ks = (0.0f * 1.0f) * P.lightIntensity;
            const F3 sc = P.matSpec[hitCh];
            const float mr = fmaf(ar, 0.75f, sc.x * 0.25f);
            const float mg = fmaf(ag, 0.75f, sc.y * 0.25f);
            const float mb = fmaf(ab, 0.75f, sc.z * 0.25f);
            cr = fmaf(P.ambient, mr, fmaf(ks, mr, kd * ar));
            cg = fmaf(P.ambient, mg, fmaf(ks, mg, kd * ag));
            cb = fmaf(P.ambient, mb, fmaf(ks, mb, kd * ab));
            ca = 1.0f;
          }
          const float oma = 1.0f - ca;
          fr += fmaf(P.bg.x * 1.0f, oma, cr);
          fg += fmaf(P.bg.y * 1.0f, oma, cg);
          fbb += fmaf(P.bg.z * 1.0f, oma, cb);
          fa += fmaf(oma, 1.0f, ca);
          totPaths++;
          if (capped) totCap++;
          s++;
          state = ST_SAMPLE;
        } break;

        default: state = ST_DONE; break;
      }
    }
    if (__all_sync(0xffffffffu, state == ST_DONE)) break;
    if (state != ST_STEP) continue;

    // ---------------- one Woodcock step (the converged part of the loop)
    if (++steps >= kMaxStepsPerSample) { capped = true; hit = false; state = ST_FINISH; continue; }
    {
      const float u = rng_next(rng);
      t = fmaf(-((mlog(1.0f - u) / maj) * P.dt), w2g, t);
      if (MODE == 2) {
        if (t >= lim) { ch++; state = ST_CHAN; continue; }
      } else {
        if (t >= ct1) { state = ST_ADVANCE; continue; }
        if (lim < t) { ch++; state = ST_DDAINIT; continue; }
      }
      const float tW = t * g2w;
      const float xs = fmaf(tW, wdx, P.camOrg.x) * P.w2u.x;
      const float ys = fmaf(tW, wdy, P.camOrg.y) * P.w2u.y;
      const float zs = fmaf(tW, wdz, P.camOrg.z) * P.w2u.z;
      if (tW >= t1w) {
        nrej++;
        if (MODE == 2) {
          if (ch == C - 1) state = ST_FINISH;
          else { ch++; state = ST_CHAN; }
        } else {
          ch++;
          state = ST_DDAINIT;
        }
        continue;
      }
      const float thr = rng_next(rng) * maj;
      const float v = sample_volume<SK>(P, ch, xs, ys, zs);
      nsamp++;
      if (v == v) {
        Axis tax;
        const float a = tf_alpha(P, ch, v, tax);
        if (a > 0.0f && thr < a) {
          const float *R = P.tfRgba[ch];
          ar = lerpf(tax.a, __ldg(R + 4 * tax.i0 + 0), __ldg(R + 4 * tax.i1 + 0));
          ag = lerpf(tax.a, __ldg(R + 4 * tax.i0 + 1), __ldg(R + 4 * tax.i1 + 1));
          ab = lerpf(tax.a, __ldg(R + 4 * tax.i0 + 2), __ldg(R + 4 * tax.i1 + 2));
          hit = true;
          hitCh = ch;
          lim = fminf(t, lim);
          if (MODE == 0) { ch++; state = ST_DDAINIT; continue; }
        } else if (MODE == 0) {
          nrej++;
        }
      }
      if (MODE == 2) nrej++;
    }
  }

  // ---------------- counters: warp reduction, one atomic per warp and counter
  unsigned long long v[5] = {totSamp, totRej, totCell, totPaths, totCap};
#pragma unroll
  for (int k = 0; k < 5; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < 5; k++)
      if (v[k]) atomicAdd(P.counters + k, v[k]);
  }
}

// ------------------------------------------------------------------ value ranges
// Pass 1: per (z, cy, cx), min/max over voxels y in ivy[cy], x in ivx[cx] of slice z.
template <int SK>
__global__ void range_xy_kernel(const void *__restrict__ vol, int X, int Y, int Z,
                                const int *__restrict__ ivx, const int *__restrict__ ivy,
                                int mcx, int mcy, float2 *__restrict__ out) {
  const size_t n = (size_t)Z * mcy * mcx;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int cx = (int)(i % mcx);
    const int cy = (int)((i / mcx) % mcy);
    const int z = (int)(i / ((size_t)mcx * mcy));
    const int x0 = __ldg(ivx + 2 * cx), x1 = __ldg(ivx + 2 * cx + 1);
    const int y0 = __ldg(ivy + 2 * cy), y1 = __ldg(ivy + 2 * cy + 1);
    float mn = __int_as_float(0x7f800000), mx = __int_as_float(0xff800000);
    for (int y = y0; y <= y1; y++) {
      const size_t row = ((size_t)z * Y + y) * X;
      for (int x = x0; x <= x1; x++) {
        const float v = vox<SK>(vol, row + x);
        if (v < mn) mn = v;   // NaN never enters (atomicMin CAS loop: `while (val < old)`)
        if (v > mx) mx = v;
      }
    }
    out[i] = make_float2(mn, mx);
  }
}

// Pass 2: per (cz, cy, cx), min/max over z in ivz[cz]; merged with the sizeMCs value
// (1e20, -1e20) into ranges[(cell*C + ch)].
__global__ void range_z_kernel(const float2 *__restrict__ in, const int *__restrict__ ivz, int mcx, int mcy, int mcz,
                               int C, int ch, float2 *__restrict__ ranges) {
  const size_t n = (size_t)mcz * mcy * mcx;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t cxy = i % ((size_t)mcx * mcy);
    const int cz = (int)(i / ((size_t)mcx * mcy));
    const int z0 = __ldg(ivz + 2 * cz), z1 = __ldg(ivz + 2 * cz + 1);
    float2 r = ranges[i * C + ch];
    for (int z = z0; z <= z1; z++) {
      const float2 a = in[(size_t)z * mcx * mcy + cxy];
      if (a.x < r.x) r.x = a.x;
      if (a.y > r.y) r.y = a.y;
    }
    ranges[i * C + ch] = r;
  }
}

__global__ void range_init_kernel(float2 *ranges, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    ranges[i] = make_float2(1e20f, -1e20f);
}

// ------------------------------------------------------------------ majorants
__device__ __forceinline__ float tf_probe(const float *A, int n, float u) {
  const Axis a = axis(u, n);
  return lerpf(a.a, __ldg(A + a.i0), __ldg(A + a.i1));
}

__device__ float channel_majorant(const MajorantParams &p, int c, float mn, float mx) {
  if (mx < mn) return 0.f;
  const int n = p.tfN[c];
  if (n <= 0) return 0.f;
  const float *A = p.tfAlpha[c];
  const float os = p.os[c];
  const float v0 = p.vd[c][0], v1 = p.vd[c][1], x0 = p.xd[c][0], x1 = p.xd[c][1];
  const float rmin1 = (mn - v0) / (v1 - v0);
  const float rmin = (rmin1 - x0) / (x1 - x0);
  const float rmax1 = (mx - v0) / (v1 - v0);
  const float rmax = (rmax1 - x0) / (x1 - x0);
  const float addr1 = rmin * (float)n;
  const float addr2 = rmax * (float)n;
  const int aMin = clampi(f2i(fminf(floorf(addr1), floorf(addr2))), 0, n - 1);
  const int aMax = clampi(f2i(fmaxf(ceilf(addr1), ceilf(addr2))), 0, n - 1);
  float m = 0.f;
  for (int i = aMin; i <= aMax; ++i) {
    const float dns = tf_probe(A, n, ((float)i + 0.5f) / (float)n) * os;
    m = (i == aMin) ? dns : fmaxf(m, dns);
  }
  m = fmaxf(m, tf_probe(A, n, (addr1 + 0.5f) / (float)n) * os);
  m = fmaxf(m, tf_probe(A, n, (addr2 + 0.5f) / (float)n) * os);
  return m;
}

__global__ void majorant_kernel(const __grid_constant__ MajorantParams p) {
  const int C = p.C;
  for (size_t cell = (size_t)blockIdx.x * blockDim.x + threadIdx.x; cell < p.M; cell += (size_t)gridDim.x * blockDim.x) {
    const float2 *r = reinterpret_cast<const float2 *>(p.ranges) + cell * C;
    if (p.mode == 3) {
      float sum = 0.f;
      for (int c = 0; c < C; c++) {
        const float2 rc = r[c];
        if (rc.y < rc.x) continue;
        sum += channel_majorant(p, c, rc.x, rc.y);
      }
      p.majorants[cell] = sum;
    } else {
      for (int c = 0; c < C; c++) {
        const float2 rc = r[c];
        p.majorants[cell * C + c] = channel_majorant(p, c, rc.x, rc.y);
      }
    }
  }
}

inline int grid_for(size_t n, int tpb, int cap) {
  size_t g = (n + tpb - 1) / tpb;
  if (g < 1) g = 1;
  if (g > (size_t)cap) g = cap;
  return (int)g;
}

}  // namespace

// ------------------------------------------------------------------ launchers
// Persistent launch: as many CTAs as fit on the device at once.
template <int MODE, int SK>
static int launch_track_t(const TrackParams &p, cudaStream_t st, int numSMs, int *grid) {
  int bps = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, track_kernel<MODE, SK>, kTrackTPB, 0);
  if (e != cudaSuccess) return (int)e;
  if (bps < 1) bps = 1;
  *grid = numSMs * bps;
  track_kernel<MODE, SK><<<*grid, kTrackTPB, 0, st>>>(p);
  return (int)cudaGetLastError();
}

int launch_track(const TrackParams &p, int storeKind, void *stream, int numSMs, int *launches, int *grid, int *block) {
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (p.mode == 2) rc = storeKind == kStoreU8 ? launch_track_t<2, kStoreU8>(p, st, numSMs, grid) : launch_track_t<2, kStoreF32>(p, st, numSMs, grid);
  else if (p.mode == 0) rc = storeKind == kStoreU8 ? launch_track_t<0, kStoreU8>(p, st, numSMs, grid) : launch_track_t<0, kStoreF32>(p, st, numSMs, grid);
  else return (int)cudaErrorInvalidValue;
  *block = kTrackTPB;
  if (launches) *launches += 1;
  return rc;
}

int track_occupancy(int storeKind, int mode, int *blocksPerSM, int *threadsPerBlock) {
  cudaError_t e;
  if (mode == 2) e = storeKind == kStoreU8 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSM, track_kernel<2, kStoreU8>, kTrackTPB, 0)
                                           : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSM, track_kernel<2, kStoreF32>, kTrackTPB, 0);
  else e = storeKind == kStoreU8 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSM, track_kernel<0, kStoreU8>, kTrackTPB, 0)
                                 : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSM, track_kernel<0, kStoreF32>, kTrackTPB, 0);
  *threadsPerBlock = kTrackTPB;
  return (int)e;
}

int launch_ranges_init(float *ranges, size_t count, void *stream, int *launches) {
  range_init_kernel<<<grid_for(count, 256, 4096), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<float2 *>(ranges), count);
  if (launches) *launches += 1;
  return (int)cudaGetLastError();
}

int launch_ranges(const void *vol, int storeKind, const int dims[3], const uint32_t mc[3],
                  const int *ivx, const int *ivy, const int *ivz, int C, int ch,
                  float *ranges, float *scratchA, float * /*scratchB*/, void *stream, int *launches) {
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n1 = (size_t)dims[2] * mc[1] * mc[0];
  float2 *A = reinterpret_cast<float2 *>(scratchA);
  if (storeKind == kStoreU8)
    range_xy_kernel<kStoreU8><<<grid_for(n1, 256, 148 * 64), 256, 0, st>>>(vol, dims[0], dims[1], dims[2], ivx, ivy, (int)mc[0], (int)mc[1], A);
  else
    range_xy_kernel<kStoreF32><<<grid_for(n1, 256, 148 * 64), 256, 0, st>>>(vol, dims[0], dims[1], dims[2], ivx, ivy, (int)mc[0], (int)mc[1], A);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  const size_t n2 = (size_t)mc[2] * mc[1] * mc[0];
  range_z_kernel<<<grid_for(n2, 256, 148 * 64), 256, 0, st>>>(A, ivz, (int)mc[0], (int)mc[1], (int)mc[2], C, ch,
                                                              reinterpret_cast<float2 *>(ranges));
  if (launches) *launches += 2;
  return (int)cudaGetLastError();
}

int launch_majorants(const MajorantParams &p, void *stream, int *launches) {
  majorant_kernel<<<grid_for(p.M, 128, 148 * 32), 128, 0, (cudaStream_t)stream>>>(p);
  if (launches) *launches += 1;
  return (int)cudaGetLastError();
}

// ------------------------------------------------------------------ range build without allocation
// Scratch of mdwt_build_ranges_noalloc: the per-(z, cell-y, cell-x) partial ranges and
// the voxel intervals.  Module globals: every device that loads the library holds them
// (8 MiB + 24 KiB) until the process exits.
namespace {
constexpr size_t kNoAllocPairs = size_t(1) << 20;
constexpr int kNoAllocMaxCells = 1024;
static __device__ __align__(256) float2 g_noalloc_pairs[kNoAllocPairs];
static __device__ __align__(256) int g_noalloc_iv[3 * 2 * kNoAllocMaxCells];

__device__ __forceinline__ int project_d(float f, float lo, float hi, int dim) {
  int v = f2i((float)dim * (f - lo) / (hi - lo));
  v = v < dim - 1 ? v : dim - 1;
  return v > 0 ? v : 0;
}

// Cells [clo, chi] that the 27-neighbour box of voxel p touches on one axis.
__device__ __forceinline__ void voxel_cells(int p, int D, int md, float wlo, float whi, float len, int &clo, int &chi) {
  const float vlo = fmaf((float)p, len, wlo);
  float blo = vlo, bhi = vlo + len;
  if (p - 1 >= 0) { const float nl = fmaf((float)(p - 1), len, wlo); blo = fminf(blo, nl); bhi = fmaxf(bhi, nl); }
  if (p + 1 < D) { const float nl = fmaf((float)(p + 1), len, wlo); blo = fminf(blo, nl); bhi = fmaxf(bhi, nl); }
  clo = project_d(blo, wlo, whi, md);
  const int h = project_d(bhi, wlo, whi, md);
  chi = h < md - 1 ? h : md - 1;
}

// One thread per (axis, cell index): the voxel interval of the separable range build,
// found by binary search (clo and chi are non-decreasing in p for these bounds).
__global__ void noalloc_intervals_kernel(int dx, int dy, int dz, int mx, int my, int mz, float lx, float ly, float lz,
                                         float hx, float hy, float hz, int *iv) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int D, md, off;
  float wlo, whi;
  if (t < mx) { D = dx; md = mx; wlo = lx; whi = hx; off = 0; }
  else if (t < mx + my) { t -= mx; D = dy; md = my; wlo = ly; whi = hy; off = 2 * mx; }
  else if (t < mx + my + mz) { t -= mx + my; D = dz; md = mz; wlo = lz; whi = hz; off = 2 * (mx + my); }
  else return;
  const int k = t;
  const float len = (whi - wlo) / (float)D;
  int lo = 0, hi = D;
  while (lo < hi) {  // first p with chi(p) >= k
    const int mid = (lo + hi) >> 1;
    int cl, ch;
    voxel_cells(mid, D, md, wlo, whi, len, cl, ch);
    if (ch >= k) hi = mid; else lo = mid + 1;
  }
  const int pmin = lo;
  lo = 0; hi = D;
  while (lo < hi) {  // first p with clo(p) > k
    const int mid = (lo + hi) >> 1;
    int cl, ch;
    voxel_cells(mid, D, md, wlo, whi, len, cl, ch);
    if (cl > k) hi = mid; else lo = mid + 1;
  }
  const int pmax = lo - 1;
  if (pmin > pmax) { iv[off + 2 * k] = 1; iv[off + 2 * k + 1] = 0; return; }
  iv[off + 2 * k] = pmin - 1 > 0 ? pmin - 1 : 0;
  iv[off + 2 * k + 1] = pmax + 1 < D - 1 ? pmax + 1 : D - 1;
}

std::mutex g_noalloc_mu;
constexpr int kNoAllocMaxDevices = 64;
void *g_noalloc_pairs_ptr[kNoAllocMaxDevices];
int *g_noalloc_iv_ptr[kNoAllocMaxDevices];
bool g_noalloc_ready[kNoAllocMaxDevices];

bool bounds_ok(float lo, float hi, int64_t D) {
  if (!std::isfinite(lo) || !std::isfinite(hi) || !(hi > lo)) return false;
  const float scale = std::fmax(std::fabs(lo), std::fabs(hi));
  return (hi - lo) / (float)D >= 1e-6f * scale;
}
}  // namespace

}  // namespace mdwt

// Value ranges of one channel computed without allocating any memory.  For callers that
// must not allocate device memory: code running inside an application's own memory pool
// or under an allocator that forbids cudaMalloc, or plug-ins that are handed device
// buffers and a stream but no allocation rights.  The scratch is the module-global
// g_noalloc_pairs / g_noalloc_iv; the first call on a device looks up their addresses
// (cudaGetSymbolAddress), so make that first call before any stream capture.  All calls
// share the scratch: calls that overlap on the GPU (two streams, two threads) race.
extern "C" mdwt_status mdwt_build_ranges_noalloc(const void *d_volume, int format, const int64_t dims[3],
                                                 const uint32_t macrocells[3], const float world_lo[3],
                                                 const float world_hi[3], float *d_ranges_out, void *cuda_stream) {
  using namespace mdwt;
  if (!d_volume || !dims || !macrocells || !world_lo || !world_hi || !d_ranges_out) return MDWT_ERR_BAD_ARG;
  if (format != MDWT_FMT_UINT8 && format != MDWT_FMT_FLOAT32) return MDWT_ERR_UNSUPPORTED;
  for (int a = 0; a < 3; a++) {
    if (dims[a] <= 0 || dims[a] > (1 << 20) || macrocells[a] == 0) return MDWT_ERR_BAD_ARG;
    if (macrocells[a] > (uint32_t)kNoAllocMaxCells) return MDWT_ERR_SCRATCH_LIMIT;
    if (!bounds_ok(world_lo[a], world_hi[a], dims[a])) return MDWT_ERR_UNSUPPORTED;
  }
  if ((size_t)dims[2] * macrocells[1] * macrocells[0] > kNoAllocPairs) return MDWT_ERR_SCRATCH_LIMIT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) { cudaGetLastError(); return MDWT_ERR_CUDA; }
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ready[dev]) {
      void *p = nullptr, *q = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_pairs) != cudaSuccess ||
          cudaGetSymbolAddress(&q, g_noalloc_iv) != cudaSuccess) {
        cudaGetLastError();
        return MDWT_ERR_CUDA;
      }
      g_noalloc_pairs_ptr[dev] = p;
      g_noalloc_iv_ptr[dev] = (int *)q;
      g_noalloc_ready[dev] = true;
    }
  }
  cudaStream_t st = (cudaStream_t)cuda_stream;
  const int mx = (int)macrocells[0], my = (int)macrocells[1], mz = (int)macrocells[2];
  int *iv = g_noalloc_iv_ptr[dev];
  noalloc_intervals_kernel<<<(mx + my + mz + 127) / 128, 128, 0, st>>>(
      (int)dims[0], (int)dims[1], (int)dims[2], mx, my, mz, world_lo[0], world_lo[1], world_lo[2],
      world_hi[0], world_hi[1], world_hi[2], iv);
  if (cudaGetLastError() != cudaSuccess) return MDWT_ERR_CUDA;
  const size_t M = (size_t)mx * my * mz;
  if (launch_ranges_init(d_ranges_out, M, st, nullptr) != 0) return MDWT_ERR_CUDA;
  const int d3[3] = {(int)dims[0], (int)dims[1], (int)dims[2]};
  const uint32_t mc3[3] = {macrocells[0], macrocells[1], macrocells[2]};
  const int sk = format == MDWT_FMT_UINT8 ? kStoreU8 : kStoreF32;
  if (launch_ranges(d_volume, sk, d3, mc3, iv, iv + 2 * mx, iv + 2 * (mx + my), 1, 0, d_ranges_out,
                    (float *)g_noalloc_pairs_ptr[dev], nullptr, st, nullptr) != 0)
    return MDWT_ERR_CUDA;
  return MDWT_OK;
}
