// mdwt_track.cu -- the sm_100a tracker: mainRG + baseLineDTCH (-m 0, N-DDA) and
// altMultiMajDTCH (-m 2, syncDDA) of the reference (deviceCode.cu:283-471, 747-970) with
// dda3 (dda.h:81-202), as two kernels per batch of samples.
//
// trace_kernel: one path-sample per lane at a time.  Work items are (8x4 pixel tile,
//   sample) pairs, a warp's 32 consecutive items being one tile at one sample; warps take
//   items in chunks from a global dispenser.  The warp loop has three lane states:
//   NEED lanes start their next path (TEA seed, jitter, ray, root box, grid transform,
//   DDA start) together, once `pool` lanes wait or nothing else runs; TRANS lanes walk
//   channels and macrocells to the next non-zero majorant; STEP lanes take one
//   Woodcock step (free flight, world-exit test, null-collision test with the trilinear
//   fetch and the TF).  A finished path writes a 4-byte record: hit flag, channel, TF
//   texel index and quantized weight -- everything its shaded colour depends on.
// resolve_kernel: per pixel, the records of the batch in sample order -> shading,
//   over(colour, background), running sum; after the last batch /spp, the running
//   mean into the accumulation buffer and RGBA8 (deviceCode.cu:323-471).  Keeping the
//   reference's per-pixel summation order makes the result bit-identical to a
//   sequential spp loop.
// Pixels whose rays certainly miss the root box (outside a conservative screen-space
// rectangle) are not traced; resolve gives them the background result.
// Compiled with --fmad=false; fused multiply-adds are the explicit fmaf() of the
// arithmetic specification shared with the CPU oracle.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>

#include "../../include/mdwt.h"
#include "mdwt_internal.h"
#include "mdwt_math.cuh"

namespace mdwt {
namespace {

constexpr int kTPB = 128;
constexpr int kMinBlocks = 8;   // 64 registers: 32 warps per SM (measured fastest)
constexpr unsigned kFull = 0xffffffffu;

// Path record: bit 31 hit, bits 27..30 channel, bits 13..26 TF texel i0, bit 12 set when
// i1 == i0 (clamped edge), bits 0..8 quantized weight * 256.  0 = miss.
// A free flight from t with draw u (deviceCode.cu:564, 805, 913, 1023) in the arithmetic of
// the request: the exact chain, or the fast arithmetic's length (fast_flight; rmaj = 1 / maj
// there).  The exit filter runs unchanged under both: a flight it passes as leaving the
// cell leaves it in either arithmetic (its margin is non-negative), and the others reach
// this function, whose length the sample stage tests against the cell exit itself.
__device__ __forceinline__ float any_flight(const TrackParams &P, float t, float u, float maj, float rmaj, float w2g) {
  if (P.fast) return fast_flight(t, u, rmaj * (P.dt * w2g * kLn2));
  return flight(t, u, maj, rmaj, P.dt, w2g);
}
// -m 1's per-channel flights (deviceCode.cu:676, 739): t - (log(1 - u) / maj) * dt * w2g.
__device__ __forceinline__ float mode1_flight(const TrackParams &P, float t, float u, float maj, float w2g) {
  if (P.fast) return fast_flight(t, u, (P.dt * w2g * kLn2) / maj);
  return fmaf(-((mlog(1.0f - u) / maj) * P.dt), w2g, t);
}
__device__ __forceinline__ uint32_t make_record(int ch, const Axis &a) {
  const uint32_t k = (uint32_t)(a.a * 256.0f);
  return 0x80000000u | ((uint32_t)ch << 27) | ((uint32_t)a.i0 << 13) | ((a.i1 == a.i0) ? (1u << 12) : 0u) | k;
}

// Texture axis of a coordinate known to be finite and in [0, 1] (so x in [-0.5, n-0.5]):
// the same values as axis(), with floor and conversion in one instruction.
__device__ __forceinline__ Axis axis_in_range(float u, int n) {
  const float x = fmaf(u, (float)n, -0.5f);
  const int i = __float2int_rd(x);
  Axis r;
  r.a = quant(x - (float)i);
  r.i0 = i < 0 ? 0 : i;
  r.i1 = (i < n - 1 ? i : n - 2) + 1;
  return r;
}

template <int SK, typename IDX>
__device__ __forceinline__ float trilinear(const void *base, int X, int Y, const Axis &ax, const Axis &ay, const Axis &az) {
  float v000, v100, v010, v110, v001, v101, v011, v111;
  if (SK == kStoreF32) {   // micro-bricks: the eight corners from at most eight 8-voxel bricks
    v000 = vox<SK>(base, vidx<SK, IDX>(ax.i0, ay.i0, az.i0, X, Y)); v100 = vox<SK>(base, vidx<SK, IDX>(ax.i1, ay.i0, az.i0, X, Y));
    v010 = vox<SK>(base, vidx<SK, IDX>(ax.i0, ay.i1, az.i0, X, Y)); v110 = vox<SK>(base, vidx<SK, IDX>(ax.i1, ay.i1, az.i0, X, Y));
    v001 = vox<SK>(base, vidx<SK, IDX>(ax.i0, ay.i0, az.i1, X, Y)); v101 = vox<SK>(base, vidx<SK, IDX>(ax.i1, ay.i0, az.i1, X, Y));
    v011 = vox<SK>(base, vidx<SK, IDX>(ax.i0, ay.i1, az.i1, X, Y)); v111 = vox<SK>(base, vidx<SK, IDX>(ax.i1, ay.i1, az.i1, X, Y));
  } else {
    const IDX sXY = (IDX)X * (IDX)Y;
    const IDX z0 = (IDX)az.i0 * sXY, z1 = (IDX)az.i1 * sXY;
    const IDX y0 = (IDX)ay.i0 * (IDX)X, y1 = (IDX)ay.i1 * (IDX)X;
    v000 = vox<SK>(base, z0 + y0 + ax.i0); v100 = vox<SK>(base, z0 + y0 + ax.i1);
    v010 = vox<SK>(base, z0 + y1 + ax.i0); v110 = vox<SK>(base, z0 + y1 + ax.i1);
    v001 = vox<SK>(base, z1 + y0 + ax.i0); v101 = vox<SK>(base, z1 + y0 + ax.i1);
    v011 = vox<SK>(base, z1 + y1 + ax.i0); v111 = vox<SK>(base, z1 + y1 + ax.i1);
  }
  const float c00 = lerpf(ax.a, v000, v100);
  const float c10 = lerpf(ax.a, v010, v110);
  const float c01 = lerpf(ax.a, v001, v101);
  const float c11 = lerpf(ax.a, v011, v111);
  const float c0 = lerpf(ay.a, c00, c10);
  const float c1 = lerpf(ay.a, c01, c11);
  return lerpf(az.a, c0, c1);
}

// Per-channel parameters, staged in shared memory at kernel start: lanes index them by
// their own channel, which in the constant bank would serialise on divergent indices.
struct ChanSm {
  const void *vol;
  const float *tfAlpha;
  int X, Y, Z, n;
  float vd0, vd1, xd0, xd1, os;
  float ry1, ry2;   // recip_for_div of the TF remap divisors vd1 - vd0 and xd1 - xd0
};

// The per-cell table (TrackParams::cellTab): a cell's non-zero-majorant channel mask, and
// channel c's (majorant, reciprocal) pair.
__device__ __forceinline__ uint32_t cell_mask(const TrackParams &P, int cellID) {
  return __float_as_uint(__ldg(reinterpret_cast<const float *>(P.cellTab + (size_t)cellID * P.tabStride)));
}
__device__ __forceinline__ float2 cell_maj(const TrackParams &P, int cellID, int c) {
  return __ldg(P.cellTab + (size_t)cellID * P.tabStride + 1 + c);
}

// sampleVolumeTexture (deviceCode.cu:122-132): NaN outside [0,1]^3, else trilinear.
template <int SK>
__device__ __forceinline__ float sample_volume(const TrackParams &P, const ChanSm &cs, float px, float py, float pz) {
  if (px < 0.0f || px > 1.0f || py < 0.0f || py > 1.0f || pz < 0.0f || pz > 1.0f) return __int_as_float(0x7fc00000);
  const Axis ax = axis_in_range(px, cs.X), ay = axis_in_range(py, cs.Y), az = axis_in_range(pz, cs.Z);
  if (P.vol32) return trilinear<SK, uint32_t>(cs.vol, cs.X, cs.Y, ax, ay, az);
  return trilinear<SK, size_t>(cs.vol, cs.X, cs.Y, ax, ay, az);
}

// transferFunction (deviceCode.cu:27-42), alpha part; the lookup axis is returned for
// the colour of a hit.
__device__ __forceinline__ float tf_alpha(const ChanSm &cs, float f, Axis &ax) {
  if (cs.n <= 0) return 0.f;
  if (f < cs.vd0 || f > cs.vd1) return 0.f;
  const float r1 = div_by(f - cs.vd0, cs.vd1 - cs.vd0, cs.ry1);
  const float r2 = div_by(r1 - cs.xd0, cs.xd1 - cs.xd0, cs.ry2);
  ax = axis(r2, cs.n);
  return lerpf(ax.a, __ldg(cs.tfAlpha + ax.i0), __ldg(cs.tfAlpha + ax.i1)) * cs.os;
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
  float rt0, ncb;        // ray_t0, next_cell_begin
  uint32_t visits;
};

__device__ __forceinline__ bool dda_init(const TrackParams &P, float ox, float oy, float oz, float dx, float dy, float dz,
                                         DDA &d) {
  const float fsx = (float)P.mc[0], fsy = (float)P.mc[1], fsz = (float)P.mc[2];
  const float rx = 1.0f / dx, ry = 1.0f / dy, rz = 1.0f / dz;
  const float tlx = (0.0f - ox) * rx, thx = (fsx - ox) * rx;
  const float tly = (0.0f - oy) * ry, thy = (fsy - oy) * ry;
  const float tlz = (0.0f - oz) * rz, thz = (fsz - oz) * rz;
  float nrx = fminf(tlx, thx), nry = fminf(tly, thy), nrz = fminf(tlz, thz);
  const float frx = fmaxf(tlx, thx), fry = fmaxf(tly, thy), frz = fmaxf(tlz, thz);
  const float inf = __int_as_float(0x7f800000);
  if (dx == 0.f) { if (ox < 0.f || ox > fsx) return false; nrx = inf; }   // dda.h:100-101 (t_nr set twice)
  if (dy == 0.f) { if (oy < 0.f || oy > fsy) return false; nry = inf; }
  if (dz == 0.f) { if (oz < 0.f || oz > fsz) return false; nrz = inf; }
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
  d.tnx = (dx == 0.f) ? inf : fabsf(ex - ivx) * d.tsx;
  d.tny = (dy == 0.f) ? inf : fabsf(ey - ivy) * d.tsy;
  d.tnz = (dz == 0.f) ? inf : fabsf(ez - ivz) * d.tsz;
  d.cx = (int)fcx; d.cy = (int)fcy; d.cz = (int)fcz;
  d.rt0 = rt0;
  d.ncb = 0.f;
  d.visits = 0;
  return true;
}

// Advance past the current cell (the step direction per axis is the sign of the ray
// direction, which the world and grid directions share); false when the walk leaves.
__device__ __forceinline__ bool dda_advance(const TrackParams &P, DDA &d, float wdx, float wdy, float wdz,
                                            uint32_t maxCells) {
  const float tc = fminf(fminf(d.tnx, d.tny), d.tnz);
  d.ncb = tc;
  if (d.tnx == tc) {
    d.tnx += d.tsx;
    if (wdx > 0.f) { if (++d.cx == (int)P.mc[0]) return false; } else { if (--d.cx == -1) return false; }
  }
  if (d.tny == tc) {
    d.tny += d.tsy;
    if (wdy > 0.f) { if (++d.cy == (int)P.mc[1]) return false; } else { if (--d.cy == -1) return false; }
  }
  if (d.tnz == tc) {
    d.tnz += d.tsz;
    if (wdz > 0.f) { if (++d.cz == (int)P.mc[2]) return false; } else { if (--d.cz == -1) return false; }
  }
  return d.visits < maxCells;
}

// Normalised grid-space direction of a world direction (deviceCode.cu:773-778).
__device__ __forceinline__ void grid_dir(const TrackParams &P, float wdx, float wdy, float wdz, float &gx, float &gy,
                                         float &gz, float &w2g, float &g2w) {
  gx = P.gScale.x * wdx; gy = P.gScale.y * wdy; gz = P.gScale.z * wdz;
  const float n2 = fmaf(gz, gz, fmaf(gy, gy, gx * gx));
  w2g = sqrtf(n2);
  g2w = 1.f / w2g;
  const float inv = 1.0f / sqrtf(n2);
  gx = gx * inv; gy = gy * inv; gz = gz * inv;
}

// Seeding, jitter and generateRay of one path-sample (deviceCode.cu:293-298, 61-76):
// the normalised world direction; returns the generator state after the jitter draw.
__device__ __forceinline__ uint32_t primary_ray(const TrackParams &P, int px, int py, uint32_t frame, int s, float &wdx,
                                                float &wdy, float &wdz) {
  const uint32_t seed = (uint32_t)P.W * (uint32_t)P.H * (frame + 1u) * (uint32_t)(s + 1);
  uint32_t rng = tea4(((uint32_t)px & P.seedMask) + seed, ((uint32_t)py & P.seedMask) + seed);
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
  return rng;
}

// Frame id and sample of sample j of the launch.
__device__ __forceinline__ uint32_t sample_frame(const TrackParams &P, int j, int &s) {
  if (P.nFrames <= 1) { s = j; return P.frameParam; }
  const int k = j / P.spp;
  s = j - k * P.spp;
  return k == 0 ? P.frameParam : P.frameParam1 + (uint32_t)(k - 1);
}
__device__ __forceinline__ uint32_t frame_accum(const TrackParams &P, int k) {
  return k == 0 ? P.accumParam : P.accumParam1 + (uint32_t)(k - 1);
}

enum : int { S_NEED = 0, S_TRANS = 1, S_STEP = 2, S_SAMPLE = 3, S_DONE = 4 };
enum : int { A_CHAN = 0, A_ADVANCE = 1, A_NEWDDA = 2 };

__device__ __forceinline__ ChanSm chan_params(const TrackParams &P, int c) {
  ChanSm cs;
  cs.vol = P.vol[c];
  cs.tfAlpha = P.tfAlpha[c];
  cs.X = P.dims[c][0]; cs.Y = P.dims[c][1]; cs.Z = P.dims[c][2];
  cs.n = P.tfN[c];
  cs.vd0 = P.vd[c][0]; cs.vd1 = P.vd[c][1];
  cs.xd0 = P.xd[c][0]; cs.xd1 = P.xd[c][1];
  cs.os = P.os[c];
  cs.ry1 = recip_for_div(cs.vd1 - cs.vd0);
  cs.ry2 = recip_for_div(cs.xd1 - cs.xd0);
  return cs;
}

// The warp's tracking loop over work items [qBegin, limit) of one request: with a
// dispenser, the warp takes `chunk` items at a time from it (qBegin = limit = the
// request's item count); without, the warp owns the whole range.  Event counts are
// added to tot[0..4] (samples, rejections, cells, paths, capped).
template <int MODE, int SK, bool STATS, bool SH>
__device__ __forceinline__ void trace_items(const TrackParams &P, const ChanSm *sch, unsigned qBegin, unsigned limit,
                                            unsigned *dispenser, unsigned chunk, uint32_t (&tot)[5]) {
  const int C = P.C;
  const uint32_t maxCells = P.mc[0] + P.mc[1] + P.mc[2] + 3u;
  const unsigned lane = threadIdx.x & 31u;
  const int rw = P.cullX1 - P.cullX0 + 1;
  const size_t nrect = (size_t)rw * (size_t)(P.cullY1 - P.cullY0 + 1);
  uint32_t &totSamp = tot[0], &totRej = tot[1], &totCell = tot[2], &totPaths = tot[3], &totCap = tot[4];

  unsigned qNext = dispenser ? 0u : qBegin, qEnd = dispenser ? 0u : limit;   // the warp's items in hand
  int st = S_NEED, act = A_CHAN;
  size_t recIdx = 0;
  uint32_t pSamp = 0, pRej = 0;                // per-path event counts (STATS)
  uint32_t rng = 0, steps = 0, record = 0;
  float wdx = 1.f, wdy = 1.f, wdz = 1.f, t1w = 0.f, w2g = 0.f, g2w = 0.f;
  DDA d;
  d.visits = 0;
  int ch = 0, cellID = 0;
  uint32_t cmask = 0;                          // non-zero-majorant channels of the current cell
  float maj = 0.f, rmaj = 0.f, t = 0.f, lim = 0.f, ct0 = 0.f, ct1 = 0.f, tW = 0.f;
  float rnd = 0.f;                              // -m 1: the draw taken before a selection
  float pendU = 0.f;                            // the draw of a flight pending in phase 2
  float majs[MODE == 1 ? kMaxChannels : 1], ts[MODE == 1 ? kMaxChannels : 1];   // -m 1 per-channel state
  bool capped = false;
  float tHitW = 0.f;                            // world t of the recorded hit
  // the current leg's world origin: the camera, or the hit point for a shadow ray
  float lox = P.camOrg.x, loy = P.camOrg.y, loz = P.camOrg.z;
  int leg = 0;                                  // 0 primary, 1 shadow ray (SH)
  uint32_t primRec = 0, pxy = 0;
  float primT = 0.f;
  uint32_t pathFrame = 0;                       // frame id of the current path (shadow seed)

  auto enter_cell = [&]() {  // cell_t0 / cell_t1 of the DDA lambda call (dda.h:164-170)
    const float tc = fminf(fminf(d.tnx, d.tny), d.tnz);
    ct0 = d.rt0 + d.ncb;
    ct1 = d.rt0 + fminf(tc, 1e20f);
    d.visits++;
    totCell++;
    cellID = d.cx + d.cy * (int)P.mc[0] + d.cz * (int)P.mc[0] * (int)P.mc[1];
    cmask = cell_mask(P, cellID);
  };
  // Start a tracking leg (volumeIntersection + the tracker's set-up, deviceCode.cu:759-778,
  // 1676-1726) from the leg origin along (dx, dy, dz); false when it misses the volume.
  auto start_leg = [&](float dx, float dy, float dz) -> bool {
    wdx = dx; wdy = dy; wdz = dz;
    const float frx = 1.0f / wdx, fry = 1.0f / wdy, frz = 1.0f / wdz;
    const float ox = SH ? lox : P.camOrg.x, oy = SH ? loy : P.camOrg.y, oz = SH ? loz : P.camOrg.z;
    const float t1 = (P.rootLo.x - ox) * frx, t2 = (P.rootHi.x - ox) * frx;
    const float t3 = (P.rootLo.y - oy) * fry, t4 = (P.rootHi.y - oy) * fry;
    const float t5 = (P.rootLo.z - oz) * frz, t6 = (P.rootHi.z - oz) * frz;
    const float th0 = fmaxf(fmaxf(fminf(t1, t2), fminf(t3, t4)), fminf(t5, t6));
    const float th1 = fminf(fminf(fmaxf(t1, t2), fmaxf(t3, t4)), fmaxf(t5, t6));
    if (th1 < 0 || th0 >= th1) return false;
    t1w = fminf(1e20f, th1);
    float gx, gy, gz;
    grid_dir(P, wdx, wdy, wdz, gx, gy, gz, w2g, g2w);
    ch = 0;
    record = 0;
    steps = 0;
    capped = false;
    st = S_TRANS;
    if (MODE != 0) {
      const float gox = SH ? P.gScale.x * (lox - P.gLo.x) : P.gOrg.x;
      const float goy = SH ? P.gScale.y * (loy - P.gLo.y) : P.gOrg.y;
      const float goz = SH ? P.gScale.z * (loz - P.gLo.z) : P.gOrg.z;
      if (!dda_init(P, gox, goy, goz, gx, gy, gz, d)) return false;
      enter_cell();
      lim = ct1;
      act = A_CHAN;
    } else {
      lim = 1e20f;
      act = A_NEWDDA;
    }
    return true;
  };
  // End of a leg: a primary hit with shadows on continues as the shadow ray
  // (deviceCode.cu:380-397), otherwise the path record is written.
  auto finish = [&]() {
    bool shadowed = false;
    if constexpr (SH) {
      if (P.shadows && leg == 0 && record != 0u && !capped) {
        primRec = record;
        primT = tHitW;
        leg = 1;
        lox = fmaf(tHitW, wdx, P.camOrg.x);
        loy = fmaf(tHitW, wdy, P.camOrg.y);
        loz = fmaf(tHitW, wdz, P.camOrg.z);
        const uint32_t sseed = (uint32_t)P.W * (uint32_t)P.H * pathFrame;
        rng = tea4((pxy & 0xffffu & P.seedMask) + sseed + 1u, ((pxy >> 16) & P.seedMask) + sseed + 1u);
        if (start_leg(-P.lightDir.x, -P.lightDir.y, -P.lightDir.z)) return;
        record = 0u;
        capped = false;
      }
      if (leg == 1) {
        shadowed = record != 0u && !capped;
        if (capped) totCap++;
        record = primRec;
        tHitW = primT;
        capped = false;
      }
    }
    P.records[recIdx] = capped ? 0u : (record | (shadowed ? (1u << 9) : 0u));
    if (SH && P.recT) P.recT[recIdx] = tHitW;
    if (STATS) P.recStats[recIdx] = (pSamp < 0xffffu ? pSamp : 0xffffu) | ((pRej < 0xffffu ? pRej : 0xffffu) << 16);
    totPaths++;
    if (capped) totCap++;
    if constexpr (SH) {
      leg = 0;
      lox = P.camOrg.x; loy = P.camOrg.y; loz = P.camOrg.z;
    }
    st = S_NEED;
  };

  while (true) {
    // ---------------- pooled path start: waiting lanes take consecutive items together
    const unsigned need = __ballot_sync(kFull, st == S_NEED);
    const unsigned busy = __ballot_sync(kFull, st == S_TRANS || st == S_STEP || st == S_SAMPLE);
    if (need == 0u && busy == 0u) break;  // every lane is done
    if (need != 0u && (busy == 0u || __popc(need) >= P.pool)) {
      const unsigned n = __popc(need);
      const unsigned rank = __popc(need & ((1u << lane) - 1u));
      unsigned avail = qEnd - qNext, base = 0;
      if (avail < n) {
        if (lane == 0) base = dispenser ? atomicAdd(dispenser, chunk) : limit;
        base = __shfl_sync(kFull, base, 0);
      }
      unsigned item = rank < avail ? qNext + rank : base + (rank - avail);
      if (avail < n) { qNext = base + (n - avail); qEnd = base + chunk; }
      else qNext += n;
      if (st == S_NEED) {
        if (item >= limit) {
          st = S_DONE;
        } else {
          const unsigned tile = item / (32u * (unsigned)P.sCount);
          const unsigned rem = item - tile * 32u * (unsigned)P.sCount;
          const int k = (int)(rem >> 5), w = (int)(rem & 31u);
          const int lx = (int)(tile % (unsigned)P.tilesX) * 8 + (w & 7);
          const int ly = (int)(tile / (unsigned)P.tilesX) * 4 + (w >> 3);
          const int px = P.cullX0 + lx, py = P.cullY0 + ly;
          if (px <= P.cullX1 && py <= P.cullY1) {
            int s;
            const uint32_t fr = sample_frame(P, P.sBase + k, s);
            if constexpr (SH) pathFrame = fr;
            recIdx = (size_t)k * nrect + (size_t)ly * rw + lx;
            pxy = (uint32_t)px | ((uint32_t)py << 16);
            record = 0;
            capped = false;
            steps = 0;
            tHitW = 0.f;
            pSamp = pRej = 0;
            float dx, dy, dz;
            rng = primary_ray(P, px, py, fr, s, dx, dy, dz);
            if (!start_leg(dx, dy, dz)) finish();
          }
        }
      }
    }

    // ---------------- phase 1: each lane transitions and draws until it holds a
    // tentative collision inside the volume (a pending density sample) or its path ends;
    // a few trips per round, the lanes that are ready wait
    for (int trip = 0; trip < P.trips; trip++) {
      if (!__any_sync(kFull, st == S_TRANS || st == S_STEP)) break;
      // enough lanes hold a pending density sample: sample them together now
      if (trip > 0 && __popc(__ballot_sync(kFull, st == S_SAMPLE)) >= P.quorum) break;
      // transitions: walk channels / cells to the next non-zero majorant
      if (st == S_TRANS) {
        bool stepping = false;
        while (true) {
          if constexpr (MODE == 2) {
            if (act == A_ADVANCE) {
              if (!dda_advance(P, d, wdx, wdy, wdz, maxCells)) break;
              enter_cell();
              lim = ct1;
              ch = 0;
              act = A_CHAN;
            }
            // next channel of this cell with a non-zero majorant (zero ones are skipped
            // without draws, deviceCode.cu:794-797)
            const uint32_t rem = ch < 16 ? (cmask >> ch) : 0u;
            if (rem == 0u) {  // end of the cell: a hit ends the traversal (deviceCode.cu:851-854)
              if (record) break;
              act = A_ADVANCE;
              continue;
            }
            ch += __ffs(rem) - 1;
            const float2 mr = cell_maj(P, cellID, ch);
            maj = mr.x;
            rmaj = mr.y;
            t = ct0;
            stepping = true;
            break;
          } else if constexpr (MODE == 0) {
            if (act == A_NEWDDA) {  // one full traversal per channel (deviceCode.cu:965-969)
              if (ch >= C) break;
              float gx, gy, gz, a, b;
              grid_dir(P, wdx, wdy, wdz, gx, gy, gz, a, b);
              const float gox = SH ? P.gScale.x * (lox - P.gLo.x) : P.gOrg.x;
              const float goy = SH ? P.gScale.y * (loy - P.gLo.y) : P.gOrg.y;
              const float goz = SH ? P.gScale.z * (loz - P.gLo.z) : P.gOrg.z;
              if (!dda_init(P, gox, goy, goz, gx, gy, gz, d)) { ch++; continue; }
              enter_cell();
            } else if (act == A_ADVANCE) {
              if (!dda_advance(P, d, wdx, wdy, wdz, maxCells)) { ch++; act = A_NEWDDA; continue; }
              enter_cell();
            }
            act = A_CHAN;
            if ((cmask >> ch) & 1u) {  // zero-majorant cells are skipped (deviceCode.cu:893-894)
              const float2 mr = cell_maj(P, cellID, ch);
              maj = mr.x;
              rmaj = mr.y;
              t = ct0;
              stepping = true;
              break;
            }
            act = A_ADVANCE;
          } else {  // MODE 1 and 3: one traversal, the cell entered or advanced past
            if (act == A_ADVANCE) {
              if (!dda_advance(P, d, wdx, wdy, wdz, maxCells)) break;
              enter_cell();
              act = A_CHAN;
            }
            if constexpr (MODE >= 3) {  // summed majorant (deviceCode.cu:541-548, 1003-1007)
              if (cmask & 1u) {
                const float2 mr = cell_maj(P, cellID, 0);
                maj = mr.x;
                rmaj = mr.y;
                t = ct0;
                stepping = true;
                break;
              }
              act = A_ADVANCE;
            } else {  // MODE 1: per-channel free flights from the cell entry (deviceCode.cu:652-674)
              float sum = 0.0f;
              for (int i = 0; i < C; i++) {
                majs[i] = cell_maj(P, cellID, i).x;
                sum += majs[i];
                ts[i] = ct0;
              }
              if (sum <= 0.0000001f) { act = A_ADVANCE; continue; }
              for (int i = 0; i < C; i++)
                ts[i] = majs[i] > 0.0f ? mode1_flight(P, ts[i], rng_next(rng), majs[i], w2g) : 1e20f;
              stepping = true;
              break;
            }
          }
        }
        if (stepping) st = S_STEP;
        else finish();
      }
      // free-flight draw (deviceCode.cu:568-583, 677-703, 800-820, 908-930)
      if (st == S_STEP) {
        if (++steps >= kMaxStepsPerSample) {
          capped = true;
          finish();
        } else {
          bool exitCell, skipChannel = false;
          if constexpr (MODE == 1) {
            rnd = rng_next(rng);  // drawn before the selection (deviceCode.cu:681)
            float minT = ts[0];
            int sel = 0;
            for (int i = 1; i < C; i++)
              if (ts[i] < minT && majs[i] > 0.f) { sel = i; minT = ts[i]; }
            ch = sel;
            t = minT;
            exitCell = minT >= ct1;
          } else {
            // A flight that certainly leaves the cell needs no exact length (the next
            // channel or cell starts again from its entry distance).  The others -- the
            // few that end inside the cell -- compute it in phase 2, together, before
            // their density sample.
            pendU = rng_next(rng);
            exitCell = flight_surely_exits(t, pendU, rmaj * (P.dt * w2g * kLn2), MODE == 2 ? lim : ct1);
            if (!exitCell) {
              st = S_SAMPLE;
              continue;
            }
          }
          if (exitCell) {
            if (MODE == 2) { ch++; act = A_CHAN; } else act = A_ADVANCE;
            st = S_TRANS;
          } else if (skipChannel) {
            ch++; act = A_NEWDDA; st = S_TRANS;
          } else {
            tW = t * g2w;
            if (tW >= t1w) {  // world exit
              if (STATS) pRej++;
              totRej++;
              if ((MODE == 2 && ch == C - 1) || MODE == 1 || MODE >= 3) finish();
              else { ch++; act = MODE == 2 ? A_CHAN : A_NEWDDA; st = S_TRANS; }
            } else {
              st = S_SAMPLE;
            }
          }
        }
      }
    }
    __syncwarp();

    // ---------------- phase 2: the pending flights and density samples, together
    if (MODE != 1 && st == S_SAMPLE) {   // the exact flight and its tests (deviceCode.cu:805-821, 915-931)
      t = any_flight(P, t, pendU, maj, rmaj, w2g);
      if (t >= (MODE == 2 ? lim : ct1)) {   // leaves the cell after all
        if (MODE == 2) { ch++; act = A_CHAN; } else act = A_ADVANCE;
        st = S_TRANS;
      } else if (MODE == 0 && lim < t) {    // beyond the closest hit so far: next channel
        ch++; act = A_NEWDDA; st = S_TRANS;
      } else {
        tW = t * g2w;
        if (tW >= t1w) {  // world exit
          if (STATS) pRej++;
          totRej++;
          if ((MODE == 2 && ch == C - 1) || MODE >= 3) finish();
          else { ch++; act = MODE == 2 ? A_CHAN : A_NEWDDA; st = S_TRANS; }
        }
      }
    }
    if (st == S_SAMPLE) {
      const float xs = fmaf(tW, wdx, SH ? lox : P.camOrg.x) * P.w2u.x;
      const float ys = fmaf(tW, wdy, SH ? loy : P.camOrg.y) * P.w2u.y;
      const float zs = fmaf(tW, wdz, SH ? loz : P.camOrg.z) * P.w2u.z;
      st = S_STEP;
      if constexpr (MODE == 4) {  // blended sample, -m 4 and -m 5 (deviceCode.cu:165-241, 1031-1058)
        // both blends have the maximum channel opacity as their opacity; the colour is
        // recomputed from the hit position by the resolve pass
        float w = 0.f;
        if (!(xs < 0.0f || xs > 1.0f || ys < 0.0f || ys > 1.0f || zs < 0.0f || zs > 1.0f)) {
          for (int c = 0; c < C; c++) {
            const ChanSm &cs = sch[c];
            Axis tax;
            const float a = tf_alpha(cs, sample_volume<SK>(P, cs, xs, ys, zs), tax);
            if (a > w) w = a;
          }
        }
        if (STATS) pSamp++;
        totSamp++;
        if (w > 0.0f && rng_next(rng) * maj < w) {   // the draw only when w > 0 (deviceCode.cu:1049)
          record = 0x80000000u;
          if constexpr (SH) tHitW = tW;
          finish();
        } else {
          if (STATS) pRej++;
          totRej++;
        }
      } else if constexpr (MODE == 3) {  // one threshold walked down through the channels (deviceCode.cu:590-613)
        float thr = rng_next(rng) * maj;
        bool hitNow = false;
        for (int c = 0; c < C; c++) {
          const ChanSm &cs = sch[c];
          const float v = sample_volume<SK>(P, cs, xs, ys, zs);
          if (STATS) pSamp++;
          totSamp++;
          if (!(v == v)) continue;
          Axis tax;
          const float a = tf_alpha(cs, v, tax);
          if (a > 0.0f && thr < a) {
            record = make_record(c, tax);
            if constexpr (SH) tHitW = tW;
            hitNow = true;
            break;
          }
          thr -= a;
        }
        if (hitNow) {
          finish();
        } else {
          if (STATS) pRej++;
          totRej++;
        }
      } else {
        const float mj = MODE == 1 ? majs[ch] : maj;
        const float thr = rng_next(rng) * mj;
        const ChanSm &cs = sch[ch];
        const float v = sample_volume<SK>(P, cs, xs, ys, zs);
        if (STATS) pSamp++;
        totSamp++;
        bool rejected = MODE != 0;
        if (v == v) {
          Axis tax;
          const float a = tf_alpha(cs, v, tax);
          if (a > 0.0f && thr < a) {
            record = make_record(ch, tax);
            if constexpr (SH) tHitW = tW;
            if constexpr (MODE == 2) lim = fminf(t, lim);
            if constexpr (MODE == 0) { lim = fminf(t, lim); ch++; act = A_NEWDDA; st = S_TRANS; }
            if constexpr (MODE == 1) finish();
            rejected = MODE == 2;
          } else {
            rejected = true;
          }
        }
        if (rejected) {
          if (STATS) pRej++;
          totRej++;
        }
        if constexpr (MODE == 1) {
          if (st == S_STEP) ts[ch] = mode1_flight(P, ts[ch], rnd, majs[ch], w2g);
        }
      }
    }
    __syncwarp();
  }
}

// counters: warp reduction, one atomic per warp and counter
__device__ __forceinline__ void flush_counters(unsigned long long *counters, const uint32_t (&tot)[5]) {
  unsigned long long v[5] = {tot[0], tot[1], tot[2], tot[3], tot[4]};
#pragma unroll
  for (int k = 0; k < 5; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(kFull, v[k], o);
  }
  if ((threadIdx.x & 31u) == 0) {
#pragma unroll
    for (int k = 0; k < 5; k++)
      if (v[k]) atomicAdd(counters + k, v[k]);
  }
}

// SH: extended variant -- shadow rays (when P.shadows) and the hit distance of every path
// (when P.recT: gradient shading, denoiser features).
template <int MODE, int SK, bool STATS, bool SH>
__global__ void __launch_bounds__(kTPB, kMinBlocks) trace_kernel(const __grid_constant__ TrackParams P) {
  __shared__ ChanSm sch[kMaxChannels];
  if (threadIdx.x < (unsigned)P.C) sch[threadIdx.x] = chan_params(P, threadIdx.x);
  __syncthreads();
  const unsigned total = (unsigned)P.numTiles * 32u * (unsigned)P.sCount;
  uint32_t tot[5] = {0, 0, 0, 0, 0};
  trace_items<MODE, SK, STATS, SH>(P, sch, total, total, P.workCounter, (unsigned)P.chunk, tot);
  flush_counters(P.counters, tot);
}

// ------------------------------------------------------------------ regrouped tracker
// trace_regroup_kernel: the syncDDA (-m 2) and N-DDA (-m 0) trackers, without shadow rays
// or per-pixel statistics, with each warp's paths regrouped by their next operation.  A
// warp keeps 64 path states in shared memory (structure of arrays), twice its lanes.
// Each iteration it counts its slots per stage -- start a path, walk (cell and channel
// transitions with free-flight draws, at most `trips` draws), evaluate a pending density
// sample -- and runs the most populated stage with lane i on the i-th slot of that stage,
// so at least 22 of its 32 lanes work on the same operation.  Warps run independently (no
// block barrier).  Every path runs exactly the arithmetic of trace_items (the same
// helpers, in the same order), so records, hit distances and counters are identical;
// only which lane runs which path when changes.  The loop ends when every slot has run
// out of work items; each path is bounded by kMaxStepsPerSample draws and maxCells cells
// per traversal.
//   -m 2: one traversal; `lim` is min(the cell's exit, the closest hit so far).
//   -m 0: one traversal per channel (deviceCode.cu:965-969); `lim` is the closest hit so
//   far (1e20 before the first), the cell's exit comes from the walk's DDA state.  A
//   channel's traversal is set up by a fourth operation, restart, which the stage count
//   treats as a stage of its own.
namespace rg {
constexpr int kTPB = 256;
constexpr int kSPT = 2;                  // path slots per thread
constexpr int kSlots = kTPB * kSPT;
constexpr int kMinBlocks = 4;            // 64 registers, 32 warps per SM
enum : uint32_t { NEED = 0, WALK = 1, SAMPLE = 2, DONE = 3 };
// meta word: bits 0-1 stage, bit 2 a channel is selected (free flights pending), bit 3
// the cell's channels are exhausted (advance the walk), bits 4-7 channel, bit 8 (-m 0)
// start the next channel's traversal (a WALK slot with it set waits for the restart
// operation), bits 9-20 the cell's non-zero-majorant channels, bits 21-31 cells entered
// by the current traversal
constexpr uint32_t kDraw = 4u, kAdvance = 8u, kNewDda = 256u;
struct Slots {
  uint32_t meta[kSlots], recIdx[kSlots], rng[kSlots], steps[kSlots], record[kSlots], cell[kSlots];
  float wdx[kSlots], wdy[kSlots], wdz[kSlots], t1w[kSlots], w2g[kSlots], g2w[kSlots];
  float tnx[kSlots], tny[kSlots], tnz[kSlots], tsx[kSlots], tsy[kSlots], tsz[kSlots];
  float rt0[kSlots], ncb[kSlots], maj[kSlots], rmaj[kSlots], t[kSlots], lim[kSlots];
};
// MODE of the regrouped loop: 0 (N-DDA) or 2 (syncDDA) at compile time, or -1 to read the
// request's method at run time (the fused batch kernel: one copy of the code for every
// request).  SK likewise: a store kind, or -1 for the request's.
template <int MODE>
__device__ __forceinline__ bool ndda(const TrackParams &P) { return MODE == 0 || (MODE < 0 && P.mode == 0); }
template <int SK>
__device__ __forceinline__ float sample_any(const TrackParams &P, const ChanSm &cs, float x, float y, float z) {
  if constexpr (SK >= 0) return sample_volume<SK>(P, cs, x, y, z);
  else return P.store == kStoreU8 ? sample_volume<kStoreU8>(P, cs, x, y, z) : sample_volume<kStoreF32>(P, cs, x, y, z);
}
// The draw a generator state was left at by its last rng_next: the top 24 bits of the
// state (the sample stage re-reads the walk's pending flight draw this way).
__device__ __forceinline__ float last_draw(uint32_t s) { return (float)(s >> 8) * (1.0f / 16777216.0f); }
__device__ __forceinline__ uint32_t pack_meta(uint32_t stage, uint32_t flags, int ch, uint32_t cmask, uint32_t visits) {
  return stage | flags | ((uint32_t)ch << 4) | ((cmask & 0xfffu) << 9) | (visits << 21);
}
__device__ __forceinline__ void load_dda(const Slots &S, unsigned s, DDA &d) {
  d.tnx = S.tnx[s]; d.tny = S.tny[s]; d.tnz = S.tnz[s];
  d.tsx = S.tsx[s]; d.tsy = S.tsy[s]; d.tsz = S.tsz[s];
  const uint32_t c = S.cell[s];
  d.cx = (int)(c & 1023u); d.cy = (int)((c >> 10) & 1023u); d.cz = (int)(c >> 20);
  d.rt0 = S.rt0[s]; d.ncb = S.ncb[s];
}
__device__ __forceinline__ void store_dda(Slots &S, unsigned s, const DDA &d) {
  S.tnx[s] = d.tnx; S.tny[s] = d.tny; S.tnz[s] = d.tnz;
  S.cell[s] = (uint32_t)d.cx | ((uint32_t)d.cy << 10) | ((uint32_t)d.cz << 20);
  S.ncb[s] = d.ncb;
}
// the exit distance of the DDA's current cell (cell_t1 of dda.h:164-170)
__device__ __forceinline__ float cell_exit(const DDA &d) {
  return d.rt0 + fminf(fminf(fminf(d.tnx, d.tny), d.tnz), 1e20f);
}
// enter_cell of trace_items: the cell's id and channel mask
__device__ __forceinline__ int enter(const TrackParams &P, const DDA &d, uint32_t &cmask) {
  const int cellID = d.cx + d.cy * (int)P.mc[0] + d.cz * (int)P.mc[0] * (int)P.mc[1];
  cmask = cell_mask(P, cellID);
  return cellID;
}
// The index of the DDA cell's first majorant entry in the cell table (its mask entry + 1);
// regroup_fits keeps every table index below 2^32.
__device__ __forceinline__ uint32_t cell_tab(const TrackParams &P, const DDA &d) {
  return ((uint32_t)d.cx + (uint32_t)d.cy * P.mc[0] + (uint32_t)d.cz * P.mc[0] * P.mc[1]) * (uint32_t)P.tabStride + 1u;
}
// enter with the table index: the cell's channel mask, and its first majorant entry
__device__ __forceinline__ uint32_t enter_tab(const TrackParams &P, const DDA &d, uint32_t &cmask) {
  const uint32_t tab = cell_tab(P, d);
  cmask = __float_as_uint(__ldg(reinterpret_cast<const float *>(P.cellTab + (tab - 1u))));
  return tab;
}
// End of a path: its record and, for features and gradient shading, the world distance
// of its hit (0 for a miss); `lim` holds the grid distance of the recorded hit.
__device__ __forceinline__ void finish(const TrackParams &P, Slots &S, unsigned s, uint32_t record, bool capped,
                                       float lim, uint32_t (&tot)[5]) {
  const uint32_t i = S.recIdx[s];
  P.records[i] = capped ? 0u : record;
  if (P.recT) P.recT[i] = record ? lim * S.g2w[s] : 0.f;
  tot[3]++;
  if (capped) tot[4]++;
  S.meta[s] = NEED;
}

// Start the path of work item `item` in slot s (the pooled start of trace_items).
template <int MODE>
__device__ __forceinline__ void start(const TrackParams &P, Slots &S, unsigned s, unsigned item, unsigned limit,
                                      uint32_t (&tot)[5]) {
  if (item >= limit) { S.meta[s] = DONE; return; }
  const int rw = P.cullX1 - P.cullX0 + 1;
  const uint32_t nrect = (uint32_t)rw * (uint32_t)(P.cullY1 - P.cullY0 + 1);
  const unsigned tile = item / (32u * (unsigned)P.sCount);
  const unsigned rem = item - tile * 32u * (unsigned)P.sCount;
  const int k = (int)(rem >> 5), w = (int)(rem & 31u);
  const int lx = (int)(tile % (unsigned)P.tilesX) * 8 + (w & 7);
  const int ly = (int)(tile / (unsigned)P.tilesX) * 4 + (w >> 3);
  const int px = P.cullX0 + lx, py = P.cullY0 + ly;
  if (px > P.cullX1 || py > P.cullY1) return;   // outside the traced rectangle: take another item
  int smp;
  const uint32_t fr = sample_frame(P, P.sBase + k, smp);
  S.recIdx[s] = (uint32_t)k * nrect + (uint32_t)(ly * rw + lx);
  float wdx, wdy, wdz;
  const uint32_t rng = primary_ray(P, px, py, fr, smp, wdx, wdy, wdz);
  // start_leg of trace_items (volumeIntersection, grid transform, DDA start)
  const float frx = 1.0f / wdx, fry = 1.0f / wdy, frz = 1.0f / wdz;
  const float t1 = (P.rootLo.x - P.camOrg.x) * frx, t2 = (P.rootHi.x - P.camOrg.x) * frx;
  const float t3 = (P.rootLo.y - P.camOrg.y) * fry, t4 = (P.rootHi.y - P.camOrg.y) * fry;
  const float t5 = (P.rootLo.z - P.camOrg.z) * frz, t6 = (P.rootHi.z - P.camOrg.z) * frz;
  const float th0 = fmaxf(fmaxf(fminf(t1, t2), fminf(t3, t4)), fminf(t5, t6));
  const float th1 = fminf(fminf(fmaxf(t1, t2), fmaxf(t3, t4)), fmaxf(t5, t6));
  if (th1 < 0 || th0 >= th1) { finish(P, S, s, 0u, false, 0.f, tot); return; }
  float gx, gy, gz, w2g, g2w;
  grid_dir(P, wdx, wdy, wdz, gx, gy, gz, w2g, g2w);
  S.rng[s] = rng; S.steps[s] = 0u; S.record[s] = 0u;
  S.wdx[s] = wdx; S.wdy[s] = wdy; S.wdz[s] = wdz;
  S.t1w[s] = fminf(1e20f, th1); S.w2g[s] = w2g; S.g2w[s] = g2w;
  if (ndda<MODE>(P)) {   // the first channel's traversal starts in the walk
    S.lim[s] = 1e20f;
    S.meta[s] = pack_meta(WALK, kNewDda, 0, 0u, 0u);
    return;
  }
  DDA d;
  if (!dda_init(P, P.gOrg.x, P.gOrg.y, P.gOrg.z, gx, gy, gz, d)) { finish(P, S, s, 0u, false, 0.f, tot); return; }
  uint32_t cmask;
  enter(P, d, cmask);
  tot[2]++;
  store_dda(S, s, d);
  S.tsx[s] = d.tsx; S.tsy[s] = d.tsy; S.tsz[s] = d.tsz;
  S.rt0[s] = d.rt0;
  S.lim[s] = cell_exit(d);
  S.meta[s] = pack_meta(WALK, 0u, 0, cmask, 1u);
}

// Walk: transitions to the next channel (-m 2) or cell (-m 0) with a non-zero majorant,
// then free-flight draws, until a tentative collision (-> SAMPLE), the end of the path,
// or `trips` draws.
template <int MODE>
__device__ __forceinline__ void walk(const TrackParams &P, Slots &S, unsigned s, uint32_t maxCells,
                                     uint32_t (&tot)[5]) {
  const uint32_t m0 = S.meta[s];
  bool drawing = (m0 & kDraw) != 0u, advance = (m0 & kAdvance) != 0u, newdda = (m0 & kNewDda) != 0u;
  int ch = (int)((m0 >> 4) & 15u);
  uint32_t cmask = (m0 >> 9) & 0xfffu, visits = m0 >> 21;
  uint32_t record = S.record[s], rng = S.rng[s];
  // the path's draws so far: a draw that would make them kMaxStepsPerSample ends it as
  // capped, so this walk has kLeft draws before that one; it stops after kStop
  const uint32_t steps0 = S.steps[s];
  const uint32_t kLeft = kMaxStepsPerSample - 1u - steps0;
  const uint32_t kStop = min((uint32_t)P.trips, kLeft);
  float maj = S.maj[s], rmaj = S.rmaj[s], t = S.t[s], lim = S.lim[s];
  const float w2g = S.w2g[s];
  const float kd = P.dt * w2g * kLn2;   // the exit filter's scale, times the majorant's reciprocal
  const float wdx = S.wdx[s], wdy = S.wdy[s], wdz = S.wdz[s];
  DDA d;
  load_dda(S, s, d);
  d.visits = visits;
  uint32_t tab = cell_tab(P, d);   // the current cell's first majorant entry
  bool moved = false;
  uint32_t stage = WALK;
  uint32_t k = 0;   // draws of this walk
  for (;;) {
    if (!drawing) {
      bool ended = false, restartNext = false;
      while (true) {
        if (ndda<MODE>(P)) {
          if (newdda) {   // the next channel's traversal: an operation of its own (restart)
            restartNext = true;
            break;
          } else if (advance) {
            advance = false;
            if (!dda_advance(P, d, wdx, wdy, wdz, maxCells)) { ch++; newdda = true; continue; }
            tab = enter_tab(P, d, cmask);
            d.visits++;
            tot[2]++;
            moved = true;
          }
          if ((cmask >> ch) & 1u) {   // zero-majorant cells are skipped (deviceCode.cu:893-894)
            const float2 mr = __ldg(P.cellTab + (tab + (uint32_t)ch));
            maj = mr.x;
            rmaj = mr.y;
            t = d.rt0 + d.ncb;   // the cell's entry distance
            break;
          }
          advance = true;
        } else {
          if (advance) {
            if (!dda_advance(P, d, wdx, wdy, wdz, maxCells)) { ended = true; break; }
            tab = enter_tab(P, d, cmask);
            d.visits++;
            tot[2]++;
            moved = true;
            lim = cell_exit(d);
            ch = 0;
            advance = false;
          }
          const uint32_t rem = cmask >> ch;   // ch <= C <= 12
          if (rem == 0u) {   // end of the cell: a hit ends the traversal (deviceCode.cu:851-854)
            if (record) { ended = true; break; }
            advance = true;
            continue;
          }
          ch += __ffs(rem) - 1;
          const float2 mr = __ldg(P.cellTab + (tab + (uint32_t)ch));
          maj = mr.x;
          rmaj = mr.y;
          t = d.rt0 + d.ncb;   // the cell's entry distance
          break;
        }
      }
      if (ended) { finish(P, S, s, record, false, lim, tot); return; }
      if (restartNext) break;
      drawing = true;
    }
    // free-flight draw (deviceCode.cu:800-820, 908-930).  A flight that certainly leaves
    // the cell needs no exact length: the next channel or cell starts again from its
    // entry distance.  The others -- the few that end inside the cell -- go to the sample
    // stage, which computes the exact flight, its tests and the density sample together.
    if (k >= kLeft) { finish(P, S, s, record, true, lim, tot); return; }
    const float u = rng_next(rng);
    const float exitAt = ndda<MODE>(P) ? cell_exit(d) : lim;
    if (!flight_surely_exits(t, u, rmaj * kd, exitAt)) {
      stage = SAMPLE;   // the state left at this draw (S.rng) gives it back to the sample stage
      k++;
      break;
    }
    if (ndda<MODE>(P)) advance = true;
    else ch++;
    drawing = false;
    if (++k >= kStop) break;
  }
  S.meta[s] = pack_meta(stage, (drawing ? kDraw : 0u) | (advance ? kAdvance : 0u) | (newdda ? kNewDda : 0u), ch,
                        cmask, d.visits);
  S.steps[s] = steps0 + k; S.rng[s] = rng; S.maj[s] = maj; S.rmaj[s] = rmaj; S.t[s] = t; S.lim[s] = lim;
  if (moved) store_dda(S, s, d);
}

// -m 0: the next channel's traversal (deviceCode.cu:965-969) as an operation of its own,
// run together by the lanes that need one, so that no walk sets a traversal up while its
// other lanes draw.  Every channel's traversal starts from the same grid origin and
// direction, so when the ray misses the grid for one channel it misses it for all and the
// path ends.
template <int MODE>
__device__ __forceinline__ void restart(const TrackParams &P, Slots &S, unsigned s, uint32_t (&tot)[5]) {
  const uint32_t m0 = S.meta[s];
  int ch = (int)((m0 >> 4) & 15u);
  const float wdx = S.wdx[s], wdy = S.wdy[s], wdz = S.wdz[s];
  DDA d;
  for (;; ch++) {
    if (ch >= P.C) { finish(P, S, s, S.record[s], false, S.lim[s], tot); return; }
    float gx, gy, gz, a, b;
    grid_dir(P, wdx, wdy, wdz, gx, gy, gz, a, b);
    if (dda_init(P, P.gOrg.x, P.gOrg.y, P.gOrg.z, gx, gy, gz, d)) break;
  }
  uint32_t cmask;
  enter_tab(P, d, cmask);
  tot[2]++;
  store_dda(S, s, d);
  S.rt0[s] = d.rt0;   // the same for every channel's traversal of the ray
  S.tsx[s] = d.tsx; S.tsy[s] = d.tsy; S.tsz[s] = d.tsz;
  S.meta[s] = pack_meta(WALK, 0u, ch, cmask, 1u);
}

// The pending flight of slot s, then its density sample (phase 2 of trace_items, -m 2
// and -m 0): the exact free flight from the walk's draw and its tests (cell exit, -m 0's
// closest hit, world exit, deviceCode.cu:805-821, 915-931), then the collision test.
template <int MODE, int SK>
__device__ __forceinline__ void sample(const TrackParams &P, Slots &S, const ChanSm *sch, unsigned s,
                                       uint32_t (&tot)[5]) {
  const uint32_t m0 = S.meta[s];
  const int ch = (int)((m0 >> 4) & 15u);
  const float lim = S.lim[s];
  uint32_t rng = S.rng[s];
  const float t = any_flight(P, S.t[s], last_draw(rng), S.maj[s], S.rmaj[s], S.w2g[s]);
  S.t[s] = t;
  float exitAt = lim;
  const bool n0 = ndda<MODE>(P);
  if (n0) {   // the walk's current cell: its exit distance from the DDA state
    DDA d;
    d.tnx = S.tnx[s]; d.tny = S.tny[s]; d.tnz = S.tnz[s]; d.rt0 = S.rt0[s];
    exitAt = cell_exit(d);
  }
  const uint32_t keep = m0 & ~(0xfu | kNewDda);   // channel, cell channels and cells entered
  if (t >= exitAt) {   // leaves the cell after all
    S.meta[s] = n0 ? (keep | WALK | kAdvance) : ((keep & ~0xf0u) | WALK | ((uint32_t)(ch + 1) << 4));
    return;
  }
  if (n0 && lim < t) {   // beyond the closest hit so far: the next channel's traversal
    S.meta[s] = pack_meta(WALK, kNewDda, ch + 1, 0u, 0u);
    return;
  }
  const float tW = t * S.g2w[s];
  if (tW >= S.t1w[s]) {   // world exit
    tot[1]++;
    if (!n0 && ch == P.C - 1) { finish(P, S, s, S.record[s], false, lim, tot); return; }
    S.meta[s] = n0 ? pack_meta(WALK, kNewDda, ch + 1, 0u, 0u) : ((keep & ~0xf0u) | WALK | ((uint32_t)(ch + 1) << 4));
    return;
  }
  const float xs = fmaf(tW, S.wdx[s], P.camOrg.x) * P.w2u.x;
  const float ys = fmaf(tW, S.wdy[s], P.camOrg.y) * P.w2u.y;
  const float zs = fmaf(tW, S.wdz[s], P.camOrg.z) * P.w2u.z;
  const float thr = rng_next(rng) * S.maj[s];
  const ChanSm &cs = sch[ch];
  const float v = sample_any<SK>(P, cs, xs, ys, zs);
  tot[0]++;
  uint32_t next = (m0 & ~3u) | WALK | kDraw;
  if (v == v) {
    Axis tax;
    const float a = tf_alpha(cs, v, tax);
    if (a > 0.0f && thr < a) {
      S.record[s] = make_record(ch, tax);
      S.lim[s] = fminf(t, lim);
      if (n0) {   // the channel's traversal ends at its hit; the next channel's starts
        next = pack_meta(WALK, kNewDda, ch + 1, 0u, 0u);
      }
    } else if (n0) {
      tot[1]++;
    }
  }
  if (!n0) tot[1]++;   // -m 2 counts every sample as a rejection, hits included (deviceCode.cu:836-846)
  S.rng[s] = rng;
  S.meta[s] = next;
}
}  // namespace rg

namespace rg {
// One warp's regrouped tracking loop over the work items [0, limit) of request P, drawn
// from `dispenser`: its 64 slots start empty and the loop ends when each has run out of
// items.  sel is the warp's 32-entry lane table in shared memory.
template <int MODE, int SK>
__device__ __forceinline__ void run_warp(const TrackParams &P, Slots &S, uint16_t *sel, unsigned wbase, unsigned lane,
                                         const ChanSm *sch, unsigned *dispenser, unsigned limit, uint32_t (&tot)[5]) {
  const uint32_t maxCells = P.mc[0] + P.mc[1] + P.mc[2] + 3u;
#pragma unroll
  for (int g = 0; g < kSPT; g++) S.meta[wbase + 32u * g + lane] = NEED;
  __syncwarp();
  while (true) {
    // the warp's slots by stage (two stage bits per slot); the most populated stage runs,
    // lane i on the i-th slot of that stage in slot order
    // (-m 0: walks waiting for their next channel's traversal form a fourth group, kRestart)
    constexpr int kRestart = 3;
    constexpr bool maybeRestart = MODE != 2;   // syncDDA never restarts a traversal
    const bool n0 = maybeRestart && ndda<MODE>(P);
    unsigned ms[kSPT][4];
    int n[4] = {0, 0, 0, 0};
#pragma unroll
    for (int g = 0; g < kSPT; g++) {
      const uint32_t st = S.meta[wbase + 32u * g + lane];
      const unsigned b0 = __ballot_sync(kFull, st & 1u), b1 = __ballot_sync(kFull, st & 2u);
      const unsigned bR = n0 ? __ballot_sync(kFull, st & kNewDda) : 0u;
      ms[g][NEED] = ~b0 & ~b1;
      ms[g][WALK] = b0 & ~b1 & ~bR;
      ms[g][SAMPLE] = ~b0 & b1;
      ms[g][kRestart] = b0 & ~b1 & bR;
#pragma unroll
      for (int X = 0; X < 4; X++) n[X] += __popc(ms[g][X]);
    }
    if (n[0] + n[1] + n[2] + (maybeRestart ? n[3] : 0) == 0) break;   // every slot is out of work items
    int X = SAMPLE, nX = n[SAMPLE];
    if (n[WALK] > nX) { X = WALK; nX = n[WALK]; }
    if (maybeRestart && n[kRestart] > nX) { X = kRestart; nX = n[kRestart]; }
    if (n[NEED] > nX) { X = NEED; nX = n[NEED]; }
    const int nx = nX < 32 ? nX : 32;
    const bool mine = (int)lane < nx;
    // each slot of stage X goes to the lane of its rank (the first 32 in slot order)
    const unsigned lt = (1u << lane) - 1u;
    int below = 0;
#pragma unroll
    for (int g = 0; g < kSPT; g++) {
      const unsigned m = X == SAMPLE ? ms[g][SAMPLE]
                         : (X == WALK ? ms[g][WALK] : ((maybeRestart && X == kRestart) ? ms[g][kRestart] : ms[g][NEED]));
      const int r = below + __popc(m & lt);
      if (((m >> lane) & 1u) && r < 32) sel[r] = (uint16_t)(wbase + 32u * g + lane);
      below += __popc(m);
    }
    __syncwarp();
    const unsigned s = mine ? (unsigned)sel[lane] : 0u;
    if (X == SAMPLE) {
      if (mine) sample<MODE, SK>(P, S, sch, s, tot);
    } else if (X == WALK) {
      if (mine) walk<MODE>(P, S, s, maxCells, tot);
    } else if (maybeRestart && X == kRestart) {
      if (mine) restart<MODE>(P, S, s, tot);
    } else {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(dispenser, (unsigned)nx);
      base = __shfl_sync(kFull, base, 0);
      if (mine) start<MODE>(P, S, s, base + lane, limit, tot);
    }
    __syncwarp();
  }
}
}  // namespace rg

template <int MODE, int SK>
__global__ void __launch_bounds__(rg::kTPB, rg::kMinBlocks) trace_regroup_kernel(const __grid_constant__ TrackParams P) {
  extern __shared__ __align__(16) unsigned char rgSmem[];
  rg::Slots &S = *reinterpret_cast<rg::Slots *>(rgSmem);
  __shared__ ChanSm sch[kMaxChannels];
  __shared__ uint16_t selAll[rg::kTPB];                    // per warp: the slot each lane runs
  const unsigned tid = threadIdx.x, lane = tid & 31u;
  const unsigned wbase = (tid >> 5) * (32u * rg::kSPT);   // the warp's slots: group g is wbase + 32 g + lane
  if (tid < (unsigned)P.C) sch[tid] = chan_params(P, (int)tid);
  __syncthreads();   // the channel table
  uint32_t tot[5] = {0, 0, 0, 0, 0};
  rg::run_warp<MODE, SK>(P, S, selAll + (tid & ~31u), wbase, lane, sch, P.workCounter,
                         (unsigned)P.numTiles * 32u * (unsigned)P.sCount, tot);
  flush_counters(P.counters, tot);
}

// Batched variant of the regrouped tracker: a warp takes the requests in turn, as
// trace_batch_kernel does, and runs the regrouped loop on each with that request's
// dispenser and channel table.
template <int MODE, int SK>
__global__ void __launch_bounds__(rg::kTPB, rg::kMinBlocks)
    trace_batch_regroup_kernel(const TrackParams *__restrict__ reqs, int nReq, unsigned *dispensers) {
  extern __shared__ __align__(16) unsigned char rgSmem[];
  rg::Slots &S = *reinterpret_cast<rg::Slots *>(rgSmem);
  __shared__ ChanSm sch[rg::kTPB / 32][kMaxChannels];
  __shared__ uint16_t selAll[rg::kTPB];
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned gw = blockIdx.x * (rg::kTPB / 32) + warp;
  const unsigned wbase = warp * (32u * rg::kSPT);
  for (int i = 0; i < nReq; i++) {
    const int r = (int)((gw + (unsigned)i) % (unsigned)nReq);
    const TrackParams &P = reqs[r];
    const unsigned total = (unsigned)P.numTiles * 32u * (unsigned)P.sCount;
    unsigned peek = 0;
    if (lane == 0) peek = *(volatile unsigned *)(dispensers + r);
    peek = __shfl_sync(kFull, peek, 0);
    if (peek >= total) continue;   // nothing left of this request
    if (lane < (unsigned)P.C) sch[warp][lane] = chan_params(P, (int)lane);
    __syncwarp();
    uint32_t tot[5] = {0, 0, 0, 0, 0};
    rg::run_warp<MODE, SK>(P, S, selAll + warp * 32u, wbase, lane, sch[warp], dispensers + r, total, tot);
    flush_counters(P.counters, tot);
    __syncwarp();
  }
}
// The regroupable requests of a whole batch in ONE persistent launch, whatever their
// method (-m 0 or -m 2) and voxel format: a warp takes the requests in turn, as
// trace_batch_regroup_kernel does, and runs the regrouped loop of each request's variant,
// so every request shares the launch's single tail.
__global__ void __launch_bounds__(rg::kTPB, rg::kMinBlocks)
    trace_batch_fused_kernel(const TrackParams *__restrict__ reqs, int nReq, unsigned *dispensers) {
  extern __shared__ __align__(16) unsigned char rgSmem[];
  rg::Slots &S = *reinterpret_cast<rg::Slots *>(rgSmem);
  __shared__ ChanSm sch[rg::kTPB / 32][kMaxChannels];
  __shared__ uint16_t selAll[rg::kTPB];
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned gw = blockIdx.x * (rg::kTPB / 32) + warp;
  const unsigned wbase = warp * (32u * rg::kSPT);
  for (int i = 0; i < nReq; i++) {
    const int r = (int)((gw + (unsigned)i) % (unsigned)nReq);
    const TrackParams &P = reqs[r];
    const unsigned total = (unsigned)P.numTiles * 32u * (unsigned)P.sCount;
    unsigned peek = 0;
    if (lane == 0) peek = *(volatile unsigned *)(dispensers + r);
    peek = __shfl_sync(kFull, peek, 0);
    if (peek >= total) continue;   // nothing left of this request
    if (lane < (unsigned)P.C) sch[warp][lane] = chan_params(P, (int)lane);
    __syncwarp();
    uint32_t tot[5] = {0, 0, 0, 0, 0};
    // one copy of the loop for every request: method and voxel format are read at run
    // time, so the kernel's code stays the size of one variant
    rg::run_warp<-1, -1>(P, S, selAll + warp * 32u, wbase, lane, sch[warp], dispensers + r, total, tot);
    flush_counters(P.counters, tot);
    __syncwarp();
  }
}

// Batched variant: many requests (render contexts) in one persistent launch.  Every
// request has its own work dispenser; a warp starts at request (global warp id mod nReq),
// takes chunks of that request's items until they run out, then moves on to the next
// request with items left, so it drains its lanes only when it changes request.  The
// request's channel table is staged per warp in shared memory; the counters go to the
// request.
template <int MODE, int SK, bool STATS, bool SH>
__global__ void __launch_bounds__(kTPB, kMinBlocks)
    trace_batch_kernel(const TrackParams *__restrict__ reqs, int nReq, unsigned *dispensers) {
  __shared__ ChanSm sch[kTPB / 32][kMaxChannels];
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned gw = blockIdx.x * (kTPB / 32) + warp;
  for (int i = 0; i < nReq; i++) {
    const int r = (int)((gw + (unsigned)i) % (unsigned)nReq);
    const TrackParams &P = reqs[r];
    const unsigned total = (unsigned)P.numTiles * 32u * (unsigned)P.sCount;
    unsigned peek = 0;
    if (lane == 0) peek = *(volatile unsigned *)(dispensers + r);
    peek = __shfl_sync(kFull, peek, 0);
    if (peek >= total) continue;   // nothing left of this request
    if (lane < (unsigned)P.C) sch[warp][lane] = chan_params(P, (int)lane);
    __syncwarp();
    uint32_t tot[5] = {0, 0, 0, 0, 0};
    trace_items<MODE, SK, STATS, SH>(P, sch[warp], total, total, dispensers + r, (unsigned)P.chunk, tot);
    flush_counters(P.counters, tot);
    __syncwarp();
  }
}

// Running mean into the accumulation buffer, RGBA8 write (deviceCode.cu:435, 463-471).
// Denoiser input features of a pixel for this frame (16 floats): mean radiance RGB,
// first-collision depth (mean hit distance times featScale, 0 without hits), the
// transmittance estimate (miss fraction), the hit fractions of channels 0..7, the noise
// level 1/sqrt(spp), zeros.
__device__ __forceinline__ void write_features(const TrackParams &P, int px, int py, float r, float g, float b,
                                               uint32_t hits, float sT, uint4 cnt) {
  const float fs = (float)P.spp;
  float4 *o = reinterpret_cast<float4 *>(P.feat) + 4 * ((size_t)px + (size_t)P.W * (size_t)py);
  const float depth = hits ? (sT / (float)hits) * P.featScale : 0.f;
  o[0] = make_float4(r, g, b, depth);
  o[1] = make_float4((float)((uint32_t)P.spp - hits) / fs, (float)(cnt.x & 0xffffu) / fs, (float)(cnt.x >> 16) / fs,
                     (float)(cnt.y & 0xffffu) / fs);
  o[2] = make_float4((float)(cnt.y >> 16) / fs, (float)(cnt.z & 0xffffu) / fs, (float)(cnt.z >> 16) / fs,
                     (float)(cnt.w & 0xffffu) / fs);
  o[3] = make_float4((float)(cnt.w >> 16) / fs, 1.0f / sqrtf(fs), 0.f, 0.f);
}

template <bool STATS>
__device__ __forceinline__ void write_pixel(const TrackParams &P, int px, int py, float o0, float o1, float o2, float o3,
                                            uint4 st, uint32_t accumId) {
  const size_t pix = (size_t)px + (size_t)P.W * (size_t)py;
  if (P.accumulate) {
    float4 *ap = reinterpret_cast<float4 *>(P.accum) + pix;
    const float4 prev = *ap;
    const float k = (float)accumId, k1 = (float)(accumId + 1u);
    o0 = fmaf(k, prev.x, o0) / k1;
    o1 = fmaf(k, prev.y, o1) / k1;
    o2 = fmaf(k, prev.z, o2) / k1;
    o3 = fmaf(k, prev.w, o3) / k1;
    *ap = make_float4(o0, o1, o2, o3);
  }
  const int fx = P.mirror ? (P.W - 1 - px) : px;
  P.fb[(size_t)fx + (size_t)P.W * (size_t)py] = q8(o0) | (q8(o1) << 8) | (q8(o2) << 16) | (q8(o3) << 24);
  if (STATS) reinterpret_cast<uint4 *>(P.stats)[pix] = st;
}

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
  return fmaf(az, bz, fmaf(ay, by, ax * bx));
}
__device__ __forceinline__ void normalize3(float &x, float &y, float &z) {
  const float s = 1.0f / sqrtf(fmaf(z, z, fmaf(y, y, x * x)));
  x = s * x; y = s * y; z = s * z;
}

// transferFunction(sampleVolumeTexture(p, c), c).w (deviceCode.cu:27-42, 122-132) for any
// position, outside positions giving NaN.
template <int SK>
__device__ __forceinline__ float alpha_at(const ChanSm &cs, float x, float y, float z) {
  float v;
  if (x < 0.0f || x > 1.0f || y < 0.0f || y > 1.0f || z < 0.0f || z > 1.0f) {
    v = __int_as_float(0x7fc00000);
  } else {
    const Axis ax = axis(x, cs.X), ay = axis(y, cs.Y), az = axis(z, cs.Z);
    v = trilinear<SK, size_t>(cs.vol, cs.X, cs.Y, ax, ay, az);
  }
  Axis t;
  return tf_alpha(cs, v, t);
}

// Gradient (Blinn-Phong) shading of a hit (deviceCode.cu:327-378, calculateGradient
// deviceCode.cu:243-281): diffuse and specular factors.
template <int SK>
__device__ void gradient_shading(const TrackParams &P, int ch, float tHit, float dx, float dy, float dz, float &diffuse,
                                 float &specular) {
  ChanSm cs;
  cs.vol = P.vol[ch];
  cs.tfAlpha = P.tfAlpha[ch];
  cs.X = P.dims[ch][0]; cs.Y = P.dims[ch][1]; cs.Z = P.dims[ch][2];
  cs.n = P.tfN[ch];
  cs.vd0 = P.vd[ch][0]; cs.vd1 = P.vd[ch][1];
  cs.xd0 = P.xd[ch][0]; cs.xd1 = P.xd[ch][1];
  cs.os = P.os[ch];
  const float tp[3] = {fmaf(tHit, dx, P.camOrg.x) * P.w2u.x, fmaf(tHit, dy, P.camOrg.y) * P.w2u.y,
                       fmaf(tHit, dz, P.camOrg.z) * P.w2u.z};
  const float eps = P.matGradStep[ch];
  float g[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    float p1[3] = {tp[0], tp[1], tp[2]}, p2[3] = {tp[0], tp[1], tp[2]};
    p1[i] -= eps;
    p2[i] += eps;
    float den;
    if (p1[i] < 0.0f) {          // forward difference at the lower boundary
      p1[i] = tp[i];
      p2[i] = tp[i] + eps;
      den = eps;
    } else if (p2[i] > 1.0f) {   // backward difference at the upper boundary
      p1[i] = tp[i] - eps;
      p2[i] = tp[i];
      den = eps;
    } else {
      den = 2.0f * eps;
    }
    const float a1 = alpha_at<SK>(cs, p1[0], p1[1], p1[2]);
    const float a2 = alpha_at<SK>(cs, p2[0], p2[1], p2[2]);
    g[i] = (a2 - a1) / den;
  }
  if (sqrtf(fmaf(g[2], g[2], fmaf(g[1], g[1], g[0] * g[0]))) > 1e-6f) {
    float nx = -g[0], ny = -g[1], nz = -g[2];
    normalize3(nx, ny, nz);
    float lx = P.lightDir.x, ly = P.lightDir.y, lz = P.lightDir.z;
    normalize3(lx, ly, lz);
    float vx = -dx, vy = -dy, vz = -dz;
    normalize3(vx, vy, vz);
    float hx = lx + vx, hy = ly + vy, hz = lz + vz;
    normalize3(hx, hy, hz);
    const float NdotL = fmaxf(dot3(nx, ny, nz, lx, ly, lz), 0.0f);
    const float NdotH = fmaxf(dot3(nx, ny, nz, hx, hy, hz), 0.0f);
    diffuse = P.matDiffuse[ch] * NdotL;
    if (NdotL > 0.0f && NdotH > 0.001f) {
      const float sh = P.matShininess[ch];
      const float normalization = (sh + 8.0f) / (8.0f * 3.14159265f);
      specular = (P.matSpecular[ch] * normalization) * mpow(NdotH, sh);
    } else {
      specular = 0.0f;
    }
  } else {
    diffuse = P.matDiffuse[ch];
    specular = 0.0f;
  }
}

// transferFunction (deviceCode.cu:27-42) with its colour: alpha * opacityScale, rgb;
// (1, 0, 1) and alpha 0 outside the volume domain.
__device__ __forceinline__ float tf_sample(const TrackParams &P, const ChanSm &cs, int c, float f, float &r, float &g,
                                           float &b) {
  r = 1.f; g = 0.f; b = 1.f;
  if (cs.n <= 0 || f < cs.vd0 || f > cs.vd1) return 0.f;
  const float r1 = (f - cs.vd0) / (cs.vd1 - cs.vd0);
  const float r2 = (r1 - cs.xd0) / (cs.xd1 - cs.xd0);
  const Axis ax = axis(r2, cs.n);
  const float *R = P.tfRgba[c];
  r = lerpf(ax.a, __ldg(R + 4 * ax.i0 + 0), __ldg(R + 4 * ax.i1 + 0));
  g = lerpf(ax.a, __ldg(R + 4 * ax.i0 + 1), __ldg(R + 4 * ax.i1 + 1));
  b = lerpf(ax.a, __ldg(R + 4 * ax.i0 + 2), __ldg(R + 4 * ax.i1 + 2));
  return lerpf(ax.a, __ldg(cs.tfAlpha + ax.i0), __ldg(cs.tfAlpha + ax.i1)) * cs.os;
}

// Colour of a blended hit (-m 4 maxOpacityBlend, -m 5 mixBlend; deviceCode.cu:165-200)
// recomputed at the hit: the primary ray of (px, py, sample s), world t = tHit.
template <int SK>
__device__ void blend_colour(const TrackParams &P, int px, int py, uint32_t frame, int s, float tHit, float &r, float &g,
                             float &b) {
  float dx, dy, dz;
  primary_ray(P, px, py, frame, s, dx, dy, dz);
  const float x = fmaf(tHit, dx, P.camOrg.x) * P.w2u.x;
  const float y = fmaf(tHit, dy, P.camOrg.y) * P.w2u.y;
  const float z = fmaf(tHit, dz, P.camOrg.z) * P.w2u.z;
  r = g = b = 0.f;
  if (x < 0.0f || x > 1.0f || y < 0.0f || y > 1.0f || z < 0.0f || z > 1.0f) return;
  if (P.mode == 4) {   // the sample of the most opaque channel
    float best = 0.f;
    for (int c = 0; c < P.C; c++) {
      const ChanSm cs = chan_params(P, c);
      float cr, cg, cb;
      const float a = tf_sample(P, cs, c, sample_volume<SK>(P, cs, x, y, z), cr, cg, cb);
      if (a > best) { best = a; r = cr; g = cg; b = cb; }
    }
  } else {             // opacity-weighted colours over the maximum opacity
    float sr = 0.f, sg = 0.f, sb = 0.f, mo = 0.f;
    for (int c = 0; c < P.C; c++) {
      const ChanSm cs = chan_params(P, c);
      float cr, cg, cb;
      const float a = tf_sample(P, cs, c, sample_volume<SK>(P, cs, x, y, z), cr, cg, cb);
      sr = fmaf(cr, a, sr);
      sg = fmaf(cg, a, sg);
      sb = fmaf(cb, a, sb);
      if (a > mo) mo = a;
    }
    if (mo <= 0.0f) return;
    r = sr / mo; g = sg / mo; b = sb / mo;
  }
}

// One pixel of the resolve pass; returns the path-samples it accounts for without
// tracing (culled pixels).
template <bool STATS, bool SHADE, int SK>
__device__ __forceinline__ uint32_t resolve_pixel(const TrackParams &P, int px, int py) {
  const int rw = P.cullX1 - P.cullX0 + 1;
  const size_t nrect = (size_t)rw * (size_t)(P.cullY1 - P.cullY0 + 1);
  const bool last = P.nFrames > 1 || P.sBase + P.sCount == P.spp;   // multi-frame launches are one batch
  const float kd0 = (1.0f * 1.0f) * P.lightIntensity;   // diffuse * shadow * lightIntensity (unshaded)
  const float ks0 = (0.0f * 1.0f) * P.lightIntensity;   // specular * shadow * lightIntensity
  const bool feat = P.feat != nullptr;   // denoiser features (one batch per frame)
  {
    const int nF = P.nFrames > 1 ? P.nFrames : 1;
    if (px < P.cullX0 || px > P.cullX1 || py < P.cullY0 || py > P.cullY1) {
      if (last) {
        for (int fi = 0; fi < nF; fi++)
          write_pixel<STATS>(P, px, py, P.bgFin[0], P.bgFin[1], P.bgFin[2], P.bgFin[3], make_uint4(0u, 0u, 0u, 0u),
                             frame_accum(P, fi));
        if (feat) write_features(P, px, py, P.bgFin[0], P.bgFin[1], P.bgFin[2], 0u, 0.f, make_uint4(0u, 0u, 0u, 0u));
        return (uint32_t)P.spp * (uint32_t)nF;
      }
      return 0u;
    }
    uint32_t hits = 0;
    uint4 cnt = make_uint4(0u, 0u, 0u, 0u);   // hits of channels 0..7, 16 bits each
    float sT = 0.f;                           // sum of the hits' world t, in sample order
    const size_t q = (size_t)(py - P.cullY0) * rw + (px - P.cullX0);
    float4 f = make_float4(0.f, 0.f, 0.f, 1.f);
    uint4 sv = make_uint4(0u, 0u, 0u, 0u);
    if (P.sBase > 0) {
      f = reinterpret_cast<const float4 *>(P.partial)[q];
      if (STATS) sv = reinterpret_cast<const uint4 *>(P.partialStats)[q];
    }
    // the records of the next samples are loaded ahead (kAhead in flight per thread), so the
    // pass streams them instead of waiting on one load per sample; the sums stay in sample
    // order
    constexpr int kAhead = 4;
    const uint32_t *rec = P.records + q;
    const int nS = P.sCount;
    uint32_t ra[kAhead];
#pragma unroll
    for (int j = 0; j < kAhead; j++) ra[j] = j < nS ? __ldcs(rec + (size_t)j * nrect) : 0u;
    for (int k = 0; k < nS; k++) {
      int s;   // this record's frame and sample
      const uint32_t fr = sample_frame(P, P.sBase + k, s);
      const uint32_t r = ra[0];
#pragma unroll
      for (int j = 0; j + 1 < kAhead; j++) ra[j] = ra[j + 1];
      ra[kAhead - 1] = k + kAhead < nS ? __ldcs(rec + (size_t)(k + kAhead) * nrect) : 0u;
      float cr = 0.f, cg = 0.f, cb = 0.f, ca = 0.f;
      if (r) {
        const int ch = (int)((r >> 27) & 15u);
        float ar, ag, ab;
        if (P.mode >= 4) {
          blend_colour<SK>(P, px, py, fr, s, P.recT[(size_t)k * nrect + q], ar, ag, ab);
        } else {
          const int i0 = (int)((r >> 13) & 0x3fffu);
          const int i1 = ((r >> 12) & 1u) ? i0 : i0 + 1;
          const float a = (float)(r & 0x1ffu) * (1.0f / 256.0f);
          const float *R = P.tfRgba[ch];
          ar = lerpf(a, __ldg(R + 4 * i0 + 0), __ldg(R + 4 * i1 + 0));
          ag = lerpf(a, __ldg(R + 4 * i0 + 1), __ldg(R + 4 * i1 + 1));
          ab = lerpf(a, __ldg(R + 4 * i0 + 2), __ldg(R + 4 * i1 + 2));
        }
        float kd = kd0, ks = ks0;
        if constexpr (SHADE) {
          float diffuse = 1.0f, specular = 0.0f, shadow = 1.0f;
          if (P.gradient && sqrtf(fmaf(ab, ab, fmaf(ag, ag, ar * ar))) > 0.001f) {
            float dx, dy, dz;
            primary_ray(P, px, py, fr, s, dx, dy, dz);
            gradient_shading<SK>(P, ch, P.recT[(size_t)k * nrect + q], dx, dy, dz, diffuse, specular);
          }
          if (P.shadows) shadow = (1.f - P.ambient) * (1.f - (((r >> 9) & 1u) ? 1.0f : 0.0f));
          kd = (diffuse * shadow) * P.lightIntensity;
          ks = (specular * shadow) * P.lightIntensity;
        }
        const F3 sc = P.matSpec[ch];
        const float mr = fmaf(ar, 0.75f, sc.x * 0.25f);
        const float mg = fmaf(ag, 0.75f, sc.y * 0.25f);
        const float mb = fmaf(ab, 0.75f, sc.z * 0.25f);
        cr = fmaf(P.ambient, mr, fmaf(ks, mr, kd * ar));
        cg = fmaf(P.ambient, mg, fmaf(ks, mg, kd * ag));
        cb = fmaf(P.ambient, mb, fmaf(ks, mb, kd * ab));
        ca = 1.0f;
        if (STATS) { sv.z++; sv.w ^= (uint32_t)(ch + 1) << (s & 15); }
        if (feat) {
          hits++;
          sT += P.recT[(size_t)k * nrect + q];
          const uint32_t inc = ch < 8 ? (1u << ((ch & 1) * 16)) : 0u;
          const int w = ch >> 1;
          cnt.x += w == 0 ? inc : 0u;
          cnt.y += w == 1 ? inc : 0u;
          cnt.z += w == 2 ? inc : 0u;
          cnt.w += w == 3 ? inc : 0u;
        }
      }
      if (STATS) {
        const uint32_t e = P.recStats[(size_t)k * nrect + q];
        sv.x += e & 0xffffu;
        sv.y += e >> 16;
      }
      const float oma = 1.0f - ca;
      f.x += fmaf(P.bg.x * 1.0f, oma, cr);
      f.y += fmaf(P.bg.y * 1.0f, oma, cg);
      f.z += fmaf(P.bg.z * 1.0f, oma, cb);
      f.w += fmaf(oma, 1.0f, ca);
      if (nF > 1 && s == P.spp - 1) {   // end of one of the launch's frames
        const float fs = (float)P.spp;
        const int fi = (P.sBase + k) / P.spp;
        write_pixel<STATS>(P, px, py, f.x / fs, f.y / fs, f.z / fs, f.w / fs, sv, frame_accum(P, fi));
        if (feat && fi == nF - 1) write_features(P, px, py, f.x / fs, f.y / fs, f.z / fs, hits, sT, cnt);
        f = make_float4(0.f, 0.f, 0.f, 1.f);
        sv = make_uint4(0u, 0u, 0u, 0u);
        hits = 0;
        cnt = make_uint4(0u, 0u, 0u, 0u);
        sT = 0.f;
      }
    }
    if (nF > 1) {
    } else if (last) {
      const float fs = (float)P.spp;
      write_pixel<STATS>(P, px, py, f.x / fs, f.y / fs, f.z / fs, f.w / fs, sv, P.accumParam);
      if (feat) write_features(P, px, py, f.x / fs, f.y / fs, f.z / fs, hits, sT, cnt);
    } else {
      reinterpret_cast<float4 *>(P.partial)[q] = f;
      if (STATS) reinterpret_cast<uint4 *>(P.partialStats)[q] = sv;
    }
  }
  return 0u;
}

template <bool STATS, bool SHADE, int SK>
__global__ void __launch_bounds__(256) resolve_kernel(const __grid_constant__ TrackParams P) {
  const unsigned npix = (unsigned)P.W * (unsigned)(P.rowHi - P.rowLo);   // the rendered row band
  uint32_t culledPaths = 0;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x)
    culledPaths += resolve_pixel<STATS, SHADE, SK>(P, (int)(i % (unsigned)P.W), P.rowLo + (int)(i / (unsigned)P.W));
  unsigned long long cp = culledPaths;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cp += __shfl_down_sync(kFull, cp, o);
  if ((threadIdx.x & 31) == 0 && cp) atomicAdd(P.counters + 3, cp);
}

// Batched resolve: the pixels of every request of a group, request r owning global
// pixel indices [pixOfs[r], pixOfs[r + 1]).
template <bool STATS, bool SHADE, int SK>
__global__ void __launch_bounds__(256) resolve_batch_kernel(const TrackParams *__restrict__ reqs,
                                                            const unsigned long long *__restrict__ pixOfs, int nReq) {
  const unsigned long long total = pixOfs[nReq];
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < total;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nReq - 1;   // the request owning pixel i
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (pixOfs[mid] <= i) lo = mid; else hi = mid - 1;
    }
    const TrackParams &P = reqs[lo];
    const unsigned j = (unsigned)(i - pixOfs[lo]);
    const uint32_t c = resolve_pixel<STATS, SHADE, SK>(P, (int)(j % (unsigned)P.W), (int)(j / (unsigned)P.W));
    if (c) atomicAdd(P.counters + 3, (unsigned long long)c);
  }
}

template <int SK>
int launch_resolve(const TrackParams &p, cudaStream_t st, int numSMs) {
  const size_t npix = (size_t)p.W * (size_t)(p.rowHi - p.rowLo);
  if (npix == 0) return (int)cudaGetLastError();
  size_t g = (npix + 255) / 256;
  if (g > (size_t)numSMs * 8) g = (size_t)numSMs * 8;
  if (p.shadows || p.gradient) {
    if (p.stats) resolve_kernel<true, true, SK><<<(unsigned)g, 256, 0, st>>>(p);
    else resolve_kernel<false, true, SK><<<(unsigned)g, 256, 0, st>>>(p);
  } else {
    if (p.stats) resolve_kernel<true, false, SK><<<(unsigned)g, 256, 0, st>>>(p);
    else resolve_kernel<false, false, SK><<<(unsigned)g, 256, 0, st>>>(p);
  }
  return (int)cudaGetLastError();
}

// The shared-memory carveout for `blocks` regrouped-tracker blocks per SM, in percent of
// the largest carveout (the rest of the SM's 256 KB is L1 cache); -1 = the default.
template <typename K>
int regroup_carveout(K kernel, int blocks, int smem) {
  if (blocks <= 0) return -1;
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return -1;
  int dev = 0, maxSm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxSm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (maxSm <= 0) return -1;
  const long need = (long)blocks * ((long)smem + (long)fa.sharedSizeBytes + 1024L);   // 1 KB reserved per block
  const int pct = (int)((need * 100 + maxSm - 1) / maxSm);
  return pct > 100 ? 100 : pct;
}

template <int MODE, int SK>
int launch_regroup(const TrackParams &p, cudaStream_t st, int numSMs, int *grid, void *evMid) {
  const int smem = (int)sizeof(rg::Slots);
  cudaError_t e = cudaFuncSetAttribute(trace_regroup_kernel<MODE, SK>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(trace_regroup_kernel<MODE, SK>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           regroup_carveout(trace_regroup_kernel<MODE, SK>, p.rgBlocks, smem));
  if (e != cudaSuccess) return (int)e;
  int bps = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, trace_regroup_kernel<MODE, SK>, rg::kTPB, smem);
  if (e != cudaSuccess) return (int)e;
  if (bps < 1) bps = 1;
  if (p.rgBlocks > 0 && p.rgBlocks < bps) bps = p.rgBlocks;
  *grid = numSMs * bps;
  if (p.numTiles > 0) trace_regroup_kernel<MODE, SK><<<*grid, rg::kTPB, smem, st>>>(p);
  if (evMid) cudaEventRecord((cudaEvent_t)evMid, st);
  e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  return launch_resolve<SK>(p, st, numSMs);
}

template <int MODE, int SK, bool STATS, bool SH>
int launch_t(const TrackParams &p, cudaStream_t st, int numSMs, int *grid, void *evMid) {
  if constexpr ((MODE == 2 || MODE == 0) && !STATS) {
    if (!p.shadows && regroup_fits(p)) return launch_regroup<MODE, SK>(p, st, numSMs, grid, evMid);
  }
  int bps = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, trace_kernel<MODE, SK, STATS, SH>, kTPB, 0);
  if (e != cudaSuccess) return (int)e;
  if (bps < 1) bps = 1;
  *grid = numSMs * bps;
  // dispenser chunk: about 8 chunks per warp, 32..256 items (multiples of a tile)
  TrackParams q = p;
  const size_t items = (size_t)p.numTiles * 32u * (size_t)p.sCount;
  size_t chunk = items / ((size_t)*grid * (kTPB / 32) * 8);
  chunk = chunk < 32 ? 32 : (chunk > 256 ? 256 : chunk & ~(size_t)31);
  q.chunk = (int)chunk;
  if (p.numTiles > 0) trace_kernel<MODE, SK, STATS, SH><<<*grid, kTPB, 0, st>>>(q);
  if (evMid) cudaEventRecord((cudaEvent_t)evMid, st);
  e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  return launch_resolve<SK>(p, st, numSMs);
}

template <int MODE, int SK>
int launch_s(const TrackParams &p, cudaStream_t st, int numSMs, int *grid, void *evMid) {
  if (p.shadows || p.recT) return p.stats ? launch_t<MODE, SK, true, true>(p, st, numSMs, grid, evMid) : launch_t<MODE, SK, false, true>(p, st, numSMs, grid, evMid);
  return p.stats ? launch_t<MODE, SK, true, false>(p, st, numSMs, grid, evMid) : launch_t<MODE, SK, false, false>(p, st, numSMs, grid, evMid);
}

template <int MODE, int SK, bool STATS, bool SH>
int launch_tb(const BatchGroup &g, cudaStream_t st, int numSMs, int *grid) {
  int bps = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, trace_batch_kernel<MODE, SK, STATS, SH>, kTPB, 0);
  if (e != cudaSuccess) return (int)e;
  if (bps < 1) bps = 1;
  *grid = numSMs * bps;
  if (g.totalItems > 0) trace_batch_kernel<MODE, SK, STATS, SH><<<*grid, kTPB, 0, st>>>(g.reqs, g.nReq, g.dispensers);
  e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  size_t rg = (size_t)((g.totalPix + 255) / 256);
  if (rg > (size_t)numSMs * 8) rg = (size_t)numSMs * 8;
  if (rg == 0) return (int)cudaSuccess;
  if (g.shade) resolve_batch_kernel<STATS, true, SK><<<(unsigned)rg, 256, 0, st>>>(g.reqs, g.pixOfs, g.nReq);
  else resolve_batch_kernel<STATS, false, SK><<<(unsigned)rg, 256, 0, st>>>(g.reqs, g.pixOfs, g.nReq);
  return (int)cudaGetLastError();
}

template <int MODE, int SK>
int launch_tb_regroup(const BatchGroup &g, cudaStream_t st, int numSMs, int *grid) {
  const int smem = (int)sizeof(rg::Slots);
  cudaError_t e = cudaFuncSetAttribute(trace_batch_regroup_kernel<MODE, SK>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return (int)e;
  int bps = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, trace_batch_regroup_kernel<MODE, SK>, rg::kTPB, smem);
  if (e != cudaSuccess) return (int)e;
  if (bps < 1) bps = 1;
  *grid = numSMs * bps;
  if (g.totalItems > 0) trace_batch_regroup_kernel<MODE, SK><<<*grid, rg::kTPB, smem, st>>>(g.reqs, g.nReq, g.dispensers);
  e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  size_t rg = (size_t)((g.totalPix + 255) / 256);
  if (rg > (size_t)numSMs * 8) rg = (size_t)numSMs * 8;
  if (rg == 0) return (int)cudaSuccess;
  resolve_batch_kernel<false, false, SK><<<(unsigned)rg, 256, 0, st>>>(g.reqs, g.pixOfs, g.nReq);
  return (int)cudaGetLastError();
}

template <int MODE, int SK>
int launch_tbs(const BatchGroup &g, cudaStream_t st, int numSMs, int *grid) {
  if constexpr (MODE == 2 || MODE == 0) {
    if (g.regroup && !g.stats && !g.ext) return launch_tb_regroup<MODE, SK>(g, st, numSMs, grid);
  }
  if (g.ext) return g.stats ? launch_tb<MODE, SK, true, true>(g, st, numSMs, grid) : launch_tb<MODE, SK, false, true>(g, st, numSMs, grid);
  return g.stats ? launch_tb<MODE, SK, true, false>(g, st, numSMs, grid) : launch_tb<MODE, SK, false, false>(g, st, numSMs, grid);
}

template <int MODE, int SK>
int occ_tbs(bool stats, bool ext) {
  int bps = 0;
  cudaError_t e;
  if (ext) e = stats ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, trace_batch_kernel<MODE, SK, true, true>, kTPB, 0)
                     : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, trace_batch_kernel<MODE, SK, false, true>, kTPB, 0);
  else e = stats ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, trace_batch_kernel<MODE, SK, true, false>, kTPB, 0)
                 : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, trace_batch_kernel<MODE, SK, false, false>, kTPB, 0);
  return (e == cudaSuccess && bps > 0) ? bps : 1;
}

}  // namespace

int launch_track_batch_fused(const TrackParams *reqs, int nReq, unsigned *dispensers, unsigned long long totalItems,
                             const unsigned long long *pixOfs, unsigned long long totalPix, void *stream, int numSMs,
                             int *launches, int *grid) {
  cudaStream_t st = (cudaStream_t)stream;
  const int smem = (int)sizeof(rg::Slots);
  cudaError_t e = cudaFuncSetAttribute(trace_batch_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return (int)e;
  int bps = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, trace_batch_fused_kernel, rg::kTPB, smem);
  if (e != cudaSuccess) return (int)e;
  if (bps < 1) bps = 1;
  *grid = numSMs * bps;
  if (totalItems > 0) trace_batch_fused_kernel<<<*grid, rg::kTPB, smem, st>>>(reqs, nReq, dispensers);
  e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  size_t g = (size_t)((totalPix + 255) / 256);
  if (g > (size_t)numSMs * 8) g = (size_t)numSMs * 8;
  // the resolve pass of -m 0 / -m 2 without shading extras reads no voxels: one variant
  // serves every voxel format
  if (g > 0) resolve_batch_kernel<false, false, kStoreF32><<<(unsigned)g, 256, 0, st>>>(reqs, pixOfs, nReq);
  if (launches) *launches += (totalItems > 0 ? 1 : 0) + (g > 0 ? 1 : 0);
  return (int)cudaGetLastError();
}

// The regrouped tracker's packed slot fields: cells < 1024 per axis, at most 2047 cells
// entered, 32-bit record indices.
bool regroup_fits(const TrackParams &p) {
  const size_t nrect = (size_t)(p.cullX1 - p.cullX0 + 1) * (size_t)(p.cullY1 - p.cullY0 + 1);
  return (p.mode == 2 || p.mode == 0) && p.regroup && p.mc[0] <= 1024u && p.mc[1] <= 1024u && p.mc[2] <= 1024u &&
         p.mc[0] + p.mc[1] + p.mc[2] + 3u <= 2047u && nrect * (size_t)p.sCount < ((size_t)1 << 32) &&
         (size_t)p.mc[0] * p.mc[1] * p.mc[2] * (size_t)p.tabStride < ((size_t)1 << 32);
}

int batch_trace_occupancy(int mode, int storeKind, bool stats, bool ext) {
  const bool u8 = storeKind == kStoreU8;
  switch (mode) {
    case 0: return u8 ? occ_tbs<0, kStoreU8>(stats, ext) : occ_tbs<0, kStoreF32>(stats, ext);
    case 1: return u8 ? occ_tbs<1, kStoreU8>(stats, ext) : occ_tbs<1, kStoreF32>(stats, ext);
    case 2: return u8 ? occ_tbs<2, kStoreU8>(stats, ext) : occ_tbs<2, kStoreF32>(stats, ext);
    case 3: return u8 ? occ_tbs<3, kStoreU8>(stats, ext) : occ_tbs<3, kStoreF32>(stats, ext);
    default: return u8 ? occ_tbs<4, kStoreU8>(stats, ext) : occ_tbs<4, kStoreF32>(stats, ext);
  }
}

// One group of a batch: every request with the same kernel variant, in one persistent
// trace launch and one resolve launch.
int launch_track_batch(const BatchGroup &g, void *stream, int numSMs, int *launches, int *grid) {
  cudaStream_t st = (cudaStream_t)stream;
  const bool u8 = g.storeKind == kStoreU8;
  int rc;
  switch (g.mode) {
    case 0: rc = u8 ? launch_tbs<0, kStoreU8>(g, st, numSMs, grid) : launch_tbs<0, kStoreF32>(g, st, numSMs, grid); break;
    case 1: rc = u8 ? launch_tbs<1, kStoreU8>(g, st, numSMs, grid) : launch_tbs<1, kStoreF32>(g, st, numSMs, grid); break;
    case 2: rc = u8 ? launch_tbs<2, kStoreU8>(g, st, numSMs, grid) : launch_tbs<2, kStoreF32>(g, st, numSMs, grid); break;
    case 3: rc = u8 ? launch_tbs<3, kStoreU8>(g, st, numSMs, grid) : launch_tbs<3, kStoreF32>(g, st, numSMs, grid); break;
    case 4:
    case 5: rc = u8 ? launch_tbs<4, kStoreU8>(g, st, numSMs, grid) : launch_tbs<4, kStoreF32>(g, st, numSMs, grid); break;
    default: return (int)cudaErrorInvalidValue;
  }
  if (launches) *launches += (g.totalItems > 0 ? 1 : 0) + (g.totalPix > 0 ? 1 : 0);
  return rc;
}

// One batch of samples [sBase, sBase + sCount): trace + resolve on `stream`.
int launch_track(const TrackParams &p, int storeKind, void *stream, int numSMs, int *launches, int *grid, int *block,
                 void *evMid) {
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  const bool u8 = storeKind == kStoreU8;
  switch (p.mode) {
    case 0: rc = u8 ? launch_s<0, kStoreU8>(p, st, numSMs, grid, evMid) : launch_s<0, kStoreF32>(p, st, numSMs, grid, evMid); break;
    case 1: rc = u8 ? launch_s<1, kStoreU8>(p, st, numSMs, grid, evMid) : launch_s<1, kStoreF32>(p, st, numSMs, grid, evMid); break;
    case 2: rc = u8 ? launch_s<2, kStoreU8>(p, st, numSMs, grid, evMid) : launch_s<2, kStoreF32>(p, st, numSMs, grid, evMid); break;
    case 3: rc = u8 ? launch_s<3, kStoreU8>(p, st, numSMs, grid, evMid) : launch_s<3, kStoreF32>(p, st, numSMs, grid, evMid); break;
    case 4:
    case 5: rc = u8 ? launch_s<4, kStoreU8>(p, st, numSMs, grid, evMid) : launch_s<4, kStoreF32>(p, st, numSMs, grid, evMid); break;
    default: return (int)cudaErrorInvalidValue;
  }
  *block = (regroup_fits(p) && !p.stats && !p.shadows) ? rg::kTPB : kTPB;
  if (launches) *launches += p.numTiles > 0 ? 2 : 1;
  return rc;
}

}  // namespace mdwt

// ------------------------------------------------------------------ exit-filter premise
namespace mdwt {
namespace {
// The largest |lg2.approx(x) - log2(x)| / (1 + |log2 x|) over every argument a free
// flight takes, x = 1 - k 2^-24 for k < 2^24, against the double-precision log2.
__global__ void flight_log2_bound_kernel(unsigned *worst) {
  float w = 0.f;
  for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < (1u << 24); k += gridDim.x * blockDim.x) {
    const float x = 1.0f - (float)k * (1.0f / 16777216.0f);
    const double e = log2((double)x);
    const double g = (double)__log2f(x);
    w = fmaxf(w, (float)(fabs(g - e) / (1.0 + fabs(e))));
  }
  for (int o = 16; o > 0; o >>= 1) w = fmaxf(w, __shfl_xor_sync(kFull, w, o));
  if ((threadIdx.x & 31u) == 0) atomicMax(worst, __float_as_uint(w));   // w >= 0: bit order is value order
}
}  // namespace
}  // namespace mdwt

// Checks the premise of the trackers' free-flight exit filter on this device: writes the
// largest relative error of the hardware log2 over the 2^24 flight arguments.
extern "C" mdwt_status mdwt_check_flight_filter(float *worst_out) {
  if (!worst_out) return MDWT_ERR_BAD_ARG;
  unsigned *d = nullptr;
  if (cudaMalloc(&d, sizeof(unsigned)) != cudaSuccess) { cudaGetLastError(); return MDWT_ERR_CUDA; }
  unsigned h = 0;
  cudaError_t e = cudaMemset(d, 0, sizeof(unsigned));
  if (e == cudaSuccess) {
    mdwt::flight_log2_bound_kernel<<<1184, 256>>>(d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(unsigned), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return MDWT_ERR_CUDA;
  std::memcpy(worst_out, &h, sizeof(float));
  return MDWT_OK;
}
