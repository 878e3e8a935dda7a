// mdwt_oracle.cpp -- CPU oracle of the multi-density Woodcock tracker.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the B200 library
// (mdwtracker_b200/csrc); only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg may load it.  It is never part of the product path.
//
// What it is: a straightforward OpenMP C++17 restatement of the reference
// renderer's raw-volume path (alpers-git/MDWTracker), written in the structure of
// the reference (nested per-sample loops, a per-voxel scatter for the macrocell
// value ranges) so that it can be read side by side with it:
//   raw load        rawFile.cpp:31-128
//   TF upload       renderer.cpp:1094-1165 (alpha^3)
//   TF lookup       deviceCode.cu:27-42
//   volume fetch    deviceCode.cu:91-132 (tex3D, normalized, linear, clamp)
//   range raster    renderer.cu:330-347, 387-403, 487-519, 835-893, 1116-1179
//   majorants       renderer.cu:111-157 (sum), 159-203 (per channel), 206-274
//   3D-DDA          dda.h:81-202
//   trackers        deviceCode.cu:513-617 (-m 3), 619-745 (-m 1), 747-856 (-m 2), 858-970 (-m 0)
//   raygen          deviceCode.cu:44-76, 283-471; root box deviceCode.cu:1676-1726
//   camera          camera.h:83-125, renderer.cpp:1058-1092
//   dt / mc dims    renderer.cpp:1317-1361, 1363-1466
//
// PARITY PARTLY PINNED: the reference renderer cannot be built here (OptiX SDK and the
// OWL, GLFW, ImGui, argparse and umesh submodules are absent) and it ships no tests or
// golden vectors.  Two parts compile on their own and pin this restatement bit for bit
// (tests/test_ref_pins.py): the 3-D DDA (dda.h) and the raw loader (rawFile.cpp), built
// where they lie with a stand-in for OWL's vector types (oracle/ref_shim, `make ref`).
// The rest is pinned by analytic known-answer tests (tests/test_oracle_known_answers.py):
// empty volume -> background, constant slab -> Beer-Lambert transmittance, hand-checked
// majorants, zero-alpha TF -> zero majorant.
//
// Arithmetic specification shared with the CUDA kernels (both sides implement it
// independently; bit-identical results are the parity bar):
//  * IEEE-754 binary32, round to nearest, no contraction: a*b+c is fused only where
//    written as fmaf(), which is where the reference's expression has the a*b+c form
//    that nvcc contracts by default (the reference builds without fast-math).
//  * Texture filtering is done in software: coordinate x = fmaf(u, N, -0.5),
//    i = floor(x), weight a = rint((x-i)*256)/256 (the 8-bit fractional weight of
//    the CUDA texture unit, CUDA C Programming Guide "Linear Filtering"), clamp
//    addressing, lerp(a,p,q) = fmaf(a, q, (1-a)*p), x first, then y, then z.
//  * RNG: the reference uses owl::common::LCG<4> (OWL submodule, not vendored).  The
//    project restates the published method it is built from: a 4-round TEA hash
//    (Wheeler & Needham 1994, delta 0x9E3779B9) of the two seed words, key =
//    the first four SHA-256 initial hash words (FIPS 180-4), feeding a 32-bit LCG
//    with the Numerical Recipes constants (1664525, 1013904223); a draw is the top
//    24 bits of the state times 2^-24.
//  * log: the project's own, from log(m) = 2 atanh((m-1)/(m+1)) on m in
//    (sqrt(1/2), sqrt(2)] (Taylor series to s^9) plus e*ln2 (ln2 split hi/lo).
//  * float->int is truncation with saturation and NaN -> 0 (the GPU cvt.rzi rule).
//  * DDA walks at most X+Y+Z+3 cells and a sample takes at most kMaxSteps Woodcock
//    steps; a sample that reaches the cap counts as a miss and is reported.  Neither
//    bound is reached by finite inputs (the reference would loop forever on NaN).

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <sstream>
#include <algorithm>
#include <limits>
#include <omp.h>

namespace orc {

static const int kMaxChannels = 12;
static const uint32_t kMaxSteps = 1u << 22;

// ---------------------------------------------------------------- small math
struct V3 { float x, y, z; };
static inline V3 v3(float x, float y, float z) { return {x, y, z}; }
static inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 mul(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
static inline V3 muls(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline V3 neg(V3 a) { return {-a.x, -a.y, -a.z}; }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// host-side normalize (camera): v * (1/sqrt(dot))
static inline V3 normalize_h(V3 v) { float s = 1.0f / std::sqrt(dot(v, v)); return muls(s, v); }
// device-side squared length with the nvcc contraction of x*x+y*y+z*z
static inline float len2_d(V3 v) { return std::fma(v.z, v.z, std::fma(v.y, v.y, v.x * v.x)); }

static inline int f2i(float x) {
  if (!(x == x)) return 0;
  if (x >= 2147483648.0f) return 2147483647;
  if (x <= -2147483648.0f) return (-2147483647 - 1);
  return (int)x;
}
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------- RNG (S1)
struct Rng {
  uint32_t state;
  void init(uint32_t v0, uint32_t v1) {
    const uint32_t k0 = 0x6a09e667u, k1 = 0xbb67ae85u, k2 = 0x3c6ef372u, k3 = 0xa54ff53au;
    uint32_t sum = 0;
    for (int n = 0; n < 4; n++) {
      sum += 0x9E3779B9u;
      v0 += ((v1 << 4) + k0) ^ (v1 + sum) ^ ((v1 >> 5) + k1);
      v1 += ((v0 << 4) + k2) ^ (v0 + sum) ^ ((v0 >> 5) + k3);
    }
    state = v0;
  }
  float next() {
    state = 1664525u * state + 1013904223u;
    return (float)(state >> 8) * (1.0f / 16777216.0f);
  }
};

// ---------------------------------------------------------------- log (S2)
static inline float mlog(float x) {
  uint32_t b; std::memcpy(&b, &x, 4);
  int e = (int)((b >> 23) & 0xff) - 127;
  uint32_t mb = (b & 0x007fffffu) | 0x3f800000u;
  float m; std::memcpy(&m, &mb, 4);
  if (m > 1.41421353816986083984375f) { m = m * 0.5f; e = e + 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float z = s * s;
  float p = std::fma(z, 1.0f / 9.0f, 1.0f / 7.0f);
  p = std::fma(z, p, 1.0f / 5.0f);
  p = std::fma(z, p, 1.0f / 3.0f);
  float s2 = s + s;
  float r = std::fma(s2 * z, p, s2);
  float fe = (float)e;
  return std::fma(fe, 0.693145751953125f, std::fma(fe, 1.428606765330187e-06f, r));
}

// exp(z): z = k*ln2 + r (Cody-Waite, ln2 split hi/lo), |r| <= ln2/2, degree-7 Taylor
// polynomial of e^r, times 2^k built in the exponent field; 0 below 2^-126.
static inline float mexp(float z) {
  if (!(z == z)) return z;
  if (z > 88.0f) return INFINITY;
  if (z < -87.0f) return 0.0f;
  const float kf = std::rint(z * 1.44269502162933349609375f);
  float r = std::fma(-kf, 0.693145751953125f, z);
  r = std::fma(-kf, 1.428606765330187e-06f, r);
  float p = std::fma(r, 1.0f / 5040.0f, 1.0f / 720.0f);
  p = std::fma(r, p, 1.0f / 120.0f);
  p = std::fma(r, p, 1.0f / 24.0f);
  p = std::fma(r, p, 1.0f / 6.0f);
  p = std::fma(r, p, 0.5f);
  p = std::fma(r, p, 1.0f);
  p = std::fma(r, p, 1.0f);
  const int k = (int)kf;
  if (k < -126) return 0.0f;
  uint32_t sb = (uint32_t)(k + 127) << 23;
  float scale; std::memcpy(&scale, &sb, 4);
  return p * scale;
}
// pow(x, y) for x > 0: exp(y * log(x)); pow(0, y > 0) = 0.
static inline float mpow(float x, float y) {
  if (x == 0.0f) return 0.0f;
  return mexp(y * mlog(x));
}

// ---------------------------------------------------------------- filtering (S4-S6)
static inline float quant(float a) { return std::rint(a * 256.0f) * (1.0f / 256.0f); }
static inline float lerpf(float a, float p, float q) { return std::fma(a, q, (1.0f - a) * p); }

struct Axis { int i0, i1; float a; };
static inline Axis axis(float u, int n) {
  float x = std::fma(u, (float)n, -0.5f);
  float fl = std::floor(x);
  Axis r;
  r.a = quant(x - fl);
  int i = f2i(fl);
  r.i0 = clampi(i, 0, n - 1);
  r.i1 = clampi(i, -1, n - 2) + 1;
  return r;
}

// ---------------------------------------------------------------- scene state
struct Channel {
  int64_t dims[3];
  std::vector<float> data;     // converted to float exactly like RawR (rawFile.cpp:98-121)
  std::vector<uint8_t> bytes;  // uint8 channels: the bytes, value = byte * 255 (exact in float)
  float lo[4], hi[4];          // box4f bounds_ = {{0,0,0,0},{1,1,1,1}} (rawFile.h:162)
  float at(size_t i) const { return bytes.empty() ? data[i] : (float)bytes[i] * 255; }
};

struct TFData {
  std::vector<float> rgba;   // alpha already cubed
  int n = 0;
  float vd[2] = {0, 1};
  float xd[2] = {0, 1};
  float os = 1.0f;
};

struct Material {
  float diffuse = 0.8f, specular = 0.3f, shininess = 8.0f, gradStep = 0.01f;
  V3 spec = {1, 1, 1};
};

struct Camera {  // camera.h:46-142
  V3 vx = {1, 0, 0}, vy = {0, 1, 0}, vz = {0, 0, 1};
  V3 position = {0, -1, 0};
  V3 upVector = {0, 1, 0};
  float poiDistance = 1.f, focalDistance = 1.f;
  float fovy = 60.f;
  void forceUpFrame() {
    if (std::fabs(dot(vz, upVector)) < 1e-6f) return;
    vx = normalize_h(cross(upVector, vz));
    vy = normalize_h(cross(vz, vx));
  }
  void setOrientation(V3 origin, V3 interest, V3 up, float fovyDeg) {
    fovy = fovyDeg;
    position = origin;
    upVector = up;
    bool same = interest.x == origin.x && interest.y == origin.y && interest.z == origin.z;
    vz = same ? v3(0, 0, 1) : neg(normalize_h(sub(interest, origin)));
    vx = cross(up, vz);
    if (dot(vx, vx) < 1e-8f) vx = v3(0, 1, 0); else vx = normalize_h(vx);
    vy = normalize_h(cross(vz, vx));
    poiDistance = std::sqrt(dot(sub(interest, origin), sub(interest, origin)));
    focalDistance = poiDistance;
    forceUpFrame();
  }
};

struct Oracle {
  std::vector<Channel> ch;
  uint32_t mcReq[3] = {0, 0, 0};
  uint32_t mc[3] = {0, 0, 0};
  int mode = 0;
  bool inited = false;
  std::vector<float> ranges;     // float2 per (cell, channel)
  std::vector<float> majorants;
  std::vector<TFData> tf;
  std::vector<Material> mats;
  float dt = 0.05f;
  int W = 1024, H = 1024;
  int spp = 1;
  bool accum = true;
  V3 bg = {0, 0, 0};
  bool shadows = false, gradient = false;
  V3 lightDir = {0.0001f, -1.f, 0.0001f};
  float lightIntensity = 1.0f, ambient = 0.1f;
  bool mirror = false;
  uint32_t seedMask = 0xffffffffu;   // orc_set_seed_block
  Camera cam;
  V3 cOrg{}, cLlc{}, cHor{}, cVer{};
  int frameID = 0, accumID = 0, frameParam = 0, accumParam = 0;
  std::vector<float> accumBuf;
  std::vector<uint32_t> fb;
  bool statsOn = false;
  std::vector<uint32_t> stats;
  bool featOn = false;
  std::vector<float> feat;       // 16 per pixel
  float featScale = 1.0f;
  uint64_t counters[4] = {0, 0, 0, 0};
  uint64_t capped = 0;
  float rootLo[3], rootHi[3];    // union of channel bounds (renderer.cpp:698-716)
  float gLo[4], gHi[4];          // bounds of the LAST channel (renderer.cpp:748-754)
  std::string err;
};

// ---------------------------------------------------------------- raw loader (L)
static bool parse_raw_name(const std::string &path, int64_t dims[3], int &fmt) {
  // rawFile.cpp:36-84: split on '_', drop from the first '.', "%dx%dx%d" gives dims,
  // a type token sets the format, any other token resets it to Unspecified.
  dims[0] = dims[1] = dims[2] = 0;
  fmt = 4;  // DataFormat::UInt8 default (rawFile.h:164)
  std::istringstream st(path);
  std::string tok;
  while (std::getline(st, tok, '_')) {
    size_t dp = tok.find('.');
    if (dp != std::string::npos) tok = tok.substr(0, dp);
    int x = 0, y = 0, z = 0;
    if (std::sscanf(tok.c_str(), "%dx%dx%d", &x, &y, &z) == 3) {
      dims[0] = x; dims[1] = y; dims[2] = z;
      continue;
    }
    if (tok == "int8") fmt = 1;
    else if (tok == "int16") fmt = 2;
    else if (tok == "int32") fmt = 3;
    else if (tok == "uint8") fmt = 4;
    else if (tok == "uint16") fmt = 5;
    else if (tok == "uint32") fmt = 6;
    else if (tok == "float32") fmt = 7;
    else if (tok == "double64") fmt = 8;
    else fmt = 0;
  }
  return dims[0] > 0 && dims[1] > 0 && dims[2] > 0;
}

static int fmt_bytes(int f) {
  switch (f) { case 1: case 4: return 1; case 2: case 5: return 2; case 3: case 6: case 7: return 4; case 8: return 8; }
  return 0;
}

static void convert(Channel &c, const void *buf, int fmt, size_t n) {
  c.lo[0] = c.lo[1] = c.lo[2] = c.lo[3] = 0.f;
  c.hi[0] = c.hi[1] = c.hi[2] = c.hi[3] = 1.f;
  if (fmt == 4) {  // uint8 kept as bytes (a quarter of the memory); the values are the same
    c.bytes.assign((const uint8_t *)buf, (const uint8_t *)buf + n);
    for (size_t i = 0; i < n; i++) {
      const float v = (float)c.bytes[i] * 255;
      if (v > c.hi[3]) c.hi[3] = v;
      if (v < c.lo[3]) c.lo[3] = v;
    }
    return;
  }
  c.data.resize(n);
  for (size_t i = 0; i < n; i++) {
    float v = 0.f;
    switch (fmt) {
      case 1: v = (float)((const int8_t *)buf)[i] * 255 - 128; break;
      case 2: v = (float)((const int16_t *)buf)[i] * 65535 - 32768; break;
      case 3: v = (float)((const int32_t *)buf)[i] * 4294967295.0f - 2147483648.0f; break;
      case 4: v = (float)((const uint8_t *)buf)[i] * 255; break;
      case 5: v = (float)((const uint16_t *)buf)[i] * 65535; break;
      case 6: v = (float)((const uint32_t *)buf)[i] * 4294967295.0f; break;
      case 7: v = ((const float *)buf)[i]; break;
      case 8: v = (float)((const double *)buf)[i]; break;
      default: v = 0.f;
    }
    c.data[i] = v;
    if (v > c.hi[3]) c.hi[3] = v;
    if (v < c.lo[3]) c.lo[3] = v;
  }
}

// ---------------------------------------------------------------- camera (G)
static void update_camera(Oracle &o) {
  // renderer.cpp:1058-1092
  const V3 lookFrom = o.cam.position;
  const V3 lookAt = sub(o.cam.position, o.cam.vz);
  const V3 lookUp = o.cam.vy;
  const float cosFovy = std::cos(o.cam.fovy * (float)(M_PI / 180.f));
  const float vfov = std::acos(cosFovy) / (float)(M_PI / 180.f);
  const float aspect = o.W / float(o.H);
  const float theta = vfov * ((float)M_PI) / 180.0f;
  const float half_height = std::tan(theta / 2.0f);
  const float half_width = aspect * half_height;
  const float focusDist = 10.f;
  const V3 w = normalize_h(sub(lookFrom, lookAt));
  const V3 u = normalize_h(cross(lookUp, w));
  const V3 v = cross(w, u);
  o.cOrg = lookFrom;
  V3 llc = sub(lookFrom, muls(half_width * focusDist, u));
  llc = sub(llc, muls(half_height * focusDist, v));
  llc = sub(llc, muls(focusDist, w));
  o.cLlc = llc;
  o.cHor = muls(2.0f * half_width * focusDist, u);
  o.cVer = muls(2.0f * half_height * focusDist, v);
  o.accumID = 0; o.accumParam = 0;
}

// ---------------------------------------------------------------- ranges (R)
static inline int project(float f, float lo, float hi, int dim) {
  // renderer.cu:387-392
  int v = f2i((float)dim * (f - lo) / (hi - lo));
  v = v < dim - 1 ? v : dim - 1;
  return v > 0 ? v : 0;
}

static void build_ranges(Oracle &o) {
  const int C = (int)o.ch.size();
  const size_t M = (size_t)o.mc[0] * o.mc[1] * o.mc[2];
  o.ranges.assign(2 * M * C, 0.f);
  for (size_t i = 0; i < M * C; i++) { o.ranges[2 * i] = 1e20f; o.ranges[2 * i + 1] = -1e20f; }  // sizeMCs
  const int md[3] = {(int)o.mc[0], (int)o.mc[1], (int)o.mc[2]};
  const float *wlo = o.rootLo, *whi = o.rootHi;
  for (int c = 0; c < C; c++) {
    const Channel &chn = o.ch[c];
    const int64_t X = chn.dims[0], Y = chn.dims[1], Z = chn.dims[2];
    float len[3];
    for (int a = 0; a < 3; a++) len[a] = (whi[a] - wlo[a]) / (float)chn.dims[a];
    const int nt = omp_get_max_threads();
    std::vector<std::vector<float>> part(nt);
#pragma omp parallel
    {
      int tid = omp_get_thread_num();
      std::vector<float> &r = part[tid];
      r.assign(2 * M, 0.f);
      for (size_t i = 0; i < M; i++) { r[2 * i] = 1e20f; r[2 * i + 1] = -1e20f; }
#pragma omp for schedule(static)
      for (int64_t z = 0; z < Z; z++)
        for (int64_t y = 0; y < Y; y++)
          for (int64_t x = 0; x < X; x++) {
            // renderer.cu:835-893, one voxel
            const int64_t p[3] = {x, y, z};
            const float s = chn.at((size_t)((z * Y + y) * X + x));
            float blo[4], bhi[4];
            for (int a = 0; a < 3; a++) {
              blo[a] = std::fma((float)p[a], len[a], wlo[a]);
              bhi[a] = blo[a] + len[a];
            }
            blo[3] = s; bhi[3] = s;
            for (int iz = -1; iz <= 1; iz++)
              for (int iy = -1; iy <= 1; iy++)
                for (int ix = -1; ix <= 1; ix++) {
                  int64_t n[3] = {x + ix, y + iy, z + iz};
                  if (n[0] < 0 || n[0] >= X || n[1] < 0 || n[1] >= Y || n[2] < 0 || n[2] >= Z) continue;
                  float pt[4];
                  for (int a = 0; a < 3; a++) pt[a] = std::fma((float)n[a], len[a], wlo[a]);
                  pt[3] = chn.at((size_t)((n[2] * Y + n[1]) * X + n[0]));
                  for (int a = 0; a < 4; a++) { blo[a] = std::fmin(blo[a], pt[a]); bhi[a] = std::fmax(bhi[a], pt[a]); }
                }
            // rasterBox(float2*) renderer.cu:487-519
            if (blo[0] >= bhi[0] || blo[1] >= bhi[1] || blo[2] >= bhi[2]) continue;
            int lo[3], hi[3];
            for (int a = 0; a < 3; a++) {
              lo[a] = project(blo[a], wlo[a], whi[a], md[a]);
              hi[a] = project(bhi[a], wlo[a], whi[a], md[a]);
              hi[a] = std::min(hi[a], md[a] - 1);
            }
            for (int cz = lo[2]; cz <= hi[2]; cz++)
              for (int cy = lo[1]; cy <= hi[1]; cy++)
                for (int cx = lo[0]; cx <= hi[0]; cx++) {
                  size_t cell = (size_t)cx + (size_t)cy * md[0] + (size_t)cz * md[0] * md[1];
                  float &mn = r[2 * cell], &mx = r[2 * cell + 1];
                  if (blo[3] < mn) mn = blo[3];   // atomicMin CAS loop: `while (val < old)`
                  if (bhi[3] > mx) mx = bhi[3];
                }
          }
    }
    for (int t = 0; t < nt; t++) {
      const std::vector<float> &r = part[t];
      if (r.empty()) continue;
      for (size_t cell = 0; cell < M; cell++) {
        float &mn = o.ranges[2 * (cell * C + c)], &mx = o.ranges[2 * (cell * C + c) + 1];
        if (r[2 * cell] < mn) mn = r[2 * cell];
        if (r[2 * cell + 1] > mx) mx = r[2 * cell + 1];
      }
    }
  }
}

// ---------------------------------------------------------------- TF (T, TF)
static inline float tex1d_comp(const TFData &t, float u, int comp) {
  Axis a = axis(u, t.n);
  return lerpf(a.a, t.rgba[4 * a.i0 + comp], t.rgba[4 * a.i1 + comp]);
}

// transferFunction (deviceCode.cu:27-42); returns alpha*opacityScale, rgb optional
static inline float tf_eval(const TFData &t, float f, float *rgb) {
  if (t.n <= 0) { if (rgb) { rgb[0] = 1.f; rgb[1] = 0.f; rgb[2] = 1.f; } return 0.f; }
  if (f < t.vd[0] || f > t.vd[1]) {
    if (rgb) { rgb[0] = 1.f; rgb[1] = 0.f; rgb[2] = 1.f; }
    return 0.f;
  }
  float r1 = (f - t.vd[0]) / (t.vd[1] - t.vd[0]);
  float r2 = (r1 - t.xd[0]) / (t.xd[1] - t.xd[0]);
  Axis a = axis(r2, t.n);
  if (rgb)
    for (int k = 0; k < 3; k++) rgb[k] = lerpf(a.a, t.rgba[4 * a.i0 + k], t.rgba[4 * a.i1 + k]);
  return lerpf(a.a, t.rgba[4 * a.i0 + 3], t.rgba[4 * a.i1 + 3]) * t.os;
}

// transferFunction(...).w for any input, NaN included (gradient samples may fall outside
// the volume): the domain test fails for NaN, so the remap and lookup run on NaN.
static inline float tf_eval_any(const TFData &t, float f) {
  if (t.n <= 0) return 0.f;
  if (f < t.vd[0] || f > t.vd[1]) return 0.f;
  float r1 = (f - t.vd[0]) / (t.vd[1] - t.vd[0]);
  float r2 = (r1 - t.xd[0]) / (t.xd[1] - t.xd[0]);
  Axis a = axis(r2, t.n);
  return lerpf(a.a, t.rgba[4 * a.i0 + 3], t.rgba[4 * a.i1 + 3]) * t.os;
}

// ---------------------------------------------------------------- majorants (M)
static float channel_majorant(const TFData &t, float mn, float mx) {
  // renderer.cu:159-203 body for one (cell, channel)
  if (mx < mn) return 0.f;
  if (t.n <= 0) return 0.f;
  float rmin1 = (mn - t.vd[0]) / (t.vd[1] - t.vd[0]);
  float rmin = (rmin1 - t.xd[0]) / (t.xd[1] - t.xd[0]);
  float rmax1 = (mx - t.vd[0]) / (t.vd[1] - t.vd[0]);
  float rmax = (rmax1 - t.xd[0]) / (t.xd[1] - t.xd[0]);
  float addr1 = rmin * (float)t.n;
  float addr2 = rmax * (float)t.n;
  int addrMin = clampi(f2i(std::fmin(std::floor(addr1), std::floor(addr2))), 0, t.n - 1);
  int addrMax = clampi(f2i(std::fmax(std::ceil(addr1), std::ceil(addr2))), 0, t.n - 1);
  float m = 0.f;
  for (int i = addrMin; i <= addrMax; ++i) {
    float d = tex1d_comp(t, ((float)i + 0.5f) / (float)t.n, 3) * t.os;
    if (i == addrMin) m = d; else m = std::fmax(m, d);
  }
  float d = tex1d_comp(t, (addr1 + 0.5f) / (float)t.n, 3) * t.os;
  m = std::fmax(m, d);
  d = tex1d_comp(t, (addr2 + 0.5f) / (float)t.n, 3) * t.os;
  m = std::fmax(m, d);
  return m;
}

static void recalc_majorants(Oracle &o) {
  const int C = (int)o.ch.size();
  const size_t M = (size_t)o.mc[0] * o.mc[1] * o.mc[2];
  if (o.mode >= 3) {
    // _recalculateDensityRanges(float2*) renderer.cu:111-157: sum over channels (-m 3, and
    // the blending modes -m 4/5, renderer.cu:255-258)
    o.majorants.assign(M, 0.f);
    for (size_t cell = 0; cell < M; cell++) {
      float s = 0.f;
      for (int c = 0; c < C; c++) {
        float mn = o.ranges[2 * (cell * C + c)], mx = o.ranges[2 * (cell * C + c) + 1];
        if (mx < mn) continue;
        s += channel_majorant(o.tf[c], mn, mx);
      }
      o.majorants[cell] = s;
    }
  } else {
    o.majorants.assign(M * C, 0.f);
    for (size_t cell = 0; cell < M; cell++)
      for (int c = 0; c < C; c++)
        o.majorants[cell * C + c] =
            channel_majorant(o.tf[c], o.ranges[2 * (cell * C + c)], o.ranges[2 * (cell * C + c) + 1]);
  }
}

// ---------------------------------------------------------------- volume fetch (V)
static inline float sample_volume(const Oracle &o, int c, V3 p) {
  // deviceCode.cu:122-132 + tex3D normalized/linear/clamp
  if (p.x < 0.0f || p.x > 1.0f || p.y < 0.0f || p.y > 1.0f || p.z < 0.0f || p.z > 1.0f) return NAN;
  const Channel &h = o.ch[c];
  const int X = (int)h.dims[0], Y = (int)h.dims[1], Z = (int)h.dims[2];
  Axis ax = axis(p.x, X), ay = axis(p.y, Y), az = axis(p.z, Z);
  auto at = [&](int x, int y, int z) { return h.at(((size_t)z * Y + y) * X + x); };
  float c00 = lerpf(ax.a, at(ax.i0, ay.i0, az.i0), at(ax.i1, ay.i0, az.i0));
  float c10 = lerpf(ax.a, at(ax.i0, ay.i1, az.i0), at(ax.i1, ay.i1, az.i0));
  float c01 = lerpf(ax.a, at(ax.i0, ay.i0, az.i1), at(ax.i1, ay.i0, az.i1));
  float c11 = lerpf(ax.a, at(ax.i0, ay.i1, az.i1), at(ax.i1, ay.i1, az.i1));
  float c0 = lerpf(ay.a, c00, c10);
  float c1 = lerpf(ay.a, c01, c11);
  return lerpf(az.a, c0, c1);
}

// ---------------------------------------------------------------- DDA (D)
struct RayPayload {
  float t0, t1;
  Rng rng;
  float rgb[3];
  float tHit;
  uint32_t samples, rejections, cells;
  bool missed;
  int channelID;
  uint32_t steps;
  bool capped;
};

// dda.h:81-202.  Calls lam(cell[3], t0, t1) -> bool.
template <typename L>
static void dda3(V3 org, V3 dir, float tMax, const uint32_t gs[3], L &&lam) {
  const float fs[3] = {(float)gs[0], (float)gs[1], (float)gs[2]};
  const float o[3] = {org.x, org.y, org.z}, d[3] = {dir.x, dir.y, dir.z};
  float rcp[3], tnr[3], tfr[3];
  for (int a = 0; a < 3; a++) {
    rcp[a] = 1.0f / d[a];
    float tlo = (0.0f - o[a]) * rcp[a];
    float thi = (fs[a] - o[a]) * rcp[a];
    tnr[a] = std::fmin(tlo, thi);
    tfr[a] = std::fmax(tlo, thi);
  }
  for (int a = 0; a < 3; a++)
    if (d[a] == 0.f) {
      if (o[a] < 0.f || o[a] > fs[a]) return;
      tnr[a] = INFINITY;  // dda.h:100-101: t_nr assigned -inf then +inf (reference bug kept)
    }
  float ray_t0 = std::fmax(0.f, std::fmax(std::fmax(tnr[0], tnr[1]), tnr[2]));
  float ray_t1 = std::fmin(tMax, std::fmin(std::fmin(tfr[0], tfr[1]), tfr[2]));
  if (ray_t0 > ray_t1) return;
  float oiv[3], fcell[3], fend[3], tstep[3], tnext[3];
  int stop[3], delta[3], cell[3];
  for (int a = 0; a < 3; a++) {
    oiv[a] = std::fma(ray_t0, d[a], o[a]);
    fcell[a] = std::fmax(0.f, std::fmin(fs[a] - 1.f, std::floor(oiv[a])));
    fend[a] = d[a] > 0.f ? fcell[a] + 1.f : fcell[a];
    tstep[a] = std::fabs(rcp[a]);
    tnext[a] = (d[a] == 0.f) ? INFINITY : std::fabs(fend[a] - oiv[a]) * tstep[a];
    stop[a] = d[a] > 0.f ? (int)gs[a] : -1;
    delta[a] = d[a] > 0.f ? 1 : -1;
    cell[a] = (int)fcell[a];
  }
  float next_cell_begin = 0.f;
  const uint32_t maxCells = gs[0] + gs[1] + gs[2] + 3;
  for (uint32_t it = 0; it < maxCells; it++) {
    float t_closest = std::fmin(std::fmin(tnext[0], tnext[1]), tnext[2]);
    const float cell_t0 = ray_t0 + next_cell_begin;
    const float cell_t1 = ray_t0 + std::fmin(t_closest, tMax);
    if (!lam(cell, cell_t0, cell_t1)) return;
    next_cell_begin = t_closest;
    for (int a = 0; a < 3; a++) {
      if (tnext[a] == t_closest) {
        tnext[a] += tstep[a];
        cell[a] += delta[a];
        if (cell[a] == stop[a]) return;
      }
    }
  }
}

// device-side dot / normalize (x*x+y*y+z*z contracted like nvcc)
static inline float dot_d(V3 a, V3 b) { return std::fma(a.z, b.z, std::fma(a.y, b.y, a.x * b.x)); }
static inline V3 normalize_d(V3 v) { const float s = 1.0f / std::sqrt(len2_d(v)); return muls(s, v); }

// calculateGradient (deviceCode.cu:243-281): central differences of the TF opacity,
// one-sided at the [0,1] boundary.
static V3 gradient_at(const Oracle &o, V3 p, float eps, int c) {
  const float pp[3] = {p.x, p.y, p.z};
  float g[3];
  auto alpha_at = [&](const float q[3]) {
    const float v = sample_volume(o, c, v3(q[0], q[1], q[2]));
    return tf_eval_any(o.tf[c], v);
  };
  for (int i = 0; i < 3; i++) {
    float p1[3] = {pp[0], pp[1], pp[2]}, p2[3] = {pp[0], pp[1], pp[2]};
    p1[i] -= eps;
    p2[i] += eps;
    if (p1[i] < 0.0f) {
      p1[i] = pp[i];
      p2[i] = pp[i] + eps;
      g[i] = (alpha_at(p2) - alpha_at(p1)) / eps;
    } else if (p2[i] > 1.0f) {
      p1[i] = pp[i] - eps;
      p2[i] = pp[i];
      g[i] = (alpha_at(p2) - alpha_at(p1)) / eps;
    } else {
      g[i] = (alpha_at(p2) - alpha_at(p1)) / (2.0f * eps);
    }
  }
  return v3(g[0], g[1], g[2]);
}

// ---------------------------------------------------------------- trackers (W)
struct TrackCtx {
  V3 worldOrg, worldDir, org, dir;
  float w2g, g2w;
  V3 w2u;
};

static void track_setup(const Oracle &o, V3 worldOrg, V3 worldDir, TrackCtx &tc) {
  // deviceCode.cu:759-778 (identical in all trackers)
  const V3 lo = v3(o.gLo[0], o.gLo[1], o.gLo[2]), hi = v3(o.gHi[0], o.gHi[1], o.gHi[2]);
  tc.worldOrg = worldOrg;
  tc.worldDir = worldDir;
  V3 org = sub(worldOrg, lo);
  const V3 w2u = v3(1.f / (hi.x - lo.x), 1.f / (hi.y - lo.y), 1.f / (hi.z - lo.z));
  const V3 u2g = v3((float)o.mc[0], (float)o.mc[1], (float)o.mc[2]);
  org = mul(mul(u2g, w2u), org);
  V3 dir = mul(mul(w2u, u2g), worldDir);
  const float n2 = len2_d(dir);
  tc.w2g = std::sqrt(n2);
  tc.g2w = 1.f / tc.w2g;
  const float inv = 1.0f / std::sqrt(n2);
  tc.dir = muls(inv, dir);
  tc.org = org;
  tc.w2u = w2u;
}

static inline float woodcock_step(float t, float u, float maj, float dt, float w2g) {
  float L = mlog(1.0f - u);
  float X = (L / maj) * dt;
  return std::fma(-X, w2g, t);
}
static inline V3 tex_pos(const TrackCtx &tc, float tW) {
  V3 p;
  p.x = std::fma(tW, tc.worldDir.x, tc.worldOrg.x) * tc.w2u.x;
  p.y = std::fma(tW, tc.worldDir.y, tc.worldOrg.y) * tc.w2u.y;
  p.z = std::fma(tW, tc.worldDir.z, tc.worldOrg.z) * tc.w2u.z;
  return p;
}

static inline bool count_step(RayPayload &prd) {
  if (++prd.steps >= kMaxSteps) { prd.capped = true; prd.missed = true; return false; }
  return true;
}

static void hit_record(const Oracle &o, RayPayload &prd, int c, float v, float tW) {
  float rgb[3];
  tf_eval(o.tf[c], v, rgb);
  prd.tHit = tW;
  prd.rgb[0] = rgb[0]; prd.rgb[1] = rgb[1]; prd.rgb[2] = rgb[2];
  prd.missed = false;
  prd.channelID = c;
}

// baseLineDTCH, -m 0 (deviceCode.cu:858-970)
static void track_ndda(const Oracle &o, TrackCtx &tc, RayPayload &prd) {
  const int C = (int)o.ch.size();
  const float *M = o.majorants.data();
  const uint32_t *mc = o.mc;
  int curMesh = 0;
  float tMax = 1e20f;
  auto lam = [&](const int cell[3], float t0, float t1) -> bool {
    prd.cells++;
    const int cellID = cell[0] + cell[1] * (int)mc[0] + cell[2] * (int)mc[0] * (int)mc[1];
    float majorant = M[(size_t)cellID * C + curMesh];
    if (majorant == 0.00f) return true;
    float t = t0;
    while (true) {
      if (!count_step(prd)) return false;
      t = woodcock_step(t, prd.rng.next(), majorant, o.dt, tc.w2g);
      if (t >= t1) break;
      if (tMax < t) return false;
      const float tWorld = t * tc.g2w;
      const V3 x = tex_pos(tc, tWorld);
      if (tWorld >= prd.t1) { prd.rejections++; return false; }
      float thr = prd.rng.next() * majorant;
      const float value = sample_volume(o, curMesh, x);
      prd.samples++;
      if (std::isnan(value)) continue;
      const float a = tf_eval(o.tf[curMesh], value, nullptr);
      if (a > 0.0f && thr < a) {
        hit_record(o, prd, curMesh, value, tWorld);
        tMax = std::fmin(tMax, t);
        return false;
      }
      prd.rejections++;
    }
    return true;
  };
  for (int i = 0; i < C; i++) {
    curMesh = i;
    dda3(tc.org, tc.dir, 1e20f, mc, lam);
    if (prd.capped) return;
  }
}

// altMultiMajDTCH, -m 2 (deviceCode.cu:747-856)
static void track_syncdda(const Oracle &o, TrackCtx &tc, RayPayload &prd) {
  const int C = (int)o.ch.size();
  const float *M = o.majorants.data();
  const uint32_t *mc = o.mc;
  auto lam = [&](const int cell[3], float t0, float t1) -> bool {
    prd.cells++;
    const int cellID = cell[0] + cell[1] * (int)mc[0] + cell[2] * (int)mc[0] * (int)mc[1];
    float minT = t1;
    for (int channelID = 0; channelID < C; channelID++) {
      float majorant = M[(size_t)cellID * C + channelID];
      float t = t0;
      if (majorant == 0.0f) continue;
      while (true) {
        if (!count_step(prd)) return false;
        t = woodcock_step(t, prd.rng.next(), majorant, o.dt, tc.w2g);
        if (t >= minT) break;
        const float tWorld = t * tc.g2w;
        const V3 x = tex_pos(tc, tWorld);
        if (tWorld >= prd.t1) {
          prd.rejections++;
          if (channelID == C - 1) return false;
          else break;
        }
        float thr = prd.rng.next() * majorant;
        const float value = sample_volume(o, channelID, x);
        prd.samples++;
        if (!std::isnan(value)) {
          const float a = tf_eval(o.tf[channelID], value, nullptr);
          if (a > 0.0f && thr < a) {
            hit_record(o, prd, channelID, value, tWorld);
            minT = std::fmin(t, minT);
          }
        }
        prd.rejections++;
      }
    }
    return prd.missed;
  };
  dda3(tc.org, tc.dir, 1e20f, mc, lam);
}

// multiMajDTCH, -m 1 (deviceCode.cu:619-745)
static void track_multi(const Oracle &o, TrackCtx &tc, RayPayload &prd) {
  const int C = (int)o.ch.size();
  const float *M = o.majorants.data();
  const uint32_t *mc = o.mc;
  float majorants[kMaxChannels];
  float ts[kMaxChannels];
  auto lam = [&](const int cell[3], float t0, float t1) -> bool {
    prd.cells++;
    const int cellID = cell[0] + cell[1] * (int)mc[0] + cell[2] * (int)mc[0] * (int)mc[1];
    float majorantSum = 0.0f;
    for (int i = 0; i < C; i++) {
      majorants[i] = M[(size_t)cellID * C + i];
      majorantSum += majorants[i];
      ts[i] = t0;
    }
    if (majorantSum <= 0.0000001f) return true;
    for (int i = 0; i < C; i++) {
      if (majorants[i] > 0.0f) ts[i] = woodcock_step(ts[i], prd.rng.next(), majorants[i], o.dt, tc.w2g);
      else ts[i] = 1e20f;
    }
    while (true) {
      if (!count_step(prd)) return false;
      float minT = ts[0];
      int sel = 0;
      float rnd = prd.rng.next();
      for (int i = 1; i < C; i++)
        if (ts[i] < minT && majorants[i] > 0.f) { sel = i; minT = ts[i]; }
      if (minT >= t1) break;
      const float tWorld = minT * tc.g2w;
      const V3 x = tex_pos(tc, tWorld);
      if (tWorld >= prd.t1) { prd.rejections++; return false; }
      float thr = prd.rng.next() * majorants[sel];
      const float value = sample_volume(o, sel, x);
      prd.samples++;
      if (!std::isnan(value)) {
        const float a = tf_eval(o.tf[sel], value, nullptr);
        if (a > 0.0f && thr < a) { hit_record(o, prd, sel, value, tWorld); return false; }
      }
      prd.rejections++;
      ts[sel] = woodcock_step(ts[sel], rnd, majorants[sel], o.dt, tc.w2g);
    }
    return true;
  };
  dda3(tc.org, tc.dir, 1e20f, mc, lam);
}

// cummilativeDTCH, -m 3 (deviceCode.cu:513-617)
static void track_cumulative(const Oracle &o, TrackCtx &tc, RayPayload &prd) {
  const int C = (int)o.ch.size();
  const float *M = o.majorants.data();
  const uint32_t *mc = o.mc;
  auto lam = [&](const int cell[3], float t0, float t1) -> bool {
    prd.cells++;
    const int cellID = cell[0] + cell[1] * (int)mc[0] + cell[2] * (int)mc[0] * (int)mc[1];
    float majorant = M[cellID];
    if (majorant == 0.00f) return true;
    float t = t0;
    while (true) {
      if (!count_step(prd)) return false;
      t = woodcock_step(t, prd.rng.next(), majorant, o.dt, tc.w2g);
      if (t >= t1) break;
      const float tWorld = t * tc.g2w;
      const V3 x = tex_pos(tc, tWorld);
      if (tWorld >= prd.t1) { prd.rejections++; return false; }
      float thr = prd.rng.next() * majorant;
      for (int c = 0; c < C; c++) {
        const float value = sample_volume(o, c, x);
        prd.samples++;
        if (std::isnan(value)) continue;
        const float a = tf_eval(o.tf[c], value, nullptr);
        if (a > 0.0f && thr < a) { hit_record(o, prd, c, value, tWorld); return false; }
        thr -= a;
      }
      prd.rejections++;
    }
    return true;
  };
  dda3(tc.org, tc.dir, 1e20f, mc, lam);
}

// blendChannels (deviceCode.cu:165-241): opacity of the blended sample, its colour.
static float blend_sample(const Oracle &o, V3 x, float rgb[3]) {
  rgb[0] = rgb[1] = rgb[2] = 0.f;
  if (x.x < 0.0f || x.x > 1.0f || x.y < 0.0f || x.y > 1.0f || x.z < 0.0f || x.z > 1.0f) return 0.f;
  const int C = (int)o.ch.size();
  if (o.mode == 4) {   // maxOpacityBlend
    float best = 0.f;
    for (int c = 0; c < C; c++) {
      float crgb[3];
      const float a = tf_eval(o.tf[c], sample_volume(o, c, x), crgb);
      if (a > best) { best = a; rgb[0] = crgb[0]; rgb[1] = crgb[1]; rgb[2] = crgb[2]; }
    }
    return best;
  }
  float col[3] = {0.f, 0.f, 0.f}, mo = 0.f;   // mixBlend
  for (int c = 0; c < C; c++) {
    float crgb[3];
    const float a = tf_eval(o.tf[c], sample_volume(o, c, x), crgb);
    for (int k = 0; k < 3; k++) col[k] = std::fma(crgb[k], a, col[k]);
    if (a > mo) mo = a;
  }
  if (mo <= 0.0f) return 0.f;
  for (int k = 0; k < 3; k++) rgb[k] = col[k] / mo;
  return mo;
}

// blendDTCH, -m 4 / -m 5 (deviceCode.cu:972-1065)
static void track_blend(const Oracle &o, TrackCtx &tc, RayPayload &prd) {
  const float *M = o.majorants.data();
  const uint32_t *mc = o.mc;
  auto lam = [&](const int cell[3], float t0, float t1) -> bool {
    prd.cells++;
    const int cellID = cell[0] + cell[1] * (int)mc[0] + cell[2] * (int)mc[0] * (int)mc[1];
    const float majorant = M[cellID];
    if (majorant == 0.00f) return true;
    float t = t0;
    while (true) {
      if (!count_step(prd)) return false;
      t = woodcock_step(t, prd.rng.next(), majorant, o.dt, tc.w2g);
      if (t >= t1) break;
      const float tWorld = t * tc.g2w;
      const V3 x = tex_pos(tc, tWorld);
      if (tWorld >= prd.t1) { prd.rejections++; return false; }
      float rgb[3];
      const float w = blend_sample(o, x, rgb);
      prd.samples++;
      if (w > 0.0f && prd.rng.next() * majorant < w) {   // the draw only when w > 0
        prd.tHit = tWorld;
        prd.rgb[0] = rgb[0]; prd.rgb[1] = rgb[1]; prd.rgb[2] = rgb[2];
        prd.missed = false;
        prd.channelID = 0;   // blendDTCH leaves the payload's channel at its initial 0
        return false;
      }
      prd.rejections++;
    }
    return true;
  };
  dda3(tc.org, tc.dir, 1e20f, mc, lam);
}

static void trace_volume(const Oracle &o, V3 worldOrg, V3 worldDir, RayPayload &prd) {
  prd.missed = true;
  prd.rgb[0] = prd.rgb[1] = prd.rgb[2] = 0.f;
  // volumeIntersection (deviceCode.cu:1676-1726) against the union box
  float fr[3] = {1.0f / worldDir.x, 1.0f / worldDir.y, 1.0f / worldDir.z};
  const float og[3] = {worldOrg.x, worldOrg.y, worldOrg.z};
  float tt[6];
  for (int a = 0; a < 3; a++) {
    tt[2 * a] = (o.rootLo[a] - og[a]) * fr[a];
    tt[2 * a + 1] = (o.rootHi[a] - og[a]) * fr[a];
  }
  float thit0 = std::fmax(std::fmax(std::fmin(tt[0], tt[1]), std::fmin(tt[2], tt[3])), std::fmin(tt[4], tt[5]));
  float thit1 = std::fmin(std::fmin(std::fmax(tt[0], tt[1]), std::fmax(tt[2], tt[3])), std::fmax(tt[4], tt[5]));
  if (thit1 < 0) return;
  if (thit0 >= thit1) return;
  thit0 = std::fmax(thit0, 0.f);
  prd.t0 = std::fmax(prd.t0, thit0);
  prd.t1 = std::fmin(prd.t1, thit1);
  TrackCtx tc;
  track_setup(o, worldOrg, worldDir, tc);
  switch (o.mode) {
    case 0: track_ndda(o, tc, prd); break;
    case 1: track_multi(o, tc, prd); break;
    case 2: track_syncdda(o, tc, prd); break;
    case 3: track_cumulative(o, tc, prd); break;
    case 4:
    case 5: track_blend(o, tc, prd); break;
  }
}

static inline uint32_t q8(float c) {
  float v = std::fmin(std::fmax(c, 0.f), 1.f);
  return (uint32_t)f2i(v * 255.0f + 0.5f);
}

// mainRG (deviceCode.cu:283-471) for one pixel
static void render_pixel(Oracle &o, int px, int py, uint64_t cnt[4], uint64_t &capped) {
  const int fbOfs = px + o.W * py;
  float fin[4] = {0.f, 0.f, 0.f, 1.f};
  RayPayload prd;
  prd.samples = prd.rejections = prd.cells = 0;
  uint32_t hits = 0, chx = 0;
  uint32_t chcnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  float sT = 0.f;
  for (int sampleID = 0; sampleID < o.spp; sampleID++) {
    uint32_t seed = (uint32_t)o.W * (uint32_t)o.H * (uint32_t)(o.frameParam + 1) * (uint32_t)(sampleID + 1);
    Rng rng;
    rng.init(((uint32_t)px & o.seedMask) + seed, ((uint32_t)py & o.seedMask) + seed);
    float jit = rng.next();
    const float sx = ((float)px + jit) / (float)o.W;
    const float sy = ((float)py + jit) / (float)o.H;
    // generateRay (deviceCode.cu:61-76)
    V3 d;
    d.x = std::fma(sy, o.cVer.x, std::fma(sx, o.cHor.x, o.cLlc.x));
    d.y = std::fma(sy, o.cVer.y, std::fma(sx, o.cHor.y, o.cLlc.y));
    d.z = std::fma(sy, o.cVer.z, std::fma(sx, o.cHor.z, o.cLlc.z));
    if (std::fabs(d.x) < 1e-5f) d.x = 1e-5f;
    if (std::fabs(d.y) < 1e-5f) d.y = 1e-5f;
    if (std::fabs(d.z) < 1e-5f) d.z = 1e-5f;
    V3 dv = sub(d, o.cOrg);
    float inv = 1.0f / std::sqrt(len2_d(dv));
    V3 dir = muls(inv, dv);
    float color[4] = {0.f, 0.f, 0.f, 0.f};
    prd.t0 = 0.f;
    prd.t1 = 1e20f;
    prd.rng = rng;
    prd.steps = 0;
    prd.capped = false;
    trace_volume(o, o.cOrg, dir, prd);
    cnt[3]++;
    if (prd.capped) capped++;
    if (!prd.missed) {
      hits++;
      chx ^= (uint32_t)(prd.channelID + 1) << (sampleID & 15);
      sT += prd.tHit;
      if (prd.channelID < 8) chcnt[prd.channelID]++;
      const float *alb = prd.rgb;
      const Material &m = o.mats[prd.channelID];
      float diffuse = 1.0f, specular = 0.0f, shadow = 1.0f;
      // deviceCode.cu:327-403: gradient (Blinn-Phong) shading and the shadow ray
      const bool calcShading = o.gradient && o.mode < 6 &&
                               std::sqrt(len2_d(v3(alb[0], alb[1], alb[2]))) > 0.001f;
      const bool calcShadows = o.shadows && o.mode < 6;
      if (calcShading) {
        const V3 w2u = v3(1.f / (o.gHi[0] - o.gLo[0]), 1.f / (o.gHi[1] - o.gLo[1]), 1.f / (o.gHi[2] - o.gLo[2]));
        V3 tp;
        tp.x = std::fma(prd.tHit, dir.x, o.cOrg.x) * w2u.x;
        tp.y = std::fma(prd.tHit, dir.y, o.cOrg.y) * w2u.y;
        tp.z = std::fma(prd.tHit, dir.z, o.cOrg.z) * w2u.z;
        const V3 g = gradient_at(o, tp, m.gradStep, prd.channelID);
        if (std::sqrt(len2_d(g)) > 1e-6f) {
          const V3 N = normalize_d(neg(g));
          const V3 L = normalize_d(o.lightDir);
          const V3 Vv = normalize_d(neg(dir));
          const V3 Hh = normalize_d(add(L, Vv));
          const float NdotL = std::fmax(dot_d(N, L), 0.0f);
          const float NdotH = std::fmax(dot_d(N, Hh), 0.0f);
          diffuse = m.diffuse * NdotL;
          if (NdotL > 0.0f && NdotH > 0.001f) {
            const float normalization = (m.shininess + 8.0f) / (8.0f * 3.14159265f);
            specular = (m.specular * normalization) * mpow(NdotH, m.shininess);
          } else {
            specular = 0.0f;
          }
        } else {
          diffuse = m.diffuse;
          specular = 0.0f;
        }
      }
      if (calcShadows) {
        // shadow payload: t0 0, t1 1e20, LCG seeded from the frame (not the sample) and
        // pixel + 1 (deviceCode.cu:380-397)
        RayPayload sh;
        sh.samples = sh.rejections = sh.cells = 0;
        sh.t0 = 0.f;
        sh.t1 = 1e20f;
        const uint32_t sseed = (uint32_t)o.W * (uint32_t)o.H * (uint32_t)o.frameParam;
        sh.rng.init(((uint32_t)px & o.seedMask) + sseed + 1u, ((uint32_t)py & o.seedMask) + sseed + 1u);
        sh.steps = 0;
        sh.capped = false;
        V3 so;
        so.x = std::fma(prd.tHit, dir.x, o.cOrg.x);
        so.y = std::fma(prd.tHit, dir.y, o.cOrg.y);
        so.z = std::fma(prd.tHit, dir.z, o.cOrg.z);
        trace_volume(o, so, neg(o.lightDir), sh);
        shadow = (1.f - o.ambient) * (1.f - (sh.missed ? 0.0f : 1.0f));
        prd.samples += sh.samples;
        prd.rejections += sh.rejections;
        prd.cells += sh.cells;
        if (sh.capped) capped++;
      }
      const float kd = (diffuse * shadow) * o.lightIntensity;
      const float ks = (specular * shadow) * o.lightIntensity;
      const float sc[3] = {m.spec.x, m.spec.y, m.spec.z};
      for (int k = 0; k < 3; k++) {
        float mix = std::fma(alb[k], 0.75f, sc[k] * 0.25f);
        color[k] = std::fma(o.ambient, mix, std::fma(ks, mix, kd * alb[k]));
      }
      color[3] = 1.0f;
    }
    // finalColor += over(color, vec4f(bg, 1))  (deviceCode.cu:44-59, 433)
    const float bgc[3] = {o.bg.x, o.bg.y, o.bg.z};
    const float oneMinusA = 1.0f - color[3];
    for (int k = 0; k < 3; k++) fin[k] += std::fma(bgc[k] * 1.0f, oneMinusA, color[k]);
    fin[3] += std::fma(oneMinusA, 1.0f, color[3]);
  }
  for (int k = 0; k < 4; k++) fin[k] = fin[k] / (float)o.spp;
  if (o.featOn) {
    float *f = &o.feat[16 * (size_t)fbOfs];
    const float fs = (float)o.spp;
    f[0] = fin[0]; f[1] = fin[1]; f[2] = fin[2];
    f[3] = hits ? (sT / (float)hits) * o.featScale : 0.f;
    f[4] = (float)((uint32_t)o.spp - hits) / fs;
    for (int c = 0; c < 8; c++) f[5 + c] = (float)chcnt[c] / fs;
    f[13] = 1.0f / std::sqrt(fs);
    f[14] = f[15] = 0.f;
  }
  float *acc = &o.accumBuf[4 * (size_t)fbOfs];
  float out[4];
  if (o.accum) {
    for (int k = 0; k < 4; k++) out[k] = std::fma((float)o.accumParam, acc[k], fin[k]) / (float)(o.accumParam + 1);
    for (int k = 0; k < 4; k++) acc[k] = out[k];
  } else {
    for (int k = 0; k < 4; k++) out[k] = fin[k];
  }
  const int fx = o.mirror ? (o.W - 1 - px) : px;
  o.fb[(size_t)fx + (size_t)o.W * py] = q8(out[0]) | (q8(out[1]) << 8) | (q8(out[2]) << 16) | (q8(out[3]) << 24);
  cnt[0] += prd.samples;
  cnt[1] += prd.rejections;
  cnt[2] += prd.cells;
  if (o.statsOn) {
    uint32_t *s = &o.stats[4 * (size_t)fbOfs];
    s[0] = prd.samples; s[1] = prd.rejections; s[2] = hits; s[3] = chx;
  }
}

// ---------------------------------------------------------------- FP64 expected image
// The expected value of the tracker's per-sample estimate (unshaded: no shadow rays, no
// gradient shading), per pixel, in double precision.  Every tracker (-m 0..3) samples
// the first collision of the superposed channels: a channel-c collision at world
// distance t has density T(t) * mu_c(t), mu_c = alpha_c / dt (dt scales every free
// flight, deviceCode.cu:800-806), T the transmittance exp(-integral of sum_c mu_c), and
// shows channel c's shaded TF colour (deviceCode.cu:408-433); no collision before the
// root-box exit shows the background.  So
//   E = mean over the pixel's jitter j of
//       integral_{t0}^{t1} T(t) sum_c mu_c(t) C_c(t) dt + T(t1) bg,
// j on the pixel diagonal (one jitter draw for x and y, deviceCode.cu:298).  The
// integral is a midpoint rule in `stepVoxels` of the smallest voxel edge with the
// extinction held constant over each step (exact exponential attenuation per step);
// the jitter average is a J-point midpoint rule.  Opacity and colour use the tracker's
// filtering semantics (8-bit fractional weights, clamp) evaluated in double.
struct AxisD { int i0, i1; double a; };
static inline AxisD axis_d(double u, int n) {
  const double x = u * (double)n - 0.5;
  const double fl = std::floor(x);
  AxisD r;
  r.a = std::rint((x - fl) * 256.0) / 256.0;
  const long long i = (long long)fl;
  r.i0 = (int)std::min<long long>(std::max<long long>(i, 0), n - 1);
  r.i1 = (int)std::min<long long>(std::max<long long>(i, -1), n - 2) + 1;
  return r;
}
static inline double lerp_d(double a, double p, double q) { return (1.0 - a) * p + a * q; }

static double volume_d(const Oracle &o, int c, const double p[3]) {
  for (int a = 0; a < 3; a++)
    if (!(p[a] >= 0.0 && p[a] <= 1.0)) return NAN;
  const Channel &h = o.ch[c];
  const int X = (int)h.dims[0], Y = (int)h.dims[1], Z = (int)h.dims[2];
  const AxisD ax = axis_d(p[0], X), ay = axis_d(p[1], Y), az = axis_d(p[2], Z);
  auto at = [&](int x, int y, int z) { return (double)h.at(((size_t)z * Y + y) * X + x); };
  const double c00 = lerp_d(ax.a, at(ax.i0, ay.i0, az.i0), at(ax.i1, ay.i0, az.i0));
  const double c10 = lerp_d(ax.a, at(ax.i0, ay.i1, az.i0), at(ax.i1, ay.i1, az.i0));
  const double c01 = lerp_d(ax.a, at(ax.i0, ay.i0, az.i1), at(ax.i1, ay.i0, az.i1));
  const double c11 = lerp_d(ax.a, at(ax.i0, ay.i1, az.i1), at(ax.i1, ay.i1, az.i1));
  return lerp_d(az.a, lerp_d(ay.a, c00, c10), lerp_d(ay.a, c01, c11));
}

// alpha (times opacity scale) and rgb of channel c's TF at value f, in double
static double tf_d(const TFData &t, double f, double rgb[3]) {
  rgb[0] = rgb[1] = rgb[2] = 0.0;
  if (t.n <= 0 || !(f >= (double)t.vd[0] && f <= (double)t.vd[1])) return 0.0;
  const double r1 = (f - (double)t.vd[0]) / ((double)t.vd[1] - (double)t.vd[0]);
  const double r2 = (r1 - (double)t.xd[0]) / ((double)t.xd[1] - (double)t.xd[0]);
  const AxisD a = axis_d(r2, t.n);
  for (int k = 0; k < 3; k++) rgb[k] = lerp_d(a.a, t.rgba[4 * a.i0 + k], t.rgba[4 * a.i1 + k]);
  return lerp_d(a.a, t.rgba[4 * a.i0 + 3], t.rgba[4 * a.i1 + 3]) * (double)t.os;
}

static void expected_pixel(const Oracle &o, int px, int py, int J, double stepVoxels, double out[3]) {
  const int C = (int)o.ch.size();
  double h0 = 1e300;
  for (auto &h : o.ch)
    for (int a = 0; a < 3; a++) h0 = std::min(h0, ((double)h.hi[a] - (double)h.lo[a]) / (double)h.dims[a]);
  h0 *= stepVoxels;
  const double org[3] = {o.cOrg.x, o.cOrg.y, o.cOrg.z};
  const double llc[3] = {o.cLlc.x, o.cLlc.y, o.cLlc.z}, hor[3] = {o.cHor.x, o.cHor.y, o.cHor.z};
  const double ver[3] = {o.cVer.x, o.cVer.y, o.cVer.z};
  const double w2u[3] = {1.0 / ((double)o.gHi[0] - o.gLo[0]), 1.0 / ((double)o.gHi[1] - o.gLo[1]),
                         1.0 / ((double)o.gHi[2] - o.gLo[2])};
  const double bg[3] = {o.bg.x, o.bg.y, o.bg.z};
  const double dt = o.dt, amb = o.ambient, li = o.lightIntensity;
  double acc[3] = {0, 0, 0};
  for (int m = 0; m < J; m++) {
    const double j = (m + 0.5) / J;
    const double sx = (px + j) / o.W, sy = (py + j) / o.H;
    double d[3];
    for (int a = 0; a < 3; a++) {
      d[a] = llc[a] + sx * hor[a] + sy * ver[a];
      if (std::fabs(d[a]) < 1e-5) d[a] = 1e-5;   // generateRay clamps the point (deviceCode.cu:70-72)
      d[a] -= org[a];
    }
    const double inv = 1.0 / std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int a = 0; a < 3; a++) d[a] *= inv;
    // root box and macrocell-grid box clip
    double ta = 0.0, tb = 1e300;
    for (int a = 0; a < 3; a++) {
      const double lo[2] = {(double)o.rootLo[a], (double)o.gLo[a]}, hi[2] = {(double)o.rootHi[a], (double)o.gHi[a]};
      for (int b = 0; b < 2; b++) {
        const double t1 = (lo[b] - org[a]) / d[a], t2 = (hi[b] - org[a]) / d[a];
        ta = std::max(ta, std::min(t1, t2));
        tb = std::min(tb, std::max(t1, t2));
      }
    }
    double L[3] = {0, 0, 0}, T = 1.0;
    if (tb > ta) {
      const long long n = (long long)std::ceil((tb - ta) / h0);
      const double h = (tb - ta) / (double)n;
      for (long long i = 0; i < n && T > 1e-300; i++) {
        const double t = ta + (i + 0.5) * h;
        double p[3];
        for (int a = 0; a < 3; a++) p[a] = (org[a] + t * d[a]) * w2u[a];
        double mu = 0.0, cw[3] = {0, 0, 0};
        for (int c = 0; c < C; c++) {
          const double v = volume_d(o, c, p);
          if (v != v) continue;
          double alb[3];
          const double al = tf_d(o.tf[c], v, alb);
          if (!(al > 0.0)) continue;
          const double mc = al / dt;
          mu += mc;
          const Material &mt = o.mats[c];
          const double sc[3] = {mt.spec.x, mt.spec.y, mt.spec.z};
          for (int k = 0; k < 3; k++) cw[k] += mc * (amb * (0.75 * alb[k] + 0.25 * sc[k]) + li * alb[k]);
        }
        if (mu > 0.0) {
          const double att = std::exp(-mu * h);
          for (int k = 0; k < 3; k++) L[k] += T * (1.0 - att) * (cw[k] / mu);
          T *= att;
        }
      }
    }
    for (int k = 0; k < 3; k++) acc[k] += L[k] + T * bg[k];
  }
  for (int k = 0; k < 3; k++) out[k] = acc[k] / J;
}

}  // namespace orc

// ======================================================================= C ABI
using namespace orc;

#define ORC_OK 0
#define ORC_BAD 1
#define ORC_IO 3
#define ORC_TOO_MANY 4
#define ORC_UNSUP 5
#define ORC_STATE 6
#define ORC_FORMAT 9

extern "C" {

int orc_create(Oracle **out) { *out = new Oracle(); return ORC_OK; }
int orc_destroy(Oracle *o) { delete o; return ORC_OK; }
const char *orc_last_error(Oracle *o) { return o->err.c_str(); }
int orc_set_threads(int n) { if (n > 0) omp_set_num_threads(n); return omp_get_max_threads(); }

static int push_common(Oracle *o, const void *buf, int fmt, const int64_t dims[3]) {
  if ((int)o->ch.size() >= kMaxChannels) { o->err = "too many channels"; return ORC_TOO_MANY; }
  if (o->inited) { o->err = "push after init"; return ORC_STATE; }
  Channel c;
  for (int a = 0; a < 3; a++) c.dims[a] = dims[a];
  convert(c, buf, fmt, (size_t)(dims[0] * dims[1] * dims[2]));
  o->ch.push_back(std::move(c));
  return ORC_OK;
}

int orc_push_channel(Oracle *o, const void *data, int fmt, const int64_t dims[3]) {
  if (!data || !dims || dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0) { o->err = "bad dims"; return ORC_BAD; }
  if (fmt_bytes(fmt) == 0) { o->err = "unsupported format"; return ORC_UNSUP; }
  return push_common(o, data, fmt, dims);
}

int orc_push_channel_raw(Oracle *o, const char *path) {
  int64_t dims[3]; int fmt;
  if (!parse_raw_name(path, dims, fmt)) { o->err = "no dims in file name"; return ORC_FORMAT; }
  int bpv = fmt_bytes(fmt);
  if (bpv == 0) { o->err = "unknown voxel type"; return ORC_FORMAT; }
  size_t n = (size_t)(dims[0] * dims[1] * dims[2]);
  FILE *f = std::fopen(path, "rb");
  if (!f) { o->err = "cannot open"; return ORC_IO; }
  std::vector<char> buf(n * bpv);
  size_t got = std::fread(buf.data(), 1, buf.size(), f);
  std::fclose(f);
  if (got != buf.size()) { o->err = "truncated"; return ORC_IO; }
  return push_common(o, buf.data(), fmt, dims);
}

int orc_reshape_bounds(Oracle *o, int c, const float *scale3) {
  if (c < 0 || c >= (int)o->ch.size()) return ORC_BAD;
  Channel &h = o->ch[c];
  for (int a = 0; a < 3; a++) {
    float s = scale3 ? scale3[a] : (float)h.dims[a];
    h.lo[a] = h.lo[a] * s;
    h.hi[a] = h.hi[a] * s;
  }
  return ORC_OK;
}

int orc_get_channel_info(Oracle *o, int c, int64_t dims[3], float b8[8]) {
  if (c < 0 || c >= (int)o->ch.size()) return ORC_BAD;
  for (int a = 0; a < 3; a++) dims[a] = o->ch[c].dims[a];
  for (int a = 0; a < 4; a++) { b8[a] = o->ch[c].lo[a]; b8[4 + a] = o->ch[c].hi[a]; }
  return ORC_OK;
}

int orc_set_macrocells(Oracle *o, const uint32_t d[3]) {
  for (int a = 0; a < 3; a++) o->mcReq[a] = d[a];
  if (o->inited) {   // after init: a new grid with the same transfer functions
    uint32_t acc[3] = {0, 0, 0};
    for (auto &h : o->ch)
      for (int a = 0; a < 3; a++) acc[a] += (uint32_t)((float)(uint32_t)h.dims[a] / 4.0f);
    for (int a = 0; a < 3; a++) acc[a] = (uint32_t)((float)acc[a] / (float)o->ch.size());
    for (int a = 0; a < 3; a++) o->mc[a] = o->mcReq[a] ? o->mcReq[a] : acc[a];
    if (o->mc[0] == 0 || o->mc[1] == 0 || o->mc[2] == 0) { o->err = "zero macrocell dims"; return ORC_BAD; }
    build_ranges(*o);
    recalc_majorants(*o);
    o->accumID = 0; o->accumParam = 0;
  }
  return ORC_OK;
}

static void reset_dt(Oracle *o) {
  // renderer.cpp:1444-1454: the loop overwrites, so the LAST channel decides
  float minVoxelSideLength = std::numeric_limits<float>::max();
  for (size_t i = 0; i < o->ch.size(); ++i) {
    const Channel &h = o->ch[i];
    float sx = (h.hi[0] - h.lo[0]) / (float)h.dims[0];
    float sy = (h.hi[1] - h.lo[1]) / (float)h.dims[1];
    float sz = (h.hi[2] - h.lo[2]) / (float)h.dims[2];
    minVoxelSideLength = std::min(sx, std::min(sy, sz));
  }
  o->dt = std::max(minVoxelSideLength * 0.5f, 1e-4f);
  o->accumID = 0; o->accumParam = 0;
}

int orc_init(Oracle *o, int mode, int autoCam) {
  if (o->ch.empty()) { o->err = "no channels"; return ORC_STATE; }
  if (mode < 0 || mode > 5) { o->err = "mode"; return ORC_UNSUP; }
  o->mode = mode;
  // CalculateMCGridDims(4) (renderer.cpp:1342-1355)
  if (o->mcReq[0] == 0 || o->mcReq[1] == 0 || o->mcReq[2] == 0) {
    uint32_t acc[3] = {0, 0, 0};
    for (auto &h : o->ch)
      for (int a = 0; a < 3; a++) acc[a] += (uint32_t)((float)(uint32_t)h.dims[a] / 4.0f);
    for (int a = 0; a < 3; a++) acc[a] = (uint32_t)((float)acc[a] / (float)o->ch.size());
    for (int a = 0; a < 3; a++) o->mc[a] = o->mcReq[a] ? o->mcReq[a] : acc[a];
  } else {
    for (int a = 0; a < 3; a++) o->mc[a] = o->mcReq[a];
  }
  if (o->mc[0] == 0 || o->mc[1] == 0 || o->mc[2] == 0) { o->err = "zero macrocell dims"; return ORC_BAD; }
  for (int a = 0; a < 3; a++) {
    float lo = std::numeric_limits<float>::infinity(), hi = -std::numeric_limits<float>::infinity();
    for (auto &h : o->ch) { lo = std::fmin(lo, h.lo[a]); hi = std::fmax(hi, h.hi[a]); }
    o->rootLo[a] = lo; o->rootHi[a] = hi;
  }
  for (int a = 0; a < 4; a++) { o->gLo[a] = o->ch.back().lo[a]; o->gHi[a] = o->ch.back().hi[a]; }
  build_ranges(*o);
  o->tf.assign(o->ch.size(), TFData());
  o->mats.assign(o->ch.size(), Material());
  for (size_t i = 0; i < o->ch.size(); i++) { o->tf[i].vd[0] = o->ch[i].lo[3]; o->tf[i].vd[1] = o->ch[i].hi[3]; }
  recalc_majorants(*o);
  if (autoCam) {
    V3 center = v3(0.5f, 0.5f, 0.5f);
    V3 eye = v3(center.x, center.y, center.z + 2.5f);
    o->cam.setOrientation(eye, center, v3(0, 1, 0), 45.0f);
  }
  update_camera(*o);
  o->accumBuf.assign(4 * (size_t)o->W * o->H, 0.f);
  o->fb.assign((size_t)o->W * o->H, 0u);
  o->frameID = 0; o->frameParam = 0;
  o->accumID = 0; o->accumParam = 0;
  reset_dt(o);
  o->inited = true;
  return ORC_OK;
}

int orc_get_macrocell_dims(Oracle *o, uint32_t d[3]) { for (int a = 0; a < 3; a++) d[a] = o->mc[a]; return ORC_OK; }

int orc_set_tf(Oracle *o, int c, const float *rgba, int n) {
  if (!o->inited || c < 0 || c >= (int)o->ch.size() || n <= 0 || !rgba) return ORC_BAD;
  TFData &t = o->tf[c];
  t.rgba.assign(rgba, rgba + 4 * n);
  for (int i = 0; i < n; i++) t.rgba[4 * i + 3] = std::pow(t.rgba[4 * i + 3], 3.f);
  t.n = n;
  o->accumID = 0; o->accumParam = 0;
  recalc_majorants(*o);
  return ORC_OK;
}
int orc_set_opacity_scale(Oracle *o, int c, float s) {
  if (!o->inited || c < 0 || c >= (int)o->ch.size()) return ORC_BAD;
  o->tf[c].os = s;
  o->accumID = 0; o->accumParam = 0;
  recalc_majorants(*o);
  return ORC_OK;
}
int orc_set_tf_range(Oracle *o, int c, float lo, float hi) {
  if (!o->inited || c < 0 || c >= (int)o->ch.size()) return ORC_BAD;
  o->tf[c].xd[0] = lo; o->tf[c].xd[1] = hi;
  o->accumID = 0; o->accumParam = 0;
  recalc_majorants(*o);
  return ORC_OK;
}
int orc_set_dt(Oracle *o, float dt) { o->dt = std::max(dt, 1e-4f); o->accumID = 0; o->accumParam = 0; return ORC_OK; }
int orc_reset_dt(Oracle *o) { reset_dt(o); return ORC_OK; }
int orc_get_dt(Oracle *o, float *dt) { *dt = o->dt; return ORC_OK; }
int orc_set_camera(Oracle *o, const float f[3], const float at[3], const float up[3], float fovy) {
  o->cam.setOrientation(v3(f[0], f[1], f[2]), v3(at[0], at[1], at[2]), v3(up[0], up[1], up[2]), fovy);
  update_camera(*o);
  return ORC_OK;
}
int orc_get_camera_basis(Oracle *o, float out[12]) {
  V3 v[4] = {o->cOrg, o->cLlc, o->cHor, o->cVer};
  for (int i = 0; i < 4; i++) { out[3 * i] = v[i].x; out[3 * i + 1] = v[i].y; out[3 * i + 2] = v[i].z; }
  return ORC_OK;
}
int orc_resize(Oracle *o, int w, int h) {
  if (w <= 0 || h <= 0) return ORC_BAD;
  o->W = w; o->H = h;
  o->accumBuf.assign(4 * (size_t)w * h, 0.f);
  o->fb.assign((size_t)w * h, 0u);
  if (o->statsOn) o->stats.assign(4 * (size_t)w * h, 0u);
  update_camera(*o);
  return ORC_OK;
}
int orc_set_spp(Oracle *o, int s) { if (s <= 0) return ORC_BAD; o->spp = s; return ORC_OK; }
int orc_set_accumulation(Oracle *o, int e) { o->accum = e != 0; return ORC_OK; }
int orc_set_background(Oracle *o, const float rgb[3]) { o->bg = v3(rgb[0], rgb[1], rgb[2]); return ORC_OK; }
int orc_set_light(Oracle *o, int sh, int gr, const float d[3], float in, float amb) {
  o->shadows = sh != 0; o->gradient = gr != 0;
  o->lightDir = v3(d[0], d[1], d[2]); o->lightIntensity = in; o->ambient = amb;
  o->accumID = 0; o->accumParam = 0;
  return ORC_OK;
}
int orc_set_material(Oracle *o, int c, float di, float sp, float shin, float gs, const float rgb[3]) {
  if (c < 0 || c >= (int)o->mats.size()) return ORC_BAD;
  Material &m = o->mats[c];
  m.diffuse = di; m.specular = sp; m.shininess = shin; m.gradStep = gs; m.spec = v3(rgb[0], rgb[1], rgb[2]);
  o->accumID = 0; o->accumParam = 0;
  return ORC_OK;
}
int orc_set_mirror(Oracle *o, int e) { o->mirror = e != 0; return ORC_OK; }
// The reference seeds from threadIdx (deviceCode.cu:296-297, 385-386): 0 = the pixel's
// coordinates, a power of two = the pixel's position in an edge x edge thread block.
int orc_set_seed_block(Oracle *o, int edge) {
  if (edge == 0) { o->seedMask = 0xffffffffu; return ORC_OK; }
  if (edge < 1 || edge > 1024 || (edge & (edge - 1)) != 0) { o->err = "bad seed block"; return ORC_BAD; }
  o->seedMask = (uint32_t)edge - 1u;
  return ORC_OK;
}
int orc_enable_pixel_stats(Oracle *o, int e) {
  o->statsOn = e != 0;
  if (o->statsOn) o->stats.assign(4 * (size_t)o->W * o->H, 0u);
  return ORC_OK;
}

// Render one frame over the pixel rows row0, row0 + stride, ... (nrows of them, all
// inside the frame); the frame ids advance as for a whole frame.
static int render_row_set(Oracle *o, int row0, int stride, int nrows) {
  if (o->featOn) {
    // depth-feature scale: 1 / (camera-to-root-box-centre distance + box diagonal)
    const float cx = (o->rootLo[0] + o->rootHi[0]) * 0.5f, cy = (o->rootLo[1] + o->rootHi[1]) * 0.5f,
                cz = (o->rootLo[2] + o->rootHi[2]) * 0.5f;
    const float dx = o->cOrg.x - cx, dy = o->cOrg.y - cy, dz = o->cOrg.z - cz;
    const float ex = o->rootHi[0] - o->rootLo[0], ey = o->rootHi[1] - o->rootLo[1], ez = o->rootHi[2] - o->rootLo[2];
    o->featScale = 1.0f / (std::sqrt(dx * dx + dy * dy + dz * dz) + std::sqrt(ex * ex + ey * ey + ez * ez));
    o->feat.resize(16 * (size_t)o->W * o->H, 0.f);
  }
  uint64_t c0 = 0, c1 = 0, c2 = 0, c3 = 0, cap = 0;
  const int W = o->W;
  const int64_t n = (int64_t)nrows * W;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : c0, c1, c2, c3, cap)
  for (int64_t i = 0; i < n; i++) {
    uint64_t cnt[4] = {0, 0, 0, 0};
    uint64_t capped = 0;
    render_pixel(*o, (int)(i % W), row0 + stride * (int)(i / W), cnt, capped);
    c0 += cnt[0]; c1 += cnt[1]; c2 += cnt[2]; c3 += cnt[3]; cap += capped;
  }
  o->counters[0] += c0; o->counters[1] += c1; o->counters[2] += c2; o->counters[3] += c3;
  o->capped += cap;
  // Renderer::Render (renderer.cpp:957-958): params take the pre-increment values
  o->accumParam = o->accumID++;
  o->frameParam = o->frameID++;
  return ORC_OK;
}

// Render one frame over the pixel rows [row0, row1) (all rows when row1 <= row0).
int orc_render_rows(Oracle *o, int row0, int row1) {
  if (!o->inited) return ORC_STATE;
  if (row1 <= row0) { row0 = 0; row1 = o->H; }
  if (row0 < 0 || row1 > o->H) return ORC_BAD;
  return render_row_set(o, row0, 1, row1 - row0);
}
// Render one frame over the rows row0, row0 + stride, ... below the frame's height
// (rows spread over the frame, for timing samples).
int orc_render_row_stride(Oracle *o, int row0, int stride) {
  if (!o->inited) return ORC_STATE;
  if (row0 < 0 || row0 >= o->H || stride <= 0) return ORC_BAD;
  return render_row_set(o, row0, stride, (o->H - 1 - row0) / stride + 1);
}
int orc_render(Oracle *o) { return orc_render_rows(o, 0, 0); }
// Rows [row0, row1) of the accumulation and RGBA8 buffers from caller memory (the row-band
// hand-over of mdwt_load_frame_rows; the stream argument is ignored on the host).
int orc_load_frame_rows(Oracle *o, int row0, int row1, const float *accum, const uint32_t *fb, void * /*stream*/) {
  if (row0 < 0 || row1 > o->H || row0 > row1) return ORC_BAD;
  const size_t off = (size_t)row0 * o->W, n = (size_t)(row1 - row0) * o->W;
  if (accum) std::memcpy(o->accumBuf.data() + 4 * off, accum, n * 16);
  if (fb) std::memcpy(o->fb.data() + off, fb, n * 4);
  return ORC_OK;
}
int orc_set_features(Oracle *o, int e) { o->featOn = e != 0; return ORC_OK; }
int orc_get_features(Oracle *o, float *out) {
  if (!o->featOn || o->feat.empty()) return ORC_STATE;
  std::memcpy(out, o->feat.data(), o->feat.size() * 4);
  return ORC_OK;
}
// FP64 expected image (W*H*3 doubles, row-major like the accumulation buffer).
int orc_expected_image(Oracle *o, int J, double stepVoxels, double *out) {
  if (!o->inited) return ORC_STATE;
  if (J <= 0 || !(stepVoxels > 0.0) || !out) return ORC_BAD;
  if (o->shadows || o->gradient) { o->err = "expected image: unshaded only"; return ORC_UNSUP; }
  const int W = o->W;
  const int64_t n = (int64_t)o->W * o->H;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < n; i++) expected_pixel(*o, (int)(i % W), (int)(i / W), J, stepVoxels, out + 3 * i);
  return ORC_OK;
}
int orc_sync(Oracle *) { return ORC_OK; }
int orc_reset_accumulation(Oracle *o) { o->accumID = 0; o->accumParam = 0; return ORC_OK; }
int orc_set_frame_id(Oracle *o, int f) {
  if (f < 0 || f == 2147483647) return ORC_BAD;
  o->frameParam = f;
  o->frameID = f + 1;
  return ORC_OK;
}
// The state a launch of the reference's mainRG reads (for the pins against the
// reference's own device code): f = dt, root box lo[3] hi[3] (union of the channels),
// last channel's box4f lo[4] hi[4], background[3], light direction[3], intensity, ambient;
// i = mode, spp, accumulation, shadows, gradient shading, W, H, channels.
int orc_get_launch_state(Oracle *o, float f[23], int i[8]) {
  if (!o->inited) return ORC_STATE;
  int k = 0;
  f[k++] = o->dt;
  for (int a = 0; a < 3; a++) f[k++] = o->rootLo[a];
  for (int a = 0; a < 3; a++) f[k++] = o->rootHi[a];
  for (int a = 0; a < 4; a++) f[k++] = o->gLo[a];
  for (int a = 0; a < 4; a++) f[k++] = o->gHi[a];
  f[k++] = o->bg.x; f[k++] = o->bg.y; f[k++] = o->bg.z;
  f[k++] = o->lightDir.x; f[k++] = o->lightDir.y; f[k++] = o->lightDir.z;
  f[k++] = o->lightIntensity;
  f[k++] = o->ambient;
  i[0] = o->mode; i[1] = o->spp; i[2] = o->accum; i[3] = o->shadows; i[4] = o->gradient;
  i[5] = o->W; i[6] = o->H; i[7] = (int)o->ch.size();
  return ORC_OK;
}
// Channel c's transfer function as uploaded (alpha cubed): texels (4 floats each, at
// most cap texels written), count, volume domain, TF range and opacity scale.
int orc_get_tf(Oracle *o, int c, float *rgba, int cap, int *n, float vd[2], float xd[2], float *os) {
  if (c < 0 || c >= (int)o->tf.size()) return ORC_BAD;
  const TFData &t = o->tf[c];
  *n = t.n;
  if (rgba) std::memcpy(rgba, t.rgba.data(), sizeof(float) * 4 * (size_t)std::min(cap, t.n));
  vd[0] = t.vd[0]; vd[1] = t.vd[1]; xd[0] = t.xd[0]; xd[1] = t.xd[1];
  *os = t.os;
  return ORC_OK;
}
// Channel c's material: diffuse, specular, shininess, gradient step, specular colour.
int orc_get_material(Oracle *o, int c, float out[7]) {
  if (c < 0 || c >= (int)o->mats.size()) return ORC_BAD;
  const Material &m = o->mats[c];
  out[0] = m.diffuse; out[1] = m.specular; out[2] = m.shininess; out[3] = m.gradStep;
  out[4] = m.spec.x; out[5] = m.spec.y; out[6] = m.spec.z;
  return ORC_OK;
}
float orc_pow(float x, float y) { return mpow(x, y); }
int orc_get_frame_ids(Oracle *o, int out[4]) {
  out[0] = o->frameID; out[1] = o->accumID; out[2] = o->frameParam; out[3] = o->accumParam; return ORC_OK;
}
int orc_get_framebuffer(Oracle *o, uint32_t *out) { std::memcpy(out, o->fb.data(), o->fb.size() * 4); return ORC_OK; }
int orc_get_accum(Oracle *o, float *out) { std::memcpy(out, o->accumBuf.data(), o->accumBuf.size() * 4); return ORC_OK; }
int orc_get_counters(Oracle *o, uint64_t out[4]) { for (int i = 0; i < 4; i++) out[i] = o->counters[i]; return ORC_OK; }
int orc_reset_counters(Oracle *o) { for (int i = 0; i < 4; i++) o->counters[i] = 0; o->capped = 0; return ORC_OK; }
uint64_t orc_capped_samples(Oracle *o) { return o->capped; }
int orc_get_pixel_stats(Oracle *o, uint32_t *out) {
  if (!o->statsOn) return ORC_STATE;
  std::memcpy(out, o->stats.data(), o->stats.size() * 4);
  return ORC_OK;
}
int orc_get_majorants(Oracle *o, float *out) { std::memcpy(out, o->majorants.data(), o->majorants.size() * 4); return ORC_OK; }
int orc_get_ranges(Oracle *o, float *out) { std::memcpy(out, o->ranges.data(), o->ranges.size() * 4); return ORC_OK; }
int orc_num_channels(Oracle *o, int *n) { *n = (int)o->ch.size(); return ORC_OK; }
// The converted float values of channel c (RawR::getDataVector, rawFile.cpp:201-204).
int orc_get_channel_data(Oracle *o, int c, float *out) {
  if (c < 0 || c >= (int)o->ch.size()) return ORC_BAD;
  const Channel &h = o->ch[c];
  const size_t n = (size_t)(h.dims[0] * h.dims[1] * h.dims[2]);
  for (size_t i = 0; i < n; i++) out[i] = h.at(i);
  return ORC_OK;
}
// The oracle's dda3 over a grid of gs cells: the cells visited and their (t0, t1), at
// most maxOut of them (the callback stops the walk there).  Returns the number written.
int orc_dda_trace(const float org[3], const float dir[3], float tMax, const uint32_t gs[3], int maxOut,
                  int32_t *cells, float *t0, float *t1) {
  int n = 0;
  if (maxOut <= 0) return 0;
  dda3(v3(org[0], org[1], org[2]), v3(dir[0], dir[1], dir[2]), tMax, gs, [&](const int *c, float a, float b) {
    cells[3 * n] = c[0]; cells[3 * n + 1] = c[1]; cells[3 * n + 2] = c[2];
    t0[n] = a; t1[n] = b;
    return ++n < maxOut;
  });
  return n;
}

// Test hooks: the primitives of the arithmetic specification.
float orc_log(float x) { return mlog(x); }
// The project's statement of the texture unit's linear filter, exposed for the tests that
// hold it against the hardware: tex3D<float> on an X x Y x Z float volume (x fastest) and
// tex2D<float4> on an N x 1 float4 array, at n normalized coordinates each.
int orc_sample_tex3d(const float *vol, const int dims[3], const float *xyz, int n, float *out) {
  const int X = dims[0], Y = dims[1], Z = dims[2];
  auto at = [&](int x, int y, int z) { return vol[((size_t)z * Y + y) * X + x]; };
  for (int i = 0; i < n; i++) {
    const Axis ax = axis(xyz[3 * i], X), ay = axis(xyz[3 * i + 1], Y), az = axis(xyz[3 * i + 2], Z);
    const float c00 = lerpf(ax.a, at(ax.i0, ay.i0, az.i0), at(ax.i1, ay.i0, az.i0));
    const float c10 = lerpf(ax.a, at(ax.i0, ay.i1, az.i0), at(ax.i1, ay.i1, az.i0));
    const float c01 = lerpf(ax.a, at(ax.i0, ay.i0, az.i1), at(ax.i1, ay.i0, az.i1));
    const float c11 = lerpf(ax.a, at(ax.i0, ay.i1, az.i1), at(ax.i1, ay.i1, az.i1));
    out[i] = lerpf(az.a, lerpf(ay.a, c00, c10), lerpf(ay.a, c01, c11));
  }
  return ORC_OK;
}
int orc_sample_tex2d(const float *rgba, int N, const float *uv, int n, float *out) {
  for (int i = 0; i < n; i++) {
    const Axis ax = axis(uv[2 * i], N), ay = axis(uv[2 * i + 1], 1);
    for (int k = 0; k < 4; k++) {
      const float r = lerpf(ax.a, rgba[4 * ax.i0 + k], rgba[4 * ax.i1 + k]);
      out[4 * i + k] = lerpf(ay.a, r, r);
    }
  }
  return ORC_OK;
}
// The trackers' quotient from a stored reciprocal (Markstein 1990: q = RN(a y), then
// RN(q + y (a - q b)) with y = RN(1/b); the IEEE division outside the safe range), restated
// on the host, against the IEEE quotient: the number of mismatches over `n` seeded pairs
// with random mantissas and exponents in [-40, 40], plus every divisor mantissa in [1, 2)
// with `per` dividends each.
static inline float host_recip_for_div(float b) {
  const float ab = std::fabs(b);
  return (ab >= 8.271806125530277e-25f && ab <= 1.2089258196146292e24f) ? 1.0f / b : 0.0f;
}
static inline float host_div_by(float a, float b, float y) {
  const float q = a * y;
  const float aq = std::fabs(q);
  if (std::fabs(a) >= 8.271806125530277e-25f && aq >= 8.271806125530277e-25f && aq <= 1.2089258196146292e24f)
    return std::fma(std::fma(-q, b, a), y, q);
  return a / b;
}
uint64_t orc_quotient_check(uint64_t n, int per, uint64_t seed) {
  uint64_t bad = 0;
#pragma omp parallel for reduction(+ : bad) schedule(static)
  for (int64_t t = 0; t < 64; t++) {
    uint64_t s = seed + 0x9e3779b97f4a7c15ull * (uint64_t)(t + 1);
    auto next = [&s]() {
      uint64_t z = (s += 0x9e3779b97f4a7c15ull);
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
      return z ^ (z >> 31);
    };
    for (uint64_t i = 0; i < n / 64; i++) {
      const uint64_t r = next();
      const uint32_t ea = 127u + (uint32_t)((r >> 8) % 81u) - 40u, eb = 127u + (uint32_t)((r >> 16) % 81u) - 40u;
      float a, b;
      const uint32_t ua = (ea << 23) | (uint32_t)((r >> 40) & 0x7fffffu) | ((uint32_t)(r & 1u) << 31);
      const uint32_t ub = (eb << 23) | (uint32_t)((r >> 20) & 0x7fffffu);
      std::memcpy(&a, &ua, 4);
      std::memcpy(&b, &ub, 4);
      const float q1 = host_div_by(a, b, host_recip_for_div(b)), q2 = a / b;
      if (std::memcmp(&q1, &q2, 4) != 0) bad++;
    }
  }
#pragma omp parallel for reduction(+ : bad) schedule(static)
  for (int64_t m = 0; m < (1 << 23); m++) {
    const uint32_t ub = (127u << 23) | (uint32_t)m;
    float b;
    std::memcpy(&b, &ub, 4);
    const float y = host_recip_for_div(b);
    uint32_t st = (uint32_t)m * 2654435761u + (uint32_t)seed;
    for (int k = 0; k < per; k++) {
      st = 1664525u * st + 1013904223u;
      const uint32_t ua = (127u << 23) | (st >> 9);
      float a;
      std::memcpy(&a, &ua, 4);
      const float q1 = host_div_by(a, b, y), q2 = a / b;
      if (std::memcmp(&q1, &q2, 4) != 0) bad++;
    }
  }
  return bad;
}

// The largest relative error of mlog against a double-precision log over every argument
// a free flight takes, 1 - k 2^-24 for k < 2^24 (the premise of the tracker kernels'
// exit filter, which bounds it by 2^-18); also counts k where mlog increases with k.
double orc_flight_log_bound(uint64_t *nonmonotone) {
  double worst = 0.0;
  uint64_t up = 0;
  float prev = 1.0f;
  for (uint32_t k = 0; k < (1u << 24); k++) {
    const float x = 1.0f - (float)k * (1.0f / 16777216.0f);
    const float L = mlog(x);
    const double e = std::log((double)x);
    if (e != 0.0) worst = std::max(worst, std::fabs((double)L - e) / std::fabs(e));
    else if (L != 0.0f) worst = INFINITY;
    if (k > 0 && L > prev) up++;
    prev = L;
  }
  if (nonmonotone) *nonmonotone = up;
  return worst;
}
// Published-algorithm checks: TEA with an arbitrary key and round count (32 rounds is
// the cipher of Wheeler & Needham), and the raw LCG state sequence.
void orc_tea(uint32_t v0, uint32_t v1, const uint32_t k[4], int rounds, uint32_t out[2]) {
  uint32_t sum = 0;
  for (int n = 0; n < rounds; n++) {
    sum += 0x9E3779B9u;
    v0 += ((v1 << 4) + k[0]) ^ (v1 + sum) ^ ((v1 >> 5) + k[1]);
    v1 += ((v0 << 4) + k[2]) ^ (v0 + sum) ^ ((v0 >> 5) + k[3]);
  }
  out[0] = v0; out[1] = v1;
}
void orc_lcg_states(uint32_t seed, int n, uint32_t *out) {
  Rng r; r.state = seed;
  for (int i = 0; i < n; i++) { r.next(); out[i] = r.state; }
}
void orc_rng_stream(uint32_t v0, uint32_t v1, int n, float *out) {
  Rng r; r.init(v0, v1);
  for (int i = 0; i < n; i++) out[i] = r.next();
}

}  // extern "C"
