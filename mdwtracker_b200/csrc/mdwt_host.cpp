// mdwt_host.cpp -- host side of libmdwt.so: the C ABI of include/mdwt.h.
//
// Stands in for dtracker::Renderer (renderer.h:52-222, renderer.cpp:313-1497) and
// raw::RawR (rawFile.cpp:31-128) on the raw-volume path.  Owns the device buffers of
// one scene and launches the sm_100a kernels of mdwt_kernels.cu.  There is no CPU
// rendering path: every frame and every majorant rebuild runs on the GPU, and a
// context on a machine without a usable CUDA device fails at mdwt_create.
//
// Host arithmetic (camera basis, dt, macrocell projection intervals) is compiled
// with -ffp-contract=off and fuses only through explicit std::fma, so it matches
// the oracle's restatement of the same reference code bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mdwt.h"
#include "../../include/mdwt_denoiser.h"
#include "../../include/mdwt_batch.h"
#include "mdwt_internal.h"

using namespace mdwt;

namespace {

struct V3 { float x, y, z; };
inline V3 v3(float x, float y, float z) { return {x, y, z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 muls(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 neg(V3 a) { return {-a.x, -a.y, -a.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V3 normalize(V3 v) { float s = 1.0f / std::sqrt(dot(v, v)); return muls(s, v); }
inline F3 f3(V3 v) { return {v.x, v.y, v.z}; }

inline int f2i(float x) {
  if (!(x == x)) return 0;
  if (x >= 2147483648.0f) return 2147483647;
  if (x <= -2147483648.0f) return (-2147483647 - 1);
  return (int)x;
}

int fmt_bytes(int f) {
  switch (f) {
    case MDWT_FMT_INT8: case MDWT_FMT_UINT8: return 1;
    case MDWT_FMT_INT16: case MDWT_FMT_UINT16: return 2;
    case MDWT_FMT_INT32: case MDWT_FMT_UINT32: case MDWT_FMT_FLOAT32: return 4;
    case MDWT_FMT_DOUBLE64: return 8;
  }
  return 0;
}

struct Channel {
  int64_t dims[3];
  int store = kStoreF32;
  std::vector<uint8_t> u8;    // kStoreU8: the raw bytes (value = b * 255)
  std::vector<float> f32;     // kStoreF32: the converted floats
  float lo[4], hi[4];
  void *dVol = nullptr;
};

struct TFState {
  std::vector<float> rgba;    // alpha cubed
  int n = 0;
  float vd[2] = {0.f, 1.f};
  float xd[2] = {0.f, 1.f};
  float os = 1.0f;
  float *dAlpha = nullptr;
  float *dRgba = nullptr;
  int cap = 0;
};

struct Material {
  float diffuse = 0.8f, specular = 0.3f, shininess = 8.0f, gradStep = 0.01f;
  V3 spec = {1.f, 1.f, 1.f};
};

struct Camera {  // camera::Camera (camera.h:46-142), the fields UpdateCamera reads
  V3 vx = {1, 0, 0}, vy = {0, 1, 0}, vz = {0, 0, 1};
  V3 position = {0, -1, 0};
  V3 upVector = {0, 1, 0};
  float fovy = 60.f;
  void forceUpFrame() {
    if (std::fabs(dot(vz, upVector)) < 1e-6f) return;
    vx = normalize(cross(upVector, vz));
    vy = normalize(cross(vz, vx));
  }
  void setOrientation(V3 origin, V3 interest, V3 up, float fovyDeg) {
    fovy = fovyDeg;
    position = origin;
    upVector = up;
    const bool same = interest.x == origin.x && interest.y == origin.y && interest.z == origin.z;
    vz = same ? v3(0, 0, 1) : neg(normalize(sub(interest, origin)));
    vx = cross(up, vz);
    if (dot(vx, vx) < 1e-8f) vx = v3(0, 1, 0);
    else vx = normalize(vx);
    vy = normalize(cross(vz, vx));
    forceUpFrame();
  }
};

}  // namespace

struct mdwt_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int numSMs = 0;
  std::vector<Channel> ch;
  uint32_t mcReq[3] = {0, 0, 0};
  uint32_t mc[3] = {0, 0, 0};
  int mode = 0;
  bool inited = false;
  int store = kStoreF32;
  float dt = 0.05f;
  int W = 1024, H = 1024;
  int spp = 1;
  bool accum = true;
  V3 bg = {0, 0, 0};
  bool shadows = false, gradient = false;
  V3 lightDir = {0.0001f, -1.f, 0.0001f};
  float lightIntensity = 1.0f, ambient = 0.1f;
  std::vector<Material> mats;
  std::vector<TFState> tf;
  bool mirror = false;
  uint32_t seedMask = 0xffffffffu;   // mdwt_set_seed_block: the pixel's coordinates, or its position in a block
  int arith = MDWT_ARITH_EXACT;      // mdwt_set_arithmetic
  Camera cam;
  V3 cOrg{}, cLlc{}, cHor{}, cVer{};
  int frameID = 0, accumID = 0, frameParam = 0, accumParam = 0;
  float *dAccum = nullptr;
  uint32_t *dFb = nullptr;
  uint32_t *dStats = nullptr;
  bool statsOn = false;
  unsigned long long *dCounters = nullptr;
  unsigned int *dWork = nullptr;
  uint32_t *dRec = nullptr, *dRecStats = nullptr;   // per-path records of one sample batch
  float *dPartial = nullptr;                          // running sums between batches
  uint32_t *dPartialStats = nullptr;
  size_t recCap = 0, recStatsCap = 0, partialCap = 0, partialStatsCap = 0;
  float *dRecT = nullptr;                             // per-path primary hit t (gradient shading)
  size_t recTCap = 0;
  bool featOn = false;                                // denoiser features per frame
  float *dFeat = nullptr;                             // W*H*16 floats
  size_t featCap = 0;
  double *dExpected = nullptr;                        // FP64 expected image, W*H*3
  size_t expectedCap = 0;
  bool expectedValid = false;                         // matches the current W x H
  double *dSqSum = nullptr;                           // RMSE reduction target
  int expW = 0, expH = 0;
  float *dRanges = nullptr;
  float *dMaj = nullptr;
  float2 *dCellTab = nullptr;   // the trackers' per-cell table: channel mask, (majorant, reciprocal) pairs
  size_t M = 0;
  float rootLo[3] = {0, 0, 0}, rootHi[3] = {1, 1, 1};
  float gLo[4] = {0, 0, 0, 0}, gHi[4] = {1, 1, 1, 1};
  std::string err;
  int launches = 0;
  int lastGrid = 0, lastBlock = 0;
  int pool = 8;       // regeneration pool of the tracker (MDWT_TUNE_POOL)
  int batchCap = 0;   // samples per trace pass, 0 = automatic (MDWT_TUNE_BATCH)
  int trips = 4;      // transition/draw trips per warp round (MDWT_TUNE_TRIPS)
  int quorum = 16;    // end a round's trips early once this many lanes wait to sample (33: never)
  int regroup = -1;   // the tracker that regroups each warp's paths by operation (MDWT_TUNE_REGROUP);
                      // -1 until set: on for -m 2, off for -m 0 (see regroup_on)
  int rgBlocks = 0;   // its blocks per SM, 0 = as many as fit (MDWT_TUNE_RG_BLOCKS)
  int rowLo = 0, rowHi = 0;   // rendered row band, empty = all rows (mdwt_set_render_rows)
  bool timing = false;        // CUDA events around the trace and resolve kernels
  static constexpr int kTimedPasses = 8;   // sample passes of a frame that can be timed
  cudaEvent_t ev[3 * kTimedPasses] = {};   // per pass: start, trace end, resolve end
  int timedPasses = 0;
  bool timed = false;
};

namespace {

mdwt_status fail(mdwt_ctx *c, mdwt_status s, const std::string &msg) {
  if (c) c->err = msg;
  return s;
}
mdwt_status cuda_fail(mdwt_ctx *c, cudaError_t e, const char *what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  if (e == cudaErrorMemoryAllocation) return fail(c, MDWT_ERR_OOM, m);
  return fail(c, MDWT_ERR_CUDA, m);
}
#define CK(call, what)                                 \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, what); \
  } while (0)
#define CKI(rc, what)                                  \
  do {                                                 \
    int r_ = (rc);                                     \
    if (r_ != 0) return cuda_fail(c, (cudaError_t)r_, what); \
  } while (0)

void reset_accum_ids(mdwt_ctx *c) { c->accumID = 0; c->accumParam = 0; }

// Renderer::UpdateCamera (renderer.cpp:1058-1092)
void update_camera(mdwt_ctx *c) {
  const V3 lookFrom = c->cam.position;
  const V3 lookAt = sub(c->cam.position, c->cam.vz);
  const V3 lookUp = c->cam.vy;
  const float cosFovy = std::cos(c->cam.fovy * (float)(M_PI / 180.f));
  const float vfov = std::acos(cosFovy) / (float)(M_PI / 180.f);
  const float aspect = c->W / float(c->H);
  const float theta = vfov * ((float)M_PI) / 180.0f;
  const float half_height = std::tan(theta / 2.0f);
  const float half_width = aspect * half_height;
  const float focusDist = 10.f;
  const V3 w = normalize(sub(lookFrom, lookAt));
  const V3 u = normalize(cross(lookUp, w));
  const V3 v = cross(w, u);
  c->cOrg = lookFrom;
  V3 llc = sub(lookFrom, muls(half_width * focusDist, u));
  llc = sub(llc, muls(half_height * focusDist, v));
  llc = sub(llc, muls(focusDist, w));
  c->cLlc = llc;
  c->cHor = muls(2.0f * half_width * focusDist, u);
  c->cVer = muls(2.0f * half_height * focusDist, v);
  reset_accum_ids(c);
}

// Renderer::Resetdt, raw branch (renderer.cpp:1444-1454): the loop overwrites its
// running value, so the last channel decides.
void reset_dt(mdwt_ctx *c) {
  float minVoxelSideLength = std::numeric_limits<float>::max();
  for (size_t i = 0; i < c->ch.size(); ++i) {
    const Channel &h = c->ch[i];
    const float sx = (h.hi[0] - h.lo[0]) / (float)h.dims[0];
    const float sy = (h.hi[1] - h.lo[1]) / (float)h.dims[1];
    const float sz = (h.hi[2] - h.lo[2]) / (float)h.dims[2];
    minVoxelSideLength = std::min(sx, std::min(sy, sz));
  }
  c->dt = std::max(minVoxelSideLength * 0.5f, 1e-4f);
  reset_accum_ids(c);
}

// Grow a context-owned device buffer to at least `bytes` (contents are not kept).
mdwt_status grow(mdwt_ctx *c, void **buf, size_t &cap, size_t bytes, const char *what) {
  if (bytes <= cap && *buf) return MDWT_OK;
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc(buf, bytes);
  if (e != cudaSuccess) return cuda_fail(c, e, what);
  cap = bytes;
  return MDWT_OK;
}

// Conservative screen-space rectangle {x0, y0, x1, y1} (inclusive pixel indices) of the
// root box: a pixel's rays pass through screen points ((px+j)/W, (py+j)/H), j in [0,1),
// and hit the box only inside the convex hull of its projected corners.  With a corner
// at or behind the eye plane the whole frame is traced.  Margin: 3 pixels.
void cull_rect(const mdwt_ctx *c, int out[4]) {
  const int W = c->W, H = c->H;
  out[0] = 0; out[1] = 0; out[2] = W - 1; out[3] = H - 1;
  const double o[3] = {c->cOrg.x, c->cOrg.y, c->cOrg.z};
  const double l[3] = {c->cLlc.x, c->cLlc.y, c->cLlc.z};
  const double h[3] = {c->cHor.x, c->cHor.y, c->cHor.z};
  const double v[3] = {c->cVer.x, c->cVer.y, c->cVer.z};
  double n[3], nn = 0, hh = 0, vv = 0, dp = 0;
  for (int a = 0; a < 3; a++) {
    n[a] = l[a] + 0.5 * h[a] + 0.5 * v[a] - o[a];
    nn += n[a] * n[a]; hh += h[a] * h[a]; vv += v[a] * v[a];
  }
  nn = std::sqrt(nn);
  if (!(nn > 0) || !(hh > 0) || !(vv > 0)) return;
  for (int a = 0; a < 3; a++) { n[a] /= nn; dp += (l[a] - o[a]) * n[a]; }
  if (!(dp > 0)) return;
  double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
  for (int k = 0; k < 8; k++) {
    const double P[3] = {(k & 1) ? c->rootHi[0] : c->rootLo[0], (k & 2) ? c->rootHi[1] : c->rootLo[1],
                         (k & 4) ? c->rootHi[2] : c->rootLo[2]};
    double e[3], z = 0, el = 0;
    for (int a = 0; a < 3; a++) { e[a] = P[a] - o[a]; z += e[a] * n[a]; el += e[a] * e[a]; }
    if (!std::isfinite(z) || !(z > 1e-3 * std::sqrt(el))) return;
    const double lam = dp / z;
    double qa = 0, qb = 0;
    for (int a = 0; a < 3; a++) {
      const double q = o[a] + lam * e[a] - l[a];
      qa += q * h[a];
      qb += q * v[a];
    }
    const double X = qa / hh * W, Y = qb / vv * H;
    xmin = std::min(xmin, X); xmax = std::max(xmax, X);
    ymin = std::min(ymin, Y); ymax = std::max(ymax, Y);
  }
  if (!std::isfinite(xmin + xmax + ymin + ymax)) return;
  const double x0 = std::floor(xmin) - 3, x1 = std::floor(xmax) + 3;
  const double y0 = std::floor(ymin) - 3, y1 = std::floor(ymax) + 3;
  out[0] = (int)std::max(0.0, std::min((double)W, x0));
  out[2] = (int)std::max(-1.0, std::min((double)(W - 1), x1));
  out[1] = (int)std::max(0.0, std::min((double)H, y0));
  out[3] = (int)std::max(-1.0, std::min((double)(H - 1), y1));
}

// Per-pixel result of a pixel whose every sample misses: finalColor starts at (0,0,0,1)
// and gains over((0,0,0,0), (bg,1)) = (bg, 1) per sample (deviceCode.cu:289, 433),
// summed in sample order, then / spp (deviceCode.cu:435).
void background_result(const mdwt_ctx *c, float out[4]) {
  float f[4] = {0.f, 0.f, 0.f, 1.f};
  const float bg[3] = {c->bg.x, c->bg.y, c->bg.z};
  for (int s = 0; s < c->spp; s++) {
    for (int k = 0; k < 3; k++) f[k] += std::fma(bg[k] * 1.0f, 1.0f - 0.0f, 0.0f);
    f[3] += std::fma(1.0f - 0.0f, 1.0f, 0.0f);
  }
  for (int k = 0; k < 4; k++) out[k] = f[k] / (float)c->spp;
}

// project (renderer.cu:387-392)
inline int project(float f, float lo, float hi, int dim) {
  int v = f2i((float)dim * (f - lo) / (hi - lo));
  v = v < dim - 1 ? v : dim - 1;
  return v > 0 ? v : 0;
}

// Voxel intervals of one axis for the separable range build.  A voxel p enters
// macrocell k on this axis when its 27-neighbour box (rasterElements,
// renderer.cu:856-884) projects onto [clo(p), chi(p)] containing k; the cell's value
// range is then the min/max over the neighbourhoods of those voxels, i.e. over the
// voxel interval [pmin-1, pmax+1] clipped to the grid.
bool axis_intervals(int64_t D, int md, float wlo, float whi, std::vector<int> &out) {
  const float len = (whi - wlo) / (float)D;
  std::vector<int> clo((size_t)D), chi((size_t)D);
  std::vector<char> valid((size_t)D);
  auto corner = [&](int64_t p) { return std::fma((float)p, len, wlo); };
  for (int64_t p = 0; p < D; p++) {
    const float vlo = corner(p);
    float blo = vlo, bhi = vlo + len;
    for (int64_t n = p - 1; n <= p + 1; n += 2) {
      if (n < 0 || n >= D) continue;
      const float nl = corner(n);
      blo = std::fmin(blo, nl);
      bhi = std::fmax(bhi, nl);
    }
    valid[(size_t)p] = blo < bhi;
    clo[(size_t)p] = project(blo, wlo, whi, md);
    chi[(size_t)p] = std::min(project(bhi, wlo, whi, md), md - 1);
  }
  out.assign(2 * (size_t)md, 0);
  for (int k = 0; k < md; k++) {
    int64_t pmin = -1, pmax = -1, cnt = 0;
    for (int64_t p = 0; p < D; p++) {
      if (!valid[(size_t)p] || clo[(size_t)p] > k || chi[(size_t)p] < k) continue;
      if (pmin < 0) pmin = p;
      pmax = p;
      cnt++;
    }
    if (cnt == 0) { out[2 * k] = 1; out[2 * k + 1] = 0; continue; }
    if (cnt != pmax - pmin + 1) return false;  // non-monotone projection: degenerate bounds
    out[2 * k] = (int)std::max<int64_t>(pmin - 1, 0);
    out[2 * k + 1] = (int)std::min<int64_t>(pmax + 1, D - 1);
  }
  return true;
}

bool parse_raw_name(const std::string &path, int64_t dims[3], int &fmt) {
  // rawFile.cpp:36-84
  dims[0] = dims[1] = dims[2] = 0;
  fmt = MDWT_FMT_UINT8;
  std::istringstream st(path);
  std::string tok;
  while (std::getline(st, tok, '_')) {
    const size_t dp = tok.find('.');
    if (dp != std::string::npos) tok = tok.substr(0, dp);
    int x = 0, y = 0, z = 0;
    if (std::sscanf(tok.c_str(), "%dx%dx%d", &x, &y, &z) == 3) {
      dims[0] = x; dims[1] = y; dims[2] = z;
      continue;
    }
    if (tok == "int8") fmt = MDWT_FMT_INT8;
    else if (tok == "int16") fmt = MDWT_FMT_INT16;
    else if (tok == "int32") fmt = MDWT_FMT_INT32;
    else if (tok == "uint8") fmt = MDWT_FMT_UINT8;
    else if (tok == "uint16") fmt = MDWT_FMT_UINT16;
    else if (tok == "uint32") fmt = MDWT_FMT_UINT32;
    else if (tok == "float32") fmt = MDWT_FMT_FLOAT32;
    else if (tok == "double64") fmt = MDWT_FMT_DOUBLE64;
    else fmt = MDWT_FMT_UNSPECIFIED;
  }
  return dims[0] > 0 && dims[1] > 0 && dims[2] > 0;
}

// RawR conversion (rawFile.cpp:94-121) and value range.
void convert_channel(Channel &h, const void *buf, int fmt, size_t n) {
  h.lo[0] = h.lo[1] = h.lo[2] = h.lo[3] = 0.f;
  h.hi[0] = h.hi[1] = h.hi[2] = h.hi[3] = 1.f;
  if (fmt == MDWT_FMT_UINT8) {
    h.store = kStoreU8;
    h.u8.assign((const uint8_t *)buf, (const uint8_t *)buf + n);
    uint8_t bmin = 255, bmax = 0;
    for (size_t i = 0; i < n; i++) { bmin = std::min(bmin, h.u8[i]); bmax = std::max(bmax, h.u8[i]); }
    if (n) {
      const float vmin = (float)bmin * 255, vmax = (float)bmax * 255;
      if (vmax > h.hi[3]) h.hi[3] = vmax;
      if (vmin < h.lo[3]) h.lo[3] = vmin;
    }
    return;
  }
  h.store = kStoreF32;
  h.f32.resize(n);
  for (size_t i = 0; i < n; i++) {
    float v = 0.f;
    switch (fmt) {
      case MDWT_FMT_INT8: v = (float)((const int8_t *)buf)[i] * 255 - 128; break;
      case MDWT_FMT_INT16: v = (float)((const int16_t *)buf)[i] * 65535 - 32768; break;
      case MDWT_FMT_INT32: v = (float)((const int32_t *)buf)[i] * 4294967295.0f - 2147483648.0f; break;
      case MDWT_FMT_UINT16: v = (float)((const uint16_t *)buf)[i] * 65535; break;
      case MDWT_FMT_UINT32: v = (float)((const uint32_t *)buf)[i] * 4294967295.0f; break;
      case MDWT_FMT_FLOAT32: v = ((const float *)buf)[i]; break;
      case MDWT_FMT_DOUBLE64: v = (float)((const double *)buf)[i]; break;
      default: v = 0.f;
    }
    h.f32[i] = v;
    if (v > h.hi[3]) h.hi[3] = v;
    if (v < h.lo[3]) h.lo[3] = v;
  }
}

mdwt_status push_common(mdwt_ctx *c, const void *buf, int fmt, const int64_t dims[3]) {
  if ((int)c->ch.size() >= MDWT_MAX_CHANNELS)
    return fail(c, MDWT_ERR_TOO_MANY_CHANNELS, "at most 12 channels (deviceCode.h:13)");
  if (c->inited) return fail(c, MDWT_ERR_STATE, "channels must be pushed before mdwt_init");
  const size_t n = (size_t)(dims[0] * dims[1] * dims[2]);
  Channel h;
  for (int a = 0; a < 3; a++) h.dims[a] = dims[a];
  try {
    convert_channel(h, buf, fmt, n);
  } catch (const std::bad_alloc &) {
    return fail(c, MDWT_ERR_OOM, "host allocation failed");
  }
  c->ch.push_back(std::move(h));
  return MDWT_OK;
}

mdwt_status check_ch(mdwt_ctx *c, int ch) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (ch < 0 || ch >= (int)c->ch.size()) return fail(c, MDWT_ERR_BAD_ARG, "channel id out of range");
  return MDWT_OK;
}

void free_device(mdwt_ctx *c) {
  for (auto &h : c->ch) { if (h.dVol) cudaFree(h.dVol); h.dVol = nullptr; }
  for (auto &t : c->tf) {
    if (t.dAlpha) cudaFree(t.dAlpha);
    if (t.dRgba) cudaFree(t.dRgba);
    t.dAlpha = t.dRgba = nullptr;
  }
  if (c->dAccum) cudaFree(c->dAccum);
  if (c->dFb) cudaFree(c->dFb);
  if (c->dStats) cudaFree(c->dStats);
  if (c->dCounters) cudaFree(c->dCounters);
  if (c->dWork) cudaFree(c->dWork);
  if (c->dRanges) cudaFree(c->dRanges);
  if (c->dMaj) cudaFree(c->dMaj);
  if (c->dCellTab) cudaFree(c->dCellTab);
  c->dCellTab = nullptr;
  if (c->dRec) cudaFree(c->dRec);
  if (c->dRecStats) cudaFree(c->dRecStats);
  if (c->dRecT) cudaFree(c->dRecT);
  c->dRecT = nullptr;
  c->recTCap = 0;
  if (c->dFeat) cudaFree(c->dFeat);
  c->dFeat = nullptr;
  c->featCap = 0;
  if (c->dExpected) cudaFree(c->dExpected);
  if (c->dSqSum) cudaFree(c->dSqSum);
  c->dExpected = nullptr;
  c->dSqSum = nullptr;
  c->expectedCap = 0;
  c->expectedValid = false;
  if (c->dPartial) cudaFree(c->dPartial);
  if (c->dPartialStats) cudaFree(c->dPartialStats);
  c->dRec = c->dRecStats = c->dPartialStats = nullptr;
  c->dPartial = nullptr;
  c->recCap = c->recStatsCap = c->partialCap = c->partialStatsCap = 0;
  c->dAccum = nullptr; c->dFb = nullptr; c->dStats = nullptr; c->dCounters = nullptr;
  c->dWork = nullptr; c->dRanges = nullptr; c->dMaj = nullptr;
}

mdwt_status alloc_frame(mdwt_ctx *c) {
  if (c->dAccum) cudaFree(c->dAccum);
  if (c->dFb) cudaFree(c->dFb);
  if (c->dStats) cudaFree(c->dStats);
  c->dAccum = nullptr; c->dFb = nullptr; c->dStats = nullptr;
  const size_t np = (size_t)c->W * c->H;
  CK(cudaMalloc(&c->dAccum, np * 16), "cudaMalloc accum");
  CK(cudaMalloc(&c->dFb, np * 4), "cudaMalloc framebuffer");
  CK(cudaMemsetAsync(c->dAccum, 0, np * 16, c->stream), "memset accum");
  CK(cudaMemsetAsync(c->dFb, 0, np * 4, c->stream), "memset framebuffer");
  if (c->statsOn) {
    CK(cudaMalloc(&c->dStats, np * 16), "cudaMalloc stats");
    CK(cudaMemsetAsync(c->dStats, 0, np * 16, c->stream), "memset stats");
  }
  return MDWT_OK;
}

// RecalculateDensityRanges (renderer.cu:206-274)
mdwt_status recalc(mdwt_ctx *c) {
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  MajorantParams p;
  std::memset(&p, 0, sizeof(p));
  p.ranges = c->dRanges;
  p.majorants = c->dMaj;
  p.cellTab = c->dCellTab;
  p.fast = c->arith == MDWT_ARITH_FAST ? 1 : 0;
  p.C = (int)c->ch.size();
  p.mode = c->mode;
  p.M = c->M;
  for (int i = 0; i < p.C; i++) {
    const TFState &t = c->tf[i];
    p.tfAlpha[i] = t.dAlpha;
    p.tfN[i] = t.n;
    p.vd[i][0] = t.vd[0]; p.vd[i][1] = t.vd[1];
    p.xd[i][0] = t.xd[0]; p.xd[i][1] = t.xd[1];
    p.os[i] = t.os;
  }
  CKI(launch_majorants(p, c->stream, &c->launches), "majorant kernel");
  return MDWT_OK;
}

// Macrocell counts per side: the requested ones, zero components from
// CalculateMCGridDims(4) (renderer.cpp:641-647, 1342-1355).
void resolve_mc(const mdwt_ctx *c, uint32_t out[3]) {
  uint32_t acc[3] = {0, 0, 0};
  for (auto &h : c->ch)
    for (int a = 0; a < 3; a++) acc[a] += (uint32_t)((float)(uint32_t)h.dims[a] / 4.0f);
  if (!c->ch.empty())
    for (int a = 0; a < 3; a++) acc[a] = (uint32_t)((float)acc[a] / (float)c->ch.size());
  for (int a = 0; a < 3; a++) out[a] = c->mcReq[a] ? c->mcReq[a] : acc[a];
}

mdwt_status build_ranges(mdwt_ctx *c) {
  const int C = (int)c->ch.size();
  const size_t M = c->M;
  CKI(launch_ranges_init(c->dRanges, M * C, c->stream, &c->launches), "range init kernel");
  size_t scratch = 0;
  for (auto &h : c->ch) scratch = std::max(scratch, (size_t)h.dims[2] * c->mc[1] * c->mc[0]);
  float *dA = nullptr;
  int *dIv = nullptr;
  CK(cudaMalloc(&dA, scratch * 8), "cudaMalloc range scratch");
  const size_t ivn = 2 * ((size_t)c->mc[0] + c->mc[1] + c->mc[2]);
  cudaError_t e = cudaMalloc(&dIv, ivn * sizeof(int) * C);
  if (e != cudaSuccess) { cudaFree(dA); return cuda_fail(c, e, "cudaMalloc intervals"); }
  std::vector<int> all;
  all.reserve(ivn * C);
  for (int i = 0; i < C; i++) {
    const Channel &h = c->ch[i];
    for (int a = 0; a < 3; a++) {
      std::vector<int> iv;
      if (!axis_intervals(h.dims[a], (int)c->mc[a], c->rootLo[a], c->rootHi[a], iv)) {
        cudaFree(dA); cudaFree(dIv);
        return fail(c, MDWT_ERR_UNSUPPORTED, "degenerate channel bounds: macrocell projection is not monotone");
      }
      all.insert(all.end(), iv.begin(), iv.end());
    }
  }
  e = cudaMemcpyAsync(dIv, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) { cudaFree(dA); cudaFree(dIv); return cuda_fail(c, e, "copy intervals"); }
  size_t off = 0;
  for (int i = 0; i < C; i++) {
    const Channel &h = c->ch[i];
    const int dims[3] = {(int)h.dims[0], (int)h.dims[1], (int)h.dims[2]};
    const int *ivx = dIv + off;
    const int *ivy = ivx + 2 * c->mc[0];
    const int *ivz = ivy + 2 * c->mc[1];
    off += ivn;
    int rc = launch_ranges(h.dVol, c->store, dims, c->mc, ivx, ivy, ivz, C, i, c->dRanges, dA, nullptr, c->stream, &c->launches);
    if (rc != 0) { cudaFree(dA); cudaFree(dIv); return cuda_fail(c, (cudaError_t)rc, "range kernels"); }
  }
  e = cudaStreamSynchronize(c->stream);
  cudaFree(dA);
  cudaFree(dIv);
  if (e != cudaSuccess) return cuda_fail(c, e, "range build");
  return MDWT_OK;
}

}  // namespace

// ========================================================================= C ABI
extern "C" {

int mdwt_version(void) { return (1 << 16) | 0; }

const char *mdwt_status_string(mdwt_status s) {
  switch (s) {
    case MDWT_OK: return "ok";
    case MDWT_ERR_BAD_ARG: return "bad argument";
    case MDWT_ERR_CUDA: return "CUDA error";
    case MDWT_ERR_IO: return "I/O error";
    case MDWT_ERR_TOO_MANY_CHANNELS: return "too many channels";
    case MDWT_ERR_UNSUPPORTED: return "unsupported";
    case MDWT_ERR_STATE: return "wrong call order";
    case MDWT_ERR_OOM: return "out of memory";
    case MDWT_ERR_TIMEOUT: return "device wait timed out";
    case MDWT_ERR_FORMAT: return "bad raw file name";
    case MDWT_ERR_NUMERIC: return "sample step cap reached";
    case MDWT_ERR_SCRATCH_LIMIT: return "input exceeds the fixed scratch of a no-alloc entry point";
  }
  return "unknown status";
}

const char *mdwt_last_error(const mdwt_ctx *c) { return c ? c->err.c_str() : "null context"; }

mdwt_status mdwt_create(mdwt_ctx **out, int device) {
  if (!out) return MDWT_ERR_BAD_ARG;
  *out = nullptr;
  if (device == MDWT_HOST_ONLY) {
    mdwt_ctx *h = new (std::nothrow) mdwt_ctx();
    if (!h) return MDWT_ERR_OOM;
    h->device = MDWT_HOST_ONLY;
    *out = h;
    return MDWT_OK;
  }
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n <= 0) { cudaGetLastError(); return MDWT_ERR_CUDA; }
  if (device < 0 || device >= n) return MDWT_ERR_BAD_ARG;
  mdwt_ctx *c = new (std::nothrow) mdwt_ctx();
  if (!c) return MDWT_ERR_OOM;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaDeviceGetAttribute(&c->numSMs, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->dCounters, 8 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&c->dWork, 64) != cudaSuccess ||
      cudaMemset(c->dCounters, 0, 8 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->dCounters) cudaFree(c->dCounters);
    if (c->dWork) cudaFree(c->dWork);
    delete c;
    return MDWT_ERR_CUDA;
  }
  *out = c;
  return MDWT_OK;
}

mdwt_status mdwt_destroy(mdwt_ctx *c) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (c->device == MDWT_HOST_ONLY) { delete c; return MDWT_OK; }
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  free_device(c);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return MDWT_OK;
}

mdwt_status mdwt_push_channel(mdwt_ctx *c, const void *data, int fmt, const int64_t dims[3]) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (!data || !dims || dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0)
    return fail(c, MDWT_ERR_BAD_ARG, "null data or non-positive dims");
  if (dims[0] > (1 << 20) || dims[1] > (1 << 20) || dims[2] > (1 << 20))
    return fail(c, MDWT_ERR_BAD_ARG, "dimension above 2^20");
  if (fmt_bytes(fmt) == 0) return fail(c, MDWT_ERR_UNSUPPORTED, "unspecified voxel format");
  return push_common(c, data, fmt, dims);
}

mdwt_status mdwt_push_channel_raw(mdwt_ctx *c, const char *path) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (!path) return fail(c, MDWT_ERR_BAD_ARG, "null path");
  int64_t dims[3];
  int fmt;
  if (!parse_raw_name(path, dims, fmt)) return fail(c, MDWT_ERR_FORMAT, std::string("no <X>x<Y>x<Z> token in ") + path);
  const int bpv = fmt_bytes(fmt);
  if (bpv == 0) return fail(c, MDWT_ERR_FORMAT, std::string("no voxel type token in ") + path);
  const size_t n = (size_t)(dims[0] * dims[1] * dims[2]);
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(c, MDWT_ERR_IO, std::string("cannot open ") + path);
  std::vector<char> buf;
  try {
    buf.resize(n * bpv);
  } catch (const std::bad_alloc &) {
    std::fclose(f);
    return fail(c, MDWT_ERR_OOM, "host allocation failed");
  }
  const size_t got = std::fread(buf.data(), 1, buf.size(), f);
  std::fclose(f);
  if (got != buf.size()) return fail(c, MDWT_ERR_IO, std::string("truncated raw file ") + path);
  return push_common(c, buf.data(), fmt, dims);
}

mdwt_status mdwt_reshape_bounds(mdwt_ctx *c, int chn, const float *scale3) {
  mdwt_status s = check_ch(c, chn);
  if (s) return s;
  if (c->inited) return fail(c, MDWT_ERR_STATE, "reshape bounds before mdwt_init");
  Channel &h = c->ch[chn];
  for (int a = 0; a < 3; a++) {
    const float k = scale3 ? scale3[a] : (float)h.dims[a];
    h.lo[a] = h.lo[a] * k;
    h.hi[a] = h.hi[a] * k;
  }
  return MDWT_OK;
}

mdwt_status mdwt_num_channels(const mdwt_ctx *c, int *n) {
  if (!c || !n) return MDWT_ERR_BAD_ARG;
  *n = (int)c->ch.size();
  return MDWT_OK;
}

mdwt_status mdwt_get_channel_info(const mdwt_ctx *c, int chn, int64_t dims[3], float b8[8]) {
  if (!c || chn < 0 || chn >= (int)c->ch.size() || !dims || !b8) return MDWT_ERR_BAD_ARG;
  for (int a = 0; a < 3; a++) dims[a] = c->ch[chn].dims[a];
  for (int a = 0; a < 4; a++) { b8[a] = c->ch[chn].lo[a]; b8[4 + a] = c->ch[chn].hi[a]; }
  return MDWT_OK;
}

static mdwt_status regrid(mdwt_ctx *c);

mdwt_status mdwt_set_macrocells(mdwt_ctx *c, const uint32_t d[3]) {
  if (!c || !d) return MDWT_ERR_BAD_ARG;
  for (int a = 0; a < 3; a++) c->mcReq[a] = d[a];
  if (c->inited) return regrid(c);   // after init: new grid, same transfer functions
  return MDWT_OK;
}

mdwt_status mdwt_init(mdwt_ctx *c, int mode, int auto_camera) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (c->inited) return fail(c, MDWT_ERR_STATE, "already initialised");
  if (c->ch.empty()) return fail(c, MDWT_ERR_STATE, "No data source specified (renderer.cpp:326-330)");
  if (mode < MDWT_MODE_NDDA || mode > MDWT_MODE_MIX)
    return fail(c, MDWT_ERR_UNSUPPORTED, "mode not supported (0..5 are; 6..9 are the ray marchers)");
  if (c->device == MDWT_HOST_ONLY) return fail(c, MDWT_ERR_STATE, "host-only context: no device to initialise");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  c->mode = mode;
  resolve_mc(c, c->mc);
  if (c->mc[0] == 0 || c->mc[1] == 0 || c->mc[2] == 0) return fail(c, MDWT_ERR_BAD_ARG, "zero macrocell dims");
  if ((uint64_t)c->mc[0] * c->mc[1] * c->mc[2] > (1ull << 30)) return fail(c, MDWT_ERR_BAD_ARG, "macrocell grid above 2^30 cells");
  c->M = (size_t)c->mc[0] * c->mc[1] * c->mc[2];
  // root box = union of bounds (renderer.cpp:698-716); trackers use the last channel's
  // bounds (globalBoundsLo/Hi are set in the per-channel loop, renderer.cpp:748-754)
  for (int a = 0; a < 3; a++) {
    float lo = std::numeric_limits<float>::infinity(), hi = -std::numeric_limits<float>::infinity();
    for (auto &h : c->ch) { lo = std::fmin(lo, h.lo[a]); hi = std::fmax(hi, h.hi[a]); }
    c->rootLo[a] = lo; c->rootHi[a] = hi;
  }
  for (int a = 0; a < 4; a++) { c->gLo[a] = c->ch.back().lo[a]; c->gHi[a] = c->ch.back().hi[a]; }
  // one storage kind for all channels: native uint8 only when every channel is uint8
  bool allU8 = true;
  for (auto &h : c->ch) allU8 = allU8 && h.store == kStoreU8;
  c->store = allU8 ? kStoreU8 : kStoreF32;
  for (auto &h : c->ch) {
    const size_t n = (size_t)(h.dims[0] * h.dims[1] * h.dims[2]);
    if (!allU8 && h.store == kStoreU8) {
      h.f32.resize(n);
      for (size_t i = 0; i < n; i++) h.f32[i] = (float)h.u8[i] * 255;
      h.u8.clear(); h.u8.shrink_to_fit();
      h.store = kStoreF32;
    }
    if (c->store == kStoreU8) {
      CK(cudaMalloc(&h.dVol, n), "cudaMalloc volume");
      CK(cudaMemcpyAsync(h.dVol, h.u8.data(), n, cudaMemcpyHostToDevice, c->stream), "upload volume");
    } else {
      // float32: uploaded x fastest, then rearranged into 2x2x2 micro-bricks on the device
      // (kStoreF32); the linear copy lives only for this channel's upload
      const int d3[3] = {(int)h.dims[0], (int)h.dims[1], (int)h.dims[2]};
      float *lin = nullptr;
      CK(cudaMalloc(&lin, n * 4), "cudaMalloc volume upload");
      cudaError_t e = cudaMemcpyAsync(lin, h.f32.data(), n * 4, cudaMemcpyHostToDevice, c->stream);
      if (e == cudaSuccess) e = cudaMalloc(&h.dVol, stored_voxels(kStoreF32, h.dims) * 4);
      if (e == cudaSuccess) e = (cudaError_t)launch_brick_f32(lin, (float *)h.dVol, d3, c->stream, &c->launches);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
      cudaFree(lin);
      CK(e, "micro-brick upload");
    }
  }
  const int C = (int)c->ch.size();
  CK(cudaMalloc(&c->dRanges, c->M * C * 8), "cudaMalloc ranges");
  CK(cudaMalloc(&c->dMaj, c->M * (mode >= 3 ? 1 : C) * 4), "cudaMalloc majorants");
  CK(cudaMalloc(&c->dCellTab, c->M * ((mode >= 3 ? 1 : C) + 1) * sizeof(float2)), "cudaMalloc cell table");
  c->inited = true;
  mdwt_status s = build_ranges(c);
  if (s) { c->inited = false; return s; }
  // host copies are no longer needed (the reference frees its scalar buffers too)
  for (auto &h : c->ch) { h.u8.clear(); h.u8.shrink_to_fit(); h.f32.clear(); h.f32.shrink_to_fit(); }
  c->tf.assign(C, TFState());
  c->mats.assign(C, Material());
  for (int i = 0; i < C; i++) { c->tf[i].vd[0] = c->ch[i].lo[3]; c->tf[i].vd[1] = c->ch[i].hi[3]; }
  s = recalc(c);
  if (s) return s;
  if (auto_camera) {
    const V3 center = v3(0.5f, 0.5f, 0.5f);
    const V3 eye = v3(center.x, center.y, center.z + 2.5f);
    c->cam.setOrientation(eye, center, v3(0, 1, 0), 45.0f);
  }
  update_camera(c);
  s = alloc_frame(c);
  if (s) return s;
  c->frameID = 0; c->frameParam = 0;
  reset_accum_ids(c);
  reset_dt(c);
  CK(cudaStreamSynchronize(c->stream), "init");
  return MDWT_OK;
}

mdwt_status mdwt_get_macrocell_dims(const mdwt_ctx *c, uint32_t d[3]) {
  if (!c || !d) return MDWT_ERR_BAD_ARG;
  if (c->inited) for (int a = 0; a < 3; a++) d[a] = c->mc[a];
  else resolve_mc(c, d);
  return MDWT_OK;
}

mdwt_status mdwt_set_tf(mdwt_ctx *c, int chn, const float *rgba, int n) {
  mdwt_status s = check_ch(c, chn);
  if (s) return s;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  if (!rgba || n <= 0 || n > kMaxTexels) return fail(c, MDWT_ERR_BAD_ARG, "colormap needs 1..16384 texels");
  for (int i = 0; i < 4 * n; i++)
    if (!std::isfinite(rgba[i])) return fail(c, MDWT_ERR_BAD_ARG, "colormap values must be finite");
  TFState &t = c->tf[chn];
  t.rgba.assign(rgba, rgba + 4 * (size_t)n);
  std::vector<float> alpha((size_t)n);
  for (int i = 0; i < n; i++) {
    t.rgba[4 * i + 3] = std::pow(t.rgba[4 * i + 3], 3.f);  // renderer.cpp:1100
    alpha[i] = t.rgba[4 * i + 3];
  }
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  if (t.cap < n) {
    if (t.dAlpha) cudaFree(t.dAlpha);
    if (t.dRgba) cudaFree(t.dRgba);
    t.dAlpha = t.dRgba = nullptr;
    t.cap = 0;
    CK(cudaMalloc(&t.dAlpha, (size_t)n * 4), "cudaMalloc tf");
    CK(cudaMalloc(&t.dRgba, (size_t)n * 16), "cudaMalloc tf");
    t.cap = n;
  }
  CK(cudaMemcpyAsync(t.dAlpha, alpha.data(), (size_t)n * 4, cudaMemcpyHostToDevice, c->stream), "upload tf");
  CK(cudaMemcpyAsync(t.dRgba, t.rgba.data(), (size_t)n * 16, cudaMemcpyHostToDevice, c->stream), "upload tf");
  CK(cudaStreamSynchronize(c->stream), "upload tf");
  t.n = n;
  reset_accum_ids(c);
  return recalc(c);
}

mdwt_status mdwt_set_opacity_scale(mdwt_ctx *c, int chn, float scale) {
  mdwt_status s = check_ch(c, chn);
  if (s) return s;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  if (!std::isfinite(scale)) return fail(c, MDWT_ERR_BAD_ARG, "opacity scale must be finite");
  c->tf[chn].os = scale;
  reset_accum_ids(c);
  return recalc(c);
}

mdwt_status mdwt_set_tf_range(mdwt_ctx *c, int chn, float lo, float hi) {
  mdwt_status s = check_ch(c, chn);
  if (s) return s;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  c->tf[chn].xd[0] = lo;
  c->tf[chn].xd[1] = hi;
  reset_accum_ids(c);
  return recalc(c);
}

mdwt_status mdwt_recalculate_majorants(mdwt_ctx *c) {
  if (!c) return MDWT_ERR_BAD_ARG;
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  return recalc(c);
}

mdwt_status mdwt_set_dt(mdwt_ctx *c, float dt) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (!(dt == dt)) return fail(c, MDWT_ERR_BAD_ARG, "dt is NaN");
  c->dt = std::max(dt, 1e-4f);
  reset_accum_ids(c);
  return MDWT_OK;
}
mdwt_status mdwt_reset_dt(mdwt_ctx *c) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (c->ch.empty()) return fail(c, MDWT_ERR_STATE, "no channels");
  reset_dt(c);
  return MDWT_OK;
}
mdwt_status mdwt_get_dt(const mdwt_ctx *c, float *dt) {
  if (!c || !dt) return MDWT_ERR_BAD_ARG;
  *dt = c->dt;
  return MDWT_OK;
}

mdwt_status mdwt_set_camera(mdwt_ctx *c, const float f[3], const float at[3], const float up[3], float fovy) {
  if (!c || !f || !at || !up) return MDWT_ERR_BAD_ARG;
  c->cam.setOrientation(v3(f[0], f[1], f[2]), v3(at[0], at[1], at[2]), v3(up[0], up[1], up[2]), fovy);
  update_camera(c);
  return MDWT_OK;
}

mdwt_status mdwt_get_camera_basis(const mdwt_ctx *c, float out[12]) {
  if (!c || !out) return MDWT_ERR_BAD_ARG;
  const V3 v[4] = {c->cOrg, c->cLlc, c->cHor, c->cVer};
  for (int i = 0; i < 4; i++) { out[3 * i] = v[i].x; out[3 * i + 1] = v[i].y; out[3 * i + 2] = v[i].z; }
  return MDWT_OK;
}

mdwt_status mdwt_resize(mdwt_ctx *c, int w, int h) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (w <= 0 || h <= 0 || (int64_t)w * h > (1ll << 28)) return fail(c, MDWT_ERR_BAD_ARG, "bad resolution");
  c->W = w;
  c->H = h;
  if (c->inited) {
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(c->stream), "resize");
    mdwt_status s = alloc_frame(c);
    if (s) return s;
  }
  update_camera(c);
  return MDWT_OK;
}

mdwt_status mdwt_set_spp(mdwt_ctx *c, int spp) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (spp <= 0) return fail(c, MDWT_ERR_BAD_ARG, "spp must be positive");
  c->spp = spp;
  return MDWT_OK;
}
mdwt_status mdwt_set_accumulation(mdwt_ctx *c, int e) {
  if (!c) return MDWT_ERR_BAD_ARG;
  c->accum = e != 0;
  return MDWT_OK;
}
mdwt_status mdwt_set_background(mdwt_ctx *c, const float rgb[3]) {
  if (!c || !rgb) return MDWT_ERR_BAD_ARG;
  c->bg = v3(rgb[0], rgb[1], rgb[2]);
  return MDWT_OK;
}
mdwt_status mdwt_set_light(mdwt_ctx *c, int shadows, int gradient, const float dir[3], float intensity, float ambient) {
  if (!c || !dir) return MDWT_ERR_BAD_ARG;
  // a shadow ray along a zero or non-finite direction would walk NaN distances until the
  // step cap of every sample
  const float n2 = dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2];
  if (shadows && !(n2 > 0.0f && std::isfinite(n2)))
    return fail(c, MDWT_ERR_BAD_ARG, "light direction must be finite and non-zero with shadows on");
  c->shadows = shadows != 0;
  c->gradient = gradient != 0;
  c->lightDir = v3(dir[0], dir[1], dir[2]);
  c->lightIntensity = intensity;
  c->ambient = ambient;
  reset_accum_ids(c);
  return MDWT_OK;
}
mdwt_status mdwt_set_material(mdwt_ctx *c, int chn, float di, float sp, float sh, float gs, const float rgb[3]) {
  mdwt_status s = check_ch(c, chn);
  if (s) return s;
  if (!rgb) return fail(c, MDWT_ERR_BAD_ARG, "null colour");
  if (chn >= (int)c->mats.size()) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  Material &m = c->mats[chn];
  m.diffuse = di; m.specular = sp; m.shininess = sh; m.gradStep = gs;
  m.spec = v3(rgb[0], rgb[1], rgb[2]);
  reset_accum_ids(c);
  return MDWT_OK;
}
mdwt_status mdwt_set_mirror(mdwt_ctx *c, int e) {
  if (!c) return MDWT_ERR_BAD_ARG;
  c->mirror = e != 0;
  return MDWT_OK;
}

mdwt_status mdwt_set_seed_block(mdwt_ctx *c, int edge) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (edge == 0) { c->seedMask = 0xffffffffu; return MDWT_OK; }
  if (edge < 1 || edge > 1024 || (edge & (edge - 1)) != 0)
    return fail(c, MDWT_ERR_BAD_ARG, "seed block edge must be 0 or a power of two in 1..1024");
  c->seedMask = (uint32_t)edge - 1u;
  return MDWT_OK;
}

mdwt_status mdwt_set_arithmetic(mdwt_ctx *c, int arith) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (arith != MDWT_ARITH_EXACT && arith != MDWT_ARITH_FAST)
    return fail(c, MDWT_ERR_BAD_ARG, "arithmetic must be MDWT_ARITH_EXACT or MDWT_ARITH_FAST");
  if (arith == c->arith) return MDWT_OK;
  c->arith = arith;
  if (!c->inited) return MDWT_OK;
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  return recalc(c);   // the cell table's reciprocals follow the arithmetic
}

mdwt_status mdwt_get_arithmetic(const mdwt_ctx *c, int *arith) {
  if (!c || !arith) return MDWT_ERR_BAD_ARG;
  *arith = c->arith;
  return MDWT_OK;
}

// Depth-feature scale: 1 / (distance from the camera to the root-box centre + the box
// diagonal), so that hit distances map into [0, 1].
static float feature_scale(const mdwt_ctx *c) {
  const float cx = (c->rootLo[0] + c->rootHi[0]) * 0.5f, cy = (c->rootLo[1] + c->rootHi[1]) * 0.5f,
              cz = (c->rootLo[2] + c->rootHi[2]) * 0.5f;
  const float dx = c->cOrg.x - cx, dy = c->cOrg.y - cy, dz = c->cOrg.z - cz;
  const float ex = c->rootHi[0] - c->rootLo[0], ey = c->rootHi[1] - c->rootLo[1], ez = c->rootHi[2] - c->rootLo[2];
  return 1.0f / (std::sqrt(dx * dx + dy * dy + dz * dz) + std::sqrt(ex * ex + ey * ey + ez * ez));
}

// Scene, camera, transfer functions and shading of the next frame.
// Whether frames run the regrouped tracker (MDWT_TUNE_REGROUP): as set, or by default for
// syncDDA only -- for N-DDA on the 1080p 6 x 512^3 float32 scene the warp-local tracker
// measured faster with 16-voxel macrocells (2.22 vs 2.07 Gpath/s) and the regrouped one
// with 32-voxel macrocells; the schedule autotuner picks per scene.
static int regroup_on(const mdwt_ctx *c) { return c->regroup >= 0 ? c->regroup : (c->mode == 2 ? 1 : 0); }

static void fill_scene(const mdwt_ctx *c, TrackParams &p) {
  std::memset(&p, 0, sizeof(p));
  p.W = c->W; p.H = c->H; p.spp = c->spp;
  p.frameParam = (uint32_t)c->frameParam;
  p.accumParam = (uint32_t)c->accumParam;
  p.accumulate = c->accum ? 1 : 0;
  p.mirror = c->mirror ? 1 : 0;
  p.seedMask = c->seedMask;
  p.fast = c->arith == MDWT_ARITH_FAST ? 1 : 0;
  p.bg = f3(c->bg);
  p.camOrg = f3(c->cOrg); p.camLlc = f3(c->cLlc); p.camHor = f3(c->cHor); p.camVer = f3(c->cVer);
  p.rootLo = {c->rootLo[0], c->rootLo[1], c->rootLo[2]};
  p.rootHi = {c->rootHi[0], c->rootHi[1], c->rootHi[2]};
  p.gLo = {c->gLo[0], c->gLo[1], c->gLo[2]};
  p.gHi = {c->gHi[0], c->gHi[1], c->gHi[2]};
  p.w2u = {1.f / (c->gHi[0] - c->gLo[0]), 1.f / (c->gHi[1] - c->gLo[1]), 1.f / (c->gHi[2] - c->gLo[2])};
  p.gScale = {(float)c->mc[0] * p.w2u.x, (float)c->mc[1] * p.w2u.y, (float)c->mc[2] * p.w2u.z};
  for (int a = 0; a < 3; a++) p.mc[a] = c->mc[a];
  p.C = (int)c->ch.size();
  p.mode = c->mode;
  p.dt = c->dt;
  p.majorants = c->dMaj;
  p.cellTab = c->dCellTab;
  p.tabStride = (c->mode >= 3 ? 1 : p.C) + 1;
  for (int i = 0; i < p.C; i++) {
    p.vol[i] = c->ch[i].dVol;
    for (int a = 0; a < 3; a++) p.dims[i][a] = (int)c->ch[i].dims[a];
    const TFState &t = c->tf[i];
    p.tfAlpha[i] = t.dAlpha;
    p.tfRgba[i] = t.dRgba;
    p.tfN[i] = t.n;
    p.vd[i][0] = t.vd[0]; p.vd[i][1] = t.vd[1];
    p.xd[i][0] = t.xd[0]; p.xd[i][1] = t.xd[1];
    p.os[i] = t.os;
    p.matSpec[i] = f3(c->mats[i].spec);
    p.matDiffuse[i] = c->mats[i].diffuse;
    p.matSpecular[i] = c->mats[i].specular;
    p.matShininess[i] = c->mats[i].shininess;
    p.matGradStep[i] = c->mats[i].gradStep;
  }
  p.lightIntensity = c->lightIntensity;
  p.ambient = c->ambient;
  p.shadows = c->shadows ? 1 : 0;
  p.gradient = c->gradient ? 1 : 0;
  p.lightDir = f3(c->lightDir);
}

// Everything a frame's kernels need: parameters, the traced rectangle, record buffers
// (grown as needed); *batchOut = samples per record batch.
static mdwt_status prepare_frame(mdwt_ctx *c, TrackParams &p, int *batchOut) {
  fill_scene(c, p);
  p.accum = c->dAccum;
  p.fb = c->dFb;
  p.stats = c->statsOn ? c->dStats : nullptr;
  p.counters = c->dCounters;
  p.workCounter = c->dWork;
  int rect[4];
  cull_rect(c, rect);
  // a row band (mdwt_set_render_rows) restricts tracing and resolve to its rows
  p.rowLo = std::max(0, std::min(c->H, c->rowLo));
  p.rowHi = c->rowHi > c->rowLo ? std::max(p.rowLo, std::min(c->H, c->rowHi)) : c->H;
  if (c->rowHi <= c->rowLo) p.rowLo = 0;
  rect[1] = std::max(rect[1], p.rowLo);
  rect[3] = std::min(rect[3], p.rowHi - 1);
  p.cullX0 = rect[0]; p.cullY0 = rect[1]; p.cullX1 = rect[2]; p.cullY1 = rect[3];
  const int rw = rect[2] - rect[0] + 1, rh = rect[3] - rect[1] + 1;
  p.tilesX = rw > 0 ? (rw + 7) / 8 : 0;
  p.numTiles = (rw > 0 && rh > 0) ? p.tilesX * ((rh + 3) / 4) : 0;
  background_result(c, p.bgFin);
  p.gOrg = {p.gScale.x * (c->cOrg.x - p.gLo.x), p.gScale.y * (c->cOrg.y - p.gLo.y), p.gScale.z * (c->cOrg.z - p.gLo.z)};
  p.pool = c->pool;
  p.trips = c->trips;
  p.quorum = c->quorum;
  p.regroup = regroup_on(c);
  p.rgBlocks = c->rgBlocks;
  p.store = c->store;
  p.vol32 = 1;
  for (auto &h : c->ch)
    if ((uint64_t)stored_voxels(c->store, h.dims) >= (1ull << 32)) p.vol32 = 0;
  // samples in batches whose path records fit the record budget; the resolve pass
  // carries the per-pixel running sums across batches in sample order
  const size_t nrect = p.numTiles > 0 ? (size_t)rw * (size_t)rh : 0;
  int batch = c->spp;
  if (nrect > 0 && (size_t)batch * nrect > kRecordBudget) batch = (int)std::max<size_t>(1, kRecordBudget / nrect);
  if (c->batchCap > 0) batch = std::min(batch, c->batchCap);
  const bool stats = c->statsOn;
  mdwt_status s = MDWT_OK;
  (void)s;
  if (nrect > 0) {
    if ((s = grow(c, (void **)&c->dRec, c->recCap, (size_t)batch * nrect * 4, "records")) != MDWT_OK) return s;
    if (stats && (s = grow(c, (void **)&c->dRecStats, c->recStatsCap, (size_t)batch * nrect * 4, "record stats")) != MDWT_OK) return s;
    if ((c->gradient || c->featOn || c->mode >= MDWT_MODE_MAX) &&
        (s = grow(c, (void **)&c->dRecT, c->recTCap, (size_t)batch * nrect * 4, "hit distances")) != MDWT_OK)
      return s;
    if (batch < c->spp) {
      if ((s = grow(c, (void **)&c->dPartial, c->partialCap, nrect * 16, "partial sums")) != MDWT_OK) return s;
      if (stats && (s = grow(c, (void **)&c->dPartialStats, c->partialStatsCap, nrect * 16, "partial stats")) != MDWT_OK) return s;
    }
  }
  p.records = c->dRec;
  p.recStats = stats ? c->dRecStats : nullptr;
  // hit distances: gradient shading, features, and the blending modes (the resolve pass
  // recomputes the blended colour at the hit)
  p.recT = (c->gradient || c->featOn || c->mode >= MDWT_MODE_MAX) ? c->dRecT : nullptr;
  if (c->featOn) {
    if (batch < c->spp || c->spp > 65535)
      return fail(c, MDWT_ERR_UNSUPPORTED, "denoiser features need the frame in one sample batch and spp < 65536");
    if ((s = grow(c, (void **)&c->dFeat, c->featCap, (size_t)c->W * c->H * 16 * sizeof(float), "features")) != MDWT_OK)
      return s;
    p.feat = c->dFeat;
    p.featScale = feature_scale(c);
  }
  p.partial = c->dPartial;
  p.partialStats = stats ? c->dPartialStats : nullptr;
  p.nFrames = 1;
  *batchOut = batch;
  return MDWT_OK;
}

// Frames traced per launch by mdwt_render_frames: their path records fit the budget.
static int frames_per_launch(const TrackParams &p, int spp, int n) {
  const int rw = p.cullX1 - p.cullX0 + 1, rh = p.cullY1 - p.cullY0 + 1;
  const size_t nrect = p.numTiles > 0 ? (size_t)rw * (size_t)rh : 0;
  if (nrect == 0) return n;
  const size_t g = kRecordBudget / (nrect * (size_t)spp);
  return (int)std::min<size_t>((size_t)n, g);
}

mdwt_status mdwt_render(mdwt_ctx *c, void *stream) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  TrackParams p;
  int batch = 0;
  mdwt_status s = prepare_frame(c, p, &batch);
  if (s) return s;
  // kernel timing: events around the trace and the resolve kernel of every sample pass
  // of the frame (frames of up to kTimedPasses passes)
  const int passes = (c->spp + batch - 1) / batch;
  const bool timeIt = c->timing && passes <= mdwt_ctx::kTimedPasses;
  c->timed = false;
  if (timeIt) {
    for (int i = 0; i < 3 * passes; i++)
      if (!c->ev[i]) CK(cudaEventCreate(&c->ev[i]), "cudaEventCreate");
  }
  for (int s0 = 0, b = 0; s0 < c->spp; s0 += batch, b++) {
    p.sBase = s0;
    p.sCount = std::min(batch, c->spp - s0);
    if (timeIt) CK(cudaEventRecord(c->ev[3 * b], st), "event");
    CK(cudaMemsetAsync(c->dWork, 0, sizeof(unsigned int), st), "reset work counter");
    CKI(launch_track(p, c->store, st, c->numSMs, &c->launches, &c->lastGrid, &c->lastBlock,
                     timeIt ? c->ev[3 * b + 1] : nullptr),
        "tracker kernels");
    if (timeIt) CK(cudaEventRecord(c->ev[3 * b + 2], st), "event");
  }
  if (timeIt) {
    c->timedPasses = passes;
    c->timed = true;
  }
  // Renderer::Render (renderer.cpp:957-958): the ids the next frame sees are the
  // pre-increment values
  c->accumParam = c->accumID++;
  c->frameParam = c->frameID++;
  return MDWT_OK;
}

mdwt_status mdwt_set_features(mdwt_ctx *c, int enable) {
  if (!c) return MDWT_ERR_BAD_ARG;
  c->featOn = enable != 0;
  return MDWT_OK;
}

mdwt_status mdwt_get_features(mdwt_ctx *c, float *out) {
  if (!c || !out) return MDWT_ERR_BAD_ARG;
  if (!c->featOn || !c->dFeat) return fail(c, MDWT_ERR_STATE, "mdwt_set_features(1) and a frame first");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  CK(cudaDeviceSynchronize(), "sync");
  CK(cudaMemcpy(out, c->dFeat, (size_t)c->W * c->H * 16 * sizeof(float), cudaMemcpyDeviceToHost), "copy features");
  return MDWT_OK;
}

mdwt_status mdwt_copy_features(mdwt_ctx *c, void *dst, void *stream) {
  if (!c || !dst) return MDWT_ERR_BAD_ARG;
  if (!c->featOn || !c->dFeat) return fail(c, MDWT_ERR_STATE, "mdwt_set_features(1) and a frame first");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  CK(cudaMemcpyAsync(dst, c->dFeat, (size_t)c->W * c->H * 16 * sizeof(float), cudaMemcpyDeviceToDevice,
                     stream ? (cudaStream_t)stream : c->stream),
     "copy features");
  return MDWT_OK;
}

mdwt_status mdwt_get_device_features(mdwt_ctx *c, void **feat) {
  if (!c || !feat) return MDWT_ERR_BAD_ARG;
  *feat = c->featOn ? c->dFeat : nullptr;
  return MDWT_OK;
}

mdwt_status mdwt_render_expected(mdwt_ctx *c, int jitter, float step_voxels, void *stream) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  if (jitter <= 0 || jitter > 1024 || !(step_voxels > 0.0f) || !std::isfinite(step_voxels))
    return fail(c, MDWT_ERR_BAD_ARG, "jitter in [1, 1024] and a positive step");
  if (c->shadows || c->gradient) return fail(c, MDWT_ERR_UNSUPPORTED, "expected image of the unshaded estimator only");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  TrackParams p;
  fill_scene(c, p);
  double h0 = 1e300;   // step: step_voxels times the smallest voxel edge in world units
  for (auto &h : c->ch)
    for (int a = 0; a < 3; a++) h0 = std::min(h0, ((double)h.hi[a] - (double)h.lo[a]) / (double)h.dims[a]);
  h0 *= (double)step_voxels;
  const size_t bytes = (size_t)c->W * c->H * 3 * sizeof(double);
  mdwt_status s = grow(c, (void **)&c->dExpected, c->expectedCap, bytes, "expected image");
  if (s != MDWT_OK) return s;
  CKI(launch_expected(p, c->store, jitter, h0, c->dExpected, st, c->numSMs, &c->launches), "expected image kernel");
  c->expectedValid = true;
  c->expW = c->W;
  c->expH = c->H;
  return MDWT_OK;
}

mdwt_status mdwt_get_expected(mdwt_ctx *c, double *out) {
  if (!c || !out) return MDWT_ERR_BAD_ARG;
  if (!c->expectedValid || c->expW != c->W || c->expH != c->H)
    return fail(c, MDWT_ERR_STATE, "mdwt_render_expected first (at the current size)");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  CK(cudaDeviceSynchronize(), "sync");
  CK(cudaMemcpy(out, c->dExpected, (size_t)c->W * c->H * 3 * sizeof(double), cudaMemcpyDeviceToHost), "copy expected");
  return MDWT_OK;
}

mdwt_status mdwt_accum_rmse(mdwt_ctx *c, double *rmse) {
  if (!c || !rmse) return MDWT_ERR_BAD_ARG;
  if (!c->expectedValid || c->expW != c->W || c->expH != c->H)
    return fail(c, MDWT_ERR_STATE, "mdwt_render_expected first (at the current size)");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  if (!c->dSqSum) CK(cudaMalloc((void **)&c->dSqSum, sizeof(double)), "rmse scratch");
  CK(cudaMemsetAsync(c->dSqSum, 0, sizeof(double), c->stream), "rmse scratch");
  const size_t npix = (size_t)c->W * c->H;
  CKI(launch_rmse(c->dAccum, c->dExpected, npix, c->dSqSum, c->stream, c->numSMs, &c->launches), "rmse kernel");
  double sum = 0.0;
  CK(cudaMemcpyAsync(&sum, c->dSqSum, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "rmse copy");
  CK(cudaStreamSynchronize(c->stream), "rmse sync");
  *rmse = std::sqrt(sum / (3.0 * (double)npix));
  return MDWT_OK;
}

mdwt_status mdwt_denoise(mdwt_ctx *c, mdwt_denoiser *d, float *out) {
  if (!c || !d || !out) return MDWT_ERR_BAD_ARG;
  if (!c->featOn || !c->dFeat) return fail(c, MDWT_ERR_STATE, "mdwt_set_features(1) and a frame first");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  const mdwt_status s = mdwt_denoiser_infer(d, c->dFeat, out, 1, c->H, c->W, c->stream);
  if (s != MDWT_OK) return fail(c, s, std::string("denoiser: ") + mdwt_denoiser_last_error(d));
  return MDWT_OK;
}

mdwt_status mdwt_image_rmse(mdwt_ctx *c, const float *img, double *rmse) {
  if (!c || !img || !rmse) return MDWT_ERR_BAD_ARG;
  if (!c->expectedValid || c->expW != c->W || c->expH != c->H)
    return fail(c, MDWT_ERR_STATE, "mdwt_render_expected first (at the current size)");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  if (!c->dSqSum) CK(cudaMalloc((void **)&c->dSqSum, sizeof(double)), "rmse scratch");
  CK(cudaMemsetAsync(c->dSqSum, 0, sizeof(double), c->stream), "rmse scratch");
  const size_t npix = (size_t)c->W * c->H;
  CKI(launch_rmse(img, c->dExpected, npix, c->dSqSum, c->stream, c->numSMs, &c->launches), "rmse kernel");
  double sum = 0.0;
  CK(cudaMemcpyAsync(&sum, c->dSqSum, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "rmse copy");
  CK(cudaStreamSynchronize(c->stream), "rmse sync");
  *rmse = std::sqrt(sum / (3.0 * (double)npix));
  return MDWT_OK;
}

// ------------------------------------------------------------------ macrocell regrid
// The value ranges and majorants of a new macrocell grid, transfer functions kept;
// resets the accumulation like a transfer-function change.
static mdwt_status regrid(mdwt_ctx *c) {
  uint32_t mc[3];
  resolve_mc(c, mc);
  if (mc[0] == 0 || mc[1] == 0 || mc[2] == 0) return fail(c, MDWT_ERR_BAD_ARG, "zero macrocell dims");
  if ((uint64_t)mc[0] * mc[1] * mc[2] > (1ull << 30)) return fail(c, MDWT_ERR_BAD_ARG, "macrocell grid above 2^30 cells");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(c->stream), "regrid");
  if (c->dRanges) cudaFree(c->dRanges);
  if (c->dMaj) cudaFree(c->dMaj);
  if (c->dCellTab) cudaFree(c->dCellTab);
  c->dRanges = nullptr; c->dMaj = nullptr; c->dCellTab = nullptr;
  for (int a = 0; a < 3; a++) c->mc[a] = mc[a];
  c->M = (size_t)mc[0] * mc[1] * mc[2];
  const int C = (int)c->ch.size();
  CK(cudaMalloc(&c->dRanges, c->M * C * 8), "cudaMalloc ranges");
  CK(cudaMalloc(&c->dMaj, c->M * (c->mode >= 3 ? 1 : C) * 4), "cudaMalloc majorants");
  CK(cudaMalloc(&c->dCellTab, c->M * ((c->mode >= 3 ? 1 : C) + 1) * sizeof(float2)), "cudaMalloc cell table");
  mdwt_status s = build_ranges(c);
  if (s) return s;
  s = recalc(c);
  if (s) return s;
  reset_accum_ids(c);
  CK(cudaStreamSynchronize(c->stream), "regrid");
  return MDWT_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ batches
struct mdwt_batch {
  int device = 0, numSMs = 0;
  cudaStream_t stream = nullptr;
  std::vector<mdwt_ctx *> reqs;
  int unitItems = 0, pool = 0, trips = 0;   // unitItems: dispenser chunk (0 = sized per request)
  bool useGraph = true;
  bool fuse = false;                         // regroupable requests share one launch (mdwt_batch_set_fusion)
  // pinned host staging and device copies: params, units, pixel offsets, unit counters
  TrackParams *hParams = nullptr, *dParams = nullptr;
  unsigned long long *hPix = nullptr, *dPix = nullptr;
  unsigned *dDisp = nullptr;                 // one work dispenser per request
  size_t capParams = 0, capPix = 0, capDisp = 0;
  cudaGraphExec_t graph = nullptr;
  std::vector<long long> graphSig;
  cudaStream_t graphStream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int64_t launches = 0, replays = 0, captures = 0, lastUnitsLaunch = 0;
  int lastGroups = 0, lastUnits = 0, lastTraceLaunches = 0;
  std::string err;
};

namespace {

mdwt_status bfail(mdwt_batch *b, mdwt_status s, const std::string &m) {
  if (b) b->err = m;
  return s;
}
#define BCK(call, what)                                                                         \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) return bfail(b, MDWT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
mdwt_status grow_pair(mdwt_batch *b, T **h, T **d, size_t &cap, size_t n) {
  if (n <= cap && *d) return MDWT_OK;
  if (*h) cudaFreeHost(*h);
  if (*d) cudaFree(*d);
  *h = nullptr; *d = nullptr; cap = 0;
  const size_t m = n < 16 ? 16 : n;
  BCK(cudaMallocHost((void **)h, m * sizeof(T)), "pinned staging");
  BCK(cudaMalloc((void **)d, m * sizeof(T)), "batch buffers");
  cap = m;
  if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; b->graphSig.clear(); }   // pointers baked
  return MDWT_OK;
}

struct GroupPlan {
  int mode, store;
  bool stats, ext, shade, regroup;
  int first, count;           // request slots [first, first + count) of the params array
  int pixFirst;               // offset of the group's nReq + 1 pixel offsets
  unsigned long long totalItems, totalPix;
};

// Kernel variant of a batched request; the regroupable variants sort first (bit 40 clear)
// so that they form one prefix of the batch, which a fused launch covers.
long long variant_key(const TrackParams &p, int store, bool stats) {
  const bool ext = p.shadows || p.recT;
  const bool shade = p.shadows || p.gradient;
  const bool rg = !stats && !ext && regroup_fits(p);
  return (rg ? 0LL : (1LL << 40)) + (long long)p.mode * 32 + (rg ? 16 : 0) + store * 8 + (stats ? 4 : 0) +
         (ext ? 2 : 0) + (shade ? 1 : 0);
}

}  // namespace

extern "C" {

mdwt_status mdwt_batch_create(mdwt_batch **out, int device) {
  if (!out) return MDWT_ERR_BAD_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return MDWT_ERR_CUDA;
  if (device < 0 || device >= count) return MDWT_ERR_BAD_ARG;
  mdwt_batch *b = new mdwt_batch();
  b->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess) {
    delete b;
    return MDWT_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&b->numSMs, cudaDevAttrMultiProcessorCount, device);
  *out = b;
  return MDWT_OK;
}

mdwt_status mdwt_batch_destroy(mdwt_batch *b) {
  if (!b) return MDWT_ERR_BAD_ARG;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->hParams) cudaFreeHost(b->hParams);
  if (b->dParams) cudaFree(b->dParams);
  if (b->hPix) cudaFreeHost(b->hPix);
  if (b->dPix) cudaFree(b->dPix);
  if (b->dDisp) cudaFree(b->dDisp);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->graphStream) cudaStreamDestroy(b->graphStream);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return MDWT_OK;
}

const char *mdwt_batch_last_error(const mdwt_batch *b) { return b ? b->err.c_str() : "null batch"; }

mdwt_status mdwt_batch_add(mdwt_batch *b, mdwt_ctx *c) {
  if (!b || !c) return MDWT_ERR_BAD_ARG;
  if (!c->inited) return bfail(b, MDWT_ERR_STATE, "request not initialised");
  if (c->device != b->device) return bfail(b, MDWT_ERR_BAD_ARG, "request on another device");
  for (auto *r : b->reqs)   // one frame per request and batch frame: its buffers are per context
    if (r == c) return bfail(b, MDWT_ERR_BAD_ARG, "request already in the batch");
  b->reqs.push_back(c);
  return MDWT_OK;
}

mdwt_status mdwt_batch_clear(mdwt_batch *b) {
  if (!b) return MDWT_ERR_BAD_ARG;
  b->reqs.clear();
  return MDWT_OK;
}

mdwt_status mdwt_batch_set_schedule(mdwt_batch *b, int unitItems, int pool, int trips) {
  if (!b || unitItems < 0 || (unitItems % 32) || pool < 0 || pool > 32 || trips < 0 || trips > 64)
    return MDWT_ERR_BAD_ARG;
  if (unitItems) b->unitItems = unitItems;   // dispenser chunk for every request
  if (pool) b->pool = pool;
  if (trips) b->trips = trips;
  return MDWT_OK;
}

mdwt_status mdwt_batch_set_graph(mdwt_batch *b, int enable) {
  if (!b) return MDWT_ERR_BAD_ARG;
  b->useGraph = enable != 0;
  return MDWT_OK;
}

mdwt_status mdwt_batch_set_fusion(mdwt_batch *b, int enable) {
  if (!b) return MDWT_ERR_BAD_ARG;
  b->fuse = enable != 0;
  return MDWT_OK;
}

mdwt_status mdwt_batch_render(mdwt_batch *b, void *stream) {
  if (!b) return MDWT_ERR_BAD_ARG;
  if (b->reqs.empty()) return bfail(b, MDWT_ERR_STATE, "empty batch");
  BCK(cudaSetDevice(b->device), "cudaSetDevice");
  const int n = (int)b->reqs.size();
  // per-request frame parameters, in variant order
  std::vector<TrackParams> ps(n);
  std::vector<long long> keys(n);
  for (int i = 0; i < n; i++) {
    mdwt_ctx *c = b->reqs[i];
    int batch = 0;
    if (c->rowHi > c->rowLo) return bfail(b, MDWT_ERR_UNSUPPORTED, "batched requests render all rows");
    mdwt_status s = prepare_frame(c, ps[i], &batch);
    if (s) return bfail(b, s, std::string("request ") + std::to_string(i) + ": " + c->err);
    if (batch < c->spp) return bfail(b, MDWT_ERR_UNSUPPORTED, "a batched request's frame exceeds one record batch");
    ps[i].sBase = 0;          // the whole frame is one sample batch
    ps[i].sCount = c->spp;
    if (b->pool) ps[i].pool = b->pool;
    if (b->trips) ps[i].trips = b->trips;
    keys[i] = variant_key(ps[i], c->store, c->statsOn);
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return keys[a] < keys[c]; });
  // groups, dispenser chunks, pixel offsets
  std::vector<GroupPlan> groups;
  std::vector<unsigned long long> pix;
  for (int k = 0; k < n;) {
    int e = k;
    while (e < n && keys[order[e]] == keys[order[k]]) e++;
    const TrackParams &p0 = ps[order[k]];
    GroupPlan g;
    g.mode = p0.mode; g.store = b->reqs[order[k]]->store; g.stats = b->reqs[order[k]]->statsOn;
    g.ext = p0.shadows || p0.recT; g.shade = p0.shadows || p0.gradient;
    g.regroup = !g.stats && !g.ext && regroup_fits(p0);   // the whole group, by its key
    g.first = k; g.count = e - k;
    g.pixFirst = (int)pix.size();
    // the group's persistent grid: chunks sized like the single-request launch
    const size_t warps = (size_t)b->numSMs * batch_trace_occupancy(g.mode, g.store, g.stats, g.ext) * 4;
    unsigned long long acc = 0, items = 0;
    for (int j = k; j < e; j++) {
      TrackParams &p = ps[order[j]];
      pix.push_back(acc);
      acc += (unsigned long long)p.W * p.H;
      const size_t it = (size_t)p.numTiles * 32u * (size_t)p.spp;
      items += it;
      size_t chunk = b->unitItems > 0 ? (size_t)b->unitItems : it / (warps * 8);
      chunk = chunk < 32 ? 32 : (chunk > 256 && b->unitItems <= 0 ? 256 : chunk & ~(size_t)31);
      p.chunk = (int)chunk;
    }
    pix.push_back(acc);
    g.totalPix = acc;
    g.totalItems = items;
    groups.push_back(g);
    k = e;
  }
  // the regroupable prefix (its groups come first in key order): one fused launch with
  // pixel offsets over all its requests
  int nFused = 0, fusedGroups = 0, fusedPixFirst = 0;
  unsigned long long fusedItems = 0, fusedPix = 0;
  if (b->fuse) {
    for (auto &g : groups) {
      if (!g.regroup) break;
      nFused += g.count;
      fusedGroups++;
      fusedItems += g.totalItems;
    }
    if (fusedGroups >= 1) {
      fusedPixFirst = (int)pix.size();
      for (int j = 0; j < nFused; j++) {
        pix.push_back(fusedPix);
        fusedPix += (unsigned long long)ps[order[j]].W * ps[order[j]].H;
      }
      pix.push_back(fusedPix);
    }
  }
  mdwt_status s;
  if ((s = grow_pair(b, &b->hParams, &b->dParams, b->capParams, (size_t)n))) return s;
  if ((s = grow_pair(b, &b->hPix, &b->dPix, b->capPix, pix.size()))) return s;
  if (b->capDisp < (size_t)n) {
    if (b->dDisp) cudaFree(b->dDisp);
    b->dDisp = nullptr;
    BCK(cudaMalloc((void **)&b->dDisp, std::max<size_t>(64, n) * sizeof(unsigned)), "dispensers");
    b->capDisp = std::max<size_t>(64, n);
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; b->graphSig.clear(); }
  }
  for (int j = 0; j < n; j++) b->hParams[j] = ps[order[j]];
  std::copy(pix.begin(), pix.end(), b->hPix);
  // structure signature: what a captured graph bakes in
  std::vector<long long> sig = {n, (long long)pix.size(), (long long)b->numSMs, (long long)fusedGroups};
  for (auto &g : groups) {
    sig.push_back(keys[order[g.first]]);
    sig.push_back(g.count);
    sig.push_back((long long)(g.totalItems > 0));
    sig.push_back((long long)g.totalPix);
  }
  cudaStream_t user = stream ? (cudaStream_t)stream : b->stream;
  auto enqueue = [&](cudaStream_t st) -> mdwt_status {
    BCK(cudaMemcpyAsync(b->dParams, b->hParams, (size_t)n * sizeof(TrackParams), cudaMemcpyHostToDevice, st), "params");
    BCK(cudaMemcpyAsync(b->dPix, b->hPix, pix.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice, st), "pix");
    BCK(cudaMemsetAsync(b->dDisp, 0, (size_t)n * sizeof(unsigned), st), "dispensers");
    if (fusedGroups >= 1) {   // every regroupable request: one trace launch, one resolve launch
      int launches = 0, grid = 0;
      const int rc = launch_track_batch_fused(b->dParams, nFused, b->dDisp, fusedItems, b->dPix + fusedPixFirst,
                                              fusedPix, st, b->numSMs, &launches, &grid);
      if (rc) return bfail(b, MDWT_ERR_CUDA, std::string("batched tracker: ") + cudaGetErrorString((cudaError_t)rc));
      b->launches += launches;
    }
    for (size_t gi = (size_t)fusedGroups; gi < groups.size(); gi++) {
      const GroupPlan &g = groups[gi];
      BatchGroup bg;
      bg.mode = g.mode; bg.storeKind = g.store; bg.stats = g.stats; bg.ext = g.ext; bg.shade = g.shade;
      bg.regroup = g.regroup;
      bg.reqs = b->dParams + g.first;
      bg.nReq = g.count;
      bg.dispensers = b->dDisp + g.first;
      bg.totalItems = g.totalItems;
      bg.pixOfs = b->dPix + g.pixFirst;
      bg.totalPix = g.totalPix;
      int launches = 0, grid = 0;
      const int rc = launch_track_batch(bg, st, b->numSMs, &launches, &grid);
      if (rc) return bfail(b, MDWT_ERR_CUDA, std::string("batched tracker: ") + cudaGetErrorString((cudaError_t)rc));
      b->launches += launches;
    }
    return MDWT_OK;
  };
  BCK(cudaEventRecord(b->ev0, user), "event");
  if (b->useGraph) {
    if (!b->graph || b->graphSig != sig) {
      if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
      cudaStream_t cs = b->stream;
      if (cs == user) {   // capture on a private stream, replay on the caller's
        if (!b->graphStream) BCK(cudaStreamCreateWithFlags(&b->graphStream, cudaStreamNonBlocking), "stream");
        cs = b->graphStream;
      }
      BCK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
      const int64_t l0 = b->launches;
      s = enqueue(cs);
      cudaGraph_t gr = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(cs, &gr);
      if (s) { if (gr) cudaGraphDestroy(gr); return s; }
      if (ec != cudaSuccess) return bfail(b, MDWT_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ec));
      const cudaError_t ei = cudaGraphInstantiate(&b->graph, gr, 0);
      cudaGraphDestroy(gr);
      if (ei != cudaSuccess) { b->graph = nullptr; return bfail(b, MDWT_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(ei)); }
      b->graphSig = sig;
      b->captures++;
      b->lastUnitsLaunch = b->launches - l0;
      b->launches = l0;
    }
    BCK(cudaGraphLaunch(b->graph, user), "graph launch");
    b->launches += b->lastUnitsLaunch;
    b->replays++;
  } else {
    if ((s = enqueue(user))) return s;
  }
  BCK(cudaEventRecord(b->ev1, user), "event");
  for (auto *c : b->reqs) {   // Renderer::Render id increments (renderer.cpp:957-958)
    c->accumParam = c->accumID++;
    c->frameParam = c->frameID++;
  }
  b->lastGroups = (int)groups.size();
  b->lastTraceLaunches = (int)groups.size() - (fusedGroups >= 1 ? fusedGroups - 1 : 0);
  b->lastUnits = n;
  return MDWT_OK;
}

mdwt_status mdwt_batch_sync(mdwt_batch *b) {
  if (!b) return MDWT_ERR_BAD_ARG;
  BCK(cudaSetDevice(b->device), "cudaSetDevice");
  BCK(cudaDeviceSynchronize(), "sync");
  return MDWT_OK;
}

mdwt_status mdwt_batch_last_ms(mdwt_batch *b, float *ms) {
  if (!b || !ms) return MDWT_ERR_BAD_ARG;
  BCK(cudaEventSynchronize(b->ev1), "event");
  BCK(cudaEventElapsedTime(ms, b->ev0, b->ev1), "elapsed");
  return MDWT_OK;
}

mdwt_status mdwt_batch_info(mdwt_batch *b, int64_t out[8]) {
  if (!b || !out) return MDWT_ERR_BAD_ARG;
  out[0] = b->launches; out[1] = b->lastGroups; out[2] = b->lastUnits; out[3] = b->replays; out[4] = b->captures;
  out[5] = b->unitItems; out[6] = b->pool; out[7] = b->trips;
  return MDWT_OK;
}

mdwt_status mdwt_batch_fusion_info(mdwt_batch *b, int out[2]) {
  if (!b || !out) return MDWT_ERR_BAD_ARG;
  out[0] = b->lastTraceLaunches;
  out[1] = b->fuse ? 1 : 0;
  return MDWT_OK;
}

mdwt_status mdwt_batch_autotune(mdwt_batch *b, int frames, int best[3]) {
  if (!b || frames <= 0) return MDWT_ERR_BAD_ARG;
  if (b->reqs.empty()) return bfail(b, MDWT_ERR_STATE, "empty batch");
  struct Ids { int f, a, fp, ap; };
  std::vector<Ids> saved;
  for (auto *c : b->reqs) saved.push_back({c->frameID, c->accumID, c->frameParam, c->accumParam});
  auto trial = [&](double *ms) -> mdwt_status {
    mdwt_status s = mdwt_batch_render(b, nullptr);   // warm-up (and capture)
    if (s) return s;
    double tot = 0.0;
    for (int f = 0; f < frames; f++) {
      if ((s = mdwt_batch_render(b, nullptr))) return s;
      float m = 0.f;
      if ((s = mdwt_batch_last_ms(b, &m))) return s;
      tot += m;
    }
    *ms = tot / frames;
    return MDWT_OK;
  };
  if (!b->pool) b->pool = b->reqs[0]->pool;
  if (!b->trips) b->trips = b->reqs[0]->trips;
  const int unitsC[] = {0, 32, 64, 128, 256};   // dispenser chunk (0 = sized per request)
  const int poolsC[] = {4, 8, 16, 32};
  const int tripsC[] = {1, 2, 3, 4, 6, 8};
  mdwt_status s = MDWT_OK;
  double bestMs = 1e300;
  auto tune = [&](int *knob, const int *cand, int nc) -> mdwt_status {
    int bestV = *knob;
    for (int i = 0; i < nc; i++) {
      *knob = cand[i];
      double ms = 0.0;
      mdwt_status st = trial(&ms);
      if (st) return st;
      if (ms < bestMs) { bestMs = ms; bestV = cand[i]; }
    }
    *knob = bestV;
    return MDWT_OK;
  };
  if (!(s = tune(&b->trips, tripsC, 6)) && !(s = tune(&b->pool, poolsC, 4))) s = tune(&b->unitItems, unitsC, 5);
  for (size_t i = 0; i < b->reqs.size(); i++) {
    mdwt_ctx *c = b->reqs[i];
    c->frameID = saved[i].f; c->accumID = saved[i].a; c->frameParam = saved[i].fp; c->accumParam = saved[i].ap;
    reset_accum_ids(c);
  }
  if (s) return s;
  if (best) { best[0] = b->unitItems; best[1] = b->pool; best[2] = b->trips; }
  return MDWT_OK;
}

mdwt_status mdwt_autotune_schedule(mdwt_ctx *c, int frames, int best[2]) {
  if (!c || frames <= 0) return MDWT_ERR_BAD_ARG;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  const int f0 = c->frameID, a0 = c->accumID, fp0 = c->frameParam, ap0 = c->accumParam;
  // the trial frames must not show in the context's event counters
  unsigned long long counters0[8];
  CK(cudaStreamSynchronize(c->stream), "sync");
  CK(cudaMemcpy(counters0, c->dCounters, sizeof(counters0), cudaMemcpyDeviceToHost), "save counters");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0), "event");
  CK(cudaEventCreate(&e1), "event");
  mdwt_status s = MDWT_OK;
  double bestMs = 1e300;
  // a candidate renders `frames` frames as one multi-frame launch sequence (the shape
  // of an accumulation loop), after a warm-up of the same
  auto trial = [&](double *ms) -> mdwt_status {
    mdwt_status st = mdwt_render_frames(c, frames, nullptr);   // warm-up
    if (st) return st;
    cudaEventRecord(e0, c->stream);
    st = mdwt_render_frames(c, frames, nullptr);
    cudaEventRecord(e1, c->stream);
    cudaEventSynchronize(e1);
    float m = 0.f;
    cudaEventElapsedTime(&m, e0, e1);
    *ms = m / frames;
    return st;
  };
  auto tune = [&](int *knob, const int *cand, int nc) -> mdwt_status {
    int bestV = *knob;
    for (int i = 0; i < nc; i++) {
      *knob = cand[i];
      double ms = 0.0;
      mdwt_status st = trial(&ms);
      if (st) return st;
      if (ms < bestMs) { bestMs = ms; bestV = cand[i]; }
    }
    *knob = bestV;
    return MDWT_OK;
  };
  const int regroupC[] = {1, 0};
  const int tripsC[] = {1, 2, 3, 4, 6, 8, 12, 16};
  const int poolsC[] = {4, 8, 16, 32};
  const int quorumC[] = {8, 16, 24, 33};
  const int rgBlocksC[] = {0, 3, 2};
  // the regrouped tracker runs -m 2 and -m 0 frames without shadow rays or per-pixel
  // statistics; other frames run the warp-local tracker whatever the knob says
  const bool regroupable = (c->mode == 2 || c->mode == 0) && !c->shadows && !c->statsOn;
  if (regroupable) s = tune(&c->regroup, regroupC, 2);
  if (!s && regroupable && regroup_on(c)) s = tune(&c->rgBlocks, rgBlocksC, 3);
  if (!s && !(s = tune(&c->trips, tripsC, 8)) && !(regroupable && regroup_on(c))) {
    // the regeneration pool and the sample quorum belong to the warp-local tracker
    if (!(s = tune(&c->pool, poolsC, 4))) s = tune(&c->quorum, quorumC, 4);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->frameID = f0; c->accumID = a0; c->frameParam = fp0; c->accumParam = ap0;
  reset_accum_ids(c);
  CK(cudaStreamSynchronize(c->stream), "sync");
  CK(cudaMemcpy(c->dCounters, counters0, sizeof(counters0), cudaMemcpyHostToDevice), "restore counters");
  if (s) return s;
  if (best) { best[0] = c->pool; best[1] = c->trips; }
  return MDWT_OK;
}

mdwt_status mdwt_autotune_macrocells(mdwt_ctx *c, const int *edges, int n, int frames, int *bestEdge) {
  if (!c || !edges || n <= 0 || frames <= 0) return MDWT_ERR_BAD_ARG;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  for (int i = 0; i < n; i++)
    if (edges[i] <= 0) return fail(c, MDWT_ERR_BAD_ARG, "macrocell edge must be positive");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  const int f0 = c->frameID, a0 = c->accumID, fp0 = c->frameParam, ap0 = c->accumParam;
  int64_t dims[3] = {0, 0, 0};
  for (auto &h : c->ch)
    for (int a = 0; a < 3; a++) dims[a] = std::max<int64_t>(dims[a], h.dims[a]);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0), "event");
  CK(cudaEventCreate(&e1), "event");
  double bestMs = 1e300;
  int best = edges[0];
  mdwt_status s = MDWT_OK;
  for (int i = 0; i < n && !s; i++) {
    uint32_t mc[3];
    for (int a = 0; a < 3; a++) mc[a] = (uint32_t)((dims[a] + edges[i] - 1) / edges[i]);
    if ((s = mdwt_set_macrocells(c, mc))) break;
    if ((s = mdwt_render(c, nullptr))) break;   // warm-up
    cudaEventRecord(e0, c->stream);
    for (int f = 0; f < frames && !s; f++) s = mdwt_render(c, nullptr);
    cudaEventRecord(e1, c->stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (!s && ms < bestMs) { bestMs = ms; best = edges[i]; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (s) return s;
  uint32_t mc[3];
  for (int a = 0; a < 3; a++) mc[a] = (uint32_t)((dims[a] + best - 1) / best);
  if ((s = mdwt_set_macrocells(c, mc))) return s;
  c->frameID = f0; c->accumID = a0; c->frameParam = fp0; c->accumParam = ap0;
  reset_accum_ids(c);
  if (bestEdge) *bestEdge = best;
  return MDWT_OK;
}

mdwt_status mdwt_render_frames(mdwt_ctx *c, int n, void *stream) {
  if (!c || n <= 0) return MDWT_ERR_BAD_ARG;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  if (n == 1) return mdwt_render(c, stream);
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  while (n > 0) {
    TrackParams p;
    int batch = 0;
    mdwt_status s = prepare_frame(c, p, &batch);
    if (s) return s;
    const int g = batch >= c->spp ? frames_per_launch(p, c->spp, n) : 1;
    if (g < 2) {   // a frame alone fills the record budget: one launch sequence per frame
      if ((s = mdwt_render(c, stream))) return s;
      n--;
      continue;
    }
    const int rw = p.cullX1 - p.cullX0 + 1, rh = p.cullY1 - p.cullY0 + 1;
    const size_t nrect = p.numTiles > 0 ? (size_t)rw * (size_t)rh : 0;
    const size_t samples = (size_t)g * c->spp;
    if (nrect > 0) {
      if ((s = grow(c, (void **)&c->dRec, c->recCap, samples * nrect * 4, "records")) != MDWT_OK) return s;
      if (c->statsOn &&
          (s = grow(c, (void **)&c->dRecStats, c->recStatsCap, samples * nrect * 4, "record stats")) != MDWT_OK)
        return s;
      if ((c->gradient || c->featOn || c->mode >= MDWT_MODE_MAX) &&
          (s = grow(c, (void **)&c->dRecT, c->recTCap, samples * nrect * 4, "hit distances")) != MDWT_OK)
        return s;
      p.records = c->dRec;
      p.recStats = c->statsOn ? c->dRecStats : nullptr;
      p.recT = (c->gradient || c->featOn || c->mode >= MDWT_MODE_MAX) ? c->dRecT : nullptr;
    }
    // the ids g successive Render calls hand their frames (renderer.cpp:957-958)
    p.nFrames = g;
    p.frameParam1 = (uint32_t)c->frameID;
    p.accumParam1 = (uint32_t)c->accumID;
    p.sBase = 0;
    p.sCount = (int)samples;
    CK(cudaMemsetAsync(c->dWork, 0, sizeof(unsigned int), st), "reset work counter");
    CKI(launch_track(p, c->store, st, c->numSMs, &c->launches, &c->lastGrid, &c->lastBlock, nullptr), "tracker kernels");
    for (int k = 0; k < g; k++) {
      c->accumParam = c->accumID++;
      c->frameParam = c->frameID++;
    }
    n -= g;
  }
  return MDWT_OK;
}

mdwt_status mdwt_sync(mdwt_ctx *c) {
  if (!c) return MDWT_ERR_BAD_ARG;
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(c->stream), "stream");
  CK(cudaDeviceSynchronize(), "device");
  return MDWT_OK;
}

mdwt_status mdwt_reset_accumulation(mdwt_ctx *c) {
  if (!c) return MDWT_ERR_BAD_ARG;
  reset_accum_ids(c);
  return MDWT_OK;
}

mdwt_status mdwt_set_frame_id(mdwt_ctx *c, int f) {
  if (!c || f < 0 || f == INT32_MAX) return MDWT_ERR_BAD_ARG;
  c->frameParam = f;
  c->frameID = f + 1;
  return MDWT_OK;
}

mdwt_status mdwt_get_frame_ids(const mdwt_ctx *c, int out[4]) {
  if (!c || !out) return MDWT_ERR_BAD_ARG;
  out[0] = c->frameID; out[1] = c->accumID; out[2] = c->frameParam; out[3] = c->accumParam;
  return MDWT_OK;
}

mdwt_status mdwt_get_framebuffer(mdwt_ctx *c, uint32_t *out) {
  if (!c || !out) return MDWT_ERR_BAD_ARG;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  CK(cudaDeviceSynchronize(), "sync");
  CK(cudaMemcpy(out, c->dFb, (size_t)c->W * c->H * 4, cudaMemcpyDeviceToHost), "copy framebuffer");
  return MDWT_OK;
}

mdwt_status mdwt_get_accum(mdwt_ctx *c, float *out) {
  if (!c || !out) return MDWT_ERR_BAD_ARG;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  CK(cudaDeviceSynchronize(), "sync");
  CK(cudaMemcpy(out, c->dAccum, (size_t)c->W * c->H * 16, cudaMemcpyDeviceToHost), "copy accum");
  return MDWT_OK;
}

mdwt_status mdwt_get_device_buffers(mdwt_ctx *c, void **accum, void **fb) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (accum) *accum = c->dAccum;
  if (fb) *fb = c->dFb;
  return MDWT_OK;
}

mdwt_status mdwt_get_counters(mdwt_ctx *c, uint64_t out[4]) {
  if (!c || !out) return MDWT_ERR_BAD_ARG;
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  unsigned long long h[8];
  CK(cudaDeviceSynchronize(), "sync");
  CK(cudaMemcpy(h, c->dCounters, sizeof(h), cudaMemcpyDeviceToHost), "copy counters");
  for (int i = 0; i < 4; i++) out[i] = h[i];
  if (h[4]) return fail(c, MDWT_ERR_NUMERIC, "samples reached the per-sample step cap");
  return MDWT_OK;
}

mdwt_status mdwt_reset_counters(mdwt_ctx *c) {
  if (!c) return MDWT_ERR_BAD_ARG;
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  CK(cudaMemsetAsync(c->dCounters, 0, 8 * sizeof(unsigned long long), c->stream), "reset counters");
  CK(cudaStreamSynchronize(c->stream), "reset counters");
  return MDWT_OK;
}

mdwt_status mdwt_enable_pixel_stats(mdwt_ctx *c, int e) {
  if (!c) return MDWT_ERR_BAD_ARG;
  c->statsOn = e != 0;
  if (c->inited) {
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    if (c->statsOn && !c->dStats) {
      const size_t np = (size_t)c->W * c->H;
      CK(cudaMalloc(&c->dStats, np * 16), "cudaMalloc stats");
      CK(cudaMemsetAsync(c->dStats, 0, np * 16, c->stream), "memset stats");
    }
  }
  return MDWT_OK;
}

mdwt_status mdwt_get_pixel_stats(mdwt_ctx *c, uint32_t *out) {
  if (!c || !out) return MDWT_ERR_BAD_ARG;
  if (!c->statsOn || !c->dStats) return fail(c, MDWT_ERR_STATE, "pixel stats are off");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  CK(cudaDeviceSynchronize(), "sync");
  CK(cudaMemcpy(out, c->dStats, (size_t)c->W * c->H * 16, cudaMemcpyDeviceToHost), "copy stats");
  return MDWT_OK;
}

mdwt_status mdwt_set_render_rows(mdwt_ctx *c, int row0, int row1) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (row0 < 0 || row1 < 0) return fail(c, MDWT_ERR_BAD_ARG, "negative row");
  c->rowLo = row0;
  c->rowHi = row1;
  return MDWT_OK;
}

mdwt_status mdwt_copy_frame_rows(mdwt_ctx *c, int row0, int row1, float *accum_dst, uint32_t *fb_dst, void *stream) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  if (row0 < 0 || row1 > c->H || row0 > row1) return fail(c, MDWT_ERR_BAD_ARG, "row range outside the frame");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const size_t off = (size_t)row0 * c->W, n = (size_t)(row1 - row0) * c->W;
  if (accum_dst) CK(cudaMemcpyAsync(accum_dst, c->dAccum + 4 * off, n * 16, cudaMemcpyDefault, st), "copy accum rows");
  if (fb_dst) CK(cudaMemcpyAsync(fb_dst, c->dFb + off, n * 4, cudaMemcpyDefault, st), "copy framebuffer rows");
  return MDWT_OK;
}

mdwt_status mdwt_load_frame_rows(mdwt_ctx *c, int row0, int row1, const float *accum_src, const uint32_t *fb_src,
                                 void *stream) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  if (row0 < 0 || row1 > c->H || row0 > row1) return fail(c, MDWT_ERR_BAD_ARG, "row range outside the frame");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const size_t off = (size_t)row0 * c->W, n = (size_t)(row1 - row0) * c->W;
  if (accum_src) CK(cudaMemcpyAsync(c->dAccum + 4 * off, accum_src, n * 16, cudaMemcpyDefault, st), "load accum rows");
  if (fb_src) CK(cudaMemcpyAsync(c->dFb + off, fb_src, n * 4, cudaMemcpyDefault, st), "load framebuffer rows");
  return MDWT_OK;
}

mdwt_status mdwt_set_timing(mdwt_ctx *c, int enable) {
  if (!c) return MDWT_ERR_BAD_ARG;
  c->timing = enable != 0;
  return MDWT_OK;
}

mdwt_status mdwt_get_kernel_times(mdwt_ctx *c, float out_ms[2]) {
  if (!c || !out_ms) return MDWT_ERR_BAD_ARG;
  if (!c->timed) return fail(c, MDWT_ERR_STATE, "no timed frame (enable timing; frames of at most 8 sample passes)");
  CK(cudaEventSynchronize(c->ev[3 * c->timedPasses - 1]), "event sync");
  out_ms[0] = out_ms[1] = 0.0f;
  for (int b = 0; b < c->timedPasses; b++) {
    float a = 0.0f, r = 0.0f;
    CK(cudaEventElapsedTime(&a, c->ev[3 * b], c->ev[3 * b + 1]), "elapsed");
    CK(cudaEventElapsedTime(&r, c->ev[3 * b + 1], c->ev[3 * b + 2]), "elapsed");
    out_ms[0] += a;
    out_ms[1] += r;
  }
  return MDWT_OK;
}

mdwt_status mdwt_set_tuning(mdwt_ctx *c, int key, int value) {
  if (!c) return MDWT_ERR_BAD_ARG;
  if (key == MDWT_TUNE_POOL) {
    if (value < 1 || value > 32) return fail(c, MDWT_ERR_BAD_ARG, "pool must be in 1..32");
    c->pool = value;
    return MDWT_OK;
  }
  if (key == MDWT_TUNE_TRIPS) {
    if (value < 1 || value > 64) return fail(c, MDWT_ERR_BAD_ARG, "trips must be in 1..64");
    c->trips = value;
    return MDWT_OK;
  }
  if (key == MDWT_TUNE_QUORUM) {
    if (value < 1 || value > 33) return fail(c, MDWT_ERR_BAD_ARG, "quorum must be in 1..33");
    c->quorum = value;
    return MDWT_OK;
  }
  if (key == MDWT_TUNE_REGROUP) {
    if (value < 0 || value > 1) return fail(c, MDWT_ERR_BAD_ARG, "regroup must be 0 or 1");
    c->regroup = value;
    return MDWT_OK;
  }
  if (key == MDWT_TUNE_RG_BLOCKS) {
    if (value < 0 || value > 8) return fail(c, MDWT_ERR_BAD_ARG, "regrouped-tracker blocks per SM must be in 0..8");
    c->rgBlocks = value;
    return MDWT_OK;
  }
  if (key == MDWT_TUNE_BATCH) {
    if (value < 0) return fail(c, MDWT_ERR_BAD_ARG, "batch must be >= 0");
    c->batchCap = value;
    return MDWT_OK;
  }
  return fail(c, MDWT_ERR_BAD_ARG, "unknown tuning key");
}

mdwt_status mdwt_get_tuning(const mdwt_ctx *c, int key, int *value) {
  if (!c || !value) return MDWT_ERR_BAD_ARG;
  switch (key) {
    case MDWT_TUNE_POOL: *value = c->pool; return MDWT_OK;
    case MDWT_TUNE_BATCH: *value = c->batchCap; return MDWT_OK;
    case MDWT_TUNE_TRIPS: *value = c->trips; return MDWT_OK;
    case MDWT_TUNE_QUORUM: *value = c->quorum; return MDWT_OK;
    case MDWT_TUNE_REGROUP: *value = regroup_on(c); return MDWT_OK;
    case MDWT_TUNE_RG_BLOCKS: *value = c->rgBlocks; return MDWT_OK;
    default: return MDWT_ERR_BAD_ARG;
  }
}

mdwt_status mdwt_get_render_info(const mdwt_ctx *c, int64_t out[4]) {
  if (!c || !out) return MDWT_ERR_BAD_ARG;
  out[0] = c->launches;
  out[1] = (int64_t)sizeof(TrackParams);
  out[2] = c->lastGrid;
  out[3] = c->lastBlock;
  return MDWT_OK;
}

mdwt_status mdwt_get_majorants(mdwt_ctx *c, float *out) {
  if (!c || !out) return MDWT_ERR_BAD_ARG;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  CK(cudaDeviceSynchronize(), "sync");
  const size_t n = c->M * (c->mode >= 3 ? 1 : c->ch.size());
  CK(cudaMemcpy(out, c->dMaj, n * 4, cudaMemcpyDeviceToHost), "copy majorants");
  return MDWT_OK;
}

mdwt_status mdwt_get_ranges(mdwt_ctx *c, float *out) {
  if (!c || !out) return MDWT_ERR_BAD_ARG;
  if (!c->inited) return fail(c, MDWT_ERR_STATE, "mdwt_init first");
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  CK(cudaDeviceSynchronize(), "sync");
  CK(cudaMemcpy(out, c->dRanges, c->M * c->ch.size() * 8, cudaMemcpyDeviceToHost), "copy ranges");
  return MDWT_OK;
}

}  // extern "C"
