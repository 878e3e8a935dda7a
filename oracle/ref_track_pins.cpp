// TEST INFRASTRUCTURE ONLY: the reference's own per-pixel program, compiled where it lies
// and run on the host, so that the tests can check the oracle's restatement of the
// tracking path against it.  oracle/Makefile (target `ref`) compiles this file, which
// includes the reference's deviceCode.cu unchanged, into oracle/_ref/libref_track.so.
// Nothing of the reference is copied here; the product never loads this library.
//
// deviceCode.cu is OptiX 7 device code (raygen mainRG, deviceCode.cu:283-471; the
// closest-hit trackers, :513-1065; the root-box intersection, :1676-1726; the miss
// program, :1278-1282).  The stand-ins of oracle/ref_shim supply what it names from the
// OptiX SDK, OWL and CUDA, none of which is vendored:
//   * the OptiX/OWL device API (launch index, payload, program data, ray queries,
//     optixReportIntersection, traceRay) reads and drives the host-side pipeline below;
//   * tex3D<float> / tex2D<float4> are the CUDA texture unit's linear filter
//     (oracle/ref_shim_units.cpp);
//   * OWL's LCG<4>, vector helpers and make_rgba follow this project's restatement;
//   * the float log(...) and pow(...) the trackers and the shading call are this project's
//     log and pow (the oracle's orc_log / orc_pow), which stand in for CUDA's logf/powf.
// deviceCode.cu is device code, and nvcc contracts a*b+c into FMA there, so this file is
// compiled with contraction (-ffp-contract=fast); the texture unit and the RGBA8 packing
// are compiled without it.
//
// The pipeline follows how the reference's Renderer sets OptiX up for the raw-volume path
// (renderer.cpp:660-685): one user geometry, the root macrocell, whose intersection
// program is volumeIntersection and whose closest-hit program is chosen by the method
// (baseLineDTCH, multiMajDTCH, altMultiMajDTCH, cummilativeDTCH, blendDTCH for -m 0..5);
// the triangle TLAS is never built for raw data, so a trace against it misses.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <limits>
#include <memory>
#include <string>
#include <vector>
#include <omp.h>

#include <cuda_runtime.h>

#include "ref_cuda_builtins.h"
#include "ref_texture.h"

extern "C" float orc_log(float x);
extern "C" float orc_pow(float x, float y);
static inline float ref_log(float x) { return orc_log(x); }
static inline float ref_pow(float x, float y) { return orc_pow(x, y); }
#define log(x) ref_log(x)
#define pow(x, y) ref_pow(x, y)
#include "deviceCode.cu"
#undef log
#undef pow

extern "C" {
LaunchParams optixLaunchParams;
}
thread_local uint3 threadIdx;

namespace {

constexpr OptixTraversableHandle kTriangleTLAS = 0;   // never built for raw data
constexpr OptixTraversableHandle kRootTLAS = 1;

struct TraceState {
  void *prd = nullptr;
  const void *data = nullptr;
  owl::vec3f org, dir;
  float tmin = 0.f, tmax = 0.f;
  bool reported = false;
};
thread_local TraceState g_trace;
thread_local owl::vec2i g_launchIndex;
owl::vec2i g_launchDims;
MacrocellData g_rootData;   // the root macrocell's program data
unsigned g_seedMask = 0xffffffffu;   // threadIdx = launch index & g_seedMask
box4f g_rootBox;

// renderer.cpp:671-685
void closest_hit(int mode) {
  switch (mode) {
    case 0: __closesthit__baseLineDTCH(); break;
    case 1: __closesthit__multiMajDTCH(); break;
    case 2: __closesthit__altMultiMajDTCH(); break;
    case 3: __closesthit__cummilativeDTCH(); break;
    default: __closesthit__blendDTCH(); break;
  }
}

}  // namespace

namespace owl {
namespace shim {
vec2i launch_index() { return g_launchIndex; }
vec2i launch_dims() { return g_launchDims; }
void *payload() { return g_trace.prd; }
const void *program_data() { return g_trace.data; }
void trace(OptixTraversableHandle handle, const Ray &ray, void *prd, unsigned) {
  const TraceState saved = g_trace;
  g_trace = TraceState();
  g_trace.prd = prd;
  g_trace.org = ray.origin;
  g_trace.dir = ray.direction;
  g_trace.tmin = ray.tmin;
  g_trace.tmax = ray.tmax;
  bool hit = false;
  if (handle == kRootTLAS) {
    g_trace.data = &g_rootData;
    __intersection__volumeIntersection();
    if (g_trace.reported) {
      closest_hit(optixLaunchParams.mode);
      hit = true;
    }
  }
  if (!hit) __miss__miss();
  g_trace = saved;
}
}  // namespace shim
}  // namespace owl

float3 optixGetWorldRayOrigin() { return g_trace.org; }
float3 optixGetWorldRayDirection() { return g_trace.dir; }
float3 optixGetObjectRayOrigin() { return g_trace.org; }
float3 optixGetObjectRayDirection() { return g_trace.dir; }
float optixGetRayTmin() { return g_trace.tmin; }
float optixGetRayTmax() { return g_trace.tmax; }
unsigned int optixGetPrimitiveIndex() { return 0u; }
float2 optixGetTriangleBarycentrics() { return float2{0.f, 0.f}; }
// OptiX accepts a reported hit inside the ray's current [tmin, tmax] and makes it the
// new tmax (the closest hit so far).
bool optixReportIntersection(float hitT, unsigned int) {
  if (!(hitT >= g_trace.tmin && hitT <= g_trace.tmax)) return false;
  g_trace.tmax = hitT;
  g_trace.reported = true;
  return true;
}

// ---------------------------------------------------------------- the launch
extern "C" {

// Texture registry of oracle/ref_shim_units.cpp: handles of a volume channel (float
// voxels, x fastest) and of a transfer function (n RGBA texels).
cudaTextureObject_t ref_texture_volume(const float *data, int X, int Y, int Z);
cudaTextureObject_t ref_texture_tf(const float *rgba, int n);
void ref_textures_clear();

struct RefScene {
  int W, H, C;
  int mode, spp, accumulate, shadows, gradient;
  const float *vol[12];
  int dims[12][3];
  const float *tf[12];
  int tfN[12];
  float vd[12][2], xd[12][2], os[12];
  float material[12][7];   // diffuse, specular, shininess, gradient step, specular rgb
  const float *majorants;
  unsigned mc[3];
  float lastLo[4], lastHi[4];   // the last channel's box4f (renderer.cpp:748-754)
  float rootLo[4], rootHi[4];   // union of the channels' box4f (renderer.cpp:698-704)
  float dt;
  float cam[12];                // origin, lower-left corner, horizontal, vertical
  float lightDir[3], lightIntensity, ambient, bg[3];
};

// threadIdx for the launches that follow: the launch index (edge 0), or its position in an
// edge x edge thread block (edge a power of two).
void ref_set_seed_block(int edge) { g_seedMask = edge > 0 ? (unsigned)edge - 1u : 0xffffffffu; }

// One launch of mainRG (owlLaunch2D(rayGen, W, H), renderer.cpp:949) with frameID and
// accumID as the launch parameters, over the rows row0, row0 + stride, ... of the frame.
// accum (W*H float4) is read and written, fb (W*H RGBA8) written, for those rows.
int ref_mainrg_frame(const RefScene *s, int frameID, int accumID, float *accum, uint32_t *fb, int row0,
                     int stride, int threads) {
  if (!s || s->C < 1 || s->C > 12 || !accum || !fb || row0 < 0 || stride < 1) return 1;
  LaunchParams lp;
  lp.fbPtr = fb;
  lp.fbSize = owl::vec2i(s->W, s->H);
  lp.accumBuffer = reinterpret_cast<vec4f *>(accum);
  lp.frameID = (uint32_t)frameID;
  lp.accumID = (uint32_t)accumID;
  lp.spp = s->spp;
  lp.triangleTLAS = kTriangleTLAS;
  lp.mode = s->mode;
  lp.enableShadows = s->shadows != 0;
  lp.enableGradientShading = s->gradient != 0;
  lp.heatMapMode = 0;
  lp.enableAccumulation = s->accumulate != 0;
  lp.lightDir = vec3f(s->lightDir[0], s->lightDir[1], s->lightDir[2]);
  lp.lightIntensity = s->lightIntensity;
  lp.ambient = s->ambient;
  lp.bgColor = vec3f(s->bg[0], s->bg[1], s->bg[2]);
  lp.volume.numChannels = s->C;
  lp.volume.rootMacrocellTLAS = kRootTLAS;
  lp.volume.meshType = 2;   // MeshType::RAW
  lp.volume.dt = s->dt;
  lp.volume.macrocellDims = vec3ui(s->mc[0], s->mc[1], s->mc[2]);
  lp.volume.majorants = const_cast<float *>(s->majorants);
  lp.volume.globalBoundsLo = float4{s->lastLo[0], s->lastLo[1], s->lastLo[2], s->lastLo[3]};
  lp.volume.globalBoundsHi = float4{s->lastHi[0], s->lastHi[1], s->lastHi[2], s->lastHi[3]};
  ref_textures_clear();
  for (int c = 0; c < s->C; c++) {
    StructuredVolumeChannel &g = lp.volume.sGrid[c];
    g.dims = vec3ui((uint32_t)s->dims[c][0], (uint32_t)s->dims[c][1], (uint32_t)s->dims[c][2]);
    g.scalarTex[0] = ref_texture_volume(s->vol[c], s->dims[c][0], s->dims[c][1], s->dims[c][2]);
    g.splitAxis = 3;
    lp.transferFunction[c].xf = ref_texture_tf(s->tf[c], s->tfN[c]);
    lp.transferFunction[c].volumeDomain = float2{s->vd[c][0], s->vd[c][1]};
    lp.transferFunction[c].xfDomain = float2{s->xd[c][0], s->xd[c][1]};
    lp.transferFunction[c].opacityScale = s->os[c];
    lp.material[c].diffuse = s->material[c][0];
    lp.material[c].specular = s->material[c][1];
    lp.material[c].shininess = s->material[c][2];
    lp.material[c].gradientStep = s->material[c][3];
    lp.material[c].specularColor = float3{s->material[c][4], s->material[c][5], s->material[c][6]};
  }
  lp.camera.origin = vec3f(s->cam[0], s->cam[1], s->cam[2]);
  lp.camera.lower_left_corner = vec3f(s->cam[3], s->cam[4], s->cam[5]);
  lp.camera.horizontal = vec3f(s->cam[6], s->cam[7], s->cam[8]);
  lp.camera.vertical = vec3f(s->cam[9], s->cam[10], s->cam[11]);
  optixLaunchParams = lp;
  g_rootBox = box4f(vec4f(s->rootLo[0], s->rootLo[1], s->rootLo[2], s->rootLo[3]),
                    vec4f(s->rootHi[0], s->rootHi[1], s->rootHi[2], s->rootHi[3]));
  g_rootData = MacrocellData();
  g_rootData.bboxes = &g_rootBox;
  g_rootData.offset = 0;
  g_launchDims = owl::vec2i(s->W, s->H);
  const int nrows = row0 < s->H ? (s->H - 1 - row0) / stride + 1 : 0;
  const int64_t n = (int64_t)nrows * s->W;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t i = 0; i < n; i++) {
    const int x = (int)(i % s->W), y = row0 + stride * (int)(i / s->W);
    // the reference's threadIdx under OptiX is not a function of the pixel: the launch
    // index stands for it, or (ref_set_seed_block) the pixel's position in a thread block
    g_launchIndex = owl::vec2i(x, y);
    threadIdx.x = (unsigned)x & g_seedMask;
    threadIdx.y = (unsigned)y & g_seedMask;
    threadIdx.z = 0;
    __raygen__mainRG();
  }
  return 0;
}

}  // extern "C"
