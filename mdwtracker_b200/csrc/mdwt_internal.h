// mdwt_internal.h -- plain-data structures shared by the host (mdwt_host.cpp) and the
// sm_100a kernels (mdwt_kernels.cu).  No CUDA or torch types cross the public ABI;
// these structs only cross the host/kernel-launcher boundary inside libmdwt.so.
#pragma once
#include <stdint.h>
#include <stddef.h>

namespace mdwt {

constexpr int kMaxChannels = 12;          // deviceCode.h:13
constexpr uint32_t kMaxStepsPerSample = 1u << 22;

// Device voxel storage.  uint8 channels stay one byte per voxel (value = b * 255,
// the exact float the reference's RawR conversion produces, rawFile.cpp:103-105);
// everything else is stored as the float32 the reference would have uploaded.
enum StoreKind : int { kStoreU8 = 0, kStoreF32 = 1 };

struct F3 { float x, y, z; };

// Parameters of one tracker launch (one frame).  Passed by value as a
// __grid_constant__ kernel parameter.
struct TrackParams {
  // frame
  int W, H, spp;
  uint32_t frameParam, accumParam;  // LaunchParams::frameID / accumID as the frame sees them
  int accumulate, mirror;
  F3 bg;
  // camera basis (LaunchParams::camera)
  F3 camOrg, camLlc, camHor, camVer;
  // root box = union of channel bounds (renderer.cpp:698-716)
  F3 rootLo, rootHi;
  // grid transform of the trackers (deviceCode.cu:759-778), bounds of the last channel
  F3 gLo;        // worlddim.lower
  F3 w2u;        // 1 / (upper - lower)
  F3 gScale;     // unitToGrid * worldToUnit (== worldToUnit * unitToGrid)
  uint32_t mc[3];
  int C, mode;
  float dt;
  const float *majorants;      // [cell*C + ch] (modes 0..2) or [cell] (mode 3)
  // channels
  const void *vol[kMaxChannels];
  int dims[kMaxChannels][3];
  // transfer functions (alpha already cubed, as in renderer.cpp:1100)
  const float *tfAlpha[kMaxChannels];   // n floats
  const float *tfRgba[kMaxChannels];    // 4n floats
  int tfN[kMaxChannels];
  float vd[kMaxChannels][2];
  float xd[kMaxChannels][2];
  float os[kMaxChannels];
  // shading (defaults of renderer.h:125-130 unless set)
  float lightIntensity, ambient;
  F3 matSpec[kMaxChannels];
  // outputs
  float *accum;                  // float4 per pixel
  uint32_t *fb;                  // RGBA8 per pixel
  uint32_t *stats;               // 4 per pixel or null
  unsigned long long *counters;  // [0]=samples [1]=rejections [2]=cells [3]=path-samples [4]=capped
  unsigned int *workCounter;     // pixel dispenser, zeroed before the launch
  int numTiles;                  // 8x4 pixel tiles covering the image
  int tilesX;
};

// Per-axis voxel intervals of the separable range build: for macrocell index k on
// one axis, voxels [lo[k], hi[k]] (empty when lo > hi) enter its value range.
struct AxisIntervals {
  const int *lo;
  const int *hi;
};

// ---- launchers implemented in mdwt_kernels.cu (return cudaError_t as int) ----
int launch_track(const TrackParams &p, int storeKind, void *stream, int numSMs, int *launches, int *grid, int *block);
int track_occupancy(int storeKind, int mode, int *blocksPerSM, int *threadsPerBlock);

// Value ranges of one channel into ranges[(cell*C + ch)*2 + {0,1}].
//   vol: channel voxels; dims; mc grid; intervals per axis (device arrays);
//   scratchA: >= Z*Y*mc[0] float2, scratchB: >= Z*mc[1]*mc[0] float2.
int launch_ranges(const void *vol, int storeKind, const int dims[3], const uint32_t mc[3],
                  const int *ivx, const int *ivy, const int *ivz, int C, int ch,
                  float *ranges, float *scratchA, float *scratchB, void *stream, int *launches);
// ranges initialised to (1e20, -1e20) (sizeMCs, renderer.cu:330-347)
int launch_ranges_init(float *ranges, size_t count, void *stream, int *launches);

struct MajorantParams {
  const float *ranges;
  float *majorants;
  int C, mode;
  size_t M;
  const float *tfAlpha[kMaxChannels];
  int tfN[kMaxChannels];
  float vd[kMaxChannels][2];
  float xd[kMaxChannels][2];
  float os[kMaxChannels];
};
int launch_majorants(const MajorantParams &p, void *stream, int *launches);

}  // namespace mdwt
