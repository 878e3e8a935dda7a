// mdwt_internal.h -- plain-data structures shared by the host (mdwt_host.cpp) and the
// sm_100a kernels (mdwt_kernels.cu).  No CUDA or torch types cross the public ABI;
// these structs only cross the host/kernel-launcher boundary inside libmdwt.so.
#pragma once
#include <stdint.h>
#include <stddef.h>

namespace mdwt {

constexpr int kMaxChannels = 12;          // deviceCode.h:13
constexpr uint32_t kMaxStepsPerSample = 1u << 22;
// Margin terms of the free-flight exit filter (flight_surely_exits in mdwt_math.cuh):
// factors of |xf|, |k| and |tf|.
constexpr float kFlightRel = 3.814697265625e-06f;   // 2^-18
constexpr float kFlightAbs = 3.814697265625e-06f;   // 2^-18 (log2 units, times k)
constexpr float kFlightTf = 2.384185791015625e-07f;  // 2^-22

// Device voxel storage.  uint8 channels stay one byte per voxel (value = b * 255,
// the exact float the reference's RawR conversion produces, rawFile.cpp:103-105);
// everything else is stored as the float32 the reference would have uploaded.
// Voxel storage on the device.  kStoreU8: bytes, x fastest (value = byte * 255).
// kStoreF32: float32 in 2x2x2 micro-bricks -- voxel (x, y, z) at
// ((((z>>1) * Yb + (y>>1)) * Xb + (x>>1)) * 8) + 4 (z&1) + 2 (y&1) + (x&1), with
// Xb = ceil(X/2), Yb = ceil(Y/2): a trilinear footprint whose lower corner has even
// coordinates is one 32-byte sector, and any footprint spans at most eight.
// kStoreF32Lin: float32, x fastest (a caller's buffer: mdwt_build_ranges_noalloc).
enum StoreKind : int { kStoreU8 = 0, kStoreF32 = 1, kStoreF32Lin = 2 };

struct F3 { float x, y, z; };

// Parameters of one tracker launch (one frame).  Passed by value as a
// __grid_constant__ kernel parameter.
struct TrackParams {
  // frame
  int W, H, spp;
  uint32_t frameParam, accumParam;  // LaunchParams::frameID / accumID as the frame sees them
  // frames traced in one launch: frame k >= 1 sees frameParam1 + k - 1, accumParam1 + k - 1
  // (the ids n successive Render calls hand their frames); sample j of the launch is
  // sample j % spp of frame j / spp
  int nFrames;
  uint32_t frameParam1, accumParam1;
  int accumulate, mirror;
  uint32_t seedMask;             // seed words from (pixel & seedMask): ~0 per pixel, edge - 1 per thread block
  F3 bg;
  // camera basis (LaunchParams::camera)
  F3 camOrg, camLlc, camHor, camVer;
  // root box = union of channel bounds (renderer.cpp:698-716)
  F3 rootLo, rootHi;
  // grid transform of the trackers (deviceCode.cu:759-778), bounds of the last channel
  F3 gLo;        // worlddim.lower
  F3 gHi;        // worlddim.upper
  F3 w2u;        // 1 / (upper - lower)
  F3 gScale;     // unitToGrid * worldToUnit (== worldToUnit * unitToGrid)
  uint32_t mc[3];
  int C, mode;
  float dt;
  const float *majorants;      // [cell*C + ch] (modes 0..2) or [cell] (mode 3)
  // The trackers' per-cell table, tabStride = Ce + 1 float2 per cell (Ce = C, or 1 for the
  // summed majorant): entry 0 holds the cell's non-zero-majorant channel mask (as bits in
  // .x), entry 1 + c the majorant of channel c and its recip_for_div -- the mask and the
  // first majorants share a sector, and a majorant comes with its reciprocal in one load.
  const float2 *cellTab;
  int tabStride;
  // Free-flight arithmetic (mdwt_set_arithmetic).  fast = 0: the flights the exit filter
  // does not settle run the exact chain.  fast = 1: they run the filter's hardware-log2
  // estimate as the flight itself, and cellTab holds 1 / majorant for every non-zero
  // majorant.
  int fast;
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
  int shadows, gradient;         // shadow rays; gradient (Blinn-Phong) shading
  F3 lightDir;
  float matDiffuse[kMaxChannels], matSpecular[kMaxChannels], matShininess[kMaxChannels], matGradStep[kMaxChannels];
  // outputs
  float *accum;                  // float4 per pixel
  uint32_t *fb;                  // RGBA8 per pixel
  uint32_t *stats;               // 4 per pixel or null
  unsigned long long *counters;  // [0]=samples [1]=rejections [2]=cells [3]=path-samples [4]=capped
  unsigned int *workCounter;     // pixel dispenser, zeroed before the launch
  // Pixels outside [cullX0, cullX1] x [cullY0, cullY1] certainly miss the root box
  // (conservative screen-space bound of its 8 corners, 3 px margin): each of their
  // samples composites the background, so their per-pixel result is the constant
  // bgFin (sum over spp of the background, / spp), computed on the host.
  int cullX0, cullY0, cullX1, cullY1;
  int rowLo, rowHi;              // rows [rowLo, rowHi) of the frame are rendered (a band)
  float bgFin[4];
  int numTiles;                  // 8x4 pixel tiles covering the traced rectangle
  int tilesX;
  F3 gOrg;                       // gScale * (camOrg - gLo): grid-space ray origin
  int pool;                      // regenerate paths when this many lanes of a warp wait
  int chunk;                     // work items a warp takes from the dispenser at once
  int trips;                     // phase-1 transition/draw trips per warp round (at most)
  int quorum;                    // ... ending early once this many lanes hold a pending sample
  int regroup;                   // -m 2 / -m 0: the regrouped tracker (trace_regroup_kernel)
  int rgBlocks;                  // its blocks per SM (0: as many as fit); fewer leave more L1 cache
  int vol32;                     // every channel has < 2^32 voxels: 32-bit voxel offsets
  int store;                     // voxel storage of every channel: kStoreU8 or kStoreF32 (micro-bricks)
  // sample batch [sBase, sBase + sCount) of the frame; one 4-byte record per traced
  // path, [k * nrect + rect-local pixel], nrect = pixels of the traced rectangle
  int sBase, sCount;
  uint32_t *records;
  uint32_t *recStats;            // per-path density samples | rejections << 16 (stats only)
  float *recT;                   // per-path world t of the primary hit (gradient shading, features)
  float *feat;                   // 16 floats per pixel of denoiser features, or null
  float featScale;               // depth feature = mean hit distance * featScale
  float *partial;                // float4 running sums per rect pixel between batches
  uint32_t *partialStats;        // uint4 per rect pixel between batches (stats only)
};

// A group of batched requests sharing one kernel variant (device arrays).
struct BatchGroup {
  int mode, storeKind;
  bool stats, ext, shade;                // per-pixel stats; extended trace; shaded resolve
  bool regroup;                          // -m 2, every request regroupable (regroup_fits)
  const TrackParams *reqs;               // the group's requests (chunk = dispenser chunk)
  int nReq;
  unsigned *dispensers;                  // one work counter per request, zeroed before the launch
  unsigned long long totalItems;         // work items of the group
  const unsigned long long *pixOfs;      // nReq + 1 prefix offsets of W*H
  unsigned long long totalPix;
};
// -m 2 with MDWT_TUNE_REGROUP on and slot fields that fit the regrouped tracker's packing.
bool regroup_fits(const TrackParams &p);
// Regroupable requests of any method (-m 0, -m 2) and voxel format in ONE persistent trace
// launch and one resolve launch (no per-pixel statistics, shadows or hit distances).
int launch_track_batch_fused(const TrackParams *reqs, int nReq, unsigned *dispensers, unsigned long long totalItems,
                             const unsigned long long *pixOfs, unsigned long long totalPix, void *stream, int numSMs,
                             int *launches, int *grid);
// Blocks per SM of the batched trace kernel of a variant (for chunk sizing).
int batch_trace_occupancy(int mode, int storeKind, bool stats, bool ext);
int launch_track_batch(const BatchGroup &g, void *stream, int numSMs, int *launches, int *grid);

constexpr int kMaxTexels = 16384;          // TF texels addressable by a path record
constexpr size_t kRecordBudget = size_t(1) << 30;   // records per sample pass (4 GiB)

// Per-axis voxel intervals of the separable range build: for macrocell index k on
// one axis, voxels [lo[k], hi[k]] (empty when lo > hi) enter its value range.
struct AxisIntervals {
  const int *lo;
  const int *hi;
};

// ---- launchers implemented in mdwt_kernels.cu (return cudaError_t as int) ----
// trace + resolve of one sample batch; evMid (a cudaEvent_t or null) is recorded between them
int launch_track(const TrackParams &p, int storeKind, void *stream, int numSMs, int *launches, int *grid, int *block,
                 void *evMid);

// Value ranges of one channel into ranges[(cell*C + ch)*2 + {0,1}].
//   vol: channel voxels; dims; mc grid; intervals per axis (device arrays);
//   scratchA: >= Z*Y*mc[0] float2, scratchB: >= Z*mc[1]*mc[0] float2.
int launch_ranges(const void *vol, int storeKind, const int dims[3], const uint32_t mc[3],
                  const int *ivx, const int *ivy, const int *ivz, int C, int ch,
                  float *ranges, float *scratchA, float *scratchB, void *stream, int *launches);
// ranges initialised to (1e20, -1e20) (sizeMCs, renderer.cu:330-347)
// FP64 expected image (W*H*3 doubles) of the unshaded estimator; J jitter points, world
// step h0.  RMSE helper: *sum += sum over pixels of |accum.rgb - ref|^2 (sum zeroed by
// the caller).
int launch_expected(const TrackParams &p, int storeKind, int J, double h0, double *out, void *stream, int numSMs,
                    int *launches);
int launch_rmse(const float *accum, const double *ref, size_t npix, double *sum, void *stream, int numSMs,
                int *launches);
int launch_ranges_init(float *ranges, size_t count, void *stream, int *launches);

struct MajorantParams {
  const float *ranges;
  float *majorants;
  float2 *cellTab;             // the trackers' per-cell table (TrackParams::cellTab), or null
  int fast;                    // TrackParams::fast: the table's reciprocals are 1 / majorant
  int C, mode;
  size_t M;
  const float *tfAlpha[kMaxChannels];
  int tfN[kMaxChannels];
  float vd[kMaxChannels][2];
  float xd[kMaxChannels][2];
  float os[kMaxChannels];
};
int launch_majorants(const MajorantParams &p, void *stream, int *launches);
// Float32 voxels, x fastest, into the micro-brick layout of kStoreF32 (dst holds
// 8 ceil(X/2) ceil(Y/2) ceil(Z/2) floats; the padding voxels are written as 0).
int launch_brick_f32(const float *src, float *dst, const int dims[3], void *stream, int *launches);
// Floats of a channel's device buffer in the layout of `storeKind` (bytes / 4 for uint8).
size_t stored_voxels(int storeKind, const int64_t dims[3]);

}  // namespace mdwt
