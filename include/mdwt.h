/*
 * mdwt.h -- C ABI of the B200-native multi-density Woodcock tracker (libmdwt.so).
 *
 * The ABI replaces the `dtracker::Renderer` class of alpers-git/MDWTracker
 * (renderer.h:52-222, renderer.cpp, renderer.cu) for the raw-volume render path,
 * headless.  Each entry point names the reference member it stands in for.
 *
 * Conventions
 *   - Every call returns an mdwt_status (MDWT_OK == 0).  No call throws, exits or
 *     prints; mdwt_last_error() returns a text for the last failing call.
 *   - A context owns one CUDA device and every device buffer of one scene.  A
 *     context is driven by one host thread at a time (like the reference).
 *   - Host pointers passed in are only read during the call (the library copies).
 *   - Setters take effect immediately.  In the reference some members (spp,
 *     accumulation, dt, materials) reach the device only in Renderer::Update()
 *     (renderer.cpp:975-1008); here each setter is that member write plus Update().
 */
#ifndef MDWT_H
#define MDWT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mdwt_ctx mdwt_ctx;
typedef int mdwt_status;

enum {
  MDWT_OK = 0,
  MDWT_ERR_BAD_ARG = 1,            /* argument out of range, null pointer, bad channel id */
  MDWT_ERR_CUDA = 2,               /* a CUDA call failed (text in mdwt_last_error) */
  MDWT_ERR_IO = 3,                 /* file missing or truncated */
  MDWT_ERR_TOO_MANY_CHANNELS = 4,  /* more than MDWT_MAX_CHANNELS channels */
  MDWT_ERR_UNSUPPORTED = 5,        /* mode or data format not supported */
  MDWT_ERR_STATE = 6,              /* call order violated (e.g. render before init) */
  MDWT_ERR_OOM = 7,                /* device or host allocation failed */
  MDWT_ERR_TIMEOUT = 8,            /* a device-side bounded wait gave up */
  MDWT_ERR_FORMAT = 9,             /* raw file name carries no dims / unknown type */
  MDWT_ERR_NUMERIC = 10,           /* a sample hit the per-sample step cap (NaN/inf input) */
  MDWT_ERR_SCRATCH_LIMIT = 11      /* input larger than the fixed scratch of mdwt_build_ranges_noalloc */
};

#define MDWT_MAX_CHANNELS 12       /* deviceCode.h:13 */

/* Voxel formats, numbered like raw::DataFormat (rawFile.h:21-35). */
enum {
  MDWT_FMT_UNSPECIFIED = 0,
  MDWT_FMT_INT8 = 1,
  MDWT_FMT_INT16 = 2,
  MDWT_FMT_INT32 = 3,
  MDWT_FMT_UINT8 = 4,
  MDWT_FMT_UINT16 = 5,
  MDWT_FMT_UINT32 = 6,
  MDWT_FMT_FLOAT32 = 7,
  MDWT_FMT_DOUBLE64 = 8
};

/* Tracking methods, numbered like dtracker::Mode (renderer.h:24-36). */
enum {
  MDWT_MODE_NDDA = 0,        /* Mode::BASELINE: one DDA per channel (deviceCode.cu:858-970) */
  MDWT_MODE_MULTI = 1,       /* Mode::MULTI: min-of-channels free flight (deviceCode.cu:619-745) */
  MDWT_MODE_SYNCDDA = 2,     /* Mode::MULTI_ALT: one DDA, per-channel samplers (deviceCode.cu:747-856) */
  MDWT_MODE_CUMULATIVE = 3,  /* Mode::CUMMULATIVE: summed majorant (deviceCode.cu:513-617) */
  MDWT_MODE_MAX = 4,         /* Mode::MAX: max-opacity blended sample, summed majorant (deviceCode.cu:165-180, 972-1065) */
  MDWT_MODE_MIX = 5          /* Mode::MIX: opacity-weighted colour mix (deviceCode.cu:182-200, 972-1065) */
};

/* ---- context ---------------------------------------------------------- */

/* Renderer() + the context part of Init (renderer.cpp:334): one context on `device`.
 * device == MDWT_HOST_ONLY makes a context that touches no GPU: it parses and holds
 * channels and answers the host-side queries (channel info, dt, macrocell dims,
 * camera basis) but refuses mdwt_init.  Fails with MDWT_ERR_CUDA when no device. */
#define MDWT_HOST_ONLY (-1)
mdwt_status mdwt_create(mdwt_ctx **out, int device);
/* Renderer::Terminate (renderer.cpp:1010-1014). Frees every device buffer. */
mdwt_status mdwt_destroy(mdwt_ctx *ctx);
/* Text of the last failing call on ctx ("" if none).  Valid until the next call. */
const char *mdwt_last_error(const mdwt_ctx *ctx);
const char *mdwt_status_string(mdwt_status s);
/* ABI version, (major << 16) | minor. */
int mdwt_version(void);

/* ---- data (raw::RawR + Renderer::PushMesh) ----------------------------- */

/* raw::RawR::RawR (rawFile.cpp:31-128) + PushMesh (renderer.cpp:1031-1044):
 * parse `<name>_<X>x<Y>x<Z>_<type>.raw`, read, convert to float exactly as the
 * reference (uint8 -> v*255, int8 -> v*255-128, ...), bounds [0,1]^3, value range
 * seeded with [0,1] and extended by the data.  Fails with MDWT_ERR_TOO_MANY_CHANNELS
 * at the 13th channel (the reference's `<=` test admits a 13th, renderer.cpp:1033). */
mdwt_status mdwt_push_channel_raw(mdwt_ctx *ctx, const char *path);
/* The same from memory: `data` holds dims[0]*dims[1]*dims[2] voxels of `format`, x fastest. */
mdwt_status mdwt_push_channel(mdwt_ctx *ctx, const void *data, int format, const int64_t dims[3]);
/* raw::RawR::reshapeBounds (rawFile.cpp:217-237, viewer `-cb`): scale the xyz bounds
 * of channel ch by scale[3], or by the grid dims when scale is NULL.  Before mdwt_init. */
mdwt_status mdwt_reshape_bounds(mdwt_ctx *ctx, int ch, const float *scale3);
/* Channel count, dims and box4f bounds (lo.xyzw, hi.xyzw) of channel ch (RawR::getBounds4f). */
mdwt_status mdwt_num_channels(const mdwt_ctx *ctx, int *n);
mdwt_status mdwt_get_channel_info(const mdwt_ctx *ctx, int ch, int64_t dims[3], float bounds8[8]);

/* ---- scene set-up (Renderer::Init) -------------------------------------- */

/* Renderer::macrocellDims (renderer.h:164) / viewer `-mc` (viewer.cpp:204-224):
 * macrocell COUNT per side.  A zero component takes the default
 * CalculateMCGridDims(4) (renderer.cpp:641-647, 1342-1355).  Before mdwt_init. */
mdwt_status mdwt_set_macrocells(mdwt_ctx *ctx, const uint32_t dims[3]);
/* Renderer::Init(mode, autoSetCamera) (renderer.cpp:324-942), raw branch: uploads the
 * channels, builds the per-(cell,channel) value ranges (renderer.cu:1116-1179), sets
 * the default camera when auto_camera != 0, dt from Resetdt, fb 1024x1024 unless resized.
 * Modes 0..3 are supported; others return MDWT_ERR_UNSUPPORTED. */
mdwt_status mdwt_init(mdwt_ctx *ctx, int mode, int auto_camera);
mdwt_status mdwt_get_macrocell_dims(const mdwt_ctx *ctx, uint32_t dims[3]);

/* ---- transfer functions -------------------------------------------------- */

/* Renderer::SetXFColormap (renderer.cpp:1094-1165): n RGBA texels (float, 4*n values);
 * alpha is raised to the third power, accumulation reset, majorants rebuilt. */
mdwt_status mdwt_set_tf(mdwt_ctx *ctx, int ch, const float *rgba, int n);
/* Renderer::SetXFOpacityScale (renderer.cpp:1167-1179). */
mdwt_status mdwt_set_opacity_scale(mdwt_ctx *ctx, int ch, float scale);
/* Renderer::SetXFRange (renderer.cpp:1182-1193): the xfDomain of channel ch. */
mdwt_status mdwt_set_tf_range(mdwt_ctx *ctx, int ch, float lo, float hi);
/* Renderer::RecalculateDensityRanges (renderer.cu:206-274). Called by the three above. */
mdwt_status mdwt_recalculate_majorants(mdwt_ctx *ctx);

/* ---- render parameters ---------------------------------------------------- */

/* Renderer::Setdt (renderer.cpp:1460-1466): dt = max(dt, 1e-4). */
mdwt_status mdwt_set_dt(mdwt_ctx *ctx, float dt);
/* Renderer::Resetdt, raw branch (renderer.cpp:1444-1454). */
mdwt_status mdwt_reset_dt(mdwt_ctx *ctx);
mdwt_status mdwt_get_dt(const mdwt_ctx *ctx, float *dt);
/* camera::Camera::setOrientation (camera.h:83-110) + Renderer::UpdateCamera
 * (renderer.cpp:1058-1092); viewer `-c` (viewer.cpp:195-203). */
mdwt_status mdwt_set_camera(mdwt_ctx *ctx, const float from[3], const float at[3],
                            const float up[3], float fovy_deg);
/* The pinhole basis the kernels use: origin, lower-left corner, horizontal, vertical. */
mdwt_status mdwt_get_camera_basis(const mdwt_ctx *ctx, float out12[12]);
/* Renderer::Resize (renderer.cpp:1046-1056). */
mdwt_status mdwt_resize(mdwt_ctx *ctx, int width, int height);
/* Renderer::spp / enableAccumulation / bgColor (renderer.h:111,124,129). */
mdwt_status mdwt_set_spp(mdwt_ctx *ctx, int spp);
mdwt_status mdwt_set_accumulation(mdwt_ctx *ctx, int enable);
mdwt_status mdwt_set_background(mdwt_ctx *ctx, const float rgb[3]);
/* viewer `-l` (viewer.cpp:274-284): shadows, gradient shading, light dir, intensity, ambient. */
mdwt_status mdwt_set_light(mdwt_ctx *ctx, int shadows, int gradient, const float dir[3],
                           float intensity, float ambient);
/* Renderer::SetMaterial* (renderer.cpp:1195-1315). */
mdwt_status mdwt_set_material(mdwt_ctx *ctx, int ch, float diffuse, float specular,
                              float shininess, float gradient_step, const float spec_rgb[3]);
/* Renderer::mirrorFramebuffer (renderer.h:177, renderer.cpp:962-972). */
mdwt_status mdwt_set_mirror(mdwt_ctx *ctx, int enable);
/* Seed words of the per-sample generator.  The reference seeds LCG<4>(threadIdx.x + seed,
 * threadIdx.y + seed) for the camera ray and (threadIdx.x + seed + 1, threadIdx.y + seed + 1)
 * for the shadow ray (deviceCode.cu:296-297, 385-386); under OptiX threadIdx is not a
 * function of the pixel.  edge 0 (the default): the pixel's coordinates stand for
 * threadIdx.  edge = a power of two in 1..1024: the pixel's position inside an edge x edge
 * thread block, as a 2-D CUDA launch of such blocks would give threadIdx -- pixels at the
 * same position in different blocks then share their generator streams, as they would in
 * that launch.  Other values: MDWT_ERR_BAD_ARG. */
mdwt_status mdwt_set_seed_block(mdwt_ctx *ctx, int edge);
/* No reference counterpart: the arithmetic of the free flights t - log(1 - u) / majorant
 * * dt * w2g (deviceCode.cu:564, 676, 739, 805, 913, 1023).
 * MDWT_ARITH_EXACT (the default): the project's own log and correctly rounded quotients,
 * the same on the CPU oracle and the GPU, so frames are bit-identical to the oracle's; a
 * flight that certainly leaves its macrocell is still decided from the hardware log2,
 * within a proven margin.
 * MDWT_ARITH_FAST: a flight length is the hardware log2 (lg2.approx) times
 * dt * w2g * ln 2 / majorant, with no exact chain.  Lengths differ from the exact ones
 * by a few units in the last place, so a path's events differ only where a flight ends
 * that close to a cell or volume boundary or a density lands that close to its
 * acceptance threshold: per-pixel collision events match the oracle on at least 99.9 %
 * of pixels at equal spp (tested), and converged images match the exact ones within
 * their noise.  Most flights leave their cell and are settled by the same exit filter
 * under both arithmetics, so the fast one gains little time (its flights inside a cell
 * skip the exact chain).
 * The accumulation is not reset.  After mdwt_init, the call rebuilds the majorant
 * table (the fast flights use 1 / majorant); other values: MDWT_ERR_BAD_ARG. */
#define MDWT_ARITH_EXACT 0
#define MDWT_ARITH_FAST 1
mdwt_status mdwt_set_arithmetic(mdwt_ctx *ctx, int arith);
mdwt_status mdwt_get_arithmetic(const mdwt_ctx *ctx, int *arith);

/* ---- frames ------------------------------------------------------------------ */

/* Renderer::Render (renderer.cpp:944-973): one frame, asynchronous on `cuda_stream`
 * (a cudaStream_t, NULL = the context's own stream).  The frame uses the current
 * frame/accumulation ids; afterwards they advance exactly like the reference
 * (owlParamsSet1i(.., accumID++) after the launch). */
mdwt_status mdwt_render(mdwt_ctx *ctx, void *cuda_stream);
/* n successive frames (n Renderer::Render calls) with their paths traced in one launch
 * when their path records fit the record budget together (no counterpart in the
 * reference): the same frames, ids, accumulation and counters as n mdwt_render calls,
 * bit for bit; the framebuffer, statistics and features are the last frame's. */
mdwt_status mdwt_render_frames(mdwt_ctx *ctx, int n, void *cuda_stream);
/* No reference counterpart: render only the rows [row0, row1) of the frame (other rows
 * keep their contents; row1 <= row0 = all rows).  Frame and accumulation ids advance
 * as for a full frame, so N contexts rendering disjoint bands of the same frame
 * together produce exactly the single-context frame (multi-GPU row split). */
mdwt_status mdwt_set_render_rows(mdwt_ctx *ctx, int row0, int row1);
/* Copy rows [row0, row1) of the accumulation (float4) and RGBA8 buffers to caller
 * memory (device or pinned/pageable host; either pointer may be NULL), enqueued on
 * `cuda_stream` (NULL = the context's stream). */
mdwt_status mdwt_copy_frame_rows(mdwt_ctx *ctx, int row0, int row1, float *accum_dst, uint32_t *fb_dst,
                                 void *cuda_stream);
/* No counterpart in the reference (row bands).  The inverse of mdwt_copy_frame_rows: rows
 * [row0, row1) of the accumulation (float4) and RGBA8 buffers from caller memory (either
 * pointer may be NULL), enqueued on `cuda_stream` (NULL = the context's stream).  A
 * context whose band grows takes over the running mean of its new rows this way. */
mdwt_status mdwt_load_frame_rows(mdwt_ctx *ctx, int row0, int row1, const float *accum_src, const uint32_t *fb_src,
                                 void *cuda_stream);
/* Wait for every frame issued on the context's streams; reports device-side errors. */
mdwt_status mdwt_sync(mdwt_ctx *ctx);
/* Renderer::ResetAccumulation (renderer.cpp:1488-1495). */
mdwt_status mdwt_reset_accumulation(mdwt_ctx *ctx);
/* frameID, accumID (host counters) and the values the next frame uses. */
mdwt_status mdwt_get_frame_ids(const mdwt_ctx *ctx, int out4[4]);
/* Writes the reference's public Renderer::frameID member (renderer.h:110): the next frame
 * renders with frame id `frame_id` (seed factor frame_id + 1), the one after with
 * frame_id + 1, and so on.  Sample seeds of frames far apart do not repeat. */
mdwt_status mdwt_set_frame_id(mdwt_ctx *ctx, int frame_id);
/* RGBA8 framebuffer (LaunchParams::fbPtr), W*H words, row-major from the bottom row. */
mdwt_status mdwt_get_framebuffer(mdwt_ctx *ctx, uint32_t *host_out);
/* Accumulation buffer (LaunchParams::accumBuffer), 4*W*H floats. */
mdwt_status mdwt_get_accum(mdwt_ctx *ctx, float *host_out);
/* Device pointers of the accumulation (float4) and RGBA8 buffers, for zero-copy readers. */
mdwt_status mdwt_get_device_buffers(mdwt_ctx *ctx, void **accum, void **fb);
/* Sum over all frames since the last reset of the per-ray counters of the reference
 * (prd.samples, prd.rejections, deviceCode.cu:829,847) plus macrocell visits and
 * path-samples: out[0]=density samples, [1]=rejections, [2]=cells visited, [3]=path-samples. */
mdwt_status mdwt_get_counters(mdwt_ctx *ctx, uint64_t out4[4]);
mdwt_status mdwt_reset_counters(mdwt_ctx *ctx);
/* Per-pixel statistics of the last frame: 4 uint32 per pixel = samples, rejections,
 * hits (over spp), xor-fold of the hit channel ids.  Off by default (costs a buffer). */
mdwt_status mdwt_enable_pixel_stats(mdwt_ctx *ctx, int enable);
mdwt_status mdwt_get_pixel_stats(mdwt_ctx *ctx, uint32_t *host_out);

/* Tracker tuning knobs (no reference counterpart; results do not depend on them).
 * MDWT_TUNE_POOL: a warp starts new paths only when at least `value` (1..32) of its
 * lanes wait for one, or when no lane is busy.
 * MDWT_TUNE_BATCH: at most `value` samples per pixel per trace pass (0 = as many as the
 * 4 GiB path-record budget allows); the per-pixel sums still run in sample order.
 * MDWT_TUNE_TRIPS: transition/free-flight trips (1..64) a warp takes per round before
 * it evaluates its pending density samples together.
 * MDWT_TUNE_QUORUM: a round's trips also end once `value` (1..33; 33 = never) of the
 * warp's lanes hold a pending density sample.
 * MDWT_TUNE_REGROUP: 1 = -m 2 and -m 0 frames without shadow rays or per-pixel
 * statistics run the tracker that keeps 64 paths per warp and runs, at each step, the
 * operation most of them need next (path start, walk, density sample), one path per
 * lane; a walk takes at most TRIPS free-flight draws.  0 = the warp-local tracker (32
 * paths per warp; POOL and QUORUM apply to it only).  Until set: 1 for -m 2, 0 for -m 0
 * (on the 1080p 6 x 512^3 float32 scene the warp-local tracker is the faster N-DDA
 * tracker with macrocells of 16 voxels or fewer, the regrouped one with 32); the
 * schedule autotuner tries both.
 * MDWT_TUNE_RG_BLOCKS: blocks of 256 threads per SM the regrouped tracker runs (0, the
 * default: as many as its path slots' shared memory allows, 4); fewer blocks leave more of
 * the SM's 256 KB of L1/shared memory to the L1 cache, which holds the majorant grid. */
enum { MDWT_TUNE_POOL = 0, MDWT_TUNE_BATCH = 1, MDWT_TUNE_TRIPS = 2, MDWT_TUNE_QUORUM = 3, MDWT_TUNE_REGROUP = 4,
       MDWT_TUNE_RG_BLOCKS = 5 };
mdwt_status mdwt_set_tuning(mdwt_ctx *ctx, int key, int value);
/* The current value of a tuning knob (defaults: pool 8, batch 0, trips 4, quorum 16,
 * regroup 1 for -m 2 and 0 otherwise, regrouped-tracker blocks 0). */
mdwt_status mdwt_get_tuning(const mdwt_ctx *ctx, int key, int *value);

/* No reference counterpart: CUDA events on the render stream around the trace kernel
 * (with the work-counter reset before it) and the resolve kernel of every sample pass of
 * each frame of at most 8 passes (a pass holds the samples whose path records fit
 * 2^30 records); mdwt_get_kernel_times returns the last frame's {trace, resolve}
 * milliseconds summed over its passes (it waits for that frame). */
mdwt_status mdwt_set_timing(mdwt_ctx *ctx, int enable);
mdwt_status mdwt_get_kernel_times(mdwt_ctx *ctx, float out_ms2[2]);

/* Launch bookkeeping: out[0] = kernels launched by this context so far, out[1] = bytes
 * of per-frame parameters a render sends host->device, out[2] = grid and out[3] = block
 * size of the last tracker launch. */
mdwt_status mdwt_get_render_info(const mdwt_ctx *ctx, int64_t out4[4]);

/* ---- majorant grid ------------------------------------------------------------ */

/* gridMaximaBuffer (renderer.cpp:706-711): M*C floats (cell-major, channel-minor) for
 * modes 0..2, M floats for mode 3 (the summed majorant, renderer.cu:111-157). */
mdwt_status mdwt_get_majorants(mdwt_ctx *ctx, float *host_out);
/* macrocellsBuffer (renderer.cu:1116-1179): per (cell, channel) value range, 2*M*C floats. */
mdwt_status mdwt_get_ranges(mdwt_ctx *ctx, float *host_out);

/* ---- denoiser features (no counterpart in the reference: the input of the learned
 * denoiser).  With features on, every frame also writes 16 floats per pixel: the frame's
 * mean radiance RGB, the first-collision depth (mean hit distance / (camera-to-box-centre
 * distance + box diagonal), 0 without hits), the miss fraction (transmittance estimate),
 * the hit fractions of channels 0..7, the noise level 1/sqrt(spp) and two zeros.  Needs the frame in one sample batch
 * and spp < 65536 (MDWT_ERR_UNSUPPORTED otherwise). */
mdwt_status mdwt_set_features(mdwt_ctx *ctx, int enable);
mdwt_status mdwt_get_features(mdwt_ctx *ctx, float *host_out);        /* W*H*16 */
mdwt_status mdwt_get_device_features(mdwt_ctx *ctx, void **d_features);
/* Device-to-device copy of the last frame's features (W*H*16 floats) on `stream`. */
mdwt_status mdwt_copy_features(mdwt_ctx *ctx, void *d_dst, void *stream);

/* ---- FP64 ground truth (no counterpart in the reference: the convergence measurement
 * "RMSE of the accumulation buffer against an FP64 expected image")
 * mdwt_render_expected: per pixel, the expected value of the unshaded estimator in double
 * precision -- the integral over the root-box segment of T(t) * sum_c (alpha_c / dt) *
 * colour_c plus T(exit) * background (every tracker -m 0..3 samples this first-collision
 * distribution), midpoint rule with `step_voxels` of the smallest voxel edge, averaged over
 * `jitter` points of the pixel's diagonal jitter.  Asynchronous on `stream` (NULL: the
 * context's).  MDWT_ERR_UNSUPPORTED with shadows or gradient shading on.
 * mdwt_get_expected: copy of the last expected image, W*H*3 doubles (row py*W + px, like
 * the accumulation buffer).
 * mdwt_accum_rmse: sqrt(mean over pixels and R, G, B of (accum - expected)^2), in double,
 * synchronous. */
mdwt_status mdwt_render_expected(mdwt_ctx *ctx, int jitter, float step_voxels, void *stream);
mdwt_status mdwt_get_expected(mdwt_ctx *ctx, double *host_out);
mdwt_status mdwt_accum_rmse(mdwt_ctx *ctx, double *rmse);

/* No counterpart in the reference: a self-check of the trackers' free-flight exit filter.
 * A flight t - log(1 - u) / majorant * dt * w2g (deviceCode.cu:805, 915) that certainly
 * leaves the current cell is decided from the hardware log2 with a margin, without the
 * exact log; the margin assumes |log2_hw(x) - log2(x)| <= 2^-20 * (1 + |log2 x|) for every
 * flight argument x = 1 - k 2^-24.  Writes the largest observed value of
 * |log2_hw(x) - log2(x)| / (1 + |log2 x|) over all 2^24 of them on the current device
 * (synchronous; allocates 4 bytes). */
mdwt_status mdwt_check_flight_filter(float *worst_out);

/* No counterpart in the reference.  The value ranges of ONE channel, built on the GPU
 * without allocating any memory, for callers that may not allocate device memory: code
 * that runs inside an application's own memory pool or under an allocator that forbids
 * cudaMalloc, and plug-ins that are handed device buffers and a stream but no right to
 * allocate.  The caller passes the channel's voxels on the device (`format`
 * MDWT_FMT_UINT8, value = byte * 255, or MDWT_FMT_FLOAT32; x fastest), its dims, the
 * macrocell counts, the box the grid spans (the union of the channel bounds,
 * renderer.cpp:698-716) and a device output of 2 * mc[0]*mc[1]*mc[2] floats (min, max per
 * cell, cell-major).  The result equals the ranges mdwt_init builds for that channel.
 * Work is enqueued on `cuda_stream` (a cudaStream_t; NULL = legacy default stream).
 * Limits: at most 1024 macrocells per axis and dims[2] * mc[1] * mc[0] <= 2^20, else
 * MDWT_ERR_SCRATCH_LIMIT.  Bounds for which some voxel's neighbour box is empty in float
 * or the cells touched are not non-decreasing along an axis give MDWT_ERR_UNSUPPORTED
 * (mdwt_init rejects the non-monotone ones too).  The scratch is fixed device memory
 * inside the library (8 MiB + 24 KiB, held by every GPU that loads the library until the
 * process exits).  A call outside stream capture looks up its address on the current
 * device; a call under capture reuses the address found by the last call on that device
 * and fails with MDWT_ERR_STATE if there was none, so make the first call on a device
 * before any stream capture.  An error left pending by earlier CUDA work is reported as
 * MDWT_ERR_CUDA before anything is launched and is not cleared.  Calls share the
 * scratch: calls that overlap on the GPU race. */
mdwt_status mdwt_build_ranges_noalloc(const void *d_volume, int format, const int64_t dims[3],
                                      const uint32_t macrocells[3], const float world_lo[3],
                                      const float world_hi[3], float *d_ranges_out, void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* MDWT_H */
