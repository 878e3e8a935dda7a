/* mdwt_batch.h -- batched rendering of many requests and the autotuner (libmdwt.so).
 *
 * No counterpart in the reference renderer, which renders one scene per Renderer and
 * launch (renderer.cpp:944-973).  A request is a fully set-up render context (its own
 * channels, transfer functions, camera, resolution, spp, mode); a batch renders one frame
 * of every request with one persistent trace launch (and one resolve launch) per kernel
 * variant -- requests with the same mode, voxel storage (uint8 / float32), statistics and
 * shading flags share a launch -- instead of one launch sequence per request.  The
 * per-request results are the ones mdwt_render gives, bit for bit (frame and accumulation
 * ids advance per request as in mdwt_render).  Each request's frame must fit one sample
 * batch of path records (MDWT_ERR_UNSUPPORTED otherwise) and render all rows.
 *
 * Launch structure: every request has a work dispenser of (8x4-tile, sample) items; a
 * warp starts at one request, takes chunks of its items until they run out, then moves
 * to the next request with items left (draining its lanes only at a change of request).
 * With graphs on, the launch sequence (parameter uploads from pinned memory, dispenser
 * resets, kernels) is captured once into a CUDA graph and replayed while the batch's
 * structure (variants, request counts, pixel totals) stays the same.
 */
#ifndef MDWT_BATCH_H
#define MDWT_BATCH_H

#include <stdint.h>

#include "mdwt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mdwt_batch mdwt_batch;

mdwt_status mdwt_batch_create(mdwt_batch **out, int device);
mdwt_status mdwt_batch_destroy(mdwt_batch *b);
const char *mdwt_batch_last_error(const mdwt_batch *b);
/* Add a request (an initialised context on the batch's device; the batch does not own it:
 * the context must stay alive while the batch renders it; adding it twice is
 * MDWT_ERR_BAD_ARG). */
mdwt_status mdwt_batch_add(mdwt_batch *b, mdwt_ctx *request);
mdwt_status mdwt_batch_clear(mdwt_batch *b);
/* One frame of every request, asynchronous on `stream` (NULL: the batch's own stream). */
mdwt_status mdwt_batch_render(mdwt_batch *b, void *stream);
mdwt_status mdwt_batch_sync(mdwt_batch *b);
/* Schedule knobs (0 keeps the current value): dispenser chunk in items (a multiple of 32;
 * by default sized per request like a single-request launch), regeneration pool and
 * phase-1 trips for every request of the batch. */
mdwt_status mdwt_batch_set_schedule(mdwt_batch *b, int unit_items, int pool, int trips);
mdwt_status mdwt_batch_set_graph(mdwt_batch *b, int enable);
/* 1: the requests that run the regrouped tracker (-m 0 and -m 2 without per-pixel
 * statistics, shadow rays, gradient shading or features), whatever their voxel format,
 * resolution and spp, share ONE persistent trace launch and one resolve launch; the other
 * requests get one launch per kernel variant.  0 (default): one launch per kernel variant
 * for all -- measured faster on the mixed 64-request workload (412 vs 424 ms per batch
 * frame).  Results do not depend on it. */
mdwt_status mdwt_batch_set_fusion(mdwt_batch *b, int enable);
/* out[0] trace launches of the last frame, out[1] fusion on (1) or off (0). */
mdwt_status mdwt_batch_fusion_info(mdwt_batch *b, int out[2]);
/* Device time (ms) of the last mdwt_batch_render, from events on its stream; synchronous. */
mdwt_status mdwt_batch_last_ms(mdwt_batch *b, float *ms);
/* out[0] kernels launched so far, [1] kernel-variant groups of the last frame, [2]
 * requests, [3] graph replays, [4] graph captures, [5] chunk items (0 = per request),
 * [6] pool, [7] trips. */
mdwt_status mdwt_batch_info(mdwt_batch *b, int64_t out[8]);
/* Autotuner: coordinate descent over the phase-1 trips {1, 2, 3, 4, 6, 8}, the
 * regeneration pool {4, 8, 16, 32} and the dispenser chunk {per request, 32..256}, each
 * candidate timed over `frames` batch frames after one warm-up frame; keeps the fastest.
 * Results do not depend on these knobs; the requests' frame ids are restored and their
 * accumulation reset afterwards.  best[3] (optional) = chunk items, pool, trips. */
mdwt_status mdwt_batch_autotune(mdwt_batch *b, int frames, int best[3]);

/* Schedule autotuner for one context: coordinate descent over, for -m 2 and -m 0, the tracker
 * (MDWT_TUNE_REGROUP {1, 0}), for the regrouped tracker its blocks per SM
 * (MDWT_TUNE_RG_BLOCKS {0, 3, 2}), then the trips {1, 2, 3, 4, 6, 8, 12, 16}, then -- for the
 * warp-local tracker -- the regeneration pool {4, 8, 16, 32} and the sample quorum
 * {8, 16, 24, never} (MDWT_TUNE_*), each candidate timed on `frames` frames rendered by
 * mdwt_render_frames (after a warm-up of the same), so pass the frames per call of the
 * loop being tuned; keeps the fastest (results do not depend on them).  Frame ids and the
 * event counters are restored and the accumulation reset.  best[2] (optional) = pool,
 * trips; mdwt_get_tuning reads every knob. */
mdwt_status mdwt_autotune_schedule(mdwt_ctx *ctx, int frames, int best[2]);

/* Macrocell autotuner for one context: for each candidate edge length (voxels per
 * macrocell side; cells per side = ceil(dims / edge)) rebuild the value ranges and
 * majorants (transfer functions kept), time `frames` frames, keep the fastest.  Frame ids
 * are restored and the accumulation reset afterwards.  *best_edge (optional). */
mdwt_status mdwt_autotune_macrocells(mdwt_ctx *ctx, const int *edges, int n_edges, int frames, int *best_edge);

#ifdef __cplusplus
}
#endif

#endif
