/*
 * gsplat_cuda.h — additive exports of the B200 CUDA SortedAlpha renderer.
 *
 * Nothing here changes the v0.1 ABI in gsplat.h; these entry points add what
 * the reference's ABI lacks (reference gsplat.h:105-111 has no pixel readback
 * and no load from memory) plus the debug taps the parity tests read, the
 * standalone GPU sort that replaces gsplat-sort's backends, and batched
 * rendering. Error convention as in gsplat.h: int32_t GsplatErrorCode plus a
 * thread-local gsplat_last_error_message().
 */
#ifndef GSPLAT_CUDA_H
#define GSPLAT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#include "gsplat.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Compositing of the per-tile splat lists. */
typedef enum GsplatBlendMode {
  /* Default. FP32 front-to-back: C += (rgb*a*g)*T, T *= (1 - a*g); a pixel
   * stops once T < 1e-4 (after adding the splat that crossed it) and a warp
   * stops when all its pixels have. One UNORM8 rounding at the end. */
  GSPLAT_BLEND_FP32_FRONT_TO_BACK = 0,
  /* Parity mode with the reference's Rgba8Unorm target: back-to-front,
   * dst = src + dst*(1 - src.a) rounded to UNORM8 after every splat, as the
   * reference's premultiplied-alpha blend state does
   * (crates/gsplat-render-wgpu/src/draw_pass.rs:75, lib.rs:53). */
  GSPLAT_BLEND_UNORM8_BACK_TO_FRONT = 1,
} GsplatBlendMode;

/* A scene in the reference's SceneBuffers layout
 * (crates/gsplat-core/src/lib.rs:201-213): RUF positions, opacity logits,
 * log-scales, xyzw rotations, DC coefficients and, for sh_degree > 0,
 * channel-major sh_rest ([R c1..cK, G c1..cK, B c1..cK] per splat,
 * K = (sh_degree+1)^2 - 1). Host pointers; the library copies the data. */
typedef struct GsplatSceneDesc {
  uint64_t count;
  uint32_t sh_degree;
  uint32_t reserved;
  const float *positions;     /* 3*count */
  const float *opacity;       /* count */
  const float *scale_xyz;     /* 3*count */
  const float *rotation_xyzw; /* 4*count */
  const float *color_dc;      /* 3*count */
  const float *sh_rest;       /* count*3*K, or NULL when sh_degree == 0 */
} GsplatSceneDesc;

/* One splat after the vertex stage of the reference shader
 * (crates/gsplat-render-wgpu/shaders/splat_surface_direct.wgsl:131-217,
 * 328-334); 64 bytes. Written for every splat id by the debug tap. */
typedef struct GsplatProjectedSplat {
  float center_ndc[2];
  float axis_u[2];
  float axis_v[2];
  float color[4]; /* premultiplied rgb, alpha */
  float extent_scale;
  float depth;
  uint32_t flags; /* bit0 depth-visible, bit1 drawn (inside the frustum) */
  uint16_t tile_x0, tile_y0, tile_x1, tile_y1; /* tile rect, ends exclusive */
  uint32_t reserved;
} GsplatProjectedSplat;

/* Counters and device timings of the last frame of a context. */
typedef struct GsplatFrameCounts {
  uint64_t visible;      /* depth-visible splats (= GsplatStats.visible_count) */
  uint64_t drawn;        /* visible splats inside the frustum */
  uint64_t tile_keys;    /* (tile, splat) pairs emitted */
  uint64_t key_capacity; /* pair capacity of the context's workspace */
  uint32_t tiles_x, tiles_y, tile_size, blend_mode;
  float preprocess_ms, sort_ms, raster_ms, frame_ms;
  uint32_t frame_reruns; /* frames re-run after growing the pair buffers */
  uint32_t sort_refreshed; /* 1: the frame sorted its depth order; 0: it reused the last one */
} GsplatFrameCounts;

/* ---- context extensions ---- */

/* Renderer::set_size (crates/gsplat-render-wgpu/src/lib.rs:383-399). */
int32_t gsplat_context_set_size(GsplatContext *ctx, uint32_t width, uint32_t height);
int32_t gsplat_context_get_config(const GsplatContext *ctx, GsplatConfig *out_config);
int32_t gsplat_context_get_camera(const GsplatContext *ctx, GsplatCamera *out_camera);
int32_t gsplat_context_set_blend_mode(GsplatContext *ctx, uint32_t mode);
/* Tile edge in pixels: 8 or 16 (default 16). Images do not depend on it. */
int32_t gsplat_context_set_tile_size(GsplatContext *ctx, uint32_t tile);
/* When enabled, render_frame also keeps the per-splat projected records for
 * gsplat_context_debug_projected. Off by default. */
int32_t gsplat_context_set_debug_taps(GsplatContext *ctx, uint32_t enabled);
/* When enabled (the default), a frame's launches are captured once into a
 * CUDA graph and replayed while the image size, tile size, blend mode, debug
 * taps and pair capacity stay the same; disabled, every launch is issued
 * separately. Images are identical either way. */
int32_t gsplat_context_set_cuda_graph(GsplatContext *ctx, uint32_t enabled);
/* Raster launch shape of the FP32 mode: records staged per step (`chunk`:
 * 64, 128 or 256 at tile size 16; 32 or 64 at tile size 8) and persistent
 * blocks per SM that pull tiles from a global queue (0 = one block per tile,
 * at most 32). Changing the tile size resets an invalid chunk to the full
 * tile. Images do not depend on either setting. */
int32_t gsplat_context_set_raster_config(GsplatContext *ctx, uint32_t chunk, uint32_t blocks_per_sm);
/* Depth-order refresh cadence. 0 (the default) sorts every frame, as the
 * reference's gsplat_context_render_frame does. interval >= 1 applies the
 * reference's surface sort interval (crates/gsplat-render-wgpu/src/
 * surface_session.rs:17, 536-596; gsplat_surface_renderer_set_sort_interval
 * there): the visible splats are re-sorted when the camera has changed
 * `interval` times since the last sort, and always after a scene load or
 * resize. Frames in between (an unchanged camera included) project every
 * splat with their own camera but draw only the splats of the last sorted
 * order, in that order (stale-order frames, as in the reference). */
int32_t gsplat_context_set_sort_interval(GsplatContext *ctx, uint32_t interval);

/* No counterpart in the reference: frame lanes (1 to 8, default 1).
 * Frames enqueued with gsplat_context_render_frame_async rotate over `lanes`
 * independent pipelines, each on its own CUDA stream with its own workspace
 * and image, so consecutive frames overlap on the device (one frame's sorts
 * run beside another's raster). Every image is the one a single lane gives;
 * readbacks, stats and debug taps refer to the last frame. Waits for the
 * frames in flight. A sort interval other than 0 runs frames on one lane. */
int32_t gsplat_context_set_frame_lanes(GsplatContext *ctx, uint32_t lanes);

/* Load a scene from host memory (validated like SceneBuffers::validate,
 * crates/gsplat-core/src/lib.rs:224-276). Replaces any loaded scene. */
int32_t gsplat_context_load_scene_buffers(GsplatContext *ctx, const GsplatSceneDesc *scene);

/* Load a scene in the packed resident format of the reference's packed atlas
 * (crates/gsplat-render-wgpu/src/packed_atlas.rs: 20-byte hot record of
 * quantised position, opacity, log scales, rotation and baked colour, plus a
 * 48-byte i8 SH sidecar): 68 instead of 240 bytes per SH3 splat, decoded per
 * frame by the preprocess kernel. SH degree <= 3 (else UNSUPPORTED). No
 * reference counterpart in the C ABI (the reference's packed path is a
 * renderer-internal diagnostic). */
int32_t gsplat_context_load_scene_packed(GsplatContext *ctx, const GsplatSceneDesc *scene);

/* Copy the last frame's RGBA8 image (row 0 = top, tight rows of width*4
 * bytes) into `out`, which must hold width*height*4 bytes. Stands in for
 * Renderer::readback_rgba8 (lib.rs:779-795). */
int32_t gsplat_context_readback_rgba8(GsplatContext *ctx, uint8_t *out, uint64_t out_len);
/* Enqueue that copy on the context's copy stream and return: `out` (pinned
 * host memory for an asynchronous copy) must stay valid until
 * gsplat_context_sync. Frames alternate between two device images, so the
 * next frame renders while this one is copied. No reference counterpart. */
int32_t gsplat_context_readback_rgba8_async(GsplatContext *ctx, uint8_t *out, uint64_t out_len);

int32_t gsplat_context_get_frame_counts(const GsplatContext *ctx, GsplatFrameCounts *out);

/* Device time of each phase of the last frame, in this order: preprocess,
 * depth sort, pair emission, tile sort, tile ranges, raster. Writes up to
 * `capacity` values and the phase count to *out_count. */
int32_t gsplat_context_get_phase_times(const GsplatContext *ctx, float *out, uint32_t capacity,
                                       uint32_t *out_count);

/* Enqueue one frame on the context's stream without waiting for it (the
 * tile-pair buffers keep the size of the last synchronous frame). Errors of
 * enqueued frames, including a pair-buffer overflow, are reported by the next
 * gsplat_context_sync, after which stats describe the last enqueued frame. */
int32_t gsplat_context_render_frame_async(GsplatContext *ctx);
int32_t gsplat_context_sync(GsplatContext *ctx);

/* The context's cudaStream_t, for callers that order their own device work
 * (events, copies) with the renderer's frames. */
int32_t gsplat_context_get_stream(const GsplatContext *ctx, void **out_stream);

/* ---- debug taps of the last frame (copies to host memory) ---- */

/* Depth-sorted visible splat ids: back-to-front, ties by ascending id — the
 * order Renderer::current_sorted_indices returns after a CPU sort
 * (lib.rs:605-607). */
int32_t gsplat_context_debug_order(GsplatContext *ctx, uint32_t *out, uint64_t capacity,
                                   uint64_t *out_len);
/* Per splat id (needs gsplat_context_set_debug_taps(ctx, 1) before the frame). */
int32_t gsplat_context_debug_projected(GsplatContext *ctx, GsplatProjectedSplat *out,
                                       uint64_t capacity, uint64_t *out_len);
/* Per splat id, two floats: the log2(alpha) and the coverage bound on r^2
 * (the largest float below (log2 alpha + 8) / (4.5 log2 e), capped at s^2;
 * -1 when that bound is not positive) the FP32 raster blended the splat with;
 * NaN for splats in no tile list and for UNORM8-mode frames. `capacity` and
 * `out_len` count splats. */
int32_t gsplat_context_debug_coverage(GsplatContext *ctx, float *out, uint64_t capacity,
                                      uint64_t *out_len);
/* (tile, splat id) pairs in emission order (depth order, rect rows outer). */
int32_t gsplat_context_debug_tile_pairs(GsplatContext *ctx, uint32_t *tiles, uint32_t *ids,
                                        uint64_t capacity, uint64_t *out_len);
/* Per-tile [start, end) ranges (2 words per tile) and the tile-sorted ids. */
int32_t gsplat_context_debug_tile_ranges(GsplatContext *ctx, uint32_t *ranges,
                                         uint64_t ranges_capacity, uint32_t *ids,
                                         uint64_t ids_capacity, uint64_t *out_keys);

/* A packed scene's resident data: the header and tables (1,292 floats: bounds
 * min and span, log-scale min and extent, SH scales, pad, 1,024 axis
 * variances, 256 extent scales), the hot records (5 words per splat) and the
 * SH sidecars (48 bytes per splat, when the degree is >= 1). Any output may be
 * null; *out_splats = n. No reference counterpart. */
int32_t gsplat_context_debug_packed_scene(GsplatContext *ctx, float *table, uint32_t *hot,
                                          int8_t *sidecar, uint64_t *out_splats);
/* The loaded scene's resident planes as floats: pos_alpha (4n), cov_a (4n),
 * cov_b (4n), then the colour planes (4 * planes * n); *out_len = total.
 * No reference counterpart: lets tests compare the device PLY decode with
 * the host load path bit for bit. */
int32_t gsplat_context_debug_scene(GsplatContext *ctx, float *out, uint64_t capacity,
                                   uint64_t *out_len);

/* ---- standalone GPU sort (replaces gsplat-sort's CPU and GPU backends) ---- */

/* CpuSortBackend::sort_values_by_keys (crates/gsplat-sort/src/lib.rs:36-61):
 * permute `values` so that keys are descending; equal keys keep their input
 * order. `keys` is not modified. Host pointers; len < 2^30. */
int32_t gsplat_cuda_sort_values_by_keys(const uint32_t *keys, uint32_t *values, uint64_t len);
/* CpuSortBackend::sort_pairs (lib.rs:81-101): keys descending, equal keys by
 * ascending value; both arrays are permuted. */
int32_t gsplat_cuda_sort_pairs(uint32_t *keys, uint32_t *values, uint64_t len);

/* No counterpart in the reference: an allocation-free form of
 * gsplat_cuda_sort_values_by_keys for callers that cannot allocate device
 * memory — hosts that own all GPU memory through their own pool and forbid
 * libraries to call cudaMalloc, or latency-critical threads where
 * cudaMalloc/cudaFree (which can synchronise the device) are not allowed.
 * `keys` and `values` are caller-owned DEVICE pointers of `len` elements;
 * `values` is permuted in place so that keys descend, equal keys keeping
 * their input order, and `keys` is left unchanged. `stream` is a
 * cudaStream_t (NULL for the default stream); the call waits for it before
 * returning. All scratch lives in one static device array of about 14.7 MB
 * that every GPU loading the library holds until exit; len above
 * 1,048,576 (2^20) is rejected with GSPLAT_ERROR_INVALID_ARGUMENT. The first
 * call on a device looks the array's address up (cudaGetSymbolAddress), so
 * make it before any stream capture starts on that device. The call waits
 * for `stream`, so a stream that is being captured is refused with
 * GSPLAT_ERROR_INVALID_ARGUMENT; a CUDA error left pending by earlier work is
 * returned (and cleared) as GSPLAT_ERROR_INTERNAL before anything launches.
 * Calls share the array; overlapping calls would race, so calls are
 * serialised inside the process. Nothing here calls cudaMalloc or cudaFree. */
int32_t gsplat_cuda_sort_values_by_keys_noalloc(const uint32_t *keys, uint32_t *values,
                                                uint64_t len, void *stream);

/* ---- batched frames -------------------------------------------------------
 * No counterpart in the reference: its renderer draws one camera per call.
 * A batch holds several HBM-resident scenes and renders many views (scene,
 * camera, image size) in one call: the views are split into launch groups of
 * up to 1024 views (one CUDA-graph launch each, with one shared sort over
 * (view, tile, depth) keys), and every view's image equals, bit for bit, the
 * image gsplat_context_render_frame gives for the same scene, camera, size,
 * tile size and blend mode. A batch handle is confined to one thread at a
 * time, like a context. */
typedef struct GsplatBatch GsplatBatch;

typedef struct GsplatBatchView {
  uint32_t scene;       /* id returned by gsplat_batch_add_scene_* */
  uint32_t width;
  uint32_t height;
  uint32_t reserved;    /* 0 */
  GsplatCamera camera;
} GsplatBatchView;      /* 56 bytes */

typedef struct GsplatBatchViewStats {
  uint32_t visible_count;  /* depth-visible splats (GsplatStats.visible_count) */
  uint32_t drawn_count;    /* splats with a raster record */
  uint32_t tile_pairs;     /* (tile, splat) pairs the view emitted */
  uint32_t group;          /* launch group the view ran in */
} GsplatBatchViewStats;

typedef struct GsplatBatchTimes {
  float device_ms;       /* CUDA-event time of all launch groups */
  float wall_ms;         /* host time of the call */
  uint32_t groups;       /* launch groups */
  uint32_t reruns;       /* groups re-run after outgrowing their pair buffers */
  uint32_t kernel_launches;
  uint32_t graph_launches; /* CUDA graph launches of the first pass: 1 once the same batch layout
                              repeats (every group captured in one graph), 0 the first time */
  uint64_t tile_pairs;   /* over all views */
} GsplatBatchTimes;

/* Creates a batch on the current CUDA device (UNSUPPORTED without an sm_100
 * device). Scenes are held under a budget of 150 GiB unless changed. */
int32_t gsplat_batch_create(GsplatBatch **out_batch);
void gsplat_batch_destroy(GsplatBatch *batch);
int32_t gsplat_batch_set_scene_budget(GsplatBatch *batch, uint64_t bytes);
/* Uploads a scene (validated like gsplat_context_load_scene_buffers); the id
 * numbers scenes from 0 in the order they were added. UNSUPPORTED when the
 * scene would exceed the budget. */
int32_t gsplat_batch_add_scene_buffers(GsplatBatch *batch, const GsplatSceneDesc *scene,
                                       uint32_t *out_scene);
int32_t gsplat_batch_add_scene_path(GsplatBatch *batch, const char *path, uint32_t *out_scene);
/* As gsplat_batch_add_scene_buffers, stored in the packed resident format. */
int32_t gsplat_batch_add_scene_packed(GsplatBatch *batch, const GsplatSceneDesc *scene,
                                      uint32_t *out_scene);
int32_t gsplat_batch_set_tile_size(GsplatBatch *batch, uint32_t tile);       /* 8 or 16 */
int32_t gsplat_batch_set_blend_mode(GsplatBatch *batch, uint32_t mode);      /* GsplatBlendMode */
/* Launch-group limits: views (1..1024), predicted tile pairs, splats and
 * image tiles per group (0 keeps the current value). Up to 65,536 tiles a
 * group's tile sort takes two passes, above that three. */
int32_t gsplat_batch_set_limits(GsplatBatch *batch, uint32_t max_views, uint64_t max_pairs,
                                uint64_t max_splats, uint64_t max_tiles);
/* As gsplat_context_set_raster_config. */
int32_t gsplat_batch_set_raster_config(GsplatBatch *batch, uint32_t chunk, uint32_t blocks_per_sm);

typedef struct GsplatTuneResult {
  uint32_t tile_size;      /* chosen launch shape, now set on the batch */
  uint32_t chunk;
  uint32_t blocks_per_sm;
  uint32_t candidates;     /* shapes timed (0 when taken from the cache) */
  float best_ms;           /* median device time of the views with it */
  float default_ms;        /* the same with tile 16, chunk 256, one block per tile */
  uint32_t from_cache;
  uint32_t reserved;
} GsplatTuneResult;        /* 32 bytes */

/* Autotunes the batch's launch shape on `views`: renders them with every
 * candidate (tile 16 with chunks 256/128/64, tile 8 with chunks 64/32, each
 * with one block per tile or 2/4 resp. 8/16 persistent blocks per SM), keeps
 * the fastest by median device time over `reps` renders and sets it on the
 * batch. With a `cache_path`, results are kept in that text file keyed by GPU
 * name, blend mode, image sizes and scene-size class, and a later call with
 * the same key takes the stored shape without rendering. Images are the same
 * under every candidate. */
int32_t gsplat_batch_autotune(GsplatBatch *batch, const GsplatBatchView *views, uint32_t count,
                              const char *cache_path, uint32_t reps, GsplatTuneResult *out_result);
/* Renders all `count` views and waits until every image is in device memory. */
int32_t gsplat_batch_render(GsplatBatch *batch, const GsplatBatchView *views, uint32_t count);
int32_t gsplat_batch_get_times(const GsplatBatch *batch, GsplatBatchTimes *out_times);
/* Phase timing (off by default): while on, a render runs its launch groups one
 * after another, waiting after each, in place of the whole-batch graph, and
 * records per-phase CUDA-event times summed over the groups. A measurement
 * mode: the images are the same, the device time is not the production one. */
int32_t gsplat_batch_set_phase_timing(GsplatBatch *batch, uint32_t on);
/* Per-phase device ms of the last render, in the order preprocess, depth sort,
 * emission, tile sort, tile ranges, raster; `count` of them (at most 6) are
 * written. All zero unless that render was phase-timed. Groups re-run after
 * outgrowing their pair buffers add their first run only. */
int32_t gsplat_batch_get_phase_times(const GsplatBatch *batch, float *out_ms, uint32_t count);
int32_t gsplat_batch_get_view_stats(const GsplatBatch *batch, uint32_t view,
                                    GsplatBatchViewStats *out_stats);
/* RGBA8 image of view `view` of the last render (row 0 = top, tight rows). */
int32_t gsplat_batch_readback_rgba8(GsplatBatch *batch, uint32_t view, uint8_t *out,
                                    uint64_t out_len);
/* Device address and size of that image (valid until the next render or
 * destroy), and the cudaStream_t the batch renders on. */
int32_t gsplat_batch_image_device(const GsplatBatch *batch, uint32_t view, const void **out_ptr,
                                  uint64_t *out_bytes);
int32_t gsplat_batch_get_stream(const GsplatBatch *batch, void **out_stream);

/* ---- served rendering --------------------------------------------------------
 * No counterpart in the reference. A server keeps scenes resident in HBM and
 * renders requests (one GsplatBatchView each) with continuous batching: a
 * scheduler thread takes the queued requests into a batch whenever one of
 * its lanes (a CUDA stream with its own workspace) is free, admitting them in
 * arrival order while the batch's predicted memory -- tile-pair buffers sized
 * from predicted tile-overlap counts, splat workspace and images -- fits the
 * lane's share of the work budget. Batches on different lanes overlap on the
 * device. A request is done when its RGBA8 image is in host memory; it is
 * identical, bit for bit, to gsplat_context_render_frame's image for the same
 * scene, camera and size at the server's tile size. Every call except create
 * and destroy may be made from any thread. */
typedef struct GsplatServer GsplatServer;

typedef struct GsplatServeConfig {
  uint64_t scene_budget_bytes;  /* resident scenes; 0 = 150 GiB */
  uint64_t work_budget_bytes;   /* workspace over all lanes; 0 = 24 GiB */
  uint32_t lanes;               /* batches in flight, 1..8; 0 = 2 */
  uint32_t max_views_per_batch; /* 1..1024; 0 = 256 */
  uint32_t tile_size;           /* 8 or 16; 0 = 16 */
  uint32_t raster_chunk;        /* as gsplat_context_set_raster_config; 0 = full tile */
  uint32_t raster_blocks_per_sm;/* 0 = one block per tile */
  uint32_t result_pool_mib;     /* pinned result memory reserved at creation, MiB; 0 = none
                                   (pinning on demand stalls the request loop for tens of ms
                                   per 64 MiB, so a server that must keep its latency under
                                   load reserves what its outstanding results will hold) */
  uint32_t max_queue_ms;        /* a request still queued this long after submit is shed:
                                   it fails with GSPLAT_ERROR_UNSUPPORTED ("request shed") when a
                                   lane next takes work, so under overload the requests that run
                                   keep a bounded queueing delay; 0 = never shed */
  uint32_t reserved;
} GsplatServeConfig;            /* 48 bytes */

typedef enum GsplatRequestStatus {
  GSPLAT_REQUEST_QUEUED = 0,
  GSPLAT_REQUEST_RUNNING = 1,
  GSPLAT_REQUEST_DONE = 2,
  GSPLAT_REQUEST_FAILED = 3
} GsplatRequestStatus;

typedef struct GsplatRequestInfo {
  uint32_t status;          /* GsplatRequestStatus */
  int32_t error_code;       /* GsplatErrorCode of a failed request */
  uint32_t batch_views;     /* requests in the batch it ran in */
  uint32_t visible_count;
  uint32_t drawn_count;
  uint32_t tile_pairs;
  float latency_ms;         /* submit -> image in host memory */
  float queue_ms;           /* submit -> batch launch */
} GsplatRequestInfo;        /* 32 bytes */

typedef struct GsplatServeStats {
  uint64_t submitted, completed, failed, batches, reruns;
  uint64_t peak_admitted_bytes;  /* predicted workspace of the batches in flight */
  double p50_ms, p99_ms, mean_ms, max_ms;  /* request latency, nearest rank */
  double views_per_s;        /* completed / (last completion - first submit) */
  double mean_batch_views;
  double device_ms;          /* CUDA-event time of the batches' launch sequences, summed */
  double launch_ms;          /* host time spent enqueuing batches, summed */
  double retire_ms;          /* host time spent retiring batches, summed */
  uint64_t graph_captures;   /* launch graphs the lanes captured */
  uint64_t pinned_slabs;     /* pinned result slabs allocated (on demand or in the background) */
  double capture_ms;         /* host time in those captures (part of launch_ms) */
  double pinned_alloc_ms;    /* host time launches waited on allocations (part of launch_ms) */
  uint64_t workspace_regrowths; /* lane workspace reallocations (each waits for an idle device) */
  double regrowth_ms;        /* host time in them (part of launch_ms) */
  uint64_t shed;             /* requests shed after max_queue_ms in the queue (counted in failed) */
} GsplatServeStats;          /* 176 bytes */

int32_t gsplat_server_create(const GsplatServeConfig *config, GsplatServer **out_server);
/* Finishes the batches in flight, fails queued requests and frees everything. */
void gsplat_server_destroy(GsplatServer *server);
int32_t gsplat_server_add_scene_buffers(GsplatServer *server, const GsplatSceneDesc *scene,
                                        uint32_t *out_scene);
int32_t gsplat_server_add_scene_path(GsplatServer *server, const char *path, uint32_t *out_scene);
int32_t gsplat_server_add_scene_packed(GsplatServer *server, const GsplatSceneDesc *scene,
                                       uint32_t *out_scene);
/* Validates the view (scene id, camera, size) and queues it. */
int32_t gsplat_server_submit(GsplatServer *server, const GsplatBatchView *view,
                             uint64_t *out_request);
int32_t gsplat_server_poll(GsplatServer *server, uint64_t request, GsplatRequestInfo *out_info);
/* Waits up to timeout_ms for the request to finish; *out_info tells whether it did. */
int32_t gsplat_server_wait(GsplatServer *server, uint64_t request, uint32_t timeout_ms,
                           GsplatRequestInfo *out_info);
int32_t gsplat_server_read_rgba8(GsplatServer *server, uint64_t request, uint8_t *out,
                                 uint64_t out_len);
/* Forgets a finished request and recycles its image buffer. */
int32_t gsplat_server_release(GsplatServer *server, uint64_t request);
int32_t gsplat_server_get_stats(GsplatServer *server, GsplatServeStats *out_stats);
int32_t gsplat_server_reset_stats(GsplatServer *server);

/* ---- host utilities ---- */

/* Parsed PLY scene owned by the library (crates/gsplat-io-ply/src/lib.rs:178-235). */
typedef struct GsplatHostScene GsplatHostScene;
int32_t gsplat_ply_load(const char *path, GsplatHostScene **out_scene);
void gsplat_host_scene_destroy(GsplatHostScene *scene);
int32_t gsplat_host_scene_view(const GsplatHostScene *scene, GsplatSceneDesc *out_desc);

/* camera_rotation_looking_at (crates/gsplat-ffi-c/src/lib.rs:1677-1733). */
int32_t gsplat_camera_look_at(const float position[3], const float target[3],
                              float vertical_fov_radians, float near_plane, float far_plane,
                              GsplatCamera *out_camera);

/* No counterpart in the reference: the FP32 FMA throughput of the current
 * device, measured by an FMA-only kernel (best of five launches after a
 * warm-up; about 20 ms), in TFLOP/s, and the best launch's time in ms
 * (out_ms may be NULL). The benchmark uses it as the FP32 roofline. */
int32_t gsplat_cuda_measure_fp32_peak(double *out_tflops, double *out_ms);

/* Name, SM count and compute capability of the current CUDA device. */
int32_t gsplat_cuda_device_info(char *name, uint64_t name_capacity, int32_t *sm_count,
                                int32_t *cc_major, int32_t *cc_minor);

#ifdef __cplusplus
}
#endif

#endif /* GSPLAT_CUDA_H */
