/*
 * gsplat.h — the gsplat-rs v0.1 C ABI, served by the B200 CUDA renderer.
 *
 * This header declares the same symbols, enum values and struct layouts as
 * the reference's crates/gsplat-ffi-c/include/gsplat.h (v0.1), so a caller
 * built against that header links against libgsplat_ffi_c.so from this
 * project without source changes. Each declaration cites the reference
 * declaration it stands in for.
 *
 * Conventions (reference gsplat.h:10-23):
 *   - int32_t results are GsplatErrorCode values; gsplat_last_error_message()
 *     describes the last failure on the calling thread ("ok" after success).
 *   - Handles are opaque, owned by the caller after a successful create and
 *     released exactly once by the matching destroy; destroy accepts NULL.
 *   - A handle is confined to one thread (or one serial queue) at a time; the
 *     library adds no locking. Each context owns one CUDA stream on the device
 *     that was current when it was created.
 *   - Rendering is offscreen into device memory; the additive header
 *     gsplat_cuda.h adds readback, in-memory scene loading and debug taps.
 *   - gsplat_surface_renderer_* needs native Android/UIKit window handles and
 *     is not served here: every such call returns GSPLAT_ERROR_UNSUPPORTED
 *     (destroy is a no-op), so the full v0.1 symbol set still links.
 */
#ifndef GSPLAT_FFI_C_GSPLAT_H
#define GSPLAT_FFI_C_GSPLAT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* reference gsplat.h:25-26 */
#define GSPLAT_API_VERSION_MAJOR_VALUE 0
#define GSPLAT_API_VERSION_MINOR_VALUE 1

/* reference gsplat.h:28-36 */
typedef enum GsplatErrorCode {
  GSPLAT_OK = 0,
  GSPLAT_ERROR_INVALID_ARGUMENT = 1,
  GSPLAT_ERROR_NOT_FOUND = 2,
  GSPLAT_ERROR_PARSE_FAILED = 3,
  GSPLAT_ERROR_UNSUPPORTED = 4,
  GSPLAT_ERROR_SCENE_NOT_LOADED = 5,
  GSPLAT_ERROR_INTERNAL = 100,
} GsplatErrorCode;

/* reference gsplat.h:38-41 */
typedef enum GsplatRenderMode {
  GSPLAT_RENDER_MODE_SORTED_ALPHA = 0,
} GsplatRenderMode;

/* reference gsplat.h:47-51 (surface knob; accepted values only) */
typedef enum GsplatGeometryPath {
  GSPLAT_GEOMETRY_PATH_DIRECT = 0,
  GSPLAT_GEOMETRY_PATH_PACKED_ATLAS = 1,
  GSPLAT_GEOMETRY_PATH_PAGED_ACTIVE_ATLAS = 2,
} GsplatGeometryPath;

/* reference gsplat.h:53-58; 12 bytes */
typedef struct GsplatConfig {
  uint32_t width;
  uint32_t height;
  uint32_t mode; /* GsplatRenderMode */
} GsplatConfig;

/* reference gsplat.h:60-67; 24 bytes. frame_ms is the host wall time of the
 * render call; preprocess_ms, sort_ms and raster_ms are device times of the
 * kernel phases measured with CUDA events. */
typedef struct GsplatStats {
  float frame_ms;
  float preprocess_ms;
  float sort_ms;
  float raster_ms;
  uint32_t visible_count;
  uint32_t drawn_count;
} GsplatStats;

/* reference gsplat.h:69-84; 44 bytes + padding */
typedef struct GsplatSurfaceSortStats {
  uint64_t camera_revision;
  uint64_t applied_order_revision;
  uint64_t scheduled_revision;
  uint64_t completed_revision;
  uint32_t presented_order_revision_lag;
  uint32_t observed_result_revision_lag;
  uint32_t flags;
} GsplatSurfaceSortStats;

/* reference gsplat.h:86-92; 40 bytes. RUF world: +X right, +Y up, +Z forward. */
typedef struct GsplatCamera {
  float position[3];
  float rotation_xyzw[4];
  float vertical_fov_radians;
  float near_plane;
  float far_plane;
} GsplatCamera;

typedef struct GsplatContext GsplatContext;
typedef struct GsplatSurfaceRenderer GsplatSurfaceRenderer;

/* reference gsplat.h:97-103 */
uint32_t gsplat_version_major(void);
uint32_t gsplat_version_minor(void);
const char *gsplat_error_message(int32_t code);
const char *gsplat_last_error_message(void);
GsplatConfig gsplat_config_default(void);
GsplatCamera gsplat_camera_default(void);

/* reference gsplat.h:105-111 */
int32_t gsplat_context_create(GsplatConfig config, GsplatContext **out_ctx);
void gsplat_context_destroy(GsplatContext *ctx);
int32_t gsplat_context_set_camera(GsplatContext *ctx, GsplatCamera camera);
int32_t gsplat_context_set_auto_camera(GsplatContext *ctx);
int32_t gsplat_context_load_scene_path(GsplatContext *ctx, const char *path);
int32_t gsplat_context_render_frame(GsplatContext *ctx);
int32_t gsplat_context_get_stats(const GsplatContext *ctx, GsplatStats *out_stats);

/* reference gsplat.h:113-201 — not served here (no native window surfaces);
 * each returns GSPLAT_ERROR_UNSUPPORTED and nulls any out handle. */
int32_t gsplat_surface_renderer_create_android(void *native_window, const char *path,
                                               uint32_t width, uint32_t height,
                                               GsplatSurfaceRenderer **out_renderer);
int32_t gsplat_surface_renderer_create_android_with_geometry_path(
    void *native_window, const char *path, uint32_t width, uint32_t height,
    uint32_t geometry_path, GsplatSurfaceRenderer **out_renderer);
int32_t gsplat_surface_renderer_create_uikit(void *ui_view, void *ui_view_controller,
                                             const char *path, uint32_t width, uint32_t height,
                                             GsplatSurfaceRenderer **out_renderer);
int32_t gsplat_surface_renderer_create_uikit_with_geometry_path(
    void *ui_view, void *ui_view_controller, const char *path, uint32_t width, uint32_t height,
    uint32_t geometry_path, GsplatSurfaceRenderer **out_renderer);
void gsplat_surface_renderer_destroy(GsplatSurfaceRenderer *renderer);
int32_t gsplat_surface_renderer_resize(GsplatSurfaceRenderer *renderer, uint32_t width,
                                       uint32_t height);
int32_t gsplat_surface_renderer_set_sort_interval(GsplatSurfaceRenderer *renderer,
                                                  uint32_t interval);
int32_t gsplat_surface_renderer_set_geometry_path(GsplatSurfaceRenderer *renderer, uint32_t path);
int32_t gsplat_surface_renderer_set_gpu_preproject(GsplatSurfaceRenderer *renderer,
                                                   uint32_t enabled);
int32_t gsplat_surface_renderer_set_gpu_preproject_double_buffer(GsplatSurfaceRenderer *renderer,
                                                                 uint32_t enabled);
int32_t gsplat_surface_renderer_set_async_sort(GsplatSurfaceRenderer *renderer, uint32_t enabled);
int32_t gsplat_surface_renderer_set_async_geometry(GsplatSurfaceRenderer *renderer,
                                                   uint32_t enabled);
int32_t gsplat_surface_renderer_set_instance_buffer_count(GsplatSurfaceRenderer *renderer,
                                                          uint32_t count);
int32_t gsplat_surface_renderer_set_frame_latency(GsplatSurfaceRenderer *renderer,
                                                  uint32_t latency);
int32_t gsplat_surface_renderer_reset_camera(GsplatSurfaceRenderer *renderer);
int32_t gsplat_surface_renderer_orbit(GsplatSurfaceRenderer *renderer, float delta_yaw_radians,
                                      float delta_pitch_radians);
int32_t gsplat_surface_renderer_zoom(GsplatSurfaceRenderer *renderer, float distance_scale);
int32_t gsplat_surface_renderer_pan(GsplatSurfaceRenderer *renderer, float normalized_delta_x,
                                    float normalized_delta_y);
int32_t gsplat_surface_renderer_render_frame(GsplatSurfaceRenderer *renderer);
int32_t gsplat_surface_renderer_get_stats(const GsplatSurfaceRenderer *renderer,
                                          GsplatStats *out_stats);
int32_t gsplat_surface_renderer_get_sort_stats(const GsplatSurfaceRenderer *renderer,
                                               GsplatSurfaceSortStats *out_stats);

#ifdef __cplusplus
}
#endif

#endif /* GSPLAT_FFI_C_GSPLAT_H */
