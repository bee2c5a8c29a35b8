// extern "C" surface: the gsplat.h v0.1 ABI (crates/gsplat-ffi-c/src/lib.rs)
// plus the additive gsplat_cuda.h exports. Every entry catches exceptions and
// turns them into a GsplatErrorCode and a thread-local message, like the
// reference's ffi_catch_* wrappers (lib.rs:225-255).

#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "../../include/gsplat.h"
#include "../../include/gsplat_cuda.h"
#include "gsr_host.h"
#include "autotune.h"
#include "cuda_check.h"
#include "batch.h"
#include "renderer.h"
#include "server.h"
#include "sort_api.h"

using gsr::Code;
using gsr::Error;

struct GsplatContext {
  GsplatConfig config;
  GsplatCamera camera;
  std::unique_ptr<gsr::Renderer> renderer;
  GsplatStats stats;
};

struct GsplatBatch {
  std::unique_ptr<gsr::Batch> batch;
};

struct GsplatServer {
  std::unique_ptr<gsr::Server> server;
};

struct GsplatHostScene {
  gsr::HostScene scene;
};

namespace {

thread_local std::string g_last_error = "ok";

int32_t ok() {
  g_last_error = "ok";
  return 0;
}

int32_t fail(Code c, const std::string &msg) {
  g_last_error = msg;
  return (int32_t)c;
}

// Runs `body`, mapping exceptions to error codes with "<op>: <what>".
template <typename F>
int32_t guarded(const char *op, F &&body) {
  try {
    return body();
  } catch (const Error &e) {
    return fail(e.code, std::string(op) + ": " + e.what());
  } catch (const std::bad_alloc &) {
    return fail(Code::Internal, std::string(op) + ": host allocation failed");
  } catch (const std::exception &e) {
    return fail(Code::Internal, std::string(op) + ": " + e.what());
  } catch (...) {
    return fail(Code::Internal, std::string(op) + ": exception caught at C ABI boundary");
  }
}

// str::from_utf8 check of the reference (lib.rs:481-489).
bool valid_utf8(const std::string &p) {
  for (size_t i = 0; i < p.size();) {
    unsigned char c = (unsigned char)p[i];
    size_t len = c < 0x80 ? 1 : (c >> 5) == 6 ? 2 : (c >> 4) == 14 ? 3 : (c >> 3) == 30 ? 4 : 0;
    bool good = len != 0 && i + len <= p.size();
    for (size_t k = 1; good && k < len; ++k) good = ((unsigned char)p[i + k] & 0xC0) == 0x80;
    if (!good) return false;
    i += len;
  }
  return true;
}

gsr::HostScene host_scene_from_desc(const GsplatSceneDesc &d) {
  gsr::HostScene s;
  const uint64_t n = d.count;
  if (n && (!d.positions || !d.opacity || !d.scale_xyz || !d.rotation_xyzw || !d.color_dc))
    throw Error(Code::InvalidArgument, "scene arrays must not be null");
  s.positions.assign(d.positions, d.positions + 3 * n);
  s.opacity.assign(d.opacity, d.opacity + n);
  s.scale_xyz.assign(d.scale_xyz, d.scale_xyz + 3 * n);
  s.rotation_xyzw.assign(d.rotation_xyzw, d.rotation_xyzw + 4 * n);
  s.color_dc.assign(d.color_dc, d.color_dc + 3 * n);
  s.sh_degree = d.sh_degree;
  if (d.sh_rest) {
    if (d.sh_degree == 0 || d.sh_degree > 4)
      throw Error(d.sh_degree > 4 ? Code::Unsupported : Code::InvalidArgument,
                  "sh_rest given for an unsupported SH degree");
    s.has_sh_rest = true;
    s.sh_rest.assign(d.sh_rest, d.sh_rest + n * gsr::sh_rest_stride(d.sh_degree));
  }
  return s;
}

}  // namespace

extern "C" {

// ---- shared functions: reference gsplat.h:97-103, ffi-c/src/lib.rs:257-320 ----

uint32_t gsplat_version_major(void) { return GSPLAT_API_VERSION_MAJOR_VALUE; }
uint32_t gsplat_version_minor(void) { return GSPLAT_API_VERSION_MINOR_VALUE; }

const char *gsplat_error_message(int32_t code) {
  switch (code) {
    case 0: return "ok";
    case 1: return "invalid argument";
    case 2: return "not found";
    case 3: return "parse failed";
    case 4: return "unsupported";
    case 5: return "scene not loaded";
    case 100: return "internal error";
    default: return "unknown error";
  }
}

const char *gsplat_last_error_message(void) { return g_last_error.c_str(); }

GsplatConfig gsplat_config_default(void) { return gsr::config_default(); }
GsplatCamera gsplat_camera_default(void) { return gsr::camera_default(); }

// ---- context: reference gsplat.h:105-111, ffi-c/src/lib.rs:329-570 ----

int32_t gsplat_context_create(GsplatConfig config, GsplatContext **out_ctx) {
  return guarded("gsplat_context_create", [&]() -> int32_t {
    if (!out_ctx) return fail(Code::InvalidArgument, "gsplat_context_create: out_ctx is null");
    *out_ctx = nullptr;
    if (config.mode != GSPLAT_RENDER_MODE_SORTED_ALPHA)
      return fail(Code::InvalidArgument, "gsplat_context_create: unsupported render mode");
    if (config.width == 0 || config.height == 0)
      return fail(Code::InvalidArgument,
                  "gsplat_context_create: invalid renderer configuration");
    auto ctx = std::make_unique<GsplatContext>();
    ctx->config = config;
    ctx->camera = gsr::camera_default();
    std::memset(&ctx->stats, 0, sizeof(ctx->stats));
    ctx->renderer = std::make_unique<gsr::Renderer>(config.width, config.height);
    *out_ctx = ctx.release();
    return ok();
  });
}

void gsplat_context_destroy(GsplatContext *ctx) {
  try {
    delete ctx;
  } catch (...) {
    g_last_error = "gsplat_context_destroy: exception caught at C ABI boundary";
  }
}

int32_t gsplat_context_set_camera(GsplatContext *ctx, GsplatCamera camera) {
  return guarded("gsplat_context_set_camera", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_set_camera: ctx is null");
    if (!gsr::camera_valid(camera))
      return fail(Code::InvalidArgument, "gsplat_context_set_camera: invalid camera");
    ctx->camera = camera;
    return ok();
  });
}

int32_t gsplat_context_set_auto_camera(GsplatContext *ctx) {
  return guarded("gsplat_context_set_auto_camera", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_set_auto_camera: ctx is null");
    const gsr::DeviceScene *sc = ctx->renderer->scene();
    if (!sc)
      return fail(Code::SceneNotLoaded, "gsplat_context_set_auto_camera: scene is not loaded");
    if (sc->n == 0)
      return fail(Code::InvalidArgument, "gsplat_context_set_auto_camera: scene is not loaded");
    ctx->camera = gsr::auto_camera(sc->positions.data(), sc->n, ctx->config.width,
                                   ctx->config.height);
    return ok();
  });
}

int32_t gsplat_context_load_scene_path(GsplatContext *ctx, const char *path) {
  return guarded("gsplat_context_load_scene_path", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_load_scene_path: ctx is null");
    if (!path) return fail(Code::InvalidArgument, "gsplat_context_load_scene_path: path is null");
    std::string p(path);
    if (!valid_utf8(p))
      return fail(Code::InvalidArgument, "gsplat_context_load_scene_path: path is not valid UTF-8");
    ctx->renderer->load_scene_path(p);
    return ok();
  });
}

int32_t gsplat_context_render_frame(GsplatContext *ctx) {
  return guarded("gsplat_context_render_frame", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_render_frame: ctx is null");
    gsr::FrameResult r = ctx->renderer->render(ctx->camera);
    ctx->stats.frame_ms = r.frame_ms;
    ctx->stats.preprocess_ms = r.preprocess_ms;
    ctx->stats.sort_ms = r.sort_ms;
    ctx->stats.raster_ms = r.raster_ms;
    ctx->stats.visible_count = (uint32_t)r.visible;
    // drawn_count is the number of instances handed to the raster, which on
    // the reference's CPU-order path is every depth-visible splat (lib.rs:736).
    ctx->stats.drawn_count = (uint32_t)r.visible;
    return ok();
  });
}

int32_t gsplat_context_get_stats(const GsplatContext *ctx, GsplatStats *out_stats) {
  return guarded("gsplat_context_get_stats", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_get_stats: ctx is null");
    if (!out_stats) return fail(Code::InvalidArgument, "gsplat_context_get_stats: out_stats is null");
    *out_stats = ctx->stats;
    return ok();
  });
}

// ---- surface renderer: reference gsplat.h:113-201 (not served here) ----

#define GSR_SURFACE_UNSUPPORTED(name)                                                       \
  return fail(Code::Unsupported, std::string(name) +                                        \
                                     ": native window surfaces are not served by the CUDA " \
                                     "renderer; use gsplat_context_* for offscreen frames")

int32_t gsplat_surface_renderer_create_android(void *, const char *, uint32_t, uint32_t,
                                               GsplatSurfaceRenderer **out) {
  if (out) *out = nullptr;
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_create_android");
}
int32_t gsplat_surface_renderer_create_android_with_geometry_path(void *, const char *, uint32_t,
                                                                  uint32_t, uint32_t,
                                                                  GsplatSurfaceRenderer **out) {
  if (out) *out = nullptr;
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_create_android_with_geometry_path");
}
int32_t gsplat_surface_renderer_create_uikit(void *, void *, const char *, uint32_t, uint32_t,
                                             GsplatSurfaceRenderer **out) {
  if (out) *out = nullptr;
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_create_uikit");
}
int32_t gsplat_surface_renderer_create_uikit_with_geometry_path(void *, void *, const char *,
                                                                uint32_t, uint32_t, uint32_t,
                                                                GsplatSurfaceRenderer **out) {
  if (out) *out = nullptr;
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_create_uikit_with_geometry_path");
}
void gsplat_surface_renderer_destroy(GsplatSurfaceRenderer *) {}
int32_t gsplat_surface_renderer_resize(GsplatSurfaceRenderer *, uint32_t, uint32_t) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_resize");
}
int32_t gsplat_surface_renderer_set_sort_interval(GsplatSurfaceRenderer *, uint32_t) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_set_sort_interval");
}
int32_t gsplat_surface_renderer_set_geometry_path(GsplatSurfaceRenderer *, uint32_t) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_set_geometry_path");
}
int32_t gsplat_surface_renderer_set_gpu_preproject(GsplatSurfaceRenderer *, uint32_t) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_set_gpu_preproject");
}
int32_t gsplat_surface_renderer_set_gpu_preproject_double_buffer(GsplatSurfaceRenderer *, uint32_t) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_set_gpu_preproject_double_buffer");
}
int32_t gsplat_surface_renderer_set_async_sort(GsplatSurfaceRenderer *, uint32_t) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_set_async_sort");
}
int32_t gsplat_surface_renderer_set_async_geometry(GsplatSurfaceRenderer *, uint32_t) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_set_async_geometry");
}
int32_t gsplat_surface_renderer_set_instance_buffer_count(GsplatSurfaceRenderer *, uint32_t) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_set_instance_buffer_count");
}
int32_t gsplat_surface_renderer_set_frame_latency(GsplatSurfaceRenderer *, uint32_t) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_set_frame_latency");
}
int32_t gsplat_surface_renderer_reset_camera(GsplatSurfaceRenderer *) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_reset_camera");
}
int32_t gsplat_surface_renderer_orbit(GsplatSurfaceRenderer *, float, float) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_orbit");
}
int32_t gsplat_surface_renderer_zoom(GsplatSurfaceRenderer *, float) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_zoom");
}
int32_t gsplat_surface_renderer_pan(GsplatSurfaceRenderer *, float, float) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_pan");
}
int32_t gsplat_surface_renderer_render_frame(GsplatSurfaceRenderer *) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_render_frame");
}
int32_t gsplat_surface_renderer_get_stats(const GsplatSurfaceRenderer *, GsplatStats *) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_get_stats");
}
int32_t gsplat_surface_renderer_get_sort_stats(const GsplatSurfaceRenderer *,
                                               GsplatSurfaceSortStats *) {
  GSR_SURFACE_UNSUPPORTED("gsplat_surface_renderer_get_sort_stats");
}

// ---- additive exports (gsplat_cuda.h) ----

int32_t gsplat_context_set_size(GsplatContext *ctx, uint32_t width, uint32_t height) {
  return guarded("gsplat_context_set_size", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_set_size: ctx is null");
    ctx->renderer->set_size(width, height);
    ctx->config.width = width;
    ctx->config.height = height;
    return ok();
  });
}

int32_t gsplat_context_get_config(const GsplatContext *ctx, GsplatConfig *out) {
  return guarded("gsplat_context_get_config", [&]() -> int32_t {
    if (!ctx || !out) return fail(Code::InvalidArgument, "gsplat_context_get_config: null argument");
    *out = ctx->config;
    return ok();
  });
}

int32_t gsplat_context_get_camera(const GsplatContext *ctx, GsplatCamera *out) {
  return guarded("gsplat_context_get_camera", [&]() -> int32_t {
    if (!ctx || !out) return fail(Code::InvalidArgument, "gsplat_context_get_camera: null argument");
    *out = ctx->camera;
    return ok();
  });
}

int32_t gsplat_context_set_blend_mode(GsplatContext *ctx, uint32_t mode) {
  return guarded("gsplat_context_set_blend_mode", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_set_blend_mode: ctx is null");
    if (mode > 1) return fail(Code::InvalidArgument, "gsplat_context_set_blend_mode: unknown mode");
    ctx->renderer->set_blend_mode(mode);
    return ok();
  });
}

int32_t gsplat_context_set_tile_size(GsplatContext *ctx, uint32_t tile) {
  return guarded("gsplat_context_set_tile_size", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_set_tile_size: ctx is null");
    ctx->renderer->set_tile(tile);
    return ok();
  });
}

int32_t gsplat_context_set_debug_taps(GsplatContext *ctx, uint32_t enabled) {
  return guarded("gsplat_context_set_debug_taps", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_set_debug_taps: ctx is null");
    ctx->renderer->set_debug(enabled != 0);
    return ok();
  });
}

int32_t gsplat_context_set_cuda_graph(GsplatContext *ctx, uint32_t enabled) {
  return guarded("gsplat_context_set_cuda_graph", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_set_cuda_graph: ctx is null");
    ctx->renderer->set_use_graph(enabled != 0);
    return ok();
  });
}

int32_t gsplat_context_set_raster_config(GsplatContext *ctx, uint32_t chunk, uint32_t blocks_per_sm) {
  return guarded("gsplat_context_set_raster_config", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_set_raster_config: ctx is null");
    gsr::RasterConfig c;
    c.chunk = chunk;
    c.blocks_per_sm = blocks_per_sm;
    ctx->renderer->set_raster_config(c);
    return ok();
  });
}

int32_t gsplat_context_set_sort_interval(GsplatContext *ctx, uint32_t interval) {
  return guarded("gsplat_context_set_sort_interval", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_set_sort_interval: ctx is null");
    ctx->renderer->set_sort_interval(interval);
    return ok();
  });
}

int32_t gsplat_context_set_frame_lanes(GsplatContext *ctx, uint32_t lanes) {
  return guarded("gsplat_context_set_frame_lanes", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_set_frame_lanes: ctx is null");
    ctx->renderer->set_frame_lanes(lanes);
    return ok();
  });
}

int32_t gsplat_context_load_scene_buffers(GsplatContext *ctx, const GsplatSceneDesc *scene) {
  return guarded("gsplat_context_load_scene_buffers", [&]() -> int32_t {
    if (!ctx || !scene)
      return fail(Code::InvalidArgument, "gsplat_context_load_scene_buffers: null argument");
    gsr::HostScene s = host_scene_from_desc(*scene);
    ctx->renderer->load_scene(s);
    return ok();
  });
}

int32_t gsplat_context_load_scene_packed(GsplatContext *ctx, const GsplatSceneDesc *scene) {
  return guarded("gsplat_context_load_scene_packed", [&]() -> int32_t {
    if (!ctx || !scene)
      return fail(Code::InvalidArgument, "gsplat_context_load_scene_packed: null argument");
    gsr::HostScene s = host_scene_from_desc(*scene);
    ctx->renderer->load_scene_packed(s);
    return ok();
  });
}

int32_t gsplat_context_readback_rgba8(GsplatContext *ctx, uint8_t *out, uint64_t out_len) {
  return guarded("gsplat_context_readback_rgba8", [&]() -> int32_t {
    if (!ctx || !out) return fail(Code::InvalidArgument, "gsplat_context_readback_rgba8: null argument");
    ctx->renderer->readback_rgba8(out, out_len);
    return ok();
  });
}

int32_t gsplat_context_readback_rgba8_async(GsplatContext *ctx, uint8_t *out, uint64_t out_len) {
  return guarded("gsplat_context_readback_rgba8_async", [&]() -> int32_t {
    if (!ctx || !out)
      return fail(Code::InvalidArgument, "gsplat_context_readback_rgba8_async: null argument");
    ctx->renderer->readback_rgba8_async(out, out_len);
    return ok();
  });
}

int32_t gsplat_context_get_frame_counts(const GsplatContext *ctx, GsplatFrameCounts *out) {
  return guarded("gsplat_context_get_frame_counts", [&]() -> int32_t {
    if (!ctx || !out) return fail(Code::InvalidArgument, "gsplat_context_get_frame_counts: null argument");
    const gsr::Renderer &r = *ctx->renderer;
    const gsr::FrameResult &f = r.last();
    std::memset(out, 0, sizeof(*out));
    out->visible = f.visible;
    out->drawn = f.drawn;
    out->tile_keys = f.keys;
    out->key_capacity = r.key_capacity();
    out->tile_size = r.tile();
    out->tiles_x = (r.width() + r.tile() - 1) / r.tile();
    out->tiles_y = (r.height() + r.tile() - 1) / r.tile();
    out->blend_mode = r.blend_mode();
    out->preprocess_ms = f.preprocess_ms;
    out->sort_ms = f.sort_ms;
    out->raster_ms = f.raster_ms;
    out->frame_ms = f.frame_ms;
    out->frame_reruns = f.reruns;
    out->sort_refreshed = f.sorted ? 1u : 0u;
    return ok();
  });
}

int32_t gsplat_context_get_phase_times(const GsplatContext *ctx, float *out, uint32_t capacity,
                                       uint32_t *out_count) {
  return guarded("gsplat_context_get_phase_times", [&]() -> int32_t {
    if (!ctx || !out_count) return fail(Code::InvalidArgument, "gsplat_context_get_phase_times: null argument");
    const gsr::FrameResult &f = ctx->renderer->last();
    *out_count = gsr::kPhaseCount;
    for (uint32_t k = 0; out && k < capacity && k < (uint32_t)gsr::kPhaseCount; ++k) out[k] = f.phase_ms[k];
    return ok();
  });
}

int32_t gsplat_context_render_frame_async(GsplatContext *ctx) {
  return guarded("gsplat_context_render_frame_async", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_render_frame_async: ctx is null");
    ctx->renderer->render_async(ctx->camera);
    return ok();
  });
}

int32_t gsplat_context_sync(GsplatContext *ctx) {
  return guarded("gsplat_context_sync", [&]() -> int32_t {
    if (!ctx) return fail(Code::InvalidArgument, "gsplat_context_sync: ctx is null");
    ctx->renderer->sync();
    const gsr::FrameResult &r = ctx->renderer->last();
    ctx->stats.preprocess_ms = r.preprocess_ms;
    ctx->stats.sort_ms = r.sort_ms;
    ctx->stats.raster_ms = r.raster_ms;
    ctx->stats.frame_ms = r.preprocess_ms + r.sort_ms + r.raster_ms;
    ctx->stats.visible_count = (uint32_t)r.visible;
    ctx->stats.drawn_count = (uint32_t)r.visible;
    return ok();
  });
}

int32_t gsplat_context_get_stream(const GsplatContext *ctx, void **out_stream) {
  return guarded("gsplat_context_get_stream", [&]() -> int32_t {
    if (!ctx || !out_stream) return fail(Code::InvalidArgument, "gsplat_context_get_stream: null argument");
    *out_stream = (void *)ctx->renderer->stream();
    return ok();
  });
}

int32_t gsplat_context_debug_order(GsplatContext *ctx, uint32_t *out, uint64_t capacity,
                                   uint64_t *out_len) {
  return guarded("gsplat_context_debug_order", [&]() -> int32_t {
    if (!ctx || !out_len) return fail(Code::InvalidArgument, "gsplat_context_debug_order: null argument");
    auto v = ctx->renderer->debug_order();
    *out_len = v.size();
    if (out) std::memcpy(out, v.data(), 4 * std::min<uint64_t>(capacity, v.size()));
    return ok();
  });
}

int32_t gsplat_context_debug_scene(GsplatContext *ctx, float *out, uint64_t capacity,
                                   uint64_t *out_len) {
  return guarded("gsplat_context_debug_scene", [&]() -> int32_t {
    if (!ctx || !out_len) return fail(Code::InvalidArgument, "gsplat_context_debug_scene: null argument");
    const gsr::DeviceScene *sc = ctx->renderer->scene();
    if (!sc) return fail(Code::SceneNotLoaded, "gsplat_context_debug_scene: no scene loaded");
    if (sc->dev.hot)
      return fail(Code::InvalidArgument, "gsplat_context_debug_scene: scene is packed");
    const uint64_t n = sc->n, planes = sc->dev.planes;
    *out_len = 4 * n * (3 + planes);
    if (!out || n == 0) return ok();
    const float4 *src[4] = {sc->dev.pos_alpha, sc->dev.cov_a, sc->dev.cov_b, sc->dev.color};
    const uint64_t count[4] = {n, n, n, n * planes};
    uint64_t at = 0;
    for (int k = 0; k < 4 && at < capacity; ++k) {
      const uint64_t floats = std::min<uint64_t>(4 * count[k], capacity - at);
      GSR_CUDA(cudaMemcpy(out + at, src[k], 4 * floats, cudaMemcpyDeviceToHost));
      at += floats;
    }
    return ok();
  });
}

int32_t gsplat_context_debug_packed_scene(GsplatContext *ctx, float *table, uint32_t *hot,
                                          int8_t *sidecar, uint64_t *out_splats) {
  return guarded("gsplat_context_debug_packed_scene", [&]() -> int32_t {
    if (!ctx || !out_splats)
      return fail(Code::InvalidArgument, "gsplat_context_debug_packed_scene: null argument");
    const gsr::DeviceScene *sc = ctx->renderer->scene();
    if (!sc) return fail(Code::SceneNotLoaded, "gsplat_context_debug_packed_scene: no scene loaded");
    if (!sc->dev.hot)
      return fail(Code::InvalidArgument, "gsplat_context_debug_packed_scene: scene is not packed");
    const uint64_t n = sc->n;
    *out_splats = n;
    if (table)
      GSR_CUDA(cudaMemcpy(table, sc->dev.packed, 4 * gsr::kPackedFloats, cudaMemcpyDeviceToHost));
    if (hot && n) GSR_CUDA(cudaMemcpy(hot, sc->dev.hot, 20 * n, cudaMemcpyDeviceToHost));
    if (sidecar && n && sc->dev.sidecar)
      GSR_CUDA(cudaMemcpy(sidecar, sc->dev.sidecar, 48 * n, cudaMemcpyDeviceToHost));
    return ok();
  });
}

int32_t gsplat_context_debug_projected(GsplatContext *ctx, GsplatProjectedSplat *out,
                                       uint64_t capacity, uint64_t *out_len) {
  return guarded("gsplat_context_debug_projected", [&]() -> int32_t {
    if (!ctx || !out_len) return fail(Code::InvalidArgument, "gsplat_context_debug_projected: null argument");
    static_assert(sizeof(GsplatProjectedSplat) == sizeof(gsr::ProjectedDev), "layout");
    auto v = ctx->renderer->debug_projected();
    *out_len = v.size();
    if (out) std::memcpy(out, v.data(), sizeof(GsplatProjectedSplat) * std::min<uint64_t>(capacity, v.size()));
    return ok();
  });
}

int32_t gsplat_context_debug_coverage(GsplatContext *ctx, float *out, uint64_t capacity,
                                      uint64_t *out_len) {
  return guarded("gsplat_context_debug_coverage", [&]() -> int32_t {
    if (!ctx || !out_len) return fail(Code::InvalidArgument, "gsplat_context_debug_coverage: null argument");
    auto v = ctx->renderer->debug_coverage();
    *out_len = v.size();
    if (out) std::memcpy(out, v.data(), sizeof(float2) * std::min<uint64_t>(capacity, v.size()));
    return ok();
  });
}

int32_t gsplat_context_debug_tile_pairs(GsplatContext *ctx, uint32_t *tiles, uint32_t *ids,
                                        uint64_t capacity, uint64_t *out_len) {
  return guarded("gsplat_context_debug_tile_pairs", [&]() -> int32_t {
    if (!ctx || !out_len) return fail(Code::InvalidArgument, "gsplat_context_debug_tile_pairs: null argument");
    std::vector<uint32_t> t, i;
    ctx->renderer->debug_tile_pairs(t, i);
    *out_len = t.size();
    uint64_t m = std::min<uint64_t>(capacity, t.size());
    if (tiles) std::memcpy(tiles, t.data(), 4 * m);
    if (ids) std::memcpy(ids, i.data(), 4 * m);
    return ok();
  });
}

int32_t gsplat_context_debug_tile_ranges(GsplatContext *ctx, uint32_t *ranges,
                                         uint64_t ranges_capacity, uint32_t *ids,
                                         uint64_t ids_capacity, uint64_t *out_keys) {
  return guarded("gsplat_context_debug_tile_ranges", [&]() -> int32_t {
    if (!ctx || !out_keys) return fail(Code::InvalidArgument, "gsplat_context_debug_tile_ranges: null argument");
    std::vector<uint32_t> r, i;
    ctx->renderer->debug_tile_ranges(r, i);
    *out_keys = i.size();
    if (ranges) std::memcpy(ranges, r.data(), 4 * std::min<uint64_t>(ranges_capacity, r.size()));
    if (ids) std::memcpy(ids, i.data(), 4 * std::min<uint64_t>(ids_capacity, i.size()));
    return ok();
  });
}

int32_t gsplat_cuda_sort_values_by_keys(const uint32_t *keys, uint32_t *values, uint64_t len) {
  return guarded("gsplat_cuda_sort_values_by_keys", [&]() -> int32_t {
    if (len && (!keys || !values))
      return fail(Code::InvalidArgument, "gsplat_cuda_sort_values_by_keys: null argument");
    gsr::sort_values_by_keys_host(keys, values, len);
    return ok();
  });
}

int32_t gsplat_cuda_sort_pairs(uint32_t *keys, uint32_t *values, uint64_t len) {
  return guarded("gsplat_cuda_sort_pairs", [&]() -> int32_t {
    if (len && (!keys || !values))
      return fail(Code::InvalidArgument, "gsplat_cuda_sort_pairs: null argument");
    gsr::sort_pairs_host(keys, values, len);
    return ok();
  });
}

int32_t gsplat_cuda_sort_values_by_keys_noalloc(const uint32_t *keys, uint32_t *values,
                                                uint64_t len, void *stream) {
  return guarded("gsplat_cuda_sort_values_by_keys_noalloc", [&]() -> int32_t {
    std::string msg;
    Code c = gsr::sort_values_by_keys_noalloc(keys, values, len, (cudaStream_t)stream, msg);
    if (c != Code::Ok) return fail(c, "gsplat_cuda_sort_values_by_keys_noalloc: " + msg);
    return ok();
  });
}

int32_t gsplat_ply_load(const char *path, GsplatHostScene **out_scene) {
  return guarded("gsplat_ply_load", [&]() -> int32_t {
    if (!out_scene) return fail(Code::InvalidArgument, "gsplat_ply_load: out_scene is null");
    *out_scene = nullptr;
    if (!path) return fail(Code::InvalidArgument, "gsplat_ply_load: path is null");
    auto hs = std::make_unique<GsplatHostScene>();
    hs->scene = gsr::load_ply(path);
    *out_scene = hs.release();
    return ok();
  });
}

void gsplat_host_scene_destroy(GsplatHostScene *scene) { delete scene; }

int32_t gsplat_host_scene_view(const GsplatHostScene *scene, GsplatSceneDesc *out) {
  return guarded("gsplat_host_scene_view", [&]() -> int32_t {
    if (!scene || !out) return fail(Code::InvalidArgument, "gsplat_host_scene_view: null argument");
    const gsr::HostScene &s = scene->scene;
    out->count = s.size();
    out->sh_degree = s.sh_degree;
    out->reserved = 0;
    out->positions = s.positions.data();
    out->opacity = s.opacity.data();
    out->scale_xyz = s.scale_xyz.data();
    out->rotation_xyzw = s.rotation_xyzw.data();
    out->color_dc = s.color_dc.data();
    out->sh_rest = s.has_sh_rest ? s.sh_rest.data() : nullptr;
    return ok();
  });
}

int32_t gsplat_camera_look_at(const float position[3], const float target[3],
                              float vertical_fov_radians, float near_plane, float far_plane,
                              GsplatCamera *out) {
  return guarded("gsplat_camera_look_at", [&]() -> int32_t {
    if (!position || !target || !out) return fail(Code::InvalidArgument, "gsplat_camera_look_at: null argument");
    GsplatCamera c;
    for (int k = 0; k < 3; ++k) c.position[k] = position[k];
    gsr::camera_rotation_looking_at(position, target, c.rotation_xyzw);
    c.vertical_fov_radians = vertical_fov_radians;
    c.near_plane = near_plane;
    c.far_plane = far_plane;
    if (!gsr::camera_valid(c)) return fail(Code::InvalidArgument, "gsplat_camera_look_at: invalid camera");
    *out = c;
    return ok();
  });
}

int32_t gsplat_cuda_device_info(char *name, uint64_t name_capacity, int32_t *sm_count,
                                int32_t *cc_major, int32_t *cc_minor) {
  return guarded("gsplat_cuda_device_info", [&]() -> int32_t {
    gsr::device_info(name, name_capacity, sm_count, cc_major, cc_minor);
    return ok();
  });
}

int32_t gsplat_cuda_measure_fp32_peak(double *out_tflops, double *out_ms) {
  return guarded("gsplat_cuda_measure_fp32_peak", [&]() -> int32_t {
    if (!out_tflops) return fail(Code::InvalidArgument, "gsplat_cuda_measure_fp32_peak: out is null");
    gsr::measure_fp32_peak(out_tflops, out_ms);
    return ok();
  });
}

// ---- batched frames (gsplat_cuda.h) ----------------------------------------

int32_t gsplat_batch_create(GsplatBatch **out_batch) {
  return guarded("gsplat_batch_create", [&]() -> int32_t {
    if (!out_batch) return fail(Code::InvalidArgument, "gsplat_batch_create: out_batch is null");
    *out_batch = nullptr;
    auto b = std::make_unique<GsplatBatch>();
    b->batch = std::make_unique<gsr::Batch>();
    *out_batch = b.release();
    return ok();
  });
}

void gsplat_batch_destroy(GsplatBatch *batch) {
  try {
    delete batch;
  } catch (...) {
  }
}

#define GSR_BATCH_CHECK(op) \
  if (!batch || !batch->batch) return fail(Code::InvalidArgument, op ": batch is null")

int32_t gsplat_batch_set_scene_budget(GsplatBatch *batch, uint64_t bytes) {
  return guarded("gsplat_batch_set_scene_budget", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_set_scene_budget");
    batch->batch->scenes().set_budget(bytes);
    return ok();
  });
}

int32_t gsplat_batch_add_scene_buffers(GsplatBatch *batch, const GsplatSceneDesc *scene,
                                       uint32_t *out_scene) {
  return guarded("gsplat_batch_add_scene_buffers", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_add_scene_buffers");
    if (!scene || !out_scene)
      return fail(Code::InvalidArgument, "gsplat_batch_add_scene_buffers: null argument");
    gsr::HostScene s = host_scene_from_desc(*scene);
    *out_scene = batch->batch->scenes().add(s, batch->batch->stream());
    return ok();
  });
}

int32_t gsplat_batch_add_scene_packed(GsplatBatch *batch, const GsplatSceneDesc *scene,
                                      uint32_t *out_scene) {
  return guarded("gsplat_batch_add_scene_packed", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_add_scene_packed");
    if (!scene || !out_scene)
      return fail(Code::InvalidArgument, "gsplat_batch_add_scene_packed: null argument");
    gsr::HostScene s = host_scene_from_desc(*scene);
    *out_scene = batch->batch->scenes().add_packed(s, batch->batch->stream());
    return ok();
  });
}

int32_t gsplat_batch_add_scene_path(GsplatBatch *batch, const char *path, uint32_t *out_scene) {
  return guarded("gsplat_batch_add_scene_path", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_add_scene_path");
    if (!path || !out_scene)
      return fail(Code::InvalidArgument, "gsplat_batch_add_scene_path: null argument");
    std::string p(path);
    if (!valid_utf8(p))
      return fail(Code::InvalidArgument, "gsplat_batch_add_scene_path: path is not valid UTF-8");
    *out_scene = batch->batch->scenes().add_path(p, batch->batch->stream());
    return ok();
  });
}

int32_t gsplat_batch_set_tile_size(GsplatBatch *batch, uint32_t tile) {
  return guarded("gsplat_batch_set_tile_size", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_set_tile_size");
    batch->batch->set_tile(tile);
    return ok();
  });
}

int32_t gsplat_batch_set_blend_mode(GsplatBatch *batch, uint32_t mode) {
  return guarded("gsplat_batch_set_blend_mode", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_set_blend_mode");
    batch->batch->set_blend_mode(mode);
    return ok();
  });
}

int32_t gsplat_batch_set_limits(GsplatBatch *batch, uint32_t max_views, uint64_t max_pairs,
                                uint64_t max_splats, uint64_t max_tiles) {
  return guarded("gsplat_batch_set_limits", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_set_limits");
    gsr::GroupLimits l = batch->batch->limits();
    if (max_views) l.max_views = max_views;
    if (max_pairs) l.max_pairs = max_pairs;
    if (max_splats) l.max_splats = max_splats;
    if (max_tiles) l.max_tiles = max_tiles;
    batch->batch->set_limits(l);
    return ok();
  });
}

int32_t gsplat_batch_set_raster_config(GsplatBatch *batch, uint32_t chunk, uint32_t blocks_per_sm) {
  return guarded("gsplat_batch_set_raster_config", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_set_raster_config");
    gsr::RasterConfig c;
    c.chunk = chunk;
    c.blocks_per_sm = blocks_per_sm;
    batch->batch->set_raster_config(c);
    return ok();
  });
}

static std::vector<gsr::BatchView> to_batch_views(const GsplatBatchView *views, uint32_t count) {
  std::vector<gsr::BatchView> v(count);
  for (uint32_t i = 0; i < count; ++i) {
    if (views[i].reserved != 0) throw Error(Code::InvalidArgument, "reserved field must be 0");
    v[i] = gsr::BatchView{views[i].scene, views[i].camera, views[i].width, views[i].height};
  }
  return v;
}

int32_t gsplat_batch_autotune(GsplatBatch *batch, const GsplatBatchView *views, uint32_t count,
                              const char *cache_path, uint32_t reps, GsplatTuneResult *out_result) {
  return guarded("gsplat_batch_autotune", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_autotune");
    if (!views || count == 0 || !out_result)
      return fail(Code::InvalidArgument, "gsplat_batch_autotune: null argument or no views");
    gsr::TuneResult r = gsr::autotune(*batch->batch, to_batch_views(views, count),
                                      cache_path ? std::string(cache_path) : std::string(), reps);
    *out_result = GsplatTuneResult{r.best.tile, r.best.raster.chunk, r.best.raster.blocks_per_sm,
                                   (uint32_t)r.tried.size(), r.best.ms, r.default_ms,
                                   r.from_cache ? 1u : 0u, 0};
    return ok();
  });
}

int32_t gsplat_batch_render(GsplatBatch *batch, const GsplatBatchView *views, uint32_t count) {
  return guarded("gsplat_batch_render", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_render");
    if (!views || count == 0) return fail(Code::InvalidArgument, "gsplat_batch_render: no views");
    batch->batch->render(to_batch_views(views, count));
    return ok();
  });
}

int32_t gsplat_batch_get_times(const GsplatBatch *batch, GsplatBatchTimes *out_times) {
  return guarded("gsplat_batch_get_times", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_get_times");
    if (!out_times) return fail(Code::InvalidArgument, "gsplat_batch_get_times: out_times is null");
    const gsr::BatchResult &r = batch->batch->last();
    *out_times = GsplatBatchTimes{r.device_ms, r.wall_ms, r.groups, r.reruns, r.launches, r.graph_launches, r.pairs};
    return ok();
  });
}

int32_t gsplat_batch_set_phase_timing(GsplatBatch *batch, uint32_t on) {
  return guarded("gsplat_batch_set_phase_timing", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_set_phase_timing");
    if (on > 1) return fail(Code::InvalidArgument, "gsplat_batch_set_phase_timing: on must be 0 or 1");
    batch->batch->set_phase_timing(on != 0);
    return ok();
  });
}

int32_t gsplat_batch_get_phase_times(const GsplatBatch *batch, float *out_ms, uint32_t count) {
  return guarded("gsplat_batch_get_phase_times", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_get_phase_times");
    if (!out_ms && count > 0)
      return fail(Code::InvalidArgument, "gsplat_batch_get_phase_times: out_ms is null");
    const gsr::BatchResult &r = batch->batch->last();
    for (uint32_t k = 0; k < count && k < (uint32_t)gsr::kPhaseCount; ++k)
      out_ms[k] = r.phase_timed ? r.phase_ms[k] : 0.0f;
    return ok();
  });
}

int32_t gsplat_batch_get_view_stats(const GsplatBatch *batch, uint32_t view,
                                    GsplatBatchViewStats *out_stats) {
  return guarded("gsplat_batch_get_view_stats", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_get_view_stats");
    if (!out_stats)
      return fail(Code::InvalidArgument, "gsplat_batch_get_view_stats: out_stats is null");
    const gsr::ViewCounters &c = batch->batch->view_stats(view);
    *out_stats = GsplatBatchViewStats{c.visible, c.drawn, c.pairs, batch->batch->view_group(view)};
    return ok();
  });
}

int32_t gsplat_batch_readback_rgba8(GsplatBatch *batch, uint32_t view, uint8_t *out,
                                    uint64_t out_len) {
  return guarded("gsplat_batch_readback_rgba8", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_readback_rgba8");
    if (!out) return fail(Code::InvalidArgument, "gsplat_batch_readback_rgba8: out is null");
    batch->batch->readback_rgba8(view, out, out_len);
    return ok();
  });
}

int32_t gsplat_batch_image_device(const GsplatBatch *batch, uint32_t view, const void **out_ptr,
                                  uint64_t *out_bytes) {
  return guarded("gsplat_batch_image_device", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_image_device");
    if (!out_ptr || !out_bytes)
      return fail(Code::InvalidArgument, "gsplat_batch_image_device: null argument");
    *out_ptr = batch->batch->image_device(view, out_bytes);
    return ok();
  });
}

int32_t gsplat_batch_get_stream(const GsplatBatch *batch, void **out_stream) {
  return guarded("gsplat_batch_get_stream", [&]() -> int32_t {
    GSR_BATCH_CHECK("gsplat_batch_get_stream");
    if (!out_stream)
      return fail(Code::InvalidArgument, "gsplat_batch_get_stream: out_stream is null");
    *out_stream = (void *)batch->batch->stream();
    return ok();
  });
}

// ---- served rendering (gsplat_cuda.h) ----------------------------------------

static_assert(sizeof(GsplatServeConfig) == 48, "GsplatServeConfig layout");
static_assert(sizeof(GsplatServeStats) == 176, "GsplatServeStats layout");

int32_t gsplat_server_create(const GsplatServeConfig *config, GsplatServer **out_server) {
  return guarded("gsplat_server_create", [&]() -> int32_t {
    if (!out_server) return fail(Code::InvalidArgument, "gsplat_server_create: out_server is null");
    *out_server = nullptr;
    gsr::ServeConfig c;
    if (config) {
      c.result_pool_mib = config->result_pool_mib;
      c.max_queue_ms = config->max_queue_ms;
      if (config->scene_budget_bytes) c.scene_budget = config->scene_budget_bytes;
      if (config->work_budget_bytes) c.work_budget = config->work_budget_bytes;
      if (config->lanes) c.lanes = config->lanes;
      if (config->max_views_per_batch) c.max_views = config->max_views_per_batch;
      if (config->tile_size) c.tile = config->tile_size;
      c.raster.chunk = config->raster_chunk;
      c.raster.blocks_per_sm = config->raster_blocks_per_sm;
    }
    auto s = std::make_unique<GsplatServer>();
    s->server = std::make_unique<gsr::Server>(c);
    *out_server = s.release();
    return ok();
  });
}

void gsplat_server_destroy(GsplatServer *server) {
  try {
    delete server;
  } catch (...) {
  }
}

#define GSR_SERVER_CHECK(op) \
  if (!server || !server->server) return fail(Code::InvalidArgument, op ": server is null")

int32_t gsplat_server_add_scene_packed(GsplatServer *server, const GsplatSceneDesc *scene,
                                       uint32_t *out_scene) {
  return guarded("gsplat_server_add_scene_packed", [&]() -> int32_t {
    GSR_SERVER_CHECK("gsplat_server_add_scene_packed");
    if (!scene || !out_scene)
      return fail(Code::InvalidArgument, "gsplat_server_add_scene_packed: null argument");
    gsr::HostScene s = host_scene_from_desc(*scene);
    *out_scene = server->server->add_scene_packed(s);
    return ok();
  });
}

int32_t gsplat_server_add_scene_buffers(GsplatServer *server, const GsplatSceneDesc *scene,
                                        uint32_t *out_scene) {
  return guarded("gsplat_server_add_scene_buffers", [&]() -> int32_t {
    GSR_SERVER_CHECK("gsplat_server_add_scene_buffers");
    if (!scene || !out_scene)
      return fail(Code::InvalidArgument, "gsplat_server_add_scene_buffers: null argument");
    *out_scene = server->server->add_scene(host_scene_from_desc(*scene));
    return ok();
  });
}

int32_t gsplat_server_add_scene_path(GsplatServer *server, const char *path, uint32_t *out_scene) {
  return guarded("gsplat_server_add_scene_path", [&]() -> int32_t {
    GSR_SERVER_CHECK("gsplat_server_add_scene_path");
    if (!path || !out_scene)
      return fail(Code::InvalidArgument, "gsplat_server_add_scene_path: null argument");
    std::string p(path);
    if (!valid_utf8(p))
      return fail(Code::InvalidArgument, "gsplat_server_add_scene_path: path is not valid UTF-8");
    *out_scene = server->server->add_scene_path(p);
    return ok();
  });
}

int32_t gsplat_server_submit(GsplatServer *server, const GsplatBatchView *view,
                             uint64_t *out_request) {
  return guarded("gsplat_server_submit", [&]() -> int32_t {
    GSR_SERVER_CHECK("gsplat_server_submit");
    if (!view || !out_request)
      return fail(Code::InvalidArgument, "gsplat_server_submit: null argument");
    if (view->reserved != 0)
      return fail(Code::InvalidArgument, "gsplat_server_submit: reserved field must be 0");
    *out_request =
        server->server->submit(gsr::BatchView{view->scene, view->camera, view->width, view->height});
    return ok();
  });
}

static GsplatRequestInfo to_c_info(const gsr::RequestInfo &i) {
  return GsplatRequestInfo{(uint32_t)i.status, i.error_code, i.batch_views, i.counters.visible,
                           i.counters.drawn, i.counters.pairs, i.latency_ms, i.queue_ms};
}

int32_t gsplat_server_poll(GsplatServer *server, uint64_t request, GsplatRequestInfo *out_info) {
  return guarded("gsplat_server_poll", [&]() -> int32_t {
    GSR_SERVER_CHECK("gsplat_server_poll");
    if (!out_info) return fail(Code::InvalidArgument, "gsplat_server_poll: out_info is null");
    *out_info = to_c_info(server->server->poll(request));
    return ok();
  });
}

int32_t gsplat_server_wait(GsplatServer *server, uint64_t request, uint32_t timeout_ms,
                           GsplatRequestInfo *out_info) {
  return guarded("gsplat_server_wait", [&]() -> int32_t {
    GSR_SERVER_CHECK("gsplat_server_wait");
    if (!out_info) return fail(Code::InvalidArgument, "gsplat_server_wait: out_info is null");
    *out_info = to_c_info(server->server->wait(request, timeout_ms));
    return ok();
  });
}

int32_t gsplat_server_read_rgba8(GsplatServer *server, uint64_t request, uint8_t *out,
                                 uint64_t out_len) {
  return guarded("gsplat_server_read_rgba8", [&]() -> int32_t {
    GSR_SERVER_CHECK("gsplat_server_read_rgba8");
    if (!out) return fail(Code::InvalidArgument, "gsplat_server_read_rgba8: out is null");
    server->server->read_rgba8(request, out, out_len);
    return ok();
  });
}

int32_t gsplat_server_release(GsplatServer *server, uint64_t request) {
  return guarded("gsplat_server_release", [&]() -> int32_t {
    GSR_SERVER_CHECK("gsplat_server_release");
    server->server->release(request);
    return ok();
  });
}

int32_t gsplat_server_get_stats(GsplatServer *server, GsplatServeStats *out_stats) {
  return guarded("gsplat_server_get_stats", [&]() -> int32_t {
    GSR_SERVER_CHECK("gsplat_server_get_stats");
    if (!out_stats) return fail(Code::InvalidArgument, "gsplat_server_get_stats: out_stats is null");
    const gsr::ServeStats s = server->server->stats();
    *out_stats = GsplatServeStats{s.submitted, s.completed, s.failed, s.batches, s.reruns,
                                  s.peak_admitted_bytes, s.p50_ms, s.p99_ms, s.mean_ms, s.max_ms,
                                  s.views_per_s, s.mean_batch_views, s.device_ms, s.launch_ms,
                                  s.retire_ms, s.graph_captures, s.pinned_slabs, s.capture_ms,
                                  s.pinned_alloc_ms, s.workspace_regrowths, s.regrowth_ms, s.shed};
    return ok();
  });
}

int32_t gsplat_server_reset_stats(GsplatServer *server) {
  return guarded("gsplat_server_reset_stats", [&]() -> int32_t {
    GSR_SERVER_CHECK("gsplat_server_reset_stats");
    server->server->reset_stats();
    return ok();
  });
}

}  // extern "C"
