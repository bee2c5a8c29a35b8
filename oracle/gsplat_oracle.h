/*
 * CPU oracle for the SortedAlpha hot path of misotofu0525/gsplat-rs.
 *
 * TEST INFRASTRUCTURE ONLY. This library restates, in plain C++, the
 * reference's CPU code and WGSL shader math for the SortedAlpha path so that
 * the CUDA product can be checked against it. It is loaded only by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg; the product never
 * links, loads or calls it.
 *
 * Citations are `path:line` inside the reference project.
 *
 * Parity pins (see tests/test_oracle_golden.py):
 *   - sort KATs from crates/gsplat-sort/src/lib.rs:602-688 and the LCG edge
 *     lengths (radix.rs tests, lib.rs:614-647);
 *   - back-to-front order [1,2,0] from crates/gsplat-render-wgpu/src/lib.rs:4062-4089;
 *   - covariance/axes properties from lib.rs:4442-4528;
 *   - camera validation from crates/gsplat-core/src/lib.rs:312-340;
 *   - conformance channel means of minimal_ascii.ply at 64x64
 *     (crates/gsplat-render-wgpu/tests/conformance_sorted_alpha.rs:47-76).
 * Per-pixel parity with the reference's wgpu image is not pinned: the
 * reference's rasteriser and blender live in the GPU driver behind wgpu 28 and
 * cannot run on this machine (no Rust toolchain, no graphics stack).
 */
#ifndef GSPLAT_ORACLE_H
#define GSPLAT_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same field order and sizes as GsplatCamera in gsplat.h (40 bytes). */
typedef struct OrcCamera {
  float position[3];
  float rotation_xyzw[4];
  float vertical_fov_radians;
  float near_plane;
  float far_plane;
} OrcCamera;

/* SceneBuffers (crates/gsplat-core/src/lib.rs:201-213) as flat arrays. */
typedef struct OrcScene {
  uint64_t count;
  uint32_t sh_degree;
  uint32_t reserved;
  const float *positions;     /* 3*count */
  const float *opacity;       /* count, logit */
  const float *scale_xyz;     /* 3*count, log scale */
  const float *rotation_xyzw; /* 4*count */
  const float *color_dc;      /* 3*count */
  const float *sh_rest;       /* count*3*((d+1)^2-1), channel-major per splat, or NULL */
} OrcScene;

/* One splat after the WGSL vertex stage; same layout as GsplatProjectedSplat
 * in gsplat_cuda.h (64 bytes). */
typedef struct OrcProjected {
  float center_ndc[2];
  float axis_u[2];
  float axis_v[2];
  float color[4]; /* premultiplied rgb, alpha */
  float extent_scale;
  float depth;
  uint32_t flags; /* bit0 depth-visible, bit1 drawn (inside the frustum) */
  uint16_t tile_x0, tile_y0, tile_x1, tile_y1; /* tile rect, ends exclusive */
  uint32_t reserved;
} OrcProjected;

/* Raster record in pixel space (48 bytes), same as the CUDA record. */
typedef struct OrcRecord {
  float cx, cy, ax, ay;
  float bx, by, s, alpha;
  float cr, cg, cb, log2a;  /* colour (not premultiplied) and log2(alpha) */
} OrcRecord;

typedef struct OrcFrameParams {
  float cam[3];
  float view_rot[9];
  float f, aspect, tan_half_fovy, lim_x, lim_y, fx, fy, blur_x, blur_y;
  float near_plane, far_plane;
  float half_w, half_h, sx, sy;
  uint32_t width, height, tile, tiles_x, tiles_y, sh_degree;
} OrcFrameParams;

/* ---- gsplat-core ---- */
int32_t orc_camera_validate(const OrcCamera *camera);
/* Automatic framing of gsplat_context_set_auto_camera
 * (crates/gsplat-ffi-c/src/lib.rs:1593-1779); 1 for an empty scene. */
int32_t orc_auto_camera(const float *positions, uint64_t n, uint32_t width, uint32_t height,
                        OrcCamera *out);
/* camera_rotation_looking_at (crates/gsplat-ffi-c/src/lib.rs:1679-1733). */
void orc_camera_look_at(const float position[3], const float target[3], float q[4]);
int32_t orc_config_validate(uint32_t width, uint32_t height);
int32_t orc_scene_validate(const OrcScene *scene, uint64_t sh_rest_len);

/* ---- quaternions and per-frame parameters ---- */
void orc_quat_inverse(const float q[4], float out[4]);
void orc_quat_to_mat3(const float q[4], float out[9]);
void orc_view_rotation(const float q[4], float out[9]);
void orc_frame_params(const OrcCamera *camera, uint32_t width, uint32_t height,
                      uint32_t tile, uint32_t sh_degree, OrcFrameParams *out);

/* ---- load-time precompute ---- */
/* ---- packed resident format (packed_atlas.rs; decode of the CUDA design) ---- */
/* header[11]: bounds min (3), bounds span (3), log-scale min, log-scale
 * extent, SH scales (3). hot: 5 words per splat; sidecar: 48 bytes per splat
 * (or NULL). SH degree <= 3. */
void orc_pack_scene(const OrcScene *sc, float *header, uint32_t *hot, int8_t *sidecar);
/* The packed scene decoded to positions (3n), alpha (n), extent scale (n),
 * covariance (6n), DC (3n) and rest coefficients (n*3*((d+1)^2-1)). */
void orc_unpack_scene(uint64_t n, uint32_t sh_degree, const float *header, const uint32_t *hot,
                      const int8_t *sidecar, float *positions, float *alpha, float *extent,
                      float *cov6, float *color_dc, float *sh_rest);

/* Test helper: dividends whose refined constant division (product with
 * RN(1/d) and one fma correction) differs from the IEEE quotient. */
uint64_t orc_const_div_mismatches(float d, const float *x, uint64_t n);

void orc_precompute_alpha(const float *opacity, uint64_t n, float *alpha);
void orc_precompute_extent_scale(const float *alpha, uint64_t n, float *s);
void orc_precompute_cov(const float *scale_xyz, const float *rotation_xyzw, uint64_t n,
                        float *cov6);

/* ---- preprocess + CPU sort ---- */
uint64_t orc_preprocess_visible(const float *positions, uint64_t n, const OrcCamera *camera,
                                uint32_t *depth_keys, uint32_t *indices);
int32_t orc_sort_values_by_keys(const uint32_t *keys, uint32_t *values, uint64_t n);
int32_t orc_sort_pairs(uint32_t *keys, uint32_t *values, uint64_t n);
void orc_radix_count(const uint64_t *values, uint64_t n, uint32_t shift, int32_t use_simd,
                     uint64_t counts[256]);
void orc_pack_pairs(const uint32_t *keys, const uint32_t *values, uint64_t n, int32_t use_simd,
                    uint64_t *out);

/* ---- projection (WGSL vertex stage) and CPU instance builder ---- */
void orc_project_all(const OrcScene *scene, const float *alpha, const float *extent_scale,
                     const float *cov6, const OrcFrameParams *params, OrcProjected *out,
                     OrcRecord *records);
uint64_t orc_build_instances(const OrcScene *scene, const float *alpha, const float *cov6,
                             const OrcCamera *camera, uint32_t width, uint32_t height,
                             const uint32_t *indices, uint64_t m, float *out12,
                             uint32_t *out_index);

/* ---- tile keys (the CUDA design's key contract) ---- */
/* (tile, id) pairs in depth order; with `exact` each drawn splat covers, per
 * row of its tile rect, only the columns its ellipse reaches (exact row
 * spans, the CUDA design), else its whole tile rect. */
uint64_t orc_emit_tile_pairs(const OrcProjected *proj, const OrcRecord *rec, const uint32_t *order,
                             uint64_t v, uint32_t tiles_x, uint32_t tile, uint32_t exact,
                             uint32_t *tile_out, uint32_t *id_out, uint64_t capacity);
void orc_tile_lists(const uint32_t *tiles, const uint32_t *ids, uint64_t k, uint32_t num_tiles,
                    uint32_t *ranges, uint32_t *sorted_ids);
void orc_sort_u64_pairs_stable(uint64_t *keys, uint32_t *values, uint64_t n);

/* ---- compositing ---- */
float orc_exp_neg(float x);
/* Row ranges [y0, y1) of the compositors below (other rows zero). */
void orc_raster_unorm8_rows(const OrcRecord *records, const OrcProjected *proj,
                            const uint32_t *order, uint64_t v, uint32_t width, uint32_t height,
                            uint8_t *rgba, int32_t threads, uint32_t y0, uint32_t y1);
void orc_raster_f64_rows(const OrcRecord *records, const OrcProjected *proj,
                         const uint32_t *order, uint64_t v, uint32_t width, uint32_t height,
                         uint8_t *rgba, double *rgba_f64, int32_t threads, uint32_t y0,
                         uint32_t y1);
void orc_raster_tiles_fp32_rows(const OrcRecord *records, const uint32_t *ranges,
                                const uint32_t *sorted_ids, uint32_t width, uint32_t height,
                                uint32_t tile, uint32_t tiles_x, uint8_t *rgba, int32_t threads,
                                uint32_t y0, uint32_t y1);
void orc_raster_unorm8(const OrcRecord *records, const OrcProjected *proj,
                       const uint32_t *order, uint64_t v, uint32_t width, uint32_t height,
                       uint8_t *rgba, int32_t threads);
void orc_raster_f64(const OrcRecord *records, const OrcProjected *proj, const uint32_t *order,
                    uint64_t v, uint32_t width, uint32_t height, uint8_t *rgba,
                    double *rgba_f64, int32_t threads);
void orc_raster_tiles_fp32(const OrcRecord *records, const uint32_t *ranges,
                           const uint32_t *sorted_ids, uint32_t width, uint32_t height,
                           uint32_t tile, uint32_t tiles_x, uint8_t *rgba, int32_t threads);

/* ---- whole frame (the reference SortedAlpha path on the CPU) ---- */
typedef struct OrcFrameTiming {
  double preprocess_ms, sort_ms, project_ms, raster_ms, total_ms;
  uint64_t visible, drawn;
} OrcFrameTiming;
int32_t orc_render_reference_frame(const OrcScene *scene, const float *alpha,
                                   const float *extent_scale, const float *cov6,
                                   const OrcCamera *camera, uint32_t width, uint32_t height,
                                   uint32_t raster_rows, uint8_t *rgba, int32_t threads,
                                   OrcFrameTiming *timing);

#ifdef __cplusplus
}
#endif

#endif
