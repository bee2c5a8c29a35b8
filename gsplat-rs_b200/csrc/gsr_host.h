// Host-side types of the CUDA renderer: the gsplat-core value types
// (crates/gsplat-core/src/lib.rs), their validation, the per-frame uniforms
// and the camera helpers of the C ABI layer.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/gsplat.h"

namespace gsr {

// crates/gsplat-core/src/lib.rs:154-170
enum class Code : int32_t {
  Ok = 0,
  InvalidArgument = 1,
  NotFound = 2,
  ParseFailed = 3,
  Unsupported = 4,
  SceneNotLoaded = 5,
  Internal = 100,
};

// Every failure inside the library is thrown as an Error and turned into a
// GsplatErrorCode plus a last-error message at the C boundary.
struct Error : std::runtime_error {
  Code code;
  Error(Code c, const std::string &msg) : std::runtime_error(msg), code(c) {}
};

// SceneBuffers (crates/gsplat-core/src/lib.rs:201-213), owned host copy.
struct HostScene {
  std::vector<float> positions;      // 3n
  std::vector<float> opacity;        // n
  std::vector<float> scale_xyz;      // 3n
  std::vector<float> rotation_xyzw;  // 4n
  std::vector<float> color_dc;       // 3n
  uint32_t sh_degree = 0;
  bool has_sh_rest = false;
  std::vector<float> sh_rest;        // n * 3 * ((d+1)^2 - 1), channel-major
  uint64_t size() const { return opacity.size(); }
};

// Validation with the reference's error codes.
bool camera_valid(const GsplatCamera &c);                 // lib.rs:40-107
Code scene_validate(const HostScene &s);                  // lib.rs:224-276
inline uint32_t sh_rest_stride(uint32_t degree) { return 3u * ((degree + 1) * (degree + 1) - 1); }

GsplatCamera camera_default();  // lib.rs:64-72
GsplatConfig config_default();  // lib.rs:139-147

// Load-time scalars of one splat with the reference's f32 expressions and
// the C library's exp/log: alpha = clamp(sigmoid(opacity)), the extent scale
// s (splat_surface_direct.wgsl:74-77) and max(exp(log_scale), 1e-6) per axis
// (lib.rs:1251-1261, 1654-1674). out = {alpha, s, sx, sy, sz}.
void splat_scalars(float opacity_logit, const float log_scale[3], float out[5]);

// Quaternion helpers (crates/gsplat-render-wgpu/src/lib.rs:1374-1407).
void quat_normalize(const float q[4], float out[4]);
void quat_inverse(const float q[4], float out[4]);
void quat_to_mat3(const float q[4], float m[9]);

// camera_rotation_looking_at (crates/gsplat-ffi-c/src/lib.rs:1714-1733).
void camera_rotation_looking_at(const float position[3], const float target[3], float out_q[4]);
// auto_camera (crates/gsplat-ffi-c/src/lib.rs:1596-1675); throws
// SceneNotLoaded / InvalidArgument like the reference.
GsplatCamera auto_camera(const float *positions, uint64_t n, uint32_t width, uint32_t height);

// Per-frame uniforms, shared by every kernel of the frame. Field meaning
// follows GpuSurfaceRenderParams (lib.rs:998-1016) and the constants that
// project_splat derives from it (splat_surface_direct.wgsl:131-217), plus the
// pixel-space and tile terms of this renderer.
struct FrameParams {
  float cam[3];
  float r0[3], r1[3], r2[3];  // view rotation rows
  float f, aspect, lim_x, lim_y, fx, fy, blur_x, blur_y;
  float near_plane, far_plane;
  float half_w, half_h, sx, sy;
  uint32_t width, height, tile, tiles_x, tiles_y, num_tiles;
  uint32_t sh_degree, color_planes, splat_count, pad;
};
FrameParams make_frame_params(const GsplatCamera &cam, uint32_t width, uint32_t height,
                              uint32_t tile, uint32_t sh_degree, uint32_t splat_count);

// Number of float4 colour planes for an SH degree: DC + rest coefficients,
// three channels each, packed four floats per plane.
inline uint32_t color_planes(uint32_t degree) {
  uint32_t floats = 3u * (degree + 1) * (degree + 1);
  return (floats + 3) / 4;
}

// Load-time precompute (lib.rs:1251-1261, 1654-1674, wgsl:74-77), bit for bit
// the reference's f32 arithmetic; spread over host threads.
struct ScenePacked {
  std::vector<float> pos_alpha;  // 4n: x y z alpha
  std::vector<float> cov_a;      // 4n: xx xy xz yy
  std::vector<float> cov_b;      // 4n: yz zz extent_scale 0
  std::vector<float> color;      // 4 * planes * n: plane-major
  uint32_t planes = 0;
};
void pack_scene(const HostScene &s, ScenePacked &out);

// PLY loader (crates/gsplat-io-ply/src/lib.rs).
HostScene load_ply(const std::string &path);

}  // namespace gsr
