// Host-side value types, validation, per-frame uniforms and scene packing.
// Compiled with -ffp-contract=off so every f32 expression rounds per
// operation, as the reference's Rust f32 code does.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

#include "gsr_host.h"

namespace gsr {

static const float kPi = 3.14159265358979323846f;

// crates/gsplat-core/src/lib.rs:40-56 and 76-93
bool camera_valid(const GsplatCamera &c) {
  for (float v : c.position)
    if (!std::isfinite(v)) return false;
  for (float v : c.rotation_xyzw)
    if (!std::isfinite(v)) return false;
  float norm2 = 0.0f;
  for (float v : c.rotation_xyzw) norm2 = norm2 + v * v;
  if (norm2 <= 0.0f || !std::isfinite(norm2)) return false;
  if (std::fabs(norm2 - 1.0f) > 1.0e-3f) return false;
  if (!std::isfinite(c.vertical_fov_radians) || !std::isfinite(c.near_plane) ||
      !std::isfinite(c.far_plane))
    return false;
  if (c.vertical_fov_radians <= 0.0f || c.vertical_fov_radians >= kPi || c.near_plane <= 0.0f ||
      c.far_plane <= c.near_plane)
    return false;
  return true;
}

// crates/gsplat-core/src/lib.rs:224-276
Code scene_validate(const HostScene &s) {
  const uint64_t n = s.positions.size() / 3;
  if (s.positions.size() != 3 * n || s.opacity.size() != n || s.scale_xyz.size() != 3 * n ||
      s.rotation_xyzw.size() != 4 * n || s.color_dc.size() != 3 * n)
    return Code::ParseFailed;
  auto all_finite = [](const std::vector<float> &v) {
    for (float x : v)
      if (!std::isfinite(x)) return false;
    return true;
  };
  if (!all_finite(s.positions) || !all_finite(s.opacity) || !all_finite(s.scale_xyz) ||
      !all_finite(s.rotation_xyzw) || !all_finite(s.color_dc))
    return Code::ParseFailed;
  if (s.sh_degree > 4) return Code::Unsupported;
  const uint64_t stride = sh_rest_stride(s.sh_degree);
  if (!s.has_sh_rest) return stride == 0 ? Code::Ok : Code::ParseFailed;
  if (stride == 0) return Code::ParseFailed;
  if (s.sh_rest.size() != n * stride) return Code::ParseFailed;
  if (!all_finite(s.sh_rest)) return Code::ParseFailed;
  return Code::Ok;
}

// crates/gsplat-core/src/lib.rs:64-72 (CameraPose/CameraIntrinsics defaults):
// fov = 60.0_f32.to_radians() = 60 * (PI / 180) in f32.
GsplatCamera camera_default() {
  GsplatCamera c;
  std::memset(&c, 0, sizeof(c));
  c.rotation_xyzw[3] = 1.0f;
  const float rads_per_deg = kPi / 180.0f;
  c.vertical_fov_radians = 60.0f * rads_per_deg;
  c.near_plane = 0.01f;
  c.far_plane = 1000.0f;
  return c;
}

GsplatConfig config_default() { return GsplatConfig{1280, 720, 0}; }

// crates/gsplat-render-wgpu/src/lib.rs:1380-1388
void quat_normalize(const float q[4], float out[4]) {
  float norm2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  if (norm2 <= 0.0f) {
    out[0] = 0.0f; out[1] = 0.0f; out[2] = 0.0f; out[3] = 1.0f;
    return;
  }
  float inv = 1.0f / std::sqrt(norm2);
  out[0] = q[0] * inv; out[1] = q[1] * inv; out[2] = q[2] * inv; out[3] = q[3] * inv;
}

// lib.rs:1374-1378
void quat_inverse(const float q[4], float out[4]) {
  float n[4];
  quat_normalize(q, n);
  out[0] = -n[0]; out[1] = -n[1]; out[2] = -n[2]; out[3] = n[3];
}

// lib.rs:1390-1407 (normalizes its input first)
void quat_to_mat3(const float qin[4], float m[9]) {
  float q[4];
  quat_normalize(qin, q);
  float x = q[0], y = q[1], z = q[2], w = q[3];
  float xx = x * x, yy = y * y, zz = z * z;
  float xy = x * y, xz = x * z, yz = y * z;
  float wx = w * x, wy = w * y, wz = w * z;
  m[0] = 1.0f - 2.0f * (yy + zz); m[1] = 2.0f * (xy - wz);        m[2] = 2.0f * (xz + wy);
  m[3] = 2.0f * (xy + wz);        m[4] = 1.0f - 2.0f * (xx + zz); m[5] = 2.0f * (yz - wx);
  m[6] = 2.0f * (xz - wy);        m[7] = 2.0f * (yz + wx);        m[8] = 1.0f - 2.0f * (xx + yy);
}

static bool vec3_normalize(const float v[3], float out[3]) {
  // crates/gsplat-ffi-c/src/lib.rs:1755-1762
  float len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if (!std::isfinite(len) || len <= 1.0e-6f) return false;
  float inv = 1.0f / len;
  out[0] = v[0] * inv; out[1] = v[1] * inv; out[2] = v[2] * inv;
  return true;
}

static void vec3_cross(const float a[3], const float b[3], float out[3]) {
  out[0] = a[1] * b[2] - a[2] * b[1];
  out[1] = a[2] * b[0] - a[0] * b[2];
  out[2] = a[0] * b[1] - a[1] * b[0];
}

// crates/gsplat-ffi-c/src/lib.rs:1714-1733 (camera_rotation_looking_at) and
// 1690-1712 (quat_from_camera_basis).
void camera_rotation_looking_at(const float position[3], const float target[3], float q[4]) {
  float d[3] = {target[0] - position[0], target[1] - position[1], target[2] - position[2]};
  float fwd[3];
  if (!vec3_normalize(d, fwd)) { fwd[0] = 0.0f; fwd[1] = 0.0f; fwd[2] = 1.0f; }
  float up_w[3] = {0.0f, 1.0f, 0.0f};
  if (std::fabs(fwd[1]) > 0.98f) { up_w[1] = 0.0f; up_w[2] = 1.0f; }
  float rc[3], right[3], up[3];
  vec3_cross(up_w, fwd, rc);
  if (!vec3_normalize(rc, right)) { right[0] = 1.0f; right[1] = 0.0f; right[2] = 0.0f; }
  vec3_cross(fwd, right, up);
  float m00 = right[0], m01 = up[0], m02 = fwd[0];
  float m10 = right[1], m11 = up[1], m12 = fwd[1];
  float m20 = right[2], m21 = up[2], m22 = fwd[2];
  float trace = m00 + m11 + m22;
  float x, y, z, w;
  if (trace > 0.0f) {
    float s = std::sqrt(trace + 1.0f) * 2.0f;
    x = (m21 - m12) / s; y = (m02 - m20) / s; z = (m10 - m01) / s; w = 0.25f * s;
  } else if (m00 > m11 && m00 > m22) {
    float s = std::sqrt(1.0f + m00 - m11 - m22) * 2.0f;
    x = 0.25f * s; y = (m01 + m10) / s; z = (m02 + m20) / s; w = (m21 - m12) / s;
  } else if (m11 > m22) {
    float s = std::sqrt(1.0f + m11 - m00 - m22) * 2.0f;
    x = (m01 + m10) / s; y = 0.25f * s; z = (m12 + m21) / s; w = (m02 - m20) / s;
  } else {
    float s = std::sqrt(1.0f + m22 - m00 - m11) * 2.0f;
    x = (m02 + m20) / s; y = (m12 + m21) / s; z = 0.25f * s; w = (m10 - m01) / s;
  }
  float norm = std::fmax(std::sqrt(x * x + y * y + z * z + w * w), 1.0e-6f);
  q[0] = x / norm; q[1] = y / norm; q[2] = z / norm; q[3] = w / norm;
}

// crates/gsplat-ffi-c/src/lib.rs:1596-1630 (auto_surface_camera_control),
// 1645-1675 (surface_camera_from_control) with yaw = pitch = 0.
GsplatCamera auto_camera(const float *p, uint64_t n, uint32_t width, uint32_t height) {
  if (n == 0) throw Error(Code::InvalidArgument, "scene has no splats");
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      mn[k] = std::fmin(mn[k], p[3 * i + k]);
      mx[k] = std::fmax(mx[k], p[3 * i + k]);
    }
  float center[3], half[3];
  for (int k = 0; k < 3; ++k) {
    center[k] = (mn[k] + mx[k]) * 0.5f;
    half[k] = std::fmax((mx[k] - mn[k]) * 0.5f, 1e-3f);
  }
  GsplatCamera cam = camera_default();
  float aspect = (float)width / (float)height;
  // Read through a volatile: tan/atan of the default fov must come from the
  // C library at run time, as the reference's f32 methods do, never from
  // the compiler folding a constant (correctly rounded, which can differ in
  // the last bit).
  volatile float fov_v = cam.vertical_fov_radians;
  float vfov = std::fmax((float)fov_v, 1e-3f);
  float hfov = 2.0f * std::atan(std::tan(vfov * 0.5f) * aspect);
  float dist_y = half[1] / std::tan(vfov * 0.5f);
  float dist_x = half[0] / std::tan(hfov * 0.5f);
  float dist = (std::fmax(dist_y, dist_x) + half[2]) * 1.2f;
  float radius = std::fmax(std::fmax(half[0], half[1]), half[2]);
  // yaw = pitch = 0: offset = (0, 0, -distance).
  const float pitch = 0.0f, yaw = 0.0f;
  float cos_pitch = std::cos(pitch);
  float offset[3] = {std::sin(yaw) * cos_pitch * dist, std::sin(pitch) * dist,
                     -std::cos(yaw) * cos_pitch * dist};
  float pos[3] = {center[0] + offset[0], center[1] + offset[1], center[2] + offset[2]};
  cam.position[0] = pos[0]; cam.position[1] = pos[1]; cam.position[2] = pos[2];
  camera_rotation_looking_at(pos, center, cam.rotation_xyzw);
  float r = std::fmax(radius, 1.0e-3f);
  cam.near_plane = std::fmax(dist - r * 2.0f, 0.01f);
  cam.far_plane = std::fmax(dist + r * 8.0f, 100.0f);
  float asp = std::fmax((float)width / (float)std::max<uint32_t>(height, 1u), 1.0e-3f);
  if (asp < 0.6f) cam.vertical_fov_radians = 65.0f * (kPi / 180.0f);
  return cam;
}

// GpuSurfaceRenderParams (crates/gsplat-render-wgpu/src/lib.rs:922-953) and
// the per-vertex constants of project_splat (splat_surface_direct.wgsl:143-187).
FrameParams make_frame_params(const GsplatCamera &cam, uint32_t width, uint32_t height,
                              uint32_t tile, uint32_t sh_degree, uint32_t splat_count) {
  FrameParams p;
  std::memset(&p, 0, sizeof(p));
  float inv_q[4], view[9];
  quat_inverse(cam.rotation_xyzw, inv_q);
  quat_to_mat3(inv_q, view);
  for (int k = 0; k < 3; ++k) {
    p.cam[k] = cam.position[k];
    p.r0[k] = view[k];
    p.r1[k] = view[3 + k];
    p.r2[k] = view[6 + k];
  }
  p.aspect = (float)width / (float)std::max<uint32_t>(height, 1u);
  if (!(p.aspect >= 1e-6f)) p.aspect = 1e-6f;
  float half_fov = cam.vertical_fov_radians * 0.5f;
  p.f = 1.0f / std::tan(half_fov);
  float tan_half_fovy = std::tan(half_fov);
  float tan_half_fovx = tan_half_fovy * p.aspect;
  p.lim_x = 1.3f * tan_half_fovx;
  p.lim_y = 1.3f * tan_half_fovy;
  p.fx = p.f / p.aspect;
  p.fy = p.f;
  float bx = 0.3f * (2.0f / std::fmax((float)width, 1.0f));
  float by = 0.3f * (2.0f / std::fmax((float)height, 1.0f));
  p.blur_x = bx * bx;
  p.blur_y = by * by;
  p.near_plane = cam.near_plane;
  p.far_plane = cam.far_plane;
  p.half_w = 0.5f * (float)width;
  p.half_h = 0.5f * (float)height;
  p.sx = 2.0f / (float)width;
  p.sy = -2.0f / (float)height;
  p.width = width;
  p.height = height;
  p.tile = tile;
  p.tiles_x = (width + tile - 1) / tile;
  p.tiles_y = (height + tile - 1) / tile;
  p.num_tiles = p.tiles_x * p.tiles_y;
  p.sh_degree = std::min<uint32_t>(sh_degree, 4u);
  p.color_planes = color_planes(p.sh_degree);
  p.splat_count = splat_count;
  return p;
}

static void mat3_mul(const float a[9], const float b[9], float out[9]) {
  // lib.rs:1409-1417
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      out[3 * r + c] = a[3 * r + 0] * b[0 + c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c];
}

void splat_scalars(float opacity_logit, const float log_scale[3], float out[5]) {
  // alpha: lib.rs:1251-1261
  float a = 1.0f / (1.0f + std::exp(-opacity_logit));
  a = std::fmin(std::fmax(a, 0.0f), 1.0f);
  // alpha_extent_scale: splat_surface_direct.wgsl:74-77
  float s2 = std::log(std::fmax(a, 1e-12f) * 256.0f) / 4.5f;
  out[0] = a;
  out[1] = std::sqrt(std::fmin(std::fmax(s2, 0.0f), 1.0f));
  // axis scales of the world covariance: lib.rs:1654-1674
  for (int k = 0; k < 3; ++k) out[2 + k] = std::fmax(std::exp(log_scale[k]), 1e-6f);
}

static void pack_range(const HostScene &s, ScenePacked &o, uint64_t begin, uint64_t end) {
  const uint64_t n = s.size();
  const uint32_t degree = s.sh_degree;
  const uint32_t per_channel = (degree + 1) * (degree + 1) - 1;
  const uint32_t planes = o.planes;
  for (uint64_t i = begin; i < end; ++i) {
    float sc[5];
    splat_scalars(s.opacity[i], &s.scale_xyz[3 * i], sc);
    const float a = sc[0], ext = sc[1], sx = sc[2], sy = sc[3], sz = sc[4];
    // world covariance: lib.rs:1654-1674
    float obj[9] = {sx * sx, 0.0f, 0.0f, 0.0f, sy * sy, 0.0f, 0.0f, 0.0f, sz * sz};
    float qn[4], rot[9], rt[9], tmp[9], w[9];
    quat_normalize(&s.rotation_xyzw[4 * i], qn);
    quat_to_mat3(qn, rot);
    mat3_mul(rot, obj, tmp);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) rt[3 * r + c] = rot[3 * c + r];
    mat3_mul(tmp, rt, w);
    float *pa = &o.pos_alpha[4 * i];
    pa[0] = s.positions[3 * i]; pa[1] = s.positions[3 * i + 1]; pa[2] = s.positions[3 * i + 2];
    pa[3] = a;
    float *ca = &o.cov_a[4 * i];
    ca[0] = w[0]; ca[1] = w[1]; ca[2] = w[2]; ca[3] = w[4];
    float *cb = &o.cov_b[4 * i];
    cb[0] = w[5]; cb[1] = w[8]; cb[2] = ext; cb[3] = 0.0f;
    // colour planes: float f[3*c + ch] for coefficient c (0 = DC), channel ch;
    // plane p holds f[4p .. 4p+3] of every splat.
    float f[4 * 19];
    std::memset(f, 0, sizeof(f));
    for (int ch = 0; ch < 3; ++ch) f[ch] = s.color_dc[3 * i + ch];
    if (degree > 0 && s.has_sh_rest) {
      const float *rest = &s.sh_rest[i * per_channel * 3];
      for (uint32_t k = 0; k < per_channel; ++k)
        for (int ch = 0; ch < 3; ++ch) f[3 * (k + 1) + ch] = rest[ch * per_channel + k];
    }
    for (uint32_t pl = 0; pl < planes; ++pl)
      std::memcpy(&o.color[4 * ((uint64_t)pl * n + i)], &f[4 * pl], 16);
  }
}

void pack_scene(const HostScene &s, ScenePacked &o) {
  const uint64_t n = s.size();
  o.planes = color_planes(s.sh_degree);
  o.pos_alpha.assign(4 * n, 0.0f);
  o.cov_a.assign(4 * n, 0.0f);
  o.cov_b.assign(4 * n, 0.0f);
  o.color.assign(4 * (uint64_t)o.planes * n, 0.0f);
  unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  if (n < 65536) hw = 1;
  std::vector<std::thread> pool;
  uint64_t chunk = (n + hw - 1) / hw;
  for (unsigned t = 0; t < hw; ++t) {
    uint64_t b = t * chunk, e = std::min<uint64_t>(n, b + chunk);
    if (b >= e) break;
    pool.emplace_back(pack_range, std::cref(s), std::ref(o), b, e);
  }
  for (auto &th : pool) th.join();
}

}  // namespace gsr
