// CPU oracle, part 1: core types, quaternions, load-time precompute,
// depth preprocess and the reference CPU radix sort.
//
// TEST INFRASTRUCTURE ONLY (see gsplat_oracle.h). Built with
// -ffp-contract=off so every f32 expression rounds after each operation,
// as Rust's f32 arithmetic does.

#include <cmath>
#include <cstring>
#include <vector>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include "gsplat_oracle.h"
#include "oracle_internal.h"

namespace orc {

// crates/gsplat-core/src/lib.rs:40-56 (CameraPose::validate)
static bool pose_valid(const OrcCamera &c) {
  for (float v : c.position)
    if (!std::isfinite(v)) return false;
  for (float v : c.rotation_xyzw)
    if (!std::isfinite(v)) return false;
  // iter().map(v*v).sum(): left-to-right fold.
  float norm2 = 0.0f;
  for (float v : c.rotation_xyzw) norm2 = norm2 + v * v;
  if (norm2 <= 0.0f || !std::isfinite(norm2)) return false;
  if (std::fabs(norm2 - 1.0f) > 1.0e-3f) return false;
  return true;
}

// crates/gsplat-core/src/lib.rs:76-93 (CameraIntrinsics::validate)
static bool intrinsics_valid(const OrcCamera &c) {
  if (!std::isfinite(c.vertical_fov_radians) || !std::isfinite(c.near_plane) ||
      !std::isfinite(c.far_plane))
    return false;
  const float pi = 3.14159265358979323846f;
  if (c.vertical_fov_radians <= 0.0f || c.vertical_fov_radians >= pi || c.near_plane <= 0.0f ||
      c.far_plane <= c.near_plane)
    return false;
  return true;
}

// crates/gsplat-render-wgpu/src/lib.rs:1380-1388 (quat_normalize)
void quat_normalize(const float q[4], float out[4]) {
  float norm2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  if (norm2 <= 0.0f) {
    out[0] = 0.0f; out[1] = 0.0f; out[2] = 0.0f; out[3] = 1.0f;
    return;
  }
  float inv = 1.0f / std::sqrt(norm2);
  out[0] = q[0] * inv; out[1] = q[1] * inv; out[2] = q[2] * inv; out[3] = q[3] * inv;
}

// lib.rs:1374-1378 (quat_inverse)
void quat_inverse(const float q[4], float out[4]) {
  float n[4];
  quat_normalize(q, n);
  out[0] = -n[0]; out[1] = -n[1]; out[2] = -n[2]; out[3] = n[3];
}

// lib.rs:1390-1407 (quat_to_mat3), row-major out[3*r+c]
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

// lib.rs:1409-1425 (mat3_mul, mat3_transpose)
static void mat3_mul(const float a[9], const float b[9], float out[9]) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      out[3 * r + c] = a[3 * r + 0] * b[0 + c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c];
}
static void mat3_transpose(const float m[9], float out[9]) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) out[3 * r + c] = m[3 * c + r];
}

// Per-frame uniforms: make_surface_render_params (lib.rs:922-953) plus the
// per-vertex constants project_splat derives from them
// (splat_surface_direct.wgsl:143-187) and the pixel-space terms of the tile
// design.
void frame_params(const OrcCamera &cam, uint32_t width, uint32_t height, uint32_t tile,
                  uint32_t sh_degree, OrcFrameParams &p) {
  std::memset(&p, 0, sizeof(p));
  float inv_q[4];
  quat_inverse(cam.rotation_xyzw, inv_q);
  quat_to_mat3(inv_q, p.view_rot);
  p.cam[0] = cam.position[0]; p.cam[1] = cam.position[1]; p.cam[2] = cam.position[2];
  float hmax = (float)(height > 1 ? height : 1);
  p.aspect = (float)width / hmax;
  if (!(p.aspect >= 1e-6f)) p.aspect = 1e-6f;
  float half_fov = cam.vertical_fov_radians * 0.5f;
  p.f = 1.0f / std::tan(half_fov);
  p.tan_half_fovy = std::tan(half_fov);
  float tan_half_fovx = p.tan_half_fovy * p.aspect;
  p.lim_x = 1.3f * tan_half_fovx;
  p.lim_y = 1.3f * p.tan_half_fovy;
  p.fx = p.f / p.aspect;
  p.fy = p.f;
  // blur_pixels = 0.3, px_ndc = 2 / max(extent, 1); the CPU path squares with powi(2).
  float px_ndc_x = 2.0f / std::fmax((float)width, 1.0f);
  float px_ndc_y = 2.0f / std::fmax((float)height, 1.0f);
  float bx = 0.3f * px_ndc_x, by = 0.3f * px_ndc_y;
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
  p.sh_degree = sh_degree;
}

// ---------------------------------------------------------------------------
// CPU radix sort: crates/gsplat-sort/src/radix.rs and lib.rs:36-210.

static inline uint64_t pack_sort_pair(uint32_t key, uint32_t value) {
  // lib.rs:104-107
  return ((uint64_t)key << 32) | (uint64_t)(uint32_t)(~value);
}

static bool have_avx2() {
#if defined(__x86_64__)
  return __builtin_cpu_supports("avx2");
#else
  return false;
#endif
}

#if defined(__x86_64__)
// lib.rs:180-210 (pack_pairs_avx2): widen key and !value to u64 lanes.
__attribute__((target("avx2"))) static void pack_pairs_avx2(const uint32_t *keys,
                                                            const uint32_t *values, uint64_t n,
                                                            uint64_t *out) {
  uint64_t i = 0;
  const __m128i ones = _mm_set1_epi32(-1);
  for (; i + 4 <= n; i += 4) {
    __m128i k = _mm_loadu_si128((const __m128i *)(keys + i));
    __m128i v = _mm_xor_si128(_mm_loadu_si128((const __m128i *)(values + i)), ones);
    __m256i k64 = _mm256_slli_epi64(_mm256_cvtepu32_epi64(k), 32);
    __m256i v64 = _mm256_cvtepu32_epi64(v);
    _mm256_storeu_si256((__m256i *)(out + i), _mm256_or_si256(k64, v64));
  }
  for (; i < n; ++i) out[i] = pack_sort_pair(keys[i], values[i]);
}

// radix.rs:176-219 (count_histograms_avx2): four lane histograms, merged.
__attribute__((target("avx2"))) static void count_avx2(const uint64_t *in, uint64_t n,
                                                       uint32_t shift, uint64_t *counts) {
  static thread_local uint32_t hist[4][256];
  std::memset(hist, 0, sizeof(hist));
  const __m256i mask = _mm256_set1_epi64x(0xff);
  const __m128i sh = _mm_cvtsi32_si128((int)shift);
  uint64_t i = 0;
  alignas(32) uint64_t d[4];
  for (; i + 4 <= n; i += 4) {
    __m256i p = _mm256_loadu_si256((const __m256i *)(in + i));
    __m256i digits = _mm256_and_si256(_mm256_srl_epi64(p, sh), mask);
    _mm256_store_si256((__m256i *)d, digits);
    hist[0][d[0]]++; hist[1][d[1]]++; hist[2][d[2]]++; hist[3][d[3]]++;
  }
  for (; i < n; ++i) hist[0][(in[i] >> shift) & 0xff]++;
  for (int b = 0; b < 256; ++b)
    counts[b] = (uint64_t)hist[0][b] + hist[1][b] + hist[2][b] + hist[3][b];
}
#endif

// radix.rs:92-98 (count_histograms_scalar)
static void count_scalar(const uint64_t *in, uint64_t n, uint32_t shift, uint64_t *counts) {
  for (int b = 0; b < 256; ++b) counts[b] = 0;
  for (uint64_t i = 0; i < n; ++i) counts[(in[i] >> shift) & 0xff]++;
}

static void count_digits(const uint64_t *in, uint64_t n, uint32_t shift, bool simd,
                         uint64_t *counts) {
#if defined(__x86_64__)
  if (simd && have_avx2()) {
    count_avx2(in, n, shift, counts);
    return;
  }
#endif
  (void)simd;
  count_scalar(in, n, shift, counts);
}

// radix.rs:110-117: offsets handed out from the largest digit down.
static void descending_prefix_offsets(uint64_t *counts) {
  uint64_t offset = 0;
  for (int b = 255; b >= 0; --b) {
    uint64_t len = counts[b];
    counts[b] = offset;
    offset += len;
  }
}

// radix.rs:119-126: stable scatter.
static void scatter_digits(const uint64_t *in, uint64_t *out, uint64_t n, uint32_t shift,
                           uint64_t *offsets) {
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t d = (in[i] >> shift) & 0xff;
    out[offsets[d]++] = in[i];
  }
}

// radix.rs:27-58: descending LSD passes over bit range [lo, hi).
void radix_sort_desc_u64_passes(uint64_t *values, uint64_t *scratch, uint64_t n, uint32_t lo,
                                uint32_t hi) {
  uint64_t counts[256];
  bool to_scratch = true;
  for (uint32_t shift = lo; shift < hi; shift += 8) {
    const uint64_t *src = to_scratch ? values : scratch;
    uint64_t *dst = to_scratch ? scratch : values;
    count_digits(src, n, shift, true, counts);
    descending_prefix_offsets(counts);
    scatter_digits(src, dst, n, shift, counts);
    to_scratch = !to_scratch;
  }
  if (!to_scratch) std::memcpy(values, scratch, n * sizeof(uint64_t));
}

}  // namespace orc

using namespace orc;

extern "C" {

int32_t orc_camera_validate(const OrcCamera *camera) {
  if (!camera) return 1;
  return (pose_valid(*camera) && intrinsics_valid(*camera)) ? 0 : 1;
}

// crates/gsplat-core/src/lib.rs:141-149
int32_t orc_config_validate(uint32_t width, uint32_t height) {
  return (width == 0 || height == 0) ? 1 : 0;
}

// crates/gsplat-core/src/lib.rs:224-276 (SceneBuffers::validate):
// 0 ok, 3 ParseFailed, 4 Unsupported.
int32_t orc_scene_validate(const OrcScene *s, uint64_t sh_rest_len) {
  uint64_t n = s->count;
  for (uint64_t i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(s->positions[3 * i + k]) || !std::isfinite(s->scale_xyz[3 * i + k]) ||
          !std::isfinite(s->color_dc[3 * i + k]))
        return 3;
    for (int k = 0; k < 4; ++k)
      if (!std::isfinite(s->rotation_xyzw[4 * i + k])) return 3;
    if (!std::isfinite(s->opacity[i])) return 3;
  }
  if (s->sh_degree > 4) return 4;
  uint64_t coeff_total = (uint64_t)(s->sh_degree + 1) * (s->sh_degree + 1);
  uint64_t stride = (coeff_total - 1) * 3;
  if (s->sh_rest == nullptr) return stride == 0 ? 0 : 3;
  if (stride == 0) return 3;
  if (sh_rest_len != n * stride) return 3;
  for (uint64_t i = 0; i < sh_rest_len; ++i)
    if (!std::isfinite(s->sh_rest[i])) return 3;
  return 0;
}

void orc_quat_inverse(const float q[4], float out[4]) { quat_inverse(q, out); }
void orc_quat_to_mat3(const float q[4], float out[9]) { quat_to_mat3(q, out); }

// lib.rs:1283-1285: view rotation = quat_to_mat3(quat_inverse(q)).
void orc_view_rotation(const float q[4], float out[9]) {
  float inv[4];
  quat_inverse(q, inv);
  quat_to_mat3(inv, out);
}

void orc_frame_params(const OrcCamera *camera, uint32_t width, uint32_t height, uint32_t tile,
                      uint32_t sh_degree, OrcFrameParams *out) {
  frame_params(*camera, width, height, tile, sh_degree, *out);
}

// lib.rs:1251-1261 (precompute_alpha_values, sigmoid)
void orc_precompute_alpha(const float *opacity, uint64_t n, float *alpha) {
  for (uint64_t i = 0; i < n; ++i) {
    float a = 1.0f / (1.0f + std::exp(-opacity[i]));
    alpha[i] = std::fmin(std::fmax(a, 0.0f), 1.0f);
  }
}

// splat_surface_direct.wgsl:74-77 (alpha_extent_scale)
void orc_precompute_extent_scale(const float *alpha, uint64_t n, float *s) {
  for (uint64_t i = 0; i < n; ++i) {
    float s2 = std::log(std::fmax(alpha[i], 1e-12f) * 256.0f) / 4.5f;
    s[i] = std::sqrt(std::fmin(std::fmax(s2, 0.0f), 1.0f));
  }
}

// lib.rs:1654-1674 (precompute_world_covariances) + CameraCovarianceTerms::from_matrix
// (lib.rs:1518-1529): cov6 = xx, xy, xz, yy, yz, zz.
void orc_precompute_cov(const float *scale_xyz, const float *rotation_xyzw, uint64_t n,
                        float *cov6) {
  for (uint64_t i = 0; i < n; ++i) {
    float sx = std::fmax(std::exp(scale_xyz[3 * i + 0]), 1e-6f);
    float sy = std::fmax(std::exp(scale_xyz[3 * i + 1]), 1e-6f);
    float sz = std::fmax(std::exp(scale_xyz[3 * i + 2]), 1e-6f);
    float obj[9] = {sx * sx, 0.0f, 0.0f, 0.0f, sy * sy, 0.0f, 0.0f, 0.0f, sz * sz};
    float qn[4], rot[9], rt[9], tmp[9], w[9];
    quat_normalize(&rotation_xyzw[4 * i], qn);
    quat_to_mat3(qn, rot);
    mat3_mul(rot, obj, tmp);
    mat3_transpose(rot, rt);
    mat3_mul(tmp, rt, w);
    float *c = &cov6[6 * i];
    c[0] = w[0]; c[1] = w[1]; c[2] = w[2]; c[3] = w[4]; c[4] = w[5]; c[5] = w[8];
  }
}

// lib.rs:1263-1296 (preprocess_visible_into), 1346-1354
// (world_to_camera_depth_with_view_row), 969-976 (is_visible, depth_to_key).
// Returns the visible count, or UINT64_MAX for an invalid camera.
uint64_t orc_preprocess_visible(const float *positions, uint64_t n, const OrcCamera *camera,
                                uint32_t *depth_keys, uint32_t *indices) {
  if (orc_camera_validate(camera) != 0) return UINT64_MAX;
  float view[9];
  orc_view_rotation(camera->rotation_xyzw, view);
  const float r0 = view[6], r1 = view[7], r2 = view[8];
  const float cx = camera->position[0], cy = camera->position[1], cz = camera->position[2];
  uint64_t v = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const float *p = &positions[3 * i];
    float depth = r0 * (p[0] - cx) + r1 * (p[1] - cy) + r2 * (p[2] - cz);
    if (depth >= camera->near_plane && depth <= camera->far_plane) {
      indices[v] = (uint32_t)i;
      float d = std::fmax(depth, 0.0f);
      uint32_t bits;
      std::memcpy(&bits, &d, 4);
      depth_keys[v] = bits;
      ++v;
    }
  }
  return v;
}

// crates/gsplat-sort/src/lib.rs:36-61 (sort_values_by_keys): pack key<<32|!value,
// sort descending on the high 32 bits, unpack !low32.
int32_t orc_sort_values_by_keys(const uint32_t *keys, uint32_t *values, uint64_t n) {
  if (n <= 1) return 0;
  std::vector<uint64_t> packed(n), scratch(n);
  orc_pack_pairs(keys, values, n, 1, packed.data());
  radix_sort_desc_u64_passes(packed.data(), scratch.data(), n, 32, 64);
  for (uint64_t i = 0; i < n; ++i) values[i] = ~(uint32_t)packed[i];
  return 0;
}

// crates/gsplat-sort/src/lib.rs:81-101 (sort_pairs): all 64 bits.
int32_t orc_sort_pairs(uint32_t *keys, uint32_t *values, uint64_t n) {
  if (n <= 1) return 0;
  std::vector<uint64_t> packed(n), scratch(n);
  orc_pack_pairs(keys, values, n, 1, packed.data());
  radix_sort_desc_u64_passes(packed.data(), scratch.data(), n, 0, 64);
  for (uint64_t i = 0; i < n; ++i) {
    keys[i] = (uint32_t)(packed[i] >> 32);
    values[i] = ~(uint32_t)packed[i];
  }
  return 0;
}

void orc_radix_count(const uint64_t *values, uint64_t n, uint32_t shift, int32_t use_simd,
                     uint64_t counts[256]) {
  count_digits(values, n, shift, use_simd != 0, counts);
}

void orc_pack_pairs(const uint32_t *keys, const uint32_t *values, uint64_t n, int32_t use_simd,
                    uint64_t *out) {
#if defined(__x86_64__)
  if (use_simd && have_avx2()) {
    pack_pairs_avx2(keys, values, n, out);
    return;
  }
#endif
  for (uint64_t i = 0; i < n; ++i) out[i] = pack_sort_pair(keys[i], values[i]);
}

}  // extern "C"

// ---- automatic framing (crates/gsplat-ffi-c/src/lib.rs:1593-1779) --------
// The reference's context camera for gsplat_context_set_auto_camera: the
// scene's bounding box (scene_bounds, :1764-1779), a distance that frames it
// at the default camera's field of view (auto_surface_camera_control,
// :1601-1637), and the camera placed at yaw = pitch = 0 looking at the box
// centre (surface_camera_from_control, :1652-1677) with the rotation of
// camera_rotation_looking_at / quat_from_camera_basis (:1679-1733). Every
// step is one f32 operation in the reference's order.
namespace {
struct V3 {
  float x, y, z;
};
V3 v3_sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 v3_cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
bool v3_normalize(V3 v, V3 &out) {
  const float len = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
  if (!std::isfinite(len) || len <= 1.0e-6f) return false;
  const float inv = 1.0f / len;
  out = {v.x * inv, v.y * inv, v.z * inv};
  return true;
}
void look_at_rotation(V3 position, V3 target, float q[4]) {
  V3 forward;
  if (!v3_normalize(v3_sub(target, position), forward)) forward = {0.0f, 0.0f, 1.0f};
  const V3 world_up = std::fabs(forward.y) > 0.98f ? V3{0.0f, 0.0f, 1.0f} : V3{0.0f, 1.0f, 0.0f};
  V3 right;
  if (!v3_normalize(v3_cross(world_up, forward), right)) right = {1.0f, 0.0f, 0.0f};
  const V3 up = v3_cross(forward, right);
  // rotation matrix with columns right, up, forward -> quaternion
  const float m00 = right.x, m01 = up.x, m02 = forward.x;
  const float m10 = right.y, m11 = up.y, m12 = forward.y;
  const float m20 = right.z, m21 = up.z, m22 = forward.z;
  const float trace = m00 + m11 + m22;
  float x, y, z, w;
  if (trace > 0.0f) {
    const float s = std::sqrt(trace + 1.0f) * 2.0f;
    x = (m21 - m12) / s; y = (m02 - m20) / s; z = (m10 - m01) / s; w = 0.25f * s;
  } else if (m00 > m11 && m00 > m22) {
    const float s = std::sqrt(1.0f + m00 - m11 - m22) * 2.0f;
    x = 0.25f * s; y = (m01 + m10) / s; z = (m02 + m20) / s; w = (m21 - m12) / s;
  } else if (m11 > m22) {
    const float s = std::sqrt(1.0f + m11 - m00 - m22) * 2.0f;
    x = (m01 + m10) / s; y = 0.25f * s; z = (m12 + m21) / s; w = (m02 - m20) / s;
  } else {
    const float s = std::sqrt(1.0f + m22 - m00 - m11) * 2.0f;
    x = (m02 + m20) / s; y = (m12 + m21) / s; z = 0.25f * s; w = (m10 - m01) / s;
  }
  const float norm = std::fmax(std::sqrt(x * x + y * y + z * z + w * w), 1.0e-6f);
  q[0] = x / norm; q[1] = y / norm; q[2] = z / norm; q[3] = w / norm;
}
// f32::to_radians: the value times (PI / 180) formed in f32.
float to_radians_f32(float deg) { return deg * (3.14159265358979323846f / 180.0f); }
}  // namespace

extern "C" void orc_camera_look_at(const float position[3], const float target[3], float q[4]) {
  look_at_rotation({position[0], position[1], position[2]}, {target[0], target[1], target[2]}, q);
}

extern "C" int32_t orc_auto_camera(const float *positions, uint64_t n, uint32_t width,
                                   uint32_t height, OrcCamera *out) {
  if (n == 0) return 1;  // the reference's InvalidArgument for an empty scene
  V3 mn{INFINITY, INFINITY, INFINITY}, mx{-INFINITY, -INFINITY, -INFINITY};
  for (uint64_t i = 0; i < n; ++i) {
    const float *p = positions + 3 * i;
    mn.x = std::fmin(mn.x, p[0]); mn.y = std::fmin(mn.y, p[1]); mn.z = std::fmin(mn.z, p[2]);
    mx.x = std::fmax(mx.x, p[0]); mx.y = std::fmax(mx.y, p[1]); mx.z = std::fmax(mx.z, p[2]);
  }
  const V3 center{(mn.x + mx.x) * 0.5f, (mn.y + mx.y) * 0.5f, (mn.z + mx.z) * 0.5f};
  const V3 extent{mx.x - mn.x, mx.y - mn.y, mx.z - mn.z};
  const float half_x = std::fmax(extent.x * 0.5f, 1e-3f);
  const float half_y = std::fmax(extent.y * 0.5f, 1e-3f);
  const float half_z = std::fmax(extent.z * 0.5f, 1e-3f);
  const float aspect = (float)width / (float)height;
  // Camera::default(). Read through a volatile so that the compiler cannot
  // fold tan/atan of a constant at build time (correctly rounded) where the
  // reference calls the platform's f32 libm at run time.
  volatile float default_fov_v = to_radians_f32(60.0f);
  const float default_fov = default_fov_v;
  const float vfov = std::fmax(default_fov, 1e-3f);
  const float hfov = 2.0f * std::atan(std::tan(vfov * 0.5f) * aspect);
  const float dist_y = half_y / std::tan(vfov * 0.5f);
  const float dist_x = half_x / std::tan(hfov * 0.5f);
  const float distance = (std::fmax(dist_y, dist_x) + half_z) * 1.2f;
  const float radius = std::fmax(std::fmax(half_x, half_y), half_z);
  // surface_camera_from_control with yaw = pitch = 0 (pitch clamped to +-1.45)
  const float yaw = 0.0f, pitch = 0.0f;
  const float cos_pitch = std::cos(pitch);
  const V3 offset{std::sin(yaw) * cos_pitch * distance, std::sin(pitch) * distance,
                  -std::cos(yaw) * cos_pitch * distance};
  const V3 pos{center.x + offset.x, center.y + offset.y, center.z + offset.z};
  OrcCamera c;
  c.position[0] = pos.x; c.position[1] = pos.y; c.position[2] = pos.z;
  look_at_rotation(pos, center, c.rotation_xyzw);
  c.vertical_fov_radians = default_fov;
  const float r = std::fmax(radius, 1.0e-3f);
  c.near_plane = std::fmax(distance - r * 2.0f, 0.01f);
  c.far_plane = std::fmax(distance + r * 8.0f, 100.0f);
  const float asp = std::fmax((float)width / (float)std::max<uint32_t>(height, 1u), 1.0e-3f);
  if (asp < 0.6f) c.vertical_fov_radians = to_radians_f32(65.0f);
  *out = c;
  return 0;
}
