// Oracle (test infrastructure only): the packed 20-byte hot record and the
// degree-3 SH sidecar of crates/gsplat-render-wgpu/src/packed_atlas.rs, and the
// decode that the CUDA renderer runs on a packed scene before its vertex stage
// (after splat_surface_packed.wgsl:128-241).
//
// Encoding (packed_atlas.rs): positions as u16 within the scene bounds
// (SceneBounds 53-102), opacity as the u8 of sigmoid(logit) (279-282), three
// u10 log scales over the scene's log-scale range (LogScaleRange 160-192),
// the smallest-three quaternion (285-316), the baked degree-0 colour
// clamp(C0 dc + 0.5) as RGB10 (335-342, 509-526) and the rest coefficients
// as i8 over per-channel maxima (386-400, 432-458; degree <= 3).
//
// Decode (the CUDA renderer's definition, following the WGSL): position =
// min + (u / 65535) span; alpha = clamp(u8 / 255, 1e-4, 1 - 1e-4) and its
// extent scale; axis variances exp(2 log_scale) from a per-scene table of the
// 1,024 codes; the quaternion unpacked, normalised (q / |q|) and turned into
// a rotation with the WGSL's doubled-component formulas; covariance terms
// sum_k s_k^2 r_ik r_jk; colour as the DC coefficient (rgb10 - 0.5) / C0 and
// the rest coefficients i8 / 127 * scale, so that the vertex stage's SH
// evaluation sees an ordinary (quantised) scene.

#include <cmath>
#include <cstdint>
#include <cstring>

#include "gsplat_oracle.h"

namespace {

float clamp01(float v) { return std::fmin(std::fmax(v, 0.0f), 1.0f); }

// Rust f32::round: half away from zero.
float round_away(float v) { return std::round(v); }

uint32_t to_u(float v) { return v > 0.0f ? (uint32_t)v : 0u; }  // saturating `as u32` of a clamped value

void quat_normalize_packed(const float q[4], float out[4]) {
  // packed_atlas.rs:377-384
  const float len2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  if (len2 <= 1e-20f) {
    out[0] = 0.0f; out[1] = 0.0f; out[2] = 0.0f; out[3] = 1.0f;
    return;
  }
  const float inv = 1.0f / std::sqrt(len2);
  for (int k = 0; k < 4; ++k) out[k] = q[k] * inv;
}

uint32_t pack_quat(const float qin[4]) {
  // packed_atlas.rs:285-316
  float q[4];
  quat_normalize_packed(qin, q);
  int max_index = 0;
  float max_abs = std::fabs(q[0]);
  for (int k = 1; k < 4; ++k)
    if (std::fabs(q[k]) > max_abs) {
      max_abs = std::fabs(q[k]);
      max_index = k;
    }
  if (q[max_index] < 0.0f)
    for (int k = 0; k < 4; ++k) q[k] = -q[k];
  const float scale = 0.70710678118654752440f;
  uint32_t packed = (uint32_t)max_index & 3u;
  int lane = 0;
  for (int k = 0; k < 4; ++k) {
    if (k == max_index) continue;
    const float t = clamp01((q[k] / scale) * 0.5f + 0.5f);
    packed |= (to_u(round_away(t * 1023.0f)) & 0x3FFu) << (2 + 10 * lane);
    ++lane;
  }
  return packed;
}

}  // namespace

extern "C" {

void orc_pack_scene(const OrcScene *sc, float *header, uint32_t *hot, int8_t *sidecar) {
  const uint64_t n = sc->count;
  // SceneBounds::from_positions
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::fmin(mn[a], sc->positions[3 * i + a]);
      mx[a] = std::fmax(mx[a], sc->positions[3 * i + a]);
    }
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(mn[a]) || !std::isfinite(mx[a]) || std::fabs(mx[a] - mn[a]) < 1e-6f) {
      mn[a] = 0.0f;
      mx[a] = 1.0f;
    }
  // LogScaleRange::from_scales
  float lmin = INFINITY, lmax = -INFINITY;
  for (uint64_t i = 0; i < 3 * n; ++i)
    if (std::isfinite(sc->scale_xyz[i])) {
      lmin = std::fmin(lmin, sc->scale_xyz[i]);
      lmax = std::fmax(lmax, sc->scale_xyz[i]);
    }
  if (!std::isfinite(lmin) || !std::isfinite(lmax)) {
    lmin = -8.0f;
    lmax = 8.0f;
  } else if (std::fabs(lmax - lmin) < 1e-6f) {
    lmax = lmin + 1e-3f;
  }
  // scene_sh_scales (degree <= 3: every rest coefficient fits the sidecar)
  const uint32_t degree = sc->sh_degree;
  const uint32_t pc = (degree + 1) * (degree + 1) - 1;
  float shs[3] = {1e-6f, 1e-6f, 1e-6f};
  if (sc->sh_rest && pc)
    for (uint64_t i = 0; i < n; ++i)
      for (int ch = 0; ch < 3; ++ch)
        for (uint32_t k = 0; k < pc; ++k)
          shs[ch] = std::fmax(shs[ch], std::fabs(sc->sh_rest[i * 3 * pc + ch * pc + k]));
  float span[3];
  for (int a = 0; a < 3; ++a) span[a] = std::fmax(mx[a] - mn[a], 1e-6f);
  const float lrange = std::fmax(lmax - lmin, 1e-6f);
  for (int a = 0; a < 3; ++a) {
    header[a] = mn[a];
    header[3 + a] = span[a];
    header[8 + a] = shs[a];
  }
  header[6] = lmin;
  header[7] = lmax - lmin;
  const float c0 = 0.2820948f;
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t *w = &hot[5 * i];
    uint32_t pos[3];
    for (int a = 0; a < 3; ++a) {
      const float t = clamp01((sc->positions[3 * i + a] - mn[a]) / span[a]);
      pos[a] = to_u(round_away(t * 65535.0f));
    }
    const float alpha = clamp01(1.0f / (1.0f + std::exp(-sc->opacity[i])));
    const uint32_t op = to_u(round_away(alpha * 255.0f));
    uint32_t scale_bits = 0;
    for (int a = 0; a < 3; ++a) {
      const float t = clamp01((sc->scale_xyz[3 * i + a] - lmin) / lrange);
      scale_bits |= to_u(round_away(t * 1023.0f)) << (10 * a);
    }
    uint32_t color = 0;
    for (int ch = 0; ch < 3; ++ch) {
      const float v = clamp01(c0 * sc->color_dc[3 * i + ch] + 0.5f);
      color |= (to_u(round_away(v * 1023.0f)) & 0x3FFu) << (10 * ch);
    }
    w[0] = pos[0] | (pos[1] << 16);
    w[1] = pos[2] | (op << 16);
    w[2] = scale_bits;
    w[3] = pack_quat(&sc->rotation_xyzw[4 * i]);
    w[4] = color;
    if (!sidecar) continue;
    int8_t *s = &sidecar[48 * i];
    std::memset(s, 0, 48);
    if (!sc->sh_rest) continue;
    for (int ch = 0; ch < 3; ++ch)
      for (uint32_t k = 0; k < pc && k < 15; ++k) {
        const float v = sc->sh_rest[i * 3 * pc + ch * pc + k];
        float q = round_away(v / std::fmax(shs[ch], 1e-6f) * 127.0f);
        q = std::fmin(std::fmax(q, -127.0f), 127.0f);
        s[ch * 15 + k] = (int8_t)q;
      }
  }
}

void orc_unpack_scene(uint64_t n, uint32_t sh_degree, const float *header, const uint32_t *hot,
                      const int8_t *sidecar, float *positions, float *alpha, float *extent,
                      float *cov6, float *color_dc, float *sh_rest) {
  // Per-scene tables: the 1,024 axis variances and the 256 extent scales.
  float var_lut[1024], ext_lut[256];
  for (uint32_t u = 0; u < 1024; ++u) {
    const float log_scale = header[6] + ((float)u / 1023.0f) * header[7];
    var_lut[u] = std::exp(2.0f * log_scale);
  }
  for (uint32_t u = 0; u < 256; ++u) {
    const float a = std::fmin(std::fmax((float)u / 255.0f, 1e-4f), 1.0f - 1e-4f);
    const float s2 = std::log(std::fmax(a, 1e-12f) * 256.0f) / 4.5f;
    ext_lut[u] = std::sqrt(std::fmin(std::fmax(s2, 0.0f), 1.0f));
  }
  const uint32_t pc = (sh_degree + 1) * (sh_degree + 1) - 1;
  const float c0 = 0.28209479177387814f, inv_sqrt2 = 0.70710678118654752440f;
  for (uint64_t i = 0; i < n; ++i) {
    const uint32_t *w = &hot[5 * i];
    const uint32_t pu[3] = {w[0] & 0xffffu, w[0] >> 16, w[1] & 0xffffu};
    for (int a = 0; a < 3; ++a)
      positions[3 * i + a] = header[a] + ((float)pu[a] / 65535.0f) * header[3 + a];
    const uint32_t op = (w[1] >> 16) & 0xffu;
    alpha[i] = std::fmin(std::fmax((float)op / 255.0f, 1e-4f), 1.0f - 1e-4f);
    extent[i] = ext_lut[op];
    const float sx2 = var_lut[w[2] & 0x3ffu], sy2 = var_lut[(w[2] >> 10) & 0x3ffu],
                sz2 = var_lut[(w[2] >> 20) & 0x3ffu];
    // smallest-three unpack, then q / |q|
    const uint32_t mi = w[3] & 3u;
    float c[3];
    for (int k = 0; k < 3; ++k)
      c[k] = ((float)((w[3] >> (2 + 10 * k)) & 0x3ffu) / 1023.0f * 2.0f - 1.0f) * inv_sqrt2;
    const float sum_sq = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
    const float dropped = std::sqrt(std::fmax(1.0f - sum_sq, 0.0f));
    float q[4];
    int r = 0;
    for (uint32_t k = 0; k < 4; ++k) q[k] = k == mi ? dropped : c[r++];
    const float len = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int k = 0; k < 4; ++k) q[k] = q[k] / len;
    const float x = q[0], y = q[1], z = q[2], ww = q[3];
    const float x2 = x + x, y2 = y + y, z2 = z + z;
    const float xx = x * x2, yy = y * y2, zz = z * z2;
    const float xy = x * y2, xz = x * z2, yz = y * z2;
    const float wx = ww * x2, wy = ww * y2, wz = ww * z2;
    const float rot[9] = {1.0f - (yy + zz), xy - wz, xz + wy,
                          xy + wz, 1.0f - (xx + zz), yz - wx,
                          xz - wy, yz + wx, 1.0f - (xx + yy)};
    auto term = [&](int a, int b) {
      return sx2 * rot[3 * a] * rot[3 * b] + sy2 * rot[3 * a + 1] * rot[3 * b + 1] +
             sz2 * rot[3 * a + 2] * rot[3 * b + 2];
    };
    float *cv = &cov6[6 * i];
    cv[0] = term(0, 0); cv[1] = term(0, 1); cv[2] = term(0, 2);
    cv[3] = term(1, 1); cv[4] = term(1, 2); cv[5] = term(2, 2);
    for (int ch = 0; ch < 3; ++ch) {
      const float v = (float)((w[4] >> (10 * ch)) & 0x3ffu) / 1023.0f;
      color_dc[3 * i + ch] = (v - 0.5f) / c0;
    }
    if (!sh_rest || !pc) continue;
    const int8_t *s = &sidecar[48 * i];
    for (int ch = 0; ch < 3; ++ch)
      for (uint32_t k = 0; k < pc; ++k)
        sh_rest[i * 3 * pc + ch * pc + k] = (float)s[ch * 15 + k] / 127.0f * header[8 + ch];
  }
}

// Test helper: how many of the given dividends x give a different f32 than
// the IEEE quotient x / d when divided as the CUDA packed decode does it (the
// product with RN(1/d), then one fma correction).
uint64_t orc_const_div_mismatches(float d, const float *x, uint64_t n) {
  const float r = 1.0f / d;
  uint64_t bad = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const float q = x[i] * r;
    const float refined = std::fma(std::fma(-q, d, x[i]), r, q);
    const float exact = x[i] / d;
    if (std::memcmp(&refined, &exact, 4) != 0) ++bad;
  }
  return bad;
}

}  // extern "C"
