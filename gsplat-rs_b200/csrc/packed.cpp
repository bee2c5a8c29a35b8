// Packed resident scenes: the reference's compact encoding
// (crates/gsplat-render-wgpu/src/packed_atlas.rs) as a storage format that
// fits 3.5x more SH3 splats in HBM (68 instead of 240 bytes per splat); the
// preprocess kernel decodes it per frame.
//
// Encoding, as pack_scene does it (packed_atlas.rs:53-192, 279-342, 386-526):
// scene bounds and log-scale range over the scene, per-channel SH maxima,
// then per splat the u16 position within the bounds, the u8 of the clamped
// sigmoid opacity, three u10 log scales, the smallest-three quaternion, the
// RGB10 of clamp(C0 dc + 0.5) and the rest coefficients as i8 of
// value / max * 127 (Rust's round: half away from zero). The per-scene
// tables hold the values the decode needs from exp/log — the axis variance
// exp(2 log_scale) of each of the 1,024 scale codes and the extent scale of
// each of the 256 opacity codes — computed here with the C library's exp and
// log, so no transcendental function runs on the device.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

#include "cuda_check.h"
#include "pipeline.h"

namespace gsr {
namespace {

float clamp01(float v) { return std::fmin(std::fmax(v, 0.0f), 1.0f); }
uint32_t to_u(float v) { return v > 0.0f ? (uint32_t)v : 0u; }

uint32_t pack_quat(const float qin[4]) {
  // packed_atlas.rs:285-316, normalising as quat_normalize (377-384) does
  const float len2 = qin[0] * qin[0] + qin[1] * qin[1] + qin[2] * qin[2] + qin[3] * qin[3];
  float q[4] = {0.0f, 0.0f, 0.0f, 1.0f};
  if (!(len2 <= 1e-20f)) {
    const float inv = 1.0f / std::sqrt(len2);
    for (int k = 0; k < 4; ++k) q[k] = qin[k] * inv;
  }
  int mi = 0;
  for (int k = 1; k < 4; ++k)
    if (std::fabs(q[k]) > std::fabs(q[mi])) mi = k;
  if (q[mi] < 0.0f)
    for (float &v : q) v = -v;
  const float scale = 0.70710678118654752440f;
  uint32_t packed = (uint32_t)mi;
  for (int k = 0, lane = 0; k < 4; ++k) {
    if (k == mi) continue;
    const float t = clamp01((q[k] / scale) * 0.5f + 0.5f);
    packed |= (to_u(std::round(t * 1023.0f)) & 0x3FFu) << (2 + 10 * lane++);
  }
  return packed;
}

}  // namespace

PackedHost pack_scene_packed(const HostScene &s) {
  if (s.sh_degree > 3)
    throw Error(Code::Unsupported, "the packed scene format holds SH degree <= 3");
  const uint64_t n = s.size();
  PackedHost o;
  o.n = n;
  o.sh_degree = s.sh_degree;
  // SceneBounds::from_positions, LogScaleRange::from_scales, scene_sh_scales
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  float lmin = INFINITY, lmax = -INFINITY;
  const uint32_t pc = (s.sh_degree + 1) * (s.sh_degree + 1) - 1;
  float shs[3] = {1e-6f, 1e-6f, 1e-6f};
  for (uint64_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::fmin(mn[a], s.positions[3 * i + a]);
      mx[a] = std::fmax(mx[a], s.positions[3 * i + a]);
      const float l = s.scale_xyz[3 * i + a];
      if (std::isfinite(l)) {
        lmin = std::fmin(lmin, l);
        lmax = std::fmax(lmax, l);
      }
    }
    if (s.has_sh_rest)
      for (int ch = 0; ch < 3; ++ch)
        for (uint32_t k = 0; k < pc; ++k)
          shs[ch] = std::fmax(shs[ch], std::fabs(s.sh_rest[i * 3 * pc + ch * pc + k]));
  }
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(mn[a]) || !std::isfinite(mx[a]) || std::fabs(mx[a] - mn[a]) < 1e-6f) {
      mn[a] = 0.0f;
      mx[a] = 1.0f;
    }
  if (!std::isfinite(lmin) || !std::isfinite(lmax)) {
    lmin = -8.0f;
    lmax = 8.0f;
  } else if (std::fabs(lmax - lmin) < 1e-6f) {
    lmax = lmin + 1e-3f;
  }
  float span[3];
  for (int a = 0; a < 3; ++a) span[a] = std::fmax(mx[a] - mn[a], 1e-6f);
  const float lrange = std::fmax(lmax - lmin, 1e-6f);

  o.table.assign(kPackedFloats, 0.0f);
  float *h = o.table.data();
  for (int a = 0; a < 3; ++a) {
    h[a] = mn[a];
    h[3 + a] = span[a];
    h[8 + a] = shs[a];
  }
  h[6] = lmin;
  h[7] = lmax - lmin;
  for (uint32_t u = 0; u < kPackedVarLut; ++u)
    h[kPackedHeaderFloats + u] = std::exp(2.0f * (h[6] + ((float)u / 1023.0f) * h[7]));
  for (uint32_t u = 0; u < kPackedExtLut; ++u) {
    const float a = std::fmin(std::fmax((float)u / 255.0f, 1e-4f), 1.0f - 1e-4f);
    const float s2 = std::log(std::fmax(a, 1e-12f) * 256.0f) / 4.5f;
    h[kPackedHeaderFloats + kPackedVarLut + u] = std::sqrt(std::fmin(std::fmax(s2, 0.0f), 1.0f));
  }

  const uint64_t slots = std::max<uint64_t>(1, (n + 255) / 256) * 256;
  o.hot.assign(5 * slots, 0u);
  if (s.sh_degree > 0) o.sidecar.assign(48 * slots, 0);
  const float c0 = 0.2820948f;
  auto encode = [&](uint64_t b, uint64_t e) {
    for (uint64_t i = b; i < e; ++i) {
      uint32_t pos[3], scale_bits = 0, color = 0;
      for (int a = 0; a < 3; ++a) {
        pos[a] = to_u(std::round(clamp01((s.positions[3 * i + a] - mn[a]) / span[a]) * 65535.0f));
        scale_bits |=
            to_u(std::round(clamp01((s.scale_xyz[3 * i + a] - lmin) / lrange) * 1023.0f)) << (10 * a);
        color |= (to_u(std::round(clamp01(c0 * s.color_dc[3 * i + a] + 0.5f) * 1023.0f)) & 0x3FFu)
                 << (10 * a);
      }
      const float alpha = clamp01(1.0f / (1.0f + std::exp(-s.opacity[i])));
      uint32_t *w = &o.hot[5 * i];
      w[0] = pos[0] | (pos[1] << 16);
      w[1] = pos[2] | (to_u(std::round(alpha * 255.0f)) << 16);
      w[2] = scale_bits;
      w[3] = pack_quat(&s.rotation_xyzw[4 * i]);
      w[4] = color;
      if (o.sidecar.empty() || !s.has_sh_rest) continue;
      int8_t *sc = &o.sidecar[48 * i];
      for (int ch = 0; ch < 3; ++ch)
        for (uint32_t k = 0; k < pc; ++k) {
          const float v = s.sh_rest[i * 3 * pc + ch * pc + k];
          const float q = std::round(v / std::fmax(shs[ch], 1e-6f) * 127.0f);
          sc[ch * 15 + k] = (int8_t)std::fmin(std::fmax(q, -127.0f), 127.0f);
        }
    }
  };
  const unsigned hw = n < 65536 ? 1u : std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  const uint64_t chunk = (n + hw - 1) / hw;
  for (unsigned t = 0; t < hw; ++t) {
    const uint64_t b = t * chunk, e = std::min(n, b + chunk);
    if (b < e) pool.emplace_back(encode, b, e);
  }
  for (auto &th : pool) th.join();
  return o;
}

uint64_t packed_device_bytes(uint64_t n, uint32_t sh_degree) {
  const uint64_t slots = std::max<uint64_t>(1, (n + 255) / 256) * 256;
  return ((20 * slots + 255) & ~255ull) + (sh_degree ? 48 * slots : 0) + 4 * kPackedFloats;
}

std::unique_ptr<DeviceScene> upload_scene_packed(const HostScene &s, cudaStream_t stream) {
  if (s.size() > (1u << 30) - 1)
    throw Error(Code::Unsupported, "scene has more splats than the renderer supports (2^30 - 1)");
  PackedHost p = pack_scene_packed(s);
  auto sc = std::make_unique<DeviceScene>();
  sc->n = (uint32_t)p.n;
  sc->sh_degree = p.sh_degree;
  sc->positions = s.positions;
  const uint64_t hot_bytes = (4 * p.hot.size() + 255) & ~255ull;
  const uint64_t side_bytes = p.sidecar.size();
  sc->mem.reset(packed_device_bytes(p.n, p.sh_degree));
  char *base = sc->mem.as<char>();
  GSR_CUDA(cudaMemcpyAsync(base, p.hot.data(), 4 * p.hot.size(), cudaMemcpyHostToDevice, stream));
  if (side_bytes)
    GSR_CUDA(cudaMemcpyAsync(base + hot_bytes, p.sidecar.data(), side_bytes,
                             cudaMemcpyHostToDevice, stream));
  GSR_CUDA(cudaMemcpyAsync(base + hot_bytes + side_bytes, p.table.data(), 4 * p.table.size(),
                           cudaMemcpyHostToDevice, stream));
  GSR_CUDA(cudaStreamSynchronize(stream));
  sc->dev = SceneDev{};
  sc->dev.n = sc->n;
  sc->dev.planes = color_planes(p.sh_degree);
  sc->dev.hot = reinterpret_cast<const uint32_t *>(base);
  sc->dev.sidecar = side_bytes ? reinterpret_cast<const int8_t *>(base + hot_bytes) : nullptr;
  sc->dev.packed = reinterpret_cast<const float *>(base + hot_bytes + side_bytes);
  return sc;
}

}  // namespace gsr
