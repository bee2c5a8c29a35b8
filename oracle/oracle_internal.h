// Shared helpers of the CPU oracle (test infrastructure only).
#ifndef GSPLAT_ORACLE_INTERNAL_H
#define GSPLAT_ORACLE_INTERNAL_H

#include <cmath>
#include <cstdint>
#include <cstring>

#include "gsplat_oracle.h"

namespace orc {

void quat_normalize(const float q[4], float out[4]);
void quat_inverse(const float q[4], float out[4]);
void quat_to_mat3(const float q[4], float m[9]);
void frame_params(const OrcCamera &cam, uint32_t width, uint32_t height, uint32_t tile,
                  uint32_t sh_degree, OrcFrameParams &p);
void radix_sort_desc_u64_passes(uint64_t *values, uint64_t *scratch, uint64_t n, uint32_t lo,
                                uint32_t hi);

// f32::clamp / WGSL clamp for finite inputs.
inline float clamp_f(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }

inline float bits_to_float(uint32_t b) {
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}
inline uint32_t float_to_bits(float f) {
  uint32_t b;
  std::memcpy(&b, &f, 4);
  return b;
}

// e^x for x in [-4.5, 0]: Cody-Waite reduction to base 2 (t = x*log2(e),
// n = rint(t), f = t - n in [-0.5, 0.5]) and the degree-6 Taylor polynomial of
// 2^f = e^(f ln 2), coefficients ln(2)^k / k!. Relative error about 2e-7.
// The CUDA raster uses the same operation sequence, so CPU and GPU agree bit
// for bit.
inline float exp_neg(float x) {
  float t = x * 1.44269504088896341f;
  float n = std::nearbyint(t);
  float f = t - n;
  float p = std::fma(1.54035304e-4f, f, 1.33335581e-3f);
  p = std::fma(p, f, 9.61812911e-3f);
  p = std::fma(p, f, 5.55041087e-2f);
  p = std::fma(p, f, 2.40226507e-1f);
  p = std::fma(p, f, 6.93147181e-1f);
  p = std::fma(p, f, 1.0f);
  int32_t e = (int32_t)n;
  return bits_to_float(float_to_bits(p) + (uint32_t)(e * (1 << 23)));
}

// The FP32 tile model's blend weight alpha e^(-4.5 r2) = 2^t with
// t = fma(r2, -4.5 log2 e, log2 alpha): the 1.5 * 2^23 shifter gives the
// nearest integer n of t, f = t - n in [-0.5, 0.5] feeds the degree-6 Taylor
// polynomial of 2^f, and n is added to the exponent bits (relative error about
// 2e-7). The CUDA raster takes 2^t from the hardware base-2 exponential (a few
// ulp) and log2 alpha from the hardware logarithm, so its images equal this
// model's up to rare single UNORM8 steps: a weight on the 1/256 threshold, or
// a channel on a rounding boundary.
inline float blend_weight(float r2, float log2_alpha) {
  const float kShift = 12582912.0f;
  float t = std::fma(r2, -6.49212768f, log2_alpha);
  float tr = t + kShift;
  float n = tr - kShift;
  float f = t - n;
  float p = std::fma(1.54035304e-4f, f, 1.33335581e-3f);
  p = std::fma(p, f, 9.61812911e-3f);
  p = std::fma(p, f, 5.55041087e-2f);
  p = std::fma(p, f, 2.40226507e-1f);
  p = std::fma(p, f, 6.93147181e-1f);
  p = std::fma(p, f, 1.0f);
  return bits_to_float(float_to_bits(p) + (float_to_bits(tr) << 23));
}

// Round-to-nearest-even UNORM8 conversion of a value clamped to [0, 1].
inline uint8_t to_unorm8(float x) {
  float c = std::fmin(std::fmax(x, 0.0f), 1.0f);
  return (uint8_t)std::nearbyint(c * 255.0f);
}

// Per-pixel coverage and weight of one splat at integer pixel (px, py):
// fs_main (splat_surface_direct.wgsl:356-369) on the local quad coordinate,
// with the quad clip |lx|,|ly| <= s from vs_main (wgsl:336-354). Returns false
// when the fragment is discarded.
inline bool pixel_weight(const OrcRecord &r, int px, int py, float &g, float &w) {
  float dpx = (float)px - r.cx;
  float dpy = (float)py - r.cy;
  float lx = std::fma(r.ax, dpx, r.ay * dpy);
  float ly = std::fma(r.bx, dpx, r.by * dpy);
  if (!(std::fabs(lx) <= r.s && std::fabs(ly) <= r.s)) return false;
  float r2 = std::fma(lx, lx, ly * ly);
  if (!(r2 <= 1.0f)) return false;
  g = exp_neg(-4.5f * r2);
  w = r.alpha * g;
  return w > (1.0f / 256.0f);
}

// Exact tile-row culling (the CUDA design's pair emission): for row ty of a
// drawn splat's tile rect [x0, x1) x [y0, y1), the tile columns [c0, c1)
// whose pixel centres the ellipse |local| <= s can reach. q(dx, dy) =
// qa dx^2 + 2 qb dx dy + qc dy^2 is |local|^2 in pixel units; s^2 is widened
// by a relative 1e-5 and an absolute 1e-6, far above the rounding of the
// weight threshold (alpha * exp(-4.5 r2) > 1/256 holds only for r2 < s^2 up
// to that rounding). The row's band is its pixel-centre rows +-0.5 px; within
// it the ellipse's x-extent (at the band ends, or the leftmost/rightmost
// point when it lies inside the band) +-0.5 px selects the columns. A
// degenerate conic keeps the whole row. Every operation is a single IEEE f32
// operation (no contraction), as on the device.
struct SpanPre {
  float qa, qb, qc, det, hx, hy, dy_left, s2a, inv_qa;
  bool degenerate;
};

inline SpanPre span_pre(const OrcRecord &r) {
  SpanPre p;
  p.qa = std::fma(r.ax, r.ax, r.bx * r.bx);
  p.qb = std::fma(r.ax, r.ay, r.bx * r.by);
  p.qc = std::fma(r.ay, r.ay, r.by * r.by);
  const float s2 = std::fma(r.s * r.s, 1.00001f, 1e-6f);
  p.det = std::fma(p.qa, p.qc, -(p.qb * p.qb));
  p.hx = std::sqrt(s2 * p.qc / p.det);
  p.hy = std::sqrt(s2 * p.qa / p.det);
  p.dy_left = p.qb * p.hx / p.qc;
  p.s2a = s2 * p.qa;
  p.inv_qa = 1.0f / p.qa;
  p.degenerate = !(p.det > 0.0f) || !(p.hx < 3.0e38f) || !(p.hy < 3.0e38f);
  return p;
}

// inv_tile = 1 / tile, exact (tile is 8 or 16).
inline void row_span(const OrcRecord &r, const SpanPre &p, uint32_t ty, uint32_t tile,
                     float inv_tile, uint32_t x0, uint32_t x1, uint32_t &c0, uint32_t &c1) {
  c0 = x0;
  c1 = x1;
  if (p.degenerate) return;
  const float lo = std::fmax((float)(ty * tile) - 0.5f - r.cy, -p.hy);
  const float hi = std::fmin((float)(ty * tile + tile) - 0.5f - r.cy, p.hy);
  if (!(lo <= hi)) {
    c1 = x0;
    return;
  }
  const float r_lo = std::sqrt(std::fmax(p.s2a - p.det * lo * lo, 0.0f));
  const float r_hi = std::sqrt(std::fmax(p.s2a - p.det * hi * hi, 0.0f));
  const float blo = -p.qb * lo, bhi = -p.qb * hi;
  float xmin = std::fmin((blo - r_lo) * p.inv_qa, (bhi - r_hi) * p.inv_qa);
  float xmax = std::fmax((blo + r_lo) * p.inv_qa, (bhi + r_hi) * p.inv_qa);
  if (p.dy_left >= lo && p.dy_left <= hi) xmin = -p.hx;
  if (-p.dy_left >= lo && -p.dy_left <= hi) xmax = p.hx;
  const float f0 = std::fmax(std::floor((r.cx + xmin - 0.5f) * inv_tile), (float)x0);
  const float f1 = std::fmin(std::floor((r.cx + xmax + 0.5f) * inv_tile) + 1.0f, (float)x1);
  if (!(f0 < f1)) {
    c1 = x0;
    return;
  }
  c0 = (uint32_t)f0;
  c1 = (uint32_t)f1;
}

}  // namespace orc

#endif
