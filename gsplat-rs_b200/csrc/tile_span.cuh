// Exact tile-row spans of a drawn splat, computed by the pair emission.
//
// For row ty of the splat's tile rect [x0, x1), the tile columns [c0, c1)
// whose pixel centres the ellipse |local| <= s can reach. q(dx, dy) =
// qa dx^2 + 2 qb dx dy + qc dy^2 is |local|^2 in pixel units; s^2 is widened
// by a relative 1e-5 and an absolute 1e-6, far above the rounding of the
// raster's weight threshold (alpha * exp(-4.5 r2) > 1/256 holds only for
// r2 < s^2 up to that rounding). The row's band is its pixel-centre rows
// +-0.5 px; within it the ellipse's x-extent (at the band ends, or at the
// leftmost/rightmost point when that lies inside the band) +-0.5 px selects
// the columns. A degenerate conic keeps the whole row.
//
// Every operation is one explicitly rounded IEEE f32 intrinsic, so the
// spans do not depend on the compiler's contraction setting and equal the
// CPU restatement bit for bit; no pixel changes, since the spans only drop
// tiles no pixel of which the splat reaches.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_types.h"

namespace gsr {

struct SpanPre {
  float qa, qb, qc, det, hx, hy, dy_left, s2a, inv_qa;
  bool degenerate;
};

// r.a = (cx, cy, ax, ay), r.b = (bx, by, s, alpha).
__device__ __forceinline__ SpanPre span_pre(float4 ra, float4 rb) {
  SpanPre p;
  p.qa = __fmaf_rn(ra.z, ra.z, __fmul_rn(rb.x, rb.x));
  p.qb = __fmaf_rn(ra.z, ra.w, __fmul_rn(rb.x, rb.y));
  p.qc = __fmaf_rn(ra.w, ra.w, __fmul_rn(rb.y, rb.y));
  const float s2 = __fmaf_rn(__fmul_rn(rb.z, rb.z), 1.00001f, 1e-6f);
  p.det = __fmaf_rn(p.qa, p.qc, -__fmul_rn(p.qb, p.qb));
  p.hx = __fsqrt_rn(__fdiv_rn(__fmul_rn(s2, p.qc), p.det));
  p.hy = __fsqrt_rn(__fdiv_rn(__fmul_rn(s2, p.qa), p.det));
  p.dy_left = __fdiv_rn(__fmul_rn(p.qb, p.hx), p.qc);
  p.s2a = __fmul_rn(s2, p.qa);
  p.inv_qa = __fdiv_rn(1.0f, p.qa);
  p.degenerate = !(p.det > 0.0f) || !(p.hx < 3.0e38f) || !(p.hy < 3.0e38f);
  return p;
}

// x-extent of the ellipse at band boundary y (relative to the centre): the
// left and right solutions of q(x, y) = s^2, NaN-free (the root is clamped).
__device__ __forceinline__ void boundary_x(const SpanPre &p, float y, float &xl, float &xr) {
  const float r = __fsqrt_rn(fmaxf(__fsub_rn(p.s2a, __fmul_rn(__fmul_rn(p.det, y), y)), 0.0f));
  const float by = __fmul_rn(-p.qb, y);
  xl = __fmul_rn(__fsub_rn(by, r), p.inv_qa);
  xr = __fmul_rn(__fadd_rn(by, r), p.inv_qa);
}

// Band [lo, hi] of tile row ty, clamped to the ellipse's y-extent.
__device__ __forceinline__ void row_band(float cy, const SpanPre &p, uint32_t ty, uint32_t tile,
                                         float &lo, float &hi) {
  lo = fmaxf(__fsub_rn(__fsub_rn((float)(ty * tile), 0.5f), cy), -p.hy);
  hi = fminf(__fsub_rn(__fsub_rn((float)(ty * tile + tile), 0.5f), cy), p.hy);
}

// Columns of a non-empty band from the x-extents at its two boundaries.
__device__ __forceinline__ uint2 band_columns(float cx, const SpanPre &p, float lo, float hi,
                                              float xl_lo, float xr_lo, float xl_hi, float xr_hi,
                                              float inv_tile, uint32_t x0, uint32_t x1) {
  float xmin = fminf(xl_lo, xl_hi);
  float xmax = fmaxf(xr_lo, xr_hi);
  if (p.dy_left >= lo && p.dy_left <= hi) xmin = -p.hx;
  if (-p.dy_left >= lo && -p.dy_left <= hi) xmax = p.hx;
  const float f0 =
      fmaxf(floorf(__fmul_rn(__fsub_rn(__fadd_rn(cx, xmin), 0.5f), inv_tile)), (float)x0);
  const float f1 = fminf(
      __fadd_rn(floorf(__fmul_rn(__fadd_rn(__fadd_rn(cx, xmax), 0.5f), inv_tile)), 1.0f),
      (float)x1);
  if (!(f0 < f1)) return make_uint2(x0, x0);
  return make_uint2((uint32_t)f0, (uint32_t)f1);
}

// Columns [c0, c1) of tile row ty (c0 == c1: none); inv_tile = 1 / tile
// exactly (tile is 8 or 16).
__device__ __forceinline__ uint2 row_span(float cx, float cy, const SpanPre &p, uint32_t ty,
                                          uint32_t tile, float inv_tile, uint32_t x0,
                                          uint32_t x1) {
  if (p.degenerate) return make_uint2(x0, x1);
  float lo, hi;
  row_band(cy, p, ty, tile, lo, hi);
  if (!(lo <= hi)) return make_uint2(x0, x0);
  float xl_lo, xr_lo, xl_hi, xr_hi;
  boundary_x(p, lo, xl_lo, xr_lo);
  boundary_x(p, hi, xl_hi, xr_hi);
  return band_columns(cx, p, lo, hi, xl_lo, xr_lo, xl_hi, xr_hi, inv_tile, x0, x1);
}

}  // namespace gsr
