// K4: per-tile raster. Built with --fmad=false; every fused multiply-add is
// an explicit fmaf, so a C++ restatement reproduces each pixel bit for bit.
//
// One block per tile; one thread per pixel, or two pixels of one row per
// thread for FP32 on 16x16 tiles (GSR_RASTER_PX, default 2). The tile's
// splat list (reference back-to-front order restricted to the tile) is
// staged into shared memory in chunks of records with cp.async (16-byte
// async copies, the record gather is random so tiled TMA does not apply),
// double-buffered so the next chunk's gather overlaps the current chunk's
// blending.
//
// Per pixel, the fragment rule of the reference shader
// (crates/gsplat-render-wgpu/shaders/splat_surface_direct.wgsl:336-369):
// local = inverse axis matrix * (pixel - centre); discard unless
// |local.x|, |local.y| <= s (the quad), r^2 = |local|^2 <= 1, and
// w = alpha * exp(-4.5 r^2) > 1/256; the source is (premult rgb * g, w).
//   FP32 mode: front to back (walks the list from its end); coverage is
//     r^2 <= s^2 and r^2 below the bound where w = 1/256 (in exact arithmetic
//     the same set as the quad clip, r^2 <= 1 and the alpha threshold);
//     C += rgb * (w T), T -= w T;
//     a pixel finishes once T < 1e-4, a warp when all its pixels have, the
//     block stops loading once all are done.
//   UNORM8 mode: back to front, dst = src + dst * (1 - w) rounded to UNORM8
//     after every splat (the reference's Rgba8Unorm premultiplied blend).

#include <algorithm>

#include "device_common.cuh"
#include "kernels.h"

#ifndef GSR_RASTER_PX
#define GSR_RASTER_PX 2
#endif
// Paired FP32 arithmetic for the two pixels of a thread (f32x2).
#ifndef GSR_RASTER_F32X2
#define GSR_RASTER_F32X2 1
#endif
// Resident blocks per SM the two-pixel FP32 kernel is compiled for: 8
// blocks of 4 warps fit 64 registers a thread without spills and 27 KB of
// shared memory a block (256-entry chunks); 10 or 12 spill and run slower.
#ifndef GSR_RASTER_MIN_BLOCKS
#define GSR_RASTER_MIN_BLOCKS 8
#endif


namespace gsr {
namespace {

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Block 0 folds the frame's error and overflow bits into the sticky word
// that gsplat_context_sync reports for enqueued frames.
__device__ __forceinline__ void fold_errors(const RasterArgs &a) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    uint32_t bits = a.counters->error | (a.counters->overflow ? 0x80000000u : 0u);
    if (bits) atomicOr(a.sticky, bits);
  }
}

// Which 8x4-pixel warp blocks of a kTile x kTile tile the ellipse
// |local|^2 <= thr reaches (bit band * kTile/8 + column block): for each
// 4-row band, the x-interval the ellipse spans within the band, plus half a
// pixel on every side, tested against the 8-column blocks. q(dx, dy) =
// A dx^2 + 2B dx dy + C dy^2 is |local|^2 in pixel units; (cxl, cyl) is the
// centre relative to the tile's first pixel. The mask only culls: hardware
// reciprocal/rsqrt (a few ulp) plus an inflation of the extents far above
// their error keeps it conservative.
template <int kTile>
__device__ __forceinline__ uint32_t ellipse_block_mask(float4 ra, float4 rb, float thr, float cxl,
                                                       float cyl) {
  constexpr int kBlocksX = kTile / 8;
  constexpr int kWarps = kTile * kTile / 32;
  const float qa = fmaf(ra.z, ra.z, rb.x * rb.x);
  const float qb = fmaf(ra.z, ra.w, rb.x * rb.y);
  const float qc = fmaf(ra.w, ra.w, rb.y * rb.y);
  const float det = fmaf(qa, qc, -qb * qb);
  const float inv_a = __fdividef(1.0f, qa);
  const float inv_det = __fdividef(1.0f, det);
  const float hx2 = thr * qc * inv_det, hy2 = thr * qa * inv_det;
  const float hx_raw = hx2 * rsqrtf(fmaxf(hx2, 1e-30f));
  const float hx = fmaf(hx_raw, 1.0001f, 1e-3f);
  const float hy = fmaf(hy2 * rsqrtf(fmaxf(hy2, 1e-30f)), 1.0001f, 1e-3f);
  // dy of the leftmost point (rightmost at -dy_left), from the unpadded extent
  const float dy_left = qb * hx_raw * __fdividef(1.0f, qc);
  const float s2a = thr * qa;
  constexpr float kPad = 0.5f + 1.0f / 64.0f;
  uint32_t mask = 0;
#pragma unroll
  for (int band = 0; band < kTile / 4; ++band) {
    const float lo = fmaxf((float)(4 * band) - 0.5f - cyl, -hy);
    const float hi = fminf((float)(4 * band) + 3.5f - cyl, hy);
    if (!(lo <= hi)) continue;
    const float qlo = fmaxf(s2a - det * lo * lo, 0.0f), qhi = fmaxf(s2a - det * hi * hi, 0.0f);
    const float r_lo = fmaf(qlo * rsqrtf(fmaxf(qlo, 1e-30f)), 1.0001f, 1e-3f);
    const float r_hi = fmaf(qhi * rsqrtf(fmaxf(qhi, 1e-30f)), 1.0001f, 1e-3f);
    float xmin = fminf((-qb * lo - r_lo) * inv_a, (-qb * hi - r_hi) * inv_a);
    float xmax = fmaxf((-qb * lo + r_lo) * inv_a, (-qb * hi + r_hi) * inv_a);
    if (dy_left >= lo && dy_left <= hi) xmin = -hx;
    if (-dy_left >= lo && -dy_left <= hi) xmax = hx;
    const float bx0f = cxl + xmin - kPad, bx1f = cxl + xmax + kPad;
#pragma unroll
    for (int colb = 0; colb < kBlocksX; ++colb)
      if (bx1f >= (float)(8 * colb) && bx0f <= (float)(8 * colb + 7))
        mask |= 1u << (band * kBlocksX + colb);
  }
  // A degenerate conic (never expected: axes are clamped to an anisotropy of
  // 64) falls back to every block.
  if (!(det > 0.0f) || !(hx < 3.0e38f) || !(hy < 3.0e38f)) mask = (1u << kWarps) - 1u;
  if (!(thr >= 0.0f)) mask = 0;
  return mask;
}

// Ordered compaction of the chunk entries whose mask meets sel (the warp's
// blocks) into list[] (ballots keep the list order); returns their count.
// Entries are stored as k << shift (shift 4: the byte offset of a float4
// array element).
__device__ __forceinline__ uint32_t compact_warp_entries(const uint8_t *mask, uint32_t n_in,
                                                        uint32_t sel, uint32_t lane,
                                                        uint16_t *list, uint32_t shift = 0) {
  uint32_t n_w = 0;
  for (uint32_t k0 = 0; k0 < n_in; k0 += 32) {
    const uint32_t k = k0 + lane;
    const bool hit = k < n_in && (mask[k] & sel) != 0;
    const uint32_t bal = __ballot_sync(0xffffffffu, hit);
    if (hit) list[n_w + __popc(bal & lanemask_lt())] = (uint16_t)(k << shift);
    n_w += __popc(bal);
  }
  __syncwarp();
  return n_w;
}

// UNORM8 parity mode: back to front over the tile list (forwards), the
// reference fragment rule with the quad clip, and the premultiplied OVER
// blend rounded to UNORM8 after every splat, exactly as the oracle's
// reference image model evaluates it. The blend has no early exit (a pixel's
// final value depends on every splat behind it), so the work it saves is
// culling: threads map to 8x4-pixel warp blocks as in the FP32 mode, one
// thread per chunk entry forms the entry's premultiplied colour (rgb * alpha,
// the vertex stage's product) and a conservative mask of the warp blocks the
// ellipse reaches (r^2 <= s^2, widened by a relative 1e-5 and an absolute
// 1e-6: alpha e^(-4.5 r^2) > 1/256 holds only below s^2 up to rounding), and
// each warp walks only the entries whose mask has its bit. A channel keeps
// its stored value both as the integer t and as f = RN(t / 255), the float
// the next blend reads.
template <int kTile>
struct U8Smem {
  static constexpr int kThreads = kTile * kTile;
  static constexpr int kWarps = kThreads / 32;
  static constexpr int kChunk = kTile * kTile;
  float4 raw[2][3][kChunk];  // (cx, cy, ax, ay), (bx, by, s, alpha), premultiplied rgb
  uint8_t mask[kChunk];
  uint16_t list[kWarps][kChunk];
  uint32_t view;
};

// RN(t / 255) for integer t in [0, 255] as t * 2^-8 + t * (1/255 - 2^-8)
// in one fma: exact for every such t (the first product is exact and the
// second's rounding never moves the sum across a rounding boundary), in two
// instructions instead of a division.
constexpr float kInv255Lo = 0x1.010102p-16f;  // RN(1/255 - 2^-8)

// One channel's blend step, dst = to_unorm8(fma(dst / 255, 1 - w, src)):
// saturate, scale by 255 and round to the nearest integer (ties to even) by
// the 1.5 * 2^23 addition, then the float the next step reads.
__device__ __forceinline__ void unorm8_step(float &f, float &t, float om, float src) {
  const float v = __saturatef(__fmaf_rn(f, om, src));
  t = __fsub_rn(__fadd_rn(__fmul_rn(v, 255.0f), kRoundMagic), kRoundMagic);
  f = __fmaf_rn(t, 0x1p-8f, __fmul_rn(t, kInv255Lo));
}

// 16x16 tiles: compiled for 4 resident blocks per SM (up to 64 registers a
// thread), which measured 2% faster than 5 blocks at 48 registers.
template <int kTile>
__global__ void __launch_bounds__(kTile *kTile, kTile == 16 ? 4 : 1)
    raster_unorm8_kernel(RasterArgs a) {
  using Smem = U8Smem<kTile>;
  constexpr int kN = Smem::kChunk;
  constexpr int kThreads = Smem::kThreads;
  constexpr int kBlocksX = kTile / 8;
  __shared__ Smem sm;
  fold_errors(a);
  const uint32_t tile = blockIdx.x;
  if (threadIdx.x == 0)
    sm.view = find_view(a.num_views, tile, [&](uint32_t v) { return a.views[v].tile_base; });
  __syncthreads();
  const uint32_t view = sm.view;
  const uint32_t width = a.views[view].p.width, height = a.views[view].p.height;
  const uint32_t tiles_x = a.views[view].p.tiles_x;
  uint32_t *__restrict__ image = a.images + a.views[view].image_base;
  const uint32_t local_tile = tile - a.views[view].tile_base;
  const uint32_t tx = local_tile % tiles_x, ty = local_tile / tiles_x;
  const uint32_t x0 = tx * kTile, y0 = ty * kTile;
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t px = x0 + (warp % kBlocksX) * 8 + (lane & 7);
  const uint32_t py = y0 + (warp / kBlocksX) * 4 + (lane >> 3);
  const bool inside = px < width && py < height;
  const float fpx = (float)px, fpy = (float)py;
  const float ftx = (float)x0, fty = (float)y0;
  const uint32_t *__restrict__ ids = a.plan->final_buffer == 0 ? a.ids0 : a.ids1;
  const uint2 range = a.ranges[tile];
  const uint32_t count = range.y - range.x;
  const uint32_t chunks = (count + kN - 1) / kN;
  auto issue = [&](uint32_t c, int buf) {
#pragma unroll
    for (uint32_t e = tid; e < (uint32_t)kN; e += kThreads) {
      const uint32_t k = c * kN + e;
      if (k < count) {
        const Record *r = &a.records[ids[range.x + k]];
        cp_async16(&sm.raw[buf][0][e], &r->a);
        cp_async16(&sm.raw[buf][1][e], &r->b);
        cp_async16(&sm.raw[buf][2][e], &r->c);
      }
    }
    cp_async_commit();
  };
  // j is the entry's byte offset into a float4 array of the chunk
  auto at = [&](const float4 *arr, uint32_t j) {
    return *reinterpret_cast<const float4 *>(reinterpret_cast<const char *>(arr) + j);
  };
  // Coverage and weight of entry j at this pixel (the reference fragment
  // rule), branch-free: a discarded fragment gets g = 0, om = 1 and alpha 0,
  // a step that leaves the stored value bit for bit as it is (sat(f) = f,
  // rint(f * 255) = t and RN(t / 255) = f for every stored t).
  auto weight = [&](int buf, uint32_t j, float &g, float &om, float &wa) {
    const float4 d0 = at(sm.raw[buf][0], j);
    const float4 d1 = at(sm.raw[buf][1], j);
    const float dpx = __fsub_rn(fpx, d0.x), dpy = __fsub_rn(fpy, d0.y);
    const float lx = __fmaf_rn(d0.z, dpx, __fmul_rn(d0.w, dpy));
    const float ly = __fmaf_rn(d1.x, dpx, __fmul_rn(d1.y, dpy));
    const float r2 = __fmaf_rn(lx, lx, __fmul_rn(ly, ly));
    // the exponential's argument stays in its domain [-4.5, 0]
    const float gg = exp_neg(__fmul_rn(-4.5f, fminf(r2, 1.0f)));
    const float w = __fmul_rn(d1.w, gg);
    const bool cov = fabsf(lx) <= d1.z && fabsf(ly) <= d1.z && r2 <= 1.0f && w > 1.0f / 256.0f;
    g = cov ? gg : 0.0f;
    om = cov ? __fsub_rn(1.0f, w) : 1.0f;
    wa = cov ? w : 0.0f;
  };
  float f[4] = {0.0f, 0.0f, 0.0f, 0.0f}, t[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  auto blend = [&](int buf, uint32_t j, float g, float om, float wa) {
    const float4 pc = at(sm.raw[buf][2], j);
    unorm8_step(f[0], t[0], om, __fmul_rn(pc.x, g));
    unorm8_step(f[1], t[1], om, __fmul_rn(pc.y, g));
    unorm8_step(f[2], t[2], om, __fmul_rn(pc.z, g));
    unorm8_step(f[3], t[3], om, wa);
  };
  if (chunks > 0) issue(0, 0);
  for (uint32_t c = 0; c < chunks; ++c) {
    const int buf = c & 1;
    if (c + 1 < chunks) issue(c + 1, buf ^ 1);
    else cp_async_commit();
    cp_async_wait_1();
    const uint32_t n_in = min((uint32_t)kN, count - c * kN);
#pragma unroll
    for (uint32_t e = tid; e < (uint32_t)kN; e += kThreads) {
      if (e < n_in) {
        const float4 ra = sm.raw[buf][0][e], rb = sm.raw[buf][1][e], rc = sm.raw[buf][2][e];
        sm.raw[buf][2][e] = make_float4(__fmul_rn(rc.x, rb.w), __fmul_rn(rc.y, rb.w),
                                        __fmul_rn(rc.z, rb.w), 0.0f);
        const float thr = __fmaf_rn(__fmul_rn(rb.z, rb.z), 1.00001f, 1e-6f);
        sm.mask[e] = (uint8_t)ellipse_block_mask<kTile>(ra, rb, thr, ra.x - ftx, ra.y - fty);
      }
    }
    __syncthreads();
    const uint32_t n_w = compact_warp_entries(sm.mask, n_in, 1u << warp, lane, sm.list[warp], 4);
    if (inside) {
      uint32_t i = 0;
      // two entries per step: the second's coverage and weight do not wait
      // for the first's blend
      for (; i + 1 < n_w; i += 2) {
        const uint32_t jj = *reinterpret_cast<const uint32_t *>(&sm.list[warp][i]);
        const uint32_t ja = jj & 0xffffu, jb = jj >> 16;
        float ga, oa, wa, gb, ob, wb;
        weight(buf, ja, ga, oa, wa);
        weight(buf, jb, gb, ob, wb);
        blend(buf, ja, ga, oa, wa);
        blend(buf, jb, gb, ob, wb);
      }
      if (i < n_w) {
        const uint32_t ja = sm.list[warp][i];
        float ga, oa, wa;
        weight(buf, ja, ga, oa, wa);
        blend(buf, ja, ga, oa, wa);
      }
    }
    __syncthreads();  // the next chunk's entries overwrite mask and list
  }
  cp_async_wait_all();
  if (inside)
    image[(size_t)py * width + px] =
        (uint32_t)t[0] | ((uint32_t)t[1] << 8) | ((uint32_t)t[2] << 16) | ((uint32_t)t[3] << 24);
}

// FP32 front-to-back mode. kPx = 1: threads map to 8x4-pixel warp blocks
// (lane l of warp w covers column (w % (kTile/8))*8 + (l & 7), row
// (w / (kTile/8))*4 + (l >> 3)). kPx = 2 (16x16 tiles): warp w covers the
// 16x4 band of rows 4w..4w+3, lane l the pixels (l & 7, 4w + (l >> 3)) and
// (8 + (l & 7), 4w + (l >> 3)): both share a row, so the row term of the
// local coordinates, fma(ay, y, ox), and the entry's three shared loads serve
// two pixels, and each pixel still evaluates the same expressions as with
// kPx = 1. Per chunk of kChunk list entries:
//   1. raw records arrive by cp.async (double-buffered, next chunk in flight);
//   2. one thread per entry derives, for this tile, the local offsets ox, oy
//      (local = (ax*lx + ay*ly + ox, bx*lx + by*ly + oy) for pixel coordinates
//      relative to the 16-pixel grid corner), s^2, and a bit mask of the 8x4
//      blocks the ellipse |local| <= s reaches (band intervals plus half a
//      pixel);
//   3. each warp compacts the entries whose mask meets its blocks (ballots
//      keep the list order) and blends only those; a pixel stops at
//      T < 1e-4, a warp when all its pixels have, the block when all pixels
//      have.
// Culling is conservative, so results equal the unculled per-pixel walk, and
// neither the chunk size, the pixels per thread nor the tile order changes
// any pixel.
template <int kTile, int kChunk, int kPx>
struct Fp32Smem {
  static_assert(kPx == 1 || (kPx == 2 && kTile == 16), "two pixels per thread on 16x16 tiles");
  static constexpr int kThreads = kTile * kTile / kPx;
  static constexpr int kWarps = kThreads / 32;
  // Chunk records as they arrive (a, b, c), overwritten in place by the
  // per-tile entry data: [0] = ax, ay, ox, thr (coverage bound on r^2);
  // [1] = bx, by, oy, -; [2] = r, g, b, log2 alpha (the record's c).
  float4 raw[2][3][kChunk];
  uint8_t mask[kChunk];
  uint16_t list[kWarps][kChunk];
  uint32_t view;
  uint32_t next;
};

template <int kTile, int kChunk, int kPx>
__device__ __forceinline__ void raster_fp32_tile(const RasterArgs &a, uint32_t tile,
                                                 Fp32Smem<kTile, kChunk, kPx> &sm) {
  constexpr int kBlocksX = kTile / 8;
  constexpr int kThreads = Fp32Smem<kTile, kChunk, kPx>::kThreads;
  if (threadIdx.x == 0)
    sm.view = find_view(a.num_views, tile, [&](uint32_t v) { return a.views[v].tile_base; });
  __syncthreads();
  const uint32_t view = sm.view;
  const uint32_t width = a.views[view].p.width, height = a.views[view].p.height;
  const uint32_t tiles_x = a.views[view].p.tiles_x;
  uint32_t *__restrict__ image = a.images + a.views[view].image_base;
  const uint32_t local_tile = tile - a.views[view].tile_base;
  const uint32_t tx = local_tile % tiles_x, ty = local_tile / tiles_x;
  const uint32_t x0 = tx * kTile, y0 = ty * kTile;
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t bx0 = kPx == 1 ? (warp % kBlocksX) * 8 : 0;
  const uint32_t by0 = kPx == 1 ? (warp / kBlocksX) * 4 : warp * 4;
  // the 8x4 blocks this warp's pixels lie in
  const uint32_t sel = kPx == 1 ? 1u << warp : 3u << (2 * warp);
  const uint32_t lxp = bx0 + (lane & 7), lyp = by0 + (lane >> 3);
  const uint32_t px = x0 + lxp, py = y0 + lyp;
  // Local coordinates are taken from the 16-pixel grid corner at or before
  // the tile, so 8x8 and 16x16 tiles evaluate every pixel identically.
  const uint32_t ax0 = x0 & ~15u, ay0 = y0 & ~15u;
  const float fy = (float)(py - ay0);
  float fx[kPx];
  bool inside[kPx];
#pragma unroll
  for (int p = 0; p < kPx; ++p) {
    fx[p] = (float)(px + 8 * p - ax0);
    inside[p] = px + 8 * p < width && py < height;
  }
  const float fax = (float)ax0, fay = (float)ay0;
  const float ftx = (float)x0, fty = (float)y0;
  const uint32_t *__restrict__ ids = a.plan->final_buffer == 0 ? a.ids0 : a.ids1;
  const uint2 range = a.ranges[tile];
  const uint32_t count = range.y - range.x;
  const uint32_t chunks = (count + kChunk - 1) / kChunk;

  auto issue = [&](uint32_t c, int buf) {
#pragma unroll
    for (uint32_t t = tid; t < (uint32_t)kChunk; t += kThreads) {
      const uint32_t k = c * kChunk + t;
      if (k < count) {
        const Record *r = &a.records[ids[range.y - 1 - k]];
        cp_async16(&sm.raw[buf][0][t], &r->a);
        cp_async16(&sm.raw[buf][1][t], &r->b);
        cp_async16(&sm.raw[buf][2][t], &r->c);
      }
    }
    cp_async_commit();
  };

  float T[kPx], c0[kPx], c1[kPx], c2[kPx];
  bool done[kPx];
#pragma unroll
  for (int p = 0; p < kPx; ++p) {
    T[p] = 1.0f;
    c0[p] = c1[p] = c2[p] = 0.0f;
    done[p] = !inside[p];
  }
  auto all_done = [&]() {
    bool d = true;
#pragma unroll
    for (int p = 0; p < kPx; ++p) d = d && done[p];
    return d;
  };
  if (chunks > 0) issue(0, 0);
  for (uint32_t c = 0; c < chunks; ++c) {
    const int buf = c & 1;
    if (c + 1 < chunks) issue(c + 1, buf ^ 1);
    else cp_async_commit();
    cp_async_wait_1();
    const uint32_t n_in = min((uint32_t)kChunk, count - c * kChunk);
#pragma unroll
    for (uint32_t t = tid; t < (uint32_t)kChunk; t += kThreads) {
      if (t < n_in) {
        const float4 ra = sm.raw[buf][0][t], rb = sm.raw[buf][1][t], col = sm.raw[buf][2][t];
        float cxa = ra.x - fax, cya = ra.y - fay;
        float ox = -fmaf(ra.z, cxa, ra.w * cya);
        float oy = -fmaf(rb.x, cxa, rb.y * cya);
        float cxl = ra.x - ftx, cyl = ra.y - fty;
        // w > 1/256 exactly when r2 < (log2 alpha + 8) / (4.5 log2 e), so a
        // pixel is covered when r2 <= thr: the largest float below that
        // bound, capped at s^2 (nothing is covered when the bound is not
        // positive).
        const float s2 = rb.z * rb.z;
        const float wlim = __fdiv_rn(col.w + 8.0f, 6.49212768f);
        const float thr =
            wlim > 0.0f ? fminf(s2, __int_as_float(__float_as_int(wlim) - 1)) : -1.0f;
        sm.raw[buf][0][t] = make_float4(ra.z, ra.w, ox, thr);
        sm.raw[buf][1][t] = make_float4(rb.x, rb.y, oy, rb.w);
        // debug tap: the inputs and the bound this kernel blends with (every
        // tile of a splat writes the same pair)
        if (a.debug_cov) a.debug_cov[ids[range.y - 1 - (c * kChunk + t)]] = make_float2(col.w, thr);
        sm.mask[t] = (uint8_t)ellipse_block_mask<kTile>(ra, rb, thr, cxl, cyl);
      }
    }
    __syncthreads();
    // Ordered compaction of this warp's entries (as byte offsets).
    const uint32_t n_w = compact_warp_entries(sm.mask, n_in, sel, lane, sm.list[warp], 4);
    // Four list entries per step (one early-out vote, one packed index
    // load); each pixel still takes them strictly in list order.
    // w = alpha e^(-4.5 r2) = 2^(log2 alpha - 4.5 log2(e) r2) (the entry's
    // log2 alpha in its colour's w), so the colour takes rgb * (w T) and the
    // transmittance loses w T.
    // j is the entry's byte offset into the float4 arrays
    auto at = [&](const float4 *arr, uint32_t j) {
      return *reinterpret_cast<const float4 *>(reinterpret_cast<const char *>(arr) + j);
    };
    // Branch-free: a pixel that does not take the entry (finished, or not
    // covered) blends with wT = 0, which leaves C and T bit for bit as they
    // are (fma(x, 0, c) = c and T - 0 = T for finite x).
    const float4 *e0 = sm.raw[buf][0], *e1 = sm.raw[buf][1], *e2 = sm.raw[buf][2];
    auto entry = [&](uint32_t j) {
      const float4 d0 = at(e0, j);
      const float4 d1 = at(e1, j);
      const float4 col = at(e2, j);
      const float rx = fmaf(d0.y, fy, d0.z), ry = fmaf(d1.y, fy, d1.z);
      if constexpr (kPx == 2 && GSR_RASTER_F32X2) {
        // The two pixels' arithmetic as paired FP32 instructions (sm_100
        // f32x2, documented to round each component as the scalar operation;
        // T - wT is fma(wT, -1, T), the same single rounding). The images
        // equal the scalar build's byte for byte on the test workloads; the
        // FP32 mode is held to its tolerance, not to bit equality.
        const float2 fxp = make_float2(fx[0], fx[1]);
        const float2 lx = __ffma2_rn(make_float2(d0.x, d0.x), fxp, make_float2(rx, rx));
        const float2 ly = __ffma2_rn(make_float2(d1.x, d1.x), fxp, make_float2(ry, ry));
        const float2 r2 = __ffma2_rn(lx, lx, __fmul2_rn(ly, ly));
        const float2 arg =
            __ffma2_rn(r2, make_float2(-6.49212768f, -6.49212768f), make_float2(col.w, col.w));
        const float2 wt = __fmul2_rn(make_float2(ex2_approx(arg.x), ex2_approx(arg.y)),
                                     make_float2(T[0], T[1]));
        const bool take0 = !done[0] && r2.x <= d0.w, take1 = !done[1] && r2.y <= d0.w;
        const float2 wT = make_float2(take0 ? wt.x : 0.0f, take1 ? wt.y : 0.0f);
        const float2 n0 = __ffma2_rn(make_float2(col.x, col.x), wT, make_float2(c0[0], c0[1]));
        const float2 n1 = __ffma2_rn(make_float2(col.y, col.y), wT, make_float2(c1[0], c1[1]));
        const float2 n2 = __ffma2_rn(make_float2(col.z, col.z), wT, make_float2(c2[0], c2[1]));
        const float2 nt = __ffma2_rn(wT, make_float2(-1.0f, -1.0f), make_float2(T[0], T[1]));
        c0[0] = n0.x, c0[1] = n0.y;
        c1[0] = n1.x, c1[1] = n1.y;
        c2[0] = n2.x, c2[1] = n2.y;
        T[0] = nt.x, T[1] = nt.y;
        done[0] = done[0] || T[0] < 1e-4f;
        done[1] = done[1] || T[1] < 1e-4f;
      } else {
#pragma unroll
        for (int p = 0; p < kPx; ++p) {
          const float lx = fmaf(d0.x, fx[p], rx);
          const float ly = fmaf(d1.x, fx[p], ry);
          const float r2 = fmaf(lx, lx, ly * ly);
          const bool take = !done[p] && r2 <= d0.w;
          const float w = blend_weight(r2, col.w);
          const float wT = take ? w * T[p] : 0.0f;
          c0[p] = fmaf(col.x, wT, c0[p]);
          c1[p] = fmaf(col.y, wT, c1[p]);
          c2[p] = fmaf(col.z, wT, c2[p]);
          T[p] = T[p] - wT;
          done[p] = done[p] || T[p] < 1e-4f;
        }
      }
    };
    uint32_t i = 0;
    for (; i + 3 < n_w; i += 4) {
      if (__all_sync(0xffffffffu, all_done())) break;
      const uint2 jj = *reinterpret_cast<const uint2 *>(&sm.list[warp][i]);
      entry(jj.x & 0xffffu);
      entry(jj.x >> 16);
      entry(jj.y & 0xffffu);
      entry(jj.y >> 16);
    }
    for (; i < n_w; ++i) {
      if (__all_sync(0xffffffffu, all_done())) break;
      entry(sm.list[warp][i]);
    }
    if (__syncthreads_count(all_done()) == kThreads) break;
  }
  cp_async_wait_all();
#pragma unroll
  for (int p = 0; p < kPx; ++p)
    if (inside[p])
      image[(size_t)py * width + px + 8 * p] =
          to_unorm8(c0[p]) | (to_unorm8(c1[p]) << 8) | (to_unorm8(c2[p]) << 16) |
          (to_unorm8(1.0f - T[p]) << 24);
}

// One block per tile (kPersistent false), or a fixed grid of blocks that take
// tiles from a global queue (an atomic ticket over the batch's tiles) until
// it is empty.
template <int kTile, int kChunk, int kPx, bool kPersistent>
__global__ void __launch_bounds__(kTile *kTile / kPx, kPx == 2 ? GSR_RASTER_MIN_BLOCKS : 1)
    raster_fp32_kernel(RasterArgs a) {
  __shared__ Fp32Smem<kTile, kChunk, kPx> sm;
  fold_errors(a);
  if constexpr (!kPersistent) {
    raster_fp32_tile<kTile, kChunk, kPx>(a, blockIdx.x, sm);
  } else {
    for (;;) {
      if (threadIdx.x == 0) sm.next = atomicAdd(&a.counters->raster_ticket, 1u);
      __syncthreads();
      const uint32_t tile = sm.next;
      if (tile >= a.total_tiles) break;
      raster_fp32_tile<kTile, kChunk, kPx>(a, tile, sm);
      __syncthreads();  // shared memory is reused by the next tile
    }
  }
}

}  // namespace

void launch_raster(const RasterArgs &a, uint32_t tile, uint32_t blend_mode,
                   const RasterConfig &cfg, uint32_t sm_count, cudaStream_t stream) {
  if (a.total_tiles == 0) return;
  if (blend_mode == 1) {
    if (tile == 16)
      raster_unorm8_kernel<16><<<a.total_tiles, 256, 0, stream>>>(a);
    else
      raster_unorm8_kernel<8><<<a.total_tiles, 64, 0, stream>>>(a);
    return;
  }
  const bool persistent = cfg.blocks_per_sm > 0;
  const uint32_t grid =
      persistent ? std::min<uint32_t>(a.total_tiles, cfg.blocks_per_sm * sm_count) : a.total_tiles;
#define GSR_FP32(T, C, P)                                                        \
  do {                                                                           \
    if (persistent)                                                              \
      raster_fp32_kernel<T, C, P, true><<<grid, T * T / P, 0, stream>>>(a);      \
    else                                                                         \
      raster_fp32_kernel<T, C, P, false><<<grid, T * T / P, 0, stream>>>(a);     \
  } while (0)
  if (tile == 16) {
    if (cfg.chunk == 64) GSR_FP32(16, 64, GSR_RASTER_PX);
    else if (cfg.chunk == 128) GSR_FP32(16, 128, GSR_RASTER_PX);
    else GSR_FP32(16, 256, GSR_RASTER_PX);
  } else {
    if (cfg.chunk == 32) GSR_FP32(8, 32, 1);
    else GSR_FP32(8, 64, 1);
  }
#undef GSR_FP32
}

bool raster_config_valid(uint32_t tile, const RasterConfig &cfg) {
  const bool chunk_ok = tile == 16 ? (cfg.chunk == 64 || cfg.chunk == 128 || cfg.chunk == 256)
                                   : (cfg.chunk == 32 || cfg.chunk == 64);
  return chunk_ok && cfg.blocks_per_sm <= 32;
}

}  // namespace gsr
