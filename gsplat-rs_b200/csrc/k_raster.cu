// K4: per-tile raster. Built with --fmad=false; every fused multiply-add is
// an explicit fmaf, so a C++ restatement reproduces each pixel bit for bit.
//
// One block per tile, one thread per pixel. The tile's splat list (reference
// back-to-front order restricted to the tile) is staged into shared memory in
// chunks of one record per thread with cp.async (16-byte async copies, the
// record gather is random so tiled TMA does not apply), double-buffered so
// the next chunk's gather overlaps the current chunk's blending.
//
// Per pixel, the fragment rule of the reference shader
// (crates/gsplat-render-wgpu/shaders/splat_surface_direct.wgsl:336-369):
// local = inverse axis matrix * (pixel - centre); discard unless
// |local.x|, |local.y| <= s (the quad), r^2 = |local|^2 <= 1, and
// w = alpha * exp(-4.5 r^2) > 1/256; the source is (premult rgb * g, w).
//   FP32 mode: front to back (walks the list from its end); coverage is
//     r^2 <= s^2 and w > 1/256 (in exact arithmetic the same set as the quad
//     clip, r^2 <= 1 and the alpha threshold); C += premult * (g T),
//     T *= 1 - w; a pixel finishes once T < 1e-4, a warp when all its pixels
//     have, the block stops loading once all are done.
//   UNORM8 mode: back to front, dst = src + dst * (1 - w) rounded to UNORM8
//     after every splat (the reference's Rgba8Unorm premultiplied blend).

#include "device_common.cuh"
#include "kernels.h"

namespace gsr {
namespace {

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// UNORM8 parity mode: back to front over the tile list, the reference
// fragment rule with the quad clip, rounding to UNORM8 after every blend.
// Per-block prologue shared by both raster kernels: fold the frame's error
// bits into the sticky word (block 0) and find the view of this global tile.
__device__ __forceinline__ uint32_t raster_view(const ViewDev *__restrict__ views,
                                                uint32_t num_views,
                                                const FrameCounters *__restrict__ counters,
                                                uint32_t *sticky, uint32_t *s_view) {
  if (threadIdx.x == 0) {
    if (blockIdx.x == 0) {
      uint32_t bits = counters->error | (counters->overflow ? 0x80000000u : 0u);
      if (bits) atomicOr(sticky, bits);
    }
    *s_view = find_view(num_views, blockIdx.x, [&](uint32_t v) { return views[v].tile_base; });
  }
  __syncthreads();
  return *s_view;
}

template <int kTile>
__global__ void __launch_bounds__(kTile *kTile) raster_unorm8_kernel(
    const ViewDev *__restrict__ views, uint32_t num_views, const uint2 *__restrict__ ranges,
    const SortPlan *__restrict__ plan, const uint32_t *__restrict__ ids0,
    const uint32_t *__restrict__ ids1, const Record *__restrict__ records,
    uint32_t *__restrict__ images, const FrameCounters *__restrict__ counters, uint32_t *sticky) {
  constexpr int kN = kTile * kTile;
  __shared__ float4 s_a[2][kN];
  __shared__ float4 s_b[2][kN];
  __shared__ float4 s_c[2][kN];
  __shared__ uint32_t s_view;
  const uint32_t view = raster_view(views, num_views, counters, sticky, &s_view);
  const FrameParams p = views[view].p;
  uint32_t *__restrict__ image = images + views[view].image_base;
  const uint32_t tile = blockIdx.x;
  const uint32_t local_tile = tile - views[view].tile_base;
  const uint32_t tx = local_tile % p.tiles_x, ty = local_tile / p.tiles_x;
  const uint32_t tid = threadIdx.x;
  const uint32_t px = tx * kTile + (tid % kTile);
  const uint32_t py = ty * kTile + (tid / kTile);
  const bool inside = px < p.width && py < p.height;
  const float fpx = (float)px, fpy = (float)py;
  const uint32_t *__restrict__ ids = plan->final_buffer == 0 ? ids0 : ids1;
  const uint2 range = ranges[tile];
  const uint32_t count = range.y - range.x;
  const uint32_t chunks = (count + kN - 1) / kN;
  auto issue = [&](uint32_t c, int buf) {
    uint32_t k = c * kN + tid;
    if (k < count) {
      const Record *r = &records[ids[range.x + k]];
      cp_async16(&s_a[buf][tid], &r->a);
      cp_async16(&s_b[buf][tid], &r->b);
      cp_async16(&s_c[buf][tid], &r->c);
    }
    cp_async_commit();
  };
  uint32_t d0 = 0, d1 = 0, d2 = 0, d3 = 0;
  if (chunks > 0) issue(0, 0);
  for (uint32_t c = 0; c < chunks; ++c) {
    const int buf = c & 1;
    if (c + 1 < chunks) issue(c + 1, buf ^ 1);
    else cp_async_commit();
    cp_async_wait_1();
    __syncthreads();
    const uint32_t n_in = min((uint32_t)kN, count - c * kN);
    if (inside) {
      for (uint32_t j = 0; j < n_in; ++j) {
        const float4 a = s_a[buf][j], b = s_b[buf][j], col = s_c[buf][j];
        float dpx = fpx - a.x, dpy = fpy - a.y;
        float lx = fmaf(a.z, dpx, a.w * dpy);
        float ly = fmaf(b.x, dpx, b.y * dpy);
        if (!(fabsf(lx) <= b.z && fabsf(ly) <= b.z)) continue;
        float r2 = fmaf(lx, lx, ly * ly);
        if (!(r2 <= 1.0f)) continue;
        float g = exp_neg(-4.5f * r2);
        float w = b.w * g;
        if (!(w > 1.0f / 256.0f)) continue;
        float om = 1.0f - w;
        d0 = to_unorm8(fmaf((float)d0 / 255.0f, om, col.x * g));
        d1 = to_unorm8(fmaf((float)d1 / 255.0f, om, col.y * g));
        d2 = to_unorm8(fmaf((float)d2 / 255.0f, om, col.z * g));
        d3 = to_unorm8(fmaf((float)d3 / 255.0f, om, w));
      }
    }
    __syncthreads();
  }
  cp_async_wait_all();
  if (inside) image[(size_t)py * p.width + px] = d0 | (d1 << 8) | (d2 << 16) | (d3 << 24);
}

// FP32 front-to-back mode. Threads map to 8x4-pixel warp blocks (lane l of
// warp w covers column (w % (kTile/8))*8 + (l & 7), row (w / (kTile/8))*4 +
// (l >> 3)). Per chunk of kN list entries:
//   1. raw records arrive by cp.async (double-buffered, next chunk in flight);
//   2. each thread derives, for its entry and this tile, the tile-local
//      offsets ox, oy (local = (ax*lx + ay*ly + ox, bx*lx + by*ly + oy) for
//      tile-local pixel coordinates), s^2, and a bit mask of the warp blocks
//      the splat's ellipse bounding box (plus one pixel) touches;
//   3. each warp compacts the entries whose mask has its bit (ballots keep the
//      list order) and blends only those; a pixel stops at T < 1e-4, a warp
//      when all 32 pixels have, the block when all pixels have.
// Culling is conservative, so results equal the unculled per-pixel walk.
template <int kTile>
__global__ void __launch_bounds__(kTile *kTile) raster_fp32_kernel(
    const ViewDev *__restrict__ views, uint32_t num_views, const uint2 *__restrict__ ranges,
    const SortPlan *__restrict__ plan, const uint32_t *__restrict__ ids0,
    const uint32_t *__restrict__ ids1, const Record *__restrict__ records,
    uint32_t *__restrict__ images, const FrameCounters *__restrict__ counters, uint32_t *sticky) {
  constexpr int kN = kTile * kTile;
  constexpr int kWarps = kN / 32;
  constexpr int kBlocksX = kTile / 8;
  __shared__ uint32_t s_view;
  __shared__ float4 s_raw[2][3][kN];
  __shared__ float4 s_d0[kN];  // ax, ay, ox, s2
  __shared__ float4 s_d1[kN];  // bx, by, oy, alpha
  __shared__ float4 s_d2[kN];  // r*alpha, g*alpha, b*alpha, -
  __shared__ uint8_t s_mask[kN];
  __shared__ uint16_t s_list[kWarps][kN];

  const uint32_t view = raster_view(views, num_views, counters, sticky, &s_view);
  const uint32_t width = views[view].p.width, height = views[view].p.height;
  const uint32_t tiles_x = views[view].p.tiles_x;
  uint32_t *__restrict__ image = images + views[view].image_base;
  const uint32_t tile = blockIdx.x;
  const uint32_t local_tile = tile - views[view].tile_base;
  const uint32_t tx = local_tile % tiles_x, ty = local_tile / tiles_x;
  const uint32_t x0 = tx * kTile, y0 = ty * kTile;
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t bx0 = (warp % kBlocksX) * 8, by0 = (warp / kBlocksX) * 4;
  const uint32_t lxp = bx0 + (lane & 7), lyp = by0 + (lane >> 3);
  const uint32_t px = x0 + lxp, py = y0 + lyp;
  const bool inside = px < width && py < height;
  // Local coordinates are taken from the 16-pixel grid corner at or before
  // the tile, so 8x8 and 16x16 tiles evaluate every pixel identically.
  const uint32_t ax0 = x0 & ~15u, ay0 = y0 & ~15u;
  const float fx = (float)(px - ax0), fy = (float)(py - ay0);
  const float fax = (float)ax0, fay = (float)ay0;
  const float ftx = (float)x0, fty = (float)y0;
  const uint32_t *__restrict__ ids = plan->final_buffer == 0 ? ids0 : ids1;
  const uint2 range = ranges[tile];
  const uint32_t count = range.y - range.x;
  const uint32_t chunks = (count + kN - 1) / kN;

  auto issue = [&](uint32_t c, int buf) {
    uint32_t k = c * kN + tid;
    if (k < count) {
      const Record *r = &records[ids[range.y - 1 - k]];
      cp_async16(&s_raw[buf][0][tid], &r->a);
      cp_async16(&s_raw[buf][1][tid], &r->b);
      cp_async16(&s_raw[buf][2][tid], &r->c);
    }
    cp_async_commit();
  };

  float T = 1.0f, c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
  bool done = !inside;
  if (chunks > 0) issue(0, 0);
  for (uint32_t c = 0; c < chunks; ++c) {
    const int buf = c & 1;
    if (c + 1 < chunks) issue(c + 1, buf ^ 1);
    else cp_async_commit();
    cp_async_wait_1();
    const uint32_t n_in = min((uint32_t)kN, count - c * kN);
    if (tid < n_in) {
      const float4 a = s_raw[buf][0][tid], b = s_raw[buf][1][tid], col = s_raw[buf][2][tid];
      float cxa = a.x - fax, cya = a.y - fay;
      float ox = -fmaf(a.z, cxa, a.w * cya);
      float oy = -fmaf(b.x, cxa, b.y * cya);
      float cxl = a.x - ftx, cyl = a.y - fty;
      s_d0[tid] = make_float4(a.z, a.w, ox, b.z * b.z);
      s_d1[tid] = make_float4(b.x, b.y, oy, b.w);
      s_d2[tid] = col;
      // Which 8x4 warp blocks the ellipse |local| <= s reaches: for each
      // 4-row band, the x-interval the ellipse spans within the band (plus
      // half a pixel on every side), tested against the two 8-column blocks.
      // q(dx, dy) = A dx^2 + 2B dx dy + C dy^2 is |local|^2 in pixel units.
      const float qa = fmaf(a.z, a.z, b.x * b.x);
      const float qb = fmaf(a.z, a.w, b.x * b.y);
      const float qc = fmaf(a.w, a.w, b.y * b.y);
      const float s2 = b.z * b.z;
      const float det = fmaf(qa, qc, -qb * qb);
      const float inv_a = 1.0f / qa;
      const float hx = sqrtf(s2 * qc / det);
      const float hy = sqrtf(s2 * qa / det);
      const float dy_left = qb * hx / qc;  // dy of the leftmost point; rightmost at -dy_left
      const float s2a = s2 * qa;
      uint32_t mask = 0;
#pragma unroll
      for (int band = 0; band < kTile / 4; ++band) {
        const float lo = fmaxf((float)(4 * band) - 0.5f - cyl, -hy);
        const float hi = fminf((float)(4 * band) + 3.5f - cyl, hy);
        if (!(lo <= hi)) continue;
        const float r_lo = sqrtf(fmaxf(s2a - det * lo * lo, 0.0f));
        const float r_hi = sqrtf(fmaxf(s2a - det * hi * hi, 0.0f));
        float xmin = fminf((-qb * lo - r_lo) * inv_a, (-qb * hi - r_hi) * inv_a);
        float xmax = fmaxf((-qb * lo + r_lo) * inv_a, (-qb * hi + r_hi) * inv_a);
        if (dy_left >= lo && dy_left <= hi) xmin = -hx;
        if (-dy_left >= lo && -dy_left <= hi) xmax = hx;
        const float x0 = cxl + xmin - 0.5f, x1 = cxl + xmax + 0.5f;
#pragma unroll
        for (int col = 0; col < kBlocksX; ++col)
          if (x1 >= (float)(8 * col) && x0 <= (float)(8 * col + 7))
            mask |= 1u << (band * kBlocksX + col);
      }
      // A degenerate conic (never expected: axes are clamped to an
      // anisotropy of 64) falls back to every block.
      if (!(det > 0.0f) || !(hx < 3.0e38f) || !(hy < 3.0e38f)) mask = (1u << kWarps) - 1u;
      s_mask[tid] = (uint8_t)mask;
    }
    __syncthreads();
    // Ordered compaction of this warp's entries.
    uint32_t n_w = 0;
    for (uint32_t k0 = 0; k0 < n_in; k0 += 32) {
      uint32_t k = k0 + lane;
      bool hit = k < n_in && ((s_mask[k] >> warp) & 1u);
      uint32_t bal = __ballot_sync(0xffffffffu, hit);
      if (hit) s_list[warp][n_w + __popc(bal & lanemask_lt())] = (uint16_t)k;
      n_w += __popc(bal);
    }
    __syncwarp();
    for (uint32_t i = 0; i < n_w; ++i) {
      if (__all_sync(0xffffffffu, done)) break;
      const uint32_t j = s_list[warp][i];
      const float4 d0 = s_d0[j];
      const float4 d1 = s_d1[j];
      float lx = fmaf(d0.x, fx, fmaf(d0.y, fy, d0.z));
      float ly = fmaf(d1.x, fx, fmaf(d1.y, fy, d1.z));
      float r2 = fmaf(lx, lx, ly * ly);
      if (done || !(r2 <= d0.w)) continue;
      float g = gauss_weight(r2);
      float w = d1.w * g;
      if (!(w > 1.0f / 256.0f)) continue;
      const float4 col = s_d2[j];
      float gT = g * T;
      c0 = fmaf(col.x, gT, c0);
      c1 = fmaf(col.y, gT, c1);
      c2 = fmaf(col.z, gT, c2);
      T = T * (1.0f - w);
      if (T < 1e-4f) done = true;
    }
    if (__syncthreads_count(done) == kN) break;
  }
  cp_async_wait_all();
  if (inside)
    image[(size_t)py * width + px] = to_unorm8(c0) | (to_unorm8(c1) << 8) |
                                       (to_unorm8(c2) << 16) | (to_unorm8(1.0f - T) << 24);
}

}  // namespace

void launch_raster(const ViewDev *views, uint32_t num_views, uint32_t total_tiles, uint32_t tile,
                   const uint2 *ranges, const SortPlan *tile_plan, const uint32_t *ids0,
                   const uint32_t *ids1, const Record *records, uint32_t *images,
                   uint32_t blend_mode, const FrameCounters *counters, uint32_t *sticky,
                   cudaStream_t stream) {
  if (total_tiles == 0) return;
  if (tile == 16) {
    if (blend_mode == 1)
      raster_unorm8_kernel<16><<<total_tiles, 256, 0, stream>>>(views, num_views, ranges, tile_plan, ids0, ids1, records, images, counters, sticky);
    else
      raster_fp32_kernel<16><<<total_tiles, 256, 0, stream>>>(views, num_views, ranges, tile_plan, ids0, ids1, records, images, counters, sticky);
  } else {
    if (blend_mode == 1)
      raster_unorm8_kernel<8><<<total_tiles, 64, 0, stream>>>(views, num_views, ranges, tile_plan, ids0, ids1, records, images, counters, sticky);
    else
      raster_fp32_kernel<8><<<total_tiles, 64, 0, stream>>>(views, num_views, ranges, tile_plan, ids0, ids1, records, images, counters, sticky);
  }
}

}  // namespace gsr
