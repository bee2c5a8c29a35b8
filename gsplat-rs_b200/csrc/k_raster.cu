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
//   FP32 mode: front to back (walks the list from its end); C += src * T,
//     T *= 1 - w; a pixel finishes once T < 1e-4, a warp leaves the chunk
//     when all its pixels have, the block stops loading once all are done.
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

template <int kTile, bool kUnorm8>
__global__ void __launch_bounds__(kTile *kTile) raster_kernel(
    FrameParams p, const uint2 *__restrict__ ranges, const SortPlan *__restrict__ plan,
    const uint32_t *__restrict__ ids0, const uint32_t *__restrict__ ids1,
    const Record *__restrict__ records, uint32_t *__restrict__ image,
    const FrameCounters *__restrict__ counters, uint32_t *sticky) {
  constexpr int kN = kTile * kTile;
  // The raster is the last kernel of a frame: fold the frame's error and
  // overflow flags into the word a deferred sync reads.
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    uint32_t bits = counters->error | (counters->overflow ? 0x80000000u : 0u);
    if (bits) atomicOr(sticky, bits);
  }
  __shared__ float4 s_a[2][kN];
  __shared__ float4 s_b[2][kN];
  __shared__ float4 s_c[2][kN];

  const uint32_t tile = blockIdx.x;
  const uint32_t tx = tile % p.tiles_x, ty = tile / p.tiles_x;
  const uint32_t tid = threadIdx.x;
  const uint32_t px = tx * kTile + (tid % kTile);
  const uint32_t py = ty * kTile + (tid / kTile);
  const bool inside = px < p.width && py < p.height;
  const float fpx = (float)px, fpy = (float)py;
  const uint32_t *__restrict__ ids = plan->final_buffer == 0 ? ids0 : ids1;
  const uint2 range = ranges[tile];
  const uint32_t count = range.y - range.x;
  const uint32_t chunks = (count + kN - 1) / kN;

  // Chunk c holds list positions (in processing order) c*kN .. c*kN+kN-1.
  auto issue = [&](uint32_t c, int buf) {
    uint32_t k = c * kN + tid;
    if (k < count) {
      uint32_t pos = kUnorm8 ? range.x + k : range.y - 1 - k;
      const Record *r = &records[ids[pos]];
      cp_async16(&s_a[buf][tid], &r->a);
      cp_async16(&s_b[buf][tid], &r->b);
      cp_async16(&s_c[buf][tid], &r->c);
    }
    cp_async_commit();
  };

  float T = 1.0f, c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
  uint32_t d0 = 0, d1 = 0, d2 = 0, d3 = 0;
  bool done = !inside;
  if (chunks > 0) issue(0, 0);
  for (uint32_t c = 0; c < chunks; ++c) {
    const int buf = c & 1;
    if (c + 1 < chunks) issue(c + 1, buf ^ 1);
    else cp_async_commit();
    cp_async_wait_1();
    __syncthreads();
    const uint32_t n_in = min((uint32_t)kN, count - c * kN);
    if (kUnorm8) {
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
    } else {
      for (uint32_t j = 0; j < n_in; ++j) {
        if (__all_sync(0xffffffffu, done)) break;
        if (done) continue;
        const float4 a = s_a[buf][j], b = s_b[buf][j];
        float dpx = fpx - a.x, dpy = fpy - a.y;
        float lx = fmaf(a.z, dpx, a.w * dpy);
        float ly = fmaf(b.x, dpx, b.y * dpy);
        if (!(fabsf(lx) <= b.z && fabsf(ly) <= b.z)) continue;
        float r2 = fmaf(lx, lx, ly * ly);
        if (!(r2 <= 1.0f)) continue;
        float g = exp_neg(-4.5f * r2);
        float w = b.w * g;
        if (!(w > 1.0f / 256.0f)) continue;
        const float4 col = s_c[buf][j];
        float tn = T * (1.0f - w);
        c0 = fmaf(col.x * g, T, c0);
        c1 = fmaf(col.y * g, T, c1);
        c2 = fmaf(col.z * g, T, c2);
        T = tn;
        if (T < 1e-4f) done = true;
      }
      if (__syncthreads_count(done) == kN) break;
    }
  }
  cp_async_wait_all();
  if (!inside) return;
  uint32_t out;
  if (kUnorm8) {
    out = d0 | (d1 << 8) | (d2 << 16) | (d3 << 24);
  } else {
    out = to_unorm8(c0) | (to_unorm8(c1) << 8) | (to_unorm8(c2) << 16) |
          (to_unorm8(1.0f - T) << 24);
  }
  image[(size_t)py * p.width + px] = out;
}

}  // namespace

void launch_raster(const FrameParams &p, const uint2 *ranges, const SortPlan *tile_plan,
                   const uint32_t *ids0, const uint32_t *ids1, const Record *records,
                   uint32_t *image, uint32_t blend_mode, const FrameCounters *counters,
                   uint32_t *sticky, cudaStream_t stream) {
  const uint32_t blocks = p.num_tiles;
  if (blocks == 0) return;
  if (p.tile == 16) {
    if (blend_mode == 1)
      raster_kernel<16, true><<<blocks, 256, 0, stream>>>(p, ranges, tile_plan, ids0, ids1, records, image, counters, sticky);
    else
      raster_kernel<16, false><<<blocks, 256, 0, stream>>>(p, ranges, tile_plan, ids0, ids1, records, image, counters, sticky);
  } else {
    if (blend_mode == 1)
      raster_kernel<8, true><<<blocks, 64, 0, stream>>>(p, ranges, tile_plan, ids0, ids1, records, image, counters, sticky);
    else
      raster_kernel<8, false><<<blocks, 64, 0, stream>>>(p, ranges, tile_plan, ids0, ids1, records, image, counters, sticky);
  }
}

}  // namespace gsr
