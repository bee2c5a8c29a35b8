// K2: (tile, splat) pair emission, and the tile-range build. Tile ids are
// global over the views of a batch: views[v].tile_base + local tile.
//
// Emission walks the depth-sorted visible ids. Each block takes the next
// 1024 sorted positions from an atomic ticket, sums their tile counts (area
// of each splat's tile rect), and gets its global pair offset from a
// decoupled look-back, so pairs land in exactly the order a sequential walk
// would write them: depth order, then rect rows, then rect columns. The
// block then writes its pairs cooperatively: each warp walks the pairs of
// its 128 items 32 at a time, every lane finding its splat with a shuffle
// search over the items' inclusive pair counts, so a splat covering thousands
// of tiles is spread over the lanes. The digit histograms the tile sort needs
// are accumulated while the pairs are written.

#include "device_common.cuh"
#include "kernels.h"

namespace gsr {
namespace {

constexpr int kEmitThreads = 256;
constexpr int kEmitIpt = 4;
constexpr int kEmitItems = kEmitThreads * kEmitIpt;
constexpr int kEmitWarps = kEmitThreads / 32;

__global__ void __launch_bounds__(kEmitThreads) emit_kernel(EmitBuffers b) {
  __shared__ uint32_t s_incl[kEmitItems];
  __shared__ uint32_t s_id[kEmitItems];
  __shared__ uint2 s_rect[kEmitItems];
  __shared__ uint16_t s_vi[kEmitItems];
  __shared__ uint32_t s_wsum[kEmitThreads / 32];
  __shared__ uint32_t s_hist[3][256];
  __shared__ uint32_t s_block;
  __shared__ unsigned long long s_prefix;
  // View table columns: splat base, tile base, tiles per row.
  extern __shared__ uint32_t s_views[];
  uint32_t *s_vsb = s_views, *s_vtb = s_views + b.num_views, *s_vtx = s_views + 2 * b.num_views;
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_block = atomicAdd(&b.counters->emit_ticket, 1u);
  for (uint32_t k = tid; k < 3 * 256; k += kEmitThreads) (&s_hist[0][0])[k] = 0;
  for (uint32_t v = tid; v < b.num_views; v += kEmitThreads) {
    s_vsb[v] = b.views[v].splat_base;
    s_vtb[v] = b.views[v].tile_base;
    s_vtx[v] = b.views[v].p.tiles_x;
  }
  __syncthreads();
  // The sorted visible ids: this frame's, or the order reused from the last
  // sort (the plan keeps its count).
  const uint32_t V = b.depth_plan->n;
  const uint32_t block = s_block;
  const uint32_t start = block * kEmitItems;
  if (start >= V) return;
  const uint32_t *ids = b.depth_plan->final_buffer == 0 ? b.ids0 : b.ids1;

  uint32_t cnt[kEmitIpt];
  uint32_t local = 0;
#pragma unroll
  for (int k = 0; k < kEmitIpt; ++k) {
    uint32_t slot = tid * kEmitIpt + k;
    uint32_t j = start + slot;
    uint32_t id = 0, c = 0, vi = 0;
    uint2 r = make_uint2(0u, 0u);
    if (j < V) {
      id = ids[j];
      r = b.rects[id];
      uint32_t w = (r.y & 0xffffu) - (r.x & 0xffffu);
      uint32_t h = (r.y >> 16) - (r.x >> 16);
      c = w * h;
      uint32_t lo = 0, hi = b.num_views - 1;
      while (lo < hi) {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (s_vsb[mid] <= id) lo = mid;
        else hi = mid - 1;
      }
      vi = lo;
    }
    s_id[slot] = id;
    s_rect[slot] = r;
    s_vi[slot] = (uint16_t)vi;
    cnt[k] = c;
    local += c;
  }
  // Block exclusive scan of the per-thread sums.
  uint32_t inc = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= (uint32_t)o) inc += t;
  }
  if (lane == 31) s_wsum[warp] = inc;
  __syncthreads();
  uint32_t before = 0, total = 0;
#pragma unroll
  for (int w = 0; w < kEmitThreads / 32; ++w) {
    uint32_t c = s_wsum[w];
    before += (w < (int)warp) ? c : 0u;
    total += c;
  }
  uint32_t run = before + inc - local;
#pragma unroll
  for (int k = 0; k < kEmitIpt; ++k) {
    run += cnt[k];
    s_incl[tid * kEmitIpt + k] = run;
  }
  if (warp == 0) {
    unsigned long long ex = lookback_warp(b.status, block, total, &b.counters->error);
    if (lane == 0) s_prefix = ex;
  }
  __syncthreads();
  const unsigned long long prefix = s_prefix;
  if (tid == 0 && block == (V - 1) / kEmitItems) {
    unsigned long long all = prefix + total;
    b.counters->keys = all;
    b.counters->pairs = (uint32_t)(all < b.capacity ? all : b.capacity);
    if (all > b.capacity) b.counters->overflow = 1u;
  }

  // Each warp writes the pairs of its own 128 items, 32 pairs per round. For
  // pair `my` a lane finds its item by a 5-step shuffle search over the
  // inclusive ends of a 32-item window starting at the round's first item.
  const uint32_t ib = warp * (kEmitItems / kEmitWarps);
  const uint32_t il = ib + kEmitItems / kEmitWarps - 1;
  uint32_t k = ib ? s_incl[ib - 1] : 0u;
  const uint32_t kend = s_incl[il];
  uint32_t it = ib;
  while (k < kend) {
    const uint32_t inc_w = s_incl[min(it + lane, il)];
    const uint32_t win_start = it ? s_incl[it - 1] : 0u;
    const uint32_t win_end = __shfl_sync(0xffffffffu, inc_w, 31);
    const uint32_t round_end = min(k + 32u, win_end);
    const uint32_t my = k + lane;
    uint32_t c = 0;
#pragma unroll
    for (uint32_t step = 16; step >= 1; step >>= 1) {
      uint32_t v = __shfl_sync(0xffffffffu, inc_w, c + step - 1);
      if (v <= my) c += step;
    }
    const uint32_t prev = __shfl_sync(0xffffffffu, inc_w, c ? c - 1 : 0);
    const unsigned long long g = prefix + my;
    if (my < round_end && g < b.capacity) {
      const uint32_t item = it + c;
      const uint32_t off = my - (c ? prev : win_start);
      const uint2 r = s_rect[item];
      const uint32_t x0 = r.x & 0xffffu, y0 = r.x >> 16;
      const uint32_t w = (r.y & 0xffffu) - x0;
      uint32_t row = (uint32_t)((float)off * (1.0f / (float)w));
      if (row * w > off) --row;
      else if ((row + 1) * w <= off) ++row;
      const uint32_t vi = s_vi[item];
      const uint32_t tile = s_vtb[vi] + (y0 + row) * s_vtx[vi] + x0 + (off - row * w);
      b.tile_keys[g] = tile;
      b.tile_vals[g] = s_id[item];
      atomicAdd(&s_hist[0][tile & 255u], 1u);
      // The higher digits of a round's tiles are mostly equal: one add per
      // distinct digit instead of up to 32 colliding ones.
      const uint32_t act = __activemask();
      const uint32_t lt = lanemask_lt();
      if (b.tile_passes > 1) {
        const uint32_t d1 = (tile >> 8) & 255u;
        const uint32_t peers = __match_any_sync(act, d1);
        if ((peers & lt) == 0) atomicAdd(&s_hist[1][d1], __popc(peers));
      }
      if (b.tile_passes > 2) {
        const uint32_t d2 = (tile >> 16) & 255u;
        const uint32_t peers = __match_any_sync(act, d2);
        if ((peers & lt) == 0) atomicAdd(&s_hist[2][d2], __popc(peers));
      }
    }
    it += __popc(__ballot_sync(0xffffffffu, inc_w <= round_end));
    k = round_end;
  }
  __syncthreads();
  for (uint32_t q = tid; q < b.tile_passes * 256; q += kEmitThreads) {
    uint32_t c = (&s_hist[0][0])[q];
    if (c) atomicAdd(&b.tile_hist[q], c);
  }
}

// Tile boundaries of the sorted keys: four keys per thread (one 16-byte
// load) plus the neighbour on each side.
__global__ void ranges_kernel(const SortPlan *__restrict__ plan, const uint32_t *k0,
                              const uint32_t *k1, const FrameCounters *__restrict__ counters,
                              uint2 *__restrict__ ranges) {
  const uint32_t K = counters->pairs;
  const uint32_t *keys = plan->final_buffer == 0 ? k0 : k1;
  const uint32_t groups = (K + 3) / 4;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < groups;
       q += gridDim.x * blockDim.x) {
    const uint32_t i0 = 4 * q;
    uint32_t v[6];
    if (i0 + 4 <= K) {
      const uint4 x = *reinterpret_cast<const uint4 *>(keys + i0);
      v[1] = x.x;
      v[2] = x.y;
      v[3] = x.z;
      v[4] = x.w;
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) v[1 + k] = i0 + k < K ? keys[i0 + k] : 0xffffffffu;
    }
    v[0] = i0 > 0 ? keys[i0 - 1] : 0xffffffffu;
    v[5] = i0 + 4 < K ? keys[i0 + 4] : 0xffffffffu;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t i = i0 + k;
      if (i >= K) break;
      const uint32_t t = v[1 + k];
      if (i == 0 || v[k] != t) ranges[t].x = i;
      if (i + 1 == K || v[2 + k] != t) ranges[t].y = i + 1;
    }
  }
}

__global__ void fill_kernel(uint32_t *dst, uint32_t value, uint64_t count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = value;
}

}  // namespace

void launch_emit(const EmitBuffers &b, cudaStream_t stream) {
  uint32_t blocks = (b.n + kEmitItems - 1) / kEmitItems;
  if (blocks == 0 || b.num_views == 0) return;
  emit_kernel<<<blocks, kEmitThreads, 3 * 4 * b.num_views, stream>>>(b);
}

void launch_ranges(const SortPlan *tile_plan, const uint32_t *keys0, const uint32_t *keys1,
                   const FrameCounters *counters, uint32_t capacity, uint2 *ranges,
                   cudaStream_t stream) {
  uint32_t blocks = (capacity + 255) / 256;
  blocks = blocks < 148 * 8 ? (blocks ? blocks : 1) : 148 * 8;
  ranges_kernel<<<blocks, 256, 0, stream>>>(tile_plan, keys0, keys1, counters, ranges);
}

void launch_fill_u32(uint32_t *dst, uint32_t value, uint64_t count, cudaStream_t stream) {
  if (count == 0) return;
  uint64_t blocks = (count + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  fill_kernel<<<(uint32_t)blocks, 256, 0, stream>>>(dst, value, count);
}

}  // namespace gsr
