// K2: (tile, splat) pair emission, and the tile-range build. Tile ids are
// global over the views of a batch: views[v].tile_base + local tile.
//
// Emission walks the depth-sorted visible ids. Each block takes the next
// kEmitThreads * kEmitIpt sorted positions from an atomic ticket. A splat
// covers, per row of its tile rect, only the span of columns its ellipse
// reaches (tile_span.cuh), so the block first computes every row's span: each
// warp walks the rows of its own items 32 at a time (a lane finds its item by
// a 5-step shuffle search over the items' inclusive row counts), keeps the
// spans in shared memory and adds their widths to the items' pair counts.
// The block's total then gets its global pair offset from a decoupled
// look-back, so pairs land in exactly the order a sequential walk would write
// them: depth order, then rect rows, then the row's columns. Each warp then
// walks the same row windows again and writes the window's pairs 32 at a
// time (a lane finds its row by a second search over the rows' inclusive
// widths), so a splat covering thousands of tiles is spread over the lanes.
// The digit histograms the tile sort needs are accumulated while the pairs
// are written.

#include <algorithm>

#include "device_common.cuh"
#include "kernels.h"
#include "tile_span.cuh"

namespace gsr {
namespace {

// Sorted ids per thread: 2 up to GSR_EMIT_SMALL_IDS ids (more blocks in
// flight for a single frame), 4 above (fewer blocks, each reading the view
// table once) (tuning knob).
#ifndef GSR_EMIT_SMALL_IDS
#define GSR_EMIT_SMALL_IDS (1u << 21)
#endif
// Row spans each warp keeps between its two walks (tuning knob); rows past
// them are computed again in the second walk.
#ifndef GSR_EMIT_ROW_SLOTS
#define GSR_EMIT_ROW_SLOTS 256
#endif
constexpr int kEmitThreads = 256;
constexpr int kEmitWarps = kEmitThreads / 32;
constexpr uint32_t kRowSlots = GSR_EMIT_ROW_SLOTS;
constexpr uint64_t kEmitSmallIds = GSR_EMIT_SMALL_IDS;

inline uint32_t emit_ipt(uint64_t ids) { return ids <= kEmitSmallIds ? 2u : 4u; }

// Index of the first lane whose inclusive end exceeds x (31 when none does),
// by a 5-step shuffle search over the warp's ascending inclusive ends.
__device__ __forceinline__ uint32_t lane_search(uint32_t incl, uint32_t x) {
  uint32_t c = 0;
#pragma unroll
  for (uint32_t step = 16; step >= 1; step >>= 1) {
    const uint32_t v = __shfl_sync(0xffffffffu, incl, c + step - 1);
    if (v <= x) c += step;
  }
  return c;
}

// One window of a warp's row walk: rows r .. round_end-1 of the items from
// `it` on, one per lane. Both walks take the same windows.
struct RowWindow {
  uint32_t inc_w;      // inclusive row end of item it + lane (clamped to the warp's last)
  uint32_t round_end;  // one past the window's last row
  uint32_t item;       // the lane's item (valid when r + lane < round_end)
  uint32_t row;        // the lane's row within its item
};

__device__ __forceinline__ RowWindow row_window(const uint32_t *s_rinc, uint32_t ib, uint32_t il,
                                                uint32_t it, uint32_t r, uint32_t lane) {
  RowWindow w;
  w.inc_w = s_rinc[min(it + lane, il)];
  const uint32_t win_start = it > ib ? s_rinc[it - 1] : 0u;
  const uint32_t win_end = __shfl_sync(0xffffffffu, w.inc_w, 31);
  w.round_end = min(r + 32u, win_end);
  const uint32_t my = r + lane;
  const uint32_t c = lane_search(w.inc_w, my);
  const uint32_t prev = __shfl_sync(0xffffffffu, w.inc_w, c ? c - 1 : 0);
  w.item = it + c;
  w.row = my - (c ? prev : win_start);
  return w;
}

// Span [c0, c1) of row `ty` of splat `id` with tile rect rc.
__device__ __forceinline__ uint2 compute_row(const EmitBuffers &b, uint32_t id, uint2 rc,
                                             uint32_t ty, float inv_tile) {
  const Record *rec = &b.records[id];
  const float4 ra = rec->a, rb = rec->b;
  const SpanPre pre = span_pre(ra, rb);
  return row_span(ra.x, ra.y, pre, ty, b.tile, inv_tile, rc.x & 0xffffu, rc.y & 0xffffu);
}

template <int kEmitIpt>
__global__ void __launch_bounds__(kEmitThreads) emit_kernel(EmitBuffers b) {
  constexpr int kEmitItems = kEmitThreads * kEmitIpt;
  constexpr int kWarpItems = kEmitItems / kEmitWarps;
  __shared__ uint32_t s_rinc[kEmitItems];  // inclusive row counts within the warp's items
  __shared__ uint32_t s_cnt[kEmitItems];   // pair counts
  __shared__ uint32_t s_id[kEmitItems];
  __shared__ uint2 s_rect[kEmitItems];
  __shared__ uint16_t s_vi[kEmitItems];
  __shared__ uint32_t s_span[kEmitWarps][kRowSlots];  // c0 | c1 << 16 per warp row
  __shared__ uint32_t s_wsum[kEmitWarps];
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

  uint32_t rows[kEmitIpt];
  uint32_t local_rows = 0;
#pragma unroll
  for (int k = 0; k < kEmitIpt; ++k) {
    const uint32_t slot = tid * kEmitIpt + k;
    const uint32_t j = start + slot;
    uint32_t id = 0, h = 0, vi = 0;
    uint2 r = make_uint2(0u, 0u);
    if (j < V) {
      id = ids[j];
      r = b.rects[id];
      if ((r.y & 0xffffu) > (r.x & 0xffffu) && (r.y >> 16) > (r.x >> 16)) {
        h = (r.y >> 16) - (r.x >> 16);
        vi = find_view(b.num_views, id, [&](uint32_t v) { return s_vsb[v]; });
      }
    }
    s_id[slot] = id;
    s_rect[slot] = r;
    s_vi[slot] = (uint16_t)vi;
    s_cnt[slot] = 0;
    rows[k] = h;
    local_rows += h;
  }
  uint32_t rinc = local_rows;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, rinc, o);
    if (lane >= (uint32_t)o) rinc += t;
  }
  uint32_t rrun = rinc - local_rows;
#pragma unroll
  for (int k = 0; k < kEmitIpt; ++k) {
    rrun += rows[k];
    s_rinc[tid * kEmitIpt + k] = rrun;
  }
  __syncwarp();

  const uint32_t tile = b.tile;
  const float inv_tile = __fdiv_rn(1.0f, (float)tile);
  const uint32_t ib = warp * kWarpItems, il = ib + kWarpItems - 1;
  const uint32_t rows_total = s_rinc[il];
  // First walk: every row's span, kept for the second walk, summed per item.
  for (uint32_t r = 0, it = ib; r < rows_total;) {
    const RowWindow w = row_window(s_rinc, ib, il, it, r, lane);
    const uint32_t my = r + lane;
    if (my < w.round_end) {
      const uint2 rc = s_rect[w.item];
      const uint2 sp = compute_row(b, s_id[w.item], rc, (rc.x >> 16) + w.row, inv_tile);
      if (my < kRowSlots) s_span[warp][my] = sp.x | (sp.y << 16);
      if (sp.y > sp.x) atomicAdd(&s_cnt[w.item], sp.y - sp.x);
    }
    it += __popc(__ballot_sync(0xffffffffu, w.inc_w <= w.round_end));
    r = w.round_end;
  }
  __syncwarp();

  // Block exclusive scan of the per-thread pair sums.
  uint32_t local = 0;
#pragma unroll
  for (int k = 0; k < kEmitIpt; ++k) {
    const uint32_t slot = tid * kEmitIpt + k;
    local += s_cnt[slot];
  }
  uint32_t inc = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= (uint32_t)o) inc += t;
  }
  if (lane == 31) s_wsum[warp] = inc;
  __syncthreads();
  uint32_t before = 0, total = 0;
#pragma unroll
  for (int w = 0; w < kEmitWarps; ++w) {
    const uint32_t c = s_wsum[w];
    before += (w < (int)warp) ? c : 0u;
    total += c;
  }
  if (warp == 0) {
    const unsigned long long ex = lookback_warp(b.status, block, total, &b.counters->error);
    if (lane == 0) s_prefix = ex;
  }
  __syncthreads();
  const unsigned long long prefix = s_prefix;
  if (tid == 0 && block == (V - 1) / kEmitItems) {
    const unsigned long long all = prefix + total;
    b.counters->keys = all;
    b.counters->pairs = (uint32_t)(all < b.capacity ? all : b.capacity);
    if (all > b.capacity) b.counters->overflow = 1u;
  }

  // Second walk: the pairs of each row window, 32 per round.
  unsigned long long kpos = prefix + before;  // position of the warp's next pair
  for (uint32_t r = 0, it = ib; r < rows_total;) {
    const RowWindow w = row_window(s_rinc, ib, il, it, r, lane);
    const uint32_t my = r + lane;
    uint32_t c0 = 0, c1 = 0, row_tile = 0, id = 0;
    if (my < w.round_end) {
      const uint2 rc = s_rect[w.item];
      const uint32_t ty = (rc.x >> 16) + w.row;
      id = s_id[w.item];
      if (my < kRowSlots) {
        const uint32_t sp = s_span[warp][my];
        c0 = sp & 0xffffu;
        c1 = sp >> 16;
      } else {
        const uint2 sp = compute_row(b, id, rc, ty, inv_tile);
        c0 = sp.x;
        c1 = sp.y;
      }
      const uint32_t vi = s_vi[w.item];
      row_tile = s_vtb[vi] + ty * s_vtx[vi] + c0;  // global id of the span's first tile
    }
    uint32_t winc = c1 - c0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, winc, o);
      if (lane >= (uint32_t)o) winc += t;
    }
    const uint32_t W = __shfl_sync(0xffffffffu, winc, 31);
    for (uint32_t q = 0; q < W; q += 32) {
      const uint32_t myp = q + lane;
      const uint32_t j = lane_search(winc, myp);
      const uint32_t pj = __shfl_sync(0xffffffffu, winc, j ? j - 1 : 0);
      const uint32_t tj = __shfl_sync(0xffffffffu, row_tile, j);
      const uint32_t idj = __shfl_sync(0xffffffffu, id, j);
      const unsigned long long g = kpos + myp;
      if (myp < W && g < b.capacity) {
        const uint32_t t = tj + myp - (j ? pj : 0u);
        b.tile_keys[g] = t;
        b.tile_vals[g] = idj;
        atomicAdd(&s_hist[0][t & 255u], 1u);
        // The higher digits of a round's tiles are mostly equal: one add per
        // distinct digit instead of up to 32 colliding ones.
        const uint32_t act = __activemask();
        const uint32_t lt = lanemask_lt();
        if (b.tile_passes > 1) {
          const uint32_t d1 = (t >> 8) & 255u;
          const uint32_t peers = __match_any_sync(act, d1);
          if ((peers & lt) == 0) atomicAdd(&s_hist[1][d1], __popc(peers));
        }
        if (b.tile_passes > 2) {
          const uint32_t d2 = (t >> 16) & 255u;
          const uint32_t peers = __match_any_sync(act, d2);
          if ((peers & lt) == 0) atomicAdd(&s_hist[2][d2], __popc(peers));
        }
      }
    }
    kpos += W;
    it += __popc(__ballot_sync(0xffffffffu, w.inc_w <= w.round_end));
    r = w.round_end;
  }
  __syncthreads();
  for (uint32_t q = tid; q < b.tile_passes * 256; q += kEmitThreads) {
    const uint32_t n = (&s_hist[0][0])[q];
    if (n) atomicAdd(&b.tile_hist[q], n);
  }
}

// First position of a key >= t in the ascending keys[0, K).
__device__ __forceinline__ uint32_t lower_bound(const uint32_t *keys, uint32_t K, uint32_t t) {
  uint32_t lo = 0, hi = K;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (keys[mid] < t) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Tile boundaries of the sorted keys: four keys per thread (one 16-byte
// load) plus the neighbour on each side. The first num_views threads also
// count each view's pairs: its tiles are one contiguous id range, so its
// pairs are one run of the sorted keys.
__global__ void ranges_kernel(const SortPlan *__restrict__ plan, const uint32_t *k0,
                              const uint32_t *k1, const FrameCounters *__restrict__ counters,
                              uint2 *__restrict__ ranges, const ViewDev *__restrict__ views,
                              uint32_t num_views, ViewCounters *__restrict__ view_counters) {
  const uint32_t K = counters->pairs;
  const uint32_t *keys = plan->final_buffer == 0 ? k0 : k1;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid < num_views) {  // the first view starts at 0, the last ends at K
    const uint32_t first = tid ? lower_bound(keys, K, views[tid].tile_base) : 0u;
    const uint32_t end =
        tid + 1 < num_views ? lower_bound(keys, K, views[tid + 1].tile_base) : K;
    view_counters[tid].pairs = end - first;
  }
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

__global__ void run_init_kernel(RunInit a) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  if (blockIdx.x == 0 && a.inline_views) {
    static_assert(sizeof(ViewSetDev) % 4 == 0 && sizeof(ViewDev) % 4 == 0, "word copies");
    const uint32_t sw = a.inline_sets * (uint32_t)(sizeof(ViewSetDev) / 4);
    const uint32_t vw = a.inline_views * (uint32_t)(sizeof(ViewDev) / 4);
    const uint32_t *ss = reinterpret_cast<const uint32_t *>(a.sets);
    const uint32_t *vs = reinterpret_cast<const uint32_t *>(a.views);
    uint32_t *sd = reinterpret_cast<uint32_t *>(a.sets_dst);
    uint32_t *vd = reinterpret_cast<uint32_t *>(a.views_dst);
    for (uint32_t i = threadIdx.x; i < sw; i += blockDim.x) sd[i] = ss[i];
    for (uint32_t i = threadIdx.x; i < vw; i += blockDim.x) vd[i] = vs[i];
  }
#pragma unroll
  for (int r = 0; r < kRunZeroRegions; ++r)
    for (uint64_t i = t; i < a.zero_words[r]; i += stride) a.zero[r][i] = 0u;
}

__global__ void fill_kernel(uint32_t *dst, uint32_t value, uint64_t count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = value;
}

}  // namespace

uint64_t emit_blocks(uint64_t ids) {
  const uint64_t items = kEmitThreads * emit_ipt(ids);
  return (ids + items - 1) / items;
}

uint64_t emit_status_words(uint64_t capacity) {
  return std::max(emit_blocks(std::min(capacity, kEmitSmallIds)), emit_blocks(capacity));
}

void launch_emit(const EmitBuffers &b, cudaStream_t stream) {
  const uint32_t blocks = (uint32_t)emit_blocks(b.n);
  if (blocks == 0 || b.num_views == 0) return;
  const size_t smem = 3 * 4 * b.num_views;
  if (emit_ipt(b.n) == 2)
    emit_kernel<2><<<blocks, kEmitThreads, smem, stream>>>(b);
  else
    emit_kernel<4><<<blocks, kEmitThreads, smem, stream>>>(b);
}

void launch_ranges(const SortPlan *tile_plan, const uint32_t *keys0, const uint32_t *keys1,
                   const FrameCounters *counters, uint32_t capacity, uint2 *ranges,
                   const ViewDev *views, uint32_t num_views, ViewCounters *view_counters,
                   cudaStream_t stream) {
  uint32_t blocks = (capacity + 255) / 256;
  const uint32_t cap = 8 * device_sm_count();
  blocks = blocks < cap ? (blocks ? blocks : 1) : cap;
  blocks = std::max(blocks, (num_views + 255) / 256);
  ranges_kernel<<<blocks, 256, 0, stream>>>(tile_plan, keys0, keys1, counters, ranges, views,
                                            num_views, view_counters);
}

const void *run_init_kernel_entry() { return reinterpret_cast<const void *>(&run_init_kernel); }

void launch_run_init(const RunInit &a, cudaStream_t stream) {
  uint64_t words = 0;
  for (int r = 0; r < kRunZeroRegions; ++r) words = std::max(words, a.zero_words[r]);
  const uint64_t blocks = std::min<uint64_t>(std::max<uint64_t>((words + 255) / 256, 1), 8ull * device_sm_count());
  run_init_kernel<<<(uint32_t)blocks, 256, 0, stream>>>(a);
}

void launch_fill_u32(uint32_t *dst, uint32_t value, uint64_t count, cudaStream_t stream) {
  if (count == 0) return;
  uint64_t blocks = (count + 255) / 256;
  if (blocks > 16ull * device_sm_count()) blocks = 16ull * device_sm_count();
  fill_kernel<<<(uint32_t)blocks, 256, 0, stream>>>(dst, value, count);
}

}  // namespace gsr
