// K3: onesweep LSD radix sort of (u32 key, u32 value) pairs, ascending and
// stable, 8-bit digits, 256 threads and 8 or 16 keys per thread.
//
//   1. histogram kernel: one read of the keys builds the digit histograms of
//      every pass (shared-memory histograms, one global add per bin and block);
//   2. plan kernel (one block): exclusive digit offsets per pass; a pass whose
//      keys all share one digit is marked skipped, and the ping-pong buffer of
//      every remaining pass is fixed on the device, so no host round trip is
//      needed between passes;
//   3. one kernel per pass: each block takes the next tile of 256*IPT keys
//      from an atomic ticket (launch order, so look-back never waits on a
//      block that has not started), ranks its keys stably per digit with warp
//      ballots, publishes its digit counts, resolves its global digit
//      offsets by decoupled look-back over the predecessor tiles (bounded
//      waits), reorders the tile in shared memory and writes digit runs
//      contiguously.
//
// Stability over equal keys is what reproduces the reference's tie order
// (crates/gsplat-sort/src/radix.rs:11-58: stable LSD passes, equal keys keep
// their input order).

#include <algorithm>
#include <atomic>

#include "device_common.cuh"
#include "kernels.h"

namespace gsr {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
// Tuning knobs: resident pass blocks per SM the register allocation must
// allow (for 8 keys per thread, and for the large tile), and predecessor
// tiles read per look-back step.
#ifndef GSR_SORT_MIN_BLOCKS
#define GSR_SORT_MIN_BLOCKS 3
#endif
#ifndef GSR_SORT_MIN_BLOCKS_LARGE
#define GSR_SORT_MIN_BLOCKS_LARGE GSR_SORT_MIN_BLOCKS
#endif
#ifndef GSR_LOOKBACK_WIDTH
#define GSR_LOOKBACK_WIDTH 4
#endif
constexpr int kLookback = GSR_LOOKBACK_WIDTH;
constexpr uint32_t kFlagA = 1u << 30;
constexpr uint32_t kFlagP = 2u << 30;
constexpr uint32_t kMask = (1u << 30) - 1;

template <int kIpt>
__global__ void __launch_bounds__(kThreads) hist_kernel(const uint32_t *__restrict__ keys,
                                                        const uint32_t *__restrict__ count,
                                                        uint32_t begin_bit, uint32_t passes,
                                                        uint32_t *__restrict__ hist) {
  constexpr uint32_t kTile = kThreads * kIpt;
  __shared__ uint32_t s_hist[4][256];
  const uint32_t n = *count;
  const uint32_t base = blockIdx.x * kTile;
  if (base >= n) return;
  for (uint32_t k = threadIdx.x; k < 4 * 256; k += kThreads) (&s_hist[0][0])[k] = 0;
  __syncthreads();
  const uint32_t end = min(n, base + kTile);
  for (uint32_t idx = base + threadIdx.x; idx < end; idx += kThreads) {
    uint32_t key = keys[idx];
    for (uint32_t p = 0; p < passes; ++p) atomicAdd(&s_hist[p][(key >> (begin_bit + 8 * p)) & 255u], 1u);
  }
  __syncthreads();
  for (uint32_t p = 0; p < passes; ++p) {
    uint32_t c = s_hist[p][threadIdx.x];
    if (c) atomicAdd(&hist[p * 256 + threadIdx.x], c);
  }
}

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *s_wsum,
                                                         uint32_t &total) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= (uint32_t)o) inc += t;
  }
  if (lane == 31) s_wsum[warp] = inc;
  __syncthreads();
  uint32_t before = 0;
  total = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    uint32_t c = s_wsum[w];
    before += (w < (int)warp) ? c : 0u;
    total += c;
  }
  __syncthreads();
  return before + inc - v;
}

// Block 0 plans the passes; every block zeroes the look-back status words
// of the tiles the actual item count needs (not the capacity's).
__global__ void __launch_bounds__(kThreads) plan_kernel(const uint32_t *__restrict__ count,
                                                        const uint32_t *__restrict__ hist,
                                                        uint32_t passes, SortPlan *plan,
                                                        uint32_t *status, uint32_t tile_stride,
                                                        uint32_t tile_items) {
  const uint32_t n = *count;
  const uint64_t used = (uint64_t)((n + tile_items - 1) / tile_items) * 256u;  // words per pass
  for (uint32_t p = 0; p < passes; ++p) {
    uint4 *dst = reinterpret_cast<uint4 *>(status + (size_t)p * tile_stride * 256u);
    for (uint64_t k = blockIdx.x * (uint64_t)kThreads + threadIdx.x; k < used / 4;
         k += (uint64_t)gridDim.x * kThreads)
      dst[k] = make_uint4(0u, 0u, 0u, 0u);
  }
  if (blockIdx.x != 0) return;
  __shared__ uint32_t s_wsum[kWarps];
  __shared__ uint32_t s_trivial[4];
  const uint32_t d = threadIdx.x;
  if (d < 4) s_trivial[d] = 0;
  __syncthreads();
  for (uint32_t p = 0; p < passes; ++p) {
    uint32_t c = hist[p * 256 + d];
    uint32_t total;
    uint32_t ex = block_exclusive_scan(c, s_wsum, total);
    plan->digit_offset[p][d] = ex;
    if (c == n) s_trivial[p] = 1;  // n == 0 marks every pass trivial
  }
  __syncthreads();
  if (d == 0) {
    uint32_t buf = 0;
    for (uint32_t p = 0; p < 8; ++p) {
      uint32_t skip = p < passes ? s_trivial[p] : 1u;
      plan->skip[p] = skip;
      plan->src[p] = buf;
      if (!skip) buf ^= 1u;
    }
    plan->final_buffer = buf;
    plan->n = n;
    plan->passes = passes;
  }
}

template <int kIpt>
struct PassSmem {
  static constexpr uint32_t kTile = kThreads * kIpt;
  uint32_t warp_hist[kWarps][256];
  uint32_t keys[kTile];
  uint32_t vals[kTile];
  uint32_t block_start[256];
  uint32_t global[256];
  uint32_t wsum[kWarps];
  uint32_t tile;
};

// One tile of one pass: rank, publish, look back, reorder, scatter.
template <int kIpt>
__device__ __forceinline__ void pass_tile(const SortPlan *__restrict__ plan, uint32_t pass,
                                          uint32_t shift, uint32_t n, uint32_t tile,
                                          const uint32_t *__restrict__ in_k,
                                          const uint32_t *__restrict__ in_v,
                                          uint32_t *__restrict__ out_k,
                                          uint32_t *__restrict__ out_v, uint32_t *status,
                                          uint32_t *error, PassSmem<kIpt> &sm) {
  constexpr uint32_t kTile = PassSmem<kIpt>::kTile;
  auto &s_warp_hist = sm.warp_hist;
  auto &s_keys = sm.keys;
  auto &s_vals = sm.vals;
  auto &s_block_start = sm.block_start;
  auto &s_global = sm.global;
  const uint32_t base = tile * kTile;

  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t warp_base = base + warp * 32 * kIpt;
  // Large tiles (16 keys per thread) place their keys in shared memory
  // before the look-back and read the values from global memory only then,
  // which keeps keys, ranks and values from being live at once (fewer
  // registers and spills); small tiles load the values with the keys and
  // place both after the look-back (their look-back is short, and the
  // value loads stay off the critical path).
  constexpr bool kEarlyReorder = kIpt >= 16;
  uint32_t key[kIpt], val[kEarlyReorder ? 1 : kIpt], rank[kIpt];
#pragma unroll
  for (int i = 0; i < kIpt; ++i) {
    uint32_t idx = warp_base + i * 32 + lane;
    if (idx < n) {
      key[i] = in_k[idx];
      if constexpr (!kEarlyReorder) val[i] = in_v[idx];
    } else {
      key[i] = 0xffffffffu;  // ranks after every real key of digit 255
      if constexpr (!kEarlyReorder) val[i] = 0;
    }
  }
  // Stable per-warp ranking: items are visited in position order
  // (i outer, lane inner); the lanes holding the same digit are the AND of
  // one ballot per digit bit (or its complement), a fixed 8 votes whatever
  // the number of distinct digits in the warp.
  uint32_t *wh = s_warp_hist[warp];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int i = 0; i < kIpt; ++i) {
    uint32_t d = (key[i] >> shift) & 255u;
    uint32_t peers = 0xffffffffu;
#pragma unroll
    for (int bit = 0; bit < 8; ++bit) {
      const bool set = (d >> bit) & 1u;
      const uint32_t bal = __ballot_sync(0xffffffffu, set);
      peers &= set ? bal : ~bal;
    }
    uint32_t before = wh[d];
    rank[i] = before + __popc(peers & lt);
    __syncwarp();
    if (lane == (uint32_t)(__ffs(peers) - 1)) wh[d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();

  // Per digit: exclusive prefix over warps, block count, publish, look back.
  const uint32_t d = threadIdx.x;
  uint32_t block_count = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    uint32_t c = s_warp_hist[w][d];
    s_warp_hist[w][d] = block_count;
    block_count += c;
  }
  uint32_t *my_status = &status[(size_t)tile * 256];
  st_relaxed_u32(&my_status[d], (tile == 0 ? kFlagP : kFlagA) | block_count);
  uint32_t total;
  s_block_start[d] = block_exclusive_scan(block_count, sm.wsum, total);
  if constexpr (kEarlyReorder) {
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kIpt; ++i) {
      uint32_t idx = warp_base + i * 32 + lane;
      uint32_t dg = (key[i] >> shift) & 255u;
      uint32_t pos = s_block_start[dg] + s_warp_hist[warp][dg] + rank[i];
      s_keys[pos] = key[i];
      s_vals[pos] = idx < n ? in_v[idx] : 0u;
    }
  }

  // Look back over the predecessor tiles, kLookback status words per step:
  // add aggregates until the nearest inclusive prefix; restart a step when
  // one of the words it needs is not published yet.
  uint32_t exclusive = 0;
  if (tile > 0) {
    int32_t t = (int32_t)tile - 1;
    uint32_t spins = 0;
    while (t >= 0) {
      uint32_t w[kLookback];
#pragma unroll
      for (int q = 0; q < kLookback; ++q)
        w[q] = (t - q >= 0) ? ld_relaxed_u32(&status[(size_t)(t - q) * 256 + d]) : kFlagP;
      bool found = false, stalled = false;
      uint32_t add = 0;
      int used = 0;
#pragma unroll
      for (int q = 0; q < kLookback; ++q) {
        if (found || stalled) continue;
        uint32_t flag = w[q] & ~kMask;
        if (flag == 0) {
          stalled = true;
          continue;
        }
        add += (t - q >= 0) ? (w[q] & kMask) : 0u;
        ++used;
        if (flag == kFlagP) found = true;
      }
      exclusive += add;
      t -= used;
      if (found) break;
      if (stalled) {
        if (++spins > kSpinLimit) {
          atomicOr(error, kErrLookbackTimeout);
          break;
        }
        __nanosleep(20);
      }
    }
    st_relaxed_u32(&my_status[d], kFlagP | (exclusive + block_count));
  }
  s_global[d] = plan->digit_offset[pass][d] + exclusive;
  __syncthreads();

  // Reorder the tile by digit in shared memory (small tiles).
  if constexpr (!kEarlyReorder) {
#pragma unroll
    for (int i = 0; i < kIpt; ++i) {
      uint32_t dg = (key[i] >> shift) & 255u;
      uint32_t pos = s_block_start[dg] + s_warp_hist[warp][dg] + rank[i];
      s_keys[pos] = key[i];
      s_vals[pos] = val[i];
    }
    __syncthreads();
  }
  // Each digit run lands contiguously in the output.
#pragma unroll 4
  for (uint32_t s = threadIdx.x; s < kTile; s += kThreads) {
    uint32_t k = s_keys[s];
    uint32_t dg = (k >> shift) & 255u;
    uint32_t g = s_global[dg] + (s - s_block_start[dg]);
    if (g < n) {
      out_k[g] = k;
      out_v[g] = s_vals[s];
    }
  }
}

// Persistent pass: a fixed grid of blocks takes tiles from an atomic ticket
// (so look-back only ever waits on tiles already taken by running blocks)
// until the item count, read on the device, is covered.
// kMinBlocks: resident blocks per SM the register allocation must allow.
// Sorts that leave L2 (tens of millions of keys and more) are latency bound
// on their memory traffic and gain from a fourth resident block, though it
// costs spills (64 registers); L2-resident sorts (a 1080p frame's 1.9 M tile
// pairs) are faster with three.
template <int kIpt, int kMinBlocks = (kIpt > 8 ? GSR_SORT_MIN_BLOCKS_LARGE : GSR_SORT_MIN_BLOCKS)>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
    pass_kernel(const SortPlan *__restrict__ plan, uint32_t pass, uint32_t shift, uint32_t *k0,
                uint32_t *v0, uint32_t *k1, uint32_t *v1, uint32_t *status, uint32_t *ticket,
                uint32_t *error) {
  __shared__ PassSmem<kIpt> sm;
  if (plan->skip[pass]) return;
  const uint32_t n = plan->n;
  const bool from0 = plan->src[pass] == 0;
  const uint32_t *in_k = from0 ? k0 : k1;
  const uint32_t *in_v = from0 ? v0 : v1;
  uint32_t *out_k = from0 ? k1 : k0;
  uint32_t *out_v = from0 ? v1 : v0;
  for (;;) {
    if (threadIdx.x == 0) sm.tile = atomicAdd(ticket, 1u);
    for (uint32_t k = threadIdx.x; k < kWarps * 256; k += kThreads) (&sm.warp_hist[0][0])[k] = 0;
    __syncthreads();
    const uint32_t tile = sm.tile;
    if ((uint64_t)tile * PassSmem<kIpt>::kTile >= n) break;
    pass_tile<kIpt>(plan, pass, shift, n, tile, in_k, in_v, out_k, out_v, status, error, sm);
    __syncthreads();  // shared memory is reused by the next tile
  }
}

// Keys per thread: 8 up to 2M keys, 16 above.
#ifndef GSR_SORT_IPT_LARGE
#define GSR_SORT_IPT_LARGE 16
#endif
constexpr int kIptLarge = GSR_SORT_IPT_LARGE;
static_assert(kIptLarge > 8, "the large tile must hold more keys per thread than the small one");
// Sorts sized for this many keys or more run the four-blocks-per-SM pass.
constexpr uint32_t kHugeSort = 1u << 24;
inline uint32_t ipt_for(uint32_t capacity) {
  return capacity <= (1u << 21) ? 8u : (uint32_t)kIptLarge;
}
inline uint32_t tiles_for(uint32_t capacity) {
  uint32_t tile = kThreads * ipt_for(capacity);
  return (capacity + tile - 1) / tile;
}

}  // namespace

// Scratch layout: [tickets: 64 words][hist: 4*256][status: passes*tiles*256].
// A workspace sized for `capacity` serves every sort of up to `capacity`
// items: smaller sorts may run 8 items per thread where a larger one runs 16,
// and so use more tiles, so the bound takes the 8-per-thread tile count.
uint64_t sort_work_words(uint32_t capacity, uint32_t passes) {
  const uint64_t max_tiles = ((uint64_t)capacity + kThreads * 8 - 1) / (kThreads * 8);
  return 64ull + 4ull * 256ull + (uint64_t)passes * max_tiles * 256ull;
}

namespace {
constexpr int kMaxDevices = 64;
int current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    dev = 0;
  }
  return dev;
}
// Resident pass blocks on the current device (the persistent grid), looked
// up once per device.
template <int kIpt, int kMinBlocks>
uint32_t resident_pass_blocks() {
  static std::atomic<uint32_t> cache[kMaxDevices];
  const int dev = current_device();
  uint32_t blocks = cache[dev].load(std::memory_order_relaxed);
  if (blocks == 0) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pass_kernel<kIpt, kMinBlocks>,
                                                  kThreads, 0);
    blocks = device_sm_count() * (uint32_t)std::max(per_sm, 1);
    cache[dev].store(blocks, std::memory_order_relaxed);
  }
  return blocks;
}
}  // namespace

uint32_t device_sm_count() {
  static std::atomic<uint32_t> cache[kMaxDevices];
  const int dev = current_device();
  uint32_t sms = cache[dev].load(std::memory_order_relaxed);
  if (sms == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
      cudaGetLastError();
      v = 1;
    }
    sms = (uint32_t)v;
    cache[dev].store(sms, std::memory_order_relaxed);
  }
  return sms;
}

void launch_sort(const SortBuffers &b, cudaStream_t stream) {
  const uint32_t tiles = tiles_for(b.capacity);
  const uint32_t ipt = ipt_for(b.capacity);
  uint32_t *tickets = b.work;
  uint32_t *hist = b.work + 64;
  uint32_t *status = b.work + 64 + 4 * 256;
  // tickets and histograms; the status words are zeroed by the plan kernel
  if (!b.scratch_zeroed) cudaMemsetAsync(b.work, 0, kSortScratchHeadWords * sizeof(uint32_t), stream);
  const uint32_t grid = tiles ? tiles : 1;
  if (!b.hist) {
    if (ipt == 8)
      hist_kernel<8><<<grid, kThreads, 0, stream>>>(b.keys0, b.count, b.begin_bit, b.passes, hist);
    else
      hist_kernel<kIptLarge>
          <<<grid, kThreads, 0, stream>>>(b.keys0, b.count, b.begin_bit, b.passes, hist);
  }
  const uint32_t zero_blocks = std::min<uint32_t>(grid, 2 * device_sm_count());
  plan_kernel<<<zero_blocks, kThreads, 0, stream>>>(b.count, b.hist ? b.hist : hist, b.passes,
                                                    b.plan, status, tiles, kThreads * ipt);
  for (uint32_t p = 0; p < b.passes; ++p) {
    uint32_t *st = status + (size_t)p * tiles * 256;
    constexpr int kSmall = GSR_SORT_MIN_BLOCKS, kLarge = GSR_SORT_MIN_BLOCKS_LARGE;
    if (ipt == 8) {
      const uint32_t g = std::min(grid, resident_pass_blocks<8, kSmall>());
      pass_kernel<8, kSmall><<<g, kThreads, 0, stream>>>(b.plan, p, b.begin_bit + 8 * p, b.keys0,
                                                         b.vals0, b.keys1, b.vals1, st,
                                                         tickets + p, b.error);
    } else if (b.capacity < kHugeSort) {
      const uint32_t g = std::min(grid, resident_pass_blocks<kIptLarge, kLarge>());
      pass_kernel<kIptLarge, kLarge><<<g, kThreads, 0, stream>>>(
          b.plan, p, b.begin_bit + 8 * p, b.keys0, b.vals0, b.keys1, b.vals1, st, tickets + p,
          b.error);
    } else {
      const uint32_t g = std::min(grid, resident_pass_blocks<kIptLarge, 4>());
      pass_kernel<kIptLarge, 4><<<g, kThreads, 0, stream>>>(b.plan, p, b.begin_bit + 8 * p,
                                                            b.keys0, b.vals0, b.keys1, b.vals1,
                                                            st, tickets + p, b.error);
    }
  }
}

}  // namespace gsr
