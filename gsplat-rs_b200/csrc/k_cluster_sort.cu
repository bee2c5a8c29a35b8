// K3a for frames of up to 294,912 splats: the depth-order sort in one launch
// of one 16-CTA thread-block cluster, every pass in distributed shared
// memory.
//
// The same stable ascending LSD radix sort over the 32-bit depth keys as the
// onesweep sort (k_sort.cu), 8-bit digits, four passes: only the scheduling
// differs. A frame's visible keys (279,044 at the 1080p workload, 2.2 MB of
// keys and ids) are far too few to fill the GPU, so the onesweep sort's time
// is latency: five launches and a decoupled look-back per pass. Here the
// cluster's 16 CTAs hold the whole sequence, 18,432 positions each (1,024
// threads x 18 keys in registers), and one pass is:
//   1. rank: each warp ranks its 576 keys stably per digit (8 ballots per
//      key, as in the onesweep sort), each CTA forms its digit counts and its
//      warps' digit prefixes;
//   2. cluster barrier; every CTA reads all 16 CTAs' digit counts from their
//      shared memory and forms its global digit offsets (earlier digits of
//      every CTA, the same digit of earlier CTAs);
//   3. scatter: each key and id is stored straight into the shared memory of
//      the CTA that owns its destination position;
//   4. cluster barrier; each thread reloads its positions.
// A pass whose keys all share one digit is skipped by every CTA alike. The
// position order (CTA, warp, key slot, lane) is the sequence order, so
// every pass is stable and the result equals the onesweep sort's, id for id.
// No global scratch, no spin-wait: the only waits are the hardware cluster
// barriers, which every CTA reaches the same number of times.

#include <cooperative_groups.h>

#include <atomic>

#include "device_common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace gsr {
namespace {

constexpr int kCsCtas = 16;
constexpr int kCsThreads = 1024;
constexpr int kCsWarps = kCsThreads / 32;
constexpr int kCsIpt = 18;
constexpr uint32_t kCsSegment = 32 * kCsIpt;             // positions per warp
constexpr uint32_t kCsPerCta = kCsThreads * kCsIpt;      // 18,432
static_assert(kCsPerCta * kCsCtas == kClusterSortMaxItems, "cluster sort capacity");

struct ClusterSortSmem {
  uint32_t recv_keys[kCsPerCta];       // this CTA's positions, written by every CTA's scatter
  uint32_t recv_vals[kCsPerCta];
  uint16_t rank[kCsIpt][kCsThreads];   // warp-local rank of each key slot
  uint32_t warp_hist[kCsWarps][256];   // digit counts, then exclusive prefixes over warps
  uint32_t cta_hist[256];              // this CTA's digit counts, read by the whole cluster
  uint32_t digit_start[256];           // global position of this CTA's first key per digit
  uint32_t wsum[8];
  uint32_t trivial;
};

__device__ __forceinline__ uint32_t cluster_addr(const void *local, uint32_t cta) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_addr(local)), "r"(cta));
  return r;
}
__device__ __forceinline__ void st_cluster_u32(uint32_t addr, uint32_t v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_cluster_u32(uint32_t addr) {
  uint32_t v;
  asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
  return v;
}

__global__ void __launch_bounds__(kCsThreads, 1)
    cluster_sort_kernel(const uint32_t *__restrict__ count, const uint32_t *__restrict__ in_k,
                        const uint32_t *__restrict__ in_v, uint32_t *__restrict__ out_k,
                        uint32_t *__restrict__ out_v, SortPlan *__restrict__ plan) {
  extern __shared__ __align__(16) unsigned char cs_dyn[];
  ClusterSortSmem &sm = *reinterpret_cast<ClusterSortSmem *>(cs_dyn);
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t cta = cluster.block_rank();
  // The host takes this path only when the run's splat count (an upper
  // bound of the visible count) fits; the clamp keeps every access in bounds
  // whatever the count says.
  const uint32_t n = min(*count, kClusterSortMaxItems);
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t lt = lanemask_lt();
  const uint32_t seg = warp * kCsSegment;
  const uint32_t first = cta * kCsPerCta;

  uint32_t key[kCsIpt], val[kCsIpt];
#pragma unroll
  for (int i = 0; i < kCsIpt; ++i) {
    const uint32_t pos = first + seg + i * 32 + lane;
    key[i] = pos < n ? in_k[pos] : 0u;
    val[i] = pos < n ? in_v[pos] : 0u;
  }

  for (uint32_t pass = 0; pass < 4; ++pass) {
    const uint32_t shift = 8 * pass;
    uint32_t *wh = sm.warp_hist[warp];
#pragma unroll
    for (int k = 0; k < 8; ++k) wh[lane + 32 * k] = 0u;
    __syncwarp();
    // 1. Stable ranking within the warp's segment, in position order
    //    (slot outer, lane inner); positions at or beyond n are not keys.
#pragma unroll
    for (int i = 0; i < kCsIpt; ++i) {
      const bool valid = first + seg + i * 32 + lane < n;
      const uint32_t d = (key[i] >> shift) & 255u;
      uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
      for (int bit = 0; bit < 8; ++bit) {
        const bool set = (d >> bit) & 1u;
        const uint32_t bal = __ballot_sync(0xffffffffu, set);
        peers &= set ? bal : ~bal;
      }
      const uint32_t before = wh[d];
      if (valid) sm.rank[i][tid] = (uint16_t)(before + __popc(peers & lt));
      __syncwarp();
      if (valid && lane == (uint32_t)(__ffs(peers) - 1)) wh[d] = before + __popc(peers);
      __syncwarp();
    }
    __syncthreads();
    if (tid < 256) {
      uint32_t running = 0;
#pragma unroll 8
      for (int w = 0; w < kCsWarps; ++w) {
        const uint32_t c = sm.warp_hist[w][tid];
        sm.warp_hist[w][tid] = running;
        running += c;
      }
      sm.cta_hist[tid] = running;
      if (tid == 0) sm.trivial = 0;
    }
    // 2. Every CTA's digit counts are complete and visible cluster-wide.
    cluster.sync();
    if (tid < 256) {
      const uint32_t d = tid;
      uint32_t total = 0, before = 0;
#pragma unroll
      for (uint32_t c = 0; c < (uint32_t)kCsCtas; ++c) {
        const uint32_t h = ld_cluster_u32(cluster_addr(&sm.cta_hist[d], c));
        total += h;
        before += c < cta ? h : 0u;
      }
      if (total == n) sm.trivial = 1;  // every key has this digit: nothing moves
      // exclusive scan of the digit totals over the 256 digits (warps 0..7)
      uint32_t inc = total;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += t;
      }
      if (lane == 31) sm.wsum[warp] = inc;
      asm volatile("bar.sync 1, 256;" ::: "memory");  // the 256 digit threads only
      uint32_t below = 0;
#pragma unroll
      for (int w = 0; w < 8; ++w) below += w < (int)warp ? sm.wsum[w] : 0u;
      sm.digit_start[d] = below + inc - total + before;
    }
    __syncthreads();
    const bool trivial = sm.trivial != 0;  // the same in every CTA (cluster-wide totals)
    if (!trivial) {
      // 3. Scatter into the owners' shared memory.
      const uint32_t rk = smem_addr(sm.recv_keys), rv = smem_addr(sm.recv_vals);
      (void)rk;
      (void)rv;
#pragma unroll
      for (int i = 0; i < kCsIpt; ++i) {
        if (first + seg + i * 32 + lane < n) {
          const uint32_t d = (key[i] >> shift) & 255u;
          const uint32_t pos = sm.digit_start[d] + sm.warp_hist[warp][d] + sm.rank[i][tid];
          const uint32_t owner = pos / kCsPerCta, off = pos - owner * kCsPerCta;
          st_cluster_u32(cluster_addr(&sm.recv_keys[off], owner), key[i]);
          st_cluster_u32(cluster_addr(&sm.recv_vals[off], owner), val[i]);
        }
      }
    }
    // 4. All stores have landed (and every CTA is done reading the digit
    //    counts, which the next pass rewrites).
    cluster.sync();
    if (!trivial) {
#pragma unroll
      for (int i = 0; i < kCsIpt; ++i) {
        const uint32_t local = seg + i * 32 + lane;
        if (first + local < n) {
          key[i] = sm.recv_keys[local];
          val[i] = sm.recv_vals[local];
        }
      }
      __syncthreads();  // the next pass's scatter may target this CTA again
    }
  }
  // The next pass's scatter above is ordered after every CTA's reload by the
  // next pass's first cluster barrier; after the last pass the sorted
  // sequence is in registers, in position order.
#pragma unroll
  for (int i = 0; i < kCsIpt; ++i) {
    const uint32_t pos = first + seg + i * 32 + lane;
    if (pos < n) {
      out_k[pos] = key[i];
      out_v[pos] = val[i];
    }
  }
  if (cta == 0 && tid == 0) {
    plan->n = n;
    plan->passes = 4;
    plan->final_buffer = 1;
    for (int p = 0; p < 8; ++p) {
      plan->skip[p] = p < 4 ? 0u : 1u;
      plan->src[p] = 0u;
    }
  }
}

struct ClusterSortState {
  std::atomic<int> ready{0};  // 0 unknown, 1 usable, -1 not usable
};
ClusterSortState g_cluster_state[64];

cudaLaunchConfig_t make_config(cudaLaunchAttribute *attr, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kCsCtas, 1, 1);
  cfg.blockDim = dim3(kCsThreads, 1, 1);
  cfg.dynamicSmemBytes = sizeof(ClusterSortSmem);
  cfg.stream = stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kCsCtas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

}  // namespace

// Whether the current device can run one 16-CTA cluster of the sort (a
// non-portable cluster size, opted into here; the occupancy query answers
// whether 16 such CTAs can be co-resident). Looked up once per device.
bool cluster_sort_available() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return false;
  }
  int state = g_cluster_state[dev].ready.load(std::memory_order_relaxed);
  if (state == 0) {
    state = -1;
    if (cudaFuncSetAttribute(cluster_sort_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed,
                             1) == cudaSuccess &&
        cudaFuncSetAttribute(cluster_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(ClusterSortSmem)) == cudaSuccess) {
      cudaLaunchAttribute attr[1];
      cudaLaunchConfig_t cfg = make_config(attr, nullptr);
      int clusters = 0;
      if (cudaOccupancyMaxActiveClusters(&clusters, cluster_sort_kernel, &cfg) == cudaSuccess &&
          clusters >= 1)
        state = 1;
    }
    cudaGetLastError();
    g_cluster_state[dev].ready.store(state, std::memory_order_relaxed);
  }
  return state == 1;
}

void launch_cluster_sort(const uint32_t *count, const uint32_t *keys0, const uint32_t *vals0,
                         uint32_t *keys1, uint32_t *vals1, SortPlan *plan, cudaStream_t stream) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = make_config(attr, stream);
  cudaLaunchKernelEx(&cfg, cluster_sort_kernel, count, keys0, vals0, keys1, vals1, plan);
}

}  // namespace gsr
