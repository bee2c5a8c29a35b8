// gsplat_cuda_sort_values_by_keys_noalloc: the depth-order sort for callers
// that must not allocate device memory.
//
// Who needs it: hosts that own every byte of GPU memory through their own
// pool or arena (game engines, compositors, plugins inside a larger
// renderer) and do not allow a library to call cudaMalloc behind their back,
// and latency-critical threads where cudaMalloc/cudaFree are off limits
// because they can synchronise the whole device and take unbounded time.
// Such callers hand over device buffers they already own; everything else
// the sort needs lives in one statically sized device array defined below.
//
// The array is a file-scope __device__ variable: every GPU that loads this
// library holds it (kNoAllocBytes, about 14.7 MB) until the process exits.
// Host code cannot use the symbol as a pointer, so the first call on each
// device looks its address up once with cudaGetSymbolAddress (with that
// device current) and caches it; make that first call before any stream
// capture begins on the device. All calls share the array and it keeps the
// previous call's contents, so every call zeroes the parts that must start at
// zero. Two calls running on the GPU at the same time would race on it; this
// entry point prevents that inside one process by holding a process-wide
// lock and waiting for its stream before it returns. Because it waits for
// its stream, it refuses a stream that is being captured.

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/gsplat_cuda.h"
#include "device_types.h"
#include "kernels.h"
#include "sort_api.h"

namespace gsr {
namespace {

constexpr uint32_t kNoAllocMaxItems = 1u << 20;
inline constexpr uint64_t align256(uint64_t v) { return (v + 255) & ~uint64_t(255); }

// Layout: inverted keys | alternate keys | alternate values | plan | count,
// error | sort work words (tickets, histograms, look-back status).
constexpr uint64_t kOffKeys0 = 0;
constexpr uint64_t kOffKeys1 = kOffKeys0 + align256(4ull * kNoAllocMaxItems);
constexpr uint64_t kOffVals1 = kOffKeys1 + align256(4ull * kNoAllocMaxItems);
constexpr uint64_t kOffPlan = kOffVals1 + align256(4ull * kNoAllocMaxItems);
constexpr uint64_t kOffCount = kOffPlan + align256(sizeof(SortPlan));
constexpr uint64_t kOffWork = kOffCount + 256;
// Work words for 8-key-per-thread tiles (2048 keys) and 4 passes.
constexpr uint64_t kWorkWords = 64ull + 4ull * 256ull + 4ull * ((kNoAllocMaxItems + 2047) / 2048) * 256ull;
constexpr uint64_t kNoAllocBytes = kOffWork + align256(4 * kWorkWords);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

__global__ void noalloc_prepare_kernel(const uint32_t *__restrict__ keys, uint32_t *__restrict__ inv,
                                       uint32_t *__restrict__ count_error, uint32_t n) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    count_error[0] = n;
    count_error[1] = 0;
  }
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    inv[i] = ~keys[i];
}

// Moves the sorted values into the caller's buffer when the last pass left
// them in the alternate buffer.
__global__ void noalloc_finish_kernel(const SortPlan *__restrict__ plan,
                                      const uint32_t *__restrict__ alt, uint32_t *__restrict__ values,
                                      uint32_t n) {
  if (plan->final_buffer == 0) return;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    values[i] = alt[i];
}

std::mutex g_noalloc_mutex;
constexpr int kMaxDevices = 64;
unsigned char *g_noalloc_ptr[kMaxDevices] = {};

Code fail_code(cudaError_t e, const char *what, std::string &msg) {
  msg = std::string(what) + ": " + cudaGetErrorString(e);
  return Code::Internal;
}

}  // namespace

Code sort_values_by_keys_noalloc(const uint32_t *keys, uint32_t *values, uint64_t n,
                                 cudaStream_t stream, std::string &msg) {
  if (n > kNoAllocMaxItems) {
    msg = "length " + std::to_string(n) + " exceeds the no-allocation limit of " +
          std::to_string(kNoAllocMaxItems) + " items";
    return Code::InvalidArgument;
  }
  if (n <= 1) return Code::Ok;
  if (!keys || !values) {
    msg = "keys and values must be device pointers";
    return Code::InvalidArgument;
  }
  // An error left pending by the caller's earlier work is reported as such
  // (and cleared), not blamed on the sort's own launches below.
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    msg = std::string("pending CUDA error before the sort: ") + cudaGetErrorString(e);
    return Code::Internal;
  }
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(stream, &capture);
  if (e != cudaSuccess) return fail_code(e, "cudaStreamIsCapturing", msg);
  if (capture != cudaStreamCaptureStatusNone) {
    msg = "the stream is being captured: this sort synchronises its stream before returning";
    return Code::InvalidArgument;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    msg = std::string("no CUDA device: ") + cudaGetErrorString(e);
    return Code::Unsupported;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    msg = "device ordinal out of range";
    return Code::Unsupported;
  }
  if (!g_noalloc_ptr[dev]) {
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return fail_code(e, "cudaGetSymbolAddress", msg);
    g_noalloc_ptr[dev] = static_cast<unsigned char *>(ptr);
  }
  unsigned char *base = g_noalloc_ptr[dev];
  uint32_t *k0 = reinterpret_cast<uint32_t *>(base + kOffKeys0);
  uint32_t *k1 = reinterpret_cast<uint32_t *>(base + kOffKeys1);
  uint32_t *v1 = reinterpret_cast<uint32_t *>(base + kOffVals1);
  SortPlan *plan = reinterpret_cast<SortPlan *>(base + kOffPlan);
  uint32_t *count_error = reinterpret_cast<uint32_t *>(base + kOffCount);
  uint32_t *work = reinterpret_cast<uint32_t *>(base + kOffWork);
  const uint32_t n32 = (uint32_t)n;
  const unsigned grid = std::min<uint32_t>((n32 + 255) / 256, 8 * device_sm_count());
  noalloc_prepare_kernel<<<grid, 256, 0, stream>>>(keys, k0, count_error, n32);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_code(e, "key preparation launch", msg);
  // launch_sort zeroes the tickets, histograms and look-back words itself.
  SortBuffers b{k0, values, k1, v1, count_error, n32, 0, 4, plan, work, count_error + 1, nullptr};
  launch_sort(b, stream);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_code(e, "radix sort launch", msg);
  noalloc_finish_kernel<<<grid, 256, 0, stream>>>(plan, v1, values, n32);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_code(e, "result copy launch", msg);
  uint32_t err = 0;
  e = cudaMemcpyAsync(&err, count_error + 1, 4, cudaMemcpyDeviceToHost, stream);
  if (e != cudaSuccess) return fail_code(e, "cudaMemcpyAsync", msg);
  e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail_code(e, "cudaStreamSynchronize", msg);
  if (err) {
    msg = "device wait limit reached in the radix sort look-back";
    return Code::Internal;
  }
  return Code::Ok;
}

uint64_t noalloc_scratch_bytes() { return kNoAllocBytes; }
uint32_t noalloc_max_items() { return kNoAllocMaxItems; }

}  // namespace gsr
