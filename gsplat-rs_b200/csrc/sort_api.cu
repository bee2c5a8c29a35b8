// Host-pointer wrappers of the onesweep sort. Each call stages the arrays in
// device memory, sorts ascending on inverted keys (so keys descend) with the
// stable radix sort, and copies the permutation back.

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "device_types.h"
#include "kernels.h"
#include "renderer.h"
#include "sort_api.h"

namespace gsr {
namespace {

#define GSR_CUDA_S(expr)                                                                  \
  do {                                                                                    \
    cudaError_t err__ = (expr);                                                           \
    if (err__ != cudaSuccess)                                                             \
      throw Error(Code::Internal, std::string("CUDA error: ") + cudaGetErrorString(err__) + \
                                      " (" #expr ")");                                    \
  } while (0)

constexpr uint64_t kMaxItems = (1u << 30) - 1;
inline uint64_t align256(uint64_t v) { return (v + 255) & ~uint64_t(255); }


__global__ void invert_copy_kernel(const uint32_t *src, uint32_t *dst, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i] = ~src[i];
}

struct SortScratch {
  DeviceBuffer mem;
  uint32_t *k[2], *v[2], *count, *error, *work;
  SortPlan *plan;
  SortScratch(uint32_t n) {
    const uint64_t words = sort_work_words(n, 4);
    uint64_t off = 0, o[8];
    for (int i = 0; i < 4; ++i) { o[i] = off; off += align256(4ull * n); }
    o[4] = off; off += align256(sizeof(SortPlan));
    o[5] = off; off += 256;
    o[6] = off; off += align256(4 * words);
    mem.reset(off);
    k[0] = mem.as<uint32_t>(o[0]); v[0] = mem.as<uint32_t>(o[1]);
    k[1] = mem.as<uint32_t>(o[2]); v[1] = mem.as<uint32_t>(o[3]);
    plan = mem.as<SortPlan>(o[4]);
    count = mem.as<uint32_t>(o[5]);
    error = count + 1;
    work = mem.as<uint32_t>(o[6]);
  }
};

// Sorts (k[src], v[src]) ascending; returns the buffer index of the result.
int run_sort(SortScratch &s, int src, uint32_t n, cudaStream_t st) {
  SortBuffers b{s.k[src], s.v[src], s.k[1 - src], s.v[1 - src], s.count, n, 0, 4, s.plan,
                s.work, s.error, nullptr};
  launch_sort(b, st);
  SortPlan plan;
  uint32_t err = 0;
  GSR_CUDA_S(cudaMemcpyAsync(&plan, s.plan, sizeof(plan), cudaMemcpyDeviceToHost, st));
  GSR_CUDA_S(cudaMemcpyAsync(&err, s.error, 4, cudaMemcpyDeviceToHost, st));
  GSR_CUDA_S(cudaStreamSynchronize(st));
  GSR_CUDA_S(cudaGetLastError());
  if (err) throw Error(Code::Internal, "device wait limit reached in the radix sort look-back");
  return plan.final_buffer == 0 ? src : 1 - src;
}

struct Stream {
  cudaStream_t s = nullptr;
  Stream() { GSR_CUDA_S(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
  ~Stream() { if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); } }
};

}  // namespace

void require_device() {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    throw Error(Code::Unsupported, "no CUDA device");
  }
}

void sort_values_by_keys_host(const uint32_t *keys, uint32_t *values, uint64_t n) {
  if (n <= 1) return;
  if (n > kMaxItems) throw Error(Code::Unsupported, "sort length exceeds 2^30 - 1");
  require_device();
  Stream st;
  SortScratch s((uint32_t)n);
  uint32_t n32 = (uint32_t)n;
  GSR_CUDA_S(cudaMemcpyAsync(s.k[1], keys, 4 * n, cudaMemcpyHostToDevice, st.s));
  GSR_CUDA_S(cudaMemcpyAsync(s.v[0], values, 4 * n, cudaMemcpyHostToDevice, st.s));
  GSR_CUDA_S(cudaMemcpyAsync(s.count, &n32, 4, cudaMemcpyHostToDevice, st.s));
  GSR_CUDA_S(cudaMemsetAsync(s.error, 0, 4, st.s));
  invert_copy_kernel<<<std::min<uint32_t>((n32 + 255) / 256, 8 * device_sm_count()), 256, 0, st.s>>>(s.k[1], s.k[0], n32);
  int fin = run_sort(s, 0, n32, st.s);
  GSR_CUDA_S(cudaMemcpy(values, s.v[fin], 4 * n, cudaMemcpyDeviceToHost));
}

void sort_pairs_host(uint32_t *keys, uint32_t *values, uint64_t n) {
  if (n <= 1) return;
  if (n > kMaxItems) throw Error(Code::Unsupported, "sort length exceeds 2^30 - 1");
  require_device();
  Stream st;
  SortScratch s((uint32_t)n);
  uint32_t n32 = (uint32_t)n;
  // Pass 1: order by value ascending, carrying the keys.
  GSR_CUDA_S(cudaMemcpyAsync(s.k[0], values, 4 * n, cudaMemcpyHostToDevice, st.s));
  GSR_CUDA_S(cudaMemcpyAsync(s.v[0], keys, 4 * n, cudaMemcpyHostToDevice, st.s));
  GSR_CUDA_S(cudaMemcpyAsync(s.count, &n32, 4, cudaMemcpyHostToDevice, st.s));
  GSR_CUDA_S(cudaMemsetAsync(s.error, 0, 4, st.s));
  int a = run_sort(s, 0, n32, st.s);
  // Pass 2: stable order by inverted key, carrying the values.
  int b = 1 - a;
  const unsigned grid = std::min<uint32_t>((n32 + 255) / 256, 8 * device_sm_count());
  invert_copy_kernel<<<grid, 256, 0, st.s>>>(s.v[a], s.k[b], n32);
  GSR_CUDA_S(cudaMemcpyAsync(s.v[b], s.k[a], 4 * n, cudaMemcpyDeviceToDevice, st.s));
  int fin = run_sort(s, b, n32, st.s);
  std::vector<uint32_t> inv(n);
  GSR_CUDA_S(cudaMemcpy(inv.data(), s.k[fin], 4 * n, cudaMemcpyDeviceToHost));
  GSR_CUDA_S(cudaMemcpy(values, s.v[fin], 4 * n, cudaMemcpyDeviceToHost));
  for (uint64_t i = 0; i < n; ++i) keys[i] = ~inv[i];
}

void device_info(char *name, uint64_t name_capacity, int32_t *sm_count, int32_t *cc_major,
                 int32_t *cc_minor) {
  require_device();
  int dev = 0;
  GSR_CUDA_S(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  GSR_CUDA_S(cudaGetDeviceProperties(&prop, dev));
  if (name && name_capacity) {
    std::strncpy(name, prop.name, name_capacity - 1);
    name[name_capacity - 1] = '\0';
  }
  if (sm_count) *sm_count = prop.multiProcessorCount;
  if (cc_major) *cc_major = prop.major;
  if (cc_minor) *cc_minor = prop.minor;
}

}  // namespace gsr
