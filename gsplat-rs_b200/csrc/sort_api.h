// Standalone GPU sort entry points (host-pointer API) and device queries.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "gsr_host.h"

namespace gsr {

// CpuSortBackend::sort_values_by_keys semantics
// (crates/gsplat-sort/src/lib.rs:36-61): values permuted so keys descend,
// equal keys keep input order.
void sort_values_by_keys_host(const uint32_t *keys, uint32_t *values, uint64_t n);
// CpuSortBackend::sort_pairs semantics (lib.rs:81-101): keys descending,
// equal keys by ascending value; both permuted.
void sort_pairs_host(uint32_t *keys, uint32_t *values, uint64_t n);

void device_info(char *name, uint64_t name_capacity, int32_t *sm_count, int32_t *cc_major,
                 int32_t *cc_minor);
// Throws Error(Unsupported) when no CUDA device is present.
void require_device();
// FP32 FMA throughput of the current device (probe.cu): the best of five
// timed launches of an FMA-only kernel, in TFLOP/s, and that launch's time.
void measure_fp32_peak(double *tflops, double *best_ms);

// The same sort on caller-owned device buffers, with all scratch in a static
// device array (sort_noalloc.cu); never allocates. Returns Ok or an error code
// with `msg` set.
Code sort_values_by_keys_noalloc(const uint32_t *keys, uint32_t *values, uint64_t n,
                                 cudaStream_t stream, std::string &msg);
uint64_t noalloc_scratch_bytes();
uint32_t noalloc_max_items();

}  // namespace gsr
