// Standalone GPU sort entry points (host-pointer API) and device queries.
#pragma once

#include <cstdint>

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

}  // namespace gsr
