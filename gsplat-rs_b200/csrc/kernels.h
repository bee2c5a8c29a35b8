// Launch interface of the CUDA kernels (host-callable, plain pointers).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_types.h"
#include "gsr_host.h"

namespace gsr {

struct SceneDev;
struct ViewDev;
struct ViewSetDev;
struct ViewCounters;
struct Record;
struct ProjectedDev;
struct FrameCounters;
struct SortPlan;

// ---- K1: preprocess -------------------------------------------------------
// Splats are indexed by gid = views[v].splat_base + i across all views.
struct K1Buffers {
  uint32_t *vis_keys;          // [total splats] ~depth bits of visible splats, compacted
  uint32_t *vis_ids;           // [total splats] their gids, view-major then ascending id
  uint2 *rects;                // [gid] tile rect per visible splat ((0, 0): none)
  Record *records;             // [gid] raster record per drawn splat
  unsigned long long *status;  // [total blocks] look-back words, zeroed
  FrameCounters *counters;
  uint32_t *key_hist;          // [4][256] digit histograms of the depth keys, zeroed
  ViewCounters *view_counters; // [views], zeroed
  ProjectedDev *projected;     // [gid] debug tap, or null
  // Reuse of the last sorted order: project and count as usual, but write no
  // keys, ids or histograms, and clear the rects of splats not visible now.
  bool reuse_order;
};
uint32_t preprocess_blocks(uint32_t splats);  // blocks one view set of `splats` splats needs
// One block per 256 splats of each view set (views of one scene handled
// together); total_blocks = sum over sets of preprocess_blocks(scene splats).
void launch_preprocess(const ViewDev *views, const ViewSetDev *sets, uint32_t num_sets,
                       uint32_t total_blocks, uint32_t max_planes, const K1Buffers &b, bool debug,
                       cudaStream_t stream);

// ---- K3: onesweep LSD radix sort of (u32 key, u32 value) pairs -----------
// Sorts ascending and stably over bits [begin_bit, begin_bit + 8*passes) of
// the key. The item count is read from device memory (*count), the grids are
// sized from `capacity`. The result ends in (keys0, vals0) or (keys1, vals1)
// as plan->final_buffer says.
struct SortBuffers {
  uint32_t *keys0, *vals0, *keys1, *vals1;
  const uint32_t *count;
  uint32_t capacity;
  uint32_t begin_bit;
  uint32_t passes;  // 1..4
  SortPlan *plan;
  uint32_t *work;   // sort_work_words(capacity, passes) words of scratch
  uint32_t *error;
  // Digit histograms [passes][256] already accumulated by the producer of
  // the keys (then no histogram kernel runs), or null.
  const uint32_t *hist;
  // The scratch's tickets and histograms are already zero (else one memset).
  bool scratch_zeroed = false;
};
constexpr uint32_t kSortScratchHeadWords = 64 + 4 * 256;  // tickets and histograms
uint64_t sort_work_words(uint32_t capacity, uint32_t passes);
// Zeroes the scratch (one memset) and launches the histogram (unless given),
// plan and pass kernels on `stream`.
void launch_sort(const SortBuffers &b, cudaStream_t stream);

// ---- K2: tile-pair emission over the depth-sorted visible ids ------------
struct EmitBuffers {
  const SortPlan *depth_plan;      // selects the buffer holding the sorted ids; n = their count
  const uint32_t *ids0, *ids1;     // depth-sorted gids, [visible]
  const uint2 *rects;              // [gid] tile rects
  const Record *records;           // [gid] raster records (row spans)
  uint32_t *tile_keys, *tile_vals; // [capacity] output pairs (global tile id, gid)
  uint64_t capacity;
  unsigned long long *status;      // [emit_blocks(n)] look-back words, zeroed
  FrameCounters *counters;
  uint32_t *tile_hist;             // [passes][256] digit histograms of the tile ids, zeroed
  uint32_t tile_passes;
  uint32_t n;                      // total splats over the views (upper bound of visible)
  const ViewDev *views;
  uint32_t num_views;              // at most kMaxViewsPerLaunch
  uint32_t tile;                   // tile size in pixels (8 or 16)
};
constexpr uint32_t kMaxViewsPerLaunch = 1024;
uint64_t emit_blocks(uint64_t ids);              // emission blocks (look-back words) for n ids
uint64_t emit_status_words(uint64_t capacity);   // look-back words any n <= capacity needs
void launch_emit(const EmitBuffers &b, cudaStream_t stream);

// ---- tile ranges from the tile-sorted keys -------------------------------
// Also writes each view's pair count (view_counters[v].pairs).
void launch_ranges(const SortPlan *tile_plan, const uint32_t *keys0, const uint32_t *keys1,
                   const FrameCounters *counters, uint32_t capacity, uint2 *ranges,
                   const ViewDev *views, uint32_t num_views, ViewCounters *view_counters,
                   cudaStream_t stream);

// ---- K4: tile raster ------------------------------------------------------
// images holds every view's RGBA8 pixels at views[v].image_base.
struct RasterArgs {
  const ViewDev *views;
  uint32_t num_views;
  uint32_t total_tiles;            // global tiles over the views
  const uint2 *ranges;             // [total_tiles] list ranges
  const SortPlan *plan;            // selects the buffer holding the sorted ids
  const uint32_t *ids0, *ids1;
  const Record *records;
  uint32_t *images;
  FrameCounters *counters;         // raster_ticket is the persistent tile queue
  uint32_t *sticky;
  float2 *debug_cov = nullptr;     // debug tap: (log2 alpha, coverage bound) per splat slot
};
// Raster launch shape: records staged per step (tile 16: 64/128/256; tile 8:
// 32/64) and persistent blocks per SM pulling tiles from a global queue
// (0 = one block per tile). The FP32 mode honours both; UNORM8 parity mode
// always runs one block per tile with full-tile chunks. No setting changes a
// pixel.
struct RasterConfig {
  uint32_t chunk = 256;
  uint32_t blocks_per_sm = 0;
  bool operator==(const RasterConfig &o) const {
    return chunk == o.chunk && blocks_per_sm == o.blocks_per_sm;
  }
};
bool raster_config_valid(uint32_t tile, const RasterConfig &cfg);
void launch_raster(const RasterArgs &a, uint32_t tile, uint32_t blend_mode,
                   const RasterConfig &cfg, uint32_t sm_count, cudaStream_t stream);

// ---- run start ------------------------------------------------------------
// One kernel zeroes a run's scratch (in place of memsets: a plain frame then
// issues no copy-engine work, so a caller's own host<->device copies never
// queue in front of it).
constexpr int kRunZeroRegions = 5;
// Runs of up to kRunInlineViews views carry their view table in the
// zeroing kernel's parameters, which writes it to the device table: no
// host-to-device copy precedes the run (a replayed graph gets the new table
// by a parameter update of that one kernel node).
constexpr uint32_t kRunInlineViews = 8;
struct RunInit {
  uint32_t *zero[kRunZeroRegions];       // regions zeroed at the start of a run
  uint64_t zero_words[kRunZeroRegions];
  uint32_t inline_views = 0;  // 0: the table was copied to the device beforehand
  uint32_t inline_sets = 0;
  ViewSetDev *sets_dst = nullptr;
  ViewDev *views_dst = nullptr;
  ViewSetDev sets[kRunInlineViews];
  ViewDev views[kRunInlineViews];
};
void launch_run_init(const RunInit &a, cudaStream_t stream);
// The zeroing kernel's entry, to find its node in a captured graph.
const void *run_init_kernel_entry();

// ---- small helpers ----------------------------------------------------------
// Streaming multiprocessors of the current device (looked up once per
// device); grid-stride kernels cap their grids at a few blocks per SM.
uint32_t device_sm_count();
void launch_fill_u32(uint32_t *dst, uint32_t value, uint64_t count, cudaStream_t stream);

}  // namespace gsr
