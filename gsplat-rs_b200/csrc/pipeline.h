// The frame pipeline over a list of views (a plain frame is one view):
// K1 -> depth sort -> K2 -> tile sort -> ranges -> K4 on one CUDA stream.
#pragma once

#include <atomic>

#include <cstdint>
#include <cuda_runtime.h>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "device_types.h"
#include "gsr_host.h"
#include "kernels.h"

namespace gsr {

// One device allocation, freed on destruction.
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  ~DeviceBuffer();
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  void reset(uint64_t bytes);  // frees, then allocates `bytes` (0 = free only)
  // The same in stream order on `stream` (cudaFreeAsync / cudaMallocAsync):
  // no host or device-wide wait, so a workspace can grow while other streams
  // run. The buffer must then only be used on `stream` (or after it), and
  // it is freed in stream order there when destroyed, so the stream must
  // outlive it.
  void reset(uint64_t bytes, cudaStream_t stream);
  void *get() const { return ptr_; }
  uint64_t size() const { return bytes_; }
  template <typename T>
  T *as(uint64_t byte_offset = 0) const {
    return reinterpret_cast<T *>(static_cast<char *>(ptr_) + byte_offset);
  }

 private:
  void release();
  void *ptr_ = nullptr;
  uint64_t bytes_ = 0;
  cudaStream_t stream_ = nullptr;  // set when allocated in stream order
  bool ordered_ = false;
};

// Scene resident in HBM (SoA float4 planes, see device_types.h SceneDev).
struct DeviceScene {
  DeviceBuffer mem;
  SceneDev dev{};
  uint32_t n = 0;
  uint32_t sh_degree = 0;
  std::vector<float> positions;  // host copy for automatic camera framing
  uint64_t bytes() const { return mem.size(); }
};
// A scene encoded in the packed resident format (packed.cpp): hot words and
// sidecar padded to whole 256-splat slices, and the header with its tables.
struct PackedHost {
  uint64_t n = 0;
  uint32_t sh_degree = 0;
  std::vector<uint32_t> hot;     // 5 words per slot
  std::vector<int8_t> sidecar;   // 48 bytes per slot (SH degree >= 1)
  std::vector<float> table;      // kPackedFloats
};
PackedHost pack_scene_packed(const HostScene &s);  // Unsupported above SH degree 3
uint64_t packed_device_bytes(uint64_t n, uint32_t sh_degree);
std::unique_ptr<DeviceScene> upload_scene_packed(const HostScene &s, cudaStream_t stream);

// Allocates the planes of an n-splat scene (Unsupported above 2^30 - 1 splats).
std::unique_ptr<DeviceScene> alloc_scene(uint64_t n, uint32_t sh_degree);
std::unique_ptr<DeviceScene> upload_scene(const HostScene &s, cudaStream_t stream);
// HBM bytes a scene's planes take.
uint64_t scene_device_bytes(uint64_t splats, uint32_t sh_degree);
uint64_t scene_device_bytes(const HostScene &s);
// Loads a PLY file into HBM: a binary body is decoded on the device
// (ply_device.cu), an ASCII one parsed on the host (load_ply) and uploaded.
// `admit(bytes)` runs with the scene's HBM size before any allocation (a
// budget check may throw). Same checks and error codes as load_ply; the
// planes equal upload_scene(load_ply(path)) bit for bit.
std::unique_ptr<DeviceScene> load_scene_file(const std::string &path, cudaStream_t stream,
                                             const std::function<void(uint64_t)> &admit);

// Device-timed phases of one run (CUDA events on the pipeline's stream).
enum Phase : int { kPhasePreprocess, kPhaseDepthSort, kPhaseEmit, kPhaseTileSort, kPhaseRanges,
                   kPhaseRaster, kPhaseCount };

struct ViewSpec {
  const DeviceScene *scene;
  GsplatCamera camera;
  uint32_t width, height;
};

struct RunResult {
  float phase_ms[kPhaseCount] = {};
  float preprocess_ms = 0, sort_ms = 0, raster_ms = 0, frame_ms = 0;
  uint64_t visible = 0, drawn = 0, keys = 0;
  uint32_t reruns = 0;
  bool sorted = true;  // false: the last sorted order was reused
};

// Pinned host destinations of a run's counters (default: the pipeline's own).
struct HostSinks {
  FrameCounters *counters = nullptr;
  ViewCounters *views = nullptr;  // one entry per view of the run
};

class Pipeline {
 public:
  Pipeline(int device, cudaStream_t stream);
  ~Pipeline();

  // Tile size 8 or 16; the raster chunk follows to the nearest valid size.
  void set_tile(uint32_t tile);
  uint32_t tile() const { return tile_; }
  void set_blend_mode(uint32_t mode) { blend_mode_ = mode; }
  uint32_t blend_mode() const { return blend_mode_; }
  void set_debug(bool on) { debug_ = on; }
  bool debug() const { return debug_; }
  void set_use_graph(bool on) { use_graph_ = on; }
  bool use_graph() const { return use_graph_; }
  // Asks the next runs to reuse the last sorted visible order instead of
  // sorting (honoured only for a layout identical to the one last sorted):
  // splats are projected with the new camera, but only those in the reused
  // order can be drawn, in its order.
  void set_reuse_order(bool on) { reuse_request_ = on; }
  bool last_reused_order() const { return last_reused_; }
  // Throws InvalidArgument unless valid for the current tile size.
  void set_raster_config(const RasterConfig &c);
  const RasterConfig &raster_config() const { return raster_cfg_; }

  // Renders `count` views into `images` (device, RGBA8 words) at the given
  // pixel offsets and waits. Grows the pair buffers and re-runs on overflow.
  RunResult run(const ViewSpec *views, uint32_t count, uint32_t *images,
                const uint64_t *image_bases);
  RunResult run(const std::vector<ViewSpec> &views, uint32_t *images,
                const std::vector<uint64_t> &image_bases) {
    return run(views.data(), (uint32_t)views.size(), images, image_bases.data());
  }
  // Enqueues without waiting (pair capacity as sized by earlier runs);
  // errors and overflow of enqueued runs surface at sync(), or in the
  // counters written to `sinks` once the stream reaches them.
  void enqueue(const ViewSpec *views, uint32_t count, uint32_t *images,
               const uint64_t *image_bases, HostSinks sinks = {});
  void enqueue(const std::vector<ViewSpec> &views, uint32_t *images,
               const std::vector<uint64_t> &image_bases, HostSinks sinks = {}) {
    enqueue(views.data(), (uint32_t)views.size(), images, image_bases.data(), sinks);
  }
  RunResult sync();
  // One batch of launch groups: group g renders views [first, first + count)
  // into `images` with host sinks `sinks`. With graphs on, the whole
  // sequence becomes one CUDA graph from the second time the same group
  // layouts are seen: every group's view table is a captured copy from a
  // pinned staging area that the host refills before each launch (the
  // previous launch having read it). Otherwise the groups are enqueued one
  // by one, as by enqueue().
  struct GroupRun {
    uint32_t first, count;
    HostSinks sinks;
  };
  void enqueue_groups(const ViewSpec *views, uint32_t *images, const uint64_t *image_bases,
                      const std::vector<GroupRun> &groups);
  uint64_t batch_graph_launches() const { return batch_graph_launches_; }
  // Grows the pair buffers to hold at least `pairs` tile pairs.
  void reserve_pairs(uint64_t pairs) { ensure_key_workspace(pairs); }

  uint64_t key_capacity() const { return key_cap_; }
  cudaStream_t stream() const { return stream_; }
  int device() const { return device_; }
  // Kernel launches of one run with the current settings (excluding copies
  // and memsets).
  uint32_t launches_per_run() const;
  const std::vector<ViewCounters> &view_counters() const { return view_counters_host_; }

  // Debug taps of the last run (valid until the next run).
  std::vector<uint32_t> debug_order();
  std::vector<ProjectedDev> debug_projected(uint32_t count);
  // (log2 alpha, coverage bound) the FP32 raster used per splat slot; NaN for
  // splats in no tile list (or frames in the UNORM8 mode).
  std::vector<float2> debug_coverage(uint32_t count);
  void debug_tile_pairs(std::vector<uint32_t> &tiles, std::vector<uint32_t> &ids);
  void debug_tile_ranges(uint32_t num_tiles, std::vector<uint32_t> &ranges,
                         std::vector<uint32_t> &ids);

 private:
  struct Layout {
    uint32_t views = 0, total_splats = 0, total_blocks = 0, total_tiles = 0, max_planes = 1;
    uint32_t tile_passes = 1, sets = 0;
    bool operator==(const Layout &o) const {
      return views == o.views && sets == o.sets && total_splats == o.total_splats &&
             total_blocks == o.total_blocks && total_tiles == o.total_tiles &&
             max_planes == o.max_planes && tile_passes == o.tile_passes;
    }
  };
  Layout plan_views(const ViewSpec *views, uint32_t count, const uint64_t *image_bases);
  void ensure_workspace(const Layout &l);
  void ensure_key_workspace(uint64_t capacity);
  void launch_all(const Layout &l, uint32_t *images, const HostSinks &sinks, bool reuse,
                  const ViewDev *views_dev, const ViewSetDev *sets_dev);
  void fetch_counters();  // device-resident counters of the last run -> host (stream synchronised)

 public:
  // Recorded, in the last enqueued run, just before its raster launch.
  cudaEvent_t raster_start_event() const { return ev_[kPhaseRaster]; }
  // Phase times of the last run enqueued without batch mode (its stream
  // must have reached the run's end).
  void phase_times(float out[kPhaseCount]) const;

 private:
  void collect(RunResult &r);
  SortPlan read_plan(int which);
  void drop_graph();
  // The zeroing kernel's parameters for a run of layout l (with the view
  // table inline when the layout is small enough).
  RunInit make_run_init(const Layout &l) const;

 public:
  // Launch graphs captured so far and the host milliseconds spent capturing
  // and instantiating them (readable from any thread).
  uint64_t graph_captures() const { return captures_.load(std::memory_order_relaxed); }
  double capture_ms() const { return capture_ms_.load(std::memory_order_relaxed); }
  // Workspace reallocations so far (each waits for the device to go idle:
  // cudaFree synchronises it) and the host milliseconds they took.
  uint64_t workspace_regrowths() const { return regrowths_.load(std::memory_order_relaxed); }
  double regrowth_ms() const { return regrowth_ms_.load(std::memory_order_relaxed); }
  void note_regrowth(double ms) {
    regrowths_.fetch_add(1, std::memory_order_relaxed);
    regrowth_ms_.store(regrowth_ms_.load(std::memory_order_relaxed) + ms,
                       std::memory_order_relaxed);
  }

 private:
  std::atomic<uint64_t> regrowths_{0};
  std::atomic<double> regrowth_ms_{0.0};
  std::atomic<uint64_t> captures_{0};
  std::atomic<double> capture_ms_{0.0};
  void record(int k);  // phase event k (a graph node while capturing)

  int device_;
  cudaStream_t stream_;
  cudaEvent_t ev_[kPhaseCount + 1] = {};
  uint32_t tile_ = 16, blend_mode_ = 0, sm_count_ = 148;
  RasterConfig raster_cfg_;
  bool debug_ = false, use_graph_ = true, has_run_ = false, capturing_ = false;
  bool reuse_request_ = false, last_reused_ = false, sorted_valid_ = false;
  Layout sorted_layout_;
  std::vector<const DeviceScene *> sorted_scenes_;  // scenes of the last sorted run
  Layout last_layout_;
  HostSinks last_sinks_;
  RunResult last_;
  std::vector<ViewDev> views_host_;
  std::vector<ViewSetDev> sets_host_;
  std::vector<ViewCounters> view_counters_host_;

  // Fixed-size scratch: counters, plans, histograms, sticky word; zeroed
  // region first (one memset per run).
  DeviceBuffer fixed_;
  FrameCounters *counters_ = nullptr;
  uint32_t *key_hist_ = nullptr, *tile_hist_ = nullptr, *sticky_ = nullptr;
  SortPlan *depth_plan_ = nullptr, *tile_plan_ = nullptr;
  FrameCounters *counters_host_ = nullptr;  // pinned
  // Per-layout scratch.
  DeviceBuffer view_ws_;  // view table + view counters + look-back words (zeroed part)
  uint64_t view_zero_bytes_ = 0;
  ViewDev *views_dev_ = nullptr;
  ViewSetDev *sets_dev_ = nullptr;
  ViewCounters *view_counters_ = nullptr;
  unsigned long long *k1_status_ = nullptr, *emit_status_ = nullptr;
  uint32_t view_cap_ = 0, splat_cap_ = 0, tile_cap_ = 0;
  DeviceBuffer splat_ws_;
  uint32_t *vis_keys0_ = nullptr, *vis_vals0_ = nullptr, *vis_keys1_ = nullptr,
           *vis_vals1_ = nullptr, *depth_sort_work_ = nullptr;
  uint2 *rects_ = nullptr;
  Record *records_ = nullptr;
  DeviceBuffer projected_;
  DeviceBuffer tile_ws_;
  uint2 *ranges_ = nullptr;
  DeviceBuffer key_ws_;
  uint64_t key_cap_ = 0;
  uint32_t *tile_keys0_ = nullptr, *tile_vals0_ = nullptr, *tile_keys1_ = nullptr,
           *tile_vals1_ = nullptr, *tile_sort_work_ = nullptr;
  DeviceBuffer debug_pairs_;
  DeviceBuffer debug_cov_;
  ViewCounters *view_counters_pinned_ = nullptr;
  uint32_t view_counters_pinned_cap_ = 0;
  // Pinned staging ring for the view table: slot s is rewritten only after
  // the copy that last read it has completed (slot_ev_[s]). A slot mirrors
  // the device table: the view sets (table_sets_bytes_) and then the views,
  // so one copy moves both.
  static constexpr int kViewSlots = 4;
  unsigned char *table_pinned_ = nullptr;
  uint64_t table_slot_bytes_ = 0;
  uint64_t table_sets_bytes_ = 0;
  cudaEvent_t slot_ev_[kViewSlots] = {};
  bool last_device_sinks_ = false;
  int slot_ = 0;
  // CUDA graphs of launch_all, one per layout, buffer set and setting.
  struct GraphKey {
    Layout layout;
    uint32_t *images;
    uint64_t key_cap;
    uint32_t tile, blend;
    bool debug;
    RasterConfig raster;
    FrameCounters *host_counters;
    ViewCounters *host_views;
    bool reuse;
    bool operator==(const GraphKey &o) const {
      return layout == o.layout && images == o.images && key_cap == o.key_cap &&
             tile == o.tile && blend == o.blend && debug == o.debug && raster == o.raster &&
             host_counters == o.host_counters && host_views == o.host_views &&
             reuse == o.reuse;
    }
  };
  struct GraphEntry {
    GraphKey key;
    cudaGraphExec_t exec;
    uint64_t last_use;
    cudaGraph_t graph;             // kept: its zeroing node takes parameter updates
    cudaGraphNode_t init_node;     // the zeroing kernel (null if not found)
    cudaKernelNodeParams init_params;
  };
  static constexpr size_t kGraphCacheSize = 64;
  std::vector<GraphEntry> graphs_;
  std::vector<GraphKey> seen_keys_;  // layouts launched once without a graph
  // Whole-batch graphs (enqueue_groups).
  struct BatchKey {
    std::vector<Layout> layouts;
    std::vector<FrameCounters *> counters;
    std::vector<ViewCounters *> views;
    uint32_t *images;
    uint64_t key_cap;
    uint32_t tile, blend;
    bool debug;
    RasterConfig raster;
    bool operator==(const BatchKey &o) const {
      return layouts == o.layouts && counters == o.counters && views == o.views &&
             images == o.images && key_cap == o.key_cap && tile == o.tile && blend == o.blend &&
             debug == o.debug && raster == o.raster;
    }
  };
  struct BatchGraph {
    BatchKey key;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    uint64_t last_use;
  };
  static constexpr size_t kBatchGraphCacheSize = 8;
  std::vector<BatchGraph> batch_graphs_;
  std::vector<BatchKey> batch_seen_;
  unsigned char *batch_stage_ = nullptr;  // pinned: every group's view table, back to back
  uint64_t batch_stage_bytes_ = 0;
  cudaEvent_t batch_ev_ = nullptr;        // the last batch launch has read the staging area
  bool batch_mode_ = false;               // launch_all: table copied, no phase events
  uint64_t batch_graph_launches_ = 0;
  void drop_batch_graphs();
  uint64_t graph_clock_ = 0;
};

uint32_t tile_sort_passes(uint32_t num_tiles);

}  // namespace gsr
