// Batched frames: many cameras over several HBM-resident scenes of uneven
// sizes, rendered by the frame pipeline in launch groups of up to 1024 views
// (one CUDA-graph launch per group). Images are identical, bit for bit, to
// rendering each view alone: every view keeps its own tile ids and its own
// depth order inside the shared (view, tile, depth) key space.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "pipeline.h"

namespace gsr {

// A request for one image: scene id, camera and image size.
struct BatchView {
  uint32_t scene;
  GsplatCamera camera;
  uint32_t width, height;
};

// HBM-resident scenes under a byte budget (admission of scenes).
class SceneStore {
 public:
  explicit SceneStore(uint64_t budget_bytes) : budget_(budget_bytes) {}
  // Uploads and returns the new scene's id; Unsupported if the budget would
  // be exceeded.
  uint32_t add(const HostScene &s, cudaStream_t stream);
  // Throws Unsupported if `bytes` more would exceed the budget.
  void check_budget(uint64_t bytes) const;
  // Uploads the scene in the packed resident format (SH degree <= 3).
  uint32_t add_packed(const HostScene &s, cudaStream_t stream);
  // Loads a PLY file (a binary body decoded on the device), budget checked
  // before any allocation.
  uint32_t add_path(const std::string &path, cudaStream_t stream);
  // Takes an uploaded scene (budget checked again).
  uint32_t insert(std::unique_ptr<DeviceScene> sc);
  const DeviceScene &get(uint32_t id) const;
  uint32_t count() const { return (uint32_t)scenes_.size(); }
  uint64_t bytes() const { return bytes_; }
  uint64_t budget() const { return budget_; }
  void set_budget(uint64_t b) { budget_ = b; }

 private:
  std::vector<std::unique_ptr<DeviceScene>> scenes_;
  uint64_t bytes_ = 0, budget_;
};

// Predicted tile pairs of a view, learned from measured per-view counts: the
// largest pairs-per-splat ratio seen for the same (scene, size, tile), else
// for the scene scaled by pixel count, else a default ratio.
class PairPredictor {
 public:
  uint64_t predict(uint32_t scene, uint32_t n, uint32_t w, uint32_t h, uint32_t tile) const;
  void observe(uint32_t scene, uint32_t n, uint32_t w, uint32_t h, uint32_t tile, uint64_t pairs);

 private:
  using Key = std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>;
  std::map<Key, double> ratio_;                 // max pairs per splat
  std::map<uint32_t, double> scene_ratio_px_;   // max pairs per splat per megapixel
};

// Limits of one launch group.
struct GroupLimits {
  uint32_t max_views = 1024;
  uint64_t max_pairs = 1ull << 28;   // predicted tile pairs (sizes the key buffers)
  uint64_t max_splats = 1ull << 28;  // splats over the views (sizes the splat workspace)
  // Tiles over the views: at most 2^16 keeps the tile sort at two passes,
  // above that it takes three (limit 2^24).
  uint64_t max_tiles = 1ull << 24;
};

struct ViewGroup {
  uint32_t first, count;
  uint64_t predicted_pairs;
};

// Splits views, in order, into launch groups within `limits`.
std::vector<ViewGroup> plan_groups(const std::vector<ViewSpec> &views,
                                   const std::vector<uint64_t> &predicted, uint32_t tile,
                                   const GroupLimits &limits);

struct BatchResult {
  float device_ms = 0;     // CUDA-event time of all groups on the batch stream
  float wall_ms = 0;       // host time of the call
  uint32_t groups = 0, reruns = 0, launches = 0;
  uint32_t graph_launches = 0;  // whole-batch graph launches of the first pass (0 or 1)
  uint64_t pairs = 0;      // tile pairs over all views
  // per-phase device ms summed over the groups (phase-timed renders only)
  float phase_ms[kPhaseCount] = {};
  bool phase_timed = false;
};

// Pinned host array that only grows (pointer stable while the size fits).
template <typename T>
class PinnedArray {
 public:
  ~PinnedArray() {
    if (p_) cudaFreeHost(p_);
  }
  T *ensure(size_t n);  // frees and reallocates when n exceeds the capacity
  T *get() const { return p_; }
  size_t capacity() const { return cap_; }

 private:
  T *p_ = nullptr;
  size_t cap_ = 0;
};

// One stream with its own pipeline, image arena and pinned counters: the
// unit a batch runs on (a server owns several and overlaps them).
class Lane {
 public:
  explicit Lane(int device);
  ~Lane();
  Lane(const Lane &) = delete;
  Lane &operator=(const Lane &) = delete;
  Pipeline &pipe() { return *pipe_; }
  cudaStream_t stream() const { return stream_; }
  // Enqueues `groups` of `views` (image offsets in `bases`, pixels) without
  // waiting; per-view counters land in view_counters(), per-group counters
  // in group_counters() once the stream reaches them. one_graph: every group
  // in one CUDA graph (Pipeline::enqueue_groups; for repeated batches), else
  // one graph per group layout (served batches, which rarely repeat whole).
  // phase_sums (not with one_graph): waits for each group and adds its
  // per-phase device times there (a measurement mode: the host sees every
  // group boundary).
  void enqueue(const std::vector<ViewSpec> &views, const std::vector<uint64_t> &bases,
               uint64_t total_pixels, const std::vector<ViewGroup> &groups, uint64_t reserve,
               bool one_graph = false, float *phase_sums = nullptr);
  // Waits, re-runs groups that overflowed their pair buffers and throws on
  // device errors. Returns the reruns.
  uint32_t finish(const std::vector<ViewSpec> &views, const std::vector<uint64_t> &bases,
                  const std::vector<ViewGroup> &groups);
  float device_ms();  // start..end events of the last enqueue (+ reruns)
  bool done();        // the last enqueue has completed (non-blocking)
  uint32_t *images() const { return images_.as<uint32_t>(); }
  const ViewCounters *view_counters() const { return view_counters_.get(); }
  const FrameCounters *group_counters() const { return group_counters_.get(); }

 private:
  int device_;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t start_ = nullptr, end_ = nullptr;
  std::unique_ptr<Pipeline> pipe_;
  DeviceBuffer images_;
  PinnedArray<ViewCounters> view_counters_;
  PinnedArray<FrameCounters> group_counters_;
};

class Batch {
 public:
  Batch();
  ~Batch();
  SceneStore &scenes() { return scenes_; }
  void set_tile(uint32_t tile);
  uint32_t tile() const { return tile_; }
  void set_blend_mode(uint32_t mode);
  void set_use_graph(bool on) { lane_->pipe().set_use_graph(on); }
  void set_raster_config(const RasterConfig &c) { lane_->pipe().set_raster_config(c); }
  const RasterConfig &raster_config() { return lane_->pipe().raster_config(); }
  uint32_t blend_mode() { return lane_->pipe().blend_mode(); }
  int device() const { return device_; }
  void set_limits(const GroupLimits &l);
  // Phase timing: renders run their groups one by one, waiting after each,
  // and report per-phase device times (BatchResult::phase_ms) in place of
  // the whole-batch graph.
  void set_phase_timing(bool on) { phase_timing_ = on; }
  bool phase_timing() const { return phase_timing_; }
  const GroupLimits &limits() const { return limits_; }

  // Renders every view; blocks until all images are in HBM.
  BatchResult render(const std::vector<BatchView> &views);
  uint32_t view_count() const { return (uint32_t)specs_.size(); }
  // Per-view results by the caller's view index.
  const ViewCounters &view_stats(uint32_t view) const;
  uint32_t view_group(uint32_t view) const;
  // Device pointer to a view's RGBA8 image (valid until the next render).
  const uint32_t *image_device(uint32_t view, uint64_t *bytes) const;
  void readback_rgba8(uint32_t view, uint8_t *out, uint64_t len);
  cudaStream_t stream() const { return lane_->stream(); }
  const BatchResult &last() const { return last_; }

 private:
  int device_;
  uint32_t tile_ = 16;
  GroupLimits limits_;
  SceneStore scenes_;
  PairPredictor predictor_;
  std::unique_ptr<Lane> lane_;
  uint32_t position(uint32_t view) const;  // caller index -> render position
  std::vector<ViewSpec> specs_;            // render order (views grouped by scene)
  std::vector<uint64_t> bases_;
  std::vector<uint32_t> pos_;
  std::vector<ViewGroup> groups_;
  std::vector<ViewCounters> stats_;
  BatchResult last_;
  bool has_images_ = false;
  bool phase_timing_ = false;
};

// Validates batch views against the store and builds pipeline view specs and
// image offsets (pixels); returns the total pixel count.
uint64_t make_view_specs(const SceneStore &store, const BatchView *views, uint32_t count,
                         std::vector<ViewSpec> &specs, std::vector<uint64_t> &bases);

}  // namespace gsr
