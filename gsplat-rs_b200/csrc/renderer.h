// The CUDA SortedAlpha renderer behind one GsplatContext: owns a CUDA
// stream, the HBM-resident scene and the image, and runs the frame pipeline
// (pipeline.h) over one view.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <memory>
#include <string>
#include <vector>

#include "pipeline.h"

namespace gsr {

using FrameResult = RunResult;

// True when an order sorted for camera `a` may still be drawn for camera `b`
// (the reference's stale-order pose bound; `limit` is the translation bound).
bool order_pose_compatible(const GsplatCamera &a, const GsplatCamera &b, float limit);

// Checks for a usable sm_100 device and returns its ordinal; throws
// Error(Unsupported) otherwise.
int require_b200();
constexpr uint32_t kMaxImageDimension = 16384;

class Renderer {
 public:
  Renderer(uint32_t width, uint32_t height);
  ~Renderer();

  void set_size(uint32_t width, uint32_t height);
  uint32_t width() const { return width_; }
  uint32_t height() const { return height_; }
  void set_tile(uint32_t tile);
  uint32_t tile() const { return lanes_[0].pipe->tile(); }
  void set_blend_mode(uint32_t mode);
  uint32_t blend_mode() const { return lanes_[0].pipe->blend_mode(); }
  void set_debug(bool on);
  void set_use_graph(bool on);
  void set_raster_config(const RasterConfig &c);
  // Frame lanes: enqueued frames rotate over `lanes` pipelines, each on its
  // own stream with its own workspace and image, so consecutive frames
  // overlap on the device (one frame's latency-bound sorts beside another's
  // raster). 1 (the default) runs every frame on one stream. Frames stay
  // independent and each image is exactly the single-lane image. A sort
  // interval other than 0 runs on one lane (its reused order lives in that
  // lane's workspace).
  static constexpr uint32_t kMaxLanes = 8;
  void set_frame_lanes(uint32_t lanes);
  uint32_t frame_lanes() const { return lane_count_; }
  // Depth-order refresh cadence. 0 (the default): every frame sorts, as the
  // reference's context does. k >= 1: the reference's surface sort interval —
  // the order is re-sorted when the camera has changed k times since the
  // last sort; other frames reuse the last sorted visible order with the new
  // camera's projection, but only while the camera stays within the
  // reference's stale-order pose bound of the camera that order was sorted
  // for (translation at most 2% of the scene's bounding-box diagonal, at
  // least 1e-4; rotation at most 0.01 rad; surface_session.rs:23-24,
  // 670-674, 1255-1272): a larger move re-sorts at once.
  void set_sort_interval(uint32_t interval);
  uint32_t sort_interval() const { return sort_interval_; }

  void load_scene(const HostScene &s);
  // The scene in the packed resident format (68 bytes per SH3 splat; SH degree <= 3).
  void load_scene_packed(const HostScene &s);
  // PLY file; a binary body is decoded on the device (load_scene_file).
  void load_scene_path(const std::string &path);
  bool has_scene() const { return scene_ != nullptr; }
  const DeviceScene *scene() const { return scene_.get(); }

  // Renders one frame; throws Error on failure. Blocks until the frame's
  // counters are on the host.
  FrameResult render(const GsplatCamera &cam);
  // Enqueues one frame without waiting for it; the pair capacity of the last
  // synchronous frame is used. Overflow or device-wait errors of any enqueued
  // frame surface at the next sync().
  void render_async(const GsplatCamera &cam);
  // Waits for enqueued frames, refreshes last() and throws if one of them
  // overflowed its pair buffers or hit a device wait limit.
  void sync();
  const FrameResult &last() const { return last_; }
  uint64_t key_capacity() const { return front_pipe().key_capacity(); }
  bool has_frame() const { return has_frame_; }

  void readback_rgba8(uint8_t *out, uint64_t len);
  // Requests the copy of the last frame's image into `out` (pinned host
  // memory, kept valid until sync()) and returns. The copy runs on a copy
  // stream while the next frame renders: it is issued with that frame, timed
  // to its raster, or at sync(). Frames alternate between two image buffers;
  // a buffer is rendered into again only after its copy.
  void readback_rgba8_async(uint8_t *out, uint64_t len);
  std::vector<uint32_t> debug_order();
  std::vector<ProjectedDev> debug_projected();
  std::vector<float2> debug_coverage();
  void debug_tile_pairs(std::vector<uint32_t> &tiles, std::vector<uint32_t> &ids);
  void debug_tile_ranges(std::vector<uint32_t> &ranges, std::vector<uint32_t> &ids);

  int device() const { return device_; }
  // The first lane's stream (the only one while frame lanes are 1).
  cudaStream_t stream() const { return lanes_[0].stream; }

 private:
  struct Lane {
    cudaStream_t stream = nullptr;
    std::unique_ptr<Pipeline> pipe;
  };
  std::vector<ViewSpec> one_view(const GsplatCamera &cam);
  void ensure_image();
  void plan_order(Pipeline &pipe, const GsplatCamera &cam);  // sets the lane's order reuse
  void finish_order(const Pipeline &pipe);
  void scene_changed();  // forces a sort and takes the scene's translation bound
  void sync_all_lanes();  // waits for every lane's stream (no error checks)
  uint32_t lanes_in_use() const { return sort_interval_ == 0 ? lane_count_ : 1u; }
  uint32_t image_slots() const { return lanes_in_use() < 2 ? 2u : lanes_in_use(); }
  Pipeline &front_pipe() const { return *lanes_[front_lane_].pipe; }
  // The lane and image slot of the next frame; makes the lane wait for
  // whatever still reads or writes that slot.
  void next_frame(uint32_t &lane, uint32_t &slot);
  void frame_enqueued(uint32_t lane, uint32_t slot);  // the slot now holds the last frame

  int device_ = 0;
  std::vector<Lane> lanes_;  // lanes_[0] always exists
  uint32_t lane_count_ = 1;
  uint64_t frame_seq_ = 0;   // frames enqueued: selects the lane and the image slot
  uint32_t front_lane_ = 0;  // lane of the last frame
  uint64_t pair_capacity_ = 0;  // largest tile-pair capacity a synchronous frame needed
  uint32_t width_, height_;
  bool has_frame_ = false;
  uint32_t sort_interval_ = 0, changes_since_sort_ = 0;
  bool force_sort_ = true, has_last_camera_ = false;
  GsplatCamera last_camera_{};
  GsplatCamera sorted_camera_{};      // the camera the current order was sorted for
  float order_translation_limit_ = 1e-4f;
  std::unique_ptr<DeviceScene> scene_;
  FrameResult last_;
  // Image slots: frames rotate over max(2, lanes in use) buffers (front_ =
  // the last frame's), so a frame's readback overlaps the next frames.
  DeviceBuffer image_[kMaxLanes];
  uint32_t front_ = 0;
  cudaStream_t copy_stream_ = nullptr;
  cudaEvent_t rendered_[kMaxLanes] = {};  // the frame into image_[k] is complete
  cudaEvent_t copied_[kMaxLanes] = {};    // the async readback of image_[k] is complete
  bool copy_pending_[kMaxLanes] = {};
  // A readback requested but not yet issued: it starts with the next frame's
  // raster (one long kernel, so the copy's PCIe traffic does not delay that
  // frame's other launches), or at sync().
  struct DeferredCopy {
    bool pending = false;
    int image = 0;
    uint8_t *out = nullptr;
    uint64_t bytes = 0;
  } deferred_;
  void issue_copy(bool after_next_raster);
  const std::vector<uint64_t> image_base_{0};
};

}  // namespace gsr
