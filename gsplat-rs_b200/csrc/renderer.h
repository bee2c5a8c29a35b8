// The CUDA SortedAlpha renderer behind one GsplatContext: owns a CUDA
// stream, the HBM-resident scene and the frame workspace, and runs the
// K1 -> depth sort -> K2 -> tile sort -> ranges -> K4 frame pipeline.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <memory>
#include <vector>

#include "device_types.h"
#include "gsr_host.h"

namespace gsr {

// One device allocation, freed on destruction.
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  ~DeviceBuffer();
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  void reset(uint64_t bytes);  // frees, then allocates `bytes` (0 = free only)
  void *get() const { return ptr_; }
  uint64_t size() const { return bytes_; }
  template <typename T>
  T *as(uint64_t byte_offset = 0) const {
    return reinterpret_cast<T *>(static_cast<char *>(ptr_) + byte_offset);
  }

 private:
  void *ptr_ = nullptr;
  uint64_t bytes_ = 0;
};

// Scene resident in HBM (SoA float4 planes, see device_types.h SceneDev).
struct DeviceScene {
  DeviceBuffer mem;
  SceneDev dev{};
  uint32_t n = 0;
  uint32_t sh_degree = 0;
  std::vector<float> positions;  // host copy for automatic camera framing
};
std::unique_ptr<DeviceScene> upload_scene(const HostScene &s, cudaStream_t stream);

// Device-timed phases of one frame (CUDA events on the context stream).
enum Phase : int { kPhasePreprocess, kPhaseDepthSort, kPhaseEmit, kPhaseTileSort, kPhaseRanges,
                   kPhaseRaster, kPhaseCount };

struct FrameResult {
  float frame_ms = 0, preprocess_ms = 0, sort_ms = 0, raster_ms = 0;
  float phase_ms[kPhaseCount] = {};
  uint64_t visible = 0, drawn = 0, keys = 0;
  uint32_t reruns = 0;
};

class Renderer {
 public:
  Renderer(uint32_t width, uint32_t height);
  ~Renderer();

  void set_size(uint32_t width, uint32_t height);
  uint32_t width() const { return width_; }
  uint32_t height() const { return height_; }
  void set_tile(uint32_t tile);
  uint32_t tile() const { return tile_; }
  void set_blend_mode(uint32_t mode) { blend_mode_ = mode; }
  uint32_t blend_mode() const { return blend_mode_; }
  void set_debug(bool on) { debug_ = on; }

  void load_scene(const HostScene &s);
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
  uint64_t key_capacity() const { return key_cap_; }
  bool has_frame() const { return has_frame_; }

  void readback_rgba8(uint8_t *out, uint64_t len);
  std::vector<uint32_t> debug_order();
  std::vector<ProjectedDev> debug_projected();
  void debug_tile_pairs(std::vector<uint32_t> &tiles, std::vector<uint32_t> &ids);
  void debug_tile_ranges(std::vector<uint32_t> &ranges, std::vector<uint32_t> &ids);

  int device() const { return device_; }
  cudaStream_t stream() const { return stream_; }

 private:
  void ensure_scene_workspace();
  void ensure_key_workspace(uint64_t capacity);
  void ensure_image_workspace();
  void prepare_frame();
  void enqueue_frame(const FrameParams &p);
  void run_frame(const FrameParams &p);
  void collect(FrameResult &r);
  SortPlan read_plan(int which);

  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev_[kPhaseCount + 1] = {};
  uint32_t width_, height_;
  uint32_t tile_ = 16;
  uint32_t blend_mode_ = 0;
  bool debug_ = false;
  bool has_frame_ = false;
  std::unique_ptr<DeviceScene> scene_;
  FrameResult last_;

  // Small per-frame scratch: counters, two sort plans and the K1 / K2
  // look-back words (zeroed with one memset per frame).
  DeviceBuffer frame_scratch_;
  uint64_t frame_scratch_zero_bytes_ = 0;
  FrameCounters *counters_ = nullptr;
  SortPlan *depth_plan_ = nullptr;
  SortPlan *tile_plan_ = nullptr;
  unsigned long long *k1_status_ = nullptr;
  unsigned long long *emit_status_ = nullptr;
  uint32_t *sticky_ = nullptr;  // OR of error bits of every frame since the last sync
  uint32_t *key_hist_ = nullptr;   // [4][256] depth-key digit histograms (from K1)
  uint32_t *tile_hist_ = nullptr;  // [4][256] tile-id digit histograms (from K2)
  // Splat-sized workspace.
  DeviceBuffer splat_ws_;
  uint32_t splat_cap_ = 0;
  uint32_t *vis_keys0_ = nullptr, *vis_vals0_ = nullptr, *vis_keys1_ = nullptr,
           *vis_vals1_ = nullptr;
  uint2 *rects_ = nullptr;
  Record *records_ = nullptr;
  uint32_t *depth_sort_work_ = nullptr;
  DeviceBuffer projected_;
  // Pair-sized workspace.
  DeviceBuffer key_ws_;
  uint64_t key_cap_ = 0;
  uint32_t *tile_keys0_ = nullptr, *tile_vals0_ = nullptr, *tile_keys1_ = nullptr,
           *tile_vals1_ = nullptr;
  uint32_t *tile_sort_work_ = nullptr;
  DeviceBuffer debug_pairs_;
  // Image-sized workspace.
  DeviceBuffer image_ws_;
  uint32_t image_w_ = 0, image_h_ = 0, image_tile_ = 0;
  uint2 *ranges_ = nullptr;
  uint32_t *image_ = nullptr;
  // Pinned host copy of the counters.
  FrameCounters *counters_host_ = nullptr;
};

uint32_t tile_sort_passes(uint32_t num_tiles);

}  // namespace gsr
