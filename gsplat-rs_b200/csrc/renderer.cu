#include <algorithm>
#include <cmath>
// Plain frames: one view of the frame pipeline (no device code in this file).

#include <cstring>
#include <exception>
#include <string>

#include "cuda_check.h"
#include "renderer.h"

namespace gsr {

int require_b200() {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    throw Error(Code::Unsupported, "gpu rasterizer unavailable: no CUDA device");
  }
  int device = 0;
  GSR_CUDA(cudaGetDevice(&device));
  cudaDeviceProp prop;
  GSR_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10 || prop.minor != 0)
    throw Error(Code::Unsupported, std::string("gpu rasterizer unavailable: device ") + prop.name +
                                       " is not sm_100 (B200)");
  return device;
}

Renderer::Renderer(uint32_t width, uint32_t height) : width_(width), height_(height) {
  device_ = require_b200();
  if (width > kMaxImageDimension || height > kMaxImageDimension)
    throw Error(Code::Unsupported, "requested dimensions exceed the maximum of 16384");
  lanes_.reserve(kMaxLanes);
  lanes_.emplace_back();
  GSR_CUDA(cudaStreamCreateWithFlags(&lanes_[0].stream, cudaStreamNonBlocking));
  GSR_CUDA(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
  for (uint32_t k = 0; k < kMaxLanes; ++k) {
    GSR_CUDA(cudaEventCreateWithFlags(&rendered_[k], cudaEventDisableTiming));
    GSR_CUDA(cudaEventCreateWithFlags(&copied_[k], cudaEventDisableTiming));
  }
  lanes_[0].pipe = std::make_unique<Pipeline>(device_, lanes_[0].stream);
}

Renderer::~Renderer() {
  cudaSetDevice(device_);
  for (auto &lane : lanes_)
    if (lane.stream) cudaStreamSynchronize(lane.stream);
  if (copy_stream_) cudaStreamSynchronize(copy_stream_);
  for (auto &lane : lanes_) lane.pipe.reset();
  scene_.reset();
  for (uint32_t k = 0; k < kMaxLanes; ++k) {
    image_[k].reset(0);
    if (rendered_[k]) cudaEventDestroy(rendered_[k]);
    if (copied_[k]) cudaEventDestroy(copied_[k]);
  }
  if (copy_stream_) cudaStreamDestroy(copy_stream_);
  for (auto &lane : lanes_)
    if (lane.stream) cudaStreamDestroy(lane.stream);
}

void Renderer::sync_all_lanes() {
  for (auto &lane : lanes_) GSR_CUDA(cudaStreamSynchronize(lane.stream));
}

// New lanes copy the first lane's settings and its tile-pair capacity (an
// enqueued frame keeps the capacity it finds, so a fresh lane must not start
// smaller than the frames it will take over).
void Renderer::set_frame_lanes(uint32_t lanes) {
  if (lanes < 1 || lanes > kMaxLanes)
    throw Error(Code::InvalidArgument, "frame lanes must be 1 to 8");
  GSR_CUDA(cudaSetDevice(device_));
  if (deferred_.pending) issue_copy(false);
  sync_all_lanes();
  GSR_CUDA(cudaStreamSynchronize(copy_stream_));
  const Pipeline &first = *lanes_[0].pipe;
  while (lanes_.size() < lanes) {
    Lane lane;
    GSR_CUDA(cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking));
    lane.pipe = std::make_unique<Pipeline>(device_, lane.stream);
    lane.pipe->set_tile(first.tile());
    lane.pipe->set_blend_mode(first.blend_mode());
    lane.pipe->set_debug(first.debug());
    lane.pipe->set_use_graph(first.use_graph());
    lane.pipe->set_raster_config(first.raster_config());
    lanes_.push_back(std::move(lane));
  }
  for (auto &lane : lanes_) pair_capacity_ = std::max(pair_capacity_, lane.pipe->key_capacity());
  for (uint32_t k = 0; k < lanes; ++k)
    if (pair_capacity_) lanes_[k].pipe->reserve_pairs(pair_capacity_);
  lane_count_ = lanes;
  ensure_image();
}

void Renderer::set_blend_mode(uint32_t mode) {
  for (auto &lane : lanes_) lane.pipe->set_blend_mode(mode);
}
void Renderer::set_debug(bool on) {
  for (auto &lane : lanes_) lane.pipe->set_debug(on);
}
void Renderer::set_use_graph(bool on) {
  for (auto &lane : lanes_) lane.pipe->set_use_graph(on);
}
void Renderer::set_raster_config(const RasterConfig &c) {
  for (auto &lane : lanes_) lane.pipe->set_raster_config(c);
}

void Renderer::set_size(uint32_t width, uint32_t height) {
  if (width == 0 || height == 0) throw Error(Code::InvalidArgument, "invalid renderer configuration");
  if (width > kMaxImageDimension || height > kMaxImageDimension)
    throw Error(Code::Unsupported, "requested dimensions exceed the maximum of 16384");
  width_ = width;
  height_ = height;
  has_frame_ = false;
  force_sort_ = true;
}

void Renderer::set_tile(uint32_t tile) {
  if (tile != 8 && tile != 16) throw Error(Code::InvalidArgument, "tile size must be 8 or 16");
  for (auto &lane : lanes_) lane.pipe->set_tile(tile);
}

void Renderer::load_scene(const HostScene &s) {
  Code c = scene_validate(s);
  if (c != Code::Ok) throw Error(Code::InvalidArgument, "invalid scene buffers");
  GSR_CUDA(cudaSetDevice(device_));
  sync_all_lanes();
  scene_.reset();
  scene_ = upload_scene(s, lanes_[0].stream);
  scene_changed();
}

void Renderer::load_scene_packed(const HostScene &s) {
  Code c = scene_validate(s);
  if (c != Code::Ok) throw Error(Code::InvalidArgument, "invalid scene buffers");
  GSR_CUDA(cudaSetDevice(device_));
  sync_all_lanes();
  std::unique_ptr<DeviceScene> sc = upload_scene_packed(s, lanes_[0].stream);
  scene_ = std::move(sc);
  scene_changed();
}

void Renderer::load_scene_path(const std::string &path) {
  GSR_CUDA(cudaSetDevice(device_));
  sync_all_lanes();
  // The current scene stays loaded until the new one is complete.
  std::unique_ptr<DeviceScene> sc = load_scene_file(path, lanes_[0].stream, {});
  scene_ = std::move(sc);
  scene_changed();
}

// Image slots only grow (a context that alternates sizes keeps its buffers,
// and with them the pointers its captured graphs use: a reallocation costs a
// device synchronisation, a free and an allocation, milliseconds under a
// loaded allocator); they shrink only when 64 times larger than needed.
void Renderer::ensure_image() {
  const uint64_t need = 4ull * width_ * height_;
  const uint32_t slots = image_slots();
  bool ok = true;
  for (uint32_t k = 0; k < slots; ++k)
    ok = ok && image_[k].size() >= need &&
         (image_[k].size() <= 64 * need || image_[k].size() <= (64ull << 20));
  if (!ok) {
    if (deferred_.pending) issue_copy(false);
    sync_all_lanes();
    GSR_CUDA(cudaStreamSynchronize(copy_stream_));
    for (uint32_t k = 0; k < kMaxLanes; ++k) {
      image_[k].reset(k < slots ? need : 0);
      copy_pending_[k] = false;
    }
  }
}

void Renderer::next_frame(uint32_t &lane, uint32_t &slot) {
  lane = (uint32_t)(frame_seq_ % lanes_in_use());
  slot = (uint32_t)(frame_seq_ % image_slots());
  ++frame_seq_;
  const cudaStream_t st = lanes_[lane].stream;
  // a requested readback of this buffer has to be issued before it is reused
  if (deferred_.pending && deferred_.image == (int)slot) issue_copy(false);
  // the buffer's last frame (another lane's, after a change of lanes) and
  // its last readback must complete before this frame overwrites it
  GSR_CUDA(cudaStreamWaitEvent(st, rendered_[slot], 0));
  if (copy_pending_[slot]) {
    GSR_CUDA(cudaStreamWaitEvent(st, copied_[slot], 0));
    copy_pending_[slot] = false;
  }
}

void Renderer::frame_enqueued(uint32_t lane, uint32_t slot) {
  front_ = slot;
  front_lane_ = lane;
  GSR_CUDA(cudaEventRecord(rendered_[slot], lanes_[lane].stream));
  if (deferred_.pending) issue_copy(true);
}

void Renderer::issue_copy(bool after_next_raster) {
  const int k = deferred_.image;
  // The image is complete once its frame is; with a frame enqueued after it,
  // the copy also waits for that frame's raster to start (one long kernel,
  // so the copy's PCIe traffic does not delay that frame's other launches).
  GSR_CUDA(cudaStreamWaitEvent(copy_stream_, rendered_[k], 0));
  if (after_next_raster)
    GSR_CUDA(cudaStreamWaitEvent(copy_stream_, front_pipe().raster_start_event(), 0));
  GSR_CUDA(cudaMemcpyAsync(deferred_.out, image_[k].get(), deferred_.bytes, cudaMemcpyDeviceToHost,
                           copy_stream_));
  GSR_CUDA(cudaEventRecord(copied_[k], copy_stream_));
  copy_pending_[k] = true;
  deferred_.pending = false;
}

std::vector<ViewSpec> Renderer::one_view(const GsplatCamera &cam) {
  if (!camera_valid(cam)) throw Error(Code::InvalidArgument, "invalid camera");
  if (!scene_) throw Error(Code::SceneNotLoaded, "scene not loaded");
  GSR_CUDA(cudaSetDevice(device_));
  ensure_image();
  return {ViewSpec{scene_.get(), cam, width_, height_}};
}

void Renderer::set_sort_interval(uint32_t interval) { sort_interval_ = interval; }

void Renderer::scene_changed() {
  has_frame_ = false;
  force_sort_ = true;
  // The stale-order translation bound: 2% of the scene's bounding-box
  // diagonal, at least 1e-4 (surface_session.rs:660-674, f32 as there).
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  const std::vector<float> &pos = scene_->positions;
  for (size_t i = 0; i + 2 < pos.size(); i += 3)
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::fmin(mn[a], pos[i + a]);
      mx[a] = std::fmax(mx[a], pos[i + a]);
    }
  const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
  const float diagonal = std::sqrt(dx * dx + dy * dy + dz * dz);
  order_translation_limit_ = pos.empty() ? 1e-4f : std::fmax(diagonal * 0.02f, 1e-4f);
}

// The reference's async_order_pose_compatible (surface_session.rs:1255-1272):
// an order sorted for camera `a` may be drawn for camera `b` while b's
// position is within `limit` of a's and the rotation between them is at
// most 0.01 rad.
bool order_pose_compatible(const GsplatCamera &a, const GsplatCamera &b, float limit) {
  const float dx = b.position[0] - a.position[0];
  const float dy = b.position[1] - a.position[1];
  const float dz = b.position[2] - a.position[2];
  if (dx * dx + dy * dy + dz * dz > limit * limit) return false;
  const float *qa = a.rotation_xyzw, *qb = b.rotation_xyzw;
  const float dot =
      std::fmin(std::fmax(std::fabs(qa[0] * qb[0] + qa[1] * qb[1] + qa[2] * qb[2] + qa[3] * qb[3]),
                          0.0f),
                1.0f);
  return 2.0f * std::acos(dot) <= 0.01f;
}

// Interval 0 sorts every frame, as the reference's Renderer::render_frame
// does. Otherwise the reference's SurfaceFrameState::plan
// (surface_session.rs:536-596): sort when forced, when there is no order
// yet, or when the camera has changed `interval` times since the last sort;
// and, as for the reference's reused orders (surface_session.rs:1149-1153),
// when the camera has left the pose bound of the order's own camera.
void Renderer::plan_order(Pipeline &pipe, const GsplatCamera &cam) {
  const bool changed = !has_last_camera_ || std::memcmp(&cam, &last_camera_, sizeof cam) != 0;
  if (changed) ++changes_since_sort_;
  const bool refresh = sort_interval_ == 0 || force_sort_ ||
                       (changed && changes_since_sort_ >= sort_interval_) ||
                       !order_pose_compatible(sorted_camera_, cam, order_translation_limit_);
  pipe.set_reuse_order(!refresh);
  last_camera_ = cam;
  has_last_camera_ = true;
}

void Renderer::finish_order(const Pipeline &pipe) {
  if (!pipe.last_reused_order()) {
    changes_since_sort_ = 0;
    force_sort_ = false;
    sorted_camera_ = last_camera_;
  }
}

FrameResult Renderer::render(const GsplatCamera &cam) {
  auto views = one_view(cam);
  uint32_t lane, slot;
  next_frame(lane, slot);
  Pipeline &pipe = *lanes_[lane].pipe;
  plan_order(pipe, cam);
  last_ = pipe.run(views, image_[slot].as<uint32_t>(), image_base_);
  pair_capacity_ = std::max(pair_capacity_, pipe.key_capacity());
  frame_enqueued(lane, slot);
  finish_order(pipe);
  has_frame_ = true;
  return last_;
}

void Renderer::render_async(const GsplatCamera &cam) {
  auto views = one_view(cam);
  uint32_t lane, slot;
  next_frame(lane, slot);
  Pipeline &pipe = *lanes_[lane].pipe;
  // an enqueued frame keeps the pair capacity it finds: every lane gets the
  // largest a synchronous frame has needed
  if (pipe.key_capacity() < pair_capacity_) pipe.reserve_pairs(pair_capacity_);
  plan_order(pipe, cam);
  pipe.enqueue(views, image_[slot].as<uint32_t>(), image_base_);
  frame_enqueued(lane, slot);
  finish_order(pipe);
  has_frame_ = true;
}

void Renderer::sync() {
  if (deferred_.pending) issue_copy(false);
  // Every lane is waited for; the first error is reported after all of
  // them, and the result is the last frame's.
  std::exception_ptr first;
  bool internal = false;
  for (uint32_t k = 0; k < lanes_.size(); ++k) {
    try {
      FrameResult r = lanes_[k].pipe->sync();
      if (k == front_lane_) last_ = r;
    } catch (const Error &e) {
      if (!first) first = std::current_exception();
      internal = internal || e.code == Code::Internal;
    }
  }
  GSR_CUDA(cudaStreamSynchronize(copy_stream_));
  if (first) {
    if (internal) has_frame_ = false;
    std::rethrow_exception(first);
  }
}

void Renderer::readback_rgba8(uint8_t *out, uint64_t len) {
  const uint64_t need = 4ull * width_ * height_;
  if (!has_frame_) throw Error(Code::InvalidArgument, "no rendered frame to read back");
  if (len < need) throw Error(Code::InvalidArgument, "output buffer too small for the RGBA8 image");
  GSR_CUDA(cudaSetDevice(device_));
  if (deferred_.pending) issue_copy(false);
  const cudaStream_t st = lanes_[front_lane_].stream;
  GSR_CUDA(cudaMemcpyAsync(out, image_[front_].get(), need, cudaMemcpyDeviceToHost, st));
  GSR_CUDA(cudaStreamSynchronize(st));
}

void Renderer::readback_rgba8_async(uint8_t *out, uint64_t len) {
  const uint64_t need = 4ull * width_ * height_;
  if (!has_frame_) throw Error(Code::InvalidArgument, "no rendered frame to read back");
  if (len < need) throw Error(Code::InvalidArgument, "output buffer too small for the RGBA8 image");
  GSR_CUDA(cudaSetDevice(device_));
  if (deferred_.pending) issue_copy(false);
  deferred_ = DeferredCopy{true, (int)front_, out, need};
}

std::vector<uint32_t> Renderer::debug_order() {
  if (!has_frame_) throw Error(Code::InvalidArgument, "no rendered frame");
  return front_pipe().debug_order();
}

std::vector<ProjectedDev> Renderer::debug_projected() {
  if (!has_frame_) throw Error(Code::InvalidArgument, "debug taps were not enabled for the last frame");
  return front_pipe().debug_projected(scene_->n);
}

std::vector<float2> Renderer::debug_coverage() {
  if (!has_frame_) throw Error(Code::InvalidArgument, "debug taps were not enabled for the last frame");
  return front_pipe().debug_coverage(scene_->n);
}

void Renderer::debug_tile_pairs(std::vector<uint32_t> &tiles, std::vector<uint32_t> &ids) {
  if (!has_frame_) throw Error(Code::InvalidArgument, "debug taps were not enabled for the last frame");
  front_pipe().debug_tile_pairs(tiles, ids);
}

void Renderer::debug_tile_ranges(std::vector<uint32_t> &ranges, std::vector<uint32_t> &ids) {
  if (!has_frame_) throw Error(Code::InvalidArgument, "no rendered frame");
  const uint32_t t = front_pipe().tile();
  const uint32_t tiles = ((width_ + t - 1) / t) * ((height_ + t - 1) / t);
  front_pipe().debug_tile_ranges(tiles, ranges, ids);
}

}  // namespace gsr
