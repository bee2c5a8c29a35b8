#include <cmath>
// Plain frames: one view of the frame pipeline (no device code in this file).

#include <cstring>
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
  GSR_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  GSR_CUDA(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
  for (int k = 0; k < 2; ++k) {
    GSR_CUDA(cudaEventCreateWithFlags(&rendered_[k], cudaEventDisableTiming));
    GSR_CUDA(cudaEventCreateWithFlags(&copied_[k], cudaEventDisableTiming));
  }
  pipe_ = std::make_unique<Pipeline>(device_, stream_);
}

Renderer::~Renderer() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  if (copy_stream_) cudaStreamSynchronize(copy_stream_);
  pipe_.reset();
  scene_.reset();
  image_[0].reset(0);
  image_[1].reset(0);
  for (int k = 0; k < 2; ++k) {
    if (rendered_[k]) cudaEventDestroy(rendered_[k]);
    if (copied_[k]) cudaEventDestroy(copied_[k]);
  }
  if (copy_stream_) cudaStreamDestroy(copy_stream_);
  if (stream_) cudaStreamDestroy(stream_);
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
  pipe_->set_tile(tile);
}

void Renderer::load_scene(const HostScene &s) {
  Code c = scene_validate(s);
  if (c != Code::Ok) throw Error(Code::InvalidArgument, "invalid scene buffers");
  GSR_CUDA(cudaSetDevice(device_));
  GSR_CUDA(cudaStreamSynchronize(stream_));
  scene_.reset();
  scene_ = upload_scene(s, stream_);
  scene_changed();
}

void Renderer::load_scene_packed(const HostScene &s) {
  Code c = scene_validate(s);
  if (c != Code::Ok) throw Error(Code::InvalidArgument, "invalid scene buffers");
  GSR_CUDA(cudaSetDevice(device_));
  GSR_CUDA(cudaStreamSynchronize(stream_));
  std::unique_ptr<DeviceScene> sc = upload_scene_packed(s, stream_);
  scene_ = std::move(sc);
  scene_changed();
}

void Renderer::load_scene_path(const std::string &path) {
  GSR_CUDA(cudaSetDevice(device_));
  GSR_CUDA(cudaStreamSynchronize(stream_));
  // The current scene stays loaded until the new one is complete.
  std::unique_ptr<DeviceScene> sc = load_scene_file(path, stream_, {});
  scene_ = std::move(sc);
  scene_changed();
}

void Renderer::ensure_image() {
  const uint64_t need = 4ull * width_ * height_;
  if (image_[0].size() < need || image_[0].size() > 2 * need) {
    if (deferred_.pending) issue_copy(false);
    GSR_CUDA(cudaStreamSynchronize(stream_));
    GSR_CUDA(cudaStreamSynchronize(copy_stream_));
    image_[0].reset(need);
    image_[1].reset(need);
    copy_pending_[0] = copy_pending_[1] = false;
  }
}

uint32_t *Renderer::next_image() {
  const int k = front_ ^ 1;
  // a requested readback of this buffer has to be issued before it is reused
  if (deferred_.pending && deferred_.image == k) issue_copy(false);
  // the buffer's last readback must land before the frame overwrites it
  if (copy_pending_[k]) {
    GSR_CUDA(cudaStreamWaitEvent(stream_, copied_[k], 0));
    copy_pending_[k] = false;
  }
  return image_[k].as<uint32_t>();
}

void Renderer::frame_enqueued() {
  front_ ^= 1;
  GSR_CUDA(cudaEventRecord(rendered_[front_], stream_));
  if (deferred_.pending) issue_copy(true);
}

void Renderer::issue_copy(bool after_next_raster) {
  const int k = deferred_.image;
  // The image is complete once its frame is; with a frame enqueued after it,
  // that frame's raster start is later still.
  GSR_CUDA(cudaStreamWaitEvent(copy_stream_,
                               after_next_raster ? pipe_->raster_start_event() : rendered_[k], 0));
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
void Renderer::plan_order(const GsplatCamera &cam) {
  const bool changed = !has_last_camera_ || std::memcmp(&cam, &last_camera_, sizeof cam) != 0;
  if (changed) ++changes_since_sort_;
  const bool refresh = sort_interval_ == 0 || force_sort_ ||
                       (changed && changes_since_sort_ >= sort_interval_) ||
                       !order_pose_compatible(sorted_camera_, cam, order_translation_limit_);
  pipe_->set_reuse_order(!refresh);
  last_camera_ = cam;
  has_last_camera_ = true;
}

void Renderer::finish_order() {
  if (!pipe_->last_reused_order()) {
    changes_since_sort_ = 0;
    force_sort_ = false;
    sorted_camera_ = last_camera_;
  }
}

FrameResult Renderer::render(const GsplatCamera &cam) {
  auto views = one_view(cam);
  plan_order(cam);
  last_ = pipe_->run(views, next_image(), image_base_);
  frame_enqueued();
  finish_order();
  has_frame_ = true;
  return last_;
}

void Renderer::render_async(const GsplatCamera &cam) {
  auto views = one_view(cam);
  plan_order(cam);
  pipe_->enqueue(views, next_image(), image_base_);
  frame_enqueued();
  finish_order();
  has_frame_ = true;
}

void Renderer::sync() {
  if (deferred_.pending) issue_copy(false);
  try {
    last_ = pipe_->sync();
  } catch (const Error &e) {
    if (e.code == Code::Internal) has_frame_ = false;
    throw;
  }
  GSR_CUDA(cudaStreamSynchronize(copy_stream_));
}

void Renderer::readback_rgba8(uint8_t *out, uint64_t len) {
  const uint64_t need = 4ull * width_ * height_;
  if (!has_frame_) throw Error(Code::InvalidArgument, "no rendered frame to read back");
  if (len < need) throw Error(Code::InvalidArgument, "output buffer too small for the RGBA8 image");
  GSR_CUDA(cudaSetDevice(device_));
  if (deferred_.pending) issue_copy(false);
  GSR_CUDA(cudaMemcpyAsync(out, image_[front_].get(), need, cudaMemcpyDeviceToHost, stream_));
  GSR_CUDA(cudaStreamSynchronize(stream_));
}

void Renderer::readback_rgba8_async(uint8_t *out, uint64_t len) {
  const uint64_t need = 4ull * width_ * height_;
  if (!has_frame_) throw Error(Code::InvalidArgument, "no rendered frame to read back");
  if (len < need) throw Error(Code::InvalidArgument, "output buffer too small for the RGBA8 image");
  GSR_CUDA(cudaSetDevice(device_));
  if (deferred_.pending) issue_copy(false);
  deferred_ = DeferredCopy{true, front_, out, need};
}

std::vector<uint32_t> Renderer::debug_order() {
  if (!has_frame_) throw Error(Code::InvalidArgument, "no rendered frame");
  return pipe_->debug_order();
}

std::vector<ProjectedDev> Renderer::debug_projected() {
  if (!has_frame_) throw Error(Code::InvalidArgument, "debug taps were not enabled for the last frame");
  return pipe_->debug_projected(scene_->n);
}

void Renderer::debug_tile_pairs(std::vector<uint32_t> &tiles, std::vector<uint32_t> &ids) {
  if (!has_frame_) throw Error(Code::InvalidArgument, "debug taps were not enabled for the last frame");
  pipe_->debug_tile_pairs(tiles, ids);
}

void Renderer::debug_tile_ranges(std::vector<uint32_t> &ranges, std::vector<uint32_t> &ids) {
  if (!has_frame_) throw Error(Code::InvalidArgument, "no rendered frame");
  const uint32_t t = pipe_->tile();
  const uint32_t tiles = ((width_ + t - 1) / t) * ((height_ + t - 1) / t);
  pipe_->debug_tile_ranges(tiles, ranges, ids);
}

}  // namespace gsr
