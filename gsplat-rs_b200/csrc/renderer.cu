// Host orchestration of the frame pipeline (no device code in this file).

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>

#include "kernels.h"
#include "renderer.h"

namespace gsr {

#define GSR_CUDA(expr)                                                                    \
  do {                                                                                    \
    cudaError_t err__ = (expr);                                                           \
    if (err__ != cudaSuccess)                                                             \
      throw Error(Code::Internal, std::string("CUDA error: ") + cudaGetErrorString(err__) + \
                                      " (" #expr ")");                                    \
  } while (0)

namespace {
inline uint64_t align256(uint64_t v) { return (v + 255) & ~uint64_t(255); }
constexpr uint32_t kMaxSortItems = (1u << 30) - 1;
constexpr uint32_t kMaxImageDimension = 16384;
}  // namespace

DeviceBuffer::~DeviceBuffer() {
  if (ptr_) cudaFree(ptr_);
}

void DeviceBuffer::reset(uint64_t bytes) {
  if (ptr_) {
    cudaFree(ptr_);
    ptr_ = nullptr;
    bytes_ = 0;
  }
  if (bytes == 0) return;
  cudaError_t e = cudaMalloc(&ptr_, bytes);
  if (e != cudaSuccess) {
    ptr_ = nullptr;
    cudaGetLastError();
    throw Error(Code::Internal, "device allocation of " + std::to_string(bytes) +
                                    " bytes failed: " + cudaGetErrorString(e));
  }
  bytes_ = bytes;
}

uint32_t tile_sort_passes(uint32_t num_tiles) {
  uint32_t bits = 0;
  while (bits < 32 && (1ull << bits) < num_tiles) ++bits;
  return std::max(1u, (bits + 7) / 8);
}

std::unique_ptr<DeviceScene> upload_scene(const HostScene &s, cudaStream_t stream) {
  const uint64_t n = s.size();
  if (n > kMaxSortItems)
    throw Error(Code::Unsupported, "scene has more splats than the renderer supports (2^30 - 1)");
  ScenePacked packed;
  pack_scene(s, packed);
  auto sc = std::make_unique<DeviceScene>();
  sc->n = (uint32_t)n;
  sc->sh_degree = s.sh_degree;
  sc->positions = s.positions;
  // Three geometry planes, then the colour planes as one tight region so
  // that plane p of splat i sits at color[p * n + i].
  const uint64_t plane = align256(16 * std::max<uint64_t>(n, 1));
  const uint64_t color_bytes = align256(16 * std::max<uint64_t>(n, 1) * packed.planes);
  sc->mem.reset(3 * plane + color_bytes);
  char *base = sc->mem.as<char>();
  if (n) {
    GSR_CUDA(cudaMemcpyAsync(base, packed.pos_alpha.data(), 16 * n, cudaMemcpyHostToDevice, stream));
    GSR_CUDA(cudaMemcpyAsync(base + plane, packed.cov_a.data(), 16 * n, cudaMemcpyHostToDevice, stream));
    GSR_CUDA(cudaMemcpyAsync(base + 2 * plane, packed.cov_b.data(), 16 * n, cudaMemcpyHostToDevice, stream));
    GSR_CUDA(cudaMemcpyAsync(base + 3 * plane, packed.color.data(), 16 * n * packed.planes,
                             cudaMemcpyHostToDevice, stream));
  }
  GSR_CUDA(cudaStreamSynchronize(stream));
  sc->dev.pos_alpha = reinterpret_cast<const float4 *>(base);
  sc->dev.cov_a = reinterpret_cast<const float4 *>(base + plane);
  sc->dev.cov_b = reinterpret_cast<const float4 *>(base + 2 * plane);
  sc->dev.color = reinterpret_cast<const float4 *>(base + 3 * plane);
  sc->dev.n = (uint32_t)n;
  sc->dev.planes = packed.planes;
  return sc;
}

Renderer::Renderer(uint32_t width, uint32_t height) : width_(width), height_(height) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    throw Error(Code::Unsupported, "gpu rasterizer unavailable: no CUDA device");
  }
  GSR_CUDA(cudaGetDevice(&device_));
  cudaDeviceProp prop;
  GSR_CUDA(cudaGetDeviceProperties(&prop, device_));
  if (prop.major != 10 || prop.minor != 0)
    throw Error(Code::Unsupported, std::string("gpu rasterizer unavailable: device ") + prop.name +
                                       " is not sm_100 (B200)");
  if (width > kMaxImageDimension || height > kMaxImageDimension)
    throw Error(Code::Unsupported, "requested dimensions exceed the maximum of 16384");
  GSR_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  for (auto &ev : ev_) GSR_CUDA(cudaEventCreate(&ev));
  GSR_CUDA(cudaMallocHost(&counters_host_, sizeof(FrameCounters)));
  // Frame scratch: counters, plans (fixed), look-back words (splat-sized,
  // allocated with the splat workspace).
}

Renderer::~Renderer() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  for (auto &ev : ev_)
    if (ev) cudaEventDestroy(ev);
  if (stream_) cudaStreamDestroy(stream_);
  if (counters_host_) cudaFreeHost(counters_host_);
}

void Renderer::set_size(uint32_t width, uint32_t height) {
  if (width == 0 || height == 0) throw Error(Code::InvalidArgument, "invalid renderer configuration");
  if (width > kMaxImageDimension || height > kMaxImageDimension)
    throw Error(Code::Unsupported, "requested dimensions exceed the maximum of 16384");
  width_ = width;
  height_ = height;
  has_frame_ = false;
}

void Renderer::set_tile(uint32_t tile) {
  if (tile != 8 && tile != 16) throw Error(Code::InvalidArgument, "tile size must be 8 or 16");
  tile_ = tile;
}

void Renderer::load_scene(const HostScene &s) {
  Code c = scene_validate(s);
  if (c != Code::Ok) throw Error(Code::InvalidArgument, "invalid scene buffers");
  GSR_CUDA(cudaSetDevice(device_));
  GSR_CUDA(cudaStreamSynchronize(stream_));
  scene_.reset();
  scene_ = upload_scene(s, stream_);
  has_frame_ = false;
  ensure_scene_workspace();
}

void Renderer::ensure_scene_workspace() {
  const uint32_t n = std::max<uint32_t>(scene_->n, 1);
  if (splat_cap_ >= n && frame_scratch_.get()) return;
  // frame scratch: counters | depth plan | tile plan | k1 status | emit status
  const uint64_t k1_words = (n + 255) / 256;
  const uint64_t emit_words = (n + 1023) / 1024;
  uint64_t off = 0;
  const uint64_t off_counters = off; off += align256(sizeof(FrameCounters));
  const uint64_t off_k1 = off; off += align256(8 * k1_words);
  const uint64_t off_emit = off; off += align256(8 * emit_words);
  const uint64_t off_khist = off; off += align256(4 * 4 * 256);
  const uint64_t off_thist = off; off += align256(4 * 4 * 256);
  frame_scratch_zero_bytes_ = off;
  const uint64_t off_dplan = off; off += align256(sizeof(SortPlan));
  const uint64_t off_tplan = off; off += align256(sizeof(SortPlan));
  const uint64_t off_sticky = off; off += 256;
  frame_scratch_.reset(off);
  GSR_CUDA(cudaMemset(frame_scratch_.get(), 0, off));
  counters_ = frame_scratch_.as<FrameCounters>(off_counters);
  k1_status_ = frame_scratch_.as<unsigned long long>(off_k1);
  emit_status_ = frame_scratch_.as<unsigned long long>(off_emit);
  key_hist_ = frame_scratch_.as<uint32_t>(off_khist);
  tile_hist_ = frame_scratch_.as<uint32_t>(off_thist);
  depth_plan_ = frame_scratch_.as<SortPlan>(off_dplan);
  tile_plan_ = frame_scratch_.as<SortPlan>(off_tplan);
  sticky_ = frame_scratch_.as<uint32_t>(off_sticky);

  const uint64_t words = sort_work_words(n, 4);
  off = 0;
  uint64_t o_k0 = off; off += align256(4ull * n);
  uint64_t o_v0 = off; off += align256(4ull * n);
  uint64_t o_k1 = off; off += align256(4ull * n);
  uint64_t o_v1 = off; off += align256(4ull * n);
  uint64_t o_rect = off; off += align256(8ull * n);
  uint64_t o_rec = off; off += align256(sizeof(Record) * (uint64_t)n);
  uint64_t o_work = off; off += align256(4 * words);
  splat_ws_.reset(off);
  vis_keys0_ = splat_ws_.as<uint32_t>(o_k0);
  vis_vals0_ = splat_ws_.as<uint32_t>(o_v0);
  vis_keys1_ = splat_ws_.as<uint32_t>(o_k1);
  vis_vals1_ = splat_ws_.as<uint32_t>(o_v1);
  rects_ = splat_ws_.as<uint2>(o_rect);
  records_ = splat_ws_.as<Record>(o_rec);
  depth_sort_work_ = splat_ws_.as<uint32_t>(o_work);
  splat_cap_ = n;
  projected_.reset(0);
}

void Renderer::ensure_key_workspace(uint64_t capacity) {
  const uint32_t passes = 3;  // enough for any tile count below 2^24
  if (key_cap_ >= capacity && key_ws_.get()) return;
  if (capacity > kMaxSortItems)
    throw Error(Code::Unsupported, "tile pair count " + std::to_string(capacity) +
                                       " exceeds the renderer's limit of 2^30 - 1");
  const uint32_t cap = (uint32_t)capacity;
  const uint64_t words = sort_work_words(cap, passes);
  uint64_t off = 0;
  uint64_t o_k0 = off; off += align256(4ull * cap);
  uint64_t o_v0 = off; off += align256(4ull * cap);
  uint64_t o_k1 = off; off += align256(4ull * cap);
  uint64_t o_v1 = off; off += align256(4ull * cap);
  uint64_t o_work = off; off += align256(4 * words);
  key_ws_.reset(0);
  key_ws_.reset(off);
  tile_keys0_ = key_ws_.as<uint32_t>(o_k0);
  tile_vals0_ = key_ws_.as<uint32_t>(o_v0);
  tile_keys1_ = key_ws_.as<uint32_t>(o_k1);
  tile_vals1_ = key_ws_.as<uint32_t>(o_v1);
  tile_sort_work_ = key_ws_.as<uint32_t>(o_work);
  key_cap_ = cap;
  debug_pairs_.reset(0);
}

void Renderer::ensure_image_workspace() {
  if (image_w_ == width_ && image_h_ == height_ && image_tile_ == tile_ && image_ws_.get()) return;
  const uint32_t tiles_x = (width_ + tile_ - 1) / tile_, tiles_y = (height_ + tile_ - 1) / tile_;
  const uint64_t tiles = (uint64_t)tiles_x * tiles_y;
  if (tiles > (1u << 24)) throw Error(Code::Unsupported, "too many tiles");
  uint64_t off = 0;
  uint64_t o_r = off; off += align256(8 * tiles);
  uint64_t o_i = off; off += align256(4ull * width_ * height_);
  image_ws_.reset(off);
  ranges_ = image_ws_.as<uint2>(o_r);
  image_ = image_ws_.as<uint32_t>(o_i);
  image_w_ = width_;
  image_h_ = height_;
  image_tile_ = tile_;
}

void Renderer::enqueue_frame(const FrameParams &p) {
  const uint32_t n = scene_->n;
  GSR_CUDA(cudaMemsetAsync(frame_scratch_.get(), 0, frame_scratch_zero_bytes_, stream_));
  GSR_CUDA(cudaMemsetAsync(ranges_, 0, 8ull * p.num_tiles, stream_));
  GSR_CUDA(cudaEventRecord(ev_[0], stream_));

  K1Buffers k1{vis_keys0_, vis_vals0_, rects_, records_, k1_status_, counters_, key_hist_,
               debug_ ? projected_.as<ProjectedDev>() : nullptr};
  launch_preprocess(scene_->dev, p, k1, debug_, stream_);
  GSR_CUDA(cudaEventRecord(ev_[1], stream_));

  SortBuffers ds{vis_keys0_, vis_vals0_, vis_keys1_, vis_vals1_, &counters_->visible,
                 std::max<uint32_t>(n, 1), 0, 4, depth_plan_, depth_sort_work_, &counters_->error,
                 key_hist_};
  launch_sort(ds, stream_);
  GSR_CUDA(cudaEventRecord(ev_[2], stream_));

  const uint32_t tpasses = tile_sort_passes(p.num_tiles);
  EmitBuffers eb{depth_plan_, vis_vals0_, vis_vals1_, rects_, tile_keys0_, tile_vals0_,
                 key_cap_, emit_status_, counters_, tile_hist_, tpasses, n};
  launch_emit(eb, p, stream_);
  if (debug_) {
    GSR_CUDA(cudaMemcpyAsync(debug_pairs_.as<uint32_t>(), tile_keys0_, 4 * key_cap_,
                             cudaMemcpyDeviceToDevice, stream_));
    GSR_CUDA(cudaMemcpyAsync(debug_pairs_.as<uint32_t>(4 * key_cap_), tile_vals0_, 4 * key_cap_,
                             cudaMemcpyDeviceToDevice, stream_));
  }
  GSR_CUDA(cudaEventRecord(ev_[3], stream_));
  SortBuffers ts{tile_keys0_, tile_vals0_, tile_keys1_, tile_vals1_, &counters_->pairs,
                 (uint32_t)key_cap_, 0, tpasses, tile_plan_, tile_sort_work_, &counters_->error,
                 tile_hist_};
  launch_sort(ts, stream_);
  GSR_CUDA(cudaEventRecord(ev_[4], stream_));
  launch_ranges(tile_plan_, tile_keys0_, tile_keys1_, counters_, (uint32_t)key_cap_, ranges_, stream_);
  GSR_CUDA(cudaEventRecord(ev_[5], stream_));

  launch_raster(p, ranges_, tile_plan_, tile_vals0_, tile_vals1_, records_, image_, blend_mode_,
                counters_, sticky_, stream_);
  GSR_CUDA(cudaEventRecord(ev_[6], stream_));
  GSR_CUDA(cudaGetLastError());
  GSR_CUDA(cudaMemcpyAsync(counters_host_, counters_, sizeof(FrameCounters),
                           cudaMemcpyDeviceToHost, stream_));
}

void Renderer::run_frame(const FrameParams &p) {
  enqueue_frame(p);
  GSR_CUDA(cudaStreamSynchronize(stream_));
}

void Renderer::prepare_frame() {
  GSR_CUDA(cudaSetDevice(device_));
  ensure_scene_workspace();
  ensure_image_workspace();
  if (key_cap_ == 0)
    ensure_key_workspace(std::min<uint64_t>(std::max<uint64_t>(16ull * scene_->n, 1u << 20),
                                            kMaxSortItems));
  if (debug_) {
    if (projected_.size() < sizeof(ProjectedDev) * std::max<uint32_t>(scene_->n, 1))
      projected_.reset(sizeof(ProjectedDev) * std::max<uint32_t>(scene_->n, 1));
    if (debug_pairs_.size() < 8 * key_cap_) debug_pairs_.reset(8 * key_cap_);
  }
}

void Renderer::collect(FrameResult &r) {
  float t[kPhaseCount];
  for (int k = 0; k < kPhaseCount; ++k) GSR_CUDA(cudaEventElapsedTime(&t[k], ev_[k], ev_[k + 1]));
  for (int k = 0; k < kPhaseCount; ++k) r.phase_ms[k] = t[k];
  r.preprocess_ms = t[kPhasePreprocess];
  r.sort_ms = t[kPhaseDepthSort] + t[kPhaseEmit] + t[kPhaseTileSort] + t[kPhaseRanges];
  r.raster_ms = t[kPhaseRaster];
  r.visible = counters_host_->visible;
  r.drawn = counters_host_->drawn;
  r.keys = counters_host_->keys;
}

FrameResult Renderer::render(const GsplatCamera &cam) {
  auto t0 = std::chrono::steady_clock::now();
  if (!camera_valid(cam)) throw Error(Code::InvalidArgument, "invalid camera");
  if (!scene_) throw Error(Code::SceneNotLoaded, "scene not loaded");
  prepare_frame();
  const FrameParams p = make_frame_params(cam, width_, height_, tile_, scene_->sh_degree, scene_->n);
  FrameResult r;
  for (;;) {
    run_frame(p);
    if (counters_host_->error)
      throw Error(Code::Internal, "device wait limit reached in a look-back scan (error bits " +
                                      std::to_string(counters_host_->error) + ")");
    if (!counters_host_->overflow) break;
    // Grow the pair buffers to the exact need plus headroom and run again.
    uint64_t need = counters_host_->keys;
    if (need > kMaxSortItems)
      throw Error(Code::Unsupported, "tile pair count " + std::to_string(need) +
                                         " exceeds the renderer's limit of 2^30 - 1");
    ensure_key_workspace(std::min<uint64_t>(need + need / 4 + 1024, kMaxSortItems));
    if (debug_) debug_pairs_.reset(8 * key_cap_);
    ++r.reruns;
  }
  GSR_CUDA(cudaMemsetAsync(sticky_, 0, 4, stream_));
  collect(r);
  r.frame_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  last_ = r;
  has_frame_ = true;
  return r;
}

void Renderer::render_async(const GsplatCamera &cam) {
  if (!camera_valid(cam)) throw Error(Code::InvalidArgument, "invalid camera");
  if (!scene_) throw Error(Code::SceneNotLoaded, "scene not loaded");
  prepare_frame();
  enqueue_frame(make_frame_params(cam, width_, height_, tile_, scene_->sh_degree, scene_->n));
  has_frame_ = true;
}

void Renderer::sync() {
  GSR_CUDA(cudaSetDevice(device_));
  uint32_t sticky = 0;
  GSR_CUDA(cudaMemcpyAsync(&sticky, sticky_, 4, cudaMemcpyDeviceToHost, stream_));
  GSR_CUDA(cudaMemsetAsync(sticky_, 0, 4, stream_));
  GSR_CUDA(cudaStreamSynchronize(stream_));
  if (!has_frame_) return;
  FrameResult r;
  collect(r);
  last_ = r;
  if (sticky & 0x7fffffffu)
    throw Error(Code::Internal, "device wait limit reached in a look-back scan");
  if (sticky & 0x80000000u) {
    has_frame_ = false;
    throw Error(Code::Internal,
                "an enqueued frame overflowed its tile-pair buffers; render it synchronously "
                "once to size them");
  }
}

void Renderer::readback_rgba8(uint8_t *out, uint64_t len) {
  const uint64_t need = 4ull * width_ * height_;
  if (!has_frame_) throw Error(Code::InvalidArgument, "no rendered frame to read back");
  if (len < need) throw Error(Code::InvalidArgument, "output buffer too small for the RGBA8 image");
  GSR_CUDA(cudaSetDevice(device_));
  GSR_CUDA(cudaMemcpyAsync(out, image_, need, cudaMemcpyDeviceToHost, stream_));
  GSR_CUDA(cudaStreamSynchronize(stream_));
}

SortPlan Renderer::read_plan(int which) {
  SortPlan plan;
  GSR_CUDA(cudaMemcpyAsync(&plan, which == 0 ? depth_plan_ : tile_plan_, sizeof(SortPlan),
                           cudaMemcpyDeviceToHost, stream_));
  GSR_CUDA(cudaStreamSynchronize(stream_));
  return plan;
}

std::vector<uint32_t> Renderer::debug_order() {
  if (!has_frame_) throw Error(Code::InvalidArgument, "no rendered frame");
  GSR_CUDA(cudaSetDevice(device_));
  SortPlan plan = read_plan(0);
  std::vector<uint32_t> out(last_.visible);
  if (!out.empty())
    GSR_CUDA(cudaMemcpy(out.data(), plan.final_buffer == 0 ? vis_vals0_ : vis_vals1_,
                        4 * out.size(), cudaMemcpyDeviceToHost));
  return out;
}

std::vector<ProjectedDev> Renderer::debug_projected() {
  if (!has_frame_ || !debug_ || !projected_.get())
    throw Error(Code::InvalidArgument, "debug taps were not enabled for the last frame");
  GSR_CUDA(cudaSetDevice(device_));
  std::vector<ProjectedDev> out(scene_->n);
  if (!out.empty())
    GSR_CUDA(cudaMemcpy(out.data(), projected_.get(), sizeof(ProjectedDev) * out.size(),
                        cudaMemcpyDeviceToHost));
  return out;
}

void Renderer::debug_tile_pairs(std::vector<uint32_t> &tiles, std::vector<uint32_t> &ids) {
  if (!has_frame_ || !debug_ || !debug_pairs_.get())
    throw Error(Code::InvalidArgument, "debug taps were not enabled for the last frame");
  GSR_CUDA(cudaSetDevice(device_));
  const uint64_t k = std::min<uint64_t>(last_.keys, key_cap_);
  tiles.resize(k);
  ids.resize(k);
  if (k) {
    GSR_CUDA(cudaMemcpy(tiles.data(), debug_pairs_.get(), 4 * k, cudaMemcpyDeviceToHost));
    GSR_CUDA(cudaMemcpy(ids.data(), debug_pairs_.as<uint32_t>(4 * key_cap_), 4 * k,
                        cudaMemcpyDeviceToHost));
  }
}

void Renderer::debug_tile_ranges(std::vector<uint32_t> &ranges, std::vector<uint32_t> &ids) {
  if (!has_frame_) throw Error(Code::InvalidArgument, "no rendered frame");
  GSR_CUDA(cudaSetDevice(device_));
  SortPlan plan = read_plan(1);
  const uint32_t tiles_x = (width_ + tile_ - 1) / tile_, tiles_y = (height_ + tile_ - 1) / tile_;
  ranges.resize(2ull * tiles_x * tiles_y);
  GSR_CUDA(cudaMemcpy(ranges.data(), ranges_, 4 * ranges.size(), cudaMemcpyDeviceToHost));
  const uint64_t k = std::min<uint64_t>(last_.keys, key_cap_);
  ids.resize(k);
  if (k)
    GSR_CUDA(cudaMemcpy(ids.data(), plan.final_buffer == 0 ? tile_vals0_ : tile_vals1_, 4 * k,
                        cudaMemcpyDeviceToHost));
}

}  // namespace gsr
