// Batched frames over resident scenes (host orchestration only).

#include "batch.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "cuda_check.h"
#include "kernels.h"
#include "renderer.h"

namespace gsr {

namespace {
constexpr double kDefaultPairsPerSplatPerMpx = 8.0;
constexpr double kHeadroom = 1.25;
constexpr uint64_t kMaxPairs = (1u << 30) - 1;
}  // namespace

// ---- SceneStore ------------------------------------------------------------

void SceneStore::check_budget(uint64_t bytes) const {
  if (bytes_ + bytes > budget_)
    throw Error(Code::Unsupported, "scene memory budget exceeded: " + std::to_string(bytes_ + bytes) +
                                       " > " + std::to_string(budget_) + " bytes");
}

uint32_t SceneStore::add(const HostScene &s, cudaStream_t stream) {
  if (scene_validate(s) != Code::Ok) throw Error(Code::InvalidArgument, "invalid scene buffers");
  check_budget(scene_device_bytes(s));
  return insert(upload_scene(s, stream));
}

uint32_t SceneStore::add_packed(const HostScene &s, cudaStream_t stream) {
  if (scene_validate(s) != Code::Ok) throw Error(Code::InvalidArgument, "invalid scene buffers");
  check_budget(packed_device_bytes(s.size(), s.sh_degree));
  return insert(upload_scene_packed(s, stream));
}

uint32_t SceneStore::add_path(const std::string &path, cudaStream_t stream) {
  return insert(load_scene_file(path, stream, [this](uint64_t bytes) { check_budget(bytes); }));
}

uint32_t SceneStore::insert(std::unique_ptr<DeviceScene> sc) {
  check_budget(sc->bytes());
  bytes_ += sc->bytes();
  scenes_.push_back(std::move(sc));
  return (uint32_t)scenes_.size() - 1;
}

const DeviceScene &SceneStore::get(uint32_t id) const {
  if (id >= scenes_.size()) throw Error(Code::InvalidArgument, "unknown scene id " + std::to_string(id));
  return *scenes_[id];
}

// ---- PairPredictor ---------------------------------------------------------

uint64_t PairPredictor::predict(uint32_t scene, uint32_t n, uint32_t w, uint32_t h,
                                uint32_t tile) const {
  const double mpx = (double)w * h / 1e6;
  double ratio;
  auto it = ratio_.find(Key{scene, w, h, tile});
  if (it != ratio_.end()) {
    ratio = it->second;
  } else {
    auto js = scene_ratio_px_.find(scene);
    ratio = (js != scene_ratio_px_.end() ? js->second : kDefaultPairsPerSplatPerMpx) *
            std::max(mpx, 0.05) * (tile == 8 ? 4.0 : 1.0);
  }
  const double p = std::ceil(ratio * kHeadroom * n) + 64;
  return (uint64_t)std::min<double>(p, (double)kMaxPairs);
}

void PairPredictor::observe(uint32_t scene, uint32_t n, uint32_t w, uint32_t h, uint32_t tile,
                            uint64_t pairs) {
  if (n == 0) return;
  const double r = (double)pairs / n;
  double &cur = ratio_[Key{scene, w, h, tile}];
  cur = std::max(cur, r);
  const double mpx = std::max((double)w * h / 1e6, 0.05) * (tile == 8 ? 4.0 : 1.0);
  double &px = scene_ratio_px_[scene];
  px = std::max(px, r / mpx);
}

// ---- grouping ----------------------------------------------------------------

std::vector<ViewGroup> plan_groups(const std::vector<ViewSpec> &views,
                                   const std::vector<uint64_t> &predicted, uint32_t tile,
                                   const GroupLimits &limits) {
  std::vector<ViewGroup> groups;
  ViewGroup cur{0, 0, 0};
  uint64_t splats = 0, tiles = 0;
  const uint32_t max_views = std::min<uint32_t>(std::max(limits.max_views, 1u), kMaxViewsPerLaunch);
  for (uint32_t v = 0; v < views.size(); ++v) {
    const uint64_t n = views[v].scene->n;
    const uint64_t t = (uint64_t)((views[v].width + tile - 1) / tile) * ((views[v].height + tile - 1) / tile);
    const bool fits = cur.count < max_views && splats + n <= std::min<uint64_t>(limits.max_splats, kMaxPairs) &&
                      tiles + t <= std::min<uint64_t>(limits.max_tiles, 1u << 24) &&
                      cur.predicted_pairs + predicted[v] <= std::min<uint64_t>(limits.max_pairs, kMaxPairs);
    if (cur.count && !fits) {
      groups.push_back(cur);
      cur = ViewGroup{v, 0, 0};
      splats = tiles = 0;
    }
    cur.count++;
    cur.predicted_pairs += predicted[v];
    splats += n;
    tiles += t;
  }
  if (cur.count) groups.push_back(cur);
  return groups;
}

uint64_t make_view_specs(const SceneStore &store, const BatchView *views, uint32_t count,
                         std::vector<ViewSpec> &specs, std::vector<uint64_t> &bases) {
  specs.resize(count);
  bases.resize(count);
  uint64_t pixels = 0;
  for (uint32_t v = 0; v < count; ++v) {
    const BatchView &b = views[v];
    if (!camera_valid(b.camera)) throw Error(Code::InvalidArgument, "invalid camera for view " + std::to_string(v));
    if (b.width == 0 || b.height == 0)
      throw Error(Code::InvalidArgument, "invalid image size for view " + std::to_string(v));
    if (b.width > kMaxImageDimension || b.height > kMaxImageDimension)
      throw Error(Code::Unsupported, "requested dimensions exceed the maximum of 16384");
    specs[v] = ViewSpec{&store.get(b.scene), b.camera, b.width, b.height};
    bases[v] = pixels;
    pixels += (uint64_t)b.width * b.height;
  }
  return pixels;
}

// ---- PinnedArray / Lane ------------------------------------------------------

template <typename T>
T *PinnedArray<T>::ensure(size_t n) {
  if (n <= cap_ && p_) return p_;
  if (p_) cudaFreeHost(p_);
  p_ = nullptr;
  cap_ = 0;
  const size_t cap = std::max<size_t>(std::max<size_t>(n, 64), 2 * cap_);
  GSR_CUDA(cudaMallocHost(&p_, sizeof(T) * cap));
  std::memset(p_, 0, sizeof(T) * cap);
  cap_ = cap;
  return p_;
}
template class PinnedArray<ViewCounters>;
template class PinnedArray<FrameCounters>;

Lane::Lane(int device) : device_(device) {
  GSR_CUDA(cudaSetDevice(device_));
  GSR_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  GSR_CUDA(cudaEventCreate(&start_));
  GSR_CUDA(cudaEventCreate(&end_));
  pipe_ = std::make_unique<Pipeline>(device_, stream_);
  // pinned once for a full launch of views (growing them later frees pinned
  // memory, which waits for the whole device)
  view_counters_.ensure(kMaxViewsPerLaunch);
  group_counters_.ensure(kMaxViewsPerLaunch);
}

Lane::~Lane() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  pipe_.reset();
  images_.reset(0);
  if (start_) cudaEventDestroy(start_);
  if (end_) cudaEventDestroy(end_);
  if (stream_) cudaStreamDestroy(stream_);
}

void Lane::enqueue(const std::vector<ViewSpec> &views, const std::vector<uint64_t> &bases,
                   uint64_t total_pixels, const std::vector<ViewGroup> &groups, uint64_t reserve,
                   bool one_graph, float *phase_sums) {
  GSR_CUDA(cudaSetDevice(device_));
  const uint64_t need = 4 * std::max<uint64_t>(total_pixels, 1);
  if (images_.size() < need) {
    const auto t_grow = std::chrono::steady_clock::now();
    GSR_CUDA(cudaStreamSynchronize(stream_));
    images_.reset(need + need / 4, stream_);  // stream order: no device-wide wait
    pipe_->note_regrowth(std::chrono::duration<double, std::milli>(
                             std::chrono::steady_clock::now() - t_grow).count());
  }
  // pinned sinks: the pointers stay put while sizes fit, so the pipeline's
  // captured graphs keep matching
  if (view_counters_.capacity() < views.size() || group_counters_.capacity() < groups.size()) {
    GSR_CUDA(cudaStreamSynchronize(stream_));  // earlier runs may still write the old arrays
    view_counters_.ensure(views.size());
    group_counters_.ensure(groups.size());
  }
  pipe_->reserve_pairs(std::min<uint64_t>(std::max<uint64_t>(reserve, 1u << 20), kMaxPairs));
  GSR_CUDA(cudaEventRecord(start_, stream_));
  if (one_graph) {
    std::vector<Pipeline::GroupRun> runs(groups.size());
    for (size_t g = 0; g < groups.size(); ++g)
      runs[g] = Pipeline::GroupRun{groups[g].first, groups[g].count,
                                   HostSinks{group_counters_.get() + g,
                                             view_counters_.get() + groups[g].first}};
    pipe_->enqueue_groups(views.data(), images_.as<uint32_t>(), bases.data(), runs);
  } else {
    for (size_t g = 0; g < groups.size(); ++g) {
      const ViewGroup &gr = groups[g];
      HostSinks sinks{group_counters_.get() + g, view_counters_.get() + gr.first};
      pipe_->enqueue(views.data() + gr.first, gr.count, images_.as<uint32_t>(),
                     bases.data() + gr.first, sinks);
      if (phase_sums) {
        GSR_CUDA(cudaStreamSynchronize(stream_));
        float t[kPhaseCount];
        pipe_->phase_times(t);
        for (int k = 0; k < kPhaseCount; ++k) phase_sums[k] += t[k];
      }
    }
  }
  GSR_CUDA(cudaEventRecord(end_, stream_));
}

uint32_t Lane::finish(const std::vector<ViewSpec> &views, const std::vector<uint64_t> &bases,
                      const std::vector<ViewGroup> &groups) {
  GSR_CUDA(cudaSetDevice(device_));
  GSR_CUDA(cudaStreamSynchronize(stream_));
  uint32_t reruns = 0;
  for (size_t g = 0; g < groups.size(); ++g) {
    FrameCounters &fc = group_counters_.get()[g];
    if (fc.error)
      throw Error(Code::Internal, "device wait limit reached in a look-back scan (error bits " +
                                      std::to_string(fc.error) + ")");
    while (fc.overflow) {
      // Too few pair slots for this group: grow to the exact need plus
      // headroom and render the group again.
      const uint64_t need = fc.keys;
      if (need > kMaxPairs)
        throw Error(Code::Unsupported, "tile pair count " + std::to_string(need) +
                                           " of one launch group exceeds 2^30 - 1");
      pipe_->reserve_pairs(std::min<uint64_t>(need + need / 4 + 1024, kMaxPairs));
      const ViewGroup &gr = groups[g];
      HostSinks sinks{&fc, view_counters_.get() + gr.first};
      pipe_->enqueue(views.data() + gr.first, gr.count, images_.as<uint32_t>(),
                     bases.data() + gr.first, sinks);
      GSR_CUDA(cudaEventRecord(end_, stream_));
      GSR_CUDA(cudaStreamSynchronize(stream_));
      ++reruns;
      if (fc.error)
        throw Error(Code::Internal, "device wait limit reached in a look-back scan");
    }
  }
  return reruns;
}

float Lane::device_ms() {
  float ms = 0;
  GSR_CUDA(cudaEventElapsedTime(&ms, start_, end_));
  return ms;
}

bool Lane::done() {
  cudaError_t e = cudaEventQuery(end_);
  if (e == cudaErrorNotReady) return false;
  GSR_CUDA(e);
  return true;
}

// ---- Batch -------------------------------------------------------------------

Batch::Batch() : scenes_(150ull << 30) {
  device_ = require_b200();
  lane_ = std::make_unique<Lane>(device_);
}

Batch::~Batch() { lane_.reset(); }

void Batch::set_tile(uint32_t tile) {
  if (tile != 8 && tile != 16) throw Error(Code::InvalidArgument, "tile size must be 8 or 16");
  tile_ = tile;
  lane_->pipe().set_tile(tile);
}

void Batch::set_blend_mode(uint32_t mode) {
  if (mode > 1) throw Error(Code::InvalidArgument, "unknown blend mode");
  lane_->pipe().set_blend_mode(mode);
}

void Batch::set_limits(const GroupLimits &l) {
  if (l.max_views == 0 || l.max_views > kMaxViewsPerLaunch || l.max_pairs == 0 || l.max_splats == 0 ||
      l.max_tiles == 0)
    throw Error(Code::InvalidArgument, "invalid batch limits");
  limits_ = l;
}

BatchResult Batch::render(const std::vector<BatchView> &in) {
  auto t0 = std::chrono::steady_clock::now();
  if (in.empty()) throw Error(Code::InvalidArgument, "no views to render");
  has_images_ = false;
  // Views of one scene render next to each other, so the pipeline's view
  // sets read each scene once for all of them; results keep the caller's
  // order through pos_.
  const uint32_t n = (uint32_t)in.size();
  std::vector<uint32_t> order(n);
  for (uint32_t v = 0; v < n; ++v) order[v] = v;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return in[a].scene < in[b].scene; });
  std::vector<BatchView> views(n);
  pos_.resize(n);
  for (uint32_t j = 0; j < n; ++j) {
    views[j] = in[order[j]];
    pos_[order[j]] = j;
  }
  const uint64_t pixels = make_view_specs(scenes_, views.data(), n, specs_, bases_);
  std::vector<uint64_t> predicted(n);
  for (uint32_t v = 0; v < n; ++v)
    predicted[v] = predictor_.predict(views[v].scene, specs_[v].scene->n, views[v].width,
                                      views[v].height, tile_);
  groups_ = plan_groups(specs_, predicted, tile_, limits_);
  uint64_t reserve = 0;
  for (const auto &g : groups_) reserve = std::max(reserve, g.predicted_pairs);
  // the whole batch, every launch group, as one CUDA graph (group by group
  // when phase-timed)
  const uint64_t graphs_before = lane_->pipe().batch_graph_launches();
  BatchResult r;
  r.phase_timed = phase_timing_;
  lane_->enqueue(specs_, bases_, pixels, groups_, reserve, !phase_timing_,
                 phase_timing_ ? r.phase_ms : nullptr);
  r.reruns = lane_->finish(specs_, bases_, groups_);
  r.device_ms = lane_->device_ms();
  r.groups = (uint32_t)groups_.size();
  r.launches = r.groups * lane_->pipe().launches_per_run();
  r.graph_launches = (uint32_t)(lane_->pipe().batch_graph_launches() - graphs_before);
  stats_.assign(lane_->view_counters(), lane_->view_counters() + n);
  for (uint32_t v = 0; v < n; ++v) {
    predictor_.observe(views[v].scene, specs_[v].scene->n, views[v].width, views[v].height, tile_,
                       stats_[v].pairs);
    r.pairs += stats_[v].pairs;
  }
  has_images_ = true;
  r.wall_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  last_ = r;
  return r;
}

uint32_t Batch::position(uint32_t view) const {
  if (!has_images_ || view >= pos_.size())
    throw Error(Code::InvalidArgument, "no rendered view " + std::to_string(view));
  return pos_[view];
}

const ViewCounters &Batch::view_stats(uint32_t view) const { return stats_[position(view)]; }

uint32_t Batch::view_group(uint32_t view) const {
  const uint32_t j = position(view);
  for (uint32_t g = 0; g < groups_.size(); ++g)
    if (j >= groups_[g].first && j < groups_[g].first + groups_[g].count) return g;
  throw Error(Code::InvalidArgument, "no rendered view " + std::to_string(view));
}

const uint32_t *Batch::image_device(uint32_t view, uint64_t *bytes) const {
  const uint32_t j = position(view);
  if (bytes) *bytes = 4ull * specs_[j].width * specs_[j].height;
  return lane_->images() + bases_[j];
}

void Batch::readback_rgba8(uint32_t view, uint8_t *out, uint64_t len) {
  uint64_t bytes = 0;
  const uint32_t *src = image_device(view, &bytes);
  if (len < bytes) throw Error(Code::InvalidArgument, "output buffer too small for the RGBA8 image");
  GSR_CUDA(cudaSetDevice(device_));
  GSR_CUDA(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToHost, lane_->stream()));
  GSR_CUDA(cudaStreamSynchronize(lane_->stream()));
}

}  // namespace gsr
