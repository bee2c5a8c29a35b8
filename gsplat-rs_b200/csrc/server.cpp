// Served rendering with continuous batching (host orchestration only).

#include "server.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "cuda_check.h"
#include "kernels.h"
#include "renderer.h"

namespace gsr {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// ---- PinnedPool --------------------------------------------------------------

PinnedPool::PinnedPool() : thread_([this] { grower(); }) {}

PinnedPool::~PinnedPool() {
  {
    std::lock_guard<std::mutex> g(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  thread_.join();
  for (uint8_t *p : slabs_) cudaFreeHost(p);
}

// One slab of buffers of `bytes` (portable pinned memory: any device's
// context can copy into it). The buffers go to the free list, except the
// first when the caller keeps it.
uint8_t *PinnedPool::allocate_slab(uint64_t bytes, bool keep_one) {
  const uint64_t stride = (bytes + 255) & ~uint64_t(255);
  {
    // a reserved slab first, when the size fits one
    std::lock_guard<std::mutex> g(mu_);
    const uint64_t fit = std::min<uint64_t>(64, kSlabBytes / stride);
    if (fit > 0 && !raw_.empty()) {
      uint8_t *slab = raw_.back();
      raw_.pop_back();
      auto &list = free_[bytes];
      for (uint64_t k = keep_one ? 1 : 0; k < fit; ++k) list.push_back(slab + k * stride);
      return keep_one ? slab : nullptr;
    }
  }
  const uint64_t count = std::max<uint64_t>(1, std::min<uint64_t>(64, (kSlabBytes + stride - 1) / stride));
  void *slab = nullptr;
  GSR_CUDA(cudaHostAlloc(&slab, stride * count, cudaHostAllocPortable));
  std::lock_guard<std::mutex> g(mu_);
  slabs_.push_back((uint8_t *)slab);
  auto &list = free_[bytes];
  for (uint64_t k = keep_one ? 1 : 0; k < count; ++k) list.push_back((uint8_t *)slab + k * stride);
  return keep_one ? (uint8_t *)slab : nullptr;
}

void PinnedPool::grower() {
  std::unique_lock<std::mutex> lk(mu_);
  for (;;) {
    cv_.wait(lk, [&] { return stop_ || !wanted_.empty(); });
    if (stop_) return;
    const uint64_t bytes = wanted_.front();
    wanted_.pop_front();
    const int device = device_;
    lk.unlock();
    bool ok = true;
    try {
      if (device >= 0) GSR_CUDA(cudaSetDevice(device));
      allocate_slab(bytes, false);
    } catch (const Error &) {
      ok = false;  // out of pinned memory: take() allocates (and reports) on demand
    }
    lk.lock();
    // still short of the low-water mark (demand outran the slab): go on
    if (ok && !stop_ && free_[bytes].size() < kLowWater) wanted_.push_back(bytes);
    else growing_[bytes] = false;
  }
}

uint8_t *PinnedPool::take(uint64_t bytes) {
  {
    std::lock_guard<std::mutex> g(mu_);
    auto &list = free_[bytes];
    if (!list.empty()) {
      uint8_t *p = list.back();
      list.pop_back();
      if (list.size() < kLowWater && !growing_[bytes]) {
        growing_[bytes] = true;
        wanted_.push_back(bytes);
        cv_.notify_one();
      }
      return p;
    }
  }
  // No free buffer of this size: allocate a slab here and keep one buffer.
  const double t0 = now_ms();
  uint8_t *p = allocate_slab(bytes, true);
  const double t1 = now_ms();
  std::lock_guard<std::mutex> g(mu_);
  wait_ms_ += t1 - t0;
  return p;
}

void PinnedPool::reserve(uint64_t bytes) {
  for (uint64_t k = 0; k < (bytes + kSlabBytes - 1) / kSlabBytes; ++k) {
    void *slab = nullptr;
    GSR_CUDA(cudaHostAlloc(&slab, kSlabBytes, cudaHostAllocPortable));
    std::lock_guard<std::mutex> g(mu_);
    slabs_.push_back((uint8_t *)slab);
    raw_.push_back((uint8_t *)slab);
  }
}

void PinnedPool::set_device(int device) {
  std::lock_guard<std::mutex> g(mu_);
  device_ = device;
}

void PinnedPool::allocations(uint64_t &slabs, double &wait_ms) {
  std::lock_guard<std::mutex> g(mu_);
  slabs = slabs_.size();
  wait_ms = wait_ms_;
}

void PinnedPool::give(uint8_t *p, uint64_t bytes) {
  if (!p) return;
  std::lock_guard<std::mutex> g(mu_);
  free_[bytes].push_back(p);
}

// ---- Server ------------------------------------------------------------------

Server::Server(const ServeConfig &cfg) : cfg_(cfg), scenes_(cfg.scene_budget) {
  if (cfg.lanes == 0 || cfg.lanes > 8) throw Error(Code::InvalidArgument, "lanes must be 1..8");
  if (cfg.max_views == 0 || cfg.max_views > kMaxViewsPerLaunch)
    throw Error(Code::InvalidArgument, "max_views must be 1..1024");
  if (cfg.tile != 8 && cfg.tile != 16) throw Error(Code::InvalidArgument, "tile size must be 8 or 16");
  device_ = require_b200();
  pool_.set_device(device_);
  pool_.reserve((uint64_t)cfg.result_pool_mib << 20);
  GSR_CUDA(cudaStreamCreateWithFlags(&upload_stream_, cudaStreamNonBlocking));
  for (uint32_t k = 0; k < cfg.lanes; ++k) {
    auto ls = std::make_unique<LaneState>();
    ls->lane = std::make_unique<Lane>(device_);
    ls->lane->pipe().set_tile(cfg.tile);
    RasterConfig rc = cfg.raster;
    if (rc.chunk == 0) rc.chunk = cfg.tile * cfg.tile;
    ls->lane->pipe().set_raster_config(rc);
    ls->server = this;
    lanes_.push_back(std::move(ls));
  }
  thread_ = std::thread([this] { loop(); });
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> g(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  if (thread_.joinable()) thread_.join();
  cudaSetDevice(device_);
  for (auto &ls : lanes_) cudaStreamSynchronize(ls->lane->stream());
  for (auto &kv : requests_) pool_.give(kv.second.result, kv.second.bytes);
  lanes_.clear();
  if (upload_stream_) cudaStreamDestroy(upload_stream_);
}

uint32_t Server::add_scene(const HostScene &s) {
  GSR_CUDA(cudaSetDevice(device_));
  if (scene_validate(s) != Code::Ok) throw Error(Code::InvalidArgument, "invalid scene buffers");
  {
    std::lock_guard<std::mutex> g(mu_);
    scenes_.check_budget(scene_device_bytes(s));
  }
  // Upload without the lock (lane callbacks take it); the store's list is
  // only touched under the lock, where the scheduler reads it too.
  auto sc = upload_scene(s, upload_stream_);
  std::lock_guard<std::mutex> g(mu_);
  return scenes_.insert(std::move(sc));
}

uint32_t Server::add_scene_packed(const HostScene &s) {
  GSR_CUDA(cudaSetDevice(device_));
  if (scene_validate(s) != Code::Ok) throw Error(Code::InvalidArgument, "invalid scene buffers");
  {
    std::lock_guard<std::mutex> g(mu_);
    scenes_.check_budget(packed_device_bytes(s.size(), s.sh_degree));
  }
  auto sc = upload_scene_packed(s, upload_stream_);
  std::lock_guard<std::mutex> g(mu_);
  return scenes_.insert(std::move(sc));
}

uint32_t Server::add_scene_path(const std::string &path) {
  GSR_CUDA(cudaSetDevice(device_));
  auto admit = [this](uint64_t bytes) {
    std::lock_guard<std::mutex> g(mu_);
    scenes_.check_budget(bytes);
  };
  auto sc = load_scene_file(path, upload_stream_, admit);
  std::lock_guard<std::mutex> g(mu_);
  return scenes_.insert(std::move(sc));
}

uint64_t Server::submit(const BatchView &v) {
  std::lock_guard<std::mutex> g(mu_);
  if (stop_) throw Error(Code::Internal, "server is stopping");
  std::vector<ViewSpec> spec;
  std::vector<uint64_t> base;
  make_view_specs(scenes_, &v, 1, spec, base);  // validates scene id, camera, size
  Request r;
  r.id = next_id_++;
  r.view = v;
  r.t_submit = now_ms();
  if (first_submit_ < 0) first_submit_ = r.t_submit;
  ++submitted_;
  const uint64_t id = r.id;
  requests_.emplace(id, std::move(r));
  queue_.push_back(id);
  cv_.notify_all();
  return id;
}

RequestInfo Server::poll(uint64_t id) {
  std::lock_guard<std::mutex> g(mu_);
  auto it = requests_.find(id);
  if (it == requests_.end()) throw Error(Code::InvalidArgument, "unknown request " + std::to_string(id));
  return it->second.info;
}

RequestInfo Server::wait(uint64_t id, uint32_t timeout_ms) {
  std::unique_lock<std::mutex> lk(mu_);
  auto finished = [&] {
    auto it = requests_.find(id);
    return it == requests_.end() || it->second.info.status == RequestStatus::Done ||
           it->second.info.status == RequestStatus::Failed;
  };
  done_cv_.wait_for(lk, std::chrono::milliseconds(timeout_ms), finished);
  auto it = requests_.find(id);
  if (it == requests_.end()) throw Error(Code::InvalidArgument, "unknown request " + std::to_string(id));
  return it->second.info;
}

void Server::read_rgba8(uint64_t id, uint8_t *out, uint64_t len) {
  std::lock_guard<std::mutex> g(mu_);
  auto it = requests_.find(id);
  if (it == requests_.end()) throw Error(Code::InvalidArgument, "unknown request " + std::to_string(id));
  const Request &r = it->second;
  if (r.info.status != RequestStatus::Done)
    throw Error(Code::InvalidArgument, "request " + std::to_string(id) + " has no finished image");
  if (len < r.bytes) throw Error(Code::InvalidArgument, "output buffer too small for the RGBA8 image");
  std::memcpy(out, r.result, r.bytes);
}

void Server::release(uint64_t id) {
  std::lock_guard<std::mutex> g(mu_);
  auto it = requests_.find(id);
  if (it == requests_.end()) throw Error(Code::InvalidArgument, "unknown request " + std::to_string(id));
  if (it->second.info.status == RequestStatus::Queued || it->second.info.status == RequestStatus::Running)
    throw Error(Code::InvalidArgument, "request " + std::to_string(id) + " is still in flight");
  pool_.give(it->second.result, it->second.bytes);
  requests_.erase(it);
}

ServeStats Server::stats() {
  std::lock_guard<std::mutex> g(mu_);
  ServeStats s;
  s.submitted = submitted_;
  s.completed = latencies_.size();
  s.failed = failed_;
  s.shed = shed_;
  s.batches = batches_;
  s.reruns = reruns_;
  s.peak_admitted_bytes = peak_admitted_;
  if (!latencies_.empty()) {
    std::vector<double> l = latencies_;
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) {
      // nearest-rank percentile
      size_t k = (size_t)std::ceil(q * l.size());
      return l[std::min(l.size() - 1, k ? k - 1 : 0)];
    };
    s.p50_ms = pct(0.50);
    s.p99_ms = pct(0.99);
    double sum = 0;
    for (double x : l) sum += x;
    s.mean_ms = sum / l.size();
    s.max_ms = l.back();
    if (last_done_ > first_submit_ && first_submit_ >= 0)
      s.views_per_s = 1000.0 * l.size() / (last_done_ - first_submit_);
  }
  s.mean_batch_views = batches_ ? (double)batch_views_ / batches_ : 0.0;
  s.device_ms = device_ms_;
  s.launch_ms = launch_ms_;
  s.retire_ms = retire_ms_;
  uint64_t captures = 0, slabs = 0, regrowths = 0;
  double capture_ms = 0, alloc_ms = 0, regrowth_ms = 0;
  host_costs(captures, capture_ms, slabs, alloc_ms, regrowths, regrowth_ms);
  s.workspace_regrowths = regrowths - base_regrowths_;
  s.regrowth_ms = regrowth_ms - base_regrowth_ms_;
  s.graph_captures = captures - base_captures_;
  s.capture_ms = capture_ms - base_capture_ms_;
  s.pinned_slabs = slabs - base_slabs_;
  s.pinned_alloc_ms = alloc_ms - base_alloc_ms_;
  return s;
}

void Server::host_costs(uint64_t &captures, double &capture_ms, uint64_t &slabs,
                        double &alloc_ms, uint64_t &regrowths, double &regrowth_ms) {
  captures = 0;
  capture_ms = 0;
  regrowths = 0;
  regrowth_ms = 0;
  for (auto &ls : lanes_) {
    captures += ls->lane->pipe().graph_captures();
    capture_ms += ls->lane->pipe().capture_ms();
    regrowths += ls->lane->pipe().workspace_regrowths();
    regrowth_ms += ls->lane->pipe().regrowth_ms();
  }
  pool_.allocations(slabs, alloc_ms);
}

void Server::reset_stats() {
  std::lock_guard<std::mutex> g(mu_);
  latencies_.clear();
  submitted_ = failed_ = batches_ = batch_views_ = reruns_ = shed_ = 0;
  peak_admitted_ = 0;
  first_submit_ = -1;
  last_done_ = 0;
  device_ms_ = launch_ms_ = retire_ms_ = 0;
  host_costs(base_captures_, base_capture_ms_, base_slabs_, base_alloc_ms_, base_regrowths_,
             base_regrowth_ms_);
}

uint64_t Server::view_bytes(const ViewSpec &s, uint64_t pairs) const {
  // pair keys and values, double-buffered, plus sort scratch; splat
  // workspace (keys, ids, rect, record, sort scratch); the image
  return pairs * 17 + (uint64_t)s.scene->n * 80 + 4ull * s.width * s.height;
}

void Server::on_lane_done(void *arg) {
  auto *ls = static_cast<LaneState *>(arg);
  ls->t_complete.store(now_ms());
  {
    std::lock_guard<std::mutex> g(ls->server->mu_);
    ls->completed.store(true);
  }
  ls->server->cv_.notify_all();
}

bool Server::launch(LaneState &ls, std::unique_lock<std::mutex> &lk) {
  // Shed the requests that have waited longer than the queueing bound (the
  // queue is in arrival order, so they are at its front).
  if (cfg_.max_queue_ms) {
    const double now = now_ms();
    bool shed = false;
    while (!queue_.empty()) {
      Request &r = requests_.at(queue_.front());
      if (now - r.t_submit <= (double)cfg_.max_queue_ms) break;
      queue_.pop_front();
      r.info.status = RequestStatus::Failed;
      r.info.error_code = (int32_t)Code::Unsupported;
      r.info.error = "request shed: queued longer than the server's max_queue_ms (" +
                     std::to_string(cfg_.max_queue_ms) + " ms)";
      r.info.queue_ms = (float)(now - r.t_submit);
      ++failed_;
      ++shed_;
      shed = true;
    }
    if (shed) done_cv_.notify_all();
  }
  if (queue_.empty()) return false;
  const uint64_t lane_budget = cfg_.work_budget / cfg_.lanes;
  ls.ids.clear();
  ls.specs.clear();
  ls.bases.clear();
  std::vector<uint64_t> predicted;
  uint64_t bytes = 0, pixels = 0;
  // Admit in arrival order while the batch fits the lane's budget and view limit.
  while (!queue_.empty() && ls.ids.size() < cfg_.max_views) {
    Request &r = requests_.at(queue_.front());
    const ViewSpec spec{&scenes_.get(r.view.scene), r.view.camera, r.view.width, r.view.height};
    const uint64_t pred = predictor_.predict(r.view.scene, spec.scene->n, spec.width, spec.height, cfg_.tile);
    const uint64_t b = view_bytes(spec, pred);
    if (!ls.ids.empty() && bytes + b > lane_budget) break;
    queue_.pop_front();
    ls.ids.push_back(r.id);
    ls.specs.push_back(spec);
    ls.bases.push_back(pixels);
    predicted.push_back(pred);
    pixels += (uint64_t)spec.width * spec.height;
    bytes += b;
    r.info.status = RequestStatus::Running;
    r.t_launch = now_ms();
  }
  // Requests of one scene run next to each other (one scene read per view
  // set in the preprocess kernel); image offsets follow the new order.
  {
    const size_t m = ls.ids.size();
    std::vector<size_t> order(m);
    for (size_t k = 0; k < m; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
      return requests_.at(ls.ids[a]).view.scene < requests_.at(ls.ids[b]).view.scene;
    });
    std::vector<uint64_t> ids(m), pred(m), bases(m);
    std::vector<ViewSpec> specs(m);
    uint64_t px = 0;
    for (size_t k = 0; k < m; ++k) {
      ids[k] = ls.ids[order[k]];
      specs[k] = ls.specs[order[k]];
      pred[k] = predicted[order[k]];
      bases[k] = px;
      px += (uint64_t)specs[k].width * specs[k].height;
    }
    ls.ids.swap(ids);
    ls.specs.swap(specs);
    ls.bases.swap(bases);
    predicted.swap(pred);
  }
  ls.admitted_bytes = bytes;
  peak_admitted_ = std::max<uint64_t>(peak_admitted_, bytes);
  for (auto &o : lanes_)
    if (o.get() != &ls && o->busy) peak_admitted_ = std::max(peak_admitted_, bytes + o->admitted_bytes);
  GroupLimits limits;
  limits.max_views = cfg_.max_views;
  ls.groups = plan_groups(ls.specs, predicted, cfg_.tile, limits);
  uint64_t reserve = 0;
  for (const auto &g : ls.groups) reserve = std::max(reserve, g.predicted_pairs);
  ls.dst.assign(ls.ids.size(), nullptr);
  ls.busy = true;
  ls.completed.store(false);
  lk.unlock();
  const double t_enqueue = now_ms();
  try {
    for (size_t k = 0; k < ls.ids.size(); ++k)
      ls.dst[k] = pool_.take(4ull * ls.specs[k].width * ls.specs[k].height);
    ls.lane->enqueue(ls.specs, ls.bases, pixels, ls.groups, reserve);
    const uint32_t *img = ls.lane->images();
    for (size_t k = 0; k < ls.ids.size(); ++k)
      GSR_CUDA(cudaMemcpyAsync(ls.dst[k], img + ls.bases[k], 4ull * ls.specs[k].width * ls.specs[k].height,
                               cudaMemcpyDeviceToHost, ls.lane->stream()));
    GSR_CUDA(cudaLaunchHostFunc(ls.lane->stream(), &Server::on_lane_done, &ls));
  } catch (const Error &e) {
    lk.lock();
    for (size_t k = 0; k < ls.ids.size(); ++k) {
      Request &r = requests_.at(ls.ids[k]);
      r.info.status = RequestStatus::Failed;
      r.info.error_code = (int32_t)e.code;
      r.info.error = e.what();
      r.result = ls.dst[k];
      r.bytes = ls.dst[k] ? 4ull * ls.specs[k].width * ls.specs[k].height : 0;
      ++failed_;
    }
    ls.busy = false;
    done_cv_.notify_all();
    return true;
  }
  const double t_enqueued = now_ms();
  lk.lock();
  ++batches_;
  batch_views_ += ls.ids.size();
  launch_ms_ += t_enqueued - t_enqueue;
  return true;
}

void Server::retire(LaneState &ls, std::unique_lock<std::mutex> &lk) {
  const double t_done = ls.t_complete.load();
  lk.unlock();
  const double t_retire = now_ms();
  uint32_t reruns = 0;
  float batch_device_ms = 0;
  std::string err;
  int32_t code = 0;
  try {
    reruns = ls.lane->finish(ls.specs, ls.bases, ls.groups);
    batch_device_ms = ls.lane->device_ms();
    if (reruns) {
      // images were re-rendered: copy them again
      const uint32_t *img = ls.lane->images();
      for (size_t k = 0; k < ls.ids.size(); ++k)
        GSR_CUDA(cudaMemcpyAsync(ls.dst[k], img + ls.bases[k],
                                 4ull * ls.specs[k].width * ls.specs[k].height,
                                 cudaMemcpyDeviceToHost, ls.lane->stream()));
      GSR_CUDA(cudaStreamSynchronize(ls.lane->stream()));
    }
  } catch (const Error &e) {
    err = e.what();
    code = (int32_t)e.code;
  }
  const double t_final = reruns ? now_ms() : t_done;
  const double t_retired = now_ms();
  lk.lock();
  device_ms_ += batch_device_ms;
  retire_ms_ += t_retired - t_retire;
  for (size_t k = 0; k < ls.ids.size(); ++k) {
    Request &r = requests_.at(ls.ids[k]);
    r.result = ls.dst[k];
    r.bytes = 4ull * ls.specs[k].width * ls.specs[k].height;
    r.info.batch_views = (uint32_t)ls.ids.size();
    r.info.queue_ms = (float)(r.t_launch - r.t_submit);
    if (code) {
      r.info.status = RequestStatus::Failed;
      r.info.error_code = code;
      r.info.error = err;
      ++failed_;
      continue;
    }
    r.info.counters = ls.lane->view_counters()[k];
    r.t_done = t_final;
    r.info.latency_ms = (float)(t_final - r.t_submit);
    r.info.status = RequestStatus::Done;
    latencies_.push_back(t_final - r.t_submit);
    predictor_.observe(r.view.scene, ls.specs[k].scene->n, ls.specs[k].width, ls.specs[k].height,
                       cfg_.tile, r.info.counters.pairs);
  }
  last_done_ = std::max(last_done_, t_final);
  reruns_ += reruns;
  ls.busy = false;
  ls.completed.store(false);
  done_cv_.notify_all();
}

void Server::loop() {
  cudaSetDevice(device_);
  std::unique_lock<std::mutex> lk(mu_);
  while (true) {
    bool progressed = false;
    for (auto &ls : lanes_)
      if (ls->busy && ls->completed.load()) {
        retire(*ls, lk);
        progressed = true;
      }
    if (stop_) {
      bool any_busy = false;
      for (auto &ls : lanes_) any_busy |= ls->busy;
      if (!any_busy) break;
    } else {
      for (auto &ls : lanes_)
        if (!ls->busy && !queue_.empty()) progressed |= launch(*ls, lk);
    }
    if (!progressed) cv_.wait(lk);
  }
  // fail whatever is still queued
  for (uint64_t id : queue_) {
    Request &r = requests_.at(id);
    r.info.status = RequestStatus::Failed;
    r.info.error_code = (int32_t)Code::Internal;
    r.info.error = "server stopped";
  }
  queue_.clear();
  done_cv_.notify_all();
}

}  // namespace gsr
