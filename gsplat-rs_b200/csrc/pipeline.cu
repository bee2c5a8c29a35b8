// Host orchestration of the frame pipeline over a list of views (no device
// code in this file).

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>

#include "kernels.h"
#include "cuda_check.h"
#include "pipeline.h"

namespace gsr {

namespace {
inline uint64_t align256(uint64_t v) { return (v + 255) & ~uint64_t(255); }
constexpr uint64_t kMaxSortItems = (1u << 30) - 1;
constexpr uint64_t kInitialPairsPerSplat = 16;
}  // namespace

DeviceBuffer::~DeviceBuffer() { release(); }

void DeviceBuffer::release() {
  if (ptr_) {
    if (ordered_) cudaFreeAsync(ptr_, stream_);
    else cudaFree(ptr_);
  }
  ptr_ = nullptr;
  bytes_ = 0;
  ordered_ = false;
  stream_ = nullptr;
}

void DeviceBuffer::reset(uint64_t bytes, cudaStream_t stream) {
  release();
  if (bytes == 0) return;
  cudaError_t e = cudaMallocAsync(&ptr_, bytes, stream);
  if (e != cudaSuccess) {
    ptr_ = nullptr;
    cudaGetLastError();
    throw Error(Code::Internal, "device allocation of " + std::to_string(bytes) +
                                    " bytes failed: " + cudaGetErrorString(e));
  }
  bytes_ = bytes;
  stream_ = stream;
  ordered_ = true;
}

void DeviceBuffer::reset(uint64_t bytes) {
  release();
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

uint64_t scene_device_bytes(uint64_t splats, uint32_t sh_degree) {
  const uint64_t n = std::max<uint64_t>(splats, 1);
  return 3 * align256(16 * n) + align256(16 * n * color_planes(sh_degree));
}

uint64_t scene_device_bytes(const HostScene &s) { return scene_device_bytes(s.size(), s.sh_degree); }

std::unique_ptr<DeviceScene> alloc_scene(uint64_t n, uint32_t sh_degree) {
  if (n > kMaxSortItems)
    throw Error(Code::Unsupported, "scene has more splats than the renderer supports (2^30 - 1)");
  auto sc = std::make_unique<DeviceScene>();
  sc->n = (uint32_t)n;
  sc->sh_degree = sh_degree;
  const uint32_t planes = color_planes(sh_degree);
  // Three geometry planes, then the colour planes as one tight region so
  // that plane p of splat i sits at color[p * n + i].
  const uint64_t plane = align256(16 * std::max<uint64_t>(n, 1));
  sc->mem.reset(scene_device_bytes(n, sh_degree));
  char *base = sc->mem.as<char>();
  sc->dev.pos_alpha = reinterpret_cast<const float4 *>(base);
  sc->dev.cov_a = reinterpret_cast<const float4 *>(base + plane);
  sc->dev.cov_b = reinterpret_cast<const float4 *>(base + 2 * plane);
  sc->dev.color = reinterpret_cast<const float4 *>(base + 3 * plane);
  sc->dev.n = (uint32_t)n;
  sc->dev.planes = planes;
  return sc;
}

std::unique_ptr<DeviceScene> upload_scene(const HostScene &s, cudaStream_t stream) {
  const uint64_t n = s.size();
  auto sc = alloc_scene(n, s.sh_degree);
  ScenePacked packed;
  pack_scene(s, packed);
  sc->positions = s.positions;
  if (n) {
    const SceneDev &d = sc->dev;
    GSR_CUDA(cudaMemcpyAsync((void *)d.pos_alpha, packed.pos_alpha.data(), 16 * n,
                             cudaMemcpyHostToDevice, stream));
    GSR_CUDA(cudaMemcpyAsync((void *)d.cov_a, packed.cov_a.data(), 16 * n, cudaMemcpyHostToDevice,
                             stream));
    GSR_CUDA(cudaMemcpyAsync((void *)d.cov_b, packed.cov_b.data(), 16 * n, cudaMemcpyHostToDevice,
                             stream));
    GSR_CUDA(cudaMemcpyAsync((void *)d.color, packed.color.data(), 16 * n * packed.planes,
                             cudaMemcpyHostToDevice, stream));
  }
  GSR_CUDA(cudaStreamSynchronize(stream));
  return sc;
}

Pipeline::Pipeline(int device, cudaStream_t stream) : device_(device), stream_(stream) {
  int sms = 0;
  GSR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
  sm_count_ = (uint32_t)sms;
  for (auto &ev : ev_) GSR_CUDA(cudaEventCreate(&ev));
  for (auto &ev : slot_ev_) GSR_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));

  GSR_CUDA(cudaMallocHost(&counters_host_, sizeof(FrameCounters)));
  std::memset(counters_host_, 0, sizeof(FrameCounters));
  // fixed scratch: [counters | key hist | tile hist] zeroed per run, then
  // plans and the sticky word.
  uint64_t off = 0;
  const uint64_t o_counters = off; off += align256(sizeof(FrameCounters));
  const uint64_t o_khist = off; off += align256(4 * 4 * 256);
  const uint64_t o_thist = off; off += align256(4 * 4 * 256);
  const uint64_t zero_end = off;
  const uint64_t o_dplan = off; off += align256(sizeof(SortPlan));
  const uint64_t o_tplan = off; off += align256(sizeof(SortPlan));
  const uint64_t o_sticky = off; off += 256;
  fixed_.reset(off);
  GSR_CUDA(cudaMemset(fixed_.get(), 0, off));
  counters_ = fixed_.as<FrameCounters>(o_counters);
  key_hist_ = fixed_.as<uint32_t>(o_khist);
  tile_hist_ = fixed_.as<uint32_t>(o_thist);
  depth_plan_ = fixed_.as<SortPlan>(o_dplan);
  tile_plan_ = fixed_.as<SortPlan>(o_tplan);
  sticky_ = fixed_.as<uint32_t>(o_sticky);
  (void)zero_end;
}

Pipeline::~Pipeline() {
  cudaSetDevice(device_);
  cudaStreamSynchronize(stream_);
  drop_graph();
  for (auto &ev : ev_)
    if (ev) cudaEventDestroy(ev);
  for (auto &ev : slot_ev_)
    if (ev) cudaEventDestroy(ev);

  if (counters_host_) cudaFreeHost(counters_host_);
  if (view_counters_pinned_) cudaFreeHost(view_counters_pinned_);
  if (table_pinned_) cudaFreeHost(table_pinned_);
  if (batch_stage_) cudaFreeHost(batch_stage_);
  if (batch_ev_) cudaEventDestroy(batch_ev_);
}

void Pipeline::record(int k) {
  if (batch_mode_) return;  // a batch of groups is timed by its caller
  if (capturing_)
    GSR_CUDA(cudaEventRecordWithFlags(ev_[k], stream_, cudaEventRecordExternal));
  else
    GSR_CUDA(cudaEventRecord(ev_[k], stream_));
}

void Pipeline::set_tile(uint32_t tile) {
  tile_ = tile;
  if (!raster_config_valid(tile_, raster_cfg_)) raster_cfg_.chunk = tile_ * tile_;
}

void Pipeline::set_raster_config(const RasterConfig &c) {
  if (!raster_config_valid(tile_, c))
    throw Error(Code::InvalidArgument, "raster chunk " + std::to_string(c.chunk) +
                                           " or blocks per SM " + std::to_string(c.blocks_per_sm) +
                                           " not valid for tile size " + std::to_string(tile_));
  raster_cfg_ = c;
}

void Pipeline::drop_graph() {
  for (auto &g : graphs_) {
    cudaGraphExecDestroy(g.exec);
    cudaGraphDestroy(g.graph);
  }
  graphs_.clear();
  seen_keys_.clear();
  drop_batch_graphs();
}

void Pipeline::drop_batch_graphs() {
  for (auto &g : batch_graphs_) {
    cudaGraphExecDestroy(g.exec);
    cudaGraphDestroy(g.graph);
  }
  batch_graphs_.clear();
  batch_seen_.clear();
}

Pipeline::Layout Pipeline::plan_views(const ViewSpec *views, uint32_t count,
                                      const uint64_t *image_bases) {
  if (count == 0) throw Error(Code::InvalidArgument, "no views to render");
  if (count > kMaxViewsPerLaunch)
    throw Error(Code::Unsupported, "more than 1024 views in one pipeline run");
  Layout l;
  l.views = count;
  views_host_.resize(count);
  sets_host_.clear();
  uint64_t splats = 0, blocks = 0, tiles = 0;
  for (uint32_t v = 0; v < count; ++v) {
    const ViewSpec &vs = views[v];
    if (!camera_valid(vs.camera)) throw Error(Code::InvalidArgument, "invalid camera");
    if (vs.width == 0 || vs.height == 0)
      throw Error(Code::InvalidArgument, "invalid renderer configuration");
    ViewDev &d = views_host_[v];
    std::memset(&d, 0, sizeof(d));
    d.p = make_frame_params(vs.camera, vs.width, vs.height, tile_, vs.scene->sh_degree,
                            vs.scene->n);
    d.sc = vs.scene->dev;
    d.splat_base = (uint32_t)splats;
    d.tile_base = (uint32_t)tiles;
    d.image_base = image_bases[v];
    // Consecutive views of one scene form a view set (one scene read in K1).
    if (sets_host_.empty() || views[v - 1].scene != vs.scene ||
        sets_host_.back().count == kMaxSetViews) {
      sets_host_.push_back(ViewSetDev{v, 0, (uint32_t)blocks, 0});
      blocks += preprocess_blocks(vs.scene->n);
    }
    sets_host_.back().count++;
    d.set = (uint32_t)sets_host_.size() - 1;
    splats += vs.scene->n;
    tiles += d.p.num_tiles;
    l.max_planes = std::max(l.max_planes, vs.scene->dev.planes);
  }
  if (splats > kMaxSortItems)
    throw Error(Code::Unsupported, "splats over the views of one run exceed 2^30 - 1");
  if (tiles > (1u << 24)) throw Error(Code::Unsupported, "too many tiles in one run");
  l.total_splats = (uint32_t)splats;
  l.sets = (uint32_t)sets_host_.size();
  l.total_blocks = (uint32_t)blocks;
  l.total_tiles = (uint32_t)tiles;
  l.tile_passes = tile_sort_passes(l.total_tiles);
  return l;
}

void Pipeline::ensure_workspace(const Layout &l) {
  const uint32_t n = std::max<uint32_t>(l.total_splats, 1);
  if (l.views > view_cap_ || n > splat_cap_ || !view_ws_.get()) {
    const auto t_grow = std::chrono::steady_clock::now();
    GSR_CUDA(cudaStreamSynchronize(stream_));  // earlier runs may still use the old buffers
    drop_graph();
    // Growth is geometric: a reallocation synchronises the device (cudaFree),
    // so a stream of batches of varying size must not regrow every time.
    const uint32_t vcap = l.views > view_cap_
                              ? std::min<uint32_t>(std::max(l.views, view_cap_ + view_cap_ / 2),
                                                   kMaxViewsPerLaunch)
                              : view_cap_;
    const uint32_t ncap = n > splat_cap_
                              ? (uint32_t)std::min<uint64_t>(
                                    std::max<uint64_t>(n, splat_cap_ + (uint64_t)splat_cap_ / 2),
                                    kMaxSortItems)
                              : splat_cap_;
    // view workspace: [view counters | K1 status | emit status] zeroed, then the table.
    const uint64_t k1_words = (ncap + 255) / 256 + 1;  // + views: blocks round up per set
    const uint64_t k1_total = k1_words + vcap;
    const uint64_t emit_words = emit_status_words(ncap);
    uint64_t off = 0;
    const uint64_t o_vc = off; off += align256(sizeof(ViewCounters) * vcap);
    const uint64_t o_k1 = off; off += align256(8 * k1_total);
    const uint64_t o_em = off; off += align256(8 * emit_words);
    view_zero_bytes_ = off;
    // the table: view sets, then views (one host-to-device copy per run);
    // the sets region is sized for the largest launch, so the table's layout
    // (and the pinned staging slots that mirror it) never changes
    const uint64_t o_sets = off; off += align256(sizeof(ViewSetDev) * kMaxViewsPerLaunch);
    const uint64_t o_tab = off; off += align256(sizeof(ViewDev) * vcap);
    view_ws_.reset(off, stream_);
    sets_dev_ = view_ws_.as<ViewSetDev>(o_sets);
    view_counters_ = view_ws_.as<ViewCounters>(o_vc);
    k1_status_ = view_ws_.as<unsigned long long>(o_k1);
    emit_status_ = view_ws_.as<unsigned long long>(o_em);
    views_dev_ = view_ws_.as<ViewDev>(o_tab);
    view_cap_ = vcap;
    // A staging slot has the device table's layout (sets, then views at
    // o_tab). The pinned host arrays are pinned once, for the largest launch
    // (freeing pinned memory waits for the whole device, which would stall
    // a growing lane behind every other stream's work).
    if (!table_pinned_) {
      const uint64_t slot_bytes = (o_tab - o_sets) + align256(sizeof(ViewDev) * kMaxViewsPerLaunch);
      GSR_CUDA(cudaMallocHost(&view_counters_pinned_, sizeof(ViewCounters) * kMaxViewsPerLaunch));
      GSR_CUDA(cudaMallocHost((void **)&table_pinned_, slot_bytes * kViewSlots));
      view_counters_pinned_cap_ = kMaxViewsPerLaunch;
      table_slot_bytes_ = slot_bytes;
    }
    table_sets_bytes_ = o_tab - o_sets;
    if (n > splat_cap_) {
      const uint64_t words = sort_work_words(ncap, 4);
      off = 0;
      uint64_t o_k0 = off; off += align256(4ull * ncap);
      uint64_t o_v0 = off; off += align256(4ull * ncap);
      uint64_t o_k1b = off; off += align256(4ull * ncap);
      uint64_t o_v1 = off; off += align256(4ull * ncap);
      uint64_t o_rect = off; off += align256(8ull * ncap);
      uint64_t o_rec = off; off += align256(sizeof(Record) * (uint64_t)ncap);
      uint64_t o_work = off; off += align256(4 * words);
      splat_ws_.reset(off, stream_);
      sorted_valid_ = false;  // the sorted ids lived in the old buffers
      vis_keys0_ = splat_ws_.as<uint32_t>(o_k0);
      vis_vals0_ = splat_ws_.as<uint32_t>(o_v0);
      vis_keys1_ = splat_ws_.as<uint32_t>(o_k1b);
      vis_vals1_ = splat_ws_.as<uint32_t>(o_v1);
      rects_ = splat_ws_.as<uint2>(o_rect);
      records_ = splat_ws_.as<Record>(o_rec);
      depth_sort_work_ = splat_ws_.as<uint32_t>(o_work);
      splat_cap_ = ncap;
      projected_.reset(0, stream_);
      debug_cov_.reset(0, stream_);
    }
    note_regrowth(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() -
                                                            t_grow).count());
  }
  if (l.total_tiles > tile_cap_ || !tile_ws_.get()) {
    const auto t_grow = std::chrono::steady_clock::now();
    GSR_CUDA(cudaStreamSynchronize(stream_));
    drop_graph();
    tile_cap_ = std::max(l.total_tiles, tile_cap_ + tile_cap_ / 2);
    tile_ws_.reset(align256(8ull * std::max<uint32_t>(tile_cap_, 1)), stream_);
    ranges_ = tile_ws_.as<uint2>();
    note_regrowth(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() -
                                                            t_grow).count());
  }
  if (key_cap_ == 0)
    ensure_key_workspace(std::min<uint64_t>(std::max<uint64_t>(kInitialPairsPerSplat * n, 1u << 20),
                                            kMaxSortItems));
  if (debug_) {
    const uint64_t need = sizeof(ProjectedDev) * (uint64_t)splat_cap_;
    if (projected_.size() < need) {
      GSR_CUDA(cudaStreamSynchronize(stream_));
      drop_graph();
      projected_.reset(need, stream_);
    }
    if (debug_cov_.size() < 8ull * splat_cap_) {
      GSR_CUDA(cudaStreamSynchronize(stream_));
      drop_graph();
      debug_cov_.reset(8ull * splat_cap_, stream_);
    }
    if (debug_pairs_.size() < 8 * key_cap_) {
      GSR_CUDA(cudaStreamSynchronize(stream_));
      drop_graph();
      debug_pairs_.reset(8 * key_cap_, stream_);
    }
  }
}

void Pipeline::ensure_key_workspace(uint64_t capacity) {
  const uint32_t passes = 3;  // enough for any tile count below 2^24
  if (key_cap_ >= capacity && key_ws_.get()) return;
  if (capacity > kMaxSortItems)
    throw Error(Code::Unsupported, "tile pair count " + std::to_string(capacity) +
                                       " exceeds the renderer's limit of 2^30 - 1");
  const auto t_grow = std::chrono::steady_clock::now();
  GSR_CUDA(cudaStreamSynchronize(stream_));
  drop_graph();
  // geometric growth, as for the other workspaces
  const uint32_t cap = (uint32_t)std::min<uint64_t>(
      std::max<uint64_t>(capacity, key_cap_ + key_cap_ / 4), kMaxSortItems);
  const uint64_t words = sort_work_words(cap, passes);
  uint64_t off = 0;
  uint64_t o_k0 = off; off += align256(4ull * cap);
  uint64_t o_v0 = off; off += align256(4ull * cap);
  uint64_t o_k1 = off; off += align256(4ull * cap);
  uint64_t o_v1 = off; off += align256(4ull * cap);
  uint64_t o_work = off; off += align256(4 * words);
  key_ws_.reset(off, stream_);
  tile_keys0_ = key_ws_.as<uint32_t>(o_k0);
  tile_vals0_ = key_ws_.as<uint32_t>(o_v0);
  tile_keys1_ = key_ws_.as<uint32_t>(o_k1);
  tile_vals1_ = key_ws_.as<uint32_t>(o_v1);
  tile_sort_work_ = key_ws_.as<uint32_t>(o_work);
  key_cap_ = cap;
  debug_pairs_.reset(0, stream_);
  note_regrowth(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() -
                                                          t_grow).count());
}

RunInit Pipeline::make_run_init(const Layout &l) const {
  RunInit init{};
  init.zero[0] = fixed_.as<uint32_t>();
  init.zero_words[0] = ((char *)depth_plan_ - (char *)fixed_.get()) / 4;
  init.zero[1] = view_ws_.as<uint32_t>();
  init.zero_words[1] = view_zero_bytes_ / 4;
  init.zero[2] = reinterpret_cast<uint32_t *>(ranges_);
  init.zero_words[2] = 2ull * l.total_tiles;
  init.zero[3] = depth_sort_work_;
  init.zero_words[3] = kSortScratchHeadWords;
  init.zero[4] = tile_sort_work_;
  init.zero_words[4] = kSortScratchHeadWords;
  if (l.views <= kRunInlineViews && !batch_mode_) {
    init.inline_views = l.views;
    init.inline_sets = l.sets;
    init.sets_dst = sets_dev_;
    init.views_dst = views_dev_;
    std::memcpy(init.sets, sets_host_.data(), sizeof(ViewSetDev) * l.sets);
    std::memcpy(init.views, views_host_.data(), sizeof(ViewDev) * l.views);
  }
  return init;
}

void Pipeline::launch_all(const Layout &l, uint32_t *images, const HostSinks &sinks,
                          bool reuse, const ViewDev *views_dev, const ViewSetDev *sets_dev) {
  const uint32_t n = std::max<uint32_t>(l.total_splats, 1);
  launch_run_init(make_run_init(l), stream_);
  record(0);

  K1Buffers k1{vis_keys0_, vis_vals0_, rects_,         records_,
               k1_status_, counters_,  key_hist_,      view_counters_,
               debug_ ? projected_.as<ProjectedDev>() : nullptr, reuse};
  launch_preprocess(views_dev, sets_dev, l.sets, l.total_blocks, l.max_planes, k1, debug_,
                    stream_);
  record(1);

  if (!reuse) {  // a reused order keeps the last sort's ids and plan
    SortBuffers ds{vis_keys0_, vis_vals0_, vis_keys1_, vis_vals1_, &counters_->visible, n, 0, 4,
                   depth_plan_, depth_sort_work_, &counters_->error, key_hist_, true};
    launch_sort(ds, stream_);
  }
  record(2);

  EmitBuffers eb{depth_plan_, vis_vals0_,  vis_vals1_, rects_,        records_,
                 tile_keys0_, tile_vals0_, key_cap_,   emit_status_,  counters_,
                 tile_hist_,  l.tile_passes, l.total_splats, views_dev,  l.views,
                 tile_};
  launch_emit(eb, stream_);
  if (debug_) {
    GSR_CUDA(cudaMemcpyAsync(debug_pairs_.as<uint32_t>(), tile_keys0_, 4 * key_cap_,
                             cudaMemcpyDeviceToDevice, stream_));
    GSR_CUDA(cudaMemcpyAsync(debug_pairs_.as<uint32_t>(4 * key_cap_), tile_vals0_, 4 * key_cap_,
                             cudaMemcpyDeviceToDevice, stream_));
  }
  record(3);
  SortBuffers ts{tile_keys0_, tile_vals0_, tile_keys1_, tile_vals1_, &counters_->pairs,
                 (uint32_t)key_cap_, 0, l.tile_passes, tile_plan_, tile_sort_work_,
                 &counters_->error, tile_hist_, true};
  launch_sort(ts, stream_);
  record(4);
  launch_ranges(tile_plan_, tile_keys0_, tile_keys1_, counters_, (uint32_t)key_cap_, ranges_,
                views_dev, l.views, view_counters_, stream_);
  record(5);
  RasterArgs ra{views_dev,  l.views,  l.total_tiles, ranges_,   tile_plan_,
                tile_vals0_, tile_vals1_, records_,  images, counters_, sticky_};
  if (debug_) {
    GSR_CUDA(cudaMemsetAsync(debug_cov_.get(), 0xff, 8ull * std::max<uint32_t>(l.total_splats, 1),
                             stream_));
    ra.debug_cov = debug_cov_.as<float2>();
  }
  launch_raster(ra, tile_, blend_mode_, raster_cfg_, sm_count_, stream_);
  record(6);
  // Runs with host sinks copy their counters there; the others leave them in
  // device memory, read after the stream is synchronised.
  if (sinks.counters) {
    GSR_CUDA(cudaMemcpyAsync(sinks.counters, counters_, sizeof(FrameCounters),
                             cudaMemcpyDeviceToHost, stream_));
    GSR_CUDA(cudaMemcpyAsync(sinks.views, view_counters_, sizeof(ViewCounters) * l.views,
                             cudaMemcpyDeviceToHost, stream_));
  }
}

void Pipeline::enqueue(const ViewSpec *views, uint32_t count, uint32_t *images,
                       const uint64_t *image_bases, HostSinks sinks) {
  GSR_CUDA(cudaSetDevice(device_));
  const Layout l = plan_views(views, count, image_bases);
  ensure_workspace(l);
  // No sinks given: the counters stay in device memory until the host reads
  // them after a synchronisation (no host memory traffic inside the run).
  const bool device_sinks = !sinks.counters;
  if (device_sinks) sinks = HostSinks{};
  // The last sorted order can be reused only for the identical layout (same
  // scenes, sizes and tile grid) and while its buffers are intact.
  const bool reuse = reuse_request_ && sorted_valid_ && l == sorted_layout_ &&
                     std::equal(views, views + count, sorted_scenes_.begin(), sorted_scenes_.end(),
                                [](const ViewSpec &v, const DeviceScene *s) { return v.scene == s; });
  // A small view table rides in the zeroing kernel's parameters. A larger
  // one goes up from a pinned ring slot, ahead of the run on its stream
  // (outside the run's graph, so the graph serves every frame of the
  // layout); the slot's previous copy is long done in steady state.
  const bool inline_table = l.views <= kRunInlineViews;
  if (!inline_table) {
    const uint32_t slot = slot_;
    GSR_CUDA(cudaEventSynchronize(slot_ev_[slot]));
    unsigned char *staged = table_pinned_ + (uint64_t)slot * table_slot_bytes_;
    std::memcpy(staged, sets_host_.data(), sizeof(ViewSetDev) * l.sets);
    std::memcpy(staged + table_sets_bytes_, views_host_.data(), sizeof(ViewDev) * l.views);
    GSR_CUDA(cudaMemcpyAsync(sets_dev_, staged, table_sets_bytes_ + sizeof(ViewDev) * l.views,
                             cudaMemcpyHostToDevice, stream_));
    GSR_CUDA(cudaEventRecord(slot_ev_[slot], stream_));
    slot_ = (slot_ + 1) % kViewSlots;
  }
  ViewDev *run_views = views_dev_;
  ViewSetDev *run_sets = sets_dev_;

  if (!use_graph_) {
    launch_all(l, images, sinks, reuse, run_views, run_sets);
  } else {
    const GraphKey key{l,     images,      key_cap_,       tile_,       blend_mode_,
                       debug_, raster_cfg_, sinks.counters, sinks.views, reuse};
    GraphEntry *hit = nullptr;
    for (auto &g : graphs_)
      if (g.key == key) hit = &g;
    // A layout is captured the second time it is seen: one-off layouts (a
    // served batch of a new size) launch directly instead of paying for a
    // capture they would never replay.
    bool seen = false;
    if (!hit) {
      for (auto &k : seen_keys_)
        if (k == key) seen = true;
      if (!seen) {
        if (seen_keys_.size() >= kGraphCacheSize) seen_keys_.erase(seen_keys_.begin());
        seen_keys_.push_back(key);
      }
    }
    if (!hit && !seen) {
      launch_all(l, images, sinks, reuse, run_views, run_sets);
    } else if (!hit) {
      if (graphs_.size() >= kGraphCacheSize) {
        auto lru = std::min_element(graphs_.begin(), graphs_.end(),
                                    [](const GraphEntry &a, const GraphEntry &b) {
                                      return a.last_use < b.last_use;
                                    });
        cudaGraphExecDestroy(lru->exec);
        cudaGraphDestroy(lru->graph);
        graphs_.erase(lru);
      }
      cudaGraph_t g = nullptr;
      const auto t_capture = std::chrono::steady_clock::now();
      GSR_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      capturing_ = true;
      try {
        launch_all(l, images, sinks, reuse, run_views, run_sets);
      } catch (...) {
        capturing_ = false;
        cudaStreamEndCapture(stream_, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
      }
      capturing_ = false;
      GSR_CUDA(cudaStreamEndCapture(stream_, &g));
      cudaGraphExec_t exec = nullptr;
      cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
      if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        throw Error(Code::Internal, std::string("CUDA graph instantiation failed: ") +
                                        cudaGetErrorString(e));
      }
      GraphEntry entry{key, exec, 0, g, nullptr, {}};
      size_t count = 0;
      GSR_CUDA(cudaGraphGetNodes(g, nullptr, &count));
      std::vector<cudaGraphNode_t> nodes(count);
      GSR_CUDA(cudaGraphGetNodes(g, nodes.data(), &count));
      for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType type;
        GSR_CUDA(cudaGraphNodeGetType(node, &type));
        if (type != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp{};
        GSR_CUDA(cudaGraphKernelNodeGetParams(node, &kp));
        if (kp.func == run_init_kernel_entry()) {
          entry.init_node = node;
          entry.init_params = kp;
          break;
        }
      }
      if (inline_table && !entry.init_node) {
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(g);
        throw Error(Code::Internal, "captured run has no zeroing kernel node");
      }
      graphs_.push_back(entry);
      hit = &graphs_.back();
      captures_.fetch_add(1, std::memory_order_relaxed);
      const double ms = std::chrono::duration<double, std::milli>(
                            std::chrono::steady_clock::now() - t_capture).count();
      capture_ms_.store(capture_ms_.load(std::memory_order_relaxed) + ms,
                        std::memory_order_relaxed);
    }
    if (hit) {
      hit->last_use = ++graph_clock_;
      if (inline_table) {
        // this run's view table, in the zeroing node's parameters
        RunInit init = make_run_init(l);
        void *args[] = {&init};
        cudaKernelNodeParams kp = hit->init_params;
        kp.kernelParams = args;
        kp.extra = nullptr;
        GSR_CUDA(cudaGraphExecKernelNodeSetParams(hit->exec, hit->init_node, &kp));
      }
      GSR_CUDA(cudaGraphLaunch(hit->exec, stream_));
    }
  }
  GSR_CUDA(cudaGetLastError());
  last_layout_ = l;
  last_sinks_ = sinks;
  last_device_sinks_ = device_sinks;
  has_run_ = true;
  last_reused_ = reuse;
  if (!reuse) {
    sorted_layout_ = l;
    sorted_valid_ = true;
    sorted_scenes_.clear();
    for (uint32_t v = 0; v < count; ++v) sorted_scenes_.push_back(views[v].scene);
  }
}

void Pipeline::enqueue_groups(const ViewSpec *views, uint32_t *images,
                              const uint64_t *image_bases, const std::vector<GroupRun> &groups) {
  GSR_CUDA(cudaSetDevice(device_));
  if (!use_graph_ || groups.empty()) {
    for (const GroupRun &g : groups)
      enqueue(views + g.first, g.count, images, image_bases + g.first, g.sinks);
    return;
  }
  // Size the workspace for every group first (growing it drops the graphs),
  // then stage every group's view table in the pinned area.
  std::vector<Layout> layouts;
  layouts.reserve(groups.size());
  for (const GroupRun &g : groups) {
    layouts.push_back(plan_views(views + g.first, g.count, image_bases + g.first));
    ensure_workspace(layouts.back());
  }
  std::vector<uint64_t> offs(groups.size());
  uint64_t total = 0;
  for (size_t k = 0; k < groups.size(); ++k) {
    offs[k] = total;
    total += (table_sets_bytes_ + sizeof(ViewDev) * layouts[k].views + 255) & ~uint64_t(255);
  }
  // the previous batch launch must have read the staging area
  if (batch_ev_) GSR_CUDA(cudaEventSynchronize(batch_ev_));
  else GSR_CUDA(cudaEventCreateWithFlags(&batch_ev_, cudaEventDisableTiming));
  if (total > batch_stage_bytes_) {
    drop_batch_graphs();  // the captured copies read the old area
    if (batch_stage_) cudaFreeHost(batch_stage_);
    batch_stage_ = nullptr;
    batch_stage_bytes_ = 0;
    GSR_CUDA(cudaMallocHost((void **)&batch_stage_, total + total / 4));
    batch_stage_bytes_ = total + total / 4;
  }
  for (size_t k = 0; k < groups.size(); ++k) {
    plan_views(views + groups[k].first, groups[k].count, image_bases + groups[k].first);
    std::memcpy(batch_stage_ + offs[k], sets_host_.data(), sizeof(ViewSetDev) * layouts[k].sets);
    std::memcpy(batch_stage_ + offs[k] + table_sets_bytes_, views_host_.data(),
                sizeof(ViewDev) * layouts[k].views);
  }
  BatchKey key{layouts, {}, {}, images, key_cap_, tile_, blend_mode_, debug_, raster_cfg_};
  for (const GroupRun &g : groups) {
    key.counters.push_back(g.sinks.counters);
    key.views.push_back(g.sinks.views);
  }
  // The groups in stream order: each copies its table into the device table
  // (no inline tables) and runs the frame pipeline over it.
  auto launch_groups = [&]() {
    for (size_t k = 0; k < groups.size(); ++k) {
      GSR_CUDA(cudaMemcpyAsync(sets_dev_, batch_stage_ + offs[k],
                               table_sets_bytes_ + sizeof(ViewDev) * layouts[k].views,
                               cudaMemcpyHostToDevice, stream_));
      launch_all(layouts[k], images, groups[k].sinks, false, views_dev_, sets_dev_);
    }
  };
  BatchGraph *hit = nullptr;
  for (auto &g : batch_graphs_)
    if (g.key == key) hit = &g;
  const bool seen = std::find(batch_seen_.begin(), batch_seen_.end(), key) != batch_seen_.end();
#ifdef GSR_BATCH_DEBUG
  fprintf(stderr, "batch: groups %zu hit %d seen %d graphs %zu seen_list %zu key_cap %llu images %p\n",
          groups.size(), hit != nullptr, (int)seen, batch_graphs_.size(), batch_seen_.size(),
          (unsigned long long)key_cap_, (void *)images);
  if (!batch_seen_.empty()) {
    const BatchKey &o = batch_seen_.back();
    fprintf(stderr, "  vs last seen: layouts %d counters %d views %d images %d cap %d tile %d blend %d dbg %d raster %d\n",
            o.layouts == key.layouts, o.counters == key.counters, o.views == key.views,
            o.images == key.images, o.key_cap == key.key_cap, o.tile == key.tile, o.blend == key.blend,
            o.debug == key.debug, o.raster == key.raster);
  }
#endif
  batch_mode_ = true;
  try {
    if (!hit && !seen) {
      // first sighting: direct launches (a one-off batch pays no capture)
      if (batch_seen_.size() >= kBatchGraphCacheSize) batch_seen_.erase(batch_seen_.begin());
      batch_seen_.push_back(key);
      launch_groups();
    } else {
      if (!hit) {
        if (batch_graphs_.size() >= kBatchGraphCacheSize) {
          auto lru = std::min_element(
              batch_graphs_.begin(), batch_graphs_.end(),
              [](const BatchGraph &a, const BatchGraph &b) { return a.last_use < b.last_use; });
          cudaGraphExecDestroy(lru->exec);
          cudaGraphDestroy(lru->graph);
          batch_graphs_.erase(lru);
        }
        const auto t_capture = std::chrono::steady_clock::now();
        cudaGraph_t g = nullptr;
        GSR_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        capturing_ = true;
        try {
          launch_groups();
        } catch (...) {
          capturing_ = false;
          cudaStreamEndCapture(stream_, &g);
          if (g) cudaGraphDestroy(g);
          cudaGetLastError();
          throw;
        }
        capturing_ = false;
        GSR_CUDA(cudaStreamEndCapture(stream_, &g));
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        if (e != cudaSuccess) {
          cudaGraphDestroy(g);
          throw Error(Code::Internal, std::string("CUDA graph instantiation failed: ") +
                                          cudaGetErrorString(e));
        }
        batch_graphs_.push_back(BatchGraph{key, g, exec, 0});
        hit = &batch_graphs_.back();
        captures_.fetch_add(1, std::memory_order_relaxed);
        const double ms = std::chrono::duration<double, std::milli>(
                              std::chrono::steady_clock::now() - t_capture).count();
        capture_ms_.store(capture_ms_.load(std::memory_order_relaxed) + ms,
                          std::memory_order_relaxed);
      }
      hit->last_use = ++graph_clock_;
      GSR_CUDA(cudaGraphLaunch(hit->exec, stream_));
      ++batch_graph_launches_;
    }
  } catch (...) {
    batch_mode_ = false;
    throw;
  }
  batch_mode_ = false;
  GSR_CUDA(cudaEventRecord(batch_ev_, stream_));
  GSR_CUDA(cudaGetLastError());
  last_layout_ = layouts.back();
  last_sinks_ = groups.back().sinks;
  last_device_sinks_ = false;
  has_run_ = true;
  last_reused_ = false;
  sorted_valid_ = false;  // a batch never hands its order to a later frame
}

void Pipeline::fetch_counters() {
  if (!last_device_sinks_) return;
  // the stream is synchronised: counters_ hold the last run's values
  GSR_CUDA(cudaMemcpy(counters_host_, counters_, sizeof(FrameCounters), cudaMemcpyDeviceToHost));
  GSR_CUDA(cudaMemcpy(view_counters_pinned_, view_counters_,
                      sizeof(ViewCounters) * last_layout_.views, cudaMemcpyDeviceToHost));
  last_sinks_ = HostSinks{counters_host_, view_counters_pinned_};
}

void Pipeline::phase_times(float out[kPhaseCount]) const {
  for (int k = 0; k < kPhaseCount; ++k)
    GSR_CUDA(cudaEventElapsedTime(&out[k], ev_[k], ev_[k + 1]));
}

void Pipeline::collect(RunResult &r) {
  float t[kPhaseCount];
  for (int k = 0; k < kPhaseCount; ++k) GSR_CUDA(cudaEventElapsedTime(&t[k], ev_[k], ev_[k + 1]));
  for (int k = 0; k < kPhaseCount; ++k) r.phase_ms[k] = t[k];
  r.preprocess_ms = t[kPhasePreprocess];
  r.sort_ms = t[kPhaseDepthSort] + t[kPhaseEmit] + t[kPhaseTileSort] + t[kPhaseRanges];
  r.raster_ms = t[kPhaseRaster];
  r.sorted = !last_reused_;
  r.visible = last_sinks_.counters->visible;
  r.drawn = last_sinks_.counters->drawn;
  r.keys = last_sinks_.counters->keys;
  view_counters_host_.assign(last_sinks_.views, last_sinks_.views + last_layout_.views);
}

RunResult Pipeline::run(const ViewSpec *views, uint32_t count, uint32_t *images,
                        const uint64_t *image_bases) {
  auto t0 = std::chrono::steady_clock::now();
  RunResult r;
  for (;;) {
    enqueue(views, count, images, image_bases);
    GSR_CUDA(cudaStreamSynchronize(stream_));
    fetch_counters();
    if (counters_host_->error)
      throw Error(Code::Internal, "device wait limit reached in a look-back scan (error bits " +
                                      std::to_string(counters_host_->error) + ")");
    if (!counters_host_->overflow) break;
    // Grow the pair buffers to the exact need plus headroom and run again.
    const uint64_t need = counters_host_->keys;
    if (need > kMaxSortItems)
      throw Error(Code::Unsupported, "tile pair count " + std::to_string(need) +
                                         " exceeds the renderer's limit of 2^30 - 1");
    ensure_key_workspace(std::min<uint64_t>(need + need / 4 + 1024, kMaxSortItems));
    if (debug_) debug_pairs_.reset(8 * key_cap_, stream_);
    ++r.reruns;
  }
  GSR_CUDA(cudaMemsetAsync(sticky_, 0, 4, stream_));
  collect(r);
  r.frame_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  last_ = r;
  return r;
}

RunResult Pipeline::sync() {
  GSR_CUDA(cudaSetDevice(device_));
  uint32_t sticky = 0;
  GSR_CUDA(cudaMemcpyAsync(&sticky, sticky_, 4, cudaMemcpyDeviceToHost, stream_));
  GSR_CUDA(cudaMemsetAsync(sticky_, 0, 4, stream_));
  GSR_CUDA(cudaStreamSynchronize(stream_));
  RunResult r;
  if (!has_run_) return r;
  fetch_counters();
  collect(r);
  r.frame_ms = r.preprocess_ms + r.sort_ms + r.raster_ms;
  last_ = r;
  if (sticky & 0x7fffffffu)
    throw Error(Code::Internal, "device wait limit reached in a look-back scan");
  if (sticky & 0x80000000u)
    throw Error(Code::Internal,
                "an enqueued frame overflowed its tile-pair buffers; render it synchronously "
                "once to size them");
  return r;
}

uint32_t Pipeline::launches_per_run() const {
  // preprocess; depth sort plan + 4 passes (histograms come from K1); emit;
  // tile sort plan + passes (histograms from K2); ranges; raster.
  const uint32_t tile_passes = last_layout_.tile_passes;
  return 1 + (1 + 4) + 1 + (1 + tile_passes) + 1 + 1;
}

SortPlan Pipeline::read_plan(int which) {
  SortPlan plan;
  GSR_CUDA(cudaMemcpyAsync(&plan, which == 0 ? depth_plan_ : tile_plan_, sizeof(SortPlan),
                           cudaMemcpyDeviceToHost, stream_));
  GSR_CUDA(cudaStreamSynchronize(stream_));
  return plan;
}

std::vector<uint32_t> Pipeline::debug_order() {
  GSR_CUDA(cudaSetDevice(device_));
  SortPlan plan = read_plan(0);
  std::vector<uint32_t> out(plan.n);
  if (!out.empty())
    GSR_CUDA(cudaMemcpy(out.data(), plan.final_buffer == 0 ? vis_vals0_ : vis_vals1_,
                        4 * out.size(), cudaMemcpyDeviceToHost));
  return out;
}

std::vector<ProjectedDev> Pipeline::debug_projected(uint32_t count) {
  if (!debug_ || !projected_.get())
    throw Error(Code::InvalidArgument, "debug taps were not enabled for the last frame");
  GSR_CUDA(cudaSetDevice(device_));
  std::vector<ProjectedDev> out(count);
  if (count)
    GSR_CUDA(cudaMemcpy(out.data(), projected_.get(), sizeof(ProjectedDev) * count,
                        cudaMemcpyDeviceToHost));
  return out;
}

std::vector<float2> Pipeline::debug_coverage(uint32_t count) {
  if (!debug_ || !debug_cov_.get())
    throw Error(Code::InvalidArgument, "debug taps were not enabled for the last frame");
  GSR_CUDA(cudaSetDevice(device_));
  std::vector<float2> out(count);
  if (count)
    GSR_CUDA(cudaMemcpy(out.data(), debug_cov_.get(), sizeof(float2) * count,
                        cudaMemcpyDeviceToHost));
  return out;
}

void Pipeline::debug_tile_pairs(std::vector<uint32_t> &tiles, std::vector<uint32_t> &ids) {
  if (!debug_ || !debug_pairs_.get())
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

void Pipeline::debug_tile_ranges(uint32_t num_tiles, std::vector<uint32_t> &ranges,
                                 std::vector<uint32_t> &ids) {
  GSR_CUDA(cudaSetDevice(device_));
  SortPlan plan = read_plan(1);
  ranges.resize(2ull * num_tiles);
  if (num_tiles)
    GSR_CUDA(cudaMemcpy(ranges.data(), ranges_, 4 * ranges.size(), cudaMemcpyDeviceToHost));
  const uint64_t k = std::min<uint64_t>(last_.keys, key_cap_);
  ids.resize(k);
  if (k)
    GSR_CUDA(cudaMemcpy(ids.data(), plan.final_buffer == 0 ? tile_vals0_ : tile_vals1_, 4 * k,
                        cudaMemcpyDeviceToHost));
}

}  // namespace gsr
