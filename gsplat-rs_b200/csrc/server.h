// Served rendering: a request loop over HBM-resident scenes with continuous
// batching. Requests are queued by submit(); a scheduler thread takes the
// queued requests into a batch whenever one of its lanes (a CUDA stream with
// its own pipeline workspace) is free, admitting them in arrival order while
// the batch's predicted memory (tile-pair buffers from predicted tile-overlap
// counts, splat workspace, images) fits the lane's share of the work budget.
// Batches on different lanes overlap on the device; a host callback on each
// lane's stream marks its requests done as soon as their images are in host
// memory. Every result is the same, bit for bit, as the plain one-frame
// render of its scene, camera and size, whatever batch it ran in.
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.h"

namespace gsr {

struct ServeConfig {
  uint64_t scene_budget = 150ull << 30;  // resident scene bytes
  uint64_t work_budget = 24ull << 30;    // pipeline workspace over all lanes
  uint32_t lanes = 2;                    // batches in flight
  uint32_t max_views = 256;              // per batch
  uint32_t tile = 16;
  RasterConfig raster;  // chunk 0 = full tile
  uint32_t result_pool_mib = 0;  // pinned result memory reserved at creation
  // A request still queued this long after its submit is shed (fails with
  // Unsupported) when a lane next admits work, so that under overload the
  // requests that do run keep a bounded queueing delay; 0 = never shed.
  uint32_t max_queue_ms = 0;
};

enum class RequestStatus : uint32_t { Queued = 0, Running = 1, Done = 2, Failed = 3 };

struct RequestInfo {
  RequestStatus status = RequestStatus::Queued;
  uint32_t batch_views = 0;   // requests in the batch it ran in
  float latency_ms = 0;       // submit -> image in host memory
  float queue_ms = 0;         // submit -> batch launch
  ViewCounters counters{};
  int32_t error_code = 0;
  std::string error;
};

struct ServeStats {
  uint64_t submitted = 0, completed = 0, failed = 0, batches = 0, reruns = 0;
  double p50_ms = 0, p99_ms = 0, mean_ms = 0, max_ms = 0;
  double views_per_s = 0;      // completed / (last completion - first submit)
  double mean_batch_views = 0;
  uint64_t peak_admitted_bytes = 0;
  double device_ms = 0;        // CUDA-event time of the batches' pipelines (sum)
  double launch_ms = 0;        // host time spent enqueuing batches (sum)
  double retire_ms = 0;        // host time spent retiring batches (sum)
  uint64_t graph_captures = 0; // launch graphs the lanes captured
  uint64_t pinned_slabs = 0;   // pinned result slabs allocated
  double capture_ms = 0;       // host time in those captures (part of launch_ms)
  double pinned_alloc_ms = 0;  // host time launches waited on pinned allocations (part of
                               // launch_ms; slabs added in the background are not counted)
  uint64_t workspace_regrowths = 0;  // lane workspace reallocations
  double regrowth_ms = 0;            // host time in them (part of launch_ms)
  uint64_t shed = 0;                 // requests shed after max_queue_ms in the queue (in failed)
};

// Pinned host buffers recycled by size, carved from slabs of about 64 MB
// (at most 64 buffers per slab). Pinning memory takes milliseconds per slab
// (tens of milliseconds for 64 MB), so a background thread adds a slab for a
// size whenever its free buffers fall below a low-water mark; take() only
// allocates on the caller's thread when a size has no free buffer at all.
class PinnedPool {
 public:
  PinnedPool();
  ~PinnedPool();
  PinnedPool(const PinnedPool &) = delete;
  PinnedPool &operator=(const PinnedPool &) = delete;
  uint8_t *take(uint64_t bytes);
  void give(uint8_t *p, uint64_t bytes);
  // slabs allocated so far, and the milliseconds take() callers spent
  // waiting on allocations (the background thread's time is not counted)
  void allocations(uint64_t &slabs, double &wait_ms);
  // the device whose context the background thread allocates in
  void set_device(int device);
  // Pins `bytes` now (whole slabs), carved into buffers of whatever sizes
  // are asked for later before any further allocation happens.
  void reserve(uint64_t bytes);

 private:
  static constexpr uint64_t kSlabBytes = 64ull << 20;
  static constexpr size_t kLowWater = 8;  // free buffers per size kept ahead of demand
  uint8_t *allocate_slab(uint64_t bytes, bool keep_one);  // adds the rest to the free list
  void grower();
  std::mutex mu_;
  std::condition_variable cv_;
  std::map<uint64_t, std::vector<uint8_t *>> free_;
  std::map<uint64_t, bool> growing_;  // a background slab for this size is pending
  std::deque<uint64_t> wanted_;       // sizes for the background thread
  std::vector<uint8_t *> slabs_;
  std::vector<uint8_t *> raw_;  // reserved slabs (kSlabBytes each), not yet carved
  double wait_ms_ = 0;
  int device_ = -1;
  bool stop_ = false;
  std::thread thread_;
};

class Server {
 public:
  explicit Server(const ServeConfig &cfg);
  ~Server();
  Server(const Server &) = delete;
  Server &operator=(const Server &) = delete;

  uint32_t add_scene(const HostScene &s);
  uint32_t add_scene_path(const std::string &path);  // PLY, binary bodies decoded on the device
  uint32_t add_scene_packed(const HostScene &s);      // packed resident format, SH degree <= 3
  // Thread-safe. Validates the view and queues it; returns its request id.
  uint64_t submit(const BatchView &v);
  RequestInfo poll(uint64_t id);
  // Waits up to timeout_ms for the request to finish (or fail).
  RequestInfo wait(uint64_t id, uint32_t timeout_ms);
  // Copies a finished request's RGBA8 image; release() frees its buffer.
  void read_rgba8(uint64_t id, uint8_t *out, uint64_t len);
  void release(uint64_t id);
  ServeStats stats();
  void reset_stats();

 private:
  struct Request {
    uint64_t id;
    BatchView view;
    RequestInfo info;
    double t_submit = 0, t_launch = 0, t_done = 0;
    uint8_t *result = nullptr;
    uint64_t bytes = 0;
  };
  struct LaneState {
    std::unique_ptr<Lane> lane;
    bool busy = false;
    std::atomic<bool> completed{false};
    std::atomic<double> t_complete{0};
    std::vector<uint64_t> ids;          // requests of the running batch
    std::vector<ViewSpec> specs;
    std::vector<uint64_t> bases;
    std::vector<ViewGroup> groups;
    std::vector<uint8_t *> dst;         // pinned result buffers
    uint64_t admitted_bytes = 0;
    Server *server = nullptr;
  };
  static void on_lane_done(void *arg);
  void loop();
  bool launch(LaneState &ls, std::unique_lock<std::mutex> &lk);
  void retire(LaneState &ls, std::unique_lock<std::mutex> &lk);
  uint64_t view_bytes(const ViewSpec &s, uint64_t pairs) const;

  ServeConfig cfg_;
  int device_;
  cudaStream_t upload_stream_ = nullptr;
  SceneStore scenes_;
  PairPredictor predictor_;
  PinnedPool pool_;
  std::mutex mu_;
  std::condition_variable cv_;       // scheduler wake-ups
  std::condition_variable done_cv_;  // request completions
  std::deque<uint64_t> queue_;
  std::unordered_map<uint64_t, Request> requests_;
  // graph captures and pinned allocations over all lanes, so far
  void host_costs(uint64_t &captures, double &capture_ms, uint64_t &slabs, double &alloc_ms,
                  uint64_t &regrowths, double &regrowth_ms);
  uint64_t base_captures_ = 0, base_slabs_ = 0, base_regrowths_ = 0;  // at the last reset
  double base_capture_ms_ = 0, base_alloc_ms_ = 0, base_regrowth_ms_ = 0;
  std::vector<std::unique_ptr<LaneState>> lanes_;
  uint64_t next_id_ = 1;
  bool stop_ = false;
  // statistics since the last reset
  std::vector<double> latencies_;
  uint64_t submitted_ = 0, failed_ = 0, batches_ = 0, batch_views_ = 0, reruns_ = 0, shed_ = 0;
  uint64_t peak_admitted_ = 0;
  double first_submit_ = -1, last_done_ = 0;
  double device_ms_ = 0, launch_ms_ = 0, retire_ms_ = 0;
  std::thread thread_;
};

double now_ms();

}  // namespace gsr
