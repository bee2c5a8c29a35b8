// Autotuner of the batched launch shape: tile size (8 or 16), raster chunk
// size (records staged per step) and persistent raster blocks per SM. Every
// candidate renders the caller's views with the caller's batch; the fastest
// by median device time wins and is applied to the batch. Results persist in
// a small text file keyed by GPU name, blend mode, the set of image sizes and
// the scene-size class, so later processes reuse them without searching. No
// candidate changes a pixel, only the time.
#pragma once

#include <string>
#include <vector>

#include "batch.h"

namespace gsr {

struct TuneChoice {
  uint32_t tile = 16;
  RasterConfig raster;
  float ms = 0;  // median device time of the views
};

struct TuneResult {
  TuneChoice best;
  float default_ms = 0;  // tile 16, chunk 256, one block per tile
  std::vector<TuneChoice> tried;
  bool from_cache = false;
  std::string key;
};

// Candidate launch shapes, default first.
std::vector<TuneChoice> tune_candidates();
// Key of a workload: GPU name, blend mode, sorted distinct image sizes and
// log2 of the mean splat count of the views' scenes.
std::string tune_key(const std::string &gpu, uint32_t blend,
                     const std::vector<ViewSpec> &views);
// Cache file: a header line, then one "key<TAB>tile<TAB>chunk<TAB>bps<TAB>ms"
// line per entry. Unknown or malformed lines are ignored.
bool tune_cache_lookup(const std::string &path, const std::string &key, TuneChoice &out);
void tune_cache_store(const std::string &path, const std::string &key, const TuneChoice &c);

TuneResult autotune(Batch &batch, const std::vector<BatchView> &views, const std::string &cache_path,
                    uint32_t reps);

}  // namespace gsr
