// Autotuner of the batched launch shape (host only).

#include "autotune.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <set>
#include <sstream>

#include "cuda_check.h"

namespace gsr {

namespace {
const char *kHeader = "gsplat-cuda-autotune v1";
}

std::vector<TuneChoice> tune_candidates() {
  std::vector<TuneChoice> c;
  for (uint32_t bps : {0u, 2u, 4u})
    for (uint32_t chunk : {256u, 128u, 64u}) {
      TuneChoice t;
      t.tile = 16;
      t.raster.chunk = chunk;
      t.raster.blocks_per_sm = bps;
      c.push_back(t);
    }
  for (uint32_t bps : {0u, 8u, 16u})
    for (uint32_t chunk : {64u, 32u}) {
      TuneChoice t;
      t.tile = 8;
      t.raster.chunk = chunk;
      t.raster.blocks_per_sm = bps;
      c.push_back(t);
    }
  return c;
}

std::string tune_key(const std::string &gpu, uint32_t blend, const std::vector<ViewSpec> &views) {
  std::set<std::pair<uint32_t, uint32_t>> sizes;
  double splats = 0;
  for (const auto &v : views) {
    sizes.insert({v.width, v.height});
    splats += v.scene->n;
  }
  const int cls = views.empty() ? 0 : (int)std::lround(std::log2(std::max(1.0, splats / views.size())));
  std::ostringstream k;
  for (char ch : gpu) k << (ch == '\t' || ch == '\n' || ch == ' ' ? '_' : ch);
  k << "|blend" << blend << "|";
  bool first = true;
  for (auto &s : sizes) {
    k << (first ? "" : ",") << s.first << "x" << s.second;
    first = false;
  }
  k << "|splats2^" << cls;
  return k.str();
}

bool tune_cache_lookup(const std::string &path, const std::string &key, TuneChoice &out) {
  if (path.empty()) return false;
  std::ifstream f(path);
  if (!f) return false;
  std::string line;
  if (!std::getline(f, line) || line != kHeader) return false;
  bool found = false;
  while (std::getline(f, line)) {
    std::istringstream ls(line);
    std::string k;
    TuneChoice c;
    if (!std::getline(ls, k, '\t')) continue;
    if (!(ls >> c.tile >> c.raster.chunk >> c.raster.blocks_per_sm >> c.ms)) continue;
    if (k == key && (c.tile == 8 || c.tile == 16) && raster_config_valid(c.tile, c.raster)) {
      out = c;  // the last entry for a key wins
      found = true;
    }
  }
  return found;
}

void tune_cache_store(const std::string &path, const std::string &key, const TuneChoice &c) {
  if (path.empty()) return;
  std::map<std::string, std::string> entries;
  {
    std::ifstream f(path);
    std::string line;
    if (f && std::getline(f, line) && line == kHeader)
      while (std::getline(f, line)) {
        auto tab = line.find('\t');
        if (tab != std::string::npos) entries[line.substr(0, tab)] = line;
      }
  }
  std::ostringstream e;
  e << key << '\t' << c.tile << '\t' << c.raster.chunk << '\t' << c.raster.blocks_per_sm << '\t'
    << c.ms;
  entries[key] = e.str();
  const std::string tmp = path + ".tmp";
  {
    std::ofstream f(tmp, std::ios::trunc);
    if (!f) throw Error(Code::InvalidArgument, "cannot write the autotune cache " + path);
    f << kHeader << '\n';
    for (auto &kv : entries) f << kv.second << '\n';
  }
  if (std::rename(tmp.c_str(), path.c_str()) != 0)
    throw Error(Code::InvalidArgument, "cannot replace the autotune cache " + path);
}

TuneResult autotune(Batch &batch, const std::vector<BatchView> &views, const std::string &cache_path,
                    uint32_t reps) {
  if (views.empty()) throw Error(Code::InvalidArgument, "no views to tune on");
  reps = std::max(reps, 1u);
  cudaDeviceProp prop;
  GSR_CUDA(cudaGetDeviceProperties(&prop, batch.device()));
  std::vector<ViewSpec> specs;
  std::vector<uint64_t> bases;
  make_view_specs(batch.scenes(), views.data(), (uint32_t)views.size(), specs, bases);
  TuneResult r;
  r.key = tune_key(prop.name, batch.blend_mode(), specs);
  TuneChoice cached;
  if (tune_cache_lookup(cache_path, r.key, cached)) {
    batch.set_tile(cached.tile);
    batch.set_raster_config(cached.raster);
    r.best = cached;
    r.from_cache = true;
    return r;
  }
  const uint32_t saved_tile = batch.tile();
  const RasterConfig saved_raster = batch.raster_config();
  try {
    for (TuneChoice c : tune_candidates()) {
      batch.set_tile(c.tile);
      batch.set_raster_config(c.raster);
      batch.render(views);  // warm-up: buffers, pair predictions, graph
      std::vector<float> ms;
      for (uint32_t k = 0; k < reps; ++k) ms.push_back(batch.render(views).device_ms);
      std::sort(ms.begin(), ms.end());
      c.ms = ms[ms.size() / 2];
      r.tried.push_back(c);
      if (r.tried.size() == 1) r.default_ms = c.ms;
    }
  } catch (...) {
    batch.set_tile(saved_tile);
    batch.set_raster_config(saved_raster);
    throw;
  }
  r.best = *std::min_element(r.tried.begin(), r.tried.end(),
                             [](const TuneChoice &a, const TuneChoice &b) { return a.ms < b.ms; });
  batch.set_tile(r.best.tile);
  batch.set_raster_config(r.best.raster);
  tune_cache_store(cache_path, r.key, r.best);
  return r;
}

}  // namespace gsr
