// The batched engine's autotuner: a measured choice of frames per launch,
// threshold task height (seg_rows) and warps per block for one frame shape,
// kept in a tuner file that engines created without explicit tuning read.
//
// The reference makes the same kind of choice by measurement: its stage0 /
// stage2 windows default to what its benchmark harness found faster on its
// test GPU (src/dext_gpu.cc:18-37, tests/bench_dext_gpu.cc:242-337). Here the
// search runs on the caller's device, on the caller's frames, timed with
// CUDA events:
//
//   1. threshold alone, at one batch size: every warps-per-block count the
//      kernel supports x task heights around the cost model's choice (as a
//      ratio to it, so the choice carries over to other batch sizes);
//   2. the whole step, threshold + placement + 3D grouping on two slots as
//      the engine overlaps them, for each frames-per-launch candidate within
//      the caller's range, using the best ratio and warps from step 1;
//   3. at the best batch size, fewer threshold blocks per SM than fit: the
//      threshold then leaves registers and warp slots on every SM for the
//      previous batch's grouping kernels, which run beside it on the other
//      stream, instead of holding them until it ends.
//
// The tuner file holds one line per (pixel bytes, height, width, SM count,
// device name): frames per launch, warps per block, the task-height ratio,
// the measured time per frame. Results never depend on the tuning (every
// tuple gives byte-identical lists); only the time does.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/spotfinder_b200.h"
#include "sf_capi.hh"
#include "sf_engine.hh"

namespace sf {
namespace {

std::mutex g_tune_lock;

std::string device_name() {
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  cudaDeviceProp p;
  check(cudaGetDeviceProperties(&p, dev), "cudaGetDeviceProperties");
  std::string s = p.name;
  for (char &c : s)
    if (c == ' ' || c == '\t' || c == '=')
      c = '_';
  return s;
}

std::string make_key(int elem_bytes, int height, int width) {
  std::ostringstream k;
  k << "u" << 8 * elem_bytes << ":" << height << "x" << width << ":sm" << device_sm_count()
    << ":" << device_name();
  return k.str();
}

void make_parent_dirs(const std::string &path) {
  for (size_t at = path.find('/', 1); at != std::string::npos; at = path.find('/', at + 1))
    mkdir(path.substr(0, at).c_str(), 0755); // existing directories are fine
}

bool read_entry(const std::string &path, const std::string &key, TuneEntry *out) {
  std::ifstream in(path);
  if (!in)
    return false;
  std::string line;
  bool found = false;
  while (std::getline(in, line)) { // the last line for a key wins
    std::istringstream ls(line);
    std::string k;
    TuneEntry e;
    if (!(ls >> k >> e.frames >> e.warps_per_block >> e.seg_ratio >> e.us_per_frame))
      continue;
    if (!(ls >> e.blocks_per_sm) || e.blocks_per_sm < 0)
      e.blocks_per_sm = 0;
    if (k != key || e.frames < 1 || e.seg_ratio <= 0 ||
        (e.warps_per_block != 1 && e.warps_per_block != 2 && e.warps_per_block != 4))
      continue;
    *out = e;
    found = true;
  }
  return found;
}

void append_entry(const std::string &path, const std::string &key, const TuneEntry &e) {
  make_parent_dirs(path);
  std::ofstream o(path, std::ios::app);
  if (!o)
    return; // a read-only location: the result is still returned
  o << key << " " << e.frames << " " << e.warps_per_block << " " << e.seg_ratio << " "
    << e.us_per_frame << " " << e.blocks_per_sm << "\n";
}

// Milliseconds per frame of `steps` runs of an engine built for F frames of
// one shape, the sample cycled into its slots.
double time_engine(int elem_bytes, int height, int width, int F, const PlanTuning &t,
                   bool grouping, const void *const *sample, int nsample, int steps) {
  const int slots = grouping ? 2 : 1;
  std::vector<ThresholdPlan::Shape> shapes(F, ThresholdPlan::Shape{height, width});
  std::unique_ptr<Engine> e = make_engine(elem_bytes, shapes, t, slots);
  if (grouping)
    e->enable_grouping(GroupOptions{}, 0, 0);
  for (int s = 0; s < slots; s++)
    for (int f = 0; f < F; f++)
      e->upload(s, f, sample[(s * F + f) % nsample]);
  e->synchronize();
  for (int i = 0; i < 2 * slots; i++)
    e->run(i % slots);
  e->synchronize();
  e->record(e->marks[0]);
  for (int i = 0; i < steps; i++)
    e->run(i % slots);
  e->record(e->marks[1]);
  e->synchronize();
  float ms = 0;
  check(cudaEventElapsedTime(&ms, e->marks[0], e->marks[1]), "cudaEventElapsedTime");
  return static_cast<double>(ms) / (static_cast<double>(steps) * F);
}

// Rough device bytes an engine of F frames needs (arena, lists, staging and
// the labeller's live set), to keep candidates inside the budget.
uint64_t engine_bytes(int elem_bytes, int height, int width, int F) {
  const uint64_t px = static_cast<uint64_t>(height) * width;
  const uint64_t list = px * elem_bytes; // capacity x 16 B = the frame's bytes
  return 2ull * F * (px * elem_bytes + 3 * list) + 4ull * F * list;
}

} // namespace

std::string tune_cache_path(const char *given) {
  if (given && *given)
    return given;
  if (const char *env = std::getenv("SPOTFINDER_TUNE_CACHE"))
    if (*env)
      return env;
  if (const char *xdg = std::getenv("XDG_CACHE_HOME"))
    if (*xdg)
      return std::string(xdg) + "/spotfinder_b200/tune.txt";
  if (const char *home = std::getenv("HOME"))
    if (*home)
      return std::string(home) + "/.cache/spotfinder_b200/tune.txt";
  return "spotfinder_b200_tune.txt";
}

bool tune_lookup(int elem_bytes, int height, int width, const char *cache_path,
                 TuneEntry *out) {
  const std::lock_guard<std::mutex> hold(g_tune_lock);
  return read_entry(tune_cache_path(cache_path), make_key(elem_bytes, height, width), out);
}

int tune_seg_rows(int elem_bytes, const std::vector<ThresholdPlan::Shape> &shapes, int wpc,
                  double ratio, int blocks_per_sm) {
  const int base = model_seg_rows(elem_bytes, shapes, wpc, blocks_per_sm);
  int max_h = 1;
  for (const auto &s : shapes)
    max_h = std::max(max_h, s.height);
  const int seg = static_cast<int>(std::lround(base * ratio));
  return std::max(16, std::min(seg, max_h));
}

TuneResult tune_search(int elem_bytes, int height, int width, const void *const *sample,
                       int nsample, const TuneOptions &o) {
  const std::lock_guard<std::mutex> hold(g_tune_lock);
  const std::string path = tune_cache_path(o.cache_path);
  const std::string key = make_key(elem_bytes, height, width);
  TuneResult r;
  if (o.use_cache && read_entry(path, key, &r.entry) && r.entry.frames >= o.min_frames &&
      r.entry.frames <= o.max_frames) {
    r.from_cache = true;
    return r;
  }

  size_t free_b = 0, total_b = 0;
  check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
  const uint64_t budget = o.hbm_budget ? o.hbm_budget : free_b / 2;

  // 1. threshold alone at one batch size
  int F1 = std::min(std::max(16, o.min_frames), o.max_frames);
  while (F1 > 1 && engine_bytes(elem_bytes, height, width, F1) > budget)
    F1--;
  const std::vector<ThresholdPlan::Shape> shapes1(F1, ThresholdPlan::Shape{height, width});
  double best1 = 1e300;
  int best_wpc = 2;
  double best_ratio = 1.0;
  for (int wpc : {1, 2, 4}) {
    if ((elem_bytes == 2 ? threshold_occupancy<uint16_t>(wpc)
                         : threshold_occupancy<uint32_t>(wpc)) < 1)
      continue;
    int last_seg = -1;
    for (double ratio : {0.5, 0.75, 1.0, 1.5, 2.0}) {
      PlanTuning t;
      t.warps_per_block = wpc;
      t.seg_rows = tune_seg_rows(elem_bytes, shapes1, wpc, ratio);
      if (t.seg_rows == last_seg)
        continue;
      last_seg = t.seg_rows;
      const double ms =
          time_engine(elem_bytes, height, width, F1, t, false, sample, nsample, o.steps);
      r.candidates++;
      if (ms < best1) {
        best1 = ms;
        best_wpc = wpc;
        best_ratio = ratio;
      }
    }
  }

  // 2. the whole step for each batch size
  double best2 = 1e300;
  int best_f = F1;
  for (int F : {1, 2, 4, 8, 12, 16, 20, 24, 28, 32, 48, 64}) {
    if (F < o.min_frames || F > o.max_frames ||
        engine_bytes(elem_bytes, height, width, F) > budget)
      continue;
    const std::vector<ThresholdPlan::Shape> shapes(F, ThresholdPlan::Shape{height, width});
    PlanTuning t;
    t.warps_per_block = best_wpc;
    t.seg_rows = tune_seg_rows(elem_bytes, shapes, best_wpc, best_ratio);
    const double ms =
        time_engine(elem_bytes, height, width, F, t, o.grouping, sample, nsample, o.steps);
    r.candidates++;
    if (ms < best2) {
      best2 = ms;
      best_f = F;
    }
  }
  if (best2 == 1e300) { // no candidate inside the range and budget: step 1's size
    best_f = F1;
    best2 = best1;
  }
  // 3. threshold blocks per SM at that batch size
  int best_bps = 0;
  {
    const int occ = elem_bytes == 2 ? threshold_occupancy<uint16_t>(best_wpc)
                                    : threshold_occupancy<uint32_t>(best_wpc);
    const std::vector<ThresholdPlan::Shape> shapes(best_f, ThresholdPlan::Shape{height, width});
    int last = occ;
    for (int bps : {occ - 1, (3 * occ) / 4, occ / 2}) {
      if (bps < 1 || bps >= last)
        continue;
      last = bps;
      PlanTuning t;
      t.warps_per_block = best_wpc;
      t.blocks_per_sm = bps;
      t.seg_rows = tune_seg_rows(elem_bytes, shapes, best_wpc, best_ratio, bps);
      const double ms = time_engine(elem_bytes, height, width, best_f, t, o.grouping, sample,
                                    nsample, o.steps);
      r.candidates++;
      if (ms < best2) {
        best2 = ms;
        best_bps = bps;
      }
    }
  }
  r.entry.frames = best_f;
  r.entry.blocks_per_sm = best_bps;
  r.entry.warps_per_block = best_wpc;
  r.entry.seg_ratio = best_ratio;
  r.entry.us_per_frame = 1000.0 * best2;
  append_entry(path, key, r.entry);
  return r;
}

} // namespace sf

extern "C" int sf_tune(int elem_bytes, int height, int width, const void *const *sample_frames,
                       int nsample, const sf_tune_options *options, sf_tune_result *out) {
  return sf::guarded([&] {
    if ((elem_bytes != 2 && elem_bytes != 4) || height < 1 || width < 1 || out == nullptr ||
        sample_frames == nullptr || nsample < 1)
      return -1;
    for (int i = 0; i < nsample; i++)
      if (sample_frames[i] == nullptr)
        return -1;
    sf::TuneOptions o;
    if (options) {
      if (options->min_frames > 0)
        o.min_frames = options->min_frames;
      if (options->max_frames > 0)
        o.max_frames = options->max_frames;
      if (options->steps > 0)
        o.steps = options->steps;
      o.grouping = options->grouping != 0;
      o.use_cache = options->use_cache != 0;
      o.hbm_budget = options->hbm_budget;
      o.cache_path = options->cache_path;
    }
    if (o.min_frames > o.max_frames)
      return -1;
    const sf::TuneResult r =
        sf::tune_search(elem_bytes, height, width, sample_frames, nsample, o);
    const std::vector<sf::ThresholdPlan::Shape> shapes(
        r.entry.frames, sf::ThresholdPlan::Shape{height, width});
    out->frames_per_launch = r.entry.frames;
    out->warps_per_block = r.entry.warps_per_block;
    out->seg_rows = sf::tune_seg_rows(elem_bytes, shapes, r.entry.warps_per_block,
                                      r.entry.seg_ratio, r.entry.blocks_per_sm);
    out->blocks_per_sm = r.entry.blocks_per_sm;
    out->from_cache = r.from_cache ? 1 : 0;
    out->candidates = r.candidates;
    out->seg_ratio = r.entry.seg_ratio;
    out->us_per_frame = r.entry.us_per_frame;
    return 0;
  });
}
