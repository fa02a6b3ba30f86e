// The batched engine: many frames (equal or uneven shapes) thresholded per
// launch, with frames resident in `slots` device arenas so that uploads into
// one slot overlap the computation of another. Runs can be replayed from a
// CUDA graph captured per slot. This is the persistent batched form; the
// per-frame sf_find_* path (capi_find.cu) is the plain form.
//
// Streams: uploads go on a copy stream, runs on a compute stream; an event
// per slot orders "frames uploaded" before "run" and "run finished" before
// the next upload into the same slot.

#include <algorithm>
#include <memory>
#include <vector>

#include "../../include/spotfinder_b200.h"
#include "sf_capi.hh"
#include "sf_engine.hh"


namespace sf {

std::unique_ptr<Engine> make_engine(int elem_bytes, const std::vector<ThresholdPlan::Shape> &shapes,
                                    const PlanTuning &tuning, int slots) {
  auto e = std::make_unique<Engine>();
  check(cudaStreamCreateWithFlags(&e->compute, cudaStreamNonBlocking), "stream");
  check(cudaStreamCreateWithFlags(&e->copy, cudaStreamNonBlocking), "stream");
  check(cudaStreamCreateWithFlags(&e->group, cudaStreamNonBlocking), "stream");
  check(cudaEventCreateWithFlags(&e->join, cudaEventDisableTiming), "event");
  e->plan = std::make_unique<ThresholdPlan>(elem_bytes, shapes, tuning, slots);
  for (int s = 0; s < slots; s++) {
    cudaEvent_t u, c;
    check(cudaEventCreateWithFlags(&u, cudaEventDisableTiming), "event");
    e->uploaded.push_back(u);
    check(cudaEventCreateWithFlags(&c, cudaEventDisableTiming), "event");
    e->consumed.push_back(c);
    check(cudaEventRecord(u, e->copy), "event");
    check(cudaEventRecord(c, e->compute), "event");
    cudaEvent_t p, g;
    check(cudaEventCreateWithFlags(&p, cudaEventDisableTiming), "event");
    e->placed.push_back(p);
    check(cudaEventCreateWithFlags(&g, cudaEventDisableTiming), "event");
    e->grouped.push_back(g);
    check(cudaEventRecord(p, e->compute), "event");
    check(cudaEventRecord(g, e->group), "event");
  }
  e->thr_graphs.assign(slots, nullptr);
  e->graphs.assign(2 * slots, nullptr);
  e->hook_args.assign(slots, nullptr);
  for (cudaEvent_t &m : e->marks)
    check(cudaEventCreate(&m), "event");
  check(cudaMallocHost(&e->pinned, (shapes.size() + 1) * sizeof(uint32_t)), "cudaMallocHost");
  return e;
}

} // namespace sf

using sf::Engine;
using sf::guarded;

extern "C" {

int sf_engine_create(int elem_bytes, int nframes, const int32_t *heights,
                     const int32_t *widths, const sf_engine_config *config,
                     sf_engine **out) {
  return guarded([&] {
    if (out == nullptr || heights == nullptr || widths == nullptr || nframes < 1)
      return -1;
    *out = nullptr;
    std::vector<sf::ThresholdPlan::Shape> shapes;
    for (int i = 0; i < nframes; i++) {
      if (heights[i] < 1 || widths[i] < 1)
        return -1;
      shapes.push_back({heights[i], widths[i]});
    }
    sf::PlanTuning t;
    int slots = 1;
    bool automatic = true;
    if (config) {
      t.seg_rows = config->seg_rows;
      t.warps_per_block = config->warps_per_block > 0 ? config->warps_per_block : 0;
      t.blocks_per_sm = config->blocks_per_sm;
      slots = config->slots > 0 ? config->slots : 1;
      automatic = config->seg_rows == 0 && config->warps_per_block == 0;
    }
    bool uniform = true;
    for (const auto &sh : shapes)
      uniform = uniform && sh.height == shapes[0].height && sh.width == shapes[0].width;
    sf::TuneEntry tuned;
    const bool from_cache = automatic && uniform &&
                            sf::tune_lookup(elem_bytes, shapes[0].height, shapes[0].width,
                                            nullptr, &tuned);
    if (from_cache) {
      t.warps_per_block = tuned.warps_per_block;
      t.blocks_per_sm = tuned.blocks_per_sm;
      t.seg_rows = sf::tune_seg_rows(elem_bytes, shapes, tuned.warps_per_block, tuned.seg_ratio,
                                     tuned.blocks_per_sm);
    }
    auto e = sf::make_engine(elem_bytes, shapes, t, slots);
    e->tuned_from_cache = from_cache;
    *out = reinterpret_cast<sf_engine *>(e.release());
    return 0;
  });
}

void sf_engine_destroy(sf_engine *engine) { delete reinterpret_cast<Engine *>(engine); }

int sf_engine_tuning(sf_engine *engine, sf_tune_result *out) {
  return guarded([&] {
    if (!engine || !out)
      return -1;
    const Engine *e = reinterpret_cast<Engine *>(engine);
    *out = sf_tune_result{};
    out->frames_per_launch = e->plan->nframes();
    out->warps_per_block = e->plan->tuning().warps_per_block;
    out->seg_rows = e->plan->tuning().seg_rows;
    out->blocks_per_sm = e->plan->tuning().blocks_per_sm;
    out->from_cache = e->tuned_from_cache ? 1 : 0;
    return 0;
  });
}

int sf_engine_info(sf_engine *engine, int64_t *out8) {
  return guarded([&] {
    if (!engine || !out8)
      return -1;
    const Engine *e = reinterpret_cast<Engine *>(engine);
    out8[0] = e->plan->tuning().seg_rows;
    out8[1] = e->plan->tuning().warps_per_block;
    out8[2] = e->plan->grid_blocks();
    out8[3] = e->plan->ntasks();
    out8[4] = e->plan->nslots();
    out8[5] = static_cast<int64_t>(e->plan->device_bytes());
    out8[6] = static_cast<int64_t>(e->plan->pitch());
    out8[7] = static_cast<int64_t>(e->plan->total_capacity());
    return 0;
  });
}

int sf_engine_upload(sf_engine *engine, int slot, int frame, const void *host_image) {
  return guarded([&] {
    if (!engine || !host_image)
      return -1;
    reinterpret_cast<Engine *>(engine)->upload(slot, frame, host_image);
    return 0;
  });
}

int sf_engine_upload_device(sf_engine *engine, int slot, int frame, const void *device_image,
                            size_t pitch_bytes) {
  return guarded([&] {
    if (!engine || !device_image)
      return -1;
    reinterpret_cast<Engine *>(engine)->upload_device(slot, frame, device_image, pitch_bytes);
    return 0;
  });
}

int sf_engine_upload_chunk(sf_engine *engine, int slot, int frame, const void *chunk,
                           size_t nbytes, int algorithm) {
  return guarded([&] {
    if (!engine || !chunk)
      return -1;
    reinterpret_cast<Engine *>(engine)->upload_chunk(slot, frame, chunk, nbytes, algorithm);
    return 0;
  });
}

int sf_engine_upload_chunks(sf_engine *engine, int slot, size_t count, const int *frames,
                            const void *const *chunks, const size_t *nbytes, int algorithm) {
  return guarded([&] {
    if (!engine || (count && (!chunks || !nbytes)))
      return -1;
    for (size_t k = 0; k < count; k++)
      if (!chunks[k])
        return -1;
    reinterpret_cast<Engine *>(engine)->upload_chunks(slot, count, frames, chunks, nbytes,
                                                      algorithm);
    return 0;
  });
}

int sf_engine_set_pixel_mask(sf_engine *engine, int frame, const uint8_t *mask) {
  return guarded([&] {
    if (!engine)
      return -1;
    reinterpret_cast<Engine *>(engine)->set_pixel_mask(frame, mask);
    return 0;
  });
}

int sf_engine_run(sf_engine *engine, int slot) {
  return guarded([&] {
    if (!engine)
      return -1;
    reinterpret_cast<Engine *>(engine)->run(slot);
    return 0;
  });
}

int sf_engine_synchronize(sf_engine *engine) {
  return guarded([&] {
    if (!engine)
      return -1;
    reinterpret_cast<Engine *>(engine)->synchronize();
    return 0;
  });
}

int sf_engine_counts(sf_engine *engine, int slot, uint32_t *counts) {
  return guarded([&] {
    if (!engine || !counts)
      return -1;
    Engine *e = reinterpret_cast<Engine *>(engine);
    e->check_slot(slot);
    const int nf = e->plan->nframes();
    sf::check(cudaMemcpyAsync(e->pinned, e->plan->frame_count(slot), nf * sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, e->compute),
              "reading counts");
    sf::check(cudaStreamSynchronize(e->compute), "cudaStreamSynchronize");
    for (int f = 0; f < nf; f++)
      counts[f] = e->pinned[f];
    return 0;
  });
}

int sf_engine_signals(sf_engine *engine, int slot, sf_signal_pixel *out, size_t capacity,
                      uint32_t *counts) {
  return guarded([&] {
    if (!engine || !counts)
      return -1;
    Engine *e = reinterpret_cast<Engine *>(engine);
    e->check_slot(slot);
    const int nf = e->plan->nframes();
    sf::check(cudaMemcpyAsync(e->pinned, e->plan->frame_count(slot), nf * sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, e->compute),
              "reading the counts");
    sf::check(cudaStreamSynchronize(e->compute), "cudaStreamSynchronize");
    uint64_t total = 0;
    bool over = false;
    for (int f = 0; f < nf; f++) {
      counts[f] = e->pinned[f];
      over = over || counts[f] > e->plan->capacity(f);
      total += counts[f];
    }
    if (over || total > capacity)
      return -2;
    if (total > 0 && !out)
      return -1;
    uint64_t at = 0;
    for (int f = 0; f < nf; f++) {
      if (counts[f])
        sf::check(cudaMemcpyAsync(out + at, e->plan->out(slot) + e->plan->out_base(f),
                                  counts[f] * sizeof(sf::SignalPixel), cudaMemcpyDeviceToHost,
                                  e->compute),
                  "copying the signal pixels back");
      at += counts[f];
    }
    sf::check(cudaStreamSynchronize(e->compute), "cudaStreamSynchronize");
    return 0;
  });
}

int sf_engine_signal(sf_engine *engine, int slot, int frame, sf_signal_pixel *out,
                     size_t capacity, size_t *found) {
  return guarded([&] {
    if (!engine || !found)
      return -1;
    Engine *e = reinterpret_cast<Engine *>(engine);
    e->check_slot(slot);
    e->check_frame(frame);
    sf::check(cudaMemcpyAsync(e->pinned, e->plan->frame_count(slot) + frame, sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, e->compute),
              "reading the count");
    sf::check(cudaStreamSynchronize(e->compute), "cudaStreamSynchronize");
    const uint32_t n = e->pinned[0];
    *found = n;
    if (n > e->plan->capacity(frame) || n > capacity)
      return -2;
    if (n == 0)
      return 0;
    if (!out)
      return -1;
    sf::check(cudaMemcpyAsync(out, e->plan->out(slot) + e->plan->out_base(frame),
                              n * sizeof(sf::SignalPixel), cudaMemcpyDeviceToHost, e->compute),
              "copying the signal pixels back");
    sf::check(cudaStreamSynchronize(e->compute), "cudaStreamSynchronize");
    return 0;
  });
}

int sf_engine_use_graph(sf_engine *engine, int on) {
  return guarded([&] {
    if (!engine)
      return -1;
    Engine *e = reinterpret_cast<Engine *>(engine);
    if (on && e->profiling)
      throw std::invalid_argument("stage profiling is on: turn it off before graph replay");
    e->use_graph = on != 0;
    return 0;
  });
}

int sf_engine_record(sf_engine *engine, int mark) {
  return guarded([&] {
    if (!engine || mark < 0 || mark >= sf::kMarks)
      return -1;
    Engine *e = reinterpret_cast<Engine *>(engine);
    e->record(e->marks[mark]);
    return 0;
  });
}

int sf_engine_elapsed(sf_engine *engine, int from, int to, float *ms) {
  return guarded([&] {
    if (!engine || !ms || from < 0 || to < 0 || from >= sf::kMarks || to >= sf::kMarks)
      return -1;
    Engine *e = reinterpret_cast<Engine *>(engine);
    sf::check(cudaEventSynchronize(e->marks[to]), "cudaEventSynchronize");
    sf::check(cudaEventElapsedTime(ms, e->marks[from], e->marks[to]), "cudaEventElapsedTime");
    return 0;
  });
}

int sf_engine_profile(sf_engine *engine, int on) {
  return guarded([&] {
    if (!engine)
      return -1;
    Engine *e = reinterpret_cast<Engine *>(engine);
    if (on && e->ring.empty()) {
      e->ring.resize(sf::kRunEvents * sf::kRingRuns);
      for (cudaEvent_t &ev : e->ring)
        sf::check(cudaEventCreate(&ev), "event");
    }
    if (on && e->use_graph)
      throw std::invalid_argument("stage profiling times the launches one by one: "
                                  "turn graph replay off first");
    e->profiling = on != 0;
    e->ring_used = 0;
    return 0;
  });
}

int sf_engine_stage_totals(sf_engine *engine, double *out4) {
  return guarded([&] {
    if (!engine || !out4)
      return -1;
    Engine *e = reinterpret_cast<Engine *>(engine);
    double thr = 0, place = 0, group = 0;
    for (int i = 0; i < e->ring_used; i++) {
      cudaEvent_t *ev = &e->ring[sf::kRunEvents * i];
      float a = 0, b = 0, c = 0;
      sf::check(cudaEventSynchronize(ev[3]), "cudaEventSynchronize");
      sf::check(cudaEventElapsedTime(&a, ev[0], ev[1]), "elapsed");
      sf::check(cudaEventElapsedTime(&b, ev[1], ev[2]), "elapsed");
      sf::check(cudaEventElapsedTime(&c, ev[2], ev[3]), "elapsed");
      thr += a;
      place += b;
      group += c;
    }
    out4[0] = e->ring_used;
    out4[1] = thr;
    out4[2] = place;
    out4[3] = group;
    return 0;
  });
}

int sf_engine_enable_grouping(sf_engine *engine, const sf_group_options *options,
                              int64_t first_frame, uint64_t carry_capacity) {
  return guarded([&] {
    if (!engine)
      return -1;
    sf::GroupOptions opt;
    if (options) {
      opt.min_spot_size = options->min_spot_size;
      opt.max_spot_size = options->max_spot_size;
      opt.max_separation = options->max_separation;
      opt.two_d = options->two_d != 0;
    }
    reinterpret_cast<Engine *>(engine)->enable_grouping(opt, first_frame, carry_capacity);
    return 0;
  });
}

int sf_engine_nseries(sf_engine *engine) {
  if (!engine)
    return -1;
  return static_cast<int>(reinterpret_cast<Engine *>(engine)->series.size());
}

int sf_engine_series_shape(sf_engine *engine, int series, int32_t *height, int32_t *width) {
  return guarded([&] {
    if (!engine || !height || !width)
      return -1;
    const Engine::Series &se = reinterpret_cast<Engine *>(engine)->series_at(series);
    *height = se.height;
    *width = se.width;
    return 0;
  });
}

int sf_engine_series_counts(sf_engine *engine, int series, sf_counts *out, uint64_t *live) {
  return guarded([&] {
    if (!engine || !out)
      return -1;
    const sf::LabelScalars &s = reinterpret_cast<Engine *>(engine)->group_state(series);
    out->signal_pixels = s.signal_pixels;
    out->groups = s.groups;
    out->too_small = s.too_small;
    out->too_large = s.too_large;
    out->separated = s.separated;
    out->accepted = s.accepted;
    if (live)
      *live = s.carry_n;
    return 0;
  });
}

int sf_engine_series_spots(sf_engine *engine, int series, sf_spot *out, size_t capacity,
                           size_t *n) {
  return guarded([&] {
    if (!engine || !n)
      return -1;
    Engine *e = reinterpret_cast<Engine *>(engine);
    const sf::LabelScalars &s = e->group_state(series);
    *n = s.batch_spots;
    if (s.batch_spots > capacity)
      return -2;
    if (s.batch_spots) {
      // on the grouping stream, after the run that made them: a DMA straight
      // into page-locked memory, while the copy stream's uploads continue
      sf::check(cudaMemcpyAsync(out, e->series[series].lab->batch_spots(),
                                s.batch_spots * sizeof(sf::Spot), cudaMemcpyDeviceToHost, e->group),
                "reading spots");
      sf::check(cudaStreamSynchronize(e->group), "cudaStreamSynchronize");
    }
    return 0;
  });
}

int sf_engine_series_pixels(sf_engine *engine, int series, sf_pixel *out, size_t capacity,
                            size_t *n) {
  return guarded([&] {
    if (!engine || !n)
      return -1;
    Engine *e = reinterpret_cast<Engine *>(engine);
    const sf::LabelScalars &s = e->group_state(series);
    *n = s.batch_pixels;
    if (s.batch_pixels > capacity)
      return -2;
    if (s.batch_pixels) {
      // on the grouping stream, after the run that made them: a DMA straight
      // into page-locked memory, while the copy stream's uploads continue
      sf::check(cudaMemcpyAsync(out, e->series[series].lab->batch_pixels(),
                                s.batch_pixels * sizeof(sf::Pixel), cudaMemcpyDeviceToHost, e->group),
                "reading spot pixels");
      sf::check(cudaStreamSynchronize(e->group), "cudaStreamSynchronize");
    }
    return 0;
  });
}

int sf_engine_group_counts(sf_engine *engine, sf_counts *out, uint64_t *live) {
  return sf_engine_series_counts(engine, 0, out, live);
}

int sf_engine_spots(sf_engine *engine, sf_spot *out, size_t capacity, size_t *n) {
  return sf_engine_series_spots(engine, 0, out, capacity, n);
}

int sf_engine_pixels(sf_engine *engine, sf_pixel *out, size_t capacity, size_t *n) {
  return sf_engine_series_pixels(engine, 0, out, capacity, n);
}

int sf_engine_finish(sf_engine *engine) {
  return guarded([&] {
    if (!engine)
      return -1;
    Engine *e = reinterpret_cast<Engine *>(engine);
    if (e->series.empty())
      throw std::invalid_argument("grouping is not enabled");
    for (Engine::Series &se : e->series)
      se.lab->enqueue(0, e->plan->out(0), se.d_offs, e->plan->frame_count(0), se.d_map,
                      se.d_caps, true, e->group);
    e->parity ^= 1;
    return 0;
  });
}

} // extern "C"
