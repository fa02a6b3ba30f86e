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
#include "sf_codec.hh"
#include "sf_host.hh"
#include "sf_label.hh"

namespace sf {
namespace {

constexpr int kMarks = 16;
constexpr int kRingRuns = 4096;
constexpr int kRunEvents = 4;

} // namespace

struct Engine {
  std::unique_ptr<ThresholdPlan> plan;
  cudaStream_t compute = nullptr, copy = nullptr;
  std::vector<cudaEvent_t> uploaded, consumed; // per slot
  // Graphs per (slot, labeller parity): the labeller alternates between two
  // live buffers, so a captured run is only valid for the parity it saw.
  std::vector<cudaGraphExec_t> graphs;
  bool use_graph = false;
  cudaEvent_t marks[kMarks] = {};
  // Profiling: per run, events before the threshold, between threshold and
  // placement, after the placement and after the grouping.
  bool profiling = false;
  std::vector<cudaEvent_t> ring;
  int ring_used = 0;
  uint32_t *pinned = nullptr;
  // Grouping, when enabled: frames of one shape are one series, with its
  // own labeller and the device copies of its frames' list offsets,
  // capacities and plan frame numbers.
  struct Series {
    std::unique_ptr<DeviceLabeller> lab;
    uint64_t *d_offs = nullptr;
    uint32_t *d_caps = nullptr;
    int32_t *d_map = nullptr;
    int nframes = 0;
    int32_t height = 0, width = 0;
  };
  std::vector<Series> series;
  int parity = 0;
  LabelScalars *host_sc = nullptr;
  // Compressed uploads, decoded on the device in the copy stream.
  DeviceChunkDecoder decoder;

  ~Engine() {
    if (compute)
      cudaStreamSynchronize(compute);
    if (copy)
      cudaStreamSynchronize(copy);
    for (cudaGraphExec_t g : graphs)
      if (g)
        cudaGraphExecDestroy(g);
    for (Series &se : series) {
      se.lab.reset();
      cudaFree(se.d_offs);
      cudaFree(se.d_caps);
      cudaFree(se.d_map);
    }
    if (host_sc)
      cudaFreeHost(host_sc);
    for (cudaEvent_t e : uploaded)
      cudaEventDestroy(e);
    for (cudaEvent_t e : consumed)
      cudaEventDestroy(e);
    for (cudaEvent_t e : marks)
      if (e)
        cudaEventDestroy(e);
    for (cudaEvent_t e : ring)
      cudaEventDestroy(e);
    if (pinned)
      cudaFreeHost(pinned);
    plan.reset();
    if (compute)
      cudaStreamDestroy(compute);
    if (copy)
      cudaStreamDestroy(copy);
  }

  void check_slot(int slot) const {
    if (slot < 0 || slot >= plan->nslots())
      throw std::out_of_range("slot out of range");
  }
  void check_frame(int frame) const {
    if (frame < 0 || frame >= plan->nframes())
      throw std::out_of_range("frame out of range");
  }

  // Threshold, placement and (when enabled) grouping of one slot.
  void enqueue_body(int slot, cudaEvent_t b, cudaEvent_t c) {
    plan->enqueue(slot, compute, b);
    if (c)
      check(cudaEventRecord(c, compute), "cudaEventRecord");
    for (Series &se : series)
      se.lab->enqueue(se.nframes, plan->out(slot), se.d_offs, plan->frame_count(slot), se.d_map,
                      se.d_caps, false, compute);
  }

  void enqueue_run(int slot, cudaEvent_t a, cudaEvent_t b, cudaEvent_t c, cudaEvent_t d) {
    if (a)
      check(cudaEventRecord(a, compute), "cudaEventRecord");
    if (use_graph) {
      cudaGraphExec_t &exec = graphs[2 * slot + parity];
      if (!exec) {
        cudaGraph_t g = nullptr;
        check(cudaStreamBeginCapture(compute, cudaStreamCaptureModeThreadLocal),
              "beginning graph capture");
        try {
          enqueue_body(slot, nullptr, nullptr);
        } catch (...) {
          cudaStreamEndCapture(compute, &g);
          if (g)
            cudaGraphDestroy(g);
          throw;
        }
        check(cudaStreamEndCapture(compute, &g), "ending graph capture");
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        check(e, "instantiating the graph");
      } else {
        for (Series &se : series)
          se.lab->note_replayed(); // the captured run flips the live buffers too
      }
      check(cudaGraphLaunch(exec, compute), "launching the graph");
    } else {
      enqueue_body(slot, b, c);
    }
    if (d)
      check(cudaEventRecord(d, compute), "cudaEventRecord");
    if (!series.empty())
      parity ^= 1;
  }

  void run(int slot) {
    check_slot(slot);
    check(cudaStreamWaitEvent(compute, uploaded[slot], 0), "ordering after the upload");
    cudaEvent_t a = nullptr, b = nullptr, c = nullptr, d = nullptr;
    if (profiling && ring_used < kRingRuns) {
      cudaEvent_t *e = &ring[kRunEvents * ring_used];
      a = e[0];
      b = e[1];
      c = e[2];
      d = e[3];
      ring_used++;
    }
    enqueue_run(slot, a, b, c, d);
    check(cudaEventRecord(consumed[slot], compute), "cudaEventRecord");
  }

  // Frames of one shape are the consecutive frames of one series, numbered
  // from first_frame in their order within the batch and advancing run by
  // run; each series is grouped by its own labeller, in the run's stream.
  void enable_grouping(const GroupOptions &opt, int64_t first_frame, uint64_t carry_cap) {
    if (!series.empty())
      throw std::invalid_argument("grouping is already enabled");
    const int nf = plan->nframes();
    std::vector<std::vector<int32_t>> members;
    for (int f = 0; f < nf; f++) {
      size_t k = 0;
      while (k < series.size() && (series[k].height != plan->shape(f).height ||
                                   series[k].width != plan->shape(f).width))
        k++;
      if (k == series.size()) {
        series.emplace_back();
        series.back().height = plan->shape(f).height;
        series.back().width = plan->shape(f).width;
        members.emplace_back();
      }
      members[k].push_back(f);
    }
    check(cudaMallocHost(&host_sc, sizeof(LabelScalars)), "cudaMallocHost");
    for (size_t k = 0; k < series.size(); k++) {
      Series &se = series[k];
      const std::vector<int32_t> &fs = members[k];
      se.nframes = static_cast<int>(fs.size());
      std::vector<uint64_t> offs;
      std::vector<uint32_t> caps;
      uint64_t total = 0, biggest = 0;
      for (int32_t f : fs) {
        offs.push_back(plan->out_base(f));
        caps.push_back(plan->capacity(f));
        total += plan->capacity(f);
        biggest = std::max<uint64_t>(biggest, plan->capacity(f));
      }
      const size_t n = fs.size();
      check(cudaMalloc(&se.d_offs, n * sizeof(uint64_t)), "cudaMalloc");
      check(cudaMalloc(&se.d_caps, n * sizeof(uint32_t)), "cudaMalloc");
      check(cudaMalloc(&se.d_map, n * sizeof(int32_t)), "cudaMalloc");
      check(cudaMemcpy(se.d_offs, offs.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice),
            "copy");
      check(cudaMemcpy(se.d_caps, caps.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice),
            "copy");
      check(cudaMemcpy(se.d_map, fs.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice), "copy");
      se.lab = std::make_unique<DeviceLabeller>(se.height, se.width, opt);
      se.lab->reserve(total, se.nframes, carry_cap ? carry_cap : 2 * biggest + (1u << 20));
      se.lab->set_next_frame(first_frame, compute);
    }
    check(cudaStreamSynchronize(compute), "cudaStreamSynchronize");
    parity = 0;
  }

  Series &series_at(int k) {
    if (series.empty())
      throw std::invalid_argument("grouping is not enabled");
    if (k < 0 || k >= static_cast<int>(series.size()))
      throw std::out_of_range("series out of range");
    return series[k];
  }

  const LabelScalars &group_state(int k) {
    Series &se = series_at(k);
    check(cudaMemcpyAsync(host_sc, se.lab->scalars(), sizeof(LabelScalars),
                          cudaMemcpyDeviceToHost, compute),
          "reading the grouping state");
    check(cudaStreamSynchronize(compute), "cudaStreamSynchronize");
    if (host_sc->status != kLabelOk)
      throw DeviceError("grouping capacity exceeded (status " + std::to_string(host_sc->status) +
                        ")");
    return *host_sc;
  }

  void upload(int slot, int frame, const void *host) {
    check_slot(slot);
    check_frame(frame);
    check(cudaStreamWaitEvent(copy, consumed[slot], 0), "ordering after the last run");
    plan->upload(slot, frame, host, copy);
    check(cudaEventRecord(uploaded[slot], copy), "cudaEventRecord");
  }

  void upload_device(int slot, int frame, const void *dev, size_t pitch) {
    check_slot(slot);
    check_frame(frame);
    check(cudaStreamWaitEvent(copy, consumed[slot], 0), "ordering after the last run");
    plan->upload_device(slot, frame, dev, pitch, copy);
    check(cudaEventRecord(uploaded[slot], copy), "cudaEventRecord");
  }

  void upload_chunk(int slot, int frame, const void *chunk, size_t nbytes, int algorithm) {
    check_slot(slot);
    check_frame(frame);
    const ThresholdPlan::Shape &sh = plan->shape(frame);
    const size_t eb = static_cast<size_t>(plan->elem_bytes());
    const ChunkLayout L = parse_chunk(algorithm, static_cast<const uint8_t *>(chunk), nbytes,
                                      static_cast<size_t>(sh.height) * sh.width, eb);
    check(cudaStreamWaitEvent(copy, consumed[slot], 0), "ordering after the last run");
    decoder.enqueue(static_cast<const uint8_t *>(chunk), nbytes, L, sh.height, sh.width,
                    plan->frame_origin(slot, frame), plan->pitch() * eb, copy);
    check(cudaEventRecord(uploaded[slot], copy), "cudaEventRecord");
  }

  void synchronize() {
    check(cudaStreamSynchronize(copy), "cudaStreamSynchronize");
    check(cudaStreamSynchronize(compute), "cudaStreamSynchronize");
    if (decoder.take_error())
      throw DeviceError("an uploaded chunk held a malformed LZ4 block");
    for (int s = 0; s < plan->nslots(); s++) {
      int status = 0;
      check(cudaMemcpy(&status, plan->status(s), sizeof(int), cudaMemcpyDeviceToHost),
            "reading the status");
      if (status == kStatusTmaTimeout)
        throw DeviceError("a TMA load did not complete in time");
      if (status == kStatusSpinTimeout)
        throw DeviceError("a device wait gave up");
    }
  }
};

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
    if (config) {
      t.seg_rows = config->seg_rows;
      t.warps_per_block = config->warps_per_block > 0 ? config->warps_per_block : 4;
      t.blocks_per_sm = config->blocks_per_sm;
      slots = config->slots > 0 ? config->slots : 1;
    }
    auto e = std::make_unique<Engine>();
    sf::check(cudaStreamCreateWithFlags(&e->compute, cudaStreamNonBlocking), "stream");
    sf::check(cudaStreamCreateWithFlags(&e->copy, cudaStreamNonBlocking), "stream");
    e->plan = std::make_unique<sf::ThresholdPlan>(elem_bytes, shapes, t, slots);
    for (int s = 0; s < slots; s++) {
      cudaEvent_t u, c;
      sf::check(cudaEventCreateWithFlags(&u, cudaEventDisableTiming), "event");
      e->uploaded.push_back(u);
      sf::check(cudaEventCreateWithFlags(&c, cudaEventDisableTiming), "event");
      e->consumed.push_back(c);
      sf::check(cudaEventRecord(u, e->copy), "event");
      sf::check(cudaEventRecord(c, e->compute), "event");
    }
    e->graphs.assign(2 * slots, nullptr);
    for (cudaEvent_t &m : e->marks)
      sf::check(cudaEventCreate(&m), "event");
    sf::check(cudaMallocHost(&e->pinned, (nframes + 1) * sizeof(uint32_t)), "cudaMallocHost");
    *out = reinterpret_cast<sf_engine *>(e.release());
    return 0;
  });
}

void sf_engine_destroy(sf_engine *engine) { delete reinterpret_cast<Engine *>(engine); }

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
    sf::check(cudaEventRecord(e->marks[mark], e->compute), "cudaEventRecord");
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
    if (s.batch_spots)
      sf::check(cudaMemcpy(out, e->series[series].lab->batch_spots(),
                           s.batch_spots * sizeof(sf::Spot), cudaMemcpyDeviceToHost),
                "reading spots");
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
    if (s.batch_pixels)
      sf::check(cudaMemcpy(out, e->series[series].lab->batch_pixels(),
                           s.batch_pixels * sizeof(sf::Pixel), cudaMemcpyDeviceToHost),
                "reading spot pixels");
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
                      se.d_caps, true, e->compute);
    e->parity ^= 1;
    return 0;
  });
}

} // extern "C"
