// The batched engine: many frames (equal or uneven shapes) thresholded per
// launch, with frames resident in `slots` device arenas so that uploads into
// one slot overlap the computation of another. Runs can be replayed from a
// CUDA graph captured per slot. This is the persistent batched form; the
// per-frame sf_find_* path (capi_find.cu) is the plain form.
//
// Streams: uploads go on a copy stream, runs on a compute stream; an event
// per slot orders "frames uploaded" before "run" and "run finished" before
// the next upload into the same slot.

#include <memory>
#include <vector>

#include "../../include/spotfinder_b200.h"
#include "sf_capi.hh"
#include "sf_host.hh"

namespace sf {
namespace {

constexpr int kMarks = 16;
constexpr int kRingRuns = 4096;

} // namespace

struct Engine {
  std::unique_ptr<ThresholdPlan> plan;
  cudaStream_t compute = nullptr, copy = nullptr;
  std::vector<cudaEvent_t> uploaded, consumed; // per slot
  std::vector<cudaGraphExec_t> graphs;         // per slot, when in use
  bool use_graph = false;
  cudaEvent_t marks[kMarks] = {};
  // Profiling: per run, events before the threshold, between threshold and
  // placement, and after the placement.
  bool profiling = false;
  std::vector<cudaEvent_t> ring;
  int ring_used = 0;
  uint32_t *pinned = nullptr;

  ~Engine() {
    if (compute)
      cudaStreamSynchronize(compute);
    if (copy)
      cudaStreamSynchronize(copy);
    for (cudaGraphExec_t g : graphs)
      if (g)
        cudaGraphExecDestroy(g);
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

  void enqueue_run(int slot, cudaEvent_t a, cudaEvent_t b, cudaEvent_t c) {
    if (a)
      check(cudaEventRecord(a, compute), "cudaEventRecord");
    if (use_graph) {
      if (!graphs[slot]) {
        cudaGraph_t g = nullptr;
        check(cudaStreamBeginCapture(compute, cudaStreamCaptureModeThreadLocal),
              "beginning graph capture");
        try {
          plan->enqueue(slot, compute, nullptr);
        } catch (...) {
          cudaStreamEndCapture(compute, &g);
          if (g)
            cudaGraphDestroy(g);
          throw;
        }
        check(cudaStreamEndCapture(compute, &g), "ending graph capture");
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        check(e, "instantiating the graph");
        graphs[slot] = exec;
      }
      check(cudaGraphLaunch(graphs[slot], compute), "launching the graph");
      if (b)
        check(cudaEventRecord(b, compute), "cudaEventRecord");
    } else {
      plan->enqueue(slot, compute, b);
    }
    if (c)
      check(cudaEventRecord(c, compute), "cudaEventRecord");
  }

  void run(int slot) {
    check_slot(slot);
    check(cudaStreamWaitEvent(compute, uploaded[slot], 0), "ordering after the upload");
    cudaEvent_t a = nullptr, b = nullptr, c = nullptr;
    if (profiling && ring_used < kRingRuns) {
      a = ring[3 * ring_used];
      b = ring[3 * ring_used + 1];
      c = ring[3 * ring_used + 2];
      ring_used++;
    }
    enqueue_run(slot, a, b, c);
    check(cudaEventRecord(consumed[slot], compute), "cudaEventRecord");
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

  void synchronize() {
    check(cudaStreamSynchronize(copy), "cudaStreamSynchronize");
    check(cudaStreamSynchronize(compute), "cudaStreamSynchronize");
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
    e->graphs.assign(slots, nullptr);
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
    reinterpret_cast<Engine *>(engine)->use_graph = on != 0;
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
      e->ring.resize(3 * sf::kRingRuns);
      for (cudaEvent_t &ev : e->ring)
        sf::check(cudaEventCreate(&ev), "event");
    }
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
    double thr = 0, place = 0;
    for (int i = 0; i < e->ring_used; i++) {
      float a = 0, b = 0;
      sf::check(cudaEventSynchronize(e->ring[3 * i + 2]), "cudaEventSynchronize");
      sf::check(cudaEventElapsedTime(&a, e->ring[3 * i], e->ring[3 * i + 1]), "elapsed");
      sf::check(cudaEventElapsedTime(&b, e->ring[3 * i + 1], e->ring[3 * i + 2]), "elapsed");
      thr += a;
      place += b;
    }
    out4[0] = e->ring_used;
    out4[1] = thr;
    out4[2] = place;
    out4[3] = 0.0;
    return 0;
  });
}

} // extern "C"
