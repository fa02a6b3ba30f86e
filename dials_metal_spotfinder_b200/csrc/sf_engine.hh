// The batched engine's state (capi_engine.cu holds the C entry points; the
// serving loop in server.cu drives engines directly). Not part of the
// public C ABI.
#pragma once

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "sf_codec.hh"
#include "sf_host.hh"
#include "sf_label.hh"
#include "sf_pool.hh"

namespace sf {

constexpr int kMarks = 16;
constexpr int kRingRuns = 4096;
constexpr int kRunEvents = 4;

struct Engine {
  std::unique_ptr<ThresholdPlan> plan;
  bool tuned_from_cache = false; // the plan's tuning came from the tuner file
  // Streams: uploads on `copy`; threshold and placement on `compute`; the
  // grouping, when enabled, on `group`, so that the next run's threshold
  // overlaps this run's grouping. Per slot, events order the upload before
  // the threshold (uploaded), the threshold before the next upload
  // (consumed), the placement before the grouping (placed) and the grouping
  // before the slot's lists are overwritten (grouped).
  cudaStream_t compute = nullptr, copy = nullptr, group = nullptr;
  std::vector<cudaEvent_t> uploaded, consumed, placed, grouped;
  cudaEvent_t join = nullptr; // the compute stream's work, for the group stream
  int last_slot = -1;
  // Graphs: per slot, the threshold and placement; per (slot, labeller
  // parity), the grouping -- the labeller alternates between two live
  // buffers, so a captured grouping is only valid for the parity it saw.
  std::vector<cudaGraphExec_t> thr_graphs;
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
  // Host threads for the framing walks of a batch of chunks, made on first
  // use.
  std::unique_ptr<HostPool> pool;
  // Host callbacks in the run's stream, captured into its graphs too: after
  // the signal lists are placed and after the grouping, each given its
  // slot's argument. Set them before the first run.
  cudaHostFn_t on_mask = nullptr, on_done = nullptr;
  std::vector<void *> hook_args;
  // Enqueued after the grouping and before on_done, for work that must see
  // the run's results before the next run overwrites them.
  void (*post_run)(Engine &engine, int slot, void *arg) = nullptr;
  void *post_arg = nullptr;
  // The pixel mask: per frame, the masked pixels' element offsets from frame
  // 0's origin (the same in every slot), and all of them on the device.
  std::vector<std::vector<uint64_t>> mask_offsets;
  uint64_t *d_mask = nullptr;
  uint64_t mask_n = 0;

  ~Engine() {
    if (compute)
      cudaStreamSynchronize(compute);
    if (copy)
      cudaStreamSynchronize(copy);
    if (group)
      cudaStreamSynchronize(group);
    drop_graphs();
    cudaFree(d_mask);
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
    for (cudaEvent_t e : placed)
      cudaEventDestroy(e);
    for (cudaEvent_t e : grouped)
      cudaEventDestroy(e);
    if (join)
      cudaEventDestroy(join);
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
    if (group)
      cudaStreamDestroy(group);
  }

  void drop_graphs() {
    for (cudaGraphExec_t &g : graphs)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
    for (cudaGraphExec_t &g : thr_graphs)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }

  void check_slot(int slot) const {
    if (slot < 0 || slot >= plan->nslots())
      throw std::out_of_range("slot out of range");
  }
  void check_frame(int frame) const {
    if (frame < 0 || frame >= plan->nframes())
      throw std::out_of_range("frame out of range");
  }

  // Threshold and placement of one slot, on the compute stream.
  void enqueue_threshold(int slot, cudaEvent_t b, cudaEvent_t c) {
    if (mask_n)
      check(launch_stamp_mask(plan->frame_origin(slot, 0), plan->elem_bytes(), d_mask, mask_n,
                              compute),
            "launching the mask stamp");
    plan->enqueue(slot, compute, b);
    if (c)
      check(cudaEventRecord(c, compute), "cudaEventRecord");
    if (on_mask)
      check(cudaLaunchHostFunc(compute, on_mask, hook_args[slot]), "cudaLaunchHostFunc");
  }

  // Grouping of one slot's lists, on the group stream.
  void enqueue_grouping(int slot) {
    for (Series &se : series)
      se.lab->enqueue(se.nframes, plan->out(slot), se.d_offs, plan->frame_count(slot), se.d_map,
                      se.d_caps, false, group);
    if (post_run)
      post_run(*this, slot, post_arg);
    if (on_done)
      check(cudaLaunchHostFunc(group, on_done, hook_args[slot]), "cudaLaunchHostFunc");
  }

  // Enqueues `body` on `s`, through a graph captured on first use.
  template <class Body> void replay(cudaGraphExec_t &exec, cudaStream_t s, Body body) {
    if (!exec) {
      cudaGraph_t g = nullptr;
      check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal),
            "beginning graph capture");
      try {
        body();
      } catch (...) {
        cudaStreamEndCapture(s, &g);
        if (g)
          cudaGraphDestroy(g);
        throw;
      }
      check(cudaStreamEndCapture(s, &g), "ending graph capture");
      const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
      cudaGraphDestroy(g);
      check(e, "instantiating the graph");
      return; // capturing did not run it
    }
    check(cudaGraphLaunch(exec, s), "launching the graph");
  }

  void enqueue_run(int slot, cudaEvent_t a, cudaEvent_t b, cudaEvent_t c, cudaEvent_t d) {
    if (series.empty()) {
      if (a)
        check(cudaEventRecord(a, compute), "cudaEventRecord");
      if (use_graph) {
        bool fresh = !thr_graphs[slot];
        replay(thr_graphs[slot], compute, [&] { enqueue_threshold(slot, nullptr, nullptr); });
        if (fresh)
          replay(thr_graphs[slot], compute, [] {});
      } else {
        enqueue_threshold(slot, b, c);
      }
      if (d)
        check(cudaEventRecord(d, compute), "cudaEventRecord");
      return;
    }
    // the slot's lists are free once its last grouping has read them; when
    // profiling, the runs are kept apart so each stage times alone
    check(cudaStreamWaitEvent(compute, grouped[slot], 0), "ordering after the grouping");
    if (profiling && last_slot >= 0)
      check(cudaStreamWaitEvent(compute, grouped[last_slot], 0), "ordering after the grouping");
    if (a)
      check(cudaEventRecord(a, compute), "cudaEventRecord");
    if (use_graph) {
      const bool fresh = !thr_graphs[slot];
      replay(thr_graphs[slot], compute, [&] { enqueue_threshold(slot, nullptr, nullptr); });
      if (fresh)
        replay(thr_graphs[slot], compute, [] {});
    } else {
      enqueue_threshold(slot, b, c);
    }
    check(cudaEventRecord(placed[slot], compute), "cudaEventRecord");
    check(cudaStreamWaitEvent(group, placed[slot], 0), "ordering after the placement");
    if (use_graph) {
      cudaGraphExec_t &exec = graphs[2 * slot + parity];
      if (!exec) {
        // capturing records the run and flips the host's record of the live
        // buffers, as the run about to be launched will flip them
        replay(exec, group, [&] { enqueue_grouping(slot); });
        replay(exec, group, [] {});
      } else {
        replay(exec, group, [] {});
        for (Series &se : series)
          se.lab->note_replayed(); // the captured run flips the live buffers too
      }
    } else {
      enqueue_grouping(slot);
    }
    if (d)
      check(cudaEventRecord(d, group), "cudaEventRecord");
    check(cudaEventRecord(grouped[slot], group), "cudaEventRecord");
    last_slot = slot;
    parity ^= 1;
  }

  // A timing mark after everything enqueued so far, on either stream.
  void record(cudaEvent_t ev) {
    if (series.empty()) {
      check(cudaEventRecord(ev, compute), "cudaEventRecord");
      return;
    }
    check(cudaEventRecord(join, compute), "cudaEventRecord");
    check(cudaStreamWaitEvent(group, join, 0), "cudaStreamWaitEvent");
    check(cudaEventRecord(ev, group), "cudaEventRecord");
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
      se.lab->set_next_frame(first_frame, group);
    }
    check(cudaStreamSynchronize(group), "cudaStreamSynchronize");
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
                          cudaMemcpyDeviceToHost, group),
          "reading the grouping state");
    check(cudaStreamSynchronize(group), "cudaStreamSynchronize");
    if (host_sc->status != kLabelOk)
      throw DeviceError("grouping capacity exceeded (status " + std::to_string(host_sc->status) +
                        ")");
    return *host_sc;
  }

  void upload(int slot, int frame, const void *host) {
    check_slot(slot);
    check_frame(frame);
    check(cudaStreamWaitEvent(copy, consumed[slot], 0), "ordering after the last run");
    // one contiguous copy on the decoder's stream (the next frame's overlaps
    // this one's placement), laid out at the arena's pitch on `copy`
    const ThresholdPlan::Shape &sh = plan->shape(frame);
    const size_t eb = static_cast<size_t>(plan->elem_bytes());
    decoder.enqueue_raw(host, sh.height, static_cast<size_t>(sh.width) * eb,
                        plan->frame_origin(slot, frame), plan->pitch() * eb, copy);
    check(cudaEventRecord(uploaded[slot], copy), "cudaEventRecord");
  }

  void upload_device(int slot, int frame, const void *dev, size_t pitch) {
    check_slot(slot);
    check_frame(frame);
    check(cudaStreamWaitEvent(copy, consumed[slot], 0), "ordering after the last run");
    plan->upload_device(slot, frame, dev, pitch, copy);
    check(cudaEventRecord(uploaded[slot], copy), "cudaEventRecord");
  }

  // Frame `frame`'s pixel mask (height x width bytes, nonzero = masked), or
  // none with a null mask. Waits for the device; captured graphs are dropped
  // so the next runs stamp the new mask.
  void set_pixel_mask(int frame, const uint8_t *mask) {
    check_frame(frame);
    const ThresholdPlan::Shape &sh = plan->shape(frame);
    const uint64_t eb = static_cast<uint64_t>(plan->elem_bytes());
    const uint64_t at = (static_cast<uint64_t>(
                             static_cast<const char *>(plan->frame_origin(0, frame)) -
                             static_cast<const char *>(plan->frame_origin(0, 0)))) /
                        eb;
    if (mask_offsets.size() < static_cast<size_t>(plan->nframes()))
      mask_offsets.resize(plan->nframes());
    std::vector<uint64_t> &v = mask_offsets[frame];
    v.clear();
    if (mask)
      for (int64_t y = 0; y < sh.height; y++)
        for (int64_t x = 0; x < sh.width; x++)
          if (mask[y * sh.width + x])
            v.push_back(at + static_cast<uint64_t>(y) * plan->pitch() + x);
    std::vector<uint64_t> all;
    for (const auto &f : mask_offsets)
      all.insert(all.end(), f.begin(), f.end());
    check(cudaStreamSynchronize(copy), "cudaStreamSynchronize");
    check(cudaStreamSynchronize(compute), "cudaStreamSynchronize");
    check(cudaStreamSynchronize(group), "cudaStreamSynchronize");
    cudaFree(d_mask);
    d_mask = nullptr;
    mask_n = 0;
    if (!all.empty()) {
      check(cudaMalloc(&d_mask, all.size() * sizeof(uint64_t)), "cudaMalloc pixel mask");
      check(cudaMemcpy(d_mask, all.data(), all.size() * sizeof(uint64_t), cudaMemcpyHostToDevice),
            "copying the pixel mask");
      mask_n = all.size();
    }
    drop_graphs();
  }

  // Several chunks at once: their framing is walked on host threads in
  // parallel (each walk is a chain of dependent loads through its chunk),
  // all checked before anything is enqueued, then the copies and decodes go
  // in order as upload_chunk's would.
  void upload_chunks(int slot, size_t n, const int *frames, const void *const *chunks,
                     const size_t *nbytes, int algorithm) {
    check_slot(slot);
    for (size_t k = 0; k < n; k++)
      check_frame(frames ? frames[k] : static_cast<int>(k));
    const size_t eb = static_cast<size_t>(plan->elem_bytes());
    std::vector<ChunkLayout> layouts(n);
    auto frame_of = [&](size_t k) { return frames ? frames[k] : static_cast<int>(k); };
    auto parse = [&](size_t k) {
      const ThresholdPlan::Shape &sh = plan->shape(frame_of(k));
      layouts[k] = parse_chunk(algorithm, static_cast<const uint8_t *>(chunks[k]), nbytes[k],
                               static_cast<size_t>(sh.height) * sh.width, eb);
    };
    if (n > 1) {
      if (!pool) {
        const unsigned hw = std::thread::hardware_concurrency();
        pool = std::make_unique<HostPool>(static_cast<int>(std::min(7u, hw > 1 ? hw - 1 : 1u)));
      }
      pool->run(n, parse);
    } else if (n == 1) {
      parse(0);
    }
    check(cudaStreamWaitEvent(copy, consumed[slot], 0), "ordering after the last run");
    for (size_t k = 0; k < n; k++) {
      const ThresholdPlan::Shape &sh = plan->shape(frame_of(k));
      decoder.enqueue(static_cast<const uint8_t *>(chunks[k]), nbytes[k], layouts[k], sh.height,
                      sh.width, plan->frame_origin(slot, frame_of(k)), plan->pitch() * eb, copy);
    }
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
    check(cudaStreamSynchronize(group), "cudaStreamSynchronize");
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

std::unique_ptr<Engine> make_engine(int elem_bytes, const std::vector<ThresholdPlan::Shape> &shapes,
                                    const PlanTuning &tuning, int slots);

} // namespace sf
