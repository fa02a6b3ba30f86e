// The serving loop: live series admitted by device-memory budget, each with
// its own engine (threshold + placement + grouping per frame, frames decoded
// from their chunks on the device), its own streams and its own worker
// thread, so the device work of concurrent series overlaps. Frames are
// admitted into the series' slots as they free up; the union-find frontier
// and the open components stay on the device between frames. The worker
// never waits for the device: each run ends with a kernel that writes its
// results (signal count, status, counts, the spots it finished and their
// pixels) into the slot's page-locked, device-mapped sink, and a host
// callback; a second thread per series collects the sinks in frame order
// and frees the slots, so the next frames upload and run meanwhile.
//
// Latencies are taken on the host's steady clock from the moment a frame is
// submitted: to its signal list being placed on the device (a host callback
// in the run's stream, after the placement: frame-to-mask), to its grouping
// being done, and, per spot, from the submission of the spot's last frame to
// the spot's row reaching the host (frame-to-finalised-spot).
//
// This replaces the reference's series queue and -j worker pool
// (src/series.hh:66-83, src/queue.hh, src/find_spots.cc:472-591), which
// decompress and threshold frames on host threads and group them on one.

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <iterator>
#include <mutex>
#include <thread>

#include "../../include/spotfinder_b200.h"
#include "sf_capi.hh"
#include "sf_engine.hh"

namespace sf {
namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct ServerSeries;

// What a run leaves for the host, in page-locked memory the device writes.
struct SinkHeader {
  uint32_t nsig;      // the frame's signal pixels
  int32_t status;     // 0, or what failed (kSink* bits)
  uint64_t nspots, npixels;
  uint64_t counts[6]; // running grouping counts
};
enum : int32_t { kSinkPlan = 1, kSinkDecode = 2, kSinkLabel = 4, kSinkOverflow = 8 };

struct SlotState {
  ServerSeries *series = nullptr;
  std::atomic<int64_t> t_mask{0}, t_done{0};
  SinkHeader *h_sink = nullptr; // host view
  SinkHeader *d_sink = nullptr; // the same memory, device view
};

void CUDART_CB mark_mask(void *arg) {
  static_cast<SlotState *>(arg)->t_mask.store(now_ns(), std::memory_order_release);
}
void CUDART_CB mark_done(void *arg);

// One run's results to its sink: the header from one thread, the spots and
// pixels by the grid, capped at the sink's capacity (kSinkOverflow beyond).
__global__ void sink_results(const LabelScalars *sc, const Spot *spots, const Pixel *pixels,
                             const uint32_t *frame_count, const int *plan_status,
                             const int *decode_err, SinkHeader *sink, uint64_t cap_spots,
                             uint64_t cap_pixels) {
  const uint64_t ns = sc->batch_spots, np = sc->batch_pixels;
  const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  if (tid == 0) {
    int32_t st = 0;
    if (*plan_status)
      st |= kSinkPlan;
    if (decode_err && *decode_err)
      st |= kSinkDecode;
    if (sc->status)
      st |= kSinkLabel;
    if (ns > cap_spots || np > cap_pixels)
      st |= kSinkOverflow;
    sink->nsig = frame_count[0];
    sink->status = st;
    sink->nspots = ns;
    sink->npixels = np;
    const uint64_t c[6] = {sc->signal_pixels, sc->groups, sc->too_small, sc->too_large,
                           sc->separated, sc->accepted};
    for (int i = 0; i < 6; i++)
      sink->counts[i] = c[i];
  }
  if (ns > cap_spots || np > cap_pixels)
    return;
  uint64_t *spot_words = reinterpret_cast<uint64_t *>(sink + 1);
  const uint64_t *src_spots = reinterpret_cast<const uint64_t *>(spots);
  for (uint64_t i = tid; i < ns * (sizeof(Spot) / 8); i += stride)
    spot_words[i] = src_spots[i];
  uint32_t *pixel_words = reinterpret_cast<uint32_t *>(spot_words + cap_spots * (sizeof(Spot) / 8));
  const uint32_t *src_pixels = reinterpret_cast<const uint32_t *>(pixels);
  for (uint64_t i = tid; i < np * (sizeof(Pixel) / 4); i += stride)
    pixel_words[i] = src_pixels[i];
}

struct Pending {
  int slot;
  size_t nbytes;
  int algorithm;
  int64_t frame; // series-relative frame number
  int64_t t_submit;
};

// Latency samples, appended in fixed blocks: an append never moves the
// samples already stored. (A vector that doubles copies all of them, and a
// series' spot samples reach tens of millions within a minute -- a copy of
// hundreds of megabytes made while the series' lock is held, which stalls
// every submission meanwhile.)
class Samples {
public:
  void push_back(double v) {
    if (n_ == blocks_.size() * kBlock)
      blocks_.emplace_back(new double[kBlock]);
    blocks_[n_ / kBlock][n_ % kBlock] = v;
    n_++;
  }
  size_t size() const { return n_; }
  void copy_to(double *out) const {
    for (size_t b = 0; b * kBlock < n_; b++)
      std::memcpy(out + b * kBlock, blocks_[b].get(),
                  std::min(kBlock, n_ - b * kBlock) * sizeof(double));
  }

private:
  static constexpr size_t kBlock = size_t(1) << 16;
  std::vector<std::unique_ptr<double[]>> blocks_;
  size_t n_ = 0;
};

struct ServerSeries {
  int id = 0;
  int device = 0;
  int64_t first_frame = 0;
  std::unique_ptr<Engine> eng;
  uint64_t device_bytes = 0;
  size_t chunk_cap = 0;
  uint64_t cap_spots = 0, cap_pixels = 0; // per sink
  std::vector<uint8_t *> staging;         // pinned, one chunk per slot
  std::vector<void *> sinks;              // page-locked, device-mapped, one per slot
  std::vector<std::unique_ptr<SlotState>> slot_state;

  std::mutex m;
  std::condition_variable cv;
  std::mutex done_m; // only for the runs' completion callbacks
  std::condition_variable done_cv;
  std::deque<int> free_slots;
  std::deque<Pending> queue;    // submitted, not yet uploaded
  std::deque<Pending> inflight; // uploaded and running, in frame order
  int64_t next_frame = 0;       // the next frame number a submission gets
  bool closing = false, worker_idle = false, done = false;
  std::thread worker, collector;

  // results, under m; spots and pixels in one block per run
  std::vector<std::vector<Spot>> spots;
  std::vector<std::vector<Pixel>> pixels;
  std::vector<uint32_t> signal_counts;
  std::vector<int64_t> t_submit; // per frame number
  int64_t t_close = 0;           // when the series was closed
  Samples lat_mask, lat_grouped, lat_spot;
  sf_counts counts{};
  uint64_t frames_done = 0, dropped = 0;
  std::string error;

  ~ServerSeries() {
    for (uint8_t *p : staging)
      if (p)
        cudaFreeHost(p);
    for (void *p : sinks)
      if (p)
        cudaFreeHost(p);
  }
};

void CUDART_CB mark_done(void *arg) {
  SlotState *st = static_cast<SlotState *>(arg);
  st->t_done.store(now_ns(), std::memory_order_release);
  std::lock_guard<std::mutex> g(st->series->done_m);
  st->series->done_cv.notify_all();
}

void post_run_sink(Engine &e, int slot, void *arg) {
  ServerSeries *se = static_cast<ServerSeries *>(arg);
  DeviceLabeller &lab = *e.series[0].lab;
  sink_results<<<64, 256, 0, e.group>>>(lab.scalars(), lab.batch_spots(), lab.batch_pixels(),
                                          e.plan->frame_count(slot), e.plan->status(slot),
                                          e.decoder.error_flag(),
                                          se->slot_state[slot]->d_sink, se->cap_spots,
                                          se->cap_pixels);
  check(cudaGetLastError(), "launching the result sink");
}

} // namespace

struct Server {
  uint64_t budget = 0, used = 0;
  int slots = 3;
  bool use_graph = true;
  std::mutex m;
  std::vector<std::unique_ptr<ServerSeries>> series;

  ~Server() {
    for (auto &se : series)
      if (se)
        stop(*se);
  }

  ServerSeries &at(int id) {
    std::lock_guard<std::mutex> g(m);
    if (id < 0 || id >= static_cast<int>(series.size()) || !series[id])
      throw std::out_of_range("no such series");
    return *series[id];
  }

  int open(size_t h, size_t w, int eb, const GroupOptions &opt, int64_t first_frame, int *out) {
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    size_t free0 = 0, total = 0;
    check(cudaMemGetInfo(&free0, &total), "cudaMemGetInfo");
    auto se = std::make_unique<ServerSeries>();
    se->device = dev;
    se->first_frame = first_frame;
    std::vector<ThresholdPlan::Shape> shapes{{static_cast<int32_t>(h), static_cast<int32_t>(w)}};
    se->eng = make_engine(eb, shapes, PlanTuning{}, slots);
    se->eng->enable_grouping(opt, first_frame, 0);
    // the decoder's staging sets, sized for the largest chunk of this shape
    // with 8 KB blocks, count toward the series' device bytes
    se->eng->decoder.reserve(sf_chunk_bound(h, w, eb), (h * w * eb + 8191) / 8192 + 1);
    size_t free1 = 0;
    check(cudaMemGetInfo(&free1, &total), "cudaMemGetInfo");
    se->device_bytes = free0 > free1 ? free0 - free1 : 0;
    {
      std::lock_guard<std::mutex> g(m);
      if (used + se->device_bytes > budget) {
        se->eng.reset();
        return -2;
      }
      used += se->device_bytes;
    }
    se->chunk_cap = sf_chunk_bound(h, w, eb);
    // A run's spots and pixels: up to four frames' list capacities of
    // pixels (a frame can close components that began frames earlier) and
    // 256 Ki spots; a run that finishes more reports an overflow.
    se->cap_pixels = std::max<uint64_t>(4 * (h * w * eb / 16), 1u << 16);
    se->cap_spots = 1u << 18;
    const size_t sink_bytes =
        sizeof(SinkHeader) + se->cap_spots * sizeof(Spot) + se->cap_pixels * sizeof(Pixel);
    se->staging.assign(slots, nullptr);
    se->sinks.assign(slots, nullptr);
    for (int s = 0; s < slots; s++) {
      check(cudaMallocHost(&se->staging[s], se->chunk_cap), "cudaMallocHost");
      check(cudaHostAlloc(&se->sinks[s], sink_bytes, cudaHostAllocMapped), "cudaHostAlloc sink");
      auto st = std::make_unique<SlotState>();
      st->series = se.get();
      st->h_sink = static_cast<SinkHeader *>(se->sinks[s]);
      void *dev = nullptr;
      check(cudaHostGetDevicePointer(&dev, se->sinks[s], 0), "cudaHostGetDevicePointer");
      st->d_sink = static_cast<SinkHeader *>(dev);
      se->eng->hook_args[s] = st.get();
      se->slot_state.push_back(std::move(st));
      se->free_slots.push_back(s);
    }
    se->eng->decoder.error_flag();
    se->eng->on_mask = mark_mask;
    se->eng->on_done = mark_done;
    se->eng->post_run = post_run_sink;
    se->eng->post_arg = se.get();
    se->eng->use_graph = use_graph;
    try {
      warm_up(*se);
    } catch (...) {
      std::lock_guard<std::mutex> g(m);
      used -= se->device_bytes; // the series is not opened
      throw;
    }
    ServerSeries *raw = se.get();
    {
      std::lock_guard<std::mutex> g(m);
      se->id = static_cast<int>(series.size());
      series.push_back(std::move(se));
    }
    raw->worker = std::thread([this, raw] { work(*raw); });
    raw->collector = std::thread([this, raw] { collect_loop(*raw); });
    *out = raw->id;
    return 0;
  }

  // Before a series takes frames: an empty frame, as a bitshuffle/LZ4
  // chunk, through every slot and both of each slot's grouping graphs, so
  // that the kernels are loaded and the graphs instantiated now and not
  // while a detector streams its first frames (without this, two series
  // opened together stalled for about half a second at their start and
  // dropped frames); the labeller then expects the series' first frame. An
  // empty frame has no signal pixels, so no count or result changes.
  void warm_up(ServerSeries &se) {
    Engine &e = *se.eng;
    const ThresholdPlan::Shape sh = e.plan->shape(0);
    const size_t n = static_cast<size_t>(sh.height) * sh.width;
    const size_t eb = static_cast<size_t>(e.plan->elem_bytes());
    std::vector<uint8_t> chunk;
    {
      std::vector<uint8_t> zeros(n * eb, 0);
      encode_chunk(SF_CHUNK_BSLZ4, zeros.data(), n, eb, chunk);
    }
    if (chunk.size() > se.chunk_cap)
      throw DeviceError("the empty frame's chunk exceeds the chunk bound");
    std::memcpy(se.staging[0], chunk.data(), chunk.size());
    const int slots = e.plan->nslots();
    for (int k = 0; k < 2 * slots; k++) { // slot k / 2, graph parity k % 2
      e.upload_chunk(k / 2, 0, se.staging[0], chunk.size(), SF_CHUNK_BSLZ4);
      e.run(k / 2);
    }
    e.synchronize();
    e.series[0].lab->set_next_frame(se.first_frame, e.group);
    e.synchronize();
  }

  int submit(int id, const void *chunk, size_t nbytes, int algorithm, int64_t timeout_us) {
    const int64_t t0 = now_ns();
    ServerSeries &se = at(id);
    if (nbytes > se.chunk_cap)
      throw std::invalid_argument("chunk larger than any encoding of the frame");
    std::unique_lock<std::mutex> lk(se.m);
    if (se.closing)
      throw std::invalid_argument("the series is closed");
    const bool ok = se.cv.wait_for(lk, std::chrono::microseconds(std::max<int64_t>(timeout_us, 0)),
                                   [&] { return !se.free_slots.empty() || !se.error.empty(); });
    if (!se.error.empty())
      throw DeviceError(se.error);
    const int64_t frame = se.next_frame++;
    se.t_submit.push_back(t0);
    if (se.signal_counts.size() < static_cast<size_t>(frame) + 1)
      se.signal_counts.resize(frame + 1, 0);
    if (!ok) {
      se.dropped++; // its count stays 0
      return -2;
    }
    const int slot = se.free_slots.front();
    se.free_slots.pop_front();
    lk.unlock();
    std::memcpy(se.staging[slot], chunk, nbytes);
    lk.lock();
    se.queue.push_back(Pending{slot, nbytes, algorithm, frame, t0});
    se.cv.notify_all();
    return 0;
  }

  // One series' frames, in order: decode on the device and run, without
  // waiting for the device; collect_loop takes the results.
  void work(ServerSeries &se) {
    cudaSetDevice(se.device);
    int64_t expected = 0; // the frame number the labeller expects next
    try {
      while (true) {
        Pending p;
        {
          std::unique_lock<std::mutex> lk(se.m);
          se.cv.wait(lk, [&] { return !se.queue.empty() || se.closing || !se.error.empty(); });
          if (!se.error.empty() || se.queue.empty())
            break;
          p = se.queue.front();
          se.queue.pop_front();
        }
        Engine &e = *se.eng;
        if (p.frame != expected) {
          // frames were dropped: the gap closes everything open, as a gap
          // in the numbering does for the reference's Labeller
          e.series[0].lab->set_next_frame(se.first_frame + p.frame, e.group);
          expected = p.frame;
        }
        SlotState &st = *se.slot_state[p.slot];
        st.t_mask.store(0);
        st.t_done.store(0);
        e.upload_chunk(p.slot, 0, se.staging[p.slot], p.nbytes, p.algorithm);
        {
          std::lock_guard<std::mutex> g(se.m);
          se.inflight.push_back(p);
          se.cv.notify_all(); // the collector waits for this
        }
        e.run(p.slot);
        expected++;
      }
    } catch (const std::exception &ex) {
      std::lock_guard<std::mutex> g(se.m);
      se.error = ex.what();
    }
    std::unique_lock<std::mutex> lk(se.m);
    se.worker_idle = true;
    se.cv.notify_all();
    se.cv.wait(lk, [&] { return se.inflight.empty(); });
    lk.unlock();
    try {
      if (se.error.empty()) {
        Engine &e = *se.eng;
        // finish() closes what is open; its spots are read back directly
        for (Engine::Series &s : e.series)
          s.lab->enqueue(0, e.plan->out(0), s.d_offs, e.plan->frame_count(0), s.d_map,
                         s.d_caps, true, e.group);
        e.parity ^= 1;
        e.synchronize();
        collect_direct(se);
      }
    } catch (const std::exception &ex) {
      std::lock_guard<std::mutex> g(se.m);
      se.error = ex.what();
    }
    lk.lock();
    se.done = true;
    se.cv.notify_all();
  }

  // The runs' sinks, in frame order, as their host callbacks mark them. The
  // sink of an in-flight slot is not reused until the slot is freed, so it
  // is read without holding the series' lock.
  void collect_loop(ServerSeries &se) {
    while (true) {
      Pending p;
      {
        std::unique_lock<std::mutex> lk(se.m);
        se.cv.wait(lk, [&] { return !se.inflight.empty() || se.worker_idle; });
        if (se.inflight.empty())
          break;
        p = se.inflight.front();
      }
      SlotState &st = *se.slot_state[p.slot];
      {
        std::unique_lock<std::mutex> dk(se.done_m);
        se.done_cv.wait(dk, [&] { return st.t_done.load(std::memory_order_acquire) != 0; });
      }
      const SinkHeader h = *st.h_sink;
      std::vector<Spot> sp;
      std::vector<Pixel> px;
      std::vector<double> lat;
      if (!h.status) {
        const Spot *hs = reinterpret_cast<const Spot *>(st.h_sink + 1);
        const Pixel *hp = reinterpret_cast<const Pixel *>(hs + se.cap_spots);
        sp.assign(hs, hs + h.nspots);
        px.assign(hp, hp + h.npixels);
      }
      const int64_t t = now_ns();
      std::lock_guard<std::mutex> g(se.m);
      if (h.status && se.error.empty())
        se.error = h.status & kSinkOverflow
                       ? "frame " + std::to_string(p.frame) + " finished " +
                             std::to_string(h.nspots) + " spots with " +
                             std::to_string(h.npixels) + " pixels, more than its sink holds (" +
                             std::to_string(se.cap_spots) + ", " + std::to_string(se.cap_pixels) +
                             ")"
                   : h.status & kSinkDecode ? "an uploaded chunk held a malformed LZ4 block"
                   : h.status & kSinkLabel  ? "grouping capacity exceeded"
                                            : "a threshold wait gave up";
      if (!h.status) {
        for (const Spot &s : sp) {
          const int64_t last = static_cast<int64_t>(s.bbox[5]) - 1 - se.first_frame;
          if (last >= 0 && last < static_cast<int64_t>(se.t_submit.size()))
            se.lat_spot.push_back(1e-3 * static_cast<double>(t - se.t_submit[last]));
        }
        std::memcpy(&se.counts, h.counts, sizeof(se.counts));
        if (!sp.empty())
          se.spots.push_back(std::move(sp));
        if (!px.empty())
          se.pixels.push_back(std::move(px));
      }
      const int64_t tm = st.t_mask.load(std::memory_order_acquire);
      const int64_t td = st.t_done.load(std::memory_order_acquire);
      se.lat_mask.push_back(1e-3 * static_cast<double>((tm ? tm : td) - p.t_submit));
      se.lat_grouped.push_back(1e-3 * static_cast<double>(td - p.t_submit));
      se.signal_counts[p.frame] = h.nsig;
      se.frames_done++;
      se.inflight.pop_front();
      se.free_slots.push_back(p.slot);
      se.cv.notify_all();
    }
  }

  // The spots the last enqueued work finished, read from the device.
  void collect_direct(ServerSeries &se) {
    Engine &e = *se.eng;
    const LabelScalars &sc = e.group_state(0);
    const uint64_t ns = sc.batch_spots, np = sc.batch_pixels;
    sf_counts c{sc.signal_pixels, sc.groups, sc.too_small, sc.too_large, sc.separated,
                sc.accepted};
    std::vector<Spot> sp(ns);
    std::vector<Pixel> px(np);
    if (ns)
      check(cudaMemcpy(sp.data(), e.series[0].lab->batch_spots(), ns * sizeof(Spot),
                       cudaMemcpyDeviceToHost),
            "reading spots");
    if (np)
      check(cudaMemcpy(px.data(), e.series[0].lab->batch_pixels(), np * sizeof(Pixel),
                       cudaMemcpyDeviceToHost),
            "reading spot pixels");
    const int64_t t = now_ns();
    std::lock_guard<std::mutex> g(se.m);
    se.counts = c;
    // these spots were still open when the series was closed: closing is
    // what finishes them, so their latency counts from the close (or from
    // their last frame's submit, were that later)
    for (const Spot &s : sp) {
      const int64_t last = static_cast<int64_t>(s.bbox[5]) - 1 - se.first_frame;
      if (last >= 0 && last < static_cast<int64_t>(se.t_submit.size()))
        se.lat_spot.push_back(
            1e-3 * static_cast<double>(t - std::max(se.t_close, se.t_submit[last])));
    }
    if (!sp.empty())
      se.spots.push_back(std::move(sp));
    if (!px.empty())
      se.pixels.push_back(std::move(px));
  }

  void stop(ServerSeries &se) {
    {
      std::lock_guard<std::mutex> g(se.m);
      if (!se.closing)
        se.t_close = now_ns();
      se.closing = true;
      se.cv.notify_all();
    }
    if (se.worker.joinable())
      se.worker.join();
    if (se.collector.joinable())
      se.collector.join();
  }

  void close(int id) {
    ServerSeries &se = at(id);
    stop(se);
    {
      std::lock_guard<std::mutex> g(m);
      if (se.eng) {
        se.eng.reset(); // the device memory goes back to the budget
        used -= std::min(used, se.device_bytes);
      }
    }
    std::lock_guard<std::mutex> g(se.m);
    if (!se.error.empty())
      throw DeviceError(se.error);
  }
};

} // namespace sf

using sf::guarded;
using sf::Server;
using sf::ServerSeries;

namespace {

int copy_out(const sf::Samples &v, double *out, size_t capacity, size_t *n) {
  *n = v.size();
  if (v.size() > capacity)
    return -2;
  v.copy_to(out);
  return 0;
}

template <typename T>
int copy_out(const std::vector<T> &v, T *out, size_t capacity, size_t *n) {
  *n = v.size();
  if (v.size() > capacity)
    return -2;
  if (!v.empty())
    std::memcpy(out, v.data(), v.size() * sizeof(T));
  return 0;
}

template <typename T>
int copy_blocks(const std::vector<std::vector<T>> &blocks, T *out, size_t capacity, size_t *n) {
  size_t total = 0;
  for (const auto &b : blocks)
    total += b.size();
  *n = total;
  if (total > capacity)
    return -2;
  for (const auto &b : blocks) {
    std::memcpy(out, b.data(), b.size() * sizeof(T));
    out += b.size();
  }
  return 0;
}

} // namespace

extern "C" {

int sf_server_create(const sf_server_config *config, sf_server **out) {
  return guarded([&] {
    if (!out)
      return -1;
    auto s = std::make_unique<Server>();
    size_t free = 0, total = 0;
    sf::check(cudaMemGetInfo(&free, &total), "cudaMemGetInfo");
    const uint64_t reserve = 2ull << 30;
    s->budget = free > reserve ? free - reserve : 0;
    if (config) {
      if (config->hbm_budget)
        s->budget = std::min<uint64_t>(config->hbm_budget, s->budget);
      if (config->slots > 0)
        s->slots = config->slots;
      s->use_graph = config->use_graph != 0;
    }
    *out = reinterpret_cast<sf_server *>(s.release());
    return 0;
  });
}

void sf_server_destroy(sf_server *server) { delete reinterpret_cast<Server *>(server); }

int sf_server_open(sf_server *server, size_t height, size_t width, int elem_bytes,
                   const sf_group_options *options, int64_t first_frame, int *series) {
  return guarded([&] {
    if (!server || !series || height == 0 || width == 0 || (elem_bytes != 2 && elem_bytes != 4))
      return -1;
    sf::GroupOptions opt;
    if (options) {
      opt.min_spot_size = options->min_spot_size;
      opt.max_spot_size = options->max_spot_size;
      opt.max_separation = options->max_separation;
      opt.two_d = options->two_d != 0;
    }
    return reinterpret_cast<Server *>(server)->open(height, width, elem_bytes, opt, first_frame,
                                                    series);
  });
}

int sf_server_set_pixel_mask(sf_server *server, int series, const uint8_t *mask) {
  return guarded([&] {
    if (!server)
      return -1;
    ServerSeries &se = reinterpret_cast<Server *>(server)->at(series);
    std::lock_guard<std::mutex> g(se.m);
    if (se.frames_done || !se.queue.empty() || !se.inflight.empty() || !se.eng)
      throw std::invalid_argument("set a series' pixel mask before its first frame");
    se.eng->set_pixel_mask(0, mask);
    // a new mask drops the series' graphs: warm them again before frames come
    reinterpret_cast<Server *>(server)->warm_up(se);
    return 0;
  });
}

int sf_server_submit(sf_server *server, int series, const void *chunk, size_t nbytes,
                     int algorithm, int64_t timeout_us) {
  return guarded([&] {
    if (!server || !chunk)
      return -1;
    return reinterpret_cast<Server *>(server)->submit(series, chunk, nbytes, algorithm,
                                                      timeout_us);
  });
}

int sf_server_close(sf_server *server, int series) {
  return guarded([&] {
    if (!server)
      return -1;
    reinterpret_cast<Server *>(server)->close(series);
    return 0;
  });
}

int sf_server_stats(sf_server *server, int series, sf_counts *counts, uint64_t out4[4]) {
  return guarded([&] {
    if (!server)
      return -1;
    ServerSeries &se = reinterpret_cast<Server *>(server)->at(series);
    std::lock_guard<std::mutex> g(se.m);
    if (counts)
      *counts = se.counts;
    if (out4) {
      out4[0] = se.frames_done;
      out4[1] = se.dropped;
      out4[2] = se.device_bytes;
      out4[3] = se.done ? 1 : 0;
    }
    return 0;
  });
}

int sf_server_spots(sf_server *server, int series, sf_spot *out, size_t capacity, size_t *n) {
  return guarded([&] {
    if (!server || !n)
      return -1;
    ServerSeries &se = reinterpret_cast<Server *>(server)->at(series);
    std::lock_guard<std::mutex> g(se.m);
    return copy_blocks(se.spots, reinterpret_cast<sf::Spot *>(out), capacity, n);
  });
}

int sf_server_pixels(sf_server *server, int series, sf_pixel *out, size_t capacity, size_t *n) {
  return guarded([&] {
    if (!server || !n)
      return -1;
    ServerSeries &se = reinterpret_cast<Server *>(server)->at(series);
    std::lock_guard<std::mutex> g(se.m);
    return copy_blocks(se.pixels, reinterpret_cast<sf::Pixel *>(out), capacity, n);
  });
}

int sf_server_take(sf_server *server, int series, sf_spot *spots, size_t spot_capacity,
                   size_t *nspots, sf_pixel *pixels, size_t pixel_capacity, size_t *npixels) {
  return guarded([&] {
    if (!server || !nspots || !npixels)
      return -1;
    ServerSeries &se = reinterpret_cast<Server *>(server)->at(series);
    // a run's spot block and pixel block are pushed together (a spot has
    // pixels), so the blocks pair up; take whole runs while both fit. The
    // blocks are moved out under the series' lock and copied after it, so
    // the series' submits and collector do not wait on the copy.
    std::vector<std::vector<sf::Spot>> sp;
    std::vector<std::vector<sf::Pixel>> px;
    bool none_fit = false;
    {
      std::lock_guard<std::mutex> g(se.m);
      size_t ns = 0, np = 0, k = 0;
      while (k < se.spots.size() && k < se.pixels.size() &&
             ns + se.spots[k].size() <= spot_capacity &&
             np + se.pixels[k].size() <= pixel_capacity) {
        ns += se.spots[k].size();
        np += se.pixels[k].size();
        k++;
      }
      none_fit = k == 0 && !se.spots.empty();
      sp.assign(std::make_move_iterator(se.spots.begin()),
                std::make_move_iterator(se.spots.begin() + k));
      px.assign(std::make_move_iterator(se.pixels.begin()),
                std::make_move_iterator(se.pixels.begin() + k));
      se.spots.erase(se.spots.begin(), se.spots.begin() + k);
      se.pixels.erase(se.pixels.begin(), se.pixels.begin() + k);
    }
    size_t ns = 0, np = 0;
    for (size_t k = 0; k < sp.size(); k++) {
      if (!sp[k].empty())
        std::memcpy(spots + ns, sp[k].data(), sp[k].size() * sizeof(sf::Spot));
      if (!px[k].empty())
        std::memcpy(pixels + np, px[k].data(), px[k].size() * sizeof(sf::Pixel));
      ns += sp[k].size();
      np += px[k].size();
    }
    *nspots = ns;
    *npixels = np;
    return none_fit ? -2 : 0;
  });
}

int sf_server_signal_counts(sf_server *server, int series, uint32_t *out, size_t capacity,
                            size_t *n) {
  return guarded([&] {
    if (!server || !n)
      return -1;
    ServerSeries &se = reinterpret_cast<Server *>(server)->at(series);
    std::lock_guard<std::mutex> g(se.m);
    return copy_out(se.signal_counts, out, capacity, n);
  });
}

int sf_server_latencies(sf_server *server, int series, int kind, double *out, size_t capacity,
                        size_t *n) {
  return guarded([&] {
    if (!server || !n || kind < 0 || kind > 2)
      return -1;
    ServerSeries &se = reinterpret_cast<Server *>(server)->at(series);
    std::lock_guard<std::mutex> g(se.m);
    const sf::Samples &v = kind == 0 ? se.lat_mask : kind == 1 ? se.lat_grouped : se.lat_spot;
    return copy_out(v, out, capacity, n);
  });
}

} // extern "C"
