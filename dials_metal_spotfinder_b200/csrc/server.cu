// The serving loop: live series admitted by device-memory budget, each with
// its own engine (threshold + placement + grouping per frame, frames decoded
// from their chunks on the device), its own streams and its own worker
// thread, so the device work of concurrent series overlaps. Frames are
// admitted into the series' slots as they free up; the union-find frontier
// and the open components stay on the device between frames, and each
// frame's finished spots are copied out as soon as its run completes.
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

struct SlotState {
  std::atomic<int64_t> t_mask{0}, t_done{0};
};

void CUDART_CB mark_mask(void *arg) {
  static_cast<SlotState *>(arg)->t_mask.store(now_ns(), std::memory_order_release);
}
void CUDART_CB mark_done(void *arg) {
  static_cast<SlotState *>(arg)->t_done.store(now_ns(), std::memory_order_release);
}

struct Pending {
  int slot;
  size_t nbytes;
  int algorithm;
  int64_t frame; // series-relative frame number
  int64_t t_submit;
};

struct ServerSeries {
  int id = 0;
  int device = 0;
  int64_t first_frame = 0;
  std::unique_ptr<Engine> eng;
  uint64_t device_bytes = 0;
  size_t chunk_cap = 0;
  std::vector<uint8_t *> staging; // pinned, one chunk per slot
  std::vector<std::unique_ptr<SlotState>> slot_state;

  std::mutex m;
  std::condition_variable cv;
  std::deque<int> free_slots;
  std::deque<Pending> queue;
  int64_t next_frame = 0; // the next frame number a submission gets
  bool closing = false, done = false;
  std::thread worker;

  // results, under m
  std::vector<Spot> spots;
  std::vector<Pixel> pixels;
  std::vector<uint32_t> signal_counts;
  std::vector<int64_t> t_submit; // per frame number
  std::vector<double> lat_mask, lat_grouped, lat_spot;
  sf_counts counts{};
  uint64_t frames_done = 0, dropped = 0;
  std::string error;

  ~ServerSeries() {
    for (uint8_t *p : staging)
      if (p)
        cudaFreeHost(p);
  }
};

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
    se->staging.assign(slots, nullptr);
    for (int s = 0; s < slots; s++) {
      check(cudaMallocHost(&se->staging[s], se->chunk_cap), "cudaMallocHost");
      se->slot_state.push_back(std::make_unique<SlotState>());
      se->eng->hook_args[s] = se->slot_state[s].get();
      se->free_slots.push_back(s);
    }
    se->eng->on_mask = mark_mask;
    se->eng->on_done = mark_done;
    se->eng->use_graph = use_graph;
    ServerSeries *raw = se.get();
    {
      std::lock_guard<std::mutex> g(m);
      se->id = static_cast<int>(series.size());
      series.push_back(std::move(se));
    }
    raw->worker = std::thread([this, raw] { work(*raw); });
    *out = raw->id;
    return 0;
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

  // One series' frames, in order: decode on the device, run, read back.
  void work(ServerSeries &se) {
    cudaSetDevice(se.device);
    int64_t expected = 0; // the frame number the labeller expects next
    try {
      while (true) {
        Pending p;
        {
          std::unique_lock<std::mutex> lk(se.m);
          se.cv.wait(lk, [&] { return !se.queue.empty() || se.closing; });
          if (se.queue.empty())
            break;
          p = se.queue.front();
          se.queue.pop_front();
        }
        Engine &e = *se.eng;
        if (p.frame != expected) {
          // frames were dropped: the gap closes everything open, as a gap
          // in the numbering does for the reference's Labeller
          e.series[0].lab->set_next_frame(se.first_frame + p.frame, e.compute);
          expected = p.frame;
        }
        SlotState &st = *se.slot_state[p.slot];
        st.t_mask.store(0);
        st.t_done.store(0);
        e.upload_chunk(p.slot, 0, se.staging[p.slot], p.nbytes, p.algorithm);
        e.run(p.slot);
        e.synchronize();
        expected++;
        uint32_t nsig = 0;
        check(cudaMemcpy(&nsig, e.plan->frame_count(p.slot), sizeof(uint32_t),
                         cudaMemcpyDeviceToHost),
              "reading a signal count");
        collect(se);
        const int64_t t_host = now_ns();
        std::lock_guard<std::mutex> g(se.m);
        const int64_t tm = st.t_mask.load(std::memory_order_acquire);
        const int64_t td = st.t_done.load(std::memory_order_acquire);
        se.lat_mask.push_back(1e-3 * static_cast<double>((tm ? tm : t_host) - p.t_submit));
        se.lat_grouped.push_back(1e-3 * static_cast<double>((td ? td : t_host) - p.t_submit));
        se.signal_counts[p.frame] = nsig;
        se.frames_done++;
        se.free_slots.push_back(p.slot);
        se.cv.notify_all();
      }
      Engine &e = *se.eng;
      // finish() closes what is open; its spots are the last run's
      for (Engine::Series &s : e.series)
        s.lab->enqueue(0, e.plan->out(0), s.d_offs, e.plan->frame_count(0), s.d_map, s.d_caps,
                       true, e.compute);
      e.parity ^= 1;
      e.synchronize();
      collect(se);
    } catch (const std::exception &ex) {
      std::lock_guard<std::mutex> g(se.m);
      se.error = ex.what();
      se.cv.notify_all();
    }
    std::lock_guard<std::mutex> g(se.m);
    se.done = true;
    se.cv.notify_all();
  }

  // The spots the last run finished, appended with their latencies.
  void collect(ServerSeries &se) {
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
    for (const Spot &s : sp) {
      const int64_t last = static_cast<int64_t>(s.bbox[5]) - 1 - se.first_frame;
      if (last >= 0 && last < static_cast<int64_t>(se.t_submit.size()))
        se.lat_spot.push_back(1e-3 * static_cast<double>(t - se.t_submit[last]));
    }
    se.spots.insert(se.spots.end(), sp.begin(), sp.end());
    se.pixels.insert(se.pixels.end(), px.begin(), px.end());
  }

  void stop(ServerSeries &se) {
    {
      std::lock_guard<std::mutex> g(se.m);
      se.closing = true;
      se.cv.notify_all();
    }
    if (se.worker.joinable())
      se.worker.join();
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

template <typename T>
int copy_out(const std::vector<T> &v, T *out, size_t capacity, size_t *n) {
  *n = v.size();
  if (v.size() > capacity)
    return -2;
  if (!v.empty())
    std::memcpy(out, v.data(), v.size() * sizeof(T));
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
    return copy_out(se.spots, reinterpret_cast<sf::Spot *>(out), capacity, n);
  });
}

int sf_server_pixels(sf_server *server, int series, sf_pixel *out, size_t capacity, size_t *n) {
  return guarded([&] {
    if (!server || !n)
      return -1;
    ServerSeries &se = reinterpret_cast<Server *>(server)->at(series);
    std::lock_guard<std::mutex> g(se.m);
    return copy_out(se.pixels, reinterpret_cast<sf::Pixel *>(out), capacity, n);
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
    const std::vector<double> &v =
        kind == 0 ? se.lat_mask : kind == 1 ? se.lat_grouped : se.lat_spot;
    return copy_out(v, out, capacity, n);
  });
}

} // extern "C"
