// The per-frame C entry points: device queries, pinned host memory and
// sf_find_u16 / sf_find_u32, the B200 replacement for the reference's
// gpu::find<T> (src/dext_cuda.cu:585-728).
//
// Per host thread: one stream, one ThresholdPlan for the last frame shape
// seen, a pinned word for the count and five events for stage profiling --
// created on first use and reused, so a steady stream of same-shaped frames
// allocates nothing after the first.

#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>

#include "../../include/spotfinder_b200.h"
#include "sf_capi.hh"
#include "sf_host.hh"

namespace sf {

thread_local std::string g_last_error;

void set_error(const char *what) { g_last_error = what ? what : ""; }

namespace {

std::atomic<bool> g_profile{false};
thread_local double g_times[6] = {0, 0, 0, 0, 0, 0};

// Blocks until the stream is idle however the scope is left, so no exit path
// returns with work in flight over buffers the next call will reuse.
class StreamIdle {
public:
  explicit StreamIdle(cudaStream_t s) : s_(s) {}
  ~StreamIdle() {
    if (s_)
      cudaStreamSynchronize(s_);
  }

private:
  cudaStream_t s_;
};

struct FindWorkspace {
  cudaStream_t stream = nullptr;
  cudaEvent_t marks[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  uint32_t *pinned = nullptr; // count, status
  std::unique_ptr<ThresholdPlan> plan;
  int eb = 0;
  size_t h = 0, w = 0;

  ~FindWorkspace() {
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
    for (cudaEvent_t &e : marks)
      if (e)
        cudaEventDestroy(e);
    if (pinned)
      cudaFreeHost(pinned);
    plan.reset();
  }

  void prepare(int elem_bytes, size_t height, size_t width) {
    if (!stream)
      check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (!pinned)
      check(cudaMallocHost(&pinned, 4 * sizeof(uint32_t)), "cudaMallocHost");
    if (plan && eb == elem_bytes && h == height && w == width)
      return;
    cudaStreamSynchronize(stream);
    plan.reset();
    std::vector<ThresholdPlan::Shape> shapes{
        {static_cast<int32_t>(height), static_cast<int32_t>(width)}};
    // One frame per launch: the plan picks segments short enough that a
    // single frame still spreads over every SM.
    plan = std::make_unique<ThresholdPlan>(elem_bytes, shapes, PlanTuning{}, 1);
    eb = elem_bytes;
    h = height;
    w = width;
  }

  cudaEvent_t *events() {
    if (!marks[0])
      for (cudaEvent_t &e : marks)
        check(cudaEventCreate(&e), "cudaEventCreate");
    return marks;
  }
};

FindWorkspace &workspace() {
  static thread_local FindWorkspace ws;
  return ws;
}

int find_impl(int elem_bytes, const void *image, size_t height, size_t width,
              SignalPixel *out, size_t capacity, size_t *found) {
  if (found)
    *found = 0;
  if (image == nullptr || height == 0 || width == 0 || found == nullptr)
    return -1;
  if (height > 0x7fffffffu / width)
    return -1;
  FindWorkspace &ws = workspace();
  ws.prepare(elem_bytes, height, width);
  ThresholdPlan &plan = *ws.plan;
  const cudaStream_t s = ws.stream;
  const StreamIdle idle(s);
  const bool timing = g_profile.load(std::memory_order_relaxed);
  cudaEvent_t *ev = timing ? ws.events() : nullptr;

  if (timing)
    check(cudaEventRecord(ev[0], s), "cudaEventRecord");
  plan.upload(0, 0, image, s);
  if (timing)
    check(cudaEventRecord(ev[1], s), "cudaEventRecord");
  plan.enqueue(0, s, timing ? ev[2] : nullptr);
  if (timing)
    check(cudaEventRecord(ev[3], s), "cudaEventRecord");
  // The count and the status word are adjacent: one copy.
  check(cudaMemcpyAsync(ws.pinned, plan.frame_count(0), 2 * sizeof(uint32_t),
                        cudaMemcpyDeviceToHost, s),
        "reading the signal count back");
  check(cudaStreamSynchronize(s), "cudaStreamSynchronize");

  const uint32_t count = ws.pinned[0];
  const int status = static_cast<int>(ws.pinned[1]);
  if (status == kStatusTmaTimeout)
    throw DeviceError("a TMA load did not complete in time");
  *found = count;
  if (timing) {
    float ms = 0;
    check(cudaEventElapsedTime(&ms, ev[0], ev[1]), "upload time");
    g_times[0] = ms;
    check(cudaEventElapsedTime(&ms, ev[1], ev[2]), "threshold time");
    g_times[1] = ms;
    g_times[2] = 0;
    check(cudaEventElapsedTime(&ms, ev[2], ev[3]), "placement time");
    g_times[3] = ms;
    g_times[4] = 0;
    g_times[5] = 0;
  }
  if (count > plan.capacity(0) || count > capacity)
    return -2;
  if (count == 0)
    return 0;
  const auto t0 = std::chrono::steady_clock::now();
  check(cudaMemcpyAsync(out, plan.out(0) + plan.out_base(0), count * sizeof(SignalPixel),
                        cudaMemcpyDeviceToHost, s),
        "copying the signal pixels back");
  check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  if (timing)
    g_times[4] =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
            .count();
  return 0;
}

} // namespace
} // namespace sf

using sf::guarded;

extern "C" {

const char *sf_backend(void) { return "CUDA sm_100a (B200-native)"; }

int sf_available(void) {
  int n = 0;
  return cudaGetDeviceCount(&n) == cudaSuccess && n > 0 ? 1 : 0;
}

size_t sf_memory_free(void) {
  size_t f = 0, t = 0;
  if (cudaMemGetInfo(&f, &t) != cudaSuccess)
    return 0;
  return f;
}

void *sf_host_alloc(size_t bytes) {
  void *p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess)
    return nullptr;
  return p;
}

void sf_host_free(void *pointer) {
  if (pointer)
    cudaFreeHost(pointer);
}

const char *sf_last_error(void) { return sf::g_last_error.c_str(); }

int sf_set_device(int device) {
  return guarded([&] {
    sf::check(cudaSetDevice(device), "cudaSetDevice");
    return 0;
  });
}

int sf_find_u16(const uint16_t *image, size_t height, size_t width, sf_signal_pixel *out,
                size_t capacity, size_t *found) {
  return guarded([&] {
    return sf::find_impl(2, image, height, width, reinterpret_cast<sf::SignalPixel *>(out),
                         capacity, found);
  });
}

int sf_find_u32(const uint32_t *image, size_t height, size_t width, sf_signal_pixel *out,
                size_t capacity, size_t *found) {
  return guarded([&] {
    return sf::find_impl(4, image, height, width, reinterpret_cast<sf::SignalPixel *>(out),
                         capacity, found);
  });
}

void sf_profile_stages(int on) { sf::g_profile.store(on != 0); }
int sf_profile_stages_enabled(void) { return sf::g_profile.load() ? 1 : 0; }
void sf_last_stage_times(double out6[6]) {
  for (int i = 0; i < 6; i++)
    out6[i] = sf::g_times[i];
}

} // extern "C"
