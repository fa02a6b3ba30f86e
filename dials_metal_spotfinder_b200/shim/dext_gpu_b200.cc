// gpu:: (the reference's src/dext_gpu.hh) on the B200 C ABI. Linked in place
// of the reference's src/dext_cuda.cu and src/dext_gpu.cc, it lets the
// reference's host code -- the NXmx reader, the -j worker pool, the labeller
// and the .refl writer in src/find_spots.cc -- run the B200 threshold without
// a changed line. Plain C++17; the only dependency is libspotfinder_b200.so.

#include "dext_gpu.hh"

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "spotfinder_b200.h"

static_assert(sizeof(SignalPixel) == sizeof(sf_signal_pixel), "SignalPixel layout");

namespace gpu {
namespace {

// CUDA's measured preferences in the reference (src/dext_gpu.cc:18-37):
// stage0 direct, stage2 tile. Kept as the defaults so that logs read the same.
std::atomic<Window> g_stage0{Window::Direct};
std::atomic<Window> g_stage2{Window::Tile};
std::once_flag g_env_once;
std::atomic<bool> g_report{true};
std::atomic<int> g_announced{-1};

void window_from_env(const char *variable, std::atomic<Window> &into) {
  const char *asked = std::getenv(variable);
  if (asked == nullptr)
    return;
  if (std::strcmp(asked, "tile") == 0)
    into.store(Window::Tile, std::memory_order_relaxed);
  else if (std::strcmp(asked, "direct") == 0)
    into.store(Window::Direct, std::memory_order_relaxed);
  else
    std::fprintf(stderr, "warning: %s=%s is not 'tile' or 'direct'; leaving it alone\n",
                 variable, asked);
}

void read_env() {
  window_from_env("SPOTFINDER_GPU_STAGE0", g_stage0);
  window_from_env("SPOTFINDER_GPU_STAGE2", g_stage2);
}

void announce() {
  if (!g_report.load(std::memory_order_relaxed))
    return;
  const Window s0 = stage0_window(), s2 = stage2_window();
  const int now = static_cast<int>(s0) * 2 + static_cast<int>(s2);
  if (g_announced.exchange(now, std::memory_order_relaxed) == now)
    return;
  std::fprintf(stderr, "%s: stage0 %s window, stage2 %s window\n", backend(), name(s0),
               name(s2));
}

// Per host thread: page-locked room for one frame's list, grown as needed,
// so the copy back runs at full speed and nothing is allocated per frame.
struct ListBuffer {
  sf_signal_pixel *data = nullptr;
  std::size_t capacity = 0;
  bool pinned = false;
  ~ListBuffer() { release(); }
  void release() {
    if (pinned)
      sf_host_free(data);
    else
      std::free(data);
    data = nullptr;
    capacity = 0;
  }
  sf_signal_pixel *reserve(std::size_t n) {
    if (n <= capacity)
      return data;
    release();
    const std::size_t bytes = n * sizeof(sf_signal_pixel);
    data = static_cast<sf_signal_pixel *>(sf_host_alloc(bytes));
    pinned = data != nullptr;
    if (!data)
      data = static_cast<sf_signal_pixel *>(std::malloc(bytes));
    if (!data)
      throw std::runtime_error("out of host memory for the signal list");
    capacity = n;
    return data;
  }
};

ListBuffer &list_buffer() {
  static thread_local ListBuffer buffer;
  return buffer;
}

} // namespace

const char *backend() { return sf_backend(); }

const char *name(Window window) { return window == Window::Tile ? "tile" : "direct"; }

Window stage0_window() {
  std::call_once(g_env_once, read_env);
  return g_stage0.load(std::memory_order_relaxed);
}
Window stage2_window() {
  std::call_once(g_env_once, read_env);
  return g_stage2.load(std::memory_order_relaxed);
}
void stage0_window(Window window) {
  std::call_once(g_env_once, read_env); // an explicit choice outlives the environment
  g_stage0.store(window, std::memory_order_relaxed);
}
void stage2_window(Window window) {
  std::call_once(g_env_once, read_env);
  g_stage2.store(window, std::memory_order_relaxed);
}

void profile_stages(bool on) { sf_profile_stages(on ? 1 : 0); }
bool profile_stages() { return sf_profile_stages_enabled() != 0; }

StageTimes last_stage_times() {
  double t[6];
  sf_last_stage_times(t);
  StageTimes s;
  s.upload = t[0];
  s.stage0 = t[1];
  s.stage1 = t[2];
  s.stage2 = t[3];
  s.copy = t[4];
  s.sort = t[5];
  return s;
}

void report_windows(bool on) { g_report.store(on, std::memory_order_relaxed); }

bool available() { return sf_available() != 0; }
std::size_t memory_free() { return sf_memory_free(); }
void *host_alloc(std::size_t bytes) { return sf_host_alloc(bytes); }
void host_free(void *pointer) { sf_host_free(pointer); }

template <typename T>
int find(const T *image_in, std::vector<SignalPixel> &signal_out, std::size_t height,
         std::size_t width) {
  static_assert(std::is_same<T, std::uint16_t>::value || std::is_same<T, std::uint32_t>::value,
                "16- and 32-bit pixels only");
  signal_out.clear();
  announce();
  if (image_in == nullptr || height == 0 || width == 0 || height > 0x7fffffffu / width)
    return -1;
  // the device list's capacity, as the reference sizes it
  const std::size_t capacity = height * width * sizeof(T) / 16;
  sf_signal_pixel *buffer = list_buffer().reserve(capacity > 0 ? capacity : 1);
  std::size_t found = 0;
  const int status =
      std::is_same<T, std::uint16_t>::value
          ? sf_find_u16(reinterpret_cast<const std::uint16_t *>(image_in), height, width,
                        buffer, capacity, &found)
          : sf_find_u32(reinterpret_cast<const std::uint32_t *>(image_in), height, width,
                        buffer, capacity, &found);
  if (status == -3)
    throw std::runtime_error(std::string("gpu::find: ") + sf_last_error());
  if (status != 0)
    return status;
  const SignalPixel *first = reinterpret_cast<const SignalPixel *>(buffer);
  signal_out.assign(first, first + found);
  return 0;
}

template int find<std::uint16_t>(const std::uint16_t *, std::vector<SignalPixel> &,
                                 std::size_t, std::size_t);
template int find<std::uint32_t>(const std::uint32_t *, std::vector<SignalPixel> &,
                                 std::size_t, std::size_t);

} // namespace gpu
