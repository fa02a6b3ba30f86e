// C entry points over the reference's own CUDA backend (src/dext_cuda.cu,
// driven through its gpu::find, src/dext_gpu.hh:156-158), built for sm_100a
// from the reference tree. Used only by bench.py to time the reference's
// per-frame GPU form on the same box as the product, and by a GPU test that
// checks the comparison is like for like. Nothing in the product calls it.

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "dext_gpu.hh"
#include "signal_pixel.hh"

namespace {
thread_local std::string last_error;
thread_local std::vector<SignalPixel> signal;
} // namespace

extern "C" {

const char *refgpu_last_error() { return last_error.c_str(); }

int refgpu_available() { return gpu::available() ? 1 : 0; }

void refgpu_quiet() { gpu::report_windows(false); }

int refgpu_find_u16(const std::uint16_t *image, std::size_t height,
                    std::size_t width, SignalPixel *out, std::size_t capacity,
                    std::size_t *found) {
  try {
    const int status = gpu::find<std::uint16_t>(image, signal, height, width);
    *found = signal.size();
    if (status != 0)
      return status;
    if (signal.size() > capacity)
      return -2;
    if (!signal.empty())
      std::memcpy(out, signal.data(), signal.size() * sizeof(SignalPixel));
    return 0;
  } catch (const std::exception &error) {
    last_error = error.what();
    return -3;
  }
}

void *refgpu_host_alloc(std::size_t bytes) { return gpu::host_alloc(bytes); }
void refgpu_host_free(void *pointer) { gpu::host_free(pointer); }

} // extern "C"
