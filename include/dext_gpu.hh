// The gpu:: interface the reference's host code calls (src/dext_gpu.hh,
// compiled into src/find_spots.cc under SPOTFINDER_GPU), declared here with
// the same names and signatures so that the B200 build drops in under it:
// dials_metal_spotfinder_b200/shim/dext_gpu_b200.cc implements every
// function below on top of the C ABI in spotfinder_b200.h, in place of the
// reference's src/dext_cuda.cu + src/dext_gpu.cc. In the reference's tree its
// own header may stay on the include path; the two declare the same functions.
//
// Semantics kept from the reference:
//   * find<T> returns 0, -1 (null image, zero dimension, height * width beyond
//     INT32_MAX) or -2 (more signal pixels than height * width * sizeof(T) / 16),
//     clears and refills `signal_out` ascending by index, and throws
//     std::runtime_error on a device failure; it may be called from many host
//     threads at once (each gets its own stream and buffers);
//   * the window choice is read from SPOTFINDER_GPU_STAGE0 / _STAGE2 ("tile" or
//     "direct"; anything else warns on stderr and is ignored) and reported on
//     stderr when it changes, unless report_windows(false);
//   * host_alloc returns page-locked memory or nullptr, never throws.
// What differs: the B200 threshold is one fused kernel whose window sums are
// running sums along the strip, so neither window setting changes how it runs
// or what it returns; they are accepted, stored and reported so that callers
// and their logs stay as they are. StageTimes::stage0 is the whole fused
// threshold (dispersion test, erode and Poisson test), stage1 is 0 and stage2
// is the ordered compaction that replaces the host sort (sort is 0).
#ifndef SPOTFINDER_DEXT_GPU_HH
#define SPOTFINDER_DEXT_GPU_HH

#include <cstddef>
#include <cstdint>
#include <vector>

#include "signal_pixel.hh"

namespace gpu {

const char *backend();

enum class Window { Direct, Tile };

const char *name(Window window);

Window stage0_window();
void stage0_window(Window window);
Window stage2_window();
void stage2_window(Window window);

struct StageTimes {
  double upload = 0.0; // host-to-device copy of the frame
  double stage0 = 0.0; // device: the fused threshold kernel
  double stage1 = 0.0; // device: 0 (the erode is fused into stage0)
  double stage2 = 0.0; // device: ordered compaction of the signal list
  double copy = 0.0;   // host wall clock: reading the list back
  double sort = 0.0;   // host wall clock: 0 (the list arrives in order)
};

void profile_stages(bool on);
bool profile_stages();
StageTimes last_stage_times();
void report_windows(bool on);

bool available();
std::size_t memory_free();

void *host_alloc(std::size_t bytes);
void host_free(void *pointer);

template <typename T>
int find(const T *image_in, std::vector<SignalPixel> &signal_out, std::size_t height,
         std::size_t width);

extern template int find<std::uint16_t>(const std::uint16_t *, std::vector<SignalPixel> &,
                                        std::size_t, std::size_t);
extern template int find<std::uint32_t>(const std::uint32_t *, std::vector<SignalPixel> &,
                                        std::size_t, std::size_t);

} // namespace gpu

#endif // SPOTFINDER_DEXT_GPU_HH
