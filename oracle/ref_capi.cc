// C entry points over the reference spot finder's own CPU code, compiled from
// the reference sources where they lie (see oracle/Makefile). Test
// infrastructure only: the parity tests, the golden-fixture script and the
// CPU-baseline leg of bench.py load this library as the checker. Nothing in
// the product links or calls it.
//
// Wrapped, unchanged:
//   dext<T>                      src/dext.cc:9-225
//   dials_spots::Labeller        src/dials_spots.cc:36-360
//   refl::write                  src/refl.cc:223-351
//   synthetic::make_frame        tests/synthetic_frame.hh:93-157
//
// Every function returns 0 on success and a negative code on failure; a C++
// exception is caught here and its message kept for ref_last_error().

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "dext.hh"
#include "dials_spots.hh"
#include "refl.hh"
#include "signal_pixel.hh"
#include "synthetic_frame.hh"

namespace {

thread_local std::string last_error;

template <typename T>
int run_dext(const T *image, std::size_t height, std::size_t width,
             SignalPixel *out, std::size_t capacity, std::size_t *found) {
  static thread_local dext_scratch<T> scratch;
  static thread_local std::vector<SignalPixel> signal;
  const int status = dext<T>(image, signal, height, width, scratch);
  *found = signal.size();
  if (status != 0)
    return status;
  if (signal.size() > capacity)
    return -2;
  if (!signal.empty())
    std::memcpy(out, signal.data(), signal.size() * sizeof(SignalPixel));
  return 0;
}

} // namespace

extern "C" {

const char *ref_last_error() { return last_error.c_str(); }

int ref_dext_u16(const std::uint16_t *image, std::size_t height,
                 std::size_t width, SignalPixel *out, std::size_t capacity,
                 std::size_t *found) {
  return run_dext<std::uint16_t>(image, height, width, out, capacity, found);
}

int ref_dext_u32(const std::uint32_t *image, std::size_t height,
                 std::size_t width, SignalPixel *out, std::size_t capacity,
                 std::size_t *found) {
  return run_dext<std::uint32_t>(image, height, width, out, capacity, found);
}

// The reference's device-test frame generator, for golden fixtures.
int ref_make_frame(std::size_t height, std::size_t width, std::uint64_t seed,
                   double background, int with_mask, std::uint16_t *out) {
  const synthetic::Frame frame = synthetic::make_frame(
      "fixture", height, width, seed, background, with_mask != 0);
  std::memcpy(out, frame.pixels.data(), height * width * sizeof(std::uint16_t));
  return 0;
}

void *ref_labeller_new(std::size_t height, std::size_t width,
                       std::size_t min_spot_size, std::size_t max_spot_size,
                       double max_separation, int two_d) {
  try {
    dials_spots::Options options;
    options.min_spot_size = min_spot_size;
    options.max_spot_size = max_spot_size;
    options.max_separation = max_separation;
    options.two_d = two_d != 0;
    return new dials_spots::Labeller(height, width, options);
  } catch (const std::exception &error) {
    last_error = error.what();
    return nullptr;
  }
}

void ref_labeller_free(void *handle) {
  delete static_cast<dials_spots::Labeller *>(handle);
}

int ref_labeller_add(void *handle, std::int64_t frame, const SignalPixel *pixels,
                     std::size_t n) {
  try {
    std::vector<SignalPixel> signal(pixels, pixels + n);
    static_cast<dials_spots::Labeller *>(handle)->add(frame, signal);
    return 0;
  } catch (const std::exception &error) {
    last_error = error.what();
    return -1;
  }
}

int ref_labeller_finish(void *handle) {
  try {
    static_cast<dials_spots::Labeller *>(handle)->finish();
    return 0;
  } catch (const std::exception &error) {
    last_error = error.what();
    return -1;
  }
}

std::size_t ref_labeller_nspots(void *handle) {
  return static_cast<dials_spots::Labeller *>(handle)->spots().size();
}

std::size_t ref_labeller_npixels(void *handle) {
  return static_cast<dials_spots::Labeller *>(handle)->pixels().size();
}

std::size_t ref_labeller_live(void *handle) {
  return static_cast<dials_spots::Labeller *>(handle)->live();
}

// Spot rows are copied as the reference lays them out (dials_spots.hh:57-79).
int ref_labeller_spots(void *handle, void *out, std::size_t capacity) {
  const auto &spots = static_cast<dials_spots::Labeller *>(handle)->spots();
  if (spots.size() > capacity)
    return -2;
  if (!spots.empty())
    std::memcpy(out, spots.data(), spots.size() * sizeof(dials_spots::Spot));
  return 0;
}

int ref_labeller_pixels(void *handle, void *out, std::size_t capacity) {
  const auto &pixels = static_cast<dials_spots::Labeller *>(handle)->pixels();
  if (pixels.size() > capacity)
    return -2;
  if (!pixels.empty())
    std::memcpy(out, pixels.data(), pixels.size() * sizeof(dials_spots::Pixel));
  return 0;
}

// signal_pixels, groups, too_small, too_large, separated, accepted.
void ref_labeller_counts(void *handle, std::uint64_t *out) {
  const dials_spots::Counts &c =
      static_cast<dials_spots::Labeller *>(handle)->counts();
  out[0] = c.signal_pixels;
  out[1] = c.groups;
  out[2] = c.too_small;
  out[3] = c.too_large;
  out[4] = c.separated;
  out[5] = c.accepted;
}

std::size_t ref_spot_size() { return sizeof(dials_spots::Spot); }

int ref_refl_write(const char *path, void *handle, std::size_t width,
                   const char *identifier, int shoeboxes, int id) {
  try {
    const auto *labeller = static_cast<dials_spots::Labeller *>(handle);
    refl::Options options;
    options.identifier = identifier == nullptr ? "" : identifier;
    options.shoeboxes = shoeboxes != 0;
    options.id = id;
    refl::write(path, labeller->spots(), labeller->pixels(), width, options);
    return 0;
  } catch (const std::exception &error) {
    last_error = error.what();
    return -1;
  }
}

} // extern "C"
