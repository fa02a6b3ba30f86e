// Drives the C++ drop-in (gpu:: from dext_gpu.hh and the templated Labeller
// facade) the way the reference's host code does, for tests/test_shim*.py.
// Frames and results pass through raw little-endian files.
//
//   shim_check info
//       available=<0|1> backend=<...> stage0=<window> stage2=<window>
//   shim_check find16|find32 H W image.raw out.raw
//       out.raw: int32 status, uint64 count, count x 16-byte SignalPixel
//   shim_check series16 NF H W Z0 TWO_D frames.raw spots.raw pixels.raw counts.raw [out.refl]
//       gpu::find<uint16_t> on each frame, then Labeller::add(Z0 + f); finish.
//       counts.raw: six uint64 counts, then uint64 live; with out.refl also
//       write_refl(identifier "golden", shoeboxes), as find_spots.cc does
//   shim_check threads16 H W NTHREADS ROUNDS image.raw
//       every thread runs gpu::find on the frame ROUNDS times; exit 0 if all
//       lists are equal to the first
//   shim_check order H W
//       adds frame 5 then frame 4; exit 0 if the second add throws
//       std::runtime_error and leaves the labeller unchanged

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "dext_gpu.hh"
#include "spotfinder_b200.hpp"

namespace {

// Stand-ins with the reference's layouts (src/dials_spots.hh:50-106), as a
// caller in the reference's tree would pass its own.
struct Pixel {
  std::int32_t frame;
  std::uint32_t index;
  std::uint32_t value;
};
struct Spot {
  std::int32_t bbox[6] = {0, 0, 0, 0, 0, 0};
  double position[3] = {0, 0, 0};
  double variance[3] = {0, 0, 0};
  double intensity = 0, intensity_variance = 0;
  std::uint32_t n_signal = 0;
  std::uint64_t first = 0;
};
struct Counts {
  std::uint64_t signal_pixels = 0, groups = 0, too_small = 0, too_large = 0, separated = 0,
                accepted = 0;
};
struct ReflOptions {
  std::size_t panel = 0;
  int id = 0;
  std::string identifier;
  bool shoeboxes = true;
};
struct Options {
  std::size_t min_spot_size = 3;
  std::size_t max_spot_size = 1000;
  double max_separation = 2.0;
  bool two_d = false;
};

template <class T> std::vector<T> read_raw(const char *path, std::size_t n) {
  std::vector<T> v(n);
  FILE *f = std::fopen(path, "rb");
  if (!f || std::fread(v.data(), sizeof(T), n, f) != n)
    throw std::runtime_error(std::string("cannot read ") + path);
  std::fclose(f);
  return v;
}

void write_raw(const char *path, const void *data, std::size_t bytes, bool append = false) {
  FILE *f = std::fopen(path, append ? "ab" : "wb");
  if (!f || (bytes && std::fwrite(data, 1, bytes, f) != bytes))
    throw std::runtime_error(std::string("cannot write ") + path);
  std::fclose(f);
}

template <class T> int cmd_find(std::size_t h, std::size_t w, const char *in, const char *out) {
  const std::vector<T> image = read_raw<T>(in, h * w);
  std::vector<SignalPixel> signal(3); // find() must clear what is there
  const std::int32_t status = gpu::find<T>(image.data(), signal, h, w);
  const std::uint64_t n = signal.size();
  write_raw(out, &status, 4);
  write_raw(out, &n, 8, true);
  write_raw(out, signal.data(), n * sizeof(SignalPixel), true);
  return 0;
}

int cmd_series(int nf, std::size_t h, std::size_t w, std::int64_t z0, bool two_d,
               const char *in, const char *spots_out, const char *pixels_out,
               const char *counts_out, const char *refl_out) {
  const std::vector<std::uint16_t> frames = read_raw<std::uint16_t>(in, nf * h * w);
  Options opt;
  opt.two_d = two_d;
  spotfinder_b200::Labeller<Spot, Pixel, Counts> labeller(h, w, opt);
  // the frame buffer comes from host_alloc, as find_spots.cc's does
  auto *pinned = static_cast<std::uint16_t *>(gpu::host_alloc(h * w * 2));
  std::vector<SignalPixel> signal;
  for (int f = 0; f < nf; f++) {
    const std::uint16_t *src = frames.data() + f * h * w;
    const std::uint16_t *img = src;
    if (pinned) {
      std::memcpy(pinned, src, h * w * 2);
      img = pinned;
    }
    const int status = gpu::find<std::uint16_t>(img, signal, h, w);
    if (status != 0) {
      std::fprintf(stderr, "frame %d: status %d\n", f, status);
      return 2;
    }
    labeller.add(z0 + f, signal);
  }
  gpu::host_free(pinned);
  labeller.finish();
  const auto &spots = labeller.spots();
  const auto &pixels = labeller.pixels();
  write_raw(spots_out, spots.data(), spots.size() * sizeof(Spot));
  write_raw(pixels_out, pixels.data(), pixels.size() * sizeof(Pixel));
  const Counts c = labeller.counts();
  const std::uint64_t live = labeller.live();
  write_raw(counts_out, &c, sizeof(c));
  write_raw(counts_out, &live, 8, true);
  if (refl_out) {
    ReflOptions ro;
    ro.identifier = "golden";
    spotfinder_b200::write_refl(refl_out, spots, pixels, w, ro);
  }
  return 0;
}

int cmd_threads(std::size_t h, std::size_t w, int nthreads, int rounds, const char *in) {
  const std::vector<std::uint16_t> image = read_raw<std::uint16_t>(in, h * w);
  std::vector<SignalPixel> first;
  if (gpu::find<std::uint16_t>(image.data(), first, h, w) != 0)
    return 2;
  std::vector<int> bad(nthreads, 0);
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; t++)
    pool.emplace_back([&, t] {
      std::vector<SignalPixel> mine;
      for (int r = 0; r < rounds; r++) {
        if (gpu::find<std::uint16_t>(image.data(), mine, h, w) != 0 ||
            mine.size() != first.size() ||
            std::memcmp(mine.data(), first.data(), first.size() * sizeof(SignalPixel)) != 0)
          bad[t] = 1;
      }
    });
  for (auto &th : pool)
    th.join();
  for (int b : bad)
    if (b)
      return 1;
  std::printf("threads=%d rounds=%d signal=%zu ok\n", nthreads, rounds, first.size());
  return 0;
}

int cmd_order(std::size_t h, std::size_t w) {
  spotfinder_b200::Labeller<Spot, Pixel, Counts> labeller(h, w, Options{});
  std::vector<SignalPixel> one(1);
  one[0] = SignalPixel{static_cast<std::uint32_t>(w + 1), 9, 1.0f, 121, 0};
  labeller.add(5, one);
  const Counts before = labeller.counts();
  try {
    labeller.add(4, one);
  } catch (const std::runtime_error &e) {
    const Counts after = labeller.counts();
    if (std::memcmp(&before, &after, sizeof(Counts)) != 0)
      return 3;
    std::printf("refused: %s\n", e.what());
    return 0;
  }
  return 1;
}

} // namespace

int main(int argc, char **argv) {
  try {
    const std::string cmd = argc > 1 ? argv[1] : "";
    if (cmd == "info") {
      std::printf("available=%d backend=%s stage0=%s stage2=%s\n", gpu::available() ? 1 : 0,
                  gpu::backend(), gpu::name(gpu::stage0_window()),
                  gpu::name(gpu::stage2_window()));
      return 0;
    }
    if ((cmd == "find16" || cmd == "find32") && argc == 6) {
      const std::size_t h = std::strtoull(argv[2], nullptr, 10);
      const std::size_t w = std::strtoull(argv[3], nullptr, 10);
      return cmd == "find16" ? cmd_find<std::uint16_t>(h, w, argv[4], argv[5])
                             : cmd_find<std::uint32_t>(h, w, argv[4], argv[5]);
    }
    if (cmd == "series16" && (argc == 11 || argc == 12))
      return cmd_series(std::atoi(argv[2]), std::strtoull(argv[3], nullptr, 10),
                        std::strtoull(argv[4], nullptr, 10), std::strtoll(argv[5], nullptr, 10),
                        std::atoi(argv[6]) != 0, argv[7], argv[8], argv[9], argv[10],
                        argc == 12 ? argv[11] : nullptr);
    if (cmd == "threads16" && argc == 7)
      return cmd_threads(std::strtoull(argv[2], nullptr, 10),
                         std::strtoull(argv[3], nullptr, 10), std::atoi(argv[4]),
                         std::atoi(argv[5]), argv[6]);
    if (cmd == "order" && argc == 4)
      return cmd_order(std::strtoull(argv[2], nullptr, 10), std::strtoull(argv[3], nullptr, 10));
    std::fprintf(stderr, "usage: see the head of shim_check.cc\n");
    return 64;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 70;
  }
}
