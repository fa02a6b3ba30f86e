// sf_labeller_*: the device labeller behind the reference's
// dials_spots::Labeller interface (src/dials_spots.hh:108-126). Frames are
// added one at a time from host signal lists, exactly as the reference's
// add() takes them, and the spots and pixels accumulate on the host side of
// the handle as the reference's vectors do.
//
// Refusals match the reference's (src/dials_spots.cc:57-100): a frame not
// after the last one, a pixel off the frame, or pixels not ascending by
// index -- reported as -4 with the reason. Unlike the reference, a refused
// add leaves the labeller exactly as it was (the reference can be left with
// part of the refused frame appended).

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/spotfinder_b200.h"
#include "sf_capi.hh"
#include "sf_label.hh"

namespace sf {

struct HostLabeller {
  std::unique_ptr<DeviceLabeller> dev;
  cudaStream_t stream = nullptr;
  std::vector<Spot> spots;
  std::vector<Pixel> pixels;
  bool started = false;
  int64_t last = 0;
  uint64_t height = 0, width = 0;
  SignalPixel *list = nullptr;
  uint64_t list_cap = 0;
  uint32_t *meta = nullptr; // count, capacity
  uint64_t *offs = nullptr; // {0}
  LabelScalars *host_sc = nullptr;
  uint64_t carry = 0;

  ~HostLabeller() {
    if (stream)
      cudaStreamSynchronize(stream);
    dev.reset();
    cudaFree(list);
    cudaFree(meta);
    cudaFree(offs);
    if (host_sc)
      cudaFreeHost(host_sc);
    if (stream)
      cudaStreamDestroy(stream);
  }

  void validate(int64_t frame, const sf_signal_pixel *sig, size_t n) const {
    if (started && frame <= last)
      throw Refused("dials_spots: frame " + std::to_string(frame) + " arrived after frame " +
                    std::to_string(last) + "; frames must be added in ascending order");
    const uint64_t pixels_in_frame = height * width;
    for (size_t i = 0; i < n; i++) {
      if (sig[i].index >= pixels_in_frame)
        throw Refused("dials_spots: signal pixel " + std::to_string(sig[i].index) +
                      " is off the end of the frame");
      if (i > 0 && sig[i].index <= sig[i - 1].index)
        throw Refused("dials_spots: signal pixels are not ascending by index");
    }
  }

  void collect() {
    check(cudaMemcpyAsync(host_sc, dev->scalars(), sizeof(LabelScalars),
                          cudaMemcpyDeviceToHost, stream),
          "reading the labeller state");
    check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    if (host_sc->status != kLabelOk)
      throw DeviceError("labeller capacity exceeded (status " +
                        std::to_string(host_sc->status) + ")");
    const uint64_t ns = host_sc->batch_spots, np = host_sc->batch_pixels;
    const size_t s0 = spots.size(), p0 = pixels.size();
    spots.resize(s0 + ns);
    pixels.resize(p0 + np);
    if (ns)
      check(cudaMemcpyAsync(spots.data() + s0, dev->batch_spots(), ns * sizeof(Spot),
                            cudaMemcpyDeviceToHost, stream),
            "reading spots");
    if (np)
      check(cudaMemcpyAsync(pixels.data() + p0, dev->batch_pixels(), np * sizeof(Pixel),
                            cudaMemcpyDeviceToHost, stream),
            "reading spot pixels");
    check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    carry = host_sc->carry_n;
  }

  void add(int64_t frame, const sf_signal_pixel *sig, size_t n) {
    validate(frame, sig, n);
    if (n > list_cap) {
      cudaFree(list);
      list = nullptr;
      list_cap = 0;
      check(cudaMalloc(&list, std::max<size_t>(n, 1024) * sizeof(SignalPixel)), "cudaMalloc list");
      list_cap = std::max<size_t>(n, 1024);
    }
    dev->reserve(std::max<uint64_t>(n, 1), 1, carry + 1);
    if (n)
      check(cudaMemcpyAsync(list, sig, n * sizeof(SignalPixel), cudaMemcpyHostToDevice, stream),
            "copying the signal list");
    const uint32_t m[2] = {static_cast<uint32_t>(n), static_cast<uint32_t>(n)};
    check(cudaMemcpyAsync(meta, m, sizeof(m), cudaMemcpyHostToDevice, stream), "copying counts");
    dev->set_next_frame(frame, stream);
    dev->enqueue(1, list, offs, meta, nullptr, meta + 1, false, stream);
    collect();
    started = true;
    last = frame;
  }

  void finish() {
    if (!started)
      return;
    dev->reserve(1, 1, carry + 1);
    dev->enqueue(0, list, offs, meta, nullptr, meta + 1, true, stream);
    collect();
  }
};

} // namespace sf

using sf::guarded;
using sf::HostLabeller;

extern "C" {

int sf_labeller_create(size_t height, size_t width, const sf_group_options *options,
                       sf_labeller **out) {
  return guarded([&] {
    if (!out)
      return -1;
    *out = nullptr;
    sf::GroupOptions opt;
    if (options) {
      opt.min_spot_size = options->min_spot_size;
      opt.max_spot_size = options->max_spot_size;
      opt.max_separation = options->max_separation;
      opt.two_d = options->two_d != 0;
    }
    if (height == 0 || width == 0 || height > 0x7fffffffu || width > 0x7fffffffu)
      return -1;
    auto h = std::make_unique<HostLabeller>();
    h->height = height;
    h->width = width;
    h->dev = std::make_unique<sf::DeviceLabeller>(static_cast<int>(height),
                                                  static_cast<int>(width), opt);
    sf::check(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
    sf::check(cudaMalloc(&h->meta, 2 * sizeof(uint32_t)), "cudaMalloc");
    sf::check(cudaMalloc(&h->offs, sizeof(uint64_t)), "cudaMalloc");
    sf::check(cudaMemset(h->offs, 0, sizeof(uint64_t)), "cudaMemset");
    sf::check(cudaMallocHost(&h->host_sc, sizeof(sf::LabelScalars)), "cudaMallocHost");
    sf::check(cudaStreamSynchronize(cudaStreamLegacy), "cudaMemset");
    *out = reinterpret_cast<sf_labeller *>(h.release());
    return 0;
  });
}

void sf_labeller_destroy(sf_labeller *lab) { delete reinterpret_cast<HostLabeller *>(lab); }

int sf_labeller_add(sf_labeller *lab, int64_t frame, const sf_signal_pixel *signal, size_t n) {
  return guarded([&] {
    if (!lab || (n > 0 && !signal))
      return -1;
    reinterpret_cast<HostLabeller *>(lab)->add(frame, signal, n);
    return 0;
  });
}

int sf_labeller_finish(sf_labeller *lab) {
  return guarded([&] {
    if (!lab)
      return -1;
    reinterpret_cast<HostLabeller *>(lab)->finish();
    return 0;
  });
}

int sf_labeller_counts(sf_labeller *lab, sf_counts *out) {
  return guarded([&] {
    if (!lab || !out)
      return -1;
    const HostLabeller *h = reinterpret_cast<HostLabeller *>(lab);
    const sf::LabelScalars &s = *h->host_sc;
    if (!h->started) {
      *out = sf_counts{0, 0, 0, 0, 0, 0};
      return 0;
    }
    out->signal_pixels = s.signal_pixels;
    out->groups = s.groups;
    out->too_small = s.too_small;
    out->too_large = s.too_large;
    out->separated = s.separated;
    out->accepted = s.accepted;
    return 0;
  });
}

size_t sf_labeller_nspots(sf_labeller *lab) {
  return lab ? reinterpret_cast<HostLabeller *>(lab)->spots.size() : 0;
}
size_t sf_labeller_npixels(sf_labeller *lab) {
  return lab ? reinterpret_cast<HostLabeller *>(lab)->pixels.size() : 0;
}
size_t sf_labeller_live(sf_labeller *lab) {
  return lab ? reinterpret_cast<HostLabeller *>(lab)->carry : 0;
}

int sf_labeller_spots(sf_labeller *lab, sf_spot *out, size_t capacity) {
  return guarded([&] {
    if (!lab)
      return -1;
    const auto &v = reinterpret_cast<HostLabeller *>(lab)->spots;
    if (v.size() > capacity)
      return -2;
    if (!v.empty())
      std::memcpy(out, v.data(), v.size() * sizeof(sf::Spot));
    return 0;
  });
}

int sf_labeller_pixels(sf_labeller *lab, sf_pixel *out, size_t capacity) {
  return guarded([&] {
    if (!lab)
      return -1;
    const auto &v = reinterpret_cast<HostLabeller *>(lab)->pixels;
    if (v.size() > capacity)
      return -2;
    if (!v.empty())
      std::memcpy(out, v.data(), v.size() * sizeof(sf::Pixel));
    return 0;
  });
}

} // extern "C"
