// C++ facade over the C ABI's device labeller, with the public surface of the
// reference's dials_spots::Labeller (src/dials_spots.hh:108-126): add, finish,
// spots, pixels, counts, live. Header-only; link libspotfinder_b200.so.
//
// It is a template over the caller's Spot, Pixel and Counts types so that it
// hands back the very vectors the reference's refl::write takes:
//
//   using Labeller = spotfinder_b200::Labeller<dials_spots::Spot,
//                                              dials_spots::Pixel,
//                                              dials_spots::Counts>;
//   Labeller labeller(height, width, options); // any dials_spots::Options
//
// The types must have the reference's layouts (104, 12 and 48 bytes), which
// is checked at compile time. Results are byte-identical to the reference's
// Labeller: same spots, same row order, same doubles. Errors: a frame out of
// order, a pixel off the frame or pixels not ascending throw
// std::runtime_error before anything changes, as the reference's add does; a
// device failure throws std::runtime_error too.
#ifndef SPOTFINDER_B200_HPP
#define SPOTFINDER_B200_HPP

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "spotfinder_b200.h"

namespace spotfinder_b200 {

inline void throw_for(int status, const char *what) {
  if (status == 0)
    return;
  if (status == -1)
    throw std::invalid_argument(std::string(what) + ": bad argument");
  throw std::runtime_error(std::string(what) + ": " + sf_last_error());
}

template <class SpotT, class PixelT, class CountsT> class Labeller {
  static_assert(sizeof(SpotT) == sizeof(sf_spot) && std::is_trivially_copyable<SpotT>::value,
                "Spot must have the reference's 104-byte layout");
  static_assert(sizeof(PixelT) == sizeof(sf_pixel) && std::is_trivially_copyable<PixelT>::value,
                "Pixel must have the reference's 12-byte layout");
  static_assert(sizeof(CountsT) == sizeof(sf_counts) &&
                    std::is_trivially_copyable<CountsT>::value,
                "Counts must be six 64-bit counters");

public:
  // Options: anything with min_spot_size, max_spot_size, max_separation and
  // two_d members (dials_spots::Options).
  template <class OptionsT>
  Labeller(std::size_t height, std::size_t width, const OptionsT &options) {
    sf_group_options o;
    o.min_spot_size = options.min_spot_size;
    o.max_spot_size = options.max_spot_size;
    o.max_separation = options.max_separation;
    o.two_d = options.two_d ? 1 : 0;
    o.reserved = 0;
    throw_for(sf_labeller_create(height, width, &o, &handle_), "Labeller");
  }
  ~Labeller() { sf_labeller_destroy(handle_); }
  Labeller(const Labeller &) = delete;
  Labeller &operator=(const Labeller &) = delete;

  // `signal`: a frame's list ascending by index (a std::vector of the
  // reference's 16-byte SignalPixel, or of sf_signal_pixel).
  template <class SignalT> void add(std::int64_t frame, const std::vector<SignalT> &signal) {
    static_assert(sizeof(SignalT) == sizeof(sf_signal_pixel) &&
                      std::is_trivially_copyable<SignalT>::value,
                  "signal records are 16 bytes");
    throw_for(sf_labeller_add(handle_, frame,
                              reinterpret_cast<const sf_signal_pixel *>(signal.data()),
                              signal.size()),
              "Labeller::add");
  }

  void finish() { throw_for(sf_labeller_finish(handle_), "Labeller::finish"); }

  const std::vector<SpotT> &spots() const {
    const std::size_t n = sf_labeller_nspots(handle_);
    if (n != spots_.size()) {
      spots_.resize(n);
      throw_for(sf_labeller_spots(handle_, reinterpret_cast<sf_spot *>(spots_.data()), n),
                "Labeller::spots");
    }
    return spots_;
  }

  const std::vector<PixelT> &pixels() const {
    const std::size_t n = sf_labeller_npixels(handle_);
    if (n != pixels_.size()) {
      pixels_.resize(n);
      throw_for(sf_labeller_pixels(handle_, reinterpret_cast<sf_pixel *>(pixels_.data()), n),
                "Labeller::pixels");
    }
    return pixels_;
  }

  const CountsT &counts() const {
    sf_counts c;
    throw_for(sf_labeller_counts(handle_, &c), "Labeller::counts");
    std::memcpy(static_cast<void *>(&counts_), &c, sizeof(c));
    return counts_;
  }

  std::size_t live() const { return sf_labeller_live(handle_); }

private:
  sf_labeller *handle_ = nullptr;
  mutable std::vector<SpotT> spots_;
  mutable std::vector<PixelT> pixels_;
  mutable CountsT counts_{};
};

// refl::write (src/refl.hh:72-74) over sf_refl_write: the same file, byte
// for byte, with the shoebox column built on the device. Options: anything
// with panel, id, identifier (std::string) and shoeboxes members
// (refl::Options). Throws std::runtime_error on failure, as refl::write does.
template <class SpotT, class PixelT, class OptionsT>
void write_refl(const std::string &path, const std::vector<SpotT> &spots,
                const std::vector<PixelT> &pixels, std::size_t width, const OptionsT &options) {
  static_assert(sizeof(SpotT) == sizeof(sf_spot) && std::is_trivially_copyable<SpotT>::value,
                "Spot must have the reference's 104-byte layout");
  static_assert(sizeof(PixelT) == sizeof(sf_pixel) && std::is_trivially_copyable<PixelT>::value,
                "Pixel must have the reference's 12-byte layout");
  sf_refl_options o;
  o.panel = options.panel;
  o.id = options.id;
  o.shoeboxes = options.shoeboxes ? 1 : 0;
  o.identifier = options.identifier.c_str();
  const int status = sf_refl_write(path.c_str(), reinterpret_cast<const sf_spot *>(spots.data()),
                                   spots.size(),
                                   reinterpret_cast<const sf_pixel *>(pixels.data()),
                                   pixels.size(), width, &o);
  if (status != 0)
    throw std::runtime_error("refl::write " + path + ": " + sf_last_error());
}

} // namespace spotfinder_b200

#endif // SPOTFINDER_B200_HPP
