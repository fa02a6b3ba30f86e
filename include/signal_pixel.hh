// The signal record the threshold emits, as the C++ callers of gpu::find see
// it. The layout is the reference's SignalPixel (src/signal_pixel.hh:20-28)
// and sf_signal_pixel in spotfinder_b200.h: 16 bytes, so a list can be handed
// across the C ABI without a copy. In the reference's own tree its header is
// the one on the include path; this one exists so the drop-in builds and is
// tested without that tree. Both declare the same type.
#ifndef SPOTFINDER_SIGNAL_PIXEL_HH
#define SPOTFINDER_SIGNAL_PIXEL_HH

#include <cstdint>

struct SignalPixel {
  std::uint32_t index;      // row-major position in the frame
  std::uint32_t value;      // the pixel as read
  float background;         // the masked 11 x 11 local mean
  std::uint16_t population; // pixels in that mean
  std::uint16_t reserved;   // zero
};

static_assert(sizeof(SignalPixel) == 16, "SignalPixel is 16 bytes");

#endif // SPOTFINDER_SIGNAL_PIXEL_HH
