// Device-side building blocks shared by the spot-finder kernels: the
// 16-byte signal record, pixel-type traits, and thin inline-PTX wrappers for
// mbarrier waits and TMA tile loads on sm_100a.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sf {

// The record the threshold emits per signal pixel: src/signal_pixel.hh:20-26
// in the reference, kept byte-identical so a list can be handed straight to
// the reference's grouping or written by its refl code.
struct SignalPixel {
  uint32_t index;      // row-major position in the frame
  uint32_t value;      // the raw pixel (0 for a masked one, which never emits)
  float background;    // the masked 11 x 11 local mean
  uint16_t population; // pixels that mean was taken over
  uint16_t reserved;   // always 0
};
static_assert(sizeof(SignalPixel) == 16, "SignalPixel must be 16 bytes");

// Geometry of the streaming threshold. A warp owns a strip of 256 pixel
// columns (8 per lane); the outer 10 on each side are halo, 4 more on the
// right are padding, so a strip produces 232 output columns. Strips start at
// multiples of 232 elements in a buffer whose frame sits 10 columns in from
// the left, which keeps every strip's first column 16-byte aligned for TMA.
constexpr int kLaneCols = 8;
constexpr int kStripCols = 32 * kLaneCols; // 256
constexpr int kHalo = 10;                  // 3 (7x7) + 2 (5x5) + 5 (11x11)
constexpr int kStripOut = 232;             // outputs per strip
constexpr int kMarginLeft = kHalo;         // frame column 0 at buffer column 10
constexpr int kMarginRows = kHalo;         // rows of fill above and below
constexpr int kRingRows = 20;              // rows of a strip held in smem
constexpr int kBoxRows = 2;                // rows per TMA box
constexpr int kRingStages = kRingRows / kBoxRows;
constexpr uint32_t kChunkRecords = 1024;   // staging pool allocation unit
// The most records a warp stages at once (two output rows of a strip); a
// staging chunk is abandoned when that many might not fit, so each chunk
// wastes fewer than this.
constexpr uint32_t kMaxStaged = 2 * kStripOut;

// Pixel-type traits. The window sums of the reference are accumulated in
// accumulator_t<T> (uint32 for 16-bit pixels, uint64 for 32-bit) and tested
// in real_t<T> (float / double), src/dext.hh:18-38. Here the count and the
// sum of a window are packed into one accumulator word (count in the high
// bits), which is exact because both stay inside their fields; the sum of
// squares has a word of its own and wraps exactly as the reference's does.
template <typename T> struct Traits;

template <> struct Traits<uint16_t> {
  using Acc = uint32_t;
  static constexpr uint32_t kMasked = 0xfffeu; // pixels >= this are masked
  static constexpr int kShift7 = 22;  // 49 * 65533 < 2^22, count <= 49 < 2^6
  static constexpr int kShift11 = 23; // 121 * 65533 < 2^23, count <= 121 < 2^7
  static constexpr int kRowVecs = 1;  // uint4 loads per lane per row
};

template <> struct Traits<uint32_t> {
  using Acc = uint64_t;
  static constexpr uint32_t kMasked = 0xfffffffeu;
  static constexpr int kShift7 = 40;  // 49 * 2^32 < 2^40
  static constexpr int kShift11 = 40; // 121 * 2^32 < 2^40, count < 2^7
  static constexpr int kRowVecs = 2;
};

// One frame of a batch as the device sees it. The arena is a single pitched
// 2D array holding every frame of the batch one above another, each with
// kMarginRows rows of fill above and below and the fill value everywhere
// outside the frame; the fill is the masked sentinel, so the kernels need no
// border logic (a pixel off the frame and a masked pixel are treated alike
// everywhere in the reference's arithmetic).
struct FrameDesc {
  int64_t row0;         // arena row of frame row 0
  int32_t height;
  int32_t width;
  int32_t strips;       // ceil(width / kStripOut)
  int32_t segments;     // ceil(height / seg_rows)
  int32_t seg_rows;     // output rows per task
  uint32_t task_begin;  // first task of this frame
  uint64_t tile_base;   // first tile (row 0, strip 0) in the tile arrays
  uint64_t out_base;    // first record of this frame's output list
  uint32_t capacity;    // records this frame's list may hold
  uint32_t pad_;
};

// Error codes a kernel leaves in its status word.
enum : int {
  kStatusOk = 0,
  kStatusTmaTimeout = 1,
  kStatusPoolExhausted = 2,
  kStatusSpinTimeout = 3,
};

// --------------------------------------------------------------------------
// PTX wrappers
// --------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], "
               "%2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(done)
               : "r"(smem_u32(bar)), "r"(parity)
               : "memory");
  return done != 0;
}

// Waits for phase `parity` of `bar` to complete, giving up after `limit`
// polls (each try_wait itself blocks for a hardware-chosen interval). Returns
// false on timeout; the caller records the failure and stops.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint32_t limit) {
  for (uint32_t i = 0; i < limit; i++) {
    if (mbar_try_wait(bar, parity))
      return true;
  }
  return false;
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// A 2D tiled TMA load of one box into shared memory, completing on `bar`.
// Each load fills only the issuing CTA's shared memory, from this GPU's own memory.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map,
                                            uint64_t *bar, int32_t x,
                                            int32_t y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cta.global.tile.mbarrier::complete_tx::"
      "bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

} // namespace sf
