// Pixel-mask stamping: the detector's pixel mask (NXmx
// /entry/instrument/detector/pixel_mask, nonzero = a pixel not to use)
// written into the frames as the masked sentinel (the type's maximum) just
// before the threshold, so masked pixels count as masked everywhere the
// reference's rule (value >= max - 1) applies. The reference reads no pixel
// mask and relies on the sentinels in the data alone.

#include "sf_host.hh"

namespace sf {
namespace {

template <typename T>
__global__ void stamp_mask(T *base, const uint64_t *__restrict__ offsets, uint64_t n, T value) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += stride)
    base[offsets[i]] = value;
}

} // namespace

cudaError_t launch_stamp_mask(void *base, int elem_bytes, const uint64_t *offsets, uint64_t n,
                              cudaStream_t s) {
  if (n == 0)
    return cudaSuccess;
  const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 4096));
  if (elem_bytes == 2)
    stamp_mask<uint16_t><<<blocks, 256, 0, s>>>(static_cast<uint16_t *>(base), offsets, n,
                                                 static_cast<uint16_t>(0xffffu));
  else
    stamp_mask<uint32_t><<<blocks, 256, 0, s>>>(static_cast<uint32_t *>(base), offsets, n,
                                                 0xffffffffu);
  return cudaGetLastError();
}

} // namespace sf
