// Chunk codec internals shared by the host codec (codec.cu) and the device
// decoder (decode.cu). The public entry points are in spotfinder_b200.h.
#pragma once

#include <stdint.h>

#include <vector>

#include <cuda_runtime.h>

#include "../../include/spotfinder_b200.h"

namespace sf {

// The largest bitshuffle block the device decodes in shared memory (the
// formats' default is 8 KB).
constexpr uint64_t kMaxBlockBytes = 16384;

// Where each LZ4 block of a chunk is and what it decodes to.
struct ChunkLayout {
  int algorithm = SF_CHUNK_RAW;
  size_t elem = 2, n_elems = 0;
  uint64_t block_bytes = 0;
  std::vector<uint64_t> block_in;  // offset of the block's LZ4 data in the chunk
  std::vector<uint32_t> block_len; // its compressed length
  std::vector<uint64_t> block_out; // offset of its output in the frame's bytes
  std::vector<uint32_t> block_n;   // its output length in bytes
  uint64_t raw_in = 0, raw_bytes = 0; // the trailing uncompressed elements
};

void encode_chunk(int algorithm, const uint8_t *in, size_t n_elems, size_t elem,
                  std::vector<uint8_t> &out);
// Validates the framing (filter header, block lengths, trailing bytes)
// against the frame; throws std::invalid_argument on a mismatch.
ChunkLayout parse_chunk(int algorithm, const uint8_t *data, size_t nbytes, size_t n_elems,
                        size_t elem);
void decode_chunk_host(const uint8_t *data, const ChunkLayout &L, uint8_t *out);

// Decodes chunks into device frames (decode.cu): the chunk's bytes and its
// block table go to the device, one warp decodes each LZ4 block (and undoes
// the bit transpose in shared memory), and the frame lands at `dst` with
// row pitch `dst_pitch`. Staging buffers grow as needed and are reused; the
// work is ordered on the stream it is given, so one decoder serves one
// stream. A malformed block sets a sticky device flag, read by
// take_error().
class DeviceChunkDecoder {
public:
  DeviceChunkDecoder() = default;
  ~DeviceChunkDecoder();
  DeviceChunkDecoder(const DeviceChunkDecoder &) = delete;
  DeviceChunkDecoder &operator=(const DeviceChunkDecoder &) = delete;

  void enqueue(const uint8_t *chunk, size_t nbytes, const ChunkLayout &L, size_t height,
               size_t width, void *dst, size_t dst_pitch, cudaStream_t s);
  // Whether a block failed since the last call (synchronises the device).
  bool take_error();
  // The device flag itself (nonzero after a failed block), allocated and
  // cleared on first use.
  int *error_flag();

private:
  uint8_t *d_chunk_ = nullptr;
  size_t chunk_cap_ = 0;
  void *d_blocks_ = nullptr;
  size_t blocks_cap_ = 0;
  uint8_t *d_linear_ = nullptr;
  size_t linear_cap_ = 0;
  int *d_err_ = nullptr;
};

// 8 x 8 bit-matrix transpose of a 64-bit word: bit 8r + c moves to 8c + r.
__host__ __device__ inline uint64_t transpose8x8(uint64_t x) {
  uint64_t t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
  x = x ^ t ^ (t << 7);
  t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
  x = x ^ t ^ (t << 14);
  t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
  x = x ^ t ^ (t << 28);
  return x;
}

} // namespace sf
