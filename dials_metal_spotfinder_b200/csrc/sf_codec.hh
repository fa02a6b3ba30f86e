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

// Brings frames from host memory into device frames (decode.cu): compressed
// chunks (their bytes and block table go to the device, one warp decodes
// each LZ4 block in shared memory and undoes the bit transpose, and writes
// the elements straight into `dst` at row pitch `dst_pitch`) and raw frames
// (one contiguous copy, then laid out at the pitch by a kernel).
//
// Host-to-device copies run on the decoder's own stream into a ring of
// staging sets, so frame k+1 crosses the link while frame k is decoded; the
// decode itself is ordered on the stream the caller gives, so one decoder
// serves one stream and work on that stream after enqueue() sees the frame.
// The caller keeps its host buffer unchanged until that stream has passed
// the frame. A malformed block sets a sticky device flag, read by
// take_error().
class DeviceChunkDecoder {
public:
  DeviceChunkDecoder() = default;
  ~DeviceChunkDecoder();
  DeviceChunkDecoder(const DeviceChunkDecoder &) = delete;
  DeviceChunkDecoder &operator=(const DeviceChunkDecoder &) = delete;

  void enqueue(const uint8_t *chunk, size_t nbytes, const ChunkLayout &L, size_t height,
               size_t width, void *dst, size_t dst_pitch, cudaStream_t s);
  // A raw frame of height rows of row_bytes each, contiguous at `src` (host
  // or device memory).
  void enqueue_raw(const void *src, size_t height, size_t row_bytes, void *dst, size_t dst_pitch,
                   cudaStream_t s);
  // Allocates every staging set for chunks up to `chunk_bytes` with up to
  // `blocks` LZ4 blocks, so later calls allocate nothing.
  void reserve(size_t chunk_bytes, size_t blocks);
  // Whether a block failed since the last call (synchronises the device).
  bool take_error();
  // The device flag itself (nonzero after a failed block), allocated and
  // cleared on first use.
  int *error_flag();

  static constexpr int kSets = 3;    // device staging buffers for chunks
  static constexpr int kTables = 32; // block tables, so the host rarely waits

private:
  // A chunk's (or raw frame's) bytes on the device. Ordered on the device
  // only: the copy into it waits for the decode that last read it.
  struct Set {
    uint8_t *d_in = nullptr;
    size_t in_cap = 0;
    cudaEvent_t copied = nullptr; // its host-to-device copies are done
    cudaEvent_t freed = nullptr;  // the decode that read it is done
    bool used = false;
  };
  // A block table, page-locked for the copy and on the device. The host
  // rewrites one only after its copy of kTables uploads ago is done.
  struct Table {
    void *h = nullptr;
    void *d = nullptr;
    size_t cap = 0; // entries
    cudaEvent_t copied = nullptr;
    cudaEvent_t freed = nullptr;
    bool used = false;
  };
  Set &next_set(size_t in_bytes);
  Table &next_table(size_t entries);
  void prepare();

  Set sets_[kSets];
  Table tables_[kTables];
  int next_ = 0, next_table_ = 0;
  cudaStream_t h2d_ = nullptr;
  uint8_t *d_linear_ = nullptr; // a frame decoded from blocks beyond shared memory
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
