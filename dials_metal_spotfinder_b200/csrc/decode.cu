// The device side of the chunk codec: LZ4 blocks decoded one warp per block,
// bitshuffle blocks un-transposed in shared memory, the frame written to a
// linear staging buffer and copied into its destination (an engine arena
// row by row). See codec.cu for the formats.

#include <algorithm>

#include "sf_codec.hh"
#include "sf_host.hh"

namespace sf {
namespace {

constexpr int kDecodeWarps = 4;
constexpr unsigned kFull = 0xffffffffu;

struct BlockDesc {
  uint64_t in;  // the LZ4 data, in the chunk
  uint64_t out; // its output, in the frame's bytes
  uint32_t len; // compressed length
  uint32_t n;   // decoded length
};

// One warp decodes one LZ4 block of `cs` bytes into `dst` (n bytes). Lane 0
// parses each sequence; the warp copies its literals and its match in
// parallel (a match of offset d repeats with period d, so byte i of it is
// byte i mod d of the d bytes before it). Every length and offset is checked
// against both buffers before anything is written; returns false on a
// malformed block.
__device__ bool warp_lz4(const uint8_t *__restrict__ src, uint32_t cs, uint8_t *dst, uint32_t n,
                         int lane) {
  uint32_t ip = 0, op = 0;
  while (true) {
    uint32_t lit = 0, ls = 0, off = 0, ml = 0;
    int flag = 0; // 0: a full sequence, 1: the last (literals only), 2: malformed
    if (lane == 0) {
      if (ip >= cs) {
        flag = 2;
      } else {
        const uint32_t token = src[ip++];
        uint64_t l = token >> 4;
        if (l == 15) {
          uint32_t b;
          do {
            if (ip >= cs) {
              flag = 2;
              break;
            }
            b = src[ip++];
            l += b;
          } while (b == 255);
        }
        if (!flag && (l > cs - ip || l > n - op))
          flag = 2;
        if (!flag) {
          lit = static_cast<uint32_t>(l);
          ls = ip;
          ip += lit;
          if (ip == cs) {
            flag = 1;
          } else if (cs - ip < 2) {
            flag = 2;
          } else {
            off = src[ip] | (static_cast<uint32_t>(src[ip + 1]) << 8);
            ip += 2;
            uint64_t m = (token & 15) + 4;
            if ((token & 15) == 15) {
              uint32_t b;
              do {
                if (ip >= cs) {
                  flag = 2;
                  break;
                }
                b = src[ip++];
                m += b;
              } while (b == 255);
            }
            if (!flag && (off == 0 || off > op + lit || m > n - op - lit))
              flag = 2;
            ml = static_cast<uint32_t>(m);
          }
        }
      }
    }
    flag = __shfl_sync(kFull, flag, 0);
    if (flag == 2)
      return false;
    lit = __shfl_sync(kFull, lit, 0);
    ls = __shfl_sync(kFull, ls, 0);
    for (uint32_t i = lane; i < lit; i += 32)
      dst[op + i] = src[ls + i];
    op += lit;
    if (flag == 1)
      break;
    off = __shfl_sync(kFull, off, 0);
    ml = __shfl_sync(kFull, ml, 0);
    __syncwarp();
    for (uint32_t i = lane; i < ml; i += 32)
      dst[op + i] = dst[op - off + (i % off)];
    op += ml;
    __syncwarp();
  }
  __syncwarp();
  return op == n;
}

// Blocks of a chunk, one warp each. With `elem` > 0 the block is bit-
// transposed: it is decoded into shared memory and un-transposed into
// `out`, eight elements a lane at a time; otherwise it is decoded in place.
__global__ void __launch_bounds__(kDecodeWarps * 32)
    decode_blocks(const uint8_t *__restrict__ chunk, const BlockDesc *__restrict__ blocks,
                  uint32_t nblocks, uint32_t elem, uint8_t *out, int *err) {
  extern __shared__ __align__(16) uint8_t decode_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint8_t *buf = decode_smem + static_cast<size_t>(warp) * kMaxBlockBytes;
  const uint32_t nwarps = gridDim.x * kDecodeWarps;
  for (uint32_t b = blockIdx.x * kDecodeWarps + warp; b < nblocks; b += nwarps) {
    const BlockDesc d = blocks[b];
    uint8_t *dst = elem ? buf : out + d.out;
    if (!warp_lz4(chunk + d.in, d.len, dst, d.n, lane)) {
      if (lane == 0)
        atomicExch(err, 1);
      continue;
    }
    if (!elem)
      continue;
    const uint32_t ne = d.n / elem, row = ne / 8;
    uint8_t *o = out + d.out;
    for (uint32_t g = lane; g < row; g += 32) {
      uint8_t bytes[32]; // eight elements of up to four bytes
      for (uint32_t j = 0; j < elem; j++) {
        uint64_t x = 0;
#pragma unroll
        for (int k = 0; k < 8; k++)
          x |= static_cast<uint64_t>(buf[(8 * j + k) * row + g]) << (8 * k);
        const uint64_t y = transpose8x8(x);
#pragma unroll
        for (int i = 0; i < 8; i++)
          bytes[i * elem + j] = static_cast<uint8_t>(y >> (8 * i));
      }
      for (uint32_t q = 0; q < 8 * elem; q++)
        o[8 * g * elem + q] = bytes[q];
    }
    __syncwarp();
  }
}

template <typename T> void grow(T **p, size_t &cap, size_t bytes, const char *what) {
  if (bytes <= cap)
    return;
  cudaFree(*p);
  *p = nullptr;
  cap = 0;
  check(cudaMalloc(reinterpret_cast<void **>(p), bytes), what);
  cap = bytes;
}

} // namespace

DeviceChunkDecoder::~DeviceChunkDecoder() {
  cudaFree(d_chunk_);
  cudaFree(d_blocks_);
  cudaFree(d_linear_);
  cudaFree(d_err_);
}

void DeviceChunkDecoder::enqueue(const uint8_t *chunk, size_t nbytes, const ChunkLayout &L,
                                 size_t height, size_t width, void *dst, size_t dst_pitch,
                                 cudaStream_t s) {
  const size_t row_bytes = width * L.elem;
  if (L.algorithm == SF_CHUNK_RAW) {
    check(cudaMemcpy2DAsync(dst, dst_pitch, chunk, row_bytes, row_bytes, height,
                            cudaMemcpyHostToDevice, s),
          "copying a frame to the device");
    return;
  }
  error_flag();
  static bool configured = false; // setting it twice is harmless
  if (!configured) {
    check(cudaFuncSetAttribute(decode_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(kDecodeWarps * kMaxBlockBytes)),
          "cudaFuncSetAttribute");
    configured = true;
  }
  const size_t frame_bytes = height * row_bytes;
  const size_t nb = L.block_in.size();
  std::vector<BlockDesc> blocks(nb);
  for (size_t b = 0; b < nb; b++)
    blocks[b] = BlockDesc{L.block_in[b], L.block_out[b], L.block_len[b], L.block_n[b]};
  grow(&d_chunk_, chunk_cap_, std::max<size_t>(nbytes, 16), "cudaMalloc chunk");
  grow(&d_blocks_, blocks_cap_, std::max<size_t>(nb, 1) * sizeof(BlockDesc), "cudaMalloc blocks");
  grow(&d_linear_, linear_cap_, std::max<size_t>(frame_bytes, 16), "cudaMalloc frame staging");
  check(cudaMemcpyAsync(d_chunk_, chunk, nbytes, cudaMemcpyHostToDevice, s), "copying a chunk");
  if (nb)
    check(cudaMemcpyAsync(d_blocks_, blocks.data(), nb * sizeof(BlockDesc),
                          cudaMemcpyHostToDevice, s),
          "copying a block table");
  if (nb) {
    const bool bs = L.algorithm == SF_CHUNK_BSLZ4;
    const unsigned grid = static_cast<unsigned>(
        std::min<size_t>((nb + kDecodeWarps - 1) / kDecodeWarps,
                         static_cast<size_t>(device_sm_count()) * 8));
    decode_blocks<<<grid, kDecodeWarps * 32, bs ? kDecodeWarps * kMaxBlockBytes : 0, s>>>(
        d_chunk_, static_cast<const BlockDesc *>(d_blocks_), static_cast<uint32_t>(nb),
        bs ? static_cast<uint32_t>(L.elem) : 0u, d_linear_, d_err_);
    check(cudaGetLastError(), "launching the chunk decoder");
  }
  if (L.raw_bytes)
    check(cudaMemcpyAsync(d_linear_ + (frame_bytes - L.raw_bytes), d_chunk_ + L.raw_in,
                          L.raw_bytes, cudaMemcpyDeviceToDevice, s),
          "copying the raw tail");
  check(cudaMemcpy2DAsync(dst, dst_pitch, d_linear_, row_bytes, row_bytes, height,
                          cudaMemcpyDeviceToDevice, s),
        "copying the decoded frame");
}

int *DeviceChunkDecoder::error_flag() {
  if (!d_err_) {
    check(cudaMalloc(&d_err_, sizeof(int)), "cudaMalloc");
    check(cudaMemset(d_err_, 0, sizeof(int)), "clearing the decode flag");
    check(cudaStreamSynchronize(cudaStreamLegacy), "clearing the decode flag");
  }
  return d_err_;
}

bool DeviceChunkDecoder::take_error() {
  if (!d_err_)
    return false;
  int v = 0;
  check(cudaMemcpy(&v, d_err_, sizeof(int), cudaMemcpyDeviceToHost), "reading the decode flag");
  if (v)
    check(cudaMemset(d_err_, 0, sizeof(int)), "clearing the decode flag");
  return v != 0;
}

} // namespace sf
