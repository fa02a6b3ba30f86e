// The device side of the chunk codec: LZ4 blocks decoded one warp per block
// in shared memory, bitshuffle blocks un-transposed there, and the elements
// written straight into the destination frame at its row pitch (an engine
// arena). Raw frames take one contiguous copy and a re-pitching kernel. See
// codec.cu for the formats.

#include <algorithm>
#include <stdexcept>

#include "sf_capi.hh"
#include "sf_codec.hh"
#include "sf_host.hh"

namespace sf {
namespace {

constexpr int kDecodeWarps = 4;
constexpr unsigned kFull = 0xffffffffu;
// Compressed bytes a warp stages in shared memory; a longer block (nearly
// incompressible, so few sequences) is parsed from global memory instead.
constexpr uint32_t kStageCap = 4096;
// Shared memory a warp may own: the decoded block, its staged compressed
// bytes, and the list of its sequence starts (a sequence other than the last
// spans at least three bytes).
__host__ __device__ constexpr uint32_t list_bytes_for(uint32_t stage_bytes) {
  return ((stage_bytes / 3 + 2) * 2 + 15) & ~15u;
}
constexpr uint32_t kWarpSmemMax = static_cast<uint32_t>(kMaxBlockBytes) + kStageCap + 16 +
                                  list_bytes_for(kStageCap + 16);
constexpr uint16_t kSeqEnd = 0xffff, kSeqBad = 0xfffe;

// lane % d and 32 % d for match offsets d < 32, shared by a block's warps.
struct ModTable {
  uint8_t lane_mod[32][32];
  uint8_t step[32];
};

struct BlockDesc {
  uint64_t in;  // the LZ4 data, in the chunk
  uint64_t out; // its output, in the frame's bytes
  uint32_t len; // compressed length
  uint32_t n;   // decoded length
};

// A frame in device memory: rows of row_bytes at `pitch` bytes apart.
struct FrameDst {
  uint8_t *base;
  uint64_t pitch;
  uint64_t row_bytes;
};

size_t round16(size_t x) { return (x + 15) & ~static_cast<size_t>(15); }

// One warp decodes one LZ4 block of `cs` bytes at `src` (shared or global
// memory) into `dst` (shared memory, n bytes). Lane 0 parses each sequence;
// the warp copies its literals and its match in parallel (a match of offset
// d repeats with period d, so byte i of it is byte i mod d of the d bytes
// before it: each lane steps its phase by 32 mod d, no division in the
// loop). Every length and offset is checked against both buffers before
// anything is written; returns false on a malformed block.
__device__ bool warp_lz4(const uint8_t *src, uint32_t cs, uint8_t *dst, uint32_t n, int lane) {
  uint32_t ip = 0, op = 0;
  while (true) {
    // c: offset | flag << 16 (0 a full sequence, 1 the last, 2 malformed);
    // a: literal count; b: literal start; m: match length
    uint32_t a = 0, b = 0, c = 0, m = 0;
    if (lane == 0) {
      int flag = 0;
      uint32_t lit = 0, off = 0, ml = 0;
      if (ip >= cs) {
        flag = 2;
      } else {
        const uint32_t token = src[ip++];
        uint64_t l = token >> 4;
        if (l == 15) {
          uint32_t v;
          do {
            if (ip >= cs) {
              flag = 2;
              break;
            }
            v = src[ip++];
            l += v;
          } while (v == 255);
        }
        if (!flag && (l > cs - ip || l > n - op))
          flag = 2;
        if (!flag) {
          lit = static_cast<uint32_t>(l);
          b = ip;
          ip += lit;
          if (ip == cs) {
            flag = 1;
          } else if (cs - ip < 2) {
            flag = 2;
          } else {
            off = src[ip] | (static_cast<uint32_t>(src[ip + 1]) << 8);
            ip += 2;
            uint64_t mm = (token & 15) + 4;
            if ((token & 15) == 15) {
              uint32_t v;
              do {
                if (ip >= cs) {
                  flag = 2;
                  break;
                }
                v = src[ip++];
                mm += v;
              } while (v == 255);
            }
            if (!flag && (off == 0 || off > op + lit || mm > n - op - lit))
              flag = 2;
            ml = static_cast<uint32_t>(mm);
          }
        }
      }
      a = lit;
      c = off | (static_cast<uint32_t>(flag) << 16);
      m = ml;
    }
    c = __shfl_sync(kFull, c, 0);
    const uint32_t flag = c >> 16, off = c & 0xffffu;
    if (flag == 2)
      return false;
    const uint32_t lit = __shfl_sync(kFull, a, 0);
    b = __shfl_sync(kFull, b, 0);
    for (uint32_t i = lane; i < lit; i += 32)
      dst[op + i] = src[b + i];
    op += lit;
    if (flag == 1)
      break;
    const uint32_t ml = __shfl_sync(kFull, m, 0);
    __syncwarp();
    if (off >= ml) {
      for (uint32_t i = lane; i < ml; i += 32)
        dst[op + i] = dst[op - off + i];
    } else {
      uint32_t q = lane % off;
      const uint32_t step = 32 % off;
      for (uint32_t i = lane; i < ml; i += 32) {
        dst[op + i] = dst[op - off + q];
        q += step;
        if (q >= off)
          q -= off;
      }
    }
    op += ml;
    __syncwarp();
  }
  __syncwarp();
  return op == n;
}

// The same decode with the sequence parsing spread over the warp, for a
// block whose L compressed bytes sit in shared memory at `in`:
//  1. every lane parses a sequence at each of its byte positions p as if a
//     token started there, and records where the next one would start
//     (next[p]; kSeqEnd when its literals end the block, kSeqBad when it
//     runs past the end);
//  2. lane 0 follows next[] from byte 0, listing the real sequence starts;
//  3. 32 sequences at a time, one a lane: parse, an exclusive scan of the
//     output lengths for each sequence's output position, the bounds
//     checks, the literal copies (short ones by their own lane, long ones by
//     the warp), then the matches in order, each by the warp as in
//     warp_lz4 (byte i of a match of offset d is byte i mod d of the d bytes
//     before it; the phases come from the table).
// `next` (2L bytes) may share `dst`: it is dead before any output is
// written. `list` holds L / 3 + 2 entries. Returns false on a malformed
// block, having written nothing past n.
__device__ bool warp_lz4_parallel(const uint8_t *in, uint32_t L, uint16_t *next, uint16_t *list,
                                  uint8_t *dst, uint32_t n, int lane, const ModTable &mt) {
  for (uint32_t p = lane; p < L; p += 32) {
    uint32_t q = p;
    const uint32_t t = in[q++];
    uint32_t lit = t >> 4, nx = kSeqBad;
    bool ok = true;
    if (lit == 15) {
      uint32_t v;
      do {
        if (q >= L) {
          ok = false;
          break;
        }
        v = in[q++];
        lit += v;
      } while (v == 255);
    }
    if (ok && lit <= L - q) {
      q += lit;
      if (q == L) {
        nx = kSeqEnd;
      } else if (L - q >= 2) {
        q += 2;
        if ((t & 15) == 15) {
          uint32_t v;
          do {
            if (q >= L) {
              ok = false;
              break;
            }
            v = in[q++];
          } while (v == 255);
        }
        if (ok)
          nx = q; // q == L: no final sequence, refused by the walk
      }
    }
    next[p] = static_cast<uint16_t>(nx);
  }
  __syncwarp();
  uint32_t k = 0;
  int bad = 0;
  if (lane == 0) {
    uint32_t p = 0;
    while (true) {
      if (p >= L) {
        bad = 1;
        break;
      }
      list[k++] = static_cast<uint16_t>(p);
      const uint32_t nx = next[p];
      if (nx == kSeqEnd)
        break;
      if (nx == kSeqBad) {
        bad = 1;
        break;
      }
      p = nx;
    }
  }
  if (__shfl_sync(kFull, bad, 0))
    return false;
  k = __shfl_sync(kFull, k, 0);
  __syncwarp();
  uint32_t obase = 0;
  for (uint32_t base = 0; base < k; base += 32) {
    const uint32_t j = base + lane;
    const bool active = j < k, last = j + 1 == k;
    uint32_t lit = 0, ls = 0, off = 0, ml = 0;
    if (active) {
      // in bounds: the walk saw this sequence end inside the block
      uint32_t q = list[j];
      const uint32_t t = in[q++];
      lit = t >> 4;
      if (lit == 15) {
        uint32_t v;
        do {
          v = in[q++];
          lit += v;
        } while (v == 255);
      }
      ls = q;
      q += lit;
      if (!last) {
        off = in[q] | (static_cast<uint32_t>(in[q + 1]) << 8);
        q += 2;
        ml = (t & 15) + 4;
        if ((t & 15) == 15) {
          uint32_t v;
          do {
            v = in[q++];
            ml += v;
          } while (v == 255);
        }
      }
    }
    const uint32_t len = lit + ml;
    uint32_t incl = len;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, incl, d);
      if (lane >= d)
        incl += y;
    }
    const uint32_t op = obase + incl - len;
    const bool ok = !active || (op + len <= n && (last || (off != 0 && off <= op + lit)));
    if (__any_sync(kFull, !ok))
      return false;
    if (lit <= 16) {
      for (uint32_t i = 0; i < lit; i++)
        dst[op + i] = in[ls + i];
    }
    for (uint32_t mask = __ballot_sync(kFull, lit > 16); mask; mask &= mask - 1) {
      const int sl = __ffs(mask) - 1;
      const uint32_t o = __shfl_sync(kFull, op, sl), s = __shfl_sync(kFull, ls, sl);
      const uint32_t c = __shfl_sync(kFull, lit, sl);
      for (uint32_t i = lane; i < c; i += 32)
        dst[o + i] = in[s + i];
    }
    __syncwarp();
    const uint32_t mstart = op + lit;
    for (uint32_t mask = __ballot_sync(kFull, ml != 0); mask; mask &= mask - 1) {
      const int sl = __ffs(mask) - 1;
      const uint32_t m = __shfl_sync(kFull, mstart, sl), d = __shfl_sync(kFull, off, sl);
      const uint32_t c = __shfl_sync(kFull, ml, sl);
      uint32_t q, step;
      if (d >= 32) {
        q = lane;
        step = d == 32 ? 0 : 32;
      } else {
        q = mt.lane_mod[d][lane];
        step = mt.step[d];
      }
      for (uint32_t i = lane; i < c; i += 32) {
        dst[m + i] = dst[m - d + q];
        q += step;
        if (q >= d)
          q -= d;
      }
      __syncwarp();
    }
    obase += __shfl_sync(kFull, incl, 31);
  }
  return obase == n;
}

// Where linear byte `o` of the frame lives.
__device__ __forceinline__ uint8_t *frame_at(const FrameDst &D, uint64_t o, uint64_t &col) {
  const uint64_t row = ((o | D.row_bytes) >> 32)
                           ? o / D.row_bytes
                           : static_cast<uint32_t>(o) / static_cast<uint32_t>(D.row_bytes);
  col = o - row * D.row_bytes;
  return D.base + row * D.pitch;
}

// Writes `nb` (<= 32) bytes held in w[0..7] to frame bytes [o, o + nb): the
// widest stores the destination's alignment allows when they sit in one row,
// byte by byte across a row end.
__device__ __forceinline__ void put(const FrameDst &D, uint64_t o, uint32_t nb,
                                   const uint32_t (&w)[8]) {
  uint64_t col;
  uint8_t *row = frame_at(D, o, col);
  uint8_t *p = row + col;
  const uintptr_t at = reinterpret_cast<uintptr_t>(p);
  if (col + nb <= D.row_bytes) {
    if ((nb & 15) == 0 && (at & 15) == 0) {
#pragma unroll
      for (int k = 0; k < 2; k++)
        if (16u * k < nb)
          reinterpret_cast<uint4 *>(p)[k] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2],
                                                       w[4 * k + 3]);
      return;
    }
    if ((nb & 7) == 0 && (at & 7) == 0) {
#pragma unroll
      for (int k = 0; k < 4; k++)
        if (8u * k < nb)
          reinterpret_cast<uint2 *>(p)[k] = make_uint2(w[2 * k], w[2 * k + 1]);
      return;
    }
    if ((nb & 3) == 0 && (at & 3) == 0) {
#pragma unroll
      for (int k = 0; k < 8; k++)
        if (4u * k < nb)
          reinterpret_cast<uint32_t *>(p)[k] = w[k];
      return;
    }
  }
#pragma unroll
  for (uint32_t q = 0; q < 32; q++) {
    if (q < nb) {
      if (col == D.row_bytes) {
        row += D.pitch;
        col = 0;
      }
      row[col++] = static_cast<uint8_t>(w[q >> 2] >> (8 * (q & 3)));
    }
  }
}

// Eight elements of E bytes, group g of a bit-transposed block of `plane`
// bytes per bit plane, back in element order: element i's byte j is byte i
// of the 8 x 8 transpose of bytes (8j + k) * plane + g, k = 0..7.
template <int E>
__device__ __forceinline__ void untranspose(const uint8_t *buf, uint32_t plane, uint32_t g,
                                            uint32_t (&w)[8]) {
  uint32_t lo[E], hi[E];
#pragma unroll
  for (int j = 0; j < E; j++) {
    uint64_t x = 0;
#pragma unroll
    for (int k = 0; k < 8; k++)
      x |= static_cast<uint64_t>(buf[(8 * j + k) * plane + g]) << (8 * k);
    const uint64_t y = transpose8x8(x);
    lo[j] = static_cast<uint32_t>(y);
    hi[j] = static_cast<uint32_t>(y >> 32);
  }
  if constexpr (E == 1) {
    w[0] = lo[0];
    w[1] = hi[0];
  } else if constexpr (E == 2) {
    w[0] = __byte_perm(lo[0], lo[1], 0x5140);
    w[1] = __byte_perm(lo[0], lo[1], 0x7362);
    w[2] = __byte_perm(hi[0], hi[1], 0x5140);
    w[3] = __byte_perm(hi[0], hi[1], 0x7362);
  } else {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const uint32_t a0 = h ? hi[0] : lo[0], a1 = h ? hi[1] : lo[1];
      const uint32_t a2 = h ? hi[2] : lo[2], a3 = h ? hi[3] : lo[3];
      const uint32_t p = __byte_perm(a0, a1, 0x5140), q = __byte_perm(a2, a3, 0x5140);
      const uint32_t r = __byte_perm(a0, a1, 0x7362), t = __byte_perm(a2, a3, 0x7362);
      w[4 * h + 0] = __byte_perm(p, q, 0x5410);
      w[4 * h + 1] = __byte_perm(p, q, 0x7632);
      w[4 * h + 2] = __byte_perm(r, t, 0x5410);
      w[4 * h + 3] = __byte_perm(r, t, 0x7632);
    }
  }
}

// Blocks of a chunk, one warp each, grid-strided. Each warp owns out_bytes
// of shared memory for the decoded block and stage_bytes for its compressed
// bytes. E > 0: bitshuffle blocks of E-byte elements, un-transposed on the
// way out; E == 0: plain LZ4, copied out 16 bytes a lane. Warp 0 of block 0
// also copies the chunk's raw tail (elements after the last block).
template <int E>
__global__ void __launch_bounds__(kDecodeWarps * 32, 1)
    decode_blocks(const uint8_t *__restrict__ chunk, const BlockDesc *__restrict__ blocks,
                  uint32_t nblocks, uint32_t out_bytes, uint32_t stage_bytes, FrameDst D,
                  uint64_t raw_in, uint32_t raw_bytes, uint64_t raw_out, int *err) {
  extern __shared__ __align__(16) uint8_t decode_smem[];
  __shared__ ModTable mt;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t list_bytes = list_bytes_for(stage_bytes);
  uint8_t *obuf =
      decode_smem + static_cast<size_t>(warp) * (out_bytes + stage_bytes + list_bytes);
  uint8_t *ibuf = obuf + out_bytes;
  uint16_t *list = reinterpret_cast<uint16_t *>(ibuf + stage_bytes);
  for (uint32_t i = threadIdx.x; i < 32 * 32; i += blockDim.x) {
    const uint32_t d = i >> 5, l = i & 31;
    mt.lane_mod[d][l] = static_cast<uint8_t>(d ? l % d : 0);
    if (l == 0)
      mt.step[d] = static_cast<uint8_t>(d ? 32 % d : 0);
  }
  __syncthreads();
  if (blockIdx.x == 0 && warp == 0) {
    for (uint32_t i = lane; i < raw_bytes; i += 32) {
      uint64_t col;
      uint8_t *row = frame_at(D, raw_out + i, col);
      row[col] = chunk[raw_in + i];
    }
  }
  const uint32_t nwarps = gridDim.x * kDecodeWarps;
  for (uint32_t b = blockIdx.x * kDecodeWarps + warp; b < nblocks; b += nwarps) {
    const BlockDesc d = blocks[b];
    const uint32_t skew = static_cast<uint32_t>(d.in & 15);
    bool ok;
    if (skew + d.len <= stage_bytes) {
      const uint4 *g = reinterpret_cast<const uint4 *>(chunk + (d.in - skew));
      uint4 *sm = reinterpret_cast<uint4 *>(ibuf);
      const uint32_t nvec = (skew + d.len + 15) / 16;
      for (uint32_t i = lane; i < nvec; i += 32)
        sm[i] = __ldg(g + i);
      __syncwarp();
      ok = 2 * d.len <= out_bytes
               ? warp_lz4_parallel(ibuf + skew, d.len, reinterpret_cast<uint16_t *>(obuf), list,
                                   obuf, d.n, lane, mt)
               : warp_lz4(ibuf + skew, d.len, obuf, d.n, lane);
    } else {
      ok = warp_lz4(chunk + d.in, d.len, obuf, d.n, lane);
    }
    if (!ok) {
      if (lane == 0)
        atomicExch(err, 1);
      __syncwarp();
      continue;
    }
    if constexpr (E > 0) {
      const uint32_t plane = d.n / (8 * E);
      for (uint32_t g = lane; g < plane; g += 32) {
        uint32_t w[8];
        untranspose<E>(obuf, plane, g, w);
        put(D, d.out + 8ull * E * g, 8 * E, w);
      }
    } else {
      const uint32_t pieces = (d.n + 15) / 16;
      for (uint32_t p = lane; p < pieces; p += 32) {
        const uint4 v = reinterpret_cast<const uint4 *>(obuf)[p];
        uint32_t w[8] = {v.x, v.y, v.z, v.w, 0, 0, 0, 0};
        put(D, d.out + 16ull * p, min(16u, d.n - 16 * p), w);
      }
    }
    __syncwarp();
  }
}

// Plain LZ4 blocks too large for shared memory, one warp each, decoded in
// place into the frame's linear bytes at `out` (then re-pitched).
__global__ void __launch_bounds__(kDecodeWarps * 32, 1)
    decode_linear(const uint8_t *__restrict__ chunk, const BlockDesc *__restrict__ blocks,
                  uint32_t nblocks, uint8_t *out, int *err) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t nwarps = gridDim.x * kDecodeWarps;
  for (uint32_t b = blockIdx.x * kDecodeWarps + warp; b < nblocks; b += nwarps) {
    const BlockDesc d = blocks[b];
    if (!warp_lz4(chunk + d.in, d.len, out + d.out, d.n, lane) && lane == 0)
      atomicExch(err, 1);
    __syncwarp();
  }
}

// Rows of row_bytes, contiguous at `src`, to `dst` at `pitch`; one warp a
// row, V-byte words (V divides row_bytes and pitch, and both bases are
// V-aligned).
template <typename V>
__global__ void __launch_bounds__(256)
    repitch_rows(const V *__restrict__ src, uint64_t row_words, uint8_t *dst, uint64_t pitch,
                 uint64_t rows) {
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * 8;
  const int lane = threadIdx.x & 31;
  for (uint64_t r = blockIdx.x * 8ull + (threadIdx.x >> 5); r < rows; r += warps) {
    const V *s = src + r * row_words;
    V *d = reinterpret_cast<V *>(dst + r * pitch);
    for (uint64_t i = lane; i < row_words; i += 32)
      d[i] = __ldg(s + i);
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

// `height` rows of row_bytes, contiguous at device address `src` (256-byte
// aligned), to `dst` at `pitch`, in the widest words that divide both.
void repitch(const uint8_t *src, size_t height, size_t row_bytes, void *dst, size_t pitch,
             cudaStream_t s) {
  const unsigned grid = static_cast<unsigned>(
      std::min<size_t>((height + 7) / 8, static_cast<size_t>(device_sm_count()) * 8));
  uint8_t *d = static_cast<uint8_t *>(dst);
  const uintptr_t at = reinterpret_cast<uintptr_t>(dst);
  auto fits = [&](size_t v) { return row_bytes % v == 0 && pitch % v == 0 && at % v == 0; };
  if (fits(16))
    repitch_rows<uint4><<<grid, 256, 0, s>>>(reinterpret_cast<const uint4 *>(src),
                                             row_bytes / 16, d, pitch, height);
  else if (fits(8))
    repitch_rows<uint2><<<grid, 256, 0, s>>>(reinterpret_cast<const uint2 *>(src),
                                             row_bytes / 8, d, pitch, height);
  else if (fits(4))
    repitch_rows<uint32_t><<<grid, 256, 0, s>>>(reinterpret_cast<const uint32_t *>(src),
                                                row_bytes / 4, d, pitch, height);
  else if (fits(2))
    repitch_rows<uint16_t><<<grid, 256, 0, s>>>(reinterpret_cast<const uint16_t *>(src),
                                                row_bytes / 2, d, pitch, height);
  else
    repitch_rows<uint8_t><<<grid, 256, 0, s>>>(src, row_bytes, d, pitch, height);
  check(cudaGetLastError(), "launching the frame copy");
}

template <int E> void configure_decoder() {
  check(cudaFuncSetAttribute(decode_blocks<E>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kDecodeWarps * kWarpSmemMax)),
        "cudaFuncSetAttribute");
}

} // namespace

DeviceChunkDecoder::~DeviceChunkDecoder() {
  // the owner has drained the stream the decodes ran on; cudaFree waits
  // for the rest
  if (h2d_)
    cudaStreamSynchronize(h2d_);
  for (Set &S : sets_) {
    cudaFree(S.d_in);
    if (S.copied)
      cudaEventDestroy(S.copied);
    if (S.freed)
      cudaEventDestroy(S.freed);
  }
  for (Table &T : tables_) {
    cudaFree(T.d);
    if (T.h)
      cudaFreeHost(T.h);
    if (T.copied)
      cudaEventDestroy(T.copied);
    if (T.freed)
      cudaEventDestroy(T.freed);
  }
  if (h2d_)
    cudaStreamDestroy(h2d_);
  cudaFree(d_linear_);
  cudaFree(d_err_);
}

void DeviceChunkDecoder::prepare() {
  if (h2d_)
    return;
  error_flag();
  static bool configured = false; // per process; setting it twice is harmless
  if (!configured) {
    configure_decoder<0>();
    configure_decoder<1>();
    configure_decoder<2>();
    configure_decoder<4>();
    configured = true;
  }
  for (Set &S : sets_) {
    check(cudaEventCreateWithFlags(&S.copied, cudaEventDisableTiming), "cudaEventCreate");
    check(cudaEventCreateWithFlags(&S.freed, cudaEventDisableTiming), "cudaEventCreate");
  }
  for (Table &T : tables_) {
    check(cudaEventCreateWithFlags(&T.copied, cudaEventDisableTiming), "cudaEventCreate");
    check(cudaEventCreateWithFlags(&T.freed, cudaEventDisableTiming), "cudaEventCreate");
  }
  check(cudaStreamCreateWithFlags(&h2d_, cudaStreamNonBlocking), "cudaStreamCreate");
}

DeviceChunkDecoder::Set &DeviceChunkDecoder::next_set(size_t in_bytes) {
  prepare();
  Set &S = sets_[next_];
  next_ = (next_ + 1) % kSets;
  if (in_bytes > S.in_cap) {
    if (S.used)
      check(cudaEventSynchronize(S.freed), "waiting for a staging set");
    grow(&S.d_in, S.in_cap, in_bytes, "cudaMalloc chunk staging");
  }
  // the copy may overwrite the set once the decode that read it is done
  check(cudaStreamWaitEvent(h2d_, S.freed, 0), "ordering a staging set");
  S.used = true;
  return S;
}

DeviceChunkDecoder::Table &DeviceChunkDecoder::next_table(size_t entries) {
  prepare();
  Table &T = tables_[next_table_];
  next_table_ = (next_table_ + 1) % kTables;
  if (T.used)
    // the host rewrites the page-locked copy below
    check(cudaEventSynchronize(T.copied), "waiting for a block table");
  if (entries > T.cap) {
    if (T.used)
      check(cudaEventSynchronize(T.freed), "waiting for a block table");
    if (T.h)
      cudaFreeHost(T.h);
    T.h = nullptr;
    cudaFree(T.d);
    T.d = nullptr;
    T.cap = 0;
    check(cudaMallocHost(&T.h, entries * sizeof(BlockDesc)), "cudaMallocHost block table");
    check(cudaMalloc(&T.d, entries * sizeof(BlockDesc)), "cudaMalloc block table");
    T.cap = entries;
  }
  check(cudaStreamWaitEvent(h2d_, T.freed, 0), "ordering a block table");
  T.used = true;
  return T;
}

void DeviceChunkDecoder::reserve(size_t chunk_bytes, size_t blocks) {
  for (int k = 0; k < kSets; k++)
    next_set(round16(chunk_bytes) + 16);
  for (int k = 0; k < kTables; k++)
    next_table(std::max<size_t>(blocks, 1));
}

void DeviceChunkDecoder::enqueue_raw(const void *src, size_t height, size_t row_bytes, void *dst,
                                     size_t dst_pitch, cudaStream_t s) {
  const size_t bytes = height * row_bytes;
  if (bytes == 0)
    return;
  Set &S = next_set(round16(bytes));
  check(cudaMemcpyAsync(S.d_in, src, bytes, cudaMemcpyDefault, h2d_), "copying a frame");
  check(cudaEventRecord(S.copied, h2d_), "cudaEventRecord");
  check(cudaStreamWaitEvent(s, S.copied, 0), "ordering after the copy");
  repitch(S.d_in, height, row_bytes, dst, dst_pitch, s);
  check(cudaEventRecord(S.freed, s), "cudaEventRecord");
}

void DeviceChunkDecoder::enqueue(const uint8_t *chunk, size_t nbytes, const ChunkLayout &L,
                                 size_t height, size_t width, void *dst, size_t dst_pitch,
                                 cudaStream_t s) {
  const size_t row_bytes = width * L.elem;
  if (L.algorithm == SF_CHUNK_RAW) {
    enqueue_raw(chunk, height, row_bytes, dst, dst_pitch, s);
    return;
  }
  const bool bs = L.algorithm == SF_CHUNK_BSLZ4;
  if (bs && L.elem != 1 && L.elem != 2 && L.elem != 4)
    throw std::invalid_argument("the device decodes 1, 2 or 4-byte bitshuffle elements");
  const size_t nb = L.block_in.size();
  if (nb == 0 && L.raw_bytes == 0)
    return;
  Set &S = next_set(round16(nbytes) + 16);
  Table &T = next_table(std::max<size_t>(nb, 1));
  BlockDesc *t = static_cast<BlockDesc *>(T.h);
  uint32_t max_len = 0;
  for (size_t b = 0; b < nb; b++) {
    t[b] = BlockDesc{L.block_in[b], L.block_out[b], L.block_len[b], L.block_n[b]};
    max_len = std::max(max_len, L.block_len[b]);
  }
  check(cudaMemcpyAsync(S.d_in, chunk, nbytes, cudaMemcpyDefault, h2d_), "copying a chunk");
  if (nb)
    check(cudaMemcpyAsync(T.d, T.h, nb * sizeof(BlockDesc), cudaMemcpyHostToDevice, h2d_),
          "copying a block table");
  check(cudaEventRecord(S.copied, h2d_), "cudaEventRecord");
  check(cudaEventRecord(T.copied, h2d_), "cudaEventRecord");
  check(cudaStreamWaitEvent(s, S.copied, 0), "ordering after the copy");

  const uint64_t frame_bytes = static_cast<uint64_t>(height) * row_bytes;
  const auto *tbl = static_cast<const BlockDesc *>(T.d);
  const uint32_t n32 = static_cast<uint32_t>(nb);
  if (L.block_bytes > kMaxBlockBytes) {
    // plain LZ4 with blocks beyond shared memory (bitshuffle blocks never
    // are): decoded into a linear frame, then laid out at the pitch
    grow(&d_linear_, linear_cap_, round16(frame_bytes), "cudaMalloc frame staging");
    const unsigned grid = static_cast<unsigned>(std::max<size_t>(
        1, std::min<size_t>((nb + kDecodeWarps - 1) / kDecodeWarps,
                            static_cast<size_t>(device_sm_count()) * 16)));
    decode_linear<<<grid, kDecodeWarps * 32, 0, s>>>(S.d_in, tbl, n32, d_linear_, d_err_);
    check(cudaGetLastError(), "launching the chunk decoder");
    repitch(d_linear_, height, row_bytes, dst, dst_pitch, s);
    check(cudaEventRecord(S.freed, s), "cudaEventRecord");
    check(cudaEventRecord(T.freed, s), "cudaEventRecord");
    return;
  }
  const uint32_t out_bytes = static_cast<uint32_t>(round16(std::max<uint64_t>(L.block_bytes, 16)));
  const uint32_t stage_bytes = static_cast<uint32_t>(round16(std::min(max_len, kStageCap) + 15));
  const size_t smem =
      static_cast<size_t>(kDecodeWarps) * (out_bytes + stage_bytes + list_bytes_for(stage_bytes));
  const unsigned grid = static_cast<unsigned>(std::max<size_t>(
      1, std::min<size_t>((nb + kDecodeWarps - 1) / kDecodeWarps,
                          static_cast<size_t>(device_sm_count()) * 16)));
  const FrameDst D{static_cast<uint8_t *>(dst), dst_pitch, row_bytes};
  const uint64_t raw_out = frame_bytes - L.raw_bytes;
  const uint32_t raw32 = static_cast<uint32_t>(L.raw_bytes);
  const int e = bs ? static_cast<int>(L.elem) : 0;
  if (e == 0)
    decode_blocks<0><<<grid, kDecodeWarps * 32, smem, s>>>(S.d_in, tbl, n32, out_bytes,
                                                           stage_bytes, D, L.raw_in, raw32,
                                                           raw_out, d_err_);
  else if (e == 1)
    decode_blocks<1><<<grid, kDecodeWarps * 32, smem, s>>>(S.d_in, tbl, n32, out_bytes,
                                                           stage_bytes, D, L.raw_in, raw32,
                                                           raw_out, d_err_);
  else if (e == 2)
    decode_blocks<2><<<grid, kDecodeWarps * 32, smem, s>>>(S.d_in, tbl, n32, out_bytes,
                                                           stage_bytes, D, L.raw_in, raw32,
                                                           raw_out, d_err_);
  else
    decode_blocks<4><<<grid, kDecodeWarps * 32, smem, s>>>(S.d_in, tbl, n32, out_bytes,
                                                           stage_bytes, D, L.raw_in, raw32,
                                                           raw_out, d_err_);
  check(cudaGetLastError(), "launching the chunk decoder");
  check(cudaEventRecord(S.freed, s), "cudaEventRecord");
  check(cudaEventRecord(T.freed, s), "cudaEventRecord");
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

extern "C" int sf_chunk_decode_device(int algorithm, const void *chunk, size_t nbytes,
                                      size_t height, size_t width, int elem_bytes,
                                      void *device_image, size_t pitch_bytes) {
  return sf::guarded([&] {
    if (!chunk || !device_image || height == 0 || width == 0 ||
        (elem_bytes != 2 && elem_bytes != 4) || pitch_bytes < width * elem_bytes)
      return -1;
    const sf::ChunkLayout L =
        sf::parse_chunk(algorithm, static_cast<const uint8_t *>(chunk), nbytes, height * width,
                        static_cast<size_t>(elem_bytes));
    // per host thread: a stream and a decoder, reused by later calls
    struct Local {
      cudaStream_t s = nullptr;
      sf::DeviceChunkDecoder dec;
      ~Local() {
        if (s) {
          cudaStreamSynchronize(s);
          cudaStreamDestroy(s);
        }
      }
    };
    static thread_local Local loc;
    if (!loc.s)
      sf::check(cudaStreamCreateWithFlags(&loc.s, cudaStreamNonBlocking), "cudaStreamCreate");
    loc.dec.enqueue(static_cast<const uint8_t *>(chunk), nbytes, L, height, width, device_image,
                    pitch_bytes, loc.s);
    sf::check(cudaStreamSynchronize(loc.s), "cudaStreamSynchronize");
    if (loc.dec.take_error())
      throw sf::DeviceError("a malformed LZ4 block");
    return 0;
  });
}
