// Detector chunk formats (src/decompress.cc:12-134): frames as the HDF5
// filters store them -- uncompressed, "lz4" (the HDF5 LZ4 filter) or "bslz4"
// (bitshuffle + LZ4, what Eiger detectors write) -- encoded on the host (as a
// detector or a replay source would) and decoded either on the host or, for
// the engine, on the device straight into a frame arena, so that only the
// compressed bytes cross PCIe.
//
// Formats, restated from their published descriptions:
//   * HDF5 filter header: 8 bytes uncompressed size, 4 bytes block size (in
//     bytes), both big-endian.
//   * "lz4": then per block of block-size bytes (the last shorter), a 4-byte
//     big-endian compressed length and an LZ4 block.
//   * "bslz4": then per block of block-size / elem elements (the last block
//     rounded down to a multiple of 8 elements), a 4-byte big-endian
//     compressed length and an LZ4 block of the bit-transposed block; the
//     last (elements mod 8) elements follow raw. The bit transpose of n
//     elements of s bytes writes 8s rows of n/8 bytes: row 8j + k holds bit
//     k of byte j of every element, element e at bit (e mod 8) of byte e/8.
//   * LZ4 block: sequences of a token (literal length high nibble, match
//     length - 4 low nibble, 15 = more bytes follow, each 255 adds and a
//     smaller one ends), the literals, a 2-byte little-endian offset and the
//     extra match length; the last sequence is literals only, the last 5
//     bytes are literals and no match starts in the last 12.

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/spotfinder_b200.h"
#include "sf_capi.hh"
#include "sf_codec.hh"
#include "sf_host.hh"

namespace sf {
namespace {

constexpr size_t kHeader = 12;
constexpr int kMinMatch = 4;
constexpr size_t kLastLiterals = 5;
constexpr size_t kMatchLimit = 12;

void put_be(uint8_t *p, uint64_t v, int n) {
  for (int i = 0; i < n; i++)
    p[i] = static_cast<uint8_t>(v >> (8 * (n - 1 - i)));
}
uint64_t get_be(const uint8_t *p, int n) {
  uint64_t v = 0;
  for (int i = 0; i < n; i++)
    v = (v << 8) | p[i];
  return v;
}

// ---- LZ4 block ------------------------------------------------------------

void put_length(std::vector<uint8_t> &out, size_t extra) {
  while (extra >= 255) {
    out.push_back(255);
    extra -= 255;
  }
  out.push_back(static_cast<uint8_t>(extra));
}

// Greedy single-probe hash matcher over a 64 KB window.
void lz4_compress(const uint8_t *in, size_t n, std::vector<uint8_t> &out) {
  constexpr int kHashBits = 14;
  std::vector<int64_t> table(size_t(1) << kHashBits, -1);
  auto hash = [](uint32_t v) { return (v * 2654435761u) >> (32 - kHashBits); };
  auto load32 = [&](size_t p) {
    uint32_t v;
    std::memcpy(&v, in + p, 4);
    return v;
  };
  size_t anchor = 0, p = 0;
  const size_t match_end = n > kMatchLimit ? n - kMatchLimit : 0; // last match start + 1
  while (p < match_end) {
    const uint32_t v = load32(p);
    const uint32_t h = hash(v);
    const int64_t cand = table[h];
    table[h] = static_cast<int64_t>(p);
    if (cand < 0 || p - static_cast<size_t>(cand) > 65535 || load32(cand) != v) {
      p++;
      continue;
    }
    // extend the match, keeping the last 5 bytes as literals
    size_t len = kMinMatch;
    const size_t limit = n - kLastLiterals;
    while (p + len < limit && in[cand + len] == in[p + len])
      len++;
    const size_t lit = p - anchor;
    const size_t ml = len - kMinMatch;
    out.push_back(static_cast<uint8_t>((std::min<size_t>(lit, 15) << 4) | std::min<size_t>(ml, 15)));
    if (lit >= 15)
      put_length(out, lit - 15);
    out.insert(out.end(), in + anchor, in + p);
    const size_t off = p - static_cast<size_t>(cand);
    out.push_back(static_cast<uint8_t>(off & 0xff));
    out.push_back(static_cast<uint8_t>(off >> 8));
    if (ml >= 15)
      put_length(out, ml - 15);
    p += len;
    anchor = p;
  }
  const size_t lit = n - anchor;
  out.push_back(static_cast<uint8_t>(std::min<size_t>(lit, 15) << 4));
  if (lit >= 15)
    put_length(out, lit - 15);
  out.insert(out.end(), in + anchor, in + n);
}

// Returns the bytes written, or -1 on malformed input or overflow.
int64_t lz4_decompress(const uint8_t *in, size_t n, uint8_t *out, size_t cap) {
  size_t ip = 0, op = 0;
  while (true) {
    if (ip >= n)
      return -1; // the block must end with a literals-only sequence
    const uint8_t token = in[ip++];
    size_t lit = token >> 4;
    if (lit == 15) {
      uint8_t b;
      do {
        if (ip >= n)
          return -1;
        b = in[ip++];
        lit += b;
      } while (b == 255);
    }
    if (lit > n - ip || lit > cap - op)
      return -1;
    std::memcpy(out + op, in + ip, lit);
    ip += lit;
    op += lit;
    if (ip == n)
      break; // the last sequence: literals only
    if (n - ip < 2)
      return -1;
    const size_t off = in[ip] | (static_cast<size_t>(in[ip + 1]) << 8);
    ip += 2;
    if (off == 0 || off > op)
      return -1;
    size_t ml = (token & 15) + kMinMatch;
    if ((token & 15) == 15) {
      uint8_t b;
      do {
        if (ip >= n)
          return -1;
        b = in[ip++];
        ml += b;
      } while (b == 255);
    }
    if (ml > cap - op)
      return -1;
    if (off >= ml) {
      std::memcpy(out + op, out + op - off, ml);
      op += ml;
    } else {
      // overlapping: the last `off` bytes repeat; copy in doubling runs
      size_t done = 0, period = off;
      while (done < ml) {
        const size_t n = std::min(period, ml - done);
        std::memcpy(out + op + done, out + op + done - period, n);
        done += n;
        if (period < 4096 && done >= period)
          period *= 2; // the last 2*period bytes are also a whole number of periods
      }
      op += ml;
    }
  }
  return static_cast<int64_t>(op);
}

// ---- bit transpose ----------------------------------------------------------

// Eight elements at a time: byte j of elements 8g..8g+7 is one 64-bit word,
// and its 8 x 8 bit transpose holds byte g of rows 8j..8j+7.
void bit_transpose(const uint8_t *in, uint8_t *out, size_t n, size_t s) {
  const size_t row = n / 8;
  for (size_t g = 0; g < row; g++)
    for (size_t j = 0; j < s; j++) {
      uint64_t x = 0;
      for (int i = 0; i < 8; i++)
        x |= static_cast<uint64_t>(in[(8 * g + i) * s + j]) << (8 * i);
      const uint64_t y = transpose8x8(x);
      for (int k = 0; k < 8; k++)
        out[(8 * j + k) * row + g] = static_cast<uint8_t>(y >> (8 * k));
    }
}

// The inverse, a byte column of eight elements at a time through the 8 x 8
// bit transpose the device decoder uses too.
void bit_untranspose(const uint8_t *in, uint8_t *out, size_t n, size_t s) {
  const size_t row = n / 8;
  for (size_t g = 0; g < row; g++)
    for (size_t j = 0; j < s; j++) {
      uint64_t x = 0;
      for (int k = 0; k < 8; k++)
        x |= static_cast<uint64_t>(in[(8 * j + k) * row + g]) << (8 * k);
      const uint64_t y = transpose8x8(x);
      for (int i = 0; i < 8; i++)
        out[(8 * g + i) * s + j] = static_cast<uint8_t>(y >> (8 * i));
    }
}

size_t default_block_elems(size_t s) {
  // 8 KB per block, a multiple of 8 elements
  return std::max<size_t>(8, (8192 / s) / 8 * 8);
}

} // namespace

void encode_chunk(int algorithm, const uint8_t *in, size_t n_elems, size_t s,
                  std::vector<uint8_t> &out) {
  const size_t bytes = n_elems * s;
  out.clear();
  if (algorithm == SF_CHUNK_RAW) {
    out.assign(in, in + bytes);
    return;
  }
  const size_t block_elems = default_block_elems(s);
  const size_t block_bytes = block_elems * s;
  out.resize(kHeader);
  put_be(out.data(), bytes, 8);
  put_be(out.data() + 8, block_bytes, 4);
  std::vector<uint8_t> tmp, packed;
  auto emit = [&](const uint8_t *p, size_t nb) {
    packed.clear();
    lz4_compress(p, nb, packed);
    uint8_t len[4];
    put_be(len, packed.size(), 4);
    out.insert(out.end(), len, len + 4);
    out.insert(out.end(), packed.begin(), packed.end());
  };
  if (algorithm == SF_CHUNK_LZ4) {
    for (size_t at = 0; at < bytes; at += block_bytes)
      emit(in + at, std::min(block_bytes, bytes - at));
    return;
  }
  // bslz4
  const size_t full = n_elems / block_elems;
  tmp.resize(block_bytes);
  for (size_t b = 0; b < full; b++) {
    bit_transpose(in + b * block_bytes, tmp.data(), block_elems, s);
    emit(tmp.data(), block_bytes);
  }
  const size_t rest = n_elems - full * block_elems;
  const size_t last = rest - rest % 8;
  if (last) {
    bit_transpose(in + full * block_bytes, tmp.data(), last, s);
    emit(tmp.data(), last * s);
  }
  const uint8_t *raw = in + (full * block_elems + last) * s;
  out.insert(out.end(), raw, raw + (rest % 8) * s);
}

ChunkLayout parse_chunk(int algorithm, const uint8_t *data, size_t nbytes, size_t n_elems,
                        size_t s) {
  ChunkLayout L;
  L.algorithm = algorithm;
  L.elem = s;
  L.n_elems = n_elems;
  const size_t bytes = n_elems * s;
  if (algorithm == SF_CHUNK_RAW) {
    if (nbytes != bytes)
      throw std::invalid_argument("an uncompressed chunk of the wrong size for the frame");
    return L;
  }
  if (algorithm != SF_CHUNK_LZ4 && algorithm != SF_CHUNK_BSLZ4)
    throw std::invalid_argument("unknown chunk algorithm");
  if (nbytes < kHeader)
    throw std::invalid_argument("too short for a filter header");
  if (get_be(data, 8) != bytes)
    throw std::invalid_argument("the filter header's size does not match the frame");
  const uint64_t block_bytes = get_be(data + 8, 4);
  if (block_bytes == 0 || block_bytes > 0xffffffffull ||
      (algorithm == SF_CHUNK_BSLZ4 &&
       (block_bytes % s != 0 || (block_bytes / s) % 8 != 0 || block_bytes > kMaxBlockBytes)))
    throw std::invalid_argument("unsupported block size in the filter header");
  L.block_bytes = block_bytes;
  size_t at = kHeader;
  size_t done = 0; // decoded bytes so far
  const size_t coded = algorithm == SF_CHUNK_BSLZ4 ? (n_elems - n_elems % 8) * s : bytes;
  // the block count follows from the header; a chunk that claims more
  // blocks than it has bytes for fails below, so bound the reservation
  const size_t expect = std::min<size_t>((coded + block_bytes - 1) / block_bytes, nbytes / 5 + 1);
  L.block_in.reserve(expect);
  L.block_len.reserve(expect);
  L.block_out.reserve(expect);
  L.block_n.reserve(expect);
  while (done < coded) {
    if (at + 4 > nbytes)
      throw std::invalid_argument("chunk truncated");
    const uint64_t cs = get_be(data + at, 4);
    if (cs == 0 || at + 4 + cs > nbytes)
      throw std::invalid_argument("an LZ4 block length out of range");
    const size_t out_bytes = std::min<size_t>(block_bytes, coded - done);
    L.block_in.push_back(at + 4);
    L.block_len.push_back(static_cast<uint32_t>(cs));
    L.block_out.push_back(done);
    L.block_n.push_back(static_cast<uint32_t>(out_bytes));
    at += 4 + cs;
    done += out_bytes;
  }
  L.raw_in = at;
  L.raw_bytes = bytes - coded;
  if (at + L.raw_bytes != nbytes)
    throw std::invalid_argument("trailing or missing bytes after the LZ4 blocks");
  return L;
}

void decode_chunk_host(const uint8_t *data, const ChunkLayout &L, uint8_t *out) {
  if (L.algorithm == SF_CHUNK_RAW) {
    std::memcpy(out, data, L.n_elems * L.elem);
    return;
  }
  std::vector<uint8_t> tmp(L.block_bytes);
  for (size_t b = 0; b < L.block_in.size(); b++) {
    uint8_t *dst = L.algorithm == SF_CHUNK_BSLZ4 ? tmp.data() : out + L.block_out[b];
    const int64_t got = lz4_decompress(data + L.block_in[b], L.block_len[b], dst, L.block_n[b]);
    if (got != static_cast<int64_t>(L.block_n[b]))
      throw std::invalid_argument("a malformed LZ4 block");
    if (L.algorithm == SF_CHUNK_BSLZ4)
      bit_untranspose(tmp.data(), out + L.block_out[b], L.block_n[b] / L.elem, L.elem);
  }
  std::memcpy(out + (L.n_elems * L.elem - L.raw_bytes), data + L.raw_in, L.raw_bytes);
}

} // namespace sf

extern "C" {

size_t sf_chunk_bound(size_t height, size_t width, int elem_bytes) {
  const size_t bytes = height * width * static_cast<size_t>(elem_bytes);
  return 12 + bytes + bytes / 255 + 32 * (bytes / 8192 + 2);
}

int sf_chunk_encode(int algorithm, const void *image, size_t height, size_t width,
                    int elem_bytes, void *out, size_t capacity, size_t *written) {
  return sf::guarded([&] {
    if (!image || !out || !written || height == 0 || width == 0 ||
        (elem_bytes != 2 && elem_bytes != 4))
      return -1;
    std::vector<uint8_t> buf;
    sf::encode_chunk(algorithm, static_cast<const uint8_t *>(image), height * width,
                     static_cast<size_t>(elem_bytes), buf);
    *written = buf.size();
    if (buf.size() > capacity)
      return -2;
    std::memcpy(out, buf.data(), buf.size());
    return 0;
  });
}

int sf_chunk_decode(int algorithm, const void *chunk, size_t nbytes, size_t height,
                    size_t width, int elem_bytes, void *image) {
  return sf::guarded([&] {
    if (!chunk || !image || height == 0 || width == 0 || (elem_bytes != 2 && elem_bytes != 4))
      return -1;
    const sf::ChunkLayout L =
        sf::parse_chunk(algorithm, static_cast<const uint8_t *>(chunk), nbytes, height * width,
                        static_cast<size_t>(elem_bytes));
    sf::decode_chunk_host(static_cast<const uint8_t *>(chunk), L, static_cast<uint8_t *>(image));
    return 0;
  });
}

} // extern "C"
