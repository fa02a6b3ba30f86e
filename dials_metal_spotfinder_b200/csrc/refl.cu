// sf_refl_write: a DIALS reflection table (.refl) from spots and their
// pixels, byte-identical to the reference's refl::write
// (src/refl.cc:223-351, src/refl.hh:72-74).
//
// The file is a msgpack document: ["dials::af::reflection_table", 2,
// {"identifiers": {...}, "nrows": N, "data": {column: [type, [N, bin]]}}],
// columns in alphabetical order, each a raw little-endian image of N
// elements. The layout is DIALS' own format, so the bytes must match.
//
// The shoebox column (src/refl.cc:295-334) is most of the file: per spot a
// dense z x y x x box of float data, a byte mask and a float background,
// zero except at the spot's signal pixels (data = value, mask = Valid |
// Foreground). It is built on the device, directly in its serialised form,
// a chunk of spots at a time, and streamed to the file; the small columns
// are written from the host.

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/spotfinder_b200.h"
#include "sf_capi.hh"
#include "sf_host.hh"
#include "sf_label.hh"

namespace sf {
namespace {

constexpr uint8_t kMaskSignal = 1 | 4;  // Valid | Foreground
constexpr uint64_t kStrong = 1u << 5;    // dials::af::Flags::Strong
constexpr uint64_t kShoeboxHeader = 29; // panel u32, bbox 6 x i32, version byte

uint64_t box_volume(const Spot &s) {
  return static_cast<uint64_t>(s.bbox[1] - s.bbox[0]) *
         static_cast<uint64_t>(s.bbox[3] - s.bbox[2]) *
         static_cast<uint64_t>(s.bbox[5] - s.bbox[4]);
}

// One warp per spot: header, zeroed data / mask / background, then the
// signal pixels. `pixels` is the chunk's pixel range, starting at pixel
// `pix0` of the caller's list. A pixel outside its box sets *bad.
__global__ void __launch_bounds__(256) shoebox_kernel(const Spot *spots, uint32_t nspots,
                                                      const uint64_t *offsets,
                                                      const Pixel *pixels, uint64_t pix0,
                                                      uint32_t width, uint32_t panel,
                                                      uint8_t *out, int *bad) {
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = warp; i < nspots; i += nwarps) {
    const Spot s = spots[i];
    const uint32_t xs = static_cast<uint32_t>(s.bbox[1] - s.bbox[0]);
    const uint32_t ys = static_cast<uint32_t>(s.bbox[3] - s.bbox[2]);
    const uint32_t zs = static_cast<uint32_t>(s.bbox[5] - s.bbox[4]);
    const uint64_t vol = static_cast<uint64_t>(xs) * ys * zs;
    uint8_t *rec = out + offsets[i];
    if (lane < 7) {
      const uint32_t word = lane == 0 ? panel : static_cast<uint32_t>(s.bbox[lane - 1]);
      for (int b = 0; b < 4; b++)
        rec[4 * lane + b] = static_cast<uint8_t>(word >> (8 * b));
    } else if (lane == 7) {
      rec[28] = 2; // version 2: a byte mask
    }
    uint8_t *body = rec + kShoeboxHeader;
    for (uint64_t k = lane; k < 9 * vol; k += 32)
      body[k] = 0;
    __syncwarp();
    uint8_t *data = body;
    uint8_t *mask = body + 4 * vol;
    for (uint32_t k = lane; k < s.n_signal; k += 32) {
      const Pixel p = pixels[s.first - pix0 + k];
      const int64_t x = static_cast<int64_t>(p.index % width) - s.bbox[0];
      const int64_t y = static_cast<int64_t>(p.index / width) - s.bbox[2];
      const int64_t z = static_cast<int64_t>(p.frame) - s.bbox[4];
      if (x < 0 || y < 0 || z < 0 || x >= xs || y >= ys || z >= zs) {
        atomicExch(bad, 1);
        continue;
      }
      const uint64_t at = (static_cast<uint64_t>(z) * ys + y) * xs + x;
      const uint32_t bits = __float_as_uint(__uint2float_rn(p.value));
      for (int b = 0; b < 4; b++)
        data[4 * at + b] = static_cast<uint8_t>(bits >> (8 * b));
      mask[at] = kMaskSignal;
    }
  }
}

class File {
public:
  explicit File(const char *path) : path_(path) {
    f_ = std::fopen(path, "wb");
    if (!f_)
      throw DeviceError(std::string("cannot write ") + path);
  }
  ~File() {
    if (f_)
      std::fclose(f_);
  }
  void bytes(const void *p, size_t n) {
    if (n && std::fwrite(p, 1, n, f_) != n)
      throw DeviceError("short write to " + path_);
  }
  void byte(uint8_t v) { bytes(&v, 1); }
  void close() {
    FILE *f = f_;
    f_ = nullptr;
    if (std::fclose(f) != 0)
      throw DeviceError("cannot finish writing " + path_);
  }

private:
  std::string path_;
  FILE *f_ = nullptr;
};

// msgpack: big-endian headers, the smallest form that holds the value.
void big_endian(File &f, uint64_t v, int width) {
  uint8_t b[8];
  for (int i = 0; i < width; i++)
    b[i] = static_cast<uint8_t>(v >> (8 * (width - 1 - i)));
  f.bytes(b, width);
}
void mp_uint(File &f, uint64_t v) {
  if (v < 0x80) {
    f.byte(static_cast<uint8_t>(v));
  } else if (v <= 0xff) {
    f.byte(0xcc);
    big_endian(f, v, 1);
  } else if (v <= 0xffff) {
    f.byte(0xcd);
    big_endian(f, v, 2);
  } else if (v <= 0xffffffffull) {
    f.byte(0xce);
    big_endian(f, v, 4);
  } else {
    f.byte(0xcf);
    big_endian(f, v, 8);
  }
}
void mp_str(File &f, const std::string &s) {
  const uint64_t n = s.size();
  if (n < 32) {
    f.byte(static_cast<uint8_t>(0xa0 | n));
  } else if (n <= 0xff) {
    f.byte(0xd9);
    big_endian(f, n, 1);
  } else if (n <= 0xffff) {
    f.byte(0xda);
    big_endian(f, n, 2);
  } else {
    f.byte(0xdb);
    big_endian(f, n, 4);
  }
  f.bytes(s.data(), n);
}
void mp_container(File &f, uint64_t n, uint8_t fix, uint8_t c16, uint8_t c32) {
  if (n < 16) {
    f.byte(static_cast<uint8_t>(fix | n));
  } else if (n <= 0xffff) {
    f.byte(c16);
    big_endian(f, n, 2);
  } else {
    f.byte(c32);
    big_endian(f, n, 4);
  }
}
void mp_array(File &f, uint64_t n) { mp_container(f, n, 0x90, 0xdc, 0xdd); }
void mp_map(File &f, uint64_t n) { mp_container(f, n, 0x80, 0xde, 0xdf); }
void mp_bin(File &f, uint64_t n) {
  if (n > 0xffffffffull)
    throw Refused("a reflection table column would be over 4 GB, which msgpack's binary "
                  "type cannot hold; write without shoeboxes");
  if (n <= 0xff) {
    f.byte(0xc4);
    big_endian(f, n, 1);
  } else if (n <= 0xffff) {
    f.byte(0xc5);
    big_endian(f, n, 2);
  } else {
    f.byte(0xc6);
    big_endian(f, n, 4);
  }
}
// [type, [rows, bin(bytes)]] after the column's name; `bytes` follow.
void column(File &f, const char *name, const char *type, uint64_t rows, uint64_t bytes) {
  mp_str(f, name);
  mp_array(f, 2);
  mp_str(f, type);
  mp_array(f, 2);
  mp_uint(f, rows);
  mp_bin(f, bytes);
}

template <typename T, typename Fn> void fixed_column(File &f, size_t rows, Fn value) {
  std::vector<T> buf;
  buf.reserve(std::min<size_t>(rows, 1 << 16));
  for (size_t i = 0; i < rows; i++) {
    buf.push_back(value(i));
    if (buf.size() == buf.capacity()) {
      f.bytes(buf.data(), buf.size() * sizeof(T));
      buf.clear();
    }
  }
  f.bytes(buf.data(), buf.size() * sizeof(T));
}

// The device side of the shoebox column: buffers grown on demand and kept
// for the thread's next table.
struct ShoeboxStage {
  cudaStream_t stream = nullptr;
  Spot *d_spots = nullptr;
  Pixel *d_pixels = nullptr;
  uint64_t *d_offsets = nullptr;
  uint8_t *d_out = nullptr;
  int *d_bad = nullptr;
  uint8_t *h_out = nullptr; // pinned
  size_t spots_cap = 0, offsets_cap = 0, pixels_cap = 0, out_cap = 0;

  ~ShoeboxStage() {
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
    cudaFree(d_spots);
    cudaFree(d_pixels);
    cudaFree(d_offsets);
    cudaFree(d_out);
    cudaFree(d_bad);
    if (h_out)
      cudaFreeHost(h_out);
  }
  template <typename T> static void grow(T **p, size_t &cap, size_t n, const char *what) {
    if (n <= cap)
      return;
    cudaFree(*p);
    *p = nullptr;
    cap = 0;
    check(cudaMalloc(reinterpret_cast<void **>(p), n * sizeof(T)), what);
    cap = n;
  }
  void reserve(size_t nspots, size_t npixels, size_t out_bytes) {
    if (!stream)
      check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (!d_bad)
      check(cudaMalloc(&d_bad, sizeof(int)), "cudaMalloc");
    grow(&d_spots, spots_cap, nspots, "cudaMalloc shoebox spots");
    grow(&d_offsets, offsets_cap, nspots, "cudaMalloc shoebox offsets");
    grow(&d_pixels, pixels_cap, npixels, "cudaMalloc shoebox pixels");
    if (out_bytes > out_cap) {
      cudaFree(d_out);
      d_out = nullptr;
      if (h_out)
        cudaFreeHost(h_out);
      h_out = nullptr;
      out_cap = 0;
      check(cudaMalloc(&d_out, out_bytes), "cudaMalloc shoebox column");
      check(cudaMallocHost(&h_out, out_bytes), "cudaMallocHost shoebox column");
      out_cap = out_bytes;
    }
  }
};

// The shoebox column's bytes for every spot, in chunks of at most
// kChunkBytes, streamed to the file.
constexpr uint64_t kChunkBytes = 64ull << 20;

void shoebox_column(File &f, const Spot *spots, size_t nspots, const Pixel *pixels,
                    uint32_t width, uint32_t panel) {
  static thread_local ShoeboxStage st;
  size_t i = 0;
  std::vector<uint64_t> offsets;
  while (i < nspots) {
    // the chunk: spots [i, j), whose records fit kChunkBytes (one spot at least)
    size_t j = i;
    uint64_t bytes = 0;
    uint64_t pix_lo = ~0ull, pix_hi = 0;
    offsets.clear();
    while (j < nspots) {
      const uint64_t rec = kShoeboxHeader + 9 * box_volume(spots[j]);
      if (j > i && bytes + rec > kChunkBytes)
        break;
      offsets.push_back(bytes);
      bytes += rec;
      if (spots[j].n_signal) {
        pix_lo = std::min<uint64_t>(pix_lo, spots[j].first);
        pix_hi = std::max<uint64_t>(pix_hi, spots[j].first + spots[j].n_signal);
      }
      j++;
    }
    if (pix_lo > pix_hi)
      pix_lo = pix_hi = 0;
    const size_t n = j - i;
    const uint64_t npix = pix_hi - pix_lo;
    st.reserve(n, std::max<uint64_t>(npix, 1), std::max<uint64_t>(bytes, 16));
    uint64_t *d_off = st.d_offsets;
    const cudaStream_t s = st.stream;
    check(cudaMemcpyAsync(st.d_spots, spots + i, n * sizeof(Spot), cudaMemcpyHostToDevice, s),
          "copying spots");
    if (npix)
      check(cudaMemcpyAsync(st.d_pixels, pixels + pix_lo, npix * sizeof(Pixel),
                            cudaMemcpyHostToDevice, s),
            "copying pixels");
    check(cudaMemcpyAsync(d_off, offsets.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice,
                          s),
          "copying offsets");
    check(cudaMemsetAsync(st.d_bad, 0, sizeof(int), s), "clearing a flag");
    const unsigned blocks =
        static_cast<unsigned>(std::min<size_t>((n + 7) / 8, static_cast<size_t>(device_sm_count()) * 16));
    shoebox_kernel<<<blocks, 256, 0, s>>>(st.d_spots, static_cast<uint32_t>(n), d_off,
                                          st.d_pixels, pix_lo, width, panel, st.d_out, st.d_bad);
    check(cudaGetLastError(), "launching the shoebox kernel");
    int bad = 0;
    check(cudaMemcpyAsync(st.h_out, st.d_out, bytes, cudaMemcpyDeviceToHost, s),
          "copying shoeboxes back");
    check(cudaMemcpyAsync(&bad, st.d_bad, sizeof(int), cudaMemcpyDeviceToHost, s),
          "copying a flag back");
    check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (bad)
      throw Refused("a spot's pixel lies outside its bounding box");
    f.bytes(st.h_out, bytes);
    i = j;
  }
}

void write_refl(const char *path, const Spot *spots, size_t nspots, const Pixel *pixels,
                size_t npixels, uint64_t width, const sf_refl_options &opt) {
  for (size_t i = 0; i < nspots; i++) {
    const Spot &s = spots[i];
    if (s.bbox[1] < s.bbox[0] || s.bbox[3] < s.bbox[2] || s.bbox[5] < s.bbox[4])
      throw Refused("a spot with an inverted bounding box");
    if (s.first + s.n_signal > npixels || s.first + s.n_signal < s.first)
      throw Refused("a spot's pixels run past the pixel list");
  }
  const uint64_t rows = nspots;
  File f(path);
  mp_array(f, 3);
  mp_str(f, "dials::af::reflection_table");
  mp_uint(f, 2);
  mp_map(f, 3);
  mp_str(f, "identifiers");
  const std::string ident = opt.identifier ? opt.identifier : "";
  if (ident.empty()) {
    mp_map(f, 0);
  } else {
    mp_map(f, 1);
    mp_uint(f, static_cast<uint64_t>(static_cast<int64_t>(opt.id)));
    mp_str(f, ident);
  }
  mp_str(f, "nrows");
  mp_uint(f, rows);
  mp_str(f, "data");
  mp_map(f, opt.shoeboxes ? 10 : 9);

  column(f, "bbox", "int6", rows, rows * 24);
  for (size_t i = 0; i < nspots; i += 1024) {
    const size_t n = std::min<size_t>(1024, nspots - i);
    int32_t buf[1024 * 6];
    for (size_t k = 0; k < n; k++)
      std::memcpy(buf + 6 * k, spots[i + k].bbox, 24);
    f.bytes(buf, n * 24);
  }
  column(f, "flags", "std::size_t", rows, rows * 8);
  fixed_column<uint64_t>(f, nspots, [](size_t) { return kStrong; });
  column(f, "id", "int", rows, rows * 4);
  fixed_column<int32_t>(f, nspots, [&](size_t) { return opt.id; });
  column(f, "intensity.sum.value", "double", rows, rows * 8);
  fixed_column<double>(f, nspots, [&](size_t i) { return spots[i].intensity; });
  column(f, "intensity.sum.variance", "double", rows, rows * 8);
  fixed_column<double>(f, nspots, [&](size_t i) { return spots[i].intensity_variance; });
  column(f, "n_signal", "int", rows, rows * 4);
  fixed_column<int32_t>(f, nspots,
                        [&](size_t i) { return static_cast<int32_t>(spots[i].n_signal); });
  column(f, "panel", "std::size_t", rows, rows * 8);
  fixed_column<uint64_t>(f, nspots, [&](size_t) { return opt.panel; });
  if (opt.shoeboxes) {
    uint64_t total = 0;
    for (size_t i = 0; i < nspots; i++)
      total += kShoeboxHeader + 9 * box_volume(spots[i]);
    column(f, "shoebox", "Shoebox<>", rows, total);
    if (nspots)
      shoebox_column(f, spots, nspots, pixels, static_cast<uint32_t>(width),
                     static_cast<uint32_t>(opt.panel));
  }
  column(f, "xyzobs.px.value", "vec3<double>", rows, rows * 24);
  for (size_t i = 0; i < nspots; i++)
    f.bytes(spots[i].position, 24);
  column(f, "xyzobs.px.variance", "vec3<double>", rows, rows * 24);
  for (size_t i = 0; i < nspots; i++)
    f.bytes(spots[i].variance, 24);
  f.close();
}

} // namespace
} // namespace sf

extern "C" int sf_refl_write(const char *path, const sf_spot *spots, size_t nspots,
                             const sf_pixel *pixels, size_t npixels, size_t width,
                             const sf_refl_options *options) {
  return sf::guarded([&] {
    if (!path || !options || width == 0 || width > 0xffffffffu || (nspots && !spots) ||
        (npixels && !pixels))
      return -1;
    sf::write_refl(path, reinterpret_cast<const sf::Spot *>(spots), nspots,
                   reinterpret_cast<const sf::Pixel *>(pixels), npixels, width, *options);
    return 0;
  });
}
