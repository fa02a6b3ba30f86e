// The fused extended-dispersion threshold: src/dext.cc:9-225 of the
// reference (dispersion test, erode, masked background, Poisson test, emit),
// as one streaming kernel per batch of frames.
//
// Decomposition. A task is one strip of 256 buffer columns (232 output
// columns plus halo) by one segment of output rows of one frame. A warp owns
// a task at a time and walks down it row by row; warps never talk to each
// other. Each warp has a ring of 20 rows of its strip in shared memory, fed
// 2 rows at a time by TMA (one elected lane issues, an mbarrier per stage).
//
// Per input row r entering at the bottom of the ring, each lane (8 columns)
// updates, all in registers:
//   - vertical 7-row running sums of the valid count+sum (packed) and of the
//     sum of squares, from rows r and r-7;
//   - the 7 x 7 window sums at row r-3 by a horizontal pass (warp shuffles
//     for the 3 neighbour columns each side), and the dispersion test there
//     -> one bit per pixel (masked pixels are 1, src/dext.cc:113);
//   - the 5 x 5 erode at row r-5 on those bits (vertical AND of five
//     8-bit rows, then horizontal AND with 2 shuffled neighbour bits);
//   - vertical 11-row running sums of the count+sum of pixels that are valid
//     and not kept by the erode, from rows r-5 and r-16;
//   - at row r-10, for the pixels that are candidates (value > 0 and kept
//     by the erode), taken one per lane, the 11 x 11 window as the sum
//     of 11 columns' vertical sums from shared memory, the Poisson test,
//     and the emit of a SignalPixel into a staging pool.
// Every window is the reference's window clipped to the frame: the arena
// holds the masked sentinel everywhere outside the frame, and a pixel off the
// frame and a masked pixel are treated identically by every step of the
// reference's arithmetic (excluded from every sum, 1 in the erode input).
//
// Cost. The running sums are updated as if every pixel entering and leaving
// were valid -- then the packed counts cancel and an update is one add of
// (entering - leaving) -- and corrected afterwards for the few pixels that
// are not (masked, or kept by the erode), only in rows where the warp holds
// one. When no pixel of the strip in the 7 rows of a dispersion window is
// masked, every window holds 49 pixels and the test runs with m = 49 as
// constants; otherwise m, and the square root from a table built on the
// device with the reference's own operation, vary per pixel. Either way the
// test runs two pixels at a time in the sm_100 packed float2 pipe.
//
// Arithmetic. Sums are exact integers; the sum of squares wraps in 32 bits
// for 16-bit pixels (64 for 32-bit) exactly as the reference's accumulator
// does. The two tests run in float for 16-bit pixels and double for 32-bit,
// one IEEE rounding per operation in the reference's order, through _rn
// intrinsics so that nothing is contracted into an FMA (the fma forms below
// multiply by -1, which is exact, so each is one rounding of a difference:
// the same as the reference's subtraction). `lhs > rhs` is read off the sign
// of the correctly rounded rhs - lhs, which rounding cannot flip.
//
// Output order. Records for the tile (row, strip) land contiguously in the
// staging pool; the tile's count and start go to two small arrays. The
// placement kernels (place.cu) then scan the counts in row-major tile order,
// which is ascending pixel index, and copy each tile's records to the final
// list -- so the list comes out sorted by index with no sort.

#include <math_constants.h>

#include <type_traits>

#include "sf_device.cuh"
#include "sf_host.hh"

namespace sf {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kNoChunk = 0xffffffffu;
constexpr int kRadius11 = 5; // the background window is 11 x 11

template <typename T> struct Real;
template <> struct Real<uint16_t> { using type = float; };
template <> struct Real<uint32_t> { using type = double; };

// sqrt(2 (m - 1)) for m in [2, 63], +inf below 2: with +inf the test's right
// side is +inf or NaN, so `lhs > rhs` is false exactly where the reference's
// `m_sum >= 2` guard (src/dext.cc:97) is.
__device__ __forceinline__ float sqrt_term(int m, float) {
  return m >= 2 ? __fsqrt_rn(__fmul_rn(2.0f, __fsub_rn(__int2float_rn(m), 1.0f)))
                : CUDART_INF_F;
}
__device__ __forceinline__ double sqrt_term(int m, double) {
  return m >= 2 ? __dsqrt_rn(__dmul_rn(2.0, __dsub_rn(__int2double_rn(m), 1.0))) : CUDART_INF;
}

// An integer below 2^23 with its bits OR'd under the exponent of 2^23: as a
// float that is 2^23 + v exactly.
__device__ __forceinline__ float magic_bits(uint32_t v) {
  return __uint_as_float(v | 0x4b000000u);
}

// Shifts `bits` left by one and brings in the sign bit of `x`.
__device__ __forceinline__ uint32_t push_sign(uint32_t bits, float x) {
  return __funnelshift_l(__float_as_uint(x), bits, 1);
}

// --------------------------------------------------------------------------
// The two tests, in the reference's arithmetic.
// --------------------------------------------------------------------------

// src/dext.cc:97-110 with R = float, for the 8 columns of a lane: window
// count+sum packed in hs (count << 22 | sum), sum of squares in hq. `sq` is
// the per-count table (sqrt_term). Bit k set where the window is dispersed.
__device__ __forceinline__ uint32_t dispersion_bits(const uint32_t (&hs)[8],
                                                    const uint32_t (&hq)[8],
                                                    const float *sq) {
  const float2 magic = make_float2(-8388608.0f, -8388608.0f);
  const float2 neg1 = make_float2(-1.0f, -1.0f);
  const float2 six = make_float2(6.0f, 6.0f);
  uint32_t bits = 0;
#pragma unroll
  for (int k = 6; k >= 0; k -= 2) {
    const uint32_t m0 = hs[k] >> 22, m1 = hs[k + 1] >> 22;
    const float2 S = __fadd2_rn(make_float2(magic_bits(hs[k] & 0x3fffffu),
                                            magic_bits(hs[k + 1] & 0x3fffffu)),
                                magic);
    const float2 M = __fadd2_rn(make_float2(magic_bits(m0), magic_bits(m1)), magic);
    const float2 Q = make_float2(__uint2float_rn(hq[k]), __uint2float_rn(hq[k + 1]));
    const float2 R = make_float2(sq[m0], sq[m1]);
    const float2 Mm1 = __fadd2_rn(M, neg1);                   // m - 1 (exact)
    const float2 t1 = __fmul2_rn(M, Q);                       // m * s2
    const float2 t2 = __fmul2_rn(S, S);                       // s * s
    const float2 t3 = __ffma2_rn(t2, neg1, t1);               // t1 - t2
    const float2 t5 = __fmul2_rn(S, Mm1);                     // s * (m - 1)
    const float2 lhs = __ffma2_rn(t5, neg1, t3);              // t3 - t5
    const float2 rhs = __fmul2_rn(__fmul2_rn(S, six), R);     // s * 6 * sqrt(2(m-1))
    const float2 d = __ffma2_rn(lhs, neg1, rhs);              // rhs - lhs
    bits = push_sign(bits, d.y);
    bits = push_sign(bits, d.x);
  }
  return bits;
}

// The same when every window holds 49 pixels: m, m - 1 and the square root
// are constants (sq49 = sqrt_term(49)). s * 48 is formed as 8 * (s * 6):
// scaling by a power of two is exact and commutes with rounding, so
// fl(s * 48) = 8 fl(s * 6), and t3 - fl(s * 48) is one fused operation on
// the already rounded fl(s * 6), which the right side needs anyway.
__device__ __forceinline__ uint32_t dispersion_bits49(const uint32_t (&hs)[8],
                                                      const uint32_t (&hq)[8], float sq49) {
  const float2 magic = make_float2(-8388608.0f, -8388608.0f);
  const float2 neg1 = make_float2(-1.0f, -1.0f);
  const float2 neg8 = make_float2(-8.0f, -8.0f);
  const float2 six = make_float2(6.0f, 6.0f);
  const float2 c49 = make_float2(49.0f, 49.0f);
  const float2 R = make_float2(sq49, sq49);
  uint32_t bits = 0;
#pragma unroll
  for (int k = 6; k >= 0; k -= 2) {
    const float2 S = __fadd2_rn(make_float2(magic_bits(hs[k] & 0x3fffffu),
                                            magic_bits(hs[k + 1] & 0x3fffffu)),
                                magic);
    const float2 Q = make_float2(__uint2float_rn(hq[k]), __uint2float_rn(hq[k + 1]));
    const float2 t1 = __fmul2_rn(c49, Q);
    const float2 t2 = __fmul2_rn(S, S);
    const float2 t3 = __ffma2_rn(t2, neg1, t1);
    const float2 u = __fmul2_rn(S, six);                      // s * 6
    const float2 lhs = __ffma2_rn(u, neg8, t3);               // t3 - 8 (s * 6)
    const float2 rhs = __fmul2_rn(u, R);
    const float2 d = __ffma2_rn(lhs, neg1, rhs);
    bits = push_sign(bits, d.y);
    bits = push_sign(bits, d.x);
  }
  return bits;
}

// The same with R = double, for 32-bit pixels (count << 40 | sum).
__device__ __forceinline__ uint32_t dispersion_bits(const uint64_t (&hs)[8],
                                                    const uint64_t (&hq)[8],
                                                    const double *sq) {
  uint32_t bits = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const uint32_t m = static_cast<uint32_t>(hs[k] >> 40);
    const double md = __uint2double_rn(m);
    const double sd = __ull2double_rn(hs[k] & ((1ull << 40) - 1));
    const double qd = __ull2double_rn(hq[k]);
    const double lhs = __dsub_rn(__dsub_rn(__dmul_rn(md, qd), __dmul_rn(sd, sd)),
                                 __dmul_rn(sd, __dsub_rn(md, 1.0)));
    const double rhs = __dmul_rn(__dmul_rn(sd, 6.0), sq[m]);
    bits |= (lhs > rhs ? 1u : 0u) << k;
  }
  return bits;
}

// src/dext.cc:200-213: mean over the masked window, then p >= mean + 3 sqrt(mean).
__device__ __forceinline__ bool poisson(uint32_t p, uint32_t m, uint32_t s,
                                        float *background) {
  const float mean =
      m >= 2 ? __fdiv_rn(__uint2float_rn(s), __uint2float_rn(m)) : 0.0f;
  *background = mean;
  return __uint2float_rn(p) >= __fadd_rn(mean, __fmul_rn(3.0f, __fsqrt_rn(mean)));
}

__device__ __forceinline__ bool poisson(uint32_t p, uint64_t m, uint64_t s,
                                        float *background) {
  const double mean =
      m >= 2 ? __ddiv_rn(__ull2double_rn(s), __ull2double_rn(m)) : 0.0;
  *background = __double2float_rn(mean);
  return __uint2double_rn(p) >= __dadd_rn(mean, __dmul_rn(3.0, __dsqrt_rn(mean)));
}

// --------------------------------------------------------------------------
// Row access
// --------------------------------------------------------------------------

// The lane's 8 pixels of one ring row, and whether any is masked.
template <typename T> struct LaneRow;

template <> struct LaneRow<uint16_t> {
  uint4 v;
  __device__ __forceinline__ void load(const uint16_t *row, int lane) {
    v = reinterpret_cast<const uint4 *>(row)[lane];
  }
  __device__ __forceinline__ void unpack(uint32_t (&p)[8]) const {
    p[0] = v.x & 0xffffu; p[1] = v.x >> 16;
    p[2] = v.y & 0xffffu; p[3] = v.y >> 16;
    p[4] = v.z & 0xffffu; p[5] = v.z >> 16;
    p[6] = v.w & 0xffffu; p[7] = v.w >> 16;
  }
  // Nonzero iff a pixel is 0xfffe or 0xffff (masked): the halfword maxima
  // of the four words, compared with 0xfffe per half.
  __device__ __forceinline__ uint32_t any_masked() const {
    const uint32_t m = __vmaxu2(__vmaxu2(v.x, v.y), __vmaxu2(v.z, v.w));
    return __vcmpgeu2(m, 0xfffefffeu);
  }
  // Bit k set where pixel k is masked.
  __device__ __forceinline__ uint32_t masked_bits() const {
    const uint32_t x = (__vcmpgeu2(v.x, 0xfffefffeu) & 0x00010001u) |
                       ((__vcmpgeu2(v.y, 0xfffefffeu) & 0x00010001u) << 2) |
                       ((__vcmpgeu2(v.z, 0xfffefffeu) & 0x00010001u) << 4) |
                       ((__vcmpgeu2(v.w, 0xfffefffeu) & 0x00010001u) << 6);
    return (x | (x >> 15)) & 0xffu;
  }
};

template <> struct LaneRow<uint32_t> {
  uint4 a, b;
  __device__ __forceinline__ void load(const uint32_t *row, int lane) {
    const uint4 *v = reinterpret_cast<const uint4 *>(row + 8 * lane);
    a = v[0];
    b = v[1];
  }
  __device__ __forceinline__ void unpack(uint32_t (&p)[8]) const {
    p[0] = a.x; p[1] = a.y; p[2] = a.z; p[3] = a.w;
    p[4] = b.x; p[5] = b.y; p[6] = b.z; p[7] = b.w;
  }
  __device__ __forceinline__ uint32_t masked_bits() const {
    const uint32_t m = Traits<uint32_t>::kMasked;
    return (a.x >= m ? 1u : 0u) | (a.y >= m ? 2u : 0u) | (a.z >= m ? 4u : 0u) |
           (a.w >= m ? 8u : 0u) | (b.x >= m ? 16u : 0u) | (b.y >= m ? 32u : 0u) |
           (b.z >= m ? 64u : 0u) | (b.w >= m ? 128u : 0u);
  }
  __device__ __forceinline__ uint32_t any_masked() const { return masked_bits(); }
};

template <typename T>
__device__ __forceinline__ void load_pixels(const T *row, int lane, uint32_t (&p)[8]) {
  LaneRow<T> r;
  r.load(row, lane);
  r.unpack(p);
}

__device__ __forceinline__ uint32_t shfl_up(uint32_t v) { return __shfl_up_sync(kFull, v, 1); }
__device__ __forceinline__ uint32_t shfl_down(uint32_t v) { return __shfl_down_sync(kFull, v, 1); }
__device__ __forceinline__ uint64_t shfl_up(uint64_t v) {
  const uint32_t lo = __shfl_up_sync(kFull, static_cast<uint32_t>(v), 1);
  const uint32_t hi = __shfl_up_sync(kFull, static_cast<uint32_t>(v >> 32), 1);
  return (static_cast<uint64_t>(hi) << 32) | lo;
}
__device__ __forceinline__ uint64_t shfl_down(uint64_t v) {
  const uint32_t lo = __shfl_down_sync(kFull, static_cast<uint32_t>(v), 1);
  const uint32_t hi = __shfl_down_sync(kFull, static_cast<uint32_t>(v >> 32), 1);
  return (static_cast<uint64_t>(hi) << 32) | lo;
}

// Horizontal sums of width 2R+1 over the lane's 8 columns, given the lane's
// own vertical sums v[0..8) and the neighbouring lanes' by shuffle. The edge
// lanes see no neighbour; their edge columns are halo and never used.
template <int R, typename A>
__device__ __forceinline__ void hsum(const A (&v)[8], A (&h)[8]) {
  A e[8 + 2 * R];
#pragma unroll
  for (int i = 0; i < R; i++)
    e[i] = shfl_up(v[8 - R + i]);
#pragma unroll
  for (int i = 0; i < 8; i++)
    e[R + i] = v[i];
#pragma unroll
  for (int i = 0; i < R; i++)
    e[R + 8 + i] = shfl_down(v[i]);
  A run = 0;
#pragma unroll
  for (int i = 0; i < 2 * R + 1; i++)
    run += e[i];
  h[0] = run;
#pragma unroll
  for (int k = 1; k < 8; k++) {
    run += e[k + 2 * R] - e[k - 1];
    h[k] = run;
  }
}

// --------------------------------------------------------------------------
// The kernel
// --------------------------------------------------------------------------

struct ThresholdArgs {
  const FrameDesc *frames;
  int32_t nframes;
  uint32_t ntasks;
  uint32_t *tile_count; // zeroed before the launch
  uint32_t *tile_start;
  SignalPixel *pool;
  uint32_t *pool_next;
  uint32_t pool_cap; // records
  int *status;
  uint32_t wait_limit;
};

__device__ __forceinline__ int find_frame(const FrameDesc *frames, int n,
                                          uint32_t task) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (frames[mid].task_begin <= task)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Ring slot of the row `back` rows above the row in slot `slot`.
__device__ __forceinline__ int back_slot(int slot, int back) {
  const int s = slot - back;
  return s < 0 ? s + kRingRows : s;
}

// Warps per SM the registers allow: 16 for 16-bit pixels, 8 for 32-bit
// (whose ring and 11-row sums, 24 KB a warp, also fill the shared memory;
// 16-bit pixels take 12.1 KB a warp).
template <typename T> constexpr int kWarpsPerSm = sizeof(T) == 2 ? 16 : 8;

// The rows before a task's first are read as zeros: 16 rows, the farthest
// back any row's sums reach (the 11-row window's leaving row, 16 above).
constexpr int kPreRows = 16;
// A pair of rows r, r+1 reads rows r-16 .. r+1 while the next box is in
// flight; the first two boxes do not land on the zero rows.
static_assert(kRingRows >= kPreRows + 2 + kBoxRows, "ring too short");
static_assert(kRingRows - kPreRows >= 2 * kBoxRows, "prologue boxes overlap the zero rows");
static_assert(kBoxRows % 2 == 0 && kRingRows % kBoxRows == 0, "rows go in pairs");

// Per-warp shared memory (the square-root table is static).
template <typename T> struct WarpSmem {
  using A = typename Traits<T>::Acc;
  static constexpr uint32_t kRing = kStripCols * sizeof(T) * kRingRows;
  static constexpr uint32_t kWin = 2 * kStripCols * sizeof(A);
  static constexpr uint32_t kBars = kRingStages * sizeof(uint64_t);
  static constexpr uint32_t kTotal = kRing + kWin + kBars;
};

template <typename T, int WPC>
__global__ void __launch_bounds__(WPC * 32, (kWarpsPerSm<T> / WPC) > 0 ? kWarpsPerSm<T> / WPC : 1)
    threshold_kernel(const __grid_constant__ CUtensorMap arena, ThresholdArgs args) {
  using Tr = Traits<T>;
  using A = typename Tr::Acc;
  using Rl = typename Real<T>::type;
  using Sm = WarpSmem<T>;
  constexpr uint32_t kRowBytes = kStripCols * sizeof(T);
  constexpr uint32_t kBoxBytes = kRowBytes * kBoxRows;
  constexpr A C7 = A(1) << Tr::kShift7;   // one valid pixel's count in a 7 x 7 sum
  constexpr A C11 = A(1) << Tr::kShift11; // ... in an 11 x 11 sum
  constexpr int kVecs = kStripCols * sizeof(T) / (32 * 16); // 16-byte words per lane per row

  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ Rl sqrt_tab[64];
  // for each 8-bit mask, the positions of its set bits in ascending order,
  // four bits each
  __shared__ uint32_t bit_pos[256];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  unsigned char *at = smem_raw;
  T *ring = reinterpret_cast<T *>(at + warp * Sm::kRing);
  at += WPC * Sm::kRing;
  A *win = reinterpret_cast<A *>(at + warp * Sm::kWin);
  at += WPC * Sm::kWin;
  uint64_t *bars = reinterpret_cast<uint64_t *>(at + warp * Sm::kBars);

  for (int m = threadIdx.x; m < 64; m += blockDim.x)
    sqrt_tab[m] = sqrt_term(m, Rl(0));
  for (int m = threadIdx.x; m < 256; m += blockDim.x) {
    uint32_t v = 0, n = 0;
    for (int k = 0; k < 8; k++)
      if ((m >> k) & 1) {
        v |= static_cast<uint32_t>(k) << (4 * n);
        n++;
      }
    bit_pos[m] = v;
  }
  if (lane == 0) {
    for (int s = 0; s < kRingStages; s++)
      mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const float sq49 = static_cast<float>(sqrt_tab[49]);

  uint32_t phase = 0; // bit s = parity of the next wait on stage s
  uint32_t chunk = kNoChunk, fill = 0;
  bool failed = false;

  const uint32_t gwarp = blockIdx.x * WPC + warp;
  const uint32_t nwarps = gridDim.x * WPC;

  for (uint32_t task = gwarp; task < args.ntasks && !failed; task += nwarps) {
    const int f = find_frame(args.frames, args.nframes, task);
    const FrameDesc fd = args.frames[f];
    const uint32_t local = task - fd.task_begin;
    const int strip = static_cast<int>(local % fd.strips);
    const int seg = static_cast<int>(local / fd.strips);
    const int r0 = seg * fd.seg_rows;
    const int r1 = min(r0 + fd.seg_rows, fd.height);
    const int rs = r0 - kHalo;       // first input row (frame coordinates)
    const int nrows = (r1 - r0) + 2 * kHalo;
    const int nboxes = (nrows + kBoxRows - 1) / kBoxRows;
    const int nrows2 = (nrows + 1) & ~1; // rows are taken in pairs
    const int32_t tma_x = strip * kStripOut;
    const int64_t tma_y0 = fd.row0 + rs;

    // Output columns of this lane: ring columns [10, 242) inside the frame.
    uint32_t outmask = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int j = 8 * lane + k;
      const int col = strip * kStripOut + j - kHalo;
      if (j >= kHalo && j < kHalo + kStripOut && col < fd.width)
        outmask |= 1u << k;
    }

    // The kPreRows rows above the task read as valid zeros, and every
    // running sum and history starts as if they had been processed (7 and
    // 11 valid zeros per column; nothing masked, dispersed, kept or a
    // candidate), so the row body needs no warm-up branches. What those rows
    // feed is flushed out before any output row reads it: an output row's
    // windows reach 10 rows up, and the first output row is the task's
    // 11th. They live in the ring slots of rows -16 .. -1, which no TMA box
    // writes before they are last read.
#pragma unroll 1
    for (int i = 0; i < kPreRows; i++) {
      uint4 *row = reinterpret_cast<uint4 *>(ring + (kRingRows - kPreRows + i) * kStripCols);
#pragma unroll
      for (int v = 0; v < kVecs; v++)
        row[kVecs * lane + v] = make_uint4(0, 0, 0, 0);
    }
    fence_proxy_async_smem(); // these writes before any later TMA write of the slots
    __syncwarp();

    // Prologue: the first two boxes.
    if (lane == 0) {
      for (int b = 0; b < 2 && b < nboxes; b++) {
        const int st = b % kRingStages;
        mbar_expect_tx(&bars[st], kBoxBytes);
        tma_load_2d(ring + st * kBoxRows * kStripCols, &arena, &bars[st], tma_x,
                    static_cast<int32_t>(tma_y0 + b * kBoxRows));
      }
    }

    A vs[8], vq[8], vg[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      vs[k] = 7 * C7;
      vq[k] = 0;
      vg[k] = 11 * C11;
    }
    // Histories, newest row in the low byte (bit), as they stand before the
    // pair of rows r, r+1 enters:
    uint64_t hist_mk = 0;   // masked bits of rows r-1 .. r-8
    uint32_t hist_s0 = 0;   // dispersion bits of rows r-4 .. r-7
    uint64_t gv_lo = ~0ull; // valid-and-not-kept bits of rows r-6 .. r-13
    uint32_t gv_hi = ~0u;   //   rows r-14 .. r-17
    uint64_t hist_cs = 0;   // candidate bits of rows r-6 .. r-13
    uint32_t dirty = 0;     // warp-uniform: bit i = row r-1-i holds a masked pixel
    uint32_t gdirty = 0;    // warp-uniform: bit i = row r-6-i holds a non-g pixel

    auto row_at = [&](int slot) { return ring + slot * kStripCols; };

    // Rows r = rr and r+1 of the task (ring slots `slot`, slot+1) enter.
    // Row r's sums are completed before row r+1's; the stages of the two
    // rows are otherwise independent, which gives the scheduler two rows of
    // work to interleave.
    auto process_pair = [&](int rr, int slot) {
      // ---- loads, masks, and the pair's warp-wide flags -----------------
      LaneRow<T> nA, nB, lA, lB;
      nA.load(row_at(slot), lane);
      nB.load(row_at(slot + 1), lane);
      lA.load(row_at(back_slot(slot, 7)), lane);
      lB.load(row_at(back_slot(slot, 6)), lane);
      // candidates: rows c = r-10 and c+1, when they are output rows
      const bool emitA = rr >= 2 * kHalo && rr < nrows;
      const bool emitB = rr + 1 >= 2 * kHalo && rr + 1 < nrows;
      const uint32_t csA = static_cast<uint32_t>(hist_cs >> 32) & (emitA ? outmask : 0u);
      const uint32_t csB = static_cast<uint32_t>(hist_cs >> 24) & (emitB ? outmask : 0u);
      const uint32_t flags = __reduce_or_sync(
          kFull, (nA.any_masked() ? 1u : 0u) | (nB.any_masked() ? 2u : 0u) |
                     ((csA | csB) ? 4u : 0u));
      uint32_t mkA = 0, mkB = 0;
      if (flags & 3u) {
        mkA = nA.masked_bits();
        mkB = nB.masked_bits();
      }

      // ---- 7-row sums: + rows r, r+1, - rows r-7, r-6 ------------------
      uint32_t p[8], q[8];
      A vsA[8], vqA[8];
      nA.unpack(p);
      lA.unpack(q);
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const A d = static_cast<A>(p[k]) - static_cast<A>(q[k]);
        vsA[k] = vs[k] + d;
        vqA[k] = vq[k] + d * (static_cast<A>(p[k]) + static_cast<A>(q[k]));
      }
      if ((flags & 1u) | (dirty & 0x40u)) {
        const uint32_t mk7 = static_cast<uint32_t>(hist_mk >> 48) & 0xffu; // row r-7
        if (mkA | mk7) {
#pragma unroll
          for (int k = 0; k < 8; k++) {
            if ((mkA >> k) & 1u) {
              vsA[k] -= static_cast<A>(p[k]) + C7;
              vqA[k] -= static_cast<A>(p[k]) * static_cast<A>(p[k]);
            }
            if ((mk7 >> k) & 1u) {
              vsA[k] += static_cast<A>(q[k]) + C7;
              vqA[k] += static_cast<A>(q[k]) * static_cast<A>(q[k]);
            }
          }
        }
      }
      nB.unpack(p);
      lB.unpack(q);
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const A d = static_cast<A>(p[k]) - static_cast<A>(q[k]);
        vs[k] = vsA[k] + d;
        vq[k] = vqA[k] + d * (static_cast<A>(p[k]) + static_cast<A>(q[k]));
      }
      if ((flags & 2u) | (dirty & 0x20u)) {
        const uint32_t mk6 = static_cast<uint32_t>(hist_mk >> 40) & 0xffu; // row r-6
        if (mkB | mk6) {
#pragma unroll
          for (int k = 0; k < 8; k++) {
            if ((mkB >> k) & 1u) {
              vs[k] -= static_cast<A>(p[k]) + C7;
              vq[k] -= static_cast<A>(p[k]) * static_cast<A>(p[k]);
            }
            if ((mk6 >> k) & 1u) {
              vs[k] += static_cast<A>(q[k]) + C7;
              vq[k] += static_cast<A>(q[k]) * static_cast<A>(q[k]);
            }
          }
        }
      }

      // ---- dispersion test at rows a = r-3 and a+1 ---------------------
      // row a's window is rows r-6 .. r, row a+1's r-5 .. r+1
      const bool wdA = ((dirty & 0x3fu) | (flags & 1u)) != 0;
      const bool wdB = ((dirty & 0x1fu) | (flags & 3u)) != 0;
      uint32_t s0A, s0B;
      {
        A hs[8], hq[8];
        hsum<3>(vsA, hs);
        hsum<3>(vqA, hq);
        if constexpr (sizeof(T) == 2)
          s0A = wdA ? dispersion_bits(hs, hq, sqrt_tab) : dispersion_bits49(hs, hq, sq49);
        else
          s0A = dispersion_bits(hs, hq, sqrt_tab);
      }
      {
        A hs[8], hq[8];
        hsum<3>(vs, hs);
        hsum<3>(vq, hq);
        if constexpr (sizeof(T) == 2)
          s0B = wdB ? dispersion_bits(hs, hq, sqrt_tab) : dispersion_bits49(hs, hq, sq49);
        else
          s0B = dispersion_bits(hs, hq, sqrt_tab);
      }
      s0A |= static_cast<uint32_t>(hist_mk >> 16) & 0xffu; // masked -> 1 (row r-3)
      s0B |= static_cast<uint32_t>(hist_mk >> 8) & 0xffu;  // row r-2

      // ---- erode at rows b = r-5 and b+1 -------------------------------
      // row b: dispersion rows r-7 .. r-3; row b+1: r-6 .. r-2. Both rows'
      // bits travel in one word (row b in bits 0-7, b+1 in 16-23).
      const uint32_t vA = s0A & hist_s0 & (hist_s0 >> 8) & (hist_s0 >> 16) & (hist_s0 >> 24);
      const uint32_t vB = s0B & s0A & hist_s0 & (hist_s0 >> 8) & (hist_s0 >> 16);
      hist_s0 = (hist_s0 << 16) | (s0A << 8) | s0B;
      const uint32_t v2 = (vA & 0xffu) | ((vB & 0xffu) << 16);
      const uint32_t vl = shfl_up(v2), vr = shfl_down(v2);
      const uint32_t w2 = ((vl >> 6) & 0x00030003u) | (v2 << 2) | ((vr << 10) & 0x0c000c00u);
      const uint32_t hv2 = w2 & (w2 >> 1) & (w2 >> 2) & (w2 >> 3) & (w2 >> 4) & 0x00ff00ffu;
      const uint32_t mkb2 = (static_cast<uint32_t>(hist_mk >> 32) & 0xffu) |      // row r-5
                            ((static_cast<uint32_t>(hist_mk >> 24) & 0xffu) << 16); // r-4
      const uint32_t s1 = hv2 | mkb2;                 // scr1, src/dext.cc:117-142
      const uint32_t gv2 = ~s1 & 0x00ff00ffu;         // valid and not kept
      const uint32_t cs2 = s1 & ~mkb2 & 0x00ff00ffu;  // kept and not masked
      const uint32_t gvA = gv2 & 0xffu, gvB = gv2 >> 16;
      const uint32_t gflags =
          __reduce_or_sync(kFull, (gvA != 0xffu ? 1u : 0u) | (gvB != 0xffu ? 2u : 0u));

      // ---- 11-row sums at rows b, b+1: + rows r-5, r-4, - rows r-16, r-15
      const uint32_t ng16 = ~(gv_hi >> 16) & 0xffu; // row r-16
      const uint32_t ng15 = ~(gv_hi >> 8) & 0xffu;  // row r-15
      load_pixels<T>(row_at(back_slot(slot, 5)), lane, p);
      load_pixels<T>(row_at(back_slot(slot, 16)), lane, q);
#pragma unroll
      for (int k = 0; k < 8; k++)
        vg[k] += static_cast<A>(p[k]) - static_cast<A>(q[k]);
      if ((gflags & 1u) | ((gdirty >> 10) & 1u)) {
        const uint32_t ng5 = ~gvA & 0xffu;
        if (ng5 | ng16) {
#pragma unroll
          for (int k = 0; k < 8; k++) {
            if ((ng5 >> k) & 1u)
              vg[k] -= static_cast<A>(p[k]) + C11;
            if ((ng16 >> k) & 1u)
              vg[k] += static_cast<A>(q[k]) + C11;
          }
        }
      }
      A vgA[8];
#pragma unroll
      for (int k = 0; k < 8; k++)
        vgA[k] = vg[k];
      load_pixels<T>(row_at(back_slot(slot, 4)), lane, p);
      load_pixels<T>(row_at(back_slot(slot, 15)), lane, q);
#pragma unroll
      for (int k = 0; k < 8; k++)
        vg[k] += static_cast<A>(p[k]) - static_cast<A>(q[k]);
      if ((gflags & 2u) | ((gdirty >> 9) & 1u)) {
        const uint32_t ng4 = ~gvB & 0xffu;
        if (ng4 | ng15) {
#pragma unroll
          for (int k = 0; k < 8; k++) {
            if ((ng4 >> k) & 1u)
              vg[k] -= static_cast<A>(p[k]) + C11;
            if ((ng15 >> k) & 1u)
              vg[k] += static_cast<A>(q[k]) + C11;
          }
        }
      }

      // ---- histories -----------------------------------------------------
      gv_hi = (gv_hi << 16) | static_cast<uint32_t>(gv_lo >> 48);
      gv_lo = (gv_lo << 16) | (gvA << 8) | gvB;
      hist_cs = (hist_cs << 16) | ((cs2 & 0xffu) << 8) | (cs2 >> 16);
      hist_mk = (hist_mk << 16) | (mkA << 8) | mkB;
      dirty = (dirty << 2) | ((flags & 1u) << 1) | ((flags >> 1) & 1u);
      gdirty = (gdirty << 2) | ((gflags & 1u) << 1) | ((gflags >> 1) & 1u);

      // ---- Poisson test and emit at rows c = r-10 and c+1 ---------------
      if (flags & 4u) {
        // The 11-row sums of both rows, for the candidates' 11-column
        // windows; then the candidates of both rows taken one per lane
        // (row c's first, each row's in column order), so that each pays
        // for one division and one square root: a prefix count over the
        // lanes, and each lane finds its candidate by itself.
        if constexpr (sizeof(A) == 4) {
          uint4 *w0 = reinterpret_cast<uint4 *>(win + 8 * lane);
          uint4 *w1 = reinterpret_cast<uint4 *>(win + kStripCols + 8 * lane);
          w0[0] = make_uint4(vgA[0], vgA[1], vgA[2], vgA[3]);
          w0[1] = make_uint4(vgA[4], vgA[5], vgA[6], vgA[7]);
          w1[0] = make_uint4(vg[0], vg[1], vg[2], vg[3]);
          w1[1] = make_uint4(vg[4], vg[5], vg[6], vg[7]);
        } else {
#pragma unroll
          for (int k = 0; k < 8; k++) {
            win[8 * lane + k] = vgA[k];
            win[kStripCols + 8 * lane + k] = vg[k];
          }
        }
        const uint32_t cntA = __popc(csA), cntB = __popc(csB);
        uint32_t incl = cntA | (cntB << 16); // two counts of at most 256
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const uint32_t t = __shfl_up_sync(kFull, incl, d);
          if (lane >= d)
            incl += t;
        }
        const uint32_t tot = __shfl_sync(kFull, incl, 31);
        const uint32_t totA = tot & 0xffffu, total = totA + (tot >> 16);
        const uint32_t excl = incl - (cntA | (cntB << 16));
        const uint32_t posA = bit_pos[csA], posB = bit_pos[csB];

        // Room for both rows' candidates in one chunk, so each tile's
        // records are contiguous whatever the rounds below find.
        if (chunk == kNoChunk || fill + total > kChunkRecords) {
          uint32_t base = 0;
          if (lane == 0)
            base = atomicAdd(args.pool_next, kChunkRecords);
          base = __shfl_sync(kFull, base, 0);
          if (base > args.pool_cap - kChunkRecords || base + kChunkRecords < base) {
            if (lane == 0)
              atomicCAS(args.status, kStatusOk, kStatusPoolExhausted);
            chunk = kNoChunk;
          } else {
            chunk = base;
          }
          fill = 0;
        }
        const uint32_t start = chunk + fill;
        const int c = rs + rr - kHalo; // frame row of row c
        const uint32_t index0 = static_cast<uint32_t>(c) * static_cast<uint32_t>(fd.width) +
                                static_cast<uint32_t>(strip * kStripOut - kHalo);
        uint32_t foundA = 0, foundB = 0;
        for (uint32_t base = 0; base < total; base += 32) {
          const uint32_t i = base + lane;
          // Candidate i (row c's in column order, then row c+1's): the lane
          // L holding it is the first whose inclusive count for the row
          // exceeds its rank t in the row, found by a binary search over
          // the lanes' counts; then the (t - exclusive count)-th set bit of
          // L's mask.
          const bool rowB = i >= totA;
          const uint32_t t = rowB ? i - totA : i;
          const uint32_t sh = rowB ? 16u : 0u;
          uint32_t L = 0;
#pragma unroll
          for (uint32_t step = 16; step > 0; step >>= 1) {
            const uint32_t v = __shfl_sync(kFull, incl, static_cast<int>(L + step - 1));
            if (((v >> sh) & 0xffffu) <= t)
              L += step;
          }
          const uint32_t exL = __shfl_sync(kFull, excl, static_cast<int>(L));
          const uint32_t pA = __shfl_sync(kFull, posA, static_cast<int>(L));
          const uint32_t pB = __shfl_sync(kFull, posB, static_cast<int>(L));
          const uint32_t pL = rowB ? pB : pA;
          bool sig = false;
          SignalPixel px;
          if (i < total) {
            const uint32_t j = t - ((exL >> sh) & 0xffffu);
            const uint32_t col = 8 * L + ((pL >> (4 * j)) & 0xfu); // an output column
            const T *prow = row_at(back_slot(slot, rowB ? 9 : 10));
            const A *w = win + (rowB ? kStripCols : 0);
            const uint32_t pv = prow[col];
            A h = 0;
#pragma unroll
            for (int d = -kRadius11; d <= kRadius11; d++)
              h += w[col + d];
            if (pv > 0) { // a masked pixel is never a candidate
              sig = poisson(pv, h >> Tr::kShift11, h & (C11 - 1), &px.background);
              px.index = index0 + (rowB ? static_cast<uint32_t>(fd.width) : 0u) + col;
              px.value = pv;
              px.population = static_cast<uint16_t>(h >> Tr::kShift11);
              px.reserved = 0;
            }
          }
          const uint32_t ball = __ballot_sync(kFull, sig);
          if (sig && chunk != kNoChunk)
            args.pool[start + foundA + foundB + __popc(ball & ((1u << lane) - 1u))] = px;
          // the lanes holding row c's candidates: i < totA
          const uint32_t na = totA > base ? totA - base : 0u;
          const uint32_t rowA_lanes = na >= 32 ? kFull : (1u << na) - 1u;
          foundA += __popc(ball & rowA_lanes);
          foundB += __popc(ball & ~rowA_lanes);
        }
        if (lane == 0) {
          const uint64_t tile = fd.tile_base + static_cast<uint64_t>(c) * fd.strips + strip;
          // counted even if the records were dropped
          if (foundA > 0) {
            args.tile_count[tile] = foundA;
            args.tile_start[tile] = chunk == kNoChunk ? 0u : start;
          }
          if (foundB > 0) {
            args.tile_count[tile + fd.strips] = foundB;
            args.tile_start[tile + fd.strips] = chunk == kNoChunk ? 0u : start + foundA;
          }
        }
        fill += foundA + foundB;
        __syncwarp();
      }
    };

    for (int b = 0; b < nboxes && !failed; b++) {
      const int st = b % kRingStages;
      if (lane == 0 && b >= 1 && b + 1 < nboxes) {
        // Box b+1 reuses the stage of box b+1-kRingStages, whose rows are
        // all older than r-16 for every row of box b: free.
        const int nst = (b + 1) % kRingStages;
        fence_proxy_async_smem();
        mbar_expect_tx(&bars[nst], kBoxBytes);
        tma_load_2d(ring + nst * kBoxRows * kStripCols, &arena, &bars[nst], tma_x,
                    static_cast<int32_t>(tma_y0 + (b + 1) * kBoxRows));
      }
      const bool ok = mbar_wait_bounded(&bars[st], (phase >> st) & 1u, args.wait_limit);
      phase ^= 1u << st;
      if (!__all_sync(kFull, ok)) {
        if (lane == 0)
          atomicCAS(args.status, kStatusOk, kStatusTmaTimeout);
        failed = true;
        break;
      }

      // Rows in pairs; an odd last row is paired with the arena row after it
      // (its box holds it), whose results go nowhere.
      const int rr0 = b * kBoxRows;
      const int slot0 = st * kBoxRows;
      const int rend = min(kBoxRows, nrows2 - rr0);
#pragma unroll 1
      for (int i = 0; i < rend; i += 2)
        process_pair(rr0 + i, slot0 + i);
      __syncwarp();
    }
    if (failed) {
      // Let any copy still in flight land before this warp's shared memory
      // is released; bounded, like every wait here.
      for (int s = 0; s < kRingStages; s++)
        mbar_wait_bounded(&bars[s], (phase >> s) & 1u, args.wait_limit);
    }
  }
}

} // namespace

// --------------------------------------------------------------------------
// Host side
// --------------------------------------------------------------------------

template <typename T>
size_t threshold_smem_bytes(int wpc) {
  return static_cast<size_t>(wpc) * WarpSmem<T>::kTotal;
}

template <typename T, int WPC>
static cudaError_t launch_wpc(const CUtensorMap &map, const ThresholdLaunch &L,
                              cudaStream_t stream) {
  const size_t smem = threshold_smem_bytes<T>(WPC);
  static bool configured = false; // per instantiation; setting it twice is harmless
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(threshold_kernel<T, WPC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess)
      return e;
    configured = true;
  }
  ThresholdArgs a;
  a.frames = L.frames;
  a.nframes = L.nframes;
  a.ntasks = L.ntasks;
  a.tile_count = L.tile_count;
  a.tile_start = L.tile_start;
  a.pool = L.pool;
  a.pool_next = L.pool_next;
  a.pool_cap = L.pool_cap;
  a.status = L.status;
  a.wait_limit = L.wait_limit;
  uint32_t blocks = (L.ntasks + WPC - 1) / WPC;
  if (L.max_blocks > 0 && blocks > static_cast<uint32_t>(L.max_blocks))
    blocks = static_cast<uint32_t>(L.max_blocks);
  if (blocks == 0)
    return cudaSuccess;
  threshold_kernel<T, WPC><<<blocks, WPC * 32, smem, stream>>>(map, a);
  return cudaGetLastError();
}

template <typename T, int WPC> static int occupancy_wpc() {
  const size_t smem = threshold_smem_bytes<T>(WPC);
  if (cudaFuncSetAttribute(threshold_kernel<T, WPC>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) != cudaSuccess)
    return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, threshold_kernel<T, WPC>, WPC * 32,
                                                    smem) != cudaSuccess)
    return 0;
  return n;
}

template <typename T> int threshold_occupancy(int wpc) {
  switch (wpc) {
  case 1: return occupancy_wpc<T, 1>();
  case 2: return occupancy_wpc<T, 2>();
  case 4: return occupancy_wpc<T, 4>();
  default: return 0;
  }
}

template <typename T>
cudaError_t launch_threshold(const CUtensorMap &map, const ThresholdLaunch &L,
                             cudaStream_t stream) {
  switch (L.warps_per_block) {
  case 1: return launch_wpc<T, 1>(map, L, stream);
  case 2: return launch_wpc<T, 2>(map, L, stream);
  case 4: return launch_wpc<T, 4>(map, L, stream);
  default: return cudaErrorInvalidValue;
  }
}

template cudaError_t launch_threshold<uint16_t>(const CUtensorMap &, const ThresholdLaunch &,
                                                cudaStream_t);
template cudaError_t launch_threshold<uint32_t>(const CUtensorMap &, const ThresholdLaunch &,
                                                cudaStream_t);
template size_t threshold_smem_bytes<uint16_t>(int);
template size_t threshold_smem_bytes<uint32_t>(int);
template int threshold_occupancy<uint16_t>(int);
template int threshold_occupancy<uint32_t>(int);

} // namespace sf
