// Ordered compaction of the threshold's staged records into per-frame lists
// ascending by pixel index. This replaces the reference's host-side sort of
// the device emit (src/signal_order.cc:19-72 called from
// src/dext_cuda.cu:718-720): the tiles are already in index order, so an
// exclusive scan of their counts places every record directly.
//
// Three launches, none of which waits on another block:
//   place_reduce  per-block sums of kPlaceTiles tile counts
//   place_scan    one block: exclusive scan of the block sums, and each
//                 frame's starting offset and signal count
//   place_copy    per-block scan of its tiles, then a record-parallel copy:
//                 the block's records are one contiguous run of the output
//                 (within a frame), so thread k copies record k after a
//                 binary search for its tile in shared memory

#include "sf_host.hh"

namespace sf {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, v, d);
    if (lane >= d)
      v += t;
  }
  return v;
}

// Exclusive scan of one value per thread across the block; returns the
// thread's prefix and writes the block total to *total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *total) {
  __shared__ uint32_t warp_sums[kPlaceThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t incl = warp_incl_scan(v, lane);
  if (lane == 31)
    warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kPlaceThreads / 32 ? warp_sums[lane] : 0u;
    w = warp_incl_scan(w, lane);
    if (lane < kPlaceThreads / 32)
      warp_sums[lane] = w;
  }
  __syncthreads();
  const uint32_t before = warp == 0 ? 0u : warp_sums[warp - 1];
  *total = warp_sums[kPlaceThreads / 32 - 1];
  __syncthreads();
  return before + incl - v;
}

__global__ void __launch_bounds__(kPlaceThreads)
    place_reduce(const uint32_t *counts, uint64_t ntiles, uint32_t *block_sums) {
  const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kPlaceTiles +
                        static_cast<uint64_t>(threadIdx.x) * kPlaceItems;
  uint32_t sum = 0;
#pragma unroll
  for (int i = 0; i < kPlaceItems; i++)
    if (base + i < ntiles)
      sum += counts[base + i];
  uint32_t total;
  block_excl_scan(sum, &total);
  if (threadIdx.x == 0)
    block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kPlaceThreads)
    place_scan(uint32_t *block_sums, uint32_t nblocks, const uint32_t *counts,
               const FrameDesc *frames, int nframes, uint32_t *frame_prefix,
               uint32_t *frame_count) {
  // Exclusive scan of the block sums, kPlaceThreads at a time.
  __shared__ uint32_t carry_s;
  if (threadIdx.x == 0)
    carry_s = 0;
  __syncthreads();
  for (uint32_t at = 0; at < nblocks; at += kPlaceThreads) {
    const uint32_t i = at + threadIdx.x;
    const uint32_t v = i < nblocks ? block_sums[i] : 0u;
    uint32_t total;
    const uint32_t ex = block_excl_scan(v, &total);
    const uint32_t carry = carry_s;
    if (i < nblocks)
      block_sums[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0)
      carry_s = carry + total;
    __syncthreads();
  }
  const uint32_t grand = carry_s;

  // Each frame's first tile lies inside some block; its prefix is that
  // block's prefix plus the counts in the block before it. A warp per frame,
  // so the frames' reads overlap.
  const int lane = threadIdx.x & 31;
  for (int f = threadIdx.x >> 5; f < nframes; f += kPlaceThreads / 32) {
    const uint64_t t0 = frames[f].tile_base;
    const uint64_t blk = t0 / kPlaceTiles;
    const uint64_t from = blk * kPlaceTiles;
    uint32_t part = 0;
#pragma unroll 4
    for (uint64_t t = from + lane; t < t0; t += 32)
      part += counts[t];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1)
      part += __shfl_xor_sync(kFull, part, d);
    if (lane == 0)
      frame_prefix[f] = (blk < nblocks ? block_sums[blk] : grand) + part;
  }
  __syncthreads();
  if (threadIdx.x == 0)
    frame_prefix[nframes] = grand;
  __syncthreads();
  for (int f = threadIdx.x; f < nframes; f += kPlaceThreads)
    frame_count[f] = frame_prefix[f + 1] - frame_prefix[f];
}

__device__ __forceinline__ int frame_of_tile(const FrameDesc *frames, int n, uint64_t tile) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (frames[mid].tile_base <= tile)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(kPlaceThreads)
    place_copy(const uint32_t *counts, const uint32_t *starts, uint64_t ntiles,
               const uint32_t *block_sums, const FrameDesc *frames, int nframes,
               const uint32_t *frame_prefix, const SignalPixel *pool,
               SignalPixel *out) {
  __shared__ uint32_t off[kPlaceTiles]; // exclusive prefix of counts within the block
  __shared__ uint32_t src[kPlaceTiles]; // pool index of the tile's first record
  __shared__ uint32_t dst[kPlaceTiles]; // output index of the tile's first record
  __shared__ uint32_t lim[kPlaceTiles]; // records of the tile that fit its frame's list
  const uint64_t block_base = static_cast<uint64_t>(blockIdx.x) * kPlaceTiles;
  const uint64_t base = block_base + static_cast<uint64_t>(threadIdx.x) * kPlaceItems;
  uint32_t c[kPlaceItems];
  uint32_t sum = 0;
#pragma unroll
  for (int i = 0; i < kPlaceItems; i++) {
    c[i] = base + i < ntiles ? counts[base + i] : 0u;
    sum += c[i];
  }
  uint32_t total;
  uint32_t run = block_excl_scan(sum, &total);
  const uint32_t block_prefix = block_sums[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kPlaceItems; i++) {
    const int t = threadIdx.x * kPlaceItems + i;
    off[t] = run;
    if (c[i] != 0) {
      const uint64_t tile = base + i;
      const int f = frame_of_tile(frames, nframes, tile);
      const uint32_t at = block_prefix + run - frame_prefix[f]; // position in frame f's list
      const uint32_t cap = frames[f].capacity;
      src[t] = starts[tile];
      dst[t] = static_cast<uint32_t>(frames[f].out_base) + at;
      lim[t] = at >= cap ? 0u : min(c[i], cap - at);
    } else {
      lim[t] = 0;
    }
    run += c[i];
  }
  __syncthreads();

  for (uint32_t k = threadIdx.x; k < total; k += kPlaceThreads) {
    // The tile holding record k: the last t with off[t] <= k.
    int lo = 0, hi = kPlaceTiles - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (off[mid] <= k)
        lo = mid;
      else
        hi = mid - 1;
    }
    const uint32_t j = k - off[lo];
    if (j < lim[lo]) {
      const uint4 v = reinterpret_cast<const uint4 *>(pool)[src[lo] + j];
      reinterpret_cast<uint4 *>(out)[dst[lo] + j] = v;
    }
  }
}

} // namespace

cudaError_t launch_place(const PlaceLaunch &L, cudaStream_t stream) {
  const uint32_t nblocks = static_cast<uint32_t>((L.ntiles + kPlaceTiles - 1) / kPlaceTiles);
  if (nblocks == 0)
    return cudaSuccess;
  place_reduce<<<nblocks, kPlaceThreads, 0, stream>>>(L.tile_count, L.ntiles, L.block_sums);
  place_scan<<<1, kPlaceThreads, 0, stream>>>(L.block_sums, nblocks, L.tile_count, L.frames,
                                               L.nframes, L.frame_prefix, L.frame_count);
  place_copy<<<nblocks, kPlaceThreads, 0, stream>>>(L.tile_count, L.tile_start, L.ntiles,
                                                     L.block_sums, L.frames, L.nframes,
                                                     L.frame_prefix, L.pool, L.out);
  return cudaGetLastError();
}

} // namespace sf
