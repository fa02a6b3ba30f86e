// Exclusive prefix sums over device arrays whose length is itself in device
// memory, so that a pipeline of kernels can be enqueued (or captured in a
// CUDA graph) without reading sizes back to the host. Three launches, no
// inter-block waiting:
//   scan_reduce  per-tile sums of kScanTile elements
//   scan_blocks  one block: exclusive scan of the tile sums, and the total
//   scan_down    per-tile scan plus the tile's prefix
// The launches have one block per SM, which take the tiles up to the
// device-side length in turn: a grid sized for the largest length the
// caller allows would spend most of its time starting blocks that find
// nothing to do (the lengths run far below their bounds).

#include "sf_scan.cuh"

namespace sf {
namespace {

constexpr unsigned kFull = 0xffffffffu;

template <typename V> __device__ __forceinline__ V warp_incl(V v, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const V t = __shfl_up_sync(kFull, v, d);
    if (lane >= d)
      v += t;
  }
  return v;
}

// Exclusive scan of one value per thread over the block; *total gets the sum.
template <typename V> __device__ __forceinline__ V block_excl(V v, V *total) {
  __shared__ V sums[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const V incl = warp_incl(v, lane);
  if (lane == 31)
    sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    V w = lane < kScanThreads / 32 ? sums[lane] : V(0);
    w = warp_incl(w, lane);
    if (lane < kScanThreads / 32)
      sums[lane] = w;
  }
  __syncthreads();
  const V before = warp == 0 ? V(0) : sums[warp - 1];
  *total = sums[kScanThreads / 32 - 1];
  __syncthreads();
  return before + incl - v;
}

template <typename V>
__global__ void __launch_bounds__(kScanThreads)
    scan_reduce(const V *in, const uint64_t *len, uint64_t len_scale, V *block_sums) {
  const uint64_t n = *len * len_scale;
  const uint64_t ntiles = n == 0 ? 1 : (n + kScanTile - 1) / kScanTile;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint64_t base = t * kScanTile;
    V sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      const uint64_t at = base + static_cast<uint64_t>(i) * kScanThreads + threadIdx.x;
      if (at < n)
        sum += in[at];
    }
    V total;
    block_excl(sum, &total);
    if (threadIdx.x == 0)
      block_sums[t] = total;
  }
}

template <typename V>
__global__ void __launch_bounds__(kScanThreads)
    scan_blocks(V *block_sums, const uint64_t *len, uint64_t len_scale, V *total_out) {
  const uint64_t n = *len * len_scale;
  const uint64_t nblocks = n == 0 ? 1 : (n + kScanTile - 1) / kScanTile;
  __shared__ V carry_s;
  if (threadIdx.x == 0)
    carry_s = 0;
  __syncthreads();
  for (uint64_t at = 0; at < nblocks; at += kScanThreads) {
    const uint64_t i = at + threadIdx.x;
    const V v = i < nblocks ? block_sums[i] : V(0);
    V total;
    const V ex = block_excl(v, &total);
    const V carry = carry_s;
    if (i < nblocks)
      block_sums[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0)
      carry_s = carry + total;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total_out)
    *total_out = n == 0 ? V(0) : carry_s;
}

template <typename V>
__global__ void __launch_bounds__(kScanThreads)
    scan_down(const V *in, const uint64_t *len, uint64_t len_scale, const V *block_sums,
              V *out) {
  const uint64_t n = *len * len_scale;
  // Items are read strided (coalesced) and scanned per thread over a
  // transposed order: thread t owns items base + t*kScanItems + i.
  __shared__ V tile[kScanTile];
  for (uint64_t t = blockIdx.x; t * kScanTile < n; t += gridDim.x) {
    const uint64_t base = t * kScanTile;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      const uint64_t at = base + static_cast<uint64_t>(i) * kScanThreads + threadIdx.x;
      tile[i * kScanThreads + threadIdx.x] = at < n ? in[at] : V(0);
    }
    __syncthreads();
    V run = 0;
    V mine[kScanItems];
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      mine[i] = tile[threadIdx.x * kScanItems + i];
      run += mine[i];
    }
    V total;
    V pre = block_excl(run, &total) + block_sums[t];
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      tile[threadIdx.x * kScanItems + i] = pre;
      pre += mine[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      const uint64_t at = base + static_cast<uint64_t>(i) * kScanThreads + threadIdx.x;
      if (at < n)
        out[at] = tile[i * kScanThreads + threadIdx.x];
    }
    __syncthreads(); // the tile is refilled by the next turn
  }
}

} // namespace

template <typename V>
void DeviceScan<V>::reserve(uint64_t max_len) {
  const uint64_t blocks = max_len / kScanTile + 1;
  if (blocks <= max_blocks_)
    return;
  if (block_sums_)
    cudaFree(block_sums_);
  block_sums_ = nullptr;
  check(cudaMalloc(&block_sums_, blocks * sizeof(V)), "cudaMalloc scan workspace");
  max_blocks_ = blocks;
  if (!grid_cap_)
    grid_cap_ = static_cast<unsigned>(device_sm_count());
}

template <typename V> DeviceScan<V>::~DeviceScan() {
  if (block_sums_)
    cudaFree(block_sums_);
}

template <typename V>
void DeviceScan<V>::run(const V *in, V *out, const uint64_t *len, uint64_t len_scale,
                        uint64_t max_len, V *total, cudaStream_t s) {
  reserve(max_len);
  const unsigned grid =
      static_cast<unsigned>(std::min<uint64_t>(max_len / kScanTile + 1, grid_cap_));
  scan_reduce<V><<<grid, kScanThreads, 0, s>>>(in, len, len_scale, block_sums_);
  scan_blocks<V><<<1, kScanThreads, 0, s>>>(block_sums_, len, len_scale, total);
  scan_down<V><<<grid, kScanThreads, 0, s>>>(in, len, len_scale, block_sums_, out);
  check(cudaGetLastError(), "launching a scan");
}

template class DeviceScan<uint32_t>;
template class DeviceScan<uint64_t>;

} // namespace sf
