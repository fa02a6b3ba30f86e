// ThresholdPlan: the device buffers and launch geometry for thresholding one
// batch shape (one or many frames, equal or uneven sizes), built once and
// reused frame after frame. Also the TMA descriptor over the frame arena.

#include <algorithm>
#include <cstring>
#include <mutex>

#include "sf_host.hh"

namespace sf {

template <typename T> int threshold_occupancy(int wpc);

namespace {

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                 const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                 const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion,
                                 CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  if (fn == nullptr)
    throw DeviceError("cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

uint64_t round_up(uint64_t v, uint64_t m) { return (v + m - 1) / m * m; }

} // namespace

void encode_arena_map(CUtensorMap *map, void *base, int elem_bytes, uint64_t pitch_elems,
                      uint64_t rows) {
  const cuuint64_t dims[2] = {pitch_elems, rows};
  const cuuint64_t strides[1] = {pitch_elems * static_cast<uint64_t>(elem_bytes)};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(kStripCols),
                             static_cast<cuuint32_t>(kBoxRows)};
  const cuuint32_t estride[2] = {1, 1};
  const CUtensorMapDataType dt =
      elem_bytes == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT32;
  const CUresult r = encode_fn()(map, dt, 2, base, dims, strides, box, estride,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    throw DeviceError("cuTensorMapEncodeTiled failed with code " + std::to_string(r));
}

int device_sm_count() {
  int dev = 0, n = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  check(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev),
        "cudaDeviceGetAttribute");
  return n;
}

ThresholdPlan::ThresholdPlan(int elem_bytes, const std::vector<Shape> &shapes, int seg_rows,
                             int warps_per_block, int blocks_per_sm)
    : elem_bytes_(elem_bytes), shapes_(shapes), seg_rows_(seg_rows), wpc_(warps_per_block),
      blocks_per_sm_(blocks_per_sm) {
  if (elem_bytes != 2 && elem_bytes != 4)
    throw std::invalid_argument("pixels are 16 or 32 bits");
  if (shapes.empty())
    throw std::invalid_argument("a plan needs at least one frame");
  if (seg_rows < 1)
    throw std::invalid_argument("seg_rows must be positive");

  int32_t max_strips = 0;
  for (const Shape &s : shapes) {
    if (s.height < 1 || s.width < 1)
      throw std::invalid_argument("frame with no pixels");
    max_strips = std::max(max_strips, (s.width + kStripOut - 1) / kStripOut);
  }
  // Every strip reads 256 columns from a multiple of 232; the pitch is a
  // multiple of 128 bytes so each arena row starts on a TMA-friendly line.
  pitch_ = round_up(static_cast<uint64_t>(max_strips) * kStripOut + (kStripCols - kStripOut),
                    128 / elem_bytes);

  uint64_t row = 0, tile = 0, out = 0;
  uint32_t task = 0;
  for (const Shape &s : shapes) {
    FrameDesc d;
    std::memset(&d, 0, sizeof(d));
    d.row0 = static_cast<int64_t>(row + kMarginRows);
    d.height = s.height;
    d.width = s.width;
    d.strips = (s.width + kStripOut - 1) / kStripOut;
    d.seg_rows = std::min(seg_rows, s.height);
    d.segments = (s.height + d.seg_rows - 1) / d.seg_rows;
    d.task_begin = task;
    d.tile_base = tile;
    d.out_base = out;
    // The reference's list capacity: the frame's own bytes, 16 to an entry
    // (src/dext_cuda.cu:611-616), so -2 comes back on exactly the same frames.
    const uint64_t cap = static_cast<uint64_t>(s.height) * s.width * elem_bytes / 16;
    d.capacity = static_cast<uint32_t>(cap);
    host_frames_.push_back(d);
    row += static_cast<uint64_t>(s.height) + 2 * kMarginRows;
    tile += static_cast<uint64_t>(s.height) * d.strips;
    out += cap;
    task += static_cast<uint32_t>(d.strips * d.segments);
  }
  arena_rows_ = row;
  ntiles_ = tile;
  ntasks_ = task;
  total_capacity_ = out;

  const int occ = elem_bytes == 2 ? threshold_occupancy<uint16_t>(wpc_)
                                  : threshold_occupancy<uint32_t>(wpc_);
  if (occ < 1)
    throw DeviceError("the threshold kernel does not fit on this device");
  const int per_sm = blocks_per_sm_ > 0 ? std::min(blocks_per_sm_, occ) : occ;
  max_blocks_ = device_sm_count() * per_sm;
  const uint64_t blocks = std::min<uint64_t>((ntasks_ + wpc_ - 1) / wpc_, max_blocks_);
  const uint64_t warps = blocks * wpc_;

  const uint64_t chunks =
      (total_capacity_ + (kChunkRecords - kStripOut) - 1) / (kChunkRecords - kStripOut) +
      warps + 1;
  const uint64_t pool_records = chunks * kChunkRecords;
  if (pool_records >= 0xffffffffull - kChunkRecords)
    throw std::invalid_argument("batch too large for one plan");
  pool_cap_ = static_cast<uint32_t>(pool_records);

  const uint64_t arena_bytes = pitch_ * arena_rows_ * elem_bytes;
  const uint64_t nblocks = (ntiles_ + kPlaceTiles - 1) / kPlaceTiles;
  try {
    check(cudaMalloc(&arena_, arena_bytes), "cudaMalloc arena");
    check(cudaMemset(arena_, 0xff, arena_bytes), "filling the arena");
    check(cudaMalloc(&frames_, host_frames_.size() * sizeof(FrameDesc)), "cudaMalloc frames");
    check(cudaMemcpy(frames_, host_frames_.data(), host_frames_.size() * sizeof(FrameDesc),
                     cudaMemcpyHostToDevice),
          "uploading frame descriptors");
    check(cudaMalloc(&tile_count_, ntiles_ * sizeof(uint32_t)), "cudaMalloc tile counts");
    check(cudaMalloc(&tile_start_, ntiles_ * sizeof(uint32_t)), "cudaMalloc tile starts");
    check(cudaMalloc(&pool_, pool_records * sizeof(SignalPixel)), "cudaMalloc pool");
    check(cudaMalloc(&pool_next_, 2 * sizeof(uint32_t)), "cudaMalloc pool cursor");
    status_ = reinterpret_cast<int *>(pool_next_ + 1);
    check(cudaMalloc(&out_, std::max<uint64_t>(total_capacity_, 1) * sizeof(SignalPixel)),
          "cudaMalloc output lists");
    check(cudaMalloc(&block_sums_, std::max<uint64_t>(nblocks, 1) * sizeof(uint32_t)),
          "cudaMalloc block sums");
    check(cudaMalloc(&frame_prefix_, (host_frames_.size() + 1) * sizeof(uint32_t)),
          "cudaMalloc frame prefix");
    check(cudaMalloc(&frame_count_, host_frames_.size() * sizeof(uint32_t)),
          "cudaMalloc frame counts");
    encode_arena_map(&map_, arena_, elem_bytes_, pitch_, arena_rows_);
    // The fill above ran on the legacy stream; the plan's users work on
    // non-blocking streams that do not wait for it.
    check(cudaStreamSynchronize(cudaStreamLegacy), "filling the arena");
  } catch (...) {
    release();
    throw;
  }
}

ThresholdPlan::~ThresholdPlan() { release(); }

void ThresholdPlan::release() {
  cudaFree(arena_);
  cudaFree(frames_);
  cudaFree(tile_count_);
  cudaFree(tile_start_);
  cudaFree(pool_);
  cudaFree(pool_next_);
  cudaFree(out_);
  cudaFree(block_sums_);
  cudaFree(frame_prefix_);
  cudaFree(frame_count_);
  arena_ = nullptr;
  frames_ = nullptr;
  tile_count_ = tile_start_ = nullptr;
  pool_ = out_ = nullptr;
  pool_next_ = block_sums_ = frame_prefix_ = frame_count_ = nullptr;
}

void *ThresholdPlan::frame_origin(int f) const {
  const uint64_t at = static_cast<uint64_t>(host_frames_[f].row0) * pitch_ + kMarginLeft;
  return static_cast<char *>(arena_) + at * elem_bytes_;
}

void ThresholdPlan::upload(int f, const void *host, cudaStream_t stream) {
  const Shape &s = shapes_[f];
  const size_t row_bytes = static_cast<size_t>(s.width) * elem_bytes_;
  check(cudaMemcpy2DAsync(frame_origin(f), pitch_ * elem_bytes_, host, row_bytes, row_bytes,
                          s.height, cudaMemcpyDefault, stream),
        "copying a frame to the device");
}

void ThresholdPlan::upload_device(int f, const void *device, size_t pitch_bytes,
                                  cudaStream_t stream) {
  const Shape &s = shapes_[f];
  const size_t row_bytes = static_cast<size_t>(s.width) * elem_bytes_;
  check(cudaMemcpy2DAsync(frame_origin(f), pitch_ * elem_bytes_, device, pitch_bytes,
                          row_bytes, s.height, cudaMemcpyDeviceToDevice, stream),
        "copying a frame into the arena");
}

void ThresholdPlan::enqueue(cudaStream_t stream) {
  check(cudaMemsetAsync(tile_count_, 0, ntiles_ * sizeof(uint32_t), stream),
        "clearing tile counts");
  check(cudaMemsetAsync(pool_next_, 0, 2 * sizeof(uint32_t), stream), "clearing the pool");
  ThresholdLaunch L;
  L.frames = frames_;
  L.nframes = static_cast<int32_t>(host_frames_.size());
  L.ntasks = ntasks_;
  L.tile_count = tile_count_;
  L.tile_start = tile_start_;
  L.pool = pool_;
  L.pool_next = pool_next_;
  L.pool_cap = pool_cap_;
  L.status = status_;
  L.wait_limit = 1u << 22;
  L.warps_per_block = wpc_;
  L.max_blocks = max_blocks_;
  if (elem_bytes_ == 2)
    check(launch_threshold<uint16_t>(map_, L, stream), "launching the threshold");
  else
    check(launch_threshold<uint32_t>(map_, L, stream), "launching the threshold");

  PlaceLaunch P;
  P.frames = frames_;
  P.nframes = L.nframes;
  P.ntiles = ntiles_;
  P.tile_count = tile_count_;
  P.tile_start = tile_start_;
  P.pool = pool_;
  P.out = out_;
  P.block_sums = block_sums_;
  P.frame_prefix = frame_prefix_;
  P.frame_count = frame_count_;
  check(launch_place(P, stream), "launching the placement");
}

} // namespace sf
