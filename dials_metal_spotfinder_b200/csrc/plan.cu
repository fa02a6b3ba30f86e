// ThresholdPlan: the device buffers and launch geometry for thresholding one
// batch shape (one or many frames, equal or uneven sizes), built once and
// reused frame after frame. Also the TMA descriptor over each frame arena.

#include <algorithm>
#include <cstring>
#include <mutex>

#include "sf_host.hh"

namespace sf {
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

// Output rows per task. A warp's cost is its rows plus the 20 rows of halo
// it re-reads, and the launch lasts as many waves as the tasks need; pick the
// segment height that minimises waves x (rows + halo).
int choose_seg_rows(const std::vector<ThresholdPlan::Shape> &shapes, uint64_t resident) {
  int max_h = 1;
  for (const auto &s : shapes)
    max_h = std::max(max_h, s.height);
  int best = max_h;
  double best_cost = 1e300;
  for (int seg = 16; seg <= max_h; seg++) {
    uint64_t tasks = 0;
    for (const auto &s : shapes) {
      const uint64_t strips = (s.width + kStripOut - 1) / kStripOut;
      tasks += strips * ((s.height + seg - 1) / seg);
    }
    const uint64_t waves = (tasks + resident - 1) / resident;
    const double cost = static_cast<double>(waves) * (std::min(seg, max_h) + 2 * kHalo);
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = seg;
    }
  }
  return best;
}

} // namespace

int model_seg_rows(int elem_bytes, const std::vector<ThresholdPlan::Shape> &shapes, int wpc,
                   int blocks_per_sm) {
  int occ = elem_bytes == 2 ? threshold_occupancy<uint16_t>(wpc)
                            : threshold_occupancy<uint32_t>(wpc);
  if (occ < 1)
    throw DeviceError("the threshold kernel does not fit on this device");
  if (blocks_per_sm > 0)
    occ = std::min(occ, blocks_per_sm);
  return choose_seg_rows(shapes, static_cast<uint64_t>(device_sm_count()) * occ * wpc);
}

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

ThresholdPlan::ThresholdPlan(int elem_bytes, const std::vector<Shape> &shapes,
                             const PlanTuning &tuning, int slots)
    : elem_bytes_(elem_bytes), shapes_(shapes), tuning_(tuning) {
  if (elem_bytes != 2 && elem_bytes != 4)
    throw std::invalid_argument("pixels are 16 or 32 bits");
  if (shapes.empty())
    throw std::invalid_argument("a plan needs at least one frame");
  if (slots < 1)
    throw std::invalid_argument("a plan needs at least one slot");
  // 16-bit pixels: 7 two-warp blocks per SM; 32-bit: each warp's shared
  // memory is twice the size, so one-warp blocks fill the SM best
  if (tuning_.warps_per_block == 0)
    tuning_.warps_per_block = elem_bytes == 2 ? 2 : 1;
  const int wpc = tuning_.warps_per_block;
  if (wpc != 1 && wpc != 2 && wpc != 4)
    throw std::invalid_argument("warps_per_block must be 1, 2 or 4");

  int32_t max_strips = 0;
  for (const Shape &s : shapes) {
    if (s.height < 1 || s.width < 1)
      throw std::invalid_argument("frame with no pixels");
    if (static_cast<uint64_t>(s.height) * s.width > 0x7fffffffull)
      throw std::invalid_argument("frame larger than INT32_MAX pixels");
    max_strips = std::max(max_strips, (s.width + kStripOut - 1) / kStripOut);
  }
  // Every strip reads 256 columns from a multiple of 232; the pitch is a
  // multiple of 128 bytes so each arena row starts on a TMA-friendly line.
  pitch_ = round_up(static_cast<uint64_t>(max_strips) * kStripOut + (kStripCols - kStripOut),
                    128 / elem_bytes);

  const int occ = elem_bytes == 2 ? threshold_occupancy<uint16_t>(wpc)
                                  : threshold_occupancy<uint32_t>(wpc);
  if (occ < 1)
    throw DeviceError("the threshold kernel does not fit on this device");
  const int per_sm = tuning_.blocks_per_sm > 0 ? std::min(tuning_.blocks_per_sm, occ) : occ;
  max_blocks_ = device_sm_count() * per_sm;
  if (tuning_.seg_rows <= 0)
    tuning_.seg_rows = choose_seg_rows(shapes, static_cast<uint64_t>(max_blocks_) * wpc);

  uint64_t row = 0, tile = 0, out = 0;
  uint32_t task = 0;
  for (const Shape &s : shapes) {
    FrameDesc d;
    std::memset(&d, 0, sizeof(d));
    d.row0 = static_cast<int64_t>(row + kMarginRows);
    d.height = s.height;
    d.width = s.width;
    d.strips = (s.width + kStripOut - 1) / kStripOut;
    d.seg_rows = std::min(tuning_.seg_rows, s.height);
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
  if (total_capacity_ >= 0xffffffffull)
    throw std::invalid_argument("batch too large for one plan");

  grid_blocks_ = static_cast<int>(std::min<uint64_t>((ntasks_ + wpc - 1) / wpc, max_blocks_));
  const uint64_t warps = static_cast<uint64_t>(grid_blocks_) * wpc;
  const uint64_t chunks =
      (total_capacity_ + (kChunkRecords - kMaxStaged) - 1) / (kChunkRecords - kMaxStaged) +
      warps + 1;
  const uint64_t pool_records = chunks * kChunkRecords;
  if (pool_records >= 0xffffffffull - kChunkRecords)
    throw std::invalid_argument("batch too large for one plan");
  pool_cap_ = static_cast<uint32_t>(pool_records);

  const uint64_t arena_bytes = pitch_ * arena_rows_ * elem_bytes;
  const uint64_t nblocks = (ntiles_ + kPlaceTiles - 1) / kPlaceTiles;
  const size_t nf = host_frames_.size();
  slots_.resize(slots);
  try {
    auto alloc = [&](void **p, uint64_t bytes, const char *what) {
      check(cudaMalloc(p, std::max<uint64_t>(bytes, 16)), what);
      device_bytes_ += bytes;
    };
    alloc(reinterpret_cast<void **>(&frames_), nf * sizeof(FrameDesc), "cudaMalloc frames");
    check(cudaMemcpy(frames_, host_frames_.data(), nf * sizeof(FrameDesc),
                     cudaMemcpyHostToDevice),
          "uploading frame descriptors");
    alloc(reinterpret_cast<void **>(&tile_count_), ntiles_ * 4, "cudaMalloc tile counts");
    alloc(reinterpret_cast<void **>(&tile_start_), ntiles_ * 4, "cudaMalloc tile starts");
    alloc(reinterpret_cast<void **>(&pool_), pool_records * sizeof(SignalPixel),
          "cudaMalloc staging pool");
    alloc(reinterpret_cast<void **>(&pool_next_), 16, "cudaMalloc pool cursor");
    alloc(reinterpret_cast<void **>(&block_sums_), std::max<uint64_t>(nblocks, 1) * 4,
          "cudaMalloc block sums");
    for (Slot &sl : slots_) {
      alloc(&sl.arena, arena_bytes, "cudaMalloc arena");
      check(cudaMemset(sl.arena, 0xff, arena_bytes), "filling the arena");
      alloc(reinterpret_cast<void **>(&sl.out), total_capacity_ * sizeof(SignalPixel),
            "cudaMalloc output lists");
      alloc(reinterpret_cast<void **>(&sl.frame_prefix), (nf + 1) * 4,
            "cudaMalloc frame prefix");
      alloc(reinterpret_cast<void **>(&sl.frame_count), (nf + 1) * 4,
            "cudaMalloc frame counts");
      sl.status = reinterpret_cast<int *>(sl.frame_count + nf);
      check(cudaMemset(sl.frame_count, 0, (nf + 1) * 4), "clearing frame counts");
      encode_arena_map(&sl.map, sl.arena, elem_bytes_, pitch_, arena_rows_);
    }
    // The fills above ran on the legacy stream; the plan's users work on
    // non-blocking streams that do not wait for it.
    check(cudaStreamSynchronize(cudaStreamLegacy), "filling the arena");
  } catch (...) {
    release();
    throw;
  }
}

ThresholdPlan::~ThresholdPlan() { release(); }

void ThresholdPlan::release() {
  for (Slot &sl : slots_) {
    cudaFree(sl.arena);
    cudaFree(sl.out);
    cudaFree(sl.frame_prefix);
    cudaFree(sl.frame_count);
    sl = Slot();
  }
  cudaFree(frames_);
  cudaFree(tile_count_);
  cudaFree(tile_start_);
  cudaFree(pool_);
  cudaFree(pool_next_);
  cudaFree(block_sums_);
  frames_ = nullptr;
  tile_count_ = tile_start_ = nullptr;
  pool_ = nullptr;
  pool_next_ = block_sums_ = nullptr;
}

void *ThresholdPlan::frame_origin(int slot, int f) const {
  const uint64_t at = static_cast<uint64_t>(host_frames_[f].row0) * pitch_ + kMarginLeft;
  return static_cast<char *>(slots_[slot].arena) + at * elem_bytes_;
}

void ThresholdPlan::upload(int slot, int f, const void *host, cudaStream_t stream) {
  const Shape &s = shapes_[f];
  const size_t row_bytes = static_cast<size_t>(s.width) * elem_bytes_;
  check(cudaMemcpy2DAsync(frame_origin(slot, f), pitch_ * elem_bytes_, host, row_bytes,
                          row_bytes, s.height, cudaMemcpyDefault, stream),
        "copying a frame to the device");
}

void ThresholdPlan::upload_device(int slot, int f, const void *device, size_t pitch_bytes,
                                  cudaStream_t stream) {
  const Shape &s = shapes_[f];
  const size_t row_bytes = static_cast<size_t>(s.width) * elem_bytes_;
  check(cudaMemcpy2DAsync(frame_origin(slot, f), pitch_ * elem_bytes_, device, pitch_bytes,
                          row_bytes, s.height, cudaMemcpyDeviceToDevice, stream),
        "copying a frame into the arena");
}

void ThresholdPlan::enqueue(int slot, cudaStream_t stream, cudaEvent_t mid) {
  Slot &sl = slots_.at(slot);
  check(cudaMemsetAsync(tile_count_, 0, ntiles_ * sizeof(uint32_t), stream),
        "clearing tile counts");
  check(cudaMemsetAsync(pool_next_, 0, sizeof(uint32_t), stream), "clearing the pool");
  check(cudaMemsetAsync(sl.status, 0, sizeof(int), stream), "clearing the status");
  ThresholdLaunch L;
  L.frames = frames_;
  L.nframes = static_cast<int32_t>(host_frames_.size());
  L.ntasks = ntasks_;
  L.tile_count = tile_count_;
  L.tile_start = tile_start_;
  L.pool = pool_;
  L.pool_next = pool_next_;
  L.pool_cap = pool_cap_;
  L.status = sl.status;
  L.wait_limit = 1u << 22;
  L.warps_per_block = tuning_.warps_per_block;
  L.max_blocks = max_blocks_;
  if (elem_bytes_ == 2)
    check(launch_threshold<uint16_t>(sl.map, L, stream), "launching the threshold");
  else
    check(launch_threshold<uint32_t>(sl.map, L, stream), "launching the threshold");
  if (mid)
    check(cudaEventRecord(mid, stream), "cudaEventRecord");

  PlaceLaunch P;
  P.frames = frames_;
  P.nframes = L.nframes;
  P.ntiles = ntiles_;
  P.tile_count = tile_count_;
  P.tile_start = tile_start_;
  P.pool = pool_;
  P.out = sl.out;
  P.block_sums = block_sums_;
  P.frame_prefix = sl.frame_prefix;
  P.frame_count = sl.frame_count;
  check(launch_place(P, stream), "launching the placement");
}

} // namespace sf
