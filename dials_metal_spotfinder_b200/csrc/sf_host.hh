// Host-side declarations shared by the library's translation units: kernel
// launch descriptors, the threshold plan (device buffers for one batch shape)
// and the error type. Nothing here is part of the public C-ABI, which is
// include/spotfinder_b200.h.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "sf_device.cuh"

namespace sf {

// A device or runtime failure, reported through the C-ABI as -3 with the
// message kept for sf_last_error().
struct DeviceError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void check(cudaError_t status, const char *what) {
  if (status != cudaSuccess)
    throw DeviceError(std::string("CUDA: ") + what + ": " + cudaGetErrorString(status));
}

void set_error(const char *what);

struct ThresholdLaunch {
  const FrameDesc *frames;
  int32_t nframes;
  uint32_t ntasks;
  uint32_t *tile_count;
  uint32_t *tile_start;
  SignalPixel *pool;
  uint32_t *pool_next;
  uint32_t pool_cap;
  int *status;
  uint32_t wait_limit;
  int warps_per_block;
  int max_blocks; // 0: one warp per task
};

template <typename T>
cudaError_t launch_threshold(const CUtensorMap &map, const ThresholdLaunch &L,
                             cudaStream_t stream);
template <typename T> size_t threshold_smem_bytes(int wpc);
template <typename T> int threshold_occupancy(int wpc);

// Ordered compaction of the staged records (place.cu).
struct PlaceLaunch {
  const FrameDesc *frames;
  int32_t nframes;
  uint64_t ntiles;
  const uint32_t *tile_count;
  const uint32_t *tile_start;
  const SignalPixel *pool;
  SignalPixel *out;
  uint32_t *block_sums;   // ceil(ntiles / kPlaceTiles)
  uint32_t *frame_prefix; // nframes + 1
  uint32_t *frame_count;  // nframes
};
constexpr int kPlaceThreads = 256;
constexpr int kPlaceItems = 4;
constexpr int kPlaceTiles = kPlaceThreads * kPlaceItems;

cudaError_t launch_place(const PlaceLaunch &L, cudaStream_t stream);

// Writes the type's maximum at base[offsets[i]], i < n (mask.cu).
cudaError_t launch_stamp_mask(void *base, int elem_bytes, const uint64_t *offsets, uint64_t n,
                              cudaStream_t s);

// cuTensorMapEncodeTiled through the runtime's driver entry point, so the
// library needs no link against libcuda.
void encode_arena_map(CUtensorMap *map, void *base, int elem_bytes,
                      uint64_t pitch_elems, uint64_t rows);

int device_sm_count();

// Launch geometry of the threshold for one batch shape.
struct PlanTuning {
  int seg_rows = 0;        // output rows per task; 0 picks by frame count
  int warps_per_block = 0; // 1, 2 or 4; 0: 2 for 16-bit pixels, 1 for 32-bit
  int blocks_per_sm = 0;   // 0: as many as fit
};

// The device buffers for thresholding one batch shape: `slots` arenas the
// frames are copied into (each with its own TMA descriptor and output lists,
// so one slot can be filled or read while another is computed), and the tile
// arrays and staging pool the runs share. Built once per shape and reused;
// every launch it enqueues is capturable in a CUDA graph.
class ThresholdPlan {
public:
  struct Shape {
    int32_t height;
    int32_t width;
  };

  ThresholdPlan(int elem_bytes, const std::vector<Shape> &shapes, const PlanTuning &tuning,
                int slots = 1);
  ~ThresholdPlan();
  ThresholdPlan(const ThresholdPlan &) = delete;
  ThresholdPlan &operator=(const ThresholdPlan &) = delete;

  // Enqueue the threshold of slot `slot` on `stream`: clears, threshold,
  // placement. When `mid` is given it is recorded between the threshold and
  // the placement, so the two can be timed apart.
  void enqueue(int slot, cudaStream_t stream, cudaEvent_t mid = nullptr);

  // Copy a host frame (row-major, height x width) into frame f of a slot.
  void upload(int slot, int f, const void *host, cudaStream_t stream);
  // Copy a device frame (row-major, pitch in bytes) into frame f of a slot.
  void upload_device(int slot, int f, const void *device, size_t pitch_bytes,
                     cudaStream_t stream);

  int elem_bytes() const { return elem_bytes_; }
  int nframes() const { return static_cast<int>(shapes_.size()); }
  int nslots() const { return static_cast<int>(slots_.size()); }
  const Shape &shape(int f) const { return shapes_[f]; }
  uint64_t pitch() const { return pitch_; }
  // Pointer to frame f's pixel (0, 0) inside slot s's arena.
  void *frame_origin(int slot, int f) const;
  SignalPixel *out(int slot) const { return slots_[slot].out; }
  uint64_t out_base(int f) const { return host_frames_[f].out_base; }
  uint32_t capacity(int f) const { return host_frames_[f].capacity; }
  uint32_t *frame_count(int slot) const { return slots_[slot].frame_count; }
  int *status(int slot) const { return slots_[slot].status; }
  uint32_t ntasks() const { return ntasks_; }
  uint64_t ntiles() const { return ntiles_; }
  uint64_t total_capacity() const { return total_capacity_; }
  const FrameDesc *device_frames() const { return frames_; }
  const PlanTuning &tuning() const { return tuning_; }
  int grid_blocks() const { return grid_blocks_; }
  uint64_t device_bytes() const { return device_bytes_; }

private:
  struct Slot {
    void *arena = nullptr;
    CUtensorMap map;
    SignalPixel *out = nullptr;
    uint32_t *frame_prefix = nullptr;
    uint32_t *frame_count = nullptr; // followed by the status word
    int *status = nullptr;
  };

  void release();

  int elem_bytes_;
  std::vector<Shape> shapes_;
  std::vector<FrameDesc> host_frames_;
  PlanTuning tuning_;
  uint64_t pitch_ = 0, arena_rows_ = 0;
  uint32_t ntasks_ = 0;
  uint64_t ntiles_ = 0, total_capacity_ = 0;
  uint32_t pool_cap_ = 0;
  int max_blocks_ = 0, grid_blocks_ = 0;
  uint64_t device_bytes_ = 0;

  std::vector<Slot> slots_;
  FrameDesc *frames_ = nullptr;
  uint32_t *tile_count_ = nullptr;
  uint32_t *tile_start_ = nullptr;
  SignalPixel *pool_ = nullptr;
  uint32_t *pool_next_ = nullptr;
  uint32_t *block_sums_ = nullptr;
};

// The cost model's task height (plan.cu) for these shapes at `wpc` warps per
// block and as many blocks per SM as fit.
int model_seg_rows(int elem_bytes, const std::vector<ThresholdPlan::Shape> &shapes, int wpc,
                   int blocks_per_sm = 0);

// The autotuner (tune.cu). An entry is what a search measured best for one
// frame shape on one kind of device: frames per launch, warps per block, the
// task height as a ratio to the cost model's, and the time per frame.
struct TuneEntry {
  int frames = 16;
  int warps_per_block = 2;
  double seg_ratio = 1.0;
  double us_per_frame = 0.0;
  int blocks_per_sm = 0; // threshold blocks per SM; 0: as many as fit
};
struct TuneOptions {
  int min_frames = 8, max_frames = 32, steps = 4;
  bool grouping = true, use_cache = true;
  uint64_t hbm_budget = 0; // 0: half the free device memory
  const char *cache_path = nullptr;
};
struct TuneResult {
  TuneEntry entry;
  bool from_cache = false;
  int candidates = 0;
};
std::string tune_cache_path(const char *given);
bool tune_lookup(int elem_bytes, int height, int width, const char *cache_path, TuneEntry *out);
int tune_seg_rows(int elem_bytes, const std::vector<ThresholdPlan::Shape> &shapes, int wpc,
                  double ratio, int blocks_per_sm = 0);
TuneResult tune_search(int elem_bytes, int height, int width, const void *const *sample,
                       int nsample, const TuneOptions &options);

} // namespace sf
