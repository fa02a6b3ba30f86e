// Host-side declarations shared by the library's translation units: kernel
// launch descriptors, the threshold plan (device buffers for one batch shape)
// and the error type. Nothing here is part of the public C-ABI, which is
// include/spotfinder_b200.h.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

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
constexpr int kPlaceItems = 16;
constexpr int kPlaceTiles = kPlaceThreads * kPlaceItems;

cudaError_t launch_place(const PlaceLaunch &L, cudaStream_t stream);

// cuTensorMapEncodeTiled through the runtime's driver entry point, so the
// library needs no link against libcuda.
void encode_arena_map(CUtensorMap *map, void *base, int elem_bytes,
                      uint64_t pitch_elems, uint64_t rows);

int device_sm_count();

// The device buffers for thresholding one batch shape: the arena the frames
// are copied into, the tile arrays, the staging pool and the output lists.
// Built once per shape and reused; every launch it enqueues is capturable in
// a CUDA graph.
class ThresholdPlan {
public:
  struct Shape {
    int32_t height;
    int32_t width;
  };

  ThresholdPlan(int elem_bytes, const std::vector<Shape> &shapes, int seg_rows,
                int warps_per_block, int blocks_per_sm);
  ~ThresholdPlan();
  ThresholdPlan(const ThresholdPlan &) = delete;
  ThresholdPlan &operator=(const ThresholdPlan &) = delete;

  // Enqueue the threshold and the placement on `stream`. Frames must already
  // be in the arena.
  void enqueue(cudaStream_t stream);

  // Copy a host frame (row-major, height x width) into frame slot f.
  void upload(int f, const void *host, cudaStream_t stream);
  // Copy a device frame (row-major, pitch in bytes) into frame slot f.
  void upload_device(int f, const void *device, size_t pitch_bytes, cudaStream_t stream);

  int elem_bytes() const { return elem_bytes_; }
  int nframes() const { return static_cast<int>(shapes_.size()); }
  const Shape &shape(int f) const { return shapes_[f]; }
  uint64_t pitch() const { return pitch_; }
  void *arena() const { return arena_; }
  // Pointer to frame f's pixel (0, 0) inside the arena.
  void *frame_origin(int f) const;
  SignalPixel *out() const { return out_; }
  uint64_t out_base(int f) const { return host_frames_[f].out_base; }
  uint32_t capacity(int f) const { return host_frames_[f].capacity; }
  uint32_t *frame_count() const { return frame_count_; }
  int *status() const { return status_; }
  uint32_t ntasks() const { return ntasks_; }
  uint64_t ntiles() const { return ntiles_; }
  uint64_t total_capacity() const { return total_capacity_; }
  const FrameDesc *device_frames() const { return frames_; }
  int seg_rows() const { return seg_rows_; }
  int warps_per_block() const { return wpc_; }

private:
  void release();

  int elem_bytes_;
  std::vector<Shape> shapes_;
  std::vector<FrameDesc> host_frames_;
  int seg_rows_, wpc_, blocks_per_sm_;
  uint64_t pitch_ = 0, arena_rows_ = 0;
  uint32_t ntasks_ = 0;
  uint64_t ntiles_ = 0, total_capacity_ = 0;
  uint32_t pool_cap_ = 0;
  int max_blocks_ = 0;

  CUtensorMap map_;
  void *arena_ = nullptr;
  FrameDesc *frames_ = nullptr;
  uint32_t *tile_count_ = nullptr;
  uint32_t *tile_start_ = nullptr;
  SignalPixel *pool_ = nullptr;
  uint32_t *pool_next_ = nullptr; // followed by the status word
  int *status_ = nullptr;
  SignalPixel *out_ = nullptr;
  uint32_t *block_sums_ = nullptr;
  uint32_t *frame_prefix_ = nullptr;
  uint32_t *frame_count_ = nullptr;
};

} // namespace sf
