// The device labeller: 3D (or 2D) six-connected grouping of signal pixels
// across frames, and the per-spot centroid / variance / intensity pass, with
// the reference's streaming semantics (src/dials_spots.cc:36-360): frames
// arrive in ascending order, a component is finished as soon as a frame is
// added that it has no pixel on, finished components come out ordered by
// their last frame and then their first pixel, and the open ones are carried
// on the device to the next batch.
#pragma once

#include <memory>
#include <vector>

#include "sf_host.hh"
#include "sf_scan.cuh"

namespace sf {

// src/dials_spots.hh:50-54 and :57-79, byte for byte.
struct Pixel {
  int32_t frame;
  uint32_t index;
  uint32_t value;
};
struct Spot {
  int32_t bbox[6];
  double position[3];
  double variance[3];
  double intensity;
  double intensity_variance;
  uint32_t n_signal;
  uint64_t first;
};
static_assert(sizeof(Pixel) == 12, "Pixel layout");
static_assert(sizeof(Spot) == 104, "Spot layout");

struct GroupOptions {
  uint64_t min_spot_size = 3;
  uint64_t max_spot_size = 1000;
  double max_separation = 2.0;
  bool two_d = false;
};

// Device-side scalars (one struct, so the host reads them back in one copy).
struct LabelScalars {
  // this batch
  int64_t batch_z0;       // frame number of the batch's first frame
  uint64_t n;             // live pixels (carried + new)
  uint64_t nw;            // 32-pixel words over n
  uint64_t nseg;          // frame segments (carried last frame + batch frames)
  uint64_t seg_len;       // bucket-count table length: nseg * ceil(closed / 32)
  uint64_t closed;        // finished components
  uint32_t closed32, open32;
  uint32_t runs_n;        // lab_link's work list
  uint32_t big_n;         // components past the middle spot-pass buffers
  // work counters: warps take the next entries as they finish their last,
  // so a few long union-find chains or large components do not hold a
  // whole grid-stride share
  uint32_t link_next, accept_next, big_next, mid_next;
  uint32_t mid_n;         // components past the small buffers, within the middle ones
  uint32_t pad0;
  uint64_t members_pack;  // members (low 32) | components passing the size filters (high 32)
  uint64_t accepted_pack; // accepted spots (low 32) | their pixels (high 32)
  uint64_t batch_spots, batch_pixels;
  // the carry between batches
  uint64_t carry_n;
  uint64_t carry_last_start; // first carried pixel on the carry's last frame
  int64_t carry_last_z;
  // running totals over the series (src/dials_spots.hh:99-106)
  uint64_t signal_pixels, groups, too_small, too_large, separated, accepted;
  uint64_t kept_total; // pixels of accepted spots so far (Spot::first base)
  int32_t status;      // nonzero: a capacity was exceeded
  int32_t pad1;
};

enum : int32_t { kLabelOk = 0, kLabelLiveOverflow = 1, kLabelSpotOverflow = 2 };

class DeviceLabeller {
public:
  DeviceLabeller(int height, int width, const GroupOptions &options);
  ~DeviceLabeller();
  DeviceLabeller(const DeviceLabeller &) = delete;
  DeviceLabeller &operator=(const DeviceLabeller &) = delete;

  // Buffers for batches of up to `batch_pixels` new signal pixels over up to
  // `max_frames` frames, with up to `carry_pixels` carried between batches.
  // Grows (synchronising the device) only when asked for more; call before
  // any graph capture.
  void reserve(uint64_t batch_pixels, int max_frames, uint64_t carry_pixels);

  // Enqueue one batch of `nframes` consecutive frames numbered from the
  // device-side batch_z0, which the batch then advances by nframes. Frame
  // f's list is lists[offs[f] ...] holding up to caps[f] records, with
  // counts[count_map[f]] entries (counts[f] when count_map is null), all in
  // device memory. With close_all every component is finished, as the
  // reference's finish() does; nframes may then be 0.
  void enqueue(int nframes, const SignalPixel *lists, const uint64_t *offs,
               const uint32_t *counts, const int32_t *count_map, const uint32_t *caps,
               bool close_all, cudaStream_t s);

  // Sets batch_z0 for the next enqueue (an asynchronous copy from pinned
  // host memory; the labeller keeps the staging word until the next call).
  void set_next_frame(int64_t z, cudaStream_t s);

  // A batch captured in a CUDA graph was replayed: it swapped the live
  // buffers on the device, so the host's record of which holds the carry
  // swaps too.
  void note_replayed() { cur_ ^= 1; }
  int parity() const { return cur_; }

  LabelScalars *scalars() const { return sc_; }
  Spot *batch_spots() const { return spots_out_; }
  Pixel *batch_pixels() const { return kept_out_; }
  uint64_t spot_capacity() const { return spot_cap_; }
  uint64_t batch_capacity() const { return batch_cap_; }
  int frame_capacity() const { return frame_cap_; }
  int height() const { return height_; }
  int width() const { return width_; }
  const GroupOptions &options() const { return opt_; }

private:
  void release();

  int height_, width_;
  GroupOptions opt_;

  uint64_t batch_cap_ = 0, carry_cap_ = 0, live_cap_ = 0, spot_cap_ = 0;
  int frame_cap_ = 0;
  int cur_ = 0; // which live buffer holds the carry

  struct Live {
    int32_t *frame = nullptr;
    uint32_t *index = nullptr;
    uint32_t *value = nullptr;
    uint32_t *parent = nullptr;
  } live_[2];
  uint32_t *root_ = nullptr, *size_ = nullptr, *rank_of_root_ = nullptr, *cursor_ = nullptr;
  int32_t *lastz_ = nullptr;
  uint32_t *bits_ = nullptr, *bcnt_ = nullptr; // finished-root bitmap; counts (see lab_mark)
  uint32_t *flist_ = nullptr;                   // the finished roots in position order
  uint32_t *comp_root_ = nullptr, *msize_ = nullptr, *members_ = nullptr;
  uint64_t *mpk_ = nullptr; // member offset (low 32) | size-filtered index (high 32)
  uint4 *runs_ = nullptr; // lab_link's work list
  uint32_t *run_starts_ = nullptr; // per 32 positions: the run starts (lab_gather)
  Spot *spot_tmp_ = nullptr;  // spots by size-filtered index, before acceptance
  Pixel *pix_tmp_ = nullptr;  // their pixels, by member offset
  uint64_t *pack_ = nullptr;
  uint32_t *obits_ = nullptr, *ocnt_ = nullptr; // open pixels per 32 positions
  uint32_t *big_ = nullptr; // ranks of the components lab_accept's large launch takes
  uint32_t *mid_ = nullptr; // ... and its middle launch
  Spot *spots_out_ = nullptr;
  Pixel *kept_out_ = nullptr;
  uint64_t *seg_start_ = nullptr; // per batch segment: start, count (device)
  uint64_t *seg_count_ = nullptr;
  int64_t *seg_z_ = nullptr;
  uint32_t *tab_ = nullptr;       // block tables of the batch frames
  uint32_t *carry_tab_ = nullptr; // block table of the carry's last frame
  uint64_t nblk_ = 0;
  unsigned grid_ = 0;
  LabelScalars *sc_ = nullptr;
  cudaStream_t aux_ = nullptr;  // the large components' spot pass
  cudaStream_t aux2_ = nullptr; // the middle-sized components' spot pass
  cudaEvent_t fork_ = nullptr, join_ = nullptr, join2_ = nullptr;
  int64_t *z_stage_ = nullptr; // pinned

  DeviceScan<uint32_t> scan32_;
  DeviceScan<uint64_t> scan64_;
};

} // namespace sf
