// Exclusive device scans with the length read from device memory.
#pragma once

#include "sf_host.hh"

namespace sf {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename V> class DeviceScan {
public:
  DeviceScan() = default;
  ~DeviceScan();
  DeviceScan(const DeviceScan &) = delete;
  DeviceScan &operator=(const DeviceScan &) = delete;

  // out[i] = in[0] + ... + in[i-1] for i < (*len) * len_scale, and the sum
  // of all of them in *total (if given). `max_len` bounds the device-side
  // length and sizes the block-sum workspace; in and out may alias.
  void run(const V *in, V *out, const uint64_t *len, uint64_t len_scale, uint64_t max_len,
           V *total, cudaStream_t s);
  void reserve(uint64_t max_len);

private:
  V *block_sums_ = nullptr;
  uint64_t max_blocks_ = 0;
  unsigned grid_cap_ = 0; // blocks per launch: one per SM, each taking tiles in turn
};

} // namespace sf
