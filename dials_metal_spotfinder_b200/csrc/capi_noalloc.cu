// sf_find_u16_noalloc: the per-frame 16-bit threshold for callers that may
// not allocate device memory.
//
// Some hosts own all of a GPU's memory and forbid the code they load from
// calling cudaMalloc: a detector acquisition or processing framework that
// carves device memory out of its own pool (or whose caching allocator has
// already reserved it), or a real-time loop where cudaMalloc / cudaFree would
// stall, cudaFree by synchronising the whole device. sf_find_u16 keeps a
// per-thread workspace that it allocates on first use and re-allocates when
// the frame shape changes; this entry point instead works entirely in one
// fixed scratch array that is part of the library's device image.
//
// The scratch: a file-scope device array of kScratchBytes (64 MiB). Every GPU
// that loads this library holds it until the process exits. Its device
// address is looked up with cudaGetSymbolAddress once per device, on the
// first call made with that device current; that first call should come
// before any stream capture. Within it, the call lays out the same buffers
// the per-thread plan uses (frame descriptor, tile counts and starts, the
// staging pool, the padded frame arena and the output list) for the frame's
// shape, and rejects, with -1 and a message, any frame whose layout does not
// fit. On a 148-SM B200 every frame of up to 6.2 million pixels at a width of
// at least 1024 fits: a Pilatus 6M (2527 x 2463) needs about 59 MiB, an
// Eiger2 4M (2162 x 2068) about 47 MiB; an Eiger2 16M does not fit.
//
// Every call shares the array, and the array keeps what the last call left
// in it, so each call clears what must start at zero (the tile counts, the
// pool cursor, the status and count words) and refills the arena's masked
// margins, unless the previous completed call on that device had the same
// frame shape and so left them intact. Calls whose device work overlapped would race on the array; each
// call therefore holds a process-wide lock and returns only when its stream
// is idle, so calls through this entry point never overlap. Nothing here
// calls cudaMalloc, cudaFree, cudaMallocHost or any allocating library
// routine.

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/spotfinder_b200.h"
#include "sf_capi.hh"
#include "sf_host.hh"

namespace sf {

constexpr uint64_t kScratchBytes = 64ull << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
constexpr int kWarpsPerBlock = 2;
constexpr int kBlocksPerSm = 2; // bounds the staging pool: one open chunk per warp

std::mutex g_lock;
void *g_scratch_ptr[kMaxDevices] = {};
// The frame shape whose arena margins the scratch holds on each device
// (0 x 0: none, or not known to be intact), so that a run of calls with one
// shape fills the margins once.
size_t g_filled_h[kMaxDevices] = {}, g_filled_w[kMaxDevices] = {};

uint64_t align_up(uint64_t v, uint64_t m) { return (v + m - 1) / m * m; }

// Where each buffer sits in the scratch for one frame shape.
struct Layout {
  FrameDesc frame;
  uint64_t pitch = 0, rows = 0, ntiles = 0;
  uint32_t ntasks = 0, pool_cap = 0;
  int max_blocks = 0;
  uint64_t frame_at = 0, tile_count_at = 0, tile_start_at = 0, pool_at = 0, pool_next_at = 0,
           block_sums_at = 0, arena_at = 0, out_at = 0, prefix_at = 0, count_at = 0;
  uint64_t arena_bytes = 0, total = 0;
};

Layout plan_layout(uint64_t height, uint64_t width) {
  Layout L;
  const int occ = threshold_occupancy<uint16_t>(kWarpsPerBlock);
  if (occ < 1)
    throw DeviceError("the threshold kernel does not fit on this device");
  L.max_blocks = device_sm_count() * std::min(occ, kBlocksPerSm);
  const uint64_t resident = static_cast<uint64_t>(L.max_blocks) * kWarpsPerBlock;

  const uint64_t strips = (width + kStripOut - 1) / kStripOut;
  // 232 output columns per 256-column strip; rows start on 128-byte lines
  L.pitch = align_up(strips * kStripOut + (kStripCols - kStripOut), 64);
  L.rows = height + 2 * kMarginRows;

  // Output rows per task: fewest waves x (rows + 20 rows of halo).
  uint64_t seg = height, best = ~0ull;
  for (uint64_t s = 16; s <= height; s++) {
    const uint64_t tasks = strips * ((height + s - 1) / s);
    const uint64_t cost = ((tasks + resident - 1) / resident) * (s + 2 * kHalo);
    if (cost < best) {
      best = cost;
      seg = s;
    }
  }
  seg = std::min(seg, height);
  const uint64_t segments = (height + seg - 1) / seg;

  std::memset(&L.frame, 0, sizeof(L.frame));
  L.frame.row0 = kMarginRows;
  L.frame.height = static_cast<int32_t>(height);
  L.frame.width = static_cast<int32_t>(width);
  L.frame.strips = static_cast<int32_t>(strips);
  L.frame.seg_rows = static_cast<int32_t>(seg);
  L.frame.segments = static_cast<int32_t>(segments);
  L.frame.task_begin = 0;
  L.frame.tile_base = 0;
  L.frame.out_base = 0;
  // the reference's device list capacity: the frame's bytes, 16 to an entry
  const uint64_t cap = height * width * 2 / 16;
  L.frame.capacity = static_cast<uint32_t>(cap);
  L.ntiles = height * strips;
  L.ntasks = static_cast<uint32_t>(strips * segments);

  const uint64_t blocks = std::min<uint64_t>((L.ntasks + kWarpsPerBlock - 1) / kWarpsPerBlock,
                                             static_cast<uint64_t>(L.max_blocks));
  const uint64_t warps = blocks * kWarpsPerBlock;
  const uint64_t chunks =
      (cap + (kChunkRecords - kMaxStaged) - 1) / (kChunkRecords - kMaxStaged) + warps + 1;
  const uint64_t pool_records = chunks * kChunkRecords;
  const uint64_t place_blocks = (L.ntiles + kPlaceTiles - 1) / kPlaceTiles;
  L.arena_bytes = L.pitch * L.rows * sizeof(uint16_t);

  uint64_t at = 0;
  auto take = [&](uint64_t bytes) {
    const uint64_t here = at;
    at = align_up(at + std::max<uint64_t>(bytes, 16), 256);
    return here;
  };
  L.frame_at = take(sizeof(FrameDesc));
  L.tile_count_at = take(L.ntiles * 4);
  L.tile_start_at = take(L.ntiles * 4);
  L.pool_next_at = take(16);
  L.block_sums_at = take(std::max<uint64_t>(place_blocks, 1) * 4);
  L.prefix_at = take(2 * 4);
  L.count_at = take(2 * 4); // the frame's count, then the status word
  L.arena_at = take(L.arena_bytes);
  L.out_at = take(cap * sizeof(SignalPixel));
  L.pool_at = take(pool_records * sizeof(SignalPixel));
  L.total = at;
  L.pool_cap = static_cast<uint32_t>(std::min<uint64_t>(pool_records, 0xffffffffull));
  return L;
}

// The scratch's device address on the current device, looked up once.
unsigned char *scratch_address() {
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices)
    throw DeviceError("device ordinal beyond the no-allocation path's table");
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress (scratch)");
    g_scratch_ptr[dev] = p;
  }
  return static_cast<unsigned char *>(g_scratch_ptr[dev]);
}

int find_noalloc(const uint16_t *image, size_t height, size_t width, SignalPixel *out,
                 size_t capacity, size_t *found, cudaStream_t s) {
  if (found)
    *found = 0;
  if (image == nullptr || height == 0 || width == 0 || found == nullptr)
    return -1;
  if (height > 0x7fffffffu / width)
    return -1;
  const std::lock_guard<std::mutex> hold(g_lock);
  unsigned char *base = scratch_address();
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  const Layout L = plan_layout(height, width);
  if (L.total > kScratchBytes) {
    set_error(("a " + std::to_string(height) + " x " + std::to_string(width) +
               " frame needs " + std::to_string(L.total) +
               " bytes of scratch; sf_find_u16_noalloc holds " + std::to_string(kScratchBytes))
                  .c_str());
    return -1;
  }
  auto *frames = reinterpret_cast<FrameDesc *>(base + L.frame_at);
  auto *tile_count = reinterpret_cast<uint32_t *>(base + L.tile_count_at);
  auto *tile_start = reinterpret_cast<uint32_t *>(base + L.tile_start_at);
  auto *pool = reinterpret_cast<SignalPixel *>(base + L.pool_at);
  auto *pool_next = reinterpret_cast<uint32_t *>(base + L.pool_next_at);
  auto *block_sums = reinterpret_cast<uint32_t *>(base + L.block_sums_at);
  auto *prefix = reinterpret_cast<uint32_t *>(base + L.prefix_at);
  auto *count = reinterpret_cast<uint32_t *>(base + L.count_at);
  int *status = reinterpret_cast<int *>(count + 1);
  void *arena = base + L.arena_at;
  auto *list = reinterpret_cast<SignalPixel *>(base + L.out_at);

  // Whatever happens below, the stream is idle before the lock is released.
  struct Idle {
    cudaStream_t s;
    ~Idle() { cudaStreamSynchronize(s); }
  } idle{s};

  check(cudaMemcpyAsync(frames, &L.frame, sizeof(FrameDesc), cudaMemcpyHostToDevice, s),
        "uploading the frame descriptor");
  check(cudaMemsetAsync(tile_count, 0, L.ntiles * 4, s), "clearing tile counts");
  check(cudaMemsetAsync(pool_next, 0, 16, s), "clearing the pool cursor");
  check(cudaMemsetAsync(count, 0, 2 * 4, s), "clearing the count and status");
  // Off-frame pixels read as masked: every byte of the arena that the frame
  // does not cover is 0xFF. The layout is a function of the shape and only
  // the frame's own pixels are written below, so after a completed call with
  // the same shape the margins are still 0xFF and the fill is skipped. The
  // record is cleared first and set again only once this call completes, so
  // a call that fails part-way makes the next one fill.
  const bool filled = g_filled_h[dev] == height && g_filled_w[dev] == width;
  g_filled_h[dev] = g_filled_w[dev] = 0;
  if (!filled)
    check(cudaMemsetAsync(arena, 0xff, L.arena_bytes, s), "filling the arena");
  const uint64_t origin = (static_cast<uint64_t>(L.frame.row0) * L.pitch + kMarginLeft) * 2;
  // cudaMemcpyDefault, as sf_find_u16 uses: the image may be host, device or
  // managed memory.
  check(cudaMemcpy2DAsync(static_cast<unsigned char *>(arena) + origin, L.pitch * 2, image,
                          width * 2, width * 2, height, cudaMemcpyDefault, s),
        "copying the frame to the device");

  CUtensorMap map;
  encode_arena_map(&map, arena, 2, L.pitch, L.rows);
  ThresholdLaunch T;
  T.frames = frames;
  T.nframes = 1;
  T.ntasks = L.ntasks;
  T.tile_count = tile_count;
  T.tile_start = tile_start;
  T.pool = pool;
  T.pool_next = pool_next;
  T.pool_cap = L.pool_cap;
  T.status = status;
  T.wait_limit = 1u << 22;
  T.warps_per_block = kWarpsPerBlock;
  T.max_blocks = L.max_blocks;
  check(launch_threshold<uint16_t>(map, T, s), "launching the threshold");

  PlaceLaunch P;
  P.frames = frames;
  P.nframes = 1;
  P.ntiles = L.ntiles;
  P.tile_count = tile_count;
  P.tile_start = tile_start;
  P.pool = pool;
  P.out = list;
  P.block_sums = block_sums;
  P.frame_prefix = prefix;
  P.frame_count = count;
  check(launch_place(P, s), "launching the placement");

  uint32_t host_words[2] = {0, 0};
  check(cudaMemcpyAsync(host_words, count, sizeof(host_words), cudaMemcpyDeviceToHost, s),
        "reading the signal count back");
  check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  if (static_cast<int>(host_words[1]) == kStatusTmaTimeout)
    throw DeviceError("a TMA load did not complete in time");
  g_filled_h[dev] = height;
  g_filled_w[dev] = width;
  *found = host_words[0];
  if (host_words[0] > L.frame.capacity || host_words[0] > capacity)
    return -2;
  if (host_words[0] == 0)
    return 0;
  check(cudaMemcpyAsync(out, list, host_words[0] * sizeof(SignalPixel), cudaMemcpyDefault, s),
        "copying the signal pixels back");
  check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  return 0;
}

} // namespace
} // namespace sf

extern "C" int sf_find_u16_noalloc(const uint16_t *image, size_t height, size_t width,
                                   sf_signal_pixel *out, size_t capacity, size_t *found,
                                   void *stream) {
  return sf::guarded([&] {
    return sf::find_noalloc(image, height, width, reinterpret_cast<sf::SignalPixel *>(out),
                            capacity, found, static_cast<cudaStream_t>(stream));
  });
}
