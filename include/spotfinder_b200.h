/* spotfinder_b200: the B200-native spot-finder hot path behind a C ABI.
 *
 * Plain pointers and sizes only; no CUDA, C++ or torch types cross this
 * boundary. Every function that can fail returns an int status:
 *
 *     0   success
 *    -1   a bad argument (null image, zero or oversized dimensions, ...)
 *    -2   more signal pixels than the list holds (see sf_find_u16)
 *    -3   a device or runtime failure; sf_last_error() says what
 *    -4   a labelling input refused (frame out of order, pixels not
 *         ascending, pixel off the frame); sf_last_error() says which
 *
 * The reference interface each entry point replaces is cited beside it
 * (paths are within graeme-winter/dials-metal-spotfinder). The C++ drop-in
 * for the reference's own gpu:: interface (include/dext_gpu.hh) is built on
 * these functions.
 *
 * Threading: sf_find_* may be called concurrently from many host threads; each
 * thread gets its own stream and device buffers, as the reference's per-thread
 * Workspace does (src/dext_cuda.cu:466-542). A handle (labeller, engine) is
 * used by one thread at a time.
 */
#ifndef SPOTFINDER_B200_H
#define SPOTFINDER_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SF_API __attribute__((visibility("default")))
#else
#define SF_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* The 16-byte signal record; src/signal_pixel.hh:20-26, byte-identical. */
typedef struct sf_signal_pixel {
  uint32_t index;      /* row-major position in the frame */
  uint32_t value;      /* the raw pixel */
  float background;    /* the masked local mean at that pixel */
  uint16_t population; /* pixels that mean was averaged over */
  uint16_t reserved;   /* 0 */
} sf_signal_pixel;

/* One signal pixel of an accepted spot; src/dials_spots.hh:50-54. */
typedef struct sf_pixel {
  int32_t frame;
  uint32_t index;
  uint32_t value;
} sf_pixel;

/* One accepted spot; src/dials_spots.hh:57-79, byte-identical (104 bytes). */
typedef struct sf_spot {
  int32_t bbox[6];           /* x0, x1, y0, y1, z0, z1; upper bounds exclusive */
  double position[3];        /* xyzobs.px.value */
  double variance[3];        /* xyzobs.px.variance */
  double intensity;          /* intensity.sum.value */
  double intensity_variance; /* intensity.sum.variance */
  uint32_t n_signal;         /* pixels in the spot */
  uint64_t first;            /* where its pixels start in the pixel list */
} sf_spot;

/* Grouping outcome counts; src/dials_spots.hh:99-106. */
typedef struct sf_counts {
  uint64_t signal_pixels, groups, too_small, too_large, separated, accepted;
} sf_counts;

/* Grouping options; src/dials_spots.hh:81-95 (the dials.find_spots
 * defaults are 3, 1000, 2.0, 0). */
typedef struct sf_group_options {
  uint64_t min_spot_size;
  uint64_t max_spot_size;
  double max_separation; /* <= 0 turns the peak-centroid filter off */
  int32_t two_d;         /* group each frame on its own */
  int32_t reserved;
} sf_group_options;

/* ---- device and host memory: src/dext_gpu.hh:26-28, 125-139 ------------ */

/* "CUDA sm_100a (B200-native)"; replaces gpu::backend(). */
SF_API const char *sf_backend(void);
/* 1 if a usable CUDA device is present; replaces gpu::available(). */
SF_API int sf_available(void);
/* Free device memory in bytes; replaces gpu::memory_free(). */
SF_API size_t sf_memory_free(void);
/* Page-locked host memory (NULL on failure: fall back to ordinary memory);
 * replaces gpu::host_alloc() / gpu::host_free(). */
SF_API void *sf_host_alloc(size_t bytes);
SF_API void sf_host_free(void *pointer);
/* The message for the last -3 or -4 on this thread. */
SF_API const char *sf_last_error(void);
/* Make `device` current for the calling thread (one process per GPU, as
 * torchrun launches them). No reference counterpart: the reference uses the
 * default device only. */
SF_API int sf_set_device(int device);

/* ---- the threshold: src/dext_gpu.hh:141-166 (gpu::find<T>) ------------- *
 *
 * Thresholds one row-major height x width frame from host memory and writes
 * its signal pixels to `out`, ascending by index, exactly as the reference's
 * dext<T> (src/dext.cc:9-225) would. *found is set to the number of signal
 * pixels whenever the arguments are valid.
 *
 * Returns -1 for a null image, a zero dimension or height * width beyond
 * INT32_MAX; -2 if the frame has more signal pixels than the reference's
 * device list holds (height * width * sizeof(pixel) / 16, src/dext_cuda.cu:
 * 611-616) or than `capacity`; -3 on a device failure. */
SF_API int sf_find_u16(const uint16_t *image, size_t height, size_t width, sf_signal_pixel *out,
                size_t capacity, size_t *found);
SF_API int sf_find_u32(const uint32_t *image, size_t height, size_t width, sf_signal_pixel *out,
                size_t capacity, size_t *found);

/* sf_find_u16 for callers that may not allocate device memory. No
 * counterpart in the reference, whose gpu::find allocates per call.
 *
 * For plugins loaded into a host that owns the GPU's memory (a framework
 * whose pool or caching allocator holds it) and for real-time loops where
 * cudaMalloc / cudaFree would stall -- cudaFree synchronises the device.
 * Same arguments, results and status codes as sf_find_u16, plus the stream
 * to run on (NULL: the legacy default stream); it returns when the results
 * are in `out`. It allocates nothing: it works in one 64 MiB device array
 * that is part of the library (every GPU that loads the library holds it
 * until exit) and returns -1, with the reason in sf_last_error(), for a
 * frame whose buffers do not fit there (every frame of up to 6.2 million
 * pixels at a width of at least 1024 fits on a 148-SM B200). The first call
 * on each device looks the array's address up; make it before any stream
 * capture. All calls share the array, so calls whose device work overlapped
 * would race: each call holds a process-wide lock until its work is done. */
SF_API int sf_find_u16_noalloc(const uint16_t *image, size_t height, size_t width,
                               sf_signal_pixel *out, size_t capacity, size_t *found,
                               void *stream);

/* ---- stage profiling: src/dext_gpu.hh:79-116 ---------------------------- *
 * When on, sf_find_* records, for the calling thread, milliseconds spent in:
 * [0] upload (host to device), [1] the fused threshold kernel, [2] 0 (the
 * erode is fused into [1]), [3] the ordered compaction, [4] reading the list
 * back, [5] 0 (no host sort is needed). */
SF_API void sf_profile_stages(int on);
SF_API int sf_profile_stages_enabled(void);
SF_API void sf_last_stage_times(double out6[6]);

/* ---- grouping: src/dials_spots.hh:108-126 (dials_spots::Labeller) ------- *
 *
 * 3D (or, with two_d, per-frame) six-connected grouping of signal pixels on
 * the device, and the centroid / variance / intensity / filter pass, with
 * the reference's streaming semantics: frames in ascending order, a gap in
 * the numbering closes everything open, spots come out ordered by the frame
 * their component closed on and then by first pixel. Spots and pixels are
 * byte-identical to the reference's (centroids and variances included: the
 * double arithmetic runs in the reference's order). */
typedef struct sf_labeller sf_labeller;

SF_API int sf_labeller_create(size_t height, size_t width, const sf_group_options *options,
                              sf_labeller **out);
SF_API void sf_labeller_destroy(sf_labeller *labeller);
/* Labeller::add: `signal` ascending by index (what the threshold emits).
 * -4 (nothing changed) if the frame is not after the last one, a pixel is
 * off the frame or the pixels are not ascending. */
SF_API int sf_labeller_add(sf_labeller *labeller, int64_t frame, const sf_signal_pixel *signal,
                           size_t n);
/* Labeller::finish: close everything still open. */
SF_API int sf_labeller_finish(sf_labeller *labeller);
SF_API int sf_labeller_counts(sf_labeller *labeller, sf_counts *out);
SF_API size_t sf_labeller_nspots(sf_labeller *labeller);
SF_API size_t sf_labeller_npixels(sf_labeller *labeller);
/* Labeller::live: pixels held for components that may still grow. */
SF_API size_t sf_labeller_live(sf_labeller *labeller);
/* Labeller::spots / pixels, copied out; -2 if `capacity` is too small. */
SF_API int sf_labeller_spots(sf_labeller *labeller, sf_spot *out, size_t capacity);
SF_API int sf_labeller_pixels(sf_labeller *labeller, sf_pixel *out, size_t capacity);

/* ---- detector chunks: src/decompress.hh:14-31 (decompress::image) ------- *
 *
 * A frame as the HDF5 filters store it: SF_CHUNK_RAW (uncompressed),
 * SF_CHUNK_LZ4 (the HDF5 LZ4 filter: 12-byte big-endian header of size and
 * block size, then per block a 4-byte big-endian length and an LZ4 block)
 * or SF_CHUNK_BSLZ4 (bitshuffle + LZ4, as Eiger detectors write: the same
 * header, then per block of elements an LZ4 block of its bit transpose, the
 * last elements mod 8 raw). Bitshuffle blocks of up to 16 KB are accepted.
 * sf_chunk_encode writes one (8 KB blocks), as a detector or a replay source
 * would; sf_chunk_decode is the host decoder. Both return -1 for bad
 * arguments or a chunk that does not describe the frame (header size,
 * framing, malformed LZ4), -2 (encode) if `capacity` is too small. */
enum { SF_CHUNK_RAW = 0, SF_CHUNK_LZ4 = 1, SF_CHUNK_BSLZ4 = 2 };
/* An upper bound on an encoded chunk's size. */
SF_API size_t sf_chunk_bound(size_t height, size_t width, int elem_bytes);
SF_API int sf_chunk_encode(int algorithm, const void *image, size_t height, size_t width,
                           int elem_bytes, void *out, size_t capacity, size_t *written);
SF_API int sf_chunk_decode(int algorithm, const void *chunk, size_t nbytes, size_t height,
                           size_t width, int elem_bytes, void *image);
/* The device decoder on its own: `chunk` (host memory) decoded into device
 * memory at `device_image`, rows `pitch_bytes` apart (at least width *
 * elem_bytes), one warp per LZ4 block. Waits for the decode. Returns as
 * sf_chunk_decode, or -3 for a device failure, a malformed LZ4 block found
 * on the device included. The batched engine's sf_engine_upload_chunk uses
 * the same decoder. */
SF_API int sf_chunk_decode_device(int algorithm, const void *chunk, size_t nbytes, size_t height,
                                  size_t width, int elem_bytes, void *device_image,
                                  size_t pitch_bytes);

/* ---- the reflection table: src/refl.hh:72-74 (refl::write) ------------- *
 *
 * Writes `spots` (with their pixels, `width` the frame width the labeller
 * was given) to `path` as a DIALS .refl file, byte-identical to the
 * reference's refl::write: the msgpack reflection table with bbox, flags
 * (Strong), id, intensity.sum.value / .variance, n_signal, panel, the
 * optional shoebox column (src/refl.cc:295-334, built on the device) and
 * xyzobs.px.value / .variance. Returns -1 for a null argument or width 0,
 * -4 for a spot whose pixels run past the list or lie outside its box or a
 * column past msgpack's 4 GB limit, -3 when the file cannot be written or
 * the device fails. */
typedef struct sf_refl_options {
  uint64_t panel;         /* one panel: 0 */
  int32_t id;             /* the experiment every row belongs to */
  int32_t shoeboxes;      /* write the shoebox column */
  const char *identifier; /* the experiment identifier; NULL or "" for none */
} sf_refl_options;

SF_API int sf_refl_write(const char *path, const sf_spot *spots, size_t nspots,
                         const sf_pixel *pixels, size_t npixels, size_t width,
                         const sf_refl_options *options);

/* ---- the batched engine ------------------------------------------------- *
 * No single reference counterpart: it replaces the reference's pattern of
 * -j host threads each calling gpu::find on one frame (src/find_spots.cc:
 * 472-537, src/dext_cuda.cu:585-728) with many frames -- equal or uneven
 * shapes -- thresholded per launch from `slots` device-resident arenas.
 * Results per frame are exactly sf_find_*'s. Uploads run on the engine's copy
 * stream and runs on its compute stream, ordered per slot by events, so
 * filling one slot overlaps computing another. */
typedef struct sf_engine sf_engine;

typedef struct sf_engine_config {
  int32_t seg_rows;        /* output rows per warp task; 0 = tuned or the cost model's */
  int32_t warps_per_block; /* 1, 2 or 4; 0 = tuned, else 2 (16-bit) or 1 (32-bit) */
  int32_t blocks_per_sm;   /* 0 = as many as fit */
  int32_t slots;           /* device arenas; 0 = 1 */
} sf_engine_config;
/* With seg_rows and warps_per_block both 0 (or no config), an engine whose
 * frames all have one shape reads the tuner file (sf_tune) for that shape on
 * this kind of device and uses its warps per block and task height; without
 * an entry it uses the cost model and 2 warps per block (1 for 32-bit
 * pixels). */

SF_API int sf_engine_create(int elem_bytes, int nframes, const int32_t *heights,
                            const int32_t *widths, const sf_engine_config *config,
                            sf_engine **out);
SF_API void sf_engine_destroy(sf_engine *engine);
/* seg_rows, warps_per_block, grid blocks, tasks, slots, device bytes, pitch
 * (elements), total list capacity (records). */
SF_API int sf_engine_info(sf_engine *engine, int64_t out8[8]);
/* Asynchronous copy of a row-major host frame (pinned for full speed) into
 * frame `frame` of slot `slot`. */
SF_API int sf_engine_upload(sf_engine *engine, int slot, int frame, const void *host_image);
/* The same from device memory with a row pitch in bytes. */
SF_API int sf_engine_upload_device(sf_engine *engine, int slot, int frame,
                                   const void *device_image, size_t pitch_bytes);
/* A compressed chunk (SF_CHUNK_*) of frame `frame`, decoded on the device
 * into the slot: only the chunk's bytes cross PCIe. The framing is checked
 * on the host first (-1 on a mismatch); a malformed LZ4 block found on the
 * device makes the next synchronize report -3. Keep `chunk` alive and
 * unchanged until the next synchronize. */
SF_API int sf_engine_upload_chunk(sf_engine *engine, int slot, int frame, const void *chunk,
                                  size_t nbytes, int algorithm);
/* `count` chunks at once, chunk k for frame frames[k] (frame k with a null
 * `frames`): the same as count sf_engine_upload_chunk calls, but the
 * framing of every chunk is checked on host threads in parallel first, and
 * a mismatch in any (-1) enqueues none. Extends the reference's per-frame
 * decompress::image (src/decompress.hh:14-31) to a batch. */
SF_API int sf_engine_upload_chunks(sf_engine *engine, int slot, size_t count, const int *frames,
                                   const void *const *chunks, const size_t *nbytes,
                                   int algorithm);
/* The detector's pixel mask for frame `frame` (height x width bytes,
 * nonzero = a pixel not to use, as NXmx /entry/instrument/detector/
 * pixel_mask marks them), stamped into the frame as the masked sentinel
 * before every run's threshold; NULL clears it. No reference counterpart:
 * the reference reads no pixel mask (its one documented omission) and relies
 * on the sentinels in the data. Waits for the device. */
SF_API int sf_engine_set_pixel_mask(sf_engine *engine, int frame, const uint8_t *mask);
/* Enqueue the threshold of every frame of a slot, after its uploads. */
SF_API int sf_engine_run(sf_engine *engine, int slot);
/* Replay each slot's run from a CUDA graph captured on first use. */
SF_API int sf_engine_use_graph(sf_engine *engine, int on);
/* Wait for all enqueued work; -3 if a kernel reported a failure. */
SF_API int sf_engine_synchronize(sf_engine *engine);
/* Per-frame signal counts of the slot's last run (waits for it). */
SF_API int sf_engine_counts(sf_engine *engine, int slot, uint32_t *counts);
/* One frame's list of the slot's last run, as sf_find_* returns it,
 * including -2 beyond the list capacity. */
SF_API int sf_engine_signal(sf_engine *engine, int slot, int frame, sf_signal_pixel *out,
                            size_t capacity, size_t *found);
/* Every frame's list of the slot's last run, back to back in frame order
 * into `out` (`capacity` records), with each frame's count in counts[frame]
 * (nframes entries): one count read and one copy per frame, waiting once.
 * -2 (counts still filled) if a frame overflowed its list or the lists do
 * not fit in `capacity`. The per-frame gpu::find of the reference
 * (src/dext_gpu.hh:141-158) over a whole batch. */
SF_API int sf_engine_signals(sf_engine *engine, int slot, sf_signal_pixel *out, size_t capacity,
                             uint32_t *counts);
/* CUDA events on the compute stream: record mark 0..15; elapsed ms between
 * two marks (waits for the later one). */
SF_API int sf_engine_record(sf_engine *engine, int mark);
SF_API int sf_engine_elapsed(sf_engine *engine, int from, int to, float *ms);
/* Per-run events around the threshold kernel, the placement and the
 * grouping (not with graph replay, which runs them as one). Turning it on
 * resets the totals; sf_engine_stage_totals gives runs, threshold ms,
 * placement ms and grouping ms, summed over the runs since. */
SF_API int sf_engine_profile(sf_engine *engine, int on);
SF_API int sf_engine_stage_totals(sf_engine *engine, double out4[4]);

/* ---- the autotuner ------------------------------------------------------ *
 * A timed search for one frame shape on the current device: warps per block
 * x threshold task height (threshold alone), then frames per launch
 * (threshold + placement + 3D grouping, two slots, as the engine overlaps
 * them), then threshold blocks per SM at that batch size (fewer than fit
 * leave room on every SM for the grouping running beside it), on the
 * caller's sample frames (host, row-major, cycled into the
 * batches), with CUDA events. The best tuple is appended to a tuner file,
 * keyed by pixel type, shape, SM count and device name; engines created
 * without explicit tuning read it. Results never depend on the tuning, only
 * the time does. The reference chooses its stage windows by measurement
 * the same way (src/dext_gpu.cc:18-37, tests/bench_dext_gpu.cc:242-337). */
typedef struct sf_tune_options {
  int32_t min_frames;   /* frames per launch tried: 0 = 8 */
  int32_t max_frames;   /* 0 = 32 */
  int32_t steps;        /* timed runs per candidate; 0 = 4 */
  int32_t grouping;     /* time the step with 3D grouping (1) or threshold only */
  int32_t use_cache;    /* return the tuner file's entry if there is one */
  int32_t reserved;
  uint64_t hbm_budget;  /* device bytes a candidate may use; 0 = half the free */
  const char *cache_path; /* NULL: $SPOTFINDER_TUNE_CACHE, else
                             $XDG_CACHE_HOME or ~/.cache /spotfinder_b200/tune.txt */
} sf_tune_options;

typedef struct sf_tune_result {
  int32_t frames_per_launch;
  int32_t warps_per_block;
  int32_t seg_rows;       /* for frames_per_launch frames */
  int32_t from_cache;     /* 1: read from the tuner file, no search */
  int32_t candidates;     /* configurations timed */
  int32_t blocks_per_sm;  /* threshold blocks per SM; 0 = as many as fit */
  double seg_ratio;       /* task height / the cost model's */
  double us_per_frame;    /* the chosen tuple's measured time per frame */
} sf_tune_result;

SF_API int sf_tune(int elem_bytes, int height, int width, const void *const *sample_frames,
                   int nsample, const sf_tune_options *options, sf_tune_result *out);
/* The tuning an engine runs with: frames per launch, warps per block, task
 * height, and whether they came from the tuner file. */
SF_API int sf_engine_tuning(sf_engine *engine, sf_tune_result *out);

/* Grouping inside every run. The batch's frames of one shape form one
 * series (several shapes: several series, e.g. concurrent detectors or
 * interleaved stills runs); each run's frames of a series are that series'
 * next consecutive frames, numbered from `first_frame`, and go through
 * sf_labeller's arithmetic on the device right after their threshold, in
 * the same stream (and graph), one labeller per series (the reference runs
 * one dials_spots::Labeller per series, src/find_spots.cc:460-636).
 * `carry_capacity` bounds the pixels a series holds open between runs (0:
 * twice its biggest frame's list capacity plus 2^20); going past it makes
 * the run report -3. Series are numbered in order of their first frame. */
SF_API int sf_engine_enable_grouping(sf_engine *engine, const sf_group_options *options,
                                     int64_t first_frame, uint64_t carry_capacity);
/* Number of series (0 before grouping is enabled) and a series' shape. */
SF_API int sf_engine_nseries(sf_engine *engine);
SF_API int sf_engine_series_shape(sf_engine *engine, int series, int32_t *height,
                                  int32_t *width);
/* Running totals over a series and the pixels it holds open (waits). */
SF_API int sf_engine_series_counts(sf_engine *engine, int series, sf_counts *out,
                                   uint64_t *live);
/* The spots, and their pixels, of a series finished by the last run
 * (waits); -2 and *n set if `capacity` is too small. Spot::first counts from
 * the series start. */
SF_API int sf_engine_series_spots(sf_engine *engine, int series, sf_spot *out, size_t capacity,
                                  size_t *n);
SF_API int sf_engine_series_pixels(sf_engine *engine, int series, sf_pixel *out,
                                   size_t capacity, size_t *n);
/* The same for series 0 (a batch of one shape). */
SF_API int sf_engine_group_counts(sf_engine *engine, sf_counts *out, uint64_t *live);
SF_API int sf_engine_spots(sf_engine *engine, sf_spot *out, size_t capacity, size_t *n);
SF_API int sf_engine_pixels(sf_engine *engine, sf_pixel *out, size_t capacity, size_t *n);
/* Close everything still open in every series (Labeller::finish); its
 * spots are then the last run's. */
SF_API int sf_engine_finish(sf_engine *engine);

/* ---- serving: live series on one device ---------------------------------- *
 *
 * Replaces the reference's series queue and -j worker pool (src/series.hh:
 * 66-83, src/queue.hh, src/find_spots.cc:472-591). Series are admitted while
 * the device-memory budget holds them; each gets its own engine (chunks
 * decoded on the device, threshold, placement and grouping per frame, graph
 * replay), streams and worker thread, so concurrent series overlap on the
 * device; frames are admitted into a series' slots as they free up, and the
 * open components stay on the device between frames. A series' results are
 * exactly what sf_find_* and sf_labeller_* give for it alone. */
typedef struct sf_server sf_server;
typedef struct sf_server_config {
  uint64_t hbm_budget; /* device bytes for series; 0: free memory less 2 GiB */
  int32_t slots;       /* frames in flight per series; 0: 3 */
  int32_t use_graph;   /* replay each series' runs from CUDA graphs */
} sf_server_config;

SF_API int sf_server_create(const sf_server_config *config, sf_server **out);
/* Stops every worker (after its queued frames) and frees everything. */
SF_API void sf_server_destroy(sf_server *server);
/* Admits a series of height x width frames of elem_bytes (2 or 4) pixels,
 * grouped with `options`, numbered from first_frame. -2 if its device memory
 * does not fit in what is left of the budget (retry after a close). Before
 * returning, an empty frame goes through every slot, so that the series'
 * first frames do not load kernels or instantiate graphs. */
SF_API int sf_server_open(sf_server *server, size_t height, size_t width, int elem_bytes,
                          const sf_group_options *options, int64_t first_frame, int *series);
/* The series' pixel mask (height x width bytes, nonzero = masked), as
 * sf_engine_set_pixel_mask; before the series' first frame. */
SF_API int sf_server_set_pixel_mask(sf_server *server, int series, const uint8_t *mask);
/* The series' next frame, as a chunk (SF_CHUNK_*), copied before return.
 * Waits up to timeout_us for a free slot; -2 if none freed: the frame is
 * dropped (its number is skipped, which closes the open components, as a
 * gap in the numbering does). Latencies count from entry. */
SF_API int sf_server_submit(sf_server *server, int series, const void *chunk, size_t nbytes,
                            int algorithm, int64_t timeout_us);
/* No more frames: processes what is queued, finishes the grouping and
 * returns the series' device memory to the budget. Results stay readable. */
SF_API int sf_server_close(sf_server *server, int series);
/* Grouping counts and [frames done, frames dropped, device bytes, closed]. */
SF_API int sf_server_stats(sf_server *server, int series, sf_counts *counts, uint64_t out4[4]);
/* The series' spots and their pixels so far (Spot::first from its start). */
SF_API int sf_server_spots(sf_server *server, int series, sf_spot *out, size_t capacity,
                           size_t *n);
SF_API int sf_server_pixels(sf_server *server, int series, sf_pixel *out, size_t capacity,
                            size_t *n);
/* Takes the spots (and their pixels) finished so far and still held, in
 * order, whole runs at a time while both arrays have room, and lets the
 * series forget them: a live consumer (writing a reflection table, say)
 * calls this as it goes, so the series does not keep every spot of a long
 * acquisition in host memory. A spot's `first` stays the offset of its
 * pixels in the series' whole pixel sequence, taken or not. -2 if the first
 * held run does not fit (nothing taken). sf_server_spots and
 * sf_server_pixels return what is still held. The reference's series
 * consumer writes the table at the end (src/find_spots.cc:636-716). */
SF_API int sf_server_take(sf_server *server, int series, sf_spot *spots, size_t spot_capacity,
                          size_t *nspots, sf_pixel *pixels, size_t pixel_capacity,
                          size_t *npixels);
/* Signal pixels per frame, by frame number (0 for a dropped frame). */
SF_API int sf_server_signal_counts(sf_server *server, int series, uint32_t *out,
                                   size_t capacity, size_t *n);
/* Latencies in microseconds: kind 0, per finished frame, submit to its
 * signal list placed on the device (frame-to-mask); kind 1, submit to its
 * grouping done; kind 2, per spot, submit of the spot's last frame to its
 * row on the host (frame-to-finalised-spot). */
SF_API int sf_server_latencies(sf_server *server, int series, int kind, double *out,
                               size_t capacity, size_t *n);

#ifdef __cplusplus
}
#endif
#endif /* SPOTFINDER_B200_H */
