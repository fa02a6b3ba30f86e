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
 * these functions; INTEGRATION.md shows the bindings.
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

/* ---- stage profiling: src/dext_gpu.hh:79-116 ---------------------------- *
 * When on, sf_find_* records, for the calling thread, milliseconds spent in:
 * [0] upload (host to device), [1] the fused threshold kernel, [2] 0 (the
 * erode is fused into [1]), [3] the ordered compaction, [4] reading the list
 * back, [5] 0 (no host sort is needed). */
SF_API void sf_profile_stages(int on);
SF_API int sf_profile_stages_enabled(void);
SF_API void sf_last_stage_times(double out6[6]);

#ifdef __cplusplus
}
#endif
#endif /* SPOTFINDER_B200_H */
