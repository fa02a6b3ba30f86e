/* The oracle: a plain-C restatement of the reference spot finder's CPU path.
 *
 * TEST INFRASTRUCTURE ONLY. The parity tests, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this as the checker; the product never
 * links, loads or calls it.
 *
 * Parity is pinned: tests/test_oracle.py checks every function here against
 * golden vectors made by the reference's own code (tests/golden/, written by
 * tests/golden/make_golden.py from oracle/_ref/libref.so, which is compiled
 * from the reference sources by oracle/Makefile), and against libref.so
 * directly on seeded frames whenever that library is present.
 *
 * What is restated, and from where:
 *   sfo_dext_u16 / sfo_dext_u32   src/dext.cc:9-225 (threshold)
 *   sfo_lab_*                     src/dials_spots.cc:36-360 (grouping, spots)
 */
#ifndef SF_ORACLE_H
#define SF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* src/signal_pixel.hh:20-26, the 16-byte record. */
typedef struct {
  uint32_t index;
  uint32_t value;
  float background;
  uint16_t population;
  uint16_t reserved;
} sfo_signal_pixel;

/* src/dials_spots.hh:50-54. */
typedef struct {
  int32_t frame;
  uint32_t index;
  uint32_t value;
} sfo_pixel;

/* src/dials_spots.hh:57-79, byte for byte (104 bytes with padding). */
typedef struct {
  int32_t bbox[6];
  double position[3];
  double variance[3];
  double intensity;
  double intensity_variance;
  uint32_t n_signal;
  uint64_t first;
} sfo_spot;

/* 0 ok, -1 bad argument, -2 more signal than `capacity`. `found` is set to
 * the number of signal pixels either way (when the arguments are valid). */
int sfo_dext_u16(const uint16_t *image, size_t height, size_t width,
                 sfo_signal_pixel *out, size_t capacity, size_t *found);
int sfo_dext_u32(const uint32_t *image, size_t height, size_t width,
                 sfo_signal_pixel *out, size_t capacity, size_t *found);

typedef struct sfo_lab sfo_lab;

sfo_lab *sfo_lab_new(size_t height, size_t width, size_t min_spot_size,
                     size_t max_spot_size, double max_separation, int two_d);
void sfo_lab_free(sfo_lab *lab);
/* 0 ok; -1 refused (out of order, repeated frame, pixel off the frame or not
 * ascending), with the reason in sfo_lab_error(). A refused add changes
 * nothing. */
int sfo_lab_add(sfo_lab *lab, int64_t frame, const sfo_signal_pixel *signal,
                size_t n);
void sfo_lab_finish(sfo_lab *lab);
const char *sfo_lab_error(const sfo_lab *lab);
size_t sfo_lab_nspots(const sfo_lab *lab);
size_t sfo_lab_npixels(const sfo_lab *lab);
size_t sfo_lab_live(const sfo_lab *lab);
const sfo_spot *sfo_lab_spots(const sfo_lab *lab);
const sfo_pixel *sfo_lab_pixels(const sfo_lab *lab);
/* signal_pixels, groups, too_small, too_large, separated, accepted */
void sfo_lab_counts(const sfo_lab *lab, uint64_t *out6);

size_t sfo_spot_size(void);

#ifdef __cplusplus
}
#endif
#endif
