/* The oracle: a plain-C restatement of the reference spot finder's CPU path.
 * TEST INFRASTRUCTURE ONLY -- see sf_oracle.h for what is restated, from
 * where, and how it is pinned to the reference's own outputs.
 *
 * Compiled with -ffp-contract=off and no -march (oracle/Makefile) so that
 * every float and double operation below rounds once, in the order written,
 * as the reference's x86-64 build does.
 */
#include "sf_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Threshold (src/dext.cc:9-225)                                             */
/* ------------------------------------------------------------------------ */

/* Box sums over the window [i-r, i+r] x [j-r, j+r] clipped to the frame,
 * which is exactly what the reference's summed-area differences select
 * (src/dext.cc:69-88 for r = 3, :157-176 for r = 5). Computed here as a
 * vertical running sum followed by a horizontal one. All arithmetic is in
 * uint64; the 16-bit caller truncates its sum of squares to 32 bits, which
 * equals the reference's wrapping uint32 accumulation because that sum never
 * wraps 64 bits. */
static void box_sums(const uint64_t *in, uint64_t *tmp, uint64_t *out,
                     int32_t ny, int32_t nx, int32_t r) {
  for (int32_t j = 0; j < nx; j++) {
    uint64_t run = 0;
    /* run holds rows [i - r, i + r] clipped */
    for (int32_t i = 0; i < r && i < ny; i++)
      run += in[(size_t)i * nx + j];
    for (int32_t i = 0; i < ny; i++) {
      if (i + r < ny)
        run += in[(size_t)(i + r) * nx + j];
      if (i - r - 1 >= 0)
        run -= in[(size_t)(i - r - 1) * nx + j];
      tmp[(size_t)i * nx + j] = run;
    }
  }
  for (int32_t i = 0; i < ny; i++) {
    const uint64_t *row = tmp + (size_t)i * nx;
    uint64_t run = 0;
    for (int32_t j = 0; j < r && j < nx; j++)
      run += row[j];
    for (int32_t j = 0; j < nx; j++) {
      if (j + r < nx)
        run += row[j + r];
      if (j - r - 1 >= 0)
        run -= row[j - r - 1];
      out[(size_t)i * nx + j] = run;
    }
  }
}

/* The dispersion test of src/dext.cc:97-110, in float for 16-bit pixels.
 * Parenthesised to show the order the reference's expression evaluates in;
 * each operation rounds once. */
static int dispersion_f(uint32_t m_sum, uint32_t i_sum, uint32_t i2_sum) {
  if (m_sum < 2)
    return 0;
  const float m = (float)m_sum;
  const float s = (float)i_sum;
  const float s2 = (float)i2_sum;
  const float lhs = ((m * s2) - (s * s)) - (s * (m - 1.0f));
  const float rhs = (s * 6.0f) * sqrtf(2.0f * (m - 1.0f));
  return lhs > rhs;
}

/* The same in double for 32-bit pixels (real_t<uint32_t> is double). */
static int dispersion_d(uint64_t m_sum, uint64_t i_sum, uint64_t i2_sum) {
  if (m_sum < 2)
    return 0;
  const double m = (double)m_sum;
  const double s = (double)i_sum;
  const double s2 = (double)i2_sum;
  const double lhs = ((m * s2) - (s * s)) - (s * (m - 1.0));
  const double rhs = (s * 6.0) * sqrt(2.0 * (m - 1.0));
  return lhs > rhs;
}

/* One threshold over a frame whose pixels have been widened to uint64.
 * `wide` selects the 32-bit pixel rules (double arithmetic, 64-bit sums). */
static int dext_any(const uint64_t *px, size_t height, size_t width, int wide,
                    sfo_signal_pixel *out, size_t capacity, size_t *found) {
  const uint64_t masked = wide ? 0xfffffffeull : 0xfffeull;
  const int32_t ny = (int32_t)height, nx = (int32_t)width;
  const size_t n = height * width;

  uint64_t *a = malloc(n * sizeof(uint64_t));
  uint64_t *b = malloc(n * sizeof(uint64_t));
  uint64_t *c = malloc(n * sizeof(uint64_t));
  uint64_t *m_box = malloc(n * sizeof(uint64_t));
  uint64_t *s_box = malloc(n * sizeof(uint64_t));
  uint64_t *q_box = malloc(n * sizeof(uint64_t));
  uint8_t *scr0 = malloc(n);
  uint8_t *scr1 = malloc(n);
  if (!a || !b || !c || !m_box || !s_box || !q_box || !scr0 || !scr1) {
    free(a); free(b); free(c); free(m_box); free(s_box); free(q_box);
    free(scr0); free(scr1);
    return -3;
  }

  /* Pass 1: 7 x 7 count, sum and sum of squares of the valid pixels. */
  for (size_t k = 0; k < n; k++)
    a[k] = px[k] < masked ? 1u : 0u;
  box_sums(a, c, m_box, ny, nx, 3);
  for (size_t k = 0; k < n; k++)
    a[k] = px[k] < masked ? px[k] : 0u;
  box_sums(a, c, s_box, ny, nx, 3);
  for (size_t k = 0; k < n; k++) {
    const uint64_t p = px[k] < masked ? px[k] : 0u;
    a[k] = p * p; /* wraps mod 2^64 for 32-bit pixels, as uint64_t does */
  }
  box_sums(a, c, q_box, ny, nx, 3);

  /* The dispersion test; a masked pixel is 1 so the erode cannot grow
   * through it (src/dext.cc:113). */
  for (size_t k = 0; k < n; k++) {
    int signal;
    if (wide)
      signal = dispersion_d(m_box[k], s_box[k], q_box[k]);
    else
      signal = dispersion_f((uint32_t)m_box[k], (uint32_t)s_box[k],
                            (uint32_t)q_box[k]);
    scr0[k] = (signal || px[k] >= masked) ? 1 : 0;
  }

  /* 5 x 5 erode, neighbours off the frame ignored; masked pixels are 1
   * (src/dext.cc:117-142). */
  for (int32_t i = 0; i < ny; i++) {
    for (int32_t j = 0; j < nx; j++) {
      const size_t k = (size_t)i * nx + j;
      if (px[k] >= masked) {
        scr1[k] = 1;
        continue;
      }
      uint8_t keep = scr0[k];
      for (int32_t di = -2; di <= 2 && keep; di++) {
        const int32_t y = i + di;
        if (y < 0 || y >= ny)
          continue;
        for (int32_t dj = -2; dj <= 2; dj++) {
          const int32_t x = j + dj;
          if (x < 0 || x >= nx)
            continue;
          if (!scr0[(size_t)y * nx + x]) {
            keep = 0;
            break;
          }
        }
      }
      scr1[k] = keep;
    }
  }

  /* Pass 2: 11 x 11 count and sum over pixels that are valid and were not
   * kept by the erode (src/dext.cc:151-161). */
  for (size_t k = 0; k < n; k++)
    a[k] = (px[k] < masked && !scr1[k]) ? 1u : 0u;
  box_sums(a, c, m_box, ny, nx, 5);
  for (size_t k = 0; k < n; k++)
    a[k] = (px[k] < masked && !scr1[k]) ? px[k] : 0u;
  box_sums(a, c, s_box, ny, nx, 5);

  /* The Poisson test and the emit, in scan order (src/dext.cc:165-222). */
  size_t count = 0;
  for (size_t k = 0; k < n; k++) {
    const uint64_t p = px[k] >= masked ? 0u : px[k];
    if (!(p > 0 && scr1[k]))
      continue;
    int signal;
    float background;
    if (wide) {
      const double mean =
          m_box[k] >= 2 ? (double)s_box[k] / (double)m_box[k] : 0.0;
      signal = (double)p >= (mean + (3.0 * sqrt(mean)));
      background = (float)mean;
    } else {
      const float mean = (uint32_t)m_box[k] >= 2
                             ? (float)(uint32_t)s_box[k] /
                                   (float)(uint32_t)m_box[k]
                             : 0.0f;
      signal = (float)(uint32_t)p >= (mean + (3.0f * sqrtf(mean)));
      background = mean;
    }
    if (!signal)
      continue;
    if (count < capacity) {
      out[count].index = (uint32_t)k;
      out[count].value = (uint32_t)p;
      out[count].background = background;
      out[count].population = (uint16_t)m_box[k];
      out[count].reserved = 0;
    }
    count++;
  }
  *found = count;

  free(a); free(b); free(c); free(m_box); free(s_box); free(q_box);
  free(scr0); free(scr1);
  return count > capacity ? -2 : 0;
}

static int check_dims(const void *image, size_t height, size_t width) {
  if (image == NULL || height == 0 || width == 0)
    return -1;
  if (height > (size_t)INT32_MAX / width)
    return -1;
  if (height * width > (size_t)INT32_MAX)
    return -1;
  return 0;
}

int sfo_dext_u16(const uint16_t *image, size_t height, size_t width,
                 sfo_signal_pixel *out, size_t capacity, size_t *found) {
  *found = 0;
  if (check_dims(image, height, width) != 0)
    return -1;
  const size_t n = height * width;
  uint64_t *px = malloc(n * sizeof(uint64_t));
  if (!px)
    return -3;
  for (size_t k = 0; k < n; k++)
    px[k] = image[k];
  const int status = dext_any(px, height, width, 0, out, capacity, found);
  free(px);
  return status;
}

int sfo_dext_u32(const uint32_t *image, size_t height, size_t width,
                 sfo_signal_pixel *out, size_t capacity, size_t *found) {
  *found = 0;
  if (check_dims(image, height, width) != 0)
    return -1;
  const size_t n = height * width;
  uint64_t *px = malloc(n * sizeof(uint64_t));
  if (!px)
    return -3;
  for (size_t k = 0; k < n; k++)
    px[k] = image[k];
  const int status = dext_any(px, height, width, 1, out, capacity, found);
  free(px);
  return status;
}

/* ------------------------------------------------------------------------ */
/* Grouping and spots (src/dials_spots.cc:36-360)                            */
/* ------------------------------------------------------------------------ */

struct sfo_lab {
  size_t height, width;
  size_t min_size, max_size;
  double max_separation;
  int two_d;

  sfo_pixel *live;
  uint32_t *parent;
  size_t nlive, cap_live;
  size_t previous; /* where the last frame's pixels start in live */
  int64_t last_frame;
  int started;

  sfo_spot *spots;
  size_t nspots, cap_spots;
  sfo_pixel *kept;
  size_t nkept, cap_kept;
  uint64_t counts[6];
  char error[160];
};

#define GROW(ptr, cap, need)                                                   \
  do {                                                                         \
    if ((need) > (cap)) {                                                      \
      size_t grown = (cap) ? (cap) : 64;                                       \
      while (grown < (need))                                                   \
        grown *= 2;                                                            \
      (ptr) = realloc((ptr), grown * sizeof(*(ptr)));                          \
      (cap) = grown;                                                           \
    }                                                                          \
  } while (0)

sfo_lab *sfo_lab_new(size_t height, size_t width, size_t min_spot_size,
                     size_t max_spot_size, double max_separation, int two_d) {
  if (height == 0 || width == 0 || max_spot_size < min_spot_size ||
      min_spot_size == 0)
    return NULL;
  sfo_lab *lab = calloc(1, sizeof(sfo_lab));
  lab->height = height;
  lab->width = width;
  lab->min_size = min_spot_size;
  lab->max_size = max_spot_size;
  lab->max_separation = max_separation;
  lab->two_d = two_d;
  return lab;
}

void sfo_lab_free(sfo_lab *lab) {
  if (!lab)
    return;
  free(lab->live);
  free(lab->parent);
  free(lab->spots);
  free(lab->kept);
  free(lab);
}

/* Path halving; roots are the lowest index of their component. */
static uint32_t uf_find(uint32_t *parent, uint32_t i) {
  while (parent[i] != i) {
    parent[i] = parent[parent[i]];
    i = parent[i];
  }
  return i;
}

static void uf_merge(uint32_t *parent, uint32_t a, uint32_t b) {
  const uint32_t ra = uf_find(parent, a), rb = uf_find(parent, b);
  if (ra == rb)
    return;
  if (ra < rb)
    parent[rb] = ra;
  else
    parent[ra] = rb;
}

/* The per-component pass (src/dials_spots.cc:221-360): filters, bbox, sums
 * in member order, centroid, variance, and the peak-centroid filter. The
 * floating-point steps are written in the order the reference performs them,
 * which is what makes the doubles identical. */
static void emit(sfo_lab *lab, const uint32_t *members, size_t n) {
  const double pixel_variance = 1.0 / 12.0;
  lab->counts[1]++;
  if (n < lab->min_size) {
    lab->counts[2]++;
    return;
  }
  if (n > lab->max_size) {
    lab->counts[3]++;
    return;
  }

  sfo_spot spot;
  memset(&spot, 0, sizeof(spot));
  spot.n_signal = (uint32_t)n;

  double sum = 0.0, sum_sq = 0.0, weighted[3] = {0.0, 0.0, 0.0};
  int32_t x0 = 0, x1 = 0, y0 = 0, y1 = 0, z0 = 0, z1 = 0;
  uint32_t peak_value = 0;
  double peak[3] = {0.0, 0.0, 0.0};
  const size_t width = lab->width;

  for (size_t k = 0; k < n; k++) {
    const sfo_pixel *p = &lab->live[members[k]];
    const int32_t x = (int32_t)(p->index % width);
    const int32_t y = (int32_t)(p->index / width);
    const int32_t z = p->frame;
    if (k == 0) {
      x0 = x; x1 = x + 1; y0 = y; y1 = y + 1; z0 = z; z1 = z + 1;
    } else {
      if (x < x0) x0 = x;
      if (x + 1 > x1) x1 = x + 1;
      if (y < y0) y0 = y;
      if (y + 1 > y1) y1 = y + 1;
      if (z < z0) z0 = z;
      if (z + 1 > z1) z1 = z + 1;
    }
    const double value = (double)p->value;
    const double pos[3] = {(double)x + 0.5, (double)y + 0.5, (double)z + 0.5};
    sum = sum + value;
    sum_sq = sum_sq + (value * value);
    for (int axis = 0; axis < 3; axis++)
      weighted[axis] = weighted[axis] + (value * pos[axis]);
    if (p->value > peak_value) {
      peak_value = p->value;
      peak[0] = pos[0]; peak[1] = pos[1]; peak[2] = pos[2];
    }
  }

  spot.bbox[0] = x0; spot.bbox[1] = x1;
  spot.bbox[2] = y0; spot.bbox[3] = y1;
  spot.bbox[4] = z0; spot.bbox[5] = z1;
  spot.intensity = sum;
  spot.intensity_variance = sum;

  if (sum > 0.0) {
    for (int axis = 0; axis < 3; axis++)
      spot.position[axis] = weighted[axis] / sum;
    double delta_sq[3] = {0.0, 0.0, 0.0};
    for (size_t k = 0; k < n; k++) {
      const sfo_pixel *p = &lab->live[members[k]];
      const double value = (double)p->value;
      const double pos[3] = {(double)(p->index % width) + 0.5,
                             (double)(p->index / width) + 0.5,
                             (double)p->frame + 0.5};
      for (int axis = 0; axis < 3; axis++) {
        const double delta = pos[axis] - spot.position[axis];
        delta_sq[axis] = delta_sq[axis] + ((value * delta) * delta);
      }
    }
    if ((sum * sum) > sum_sq) {
      for (int axis = 0; axis < 3; axis++) {
        const double variance =
            (delta_sq[axis] * sum) / ((sum * sum) - sum_sq);
        spot.variance[axis] = (variance / sum) + pixel_variance;
      }
    } else {
      for (int axis = 0; axis < 3; axis++)
        spot.variance[axis] = pixel_variance;
    }
    if (spot.bbox[5] == spot.bbox[4] + 1)
      spot.position[2] = (double)spot.bbox[4] + 0.5;
  } else {
    spot.position[0] = (double)(spot.bbox[1] + spot.bbox[0]) / 2.0;
    spot.position[1] = (double)(spot.bbox[3] + spot.bbox[2]) / 2.0;
    spot.position[2] = (double)(spot.bbox[5] + spot.bbox[4]) / 2.0;
  }

  if (lab->max_separation > 0.0) {
    const double dx = peak[0] - spot.position[0];
    const double dy = peak[1] - spot.position[1];
    const double dz = peak[2] - spot.position[2];
    if (sqrt(((dx * dx) + (dy * dy)) + (dz * dz)) > lab->max_separation) {
      lab->counts[4]++;
      return;
    }
  }

  spot.first = lab->nkept;
  GROW(lab->kept, lab->cap_kept, lab->nkept + n);
  for (size_t k = 0; k < n; k++)
    lab->kept[lab->nkept++] = lab->live[members[k]];
  GROW(lab->spots, lab->cap_spots, lab->nspots + 1);
  lab->spots[lab->nspots++] = spot;
  lab->counts[5]++;
}

/* Close every component with no pixel on keep_frame, emitting in order of
 * first pixel, and compact the rest in (frame, index) order, re-rooted at
 * their first pixel (src/dials_spots.cc:153-219). */
static void close_components(sfo_lab *lab, int64_t keep_frame) {
  const size_t n = lab->nlive;
  if (n == 0) {
    lab->previous = 0;
    return;
  }
  uint32_t *comp = malloc(n * sizeof(uint32_t));
  uint32_t *label = malloc(n * sizeof(uint32_t));
  for (size_t i = 0; i < n; i++)
    label[i] = UINT32_MAX;
  uint32_t components = 0;
  for (size_t i = 0; i < n; i++) {
    const uint32_t r = uf_find(lab->parent, (uint32_t)i);
    if (label[r] == UINT32_MAX)
      label[r] = components++;
    comp[i] = label[r];
  }
  uint32_t *offset = calloc((size_t)components + 1, sizeof(uint32_t));
  uint32_t *cursor = malloc(((size_t)components + 1) * sizeof(uint32_t));
  uint32_t *member = malloc(n * sizeof(uint32_t));
  char *open = calloc(components ? components : 1, 1);
  for (size_t i = 0; i < n; i++)
    offset[comp[i] + 1]++;
  for (uint32_t c = 0; c < components; c++)
    offset[c + 1] += offset[c];
  for (uint32_t c = 0; c < components; c++)
    cursor[c] = offset[c];
  for (size_t i = 0; i < n; i++)
    member[cursor[comp[i]]++] = (uint32_t)i;
  for (size_t i = 0; i < n; i++)
    if (lab->live[i].frame == keep_frame)
      open[comp[i]] = 1;
  for (uint32_t c = 0; c < components; c++)
    if (!open[c])
      emit(lab, member + offset[c], offset[c + 1] - offset[c]);

  for (uint32_t c = 0; c < components; c++)
    cursor[c] = UINT32_MAX;
  size_t write = 0;
  for (size_t i = 0; i < n; i++) {
    const uint32_t c = comp[i];
    if (!open[c])
      continue;
    if (cursor[c] == UINT32_MAX)
      cursor[c] = (uint32_t)write;
    lab->live[write] = lab->live[i];
    lab->parent[write] = cursor[c];
    write++;
  }
  lab->nlive = write;
  lab->previous = write;
  while (lab->previous > 0 && lab->live[lab->previous - 1].frame == keep_frame)
    lab->previous--;
  free(comp); free(label); free(offset); free(cursor); free(member); free(open);
}

int sfo_lab_add(sfo_lab *lab, int64_t frame, const sfo_signal_pixel *signal,
                size_t n) {
  if (lab->started && frame <= lab->last_frame) {
    snprintf(lab->error, sizeof(lab->error),
             "frame %lld arrived after frame %lld", (long long)frame,
             (long long)lab->last_frame);
    return -1;
  }
  const size_t pixels = lab->height * lab->width;
  for (size_t i = 0; i < n; i++) {
    if (signal[i].index >= pixels) {
      snprintf(lab->error, sizeof(lab->error),
               "signal pixel %u is off the end of the frame", signal[i].index);
      return -1;
    }
    if (i > 0 && signal[i].index <= signal[i - 1].index) {
      snprintf(lab->error, sizeof(lab->error),
               "signal pixels are not ascending by index");
      return -1;
    }
  }
  if (lab->nlive + n > (size_t)UINT32_MAX) {
    snprintf(lab->error, sizeof(lab->error), "too many pixels held open");
    return -1;
  }

  if (lab->started && frame != lab->last_frame + 1)
    close_components(lab, frame);

  const size_t base = lab->nlive;
  GROW(lab->live, lab->cap_live, base + n);
  {
    size_t cap = lab->cap_live;
    lab->parent = realloc(lab->parent, (cap ? cap : 1) * sizeof(uint32_t));
  }
  for (size_t i = 0; i < n; i++) {
    lab->live[base + i].frame = (int32_t)frame;
    lab->live[base + i].index = signal[i].index;
    lab->live[base + i].value = signal[i].value;
    lab->parent[base + i] = (uint32_t)(base + i);
  }
  lab->nlive = base + n;
  lab->counts[0] += n;
  const size_t end = lab->nlive;
  const uint32_t columns = (uint32_t)lab->width;
  sfo_pixel *live = lab->live;

  /* left, within the row */
  for (size_t i = base + 1; i < end; i++)
    if (live[i].index % columns != 0 && live[i].index == live[i - 1].index + 1)
      uf_merge(lab->parent, (uint32_t)i, (uint32_t)(i - 1));
  /* up, within the frame */
  for (size_t i = base, up = base; i < end; i++) {
    if (live[i].index < columns)
      continue;
    const uint32_t target = live[i].index - columns;
    while (up < i && live[up].index < target)
      up++;
    if (up < i && live[up].index == target)
      uf_merge(lab->parent, (uint32_t)i, (uint32_t)up);
  }
  /* the same pixel on the previous frame */
  if (!lab->two_d && lab->started && lab->last_frame + 1 == frame &&
      lab->previous < base) {
    for (size_t i = base, back = lab->previous; i < end; i++) {
      const uint32_t target = live[i].index;
      while (back < base && live[back].index < target)
        back++;
      if (back < base && live[back].index == target)
        uf_merge(lab->parent, (uint32_t)i, (uint32_t)back);
    }
  }
  lab->started = 1;
  lab->last_frame = frame;
  close_components(lab, lab->two_d ? frame + 1 : frame);
  return 0;
}

void sfo_lab_finish(sfo_lab *lab) {
  if (!lab->started)
    return;
  close_components(lab, lab->last_frame + 1);
}

const char *sfo_lab_error(const sfo_lab *lab) { return lab->error; }
size_t sfo_lab_nspots(const sfo_lab *lab) { return lab->nspots; }
size_t sfo_lab_npixels(const sfo_lab *lab) { return lab->nkept; }
size_t sfo_lab_live(const sfo_lab *lab) { return lab->nlive; }
const sfo_spot *sfo_lab_spots(const sfo_lab *lab) { return lab->spots; }
const sfo_pixel *sfo_lab_pixels(const sfo_lab *lab) { return lab->kept; }
void sfo_lab_counts(const sfo_lab *lab, uint64_t *out6) {
  memcpy(out6, lab->counts, sizeof(lab->counts));
}
size_t sfo_spot_size(void) { return sizeof(sfo_spot); }
