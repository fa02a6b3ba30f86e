// 3D / 2D six-connected grouping and the spot pass on the device, with the
// streaming semantics of the reference's Labeller (src/dials_spots.cc:
// 57-219) and its per-component arithmetic (src/dials_spots.cc:221-360).
//
// One batch (enqueue) is a fixed sequence of launches whose sizes all live
// in device memory, so a batch can follow the threshold on the same stream
// and be captured in the same CUDA graph:
//
//   setup     frame segments of the live set: the carry's last frame, then
//             the batch frames; live size n
//   gather    the batch's signal lists appended after the carried pixels,
//             so the live set is in (frame, index) order; per-root fields
//             cleared
//   link      left, up and previous-frame neighbours joined by a lock-free
//             union-find that links toward the lower position, so a root is
//             its component's first pixel in (frame, index) order
//   flatten   root of every pixel; component size and last frame
//   mark      finished roots (no pixel on the batch's last frame) as a
//             bitmap, with a count per 32-position word
//   scan      of the counts
//   compact   the finished roots, in position order
//   count     per 32 roots of that list, how many close on each frame
//             (last-frame bucket)
//   scan      of those counts, bucket-major: the reference's emission order
//             is (last frame, first pixel), which is exactly bucket then
//             position
//   rank      each finished component's emission rank; size filters
//   scan      member offsets of the components that pass the size filters
//   scatter   members, in any order; the open pixels (their component is
//             not finished) as a bitmap with a count per 32 positions
//   accept    per component: members sorted by position (so (frame, index)
//             order), then the FP64 pass in that order, peak-centroid
//             filter
//   scan      output rows and pixel offsets of the accepted spots
//   write     spots and their pixels
//   scan      of the open counts
//   carry     the open components' pixels compacted, in order, into
//             the other live buffer and re-rooted at their first pixel
//   finalize  running counts and the carry for the next batch
//
// Every loop here walks a bounded range; union-find paths strictly decrease
// in position, so no loop depends on another thread making progress.

#include <climits>
#include <cstddef>

#include "sf_label.hh"

namespace sf {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kNone = 0xffffffffu;
constexpr int kThreads = 256;
// Components up to kSmallCap members take lab_accept's launch with small
// per-warp buffers (many warps per SM); the larger ones are listed by
// lab_rank in two lists, up to kMidCap members and beyond, and taken by
// launches with larger buffers.
constexpr uint32_t kSmallCap = 256;
constexpr uint32_t kMidCap = 512;

// Quotients by one divisor fixed for a whole launch (the frame width), by a
// multiply-high and two shifts: Granlund and Montgomery, "Division by
// invariant integers using multiplication" (PLDI 1994), the form with a
// 33-bit multiplier whose top bit is folded into an add. Exact for every
// 32-bit dividend and divisor >= 1.
struct DivU32 {
  uint32_t d, m, s1, s2;
  static DivU32 of(uint32_t d) {
    uint32_t l = 0;
    while (l < 32 && (1ull << l) < d)
      l++; // ceil(log2 d)
    DivU32 v;
    v.d = d;
    v.m = static_cast<uint32_t>((((1ull << l) - d) << 32) / d + 1);
    v.s1 = l < 1 ? l : 1;
    v.s2 = l > 1 ? l - 1 : 0;
    return v;
  }
  __device__ __forceinline__ uint32_t quo(uint32_t n) const {
    const uint32_t t = __umulhi(m, n);
    return (t + ((n - t) >> s1)) >> s2;
  }
  __device__ __forceinline__ uint32_t rem(uint32_t n) const { return n - quo(n) * d; }
};

struct LabArgs {
  int32_t width;
  DivU32 wdiv; // division by the width
  int32_t nframes;
  int32_t close_all;
  int32_t two_d;
  uint64_t min_size, max_size;
  double max_sep;
  uint64_t live_cap, spot_cap;
  const SignalPixel *lists;
  const uint64_t *offs;
  const uint32_t *counts;
  const int32_t *count_map; // frame f's count is counts[count_map[f]]; null: counts[f]
  const uint32_t *caps;
  int32_t *fr;
  uint32_t *ix, *val, *par;
  int32_t *nfr;
  uint32_t *nix, *nval, *npar;
  uint32_t *root, *size;
  int32_t *lastz;
  uint32_t *rank_of_root, *cursor;
  uint32_t *bits, *bcnt; // finished-root bitmap; word counts, then bucket counts
  uint32_t *flist;       // the finished roots in position order
  uint32_t *comp_root, *msize, *members;
  uint64_t *mpk;
  uint4 *runs; // per batch: lab_link's entries, see lab_gather
  uint32_t *run_starts; // bit p & 31 of word p >> 5: position p starts a run
  Spot *spot_tmp;
  Pixel *pix_tmp;
  uint64_t *pack;
  uint32_t *obits, *ocnt; // open pixels: bitmap and (scanned) count per 32 positions
  uint32_t *big; // ranks of the kept components with more than kMidCap members
  uint32_t *mid; // ... with more than kSmallCap and at most kMidCap
  Spot *spots;
  Pixel *kept;
  uint64_t *seg_start, *seg_count;
  int64_t *seg_z;
  uint32_t *tab;       // block tables of the batch frames, nblk each
  uint32_t *carry_tab; // block table of the carry's last frame
  uint64_t nblk;
  LabelScalars *sc;
};

__device__ __forceinline__ uint64_t gtid() {
  return static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
}
__device__ __forceinline__ uint64_t gstride() {
  return static_cast<uint64_t>(gridDim.x) * blockDim.x;
}

// The root of x when no link can happen any more: read only.
__device__ __forceinline__ uint32_t uf_root(const uint32_t *parent, uint32_t x) {
  while (true) {
    const uint32_t px = parent[x];
    if (px == x)
      return x;
    x = px;
  }
}

// Union-find on positions. Parents only ever point to lower positions.
// Path halving: each step reads a parent and a grandparent, points the node
// at the grandparent (still an ancestor, still lower) and moves there, so a
// step covers two levels; a grandparent equal to its parent is the root.
// Returns the root of x, given x's parent px already read.
__device__ __forceinline__ uint32_t uf_find_from(volatile uint32_t *p, uint32_t x, uint32_t px) {
  while (px != x) {
    const uint32_t gp = p[px];
    if (gp == px)
      return px;
    p[x] = gp;
    x = gp;
    px = p[x];
  }
  return x;
}

// Joins the trees of a and b; returns the merged tree's root as it was at
// the link (an ancestor of both from then on), so a caller uniting one
// element with several others can pass it back as `a`.
__device__ __forceinline__ uint32_t uf_unite(uint32_t *parent, uint32_t a, uint32_t b) {
  volatile uint32_t *p = parent;
  while (true) {
    // both parents' reads in flight before either walk
    const uint32_t pa = p[a], pb = p[b];
    a = uf_find_from(p, a, pa);
    b = uf_find_from(p, b, pb);
    if (a == b)
      return a;
    if (a < b) {
      const uint32_t t = a;
      a = b;
      b = t;
    }
    // Link the higher root under the lower one, if it is still a root.
    const uint32_t old = atomicCAS(&parent[a], a, b);
    if (old == a)
      return b;
    a = old;
  }
}

__device__ __forceinline__ int segment_of(const uint64_t *seg_start, int nseg, uint64_t g) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seg_start[mid] <= g)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int bucket_of(const int64_t *seg_z, int nseg, int64_t z) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seg_z[mid] <= z)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int64_t last_batch_frame(const LabArgs &a) {
  return a.sc->batch_z0 + a.nframes - 1;
}

// A root whose component is finished by this batch.
__device__ __forceinline__ bool finished_root(const LabArgs &a, uint64_t g, uint64_t n) {
  if (g >= n || a.root[g] != g)
    return false;
  if (a.close_all || a.two_d || a.nframes == 0)
    return true;
  return static_cast<int64_t>(a.lastz[g]) < last_batch_frame(a);
}

// --------------------------------------------------------------------------

__global__ void lab_setup(LabArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0)
    return;
  LabelScalars *sc = a.sc;
  const uint64_t carry = sc->carry_n;
  int nseg = 0;
  if (carry > 0) {
    a.seg_z[0] = sc->carry_last_z;
    a.seg_start[0] = sc->carry_last_start;
    a.seg_count[0] = carry - sc->carry_last_start;
    nseg = 1;
  }
  uint64_t pos = carry;
  for (int f = 0; f < a.nframes; f++) {
    uint32_t c = a.counts[a.count_map ? a.count_map[f] : f];
    if (c > a.caps[f]) // an over-dense frame: its list holds only this many
      c = a.caps[f];
    if (pos + c > a.live_cap) {
      sc->status = kLabelLiveOverflow;
      c = static_cast<uint32_t>(a.live_cap - pos);
    }
    a.seg_z[nseg] = sc->batch_z0 + f;
    a.seg_start[nseg] = pos;
    a.seg_count[nseg] = c;
    pos += c;
    nseg++;
  }
  if (nseg == 0) { // nothing held and nothing added: one empty segment
    a.seg_z[0] = sc->batch_z0;
    a.seg_start[0] = 0;
    a.seg_count[0] = 0;
    nseg = 1;
  }
  sc->n = pos;
  sc->nw = (pos + 31) / 32;
  sc->nseg = nseg;
  sc->signal_pixels += pos - carry;
  sc->closed32 = sc->open32 = 0;
  sc->runs_n = 0;
  sc->big_n = 0;
  sc->mid_n = 0;
  sc->link_next = sc->accept_next = sc->big_next = sc->mid_next = 0;
  sc->members_pack = 0;
  sc->accepted_pack = 0;
}

// Block tables. For a frame's list, entry b is the position (within the
// list) of the first pixel whose index is at least 64 b, or kNone when there
// is none; so the pixels of block b are the positions [tab[b], tab[b+1]).
// A lookup of one index is then a scan of about two entries.
constexpr int kBlockShift = 6;

// Frame segments lab_gather and lab_link keep in shared memory (batches of
// up to 128 frames; longer ones read them from global memory).
constexpr int kMaxSegments = 129;

__device__ __forceinline__ const uint32_t *table_of(const LabArgs &a, int s, int first_batch_seg) {
  return s < first_batch_seg ? a.carry_tab : a.tab + static_cast<uint64_t>(s - first_batch_seg) * a.nblk;
}

// The new pixels' lists are copied after the carried pixels; per-root
// fields are cleared. Each new pixel's parent is set to the first pixel of
// its horizontal run (left neighbours, src/dials_spots.cc:106-110) within its
// 32-aligned chunk of positions, found with one ballot, so that the trees
// start one level deep; a run that enters a chunk from the previous one is
// joined by lab_link at the chunk's first position.
__global__ void __launch_bounds__(kThreads) lab_gather(LabArgs a) {
  LabelScalars *sc = a.sc;
  const uint64_t n = sc->n, carry = sc->carry_n;
  const int nseg = static_cast<int>(sc->nseg);
  const int first_batch_seg = carry > 0 ? 1 : 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ uint32_t warp_count[kThreads / 32];
  __shared__ uint32_t block_at;
  // the segments' starts and frame numbers, for every pixel's lookup
  __shared__ uint64_t sh_start[kMaxSegments];
  __shared__ int64_t sh_z[kMaxSegments];
  const bool in_shared = nseg <= kMaxSegments;
  if (in_shared)
    for (int k = threadIdx.x; k < nseg; k += blockDim.x) {
      sh_start[k] = a.seg_start[k];
      sh_z[k] = a.seg_z[k];
    }
  __syncthreads();
  const uint64_t *seg_start = in_shared ? sh_start : a.seg_start;
  const int64_t *seg_z = in_shared ? sh_z : a.seg_z;
  // block-uniform trip count: the run list is appended to once per block
  for (uint64_t block_base = static_cast<uint64_t>(blockIdx.x) * kThreads; block_base < n;
       block_base += static_cast<uint64_t>(gridDim.x) * kThreads) {
    const uint64_t base = block_base + static_cast<uint64_t>(warp) * 32;
    const uint64_t g = base + lane;
    bool left = false;
    int seg = 0;       // a new pixel's frame segment
    uint32_t pidx = 0; // and its index, for the work list
    if (g < n) {
      a.size[g] = 0;
      a.lastz[g] = INT_MIN;
      a.rank_of_root[g] = kNone;
      a.cursor[g] = 0;
      if (g >= carry) {
        const int s = segment_of(seg_start, nseg, g);
        seg = s;
        const int f = s - first_batch_seg;
        const uint64_t i = g - seg_start[s];
        const SignalPixel *list = a.lists + a.offs[f];
        const SignalPixel px = list[i];
        a.fr[g] = static_cast<int32_t>(seg_z[s]);
        a.ix[g] = px.index;
        a.val[g] = px.value;
        pidx = px.index;
        const uint32_t prev = i == 0 ? 0u : list[i - 1].index;
        left = i > 0 && prev + 1 == px.index && a.wdiv.rem(px.index) != 0;
        // This pixel is the first of every block from the one after the
        // previous pixel's up to its own.
        uint32_t *tab = a.tab + static_cast<uint64_t>(f) * a.nblk;
        const uint64_t b1 = px.index >> kBlockShift;
        const uint64_t b0 = i == 0 ? 0 : (prev >> kBlockShift) + 1;
        for (uint64_t b = b0; b <= b1; b++)
          tab[b] = static_cast<uint32_t>(i);
      } else if (g > sc->carry_last_start) {
        // the carried last frame, which the first batch frame links to
        const uint32_t v = a.ix[g];
        left = a.ix[g - 1] + 1 == v && a.wdiv.rem(v) != 0;
      }
    }
    const uint32_t linked = __ballot_sync(kFull, left);
    if (lane == 0 && base < n)
      a.run_starts[base >> 5] = ~linked;
    const bool mine = g < n && g >= carry;
    if (mine) {
      // the run's first lane in this chunk: the highest lane at or below
      // this one that is not joined to its left neighbour
      const uint32_t starts = ~linked & (0xffffffffu >> (31 - lane));
      const int first = starts ? 31 - __clz(starts) : 0;
      a.par[g] = static_cast<uint32_t>(base + first);
    }
    // lab_link's work list: one entry per piece of a run within a chunk --
    // its first position, its first pixel's index, its length, whether it
    // continues a run from the chunk before (lane 0 joined to its left
    // neighbour) and its frame segment, so that lab_link starts from one
    // 16-byte load
    const bool boundary = left && lane == 0;
    const bool entry = mine && (!left || boundary);
    const uint32_t want = __ballot_sync(kFull, entry);
    // pieces end at the next piece, at a lane that is not ours, or at the
    // chunk's end
    const uint32_t stops = want | ~__ballot_sync(kFull, mine);
    const uint32_t after = lane == 31 ? 0u : stops & (0xfffffffeu << lane);
    const uint32_t len = (after ? __ffs(after) - 1 : 32) - lane;
    if (lane == 0)
      warp_count[warp] = __popc(want);
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t total = 0;
      for (int w = 0; w < kThreads / 32; w++) {
        const uint32_t c = warp_count[w];
        warp_count[w] = total;
        total += c;
      }
      block_at = total ? atomicAdd(&sc->runs_n, total) : 0u;
    }
    __syncthreads();
    if (entry)
      a.runs[block_at + warp_count[warp] + __popc(want & ((1u << lane) - 1u))] =
          make_uint4(static_cast<uint32_t>(g), pidx,
                     len | (boundary ? 0x40u : 0u) | (static_cast<uint32_t>(seg) << 8), 0u);
    __syncthreads();
  }
}

// First position (relative to the list at s0) whose index is at least t,
// or count, given the block table's entries p for t's block and p1 for the
// next block (loaded by the caller, so that independent lookups overlap);
// *iq gets that position's index (not set at count), which the caller's
// next step needs. Indices rise by at least one a position, so position
// p + (t mod 64) holds an index of at least t, and p1 one above t's block:
// the answer lies in [p, min(p + t mod 64, p1)]. When that first bound
// holds t itself (a dense stretch: every index from the block's start is
// present) it is the answer; otherwise a binary search of the range.
__device__ __forceinline__ uint64_t first_at_least(const LabArgs &a, uint32_t p, uint32_t p1,
                                                   uint64_t s0, uint64_t count, uint32_t t,
                                                   uint32_t *iq) {
  if (p == kNone)
    return count;
  uint64_t lo = p;
  uint64_t hi = min(lo + (t & ((1u << kBlockShift) - 1u)), count);
  if (p1 != kNone)
    hi = min(hi, static_cast<uint64_t>(p1));
  if (hi < count) {
    const uint32_t v = a.ix[s0 + hi];
    *iq = v;
    if (v == t)
      return hi;
  }
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    const uint32_t v = a.ix[s0 + mid];
    if (v >= t) {
      hi = mid;
      *iq = v;
    } else {
      lo = mid + 1;
    }
  }
  return hi;
}

// Unites the tree of `ra` (the run whose first pixel is g, or an ancestor)
// with every run of the list at s0 that has a pixel with an index in
// [lo, hi] (one row's span, at most 32 indices), q being the first position
// at or past lo: the run holding that pixel, then the later run starts,
// found in the run-start bitmap; returns the merged root.
__device__ __forceinline__ uint32_t unite_overlaps(const LabArgs &a, uint32_t ra, uint64_t q,
                                                   uint32_t iq, uint64_t s0, uint64_t count,
                                                   uint32_t hi) {
  if (q >= count || iq > hi) // iq: the index at q
    return ra;
  uint64_t p = s0 + q;
  const uint64_t end = s0 + count;
  // the run-start word of the next position, read before the union so that
  // the two reads overlap; `wp` is a position of the word held in `word`
  uint64_t wp = p + 1;
  uint32_t word = wp < end ? a.run_starts[wp >> 5] : 0u;
  ra = uf_unite(a.par, ra, static_cast<uint32_t>(p));
  for (p++; p < end;) {
    if ((p >> 5) != (wp >> 5)) {
      wp = p;
      word = a.run_starts[p >> 5];
    }
    const uint32_t w = word & (0xffffffffu << (p & 31));
    if (!w) {
      // the rest of the chunk continues the run; the next start is after it
      const uint64_t lastp = p | 31;
      if (lastp + 1 >= end || a.ix[lastp] >= hi)
        break;
      p = lastp + 1;
      continue;
    }
    p = (p & ~31ull) + static_cast<uint64_t>(__ffs(w) - 1);
    if (p >= end || a.ix[p] > hi)
      break;
    ra = uf_unite(a.par, ra, static_cast<uint32_t>(p));
    p++;
  }
  return ra;
}

// The links of src/dials_spots.cc:106-137 -- left, up, and the same pixel on
// the frame before -- taken a run at a time. A pixel joined to its left
// neighbour already shares a tree with its run's first pixel (lab_gather),
// except where the run crosses into a new 32-position chunk, which is joined
// here. The first pixel of each run then unites it with every run of the row
// above, and of the previous frame's same row, that overlaps its span: each
// up or previous-frame edge of the run's pixels ends in one of those runs.
__global__ void __launch_bounds__(kThreads) lab_link(LabArgs a) {
  // the batch's frame segments, read once per block
  __shared__ uint64_t sh_start[kMaxSegments], sh_count[kMaxSegments];
  __shared__ int64_t sh_z[kMaxSegments];
  LabelScalars *sc = a.sc;
  const uint64_t carry = sc->carry_n;
  const int first_batch_seg = carry > 0 ? 1 : 0;
  const uint32_t W = static_cast<uint32_t>(a.width);
  const uint32_t nruns = sc->runs_n;
  const int nseg = static_cast<int>(sc->nseg);
  const bool in_shared = nseg <= kMaxSegments;
  if (in_shared)
    for (int k = threadIdx.x; k < nseg; k += blockDim.x) {
      sh_start[k] = a.seg_start[k];
      sh_count[k] = a.seg_count[k];
      sh_z[k] = a.seg_z[k];
    }
  __syncthreads();
  const uint64_t *seg_start = in_shared ? sh_start : a.seg_start;
  const uint64_t *seg_count = in_shared ? sh_count : a.seg_count;
  const int64_t *seg_z = in_shared ? sh_z : a.seg_z;
  const int lane = threadIdx.x & 31;
  // one entry of lab_gather's list per lane, so the lanes of a warp all
  // have a run to link; a warp takes the next 32 entries when its last are
  // done (chains vary in length, so fixed shares would leave warps idle)
  while (true) {
    uint32_t base = 0;
    if (lane == 0)
      base = atomicAdd(&sc->link_next, 32u);
    base = __shfl_sync(kFull, base, 0);
    if (base >= nruns)
      break;
    const uint64_t i = base + static_cast<uint64_t>(lane);
    if (i >= nruns)
      continue;
    const uint4 e = a.runs[i];
    const uint32_t g = e.x, idx = e.y;
    const uint32_t len = e.z & 0x3fu;
    const int s = static_cast<int>(e.z >> 8);
    uint32_t ra = g;
    if (e.z & 0x40u) // a run crossing into a new chunk: join the pieces
      ra = uf_unite(a.par, ra, g - 1);
    const uint64_t s0 = seg_start[s];
    const uint64_t end = s0 + seg_count[s];
    const uint32_t last = idx + len - 1; // the piece's last index (one row, one chunk)
    const bool up = idx >= W;
    const bool prev = !a.two_d && s > 0 && seg_z[s - 1] + 1 == seg_z[s];
    // both lookups' first loads before either walk
    const uint32_t *tabu = up ? table_of(a, s, first_batch_seg) + ((idx - W) >> kBlockShift)
                              : nullptr;
    const uint32_t *tabp = prev ? table_of(a, s - 1, first_batch_seg) + (idx >> kBlockShift)
                                : nullptr;
    const uint32_t tu = up ? tabu[0] : kNone, tu1 = up ? tabu[1] : kNone;
    const uint32_t tp = prev ? tabp[0] : kNone, tp1 = prev ? tabp[1] : kNone;
    uint32_t iu = 0, ip = 0;
    const uint64_t qu = up ? first_at_least(a, tu, tu1, s0, end - s0, idx - W, &iu) : end - s0;
    uint64_t ps0 = 0, pcount = 0, qp = 0;
    if (prev) {
      ps0 = seg_start[s - 1];
      pcount = seg_count[s - 1];
      qp = first_at_least(a, tp, tp1, ps0, pcount, idx, &ip);
    }
    if (up)
      ra = unite_overlaps(a, ra, qu, iu, s0, end - s0, last - W);
    if (prev)
      unite_overlaps(a, ra, qp, ip, ps0, pcount, last);
  }
}

// After the batch: the last frame's table becomes the carry's, since every
// pixel of the last frame is carried, in the same order.
__global__ void __launch_bounds__(kThreads) lab_keep_table(LabArgs a) {
  if (a.nframes == 0 || a.close_all || a.two_d)
    return;
  const uint32_t *last = a.tab + static_cast<uint64_t>(a.nframes - 1) * a.nblk;
  for (uint64_t b = gtid(); b < a.nblk; b += gstride())
    a.carry_tab[b] = last[b];
}

// Roots, component sizes and last frames. A warp's lanes hold 32
// consecutive positions; each stretch of adjacent lanes with one root (a
// run, mostly) makes one update. Positions are in (frame, index) order, so
// a stretch's last frame is its last lane's.
__global__ void __launch_bounds__(kThreads) lab_flatten(LabArgs a) {
  const uint64_t n = a.sc->n;
  const int lane = threadIdx.x & 31;
  const uint64_t warps = gstride() >> 5;
  for (uint64_t base = (gtid() >> 5) * 32; base < n; base += warps * 32) {
    const uint64_t g = base + lane;
    uint32_t r = kNone;
    int32_t z = INT_MIN;
    if (g < n) {
      z = a.fr[g]; // read before the walk, which it does not depend on
      r = uf_root(a.par, static_cast<uint32_t>(g)); // lab_link is done: no more links
      a.root[g] = r;
    }
    const uint32_t before = __shfl_up_sync(kFull, r, 1);
    const bool head = lane == 0 || before != r;
    const uint32_t heads = __ballot_sync(kFull, head);
    // the stretch ends before the next head (bits above this lane)
    const uint32_t later = lane == 31 ? 0u : heads & (0xfffffffeu << lane);
    const int end = later ? __ffs(later) - 2 : 31;
    const int32_t zlast = __shfl_sync(kFull, z, end);
    if (head && r != kNone) {
      atomicAdd(&a.size[r], static_cast<uint32_t>(end - lane + 1));
      atomicMax(&a.lastz[r], zlast);
    }
  }
}

__global__ void __launch_bounds__(kThreads) lab_mark(LabArgs a) {
  const LabelScalars *sc = a.sc;
  const uint64_t n = sc->n, nw = sc->nw;
  const int lane = threadIdx.x & 31;
  const uint64_t warp = gtid() >> 5, nwarps = gstride() >> 5;
  for (uint64_t w = warp; w < nw; w += nwarps) {
    const uint32_t m = __ballot_sync(kFull, finished_root(a, w * 32 + lane, n));
    if (lane == 0) {
      a.bits[w] = m;
      a.bcnt[w] = __popc(m);
    }
  }
}

// The finished roots in position order, from the bitmap and the scanned
// word counts (a thread per word: most words hold none, few more than one).
// Also the length of the bucket-count table that the next scan covers.
__global__ void __launch_bounds__(kThreads) lab_compact(LabArgs a) {
  LabelScalars *sc = a.sc;
  const uint64_t nw = sc->nw;
  if (gtid() == 0) {
    const uint64_t closed = sc->closed32;
    sc->closed = closed;
    sc->seg_len = sc->nseg * ((closed + 31) / 32);
  }
  for (uint64_t w = gtid(); w < nw; w += gstride()) {
    uint32_t m = a.bits[w];
    uint32_t at = a.bcnt[w];
    while (m) {
      a.flist[at++] = static_cast<uint32_t>(w * 32 + __ffs(m) - 1);
      m &= m - 1;
    }
  }
}

// Per 32 consecutive roots of the list, how many close in each bucket, laid
// out bucket-major (bucket s, group j at s * groups + j).
__global__ void __launch_bounds__(kThreads) lab_count(LabArgs a) {
  const LabelScalars *sc = a.sc;
  const uint64_t closed = sc->closed, groups = (closed + 31) / 32;
  const int nseg = static_cast<int>(sc->nseg);
  const int lane = threadIdx.x & 31;
  const uint64_t warp = gtid() >> 5, nwarps = gstride() >> 5;
  for (uint64_t j = warp; j < groups; j += nwarps) {
    const uint64_t k = j * 32 + lane;
    const int b = k < closed ? bucket_of(a.seg_z, nseg, a.lastz[a.flist[k]]) : -1;
    for (int s = 0; s < nseg; s++) {
      const uint32_t m = __ballot_sync(kFull, b == s);
      if (lane == 0)
        a.bcnt[s * groups + j] = __popc(m);
    }
  }
}

__global__ void __launch_bounds__(kThreads) lab_rank(LabArgs a) {
  LabelScalars *sc = a.sc;
  const uint64_t closed = sc->closed, groups = (closed + 31) / 32;
  const int nseg = static_cast<int>(sc->nseg);
  const int lane = threadIdx.x & 31;
  const uint64_t warp = gtid() >> 5, nwarps = gstride() >> 5;
  uint32_t small = 0, large = 0;
  for (uint64_t j = warp; j < groups; j += nwarps) {
    const uint64_t k = j * 32 + lane;
    const bool valid = k < closed;
    const uint32_t g = valid ? a.flist[k] : 0u;
    const int b = valid ? bucket_of(a.seg_z, nseg, a.lastz[g]) : -1;
    // earlier roots of this group in the same bucket come first
    const uint32_t peers = __match_any_sync(kFull, b);
    if (!valid)
      continue;
    const uint32_t rank =
        a.bcnt[b * groups + j] + __popc(peers & ((1u << lane) - 1u));
    a.rank_of_root[g] = rank;
    a.comp_root[rank] = g;
    const uint32_t size = a.size[g];
    const bool keep = size >= a.min_size && size <= a.max_size;
    a.msize[rank] = keep ? size : 0u;
    a.mpk[rank] = keep ? (static_cast<uint64_t>(size) | (1ull << 32)) : 0ull;
    if (keep && size > kMidCap)
      a.big[atomicAdd(&sc->big_n, 1u)] = rank;
    else if (keep && size > kSmallCap)
      a.mid[atomicAdd(&sc->mid_n, 1u)] = rank;
    small += size < a.min_size;
    large += size > a.max_size;
  }
  if (small)
    atomicAdd(reinterpret_cast<unsigned long long *>(&sc->too_small), small);
  if (large)
    atomicAdd(reinterpret_cast<unsigned long long *>(&sc->too_large), large);
}

// Member lists, and the open pixels (their component is not finished by
// this batch, so they are carried) as a bitmap and count per 32 positions. A warp takes 32 consecutive
// positions; the lanes of one component claim their slots with one atomic
// and fill them in lane order.
// So each component's list is a set of runs, one per 32-position chunk it
// has pixels in, each run ascending and within its chunk; lab_accept orders
// the runs rather than the members.
__global__ void __launch_bounds__(kThreads) lab_scatter(LabArgs a) {
  const uint64_t n = a.sc->n;
  const int lane = threadIdx.x & 31;
  const uint64_t warps = gstride() >> 5;
  for (uint64_t base = (gtid() >> 5) * 32; base < n; base += warps * 32) {
    const uint64_t g = base + lane;
    uint32_t r = kNone, rank = kNone, moff = 0;
    bool open = false;
    if (g < n) {
      r = a.root[g];
      rank = a.rank_of_root[r];
      open = rank == kNone; // not finished by this batch: carried
      if (rank != kNone) {
        // the component's size and member offset read together
        const uint32_t size = a.msize[rank];
        moff = static_cast<uint32_t>(a.mpk[rank]);
        if (size == 0)
          rank = kNone;
      }
    }
    const uint32_t ob = __ballot_sync(kFull, open);
    if (lane == 0) {
      a.obits[base >> 5] = ob;
      a.ocnt[base >> 5] = __popc(ob);
    }
    const uint32_t key = rank == kNone ? kNone : r;
    const uint32_t peers = __match_any_sync(kFull, key);
    if (key == kNone)
      continue;
    const int leader = __ffs(peers) - 1;
    uint32_t at = 0;
    if (lane == leader)
      at = atomicAdd(&a.cursor[r], static_cast<uint32_t>(__popc(peers)));
    at = __shfl_sync(peers, at, leader) + __popc(peers & ((1u << lane) - 1u));
    a.members[moff + at] = static_cast<uint32_t>(g);
  }
}

// Shell sort of a short array (a spot has at most max_spot_size members).
__device__ void sort_positions(uint32_t *v, uint32_t n) {
  const uint32_t gaps[] = {701, 301, 132, 57, 23, 10, 4, 1};
  for (uint32_t gap : gaps) {
    if (gap >= n)
      continue;
    for (uint32_t i = gap; i < n; i++) {
      const uint32_t t = v[i];
      uint32_t j = i;
      while (j >= gap && v[j - gap] > t) {
        v[j] = v[j - gap];
        j -= gap;
      }
      v[j] = t;
    }
  }
}

// The member data a spot pass reads: from global memory through the member
// positions, or from the per-warp copy in shared memory.
struct GlobalMembers {
  const LabArgs *a;
  const uint32_t *m;
  __device__ __forceinline__ void get(uint32_t k, uint32_t *idx, uint32_t *v, int32_t *z) const {
    const uint32_t g = m[k];
    *idx = a->ix[g];
    *v = a->val[g];
    *z = a->fr[g];
  }
};
struct SharedMembers {
  const uint32_t *ix, *val;
  const int32_t *fr;
  __device__ __forceinline__ void get(uint32_t k, uint32_t *idx, uint32_t *v, int32_t *z) const {
    *idx = ix[k];
    *v = val[k];
    *z = fr[k];
  }
};

// The per-component arithmetic of src/dials_spots.cc:221-360, in the
// reference's order, one IEEE rounding per operation (explicit _rn so that
// nothing is fused). Returns whether the spot passes the peak-centroid
// filter; fills *spot either way.
template <typename Members>
__device__ bool spot_pass(const DivU32 &W, double max_sep, const Members &mem, uint32_t n,
                          Spot *spot) {
  const double pixel_variance = 1.0 / 12.0;
  double sum = 0.0, sum_sq = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
  int32_t x0 = 0, x1 = 0, y0 = 0, y1 = 0, z0 = 0, z1 = 0;
  uint32_t peak_value = 0;
  double px = 0.0, py = 0.0, pz = 0.0;
  for (uint32_t k = 0; k < n; k++) {
    uint32_t idx, v;
    int32_t z;
    mem.get(k, &idx, &v, &z);
    const uint32_t yq = W.quo(idx);
    const int32_t x = static_cast<int32_t>(idx - yq * W.d);
    const int32_t y = static_cast<int32_t>(yq);
    if (k == 0) {
      x0 = x; x1 = x + 1; y0 = y; y1 = y + 1; z0 = z; z1 = z + 1;
    } else {
      x0 = min(x0, x); x1 = max(x1, x + 1);
      y0 = min(y0, y); y1 = max(y1, y + 1);
      z0 = min(z0, z); z1 = max(z1, z + 1);
    }
    const double value = __uint2double_rn(v);
    const double cx = __dadd_rn(__int2double_rn(x), 0.5);
    const double cy = __dadd_rn(__int2double_rn(y), 0.5);
    const double cz = __dadd_rn(__int2double_rn(z), 0.5);
    sum = __dadd_rn(sum, value);
    sum_sq = __dadd_rn(sum_sq, __dmul_rn(value, value));
    wx = __dadd_rn(wx, __dmul_rn(value, cx));
    wy = __dadd_rn(wy, __dmul_rn(value, cy));
    wz = __dadd_rn(wz, __dmul_rn(value, cz));
    if (v > peak_value) {
      peak_value = v;
      px = cx; py = cy; pz = cz;
    }
  }
  spot->bbox[0] = x0; spot->bbox[1] = x1;
  spot->bbox[2] = y0; spot->bbox[3] = y1;
  spot->bbox[4] = z0; spot->bbox[5] = z1;
  spot->intensity = sum;
  spot->intensity_variance = sum;
  spot->n_signal = n;
  if (sum > 0.0) {
    const double mx = __ddiv_rn(wx, sum), my = __ddiv_rn(wy, sum);
    double mz = __ddiv_rn(wz, sum);
    double dx2 = 0.0, dy2 = 0.0, dz2 = 0.0;
    for (uint32_t k = 0; k < n; k++) {
      uint32_t idx, v;
      int32_t z;
      mem.get(k, &idx, &v, &z);
      const double value = __uint2double_rn(v);
      const uint32_t yq = W.quo(idx);
      const double dx = __dsub_rn(__dadd_rn(__uint2double_rn(idx - yq * W.d), 0.5), mx);
      const double dy = __dsub_rn(__dadd_rn(__uint2double_rn(yq), 0.5), my);
      const double dz = __dsub_rn(__dadd_rn(__int2double_rn(z), 0.5), mz);
      dx2 = __dadd_rn(dx2, __dmul_rn(__dmul_rn(value, dx), dx));
      dy2 = __dadd_rn(dy2, __dmul_rn(__dmul_rn(value, dy), dy));
      dz2 = __dadd_rn(dz2, __dmul_rn(__dmul_rn(value, dz), dz));
    }
    const double ss = __dmul_rn(sum, sum);
    if (ss > sum_sq) {
      const double den = __dsub_rn(ss, sum_sq);
      spot->variance[0] = __dadd_rn(__ddiv_rn(__ddiv_rn(__dmul_rn(dx2, sum), den), sum), pixel_variance);
      spot->variance[1] = __dadd_rn(__ddiv_rn(__ddiv_rn(__dmul_rn(dy2, sum), den), sum), pixel_variance);
      spot->variance[2] = __dadd_rn(__ddiv_rn(__ddiv_rn(__dmul_rn(dz2, sum), den), sum), pixel_variance);
    } else {
      spot->variance[0] = spot->variance[1] = spot->variance[2] = pixel_variance;
    }
    if (z1 == z0 + 1)
      mz = __dadd_rn(__int2double_rn(z0), 0.5);
    spot->position[0] = mx;
    spot->position[1] = my;
    spot->position[2] = mz;
  } else {
    spot->variance[0] = spot->variance[1] = spot->variance[2] = 0.0;
    spot->position[0] = __ddiv_rn(__int2double_rn(x1 + x0), 2.0);
    spot->position[1] = __ddiv_rn(__int2double_rn(y1 + y0), 2.0);
    spot->position[2] = __ddiv_rn(__int2double_rn(z1 + z0), 2.0);
  }
  if (max_sep > 0.0) {
    const double dx = __dsub_rn(px, spot->position[0]);
    const double dy = __dsub_rn(py, spot->position[1]);
    const double dz = __dsub_rn(pz, spot->position[2]);
    const double d = __dsqrt_rn(
        __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    if (d > max_sep)
      return false;
  }
  return true;
}

// One warp per finished component. The members (positions in the live set)
// are sorted in shared memory by a warp bitonic network -- position order is
// (frame, index) order -- and their pixels gathered there; every lane then
// runs the same sequential pass, so the doubles accumulate in the
// reference's order and the result is warp-uniform. Components larger than
// the per-warp buffer (possible only with max_spot_size above it) take a
// slower path through global memory.
constexpr int kCompWarps = 4;
constexpr uint32_t kCompCap = 1024;

struct WarpBuffers {
  uint32_t *g, *ix, *val;
  int32_t *fr;
  double *t; // 3 x 32 second-pass terms
};

// Per warp: four CAP-member arrays and the terms. Three launches split the
// components by size: up to kSmallCap members with small buffers, so that
// many warps fit on an SM, up to kMidCap with middle ones, and the rest with
// kCompCap-member buffers.

template <uint32_t CAP> __host__ __device__ constexpr size_t warp_comp_bytes() {
  return 4 * CAP * sizeof(uint32_t) + 3 * 32 * sizeof(double);
}

template <uint32_t CAP>
__device__ __forceinline__ WarpBuffers warp_buffers(unsigned char *smem, int warp) {
  WarpBuffers b;
  unsigned char *at = smem + static_cast<size_t>(warp) * warp_comp_bytes<CAP>();
  uint32_t *base = reinterpret_cast<uint32_t *>(at);
  b.g = base;
  b.ix = base + CAP;
  b.val = base + 2 * CAP;
  b.fr = reinterpret_cast<int32_t *>(base + 3 * CAP);
  b.t = reinterpret_cast<double *>(base + 4 * CAP);
  return b;
}

__device__ void warp_sort(uint32_t *s, uint32_t n, int lane) {
  uint32_t p = 2;
  while (p < n)
    p <<= 1;
  for (uint32_t i = n + lane; i < p; i += 32)
    s[i] = kNone;
  __syncwarp();
  for (uint32_t k = 2; k <= p; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = lane; i < p; i += 32) {
        const uint32_t l = i ^ j;
        if (l > i) {
          const uint32_t x = s[i], y = s[l];
          if ((x > y) == ((i & k) == 0)) {
            s[i] = y;
            s[l] = x;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Member k of b.g starts a run: the first member, or a different 32-position
// chunk from the member before it.
__device__ __forceinline__ bool run_start(const uint32_t *g, uint32_t k, uint32_t n) {
  return k < n && (k == 0 || (g[k] >> 5) != (g[k - 1] >> 5));
}

// Puts the member positions in b.g (n <= kCompCap, as lab_scatter left them:
// runs, one per chunk, each ascending) into ascending order by ordering the
// runs: their chunks are sorted (the chunks of one component are distinct),
// each run finds its rank by binary search, and every member moves once.
// Uses b.ix, b.val and b.fr as scratch.
__device__ void move_runs(const WarpBuffers &b, uint32_t n, int lane);

__device__ void order_members(const WarpBuffers &b, uint32_t n, int lane) {
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t runs = 0;
  for (uint32_t c = 0; c < n; c += 32) {
    const uint32_t k = c + lane;
    const bool st = run_start(b.g, k, n);
    const uint32_t flags = __ballot_sync(kFull, st);
    if (st)
      b.ix[runs + __popc(flags & lt)] = k; // where run j starts
    runs += __popc(flags);
  }
  __syncwarp();
  if (runs == 1)
    return; // one chunk: already ascending
  if (runs <= 32) {
    // One run per lane. Sort the keys chunk << 5 | run (chunks are below
    // 2^27) across the lanes with a bitonic network in registers; lane q then
    // holds the run of rank q, whose place is the sum of the lengths of the
    // runs ranked before it.
    const bool have = static_cast<uint32_t>(lane) < runs;
    const uint32_t s0 = have ? b.ix[lane] : 0u;
    const uint32_t s1 = static_cast<uint32_t>(lane) + 1 < runs ? b.ix[lane + 1] : n;
    const uint32_t len = have ? s1 - s0 : 0u;
    uint32_t key = have ? (b.g[s0] & ~31u) | static_cast<uint32_t>(lane) : 0xffffffffu;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
      for (int j = k >> 1; j > 0; j >>= 1) {
        const uint32_t other = __shfl_xor_sync(kFull, key, j);
        const bool ascending = (lane & k) == 0, lower = (lane & j) == 0;
        key = lower == ascending ? min(key, other) : max(key, other);
      }
    }
    const int run = static_cast<int>(key & 31u); // valid on lanes below runs
    const uint32_t rlen = __shfl_sync(kFull, len, run);
    const uint32_t rs0 = __shfl_sync(kFull, s0, run);
    uint32_t incl = have ? rlen : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(kFull, incl, d);
      if (lane >= d)
        incl += v;
    }
    __syncwarp(); // every lane has read its start before any is overwritten
    if (have)
      b.ix[run] = rs0 | ((incl - rlen) << 16); // start and place, both below kCompCap
    __syncwarp();
    move_runs(b, n, lane);
    return;
  }
  if (runs <= 64) {
    // Two runs per lane, run lane in A and run lane + 32 in B: the keys
    // chunk << 6 | run (while every position is below 2^30, so that no key
    // reaches the empty slots' all-ones) sorted as 64
    // elements, element lane in A and lane + 32 in B, by the same bitonic
    // network; the pairs at distance 32 meet within a lane.
    const bool hb = static_cast<uint32_t>(lane) + 32 < runs;
    const uint32_t s0a = b.ix[lane]; // runs > 32: lanes 0-31 all hold a run
    const uint32_t s1a = b.ix[lane + 1];
    const uint32_t s0b = hb ? b.ix[lane + 32] : 0u;
    const uint32_t s1b = static_cast<uint32_t>(lane) + 33 < runs ? b.ix[lane + 33] : n;
    const uint32_t ga = b.g[s0a], gb = hb ? b.g[s0b] : 0u;
    if (!__any_sync(kFull, ((ga | gb) & 0xc0000000u) != 0)) {
      const uint32_t lena = s1a - s0a, lenb = hb ? s1b - s0b : 0u;
      uint32_t ka = ((ga & ~31u) << 1) | static_cast<uint32_t>(lane);
      uint32_t kb = hb ? ((gb & ~31u) << 1) | static_cast<uint32_t>(lane + 32) : 0xffffffffu;
#pragma unroll
      for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
          if (j == 32) { // k == 64: ascending, A the lower element
            const uint32_t lo = min(ka, kb), hi = max(ka, kb);
            ka = lo;
            kb = hi;
          } else {
            const uint32_t oa = __shfl_xor_sync(kFull, ka, j);
            const uint32_t ob = __shfl_xor_sync(kFull, kb, j);
            const bool lower = (lane & j) == 0;
            const bool asc_a = (lane & k) == 0, asc_b = ((lane + 32) & k) == 0;
            ka = lower == asc_a ? min(ka, oa) : max(ka, oa);
            kb = lower == asc_b ? min(kb, ob) : max(kb, ob);
          }
        }
      }
      // lane q holds ranks q (A) and q + 32 (B, a run while q + 32 < runs)
      const bool rb = static_cast<uint32_t>(lane) + 32 < runs;
      const uint32_t run_a = ka & 63u, run_b = kb & 63u;
      auto of_run = [&](uint32_t va, uint32_t vb, uint32_t r) {
        const uint32_t xa = __shfl_sync(kFull, va, static_cast<int>(r & 31u));
        const uint32_t xb = __shfl_sync(kFull, vb, static_cast<int>(r & 31u));
        return r < 32 ? xa : xb;
      };
      const uint32_t len_ra = of_run(lena, lenb, run_a), s0_ra = of_run(s0a, s0b, run_a);
      const uint32_t len_rb = of_run(lena, lenb, run_b), s0_rb = of_run(s0a, s0b, run_b);
      uint32_t inca = len_ra, incb = rb ? len_rb : 0u;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t va = __shfl_up_sync(kFull, inca, d);
        const uint32_t vb = __shfl_up_sync(kFull, incb, d);
        if (lane >= d) {
          inca += va;
          incb += vb;
        }
      }
      const uint32_t half = __shfl_sync(kFull, inca, 31); // ranks 0-31's lengths
      __syncwarp(); // every lane has read its starts before any is overwritten
      b.ix[run_a] = s0_ra | ((inca - len_ra) << 16); // start and place, below kCompCap
      if (rb)
        b.ix[run_b] = s0_rb | ((half + incb - len_rb) << 16);
      __syncwarp();
      move_runs(b, n, lane);
      return;
    }
  }
  for (uint32_t j = lane; j < runs; j += 32)
    b.val[j] = b.g[b.ix[j]] >> 5;
  __syncwarp();
  warp_sort(b.val, runs, lane); // the chunks, ascending
  auto rank_of = [&](uint32_t key) {
    uint32_t lo = 0, hi = runs;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (b.val[mid] < key)
        lo = mid + 1;
      else
        hi = mid;
    }
    return lo;
  };
  for (uint32_t j = lane; j < runs; j += 32) {
    const uint32_t s0 = b.ix[j];
    const uint32_t s1 = j + 1 < runs ? b.ix[j + 1] : n;
    b.fr[rank_of(b.g[s0] >> 5)] = static_cast<int32_t>(s1 - s0); // lengths in chunk order
  }
  __syncwarp();
  uint32_t carry = 0; // exclusive scan of the lengths: each run's place
  for (uint32_t c = 0; c < runs; c += 32) {
    const uint32_t q = c + lane;
    const uint32_t len = q < runs ? static_cast<uint32_t>(b.fr[q]) : 0u;
    uint32_t inc = len;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(kFull, inc, d);
      if (lane >= d)
        inc += v;
    }
    if (q < runs)
      b.fr[q] = static_cast<int32_t>(carry + inc - len);
    carry += __shfl_sync(kFull, inc, 31);
  }
  __syncwarp();
  for (uint32_t j = lane; j < runs; j += 32) {
    const uint32_t s0 = b.ix[j];
    const uint32_t off = static_cast<uint32_t>(b.fr[rank_of(b.g[s0] >> 5)]);
    b.ix[j] = s0 | (off << 16); // start and place, both below kCompCap
  }
  __syncwarp();
  move_runs(b, n, lane);
}

// Moves every member to its run's place plus its offset in the run (b.ix
// holds start | place << 16 per run, in run order) through b.fr.
__device__ void move_runs(const WarpBuffers &b, uint32_t n, int lane) {
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t base = 0;
  for (uint32_t c = 0; c < n; c += 32) {
    const uint32_t k = c + lane;
    const uint32_t flags = __ballot_sync(kFull, run_start(b.g, k, n));
    // the run this member belongs to: the last start at or before it
    const uint32_t r = base + __popc(flags & (lt | (1u << lane))) - 1;
    if (k < n) {
      const uint32_t packed = b.ix[r];
      b.fr[(packed >> 16) + (k - (packed & 0xffffu))] = static_cast<int32_t>(b.g[k]);
    }
    base += __popc(flags);
  }
  __syncwarp();
  for (uint32_t k = lane; k < n; k += 32)
    b.g[k] = static_cast<uint32_t>(b.fr[k]);
  __syncwarp();
}

// Loads (ordering if asked) a component's members and their pixels into the
// warp's buffers.
template <uint32_t kU>
__device__ void load_members(const LabArgs &a, uint32_t *m, uint32_t n, bool sort,
                             const WarpBuffers &b, int lane) {
  // kU members a lane at a time, every load issued before the first store,
  // so that a large component's reads overlap instead of following one
  // another (the small components' launch takes one: its 64 registers are
  // spoken for).
  for (uint32_t k0 = lane; k0 < n; k0 += 32 * kU) {
    uint32_t v[kU];
#pragma unroll
    for (uint32_t u = 0; u < kU; u++)
      v[u] = k0 + 32 * u < n ? m[k0 + 32 * u] : 0u;
#pragma unroll
    for (uint32_t u = 0; u < kU; u++)
      if (k0 + 32 * u < n)
        b.g[k0 + 32 * u] = v[u];
  }
  __syncwarp();
  if (sort)
    order_members(b, n, lane);
  for (uint32_t k0 = lane; k0 < n; k0 += 32 * kU) {
    uint32_t g[kU], ix[kU], val[kU];
    int32_t fr[kU];
#pragma unroll
    for (uint32_t u = 0; u < kU; u++)
      g[u] = k0 + 32 * u < n ? b.g[k0 + 32 * u] : 0u;
#pragma unroll
    for (uint32_t u = 0; u < kU; u++)
      if (k0 + 32 * u < n) {
        ix[u] = a.ix[g[u]];
        val[u] = a.val[g[u]];
        fr[u] = a.fr[g[u]];
      }
#pragma unroll
    for (uint32_t u = 0; u < kU; u++)
      if (k0 + 32 * u < n) {
        b.ix[k0 + 32 * u] = ix[u];
        b.val[k0 + 32 * u] = val[u];
        b.fr[k0 + 32 * u] = fr[u];
      }
  }
  __syncwarp();
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1)
    v += __shfl_xor_sync(kFull, v, d);
  return v;
}
__device__ __forceinline__ int32_t warp_min(int32_t v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1)
    v = min(v, __shfl_xor_sync(kFull, v, d));
  return v;
}
__device__ __forceinline__ int32_t warp_max(int32_t v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1)
    v = max(v, __shfl_xor_sync(kFull, v, d));
  return v;
}

// The spot pass with the warp's 32 lanes sharing the work, for members in
// shared memory. The first pass (count, sums, weighted sums, bbox, peak) is
// a parallel reduction; it is taken only when every partial sum it can form
// is exact in double -- integers (and halves, for the weighted sums) below
// 2^52 -- so its result is the reference's sequential one bit for bit. The
// second pass's terms value * d * d are rounded, so they are formed in
// parallel but added in member order, one after another, as the reference
// adds them. Returns false (and leaves *spot alone) if the first pass is not
// exact for this component; *ok is the peak-centroid filter's verdict.
__device__ bool spot_pass_warp(const DivU32 &W, double max_sep, const WarpBuffers &b,
                               uint32_t n, int lane, Spot *spot, bool *ok) {
  double sum = 0.0, sum_sq = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
  int32_t x0 = INT_MAX, x1 = INT_MIN, y0 = INT_MAX, y1 = INT_MIN, z0 = INT_MAX, z1 = INT_MIN;
  uint32_t peak_v = 0, peak_k = kNone, max_v = 0;
  uint32_t max_c = 0;
  for (uint32_t k = lane; k < n; k += 32) {
    const uint32_t idx = b.ix[k], v = b.val[k];
    const int32_t z = b.fr[k];
    const uint32_t yq = W.quo(idx);
    const int32_t x = static_cast<int32_t>(idx - yq * W.d), y = static_cast<int32_t>(yq);
    const double value = __uint2double_rn(v);
    sum = __dadd_rn(sum, value);
    sum_sq = __dadd_rn(sum_sq, __dmul_rn(value, value));
    wx = __dadd_rn(wx, __dmul_rn(value, __dadd_rn(__int2double_rn(x), 0.5)));
    wy = __dadd_rn(wy, __dmul_rn(value, __dadd_rn(__int2double_rn(y), 0.5)));
    wz = __dadd_rn(wz, __dmul_rn(value, __dadd_rn(__int2double_rn(z), 0.5)));
    x0 = min(x0, x); x1 = max(x1, x + 1);
    y0 = min(y0, y); y1 = max(y1, y + 1);
    z0 = min(z0, z); z1 = max(z1, z + 1);
    if (v > peak_v) { // k rises within a lane: the lane's first maximum
      peak_v = v;
      peak_k = k;
    }
    max_c = max(max_c, max(max(static_cast<uint32_t>(x), static_cast<uint32_t>(y)),
                           static_cast<uint32_t>(z < 0 ? -z : z)));
  }
  max_v = peak_v;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    max_v = max(max_v, __shfl_xor_sync(kFull, max_v, d));
    max_c = max(max_c, __shfl_xor_sync(kFull, max_c, d));
  }
  // |every partial sum| <= n * max_v * max(max_v, 2 (max_c + 1)), in units
  // of 0.5 for the weighted sums: exact below 2^52.
  const double bound = static_cast<double>(n) * static_cast<double>(max_v) *
                       fmax(static_cast<double>(max_v), 2.0 * (static_cast<double>(max_c) + 1.0));
  if (!(bound < 4503599627370496.0)) // 2^52
    return false;
  sum = warp_sum(sum);
  sum_sq = warp_sum(sum_sq);
  wx = warp_sum(wx);
  wy = warp_sum(wy);
  wz = warp_sum(wz);
  x0 = warp_min(x0); x1 = warp_max(x1);
  y0 = warp_min(y0); y1 = warp_max(y1);
  z0 = warp_min(z0); z1 = warp_max(z1);
  // the first maximum over the whole component: the largest value, then
  // the lowest member index among lanes that hold it
  uint32_t pk = peak_v == max_v ? peak_k : kNone;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1)
    pk = min(pk, __shfl_xor_sync(kFull, pk, d));
  double px = 0.0, py = 0.0, pz = 0.0;
  if (max_v > 0 && pk != kNone) {
    const uint32_t pidx = b.ix[pk], pq = W.quo(pidx);
    px = __dadd_rn(__uint2double_rn(pidx - pq * W.d), 0.5);
    py = __dadd_rn(__uint2double_rn(pq), 0.5);
    pz = __dadd_rn(__int2double_rn(b.fr[pk]), 0.5);
  }

  const double pixel_variance = 1.0 / 12.0;
  spot->bbox[0] = x0; spot->bbox[1] = x1;
  spot->bbox[2] = y0; spot->bbox[3] = y1;
  spot->bbox[4] = z0; spot->bbox[5] = z1;
  spot->intensity = sum;
  spot->intensity_variance = sum;
  spot->n_signal = n;
  if (sum > 0.0) {
    const double mx = __ddiv_rn(wx, sum), my = __ddiv_rn(wy, sum);
    double mz = __ddiv_rn(wz, sum);
    // lanes 0, 1 and 2 each run one of the three sums, over terms the
    // whole warp computes 32 at a time. Every term value * d * d is +0 or
    // positive (value >= 0, and the two factors d have one sign), so the
    // sums are too, and the +0 terms past the last member leave them
    // unchanged: each chunk is 32 additions with no bound to test.
    double acc = 0.0;
    for (uint32_t c = 0; c < n; c += 32) {
      const uint32_t k = c + lane;
      double tx = 0.0, ty = 0.0, tz = 0.0;
      if (k < n) {
        const uint32_t idx = b.ix[k], yq = W.quo(idx);
        const double value = __uint2double_rn(b.val[k]);
        const double dx = __dsub_rn(__dadd_rn(__uint2double_rn(idx - yq * W.d), 0.5), mx);
        const double dy = __dsub_rn(__dadd_rn(__uint2double_rn(yq), 0.5), my);
        const double dz = __dsub_rn(__dadd_rn(__int2double_rn(b.fr[k]), 0.5), mz);
        tx = __dmul_rn(__dmul_rn(value, dx), dx);
        ty = __dmul_rn(__dmul_rn(value, dy), dy);
        tz = __dmul_rn(__dmul_rn(value, dz), dz);
      }
      b.t[lane] = tx;
      b.t[32 + lane] = ty;
      b.t[64 + lane] = tz;
      __syncwarp();
      if (lane < 3) {
        const double2 *t = reinterpret_cast<const double2 *>(b.t + 32 * lane);
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const double2 u = t[j];
          acc = __dadd_rn(__dadd_rn(acc, u.x), u.y);
        }
      }
      __syncwarp();
    }
    const double dx2 = __shfl_sync(kFull, acc, 0);
    const double dy2 = __shfl_sync(kFull, acc, 1);
    const double dz2 = __shfl_sync(kFull, acc, 2);
    const double ss = __dmul_rn(sum, sum);
    if (ss > sum_sq) {
      const double den = __dsub_rn(ss, sum_sq);
      spot->variance[0] = __dadd_rn(__ddiv_rn(__ddiv_rn(__dmul_rn(dx2, sum), den), sum), pixel_variance);
      spot->variance[1] = __dadd_rn(__ddiv_rn(__ddiv_rn(__dmul_rn(dy2, sum), den), sum), pixel_variance);
      spot->variance[2] = __dadd_rn(__ddiv_rn(__ddiv_rn(__dmul_rn(dz2, sum), den), sum), pixel_variance);
    } else {
      spot->variance[0] = spot->variance[1] = spot->variance[2] = pixel_variance;
    }
    if (z1 == z0 + 1)
      mz = __dadd_rn(__int2double_rn(z0), 0.5);
    spot->position[0] = mx;
    spot->position[1] = my;
    spot->position[2] = mz;
  } else {
    spot->variance[0] = spot->variance[1] = spot->variance[2] = 0.0;
    spot->position[0] = __ddiv_rn(__int2double_rn(x1 + x0), 2.0);
    spot->position[1] = __ddiv_rn(__int2double_rn(y1 + y0), 2.0);
    spot->position[2] = __ddiv_rn(__int2double_rn(z1 + z0), 2.0);
  }
  *ok = true;
  if (max_sep > 0.0) {
    const double dx = __dsub_rn(px, spot->position[0]);
    const double dy = __dsub_rn(py, spot->position[1]);
    const double dz = __dsub_rn(pz, spot->position[2]);
    const double d = __dsqrt_rn(
        __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    if (d > max_sep)
      *ok = false;
  }
  return true;
}

// Per finished component that passes the size filters: sort its members,
// run the spot pass, and park the spot and its pixel records by the
// component's size-filtered index and member offset until lab_write knows
// where the accepted ones go.
// Components of lo < size <= hi; the launch with lo = 0 also clears the
// pack word of those the size filter removed.
// `list` says which components a launch walks: 0 every finished root, 1
// lab_rank's list of the large ones, 2 its list of the middle-sized ones.
// Blocks per SM for a buffer size: as many as its shared memory allows.
template <uint32_t CAP> constexpr int kAcceptBlocks = CAP <= 256 ? 8 : CAP <= 512 ? 6 : 1;

template <uint32_t CAP>
__global__ void __launch_bounds__(kCompWarps * 32, kAcceptBlocks<CAP>)
    lab_accept(LabArgs a, uint32_t lo, uint32_t hi, int list) {
  extern __shared__ __align__(16) unsigned char comp_smem[];
  LabelScalars *sc = a.sc;
  const uint64_t closed = list == 0 ? sc->closed : list == 1 ? sc->big_n : sc->mid_n;
  uint32_t *next = list == 0 ? &sc->accept_next : list == 1 ? &sc->big_next : &sc->mid_next;
  const uint32_t *listed = list == 1 ? a.big : a.mid;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const WarpBuffers b = warp_buffers<CAP>(comp_smem, warp);
  const DivU32 W = a.wdiv;
  uint32_t separated = 0;
  // a warp takes the next component when it has finished its last
  while (true) {
    uint32_t i = 0;
    if (lane == 0)
      i = atomicAdd(next, 1u);
    i = __shfl_sync(kFull, i, 0);
    if (i >= closed)
      break;
    const uint64_t r = list == 0 ? i : listed[i];
    const uint32_t n = a.msize[r];
    const uint64_t mp = a.mpk[r]; // read beside the size, not after it
    if (n == 0) {
      if (lane == 0 && lo == 0)
        a.pack[r] = 0;
      continue;
    }
    if (n <= lo || n > hi)
      continue;
    const uint32_t moff = static_cast<uint32_t>(mp);
    const uint32_t sidx = static_cast<uint32_t>(mp >> 32);
    uint32_t *m = a.members + moff;
    Spot spot{}; // zeroed, padding included, so rows compare byte for byte
    bool ok;
    if (n <= CAP) {
      load_members<CAP <= 256 ? 1 : 4>(a, m, n, true, b, lane);
      if (!spot_pass_warp(W, a.max_sep, b, n, lane, &spot, &ok))
        ok = spot_pass(W, a.max_sep, SharedMembers{b.ix, b.val, b.fr}, n, &spot);
      for (uint32_t k = lane; k < n; k += 32) {
        Pixel p;
        p.frame = b.fr[k];
        p.index = b.ix[k];
        p.value = b.val[k];
        a.pix_tmp[moff + k] = p;
      }
    } else {
      if (lane == 0)
        sort_positions(m, n);
      __syncwarp();
      __threadfence_block();
      ok = spot_pass(W, a.max_sep, GlobalMembers{&a, m}, n, &spot);
      for (uint32_t k = lane; k < n; k += 32) {
        const uint32_t g = m[k];
        Pixel p;
        p.frame = a.fr[g];
        p.index = a.ix[g];
        p.value = a.val[g];
        a.pix_tmp[moff + k] = p;
      }
    }
    if (lane == 0) {
      if (sidx < a.spot_cap)
        a.spot_tmp[sidx] = spot;
      else
        sc->status = kLabelSpotOverflow;
      if (!ok) {
        separated++;
        a.msize[r] = 0;
        a.pack[r] = 0;
      } else {
        a.pack[r] = (static_cast<uint64_t>(n) << 32) | 1u;
      }
    }
    __syncwarp();
  }
  if (lane == 0 && separated)
    atomicAdd(reinterpret_cast<unsigned long long *>(&sc->separated), separated);
}

// The accepted spots to their rows and their pixels to the kept list.
__global__ void __launch_bounds__(kThreads) lab_write(LabArgs a) {
  LabelScalars *sc = a.sc;
  const uint64_t closed = sc->closed;
  const uint64_t kept_base = sc->kept_total;
  const int lane = threadIdx.x & 31;
  const uint64_t gw = gtid() >> 5, nw = gstride() >> 5;
  static_assert(offsetof(Spot, first) == 96, "Spot::first is the row's last word");
  for (uint64_t r = gw; r < closed; r += nw) {
    // the component's three words read together, not one after another
    const uint32_t n = a.msize[r];
    const uint64_t pk = a.pack[r], mp = a.mpk[r];
    if (n == 0)
      continue;
    const uint64_t row = pk & 0xffffffffu;
    const uint64_t pix = pk >> 32;
    const uint32_t moff = static_cast<uint32_t>(mp);
    const uint32_t sidx = static_cast<uint32_t>(mp >> 32);
    if (row >= a.spot_cap || sidx >= a.spot_cap || pix + n > a.live_cap) {
      if (lane == 0)
        sc->status = kLabelSpotOverflow;
      continue;
    }
    // the 104-byte row as 13 words, one a lane; the last is Spot::first
    if (lane < 13) {
      const uint64_t *src = reinterpret_cast<const uint64_t *>(a.spot_tmp + sidx);
      uint64_t *dst = reinterpret_cast<uint64_t *>(a.spots + row);
      dst[lane] = lane == 12 ? kept_base + pix : src[lane];
    }
    for (uint32_t k = lane; k < n; k += 32)
      a.kept[pix + k] = a.pix_tmp[moff + k];
  }
}


// Where an open pixel lands in the carry: the scanned count of open pixels
// in the 32-position words before its own, plus the open ones before it in
// its word.
__device__ __forceinline__ uint32_t open_position(const LabArgs &a, uint64_t g) {
  return a.ocnt[g >> 5] + __popc(a.obits[g >> 5] & ((1u << (g & 31)) - 1u));
}

// The open pixels to the other live buffer, in order, a warp per
// 32-position word (most words hold none).
__global__ void __launch_bounds__(kThreads) lab_carry(LabArgs a) {
  LabelScalars *sc = a.sc;
  const uint64_t nw = sc->nw;
  const int lane = threadIdx.x & 31;
  const uint64_t warps = gstride() >> 5;
  for (uint64_t w = gtid() >> 5; w < nw; w += warps) {
    const uint32_t bits = a.obits[w], cnt = a.ocnt[w]; // read together
    if (!((bits >> lane) & 1u))
      continue;
    const uint64_t g = w * 32 + static_cast<uint64_t>(lane);
    const uint32_t at = cnt + __popc(bits & ((1u << lane) - 1u));
    const uint32_t r = a.root[g];
    a.nfr[at] = a.fr[g];
    a.nix[at] = a.ix[g];
    a.nval[at] = a.val[g];
    a.npar[at] = open_position(a, r); // the root is open too, and comes first
  }
}

__global__ void lab_finalize(LabArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0)
    return;
  LabelScalars *sc = a.sc;
  const bool all = a.close_all || a.two_d || a.nframes == 0;
  sc->groups += sc->closed;
  const uint64_t rows = sc->accepted_pack & 0xffffffffu;
  const uint64_t pixels = sc->accepted_pack >> 32;
  sc->accepted += rows;
  sc->kept_total += pixels;
  sc->batch_spots = rows;
  sc->batch_pixels = pixels;
  sc->carry_n = all ? 0 : sc->open32;
  sc->carry_last_z = last_batch_frame(a);
  // Every pixel of the last frame stays open (its components can still
  // grow), so the carry's last frame starts where that frame's first pixel
  // lands (with anything carried, the last frame has pixels).
  sc->carry_last_start = sc->carry_n > 0 ? open_position(a, a.seg_start[sc->nseg - 1]) : 0;
  sc->batch_z0 += a.nframes;
}

} // namespace

// --------------------------------------------------------------------------

DeviceLabeller::DeviceLabeller(int height, int width, const GroupOptions &options)
    : height_(height), width_(width), opt_(options) {
  if (height < 1 || width < 1)
    throw std::invalid_argument("dials_spots: a frame with no pixels in it");
  if (opt_.max_spot_size < opt_.min_spot_size)
    throw std::invalid_argument("dials_spots: max_spot_size is below min_spot_size");
  if (opt_.min_spot_size == 0)
    throw std::invalid_argument("dials_spots: min_spot_size must be at least 1");
  if (static_cast<uint64_t>(height) * width > 0xffffffffull)
    throw std::invalid_argument("dials_spots: frame too large");
  check(cudaMalloc(&sc_, sizeof(LabelScalars)), "cudaMalloc labeller scalars");
  check(cudaMemset(sc_, 0, sizeof(LabelScalars)), "clearing labeller scalars");
  nblk_ = ((static_cast<uint64_t>(height) * width) >> kBlockShift) + 2;
  check(cudaMalloc(&carry_tab_, nblk_ * sizeof(uint32_t)), "cudaMalloc carry table");
  check(cudaFuncSetAttribute(lab_accept<kCompCap>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kCompWarps * warp_comp_bytes<kCompCap>())),
        "cudaFuncSetAttribute");
  grid_ = static_cast<unsigned>(device_sm_count() * 8);
  check(cudaMallocHost(&z_stage_, sizeof(int64_t)), "cudaMallocHost");
  check(cudaStreamCreateWithFlags(&aux_, cudaStreamNonBlocking), "cudaStreamCreate");
  check(cudaStreamCreateWithFlags(&aux2_, cudaStreamNonBlocking), "cudaStreamCreate");
  check(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaEventCreateWithFlags(&join2_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaStreamSynchronize(cudaStreamLegacy), "clearing labeller scalars");
}

DeviceLabeller::~DeviceLabeller() {
  if (aux2_) {
    cudaStreamSynchronize(aux2_);
    cudaStreamDestroy(aux2_);
  }
  if (join2_)
    cudaEventDestroy(join2_);
  if (aux_) {
    cudaStreamSynchronize(aux_);
    cudaStreamDestroy(aux_);
  }
  if (fork_)
    cudaEventDestroy(fork_);
  if (join_)
    cudaEventDestroy(join_);
  release();
  cudaFree(sc_);
  cudaFree(carry_tab_);
  if (z_stage_)
    cudaFreeHost(z_stage_);
}

void DeviceLabeller::release() {
  for (Live &l : live_) {
    cudaFree(l.frame);
    cudaFree(l.index);
    cudaFree(l.value);
    cudaFree(l.parent);
    l = Live();
  }
  void *ptrs[] = {root_, size_, rank_of_root_, cursor_, lastz_, bits_, bcnt_, flist_, comp_root_,
                  msize_, mpk_, runs_, run_starts_, spot_tmp_, pix_tmp_, members_, pack_, obits_, ocnt_, spots_out_, kept_out_, seg_start_,
                  seg_count_, seg_z_, tab_, big_, mid_};
  for (void *p : ptrs)
    cudaFree(p);
  tab_ = nullptr;
  root_ = size_ = rank_of_root_ = cursor_ = nullptr;
  lastz_ = nullptr;
  bits_ = bcnt_ = flist_ = comp_root_ = msize_ = members_ = obits_ = ocnt_ = big_ = mid_ = nullptr;
  mpk_ = pack_ = nullptr;
  runs_ = nullptr;
  run_starts_ = nullptr;
  spot_tmp_ = nullptr;
  pix_tmp_ = nullptr;
  spots_out_ = nullptr;
  kept_out_ = nullptr;
  seg_start_ = seg_count_ = nullptr;
  seg_z_ = nullptr;
}

void DeviceLabeller::reserve(uint64_t batch_pixels, int max_frames, uint64_t carry_pixels) {
  if (batch_pixels <= batch_cap_ && max_frames <= frame_cap_ && carry_pixels <= carry_cap_)
    return;
  const uint64_t bc = std::max(batch_pixels, batch_cap_);
  const int fc = std::max(max_frames, frame_cap_);
  const uint64_t cc = std::max(carry_pixels, carry_cap_);
  const uint64_t live = bc + cc;
  if (live >= 0x7fffffffull)
    throw std::invalid_argument("labelling batch too large");
  // Growing keeps the carry: copy it across after reallocating.
  check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
  LabelScalars host;
  check(cudaMemcpy(&host, sc_, sizeof(host), cudaMemcpyDeviceToHost), "reading scalars");
  std::vector<int32_t> fr(host.carry_n);
  std::vector<uint32_t> ix(host.carry_n), val(host.carry_n), par(host.carry_n);
  if (host.carry_n) {
    const Live &c = live_[cur_];
    check(cudaMemcpy(fr.data(), c.frame, host.carry_n * 4, cudaMemcpyDeviceToHost), "carry");
    check(cudaMemcpy(ix.data(), c.index, host.carry_n * 4, cudaMemcpyDeviceToHost), "carry");
    check(cudaMemcpy(val.data(), c.value, host.carry_n * 4, cudaMemcpyDeviceToHost), "carry");
    check(cudaMemcpy(par.data(), c.parent, host.carry_n * 4, cudaMemcpyDeviceToHost), "carry");
  }
  release();
  const uint64_t nwmax = live / 32 + 1;
  const uint64_t spot_cap = live / opt_.min_spot_size + 1;
  try {
    auto alloc = [](auto **p, uint64_t count, const char *what) {
      check(cudaMalloc(reinterpret_cast<void **>(p), std::max<uint64_t>(count, 1) * sizeof(**p)),
            what);
    };
    for (Live &l : live_) {
      alloc(&l.frame, live, "live frames");
      alloc(&l.index, live, "live indices");
      alloc(&l.value, live, "live values");
      alloc(&l.parent, live, "live parents");
    }
    alloc(&root_, live, "roots");
    alloc(&size_, live, "sizes");
    alloc(&rank_of_root_, live, "ranks");
    alloc(&cursor_, live, "cursors");
    alloc(&lastz_, live, "last frames");
    alloc(&bits_, nwmax, "finished-root bitmap");
    alloc(&bcnt_, (fc + 1) * nwmax, "bucket counts");
    alloc(&flist_, live, "finished roots");
    alloc(&comp_root_, live, "components");
    alloc(&msize_, live, "member sizes");
    alloc(&mpk_, live, "member offsets");
    alloc(&runs_, live, "run list");
    alloc(&run_starts_, live / 32 + 1, "run starts");
    alloc(&members_, live, "members");
    alloc(&pack_, live, "spot offsets");
    alloc(&obits_, nwmax, "open bitmap");
    alloc(&ocnt_, nwmax, "open counts");
    alloc(&big_, live / (kMidCap + 1) + 1, "large components");
    alloc(&mid_, live / (kSmallCap + 1) + 1, "middle-sized components");
    alloc(&spots_out_, spot_cap, "spots");
    alloc(&spot_tmp_, spot_cap, "spot scratch");
    alloc(&pix_tmp_, live, "spot pixel scratch");
    alloc(&kept_out_, live, "spot pixels");
    alloc(&seg_start_, fc + 1, "segments");
    alloc(&seg_count_, fc + 1, "segments");
    alloc(&seg_z_, fc + 1, "segments");
    alloc(&tab_, static_cast<uint64_t>(fc) * nblk_, "block tables");
    scan32_.reserve((fc + 1) * nwmax);
    scan32_.reserve(live);
    scan64_.reserve(live);
  } catch (...) {
    release();
    batch_cap_ = carry_cap_ = live_cap_ = spot_cap_ = 0;
    frame_cap_ = 0;
    throw;
  }
  if (host.carry_n) {
    const Live &c = live_[cur_];
    check(cudaMemcpy(c.frame, fr.data(), host.carry_n * 4, cudaMemcpyHostToDevice), "carry");
    check(cudaMemcpy(c.index, ix.data(), host.carry_n * 4, cudaMemcpyHostToDevice), "carry");
    check(cudaMemcpy(c.value, val.data(), host.carry_n * 4, cudaMemcpyHostToDevice), "carry");
    check(cudaMemcpy(c.parent, par.data(), host.carry_n * 4, cudaMemcpyHostToDevice), "carry");
  }
  batch_cap_ = bc;
  frame_cap_ = fc;
  carry_cap_ = cc;
  live_cap_ = live;
  spot_cap_ = spot_cap;
}

void DeviceLabeller::set_next_frame(int64_t z, cudaStream_t s) {
  check(cudaStreamSynchronize(s), "cudaStreamSynchronize"); // the staging word is reused
  *z_stage_ = z;
  check(cudaMemcpyAsync(&sc_->batch_z0, z_stage_, sizeof(int64_t), cudaMemcpyHostToDevice, s),
        "setting the frame number");
}

void DeviceLabeller::enqueue(int nframes, const SignalPixel *lists, const uint64_t *offs,
                             const uint32_t *counts, const int32_t *count_map,
                             const uint32_t *caps, bool close_all,
                             cudaStream_t s) {
  if (nframes > frame_cap_)
    throw std::invalid_argument("more frames than the labeller was sized for");
  if (live_cap_ == 0)
    throw std::invalid_argument("the labeller has no capacity: reserve() first");
  LabArgs a;
  a.width = width_;
  a.wdiv = DivU32::of(static_cast<uint32_t>(width_));
  a.nframes = nframes;
  a.close_all = close_all ? 1 : 0;
  a.two_d = opt_.two_d ? 1 : 0;
  a.min_size = opt_.min_spot_size;
  a.max_size = opt_.max_spot_size;
  a.max_sep = opt_.max_separation;
  a.live_cap = live_cap_;
  a.spot_cap = spot_cap_;
  a.lists = lists;
  a.offs = offs;
  a.counts = counts;
  a.count_map = count_map;
  a.caps = caps;
  const Live &cur = live_[cur_];
  const Live &nxt = live_[cur_ ^ 1];
  a.fr = cur.frame;
  a.ix = cur.index;
  a.val = cur.value;
  a.par = cur.parent;
  a.nfr = nxt.frame;
  a.nix = nxt.index;
  a.nval = nxt.value;
  a.npar = nxt.parent;
  a.root = root_;
  a.size = size_;
  a.lastz = lastz_;
  a.rank_of_root = rank_of_root_;
  a.cursor = cursor_;
  a.bits = bits_;
  a.bcnt = bcnt_;
  a.flist = flist_;
  a.comp_root = comp_root_;
  a.msize = msize_;
  a.mpk = mpk_;
  a.runs = runs_;
  a.run_starts = run_starts_;
  a.spot_tmp = spot_tmp_;
  a.pix_tmp = pix_tmp_;
  a.members = members_;
  a.pack = pack_;
  a.obits = obits_;
  a.ocnt = ocnt_;
  a.big = big_;
  a.mid = mid_;
  a.spots = spots_out_;
  a.kept = kept_out_;
  a.seg_start = seg_start_;
  a.seg_count = seg_count_;
  a.seg_z = seg_z_;
  a.tab = tab_;
  a.carry_tab = carry_tab_;
  a.nblk = nblk_;
  a.sc = sc_;

  const unsigned grid = grid_;
  LabelScalars *sc = sc_;
  if (nframes > 0)
    check(cudaMemsetAsync(tab_, 0xff, static_cast<uint64_t>(nframes) * nblk_ * sizeof(uint32_t), s),
          "clearing block tables");
  lab_setup<<<1, 32, 0, s>>>(a);
  lab_gather<<<grid, kThreads, 0, s>>>(a);
  lab_link<<<grid, kThreads, 0, s>>>(a);
  lab_keep_table<<<grid, kThreads, 0, s>>>(a);
  lab_flatten<<<grid, kThreads, 0, s>>>(a);
  lab_mark<<<grid, kThreads, 0, s>>>(a);
  const uint64_t nwmax = live_cap_ / 32 + 1;
  scan32_.run(bcnt_, bcnt_, &sc->nw, 1, nwmax, &sc->closed32, s);
  lab_compact<<<grid, kThreads, 0, s>>>(a);
  lab_count<<<grid, kThreads, 0, s>>>(a);
  scan32_.run(bcnt_, bcnt_, &sc->seg_len, 1, static_cast<uint64_t>(frame_cap_ + 1) * nwmax,
              nullptr, s);
  lab_rank<<<grid, kThreads, 0, s>>>(a);
  scan64_.run(mpk_, mpk_, &sc->closed, 1, live_cap_, &sc->members_pack, s);
  lab_scatter<<<grid, kThreads, 0, s>>>(a);
  // The few large and middle-sized components on streams of their own,
  // launched first so that their blocks are placed before the many small
  // components' launch fills the SMs: each of them is one warp's long walk,
  // which then runs beside the small ones instead of after them.
  check(cudaEventRecord(fork_, s), "cudaEventRecord");
  check(cudaStreamWaitEvent(aux_, fork_, 0), "cudaStreamWaitEvent");
  check(cudaStreamWaitEvent(aux2_, fork_, 0), "cudaStreamWaitEvent");
  lab_accept<kCompCap><<<grid_ / 4, kCompWarps * 32, kCompWarps * warp_comp_bytes<kCompCap>(),
                         aux_>>>(a, kMidCap, 0xffffffffu, 1);
  lab_accept<kMidCap><<<grid_ / 8 * kAcceptBlocks<kMidCap>, kCompWarps * 32,
                        kCompWarps * warp_comp_bytes<kMidCap>(), aux2_>>>(a, kSmallCap, kMidCap, 2);
  lab_accept<kSmallCap><<<grid, kCompWarps * 32, kCompWarps * warp_comp_bytes<kSmallCap>(), s>>>(
      a, 0u, kSmallCap, 0);
  check(cudaEventRecord(join_, aux_), "cudaEventRecord");
  check(cudaEventRecord(join2_, aux2_), "cudaEventRecord");
  check(cudaStreamWaitEvent(s, join_, 0), "cudaStreamWaitEvent");
  check(cudaStreamWaitEvent(s, join2_, 0), "cudaStreamWaitEvent");
  scan64_.run(pack_, pack_, &sc->closed, 1, live_cap_, &sc->accepted_pack, s);
  lab_write<<<grid, kThreads, 0, s>>>(a);
  scan32_.run(ocnt_, ocnt_, &sc->nw, 1, nwmax, &sc->open32, s);
  lab_carry<<<grid, kThreads, 0, s>>>(a);
  lab_finalize<<<1, 32, 0, s>>>(a);
  check(cudaGetLastError(), "launching the labeller");
  cur_ ^= 1;
}

} // namespace sf
