// Deblocking of one plane (src/loopfilter.rs:98-648, the dav1d loop-filter
// port driven per superblock row).
//
// Order.  The reference walks superblock rows top to bottom; in each it filters
// every vertical edge (per row of samples, left to right), then every
// horizontal edge (per column, top to bottom).  A line of samples across a
// vertical edge only touches its own row, and one across a horizontal edge
// only its own column, so the reference's result is fixed by two orders: along
// each row, vertical edges left to right; along each column, horizontal edges
// top to bottom -- plus the interleaving of the two directions per superblock
// row.  A horizontal edge reaches at most 6 rows below itself (the 16-wide
// luma filter), so only a 16-wide horizontal edge on the last 4-row of a
// superblock row reaches the next superblock row, whose vertical edges the
// reference filters after it.  No AV1 block geometry puts one there (a block
// >= 16 rows high starts on a multiple of 16 rows); without one, two
// frame-wide passes -- all vertical edges, then all horizontal edges -- give
// the reference's samples.  mt_deblock_plane rejects maps that have one.
//
// Parallelism.  One thread filters one line across one edge.  Two edges of one
// direction whose taps overlap (possible only with edge maps that do not
// follow the block sizes: AV1 geometry keeps the taps of neighbouring edges
// apart, 1+2 < 4, 3+4 < 8, 6+7 < 16 samples) must run in the reference's order:
// such edges form runs of consecutive overlapping edges, and the thread of a
// run's first edge filters the whole run in order while the others return.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/maroontree_b200.h"

namespace {

struct LfLimits {
  int e, i, h;
};

__host__ __device__ inline LfLimits lf_limits(int level, int sharp) {
  int i = level;
  if (sharp > 0) {
    i >>= (sharp + 3) >> 2;
    i = i < 9 - sharp ? i : 9 - sharp;
  }
  i = i > 1 ? i : 1;
  return {2 * (level + 2) + i, i, level >> 4};
}

__device__ __forceinline__ int clip3(int v, int lo, int hi) { return max(lo, min(v, hi)); }

// One line of the filter across an edge (src/loopfilter.rs:98-292): v[7 + k]
// holds the sample k places past the edge (v[6] = p0, v[7] = q0); WD is the
// filter width, so only v[7 - reach .. 7 + reach) is read.
template <int WD>
__device__ __forceinline__ void lf_core(int (&v)[14], const LfLimits L, int bd) {
  const int bm8 = bd - 8;
  const int f_flat = 1 << bm8;
  const int e = L.e << bm8, il = L.i << bm8, ht = L.h << bm8;
  const int px_max = (1 << bd) - 1;
  const int clip_lo = -128 * (1 << bm8), clip_hi = 128 * (1 << bm8) - 1;
  const int p1 = v[5], p0 = v[6], q0 = v[7], q1 = v[8];
  bool fm = abs(p1 - p0) <= il && abs(q1 - q0) <= il && abs(p0 - q0) * 2 + (abs(p1 - q1) >> 1) <= e;
  int p2 = 0, q2 = 0, p3 = 0, q3 = 0;
  if (WD > 4) {
    p2 = v[4];
    q2 = v[9];
    fm = fm && abs(p2 - p1) <= il && abs(q2 - q1) <= il;
    if (WD > 6) {
      p3 = v[3];
      q3 = v[10];
      fm = fm && abs(p3 - p2) <= il && abs(q3 - q2) <= il;
    }
  }
  if (!fm) return;
  bool flat8in = false;
  if (WD >= 6)
    flat8in = abs(p2 - p0) <= f_flat && abs(p1 - p0) <= f_flat && abs(q1 - q0) <= f_flat && abs(q2 - q0) <= f_flat;
  if (WD >= 8) flat8in = flat8in && abs(p3 - p0) <= f_flat && abs(q3 - q0) <= f_flat;
  if (WD >= 16 && flat8in) {
    const int p6 = v[0], p5 = v[1], p4 = v[2], q4 = v[11], q5 = v[12], q6 = v[13];
    const bool flat8out = abs(p6 - p0) <= f_flat && abs(p5 - p0) <= f_flat && abs(p4 - p0) <= f_flat &&
                          abs(q4 - q0) <= f_flat && abs(q5 - q0) <= f_flat && abs(q6 - q0) <= f_flat;
    if (flat8out) {
      v[1] = (p6 * 7 + p5 * 2 + p4 * 2 + p3 + p2 + p1 + p0 + q0 + 8) >> 4;
      v[2] = (p6 * 5 + p5 * 2 + p4 * 2 + p3 * 2 + p2 + p1 + p0 + q0 + q1 + 8) >> 4;
      v[3] = (p6 * 4 + p5 + p4 * 2 + p3 * 2 + p2 * 2 + p1 + p0 + q0 + q1 + q2 + 8) >> 4;
      v[4] = (p6 * 3 + p5 + p4 + p3 * 2 + p2 * 2 + p1 * 2 + p0 + q0 + q1 + q2 + q3 + 8) >> 4;
      v[5] = (p6 * 2 + p5 + p4 + p3 + p2 * 2 + p1 * 2 + p0 * 2 + q0 + q1 + q2 + q3 + q4 + 8) >> 4;
      v[6] = (p6 + p5 + p4 + p3 + p2 + p1 * 2 + p0 * 2 + q0 * 2 + q1 + q2 + q3 + q4 + q5 + 8) >> 4;
      v[7] = (p5 + p4 + p3 + p2 + p1 + p0 * 2 + q0 * 2 + q1 * 2 + q2 + q3 + q4 + q5 + q6 + 8) >> 4;
      v[8] = (p4 + p3 + p2 + p1 + p0 + q0 * 2 + q1 * 2 + q2 * 2 + q3 + q4 + q5 + q6 + q6 + 8) >> 4;
      v[9] = (p3 + p2 + p1 + p0 + q0 + q1 * 2 + q2 * 2 + q3 * 2 + q4 + q5 + q6 + q6 + q6 + 8) >> 4;
      v[10] = (p2 + p1 + p0 + q0 + q1 + q2 * 2 + q3 * 2 + q4 * 2 + q5 + q6 + q6 + q6 + q6 + 8) >> 4;
      v[11] = (p1 + p0 + q0 + q1 + q2 + q3 * 2 + q4 * 2 + q5 * 2 + q6 * 5 + 8) >> 4;
      v[12] = (p0 + q0 + q1 + q2 + q3 + q4 * 2 + q5 * 2 + q6 * 7 + 8) >> 4;
      return;
    }
  }
  if (WD >= 8 && flat8in) {
    v[4] = (p3 * 3 + 2 * p2 + p1 + p0 + q0 + 4) >> 3;
    v[5] = (p3 * 2 + p2 + 2 * p1 + p0 + q0 + q1 + 4) >> 3;
    v[6] = (p3 + p2 + p1 + 2 * p0 + q0 + q1 + q2 + 4) >> 3;
    v[7] = (p2 + p1 + p0 + 2 * q0 + q1 + q2 + q3 + 4) >> 3;
    v[8] = (p1 + p0 + q0 + 2 * q1 + q2 + q3 + q3 + 4) >> 3;
    v[9] = (p0 + q0 + q1 + 2 * q2 + q3 + q3 + q3 + 4) >> 3;
  } else if (WD == 6 && flat8in) {
    v[5] = (p2 * 3 + 2 * p1 + 2 * p0 + q0 + 4) >> 3;
    v[6] = (p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3;
    v[7] = (p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3;
    v[8] = (p0 + 2 * q0 + 2 * q1 + 2 * q2 + q2 + 4) >> 3;
  } else {
    const bool hev = abs(p1 - p0) > ht || abs(q1 - q0) > ht;
    int fv = hev ? clip3(p1 - q1, clip_lo, clip_hi) : 0;
    fv = clip3(3 * (q0 - p0) + fv, clip_lo, clip_hi);
    const int f1 = min(fv + 4, clip_hi) >> 3;
    const int f2 = min(fv + 3, clip_hi) >> 3;
    v[6] = clip3(p0 + f2, 0, px_max);
    v[7] = clip3(q0 - f1, 0, px_max);
    if (!hev) {
      const int f = (f1 + 1) >> 1;
      v[5] = clip3(p1 + f, 0, px_max);
      v[8] = clip3(q1 - f, 0, px_max);
    }
  }
}

// Samples a filter of width WD reads / writes on each side: reads
// [7 - RLO, 7 + RHI], writes [7 - WLO, 7 + WHI].
template <int WD> struct Reach;
template <> struct Reach<4> { static constexpr int RLO = 2, RHI = 1, WLO = 2, WHI = 1; };
template <> struct Reach<6> { static constexpr int RLO = 3, RHI = 2, WLO = 2, WHI = 1; };
template <> struct Reach<8> { static constexpr int RLO = 4, RHI = 3, WLO = 3, WHI = 2; };
template <> struct Reach<16> { static constexpr int RLO = 7, RHI = 6, WLO = 6, WHI = 5; };

// One line across a vertical edge at row[x0] (samples contiguous).
template <int WD>
__device__ __forceinline__ void lf_row(uint16_t* __restrict__ row, const LfLimits L, int bd) {
  using R = Reach<WD>;
  int v[14];
#pragma unroll
  for (int k = -R::RLO; k <= R::RHI; k++) v[7 + k] = row[k];
  lf_core<WD>(v, L, bd);
#pragma unroll
  for (int k = -R::WLO; k <= R::WHI; k++) row[k] = (uint16_t)v[7 + k];
}

// Four columns (x0 .. x0 + 3) across a horizontal edge at row y0: 8-byte row
// loads and stores (col points at sample (x0, y0), 8-byte aligned).
template <int WD>
__device__ __forceinline__ void lf_cols4(uint16_t* __restrict__ col, long stride, const LfLimits L, int bd) {
  using R = Reach<WD>;
  int v[4][14];
#pragma unroll
  for (int k = -R::RLO; k <= R::RHI; k++) {
    const uint2 q = *reinterpret_cast<const uint2*>(col + k * stride);
    v[0][7 + k] = q.x & 0xffff;
    v[1][7 + k] = q.x >> 16;
    v[2][7 + k] = q.y & 0xffff;
    v[3][7 + k] = q.y >> 16;
  }
#pragma unroll
  for (int l = 0; l < 4; l++) lf_core<WD>(v[l], L, bd);
#pragma unroll
  for (int k = -R::WLO; k <= R::WHI; k++) {
    uint2 q;
    q.x = (unsigned)v[0][7 + k] | ((unsigned)v[1][7 + k] << 16);
    q.y = (unsigned)v[2][7 + k] | ((unsigned)v[3][7 + k] << 16);
    *reinterpret_cast<uint2*>(col + k * stride) = q;
  }
}

// Filter width class of a block dimension in 4-sample units
// (src/loopfilter.rs:396-412): luma 4/8/16, chroma 4/6.
__host__ __device__ __forceinline__ int lf_cls(int d, bool luma) {
  return luma ? (d == 1 ? 0 : (d == 2 ? 1 : 2)) : (d >= 2);
}
__host__ __device__ __forceinline__ int lf_wd(int wcls, bool luma) { return luma ? 4 << wcls : 4 + 2 * wcls; }
// Samples a filter of width wd reads before / after the edge (it writes fewer).
__host__ __device__ __forceinline__ int lf_reach_lo(int wd) {
  return wd == 16 ? 7 : (wd == 8 ? 4 : (wd == 6 ? 3 : 2));
}
__host__ __device__ __forceinline__ int lf_reach_hi(int wd) {
  return wd == 16 ? 6 : (wd == 8 ? 3 : (wd == 6 ? 2 : 1));
}

// The edges of one row of cells (vertical edges, i = 4x4 column) or one
// column of cells (horizontal edges, i = 4x4 row): cell i sits at
// map[base + i * step], the block before the edge at map[base + (i-1) * step].
struct EdgeLine {
  const uint8_t* dim;   // block extent across the edge, in 4-sample units
  const uint8_t* flag;  // block-start flags, or null for the alignment rule
  long base, step;
  int n4;               // cells along the line inside the visible window
  int len;              // samples along the line in the padded plane
  bool luma;
};

// Filter width of the edge at cell i, 0 where none is filtered: outside
// 1..n4-1, no block start there, or taps that would leave the row / plane (the
// reference indexes outside its row there; no AV1 geometry reaches it).
__host__ __device__ __forceinline__ int edge_wd(const EdgeLine& e, int i) {
  if (i < 1 || i >= e.n4) return 0;
  const long idx = e.base + (long)i * e.step;
  const int cur = e.dim[idx];
  if (cur == 0) return 0;
  const bool present = e.flag ? e.flag[idx] != 0 : (i % cur == 0);
  if (!present) return 0;
  const int prev = e.dim[idx - e.step];
  const int a = lf_cls(cur, e.luma), b = lf_cls(prev, e.luma);
  const int wd = lf_wd(a < b ? a : b, e.luma);
  if (4 * i - lf_reach_lo(wd) < 0 || 4 * i + lf_reach_hi(wd) >= e.len) return 0;
  return wd;
}

// Do the taps of edges i < k (widths wi, wk) share a sample?
__host__ __device__ __forceinline__ bool taps_overlap(int i, int wi, int k, int wk) {
  return 4 * i + lf_reach_hi(wi) >= 4 * k - lf_reach_lo(wk);
}

// Window of edge widths for cells i-6 .. i+3 (taps reach at most 3 cells).
struct EdgeWindow {
  int wd[10];
  __device__ __forceinline__ int at(int d) const { return wd[d + 6]; }  // d in -6..3
};

// Does the edge at offset d (-3..0) of the window overlap a neighbour within 3 cells?
__device__ __forceinline__ bool window_involved(const EdgeWindow& w, int i, int d) {
  const int wd = w.at(d);
  for (int k = d - 3; k <= d + 3; k++) {
    if (k == d || k < -6 || k > 3) continue;
    const int wk = w.at(k);
    if (!wk) continue;
    if (k < d ? taps_overlap(i + k, wk, i + d, wd) : taps_overlap(i + d, wd, i + k, wk)) return true;
  }
  return false;
}

__device__ __forceinline__ bool involved_at(const EdgeLine& e, int i, int wd) {
  for (int k = i - 3; k <= i + 3; k++) {
    if (k == i) continue;
    const int wk = edge_wd(e, k);
    if (!wk) continue;
    if (k < i ? taps_overlap(k, wk, i, wd) : taps_overlap(i, wd, k, wk)) return true;
  }
  return false;
}

// Is the edge at cell i filtered by this thread, and which edges follow it?
// Returns the width of edge i when this thread owns it (0 otherwise); *run is
// set when i heads a run of edges whose taps overlap (the thread then filters
// the whole run in order, see run_next).
__device__ __forceinline__ int own_edge(const EdgeLine& e, int i, bool* run) {
  EdgeWindow w;
#pragma unroll
  for (int d = -6; d <= 3; d++) w.wd[d + 6] = edge_wd(e, i + d);
  const int wd = w.at(0);
  *run = false;
  if (!wd) return 0;
  if (!window_involved(w, i, 0)) return wd;
  // Part of a run: only the run's first edge proceeds.
#pragma unroll
  for (int d = -1; d >= -3; d--) {
    if (w.at(d)) {
      if (window_involved(w, i, d)) return 0;
      break;
    }
  }
  *run = true;
  return wd;
}

// The edge after cur in its run, or 0 (with its width in *nw).
__device__ __forceinline__ int run_next(const EdgeLine& e, int cur, int* nw) {
  for (int k = cur + 1; k <= cur + 3; k++) {
    const int wk = edge_wd(e, k);
    if (wk) {
      *nw = involved_at(e, k, wk) ? wk : 0;
      return *nw ? k : 0;
    }
  }
  *nw = 0;
  return 0;
}

struct PlaneArgs {
  int w, h, w4, h4, nc4, bd, luma;
  LfLimits L;
};

__device__ __forceinline__ void vert_cell(uint16_t* __restrict__ px, const PlaneArgs& a, int r4, int c4, int wd) {
  uint16_t* base = px + (size_t)(r4 * 4) * a.w + c4 * 4;
#pragma unroll 1
  for (int l = 0; l < 4; l++) {
    uint16_t* row = base + (size_t)l * a.w;
    switch (wd) {
      case 4: lf_row<4>(row, a.L, a.bd); break;
      case 6: lf_row<6>(row, a.L, a.bd); break;
      case 8: lf_row<8>(row, a.L, a.bd); break;
      default: lf_row<16>(row, a.L, a.bd); break;
    }
  }
}

__device__ __forceinline__ void horz_cell(uint16_t* __restrict__ px, const PlaneArgs& a, int r4, int c4, int wd) {
  uint16_t* col = px + (size_t)(r4 * 4) * a.w + c4 * 4;
  switch (wd) {
    case 4: lf_cols4<4>(col, a.w, a.L, a.bd); break;
    case 6: lf_cols4<6>(col, a.w, a.L, a.bd); break;
    case 8: lf_cols4<8>(col, a.w, a.L, a.bd); break;
    default: lf_cols4<16>(col, a.w, a.L, a.bd); break;
  }
}

// Vertical edges: one thread per 4x4 cell (edge column c4, cell row r4),
// filtering the cell's four rows.
__global__ void __launch_bounds__(128) lf_vert_kernel(uint16_t* __restrict__ px, PlaneArgs a,
                                                      const uint8_t* __restrict__ bw4,
                                                      const uint8_t* __restrict__ vedge4) {
  const int c4 = blockIdx.x * blockDim.x + threadIdx.x;
  const int r4 = blockIdx.y;
  if (c4 >= a.w4) return;
  const EdgeLine e{bw4, vedge4, (long)r4 * a.nc4, 1, a.w4, a.w, a.luma != 0};
  bool run;
  int wd = own_edge(e, c4, &run);
  if (!wd) return;
  int cur = c4;
  while (true) {
    vert_cell(px, a, r4, cur, wd);
    if (!run) return;
    cur = run_next(e, cur, &wd);
    if (!cur) return;
  }
}

// Horizontal edges: one thread per 4x4 cell (cell column c4, edge row r4),
// filtering the cell's four columns with 8-byte row accesses.
__global__ void __launch_bounds__(128) lf_horz_kernel(uint16_t* __restrict__ px, PlaneArgs a,
                                                      const uint8_t* __restrict__ bh4,
                                                      const uint8_t* __restrict__ hedge4) {
  const int c4 = blockIdx.x * blockDim.x + threadIdx.x;
  const int r4 = blockIdx.y;
  if (c4 >= a.w4) return;
  const EdgeLine e{bh4, hedge4, (long)c4, a.nc4, a.h4, a.h, a.luma != 0};
  bool run;
  int wd = own_edge(e, r4, &run);
  if (!wd) return;
  int cur = r4;
  while (true) {
    horz_cell(px, a, cur, c4, wd);
    if (!run) return;
    cur = run_next(e, cur, &wd);
    if (!cur) return;
  }
}

// ---------------------------------------------------------------------------
// The frame path.  The fused kernel filters each 64x64 tile in shared memory:
// the tile's region (a 16-sample halo holds every tap its samples depend on)
// and the block maps of the region's cells are loaded once, the edge widths
// computed there, then all vertical edges and all horizontal edges filtered,
// reading the unfiltered plane and writing the tile once into the filtered
// plane (a separate buffer: neighbouring tiles read their halos while others
// are being written) -- the samples of the frame-wide two-pass order.  Each
// tile also checks whether an edge of its own cells has taps overlapping one
// of the next three edges of its line (never with AV1 block geometry); if any
// tile finds one, it raises a flag, the unfiltered planes are copied over the
// filtered ones, and the two-pass kernels above (which keep overlapping runs
// in the reference's order) filter them in place.

struct FramePlane {
  const uint16_t* in;  // the unfiltered plane (never written while the fused kernel runs)
  uint16_t* px;        // the filtered plane
  const uint8_t* bw4;
  const uint8_t* bh4;
  const uint8_t* vedge4;
  const uint8_t* hedge4;
  PlaneArgs a;
  int nr4;  // map rows
  int on;
};
struct FrameArgs {
  FramePlane p[3];
};

// One line across a horizontal edge in shared memory (col: the sample on the
// edge's lower side, rows pitch apart).
template <int WD>
__device__ __forceinline__ void lf_col(uint16_t* col, int pitch, const LfLimits L, int bd) {
  using R = Reach<WD>;
  int v[14];
#pragma unroll
  for (int k = -R::RLO; k <= R::RHI; k++) v[7 + k] = col[k * pitch];
  lf_core<WD>(v, L, bd);
#pragma unroll
  for (int k = -R::WLO; k <= R::WHI; k++) col[k * pitch] = (uint16_t)v[7 + k];
}

constexpr int kFT = 64;              // output tile
constexpr int kFH = 16;              // halo: every tap of an edge that writes the tile
constexpr int kFR = kFT + 2 * kFH;   // region side, samples
constexpr int kFP = kFR + 2;         // row pitch (odd in 4-byte words: column walks are conflict-free)
constexpr int kFC = kFR / 4;         // region side, cells
constexpr int kFM = kFC + 1;         // map block side: the region's cells and the cells before them
constexpr int kFE0 = 3, kFE1 = 21;   // region cells whose edges write the tile (4c - 6 <= 79, 4c + 5 >= 16)
constexpr int kFThreads = 256;

// edge_wd on the map block in shared memory: the edge before map cell (mr, mc)
// along a line (dv = 1: vertical edge, the previous cell to the left; else
// horizontal, the previous cell above), i its cell index along the line.
__device__ __forceinline__ int smem_edge_wd(const uint8_t* dim, const uint8_t* flag, bool has_flag, int mr, int mc,
                                            bool vert, int i, int n4, int len, bool luma) {
  if (i < 1 || i >= n4) return 0;
  const int cur = dim[mr * kFM + mc];
  if (cur == 0) return 0;
  const bool present = has_flag ? flag[mr * kFM + mc] != 0 : (i % cur == 0);
  if (!present) return 0;
  const int prev = vert ? dim[mr * kFM + mc - 1] : dim[(mr - 1) * kFM + mc];
  const int a = lf_cls(cur, luma), b = lf_cls(prev, luma);
  const int wd = lf_wd(a < b ? a : b, luma);
  if (4 * i - lf_reach_lo(wd) < 0 || 4 * i + lf_reach_hi(wd) >= len) return 0;
  return wd;
}

// Width class of a filter width (4, 6, 8, 16 -> 0..3).
__device__ __forceinline__ int wd_class(int wd) { return wd == 4 ? 0 : (wd == 6 ? 1 : (wd == 8 ? 2 : 3)); }

constexpr int kFMaxV = (kFC - 2) * (kFE1 - kFE0 + 1);  // vertical edges filtered: cell rows 1..kFC-2
constexpr int kFMaxH = (kFE1 - kFE0 + 1) * (kFT / 4);  // horizontal edges filtered: the tile's cell columns

__global__ void __launch_bounds__(kFThreads) lf_fused_kernel(FrameArgs fa, int* __restrict__ overlap) {
  const FramePlane& P = fa.p[blockIdx.z];
  if (!P.px || (!P.on && P.in == P.px)) return;  // no plane, or unfiltered in place
  const PlaneArgs& a = P.a;
  const int x0 = blockIdx.x * kFT, y0 = blockIdx.y * kFT;
  if (x0 >= a.w || y0 >= a.h) return;
  __shared__ __align__(16) uint16_t S[kFR * kFP];
  __shared__ uint8_t vw[kFC * kFC], hw[kFC * kFC];
  __shared__ uint8_t mb[4][kFM * kFM];  // bw4, bh4, vedge4, hedge4 of the map block
  __shared__ uint16_t vlist[4][kFMaxV], hlist[4][kFMaxH];  // active edges by width class: cell row << 8 | col
  __shared__ int nv[4], nh[4], bad;
  const int rx0 = x0 - kFH, ry0 = y0 - kFH, c0 = rx0 / 4, r0 = ry0 / 4;
  const int t = threadIdx.x;
  const bool on = P.on;  // an unfiltered plane is copied through
  if (t < 4) {
    nv[t] = 0;
    nh[t] = 0;
  }
  if (t == 0) bad = 0;
  // the region's samples, 4 at a time (8-byte loads: rx0, the plane width and
  // the row starts are multiples of 4 samples)
  for (int i = t; i < kFR * (kFR / 4); i += kFThreads) {
    const int r = i / (kFR / 4), c4 = (i - r * (kFR / 4)) * 4;
    const int gy = ry0 + r, gx = rx0 + c4;
    uint2 v = make_uint2(0, 0);
    if (gy >= 0 && gy < a.h && gx >= 0 && gx < a.w)
      v = *reinterpret_cast<const uint2*>(P.in + (size_t)gy * a.w + gx);
    uint32_t* d = reinterpret_cast<uint32_t*>(&S[r * kFP + c4]);
    d[0] = v.x;
    d[1] = v.y;
  }
  // the map block: cells (r0 - 1 .. r0 + kFC - 1) x (c0 - 1 .. c0 + kFC - 1)
  if (on)
    for (int i = t; i < kFM * kFM; i += kFThreads) {
      const int mr = i / kFM, mc = i - mr * kFM;
      const int gr = r0 - 1 + mr, gc = c0 - 1 + mc;
      const bool in = gr >= 0 && gr < P.nr4 && gc >= 0 && gc < a.nc4;
      const long idx = (long)gr * a.nc4 + gc;
      mb[0][i] = in ? P.bw4[idx] : 0;
      mb[1][i] = in ? P.bh4[idx] : 0;
      mb[2][i] = in && P.vedge4 ? P.vedge4[idx] : 0;
      mb[3][i] = in && P.hedge4 ? P.hedge4[idx] : 0;
    }
  __syncthreads();
  // the region's edge widths (none outside the visible cells), and the lists
  // of the edges this tile filters
  if (on)
    for (int i = t; i < kFC * kFC; i += kFThreads) {
      const int cr = i / kFC, cc = i - cr * kFC;
      const int gr = r0 + cr, gc = c0 + cc;
      const bool in = gr >= 0 && gr < a.h4 && gc >= 0 && gc < a.w4;
      const int v = in ? smem_edge_wd(mb[0], mb[2], P.vedge4 != nullptr, cr + 1, cc + 1, true, gc, a.w4, a.w, a.luma)
                       : 0;
      const int h = in ? smem_edge_wd(mb[1], mb[3], P.hedge4 != nullptr, cr + 1, cc + 1, false, gr, a.h4, a.h, a.luma)
                       : 0;
      vw[i] = (uint8_t)v;
      hw[i] = (uint8_t)h;
      if (v && cr >= 1 && cr <= kFC - 2 && cc >= kFE0 && cc <= kFE1) {
        const int k = wd_class(v);
        vlist[k][atomicAdd(&nv[k], 1)] = (uint16_t)(cr << 8 | cc);
      }
      if (h && cr >= kFE0 && cr <= kFE1 && cc >= kFH / 4 && cc < (kFH + kFT) / 4) {
        const int k = wd_class(h);
        hlist[k][atomicAdd(&nh[k], 1)] = (uint16_t)(cr << 8 | cc);
      }
    }
  __syncthreads();
  // overlapping taps between an edge of the tile's own cells and the next
  // three edges of its line (every such pair has its first edge in exactly
  // one tile): the two-pass kernels then redo the whole frame
  if (on) {
    bool o = false;
    for (int i = t; i < 2 * (kFT / 4) * (kFT / 4); i += kFThreads) {
      const bool vert = i < (kFT / 4) * (kFT / 4);
      const int j = vert ? i : i - (kFT / 4) * (kFT / 4);
      const int ar = kFH / 4 + j / (kFT / 4), ac = kFH / 4 + j % (kFT / 4);  // line, and position along it
      const uint8_t* w = vert ? vw : hw;
      const int cell = vert ? ar * kFC + ac : ac * kFC + ar;
      const int wd = w[cell];
      if (!wd) continue;
      const int gi = vert ? c0 + ac : r0 + ac;
      for (int k = 1; k <= 3; k++) {
        const int wk = w[vert ? cell + k : cell + k * kFC];
        if (wk && taps_overlap(gi, wd, gi + k, wk)) o = true;
      }
    }
    if (o) bad = 1;
  }
  __syncthreads();
  if (bad) {
    if (t == 0) atomicExch(overlap, 1);
    return;
  }
  // vertical edges, width class by class (four rows per edge; the rows of
  // cell rows 1 .. kFC-2 cover every row the horizontal pass reads)
  if (on) {
    int base = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int n = 4 * nv[k];
      for (int i = (t - base) & (kFThreads - 1); i < n; i += kFThreads) {
        const int e = vlist[k][i >> 2];
        uint16_t* row = &S[(4 * (e >> 8) + (i & 3)) * kFP + 4 * (e & 255)];
        switch (k) {  // 8-bit samples: the entry accepts no other depth
          case 0: lf_row<4>(row, a.L, 8); break;
          case 1: lf_row<6>(row, a.L, 8); break;
          case 2: lf_row<8>(row, a.L, 8); break;
          default: lf_row<16>(row, a.L, 8); break;
        }
      }
      base = (base + n) & (kFThreads - 1);
    }
  }
  __syncthreads();
  // horizontal edges on the tile's columns, width class by class
  if (on) {
    int base = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int n = 4 * nh[k];
      for (int i = (t - base) & (kFThreads - 1); i < n; i += kFThreads) {
        const int e = hlist[k][i >> 2];
        uint16_t* cp = &S[(4 * (e >> 8)) * kFP + 4 * (e & 255) + (i & 3)];
        switch (k) {
          case 0: lf_col<4>(cp, kFP, a.L, 8); break;
          case 1: lf_col<6>(cp, kFP, a.L, 8); break;
          case 2: lf_col<8>(cp, kFP, a.L, 8); break;
          default: lf_col<16>(cp, kFP, a.L, 8); break;
        }
      }
      base = (base + n) & (kFThreads - 1);
    }
  }
  __syncthreads();
  for (int i = t; i < kFT * (kFT / 4); i += kFThreads) {
    const int r = i / (kFT / 4), c4 = (i - r * (kFT / 4)) * 4;
    const int gy = y0 + r, gx = x0 + c4;
    if (gy < a.h && gx < a.w) {
      const uint32_t* sp = reinterpret_cast<const uint32_t*>(&S[(kFH + r) * kFP + kFH + c4]);
      *reinterpret_cast<uint2*>(P.px + (size_t)gy * a.w + gx) = make_uint2(sp[0], sp[1]);
    }
  }
}

// With overlapping taps: the unfiltered planes into the filtered ones (where
// they are separate buffers), for the two-pass kernels to filter in place.
__global__ void __launch_bounds__(256) lf_copy_frame_kernel(FrameArgs fa, const int* __restrict__ overlap) {
  if (!*overlap) return;
  const FramePlane& P = fa.p[blockIdx.z];
  if (!P.px || P.in == P.px) return;
  const long n = (long)P.a.w * P.a.h / 2;  // sample pairs
  const uint32_t* src = reinterpret_cast<const uint32_t*>(P.in);
  uint32_t* dst = reinterpret_cast<uint32_t*>(P.px);
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) dst[i] = src[i];
}

// The two-pass kernels over all planes of the frame, run only when the
// classify pass found overlapping taps.
__global__ void __launch_bounds__(128) lf_vert_frame_kernel(FrameArgs fa, const int* __restrict__ overlap) {
  if (!*overlap) return;
  const FramePlane& P = fa.p[blockIdx.z];
  if (!P.on) return;
  const PlaneArgs& a = P.a;
  const long n = (long)a.w4 * a.h4;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int r4 = (int)(i / a.w4), c4 = (int)(i - (long)r4 * a.w4);
    const EdgeLine e{P.bw4, P.vedge4, (long)r4 * a.nc4, 1, a.w4, a.w, a.luma != 0};
    bool run;
    int wd = own_edge(e, c4, &run);
    int cur = c4;
    while (wd) {
      vert_cell(P.px, a, r4, cur, wd);
      if (!run) break;
      cur = run_next(e, cur, &wd);
      if (!cur) break;
    }
  }
}

__global__ void __launch_bounds__(128) lf_horz_frame_kernel(FrameArgs fa, const int* __restrict__ overlap) {
  if (!*overlap) return;
  const FramePlane& P = fa.p[blockIdx.z];
  if (!P.on) return;
  const PlaneArgs& a = P.a;
  const long n = (long)a.w4 * a.h4;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int r4 = (int)(i / a.w4), c4 = (int)(i - (long)r4 * a.w4);
    const EdgeLine e{P.bh4, P.hedge4, (long)c4, a.nc4, a.h4, a.h, a.luma != 0};
    bool run;
    int wd = own_edge(e, r4, &run);
    int cur = r4;
    while (wd) {
      horz_cell(P.px, a, cur, c4, wd);
      if (!run) break;
      cur = run_next(e, cur, &wd);
      if (!cur) break;
    }
  }
}

int check_plane(int32_t w, int32_t h, int32_t vis_w, int32_t vis_h, int32_t nc4, int32_t level, int32_t sharp,
                int32_t bd) {
  if (w <= 0 || h <= 0 || (w & 3) || (h & 3)) return MT_ERR_INVALID_INPUT;
  if (vis_w <= 0 || vis_h <= 0 || vis_w > w || vis_h > h) return MT_ERR_INVALID_INPUT;
  if (nc4 < (vis_w + 3) / 4 || level < 0 || level > 63 || sharp < 0 || sharp > 7) return MT_ERR_INVALID_INPUT;
  if (bd != 8) return MT_ERR_UNSUPPORTED;
  return MT_OK;
}

// A 16-wide horizontal edge on the last 4-row of a 64-row superblock row
// (the only edge the two-pass order would filter out of the reference's order).
bool has_superblock_crossing(int32_t w, int32_t h, int32_t vis_w, int32_t vis_h, const uint8_t* bh4,
                             const uint8_t* hedge4, int32_t nc4) {
  const int w4 = (vis_w + 3) / 4, h4 = (vis_h + 3) / 4;
  (void)w;
  for (int t = 16; t < h4; t += 16)
    for (int c4 = 0; c4 < w4; c4++) {
      const EdgeLine e{bh4, hedge4, (long)c4, nc4, h4, h, true};
      if (edge_wd(e, t - 1) == 16) return true;
    }
  return false;
}

// Chroma deblocking geometry (src/coder/frame_deblock.rs:87-152, variant 1):
// per chroma 4x4 cell, the covering luma PREDICTION block's size >> subsampling,
// at least 1 and at most 8 (32 px, the largest chroma transform); edges by the
// alignment rule.
__global__ void chroma_geom_kernel(const uint8_t* __restrict__ pbw4, const uint8_t* __restrict__ pbh4, int nc4,
                                   int cnc4, int cnr4, int ss_hor, int ss_ver, uint8_t* __restrict__ cbw4,
                                   uint8_t* __restrict__ cbh4) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnc4 * cnr4) return;
  const int cr = i / cnc4, cc = i - cr * cnc4;
  const long li = (long)(cr << ss_ver) * nc4 + (cc << ss_hor);
  cbw4[i] = (uint8_t)min(max(pbw4[li] >> ss_hor, 1), 8);
  cbh4[i] = (uint8_t)min(max(pbh4[li] >> ss_ver, 1), 8);
}

int check_frame(const mt_deblock_frame_params* p) {
  if (!p) return MT_ERR_INVALID_INPUT;
  if (p->w8 <= 0 || p->h8 <= 0 || (p->w8 & 7) || (p->h8 & 7)) return MT_ERR_INVALID_INPUT;
  if (p->disp_w <= p->w8 - 8 || p->disp_w > p->w8 || p->disp_h <= p->h8 - 8 || p->disp_h > p->h8)
    return MT_ERR_INVALID_INPUT;
  if (p->sub_x < 0 || p->sub_x > 1 || p->sub_y < 0 || p->sub_y > p->sub_x) return MT_ERR_INVALID_INPUT;
  if (p->bd != 8) return MT_ERR_UNSUPPORTED;
  return MT_OK;
}

// Scratch of the frame entries: the chroma block maps, the overlap flag and
// the unfiltered planes of an in-place call.
struct FrameLayout {
  size_t cbw4, cbh4, flag, snap[3], total;
};

FrameLayout frame_layout(const mt_deblock_frame_params& p) {
  auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
  const size_t nch = (size_t)((p.w8 >> p.sub_x) / 4) * ((p.h8 >> p.sub_y) / 4);
  FrameLayout L;
  size_t o = 0;
  L.cbw4 = o;
  o += up(nch);
  L.cbh4 = o;
  o += up(nch);
  L.flag = o;
  o += 256;
  const size_t ny = (size_t)p.w8 * p.h8 * 2, nc = (size_t)(p.w8 >> p.sub_x) * (p.h8 >> p.sub_y) * 2;
  for (int pl = 0; pl < 3; pl++) {  // the unfiltered planes of an in-place call
    L.snap[pl] = o;
    o += up(pl ? (p.mono ? 0 : nc) : ny);
  }
  L.total = o;
  return L;
}

}  // namespace

namespace mth {
// Kernels the calling thread's last mt_deblock_frame_device launched.
thread_local int deblock_last_launches = 0;
}  // namespace mth

namespace {

// The frame deblocking from the unfiltered planes in_* (null: the filtered
// planes themselves, snapshotted into the scratch first) into the filtered
// planes d_*.
int deblock_frame(const uint16_t* in_y, const uint16_t* in_u, const uint16_t* in_v, uint16_t* d_y, uint16_t* d_u,
                  uint16_t* d_v, const uint8_t* d_blk4, const uint8_t* d_blk4h, const uint8_t* d_blk4v,
                  const uint8_t* d_blk4t, const uint8_t* d_pblk4, const uint8_t* d_pblk4h,
                  const mt_deblock_frame_params* prm, int32_t lvl_y, int32_t lvl_u, int32_t lvl_v, void* d_scratch,
                  void* stream) {
  mth::deblock_last_launches = 0;
  int rc = check_frame(prm);
  if (rc != MT_OK) return rc;
  if (lvl_y < 0 || lvl_y > 63 || lvl_u < 0 || lvl_u > 63 || lvl_v < 0 || lvl_v > 63) return MT_ERR_INVALID_INPUT;
  const bool in_place = in_y == nullptr;
  if (in_place && lvl_y == 0) return MT_OK;  // chroma is filtered only with luma
  const bool want_uv = !prm->mono && lvl_y > 0 && (lvl_u > 0 || lvl_v > 0);  // chroma is filtered
  if (!d_y || !d_scratch) return MT_ERR_INVALID_INPUT;
  if (want_uv && (!d_u || !d_v || (!in_place && (!in_u || !in_v)))) return MT_ERR_INVALID_INPUT;
  // chroma planes to carry (filtered, or copied through by an out-of-place call)
  const bool planes_uv = !prm->mono && d_u && d_v && (in_place || (in_u && in_v));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int cw8 = prm->w8 >> prm->sub_x, ch8 = prm->h8 >> prm->sub_y;
  const size_t ny = (size_t)prm->w8 * prm->h8 * 2, nc = (size_t)cw8 * ch8 * 2;
  if (lvl_y == 0) {  // the planes as they are
    if (cudaMemcpyAsync(d_y, in_y, ny, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return MT_ERR_DEVICE;
    if (planes_uv && (cudaMemcpyAsync(d_u, in_u, nc, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
                      cudaMemcpyAsync(d_v, in_v, nc, cudaMemcpyDeviceToDevice, st) != cudaSuccess))
      return MT_ERR_DEVICE;
    return MT_OK;
  }
  const int sharp = 7;
  const int nc4 = prm->w8 / 4;
  const bool chroma = want_uv;
  if (!d_blk4 || !d_blk4h) return MT_ERR_INVALID_INPUT;
  if (chroma && (!d_pblk4 || !d_pblk4h)) return MT_ERR_INVALID_INPUT;
  const FrameLayout L = frame_layout(*prm);
  uint8_t* s = static_cast<uint8_t*>(d_scratch);
  FrameArgs fa = {};
  int launches = 0;
  auto plane = [&](int k, const uint16_t* in, uint16_t* px, int w, int h, int vis_w, int vis_h, const uint8_t* bw4,
                   const uint8_t* bh4, const uint8_t* ve, const uint8_t* he, int pnc4, int level, bool luma) -> int {
    const int r = check_plane(w, h, vis_w, vis_h, pnc4, level, sharp, prm->bd);
    if (r != MT_OK) return r;
    if ((reinterpret_cast<uintptr_t>(px) | reinterpret_cast<uintptr_t>(in)) & 7)
      return MT_ERR_INVALID_INPUT;  // paired and 8-byte row accesses
    FramePlane& P = fa.p[k];
    P.in = in;
    P.px = px;
    P.bw4 = bw4;
    P.bh4 = bh4;
    P.vedge4 = ve;
    P.hedge4 = he;
    P.nr4 = h / 4;
    P.a.w = w;
    P.a.h = h;
    P.a.w4 = (vis_w + 3) / 4;
    P.a.h4 = (vis_h + 3) / 4;
    P.a.nc4 = pnc4;
    P.a.bd = prm->bd;
    P.a.luma = luma;
    P.a.L = lf_limits(level, sharp);
    P.on = level > 0;
    if (in_place && P.on) {  // the unfiltered plane, read by the fused kernel
      uint16_t* snap = reinterpret_cast<uint16_t*>(s + L.snap[k]);
      if (cudaMemcpyAsync(snap, px, (size_t)w * h * 2, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return MT_ERR_DEVICE;
      P.in = snap;
    }
    return MT_OK;
  };
  if ((rc = plane(0, in_y, d_y, prm->w8, prm->h8, prm->disp_w, prm->disp_h, d_blk4, d_blk4h, d_blk4v, d_blk4t, nc4,
                  lvl_y, true)) != MT_OK)
    return rc;
  if (planes_uv) {
    const int cnc4 = cw8 / 4, cnr4 = ch8 / 4;
    uint8_t* cbw4 = s + L.cbw4;
    uint8_t* cbh4 = s + L.cbh4;
    if (chroma) {
      const size_t n = (size_t)cnc4 * cnr4;
      chroma_geom_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_pblk4, d_pblk4h, nc4, cnc4, cnr4, prm->sub_x,
                                                                      prm->sub_y, cbw4, cbh4);
      ++launches;
    }
    const int vis_w = (prm->disp_w + (1 << prm->sub_x) - 1) >> prm->sub_x;
    const int vis_h = (prm->disp_h + (1 << prm->sub_y) - 1) >> prm->sub_y;
    if ((rc = plane(1, in_place ? d_u : in_u, d_u, cw8, ch8, vis_w, vis_h, cbw4, cbh4, nullptr, nullptr, cnc4,
                    chroma ? lvl_u : 0, false)) != MT_OK ||
        (rc = plane(2, in_place ? d_v : in_v, d_v, cw8, ch8, vis_w, vis_h, cbw4, cbh4, nullptr, nullptr, cnc4,
                    chroma ? lvl_v : 0, false)) != MT_OK)
      return rc;
  }
  int* flag = reinterpret_cast<int*>(s + L.flag);
  if (cudaMemsetAsync(flag, 0, sizeof(int), st) != cudaSuccess) return MT_ERR_DEVICE;
  const long cells = (long)fa.p[0].a.w4 * fa.p[0].a.h4;  // the largest plane
  lf_fused_kernel<<<dim3((prm->w8 + kFT - 1) / kFT, (prm->h8 + kFT - 1) / kFT, 3), kFThreads, 0, st>>>(fa, flag);
  // the fallback, gated on the flag (small grids: they return at once without it)
  const int gs = (int)std::min<long>((cells + 255) / 256, 296);
  lf_copy_frame_kernel<<<dim3(gs, 1, 3), 256, 0, st>>>(fa, flag);
  launches += 2;
  const int g2 = (int)std::min<long>((cells + 127) / 128, 592);
  lf_vert_frame_kernel<<<dim3(g2, 1, 3), 128, 0, st>>>(fa, flag);
  lf_horz_frame_kernel<<<dim3(g2, 1, 3), 128, 0, st>>>(fa, flag);
  launches += 2;
  mth::deblock_last_launches = launches;
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // namespace

extern "C" {

int mt_loop_filter_levels(int32_t base_q_idx, int32_t sub_x, int32_t sub_y, int32_t* lvl_y, int32_t* lvl_uv,
                          int32_t* sharp) {
  if (base_q_idx < 0 || base_q_idx > 255 || sub_x < 0 || sub_x > 1 || sub_y < 0 || sub_y > 1)
    return MT_ERR_INVALID_INPUT;
  const int q = base_q_idx;
  const int sub = sub_x + sub_y;
  const float uv_scale = sub == 2 ? 0.5f : 1.0f;
  const int ly = std::min(std::max((int)roundf((float)(q / 8) * 1.0f), 0), 40);
  int luv = 0;
  if (ly > 0) luv = std::min(std::max(std::max((int)roundf((float)(q / 10) * uv_scale), 1), 0), 32);
  if (lvl_y) *lvl_y = ly;
  if (lvl_uv) *lvl_uv = luv;
  if (sharp) *sharp = 7;
  return MT_OK;
}

size_t mt_deblock_frame_scratch_bytes(const mt_deblock_frame_params* prm) {
  if (check_frame(prm) != MT_OK) return 0;
  return frame_layout(*prm).total;
}

int mt_deblock_plane_device(uint16_t* d_px, int32_t w, int32_t h, int32_t vis_w, int32_t vis_h, const uint8_t* d_bw4,
                            const uint8_t* d_bh4, const uint8_t* d_vedge4, const uint8_t* d_hedge4, int32_t nc4,
                            int32_t level, int32_t sharp, int32_t is_luma, int32_t bd, void* stream) {
  int rc = check_plane(w, h, vis_w, vis_h, nc4, level, sharp, bd);
  if (rc != MT_OK) return rc;
  if (level == 0) return MT_OK;
  if (!d_px || !d_bw4 || !d_bh4) return MT_ERR_INVALID_INPUT;
  if (reinterpret_cast<uintptr_t>(d_px) & 7) return MT_ERR_INVALID_INPUT;  // 8-byte row accesses
  PlaneArgs a;
  a.w = w;
  a.h = h;
  a.w4 = (vis_w + 3) / 4;
  a.h4 = (vis_h + 3) / 4;
  a.nc4 = nc4;
  a.bd = bd;
  a.luma = is_luma;
  a.L = lf_limits(level, sharp);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int T = 128;
  if (a.w4 > 1) lf_vert_kernel<<<dim3((a.w4 + T - 1) / T, a.h4), T, 0, st>>>(d_px, a, d_bw4, d_vedge4);
  if (a.h4 > 1) lf_horz_kernel<<<dim3((a.w4 + T - 1) / T, a.h4), T, 0, st>>>(d_px, a, d_bh4, d_hedge4);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_deblock_frame_device(uint16_t* d_y, uint16_t* d_u, uint16_t* d_v, const uint8_t* d_blk4,
                            const uint8_t* d_blk4h, const uint8_t* d_blk4v, const uint8_t* d_blk4t,
                            const uint8_t* d_pblk4, const uint8_t* d_pblk4h, const mt_deblock_frame_params* prm,
                            int32_t lvl_y, int32_t lvl_u, int32_t lvl_v, void* d_scratch, void* stream) {
  return deblock_frame(nullptr, nullptr, nullptr, d_y, d_u, d_v, d_blk4, d_blk4h, d_blk4v, d_blk4t, d_pblk4, d_pblk4h,
                       prm, lvl_y, lvl_u, lvl_v, d_scratch, stream);
}

int mt_deblock_frame_device_to(const uint16_t* d_in_y, const uint16_t* d_in_u, const uint16_t* d_in_v, uint16_t* d_y,
                               uint16_t* d_u, uint16_t* d_v, const uint8_t* d_blk4, const uint8_t* d_blk4h,
                               const uint8_t* d_blk4v, const uint8_t* d_blk4t, const uint8_t* d_pblk4,
                               const uint8_t* d_pblk4h, const mt_deblock_frame_params* prm, int32_t lvl_y,
                               int32_t lvl_u, int32_t lvl_v, void* d_scratch, void* stream) {
  if (!prm || !d_in_y) return MT_ERR_INVALID_INPUT;
  return deblock_frame(d_in_y, d_in_u, d_in_v, d_y, d_u, d_v, d_blk4, d_blk4h, d_blk4v, d_blk4t, d_pblk4, d_pblk4h,
                       prm, lvl_y, lvl_u, lvl_v, d_scratch, stream);
}

int mt_deblock_frame(uint16_t* y, uint16_t* u, uint16_t* v, const uint8_t* blk4, const uint8_t* blk4h,
                     const uint8_t* blk4v, const uint8_t* blk4t, const uint8_t* pblk4, const uint8_t* pblk4h,
                     const mt_deblock_frame_params* prm, int32_t lvl_y, int32_t lvl_u, int32_t lvl_v) {
  int rc = check_frame(prm);
  if (rc != MT_OK) return rc;
  if (!y || !blk4 || !blk4h || !blk4v || !blk4t) return MT_ERR_INVALID_INPUT;
  const bool chroma = !prm->mono && lvl_y > 0 && (lvl_u > 0 || lvl_v > 0);
  if (chroma && (!u || !v || !pblk4 || !pblk4h)) return MT_ERR_INVALID_INPUT;
  const int nc4 = prm->w8 / 4, nr4 = prm->h8 / 4;
  if (lvl_y > 0 && has_superblock_crossing(prm->w8, prm->h8, prm->disp_w, prm->disp_h, blk4h, blk4t, nc4))
    return MT_ERR_UNSUPPORTED;
  const size_t ny = (size_t)prm->w8 * prm->h8 * 2, nm = (size_t)nc4 * nr4;
  const size_t nc = chroma ? (size_t)(prm->w8 >> prm->sub_x) * (prm->h8 >> prm->sub_y) * 2 : 0;
  auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
  const size_t o_y = 0, o_u = up(ny), o_v = o_u + up(nc), o_m = o_v + up(nc), o_s = o_m + 6 * up(nm);
  const size_t total = o_s + mt_deblock_frame_scratch_bytes(prm);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, total) != cudaSuccess) return MT_ERR_ALLOC;
  const uint8_t* maps[6] = {blk4, blk4h, blk4v, blk4t, pblk4, pblk4h};
  cudaError_t e = cudaMemcpy(d + o_y, y, ny, cudaMemcpyHostToDevice);
  for (int k = 0; k < 6 && e == cudaSuccess; k++)
    if (maps[k] && (k < 4 || chroma)) e = cudaMemcpy(d + o_m + k * up(nm), maps[k], nm, cudaMemcpyHostToDevice);
  if (chroma && e == cudaSuccess) e = cudaMemcpy(d + o_u, u, nc, cudaMemcpyHostToDevice);
  if (chroma && e == cudaSuccess) e = cudaMemcpy(d + o_v, v, nc, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    auto m = [&](int k) { return (const uint8_t*)(d + o_m + k * up(nm)); };
    rc = mt_deblock_frame_device((uint16_t*)(d + o_y), chroma ? (uint16_t*)(d + o_u) : nullptr,
                                 chroma ? (uint16_t*)(d + o_v) : nullptr, m(0), m(1), m(2), m(3),
                                 chroma ? m(4) : nullptr, chroma ? m(5) : nullptr, prm, lvl_y, chroma ? lvl_u : 0,
                                 chroma ? lvl_v : 0, d + o_s, nullptr);
    if (rc == MT_OK) e = cudaMemcpy(y, d + o_y, ny, cudaMemcpyDeviceToHost);
    if (rc == MT_OK && chroma && e == cudaSuccess) e = cudaMemcpy(u, d + o_u, nc, cudaMemcpyDeviceToHost);
    if (rc == MT_OK && chroma && e == cudaSuccess) e = cudaMemcpy(v, d + o_v, nc, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_deblock_plane(uint16_t* px, int32_t w, int32_t h, int32_t vis_w, int32_t vis_h, const uint8_t* bw4,
                     const uint8_t* bh4, const uint8_t* vedge4, const uint8_t* hedge4, int32_t nc4, int32_t level,
                     int32_t sharp, int32_t is_luma, int32_t bd) {
  int rc = check_plane(w, h, vis_w, vis_h, nc4, level, sharp, bd);
  if (rc != MT_OK) return rc;
  if (level == 0) return MT_OK;
  if (!px || !bw4 || !bh4) return MT_ERR_INVALID_INPUT;
  if (is_luma && has_superblock_crossing(w, h, vis_w, vis_h, bh4, hedge4, nc4)) return MT_ERR_UNSUPPORTED;
  const int nr4 = (vis_h + 3) / 4;
  const size_t n_px = (size_t)w * h * 2, n_map = (size_t)nr4 * nc4;
  const size_t o_bw = (n_px + 255) & ~(size_t)255, o_bh = o_bw + ((n_map + 255) & ~(size_t)255);
  const size_t o_ve = o_bh + ((n_map + 255) & ~(size_t)255), o_he = o_ve + ((n_map + 255) & ~(size_t)255);
  const size_t total = o_he + n_map;
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, total) != cudaSuccess) return MT_ERR_ALLOC;
  cudaError_t e = cudaMemcpy(d, px, n_px, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_bw, bw4, n_map, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_bh, bh4, n_map, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && vedge4) e = cudaMemcpy(d + o_ve, vedge4, n_map, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && hedge4) e = cudaMemcpy(d + o_he, hedge4, n_map, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = mt_deblock_plane_device((uint16_t*)d, w, h, vis_w, vis_h, d + o_bw, d + o_bh, vedge4 ? d + o_ve : nullptr,
                                 hedge4 ? d + o_he : nullptr, nc4, level, sharp, is_luma, bd, nullptr);
    if (rc == MT_OK) e = cudaMemcpy(px, d, n_px, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"
