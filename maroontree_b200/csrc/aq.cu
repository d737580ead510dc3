// Adaptive quantisation: the per-superblock qindex grid of every tile
// (precompute_aq_grid, src/coder/lossy_state.rs:3937-3963), as two kernels.
//
// aq_sb_kernel (one CTA of 256 threads per 64x64 superblock): stages the
// superblock's luma in shared memory (one 16-byte load per 8 samples) and
// computes everything that depends on that superblock alone: the whole-SB
// log-activity (sb_activity, src/coder/aq.rs:140-160), the 64 8x8 variances and
// their octile pick (aq_sb_subblock_variances / sb_octile_variance,
// src/coder/aq.rs:216-252, src/aq_common.rs:58-63) and the dark-structure
// protection (src/aq_common.rs:216-345).  Moments are exact integers; every f32
// sum of the reference that is order-sensitive is either proven exact (all
// partial sums are integer multiples of the sample scale below 2^24) and formed
// from the integer total, or, when that bound fails (12-bit Laplacian sums),
// re-run by one thread in the reference's order.
//
// aq_tile_kernel (one CTA per (tile, chunk of 32 superblocks)): the tile means
// ref_act / ref_pick are sequential f32 sums in raster order (tile_ref_activity
// / tile_ref_picked, src/coder/aq.rs:162-192), so each CTA forms them in that
// order; it then evaluates aq_sb_target (src/coder/lossy_state.rs:3796-3902)
// for its chunk and tabulates the chunk's delta-q chain as a map of all 256
// entry qindices to the exit qindex.  The last CTA of a tile composes the
// chunk maps from base_q_idx (one lookup per chunk) and every chunk then walks
// its 32 superblocks from its known entry, writing the cells.  The chain is a
// sequence of clamped rounding steps, so a map composition replaces the
// reference's serial raster walk without changing a single value.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/maroontree_b200.h"
#include "av1_tables.h"
#include "dark_pow_table.h"

namespace {

constexpr int kChunk = 32;         // superblocks per chain chunk
constexpr int kMaxTileSbCols = 64;  // AV1 MAX_TILE_WIDTH / 64
constexpr int kMaxTileSbs = 2304;   // AV1 MAX_TILE_AREA / (64 * 64)
constexpr int kMaxChunks = (kMaxTileSbs + kChunk - 1) / kChunk;
constexpr int kDarkMinQ = 90;       // DarkAq::on (src/aq_common.rs:206-212)

// Ac_Qlookup at 8 / 10 / 12 bits (src/coef_q.rs), for the relative step clamp.
__device__ const uint16_t kAcQ[3][256] = {{MT_AC_QLOOKUP_8_LIST}, {MT_AC_QLOOKUP_10_LIST}, {MT_AC_QLOOKUP_12_LIST}};

struct AqGeom {
  int w8, h8, sb_cols, sb_rows;
  int tc_size, tr_size;      // tile size in superblocks (uniform spacing)
  int tile_cols, tile_rows;  // tiles actually present
  int chunks_per_tile;       // chunk slots per tile: ceil(tc_size * tr_size / 32)
  int base_q, bd, vb, dark, octile, boost_only;
  float strength;
};

struct SbStat {
  float act;       // sb_activity
  float pick_log;  // dirty_log1pf(octile pick * var_scale)
  int32_t dark;    // dark_protection
  int32_t filled;  // in-frame 8x8 blocks
};

// util.rs:36-59 fast_round: one ulp up, then round-to-nearest through 1.5*2^23.
__device__ __forceinline__ float fast_round(float x) {
  const float m = 12582912.0f;
  return __fsub_rn(__fadd_rn(__int_as_float(__float_as_int(x) + 1), m), m);
}

// Rust `f32 as i32` (saturating, NaN -> 0) is what cvt.rzi.s32.f32 does.
__device__ __forceinline__ int32_t to_i32(float v) { return __float2int_rz(v); }

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// aq_common.rs:89-109 dirty_log1pf, f_fmlaf unfused (multiply, round, add, round).
__device__ __forceinline__ float dirty_log1pf(float d) {
  const uint32_t ix = __float_as_uint(__fadd_rn(1.0f, d));
  const int32_t n = (int32_t)((ix & 0x7f800000u) >> 23) - 0x7f;
  const float mant = __uint_as_float((ix & 0x007fffffu) | 0x3f800000u);
  const float t = n == 0 ? d : __fsub_rn(mant, 1.0f);
  float p = 0.014539075084030628f;
  p = __fadd_rn(__fmul_rn(p, t), -0.0675969123840332f);
  p = __fadd_rn(__fmul_rn(p, t), 0.15056970715522766f);
  p = __fadd_rn(__fmul_rn(p, t), -0.23573730885982513f);
  p = __fadd_rn(__fmul_rn(p, t), 0.33125850558280945f);
  p = __fadd_rn(__fmul_rn(p, t), -0.4998837411403656f);
  p = __fadd_rn(__fmul_rn(p, t), 0.999998927116394f);
  return __fadd_rn(__fmul_rn((float)n, 0.693147180559945309417232121458176568f), __fmul_rn(t, p));
}

// powf(x, 1.2f) as the host C library rounds it: the binary64 power rounded
// once, except on the listed inputs where the library's result is taken (a
// bucket of at most 15 entries, found through the 4096-float bucket index).
__device__ float dark_pow(float x) {
  const uint32_t u = __float_as_uint(x);
  if (u > MT_DARK_POW_BASE && u <= MT_DARK_POW_BASE + ((uint32_t)(MT_DARK_POW_NB - 1) << MT_DARK_POW_SHIFT)) {
    const uint32_t b = (u - MT_DARK_POW_BASE) >> MT_DARK_POW_SHIFT;
    for (int i = kDarkPowB[b], e = kDarkPowB[b + 1]; i < e; i++)
      if (kDarkPowX[i] == u) return __uint_as_float(kDarkPowR[i]);
  }
  return __double2float_rn(pow((double)x, (double)1.2f));
}

// var = max(sum_sq / n - mean^2, 0) from exact moments (aq.rs:150-153, :235-238).
__device__ __forceinline__ float var_of(long long sum, unsigned long long ssq, int n) {
  const float nf = (float)n;
  const float mean = __fdiv_rn(__ll2float_rn(sum), nf);
  const float v = __fsub_rn(__fdiv_rn(__ull2float_rn(ssq), nf), __fmul_rn(mean, mean));
  return fmaxf(v, 0.0f);
}

__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int lap_at(const uint16_t (*p)[64], int r, int c) {
  return 4 * (int)p[r][c] - p[r - 1][c] - p[r + 1][c] - p[r][c - 1] - p[r][c + 1];
}
__device__ __forceinline__ int lap_at(const int32_t (*p)[32], int r, int c) {
  return 4 * p[r][c] - p[r - 1][c] - p[r + 1][c] - p[r][c - 1] - p[r][c + 1];
}

__global__ void __launch_bounds__(256) aq_sb_kernel(const uint16_t* __restrict__ luma, const AqGeom g,
                                                    SbStat* __restrict__ stats, uint32_t* __restrict__ counters,
                                                    int n_counters) {
  __shared__ __align__(16) uint16_t s_px[64][64];
  __shared__ int32_t s_half[32][32];
  __shared__ float s_var[64];
  __shared__ uint32_t s_bsum[64], s_bssq[64];
  __shared__ int s_red[2][8];
  __shared__ float s_pick, s_wgt;
  const int tid = threadIdx.x;
  const int sb = blockIdx.x;
  if (sb == 0)
    for (int i = tid; i < n_counters; i += 256) counters[i] = 0;
  const int sbr = sb / g.sb_cols, sbc = sb - sbr * g.sb_cols;
  const int y0 = sbr * 64, x0 = sbc * 64;
  const int h = min(g.h8 - y0, 64), w = min(g.w8 - x0, 64);  // multiples of 8
  const int bd = g.bd;
  const bool dark_on = g.dark && g.base_q >= kDarkMinQ;
  // Stage: 64 rows x 8 segments of 8 samples, two segments per thread.
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const int seg = tid + k * 256, row = seg >> 3, c8 = seg & 7;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (row < h && c8 * 8 < w) v = *reinterpret_cast<const uint4*>(luma + (size_t)(y0 + row) * g.w8 + x0 + c8 * 8);
    *reinterpret_cast<uint4*>(&s_px[row][c8 * 8]) = v;
  }
  __syncthreads();
  // 8x8 moments: four threads per block, two rows each.
  {
    const int b = tid >> 2, qd = tid & 3, by = b >> 3, bx = b & 7;
    uint32_t s = 0, q = 0;
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const uint32_t v = s_px[by * 8 + qd * 2 + r][bx * 8 + c];
        s += v;
        q += v * v;
      }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    q += __shfl_xor_sync(0xffffffffu, q, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    q += __shfl_xor_sync(0xffffffffu, q, 2);
    if (qd == 0) {
      const bool valid = by * 8 < h && bx * 8 < w;
      s_bsum[b] = valid ? s : 0u;
      s_bssq[b] = valid ? q : 0u;
      s_var[b] = valid ? var_of((long long)s, q, 64) : __int_as_float(0x7fc00000);
    }
  }
  // 2x box sums for the dark statistics (value = Q * scale / 4).
  const int hh = h >> 1, ww = w >> 1;
  if (dark_on)
    for (int i = tid; i < hh * ww; i += 256) {
      const int y = i / ww, x = i - y * ww;
      s_half[y][x] = (int)s_px[2 * y][2 * x] + s_px[2 * y][2 * x + 1] + s_px[2 * y + 1][2 * x] +
                     s_px[2 * y + 1][2 * x + 1];
    }
  __syncthreads();
  const int nblk = (h >> 3) * (w >> 3);
  const float scale = __fdiv_rn(1.0f, (float)(1u << (bd - 8)));
  float act = 0.0f, pick_log = 0.0f;
  if (tid < 32) {
    // Whole-SB moments from the block moments (exact).
    unsigned long long q = (unsigned long long)s_bssq[tid] + s_bssq[tid + 32];
    long long s = (long long)s_bsum[tid] + s_bsum[tid + 32];
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      q += __shfl_xor_sync(0xffffffffu, q, o);
      s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    const float var = var_of(s, q, h * w);
    act = dirty_log1pf(__fdiv_rn(var, (float)(1u << (2 * (bd - 8)))));
    // Out-of-frame 8x8s take the mean of the in-frame variances (raster f32 sum).
    float fill = 0.0f;
    if (nblk < 64 && tid == 0) {
      float acc = 0.0f;
      for (int b = 0; b < 64; b++)
        if ((b >> 3) * 8 < h && (b & 7) * 8 < w) acc = __fadd_rn(acc, s_var[b]);
      fill = __fdiv_rn(acc, (float)nblk);
    }
    fill = __shfl_sync(0xffffffffu, fill, 0);
    float v0 = s_var[tid], v1 = s_var[tid + 32];
    if (v0 != v0) v0 = fill;
    if (v1 != v1) v1 = fill;
    // The k-th smallest of the 64 (k = octile * 8 - 1): a value whose count of
    // smaller values is <= k and whose count of smaller-or-equal values is > k.
    const int k = min(g.octile * 8 - 1, 63);
    int lt0 = 0, le0 = 0, lt1 = 0, le1 = 0;
#pragma unroll 16
    for (int j = 0; j < 64; j++) {
      const float vj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
      lt0 += vj < v0;
      le0 += vj <= v0;
      lt1 += vj < v1;
      le1 += vj <= v1;
    }
    if (lt0 <= k && k < le0) s_pick = v0;
    if (lt1 <= k && k < le1) s_pick = v1;
    __syncwarp();
    const float var_scale = __fdiv_rn(1.0f, (float)(1u << (2 * (bd - 8))));
    pick_log = dirty_log1pf(__fmul_rn(s_pick, var_scale));
  }
  // Dark-structure protection (src/aq_common.rs:262-345).
  int dark = 0;
  if (dark_on) {
    if (tid == 32) {
      // The weight's power, started early: its table walk overlaps the Laplacians.
      // The sample sum is exact in f32 at every depth (< 2^24 sample units):
      // sum(px * scale) = S * scale.
      float mean;
      {
        long long s = 0;
        for (int b = 0; b < 64; b++) s += s_bsum[b];
        mean = __fdiv_rn(__fmul_rn(__ll2float_rn(s), scale), (float)(h * w));
      }
      const float x = __fdiv_rn(72.0f, __fadd_rn(16.0f, mean));
      s_wgt = x > 1.0f ? clampf(dark_pow(x), 1.0f, 4.5f) : 1.0f;
    }
    // |Laplacian| sums in integer units of the sample scale (full) and of a quarter of it (half).
    int lf = 0, lh = 0;
    const int iw = w - 2, ni = (h - 2) * iw;
    for (int i = tid; i < ni; i += 256) {
      const int r = 1 + i / iw, c = 1 + i % iw;
      lf += abs(lap_at(s_px, r, c));
    }
    const int hw = ww - 2, nh = (hh - 2) * hw;
    for (int i = tid; i < nh; i += 256) {
      const int r = 1 + i / hw, c = 1 + i % hw;
      lh += abs(lap_at(s_half, r, c));
    }
    lf = warp_sum_i(lf);
    lh = warp_sum_i(lh);
    if ((tid & 31) == 0) {
      s_red[0][tid >> 5] = lf;
      s_red[1][tid >> 5] = lh;
    }
    __syncthreads();
    if (tid == 0) {
      long long tf = 0, th = 0;
      for (int i = 0; i < 8; i++) {
        tf += s_red[0][i];
        th += s_red[1][i];
      }
      // Every partial sum of the reference's f32 loop is an integer multiple of
      // the unit below 2^24 units, hence exact, when the integer total is; else
      // (busy 12-bit content) the loop is re-run in the reference's order.
      float sf, sh;
      if (tf < (1 << 24)) {
        sf = __fmul_rn(__ll2float_rn(tf), scale);
      } else {
        sf = 0.0f;
        for (int r = 1; r + 1 < h; r++)
          for (int c = 1; c + 1 < w; c++) sf = __fadd_rn(sf, __fmul_rn((float)abs(lap_at(s_px, r, c)), scale));
      }
      const float qs = __fmul_rn(scale, 0.25f);
      if (th < (1 << 24)) {
        sh = __fmul_rn(__ll2float_rn(th), qs);
      } else {
        sh = 0.0f;
        for (int r = 1; r + 1 < hh; r++)
          for (int c = 1; c + 1 < ww; c++) sh = __fadd_rn(sh, __fmul_rn((float)abs(lap_at(s_half, r, c)), qs));
      }
      const float lap_full = __fdiv_rn(sf, (float)((h - 2) * (w - 2)));
      const float lap_half = __fdiv_rn(sh, (float)((hh - 2) * (ww - 2)));
      const float mid = __fsqrt_rn(__fmul_rn(lap_full, lap_half));
      if (mid > 0.0f) {
        const float darkness = __fsub_rn(s_wgt, 1.0f);
        if (darkness > 0.0f) {
          const float ds = dirty_log1pf(__fmul_rn(mid, darkness));
          dark = to_i32(fast_round(fmaxf(fminf(__fmul_rn(ds, 4.0f), 16.0f), 0.0f)));
        }
      }
    }
  }
  if (tid == 0) {
    SbStat st;
    st.act = act;
    st.pick_log = pick_log;
    st.dark = dark;
    st.filled = nblk;
    stats[sb] = st;
  }
}

// The frame constants aq_sb_target reads.
struct TargetConsts {
  int base_q, vb, boost_only;
  float strength, mid_t, low_log, boost_slope, cut_slope, ease;
};

// clamp_aq_delta_relative (lossy_state.rs:133-154), aq_r 1.35; acq = Ac_Qlookup.
__device__ __forceinline__ int32_t clamp_delta_relative(const uint16_t* acq, int32_t base_q, int32_t delta) {
  if (delta == 0) return 0;
  const float r = delta > 0 ? 1.35f : fmaxf(1.35f, 1.05f);
  const float base_step = (float)acq[min(max(base_q, 1), 255)];
  const float lo = __fdiv_rn(base_step, r), hi = __fmul_rn(base_step, r);
  int32_t d = delta;
  while (d != 0) {
    const float s = (float)acq[min(max(base_q + d, 1), 255)];
    if (s >= lo && s <= hi) break;
    d -= d > 0 ? 1 : -1;
  }
  return d;
}

// aq_sb_target (lossy_state.rs:3796-3902) from the superblock's statistics.
__device__ __forceinline__ int32_t sb_target(const TargetConsts& k, const uint16_t* acq, const SbStat& st,
                                             float ref_act, float ref_pick) {
  const int32_t base_q = k.base_q;
  const int32_t dark = st.dark;
  int32_t delta;
  if (k.vb) {
    if (st.filled == 0) return base_q;
    // variance_boost_delta (aq_common.rs:115-150), cut_wide_t 0.
    const float v_log = st.pick_log;
    int32_t vb_delta;
    if (v_log < k.low_log) {
      const float d = fminf(__fmul_rn(__fmul_rn(__fsub_rn(k.low_log, v_log), k.boost_slope), k.strength), 18.0f);
      vb_delta = -to_i32(fast_round(d));
    } else if (k.boost_only) {
      vb_delta = 0;
    } else {
      const float anchor = ref_pick > 0.0f ? ref_pick : __fmul_rn(ref_act, 0.95f);
      const float over = fmaxf(__fsub_rn(v_log, fmaxf(anchor, k.low_log)), 0.0f);
      const float d = fminf(__fmul_rn(__fmul_rn(over, k.cut_slope), k.strength), 16.0f);
      vb_delta = to_i32(fast_round(d));
    }
    const int32_t flat_boost = max(-vb_delta, 0);
    const int32_t protection = max(flat_boost, dark);
    if (vb_delta > 0 && dark > 0) delta = vb_delta - dark;
    else if (protection > 0) delta = -protection;
    else delta = vb_delta;
    if (delta > 0) delta = to_i32(fast_round(__fmul_rn((float)delta, k.ease)));
  } else {
    // aq_target_qidx (aq.rs:201-214): slope 5, max delta 28.
    const float dl = clampf(__fmul_rn(__fsub_rn(st.act, ref_act), 5.0f), -28.0f, 28.0f);
    const int32_t tq = min(max(base_q + to_i32(fast_round(dl)), 1), 255);
    const int32_t vb_delta = tq - base_q;
    const int32_t protection = max(max(-vb_delta, 0), dark);
    delta = protection > 0 ? -protection : vb_delta;
  }
  delta = clamp_delta_relative(acq, base_q, delta);
  return min(max(base_q + delta, 1), 255);
}

// One raster step of the delta-q chain (precompute_aq_grid): steps of 4 qindex,
// at most 12, the decoder's Clip3(1, 255).  (target - cur) / 4 is exact as a
// product with 0.25.
__device__ __forceinline__ int32_t chain_step(int32_t cur, int32_t target, int32_t* steps_out) {
  const float st = clampf(fast_round(__fmul_rn((float)(target - cur), 0.25f)), -12.0f, 12.0f);
  const int32_t steps = to_i32(st);
  *steps_out = steps;
  return min(max(cur + steps * 4, 1), 255);
}

__global__ void __launch_bounds__(256) aq_tile_kernel(const AqGeom g, const SbStat* __restrict__ stats,
                                                      uint8_t* __restrict__ targets, uint8_t* __restrict__ maps,
                                                      uint32_t* __restrict__ counters, mt_aq_cell* __restrict__ cells,
                                                      float* __restrict__ tile_refs) {
  __shared__ __align__(16) float s_val[2][kMaxTileSbs];  // per SB of the tile: act, pick_log (0 if unfilled)
  __shared__ uint8_t s_tq[kMaxTileSbs];                  // target qindex per SB (last CTA)
  __shared__ uint8_t s_map[kMaxChunks][256];
  __shared__ uint16_t s_acq[256];
  __shared__ int32_t s_entry[kMaxChunks];
  __shared__ float s_refs[2];
  __shared__ int32_t s_target[kChunk];
  __shared__ int s_filled, s_last;
  const int tid = threadIdx.x;
  const int tile = blockIdx.x / g.chunks_per_tile, chunk = blockIdx.x - tile * g.chunks_per_tile;
  const int tr = tile / g.tile_cols, tc = tile - tr * g.tile_cols;
  const int sb_cols = g.sb_cols;
  const int sx0 = tc * g.tc_size, sy0 = tr * g.tr_size;
  const int sw = min(g.tc_size, sb_cols - sx0), sh = min(g.tr_size, g.sb_rows - sy0);
  const int n = sw * sh, nchunks = (n + kChunk - 1) / kChunk;
  if (chunk >= nchunks) return;
  s_acq[tid] = kAcQ[g.bd == 10 ? 1 : (g.bd == 12 ? 2 : 0)][tid];
  if (tid == 0) s_filled = 0;
  __syncthreads();
  int filled = 0;
  for (int i = tid; i < n; i += 256) {
    const int r = i / sw;
    const SbStat st = stats[(sy0 + r) * sb_cols + sx0 + (i - r * sw)];
    s_val[0][i] = st.act;
    s_val[1][i] = st.filled != 0 ? st.pick_log : 0.0f;
    filled += st.filled != 0;
  }
  if (filled) atomicAdd(&s_filled, filled);
  __syncthreads();
  // Tile means in raster order (tile_ref_activity / tile_ref_picked): warp 0
  // sums the activities, warp 1 the picks.  Adding the +0 of an unfilled SB
  // leaves the sum unchanged (no value is -0), and the counts are exact.
  if (tid == 0 || tid == 32) {
    const int which = tid >> 5;
    const float4* v4 = reinterpret_cast<const float4*>(s_val[which]);
    float sum = 0.0f;
    int i = 0;
#pragma unroll 4
    for (; i + 4 <= n; i += 4) {
      const float4 v = v4[i >> 2];
      sum = __fadd_rn(sum, v.x);
      sum = __fadd_rn(sum, v.y);
      sum = __fadd_rn(sum, v.z);
      sum = __fadd_rn(sum, v.w);
    }
    for (; i < n; i++) sum = __fadd_rn(sum, s_val[which][i]);
    const int cnt = which == 0 ? n : s_filled;
    s_refs[which] = cnt > 0 ? __fdiv_rn(sum, (float)cnt) : 5.0f;
  }
  __syncthreads();
  const float ref_act = s_refs[0], ref_pick = s_refs[1];
  if (chunk == 0 && tid == 0 && tile_refs) {
    tile_refs[2 * tile] = ref_act;
    tile_refs[2 * tile + 1] = ref_pick;
  }
  const int first = chunk * kChunk, len = min(kChunk, n - first);
  if (tid < len) {
    TargetConsts k;
    k.base_q = g.base_q;
    k.vb = g.vb;
    k.boost_only = g.boost_only;
    k.strength = fmaxf(g.strength, 0.0f);
    k.mid_t = clampf(__fdiv_rn(__fsub_rn((float)g.base_q, 48.0f), 48.0f), 0.0f, 1.0f);
    k.low_log = __fadd_rn(__fmul_rn(0.5f, k.mid_t), 5.549076f);
    k.boost_slope = __fadd_rn(5.0f, __fmul_rn(1.5f, k.mid_t));
    k.cut_slope = __fadd_rn(6.0f, __fmul_rn(2.0f, k.mid_t));
    // top_ease_t (quant.rs:122-125): knee 20, width 12, top_ease 1.
    const float t = clampf(__fdiv_rn(__fsub_rn(20.0f, (float)g.base_q), 12.0f), 0.0f, 1.0f);
    k.ease = __fsub_rn(1.0f, __fmul_rn(1.0f, t));
    const int i = first + tid, r = i / sw;
    const int sb = (sy0 + r) * sb_cols + sx0 + (i - r * sw);
    const int32_t tq = sb_target(k, s_acq, stats[sb], ref_act, ref_pick);
    s_target[tid] = tq;
    targets[sb] = (uint8_t)tq;
  }
  __syncthreads();
  // Exit qindex of this chunk for every entry qindex.
  {
    int32_t cur = tid, steps;
    for (int j = 0; j < len; j++) cur = chain_step(cur, s_target[j], &steps);
    maps[((size_t)tile * g.chunks_per_tile + chunk) * 256 + tid] = (uint8_t)cur;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) s_last = atomicAdd(&counters[tile], 1u) == (unsigned)(nchunks - 1);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // Last CTA of the tile: compose the maps from base_q_idx, then walk every chunk.
  const uint8_t* tmaps = maps + (size_t)tile * g.chunks_per_tile * 256;
  for (int i = tid; i < nchunks * 64; i += 256)
    reinterpret_cast<uint32_t*>(&s_map[0][0])[i] = __ldcg(reinterpret_cast<const uint32_t*>(tmaps) + i);
  for (int i = tid; i < n; i += 256) {
    const int r = i / sw;
    s_tq[i] = __ldcg(targets + (sy0 + r) * sb_cols + sx0 + (i - r * sw));
  }
  __syncthreads();
  if (tid == 0) {
    int32_t cur = g.base_q;
    for (int c = 0; c < nchunks; c++) {
      s_entry[c] = cur;
      cur = s_map[c][cur];
    }
  }
  __syncthreads();
  if (tid < nchunks) {
    int32_t cur = s_entry[tid];
    const int f = tid * kChunk, l = min(kChunk, n - f);
    int r = f / sw, c = f - r * sw;
    for (int j = 0; j < l; j++) {
      const int32_t t = s_tq[f + j];
      int32_t steps;
      const int32_t nq = chain_step(cur, t, &steps);
      mt_aq_cell cell;
      cell.prev = (uint8_t)cur;
      cell.newq = (uint8_t)nq;
      cell.steps = (int8_t)steps;
      cell.target = (uint8_t)t;
      cells[(sy0 + r) * sb_cols + sx0 + c] = cell;
      cur = nq;
      if (++c == sw) {
        c = 0;
        r++;
      }
    }
  }
}

__global__ void dark_pow_kernel(const float* __restrict__ x, float* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = dark_pow(x[i]);
}

struct Layout {
  size_t stats, targets, maps, counters, total;
  int ntiles;
};

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

int make_geom(const mt_aq_params* p, AqGeom* g) {
  if (!p) return MT_ERR_INVALID_INPUT;
  if (p->w8 <= 0 || p->h8 <= 0 || (p->w8 & 7) || (p->h8 & 7) || p->w8 > 16384 || p->h8 > 16384)
    return MT_ERR_INVALID_INPUT;
  if (p->bd != 8 && p->bd != 10 && p->bd != 12) return MT_ERR_UNSUPPORTED;
  if (p->base_q_idx < 0 || p->base_q_idx > 255) return MT_ERR_INVALID_INPUT;
  if (p->tile_cols_log2 < 0 || p->tile_cols_log2 > 6 || p->tile_rows_log2 < 0 || p->tile_rows_log2 > 6)
    return MT_ERR_INVALID_INPUT;
  if (p->strength != p->strength) return MT_ERR_INVALID_INPUT;
  g->w8 = p->w8;
  g->h8 = p->h8;
  g->sb_cols = (p->w8 + 63) / 64;
  g->sb_rows = (p->h8 + 63) / 64;
  g->tc_size = (g->sb_cols + (1 << p->tile_cols_log2) - 1) >> p->tile_cols_log2;
  g->tr_size = (g->sb_rows + (1 << p->tile_rows_log2) - 1) >> p->tile_rows_log2;
  if (g->tc_size > kMaxTileSbCols || g->tc_size * g->tr_size > kMaxTileSbs) return MT_ERR_INVALID_INPUT;
  g->tile_cols = (g->sb_cols + g->tc_size - 1) / g->tc_size;
  g->tile_rows = (g->sb_rows + g->tr_size - 1) / g->tr_size;
  g->chunks_per_tile = (g->tc_size * g->tr_size + kChunk - 1) / kChunk;
  g->base_q = p->base_q_idx;
  g->bd = p->bd;
  g->vb = p->variance_boost != 0;
  g->dark = p->dark_aq != 0;
  g->octile = std::min(std::max(p->octile, 1), 8);
  g->boost_only = p->boost_only != 0;
  g->strength = p->strength;
  return MT_OK;
}

Layout make_layout(const AqGeom& g) {
  Layout L;
  const size_t nsb = (size_t)g.sb_cols * g.sb_rows;
  L.ntiles = g.tile_cols * g.tile_rows;
  L.stats = 0;
  L.targets = up256(nsb * sizeof(SbStat));
  L.maps = L.targets + up256(nsb);
  L.counters = L.maps + up256((size_t)L.ntiles * g.chunks_per_tile * 256);
  L.total = L.counters + up256((size_t)L.ntiles * 4);
  return L;
}

}  // namespace

extern "C" {

int mt_tiling_spec_min(int32_t w8, int32_t h8, int32_t* cols_log2, int32_t* rows_log2) {
  if (w8 <= 0 || h8 <= 0 || !cols_log2 || !rows_log2) return MT_ERR_INVALID_INPUT;
  auto tile_log2 = [](int blk, int target) {
    int k = 0;
    while ((blk << k) < target) k++;
    return k;
  };
  const int sb_cols = (w8 + 63) / 64, sb_rows = (h8 + 63) / 64;
  const int min_c = tile_log2(64, sb_cols);
  const int max_c = tile_log2(1, std::min(sb_cols, 64));
  const int max_r = tile_log2(1, std::min(sb_rows, 64));
  const int min_tiles = std::max(min_c, tile_log2(2304, sb_rows * sb_cols));
  const int tcl = std::min(min_c, max_c);
  *cols_log2 = tcl;
  *rows_log2 = std::min(std::max(min_tiles - tcl, 0), max_r);
  return MT_OK;
}

size_t mt_aq_grid_scratch_bytes(const mt_aq_params* prm) {
  AqGeom g;
  if (make_geom(prm, &g) != MT_OK) return 0;
  return make_layout(g).total;
}

int mt_aq_grid_device(const uint16_t* d_luma, const mt_aq_params* prm, mt_aq_cell* d_cells, float* d_tile_refs,
                      void* d_scratch, void* stream) {
  AqGeom g;
  int rc = make_geom(prm, &g);
  if (rc != MT_OK) return rc;
  if (!d_luma || !d_cells || !d_scratch) return MT_ERR_INVALID_INPUT;
  if (reinterpret_cast<uintptr_t>(d_luma) & 15) return MT_ERR_INVALID_INPUT;
  const Layout L = make_layout(g);
  uint8_t* s = static_cast<uint8_t*>(d_scratch);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  SbStat* stats = reinterpret_cast<SbStat*>(s + L.stats);
  uint32_t* counters = reinterpret_cast<uint32_t*>(s + L.counters);
  const int nsb = g.sb_cols * g.sb_rows;
  aq_sb_kernel<<<nsb, 256, 0, st>>>(d_luma, g, stats, counters, L.ntiles);
  aq_tile_kernel<<<L.ntiles * g.chunks_per_tile, 256, 0, st>>>(g, stats, s + L.targets, s + L.maps, counters, d_cells,
                                                                d_tile_refs);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_aq_grid(const uint16_t* luma, const mt_aq_params* prm, mt_aq_cell* cells, float* tile_refs) {
  AqGeom g;
  int rc = make_geom(prm, &g);
  if (rc != MT_OK) return rc;
  if (!luma || !cells) return MT_ERR_INVALID_INPUT;
  const Layout L = make_layout(g);
  const size_t ny = (size_t)g.w8 * g.h8 * 2, nsb = (size_t)g.sb_cols * g.sb_rows, nref = (size_t)L.ntiles * 8;
  const size_t o_y = 0, o_c = up256(ny), o_r = o_c + up256(nsb * sizeof(mt_aq_cell)), o_s = o_r + up256(nref);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, o_s + L.total) != cudaSuccess) return MT_ERR_ALLOC;
  cudaError_t e = cudaMemcpy(d + o_y, luma, ny, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = mt_aq_grid_device(reinterpret_cast<const uint16_t*>(d + o_y), prm, reinterpret_cast<mt_aq_cell*>(d + o_c),
                           reinterpret_cast<float*>(d + o_r), d + o_s, nullptr);
    if (rc == MT_OK) e = cudaMemcpy(cells, d + o_c, nsb * sizeof(mt_aq_cell), cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && tile_refs) e = cudaMemcpy(tile_refs, d + o_r, nref, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_dark_pow_device(const float* d_x, float* d_out, int64_t n, void* stream) {
  if (n < 0 || (n > 0 && (!d_x || !d_out))) return MT_ERR_INVALID_INPUT;
  if (n == 0) return MT_OK;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 16);
  dark_pow_kernel<<<(unsigned)blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_x, d_out, n);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"
