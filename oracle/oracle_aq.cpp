// Oracle (test infrastructure, the CPU checker of the CUDA path): the adaptive
// quantiser's per-superblock qindex grid, restated from the reference in its
// scalar order.  Variance Boost and classic AQ targets, dark-structure
// protection, the relative step clamp and the raster delta-q chain of each
// tile.
//
//   src/aq_common.rs:58-63    sb_octile_variance
//   src/aq_common.rs:89-109   dirty_log1pf (f_fmlaf unfused: no FMA target feature in the default build)
//   src/aq_common.rs:115-150  variance_boost_delta
//   src/aq_common.rs:177-214  DarkAq::on constants
//   src/aq_common.rs:216-345  laplacian_abs_sum, box_downsample_2x, dark_structure_stats, dark_protection
//   src/coder/aq.rs:140-262   sb_activity, tile_ref_activity, tile_ref_picked, aq_target_qidx,
//                             aq_sb_subblock_variances
//   src/coder/lossy_state.rs:91-109    block_moments_i32
//   src/coder/lossy_state.rs:133-154   clamp_aq_delta_relative
//   src/coder/lossy_state.rs:3746-3770 enable_aq (refs per tile)
//   src/coder/lossy_state.rs:3796-3963 aq_sb_target, precompute_aq_grid
//   src/coder/tiling.rs:92-147         plan_tiling (target 1), tile_starts_sb
//   src/util.rs:36-59                  fast_round
//   src/tuning.rs:750-752, :858-860    top_ease 1 / knee 20 / width 12; aq_slope 5, aq_max_delta 28, aq_r 1.35
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../maroontree_b200/csrc/av1_tables.h"
#include "oracle.h"

namespace {

float bits_f(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}
uint32_t f_bits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}

// Rust `f32 as i32`: saturating, NaN -> 0.
int32_t sat_i32(float v) {
  if (v != v) return 0;
  if (v >= 2147483648.0f) return INT32_MAX;
  if (v <= -2147483648.0f) return INT32_MIN;
  return (int32_t)v;
}

float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
// Rust f32::min / f32::max (NaN-ignoring; no NaN reaches them here).
float fminr(float a, float b) { return a < b ? a : (b < a ? b : a); }
float fmaxr(float a, float b) { return a > b ? a : (b > a ? b : a); }

uint16_t ac_q(int q, int bd) {
  const uint16_t* t = bd == 10 ? MT_AC_QLOOKUP_10 : (bd == 12 ? MT_AC_QLOOKUP_12 : MT_AC_QLOOKUP_8);
  return t[q];
}

// block_moments_i32 (lossy_state.rs:91-109).
void block_moments(const uint16_t* p, int stride, int px, int py, int w, int h, int64_t* sum, int64_t* ssq) {
  int64_t s = 0, q = 0;
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      const int64_t v = p[(size_t)(py + y) * stride + px + x];
      s += v;
      q += v * v;
    }
  *sum = s;
  *ssq = q;
}

float var_of(int64_t sum, int64_t ssq, int n) {
  const float nf = (float)n;
  const float mean = (float)sum / nf;
  const float v = (float)ssq / nf - mean * mean;
  return fmaxr(v, 0.0f);
}

// DarkAq::on (aq_common.rs:177-214).
constexpr int kDarkMinQ = 90;
constexpr float kDarkMeanFloor = 16.0f, kDarkRef = 56.0f, kDarkGamma = 1.2f, kDarkMaxWeight = 4.5f,
                kDarkScale = 4.0f;
constexpr int kDarkMaxQidx = 16;

// laplacian_abs_sum (aq_common.rs:216-233) over a row-major f32 buffer.
void laplacian_abs_sum(const float* buf, int stride, int h, int w, float* sum_out, uint32_t* n_out) {
  float sum = 0.0f;
  uint32_t n = 0;
  for (int r = 1; r + 1 < h; r++)
    for (int c = 1; c + 1 < w; c++) {
      const float up = buf[(r - 1) * stride + c], down = buf[(r + 1) * stride + c];
      const float left = buf[r * stride + c - 1], center = buf[r * stride + c], right = buf[r * stride + c + 1];
      const float l = 4.0f * center - up - down - left - right;
      sum += fabsf(l);
      n++;
    }
  *sum_out = sum;
  *n_out = n;
}

// dark_structure_stats (aq_common.rs:262-305).
void dark_structure_stats(const uint16_t* yp, int pw, int sb_y, int sb_x, int width, int height, float scale,
                          float* mean_out, float* mid_out) {
  const int h = std::min(std::max(height - sb_y, 0), 64);
  const int w = std::min(std::max(width - sb_x, 0), 64);
  *mean_out = 0.0f;
  *mid_out = 0.0f;
  if (h == 0 || w == 0) return;
  static thread_local float buf[64 * 64];
  float sum = 0.0f;
  for (int r = 0; r < h; r++)
    for (int c = 0; c < w; c++) {
      const float v = (float)yp[(size_t)(sb_y + r) * pw + sb_x + c] * scale;
      buf[r * 64 + c] = v;
      sum += v;
    }
  const float mean = sum / (float)(h * w);
  *mean_out = mean;
  if (h < 3 || w < 3) return;
  float lf;
  uint32_t nf;
  laplacian_abs_sum(buf, 64, h, w, &lf, &nf);
  const float lap_full = lf / (float)nf;
  const int hh = h / 2, ww = w / 2;
  if (hh < 3 || ww < 3) return;
  static thread_local float half[32 * 32];
  for (int y = 0; y < hh; y++)
    for (int x = 0; x < ww; x++) {
      const float tl = buf[(2 * y) * 64 + 2 * x], tr = buf[(2 * y) * 64 + 2 * x + 1];
      const float bl = buf[(2 * y + 1) * 64 + 2 * x], br = buf[(2 * y + 1) * 64 + 2 * x + 1];
      half[y * 32 + x] = 0.25f * (tl + tr + bl + br);
    }
  float lh;
  uint32_t nh;
  laplacian_abs_sum(half, 32, hh, ww, &lh, &nh);
  const float lap_half = lh / (float)nh;
  *mid_out = sqrtf(lap_full * lap_half);
}

// sb_activity (aq.rs:140-160).
float sb_activity(const uint16_t* yp, int pw, int sb_y, int sb_x, int width, int height, int bd) {
  const int h = std::min(std::max(height - sb_y, 0), 64);
  const int w = std::min(std::max(width - sb_x, 0), 64);
  if (h == 0 || w == 0) return 0.0f;
  int64_t s, q;
  block_moments(yp, pw, sb_x, sb_y, w, h, &s, &q);
  const float var = var_of(s, q, h * w);
  const int b = bd > 8 ? bd : 8;
  return or_dirty_log1pf(var / (float)(1u << (2 * (b - 8))));
}

// aq_sb_subblock_variances (aq.rs:216-252).
int sb_subblock_variances(const uint16_t* yp, int pw, int sb_y, int sb_x, int width, int height, float* out) {
  int filled = 0;
  float acc = 0.0f;
  for (int by = 0; by < 8; by++)
    for (int bx = 0; bx < 8; bx++) {
      const int y0 = sb_y + by * 8, x0 = sb_x + bx * 8;
      const int h = std::min(std::max(height - y0, 0), 8), w = std::min(std::max(width - x0, 0), 8);
      float& o = out[by * 8 + bx];
      if (h == 0 || w == 0) {
        o = NAN;
        continue;
      }
      int64_t s, q;
      block_moments(yp, pw, x0, y0, w, h, &s, &q);
      o = var_of(s, q, h * w);
      acc += o;
      filled++;
    }
  if (filled == 0) {
    for (int i = 0; i < 64; i++) out[i] = 0.0f;
    return 0;
  }
  const float mean = acc / (float)filled;
  for (int i = 0; i < 64; i++)
    if (out[i] != out[i]) out[i] = mean;
  return filled;
}

// sb_octile_variance (aq_common.rs:58-63).
float octile_pick(float* v, int octile) {
  std::sort(v, v + 64);
  const int o = std::min(std::max(octile, 1), 8);
  return v[std::min(o * 8 - 1, 63)];
}

// variance_boost_delta (aq_common.rs:115-150).
int32_t variance_boost_delta(float picked_var, float ref_log, float ref_pick, float strength, bool boost_only,
                             float mid_t, float cut_wide_t) {
  const float v_log = or_dirty_log1pf(picked_var);
  const float low_log = 0.5f * mid_t + 5.549076f;
  const float max_boost = 18.0f;
  const float max_cut = 16.0f + 24.0f * cut_wide_t;
  const float boost_slope = 5.0f + 1.5f * mid_t;
  const float cut_slope = 6.0f + 2.0f * mid_t;
  if (v_log < low_log) {
    const float d = fminr((low_log - v_log) * boost_slope * strength, max_boost);
    return -sat_i32(or_fast_round(d));
  }
  if (boost_only) return 0;
  const float anchor = ref_pick > 0.0f ? ref_pick : ref_log * 0.95f;
  const float over = fmaxr(v_log - fmaxr(anchor, low_log), 0.0f);
  const float d = fminr(over * cut_slope * strength, max_cut);
  return sat_i32(or_fast_round(d));
}

// aq_target_qidx (aq.rs:201-214) with aq_params() = (5.0, 28.0, 1.0).
int32_t aq_target_qidx(int32_t base_q, float activity, float ref_act) {
  const float slope = 5.0f, maxd = 28.0f, coarsen = 1.0f;
  float delta = (activity - ref_act) * slope;
  if (delta > 0.0f) delta *= coarsen;
  delta = clampf(delta, -maxd, maxd);
  const int32_t q = base_q + sat_i32(or_fast_round(delta));
  return std::min(std::max(q, 1), 255);
}

// clamp_aq_delta_relative (lossy_state.rs:133-154), aq_r = 1.35.
int32_t clamp_aq_delta_relative(int32_t base_q, int32_t delta, int bd) {
  float r = 1.35f;
  r = delta > 0 ? r : fmaxr(r, 1.05f);
  if (delta == 0) return delta;
  const float base_step = (float)ac_q(std::min(std::max(base_q, 1), 255), bd);
  const float lo = base_step / r, hi = base_step * r;
  int32_t d = delta;
  while (d != 0) {
    const float s = (float)ac_q(std::min(std::max(base_q + d, 1), 255), bd);
    if (s >= lo && s <= hi) break;
    d -= d > 0 ? 1 : -1;
  }
  return d;
}

// top_ease_t (quant.rs:122-125), knee 20, width 12.
float top_ease_t(int base_q) { return clampf((20.0f - (float)base_q) / 12.0f, 0.0f, 1.0f); }

struct TileRefs {
  float ref_act, ref_pick;
};

// aq_sb_target (lossy_state.rs:3796-3902) for one SB at tile-local (sb_x, sb_y)
// of a tile whose luma starts at yp with stride pw.
int32_t aq_sb_target(const uint16_t* yp, int pw, int tw, int th, int sb_x, int sb_y, const mt_aq_params* p,
                     const TileRefs& refs) {
  const int32_t base_q = p->base_q_idx;
  const int bd = p->bd;
  const float dark_scale = 1.0f / (float)(1u << (bd - 8));
  const int32_t dark = or_dark_protection(p->dark_aq, base_q, yp, pw, sb_y, sb_x, tw, th, dark_scale);
  if (p->variance_boost) {
    float subvars[64];
    const int filled = sb_subblock_variances(yp, pw, sb_y, sb_x, tw, th, subvars);
    if (filled == 0) return base_q;
    const float picked = octile_pick(subvars, std::min(std::max(p->octile, 1), 8));
    const float var_scale = 1.0f / (float)(1u << (2 * (bd - 8)));
    const float mid_t = clampf(((float)base_q - 48.0f) / 48.0f, 0.0f, 1.0f);
    const int32_t vb_delta = variance_boost_delta(picked * var_scale, refs.ref_act, refs.ref_pick,
                                                  fmaxr(p->strength, 0.0f), p->boost_only != 0, mid_t, 0.0f);
    const int32_t flat_boost = std::max(-vb_delta, 0);
    const int32_t protection = std::max(flat_boost, dark);
    int32_t delta;
    if (vb_delta > 0 && dark > 0)
      delta = vb_delta - dark;
    else if (protection > 0)
      delta = -protection;
    else
      delta = vb_delta;
    if (delta > 0) {
      const float g = 1.0f - 1.0f * top_ease_t(base_q);
      delta = sat_i32(or_fast_round((float)delta * g));
    }
    delta = clamp_aq_delta_relative(base_q, delta, bd);
    return std::min(std::max(base_q + delta, 1), 255);
  }
  const float act = sb_activity(yp, pw, sb_y, sb_x, tw, th, bd);
  const int32_t vb_delta = aq_target_qidx(base_q, act, refs.ref_act) - base_q;
  const int32_t flat_boost = std::max(-vb_delta, 0);
  const int32_t protection = std::max(flat_boost, dark);
  int32_t delta = protection > 0 ? -protection : vb_delta;
  delta = clamp_aq_delta_relative(base_q, delta, bd);
  return std::min(std::max(base_q + delta, 1), 255);
}

// tile_ref_activity / tile_ref_picked (aq.rs:162-192): raster means over the tile's SBs.
TileRefs tile_refs(const uint16_t* yp, int pw, int tw, int th, const mt_aq_params* p) {
  float sa = 0.0f, ca = 0.0f, sp = 0.0f, cp = 0.0f;
  const float var_scale = 1.0f / (float)(1u << (2 * (p->bd - 8)));
  const int octile = std::min(std::max(p->octile, 1), 8);
  for (int sb_y = 0; sb_y < th; sb_y += 64)
    for (int sb_x = 0; sb_x < tw; sb_x += 64) {
      sa += sb_activity(yp, pw, sb_y, sb_x, tw, th, p->bd);
      ca += 1.0f;
    }
  for (int sb_y = 0; sb_y < th; sb_y += 64)
    for (int sb_x = 0; sb_x < tw; sb_x += 64) {
      float subvars[64];
      if (sb_subblock_variances(yp, pw, sb_y, sb_x, tw, th, subvars) == 0) continue;
      const float picked = octile_pick(subvars, octile);
      sp += or_dirty_log1pf(picked * var_scale);
      cp += 1.0f;
    }
  TileRefs r;
  r.ref_act = ca > 0.0f ? sa / ca : 5.0f;
  r.ref_pick = cp > 0.0f ? sp / cp : 5.0f;
  return r;
}

int tile_log2(int blk, int target) {
  int k = 0;
  while ((blk << k) < target) k++;
  return k;
}

void tile_starts(int sbs, int log2, std::vector<int>& out) {
  const int size = (sbs + (1 << log2) - 1) >> log2;
  out.clear();
  for (int s = 0; s < sbs; s += size) out.push_back(s);
}

}  // namespace

extern "C" {

float or_fast_round(float x) {
  const float magic = (float)((1u << 23) + (1u << 22));
  return (bits_f(f_bits(x) + 1) + magic) - magic;
}

float or_dirty_log1pf(float d) {
  const uint32_t ix = f_bits(1.0f + d);
  const uint32_t exponent = ix & 0x7f800000u;
  const int32_t n = (int32_t)(exponent >> 23) - 0x7f;
  const float mantissa = bits_f((ix & 0x007fffffu) | 0x3f800000u);
  const float t = n == 0 ? d : mantissa - 1.0f;
  float p = 0.014539075084030628f;
  p = p * t + -0.0675969123840332f;
  p = p * t + 0.15056970715522766f;
  p = p * t + -0.23573730885982513f;
  p = p * t + 0.33125850558280945f;
  p = p * t + -0.4998837411403656f;
  p = p * t + 0.999998927116394f;
  return (float)n * 0.693147180559945309417232121458176568f + t * p;
}

void or_dark_pow(const float* x, float* out, int64_t n) {
  for (int64_t i = 0; i < n; i++) out[i] = powf(x[i], kDarkGamma);
}

// dark_protection (aq_common.rs:312-345) with DarkAq::on when enabled.
int32_t or_dark_protection(int32_t enabled, int32_t base_q, const uint16_t* yp, int32_t pw, int32_t sb_y, int32_t sb_x,
                           int32_t width, int32_t height, float scale) {
  if (!enabled || base_q < kDarkMinQ) return 0;
  float mean, mid;
  dark_structure_stats(yp, pw, sb_y, sb_x, width, height, scale, &mean, &mid);
  if (mid <= 0.0f) return 0;
  const float w = clampf(powf((kDarkMeanFloor + kDarkRef) / (kDarkMeanFloor + mean), kDarkGamma), 1.0f,
                         kDarkMaxWeight);
  const float darkness = w - 1.0f;
  if (darkness <= 0.0f) return 0;
  const float ds = or_dirty_log1pf(mid * darkness);
  return sat_i32(or_fast_round(fmaxr(fminr(ds * kDarkScale, (float)kDarkMaxQidx), 0.0f)));
}

int or_tiling_spec_min(int32_t w8, int32_t h8, int32_t* cols_log2, int32_t* rows_log2) {
  if (w8 <= 0 || h8 <= 0) return MT_ERR_INVALID_INPUT;
  const int sb_cols = (w8 + 63) / 64, sb_rows = (h8 + 63) / 64;
  const int min_c = tile_log2(64, sb_cols);
  const int max_c = tile_log2(1, std::min(sb_cols, 64));
  const int max_r = tile_log2(1, std::min(sb_rows, 64));
  const int min_tiles = std::max(min_c, tile_log2(2304, sb_rows * sb_cols));
  const int tcl = std::min(min_c, max_c);
  const int trl = std::min(std::max(min_tiles - tcl, 0), max_r);
  *cols_log2 = tcl;
  *rows_log2 = trl;
  return MT_OK;
}

// precompute_aq_grid (lossy_state.rs:3937-3963) for every tile of the frame;
// cells in frame raster order of superblocks, refs two floats per tile.
int or_aq_grid(const uint16_t* luma, const mt_aq_params* p, mt_aq_cell* cells, float* refs_out) {
  const int sb_cols = (p->w8 + 63) / 64, sb_rows = (p->h8 + 63) / 64;
  std::vector<int> cs, rs;
  tile_starts(sb_cols, p->tile_cols_log2, cs);
  tile_starts(sb_rows, p->tile_rows_log2, rs);
  int ti = 0;
  for (size_t r = 0; r < rs.size(); r++) {
    const int y0 = rs[r] * 64;
    const int y1 = std::min((r + 1 < rs.size() ? rs[r + 1] : sb_rows) * 64, p->h8);
    for (size_t c = 0; c < cs.size(); c++, ti++) {
      const int x0 = cs[c] * 64;
      const int x1 = std::min((c + 1 < cs.size() ? cs[c + 1] : sb_cols) * 64, p->w8);
      const int tw = x1 - x0, th = y1 - y0;
      const uint16_t* yp = luma + (size_t)y0 * p->w8 + x0;
      const TileRefs refs = tile_refs(yp, p->w8, tw, th, p);
      if (refs_out) {
        refs_out[2 * ti] = refs.ref_act;
        refs_out[2 * ti + 1] = refs.ref_pick;
      }
      int32_t cur = p->base_q_idx;
      for (int sy = 0; sy < th; sy += 64)
        for (int sx = 0; sx < tw; sx += 64) {
          const int32_t target = aq_sb_target(yp, p->w8, tw, th, sx, sy, p, refs);
          const float st = clampf(or_fast_round((float)(target - cur) / 4.0f), -12.0f, 12.0f);
          const int32_t steps = sat_i32(st);
          const int32_t newq = std::min(std::max(cur + steps * 4, 1), 255);
          mt_aq_cell& o = cells[(size_t)((y0 + sy) / 64) * sb_cols + (x0 + sx) / 64];
          o.prev = (uint8_t)cur;
          o.newq = (uint8_t)newq;
          o.steps = (int8_t)steps;
          o.target = (uint8_t)target;
          cur = newq;
        }
    }
  }
  return MT_OK;
}

}  // extern "C"
