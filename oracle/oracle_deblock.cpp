// Oracle (test infrastructure only): the reference's deblocking filter,
// restated in the reference's own processing order.
//   limits                src/loopfilter.rs:31-44  (dav1d_calc_eih)
//   loop_filter_scalar    src/loopfilter.rs:98-292 (dav1d loop_filter port)
//   luma_cls / chroma_cls src/loopfilter.rs:396-412
//   filter_plane_impl     src/loopfilter.rs:482-648 (per superblock row: vertical
//                         edges, then horizontal edges; scalar edge path)
//   frame_deblock         src/coder/frame_deblock.rs:87-224, src/obu.rs:306-334
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include <vector>

#include "oracle.h"

namespace {

void limits(int level, int sharp, int* e, int* i_lim, int* h) {
  int i = level;
  if (sharp > 0) {
    i >>= (sharp + 3) >> 2;
    if (i > 9 - sharp) i = 9 - sharp;
  }
  if (i < 1) i = 1;
  *e = 2 * (level + 2) + i;
  *i_lim = i;
  *h = level >> 4;
}

inline int iclip(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// One line of src/loopfilter.rs:98-292 (the reference loops this over the
// edge segment's four lines, each line deciding on its own samples).
void loop_filter_line(uint16_t* dst, long o, int e, int i_lim, int h_thresh, long sb, int wd, int bd) {
  const int bm8 = bd - 8;
  const int f_flat = 1 << bm8;
  e <<= bm8;
  i_lim <<= bm8;
  h_thresh <<= bm8;
  const int px_max = (1 << bd) - 1;
  const int clip_lo = -128 * (1 << bm8), clip_hi = 128 * (1 << bm8) - 1;
  {
    auto g = [&](int k) -> int { return dst[o + k * sb]; };
    auto put = [&](int k, int v) { dst[o + k * sb] = (uint16_t)v; };
    int p1 = g(-2), p0 = g(-1), q0 = g(0), q1 = g(1);
    bool fm = abs(p1 - p0) <= i_lim && abs(q1 - q0) <= i_lim && abs(p0 - q0) * 2 + (abs(p1 - q1) >> 1) <= e;
    int p2 = 0, q2 = 0, p3 = 0, q3 = 0;
    if (wd > 4) {
      p2 = g(-3);
      q2 = g(2);
      fm = fm && abs(p2 - p1) <= i_lim && abs(q2 - q1) <= i_lim;
      if (wd > 6) {
        p3 = g(-4);
        q3 = g(3);
        fm = fm && abs(p3 - p2) <= i_lim && abs(q3 - q2) <= i_lim;
      }
    }
    if (!fm) return;
    int p6 = 0, p5 = 0, p4 = 0, q4 = 0, q5 = 0, q6 = 0;
    bool flat8out = false;
    if (wd >= 16) {
      p6 = g(-7);
      p5 = g(-6);
      p4 = g(-5);
      q4 = g(4);
      q5 = g(5);
      q6 = g(6);
      flat8out = abs(p6 - p0) <= f_flat && abs(p5 - p0) <= f_flat && abs(p4 - p0) <= f_flat &&
                 abs(q4 - q0) <= f_flat && abs(q5 - q0) <= f_flat && abs(q6 - q0) <= f_flat;
    }
    bool flat8in = false;
    if (wd >= 6)
      flat8in = abs(p2 - p0) <= f_flat && abs(p1 - p0) <= f_flat && abs(q1 - q0) <= f_flat && abs(q2 - q0) <= f_flat;
    if (wd >= 8) flat8in = flat8in && abs(p3 - p0) <= f_flat && abs(q3 - q0) <= f_flat;
    if (wd >= 16 && flat8out && flat8in) {
      put(-6, (p6 * 7 + p5 * 2 + p4 * 2 + p3 + p2 + p1 + p0 + q0 + 8) >> 4);
      put(-5, (p6 * 5 + p5 * 2 + p4 * 2 + p3 * 2 + p2 + p1 + p0 + q0 + q1 + 8) >> 4);
      put(-4, (p6 * 4 + p5 + p4 * 2 + p3 * 2 + p2 * 2 + p1 + p0 + q0 + q1 + q2 + 8) >> 4);
      put(-3, (p6 * 3 + p5 + p4 + p3 * 2 + p2 * 2 + p1 * 2 + p0 + q0 + q1 + q2 + q3 + 8) >> 4);
      put(-2, (p6 * 2 + p5 + p4 + p3 + p2 * 2 + p1 * 2 + p0 * 2 + q0 + q1 + q2 + q3 + q4 + 8) >> 4);
      put(-1, (p6 + p5 + p4 + p3 + p2 + p1 * 2 + p0 * 2 + q0 * 2 + q1 + q2 + q3 + q4 + q5 + 8) >> 4);
      put(0, (p5 + p4 + p3 + p2 + p1 + p0 * 2 + q0 * 2 + q1 * 2 + q2 + q3 + q4 + q5 + q6 + 8) >> 4);
      put(1, (p4 + p3 + p2 + p1 + p0 + q0 * 2 + q1 * 2 + q2 * 2 + q3 + q4 + q5 + q6 + q6 + 8) >> 4);
      put(2, (p3 + p2 + p1 + p0 + q0 + q1 * 2 + q2 * 2 + q3 * 2 + q4 + q5 + q6 + q6 + q6 + 8) >> 4);
      put(3, (p2 + p1 + p0 + q0 + q1 + q2 * 2 + q3 * 2 + q4 * 2 + q5 + q6 + q6 + q6 + q6 + 8) >> 4);
      put(4, (p1 + p0 + q0 + q1 + q2 + q3 * 2 + q4 * 2 + q5 * 2 + q6 * 5 + 8) >> 4);
      put(5, (p0 + q0 + q1 + q2 + q3 + q4 * 2 + q5 * 2 + q6 * 7 + 8) >> 4);
    } else if (wd >= 8 && flat8in) {
      put(-3, (p3 * 3 + 2 * p2 + p1 + p0 + q0 + 4) >> 3);
      put(-2, (p3 * 2 + p2 + 2 * p1 + p0 + q0 + q1 + 4) >> 3);
      put(-1, (p3 + p2 + p1 + 2 * p0 + q0 + q1 + q2 + 4) >> 3);
      put(0, (p2 + p1 + p0 + 2 * q0 + q1 + q2 + q3 + 4) >> 3);
      put(1, (p1 + p0 + q0 + 2 * q1 + q2 + q3 + q3 + 4) >> 3);
      put(2, (p0 + q0 + q1 + 2 * q2 + q3 + q3 + q3 + 4) >> 3);
    } else if (wd == 6 && flat8in) {
      put(-2, (p2 * 3 + 2 * p1 + 2 * p0 + q0 + 4) >> 3);
      put(-1, (p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3);
      put(0, (p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3);
      put(1, (p0 + 2 * q0 + 2 * q1 + 2 * q2 + q2 + 4) >> 3);
    } else {
      const bool hev = abs(p1 - p0) > h_thresh || abs(q1 - q0) > h_thresh;
      if (hev) {
        int fv = iclip(p1 - q1, clip_lo, clip_hi);
        fv = iclip(3 * (q0 - p0) + fv, clip_lo, clip_hi);
        const int f1 = (fv + 4 < clip_hi ? fv + 4 : clip_hi) >> 3;
        const int f2 = (fv + 3 < clip_hi ? fv + 3 : clip_hi) >> 3;
        put(-1, iclip(p0 + f2, 0, px_max));
        put(0, iclip(q0 - f1, 0, px_max));
      } else {
        const int fv = iclip(3 * (q0 - p0), clip_lo, clip_hi);
        const int f1 = (fv + 4 < clip_hi ? fv + 4 : clip_hi) >> 3;
        const int f2 = (fv + 3 < clip_hi ? fv + 3 : clip_hi) >> 3;
        put(-1, iclip(p0 + f2, 0, px_max));
        put(0, iclip(q0 - f1, 0, px_max));
        const int f = (f1 + 1) >> 1;
        put(-2, iclip(p1 + f, 0, px_max));
        put(1, iclip(q1 - f, 0, px_max));
      }
    }
  }
}

inline int cls_of(int d, bool luma) {
  if (luma) return d == 1 ? 0 : (d == 2 ? 1 : 2);
  return d >= 2 ? 1 : 0;
}
inline int wd_of(int wcls, bool luma) { return luma ? 4 << wcls : 4 + 2 * wcls; }
// Samples a filter of width wd reads before / after the edge.  Edges whose taps
// would leave their row (vertical edges) or the plane (horizontal edges) are
// skipped: the reference indexes outside the row there (a panic or a read of
// the neighbouring row, by SIMD dispatch), which no AV1 block geometry reaches.
inline int reach_lo(int wd) { return wd == 16 ? 7 : (wd == 8 ? 4 : (wd == 6 ? 3 : 2)); }
inline int reach_hi(int wd) { return wd == 16 ? 6 : (wd == 8 ? 3 : (wd == 6 ? 2 : 1)); }

}  // namespace

extern "C" int or_deblock_plane(uint16_t* px, int32_t w, int32_t h, int32_t vis_w, int32_t vis_h, const uint8_t* bw4,
                                const uint8_t* bh4, const uint8_t* vedge4, const uint8_t* hedge4, int32_t nc4,
                                int32_t level, int32_t sharp, int32_t is_luma, int32_t sb_rows4, int32_t bd) {
  if (level <= 0) return MT_OK;
  int e, i_lim, h_thresh;
  limits(level, sharp, &e, &i_lim, &h_thresh);
  const int w4 = (vis_w + 3) / 4, h4 = (vis_h + 3) / 4;
  const bool luma = is_luma != 0;
  for (int sb_top = 0; sb_top < h4; sb_top += sb_rows4) {
    const int sb_bot = sb_top + sb_rows4 < h4 ? sb_top + sb_rows4 : h4;
    // vertical edges (scalar path of filter_plane_impl)
    for (int r4 = sb_top; r4 < sb_bot; r4++) {
      if (r4 * 4 >= h) continue;
      for (int c4 = 1; c4 < w4; c4++) {
        const int x0 = c4 * 4;
        if (x0 >= w) continue;
        const int idx = r4 * nc4 + c4;
        const int cur = bw4[idx], left = bw4[idx - 1];
        if (cur == 0) continue;  // not a block size (the reference divides by it)
        const bool present = vedge4 ? vedge4[idx] != 0 : (c4 % cur == 0);
        if (!present) continue;
        const int wcls = cls_of(cur, luma) < cls_of(left, luma) ? cls_of(cur, luma) : cls_of(left, luma);
        const int wd = wd_of(wcls, luma);
        if (x0 - reach_lo(wd) < 0 || x0 + reach_hi(wd) >= w) continue;
        for (int line = 0; line < 4; line++)
          loop_filter_line(px, (long)(r4 * 4 + line) * w + x0, e, i_lim, h_thresh, 1, wd, bd);
      }
    }
    // horizontal edges
    for (int r4 = sb_top; r4 < sb_bot; r4++) {
      if (r4 == 0) continue;
      for (int c4 = 0; c4 < w4; c4++) {
        const int idx = r4 * nc4 + c4;
        const int cur = bh4[idx], top = bh4[(r4 - 1) * nc4 + c4];
        if (cur == 0) continue;
        const bool present = hedge4 ? hedge4[idx] != 0 : (r4 % cur == 0);
        if (!present) continue;
        const int wcls = cls_of(cur, luma) < cls_of(top, luma) ? cls_of(cur, luma) : cls_of(top, luma);
        const int y0 = r4 * 4, x0 = c4 * 4;
        if (y0 >= h || x0 >= w) continue;
        const int wd = wd_of(wcls, luma);
        if (y0 - reach_lo(wd) < 0 || y0 + reach_hi(wd) >= h) continue;
        for (int line = 0; line < 4; line++) loop_filter_line(px, (long)y0 * w + x0 + line, e, i_lim, h_thresh, w, wd, bd);
      }
    }
  }
  return MT_OK;
}

// src/obu.rs:306-334 with the shipped tuning (lf_level_scale 1, lf_uv_level_scale
// 1, lf_uv_level_scale_420 0.5, lf_sharpness 7; src/tuning.rs:764-767).
extern "C" void or_loop_filter_levels(int32_t base_q_idx, int32_t sub, int32_t* lvl_y, int32_t* lvl_uv,
                                      int32_t* sharp) {
  const int q = base_q_idx;
  const float uv_scale = sub == 2 ? 0.5f : 1.0f;
  int ly = (int)roundf((float)(q / 8) * 1.0f);
  ly = ly < 0 ? 0 : (ly > 40 ? 40 : ly);
  int luv = 0;
  if (ly > 0) {
    luv = (int)roundf((float)(q / 10) * uv_scale);
    if (luv < 1) luv = 1;
    luv = luv > 32 ? 32 : luv;
  }
  *lvl_y = ly;
  *lvl_uv = luv;
  *sharp = 7;
}

// src/coder/frame_deblock.rs:87-224: frame_deblock with chroma_deblock_geom
// (cdblk_variant 1: prediction geometry, alignment-rule chroma edges).
extern "C" int or_deblock_frame(uint16_t* y, uint16_t* u, uint16_t* v, const uint8_t* blk4, const uint8_t* blk4h,
                                const uint8_t* blk4v, const uint8_t* blk4t, const uint8_t* pblk4,
                                const uint8_t* pblk4h, const mt_deblock_frame_params* g, int32_t lvl_y,
                                int32_t lvl_u, int32_t lvl_v) {
  const int nc4 = g->w8 / 4;
  if (lvl_y > 0)
    or_deblock_plane(y, g->w8, g->h8, g->disp_w, g->disp_h, blk4, blk4h, blk4v, blk4t, nc4, lvl_y, 7, 1, 16, g->bd);
  if (g->mono || lvl_y <= 0 || (lvl_u <= 0 && lvl_v <= 0)) return MT_OK;
  const int ss_hor = g->sub_x, ss_ver = g->sub_y;
  const int cw8 = g->w8 >> ss_hor, ch8 = g->h8 >> ss_ver;
  const int cnc4 = cw8 / 4, cnr4 = ch8 / 4;
  std::vector<uint8_t> cbw4(cnc4 * cnr4), cbh4(cnc4 * cnr4);
  for (int cr = 0; cr < cnr4; cr++)
    for (int cc = 0; cc < cnc4; cc++) {
      const int li = (cr << ss_ver) * nc4 + (cc << ss_hor), ci = cr * cnc4 + cc;
      int sw = pblk4[li] >> ss_hor, sh = pblk4h[li] >> ss_ver;
      sw = sw < 1 ? 1 : (sw > 8 ? 8 : sw);
      sh = sh < 1 ? 1 : (sh > 8 ? 8 : sh);
      cbw4[ci] = (uint8_t)sw;
      cbh4[ci] = (uint8_t)sh;
    }
  const int vis_w = (g->disp_w + (1 << ss_hor) - 1) >> ss_hor, vis_h = (g->disp_h + (1 << ss_ver) - 1) >> ss_ver;
  const int sb_rows4 = 16 >> ss_ver;
  if (lvl_u > 0)
    or_deblock_plane(u, cw8, ch8, vis_w, vis_h, cbw4.data(), cbh4.data(), nullptr, nullptr, cnc4, lvl_u, 7, 0,
                     sb_rows4, g->bd);
  if (lvl_v > 0)
    or_deblock_plane(v, cw8, ch8, vis_w, vis_h, cbw4.data(), cbh4.data(), nullptr, nullptr, cnc4, lvl_v, 7, 0,
                     sb_rows4, g->bd);
  return MT_OK;
}
