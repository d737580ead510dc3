// Device AV1 intra prediction for one block per thread (src/intrapred.rs:1357-1810
// semantics): edge gathering with the reference's availability and fill rules,
// corner/edge filtering, 2x edge upsampling, directional zones 1-3, PAETH,
// SMOOTH*, and DC.  Edges live in a per-thread array with logical origin 2
// (indices -2 .. 2*(bw+bh)), the reference's IntraEdge layout.
#pragma once
#include <stdint.h>

#include "../../include/maroontree_b200.h"
#include "common.cuh"

namespace mtd {

__constant__ int16_t kDrDeriv[44] = {0,  1023, 0,  547, 372, 0,  0,  273, 215, 0,  178, 151, 0,  132, 116,
                                     0,  102,  0,  90,  80,  0,  71, 64,  0,   57, 51,  0,   45, 0,   40,
                                     35, 0,    31, 27,  0,   23, 19, 0,   15,  0,  11,  0,   7,  3};
__constant__ int16_t kSmW8[8] = {255, 197, 146, 105, 73, 50, 37, 32};
__constant__ int16_t kSmW4[4] = {255, 149, 85, 64};
__constant__ int16_t kSmW16[16] = {255, 225, 196, 170, 145, 123, 102, 84, 68, 54, 43, 33, 26, 20, 17, 16};
__constant__ int16_t kSmW32[32] = {255, 240, 225, 210, 196, 182, 169, 157, 145, 133, 122, 111, 101, 92, 83, 74,
                                   66,  59,  52,  45,  39,  34,  29,  25,  21,  17,  14,  12,  10,  9,  8,  8};

template <int N>
__device__ __forceinline__ int32_t sm_weight(int i) {
  return N == 4 ? kSmW4[i] : (N == 8 ? kSmW8[i] : (N == 16 ? kSmW16[i] : kSmW32[i]));
}

constexpr int kEdgeOrigin = 2;
// Words of one edge array for an N x N block: origin 2 plus the upsampled
// reach 2 * (2N) and slack.
template <int N>
__host__ __device__ constexpr int edge_cap() {
  return 2 + 4 * N + 4;
}
constexpr int kEdgeCap8 = edge_cap<8>();

__device__ __forceinline__ int edge_strength(int w, int h, bool ft, int delta) {
  const int d = abs(delta), wh = w + h;
  int s = 0;
  if (!ft) {
    if (wh <= 8) s = d >= 56;
    else if (wh <= 16) s = d >= 40;
    else if (wh <= 24) s = d >= 32 ? 3 : (d >= 16 ? 2 : (d >= 8 ? 1 : 0));
    else if (wh <= 32) s = d >= 32 ? 3 : (d >= 4 ? 2 : (d >= 1 ? 1 : 0));
    else s = d >= 1 ? 3 : 0;
  } else {
    if (wh <= 8) s = d >= 64 ? 2 : (d >= 40 ? 1 : 0);
    else if (wh <= 16) s = d >= 48 ? 2 : (d >= 20 ? 1 : 0);
    else if (wh <= 24) s = d >= 4 ? 3 : 0;
    else s = d >= 1 ? 3 : 0;
  }
  return s;
}

// 5-tap edge smoothing of positions 0..size-2 from the unfiltered window
// src[k] = edge[k-1] with clamped reads (src/intrapred.rs:977-1012).
__device__ __forceinline__ void filter_edge(int32_t* e, int size, int strength, int32_t* src) {
  if (strength == 0) return;
  int32_t k0, k1, k2;  // symmetric taps: (k0, k1, k2, k1, k0)
  if (strength == 1) { k0 = 0; k1 = 4; k2 = 8; }
  else if (strength == 2) { k0 = 0; k1 = 5; k2 = 6; }
  else { k0 = 2; k1 = 4; k2 = 4; }
  for (int i = 0; i < size; i++) src[i] = e[kEdgeOrigin + i - 1];
  const int last = size - 1;
  for (int o = 0; o < size - 1; o++) {
    const int32_t a = src[max(o - 1, 0)], b = src[min(max(o, 0), last)], c = src[min(o + 1, last)];
    const int32_t d = src[min(o + 2, last)], f = src[min(o + 3, last)];
    e[kEdgeOrigin + o] = (k0 * a + k1 * b + k2 * c + k1 * d + k0 * f + 8) >> 4;
  }
}

// 2x upsampling of num_px edge samples (src/intrapred.rs:1026-1048).
__device__ __forceinline__ void upsample_edge(int32_t* e, int num_px, int32_t maxv, int32_t* in) {
  in[0] = e[kEdgeOrigin - 1];
  in[1] = e[kEdgeOrigin - 1];
  for (int i = 0; i < num_px; i++) in[i + 2] = e[kEdgeOrigin + i];
  in[num_px + 2] = e[kEdgeOrigin + num_px - 1];
  e[kEdgeOrigin - 2] = in[0];
  for (int i = 0; i < num_px; i++) {
    const int32_t v = -in[i] + 9 * in[i + 1] + 9 * in[i + 2] - in[i + 3];
    e[kEdgeOrigin + 2 * i - 1] = clampi((v + 8) >> 4, 0, maxv);
    e[kEdgeOrigin + 2 * i] = in[i + 2];
  }
}

// Neighbour reads of the predictors: sample (x, y) of the reconstruction
// plane.  Other readers (a plane with a trial-coded patch laid over it) supply
// the same call.
struct PlaneRead {
  const uint16_t* __restrict__ p;
  int stride;
  __device__ __forceinline__ int32_t operator()(int x, int y) const { return p[(size_t)y * stride + x]; }
};

// DC predictor (src/intrapred.rs:1740-1789) for square power-of-two blocks.
template <typename R>
__device__ __forceinline__ int32_t dc_pred_sq_at(const R& rd, int ox, int oy, int n, int log2n, int bd) {
  const bool top = oy > 0, left = ox > 0;
  int32_t sum = 0;
  if (top)
    for (int x = 0; x < n; x++) sum += rd(ox + x, oy - 1);
  if (left)
    for (int y = 0; y < n; y++) sum += rd(ox - 1, oy + y);
  if (top && left) return (n + sum) >> (log2n + 1);
  if (top || left) return ((n >> 1) + sum) >> log2n;
  return 1 << (bd - 1);
}
__device__ __forceinline__ int32_t dc_pred_sq(const uint16_t* __restrict__ rec, int stride, int ox, int oy, int n,
                                              int log2n, int bd) {
  return dc_pred_sq_at(PlaneRead{rec, stride}, ox, oy, n, log2n, bd);
}

// Prediction of an N x N block (N = 4, 8, 16 or 32) into out[N*N] (row-major),
// neighbours read through `rd`.  `scratch` holds 3 * edge_cap<N>() words: the
// above and left edges and a filter temporary.  Only rows [y0, y1) of out are
// written (the edges are always built whole), so several threads can share
// one block's rows.
template <int N, typename R, typename O>
__device__ void predict_sq_at(const R& rd, int fw, int fh, int ox, int oy, int mode, int delta, bool have_tr,
                              bool have_bl, bool ft, int bd, O* __restrict__ out, int32_t* __restrict__ scratch,
                              int y0 = 0, int y1 = N) {
  static_assert(N == 4 || N == 8 || N == 16 || N == 32, "square sizes 4, 8, 16 and 32");
  constexpr int bw = N, bh = N, edge_len = 2 * N, cap = edge_cap<N>();
  if (mode == MT_DC_PRED) {
    const int32_t d = dc_pred_sq_at(rd, ox, oy, N, N == 4 ? 2 : (N == 8 ? 3 : (N == 16 ? 4 : 5)), bd);
    for (int i = y0 * N; i < y1 * N; i++) out[i] = (O)(d);
    return;
  }
  // Every edge entry the predictor reads is written below (logical -1 ..
  // 2N-1, and -2 .. 4N-2 once upsampled), so the arrays are not cleared.
  int32_t* A = scratch;
  int32_t* L = scratch + cap;
  int32_t* tmp = scratch + 2 * cap;
  const bool have_top = oy > 0, have_left = ox > 0;
  const int32_t base = 1 << (bd - 1);
  // above row at y = oy - 1 (valid when have_top), left column at x = ox - 1
  // (valid when have_left)
  if (have_top) {
    for (int i = 0; i < bw; i++) A[kEdgeOrigin + i] = rd(ox + i, oy - 1);
  } else {
    const int32_t fill = have_left ? rd(ox - 1, oy) : base - 1;
    for (int i = 0; i < edge_len; i++) A[kEdgeOrigin + i] = fill;
  }
  if (have_left) {
    for (int j = 0; j < bh; j++) L[kEdgeOrigin + j] = rd(ox - 1, oy + j);
  } else {
    const int32_t fill = have_top ? rd(ox, oy - 1) : base + 1;
    for (int i = 0; i < edge_len; i++) L[kEdgeOrigin + i] = fill;
  }
  const int32_t corner =
      have_left ? (have_top ? rd(ox - 1, oy - 1) : rd(ox - 1, oy)) : (have_top ? rd(ox, oy - 1) : base);
  A[kEdgeOrigin - 1] = corner;
  L[kEdgeOrigin - 1] = corner;
  if (have_top) {
    const int px_have = have_tr ? min(bw, max(fw - (ox + bw), 0)) : 0;
    for (int i = 0; i < px_have; i++) A[kEdgeOrigin + bw + i] = rd(ox + bw + i, oy - 1);
    const int32_t fill = A[kEdgeOrigin + bw + px_have - 1];
    for (int i = bw + px_have; i < edge_len; i++) A[kEdgeOrigin + i] = fill;
  }
  if (have_left) {
    const int px_have = have_bl ? min(bh, max(fh - (oy + bh), 0)) : 0;
    for (int i = 0; i < px_have; i++) L[kEdgeOrigin + bh + i] = rd(ox - 1, oy + bh + i);
    const int32_t fill = L[kEdgeOrigin + bh + px_have - 1];
    for (int i = bh + px_have; i < edge_len; i++) L[kEdgeOrigin + i] = fill;
  }
  const bool directional = mode >= MT_V_PRED && mode <= MT_D67_PRED;
  if (directional) {
    const int base_angle[9] = {0, 90, 180, 45, 135, 113, 157, 203, 67};
    const int angle = base_angle[mode] + delta * 3;
    int up_a = 0, up_l = 0;
    if (angle != 90 && angle != 180) {
      // The corner filter (src/intrapred.rs:1014-1019) for edge_len >= 24,
      // i.e. 16x16 and 32x32 here, before the edges are smoothed.
      if (edge_len >= 24 && angle > 90 && angle < 180) {
        const int32_t f = (5 * L[kEdgeOrigin] + 6 * A[kEdgeOrigin - 1] + 5 * A[kEdgeOrigin] + 8) >> 4;
        A[kEdgeOrigin - 1] = f;
        L[kEdgeOrigin - 1] = f;
      }
      filter_edge(A, bw + 1 + (angle < 90 ? bh : 0), edge_strength(bw, bh, ft, angle - 90), tmp);
      filter_edge(L, bh + 1 + (angle > 180 ? bw : 0), edge_strength(bh, bw, ft, angle - 180), tmp);
      const int da = abs(angle - 90), dl = abs(angle - 180);
      const int lim = ft ? 8 : 16;
      up_a = (da != 0 && da < 40 && bw + bh <= lim);
      up_l = (dl != 0 && dl < 40 && bw + bh <= lim);
      const int32_t maxv = (1 << bd) - 1;
      if (up_a) upsample_edge(A, bw + (angle < 90 ? bh : 0), maxv, tmp);
      if (up_l) upsample_edge(L, bh + (angle > 180 ? bw : 0), maxv, tmp);
    }
    const int32_t* a = A + kEdgeOrigin;  // logical index 0
    const int32_t* l = L + kEdgeOrigin;
    if (angle == 90) {
      for (int y = y0; y < y1; y++)
        for (int x = 0; x < bw; x++) out[y * bw + x] = (O)(a[x]);
    } else if (angle == 180) {
      for (int y = y0; y < y1; y++)
        for (int x = 0; x < bw; x++) out[y * bw + x] = (O)(l[y]);
    } else if (angle < 90) {
      const int dx = kDrDeriv[angle >> 1];
      const int max_base_x = (edge_len - 1) << up_a;
      const int frac_bits = 6 - up_a, inc = 1 << up_a;
      for (int y = y0; y < y1; y++) {
        const int xpos = dx * (y + 1);
        const int shift = ((xpos << up_a) & 0x3f) >> 1;
        const int b0 = xpos >> frac_bits;
        for (int x = 0; x < bw; x++) {
          const int b = b0 + x * inc;
          out[y * bw + x] = (O)(b < max_base_x ? (a[b] * (32 - shift) + a[b + 1] * shift + 16) >> 5 : a[max_base_x]);
        }
      }
    } else if (angle > 180) {
      const int dy = kDrDeriv[(270 - angle) >> 1];
      const int max_base_y = (edge_len - 1) << up_l;
      const int frac_bits = 6 - up_l, inc = 1 << up_l;
      for (int y = y0; y < y1; y++)
        for (int x = 0; x < bw; x++) {
          const int ypos = dy * (x + 1);
          const int shift = ((ypos << up_l) & 0x3f) >> 1;
          const int b = (ypos >> frac_bits) + y * inc;
          out[y * bw + x] = (O)(b >= max_base_y ? l[max_base_y] : (l[b] * (32 - shift) + l[b + 1] * shift + 16) >> 5);
        }
    } else {
      const int dy = kDrDeriv[(angle - 90) >> 1];
      const int dx = kDrDeriv[(180 - angle) >> 1];
      for (int y = y0; y < y1; y++) {
        const int t = (y + 1) * dx - 64;
        const int x0 = t <= 0 ? 0 : min((t + 63) >> 6, bw);
        const int xpos0 = (x0 << 6) - (y + 1) * dx;
        const int ba0 = xpos0 >> (6 - up_a);
        const int sha = ((xpos0 * (1 << up_a)) & 0x3f) >> 1;
        for (int x = 0; x < bw; x++) {
          if (x < x0) {
            const int ypos = (y << 6) - (x + 1) * dy;
            const int b = ypos >> (6 - up_l);
            const int sh = ((ypos * (1 << up_l)) & 0x3f) >> 1;
            out[y * bw + x] = (O)((l[b] * (32 - sh) + l[b + 1] * sh + 16) >> 5);
          } else {
            const int b = ba0 + (x - x0) * (1 << up_a);
            out[y * bw + x] = (O)((a[b] * (32 - sha) + a[b + 1] * sha + 16) >> 5);
          }
        }
      }
    }
    return;
  }
  const int32_t* a = A + kEdgeOrigin;
  const int32_t* l = L + kEdgeOrigin;
  if (mode == MT_PAETH_PRED) {
    for (int y = y0; y < y1; y++)
      for (int x = 0; x < bw; x++) {
        const int32_t lv = l[y], tv = a[x], b = lv + tv - corner;
        const int32_t ld = abs(lv - b), td = abs(tv - b), cd = abs(corner - b);
        out[y * bw + x] = (O)((ld <= td && ld <= cd) ? lv : (td <= cd ? tv : corner));
      }
  } else if (mode == MT_SMOOTH_PRED) {
    const int32_t right = a[bw - 1], bottom = l[bh - 1];
    for (int y = y0; y < y1; y++)
      for (int x = 0; x < bw; x++) {
        const int32_t wv = sm_weight<N>(y), wh = sm_weight<N>(x);
        const int32_t p = wv * a[x] + (256 - wv) * bottom + wh * l[y] + (256 - wh) * right;
        out[y * bw + x] = (O)((p + 256) >> 9);
      }
  } else if (mode == MT_SMOOTH_V_PRED) {
    const int32_t bottom = l[bh - 1];
    for (int y = y0; y < y1; y++)
      for (int x = 0; x < bw; x++)
        out[y * bw + x] = (O)((sm_weight<N>(y) * a[x] + (256 - sm_weight<N>(y)) * bottom + 128) >> 8);
  } else {  // SMOOTH_H
    const int32_t right = a[bw - 1];
    for (int y = y0; y < y1; y++)
      for (int x = 0; x < bw; x++)
        out[y * bw + x] = (O)((sm_weight<N>(x) * l[y] + (256 - sm_weight<N>(x)) * right + 128) >> 8);
  }
}

template <int N, typename O>
__device__ __forceinline__ void predict_sq(const uint16_t* __restrict__ rec, int stride, int fw, int fh, int ox, int oy,
                                           int mode, int delta, bool have_tr, bool have_bl, bool ft, int bd,
                                           O* __restrict__ out, int32_t* __restrict__ scratch, int y0 = 0,
                                           int y1 = N) {
  predict_sq_at<N>(PlaneRead{rec, stride}, fw, fh, ox, oy, mode, delta, have_tr, have_bl, ft, bd, out, scratch, y0,
                   y1);
}

template <typename O>
__device__ __forceinline__ void predict8(const uint16_t* __restrict__ rec, int stride, int fw, int fh, int ox, int oy,
                                         int mode, int delta, bool have_tr, bool have_bl, bool ft, int bd,
                                         O* __restrict__ out, int32_t* __restrict__ scratch) {
  predict_sq<8>(rec, stride, fw, fh, ox, oy, mode, delta, have_tr, have_bl, ft, bd, out, scratch);
}

}  // namespace mtd
