// The 8x8 candidate chain of chain8.cuh evaluated by EIGHT lanes of one warp
// (an "octet") instead of one thread, for launches whose latency, not their
// throughput, bounds the run: the superblock wavefront of the encoder, where
// a few dozen blocks per dependency level are all the work there is.
//
// Same arithmetic, same order, same results as chain8_tx (bit for bit):
//   * lane j owns row j of the residual, the row passes and the prediction,
//     and column j of the column passes; the octet's working set lives in
//     shared memory (Oct8) and the lanes meet at __syncwarp on the octet mask;
//   * quantisation, the QM step and the trellis round-down decisions are
//     per coefficient (the reference's AVX2 chunks decide each position from
//     the chunk's starting values, so only the chunk's "any level > 63" flag
//     is shared, by ballot);
//   * the float chains that have an order (the trellis suffix sums of the
//     zeroing distortion, its running prefix cost, the rate walk's sum) keep
//     it: their terms are computed by all lanes in parallel and added by one
//     lane in the reference's order; integer sums (SATD, counts) are reduced
//     across lanes in any order.
#pragma once
#include <stdint.h>

#include "chain8.cuh"

namespace mtd {

// Shared-memory working set of one octet.  t: the transform scratch (68 words:
// 64 + the suffix sums' extra entry); tf: targets (column-major rc), later the
// trellis rate terms; x: the trellis prefix terms, later the rate terms; cf:
// levels (column-major); rr: residual and then the inverse residual
// (row-major).
struct Oct8 {
  int32_t t[68];
  float tf[64];
  float x[64];
  int16_t cf[64];
  int16_t rr[64];
};

// Scan tables read with lane-dependent indices: in shared memory, where
// eight different addresses cost one access (the constant cache would
// serialise them).
struct CoopTabs {
  uint8_t scan[64];   // kScan8
  uint8_t iscan[64];  // kIScan8
  uint8_t loctx[32];  // kLoCtxOff
  // vmask[rc] bit k: the rate walk's neighbour rc + {1, 8, 9, 2, 16}[k] lies in
  // the block and comes later in the scan (so the reverse walk has already
  // entered its level when it reaches rc)
  uint8_t vmask[64];
  __device__ __forceinline__ void load(int t, int nthreads) {
    for (int i = t; i < 64; i += nthreads) {
      scan[i] = kScan8[i];
      iscan[i] = kIScan8[i];
      if (i < 25) loctx[i] = kLoCtxOff[i];
      const int off[5] = {1, 8, 9, 2, 16};
      uint8_t m = 0;
#pragma unroll
      for (int k = 0; k < 5; k++)
        if (i + off[k] < 64 && kIScan8[i + off[k]] > kIScan8[i]) m |= (uint8_t)(1 << k);
      vmask[i] = m;
    }
  }
};

// Column / row kinds of the seven 8x8 intra types (0 identity, 1 DCT, 2 ADST),
// col_kind / row_kind of txfm8.cuh without the local array.
__device__ __forceinline__ int coop_col_kind(int tx) { return (0x1A14 >> (2 * tx)) & 3; }
__device__ __forceinline__ int coop_row_kind(int tx) { return (0x2644 >> (2 * tx)) & 3; }

struct Octet {
  unsigned mask;  // the octet's 8 lanes within the warp
  int j;          // lane within the octet
  __device__ __forceinline__ Octet() : mask(0xFFu << (threadIdx.x & 24)), j(threadIdx.x & 7) {}
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
  __device__ __forceinline__ int max(int v) const { return (int)__reduce_max_sync(mask, (unsigned)v); }
  __device__ __forceinline__ unsigned sum(unsigned v) const { return __reduce_add_sync(mask, v); }
  __device__ __forceinline__ bool any(bool v) const { return (__ballot_sync(mask, v) & mask) != 0; }
};

// The neighbours an 8x8 (or smaller) intra predictor can read, staged in
// shared memory: above[k] = sample (ox - 1 + k, oy - 1) for k in [0, 17) and
// left[k] = sample (ox - 1, oy + k) for k in [0, 16).  The predictor reads
// only samples its availability rules allow, all of which are in these two
// runs.
struct EdgeRead {
  const int16_t* above;
  const int16_t* left;
  int ox, oy;
  __device__ __forceinline__ int32_t operator()(int x, int y) const {
    return y < oy ? above[x - ox + 1] : left[y - oy];
  }
};

// Rows [j, j+1) of the prediction of candidate cd (delta, flags as in
// chain8_predict) into pred (shared, row-major), neighbours read through
// `rd`; every lane builds the edges itself in `scratch` (3 * kEdgeCap8
// words).
template <typename R>
__device__ __forceinline__ void coop8_predict_row(const R& rd, const mt_chain_params& p, const mt_candidate& cd,
                                                  int16_t* pred, int32_t* scratch, const Octet& g) {
  predict_sq_at<8>(rd, p.frame_w, p.frame_h, cd.px, cd.py, cd.mode, cd.angle_delta, cd.flags & 1,
                   (cd.flags >> 1) & 1, (cd.flags >> 2) & 1, p.bd, pred, scratch, g.j, g.j + 1);
}

// Shared scratch of the lane-parallel 8x8 predictor: the above and left edges
// (logical index -2 .. 33 at offset 2, predict_sq_at's IntraEdge layout) and
// their copies, which the edge filter and the upsampler read.
struct Edge8 {
  int32_t a[40], l[40], ca[40], cl[40];
};

// One output of filter_edge (src/intrapred.rs:977-1012) at position o of an
// edge of `size` entries, from the unfiltered copy src[k] = e[k - 1].
__device__ __forceinline__ int32_t edge_tap(const int32_t* src, int o, int size, int strength) {
  const int32_t k0 = strength == 3 ? 2 : 0, k1 = strength == 1 ? 4 : (strength == 2 ? 5 : 4),
                k2 = strength == 1 ? 8 : (strength == 2 ? 6 : 4);
  const int last = size - 1;
  const int32_t a = src[::max(o - 1, 0)], b = src[::min(::max(o, 0), last)], c = src[::min(o + 1, last)];
  const int32_t d = src[::min(o + 2, last)], f = src[::min(o + 3, last)];
  return (k0 * a + k1 * b + k2 * c + k1 * d + k0 * f + 8) >> 4;
}

// predict_sq_at<8> (intrapred.cuh) split over the octet: the edges are built,
// filtered and upsampled position by position in E (each lane a few
// positions from copies taken before the step), then lane j writes row j of
// the prediction into pred (shared, row-major).  Same values as
// predict_sq_at<8> for every mode, angle delta and availability.
template <typename R>
__device__ void coop8_predict(const R& rd, const mt_chain_params& p, const mt_candidate& cd, int16_t* pred, Edge8& E,
                              const Octet& g) {
  constexpr int bw = 8, bh = 8, edge_len = 16;
  const int j = g.j, y = j;
  const int ox = cd.px, oy = cd.py, mode = cd.mode;
  const bool have_tr = cd.flags & 1, have_bl = (cd.flags >> 1) & 1, ft = (cd.flags >> 2) & 1;
  const int bd = p.bd;
  const bool have_top = oy > 0, have_left = ox > 0;
  const int32_t base = 1 << (bd - 1);
  int16_t* out = pred + y * 8;
  if (mode == MT_DC_PRED) {  // dc_pred_sq_at: (n + sum) >> (log2n + 1), or one side >> log2n
    const int32_t s = (have_top ? rd(ox + j, oy - 1) : 0) + (have_left ? rd(ox - 1, oy + j) : 0);
    const int32_t sum = (int32_t)g.sum((unsigned)s);
    const int32_t d = (have_top && have_left) ? (8 + sum) >> 4 : ((have_top || have_left) ? (4 + sum) >> 3 : base);
#pragma unroll
    for (int x = 0; x < 8; x++) out[x] = (int16_t)d;
    return;
  }
  int32_t* A = E.a + 2;
  int32_t* L = E.l + 2;
  // edges: lane j fills positions j and 8 + j of each
  if (have_top) {
    const int px_have = have_tr ? ::min(bw, ::max(p.frame_w - (ox + bw), 0)) : 0;
    A[j] = rd(ox + j, oy - 1);
    A[8 + j] = rd(ox + 8 + (j < px_have ? j : px_have - 1), oy - 1);  // the last available sample repeated
  } else {
    const int32_t fill = have_left ? rd(ox - 1, oy) : base - 1;
    A[j] = fill;
    A[8 + j] = fill;
  }
  if (have_left) {
    const int px_have = have_bl ? ::min(bh, ::max(p.frame_h - (oy + bh), 0)) : 0;
    L[j] = rd(ox - 1, oy + j);
    L[8 + j] = rd(ox - 1, oy + 8 + (j < px_have ? j : px_have - 1));
  } else {
    const int32_t fill = have_top ? rd(ox, oy - 1) : base + 1;
    L[j] = fill;
    L[8 + j] = fill;
  }
  const int32_t corner =
      have_left ? (have_top ? rd(ox - 1, oy - 1) : rd(ox - 1, oy)) : (have_top ? rd(ox, oy - 1) : base);
  if (j == 0) A[-1] = L[-1] = corner;
  g.sync();
  const bool directional = mode >= MT_V_PRED && mode <= MT_D67_PRED;
  if (directional) {
    const int base_angle = mode == MT_V_PRED ? 90 : mode == MT_H_PRED ? 180 : mode == MT_D45_PRED ? 45
                         : mode == MT_D135_PRED ? 135 : mode == MT_D113_PRED ? 113 : mode == MT_D157_PRED ? 157
                         : mode == MT_D203_PRED ? 203 : 67;
    const int angle = base_angle + cd.angle_delta * 3;
    int up_a = 0, up_l = 0;
    if (angle != 90 && angle != 180) {  // (the corner filter needs edges of 24 or more)
      const int sa = edge_strength(bw, bh, ft, angle - 90), sl = edge_strength(bh, bw, ft, angle - 180);
      const int na = bw + 1 + (angle < 90 ? bh : 0), nl = bh + 1 + (angle > 180 ? bw : 0);
      for (int k = j; k < 18; k += 8) {  // copies src[k] = e[k - 1]
        E.ca[k] = A[k - 1];
        E.cl[k] = L[k - 1];
      }
      g.sync();
      if (sa)
        for (int o = j; o < na - 1; o += 8) A[o] = edge_tap(E.ca, o, na, sa);
      if (sl)
        for (int o = j; o < nl - 1; o += 8) L[o] = edge_tap(E.cl, o, nl, sl);
      g.sync();
      const int da = abs(angle - 90), dl = abs(angle - 180), lim = ft ? 8 : 16;
      up_a = (da != 0 && da < 40 && bw + bh <= lim);
      up_l = (dl != 0 && dl < 40 && bw + bh <= lim);
      if (up_a || up_l) {  // upsample_edge (src/intrapred.rs:1026-1048)
        const int32_t maxv = (1 << bd) - 1;
        const int numa = bw + (angle < 90 ? bh : 0), numl = bh + (angle > 180 ? bw : 0);
        for (int k = j; k < 18; k += 8) {  // copies c[m] = e[m - 1], m = 0 .. num
          if (up_a && k <= numa) E.ca[k] = A[k - 1];
          if (up_l && k <= numl) E.cl[k] = L[k - 1];
        }
        g.sync();
        auto in = [](const int32_t* c, int k, int num) { return c[k <= 1 ? 0 : ::min(k - 1, num)]; };
        if (up_a) {
          if (j == 0) A[-2] = E.ca[0];
          for (int i = j; i < numa; i += 8) {
            const int32_t v = -in(E.ca, i, numa) + 9 * in(E.ca, i + 1, numa) + 9 * in(E.ca, i + 2, numa) -
                              in(E.ca, i + 3, numa);
            A[2 * i - 1] = clampi((v + 8) >> 4, 0, maxv);
            A[2 * i] = in(E.ca, i + 2, numa);
          }
        }
        if (up_l) {
          if (j == 0) L[-2] = E.cl[0];
          for (int i = j; i < numl; i += 8) {
            const int32_t v = -in(E.cl, i, numl) + 9 * in(E.cl, i + 1, numl) + 9 * in(E.cl, i + 2, numl) -
                              in(E.cl, i + 3, numl);
            L[2 * i - 1] = clampi((v + 8) >> 4, 0, maxv);
            L[2 * i] = in(E.cl, i + 2, numl);
          }
        }
        g.sync();
      }
    }
    const int32_t* a = A;
    const int32_t* l = L;
    if (angle == 90) {
#pragma unroll
      for (int x = 0; x < 8; x++) out[x] = (int16_t)a[x];
    } else if (angle == 180) {
#pragma unroll
      for (int x = 0; x < 8; x++) out[x] = (int16_t)l[y];
    } else if (angle < 90) {
      const int dx = kDrDeriv[angle >> 1];
      const int max_base_x = (edge_len - 1) << up_a;
      const int frac_bits = 6 - up_a, inc = 1 << up_a;
      const int xpos = dx * (y + 1);
      const int shift = ((xpos << up_a) & 0x3f) >> 1;
      const int b0 = xpos >> frac_bits;
#pragma unroll
      for (int x = 0; x < 8; x++) {
        const int b = b0 + x * inc;
        out[x] = (int16_t)(b < max_base_x ? (a[b] * (32 - shift) + a[b + 1] * shift + 16) >> 5 : a[max_base_x]);
      }
    } else if (angle > 180) {
      const int dy = kDrDeriv[(270 - angle) >> 1];
      const int max_base_y = (edge_len - 1) << up_l;
      const int frac_bits = 6 - up_l, inc = 1 << up_l;
#pragma unroll
      for (int x = 0; x < 8; x++) {
        const int ypos = dy * (x + 1);
        const int shift = ((ypos << up_l) & 0x3f) >> 1;
        const int b = (ypos >> frac_bits) + y * inc;
        out[x] = (int16_t)(b >= max_base_y ? l[max_base_y] : (l[b] * (32 - shift) + l[b + 1] * shift + 16) >> 5);
      }
    } else {
      const int dy = kDrDeriv[(angle - 90) >> 1];
      const int dx = kDrDeriv[(180 - angle) >> 1];
      const int t = (y + 1) * dx - 64;
      const int x0 = t <= 0 ? 0 : ::min((t + 63) >> 6, bw);
      const int xpos0 = (x0 << 6) - (y + 1) * dx;
      const int ba0 = xpos0 >> (6 - up_a);
      const int sha = ((xpos0 * (1 << up_a)) & 0x3f) >> 1;
#pragma unroll
      for (int x = 0; x < 8; x++) {
        if (x < x0) {
          const int ypos = (y << 6) - (x + 1) * dy;
          const int b = ypos >> (6 - up_l);
          const int sh = ((ypos * (1 << up_l)) & 0x3f) >> 1;
          out[x] = (int16_t)((l[b] * (32 - sh) + l[b + 1] * sh + 16) >> 5);
        } else {
          const int b = ba0 + (x - x0) * (1 << up_a);
          out[x] = (int16_t)((a[b] * (32 - sha) + a[b + 1] * sha + 16) >> 5);
        }
      }
    }
    return;
  }
  const int32_t* a = A;
  const int32_t* l = L;
  if (mode == MT_PAETH_PRED) {
#pragma unroll
    for (int x = 0; x < 8; x++) {
      const int32_t lv = l[y], tv = a[x], b = lv + tv - corner;
      const int32_t ld = abs(lv - b), td = abs(tv - b), cdd = abs(corner - b);
      out[x] = (int16_t)((ld <= td && ld <= cdd) ? lv : (td <= cdd ? tv : corner));
    }
  } else if (mode == MT_SMOOTH_PRED) {
    const int32_t right = a[bw - 1], bottom = l[bh - 1];
#pragma unroll
    for (int x = 0; x < 8; x++) {
      const int32_t wv = kSmW8[y], wh = kSmW8[x];
      const int32_t pp = wv * a[x] + (256 - wv) * bottom + wh * l[y] + (256 - wh) * right;
      out[x] = (int16_t)((pp + 256) >> 9);
    }
  } else if (mode == MT_SMOOTH_V_PRED) {
    const int32_t bottom = l[bh - 1];
#pragma unroll
    for (int x = 0; x < 8; x++) out[x] = (int16_t)((kSmW8[y] * a[x] + (256 - kSmW8[y]) * bottom + 128) >> 8);
  } else {  // SMOOTH_H
    const int32_t right = a[bw - 1];
#pragma unroll
    for (int x = 0; x < 8; x++) out[x] = (int16_t)((kSmW8[x] * l[y] + (256 - kSmW8[x]) * right + 128) >> 8);
  }
}

// Forward transform + quantisation (+ QM for the 2-D types) of src - pred
// into o.cf / o.tf: fwd8x8 and apply_qm split over the lanes.
__device__ __forceinline__ void coop8_fwd(const uint16_t* __restrict__ src, int stride, int px, int py,
                                          const int16_t* pred, int TX, const mt_quant& q, const float* qs,
                                          bool use_qm, Oct8& o, const Octet& g) {
  const int j = g.j;
#pragma unroll
  for (int x = 0; x < 8; x++)
    o.t[j * 8 + x] = (int32_t)src[(size_t)(py + j) * stride + px + x] - pred[j * 8 + x];
  if (TX == MT_TX_IDTX) {
#pragma unroll
    for (int x = 0; x < 8; x++) {
      const int rc = j + x * 8;
      const int32_t qd = rc == 0 ? q.dc_q : q.ac_q;
      const int32_t num = o.t[j * 8 + x] * 8;
      o.tf[rc] = __fdiv_rn((float)num, (float)qd);
      const int32_t am = (int32_t)uabs(num);
      const int32_t level = (am + qd / 2) / qd;
      o.cf[rc] = (int16_t)(am < qd ? 0 : (num < 0 ? -level : level));
    }
    g.sync();
    return;
  }
  if (TX == MT_TX_H_DCT) {  // rows: lane j transforms row j
    int32_t v[8];
#pragma unroll
    for (int x = 0; x < 8; x++) v[x] = o.t[j * 8 + x];
    fdct8(v);
#pragma unroll
    for (int x = 0; x < 8; x++) {
      const int rc = j + x * 8;
      int32_t lv;
      quant_fullstep(v[x] * 2, rc == 0 ? q.q_mult_dc : q.q_mult_ac, &lv, &o.tf[rc]);
      o.cf[rc] = (int16_t)lv;
    }
    g.sync();
    return;
  }
  g.sync();  // the column passes read other lanes' rows
  int32_t v[8];
#pragma unroll
  for (int r = 0; r < 8; r++) v[r] = o.t[r * 8 + j];
  if (TX == MT_TX_V_DCT) {  // columns only: lane j transforms column j
    fdct8(v);
#pragma unroll
    for (int y = 0; y < 8; y++) {
      const int rc = y + j * 8;
      int32_t lv;
      quant_fullstep(v[y] * 2, rc == 0 ? q.q_mult_dc : q.q_mult_ac, &lv, &o.tf[rc]);
      o.cf[rc] = (int16_t)lv;
    }
    g.sync();
    return;
  }
  if (coop_col_kind(TX) == 1) fdct8(v); else fadst8(v);
  g.sync();  // every lane has read its column before any is overwritten
#pragma unroll
  for (int r = 0; r < 8; r++) o.t[r * 8 + j] = v[r];
  g.sync();
#pragma unroll
  for (int u = 0; u < 8; u++) v[u] = o.t[j * 8 + u];
  if (coop_row_kind(TX) == 1) fdct8(v); else fadst8(v);
#pragma unroll
  for (int u = 0; u < 8; u++) {
    const int idx = u * 8 + j;
    const int32_t m = idx == 0 ? q.q_mult_dc : q.q_mult_ac;
    int32_t c = quant_q16(v[u], m);
    float tf = __fmul_rn(__fmul_rn((float)v[u], (float)m), 1.0f / 65536.0f);
    if (use_qm) {  // apply_qm
      const float xs = __fmul_rn(tf, qs[idx]);
      tf = xs;
      const float tr = truncf(xs);
      const float frac = fabsf(__fsub_rn(xs, tr));
      const float step = frac >= 0.5f ? copysignf(1.0f, xs) : 0.0f;
      c = (int32_t)__fadd_rn(tr, step);
    }
    o.cf[idx] = (int16_t)c;
    o.tf[idx] = tf;
  }
  g.sync();
}

// The last nonzero scan index of o.cf (-1 when all zero).
__device__ __forceinline__ int coop8_eob(const Oct8& o, const CoopTabs& tb, const Octet& g) {
  int e1 = 0;
#pragma unroll
  for (int y = 0; y < 8; y++) {
    const int rc = g.j * 8 + y;
    if (o.cf[rc] != 0) e1 = ::max(e1, (int)tb.iscan[rc] + 1);
  }
  return g.max(e1) - 1;
}

// trellis8 over the octet, lane j holding column j of the block (positions
// rc = 8j + y, y = 0..7, in registers).  Returns the final EOB scan index.
__device__ __forceinline__ int coop8_trellis(Oct8& o, float dc_q, float ac_q, float lambda, const float* lut,
                                             const CoopTabs& tb, const Octet& g) {
  const int j = g.j;
  const float dq2 = __fmul_rn(dc_q, dc_q), aq2 = __fmul_rn(ac_q, ac_q);
  int32_t c[8];
  float at[8];
  int e[8];
  int e1 = 0;
#pragma unroll
  for (int y = 0; y < 8; y++) {
    const int rc = j * 8 + y;
    c[y] = o.cf[rc];
    at[y] = fabsf(o.tf[rc]);
    e[y] = tb.iscan[rc];
    if (c[y] != 0) e1 = ::max(e1, e[y] + 1);
  }
  const int m = g.max(e1);
  if (m == 0) return -1;
  const int full8 = m & ~7;
  const bool has4 = (m - full8) >= 4;
  // step A.  The reference decides each position of a chunk from the chunk's
  // starting values, in the AVX2 FMA form unless the chunk holds a level
  // above 63 (then, and in the scalar tail, the plain form): positions are
  // independent given each chunk's flag (bits 0-7: the 8-wide chunks, bit 8:
  // the 4-wide one).
  unsigned bigb = 0;
#pragma unroll
  for (int y = 0; y < 8; y++) {
    if (uabs(c[y]) > 63u && e[y] < m) {
      if (e[y] < full8) bigb |= 1u << (e[y] >> 3);
      else if (has4 && e[y] < full8 + 4) bigb |= 1u << 8;
    }
  }
  const unsigned big = __reduce_or_sync(g.mask, bigb);
#pragma unroll
  for (int y = 0; y < 8; y++) {
    if (e[y] < m && c[y] != 0) {
      const float q2 = (j == 0 && y == 0) ? dq2 : aq2;
      const bool fma_form = e[y] < full8 ? !((big >> (e[y] >> 3)) & 1) : (has4 && e[y] < full8 + 4 && !((big >> 8) & 1));
      bool dn;
      if (fma_form) {
        const int32_t li = (int32_t)uabs(c[y]), ldi = ::max(li - 1, 0);
        const float el = __fsub_rn(at[y], (float)li), ed = __fsub_rn(at[y], (float)ldi);
        const float cl = __fmaf_rn(q2, __fmul_rn(el, el), __fmul_rn(lambda, lut[li]));
        const float cd = __fmaf_rn(q2, __fmul_rn(ed, ed), __fmul_rn(lambda, lut[ldi]));
        dn = cd < cl;
      } else {
        dn = round_down_plain(at[y], uabs(c[y]), q2, lambda);
      }
      if (dn) c[y] = c[y] < 0 ? c[y] + 1 : c[y] - 1;
    }
  }
  g.sync();  // every lane has read tf before R overwrites it
  // Terms of the two ordered float chains, by scan position e < m:
  //   S[e] = q2 * at^2 (the zeroing distortion; becomes the suffix sums),
  //   B[e] = q2 * (at - l)^2 (becomes the running prefix cost base_c),
  //   R[e] = lambda * rate(l).
  float* S = reinterpret_cast<float*>(o.t);
  float* B = o.x;
  float* R = o.tf;
#pragma unroll
  for (int y = 0; y < 8; y++) {
    if (e[y] < m) {
      const float q2 = (j == 0 && y == 0) ? dq2 : aq2;
      const uint32_t l = uabs(c[y]);
      S[e[y]] = __fmul_rn(q2, __fmul_rn(at[y], at[y]));
      const float ecur = __fsub_rn(at[y], (float)l);
      B[e[y]] = __fmul_rn(q2, __fmul_rn(ecur, ecur));
      R[e[y]] = __fmul_rn(lambda, l < 64 ? lut[l] : coef_rate_bits(l));
    }
  }
  g.sync();
  // Two ordered chains in one loop: lane 0 the suffix sums right to left
  // (acc += S[e]; S[e] = acc), lane 1 the prefix cost left to right
  // (base_c = pre + B[e]; B[e] = base_c; pre = base_c + R[e]).  Lane 0 adds
  // +0 in the second step, which leaves its non-negative sum unchanged.  The
  // terms are loaded eight at a time ahead of the ordered additions.
  if (j < 2) {
    if (j == 0) S[m] = 0.0f;
    float* arr = j == 0 ? S : B;
    float acc = 0.0f;
    int s = 0;
    for (; s + 8 <= m; s += 8) {
      float v[8], r[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int ee = j == 0 ? m - 1 - (s + u) : s + u;
        v[u] = arr[ee];
        r[u] = j == 0 ? 0.0f : R[ee];
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int ee = j == 0 ? m - 1 - (s + u) : s + u;
        const float x = __fadd_rn(acc, v[u]);
        arr[ee] = x;
        acc = __fadd_rn(x, r[u]);
      }
    }
    for (; s < m; s++) {
      const int ee = j == 0 ? m - 1 - s : s;
      const float x = __fadd_rn(acc, arr[ee]);
      arr[ee] = x;
      acc = __fadd_rn(x, j == 0 ? 0.0f : R[ee]);
    }
  }
  g.sync();
  // candidate ends: the lowest cost, the first position on ties
  float best = __int_as_float(0x7f800000);
  int best_e = 64;
#pragma unroll
  for (int y = 0; y < 8; y++) {
    if (e[y] < m && c[y] != 0) {
      const int ee = e[y];
      const int bin = ee < 2 ? ee : 32 - __clz(ee);
      const int extra = bin > 1 ? bin - 2 : 0;
      const float sig = __fadd_rn(__fmul_rn((float)bin, 0.9f), __fadd_rn((float)extra, 2.0f));
      const float cst = __fadd_rn(__fadd_rn(B[ee], __fmul_rn(lambda, sig)), S[ee + 1]);
      if (cst < best || (cst == best && ee < best_e)) {
        best = cst;
        best_e = ee;
      }
    }
  }
#pragma unroll
  for (int sh = 1; sh < 8; sh <<= 1) {
    const float ob = __shfl_xor_sync(g.mask, best, sh);
    const int oe = __shfl_xor_sync(g.mask, best_e, sh);
    if (ob < best || (ob == best && oe < best_e)) {
      best = ob;
      best_e = oe;
    }
  }
  const float skip = __fadd_rn(S[0], lambda);
  const int keep = (best_e == 64 || skip < best) ? 0 : best_e + 1;
#pragma unroll
  for (int y = 0; y < 8; y++) o.cf[j * 8 + y] = (int16_t)((e[y] >= keep && e[y] < m) ? 0 : c[y]);
  g.sync();
  return keep - 1;
}

// Dequantisation + inverse transform of o.cf into o.rr (inv8x8).
__device__ __forceinline__ void coop8_inv(int TX, const mt_quant& q, const uint8_t* qm, Oct8& o, const Octet& g) {
  const int j = g.j;
  const bool flat = TX == MT_TX_IDTX || TX == MT_TX_V_DCT || TX == MT_TX_H_DCT;
  const uint8_t* w = flat ? nullptr : qm;
  int32_t* t = o.t;
#pragma unroll
  for (int y = 0; y < 8; y++) {  // rc = j * 8 + y: column j of t
    const int rc = j * 8 + y;
    const int32_t l = o.cf[rc];
    const int32_t base = rc == 0 ? q.dc_q : q.ac_q;
    const int32_t step = w ? ((base * (int32_t)w[rc] + 16) >> 5) : base;
    int32_t mag = (int32_t)((uabs(l) * (uint32_t)step) & 0xffffffu);
    mag = ::min(mag, q.cf_max + (l < 0 ? 1 : 0));
    t[y * 8 + j] = l == 0 ? 0 : (l < 0 ? -mag : mag);
  }
  g.sync();
  const int ck = coop_col_kind(TX), rk = coop_row_kind(TX);
  int32_t* row = t + j * 8;
  if (rk == 0) {
#pragma unroll
    for (int x = 0; x < 8; x++) row[x] *= 2;
  } else if (rk == 1) {
    idct8s(row, 1, q.rmin, q.rmax);
  } else {
    iadst8s(row, 1, q.rmin, q.rmax);
  }
#pragma unroll
  for (int x = 0; x < 8; x++) row[x] = clampi((row[x] + 1) >> 1, q.cmin, q.cmax);
  g.sync();
  int32_t* col = t + j;
  if (ck == 0) {
#pragma unroll
    for (int y = 0; y < 8; y++) col[y * 8] *= 2;
  } else if (ck == 1) {
    idct8s(col, 8, q.cmin, q.cmax);
  } else {
    iadst8s(col, 8, q.cmin, q.cmax);
  }
#pragma unroll
  for (int y = 0; y < 8; y++) o.rr[y * 8 + j] = (int16_t)((col[y * 8] + 8) >> 4);
  g.sync();
}

// satd8 (no display mask): lanes 0..3 take one 4x4 Hadamard each.
__device__ __forceinline__ uint32_t coop8_satd(const uint16_t* __restrict__ src, int stride, int px, int py,
                                               const int16_t* pred, const Oct8& o, int32_t maxv, const Octet& g) {
  uint32_t satd = 0;
  if (g.j < 4) {
    const int ty = (g.j >> 1) * 4, tx = (g.j & 1) * 4;
    int32_t r[4][4];
#pragma unroll
    for (int y = 0; y < 4; y++) {
      int32_t d[4];
#pragma unroll
      for (int x = 0; x < 4; x++) {
        const int i = (ty + y) * 8 + tx + x;
        d[x] = (int32_t)src[(size_t)(py + ty + y) * stride + px + tx + x] - clampi(pred[i] + o.rr[i], 0, maxv);
      }
      const int32_t e = d[0] + d[2], f = d[0] - d[2], gg = d[1] + d[3], h = d[1] - d[3];
      r[y][0] = e + gg;
      r[y][1] = f + h;
      r[y][2] = f - h;
      r[y][3] = e - gg;
    }
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const int32_t e = r[0][x] + r[2][x], f = r[0][x] - r[2][x], gg = r[1][x] + r[3][x], h = r[1][x] - r[3][x];
      satd += uabs(e + gg) + uabs(f + h) + uabs(f - h) + uabs(e - gg);
    }
  }
  return g.sum(satd);
}

// rate8 over the octet, lane j holding column j.  The level map the
// reference fills as its reverse walk goes holds, at scan index i,
// level_byte(|level|) of exactly the positions of scan index > i (its
// neighbours are entered before it when they come later in the scan:
// CoopTabs::vmask), so every position's context is known from the final
// levels; the neighbours' level bytes come from the lanes of columns j + 1
// and j + 2.  The per-position terms go to shared memory and lane 0 adds them
// in the walk's order (base token, then the br cost, then the golomb cost; an
// absent term is +0, which leaves the positive sum unchanged).  Every lane
// returns the bits.
__device__ __forceinline__ float coop8_rate(Oct8& o, int eob, const mt_coef_costs& T, int skip_ctx, int dcs,
                                            int mode, int tx, bool use_skip_bits, float skip1, float skip0,
                                            const CoopTabs& tb, const Octet& g) {
  if (eob < 0) return use_skip_bits ? skip1 : T.txb_skip[skip_ctx][1];
  const int j = g.j;
  float* T1 = o.tf;
  float* T2 = o.x;
  float* T3 = reinterpret_cast<float*>(o.t);
  unsigned nz = 0;
  uint32_t m[8], lb[8], lb1[8], lb2[8];
#pragma unroll
  for (int y = 0; y < 8; y++) {
    m[y] = uabs(o.cf[j * 8 + y]);
    lb[y] = level_byte(m[y]);
  }
#pragma unroll
  for (int y = 0; y < 8; y++) {  // columns j + 1 and j + 2 (none past column 7)
    const uint32_t v1 = __shfl_down_sync(g.mask, lb[y], 1, 8), v2 = __shfl_down_sync(g.mask, lb[y], 2, 8);
    lb1[y] = j + 1 < 8 ? v1 : 0u;
    lb2[y] = j + 2 < 8 ? v2 : 0u;
  }
  if (eob > 0) {
#pragma unroll
    for (int y = 0; y < 8; y++) {
      const int rc = j * 8 + y;
      const int i = tb.iscan[rc];
      if (i >= 1 && i < eob) {
        const unsigned vm = tb.vmask[rc];
        // neighbours rc + 1, + 8, + 9, + 2, + 16 (rc + 1 and + 2 run on into the next column)
        const uint32_t n1 = y < 7 ? lb[y + 1] : lb1[0];
        const uint32_t n8 = lb1[y];
        const uint32_t n9 = y < 7 ? lb1[y + 1] : lb2[0];
        const uint32_t n2 = y < 6 ? lb[y + 2] : lb1[y - 6];
        const uint32_t n16 = lb2[y];
        const uint32_t hm = ((vm & 1) ? n1 : 0u) + ((vm & 2) ? n8 : 0u) + ((vm & 4) ? n9 : 0u);
        const uint32_t mag = hm + ((vm & 8) ? n2 : 0u) + ((vm & 16) ? n16 : 0u);
        const int ctx = tb.loctx[::min(y, 4) * 5 + ::min(j, 4)] + (mag > 512 ? 4 : (int)((mag + 64) >> 7));
        const uint32_t tok = ::min(m[y], 3u);
        T1[i] = T.base_tok[ctx][tok];
        float t2 = 0.0f, t3 = 0.0f;
        if (tok == 3) {
          const uint32_t hmag = hm & 63;
          const int bc = ((y | j) > 1 ? 14 : 7) + (hmag > 12 ? 6 : (int)((hmag + 1) >> 1));
          t2 = T.br_cum[bc][::min((int32_t)m[y] - 3, 12)];
          if (m[y] >= 15) t3 = golomb_cost(m[y] - 15);
        }
        T2[i] = t2;
        T3[i] = t3;
        nz += m[y] != 0;
      }
    }
    nz = g.sum(nz);
  }
  // the DC context's neighbours (0, 1), (1, 0), (1, 1): lane 0's column and lane 1's
  const uint32_t dcmag = (lb[1] + lb1[0] + lb1[1]) & 63;
  g.sync();
  float bits = 0.0f;
  if (j == 0) {
    bits = use_skip_bits ? skip0 : T.txb_skip[skip_ctx][0];
    bits = __fadd_rn(bits, T.txtp[mode][tx]);
    const float* dcs_c = T.dc_sign[dcs];
    if (eob == 0) {
      const uint32_t mm = ::min(m[0], 3u);
      bits = __fadd_rn(bits, T.eob_bin[0]);
      bits = __fadd_rn(bits, T.eob_base[0][mm - 1]);
      if (mm == 3) {
        float h = T.br_cum[0][::min((int32_t)m[0] - 3, 12)];
        if (m[0] >= 15) h = __fadd_rn(h, golomb_cost(m[0] - 15));
        bits = __fadd_rn(bits, h);
      }
      bits = __fadd_rn(bits, dcs_c[o.cf[0] < 0]);
    } else {
      const int eob_bin = eob < 2 ? eob : 32 - __clz(eob);
      bits = __fadd_rn(bits, T.eob_bin[eob_bin]);
      if (eob_bin > 1) {
        const int nb = eob_bin - 2;
        bits = __fadd_rn(bits, T.eob_hi[eob_bin][(eob >> nb) & 1]);
        bits = __fadd_rn(bits, (float)nb);
      }
      const int ctx_e = 1 + (eob > 8) + (eob > 16);
      {
        const int rc = tb.scan[eob];
        const int ex = rc >> 3, ey = rc & 7;
        const uint32_t me = uabs(o.cf[rc]);
        const uint32_t tok = ::min(me, 3u) - 1;
        bits = __fadd_rn(bits, T.eob_base[ctx_e][tok]);
        if (tok == 2) {
          float h = T.br_cum[(ex | ey) > 1 ? 14 : 7][::min((int32_t)me - 3, 12)];
          if (me >= 15) h = __fadd_rn(h, golomb_cost(me - 15));
          bits = __fadd_rn(bits, h);
        }
      }
      int i = eob - 1;
      for (; i >= 8; i -= 8) {  // loads ahead of the ordered additions
        float a[8], b2[8], c3[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          a[u] = T1[i - u];
          b2[u] = T2[i - u];
          c3[u] = T3[i - u];
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
          bits = __fadd_rn(bits, a[u]);
          bits = __fadd_rn(bits, b2[u]);
          bits = __fadd_rn(bits, c3[u]);
        }
      }
      for (; i >= 1; i--) {
        bits = __fadd_rn(bits, T1[i]);
        bits = __fadd_rn(bits, T2[i]);
        bits = __fadd_rn(bits, T3[i]);
      }
      const uint32_t dm = m[0], dtok = ::min(dm, 3u);
      bits = __fadd_rn(bits, T.base_tok[0][dtok]);
      if (dtok == 3) {
        float h = T.br_cum[dcmag > 12 ? 6 : (int)((dcmag + 1) >> 1)][::min((int32_t)dm - 3, 12)];
        if (dm >= 15) h = __fadd_rn(h, golomb_cost(dm - 15));
        bits = __fadd_rn(bits, h);
      }
      if (o.cf[0] != 0) bits = __fadd_rn(bits, dcs_c[o.cf[0] < 0]);
      const int ac_nz = 1 + (int)nz;
      for (int k = 0; k < ac_nz; k++) bits = __fadd_rn(bits, 1.0f);
    }
  }
  bits = __shfl_sync(g.mask, bits, threadIdx.x & 24);
  g.sync();
  return bits;
}

// chain8_tx<false> over the octet: from the prediction `pred` (shared,
// row-major) and the source block at (sx, sy) of src (row stride sstride: the
// plane, or the block staged in shared memory), leaves the levels in o.cf,
// the inverse residual in o.rr and the result in r (all lanes).
__device__ __forceinline__ void coop8_tx(const uint16_t* __restrict__ src, int sstride, int sx, int sy,
                                         const mt_chain_params& p, const mt_quant& q, float trellis_lambda,
                                         const uint8_t* qm, const float* qs,
                                         const float* lut, const mt_coef_costs& T, const mt_candidate& cd,
                                         const int16_t* pred, mt_candidate_result& r, Oct8& o, const CoopTabs& tb,
                                         const Octet& g) {
  const int32_t maxv = (1 << p.bd) - 1;
  const int TX = cd.tx_type;
  const bool two_d = TX == MT_TX_DCT_DCT || TX >= MT_TX_ADST_ADST;
  coop8_fwd(src, sstride, sx, sy, pred, TX, q, qs, two_d && qm, o, g);
  int eob;
  if (p.trellis_lambda0 > 0.0f && !(cd.flags & MT_CAND_NO_TRELLIS))
    eob = coop8_trellis(o, (float)q.dc_q, (float)q.ac_q, trellis_lambda, lut, tb, g);
  else
    eob = coop8_eob(o, tb, g);
  coop8_inv(TX, q, qm, o, g);
  const uint32_t satd = coop8_satd(src, sstride, sx, sy, pred, o, maxv, g);
  const float qstep = (float)q.ac_q;
  float price = __fmul_rn(__fmul_rn(__fmul_rn((float)satd, fmaxf(qstep, 1.0f)), 0.25f), p.satd_scale);
  if (p.satd_bridge != 0.0f) price = __fmul_rn(price, p.satd_bridge);
  const float cbits = coop8_rate(o, eob, T, cd.skip_ctx, cd.dcs_ctx, cd.mode, TX, p.use_skip_bits != 0,
                                 p.skip_bits[0], p.skip_bits[1], tb, g);
  const float bits = __fadd_rn(__fadd_rn(cbits, cd.mode_bits), cd.extra_bits);
  r.distortion = price;
  r.bits = bits;
  r.cost = __fadd_rn(price, __fmul_rn(p.mode_lambda, bits));
  r.satd = satd;
  r.eob = eob;
  r.reserved[0] = r.reserved[1] = r.reserved[2] = 0;
}

}  // namespace mtd
