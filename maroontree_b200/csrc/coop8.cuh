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
  __device__ __forceinline__ void load(int t, int nthreads) {
    for (int i = t; i < 64; i += nthreads) {
      scan[i] = kScan8[i];
      iscan[i] = kIScan8[i];
      if (i < 25) loctx[i] = kLoCtxOff[i];
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
  for (int k = 0; k < 8; k++)
    if (o.cf[tb.scan[k * 8 + g.j]] != 0) e1 = k * 8 + g.j + 1;
  return g.max(e1) - 1;
}

// trellis8 over the octet.  Returns the final EOB scan index.
__device__ __forceinline__ int coop8_trellis(Oct8& o, float dc_q, float ac_q, float lambda, const float* lut,
                                             const CoopTabs& tb, const Octet& g) {
  const int j = g.j;
  const float dq2 = __fmul_rn(dc_q, dc_q), aq2 = __fmul_rn(ac_q, ac_q);
  const int m = coop8_eob(o, tb, g) + 1;
  if (m == 0) return -1;
  const int full8 = m & ~7;
  const bool has4 = (m - full8) >= 4;
  // step A: lane j decides scan position 8k + j of chunk k
  for (int base = 0; base < m; base += 8) {
    const int e = base + j;
    const int rc = tb.scan[e];
    const int32_t c = o.cf[rc];
    const float at = fabsf(o.tf[rc]);
    const bool in_chunk = base < full8 || (has4 && j < 4);  // an 8-wide or the 4-wide chunk
    const bool big = g.any(in_chunk && uabs(c) > 63u);
    bool dn = false;
    if (e < m && c != 0) {
      const float q2 = rc == 0 ? dq2 : aq2;
      if (in_chunk && !big) {
        const int32_t li = (int32_t)uabs(c), ldi = ::max(li - 1, 0);
        const float el = __fsub_rn(at, (float)li), ed = __fsub_rn(at, (float)ldi);
        const float cl = __fmaf_rn(q2, __fmul_rn(el, el), __fmul_rn(lambda, lut[li]));
        const float cd = __fmaf_rn(q2, __fmul_rn(ed, ed), __fmul_rn(lambda, lut[ldi]));
        dn = cd < cl;
      } else {
        dn = round_down_plain(at, uabs(c), q2, lambda);
      }
    }
    if (dn) o.cf[rc] = (int16_t)(c < 0 ? c + 1 : c - 1);
  }
  g.sync();
  // Terms of the two ordered float chains, by scan position e < m:
  //   S[e] = q2 * at^2 (the zeroing distortion; becomes the suffix sums),
  //   B[e] = q2 * (at - l)^2 (becomes the running prefix cost base_c),
  //   R[e] = lambda * rate(l).
  float* S = reinterpret_cast<float*>(o.t);
  float* B = o.x;
  float* R = o.tf;
  float at_k[8];
  uint32_t l_k[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int e = k * 8 + j;
    const int rc = tb.scan[e];
    at_k[k] = fabsf(o.tf[rc]);
    l_k[k] = uabs(o.cf[rc]);
  }
  g.sync();  // tf is overwritten by R below
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int e = k * 8 + j;
    if (e < m) {
      const float q2 = tb.scan[e] == 0 ? dq2 : aq2;
      S[e] = __fmul_rn(q2, __fmul_rn(at_k[k], at_k[k]));
      const float ecur = __fsub_rn(at_k[k], (float)l_k[k]);
      B[e] = __fmul_rn(q2, __fmul_rn(ecur, ecur));
      R[e] = __fmul_rn(lambda, l_k[k] < 64 ? lut[l_k[k]] : coef_rate_bits(l_k[k]));
    }
  }
  g.sync();
  // Two ordered chains in one loop: lane 0 the suffix sums right to left
  // (acc += S[e]; S[e] = acc), lane 1 the prefix cost left to right
  // (base_c = pre + B[e]; B[e] = base_c; pre = base_c + R[e]).  Lane 0 adds
  // +0 in the second step, which leaves its non-negative sum unchanged.
  if (j < 2) {
    if (j == 0) S[m] = 0.0f;
    float* arr = j == 0 ? S : B;
    float acc = 0.0f;
    for (int s = 0; s < m; s++) {
      const int e = j == 0 ? m - 1 - s : s;
      const float r = __fadd_rn(acc, arr[e]);
      arr[e] = r;
      acc = __fadd_rn(r, j == 0 ? 0.0f : R[e]);
    }
  }
  g.sync();
  // candidate ends: the lowest cost, the first position on ties
  float best = __int_as_float(0x7f800000);
  int best_e = 64;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int e = k * 8 + j;
    if (e < m && l_k[k] != 0) {
      const int bin = e < 2 ? e : 32 - __clz(e);
      const int extra = bin > 1 ? bin - 2 : 0;
      const float sig = __fadd_rn(__fmul_rn((float)bin, 0.9f), __fadd_rn((float)extra, 2.0f));
      const float c = __fadd_rn(__fadd_rn(B[e], __fmul_rn(lambda, sig)), S[e + 1]);
      if (c < best) {
        best = c;
        best_e = e;
      }
    }
  }
#pragma unroll
  for (int s = 1; s < 8; s <<= 1) {
    const float ob = __shfl_xor_sync(g.mask, best, s);
    const int oe = __shfl_xor_sync(g.mask, best_e, s);
    if (ob < best || (ob == best && oe < best_e)) {
      best = ob;
      best_e = oe;
    }
  }
  const float skip = __fadd_rn(S[0], lambda);
  const int keep = (best_e == 64 || skip < best) ? 0 : best_e + 1;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int e = k * 8 + j;
    if (e >= keep && e < m) o.cf[tb.scan[e]] = 0;
  }
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

// rate8 over the octet.  The level map the reference fills as its reverse
// walk goes holds, at scan index i, level_byte(|level|) of exactly the
// positions of scan index > i, so every position's context is known from the
// final levels; the per-position terms go to shared memory and lane 0 adds
// them in the walk's order (base token, then the br cost, then the golomb
// cost; an absent term is +0, which leaves the positive sum unchanged).
// Every lane returns the bits.
__device__ __forceinline__ float coop8_rate(Oct8& o, int eob, const mt_coef_costs& T, int skip_ctx, int dcs,
                                            int mode, int tx, bool use_skip_bits, float skip1, float skip0,
                                            const CoopTabs& tb, const Octet& g) {
  if (eob < 0) return use_skip_bits ? skip1 : T.txb_skip[skip_ctx][1];
  const int j = g.j;
  float* T1 = o.tf;
  float* T2 = o.x;
  float* T3 = reinterpret_cast<float*>(o.t);
  unsigned nz = 0;
  if (eob > 0) {
    auto lvb = [&](int p, int i) -> uint32_t {
      return (p < 64 && (int)tb.iscan[p] > i) ? level_byte(uabs(o.cf[p])) : 0u;
    };
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int i = k * 8 + j;
      if (i >= 1 && i < eob) {
        const int rc = tb.scan[i];
        const int x = rc >> 3, y = rc & 7;
        const uint32_t hm = lvb(rc + 1, i) + lvb(rc + 8, i) + lvb(rc + 9, i);
        const uint32_t mag = hm + lvb(rc + 2, i) + lvb(rc + 16, i);
        const int ctx = tb.loctx[::min(y, 4) * 5 + ::min(x, 4)] + (mag > 512 ? 4 : (int)((mag + 64) >> 7));
        const uint32_t m = uabs(o.cf[rc]);
        const uint32_t tok = ::min(m, 3u);
        T1[i] = T.base_tok[ctx][tok];
        float t2 = 0.0f, t3 = 0.0f;
        if (tok == 3) {
          const uint32_t hmag = hm & 63;
          const int bc = ((y | x) > 1 ? 14 : 7) + (hmag > 12 ? 6 : (int)((hmag + 1) >> 1));
          t2 = T.br_cum[bc][::min((int32_t)m - 3, 12)];
          if (m >= 15) t3 = golomb_cost(m - 15);
        }
        T2[i] = t2;
        T3[i] = t3;
        nz += m != 0;
      }
    }
    nz = g.sum(nz);
  }
  g.sync();
  float bits = 0.0f;
  if (j == 0) {
    bits = use_skip_bits ? skip0 : T.txb_skip[skip_ctx][0];
    bits = __fadd_rn(bits, T.txtp[mode][tx]);
    const float* dcs_c = T.dc_sign[dcs];
    if (eob == 0) {
      const uint32_t m = uabs(o.cf[0]), mm = ::min(m, 3u);
      bits = __fadd_rn(bits, T.eob_bin[0]);
      bits = __fadd_rn(bits, T.eob_base[0][mm - 1]);
      if (mm == 3) {
        float h = T.br_cum[0][::min((int32_t)m - 3, 12)];
        if (m >= 15) h = __fadd_rn(h, golomb_cost(m - 15));
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
        const uint32_t m = uabs(o.cf[rc]);
        const uint32_t tok = ::min(m, 3u) - 1;
        bits = __fadd_rn(bits, T.eob_base[ctx_e][tok]);
        if (tok == 2) {
          float h = T.br_cum[(ex | ey) > 1 ? 14 : 7][::min((int32_t)m - 3, 12)];
          if (m >= 15) h = __fadd_rn(h, golomb_cost(m - 15));
          bits = __fadd_rn(bits, h);
        }
      }
      int i = eob - 1;
      for (; i >= 4; i -= 4) {  // loads ahead of the ordered additions
        float a[4], b2[4], c3[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          a[u] = T1[i - u];
          b2[u] = T2[i - u];
          c3[u] = T3[i - u];
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
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
      const uint32_t dm = uabs(o.cf[0]), dtok = ::min(dm, 3u);
      bits = __fadd_rn(bits, T.base_tok[0][dtok]);
      if (dtok == 3) {
        const uint32_t mag = (level_byte(uabs(o.cf[1])) + level_byte(uabs(o.cf[8])) + level_byte(uabs(o.cf[9]))) & 63;
        float h = T.br_cum[mag > 12 ? 6 : (int)((mag + 1) >> 1)][::min((int32_t)dm - 3, 12)];
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
