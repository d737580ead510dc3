// Device pieces of the luma leaf search at TX_8X8 that the proxy chain does
// not use: trellis_optimize_ctx (src/trellis.rs:55-942) with the real
// decision-CDF costs, the bounded 2-D coefficient rate walk
// (real_block_bits_bounded, src/rate.rs:149-291) in any txb_skip / dc_sign
// context, the 1-D V_DCT / H_DCT walk (luma_bits_1d_8x8,
// src/coder/lossy_state.rs:876-1008) and the coefficient result context
// (coef_res_ctx, src/coder/lossy_state.rs:630-648).
//
// One thread runs one block; every float operation is one IEEE rounding in
// the reference's order (the file is compiled with -fmad=false).  Costs come
// from the host-built mt_coef_costs: each entry is the reference's
// cdf_cost_with_table of the same symbol, br_cum the base-range ladder of
// src/cost.rs:214-241 (equal term for term to hi_tok_cost_with_table).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "chain4.cuh"
#include "chain8.cuh"
#include "chain16.cuh"

namespace mtd {

// Base-range ladder + Golomb tail of magnitude m >= 3 in br context bc
// (src/cost.rs:244-262 hi_tok_cost_with_table).
__device__ __forceinline__ float hi_cost(const mt_coef_costs& T, uint32_t m, int bc) {
  float h = T.br_cum[bc][min((int32_t)m - 3, 12)];
  if (m >= 15) h = __fadd_rn(h, golomb_cost(m - 15));
  return h;
}

__constant__ uint16_t kScan32[1024] = {MT_SCAN_32X32_LIST};
// The 32x32 default scan as trellis_sq's accessor.
struct Scan32 {
  __device__ __forceinline__ int operator()(int i) const { return kScan32[i]; }
};

// Default scan of a W x W block (scan index -> rc = x*W + y).
template <int W>
__device__ __forceinline__ int scan_rc(int i) {
  return W == 4 ? kScan4[i] : (W == 8 ? kScan8[i] : (W == 16 ? kScan16[i] : kScan32[i]));
}

// log2 of a block side 4 .. 32.
template <int W>
__host__ __device__ constexpr int log2w() {
  return W == 4 ? 2 : (W == 8 ? 3 : (W == 16 ? 4 : 5));
}

// Scratch of trellis_ctx<W>: the zero-distortion suffix sums and the level map
// (stride W with the reference's two zero columns of padding).
template <int W>
struct TrellisCtxScratchW {
  float suf0[W * W + 1];
  uint8_t lv[(W + 2) * W];
};
using TrellisCtxScratch = TrellisCtxScratchW<8>;

// trellis_optimize_ctx of one TX_WxW luma block (W = 8: class 1, 16: class 2,
// 32: class 3; plane 0; the cost slice of that class) under the
// shipped tuning: trellis_aom / eob_reprice / eob_zero_term / pad_stride off,
// dead zone 0, the DC-only terminal in eob_base context 0 with br context 0,
// skip priced at trellis_zero_bits = 1, tilt magnitude cap 2.  `lambda` is
// scaled_trellis_lambda (src/trellis.rs:50-53); qm (NULL = flat) the inverse
// QM row, weighted w/32 and squared from QM level 5 (qm_full).
template <int W, typename C>
__device__ void trellis_ctx(C* __restrict__ cf, const float* __restrict__ tf, float dc_q, float ac_q, float lambda,
                            const mt_coef_costs& T, int dcs, const uint8_t* __restrict__ qm, bool qm_full,
                            float band_t, TrellisCtxScratchW<W>& s) {
  constexpr int N = W * W, L = log2w<W>();
  constexpr float kCap = 2.0f, kNInv = 1.0f / (float)N;
  int eob = -1;
  for (int i = N - 1; i >= 0; i--)
    if (cf[scan_rc<W>(i)] != 0) {
      eob = i;
      break;
    }
  if (eob < 0) return;
  const float dq2_dc = __fmul_rn(dc_q, dc_q), dq2_ac = __fmul_rn(ac_q, ac_q);
  auto qm_at = [&](int rc) -> float {
    const float wq = __fdiv_rn((float)qm[rc], 32.0f);
    return qm_full ? __fmul_rn(wq, wq) : wq;
  };
  // trellis_dist_one (src/trellis_dist.rs:100-105) with the QM weight and the
  // band tilt as a division (the `distw` closure, src/trellis.rs:120-129).
  auto distw = [&](int idx, int rc, uint32_t lev) -> float {
    const float at = fabsf(tf[rc]);
    const float e = __fsub_rn(at, (float)lev);
    float d = __fmul_rn(rc == 0 ? dq2_dc : dq2_ac, __fmul_rn(e, e));
    if (qm) d = __fmul_rn(d, qm_at(rc));
    if (band_t != 0.0f && at < kCap) d = __fdiv_rn(d, __fadd_rn(1.0f, __fmul_rn(band_t, __fmul_rn((float)idx, kNInv))));
    return d;
  };
  uint8_t* lv = s.lv;
#pragma unroll 4
  for (int i = 0; i < (W + 2) * W / 4; i++) reinterpret_cast<uint32_t*>(lv)[i] = 0;
  for (int i = 0; i <= eob; i++) {
    const int rc = scan_rc<W>(i);
    lv[rc] = (uint8_t)level_byte(uabs(cf[rc]));
  }
  auto interior_ctx = [&](int rc, int& bc) -> int {
    const int x = rc >> L, y = rc & (W - 1);
    const uint32_t hm = (uint32_t)lv[rc + 1] + lv[rc + W] + lv[rc + W + 1];
    const uint32_t mag = hm + lv[rc + 2] + lv[rc + 2 * W];
    const uint32_t hm6 = hm & 63;
    bc = ((y | x) > 1 ? 14 : 7) + (hm6 > 12 ? 6 : (int)((hm6 + 1) >> 1));
    return kLoCtxOff[min(y, 4) * 5 + min(x, 4)] + (mag > 512 ? 4 : (int)((mag + 64) >> 7));
  };
  auto dc_brc = [&]() -> int {
    const uint32_t mag = ((uint32_t)lv[1] + lv[W] + lv[W + 1]) & 63;
    return mag > 12 ? 6 : (int)((mag + 1) >> 1);
  };

  // Step A (src/trellis.rs:514-602): reverse-scan RD-best level per interior
  // coefficient below the last nonzero, then DC.
  for (int i = eob - 1; i >= 1; i--) {
    const int rc = scan_rc<W>(i);
    const uint32_t l = uabs(cf[rc]);
    if (l == 0) continue;
    int bc;
    const int ctx = interior_ctx(rc, bc);
    const float* bt = T.base_tok[ctx];
    auto rate_k = [&](uint32_t k) -> float {
      if (k == 0) return bt[0];
      if (k < 3) return __fadd_rn(bt[k], 1.0f);
      return __fadd_rn(__fadd_rn(bt[3], hi_cost(T, k, bc)), 1.0f);
    };
    uint32_t best_k = l;
    float best_c = __fadd_rn(distw(i, rc, l), __fmul_rn(lambda, rate_k(l)));
    for (int32_t k = (int32_t)l - 1; k >= 0; k--) {
      const float dk = distw(i, rc, (uint32_t)k);
      if (dk >= best_c) break;
      const float c = __fadd_rn(dk, __fmul_rn(lambda, rate_k((uint32_t)k)));
      if (c < best_c) {
        best_c = c;
        best_k = (uint32_t)k;
      }
    }
    if (best_k != l) {
      cf[rc] = (C)(cf[rc] < 0 ? -(int32_t)best_k : (int32_t)best_k);
      lv[rc] = (uint8_t)level_byte(best_k);
    }
  }
  {
    const uint32_t l = uabs(cf[0]);
    if (l != 0) {
      const int bc = dc_brc();
      const float sgn_bits = T.dc_sign[dcs][cf[0] < 0];
      auto dc_rate = [&](uint32_t k) -> float {
        if (k == 0) return T.base_tok[0][0];
        float b = T.base_tok[0][min(k, 3u)];
        if (k >= 3) b = __fadd_rn(b, hi_cost(T, k, bc));
        return __fadd_rn(b, sgn_bits);
      };
      uint32_t best_k = l;
      float best_c = __fadd_rn(distw(0, 0, l), __fmul_rn(lambda, dc_rate(l)));
      for (int32_t k = (int32_t)l - 1; k >= 0; k--) {
        const float dk = distw(0, 0, (uint32_t)k);
        if (dk >= best_c) break;
        const float c = __fadd_rn(dk, __fmul_rn(lambda, dc_rate((uint32_t)k)));
        if (c < best_c) {
          best_c = c;
          best_k = (uint32_t)k;
        }
      }
      if (best_k != l) {
        cf[0] = (C)(cf[0] < 0 ? -(int32_t)best_k : (int32_t)best_k);
        lv[0] = (uint8_t)level_byte(best_k);
      }
    }
  }

  // Step B (src/trellis.rs:604-941).  The distortions in scan order
  // (trellis_dist_current_zero_scan, src/trellis_dist.rs:178-196), weighted by
  // the QM and multiplied by the reciprocal tilt factor.
  const int m = eob + 1;
  auto dist_pair = [&](int i, float& cur, float& zero) {
    const int rc = scan_rc<W>(i);
    const float dq2 = rc == 0 ? dq2_dc : dq2_ac;
    const float at = fabsf(tf[rc]);
    const float e = __fsub_rn(at, (float)uabs(cf[rc]));
    cur = __fmul_rn(dq2, __fmul_rn(e, e));
    zero = __fmul_rn(dq2, __fmul_rn(at, at));
    if (qm) {
      const float w2 = qm_at(rc);
      cur = __fmul_rn(cur, w2);
      zero = __fmul_rn(zero, w2);
    }
    if (band_t != 0.0f && at < kCap) {
      const float wgt = __fdiv_rn(1.0f, __fadd_rn(1.0f, __fmul_rn(band_t, __fmul_rn((float)i, kNInv))));
      zero = __fmul_rn(zero, wgt);
      cur = __fmul_rn(cur, wgt);
    }
  };
  float* suf0 = s.suf0;
  suf0[m] = 0.0f;
  float dist_zero0, dist_cur0;
  {
    float sacc = 0.0f;
    for (int i = m - 1; i >= 1; i--) {
      float cur, zero;
      dist_pair(i, cur, zero);
      sacc = __fadd_rn(sacc, zero);
      suf0[i] = sacc;
    }
    dist_pair(0, dist_cur0, dist_zero0);
  }
  const uint32_t dc_m = uabs(cf[0]);
  int best_e = -1;
  uint32_t best_m = 0;
  float best_cost = __int_as_float(0x7f800000);
  auto eob_coeff_cost = [&](int e, uint32_t k) -> float {
    const int ctx_e = 1 + (e > (N >> 3)) + (e > (N >> 2));
    const uint32_t tok = min(k, 3u);
    float c = T.eob_base[ctx_e][tok - 1];
    if (tok == 3) {
      const int rc = scan_rc<W>(e);
      c = __fadd_rn(c, hi_cost(T, k, ((rc >> L) | (rc & (W - 1))) > 1 ? 14 : 7));
    }
    return __fadd_rn(c, 1.0f);
  };
  auto eob_pt_cost = [&](int e) -> float {
    const int bin = e < 2 ? e : 32 - __clz(e);
    float c = T.eob_bin[bin];
    if (bin > 1) {
      const int nb = bin - 2;
      c = __fadd_rn(c, T.eob_hi[bin][(e >> nb) & 1]);
      c = __fadd_rn(c, (float)nb);
    }
    return c;
  };
  auto eob_cand = [&](int e, uint32_t k) -> float {
    return __fadd_rn(__fmul_rn(lambda, eob_coeff_cost(e, k)), distw(e, scan_rc<W>(e), k));
  };
  {
    float dc_cost;
    if (dc_m == 0) {
      dc_cost = __fmul_rn(lambda, T.base_tok[0][0]);
    } else {
      const int bc = dc_brc();
      float b = T.base_tok[0][min(dc_m, 3u)];
      if (dc_m >= 3) b = __fadd_rn(b, hi_cost(T, dc_m, bc));
      b = __fadd_rn(b, T.dc_sign[dcs][cf[0] < 0]);
      dc_cost = __fmul_rn(lambda, b);
    }
    dc_cost = __fadd_rn(dc_cost, dist_cur0);
    // pre[e], the rate + distortion of interior positions 1 .. e-1, as a
    // running sum in the reference's order (src/trellis.rs:849-868).
    float acc = 0.0f;
    for (int e = 1; e < m; e++) {
      const int rc = scan_rc<W>(e);
      const uint32_t k = uabs(cf[rc]);
      if (k != 0) {
        const float base =
            __fadd_rn(__fadd_rn(__fadd_rn(dc_cost, acc), __fmul_rn(lambda, eob_pt_cost(e))), suf0[e + 1]);
        uint32_t m_best = k;
        float c = __fadd_rn(base, eob_cand(e, k));
        if (k >= 2) {
          const float c_low = __fadd_rn(base, eob_cand(e, k - 1));
          if (c_low < c) {
            c = c_low;
            m_best = k - 1;
          }
        }
        if (c < best_cost) {
          best_cost = c;
          best_e = e;
          best_m = m_best;
        }
      }
      int bc;
      const int ctx = interior_ctx(rc, bc);
      float r;
      if (k == 0) {
        r = T.base_tok[ctx][0];
      } else {
        r = T.base_tok[ctx][min(k, 3u)];
        if (k >= 3) r = __fadd_rn(r, hi_cost(T, k, bc));
        r = __fadd_rn(r, 1.0f);
      }
      float cur, zero;
      dist_pair(e, cur, zero);
      acc = __fadd_rn(acc, __fadd_rn(__fmul_rn(lambda, r), cur));
    }
  }
  if (dc_m != 0) {
    float c0 = __fadd_rn(T.eob_bin[0], T.eob_base[0][min(dc_m, 3u) - 1]);
    if (dc_m >= 3) c0 = __fadd_rn(c0, hi_cost(T, dc_m, 0));
    const float r = __fadd_rn(c0, T.dc_sign[dcs][cf[0] < 0]);
    const float total0 = __fadd_rn(__fadd_rn(__fmul_rn(lambda, r), dist_cur0), suf0[1]);
    if (total0 < best_cost) {
      best_cost = total0;
      best_e = 0;
      best_m = dc_m;
    }
  }
  const float skip_cost = __fadd_rn(__fadd_rn(suf0[1], dist_zero0), __fmul_rn(lambda, 1.0f));
  if (best_e < 0 || skip_cost < best_cost) {
    for (int i = 0; i < m; i++) cf[scan_rc<W>(i)] = 0;
  } else {
    const int rc = scan_rc<W>(best_e);
    if (best_m != uabs(cf[rc])) {
      const bool neg = cf[rc] != 0 ? cf[rc] < 0 : tf[rc] < 0.0f;
      cf[rc] = (C)(neg ? -(int32_t)best_m : (int32_t)best_m);
    }
    for (int i = best_e + 1; i < m; i++) cf[scan_rc<W>(i)] = 0;
  }
}

template <typename C>
__device__ __forceinline__ void trellis_ctx8(C* __restrict__ cf, const float* __restrict__ tf, float dc_q, float ac_q,
                                             float lambda, const mt_coef_costs& T, int dcs,
                                             const uint8_t* __restrict__ qm, bool qm_full, float band_t,
                                             TrellisCtxScratch& s) {
  trellis_ctx<8>(cf, tf, dc_q, ac_q, lambda, T, dcs, qm, qm_full, band_t, s);
}

// real_block_bits_bounded of a TX_WxW luma block (W = 4, 8, 16, 32: classes
// TX_4X4 .. TX_32X32) in txb_skip context skip_ctx and dc_sign context dcs
// with the tx-type symbol of (mode, tx) (tx < 0: none, the DCT-only TX_32X32
// set): +inf once the running sum passes `bound` after the eob position or at
// an interior scan index divisible by 16.  lv: (W + 2) * W bytes of scratch
// (the level map, stride W).
template <int W, typename C>
__device__ float rate_bounded(const C* __restrict__ cf, const mt_coef_costs& T, int skip_ctx, int dcs, int mode,
                               int tx, bool use_skip_bits, float skip1, float skip0, float bound,
                               uint8_t* __restrict__ lv) {
  const float kInf = __int_as_float(0x7f800000);
  int eob = -1;
  for (int i = W * W - 1; i >= 0; i--)
    if (cf[scan_rc<W>(i)] != 0) {
      eob = i;
      break;
    }
  if (eob < 0) return use_skip_bits ? skip1 : T.txb_skip[skip_ctx][1];
  float bits = use_skip_bits ? skip0 : T.txb_skip[skip_ctx][0];
  if (tx >= 0) bits = __fadd_rn(bits, T.txtp[mode][tx]);
  const float* dcs_c = T.dc_sign[dcs];
  if (eob == 0) {
    const uint32_t m = uabs(cf[0]);
    bits = __fadd_rn(bits, T.eob_bin[0]);
    bits = __fadd_rn(bits, T.eob_base[0][min(m, 3u) - 1]);
    if (m >= 3) bits = __fadd_rn(bits, hi_cost(T, m, 0));
    return __fadd_rn(bits, dcs_c[cf[0] < 0]);
  }
  const int eob_bin = eob < 2 ? eob : 32 - __clz(eob);
  bits = __fadd_rn(bits, T.eob_bin[eob_bin]);
  if (eob_bin > 1) {
    const int nb = eob_bin - 2;
    bits = __fadd_rn(bits, T.eob_hi[eob_bin][(eob >> nb) & 1]);
    bits = __fadd_rn(bits, (float)nb);
  }
  if (bits > bound) return kInf;
  uint32_t* lv32 = reinterpret_cast<uint32_t*>(lv);
#pragma unroll
  for (int i = 0; i < (W + 2) * W / 4; i++) lv32[i] = 0;
  constexpr int L = log2w<W>();
  const int ctx_e = 1 + (eob > (W * W >> 3)) + (eob > (W * W >> 2));
  {
    const int rc = scan_rc<W>(eob);
    const uint32_t m = uabs(cf[rc]);
    bits = __fadd_rn(bits, T.eob_base[ctx_e][min(m, 3u) - 1]);
    if (m >= 3) bits = __fadd_rn(bits, hi_cost(T, m, ((rc >> L) | (rc & (W - 1))) > 1 ? 14 : 7));
    lv[rc] = (uint8_t)level_byte(m);
  }
  int ac_nz = 1;
  for (int i = eob - 1; i >= 1; i--) {
    if ((i & 15) == 0 && bits > bound) return kInf;
    const int rc = scan_rc<W>(i);
    const int x = rc >> L, y = rc & (W - 1);
    const uint32_t hm = (uint32_t)lv[rc + 1] + lv[rc + W] + lv[rc + W + 1];
    const uint32_t mag = hm + lv[rc + 2] + lv[rc + 2 * W];
    const int ctx = kLoCtxOff[min(y, 4) * 5 + min(x, 4)] + (mag > 512 ? 4 : (int)((mag + 64) >> 7));
    const uint32_t m = uabs(cf[rc]);
    const uint32_t tok = min(m, 3u);
    bits = __fadd_rn(bits, T.base_tok[ctx][tok]);
    if (tok == 3) {
      const uint32_t hmag = hm & 63;
      const int bc = ((y | x) > 1 ? 14 : 7) + (hmag > 12 ? 6 : (int)((hmag + 1) >> 1));
      bits = __fadd_rn(bits, T.br_cum[bc][min((int32_t)m - 3, 12)]);
      if (m >= 15) bits = __fadd_rn(bits, golomb_cost(m - 15));
    }
    if (m != 0) {
      lv[rc] = (uint8_t)level_byte(m);
      ac_nz++;
    }
  }
  const uint32_t dm = uabs(cf[0]);
  bits = __fadd_rn(bits, T.base_tok[0][min(dm, 3u)]);
  if (dm >= 3) {
    const uint32_t mag = ((uint32_t)lv[1] + lv[W] + lv[W + 1]) & 63;
    bits = __fadd_rn(bits, hi_cost(T, dm, mag > 12 ? 6 : (int)((mag + 1) >> 1)));
  }
  if (cf[0] != 0) bits = __fadd_rn(bits, dcs_c[cf[0] < 0]);
  for (int k = 0; k < ac_nz; k++) bits = __fadd_rn(bits, 1.0f);
  return bits;
}

// luma_bits_1d_8x8 / luma_bits_1d_4x4 (src/coder/lossy_state.rs:876-1143):
// the V_DCT (vertical) / H_DCT coefficient rate of a W x W block -- txb_skip
// context 0, tx-type symbol 2 / 3, the 1-D eob_pt CDF, the 1-D base contexts
// (offset 26 + 0 / 5 / 10 by row) over (x, y) = (i % W, i / W) of the scan
// index, eob-coefficient context thresholds W*W/8 and W*W/4, sign bits in
// place.  lv: 160 bytes of scratch (10 columns of 16).
template <int W, typename C>
__device__ float rate_1d(const C* __restrict__ cf, bool vertical, const mt_coef_costs& T, int dcs, int mode,
                          uint8_t* __restrict__ lv) {
  constexpr int L = log2w<W>();
  auto pos_rc = [&](int i) -> int { return vertical ? ((i & (W - 1)) << L) | (i >> L) : i; };
  int eob = -1;
  for (int i = W * W - 1; i >= 0; i--)
    if (cf[pos_rc(i)] != 0) {
      eob = i;
      break;
    }
  if (eob < 0) return T.txb_skip[0][1];
  float bits = __fadd_rn(T.txb_skip[0][0], T.txtp[mode][vertical ? MT_TX_V_DCT : MT_TX_H_DCT]);
  if (eob == 0) {
    const uint32_t dm = uabs(cf[0]);
    bits = __fadd_rn(bits, T.eob_bin_1d[0]);
    bits = __fadd_rn(bits, T.eob_base[0][min(dm, 3u) - 1]);
    if (dm >= 3) bits = __fadd_rn(bits, hi_cost(T, dm, 0));
    return __fadd_rn(bits, T.dc_sign[dcs][cf[0] < 0]);
  }
  const int eob_bin = eob < 2 ? eob : 32 - __clz(eob);
  bits = __fadd_rn(bits, T.eob_bin_1d[eob_bin]);
  if (eob_bin > 1) {
    const int nb = eob_bin - 2;
    bits = __fadd_rn(bits, __fadd_rn(T.eob_hi[eob_bin][(eob >> nb) & 1], (float)nb));
  }
  uint32_t* lv32 = reinterpret_cast<uint32_t*>(lv);
#pragma unroll
  for (int i = 0; i < 40; i++) lv32[i] = 0;
  auto lo_ctx_1d = [&](int x, int y, uint32_t& hm) -> int {
    uint32_t mag = (uint32_t)lv[x * 16 + y + 1] + lv[(x + 1) * 16 + y] + lv[x * 16 + y + 2];
    hm = mag;
    mag += (uint32_t)lv[x * 16 + y + 3] + lv[x * 16 + y + 4];
    return 26 + (y > 1 ? 10 : y * 5) + (mag > 512 ? 4 : (int)((mag + 64) >> 7));
  };
  const int ctx_e = 1 + (eob > (W * W >> 3)) + (eob > (W * W >> 2));
  {
    const int x = eob & (W - 1), y = eob >> L;
    const uint32_t m = uabs(cf[pos_rc(eob)]);
    bits = __fadd_rn(bits, T.eob_base[ctx_e][min(m, 3u) - 1]);
    if (m >= 3) bits = __fadd_rn(bits, hi_cost(T, m, y != 0 ? 14 : 7));
    bits = __fadd_rn(bits, 1.0f);
    lv[x * 16 + y] = (uint8_t)level_byte(m);
  }
  for (int i = eob - 1; i >= 1; i--) {
    const int x = i & (W - 1), y = i >> L;
    const uint32_t m = uabs(cf[pos_rc(i)]);
    uint32_t hm;
    const int ctx = lo_ctx_1d(x, y, hm);
    bits = __fadd_rn(bits, T.base_tok[ctx][min(m, 3u)]);
    if (m >= 3) {
      const uint32_t mag = hm & 63;
      bits = __fadd_rn(bits, hi_cost(T, m, (y != 0 ? 14 : 7) + (mag > 12 ? 6 : (int)((mag + 1) >> 1))));
    }
    if (m != 0) bits = __fadd_rn(bits, 1.0f);
    lv[x * 16 + y] = (uint8_t)level_byte(m);
  }
  uint32_t dhm;
  const int dctx = lo_ctx_1d(0, 0, dhm);
  const uint32_t dm = uabs(cf[0]);
  bits = __fadd_rn(bits, T.base_tok[dctx][min(dm, 3u)]);
  if (dm >= 3) {
    const uint32_t mag = dhm & 63;
    bits = __fadd_rn(bits, hi_cost(T, dm, mag > 12 ? 6 : (int)((mag + 1) >> 1)));
  }
  if (dm != 0) bits = __fadd_rn(bits, T.dc_sign[dcs][cf[0] < 0]);
  return bits;
}

// A one-thread-per-job kernel's working set in the CTA's dynamic shared
// memory instead of local memory: thread t's copy at t * stride bytes.
// arena_stride rounds the size up to 128 bytes and adds 16, so consecutive
// threads' copies start 4 banks apart and every copy stays 16-byte aligned.
constexpr int arena_stride(size_t bytes) { return (int)(((bytes + 127) & ~(size_t)127) + 16); }

template <typename A>
__device__ __forceinline__ A& smem_arena(int stride) {
  extern __shared__ __align__(16) unsigned char mt_arena_smem[];
  return *reinterpret_cast<A*>(mt_arena_smem + (size_t)threadIdx.x * stride);
}

// Launch shape of an arena kernel: n jobs spread over the SMs (one CTA per
// SM while they fit), at most `cap` threads per CTA and as many copies as fit
// beside the kernel's static shared memory.  False when not even one fits.
template <typename K>
__host__ bool arena_launch_shape(K kernel, int n, int stride, int cap, int* threads, size_t* dyn) {
  cudaFuncAttributes fa;
  int dev = 0, sms = 0, optin = 0;
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return false;
  const long fit = ((long)optin - (long)fa.sharedSizeBytes) / stride;
  if (fit < 1 || sms < 1) return false;
  long t = (n + sms - 1) / sms;
  t = t < 1 ? 1 : t;
  t = t > cap ? cap : t;
  t = t > fit ? fit : t;
  *threads = (int)t;
  *dyn = (size_t)t * stride;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*dyn) == cudaSuccess;
}

// The dav1d txb_skip context table of skip_ctx_split
// (src/coder/lossy_state.rs:1367-1386), indexed by the capped ORs of the above
// and left coefficient-context bytes.
__constant__ uint8_t kSkipCtxTbl[5][5] = {
    {1, 2, 2, 2, 3}, {2, 4, 4, 4, 5}, {2, 4, 4, 4, 5}, {2, 4, 4, 4, 5}, {3, 5, 5, 5, 6}};

// coef_res_ctx of a W x W transform (levels column-major, the default scan).
template <int W, typename C>
__device__ __forceinline__ uint8_t coef_res_ctx_w(const C* __restrict__ cf) {
  int eob = -1;
  for (int i = W * W - 1; i >= 0; i--)
    if (cf[scan_rc<W>(i)] != 0) {
      eob = i;
      break;
    }
  if (eob < 0) return 0x40;
  uint32_t cul = 0;
  for (int i = 0; i <= eob && cul < 63u; i++) cul += uabs(cf[scan_rc<W>(i)]);
  const uint32_t dcb = cf[0] == 0 ? 0x40u : (cf[0] < 0 ? 0u : 0x80u);
  return (uint8_t)(min(cul, 63u) | dcb);
}

// coef_res_ctx: min(cumulative level, 63) | the dc-sign marker (0x40 zero,
// 0x00 negative, 0x80 positive), or 0x40 for an all-zero block.
template <typename C>
__device__ __forceinline__ uint8_t coef_res_ctx8(const C* __restrict__ cf) {
  int eob = -1;
  for (int i = 63; i >= 0; i--)
    if (cf[kScan8[i]] != 0) {
      eob = i;
      break;
    }
  if (eob < 0) return 0x40;
  uint32_t cul = 0;
  for (int i = 0; i <= eob; i++) cul += uabs(cf[kScan8[i]]);
  const uint32_t dcb = cf[0] == 0 ? 0x40u : (cf[0] < 0 ? 0u : 0x80u);
  return (uint8_t)(min(cul, 63u) | dcb);
}

}  // namespace mtd
