// Oracle (test-only checker of the CUDA path): the 16x16 leaf's TX_8X8 split
// trial and the pieces it adds to the candidate chain -- trellis_optimize_ctx,
// the 1-D (V_DCT / H_DCT) coefficient rate walk and the progressive
// coefficient contexts.  Each function names the reference file:line it
// restates; the float order is the reference's (x86-64 AVX2 build).
#include <math.h>
#include <string.h>

#include <thread>
#include <vector>

#include "oracle.h"
#include "../maroontree_b200/csrc/av1_tables.h"

extern "C" float or_scaled_trellis_lambda(float dc_q, float ac_q, float lambda0);
extern "C" float or_real_block_bits_bounded(const int32_t* cf, const uint16_t* scan, int32_t w, int32_t h,
                                            const mt_coef_cdfs* c, int32_t skip_ctx, int32_t dcs_ctx,
                                            int32_t txtp_mode, int32_t txtp, int32_t use_skip_bits,
                                            const float* skip_bits, float bound);

namespace {

inline uint32_t uabs(int32_t v) { return v < 0 ? 0u - (uint32_t)v : (uint32_t)v; }
inline int lz32(uint32_t v) { return v ? __builtin_clz(v) : 32; }
inline int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

// tables.rs:365-373 level_byte.
inline uint8_t level_byte(uint32_t m) {
  if (m == 0) return 0;
  if (m <= 2) return (uint8_t)(m * 0x41);
  return (uint8_t)((m < 15 ? m : 15) + (3u << 6));
}
// cost.rs:196-200 golomb_cost.
inline float golomb_cost(uint32_t v) { return (float)(2 * (32 - lz32(v + 1)) - 1); }
// cost.rs:244-262 hi_tok_cost_with_table (equal, term for term, to the cached
// br_cum ladder of cost.rs:214-241 plus the Golomb tail).
float hi_tok_cost(uint32_t m, const uint16_t* br) {
  int32_t total_br = (int32_t)m - 3;
  if (total_br > 12) total_br = 12;
  int32_t coded = 0;
  float bits = 0.0f;
  for (int k = 0; k < 4; k++) {
    int32_t s = total_br - coded;
    if (s > 3) s = 3;
    bits += or_cdf_cost(br, s);
    coded += s;
    if (s < 3) break;
  }
  if (m >= 15) bits += golomb_cost(m - 15);
  return bits;
}
inline float cost(const uint16_t* cdf, int s) { return or_cdf_cost(cdf, s); }

// coeffs.rs:46-59 get_lo_ctx_2d.
inline int lo_ctx_2d(const uint8_t* lv, int x, int y, int stride, uint32_t* hi_mag) {
  auto g = [&](int dx, int dy) -> uint32_t { return lv[(x + dx) * stride + (y + dy)]; };
  const uint32_t hm = g(0, 1) + g(1, 0) + g(1, 1);
  const uint32_t mag = hm + g(0, 2) + g(2, 0);
  *hi_mag = hm;
  return MT_LO_CTX_OFF[(y < 4 ? y : 4) * 5 + (x < 4 ? x : 4)] + (mag > 512 ? 4 : (int)((mag + 64) >> 7));
}

}  // namespace

extern "C" {

// trellis.rs:55-942 trellis_optimize_ctx for a square w x w luma block (cls of
// the slice `c`, plane 0) under the shipped tuning (tuning.rs:829-961:
// trellis_aom, trellis_eob_reprice, trellis_eob_zero_term, trellis_pad_stride
// off; trellis_dz 0; trellis_dc_ctx0 on; trellis_dc_only_scan off;
// trellis_zero_bits 1.0; trellis_tilt_mag_cap 2.0).  qm: the inverse QM row of
// the block (qm_row, quant.rs:84-90), NULL when flat.
void or_trellis_optimize_ctx(int32_t* cf, const float* tf, float dc_q, float ac_q, const uint16_t* scan, int32_t w,
                             float lambda0, const mt_coef_cdfs* c, int32_t dcs_ctx, const uint8_t* qm,
                             int32_t qm_level, float band_t) {
  if (lambda0 <= 0.0f) return;
  const int h = w, n = w * h;
  const bool qm_full = qm_level >= 5;
  auto qm_at = [&](int rc) -> float {
    const float wq = (float)qm[rc] / 32.0f;
    return qm_full ? wq * wq : wq;
  };
  const float lambda = or_scaled_trellis_lambda(dc_q, ac_q, lambda0);
  const int log2h = __builtin_ctz((unsigned)h), stride = h;
  const float cap = 2.0f;
  const float dq2_dc = dc_q * dc_q, dq2_ac = ac_q * ac_q;
  const float n_inv = 1.0f / (float)n;
  // trellis_dist.rs:100-105 trellis_dist_one, with the QM weight and the tilt.
  auto distw = [&](int idx, int rc, int32_t lev) -> float {
    const float dq2 = rc == 0 ? dq2_dc : dq2_ac;
    const float e = fabsf(tf[rc]) - (float)uabs(lev);
    float d = dq2 * (e * e);
    if (qm) d *= qm_at(rc);
    if (band_t != 0.0f && fabsf(tf[rc]) < cap) d /= 1.0f + band_t * ((float)idx * n_inv);
    return d;
  };
  int eob = -1;
  for (int i = n - 1; i >= 0; i--)
    if (cf[scan[i]] != 0) {
      eob = i;
      break;
    }
  if (eob < 0) return;
  const int eu = eob, m = eu + 1;
  auto hi_cost = [&](uint32_t k, int bc) -> float { return hi_tok_cost(k, c->br_tok[bc]); };
  std::vector<uint8_t> levels((size_t)(w + 2) * (h + 2), 0);
  auto set_level = [&](int rc, uint32_t k) { levels[(rc >> log2h) * stride + (rc & (h - 1))] = level_byte(k); };
  for (int i = 0; i <= eu; i++) {
    const int rc = scan[i];
    if (cf[rc] != 0) set_level(rc, uabs(cf[rc]));
  }
  auto interior_ctx = [&](int rc, int* bc) -> int {
    const int x = rc >> log2h, y = rc & (h - 1);
    uint32_t hm;
    const int ctx = lo_ctx_2d(levels.data(), x, y, stride, &hm);
    const uint32_t mag = hm & 63;
    *bc = ((y | x) > 1 ? 14 : 7) + (mag > 12 ? 6 : (int)((mag + 1) >> 1));
    return ctx;
  };
  auto dc_brc = [&]() -> int {
    const uint32_t mag = ((uint32_t)levels[1] + levels[stride] + levels[stride + 1]) & 63;
    return mag > 12 ? 6 : (int)((mag + 1) >> 1);
  };
  auto interior_rate = [&](int ctx, int bc, uint32_t k) -> float {
    if (k == 0) return cost(c->base_tok[ctx], 0);
    const uint32_t tok = k < 3 ? k : 3;
    float b = cost(c->base_tok[ctx], (int)tok);
    if (tok == 3) b += hi_cost(k, bc);
    return b + 1.0f;
  };
  auto eob_pt_cost = [&](int e) -> float {
    const int bin = e < 2 ? e : 32 - lz32((uint32_t)e);
    float cc = cost(c->eob_bin, bin);
    if (bin > 1) {
      const int nbits = bin - 2;
      cc += cost(c->eob_hi[bin], (e >> nbits) & 1);
      cc += (float)nbits;
    }
    return cc;
  };

  // Step A (trellis.rs:514-602): reverse-scan RD-best level of each interior
  // coefficient, then DC.
  for (int i = eob - 1; i >= 1; i--) {
    const int rc = scan[i];
    const uint32_t l = uabs(cf[rc]);
    if (l == 0) continue;
    int bc;
    const int ctx = interior_ctx(rc, &bc);
    const float bt0 = cost(c->base_tok[ctx], 0), bt1 = cost(c->base_tok[ctx], 1);
    const float bt2 = cost(c->base_tok[ctx], 2), bt3 = cost(c->base_tok[ctx], 3);
    auto rate_k = [&](uint32_t k) -> float {
      switch (k) {
        case 0: return bt0;
        case 1: return bt1 + 1.0f;
        case 2: return bt2 + 1.0f;
        default: return (bt3 + hi_cost(k, bc)) + 1.0f;
      }
    };
    uint32_t best_k = l;
    float best_c = distw(i, rc, (int32_t)l) + lambda * rate_k(l);
    for (int32_t k = (int32_t)l - 1; k >= 0; k--) {
      const float dk = distw(i, rc, k);
      if (dk >= best_c) break;
      const float cc = dk + lambda * rate_k((uint32_t)k);
      if (cc < best_c) {
        best_c = cc;
        best_k = (uint32_t)k;
      }
    }
    if (best_k != l) {
      cf[rc] = cf[rc] < 0 ? -(int32_t)best_k : (int32_t)best_k;
      set_level(rc, best_k);
    }
  }
  {
    const int rc = scan[0];
    const uint32_t l = uabs(cf[rc]);
    if (l != 0) {
      const int bc = dc_brc();
      const int sgn = cf[rc] < 0;
      auto dc_rate = [&](uint32_t k) -> float {
        if (k == 0) return cost(c->base_tok[0], 0);
        const uint32_t tok = k < 3 ? k : 3;
        float b = cost(c->base_tok[0], (int)tok);
        if (tok == 3) b += hi_cost(k, bc);
        return b + cost(c->dc_sign[dcs_ctx], sgn);
      };
      uint32_t best_k = l;
      float best_c = distw(0, rc, (int32_t)l) + lambda * dc_rate(l);
      for (int32_t k = (int32_t)l - 1; k >= 0; k--) {
        const float dk = distw(0, rc, k);
        if (dk >= best_c) break;
        const float cc = dk + lambda * dc_rate((uint32_t)k);
        if (cc < best_c) {
          best_c = cc;
          best_k = (uint32_t)k;
        }
      }
      if (best_k != l) {
        cf[rc] = cf[rc] < 0 ? -(int32_t)best_k : (int32_t)best_k;
        set_level(rc, best_k);
      }
    }
  }

  // Step B (trellis.rs:604-941): EOB position with the eob_pt / eob_base costs.
  auto eob_coeff_cost = [&](int e, uint32_t k) -> float {
    const int ctx_e = 1 + (e > n / 8) + (e > n / 4);
    const uint32_t tok = k < 3 ? k : 3;
    float cc = cost(c->eob_base[ctx_e], (int)tok - 1);
    if (tok == 3) {
      const int rc = scan[e];
      const int ex = rc >> log2h, ey = rc & (h - 1);
      cc += hi_cost(k, (ex | ey) > 1 ? 14 : 7);
    }
    return cc + 1.0f;
  };
  std::vector<float> dist_cur(m), dist_zero(m), suf0(m + 1, 0.0f), pre(m + 1, 0.0f);
  // trellis_dist.rs:178-196 (the AVX2 twin avx/trellis.rs:264-318 rounds the same).
  for (int i = 0; i < m; i++) {
    const int rc = scan[i];
    const float dq2 = rc == 0 ? dq2_dc : dq2_ac;
    const float at = fabsf(tf[rc]);
    const float e = at - (float)uabs(cf[rc]);
    dist_cur[i] = dq2 * (e * e);
    dist_zero[i] = dq2 * (at * at);
  }
  if (qm)
    for (int i = 0; i < m; i++) {
      const float w2 = qm_at(scan[i]);
      dist_cur[i] *= w2;
      dist_zero[i] *= w2;
    }
  if (band_t != 0.0f)
    for (int i = 0; i < m; i++)
      if (fabsf(tf[scan[i]]) < cap) {
        const float wgt = 1.0f / (1.0f + band_t * ((float)i * n_inv));
        dist_zero[i] *= wgt;
        dist_cur[i] *= wgt;
      }
  suf0[m] = 0.0f;
  float sacc = 0.0f;
  for (int i = m - 1; i >= 1; i--) {
    sacc += dist_zero[i];
    suf0[i] = sacc;
  }
  const int dc_rc = scan[0];
  const uint32_t dc_m = uabs(cf[dc_rc]);
  int best_e = -1;
  uint32_t best_m = 0;
  float best_cost = INFINITY;
  auto eob_cand = [&](int e, uint32_t k) -> float {
    return lambda * eob_coeff_cost(e, k) + distw(e, scan[e], (int32_t)k);
  };
  {
    float acc = 0.0f;
    for (int i = 1; i <= eu; i++) {
      const int rc = scan[i];
      int bc;
      const int ctx = interior_ctx(rc, &bc);
      const float r = interior_rate(ctx, bc, uabs(cf[rc]));
      acc += lambda * r + dist_cur[i];
      pre[i + 1] = acc;
    }
    float dc_cost;
    if (dc_m == 0) {
      dc_cost = lambda * cost(c->base_tok[0], 0);
    } else {
      const int bc = dc_brc();
      const uint32_t tok = dc_m < 3 ? dc_m : 3;
      float b = cost(c->base_tok[0], (int)tok);
      if (tok == 3) b += hi_cost(dc_m, bc);
      b += cost(c->dc_sign[dcs_ctx], cf[dc_rc] < 0);
      dc_cost = lambda * b;
    }
    dc_cost = dc_cost + dist_cur[0];
    for (int e = 1; e < m; e++) {
      const int rc = scan[e];
      const uint32_t k = uabs(cf[rc]);
      if (k == 0) continue;
      const float base = dc_cost + pre[e] + lambda * eob_pt_cost(e) + suf0[e + 1];
      uint32_t m_best = k;
      float cc = base + eob_cand(e, k);
      if (k >= 2) {
        const float c_low = base + eob_cand(e, k - 1);
        if (c_low < cc) {
          cc = c_low;
          m_best = k - 1;
        }
      }
      if (cc < best_cost) {
        best_cost = cc;
        best_e = e;
        best_m = m_best;
      }
    }
  }
  if (dc_m != 0) {
    // trellis_dc_ctx0: the DC-only terminal in eob_base context 0, br context 0.
    const uint32_t tok = dc_m < 3 ? dc_m : 3;
    float c0 = cost(c->eob_bin, 0) + cost(c->eob_base[0], (int)tok - 1);
    if (tok == 3) c0 += hi_cost(dc_m, 0);
    const float r = c0 + cost(c->dc_sign[dcs_ctx], cf[dc_rc] < 0);
    const float total0 = lambda * r + dist_cur[0] + suf0[1];
    if (total0 < best_cost) {
      best_cost = total0;
      best_e = 0;
      best_m = dc_m;
    }
  }
  const float skip_cost = suf0[1] + dist_zero[0] + lambda * 1.0f;
  if (best_e < 0 || skip_cost < best_cost) {
    for (int i = 0; i < m; i++) cf[scan[i]] = 0;
  } else {
    const int rc = scan[best_e];
    if (best_m != uabs(cf[rc])) {
      const bool neg = cf[rc] != 0 ? cf[rc] < 0 : tf[rc] < 0.0f;
      cf[rc] = neg ? -(int32_t)best_m : (int32_t)best_m;
    }
    for (int i = best_e + 1; i < m; i++) cf[scan[i]] = 0;
  }
}

// lossy_state.rs:876-1008 luma_bits_1d_8x8 (w = 8) and :1010-1143
// luma_bits_1d_4x4 (w = 4): the V_DCT / H_DCT coefficient rate against the
// decision CDFs -- txb_skip in context 0, the tx-type symbol (2 = V_DCT,
// 3 = H_DCT), the 1-D eob_pt CDF, the 1-D base-token contexts (offset 26 +),
// sign bits in place.
float or_luma_bits_1d(const int32_t* cf, int32_t w, int32_t vertical, const mt_coef_cdfs* c, int32_t dcs,
                      int32_t y_mode) {
  const int n = w * w, lw = w == 4 ? 2 : 3;
  auto pos_rc = [&](int i) -> int {
    const int x = i & (w - 1), y = i >> lw;
    return vertical ? (x << lw) | y : i;
  };
  int eob = -1;
  for (int i = n - 1; i >= 0; i--)
    if (cf[pos_rc(i)] != 0) {
      eob = i;
      break;
    }
  if (eob < 0) return cost(c->txb_skip[0], 1);
  float bits = cost(c->txb_skip[0], 0) + cost(c->txtp[y_mode], vertical ? 2 : 3);
  auto hi_bits = [&](uint32_t m, int bc) -> float { return hi_tok_cost(m, c->br_tok[bc]); };
  if (eob == 0) {
    const uint32_t dm = uabs(cf[0]);
    const uint32_t mm = dm < 3 ? dm : 3;
    bits += cost(c->eob_bin_1d, 0);
    bits += cost(c->eob_base[0], (int)mm - 1);
    if (mm == 3) bits += hi_bits(dm, 0);
    bits += cost(c->dc_sign[dcs], cf[0] < 0);
    return bits;
  }
  const int eob_bin = eob < 2 ? eob : 32 - lz32((uint32_t)eob);
  bits += cost(c->eob_bin_1d, eob_bin);
  if (eob_bin > 1) {
    const int nbits = eob_bin - 2;
    bits += cost(c->eob_hi[eob_bin], (eob >> nbits) & 1) + (float)nbits;
  }
  uint8_t levels[16 * 10];
  memset(levels, 0, sizeof(levels));
  auto lvl = [&](int x, int y) -> uint32_t { return levels[x * 16 + y]; };
  auto lo_ctx_1d = [&](int x, int y, uint32_t* hi_mag) -> int {
    uint32_t mag = lvl(x, y + 1) + lvl(x + 1, y) + lvl(x, y + 2);
    *hi_mag = mag;
    mag += lvl(x, y + 3) + lvl(x, y + 4);
    const int offset = 26 + (y > 1 ? 10 : y * 5);
    return offset + (mag > 512 ? 4 : (int)((mag + 64) >> 7));
  };
  const int ctx_e = w == 4 ? 1 + (eob > 2) + (eob > 4) : 1 + (eob > 8) + (eob > 16);
  {
    const int x = eob & (w - 1), y = eob >> lw;
    const uint32_t m = uabs(cf[pos_rc(eob)]);
    const uint32_t mm = m < 3 ? m : 3;
    bits += cost(c->eob_base[ctx_e], (int)mm - 1);
    if (mm == 3) bits += hi_bits(m, y != 0 ? 14 : 7);
    bits += 1.0f;
    levels[x * 16 + y] = level_byte(m);
  }
  for (int i = eob - 1; i >= 1; i--) {
    const int x = i & (w - 1), y = i >> lw;
    const uint32_t m = uabs(cf[pos_rc(i)]);
    uint32_t hm;
    const int ctx = lo_ctx_1d(x, y, &hm);
    const uint32_t mm = m < 3 ? m : 3;
    bits += cost(c->base_tok[ctx], (int)mm);
    if (mm == 3) {
      const uint32_t mag = hm & 63;
      bits += hi_bits(m, (y != 0 ? 14 : 7) + (mag > 12 ? 6 : (int)((mag + 1) >> 1)));
    }
    if (m != 0) bits += 1.0f;
    levels[x * 16 + y] = level_byte(m);
  }
  uint32_t dhm;
  const int dc_ctx = lo_ctx_1d(0, 0, &dhm);
  const uint32_t dm = uabs(cf[0]);
  const uint32_t dmm = dm < 3 ? dm : 3;
  bits += cost(c->base_tok[dc_ctx], (int)dmm);
  if (dmm == 3) {
    const uint32_t mag = dhm & 63;
    bits += hi_bits(dm, mag > 12 ? 6 : (int)((mag + 1) >> 1));
  }
  if (dm != 0) bits += cost(c->dc_sign[dcs], cf[0] < 0);
  return bits;
}

// lossy_state.rs:630-648 coef_res_ctx.
uint8_t or_coef_res_ctx(const int32_t* cf, const uint16_t* scan, int32_t n) {
  int eob = -1;
  for (int i = n - 1; i >= 0; i--)
    if (cf[scan[i]] != 0) {
      eob = i;
      break;
    }
  if (eob < 0) return 0x40;
  uint32_t cul = 0;
  for (int i = 0; i <= eob; i++) cul += uabs(cf[scan[i]]);
  const uint8_t dcb = cf[0] == 0 ? (1 << 6) : (cf[0] < 0 ? 0 : (2 << 6));
  return (uint8_t)((cul < 63 ? cul : 63) | dcb);
}

}  // extern "C"

namespace {

// lossy_state.rs:1367-1386 skip_ctx_split over a 2 x 2 span of 4x4 units.
int skip_ctx_split(const uint8_t* a, const uint8_t* l) {
  static const uint8_t kTbl[5][5] = {
      {1, 2, 2, 2, 3}, {2, 4, 4, 4, 5}, {2, 4, 4, 4, 5}, {2, 4, 4, 4, 5}, {3, 5, 5, 5, 6}};
  const uint8_t la = a[0] | a[1], ll = l[0] | l[1];
  const int ia = (la & 0x3f) < 4 ? (la & 0x3f) : 4, il = (ll & 0x3f) < 4 ? (ll & 0x3f) : 4;
  return kTbl[ia][il];
}
// lossy_state.rs:1388-1405 dc_sign_ctx_span over a 2 x 2 span.
int dc_sign_ctx_span(const uint8_t* a, const uint8_t* l) {
  int s = 0;
  for (int i = 0; i < 2; i++) s += (a[i] >> 6) - 1;
  for (int i = 0; i < 2; i++) s += (l[i] >> 6) - 1;
  return (s != 0) + (s > 0);
}
inline float rd_cost_i64(int64_t d, float lam, float rate) { return (float)d + lam * rate; }

// One job of split16_luma_try.  `rec` is the worker's copy of the
// reconstruction plane; the 16x16 block is restored before returning.
void split16_one(const uint16_t* src, uint16_t* rec, const mt_split16_params* p, const mt_quant* q, const uint8_t* qm,
                 const mt_coef_cdfs* cd, const mt_split16_job& jb, mt_split16_result* r, int32_t* cf_out,
                 uint16_t* rec_out) {
  const int px = jb.px, py = jb.py, stride = p->stride;
  uint16_t saved[256];
  for (int y = 0; y < 16; y++)
    for (int x = 0; x < 16; x++) saved[y * 16 + x] = rec[(size_t)(py + y) * stride + px + x];
  uint8_t a[4], l[4];
  memcpy(a, jb.a_coef, 4);
  memcpy(l, jb.l_coef, 4);
  const bool have_tr = jb.flags & MT_CAND_HAVE_TR, have_bl = jb.flags & MT_CAND_HAVE_BL;
  const int ft = (jb.flags & MT_CAND_FILTER_TYPE) != 0;
  const int32_t maxv = (1 << p->bd) - 1;
  const uint16_t* scan = or_default_scan(8);
  const float dcq = (float)q->dc_q, acq = (float)q->ac_q;
  const int vis_w = p->vis_w > 0 ? p->vis_w : p->frame_w, vis_h = p->vis_h > 0 ? p->vis_h : p->frame_h;
  const float rd_lam = p->rd_lambda;
  int64_t sse_sum = 0;
  float bits_sum = 0.0f;
  uint8_t txtps[4] = {1, 1, 1, 1};
  uint16_t blk[256];
  static const int kQuad[4][2] = {{0, 0}, {8, 0}, {0, 8}, {8, 8}};
  for (int qi = 0; qi < 4; qi++) {
    const int sx = kQuad[qi][0], sy = kQuad[qi][1], bx = px + sx, by = py + sy;
    bool tr, bl;
    switch (qi) {
      case 0: tr = py > 0; bl = px > 0; break;
      case 1: tr = have_tr; bl = false; break;
      case 2: tr = true; bl = have_bl; break;
      default: tr = false; bl = false; break;
    }
    int32_t pred[64];
    if (jb.mode == MT_DC_PRED && jb.angle_delta == 0) {
      const int32_t d = or_dc_pred(rec, stride, bx, by, 8, 8, p->bd);
      for (int i = 0; i < 64; i++) pred[i] = d;
    } else {
      or_intra_predict(rec, stride, bx, by, 8, 8, jb.mode, jb.angle_delta, tr, bl, p->frame_w, p->frame_h, ft, p->bd,
                       pred);
    }
    int32_t resid[64];
    for (int y = 0; y < 8; y++)
      for (int x = 0; x < 8; x++) resid[y * 8 + x] = (int32_t)src[(size_t)(by + y) * stride + bx + x] - pred[y * 8 + x];
    const int ax = sx / 4, ly = sy / 4;
    const int sk = skip_ctx_split(a + ax, l + ly);
    const int ds = dc_sign_ctx_span(a + ax, l + ly);
    const uint16_t pos[2] = {(uint16_t)bx, (uint16_t)by};
    auto sse_of = [&](const int32_t* rr) -> int64_t {
      int64_t d = 0;
      or_sse_recon(src, stride, vis_w, vis_h, p->bd, pos, pred, rr, 1, 8, 8, p->wsse_scale, &d);
      return d;
    };
    auto bits_2d = [&](const int32_t* cf, int txtp, float bound) -> float {
      return or_real_block_bits_bounded(cf, scan, 8, 8, cd, sk, ds, jb.mode, txtp, p->use_skip_bits,
                                        p->use_skip_bits ? p->skip_bits[sk] : nullptr, bound);
    };
    int32_t cf[64], rr[64];
    float tf[64];
    or_fwd_txfm_quant(resid, MT_TX_DCT_DCT, 8, q, qm, cf, tf);
    or_trellis_optimize_ctx(cf, tf, dcq, acq, scan, 8, p->trellis_lambda0, cd, ds, qm, q->qm_level, p->band_tilt);
    or_inv_txfm_dequant(cf, MT_TX_DCT_DCT, 8, q, qm, rr);
    const int64_t dct_sse = sse_of(rr);
    const float dct_bits = bits_2d(cf, MT_TX_DCT_DCT, INFINITY);
    int32_t bcf[64], brr[64];
    memcpy(bcf, cf, sizeof(cf));
    memcpy(brr, rr, sizeof(rr));
    int64_t bsse = dct_sse;
    float bbits = dct_bits;
    uint8_t btx = MT_TX_DCT_DCT;
    if (p->tx_search) {
      static const int kTypes[6] = {MT_TX_ADST_ADST, MT_TX_ADST_DCT, MT_TX_DCT_ADST,
                                    MT_TX_IDTX,      MT_TX_V_DCT,    MT_TX_H_DCT};
      const int64_t guard = p->tx_guard_shift >= 63 ? 0 : dct_sse >> p->tx_guard_shift;
      for (int t : kTypes) {
        int32_t acf[64], arr[64];
        float atf[64];
        or_fwd_txfm_quant(resid, t, 8, q, qm, acf, atf);
        if (t >= 4)
          or_trellis_optimize_ctx(acf, atf, dcq, acq, scan, 8, p->trellis_lambda0, cd, ds, qm, q->qm_level,
                                  p->band_tilt);
        or_inv_txfm_dequant(acf, t, 8, q, qm, arr);
        const int64_t asse = sse_of(arr);
        const bool gate = t >= 4 ? asse <= dct_sse + guard : asse <= bsse;
        if (!gate) continue;
        const float bound = (rd_cost_i64(bsse, rd_lam, bbits) - (float)asse) / rd_lam;
        const float abits = (t == MT_TX_V_DCT || t == MT_TX_H_DCT)
                                ? or_luma_bits_1d(acf, 8, t == MT_TX_V_DCT, cd, ds, jb.mode)
                                : bits_2d(acf, t, bound);
        if (rd_cost_i64(asse, rd_lam, abits) < rd_cost_i64(bsse, rd_lam, bbits)) {
          memcpy(bcf, acf, sizeof(acf));
          memcpy(brr, arr, sizeof(arr));
          bsse = asse;
          bbits = abits;
          btx = (uint8_t)t;
        }
      }
    }
    txtps[qi] = btx;
    sse_sum += bsse;
    bits_sum += bbits;
    const uint8_t res = or_coef_res_ctx(bcf, scan, 64);
    a[ax] = a[ax + 1] = res;
    l[ly] = l[ly + 1] = res;
    for (int y = 0; y < 8; y++)
      for (int x = 0; x < 8; x++) {
        const uint16_t v = (uint16_t)clampi(pred[y * 8 + x] + brr[y * 8 + x], 0, maxv);
        rec[(size_t)(by + y) * stride + bx + x] = v;
        blk[(sy + y) * 16 + sx + x] = v;
      }
    if (cf_out) memcpy(cf_out + qi * 64, bcf, sizeof(bcf));
  }
  for (int y = 0; y < 16; y++)
    for (int x = 0; x < 16; x++) rec[(size_t)(py + y) * stride + px + x] = saved[y * 16 + x];
  r->sse = sse_sum;
  r->bits = bits_sum;
  memcpy(r->tx_types, txtps, 4);
  if (rec_out) memcpy(rec_out, blk, sizeof(blk));
}

}  // namespace

extern "C" {

// partition_search.rs:4235-4428 split16_luma_try over a batch of jobs.
int or_split16_luma(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
                    const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_split16_job* jobs, int32_t n,
                    mt_split16_result* results, int32_t* cf_out, uint16_t* rec_out, int32_t threads) {
  if (!p || p->bd != 8) return MT_ERR_UNSUPPORTED;
  const size_t plane = (size_t)p->stride * p->frame_h;
  auto work = [&](int lo, int hi) {
    std::vector<uint16_t> rec(recon, recon + plane);
    for (int i = lo; i < hi; i++) {
      const mt_split16_job& jb = jobs[i];
      mt_split16_result* r = &results[i];
      const bool bad = jb.px + 16 > p->frame_w || jb.py + 16 > p->frame_h || jb.mode > MT_PAETH_PRED ||
                       jb.angle_delta < -3 || jb.angle_delta > 3 ||
                       (jb.angle_delta != 0 && (jb.mode < MT_V_PRED || jb.mode > MT_D67_PRED));
      if (bad) {
        r->sse = 0;
        r->bits = 0.0f;
        memset(r->tx_types, 255, 4);
        if (cf_out) memset(cf_out + (size_t)i * 256, 0, 256 * sizeof(int32_t));
        if (rec_out) memset(rec_out + (size_t)i * 256, 0, 256 * sizeof(uint16_t));
        continue;
      }
      split16_one(src, rec.data(), p, q, qm, cdfs, jb, r, cf_out ? cf_out + (size_t)i * 256 : nullptr,
                  rec_out ? rec_out + (size_t)i * 256 : nullptr);
    }
  };
  if (threads <= 1 || n < 64) {
    work(0, n);
    return MT_OK;
  }
  std::vector<std::thread> pool;
  const int per = (n + threads - 1) / threads;
  for (int t = 0; t < threads; t++) {
    const int lo = t * per, hi = lo + per < n ? lo + per : n;
    if (lo >= hi) break;
    pool.emplace_back(work, lo, hi);
  }
  for (auto& th : pool) th.join();
  return MT_OK;
}

}  // extern "C"

namespace {

// One job of split16_depth2_try (partition_search.rs:4524-4642); `rec` as in
// split16_one.
void depth2_one(const uint16_t* src, uint16_t* rec, const mt_split16_params* p, const mt_quant* q, const uint8_t* qm,
                const mt_coef_cdfs* cd, const mt_split16_job& jb, mt_split16_d2_result* r, int32_t* cf_out,
                uint16_t* rec_out) {
  const int px = jb.px, py = jb.py, stride = p->stride;
  uint16_t saved[256], blk[256];
  for (int y = 0; y < 16; y++)
    for (int x = 0; x < 16; x++) saved[y * 16 + x] = rec[(size_t)(py + y) * stride + px + x];
  const bool have_tr = jb.flags & MT_CAND_HAVE_TR, have_bl = jb.flags & MT_CAND_HAVE_BL;
  const int ft = (jb.flags & MT_CAND_FILTER_TYPE) != 0;
  const int32_t maxv = (1 << p->bd) - 1;
  const uint16_t* scan = or_default_scan(4);
  const float dcq = (float)q->dc_q, acq = (float)q->ac_q, rd_lam = p->rd_lambda;
  const int vis_w = p->vis_w > 0 ? p->vis_w : p->frame_w, vis_h = p->vis_h > 0 ? p->vis_h : p->frame_h;
  const float* skip = p->use_skip_bits ? p->skip_bits[0] : nullptr;
  int64_t sse_sum = 0;
  float bits_sum = 0.0f;
  for (int j = 0; j < 4; j++)
    for (int i = 0; i < 4; i++) {
      const int ti = j * 4 + i, bx = px + i * 4, by = py + j * 4;
      const bool tr = j == 0 ? (py > 0 && (i < 3 || have_tr)) : i < 3;
      const bool bl = i == 0 ? (px > 0 && (j < 3 || have_bl)) : false;
      int32_t pred[16];
      if (jb.mode == MT_DC_PRED && jb.angle_delta == 0) {
        const int32_t d = or_dc_pred(rec, stride, bx, by, 4, 4, p->bd);
        for (int k = 0; k < 16; k++) pred[k] = d;
      } else {
        or_intra_predict(rec, stride, bx, by, 4, 4, jb.mode, jb.angle_delta, tr, bl, p->frame_w, p->frame_h, ft,
                         p->bd, pred);
      }
      int32_t resid[16];
      for (int y = 0; y < 4; y++)
        for (int x = 0; x < 4; x++) resid[y * 4 + x] = (int32_t)src[(size_t)(by + y) * stride + bx + x] - pred[y * 4 + x];
      // luma_bits' whole-block contexts (lossy_state.rs:495-513): txb_skip 0,
      // dc_sign over this 4x4's own above / left bytes, left untouched by the trial.
      int s = (jb.a_coef[i] >> 6) - 1 + (jb.l_coef[j] >> 6) - 1;
      const int ds = (s != 0) + (s > 0);
      const uint16_t pos[2] = {(uint16_t)bx, (uint16_t)by};
      auto sse_of = [&](const int32_t* rr) -> int64_t {
        int64_t d = 0;
        or_sse_recon(src, stride, vis_w, vis_h, p->bd, pos, pred, rr, 1, 4, 4, p->wsse_scale, &d);
        return d;
      };
      int32_t bcf[16], brr[16];
      float tf[16];
      or_fwd_txfm_quant(resid, MT_TX_DCT_DCT, 4, q, qm, bcf, tf);
      or_trellis_optimize(bcf, tf, dcq, acq, scan, 16, p->trellis_lambda0);
      or_inv_txfm_dequant(bcf, MT_TX_DCT_DCT, 4, q, qm, brr);
      const int64_t dct_sse = sse_of(brr);
      int64_t bsse = dct_sse;
      float bbits = or_real_block_bits_bounded(bcf, scan, 4, 4, cd, 0, ds, jb.mode, MT_TX_DCT_DCT,
                                               p->use_skip_bits, skip, INFINITY);
      uint8_t btx = MT_TX_DCT_DCT;
      const int64_t guard = p->tx_guard_shift >= 63 ? 0 : dct_sse >> p->tx_guard_shift;
      static const int kTypes[4] = {MT_TX_ADST_ADST, MT_TX_IDTX, MT_TX_V_DCT, MT_TX_H_DCT};
      for (int t : kTypes) {
        int32_t acf[16], arr[16];
        float atf[16];
        or_fwd_txfm_quant(resid, t, 4, q, qm, acf, atf);
        if (t == MT_TX_ADST_ADST) or_trellis_optimize(acf, atf, dcq, acq, scan, 16, p->trellis_lambda0);
        or_inv_txfm_dequant(acf, t, 4, q, qm, arr);
        const int64_t asse = sse_of(arr);
        const float best_rd = rd_cost_i64(bsse, rd_lam, bbits);
        const float bound = (best_rd - (float)asse) / rd_lam;
        const float abits = (t == MT_TX_V_DCT || t == MT_TX_H_DCT)
                                ? or_luma_bits_1d(acf, 4, t == MT_TX_V_DCT, cd, ds, jb.mode)
                                : or_real_block_bits_bounded(acf, scan, 4, 4, cd, 0, ds, jb.mode, t, p->use_skip_bits,
                                                             skip, bound);
        if (asse <= dct_sse + guard && rd_cost_i64(asse, rd_lam, abits) < best_rd) {
          memcpy(bcf, acf, sizeof(acf));
          memcpy(brr, arr, sizeof(arr));
          bsse = asse;
          bbits = abits;
          btx = (uint8_t)t;
        }
      }
      r->tx_types[ti] = btx;
      sse_sum += bsse;
      bits_sum += bbits;
      for (int y = 0; y < 4; y++)
        for (int x = 0; x < 4; x++) {
          const uint16_t v = (uint16_t)clampi(pred[y * 4 + x] + brr[y * 4 + x], 0, maxv);
          rec[(size_t)(by + y) * stride + bx + x] = v;
          blk[(j * 4 + y) * 16 + i * 4 + x] = v;
        }
      if (cf_out) memcpy(cf_out + ti * 16, bcf, sizeof(bcf));
    }
  for (int y = 0; y < 16; y++)
    for (int x = 0; x < 16; x++) rec[(size_t)(py + y) * stride + px + x] = saved[y * 16 + x];
  r->sse = sse_sum;
  r->bits = bits_sum;
  memset(r->reserved, 0, sizeof(r->reserved));
  if (rec_out) memcpy(rec_out, blk, sizeof(blk));
}

}  // namespace

extern "C" {

// partition_search.rs:4524-4642 split16_depth2_try over a batch of jobs.
int or_split16_depth2(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
                      const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_split16_job* jobs, int32_t n,
                      mt_split16_d2_result* results, int32_t* cf_out, uint16_t* rec_out, int32_t threads) {
  if (!p || p->bd != 8) return MT_ERR_UNSUPPORTED;
  const size_t plane = (size_t)p->stride * p->frame_h;
  auto work = [&](int lo, int hi) {
    std::vector<uint16_t> rec(recon, recon + plane);
    for (int i = lo; i < hi; i++) {
      const mt_split16_job& jb = jobs[i];
      mt_split16_d2_result* r = &results[i];
      const bool bad = jb.px + 16 > p->frame_w || jb.py + 16 > p->frame_h || jb.mode > MT_PAETH_PRED ||
                       jb.angle_delta < -3 || jb.angle_delta > 3 ||
                       (jb.angle_delta != 0 && (jb.mode < MT_V_PRED || jb.mode > MT_D67_PRED));
      if (bad) {
        r->sse = 0;
        r->bits = 0.0f;
        memset(r->tx_types, 255, 16);
        memset(r->reserved, 0, 4);
        if (cf_out) memset(cf_out + (size_t)i * 256, 0, 256 * sizeof(int32_t));
        if (rec_out) memset(rec_out + (size_t)i * 256, 0, 256 * sizeof(uint16_t));
        continue;
      }
      depth2_one(src, rec.data(), p, q, qm, cdfs, jb, r, cf_out ? cf_out + (size_t)i * 256 : nullptr,
                 rec_out ? rec_out + (size_t)i * 256 : nullptr);
    }
  };
  if (threads <= 1 || n < 64) {
    work(0, n);
    return MT_OK;
  }
  std::vector<std::thread> pool;
  const int per = (n + threads - 1) / threads;
  for (int t = 0; t < threads; t++) {
    const int lo = t * per, hi = lo + per < n ? lo + per : n;
    if (lo >= hi) break;
    pool.emplace_back(work, lo, hi);
  }
  for (auto& th : pool) th.join();
  return MT_OK;
}

}  // extern "C"

namespace {

// One job of split4tx_try (block8.rs:157-286); `rec` as in split16_one.
void split4tx_one(const uint16_t* src, uint16_t* rec, const mt_split16_params* p, const mt_quant* q, const uint8_t* qm,
                  const mt_coef_cdfs* cd, const mt_split16_job& jb, mt_split16_result* r, int32_t* cf_out,
                  uint16_t* rec_out) {
  const int px = jb.px, py = jb.py, stride = p->stride;
  uint16_t saved[64], blk[64];
  for (int y = 0; y < 8; y++)
    for (int x = 0; x < 8; x++) saved[y * 8 + x] = rec[(size_t)(py + y) * stride + px + x];
  const bool have_tr = jb.flags & MT_CAND_HAVE_TR, have_bl = jb.flags & MT_CAND_HAVE_BL;
  const int ft = (jb.flags & MT_CAND_FILTER_TYPE) != 0;
  const int32_t maxv = (1 << p->bd) - 1;
  const uint16_t* scan = or_default_scan(4);
  const float dcq = (float)q->dc_q, acq = (float)q->ac_q, rd_lam = p->rd_lambda;
  const int vis_w = p->vis_w > 0 ? p->vis_w : p->frame_w, vis_h = p->vis_h > 0 ? p->vis_h : p->frame_h;
  const float* skip = p->use_skip_bits ? p->skip_bits[0] : nullptr;
  static const int kQuad[4][2] = {{0, 0}, {4, 0}, {0, 4}, {4, 4}};
  int64_t sse_sum = 0;
  float bits_sum = 0.0f;
  for (int qi = 0; qi < 4; qi++) {
    const int sx = kQuad[qi][0], sy = kQuad[qi][1], bx = px + sx, by = py + sy;
    bool tr, bl;
    switch (qi) {
      case 0: tr = py > 0; bl = px > 0; break;
      case 1: tr = have_tr; bl = false; break;
      case 2: tr = true; bl = have_bl; break;
      default: tr = false; bl = false; break;
    }
    int32_t pred[16];
    if (jb.mode == MT_DC_PRED) {
      const int32_t d = or_dc_pred(rec, stride, bx, by, 4, 4, p->bd);
      for (int k = 0; k < 16; k++) pred[k] = d;
    } else {
      or_intra_predict(rec, stride, bx, by, 4, 4, jb.mode, jb.angle_delta, tr, bl, p->frame_w, p->frame_h, ft, p->bd,
                       pred);
    }
    int32_t resid[16];
    for (int y = 0; y < 4; y++)
      for (int x = 0; x < 4; x++) resid[y * 4 + x] = (int32_t)src[(size_t)(by + y) * stride + bx + x] - pred[y * 4 + x];
    // luma_bits' whole-block contexts of this 4x4 (lossy_state.rs:495-513).
    const int s = (jb.a_coef[sx / 4] >> 6) - 1 + (jb.l_coef[sy / 4] >> 6) - 1;
    const int ds = (s != 0) + (s > 0);
    const uint16_t pos[2] = {(uint16_t)bx, (uint16_t)by};
    auto sse_of = [&](const int32_t* rr) -> int64_t {
      int64_t d = 0;
      or_sse_recon(src, stride, vis_w, vis_h, p->bd, pos, pred, rr, 1, 4, 4, p->wsse_scale, &d);
      return d;
    };
    int32_t bcf[16], brr[16];
    float tf[16];
    or_fwd_txfm_quant(resid, MT_TX_DCT_DCT, 4, q, qm, bcf, tf);
    or_trellis_optimize(bcf, tf, dcq, acq, scan, 16, p->trellis_lambda0);
    or_inv_txfm_dequant(bcf, MT_TX_DCT_DCT, 4, q, qm, brr);
    const int64_t dct_sse = sse_of(brr);
    int64_t bsse = dct_sse;
    float bbits = or_real_block_bits_bounded(bcf, scan, 4, 4, cd, 0, ds, jb.mode, MT_TX_DCT_DCT, p->use_skip_bits,
                                             skip, INFINITY);
    uint8_t btx = MT_TX_DCT_DCT;
    const int64_t guard = p->tx_guard_shift >= 63 ? 0 : dct_sse >> p->tx_guard_shift;
    for (int t : {MT_TX_ADST_ADST, MT_TX_IDTX}) {
      int32_t acf[16], arr[16];
      float atf[16];
      or_fwd_txfm_quant(resid, t, 4, q, qm, acf, atf);
      if (t == MT_TX_ADST_ADST) or_trellis_optimize(acf, atf, dcq, acq, scan, 16, p->trellis_lambda0);
      or_inv_txfm_dequant(acf, t, 4, q, qm, arr);
      const int64_t asse = sse_of(arr);
      if (asse > dct_sse + guard) continue;
      const float best_rd = rd_cost_i64(bsse, rd_lam, bbits);
      const float bound = (best_rd - (float)asse) / rd_lam;
      const float abits =
          or_real_block_bits_bounded(acf, scan, 4, 4, cd, 0, ds, jb.mode, t, p->use_skip_bits, skip, bound);
      if (rd_cost_i64(asse, rd_lam, abits) < best_rd) {
        memcpy(bcf, acf, sizeof(acf));
        memcpy(brr, arr, sizeof(arr));
        bsse = asse;
        bbits = abits;
        btx = (uint8_t)t;
      }
    }
    r->tx_types[qi] = btx;
    sse_sum += bsse;
    bits_sum += bbits;
    for (int y = 0; y < 4; y++)
      for (int x = 0; x < 4; x++) {
        const uint16_t v = (uint16_t)clampi(pred[y * 4 + x] + brr[y * 4 + x], 0, maxv);
        rec[(size_t)(by + y) * stride + bx + x] = v;
        blk[(sy + y) * 8 + sx + x] = v;
      }
    if (cf_out) memcpy(cf_out + qi * 16, bcf, sizeof(bcf));
  }
  for (int y = 0; y < 8; y++)
    for (int x = 0; x < 8; x++) rec[(size_t)(py + y) * stride + px + x] = saved[y * 8 + x];
  r->sse = sse_sum;
  r->bits = bits_sum;
  if (rec_out) memcpy(rec_out, blk, sizeof(blk));
}

}  // namespace

extern "C" {

// block8.rs:157-286 split4tx_try over a batch of 8x8 jobs.
int or_split4tx(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
                const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_split16_job* jobs, int32_t n,
                mt_split16_result* results, int32_t* cf_out, uint16_t* rec_out) {
  if (!p || p->bd != 8) return MT_ERR_UNSUPPORTED;
  std::vector<uint16_t> rec(recon, recon + (size_t)p->stride * p->frame_h);
  for (int i = 0; i < n; i++) {
    const mt_split16_job& jb = jobs[i];
    mt_split16_result* r = &results[i];
    const bool bad = jb.px + 8 > p->frame_w || jb.py + 8 > p->frame_h || jb.mode > MT_PAETH_PRED ||
                     jb.angle_delta < -3 || jb.angle_delta > 3 ||
                     (jb.angle_delta != 0 && (jb.mode < MT_V_PRED || jb.mode > MT_D67_PRED));
    if (bad) {
      r->sse = 0;
      r->bits = 0.0f;
      memset(r->tx_types, 255, 4);
      if (cf_out) memset(cf_out + (size_t)i * 64, 0, 64 * sizeof(int32_t));
      if (rec_out) memset(rec_out + (size_t)i * 64, 0, 64 * sizeof(uint16_t));
      continue;
    }
    split4tx_one(src, rec.data(), p, q, qm, cdfs, jb, r, cf_out ? cf_out + (size_t)i * 64 : nullptr,
                 rec_out ? rec_out + (size_t)i * 64 : nullptr);
  }
  return MT_OK;
}

}  // extern "C"

extern "C" {

// block8.rs:738-808 (refine = 0: the Slow mode loop's candidate) and
// :1183-1404 (refine = 1: the winner's transform-type refinement) of
// pick_block8 over a batch of 8x8 jobs (N = 8), the same two stages of
// pick_luma16 over 16x16 jobs (N = 16), or pick_luma32's mode-loop candidates
// over 32x32 jobs (N = 32, refine 0: block32.rs:776-836, TX_32X32 DCT_DCT).
static int leaf_impl(int N, const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
                     const uint8_t* qm, const mt_coef_cdfs* cd, const mt_leaf8_job* jobs, int32_t n, int32_t refine,
                     mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out) {
  if (!p || p->bd != 8) return MT_ERR_UNSUPPORTED;
  const int NN = N * N;
  const int32_t maxv = (1 << p->bd) - 1;
  const uint16_t* scan = or_default_scan(N);
  const float dcq = (float)q->dc_q, acq = (float)q->ac_q, mlam = p->rd_lambda;
  const int vis_w = p->vis_w > 0 ? p->vis_w : p->frame_w, vis_h = p->vis_h > 0 ? p->vis_h : p->frame_h;
  const float* skip = p->use_skip_bits ? p->skip_bits[0] : nullptr;
  auto guard = [&](int64_t d) -> int64_t { return p->tx_guard_shift >= 63 ? 0 : d >> p->tx_guard_shift; };
  for (int i = 0; i < n; i++) {
    const mt_leaf8_job& jb = jobs[i];
    mt_leaf8_result* r = &results[i];
    memset(r->reserved, 0, sizeof(r->reserved));
    const bool bad = jb.px + N > p->frame_w || jb.py + N > p->frame_h || jb.mode > MT_PAETH_PRED ||
                     jb.angle_delta < -3 || jb.angle_delta > 3 ||
                     (jb.angle_delta != 0 && (jb.mode < MT_V_PRED || jb.mode > MT_D67_PRED)) || jb.dcs_ctx > 2;
    if (bad) {
      r->sse = 0;
      r->bits = r->cost = INFINITY;
      r->tx_type = 255;
      if (cf_out) memset(cf_out + (size_t)i * NN, 0, NN * 4);
      if (rec_out) memset(rec_out + (size_t)i * NN, 0, NN * 2);
      continue;
    }
    int32_t pred[1024];
    if (jb.mode == MT_DC_PRED) {
      const int32_t d = or_dc_pred(recon, p->stride, jb.px, jb.py, N, N, p->bd);
      for (int k = 0; k < NN; k++) pred[k] = d;
    } else {
      or_intra_predict(recon, p->stride, jb.px, jb.py, N, N, jb.mode, jb.angle_delta, jb.flags & 1,
                       (jb.flags >> 1) & 1, p->frame_w, p->frame_h, (jb.flags >> 2) & 1, p->bd, pred);
    }
    int32_t resid[1024];
    for (int y = 0; y < N; y++)
      for (int x = 0; x < N; x++)
        resid[y * N + x] = (int32_t)src[(size_t)(jb.py + y) * p->stride + jb.px + x] - pred[y * N + x];
    const int ds = jb.dcs_ctx;
    const uint16_t pos[2] = {jb.px, jb.py};
    auto sse_of = [&](const int32_t* rr) -> int64_t {
      int64_t d = 0;
      or_sse_recon(src, p->stride, vis_w, vis_h, p->bd, pos, pred, rr, 1, N, N, p->wsse_scale, &d);
      return d;
    };
    // The tx-type symbol: MT_TX_* is the 7-type TX_8X8 intra set's index;
    // the 5-type TX_16X16 set (IDTX, DCT_DCT, ADST_ADST, ADST_DCT, DCT_ADST)
    // drops V_DCT / H_DCT (cost.rs:95-108).
    auto bits2d = [&](const int32_t* cf, int t, float bound) -> float {
      const int sym = N == 16 && t >= MT_TX_ADST_ADST ? t - 2 : t;
      // TX_32X32 intra codes no tx-type symbol (lossy_state.rs:533-539)
      return or_real_block_bits_bounded(cf, scan, N, N, cd, 0, ds, N == 32 ? -1 : jb.mode, sym, p->use_skip_bits,
                                        skip, bound);
    };
    // The DCT_DCT candidate with the per-candidate trellis (block8.rs:780-805).
    int32_t lcf[1024], lrr[1024];
    float tf[1024];
    or_fwd_txfm_quant(resid, MT_TX_DCT_DCT, N, q, qm, lcf, tf);
    or_trellis_optimize_ctx(lcf, tf, dcq, acq, scan, N, p->trellis_lambda0, cd, ds, qm, q->qm_level, p->band_tilt);
    or_inv_txfm_dequant(lcf, MT_TX_DCT_DCT, N, q, qm, lrr);
    const int64_t dct_sse = sse_of(lrr);
    const float dct_bits = bits2d(lcf, MT_TX_DCT_DCT, INFINITY);
    int64_t bsse = dct_sse;
    float bbits = dct_bits;
    uint8_t btx = MT_TX_DCT_DCT;
    if (refine) {
      auto take = [&](const int32_t* cf, const int32_t* rr, int64_t s, float b, int t) {
        memcpy(lcf, cf, NN * sizeof(int32_t));
        memcpy(lrr, rr, NN * sizeof(int32_t));
        bsse = s;
        bbits = b;
        btx = (uint8_t)t;
      };
      // ADST_ADST (block8.rs:1214-1262; partition_search.rs:5276-5328): bounded
      // by the DCT's rd cost.  An aborted rate is infinite, so an accepted
      // one is exact.
      {
        int32_t acf[1024], arr[1024];
        float atf[1024];
        or_fwd_txfm_quant(resid, MT_TX_ADST_ADST, N, q, qm, acf, atf);
        or_trellis_optimize_ctx(acf, atf, dcq, acq, scan, N, p->trellis_lambda0, cd, ds, qm, q->qm_level,
                                p->band_tilt);
        or_inv_txfm_dequant(acf, MT_TX_ADST_ADST, N, q, qm, arr);
        const int64_t asse = sse_of(arr);
        const float base_rd = rd_cost_i64(dct_sse, mlam, dct_bits);
        const float abits = bits2d(acf, MT_TX_ADST_ADST, (base_rd - (float)asse) / mlam);
        if (asse <= dct_sse + guard(dct_sse) && rd_cost_i64(asse, mlam, abits) < base_rd)
          take(acf, arr, asse, abits, MT_TX_ADST_ADST);
      }
      // ADST_DCT, DCT_ADST against the running winner (block8.rs:1264-1332,
      // bounded rate; partition_search.rs:5331-5423, unbounded luma_bits, the
      // ADST_ADST winner re-priced unbounded -- the same value).
      for (int t : {MT_TX_ADST_DCT, MT_TX_DCT_ADST}) {
        int32_t acf[1024], arr[1024];
        float atf[1024];
        or_fwd_txfm_quant(resid, t, N, q, qm, acf, atf);
        or_trellis_optimize_ctx(acf, atf, dcq, acq, scan, N, p->trellis_lambda0, cd, ds, qm, q->qm_level,
                                p->band_tilt);
        or_inv_txfm_dequant(acf, t, N, q, qm, arr);
        const int64_t asse = sse_of(arr);
        const float base_rd = rd_cost_i64(bsse, mlam, bbits);
        const float abits = bits2d(acf, t, N == 8 ? (base_rd - (float)asse) / mlam : INFINITY);
        if (asse <= dct_sse + guard(dct_sse) && rd_cost_i64(asse, mlam, abits) < base_rd)
          take(acf, arr, asse, abits, t);
      }
      // IDTX without the trellis, within tx_guard of the winner's SSE
      // (block8.rs:1334-1361; partition_search.rs:5425-5474)
      {
        int32_t icf[1024], irr[1024];
        float itf[1024];
        or_fwd_txfm_quant(resid, MT_TX_IDTX, N, q, qm, icf, itf);
        or_inv_txfm_dequant(icf, MT_TX_IDTX, N, q, qm, irr);
        const int64_t isse = sse_of(irr);
        const float ibits = bits2d(icf, MT_TX_IDTX, INFINITY);
        const float base_rd = rd_cost_i64(bsse, mlam, bbits);
        if (isse <= bsse + guard(bsse) && rd_cost_i64(isse, mlam, ibits) < base_rd)
          take(icf, irr, isse, ibits, MT_TX_IDTX);
      }
      // V_DCT, H_DCT unless 4:2:0 (block8.rs:1362-1396); the 16x16 intra set
      // has no 1-D types.
      if (N == 8 && p->tx_search)
        for (int vertical = 1; vertical >= 0; vertical--) {
          const int t = vertical ? MT_TX_V_DCT : MT_TX_H_DCT;
          int32_t vcf[64], vrr[64];
          float vtf[64];
          or_fwd_txfm_quant(resid, t, 8, q, qm, vcf, vtf);
          or_inv_txfm_dequant(vcf, t, 8, q, qm, vrr);
          const int64_t vsse = sse_of(vrr);
          const float vbits = or_luma_bits_1d(vcf, 8, vertical, cd, ds, jb.mode);
          const float base_rd = rd_cost_i64(bsse, mlam, bbits);
          if (vsse <= bsse && rd_cost_i64(vsse, mlam, vbits) < base_rd) take(vcf, vrr, vsse, vbits, t);
        }
    }
    r->sse = bsse;
    r->bits = bbits;
    r->cost = refine ? rd_cost_i64(bsse, mlam, bbits) : rd_cost_i64(bsse, mlam, bbits + jb.syntax_bits);
    r->tx_type = btx;
    if (cf_out) memcpy(cf_out + (size_t)i * NN, lcf, NN * sizeof(int32_t));
    if (rec_out)
      for (int k = 0; k < NN; k++) rec_out[(size_t)i * NN + k] = (uint16_t)clampi(pred[k] + lrr[k], 0, maxv);
  }
  return MT_OK;
}

int or_leaf8(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
             const uint8_t* qm, const mt_coef_cdfs* cd, const mt_leaf8_job* jobs, int32_t n, int32_t refine,
             mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out) {
  return leaf_impl(8, src, recon, p, q, qm, cd, jobs, n, refine, results, cf_out, rec_out);
}

// partition_search.rs:4802-4880 pick_luma16's mode-loop candidates (refine 0)
// and :5252-5474 the winner's transform-type refinement (refine 1).
int or_leaf16(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
              const uint8_t* qm, const mt_coef_cdfs* cd, const mt_leaf8_job* jobs, int32_t n, int32_t refine,
              mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out) {
  return leaf_impl(16, src, recon, p, q, qm, cd, jobs, n, refine, results, cf_out, rec_out);
}

// block64.rs:1906-1958 rd_pick_luma64's four-TX_32X32 leg (Quad32) of each
// (64x64 block, mode, delta) job: the quadrants in Q64 order (:328), each
// predicted at 32x32 from the running reconstruction with quad_edges'
// flags (:2731-2745), DCT_DCT + QM, trellis_optimize_ctx in the quadrant's
// dc_sign context, the inverse, luma_pick_distortion's Wsse metric
// (chroma_sse's value x K_PART_LAMBDA, lossy_state.rs:2363-2382, :1804-1806),
// luma_bits, recon_add_pred back into the reconstruction; total =
// rate_cost(mlam, mode_bits) [+ rate_cost(mlam, delta_bits)] + the quadrants'
// rd_cost (partition_rd.rs:140-142).  Each job starts from the block's
// reconstruction as given (the reference restores it per candidate).
int or_quad32_luma(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
                   const uint8_t* qm, const mt_coef_cdfs* cd, const mt_quad32_job* jobs, int32_t n,
                   mt_quad32_result* results) {
  if (!p || p->bd != 8) return MT_ERR_UNSUPPORTED;
  const int32_t maxv = (1 << p->bd) - 1;
  const uint16_t* scan = or_default_scan(32);
  const float dcq = (float)q->dc_q, acq = (float)q->ac_q, mlam = p->rd_lambda;
  const int vis_w = p->vis_w > 0 ? p->vis_w : p->frame_w, vis_h = p->vis_h > 0 ? p->vis_h : p->frame_h;
  const float* skip = p->use_skip_bits ? p->skip_bits[0] : nullptr;
  std::vector<uint16_t> work(recon, recon + (size_t)p->stride * p->frame_h);
  std::vector<int32_t> pred(1024), resid(1024), cf(1024), rr(1024);
  std::vector<float> tf(1024);
  for (int i = 0; i < n; i++) {
    const mt_quad32_job& jb = jobs[i];
    mt_quad32_result* r = &results[i];
    r->reserved = 0;
    const bool directional = jb.mode >= MT_V_PRED && jb.mode <= MT_D67_PRED;
    const bool bad = jb.px + 64 > p->frame_w || jb.py + 64 > p->frame_h || jb.mode > MT_PAETH_PRED ||
                     jb.angle_delta < -3 || jb.angle_delta > 3 || (jb.angle_delta != 0 && !directional) ||
                     jb.dcs_ctx[0] > 2 || jb.dcs_ctx[1] > 2 || jb.dcs_ctx[2] > 2 || jb.dcs_ctx[3] > 2;
    if (bad) {
      r->total = INFINITY;
      for (int k = 0; k < 4; k++) {
        r->bits[k] = INFINITY;
        r->sse[k] = 0;
      }
      continue;
    }
    const bool have_tr = jb.flags & 1, have_bl = (jb.flags >> 1) & 1, ft = (jb.flags >> 2) & 1;
    float total = mlam * jb.mode_bits;
    if (directional) total += mlam * jb.delta_bits;
    static const int kQ64[4][2] = {{0, 0}, {32, 0}, {0, 32}, {32, 32}};
    for (int k = 0; k < 4; k++) {
      const int sx = kQ64[k][0], sy = kQ64[k][1];
      const int bx = jb.px + sx, by = jb.py + sy;
      bool tr, bl;  // quad_edges
      if (sx == 0 && sy == 0) {
        tr = jb.py > 0;
        bl = jb.px > 0;
      } else if (sy == 0) {
        tr = have_tr;
        bl = false;
      } else if (sx == 0) {
        tr = true;
        bl = have_bl;
      } else {
        tr = bl = false;
      }
      if (jb.mode == MT_DC_PRED) {
        const int32_t d = or_dc_pred(work.data(), p->stride, bx, by, 32, 32, p->bd);
        for (int t = 0; t < 1024; t++) pred[t] = d;
      } else {
        or_intra_predict(work.data(), p->stride, bx, by, 32, 32, jb.mode, jb.angle_delta, tr, bl, p->frame_w,
                         p->frame_h, ft, p->bd, pred.data());
      }
      for (int y = 0; y < 32; y++)
        for (int x = 0; x < 32; x++)
          resid[y * 32 + x] = (int32_t)src[(size_t)(by + y) * p->stride + bx + x] - pred[y * 32 + x];
      or_fwd_txfm_quant(resid.data(), MT_TX_DCT_DCT, 32, q, qm, cf.data(), tf.data());
      or_trellis_optimize_ctx(cf.data(), tf.data(), dcq, acq, scan, 32, p->trellis_lambda0, cd, jb.dcs_ctx[k], qm,
                              q->qm_level, p->band_tilt);
      or_inv_txfm_dequant(cf.data(), MT_TX_DCT_DCT, 32, q, qm, rr.data());
      const uint16_t pos[2] = {(uint16_t)bx, (uint16_t)by};
      int64_t sse = 0;
      or_sse_recon(src, p->stride, vis_w, vis_h, p->bd, pos, pred.data(), rr.data(), 1, 32, 32, p->wsse_scale, &sse);
      const float dist = (float)sse * 2.775f;
      const float bits = or_real_block_bits_bounded(cf.data(), scan, 32, 32, cd, 0, jb.dcs_ctx[k], -1, 0,
                                                    p->use_skip_bits, skip, INFINITY);
      total += dist + mlam * bits;
      r->bits[k] = bits;
      r->sse[k] = sse;
      for (int y = 0; y < 32; y++)
        for (int x = 0; x < 32; x++)
          work[(size_t)(by + y) * p->stride + bx + x] = (uint16_t)clampi(pred[y * 32 + x] + rr[y * 32 + x], 0, maxv);
    }
    r->total = total;
    for (int y = 0; y < 64; y++)  // the next job predicts from the input reconstruction
      memcpy(&work[(size_t)(jb.py + y) * p->stride + jb.px], &recon[(size_t)(jb.py + y) * p->stride + jb.px], 128);
  }
  return MT_OK;
}

// rd_pick_luma64's tx_depth-2 trial (src/coder/block64.rs:1983-2010) through
// grid16_luma_pass (:1670-1805): sixteen TX_16X16 in raster order on one
// (mode, delta), the coefficient contexts carried between transforms.
int or_grid16_luma(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
                   const uint8_t* qm, const mt_coef_cdfs* cd, const mt_grid16_job* jobs, int32_t n,
                   mt_grid16_result* results, int32_t* cf_out) {
  if (!p || p->bd != 8) return MT_ERR_UNSUPPORTED;
  const int32_t maxv = (1 << p->bd) - 1;
  const uint16_t* scan = or_default_scan(16);
  const float dcq = (float)q->dc_q, acq = (float)q->ac_q, mlam = p->rd_lambda;
  const int vis_w = p->vis_w > 0 ? p->vis_w : p->frame_w, vis_h = p->vis_h > 0 ? p->vis_h : p->frame_h;
  std::vector<uint16_t> work(recon, recon + (size_t)p->stride * p->frame_h);
  std::vector<int32_t> pred(256), resid(256), cf(256), rr(256);
  std::vector<float> tf(256);
  for (int i = 0; i < n; i++) {
    const mt_grid16_job& jb = jobs[i];
    mt_grid16_result* r = &results[i];
    r->reserved = 0;
    const bool directional = jb.mode >= MT_V_PRED && jb.mode <= MT_D67_PRED;
    const bool bad = jb.px + 64 > p->frame_w || jb.py + 64 > p->frame_h || jb.mode > MT_PAETH_PRED ||
                     jb.angle_delta < -3 || jb.angle_delta > 3 || (jb.angle_delta != 0 && !directional);
    if (bad) {
      r->total = r->dist = r->bits = INFINITY;
      r->sse = 0;
      if (cf_out) memset(cf_out + (size_t)i * 4096, 0, 4096 * sizeof(int32_t));
      continue;
    }
    uint8_t a[16], l[16];
    memcpy(a, jb.a_coef, 16);
    memcpy(l, jb.l_coef, 16);
    const bool have_tr = jb.flags & MT_CAND_HAVE_TR, have_bl = jb.flags & MT_CAND_HAVE_BL;
    const int ft = (jb.flags & MT_CAND_FILTER_TYPE) != 0;
    float dist = 0.0f, bits = 0.0f;
    int64_t sse_sum = 0;
    for (int ty = 0; ty < 4; ty++)
      for (int tx = 0; tx < 4; tx++) {
        const int bx = jb.px + tx * 16, by = jb.py + ty * 16;
        const bool tr = ty == 0 ? (jb.py > 0 && (tx < 3 || have_tr)) : tx < 3;
        const bool bl = tx == 0 ? (jb.px > 0 && (ty < 3 || have_bl)) : false;
        if (jb.mode == MT_DC_PRED) {
          const int32_t d = or_dc_pred(work.data(), p->stride, bx, by, 16, 16, p->bd);
          for (int t = 0; t < 256; t++) pred[t] = d;
        } else {
          or_intra_predict(work.data(), p->stride, bx, by, 16, 16, jb.mode, jb.angle_delta, tr, bl, p->frame_w,
                           p->frame_h, ft, p->bd, pred.data());
        }
        for (int y = 0; y < 16; y++)
          for (int x = 0; x < 16; x++)
            resid[y * 16 + x] = (int32_t)src[(size_t)(by + y) * p->stride + bx + x] - pred[y * 16 + x];
        // skip_ctx_split / dc_sign_ctx_span over the transform's four above
        // and four left context bytes
        uint8_t la = 0, ll = 0;
        int s = 0;
        for (int k = 0; k < 4; k++) {
          la |= a[tx * 4 + k];
          ll |= l[ty * 4 + k];
          s += (a[tx * 4 + k] >> 6) - 1 + (l[ty * 4 + k] >> 6) - 1;
        }
        static const uint8_t kTbl[5][5] = {
            {1, 2, 2, 2, 3}, {2, 4, 4, 4, 5}, {2, 4, 4, 4, 5}, {2, 4, 4, 4, 5}, {3, 5, 5, 5, 6}};
        const int sk = kTbl[(la & 0x3f) < 4 ? (la & 0x3f) : 4][(ll & 0x3f) < 4 ? (ll & 0x3f) : 4];
        const int ds = (s != 0) + (s > 0);
        or_fwd_txfm_quant(resid.data(), MT_TX_DCT_DCT, 16, q, qm, cf.data(), tf.data());
        or_trellis_optimize_ctx(cf.data(), tf.data(), dcq, acq, scan, 16, p->trellis_lambda0, cd, ds, qm,
                                q->qm_level, p->band_tilt);
        or_inv_txfm_dequant(cf.data(), MT_TX_DCT_DCT, 16, q, qm, rr.data());
        const uint16_t pos[2] = {(uint16_t)bx, (uint16_t)by};
        int64_t sse = 0;
        or_sse_recon(src, p->stride, vis_w, vis_h, p->bd, pos, pred.data(), rr.data(), 1, 16, 16, p->wsse_scale, &sse);
        dist += (float)sse * 2.775f;
        sse_sum += sse;
        // the DCT_DCT symbol of the TX_16X16 intra set is 1
        bits += or_real_block_bits_bounded(cf.data(), scan, 16, 16, cd, sk, ds, jb.mode, 1, p->use_skip_bits,
                                           p->skip_bits[sk], INFINITY);
        const uint8_t rc = or_coef_res_ctx(cf.data(), scan, 256);
        memset(a + tx * 4, rc, 4);
        memset(l + ty * 4, rc, 4);
        for (int y = 0; y < 16; y++)
          for (int x = 0; x < 16; x++)
            work[(size_t)(by + y) * p->stride + bx + x] = (uint16_t)clampi(pred[y * 16 + x] + rr[y * 16 + x], 0, maxv);
        if (cf_out) memcpy(cf_out + (size_t)i * 4096 + (ty * 4 + tx) * 256, cf.data(), 256 * sizeof(int32_t));
      }
    float total = mlam * jb.mode_bits;
    if (directional) total += mlam * jb.delta_bits;
    total = total + (dist + mlam * bits);
    total = total + mlam * jb.depth_bits;
    r->total = total;
    r->dist = dist;
    r->bits = bits;
    r->sse = sse_sum;
    for (int y = 0; y < 64; y++)  // the next job predicts from the input reconstruction
      memcpy(&work[(size_t)(jb.py + y) * p->stride + jb.px], &recon[(size_t)(jb.py + y) * p->stride + jb.px], 128);
  }
  return MT_OK;
}

// block32.rs:776-836 pick_luma32's mode-loop candidates.
int or_leaf32(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
              const uint8_t* qm, const mt_coef_cdfs* cd, const mt_leaf8_job* jobs, int32_t n, mt_leaf8_result* results,
              int32_t* cf_out, uint16_t* rec_out) {
  return leaf_impl(32, src, recon, p, q, qm, cd, jobs, n, 0, results, cf_out, rec_out);
}

}  // extern "C"
