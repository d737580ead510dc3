// Device 16x16 luma candidate chain (the 16x16 arm of rd_cost_square,
// src/coder/partition_search.rs:620-673): prediction -> residual -> forward
// transform + quantisation (+QM) -> trellis_optimize over the 16x16 default scan
// -> inverse -> SATD bridge distortion -> TX_16X16 coefficient rate + mode bits
// -> rd cost.  One candidate per thread, the same arithmetic order as the 8x8
// chain; working arrays in one per-thread arena (Work16).
#pragma once
#include <stdint.h>

#include "chain8.cuh"
#include "txfm16.cuh"

namespace mtd {

// The 16x16 default scan (src/coef_q.rs SCAN_16X16); coefficient indices
// are column-major (rc = y + 16 x).
__constant__ uint16_t kScan16[256] = {MT_SCAN_16X16_LIST};

// trellis_optimize (src/trellis.rs:944-1030) over an N-coefficient scan
// (scan(i): the coefficient index of scan position i): step A in
// the pinned AVX2 chunking (8-wide chunks, one 4-wide chunk, scalar tail; a
// chunk holding a level >= 64 takes the scalar form in all lanes), the exact
// right-to-left suffix sums of the zeroing distortion, and the EOB search.
// `suf` is scratch for N + 1 floats.  Returns the final EOB scan index.
template <int N, typename S, typename C>
__device__ int trellis_sq(C* cf, const float* tf, float* suf, float dc_q, float ac_q, float lambda, const float* lut,
                          S scan) {
  const float dq2 = __fmul_rn(dc_q, dc_q), aq2 = __fmul_rn(ac_q, ac_q);
  int eob_idx = -1;
#pragma unroll 8
  for (int i = 0; i < N; i++)
    if (cf[scan(i)] != 0) eob_idx = i;
  const int m = eob_idx + 1;
  const int M = warp_max(m);
  if (m == 0) return -1;
  const int full8 = m & ~7;
  const bool has4 = (m - full8) >= 4;
  for (int base = 0; base < M; base += 8) {
    if (base >= m) continue;
    const int W = base < full8 ? 8 : (has4 ? 4 : 0);
    if (W > 0) {
      // One chunk: levels and targets read first; the decisions use the
      // values at the start of the chunk.
      int32_t c[8];
      float at[8];
      int rc[8];
      bool big = false;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        if (k < W) {
          rc[k] = scan(base + k);
          c[k] = cf[rc[k]];
          at[k] = fabsf(tf[rc[k]]);
          big |= uabs(c[k]) > 63u;
        }
      }
#pragma unroll
      for (int k = 0; k < 8; k++) {
        if (k >= W) break;
        const float q2 = rc[k] == 0 ? dq2 : aq2;
        bool dn;
        if (big) {
          dn = c[k] != 0 && round_down_plain(at[k], uabs(c[k]), q2, lambda);
        } else {
          const int32_t li = (int32_t)uabs(c[k]), ldi = max(li - 1, 0);
          const float el = __fsub_rn(at[k], (float)li), ed = __fsub_rn(at[k], (float)ldi);
          const float cl = __fmaf_rn(q2, __fmul_rn(el, el), __fmul_rn(lambda, lut[li]));
          const float cd = __fmaf_rn(q2, __fmul_rn(ed, ed), __fmul_rn(lambda, lut[ldi]));
          dn = cd < cl;
        }
        if (dn && c[k] != 0) cf[rc[k]] = (C)(c[k] < 0 ? c[k] + 1 : c[k] - 1);
      }
    }
    if (base >= full8) {
      // The scalar tail after the last full chunk (and the 4-wide one).
      const int s = base + (has4 ? 4 : 0);
      for (int k = 0; k < 4; k++) {
        const int e = s + k;
        if (e >= m) break;
        const int r = scan(e);
        const int32_t v = cf[r];
        if (v != 0 && round_down_plain(fabsf(tf[r]), uabs(v), r == 0 ? dq2 : aq2, lambda))
          cf[r] = (C)(v < 0 ? v + 1 : v - 1);
      }
    }
  }
  suf[m] = 0.0f;
  float acc = 0.0f;
  for (int e = M - 1; e >= 0; e--) {
    if (e >= m) continue;
    const int rc = scan(e);
    const float at = fabsf(tf[rc]);
    acc = __fadd_rn(acc, __fmul_rn(rc == 0 ? dq2 : aq2, __fmul_rn(at, at)));
    suf[e] = acc;
  }
  int best_e = -1;
  float best = __int_as_float(0x7f800000);
  float pre = 0.0f;
  for (int e = 0; e < M; e++) {
    if (e >= m) continue;
    const int rc = scan(e);
    const float at = fabsf(tf[rc]);
    const uint32_t l = uabs(cf[rc]);
    const float ecur = __fsub_rn(at, (float)l);
    const float dcur = __fmul_rn(rc == 0 ? dq2 : aq2, __fmul_rn(ecur, ecur));
    const float base_c = __fadd_rn(pre, dcur);
    if (l != 0) {
      const int bin = e < 2 ? e : 32 - __clz(e);
      const int extra = bin > 1 ? bin - 2 : 0;
      const float sig = __fadd_rn(__fmul_rn((float)bin, 0.9f), __fadd_rn((float)extra, 2.0f));
      const float c = __fadd_rn(__fadd_rn(base_c, __fmul_rn(lambda, sig)), suf[e + 1]);
      if (c < best) {
        best = c;
        best_e = e;
      }
    }
    pre = __fadd_rn(base_c, __fmul_rn(lambda, l < 64 ? lut[l] : coef_rate_bits(l)));
  }
  const float skip = __fadd_rn(suf[0], lambda);
  const int keep = (best_e < 0 || skip < best) ? 0 : best_e + 1;
  for (int e = 0; e < M; e++)
    if (e >= keep && e < m) cf[scan(e)] = 0;
  return keep - 1;
}

// The 16x16 default scan as trellis_sq's accessor.
struct Scan16 {
  __device__ __forceinline__ int operator()(int i) const { return kScan16[i]; }
};

// trellis_optimize over the 16x16 scan; `suf` is scratch for 257 floats.
template <typename C>
__device__ __forceinline__ int trellis16(C* cf, const float* tf, float* suf, float dc_q, float ac_q, float lambda,
                                         const float* lut) {
  return trellis_sq<256>(cf, tf, suf, dc_q, ac_q, lambda, lut, Scan16{});
}

// Coefficient bits of a 16x16 luma block (src/rate.rs:149-291), float
// additions in the reference's order; the level map has the reference's
// stride 16 (column-major, reads past a column land in the next one or in the
// zeroed tail), kept in the 324-byte scratch `lv`.
template <typename C>
__device__ float rate16(const C* cf, int eob, const mt_coef_costs& T, int skip_ctx, int dcs, int mode, int tx,
                        bool use_skip_bits, float skip1, float skip0, uint8_t* lv) {
  const int E = warp_max(eob);
  if (eob < 0) return use_skip_bits ? skip1 : T.txb_skip[skip_ctx][1];
  float bits = use_skip_bits ? skip0 : T.txb_skip[skip_ctx][0];
  bits = __fadd_rn(bits, T.txtp[mode][tx]);
  const float* dcs_c = T.dc_sign[dcs];
  if (eob == 0) {
    const uint32_t m = uabs(cf[0]), mm = min(m, 3u);
    bits = __fadd_rn(bits, T.eob_bin[0]);
    bits = __fadd_rn(bits, T.eob_base[0][mm - 1]);
    if (mm == 3) {
      float h = T.br_cum[0][min((int32_t)m - 3, 12)];
      if (m >= 15) h = __fadd_rn(h, golomb_cost(m - 15));
      bits = __fadd_rn(bits, h);
    }
    return __fadd_rn(bits, dcs_c[cf[0] < 0]);
  }
  const int eob_bin = eob < 2 ? eob : 32 - __clz(eob);
  bits = __fadd_rn(bits, T.eob_bin[eob_bin]);
  if (eob_bin > 1) {
    const int nb = eob_bin - 2;
    bits = __fadd_rn(bits, T.eob_hi[eob_bin][(eob >> nb) & 1]);
    bits = __fadd_rn(bits, (float)nb);
  }
  uint32_t* lv32 = reinterpret_cast<uint32_t*>(lv);
#pragma unroll 9
  for (int i = 0; i < 81; i++) lv32[i] = 0;
  const int ctx_e = 1 + (eob > 32) + (eob > 64);
  {
    const int rc = kScan16[eob];
    const int ex = rc >> 4, ey = rc & 15;
    const uint32_t m = uabs(cf[rc]);
    const uint32_t tok = min(m, 3u) - 1;
    bits = __fadd_rn(bits, T.eob_base[ctx_e][tok]);
    if (tok == 2) {
      float h = T.br_cum[(ex | ey) > 1 ? 14 : 7][min((int32_t)m - 3, 12)];
      if (m >= 15) h = __fadd_rn(h, golomb_cost(m - 15));
      bits = __fadd_rn(bits, h);
    }
    lv[rc] = (uint8_t)level_byte(m);
  }
  int ac_nz = 1;
  for (int i = E - 1; i >= 1; i--) {
    if (i >= eob) continue;
    const int rc = kScan16[i];
    const int x = rc >> 4, y = rc & 15;
    const uint32_t hm = (uint32_t)lv[rc + 1] + lv[rc + 16] + lv[rc + 17];
    const uint32_t mag = hm + lv[rc + 2] + lv[rc + 32];
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
    lv[rc] = (uint8_t)level_byte(m);
    ac_nz += m != 0;
  }
  const uint32_t dm = uabs(cf[0]), dtok = min(dm, 3u);
  bits = __fadd_rn(bits, T.base_tok[0][dtok]);
  if (dtok == 3) {
    const uint32_t mag = ((uint32_t)lv[1] + lv[16] + lv[17]) & 63;
    float h = T.br_cum[mag > 12 ? 6 : (int)((mag + 1) >> 1)][min((int32_t)dm - 3, 12)];
    if (dm >= 15) h = __fadd_rn(h, golomb_cost(dm - 15));
    bits = __fadd_rn(bits, h);
  }
  if (cf[0] != 0) bits = __fadd_rn(bits, dcs_c[cf[0] < 0]);
  for (int k = 0; k < ac_nz; k++) bits = __fadd_rn(bits, 1.0f);
  return bits;
}

// Hadamard 4x4 SATD of src - clamp(pred + resid) over the 16 tiles of a 16x16
// block (src/partition_rd.rs:86-133).
template <bool MASK, typename P, typename R>
__device__ uint32_t satd16(const uint16_t* __restrict__ src, int stride, int px, int py, const P* pred, const R* rr,
                           int32_t maxv, int vw, int vh) {
  uint32_t satd = 0;
#pragma unroll 1
  for (int tile = 0; tile < 16; tile++) {
    const int ty = (tile >> 2) * 4, tx = (tile & 3) * 4;
    int32_t r[4][4];
#pragma unroll
    for (int y = 0; y < 4; y++) {
      int32_t d[4];
#pragma unroll
      for (int x = 0; x < 4; x++) {
        const int i = (ty + y) * 16 + tx + x;
        d[x] = (!MASK || (tx + x < vw && ty + y < vh))
                   ? (int32_t)src[(size_t)(py + ty + y) * stride + px + tx + x] - clampi(pred[i] + rr[i], 0, maxv)
                   : 0;
      }
      const int32_t e = d[0] + d[2], f = d[0] - d[2], g = d[1] + d[3], h = d[1] - d[3];
      r[y][0] = e + g;
      r[y][1] = f + h;
      r[y][2] = f - h;
      r[y][3] = e - g;
    }
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const int32_t e = r[0][x] + r[2][x], f = r[0][x] - r[2][x], g = r[1][x] + r[3][x], h = r[1][x] - r[3][x];
      satd += uabs(e + g) + uabs(f + h) + uabs(f - h) + uabs(e - g);
    }
  }
  return satd;
}

// A 16x16 candidate outside the frame or the tables (V/H_DCT have no 16x16
// intra use here) is not evaluated.
__device__ __forceinline__ bool cand16_ok(const mt_candidate& c, int fw, int fh) {
  return c.px + 16 <= fw && c.py + 16 <= fh && c.mode <= MT_PAETH_PRED && c.tx_type <= MT_TX_DCT_ADST &&
         c.tx_type != MT_TX_V_DCT && c.tx_type != MT_TX_H_DCT && c.dcs_ctx < 3 && c.skip_ctx < 13 &&
         c.angle_delta >= -3 && c.angle_delta <= 3;
}

// Per-thread arena (32-bit words): [0,256) tf | [256,513) suf, also the int32
// transform scratch and the u8 level map | [513,641) pred | [641,769) rr |
// [769,897) cf.  During prediction [0,210) holds the two edges and the filter
// temporary.
constexpr int kWork16Words = 897;
static_assert(3 * edge_cap<16>() <= 256, "prediction scratch fits the tf region");
struct Work16 {
  int32_t* w;
  __device__ __forceinline__ float* tf() { return reinterpret_cast<float*>(w); }
  __device__ __forceinline__ float* suf() { return reinterpret_cast<float*>(w + 256); }
  __device__ __forceinline__ int32_t* edges() { return w; }
  __device__ __forceinline__ int16_t* pred() { return reinterpret_cast<int16_t*>(w + 513); }
  __device__ __forceinline__ int16_t* rr() { return reinterpret_cast<int16_t*>(w + 641); }
  __device__ __forceinline__ int16_t* cf() { return reinterpret_cast<int16_t*>(w + 769); }
};

// One whole 16x16 candidate.  `qs` holds fwd_qm_scale of the 256 QM weights.
template <bool VIS>
__device__ __forceinline__ void chain16_one(const uint16_t* __restrict__ src, const uint16_t* __restrict__ rec,
                                            const mt_chain_params& p, const mt_quant& q, float trellis_lambda,
                                            const uint8_t* qm, const float* qs, const float* lut,
                                            const mt_coef_costs& T, const mt_candidate& cd, mt_candidate_result& r,
                                            Work16& w) {
  const int32_t maxv = (1 << p.bd) - 1;
  int16_t* pred = w.pred();
  int16_t* cf = w.cf();
  int16_t* rr = w.rr();
  float* tf = w.tf();
  predict_sq<16>(rec, p.stride, p.frame_w, p.frame_h, cd.px, cd.py, cd.mode, cd.angle_delta, cd.flags & 1,
                 (cd.flags >> 1) & 1, (cd.flags >> 2) & 1, p.bd, pred, w.edges());
#pragma unroll 2
  for (int y = 0; y < 16; y++)
#pragma unroll
    for (int x = 0; x < 16; x++)
      rr[y * 16 + x] = (int16_t)((int32_t)src[(size_t)(cd.py + y) * p.stride + cd.px + x] - pred[y * 16 + x]);
  const int TX = cd.tx_type;
  fwd16x16(rr, TX, q, cf, tf, reinterpret_cast<int32_t*>(w.suf()));
  if (TX != MT_TX_IDTX && qm) apply_qm(cf, tf, qs, 256);
  int eob;
  if (p.trellis_lambda0 > 0.0f && !(cd.flags & MT_CAND_NO_TRELLIS)) {
    eob = trellis16(cf, tf, w.suf(), (float)q.dc_q, (float)q.ac_q, trellis_lambda, lut);
  } else {
    eob = -1;
    for (int i = 0; i < 256; i++)
      if (cf[kScan16[i]] != 0) eob = i;
  }
  inv16x16(cf, TX, q, qm, rr, reinterpret_cast<int32_t*>(w.suf()));
  const int vw = vis_extent(p.vis_w, p.frame_w, cd.px), vh = vis_extent(p.vis_h, p.frame_h, cd.py);
  // VIS: the frame is displayed smaller than coded; samples past the
  // displayed edge carry no distortion.
  const uint32_t satd = satd16<VIS>(src, p.stride, cd.px, cd.py, pred, rr, maxv, vw, vh);
  const float qstep = (float)q.ac_q;
  float price = __fmul_rn(__fmul_rn(__fmul_rn((float)satd, fmaxf(qstep, 1.0f)), 0.25f), p.satd_scale);
  if (p.satd_bridge != 0.0f) price = __fmul_rn(price, p.satd_bridge);
  const float cbits = rate16(cf, eob, T, cd.skip_ctx, cd.dcs_ctx, cd.mode, TX, p.use_skip_bits != 0, p.skip_bits[0],
                             p.skip_bits[1], reinterpret_cast<uint8_t*>(w.suf()));
  // (luma_bits + mode_bits) + extra_bits; adding 0 leaves the sum as is.
  const float bits = __fadd_rn(__fadd_rn(cbits, cd.mode_bits), cd.extra_bits);
  r.distortion = price;
  r.bits = bits;
  r.cost = __fadd_rn(price, __fmul_rn(p.mode_lambda, bits));
  r.satd = satd;
  r.eob = eob;
  r.reserved[0] = r.reserved[1] = r.reserved[2] = 0;
}

}  // namespace mtd
