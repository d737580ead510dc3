// Device functions of the 8x8 luma candidate chain (the per-candidate body of
// the reference's luma mode search, src/coder/partition_search.rs:467-530):
//   predict -> residual -> forward transform + quantisation (+QM)
//   -> trellis_optimize -> dequantisation + inverse transform
//   -> SATD distortion (luma_partition_distortion) and coefficient rate
//   -> rd_cost = D + lambda * (bits + mode bits).
//
// Execution model: one thread evaluates one candidate; launches arrange the
// candidates so that a warp runs one (mode, transform type) pair over 32
// blocks.  Every loop over scan positions runs on a warp-uniform index (the
// warp maximum of the per-lane bound, lanes past their own bound predicated
// off), so scan tables are constant-cache broadcasts and the per-thread
// arrays are read and written with the same offset in every lane (coalesced
// local memory).
#pragma once
#include <stdint.h>

#include "intrapred.cuh"
#include "txfm8.cuh"

namespace mtd {

// Default 8x8 scan (scan index -> rc = x*8 + y) and its inverse.
__constant__ uint8_t kScan8[64] = {0,  8,  1,  2,  9,  16, 24, 17, 10, 3,  4,  11, 18, 25, 32, 40,
                                   33, 26, 19, 12, 5,  6,  13, 20, 27, 34, 41, 48, 56, 49, 42, 35,
                                   28, 21, 14, 7,  15, 22, 29, 36, 43, 50, 57, 58, 51, 44, 37, 30,
                                   23, 31, 38, 45, 52, 59, 60, 53, 46, 39, 47, 54, 61, 62, 55, 63};
__constant__ uint8_t kIScan8[64] = {0,  2,  3,  9,  10, 20, 21, 35, 1,  4,  8,  11, 19, 22, 34, 36,
                                    5,  7,  12, 18, 23, 33, 37, 48, 6,  13, 17, 24, 32, 38, 47, 49,
                                    14, 16, 25, 31, 39, 46, 50, 57, 15, 26, 30, 40, 45, 51, 56, 58,
                                    27, 29, 41, 44, 52, 55, 59, 62, 28, 42, 43, 53, 54, 60, 61, 63};
// Coefficient-base position offsets for square transforms, [min(y,4)][min(x,4)].
__constant__ uint8_t kLoCtxOff[25] = {0, 1, 6, 6, 21, 1, 6, 6, 21, 21, 6, 6, 21, 21, 21,
                                      6, 21, 21, 21, 21, 21, 21, 21, 21, 21};
// Static per-level trellis rate (src/cost.rs:70-75).
__constant__ float kCoefRateLut[64] = {
    0.9f,  2.7f,  3.6f,  5.3f,  5.3f,  5.3f,  6.6f,  6.6f,  6.6f,  7.9f,  7.9f,  7.9f,  9.2f,
    9.2f,  9.2f,  11.5f, 13.5f, 13.5f, 15.5f, 15.5f, 15.5f, 15.5f, 17.5f, 17.5f, 17.5f, 17.5f,
    17.5f, 17.5f, 17.5f, 17.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f,
    19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f,
    21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f};

// Warp maximum over the lanes currently executing this call site; every lane
// gets a bound >= its own value.
__device__ __forceinline__ int warp_max(int v) { return __reduce_max_sync(__activemask(), v); }

// Static per-level bit estimate (src/cost.rs:50-68); >= 64 takes the closed form.
__device__ __forceinline__ float coef_rate_bits(uint32_t level) {
  if (level < 64) return kCoefRateLut[level];
  float b = 4.0f;
  const int32_t total_br = min((int32_t)level - 3, 12);
  b = __fadd_rn(b, __fmul_rn((float)(total_br / 3 + 1), 1.3f));
  if (level >= 15) b = __fadd_rn(b, __fadd_rn(__fmul_rn(2.0f, (float)(32 - __clz(level - 15 + 1))), -1.0f));
  return b;
}
__device__ __forceinline__ float golomb_cost(uint32_t v) { return (float)(2 * (32 - __clz(v + 1)) - 1); }
// The byte the coefficient coder keeps per position (src/tables.rs:365-373).
__device__ __forceinline__ uint32_t level_byte(uint32_t m) {
  return m == 0 ? 0u : (m <= 2 ? m * 0x41u : min(m, 15u) + 0xC0u);
}

// Round-down decision of one coefficient: the AVX2 FMA lane form
// (src/avx/trellis.rs:79-118) or the scalar form (src/avx/trellis.rs:139-161).
__device__ __forceinline__ bool round_down_fma(float at, int32_t li, float q2, float lambda) {
  const int32_t ldi = max(li - 1, 0);
  const float el = __fsub_rn(at, (float)li), ed = __fsub_rn(at, (float)ldi);
  const float cl = __fmaf_rn(q2, __fmul_rn(el, el), __fmul_rn(lambda, kCoefRateLut[li]));
  const float cd = __fmaf_rn(q2, __fmul_rn(ed, ed), __fmul_rn(lambda, kCoefRateLut[ldi]));
  return cd < cl;
}
__device__ __forceinline__ bool round_down_plain(float at, uint32_t l, float q2, float lambda) {
  const float el = __fsub_rn(at, (float)l), ed = __fsub_rn(at, (float)(l - 1));
  const float cl = __fadd_rn(__fmul_rn(q2, __fmul_rn(el, el)), __fmul_rn(lambda, coef_rate_bits(l)));
  const float cd = __fadd_rn(__fmul_rn(q2, __fmul_rn(ed, ed)), __fmul_rn(lambda, coef_rate_bits(l - 1)));
  return cd < cl;
}

// One chunk of the trellis step A at scan positions [base, base + W).  The
// chunk's levels and targets are read once; decisions use the values at the
// start of the chunk (scan positions are distinct, as in the AVX2 gather).
// `lut` is the static per-level rate table in shared memory (per-lane
// indices, so it must not sit in the constant cache).
template <int W, typename C>
__device__ __forceinline__ void round_down_chunk(C* cf, const float* tf, int base, float dq2, float aq2, float lambda,
                                                 const float* lut) {
  int32_t c[W];
  float at[W];
  int rc[W];
  bool big = false;
#pragma unroll
  for (int k = 0; k < W; k++) {
    rc[k] = kScan8[base + k];
    c[k] = cf[rc[k]];
    at[k] = fabsf(tf[rc[k]]);
    big |= uabs(c[k]) > 63u;
  }
#pragma unroll
  for (int k = 0; k < W; k++) {
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

// trellis_optimize (src/trellis.rs:944-1030) over the 8x8 default scan with
// step A in the pinned AVX2 chunking (8-wide chunks, one 4-wide chunk, scalar
// tail; a chunk holding a level >= 64 takes the scalar form in all lanes).
// `suf` is scratch for 65 floats, `lut` the shared-memory rate table.
// Returns the final EOB scan index (-1 when every level is zero).
template <typename C>
__device__ int trellis8(C* cf, const float* tf, float* suf, float dc_q, float ac_q, float lambda, const float* lut) {
  const float dq2 = __fmul_rn(dc_q, dc_q), aq2 = __fmul_rn(ac_q, ac_q);
  int eob_idx = -1;
#pragma unroll 8
  for (int i = 0; i < 64; i++)
    if (cf[kScan8[i]] != 0) eob_idx = i;
  const int m = eob_idx + 1;
  const int M = warp_max(m);
  if (m == 0) return -1;
  const int full8 = m & ~7;
  const bool has4 = (m - full8) >= 4;
  for (int base = 0; base < M; base += 8) {
    if (base >= m) continue;
    if (base < full8) {
      round_down_chunk<8>(cf, tf, base, dq2, aq2, lambda, lut);
    } else {
      int s = base;
      if (has4) {
        round_down_chunk<4>(cf, tf, base, dq2, aq2, lambda, lut);
        s += 4;
      }
      for (int k = 0; k < 4; k++) {
        const int e = s + k;
        if (e >= m) break;
        const int rc = kScan8[e];
        const int32_t c = cf[rc];
        if (c != 0 && round_down_plain(fabsf(tf[rc]), uabs(c), rc == 0 ? dq2 : aq2, lambda))
          cf[rc] = (C)(c < 0 ? c + 1 : c - 1);
      }
    }
  }
  // Suffix sums of the zeroing distortion in exact right-to-left order.
  suf[m] = 0.0f;
  float acc = 0.0f;
  for (int e = M - 1; e >= 0; e--) {
    if (e >= m) continue;
    const int rc = kScan8[e];
    const float at = fabsf(tf[rc]);
    acc = __fadd_rn(acc, __fmul_rn(rc == 0 ? dq2 : aq2, __fmul_rn(at, at)));
    suf[e] = acc;
  }
  int best_e = -1;
  float best = __int_as_float(0x7f800000);
  float pre = 0.0f;
  for (int e = 0; e < M; e++) {
    if (e >= m) continue;
    const int rc = kScan8[e];
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
    if (e >= keep && e < m) cf[kScan8[e]] = 0;
  return keep - 1;
}

// Coefficient bits of an 8x8 luma block (src/rate.rs:149-291) from the
// host-built bit costs, float additions in the reference's order, with the
// reference's level map (stride 8, reads past the 8x8 plane land in the
// zeroed tail) kept in the 80-byte scratch `lv`.
template <typename C>
__device__ float rate8(const C* cf, int eob, const mt_coef_costs& T, int skip_ctx, int dcs, int mode, int tx,
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
#pragma unroll
  for (int i = 0; i < 20; i++) lv32[i] = 0;
  const int ctx_e = 1 + (eob > 8) + (eob > 16);
  {
    const int rc = kScan8[eob];
    const int ex = rc >> 3, ey = rc & 7;
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
    const int rc = kScan8[i];
    const int x = rc >> 3, y = rc & 7;
    const uint32_t hm = (uint32_t)lv[rc + 1] + lv[rc + 8] + lv[rc + 9];
    const uint32_t mag = hm + lv[rc + 2] + lv[rc + 16];
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
    const uint32_t mag = ((uint32_t)lv[1] + lv[8] + lv[9]) & 63;
    float h = T.br_cum[mag > 12 ? 6 : (int)((mag + 1) >> 1)][min((int32_t)dm - 3, 12)];
    if (dm >= 15) h = __fadd_rn(h, golomb_cost(dm - 15));
    bits = __fadd_rn(bits, h);
  }
  if (cf[0] != 0) bits = __fadd_rn(bits, dcs_c[cf[0] < 0]);
  for (int k = 0; k < ac_nz; k++) bits = __fadd_rn(bits, 1.0f);
  return bits;
}

// Visible columns (rows) of a block at p: the displayed size (0 = the padded
// frame) minus the block origin; samples past it are masked to the
// reconstruction (zero error), as the reference's SrcBlock does.
__device__ __forceinline__ int vis_extent(int vis, int frame, int p) { return (vis > 0 ? vis : frame) - p; }

#ifndef MT_SATD_UNROLL
#define MT_SATD_UNROLL 1
#endif
constexpr int kSatdUnroll = MT_SATD_UNROLL;

// Hadamard 4x4 SATD of src - clamp(pred + resid) (src/partition_rd.rs:86-133).
template <bool MASK, typename P, typename R>
__device__ __forceinline__ uint32_t satd8(const uint16_t* __restrict__ src, int stride, int px, int py, const P* pred,
                                          const R* rr, int32_t maxv, int vw, int vh) {
  uint32_t satd = 0;
#pragma unroll kSatdUnroll
  for (int ty = 0; ty < 8; ty += 4)
#pragma unroll kSatdUnroll
    for (int tx = 0; tx < 8; tx += 4) {
      int32_t r[4][4];
#pragma unroll
      for (int y = 0; y < 4; y++) {
        int32_t d[4];
#pragma unroll
        for (int x = 0; x < 4; x++) {
          const int i = (ty + y) * 8 + tx + x;
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

// A candidate whose block, mode, type or contexts fall outside the frame or
// the tables is not evaluated; its result carries eob = MT_EOB_INVALID.
__device__ __forceinline__ bool cand_ok(const mt_candidate& c, int fw, int fh) {
  return c.px + 8 <= fw && c.py + 8 <= fh && c.mode <= MT_PAETH_PRED && c.tx_type <= MT_TX_DCT_ADST &&
         c.angle_delta >= -3 && c.angle_delta <= 3 && c.dcs_ctx < 3 && c.skip_ctx < 13;
}

// Per-thread working set of one 8x8 candidate: a view onto ONE block of
// kWork8Words 32-bit words (a single local array, or one thread's slice of a
// shared-memory arena).  NVVM -O3 (CUDA 12.9, sm_100a) was seen to give two
// separate per-thread local arrays that are both live across an inlined
// transform the same slot (the residual input and the level output); one
// allocation cannot be split that way.  Sample-domain arrays are int16: for
// 8-bit video every prediction, residual, level and inverse output fits.
// Layout (words): [0,64) tf | [64,132) suf, later the rate walk's level map |
// [132,164) pred | [164,196) rr | [196,228) cf.  During prediction, before
// tf and suf are live, [0,114) holds the two edges and the filter temporary.
constexpr int kWork8Words = 228;
struct Work8 {
  int32_t* w;
  __device__ __forceinline__ float* tf() { return reinterpret_cast<float*>(w); }
  __device__ __forceinline__ float* suf() { return reinterpret_cast<float*>(w + 64); }
  __device__ __forceinline__ int32_t* edges() { return w; }
  __device__ __forceinline__ int16_t* pred() { return reinterpret_cast<int16_t*>(w + 132); }
  __device__ __forceinline__ int16_t* rr() { return reinterpret_cast<int16_t*>(w + 164); }
  __device__ __forceinline__ int16_t* cf() { return reinterpret_cast<int16_t*>(w + 196); }
};

// Evaluate one candidate.  Leaves the final levels (column-major) in w.cf(),
// the prediction in w.pred() and the inverse residual in w.rr().  (Compiling
// one path per transform type raised register use to the cap and was no
// faster, so the type stays a run-time value.)
// Prediction of candidate cd into w.pred() (it depends on the mode, angle
// delta and neighbour flags only, not on the transform type).
__device__ __forceinline__ void chain8_predict(const uint16_t* __restrict__ rec, const mt_chain_params& p,
                                               const mt_candidate& cd, Work8& w) {
  predict8(rec, p.stride, p.frame_w, p.frame_h, cd.px, cd.py, cd.mode, cd.angle_delta, cd.flags & 1,
           (cd.flags >> 1) & 1, (cd.flags >> 2) & 1, p.bd, w.pred(), w.edges());
}

// The rest of the chain for candidate cd from the prediction in w.pred()
// (left intact, so several transform types can share one prediction).
template <bool VIS>
__device__ __forceinline__ void chain8_tx(const uint16_t* __restrict__ src, const mt_chain_params& p,
                                          const mt_quant& q, float trellis_lambda, const uint8_t* qm,
                                          const float* qs, const float* lut, const mt_coef_costs& T,
                                          const mt_candidate& cd, mt_candidate_result& r, Work8& w) {
  const int32_t maxv = (1 << p.bd) - 1;
  int16_t* pred = w.pred();
  int16_t* cf = w.cf();
  int16_t* rr = w.rr();
  float* tf = w.tf();
#pragma unroll
  for (int y = 0; y < 8; y++)
#pragma unroll
    for (int x = 0; x < 8; x++)
      rr[y * 8 + x] = (int16_t)((int32_t)src[(size_t)(cd.py + y) * p.stride + cd.px + x] - pred[y * 8 + x]);
  const int TX = cd.tx_type;
  fwd8x8(rr, TX, q, cf, tf, reinterpret_cast<int32_t*>(w.suf()));
  const bool two_d = TX == MT_TX_DCT_DCT || TX >= MT_TX_ADST_ADST;
  if (two_d && qm) apply_qm(cf, tf, qs, 64);
  int eob;
  if (p.trellis_lambda0 > 0.0f && !(cd.flags & MT_CAND_NO_TRELLIS)) {
    eob = trellis8(cf, tf, w.suf(), (float)q.dc_q, (float)q.ac_q, trellis_lambda, lut);
  } else {
    eob = -1;
    for (int i = 0; i < 64; i++)
      if (cf[kScan8[i]] != 0) eob = i;
  }
  inv8x8(cf, TX, q, qm, rr, reinterpret_cast<int32_t*>(w.suf()));
  const int vw = vis_extent(p.vis_w, p.frame_w, cd.px), vh = vis_extent(p.vis_h, p.frame_h, cd.py);
  // VIS: the frame is displayed smaller than coded; samples past the
  // displayed edge carry no distortion.
  const uint32_t satd = satd8<VIS>(src, p.stride, cd.px, cd.py, pred, rr, maxv, vw, vh);
  const float qstep = (float)q.ac_q;
  float price = __fmul_rn(__fmul_rn(__fmul_rn((float)satd, fmaxf(qstep, 1.0f)), 0.25f), p.satd_scale);
  if (p.satd_bridge != 0.0f) price = __fmul_rn(price, p.satd_bridge);
  const float cbits = rate8(cf, eob, T, cd.skip_ctx, cd.dcs_ctx, cd.mode, TX, p.use_skip_bits != 0, p.skip_bits[0],
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

template <bool VIS>
__device__ __forceinline__ void chain8_one(const uint16_t* __restrict__ src, const uint16_t* __restrict__ rec,
                                           const mt_chain_params& p, const mt_quant& q, float trellis_lambda,
                                           const uint8_t* qm, const float* qs, const float* lut,
                                           const mt_coef_costs& T, const mt_candidate& cd, mt_candidate_result& r,
                                           Work8& w) {
  chain8_predict(rec, p, cd, w);
  chain8_tx<VIS>(src, p, q, trellis_lambda, qm, qs, lut, T, cd, r, w);
}

}  // namespace mtd
