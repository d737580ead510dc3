// Oracle (test-only checker of the CUDA path): the 16x16 leaf's chroma
// searches with the shipped tuning -- pick_uv16_420
// (src/coder/block16.rs:980-1381: uv16_joint on, uv8_joint_k from the params)
// and pick_uv16_444 (:437-978: no palette outside screen content,
// uv16_444_mlam_c off), and the 32x32 leaf's pick_uv32_420
// (src/coder/block32.rs:2797-3120), both with cfl_alpha_rd_steps 0 so cfl_alpha_rd_refine
// returns the closed-form alpha (src/cost.rs:332-341) -- and uv_mode_bits
// (src/coder/lossy_state.rs:1302-1349) priced straight from the CDFs with
// cdf_cost.  Composed of the oracle's own
// primitives: the intra predictors, the 8x8 / 16x16 forward transforms with
// the QM, trellis_optimize_ctx / trellis_optimize, the dav1d inverses, sse_recon, the rate walk and the
// CfL alpha search.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <tuple>
#include <vector>

#include "oracle.h"

namespace {

inline bool directional(int m) { return m >= MT_V_PRED && m <= MT_D67_PRED; }

// chroma_tx_for_mode (src/coder/chroma_tx.rs:46-66).
int chroma_tx(int m) {
  switch (m) {
    case MT_PAETH_PRED:
    case MT_SMOOTH_PRED:
    case MT_D135_PRED:
      return MT_TX_ADST_ADST;
    case MT_SMOOTH_V_PRED:
    case MT_V_PRED:
    case MT_D113_PRED:
    case MT_D67_PRED:
      return MT_TX_ADST_DCT;
    case MT_SMOOTH_H_PRED:
    case MT_H_PRED:
    case MT_D157_PRED:
    case MT_D203_PRED:
      return MT_TX_DCT_ADST;
    default:
      return MT_TX_DCT_DCT;
  }
}

// satd_sad_proxy (src/rd_sse.rs:559-589, :1143-1176) of an n x n block (n a
// multiple of 4): the samples past the displayed extent (vw x vh) take the
// prediction's value.
uint64_t satd_sad_proxy_n(const uint16_t* src, int stride, const int32_t* pred, int n, int vw, int vh) {
  uint64_t sad = 0, satd = 0;
  for (int ty = 0; ty < n; ty += 4)
    for (int tx = 0; tx < n; tx += 4) {
      int32_t rows[4][4];
      for (int r = 0; r < 4; r++) {
        int32_t d[4];
        for (int x = 0; x < 4; x++) {
          const bool vis = tx + x < vw && ty + r < vh;
          d[x] = vis ? (int32_t)src[(size_t)(ty + r) * stride + tx + x] - pred[(ty + r) * n + tx + x] : 0;
          sad += (uint64_t)(d[x] < 0 ? -d[x] : d[x]);
        }
        const int32_t e = d[0] + d[2], f = d[0] - d[2], g = d[1] + d[3], h = d[1] - d[3];
        rows[r][0] = e + g;
        rows[r][1] = f + h;
        rows[r][2] = f - h;
        rows[r][3] = e - g;
      }
      for (int x = 0; x < 4; x++) {
        const int32_t e = rows[0][x] + rows[2][x], f = rows[0][x] - rows[2][x];
        const int32_t g = rows[1][x] + rows[3][x], h = rows[1][x] - rows[3][x];
        const int32_t v[4] = {e + g, f + h, f - h, e - g};
        for (int k = 0; k < 4; k++) satd += (uint64_t)(v[k] < 0 ? -v[k] : v[k]);
      }
    }
  return sad + (satd >> 2);
}

struct Plane {
  const uint16_t* src;  // plane base
  const uint16_t* rec;
  int sk, ds;
};

// One plane of a candidate (pred given): residual, the transform with the
// QM, chroma_rect_trellis (trellis_optimize_ctx, lossy_state.rs:821-870),
// preserve_dc (rd_sse.rs:759-765) when keep_dc, the inverse, sse_recon and
// chroma_bits (lossy_state.rs:749-811); returns rd_cost_i64 and leaves the
// levels / inverse in cf / rr.
float plane_cost(const mt_split16_params* p, const mt_quant* q, const uint8_t* qm, const mt_coef_cdfs* cd,
                 const Plane& P, int cx, int cy, int tx, bool keep_dc, const int32_t* pred, int32_t* cf,
                 int32_t* rr) {
  int32_t resid[64];
  float tf[64];
  int32_t sum = 0;
  for (int i = 0; i < 64; i++) {
    resid[i] = (int32_t)P.src[(size_t)(cy + i / 8) * p->stride + cx + i % 8] - pred[i];
    sum += resid[i];
  }
  or_fwd_txfm_quant(resid, tx, 8, q, qm, cf, tf);
  or_trellis_optimize_ctx(cf, tf, (float)q->dc_q, (float)q->ac_q, or_default_scan(8), 8, p->trellis_lambda0, cd,
                          P.ds, qm, q->qm_level, p->band_tilt);
  if (keep_dc) {
    const int32_t mean = sum / 64;
    if (cf[0] == 0 && (mean < 0 ? -mean : mean) >= 8) cf[0] = mean > 0 ? 1 : -1;
  }
  or_inv_txfm_dequant(cf, tx, 8, q, qm, rr);
  const int vis_w = p->vis_w > 0 ? p->vis_w : p->frame_w, vis_h = p->vis_h > 0 ? p->vis_h : p->frame_h;
  const uint16_t pos[2] = {(uint16_t)cx, (uint16_t)cy};
  int64_t sse = 0;
  or_sse_recon(P.src, p->stride, vis_w, vis_h, p->bd, pos, pred, rr, 1, 8, 8, p->wsse_scale, &sse);
  const float bits = or_real_block_bits_bounded(cf, or_default_scan(8), 8, 8, cd, P.sk, P.ds, -1, 0, p->use_skip_bits,
                                                p->skip_bits[P.sk], INFINITY);
  return (float)sse + p->rd_lambda * bits;
}

// One N x N plane of a chroma candidate: the transform with the QM, the plain
// trellis_optimize (chroma_rect_trellis outside 4:2:0 / 4:2:2,
// lossy_state.rs:834-838) or, ctx, trellis_optimize_ctx (4:2:0), preserve_dc when keep_dc, the inverse, sse_recon
// and chroma_bits at TX_16X16 (lossy_state.rs:749-811); sse and bits apart.
void plane_cost_n(int N, const mt_split16_params* p, const mt_quant* q, const uint8_t* qm, const mt_coef_cdfs* cd,
                  const Plane& P, int cx, int cy, int tx, bool keep_dc, const int32_t* pred, int32_t* cf, int32_t* rr,
                  int64_t* sse, float* bits, bool ctx = false) {
  const int NN = N * N;
  std::vector<int32_t> resid((size_t)NN);
  std::vector<float> tf((size_t)NN);
  int32_t sum = 0;
  for (int i = 0; i < NN; i++) {
    resid[(size_t)i] = (int32_t)P.src[(size_t)(cy + i / N) * p->stride + cx + i % N] - pred[i];
    sum += resid[(size_t)i];
  }
  or_fwd_txfm_quant(resid.data(), tx, N, q, qm, cf, tf.data());
  if (ctx)  // the 4:2:0 chroma_rect_trellis (lossy_state.rs:821-870)
    or_trellis_optimize_ctx(cf, tf.data(), (float)q->dc_q, (float)q->ac_q, or_default_scan(N), N, p->trellis_lambda0,
                            cd, P.ds, qm, q->qm_level, p->band_tilt);
  else
    or_trellis_optimize(cf, tf.data(), (float)q->dc_q, (float)q->ac_q, or_default_scan(N), NN, p->trellis_lambda0);
  if (keep_dc) {
    const int32_t mean = sum / NN;
    if (cf[0] == 0 && (mean < 0 ? -mean : mean) >= 8) cf[0] = mean > 0 ? 1 : -1;
  }
  or_inv_txfm_dequant(cf, tx, N, q, qm, rr);
  const int vis_w = p->vis_w > 0 ? p->vis_w : p->frame_w, vis_h = p->vis_h > 0 ? p->vis_h : p->frame_h;
  const uint16_t pos[2] = {(uint16_t)cx, (uint16_t)cy};
  *sse = 0;
  or_sse_recon(P.src, p->stride, vis_w, vis_h, p->bd, pos, pred, rr, 1, N, N, p->wsse_scale, sse);
  *bits = or_real_block_bits_bounded(cf, or_default_scan(N), N, N, cd, P.sk, P.ds, -1, 0, p->use_skip_bits,
                                     p->skip_bits[P.sk], INFINITY);
}

inline void plane_cost16(const mt_split16_params* p, const mt_quant* q, const uint8_t* qm, const mt_coef_cdfs* cd,
                         const Plane& P, int cx, int cy, int tx, bool keep_dc, const int32_t* pred, int32_t* cf,
                         int32_t* rr, int64_t* sse, float* bits, bool ctx = false) {
  plane_cost_n(16, p, q, qm, cd, P, cx, cy, tx, keep_dc, pred, cf, rr, sse, bits, ctx);
}

template <int N, typename J>
int pick444(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
            const uint16_t* luma, const mt_split16_params* p, const mt_uv16_params* u, const mt_quant* q,
            const uint8_t* qm, const mt_coef_cdfs* cd, const mt_uv_mode_cdfs* mc, const J* jobs, int32_t n,
            mt_uv16_result* results, int32_t* cf_out, uint16_t* rec_out) {
  constexpr int NN = N * N, U = N / 4;
  if (!p || p->bd != 8) return MT_ERR_UNSUPPORTED;
  const int32_t maxv = (1 << p->bd) - 1;
  const float mlam = p->rd_lambda, dlam = u->dir_lambda;
  const int vis_w = p->vis_w > 0 ? p->vis_w : p->frame_w, vis_h = p->vis_h > 0 ? p->vis_h : p->frame_h;
  static const int kList[12] = {MT_SMOOTH_V_PRED, MT_PAETH_PRED, MT_SMOOTH_PRED, MT_SMOOTH_H_PRED,
                                MT_V_PRED,        MT_H_PRED,     MT_D135_PRED,   MT_D113_PRED,
                                MT_D157_PRED,     MT_D45_PRED,   MT_D67_PRED,    MT_D203_PRED};
  std::vector<int32_t> bufs(12 * NN);
  for (int j = 0; j < n; j++) {
    const J& jb = jobs[j];
    mt_uv16_result& r = results[j];
    const int cx = jb.px, cy = jb.py;
    if ((cx & (N - 1)) || (cy & (N - 1)) || cx + N > p->frame_w || cy + N > p->frame_h || jb.y_mode > MT_PAETH_PRED) {
      r.total = r.dc_total = r.cfl_total = INFINITY;
      r.uv_mode = 255;
      r.angle_delta = 0;
      r.cfl_alpha[0] = r.cfl_alpha[1] = 0;
      if (cf_out) memset(cf_out + (size_t)j * 2 * NN, 0, 2 * NN * sizeof(int32_t));
      if (rec_out) memset(rec_out + (size_t)j * 2 * NN, 0, 2 * NN * sizeof(uint16_t));
      continue;
    }
    const bool tr = jb.flags & MT_CAND_HAVE_TR, bl = jb.flags & MT_CAND_HAVE_BL, ft = jb.flags & MT_CAND_FILTER_TYPE;
    Plane P[2];
    for (int pl = 0; pl < 2; pl++) {
      P[pl].src = pl ? src_v : src_u;
      P[pl].rec = pl ? rec_v : rec_u;
      // the chroma txb_skip context and dc_sign span over the block's U + U units
      // (skip_ctx_16 / dc_sign_ctx_16 at 16x16, lossy_state.rs:1420-1440)
      bool anz = false, lnz = false;
      int s = -2 * U;
      for (int k = 0; k < U; k++) {
        anz |= jb.a_coef[pl][k] != 0x40;
        lnz |= jb.l_coef[pl][k] != 0x40;
        s += (jb.a_coef[pl][k] >> 6) + (jb.l_coef[pl][k] >> 6);
      }
      P[pl].sk = 7 + anz + lnz;
      P[pl].ds = (s != 0) + (s > 0);
    }
    int32_t* dpred = &bufs[0];  // [2][NN]
    int32_t* dcf = &bufs[2 * NN];
    int32_t* drr = &bufs[4 * NN];
    int32_t* cpred = &bufs[6 * NN];
    int32_t* ccf = &bufs[8 * NN];
    int32_t* crr = &bufs[10 * NN];
    // 1. DC
    int32_t dc[2];
    int64_t dsse[2], csse[2];
    float dbits[2], cbits[2];
    for (int pl = 0; pl < 2; pl++) {
      dc[pl] = or_dc_pred(P[pl].rec, p->stride, cx, cy, N, N, p->bd);
      for (int i = 0; i < NN; i++) dpred[pl * NN + i] = dc[pl];
      plane_cost_n(N, p, q, qm, cd, P[pl], cx, cy, MT_TX_DCT_DCT, true, dpred + pl * NN, dcf + pl * NN,
                   drr + pl * NN, &dsse[pl], &dbits[pl]);
    }
    // 2. CfL: cfl_ac_444 and cfl_best_alpha (or_cfl_alpha without subsampling)
    mt_cfl_block cb = {};
    cb.cx = (uint16_t)cx;
    cb.cy = (uint16_t)cy;
    cb.dc[0] = (int16_t)dc[0];
    cb.dc[1] = (int16_t)dc[1];
    int8_t alpha[2];
    std::vector<int32_t> ac(NN);
    or_cfl_alpha(luma, u->luma_stride, src_u, src_v, p->stride, 0, 0, N, N, vis_w, vis_h, p->bd, &cb, 1, alpha,
                 ac.data());
    for (int pl = 0; pl < 2; pl++) {
      for (int i = 0; i < NN; i++) {
        const int32_t diff = alpha[pl] * ac[i];
        const int32_t mag = ((diff < 0 ? -diff : diff) + 32) >> 6;
        const int32_t v = dc[pl] + (diff < 0 ? -mag : mag);
        cpred[pl * NN + i] = v < 0 ? 0 : (v > maxv ? maxv : v);
      }
      plane_cost_n(N, p, q, qm, cd, P[pl], cx, cy, MT_TX_DCT_DCT, false, cpred + pl * NN, ccf + pl * NN,
                   crr + pl * NN, &csse[pl], &cbits[pl]);
    }
    const float sig = or_uv_mode_bits(mc, jb.y_mode, MT_UV_CFL_PRED, 1, alpha[0], alpha[1]);
    const float dcb = or_uv_mode_bits(mc, jb.y_mode, MT_DC_PRED, 0, 0, 0);
    float dc_total, cfl_total;
    if (N == 16) {  // block16.rs:587-597
      dc_total = (float)(dsse[0] + dsse[1]) + mlam * (dbits[0] + dbits[1] + dcb);
      cfl_total = (float)(csse[0] + csse[1]) + mlam * (cbits[0] + cbits[1] + sig);
    } else {  // block32.rs:2399-2404: the planes' costs summed, then the mode bits
      dc_total = ((float)dsse[0] + mlam * dbits[0]) + ((float)dsse[1] + mlam * dbits[1]) + mlam * dcb;
      cfl_total = ((float)csse[0] + mlam * cbits[0]) + ((float)csse[1] + mlam * cbits[1]) + mlam * sig;
    }
    const bool use_cfl = cfl_total < dc_total && (alpha[0] != 0 || alpha[1] != 0);
    // the winner so far: prediction, levels, inverse
    std::vector<int32_t> bpred(use_cfl ? cpred : dpred, (use_cfl ? cpred : dpred) + 2 * NN);
    std::vector<int32_t> bcf(use_cfl ? ccf : dcf, (use_cfl ? ccf : dcf) + 2 * NN);
    std::vector<int32_t> brr(use_cfl ? crr : drr, (use_cfl ? crr : drr) + 2 * NN);
    // 3. the directional stage on dir_lambda
    float best_total = dlam * (use_cfl ? sig : dcb);
    for (int pl = 0; pl < 2; pl++)
      best_total += (float)(use_cfl ? csse[pl] : dsse[pl]) + dlam * (use_cfl ? cbits[pl] : dbits[pl]);
    int mode = MT_DC_PRED, delta = 0;
    // rank_chroma_modes + DirectionalTopK (K = 3)
    uint64_t tc[3];
    int tm[3], tn = 0;
    std::vector<int32_t> ppv(NN);
    int32_t* pp = ppv.data();
    for (int m : kList) {
      uint64_t cost = 0;
      for (int pl = 0; pl < 2; pl++) {
        or_intra_predict(P[pl].rec, p->stride, cx, cy, N, N, m, 0, tr, bl, p->frame_w, p->frame_h, ft, p->bd, pp);
        const int vw = std::min(std::max(vis_w - cx, 0), N), vh = std::min(std::max(vis_h - cy, 0), N);
        cost += satd_sad_proxy_n(P[pl].src + (size_t)cy * p->stride + cx, p->stride, pp, N, vw, vh);
      }
      int pos = tn < 3 ? tn : 2;
      if (tn == 3 && cost >= tc[pos]) continue;
      if (tn < 3) pos = tn++;
      while (pos > 0 && cost < tc[pos - 1]) {
        tc[pos] = tc[pos - 1];
        tm[pos] = tm[pos - 1];
        pos--;
      }
      tc[pos] = cost;
      tm[pos] = m;
    }
    std::vector<int32_t> nbuf(6 * NN);
    int32_t* npred = nbuf.data();
    int32_t* ncf = npred + 2 * NN;
    int32_t* nrr = ncf + 2 * NN;
    auto price = [&](int m, int d, bool etr, bool ebl, float rate_bits) {
      const int tx = N == 32 ? MT_TX_DCT_DCT : chroma_tx(m);  // forced DCT_DCT at TX_32X32
      float total = dlam * rate_bits;
      for (int pl = 0; pl < 2; pl++) {
        or_intra_predict(P[pl].rec, p->stride, cx, cy, N, N, m, d, etr, ebl, p->frame_w, p->frame_h, ft, p->bd,
                         npred + pl * NN);
        int64_t sse;
        float bits;
        plane_cost_n(N, p, q, qm, cd, P[pl], cx, cy, tx, true, npred + pl * NN, ncf + pl * NN, nrr + pl * NN, &sse,
                     &bits);
        total += (float)sse + dlam * bits;
      }
      return total;
    };
    auto take = [&]() {
      std::copy(npred, npred + 2 * NN, bpred.begin());
      std::copy(ncf, ncf + 2 * NN, bcf.begin());
      std::copy(nrr, nrr + 2 * NN, brr.begin());
    };
    for (int m : kList) {
      bool in = false;
      for (int e = 0; e < tn; e++) in |= tm[e] == m;
      if (!in) continue;
      const float total = price(m, 0, tr, bl, or_uv_mode_bits(mc, jb.y_mode, m, 0, 0, 0));
      if (total < best_total) {
        best_total = total;
        mode = m;
        take();
      }
    }
    // uv_ad: the zone-2 deltas of a directional winner (block16.rs:743-778, :2342-2349)
    if (u->angle_deltas && directional(mode)) {
      const int m = mode;
      std::vector<int> ds;
      if (m == MT_V_PRED) ds = {1, 2, 3};
      else if (m == MT_H_PRED) ds = {-3, -2, -1};
      else if (m == MT_D113_PRED || m == MT_D135_PRED || m == MT_D157_PRED) ds = {-3, -2, -1, 1, 2, 3};
      const float base_sig = or_uv_mode_bits(mc, jb.y_mode, m, 0, 0, 0) - or_cdf_cost(mc->angle_delta[m - MT_V_PRED], 3);
      for (int d : ds) {
        const float total = price(m, d, false, false, base_sig + or_cdf_cost(mc->angle_delta[m - MT_V_PRED], d + 3));
        if (total < best_total) {
          best_total = total;
          delta = d;
          take();
        }
      }
    }
    r.total = best_total;
    r.dc_total = dc_total;
    r.cfl_total = cfl_total;
    r.uv_mode = (uint8_t)(mode != MT_DC_PRED ? mode : (use_cfl ? MT_UV_CFL_PRED : MT_DC_PRED));
    r.angle_delta = (int8_t)delta;
    r.cfl_alpha[0] = alpha[0];
    r.cfl_alpha[1] = alpha[1];
    for (int i = 0; i < 2 * NN; i++) {
      if (cf_out) cf_out[(size_t)j * 2 * NN + i] = bcf[(size_t)i];
      if (rec_out) {
        const int32_t v = bpred[(size_t)i] + brr[(size_t)i];
        rec_out[(size_t)j * 2 * NN + i] = (uint16_t)(v < 0 ? 0 : (v > maxv ? maxv : v));
      }
    }
  }
  return MT_OK;
}

}  // namespace

extern "C" {

float or_uv_mode_bits(const mt_uv_mode_cdfs* c, int32_t y_mode, int32_t uv_mode, int32_t cfl, int32_t au,
                      int32_t av) {
  if (!cfl) {
    float bits = or_cdf_cost(c->uv_mode[y_mode], uv_mode);
    if (directional(uv_mode)) bits += or_cdf_cost(c->angle_delta[uv_mode - MT_V_PRED], 3);
    return bits;
  }
  const int su = au == 0 ? 0 : (au < 0 ? 1 : 2), sv = av == 0 ? 0 : (av < 0 ? 1 : 2);
  const int sign = su * 3 + sv;
  if (sign == 0) return or_cdf_cost(c->uv_mode[y_mode], MT_DC_PRED);
  float bits = or_cdf_cost(c->uv_mode[y_mode], MT_UV_CFL_PRED) + or_cdf_cost(c->cfl_sign, sign - 1);
  if (su != 0) bits += or_cdf_cost(c->cfl_alpha[(su == 2) * 3 + sv], (au < 0 ? -au : au) - 1);
  if (sv != 0) bits += or_cdf_cost(c->cfl_alpha[(sv == 2) * 3 + su], (av < 0 ? -av : av) - 1);
  return bits;
}

int or_pick_uv16_420(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* p, const mt_uv16_params* u, const mt_quant* q,
                     const uint8_t* qm, const mt_coef_cdfs* cd, const mt_uv_mode_cdfs* mc, const mt_uv16_job* jobs,
                     int32_t n, mt_uv16_result* results, int32_t* cf_out, uint16_t* rec_out) {
  if (!p || p->bd != 8) return MT_ERR_UNSUPPORTED;
  const int32_t maxv = (1 << p->bd) - 1;
  const float mlam = p->rd_lambda;
  const int vis_w = p->vis_w > 0 ? p->vis_w : p->frame_w, vis_h = p->vis_h > 0 ? p->vis_h : p->frame_h;
  static const int kJoint[12] = {MT_SMOOTH_V_PRED, MT_PAETH_PRED, MT_SMOOTH_PRED, MT_SMOOTH_H_PRED,
                                 MT_V_PRED,        MT_H_PRED,     MT_D135_PRED,   MT_D113_PRED,
                                 MT_D157_PRED,     MT_D45_PRED,   MT_D67_PRED,    MT_D203_PRED};
  for (int j = 0; j < n; j++) {
    const mt_uv16_job& jb = jobs[j];
    mt_uv16_result& r = results[j];
    const int cx = jb.px / 2, cy = jb.py / 2;
    if ((jb.px & 15) || (jb.py & 15) || cx + 8 > p->frame_w || cy + 8 > p->frame_h || jb.y_mode > MT_PAETH_PRED) {
      r.total = r.dc_total = r.cfl_total = INFINITY;
      r.uv_mode = 255;
      r.angle_delta = 0;
      r.cfl_alpha[0] = r.cfl_alpha[1] = 0;
      if (cf_out) memset(cf_out + (size_t)j * 128, 0, 128 * sizeof(int32_t));
      if (rec_out) memset(rec_out + (size_t)j * 128, 0, 128 * sizeof(uint16_t));
      continue;
    }
    const bool tr = jb.flags & MT_CAND_HAVE_TR, bl = jb.flags & MT_CAND_HAVE_BL, ft = jb.flags & MT_CAND_FILTER_TYPE;
    Plane P[2];
    for (int pl = 0; pl < 2; pl++) {
      P[pl].src = pl ? src_v : src_u;
      P[pl].rec = pl ? rec_v : rec_u;
      // skip_ctx 7 + above non-zero + left non-zero; dc_sign_ctx_span over 2 + 2
      const uint8_t* a = jb.a_coef[pl];
      const uint8_t* l = jb.l_coef[pl];
      P[pl].sk = 7 + (a[0] != 0x40 || a[1] != 0x40) + (l[0] != 0x40 || l[1] != 0x40);
      int s = 0;
      for (int k = 0; k < 2; k++) s += (a[k] >> 6) - 1 + (l[k] >> 6) - 1;
      P[pl].ds = (s != 0) + (s > 0);
    }
    // the winner's planes: prediction, levels, inverse
    int32_t bpred[2][64], bcf[2][64], brr[2][64];
    int32_t cpred[2][64], ccf[2][64], crr[2][64];
    // 1. DC
    int32_t dc[2];
    float dc_total = 0.0f;
    for (int pl = 0; pl < 2; pl++) {
      dc[pl] = or_dc_pred(P[pl].rec, p->stride, cx, cy, 8, 8, p->bd);
      for (int i = 0; i < 64; i++) bpred[pl][i] = dc[pl];
      dc_total += plane_cost(p, q, qm, cd, P[pl], cx, cy, MT_TX_DCT_DCT, true, bpred[pl], bcf[pl], brr[pl]);
    }
    float best_total = dc_total;
    int mode = MT_DC_PRED, delta = 0;
    // 2. CfL: cfl_ac_sub of the 16x16 luma, cfl_best_alpha per plane
    mt_cfl_block cb = {};
    cb.cx = (uint16_t)cx;
    cb.cy = (uint16_t)cy;
    cb.dc[0] = (int16_t)dc[0];
    cb.dc[1] = (int16_t)dc[1];
    int8_t alpha[2];
    int32_t ac[64];
    or_cfl_alpha(luma, u->luma_stride, src_u, src_v, p->stride, 1, 1, 8, 8, vis_w, vis_h, p->bd, &cb, 1, alpha, ac);
    float body = 0.0f;
    for (int pl = 0; pl < 2; pl++) {
      for (int i = 0; i < 64; i++) {
        const int32_t diff = alpha[pl] * ac[i];
        const int32_t mag = ((diff < 0 ? -diff : diff) + 32) >> 6;
        const int32_t v = dc[pl] + (diff < 0 ? -mag : mag);
        cpred[pl][i] = v < 0 ? 0 : (v > maxv ? maxv : v);
      }
      body += plane_cost(p, q, qm, cd, P[pl], cx, cy, MT_TX_DCT_DCT, false, cpred[pl], ccf[pl], crr[pl]);
    }
    const float cfl_total = body + mlam * or_uv_mode_bits(mc, jb.y_mode, MT_UV_CFL_PRED, 1, alpha[0], alpha[1]) -
                            mlam * or_uv_mode_bits(mc, jb.y_mode, MT_DC_PRED, 0, 0, 0);
    if ((alpha[0] != 0 || alpha[1] != 0) && cfl_total < best_total) {
      best_total = cfl_total;
      mode = MT_UV_CFL_PRED;
      memcpy(bpred, cpred, sizeof(bpred));
      memcpy(bcf, ccf, sizeof(bcf));
      memcpy(brr, crr, sizeof(brr));
    }
    // 3. the joint (mode, delta) shortlist, sorted by (score, mode, delta)
    std::vector<std::tuple<uint64_t, int, int>> all;
    int32_t pp[64];
    for (int m : kJoint) {
      const bool dir = directional(m) && u->angle_deltas;
      for (int d = dir ? -3 : 0; d <= (dir ? 3 : 0); d++) {
        uint64_t cost = 0;
        for (int pl = 0; pl < 2; pl++) {
          or_intra_predict(P[pl].rec, p->stride, cx, cy, 8, 8, m, d, tr, bl, p->frame_w, p->frame_h, ft, p->bd, pp);
          const int vw = std::min(std::max(vis_w - cx, 0), 8), vh = std::min(std::max(vis_h - cy, 0), 8);
          cost += satd_sad_proxy_n(P[pl].src + (size_t)cy * p->stride + cx, p->stride, pp, 8, vw, vh);
        }
        all.emplace_back(cost, m, d);
      }
    }
    std::sort(all.begin(), all.end());
    const int k = std::min(std::max(u->joint_k, 1), 12);
    for (int e = 0; e < k && e < (int)all.size(); e++) {
      const int m = std::get<1>(all[(size_t)e]), d = std::get<2>(all[(size_t)e]);
      const int tx = chroma_tx(m);
      float ad_bits = 0.0f;
      if (directional(m))
        ad_bits = or_cdf_cost(mc->angle_delta[m - MT_V_PRED], d + 3) - or_cdf_cost(mc->angle_delta[m - MT_V_PRED], 3);
      float total = mlam * (or_uv_mode_bits(mc, jb.y_mode, m, 0, 0, 0) + ad_bits);
      for (int pl = 0; pl < 2; pl++) {
        or_intra_predict(P[pl].rec, p->stride, cx, cy, 8, 8, m, d, tr, bl, p->frame_w, p->frame_h, ft, p->bd,
                         cpred[pl]);
        total += plane_cost(p, q, qm, cd, P[pl], cx, cy, tx, true, cpred[pl], ccf[pl], crr[pl]);
        if (pl == 0 && total >= best_total) break;
      }
      if (total < best_total) {
        best_total = total;
        mode = m;
        delta = d;
        memcpy(bpred, cpred, sizeof(bpred));
        memcpy(bcf, ccf, sizeof(bcf));
        memcpy(brr, crr, sizeof(brr));
      }
    }
    r.total = best_total;
    r.dc_total = dc_total;
    r.cfl_total = cfl_total;
    r.uv_mode = (uint8_t)mode;
    r.angle_delta = (int8_t)delta;
    r.cfl_alpha[0] = alpha[0];
    r.cfl_alpha[1] = alpha[1];
    for (int pl = 0; pl < 2; pl++)
      for (int i = 0; i < 64; i++) {
        if (cf_out) cf_out[(size_t)j * 128 + pl * 64 + i] = bcf[pl][i];
        if (rec_out) {
          const int32_t v = bpred[pl][i] + brr[pl][i];
          rec_out[(size_t)j * 128 + pl * 64 + i] = (uint16_t)(v < 0 ? 0 : (v > maxv ? maxv : v));
        }
      }
  }
  return MT_OK;
}


int or_pick_uv32_420(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* p, const mt_uv16_params* u, const mt_quant* q,
                     const uint8_t* qm, const mt_coef_cdfs* cd, const mt_uv_mode_cdfs* mc,
                     const mt_uv16_444_job* jobs, int32_t n, mt_uv16_result* results, int32_t* cf_out,
                     uint16_t* rec_out) {
  if (!p || p->bd != 8) return MT_ERR_UNSUPPORTED;
  const int32_t maxv = (1 << p->bd) - 1;
  const float mlam = p->rd_lambda;
  const int vis_w = p->vis_w > 0 ? p->vis_w : p->frame_w, vis_h = p->vis_h > 0 ? p->vis_h : p->frame_h;
  static const int kList[12] = {MT_SMOOTH_V_PRED, MT_PAETH_PRED, MT_SMOOTH_PRED, MT_SMOOTH_H_PRED,
                                MT_V_PRED,        MT_H_PRED,     MT_D135_PRED,   MT_D113_PRED,
                                MT_D157_PRED,     MT_D45_PRED,   MT_D67_PRED,    MT_D203_PRED};
  for (int j = 0; j < n; j++) {
    const mt_uv16_444_job& jb = jobs[j];
    mt_uv16_result& r = results[j];
    const int cx = jb.px / 2, cy = jb.py / 2;
    if ((jb.px & 31) || (jb.py & 31) || cx + 16 > p->frame_w || cy + 16 > p->frame_h || jb.y_mode > MT_PAETH_PRED) {
      r.total = r.dc_total = r.cfl_total = INFINITY;
      r.uv_mode = 255;
      r.angle_delta = 0;
      r.cfl_alpha[0] = r.cfl_alpha[1] = 0;
      if (cf_out) memset(cf_out + (size_t)j * 512, 0, 512 * sizeof(int32_t));
      if (rec_out) memset(rec_out + (size_t)j * 512, 0, 512 * sizeof(uint16_t));
      continue;
    }
    const bool tr = jb.flags & MT_CAND_HAVE_TR, bl = jb.flags & MT_CAND_HAVE_BL, ft = jb.flags & MT_CAND_FILTER_TYPE;
    Plane P[2];
    for (int pl = 0; pl < 2; pl++) {
      P[pl].src = pl ? src_v : src_u;
      P[pl].rec = pl ? rec_v : rec_u;
      bool anz = false, lnz = false;
      int s = -8;
      for (int k = 0; k < 4; k++) {
        anz |= jb.a_coef[pl][k] != 0x40;
        lnz |= jb.l_coef[pl][k] != 0x40;
        s += (jb.a_coef[pl][k] >> 6) + (jb.l_coef[pl][k] >> 6);
      }
      P[pl].sk = 7 + anz + lnz;
      P[pl].ds = (s != 0) + (s > 0);
    }
    std::vector<int32_t> bpred(512), bcf(512), brr(512), npred(512), ncf(512), nrr(512);
    int32_t dc[2];
    float dc_total = 0.0f;
    for (int pl = 0; pl < 2; pl++) {
      dc[pl] = or_dc_pred(P[pl].rec, p->stride, cx, cy, 16, 16, p->bd);
      for (int i = 0; i < 256; i++) bpred[(size_t)pl * 256 + i] = dc[pl];
      int64_t sse;
      float bits;
      plane_cost16(p, q, qm, cd, P[pl], cx, cy, MT_TX_DCT_DCT, true, &bpred[(size_t)pl * 256], &bcf[(size_t)pl * 256],
                   &brr[(size_t)pl * 256], &sse, &bits, true);
      dc_total += (float)sse + mlam * bits;
    }
    float best_total = dc_total;
    int mode = MT_DC_PRED, delta = 0;
    bool use_cfl = false;
    // CfL: cfl_ac_sub of the 32x32 luma (4:2:0) and cfl_best_alpha
    mt_cfl_block cb = {};
    cb.cx = (uint16_t)cx;
    cb.cy = (uint16_t)cy;
    cb.dc[0] = (int16_t)dc[0];
    cb.dc[1] = (int16_t)dc[1];
    int8_t alpha[2];
    std::vector<int32_t> ac(256);
    or_cfl_alpha(luma, u->luma_stride, src_u, src_v, p->stride, 1, 1, 16, 16, vis_w, vis_h, p->bd, &cb, 1, alpha,
                 ac.data());
    float body = 0.0f;
    for (int pl = 0; pl < 2; pl++) {
      for (int i = 0; i < 256; i++) {
        const int32_t diff = alpha[pl] * ac[(size_t)i];
        const int32_t mag = ((diff < 0 ? -diff : diff) + 32) >> 6;
        const int32_t v = dc[pl] + (diff < 0 ? -mag : mag);
        npred[(size_t)pl * 256 + i] = v < 0 ? 0 : (v > maxv ? maxv : v);
      }
      int64_t sse;
      float bits;
      plane_cost16(p, q, qm, cd, P[pl], cx, cy, MT_TX_DCT_DCT, false, &npred[(size_t)pl * 256], &ncf[(size_t)pl * 256],
                   &nrr[(size_t)pl * 256], &sse, &bits, true);
      body += (float)sse + mlam * bits;
    }
    const float cfl_total = body + mlam * or_uv_mode_bits(mc, jb.y_mode, MT_UV_CFL_PRED, 1, alpha[0], alpha[1]) -
                            mlam * or_uv_mode_bits(mc, jb.y_mode, MT_DC_PRED, 0, 0, 0);
    if ((alpha[0] != 0 || alpha[1] != 0) && cfl_total < best_total) {
      best_total = cfl_total;
      use_cfl = true;
      bpred = npred;
      bcf = ncf;
      brr = nrr;
    }
    // rank_chroma_modes + DirectionalTopK (K = 3)
    uint64_t tc[3];
    int tm[3], tn = 0;
    int32_t pp[256];
    for (int m : kList) {
      uint64_t cost = 0;
      for (int pl = 0; pl < 2; pl++) {
        or_intra_predict(P[pl].rec, p->stride, cx, cy, 16, 16, m, 0, tr, bl, p->frame_w, p->frame_h, ft, p->bd, pp);
        const int vw = std::min(std::max(vis_w - cx, 0), 16), vh = std::min(std::max(vis_h - cy, 0), 16);
        cost += satd_sad_proxy_n(P[pl].src + (size_t)cy * p->stride + cx, p->stride, pp, 16, vw, vh);
      }
      int pos = tn < 3 ? tn : 2;
      if (tn == 3 && cost >= tc[pos]) continue;
      if (tn < 3) pos = tn++;
      while (pos > 0 && cost < tc[pos - 1]) {
        tc[pos] = tc[pos - 1];
        tm[pos] = tm[pos - 1];
        pos--;
      }
      tc[pos] = cost;
      tm[pos] = m;
    }
    auto price = [&](int m, int d, bool etr, bool ebl, float rate_bits) {
      const int tx = chroma_tx(m);
      float total = mlam * rate_bits;
      for (int pl = 0; pl < 2; pl++) {
        or_intra_predict(P[pl].rec, p->stride, cx, cy, 16, 16, m, d, etr, ebl, p->frame_w, p->frame_h, ft, p->bd,
                         &npred[(size_t)pl * 256]);
        int64_t sse;
        float bits;
        plane_cost16(p, q, qm, cd, P[pl], cx, cy, tx, true, &npred[(size_t)pl * 256], &ncf[(size_t)pl * 256],
                     &nrr[(size_t)pl * 256], &sse, &bits, true);
        total += (float)sse + mlam * bits;
      }
      return total;
    };
    for (int m : kList) {
      bool in = false;
      for (int e = 0; e < tn; e++) in |= tm[e] == m;
      if (!in) continue;
      const float total = price(m, 0, tr, bl, or_uv_mode_bits(mc, jb.y_mode, m, 0, 0, 0));
      if (total < best_total) {
        best_total = total;
        mode = m;
        use_cfl = false;
        bpred = npred;
        bcf = ncf;
        brr = nrr;
      }
    }
    // uv_ad / uv_ad32 (block32.rs:3054-3110)
    if (!use_cfl && u->angle_deltas && directional(mode)) {
      const int m = mode;
      std::vector<int> ds;
      if (m == MT_V_PRED) ds = {1, 2, 3};
      else if (m == MT_H_PRED) ds = {-3, -2, -1};
      else if (m == MT_D113_PRED || m == MT_D135_PRED || m == MT_D157_PRED) ds = {-3, -2, -1, 1, 2, 3};
      const float base_sig = or_uv_mode_bits(mc, jb.y_mode, m, 0, 0, 0) - or_cdf_cost(mc->angle_delta[m - MT_V_PRED], 3);
      for (int d : ds) {
        const float total = price(m, d, false, false, base_sig + or_cdf_cost(mc->angle_delta[m - MT_V_PRED], d + 3));
        if (total < best_total) {
          best_total = total;
          delta = d;
          bpred = npred;
          bcf = ncf;
          brr = nrr;
        }
      }
    }
    r.total = best_total;
    r.dc_total = dc_total;
    r.cfl_total = cfl_total;
    r.uv_mode = (uint8_t)(use_cfl ? MT_UV_CFL_PRED : mode);
    r.angle_delta = (int8_t)delta;
    r.cfl_alpha[0] = alpha[0];
    r.cfl_alpha[1] = alpha[1];
    for (int i = 0; i < 512; i++) {
      if (cf_out) cf_out[(size_t)j * 512 + i] = bcf[(size_t)i];
      if (rec_out) {
        const int32_t v = bpred[(size_t)i] + brr[(size_t)i];
        rec_out[(size_t)j * 512 + i] = (uint16_t)(v < 0 ? 0 : (v > maxv ? maxv : v));
      }
    }
  }
  return MT_OK;
}

int or_pick_uv16_444(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* p, const mt_uv16_params* u, const mt_quant* q,
                     const uint8_t* qm, const mt_coef_cdfs* cd, const mt_uv_mode_cdfs* mc,
                     const mt_uv16_444_job* jobs, int32_t n, mt_uv16_result* results, int32_t* cf_out,
                     uint16_t* rec_out) {
  return pick444<16>(src_u, src_v, rec_u, rec_v, luma, p, u, q, qm, cd, mc, jobs, n, results, cf_out, rec_out);
}

// block32.rs pick_uv32_444 (:2264-2720).
int or_pick_uv32_444(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* p, const mt_uv16_params* u, const mt_quant* q,
                     const uint8_t* qm, const mt_coef_cdfs* cd, const mt_uv_mode_cdfs* mc,
                     const mt_uv32_444_job* jobs, int32_t n, mt_uv16_result* results, int32_t* cf_out,
                     uint16_t* rec_out) {
  return pick444<32>(src_u, src_v, rec_u, rec_v, luma, p, u, q, qm, cd, mc, jobs, n, results, cf_out, rec_out);
}

}  // extern "C"
