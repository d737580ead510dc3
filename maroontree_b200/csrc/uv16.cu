// The 16x16 leaf's 4:2:0 chroma search (pick_uv16_420,
// src/coder/block16.rs:980-1381) with the shipped tuning (uv16_joint on,
// uv8_joint_k 4, cfl_alpha_rd_steps 0), batched over leaves, one thread per
// leaf.  The 8x8 chroma block of each leaf runs the DC path, the CfL path
// (the AC of the 16x16 luma reconstruction, the closed-form alphas) and the
// joint (mode, delta) SATD shortlist, whose first joint_k entries are priced
// in full; every priced candidate goes through the same per-plane chain:
// prediction, the transform (DCT_DCT, or the uv mode's type for the
// shortlist) with the QM, the chroma trellis (trellis_optimize_ctx against
// the chroma TX_8X8 costs), preserve_dc where the reference applies it, the
// inverse, sse_recon and chroma_bits.  The candidate and the winner live in
// the two slots of UvWork; a candidate that wins swaps them.
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "../../include/maroontree_b200.h"
#include "common.cuh"
#include "leaf8.cuh"
#include "txfm32.cuh"
#include "wsse.cuh"

namespace mth {
float scaled_trellis_lambda_host(float dc_q, float lambda0);
}

namespace {

using namespace mtd;

constexpr int kUvThreads = 32;  // one warp per CTA: 8,040 leaves at 1080p reach every SM
constexpr int kJointModes = 12;
constexpr int kMaxJoint = 12;

struct UvArgs {
  mt_split16_params p;  // the chroma planes
  mt_uv16_params u;
  mt_quant q;           // the chroma quantiser
  float lambda;         // scaled_trellis_lambda of the chroma trellis (0: off)
  int has_qm;
};

// Both planes of one candidate: predictions, levels and inverses.
struct UvSlot {
  int16_t pred[2][64];
  int16_t cf[2][64];
  int16_t rr[2][64];
};

struct UvWork {
  UvSlot s[2];     // the candidate and the winner
  int32_t u[128];  // prediction edges, then the targets [0, 64) and the transform temporary [64, 128)
  int16_t resid[64];
  int16_t ac[64];  // CfL AC of the leaf's luma
  TrellisCtxScratch tr;
  alignas(16) uint8_t lv[160];  // the rate walk stores it as 32-bit words
};

// The shortlist's modes in the reference's order (block16.rs:1143-1156).
__constant__ uint8_t kJointList[kJointModes] = {MT_SMOOTH_V_PRED, MT_PAETH_PRED, MT_SMOOTH_PRED, MT_SMOOTH_H_PRED,
                                                MT_V_PRED,        MT_H_PRED,     MT_D135_PRED,   MT_D113_PRED,
                                                MT_D157_PRED,     MT_D45_PRED,   MT_D67_PRED,    MT_D203_PRED};

__device__ __forceinline__ bool directional(int m) { return m >= MT_V_PRED && m <= MT_D67_PRED; }

// chroma_tx_for_mode (src/coder/chroma_tx.rs:46-66): dav1d's uv-mode map.
__device__ __forceinline__ int chroma_tx(int m) {
  if (m == MT_PAETH_PRED || m == MT_SMOOTH_PRED || m == MT_D135_PRED) return MT_TX_ADST_ADST;
  if (m == MT_SMOOTH_V_PRED || m == MT_V_PRED || m == MT_D113_PRED || m == MT_D67_PRED) return MT_TX_ADST_DCT;
  if (m == MT_SMOOTH_H_PRED || m == MT_H_PRED || m == MT_D157_PRED || m == MT_D203_PRED) return MT_TX_DCT_ADST;
  return MT_TX_DCT_DCT;
}

__device__ __forceinline__ float rd_cost_i64(long long d, float lam, float rate) {
  return __fadd_rn((float)d, __fmul_rn(lam, rate));
}

// uv_mode_bits (src/coder/lossy_state.rs:1302-1349); cfl: the alphas' form.
__device__ float uv_mode_bits(const mt_uv_mode_costs& C, int y_mode, int uv, bool cfl, int au, int av) {
  if (!cfl) {
    float bits = C.uv_mode[y_mode][uv];
    if (directional(uv)) bits = __fadd_rn(bits, C.angle_delta[uv - MT_V_PRED][3]);
    return bits;
  }
  const int su = au == 0 ? 0 : (au < 0 ? 1 : 2), sv = av == 0 ? 0 : (av < 0 ? 1 : 2);
  const int sign = su * 3 + sv;
  if (sign == 0) return C.uv_mode[y_mode][MT_DC_PRED];
  float bits = __fadd_rn(C.uv_mode[y_mode][MT_UV_CFL_PRED], C.cfl_sign[sign - 1]);
  if (su != 0) bits = __fadd_rn(bits, C.cfl_alpha[(su == 2) * 3 + sv][abs(au) - 1]);
  if (sv != 0) bits = __fadd_rn(bits, C.cfl_alpha[(sv == 2) * 3 + su][abs(av) - 1]);
  return bits;
}

// Per-plane constants of a job: source / reconstruction origins, displayed
// extent, coefficient contexts.
struct UvPlane {
  const uint16_t* src;  // block origin
  const uint16_t* rec;  // plane base
  int vw, vh;
  int sk, ds;           // txb_skip context 7 + above nz + left nz, dc_sign_ctx_span
  float skip1, skip0;
};

// One plane of a candidate after its prediction: residual, transform with
// the QM, trellis, preserve_dc (src/rd_sse.rs:759-765) when `keep_dc`,
// inverse, sse_recon and the rate.  Returns the plane's rd_cost_i64.
__device__ float plane_chain(const UvArgs& a, const UvPlane& P, const mt_coef_costs& T, const uint8_t* qm,
                             const float* sQs, int tx, bool keep_dc, int16_t* pred, int16_t* cf, int16_t* rr,
                             UvWork& w) {
  const mt_split16_params& p = a.p;
  const mt_quant& q = a.q;
  int32_t sum = 0;
#pragma unroll 8
  for (int i = 0; i < 64; i++) {
    const int32_t r = (int32_t)P.src[(size_t)(i >> 3) * p.stride + (i & 7)] - pred[i];
    w.resid[i] = (int16_t)r;
    sum += r;
  }
  float* tf = reinterpret_cast<float*>(w.u);
  int32_t* tmp = w.u + 64;
  fwd8x8(w.resid, tx, q, cf, tf, tmp);
  if (qm) apply_qm(cf, tf, sQs, 64);
  if (a.lambda > 0.0f)
    trellis_ctx8(cf, tf, (float)q.dc_q, (float)q.ac_q, a.lambda, T, P.ds, qm, q.qm_level >= 5, p.band_tilt, w.tr);
  if (keep_dc) {
    const int32_t mean = sum / 64;  // truncating, as the reference's i32 division
    if (cf[0] == 0 && abs(mean) >= 8) cf[0] = (int16_t)(mean > 0 ? 1 : -1);
  }
  inv8x8(cf, tx, q, qm, rr, tmp);
  ErrBlock<int16_t, int16_t> eb;
  eb.src = P.src;
  eb.stride = p.stride;
  eb.pred = pred;
  eb.resid = rr;
  eb.w = 8;
  eb.vw = P.vw;
  eb.vh = P.vh;
  eb.maxv = (1 << p.bd) - 1;
  const long long sse = sse_recon_block(eb, p.wsse_scale);
  const float bits = rate_bounded<8>(cf, T, P.sk, P.ds, 0, -1, p.use_skip_bits != 0, P.skip1, P.skip0,
                                     __int_as_float(0x7f800000), w.lv);
  return rd_cost_i64(sse, p.rd_lambda, bits);
}

// cfl_best_alpha (src/intrapred.rs:1211-1258) over the displayed part: the
// closed-form alpha, then the first minimum of the prediction's SSE over
// alpha - 3 .. alpha + 3 within +-16.
__device__ int cfl_alpha(const int16_t* ac, const UvPlane& P, int stride, int32_t dc, int32_t maxv) {
  long long num = 0, den = 0;
  for (int y = 0; y < P.vh; y++)
    for (int x = 0; x < P.vw; x++) {
      const long long v = ac[y * 8 + x];
      num += (long long)((int32_t)P.src[(size_t)y * stride + x] - dc) * v;
      den += v * v;
    }
  if (den == 0) return 0;
  const long long sg = num > 0 ? 1 : (num < 0 ? -1 : 0);
  long long a0 = (64 * num + (den >> 1) * sg) / den;
  a0 = a0 < -16 ? -16 : (a0 > 16 ? 16 : a0);
  long long best_e = 0x7fffffffffffffffLL;
  int best_a = 0;
  for (int c = (int)a0 - 3; c <= (int)a0 + 3; c++) {
    if (c < -16 || c > 16) continue;
    long long e = 0;
    for (int y = 0; y < P.vh; y++)
      for (int x = 0; x < P.vw; x++) {
        const long long d = (int32_t)P.src[(size_t)y * stride + x] - cfl_pred_pixel(dc, ac[y * 8 + x], c, maxv);
        e += d * d;
      }
    if (e < best_e) {
      best_e = e;
      best_a = c;
    }
  }
  return best_a;
}

__global__ void __launch_bounds__(kUvThreads) uv16_420_kernel(
    const uint16_t* __restrict__ src_u, const uint16_t* __restrict__ src_v, const uint16_t* __restrict__ rec_u,
    const uint16_t* __restrict__ rec_v, const uint16_t* __restrict__ luma, UvArgs a,
    const uint8_t* __restrict__ qm_row, const mt_coef_costs* __restrict__ costs,
    const mt_uv_mode_costs* __restrict__ mode_costs, const mt_uv16_job* __restrict__ jobs, int n,
    mt_uv16_result* __restrict__ res, int32_t* __restrict__ cf_out, uint16_t* __restrict__ rec_out, int arena) {
  __shared__ mt_coef_costs sT;
  __shared__ mt_uv_mode_costs sM;
  __shared__ uint8_t sQm[64];
  __shared__ float sQs[64];
  {
    const float* g = reinterpret_cast<const float*>(costs);
    float* s = reinterpret_cast<float*>(&sT);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
    const float* gm = reinterpret_cast<const float*>(mode_costs);
    float* sm = reinterpret_cast<float*>(&sM);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_uv_mode_costs) / 4); i += blockDim.x) sm[i] = gm[i];
    for (int i = threadIdx.x; i < 64; i += blockDim.x) {
      const int wq = a.has_qm ? qm_row[i] : 32;
      sQm[i] = (uint8_t)wq;
      sQs[i] = fwd_qm_scale(wq);
    }
    __syncthreads();
  }
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const mt_split16_params& p = a.p;
  const mt_uv16_job jb = jobs[j];
  mt_uv16_result& r = res[j];
  const int cx = jb.px >> 1, cy = jb.py >> 1;
  const float kInf = __int_as_float(0x7f800000);
  const bool ok = (jb.px & 15) == 0 && (jb.py & 15) == 0 && cx + 8 <= p.frame_w && cy + 8 <= p.frame_h &&
                  jb.y_mode <= MT_PAETH_PRED;
  if (!ok) {
    r.total = r.dc_total = r.cfl_total = kInf;
    r.uv_mode = 255;
    r.angle_delta = 0;
    r.cfl_alpha[0] = r.cfl_alpha[1] = 0;
    if (cf_out)
      for (int i = 0; i < 128; i++) cf_out[(size_t)j * 128 + i] = 0;
    if (rec_out)
      for (int i = 0; i < 128; i++) rec_out[(size_t)j * 128 + i] = 0;
    return;
  }
  const mt_coef_costs& T = sT;
  const mt_uv_mode_costs& M = sM;
  const uint8_t* qm = a.has_qm ? sQm : nullptr;
  const int32_t maxv = (1 << p.bd) - 1;
  const float mlam = p.rd_lambda;
  const bool have_tr = jb.flags & MT_CAND_HAVE_TR, have_bl = jb.flags & MT_CAND_HAVE_BL;
  const bool ft = jb.flags & MT_CAND_FILTER_TYPE;
  const int vis_w = p.vis_w > 0 ? p.vis_w : p.frame_w, vis_h = p.vis_h > 0 ? p.vis_h : p.frame_h;
  UvPlane P[2];
  for (int pl = 0; pl < 2; pl++) {
    UvPlane& q = P[pl];
    q.src = (pl ? src_v : src_u) + (size_t)cy * p.stride + cx;
    q.rec = pl ? rec_v : rec_u;
    q.vw = min(max(vis_w - cx, 0), 8);
    q.vh = min(max(vis_h - cy, 0), 8);
    const uint32_t a0 = jb.a_coef[pl][0], a1 = jb.a_coef[pl][1], l0 = jb.l_coef[pl][0], l1 = jb.l_coef[pl][1];
    q.sk = 7 + (a0 != 0x40 || a1 != 0x40) + (l0 != 0x40 || l1 != 0x40);
    const int s = (int)(a0 >> 6) + (int)(a1 >> 6) + (int)(l0 >> 6) + (int)(l1 >> 6) - 4;
    q.ds = (s != 0) + (s > 0);
    q.skip1 = p.use_skip_bits ? p.skip_bits[q.sk][0] : 0.0f;
    q.skip0 = p.use_skip_bits ? p.skip_bits[q.sk][1] : 0.0f;
  }
  UvWork& w = smem_arena<UvWork>(arena);
  int best = 0;
  // 1. DC on both planes (block16.rs:999-1046): no mode bits in its total
  int32_t dc[2];
  float dc_total = 0.0f;
  for (int pl = 0; pl < 2; pl++) {
    predict_sq<8>(P[pl].rec, p.stride, p.frame_w, p.frame_h, cx, cy, MT_DC_PRED, 0, have_tr, have_bl, ft, p.bd,
                  w.s[0].pred[pl], w.u);
    dc[pl] = w.s[0].pred[pl][0];
    dc_total = __fadd_rn(dc_total, plane_chain(a, P[pl], T, qm, sQs, MT_TX_DCT_DCT, true, w.s[0].pred[pl],
                                               w.s[0].cf[pl], w.s[0].rr[pl], w));
  }
  float best_total = dc_total;
  int mode = MT_DC_PRED, delta = 0;
  // 2. CfL (:1058-1128): the AC of the 16x16 luma reconstruction, the
  // closed-form alphas, each plane's prediction through the DCT chain
  {
    const int ls = a.u.luma_stride;
    const uint16_t* l = luma + (size_t)jb.py * ls + jb.px;
    int32_t sum = 32;
    for (int i = 0; i < 64; i++) {
      const int y = i >> 3, x = i & 7;
      const uint16_t* q = l + (size_t)(2 * y) * ls + 2 * x;
      const int32_t v = ((int32_t)q[0] + q[1] + q[ls] + q[ls + 1]) << 1;
      w.ac[i] = (int16_t)v;
      sum += v;
    }
    const int32_t mean = sum >> 6;
    for (int i = 0; i < 64; i++) w.ac[i] = (int16_t)(w.ac[i] - mean);
  }
  int alpha[2];
  for (int pl = 0; pl < 2; pl++) alpha[pl] = cfl_alpha(w.ac, P[pl], p.stride, dc[pl], maxv);
  {
    UvSlot& c = w.s[1 - best];
    float body = 0.0f;
    for (int pl = 0; pl < 2; pl++) {
      for (int i = 0; i < 64; i++) c.pred[pl][i] = (int16_t)cfl_pred_pixel(dc[pl], w.ac[i], alpha[pl], maxv);
      body = __fadd_rn(body, plane_chain(a, P[pl], T, qm, sQs, MT_TX_DCT_DCT, false, c.pred[pl], c.cf[pl],
                                         c.rr[pl], w));
    }
    const float cfl_total =
        __fsub_rn(__fadd_rn(body, __fmul_rn(mlam, uv_mode_bits(M, jb.y_mode, MT_UV_CFL_PRED, true, alpha[0], alpha[1]))),
                  __fmul_rn(mlam, uv_mode_bits(M, jb.y_mode, MT_DC_PRED, false, 0, 0)));
    r.cfl_total = cfl_total;
    if ((alpha[0] != 0 || alpha[1] != 0) && cfl_total < best_total) {
      best_total = cfl_total;
      mode = MT_UV_CFL_PRED;
      best = 1 - best;
    }
  }
  // 3. the joint (mode, delta) shortlist (:1157-1240): the two planes'
  // satd_sad_proxy per candidate, the first joint_k by (score, mode, delta)
  const int k = min(max(a.u.joint_k, 1), kMaxJoint);
  unsigned long long ks[kMaxJoint];
  uint8_t km[kMaxJoint];
  int8_t kd[kMaxJoint];
  int nk = 0;
  int16_t* sp = w.s[1 - best].pred[0];  // scratch prediction
  for (int ci = 0; ci < kJointModes; ci++) {
    const int m = kJointList[ci];
    const bool dir = directional(m) && a.u.angle_deltas;
    for (int d = dir ? -3 : 0; d <= (dir ? 3 : 0); d++) {
      unsigned long long sc = 0;
      for (int pl = 0; pl < 2; pl++) {
        predict_sq<8>(P[pl].rec, p.stride, p.frame_w, p.frame_h, cx, cy, m, d, have_tr, have_bl, ft, p.bd, sp, w.u);
        sc += satd_sad_proxy<8>(pl ? src_v : src_u, p.stride, cx, cy, sp, P[pl].vw, P[pl].vh);
      }
      // insert (sc, m, d) into the ascending list of at most k entries
      auto less = [&](int e) {
        return sc < ks[e] || (sc == ks[e] && (m < km[e] || (m == km[e] && d < kd[e])));
      };
      if (nk == k && !less(nk - 1)) continue;
      int e = nk < k ? nk++ : nk - 1;
      while (e > 0 && less(e - 1)) {
        ks[e] = ks[e - 1];
        km[e] = km[e - 1];
        kd[e] = kd[e - 1];
        e--;
      }
      ks[e] = sc;
      km[e] = (uint8_t)m;
      kd[e] = (int8_t)d;
    }
  }
  for (int e = 0; e < nk; e++) {
    const int m = km[e], d = kd[e], tx = chroma_tx(m);
    float ad_bits = 0.0f;
    if (directional(m)) ad_bits = __fsub_rn(M.angle_delta[m - MT_V_PRED][d + 3], M.angle_delta[m - MT_V_PRED][3]);
    float total = __fmul_rn(mlam, __fadd_rn(uv_mode_bits(M, jb.y_mode, m, false, 0, 0), ad_bits));
    UvSlot& c = w.s[1 - best];
    for (int pl = 0; pl < 2; pl++) {
      predict_sq<8>(P[pl].rec, p.stride, p.frame_w, p.frame_h, cx, cy, m, d, have_tr, have_bl, ft, p.bd, c.pred[pl],
                    w.u);
      total = __fadd_rn(total, plane_chain(a, P[pl], T, qm, sQs, tx, true, c.pred[pl], c.cf[pl], c.rr[pl], w));
      if (pl == 0 && total >= best_total) break;  // cannot win: the second plane is skipped
    }
    if (total < best_total) {
      best_total = total;
      mode = m;
      delta = d;
      best = 1 - best;
    }
  }
  r.total = best_total;
  r.dc_total = dc_total;
  r.uv_mode = (uint8_t)mode;
  r.angle_delta = (int8_t)delta;
  r.cfl_alpha[0] = (int8_t)alpha[0];
  r.cfl_alpha[1] = (int8_t)alpha[1];
  const UvSlot& b = w.s[best];
  if (cf_out)
    for (int pl = 0; pl < 2; pl++)
      for (int i = 0; i < 64; i++) cf_out[(size_t)j * 128 + pl * 64 + i] = b.cf[pl][i];
  if (rec_out)
    for (int pl = 0; pl < 2; pl++)
      for (int i = 0; i < 64; i++)
        rec_out[(size_t)j * 128 + pl * 64 + i] = (uint16_t)clampi((int32_t)b.pred[pl][i] + b.rr[pl][i], 0, maxv);
}

// ---- 4:4:4: pick_uv16_444 and pick_uv32_444 ----

// Both planes of one N x N candidate: predictions, levels (32-bit at 32x32,
// where a full-scale DC passes 16 bits) and inverses.
template <int N>
struct UvBigSlot {
  using Coef = std::conditional_t<N == 32, int32_t, int16_t>;
  int16_t pred[2][N * N];
  Coef cf[2][N * N];
  int16_t rr[2][N * N];
};

template <int N>
struct UvBigWork {
  UvBigSlot<N> s[2];   // the current choice and the candidate
  int32_t u[2 * N * N];  // prediction edges, then the targets [0, N*N) and the transform temporary [N*N, 2N*N)
  int16_t resid[N * N];
  int16_t ac[N * N];
  float suf[N * N + 1];  // trellis_sq scratch
  std::conditional_t<N == 16, TrellisCtxScratchW<16>, char> trc;  // trellis_ctx<16> scratch (4:2:0 at 16x16)
  alignas(16) uint8_t lv[(N + 2) * N];  // the rate walk stores it as 32-bit words
};
using Uv444Slot = UvBigSlot<16>;
using Uv444Work = UvBigWork<16>;

struct PlaneCost {
  long long sse;
  float bits;
};

// One N x N plane of a candidate after its prediction: the transform with
// the QM (DCT_DCT only at 32x32), the plain trellis_optimize (the 4:4:4
// chroma_rect_trellis) or, CTX, trellis_optimize_ctx against the chroma
// costs in the plane's dc_sign context (4:2:0), preserve_dc when `keep_dc`,
// the inverse, sse_recon and chroma_bits.
template <int N, bool CTX = false>
__device__ PlaneCost plane_chain(const UvArgs& a, const UvPlane& P, const mt_coef_costs& T, const uint8_t* qm,
                                 const float* sQs, const float* lut, int tx, bool keep_dc, int16_t* pred,
                                 typename UvBigSlot<N>::Coef* cf, int16_t* rr, UvBigWork<N>& w) {
  static_assert(N == 16 || N == 32, "16x16 and 32x32 chroma blocks");
  static_assert(!CTX || N == 16, "the context trellis runs at 16x16 here");
  constexpr int NN = N * N, L = log2w<N>();
  const mt_split16_params& p = a.p;
  const mt_quant& q = a.q;
  int32_t sum = 0;
#pragma unroll 8
  for (int i = 0; i < NN; i++) {
    const int32_t r = (int32_t)P.src[(size_t)(i >> L) * p.stride + (i & (N - 1))] - pred[i];
    w.resid[i] = (int16_t)r;
    sum += r;
  }
  float* tf = reinterpret_cast<float*>(w.u);
  int32_t* tmp = w.u + NN;
  if constexpr (N == 16) fwd16x16(w.resid, tx, q, cf, tf, tmp);
  else fwd32x32(w.resid, q, cf, tf, tmp);
  if (qm) apply_qm(cf, tf, sQs, NN);
  if (a.lambda > 0.0f) {
    if constexpr (CTX)
      trellis_ctx<16>(cf, tf, (float)q.dc_q, (float)q.ac_q, a.lambda, T, P.ds, qm, q.qm_level >= 5, p.band_tilt,
                      w.trc);
    else if constexpr (N == 16)
      trellis_sq<NN>(cf, tf, w.suf, (float)q.dc_q, (float)q.ac_q, a.lambda, lut, Scan16{});
    else
      trellis_sq<NN>(cf, tf, w.suf, (float)q.dc_q, (float)q.ac_q, a.lambda, lut, Scan32{});
  }
  if (keep_dc) {
    const int32_t mean = sum / NN;
    if (cf[0] == 0 && abs(mean) >= 8) cf[0] = mean > 0 ? 1 : -1;
  }
  if constexpr (N == 16) inv16x16(cf, tx, q, qm, rr, tmp);
  else inv32x32(cf, q, qm, rr, tmp);
  ErrBlock<int16_t, int16_t> eb;
  eb.src = P.src;
  eb.stride = p.stride;
  eb.pred = pred;
  eb.resid = rr;
  eb.w = N;
  eb.vw = P.vw;
  eb.vh = P.vh;
  eb.maxv = (1 << p.bd) - 1;
  PlaneCost c;
  c.sse = sse_recon_block(eb, p.wsse_scale);
  c.bits = rate_bounded<N>(cf, T, P.sk, P.ds, 0, -1, p.use_skip_bits != 0, P.skip1, P.skip0,
                           __int_as_float(0x7f800000), w.lv);
  return c;
}

// cfl_best_alpha over an N x N block's displayed part (as cfl_alpha).
template <int N>
__device__ int cfl_alpha_n(const int16_t* ac, const UvPlane& P, int stride, int32_t dc, int32_t maxv) {
  long long num = 0, den = 0;
  for (int y = 0; y < P.vh; y++)
    for (int x = 0; x < P.vw; x++) {
      const long long v = ac[y * N + x];
      num += (long long)((int32_t)P.src[(size_t)y * stride + x] - dc) * v;
      den += v * v;
    }
  if (den == 0) return 0;
  const long long sg = num > 0 ? 1 : (num < 0 ? -1 : 0);
  long long a0 = (64 * num + (den >> 1) * sg) / den;
  a0 = a0 < -16 ? -16 : (a0 > 16 ? 16 : a0);
  long long best_e = 0x7fffffffffffffffLL;
  int best_a = 0;
  for (int c = (int)a0 - 3; c <= (int)a0 + 3; c++) {
    if (c < -16 || c > 16) continue;
    long long e = 0;
    for (int y = 0; y < P.vh; y++)
      for (int x = 0; x < P.vw; x++) {
        const long long d = (int32_t)P.src[(size_t)y * stride + x] - cfl_pred_pixel(dc, ac[y * N + x], c, maxv);
        e += d * d;
      }
    if (e < best_e) {
      best_e = e;
      best_a = c;
    }
  }
  return best_a;
}

// The 4:4:4 leaf searches: N = 16 is pick_uv16_444 (block16.rs:437-978), N =
// 32 pick_uv32_444 (block32.rs:2264-2720).  J: the job (four or eight
// context bytes per plane and side).
template <int N, typename J>
__global__ void __launch_bounds__(kUvThreads) uv444_kernel(
    const uint16_t* __restrict__ src_u, const uint16_t* __restrict__ src_v, const uint16_t* __restrict__ rec_u,
    const uint16_t* __restrict__ rec_v, const uint16_t* __restrict__ luma, UvArgs a,
    const uint8_t* __restrict__ qm_row, const mt_coef_costs* __restrict__ costs,
    const mt_uv_mode_costs* __restrict__ mode_costs, const J* __restrict__ jobs, int n,
    mt_uv16_result* __restrict__ res, int32_t* __restrict__ cf_out, uint16_t* __restrict__ rec_out, int arena) {
  constexpr int NN = N * N, U = N / 4, L = log2w<N>();
  __shared__ mt_coef_costs sT;
  __shared__ mt_uv_mode_costs sM;
  __shared__ uint8_t sQm[NN];
  __shared__ float sQs[NN];
  __shared__ float sLut[64];
  {
    const float* g = reinterpret_cast<const float*>(costs);
    float* s = reinterpret_cast<float*>(&sT);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
    const float* gm = reinterpret_cast<const float*>(mode_costs);
    float* sm = reinterpret_cast<float*>(&sM);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_uv_mode_costs) / 4); i += blockDim.x) sm[i] = gm[i];
    for (int i = threadIdx.x; i < NN; i += blockDim.x) {
      const int wq = a.has_qm ? qm_row[i] : 32;
      sQm[i] = (uint8_t)wq;
      sQs[i] = fwd_qm_scale(wq);
    }
    for (int i = threadIdx.x; i < 64; i += blockDim.x) sLut[i] = kCoefRateLut[i];
    __syncthreads();
  }
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const mt_split16_params& p = a.p;
  const J jb = jobs[j];
  mt_uv16_result& r = res[j];
  const int cx = jb.px, cy = jb.py;
  const float kInf = __int_as_float(0x7f800000);
  const bool ok = (cx & (N - 1)) == 0 && (cy & (N - 1)) == 0 && cx + N <= p.frame_w && cy + N <= p.frame_h &&
                  jb.y_mode <= MT_PAETH_PRED;
  if (!ok) {
    r.total = r.dc_total = r.cfl_total = kInf;
    r.uv_mode = 255;
    r.angle_delta = 0;
    r.cfl_alpha[0] = r.cfl_alpha[1] = 0;
    if (cf_out)
      for (int i = 0; i < 2 * NN; i++) cf_out[(size_t)j * 2 * NN + i] = 0;
    if (rec_out)
      for (int i = 0; i < 2 * NN; i++) rec_out[(size_t)j * 2 * NN + i] = 0;
    return;
  }
  const mt_coef_costs& T = sT;
  const mt_uv_mode_costs& M = sM;
  const uint8_t* qm = a.has_qm ? sQm : nullptr;
  const int32_t maxv = (1 << p.bd) - 1;
  const float mlam = p.rd_lambda, dlam = a.u.dir_lambda;
  const bool have_tr = jb.flags & MT_CAND_HAVE_TR, have_bl = jb.flags & MT_CAND_HAVE_BL;
  const bool ft = jb.flags & MT_CAND_FILTER_TYPE;
  const int vis_w = p.vis_w > 0 ? p.vis_w : p.frame_w, vis_h = p.vis_h > 0 ? p.vis_h : p.frame_h;
  UvPlane P[2];
  for (int pl = 0; pl < 2; pl++) {
    UvPlane& q = P[pl];
    q.src = (pl ? src_v : src_u) + (size_t)cy * p.stride + cx;
    q.rec = pl ? rec_v : rec_u;
    q.vw = min(max(vis_w - cx, 0), N);
    q.vh = min(max(vis_h - cy, 0), N);
    bool anz = false, lnz = false;
    int s = -2 * U;
    for (int k = 0; k < U; k++) {
      anz |= jb.a_coef[pl][k] != 0x40;
      lnz |= jb.l_coef[pl][k] != 0x40;
      s += (jb.a_coef[pl][k] >> 6) + (jb.l_coef[pl][k] >> 6);
    }
    q.sk = 7 + anz + lnz;       // the chroma txb_skip context over the block's units
    q.ds = (s != 0) + (s > 0);  // dc_sign_ctx_span over U + U units
    q.skip1 = p.use_skip_bits ? p.skip_bits[q.sk][0] : 0.0f;
    q.skip0 = p.use_skip_bits ? p.skip_bits[q.sk][1] : 0.0f;
  }
  UvBigWork<N>& w = smem_arena<UvBigWork<N>>(arena);
  // DC, slot 0
  int32_t dc[2];
  PlaneCost dcc[2], cfc[2];
  for (int pl = 0; pl < 2; pl++) {
    predict_sq<N>(P[pl].rec, p.stride, p.frame_w, p.frame_h, cx, cy, MT_DC_PRED, 0, have_tr, have_bl, ft, p.bd,
                  w.s[0].pred[pl], w.u);
    dc[pl] = w.s[0].pred[pl][0];
    dcc[pl] = plane_chain<N>(a, P[pl], T, qm, sQs, sLut, MT_TX_DCT_DCT, true, w.s[0].pred[pl], w.s[0].cf[pl],
                             w.s[0].rr[pl], w);
  }
  // CfL against DC, slot 1: cfl_ac_444 (each luma sample << 3, less the rounded mean)
  {
    const int ls = a.u.luma_stride;
    const uint16_t* l = luma + (size_t)cy * ls + cx;
    int32_t sum = NN / 2;
    for (int i = 0; i < NN; i++) {
      const int32_t v = (int32_t)l[(size_t)(i >> L) * ls + (i & (N - 1))] << 3;
      w.ac[i] = (int16_t)v;
      sum += v;
    }
    const int32_t mean = sum >> (2 * L);
    for (int i = 0; i < NN; i++) w.ac[i] = (int16_t)(w.ac[i] - mean);
  }
  int alpha[2];
  for (int pl = 0; pl < 2; pl++) alpha[pl] = cfl_alpha_n<N>(w.ac, P[pl], p.stride, dc[pl], maxv);
  for (int pl = 0; pl < 2; pl++) {
    for (int i = 0; i < NN; i++) w.s[1].pred[pl][i] = (int16_t)cfl_pred_pixel(dc[pl], w.ac[i], alpha[pl], maxv);
    cfc[pl] = plane_chain<N>(a, P[pl], T, qm, sQs, sLut, MT_TX_DCT_DCT, false, w.s[1].pred[pl], w.s[1].cf[pl],
                             w.s[1].rr[pl], w);
  }
  const float sig = uv_mode_bits(M, jb.y_mode, MT_UV_CFL_PRED, true, alpha[0], alpha[1]);
  const float dc_bits = uv_mode_bits(M, jb.y_mode, MT_DC_PRED, false, 0, 0);
  float dc_total, cfl_total;
  if constexpr (N == 16) {
    // rd_cost_i64 of the summed SSE and bits (block16.rs:587-597)
    dc_total = rd_cost_i64(dcc[0].sse + dcc[1].sse, mlam, __fadd_rn(__fadd_rn(dcc[0].bits, dcc[1].bits), dc_bits));
    cfl_total = rd_cost_i64(cfc[0].sse + cfc[1].sse, mlam, __fadd_rn(__fadd_rn(cfc[0].bits, cfc[1].bits), sig));
  } else {
    // the planes' rd_cost_i64 summed, then the mode bits (block32.rs:2399-2404)
    dc_total = __fadd_rn(__fadd_rn(rd_cost_i64(dcc[0].sse, mlam, dcc[0].bits), rd_cost_i64(dcc[1].sse, mlam, dcc[1].bits)),
                         __fmul_rn(mlam, dc_bits));
    cfl_total = __fadd_rn(__fadd_rn(rd_cost_i64(cfc[0].sse, mlam, cfc[0].bits), rd_cost_i64(cfc[1].sse, mlam, cfc[1].bits)),
                          __fmul_rn(mlam, sig));
  }
  const bool use_cfl = cfl_total < dc_total && (alpha[0] != 0 || alpha[1] != 0);
  int best = use_cfl ? 1 : 0;
  const PlaneCost* cur = use_cfl ? cfc : dcc;
  // the directional stage on dir_lambda: the current choice's total, then the ranked modes
  float best_total = __fmul_rn(dlam, use_cfl ? sig : dc_bits);
  for (int pl = 0; pl < 2; pl++) best_total = __fadd_rn(best_total, rd_cost_i64(cur[pl].sse, dlam, cur[pl].bits));
  int mode = MT_DC_PRED, delta = 0;
  // rank_chroma_modes (superblock.rs:469-513) into DirectionalTopK (coder.rs:326-365), K = 3
  unsigned long long tc[3];
  int tm[3], tn = 0;
  int16_t* sp = w.s[1 - best].pred[0];
  for (int ci = 0; ci < kJointModes; ci++) {
    const int m = kJointList[ci];
    unsigned long long sc = 0;
    for (int pl = 0; pl < 2; pl++) {
      predict_sq<N>(P[pl].rec, p.stride, p.frame_w, p.frame_h, cx, cy, m, 0, have_tr, have_bl, ft, p.bd, sp, w.u);
      sc += satd_sad_proxy<N>(pl ? src_v : src_u, p.stride, cx, cy, sp, P[pl].vw, P[pl].vh);
    }
    int pos = tn < 3 ? tn : 2;
    if (tn == 3 && sc >= tc[pos]) continue;
    if (tn < 3) pos = tn++;
    while (pos > 0 && sc < tc[pos - 1]) {
      tc[pos] = tc[pos - 1];
      tm[pos] = tm[pos - 1];
      pos--;
    }
    tc[pos] = sc;
    tm[pos] = m;
  }
  for (int ci = 0; ci < kJointModes; ci++) {
    const int m = kJointList[ci];
    bool in = false;
    for (int e = 0; e < tn; e++) in |= tm[e] == m;
    if (!in) continue;
    const int tx = N == 32 ? MT_TX_DCT_DCT : chroma_tx(m);  // forced DCT_DCT at TX_32X32
    float total = __fmul_rn(dlam, uv_mode_bits(M, jb.y_mode, m, false, 0, 0));
    UvBigSlot<N>& c = w.s[1 - best];
    for (int pl = 0; pl < 2; pl++) {
      predict_sq<N>(P[pl].rec, p.stride, p.frame_w, p.frame_h, cx, cy, m, 0, have_tr, have_bl, ft, p.bd,
                    c.pred[pl], w.u);
      const PlaneCost pc = plane_chain<N>(a, P[pl], T, qm, sQs, sLut, tx, true, c.pred[pl], c.cf[pl], c.rr[pl], w);
      total = __fadd_rn(total, rd_cost_i64(pc.sse, dlam, pc.bits));
    }
    if (total < best_total) {
      best_total = total;
      mode = m;
      best = 1 - best;
    }
  }
  // the zone-2 angle deltas of a directional winner (uv_ad; uv_ad32 at 32x32)
  if (a.u.angle_deltas && directional(mode)) {
    const int m = mode, tx = N == 32 ? MT_TX_DCT_DCT : chroma_tx(m);
    int lo = 0, hi = -1;
    if (m == MT_V_PRED) lo = 1, hi = 3;
    else if (m == MT_H_PRED) lo = -3, hi = -1;
    else if (m == MT_D113_PRED || m == MT_D135_PRED || m == MT_D157_PRED) lo = -3, hi = 3;
    const float base_sig = __fsub_rn(uv_mode_bits(M, jb.y_mode, m, false, 0, 0), M.angle_delta[m - MT_V_PRED][3]);
    for (int d = lo; d <= hi; d++) {
      if (d == 0) continue;
      float total = __fmul_rn(dlam, __fadd_rn(base_sig, M.angle_delta[m - MT_V_PRED][d + 3]));
      UvBigSlot<N>& c = w.s[1 - best];
      for (int pl = 0; pl < 2; pl++) {
        predict_sq<N>(P[pl].rec, p.stride, p.frame_w, p.frame_h, cx, cy, m, d, false, false, ft, p.bd, c.pred[pl],
                      w.u);
        const PlaneCost pc = plane_chain<N>(a, P[pl], T, qm, sQs, sLut, tx, true, c.pred[pl], c.cf[pl], c.rr[pl], w);
        total = __fadd_rn(total, rd_cost_i64(pc.sse, dlam, pc.bits));
      }
      if (total < best_total) {
        best_total = total;
        delta = d;
        best = 1 - best;
      }
    }
  }
  r.total = best_total;
  r.dc_total = dc_total;
  r.cfl_total = cfl_total;
  r.uv_mode = (uint8_t)(mode != MT_DC_PRED ? mode : (use_cfl ? MT_UV_CFL_PRED : MT_DC_PRED));
  r.angle_delta = (int8_t)delta;
  r.cfl_alpha[0] = (int8_t)alpha[0];
  r.cfl_alpha[1] = (int8_t)alpha[1];
  const UvBigSlot<N>& b = w.s[best];
  if (cf_out)
    for (int pl = 0; pl < 2; pl++)
      for (int i = 0; i < NN; i++) cf_out[(size_t)j * 2 * NN + pl * NN + i] = b.cf[pl][i];
  if (rec_out)
    for (int pl = 0; pl < 2; pl++)
      for (int i = 0; i < NN; i++)
        rec_out[(size_t)j * 2 * NN + pl * NN + i] = (uint16_t)clampi((int32_t)b.pred[pl][i] + b.rr[pl][i], 0, maxv);
}

// ---- the 32x32 leaf at 4:2:0: pick_uv32_420 ----

// pick_uv32_420 (src/coder/block32.rs:2797-3120) with the shipped tuning on
// the 32x32 leaf's 16x16 chroma blocks: DC (the 4:2:0 context trellis,
// preserve_dc), CfL from the AC of the 32x32 luma reconstruction against
// DC, the 12 modes ranked by SATD into a top-3 priced in list order, then a
// directional winner's zone-2 deltas (uv_ad, uv_ad32; not after CfL); every
// total on the one chroma lambda.
__global__ void __launch_bounds__(kUvThreads) uv32_420_kernel(
    const uint16_t* __restrict__ src_u, const uint16_t* __restrict__ src_v, const uint16_t* __restrict__ rec_u,
    const uint16_t* __restrict__ rec_v, const uint16_t* __restrict__ luma, UvArgs a,
    const uint8_t* __restrict__ qm_row, const mt_coef_costs* __restrict__ costs,
    const mt_uv_mode_costs* __restrict__ mode_costs, const mt_uv16_444_job* __restrict__ jobs, int n,
    mt_uv16_result* __restrict__ res, int32_t* __restrict__ cf_out, uint16_t* __restrict__ rec_out, int arena) {
  __shared__ mt_coef_costs sT;
  __shared__ mt_uv_mode_costs sM;
  __shared__ uint8_t sQm[256];
  __shared__ float sQs[256];
  {
    const float* g = reinterpret_cast<const float*>(costs);
    float* s = reinterpret_cast<float*>(&sT);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
    const float* gm = reinterpret_cast<const float*>(mode_costs);
    float* sm = reinterpret_cast<float*>(&sM);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_uv_mode_costs) / 4); i += blockDim.x) sm[i] = gm[i];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
      const int wq = a.has_qm ? qm_row[i] : 32;
      sQm[i] = (uint8_t)wq;
      sQs[i] = fwd_qm_scale(wq);
    }
    __syncthreads();
  }
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const mt_split16_params& p = a.p;
  const mt_uv16_444_job jb = jobs[j];
  mt_uv16_result& r = res[j];
  const int cx = jb.px >> 1, cy = jb.py >> 1;
  const float kInf = __int_as_float(0x7f800000);
  const bool ok = (jb.px & 31) == 0 && (jb.py & 31) == 0 && cx + 16 <= p.frame_w && cy + 16 <= p.frame_h &&
                  jb.y_mode <= MT_PAETH_PRED;
  if (!ok) {
    r.total = r.dc_total = r.cfl_total = kInf;
    r.uv_mode = 255;
    r.angle_delta = 0;
    r.cfl_alpha[0] = r.cfl_alpha[1] = 0;
    if (cf_out)
      for (int i = 0; i < 512; i++) cf_out[(size_t)j * 512 + i] = 0;
    if (rec_out)
      for (int i = 0; i < 512; i++) rec_out[(size_t)j * 512 + i] = 0;
    return;
  }
  const mt_coef_costs& T = sT;
  const mt_uv_mode_costs& M = sM;
  const uint8_t* qm = a.has_qm ? sQm : nullptr;
  const int32_t maxv = (1 << p.bd) - 1;
  const float mlam = p.rd_lambda;
  const bool have_tr = jb.flags & MT_CAND_HAVE_TR, have_bl = jb.flags & MT_CAND_HAVE_BL;
  const bool ft = jb.flags & MT_CAND_FILTER_TYPE;
  const int vis_w = p.vis_w > 0 ? p.vis_w : p.frame_w, vis_h = p.vis_h > 0 ? p.vis_h : p.frame_h;
  UvPlane P[2];
  for (int pl = 0; pl < 2; pl++) {
    UvPlane& q = P[pl];
    q.src = (pl ? src_v : src_u) + (size_t)cy * p.stride + cx;
    q.rec = pl ? rec_v : rec_u;
    q.vw = min(max(vis_w - cx, 0), 16);
    q.vh = min(max(vis_h - cy, 0), 16);
    bool anz = false, lnz = false;
    int s = -8;
    for (int k = 0; k < 4; k++) {
      anz |= jb.a_coef[pl][k] != 0x40;
      lnz |= jb.l_coef[pl][k] != 0x40;
      s += (jb.a_coef[pl][k] >> 6) + (jb.l_coef[pl][k] >> 6);
    }
    q.sk = 7 + anz + lnz;
    q.ds = (s != 0) + (s > 0);
    q.skip1 = p.use_skip_bits ? p.skip_bits[q.sk][0] : 0.0f;
    q.skip0 = p.use_skip_bits ? p.skip_bits[q.sk][1] : 0.0f;
  }
  Uv444Work& w = smem_arena<Uv444Work>(arena);
  int best = 0;
  int32_t dc[2];
  float dc_total = 0.0f;
  for (int pl = 0; pl < 2; pl++) {
    predict_sq<16>(P[pl].rec, p.stride, p.frame_w, p.frame_h, cx, cy, MT_DC_PRED, 0, have_tr, have_bl, ft, p.bd,
                   w.s[0].pred[pl], w.u);
    dc[pl] = w.s[0].pred[pl][0];
    const PlaneCost c = plane_chain<16, true>(a, P[pl], T, qm, sQs, nullptr, MT_TX_DCT_DCT, true, w.s[0].pred[pl],
                                           w.s[0].cf[pl], w.s[0].rr[pl], w);
    dc_total = __fadd_rn(dc_total, rd_cost_i64(c.sse, mlam, c.bits));
  }
  float best_total = dc_total;
  int mode = MT_DC_PRED, delta = 0;
  bool use_cfl = false;
  // CfL: cfl_ac_sub of the 32x32 luma into 16x16
  {
    const int ls = a.u.luma_stride;
    const uint16_t* l = luma + (size_t)jb.py * ls + jb.px;
    int32_t sum = 128;
    for (int i = 0; i < 256; i++) {
      const int y = i >> 4, x = i & 15;
      const uint16_t* q = l + (size_t)(2 * y) * ls + 2 * x;
      const int32_t v = ((int32_t)q[0] + q[1] + q[ls] + q[ls + 1]) << 1;
      w.ac[i] = (int16_t)v;
      sum += v;
    }
    const int32_t mean = sum >> 8;
    for (int i = 0; i < 256; i++) w.ac[i] = (int16_t)(w.ac[i] - mean);
  }
  int alpha[2];
  for (int pl = 0; pl < 2; pl++) alpha[pl] = cfl_alpha_n<16>(w.ac, P[pl], p.stride, dc[pl], maxv);
  {
    Uv444Slot& c = w.s[1 - best];
    float body = 0.0f;
    for (int pl = 0; pl < 2; pl++) {
      for (int i = 0; i < 256; i++) c.pred[pl][i] = (int16_t)cfl_pred_pixel(dc[pl], w.ac[i], alpha[pl], maxv);
      const PlaneCost pc = plane_chain<16, true>(a, P[pl], T, qm, sQs, nullptr, MT_TX_DCT_DCT, false, c.pred[pl],
                                               c.cf[pl], c.rr[pl], w);
      body = __fadd_rn(body, rd_cost_i64(pc.sse, mlam, pc.bits));
    }
    const float cfl_total =
        __fsub_rn(__fadd_rn(body, __fmul_rn(mlam, uv_mode_bits(M, jb.y_mode, MT_UV_CFL_PRED, true, alpha[0], alpha[1]))),
                  __fmul_rn(mlam, uv_mode_bits(M, jb.y_mode, MT_DC_PRED, false, 0, 0)));
    r.cfl_total = cfl_total;
    if ((alpha[0] != 0 || alpha[1] != 0) && cfl_total < best_total) {
      best_total = cfl_total;
      use_cfl = true;
      best = 1 - best;
    }
  }
  // rank_chroma_modes into DirectionalTopK (K = 3), then the ranked modes in list order
  unsigned long long tc[3];
  int tm[3], tn = 0;
  int16_t* sp = w.s[1 - best].pred[0];
  for (int ci = 0; ci < kJointModes; ci++) {
    const int m = kJointList[ci];
    unsigned long long sc = 0;
    for (int pl = 0; pl < 2; pl++) {
      predict_sq<16>(P[pl].rec, p.stride, p.frame_w, p.frame_h, cx, cy, m, 0, have_tr, have_bl, ft, p.bd, sp, w.u);
      sc += satd_sad_proxy<16>(pl ? src_v : src_u, p.stride, cx, cy, sp, P[pl].vw, P[pl].vh);
    }
    int pos = tn < 3 ? tn : 2;
    if (tn == 3 && sc >= tc[pos]) continue;
    if (tn < 3) pos = tn++;
    while (pos > 0 && sc < tc[pos - 1]) {
      tc[pos] = tc[pos - 1];
      tm[pos] = tm[pos - 1];
      pos--;
    }
    tc[pos] = sc;
    tm[pos] = m;
  }
  for (int ci = 0; ci < kJointModes; ci++) {
    const int m = kJointList[ci];
    bool in = false;
    for (int e = 0; e < tn; e++) in |= tm[e] == m;
    if (!in) continue;
    const int tx = chroma_tx(m);
    float total = __fmul_rn(mlam, uv_mode_bits(M, jb.y_mode, m, false, 0, 0));
    Uv444Slot& c = w.s[1 - best];
    for (int pl = 0; pl < 2; pl++) {
      predict_sq<16>(P[pl].rec, p.stride, p.frame_w, p.frame_h, cx, cy, m, 0, have_tr, have_bl, ft, p.bd,
                     c.pred[pl], w.u);
      const PlaneCost pc =
          plane_chain<16, true>(a, P[pl], T, qm, sQs, nullptr, tx, true, c.pred[pl], c.cf[pl], c.rr[pl], w);
      total = __fadd_rn(total, rd_cost_i64(pc.sse, mlam, pc.bits));
    }
    if (total < best_total) {
      best_total = total;
      mode = m;
      use_cfl = false;
      best = 1 - best;
    }
  }
  if (!use_cfl && a.u.angle_deltas && directional(mode)) {
    const int m = mode, tx = chroma_tx(m);
    int lo = 0, hi = -1;
    if (m == MT_V_PRED) lo = 1, hi = 3;
    else if (m == MT_H_PRED) lo = -3, hi = -1;
    else if (m == MT_D113_PRED || m == MT_D135_PRED || m == MT_D157_PRED) lo = -3, hi = 3;
    const float base_sig = __fsub_rn(uv_mode_bits(M, jb.y_mode, m, false, 0, 0), M.angle_delta[m - MT_V_PRED][3]);
    for (int d = lo; d <= hi; d++) {
      if (d == 0) continue;
      float total = __fmul_rn(mlam, __fadd_rn(base_sig, M.angle_delta[m - MT_V_PRED][d + 3]));
      Uv444Slot& c = w.s[1 - best];
      for (int pl = 0; pl < 2; pl++) {
        predict_sq<16>(P[pl].rec, p.stride, p.frame_w, p.frame_h, cx, cy, m, d, false, false, ft, p.bd, c.pred[pl],
                       w.u);
        const PlaneCost pc =
            plane_chain<16, true>(a, P[pl], T, qm, sQs, nullptr, tx, true, c.pred[pl], c.cf[pl], c.rr[pl], w);
        total = __fadd_rn(total, rd_cost_i64(pc.sse, mlam, pc.bits));
      }
      if (total < best_total) {
        best_total = total;
        delta = d;
        best = 1 - best;
      }
    }
  }
  r.total = best_total;
  r.dc_total = dc_total;
  r.uv_mode = (uint8_t)(use_cfl ? MT_UV_CFL_PRED : mode);
  r.angle_delta = (int8_t)delta;
  r.cfl_alpha[0] = (int8_t)alpha[0];
  r.cfl_alpha[1] = (int8_t)alpha[1];
  const Uv444Slot& b = w.s[best];
  if (cf_out)
    for (int pl = 0; pl < 2; pl++)
      for (int i = 0; i < 256; i++) cf_out[(size_t)j * 512 + pl * 256 + i] = b.cf[pl][i];
  if (rec_out)
    for (int pl = 0; pl < 2; pl++)
      for (int i = 0; i < 256; i++)
        rec_out[(size_t)j * 512 + pl * 256 + i] = (uint16_t)clampi((int32_t)b.pred[pl][i] + b.rr[pl][i], 0, maxv);
}

int uv_check(const mt_split16_params* p, const mt_uv16_params* u, const mt_quant* q, int32_t n) {
  if (!p || !u || !q || n < 0) return MT_ERR_INVALID_INPUT;
  if (p->bd != 8) return MT_ERR_UNSUPPORTED;
  if (p->frame_w < 8 || p->frame_h < 8 || p->stride < p->frame_w || p->vis_w < 0 || p->vis_h < 0)
    return MT_ERR_INVALID_INPUT;
  if (u->luma_stride < 2 * p->frame_w) return MT_ERR_INVALID_INPUT;
  if (!(p->rd_lambda > 0.0f) || !(p->wsse_scale >= 0.0f)) return MT_ERR_INVALID_INPUT;
  return MT_OK;
}

// 4:4:4: the chroma planes have the luma size, so the luma stride needs only
// the frame width.
int uv_check_444(const mt_split16_params* p, const mt_uv16_params* u, const mt_quant* q, int32_t n) {
  if (!p || !u || !q || n < 0) return MT_ERR_INVALID_INPUT;
  if (p->bd != 8) return MT_ERR_UNSUPPORTED;
  if (p->frame_w < 16 || p->frame_h < 16 || p->stride < p->frame_w || p->vis_w < 0 || p->vis_h < 0)
    return MT_ERR_INVALID_INPUT;
  if (u->luma_stride < p->frame_w) return MT_ERR_INVALID_INPUT;
  if (!(p->rd_lambda > 0.0f) || !(p->wsse_scale >= 0.0f)) return MT_ERR_INVALID_INPUT;
  return MT_OK;
}

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

template <int N, typename J>
int uv444_device(const uint16_t* su, const uint16_t* sv, const uint16_t* ru, const uint16_t* rv, const uint16_t* luma,
                 const mt_split16_params* prm, const mt_uv16_params* uvp, const mt_quant* quant, const uint8_t* d_qm,
                 const mt_coef_costs* d_costs, const mt_uv_mode_costs* d_mc, const J* d_jobs, int32_t n,
                 mt_uv16_result* d_res, int32_t* d_cf, uint16_t* d_rec, void* stream) {
  const int rc = uv_check_444(prm, uvp, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!su || !sv || !ru || !rv || !luma || !d_costs || !d_mc || !d_jobs || !d_res) return MT_ERR_INVALID_INPUT;
  if (!(uvp->dir_lambda > 0.0f) || prm->frame_w < N || prm->frame_h < N) return MT_ERR_INVALID_INPUT;
  UvArgs a;
  a.p = *prm;
  a.u = *uvp;
  a.q = *quant;
  a.lambda = prm->trellis_lambda0 > 0.0f ? mth::scaled_trellis_lambda_host((float)quant->dc_q, prm->trellis_lambda0)
                                         : 0.0f;
  a.has_qm = quant->qm_level < 15 && d_qm != nullptr;
  const int stride = arena_stride(sizeof(UvBigWork<N>));
  auto* kern = uv444_kernel<N, J>;
  int threads = 0;
  size_t dyn = 0;
  if (!arena_launch_shape(kern, n, stride, kUvThreads, &threads, &dyn)) return MT_ERR_DEVICE;
  kern<<<(unsigned)((n + threads - 1) / threads), threads, dyn, reinterpret_cast<cudaStream_t>(stream)>>>(
      su, sv, ru, rv, luma, a, d_qm, d_costs, d_mc, d_jobs, n, d_res, d_cf, d_rec, stride);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int uv32_device(const uint16_t* su, const uint16_t* sv, const uint16_t* ru, const uint16_t* rv, const uint16_t* luma,
                const mt_split16_params* prm, const mt_uv16_params* uvp, const mt_quant* quant, const uint8_t* d_qm,
                const mt_coef_costs* d_costs, const mt_uv_mode_costs* d_mc, const mt_uv16_444_job* d_jobs, int32_t n,
                mt_uv16_result* d_res, int32_t* d_cf, uint16_t* d_rec, void* stream) {
  const int rc = uv_check(prm, uvp, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!su || !sv || !ru || !rv || !luma || !d_costs || !d_mc || !d_jobs || !d_res) return MT_ERR_INVALID_INPUT;
  UvArgs a;
  a.p = *prm;
  a.u = *uvp;
  a.q = *quant;
  a.lambda = prm->trellis_lambda0 > 0.0f ? mth::scaled_trellis_lambda_host((float)quant->dc_q, prm->trellis_lambda0)
                                         : 0.0f;
  a.has_qm = quant->qm_level < 15 && d_qm != nullptr;
  const int stride = arena_stride(sizeof(Uv444Work));
  int threads = 0;
  size_t dyn = 0;
  if (!arena_launch_shape(uv32_420_kernel, n, stride, kUvThreads, &threads, &dyn)) return MT_ERR_DEVICE;
  uv32_420_kernel<<<(unsigned)((n + threads - 1) / threads), threads, dyn, reinterpret_cast<cudaStream_t>(stream)>>>(
      su, sv, ru, rv, luma, a, d_qm, d_costs, d_mc, d_jobs, n, d_res, d_cf, d_rec, stride);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int uv16_device(const uint16_t* su, const uint16_t* sv, const uint16_t* ru, const uint16_t* rv, const uint16_t* luma,
                const mt_split16_params* prm, const mt_uv16_params* uvp, const mt_quant* quant, const uint8_t* d_qm,
                const mt_coef_costs* d_costs, const mt_uv_mode_costs* d_mc, const mt_uv16_job* d_jobs, int32_t n,
                mt_uv16_result* d_res, int32_t* d_cf, uint16_t* d_rec, void* stream) {
  const int rc = uv_check(prm, uvp, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!su || !sv || !ru || !rv || !luma || !d_costs || !d_mc || !d_jobs || !d_res) return MT_ERR_INVALID_INPUT;
  UvArgs a;
  a.p = *prm;
  a.u = *uvp;
  a.q = *quant;
  a.lambda = prm->trellis_lambda0 > 0.0f ? mth::scaled_trellis_lambda_host((float)quant->dc_q, prm->trellis_lambda0)
                                         : 0.0f;
  a.has_qm = quant->qm_level < 15 && d_qm != nullptr;
  const int stride = arena_stride(sizeof(UvWork));
  int threads = 0;
  size_t dyn = 0;
  if (!arena_launch_shape(uv16_420_kernel, n, stride, kUvThreads, &threads, &dyn)) return MT_ERR_DEVICE;
  uv16_420_kernel<<<(unsigned)((n + threads - 1) / threads), threads, dyn, reinterpret_cast<cudaStream_t>(stream)>>>(
      su, sv, ru, rv, luma, a, d_qm, d_costs, d_mc, d_jobs, n, d_res, d_cf, d_rec, stride);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

// Host-buffer form of either search: the planes, tables and jobs copied to one
// device allocation, the launch, the results (and levels / reconstruction,
// per_job entries each) copied back.
template <typename J, typename L>
int uv_host(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
            const uint16_t* luma, size_t luma_rows, const mt_split16_params* prm, const mt_uv16_params* uvp,
            const mt_quant* quant, const uint8_t* qm_row, size_t qm_len, const mt_coef_costs* costs,
            const mt_uv_mode_costs* mode_costs, const J* jobs, int32_t n, mt_uv16_result* results, int32_t* cf_out,
            uint16_t* rec_out, size_t per_job, L launch) {
  if (!prm || !uvp || !quant || n < 0) return MT_ERR_INVALID_INPUT;
  if (n == 0) return MT_OK;
  if (!src_u || !src_v || !rec_u || !rec_v || !luma || !costs || !mode_costs || !jobs || !results)
    return MT_ERR_INVALID_INPUT;
  if (prm->stride <= 0 || prm->frame_h <= 0 || uvp->luma_stride <= 0) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)prm->stride * prm->frame_h * 2;
  const size_t lplane = (size_t)uvp->luma_stride * luma_rows * 2;
  size_t o = 0;
  const size_t o_su = o, o_sv = (o += up256(plane)), o_ru = (o += up256(plane)), o_rv = (o += up256(plane));
  const size_t o_l = (o += up256(plane)), o_qm = (o += up256(lplane)), o_c = (o += up256(qm_len));
  const size_t o_mc = (o += up256(sizeof(mt_coef_costs))), o_j = (o += up256(sizeof(mt_uv_mode_costs)));
  const size_t o_r = (o += up256((size_t)n * sizeof(J)));
  const size_t o_cf = (o += up256((size_t)n * sizeof(mt_uv16_result)));
  const size_t o_rec = (o += cf_out ? up256((size_t)n * per_job * 4) : 0);
  const size_t total = o + (rec_out ? up256((size_t)n * per_job * 2) : 0);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, total) != cudaSuccess) return MT_ERR_ALLOC;
  const bool has_qm = quant->qm_level < 15 && qm_row != nullptr;
  cudaError_t e = cudaMemcpy(d + o_su, src_u, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_sv, src_v, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_ru, rec_u, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_rv, rec_v, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_l, luma, lplane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && has_qm) e = cudaMemcpy(d + o_qm, qm_row, qm_len, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_c, costs, sizeof(mt_coef_costs), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_mc, mode_costs, sizeof(mt_uv_mode_costs), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_j, jobs, (size_t)n * sizeof(J), cudaMemcpyHostToDevice);
  int rc = MT_OK;
  if (e == cudaSuccess) {
    auto U = [&](size_t off) { return reinterpret_cast<const uint16_t*>(d + off); };
    rc = launch(U(o_su), U(o_sv), U(o_ru), U(o_rv), U(o_l), has_qm ? d + o_qm : nullptr,
                reinterpret_cast<const mt_coef_costs*>(d + o_c), reinterpret_cast<const mt_uv_mode_costs*>(d + o_mc),
                reinterpret_cast<const J*>(d + o_j), reinterpret_cast<mt_uv16_result*>(d + o_r),
                cf_out ? reinterpret_cast<int32_t*>(d + o_cf) : nullptr,
                rec_out ? reinterpret_cast<uint16_t*>(d + o_rec) : nullptr);
    if (rc == MT_OK) e = cudaMemcpy(results, d + o_r, (size_t)n * sizeof(mt_uv16_result), cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && cf_out)
      e = cudaMemcpy(cf_out, d + o_cf, (size_t)n * per_job * 4, cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && rec_out)
      e = cudaMemcpy(rec_out, d + o_rec, (size_t)n * per_job * 2, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // namespace

extern "C" {

int mt_pick_uv16_420_device(const uint16_t* d_src_u, const uint16_t* d_src_v, const uint16_t* d_rec_u,
                            const uint16_t* d_rec_v, const uint16_t* d_luma, const mt_split16_params* prm,
                            const mt_uv16_params* uvp, const mt_quant* quant, const uint8_t* d_qm_row,
                            const mt_coef_costs* d_costs, const mt_uv_mode_costs* d_mode_costs,
                            const mt_uv16_job* d_jobs, int32_t n, mt_uv16_result* d_results, int32_t* d_cf,
                            uint16_t* d_rec, void* stream) {
  return uv16_device(d_src_u, d_src_v, d_rec_u, d_rec_v, d_luma, prm, uvp, quant, d_qm_row, d_costs, d_mode_costs,
                     d_jobs, n, d_results, d_cf, d_rec, stream);
}

int mt_pick_uv16_420(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* prm, const mt_uv16_params* uvp,
                     const mt_quant* quant, const uint8_t* qm_row, const mt_coef_costs* costs,
                     const mt_uv_mode_costs* mode_costs, const mt_uv16_job* jobs, int32_t n,
                     mt_uv16_result* results, int32_t* cf_out, uint16_t* rec_out) {
  const int rc = uv_check(prm, uvp, quant, n);
  if (rc != MT_OK) return rc;
  return uv_host(src_u, src_v, rec_u, rec_v, luma, 2 * (size_t)prm->frame_h, prm, uvp, quant, qm_row, 64, costs,
                 mode_costs, jobs, n, results, cf_out, rec_out, 128,
                 [&](const uint16_t* su, const uint16_t* sv, const uint16_t* ru, const uint16_t* rv, const uint16_t* l,
                     const uint8_t* qm, const mt_coef_costs* c, const mt_uv_mode_costs* mc, const mt_uv16_job* j,
                     mt_uv16_result* r, int32_t* cf, uint16_t* rec) {
                   return uv16_device(su, sv, ru, rv, l, prm, uvp, quant, qm, c, mc, j, n, r, cf, rec, nullptr);
                 });
}

int mt_pick_uv32_444_device(const uint16_t* d_src_u, const uint16_t* d_src_v, const uint16_t* d_rec_u,
                            const uint16_t* d_rec_v, const uint16_t* d_luma, const mt_split16_params* prm,
                            const mt_uv16_params* uvp, const mt_quant* quant, const uint8_t* d_qm_row,
                            const mt_coef_costs* d_costs, const mt_uv_mode_costs* d_mode_costs,
                            const mt_uv32_444_job* d_jobs, int32_t n, mt_uv16_result* d_results, int32_t* d_cf,
                            uint16_t* d_rec, void* stream) {
  return uv444_device<32>(d_src_u, d_src_v, d_rec_u, d_rec_v, d_luma, prm, uvp, quant, d_qm_row, d_costs,
                          d_mode_costs, d_jobs, n, d_results, d_cf, d_rec, stream);
}

int mt_pick_uv32_444(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* prm, const mt_uv16_params* uvp,
                     const mt_quant* quant, const uint8_t* qm_row, const mt_coef_costs* costs,
                     const mt_uv_mode_costs* mode_costs, const mt_uv32_444_job* jobs, int32_t n,
                     mt_uv16_result* results, int32_t* cf_out, uint16_t* rec_out) {
  const int rc = uv_check_444(prm, uvp, quant, n);
  if (rc != MT_OK) return rc;
  if (n > 0 && !(uvp->dir_lambda > 0.0f)) return MT_ERR_INVALID_INPUT;
  return uv_host(src_u, src_v, rec_u, rec_v, luma, (size_t)prm->frame_h, prm, uvp, quant, qm_row, 1024, costs,
                 mode_costs, jobs, n, results, cf_out, rec_out, 2048,
                 [&](const uint16_t* su, const uint16_t* sv, const uint16_t* ru, const uint16_t* rv, const uint16_t* l,
                     const uint8_t* qm, const mt_coef_costs* c, const mt_uv_mode_costs* mc,
                     const mt_uv32_444_job* j, mt_uv16_result* r, int32_t* cf, uint16_t* rec) {
                   return uv444_device<32>(su, sv, ru, rv, l, prm, uvp, quant, qm, c, mc, j, n, r, cf, rec, nullptr);
                 });
}

int mt_pick_uv32_420_device(const uint16_t* d_src_u, const uint16_t* d_src_v, const uint16_t* d_rec_u,
                            const uint16_t* d_rec_v, const uint16_t* d_luma, const mt_split16_params* prm,
                            const mt_uv16_params* uvp, const mt_quant* quant, const uint8_t* d_qm_row,
                            const mt_coef_costs* d_costs, const mt_uv_mode_costs* d_mode_costs,
                            const mt_uv32_420_job* d_jobs, int32_t n, mt_uv16_result* d_results, int32_t* d_cf,
                            uint16_t* d_rec, void* stream) {
  return uv32_device(d_src_u, d_src_v, d_rec_u, d_rec_v, d_luma, prm, uvp, quant, d_qm_row, d_costs, d_mode_costs,
                     d_jobs, n, d_results, d_cf, d_rec, stream);
}

int mt_pick_uv32_420(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* prm, const mt_uv16_params* uvp,
                     const mt_quant* quant, const uint8_t* qm_row, const mt_coef_costs* costs,
                     const mt_uv_mode_costs* mode_costs, const mt_uv32_420_job* jobs, int32_t n,
                     mt_uv16_result* results, int32_t* cf_out, uint16_t* rec_out) {
  const int rc = uv_check(prm, uvp, quant, n);
  if (rc != MT_OK) return rc;
  return uv_host(src_u, src_v, rec_u, rec_v, luma, 2 * (size_t)prm->frame_h, prm, uvp, quant, qm_row, 256, costs,
                 mode_costs, jobs, n, results, cf_out, rec_out, 512,
                 [&](const uint16_t* su, const uint16_t* sv, const uint16_t* ru, const uint16_t* rv, const uint16_t* l,
                     const uint8_t* qm, const mt_coef_costs* c, const mt_uv_mode_costs* mc,
                     const mt_uv32_420_job* j, mt_uv16_result* r, int32_t* cf, uint16_t* rec) {
                   return uv32_device(su, sv, ru, rv, l, prm, uvp, quant, qm, c, mc, j, n, r, cf, rec, nullptr);
                 });
}

int mt_pick_uv16_444_device(const uint16_t* d_src_u, const uint16_t* d_src_v, const uint16_t* d_rec_u,
                            const uint16_t* d_rec_v, const uint16_t* d_luma, const mt_split16_params* prm,
                            const mt_uv16_params* uvp, const mt_quant* quant, const uint8_t* d_qm_row,
                            const mt_coef_costs* d_costs, const mt_uv_mode_costs* d_mode_costs,
                            const mt_uv16_444_job* d_jobs, int32_t n, mt_uv16_result* d_results, int32_t* d_cf,
                            uint16_t* d_rec, void* stream) {
  return uv444_device<16>(d_src_u, d_src_v, d_rec_u, d_rec_v, d_luma, prm, uvp, quant, d_qm_row, d_costs,
                          d_mode_costs, d_jobs, n, d_results, d_cf, d_rec, stream);
}

int mt_pick_uv16_444(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* prm, const mt_uv16_params* uvp,
                     const mt_quant* quant, const uint8_t* qm_row, const mt_coef_costs* costs,
                     const mt_uv_mode_costs* mode_costs, const mt_uv16_444_job* jobs, int32_t n,
                     mt_uv16_result* results, int32_t* cf_out, uint16_t* rec_out) {
  const int rc = uv_check_444(prm, uvp, quant, n);
  if (rc != MT_OK) return rc;
  if (n > 0 && !(uvp->dir_lambda > 0.0f)) return MT_ERR_INVALID_INPUT;
  return uv_host(src_u, src_v, rec_u, rec_v, luma, (size_t)prm->frame_h, prm, uvp, quant, qm_row, 256, costs,
                 mode_costs, jobs, n, results, cf_out, rec_out, 512,
                 [&](const uint16_t* su, const uint16_t* sv, const uint16_t* ru, const uint16_t* rv, const uint16_t* l,
                     const uint8_t* qm, const mt_coef_costs* c, const mt_uv_mode_costs* mc,
                     const mt_uv16_444_job* j, mt_uv16_result* r, int32_t* cf, uint16_t* rec) {
                   return uv444_device<16>(su, sv, ru, rv, l, prm, uvp, quant, qm, c, mc, j, n, r, cf, rec, nullptr);
                 });
}

}  // extern "C"
