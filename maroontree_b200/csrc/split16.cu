// The 16x16 leaf's TX_8X8 split trial (split16_luma_try,
// src/coder/partition_search.rs:4235-4428), batched over (block, mode) jobs,
// and a batched trellis_optimize_ctx.
//
// split16_kernel: one thread per job.  The four 8x8 quadrants run in raster
// order; each is predicted through PatchRead (the reconstruction with the
// quadrants already trial-coded laid over it, kept in the thread's 256-byte
// patch), transformed, trellised, inverse-transformed and measured; with the
// type search its six more types are gated on SSE before their rate is
// walked.  The winner's coefficient result context updates the thread's
// above / left context bytes for the next quadrant.  Launches order jobs as
// the caller lists them; a caller that lists them mode-major (every block for
// one mode, then the next mode) gives warps one prediction path.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/maroontree_b200.h"
#include "leaf8.cuh"
#include "wsse.cuh"

namespace mth {
float scaled_trellis_lambda_host(float dc_q, float lambda0);
}

namespace {

using namespace mtd;

constexpr int kSplitThreads = 128;
// Resident CTAs per SM each kernel is compiled for (measured on the 1080p
// level: the DCT-only path is fastest at six, 85 registers a thread; the type
// search, with far more live state, at three, no register cap).
constexpr int kSplitMinBlocksDct = 6, kSplitMinBlocksSearch = 3;

// Sample (x, y) of the reconstruction with the job's 16x16 trial patch at
// (px, py) laid over it.
template <int S>
struct PatchReadS {
  const uint16_t* __restrict__ plane;
  int stride, px, py;
  const uint8_t* patch;  // S x S, row-major
  __device__ __forceinline__ int32_t operator()(int x, int y) const {
    const unsigned dx = (unsigned)(x - px), dy = (unsigned)(y - py);
    return (dx < (unsigned)S && dy < (unsigned)S) ? (int32_t)patch[dy * S + dx]
                                                  : (int32_t)plane[(size_t)y * stride + x];
  }
};
using PatchRead = PatchReadS<16>;

struct SplitArgs {
  mt_split16_params p;
  mt_quant q;
  float lambda;  // scaled_trellis_lambda of the trellis (0: trellis off)
  int has_qm;
};

// Per-thread working set of one job.  u: the prediction edges while a
// quadrant is predicted, then the targets (u[0, 64)) and the transform
// temporary (u[64, 128)).
struct SplitWork {
  int32_t u[128];
  int16_t pred[64], resid[64];
  int16_t cfs[2][64], rrs[2][64];  // levels / inverse of the candidate and of the winner
  TrellisCtxScratch tr;
  uint8_t lv[160];
  uint8_t patch[256];
};

template <int B = 16>
__device__ __forceinline__ bool job_ok(const mt_split16_job& jb, int fw, int fh) {
  if (jb.px + B > fw || jb.py + B > fh || jb.mode > MT_PAETH_PRED) return false;
  if (jb.angle_delta < -3 || jb.angle_delta > 3) return false;
  return jb.angle_delta == 0 || (jb.mode >= MT_V_PRED && jb.mode <= MT_D67_PRED);
}

// lossy_state.rs:1367-1386 skip_ctx_split (2 x 2 span; kSkipCtxTbl indexed
// by the OR of the above / left context bytes without the dc-sign bits, each
// capped at 4) and :1388-1405 dc_sign_ctx_span.
__device__ __forceinline__ int skip_ctx_split2(uint32_t a0, uint32_t a1, uint32_t l0, uint32_t l1) {
  const uint32_t la = (a0 | a1) & 0x3f, ll = (l0 | l1) & 0x3f;
  return kSkipCtxTbl[min(la, 4u)][min(ll, 4u)];
}
__device__ __forceinline__ int dc_sign_ctx2(uint32_t a0, uint32_t a1, uint32_t l0, uint32_t l1) {
  const int s = (int)(a0 >> 6) + (int)(a1 >> 6) + (int)(l0 >> 6) + (int)(l1 >> 6) - 4;
  return (s != 0) + (s > 0);
}

__device__ __forceinline__ float rd_cost_i64(long long d, float lam, float rate) {
  return __fadd_rn((float)d, __fmul_rn(lam, rate));
}

// SEARCH: the 4:4:4 type search is compiled in (a separate kernel keeps the
// DCT-only path small for the instruction cache).
template <bool SEARCH>
__global__ void __launch_bounds__(kSplitThreads, SEARCH ? kSplitMinBlocksSearch : kSplitMinBlocksDct) split16_kernel(
    const uint16_t* __restrict__ src, const uint16_t* __restrict__ rec, SplitArgs a,
    const uint8_t* __restrict__ qm_row, const mt_coef_costs* __restrict__ costs,
    const mt_split16_job* __restrict__ jobs, int n, mt_split16_result* __restrict__ res, int32_t* __restrict__ cf_out,
    uint16_t* __restrict__ rec_out) {
  __shared__ mt_coef_costs sT;
  __shared__ uint8_t sQm[64];
  __shared__ float sQs[64];
  {
    const float* g = reinterpret_cast<const float*>(costs);
    float* s = reinterpret_cast<float*>(&sT);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
    if (threadIdx.x < 64) {
      const int w = a.has_qm ? qm_row[threadIdx.x] : 32;
      sQm[threadIdx.x] = (uint8_t)w;
      sQs[threadIdx.x] = fwd_qm_scale(w);
    }
    __syncthreads();
  }
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const mt_split16_params& p = a.p;
  const mt_quant& q = a.q;
  const mt_coef_costs& T = sT;
  const uint8_t* qm = a.has_qm ? sQm : nullptr;
  const mt_split16_job jb = jobs[j];
  mt_split16_result& r = res[j];
  if (!job_ok(jb, p.frame_w, p.frame_h)) {
    r.sse = 0;
    r.bits = 0.0f;
    *reinterpret_cast<uint32_t*>(r.tx_types) = 0xffffffffu;
    if (cf_out)
      for (int i = 0; i < 256; i++) cf_out[(size_t)j * 256 + i] = 0;
    if (rec_out)
      for (int i = 0; i < 256; i++) rec_out[(size_t)j * 256 + i] = 0;
    return;
  }
  SplitWork w;
  uint32_t actx[4], lctx[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    actx[i] = jb.a_coef[i];
    lctx[i] = jb.l_coef[i];
  }
  const bool have_tr = jb.flags & MT_CAND_HAVE_TR, have_bl = jb.flags & MT_CAND_HAVE_BL;
  const bool ft = jb.flags & MT_CAND_FILTER_TYPE;
  const int32_t maxv = (1 << p.bd) - 1;
  const float dcq = (float)q.dc_q, acq = (float)q.ac_q, rd_lam = p.rd_lambda;
  const bool qm_full = q.qm_level >= 5;
  const int vis_w = p.vis_w > 0 ? p.vis_w : p.frame_w, vis_h = p.vis_h > 0 ? p.vis_h : p.frame_h;
  const PatchRead rd{rec, p.stride, jb.px, jb.py, w.patch};
  long long sse_sum = 0;
  float bits_sum = 0.0f;
  uint32_t txtps = 0;
  for (int qi = 0; qi < 4; qi++) {
    const int sx = (qi & 1) * 8, sy = (qi >> 1) * 8, bx = jb.px + sx, by = jb.py + sy;
    const bool tr = qi == 0 ? jb.py > 0 : (qi == 1 ? have_tr : qi == 2);
    const bool bl = qi == 0 ? jb.px > 0 : (qi == 2 ? have_bl : false);
    predict_sq_at<8>(rd, p.frame_w, p.frame_h, bx, by, jb.mode, jb.angle_delta, tr, bl, ft, p.bd, w.pred, w.u);
#pragma unroll 8
    for (int i = 0; i < 64; i++)
      w.resid[i] = (int16_t)((int32_t)src[(size_t)(by + (i >> 3)) * p.stride + bx + (i & 7)] - w.pred[i]);
    const int ax = sx >> 2, ly = sy >> 2;
    const int sk = skip_ctx_split2(actx[ax], actx[ax + 1], lctx[ly], lctx[ly + 1]);
    const int ds = dc_sign_ctx2(actx[ax], actx[ax + 1], lctx[ly], lctx[ly + 1]);
    ErrBlock<int16_t, int16_t> eb;
    eb.src = src + (size_t)by * p.stride + bx;
    eb.stride = p.stride;
    eb.pred = w.pred;
    eb.w = 8;
    eb.vw = min(max(vis_w - bx, 0), 8);
    eb.vh = min(max(vis_h - by, 0), 8);
    eb.maxv = maxv;
    const float skip1 = p.use_skip_bits ? p.skip_bits[sk][0] : 0.0f;
    const float skip0 = p.use_skip_bits ? p.skip_bits[sk][1] : 0.0f;
    float* tf = reinterpret_cast<float*>(w.u);
    int32_t* tmp = w.u + 64;
    // The types in the reference's order: DCT_DCT (trellised; every other
    // type is gated against it), then with SEARCH ADST_ADST, ADST_DCT,
    // DCT_ADST (trellised), IDTX, V_DCT, H_DCT (not trellised).  One loop body
    // keeps one copy of each stage in the code; the candidate and the current
    // winner live in the two slots of cfs / rrs.
    constexpr int kTypes = SEARCH ? 7 : 1;
    constexpr uint32_t kTypeOrder = 0x3206541u;  // nibble k: the k-th type
    int best = 0, btx = MT_TX_DCT_DCT;
    long long bsse = 0, dct_sse = 0, guard = 0;
    float bbits = 0.0f;
#pragma unroll 1
    for (int k = 0; k < kTypes; k++) {
      const int t = (int)((kTypeOrder >> (4 * k)) & 15u);
      const int cur = k == 0 ? 0 : 1 - best;
      int16_t* cf = w.cfs[cur];
      int16_t* rr = w.rrs[cur];
      fwd8x8(w.resid, t, q, cf, tf, tmp);
      if (t == MT_TX_DCT_DCT || t >= MT_TX_ADST_ADST) {
        if (qm) apply_qm(cf, tf, sQs, 64);
        if (a.lambda > 0.0f) trellis_ctx8(cf, tf, dcq, acq, a.lambda, T, ds, qm, qm_full, p.band_tilt, w.tr);
      }
      inv8x8(cf, t, q, qm, rr, tmp);
      eb.resid = rr;
      const long long asse = sse_recon_block(eb, p.wsse_scale);
      if (k > 0 && !(t >= MT_TX_ADST_ADST ? asse <= dct_sse + guard : asse <= bsse)) continue;
      const float best_rd = k == 0 ? 0.0f : rd_cost_i64(bsse, rd_lam, bbits);
      float abits;
      if (t == MT_TX_V_DCT || t == MT_TX_H_DCT) {
        abits = rate_1d<8>(cf, t == MT_TX_V_DCT, T, ds, jb.mode, w.lv);
      } else {
        const float bound =
            k == 0 ? __int_as_float(0x7f800000) : __fdiv_rn(__fsub_rn(best_rd, (float)asse), rd_lam);
        abits = rate_bounded<8>(cf, T, sk, ds, jb.mode, t, p.use_skip_bits != 0, skip1, skip0, bound, w.lv);
      }
      if (k == 0 || rd_cost_i64(asse, rd_lam, abits) < best_rd) {
        best = cur;
        bsse = asse;
        bbits = abits;
        btx = t;
      }
      if (k == 0) {
        dct_sse = asse;
        guard = p.tx_guard_shift >= 63 ? 0 : (asse >> p.tx_guard_shift);
      }
    }
    const int16_t* bcf = w.cfs[best];
    const int16_t* brr = w.rrs[best];
    txtps |= (uint32_t)btx << (8 * qi);
    sse_sum += bsse;
    bits_sum = __fadd_rn(bits_sum, bbits);
    const uint32_t res_ctx = coef_res_ctx8(bcf);
    actx[ax] = actx[ax + 1] = res_ctx;
    lctx[ly] = lctx[ly + 1] = res_ctx;
#pragma unroll 8
    for (int i = 0; i < 64; i++)
      w.patch[(sy + (i >> 3)) * 16 + sx + (i & 7)] = (uint8_t)clampi((int32_t)w.pred[i] + brr[i], 0, maxv);
    if (cf_out) {
      int4* o = reinterpret_cast<int4*>(cf_out + (size_t)j * 256 + qi * 64);
#pragma unroll
      for (int i = 0; i < 16; i++) o[i] = make_int4(bcf[4 * i], bcf[4 * i + 1], bcf[4 * i + 2], bcf[4 * i + 3]);
    }
  }
  r.sse = sse_sum;
  r.bits = bits_sum;
  *reinterpret_cast<uint32_t*>(r.tx_types) = txtps;
  if (rec_out) {
    uint2* o = reinterpret_cast<uint2*>(rec_out + (size_t)j * 256);
#pragma unroll 4
    for (int i = 0; i < 64; i++)
      o[i] = make_uint2(w.patch[4 * i] | ((uint32_t)w.patch[4 * i + 1] << 16),
                        w.patch[4 * i + 2] | ((uint32_t)w.patch[4 * i + 3] << 16));
  }
}

__global__ void __launch_bounds__(kSplitThreads) trellis_ctx_kernel(int32_t* __restrict__ levels,
                                                                   const float* __restrict__ targets,
                                                                   const uint8_t* __restrict__ dcs_ctx, int n,
                                                                   float dc_q, float ac_q, float lambda,
                                                                   const uint8_t* __restrict__ qm_row, int has_qm,
                                                                   int qm_full, const mt_coef_costs* __restrict__ costs,
                                                                   float band_tilt) {
  __shared__ mt_coef_costs sT;
  __shared__ uint8_t sQm[64];
  {
    const float* g = reinterpret_cast<const float*>(costs);
    float* s = reinterpret_cast<float*>(&sT);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
    if (threadIdx.x < 64) sQm[threadIdx.x] = has_qm ? qm_row[threadIdx.x] : 32;
    __syncthreads();
  }
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int32_t cf[64];
  float tf[64];
#pragma unroll 8
  for (int i = 0; i < 64; i++) {
    cf[i] = levels[(size_t)b * 64 + i];
    tf[i] = targets[(size_t)b * 64 + i];
  }
  const int dcs = dcs_ctx[b] < 3 ? dcs_ctx[b] : 0;
  TrellisCtxScratch s;
  trellis_ctx8(cf, tf, dc_q, ac_q, lambda, sT, dcs, has_qm ? sQm : nullptr, qm_full != 0, band_tilt, s);
#pragma unroll 8
  for (int i = 0; i < 64; i++) levels[(size_t)b * 64 + i] = cf[i];
}

// The TX_4X4 split trials, one thread per job, the 4x4 blocks in raster
// order: B = 16 is split16_depth2_try (sixteen 4x4, DCT_DCT, ADST_ADST, IDTX,
// V_DCT, H_DCT), B = 8 is the 8x8 leaf's split4tx_try
// (src/coder/block8.rs:157-286: four 4x4, DCT_DCT, ADST_ADST, IDTX, with the
// quadrant edge flags (py > 0, px > 0), (have_tr, 0), (1, have_bl), (0, 0)).
// Per 4x4: prediction through the B x B patch reader, DCT_DCT (+ QM,
// trellis), then the other types through one loop body (ADST_ADST trellised),
// each kept when its SSE is within tx_guard of the DCT's and its rd cost is
// lower.  The rates use txb_skip context 0 and the dc_sign context of the job's
// own bytes for the 4x4's column and row.
struct Depth2Work {
  int32_t u[128];  // prediction edges, then targets [0, 16) and the transform temporary [64, 128)
  int16_t pred[16], resid[16];
  int16_t cfs[2][16], rrs[2][16];
  float suf[20];
  uint8_t lv[160];
  uint8_t patch[256];
};

// tx_types of the B = 16 and B = 8 results.
__device__ __forceinline__ uint8_t* result_types(mt_split16_d2_result& r) { return r.tx_types; }
__device__ __forceinline__ uint8_t* result_types(mt_split16_result& r) { return r.tx_types; }
__device__ __forceinline__ void clear_reserved(mt_split16_d2_result& r) { *reinterpret_cast<uint32_t*>(r.reserved) = 0; }
__device__ __forceinline__ void clear_reserved(mt_split16_result&) {}

template <int B, typename R>
__global__ void __launch_bounds__(kSplitThreads) tx4_split_kernel(
    const uint16_t* __restrict__ src, const uint16_t* __restrict__ rec, SplitArgs a,
    const uint8_t* __restrict__ qm_row, const mt_coef_costs* __restrict__ costs,
    const mt_split16_job* __restrict__ jobs, int n, R* __restrict__ res,
    int32_t* __restrict__ cf_out, uint16_t* __restrict__ rec_out) {
  constexpr int G = B / 4, NB = G * G;  // 4x4 blocks per row / per job
  __shared__ mt_coef_costs sT;
  __shared__ uint8_t sQm[16];
  __shared__ float sQs[16];
  __shared__ float sLut[64];
  {
    const float* g = reinterpret_cast<const float*>(costs);
    float* s = reinterpret_cast<float*>(&sT);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
    if (threadIdx.x < 16) {
      const int w = a.has_qm ? qm_row[threadIdx.x] : 32;
      sQm[threadIdx.x] = (uint8_t)w;
      sQs[threadIdx.x] = fwd_qm_scale(w);
    }
    if (threadIdx.x < 64) sLut[threadIdx.x] = kCoefRateLut[threadIdx.x];
    __syncthreads();
  }
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const mt_split16_params& p = a.p;
  const mt_quant& q = a.q;
  const mt_coef_costs& T = sT;
  const uint8_t* qm = a.has_qm ? sQm : nullptr;
  const mt_split16_job jb = jobs[j];
  R& r = res[j];
  if (!job_ok<B>(jb, p.frame_w, p.frame_h)) {
    r.sse = 0;
    r.bits = 0.0f;
    for (int i = 0; i < NB; i++) result_types(r)[i] = 0xff;
    clear_reserved(r);
    if (cf_out)
      for (int i = 0; i < B * B; i++) cf_out[(size_t)j * B * B + i] = 0;
    if (rec_out)
      for (int i = 0; i < B * B; i++) rec_out[(size_t)j * B * B + i] = 0;
    return;
  }
  Depth2Work w;
  const bool have_tr = jb.flags & MT_CAND_HAVE_TR, have_bl = jb.flags & MT_CAND_HAVE_BL;
  const bool ft = jb.flags & MT_CAND_FILTER_TYPE;
  const int32_t maxv = (1 << p.bd) - 1;
  const float dcq = (float)q.dc_q, acq = (float)q.ac_q, rd_lam = p.rd_lambda;
  const int vis_w = p.vis_w > 0 ? p.vis_w : p.frame_w, vis_h = p.vis_h > 0 ? p.vis_h : p.frame_h;
  const float skip1 = p.use_skip_bits ? p.skip_bits[0][0] : 0.0f;
  const float skip0 = p.use_skip_bits ? p.skip_bits[0][1] : 0.0f;
  const PatchReadS<B> rd{rec, p.stride, jb.px, jb.py, w.patch};
  long long sse_sum = 0;
  float bits_sum = 0.0f;
  uint8_t txtps[NB];
  for (int ti = 0; ti < NB; ti++) {
    const int i = ti % G, jr = ti / G, bx = jb.px + i * 4, by = jb.py + jr * 4;
    bool tr, bl;
    if (B == 16) {
      tr = jr == 0 ? (jb.py > 0 && (i < 3 || have_tr)) : i < 3;
      bl = i == 0 ? (jb.px > 0 && (jr < 3 || have_bl)) : false;
    } else {
      tr = ti == 0 ? jb.py > 0 : (ti == 1 ? have_tr : ti == 2);
      bl = ti == 0 ? jb.px > 0 : (ti == 2 ? have_bl : false);
    }
    predict_sq_at<4>(rd, p.frame_w, p.frame_h, bx, by, jb.mode, jb.angle_delta, tr, bl, ft, p.bd, w.pred, w.u);
#pragma unroll
    for (int k = 0; k < 16; k++)
      w.resid[k] = (int16_t)((int32_t)src[(size_t)(by + (k >> 2)) * p.stride + bx + (k & 3)] - w.pred[k]);
    const int sgn = (int)(jb.a_coef[i] >> 6) + (int)(jb.l_coef[jr] >> 6) - 2;
    const int ds = (sgn != 0) + (sgn > 0);
    ErrBlock<int16_t, int16_t> eb;
    eb.src = src + (size_t)by * p.stride + bx;
    eb.stride = p.stride;
    eb.pred = w.pred;
    eb.w = 4;
    eb.vw = min(max(vis_w - bx, 0), 4);
    eb.vh = min(max(vis_h - by, 0), 4);
    eb.maxv = maxv;
    float* tf = reinterpret_cast<float*>(w.u);
    int32_t* tmp = w.u + 64;
    // DCT_DCT, ADST_ADST, IDTX[, V_DCT, H_DCT] (nibble k: the k-th type).
    constexpr uint32_t kTypeOrder = 0x32041u;
    constexpr int kNumTypes = B == 16 ? 5 : 3;
    int best = 0, btx = MT_TX_DCT_DCT;
    long long bsse = 0, dct_sse = 0, guard = 0;
    float bbits = 0.0f;
#pragma unroll 1
    for (int k = 0; k < kNumTypes; k++) {
      const int t = (int)((kTypeOrder >> (4 * k)) & 15u);
      const int cur = k == 0 ? 0 : 1 - best;
      int16_t* cf = w.cfs[cur];
      int16_t* rr = w.rrs[cur];
      fwd4x4(w.resid, t, q, cf, tf, tmp);
      if (t == MT_TX_DCT_DCT || t == MT_TX_ADST_ADST) {
        if (qm) apply_qm(cf, tf, sQs, 16);
        if (a.lambda > 0.0f) trellis4(cf, tf, w.suf, dcq, acq, a.lambda, sLut);
      }
      inv4x4(cf, t, q, qm, rr, tmp);
      eb.resid = rr;
      const long long asse = sse_recon_block(eb, p.wsse_scale);
      if (k > 0 && !(asse <= dct_sse + guard)) continue;
      const float best_rd = k == 0 ? 0.0f : rd_cost_i64(bsse, rd_lam, bbits);
      float abits;
      if (t == MT_TX_V_DCT || t == MT_TX_H_DCT) {
        abits = rate_1d<4>(cf, t == MT_TX_V_DCT, T, ds, jb.mode, w.lv);
      } else {
        const float bound =
            k == 0 ? __int_as_float(0x7f800000) : __fdiv_rn(__fsub_rn(best_rd, (float)asse), rd_lam);
        abits = rate_bounded<4>(cf, T, 0, ds, jb.mode, t, p.use_skip_bits != 0, skip1, skip0, bound, w.lv);
      }
      if (k == 0 || rd_cost_i64(asse, rd_lam, abits) < best_rd) {
        best = cur;
        bsse = asse;
        bbits = abits;
        btx = t;
      }
      if (k == 0) {
        dct_sse = asse;
        guard = p.tx_guard_shift >= 63 ? 0 : (asse >> p.tx_guard_shift);
      }
    }
    const int16_t* bcf = w.cfs[best];
    const int16_t* brr = w.rrs[best];
    txtps[ti] = (uint8_t)btx;
    sse_sum += bsse;
    bits_sum = __fadd_rn(bits_sum, bbits);
#pragma unroll
    for (int k = 0; k < 16; k++)
      w.patch[(jr * 4 + (k >> 2)) * B + i * 4 + (k & 3)] = (uint8_t)clampi((int32_t)w.pred[k] + brr[k], 0, maxv);
    if (cf_out) {
      int4* o = reinterpret_cast<int4*>(cf_out + (size_t)j * B * B + ti * 16);
#pragma unroll
      for (int k = 0; k < 4; k++) o[k] = make_int4(bcf[4 * k], bcf[4 * k + 1], bcf[4 * k + 2], bcf[4 * k + 3]);
    }
  }
  r.sse = sse_sum;
  r.bits = bits_sum;
#pragma unroll
  for (int k = 0; k < NB; k++) result_types(r)[k] = txtps[k];
  clear_reserved(r);
  if (rec_out) {
    uint2* o = reinterpret_cast<uint2*>(rec_out + (size_t)j * B * B);
#pragma unroll 4
    for (int k = 0; k < B * B / 4; k++)
      o[k] = make_uint2(w.patch[4 * k] | ((uint32_t)w.patch[4 * k + 1] << 16),
                        w.patch[4 * k + 2] | ((uint32_t)w.patch[4 * k + 3] << 16));
  }
}

int check_split(const mt_split16_params* p, const mt_quant* q, int32_t n) {
  if (!p || !q || n < 0) return MT_ERR_INVALID_INPUT;
  if (p->bd != 8) return MT_ERR_UNSUPPORTED;
  if (p->frame_w < 16 || p->frame_h < 16 || p->stride < p->frame_w || p->vis_w < 0 || p->vis_h < 0)
    return MT_ERR_INVALID_INPUT;
  if (!(p->rd_lambda > 0.0f) || !(p->wsse_scale >= 0.0f) || p->tx_guard_shift < 0) return MT_ERR_INVALID_INPUT;
  return MT_OK;
}

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

// Launch and host-buffer forms shared by the two TX_4X4 split trials.
template <int B, typename R>
int tx4_split_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                     const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                     const mt_split16_job* d_jobs, int32_t n, R* d_results, int32_t* d_cf, uint16_t* d_rec,
                     void* stream) {
  int rc = check_split(prm, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!d_src || !d_recon || !d_costs || !d_jobs || !d_results) return MT_ERR_INVALID_INPUT;
  SplitArgs a;
  a.p = *prm;
  a.q = *quant;
  a.lambda = prm->trellis_lambda0 > 0.0f ? mth::scaled_trellis_lambda_host((float)quant->dc_q, prm->trellis_lambda0)
                                         : 0.0f;
  a.has_qm = quant->qm_level < 15 && d_qm_row != nullptr;
  tx4_split_kernel<B, R><<<(unsigned)((n + kSplitThreads - 1) / kSplitThreads), kSplitThreads, 0,
                           reinterpret_cast<cudaStream_t>(stream)>>>(d_src, d_recon, a, d_qm_row, d_costs, d_jobs, n,
                                                                     d_results, d_cf, d_rec);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

template <int B, typename R>
int tx4_split_host(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
                   const uint8_t* qm_row, const mt_coef_costs* costs, const mt_split16_job* jobs, int32_t n,
                   R* results, int32_t* cf_out, uint16_t* rec_out) {
  int rc = check_split(prm, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!src || !recon || !costs || !jobs || !results) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)prm->stride * prm->frame_h * sizeof(uint16_t), bb = (size_t)B * B;
  const size_t o_src = 0, o_rec = up256(plane), o_qm = o_rec + up256(plane), o_cost = o_qm + 256;
  const size_t o_jobs = o_cost + up256(sizeof(mt_coef_costs));
  const size_t o_res = o_jobs + up256((size_t)n * sizeof(mt_split16_job));
  const size_t o_cf = o_res + up256((size_t)n * sizeof(R));
  const size_t o_out = o_cf + (cf_out ? up256((size_t)n * bb * 4) : 0);
  const size_t total = o_out + (rec_out ? up256((size_t)n * bb * 2) : 0);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, total) != cudaSuccess) return MT_ERR_ALLOC;
  const bool has_qm = quant->qm_level < 15 && qm_row != nullptr;
  cudaError_t e = cudaMemcpy(d + o_src, src, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_rec, recon, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && has_qm) e = cudaMemcpy(d + o_qm, qm_row, 16, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_cost, costs, sizeof(mt_coef_costs), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_jobs, jobs, (size_t)n * sizeof(mt_split16_job), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = tx4_split_device<B>(reinterpret_cast<const uint16_t*>(d + o_src),
                             reinterpret_cast<const uint16_t*>(d + o_rec), prm, quant, has_qm ? d + o_qm : nullptr,
                             reinterpret_cast<const mt_coef_costs*>(d + o_cost),
                             reinterpret_cast<const mt_split16_job*>(d + o_jobs), n, reinterpret_cast<R*>(d + o_res),
                             cf_out ? reinterpret_cast<int32_t*>(d + o_cf) : nullptr,
                             rec_out ? reinterpret_cast<uint16_t*>(d + o_out) : nullptr, nullptr);
    if (rc == MT_OK) e = cudaMemcpy(results, d + o_res, (size_t)n * sizeof(R), cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && cf_out) e = cudaMemcpy(cf_out, d + o_cf, (size_t)n * bb * 4, cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && rec_out)
      e = cudaMemcpy(rec_out, d + o_out, (size_t)n * bb * 2, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // namespace

extern "C" {

int mt_trellis_optimize_ctx_device(int32_t* d_levels, const float* d_targets, const uint8_t* d_dcs_ctx, int32_t n,
                                   const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                                   float lambda0, float band_tilt, void* stream) {
  if (!quant || n < 0) return MT_ERR_INVALID_INPUT;
  if (n == 0 || lambda0 <= 0.0f) return MT_OK;
  if (!d_levels || !d_targets || !d_dcs_ctx || !d_costs) return MT_ERR_INVALID_INPUT;
  const int has_qm = quant->qm_level < 15 && d_qm_row != nullptr;
  const float lambda = mth::scaled_trellis_lambda_host((float)quant->dc_q, lambda0);
  trellis_ctx_kernel<<<(n + kSplitThreads - 1) / kSplitThreads, kSplitThreads, 0,
                       reinterpret_cast<cudaStream_t>(stream)>>>(d_levels, d_targets, d_dcs_ctx, n, (float)quant->dc_q,
                                                                 (float)quant->ac_q, lambda, d_qm_row, has_qm,
                                                                 quant->qm_level >= 5, d_costs, band_tilt);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_split16_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                           const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                           const mt_split16_job* d_jobs, int32_t n, mt_split16_result* d_results, int32_t* d_cf,
                           uint16_t* d_rec, void* stream) {
  int rc = check_split(prm, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!d_src || !d_recon || !d_costs || !d_jobs || !d_results) return MT_ERR_INVALID_INPUT;
  SplitArgs a;
  a.p = *prm;
  a.q = *quant;
  a.lambda = prm->trellis_lambda0 > 0.0f ? mth::scaled_trellis_lambda_host((float)quant->dc_q, prm->trellis_lambda0)
                                         : 0.0f;
  a.has_qm = quant->qm_level < 15 && d_qm_row != nullptr;
  const unsigned grid = (unsigned)((n + kSplitThreads - 1) / kSplitThreads);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (prm->tx_search)
    split16_kernel<true><<<grid, kSplitThreads, 0, st>>>(d_src, d_recon, a, d_qm_row, d_costs, d_jobs, n, d_results,
                                                         d_cf, d_rec);
  else
    split16_kernel<false><<<grid, kSplitThreads, 0, st>>>(d_src, d_recon, a, d_qm_row, d_costs, d_jobs, n, d_results,
                                                          d_cf, d_rec);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_split16_luma(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
                    const uint8_t* qm_row, const mt_coef_costs* costs, const mt_split16_job* jobs, int32_t n,
                    mt_split16_result* results, int32_t* cf_out, uint16_t* rec_out) {
  int rc = check_split(prm, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!src || !recon || !costs || !jobs || !results) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)prm->stride * prm->frame_h * sizeof(uint16_t);
  const size_t o_src = 0, o_rec = up256(plane), o_qm = o_rec + up256(plane), o_cost = o_qm + 256;
  const size_t o_jobs = o_cost + up256(sizeof(mt_coef_costs));
  const size_t o_res = o_jobs + up256((size_t)n * sizeof(mt_split16_job));
  const size_t o_cf = o_res + up256((size_t)n * sizeof(mt_split16_result));
  const size_t o_out = o_cf + (cf_out ? up256((size_t)n * 256 * 4) : 0);
  const size_t total = o_out + (rec_out ? up256((size_t)n * 256 * 2) : 0);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, total) != cudaSuccess) return MT_ERR_ALLOC;
  const bool has_qm = quant->qm_level < 15 && qm_row != nullptr;
  cudaError_t e = cudaMemcpy(d + o_src, src, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_rec, recon, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && has_qm) e = cudaMemcpy(d + o_qm, qm_row, 64, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_cost, costs, sizeof(mt_coef_costs), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_jobs, jobs, (size_t)n * sizeof(mt_split16_job), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = mt_split16_luma_device(
        reinterpret_cast<const uint16_t*>(d + o_src), reinterpret_cast<const uint16_t*>(d + o_rec), prm, quant,
        has_qm ? d + o_qm : nullptr, reinterpret_cast<const mt_coef_costs*>(d + o_cost),
        reinterpret_cast<const mt_split16_job*>(d + o_jobs), n, reinterpret_cast<mt_split16_result*>(d + o_res),
        cf_out ? reinterpret_cast<int32_t*>(d + o_cf) : nullptr, rec_out ? reinterpret_cast<uint16_t*>(d + o_out) : nullptr,
        nullptr);
    if (rc == MT_OK) e = cudaMemcpy(results, d + o_res, (size_t)n * sizeof(mt_split16_result), cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && cf_out) e = cudaMemcpy(cf_out, d + o_cf, (size_t)n * 256 * 4, cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && rec_out)
      e = cudaMemcpy(rec_out, d + o_out, (size_t)n * 256 * 2, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"

extern "C" {

int mt_split16_depth2_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                             const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                             const mt_split16_job* d_jobs, int32_t n, mt_split16_d2_result* d_results,
                             int32_t* d_cf, uint16_t* d_rec, void* stream) {
  return tx4_split_device<16>(d_src, d_recon, prm, quant, d_qm_row, d_costs, d_jobs, n, d_results, d_cf, d_rec,
                              stream);
}

int mt_split16_depth2(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
                      const uint8_t* qm_row, const mt_coef_costs* costs, const mt_split16_job* jobs, int32_t n,
                      mt_split16_d2_result* results, int32_t* cf_out, uint16_t* rec_out) {
  return tx4_split_host<16>(src, recon, prm, quant, qm_row, costs, jobs, n, results, cf_out, rec_out);
}

int mt_split4tx_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                       const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                       const mt_split16_job* d_jobs, int32_t n, mt_split16_result* d_results, int32_t* d_cf,
                       uint16_t* d_rec, void* stream) {
  return tx4_split_device<8>(d_src, d_recon, prm, quant, d_qm_row, d_costs, d_jobs, n, d_results, d_cf, d_rec,
                             stream);
}

int mt_split4tx(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
                const uint8_t* qm_row, const mt_coef_costs* costs, const mt_split16_job* jobs, int32_t n,
                mt_split16_result* results, int32_t* cf_out, uint16_t* rec_out) {
  return tx4_split_host<8>(src, recon, prm, quant, qm_row, costs, jobs, n, results, cf_out, rec_out);
}

}  // extern "C"
