// The 8x8 leaf's luma search (pick_block8, src/coder/block8.rs:689-1420),
// batched: the Slow mode loop's candidates (leaf8_kernel<false>) and the
// winner's transform-type refinement (leaf8_kernel<true>), one thread per job.
// The stages are the split trial's (leaf8.cuh): DCT_DCT + QM with
// trellis_optimize_ctx, the dav1d inverse, sse_recon, the bounded 2-D and the
// 1-D rate walks; every type runs through one loop body with the candidate and
// the current winner in the two slots of cfs / rrs.
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

constexpr int kLeafThreads = 128;

struct LeafArgs {
  mt_split16_params p;
  mt_quant q;
  float lambda;  // scaled_trellis_lambda (0: no trellis)
  int has_qm;
};

struct LeafWork {
  int32_t u[128];  // prediction edges, then targets [0, 64) and the transform temporary [64, 128)
  int16_t pred[64], resid[64];
  int16_t cfs[2][64], rrs[2][64];
  TrellisCtxScratch tr;
  uint8_t lv[160];
};

__device__ __forceinline__ float rd_cost_i64(long long d, float lam, float rate) {
  return __fadd_rn((float)d, __fmul_rn(lam, rate));
}

template <bool REFINE>
__global__ void __launch_bounds__(kLeafThreads) leaf8_kernel(
    const uint16_t* __restrict__ src, const uint16_t* __restrict__ rec, LeafArgs a,
    const uint8_t* __restrict__ qm_row, const mt_coef_costs* __restrict__ costs,
    const mt_leaf8_job* __restrict__ jobs, int n, mt_leaf8_result* __restrict__ res, int32_t* __restrict__ cf_out,
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
  const mt_leaf8_job jb = jobs[j];
  mt_leaf8_result& r = res[j];
  const bool ok = jb.px + 8 <= p.frame_w && jb.py + 8 <= p.frame_h && jb.mode <= MT_PAETH_PRED &&
                  jb.angle_delta >= -3 && jb.angle_delta <= 3 &&
                  (jb.angle_delta == 0 || (jb.mode >= MT_V_PRED && jb.mode <= MT_D67_PRED)) && jb.dcs_ctx < 3;
  if (!ok) {
    r.sse = 0;
    r.bits = r.cost = __int_as_float(0x7f800000);
    r.tx_type = 255;
    for (int i = 0; i < 7; i++) r.reserved[i] = 0;
    if (cf_out)
      for (int i = 0; i < 64; i++) cf_out[(size_t)j * 64 + i] = 0;
    if (rec_out)
      for (int i = 0; i < 64; i++) rec_out[(size_t)j * 64 + i] = 0;
    return;
  }
  LeafWork w;
  const int32_t maxv = (1 << p.bd) - 1;
  const float dcq = (float)q.dc_q, acq = (float)q.ac_q, rd_lam = p.rd_lambda;
  const bool qm_full = q.qm_level >= 5;
  const int vis_w = p.vis_w > 0 ? p.vis_w : p.frame_w, vis_h = p.vis_h > 0 ? p.vis_h : p.frame_h;
  predict_sq<8>(rec, p.stride, p.frame_w, p.frame_h, jb.px, jb.py, jb.mode, jb.angle_delta, jb.flags & 1,
                (jb.flags >> 1) & 1, (jb.flags >> 2) & 1, p.bd, w.pred, w.u);
#pragma unroll 8
  for (int i = 0; i < 64; i++)
    w.resid[i] = (int16_t)((int32_t)src[(size_t)(jb.py + (i >> 3)) * p.stride + jb.px + (i & 7)] - w.pred[i]);
  const int ds = jb.dcs_ctx;
  ErrBlock<int16_t, int16_t> eb;
  eb.src = src + (size_t)jb.py * p.stride + jb.px;
  eb.stride = p.stride;
  eb.pred = w.pred;
  eb.w = 8;
  eb.vw = min(max(vis_w - jb.px, 0), 8);
  eb.vh = min(max(vis_h - jb.py, 0), 8);
  eb.maxv = maxv;
  const float skip1 = p.use_skip_bits ? p.skip_bits[0][0] : 0.0f;
  const float skip0 = p.use_skip_bits ? p.skip_bits[0][1] : 0.0f;
  float* tf = reinterpret_cast<float*>(w.u);
  int32_t* tmp = w.u + 64;
  // DCT_DCT, then (refinement) ADST_ADST, ADST_DCT, DCT_ADST, IDTX[, V_DCT,
  // H_DCT]; nibble k: the k-th type.
  constexpr uint32_t kTypeOrder = 0x3206541u;
  const int ntypes = REFINE ? (p.tx_search ? 7 : 5) : 1;
  int best = 0, btx = MT_TX_DCT_DCT;
  long long bsse = 0, dct_sse = 0, dct_guard = 0;
  float bbits = 0.0f;
#pragma unroll 1
  for (int k = 0; k < ntypes; k++) {
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
    if (k > 0) {
      // the gates of block8.rs:1214-1396: the ADST family within tx_guard of
      // the DCT's SSE, IDTX within tx_guard of the current best's, V / H at
      // most the current best's
      bool gate;
      if (t >= MT_TX_ADST_ADST) gate = asse <= dct_sse + dct_guard;
      else if (t == MT_TX_IDTX) gate = asse <= bsse + (p.tx_guard_shift >= 63 ? 0 : (bsse >> p.tx_guard_shift));
      else gate = asse <= bsse;
      if (!gate) continue;
    }
    const float base_rd = k == 0 ? 0.0f : rd_cost_i64(bsse, rd_lam, bbits);
    float abits;
    if (t == MT_TX_V_DCT || t == MT_TX_H_DCT) {
      abits = rate_1d<8>(cf, t == MT_TX_V_DCT, T, ds, jb.mode, w.lv);
    } else {
      const float bound = (k == 0 || t == MT_TX_IDTX) ? __int_as_float(0x7f800000)
                                                      : __fdiv_rn(__fsub_rn(base_rd, (float)asse), rd_lam);
      abits = rate_bounded<8>(cf, T, 0, ds, jb.mode, t, p.use_skip_bits != 0, skip1, skip0, bound, w.lv);
    }
    if (k == 0 || rd_cost_i64(asse, rd_lam, abits) < base_rd) {
      best = cur;
      bsse = asse;
      bbits = abits;
      btx = t;
    }
    if (k == 0) {
      dct_sse = asse;
      dct_guard = p.tx_guard_shift >= 63 ? 0 : (asse >> p.tx_guard_shift);
    }
  }
  r.sse = bsse;
  r.bits = bbits;
  r.cost = REFINE ? rd_cost_i64(bsse, rd_lam, bbits) : rd_cost_i64(bsse, rd_lam, __fadd_rn(bbits, jb.syntax_bits));
  r.tx_type = (uint8_t)btx;
  for (int i = 0; i < 7; i++) r.reserved[i] = 0;
  const int16_t* bcf = w.cfs[best];
  const int16_t* brr = w.rrs[best];
  if (cf_out) {
    int4* o = reinterpret_cast<int4*>(cf_out + (size_t)j * 64);
#pragma unroll
    for (int i = 0; i < 16; i++) o[i] = make_int4(bcf[4 * i], bcf[4 * i + 1], bcf[4 * i + 2], bcf[4 * i + 3]);
  }
  if (rec_out) {
    uint16_t* o = rec_out + (size_t)j * 64;
#pragma unroll 8
    for (int i = 0; i < 64; i++) o[i] = (uint16_t)clampi((int32_t)w.pred[i] + brr[i], 0, maxv);
  }
}

int check(const mt_split16_params* p, const mt_quant* q, int32_t n) {
  if (!p || !q || n < 0) return MT_ERR_INVALID_INPUT;
  if (p->bd != 8) return MT_ERR_UNSUPPORTED;
  if (p->frame_w < 8 || p->frame_h < 8 || p->stride < p->frame_w || p->vis_w < 0 || p->vis_h < 0)
    return MT_ERR_INVALID_INPUT;
  if (!(p->rd_lambda > 0.0f) || !(p->wsse_scale >= 0.0f) || p->tx_guard_shift < 0) return MT_ERR_INVALID_INPUT;
  return MT_OK;
}

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

template <bool REFINE>
int leaf8_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm, const mt_quant* quant,
                 const uint8_t* d_qm_row, const mt_coef_costs* d_costs, const mt_leaf8_job* d_jobs, int32_t n,
                 mt_leaf8_result* d_results, int32_t* d_cf, uint16_t* d_rec, void* stream) {
  const int rc = check(prm, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!d_src || !d_recon || !d_costs || !d_jobs || !d_results) return MT_ERR_INVALID_INPUT;
  LeafArgs a;
  a.p = *prm;
  a.q = *quant;
  a.lambda = prm->trellis_lambda0 > 0.0f ? mth::scaled_trellis_lambda_host((float)quant->dc_q, prm->trellis_lambda0)
                                         : 0.0f;
  a.has_qm = quant->qm_level < 15 && d_qm_row != nullptr;
  leaf8_kernel<REFINE><<<(unsigned)((n + kLeafThreads - 1) / kLeafThreads), kLeafThreads, 0,
                         reinterpret_cast<cudaStream_t>(stream)>>>(d_src, d_recon, a, d_qm_row, d_costs, d_jobs, n,
                                                                   d_results, d_cf, d_rec);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // namespace

extern "C" {

int mt_leaf8_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                         const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                         const mt_leaf8_job* d_jobs, int32_t n, mt_leaf8_result* d_results, int32_t* d_cf,
                         uint16_t* d_rec, void* stream) {
  return leaf8_device<false>(d_src, d_recon, prm, quant, d_qm_row, d_costs, d_jobs, n, d_results, d_cf, d_rec, stream);
}

int mt_leaf8_tx_refine_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                              const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                              const mt_leaf8_job* d_jobs, int32_t n, mt_leaf8_result* d_results, int32_t* d_cf,
                              uint16_t* d_rec, void* stream) {
  return leaf8_device<true>(d_src, d_recon, prm, quant, d_qm_row, d_costs, d_jobs, n, d_results, d_cf, d_rec, stream);
}

int mt_leaf8(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
             const uint8_t* qm_row, const mt_coef_costs* costs, const mt_leaf8_job* jobs, int32_t n, int32_t refine,
             mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out) {
  int rc = check(prm, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!src || !recon || !costs || !jobs || !results) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)prm->stride * prm->frame_h * sizeof(uint16_t);
  const size_t o_src = 0, o_rec = up256(plane), o_qm = o_rec + up256(plane), o_cost = o_qm + 256;
  const size_t o_jobs = o_cost + up256(sizeof(mt_coef_costs));
  const size_t o_res = o_jobs + up256((size_t)n * sizeof(mt_leaf8_job));
  const size_t o_cf = o_res + up256((size_t)n * sizeof(mt_leaf8_result));
  const size_t o_out = o_cf + (cf_out ? up256((size_t)n * 64 * 4) : 0);
  const size_t total = o_out + (rec_out ? up256((size_t)n * 64 * 2) : 0);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, total) != cudaSuccess) return MT_ERR_ALLOC;
  const bool has_qm = quant->qm_level < 15 && qm_row != nullptr;
  cudaError_t e = cudaMemcpy(d + o_src, src, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_rec, recon, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && has_qm) e = cudaMemcpy(d + o_qm, qm_row, 64, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_cost, costs, sizeof(mt_coef_costs), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_jobs, jobs, (size_t)n * sizeof(mt_leaf8_job), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    auto fn = refine ? leaf8_device<true> : leaf8_device<false>;
    rc = fn(reinterpret_cast<const uint16_t*>(d + o_src), reinterpret_cast<const uint16_t*>(d + o_rec), prm, quant,
            has_qm ? d + o_qm : nullptr, reinterpret_cast<const mt_coef_costs*>(d + o_cost),
            reinterpret_cast<const mt_leaf8_job*>(d + o_jobs), n, reinterpret_cast<mt_leaf8_result*>(d + o_res),
            cf_out ? reinterpret_cast<int32_t*>(d + o_cf) : nullptr,
            rec_out ? reinterpret_cast<uint16_t*>(d + o_out) : nullptr, nullptr);
    if (rc == MT_OK) e = cudaMemcpy(results, d + o_res, (size_t)n * sizeof(mt_leaf8_result), cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && cf_out) e = cudaMemcpy(cf_out, d + o_cf, (size_t)n * 256, cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && rec_out) e = cudaMemcpy(rec_out, d + o_out, (size_t)n * 128, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"
