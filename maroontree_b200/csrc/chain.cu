// Batched luma candidate chain for 8x8 blocks (the per-candidate body of the
// reference's luma mode search, src/coder/partition_search.rs:467-530):
//   predict -> residual -> forward transform + quantisation (+QM)
//   -> trellis_optimize -> dequantisation + inverse transform
//   -> SATD distortion (luma_partition_distortion) and coefficient rate
//   -> rd_cost = D + lambda * (bits + mode bits).
// One thread evaluates one candidate; the batch-wide tables (bit costs, scan,
// QM row) are staged once per CTA in shared memory.
#include <cuda_runtime.h>
#include <stdint.h>

#include "chain8.cuh"

namespace mtd {

struct ChainArgs {
  mt_chain_params p;
  mt_quant q;
  float trellis_lambda;  // scaled_trellis_lambda(dc_q, ac_q, lambda0), computed on the host
  int has_qm;
};

__global__ void __launch_bounds__(128) chain8_kernel(const uint16_t* __restrict__ src,
                                                     const uint16_t* __restrict__ rec, ChainArgs a,
                                                     const uint8_t* __restrict__ qm_row,
                                                     const mt_coef_costs* __restrict__ costs,
                                                     const mt_candidate* __restrict__ cands, int n,
                                                     mt_candidate_result* __restrict__ res,
                                                     int32_t* __restrict__ lv_out, int32_t* __restrict__ rec_out) {
  __shared__ mt_coef_costs sC;
  __shared__ uint8_t sQm[64];
  {
    const float* g = reinterpret_cast<const float*>(costs);
    float* s = reinterpret_cast<float*>(&sC);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
    if (threadIdx.x < 64) sQm[threadIdx.x] = a.has_qm ? qm_row[threadIdx.x] : 32;
  }
  __syncthreads();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const mt_candidate cd = cands[idx];
  const int32_t maxv = (1 << a.p.bd) - 1;
  if (!cand_ok(cd, a.p.frame_w, a.p.frame_h)) {
    mt_candidate_result bad = {};
    bad.eob = MT_EOB_INVALID;
    res[idx] = bad;
    return;
  }
  Work8 w;
  mt_candidate_result r;
  chain8_one(src, rec, a.p, a.q, a.trellis_lambda, a.has_qm ? sQm : nullptr, sC, cd, r, w);
  const int32_t* pred = w.pred();
  const int32_t* cf = w.cf();
  const int32_t* rr = w.rr();
  res[idx] = r;
  if (lv_out) {
    int4* o = reinterpret_cast<int4*>(lv_out + (size_t)idx * 64);
    for (int i = 0; i < 16; i++) o[i] = make_int4(cf[4 * i], cf[4 * i + 1], cf[4 * i + 2], cf[4 * i + 3]);
  }
  if (rec_out) {
    int4* o = reinterpret_cast<int4*>(rec_out + (size_t)idx * 64);
    for (int i = 0; i < 16; i++)
      o[i] = make_int4(clampi(pred[4 * i] + rr[4 * i], 0, maxv), clampi(pred[4 * i + 1] + rr[4 * i + 1], 0, maxv),
                       clampi(pred[4 * i + 2] + rr[4 * i + 2], 0, maxv),
                       clampi(pred[4 * i + 3] + rr[4 * i + 3], 0, maxv));
  }
}


// Standalone kernels of the chain's stages, one block per thread.
__global__ void fwd8_kernel(const int32_t* __restrict__ resid, const uint8_t* __restrict__ types, int n, mt_quant q,
                            const uint8_t* __restrict__ qm_row, int32_t* __restrict__ levels,
                            float* __restrict__ targets) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  Work8 w;
  int32_t* r = w.rr();
  int32_t* cf = w.cf();
  float* tf = w.tf();
  for (int i = 0; i < 64; i++) r[i] = resid[(size_t)idx * 64 + i];
  const int tx = types[idx];
  fwd8x8(r, tx, q, cf, tf);
  if (qm_row && (tx == MT_TX_DCT_DCT || tx >= MT_TX_ADST_ADST)) apply_qm(cf, tf, qm_row, 64);
  for (int i = 0; i < 64; i++) {
    levels[(size_t)idx * 64 + i] = cf[i];
    targets[(size_t)idx * 64 + i] = tf[i];
  }
}
__global__ void inv8_kernel(const int32_t* __restrict__ levels, const uint8_t* __restrict__ types, int n, mt_quant q,
                            const uint8_t* __restrict__ qm_row, int32_t* __restrict__ out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  Work8 w;
  int32_t* cf = w.cf();
  int32_t* o = w.rr();
  for (int i = 0; i < 64; i++) cf[i] = levels[(size_t)idx * 64 + i];
  inv8x8(cf, types[idx], q, qm_row, o);
  for (int i = 0; i < 64; i++) out[(size_t)idx * 64 + i] = o[i];
}
__global__ void trellis8_kernel(int32_t* __restrict__ levels, const float* __restrict__ targets, int n, float dc_q,
                                float ac_q, float lambda) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  Work8 w;
  int32_t* cf = w.cf();
  float* tf = w.tf();
  for (int i = 0; i < 64; i++) {
    cf[i] = levels[(size_t)idx * 64 + i];
    tf[i] = targets[(size_t)idx * 64 + i];
  }
  trellis8(cf, tf, dc_q, ac_q, lambda);
  for (int i = 0; i < 64; i++) levels[(size_t)idx * 64 + i] = cf[i];
}
__global__ void pred8_kernel(const uint16_t* __restrict__ rec, mt_chain_params p, const mt_candidate* __restrict__ cands,
                             int n, int32_t* __restrict__ out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const mt_candidate cd = cands[idx];
  Work8 w;
  int32_t* pr = w.pred();
  if (!cand_ok(cd, p.frame_w, p.frame_h)) {
    for (int i = 0; i < 64; i++) out[(size_t)idx * 64 + i] = 0;
    return;
  }
  predict8(rec, p.stride, p.frame_w, p.frame_h, cd.px, cd.py, cd.mode, cd.angle_delta, cd.flags & 1,
           (cd.flags >> 1) & 1, (cd.flags >> 2) & 1, p.bd, pr);
  for (int i = 0; i < 64; i++) out[(size_t)idx * 64 + i] = pr[i];
}

}  // namespace mtd

// Host launchers used by the C ABI (capi.cu).
namespace mth {
cudaError_t launch_chain8(const uint16_t* src, const uint16_t* rec, const mt_chain_params& p, const mt_quant& q,
                          float trellis_lambda, const uint8_t* qm_row, const mt_coef_costs* costs,
                          const mt_candidate* cands, int n, mt_candidate_result* res, int32_t* lv, int32_t* ro,
                          cudaStream_t st) {
  mtd::ChainArgs a;
  a.p = p;
  a.q = q;
  a.trellis_lambda = trellis_lambda;
  a.has_qm = qm_row != nullptr;
  const int threads = 128;
  const int blocks = (n + threads - 1) / threads;
  if (blocks > 0) mtd::chain8_kernel<<<blocks, threads, 0, st>>>(src, rec, a, qm_row, costs, cands, n, res, lv, ro);
  return cudaGetLastError();
}
cudaError_t launch_fwd8(const int32_t* resid, const uint8_t* types, int n, const mt_quant& q, const uint8_t* qm,
                        int32_t* levels, float* targets, cudaStream_t st) {
  const int blocks = (n + 127) / 128;
  if (blocks > 0) mtd::fwd8_kernel<<<blocks, 128, 0, st>>>(resid, types, n, q, qm, levels, targets);
  return cudaGetLastError();
}
cudaError_t launch_inv8(const int32_t* levels, const uint8_t* types, int n, const mt_quant& q, const uint8_t* qm,
                        int32_t* out, cudaStream_t st) {
  const int blocks = (n + 127) / 128;
  if (blocks > 0) mtd::inv8_kernel<<<blocks, 128, 0, st>>>(levels, types, n, q, qm, out);
  return cudaGetLastError();
}
cudaError_t launch_trellis8(int32_t* levels, const float* targets, int n, float dc_q, float ac_q, float lambda,
                            cudaStream_t st) {
  const int blocks = (n + 127) / 128;
  if (blocks > 0) mtd::trellis8_kernel<<<blocks, 128, 0, st>>>(levels, targets, n, dc_q, ac_q, lambda);
  return cudaGetLastError();
}
cudaError_t launch_pred8(const uint16_t* rec, const mt_chain_params& p, const mt_candidate* cands, int n, int32_t* out,
                         cudaStream_t st) {
  const int blocks = (n + 127) / 128;
  if (blocks > 0) mtd::pred8_kernel<<<blocks, 128, 0, st>>>(rec, p, cands, n, out);
  return cudaGetLastError();
}
}  // namespace mth
