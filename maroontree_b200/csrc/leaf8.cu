// The leaf luma searches, batched, one thread per job: pick_block8's
// (src/coder/block8.rs:689-1420) Slow mode-loop candidates (leaf_kernel<8,
// false>) and winner transform-type refinement (leaf_kernel<8, true>), and
// pick_luma16's mode-loop candidates (leaf_kernel<16, false>).
// The stages are the split trial's (leaf8.cuh): DCT_DCT + QM with
// trellis_optimize_ctx, the dav1d inverse, sse_recon, the bounded 2-D and the
// 1-D rate walks; every type runs through one loop body with the candidate and
// the current winner in the two slots of cfs / rrs.
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "../../include/maroontree_b200.h"
#include "leaf8.cuh"
#include "txfm32.cuh"
#include "wsse.cuh"

namespace mth {
float scaled_trellis_lambda_host(float dc_q, float lambda0);
}

namespace {

using namespace mtd;

constexpr int kLeafThreads = 128;
// The 32x32 and 64x64 searches have few jobs per frame (1,980 32x32 blocks x 13
// modes, 480 64x64 blocks at 1080p) and long serial chains per job: one warp
// per CTA spreads them over every SM instead of a few.
constexpr int kBigThreads = 32;
template <int N>
constexpr int leaf_threads() {
  return N == 32 ? kBigThreads : kLeafThreads;
}

struct LeafArgs {
  mt_split16_params p;
  mt_quant q;
  float lambda;  // scaled_trellis_lambda (0: no trellis)
  int has_qm;
};

// Per-thread working set of one N x N job.  u: the prediction edges, then the
// targets [0, N*N) and the transform temporary [N*N, 2*N*N).  Levels are
// 32-bit at 32x32 (a full-scale DC at the smallest steps passes 16 bits);
// 32x32 has one transform type, so one slot.
template <int N>
struct LeafWork {
  using Coef = std::conditional_t<N == 32, int32_t, int16_t>;
  static constexpr int kSlots = N == 32 ? 1 : 2;
  int32_t u[2 * N * N];
  int16_t pred[N * N], resid[N * N];
  Coef cfs[kSlots][N * N];                // levels of the candidate and of the winner
  int16_t rrs[kSlots][N * N];             // their inverses
  TrellisCtxScratchW<N> tr;
  uint8_t lv[N == 8 ? 160 : (N + 2) * N];  // rate walks' level maps
};

__device__ __forceinline__ float rd_cost_i64(long long d, float lam, float rate) {
  return __fadd_rn((float)d, __fmul_rn(lam, rate));
}

// N = 8: pick_block8's candidates (REFINE = false) and winner refinement
// (REFINE = true); N = 16: pick_luma16's mode-loop candidates
// (src/coder/partition_search.rs:4802-4880) and winner refinement (:5252-5474:
// ADST_ADST, ADST_DCT, DCT_ADST, IDTX with the 8x8 leaf's gates); N = 32:
// pick_luma32's mode-loop candidates (src/coder/block32.rs:776-836: TX_32X32
// DCT_DCT, the only intra type of that size, trellis_optimize_ctx of class 3,
// no tx-type symbol in the rate).
template <int N, bool REFINE>
__global__ void __launch_bounds__(leaf_threads<N>()) leaf_kernel(
    const uint16_t* __restrict__ src, const uint16_t* __restrict__ rec, LeafArgs a,
    const uint8_t* __restrict__ qm_row, const mt_coef_costs* __restrict__ costs,
    const mt_leaf8_job* __restrict__ jobs, int n, mt_leaf8_result* __restrict__ res, int32_t* __restrict__ cf_out,
    uint16_t* __restrict__ rec_out) {
  __shared__ mt_coef_costs sT;
  static_assert(N == 8 || N == 16 || (N == 32 && !REFINE), "8x8 and 16x16 leaves, the 32x32 mode loop");
  constexpr int NN = N * N, L = log2w<N>();
  __shared__ uint8_t sQm[NN];
  __shared__ float sQs[NN];
  {
    const float* g = reinterpret_cast<const float*>(costs);
    float* s = reinterpret_cast<float*>(&sT);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
    for (int i = threadIdx.x; i < NN; i += blockDim.x) {
      const int w = a.has_qm ? qm_row[i] : 32;
      sQm[i] = (uint8_t)w;
      sQs[i] = fwd_qm_scale(w);
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
  const bool ok = jb.px + N <= p.frame_w && jb.py + N <= p.frame_h && jb.mode <= MT_PAETH_PRED &&
                  jb.angle_delta >= -3 && jb.angle_delta <= 3 &&
                  (jb.angle_delta == 0 || (jb.mode >= MT_V_PRED && jb.mode <= MT_D67_PRED)) && jb.dcs_ctx < 3;
  if (!ok) {
    r.sse = 0;
    r.bits = r.cost = __int_as_float(0x7f800000);
    r.tx_type = 255;
    for (int i = 0; i < 7; i++) r.reserved[i] = 0;
    if (cf_out)
      for (int i = 0; i < NN; i++) cf_out[(size_t)j * NN + i] = 0;
    if (rec_out)
      for (int i = 0; i < NN; i++) rec_out[(size_t)j * NN + i] = 0;
    return;
  }
  LeafWork<N> w;
  const int32_t maxv = (1 << p.bd) - 1;
  const float dcq = (float)q.dc_q, acq = (float)q.ac_q, rd_lam = p.rd_lambda;
  const bool qm_full = q.qm_level >= 5;
  const int vis_w = p.vis_w > 0 ? p.vis_w : p.frame_w, vis_h = p.vis_h > 0 ? p.vis_h : p.frame_h;
  predict_sq<N>(rec, p.stride, p.frame_w, p.frame_h, jb.px, jb.py, jb.mode, jb.angle_delta, jb.flags & 1,
                (jb.flags >> 1) & 1, (jb.flags >> 2) & 1, p.bd, w.pred, w.u);
#pragma unroll 8
  for (int i = 0; i < NN; i++)
    w.resid[i] = (int16_t)((int32_t)src[(size_t)(jb.py + (i >> L)) * p.stride + jb.px + (i & (N - 1))] - w.pred[i]);
  const int ds = jb.dcs_ctx;
  ErrBlock<int16_t, int16_t> eb;
  eb.src = src + (size_t)jb.py * p.stride + jb.px;
  eb.stride = p.stride;
  eb.pred = w.pred;
  eb.w = N;
  eb.vw = min(max(vis_w - jb.px, 0), N);
  eb.vh = min(max(vis_h - jb.py, 0), N);
  eb.maxv = maxv;
  const float skip1 = p.use_skip_bits ? p.skip_bits[0][0] : 0.0f;
  const float skip0 = p.use_skip_bits ? p.skip_bits[0][1] : 0.0f;
  float* tf = reinterpret_cast<float*>(w.u);
  int32_t* tmp = w.u + NN;
  // DCT_DCT, then (refinement) ADST_ADST, ADST_DCT, DCT_ADST, IDTX[, V_DCT,
  // H_DCT]; nibble k: the k-th type.
  constexpr uint32_t kTypeOrder = 0x3206541u;
  // the 16x16 refinement has no V / H (transform set INTRA_2)
  const int ntypes = REFINE ? ((N == 8 && p.tx_search) ? 7 : 5) : 1;
  int best = 0, btx = MT_TX_DCT_DCT;
  long long bsse = 0, dct_sse = 0, dct_guard = 0;
  float bbits = 0.0f;
#pragma unroll 1
  for (int k = 0; k < ntypes; k++) {
    const int t = (int)((kTypeOrder >> (4 * k)) & 15u);
    const int cur = k == 0 ? 0 : 1 - best;
    auto* cf = w.cfs[cur];
    int16_t* rr = w.rrs[cur];
    if constexpr (N == 8) fwd8x8(w.resid, t, q, cf, tf, tmp);
    else if constexpr (N == 16) fwd16x16(w.resid, t, q, cf, tf, tmp);
    else fwd32x32(w.resid, q, cf, tf, tmp);
    if (t == MT_TX_DCT_DCT || t >= MT_TX_ADST_ADST) {
      if (qm) apply_qm(cf, tf, sQs, NN);
      if (a.lambda > 0.0f) trellis_ctx<N>(cf, tf, dcq, acq, a.lambda, T, ds, qm, qm_full, p.band_tilt, w.tr);
    }
    if constexpr (N == 8) inv8x8(cf, t, q, qm, rr, tmp);
    else if constexpr (N == 16) inv16x16(cf, t, q, qm, rr, tmp);
    else inv32x32(cf, q, qm, rr, tmp);
    eb.resid = rr;
    const long long asse = sse_recon_block(eb, p.wsse_scale);
    if (k > 0) {
      // the gates of block8.rs:1214-1396 (and partition_search.rs:5320-5470
      // at 16x16): the ADST family within tx_guard of the DCT's SSE, IDTX
      // within tx_guard of the current best's, V / H at most the current
      // best's
      bool gate;
      if (t >= MT_TX_ADST_ADST) gate = asse <= dct_sse + dct_guard;
      else if (t == MT_TX_IDTX) gate = asse <= bsse + (p.tx_guard_shift >= 63 ? 0 : (bsse >> p.tx_guard_shift));
      else gate = asse <= bsse;
      if (!gate) continue;
    }
    const float base_rd = k == 0 ? 0.0f : rd_cost_i64(bsse, rd_lam, bbits);
    float abits;
    if (N == 8 && (t == MT_TX_V_DCT || t == MT_TX_H_DCT)) {
      if constexpr (N == 8) abits = rate_1d<8>(cf, t == MT_TX_V_DCT, T, ds, jb.mode, w.lv);
    } else {
      // unbounded: the DCT, IDTX and, at 16x16, ADST_DCT / DCT_ADST (priced
      // with luma_bits there, partition_search.rs:5396-5404)
      const bool unbounded = k == 0 || t == MT_TX_IDTX || (N == 16 && t != MT_TX_ADST_ADST);
      const float bound = unbounded ? __int_as_float(0x7f800000)
                                    : __fdiv_rn(__fsub_rn(base_rd, (float)asse), rd_lam);
      // tx-type symbol: the 5-type TX_16X16 intra set drops V_DCT / H_DCT;
      // TX_32X32 codes none
      const int sym = N == 32 ? -1 : (N == 16 && t >= MT_TX_ADST_ADST ? t - 2 : t);
      abits = rate_bounded<N>(cf, T, 0, ds, jb.mode, sym, p.use_skip_bits != 0, skip1, skip0, bound, w.lv);
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
  const auto* bcf = w.cfs[best];
  const int16_t* brr = w.rrs[best];
  if (cf_out) {
    int4* o = reinterpret_cast<int4*>(cf_out + (size_t)j * NN);
#pragma unroll 4
    for (int i = 0; i < NN / 4; i++) o[i] = make_int4(bcf[4 * i], bcf[4 * i + 1], bcf[4 * i + 2], bcf[4 * i + 3]);
  }
  if (rec_out) {
    uint16_t* o = rec_out + (size_t)j * NN;
#pragma unroll 8
    for (int i = 0; i < NN; i++) o[i] = (uint16_t)clampi((int32_t)w.pred[i] + brr[i], 0, maxv);
  }
}

// The 64x64 leaf's four-TX_32X32 leg (rd_pick_luma64's candidate loop,
// src/coder/block64.rs:1906-1958): for a (64x64 block, mode, delta), the
// quadrants in raster order (Q64, :328), each predicted at 32x32 from the
// running reconstruction with the per-transform edge flags (quad_edges,
// :2731-2745), TX_32X32 DCT_DCT with the QM and trellis_optimize_ctx in the
// quadrant's dc_sign context, the inverse, the decision distortion
// (luma_pick_distortion with luma64_wsse: chroma_sse's value, i.e. sse_recon,
// times K_PART_LAMBDA, src/coder/lossy_state.rs:2363-2382), luma_bits, and the
// reconstruction written back before the next quadrant.  total =
// mlam * mode_bits (+ mlam * delta_bits) + sum of (dist + mlam * bits), f32 in
// that order.
struct Patch64Read {
  const uint16_t* __restrict__ rec;
  int stride, px, py;
  const uint16_t* patch;
  __device__ __forceinline__ int32_t operator()(int x, int y) const {
    const int dx = x - px, dy = y - py;
    if ((unsigned)dx < 64u && (unsigned)dy < 64u) return patch[dy * 64 + dx];
    return rec[(size_t)y * stride + x];
  }
};

__global__ void __launch_bounds__(kBigThreads) quad32_kernel(
    const uint16_t* __restrict__ src, const uint16_t* __restrict__ rec, LeafArgs a,
    const uint8_t* __restrict__ qm_row, const mt_coef_costs* __restrict__ costs,
    const mt_quad32_job* __restrict__ jobs, int n, mt_quad32_result* __restrict__ res) {
  __shared__ mt_coef_costs sT;
  constexpr int NN = 1024;
  __shared__ uint8_t sQm[NN];
  __shared__ float sQs[NN];
  {
    const float* g = reinterpret_cast<const float*>(costs);
    float* s = reinterpret_cast<float*>(&sT);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
    for (int i = threadIdx.x; i < NN; i += blockDim.x) {
      const int w = a.has_qm ? qm_row[i] : 32;
      sQm[i] = (uint8_t)w;
      sQs[i] = fwd_qm_scale(w);
    }
    __syncthreads();
  }
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const mt_split16_params& p = a.p;
  const mt_quant& q = a.q;
  const mt_coef_costs& T = sT;
  const uint8_t* qm = a.has_qm ? sQm : nullptr;
  const mt_quad32_job jb = jobs[j];
  mt_quad32_result& r = res[j];
  const bool directional = jb.mode >= MT_V_PRED && jb.mode <= MT_D67_PRED;
  const bool ok = jb.px + 64 <= p.frame_w && jb.py + 64 <= p.frame_h && jb.mode <= MT_PAETH_PRED &&
                  jb.angle_delta >= -3 && jb.angle_delta <= 3 && (jb.angle_delta == 0 || directional) &&
                  jb.dcs_ctx[0] < 3 && jb.dcs_ctx[1] < 3 && jb.dcs_ctx[2] < 3 && jb.dcs_ctx[3] < 3;
  r.reserved = 0;
  if (!ok) {
    r.total = __int_as_float(0x7f800000);
    for (int k = 0; k < 4; k++) {
      r.bits[k] = __int_as_float(0x7f800000);
      r.sse[k] = 0;
    }
    return;
  }
  LeafWork<32> w;
  uint16_t patch[64 * 64];
  for (int y = 0; y < 64; y++)
    for (int x = 0; x < 64; x++) patch[y * 64 + x] = rec[(size_t)(jb.py + y) * p.stride + jb.px + x];
  const Patch64Read rd{rec, p.stride, jb.px, jb.py, patch};
  const int32_t maxv = (1 << p.bd) - 1;
  const float dcq = (float)q.dc_q, acq = (float)q.ac_q, mlam = p.rd_lambda;
  const bool qm_full = q.qm_level >= 5;
  const int vis_w = p.vis_w > 0 ? p.vis_w : p.frame_w, vis_h = p.vis_h > 0 ? p.vis_h : p.frame_h;
  const float skip1 = p.use_skip_bits ? p.skip_bits[0][0] : 0.0f;
  const float skip0 = p.use_skip_bits ? p.skip_bits[0][1] : 0.0f;
  const bool have_tr = jb.flags & 1, have_bl = (jb.flags >> 1) & 1, ft = (jb.flags >> 2) & 1;
  float total = __fmul_rn(mlam, jb.mode_bits);
  if (directional) total = __fadd_rn(total, __fmul_rn(mlam, jb.delta_bits));
  float* tf = reinterpret_cast<float*>(w.u);
  int32_t* tmp = w.u + NN;
  auto* cf = w.cfs[0];
  int16_t* rr = w.rrs[0];
#pragma unroll 1
  for (int k = 0; k < 4; k++) {
    const int sx = (k & 1) * 32, sy = (k >> 1) * 32;
    const int bx = jb.px + sx, by = jb.py + sy;
    const bool tr = k == 0 ? jb.py > 0 : (k == 1 ? have_tr : k == 2);
    const bool bl = k == 0 ? jb.px > 0 : (k == 2 ? have_bl : false);
    predict_sq_at<32>(rd, p.frame_w, p.frame_h, bx, by, jb.mode, jb.angle_delta, tr, bl, ft, p.bd, w.pred, w.u);
#pragma unroll 8
    for (int i = 0; i < NN; i++)
      w.resid[i] = (int16_t)((int32_t)src[(size_t)(by + (i >> 5)) * p.stride + bx + (i & 31)] - w.pred[i]);
    fwd32x32(w.resid, q, cf, tf, tmp);
    if (qm) apply_qm(cf, tf, sQs, NN);
    if (a.lambda > 0.0f) trellis_ctx<32>(cf, tf, dcq, acq, a.lambda, T, jb.dcs_ctx[k], qm, qm_full, p.band_tilt, w.tr);
    inv32x32(cf, q, qm, rr, tmp);
    ErrBlock<int16_t, int16_t> eb;
    eb.src = src + (size_t)by * p.stride + bx;
    eb.stride = p.stride;
    eb.pred = w.pred;
    eb.resid = rr;
    eb.w = 32;
    eb.vw = min(max(vis_w - bx, 0), 32);
    eb.vh = min(max(vis_h - by, 0), 32);
    eb.maxv = maxv;
    const long long sse = sse_recon_block(eb, p.wsse_scale);
    const float dist = __fmul_rn(__ll2float_rn(sse), 2.775f);  // proxy_wsse: K_PART_LAMBDA
    const float bits = rate_bounded<32>(cf, T, 0, jb.dcs_ctx[k], jb.mode, -1, p.use_skip_bits != 0, skip1, skip0,
                                        __int_as_float(0x7f800000), w.lv);
    total = __fadd_rn(total, __fadd_rn(dist, __fmul_rn(mlam, bits)));
    r.bits[k] = bits;
    r.sse[k] = sse;
    for (int i = 0; i < NN; i++)
      patch[(sy + (i >> 5)) * 64 + sx + (i & 31)] = (uint16_t)clampi((int32_t)w.pred[i] + rr[i], 0, maxv);
  }
  r.total = total;
}

// The 64x64 leaf's sixteen-TX_16X16 leg (rd_pick_luma64's tx_depth-2 trial,
// src/coder/block64.rs:1983-2010, through grid16_luma_pass, :1670-1805): the
// transforms in raster order, each predicted at 16x16 through the job's 64x64
// patch with the per-transform edge flags, TX_16X16 DCT_DCT with the QM and
// trellis_optimize_ctx in the dc_sign context of its four above / four left
// context bytes, the inverse, sse_recon x K_PART_LAMBDA, and the bounded rate
// walk in the txb_skip context skip_ctx_split of the same bytes with the
// DCT_DCT symbol (1) of the mode's TX_16X16 tx-type CDF; coef_res_ctx then
// fills the transform's context bytes.  total = mode cost + (dist + mlam x
// bits) + mlam x depth_bits, f32 in that order.
// grid16_kernel's per-job working set (in shared memory, see smem_arena).
struct Grid16Arena {
  LeafWork<16> w;
  uint16_t patch[64 * 64];
};

__global__ void __launch_bounds__(kBigThreads) grid16_kernel(
    const uint16_t* __restrict__ src, const uint16_t* __restrict__ rec, LeafArgs a,
    const uint8_t* __restrict__ qm_row, const mt_coef_costs* __restrict__ costs,
    const mt_grid16_job* __restrict__ jobs, int n, mt_grid16_result* __restrict__ res, int32_t* __restrict__ cf_out,
    int arena) {
  __shared__ mt_coef_costs sT;
  constexpr int NN = 256;
  __shared__ uint8_t sQm[NN];
  __shared__ float sQs[NN];
  {
    const float* g = reinterpret_cast<const float*>(costs);
    float* s = reinterpret_cast<float*>(&sT);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
    for (int i = threadIdx.x; i < NN; i += blockDim.x) {
      const int w = a.has_qm ? qm_row[i] : 32;
      sQm[i] = (uint8_t)w;
      sQs[i] = fwd_qm_scale(w);
    }
    __syncthreads();
  }
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const mt_split16_params& p = a.p;
  const mt_quant& q = a.q;
  const mt_coef_costs& T = sT;
  const uint8_t* qm = a.has_qm ? sQm : nullptr;
  const mt_grid16_job jb = jobs[j];
  mt_grid16_result& r = res[j];
  const bool directional = jb.mode >= MT_V_PRED && jb.mode <= MT_D67_PRED;
  const bool ok = jb.px + 64 <= p.frame_w && jb.py + 64 <= p.frame_h && jb.mode <= MT_PAETH_PRED &&
                  jb.angle_delta >= -3 && jb.angle_delta <= 3 && (jb.angle_delta == 0 || directional);
  r.reserved = 0;
  if (!ok) {
    r.total = r.dist = r.bits = __int_as_float(0x7f800000);
    r.sse = 0;
    if (cf_out)
      for (int i = 0; i < 4096; i++) cf_out[(size_t)j * 4096 + i] = 0;
    return;
  }
  Grid16Arena& A = smem_arena<Grid16Arena>(arena);
  LeafWork<16>& w = A.w;
  uint16_t* patch = A.patch;
  for (int y = 0; y < 64; y++)
    for (int x = 0; x < 64; x++) patch[y * 64 + x] = rec[(size_t)(jb.py + y) * p.stride + jb.px + x];
  const Patch64Read rd{rec, p.stride, jb.px, jb.py, patch};
  uint8_t actx[16], lctx[16];
#pragma unroll
  for (int i = 0; i < 16; i++) {
    actx[i] = jb.a_coef[i];
    lctx[i] = jb.l_coef[i];
  }
  const int32_t maxv = (1 << p.bd) - 1;
  const float dcq = (float)q.dc_q, acq = (float)q.ac_q, mlam = p.rd_lambda;
  const bool qm_full = q.qm_level >= 5;
  const int vis_w = p.vis_w > 0 ? p.vis_w : p.frame_w, vis_h = p.vis_h > 0 ? p.vis_h : p.frame_h;
  const bool have_tr = jb.flags & MT_CAND_HAVE_TR, have_bl = jb.flags & MT_CAND_HAVE_BL;
  const bool ft = jb.flags & MT_CAND_FILTER_TYPE;
  float* tf = reinterpret_cast<float*>(w.u);
  int32_t* tmp = w.u + NN;
  int16_t* cf = w.cfs[0];
  int16_t* rr = w.rrs[0];
  float dist = 0.0f, bits = 0.0f;
  long long sse_sum = 0;
#pragma unroll 1
  for (int t = 0; t < 16; t++) {
    const int tx = t & 3, ty = t >> 2;
    const int sx = tx * 16, sy = ty * 16, bx = jb.px + sx, by = jb.py + sy;
    const bool tr = ty == 0 ? (jb.py > 0 && (tx < 3 || have_tr)) : tx < 3;
    const bool bl = tx == 0 && jb.px > 0 && (ty < 3 || have_bl);
    predict_sq_at<16>(rd, p.frame_w, p.frame_h, bx, by, jb.mode, jb.angle_delta, tr, bl, ft, p.bd, w.pred, w.u);
#pragma unroll 8
    for (int i = 0; i < NN; i++)
      w.resid[i] = (int16_t)((int32_t)src[(size_t)(by + (i >> 4)) * p.stride + bx + (i & 15)] - w.pred[i]);
    uint32_t la = 0, ll = 0;
    int s = -8;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      la |= actx[tx * 4 + k];
      ll |= lctx[ty * 4 + k];
      s += (actx[tx * 4 + k] >> 6) + (lctx[ty * 4 + k] >> 6);
    }
    const int sk = kSkipCtxTbl[min(la & 0x3fu, 4u)][min(ll & 0x3fu, 4u)];
    const int ds = (s != 0) + (s > 0);
    fwd16x16(w.resid, MT_TX_DCT_DCT, q, cf, tf, tmp);
    if (qm) apply_qm(cf, tf, sQs, NN);
    if (a.lambda > 0.0f) trellis_ctx<16>(cf, tf, dcq, acq, a.lambda, T, ds, qm, qm_full, p.band_tilt, w.tr);
    inv16x16(cf, MT_TX_DCT_DCT, q, qm, rr, tmp);
    ErrBlock<int16_t, int16_t> eb;
    eb.src = src + (size_t)by * p.stride + bx;
    eb.stride = p.stride;
    eb.pred = w.pred;
    eb.resid = rr;
    eb.w = 16;
    eb.vw = min(max(vis_w - bx, 0), 16);
    eb.vh = min(max(vis_h - by, 0), 16);
    eb.maxv = maxv;
    const long long sse = sse_recon_block(eb, p.wsse_scale);
    dist = __fadd_rn(dist, __fmul_rn(__ll2float_rn(sse), 2.775f));  // proxy_wsse: K_PART_LAMBDA
    sse_sum += sse;
    const float skip1 = p.use_skip_bits ? p.skip_bits[sk][0] : 0.0f;
    const float skip0 = p.use_skip_bits ? p.skip_bits[sk][1] : 0.0f;
    bits = __fadd_rn(bits, rate_bounded<16>(cf, T, sk, ds, jb.mode, 1, p.use_skip_bits != 0, skip1, skip0,
                                            __int_as_float(0x7f800000), w.lv));
    const uint8_t rc = coef_res_ctx_w<16>(cf);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      actx[tx * 4 + k] = rc;
      lctx[ty * 4 + k] = rc;
    }
#pragma unroll 8
    for (int i = 0; i < NN; i++)
      patch[(sy + (i >> 4)) * 64 + sx + (i & 15)] = (uint16_t)clampi((int32_t)w.pred[i] + rr[i], 0, maxv);
    if (cf_out) {
      int4* o = reinterpret_cast<int4*>(cf_out + (size_t)j * 4096 + t * NN);
#pragma unroll 4
      for (int i = 0; i < NN / 4; i++) o[i] = make_int4(cf[4 * i], cf[4 * i + 1], cf[4 * i + 2], cf[4 * i + 3]);
    }
  }
  float total = __fmul_rn(mlam, jb.mode_bits);
  if (directional) total = __fadd_rn(total, __fmul_rn(mlam, jb.delta_bits));
  total = __fadd_rn(total, __fadd_rn(dist, __fmul_rn(mlam, bits)));
  r.total = __fadd_rn(total, __fmul_rn(mlam, jb.depth_bits));
  r.dist = dist;
  r.bits = bits;
  r.sse = sse_sum;
}

int check(const mt_split16_params* p, const mt_quant* q, int32_t n) {
  if (!p || !q || n < 0) return MT_ERR_INVALID_INPUT;
  if (p->bd != 8) return MT_ERR_UNSUPPORTED;
  if (p->frame_w < 4 || p->frame_h < 4 || p->stride < p->frame_w || p->vis_w < 0 || p->vis_h < 0)
    return MT_ERR_INVALID_INPUT;
  if (!(p->rd_lambda > 0.0f) || !(p->wsse_scale >= 0.0f) || p->tx_guard_shift < 0) return MT_ERR_INVALID_INPUT;
  return MT_OK;
}

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

template <int N, bool REFINE>
int leaf_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm, const mt_quant* quant,
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
  constexpr int T = leaf_threads<N>();
  leaf_kernel<N, REFINE><<<(unsigned)((n + T - 1) / T), T, 0,
                         reinterpret_cast<cudaStream_t>(stream)>>>(d_src, d_recon, a, d_qm_row, d_costs, d_jobs, n,
                                                                   d_results, d_cf, d_rec);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

template <int N>
int leaf_host(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
              const uint8_t* qm_row, const mt_coef_costs* costs, const mt_leaf8_job* jobs, int32_t n, int32_t refine,
              mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out);

int quad32_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm, const mt_quant* quant,
                  const uint8_t* d_qm_row, const mt_coef_costs* d_costs, const mt_quad32_job* d_jobs, int32_t n,
                  mt_quad32_result* d_results, void* stream) {
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
  quad32_kernel<<<(unsigned)((n + kBigThreads - 1) / kBigThreads), kBigThreads, 0,
                  reinterpret_cast<cudaStream_t>(stream)>>>(d_src, d_recon, a, d_qm_row, d_costs, d_jobs, n,
                                                            d_results);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int grid16_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm, const mt_quant* quant,
                  const uint8_t* d_qm_row, const mt_coef_costs* d_costs, const mt_grid16_job* d_jobs, int32_t n,
                  mt_grid16_result* d_results, int32_t* d_cf, void* stream) {
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
  const int stride = arena_stride(sizeof(Grid16Arena));
  int threads = 0;
  size_t dyn = 0;
  if (!arena_launch_shape(grid16_kernel, n, stride, kBigThreads, &threads, &dyn)) return MT_ERR_DEVICE;
  grid16_kernel<<<(unsigned)((n + threads - 1) / threads), threads, dyn, reinterpret_cast<cudaStream_t>(stream)>>>(
      d_src, d_recon, a, d_qm_row, d_costs, d_jobs, n, d_results, d_cf, stride);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // namespace

extern "C" {

int mt_leaf8_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                         const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                         const mt_leaf8_job* d_jobs, int32_t n, mt_leaf8_result* d_results, int32_t* d_cf,
                         uint16_t* d_rec, void* stream) {
  return leaf_device<8, false>(d_src, d_recon, prm, quant, d_qm_row, d_costs, d_jobs, n, d_results, d_cf, d_rec, stream);
}

int mt_leaf8_tx_refine_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                              const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                              const mt_leaf8_job* d_jobs, int32_t n, mt_leaf8_result* d_results, int32_t* d_cf,
                              uint16_t* d_rec, void* stream) {
  return leaf_device<8, true>(d_src, d_recon, prm, quant, d_qm_row, d_costs, d_jobs, n, d_results, d_cf, d_rec, stream);
}

int mt_leaf8(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
             const uint8_t* qm_row, const mt_coef_costs* costs, const mt_leaf8_job* jobs, int32_t n, int32_t refine,
             mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out) {
  return leaf_host<8>(src, recon, prm, quant, qm_row, costs, jobs, n, refine, results, cf_out, rec_out);
}

int mt_leaf16_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                          const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                          const mt_leaf8_job* d_jobs, int32_t n, mt_leaf8_result* d_results, int32_t* d_cf,
                          uint16_t* d_rec, void* stream) {
  return leaf_device<16, false>(d_src, d_recon, prm, quant, d_qm_row, d_costs, d_jobs, n, d_results, d_cf, d_rec,
                                stream);
}

int mt_leaf16_tx_refine_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                               const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                               const mt_leaf8_job* d_jobs, int32_t n, mt_leaf8_result* d_results, int32_t* d_cf,
                               uint16_t* d_rec, void* stream) {
  return leaf_device<16, true>(d_src, d_recon, prm, quant, d_qm_row, d_costs, d_jobs, n, d_results, d_cf, d_rec,
                               stream);
}

int mt_leaf16(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
              const uint8_t* qm_row, const mt_coef_costs* costs, const mt_leaf8_job* jobs, int32_t n, int32_t refine,
              mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out) {
  return leaf_host<16>(src, recon, prm, quant, qm_row, costs, jobs, n, refine, results, cf_out, rec_out);
}

int mt_leaf32_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                          const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                          const mt_leaf8_job* d_jobs, int32_t n, mt_leaf8_result* d_results, int32_t* d_cf,
                          uint16_t* d_rec, void* stream) {
  return leaf_device<32, false>(d_src, d_recon, prm, quant, d_qm_row, d_costs, d_jobs, n, d_results, d_cf, d_rec,
                                stream);
}

int mt_leaf32(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
              const uint8_t* qm_row, const mt_coef_costs* costs, const mt_leaf8_job* jobs, int32_t n,
              mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out) {
  return leaf_host<32>(src, recon, prm, quant, qm_row, costs, jobs, n, 0, results, cf_out, rec_out);
}

int mt_quad32_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                          const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                          const mt_quad32_job* d_jobs, int32_t n, mt_quad32_result* d_results, void* stream) {
  return quad32_device(d_src, d_recon, prm, quant, d_qm_row, d_costs, d_jobs, n, d_results, stream);
}

int mt_quad32_luma(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
                   const uint8_t* qm_row, const mt_coef_costs* costs, const mt_quad32_job* jobs, int32_t n,
                   mt_quad32_result* results) {
  int rc = check(prm, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!src || !recon || !costs || !jobs || !results) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)prm->stride * prm->frame_h * sizeof(uint16_t);
  const size_t o_src = 0, o_rec = up256(plane), o_qm = o_rec + up256(plane), o_cost = o_qm + up256(1024);
  const size_t o_jobs = o_cost + up256(sizeof(mt_coef_costs));
  const size_t o_res = o_jobs + up256((size_t)n * sizeof(mt_quad32_job));
  const size_t total = o_res + up256((size_t)n * sizeof(mt_quad32_result));
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, total) != cudaSuccess) return MT_ERR_ALLOC;
  const bool has_qm = quant->qm_level < 15 && qm_row != nullptr;
  cudaError_t e = cudaMemcpy(d + o_src, src, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_rec, recon, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && has_qm) e = cudaMemcpy(d + o_qm, qm_row, 1024, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_cost, costs, sizeof(mt_coef_costs), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_jobs, jobs, (size_t)n * sizeof(mt_quad32_job), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = quad32_device(reinterpret_cast<const uint16_t*>(d + o_src), reinterpret_cast<const uint16_t*>(d + o_rec),
                       prm, quant, has_qm ? d + o_qm : nullptr, reinterpret_cast<const mt_coef_costs*>(d + o_cost),
                       reinterpret_cast<const mt_quad32_job*>(d + o_jobs), n,
                       reinterpret_cast<mt_quad32_result*>(d + o_res), nullptr);
    if (rc == MT_OK) e = cudaMemcpy(results, d + o_res, (size_t)n * sizeof(mt_quad32_result), cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_grid16_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                          const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                          const mt_grid16_job* d_jobs, int32_t n, mt_grid16_result* d_results, int32_t* d_cf,
                          void* stream) {
  return grid16_device(d_src, d_recon, prm, quant, d_qm_row, d_costs, d_jobs, n, d_results, d_cf, stream);
}

int mt_grid16_luma(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
                   const uint8_t* qm_row, const mt_coef_costs* costs, const mt_grid16_job* jobs, int32_t n,
                   mt_grid16_result* results, int32_t* cf_out) {
  int rc = check(prm, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!src || !recon || !costs || !jobs || !results) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)prm->stride * prm->frame_h * sizeof(uint16_t);
  const size_t o_src = 0, o_rec = up256(plane), o_qm = o_rec + up256(plane), o_cost = o_qm + up256(256);
  const size_t o_jobs = o_cost + up256(sizeof(mt_coef_costs));
  const size_t o_res = o_jobs + up256((size_t)n * sizeof(mt_grid16_job));
  const size_t o_cf = o_res + up256((size_t)n * sizeof(mt_grid16_result));
  const size_t total = o_cf + (cf_out ? up256((size_t)n * 4096 * 4) : 0);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, total) != cudaSuccess) return MT_ERR_ALLOC;
  const bool has_qm = quant->qm_level < 15 && qm_row != nullptr;
  cudaError_t e = cudaMemcpy(d + o_src, src, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_rec, recon, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && has_qm) e = cudaMemcpy(d + o_qm, qm_row, 256, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_cost, costs, sizeof(mt_coef_costs), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_jobs, jobs, (size_t)n * sizeof(mt_grid16_job), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = grid16_device(reinterpret_cast<const uint16_t*>(d + o_src), reinterpret_cast<const uint16_t*>(d + o_rec),
                       prm, quant, has_qm ? d + o_qm : nullptr, reinterpret_cast<const mt_coef_costs*>(d + o_cost),
                       reinterpret_cast<const mt_grid16_job*>(d + o_jobs), n,
                       reinterpret_cast<mt_grid16_result*>(d + o_res),
                       cf_out ? reinterpret_cast<int32_t*>(d + o_cf) : nullptr, nullptr);
    if (rc == MT_OK) e = cudaMemcpy(results, d + o_res, (size_t)n * sizeof(mt_grid16_result), cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && cf_out)
      e = cudaMemcpy(cf_out, d + o_cf, (size_t)n * 4096 * 4, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"

namespace {

// Host-buffer form of the leaf searches.
template <int N>
int leaf_host(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
              const uint8_t* qm_row, const mt_coef_costs* costs, const mt_leaf8_job* jobs, int32_t n, int32_t refine,
              mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out) {
  constexpr size_t NN = (size_t)N * N;
  int rc = check(prm, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!src || !recon || !costs || !jobs || !results) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)prm->stride * prm->frame_h * sizeof(uint16_t);
  const size_t o_src = 0, o_rec = up256(plane), o_qm = o_rec + up256(plane), o_cost = o_qm + up256(NN);
  const size_t o_jobs = o_cost + up256(sizeof(mt_coef_costs));
  const size_t o_res = o_jobs + up256((size_t)n * sizeof(mt_leaf8_job));
  const size_t o_cf = o_res + up256((size_t)n * sizeof(mt_leaf8_result));
  const size_t o_out = o_cf + (cf_out ? up256((size_t)n * NN * 4) : 0);
  const size_t total = o_out + (rec_out ? up256((size_t)n * NN * 2) : 0);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, total) != cudaSuccess) return MT_ERR_ALLOC;
  const bool has_qm = quant->qm_level < 15 && qm_row != nullptr;
  cudaError_t e = cudaMemcpy(d + o_src, src, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_rec, recon, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && has_qm) e = cudaMemcpy(d + o_qm, qm_row, NN, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_cost, costs, sizeof(mt_coef_costs), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_jobs, jobs, (size_t)n * sizeof(mt_leaf8_job), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    auto fn = refine ? leaf_device<N, N != 32> : leaf_device<N, false>;
    rc = fn(reinterpret_cast<const uint16_t*>(d + o_src), reinterpret_cast<const uint16_t*>(d + o_rec), prm, quant,
            has_qm ? d + o_qm : nullptr, reinterpret_cast<const mt_coef_costs*>(d + o_cost),
            reinterpret_cast<const mt_leaf8_job*>(d + o_jobs), n, reinterpret_cast<mt_leaf8_result*>(d + o_res),
            cf_out ? reinterpret_cast<int32_t*>(d + o_cf) : nullptr,
            rec_out ? reinterpret_cast<uint16_t*>(d + o_out) : nullptr, nullptr);
    if (rc == MT_OK) e = cudaMemcpy(results, d + o_res, (size_t)n * sizeof(mt_leaf8_result), cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && cf_out) e = cudaMemcpy(cf_out, d + o_cf, (size_t)n * NN * 4, cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && rec_out) e = cudaMemcpy(rec_out, d + o_out, (size_t)n * NN * 2, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // namespace

extern "C" {

}  // extern "C"
