// C ABI of the B200 intra RD core (declared in include/maroontree_b200.h).
// Host-side helpers mirror the reference's quantiser and rate-table set-up;
// every batched entry point launches the CUDA kernels of chain.cu.  There is
// no CPU fallback: without a usable device the calls return MT_ERR_DEVICE.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "../../include/maroontree_b200.h"
#include "av1_tables.h"

namespace mth {
size_t chain8_scratch_bytes(int n);
cudaError_t launch_chain8(const uint16_t* src, const uint16_t* rec, const mt_chain_params& p, const mt_quant& q,
                          float trellis_lambda, const uint8_t* qm_row, const mt_coef_costs* costs,
                          const mt_candidate* cands, int n, mt_candidate_result* res, int32_t* lv, int32_t* ro,
                          void* scratch, cudaStream_t st);
size_t level8_scratch_bytes(int nblocks, int ncombos);
cudaError_t launch_level4(const uint16_t* src, const uint16_t* rec, const mt_chain_params& p, const mt_quant& q,
                          float trellis_lambda, const uint8_t* qm_row, const mt_coef_costs* costs,
                          const mt_block8* blocks, int nblocks, const mt_combo* combos, int ncombos,
                          mt_candidate_result* res, void* scratch, mt_block_best* best, cudaStream_t st);
cudaError_t launch_level16(const uint16_t* src, const uint16_t* rec, const mt_chain_params& p, const mt_quant& q,
                           float trellis_lambda, const uint8_t* qm_row, const mt_coef_costs* costs,
                           const mt_block8* blocks, int nblocks, const mt_combo* combos, int ncombos,
                           mt_candidate_result* res, void* scratch, mt_block_best* best, cudaStream_t st);
cudaError_t launch_level8(const uint16_t* src, const uint16_t* rec, const mt_chain_params& p, const mt_quant& q,
                          float trellis_lambda, const uint8_t* qm_row, const mt_coef_costs* costs,
                          const mt_block8* blocks, int nblocks, const mt_combo* combos, int ncombos,
                          mt_candidate_result* res, void* scratch, mt_block_best* best, cudaStream_t st);
cudaError_t launch_fwd8(const int32_t* resid, const uint8_t* types, int n, const mt_quant& q, const uint8_t* qm,
                        int32_t* levels, float* targets, cudaStream_t st);
cudaError_t launch_inv8(const int32_t* levels, const uint8_t* types, int n, const mt_quant& q, const uint8_t* qm,
                        int32_t* out, cudaStream_t st);
cudaError_t launch_trellis8(int32_t* levels, const float* targets, int n, float dc_q, float ac_q, float lambda,
                            cudaStream_t st);
cudaError_t launch_pred8(const uint16_t* rec, const mt_chain_params& p, const mt_candidate* cands, int n, int32_t* out,
                         cudaStream_t st);
}  // namespace mth

namespace {

int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Quant field set-up shared by luma and chroma (src/quant.rs:351-418; 8-bit
// clips of src/quant.rs:239-247).
void fill_quant(int32_t dc, int32_t ac, int32_t qm_level, int32_t chroma, int32_t qidx, mt_quant* q) {
  q->dc_q = dc;
  q->ac_q = ac;
  q->q_mult_dc = (int32_t)llround(65536.0 / (double)dc);
  q->q_mult_ac = (int32_t)llround(65536.0 / (double)ac);
  q->rmin = q->cmin = -32768;
  q->rmax = q->cmax = 32767;
  q->cf_max = 32767;
  q->qm_level = qm_level > 15 ? 15 : qm_level;
  q->qm_chroma = chroma;
  q->qidx = qidx;
}

// Q22 -log2 table of src/cost.rs:156-169 (glibc log2f on the host).
const uint32_t* cost_table() {
  static uint32_t tab[32769];
  static std::once_flag once;
  std::call_once(once, [] {
    tab[0] = 0;
    for (int p = 1; p <= 32768; p++) {
      float bits = -log2f((float)p * (1.0f / 32768.0f));
      tab[p] = (uint32_t)roundf(bits * (float)(1u << 22));
    }
  });
  return tab;
}
float cdf_cost(const uint16_t* cdf, int s) {
  int32_t fl = s > 0 ? cdf[s - 1] : 32768;
  int32_t p = fl - (int32_t)cdf[s];
  if (p < 1) p = 1;
  return (float)cost_table()[p] * (1.0f / 4194304.0f);
}

// scaled_trellis_lambda (src/trellis.rs:38-53) with the shipped calibration
// trellis_calib = 1.15 (src/tuning.rs:953).
float scaled_trellis_lambda(float dc_q, float lambda0) {
  const float calib = 0.045025873597302174f * 0.5525f;
  volatile float a = calib * 1.15f;  // keep the reference's left-to-right product
  float aom = a * dc_q;
  aom = aom * dc_q;
  float k = 0.0015f * dc_q;
  k = 3.3f + k;
  aom = aom * k;
  return aom * (lambda0 / 0.05f);
}

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Grow-only device workspace for the host-buffer entry points.
struct Workspace {
  std::mutex mu;
  void* ptr = nullptr;
  size_t cap = 0;
  void* get(size_t bytes) {
    if (bytes <= cap) return ptr;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    if (cudaMalloc(&ptr, bytes) != cudaSuccess) return nullptr;
    cap = bytes;
    return ptr;
  }
};
Workspace g_ws;

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

extern "C" {

const char* mt_version(void) { return "maroontree_b200 0.1 (sm_100a)"; }

int mt_quant_init(uint8_t base_q_idx, uint8_t bd, uint8_t qm_level, mt_quant* out) {
  if (!out) return MT_ERR_INVALID_INPUT;
  if (bd != 8) return MT_ERR_UNSUPPORTED;
  int dc_idx = clampi((int)base_q_idx - 8, 0, 255);
  fill_quant(MT_DC_QLOOKUP_8[dc_idx], MT_AC_QLOOKUP_8[base_q_idx], qm_level, 0, base_q_idx, out);
  return MT_OK;
}

int mt_quant_init_chroma(uint8_t base_q_idx, int32_t dc_delta, int32_t ac_delta, uint8_t bd, uint8_t qm_level,
                         mt_quant* out) {
  if (!out) return MT_ERR_INVALID_INPUT;
  if (bd != 8) return MT_ERR_UNSUPPORTED;
  int dc_idx = clampi((int)base_q_idx + dc_delta, 0, 255);
  int ac_idx = clampi((int)base_q_idx + ac_delta, 0, 255);
  fill_quant(MT_DC_QLOOKUP_8[dc_idx], MT_AC_QLOOKUP_8[ac_idx], qm_level, 1, ac_idx, out);
  return MT_OK;
}

const uint8_t* mt_qm_row(int32_t qm_level, int32_t chroma, int32_t w, int32_t h) {
  if (qm_level < 0 || qm_level >= 15 || w != h) return nullptr;
  int off;
  switch (w) {
    case 4: off = 0; break;
    case 8: off = 16; break;
    case 16: off = 80; break;
    case 32: off = 336; break;
    default: return nullptr;
  }
  return &MT_AV1_IQM[((size_t)qm_level * 2 + (chroma ? 1 : 0)) * 3344 + off];
}

const uint16_t* mt_default_scan(int32_t n) {
  switch (n) {
    case 4: return MT_SCAN_4X4;
    case 8: return MT_SCAN_8X8;
    case 16: return MT_SCAN_16X16;
    case 32: return MT_SCAN_32X32;
  }
  return nullptr;
}

int mt_coef_costs_build(const mt_coef_cdfs* c, mt_coef_costs* o) {
  if (!c || !o) return MT_ERR_INVALID_INPUT;
  memset(o, 0, sizeof(*o));
  for (int k = 0; k < 13; k++)
    for (int s = 0; s < 2; s++) o->txb_skip[k][s] = cdf_cost(c->txb_skip[k], s);
  for (int k = 0; k < 42; k++)
    for (int s = 0; s < 4; s++) o->base_tok[k][s] = cdf_cost(c->base_tok[k], s);
  for (int k = 0; k < 21; k++) {
    // Cumulative base-range ladder (src/cost.rs:214-241).
    float c0 = cdf_cost(c->br_tok[k], 0), c1 = cdf_cost(c->br_tok[k], 1);
    float c2 = cdf_cost(c->br_tok[k], 2), c3 = cdf_cost(c->br_tok[k], 3);
    float x2 = c3 + c3, x3 = x2 + c3, x4 = x3 + c3;
    float row[13] = {c0, c1, c2, c3 + c0, c3 + c1, c3 + c2, x2 + c0, x2 + c1, x2 + c2, x3 + c0, x3 + c1, x3 + c2, x4};
    memcpy(o->br_cum[k], row, sizeof(row));
  }
  for (int k = 0; k < 4; k++)
    for (int s = 0; s < 3; s++) o->eob_base[k][s] = cdf_cost(c->eob_base[k], s);
  for (int k = 0; k < 11; k++)
    for (int s = 0; s < 2; s++) o->eob_hi[k][s] = cdf_cost(c->eob_hi[k], s);
  for (int s = 0; s < 11; s++) o->eob_bin[s] = cdf_cost(c->eob_bin, s);
  for (int k = 0; k < 3; k++)
    for (int s = 0; s < 2; s++) o->dc_sign[k][s] = cdf_cost(c->dc_sign[k], s);
  for (int m = 0; m < 13; m++)
    for (int s = 0; s < 16; s++) o->txtp[m][s] = cdf_cost(c->txtp[m], s);
  for (int s = 0; s < 11; s++) o->eob_bin_1d[s] = cdf_cost(c->eob_bin_1d, s);
  return MT_OK;
}

int mt_uv_mode_costs_build(const mt_uv_mode_cdfs* c, mt_uv_mode_costs* o) {
  if (!c || !o) return MT_ERR_INVALID_INPUT;
  for (int m = 0; m < 13; m++)
    for (int s = 0; s < 14; s++) o->uv_mode[m][s] = cdf_cost(c->uv_mode[m], s);
  for (int m = 0; m < 8; m++)
    for (int s = 0; s < 7; s++) o->angle_delta[m][s] = cdf_cost(c->angle_delta[m], s);
  for (int s = 0; s < 8; s++) o->cfl_sign[s] = cdf_cost(c->cfl_sign, s);
  for (int k = 0; k < 6; k++)
    for (int s = 0; s < 16; s++) o->cfl_alpha[k][s] = cdf_cost(c->cfl_alpha[k], s);
  return MT_OK;
}

// uv_mode_bits (src/coder/lossy_state.rs:1302-1349); the same sums as the
// device's uv_mode_bits_dev.
float mt_uv_mode_bits(const mt_uv_mode_costs* c, int32_t y_mode, int32_t uv_mode, int32_t cfl, int32_t au, int32_t av) {
  if (!c || y_mode < 0 || y_mode > 12 || uv_mode < 0 || uv_mode > 13) return INFINITY;
  if (!cfl) {
    float bits = c->uv_mode[y_mode][uv_mode];
    if (uv_mode >= MT_V_PRED && uv_mode <= MT_D67_PRED) bits += c->angle_delta[uv_mode - MT_V_PRED][3];
    return bits;
  }
  if (au < -16 || au > 16 || av < -16 || av > 16) return INFINITY;
  const int su = au == 0 ? 0 : (au < 0 ? 1 : 2), sv = av == 0 ? 0 : (av < 0 ? 1 : 2);
  const int sign = su * 3 + sv;
  if (sign == 0) return c->uv_mode[y_mode][MT_DC_PRED];
  float bits = c->uv_mode[y_mode][MT_UV_CFL_PRED] + c->cfl_sign[sign - 1];
  if (su != 0) bits += c->cfl_alpha[(su == 2) * 3 + sv][(au < 0 ? -au : au) - 1];
  if (sv != 0) bits += c->cfl_alpha[(sv == 2) * 3 + su][(av < 0 ? -av : av) - 1];
  return bits;
}

extern "C++" {
namespace mth {
// scaled_trellis_lambda for the other translation units of the library.
float scaled_trellis_lambda_host(float dc_q, float lambda0) { return scaled_trellis_lambda(dc_q, lambda0); }
}  // namespace mth
}

static int check_chain(const mt_chain_params* prm, const mt_quant* q, int32_t n, int32_t tx_size = 8) {
  if (!prm || !q || n < 0) return MT_ERR_INVALID_INPUT;
  if (prm->tx_size != tx_size || prm->bd != 8) return MT_ERR_UNSUPPORTED;
  if (prm->frame_w <= 0 || prm->frame_h <= 0 || prm->stride < prm->frame_w) return MT_ERR_INVALID_INPUT;
  return MT_OK;
}

size_t mt_candidate_chain_scratch_bytes(int32_t n) { return n > 0 ? mth::chain8_scratch_bytes(n) : 0; }

int mt_candidate_chain_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_chain_params* prm,
                              const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                              const mt_candidate* d_cands, int32_t n, mt_candidate_result* d_results,
                              int32_t* d_levels_out, int32_t* d_recon_out, void* d_scratch, void* stream) {
  int rc = check_chain(prm, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!d_src || !d_recon || !d_costs || !d_cands || !d_results) return MT_ERR_INVALID_INPUT;
  float tl = scaled_trellis_lambda((float)quant->dc_q, prm->trellis_lambda0);
  cudaError_t e = mth::launch_chain8(d_src, d_recon, *prm, *quant, tl, d_qm_row, d_costs, d_cands, n, d_results,
                                     d_levels_out, d_recon_out, d_scratch, as_stream(stream));
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_rdo_level8_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_chain_params* prm,
                         const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                         const mt_block8* d_blocks, int32_t nblocks, const mt_combo* d_combos, int32_t ncombos,
                         mt_block_best* d_best, mt_candidate_result* d_results, void* d_scratch, void* stream) {
  int rc = check_chain(prm, quant, 0);
  if (rc != MT_OK) return rc;
  if (nblocks < 0 || ncombos < 0) return MT_ERR_INVALID_INPUT;
  if (nblocks == 0 || ncombos == 0) return MT_OK;
  if ((long long)nblocks * ncombos > 0x7fffffffLL) return MT_ERR_INVALID_INPUT;
  if (ncombos > MT_LEVEL_MAX_COMBOS) return MT_ERR_TOO_LARGE;
  if (!d_src || !d_recon || !d_costs || !d_blocks || !d_combos || !d_best || !d_results || !d_scratch)
    return MT_ERR_INVALID_INPUT;
  float tl = scaled_trellis_lambda((float)quant->dc_q, prm->trellis_lambda0);
  cudaError_t e = mth::launch_level8(d_src, d_recon, *prm, *quant, tl, d_qm_row, d_costs, d_blocks, nblocks, d_combos,
                                     ncombos, d_results, d_scratch, d_best, as_stream(stream));
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

size_t mt_rdo_level8_scratch_bytes(int32_t nblocks, int32_t ncombos) {
  if (nblocks <= 0 || ncombos <= 0 || ncombos > MT_LEVEL_MAX_COMBOS) return 0;
  return mth::level8_scratch_bytes(nblocks, ncombos);
}

int mt_rdo_level8(const uint16_t* src, const uint16_t* recon, const mt_chain_params* prm, const mt_quant* quant,
                  const uint8_t* qm_row, const mt_coef_costs* costs, const mt_block8* blocks, int32_t nblocks,
                  const mt_combo* combos, int32_t ncombos, mt_block_best* best_out, mt_candidate_result* results_out) {
  int rc = check_chain(prm, quant, 0);
  if (rc != MT_OK) return rc;
  if (nblocks < 0 || ncombos < 0) return MT_ERR_INVALID_INPUT;
  if (nblocks == 0 || ncombos == 0) return MT_OK;
  if ((long long)nblocks * ncombos > 0x7fffffffLL) return MT_ERR_INVALID_INPUT;
  if (ncombos > MT_LEVEL_MAX_COMBOS) return MT_ERR_TOO_LARGE;
  if (!src || !recon || !costs || !blocks || !combos || !best_out) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)prm->stride * prm->frame_h * sizeof(uint16_t);
  const size_t nres = (size_t)nblocks * ncombos;
  size_t off_src = 0, off_rec = align256(plane), off_cost = off_rec + align256(plane);
  size_t off_qm = off_cost + align256(sizeof(mt_coef_costs));
  size_t off_blk = off_qm + 256;
  size_t off_cmb = off_blk + align256((size_t)nblocks * sizeof(mt_block8));
  size_t off_best = off_cmb + align256((size_t)ncombos * sizeof(mt_combo));
  size_t off_key = off_best + align256((size_t)nblocks * sizeof(mt_block_best));
  size_t off_res = off_key + align256(mth::level8_scratch_bytes(nblocks, ncombos));
  size_t total = off_res + align256(nres * sizeof(mt_candidate_result));
  std::lock_guard<std::mutex> lock(g_ws.mu);
  char* base = (char*)g_ws.get(total);
  if (!base) return MT_ERR_ALLOC;
  cudaStream_t st = 0;
  cudaError_t e = cudaSuccess;
  auto cp = [&](size_t off, const void* h, size_t bytes) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + off, h, bytes, cudaMemcpyHostToDevice, st);
  };
  cp(off_src, src, plane);
  cp(off_rec, recon, plane);
  cp(off_cost, costs, sizeof(mt_coef_costs));
  if (qm_row) cp(off_qm, qm_row, 64);
  cp(off_blk, blocks, (size_t)nblocks * sizeof(mt_block8));
  cp(off_cmb, combos, (size_t)ncombos * sizeof(mt_combo));
  if (e != cudaSuccess) return MT_ERR_DEVICE;
  float tl = scaled_trellis_lambda((float)quant->dc_q, prm->trellis_lambda0);
  e = mth::launch_level8((const uint16_t*)(base + off_src), (const uint16_t*)(base + off_rec), *prm, *quant, tl,
                         qm_row ? (const uint8_t*)(base + off_qm) : nullptr, (const mt_coef_costs*)(base + off_cost),
                         (const mt_block8*)(base + off_blk), nblocks, (const mt_combo*)(base + off_cmb), ncombos,
                         (mt_candidate_result*)(base + off_res), base + off_key, (mt_block_best*)(base + off_best),
                         st);
  if (e != cudaSuccess) return MT_ERR_DEVICE;
  e = cudaMemcpyAsync(best_out, base + off_best, (size_t)nblocks * sizeof(mt_block_best), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && results_out)
    e = cudaMemcpyAsync(results_out, base + off_res, nres * sizeof(mt_candidate_result), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"

namespace {

using LevelLaunch = cudaError_t (*)(const uint16_t*, const uint16_t*, const mt_chain_params&, const mt_quant&, float,
                                    const uint8_t*, const mt_coef_costs*, const mt_block8*, int, const mt_combo*, int,
                                    mt_candidate_result*, void*, mt_block_best*, cudaStream_t);

// The 4x4 and 16x16 levels: scratch is the per-block argmin keys.
size_t small_level_scratch(int32_t nblocks, int32_t ncombos) {
  if (nblocks <= 0 || ncombos <= 0 || ncombos > MT_LEVEL_MAX_COMBOS) return 0;
  return (size_t)nblocks * 8;
}

int small_level_device(int tx, LevelLaunch launch, const uint16_t* d_src, const uint16_t* d_recon,
                       const mt_chain_params* prm, const mt_quant* quant, const uint8_t* d_qm_row,
                       const mt_coef_costs* d_costs, const mt_block8* d_blocks, int32_t nblocks,
                       const mt_combo* d_combos, int32_t ncombos, mt_block_best* d_best,
                       mt_candidate_result* d_results, void* d_scratch, void* stream) {
  int rc = check_chain(prm, quant, 0, tx);
  if (rc != MT_OK) return rc;
  if (nblocks < 0 || ncombos < 0) return MT_ERR_INVALID_INPUT;
  if (nblocks == 0 || ncombos == 0) return MT_OK;
  if ((long long)nblocks * ncombos > 0x7fffffffLL) return MT_ERR_INVALID_INPUT;
  if (ncombos > MT_LEVEL_MAX_COMBOS) return MT_ERR_TOO_LARGE;
  if (!d_src || !d_recon || !d_costs || !d_blocks || !d_combos || !d_best || !d_results || !d_scratch)
    return MT_ERR_INVALID_INPUT;
  float tl = scaled_trellis_lambda((float)quant->dc_q, prm->trellis_lambda0);
  cudaError_t e = launch(d_src, d_recon, *prm, *quant, tl, d_qm_row, d_costs, d_blocks, nblocks, d_combos, ncombos,
                         d_results, d_scratch, d_best, as_stream(stream));
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int small_level_host(int tx, LevelLaunch launch, const uint16_t* src, const uint16_t* recon,
                     const mt_chain_params* prm, const mt_quant* quant, const uint8_t* qm_row,
                     const mt_coef_costs* costs, const mt_block8* blocks, int32_t nblocks, const mt_combo* combos,
                     int32_t ncombos, mt_block_best* best_out, mt_candidate_result* results_out) {
  int rc = check_chain(prm, quant, 0, tx);
  if (rc != MT_OK) return rc;
  if (nblocks < 0 || ncombos < 0) return MT_ERR_INVALID_INPUT;
  if (nblocks == 0 || ncombos == 0) return MT_OK;
  if ((long long)nblocks * ncombos > 0x7fffffffLL) return MT_ERR_INVALID_INPUT;
  if (ncombos > MT_LEVEL_MAX_COMBOS) return MT_ERR_TOO_LARGE;
  if (!src || !recon || !costs || !blocks || !combos || !best_out) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)prm->stride * prm->frame_h * sizeof(uint16_t);
  const size_t nres = (size_t)nblocks * ncombos;
  const size_t qm_bytes = (size_t)tx * tx;
  size_t off_src = 0, off_rec = align256(plane), off_cost = off_rec + align256(plane);
  size_t off_qm = off_cost + align256(sizeof(mt_coef_costs));
  size_t off_blk = off_qm + 256;
  size_t off_cmb = off_blk + align256((size_t)nblocks * sizeof(mt_block8));
  size_t off_best = off_cmb + align256((size_t)ncombos * sizeof(mt_combo));
  size_t off_key = off_best + align256((size_t)nblocks * sizeof(mt_block_best));
  size_t off_res = off_key + align256((size_t)nblocks * 8);
  size_t total = off_res + align256(nres * sizeof(mt_candidate_result));
  std::lock_guard<std::mutex> lock(g_ws.mu);
  char* base = (char*)g_ws.get(total);
  if (!base) return MT_ERR_ALLOC;
  cudaStream_t st = 0;
  cudaError_t e = cudaSuccess;
  auto cp = [&](size_t off, const void* h, size_t bytes) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + off, h, bytes, cudaMemcpyHostToDevice, st);
  };
  cp(off_src, src, plane);
  cp(off_rec, recon, plane);
  cp(off_cost, costs, sizeof(mt_coef_costs));
  if (qm_row) cp(off_qm, qm_row, qm_bytes);
  cp(off_blk, blocks, (size_t)nblocks * sizeof(mt_block8));
  cp(off_cmb, combos, (size_t)ncombos * sizeof(mt_combo));
  if (e != cudaSuccess) return MT_ERR_DEVICE;
  float tl = scaled_trellis_lambda((float)quant->dc_q, prm->trellis_lambda0);
  e = launch((const uint16_t*)(base + off_src), (const uint16_t*)(base + off_rec), *prm, *quant, tl,
             qm_row ? (const uint8_t*)(base + off_qm) : nullptr, (const mt_coef_costs*)(base + off_cost),
             (const mt_block8*)(base + off_blk), nblocks, (const mt_combo*)(base + off_cmb), ncombos,
             (mt_candidate_result*)(base + off_res), base + off_key, (mt_block_best*)(base + off_best), st);
  if (e != cudaSuccess) return MT_ERR_DEVICE;
  e = cudaMemcpyAsync(best_out, base + off_best, (size_t)nblocks * sizeof(mt_block_best), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && results_out)
    e = cudaMemcpyAsync(results_out, base + off_res, nres * sizeof(mt_candidate_result), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // namespace

extern "C" {

size_t mt_rdo_level4_scratch_bytes(int32_t nblocks, int32_t ncombos) { return small_level_scratch(nblocks, ncombos); }

int mt_rdo_level4_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_chain_params* prm,
                         const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                         const mt_block8* d_blocks, int32_t nblocks, const mt_combo* d_combos, int32_t ncombos,
                         mt_block_best* d_best, mt_candidate_result* d_results, void* d_scratch, void* stream) {
  return small_level_device(4, mth::launch_level4, d_src, d_recon, prm, quant, d_qm_row, d_costs, d_blocks, nblocks,
                            d_combos, ncombos, d_best, d_results, d_scratch, stream);
}

int mt_rdo_level4(const uint16_t* src, const uint16_t* recon, const mt_chain_params* prm, const mt_quant* quant,
                  const uint8_t* qm_row, const mt_coef_costs* costs, const mt_block8* blocks, int32_t nblocks,
                  const mt_combo* combos, int32_t ncombos, mt_block_best* best_out, mt_candidate_result* results_out) {
  return small_level_host(4, mth::launch_level4, src, recon, prm, quant, qm_row, costs, blocks, nblocks, combos,
                          ncombos, best_out, results_out);
}

size_t mt_rdo_level16_scratch_bytes(int32_t nblocks, int32_t ncombos) { return small_level_scratch(nblocks, ncombos); }

int mt_rdo_level16_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_chain_params* prm,
                          const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                          const mt_block8* d_blocks, int32_t nblocks, const mt_combo* d_combos, int32_t ncombos,
                          mt_block_best* d_best, mt_candidate_result* d_results, void* d_scratch, void* stream) {
  return small_level_device(16, mth::launch_level16, d_src, d_recon, prm, quant, d_qm_row, d_costs, d_blocks,
                            nblocks, d_combos, ncombos, d_best, d_results, d_scratch, stream);
}

int mt_rdo_level16(const uint16_t* src, const uint16_t* recon, const mt_chain_params* prm, const mt_quant* quant,
                   const uint8_t* qm_row, const mt_coef_costs* costs, const mt_block8* blocks, int32_t nblocks,
                   const mt_combo* combos, int32_t ncombos, mt_block_best* best_out,
                   mt_candidate_result* results_out) {
  return small_level_host(16, mth::launch_level16, src, recon, prm, quant, qm_row, costs, blocks, nblocks, combos,
                          ncombos, best_out, results_out);
}

int mt_candidate_chain(const uint16_t* src, const uint16_t* recon, const mt_chain_params* prm, const mt_quant* quant,
                       const uint8_t* qm_row, const mt_coef_costs* costs, const mt_candidate* cands, int32_t n,
                       mt_candidate_result* results, int32_t* levels_out, int32_t* recon_out) {
  int rc = check_chain(prm, quant, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!src || !recon || !costs || !cands || !results) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)prm->stride * prm->frame_h * sizeof(uint16_t);
  const size_t blk = (size_t)n * 64 * sizeof(int32_t);
  size_t off_src = 0, off_rec = align256(plane), off_cost = off_rec + align256(plane);
  size_t off_qm = off_cost + align256(sizeof(mt_coef_costs));
  size_t off_cand = off_qm + 256;
  size_t off_res = off_cand + align256((size_t)n * sizeof(mt_candidate));
  size_t off_lv = off_res + align256((size_t)n * sizeof(mt_candidate_result));
  size_t off_ro = off_lv + (levels_out ? align256(blk) : 0);
  size_t off_scr = off_ro + (recon_out ? align256(blk) : 0);
  size_t total = off_scr + align256(mth::chain8_scratch_bytes(n));
  std::lock_guard<std::mutex> lock(g_ws.mu);
  char* base = (char*)g_ws.get(total);
  if (!base) return MT_ERR_ALLOC;
  cudaStream_t st = 0;
  cudaError_t e = cudaSuccess;
  auto cp = [&](size_t off, const void* h, size_t bytes) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + off, h, bytes, cudaMemcpyHostToDevice, st);
  };
  cp(off_src, src, plane);
  cp(off_rec, recon, plane);
  cp(off_cost, costs, sizeof(mt_coef_costs));
  if (qm_row) cp(off_qm, qm_row, 64);
  cp(off_cand, cands, (size_t)n * sizeof(mt_candidate));
  if (e != cudaSuccess) return MT_ERR_DEVICE;
  float tl = scaled_trellis_lambda((float)quant->dc_q, prm->trellis_lambda0);
  e = mth::launch_chain8((const uint16_t*)(base + off_src), (const uint16_t*)(base + off_rec), *prm, *quant, tl,
                         qm_row ? (const uint8_t*)(base + off_qm) : nullptr, (const mt_coef_costs*)(base + off_cost),
                         (const mt_candidate*)(base + off_cand), n, (mt_candidate_result*)(base + off_res),
                         levels_out ? (int32_t*)(base + off_lv) : nullptr,
                         recon_out ? (int32_t*)(base + off_ro) : nullptr, base + off_scr, st);
  if (e != cudaSuccess) return MT_ERR_DEVICE;
  e = cudaMemcpyAsync(results, base + off_res, (size_t)n * sizeof(mt_candidate_result), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && levels_out) e = cudaMemcpyAsync(levels_out, base + off_lv, blk, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && recon_out) e = cudaMemcpyAsync(recon_out, base + off_ro, blk, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_fwd_txfm_quant_device(const int32_t* d_resid, const uint8_t* d_tx_types, int32_t n, int32_t tx_size,
                             const mt_quant* quant, const uint8_t* d_qm_row, int32_t* d_levels, float* d_targets,
                             void* stream) {
  if (!quant || n < 0) return MT_ERR_INVALID_INPUT;
  if (tx_size != 8) return MT_ERR_UNSUPPORTED;
  if (n == 0) return MT_OK;
  cudaError_t e = mth::launch_fwd8(d_resid, d_tx_types, n, *quant, d_qm_row, d_levels, d_targets, as_stream(stream));
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_inv_txfm_dequant_device(const int32_t* d_levels, const uint8_t* d_tx_types, int32_t n, int32_t tx_size,
                               const mt_quant* quant, const uint8_t* d_qm_row, int32_t* d_resid, void* stream) {
  if (!quant || n < 0) return MT_ERR_INVALID_INPUT;
  if (tx_size != 8) return MT_ERR_UNSUPPORTED;
  if (n == 0) return MT_OK;
  cudaError_t e = mth::launch_inv8(d_levels, d_tx_types, n, *quant, d_qm_row, d_resid, as_stream(stream));
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_trellis_optimize_device(int32_t* d_levels, const float* d_targets, int32_t n, int32_t tx_size, float dc_q,
                               float ac_q, float lambda0, void* stream) {
  if (n < 0) return MT_ERR_INVALID_INPUT;
  if (tx_size != 8) return MT_ERR_UNSUPPORTED;
  if (n == 0 || lambda0 <= 0.0f) return MT_OK;
  cudaError_t e =
      mth::launch_trellis8(d_levels, d_targets, n, dc_q, ac_q, scaled_trellis_lambda(dc_q, lambda0), as_stream(stream));
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_intra_predict_device(const uint16_t* d_recon, const mt_chain_params* prm, const mt_candidate* d_cands, int32_t n,
                            int32_t* d_pred_out, void* stream) {
  if (!prm || n < 0) return MT_ERR_INVALID_INPUT;
  if (prm->tx_size != 8 || prm->bd != 8) return MT_ERR_UNSUPPORTED;
  if (n == 0) return MT_OK;
  cudaError_t e = mth::launch_pred8(d_recon, *prm, d_cands, n, d_pred_out, as_stream(stream));
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"
