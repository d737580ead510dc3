// Default decision-CDF snapshot: the coefficient slices of Cdfs::new(qctx)
// (src/coder/cdfs.rs:401-629) and the coefficient q context qcat
// (src/coef_q.rs:31-41).  Host code only: the slices are handed to the
// batched kernels as their mt_coef_cdfs input.
#include <stdint.h>
#include <string.h>

#include "../../include/maroontree_b200.h"
#include "av1_cdfs.h"

namespace {

// AV1 inverse-CDF entry of a stored cumulative value (src/tables.rs:31-35).
inline uint16_t inv(uint16_t v) { return (uint16_t)(32768 - v); }

// Fills `n` symbols' CDF row (n - 1 stored values, then the terminal 0).
void row(uint16_t* dst, const uint16_t* vals, int nvals) {
  for (int k = 0; k < nvals; ++k) dst[k] = inv(vals[k]);
  dst[nvals] = 0;
}

int log2i(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}

struct ClassTables {
  const uint16_t* skip;      // [4][13]
  const uint16_t* base;      // [4][rows][3]
  int base_rows;
  const uint16_t* br;        // [4][21][3], NULL for TX_64X64 (no chroma, luma unused)
  const uint16_t* eob_base;  // [4][4][2]
  const uint16_t* eob_hi;    // [4][11]
};

// Tables of one (class, plane); plane 1 of class 4 does not exist.
bool class_tables(int cls, int plane, ClassTables* t) {
  const bool c = plane != 0;
  switch (cls) {
    case 0:
      *t = {MT_CDF_SKIP_TX4, c ? MT_CDF_BASE_TOK_TX4_CHROMA_Q : MT_CDF_BASE_TOK_TX4_LUMA_Q, 41,
            c ? MT_CDF_BR_TOK_TX4_CHROMA_Q : MT_CDF_BR_TOK_TX4_LUMA_Q,
            c ? MT_CDF_EOB_BASE_TX4_CHROMA_Q : MT_CDF_EOB_BASE_TX4_LUMA_Q,
            c ? MT_CDF_EOB_HI_TX4_CHROMA : MT_CDF_EOB_HI_TX4_LUMA};
      return true;
    case 1:
      *t = {MT_CDF_SKIP_TX8, c ? MT_CDF_BASE_TOK_TX8_CHROMA_Q : MT_CDF_BASE_TOK_TX8_LUMA_Q, 41,
            c ? MT_CDF_BR_TOK_TX8_CHROMA_Q : MT_CDF_BR_TOK_TX8_LUMA_Q,
            c ? MT_CDF_EOB_BASE_TX8_CHROMA_Q : MT_CDF_EOB_BASE_TX8_LUMA_Q,
            c ? MT_CDF_EOB_HI_TX8_CHROMA : MT_CDF_EOB_HI_TX8_LUMA};
      return true;
    case 2:
      *t = {MT_CDF_SKIP_TX16, c ? MT_CDF_BASE_TOK_TX16_CHROMA_Q : MT_CDF_BASE_TOK_TX16_LUMA_Q, 42,
            c ? MT_CDF_BR_TOK_TX16_CHROMA_Q : MT_CDF_BR_TOK_TX16_LUMA_Q,
            c ? MT_CDF_EOB_BASE_TX16_CHROMA_Q : MT_CDF_EOB_BASE_TX16_LUMA_Q,
            c ? MT_CDF_EOB_HI_TX16_CHROMA : MT_CDF_EOB_HI_TX16_LUMA};
      return true;
    case 3:
      *t = {MT_CDF_SKIP_TX32, c ? MT_CDF_BASE_TOK_TX32_CHROMA_Q : MT_CDF_BASE_TOK_TX32_LUMA_Q, 42,
            c ? MT_CDF_BR_TOK_TX32_CHROMA_Q : MT_CDF_BR_TOK_TX32_LUMA_Q,
            c ? MT_CDF_EOB_BASE_TX32_CHROMA_Q : MT_CDF_EOB_BASE_TX32_LUMA_Q,
            c ? MT_CDF_EOB_HI_TX32_CHROMA : MT_CDF_EOB_HI_TX32_LUMA};
      return true;
    case 4:
      if (c) return false;
      // The br_tok ladder has four classes (src/coder/cdfs.rs:451-468); the
      // 64-point transforms are coded through the 32-point class's.
      *t = {MT_CDF_SKIP_TX64, MT_CDF_BASE_TOK_TX64_LUMA_Q, 42, MT_CDF_BR_TOK_TX32_LUMA_Q,
            MT_CDF_EOB_BASE_TX64_LUMA_Q, MT_CDF_EOB_HI_TX64_LUMA};
      return true;
    default:
      return false;
  }
}

// eob_pt CDF of a transform with `area` coefficients (capped at 1024), and the
// 1-D classes' form where the reference keeps one (luma 16 / 64 / 128).
const uint16_t* eob_bin_table(int area, int plane, int* nvals) {
  const bool c = plane != 0;
  switch (area) {
    case 16: *nvals = 4; return c ? MT_CDF_EOB_BIN_16_CHROMA : MT_CDF_EOB_BIN_16_LUMA;
    case 32: *nvals = 5; return c ? MT_CDF_EOB_BIN_32_CHROMA : MT_CDF_EOB_BIN_32_LUMA;
    case 64: *nvals = 6; return c ? MT_CDF_EOB_BIN_64_CHROMA : MT_CDF_EOB_BIN_64_LUMA;
    case 128: *nvals = 7; return c ? MT_CDF_EOB_BIN_128_CHROMA : MT_CDF_EOB_BIN_128_LUMA;
    case 256: *nvals = 8; return c ? MT_CDF_EOB_BIN_256_CHROMA : MT_CDF_EOB_BIN_256_LUMA;
    case 512: *nvals = 9; return c ? MT_CDF_EOB_BIN_512_CHROMA : MT_CDF_EOB_BIN_512_LUMA;
    case 1024: *nvals = 10; return c ? MT_CDF_EOB_BIN_1024_CHROMA : MT_CDF_EOB_BIN_1024_LUMA;
    default: *nvals = 0; return nullptr;
  }
}

const uint16_t* eob_bin_1d_table(int area, int plane, int* nvals) {
  if (plane != 0) return nullptr;
  switch (area) {
    case 16: *nvals = 4; return MT_CDF_EOB_BIN_16_LUMA_1D;
    case 64: *nvals = 6; return MT_CDF_EOB_BIN_64_LUMA_1D;
    case 128: *nvals = 7; return MT_CDF_EOB_BIN_128_LUMA_1D;
    default: return nullptr;
  }
}

}  // namespace

extern "C" int mt_qcat(int32_t base_q_idx) {
  if (base_q_idx <= 20) return 0;
  if (base_q_idx <= 60) return 1;
  if (base_q_idx <= 120) return 2;
  return 3;
}

extern "C" int mt_coef_cdfs_default(int32_t qctx, int32_t tx_w, int32_t tx_h, int32_t plane, mt_coef_cdfs* out) {
  if (!out || qctx < 0 || qctx > 3 || (plane != 0 && plane != 1)) return MT_ERR_INVALID_INPUT;
  const bool pow2 = tx_w >= 4 && tx_h >= 4 && tx_w <= 64 && tx_h <= 64 && !(tx_w & (tx_w - 1)) && !(tx_h & (tx_h - 1));
  if (!pow2) return MT_ERR_INVALID_INPUT;
  const int lw = log2i(tx_w) - 2, lh = log2i(tx_h) - 2;
  const int sqr = lw < lh ? lw : lh, sqr_up = lw < lh ? lh : lw;
  if (sqr_up - sqr > 2) return MT_ERR_INVALID_INPUT;  // no 1:8 transforms in AV1
  // AV1 txSzCtx: the mean of the square sizes below and above (1:2 and 1:4
  // rectangles take the class the reference's emitters use, e.g. 4x8 -> TX_8X8
  // at src/coeffs.rs:1054-1100, 16x8 -> TX_16X16 at :1896-1925).
  const int cls = (sqr + sqr_up + 1) >> 1;
  ClassTables t;
  if (!class_tables(cls, plane, &t)) return MT_ERR_UNSUPPORTED;
  memset(out, 0, sizeof(*out));
  for (int i = 0; i < 13; ++i) row(out->txb_skip[i], &t.skip[qctx * 13 + i], 1);
  for (int i = 0; i < t.base_rows; ++i) row(out->base_tok[i], &t.base[(qctx * t.base_rows + i) * 3], 3);
  for (int i = 0; i < 21; ++i) row(out->br_tok[i], &t.br[(qctx * 21 + i) * 3], 3);
  for (int i = 0; i < 4; ++i) row(out->eob_base[i], &t.eob_base[(qctx * 4 + i) * 2], 2);
  for (int i = 0; i < 11; ++i) row(out->eob_hi[i], &t.eob_hi[qctx * 11 + i], 1);
  for (int i = 0; i < 3; ++i) row(out->dc_sign[i], &MT_CDF_DC_SIGN_Q[(qctx * 2 + plane) * 3 + i], 1);
  int area = tx_w * tx_h;
  if (area > 1024) area = 1024;  // 64-point transforms code their 32x32 low band
  int nv = 0;
  const uint16_t* eb = eob_bin_table(area, plane, &nv);
  row(out->eob_bin, &eb[qctx * nv], nv);
  const uint16_t* e1 = eob_bin_1d_table(area, plane, &nv);
  if (e1) row(out->eob_bin_1d, &e1[qctx * nv], nv);
  // Luma signals the intra tx type from the set of the square size below
  // (src/coeffs.rs:1908 uses the TX_8X8 table for 16x8): TX_4X4 and TX_8X8 take
  // the 7-type INTRA1 set, TX_16X16 the 5-type INTRA2 set; a transform with a
  // 32- or 64-point side codes no tx type (AV1's DCT-only intra set).
  if (plane == 0 && sqr_up <= 2) {
    if (sqr == 0 || sqr == 1) {
      const uint16_t* tp = sqr == 0 ? MT_CDF_TXTP_INTRA1_TX4 : MT_CDF_TXTP_INTRA1_TX8;
      for (int m = 0; m < 13; ++m) row(out->txtp[m], &tp[m * 6], 6);
    } else if (sqr == 2) {
      for (int m = 0; m < 13; ++m) row(out->txtp[m], &MT_CDF_TXTP_INTRA2_TX16[m * 4], 4);
    }
  }
  return MT_OK;
}

// The mode CDFs uv_mode_bits reads (src/coder/lossy_state.rs:1302-1349) from
// the decision snapshot: uv_mode with CfL allowed per y mode, angle_delta per
// directional mode, cfl_sign, cfl_alpha per context.
extern "C" int mt_uv_mode_cdfs_default(mt_uv_mode_cdfs* out) {
  if (!out) return MT_ERR_INVALID_INPUT;
  memset(out, 0, sizeof(*out));
  for (int m = 0; m < 13; ++m) row(out->uv_mode[m], &MT_CDF_UV_MODE_CFL_CDF[m * 13], 13);
  for (int m = 0; m < 8; ++m) row(out->angle_delta[m], &MT_CDF_ANGLE_DELTA_CDF[m * 6], 6);
  row(out->cfl_sign, MT_CDF_CFL_SIGN_CDF, 7);
  for (int c = 0; c < 6; ++c) row(out->cfl_alpha[c], &MT_CDF_CFL_ALPHA_CDF[c * 15], 15);
  return MT_OK;
}
