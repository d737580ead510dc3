// Oracle coefficient coders (test infrastructure only): the adaptive square
// 2-D coefficient coders of src/coeffs.rs restated as token writers --
// encode_golomb :34-44, get_lo_ctx_2d :46-60, eob_and_cul :62-69,
// encode_hi_tok :71-84, encode_dc_tail :87-106, encode_tx8_coeffs_adapt
// :583-705, encode_tx16_coeffs_adapt / tx16_coeffs_tail :707-845,
// encode_4x4_chroma_coeffs :2310-2412, encode_tx4_luma_coeffs_adapt :2414-2520 --
// with the tokens of src/odec.rs:96-108 (adaptive symbol: slot << 8 | s; bool:
// 1 << 30 | f << 1 | v).
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "../include/maroontree_b200.h"
#include "../maroontree_b200/csrc/av1_tables.h"
#include "oracle.h"

namespace {

using EmitSlots = or_emit_slots;

struct Toks {
  std::vector<uint32_t> v;
  void symbol(int32_t slot, uint32_t s) { v.push_back(((uint32_t)slot << 8) | s); }
  void boolean(bool b) { v.push_back((1u << 30) | (16384u << 1) | (b ? 1u : 0u)); }
};

const uint8_t kScan4[16] = {0, 4, 1, 2, 5, 8, 12, 9, 6, 3, 7, 10, 13, 14, 11, 15};
const uint32_t kLoCtxOff[5][5] = {
    {0, 1, 6, 6, 21}, {1, 6, 6, 21, 21}, {6, 6, 21, 21, 21}, {6, 21, 21, 21, 21}, {21, 21, 21, 21, 21}};

uint32_t scan(int n, int i) {
  if (n == 4) return kScan4[i];
  if (n == 8) return MT_SCAN_8X8[i];
  return MT_SCAN_16X16[i];
}

void encode_golomb(Toks& t, uint32_t v) {
  const uint32_t x = v + 1;
  int length = 0;
  while ((x >> length) != 0) ++length;
  for (int i = 0; i < length - 1; ++i) t.boolean(false);
  for (int i = length - 1; i >= 0; --i) t.boolean(((x >> i) & 1) == 1);
}

void encode_hi_tok(Toks& t, uint32_t m, int32_t br_slot) {
  const int32_t total_br = (int32_t)m - 3 < 12 ? (int32_t)m - 3 : 12;  // NUM_BASE_LEVELS + 1, COEFF_BASE_RANGE
  int32_t coded = 0;
  for (int k = 0; k < 12 / 3; ++k) {
    const int32_t s = total_br - coded < 3 ? total_br - coded : 3;
    t.symbol(br_slot, (uint32_t)s);
    coded += s;
    if (s < 3) break;
  }
}

uint8_t level_byte(uint32_t m) {
  if (m == 0) return 0;
  if (m <= 2) return (uint8_t)(m * 0x41);
  return (uint8_t)((m < 15 ? m : 15) + (3 << 6));
}

// One coder, the four square sizes: class cls, plane pl (the reference's
// functions differ only in the size-dependent tables they name).
uint8_t encode_square(Toks& t, const EmitSlots& S, const int32_t* cf, int n, bool chroma, int skip_ctx, int dcs_ctx,
                      int y_mode, int txtp, bool code_txtp) {
  const int cls = n == 4 ? 0 : (n == 8 ? 1 : 2);
  const int pl = chroma ? 1 : 0;
  const int area = n * n;
  int eob = -1;
  for (int i = 0; i < area; ++i)
    if (cf[scan(n, i)] != 0) eob = i;
  if (eob < 0) {
    t.symbol(S.txb_skip[cls] + skip_ctx, 1);
    return 0x40;
  }
  uint32_t cul = 0;
  for (int i = 0; i <= eob; ++i) cul += (uint32_t)abs(cf[scan(n, i)]);
  t.symbol(S.txb_skip[cls] + skip_ctx, 0);
  if (!chroma && code_txtp) t.symbol((cls == 0 ? S.txtp4 : cls == 1 ? S.txtp8 : S.txtp16) + y_mode, (uint32_t)txtp);
  const uint8_t dc_sign_bits = cf[0] == 0 ? (1 << 6) : (cf[0] < 0 ? 0 : (2 << 6));
  const uint8_t res_ctx = (uint8_t)((cul < 63 ? cul : 63) | dc_sign_bits);
  // eob_pt CDFs in the frame set: 16c 16l 32c 32l 64l 16l1d 64l1d 128l1d 64c 256l 256c
  const int32_t eob_bin_cdf = S.eob_bin + (n == 4 ? (chroma ? 0 : 1) : n == 8 ? (chroma ? 8 : 4) : (chroma ? 10 : 9));
  if (eob == 0) {  // encode_dc_tail
    t.symbol(eob_bin_cdf, 0);
    const uint32_t m = (uint32_t)abs(cf[0]);
    const uint32_t base = m < 3 ? m : 3;
    t.symbol(S.eob_base[cls][pl] + 0, base - 1);
    if (base == 3) encode_hi_tok(t, m, S.br_tok[cls][pl] + 0);
    t.symbol(S.dc_sign[pl] + dcs_ctx, cf[0] < 0 ? 1 : 0);
    if (m >= 15) encode_golomb(t, m - 15);
    return res_ctx;
  }
  int eob_bin = eob;
  if (eob >= 2) {
    eob_bin = 0;
    while ((1u << eob_bin) <= (uint32_t)eob) ++eob_bin;  // 32 - leading_zeros(eob)
  }
  t.symbol(eob_bin_cdf, (uint32_t)eob_bin);
  if (eob_bin > 1) {
    const int nbits = eob_bin - 2;
    t.symbol(S.eob_hi[cls][pl] + eob_bin, (uint32_t)((eob >> nbits) & 1));
    for (int b = nbits - 1; b >= 0; --b) t.boolean(((eob >> b) & 1) == 1);
  }
  std::vector<uint8_t> levels(n == 16 ? 320 : 80, 0);
  const int ctx_e = 1 + (eob > area / 8 ? 1 : 0) + (eob > area / 4 ? 1 : 0);
  {
    const uint32_t rc = scan(n, eob);
    const uint32_t ex = rc / n, ey = rc % n;
    const uint32_t m = (uint32_t)abs(cf[rc]);
    const uint32_t eob_tok = (m < 3 ? m : 3) - 1;
    t.symbol(S.eob_base[cls][pl] + ctx_e, eob_tok);
    if (eob_tok == 2) encode_hi_tok(t, m, S.br_tok[cls][pl] + (((ex | ey) > 1) ? 14 : 7));
    levels[ex * n + ey] = level_byte(m);
  }
  for (int i = eob - 1; i >= 1; --i) {
    const uint32_t rc = scan(n, i);
    const uint32_t x = rc / n, y = rc % n;
    auto g = [&](uint32_t dx, uint32_t dy) { return (uint32_t)levels[(x + dx) * n + (y + dy)]; };
    const uint32_t hi_mag = g(0, 1) + g(1, 0) + g(1, 1);
    const uint32_t mag = hi_mag + g(0, 2) + g(2, 0);
    const uint32_t ctx = kLoCtxOff[y < 4 ? y : 4][x < 4 ? x : 4] + (mag > 512 ? 4 : (mag + 64) >> 7);
    const uint32_t m = (uint32_t)abs(cf[rc]);
    const uint32_t tok = m < 3 ? m : 3;
    t.symbol(S.base_tok[cls][pl] + (int32_t)ctx, tok);
    if (tok == 3) {
      const uint32_t mg = hi_mag & 63;
      const uint32_t bc = (((y | x) > 1) ? 14 : 7) + (mg > 12 ? 6 : (mg + 1) >> 1);
      encode_hi_tok(t, m, S.br_tok[cls][pl] + (int32_t)bc);
    }
    levels[x * n + y] = level_byte(m);
  }
  const uint32_t dm = (uint32_t)abs(cf[0]);
  const uint32_t dc_tok = dm < 3 ? dm : 3;
  t.symbol(S.base_tok[cls][pl] + 0, dc_tok);
  if (dc_tok == 3) {
    const uint32_t mg = ((uint32_t)levels[1] + (uint32_t)levels[n] + (uint32_t)levels[n + 1]) & 63;
    encode_hi_tok(t, dm, S.br_tok[cls][pl] + (int32_t)(mg > 12 ? 6 : (mg + 1) >> 1));
  }
  if (cf[0] != 0) {
    t.symbol(S.dc_sign[pl] + dcs_ctx, cf[0] < 0 ? 1 : 0);
    if (dm >= 15) encode_golomb(t, dm - 15);
  }
  for (int i = 1; i <= eob; ++i) {
    const int32_t c = cf[scan(n, i)];
    if (c != 0) {
      t.boolean(c < 0);
      if ((uint32_t)abs(c) >= 15) encode_golomb(t, (uint32_t)abs(c) - 15);
    }
  }
  return res_ctx;
}

// encode_tx4_coeffs_1d / encode_tx8_coeffs_1d (src/coeffs.rs:264-420, :109-262).
uint8_t encode_1d(Toks& t, const EmitSlots& S, const int32_t* cf, int n, bool vertical, int skip_ctx, int dcs_ctx,
                  int y_mode) {
  const int cls = n == 4 ? 0 : 1, pl = 0, sh = n == 4 ? 2 : 3;
  auto pos_rc = [&](int i) -> int {
    const int x = i & (n - 1), y = i >> sh;
    return vertical ? ((x << sh) | y) : i;
  };
  int eob = -1;
  for (int i = n * n - 1; i >= 0; --i)
    if (cf[pos_rc(i)] != 0) {
      eob = i;
      break;
    }
  if (eob < 0) {
    t.symbol(S.txb_skip[cls] + skip_ctx, 1);
    return 0x40;
  }
  uint32_t cul = 0;
  for (int i = 0; i <= eob; ++i) cul += (uint32_t)abs(cf[pos_rc(i)]);
  t.symbol(S.txb_skip[cls] + skip_ctx, 0);
  t.symbol((cls == 0 ? S.txtp4 : S.txtp8) + y_mode, vertical ? 2 : 3);
  const uint8_t dc_sign_bits = cf[0] == 0 ? (1 << 6) : (cf[0] < 0 ? 0 : (2 << 6));
  const uint8_t res_ctx = (uint8_t)((cul < 63 ? cul : 63) | dc_sign_bits);
  const int32_t eb = S.eob_bin + (cls == 0 ? 5 : 6);  // eob_bin_16_l1d, eob_bin_64_l1d
  if (eob == 0) {
    t.symbol(eb, 0);
    const uint32_t m = (uint32_t)abs(cf[0]);
    const uint32_t base = m < 3 ? m : 3;
    t.symbol(S.eob_base[cls][pl] + 0, base - 1);
    if (base == 3) encode_hi_tok(t, m, S.br_tok[cls][pl] + 0);
    t.symbol(S.dc_sign[pl] + dcs_ctx, cf[0] < 0 ? 1 : 0);
    if (m >= 15) encode_golomb(t, m - 15);
    return res_ctx;
  }
  int eob_bin = eob;
  if (eob >= 2) {
    eob_bin = 0;
    while ((1u << eob_bin) <= (uint32_t)eob) ++eob_bin;
  }
  t.symbol(eb, (uint32_t)eob_bin);
  if (eob_bin > 1) {
    const int nbits = eob_bin - 2;
    t.symbol(S.eob_hi[cls][pl] + eob_bin, (uint32_t)((eob >> nbits) & 1));
    for (int b = nbits - 1; b >= 0; --b) t.boolean(((eob >> b) & 1) == 1);
  }
  uint8_t levels[16 * 10] = {};
  auto lvl = [&](int x, int y) { return (uint32_t)levels[x * 16 + y]; };
  auto lo_ctx_1d = [&](int x, int y, uint32_t* hi_mag) {
    uint32_t mag = lvl(x, y + 1) + lvl(x + 1, y) + lvl(x, y + 2);
    *hi_mag = mag;
    mag += lvl(x, y + 3) + lvl(x, y + 4);
    const uint32_t offset = 26 + (y > 1 ? 10 : (uint32_t)y * 5);
    return offset + (mag > 512 ? 4 : (mag + 64) >> 7);
  };
  const int ctx_e = 1 + (eob > (n * n) / 8 ? 1 : 0) + (eob > (n * n) / 4 ? 1 : 0);
  {
    const int x = eob & (n - 1), y = eob >> sh;
    const uint32_t m = (uint32_t)abs(cf[pos_rc(eob)]);
    const uint32_t eob_tok = (m < 3 ? m : 3) - 1;
    t.symbol(S.eob_base[cls][pl] + ctx_e, eob_tok);
    if (eob_tok == 2) encode_hi_tok(t, m, S.br_tok[cls][pl] + (y != 0 ? 14 : 7));
    levels[x * 16 + y] = level_byte(m);
  }
  for (int i = eob - 1; i >= 1; --i) {
    const int x = i & (n - 1), y = i >> sh;
    uint32_t hi_mag;
    const uint32_t ctx = lo_ctx_1d(x, y, &hi_mag);
    const uint32_t m = (uint32_t)abs(cf[pos_rc(i)]);
    const uint32_t tok = m < 3 ? m : 3;
    t.symbol(S.base_tok[cls][pl] + (int32_t)ctx, tok);
    if (tok == 3) {
      const uint32_t mg = hi_mag & 63;
      encode_hi_tok(t, m, S.br_tok[cls][pl] + (int32_t)((y != 0 ? 14 : 7) + (mg > 12 ? 6 : (mg + 1) >> 1)));
    }
    levels[x * 16 + y] = level_byte(m);
  }
  uint32_t dc_hi;
  const uint32_t dc_ctx = lo_ctx_1d(0, 0, &dc_hi);
  const uint32_t dm = (uint32_t)abs(cf[0]);
  const uint32_t dc_tok = dm < 3 ? dm : 3;
  t.symbol(S.base_tok[cls][pl] + (int32_t)dc_ctx, dc_tok);
  if (dc_tok == 3) {
    const uint32_t mg = dc_hi & 63;
    encode_hi_tok(t, dm, S.br_tok[cls][pl] + (int32_t)(mg > 12 ? 6 : (mg + 1) >> 1));
  }
  if (cf[0] != 0) {
    t.symbol(S.dc_sign[pl] + dcs_ctx, cf[0] < 0 ? 1 : 0);
    if (dm >= 15) encode_golomb(t, dm - 15);
  }
  for (int i = 1; i <= eob; ++i) {
    const int32_t c = cf[pos_rc(i)];
    if (c != 0) {
      t.boolean(c < 0);
      if ((uint32_t)abs(c) >= 15) encode_golomb(t, (uint32_t)abs(c) - 15);
    }
  }
  return res_ctx;
}

}  // namespace

extern "C" int or_emit_coeffs(const int32_t* levels, const mt_coef_block* blocks, int32_t n, const EmitSlots* S,
                              uint32_t* tokens, size_t cap, uint32_t* offsets, uint8_t* res_ctx) {
  size_t at = 0;
  for (int32_t i = 0; i < n; ++i) {
    Toks t;
    const mt_coef_block& b = blocks[i];
    if (b.tx_class)
      res_ctx[i] = encode_1d(t, *S, levels + b.cf_offset, 1 << b.log2n, b.tx_class == 1, b.skip_ctx, b.dcs_ctx,
                             b.y_mode);
    else
      res_ctx[i] = encode_square(t, *S, levels + b.cf_offset, 1 << b.log2n, b.plane != 0, b.skip_ctx, b.dcs_ctx,
                                 b.y_mode, b.txtp, b.code_txtp != 0);
    offsets[i] = (uint32_t)at;
    if (at + t.v.size() > cap) return -1;
    memcpy(tokens + at, t.v.data(), t.v.size() * 4);
    at += t.v.size();
  }
  offsets[n] = (uint32_t)at;
  return 0;
}
