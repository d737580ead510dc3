// Oracle (test infrastructure only): scalar restatement of the reference's
// luma candidate chain.  See oracle.h for the arithmetic conventions.  Every
// function names the reference file:line it restates (awxkee/maroontree).
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <thread>
#include <algorithm>
#include <vector>

#include "../maroontree_b200/csrc/av1_tables.h"

namespace {

inline int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }
inline int32_t iabs(int32_t v) { return v < 0 ? -v : v; }
inline uint32_t uabs(int32_t v) { return v < 0 ? (uint32_t)0 - (uint32_t)v : (uint32_t)v; }

// ---------------------------------------------------------------- quant.rs
// quant.rs:351-373 Quant::new_with_qm, :393-418 new_chroma_with_delta_qm,
// :239-247 itx_clips (bd <= 8).
void fill_quant(int32_t dc, int32_t ac, int32_t qm_level, int32_t chroma, int32_t qidx, mt_quant* q) {
  q->dc_q = dc;
  q->ac_q = ac;
  q->q_mult_dc = (int32_t)llround(65536.0 / (double)dc);
  q->q_mult_ac = (int32_t)llround(65536.0 / (double)ac);
  q->rmin = -32768;
  q->rmax = 32767;
  q->cmin = -32768;
  q->cmax = 32767;
  q->cf_max = 32767;
  q->qm_level = qm_level > 15 ? 15 : qm_level;
  q->qm_chroma = chroma;
  q->qidx = qidx;
}

// quant.rs:58-77 qm_offset.
int qm_offset(int w, int h) {
  if (w == 4 && h == 4) return 0;
  if (w == 8 && h == 8) return 16;
  if (w == 16 && h == 16) return 80;
  if (w == 32 && h == 32) return 336;
  return -1;
}

// ------------------------------------------------------------------ dct.rs
// dct.rs:60-67 mul_q16 (rounding).
inline int32_t mul_q16(int32_t d, int32_t c) { return (int32_t)(((int64_t)d * (int64_t)c + 32768) >> 16); }
// dct.rs:70-79 quant_q16 (half-step dead zone).
inline int32_t quant_q16(int32_t d, int32_t c) {
  int64_t prod = (int64_t)d * (int64_t)c;
  uint64_t mag = prod < 0 ? (uint64_t)0 - (uint64_t)prod : (uint64_t)prod;
  if (mag < 32768) return 0;
  int32_t lvl = (int32_t)((mag + 32768) >> 16);
  return prod >= 0 ? lvl : -lvl;
}
const int32_t WC4_0 = 35468, WC4_1 = 85627;
const int32_t WC8[4] = {33410, 39410, 58981, 167963};
const int32_t SQRT2_Q16 = 92682;
inline int32_t fmla_sqrt2(int32_t a, int32_t b) { return mul_q16(a, SQRT2_Q16) + b; }

// dct.rs:171-191 dct1d_4_i32.
void dct1d_4(int32_t* b) {
  int32_t t0 = b[0] + b[3], t1 = b[1] + b[2];
  int32_t e0 = t0 + t1, e1 = t0 - t1;
  int32_t t2 = mul_q16(b[0] - b[3], WC4_0);
  int32_t t3 = mul_q16(b[1] - b[2], WC4_1);
  int32_t o0 = t2 + t3, o1 = t2 - t3;
  o0 = fmla_sqrt2(o0, o1);
  b[0] = e0;
  b[2] = e1;
  b[1] = o0;
  b[3] = o1;
}
// dct.rs:194-219 dct1d_8_i32.
void dct1d_8(int32_t* b) {
  int32_t t[8];
  for (int i = 0; i < 4; i++) t[i] = b[i] + b[7 - i];
  dct1d_4(t);
  for (int i = 0; i < 4; i++) t[4 + i] = mul_q16(b[i] - b[7 - i], WC8[i]);
  dct1d_4(t + 4);
  t[4] = fmla_sqrt2(t[4], t[5]);
  t[5] += t[6];
  t[6] += t[7];
  for (int i = 0; i < 4; i++) {
    b[2 * i] = t[i];
    b[2 * i + 1] = t[4 + i];
  }
}
// dct.rs:304-326 ADST8_FWD_Q12 / fwd_adst8_1d.
const int32_t ADST8_FWD[8][8] = {
    {567, 1682, 2730, 3675, 4477, 5109, 5544, 5766},
    {1682, 4480, 5766, 5109, 2732, -569, -3675, -5545},
    {2732, 5766, 3675, -1682, -5544, -4479, 569, 5109},
    {3675, 5108, -1681, -5764, -569, 5542, 2732, -4479},
    {4479, 2732, -5542, -569, 5764, -1681, -5108, 3675},
    {5109, -569, -4479, 5544, -1682, -3675, 5766, -2732},
    {5545, -3675, 569, 2732, -5109, 5766, -4480, 1682},
    {5766, -5544, 5109, -4477, 3675, -2730, 1682, -567},
};
void fwd_adst8(int32_t* b) {
  int32_t o[8];
  for (int i = 0; i < 8; i++) {
    int64_t acc = 0;
    for (int j = 0; j < 8; j++) acc += (int64_t)ADST8_FWD[i][j] * (int64_t)b[j];
    o[i] = (int32_t)((acc + 2048) >> 12);
  }
  memcpy(b, o, sizeof(o));
}

// dct.rs:1368-1383 ADST4_FWD_Q12 / fwd_adst4_1d.
const int32_t ADST4_FWD[4][4] = {
    {1868, 3510, 4730, 5379},
    {4730, 4730, 0, -4730},
    {5379, -1868, -4730, 3510},
    {3510, -5379, 4730, -1868},
};
void fwd_adst4(int32_t* b) {
  int32_t o[4];
  for (int i = 0; i < 4; i++) {
    int64_t acc = 0;
    for (int j = 0; j < 4; j++) acc += (int64_t)ADST4_FWD[i][j] * (int64_t)b[j];
    o[i] = (int32_t)((acc + 2048) >> 12);
  }
  memcpy(b, o, sizeof(o));
}

// dct.rs:1194-1205 store_quant_target_scalar (AVX2 twin avx/dct.rs:143-166 has the
// same float order: (c * m) * 2^-16).
inline void store_quant_target(int32_t* cf, float* tf, int idx, int32_t coeff, int32_t mdc, int32_t mac) {
  int32_t m = idx == 0 ? mdc : mac;
  cf[idx] = quant_q16(coeff, m);
  tf[idx] = (float)coeff * (float)m * (1.0f / 65536.0f);
}
// dct.rs:373-389 quant_fullstep.
inline void quant_fullstep(int32_t* cf, float* tf, int idx, int32_t coeff, int32_t m) {
  int64_t prod = (int64_t)coeff * (int64_t)m;
  tf[idx] = (float)prod * (1.0f / 65536.0f);
  uint64_t mag = prod < 0 ? (uint64_t)0 - (uint64_t)prod : (uint64_t)prod;
  if (mag < 65536) {
    cf[idx] = 0;
  } else {
    int32_t l = (int32_t)((mag + 32768) >> 16);
    cf[idx] = prod >= 0 ? l : -l;
  }
}

// dct.rs:93-104 FORWARD_QM_SCALES.
float fwd_qm_scale(int iwt) { return (float)((1024 + iwt / 2) / iwt) / 32.0f; }

// avx/qmatrix.rs:34-71 apply_qmatrix_avx2: the pinned x86 path.  Chunks of 8
// scale the target and round half away from zero via truncate + fraction test;
// the tail (len % 8, never reached for square sizes >= 4x4 since 16 % 8 == 0)
// would use the scalar dct.rs:111-129 form.
void apply_qmatrix(int32_t* levels, float* targets, const uint8_t* iw, int n) {
  for (int i = 0; i < n; i++) {
    float w = targets[i] * fwd_qm_scale(iw[i]);
    targets[i] = w;
    float tr = truncf(w);
    float frac = fabsf(w - tr);
    float step = frac >= 0.5f ? (w < 0.0f || (w == 0.0f && signbit(w)) ? -1.0f : 1.0f) : 0.0f;
    levels[i] = (int32_t)(tr + step);
  }
}

// dct.rs:279-301 dct8x8_quant_t_direct and the ADST variants dct.rs:1222-1293:
// columns first (1-D kernel `col`), then rows (`row`), levels at u*8 + r.
void fwd_2d_8x8(const int32_t* in, void (*colf)(int32_t*), void (*rowf)(int32_t*), int32_t mdc,
                int32_t mac, int32_t* cf, float* tf) {
  int32_t tmp[64];
  for (int x = 0; x < 8; x++) {
    int32_t col[8];
    for (int r = 0; r < 8; r++) col[r] = in[r * 8 + x];
    colf(col);
    for (int r = 0; r < 8; r++) tmp[r * 8 + x] = col[r];
  }
  for (int r = 0; r < 8; r++) {
    int32_t row[8];
    for (int u = 0; u < 8; u++) row[u] = tmp[r * 8 + u];
    rowf(row);
    for (int u = 0; u < 8; u++) store_quant_target(cf, tf, u * 8 + r, row[u], mdc, mac);
  }
}

// dct.rs:328-370 f1ddct8x8_quant_t_direct (V_DCT vertical / H_DCT).
void fwd_1d_8x8(const int32_t* in, bool vertical, int32_t mdc, int32_t mac, int32_t* cf, float* tf) {
  int32_t f[64];
  if (vertical) {
    for (int x = 0; x < 8; x++) {
      int32_t col[8];
      for (int y = 0; y < 8; y++) col[y] = in[y * 8 + x];
      dct1d_8(col);
      for (int y = 0; y < 8; y++) f[y * 8 + x] = col[y] * 2;
    }
  } else {
    for (int y = 0; y < 8; y++) {
      int32_t row[8];
      for (int x = 0; x < 8; x++) row[x] = in[y * 8 + x];
      dct1d_8(row);
      for (int x = 0; x < 8; x++) f[y * 8 + x] = row[x] * 2;
    }
  }
  for (int y = 0; y < 8; y++)
    for (int x = 0; x < 8; x++) {
      int rc = y + x * 8;
      quant_fullstep(cf, tf, rc, f[y * 8 + x], rc == 0 ? mdc : mac);
    }
}

// dct.rs:3076-3100 dct4x4_quant_t_direct and dct.rs:1398-1470 adst4x4 /
// adstdct4x4 / dctadst4x4 (AVX2 twins avx/dct.rs:717-793, :841-843 run the
// same columns-then-rows order; their 4x4 normalisation is Q16 unity):
// columns first, then rows, levels at u*4 + r.
void fwd_2d_4x4(const int32_t* in, void (*colf)(int32_t*), void (*rowf)(int32_t*), int32_t mdc, int32_t mac,
                int32_t* cf, float* tf) {
  int32_t tmp[16];
  for (int x = 0; x < 4; x++) {
    int32_t col[4];
    for (int r = 0; r < 4; r++) col[r] = in[r * 4 + x];
    colf(col);
    for (int r = 0; r < 4; r++) tmp[r * 4 + x] = col[r];
  }
  for (int r = 0; r < 4; r++) {
    int32_t row[4];
    for (int u = 0; u < 4; u++) row[u] = tmp[r * 4 + u];
    rowf(row);
    for (int u = 0; u < 4; u++) store_quant_target(cf, tf, u * 4 + r, row[u], mdc, mac);
  }
}

// dct.rs:391-431 f1ddct4x4_quant_t_direct (V_DCT / H_DCT): the 1-D DCT x 2 sqrt2
// (AVX2 avx/dct.rs:933-934 folds it into one Q16 multiply by 185364, the same
// value), full-step quantisation, transposed storage.
void fwd_1d_4x4(const int32_t* in, bool vertical, int32_t mdc, int32_t mac, int32_t* cf, float* tf) {
  int32_t f[16];
  if (vertical) {
    for (int x = 0; x < 4; x++) {
      int32_t col[4];
      for (int y = 0; y < 4; y++) col[y] = in[y * 4 + x];
      dct1d_4(col);
      for (int y = 0; y < 4; y++) f[y * 4 + x] = mul_q16(col[y] * 2, SQRT2_Q16);
    }
  } else {
    for (int y = 0; y < 4; y++) {
      int32_t row[4];
      for (int x = 0; x < 4; x++) row[x] = in[y * 4 + x];
      dct1d_4(row);
      for (int x = 0; x < 4; x++) f[y * 4 + x] = mul_q16(row[x] * 2, SQRT2_Q16);
    }
  }
  for (int y = 0; y < 4; y++)
    for (int x = 0; x < 4; x++) {
      int rc = y + x * 4;
      quant_fullstep(cf, tf, rc, f[y * 4 + x], rc == 0 ? mdc : mac);
    }
}

// dct.rs:224-238 WC16: the odd-half weights of the 16-point forward DCT (Q16).
const int32_t WC16[8] = {32927, 34242, 37155, 42390, 51653, 69513, 112882, 334309};

// dct.rs:241-276 dct1d_16_i32: even/odd split, 8-point DCTs on both halves (the
// odd one after the WC16 weights), the odd-half running combine, interleave.
void dct1d_16(int32_t* b) {
  int32_t t[16];
  for (int i = 0; i < 8; i++) {
    t[i] = b[i] + b[15 - i];
    t[8 + i] = b[i] - b[15 - i];
  }
  dct1d_8(t);
  for (int i = 0; i < 8; i++) t[8 + i] = mul_q16(t[8 + i], WC16[i]);
  dct1d_8(t + 8);
  t[8] = fmla_sqrt2(t[8], t[9]);
  for (int i = 9; i < 15; i++) t[i] += t[i + 1];
  for (int i = 0; i < 8; i++) {
    b[2 * i] = t[i];
    b[2 * i + 1] = t[8 + i];
  }
}

// dct.rs:513-523 fwd_adst16_1d: the Q12 matrix ADST16_FWD_Q12 (i64 sums).
void fwd_adst16(int32_t* b) {
  int32_t o[16];
  for (int i = 0; i < 16; i++) {
    int64_t acc = 0;
    for (int j = 0; j < 16; j++) acc += (int64_t)MT_ADST16_FWD_Q12[i * 16 + j] * b[j];
    o[i] = (int32_t)((acc + 2048) >> 12);
  }
  for (int i = 0; i < 16; i++) b[i] = o[i];
}

// dct.rs:557-580 dct16x16_quant_t_direct, :1295-1392 adst16x16 / adstdct16x16 /
// dctadst16x16: columns, then rows, each output halved by mul_q16(x, 32768)
// before store_quant_target (the Q16 multipliers are the quantiser's own).
void fwd_2d_16x16(const int32_t* in, void (*colf)(int32_t*), void (*rowf)(int32_t*), int32_t mdc, int32_t mac,
                  int32_t* cf, float* tf) {
  int32_t tmp[256];
  for (int u = 0; u < 16; u++) {
    int32_t col[16];
    for (int i = 0; i < 16; i++) col[i] = in[i * 16 + u];
    colf(col);
    for (int v = 0; v < 16; v++) tmp[v * 16 + u] = col[v];
  }
  for (int v = 0; v < 16; v++) {
    int32_t row[16];
    for (int u = 0; u < 16; u++) row[u] = tmp[v * 16 + u];
    rowf(row);
    for (int u = 0; u < 16; u++) store_quant_target(cf, tf, u * 16 + v, mul_q16(row[u], 32768), mdc, mac);
  }
}

// dct.rs:589-631 WC32 (the odd-half weights of the 32-point forward DCT) and
// dct1d_32_i32: even/odd split, the 16-point DCT of both halves (the odd one
// after the WC32 weights), the odd-half running combine, interleave.
const int32_t WC32[16] = {32808, 33127, 33780, 34802, 36248,  38203,  40796,  44224,
                          48794, 55008, 63738, 76640, 97266, 134859, 223321, 667812};
void dct1d_32(int32_t* b) {
  int32_t t[32];
  for (int i = 0; i < 16; i++) {
    t[i] = b[i] + b[31 - i];
    t[16 + i] = b[i] - b[31 - i];
  }
  dct1d_16(t);
  for (int i = 0; i < 16; i++) t[16 + i] = mul_q16(t[16 + i], WC32[i]);
  dct1d_16(t + 16);
  t[16] = mul_q16(t[16], 92682) + t[17];  // fmla_sqrt2 (dct.rs:158-160)
  for (int i = 17; i < 31; i++) t[i] += t[i + 1];
  for (int i = 0; i < 16; i++) {
    b[2 * i] = t[i];
    b[2 * i + 1] = t[16 + i];
  }
}

// dct.rs:705-736 dct32x32_quant_t_direct: the residual shifted left by B = 6,
// columns then rows, each output (x * 16384 + 2^(15+B)) >> (16+B) in i64,
// quantised into the levels at u*32 + v.
void fwd_2d_32x32(const int32_t* in, int32_t mdc, int32_t mac, int32_t* cf, float* tf) {
  const int B = 6;
  std::vector<int32_t> tmp(1024);
  for (int u = 0; u < 32; u++) {
    int32_t col[32];
    for (int i = 0; i < 32; i++) col[i] = in[i * 32 + u] * (1 << B);
    dct1d_32(col);
    for (int v = 0; v < 32; v++) tmp[(size_t)v * 32 + u] = col[v];
  }
  for (int v = 0; v < 32; v++) {
    int32_t row[32];
    for (int u = 0; u < 32; u++) row[u] = tmp[(size_t)v * 32 + u];
    dct1d_32(row);
    for (int u = 0; u < 32; u++) {
      const int64_t prod = (int64_t)row[u] * 16384;
      store_quant_target(cf, tf, u * 32 + v, (int32_t)((prod + (1ll << (15 + B))) >> (16 + B)), mdc, mac);
    }
  }
}

// dct.rs:1586-1611 identity_quant_t_direct (IDTX; QM never applied).
void fwd_idtx(const int32_t* in, int w, int h, int32_t dc_q, int32_t ac_q, int32_t* cf, float* tf) {
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      int rc = y + x * h;
      int32_t qd = rc == 0 ? dc_q : ac_q;
      int32_t num = in[y * w + x] * 8;
      tf[rc] = (float)num / (float)qd;
      int32_t am = (int32_t)uabs(num);
      if (am < qd) {
        cf[rc] = 0;
      } else {
        int32_t level = (am + qd / 2) / qd;
        cf[rc] = num < 0 ? -level : level;
      }
    }
}

// ----------------------------------------------------------------- idct.rs
// idct.rs:1432-1443 inv_dct4_1d.
void inv_dct4(int32_t* c, int s, int32_t mn, int32_t mx) {
  int32_t in0 = c[0], in1 = c[s], in2 = c[2 * s], in3 = c[3 * s];
  int32_t t0 = ((in0 + in2) * 181 + 128) >> 8;
  int32_t t1 = ((in0 - in2) * 181 + 128) >> 8;
  int32_t t2 = ((in1 * 1567 - in3 * (3784 - 4096) + 2048) >> 12) - in3;
  int32_t t3 = ((in1 * (3784 - 4096) + in3 * 1567 + 2048) >> 12) + in1;
  c[0] = clampi(t0 + t3, mn, mx);
  c[s] = clampi(t1 + t2, mn, mx);
  c[2 * s] = clampi(t1 - t2, mn, mx);
  c[3 * s] = clampi(t0 - t3, mn, mx);
}
// idct.rs:1446-1470 inv_dct8_1d.
void inv_dct8(int32_t* c, int s, int32_t mn, int32_t mx) {
  inv_dct4(c, 2 * s, mn, mx);
  int32_t in1 = c[s], in3 = c[3 * s], in5 = c[5 * s], in7 = c[7 * s];
  int32_t t4a = ((in1 * 799 - in7 * (4017 - 4096) + 2048) >> 12) - in7;
  int32_t t5a = (in5 * 1703 - in3 * 1138 + 1024) >> 11;
  int32_t t6a = (in5 * 1138 + in3 * 1703 + 1024) >> 11;
  int32_t t7a = ((in1 * (4017 - 4096) + in7 * 799 + 2048) >> 12) + in1;
  int32_t t4 = clampi(t4a + t5a, mn, mx);
  t5a = clampi(t4a - t5a, mn, mx);
  int32_t t7 = clampi(t7a + t6a, mn, mx);
  t6a = clampi(t7a - t6a, mn, mx);
  int32_t t5 = ((t6a - t5a) * 181 + 128) >> 8;
  int32_t t6 = ((t6a + t5a) * 181 + 128) >> 8;
  int32_t t0 = c[0], t1 = c[2 * s], t2 = c[4 * s], t3 = c[6 * s];
  c[0] = clampi(t0 + t7, mn, mx);
  c[s] = clampi(t1 + t6, mn, mx);
  c[2 * s] = clampi(t2 + t5, mn, mx);
  c[3 * s] = clampi(t3 + t4, mn, mx);
  c[4 * s] = clampi(t3 - t4, mn, mx);
  c[5 * s] = clampi(t2 - t5, mn, mx);
  c[6 * s] = clampi(t1 - t6, mn, mx);
  c[7 * s] = clampi(t0 - t7, mn, mx);
}
// idct.rs:1473-1509 inv_adst8_1d.
void inv_adst8(int32_t* c, int s, int32_t mn, int32_t mx) {
  int32_t in0 = c[0], in1 = c[s], in2 = c[2 * s], in3 = c[3 * s];
  int32_t in4 = c[4 * s], in5 = c[5 * s], in6 = c[6 * s], in7 = c[7 * s];
  int32_t t0a = (((4076 - 4096) * in7 + 401 * in0 + 2048) >> 12) + in7;
  int32_t t1a = ((401 * in7 - (4076 - 4096) * in0 + 2048) >> 12) - in0;
  int32_t t2a = (((3612 - 4096) * in5 + 1931 * in2 + 2048) >> 12) + in5;
  int32_t t3a = ((1931 * in5 - (3612 - 4096) * in2 + 2048) >> 12) - in2;
  int32_t t4a = (1299 * in3 + 1583 * in4 + 1024) >> 11;
  int32_t t5a = (1583 * in3 - 1299 * in4 + 1024) >> 11;
  int32_t t6a = ((1189 * in1 + (3920 - 4096) * in6 + 2048) >> 12) + in6;
  int32_t t7a = (((3920 - 4096) * in1 - 1189 * in6 + 2048) >> 12) + in1;
  int32_t t0 = clampi(t0a + t4a, mn, mx);
  int32_t t1 = clampi(t1a + t5a, mn, mx);
  int32_t t2 = clampi(t2a + t6a, mn, mx);
  int32_t t3 = clampi(t3a + t7a, mn, mx);
  int32_t t4 = clampi(t0a - t4a, mn, mx);
  int32_t t5 = clampi(t1a - t5a, mn, mx);
  int32_t t6 = clampi(t2a - t6a, mn, mx);
  int32_t t7 = clampi(t3a - t7a, mn, mx);
  int32_t u4a = (((3784 - 4096) * t4 + 1567 * t5 + 2048) >> 12) + t4;
  int32_t u5a = ((1567 * t4 - (3784 - 4096) * t5 + 2048) >> 12) - t5;
  int32_t u6a = (((3784 - 4096) * t7 - 1567 * t6 + 2048) >> 12) + t7;
  int32_t u7a = ((1567 * t7 + (3784 - 4096) * t6 + 2048) >> 12) + t6;
  c[0] = clampi(t0 + t2, mn, mx);
  c[7 * s] = -clampi(t1 + t3, mn, mx);
  int32_t v2 = clampi(t0 - t2, mn, mx);
  int32_t v3 = clampi(t1 - t3, mn, mx);
  c[s] = -clampi(u4a + u6a, mn, mx);
  c[6 * s] = clampi(u5a + u7a, mn, mx);
  int32_t v6 = clampi(u4a - u6a, mn, mx);
  int32_t v7 = clampi(u5a - u7a, mn, mx);
  c[3 * s] = -(((v2 + v3) * 181 + 128) >> 8);
  c[4 * s] = ((v2 - v3) * 181 + 128) >> 8;
  c[2 * s] = ((v6 + v7) * 181 + 128) >> 8;
  c[5 * s] = -(((v6 - v7) * 181 + 128) >> 8);
}

// idct.rs:2837-2865 inv_adst4_1d (no clamps).
void inv_adst4(int32_t* c, int s) {
  int32_t in0 = c[0], in1 = c[s], in2 = c[2 * s], in3 = c[3 * s];
  int32_t o0 = ((1321 * in0 + (3803 - 4096) * in2 + (2482 - 4096) * in3 + (3344 - 4096) * in1 + 2048) >> 12) + in2 +
               in3 + in1;
  int32_t o1 = (((2482 - 4096) * in0 - 1321 * in2 - (3803 - 4096) * in3 + (3344 - 4096) * in1 + 2048) >> 12) + in0 -
               in3 + in1;
  int32_t o2 = (209 * (in0 - in2 + in3) + 128) >> 8;
  int32_t o3 = (((3803 - 4096) * in0 + (2482 - 4096) * in2 - 1321 * in3 - (3344 - 4096) * in1 + 2048) >> 12) + in0 +
               in2 - in1;
  c[0] = o0;
  c[s] = o1;
  c[2 * s] = o2;
  c[3 * s] = o3;
}
// idct.rs:2719-2748 identity4 step: i + (i * 1697 + 2048) >> 12.
inline int32_t inv_id4(int32_t i) { return i + ((i * 1697 + 2048) >> 12); }

// idct.rs:1562-1570 IdctDequant::step and the dequant loop shared by every
// inverse (idct.rs:1581-1590): 24-bit magnitude wrap, cf_max clip.
void dequant(const int32_t* lv, int n, int h, const mt_quant* q, const uint8_t* qm, int32_t* coeff) {
  (void)h;
  for (int rc = 0; rc < n; rc++) {
    int32_t l = lv[rc];
    if (l == 0) {
      coeff[rc] = 0;
      continue;
    }
    int32_t base = rc == 0 ? q->dc_q : q->ac_q;
    int32_t step = qm ? ((base * (int32_t)qm[rc] + 16) >> 5) : base;
    int32_t mag = (int32_t)(((uint64_t)uabs(l) * (uint64_t)(uint32_t)step) & 0xffffffULL);
    int32_t cap = q->cf_max + (l < 0 ? 1 : 0);
    if (mag > cap) mag = cap;
    coeff[rc] = l < 0 ? -mag : mag;
  }
}

// idct.rs:1572-1611 (DCT_DCT), :1683-1783 (ADST family), :1613-1681 (V/H),
// :1785-1824 (IDTX).  Row pass on tmp[y*8 + x] = coeff[y + x*8], (t+1)>>1 with
// the column clip, column pass, (t+8)>>4.
void inv_8x8(const int32_t* levels, int tx, const mt_quant* q, const uint8_t* qm, int32_t* out) {
  int32_t coeff[64];
  const bool flat = (tx == MT_TX_IDTX || tx == MT_TX_V_DCT || tx == MT_TX_H_DCT);
  dequant(levels, 64, 8, q, flat ? nullptr : qm, coeff);
  int32_t tmp[64];
  for (int y = 0; y < 8; y++)
    for (int x = 0; x < 8; x++) tmp[y * 8 + x] = coeff[y + x * 8];
  // row transform kind / column transform kind
  int rowk, colk;  // 0 identity, 1 dct, 2 adst
  switch (tx) {
    case MT_TX_IDTX: rowk = 0; colk = 0; break;
    case MT_TX_DCT_DCT: rowk = 1; colk = 1; break;
    case MT_TX_V_DCT: rowk = 0; colk = 1; break;
    case MT_TX_H_DCT: rowk = 1; colk = 0; break;
    case MT_TX_ADST_ADST: rowk = 2; colk = 2; break;
    case MT_TX_ADST_DCT: rowk = 1; colk = 2; break;
    default: rowk = 2; colk = 1; break;  // DCT_ADST
  }
  for (int y = 0; y < 8; y++) {
    if (rowk == 1) inv_dct8(tmp + y * 8, 1, q->rmin, q->rmax);
    else if (rowk == 2) inv_adst8(tmp + y * 8, 1, q->rmin, q->rmax);
  }
  if (rowk == 0)
    for (int i = 0; i < 64; i++) tmp[i] *= 2;
  for (int i = 0; i < 64; i++) tmp[i] = clampi((tmp[i] + 1) >> 1, q->cmin, q->cmax);
  for (int x = 0; x < 8; x++) {
    if (colk == 1) inv_dct8(tmp + x, 8, q->cmin, q->cmax);
    else if (colk == 2) inv_adst8(tmp + x, 8, q->cmin, q->cmax);
  }
  if (colk == 0)
    for (int i = 0; i < 64; i++) tmp[i] *= 2;
  for (int i = 0; i < 64; i++) out[i] = (tmp[i] + 8) >> 4;
}

// idct.rs:2719-2948 the 4x4 inverses: rows (kind by type), no inter-pass
// shift, the column clamp, columns, (t+8)>>4; identity4 rows/columns use the
// 1697 step; the identity family (IDTX, V_DCT, H_DCT) dequantises flat.
void inv_4x4(const int32_t* levels, int tx, const mt_quant* q, const uint8_t* qm, int32_t* out) {
  int32_t coeff[16];
  const bool flat = (tx == MT_TX_IDTX || tx == MT_TX_V_DCT || tx == MT_TX_H_DCT);
  dequant(levels, 16, 4, q, flat ? nullptr : qm, coeff);
  int32_t tmp[16];
  for (int y = 0; y < 4; y++)
    for (int x = 0; x < 4; x++) tmp[y * 4 + x] = coeff[y + x * 4];
  int rowk, colk;  // 0 identity, 1 dct, 2 adst
  switch (tx) {
    case MT_TX_IDTX: rowk = 0; colk = 0; break;
    case MT_TX_DCT_DCT: rowk = 1; colk = 1; break;
    case MT_TX_V_DCT: rowk = 0; colk = 1; break;
    case MT_TX_H_DCT: rowk = 1; colk = 0; break;
    case MT_TX_ADST_ADST: rowk = 2; colk = 2; break;
    case MT_TX_ADST_DCT: rowk = 1; colk = 2; break;
    default: rowk = 2; colk = 1; break;  // DCT_ADST
  }
  for (int y = 0; y < 4; y++) {
    if (rowk == 1) inv_dct4(tmp + y * 4, 1, q->rmin, q->rmax);
    else if (rowk == 2) inv_adst4(tmp + y * 4, 1);
    else
      for (int x = 0; x < 4; x++) tmp[y * 4 + x] = inv_id4(tmp[y * 4 + x]);
  }
  for (int i = 0; i < 16; i++) tmp[i] = clampi(tmp[i], q->cmin, q->cmax);
  for (int x = 0; x < 4; x++) {
    if (colk == 1) inv_dct4(tmp + x, 4, q->cmin, q->cmax);
    else if (colk == 2) inv_adst4(tmp + x, 4);
    else
      for (int y = 0; y < 4; y++) tmp[y * 4 + x] = inv_id4(tmp[y * 4 + x]);
  }
  for (int i = 0; i < 16; i++) out[i] = (tmp[i] + 8) >> 4;
}

// ------------------------------------------------------- cost.rs / trellis
// cost.rs:70-75 COEF_RATE_LUT, cost.rs:50-68 coef_rate_bits_slow.
const float COEF_RATE_LUT[64] = {
    0.9f,  2.7f,  3.6f,  5.3f,  5.3f,  5.3f,  6.6f,  6.6f,  6.6f,  7.9f,  7.9f,  7.9f,  9.2f,
    9.2f,  9.2f,  11.5f, 13.5f, 13.5f, 15.5f, 15.5f, 15.5f, 15.5f, 17.5f, 17.5f, 17.5f, 17.5f,
    17.5f, 17.5f, 17.5f, 17.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f,
    19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 19.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f,
    21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f, 21.5f,
};
inline int lzcnt32(uint32_t v) { return v == 0 ? 32 : __builtin_clz(v); }
float coef_rate_bits(uint32_t level) {
  if (level < 64) return COEF_RATE_LUT[level];
  float b = 3.0f + 1.0f;
  int32_t total_br = (int32_t)level - 3;
  if (total_br > 12) total_br = 12;
  float steps = (float)(total_br / 3 + 1);
  b += steps * 1.3f;
  if (level >= 15) {
    uint32_t v = level - 15;
    b += 2.0f * (float)(32 - lzcnt32(v + 1)) + -1.0f;  // f_fmlaf: unfused on the pinned build
  }
  return b;
}

// trellis.rs:38-53 lambda law (SHIPPED trellis_calib = 1.15, tuning.rs:953).
const float TRELLIS_AOM_CALIB = 0.045025873597302174f * 0.5525f;
const float TRELLIS_CALIB = 1.15f;
const float TRELLIS_LAMBDA0 = 0.05f;
float scaled_trellis_lambda(float dc_q, float ac_q, float lambda0) {
  (void)ac_q;
  float aom = TRELLIS_AOM_CALIB * TRELLIS_CALIB * dc_q * dc_q * (3.3f + 0.0015f * dc_q);
  return aom * (lambda0 / TRELLIS_LAMBDA0);
}
}  // namespace
extern "C" float or_scaled_trellis_lambda(float dc_q, float ac_q, float lambda0) {
  return scaled_trellis_lambda(dc_q, ac_q, lambda0);
}
namespace {

// avx/trellis.rs:79-137 round_down_cost8/4 (FMA lanes) and :139-161
// round_down_scalar_one; driver avx/trellis.rs:163-230.
void round_down_scalar_one(int32_t* cf, const float* tf, int rc, float dc_q2, float ac_q2, float lambda) {
  int32_t c = cf[rc];
  if (c == 0) return;
  uint32_t l = uabs(c);
  float dq2 = rc == 0 ? dc_q2 : ac_q2;
  float at = fabsf(tf[rc]);
  float e_l = at - (float)l;
  float e_dn = at - (float)(l - 1);
  float cost_l = dq2 * (e_l * e_l) + lambda * coef_rate_bits(l);
  float cost_dn = dq2 * (e_dn * e_dn) + lambda * coef_rate_bits(l - 1);
  if (cost_dn < cost_l) cf[rc] = c < 0 ? -(int32_t)(l - 1) : (int32_t)(l - 1);
}
void round_down_chunk(int32_t* cf, const float* tf, const uint16_t* scan, int i, int width,
                      float dc_q2, float ac_q2, float lambda) {
  bool big = false;
  for (int k = 0; k < width; k++)
    if (uabs(cf[scan[i + k]]) > 63) big = true;
  if (big) {
    for (int k = 0; k < width; k++) round_down_scalar_one(cf, tf, scan[i + k], dc_q2, ac_q2, lambda);
    return;
  }
  bool better[8];
  for (int k = 0; k < width; k++) {
    int rc = scan[i + k];
    int32_t li = (int32_t)uabs(cf[rc]);
    int32_t ldi = li - 1 > 0 ? li - 1 : 0;
    float at = fabsf(tf[rc]);
    float q2 = (i == 0 && k == 0) ? dc_q2 : ac_q2;
    float e_l = at - (float)li;
    float e_dn = at - (float)ldi;
    float cost_l = fmaf(q2, e_l * e_l, lambda * COEF_RATE_LUT[li]);
    float cost_dn = fmaf(q2, e_dn * e_dn, lambda * COEF_RATE_LUT[ldi]);
    better[k] = cost_dn < cost_l;
  }
  for (int k = 0; k < width; k++) {
    if (!better[k]) continue;
    int rc = scan[i + k];
    int32_t c = cf[rc];
    if (c != 0) {
      int32_t l = iabs(c);
      cf[rc] = c < 0 ? -(l - 1) : (l - 1);
    }
  }
}
void round_down_scan(int32_t* cf, const float* tf, const uint16_t* scan, int n, float dc_q2, float ac_q2,
                     float lambda) {
  int i = 0;
  while (i + 8 <= n) {
    round_down_chunk(cf, tf, scan, i, 8, dc_q2, ac_q2, lambda);
    i += 8;
  }
  while (i + 4 <= n) {
    round_down_chunk(cf, tf, scan, i, 4, dc_q2, ac_q2, lambda);
    i += 4;
  }
  for (; i < n; i++) round_down_scalar_one(cf, tf, scan[i], dc_q2, ac_q2, lambda);
}

}  // namespace

extern "C" {

int or_quant_init(uint8_t base_q_idx, uint8_t bd, uint8_t qm_level, mt_quant* out) {
  if (!out || bd != 8) return MT_ERR_UNSUPPORTED;
  int dc_idx = clampi((int)base_q_idx - 8, 0, 255);  // quant.rs:347 luma_dc_delta = -8
  fill_quant(MT_DC_QLOOKUP_8[dc_idx], MT_AC_QLOOKUP_8[base_q_idx], qm_level, 0, base_q_idx, out);
  return MT_OK;
}

int or_quant_init_chroma(uint8_t base_q_idx, int32_t dc_delta, int32_t ac_delta, uint8_t bd,
                         uint8_t qm_level, mt_quant* out) {
  if (!out || bd != 8) return MT_ERR_UNSUPPORTED;
  int dc_idx = clampi((int)base_q_idx + dc_delta, 0, 255);
  int ac_idx = clampi((int)base_q_idx + ac_delta, 0, 255);
  fill_quant(MT_DC_QLOOKUP_8[dc_idx], MT_AC_QLOOKUP_8[ac_idx], qm_level, 1, ac_idx, out);
  return MT_OK;
}

const uint8_t* or_qm_row(int32_t qm_level, int32_t chroma, int32_t w, int32_t h) {
  if (qm_level >= 15 || qm_level < 0) return nullptr;
  int off = qm_offset(w, h);
  if (off < 0) return nullptr;
  return &MT_AV1_IQM[((size_t)qm_level * 2 + (chroma ? 1 : 0)) * 3344 + off];
}

// dct1d_32_i32 on one buffer of 32 (for the property tests of dct.rs:4091-4125).
void or_dct1d_32(int32_t* buf) { dct1d_32(buf); }

const uint16_t* or_default_scan(int32_t n) {
  switch (n) {
    case 4: return MT_SCAN_4X4;
    case 8: return MT_SCAN_8X8;
    case 16: return MT_SCAN_16X16;
    case 32: return MT_SCAN_32X32;
  }
  return nullptr;
}

void inv_16x16(const int32_t* levels, int tx, const mt_quant* q, const uint8_t* qm, int32_t* out);
void inv_32x32(const int32_t* levels, const mt_quant* q, const uint8_t* qm, int32_t* out);

// DctDispatch::dct8x8_t / adst8x8_t / adstdct8x8_t / dctadst8x8_t (QM applied,
// dct.rs:2751-2763, :2896-2909), fvdct8x8_t / fhdct8x8_t (flat, :2910-2920),
// idtx8x8_t (dc/ac steps, :2918-2924).
void or_fwd_txfm_quant(const int32_t* resid, int32_t tx, int32_t n, const mt_quant* q,
                       const uint8_t* qm_row, int32_t* cf, float* tf) {
  if (n == 4) {
    // DctDispatch::dct4x4_t and the dispatch_qm_ratio_methods family
    // (dct.rs:2465-2488, :2624-2637, :2876-2880): Q16 multipliers x 8/sqrt(16)
    // = 2 (RATIO_4X4_Q16); V/H flat (:2510-2523, :2899-2901); IDTX dc/ac steps.
    const int32_t r4 = 131072;
    const int32_t mdc = mul_q16(q->q_mult_dc, r4), mac = mul_q16(q->q_mult_ac, r4);
    switch (tx) {
      case MT_TX_IDTX: fwd_idtx(resid, 4, 4, q->dc_q, q->ac_q, cf, tf); return;
      case MT_TX_V_DCT: fwd_1d_4x4(resid, true, q->q_mult_dc, q->q_mult_ac, cf, tf); return;
      case MT_TX_H_DCT: fwd_1d_4x4(resid, false, q->q_mult_dc, q->q_mult_ac, cf, tf); return;
      case MT_TX_DCT_DCT: fwd_2d_4x4(resid, dct1d_4, dct1d_4, mdc, mac, cf, tf); break;
      case MT_TX_ADST_ADST: fwd_2d_4x4(resid, fwd_adst4, fwd_adst4, mdc, mac, cf, tf); break;
      case MT_TX_ADST_DCT: fwd_2d_4x4(resid, fwd_adst4, dct1d_4, mdc, mac, cf, tf); break;
      case MT_TX_DCT_ADST: fwd_2d_4x4(resid, dct1d_4, fwd_adst4, mdc, mac, cf, tf); break;
      default: return;
    }
    if (qm_row) apply_qmatrix(cf, tf, qm_row, 16);
    return;
  }
  if (n == 32) {  // TX_32X32: DCT_DCT only (dct.rs:2862-2873, QM applied)
    if (tx != MT_TX_DCT_DCT) return;
    fwd_2d_32x32(resid, q->q_mult_dc, q->q_mult_ac, cf, tf);
    if (qm_row) apply_qmatrix(cf, tf, qm_row, 1024);
    return;
  }
  if (n == 16) {
    switch (tx) {
      case MT_TX_IDTX: fwd_idtx(resid, 16, 16, q->dc_q, q->ac_q, cf, tf); return;
      case MT_TX_DCT_DCT: fwd_2d_16x16(resid, dct1d_16, dct1d_16, q->q_mult_dc, q->q_mult_ac, cf, tf); break;
      case MT_TX_ADST_ADST: fwd_2d_16x16(resid, fwd_adst16, fwd_adst16, q->q_mult_dc, q->q_mult_ac, cf, tf); break;
      case MT_TX_ADST_DCT: fwd_2d_16x16(resid, fwd_adst16, dct1d_16, q->q_mult_dc, q->q_mult_ac, cf, tf); break;
      case MT_TX_DCT_ADST: fwd_2d_16x16(resid, dct1d_16, fwd_adst16, q->q_mult_dc, q->q_mult_ac, cf, tf); break;
      default: return;
    }
    if (qm_row) apply_qmatrix(cf, tf, qm_row, 256);
    return;
  }
  if (n != 8) return;
  switch (tx) {
    case MT_TX_IDTX: fwd_idtx(resid, 8, 8, q->dc_q, q->ac_q, cf, tf); return;
    case MT_TX_V_DCT: fwd_1d_8x8(resid, true, q->q_mult_dc, q->q_mult_ac, cf, tf); return;
    case MT_TX_H_DCT: fwd_1d_8x8(resid, false, q->q_mult_dc, q->q_mult_ac, cf, tf); return;
    case MT_TX_DCT_DCT: fwd_2d_8x8(resid, dct1d_8, dct1d_8, q->q_mult_dc, q->q_mult_ac, cf, tf); break;
    case MT_TX_ADST_ADST: fwd_2d_8x8(resid, fwd_adst8, fwd_adst8, q->q_mult_dc, q->q_mult_ac, cf, tf); break;
    case MT_TX_ADST_DCT: fwd_2d_8x8(resid, fwd_adst8, dct1d_8, q->q_mult_dc, q->q_mult_ac, cf, tf); break;
    case MT_TX_DCT_ADST: fwd_2d_8x8(resid, dct1d_8, fwd_adst8, q->q_mult_dc, q->q_mult_ac, cf, tf); break;
    default: return;
  }
  if (qm_row) apply_qmatrix(cf, tf, qm_row, 64);
}

void or_inv_txfm_dequant(const int32_t* levels, int32_t tx, int32_t n, const mt_quant* q,
                         const uint8_t* qm_row, int32_t* resid) {
  if (n == 4) inv_4x4(levels, tx, q, qm_row, resid);
  if (n == 16) inv_16x16(levels, tx, q, qm_row, resid);
  if (n == 32 && tx == MT_TX_DCT_DCT) inv_32x32(levels, q, qm_row, resid);
  if (n != 8) return;
  inv_8x8(levels, tx, q, qm_row, resid);
}

// One dav1d rotation: (x * cx + y * cy + 2048) >> 12.  The reference writes
// most of them with one constant minus 4096 and the input added back, and a
// few with halved constants and >> 11; those equal this form exactly.
inline int32_t rot12(int32_t x, int32_t cx, int32_t y, int32_t cy) { return (x * cx + y * cy + 2048) >> 12; }
inline int32_t r181(int32_t v) { return (v * 181 + 128) >> 8; }

// idct.rs:1871-1924 inv_dct16_1d: the 8-point inverse on the even inputs, the
// odd half in four stages with the intermediate clip, the output butterflies.
void inv_dct16(int32_t* c, int s, int32_t mn, int32_t mx) {
  auto cl = [&](int32_t v) { return clampi(v, mn, mx); };
  inv_dct8(c, 2 * s, mn, mx);
  const int32_t in1 = c[s], in3 = c[3 * s], in5 = c[5 * s], in7 = c[7 * s];
  const int32_t in9 = c[9 * s], in11 = c[11 * s], in13 = c[13 * s], in15 = c[15 * s];
  const int32_t a8 = rot12(in1, 401, in15, -4076), a9 = rot12(in9, 3166, in7, -2598);
  const int32_t a10 = rot12(in5, 1931, in11, -3612), a11 = rot12(in13, 3920, in3, -1189);
  const int32_t a12 = rot12(in13, 1189, in3, 3920), a13 = rot12(in5, 3612, in11, 1931);
  const int32_t a14 = rot12(in9, 2598, in7, 3166), a15 = rot12(in1, 4076, in15, 401);
  const int32_t b8 = cl(a8 + a9), b9 = cl(a8 - a9), b10 = cl(a11 - a10), b11 = cl(a11 + a10);
  const int32_t b12 = cl(a12 + a13), b13 = cl(a12 - a13), b14 = cl(a15 - a14), b15 = cl(a15 + a14);
  const int32_t c9 = rot12(b14, 1567, b9, -3784), c14 = rot12(b14, 3784, b9, 1567);
  const int32_t c10 = rot12(b13, -3784, b10, -1567), c13 = rot12(b13, 1567, b10, -3784);
  const int32_t d8 = cl(b8 + b11), d9 = cl(c9 + c10), d10 = cl(c9 - c10), d11 = cl(b8 - b11);
  const int32_t d12 = cl(b15 - b12), d13 = cl(c14 - c13), d14 = cl(c14 + c13), d15 = cl(b15 + b12);
  const int32_t e10 = r181(d13 - d10), e13 = r181(d13 + d10), e11 = r181(d12 - d11), e12 = r181(d12 + d11);
  const int32_t t0 = c[0], t1 = c[2 * s], t2 = c[4 * s], t3 = c[6 * s];
  const int32_t t4 = c[8 * s], t5 = c[10 * s], t6 = c[12 * s], t7 = c[14 * s];
  c[0] = cl(t0 + d15);
  c[s] = cl(t1 + d14);
  c[2 * s] = cl(t2 + e13);
  c[3 * s] = cl(t3 + e12);
  c[4 * s] = cl(t4 + e11);
  c[5 * s] = cl(t5 + e10);
  c[6 * s] = cl(t6 + d9);
  c[7 * s] = cl(t7 + d8);
  c[8 * s] = cl(t7 - d8);
  c[9 * s] = cl(t6 - d9);
  c[10 * s] = cl(t5 - e10);
  c[11 * s] = cl(t4 - e11);
  c[12 * s] = cl(t3 - e12);
  c[13 * s] = cl(t2 - e13);
  c[14 * s] = cl(t1 - d14);
  c[15 * s] = cl(t0 - d15);
}

// idct.rs:1968-2062 inv_adst16_1d (dav1d): four rotation / butterfly stages
// with the intermediate clip and the signed 181/256 outputs.
void inv_adst16(int32_t* c, int s, int32_t mn, int32_t mx) {
  auto cl = [&](int32_t v) { return clampi(v, mn, mx); };
  int32_t in[16];
  for (int i = 0; i < 16; i++) in[i] = c[i * s];
  int32_t a[16];
  a[0] = rot12(in[15], 4091, in[0], 201);
  a[1] = rot12(in[15], 201, in[0], -4091);
  a[2] = rot12(in[13], 3973, in[2], 995);
  a[3] = rot12(in[13], 995, in[2], -3973);
  a[4] = rot12(in[11], 3703, in[4], 1751);
  a[5] = rot12(in[11], 1751, in[4], -3703);
  a[6] = rot12(in[9], 3290, in[6], 2440);
  a[7] = rot12(in[9], 2440, in[6], -3290);
  a[8] = rot12(in[7], 2751, in[8], 3035);
  a[9] = rot12(in[7], 3035, in[8], -2751);
  a[10] = rot12(in[5], 2106, in[10], 3513);
  a[11] = rot12(in[5], 3513, in[10], -2106);
  a[12] = rot12(in[3], 1380, in[12], 3857);
  a[13] = rot12(in[3], 3857, in[12], -1380);
  a[14] = rot12(in[1], 601, in[14], 4052);
  a[15] = rot12(in[1], 4052, in[14], -601);
  int32_t b[16];
  for (int i = 0; i < 8; i++) {
    b[i] = cl(a[i] + a[i + 8]);
    b[8 + i] = cl(a[i] - a[i + 8]);
  }
  const int32_t c8 = rot12(b[8], 4017, b[9], 799), c9 = rot12(b[8], 799, b[9], -4017);
  const int32_t c10 = rot12(b[10], 2276, b[11], 3406), c11 = rot12(b[10], 3406, b[11], -2276);
  const int32_t c12 = rot12(b[13], 4017, b[12], -799), c13 = rot12(b[13], 799, b[12], 4017);
  const int32_t c14 = rot12(b[15], 2276, b[14], -3406), c15 = rot12(b[15], 3406, b[14], 2276);
  const int32_t d0 = cl(b[0] + b[4]), d1 = cl(b[1] + b[5]), d2 = cl(b[2] + b[6]), d3 = cl(b[3] + b[7]);
  const int32_t d4 = cl(b[0] - b[4]), d5 = cl(b[1] - b[5]), d6 = cl(b[2] - b[6]), d7 = cl(b[3] - b[7]);
  const int32_t d8 = cl(c8 + c12), d9 = cl(c9 + c13), d10 = cl(c10 + c14), d11 = cl(c11 + c15);
  const int32_t d12 = cl(c8 - c12), d13 = cl(c9 - c13), d14 = cl(c10 - c14), d15 = cl(c11 - c15);
  const int32_t e4 = rot12(d4, 3784, d5, 1567), e5 = rot12(d4, 1567, d5, -3784);
  const int32_t e6 = rot12(d7, 3784, d6, -1567), e7 = rot12(d7, 1567, d6, 3784);
  const int32_t e12 = rot12(d12, 3784, d13, 1567), e13 = rot12(d12, 1567, d13, -3784);
  const int32_t e14 = rot12(d15, 3784, d14, -1567), e15 = rot12(d15, 1567, d14, 3784);
  const int32_t f2 = cl(d0 - d2), f3 = cl(d1 - d3), f6 = cl(e4 - e6), f7 = cl(e5 - e7);
  const int32_t f10 = cl(d8 - d10), f11 = cl(d9 - d11), f14 = cl(e12 - e14), f15 = cl(e13 - e15);
  c[0] = cl(d0 + d2);
  c[15 * s] = -cl(d1 + d3);
  c[3 * s] = -cl(e4 + e6);
  c[12 * s] = cl(e5 + e7);
  c[s] = -cl(d8 + d10);
  c[14 * s] = cl(d9 + d11);
  c[2 * s] = cl(e12 + e14);
  c[13 * s] = -cl(e13 + e15);
  c[7 * s] = -r181(f2 + f3);
  c[8 * s] = r181(f2 - f3);
  c[4 * s] = r181(f6 + f7);
  c[11 * s] = -r181(f6 - f7);
  c[6 * s] = r181(f10 + f11);
  c[9 * s] = -r181(f10 - f11);
  c[5 * s] = -r181(f14 + f15);
  c[10 * s] = r181(f14 - f15);
}

// idct.rs:1926-1966 / :2067-2128 the 16x16 inverses: tmp[y*16 + x] =
// coeff[y + x*16]; rows (row clip), (t+2)>>2 with the column clip, columns,
// (t+8)>>4.  IDTX (idct.rs:1826-1869): identity16 2x + (x*1697 + 1024) >> 11
// both passes, flat dequantisation.
void inv_16x16(const int32_t* levels, int tx, const mt_quant* q, const uint8_t* qm, int32_t* out) {
  int32_t coeff[256], tmp[256];
  const bool idtx = tx == MT_TX_IDTX;
  dequant(levels, 256, 16, q, idtx ? nullptr : qm, coeff);
  for (int y = 0; y < 16; y++)
    for (int x = 0; x < 16; x++) tmp[y * 16 + x] = coeff[y + x * 16];
  if (idtx) {
    auto id16 = [](int32_t v) { return 2 * v + ((v * 1697 + 1024) >> 11); };
    for (int i = 0; i < 256; i++) tmp[i] = clampi((id16(tmp[i]) + 2) >> 2, q->cmin, q->cmax);
    for (int i = 0; i < 256; i++) out[i] = (id16(tmp[i]) + 8) >> 4;
    return;
  }
  const bool row_adst = tx == MT_TX_ADST_ADST || tx == MT_TX_DCT_ADST;
  const bool col_adst = tx == MT_TX_ADST_ADST || tx == MT_TX_ADST_DCT;
  for (int y = 0; y < 16; y++) {
    if (row_adst) inv_adst16(tmp + y * 16, 1, q->rmin, q->rmax);
    else inv_dct16(tmp + y * 16, 1, q->rmin, q->rmax);
  }
  for (int i = 0; i < 256; i++) tmp[i] = clampi((tmp[i] + 2) >> 2, q->cmin, q->cmax);
  for (int x = 0; x < 16; x++) {
    if (col_adst) inv_adst16(tmp + x, 16, q->cmin, q->cmax);
    else inv_dct16(tmp + x, 16, q->cmin, q->cmax);
  }
  for (int i = 0; i < 256; i++) out[i] = (tmp[i] + 8) >> 4;
}

// idct.rs:2130-2279 inv_dct32_1d (dav1d), in the reference's own forms: the
// 16-point inverse on the even inputs, seven stages on the odd half.
void inv_dct32(int32_t* c, int s, int32_t mn, int32_t mx) {
  auto cl = [&](int32_t v) { return clampi(v, mn, mx); };
  inv_dct16(c, 2 * s, mn, mx);
  const int32_t in1 = c[s], in3 = c[3 * s], in5 = c[5 * s], in7 = c[7 * s];
  const int32_t in9 = c[9 * s], in11 = c[11 * s], in13 = c[13 * s], in15 = c[15 * s];
  const int32_t in17 = c[17 * s], in19 = c[19 * s], in21 = c[21 * s], in23 = c[23 * s];
  const int32_t in25 = c[25 * s], in27 = c[27 * s], in29 = c[29 * s], in31 = c[31 * s];
  int32_t t16a = ((in1 * 201 - in31 * (4091 - 4096) + 2048) >> 12) - in31;
  int32_t t17a = ((in17 * (3035 - 4096) - in15 * 2751 + 2048) >> 12) + in17;
  int32_t t18a = ((in9 * 1751 - in23 * (3703 - 4096) + 2048) >> 12) - in23;
  int32_t t19a = ((in25 * (3857 - 4096) - in7 * 1380 + 2048) >> 12) + in25;
  int32_t t20a = ((in5 * 995 - in27 * (3973 - 4096) + 2048) >> 12) - in27;
  int32_t t21a = ((in21 * (3513 - 4096) - in11 * 2106 + 2048) >> 12) + in21;
  int32_t t22a = (in13 * 1220 - in19 * 1645 + 1024) >> 11;
  int32_t t23a = ((in29 * (4052 - 4096) - in3 * 601 + 2048) >> 12) + in29;
  int32_t t24a = ((in29 * 601 + in3 * (4052 - 4096) + 2048) >> 12) + in3;
  int32_t t25a = (in13 * 1645 + in19 * 1220 + 1024) >> 11;
  int32_t t26a = ((in21 * 2106 + in11 * (3513 - 4096) + 2048) >> 12) + in11;
  int32_t t27a = ((in5 * (3973 - 4096) + in27 * 995 + 2048) >> 12) + in5;
  int32_t t28a = ((in25 * 1380 + in7 * (3857 - 4096) + 2048) >> 12) + in7;
  int32_t t29a = ((in9 * (3703 - 4096) + in23 * 1751 + 2048) >> 12) + in9;
  int32_t t30a = ((in17 * 2751 + in15 * (3035 - 4096) + 2048) >> 12) + in15;
  int32_t t31a = ((in1 * (4091 - 4096) + in31 * 201 + 2048) >> 12) + in1;
  int32_t t16 = cl(t16a + t17a), t17 = cl(t16a - t17a), t18 = cl(t19a - t18a), t19 = cl(t19a + t18a);
  int32_t t20 = cl(t20a + t21a), t21 = cl(t20a - t21a), t22 = cl(t23a - t22a), t23 = cl(t23a + t22a);
  int32_t t24 = cl(t24a + t25a), t25 = cl(t24a - t25a), t26 = cl(t27a - t26a), t27 = cl(t27a + t26a);
  int32_t t28 = cl(t28a + t29a), t29 = cl(t28a - t29a), t30 = cl(t31a - t30a), t31 = cl(t31a + t30a);
  t17a = ((t30 * 799 - t17 * (4017 - 4096) + 2048) >> 12) - t17;
  t30a = ((t30 * (4017 - 4096) + t17 * 799 + 2048) >> 12) + t30;
  t18a = ((-(t29 * (4017 - 4096) + t18 * 799) + 2048) >> 12) - t29;
  t29a = ((t29 * 799 - t18 * (4017 - 4096) + 2048) >> 12) - t18;
  t21a = (t26 * 1703 - t21 * 1138 + 1024) >> 11;
  t26a = (t26 * 1138 + t21 * 1703 + 1024) >> 11;
  t22a = (-(t25 * 1138 + t22 * 1703) + 1024) >> 11;
  t25a = (t25 * 1703 - t22 * 1138 + 1024) >> 11;
  t16a = cl(t16 + t19);
  t17 = cl(t17a + t18a);
  t18 = cl(t17a - t18a);
  t19a = cl(t16 - t19);
  t20a = cl(t23 - t20);
  t21 = cl(t22a - t21a);
  t22 = cl(t22a + t21a);
  t23a = cl(t23 + t20);
  t24a = cl(t24 + t27);
  t25 = cl(t25a + t26a);
  t26 = cl(t25a - t26a);
  t27a = cl(t24 - t27);
  t28a = cl(t31 - t28);
  t29 = cl(t30a - t29a);
  t30 = cl(t30a + t29a);
  t31a = cl(t31 + t28);
  t18a = ((t29 * 1567 - t18 * (3784 - 4096) + 2048) >> 12) - t18;
  t29a = ((t29 * (3784 - 4096) + t18 * 1567 + 2048) >> 12) + t29;
  t19 = ((t28a * 1567 - t19a * (3784 - 4096) + 2048) >> 12) - t19a;
  t28 = ((t28a * (3784 - 4096) + t19a * 1567 + 2048) >> 12) + t28a;
  t20 = ((-(t27a * (3784 - 4096) + t20a * 1567) + 2048) >> 12) - t27a;
  t27 = ((t27a * 1567 - t20a * (3784 - 4096) + 2048) >> 12) - t20a;
  t21a = ((-(t26 * (3784 - 4096) + t21 * 1567) + 2048) >> 12) - t26;
  t26a = ((t26 * 1567 - t21 * (3784 - 4096) + 2048) >> 12) - t21;
  t16 = cl(t16a + t23a);
  t17a = cl(t17 + t22);
  t18 = cl(t18a + t21a);
  t19a = cl(t19 + t20);
  t20a = cl(t19 - t20);
  t21 = cl(t18a - t21a);
  t22a = cl(t17 - t22);
  t23 = cl(t16a - t23a);
  t24 = cl(t31a - t24a);
  t25a = cl(t30 - t25);
  t26 = cl(t29a - t26a);
  t27a = cl(t28 - t27);
  t28a = cl(t28 + t27);
  t29 = cl(t29a + t26a);
  t30a = cl(t30 + t25);
  t31 = cl(t31a + t24a);
  t20 = ((t27a - t20a) * 181 + 128) >> 8;
  t27 = ((t27a + t20a) * 181 + 128) >> 8;
  t21a = ((t26 - t21) * 181 + 128) >> 8;
  t26a = ((t26 + t21) * 181 + 128) >> 8;
  t22 = ((t25a - t22a) * 181 + 128) >> 8;
  t25 = ((t25a + t22a) * 181 + 128) >> 8;
  t23a = ((t24 - t23) * 181 + 128) >> 8;
  t24a = ((t24 + t23) * 181 + 128) >> 8;
  const int32_t odd[16] = {t31, t30a, t29, t28a, t27, t26a, t25, t24a, t23a, t22, t21a, t20, t19a, t18, t17a, t16};
  int32_t even[16];
  for (int k = 0; k < 16; k++) even[k] = c[2 * k * s];
  for (int k = 0; k < 16; k++) {
    c[k * s] = cl(even[k] + odd[k]);
    c[(31 - k) * s] = cl(even[k] - odd[k]);
  }
}

// idct.rs:2281-2320 idct_dequant_32x32_scalar: the dequantised product masked
// to 24 bits and halved (dq_shift 1), clamped to cf_max; rows with the row
// clip, (t+2)>>2 with the column clip, columns, (t+8)>>4.
void inv_32x32(const int32_t* levels, const mt_quant* q, const uint8_t* qm, int32_t* out) {
  std::vector<int32_t> tmp(1024, 0);
  for (int rc = 0; rc < 1024; rc++) {
    const int32_t l = levels[rc];
    if (l == 0) continue;
    const int32_t base = rc == 0 ? q->dc_q : q->ac_q;
    const int32_t step = qm ? ((base * (int32_t)qm[rc] + 16) >> 5) : base;
    int32_t mag = (int32_t)((((uint64_t)uabs(l) * (uint64_t)(uint32_t)step) & 0xffffffULL) >> 1);
    const int32_t cap = q->cf_max + (l < 0 ? 1 : 0);
    if (mag > cap) mag = cap;
    tmp[(size_t)(rc & 31) * 32 + (rc >> 5)] = l < 0 ? -mag : mag;
  }
  for (int y = 0; y < 32; y++) inv_dct32(&tmp[(size_t)y * 32], 1, q->rmin, q->rmax);
  for (int i = 0; i < 1024; i++) tmp[i] = clampi((tmp[i] + 2) >> 2, q->cmin, q->cmax);
  for (int x = 0; x < 32; x++) inv_dct32(&tmp[x], 32, q->cmin, q->cmax);
  for (int i = 0; i < 1024; i++) out[i] = (tmp[i] + 8) >> 4;
}

// trellis.rs:944-1030 trellis_optimize with the AVX2 step A
// (avx/trellis.rs:163-230) and AVX2 dist scan (avx/trellis.rs:232-321, same
// products as trellis_dist.rs:178-196).
void or_trellis_optimize(int32_t* cf, const float* tf, float dc_q, float ac_q, const uint16_t* scan,
                         int32_t n, float lambda0) {
  if (lambda0 <= 0.0f) return;
  float lambda = scaled_trellis_lambda(dc_q, ac_q, lambda0);
  float dc_q2 = dc_q * dc_q, ac_q2 = ac_q * ac_q;
  int eob_idx = -1;
  for (int i = n - 1; i >= 0; i--)
    if (cf[scan[i]] != 0) {
      eob_idx = i;
      break;
    }
  if (eob_idx < 0) return;
  int m = eob_idx + 1;
  round_down_scan(cf, tf, scan, m, dc_q2, ac_q2, lambda);
  std::vector<float> dcur(m), dzero(m), suf0(m + 1);
  for (int i = 0; i < m; i++) {
    int rc = scan[i];
    float dq2 = rc == 0 ? dc_q2 : ac_q2;
    float at = fabsf(tf[rc]);
    float e = at - (float)uabs(cf[rc]);
    dcur[i] = dq2 * (e * e);
    dzero[i] = dq2 * (at * at);
  }
  suf0[m] = 0.0f;
  for (int i = m - 1; i >= 0; i--) suf0[i] = suf0[i + 1] + dzero[i];
  int best_e = -1;
  float best_cost = INFINITY;
  float pre = 0.0f;
  for (int e = 0; e < m; e++) {
    int rc = scan[e];
    if (cf[rc] != 0) {
      uint32_t ue = (uint32_t)e;
      int bin = e < 2 ? e : 32 - lzcnt32(ue);
      int extra = bin > 1 ? bin - 2 : 0;
      float sig = (float)bin * 0.9f + ((float)extra + 2.0f);  // f_fmlaf, unfused
      float c = pre + dcur[e] + lambda * sig + suf0[e + 1];
      if (c < best_cost) {
        best_cost = c;
        best_e = e;
      }
    }
    pre = pre + dcur[e] + lambda * coef_rate_bits(uabs(cf[rc]));
  }
  float skip_cost = suf0[0] + lambda * 1.0f;  // tuning.rs:946 trellis_zero_bits = 1.0
  if (best_e < 0 || skip_cost < best_cost) {
    for (int i = 0; i < m; i++) cf[scan[i]] = 0;
  } else {
    for (int i = best_e + 1; i < m; i++) cf[scan[i]] = 0;
  }
}

// intrapred.rs:1740-1789 dc_pred + dc_pred_from_sum.
int32_t or_dc_pred(const uint16_t* recon, int32_t stride, int32_t ox, int32_t oy, int32_t w, int32_t h,
                   int32_t bd) {
  bool have_top = oy > 0, have_left = ox > 0;
  int32_t sum = 0;
  if (have_top)
    for (int x = 0; x < w; x++) sum += recon[(size_t)(oy - 1) * stride + ox + x];
  if (have_left)
    for (int y = 0; y < h; y++) sum += recon[(size_t)(oy + y) * stride + ox - 1];
  if (have_top && have_left) {
    int32_t s = ((w + h) >> 1) + sum;
    s >>= __builtin_ctz((unsigned)(w + h));
    if (w != h) {
      uint32_t mult = (w > 2 * h || h > 2 * w) ? 0x3334u : 0x5556u;
      s = (int32_t)(((uint32_t)s * mult) >> 16);
    }
    return s;
  }
  if (have_top) return ((w >> 1) + sum) >> __builtin_ctz((unsigned)w);
  if (have_left) return ((h >> 1) + sum) >> __builtin_ctz((unsigned)h);
  return 1 << (bd - 1);
}

}  // extern "C"

namespace {
// intrapred.rs:422-423: edge storage with origin 2 (logical index -2..129).
struct Edge {
  int32_t s[132];
  int32_t& at(int i) { return s[i + 2]; }
};
// intrapred.rs:1084-1089 DR_INTRA_DERIVATIVE, :1094-1109 sm_weights.
const int32_t DR_DERIV[44] = {0,   1023, 0, 547, 372, 0,  0,  273, 215, 0,  178, 151, 0,  132, 116,
                              0,   102,  0, 90,  80,  0,  71, 64,  0,   57, 51,  0,   45, 0,   40,
                              35,  0,    31, 27, 0,   23, 19, 0,   15,  0,  11,  0,   7,  3};
const int32_t SMW4[4] = {255, 149, 85, 64};
const int32_t SMW8[8] = {255, 197, 146, 105, 73, 50, 37, 32};
const int32_t SMW16[16] = {255, 225, 196, 170, 145, 123, 102, 84, 68, 54, 43, 33, 26, 20, 17, 16};
const int32_t SMW32[32] = {255, 240, 225, 210, 196, 182, 169, 157, 145, 133, 122, 111, 101, 92, 83, 74,
                           66,  59,  52,  45,  39,  34,  29,  25,  21,  17,  14,  12,  10,  9,  8,  8};
const int32_t* sm_weights(int n) {
  switch (n) {
    case 4: return SMW4;
    case 8: return SMW8;
    case 16: return SMW16;
    default: return SMW32;
  }
}
// intrapred.rs:917-975 intra_edge_filter_strength.
int edge_filter_strength(int w, int h, bool ft, int delta) {
  int d = iabs(delta), wh = w + h, s = 0;
  if (!ft) {
    if (wh <= 8) {
      if (d >= 56) s = 1;
    } else if (wh <= 16) {
      if (d >= 40) s = 1;
    } else if (wh <= 24) {
      if (d >= 8) s = 1;
      if (d >= 16) s = 2;
      if (d >= 32) s = 3;
    } else if (wh <= 32) {
      if (d >= 1) s = 1;
      if (d >= 4) s = 2;
      if (d >= 32) s = 3;
    } else if (d >= 1) {
      s = 3;
    }
  } else if (wh <= 8) {
    if (d >= 40) s = 1;
    if (d >= 64) s = 2;
  } else if (wh <= 16) {
    if (d >= 20) s = 1;
    if (d >= 48) s = 2;
  } else if (wh <= 24) {
    if (d >= 4) s = 3;
  } else if (d >= 1) {
    s = 3;
  }
  return s;
}
// intrapred.rs:977-1012 filter_intra_edge: every output o in 0..size-1 is the
// clamped 5-tap convolution of the unfiltered window source[k] = edge[k-1].
void filter_edge(Edge& e, int size, int strength) {
  if (strength == 0) return;
  static const int32_t K[3][5] = {{0, 4, 8, 4, 0}, {0, 5, 6, 5, 0}, {2, 4, 4, 4, 2}};
  const int32_t* k = K[strength - 1];
  int32_t src[132];
  for (int i = 0; i < size; i++) src[i] = e.at(i - 1);
  for (int o = 0; o < size - 1; o++) {
    int32_t sum = 0;
    for (int j = 0; j < 5; j++) sum += k[j] * src[clampi(o - 1 + j, 0, size - 1)];
    e.at(o) = (sum + 8) >> 4;
  }
}
// intrapred.rs:1014-1019 filter_intra_corner.
void filter_corner(Edge& above, Edge& left) {
  int32_t f = (5 * left.at(0) + 6 * above.at(-1) + 5 * above.at(0) + 8) >> 4;
  above.at(-1) = f;
  left.at(-1) = f;
}
// intrapred.rs:1021-1024 use_intra_edge_upsample.
bool use_upsample(int w, int h, bool ft, int delta) {
  int d = iabs(delta);
  return d != 0 && d < 40 && (ft ? w + h <= 8 : w + h <= 16);
}
// intrapred.rs:1026-1048 upsample_intra_edge.
void upsample_edge(Edge& e, int num_px, int bd) {
  int32_t in[136];
  in[0] = e.at(-1);
  in[1] = e.at(-1);
  for (int i = 0; i < num_px; i++) in[i + 2] = e.at(i);
  in[num_px + 2] = e.at(num_px - 1);
  e.at(-2) = in[0];
  int32_t mx = (1 << bd) - 1;
  for (int i = 0; i < num_px; i++) {
    int32_t v = -in[i] + 9 * in[i + 1] + 9 * in[i + 2] - in[i + 3];
    e.at(2 * i - 1) = clampi((v + 8) >> 4, 0, mx);
    e.at(2 * i) = in[i + 2];
  }
}
}  // namespace

extern "C" {

// intrapred.rs:1357-1594 intra_predict_nd_ad_impl (enable_edge_filter = true,
// as predict_nd_ad passes at :389) with dr_predict_scalar :629-705, paeth :1596,
// smooth :1676, smooth_v :1688, smooth_h :1700.
void or_intra_predict(const uint16_t* recon, int32_t stride, int32_t ox, int32_t oy, int32_t bw, int32_t bh,
                      int32_t mode, int32_t angle_delta, int32_t have_tr, int32_t have_bl, int32_t fw,
                      int32_t fh, int32_t filter_type, int32_t bd, int32_t* out) {
  if (mode == MT_DC_PRED) {
    int32_t d = or_dc_pred(recon, stride, ox, oy, bw, bh, bd);
    for (int i = 0; i < bw * bh; i++) out[i] = d;
    return;
  }
  Edge above, left;
  memset(&above, 0, sizeof(above));
  memset(&left, 0, sizeof(left));
  const bool have_top = oy > 0, have_left = ox > 0;
  const int32_t base = 1 << (bd - 1);
  const int edge_len = bw + bh;
  auto R = [&](int y, int x) -> int32_t { return recon[(size_t)y * stride + x]; };
  if (have_top) {
    for (int i = 0; i < bw; i++) above.at(i) = R(oy - 1, ox + i);
  } else {
    int32_t fill = have_left ? R(oy, ox - 1) : base - 1;
    for (int i = 0; i < edge_len; i++) above.at(i) = fill;
  }
  if (have_left) {
    for (int j = 0; j < bh; j++) left.at(j) = R(oy + j, ox - 1);
  } else {
    int32_t fill = have_top ? R(oy - 1, ox) : base + 1;
    for (int i = 0; i < edge_len; i++) left.at(i) = fill;
  }
  int32_t corner = have_left ? (have_top ? R(oy - 1, ox - 1) : R(oy, ox - 1)) : (have_top ? R(oy - 1, ox) : base);
  above.at(-1) = corner;
  left.at(-1) = corner;
  if (have_top) {
    int px_have = 0;
    if (have_tr) {
      int rem = fw - (ox + bw);
      if (rem < 0) rem = 0;
      px_have = bw < bh ? bw : bh;
      if (rem < px_have) px_have = rem;
    }
    for (int i = 0; i < px_have; i++) above.at(bw + i) = R(oy - 1, ox + bw + i);
    int32_t fill = above.at(bw + px_have - 1);
    for (int i = bw + px_have; i < edge_len; i++) above.at(i) = fill;
  }
  if (have_left) {
    int px_have = 0;
    if (have_bl) {
      int rem = fh - (oy + bh);
      if (rem < 0) rem = 0;
      px_have = bw < bh ? bw : bh;
      if (rem < px_have) px_have = rem;
    }
    for (int i = 0; i < px_have; i++) left.at(bh + i) = R(oy + bh + i, ox - 1);
    int32_t fill = left.at(bh + px_have - 1);
    for (int i = bh + px_have; i < edge_len; i++) left.at(i) = fill;
  }
  int angle = 0;
  switch (mode) {
    case MT_V_PRED: angle = 90; break;
    case MT_H_PRED: angle = 180; break;
    case MT_D45_PRED: angle = 45; break;
    case MT_D67_PRED: angle = 67; break;
    case MT_D135_PRED: angle = 135; break;
    case MT_D113_PRED: angle = 113; break;
    case MT_D157_PRED: angle = 157; break;
    case MT_D203_PRED: angle = 203; break;
  }
  const bool directional = mode >= MT_V_PRED && mode <= MT_D67_PRED;
  if (directional) angle += angle_delta * 3;
  int up_above = 0, up_left = 0;
  const bool ft = filter_type != 0;
  if (directional && angle != 90 && angle != 180) {
    if (angle > 90 && angle < 180 && edge_len >= 24) filter_corner(above, left);
    filter_edge(above, bw + 1 + (angle < 90 ? bh : 0), edge_filter_strength(bw, bh, ft, angle - 90));
    filter_edge(left, bh + 1 + (angle > 180 ? bw : 0), edge_filter_strength(bh, bw, ft, angle - 180));
    up_above = use_upsample(bw, bh, ft, angle - 90);
    up_left = use_upsample(bh, bw, ft, angle - 180);
    if (up_above) upsample_edge(above, bw + (angle < 90 ? bh : 0), bd);
    if (up_left) upsample_edge(left, bh + (angle > 180 ? bw : 0), bd);
  }
  if (directional && angle == 90) {
    for (int y = 0; y < bh; y++)
      for (int x = 0; x < bw; x++) out[y * bw + x] = above.at(x);
  } else if (directional && angle == 180) {
    for (int y = 0; y < bh; y++)
      for (int x = 0; x < bw; x++) out[y * bw + x] = left.at(y);
  } else if (directional && angle < 90) {
    // zone 1 (intrapred.rs:632-656)
    int dx = DR_DERIV[angle >> 1];
    int max_base_x = (edge_len - 1) << up_above;
    int frac_bits = 6 - up_above, base_inc = 1 << up_above;
    for (int y = 0; y < bh; y++) {
      int xpos = dx * (y + 1);
      int shift = ((xpos << up_above) & 0x3f) >> 1;
      int b0 = xpos >> frac_bits;
      int n_fit = 0;
      if (b0 < max_base_x) {
        n_fit = (max_base_x - b0 + base_inc - 1) / base_inc;
        if (n_fit > bw) n_fit = bw;
      }
      for (int i = 0; i < n_fit; i++) {
        int b = b0 + i * base_inc;
        out[y * bw + i] = (above.at(b) * (32 - shift) + above.at(b + 1) * shift + 16) >> 5;
      }
      for (int i = n_fit; i < bw; i++) out[y * bw + i] = above.at(max_base_x);
    }
  } else if (directional && angle > 180) {
    // zone 3 (intrapred.rs:657-676)
    int dy = DR_DERIV[(270 - angle) >> 1];
    int max_base_y = (edge_len - 1) << up_left;
    int frac_bits = 6 - up_left, base_inc = 1 << up_left;
    for (int y = 0; y < bh; y++)
      for (int x = 0; x < bw; x++) {
        int ypos = dy * (x + 1);
        int shift = ((ypos << up_left) & 0x3f) >> 1;
        int b = (ypos >> frac_bits) + y * base_inc;
        out[y * bw + x] = b >= max_base_y ? left.at(max_base_y)
                                          : (left.at(b) * (32 - shift) + left.at(b + 1) * shift + 16) >> 5;
      }
  } else if (directional) {
    // zone 2 (intrapred.rs:677-701)
    int dy = DR_DERIV[(angle - 90) >> 1];
    int dx = DR_DERIV[(180 - angle) >> 1];
    int frac_bits_y = 6 - up_left;
    for (int y = 0; y < bh; y++) {
      int t = (y + 1) * dx - 64;
      int x0 = 0;
      if (t > 0) {
        x0 = (t + 63) >> 6;
        if (x0 > bw) x0 = bw;
      }
      for (int x = 0; x < x0; x++) {
        int ypos = (y << 6) - (x + 1) * dy;
        int b = ypos >> frac_bits_y;
        int shift = ((ypos * (1 << up_left)) & 0x3f) >> 1;
        out[y * bw + x] = (left.at(b) * (32 - shift) + left.at(b + 1) * shift + 16) >> 5;
      }
      if (x0 < bw) {
        int xpos = (x0 << 6) - (y + 1) * dx;
        int b0 = xpos >> (6 - up_above);
        int shift = ((xpos * (1 << up_above)) & 0x3f) >> 1;
        for (int i = 0; i < bw - x0; i++) {
          int b = b0 + i * (1 << up_above);
          out[y * bw + x0 + i] = (above.at(b) * (32 - shift) + above.at(b + 1) * shift + 16) >> 5;
        }
      }
    }
  } else if (mode == MT_PAETH_PRED) {
    for (int y = 0; y < bh; y++)
      for (int x = 0; x < bw; x++) {
        int32_t lv = left.at(y), tv = above.at(x);
        int32_t b = lv + tv - corner;
        int32_t ld = iabs(lv - b), td = iabs(tv - b), cd = iabs(corner - b);
        out[y * bw + x] = (ld <= td && ld <= cd) ? lv : (td <= cd ? tv : corner);
      }
  } else if (mode == MT_SMOOTH_PRED) {
    const int32_t *wv = sm_weights(bh), *wh = sm_weights(bw);
    int32_t right = above.at(bw - 1), bottom = left.at(bh - 1);
    for (int y = 0; y < bh; y++)
      for (int x = 0; x < bw; x++) {
        int32_t p = wv[y] * above.at(x) + (256 - wv[y]) * bottom + wh[x] * left.at(y) + (256 - wh[x]) * right;
        out[y * bw + x] = (p + 256) >> 9;
      }
  } else if (mode == MT_SMOOTH_V_PRED) {
    const int32_t* wv = sm_weights(bh);
    int32_t bottom = left.at(bh - 1);
    for (int y = 0; y < bh; y++)
      for (int x = 0; x < bw; x++) out[y * bw + x] = (wv[y] * above.at(x) + (256 - wv[y]) * bottom + 128) >> 8;
  } else if (mode == MT_SMOOTH_H_PRED) {
    const int32_t* wh = sm_weights(bw);
    int32_t right = above.at(bw - 1);
    for (int y = 0; y < bh; y++)
      for (int x = 0; x < bw; x++) out[y * bw + x] = (wh[x] * left.at(y) + (256 - wh[x]) * right + 128) >> 8;
  }
}

// partition_rd.rs:86-133 luma_satd_scalar.
// rd_sse.rs:630-655 luma_satd: outside the visible window (vis_w x vis_h from
// the block origin) the source is replaced by the reconstruction.
static uint64_t luma_satd_vis(const uint16_t* src, int32_t stride, int32_t px, int32_t py, int32_t w, int32_t h,
                              int32_t maxv, const int32_t* pred, const int32_t* resid, int32_t vis_w, int32_t vis_h);

uint64_t or_luma_satd(const uint16_t* src, int32_t stride, int32_t px, int32_t py, int32_t w, int32_t h,
                      int32_t maxv, const int32_t* pred, const int32_t* resid) {
  return luma_satd_vis(src, stride, px, py, w, h, maxv, pred, resid, w, h);
}

static uint64_t luma_satd_vis(const uint16_t* src, int32_t stride, int32_t px, int32_t py, int32_t w, int32_t h,
                              int32_t maxv, const int32_t* pred, const int32_t* resid, int32_t vis_w, int32_t vis_h) {
  std::vector<int32_t> err((size_t)w * h);
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      int i = y * w + x;
      int32_t r = pred[i] + (resid ? resid[i] : 0);
      err[i] = (x < vis_w && y < vis_h) ? (int32_t)src[(size_t)(py + y) * stride + px + x] - clampi(r, 0, maxv) : 0;
    }
  uint64_t satd = 0;
  for (int ty = 0; ty < h; ty += 4)
    for (int tx = 0; tx < w; tx += 4) {
      int32_t rows[4][4];
      for (int y = 0; y < 4; y++) {
        const int32_t* d = &err[(size_t)(ty + y) * w + tx];
        int32_t e = d[0] + d[2], f = d[0] - d[2], g = d[1] + d[3], hh = d[1] - d[3];
        rows[y][0] = e + g;
        rows[y][1] = f + hh;
        rows[y][2] = f - hh;
        rows[y][3] = e - g;
      }
      for (int x = 0; x < 4; x++) {
        int32_t a = rows[0][x], b = rows[1][x], c = rows[2][x], d = rows[3][x];
        int32_t e = a + c, f = a - c, g = b + d, hh = b - d;
        satd += uabs(e + g) + uabs(f + hh) + uabs(f - hh) + uabs(e - g);
      }
    }
  return satd;
}

// cost.rs:156-169 cost_q_table (glibc log2f, Q22) and :184-190 cdf_cost_with_table.
static uint32_t* cost_q_table() {
  static uint32_t* t = [] {
    uint32_t* tab = (uint32_t*)calloc(32769, sizeof(uint32_t));
    for (int p = 1; p <= 32768; p++) {
      float bits = -log2f((float)p * (1.0f / 32768.0f));
      tab[p] = (uint32_t)roundf(bits * (float)(1u << 22));
    }
    return tab;
  }();
  return t;
}
float or_cdf_cost(const uint16_t* cdf, int32_t s) {
  int32_t fl = s > 0 ? cdf[s - 1] : 32768;
  int32_t fh = cdf[s];
  int32_t p = fl - fh;
  if (p < 1) p = 1;
  return (float)cost_q_table()[p] * (1.0f / (float)(1u << 22));
}
}  // extern "C"

namespace {
// tables.rs:365-373 level_byte.
inline uint8_t level_byte(uint32_t m) {
  if (m == 0) return 0;
  if (m <= 2) return (uint8_t)(m * 0x41);
  return (uint8_t)((m < 15 ? m : 15) + (3u << 6));
}
// cost.rs:196-200 golomb_cost.
inline float golomb_cost(uint32_t v) { return (float)(2 * (32 - lzcnt32(v + 1)) - 1); }
// cost.rs:244-262 hi_tok_cost_with_table.
float hi_tok_cost(uint32_t m, const uint16_t* br) {
  int32_t total_br = (int32_t)m - 3;
  if (total_br > 12) total_br = 12;
  int32_t coded = 0;
  float bits = 0.0f;
  for (int k = 0; k < 4; k++) {
    int32_t s = total_br - coded;
    if (s > 3) s = 3;
    bits += or_cdf_cost(br, s);
    coded += s;
    if (s < 3) break;
  }
  if (m >= 15) bits += golomb_cost(m - 15);
  return bits;
}
}  // namespace

extern "C" {

// rate.rs:149-291 real_block_bits_bounded (bound = +inf) for a w x h block,
// with the CDF costs evaluated directly (the CoefCostTables cache at
// rate.rs:58-80 holds the same values).  txtp_mode < 0: no transform-type
// symbol (chroma, TX_32X32).  Contexts: the square, w < h or w > h lo-context
// offset table (src/tables.rs:354-360, :456-472).
// `bound`: the exact abort of rate.rs:149-157 -- +inf once the running sum
// passes it after the eob position (:208-210) or at every 16th interior index
// (:234-236).
float or_real_block_bits_bounded(const int32_t* cf, const uint16_t* scan, int32_t w, int32_t h,
                                 const mt_coef_cdfs* c, int32_t skip_ctx, int32_t dcs_ctx, int32_t txtp_mode,
                                 int32_t txtp, int32_t use_skip_bits, const float* skip_bits, float bound) {
  const int N = w * h;
  int eob = -1;
  for (int i = N - 1; i >= 0; i--)
    if (cf[scan[i]] != 0) {
      eob = i;
      break;
    }
  if (eob < 0) return use_skip_bits ? skip_bits[0] : or_cdf_cost(c->txb_skip[skip_ctx], 1);
  float bits = use_skip_bits ? skip_bits[1] : or_cdf_cost(c->txb_skip[skip_ctx], 0);
  if (txtp_mode >= 0) bits += or_cdf_cost(c->txtp[txtp_mode], txtp);
  const uint16_t* dc_sign = c->dc_sign[dcs_ctx];
  if (eob == 0) {
    uint32_t m = uabs(cf[0]);
    uint32_t mm = m < 3 ? m : 3;
    bits += or_cdf_cost(c->eob_bin, 0);
    bits += or_cdf_cost(c->eob_base[0], (int)mm - 1);
    if (mm == 3) bits += hi_tok_cost(m, c->br_tok[0]);
    bits += or_cdf_cost(dc_sign, cf[0] < 0 ? 1 : 0);
    return bits;
  }
  int eob_bin = eob < 2 ? eob : 32 - lzcnt32((uint32_t)eob);
  bits += or_cdf_cost(c->eob_bin, eob_bin);
  if (eob_bin > 1) {
    int nbits = eob_bin - 2;
    bits += or_cdf_cost(c->eob_hi[eob_bin], (eob >> nbits) & 1);
    bits += (float)nbits;
  }
  if (bits > bound) return INFINITY;
  static const uint8_t kOffWlh[25] = {0, 11, 11, 11, 11, 11, 11, 11, 11, 11, 6, 6, 21,
                                        21, 21, 6, 21, 21, 21, 21, 21, 21, 21, 21, 21};
  static const uint8_t kOffWgh[25] = {0, 16, 6, 6, 21, 16, 16, 6, 21, 21, 16, 16, 21,
                                        21, 21, 16, 16, 21, 21, 21, 16, 16, 21, 21, 21};
  const int stride = h;
  const int log2h = __builtin_ctz((unsigned)h);
  std::vector<uint8_t> levels((size_t)(w + 2) * (h + 2), 0);
  auto lo_ctx = [&](int x, int y, uint32_t* hi_mag) -> int {
    auto g = [&](int dx, int dy) -> uint32_t { return levels[(size_t)(x + dx) * stride + (y + dy)]; };
    uint32_t hm = g(0, 1) + g(1, 0) + g(1, 1);
    uint32_t mag = hm + g(0, 2) + g(2, 0);
    int yy = y < 4 ? y : 4, xx = x < 4 ? x : 4;
    int off = w < h ? kOffWlh[yy * 5 + xx] : (w > h ? kOffWgh[yy * 5 + xx] : MT_LO_CTX_OFF[yy * 5 + xx]);
    *hi_mag = hm;
    return off + (mag > 512 ? 4 : (int)((mag + 64) >> 7));
  };
  int ctx_e = 1 + (eob > (N >> 3) ? 1 : 0) + (eob > (N >> 2) ? 1 : 0);
  {
    int rc = scan[eob];
    int ex = rc >> log2h, ey = rc & (h - 1);
    uint32_t m = uabs(cf[rc]);
    uint32_t tok = (m < 3 ? m : 3) - 1;
    bits += or_cdf_cost(c->eob_base[ctx_e], (int)tok);
    if (tok == 2) {
      int bc = (ex | ey) > 1 ? 14 : 7;
      bits += hi_tok_cost(m, c->br_tok[bc]);
    }
    levels[(size_t)ex * stride + ey] = level_byte(m);
  }
  int ac_nonzero = 1;
  for (int i = eob - 1; i >= 1; i--) {
    if ((i & 15) == 0 && bits > bound) return INFINITY;
    int rc = scan[i];
    int x = rc >> log2h, y = rc & (h - 1);
    uint32_t hi_mag;
    int ctx = lo_ctx(x, y, &hi_mag);
    uint32_t m = uabs(cf[rc]);
    uint32_t tok = m < 3 ? m : 3;
    bits += or_cdf_cost(c->base_tok[ctx], (int)tok);
    if (tok == 3) {
      uint32_t mag = hi_mag & 63;
      int bc = ((y | x) > 1 ? 14 : 7) + (mag > 12 ? 6 : (int)((mag + 1) >> 1));
      // rate.rs:255-262: cached ladder br_cum[bc][total_br] then the Golomb tail.
      int32_t total_br = (int32_t)m - 3;
      if (total_br > 12) total_br = 12;
      float ladder = 0.0f;
      {
        int32_t coded = 0;
        for (int k = 0; k < 4; k++) {
          int32_t s = total_br - coded;
          if (s > 3) s = 3;
          ladder += or_cdf_cost(c->br_tok[bc], s);
          coded += s;
          if (s < 3) break;
        }
      }
      bits += ladder;
      if (m >= 15) bits += golomb_cost(m - 15);
    }
    if (m != 0) {
      levels[(size_t)x * stride + y] = level_byte(m);
      ac_nonzero++;
    }
  }
  uint32_t dm = uabs(cf[0]);
  uint32_t dtok = dm < 3 ? dm : 3;
  bits += or_cdf_cost(c->base_tok[0], (int)dtok);
  if (dtok == 3) {
    uint32_t mag = ((uint32_t)levels[1] + levels[stride] + levels[stride + 1]) & 63;
    int bc = mag > 12 ? 6 : (int)((mag + 1) >> 1);
    bits += hi_tok_cost(dm, c->br_tok[bc]);
  }
  if (cf[0] != 0) bits += or_cdf_cost(dc_sign, cf[0] < 0 ? 1 : 0);
  for (int k = 0; k < ac_nonzero; k++) bits += 1.0f;
  return bits;
}

float or_real_block_bits_wh(const int32_t* cf, const uint16_t* scan, int32_t w, int32_t h,
                            const mt_coef_cdfs* c, int32_t skip_ctx, int32_t dcs_ctx, int32_t txtp_mode,
                            int32_t txtp, int32_t use_skip_bits, const float* skip_bits) {
  return or_real_block_bits_bounded(cf, scan, w, h, c, skip_ctx, dcs_ctx, txtp_mode, txtp, use_skip_bits, skip_bits,
                                    INFINITY);
}

// The square luma form the candidate chain prices (TX_32X32 codes no txtp).
float or_real_block_bits(const int32_t* cf, const uint16_t* scan, int32_t n, int32_t cls,
                         const mt_coef_cdfs* c, int32_t skip_ctx, int32_t dcs_ctx, int32_t y_mode,
                         int32_t txtp, int32_t use_skip_bits, const float* skip_bits) {
  return or_real_block_bits_wh(cf, scan, n, n, c, skip_ctx, dcs_ctx, cls < 3 ? y_mode : -1, txtp, use_skip_bits,
                               skip_bits);
}

// rate.rs:58-80 CoefCostTables::build plus the per-symbol costs of the other
// CDFs of the slice; br_cum rows follow cost.rs:214-241 br_cum_row_with_table.
void or_coef_costs_build(const mt_coef_cdfs* c, mt_coef_costs* o) {
  memset(o, 0, sizeof(*o));
  for (int k = 0; k < 13; k++)
    for (int s = 0; s < 2; s++) o->txb_skip[k][s] = or_cdf_cost(c->txb_skip[k], s);
  for (int k = 0; k < 42; k++)
    for (int s = 0; s < 4; s++) o->base_tok[k][s] = or_cdf_cost(c->base_tok[k], s);
  for (int k = 0; k < 21; k++) {
    float cc[4];
    for (int s = 0; s < 4; s++) cc[s] = or_cdf_cost(c->br_tok[k], s);
    float c3x2 = cc[3] + cc[3], c3x3 = c3x2 + cc[3], c3x4 = c3x3 + cc[3];
    float row[13] = {cc[0],        cc[1],        cc[2],        cc[3] + cc[0], cc[3] + cc[1],
                     cc[3] + cc[2], c3x2 + cc[0], c3x2 + cc[1], c3x2 + cc[2], c3x3 + cc[0],
                     c3x3 + cc[1], c3x3 + cc[2], c3x4};
    memcpy(o->br_cum[k], row, sizeof(row));
  }
  for (int k = 0; k < 4; k++)
    for (int s = 0; s < 3; s++) o->eob_base[k][s] = or_cdf_cost(c->eob_base[k], s);
  for (int k = 0; k < 11; k++)
    for (int s = 0; s < 2; s++) o->eob_hi[k][s] = or_cdf_cost(c->eob_hi[k], s);
  for (int s = 0; s < 11; s++) o->eob_bin[s] = or_cdf_cost(c->eob_bin, s);
  for (int k = 0; k < 3; k++)
    for (int s = 0; s < 2; s++) o->dc_sign[k][s] = or_cdf_cost(c->dc_sign[k], s);
  for (int m = 0; m < 13; m++)
    for (int s = 0; s < 16; s++) o->txtp[m][s] = or_cdf_cost(c->txtp[m], s);
  for (int s = 0; s < 11; s++) o->eob_bin_1d[s] = or_cdf_cost(c->eob_bin_1d, s);
}

// partition_search.rs:467-530 (8x8) / :620-673 (16x16): predict (DC via
// dc_pred_NxN, else predict_nd_ad)
// -> residual_pred -> forward transform + quant (+QM) -> trellis_optimize ->
// inverse -> luma_partition_distortion (lossy_state.rs:2385-2409) -> luma_bits
// (lossy_state.rs:477-572) + mode_bits -> partition_rd::rd_cost.
static void chain_one(const uint16_t* src, const uint16_t* recon, const mt_chain_params* p, const mt_quant* q,
                      const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_candidate& cd, mt_candidate_result* r,
                      int32_t* lv_out, int32_t* rec_out) {
  const int n = p->tx_size, N = n * n;
  int32_t pred[256], resid[256], cf[256], rr[256];
  float tf[256];
  or_intra_predict(recon, p->stride, cd.px, cd.py, n, n, cd.mode, cd.angle_delta, (cd.flags & 1) != 0,
                   (cd.flags & 2) != 0, p->frame_w, p->frame_h, (cd.flags & 4) != 0, p->bd, pred);
  for (int y = 0; y < n; y++)
    for (int x = 0; x < n; x++)
      resid[y * n + x] = (int32_t)src[(size_t)(cd.py + y) * p->stride + cd.px + x] - pred[y * n + x];
  or_fwd_txfm_quant(resid, cd.tx_type, n, q, qm, cf, tf);
  const uint16_t* scan = or_default_scan(n);
  if (!(cd.flags & MT_CAND_NO_TRELLIS))
    or_trellis_optimize(cf, tf, (float)q->dc_q, (float)q->ac_q, scan, N, p->trellis_lambda0);
  or_inv_txfm_dequant(cf, cd.tx_type, n, q, qm, rr);
  const int32_t maxv = (1 << p->bd) - 1;
  const int32_t vis_w = (p->vis_w > 0 ? p->vis_w : p->frame_w) - cd.px;
  const int32_t vis_h = (p->vis_h > 0 ? p->vis_h : p->frame_h) - cd.py;
  uint64_t satd = luma_satd_vis(src, p->stride, cd.px, cd.py, n, n, maxv, pred, rr, vis_w, vis_h);
  float qstep = (float)q->ac_q;
  float price = (float)satd * (qstep > 1.0f ? qstep : 1.0f) * 0.25f * p->satd_scale;
  if (p->satd_bridge != 0.0f) price *= p->satd_bridge;
  const int cls = n == 4 ? 0 : (n == 8 ? 1 : (n == 16 ? 2 : 3));
  float bits = or_real_block_bits(cf, scan, n, cls, cdfs, cd.skip_ctx, cd.dcs_ctx, cd.mode, cd.tx_type,
                                  p->use_skip_bits, p->skip_bits) +
               cd.mode_bits + cd.extra_bits;
  r->distortion = price;
  r->bits = bits;
  r->cost = price + p->mode_lambda * bits;
  r->satd = (uint32_t)satd;
  int eob = -1;
  for (int i = N - 1; i >= 0; i--)
    if (cf[scan[i]] != 0) {
      eob = i;
      break;
    }
  r->eob = eob;
  r->reserved[0] = r->reserved[1] = r->reserved[2] = 0;
  if (lv_out) memcpy(lv_out, cf, sizeof(int32_t) * N);
  if (rec_out)
    for (int i = 0; i < N; i++) rec_out[i] = clampi(pred[i] + rr[i], 0, maxv);
}

// partition_search.rs:187-238 proxy_mode_beam's ranking: the 11 nd_modes
// (intrapred.rs:1712-1724) predicted at delta 0, scored by satd_sad_proxy
// (rd_sse.rs:559-589, :1143-1176; samples past the displayed window taken as
// the prediction), sorted by (score, mode).
int or_mode_beam(const uint16_t* src, const uint16_t* recon, const mt_chain_params* p, const mt_block8* blocks,
                 int32_t nblocks, uint64_t* scores, uint8_t* modes) {
  static const int ND[11] = {MT_DC_PRED,   MT_V_PRED,    MT_H_PRED,    MT_D45_PRED,    MT_D135_PRED, MT_D113_PRED,
                             MT_D157_PRED, MT_D203_PRED, MT_D67_PRED,  MT_SMOOTH_PRED, MT_PAETH_PRED};
  const int n = p->tx_size;
  std::vector<int32_t> pred((size_t)n * n);
  for (int b = 0; b < nblocks; b++) {
    const mt_block8& bk = blocks[b];
    if (bk.px + n > p->frame_w || bk.py + n > p->frame_h) {
      for (int k = 0; k < 11; k++) {
        if (scores) scores[(size_t)b * 11 + k] = UINT64_MAX;
        modes[(size_t)b * 11 + k] = 255;
      }
      continue;
    }
    const int vw = (p->vis_w > 0 ? p->vis_w : p->frame_w) - bk.px;
    const int vh = (p->vis_h > 0 ? p->vis_h : p->frame_h) - bk.py;
    std::vector<std::pair<uint64_t, int>> ranked;
    for (int m : ND) {
      or_intra_predict(recon, p->stride, bk.px, bk.py, n, n, m, 0, (bk.flags & 1) != 0, (bk.flags & 2) != 0,
                       p->frame_w, p->frame_h, (bk.flags & 4) != 0, p->bd, pred.data());
      uint64_t sad = 0, satd = 0;
      for (int ty = 0; ty < n; ty += 4)
        for (int tx = 0; tx < n; tx += 4) {
          int32_t rows[4][4];
          for (int r = 0; r < 4; r++) {
            int32_t d[4];
            for (int x = 0; x < 4; x++) {
              const bool vis = tx + x < vw && ty + r < vh;
              d[x] = vis ? (int32_t)src[(size_t)(bk.py + ty + r) * p->stride + bk.px + tx + x] -
                               pred[(size_t)(ty + r) * n + tx + x]
                         : 0;
              sad += uabs(d[x]);
            }
            const int32_t e = d[0] + d[2], f = d[0] - d[2], g = d[1] + d[3], h = d[1] - d[3];
            rows[r][0] = e + g;
            rows[r][1] = f + h;
            rows[r][2] = f - h;
            rows[r][3] = e - g;
          }
          for (int x = 0; x < 4; x++) {
            const int32_t a = rows[0][x], bb = rows[1][x], c = rows[2][x], dd = rows[3][x];
            const int32_t e = a + c, f = a - c, g = bb + dd, h = bb - dd;
            satd += (uint64_t)uabs(e + g) + uabs(f + h) + uabs(f - h) + uabs(e - g);
          }
        }
      ranked.emplace_back(sad + (satd >> 2), m);
    }
    std::sort(ranked.begin(), ranked.end());
    for (int k = 0; k < 11; k++) {
      if (scores) scores[(size_t)b * 11 + k] = ranked[k].first;
      modes[(size_t)b * 11 + k] = (uint8_t)ranked[k].second;
    }
  }
  return MT_OK;
}

// The forward 1-D integer DCT of n = 4, 8 or 16 points in place (dct.rs:175-276).
void or_dct1d(int32_t* buf, int32_t n) {
  if (n == 4) dct1d_4(buf);
  if (n == 8) dct1d_8(buf);
  if (n == 16) dct1d_16(buf);
}

int or_candidate_chain(const uint16_t* src, const uint16_t* recon, const mt_chain_params* p, const mt_quant* q,
                       const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_candidate* cands, int32_t n,
                       mt_candidate_result* results, int32_t* levels_out, int32_t* recon_out, int32_t threads) {
  if (!p || (p->tx_size != 8 && p->tx_size != 4 && p->tx_size != 16)) return MT_ERR_UNSUPPORTED;
  const int N = p->tx_size * p->tx_size;
  auto work = [&](int lo, int hi) {
    for (int i = lo; i < hi; i++)
      chain_one(src, recon, p, q, qm, cdfs, cands[i], &results[i], levels_out ? levels_out + (size_t)i * N : nullptr,
                recon_out ? recon_out + (size_t)i * N : nullptr);
  };
  if (threads <= 1 || n < 64) {
    work(0, n);
    return MT_OK;
  }
  std::vector<std::thread> pool;
  int per = (n + threads - 1) / threads;
  for (int t = 0; t < threads; t++) {
    int lo = t * per, hi = lo + per < n ? lo + per : n;
    if (lo >= hi) break;
    pool.emplace_back(work, lo, hi);
  }
  for (auto& th : pool) th.join();
  return MT_OK;
}

}  // extern "C"

extern "C" {
// Exposed for the known-answer tests of intrapred.rs:2481-2496.
int or_edge_filter_strength(int w, int h, int filter_type, int delta) {
  return edge_filter_strength(w, h, filter_type != 0, delta);
}
int or_use_edge_upsample(int w, int h, int filter_type, int delta) { return use_upsample(w, h, filter_type != 0, delta); }
}
