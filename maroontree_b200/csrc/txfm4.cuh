// Device 4x4 transforms of the luma candidate chain: forward transforms with
// quantisation and dequantisation + inverse transforms, in the reference's
// integer arithmetic (building blocks shared with the 8x8 path in txfm8.cuh).
#pragma once
#include <stdint.h>

#include "txfm8.cuh"

namespace mtd {

// Forward 4-point ADST as a Q12 matrix product (src/dct.rs:1368-1383); the
// reference accumulates in i64, and for residuals of 8-bit samples no partial
// sum of either pass leaves +-2^31 (row sums of |A| <= 15487, first-pass
// outputs <= ~1.5k), so i32 accumulation gives the same value.
__constant__ int16_t kAdst4Fwd[16] = {1868, 3510, 4730, 5379, 4730, 4730,  0,    -4730,
                                      5379, -1868, -4730, 3510, 3510, -5379, 4730, -1868};
__device__ __forceinline__ void fadst4(int32_t* v) {
  int32_t o[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    int32_t acc = 2048;
#pragma unroll
    for (int j = 0; j < 4; j++) acc += (int32_t)kAdst4Fwd[i * 4 + j] * v[j];
    o[i] = acc >> 12;
  }
#pragma unroll
  for (int i = 0; i < 4; i++) v[i] = o[i];
}
__device__ __forceinline__ void fdct4v(int32_t* v) { fdct4(v[0], v[1], v[2], v[3]); }

// Forward 4x4 transform + quantisation of a row-major residual into
// column-major levels and f32 targets: the 2-D types columns first then rows
// with the Q16 multipliers x 8/sqrt(16) = 2 (src/dct.rs:3076-3100, :1398-1470,
// :2465-2488); V/H_DCT the 1-D DCT x 2 sqrt2 with full-step quantisation
// (src/dct.rs:391-431); IDTX num*8/q (src/dct.rs:1586-1615).  The QM step of
// the 2-D types is applied by the caller.
template <typename I, typename C>
__device__ void fwd4x4(const I* __restrict__ in, int tx, const mt_quant& q, C* __restrict__ cf,
                       float* __restrict__ tf, int32_t* __restrict__ t) {
  if (tx == MT_TX_IDTX) {
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const int y = i >> 2, x = i & 3, rc = y + x * 4;
      const int32_t qd = rc == 0 ? q.dc_q : q.ac_q;
      const int32_t num = in[i] * 8;
      tf[rc] = __fdiv_rn((float)num, (float)qd);
      const int32_t am = (int32_t)uabs(num);
      const int32_t level = (am + qd / 2) / qd;
      cf[rc] = (C)(am < qd ? 0 : (num < 0 ? -level : level));
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < 16; i++) t[i] = in[i];
  if (tx == MT_TX_V_DCT || tx == MT_TX_H_DCT) {
    if (tx == MT_TX_V_DCT) {
#pragma unroll
      for (int x = 0; x < 4; x++) {
        int32_t v[4] = {t[x], t[4 + x], t[8 + x], t[12 + x]};
        fdct4v(v);
#pragma unroll
        for (int y = 0; y < 4; y++) t[y * 4 + x] = mul_q16(v[y] * 2, 92682);
      }
    } else {
#pragma unroll
      for (int y = 0; y < 4; y++) {
        fdct4v(t + y * 4);
#pragma unroll
        for (int x = 0; x < 4; x++) t[y * 4 + x] = mul_q16(t[y * 4 + x] * 2, 92682);
      }
    }
#pragma unroll
    for (int y = 0; y < 4; y++)
#pragma unroll
      for (int x = 0; x < 4; x++) {
        const int rc = y + x * 4;
        int32_t lv;
        quant_fullstep(t[y * 4 + x], rc == 0 ? q.q_mult_dc : q.q_mult_ac, &lv, &tf[rc]);
        cf[rc] = (C)lv;
      }
    return;
  }
  const int32_t mdc = mul_q16(q.q_mult_dc, 131072), mac = mul_q16(q.q_mult_ac, 131072);
  const int ck = col_kind(tx), rk = row_kind(tx);
#pragma unroll
  for (int x = 0; x < 4; x++) {
    int32_t v[4] = {t[x], t[4 + x], t[8 + x], t[12 + x]};
    if (ck == 1) fdct4v(v); else fadst4(v);
#pragma unroll
    for (int r = 0; r < 4; r++) t[r * 4 + x] = v[r];
  }
#pragma unroll
  for (int r = 0; r < 4; r++) {
    int32_t* v = t + r * 4;
    if (rk == 1) fdct4v(v); else fadst4(v);
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int idx = u * 4 + r;
      const int32_t m = idx == 0 ? mdc : mac;
      cf[idx] = (C)quant_q16(v[u], m);
      tf[idx] = __fmul_rn(__fmul_rn((float)v[u], (float)m), 1.0f / 65536.0f);
    }
  }
}

// Inverse 4-point ADST, dav1d form without clamps (src/idct.rs:2837-2865), and
// the identity4 step i + (i * 1697 + 2048) >> 12 (src/idct.rs:2719-2748).
__device__ __forceinline__ void iadst4s(int32_t* c, int s) {
  const int32_t in0 = c[0], in1 = c[s], in2 = c[2 * s], in3 = c[3 * s];
  const int32_t o0 =
      ((1321 * in0 + (3803 - 4096) * in2 + (2482 - 4096) * in3 + (3344 - 4096) * in1 + 2048) >> 12) + in2 + in3 + in1;
  const int32_t o1 =
      (((2482 - 4096) * in0 - 1321 * in2 - (3803 - 4096) * in3 + (3344 - 4096) * in1 + 2048) >> 12) + in0 - in3 + in1;
  const int32_t o2 = (209 * (in0 - in2 + in3) + 128) >> 8;
  const int32_t o3 =
      (((3803 - 4096) * in0 + (2482 - 4096) * in2 - 1321 * in3 - (3344 - 4096) * in1 + 2048) >> 12) + in0 + in2 - in1;
  c[0] = o0;
  c[s] = o1;
  c[2 * s] = o2;
  c[3 * s] = o3;
}
__device__ __forceinline__ int32_t iid4(int32_t i) { return i + ((i * 1697 + 2048) >> 12); }

// Dequantisation and the 4x4 inverses (src/idct.rs:2719-2948): tmp[y*4+x] =
// coeff[y + x*4]; row pass (DCT clamped to the row range), the column clamp
// with no inter-pass shift, column pass, (t+8)>>4.  The identity family
// dequantises flat.
template <typename C, typename O>
__device__ void inv4x4(const C* __restrict__ cf, int tx, const mt_quant& q, const uint8_t* __restrict__ qm,
                       O* __restrict__ out, int32_t* __restrict__ t) {
  const bool flat = tx == MT_TX_IDTX || tx == MT_TX_V_DCT || tx == MT_TX_H_DCT;
  const uint8_t* w = flat ? nullptr : qm;
#pragma unroll
  for (int rc = 0; rc < 16; rc++) {
    const int32_t l = cf[rc];
    const int32_t base = rc == 0 ? q.dc_q : q.ac_q;
    const int32_t step = w ? ((base * (int32_t)w[rc] + 16) >> 5) : base;
    int32_t mag = (int32_t)((uabs(l) * (uint32_t)step) & 0xffffffu);
    mag = min(mag, q.cf_max + (l < 0 ? 1 : 0));
    const int y = rc & 3, x = rc >> 2;
    t[y * 4 + x] = l == 0 ? 0 : (l < 0 ? -mag : mag);
  }
  const int ck = col_kind(tx), rk = row_kind(tx);
#pragma unroll
  for (int y = 0; y < 4; y++) {
    if (rk == 1) idct4s(t + y * 4, 1, q.rmin, q.rmax);
    else if (rk == 2) iadst4s(t + y * 4, 1);
    else
#pragma unroll
      for (int x = 0; x < 4; x++) t[y * 4 + x] = iid4(t[y * 4 + x]);
  }
#pragma unroll
  for (int i = 0; i < 16; i++) t[i] = clampi(t[i], q.cmin, q.cmax);
#pragma unroll
  for (int x = 0; x < 4; x++) {
    if (ck == 1) idct4s(t + x, 4, q.cmin, q.cmax);
    else if (ck == 2) iadst4s(t + x, 4);
    else
#pragma unroll
      for (int y = 0; y < 4; y++) t[y * 4 + x] = iid4(t[y * 4 + x]);
  }
#pragma unroll
  for (int i = 0; i < 16; i++) out[i] = (O)((t[i] + 8) >> 4);
}

}  // namespace mtd
