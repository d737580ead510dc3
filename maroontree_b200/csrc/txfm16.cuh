// Device 16x16 transforms of the luma candidate chain: forward transforms with
// quantisation (the reference's integer butterflies and Q12 ADST matrix) and
// the dav1d inverses, for DCT_DCT, ADST_ADST, ADST_DCT, DCT_ADST and IDTX.
#pragma once
#include <stdint.h>

#include "av1_tables.h"
#include "txfm8.cuh"

namespace mtd {

// Odd-half weights of the 16-point forward DCT, round(65536 / (2 cos((2k+1) pi / 32)))
// (src/dct.rs:224-238).
__constant__ int32_t kWc16[8] = {32927, 34242, 37155, 42390, 51653, 69513, 112882, 334309};
// The forward 16-point ADST as a Q12 matrix (src/dct.rs:445-523).
__constant__ int16_t kAdst16Fwd[256] = {MT_ADST16_FWD_Q12_LIST};

// dct1d_16_i32 (src/dct.rs:241-276): even/odd split, 8-point DCTs of both
// halves (the odd one after the WC16 weights), the odd running combine.
__device__ __forceinline__ void fdct16(int32_t* v) {
  int32_t t[16];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    t[i] = v[i] + v[15 - i];
    t[8 + i] = v[i] - v[15 - i];
  }
  fdct8(t);
#pragma unroll
  for (int i = 0; i < 8; i++) t[8 + i] = mul_q16(t[8 + i], kWc16[i]);
  fdct8(t + 8);
  t[8] = mul_q16(t[8], 92682) + t[9];
#pragma unroll
  for (int i = 9; i < 15; i++) t[i] += t[i + 1];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    v[2 * i] = t[i];
    v[2 * i + 1] = t[8 + i];
  }
}

// fwd_adst16_1d: (sum_j A[i][j] v[j] + 2048) >> 12.  The reference sums in
// i64; for residuals of 8-bit samples the row sums of |A| bound both passes
// well inside i32 (checked from the table by the tests).
__device__ __forceinline__ void fadst16(int32_t* v) {
  int32_t o[16];
#pragma unroll 4
  for (int i = 0; i < 16; i++) {
    int32_t acc = 2048;
#pragma unroll
    for (int j = 0; j < 16; j++) acc += (int32_t)kAdst16Fwd[i * 16 + j] * v[j];
    o[i] = acc >> 12;
  }
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = o[i];
}

// Forward 16x16 transform + quantisation of a row-major residual into
// column-major levels and f32 targets (src/dct.rs:557-580, :1295-1392): the
// columns then the rows, each output halved by mul_q16(x, 32768), quantised
// with the quantiser's own Q16 multipliers.  IDTX: num*8/q (src/dct.rs:1586-1633).
// The QM step of the 2-D types is applied by the caller.
template <typename I, typename C>
__device__ void fwd16x16(const I* __restrict__ in, int tx, const mt_quant& q, C* __restrict__ cf,
                         float* __restrict__ tf, int32_t* __restrict__ t) {
  if (tx == MT_TX_IDTX) {
#pragma unroll 4
    for (int i = 0; i < 256; i++) {
      const int y = i >> 4, x = i & 15, rc = y + x * 16;
      const int32_t qd = rc == 0 ? q.dc_q : q.ac_q;
      const int32_t num = in[i] * 8;
      tf[rc] = __fdiv_rn((float)num, (float)qd);
      const int32_t am = (int32_t)uabs(num);
      const int32_t level = (am + qd / 2) / qd;
      cf[rc] = (C)(am < qd ? 0 : (num < 0 ? -level : level));
    }
    return;
  }
  const bool col_adst = tx == MT_TX_ADST_ADST || tx == MT_TX_ADST_DCT;
  const bool row_adst = tx == MT_TX_ADST_ADST || tx == MT_TX_DCT_ADST;
#pragma unroll 1
  for (int x = 0; x < 16; x++) {
    int32_t v[16];
#pragma unroll
    for (int r = 0; r < 16; r++) v[r] = in[r * 16 + x];
    if (col_adst) fadst16(v); else fdct16(v);
#pragma unroll
    for (int r = 0; r < 16; r++) t[r * 16 + x] = v[r];
  }
#pragma unroll 1
  for (int r = 0; r < 16; r++) {
    int32_t v[16];
#pragma unroll
    for (int u = 0; u < 16; u++) v[u] = t[r * 16 + u];
    if (row_adst) fadst16(v); else fdct16(v);
#pragma unroll
    for (int u = 0; u < 16; u++) {
      const int idx = u * 16 + r;
      const int32_t m = idx == 0 ? q.q_mult_dc : q.q_mult_ac;
      const int32_t c = mul_q16(v[u], 32768);
      cf[idx] = (C)quant_q16(c, m);
      tf[idx] = __fmul_rn(__fmul_rn((float)c, (float)m), 1.0f / 65536.0f);
    }
  }
}

// One dav1d rotation, (x * cx + y * cy + 2048) >> 12 (the reference's forms
// with a constant minus 4096, or halved constants and >> 11, are equal).
__device__ __forceinline__ int32_t rot12(int32_t x, int32_t cx, int32_t y, int32_t cy) {
  return (x * cx + y * cy + 2048) >> 12;
}
__device__ __forceinline__ int32_t r181(int32_t v) { return (v * 181 + 128) >> 8; }

// inv_dct16_1d (src/idct.rs:1871-1924): the 8-point inverse on the even
// inputs, four stages on the odd half with the intermediate clip, the output
// butterflies.
__device__ __forceinline__ void idct16s(int32_t* c, int s, int32_t mn, int32_t mx) {
  idct8s(c, 2 * s, mn, mx);
  const int32_t in1 = c[s], in3 = c[3 * s], in5 = c[5 * s], in7 = c[7 * s];
  const int32_t in9 = c[9 * s], in11 = c[11 * s], in13 = c[13 * s], in15 = c[15 * s];
  const int32_t a8 = rot12(in1, 401, in15, -4076), a9 = rot12(in9, 3166, in7, -2598);
  const int32_t a10 = rot12(in5, 1931, in11, -3612), a11 = rot12(in13, 3920, in3, -1189);
  const int32_t a12 = rot12(in13, 1189, in3, 3920), a13 = rot12(in5, 3612, in11, 1931);
  const int32_t a14 = rot12(in9, 2598, in7, 3166), a15 = rot12(in1, 4076, in15, 401);
  const int32_t b8 = clampi(a8 + a9, mn, mx), b9 = clampi(a8 - a9, mn, mx);
  const int32_t b10 = clampi(a11 - a10, mn, mx), b11 = clampi(a11 + a10, mn, mx);
  const int32_t b12 = clampi(a12 + a13, mn, mx), b13 = clampi(a12 - a13, mn, mx);
  const int32_t b14 = clampi(a15 - a14, mn, mx), b15 = clampi(a15 + a14, mn, mx);
  const int32_t c9 = rot12(b14, 1567, b9, -3784), c14 = rot12(b14, 3784, b9, 1567);
  const int32_t c10 = rot12(b13, -3784, b10, -1567), c13 = rot12(b13, 1567, b10, -3784);
  const int32_t d8 = clampi(b8 + b11, mn, mx), d9 = clampi(c9 + c10, mn, mx);
  const int32_t d10 = clampi(c9 - c10, mn, mx), d11 = clampi(b8 - b11, mn, mx);
  const int32_t d12 = clampi(b15 - b12, mn, mx), d13 = clampi(c14 - c13, mn, mx);
  const int32_t d14 = clampi(c14 + c13, mn, mx), d15 = clampi(b15 + b12, mn, mx);
  const int32_t e10 = r181(d13 - d10), e13 = r181(d13 + d10), e11 = r181(d12 - d11), e12 = r181(d12 + d11);
  const int32_t t0 = c[0], t1 = c[2 * s], t2 = c[4 * s], t3 = c[6 * s];
  const int32_t t4 = c[8 * s], t5 = c[10 * s], t6 = c[12 * s], t7 = c[14 * s];
  c[0] = clampi(t0 + d15, mn, mx);
  c[s] = clampi(t1 + d14, mn, mx);
  c[2 * s] = clampi(t2 + e13, mn, mx);
  c[3 * s] = clampi(t3 + e12, mn, mx);
  c[4 * s] = clampi(t4 + e11, mn, mx);
  c[5 * s] = clampi(t5 + e10, mn, mx);
  c[6 * s] = clampi(t6 + d9, mn, mx);
  c[7 * s] = clampi(t7 + d8, mn, mx);
  c[8 * s] = clampi(t7 - d8, mn, mx);
  c[9 * s] = clampi(t6 - d9, mn, mx);
  c[10 * s] = clampi(t5 - e10, mn, mx);
  c[11 * s] = clampi(t4 - e11, mn, mx);
  c[12 * s] = clampi(t3 - e12, mn, mx);
  c[13 * s] = clampi(t2 - e13, mn, mx);
  c[14 * s] = clampi(t1 - d14, mn, mx);
  c[15 * s] = clampi(t0 - d15, mn, mx);
}

// Rotation constants of the first ADST16 stage: output pair k uses inputs
// (15 - 2k, 2k), i.e. a[2k] = rot(in[15-2k], c0, in[2k], c1) and
// a[2k+1] = rot(in[15-2k], c1, in[2k], -c0) (src/idct.rs:1974-1989).
__constant__ int16_t kIadst16S1[8][2] = {{4091, 201}, {3973, 995}, {3703, 1751}, {3290, 2440},
                                         {2751, 3035}, {2106, 3513}, {1380, 3857}, {601, 4052}};

// inv_adst16_1d (src/idct.rs:1968-2062): four rotation / butterfly stages with
// the intermediate clip and the signed 181/256 outputs.
__device__ __forceinline__ void iadst16s(int32_t* c, int s, int32_t mn, int32_t mx) {
  int32_t a[16];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int32_t hi = c[(15 - 2 * k) * s], lo = c[(2 * k) * s];
    const int32_t c0 = kIadst16S1[k][0], c1 = kIadst16S1[k][1];
    a[2 * k] = rot12(hi, c0, lo, c1);
    a[2 * k + 1] = rot12(hi, c1, lo, -c0);
  }
  int32_t b[16];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    b[i] = clampi(a[i] + a[i + 8], mn, mx);
    b[8 + i] = clampi(a[i] - a[i + 8], mn, mx);
  }
  const int32_t c8 = rot12(b[8], 4017, b[9], 799), c9 = rot12(b[8], 799, b[9], -4017);
  const int32_t c10 = rot12(b[10], 2276, b[11], 3406), c11 = rot12(b[10], 3406, b[11], -2276);
  const int32_t c12 = rot12(b[13], 4017, b[12], -799), c13 = rot12(b[13], 799, b[12], 4017);
  const int32_t c14 = rot12(b[15], 2276, b[14], -3406), c15 = rot12(b[15], 3406, b[14], 2276);
  const int32_t d0 = clampi(b[0] + b[4], mn, mx), d1 = clampi(b[1] + b[5], mn, mx);
  const int32_t d2 = clampi(b[2] + b[6], mn, mx), d3 = clampi(b[3] + b[7], mn, mx);
  const int32_t d4 = clampi(b[0] - b[4], mn, mx), d5 = clampi(b[1] - b[5], mn, mx);
  const int32_t d6 = clampi(b[2] - b[6], mn, mx), d7 = clampi(b[3] - b[7], mn, mx);
  const int32_t d8 = clampi(c8 + c12, mn, mx), d9 = clampi(c9 + c13, mn, mx);
  const int32_t d10 = clampi(c10 + c14, mn, mx), d11 = clampi(c11 + c15, mn, mx);
  const int32_t d12 = clampi(c8 - c12, mn, mx), d13 = clampi(c9 - c13, mn, mx);
  const int32_t d14 = clampi(c10 - c14, mn, mx), d15 = clampi(c11 - c15, mn, mx);
  const int32_t e4 = rot12(d4, 3784, d5, 1567), e5 = rot12(d4, 1567, d5, -3784);
  const int32_t e6 = rot12(d7, 3784, d6, -1567), e7 = rot12(d7, 1567, d6, 3784);
  const int32_t e12 = rot12(d12, 3784, d13, 1567), e13 = rot12(d12, 1567, d13, -3784);
  const int32_t e14 = rot12(d15, 3784, d14, -1567), e15 = rot12(d15, 1567, d14, 3784);
  const int32_t f2 = clampi(d0 - d2, mn, mx), f3 = clampi(d1 - d3, mn, mx);
  const int32_t f6 = clampi(e4 - e6, mn, mx), f7 = clampi(e5 - e7, mn, mx);
  const int32_t f10 = clampi(d8 - d10, mn, mx), f11 = clampi(d9 - d11, mn, mx);
  const int32_t f14 = clampi(e12 - e14, mn, mx), f15 = clampi(e13 - e15, mn, mx);
  c[0] = clampi(d0 + d2, mn, mx);
  c[15 * s] = -clampi(d1 + d3, mn, mx);
  c[3 * s] = -clampi(e4 + e6, mn, mx);
  c[12 * s] = clampi(e5 + e7, mn, mx);
  c[s] = -clampi(d8 + d10, mn, mx);
  c[14 * s] = clampi(d9 + d11, mn, mx);
  c[2 * s] = clampi(e12 + e14, mn, mx);
  c[13 * s] = -clampi(e13 + e15, mn, mx);
  c[7 * s] = -r181(f2 + f3);
  c[8 * s] = r181(f2 - f3);
  c[4 * s] = r181(f6 + f7);
  c[11 * s] = -r181(f6 - f7);
  c[6 * s] = r181(f10 + f11);
  c[9 * s] = -r181(f10 - f11);
  c[5 * s] = -r181(f14 + f15);
  c[10 * s] = r181(f14 - f15);
}

// Dequantisation and the 16x16 inverses (src/idct.rs:1826-1966, :2067-2128):
// tmp[y*16+x] = coeff[y + x*16]; rows (row clip), (t+2)>>2 with the column
// clip, columns, (t+8)>>4; IDTX: 2x + (x*1697 + 1024) >> 11 both passes,
// flat dequantisation.
template <typename C, typename O>
__device__ void inv16x16(const C* __restrict__ cf, int tx, const mt_quant& q, const uint8_t* __restrict__ qm,
                         O* __restrict__ out, int32_t* __restrict__ t) {
  const bool idtx = tx == MT_TX_IDTX;
  const uint8_t* w = idtx ? nullptr : qm;
#pragma unroll 4
  for (int rc = 0; rc < 256; rc++) {
    const int32_t l = cf[rc];
    const int32_t base = rc == 0 ? q.dc_q : q.ac_q;
    const int32_t step = w ? ((base * (int32_t)w[rc] + 16) >> 5) : base;
    int32_t mag = (int32_t)((uabs(l) * (uint32_t)step) & 0xffffffu);
    mag = min(mag, q.cf_max + (l < 0 ? 1 : 0));
    t[(rc & 15) * 16 + (rc >> 4)] = l == 0 ? 0 : (l < 0 ? -mag : mag);
  }
  if (idtx) {
#pragma unroll 4
    for (int i = 0; i < 256; i++) {
      int32_t v = t[i];
      v = clampi((2 * v + ((v * 1697 + 1024) >> 11) + 2) >> 2, q.cmin, q.cmax);
      out[i] = (O)((2 * v + ((v * 1697 + 1024) >> 11) + 8) >> 4);
    }
    return;
  }
  const bool col_adst = tx == MT_TX_ADST_ADST || tx == MT_TX_ADST_DCT;
  const bool row_adst = tx == MT_TX_ADST_ADST || tx == MT_TX_DCT_ADST;
#pragma unroll 1
  for (int y = 0; y < 16; y++) {
    if (row_adst) iadst16s(t + y * 16, 1, q.rmin, q.rmax);
    else idct16s(t + y * 16, 1, q.rmin, q.rmax);
  }
#pragma unroll 4
  for (int i = 0; i < 256; i++) t[i] = clampi((t[i] + 2) >> 2, q.cmin, q.cmax);
#pragma unroll 1
  for (int x = 0; x < 16; x++) {
    if (col_adst) iadst16s(t + x, 16, q.cmin, q.cmax);
    else idct16s(t + x, 16, q.cmin, q.cmax);
  }
#pragma unroll 4
  for (int i = 0; i < 256; i++) out[i] = (O)((t[i] + 8) >> 4);
}

}  // namespace mtd
