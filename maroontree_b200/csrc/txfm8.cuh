// Device building blocks of the 8x8 luma candidate chain: forward transforms
// with quantisation, dequantisation + inverse transforms, trellis, prediction
// edges, SATD and the coefficient rate walk.  All integer arithmetic is the
// reference's exactly (two's-complement wrap, arithmetic shifts); float
// expressions are written one rounding per operation and the file is compiled
// with -fmad=false, so the only fused multiply-adds are the explicit __fmaf_rn
// calls that stand for the AVX2 FMA lanes of the reference's trellis.
#pragma once
#include <stdint.h>

#include "../../include/maroontree_b200.h"
#include "common.cuh"

namespace mtd {

// Unroll depth of the 8-iteration row/column loops of the 8x8 transforms and
// of the 64-element sweeps.  Rolled loops keep one candidate's path small
// enough for the instruction caches, which measured faster than
// straight-line code (the kernel is bound by instruction fetch otherwise).
#ifndef MT_TX_UNROLL
#define MT_TX_UNROLL 1
#endif
#ifndef MT_VEC_UNROLL
#define MT_VEC_UNROLL 8
#endif
constexpr int kTxUnroll = MT_TX_UNROLL;
constexpr int kVecUnroll = MT_VEC_UNROLL;

// Q16 butterfly multiply with rounding (src/dct.rs:60-67).
__device__ __forceinline__ int32_t mul_q16(int32_t d, int32_t c) {
  return (int32_t)(((int64_t)d * (int64_t)c + 32768) >> 16);
}
// Half-step dead-zone quantiser (src/dct.rs:70-79).
__device__ __forceinline__ int32_t quant_q16(int32_t d, int32_t c) {
  int64_t prod = (int64_t)d * (int64_t)c;
  uint64_t mag = prod < 0 ? (uint64_t)0 - (uint64_t)prod : (uint64_t)prod;
  if (mag < 32768) return 0;
  int32_t lvl = (int32_t)((mag + 32768) >> 16);
  return prod >= 0 ? lvl : -lvl;
}
// Full-step dead-zone quantiser of the 1-D DCT family (src/dct.rs:373-389).
__device__ __forceinline__ void quant_fullstep(int32_t coeff, int32_t m, int32_t* lvl, float* tgt) {
  int64_t prod = (int64_t)coeff * (int64_t)m;
  *tgt = __fmul_rn((float)prod, 1.0f / 65536.0f);
  uint64_t mag = prod < 0 ? (uint64_t)0 - (uint64_t)prod : (uint64_t)prod;
  int32_t l = (int32_t)((mag + 32768) >> 16);
  *lvl = mag < 65536 ? 0 : (prod >= 0 ? l : -l);
}

// 4- and 8-point forward DCT butterflies in Q16 (src/dct.rs:171-219).
__device__ __forceinline__ void fdct4(int32_t& a0, int32_t& a1, int32_t& a2, int32_t& a3) {
  const int32_t s0 = a0 + a3, s1 = a1 + a2;
  const int32_t o2 = mul_q16(a0 - a3, 35468), o3 = mul_q16(a1 - a2, 85627);
  const int32_t p = o2 + o3, q = o2 - o3;
  a0 = s0 + s1;
  a2 = s0 - s1;
  a1 = mul_q16(p, 92682) + q;
  a3 = q;
}
__device__ __forceinline__ void fdct8(int32_t* v) {
  int32_t e0 = v[0] + v[7], e1 = v[1] + v[6], e2 = v[2] + v[5], e3 = v[3] + v[4];
  int32_t o0 = mul_q16(v[0] - v[7], 33410), o1 = mul_q16(v[1] - v[6], 39410);
  int32_t o2 = mul_q16(v[2] - v[5], 58981), o3 = mul_q16(v[3] - v[4], 167963);
  fdct4(e0, e1, e2, e3);
  fdct4(o0, o1, o2, o3);
  o0 = mul_q16(o0, 92682) + o1;
  o1 += o2;
  o2 += o3;
  v[0] = e0; v[2] = e1; v[4] = e2; v[6] = e3;
  v[1] = o0; v[3] = o1; v[5] = o2; v[7] = o3;
}
// 8-point forward ADST as a Q12 matrix product (src/dct.rs:304-326).
__constant__ int16_t kAdst8Fwd[64] = {
    567,  1682,  2730, 3675,  4477,  5109,  5544,  5766,  1682, 4480,  5766,  5109,  2732,
    -569, -3675, -5545, 2732, 5766,  3675,  -1682, -5544, -4479, 569,   5109,  3675,  5108,
    -1681, -5764, -569, 5542,  2732,  -4479, 4479,  2732,  -5542, -569,  5764,  -1681, -5108,
    3675,  5109,  -569, -4479, 5544,  -1682, -3675, 5766,  -2732, 5545,  -3675, 569,   2732,
    -5109, 5766,  -4480, 1682, 5766,  -5544, 5109,  -4477, 3675,  -2730, 1682,  -567};
// The reference accumulates in i64.  For residuals of 8-bit samples
// (|r| <= 255) no partial sum of either pass leaves +-2^31 (row sums of |A|
// are <= 29550, column outputs <= ~6.2k), so the i32 accumulation here is the
// same value.
__device__ __forceinline__ void fadst8(int32_t* v) {
  int32_t o[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    int32_t acc = 2048;
#pragma unroll
    for (int j = 0; j < 8; j++) acc += (int32_t)kAdst8Fwd[i * 8 + j] * v[j];
    o[i] = acc >> 12;
  }
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = o[i];
}

// Inverse 1-D kernels, dav1d integer forms (src/idct.rs:1432-1509).
__device__ __forceinline__ void idct4s(int32_t* c, int s, int32_t mn, int32_t mx) {
  const int32_t in0 = c[0], in1 = c[s], in2 = c[2 * s], in3 = c[3 * s];
  const int32_t t0 = ((in0 + in2) * 181 + 128) >> 8;
  const int32_t t1 = ((in0 - in2) * 181 + 128) >> 8;
  const int32_t t2 = ((in1 * 1567 - in3 * (3784 - 4096) + 2048) >> 12) - in3;
  const int32_t t3 = ((in1 * (3784 - 4096) + in3 * 1567 + 2048) >> 12) + in1;
  c[0] = clampi(t0 + t3, mn, mx);
  c[s] = clampi(t1 + t2, mn, mx);
  c[2 * s] = clampi(t1 - t2, mn, mx);
  c[3 * s] = clampi(t0 - t3, mn, mx);
}
__device__ __forceinline__ void idct8s(int32_t* c, int s, int32_t mn, int32_t mx) {
  idct4s(c, 2 * s, mn, mx);
  const int32_t in1 = c[s], in3 = c[3 * s], in5 = c[5 * s], in7 = c[7 * s];
  const int32_t t4a = ((in1 * 799 - in7 * (4017 - 4096) + 2048) >> 12) - in7;
  int32_t t5a = (in5 * 1703 - in3 * 1138 + 1024) >> 11;
  int32_t t6a = (in5 * 1138 + in3 * 1703 + 1024) >> 11;
  const int32_t t7a = ((in1 * (4017 - 4096) + in7 * 799 + 2048) >> 12) + in1;
  const int32_t t4 = clampi(t4a + t5a, mn, mx);
  t5a = clampi(t4a - t5a, mn, mx);
  const int32_t t7 = clampi(t7a + t6a, mn, mx);
  t6a = clampi(t7a - t6a, mn, mx);
  const int32_t t5 = ((t6a - t5a) * 181 + 128) >> 8;
  const int32_t t6 = ((t6a + t5a) * 181 + 128) >> 8;
  const int32_t e0 = c[0], e1 = c[2 * s], e2 = c[4 * s], e3 = c[6 * s];
  c[0] = clampi(e0 + t7, mn, mx);
  c[s] = clampi(e1 + t6, mn, mx);
  c[2 * s] = clampi(e2 + t5, mn, mx);
  c[3 * s] = clampi(e3 + t4, mn, mx);
  c[4 * s] = clampi(e3 - t4, mn, mx);
  c[5 * s] = clampi(e2 - t5, mn, mx);
  c[6 * s] = clampi(e1 - t6, mn, mx);
  c[7 * s] = clampi(e0 - t7, mn, mx);
}
__device__ __forceinline__ void iadst8s(int32_t* c, int s, int32_t mn, int32_t mx) {
  const int32_t in0 = c[0], in1 = c[s], in2 = c[2 * s], in3 = c[3 * s];
  const int32_t in4 = c[4 * s], in5 = c[5 * s], in6 = c[6 * s], in7 = c[7 * s];
  const int32_t t0a = (((4076 - 4096) * in7 + 401 * in0 + 2048) >> 12) + in7;
  const int32_t t1a = ((401 * in7 - (4076 - 4096) * in0 + 2048) >> 12) - in0;
  const int32_t t2a = (((3612 - 4096) * in5 + 1931 * in2 + 2048) >> 12) + in5;
  const int32_t t3a = ((1931 * in5 - (3612 - 4096) * in2 + 2048) >> 12) - in2;
  const int32_t t4a = (1299 * in3 + 1583 * in4 + 1024) >> 11;
  const int32_t t5a = (1583 * in3 - 1299 * in4 + 1024) >> 11;
  const int32_t t6a = ((1189 * in1 + (3920 - 4096) * in6 + 2048) >> 12) + in6;
  const int32_t t7a = (((3920 - 4096) * in1 - 1189 * in6 + 2048) >> 12) + in1;
  const int32_t t0 = clampi(t0a + t4a, mn, mx), t1 = clampi(t1a + t5a, mn, mx);
  const int32_t t2 = clampi(t2a + t6a, mn, mx), t3 = clampi(t3a + t7a, mn, mx);
  const int32_t t4 = clampi(t0a - t4a, mn, mx), t5 = clampi(t1a - t5a, mn, mx);
  const int32_t t6 = clampi(t2a - t6a, mn, mx), t7 = clampi(t3a - t7a, mn, mx);
  const int32_t u4 = (((3784 - 4096) * t4 + 1567 * t5 + 2048) >> 12) + t4;
  const int32_t u5 = ((1567 * t4 - (3784 - 4096) * t5 + 2048) >> 12) - t5;
  const int32_t u6 = (((3784 - 4096) * t7 - 1567 * t6 + 2048) >> 12) + t7;
  const int32_t u7 = ((1567 * t7 + (3784 - 4096) * t6 + 2048) >> 12) + t6;
  c[0] = clampi(t0 + t2, mn, mx);
  c[7 * s] = -clampi(t1 + t3, mn, mx);
  const int32_t v2 = clampi(t0 - t2, mn, mx), v3 = clampi(t1 - t3, mn, mx);
  c[s] = -clampi(u4 + u6, mn, mx);
  c[6 * s] = clampi(u5 + u7, mn, mx);
  const int32_t v6 = clampi(u4 - u6, mn, mx), v7 = clampi(u5 - u7, mn, mx);
  c[3 * s] = -(((v2 + v3) * 181 + 128) >> 8);
  c[4 * s] = ((v2 - v3) * 181 + 128) >> 8;
  c[2 * s] = ((v6 + v7) * 181 + 128) >> 8;
  c[5 * s] = -(((v6 - v7) * 181 + 128) >> 8);
}

// Row/column transform kinds per 7-type index: 0 identity, 1 DCT, 2 ADST.
// Index order IDTX, DCT_DCT, V_DCT, H_DCT, ADST_ADST, ADST_DCT, DCT_ADST;
// "col" is the vertical (first forward) pass.
__device__ __forceinline__ int col_kind(int tx) {
  const int k[7] = {0, 1, 1, 0, 2, 2, 1};
  return k[tx];
}
__device__ __forceinline__ int row_kind(int tx) {
  const int k[7] = {0, 1, 0, 1, 2, 1, 2};
  return k[tx];
}

// Forward 8x8 transform + quantisation of a row-major residual into
// column-major levels and f32 targets (src/dct.rs:279-301, :1222-1293 for the
// 2-D types; :328-370 V/H_DCT; :1586-1611 IDTX).  The QM step of the 2-D types
// is applied by the caller.
template <typename I, typename C>
__device__ void fwd8x8(const I* __restrict__ in, int tx, const mt_quant& q, C* __restrict__ cf,
                       float* __restrict__ tf, int32_t* __restrict__ t) {
  if (tx == MT_TX_IDTX) {
#pragma unroll 8
    for (int i = 0; i < 64; i++) {
      const int y = i >> 3, x = i & 7, rc = y + x * 8;
      const int32_t qd = rc == 0 ? q.dc_q : q.ac_q;
      const int32_t num = in[i] * 8;
      tf[rc] = __fdiv_rn((float)num, (float)qd);
      const int32_t am = (int32_t)uabs(num);
      const int32_t level = (am + qd / 2) / qd;
      cf[rc] = (C)(am < qd ? 0 : (num < 0 ? -level : level));
    }
    return;
  }
#pragma unroll kVecUnroll
  for (int i = 0; i < 64; i++) t[i] = in[i];
  if (tx == MT_TX_V_DCT || tx == MT_TX_H_DCT) {
    const bool vert = tx == MT_TX_V_DCT;
    if (vert) {
#pragma unroll kTxUnroll
      for (int x = 0; x < 8; x++) {
        int32_t v[8];
#pragma unroll
        for (int y = 0; y < 8; y++) v[y] = t[y * 8 + x];
        fdct8(v);
#pragma unroll
        for (int y = 0; y < 8; y++) t[y * 8 + x] = v[y] * 2;
      }
    } else {
#pragma unroll kTxUnroll
      for (int y = 0; y < 8; y++) {
        fdct8(t + y * 8);
#pragma unroll
        for (int x = 0; x < 8; x++) t[y * 8 + x] *= 2;
      }
    }
#pragma unroll
    for (int y = 0; y < 8; y++)
#pragma unroll kTxUnroll
      for (int x = 0; x < 8; x++) {
        const int rc = y + x * 8;
        int32_t lv;
        quant_fullstep(t[y * 8 + x], rc == 0 ? q.q_mult_dc : q.q_mult_ac, &lv, &tf[rc]);
        cf[rc] = (C)lv;
      }
    return;
  }
  const int ck = col_kind(tx), rk = row_kind(tx);
#pragma unroll kTxUnroll
  for (int x = 0; x < 8; x++) {
    int32_t v[8];
#pragma unroll
    for (int r = 0; r < 8; r++) v[r] = t[r * 8 + x];
    if (ck == 1) fdct8(v); else fadst8(v);
#pragma unroll
    for (int r = 0; r < 8; r++) t[r * 8 + x] = v[r];
  }
#pragma unroll kTxUnroll
  for (int r = 0; r < 8; r++) {
    int32_t* v = t + r * 8;
    if (rk == 1) fdct8(v); else fadst8(v);
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = u * 8 + r;
      const int32_t m = idx == 0 ? q.q_mult_dc : q.q_mult_ac;
      cf[idx] = (C)quant_q16(v[u], m);
      tf[idx] = __fmul_rn(__fmul_rn((float)v[u], (float)m), 1.0f / 65536.0f);
    }
  }
}

// Forward QM scale (1024 + w/2)/w / 32 (src/dct.rs:93-104) and the AVX2
// re-quantisation of the pinned x86 build (src/avx/qmatrix.rs:34-71): scale the
// target, round half away from zero by truncate + fraction test.
// Forward QM scale of an inverse weight w (src/dct.rs:93-104); exact in f32.
__device__ __forceinline__ float fwd_qm_scale(int w) { return __fmul_rn((float)((1024 + w / 2) / w), 1.0f / 32.0f); }

// `scale` holds fwd_qm_scale of each position's inverse weight.
template <typename C>
__device__ __forceinline__ void apply_qm(C* cf, float* tf, const float* scale, int n) {
#pragma unroll 8
  for (int i = 0; i < n; i++) {
    const float x = __fmul_rn(tf[i], scale[i]);
    tf[i] = x;
    const float tr = truncf(x);
    const float frac = fabsf(__fsub_rn(x, tr));
    const float step = frac >= 0.5f ? copysignf(1.0f, x) : 0.0f;
    cf[i] = (C)(int32_t)__fadd_rn(tr, step);
  }
}

// Dequantisation (src/idct.rs:1562-1590) and the 8x8 inverse transforms
// (src/idct.rs:1572-1824): tmp[y*8+x] = coeff[y + x*8]; row pass, (t+1)>>1 with
// the column clip, column pass, (t+8)>>4.
template <typename C, typename O>
__device__ void inv8x8(const C* __restrict__ cf, int tx, const mt_quant& q, const uint8_t* __restrict__ qm,
                       O* __restrict__ out, int32_t* __restrict__ t) {
  const bool flat = tx == MT_TX_IDTX || tx == MT_TX_V_DCT || tx == MT_TX_H_DCT;
  const uint8_t* w = flat ? nullptr : qm;
#pragma unroll 8
  for (int rc = 0; rc < 64; rc++) {
    const int32_t l = cf[rc];
    const int32_t base = rc == 0 ? q.dc_q : q.ac_q;
    const int32_t step = w ? ((base * (int32_t)w[rc] + 16) >> 5) : base;
    // Low 24 bits of |l| * step: the 32-bit product has the same low 24 bits
    // as the reference's 64-bit one.
    int32_t mag = (int32_t)((uabs(l) * (uint32_t)step) & 0xffffffu);
    mag = min(mag, q.cf_max + (l < 0 ? 1 : 0));
    const int y = rc & 7, x = rc >> 3;
    t[y * 8 + x] = l == 0 ? 0 : (l < 0 ? -mag : mag);
  }
  const int ck = col_kind(tx), rk = row_kind(tx);
  if (rk == 0) {
#pragma unroll kVecUnroll
    for (int i = 0; i < 64; i++) t[i] *= 2;
  } else {
#pragma unroll kTxUnroll
    for (int y = 0; y < 8; y++) {
      if (rk == 1) idct8s(t + y * 8, 1, q.rmin, q.rmax);
      else iadst8s(t + y * 8, 1, q.rmin, q.rmax);
    }
  }
#pragma unroll kVecUnroll
  for (int i = 0; i < 64; i++) t[i] = clampi((t[i] + 1) >> 1, q.cmin, q.cmax);
  if (ck == 0) {
#pragma unroll kVecUnroll
    for (int i = 0; i < 64; i++) t[i] *= 2;
  } else {
#pragma unroll kTxUnroll
    for (int x = 0; x < 8; x++) {
      if (ck == 1) idct8s(t + x, 8, q.cmin, q.cmax);
      else iadst8s(t + x, 8, q.cmin, q.cmax);
    }
  }
#pragma unroll kVecUnroll
  for (int i = 0; i < 64; i++) out[i] = (O)((t[i] + 8) >> 4);
}

}  // namespace mtd
