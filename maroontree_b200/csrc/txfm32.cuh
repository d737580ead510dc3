// Device 32x32 DCT_DCT of the luma leaf (the only TX_32X32 intra type): the
// forward transform with quantisation -- the reference's integer butterflies,
// dct1d_32_i32 built on the 16-point one (src/dct.rs:589-631), on a residual
// with 6 bits of headroom and the 64-bit rounding of
// dct32x32_quant_t_direct (src/dct.rs:705-736) -- and the dav1d inverse with
// the TX_32X32 dequantisation (src/idct.rs:2130-2320).
#pragma once
#include <stdint.h>

#include "txfm16.cuh"

namespace mtd {

// Odd-half weights of the 32-point forward DCT, round(65536 / (2 cos((2k+1) pi / 64)))
// (src/dct.rs:589-592).
__constant__ int32_t kWc32[16] = {32808, 33127, 33780, 34802, 36248,  38203,  40796,  44224,
                                  48794, 55008, 63738, 76640, 97266, 134859, 223321, 667812};

// dct1d_32_i32: even/odd split, 16-point DCTs of both halves (the odd one
// after the WC32 weights), the odd running combine, interleave.
__device__ __forceinline__ void fdct32(int32_t* v) {
  int32_t t[32];
#pragma unroll
  for (int i = 0; i < 16; i++) {
    t[i] = v[i] + v[31 - i];
    t[16 + i] = v[i] - v[31 - i];
  }
  fdct16(t);
#pragma unroll
  for (int i = 0; i < 16; i++) t[16 + i] = mul_q16(t[16 + i], kWc32[i]);
  fdct16(t + 16);
  t[16] = mul_q16(t[16], 92682) + t[17];
#pragma unroll
  for (int i = 17; i < 31; i++) t[i] += t[i + 1];
#pragma unroll
  for (int i = 0; i < 16; i++) {
    v[2 * i] = t[i];
    v[2 * i + 1] = t[16 + i];
  }
}

// Forward 32x32 DCT + quantisation of a row-major residual into column-major
// levels and f32 targets: columns (x 64 headroom), rows, each output
// (x * 16384 + 2^21) >> 22 in 64 bits, quantised with the Q16 multipliers.
// The QM step is applied by the caller.  t: 1024 words.
template <typename I, typename C>
__device__ void fwd32x32(const I* __restrict__ in, const mt_quant& q, C* __restrict__ cf, float* __restrict__ tf,
                         int32_t* __restrict__ t) {
#pragma unroll 1
  for (int x = 0; x < 32; x++) {
    int32_t v[32];
#pragma unroll
    for (int r = 0; r < 32; r++) v[r] = (int32_t)in[r * 32 + x] * 64;
    fdct32(v);
#pragma unroll
    for (int r = 0; r < 32; r++) t[r * 32 + x] = v[r];
  }
#pragma unroll 1
  for (int r = 0; r < 32; r++) {
    int32_t v[32];
#pragma unroll
    for (int u = 0; u < 32; u++) v[u] = t[r * 32 + u];
    fdct32(v);
#pragma unroll
    for (int u = 0; u < 32; u++) {
      const int idx = u * 32 + r;
      const int32_t m = idx == 0 ? q.q_mult_dc : q.q_mult_ac;
      const int32_t c = (int32_t)(((long long)v[u] * 16384 + (1ll << 21)) >> 22);
      cf[idx] = (C)quant_q16(c, m);
      tf[idx] = __fmul_rn(__fmul_rn((float)c, (float)m), 1.0f / 65536.0f);
    }
  }
}

// inv_dct32_1d (src/idct.rs:2130-2279): the 16-point inverse on the even
// inputs, then seven stages on the odd half (rotations by the AV1 cosine
// constants, butterflies with the intermediate clip, the 181/256 pairs) and
// the output butterflies.  Each rotation is (x * cx + y * cy + 2048) >> 12;
// the reference's forms with a constant minus 4096 plus or minus an input, or
// with halved constants and >> 11, are the same value.
__device__ __forceinline__ void idct32s(int32_t* c, int s, int32_t mn, int32_t mx) {
  idct16s(c, 2 * s, mn, mx);
  const int32_t i1 = c[s], i3 = c[3 * s], i5 = c[5 * s], i7 = c[7 * s];
  const int32_t i9 = c[9 * s], i11 = c[11 * s], i13 = c[13 * s], i15 = c[15 * s];
  const int32_t i17 = c[17 * s], i19 = c[19 * s], i21 = c[21 * s], i23 = c[23 * s];
  const int32_t i25 = c[25 * s], i27 = c[27 * s], i29 = c[29 * s], i31 = c[31 * s];
  auto cl = [&](int32_t v) { return clampi(v, mn, mx); };
  // stage 1
  const int32_t a16 = rot12(i1, 201, i31, -4091), a31 = rot12(i1, 4091, i31, 201);
  const int32_t a17 = rot12(i17, 3035, i15, -2751), a30 = rot12(i17, 2751, i15, 3035);
  const int32_t a18 = rot12(i9, 1751, i23, -3703), a29 = rot12(i9, 3703, i23, 1751);
  const int32_t a19 = rot12(i25, 3857, i7, -1380), a28 = rot12(i25, 1380, i7, 3857);
  const int32_t a20 = rot12(i5, 995, i27, -3973), a27 = rot12(i5, 3973, i27, 995);
  const int32_t a21 = rot12(i21, 3513, i11, -2106), a26 = rot12(i21, 2106, i11, 3513);
  const int32_t a22 = rot12(i13, 2440, i19, -3290), a25 = rot12(i13, 3290, i19, 2440);
  const int32_t a23 = rot12(i29, 4052, i3, -601), a24 = rot12(i29, 601, i3, 4052);
  // stage 2
  const int32_t b16 = cl(a16 + a17), b17 = cl(a16 - a17), b18 = cl(a19 - a18), b19 = cl(a19 + a18);
  const int32_t b20 = cl(a20 + a21), b21 = cl(a20 - a21), b22 = cl(a23 - a22), b23 = cl(a23 + a22);
  const int32_t b24 = cl(a24 + a25), b25 = cl(a24 - a25), b26 = cl(a27 - a26), b27 = cl(a27 + a26);
  const int32_t b28 = cl(a28 + a29), b29 = cl(a28 - a29), b30 = cl(a31 - a30), b31 = cl(a31 + a30);
  // stage 3
  const int32_t c17 = rot12(b30, 799, b17, -4017), c30 = rot12(b30, 4017, b17, 799);
  const int32_t c18 = rot12(b29, -4017, b18, -799), c29 = rot12(b29, 799, b18, -4017);
  const int32_t c21 = rot12(b26, 3406, b21, -2276), c26 = rot12(b26, 2276, b21, 3406);
  const int32_t c22 = rot12(b25, -2276, b22, -3406), c25 = rot12(b25, 3406, b22, -2276);
  // stage 4
  const int32_t d16 = cl(b16 + b19), d17 = cl(c17 + c18), d18 = cl(c17 - c18), d19 = cl(b16 - b19);
  const int32_t d20 = cl(b23 - b20), d21 = cl(c22 - c21), d22 = cl(c22 + c21), d23 = cl(b23 + b20);
  const int32_t d24 = cl(b24 + b27), d25 = cl(c25 + c26), d26 = cl(c25 - c26), d27 = cl(b24 - b27);
  const int32_t d28 = cl(b31 - b28), d29 = cl(c30 - c29), d30 = cl(c30 + c29), d31 = cl(b31 + b28);
  // stage 5
  const int32_t e18 = rot12(d29, 1567, d18, -3784), e29 = rot12(d29, 3784, d18, 1567);
  const int32_t e19 = rot12(d28, 1567, d19, -3784), e28 = rot12(d28, 3784, d19, 1567);
  const int32_t e20 = rot12(d27, -3784, d20, -1567), e27 = rot12(d27, 1567, d20, -3784);
  const int32_t e21 = rot12(d26, -3784, d21, -1567), e26 = rot12(d26, 1567, d21, -3784);
  // stage 6
  const int32_t f16 = cl(d16 + d23), f17 = cl(d17 + d22), f18 = cl(e18 + e21), f19 = cl(e19 + e20);
  const int32_t f20 = cl(e19 - e20), f21 = cl(e18 - e21), f22 = cl(d17 - d22), f23 = cl(d16 - d23);
  const int32_t f24 = cl(d31 - d24), f25 = cl(d30 - d25), f26 = cl(e29 - e26), f27 = cl(e28 - e27);
  const int32_t f28 = cl(e28 + e27), f29 = cl(e29 + e26), f30 = cl(d30 + d25), f31 = cl(d31 + d24);
  // stage 7
  const int32_t g20 = r181(f27 - f20), g27 = r181(f27 + f20), g21 = r181(f26 - f21), g26 = r181(f26 + f21);
  const int32_t g22 = r181(f25 - f22), g25 = r181(f25 + f22), g23 = r181(f24 - f23), g24 = r181(f24 + f23);
  // the odd half, paired with even result k: o[k] for outputs k and 31 - k
  const int32_t o[16] = {f31, f30, f29, f28, g27, g26, g25, g24, g23, g22, g21, g20, f19, f18, f17, f16};
  int32_t e[16];
#pragma unroll
  for (int k = 0; k < 16; k++) e[k] = c[2 * k * s];
#pragma unroll
  for (int k = 0; k < 16; k++) {
    c[k * s] = cl(e[k] + o[k]);
    c[(31 - k) * s] = cl(e[k] - o[k]);
  }
}

// Dequantisation of TX_32X32 (src/idct.rs:2281-2320: the product masked to
// 24 bits, then halved, clamped to cf_max) and the 2-D inverse:
// tmp[y*32+x] = coeff[y + x*32]; rows (row clip), (t+2)>>2 with the column
// clip, columns, (t+8)>>4.  qm: the dequantisation weights (NULL: flat).
template <typename C, typename O>
__device__ void inv32x32(const C* __restrict__ cf, const mt_quant& q, const uint8_t* __restrict__ qm,
                         O* __restrict__ out, int32_t* __restrict__ t) {
#pragma unroll 4
  for (int rc = 0; rc < 1024; rc++) {
    const int32_t l = cf[rc];
    const int32_t base = rc == 0 ? q.dc_q : q.ac_q;
    const int32_t step = qm ? ((base * (int32_t)qm[rc] + 16) >> 5) : base;
    int32_t mag = (int32_t)(((uabs(l) * (uint32_t)step) & 0xffffffu) >> 1);
    mag = min(mag, q.cf_max + (l < 0 ? 1 : 0));
    t[(rc & 31) * 32 + (rc >> 5)] = l == 0 ? 0 : (l < 0 ? -mag : mag);
  }
#pragma unroll 1
  for (int y = 0; y < 32; y++) idct32s(t + y * 32, 1, q.rmin, q.rmax);
#pragma unroll 4
  for (int i = 0; i < 1024; i++) t[i] = clampi((t[i] + 2) >> 2, q.cmin, q.cmax);
#pragma unroll 1
  for (int x = 0; x < 32; x++) idct32s(t + x, 32, q.cmin, q.cmax);
#pragma unroll 4
  for (int i = 0; i < 1024; i++) out[i] = (O)((t[i] + 8) >> 4);
}

}  // namespace mtd
