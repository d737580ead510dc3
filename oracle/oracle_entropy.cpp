// Oracle side of the entropy path (test infrastructure only): the AV1 range
// decoder restated from src/odec.rs:615-760 (OdEcDecoder) with the same
// update_cdf (src/odec.rs:47-60), so that the library's encoder and packer
// can be checked by decoding what they wrote.
#include <stdint.h>
#include <string.h>

namespace {
constexpr int kWindow = 32;
constexpr int16_t kLotsOfBits = 0x4000;

struct Dec {
  const uint8_t* buf;
  size_t n, bptr;
  uint32_t dif;
  uint16_t rng;
  int16_t cnt;

  void refill() {
    int s = kWindow - 9 - (cnt + 15);
    while (s >= 0 && bptr < n) {
      dif ^= (uint32_t)buf[bptr] << s;
      cnt += 8;
      s -= 8;
      ++bptr;
    }
    if (bptr >= n) cnt = kLotsOfBits;
  }
  void normalize(uint32_t d_, uint32_t r) {
    int lz = 0;
    for (uint32_t b = 0x80000000u; b && !(r & b); b >>= 1) ++lz;
    const int d = lz - 16;
    cnt -= d;
    dif = ((d_ + 1) << d) - 1;
    rng = (uint16_t)(r << d);
    if (cnt < 0) refill();
  }
  bool decode_bool(uint16_t f) {
    const uint32_t r = rng;
    const uint32_t v = (((r >> 8) * ((uint32_t)f >> 6)) >> 1) + 4;
    const uint32_t vw = v << (kWindow - 16);
    bool ret;
    uint32_t d2, r2;
    if (dif >= vw) {
      d2 = dif - vw;
      r2 = r - v;
      ret = false;
    } else {
      d2 = dif;
      r2 = v;
      ret = true;
    }
    normalize(d2, r2);
    return ret;
  }
  int decode_symbol_noupdate(const uint16_t* cdf, int len) {
    const uint32_t r = rng;
    const uint32_t n = (uint32_t)len - 1;
    const uint32_t c = dif >> (kWindow - 16);
    int ret = 0;
    uint32_t u = r;
    uint32_t v = ((r >> 8) * ((uint32_t)cdf[0] >> 6)) >> 1;
    v += 4 * n;
    while (c < v) {
      u = v;
      ++ret;
      v = ((r >> 8) * ((uint32_t)cdf[ret] >> 6)) >> 1;
      v += 4 * (n - (uint32_t)ret);
    }
    normalize(dif - (v << (kWindow - 16)), u - v);
    return ret;
  }
};

void update_cdf(uint16_t* cdf, int n, int val) {
  const uint32_t count = cdf[n - 1];
  const uint32_t rate = 3 + (uint32_t)((n >> 1) < 2 ? (n >> 1) : 2) + (count >> 4);
  cdf[n - 1] = (uint16_t)(count + 1 - (count >> 5));
  for (int i = 0; i < n - 1; ++i)
    cdf[i] = i >= val ? (uint16_t)(cdf[i] - (cdf[i] >> rate)) : (uint16_t)(cdf[i] + ((32768u - cdf[i]) >> rate));
}

}  // namespace

extern "C" {

void* or_dec_new(const uint8_t* buf, size_t n) {
  Dec* d = new Dec{buf, n, 0, (1u << 31) - 1, 0x8000, -15};
  d->refill();
  return d;
}
void or_dec_free(void* d) { delete (Dec*)d; }
int or_dec_bool(void* d, uint16_t f) { return ((Dec*)d)->decode_bool(f) ? 1 : 0; }
uint32_t or_dec_literal(void* d, uint32_t bits) {
  uint32_t v = 0;
  for (uint32_t i = 0; i < bits; ++i) v = (v << 1) | (((Dec*)d)->decode_bool(16384) ? 1u : 0u);
  return v;
}
int or_dec_symbol(void* d, uint16_t* cdf, int len, int adapt) {
  const int s = ((Dec*)d)->decode_symbol_noupdate(cdf, len);
  if (adapt) update_cdf(cdf, len, s);
  return s;
}

// decode_subexp / decode_signed_subexp_with_ref (src/odec.rs:686-728).
static uint32_t dec_ns(Dec* d, uint32_t n) {
  if (n <= 1) return 0;
  uint32_t w = 0;
  while ((1u << w) < n) ++w;
  const uint32_t m = (1u << w) - n;
  uint32_t v = 0;
  for (uint32_t i = 0; i + 1 < w; ++i) v = (v << 1) | (d->decode_bool(16384) ? 1u : 0u);
  if (v < m) return v;
  const uint32_t extra = d->decode_bool(16384) ? 1u : 0u;
  return (v << 1) - m + extra;
}
static uint32_t dec_subexp(Dec* d, uint32_t num_syms, uint32_t k) {
  uint32_t i = 0, mk = 0;
  for (;;) {
    const uint32_t b2 = i ? k + i - 1 : k;
    const uint32_t a = 1u << b2;
    if (num_syms <= mk + 3 * a) return dec_ns(d, num_syms - mk) + mk;
    if (d->decode_bool(16384)) {
      ++i;
      mk += a;
    } else {
      uint32_t v = 0;
      for (uint32_t j = 0; j < b2; ++j) v = (v << 1) | (d->decode_bool(16384) ? 1u : 0u);
      return v + mk;
    }
  }
}
static uint32_t inverse_recenter(uint32_t r, uint32_t v) {
  if (v > (r << 1)) return v;
  if (v & 1) return r - ((v + 1) >> 1);
  return r + (v >> 1);
}
int32_t or_dec_signed_subexp_with_ref(void* dv, int32_t low, int32_t high, uint32_t k, int32_t r) {
  Dec* d = (Dec*)dv;
  const uint32_t mx = (uint32_t)(high - low), rr = (uint32_t)(r - low);
  const uint32_t v = dec_subexp(d, mx, k);
  const uint32_t x = (rr << 1) <= mx ? inverse_recenter(rr, v) : mx - 1 - inverse_recenter(mx - 1 - rr, v);
  return (int32_t)x + low;
}

}  // extern "C"
