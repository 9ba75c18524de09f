// CPU oracle (test infrastructure only): GF(2^128) GHASH field and AES GF(2^8).
//
// Restates verifier/field/src/ghash.rs (modulus x^128 + x^7 + x^2 + x + 1, bit i of the u128 is
// the coefficient of x^i, ghash.rs:55-96) and verifier/field/src/aes_field.rs:26-35.  The
// multiplication is the textbook carry-less product followed by reduction modulo the GHASH
// polynomial; the PCLMULQDQ path and the portable shift-and-add path must agree (tests check it).
#include <stdint.h>
#include <string.h>

#include "oracle.h"
#include "oracle_internal.h"

#if defined(__PCLMUL__) && defined(__SSE4_1__)
#include <immintrin.h>
#define ORC_HAVE_PCLMUL 1
#endif

namespace orc {

static inline void clmul64_portable(uint64_t a, uint64_t b, uint64_t& lo, uint64_t& hi) {
  uint64_t l = 0, h = 0;
  for (int i = 0; i < 64; i++) {
    if ((b >> i) & 1) {
      l ^= a << i;
      if (i) h ^= a >> (64 - i);
    }
  }
  lo = l;
  hi = h;
}

// Reduce the 256-bit carry-less product p[0..3] (little-endian u64 limbs) modulo
// x^128 + x^7 + x^2 + x + 1.  x^128 = x^7 + x^2 + x + 1, so the high half H contributes
// H * (x^7 + x^2 + x + 1); the <= 7 bits that this pushes past x^127 are folded once more.
static inline u128 reduce256(uint64_t p0, uint64_t p1, uint64_t p2, uint64_t p3) {
  uint64_t t = (p3 >> 63) ^ (p3 >> 62) ^ (p3 >> 57);
  uint64_t lo = p0 ^ p2 ^ (p2 << 1) ^ (p2 << 2) ^ (p2 << 7) ^ t ^ (t << 1) ^ (t << 2) ^ (t << 7);
  uint64_t hi = p1 ^ p3 ^ ((p3 << 1) | (p2 >> 63)) ^ ((p3 << 2) | (p2 >> 62)) ^
                ((p3 << 7) | (p2 >> 57));
  return ((u128)hi << 64) | lo;
}

u128 gf_mul_portable(u128 a, u128 b) {
  uint64_t a0 = (uint64_t)a, a1 = (uint64_t)(a >> 64), b0 = (uint64_t)b, b1 = (uint64_t)(b >> 64);
  uint64_t l0, l1, h0, h1, m0, m1, x0, x1;
  clmul64_portable(a0, b0, l0, l1);
  clmul64_portable(a1, b1, h0, h1);
  clmul64_portable(a0, b1, m0, m1);
  clmul64_portable(a1, b0, x0, x1);
  m0 ^= x0;
  m1 ^= x1;
  return reduce256(l0, l1 ^ m0, h0 ^ m1, h1);
}

u128 gf_mul(u128 a, u128 b) {
#ifdef ORC_HAVE_PCLMUL
  __m128i va = _mm_set_epi64x((long long)(uint64_t)(a >> 64), (long long)(uint64_t)a);
  __m128i vb = _mm_set_epi64x((long long)(uint64_t)(b >> 64), (long long)(uint64_t)b);
  __m128i l = _mm_clmulepi64_si128(va, vb, 0x00);
  __m128i h = _mm_clmulepi64_si128(va, vb, 0x11);
  __m128i m = _mm_xor_si128(_mm_clmulepi64_si128(va, vb, 0x01), _mm_clmulepi64_si128(va, vb, 0x10));
  uint64_t l0 = (uint64_t)_mm_cvtsi128_si64(l), l1 = (uint64_t)_mm_extract_epi64(l, 1);
  uint64_t h0 = (uint64_t)_mm_cvtsi128_si64(h), h1 = (uint64_t)_mm_extract_epi64(h, 1);
  uint64_t m0 = (uint64_t)_mm_cvtsi128_si64(m), m1 = (uint64_t)_mm_extract_epi64(m, 1);
  return reduce256(l0, l1 ^ m0, h0 ^ m1, h1);
#else
  return gf_mul_portable(a, b);
#endif
}

u128 gf_square(u128 a) { return gf_mul(a, a); }

// a^(2^128 - 2) = (a^(2^127 - 1))^2; a^(2^k - 1) = (a^(2^(k-1) - 1))^2 * a.  Zero maps to zero
// (the reference's invert_or_zero).
u128 gf_inv(u128 a) {
  u128 r = a;
  for (int k = 2; k <= 127; k++) r = gf_mul(gf_square(r), a);
  return gf_square(r);
}

u128 gf_mul_x(u128 a) {
  u128 mask = (u128)0 - (a >> 127);
  return (a << 1) ^ ((u128)0x87 & mask);
}

u128 gf_mul_inv_x(u128 a) {
  u128 mask = (u128)0 - (a & 1);
  return (a >> 1) ^ ((((u128)1 << 127) | 0x43) & mask);
}

// AES field GF(2^8), modulus x^8 + x^4 + x^3 + x + 1 (aes_field.rs:26-35).
uint8_t aes_mul(uint8_t a, uint8_t b) {
  uint8_t r = 0;
  for (int i = 0; i < 8; i++) {
    if (b & 1) r ^= a;
    uint8_t hi = a & 0x80;
    a = (uint8_t)(a << 1);
    if (hi) a ^= 0x1b;
    b >>= 1;
  }
  return r;
}

// The field embedding GF(2^8) -> GF(2^128) used by `From<AESTowerField8b> for B128`
// (ghash.rs:520-780).  An embedding of fields is fixed by the image g of the AES generator x
// (byte 0x02): phi(b) = sum_i b_i g^i.  g is the table's entry for 0x02, a root of
// x^8 + x^4 + x^3 + x + 1 in GF(2^128); the remaining 255 entries follow from linearity.
static const u128 kAesXInGhash =
    ((u128)0x0dcb364640a222feull << 64) | (u128)0x6b8330483c2e9849ull;

void aes_to_ghash_table(u128 out[256]) {
  u128 pw[8];
  pw[0] = 1;
  for (int i = 1; i < 8; i++) pw[i] = gf_mul(pw[i - 1], kAesXInGhash);
  for (int b = 0; b < 256; b++) {
    u128 acc = 0;
    for (int i = 0; i < 8; i++)
      if ((b >> i) & 1) acc ^= pw[i];
    out[b] = acc;
  }
}

}  // namespace orc

using namespace orc;

extern "C" {

void orc_gf_mul(const uint64_t a[2], const uint64_t b[2], uint64_t out[2]) {
  store(out, gf_mul(load(a), load(b)));
}
void orc_gf_mul_portable(const uint64_t a[2], const uint64_t b[2], uint64_t out[2]) {
  store(out, gf_mul_portable(load(a), load(b)));
}
void orc_gf_inv(const uint64_t a[2], uint64_t out[2]) { store(out, gf_inv(load(a))); }
void orc_gf_mul_x(const uint64_t a[2], uint64_t out[2]) { store(out, gf_mul_x(load(a))); }
void orc_gf_mul_inv_x(const uint64_t a[2], uint64_t out[2]) { store(out, gf_mul_inv_x(load(a))); }
void orc_gf_mul_vec(const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n) {
  for (size_t i = 0; i < n; i++) store(out + 2 * i, gf_mul(load(a + 2 * i), load(b + 2 * i)));
}
uint8_t orc_aes_mul(uint8_t a, uint8_t b) { return aes_mul(a, b); }
void orc_aes_to_ghash_table(uint64_t out[512]) {
  u128 t[256];
  aes_to_ghash_table(t);
  for (int i = 0; i < 256; i++) store(out + 2 * i, t[i]);
}

}  // extern "C"
