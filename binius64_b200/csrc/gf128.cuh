// GF(2^128) GHASH-field arithmetic on the sm_100a integer pipes.
//
// Field: x^128 + x^7 + x^2 + x + 1, bit i of the little-endian u128 is the coefficient of x^i
// (BinaryField128bGhash, verifier/field/src/ghash.rs:55-96).  An element lives in a uint4
// (x = bits 0..31, ..., w = bits 96..127), which is exactly the 16-byte LE serialization, so
// HBM buffers are read and written with 128-bit vector accesses and no repacking.
//
// There is no carry-less multiply instruction on the GPU.  The 32x32 -> 64 carry-less product is
// built from integer multiplies "with holes" (the bmul technique published in BearSSL's
// constant-time GHASH, ghash_ctmul.c): split each operand into the four bit classes i = r mod 4;
// a product of two classes has at most 8 terms at any bit position, which fits in the 4-bit gap
// before the next position of the same class, so the integer product's bits in the right class
// are exactly the carry-less sums.  128x128 uses two levels of Karatsuba (9 such products).
#pragma once
#include <stdint.h>

namespace bgpu {

struct u256 {
  uint64_t p0, p1, p2, p3;
};

__device__ __forceinline__ uint64_t mulw(uint32_t a, uint32_t b) {
  return (uint64_t)a * (uint64_t)b;
}

__device__ __forceinline__ uint64_t clmul32(uint32_t x, uint32_t y) {
  const uint32_t m0 = 0x11111111u, m1 = 0x22222222u, m2 = 0x44444444u, m3 = 0x88888888u;
  uint32_t x0 = x & m0, x1 = x & m1, x2 = x & m2, x3 = x & m3;
  uint32_t y0 = y & m0, y1 = y & m1, y2 = y & m2, y3 = y & m3;
  uint64_t z0 = mulw(x0, y0) ^ mulw(x1, y3) ^ mulw(x2, y2) ^ mulw(x3, y1);
  uint64_t z1 = mulw(x0, y1) ^ mulw(x1, y0) ^ mulw(x2, y3) ^ mulw(x3, y2);
  uint64_t z2 = mulw(x0, y2) ^ mulw(x1, y1) ^ mulw(x2, y0) ^ mulw(x3, y3);
  uint64_t z3 = mulw(x0, y3) ^ mulw(x1, y2) ^ mulw(x2, y1) ^ mulw(x3, y0);
  return (z0 & 0x1111111111111111ull) | (z1 & 0x2222222222222222ull) |
         (z2 & 0x4444444444444444ull) | (z3 & 0x8888888888888888ull);
}

// 64x64 -> 128 carry-less product, one Karatsuba level over clmul32.
__device__ __forceinline__ void clmul64(uint64_t a, uint64_t b, uint64_t& lo, uint64_t& hi) {
  uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
  uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
  uint64_t l = clmul32(a0, b0);
  uint64_t h = clmul32(a1, b1);
  uint64_t m = clmul32(a0 ^ a1, b0 ^ b1) ^ l ^ h;
  lo = l ^ (m << 32);
  hi = h ^ (m >> 32);
}

__device__ __forceinline__ uint64_t lo64(uint4 a) { return ((uint64_t)a.y << 32) | a.x; }
__device__ __forceinline__ uint64_t hi64(uint4 a) { return ((uint64_t)a.w << 32) | a.z; }
__device__ __forceinline__ uint4 make_gf(uint64_t lo, uint64_t hi) {
  return make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32));
}

// Unreduced 128x128 -> 256 carry-less product (Karatsuba over clmul64).
__device__ __forceinline__ u256 clmul128(uint4 a, uint4 b) {
  uint64_t a0 = lo64(a), a1 = hi64(a), b0 = lo64(b), b1 = hi64(b);
  uint64_t l0, l1, h0, h1, m0, m1;
  clmul64(a0, b0, l0, l1);
  clmul64(a1, b1, h0, h1);
  clmul64(a0 ^ a1, b0 ^ b1, m0, m1);
  m0 ^= l0 ^ h0;
  m1 ^= l1 ^ h1;
  u256 r;
  r.p0 = l0;
  r.p1 = l1 ^ m0;
  r.p2 = h0 ^ m1;
  r.p3 = h1;
  return r;
}

__device__ __forceinline__ void xor_into(u256& acc, const u256& v) {
  acc.p0 ^= v.p0;
  acc.p1 ^= v.p1;
  acc.p2 ^= v.p2;
  acc.p3 ^= v.p3;
}

// Reduction modulo x^128 + x^7 + x^2 + x + 1: the high half H contributes H*(x^7 + x^2 + x + 1);
// the <= 7 bits pushed past x^127 by that shift are folded a second time.
__device__ __forceinline__ uint4 reduce256(const u256& p) {
  uint64_t t = (p.p3 >> 63) ^ (p.p3 >> 62) ^ (p.p3 >> 57);
  uint64_t lo = p.p0 ^ p.p2 ^ (p.p2 << 1) ^ (p.p2 << 2) ^ (p.p2 << 7) ^ t ^ (t << 1) ^ (t << 2) ^
                (t << 7);
  uint64_t hi = p.p1 ^ p.p3 ^ ((p.p3 << 1) | (p.p2 >> 63)) ^ ((p.p3 << 2) | (p.p2 >> 62)) ^
                ((p.p3 << 7) | (p.p2 >> 57));
  return make_gf(lo, hi);
}

__device__ __forceinline__ uint4 gf_mul(uint4 a, uint4 b) { return reduce256(clmul128(a, b)); }

// An out-of-line multiply for code that runs once per launch on few threads (small sumcheck
// rounds, scalar protocol steps): one copy of the multiply stays in the instruction cache, where
// inlined copies would each be fetched cold.
static __device__ __noinline__ uint4 gf_mul_nl(uint4 a, uint4 b) { return reduce256(clmul128(a, b)); }

__device__ __forceinline__ uint4 gf_add(uint4 a, uint4 b) {
  return make_uint4(a.x ^ b.x, a.y ^ b.y, a.z ^ b.z, a.w ^ b.w);
}

__device__ __forceinline__ void gf_add_into(uint4& a, uint4 b) {
  a.x ^= b.x;
  a.y ^= b.y;
  a.z ^= b.z;
  a.w ^= b.w;
}

__device__ __forceinline__ bool gf_is_zero(uint4 a) { return (a.x | a.y | a.z | a.w) == 0u; }

__device__ __forceinline__ uint4 gf_zero() { return make_uint4(0u, 0u, 0u, 0u); }
__device__ __forceinline__ uint4 gf_one() { return make_uint4(1u, 0u, 0u, 0u); }

// Multiplication by a fixed element r (the fold challenge of a sumcheck round multiplies every
// element by the same r) through nibble tables in shared memory, which each block builds for
// itself from r: entry (p, v) = r * (v x^(4p)) for the 32 nibble positions p and v < 16, so
// r * x = XOR over the nibbles x_p of x of entry (p, x_p) -- 32 lookups, no reduction.  An entry
// is kept as two 8-byte halves in separate arrays: one 16-entry table of 8-byte words spans the
// 32 banks exactly once, so the scattered lookups of a warp cost two conflict-free wavefronts
// each (16-byte entries put two entries on every bank group).  8 KiB per block.
struct NibbleTable {
  uint2 lo[32][16];
  uint2 hi[32][16];
};

// x^k * r for k < 128: r shifted left by k as a 256-bit value, reduced.
__device__ __forceinline__ uint4 gf_mul_xk(uint4 r, uint32_t k) {
  const uint64_t r0 = lo64(r), r1 = hi64(r);
  const uint32_t s = k & 63;
  const uint64_t a = r0 << s;
  const uint64_t b = s ? (r1 << s) | (r0 >> (64 - s)) : r1;
  const uint64_t c = s ? r1 >> (64 - s) : 0;
  u256 u;
  if (k < 64) {
    u.p0 = a; u.p1 = b; u.p2 = c; u.p3 = 0;
  } else {
    u.p0 = 0; u.p1 = a; u.p2 = b; u.p3 = c;
  }
  return reduce256(u);
}

// Builds r's nibble tables with the calling block (any block size >= 1; ends with a barrier, so
// every thread of the block must call it).  `basis` is 128 elements of scratch shared memory.
__device__ __forceinline__ void nibble_table_build(NibbleTable& t, uint4* basis, uint4 r) {
  for (uint32_t k = threadIdx.x; k < 128; k += blockDim.x) basis[k] = gf_mul_xk(r, k);
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < 32 * 16; e += blockDim.x) {
    const uint32_t p = e >> 4, v = e & 15;
    uint4 acc = gf_zero();
#pragma unroll
    for (int i = 0; i < 4; i++)
      if ((v >> i) & 1u) gf_add_into(acc, basis[4 * p + i]);
    t.lo[p][v] = make_uint2(acc.x, acc.y);
    t.hi[p][v] = make_uint2(acc.z, acc.w);
  }
  __syncthreads();
}

__device__ __forceinline__ uint4 gf_mul_nibble(const NibbleTable& t, uint4 x) {
  uint2 lo = make_uint2(0u, 0u), hi = make_uint2(0u, 0u);
  const uint32_t w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
  for (int p = 0; p < 32; p++) {
    const uint32_t v = (w[p >> 3] >> (4 * (p & 7))) & 15u;
    const uint2 l = t.lo[p][v], h = t.hi[p][v];
    lo.x ^= l.x;
    lo.y ^= l.y;
    hi.x ^= h.x;
    hi.y ^= h.y;
  }
  return make_uint4(lo.x, lo.y, hi.x, hi.y);
}

}  // namespace bgpu
