// SHA-256 (FIPS 180-4) on the integer pipes, plus the Binius Merkle node compression.
//
// Leaves are standard SHA-256 digests of the concatenated 16-byte LE field elements
// (prover/prover/src/hash/parallel_digest.rs:145-173 with D = sha2::Sha256).  Inner nodes are one
// compression of left||right from the state whose little-endian bytes are
// SHA-256("BINIUS SHA-256 COMPRESS"), written out as little-endian state words
// (verifier/verifier/src/hash/compress.rs:32-57).  Rotations are funnel shifts; byte swaps are
// PRMT (__byte_perm).
#pragma once
#include <stdint.h>

namespace bgpu {

__device__ __constant__ uint32_t kSha256K[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

// Node-compression initial state: the little-endian words of SHA-256("BINIUS SHA-256 COMPRESS").
// Computed once on the host and passed to kernels by value.
struct NodeIV {
  uint32_t w[8];
};

__device__ __forceinline__ uint32_t rotr32(uint32_t x, uint32_t n) {
  return __funnelshift_r(x, x, n);
}
__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

// One compression of a 16-word big-endian-parsed block into state s.
__device__ __forceinline__ void sha256_compress(uint32_t s[8], uint32_t w[16]) {
  uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
#pragma unroll
  for (int t = 0; t < 64; t++) {
    uint32_t wt;
    if (t < 16) {
      wt = w[t];
    } else {
      uint32_t w15 = w[(t - 15) & 15], w2 = w[(t - 2) & 15];
      uint32_t s0 = rotr32(w15, 7) ^ rotr32(w15, 18) ^ (w15 >> 3);
      uint32_t s1 = rotr32(w2, 17) ^ rotr32(w2, 19) ^ (w2 >> 10);
      wt = w[t & 15] + s0 + w[(t - 7) & 15] + s1;
      w[t & 15] = wt;
    }
    uint32_t S1 = rotr32(e, 6) ^ rotr32(e, 11) ^ rotr32(e, 25);
    uint32_t ch = (e & f) ^ (~e & g);
    uint32_t t1 = h + S1 + ch + kSha256K[t] + wt;
    uint32_t S0 = rotr32(a, 2) ^ rotr32(a, 13) ^ rotr32(a, 22);
    uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
    h = g;
    g = f;
    f = e;
    e = d + t1;
    d = c;
    c = b;
    b = a;
    a = t1 + S0 + mj;
  }
  s[0] += a;
  s[1] += b;
  s[2] += c;
  s[3] += d;
  s[4] += e;
  s[5] += f;
  s[6] += g;
  s[7] += h;
}

__device__ __forceinline__ void sha256_init(uint32_t s[8]) {
  s[0] = 0x6a09e667u;
  s[1] = 0xbb67ae85u;
  s[2] = 0x3c6ef372u;
  s[3] = 0xa54ff53au;
  s[4] = 0x510e527fu;
  s[5] = 0x9b05688cu;
  s[6] = 0x1f83d9abu;
  s[7] = 0x5be0cd19u;
}

// SHA-256 of n_elems consecutive 16-byte elements.  out receives the digest as the 8 words that,
// stored little-endian, give the standard digest bytes.
__device__ __forceinline__ void sha256_elems(const uint4* __restrict__ p, uint32_t n_elems,
                                             uint32_t out[8]) {
  uint32_t s[8];
  sha256_init(s);
  uint32_t w[16];
  uint32_t full_blocks = n_elems >> 2;
  for (uint32_t blk = 0; blk < full_blocks; blk++) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      uint4 v = __ldg(p + 4 * blk + q);
      w[4 * q + 0] = bswap32(v.x);
      w[4 * q + 1] = bswap32(v.y);
      w[4 * q + 2] = bswap32(v.z);
      w[4 * q + 3] = bswap32(v.w);
    }
    sha256_compress(s, w);
  }
  // Final block: the 0, 1, 2 or 3 trailing elements (at most 48 bytes), 0x80, zeros and the
  // 64-bit big-endian bit length always fit in one block.
  uint32_t rem = n_elems & 3;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    if ((uint32_t)q < rem) {
      uint4 v = __ldg(p + 4 * full_blocks + q);
      w[4 * q + 0] = bswap32(v.x);
      w[4 * q + 1] = bswap32(v.y);
      w[4 * q + 2] = bswap32(v.z);
      w[4 * q + 3] = bswap32(v.w);
    } else {
      w[4 * q + 0] = ((uint32_t)q == rem) ? 0x80000000u : 0u;
      w[4 * q + 1] = 0u;
      w[4 * q + 2] = 0u;
      w[4 * q + 3] = 0u;
    }
  }
  uint64_t bits = (uint64_t)n_elems * 128u;
  w[14] = (uint32_t)(bits >> 32);
  w[15] = (uint32_t)bits;
  sha256_compress(s, w);
#pragma unroll
  for (int i = 0; i < 8; i++) out[i] = bswap32(s[i]);
}

// Binius node compression of two 32-byte digests given as little-endian-loaded words; the result
// words, stored little-endian, are the node digest bytes.
__device__ __forceinline__ void compress_node(const NodeIV& iv, const uint32_t left[8],
                                              const uint32_t right[8], uint32_t out[8]) {
  uint32_t s[8];
#pragma unroll
  for (int i = 0; i < 8; i++) s[i] = iv.w[i];
  uint32_t w[16];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    w[i] = bswap32(left[i]);
    w[8 + i] = bswap32(right[i]);
  }
  sha256_compress(s, w);
#pragma unroll
  for (int i = 0; i < 8; i++) out[i] = s[i];
}

}  // namespace bgpu
