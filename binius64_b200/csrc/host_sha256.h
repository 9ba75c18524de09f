// Incremental SHA-256 (FIPS 180-4) for the library's host-side protocol code: the Fiat-Shamir
// challenger (HasherChallenger<Sha256>, verifier/transcript/src/fiat_shamir/hasher_challenger.rs)
// and the Merkle node-compression IV.  The reference uses the third-party `sha2` crate 0.10.x.
#pragma once
#include <stdint.h>
#include <string.h>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

namespace bgpu {

class HostSha256 {
 public:
  HostSha256() { reset(); }

  void reset() {
    static const uint32_t kH0[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                    0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
    memcpy(h_, kH0, sizeof(h_));
    buflen_ = 0;
    total_ = 0;
  }

  void update(const uint8_t* data, size_t len) {
    total_ += len;
    while (len > 0) {
      size_t take = 64 - buflen_ < len ? 64 - buflen_ : len;
      memcpy(buf_ + buflen_, data, take);
      buflen_ += take;
      data += take;
      len -= take;
      if (buflen_ == 64) {
        compress(h_, buf_);
        buflen_ = 0;
      }
    }
  }

  // Digest of everything absorbed so far; the state is left unchanged.
  void digest(uint8_t out[32]) const {
    uint32_t s[8];
    memcpy(s, h_, sizeof(s));
    uint8_t tail[128] = {0};
    memcpy(tail, buf_, buflen_);
    tail[buflen_] = 0x80;
    size_t tl = buflen_ + 9 <= 64 ? 64 : 128;
    uint64_t bits = total_ * 8;
    for (int i = 0; i < 8; i++) tail[tl - 1 - i] = (uint8_t)(bits >> (8 * i));
    compress(s, tail);
    if (tl == 128) compress(s, tail + 64);
    for (int i = 0; i < 8; i++) {
      out[4 * i] = (uint8_t)(s[i] >> 24);
      out[4 * i + 1] = (uint8_t)(s[i] >> 16);
      out[4 * i + 2] = (uint8_t)(s[i] >> 8);
      out[4 * i + 3] = (uint8_t)s[i];
    }
  }

  // Raw state, for handing the stream to the device transcript and back.
  void save(uint32_t h[8], uint8_t blk[64], uint32_t& blk_len, uint64_t& total) const {
    memcpy(h, h_, sizeof(h_));
    memcpy(blk, buf_, 64);
    blk_len = (uint32_t)buflen_;
    total = total_;
  }
  void load(const uint32_t h[8], const uint8_t blk[64], uint32_t blk_len, uint64_t total) {
    memcpy(h_, h, sizeof(h_));
    memcpy(buf_, blk, 64);
    buflen_ = blk_len & 63;
    total_ = total;
  }

  static void oneshot(const uint8_t* data, size_t len, uint8_t out[32]) {
    HostSha256 h;
    h.update(data, len);
    h.digest(out);
  }

 private:
  static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

  static void compress(uint32_t s[8], const uint8_t* blk) {
#if defined(__x86_64__)
    static const bool ni = __builtin_cpu_supports("sha") && __builtin_cpu_supports("sse4.1");
    if (ni) return compress_ni(s, blk);
#endif
    compress_scalar(s, blk);
  }

  static const uint32_t* round_constants() {
    static const uint32_t K[64] = {
        0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4,
        0xab1c5ed5, 0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe,
        0x9bdc06a7, 0xc19bf174, 0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f,
        0x4a7484aa, 0x5cb0a9dc, 0x76f988da, 0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7,
        0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967, 0x27b70a85, 0x2e1b2138, 0x4d2c6dfc,
        0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85, 0xa2bfe8a1, 0xa81a664b,
        0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070, 0x19a4c116,
        0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
        0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7,
        0xc67178f2};
    return K;
  }

#if defined(__x86_64__)
  // The same compression on the x86 SHA extensions (SHA256RNDS2 runs two rounds on the state
  // split as (A, B, E, F) / (C, D, G, H); SHA256MSG1 / SHA256MSG2 extend the schedule four words
  // at a time), following the usage Intel documents for them.
  __attribute__((target("sha,sse4.1"))) static void compress_ni(uint32_t s[8],
                                                                const uint8_t* blk) {
    const uint32_t* K = round_constants();
    const __m128i bswap = _mm_set_epi64x(0x0c0d0e0f08090a0bll, 0x0405060700010203ll);
    __m128i dcba = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s));
    __m128i hgfe = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + 4));
    const __m128i cdab = _mm_shuffle_epi32(dcba, 0xB1);
    const __m128i efgh = _mm_shuffle_epi32(hgfe, 0x1B);
    __m128i abef = _mm_alignr_epi8(cdab, efgh, 8);
    __m128i cdgh = _mm_blend_epi16(efgh, cdab, 0xF0);
    const __m128i abef0 = abef, cdgh0 = cdgh;
    __m128i w[16];  // the schedule in groups of four words
    for (int i = 0; i < 4; i++)
      w[i] = _mm_shuffle_epi8(_mm_loadu_si128(reinterpret_cast<const __m128i*>(blk + 16 * i)),
                              bswap);
    for (int i = 4; i < 16; i++) {
      __m128i t = _mm_sha256msg1_epu32(w[i - 4], w[i - 3]);
      t = _mm_add_epi32(t, _mm_alignr_epi8(w[i - 1], w[i - 2], 4));
      w[i] = _mm_sha256msg2_epu32(t, w[i - 1]);
    }
    for (int i = 0; i < 16; i++) {
      const __m128i m =
          _mm_add_epi32(w[i], _mm_loadu_si128(reinterpret_cast<const __m128i*>(K + 4 * i)));
      cdgh = _mm_sha256rnds2_epu32(cdgh, abef, m);
      abef = _mm_sha256rnds2_epu32(abef, cdgh, _mm_shuffle_epi32(m, 0x0E));
    }
    abef = _mm_add_epi32(abef, abef0);
    cdgh = _mm_add_epi32(cdgh, cdgh0);
    const __m128i feba = _mm_shuffle_epi32(abef, 0x1B);
    const __m128i dchg = _mm_shuffle_epi32(cdgh, 0xB1);
    dcba = _mm_blend_epi16(feba, dchg, 0xF0);
    hgfe = _mm_alignr_epi8(dchg, feba, 8);
    _mm_storeu_si128(reinterpret_cast<__m128i*>(s), dcba);
    _mm_storeu_si128(reinterpret_cast<__m128i*>(s + 4), hgfe);
  }
#endif

  static void compress_scalar(uint32_t s[8], const uint8_t* blk) {
    const uint32_t* K = round_constants();
    uint32_t w[64];
    for (int t = 0; t < 16; t++)
      w[t] = ((uint32_t)blk[4 * t] << 24) | ((uint32_t)blk[4 * t + 1] << 16) |
             ((uint32_t)blk[4 * t + 2] << 8) | blk[4 * t + 3];
    for (int t = 16; t < 64; t++)
      w[t] = w[t - 16] + (rotr(w[t - 15], 7) ^ rotr(w[t - 15], 18) ^ (w[t - 15] >> 3)) +
             w[t - 7] + (rotr(w[t - 2], 17) ^ rotr(w[t - 2], 19) ^ (w[t - 2] >> 10));
    uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
    for (int t = 0; t < 64; t++) {
      uint32_t t1 = h + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + K[t] +
                    w[t];
      uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
      h = g;
      g = f;
      f = e;
      e = d + t1;
      d = c;
      c = b;
      b = a;
      a = t1 + t2;
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

  uint32_t h_[8];
  uint8_t buf_[64];
  size_t buflen_;
  uint64_t total_;
};

}  // namespace bgpu
