// CPU oracle (test infrastructure only): SHA-256 per FIPS 180-4 and the Binius Merkle node
// compression.
//
// The reference uses the third-party `sha2` crate 0.10.x (workspace dependency `sha2 = "0.10.8"`,
// feature `compress`), which is not vendored under the reference tree; this file restates the
// published FIPS 180-4 algorithm.  Call sites it must match:
//   * leaves: `impl<D: Digest> ParallelDigest for D` with D = sha2::Sha256
//     (prover/prover/src/hash/parallel_digest.rs:145-173) -- a standard SHA-256 digest of the
//     concatenated 16-byte little-endian element encodings;
//   * nodes: `Sha256Compression` (verifier/verifier/src/hash/compress.rs:32-57) -- one
//     `compress256` of left||right starting from the state whose little-endian bytes are
//     SHA-256("BINIUS SHA-256 COMPRESS"), with the output state words written little-endian.
#include <string.h>

#include <thread>
#include <vector>

#include "oracle.h"
#include "oracle_internal.h"

namespace orc {

static const uint32_t K[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

static const uint32_t H0[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                               0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};

static inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

void sha256_compress(uint32_t s[8], const uint8_t block[64]) {
  uint32_t w[64];
  for (int t = 0; t < 16; t++)
    w[t] = ((uint32_t)block[4 * t] << 24) | ((uint32_t)block[4 * t + 1] << 16) |
           ((uint32_t)block[4 * t + 2] << 8) | (uint32_t)block[4 * t + 3];
  for (int t = 16; t < 64; t++) {
    uint32_t s0 = rotr(w[t - 15], 7) ^ rotr(w[t - 15], 18) ^ (w[t - 15] >> 3);
    uint32_t s1 = rotr(w[t - 2], 17) ^ rotr(w[t - 2], 19) ^ (w[t - 2] >> 10);
    w[t] = w[t - 16] + s0 + w[t - 7] + s1;
  }
  uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
  for (int t = 0; t < 64; t++) {
    uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);
    uint32_t ch = (e & f) ^ (~e & g);
    uint32_t t1 = h + S1 + ch + K[t] + w[t];
    uint32_t S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
    uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
    uint32_t t2 = S0 + mj;
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

void sha256(const uint8_t* data, size_t len, uint8_t out[32]) {
  uint32_t s[8];
  memcpy(s, H0, sizeof(s));
  size_t full = len / 64;
  for (size_t i = 0; i < full; i++) sha256_compress(s, data + 64 * i);
  uint8_t tail[128];
  memset(tail, 0, sizeof(tail));
  size_t rem = len - 64 * full;
  memcpy(tail, data + 64 * full, rem);
  tail[rem] = 0x80;
  size_t tail_len = (rem + 9 <= 64) ? 64 : 128;
  uint64_t bits = (uint64_t)len * 8;
  for (int i = 0; i < 8; i++) tail[tail_len - 1 - i] = (uint8_t)(bits >> (8 * i));
  sha256_compress(s, tail);
  if (tail_len == 128) sha256_compress(s, tail + 64);
  for (int i = 0; i < 8; i++) {
    out[4 * i] = (uint8_t)(s[i] >> 24);
    out[4 * i + 1] = (uint8_t)(s[i] >> 16);
    out[4 * i + 2] = (uint8_t)(s[i] >> 8);
    out[4 * i + 3] = (uint8_t)s[i];
  }
}

void Sha256Ctx::reset() {
  memcpy(h, H0, sizeof(h));
  buflen = 0;
  total = 0;
}

void Sha256Ctx::update(const uint8_t* data, size_t len) {
  total += len;
  while (len > 0) {
    size_t take = 64 - buflen < len ? 64 - buflen : len;
    memcpy(buf + buflen, data, take);
    buflen += take;
    data += take;
    len -= take;
    if (buflen == 64) {
      sha256_compress(h, buf);
      buflen = 0;
    }
  }
}

void Sha256Ctx::finalize(uint8_t out[32]) {
  uint32_t s[8];
  memcpy(s, h, sizeof(s));
  uint8_t tail[128];
  memset(tail, 0, sizeof(tail));
  memcpy(tail, buf, buflen);
  tail[buflen] = 0x80;
  size_t tail_len = (buflen + 9 <= 64) ? 64 : 128;
  uint64_t bits = total * 8;
  for (int i = 0; i < 8; i++) tail[tail_len - 1 - i] = (uint8_t)(bits >> (8 * i));
  sha256_compress(s, tail);
  if (tail_len == 128) sha256_compress(s, tail + 64);
  for (int i = 0; i < 8; i++) {
    out[4 * i] = (uint8_t)(s[i] >> 24);
    out[4 * i + 1] = (uint8_t)(s[i] >> 16);
    out[4 * i + 2] = (uint8_t)(s[i] >> 8);
    out[4 * i + 3] = (uint8_t)s[i];
  }
}

// The compression IV: the digest bytes of "BINIUS SHA-256 COMPRESS" read as native
// (little-endian) u32 words, as `bytes_of_mut(&mut initial_state).copy_from_slice(...)` does.
static void node_iv(uint32_t iv[8]) {
  static uint32_t cached[8];
  static bool ready = false;
  if (!ready) {
    const char* tag = "BINIUS SHA-256 COMPRESS";
    uint8_t d[32];
    sha256((const uint8_t*)tag, strlen(tag), d);
    for (int i = 0; i < 8; i++)
      cached[i] = (uint32_t)d[4 * i] | ((uint32_t)d[4 * i + 1] << 8) |
                  ((uint32_t)d[4 * i + 2] << 16) | ((uint32_t)d[4 * i + 3] << 24);
    ready = true;
  }
  memcpy(iv, cached, sizeof(cached));
}

void compress_node(const uint8_t left[32], const uint8_t right[32], uint8_t out[32]) {
  uint32_t s[8];
  node_iv(s);
  uint8_t block[64];
  memcpy(block, left, 32);
  memcpy(block + 32, right, 32);
  sha256_compress(s, block);
  // must_cast::<[u32; 8], [u8; 32]>: native little-endian bytes of the state words.
  for (int i = 0; i < 8; i++) {
    out[4 * i] = (uint8_t)s[i];
    out[4 * i + 1] = (uint8_t)(s[i] >> 8);
    out[4 * i + 2] = (uint8_t)(s[i] >> 16);
    out[4 * i + 3] = (uint8_t)(s[i] >> 24);
  }
}

static int g_threads = 1;

int num_threads() { return g_threads; }

void parallel_for(size_t n, const std::function<void(size_t, size_t)>& range_fn) {
  int t = g_threads;
  if (t <= 1 || n < 2) {
    range_fn(0, n);
    return;
  }
  if ((size_t)t > n) t = (int)n;
  std::vector<std::thread> pool;
  size_t chunk = (n + t - 1) / t;
  for (int i = 0; i < t; i++) {
    size_t lo = i * chunk, hi = lo + chunk < n ? lo + chunk : n;
    if (lo >= hi) break;
    pool.emplace_back([&, lo, hi] { range_fn(lo, hi); });
  }
  for (auto& th : pool) th.join();
}

}  // namespace orc

extern "C" {
void orc_sha256(const uint8_t* data, size_t len, uint8_t out[32]) { orc::sha256(data, len, out); }
void orc_sha256_compress_node(const uint8_t left[32], const uint8_t right[32], uint8_t out[32]) {
  orc::compress_node(left, right, out);
}
void orc_set_threads(int n) { orc::g_threads = n < 1 ? 1 : n; }
}
