// CPU oracle (test infrastructure only): the Vision-4 hash over GF(2^128) GHASH, restated from
// verifier/verifier/src/hash/vision_4/{constants,permutation,digest,compression}.rs.
//
//   permutation  (permutation.rs:104-123): add RC[0]; 8 rounds of
//                sbox(B^-1) -> MDS -> add RC[2r+1] -> sbox(B) -> MDS -> add RC[2r+2]
//   sbox         (permutation.rs:69-73): elementwise inversion (0 -> 0, batch_invert.rs:32-100),
//                then B^-1 or B on each element
//   B(x)         = c0 + c1 x + c2 x^2 + c3 x^4 (B_FWD_COEFFS, constants.rs:11-16);
//                B^-1(y) = L^-1(y) + B_INV_COEFFS[0] with L the linear part of B
//   MDS          (permutation.rs:76-93): circulant (2 3 1 1)
//   RC           compute_round_constants (constants.rs:309-338) from INITIAL_CONSTANT,
//                CONSTANTS_MATRIX and CONSTANTS_CONSTANT (constants.rs:283-307)
//   digest       (digest.rs:37-136): rate 2 elements (32 bytes) that OVERWRITE state[0..2],
//                Keccak-style padding 0x80 .. 0x01, output state[0] || state[1]
//   compression  (compression.rs:24-52): MMO, out = (p(x) + x)[0..2] for x = left || right
//
// L^-1 is found here by Gauss-Jordan elimination of L's 128x128 bit matrix; the tests pin it to the
// reference's own B_INV_COEFFS linearized polynomial and the permutation to its known answers.
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <utility>

#include "oracle.h"
#include "oracle_internal.h"

namespace orc {
namespace {

constexpr u128 H(uint64_t hi, uint64_t lo) { return ((u128)hi << 64) | lo; }

const u128 kBFwd[4] = {
    H(0xb0b849b207a0f1c7, 0x4c29e4d892ca33dd), H(0xf2240891aac3c3a5, 0x855eeb8ce24c9523),
    H(0xb017e96797ef1fbe, 0x9d79908388dd768d), H(0x2bf9f0b94c2b2ceb, 0x00dbb86a2cb472bb)};
const u128 kInitial[4] = {
    H(0xd0e015190f5e0795, 0xf4a1d28234ffdf87), H(0x6111731acd9a89f6, 0xb93ec3a23ec7681b),
    H(0x15da8de707ee3f39, 0x18a34a96728b8d29), H(0x2ea920e89fbb13a1, 0xed2a216b1d232bfb)};
const u128 kMatrix[16] = {
    H(0x1cac9af051191d2c, 0x8ef96344bc8cbd0f), H(0x3ceb350e8c2d2f4d, 0x4750ab0a854c3a4d),
    H(0x09cc78f7eafef94d, 0x8e092e899156946b), H(0x1d1ad17c8c7ee715, 0xa3d58f7eedb30dbb),
    H(0x06bee572113950b3, 0xdd0cdae9dff5dfc5), H(0x4799c3743a356042, 0x8b4bfa1a5cd3d295),
    H(0x516883bf97b07fcf, 0x4cb89ac6bf636d0b), H(0x0b681d1621d6aa1f, 0xdf1a9113b04d755b),
    H(0xe9ba2f01051f6b4b, 0x3ddfe74c125e99e5), H(0x1f58efc5ecf2e1b9, 0x33e31cfb26b916d1),
    H(0x36da671249b5444c, 0xf67efc573241fe19), H(0x056cae18b867d486, 0x615a130556e5eb99),
    H(0x1d8645dd4b1e46b7, 0x8dd9df84956bcf11), H(0x3efa34e48e3b2183, 0x95efe6255339375b),
    H(0x79bf44bae0d23793, 0x97d0812db56c5eff), H(0x7fb3b7fce84776e3, 0x9e538151daddae85)};
const u128 kConstant[4] = {
    H(0x0d42981a71a7c2e4, 0x93ca17e6bb10203f), H(0x9ceed672ccb7030f, 0xca17ed48e18717b9),
    H(0x0cec5c463024f2ba, 0x95c6ecdb4a349d15), H(0xa46023576301b995, 0x990418f3a23e3c99)};

u128 l_fwd(u128 x) {
  const u128 x2 = gf_square(x), x4 = gf_square(x2);
  return gf_mul(kBFwd[1], x) ^ gf_mul(kBFwd[2], x2) ^ gf_mul(kBFwd[3], x4);
}

struct Params {
  u128 linv[128];  // L^-1(e_j)
  u128 binv0;      // B_INV_COEFFS[0] = L^-1(c0)
  u128 rc[17][4];
};

u128 apply_cols(const u128* cols, u128 x) {
  u128 r = 0;
  for (int i = 0; i < 128; i++)
    if ((x >> i) & 1) r ^= cols[i];
  return r;
}

u128 b_fwd(u128 x) { return l_fwd(x) ^ kBFwd[0]; }

void sbox(u128 s[4], bool inverse, const Params& p) {
  for (int i = 0; i < 4; i++) {
    const u128 v = gf_inv(s[i]);  // invert_or_zero
    s[i] = inverse ? (apply_cols(p.linv, v) ^ p.binv0) : b_fwd(v);
  }
}

void mds(u128 a[4]) {
  const u128 sum = a[0] ^ a[1] ^ a[2] ^ a[3], a0 = a[0];
  a[0] ^= sum ^ gf_mul_x(a[0] ^ a[1]);
  a[1] ^= sum ^ gf_mul_x(a[1] ^ a[2]);
  a[2] ^= sum ^ gf_mul_x(a[2] ^ a[3]);
  a[3] ^= sum ^ gf_mul_x(a[3] ^ a0);
}

const Params& params() {
  static Params p;
  static std::once_flag once;
  std::call_once(once, [] {
    // L^-1 by Gauss-Jordan on the pairs (L(e_i), e_i)
    u128 v[128], u[128];
    for (int i = 0; i < 128; i++) {
      v[i] = l_fwd((u128)1 << i);
      u[i] = (u128)1 << i;
    }
    for (int j = 0; j < 128; j++) {
      int piv = j;
      while (piv < 128 && !((v[piv] >> j) & 1)) piv++;
      if (piv == 128) abort();  // L is invertible by construction of B
      std::swap(v[j], v[piv]);
      std::swap(u[j], u[piv]);
      for (int k = 0; k < 128; k++)
        if (k != j && ((v[k] >> j) & 1)) {
          v[k] ^= v[j];
          u[k] ^= u[j];
        }
    }
    for (int j = 0; j < 128; j++) p.linv[j] = u[j];
    p.binv0 = apply_cols(p.linv, kBFwd[0]);
    // compute_round_constants
    u128 state[4], inj[4];
    for (int i = 0; i < 4; i++) state[i] = inj[i] = kInitial[i];
    for (int i = 0; i < 4; i++) p.rc[0][i] = kInitial[i];
    int idx = 1;
    for (int r = 0; r < 8; r++)
      for (int half = 0; half < 2; half++) {
        u128 next[4];
        for (int i = 0; i < 4; i++) {
          next[i] = kConstant[i];
          for (int j = 0; j < 4; j++) next[i] ^= gf_mul(kMatrix[4 * i + j], inj[j]);
        }
        memcpy(inj, next, sizeof(inj));
        sbox(state, half == 0, p);
        mds(state);
        for (int i = 0; i < 4; i++) state[i] ^= inj[i];
        for (int i = 0; i < 4; i++) p.rc[idx][i] = state[i];
        idx++;
      }
  });
  return p;
}

void add_rc(u128 s[4], const u128 rc[4]) {
  for (int i = 0; i < 4; i++) s[i] ^= rc[i];
}

u128 le_load(const uint8_t* b) {
  u128 v = 0;
  for (int i = 15; i >= 0; i--) v = (v << 8) | b[i];
  return v;
}

void le_store(uint8_t* b, u128 v) {
  for (int i = 0; i < 16; i++) b[i] = (uint8_t)(v >> (8 * i));
}

}  // namespace

void vision4_permutation(u128 s[4]) {
  const Params& p = params();
  add_rc(s, p.rc[0]);
  for (int r = 0; r < 8; r++) {
    sbox(s, true, p);
    mds(s);
    add_rc(s, p.rc[1 + 2 * r]);
    sbox(s, false, p);
    mds(s);
    add_rc(s, p.rc[2 + 2 * r]);
  }
}

// VisionHasherDigest: update (digest.rs:94-120) and finalize (:66-79).
struct Vision4Digest {
  u128 state[4] = {0, 0, 0, 0};
  uint8_t buffer[32] = {0};
  size_t filled = 0;

  void permute(const uint8_t* block) {
    state[0] = le_load(block);
    state[1] = le_load(block + 16);
    vision4_permutation(state);
  }
  void update(const uint8_t* data, size_t len) {
    if (filled != 0) {
      const size_t take = len < 32 - filled ? len : 32 - filled;
      memcpy(buffer + filled, data, take);
      data += take;
      len -= take;
      filled += take;
      if (filled == 32) {
        permute(buffer);
        filled = 0;
      }
    }
    while (len >= 32) {
      permute(data);
      data += 32;
      len -= 32;
    }
    if (len) {
      memcpy(buffer, data, len);
      filled = len;
    }
  }
  void finalize(uint8_t out[32]) {
    uint8_t block[32] = {0};
    if (filled != 0) {
      memcpy(block, buffer, filled);
      block[filled] |= 0x80;
      block[31] |= 0x01;
    } else {
      block[0] = 0x80;
      block[31] |= 0x01;
    }
    permute(block);
    le_store(out, state[0]);
    le_store(out + 16, state[1]);
  }
};

void vision4_digest(const uint8_t* data, size_t len, uint8_t out[32]) {
  Vision4Digest d;
  d.update(data, len);
  d.finalize(out);
}

void vision4_compress(const uint8_t left[32], const uint8_t right[32], uint8_t out[32]) {
  u128 s[4] = {le_load(left), le_load(left + 16), le_load(right), le_load(right + 16)};
  const u128 x0 = s[0], x1 = s[1];
  vision4_permutation(s);
  le_store(out, s[0] ^ x0);
  le_store(out + 16, s[1] ^ x1);
}

void merkle_commit_vision4(const u128* elems, uint32_t log_leaves, uint32_t log_batch,
                           uint8_t* nodes) {
  const size_t n_leaves = (size_t)1 << log_leaves, batch = (size_t)1 << log_batch;
  parallel_for(n_leaves, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; i++)
      vision4_digest((const uint8_t*)(elems + i * batch), batch * 16, nodes + 32 * i);
  });
  size_t prev = 0, len = n_leaves;
  while (len > 1) {
    const size_t next = prev + len, half = len / 2;
    parallel_for(half, [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; i++)
        vision4_compress(nodes + 32 * (prev + 2 * i), nodes + 32 * (prev + 2 * i + 1),
                         nodes + 32 * (next + i));
    });
    prev = next;
    len = half;
  }
}

int g_merkle_hash = 0;

void merkle_leaf_hash(const uint8_t* data, size_t len, uint8_t out[32]) {
  if (g_merkle_hash == 1)
    vision4_digest(data, len, out);
  else
    sha256(data, len, out);
}

void merkle_node_hash(const uint8_t left[32], const uint8_t right[32], uint8_t out[32]) {
  if (g_merkle_hash == 1)
    vision4_compress(left, right, out);
  else
    compress_node(left, right, out);
}

}  // namespace orc

using namespace orc;

extern "C" {

void orc_set_merkle_hash(int kind) { g_merkle_hash = kind; }

void orc_vision4_permutation(uint64_t* state) {
  u128 s[4];
  for (int i = 0; i < 4; i++) s[i] = load(state + 2 * i);
  vision4_permutation(s);
  for (int i = 0; i < 4; i++) store(state + 2 * i, s[i]);
}

void orc_vision4_digest(const uint8_t* data, size_t len, const size_t* splits, size_t n_splits,
                        uint8_t* out) {
  Vision4Digest d;
  size_t at = 0;
  for (size_t i = 0; i < n_splits; i++) {
    d.update(data + at, splits[i] - at);
    at = splits[i];
  }
  d.update(data + at, len - at);
  d.finalize(out);
}

void orc_vision4_compress(const uint8_t* in64, uint8_t* out32) {
  vision4_compress(in64, in64 + 32, out32);
}

// which: 0 = L (linear part of B), 1 = L^-1; 2 = B, 3 = B^-1
void orc_vision4_map(int which, const uint64_t* x, uint64_t* out) {
  const Params& p = params();
  const u128 v = load(x);
  u128 r = 0;
  switch (which) {
    case 0: r = l_fwd(v); break;
    case 1: r = apply_cols(p.linv, v); break;
    case 2: r = b_fwd(v); break;
    default: r = apply_cols(p.linv, v) ^ p.binv0; break;
  }
  store(out, r);
}

// rc: 17 * 4 elements; binv0: one element
void orc_vision4_constants(uint64_t* rc, uint64_t* binv0) {
  const Params& p = params();
  for (int r = 0; r < 17; r++)
    for (int i = 0; i < 4; i++) store(rc + 8 * r + 2 * i, p.rc[r][i]);
  store(binv0, p.binv0);
}

int orc_vision4_merkle_commit(const uint64_t* elems, uint32_t log_leaves, uint32_t log_batch,
                              uint8_t* nodes_out) {
  merkle_commit_vision4(reinterpret_cast<const u128*>(elems), log_leaves, log_batch, nodes_out);
  return 0;
}

}  // extern "C"
