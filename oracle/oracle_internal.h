// CPU oracle internals (test infrastructure only).
#ifndef BINIUS_ORACLE_INTERNAL_H
#define BINIUS_ORACLE_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#include <functional>

namespace orc {

typedef unsigned __int128 u128;

static inline u128 load(const uint64_t* p) { return ((u128)p[1] << 64) | p[0]; }
static inline void store(uint64_t* p, u128 v) {
  p[0] = (uint64_t)v;
  p[1] = (uint64_t)(v >> 64);
}

u128 gf_mul(u128 a, u128 b);
u128 gf_mul_portable(u128 a, u128 b);
u128 gf_square(u128 a);
u128 gf_inv(u128 a);
u128 gf_mul_x(u128 a);
u128 gf_mul_inv_x(u128 a);
uint8_t aes_mul(uint8_t a, uint8_t b);
void aes_to_ghash_table(u128 out[256]);

void sha256(const uint8_t* data, size_t len, uint8_t out[32]);
void sha256_compress(uint32_t state[8], const uint8_t block[64]);
void compress_node(const uint8_t left[32], const uint8_t right[32], uint8_t out[32]);

// Incremental SHA-256 (FIPS 180-4): the streaming hasher behind the Fiat-Shamir challenger.
struct Sha256Ctx {
  uint32_t h[8];
  uint8_t buf[64];
  size_t buflen;
  uint64_t total;
  Sha256Ctx() { reset(); }
  void reset();
  void update(const uint8_t* data, size_t len);
  void finalize(uint8_t out[32]);  // does not reset
};

// NTT / RS / Merkle / FRI building blocks (ntt_fri.cpp).
u128 twiddle(const u128* tw, uint32_t layer, size_t block);
size_t reverse_bits(size_t x, uint32_t bits);
void ntt_forward(const u128* tw, u128* data, uint32_t log_d, uint32_t skip_early,
                 uint32_t skip_late);
void rs_encode(const u128* tw, const u128* msg, uint32_t log_dim, uint32_t log_inv_rate,
               uint32_t log_batch, u128* out);
void merkle_commit(const u128* elems, uint32_t log_leaves, uint32_t log_batch, uint8_t* nodes);
void eq_ind_partial_eval(const u128* point, uint32_t n, u128* out);
// The Merkle hash of the tree code (merkle_commit, the PCS openings and their verification):
// 0 = SHA-256 leaves + the Binius SHA-256 compression, 1 = Vision-4 leaves and compression.
// Process-wide, set by orc_set_merkle_hash (the oracle serves one test at a time).
extern int g_merkle_hash;
void merkle_leaf_hash(const uint8_t* data, size_t len, uint8_t out[32]);
void merkle_node_hash(const uint8_t left[32], const uint8_t right[32], uint8_t out[32]);
// Vision-4 (vision4.cpp)
void vision4_permutation(u128 s[4]);
void vision4_digest(const uint8_t* data, size_t len, uint8_t out[32]);
void vision4_compress(const uint8_t left[32], const uint8_t right[32], uint8_t out[32]);
void merkle_commit_vision4(const u128* elems, uint32_t log_leaves, uint32_t log_batch,
                           uint8_t* nodes);
void fold_interleaved(const u128* cw, uint32_t log_len, uint32_t log_batch, const u128* ch,
                      u128* out);
u128 fold_chunk(const u128* tw, uint32_t log_len, size_t chunk_index, u128* vals, const u128* r,
                uint32_t n);
void fold_codeword(const u128* tw, const u128* cw, uint32_t log_len, const u128* r, uint32_t n,
                   u128* out);

// Runs f(i) for i in [0, n), split into contiguous ranges over the configured thread count.
void parallel_for(size_t n, const std::function<void(size_t, size_t)>& range_fn);
int num_threads();

}  // namespace orc

#endif
