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

// Runs f(i) for i in [0, n), split into contiguous ranges over the configured thread count.
void parallel_for(size_t n, const std::function<void(size_t, size_t)>& range_fn);
int num_threads();

}  // namespace orc

#endif
