// AND reduction: the oblong zerocheck of (A & B) ^ C = 0 over the 64-bit rows of every AND
// constraint, with a univariate skip round over the 64 bit positions.
//
// Follows prove_bitand_reduction (prover/prover/src/prove.rs:329-372) and OblongZerocheckProver
// (prover/prover/src/and_reduction/prover.rs:74-276):
//  1. log_n - 3 big-field challenges are sampled; eq_big is their eq tensor.
//  2. Univariate round (and_reduction/sumcheck_round_messages.rs:62-136): each word's 64 bits are
//     the values on the subspace {0, .., 63} of GF(2^8) (AES field, basis 1, 2, .., 32) of a
//     polynomial of degree < 64; its values at the points 64 .. 127 come from byte-indexed tables of
//     Lagrange sums (ntt_lookup.rs:91-164).  Per group of 8 constraints the GF(2^8) values
//     (A*B + C) * eq_small[j] are summed (eq_small is the eq tensor of the fixed challenges 2, 4, 16,
//     config.rs:33-37), embedded into GF(2^128) and weighted by eq_big.  The 64 sums are the message.
//  3. The words are folded at the univariate challenge z (fold_lookup.rs:18-92): word -> sum of the
//     Lagrange basis at z over the set bits, through 8 byte tables.
//  4. A quadratic MLE-check (protocols/sumcheck/quadratic_mle.rs:21-196 with gruen32.rs) on
//     (a, b, c) with composition a*b - c over the point [2, 4, 16] ++ big (embedded), claim = the
//     message extended by zeros on the base domain and evaluated at z.
//
// B200 mapping: the univariate round keeps its 128 KiB of GF(2^8) tables in shared memory laid out
// [byte index][byte value][4-point group] so the 16 threads of a constraint group hit 16 distinct
// banks; GF(2^8) products use log/exp tables; the embedding into GF(2^128) is done once per group
// and bit (8 multiplies per group instead of 64).  The MLE-check rounds fuse the fold by the previous
// challenge, the truncation of the eq tensor and the next round's evaluation in one pass.
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "cs.h"
#include "dev_transcript.cuh"
#include "pdl.cuh"
#include "gf128.cuh"
#include "gf_reduce.cuh"
#include "internal.h"
#include "kernels.h"
#include "reductions.h"
#include "transcript.h"

using namespace bgpu;

namespace {

typedef unsigned __int128 u128h;

// ------------------------------------------------------------------ host constants

uint8_t aes_mul_h(uint8_t a, uint8_t b) {
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

uint8_t aes_inv_h(uint8_t a) {
  uint8_t r = 1;
  for (int i = 0; i < 254; i++) r = aes_mul_h(r, a);
  return a ? r : 0;
}

struct AndConstants {
  uint32_t ntt[8][256][16];  // [byte index][byte value][point group] -> 4 GF(2^8) values
  uint8_t mul_eq[8][256];    // x * eq_small[j]
  uint8_t log[256];
  uint8_t exp[512];
  u128h phi[256];            // the GF(2^8) -> GF(2^128) embedding
};

// The embedding is fixed by the image of the AES generator x (byte 0x02), the entry for 0x02 of
// `From<AESTowerField8b> for BinaryField128bGhash` (verifier/field/src/ghash.rs:520-530); the other
// entries follow by linearity.
const u128h kAesXInGhash = ((u128h)0x0dcb364640a222feull << 64) | (u128h)0x6b8330483c2e9849ull;

const AndConstants& and_constants() {
  static AndConstants C;
  static std::once_flag once;
  std::call_once(once, [] {
    // Lagrange basis over {0..63} evaluated at 64 + k: M[k][t]
    uint8_t denom = 1;
    for (int u = 1; u < 64; u++) denom = aes_mul_h(denom, (uint8_t)u);
    const uint8_t dinv = aes_inv_h(denom);
    static uint8_t M[64][64];
    for (int k = 0; k < 64; k++)
      for (int t = 0; t < 64; t++) {
        uint8_t num = 1;
        for (int s = 0; s < 64; s++)
          if (s != t) num = aes_mul_h(num, (uint8_t)((64 + k) ^ s));
        M[k][t] = aes_mul_h(num, dinv);
      }
    for (int bi = 0; bi < 8; bi++)
      for (int bv = 0; bv < 256; bv++)
        for (int kq = 0; kq < 16; kq++) {
          uint32_t packed = 0;
          for (int l = 0; l < 4; l++) {
            uint8_t acc = 0;
            for (int j = 0; j < 8; j++)
              if ((bv >> j) & 1) acc ^= M[4 * kq + l][8 * bi + j];
            packed |= (uint32_t)acc << (8 * l);
          }
          C.ntt[bi][bv][kq] = packed;
        }
    // eq_small = eq tensor of (2, 4, 16) in GF(2^8)
    const uint8_t r[3] = {0x2, 0x4, 0x10};
    uint8_t eq[8] = {1};
    uint32_t len = 1;
    for (int i = 0; i < 3; i++) {
      for (uint32_t j = 0; j < len; j++) {
        uint8_t prod = aes_mul_h(eq[j], r[i]);
        eq[j] ^= prod;
        eq[len + j] = prod;
      }
      len <<= 1;
    }
    for (int j = 0; j < 8; j++)
      for (int x = 0; x < 256; x++) C.mul_eq[j][x] = aes_mul_h((uint8_t)x, eq[j]);
    uint8_t e = 1;
    for (int i = 0; i < 255; i++) {
      C.exp[i] = e;
      C.exp[i + 255] = e;
      C.log[e] = (uint8_t)i;
      e = aes_mul_h(e, 3);
    }
    C.exp[510] = C.exp[0];
    C.exp[511] = C.exp[1];
    C.log[0] = 0;
    u128h pw[8];
    pw[0] = 1;
    for (int i = 1; i < 8; i++) pw[i] = host_gf_mul(pw[i - 1], kAesXInGhash);
    for (int b = 0; b < 256; b++) {
      u128h acc = 0;
      for (int i = 0; i < 8; i++)
        if ((b >> i) & 1) acc ^= pw[i];
      C.phi[b] = acc;
    }
  });
  return C;
}

// Lagrange basis of {phi(t) : t < 2^dim} at x (univariate_lagrange.rs:22-66).
void lagrange_b128(uint32_t dim, u128h x, u128h* out) {
  const AndConstants& C = and_constants();
  const uint32_t n = 1u << dim;
  // 1 / prod_{u != 0} phi(u): a constant per dimension, computed once
  static const std::vector<u128h> dinvs = [&C] {
    std::vector<u128h> v(9);
    for (uint32_t d = 0; d <= 8; d++) {
      u128h denom = 1;
      for (uint32_t u = 1; u < (1u << d); u++) denom = host_gf_mul(denom, C.phi[u & 255]);
      v[d] = host_gf_inv(denom);
    }
    return v;
  }();
  const u128h dinv = dinvs[dim];
  std::vector<u128h> diff(n), suffix(n + 1);
  for (uint32_t s = 0; s < n; s++) diff[s] = x ^ C.phi[s];
  suffix[n] = 1;
  for (int s = (int)n - 1; s >= 0; s--) suffix[s] = host_gf_mul(suffix[s + 1], diff[s]);
  u128h prefix = 1;
  for (uint32_t t = 0; t < n; t++) {
    out[t] = host_gf_mul(host_gf_mul(prefix, suffix[t + 1]), dinv);
    prefix = host_gf_mul(prefix, diff[t]);
  }
}

// ------------------------------------------------------------------ device tables

struct DevAndTables {
  uint32_t* ntt = nullptr;  // 8 * 256 * 16
  uint8_t* mul_eq = nullptr;
  uint8_t* log = nullptr;
  uint8_t* exp = nullptr;
};

struct PhiPowers {
  uint4 p[8];
};

constexpr int kUniThreads = 512;
constexpr int kUniLanes = 8;  // lanes per word, 8 of the 64 points each
constexpr int kSlots = kUniThreads / kUniLanes;
constexpr size_t kUniSmem = sizeof(uint32_t) * 8 * 256 * 16 + 8 * 256 + 256 + 512 +
                            sizeof(uint4) * kSlots * 8;

__device__ __forceinline__ uint8_t gf8_mul(const uint8_t* s_log, const uint8_t* s_exp, uint32_t a,
                                           uint32_t b) {
  return (a && b) ? s_exp[s_log[a] + s_log[b]] : 0;
}

// The word's extension values at points 8 kq .. 8 kq + 7: one 8-byte row per byte of the word.
__device__ __forceinline__ uint2 word_ntt(const uint2* sT2, uint64_t w, uint32_t kq) {
  uint2 acc = make_uint2(0u, 0u);
#pragma unroll
  for (int bi = 0; bi < 8; bi++) {
    const uint2 t = sT2[((bi << 8) | (uint32_t)((w >> (8 * bi)) & 255)) * 8 + kq];
    acc.x ^= t.x;
    acc.y ^= t.y;
  }
  return acc;
}

__device__ __forceinline__ uint32_t and_bytes(const uint8_t* s_log, const uint8_t* s_exp,
                                              const uint8_t* mj, uint32_t A, uint32_t B,
                                              uint32_t C) {
  uint32_t v = 0;
#pragma unroll
  for (int l = 0; l < 4; l++) {
    const uint32_t x = gf8_mul(s_log, s_exp, (A >> (8 * l)) & 255, (B >> (8 * l)) & 255) ^
                       ((C >> (8 * l)) & 255);
    v ^= (uint32_t)mj[x] << (8 * l);
  }
  return v;
}

__global__ void __launch_bounds__(kUniThreads, 1)
    univariate_round_kernel(const uint64_t* __restrict__ wa, const uint64_t* __restrict__ wb,
                            const uint64_t* __restrict__ wc, const uint4* __restrict__ eq_big,
                            uint64_t n_chunks, DevAndTables tab, PhiPowers phi,
                            uint32_t* __restrict__ out) {
  extern __shared__ uint4 smem4[];
  uint32_t* sT = reinterpret_cast<uint32_t*>(smem4);
  const uint2* sT2 = reinterpret_cast<const uint2*>(sT);
  uint8_t* s_mul = reinterpret_cast<uint8_t*>(sT + 8 * 256 * 16);
  uint8_t* s_log = s_mul + 8 * 256;
  uint8_t* s_exp = s_log + 256;
  uint4* s_P = reinterpret_cast<uint4*>(s_exp + 512);  // [kSlots][8], 16-byte aligned
  for (uint32_t i = threadIdx.x; i < 8 * 256 * 16; i += blockDim.x) sT[i] = tab.ntt[i];
  for (uint32_t i = threadIdx.x; i < 8 * 256; i += blockDim.x) s_mul[i] = tab.mul_eq[i];
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) s_log[i] = tab.log[i];
  for (uint32_t i = threadIdx.x; i < 512; i += blockDim.x) s_exp[i] = tab.exp[i];
  const uint32_t kq = threadIdx.x & (kUniLanes - 1), slot = threadIdx.x / kUniLanes;
  uint4 acc[8];
#pragma unroll
  for (int l = 0; l < 8; l++) acc[l] = gf_zero();
  const uint64_t stride = (uint64_t)gridDim.x * kSlots;
  const uint64_t iters = (n_chunks + stride - 1) / stride;
  for (uint64_t it = 0; it < iters; it++) {
    const uint64_t chunk = it * stride + (uint64_t)blockIdx.x * kSlots + slot;
    const bool valid = chunk < n_chunks;
    __syncthreads();
    if (valid) s_P[slot * 8 + kq] = gf_mul(eq_big[chunk], phi.p[kq]);
    __syncthreads();
    if (valid) {
      uint32_t vlo = 0, vhi = 0;
#pragma unroll 1
      for (int j = 0; j < 8; j++) {
        const uint64_t i = chunk * 8 + j;
        const uint2 A = word_ntt(sT2, __ldg(wa + i), kq);
        const uint2 B = word_ntt(sT2, __ldg(wb + i), kq);
        const uint2 Cv = word_ntt(sT2, __ldg(wc + i), kq);
        const uint8_t* mj = s_mul + (j << 8);
        vlo ^= and_bytes(s_log, s_exp, mj, A.x, B.x, Cv.x);
        vhi ^= and_bytes(s_log, s_exp, mj, A.y, B.y, Cv.y);
      }
#pragma unroll
      for (int l = 0; l < 8; l++) {
        const uint32_t v = ((l < 4 ? vlo : vhi) >> (8 * (l & 3))) & 255;
#pragma unroll
        for (int b = 0; b < 8; b++) {
          const uint32_t m = 0u - ((v >> b) & 1u);
          const uint4 P = s_P[slot * 8 + b];
          acc[l].x ^= P.x & m;
          acc[l].y ^= P.y & m;
          acc[l].z ^= P.z & m;
          acc[l].w ^= P.w & m;
        }
      }
    }
  }
  // reduce over the slots: reuse the table area as [64 points][kSlots] accumulators
  __syncthreads();
  uint4* red = smem4;
#pragma unroll
  for (int l = 0; l < 8; l++) red[(8 * kq + l) * kSlots + slot] = acc[l];
  __syncthreads();
  if (threadIdx.x < 64) {
    uint4 s = gf_zero();
    for (int q = 0; q < kSlots; q++) gf_add_into(s, red[threadIdx.x * kSlots + q]);
    uint32_t* dst = out + 4 * threadIdx.x;
    if (s.x) atomicXor(dst + 0, s.x);
    if (s.y) atomicXor(dst + 1, s.y);
    if (s.z) atomicXor(dst + 2, s.z);
    if (s.w) atomicXor(dst + 3, s.w);
  }
}

struct Lag64 {
  uint4 l[64];
};

// out[i] = sum over set bits t of words[i] of lag[t], through 8 byte tables of subset sums.
__global__ void __launch_bounds__(256)
    fold_words_kernel(const uint64_t* __restrict__ words, uint64_t n, Lag64 lag,
                      uint4* __restrict__ out) {
  __shared__ uint4 tab[8][256];
  for (uint32_t i = threadIdx.x; i < 8 * 256; i += blockDim.x) {
    const uint32_t bi = i >> 8, bv = i & 255;
    uint4 acc = gf_zero();
    for (int j = 0; j < 8; j++)
      if ((bv >> j) & 1) gf_add_into(acc, lag.l[8 * bi + j]);
    tab[bi][bv] = acc;
  }
  __syncthreads();
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t w = __ldg(words + i);
    uint4 acc = gf_zero();
#pragma unroll
    for (int bi = 0; bi < 8; bi++) gf_add_into(acc, tab[bi][(w >> (8 * bi)) & 255]);
    out[i] = acc;
  }
}

__device__ __forceinline__ uint4 shfl_gf(uint4 v, int m) {
  v.x = __shfl_xor_sync(0xffffffffu, v.x, m);
  v.y = __shfl_xor_sync(0xffffffffu, v.y, m);
  v.z = __shfl_xor_sync(0xffffffffu, v.z, m);
  v.w = __shfl_xor_sync(0xffffffffu, v.w, m);
  return v;
}

__device__ __forceinline__ void reduce2_atomic(uint4 v0, uint4 v1, uint32_t* dst) {
  __shared__ uint4 red[2][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) {
    gf_add_into(v0, shfl_gf(v0, m));
    gf_add_into(v1, shfl_gf(v1, m));
  }
  if (lane == 0) {
    red[0][warp] = v0;
    red[1][warp] = v1;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    uint4 a = lane < nw ? red[0][lane] : gf_zero();
    uint4 b = lane < nw ? red[1][lane] : gf_zero();
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) {
      gf_add_into(a, shfl_gf(a, m));
      gf_add_into(b, shfl_gf(b, m));
    }
    if (lane == 0) {
      const uint32_t v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
      for (int q = 0; q < 8; q++)
        if (v[q]) atomicXor(dst + q, v[q]);
    }
  }
}

// Round evaluation without a fold: columns of length 2*half, eq of length half.
__global__ void __launch_bounds__(256)
    and_mle_eval_kernel(const uint4* __restrict__ fa, const uint4* __restrict__ fb,
                        const uint4* __restrict__ fc, const uint4* __restrict__ eq, uint64_t half,
                        uint32_t* __restrict__ out) {
  u256 s1 = {0, 0, 0, 0}, sinf = {0, 0, 0, 0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < half;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 a0 = fa[i], a1 = fa[half + i], b0 = fb[i], b1 = fb[half + i], c1 = fc[half + i];
    const uint4 e = eq[i];
    xor_into(s1, clmul128(e, gf_add(gf_mul(a1, b1), c1)));
    xor_into(sinf, clmul128(e, gf_mul(gf_add(a0, a1), gf_add(b0, b1))));
  }
  reduce2_atomic(reduce256(s1), reduce256(sinf), out);
}

// Fold the three columns (length size) by the previous round's challenge, truncate eq (length
// size/2 -> size/4) and evaluate the next round.  Each folded position j < size/4 belongs to a
// pair of adjacent lanes: the odd lane folds a, b, c at j and truncates eq there, the even lane
// folds them at j + size/4, and each forms one of the two products (the even lane y_1's
// e (a1 b1 + c1), the odd lane y_inf's e (a0 + a1)(b0 + b1)); shuffles bring a1, b1 to the odd
// lane and e to the even one.  The six products by r (read from r_ptr) go through r's nibble
// tables, which each block builds in shared memory.
__global__ void __launch_bounds__(256)
    and_mle_fold_eval_kernel(uint4* __restrict__ fa, uint4* __restrict__ fb, uint4* __restrict__ fc,
                             uint4* __restrict__ eq, uint64_t size, const uint4* __restrict__ r_ptr,
                             uint32_t* __restrict__ out) {
  __shared__ NibbleTable tab;
  __shared__ uint4 basis[128];
  pdl_wait();
  pdl_trigger();
  nibble_table_build(tab, basis, *r_ptr);
  const uint64_t h = size >> 1, q = size >> 2;
  const uint32_t odd = threadIdx.x & 1;
  u256 acc = {0, 0, 0, 0};
  const uint64_t all = (uint64_t)gridDim.x * blockDim.x;
  // warp-uniform sweeps: every lane of a warp runs the same iterations (shuffles below)
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u); base < 2 * q;
       base += all) {
    const uint64_t j = (base + (threadIdx.x & 31)) >> 1;
    const bool live = j < q;
    uint4 f[3] = {gf_zero(), gf_zero(), gf_zero()}, e = gf_zero();
    if (live) {
      const uint64_t pos = odd ? j : q + j;
      uint4* cols[3] = {fa, fb, fc};
#pragma unroll
      for (int c = 0; c < 3; c++) {
        uint4* col = cols[c];
        const uint4 lo = col[pos], hi = col[h + pos];
        f[c] = gf_add(lo, gf_mul_nibble(tab, gf_add(hi, lo)));
        col[pos] = f[c];
      }
      if (odd) {
        e = gf_add(eq[j], eq[q + j]);
        eq[j] = e;
      }
    }
    // (qualified: this file's own shfl_gf is the xor-butterfly one)
    const uint4 pa = bgpu::shfl_gf(f[0], 0, 2), pb = bgpu::shfl_gf(f[1], 0, 2);
    e = bgpu::shfl_gf(e, 1, 2);
    // one product chain per lane, selected without divergence (zero on dead lanes)
    const uint4 x = odd ? gf_add(f[0], pa) : f[0], y = odd ? gf_add(f[1], pb) : f[1];
    xor_into(acc, clmul128(e, gf_add(gf_mul(x, y), odd ? gf_zero() : f[2])));
  }
  const uint4 v = reduce256(acc);
  reduce2_atomic(odd ? gf_zero() : v, odd ? v : gf_zero(), out);
}

// The small rounds of and_mle_fold_eval_kernel (no nibble tables) on eight lanes per position j:
// lanes 0..5 fold column k / 2 at j (k even) or q + j (k odd) by r, lane 6 truncates eq at j,
// the folded values and eq are shared by shuffles and lanes 0 and 1 form the two products.
// Three dependent multiplies per lane instead of ten on one thread.
__global__ void __launch_bounds__(256)
    and_mle_fold_eval_lanes_kernel(uint4* __restrict__ fa, uint4* __restrict__ fb,
                                   uint4* __restrict__ fc, uint4* __restrict__ eq, uint64_t size,
                                   const uint4* __restrict__ r_ptr, uint32_t* __restrict__ out) {
  pdl_wait();
  pdl_trigger();
  const uint64_t h = size >> 1, q = size >> 2;
  const uint4 r = *r_ptr;
  const uint32_t k = threadIdx.x & 7;
  uint4 s1 = gf_zero(), sinf = gf_zero();
  const uint64_t all = (uint64_t)gridDim.x * blockDim.x;
  // warp-uniform sweeps: every lane of a warp runs the same iterations (shuffles below)
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u); base < 8 * q;
       base += all) {
    const uint64_t j = (base + (threadIdx.x & 31)) >> 3;
    const bool live = j < q;
    uint4 f = gf_zero();
    if (live && k < 6) {
      uint4* col = k < 2 ? fa : k < 4 ? fb : fc;
      const uint64_t pos = j + ((k & 1) ? q : 0);
      const uint4 lo = col[pos];
      f = gf_add(lo, gf_mul_nl(r, gf_add(col[h + pos], lo)));
      col[pos] = f;
    } else if (live && k == 6) {
      f = gf_add(eq[j], eq[q + j]);
      eq[j] = f;
    }
    // (qualified: this file's own shfl_gf is the xor-butterfly one)
    const uint4 a0 = bgpu::shfl_gf(f, 0, 8), a1 = bgpu::shfl_gf(f, 1, 8);
    const uint4 b0 = bgpu::shfl_gf(f, 2, 8), b1 = bgpu::shfl_gf(f, 3, 8);
    const uint4 c1 = bgpu::shfl_gf(f, 5, 8), e = bgpu::shfl_gf(f, 6, 8);
    if (live && k == 0) gf_add_into(s1, gf_mul_nl(e, gf_add(gf_mul_nl(a1, b1), c1)));
    if (live && k == 1)
      gf_add_into(sinf, gf_mul_nl(e, gf_mul_nl(gf_add(a0, a1), gf_add(b0, b1))));
  }
  reduce2_atomic(s1, sinf, out);
}

// Per-round constants of the MLE-check: the eq coordinate alpha the round binds and
// 1 / (1 + alpha), both known before the loop starts.
struct AndRoundConst {
  uint4 alpha, inv_one_plus_alpha;
};

// The Fiat-Shamir step of one MLE-check round, on the device: the round's sums (y_1, y_inf) ->
// the round polynomial by RoundEvals2::interpolate_eq (prover/prover/src/protocols/sumcheck/
// round_evals.rs:80-86) -> the truncated proof (c_1, c_2) (mlecheck::RoundProof::truncate) ->
// the challenge r -> the next claim c_0 + c_1 r + c_2 r^2.  One warp runs the chain.
__global__ void __launch_bounds__(32)
    and_round_finish_kernel(TranscriptState* __restrict__ ts, uint8_t* __restrict__ tape,
                            const uint4* __restrict__ ys, const AndRoundConst* __restrict__ rc,
                            uint4* __restrict__ claim, uint4* __restrict__ r_out) {
  pdl_wait();
  pdl_trigger();
  {
    DevTr st;
    st.load(ts);
    const uint4 y1 = ys[0], yinf = ys[1];
    const uint4 y0 =
        gf_mul_warp(gf_add(*claim, gf_mul_warp(y1, rc->alpha)), rc->inv_one_plus_alpha);
    const uint4 c0 = y0, c2 = yinf, c1 = gf_add(gf_add(y1, c0), c2);
    const uint4 msg[2] = {c1, c2};
    st.message_elems(tape, msg, 2);
    const uint4 r = st.sample_elem();
    *r_out = r;
    *claim = gf_add(c0, gf_mul_warp(r, gf_add(c1, gf_mul_warp(c2, r))));
    st.store(ts);
  }
}

// The small last rounds of the MLE-check in one CTA (see bivariate_tail_kernel): per round fold
// the three columns (length len -> len/2) by the previous challenge, truncate eq (len/2 -> len/4),
// evaluate (y_1, y_inf) and let warp 0 run and_round_finish_kernel's Fiat-Shamir step with
// the round's constants rc[k].
constexpr int kAndTailThreads = 512;
__global__ void __launch_bounds__(kAndTailThreads)
    and_tail_kernel(TranscriptState* __restrict__ ts, uint8_t* __restrict__ tape,
                    uint4* __restrict__ fa, uint4* __restrict__ fb, uint4* __restrict__ fc,
                    uint4* __restrict__ eq, uint64_t len, uint32_t n_rounds,
                    const uint4* __restrict__ r_first, const AndRoundConst* __restrict__ rc,
                    uint4* __restrict__ claim, uint4* __restrict__ chal) {
  pdl_wait();
  pdl_trigger();
  __shared__ uint4 r_sh;
  DevTr st;
  uint4 cl = gf_zero();
  if (threadIdx.x < 32) {
    st.load(ts);
    cl = *claim;
    r_sh = *r_first;
  }
  __syncthreads();
  for (uint32_t k = 0; k < n_rounds; k++) {
    const uint4 r = r_sh;
    const uint64_t h = len >> 1, q = len >> 2;
    for (uint64_t j = threadIdx.x; j < h; j += blockDim.x) {
      const uint4 a0 = fa[j], b0 = fb[j], c0 = fc[j];
      fa[j] = gf_add(a0, gf_mul_nl(r, gf_add(fa[h + j], a0)));
      fb[j] = gf_add(b0, gf_mul_nl(r, gf_add(fb[h + j], b0)));
      fc[j] = gf_add(c0, gf_mul_nl(r, gf_add(fc[h + j], c0)));
    }
    for (uint64_t j = threadIdx.x; j < q; j += blockDim.x) eq[j] = gf_add(eq[j], eq[q + j]);
    len = h;
    __syncthreads();
    uint4 v[2] = {gf_zero(), gf_zero()};
    for (uint64_t j = threadIdx.x; j < q; j += blockDim.x) {
      const uint4 e = eq[j];
      const uint4 a0 = fa[j], a1 = fa[q + j], b0 = fb[j], b1 = fb[q + j], c1 = fc[q + j];
      gf_add_into(v[0], gf_mul_nl(e, gf_add(gf_mul_nl(a1, b1), c1)));
      gf_add_into(v[1], gf_mul_nl(e, gf_mul_nl(gf_add(a0, a1), gf_add(b0, b1))));
    }
    block_xor_sum<2>(v);
    if (threadIdx.x < 32) {
      const AndRoundConst c = rc[k];
      const uint4 y1 = v[0], yinf = v[1];
      const uint4 y0 = gf_mul_warp(gf_add(cl, gf_mul_warp(y1, c.alpha)), c.inv_one_plus_alpha);
      const uint4 c0 = y0, c2 = yinf, c1 = gf_add(gf_add(y1, c0), c2);
      const uint4 msg[2] = {c1, c2};
      st.message_elems(tape, msg, 2);
      const uint4 rr = st.sample_elem();
      chal[k] = rr;
      cl = gf_add(c0, gf_mul_warp(rr, gf_add(c1, gf_mul_warp(c2, rr))));
      r_sh = rr;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    st.store(ts);
    *claim = cl;
  }
}

struct DevTablesHolder {
  DevAndTables t;
  int device = -1;
};

int device_tables(DevAndTables& out) {
  static std::mutex m;
  static DevTablesHolder holders[64];
  int dev = 0;
  BGPU_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(BINIUS_E_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> g(m);
  DevTablesHolder& h = holders[dev];
  if (h.device != dev) {
    const AndConstants& C = and_constants();
    BGPU_CUDA(cudaMalloc(&h.t.ntt, sizeof(C.ntt)));
    BGPU_CUDA(cudaMemcpy(h.t.ntt, C.ntt, sizeof(C.ntt), cudaMemcpyHostToDevice));
    BGPU_CUDA(cudaMalloc(&h.t.mul_eq, sizeof(C.mul_eq) + 256 + 512));
    h.t.log = h.t.mul_eq + sizeof(C.mul_eq);
    h.t.exp = h.t.log + 256;
    BGPU_CUDA(cudaMemcpy(h.t.mul_eq, C.mul_eq, sizeof(C.mul_eq), cudaMemcpyHostToDevice));
    BGPU_CUDA(cudaMemcpy(h.t.log, C.log, 256, cudaMemcpyHostToDevice));
    BGPU_CUDA(cudaMemcpy(h.t.exp, C.exp, 512, cudaMemcpyHostToDevice));
    BGPU_CUDA(cudaFuncSetAttribute(univariate_round_kernel,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUniSmem));
    h.device = dev;
  }
  out = h.t;
  return BINIUS_OK;
}

uint4 to_uint4(u128h v) {
  uint4 r;
  memcpy(&r, &v, 16);
  return r;
}
u128h from_bytes16(const uint8_t* b) {
  u128h v;
  memcpy(&v, b, 16);
  return v;
}

unsigned grid_for(uint64_t n, unsigned threads, unsigned cap = 148 * 8) {
  uint64_t g = (n + threads - 1) / threads;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, cap));
}

}  // namespace

namespace bgpu {

void lagrange_phi(uint32_t dim, hu128 x, hu128* out) { lagrange_b128(dim, x, out); }
hu128 phi_elem(uint32_t b) { return and_constants().phi[b & 255]; }

int and_mle_eval(const uint4* d_a, const uint4* d_b, const uint4* d_c, const uint4* d_eq,
                 uint64_t half, uint32_t* d_out8, cudaStream_t s) {
  BGPU_CUDA(cudaMemsetAsync(d_out8, 0, 32, s));
  and_mle_eval_kernel<<<grid_for(half, 256), 256, 0, s>>>(d_a, d_b, d_c, d_eq, half, d_out8);
  BGPU_LAUNCH_CHECK("and_mle_eval_kernel");
  count_launch();
  return BINIUS_OK;
}

int fold_words64(const uint64_t* d_words, uint64_t n, const hu128* vec64, uint4* d_out,
                 cudaStream_t s) {
  if (n == 0) return BINIUS_OK;
  Lag64 l64;
  for (int i = 0; i < 64; i++) l64.l[i] = to_uint4(vec64[i]);
  fold_words_kernel<<<grid_for(n, 256), 256, 0, s>>>(d_words, n, l64, d_out);
  BGPU_LAUNCH_CHECK("fold_words_kernel");
  count_launch();
  return BINIUS_OK;
}

// d_witness: committed_total_len words; writes the AND reduction's transcript messages.
void and_prep_free(AndPrep& p, cudaStream_t s) {
  dev_free(p.words, s);
  dev_free(p.eq_big, s);
  dev_free(p.fcols, s);
  dev_free(p.eq, s);
  dev_free(p.d_acc, s);
  dev_free(p.dev, s);
  p = AndPrep();
}

int and_reduction_begin(const binius_cs* cs, const uint64_t* d_witness, AndPrep& p,
                        cudaStream_t s) {
  const uint64_t N = cs->and_ops.n_constraints;
  uint32_t log_n = 0;
  while ((1ull << log_n) < N) log_n++;
  if (log_n < 3) return set_error(BINIUS_E_ARG, "AND reduction needs at least 8 constraints");
  p = AndPrep();
  cudaError_t e;
  if ((e = dev_alloc(&p.words, 8 * 3 * N, s)) != cudaSuccess ||
      (e = dev_alloc(&p.eq_big, 16 * (N >> 3), s)) != cudaSuccess ||
      (e = dev_alloc(&p.fcols, 16 * 3 * N, s)) != cudaSuccess ||
      (e = dev_alloc(&p.eq, 16 * (N / 2), s)) != cudaSuccess ||
      // 64 univariate slots, then one (y_1, y_inf) slot pair per MLE-check round, zeroed once
      (e = dev_alloc(&p.d_acc, 16 * (64 + 2 * (log_n + 1)), s)) != cudaSuccess ||
      // round constants (2 per round), the claim slot pair, the challenges
      (e = dev_alloc(&p.dev, 16 * (2 * (log_n + 1) + log_n), s)) != cudaSuccess) {
    and_prep_free(p, s);
    return cuda_error(e, "AND reduction buffers");
  }
  if (int rc = eval_operands(cs->and_ops, d_witness, p.words, s)) {
    and_prep_free(p, s);
    return rc;
  }
  return BINIUS_OK;
}

int and_reduction_prove(const binius_cs* cs, const uint64_t* d_witness, Transcript& t,
                        AndResult& res, cudaStream_t s) {
  AndPrep p;
  if (int rc = and_reduction_begin(cs, d_witness, p, s)) return rc;
  return and_reduction_finish(cs, p, t, res, s);
}

int and_reduction_finish(const binius_cs* cs, AndPrep& p, Transcript& t, AndResult& res,
                         cudaStream_t s) {
  const uint64_t N = cs->and_ops.n_constraints;
  uint32_t log_n = 0;
  while ((1ull << log_n) < N) log_n++;
  const uint64_t n_chunks = N >> 3;
  const AndConstants& C = and_constants();
  uint64_t* const words = p.words;
  uint4* const eq_big = p.eq_big;
  uint4* const fcols = p.fcols;
  uint4* const eq = p.eq;
  uint32_t* const d_acc = p.d_acc;
  uint4* const dev = p.dev;
  DevAndTables tab;
  int rc = device_tables(tab);
  do {
    if (rc) break;
    // big-field zerocheck challenges
    std::vector<uint8_t> big(16 * (log_n - 3));
    for (uint32_t i = 0; i < log_n - 3; i++) t.sample_elem(big.data() + 16 * i);
    if ((rc = eq_tensor(reinterpret_cast<const uint4*>(big.data()), log_n - 3, eq_big, s))) break;
    // univariate round
    PhiPowers pw;
    for (int i = 0; i < 8; i++) pw.p[i] = to_uint4(C.phi[1u << i]);
    cudaError_t e = cudaMemsetAsync(d_acc, 0, 16 * (64 + 2 * (log_n + 1)), s);
    if (e != cudaSuccess) { rc = cuda_error(e, "memset"); break; }
    univariate_round_kernel<<<148, kUniThreads, kUniSmem, s>>>(words, words + N, words + 2 * N,
                                                              eq_big, n_chunks, tab, pw, d_acc);
    e = cudaGetLastError();
    if (e != cudaSuccess) { rc = cuda_error(e, "univariate_round_kernel"); break; }
    count_launch();
    uint8_t msg[64 * 16];
    if ((rc = read_sync(msg, d_acc, sizeof(msg), s))) break;
    t.message(msg, sizeof(msg));
    uint8_t zb[16];
    t.sample_elem(zb);
    const u128h z = from_bytes16(zb);
    res.z = z;
    // fold the words at z
    u128h lag[128];
    lagrange_b128(6, z, lag);
    Lag64 l64;
    for (int i = 0; i < 64; i++) l64.l[i] = to_uint4(lag[i]);
    fold_words_kernel<<<grid_for(3 * N, 256), 256, 0, s>>>(words, 3 * N, l64, fcols);
    e = cudaGetLastError();
    if (e != cudaSuccess) { rc = cuda_error(e, "fold_words_kernel"); break; }
    count_launch();
    // claim: the message (zero on the base domain) evaluated at z over the 128-point domain
    lagrange_b128(7, z, lag);
    u128h sum = 0;
    for (int k = 0; k < 64; k++) sum ^= host_gf_mul(from_bytes16(msg + 16 * k), lag[64 + k]);
    // MLE-check over the point [phi(2), phi(4), phi(16)] ++ big
    std::vector<u128h> point{C.phi[2], C.phi[4], C.phi[16]};
    for (uint32_t i = 0; i < log_n - 3; i++) point.push_back(from_bytes16(big.data() + 16 * i));
    std::vector<uint4> pt4(point.size());
    for (size_t i = 0; i < point.size(); i++) pt4[i] = to_uint4(point[i]);
    if ((rc = eq_tensor(pt4.data(), log_n - 1, eq, s))) break;
    uint4* fa = fcols;
    uint4* fb = fcols + N;
    uint4* fc = fcols + 2 * N;
    // The round loop runs on the device transcript: per round one evaluation kernel and one
    // finish kernel, no host round trip.  dev holds the claim, the round constants (rounds in
    // order log_n .. 1) and the challenges.
    std::vector<AndRoundConst> consts(log_n + 1);
    for (uint32_t n_rem = log_n; n_rem > 0; n_rem--) {
      const u128h alpha = point[n_rem - 1];
      consts[log_n - n_rem] = {to_uint4(alpha), to_uint4(host_gf_inv(1 ^ alpha))};
    }
    consts[log_n].alpha = to_uint4(sum);  // the initial claim rides in the spare slot
    AndRoundConst* d_consts = reinterpret_cast<AndRoundConst*>(dev);
    uint4* d_claim = dev + 2 * log_n;
    uint4* d_chal = dev + 2 * (log_n + 1);
    e = cudaMemcpyAsync(d_consts, consts.data(), sizeof(AndRoundConst) * (log_n + 1),
                        cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) { rc = cuda_error(e, "round constants"); break; }
    DeviceTranscript dt;
    if ((rc = dt.begin(t, s))) break;
    // rounds whose fold starts from at most tail_max_len() elements run in the single-CTA tail
    uint32_t tail_n = 0;  // n_rem of the first tail round (0: no tail)
    for (uint32_t n_rem = log_n - 1; n_rem > 0; n_rem--)
      if ((2ull << n_rem) <= tail_max_len()) {
        tail_n = n_rem;
        break;
      }
    for (uint32_t n_rem = log_n; n_rem > tail_n; n_rem--) {
      const uint32_t k = log_n - n_rem;
      uint32_t* acc = d_acc + 4 * (64 + 2 * k);
      const uint64_t size = 1ull << n_rem;
      if (n_rem == log_n) {
        and_mle_eval_kernel<<<grid_for(size / 2, 256), 256, 0, s>>>(fa, fb, fc, eq, size / 2,
                                                                    acc);
        e = cudaGetLastError();
      } else if (size * 2 >= kMulTableMinSize) {
        // two lanes per folded position (size of them)
        e = launch_pdl(and_mle_fold_eval_kernel, grid_for(size, 256), 256, 0, s, fa, fb, fc,
                       eq, size * 2, (const uint4*)(d_chal + k - 1), acc);
      } else {
        e = launch_pdl(and_mle_fold_eval_lanes_kernel, grid_for(4 * size, 256), 256, 0, s, fa,
                       fb, fc, eq, size * 2, (const uint4*)(d_chal + k - 1), acc);
      }
      if (e != cudaSuccess) { rc = cuda_error(e, "AND MLE-check round"); break; }
      e = launch_pdl(and_round_finish_kernel, 1, 32, 0, s, dt.state(), dt.tape(),
                     reinterpret_cast<const uint4*>(acc), (const AndRoundConst*)(d_consts + k),
                     d_claim, d_chal + k);
      if (e != cudaSuccess) { rc = cuda_error(e, "and_round_finish_kernel"); break; }
      count_launch(2);
    }
    if (rc) break;
    if (tail_n) {
      const uint32_t k0 = log_n - tail_n;
      e = launch_pdl(and_tail_kernel, 1, kAndTailThreads, 0, s, dt.state(), dt.tape(), fa, fb, fc,
                     eq, 2ull << tail_n, tail_n, (const uint4*)(d_chal + k0 - 1),
                     (const AndRoundConst*)(d_consts + k0), d_claim, d_chal + k0);
      if (e != cudaSuccess) { rc = cuda_error(e, "and_tail_kernel"); break; }
      count_launch();
    }
    // one read: the transcript, the challenges and the length-2 columns before the final fold
    std::vector<u128h> challenges(log_n);
    uint8_t last[96];  // (lo, hi) of a, b, c
    StagedReads rd(s);
    if ((rc = dt.read(rd, 32 * log_n))) break;
    if ((rc = rd.add(challenges.data(), d_chal, 16 * log_n))) break;
    for (int c = 0; c < 3 && !rc; c++) rc = rd.add(last + 32 * c, fcols + (uint64_t)c * N, 32);
    if (rc || (rc = rd.wait()) || (rc = dt.finish(t))) break;
    // final fold of the length-2 columns by the last challenge: lo + r (hi - lo)
    uint8_t ev[48];
    const u128h r_last = challenges[log_n - 1];
    for (int c = 0; c < 3; c++) {
      const u128h lo = from_bytes16(last + 32 * c), hi = from_bytes16(last + 32 * c + 16);
      const u128h v = lo ^ host_gf_mul(r_last, hi ^ lo);
      memcpy(ev + 16 * c, &v, 16);
    }
    t.message(ev, 48);
    res.a_eval = from_bytes16(ev);
    res.b_eval = from_bytes16(ev + 16);
    res.c_eval = from_bytes16(ev + 32);
    res.eval_point.assign(challenges.rbegin(), challenges.rend());
  } while (0);
  and_prep_free(p, s);
  return rc;
}

}  // namespace bgpu

extern "C" {

int binius_and_reduction_prove(const binius_cs* cs, const void* d_witness,
                               binius_transcript* transcript, void* h_out_meta,
                               void* h_out_point, void* stream) {
  BGPU_ARG(cs && d_witness && transcript, "NULL argument");
  AndResult res;
  int rc = and_reduction_prove(cs, static_cast<const uint64_t*>(d_witness), transcript->t, res,
                               as_stream(stream));
  if (rc) return rc;
  if (h_out_meta) {
    uint8_t* m = static_cast<uint8_t*>(h_out_meta);
    memcpy(m, &res.a_eval, 16);
    memcpy(m + 16, &res.b_eval, 16);
    memcpy(m + 32, &res.c_eval, 16);
    memcpy(m + 48, &res.z, 16);
  }
  if (h_out_point)
    memcpy(h_out_point, res.eval_point.data(), 16 * res.eval_point.size());
  return clear_error();
}

}  // extern "C"
