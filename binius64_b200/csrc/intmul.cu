// Integer multiplication reduction (IntMulProver::prove, prover/prover/src/protocols/intmul/
// prove.rs:93-194) on the device.
//
// Witness (witness.rs:47-270): GKR product trees over the 64 bit positions of each exponent
// column.  A leaf holds, per statement x, either 1 or base^(2^i) as bit i of the exponent is clear
// or set; a node is the per-vertex product of its two children, so a root holds base^exponent.
// a and c_lo use the multiplicative generator g, c_hi uses g^(2^64), and b uses the per-vertex
// variable base g^a (its leaves square the base per bit).  The a, c_lo and c_hi trees are stored
// interleaved by layer: layer k is one contiguous set of 3 * 2^k multilinears [a | c_lo | c_hi],
// so node q of a layer is the product of nodes 2q and 2q + 1 of the next one for all three trees,
// and every GKR layer of phases 4 and 5 is a contiguous run of pairs.  Multilinears of one set
// share a stride of 2^n_vars elements and shrink in place as their top variable is folded.
//
// Each phase is a batched sumcheck (batch.rs:41-135) over the MLE-check provers of the reference:
// bivariate products on multiple pairs (bivariate_product_multi_mle.rs), the selector prover
// (selector_mle.rs) and rerandomisation (rerand_mle.rs), with the Gruen eq factor
// (gruen32.rs, mle_to_sumcheck.rs).  Kernels produce the per-claim round sums (y_1, y_inf) and
// fold by the previous challenge; each round's degree-2/3 coefficient algebra over all claims and
// the Fiat-Shamir step run in intmul_round_finish_kernel on the device transcript, so a batched
// sumcheck of n rounds is one chain of launches with one read-back at its end.  The host sets each
// sumcheck up (the eq points' alphas with one batched inversion, the powers of beta) and writes the
// final evaluations.
#include <string.h>

#include <algorithm>
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

constexpr int kT = 256;
// Round kernels on multilinears of at most this many elements run few threads once per launch,
// so they take the compact out-of-line multiply (their code is fetched cold).
constexpr uint64_t kSmallRound = 1ull << 12;
// (pair, position) items of the layer rounds that run in intmul_layer_tail_kernel: a quarter of
// the other sumchecks' tail length (a layer item folds two multilinears at two positions).
inline uint64_t tail_items() { return tail_max_len() >> 2; }

struct Pow64 {
  uint4 p[64];
};

unsigned blocks_for(uint64_t n, unsigned cap = 148 * 4) {
  uint64_t g = (n + kT - 1) / kT;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, cap));
}

// ---------------------------------------------------------------- witness kernels

// out[(i) * stride + x] = bit_i(e[x]) ? pw[i] : 1 for i < 64.
__global__ void const_leaves_kernel(const uint64_t* __restrict__ e, uint64_t n, Pow64 pw,
                                    uint4* __restrict__ out, uint64_t stride) {
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < n;
       x += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t w = e[x];
#pragma unroll 8
    for (int i = 0; i < 64; i++) out[i * stride + x] = ((w >> i) & 1) ? pw.p[i] : gf_one();
  }
}

// Variable base: out[i * stride + x] = bit_i(e[x]) ? base[x]^(2^i) : 1.
__global__ void var_leaves_kernel(const uint64_t* __restrict__ e, uint64_t n,
                                  const uint4* __restrict__ base, uint4* __restrict__ out,
                                  uint64_t stride) {
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < n;
       x += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t w = e[x];
    uint4 v = base[x];
    for (int i = 0; i < 64; i++) {
      out[i * stride + x] = ((w >> i) & 1) ? v : gf_one();
      v = gf_mul(v, v);
    }
  }
}

// parent[q] = child[2q] * child[2q + 1] for q < count.
__global__ void tree_layer_kernel(const uint4* __restrict__ child, uint4* __restrict__ parent,
                                  uint32_t count, uint64_t n, uint64_t stride) {
  const uint64_t total = (uint64_t)count * n;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t q = t / n, x = t - q * n;
    parent[q * stride + x] = gf_mul(child[2 * q * stride + x], child[(2 * q + 1) * stride + x]);
  }
}

// out[k * stride + x] = bit (k + first) of e[x] as 0 / 1 for k < count.
__global__ void bit_columns_kernel(const uint64_t* __restrict__ e, uint64_t n, uint32_t first,
                                   uint32_t count, uint4* __restrict__ out, uint64_t stride) {
  const uint64_t total = (uint64_t)count * n;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = t / n, x = t - k * n;
    out[k * stride + x] = make_uint4((uint32_t)((e[x] >> (k + first)) & 1), 0u, 0u, 0u);
  }
}

// ---------------------------------------------------------------- sumcheck kernels

__device__ __forceinline__ uint4 fold1(uint4 lo, uint4 hi, uint4 r) {
  return gf_add(lo, gf_mul(r, gf_add(hi, lo)));
}

// One round of the bivariate products on pair p of `set` (multilinears 2p and 2p + 1, current
// length L): out[8p..] += (sum eq[i] a1 b1, sum eq[i] (a0 + a1)(b0 + b1)) over i < L/2.  With
// `fold`, both multilinears first shrink from 2L to L by r in place (fold_highest_var_inplace);
// thread i owns positions i and i + L/2, so the fold and the round need one pass.  Grid: (chunks,
// pairs).  The fold's r is *r_ptr (a challenge in HBM); r_ptr == nullptr means no fold.  Rounds of
// at most kSmallRound elements run in biv_round_lanes_kernel.
__global__ void __launch_bounds__(kT)
    biv_round_kernel(uint4* __restrict__ set, uint64_t L, uint64_t stride,
                     const uint4* __restrict__ eq, const uint4* __restrict__ r_ptr,
                     uint32_t* __restrict__ out) {
  pdl_wait();
  pdl_trigger();
  const bool fold = r_ptr != nullptr;
  const uint4 r = fold ? *r_ptr : gf_zero();
  const uint32_t p = blockIdx.y;
  uint4* a = set + 2 * p * stride;
  uint4* b = a + stride;
  const uint64_t h = L >> 1;
  u256 s1 = {0, 0, 0, 0}, sinf = {0, 0, 0, 0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < h;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint4 a0, a1, b0, b1;
    if (fold) {
      a0 = gf_add(a[i], gf_mul(r, gf_add(a[L + i], a[i])));
      a1 = gf_add(a[h + i], gf_mul(r, gf_add(a[L + h + i], a[h + i])));
      b0 = gf_add(b[i], gf_mul(r, gf_add(b[L + i], b[i])));
      b1 = gf_add(b[h + i], gf_mul(r, gf_add(b[L + h + i], b[h + i])));
      a[i] = a0;
      a[h + i] = a1;
      b[i] = b0;
      b[h + i] = b1;
    } else {
      a0 = a[i];
      a1 = a[h + i];
      b0 = b[i];
      b1 = b[h + i];
    }
    const uint4 e = eq[i];
    xor_into(s1, clmul128(e, gf_mul(a1, b1)));
    xor_into(sinf, clmul128(e, gf_mul(gf_add(a0, a1), gf_add(b0, b1))));
  }
  uint4 v[2] = {reduce256(s1), reduce256(sinf)};
  block_xor_reduce<2>(v, out + 8 * p);
}

// The small rounds of biv_round_kernel (L <= kSmallRound) on four lanes per position i: lane k
// folds a or b (k < 2) at i or L/2 + i (k odd), the folded values meet by shuffles and lanes 0
// and 1 form the two eq-weighted products: three dependent multiplies per lane instead of eight
// on one thread.  Grid: (chunks of four-lane groups, pairs).
__global__ void __launch_bounds__(kT)
    biv_round_lanes_kernel(uint4* __restrict__ set, uint64_t L, uint64_t stride,
                           const uint4* __restrict__ eq, const uint4* __restrict__ r_ptr,
                           uint32_t* __restrict__ out) {
  pdl_wait();
  pdl_trigger();
  const bool fold = r_ptr != nullptr;
  const uint4 r = fold ? *r_ptr : gf_zero();
  const uint32_t p = blockIdx.y, k = threadIdx.x & 3;
  uint4* a = set + 2 * p * stride;
  uint4* b = a + stride;
  const uint64_t h = L >> 1;
  uint4 v[2] = {gf_zero(), gf_zero()};
  const uint64_t all = (uint64_t)gridDim.x * blockDim.x;
  // warp-uniform sweeps: every lane of a warp runs the same iterations (shuffles below)
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u); base < 4 * h;
       base += all) {
    const uint64_t i = (base + (threadIdx.x & 31)) >> 2;
    const bool live = i < h;
    uint4 f = gf_zero();
    if (live) {
      uint4* col = k < 2 ? a : b;
      const uint64_t pos = i + ((k & 1) ? h : 0);
      f = col[pos];
      if (fold) {
        f = gf_add(f, gf_mul_nl(r, gf_add(col[L + pos], f)));
        col[pos] = f;
      }
    }
    const uint4 a0 = shfl_gf(f, 0, 4), a1 = shfl_gf(f, 1, 4), b0 = shfl_gf(f, 2, 4),
                b1 = shfl_gf(f, 3, 4);
    if (live && k == 0) gf_add_into(v[0], gf_mul_nl(eq[i], gf_mul_nl(a1, b1)));
    if (live && k == 1)
      gf_add_into(v[1], gf_mul_nl(eq[i], gf_mul_nl(gf_add(a0, a1), gf_add(b0, b1))));
  }
  block_xor_reduce<2>(v, out + 8 * p);
}

// Column k of `set` (current length L): out[4k..] += sum eq[i] col_k[L/2 + i], with the same
// optional fused fold.  Grid: (chunks, columns).
template <bool SMALL>
__global__ void __launch_bounds__(kT)
    lin_round_kernel(uint4* __restrict__ set, uint64_t L, uint64_t stride,
                     const uint4* __restrict__ eq, const uint4* __restrict__ r_ptr,
                     uint32_t* __restrict__ out) {
  pdl_wait();
  pdl_trigger();
  const bool fold = r_ptr != nullptr;
  const uint4 r = fold ? *r_ptr : gf_zero();
  const uint32_t k = blockIdx.y;
  uint4* c = set + k * stride;
  const uint64_t h = L >> 1;
  u256 s1 = {0, 0, 0, 0};
  uint4 s1r = gf_zero();
  auto mul = [](uint4 x, uint4 y) { return SMALL ? gf_mul_nl(x, y) : gf_mul(x, y); };
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < h;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint4 c1;
    if (fold) {
      c[i] = gf_add(c[i], mul(r, gf_add(c[L + i], c[i])));
      c1 = gf_add(c[h + i], mul(r, gf_add(c[L + h + i], c[h + i])));
      c[h + i] = c1;
    } else {
      c1 = c[h + i];
    }
    if constexpr (SMALL)
      gf_add_into(s1r, gf_mul_nl(eq[i], c1));
    else
      xor_into(s1, clmul128(eq[i], c1));
  }
  uint4 v[1] = {SMALL ? s1r : reduce256(s1)};
  block_xor_reduce<1>(v, out + 4 * k);
}

// Selector claim k with its own eq_k: out[8k..] += (sum eq_k[i] (s1 (sel1 + 1) + 1),
// sum eq_k[i] (s0 + s1)(sel0 + sel1)); `sel` (shared by all claims) is folded beforehand, the
// column s_k is folded here when `fold` is set.  Grid: (chunks, claims).
template <bool SMALL>
__global__ void __launch_bounds__(kT)
    selector_round_kernel(const uint4* __restrict__ sel, uint4* __restrict__ cols, uint64_t L,
                          uint64_t stride, const uint4* __restrict__ eqs, uint64_t eq_stride,
                          const uint4* __restrict__ r_ptr, uint32_t* __restrict__ out) {
  pdl_wait();
  pdl_trigger();
  const bool fold = r_ptr != nullptr;
  const uint4 r = fold ? *r_ptr : gf_zero();
  const uint32_t k = blockIdx.y;
  uint4* s = cols + k * stride;
  const uint4* eq = eqs + k * eq_stride;
  const uint64_t h = L >> 1;
  u256 s1 = {0, 0, 0, 0}, sinf = {0, 0, 0, 0};
  uint4 s1r = gf_zero(), sinfr = gf_zero();
  auto mul = [](uint4 x, uint4 y) { return SMALL ? gf_mul_nl(x, y) : gf_mul(x, y); };
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < h;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint4 c0, c1;
    if (fold) {
      c0 = gf_add(s[i], mul(r, gf_add(s[L + i], s[i])));
      c1 = gf_add(s[h + i], mul(r, gf_add(s[L + h + i], s[h + i])));
      s[i] = c0;
      s[h + i] = c1;
    } else {
      c0 = s[i];
      c1 = s[h + i];
    }
    const uint4 e = eq[i], sel0 = sel[i], sel1 = sel[h + i];
    const uint4 x1 = gf_add(mul(c1, gf_add(sel1, gf_one())), gf_one());
    const uint4 xi = mul(gf_add(c0, c1), gf_add(sel0, sel1));
    if constexpr (SMALL) {
      gf_add_into(s1r, gf_mul_nl(e, x1));
      gf_add_into(sinfr, gf_mul_nl(e, xi));
    } else {
      xor_into(s1, clmul128(e, x1));
      xor_into(sinf, clmul128(e, xi));
    }
  }
  uint4 v[2] = {SMALL ? s1r : reduce256(s1), SMALL ? sinfr : reduce256(sinf)};
  block_xor_reduce<2>(v, out + 8 * k);
}

// In-place top-variable fold of `count` multilinears of length 2 * half.
__global__ void fold_set_kernel(uint4* __restrict__ set, uint32_t count, uint64_t half,
                                uint64_t stride, const uint4* __restrict__ r_ptr) {
  pdl_wait();
  pdl_trigger();
  const uint4 r = *r_ptr;
  const uint64_t total = (uint64_t)count * half;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = t / half, i = t - k * half;
    uint4* m = set + k * stride;
    m[i] = fold1(m[i], m[half + i], r);
  }
}

// The eq tensors of `count` points over their first m' coordinates for every m' <= m (the Gruen
// eq factor of each round, gruen32.rs; in place of eq_ind_truncate_low_inplace per round):
// out[k * stride + (2^m' - 1) + i] = prod_{j < m'} (bit_j(i) ? p_kj : 1 + p_kj).
__global__ void eq_levels_kernel(const uint4* __restrict__ points, uint32_t count, uint32_t m,
                                 uint4* __restrict__ out, uint64_t stride) {
  const uint64_t per = (2ull << m) - 1, total = (uint64_t)count * per;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = t / per, rr = t - k * per;
    const uint32_t lvl = 63 - __clzll(rr + 1);
    const uint64_t i = rr + 1 - (1ull << lvl);
    // four interleaved partial products: the dependent chain is ~lvl / 4 multiplies, not lvl
    auto factor = [&](uint32_t j) {
      const uint4 p = points[k * m + j];
      return ((i >> j) & 1) ? p : gf_add(p, gf_one());
    };
    uint4 a0 = gf_one(), a1 = gf_one(), a2 = gf_one(), a3 = gf_one();
    uint32_t j = 0;
    for (; j + 4 <= lvl; j += 4) {
      a0 = gf_mul(a0, factor(j));
      a1 = gf_mul(a1, factor(j + 1));
      a2 = gf_mul(a2, factor(j + 2));
      a3 = gf_mul(a3, factor(j + 3));
    }
    for (; j < lvl; j++) a0 = gf_mul(a0, factor(j));
    out[k * stride + rr] = gf_mul(gf_mul(a0, a1), gf_mul(a2, a3));
  }
}

// out += sum eq[x] a[x] (b[x] or 1).
__global__ void __launch_bounds__(kT)
    dot_kernel(const uint4* __restrict__ a, const uint4* __restrict__ b,
               const uint4* __restrict__ eq, uint64_t n, uint32_t* __restrict__ out) {
  u256 s = {0, 0, 0, 0};
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < n;
       x += (uint64_t)gridDim.x * blockDim.x) {
    uint4 v = a[x];
    if (b) v = gf_mul(v, b[x]);
    xor_into(s, clmul128(eq[x], v));
  }
  uint4 r[1] = {reduce256(s)};
  block_xor_reduce<1>(r, out);
}

// One claim of a batched MLE-check round: the slots (uint4 index into the round's sums) of its
// y_1 and, for a bivariate product (deg 2), y_inf; deg 1 is a linear claim (RoundEvals1).  group
// selects the eq point (alphas, Gruen prefix) the claim follows.
struct ImClaim {
  uint16_t y1, yinf;
  uint8_t deg, group;
  uint16_t pad;
};
// The eq coordinate a group's MLE-check binds in one round and 1 / (1 + alpha).
struct ImAlpha {
  uint4 alpha, inv_one_plus_alpha;
};
constexpr int kImFinishThreads = 256;
constexpr uint32_t kImMaxClaims = 256;

// The Fiat-Shamir step of one round of a batched MLE-check (BatchSumcheckProver over decorated
// MLE-check provers, batch.rs:41-135 + mle_to_sumcheck.rs + gruen32.rs), on the device.  Claim i:
// prime_i = interpolate_eq(sum_i, y_1, [y_inf], alpha) (RoundEvals2 / RoundEvals1,
// round_evals.rs:23-27, 80-87), all_i = round_coeffs_by_eq(prime_i, alpha) * prefix
// (round_evals.rs:145-156); the round message is sum_i beta^i all_i without its top coefficient
// (msg_coeffs elements).  Claims are spread over the block and block-reduced; warp 0 writes the
// message and samples r; then every claim's sum becomes prime_i(r) and every group's prefix
// takes the factor (1 + r + alpha).
__global__ void __launch_bounds__(kImFinishThreads)
    intmul_round_finish_kernel(TranscriptState* __restrict__ ts, uint8_t* __restrict__ tape,
                               const uint4* __restrict__ slots, const ImClaim* __restrict__ claims,
                               uint32_t n_claims, uint4* __restrict__ sums,
                               uint4* __restrict__ prefix, const ImAlpha* __restrict__ alphas,
                               uint32_t n_groups, const uint4* __restrict__ beta_pow,
                               uint32_t msg_coeffs, uint4* __restrict__ r_out) {
  pdl_wait();
  pdl_trigger();
  __shared__ uint4 s_prime[kImMaxClaims][3];
  __shared__ uint4 s_r;
  uint4 acc[4] = {gf_zero(), gf_zero(), gf_zero(), gf_zero()};
  for (uint32_t i = threadIdx.x; i < n_claims; i += blockDim.x) {
    const ImClaim c = claims[i];
    const ImAlpha a = alphas[c.group];
    const uint4 y1 = slots[c.y1];
    const uint4 y0 = gf_mul_nl(gf_add(sums[i], gf_mul_nl(y1, a.alpha)), a.inv_one_plus_alpha);
    uint4 p0 = y0, p1, p2 = gf_zero();
    if (c.deg == 2) {
      const uint4 yinf = slots[c.yinf];
      p1 = gf_add(gf_add(y1, y0), yinf);
      p2 = yinf;
    } else {
      p1 = gf_add(y1, y0);
    }
    s_prime[i][0] = p0;
    s_prime[i][1] = p1;
    s_prime[i][2] = p2;
    uint4 oma = a.alpha;
    oma.x ^= 1u;
    const uint4 sc = gf_mul_nl(prefix[c.group], beta_pow[i]);
    gf_add_into(acc[0], gf_mul_nl(gf_mul_nl(p0, oma), sc));
    gf_add_into(acc[1], gf_mul_nl(gf_add(gf_mul_nl(p1, oma), p0), sc));
    gf_add_into(acc[2], gf_mul_nl(gf_add(gf_mul_nl(p2, oma), p1), sc));
    gf_add_into(acc[3], gf_mul_nl(p2, sc));
  }
  block_xor_sum<4>(acc);
  if (threadIdx.x < 32) {
    DevTr st;
    st.load(ts);
    st.message_elems(tape, acc, msg_coeffs);
    const uint4 r = st.sample_elem();
    __syncwarp();
    if (threadIdx.x == 0) {
      *r_out = r;
      st.store(ts);
      s_r = r;
    }
  }
  __syncthreads();
  const uint4 r = s_r;
  for (uint32_t i = threadIdx.x; i < n_claims; i += blockDim.x)
    sums[i] = gf_add(s_prime[i][0], gf_mul_nl(r, gf_add(s_prime[i][1], gf_mul_nl(r, s_prime[i][2]))));
  for (uint32_t g = threadIdx.x; g < n_groups; g += blockDim.x) {
    uint4 f = gf_add(r, alphas[g].alpha);
    f.x ^= 1u;
    prefix[g] = gf_mul_nl(prefix[g], f);
  }
}

// The small last rounds of one GKR layer's batched MLE-check (IntMulDevice::layer: `pairs`
// bivariate product claims, one eq point, messages of three coefficients) in one CTA, from round
// t0 on: per round every multilinear of the set folds 2L -> L by the previous challenge (r_first
// for round t0 when t0 > 0), the products are summed with their eq weights, and warp 0 runs the
// batch's Fiat-Shamir step with the transcript in its registers.  The step is the one of
// intmul_round_finish_kernel rewritten for a single group: the message is linear in the round's
// sums, so with Y1 = sum_p beta^p y_1,p and Yinf = sum_p beta^p y_inf,p (one block sum per
// round) and the running G = sum_p beta^p sum_p, T0 = (G + alpha Y1) / (1 + alpha),
// T1 = Y1 + T0 + Yinf, T2 = Yinf, the message is prefix ((1 + alpha) T0, (1 + alpha) T1 + T0,
// (1 + alpha) T2 + T1), and after r the batch keeps G = T0 + r T1 + r^2 T2 and
// prefix (1 + r + alpha).  Thread items are (pair, index) with the index fastest; item i of pair
// p folds positions i and L/2 + i of both multilinears and evaluates that pair of positions.
constexpr int kImTailThreads = 512;
__global__ void __launch_bounds__(kImTailThreads)
    intmul_layer_tail_kernel(TranscriptState* __restrict__ ts, uint8_t* __restrict__ tape,
                             uint4* __restrict__ set, uint32_t pairs, uint64_t stride,
                             uint32_t n, uint32_t t0, const uint4* __restrict__ eq_base,
                             const uint4* __restrict__ sums, const uint4* __restrict__ prefix,
                             const ImAlpha* __restrict__ alphas,
                             const uint4* __restrict__ beta_pow, uint4* __restrict__ chal) {
  pdl_wait();
  pdl_trigger();
  __shared__ uint4 r_sh;
  DevTr st;
  uint4 G = gf_zero(), pf = gf_zero();
  {
    uint4 v[1] = {gf_zero()};
    for (uint32_t p = threadIdx.x; p < pairs; p += blockDim.x)
      gf_add_into(v[0], gf_mul_nl(beta_pow[p], sums[p]));
    block_xor_sum<1>(v);
    if (threadIdx.x < 32) {
      G = v[0];
      pf = prefix[0];
      st.load(ts);
      if (t0 > 0) r_sh = chal[t0 - 1];
    }
    __syncthreads();
  }
  for (uint32_t t = t0; t < n; t++) {
    const bool fold = t > 0;
    const uint4 r = r_sh;
    const uint64_t L = 1ull << (n - t), h = L >> 1;
    const uint4* eq = eq_base + ((1ull << (n - t - 1)) - 1);
    uint4 v[2] = {gf_zero(), gf_zero()};
    for (uint64_t it = threadIdx.x; it < (uint64_t)pairs * h; it += blockDim.x) {
      const uint32_t p = (uint32_t)(it / h);
      const uint64_t i = it - (uint64_t)p * h;
      uint4* a = set + 2 * (uint64_t)p * stride;
      uint4* b = a + stride;
      uint4 a0 = a[i], a1 = a[h + i], b0 = b[i], b1 = b[h + i];
      if (fold) {
        a0 = gf_add(a0, gf_mul_nl(r, gf_add(a[L + i], a0)));
        a1 = gf_add(a1, gf_mul_nl(r, gf_add(a[L + h + i], a1)));
        b0 = gf_add(b0, gf_mul_nl(r, gf_add(b[L + i], b0)));
        b1 = gf_add(b1, gf_mul_nl(r, gf_add(b[L + h + i], b1)));
        a[i] = a0;
        a[h + i] = a1;
        b[i] = b0;
        b[h + i] = b1;
      }
      const uint4 w = gf_mul_nl(eq[i], beta_pow[p]);
      gf_add_into(v[0], gf_mul_nl(w, gf_mul_nl(a1, b1)));
      gf_add_into(v[1], gf_mul_nl(w, gf_mul_nl(gf_add(a0, a1), gf_add(b0, b1))));
    }
    block_xor_sum<2>(v);
    if (threadIdx.x < 32) {
      const ImAlpha al = alphas[t];
      const uint4 y1 = v[0], yinf = v[1];
      const uint4 T0 = gf_mul_warp(gf_add(G, gf_mul_warp(al.alpha, y1)), al.inv_one_plus_alpha);
      const uint4 T1 = gf_add(gf_add(y1, T0), yinf), T2 = yinf;
      uint4 oma = al.alpha;
      oma.x ^= 1u;
      const uint4 m[3] = {gf_mul_warp(pf, gf_mul_warp(oma, T0)),
                          gf_mul_warp(pf, gf_add(gf_mul_warp(oma, T1), T0)),
                          gf_mul_warp(pf, gf_add(gf_mul_warp(oma, T2), T1))};
      st.message_elems(tape, m, 3);
      const uint4 rr = st.sample_elem();
      chal[t] = rr;
      G = gf_add(T0, gf_mul_warp(rr, gf_add(T1, gf_mul_warp(rr, T2))));
      uint4 f = gf_add(rr, al.alpha);
      f.x ^= 1u;
      pf = gf_mul_warp(pf, f);
      r_sh = rr;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) st.store(ts);
}

// The small last rounds of the leaf batch (IntMulDevice phase 5) in one CTA, from round t0 on,
// with intmul_layer_tail_kernel's single-group step per group: claims 0..96 are the bivariate
// leaf pairs and 97 the linear c_lo_0 column, all on eq point 0 (eq_base); claims 98..161 are
// the 64 linear b columns on eq point 1 (eq2_base).  Per round every multilinear folds 2L -> L
// by the previous challenge and the group sums Y1_0, Yinf_0, Y1_1 (beta^claim and eq weighted)
// feed the step; deg-1 claims have no y_inf.  Items are (multilinear group m, index i) with the
// index fastest: m < 97 a leaf pair, m = 97 the c_lo_0 column, m > 97 b column m - 98.
constexpr uint32_t kLeafPairs = 97, kLeafCols = 64;
__global__ void __launch_bounds__(kImTailThreads)
    intmul_leaf_tail_kernel(TranscriptState* __restrict__ ts, uint8_t* __restrict__ tape,
                            uint4* __restrict__ leaves, uint4* __restrict__ lo0,
                            uint4* __restrict__ bcols, uint64_t stride, uint32_t n, uint32_t t0,
                            const uint4* __restrict__ eq_base, const uint4* __restrict__ eq2_base,
                            const uint4* __restrict__ sums, const uint4* __restrict__ prefix,
                            const ImAlpha* __restrict__ alphas,
                            const uint4* __restrict__ beta_pow, uint4* __restrict__ chal) {
  pdl_wait();
  pdl_trigger();
  constexpr uint32_t kClaims0 = kLeafPairs + 1, kClaims = kClaims0 + kLeafCols;
  __shared__ uint4 r_sh;
  DevTr st;
  uint4 G[2] = {gf_zero(), gf_zero()}, pf[2] = {gf_zero(), gf_zero()};
  {
    uint4 v[2] = {gf_zero(), gf_zero()};
    for (uint32_t i = threadIdx.x; i < kClaims; i += blockDim.x)
      gf_add_into(v[i < kClaims0 ? 0 : 1], gf_mul_nl(beta_pow[i], sums[i]));
    block_xor_sum<2>(v);
    if (threadIdx.x < 32) {
      G[0] = v[0];
      G[1] = v[1];
      pf[0] = prefix[0];
      pf[1] = prefix[1];
      st.load(ts);
      if (t0 > 0) r_sh = chal[t0 - 1];
    }
    __syncthreads();
  }
  auto fold2 = [](uint4* col, uint64_t i, uint64_t L, uint64_t h, uint4 r, bool fold,
                  uint4& x0, uint4& x1) {
    x0 = col[i];
    x1 = col[h + i];
    if (fold) {
      x0 = gf_add(x0, gf_mul_nl(r, gf_add(col[L + i], x0)));
      x1 = gf_add(x1, gf_mul_nl(r, gf_add(col[L + h + i], x1)));
      col[i] = x0;
      col[h + i] = x1;
    }
  };
  for (uint32_t t = t0; t < n; t++) {
    const bool fold = t > 0;
    const uint4 r = r_sh;
    const uint64_t L = 1ull << (n - t), h = L >> 1;
    const uint64_t lvl = (1ull << (n - t - 1)) - 1;
    uint4 v[3] = {gf_zero(), gf_zero(), gf_zero()};  // Y1_0, Yinf_0, Y1_1
    for (uint64_t it = threadIdx.x; it < (uint64_t)kClaims * h; it += blockDim.x) {
      const uint32_t m = (uint32_t)(it / h);
      const uint64_t i = it - (uint64_t)m * h;
      if (m < kLeafPairs) {
        uint4 a0, a1, b0, b1;
        fold2(leaves + 2 * (uint64_t)m * stride, i, L, h, r, fold, a0, a1);
        fold2(leaves + (2 * (uint64_t)m + 1) * stride, i, L, h, r, fold, b0, b1);
        const uint4 w = gf_mul_nl(eq_base[lvl + i], beta_pow[m]);
        gf_add_into(v[0], gf_mul_nl(w, gf_mul_nl(a1, b1)));
        gf_add_into(v[1], gf_mul_nl(w, gf_mul_nl(gf_add(a0, a1), gf_add(b0, b1))));
      } else {
        const bool g0 = m == kLeafPairs;
        uint4* col = g0 ? lo0 : bcols + (uint64_t)(m - kClaims0) * stride;
        uint4 c0, c1;
        fold2(col, i, L, h, r, fold, c0, c1);
        const uint4 w = gf_mul_nl(g0 ? eq_base[lvl + i] : eq2_base[lvl + i], beta_pow[m]);
        gf_add_into(v[g0 ? 0 : 2], gf_mul_nl(w, c1));
      }
    }
    block_xor_sum<3>(v);
    if (threadIdx.x < 32) {
      uint4 m3[3] = {gf_zero(), gf_zero(), gf_zero()};
      uint4 T[2][3];
      for (int g = 0; g < 2; g++) {
        const ImAlpha al = alphas[2 * t + g];
        const uint4 y1 = g == 0 ? v[0] : v[2], yinf = g == 0 ? v[1] : gf_zero();
        T[g][0] = gf_mul_warp(gf_add(G[g], gf_mul_warp(al.alpha, y1)), al.inv_one_plus_alpha);
        T[g][1] = gf_add(gf_add(y1, T[g][0]), yinf);
        T[g][2] = yinf;
        uint4 oma = al.alpha;
        oma.x ^= 1u;
        gf_add_into(m3[0], gf_mul_warp(pf[g], gf_mul_warp(oma, T[g][0])));
        gf_add_into(m3[1], gf_mul_warp(pf[g], gf_add(gf_mul_warp(oma, T[g][1]), T[g][0])));
        gf_add_into(m3[2], gf_mul_warp(pf[g], gf_add(gf_mul_warp(oma, T[g][2]), T[g][1])));
      }
      st.message_elems(tape, m3, 3);
      const uint4 rr = st.sample_elem();
      chal[t] = rr;
      for (int g = 0; g < 2; g++) {
        G[g] = gf_add(T[g][0], gf_mul_warp(rr, gf_add(T[g][1], gf_mul_warp(rr, T[g][2]))));
        uint4 f = gf_add(rr, alphas[2 * t + g].alpha);
        f.x ^= 1u;
        pf[g] = gf_mul_warp(pf[g], f);
      }
      r_sh = rr;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) st.store(ts);
}

// ---------------------------------------------------------------- host side

uint4 u4(hu128 v) {
  uint4 r;
  memcpy(&r, &v, 16);
  return r;
}
hu128 h128(const void* p) {
  hu128 v;
  memcpy(&v, p, 16);
  return v;
}
hu128 sq_n(hu128 x, int n) {
  for (int i = 0; i < n; i++) x = host_gf_mul(x, x);
  return x;
}
// 1 / (g^(2^i) - 1) for i < 128 (normalize_a_c_exponent_evals, common.rs:107-138), computed once.
const hu128* conj_inv_table() {
  static const std::vector<hu128> table = [] {
    std::vector<hu128> t(128);
    hu128 c = ((hu128)0x494ef99794d5244fULL << 64) | (hu128)0x9152df59d87a9186ULL;
    for (int i = 0; i < 128; i++, c = host_gf_mul(c, c)) t[i] = host_gf_inv(c ^ 1);
    return t;
  }();
  return table.data();
}

// normalize_a_c_exponent_evals: the 192 leaf evaluations (a, c_lo, c_hi) -> bit evaluations.
void normalize_leaves(const std::vector<hu128>& biv, IntMulResult& res) {
  const hu128* inv = conj_inv_table();
  res.a_evals.clear();
  res.c_lo_evals.clear();
  res.c_hi_evals.clear();
  for (int i = 0; i < 64; i++) {
    res.a_evals.push_back(host_gf_mul(biv[i] ^ 1, inv[i]));
    res.c_lo_evals.push_back(host_gf_mul(biv[64 + i] ^ 1, inv[i]));
    res.c_hi_evals.push_back(host_gf_mul(biv[128 + i] ^ 1, inv[64 + i]));
  }
}

// In place: v[i] <- 1 / v[i] for nonzero entries (zero stays zero, as invert_or_zero), with one
// inversion for the whole vector (Montgomery's trick).
void batch_inv(std::vector<hu128>& v) {
  std::vector<hu128> pre(v.size());
  hu128 acc = 1;
  for (size_t i = 0; i < v.size(); i++) {
    pre[i] = acc;
    if (v[i]) acc = host_gf_mul(acc, v[i]);
  }
  hu128 inv = host_gf_inv(acc);
  for (size_t i = v.size(); i-- > 0;) {
    if (!v[i]) continue;
    const hu128 x = v[i];
    v[i] = host_gf_mul(inv, pre[i]);
    inv = host_gf_mul(inv, x);
  }
}

hu128 sample(Transcript& t) {
  uint8_t b[16];
  t.sample_elem(b);
  return h128(b);
}
void write_elems(Transcript& t, const std::vector<hu128>& v) {
  if (!v.empty()) t.message(v.data(), 16 * v.size());
}
class IntMulDevice {
 public:
  IntMulDevice(cudaStream_t s, Transcript& t) : s_(s), t_(t) {}
  ~IntMulDevice() {
    for (void* p : ptrs_) dev_free(p, s_);
  }

  int run(const uint64_t* d_a, const uint64_t* d_b, const uint64_t* d_lo, const uint64_t* d_hi,
          uint32_t n_vars, IntMulResult& res);

 private:
  // One statement (n_vars = 0): every sumcheck has zero rounds, so the transcript carries the
  // tree values themselves; they are read back from the device in one copy.
  int run_single(uint4* acl, uint4* btree, uint4* bcols, uint4* lo0, const uint64_t* d_a,
                 const uint64_t* d_b, const uint64_t* d_lo, IntMulResult& res);

 private:
  template <class T>
  int alloc(T** p, size_t elems16) {
    cudaError_t e = dev_alloc(reinterpret_cast<void**>(p), 16 * std::max<size_t>(elems16, 1), s_);
    if (e != cudaSuccess) return cuda_error(e, "intmul buffers");
    ptrs_.push_back(*p);
    return BINIUS_OK;
  }
  int check(const char* what, uint64_t launches = 1) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, what);
    count_launch(launches);
    return BINIUS_OK;
  }
  int sync_read(void* dst, const void* src, size_t bytes) { return read_sync(dst, src, bytes, s_); }
  // values [0] of `count` multilinears with stride `stride`
  int read_first(const uint4* set, uint32_t count, uint64_t stride, std::vector<hu128>& out) {
    out.resize(count);
    StagedReads rd(s_);
    if (int rc = rd.add2d(out.data(), 16, set, 16 * stride, 16, count)) return rc;
    return rd.wait();
  }
  int eq_single(const std::vector<hu128>& point, uint32_t m, uint4* out) {
    std::vector<uint4> p(m);
    for (uint32_t i = 0; i < m; i++) p[i] = u4(point[i]);
    return eq_tensor(p.data(), m, out, s_);
  }
  int fold(uint4* set, uint32_t count, uint64_t half, const uint4* r_ptr) {
    if (half == 0) return BINIUS_OK;
    BGPU_CUDA(launch_pdl(fold_set_kernel, blocks_for((uint64_t)count * half), kT, 0, s_, set, count,
                         half, N_, r_ptr));
    return check("fold_set_kernel");
  }
  // Fused round launches on multilinears of current length L (fold from 2L first by *r_ptr when
  // r_ptr is set).
  int biv_round(uint4* set, uint32_t pairs, uint64_t L, const uint4* eq, const uint4* r_ptr,
                uint32_t* out) {
    dim3 grid(blocks_for(L / 2, 148 * 2), pairs);
    if (L <= kSmallRound)
      BGPU_CUDA(launch_pdl(biv_round_lanes_kernel, dim3(blocks_for(2 * L, 148 * 2), pairs), kT, 0,
                           s_, set, L, N_, eq, r_ptr, out));
    else
      BGPU_CUDA(launch_pdl(biv_round_kernel, grid, kT, 0, s_, set, L, N_, eq, r_ptr, out));
    return check("biv_round_kernel");
  }
  int lin_round(uint4* set, uint32_t cols, uint64_t L, const uint4* eq, const uint4* r_ptr,
                uint32_t* out) {
    dim3 grid(blocks_for(L / 2, 148 * 2), cols);
    if (L <= kSmallRound)
      BGPU_CUDA(launch_pdl(lin_round_kernel<true>, grid, kT, 0, s_, set, L, N_, eq, r_ptr, out));
    else
      BGPU_CUDA(launch_pdl(lin_round_kernel<false>, grid, kT, 0, s_, set, L, N_, eq, r_ptr, out));
    return check("lin_round_kernel");
  }
  // A batched MLE-check whose rounds run on the device transcript: batch_begin uploads the claims,
  // each eq point's per-round alpha and 1/(1 + alpha) (one batched inversion), the powers of
  // beta and the initial sums; each round launches its evaluation kernels into batch_slots(t)
  // (folding by batch_r(t)) and then batch_round; batch_read queues the copy-back of the
  // challenges and the transcript, batch_end hands the transcript back to the host.
  struct DevBatch {
    uint32_t n = 0, n_claims = 0, n_groups = 0, msg = 3, per_round = 0;
    ImClaim* claims = nullptr;
    ImAlpha* alphas = nullptr;
    uint4 *sums = nullptr, *prefix = nullptr, *beta = nullptr, *chal = nullptr, *slots = nullptr;
    DeviceTranscript dt;
  };
  int batch_begin(DevBatch& b, const std::vector<ImClaim>& claims,
                  const std::vector<const std::vector<hu128>*>& points,
                  const std::vector<hu128>& sums, hu128 beta, uint32_t per_round) {
    if (claims.empty() || claims.size() > kImMaxClaims || sums.size() != claims.size())
      return set_error(BINIUS_E_ARG, "intmul batch: 1..256 claims with one sum each");
    b.n = (uint32_t)points[0]->size();
    b.n_claims = (uint32_t)claims.size();
    b.n_groups = (uint32_t)points.size();
    b.per_round = per_round;
    b.msg = 2;
    for (const auto& c : claims) b.msg = c.deg == 2 ? 3 : b.msg;
    const size_t n_cl = (8 * claims.size() + 15) / 16, n_al = 2ull * b.n * b.n_groups;
    const size_t host_elems = n_cl + b.n_claims + b.n_groups + n_al + b.n_claims;
    const size_t total = host_elems + b.n + (size_t)b.n * per_round;
    uint4* base = nullptr;
    if (int rc = alloc(&base, total)) return rc;
    std::vector<uint4> h(host_elems, make_uint4(0, 0, 0, 0));
    memcpy(h.data(), claims.data(), 8 * claims.size());
    uint4* hs = h.data() + n_cl;
    for (uint32_t i = 0; i < b.n_claims; i++) hs[i] = u4(sums[i]);
    uint4* hp = hs + b.n_claims;
    for (uint32_t g = 0; g < b.n_groups; g++) hp[g] = u4(1);
    uint4* ha = hp + b.n_groups;
    std::vector<hu128> inv(b.n * b.n_groups);
    for (uint32_t t = 0; t < b.n; t++)
      for (uint32_t g = 0; g < b.n_groups; g++) {
        if (points[g]->size() != b.n) return set_error(BINIUS_E_ARG, "intmul batch: point lengths");
        inv[t * b.n_groups + g] = 1 ^ (*points[g])[b.n - 1 - t];
      }
    batch_inv(inv);
    for (uint32_t t = 0; t < b.n; t++)
      for (uint32_t g = 0; g < b.n_groups; g++) {
        ha[2 * (t * b.n_groups + g)] = u4((*points[g])[b.n - 1 - t]);
        ha[2 * (t * b.n_groups + g) + 1] = u4(inv[t * b.n_groups + g]);
      }
    uint4* hb = ha + n_al;
    hu128 bp = 1;
    for (uint32_t i = 0; i < b.n_claims; i++, bp = host_gf_mul(bp, beta)) hb[i] = u4(bp);
    BGPU_CUDA(cudaMemcpyAsync(base, h.data(), 16 * host_elems, cudaMemcpyHostToDevice, s_));
    b.claims = reinterpret_cast<ImClaim*>(base);
    b.sums = base + n_cl;
    b.prefix = b.sums + b.n_claims;
    b.alphas = reinterpret_cast<ImAlpha*>(b.prefix + b.n_groups);
    b.beta = b.prefix + b.n_groups + n_al;
    b.chal = base + host_elems;
    b.slots = b.chal + b.n;
    BGPU_CUDA(cudaMemsetAsync(b.slots, 0, 16ull * b.n * per_round, s_));
    return b.dt.begin(t_, s_);
  }
  static uint32_t* batch_slots(DevBatch& b, uint32_t t) {
    return reinterpret_cast<uint32_t*>(b.slots + (size_t)t * b.per_round);
  }
  static const uint4* batch_r(const DevBatch& b, uint32_t t) {
    return t ? b.chal + t - 1 : nullptr;
  }
  int batch_round(DevBatch& b, uint32_t t) {
    BGPU_CUDA(launch_pdl(intmul_round_finish_kernel, 1, kImFinishThreads, 0, s_, b.dt.state(),
                         b.dt.tape(), (const uint4*)(b.slots + (size_t)t * b.per_round),
                         (const ImClaim*)b.claims, b.n_claims, b.sums, b.prefix,
                         (const ImAlpha*)(b.alphas + (size_t)t * b.n_groups), b.n_groups,
                         (const uint4*)b.beta, b.msg, b.chal + t));
    return check("intmul_round_finish_kernel");
  }
  int batch_read(DevBatch& b, StagedReads& rd, std::vector<hu128>& ch) {
    ch.resize(b.n);
    if (int rc = b.dt.read(rd, 16 * b.msg * b.n)) return rc;
    return rd.add(ch.data(), b.chal, 16ull * b.n);
  }
  int batch_end(DevBatch& b) { return b.dt.finish(t_); }
  // eq levels of the given points over their first m' <= m coordinates (stride N_ per point).
  int eq_levels(const std::vector<const std::vector<hu128>*>& points, uint32_t m, uint4* out) {
    const uint32_t count = (uint32_t)points.size();
    uint4* d_pts = nullptr;
    if (m > 0) {
      std::vector<uint4> h;
      for (auto* pt : points)
        for (uint32_t j = 0; j < m; j++) h.push_back(u4((*pt)[j]));
      if (int rc = alloc(&d_pts, h.size())) return rc;
      BGPU_CUDA(cudaMemcpyAsync(d_pts, h.data(), 16 * h.size(), cudaMemcpyHostToDevice, s_));
    }
    eq_levels_kernel<<<blocks_for((uint64_t)count << (m + 1)), kT, 0, s_>>>(d_pts, count, m, out, N_);
    return check("eq_levels_kernel");
  }
  static const uint4* level(const uint4* eqs, uint32_t lvl) { return eqs + ((1ull << lvl) - 1); }
  // queue the read of entries 0 and 1 of `count` multilinears (the last round's pre-fold pairs)
  int copy_pairs(StagedReads& rd, const uint4* set, uint32_t count, hu128* dst) {
    return rd.add2d(dst, 32, set, 16 * N_, 32, count);
  }
  static std::vector<hu128> fold_pairs(const std::vector<hu128>& pairs, hu128 r) {
    std::vector<hu128> out(pairs.size() / 2);
    for (size_t m = 0; m < out.size(); m++)
      out[m] = pairs[2 * m] ^ host_gf_mul(r, pairs[2 * m + 1] ^ pairs[2 * m]);
    return out;
  }
  // One GKR layer: decorated BivariateProductMultiMlecheckProver over `pairs` pairs of `set`,
  // batched alone and its evaluations written (prove.rs:207-243, 297-330).
  int layer(uint4* set, uint32_t pairs, std::vector<hu128>& point, std::vector<hu128>& claims);

  cudaStream_t s_;
  Transcript& t_;
  std::vector<void*> ptrs_;
  uint64_t N_ = 1;
  uint32_t n_ = 0;
  uint4* eq_ = nullptr;    // shared eq scratch (N_ elements)
  uint4* eq2_ = nullptr;   // second shared eq (phase 5)
  uint32_t* acc_ = nullptr;
};

int IntMulDevice::layer(uint4* set, uint32_t pairs, std::vector<hu128>& point,
                        std::vector<hu128>& claims) {
  const uint32_t n = (uint32_t)point.size();
  const hu128 beta = sample(t_);
  std::vector<hu128> evals;
  if (n == 0) {
    if (int rc = read_first(set, 2 * pairs, N_, evals)) return rc;
  } else {
    if (int rc = eq_levels({&point}, n - 1, eq_)) return rc;
    std::vector<ImClaim> cl(pairs);
    for (uint32_t p = 0; p < pairs; p++) cl[p] = ImClaim{(uint16_t)(2 * p), (uint16_t)(2 * p + 1), 2, 0, 0};
    DevBatch b;
    if (int rc = batch_begin(b, cl, {&point}, claims, beta, 2 * pairs)) return rc;
    // rounds of at most tail_items() (pair, position) items run in one intmul_layer_tail_kernel
    uint32_t t0 = 0;
    while (t0 < n && ((uint64_t)pairs << (n - t0 - 1)) > tail_items()) t0++;
    for (uint32_t t = 0; t < t0; t++) {
      if (int rc = biv_round(set, pairs, 1ull << (n - t), level(eq_, n - t - 1), batch_r(b, t),
                             batch_slots(b, t)))
        return rc;
      if (int rc = batch_round(b, t)) return rc;
    }
    if (t0 < n) {
      BGPU_CUDA(launch_pdl(intmul_layer_tail_kernel, 1, kImTailThreads, 0, s_, b.dt.state(),
                           b.dt.tape(), set, pairs, N_, n, t0, (const uint4*)eq_,
                           (const uint4*)b.sums, (const uint4*)b.prefix,
                           (const ImAlpha*)b.alphas, (const uint4*)b.beta, b.chal));
      if (int rc = check("intmul_layer_tail_kernel")) return rc;
    }
    std::vector<hu128> ch, last(4 * pairs);
    StagedReads rd(s_);
    if (int rc = batch_read(b, rd, ch)) return rc;
    if (int rc = copy_pairs(rd, set, 2 * pairs, last.data())) return rc;
    if (int rc = rd.wait()) return rc;
    if (int rc = batch_end(b)) return rc;
    evals = fold_pairs(last, ch[n - 1]);
    point.assign(ch.rbegin(), ch.rend());
  }
  write_elems(t_, evals);
  if (n == 0) point.clear();
  claims = evals;
  return BINIUS_OK;
}

// The transcript of a one-statement IntMul (n_vars = 0: every sumcheck has zero rounds, so the
// messages are the tree values themselves) from the host copies of its trees: hacl the a / c_lo /
// c_hi tree (layer k at 3 (2^k - 1), 3 * 2^k values) with a_0 and b_0 after layer 6, hb the b
// tree (layer k at 2^k - 1), hcols the 64 bit columns of b, c_root = c_lo root * c_hi root, lo_bit
// bit 0 of c_lo (prove.rs:91-194 with the phase structure of run).
void emit_single(Transcript& t_, const std::vector<hu128>& hacl, const std::vector<hu128>& hb,
                 const std::vector<hu128>& hcols, hu128 c_root, hu128 lo_bit, IntMulResult& res) {
  auto acl_layer = [&](int k) { return hacl.begin() + 3 * ((1 << k) - 1); };
  auto b_layer = [&](int k) { return hb.begin() + ((1 << k) - 1); };
  write_elems(t_, {hb[0], c_root});
  for (int d = 0; d < 6; d++) {  // phase 1
    sample(t_);
    write_elems(t_, std::vector<hu128>(b_layer(d + 1), b_layer(d + 1) + (2 << d)));
  }
  sample(t_);  // phase 3
  std::vector<hu128> sel = hcols;
  sel.push_back(hacl[0]);
  write_elems(t_, sel);
  write_elems(t_, {hacl[1], hacl[2]});
  for (int d = 0; d < 5; d++) {  // phase 4
    sample(t_);
    write_elems(t_, std::vector<hu128>(acl_layer(d + 1), acl_layer(d + 1) + (6 << d)));
  }
  write_elems(t_, {lo_bit});  // phase 5
  sample(t_);
  std::vector<hu128> biv(acl_layer(6), acl_layer(6) + 194);
  write_elems(t_, biv);
  write_elems(t_, {lo_bit});
  write_elems(t_, hcols);
  res = IntMulResult();
  normalize_leaves(biv, res);
  res.b_evals = hcols;
}

int IntMulDevice::run_single(uint4* acl, uint4* btree, uint4* bcols, uint4* lo0,
                             const uint64_t* d_a, const uint64_t* d_b, const uint64_t* d_lo,
                             IntMulResult& res) {
  constexpr int kAcl = 3 * 127 + 2, kB = 127;
  bit_columns_kernel<<<1, kT, 0, s_>>>(d_b, 1, 0, 64, bcols, 1);
  bit_columns_kernel<<<1, kT, 0, s_>>>(d_a, 1, 0, 1, acl + 3 * 127, 1);
  bit_columns_kernel<<<1, kT, 0, s_>>>(d_b, 1, 0, 1, acl + 3 * 127 + 1, 1);
  bit_columns_kernel<<<1, kT, 0, s_>>>(d_lo, 1, 0, 1, lo0, 1);
  if (int rc = check("bit_columns_kernel", 4)) return rc;
  // c_root = c_lo_root * c_hi_root (acl nodes 1 and 2), through the dot kernel with eq = [1]
  if (int rc = eq_single({}, 0, eq_)) return rc;
  BGPU_CUDA(cudaMemsetAsync(acc_, 0, 16, s_));
  dot_kernel<<<1, kT, 0, s_>>>(acl + 1, acl + 2, eq_, 1, acc_);
  if (int rc = check("dot_kernel")) return rc;
  std::vector<hu128> hacl(kAcl), hb(kB), hcols(64);
  hu128 c_root = 0, lo_bit = 0;
  StagedReads rd(s_);
  if (int rc = rd.add(hacl.data(), acl, 16 * kAcl)) return rc;
  if (int rc = rd.add(hb.data(), btree, 16 * kB)) return rc;
  if (int rc = rd.add(hcols.data(), bcols, 16 * 64)) return rc;
  if (int rc = rd.add(&c_root, acc_, 16)) return rc;
  if (int rc = rd.add(&lo_bit, lo0, 16)) return rc;
  if (int rc = rd.wait()) return rc;
  emit_single(t_, hacl, hb, hcols, c_root, lo_bit, res);
  return BINIUS_OK;
}

int IntMulDevice::run(const uint64_t* d_a, const uint64_t* d_b, const uint64_t* d_lo,
                      const uint64_t* d_hi, uint32_t n_vars, IntMulResult& res) {
  n_ = n_vars;
  N_ = 1ull << n_vars;
  const uint64_t N = N_;
  // a / c_lo / c_hi interleaved tree: layer k at 3 (2^k - 1) N, 3 * 2^k multilinears; two more
  // slots after layer 6 hold a_0 and b_0 for phase 5.
  uint4 *acl, *btree, *bcols, *sel_eqs, *lo0;
  uint32_t* acc;
  if (int rc = alloc(&acl, (3 * 127 + 2) * N)) return rc;
  if (int rc = alloc(&btree, 127 * N)) return rc;
  if (int rc = alloc(&bcols, 64 * N)) return rc;
  if (int rc = alloc(&sel_eqs, 64 * N)) return rc;
  if (int rc = alloc(&lo0, N)) return rc;
  if (int rc = alloc(&eq_, N)) return rc;
  if (int rc = alloc(&eq2_, N)) return rc;
  if (int rc = alloc(&acc, 2 * 97 + 1 + 64)) return rc;
  acc_ = acc;
  auto acl_layer = [&](int k) { return acl + 3 * ((1ull << k) - 1) * N; };
  auto b_layer = [&](int k) { return btree + ((1ull << k) - 1) * N; };

  // ---- witness trees
  const hu128 g = ((hu128)0x494ef99794d5244fULL << 64) | (hu128)0x9152df59d87a9186ULL;
  const hu128 g_hi = sq_n(g, 64);
  const uint64_t* exps[3] = {d_a, d_lo, d_hi};
  const hu128 bases[3] = {g, g, g_hi};
  for (int t = 0; t < 3; t++) {
    Pow64 pw;
    hu128 b = bases[t];
    for (int i = 0; i < 64; i++, b = host_gf_mul(b, b)) pw.p[i] = u4(b);
    const_leaves_kernel<<<blocks_for(N), kT, 0, s_>>>(exps[t], N, pw, acl_layer(6) + 64 * t * N, N);
    if (int rc = check("const_leaves_kernel")) return rc;
  }
  for (int k = 5; k >= 0; k--) {
    const uint32_t count = 3u << k;
    tree_layer_kernel<<<blocks_for(count * N), kT, 0, s_>>>(acl_layer(k + 1), acl_layer(k), count, N, N);
    if (int rc = check("tree_layer_kernel")) return rc;
  }
  var_leaves_kernel<<<blocks_for(N), kT, 0, s_>>>(d_b, N, acl_layer(0), b_layer(6), N);
  if (int rc = check("var_leaves_kernel")) return rc;
  for (int k = 5; k >= 0; k--) {
    tree_layer_kernel<<<blocks_for((1u << k) * N), kT, 0, s_>>>(b_layer(k + 1), b_layer(k), 1u << k, N, N);
    if (int rc = check("tree_layer_kernel")) return rc;
  }

  if (n_ == 0) return run_single(acl, btree, bcols, lo0, d_a, d_b, d_lo, res);

  // ---- root evaluations at the initial point
  std::vector<hu128> point0(n_);
  for (auto& v : point0) v = sample(t_);
  if (int rc = eq_single(point0, n_, eq_)) return rc;
  BGPU_CUDA(cudaMemsetAsync(acc, 0, 32, s_));
  dot_kernel<<<blocks_for(N), kT, 0, s_>>>(b_layer(0), nullptr, eq_, N, acc);
  dot_kernel<<<blocks_for(N), kT, 0, s_>>>(acl_layer(0) + N, acl_layer(0) + 2 * N, eq_, N, acc + 4);
  if (int rc = check("dot_kernel", 2)) return rc;
  uint8_t bc[32];
  if (int rc = sync_read(bc, acc, 32)) return rc;
  const hu128 c_eval = h128(bc + 16);
  t_.message(bc, 32);

  // ---- phase 1: the b tree layers
  std::vector<hu128> pt = point0, evals{h128(bc)};
  for (int d = 0; d < 6; d++)
    if (int rc = layer(b_layer(d + 1), 1u << d, pt, evals)) return rc;

  // ---- phase 2: frobenius twist (common.rs:81-105): x -> x^(2^(128 - i)); twist i is the
  // square of twist i + 1, so the 64 twists of a value take 128 squarings in all
  std::vector<std::vector<hu128>> tw_points(64, std::vector<hu128>(n_));
  std::vector<hu128> sel_sums(64);
  {
    std::vector<hu128> cur(pt);
    for (auto& c : cur) c = sq_n(c, 65);  // i = 63: 2^(128 - 63)
    for (int i = 63; i >= 0; i--) {
      for (uint32_t j = 0; j < n_; j++) tw_points[i][j] = cur[j];
      if (i > 0)
        for (auto& c : cur) c = host_gf_mul(c, c);
    }
    for (int i = 0; i < 64; i++) sel_sums[i] = sq_n(evals[i], 128 - i);
  }

  // ---- phase 3: selector prover on (a_root, bits of b) + bivariate c root prover, on the
  // device transcript: claims 0..63 the selector (slots 2k, 2k + 1, eq point twist k), claim 64
  // the c root pair (slots 128, 129, eq point point0)
  std::vector<hu128> p3, b_exp_evals;
  hu128 selector_eval, c_lo_root_eval, c_hi_root_eval;
  {
    bit_columns_kernel<<<blocks_for(64 * N), kT, 0, s_>>>(d_b, N, 0, 64, bcols, N);
    if (int rc = check("bit_columns_kernel")) return rc;
    std::vector<const std::vector<hu128>*> tw_ptrs;
    for (int i = 0; i < 64; i++) tw_ptrs.push_back(&tw_points[i]);
    if (int rc = eq_levels(tw_ptrs, n_ - 1, sel_eqs)) return rc;
    if (int rc = eq_levels({&point0}, n_ - 1, eq_)) return rc;
    uint4* sel = acl_layer(0);
    uint4* croot = acl_layer(0) + N;
    const hu128 beta = sample(t_);
    std::vector<ImClaim> cl;
    for (int k = 0; k < 64; k++)
      cl.push_back(ImClaim{(uint16_t)(2 * k), (uint16_t)(2 * k + 1), 2, (uint8_t)k, 0});
    cl.push_back(ImClaim{128, 129, 2, 64, 0});
    std::vector<const std::vector<hu128>*> pts = tw_ptrs;
    pts.push_back(&point0);
    std::vector<hu128> sums = sel_sums;
    sums.push_back(c_eval);
    DevBatch b;
    if (int rc = batch_begin(b, cl, pts, sums, beta, 130)) return rc;
    for (uint32_t t = 0; t < n_; t++) {
      const uint64_t L = 1ull << (n_ - t);
      uint32_t* out = batch_slots(b, t);
      const uint4* rp = batch_r(b, t);
      if (rp)
        if (int rc = fold(sel, 1, L, rp)) return rc;  // a_root, shared by the 64 claims
      dim3 grid(blocks_for(L / 2, 148 * 2), 64);
      if (L <= kSmallRound)
        BGPU_CUDA(launch_pdl(selector_round_kernel<true>, grid, kT, 0, s_, (const uint4*)sel, bcols,
                             L, N, level(sel_eqs, n_ - t - 1), N, rp, out));
      else
        BGPU_CUDA(launch_pdl(selector_round_kernel<false>, grid, kT, 0, s_, (const uint4*)sel,
                             bcols, L, N, level(sel_eqs, n_ - t - 1), N, rp, out));
      if (int rc = check("selector_round_kernel")) return rc;
      if (int rc = biv_round(croot, 1, L, level(eq_, n_ - t - 1), rp, out + 4 * 128)) return rc;
      if (int rc = batch_round(b, t)) return rc;
    }
    std::vector<hu128> ch, last_cols(128), last_roots(6);
    StagedReads rd(s_);
    if (int rc = batch_read(b, rd, ch)) return rc;
    if (int rc = copy_pairs(rd, bcols, 64, last_cols.data())) return rc;
    if (int rc = copy_pairs(rd, sel, 3, last_roots.data())) return rc;
    if (int rc = rd.wait()) return rc;
    if (int rc = batch_end(b)) return rc;
    const hu128 r = ch[n_ - 1];
    const std::vector<hu128> colv = fold_pairs(last_cols, r), roots = fold_pairs(last_roots, r);
    std::vector<hu128> sel_evals = colv;
    sel_evals.push_back(roots[0]);
    write_elems(t_, sel_evals);
    write_elems(t_, {roots[1], roots[2]});
    p3.assign(ch.rbegin(), ch.rend());
    b_exp_evals = colv;
    selector_eval = roots[0];
    c_lo_root_eval = roots[1];
    c_hi_root_eval = roots[2];
  }

  // ---- phase 4: layers 1..5 of the a / c_lo / c_hi trees
  pt = p3;
  evals = {selector_eval, c_lo_root_eval, c_hi_root_eval};
  for (int d = 0; d < 5; d++)
    if (int rc = layer(acl_layer(d + 1), 3u << d, pt, evals)) return rc;

  // ---- phase 5: the leaf layers with a_0 * b_0 = c_lo_0 and the b rerandomisation
  {
    uint4* leaves = acl_layer(6);
    bit_columns_kernel<<<blocks_for(N), kT, 0, s_>>>(d_a, N, 0, 1, leaves + 192 * N, N);
    bit_columns_kernel<<<blocks_for(N), kT, 0, s_>>>(d_b, N, 0, 1, leaves + 193 * N, N);
    bit_columns_kernel<<<blocks_for(N), kT, 0, s_>>>(d_lo, N, 0, 1, lo0, N);
    bit_columns_kernel<<<blocks_for(64 * N), kT, 0, s_>>>(d_b, N, 0, 64, bcols, N);
    if (int rc = check("bit_columns_kernel", 4)) return rc;
    if (int rc = eq_single(pt, n_, eq_)) return rc;
    BGPU_CUDA(cudaMemsetAsync(acc, 0, 16, s_));
    dot_kernel<<<blocks_for(N), kT, 0, s_>>>(lo0, nullptr, eq_, N, acc);
    if (int rc = check("dot_kernel")) return rc;
    uint8_t cb[16];
    if (int rc = sync_read(cb, acc, 16)) return rc;
    const hu128 c_lo_0_eval = h128(cb);
    t_.message(cb, 16);
    if (int rc = eq_levels({&pt}, n_ - 1, eq_)) return rc;
    if (int rc = eq_levels({&p3}, n_ - 1, eq2_)) return rc;
    // claims 0..96 the leaf pairs (slots 2p, 2p + 1, point pt), 97 the linear c_lo_0 claim (slot
    // 194, point pt), 98..161 the rerandomised b columns (slots 195 + k, point p3)
    const hu128 beta = sample(t_);
    std::vector<ImClaim> cl;
    for (int p = 0; p < 97; p++)
      cl.push_back(ImClaim{(uint16_t)(2 * p), (uint16_t)(2 * p + 1), 2, 0, 0});
    cl.push_back(ImClaim{194, 0, 1, 0, 0});
    for (int k = 0; k < 64; k++) cl.push_back(ImClaim{(uint16_t)(195 + k), 0, 1, 1, 0});
    std::vector<hu128> sums = evals;
    sums.push_back(c_lo_0_eval);
    sums.push_back(c_lo_0_eval);
    sums.insert(sums.end(), b_exp_evals.begin(), b_exp_evals.end());
    constexpr uint32_t kSlots = 2 * 97 + 1 + 64;
    DevBatch b;
    if (int rc = batch_begin(b, cl, {&pt, &p3}, sums, beta, kSlots)) return rc;
    // rounds of at most tail_items() (multilinear group, position) items: intmul_leaf_tail_kernel
    uint32_t t0 = 0;
    while (t0 < n_ && ((uint64_t)(kLeafPairs + 1 + kLeafCols) << (n_ - t0 - 1)) > tail_items())
      t0++;
    for (uint32_t t = 0; t < t0; t++) {
      const uint64_t L = 1ull << (n_ - t);
      uint32_t* out = batch_slots(b, t);
      const uint4* rp = batch_r(b, t);
      if (int rc = biv_round(leaves, 97, L, level(eq_, n_ - t - 1), rp, out)) return rc;
      if (int rc = lin_round(lo0, 1, L, level(eq_, n_ - t - 1), rp, out + 4 * 194)) return rc;
      if (int rc = lin_round(bcols, 64, L, level(eq2_, n_ - t - 1), rp, out + 4 * 195)) return rc;
      if (int rc = batch_round(b, t)) return rc;
    }
    if (t0 < n_) {
      BGPU_CUDA(launch_pdl(intmul_leaf_tail_kernel, 1, kImTailThreads, 0, s_, b.dt.state(),
                           b.dt.tape(), leaves, lo0, bcols, N_, n_, t0, (const uint4*)eq_,
                           (const uint4*)eq2_, (const uint4*)b.sums, (const uint4*)b.prefix,
                           (const ImAlpha*)b.alphas, (const uint4*)b.beta, b.chal));
      if (int rc = check("intmul_leaf_tail_kernel")) return rc;
    }
    std::vector<hu128> ch, last_leaves(2 * 194), last_lo(2), last_b(2 * 64);
    StagedReads rd(s_);
    if (int rc = batch_read(b, rd, ch)) return rc;
    if (int rc = copy_pairs(rd, leaves, 194, last_leaves.data())) return rc;
    if (int rc = copy_pairs(rd, lo0, 1, last_lo.data())) return rc;
    if (int rc = copy_pairs(rd, bcols, 64, last_b.data())) return rc;
    if (int rc = rd.wait()) return rc;
    if (int rc = batch_end(b)) return rc;
    const hu128 r = ch[n_ - 1];
    const std::vector<hu128> biv = fold_pairs(last_leaves, r), lo_ev = fold_pairs(last_lo, r),
                             b_ev = fold_pairs(last_b, r);
    write_elems(t_, biv);
    write_elems(t_, lo_ev);
    write_elems(t_, b_ev);
    // normalize_a_c_exponent_evals (common.rs:107-138)
    res.eval_point.assign(ch.rbegin(), ch.rend());
    normalize_leaves(biv, res);
    res.b_evals = b_ev;
  }
  return BINIUS_OK;
}

uint32_t log2_ceil(uint64_t n) {
  uint32_t r = 0;
  while ((1ull << r) < n) r++;
  return r;
}

}  // namespace

namespace bgpu {

// One MUL constraint (padded count 1): the trees of run's witness stage are 64-leaf exponent
// trees of four words, a few hundred products, so they are formed here from the operand words
// (read back with the commit's root by the prove entry) and the proof needs no device round
// trip for this phase.  Same values as const_leaves_kernel / var_leaves_kernel /
// tree_layer_kernel / bit_columns_kernel at n = 1.
int intmul_single_from_words(uint64_t a, uint64_t b, uint64_t lo, uint64_t hi, Transcript& t,
                             IntMulResult& res) {
  const hu128 g = ((hu128)0x494ef99794d5244fULL << 64) | (hu128)0x9152df59d87a9186ULL;
  std::vector<hu128> hacl(3 * 127 + 2), hb(127), hcols(64);
  auto leaves = [](uint64_t e, hu128 base, hu128* out) {  // bit_i(e) ? base^(2^i) : 1
    for (int i = 0; i < 64; i++, base = host_gf_mul(base, base)) out[i] = ((e >> i) & 1) ? base : 1;
  };
  hu128* l6 = hacl.data() + 3 * 63;
  leaves(a, g, l6);
  leaves(lo, g, l6 + 64);
  leaves(hi, sq_n(g, 64), l6 + 128);
  for (int k = 5; k >= 0; k--) {  // parent[q] = child[2q] child[2q + 1]
    const hu128* child = hacl.data() + 3 * ((2 << k) - 1);
    hu128* parent = hacl.data() + 3 * ((1 << k) - 1);
    for (int q = 0; q < (3 << k); q++) parent[q] = host_gf_mul(child[2 * q], child[2 * q + 1]);
  }
  hacl[3 * 127] = a & 1;
  hacl[3 * 127 + 1] = b & 1;
  leaves(b, hacl[0], hb.data() + 63);
  for (int k = 5; k >= 0; k--) {
    const hu128* child = hb.data() + ((2 << k) - 1);
    hu128* parent = hb.data() + ((1 << k) - 1);
    for (int q = 0; q < (1 << k); q++) parent[q] = host_gf_mul(child[2 * q], child[2 * q + 1]);
  }
  for (int i = 0; i < 64; i++) hcols[i] = (b >> i) & 1;
  emit_single(t, hacl, hb, hcols, host_gf_mul(hacl[1], hacl[2]), lo & 1, res);
  return BINIUS_OK;
}

int intmul_reduction_prove(const binius_cs* cs, const uint64_t* d_witness, Transcript& t,
                           IntMulResult& res, cudaStream_t s) {
  const uint64_t n = cs->mul_ops.n_constraints;
  uint64_t* cols = nullptr;
  BGPU_CUDA(dev_alloc(&cols, 8 * 4 * n, s));
  int rc = eval_operands(cs->mul_ops, d_witness, cols, s);
  if (!rc) {
    // CSR slots are (a, b, hi, lo)
    IntMulDevice dev(s, t);
    rc = dev.run(cols, cols + n, cols + 3 * n, cols + 2 * n, log2_ceil(n), res);
  }
  dev_free(cols, s);
  return rc;
}

}  // namespace bgpu

extern "C" {

int binius_intmul_reduction_prove(const binius_cs* cs, const void* d_witness,
                                  binius_transcript* transcript, void* h_out_point,
                                  void* h_out_evals, void* stream) {
  BGPU_ARG(cs && d_witness && transcript, "NULL argument");
  IntMulResult res;
  int rc = intmul_reduction_prove(cs, static_cast<const uint64_t*>(d_witness), transcript->t, res,
                                  as_stream(stream));
  if (rc) return rc;
  if (h_out_point && !res.eval_point.empty())
    memcpy(h_out_point, res.eval_point.data(), 16 * res.eval_point.size());
  if (h_out_evals) {
    uint8_t* o = static_cast<uint8_t*>(h_out_evals);
    const std::vector<hu128>* cols[4] = {&res.a_evals, &res.b_evals, &res.c_lo_evals,
                                         &res.c_hi_evals};
    for (int k = 0; k < 4; k++) memcpy(o + 16 * 64 * k, cols[k]->data(), 16 * 64);
  }
  return clear_error();
}

}  // extern "C"
