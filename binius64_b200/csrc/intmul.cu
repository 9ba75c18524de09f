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
// fold; the degree-2/3 coefficient algebra and the transcript run on the host between launches.
#include <string.h>

#include <algorithm>
#include <vector>

#include "cs.h"
#include "gf128.cuh"
#include "gf_reduce.cuh"
#include "internal.h"
#include "kernels.h"
#include "reductions.h"
#include "transcript.h"

using namespace bgpu;

namespace {

constexpr int kT = 256;

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

// Pair p of `set` (multilinears 2p, 2p + 1 of length 2 * half): out[2p] += sum eq[i] a1 b1,
// out[2p + 1] += sum eq[i] (a0 + a1)(b0 + b1).  Grid: (chunks, pairs).
__global__ void __launch_bounds__(kT)
    biv_round_kernel(const uint4* __restrict__ set, uint64_t half, uint64_t stride,
                     const uint4* __restrict__ eq, uint32_t* __restrict__ out) {
  const uint32_t p = blockIdx.y;
  const uint4* a = set + 2 * p * stride;
  const uint4* b = a + stride;
  u256 s1 = {0, 0, 0, 0}, sinf = {0, 0, 0, 0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < half;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 e = eq[i];
    const uint4 a0 = a[i], a1 = a[half + i], b0 = b[i], b1 = b[half + i];
    xor_into(s1, clmul128(e, gf_mul(a1, b1)));
    xor_into(sinf, clmul128(e, gf_mul(gf_add(a0, a1), gf_add(b0, b1))));
  }
  uint4 v[2] = {reduce256(s1), reduce256(sinf)};
  block_xor_reduce<2>(v, out + 8 * p);
}

// Column k of `set`: out[k] += sum eq[i] col_k[half + i].  Grid: (chunks, columns).
__global__ void __launch_bounds__(kT)
    lin_round_kernel(const uint4* __restrict__ set, uint64_t half, uint64_t stride,
                     const uint4* __restrict__ eq, uint32_t* __restrict__ out) {
  const uint32_t k = blockIdx.y;
  const uint4* c = set + k * stride + half;
  u256 s1 = {0, 0, 0, 0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < half;
       i += (uint64_t)gridDim.x * blockDim.x)
    xor_into(s1, clmul128(eq[i], c[i]));
  uint4 v[1] = {reduce256(s1)};
  block_xor_reduce<1>(v, out + 4 * k);
}

// Selector claim k (its own eq_k): out[2k] += sum eq_k[i] (s1 (sel1 + 1) + 1),
// out[2k + 1] += sum eq_k[i] (s0 + s1)(sel0 + sel1).  Grid: (chunks, claims).
__global__ void __launch_bounds__(kT)
    selector_round_kernel(const uint4* __restrict__ sel, const uint4* __restrict__ cols,
                          uint64_t half, uint64_t stride, const uint4* __restrict__ eqs,
                          uint64_t eq_stride, uint32_t* __restrict__ out) {
  const uint32_t k = blockIdx.y;
  const uint4* s = cols + k * stride;
  const uint4* eq = eqs + k * eq_stride;
  u256 s1 = {0, 0, 0, 0}, sinf = {0, 0, 0, 0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < half;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 e = eq[i];
    const uint4 sel0 = sel[i], sel1 = sel[half + i], c0 = s[i], c1 = s[half + i];
    xor_into(s1, clmul128(e, gf_add(gf_mul(c1, gf_add(sel1, gf_one())), gf_one())));
    xor_into(sinf, clmul128(e, gf_mul(gf_add(c0, c1), gf_add(sel0, sel1))));
  }
  uint4 v[2] = {reduce256(s1), reduce256(sinf)};
  block_xor_reduce<2>(v, out + 8 * k);
}

// In-place top-variable fold of `count` multilinears of length 2 * half.
__global__ void fold_set_kernel(uint4* __restrict__ set, uint32_t count, uint64_t half,
                                uint64_t stride, uint4 r) {
  const uint64_t total = (uint64_t)count * half;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = t / half, i = t - k * half;
    uint4* m = set + k * stride;
    const uint4 lo = m[i], hi = m[half + i];
    m[i] = gf_add(lo, gf_mul(r, gf_add(hi, lo)));
  }
}

// eq over one coordinate fewer: eq_k[i] += eq_k[i + half] (eq_ind_truncate_low_inplace).
__global__ void eq_truncate_kernel(uint4* __restrict__ eqs, uint32_t count, uint64_t half,
                                   uint64_t stride) {
  const uint64_t total = (uint64_t)count * half;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = t / half, i = t - k * half;
    gf_add_into(eqs[k * stride + i], eqs[k * stride + half + i]);
  }
}

// count eq tensors over m coordinates each: out[k * stride + i] = prod_j (bit_j(i) ? p : 1 + p)
// with p = points[k * m + j].
__global__ void eq_many_kernel(const uint4* __restrict__ points, uint32_t count, uint32_t m,
                               uint4* __restrict__ out, uint64_t stride) {
  const uint64_t len = 1ull << m, total = (uint64_t)count * len;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = t / len, i = t - k * len;
    uint4 acc = gf_one();
    for (uint32_t j = 0; j < m; j++) {
      const uint4 p = points[k * m + j];
      acc = gf_mul(acc, ((i >> j) & 1) ? p : gf_add(p, gf_one()));
    }
    out[k * stride + i] = acc;
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

// ---------------------------------------------------------------- host side

typedef std::vector<hu128> Poly;

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

hu128 eval_poly(const Poly& c, hu128 x) {
  hu128 acc = 0;
  for (size_t i = c.size(); i-- > 0;) acc = host_gf_mul(acc, x) ^ c[i];
  return acc;
}
// (1 + alpha)^-1 (invert_or_zero), memoised per thread: the claims of one prover share alpha.
hu128 inv_one_plus(hu128 alpha) {
  thread_local hu128 last_alpha = 0, last_inv = 1;
  if (alpha != last_alpha) {
    last_alpha = alpha;
    last_inv = host_gf_inv(1 ^ alpha);
  }
  return last_inv;
}
// RoundEvals2 / RoundEvals1 ::interpolate_eq (round_evals.rs:23-27, 80-87).
Poly interp2(hu128 sum, hu128 y1, hu128 yinf, hu128 alpha) {
  const hu128 y0 = host_gf_mul(sum ^ host_gf_mul(y1, alpha), inv_one_plus(alpha));
  return {y0, y1 ^ y0 ^ yinf, yinf};
}
Poly interp1(hu128 sum, hu128 y1, hu128 alpha) {
  const hu128 y0 = host_gf_mul(sum ^ host_gf_mul(y1, alpha), inv_one_plus(alpha));
  return {y0, y1 ^ y0};
}
// round_coeffs_by_eq (round_evals.rs:145-156) times `scale`.
Poly by_eq(const Poly& prime, hu128 alpha, hu128 scale) {
  Poly out(prime.size() + 1, 0);
  for (size_t i = 0; i < prime.size(); i++) {
    out[i] ^= host_gf_mul(prime[i], 1 ^ alpha);
    out[i + 1] ^= prime[i];
  }
  for (auto& c : out) c = host_gf_mul(c, scale);
  return out;
}
hu128 sample(Transcript& t) {
  uint8_t b[16];
  t.sample_elem(b);
  return h128(b);
}
void write_elems(Transcript& t, const std::vector<hu128>& v) {
  if (!v.empty()) t.message(v.data(), 16 * v.size());
}
// Batched round polynomial sum_i beta^i c_i (rfold in batch.rs:76-78), truncated and written.
void write_batched(Transcript& t, const std::vector<Poly>& all, hu128 beta) {
  Poly acc;
  for (size_t i = all.size(); i-- > 0;) {
    for (auto& c : acc) c = host_gf_mul(c, beta);
    if (acc.size() < all[i].size()) acc.resize(all[i].size(), 0);
    for (size_t k = 0; k < all[i].size(); k++) acc[k] ^= all[i][k];
  }
  acc.pop_back();
  write_elems(t, acc);
}

// The Gruen eq factor of an MLE-check: eq over point[0 .. n_rem - 1) on the device plus the
// prefix product of eq_one_var over the folded coordinates.
struct GruenState {
  std::vector<hu128> point;
  uint32_t n_rem;
  hu128 prefix = 1;
  hu128 alpha() const { return point[n_rem - 1]; }
  void fold(hu128 r) {
    prefix = host_gf_mul(prefix, 1 ^ r ^ alpha());
    n_rem--;
  }
};

class IntMulDevice {
 public:
  IntMulDevice(cudaStream_t s, Transcript& t) : s_(s), t_(t) {}
  ~IntMulDevice() {
    for (void* p : ptrs_) cudaFreeAsync(p, s_);
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
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(p), 16 * std::max<size_t>(elems16, 1), s_);
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
  int sync_read(void* dst, const void* src, size_t bytes) {
    BGPU_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s_));
    BGPU_CUDA(stream_wait(s_));
    return BINIUS_OK;
  }
  // values [0] of `count` multilinears with stride `stride`
  int read_first(const uint4* set, uint32_t count, uint64_t stride, std::vector<hu128>& out) {
    out.resize(count);
    BGPU_CUDA(cudaMemcpy2DAsync(out.data(), 16, set, 16 * stride, 16, count,
                                cudaMemcpyDeviceToHost, s_));
    BGPU_CUDA(stream_wait(s_));
    return BINIUS_OK;
  }
  int eq_single(const std::vector<hu128>& point, uint32_t m, uint4* out) {
    std::vector<uint4> p(m);
    for (uint32_t i = 0; i < m; i++) p[i] = u4(point[i]);
    return eq_tensor(p.data(), m, out, s_);
  }
  int fold(uint4* set, uint32_t count, uint64_t half, hu128 r) {
    if (half == 0) return BINIUS_OK;
    fold_set_kernel<<<blocks_for((uint64_t)count * half), kT, 0, s_>>>(set, count, half, N_, u4(r));
    return check("fold_set_kernel");
  }
  int truncate(uint4* eqs, uint32_t count, uint64_t half) {
    if (half == 0) return BINIUS_OK;
    eq_truncate_kernel<<<blocks_for((uint64_t)count * half), kT, 0, s_>>>(eqs, count, half, N_);
    return check("eq_truncate_kernel");
  }
  int biv_round(const uint4* set, uint32_t pairs, uint64_t half, const uint4* eq, uint32_t* out) {
    dim3 grid(blocks_for(half, 148 * 2), pairs);
    biv_round_kernel<<<grid, kT, 0, s_>>>(set, half, N_, eq, out);
    return check("biv_round_kernel");
  }
  int lin_round(const uint4* set, uint32_t cols, uint64_t half, const uint4* eq, uint32_t* out) {
    dim3 grid(blocks_for(half, 148 * 2), cols);
    lin_round_kernel<<<grid, kT, 0, s_>>>(set, half, N_, eq, out);
    return check("lin_round_kernel");
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
  GruenState g{point, n};
  if (n > 0)
    if (int rc = eq_single(point, n - 1, eq_)) return rc;
  std::vector<hu128> sums = claims, ch;
  std::vector<uint8_t> host(32ull * pairs);
  for (uint32_t round = 0; round < n; round++) {
    const uint64_t half = 1ull << (g.n_rem - 1);
    BGPU_CUDA(cudaMemsetAsync(acc_, 0, 32ull * pairs, s_));
    if (int rc = biv_round(set, pairs, half, eq_, acc_)) return rc;
    if (int rc = sync_read(host.data(), acc_, 32ull * pairs)) return rc;
    const hu128 alpha = g.alpha();
    std::vector<Poly> primes, all;
    for (uint32_t p = 0; p < pairs; p++) {
      primes.push_back(interp2(sums[p], h128(&host[32 * p]), h128(&host[32 * p + 16]), alpha));
      all.push_back(by_eq(primes.back(), alpha, g.prefix));
    }
    write_batched(t_, all, beta);
    const hu128 r = sample(t_);
    ch.push_back(r);
    for (uint32_t p = 0; p < pairs; p++) sums[p] = eval_poly(primes[p], r);
    g.fold(r);
    if (int rc = fold(set, 2 * pairs, half, r)) return rc;
    if (int rc = truncate(eq_, 1, half / 2)) return rc;
  }
  std::vector<hu128> evals;
  if (int rc = read_first(set, 2 * pairs, N_, evals)) return rc;
  write_elems(t_, evals);
  point.assign(ch.rbegin(), ch.rend());
  claims = evals;
  return BINIUS_OK;
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
  BGPU_CUDA(cudaMemcpyAsync(hacl.data(), acl, 16 * kAcl, cudaMemcpyDeviceToHost, s_));
  BGPU_CUDA(cudaMemcpyAsync(hb.data(), btree, 16 * kB, cudaMemcpyDeviceToHost, s_));
  BGPU_CUDA(cudaMemcpyAsync(hcols.data(), bcols, 16 * 64, cudaMemcpyDeviceToHost, s_));
  BGPU_CUDA(cudaMemcpyAsync(&c_root, acc_, 16, cudaMemcpyDeviceToHost, s_));
  BGPU_CUDA(cudaMemcpyAsync(&lo_bit, lo0, 16, cudaMemcpyDeviceToHost, s_));
  BGPU_CUDA(stream_wait(s_));
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

  // ---- phase 2: frobenius twist (common.rs:81-105)
  std::vector<std::vector<hu128>> tw_points(64);
  std::vector<hu128> sel_sums(64);
  for (int i = 0; i < 64; i++) {
    for (hu128 c : pt) tw_points[i].push_back(sq_n(c, 128 - i));
    sel_sums[i] = sq_n(evals[i], 128 - i);
  }

  // ---- phase 3: selector prover on (a_root, bits of b) + bivariate c root prover
  std::vector<hu128> p3, b_exp_evals;
  hu128 selector_eval, c_lo_root_eval, c_hi_root_eval;
  {
    bit_columns_kernel<<<blocks_for(64 * N), kT, 0, s_>>>(d_b, N, 0, 64, bcols, N);
    if (int rc = check("bit_columns_kernel")) return rc;
    if (n_ > 0) {
      std::vector<uint4> pts;
      for (int i = 0; i < 64; i++)
        for (uint32_t j = 0; j + 1 < n_; j++) pts.push_back(u4(tw_points[i][j]));
      uint4* d_pts = nullptr;
      if (int rc = alloc(&d_pts, pts.size())) return rc;
      BGPU_CUDA(cudaMemcpyAsync(d_pts, pts.data(), 16 * pts.size(), cudaMemcpyHostToDevice, s_));
      eq_many_kernel<<<blocks_for(64ull << (n_ - 1)), kT, 0, s_>>>(d_pts, 64, n_ - 1, sel_eqs, N);
      if (int rc = check("eq_many_kernel")) return rc;
      if (int rc = eq_single(point0, n_ - 1, eq_)) return rc;
    }
    std::vector<GruenState> gs;
    for (int i = 0; i < 64; i++) gs.push_back(GruenState{tw_points[i], n_});
    GruenState gc{point0, n_};
    uint4* sel = acl_layer(0);
    uint4* croot = acl_layer(0) + N;
    hu128 c_sum = c_eval;
    const hu128 beta = sample(t_);
    std::vector<uint8_t> host(16 * (128 + 2));
    std::vector<hu128> ch;
    for (uint32_t round = 0; round < n_; round++) {
      const uint64_t half = 1ull << (n_ - round - 1);
      BGPU_CUDA(cudaMemsetAsync(acc, 0, 16 * 130, s_));
      dim3 grid(blocks_for(half, 148 * 2), 64);
      selector_round_kernel<<<grid, kT, 0, s_>>>(sel, bcols, half, N, sel_eqs, N, acc);
      if (int rc = check("selector_round_kernel")) return rc;
      if (int rc = biv_round(croot, 1, half, eq_, acc + 4 * 128)) return rc;
      if (int rc = sync_read(host.data(), acc, host.size())) return rc;
      std::vector<Poly> primes, all;
      for (int i = 0; i < 64; i++) {
        const hu128 a = gs[i].alpha();
        primes.push_back(interp2(sel_sums[i], h128(&host[32 * i]), h128(&host[32 * i + 16]), a));
        all.push_back(by_eq(primes.back(), a, gs[i].prefix));
      }
      primes.push_back(interp2(c_sum, h128(&host[2048]), h128(&host[2048 + 16]), gc.alpha()));
      all.push_back(by_eq(primes.back(), gc.alpha(), gc.prefix));
      write_batched(t_, all, beta);
      const hu128 r = sample(t_);
      ch.push_back(r);
      for (int i = 0; i < 64; i++) {
        sel_sums[i] = eval_poly(primes[i], r);
        gs[i].fold(r);
      }
      c_sum = eval_poly(primes[64], r);
      gc.fold(r);
      if (int rc = fold(sel, 3, half, r)) return rc;  // a_root, c_lo_root, c_hi_root
      if (int rc = fold(bcols, 64, half, r)) return rc;
      if (int rc = truncate(sel_eqs, 64, half / 2)) return rc;
      if (int rc = truncate(eq_, 1, half / 2)) return rc;
    }
    std::vector<hu128> colv, roots;
    if (int rc = read_first(bcols, 64, N, colv)) return rc;
    if (int rc = read_first(sel, 3, N, roots)) return rc;
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
    if (n_ > 0) {
      if (int rc = eq_single(pt, n_ - 1, eq_)) return rc;
      if (int rc = eq_single(p3, n_ - 1, eq2_)) return rc;
    }
    GruenState gb{pt, n_}, gl{pt, n_}, gr{p3, n_};
    std::vector<hu128> biv_sums = evals;
    biv_sums.push_back(c_lo_0_eval);
    hu128 lo_sum = c_lo_0_eval;
    std::vector<hu128> b_sums = b_exp_evals;
    const hu128 beta = sample(t_);
    const size_t nbytes = 16 * (2 * 97 + 1 + 64);
    std::vector<uint8_t> host(nbytes);
    std::vector<hu128> ch;
    for (uint32_t round = 0; round < n_; round++) {
      const uint64_t half = 1ull << (n_ - round - 1);
      BGPU_CUDA(cudaMemsetAsync(acc, 0, nbytes, s_));
      if (int rc = biv_round(leaves, 97, half, eq_, acc)) return rc;
      if (int rc = lin_round(lo0, 1, half, eq_, acc + 4 * 194)) return rc;
      if (int rc = lin_round(bcols, 64, half, eq2_, acc + 4 * 195)) return rc;
      if (int rc = sync_read(host.data(), acc, nbytes)) return rc;
      std::vector<Poly> primes, all;
      for (int p = 0; p < 97; p++) {
        primes.push_back(interp2(biv_sums[p], h128(&host[32 * p]), h128(&host[32 * p + 16]), gb.alpha()));
        all.push_back(by_eq(primes.back(), gb.alpha(), gb.prefix));
      }
      primes.push_back(interp1(lo_sum, h128(&host[16 * 194]), gl.alpha()));
      all.push_back(by_eq(primes.back(), gl.alpha(), gl.prefix));
      for (int k = 0; k < 64; k++) {
        primes.push_back(interp1(b_sums[k], h128(&host[16 * (195 + k)]), gr.alpha()));
        all.push_back(by_eq(primes.back(), gr.alpha(), gr.prefix));
      }
      write_batched(t_, all, beta);
      const hu128 r = sample(t_);
      ch.push_back(r);
      for (int p = 0; p < 97; p++) biv_sums[p] = eval_poly(primes[p], r);
      lo_sum = eval_poly(primes[97], r);
      for (int k = 0; k < 64; k++) b_sums[k] = eval_poly(primes[98 + k], r);
      gb.fold(r);
      gl.fold(r);
      gr.fold(r);
      if (int rc = fold(leaves, 194, half, r)) return rc;
      if (int rc = fold(lo0, 1, half, r)) return rc;
      if (int rc = fold(bcols, 64, half, r)) return rc;
      if (int rc = truncate(eq_, 1, half / 2)) return rc;
      if (int rc = truncate(eq2_, 1, half / 2)) return rc;
    }
    std::vector<hu128> biv, lo_ev, b_ev;
    if (int rc = read_first(leaves, 194, N, biv)) return rc;
    if (int rc = read_first(lo0, 1, N, lo_ev)) return rc;
    if (int rc = read_first(bcols, 64, N, b_ev)) return rc;
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

int intmul_reduction_prove(const binius_cs* cs, const uint64_t* d_witness, Transcript& t,
                           IntMulResult& res, cudaStream_t s) {
  const uint64_t n = cs->mul_ops.n_constraints;
  uint64_t* cols = nullptr;
  BGPU_CUDA(cudaMallocAsync(&cols, 8 * 4 * n, s));
  int rc = eval_operands(cs->mul_ops, d_witness, cols, s);
  if (!rc) {
    // CSR slots are (a, b, hi, lo)
    IntMulDevice dev(s, t);
    rc = dev.run(cols, cols + n, cols + 3 * n, cols + 2 * n, log2_ceil(n), res);
  }
  cudaFreeAsync(cols, s);
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
