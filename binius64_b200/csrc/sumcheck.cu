// Multilinear / sumcheck kernels of the PCS opening and the reductions.
//
// * eq tensor (eq_ind_partial_eval, verifier/math/src/multilinear/eq.rs:39-71): coordinate i
//   selects index bit i; built as lo[i & mask] * hi[i >> k] from two small tensors (one multiply
//   per output; the product order does not change the field value).
// * ring-switch row fold (fold_1b_rows_for_b128, prover/prover/src/ring_switch.rs:197-265):
//   out[k] = sum_i bit_k(mat[i]) * vec[i] for the 128 bit columns k.  A CTA of 128 threads gives
//   one column to each thread, streams rows through shared memory and XOR-accumulates the masked
//   vector entries; CTA partials meet in global memory through atomicXor (addition in GF(2^128)).
// * element fold (fold_b128_elems_inplace, ring_switch.rs:130-171): x -> sum_k bit_k(x) * vec[k]
//   through 16 byte-indexed tables of 256 subset sums held in shared memory.
// * bivariate product round (BivariateProductSumcheckProver::execute / fold,
//   prover/prover/src/protocols/sumcheck/bivariate_product.rs:43-95): y_1 = sum a_hi*b_hi,
//   y_inf = sum (a_lo + a_hi)(b_lo + b_hi), the top variable is folded by
//   fold_highest_var_inplace (multilinear/fold.rs:14-29).  The fold by the previous challenge and
//   the next round's evaluation run in one pass; products accumulate unreduced (256-bit) and are
//   reduced once per thread.
#include <string.h>

#include <algorithm>

#include "dev_transcript.cuh"
#include "pdl.cuh"
#include "gf128.cuh"
#include "gf_reduce.cuh"
#include "internal.h"
#include "kernels.h"

using namespace bgpu;

namespace {

constexpr int kThreads = 256;
constexpr int kTailThreads = 512;

uint4 gf_zero_host() { return make_uint4(0u, 0u, 0u, 0u); }

unsigned grid_for(uint64_t n, unsigned threads, unsigned max_blocks = 148 * 8) {
  uint64_t g = (n + threads - 1) / threads;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, max_blocks));
}

// out[j] = prod_i (bit_i(j) ? r_i : 1 + r_i) for n <= 16 coordinates.  Each block first builds
// the eq tensors of the low k = min(n, 8) and the high n - k coordinates (at most 256 entries
// each) in shared memory, then every output is one multiply lo[j mod 2^k] * hi[j >> k].  The
// tables are built by doubling (8 steps of one multiply per thread; a balanced product tree per
// entry on one thread, its multiplies sequential calls, cost ~20 us more per 2^20 proof).  These
// tensors are small and on the protocol's critical path, so latency matters: the tables depend
// only on the point (a kernel argument), so under programmatic dependent launch they are built
// while the previous kernel still runs, and only the writes wait for it.
__global__ void __launch_bounds__(256)
    eq_small_kernel(uint4* __restrict__ out, Point32 p, uint32_t off, uint32_t n) {
  __shared__ uint4 s_lo[256], s_hi[256];
  const uint32_t k = n < 8 ? n : 8, m = n - k;
  const uint32_t n_lo = 1u << k;
  // threads 0..127 build the low table, 128..255 the high one, by doubling: after step i a
  // table holds eq of its first i + 1 coordinates (entry t: factor 1 + r_i, t + 2^i: r_i)
  const bool lo_side = threadIdx.x < 128;
  const uint32_t t = threadIdx.x & 127, cnt = lo_side ? k : m, first = lo_side ? off : off + k;
  uint4* tab = lo_side ? s_lo : s_hi;
  if (t == 0) tab[0] = gf_one();
  for (uint32_t i = 0; i < 8; i++) {
    __syncthreads();
    if (i < cnt && t < (1u << i)) {
      const uint4 x = tab[t], y = gf_mul(x, p.r[first + i]);
      tab[t + (1u << i)] = y;
      tab[t] = gf_add(x, y);
    }
  }
  pdl_wait();
  pdl_trigger();
  __syncthreads();
  const uint64_t total = 1ull << n;
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < total;
       j += (uint64_t)gridDim.x * blockDim.x)
    out[j] = gf_mul(s_lo[j & (n_lo - 1)], s_hi[j >> k]);
}

__global__ void eq_expand_kernel(uint4* __restrict__ out, const uint4* __restrict__ lo,
                                 const uint4* __restrict__ hi, uint32_t k, uint64_t total) {
  pdl_wait();
  pdl_trigger();
  const uint64_t mask = (1ull << k) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = gf_mul(__ldg(lo + (i & mask)), __ldg(hi + (i >> k)));
}

constexpr int kRowTile = 256;

__global__ void __launch_bounds__(128)
    fold_rows_kernel(const uint4* __restrict__ mat, const uint4* __restrict__ vec, uint64_t n,
                     uint32_t* __restrict__ out) {
  __shared__ uint32_t s_mat[kRowTile][4];
  __shared__ uint4 s_vec[kRowTile];
  const uint32_t k = threadIdx.x;  // bit column
  const uint32_t word = k >> 5, bit = k & 31;
  uint4 acc = gf_zero();
  for (uint64_t base = (uint64_t)blockIdx.x * kRowTile; base < n;
       base += (uint64_t)gridDim.x * kRowTile) {
    const uint32_t rows = (uint32_t)((n - base) < (uint64_t)kRowTile ? (n - base) : (uint64_t)kRowTile);
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x) {
      uint4 m = __ldg(mat + base + r);
      s_mat[r][0] = m.x;
      s_mat[r][1] = m.y;
      s_mat[r][2] = m.z;
      s_mat[r][3] = m.w;
      s_vec[r] = __ldg(vec + base + r);
    }
    __syncthreads();
    for (uint32_t r = 0; r < rows; r++) {
      const uint32_t msk = 0u - ((s_mat[r][word] >> bit) & 1u);
      const uint4 v = s_vec[r];
      acc.x ^= v.x & msk;
      acc.y ^= v.y & msk;
      acc.z ^= v.z & msk;
      acc.w ^= v.w & msk;
    }
  }
  atomic_xor_gf(out + 4 * k, acc);
}

// tables[p][b] = sum over the set bits j of b of vec[8p + j].
__global__ void build_fold_tables_kernel(const uint4* __restrict__ vec, uint4* __restrict__ tables) {
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 16 * 256) return;
  const uint32_t p = idx >> 8, b = idx & 255;
  uint4 acc = gf_zero();
  for (uint32_t j = 0; j < 8; j++)
    if ((b >> j) & 1) gf_add_into(acc, vec[8 * p + j]);
  tables[idx] = acc;
}

__device__ __forceinline__ uint32_t byte_of(uint4 v, uint32_t p) {
  const uint32_t w = p < 4 ? v.x : p < 8 ? v.y : p < 12 ? v.z : v.w;
  return (w >> (8 * (p & 3))) & 255u;
}

__global__ void __launch_bounds__(kThreads)
    fold_elems_kernel(const uint4* __restrict__ in, uint4* __restrict__ out, uint64_t n,
                      const uint4* __restrict__ tables) {
  extern __shared__ uint4 s_tab[];  // 16 x 256
  for (uint32_t i = threadIdx.x; i < 16 * 256; i += blockDim.x) s_tab[i] = tables[i];
  __syncthreads();
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 x = in[i];
    uint4 acc = gf_zero();
#pragma unroll
    for (uint32_t p = 0; p < 16; p++) gf_add_into(acc, s_tab[(p << 8) | byte_of(x, p)]);
    out[i] = acc;
  }
}

// Round evaluation on (a, b) of length 2*half, no fold.
__global__ void __launch_bounds__(kThreads)
    bivariate_eval_kernel(const uint4* __restrict__ a, const uint4* __restrict__ b, uint64_t half,
                          uint32_t* __restrict__ out) {
  u256 s1 = {0, 0, 0, 0}, sinf = {0, 0, 0, 0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < half;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 a0 = a[i], a1 = a[half + i], b0 = b[i], b1 = b[half + i];
    xor_into(s1, clmul128(a1, b1));
    xor_into(sinf, clmul128(gf_add(a0, a1), gf_add(b0, b1)));
  }
  uint4 v[2] = {reduce256(s1), reduce256(sinf)};
  block_xor_reduce<2>(v, out);
}

// Folds (a, b) of length `size` by r in place (a[i] = a[i] + r (a[i + size/2] - a[i])) and
// evaluates the next round on the folded length-size/2 arrays.  Each folded position j < size/4
// belongs to a pair of adjacent lanes: the odd lane folds a and b at j, the even lane at
// j + size/4, and each forms one of the two products (the even lane y_1's fa1 fb1, the odd lane
// y_inf's after a shuffle brings fa1, fb1 over).  The products by r go through r's nibble tables,
// which each block builds in shared memory from r (read from r_ptr, else r_arg).
__global__ void __launch_bounds__(kThreads)
    bivariate_fold_eval_kernel(uint4* __restrict__ a, uint4* __restrict__ b, uint64_t size,
                               uint4 r_arg, const uint4* __restrict__ r_ptr,
                               uint32_t* __restrict__ out) {
  __shared__ NibbleTable tab;
  __shared__ uint4 basis[128];
  pdl_wait();
  pdl_trigger();
  nibble_table_build(tab, basis, r_ptr ? *r_ptr : r_arg);
  const uint64_t h = size >> 1, q = size >> 2;
  const uint32_t odd = threadIdx.x & 1;
  u256 acc = {0, 0, 0, 0};
  const uint64_t all = (uint64_t)gridDim.x * blockDim.x;
  // warp-uniform sweeps: every lane of a warp runs the same iterations (shuffles below)
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u); base < 2 * q;
       base += all) {
    const uint64_t j = (base + (threadIdx.x & 31)) >> 1;
    const bool live = j < q;
    uint4 fa = gf_zero(), fb = gf_zero();
    if (live) {
      const uint64_t pos = odd ? j : q + j;
      const uint4 a_lo = a[pos], a_hi = a[h + pos], b_lo = b[pos], b_hi = b[h + pos];
      fa = gf_add(a_lo, gf_mul_nibble(tab, gf_add(a_hi, a_lo)));
      fb = gf_add(b_lo, gf_mul_nibble(tab, gf_add(b_hi, b_lo)));
      a[pos] = fa;
      b[pos] = fb;
    }
    // the odd lane takes its even partner's (fa1, fb1)
    const uint4 pa = shfl_gf(fa, 0, 2), pb = shfl_gf(fb, 0, 2);
    // one product per lane, selected without divergence (fa, fb are zero on dead lanes)
    xor_into(acc, clmul128(odd ? gf_add(fa, pa) : fa, odd ? gf_add(fb, pb) : fb));
  }
  const uint4 s = reduce256(acc);
  uint4 v[2] = {odd ? gf_zero() : s, odd ? s : gf_zero()};
  block_xor_reduce<2>(v, out);
}

// The small rounds of bivariate_fold_eval_kernel (no nibble tables) on four lanes per position j:
// lane k folds one of a[j], a[q + j], b[j], b[q + j] by r, the four folded values are shared by
// shuffles, and lanes 0 and 1 form the two products.  One multiply then one product per lane,
// where one thread per position ran six dependent out-of-line multiplies: these rounds are
// latency chains on few CTAs.
__global__ void __launch_bounds__(kThreads)
    bivariate_fold_eval_lanes_kernel(uint4* __restrict__ a, uint4* __restrict__ b, uint64_t size,
                                     uint4 r_arg, const uint4* __restrict__ r_ptr,
                                     uint32_t* __restrict__ out) {
  pdl_wait();
  pdl_trigger();
  const uint64_t h = size >> 1, q = size >> 2;
  const uint4 r = r_ptr ? *r_ptr : r_arg;
  const uint32_t k = threadIdx.x & 3;
  uint4 v[2] = {gf_zero(), gf_zero()};
  const uint64_t all = (uint64_t)gridDim.x * blockDim.x;
  // warp-uniform sweeps: every lane of a warp runs the same iterations (shuffles below)
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u); base < 4 * q;
       base += all) {
    const uint64_t j = (base + (threadIdx.x & 31)) >> 2;
    const bool live = j < q;
    uint4 f = gf_zero();
    if (live) {
      uint4* col = k < 2 ? a : b;
      const uint64_t pos = j + ((k & 1) ? q : 0);
      const uint4 lo = col[pos];
      f = gf_add(lo, gf_mul_nl(r, gf_add(col[h + pos], lo)));
      col[pos] = f;
    }
    const uint4 fa0 = shfl_gf(f, 0, 4), fa1 = shfl_gf(f, 1, 4), fb0 = shfl_gf(f, 2, 4),
                fb1 = shfl_gf(f, 3, 4);
    if (live && k == 0) gf_add_into(v[0], gf_mul_nl(fa1, fb1));
    if (live && k == 1) gf_add_into(v[1], gf_mul_nl(gf_add(fa0, fa1), gf_add(fb0, fb1)));
  }
  block_xor_reduce<2>(v, out);
}

// The Fiat-Shamir step of a plain bivariate product round (BivariateProductSumcheckProver,
// bivariate_product.rs:43-95, through the prover's round-proof truncation) on the device: the
// sums (y_1, y_inf) and the claim give c_0 = claim + y_1, c_2 = y_inf, c_1 = y_1 + c_0 + c_2; the
// message is (c_0, c_1), then optionally a 32-byte commitment (a Merkle root the device just
// built), then the challenge r is sampled and the claim becomes c_0 + c_1 r + c_2 r^2.  The claim
// is read from claim_init when that is set (the first round).  One warp runs the step.
__global__ void __launch_bounds__(32)
    bivariate_round_finish_kernel(TranscriptState* __restrict__ ts, uint8_t* __restrict__ tape,
                                  const uint4* __restrict__ ys, const uint4* __restrict__ claim_init,
                                  uint4* __restrict__ claim, const uint8_t* __restrict__ commitment,
                                  uint4* __restrict__ r_out) {
  pdl_wait();
  pdl_trigger();
  {
    DevTr st;
    st.load(ts);
    const uint4 y1 = ys[0], yinf = ys[1];
    const uint4 c0 = gf_add(claim_init ? *claim_init : *claim, y1), c2 = yinf;
    const uint4 c1 = gf_add(gf_add(y1, c0), c2);
    const uint4 msg[2] = {c0, c1};
    st.message_elems(tape, msg, 2);
    if (commitment) {
      uint32_t root[8];
      for (int i = 0; i < 8; i++) root[i] = reinterpret_cast<const uint32_t*>(commitment)[i];
      st.message_words(tape, root, 8);
    }
    const uint4 r = st.sample_elem();
    *r_out = r;
    *claim = gf_add(c0, gf_mul_warp(r, gf_add(c1, gf_mul_warp(c2, r))));
    st.store(ts);
  }
}

// The small last rounds of a plain bivariate product sumcheck in one CTA: per round, fold (a, b)
// by the previous challenge (r_first for the first round when set), evaluate (y_1, y_inf) on the
// folded arrays, and let warp 0 run the Fiat-Shamir step of bivariate_round_finish_kernel with
// the transcript held in its registers.  The rounds of a sumcheck below a few thousand elements
// are latency chains; run as one launch, the loop body stays in the instruction cache and no
// launch gap separates the rounds.  len is the arrays' length before the first fold.
__global__ void __launch_bounds__(kTailThreads)
    bivariate_tail_kernel(TranscriptState* __restrict__ ts, uint8_t* __restrict__ tape,
                          uint4* __restrict__ a, uint4* __restrict__ b, uint64_t len,
                          uint32_t n_rounds, const uint4* __restrict__ r_first,
                          uint4* __restrict__ claim, uint4* __restrict__ chal) {
  pdl_wait();
  pdl_trigger();
  __shared__ uint4 r_sh;
  DevTr st;
  uint4 cl = gf_zero();
  if (threadIdx.x < 32) {
    st.load(ts);
    cl = *claim;
    if (r_first) r_sh = *r_first;
  }
  __syncthreads();
  for (uint32_t k = 0; k < n_rounds; k++) {
    if (k > 0 || r_first) {
      const uint4 r = r_sh;
      const uint64_t h = len >> 1;
      for (uint64_t j = threadIdx.x; j < h; j += blockDim.x) {
        const uint4 a0 = a[j], b0 = b[j];
        a[j] = gf_add(a0, gf_mul_nl(r, gf_add(a[h + j], a0)));
        b[j] = gf_add(b0, gf_mul_nl(r, gf_add(b[h + j], b0)));
      }
      len = h;
      __syncthreads();
    }
    const uint64_t h = len >> 1;
    uint4 v[2] = {gf_zero(), gf_zero()};
    for (uint64_t j = threadIdx.x; j < h; j += blockDim.x) {
      const uint4 a0 = a[j], a1 = a[h + j], b0 = b[j], b1 = b[h + j];
      gf_add_into(v[0], gf_mul_nl(a1, b1));
      gf_add_into(v[1], gf_mul_nl(gf_add(a0, a1), gf_add(b0, b1)));
    }
    block_xor_sum<2>(v);
    if (threadIdx.x < 32) {
      const uint4 y1 = v[0], yinf = v[1];
      const uint4 c0 = gf_add(cl, y1), c2 = yinf, c1 = gf_add(gf_add(y1, c0), c2);
      const uint4 msg[2] = {c0, c1};
      st.message_elems(tape, msg, 2);
      const uint4 r = st.sample_elem();
      chal[k] = r;
      cl = gf_add(c0, gf_mul_warp(r, gf_add(c1, gf_mul_warp(c2, r))));
      r_sh = r;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    st.store(ts);
    *claim = cl;
  }
}


}  // namespace

namespace bgpu {

int eq_tensor(const uint4* h_point, uint32_t n, uint4* d_out, cudaStream_t s) {
  if (n > 32) return set_error(BINIUS_E_ARG, "eq tensor: at most 32 coordinates");
  Point32 p;
  memset(&p, 0, sizeof(p));
  if (n) memcpy(p.r, h_point, 16 * (size_t)n);
  if (n <= 16) {
    BGPU_CUDA(launch_pdl(eq_small_kernel, grid_for(1ull << n, kThreads), kThreads, 0, s, d_out, p,
                         0u, n));
    count_launch();
    return BINIUS_OK;
  }
  const uint32_t k = n / 2;
  uint4* tmp = nullptr;
  const uint64_t nlo = 1ull << k, nhi = 1ull << (n - k);
  BGPU_CUDA(dev_alloc(&tmp, 16 * (nlo + nhi), s));
  cudaError_t e =
      launch_pdl(eq_small_kernel, grid_for(nlo, kThreads), kThreads, 0, s, tmp, p, 0u, k);
  if (e == cudaSuccess)
    e = launch_pdl(eq_small_kernel, grid_for(nhi, kThreads), kThreads, 0, s, tmp + nlo, p, k,
                   n - k);
  if (e == cudaSuccess)
    e = launch_pdl(eq_expand_kernel, grid_for(1ull << n, kThreads, 148 * 16), kThreads, 0, s,
                   d_out, (const uint4*)tmp, (const uint4*)(tmp + nlo), k, 1ull << n);
  dev_free(tmp, s);
  if (e != cudaSuccess) return cuda_error(e, "eq tensor kernels");
  count_launch(3);
  return BINIUS_OK;
}

int fold_1b_rows(const uint4* d_mat, const uint4* d_vec, uint64_t n, uint32_t* d_out512,
                 cudaStream_t s) {
  BGPU_CUDA(cudaMemsetAsync(d_out512, 0, 128 * 16, s));
  unsigned blocks = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>((n + kRowTile - 1) / kRowTile, 148 * 4));
  fold_rows_kernel<<<blocks, 128, 0, s>>>(d_mat, d_vec, n, d_out512);
  BGPU_LAUNCH_CHECK("fold_rows_kernel");
  count_launch();
  return BINIUS_OK;
}

int fold_b128_elems(const uint4* d_in, uint4* d_out, uint64_t n, const uint4* d_vec128,
                    cudaStream_t s) {
  uint4* tables = nullptr;
  BGPU_CUDA(dev_alloc(&tables, 16 * 16 * 256, s));
  build_fold_tables_kernel<<<16, 256, 0, s>>>(d_vec128, tables);
  const size_t smem = 16 * 256 * sizeof(uint4);
  cudaError_t e = ensure_smem_limit(reinterpret_cast<const void*>(fold_elems_kernel), smem)
                      ? cudaErrorInvalidValue
                      : cudaSuccess;
  if (e == cudaSuccess) {
    fold_elems_kernel<<<grid_for(n, kThreads, 148 * 2), kThreads, smem, s>>>(d_in, d_out, n, tables);
    e = cudaGetLastError();
  }
  dev_free(tables, s);
  if (e != cudaSuccess) return cuda_error(e, "fold_elems_kernel");
  count_launch(2);
  return BINIUS_OK;
}

int bivariate_eval(const uint4* d_a, const uint4* d_b, uint64_t half, uint32_t* d_out8,
                   cudaStream_t s) {
  BGPU_CUDA(cudaMemsetAsync(d_out8, 0, 32, s));
  bivariate_eval_kernel<<<grid_for(half, kThreads), kThreads, 0, s>>>(d_a, d_b, half, d_out8);
  BGPU_LAUNCH_CHECK("bivariate_eval_kernel");
  count_launch();
  return BINIUS_OK;
}

int bivariate_fold_eval(uint4* d_a, uint4* d_b, uint64_t size, const uint8_t r[16],
                        uint32_t* d_out8, cudaStream_t s) {
  if (size < 4) return set_error(BINIUS_E_ARG, "bivariate_fold_eval needs size >= 4");
  uint4 rv;
  memcpy(&rv, r, 16);
  BGPU_CUDA(cudaMemsetAsync(d_out8, 0, 32, s));
  const unsigned grid = grid_for(size / 2, kThreads);  // two lanes per folded position
  if (size >= kMulTableMinSize) {
    bivariate_fold_eval_kernel<<<grid, kThreads, 0, s>>>(d_a, d_b, size, rv, nullptr, d_out8);
    BGPU_LAUNCH_CHECK("bivariate_fold_eval_kernel");
    count_launch();
    return BINIUS_OK;
  }
  bivariate_fold_eval_lanes_kernel<<<grid_for(size, kThreads), kThreads, 0, s>>>(
      d_a, d_b, size, rv, nullptr, d_out8);
  BGPU_LAUNCH_CHECK("bivariate_fold_eval_lanes_kernel");
  count_launch();
  return BINIUS_OK;
}

int bivariate_fold_eval_dev(uint4* d_a, uint4* d_b, uint64_t size, const uint4* d_r,
                            uint32_t* d_out8, cudaStream_t s) {
  if (size < 4) return set_error(BINIUS_E_ARG, "bivariate_fold_eval needs size >= 4");
  const unsigned grid = grid_for(size / 2, kThreads);  // two lanes per folded position
  cudaError_t e;
  if (size >= kMulTableMinSize) {
    e = launch_pdl(bivariate_fold_eval_kernel, grid, kThreads, 0, s, d_a, d_b, size,
                   gf_zero_host(), d_r, d_out8);
  } else {
    e = launch_pdl(bivariate_fold_eval_lanes_kernel, grid_for(size, kThreads), kThreads, 0, s,
                   d_a, d_b, size, gf_zero_host(), d_r, d_out8);
  }
  if (e != cudaSuccess) return cuda_error(e, "bivariate_fold_eval_kernel");
  count_launch();
  return BINIUS_OK;
}

int bivariate_round_finish(const DeviceTranscript& dt, const uint4* d_ys, const uint4* d_claim_init,
                           uint4* d_claim, const uint8_t* d_commitment, uint4* d_r_out,
                           cudaStream_t s) {
  cudaError_t e = launch_pdl(bivariate_round_finish_kernel, 1, 32, 0, s, dt.state(), dt.tape(),
                             d_ys, d_claim_init, d_claim, d_commitment, d_r_out);
  if (e != cudaSuccess) return cuda_error(e, "bivariate_round_finish_kernel");
  count_launch();
  return BINIUS_OK;
}

int bivariate_tail(const DeviceTranscript& dt, uint4* d_a, uint4* d_b, uint64_t len,
                   uint32_t n_rounds, const uint4* d_r_first, uint4* d_claim, uint4* d_chal,
                   cudaStream_t s) {
  if (n_rounds == 0) return BINIUS_OK;
  if ((len >> (n_rounds - (d_r_first ? 0 : 1))) < 2)
    return set_error(BINIUS_E_ARG, "bivariate tail: more rounds than variables");
  cudaError_t e = launch_pdl(bivariate_tail_kernel, 1, kTailThreads, 0, s, dt.state(), dt.tape(),
                             d_a, d_b, len, n_rounds, d_r_first, d_claim, d_chal);
  if (e != cudaSuccess) return cuda_error(e, "bivariate_tail_kernel");
  count_launch();
  return BINIUS_OK;
}


}  // namespace bgpu

extern "C" {

int binius_bivariate_round_evals(const void* d_a, const void* d_b, uint32_t log_len,
                                 void* d_out2, void* stream) {
  BGPU_ARG(d_a && d_b && d_out2, "NULL argument");
  BGPU_ARG(log_len >= 1 && log_len <= 40, "log_len must be in [1, 40]");
  return bivariate_eval(static_cast<const uint4*>(d_a), static_cast<const uint4*>(d_b),
                        1ull << (log_len - 1), static_cast<uint32_t*>(d_out2), as_stream(stream))
             ? BINIUS_E_CUDA
             : clear_error();
}

int binius_bivariate_fold_round_evals(void* d_a, void* d_b, uint32_t log_len, const void* h_r,
                                      void* d_out2, void* stream) {
  BGPU_ARG(d_a && d_b && d_out2 && h_r, "NULL argument");
  BGPU_ARG(log_len >= 2 && log_len <= 40, "log_len must be in [2, 40]");
  return bivariate_fold_eval(static_cast<uint4*>(d_a), static_cast<uint4*>(d_b), 1ull << log_len,
                             static_cast<const uint8_t*>(h_r), static_cast<uint32_t*>(d_out2),
                             as_stream(stream))
             ? BINIUS_E_CUDA
             : clear_error();
}

}  // extern "C"
