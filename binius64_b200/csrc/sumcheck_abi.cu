// Round-by-round sumcheck provers behind the C ABI: the SumcheckProver trait
// (prover/prover/src/protocols/sumcheck/common.rs:29-101: execute -> RoundCoeffs, fold(challenge),
// finish -> multilinear evaluations) for the three provers of the prove path:
//
//   BivariateProductSumcheckProver (sumcheck/bivariate_product.rs:17-119): product of two
//     multilinears, high-to-low binding, degree-2 rounds from the evaluations at 1 and infinity
//     and the running sum (RoundEvals2::interpolate, round_evals.rs:70-77);
//   QuadraticMleCheckProver (sumcheck/quadratic_mle.rs:21-229) with the AND reduction's
//     composition a * b - c (infinity part a * b): evaluations weighted by the Gruen eq
//     expansion of the evaluation point's first n - 1 coordinates (gruen32.rs:29-131) and
//     interpolated by RoundEvals2::interpolate_eq (round_evals.rs:80-86);
//   InOutCheckProver (protocols/inout_check.rs:19-221): the witness against the public
//     input/output segment, degree-1 rounds, the evaluation point zero-padded above log_public.
//
// The multilinears stay in the caller's device buffers and are folded there
// (fold_highest_var_inplace, verifier/math/src/multilinear/fold.rs:14-29: a[i] += r (a[i + h] -
// a[i])); the eq expansion and the sums live in the prover object's own device memory.  Round
// sums come from the prove path's own evaluation kernels (bivariate_eval, and_mle_eval); each
// execute reads two field elements back and interpolates on the host.  Calls out of order return
// BINIUS_E_ARG with the reference's error names (ExpectedFold / ExpectedExecute,
// sumcheck/error.rs).
#include <string.h>

#include <algorithm>
#include <vector>

#include "gf128.cuh"
#include "gf_reduce.cuh"
#include "internal.h"
#include "kernels.h"

using namespace bgpu;

namespace {

constexpr int kThreads = 256;

unsigned blocks_for(uint64_t n) {
  const uint64_t g = (n + kThreads - 1) / kThreads;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, 148 * 8));
}

// Folds up to three columns of length 2 * half by r in place (null columns are skipped).
__global__ void __launch_bounds__(kThreads)
    fold_high_kernel(uint4* __restrict__ a, uint4* __restrict__ b, uint4* __restrict__ c,
                     uint64_t half, uint4 r) {
  uint4* cols[3] = {a, b, c};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < half;
       i += (uint64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      uint4* col = cols[k];
      if (!col) continue;
      const uint4 lo = col[i], hi = col[half + i];
      col[i] = gf_add(lo, gf_mul(r, gf_add(hi, lo)));
    }
  }
}

// eq_ind_truncate_low_inplace by one variable (verifier/math/src/multilinear/eq.rs:139-163):
// eq'[j] = eq[j] + eq[j + q], since eq(r, 0) + eq(r, 1) = 1.
__global__ void eq_truncate_kernel(uint4* __restrict__ eq, uint64_t q) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < q;
       j += (uint64_t)gridDim.x * blockDim.x)
    eq[j] = gf_add(eq[j], eq[q + j]);
}

// out[0..4) ^= sum_i x[i] * y[i] (inner_product_buffers), accumulated unreduced per thread.
__global__ void __launch_bounds__(kThreads)
    inner_product_kernel(const uint4* __restrict__ x, const uint4* __restrict__ y, uint64_t n,
                         uint32_t* __restrict__ out) {
  u256 acc = {0, 0, 0, 0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    xor_into(acc, clmul128(__ldg(x + i), __ldg(y + i)));
  uint4 v[1] = {reduce256(acc)};
  block_xor_reduce<1>(v, out);
}

enum Kind { kBivariate = 0, kQuadraticMle = 1, kInOut = 2 };

hu128 h128(const void* p) {
  hu128 v;
  memcpy(&v, p, 16);
  return v;
}

void put128(void* dst, hu128 v) { memcpy(dst, &v, 16); }

hu128 eval_poly(const std::vector<hu128>& c, hu128 x) {  // RoundCoeffs::evaluate (Horner)
  hu128 acc = 0;
  for (size_t i = c.size(); i-- > 0;) acc = host_gf_mul(acc, x) ^ c[i];
  return acc;
}

hu128 inv_or_zero(hu128 a) { return a ? host_gf_inv(a) : 0; }

}  // namespace

struct binius_sumcheck {
  int kind = kBivariate;
  cudaStream_t s = nullptr;
  uint4* cols[3] = {nullptr, nullptr, nullptr};
  uint32_t n_vars = 0;          // variables of the multilinears still free
  std::vector<hu128> point;     // MLE-checks: the evaluation point (InOut: zero-padded)
  uint32_t log_public = 0;      // InOut: m
  uint32_t gruen_vars = 0;      // variables of the Gruen eq expansion's point still free
  uint4* eq = nullptr;          // 2^(gruen_vars - 1) elements
  uint32_t* acc = nullptr;      // 2 x 4 words of round sums
  bool have_coeffs = false;
  std::vector<hu128> coeffs;    // the last execute's RoundCoeffs
  hu128 last = 0;               // the running sum / evaluation claim
};

namespace {

// sumcheck/error.rs: ExpectedFold when a fold is due, ExpectedExecute when an execute is due.
int state_error(const binius_sumcheck* p) {
  return set_error(BINIUS_E_ARG, p->have_coeffs ? "ExpectedFold" : "ExpectedExecute");
}

int read_two(const binius_sumcheck* p, hu128& y0, hu128& y1) {
  uint8_t buf[32];
  if (int rc = read_sync(buf, p->acc, 32, p->s)) return rc;
  y0 = h128(buf);
  y1 = h128(buf + 16);
  return BINIUS_OK;
}

// <x, y> over n elements, read back.
int inner_product(const binius_sumcheck* p, const uint4* x, const uint4* y, uint64_t n,
                  hu128& out) {
  BGPU_CUDA(cudaMemsetAsync(p->acc, 0, 16, p->s));
  inner_product_kernel<<<blocks_for(n), kThreads, 0, p->s>>>(x, y, n, p->acc);
  BGPU_LAUNCH_CHECK("inner_product_kernel");
  count_launch();
  uint8_t buf[16];
  if (int rc = read_sync(buf, p->acc, 16, p->s)) return rc;
  out = h128(buf);
  return BINIUS_OK;
}

// Gruen32 evaluate_multilinear_with_gruen32 (inout_check.rs:104-126): the multilinear x of
// 2^gruen_vars values at the full evaluation point, from its halves' inner products with the
// eq expansion, extrapolated along the last coordinate.
int eval_with_gruen(const binius_sumcheck* p, const uint4* x, hu128& out) {
  if (p->gruen_vars == 0) return read_sync(&out, x, 16, p->s);
  const uint64_t h = 1ull << (p->gruen_vars - 1);
  hu128 lo = 0, hi = 0;
  if (int rc = inner_product(p, x, p->eq, h, lo)) return rc;
  if (int rc = inner_product(p, x + h, p->eq, h, hi)) return rc;
  const hu128 alpha = p->point[p->gruen_vars - 1];
  out = lo ^ host_gf_mul(alpha, lo ^ hi);  // extrapolate_line(lo, hi, alpha)
  return BINIUS_OK;
}

int make(int kind, uint32_t n_vars, void* stream, binius_sumcheck** out) {
  binius_sumcheck* p = new binius_sumcheck();
  p->kind = kind;
  p->s = as_stream(stream);
  p->n_vars = n_vars;
  cudaError_t e = cudaMalloc(&p->acc, 32);
  if (e != cudaSuccess) {
    delete p;
    return cuda_error(e, "sumcheck round sums");
  }
  *out = p;
  return BINIUS_OK;
}

int build_eq(binius_sumcheck* p) {
  const uint32_t n = p->gruen_vars ? p->gruen_vars - 1 : 0;
  BGPU_ARG(n <= 32, "evaluation point longer than 33 coordinates");
  BGPU_CUDA(cudaMalloc(&p->eq, 16ull << n));
  std::vector<uint4> pt(n);
  for (uint32_t i = 0; i < n; i++) memcpy(&pt[i], &p->point[i], 16);
  return eq_tensor(pt.data(), n, p->eq, p->s);
}

int do_execute(binius_sumcheck* p, int kind, void* h_coeffs, uint32_t* n_coeffs) {
  BGPU_ARG(p && h_coeffs, "NULL argument");
  BGPU_ARG(p->kind == kind, "prover of another kind");
  if (p->have_coeffs) return state_error(p);
  BGPU_ARG(p->n_vars > 0, "no variables left: call finish");
  const uint64_t half = 1ull << (p->n_vars - 1);
  std::vector<hu128> c;
  if (kind == kBivariate) {
    if (int rc = bivariate_eval(p->cols[0], p->cols[1], half, p->acc, p->s)) return rc;
    hu128 y1, yinf;
    if (int rc = read_two(p, y1, yinf)) return rc;
    const hu128 y0 = p->last ^ y1;  // RoundEvals2::interpolate
    c = {y0, y1 ^ y0 ^ yinf, yinf};
  } else if (kind == kQuadraticMle) {
    if (int rc = and_mle_eval(p->cols[0], p->cols[1], p->cols[2], p->eq, half, p->acc, p->s))
      return rc;
    hu128 y1, yinf;
    if (int rc = read_two(p, y1, yinf)) return rc;
    const hu128 alpha = p->point[p->gruen_vars - 1];
    const hu128 y0 = host_gf_mul(p->last ^ host_gf_mul(y1, alpha), inv_or_zero(1 ^ alpha));
    c = {y0, y1 ^ y0 ^ yinf, yinf};
  } else {
    hu128 y0, y1;
    if (p->log_public < p->n_vars) {
      // early rounds: the point's coordinate is 0; the first 2^m values of the upper half
      if (int rc = eval_with_gruen(p, p->cols[0] + half, y1)) return rc;
      y0 = p->last;
    } else {
      // later rounds: witness and eq expansion have the same variables
      if (int rc = inner_product(p, p->cols[0] + half, p->eq, half, y1)) return rc;
      const hu128 alpha = p->point[p->gruen_vars - 1];
      y0 = host_gf_mul(p->last ^ host_gf_mul(y1, alpha), inv_or_zero(1 ^ alpha));
    }
    c = {y0, y1 ^ y0};
  }
  for (size_t i = 0; i < c.size(); i++) put128(static_cast<uint8_t*>(h_coeffs) + 16 * i, c[i]);
  if (n_coeffs) *n_coeffs = (uint32_t)c.size();
  p->coeffs = c;
  p->have_coeffs = true;
  return clear_error();
}

int do_fold(binius_sumcheck* p, int kind, const void* h_challenge) {
  BGPU_ARG(p && h_challenge, "NULL argument");
  BGPU_ARG(p->kind == kind, "prover of another kind");
  if (!p->have_coeffs) return state_error(p);
  const hu128 r = h128(h_challenge);
  const uint64_t half = 1ull << (p->n_vars - 1);
  uint4 rv;
  memcpy(&rv, &r, 16);
  fold_high_kernel<<<blocks_for(half), kThreads, 0, p->s>>>(p->cols[0], p->cols[1], p->cols[2],
                                                            half, rv);
  BGPU_LAUNCH_CHECK("fold_high_kernel");
  count_launch();
  const bool gruen_fold = kind == kQuadraticMle || (kind == kInOut && p->n_vars <= p->log_public);
  if (gruen_fold) {  // Gruen32::fold: drop the eq expansion's highest variable
    if (p->gruen_vars >= 2) {
      const uint64_t q = 1ull << (p->gruen_vars - 2);
      eq_truncate_kernel<<<blocks_for(q), kThreads, 0, p->s>>>(p->eq, q);
      BGPU_LAUNCH_CHECK("eq_truncate_kernel");
      count_launch();
    }
    p->gruen_vars--;
  }
  p->last = eval_poly(p->coeffs, r);
  p->have_coeffs = false;
  p->n_vars--;
  return clear_error();
}

int do_finish(binius_sumcheck* p, int kind, void* h_evals) {
  BGPU_ARG(p && h_evals, "NULL argument");
  BGPU_ARG(p->kind == kind, "prover of another kind");
  if (p->n_vars > 0) return state_error(p);
  StagedReads rd(p->s);
  const int n = kind == kBivariate ? 2 : kind == kQuadraticMle ? 3 : 1;
  for (int i = 0; i < n; i++)
    if (int rc = rd.add(static_cast<uint8_t*>(h_evals) + 16 * i, p->cols[i], 16)) return rc;
  if (int rc = rd.wait()) return rc;
  return clear_error();
}

int eval_point_out(const binius_sumcheck* p, int kind, void* h_out) {
  BGPU_ARG(p && h_out, "NULL argument");
  BGPU_ARG(p->kind == kind, "prover of another kind");
  // MleCheckProver::eval_point: the first n_vars coordinates still to bind
  for (uint32_t i = 0; i < p->n_vars; i++)
    put128(static_cast<uint8_t*>(h_out) + 16 * i, p->point[i]);
  return clear_error();
}

}  // namespace

extern "C" {

int binius_sumcheck_bivariate_create(void* d_a, void* d_b, uint32_t log_len, const void* h_sum,
                                     void* stream, binius_sumcheck** out) {
  BGPU_ARG(d_a && d_b && h_sum && out, "NULL argument");
  *out = nullptr;
  BGPU_ARG(log_len <= 40, "log_len must be <= 40");
  binius_sumcheck* p = nullptr;
  if (int rc = make(kBivariate, log_len, stream, &p)) return rc;
  p->cols[0] = static_cast<uint4*>(d_a);
  p->cols[1] = static_cast<uint4*>(d_b);
  p->last = h128(h_sum);
  *out = p;
  return clear_error();
}

int binius_sumcheck_quadratic_mle_create(void* d_a, void* d_b, void* d_c, uint32_t n_vars,
                                         const void* h_eval_point, const void* h_eval_claim,
                                         void* stream, binius_sumcheck** out) {
  BGPU_ARG(d_a && d_b && d_c && out && h_eval_claim && (h_eval_point || n_vars == 0),
           "NULL argument");
  *out = nullptr;
  BGPU_ARG(n_vars <= 33, "n_vars must be <= 33");
  binius_sumcheck* p = nullptr;
  if (int rc = make(kQuadraticMle, n_vars, stream, &p)) return rc;
  p->cols[0] = static_cast<uint4*>(d_a);
  p->cols[1] = static_cast<uint4*>(d_b);
  p->cols[2] = static_cast<uint4*>(d_c);
  for (uint32_t i = 0; i < n_vars; i++)
    p->point.push_back(h128(static_cast<const uint8_t*>(h_eval_point) + 16 * i));
  p->gruen_vars = n_vars;
  p->last = h128(h_eval_claim);
  if (int rc = build_eq(p)) {
    binius_sumcheck_destroy(p);
    return rc;
  }
  *out = p;
  return clear_error();
}

int binius_sumcheck_inout_create(void* d_witness, uint32_t log_len, const void* h_eval_point,
                                 uint32_t log_public, void* stream, binius_sumcheck** out) {
  BGPU_ARG(d_witness && out && (h_eval_point || log_public == 0), "NULL argument");
  *out = nullptr;
  BGPU_ARG(log_public <= log_len, "eval_point.len() must be <= witness.log_len()");
  BGPU_ARG(log_len <= 40 && log_public <= 33, "sizes out of range");
  binius_sumcheck* p = nullptr;
  if (int rc = make(kInOut, log_len, stream, &p)) return rc;
  p->cols[0] = static_cast<uint4*>(d_witness);
  p->log_public = log_public;
  for (uint32_t i = 0; i < log_len; i++)
    p->point.push_back(i < log_public ? h128(static_cast<const uint8_t*>(h_eval_point) + 16 * i)
                                      : (hu128)0);
  p->gruen_vars = log_public;
  int rc = build_eq(p);
  // InOutCheckProver::new: the claim is the public segment's evaluation at the point
  if (!rc) rc = eval_with_gruen(p, p->cols[0], p->last);
  if (rc) {
    binius_sumcheck_destroy(p);
    return rc;
  }
  *out = p;
  return clear_error();
}

int binius_sumcheck_destroy(binius_sumcheck* p) {
  if (!p) return BINIUS_OK;
  if (p->s) cudaStreamSynchronize(p->s);
  if (p->eq) cudaFree(p->eq);
  if (p->acc) cudaFree(p->acc);
  delete p;
  return BINIUS_OK;
}

uint32_t binius_sumcheck_n_vars(const binius_sumcheck* p) { return p ? p->n_vars : 0; }

int binius_sumcheck_bivariate_execute(binius_sumcheck* p, void* h_coeffs, uint32_t* n_coeffs) {
  return do_execute(p, kBivariate, h_coeffs, n_coeffs);
}
int binius_sumcheck_bivariate_fold(binius_sumcheck* p, const void* h_challenge) {
  return do_fold(p, kBivariate, h_challenge);
}
int binius_sumcheck_bivariate_finish(binius_sumcheck* p, void* h_evals2) {
  return do_finish(p, kBivariate, h_evals2);
}

int binius_sumcheck_quadratic_mle_execute(binius_sumcheck* p, void* h_coeffs,
                                          uint32_t* n_coeffs) {
  return do_execute(p, kQuadraticMle, h_coeffs, n_coeffs);
}
int binius_sumcheck_quadratic_mle_fold(binius_sumcheck* p, const void* h_challenge) {
  return do_fold(p, kQuadraticMle, h_challenge);
}
int binius_sumcheck_quadratic_mle_finish(binius_sumcheck* p, void* h_evals3) {
  return do_finish(p, kQuadraticMle, h_evals3);
}
int binius_sumcheck_quadratic_mle_eval_point(const binius_sumcheck* p, void* h_out) {
  return eval_point_out(p, kQuadraticMle, h_out);
}

int binius_sumcheck_inout_execute(binius_sumcheck* p, void* h_coeffs, uint32_t* n_coeffs) {
  return do_execute(p, kInOut, h_coeffs, n_coeffs);
}
int binius_sumcheck_inout_fold(binius_sumcheck* p, const void* h_challenge) {
  return do_fold(p, kInOut, h_challenge);
}
int binius_sumcheck_inout_finish(binius_sumcheck* p, void* h_eval) {
  return do_finish(p, kInOut, h_eval);
}
int binius_sumcheck_inout_eval_point(const binius_sumcheck* p, void* h_out) {
  return eval_point_out(p, kInOut, h_out);
}

}  // extern "C"
