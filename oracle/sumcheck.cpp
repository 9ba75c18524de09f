// CPU oracle (test infrastructure only): the round-by-round sumcheck provers of the prove path,
// run over given challenges, so that the device's trait-level entry points can be compared round
// by round.
//
// Restates:
//   SumcheckProver {execute, fold, finish}  prover/prover/src/protocols/sumcheck/common.rs:29-101
//   BivariateProductSumcheckProver         sumcheck/bivariate_product.rs:17-119
//   QuadraticMleCheckProver (a*b - c)      sumcheck/quadratic_mle.rs:21-229, gruen32.rs:29-131
//   RoundEvals2::{interpolate, interpolate_eq}  sumcheck/round_evals.rs:58-142
//   InOutCheckProver                       protocols/inout_check.rs:19-221
//   fold_highest_var_inplace               verifier/math/src/multilinear/fold.rs:14-29
//   eq_ind_partial_eval / truncate_low     verifier/math/src/multilinear/eq.rs:39-163
#include <string.h>

#include <vector>

#include "oracle.h"
#include "oracle_internal.h"

namespace orc {
namespace {

typedef std::vector<u128> Vec;

Vec load_vec(const uint64_t* p, size_t n) {
  Vec v(n);
  for (size_t i = 0; i < n; i++) v[i] = load(p + 2 * i);
  return v;
}

// fold_highest_var_inplace: a[i] = a[i] + r (a[i + h] - a[i]), then keep the low half.
void fold_high(Vec& a, u128 r) {
  const size_t h = a.size() / 2;
  for (size_t i = 0; i < h; i++) a[i] ^= gf_mul(r, a[i] ^ a[h + i]);
  a.resize(h);
}

Vec eq_expand(const Vec& point, size_t n) {
  Vec out((size_t)1 << n);
  eq_ind_partial_eval(point.data(), (uint32_t)n, out.data());
  return out;
}

// eq_ind_truncate_low_inplace by one variable: the tensor over the first n - 1 coordinates.
void eq_truncate(Vec& eq) {
  const size_t q = eq.size() / 2;
  for (size_t j = 0; j < q; j++) eq[j] ^= eq[q + j];
  eq.resize(q);
}

u128 inner(const u128* x, const u128* y, size_t n) {
  u128 acc = 0;
  for (size_t i = 0; i < n; i++) acc ^= gf_mul(x[i], y[i]);
  return acc;
}

u128 eval_poly(const u128* c, int n, u128 x) {
  u128 acc = 0;
  for (int i = n - 1; i >= 0; i--) acc = gf_mul(acc, x) ^ c[i];
  return acc;
}

u128 inv_or_zero(u128 a) { return a ? gf_inv(a) : 0; }

// RoundEvals2::interpolate_eq: y_0 = (sum - y_1 alpha) / (1 - alpha).
void interpolate_eq(u128 sum, u128 y1, u128 yinf, u128 alpha, u128* c) {
  const u128 y0 = gf_mul(sum ^ gf_mul(y1, alpha), inv_or_zero(1 ^ alpha));
  c[0] = y0;
  c[1] = y1 ^ y0 ^ yinf;
  c[2] = yinf;
}

}  // namespace
}  // namespace orc

using namespace orc;

extern "C" {

// BivariateProductSumcheckProver over [a, b] of 2^n values with the given sum and n challenges:
// coeffs_out receives 3 coefficients per round, evals_out the two final values.
int orc_bivariate_rounds(const uint64_t* a_in, const uint64_t* b_in, uint32_t n,
                         const uint64_t* sum, const uint64_t* challenges, uint64_t* coeffs_out,
                         uint64_t* evals_out) {
  Vec a = load_vec(a_in, (size_t)1 << n), b = load_vec(b_in, (size_t)1 << n);
  u128 last = load(sum);
  for (uint32_t k = 0; k < n; k++) {
    const size_t h = a.size() / 2;
    u128 y1 = 0, yinf = 0;
    for (size_t i = 0; i < h; i++) {
      y1 ^= gf_mul(a[h + i], b[h + i]);
      yinf ^= gf_mul(a[i] ^ a[h + i], b[i] ^ b[h + i]);
    }
    const u128 y0 = last ^ y1;  // RoundEvals2::interpolate
    const u128 c[3] = {y0, y1 ^ y0 ^ yinf, yinf};
    for (int j = 0; j < 3; j++) store(coeffs_out + 2 * (3 * k + j), c[j]);
    const u128 r = load(challenges + 2 * k);
    last = eval_poly(c, 3, r);
    fold_high(a, r);
    fold_high(b, r);
  }
  store(evals_out, a[0]);
  store(evals_out + 2, b[0]);
  return 0;
}

// QuadraticMleCheckProver over [a, b, c] with composition a*b - c (infinity part a*b).
int orc_quadratic_mle_rounds(const uint64_t* a_in, const uint64_t* b_in, const uint64_t* c_in,
                             uint32_t n, const uint64_t* point_in, const uint64_t* claim,
                             const uint64_t* challenges, uint64_t* coeffs_out,
                             uint64_t* evals_out) {
  const size_t N = (size_t)1 << n;
  Vec cols[3] = {load_vec(a_in, N), load_vec(b_in, N), load_vec(c_in, N)};
  const Vec point = load_vec(point_in, n);
  Vec eq = eq_expand(point, n ? n - 1 : 0);
  u128 last = load(claim);
  for (uint32_t k = 0; k < n; k++) {
    const uint32_t rem = n - k;
    const size_t h = cols[0].size() / 2;
    u128 y1 = 0, yinf = 0;
    for (size_t i = 0; i < h; i++) {
      const u128 a0 = cols[0][i], a1 = cols[0][h + i], b0 = cols[1][i], b1 = cols[1][h + i];
      const u128 c1 = cols[2][h + i];
      y1 ^= gf_mul(eq[i], gf_mul(a1, b1) ^ c1);
      yinf ^= gf_mul(eq[i], gf_mul(a0 ^ a1, b0 ^ b1));
    }
    u128 c[3];
    interpolate_eq(last, y1, yinf, point[rem - 1], c);
    for (int j = 0; j < 3; j++) store(coeffs_out + 2 * (3 * k + j), c[j]);
    const u128 r = load(challenges + 2 * k);
    last = eval_poly(c, 3, r);
    for (auto& col : cols) fold_high(col, r);
    if (eq.size() > 1) eq_truncate(eq);
  }
  for (int j = 0; j < 3; j++) store(evals_out + 2 * j, cols[j][0]);
  return 0;
}

// InOutCheckProver over a witness of 2^n values against the first 2^m, at eval_point (m
// coordinates, zero-padded to n): coeffs_out receives 2 coefficients per round, eval_out the
// witness evaluation.
int orc_inout_rounds(const uint64_t* w_in, uint32_t n, const uint64_t* point_in, uint32_t m,
                     const uint64_t* challenges, uint64_t* coeffs_out, uint64_t* eval_out) {
  Vec w = load_vec(w_in, (size_t)1 << n);
  const Vec point = load_vec(point_in, m);
  uint32_t gv = m;  // Gruen32's variables still free
  Vec eq = eq_expand(point, m ? m - 1 : 0);
  // evaluate_multilinear_with_gruen32 over x (2^gv values)
  auto eval_gruen = [&](const u128* x) -> u128 {
    if (gv == 0) return x[0];
    const size_t h = (size_t)1 << (gv - 1);
    const u128 lo = inner(x, eq.data(), h), hi = inner(x + h, eq.data(), h);
    return lo ^ gf_mul(point[gv - 1], lo ^ hi);  // extrapolate_line
  };
  u128 last = eval_gruen(w.data());
  uint32_t vars = n;
  for (uint32_t k = 0; k < n; k++) {
    const size_t h = w.size() / 2;
    u128 y0, y1;
    if (m < vars) {
      y1 = eval_gruen(w.data() + h);
      y0 = last;
    } else {
      y1 = inner(w.data() + h, eq.data(), h);
      const u128 alpha = point[gv - 1];
      y0 = gf_mul(last ^ gf_mul(y1, alpha), inv_or_zero(1 ^ alpha));
    }
    const u128 c[2] = {y0, y1 ^ y0};
    store(coeffs_out + 2 * (2 * k), c[0]);
    store(coeffs_out + 2 * (2 * k + 1), c[1]);
    const u128 r = load(challenges + 2 * k);
    last = eval_poly(c, 2, r);
    fold_high(w, r);
    if (vars <= m) {
      if (eq.size() > 1) eq_truncate(eq);
      gv--;
    }
    vars--;
  }
  store(eval_out, w[0]);
  return 0;
}

}  // extern "C"
