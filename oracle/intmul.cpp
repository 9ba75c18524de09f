// CPU oracle (test infrastructure only): the integer multiplication reduction, prover and a
// restated verifier.
//
// Restates:
//   witness trees            prover/prover/src/protocols/intmul/witness.rs:47-270
//   IntMulProver::prove      prover/prover/src/protocols/intmul/prove.rs:93-509
//   common helpers           verifier/verifier/src/protocols/intmul/common.rs:81-138
//   sumcheck provers         prover/prover/src/protocols/sumcheck/{bivariate_product_multi_mle.rs,
//                            selector_mle.rs, rerand_mle.rs, mle_to_sumcheck.rs, gruen32.rs,
//                            round_evals.rs, batch.rs}
//   verifier                 verifier/verifier/src/protocols/intmul/verify.rs:30-413
// The multiplicative generator of GF(2^128) (GHASH) is the field's MULTIPLICATIVE_GENERATOR
// constant (verifier/field/src/ghash.rs:502).
#include <string.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "oracle.h"
#include "oracle_internal.h"
#include "protocols.h"
#include "transcript.h"

namespace orc {

namespace {

typedef std::vector<u128> Vec;

const u128 kGen = ((u128)0x494ef99794d5244fULL << 64) | (u128)0x9152df59d87a9186ULL;

u128 sq_n(u128 x, int n) {
  for (int i = 0; i < n; i++) x = gf_square(x);
  return x;
}

Vec eq_vec(const u128* point, uint32_t n) {
  Vec out((size_t)1 << n);
  eq_ind_partial_eval(point, n, out.data());
  return out;
}

u128 eval_univariate(const Vec& c, u128 x) {
  u128 acc = 0;
  for (size_t i = c.size(); i-- > 0;) acc = gf_mul(acc, x) ^ c[i];
  return acc;
}

u128 mle(const Vec& v, const Vec& point) {
  Vec eq = eq_vec(point.data(), (uint32_t)point.size());
  u128 acc = 0;
  for (size_t i = 0; i < v.size(); i++) acc ^= gf_mul(v[i], eq[i]);
  return acc;
}

void fold_high(Vec& v, u128 r) {
  const size_t half = v.size() / 2;
  for (size_t i = 0; i < half; i++) v[i] ^= gf_mul(r, v[half + i] ^ v[i]);
  v.resize(half);
}

// RoundEvals2::interpolate_eq / RoundEvals1::interpolate_eq (round_evals.rs:23-27, 80-87).
Vec interp2_eq(u128 sum, u128 y1, u128 yinf, u128 alpha) {
  const u128 y0 = gf_mul(sum ^ gf_mul(y1, alpha), gf_inv(1 ^ alpha));
  return {y0, y1 ^ y0 ^ yinf, yinf};
}
Vec interp1_eq(u128 sum, u128 y1, u128 alpha) {
  const u128 y0 = gf_mul(sum ^ gf_mul(y1, alpha), gf_inv(1 ^ alpha));
  return {y0, y1 ^ y0};
}

// round_coeffs_by_eq (round_evals.rs:145-156) times a scalar.
Vec by_eq(const Vec& prime, u128 alpha, u128 scale) {
  Vec out(prime.size() + 1, 0);
  for (size_t i = 0; i < prime.size(); i++) {
    out[i] ^= gf_mul(prime[i], 1 ^ alpha);
    out[i + 1] ^= prime[i];
  }
  for (auto& c : out) c = gf_mul(c, scale);
  return out;
}

// Gruen32 (gruen32.rs): eq over the point minus its last remaining coordinate, and the prefix
// product of eq_one_var over the folded coordinates.
struct Gruen {
  Vec point;
  uint32_t n_rem;
  u128 prefix = 1;
  explicit Gruen(const Vec& p) : point(p), n_rem((uint32_t)p.size()) {}
  u128 alpha() const { return point[n_rem - 1]; }
  Vec eq() const { return eq_vec(point.data(), n_rem - 1); }
  void fold(u128 r) {
    prefix = gf_mul(prefix, 1 ^ r ^ alpha());
    n_rem--;
  }
};

struct SumcheckProver {
  virtual ~SumcheckProver() {}
  virtual uint32_t n_vars() const = 0;
  virtual std::vector<Vec> execute() = 0;
  virtual void fold(u128 r) = 0;
  virtual Vec finish() = 0;
};

struct MleCheckProver : SumcheckProver {
  virtual u128 alpha() const = 0;  // eval_point()[n_vars - 1]
};

// BivariateProductMultiMlecheckProver (bivariate_product_multi_mle.rs:15-165).
struct BivMulti : MleCheckProver {
  std::vector<Vec> ml;  // pairs flattened
  Gruen gr;
  Vec sums;
  std::vector<Vec> prime;
  BivMulti(std::vector<Vec> m, const Vec& point, Vec claims)
      : ml(std::move(m)), gr(point), sums(std::move(claims)) {}
  uint32_t n_vars() const override { return gr.n_rem; }
  u128 alpha() const override { return gr.alpha(); }
  std::vector<Vec> execute() override {
    const Vec eq = gr.eq();
    const size_t half = eq.size();
    prime.clear();
    for (size_t p = 0; p < sums.size(); p++) {
      const Vec& a = ml[2 * p];
      const Vec& b = ml[2 * p + 1];
      u128 y1 = 0, yinf = 0;
      for (size_t i = 0; i < half; i++) {
        y1 ^= gf_mul(eq[i], gf_mul(a[half + i], b[half + i]));
        yinf ^= gf_mul(eq[i], gf_mul(a[i] ^ a[half + i], b[i] ^ b[half + i]));
      }
      prime.push_back(interp2_eq(sums[p], y1, yinf, gr.alpha()));
    }
    return prime;
  }
  void fold(u128 r) override {
    for (size_t p = 0; p < sums.size(); p++) sums[p] = eval_univariate(prime[p], r);
    for (auto& m : ml) fold_high(m, r);
    gr.fold(r);
  }
  Vec finish() override {
    Vec out;
    for (auto& m : ml) out.push_back(m[0]);
    return out;
  }
};

// RerandMlecheckProver (rerand_mle.rs): claims on the bit columns 0..n_claims of `bits`.
struct Rerand : MleCheckProver {
  std::vector<Vec> cols;
  Gruen gr;
  Vec sums;
  std::vector<Vec> prime;
  Rerand(const Vec& point, Vec claims, const uint64_t* bits)
      : gr(point), sums(std::move(claims)) {
    const size_t n = (size_t)1 << point.size();
    for (size_t k = 0; k < sums.size(); k++) {
      Vec c(n);
      for (size_t x = 0; x < n; x++) c[x] = (bits[x] >> k) & 1;
      cols.push_back(std::move(c));
    }
  }
  uint32_t n_vars() const override { return gr.n_rem; }
  u128 alpha() const override { return gr.alpha(); }
  std::vector<Vec> execute() override {
    const Vec eq = gr.eq();
    const size_t half = eq.size();
    prime.clear();
    for (size_t k = 0; k < sums.size(); k++) {
      u128 y1 = 0;
      for (size_t i = 0; i < half; i++) y1 ^= gf_mul(eq[i], cols[k][half + i]);
      prime.push_back(interp1_eq(sums[k], y1, gr.alpha()));
    }
    return prime;
  }
  void fold(u128 r) override {
    for (size_t k = 0; k < sums.size(); k++) sums[k] = eval_univariate(prime[k], r);
    for (auto& c : cols) fold_high(c, r);
    gr.fold(r);
  }
  Vec finish() override {
    Vec out;
    for (auto& c : cols) out.push_back(c[0]);
    return out;
  }
};

// MleToSumCheckDecorator (mle_to_sumcheck.rs:28-77).
struct Decorator : SumcheckProver {
  std::unique_ptr<MleCheckProver> inner;
  u128 prefix = 1;
  explicit Decorator(MleCheckProver* p) : inner(p) {}
  uint32_t n_vars() const override { return inner->n_vars(); }
  std::vector<Vec> execute() override {
    std::vector<Vec> out;
    const u128 a = inner->alpha();
    for (auto& pr : inner->execute()) out.push_back(by_eq(pr, a, prefix));
    return out;
  }
  void fold(u128 r) override {
    prefix = gf_mul(prefix, 1 ^ r ^ inner->alpha());
    inner->fold(r);
  }
  Vec finish() override { return inner->finish(); }
};

// SelectorMlecheckProver (selector_mle.rs): claims on sel_k * (selected - 1) + 1 for the bit
// columns k of `bits`, each at its own point; itself a sumcheck prover (Gruen32::interpolate2).
struct Selector : SumcheckProver {
  Vec selected;
  std::vector<Vec> cols;
  std::vector<Gruen> grs;
  Vec sums;
  std::vector<Vec> prime;
  Selector(Vec sel, const std::vector<Vec>& points, Vec claims, const uint64_t* bits)
      : selected(std::move(sel)), sums(std::move(claims)) {
    const size_t n = selected.size();
    for (size_t k = 0; k < sums.size(); k++) {
      Vec c(n);
      for (size_t x = 0; x < n; x++) c[x] = (bits[x] >> k) & 1;
      cols.push_back(std::move(c));
      grs.emplace_back(points[k]);
    }
  }
  uint32_t n_vars() const override { return grs[0].n_rem; }
  std::vector<Vec> execute() override {
    const size_t half = selected.size() / 2;
    std::vector<Vec> out;
    prime.clear();
    for (size_t k = 0; k < sums.size(); k++) {
      const Vec eq = grs[k].eq();
      const Vec& s = cols[k];
      u128 y1 = 0, yinf = 0;
      for (size_t i = 0; i < half; i++) {
        y1 ^= gf_mul(eq[i], gf_mul(s[half + i], selected[half + i] ^ 1) ^ 1);
        yinf ^= gf_mul(eq[i], gf_mul(s[i] ^ s[half + i], selected[i] ^ selected[half + i]));
      }
      const u128 a = grs[k].alpha();
      prime.push_back(interp2_eq(sums[k], y1, yinf, a));
      out.push_back(by_eq(prime.back(), a, grs[k].prefix));
    }
    return out;
  }
  void fold(u128 r) override {
    for (size_t k = 0; k < sums.size(); k++) sums[k] = eval_univariate(prime[k], r);
    for (auto& g : grs) g.fold(r);
    for (auto& c : cols) fold_high(c, r);
    fold_high(selected, r);
  }
  Vec finish() override {
    Vec out;
    for (auto& c : cols) out.push_back(c[0]);
    out.push_back(selected[0]);
    return out;
  }
};

struct BatchOut {
  Vec challenges;            // reversed
  std::vector<Vec> evals;    // per prover
};

// batch_prove_and_write_evals (batch.rs:41-135).
BatchOut batch_prove(std::vector<std::unique_ptr<SumcheckProver>>& provers, Transcript& t) {
  BatchOut out;
  const uint32_t n = provers[0]->n_vars();
  const u128 beta = t.sample();
  for (uint32_t round = 0; round < n; round++) {
    std::vector<Vec> all;
    for (auto& p : provers)
      for (auto& c : p->execute()) all.push_back(std::move(c));
    Vec acc;
    for (size_t i = all.size(); i-- > 0;) {
      for (auto& c : acc) c = gf_mul(c, beta);
      if (acc.size() < all[i].size()) acc.resize(all[i].size(), 0);
      for (size_t k = 0; k < all[i].size(); k++) acc[k] ^= all[i][k];
    }
    acc.pop_back();
    t.message_elems(acc.data(), acc.size());
    const u128 r = t.sample();
    out.challenges.push_back(r);
    for (auto& p : provers) p->fold(r);
  }
  std::reverse(out.challenges.begin(), out.challenges.end());
  for (auto& p : provers) {
    Vec e = p->finish();
    t.message_elems(e.data(), e.size());
    out.evals.push_back(std::move(e));
  }
  return out;
}

std::unique_ptr<SumcheckProver> decorated(MleCheckProver* p) {
  return std::unique_ptr<SumcheckProver>(new Decorator(p));
}

// BinaryTree layers, root first: layers[k] holds 2^k multilinears of n values.
typedef std::vector<std::vector<Vec>> Layers;

Layers build_layers(std::vector<Vec> leaves) {
  Layers t;
  t.push_back(std::move(leaves));
  while (t.back().size() > 1) {
    const auto& cur = t.back();
    std::vector<Vec> next;
    for (size_t j = 0; j < cur.size() / 2; j++) {
      Vec prod(cur[0].size());
      for (size_t x = 0; x < prod.size(); x++) prod[x] = gf_mul(cur[2 * j][x], cur[2 * j + 1][x]);
      next.push_back(std::move(prod));
    }
    t.push_back(std::move(next));
  }
  std::reverse(t.begin(), t.end());
  return t;
}

Layers constant_base(u128 base, const uint64_t* e, size_t n) {
  std::vector<Vec> leaves;
  u128 b = base;
  for (int i = 0; i < 64; i++, b = gf_square(b)) {
    Vec l(n);
    for (size_t x = 0; x < n; x++) l[x] = ((e[x] >> i) & 1) ? b : 1;
    leaves.push_back(std::move(l));
  }
  return build_layers(std::move(leaves));
}

Layers variable_base(Vec bases, const uint64_t* e, size_t n) {
  std::vector<Vec> leaves;
  for (int i = 0; i < 64; i++) {
    Vec l(n);
    for (size_t x = 0; x < n; x++) {
      l[x] = ((e[x] >> i) & 1) ? bases[x] : 1;
      bases[x] = gf_square(bases[x]);
    }
    leaves.push_back(std::move(l));
  }
  return build_layers(std::move(leaves));
}

std::vector<Vec> concat_layers(std::initializer_list<const std::vector<Vec>*> ls) {
  std::vector<Vec> out;
  for (auto* l : ls) out.insert(out.end(), l->begin(), l->end());
  return out;
}

}  // namespace


IntMulResult intmul_prove(const uint64_t* a, const uint64_t* b, const uint64_t* lo,
                          const uint64_t* hi, uint32_t n_vars, Transcript& t) {
  const size_t n = (size_t)1 << n_vars;
  const u128 g = kGen;
  const u128 g_hi = sq_n(g, 64);
  Layers ta = constant_base(g, a, n);
  Layers tlo = constant_base(g, lo, n);
  Layers thi = constant_base(g_hi, hi, n);
  Layers tb = variable_base(ta[0][0], b, n);
  Vec c_root(n);
  for (size_t x = 0; x < n; x++) c_root[x] = gf_mul(tlo[0][0][x], thi[0][0][x]);

  Vec point0(n_vars);
  for (auto& v : point0) v = t.sample();
  const u128 b_eval = mle(tb[0][0], point0), c_eval = mle(c_root, point0);
  u128 be[2] = {b_eval, c_eval};
  t.message_elems(be, 2);

  // phase 1
  Vec pt = point0, evals{b_eval};
  for (int depth = 0; depth < 6; depth++) {
    std::vector<std::unique_ptr<SumcheckProver>> ps;
    ps.push_back(decorated(new BivMulti(tb[depth + 1], pt, evals)));
    BatchOut o = batch_prove(ps, t);
    pt = o.challenges;
    evals = o.evals[0];
  }
  // phase 2: frobenius twist
  std::vector<Vec> tw_points;
  Vec tw_evals;
  for (int i = 0; i < 64; i++) {
    Vec p;
    for (u128 c : pt) p.push_back(sq_n(c, 128 - i));
    tw_points.push_back(std::move(p));
    tw_evals.push_back(sq_n(evals[i], 128 - i));
  }
  // phase 3
  Vec p3, b_exp_evals;
  u128 selector_eval, c_lo_root_eval, c_hi_root_eval;
  {
    std::vector<std::unique_ptr<SumcheckProver>> ps;
    ps.emplace_back(new Selector(ta[0][0], tw_points, tw_evals, b));
    ps.push_back(decorated(new BivMulti({tlo[0][0], thi[0][0]}, point0, {c_eval})));
    BatchOut o = batch_prove(ps, t);
    p3 = o.challenges;
    b_exp_evals.assign(o.evals[0].begin(), o.evals[0].begin() + 64);
    selector_eval = o.evals[0][64];
    c_lo_root_eval = o.evals[1][0];
    c_hi_root_eval = o.evals[1][1];
  }
  // phase 4
  pt = p3;
  evals = {selector_eval, c_lo_root_eval, c_hi_root_eval};
  for (int depth = 0; depth < 5; depth++) {
    std::vector<std::unique_ptr<SumcheckProver>> ps;
    ps.push_back(decorated(
        new BivMulti(concat_layers({&ta[depth + 1], &tlo[depth + 1], &thi[depth + 1]}), pt, evals)));
    BatchOut o = batch_prove(ps, t);
    pt = o.challenges;
    evals = o.evals[0];
  }
  // phase 5
  Vec a0(n), b0(n);
  for (size_t x = 0; x < n; x++) {
    a0[x] = a[x] & 1;
    b0[x] = b[x] & 1;
  }
  u128 c_lo_0_eval = 0;
  {
    Vec eq = eq_vec(pt.data(), n_vars);
    for (size_t x = 0; x < n; x++)
      if (lo[x] & 1) c_lo_0_eval ^= eq[x];
  }
  t.message_elems(&c_lo_0_eval, 1);
  IntMulResult res;
  {
    std::vector<Vec> ml = concat_layers({&ta[6], &tlo[6], &thi[6]});
    ml.push_back(a0);
    ml.push_back(b0);
    Vec claims = evals;
    claims.push_back(c_lo_0_eval);
    std::vector<std::unique_ptr<SumcheckProver>> ps;
    ps.push_back(decorated(new BivMulti(std::move(ml), pt, claims)));
    ps.push_back(decorated(new Rerand(pt, {c_lo_0_eval}, lo)));
    ps.push_back(decorated(new Rerand(p3, b_exp_evals, b)));
    BatchOut o = batch_prove(ps, t);
    res.eval_point = o.challenges;
    // normalize_a_c_exponent_evals
    Vec conj;
    u128 c = g;
    for (int i = 0; i < 128; i++, c = gf_square(c)) conj.push_back(c);
    for (int i = 0; i < 64; i++) {
      res.a_evals.push_back(gf_mul(o.evals[0][i] ^ 1, gf_inv(conj[i] ^ 1)));
      res.c_lo_evals.push_back(gf_mul(o.evals[0][64 + i] ^ 1, gf_inv(conj[i] ^ 1)));
      res.c_hi_evals.push_back(gf_mul(o.evals[0][128 + i] ^ 1, gf_inv(conj[64 + i] ^ 1)));
    }
    res.b_evals = o.evals[2];
  }
  return res;
}

// ---------------------------------------------------------------- restated verifier

namespace {

struct BatchVerifyOut {
  u128 beta;
  Vec challenges;  // reversed
  u128 eval;
};

// batch_verify (verifier/verifier/src/protocols/sumcheck/batch.rs) for degree 3.
BatchVerifyOut batch_verify(uint32_t n_vars, const Vec& claims, Transcript& t) {
  BatchVerifyOut o;
  o.beta = t.sample();
  u128 sum = eval_univariate(claims, o.beta);
  for (uint32_t i = 0; i < n_vars; i++) {
    u128 c[3];
    t.read_message((uint8_t*)c, 48);
    const u128 r = t.sample();
    const u128 c3 = sum ^ c[1] ^ c[2];
    sum = eval_univariate({c[0], c[1], c[2], c3}, r);
    o.challenges.push_back(r);
  }
  std::reverse(o.challenges.begin(), o.challenges.end());
  o.eval = sum;
  return o;
}

Vec read_elems(Transcript& t, size_t n) {
  Vec v(n);
  t.read_message((uint8_t*)v.data(), 16 * n);
  return v;
}

u128 eq_ind(const Vec& x, const Vec& y) {
  u128 acc = 1;
  for (size_t i = 0; i < x.size(); i++) acc = gf_mul(acc, 1 ^ x[i] ^ y[i]);
  return acc;
}

bool verify_layer(Vec& point, Vec& evals, Transcript& t) {
  BatchVerifyOut o = batch_verify((uint32_t)point.size(), evals, t);
  Vec ml = read_elems(t, 2 * evals.size());
  const u128 e = eq_ind(point, o.challenges);
  Vec terms;
  for (size_t i = 0; i < evals.size(); i++) terms.push_back(gf_mul(e, gf_mul(ml[2 * i], ml[2 * i + 1])));
  if (eval_univariate(terms, o.beta) != o.eval) return false;
  point = o.challenges;
  evals = ml;
  return true;
}

}  // namespace

// Returns 0 when accepted; fills the output claims like the prover.
int intmul_verify(uint32_t n_vars, Transcript& t, IntMulResult& res) {
  Vec point0(n_vars);
  for (auto& v : point0) v = t.sample();
  Vec be = read_elems(t, 2);
  const u128 c_eval = be[1];
  Vec pt = point0, evals{be[0]};
  for (int d = 0; d < 6; d++)
    if (!verify_layer(pt, evals, t)) return 1;
  std::vector<Vec> tw_points;
  Vec claims;
  for (int i = 0; i < 64; i++) {
    Vec p;
    for (u128 c : pt) p.push_back(sq_n(c, 128 - i));
    tw_points.push_back(std::move(p));
    claims.push_back(sq_n(evals[i], 128 - i));
  }
  claims.push_back(c_eval);
  BatchVerifyOut o3 = batch_verify(n_vars, claims, t);
  Vec sel = read_elems(t, 65), croot = read_elems(t, 2);
  {
    Vec terms;
    for (int i = 0; i < 64; i++)
      terms.push_back(gf_mul(eq_ind(tw_points[i], o3.challenges), gf_mul(sel[i], sel[64] ^ 1) ^ 1));
    terms.push_back(gf_mul(eq_ind(point0, o3.challenges), gf_mul(croot[0], croot[1])));
    if (eval_univariate(terms, o3.beta) != o3.eval) return 2;
  }
  const Vec p3 = o3.challenges;
  Vec b_exp(sel.begin(), sel.begin() + 64);
  pt = p3;
  evals = {sel[64], croot[0], croot[1]};
  for (int d = 0; d < 5; d++)
    if (!verify_layer(pt, evals, t)) return 3;
  const u128 ov = read_elems(t, 1)[0];
  Vec c5 = evals;
  c5.push_back(ov);
  c5.push_back(ov);
  c5.insert(c5.end(), b_exp.begin(), b_exp.end());
  BatchVerifyOut o5 = batch_verify(n_vars, c5, t);
  Vec biv = read_elems(t, 194);
  const u128 clo0 = read_elems(t, 1)[0];
  Vec bev = read_elems(t, 64);
  {
    const u128 e = eq_ind(pt, o5.challenges);
    Vec terms;
    for (int i = 0; i < 97; i++) terms.push_back(gf_mul(e, gf_mul(biv[2 * i], biv[2 * i + 1])));
    terms.push_back(gf_mul(e, clo0));
    const u128 eb = eq_ind(p3, o5.challenges);
    for (int i = 0; i < 64; i++) terms.push_back(gf_mul(eb, bev[i]));
    if (eval_univariate(terms, o5.beta) != o5.eval) return 4;
  }
  Vec conj;
  u128 c = kGen;
  for (int i = 0; i < 128; i++, c = gf_square(c)) conj.push_back(c);
  res = IntMulResult();
  res.eval_point = o5.challenges;
  for (int i = 0; i < 64; i++) {
    res.a_evals.push_back(gf_mul(biv[i] ^ 1, gf_inv(conj[i] ^ 1)));
    res.c_lo_evals.push_back(gf_mul(biv[64 + i] ^ 1, gf_inv(conj[i] ^ 1)));
    res.c_hi_evals.push_back(gf_mul(biv[128 + i] ^ 1, gf_inv(conj[64 + i] ^ 1)));
  }
  res.b_evals = bev;
  if (res.a_evals[0] != biv[192] || res.b_evals[0] != biv[193] || res.c_lo_evals[0] != clo0)
    return 5;
  if (t.overrun) return 6;
  return 0;
}

}  // namespace orc

using namespace orc;

namespace {
void store_result(const IntMulResult& r, uint64_t* out_point, uint64_t* out_evals) {
  for (size_t i = 0; i < r.eval_point.size(); i++) store(out_point + 2 * i, r.eval_point[i]);
  const std::vector<u128>* cols[4] = {&r.a_evals, &r.b_evals, &r.c_lo_evals, &r.c_hi_evals};
  for (int k = 0; k < 4; k++)
    for (int i = 0; i < 64; i++) store(out_evals + 2 * (64 * k + i), (*cols[k])[i]);
}
}  // namespace

extern "C" {

// IntMul reduction on a fresh transcript over 2^log_n statements a * b = hi:lo.
// out_point: log_n elements; out_evals: 4 x 64 elements (a, b, lo, hi bit-column evaluations).
int orc_intmul_prove(const uint64_t* a, const uint64_t* b, const uint64_t* lo, const uint64_t* hi,
                     uint32_t log_n, uint8_t* proof, size_t cap, size_t* len,
                     uint64_t* out_point, uint64_t* out_evals) {
  Transcript t;
  IntMulResult r = intmul_prove(a, b, lo, hi, log_n, t);
  *len = t.tape.size();
  if (t.tape.size() > cap) return 2;
  memcpy(proof, t.tape.data(), t.tape.size());
  store_result(r, out_point, out_evals);
  return 0;
}

int orc_intmul_verify(uint32_t log_n, const uint8_t* proof, size_t len, uint64_t* out_point,
                      uint64_t* out_evals) {
  Transcript t;
  t.tape.assign(proof, proof + len);
  IntMulResult r;
  int rc = intmul_verify(log_n, t, r);
  if (rc == 0 && t.pos != t.tape.size()) rc = 7;
  if (rc == 0) store_result(r, out_point, out_evals);
  return rc;
}

}  // extern "C"
