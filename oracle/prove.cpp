// CPU oracle (test infrastructure only): the whole Prover::prove and a restated Verifier::verify.
//
// Restates:
//   Verifier::setup          verifier/verifier/src/verify.rs:61-108 (FRI parameters, 96-bit
//                            security, arity from estimate_optimal_arity, the standard-basis NTT
//                            domain of dim log_code_len), FRIParams::choose_with_constant_fold_arity
//                            (verifier/verifier/src/fri/common.rs:64-115)
//   Prover::prove            prover/prover/src/prove.rs:124-303: pack the witness, commit, IntMul
//                            reduction, AND reduction, the IntMul claims at the AND r_zhat', the
//                            shift reduction and the PCS opening at its point
//   Verifier::verify         verifier/verifier/src/verify.rs:143-282
#include <string.h>

#include <vector>

#include "oracle.h"
#include "protocols.h"
#include "transcript.h"

namespace orc {

namespace {

constexpr uint32_t kSecurityBits = 96;  // verify.rs:39

struct Setup {
  FriParams fri;
  std::vector<u128> tw;  // standard domain of dim log_code_len
};

uint32_t log2_ceil32(uint64_t n) {
  uint32_t r = 0;
  while ((1ull << r) < n) r++;
  return r;
}

Setup setup(uint32_t log_words, uint32_t log_inv_rate) {
  Setup s;
  const uint32_t log_witness_words = log_words < 1 ? 1 : log_words;
  const uint32_t log_witness_elems = log_witness_words - 1;
  const uint32_t log_code_len = log_witness_elems + log_inv_rate;
  const uint32_t arity = orc_estimate_optimal_arity(log_code_len, 32, 16);
  FriParams& p = s.fri;
  p.log_msg = log_witness_elems;
  p.log_batch = log_witness_elems < arity ? log_witness_elems : arity;
  p.log_inv_rate = log_inv_rate;
  p.n_queries = orc_calculate_n_test_queries(kSecurityBits, log_inv_rate);
  const uint32_t rs_log_len = p.log_msg - p.log_batch + log_inv_rate;
  uint32_t cap = ceil_log2(p.n_queries);
  uint32_t term = cap < log_inv_rate ? log_inv_rate : cap;
  if (term > rs_log_len) term = rs_log_len;
  const uint32_t q = (rs_log_len - term) / arity, rem = (rs_log_len - term) % arity;
  p.arities.assign(q, arity);
  if (rem) p.arities.push_back(rem);
  s.tw.resize(((size_t)1 << log_code_len) - 1);
  orc_domain_twiddles(nullptr, log_code_len, (uint64_t*)s.tw.data());
  return s;
}

// eval_operand over every constraint of a CSR list; out is slot-major (out[slot * n + i]).
std::vector<uint64_t> eval_ops(const uint64_t* words, const Ops& o) {
  std::vector<uint64_t> out((size_t)o.k * o.n, 0);
  parallel_for(o.n, [&](size_t c_lo, size_t c_hi) {  // constraints are independent
    for (size_t c = c_lo; c < c_hi; c++)
      for (uint32_t sl = 0; sl < o.k; sl++) {
        const uint32_t g = (uint32_t)c * o.k + sl;
        uint64_t acc = 0;
        for (uint32_t e = o.off[g]; e < o.off[g + 1]; e++)
          acc ^= shifted_word(words[o.vi[e]], o.var[e], o.amt[e]);
        out[(size_t)sl * o.n + c] = acc;
      }
  });
  return out;
}

u128 final_claim(const std::vector<u128>& evals, const u128 L[64]) {
  u128 acc = 0;
  for (int i = 0; i < 64; i++) acc ^= gf_mul(evals[i], L[i]);
  return acc;
}

void make_operator_data(const AndOutput& ao, const IntMulResult& im, OpData& band,
                        OpData& bmul) {
  band.evals = {ao.a_eval, ao.b_eval, ao.c_eval};
  band.r_zhat = ao.z;
  band.r_x = ao.eval_point;
  u128 L[64];
  l_tilde64(ao.z, L);
  bmul.evals = {final_claim(im.a_evals, L), final_claim(im.b_evals, L),
                final_claim(im.c_lo_evals, L), final_claim(im.c_hi_evals, L)};
  bmul.r_zhat = ao.z;
  bmul.r_x = im.eval_point;
}

}  // namespace

void prove(const uint64_t* words, uint32_t log_words, uint32_t log_public, const Ops& and_ops,
           const Ops& mul_ops, uint32_t log_inv_rate, Transcript& t) {
  Setup S = setup(log_words, log_inv_rate);
  const FriParams& p = S.fri;
  const u128* witness = (const u128*)words;  // pack_witness: word pairs as little-endian u128
  std::vector<u128> codeword((size_t)1 << p.log_len());
  rs_encode(S.tw.data(), witness, p.log_dim(), log_inv_rate, p.log_batch, codeword.data());
  Tree tree = build_tree(codeword.data(), p.rs_log_len(), p.log_batch);
  t.message(tree.root(), 32);

  std::vector<uint64_t> mul = eval_ops(words, mul_ops);  // slots a, b, hi, lo
  const size_t nm = mul_ops.n;
  IntMulResult im = intmul_prove(mul.data(), mul.data() + nm, mul.data() + 3 * nm,
                                 mul.data() + 2 * nm, log2_ceil32(nm), t);
  std::vector<uint64_t> abc = eval_ops(words, and_ops);
  const size_t na = and_ops.n;
  AndOutput ao = and_reduction_prove(abc.data(), abc.data() + na, abc.data() + 2 * na,
                                     log2_ceil32(na), t);
  OpData band, bmul;
  make_operator_data(ao, im, band, bmul);
  ShiftResult sh = shift_prove(words, log_words, log_public, and_ops, mul_ops, band, bmul, t);
  pcs_prove(p, S.tw.data(), codeword.data(), tree, witness, sh.challenges.data(), t);
}

int verify(const uint64_t* public_words, uint32_t log_words, uint32_t log_public,
           const Ops& and_ops, const Ops& mul_ops, uint32_t log_inv_rate, Transcript& t) {
  Setup S = setup(log_words, log_inv_rate);
  uint8_t root[32];
  if (!t.read_message(root, 32)) return 10;
  IntMulResult im;
  if (int rc = intmul_verify(log2_ceil32(mul_ops.n), t, im)) return 20 + rc;
  AndOutput ao;
  if (!and_reduction_verify(log2_ceil32(and_ops.n), t, ao)) return 30;
  OpData band, bmul;
  make_operator_data(ao, im, band, bmul);
  u128 witness_eval = 0;
  std::vector<u128> point;
  if (int rc = shift_verify(public_words, log_words, log_public, and_ops, mul_ops, band, bmul, t,
                            witness_eval, point))
    return 40 + rc;
  if (int rc = pcs_verify(S.fri, S.tw.data(), point.data(), witness_eval, root, t)) return 50 + rc;
  if (t.overrun) return 60;
  if (t.pos != t.tape.size()) return 61;
  return 0;
}

}  // namespace orc

using namespace orc;

namespace {
void make_ops(const uint32_t* const* csr, const uint8_t* var, uint32_t n, bool is_mul, Ops& o) {
  static const uint32_t and_map[3] = {0, 1, 2};
  static const uint32_t mul_map[4] = {0, 1, 3, 2};
  o = Ops{is_mul ? 4u : 3u, n, csr[0], csr[1], var, csr[2], is_mul ? mul_map : and_map};
}
}  // namespace

extern "C" {

// Setup of the FRI parameters for 2^log_words committed words: out6 = log_witness_elems,
// log_batch, n_queries, number of arities, then up to 8 arities in out_arities.
void orc_prove_params(uint32_t log_words, uint32_t log_inv_rate, uint32_t* out4,
                      uint32_t* out_arities) {
  Setup S = setup(log_words, log_inv_rate);
  out4[0] = S.fri.log_msg;
  out4[1] = S.fri.log_batch;
  out4[2] = S.fri.n_queries;
  out4[3] = (uint32_t)S.fri.arities.size();
  for (size_t i = 0; i < S.fri.arities.size() && i < 8; i++) out_arities[i] = S.fri.arities[i];
}

int orc_prove(const uint64_t* words, uint32_t log_words, uint32_t log_public,
              const uint32_t* const* and_csr, const uint8_t* and_var, uint32_t n_and,
              const uint32_t* const* mul_csr, const uint8_t* mul_var, uint32_t n_mul,
              uint32_t log_inv_rate, uint8_t* proof, size_t cap, size_t* len) {
  Ops ao, mo;
  make_ops(and_csr, and_var, n_and, false, ao);
  make_ops(mul_csr, mul_var, n_mul, true, mo);
  Transcript t;
  prove(words, log_words, log_public, ao, mo, log_inv_rate, t);
  *len = t.tape.size();
  if (t.tape.size() > cap) return 2;
  memcpy(proof, t.tape.data(), t.tape.size());
  return 0;
}

int orc_verify(const uint64_t* public_words, uint32_t log_words, uint32_t log_public,
               const uint32_t* const* and_csr, const uint8_t* and_var, uint32_t n_and,
               const uint32_t* const* mul_csr, const uint8_t* mul_var, uint32_t n_mul,
               uint32_t log_inv_rate, const uint8_t* proof, size_t len) {
  Ops ao, mo;
  make_ops(and_csr, and_var, n_and, false, ao);
  make_ops(mul_csr, mul_var, n_mul, true, mo);
  Transcript t;
  t.tape.assign(proof, proof + len);
  return verify(public_words, log_words, log_public, ao, mo, log_inv_rate, t);
}

}  // extern "C"
