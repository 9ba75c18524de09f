// CPU oracle (test infrastructure only): the Fiat-Shamir transcript and the FRI-Binius 1-bit
// multilinear polynomial commitment scheme (ring switching + BaseFold + FRI), prover and verifier.
//
// Restates:
//   transcript   verifier/transcript/src/fiat_shamir/hasher_challenger.rs:14-200,
//                verifier/transcript/src/transcript.rs:204-407, fiat_shamir/sampling.rs:34-50
//   PCS prover   prover/prover/src/pcs.rs:107-169, ring_switch.rs:130-265,
//                protocols/basefold.rs:69-166, protocols/sumcheck/bivariate_product.rs:43-95,
//                protocols/sumcheck/round_evals.rs:58-142, fri/fold.rs:117-244, fri/query.rs:51-134,
//                merkle_tree/prover.rs:67-81, merkle_tree/binary_merkle_tree.rs:142-169
//   PCS verifier verifier/verifier/src/pcs.rs:19-97, protocols/basefold.rs:16-67,
//                fri/fold.rs:132-278, fri/verify.rs:40-320, merkle_tree/scheme.rs:85-180
#include <string.h>

#include <mutex>
#include <vector>

#include "oracle.h"
#include "oracle_internal.h"
#include "protocols.h"
#include "transcript.h"

namespace orc {

// ---------------------------------------------------------------- FRI fold prover

struct FriFolder {
  const FriParams& p;
  const u128* tw;
  const u128* codeword;
  const Tree& codeword_tree;
  std::vector<std::vector<u128>> round_words;
  std::vector<Tree> round_trees;
  uint32_t curr_round = 0;
  int64_t next_commit_round;
  std::vector<u128> unprocessed;

  FriFolder(const FriParams& p_, const u128* tw_, const u128* cw, const Tree& tree)
      : p(p_), tw(tw_), codeword(cw), codeword_tree(tree), next_commit_round(p_.log_batch) {}

  // FRIFoldProver::execute_fold_round (prover/prover/src/fri/fold.rs:117-175)
  bool execute_fold_round(uint8_t root[32]) {
    if (next_commit_round < 0 || (int64_t)curr_round != next_commit_round) return false;
    std::vector<u128> folded;
    if (round_words.empty()) {
      folded.resize((size_t)1 << p.rs_log_len());
      fold_interleaved(codeword, p.rs_log_len(), p.log_batch, unprocessed.data(), folded.data());
    } else {
      const auto& prev = round_words.back();
      uint32_t log_prev = log2_exact(prev.size());
      folded.resize(prev.size() >> unprocessed.size());
      fold_codeword(tw, prev.data(), log_prev, unprocessed.data(), (uint32_t)unprocessed.size(),
                    folded.data());
    }
    unprocessed.clear();
    bool has_next = round_words.size() < p.arities.size();
    uint32_t next_arity = has_next ? p.arities[round_words.size()] : 0;
    uint32_t log_coset = has_next ? next_arity : p.n_final_challenges();
    uint32_t log_leaves = log2_exact(folded.size()) - log_coset;
    Tree t = build_tree(folded.data(), log_leaves, log_coset);
    memcpy(root, t.root(), 32);
    next_commit_round = has_next ? next_commit_round + next_arity : -1;
    round_words.push_back(std::move(folded));
    round_trees.push_back(std::move(t));
    return true;
  }

  void receive_challenge(u128 c) {
    unprocessed.push_back(c);
    curr_round++;
  }

  // prove_coset_opening (prover/prover/src/fri/query.rs:112-134)
  static void coset_opening(Transcript& t, const u128* word, const Tree& tree, size_t coset_index,
                            uint32_t log_coset, uint32_t depth) {
    t.decommit_elems(word + (coset_index << log_coset), (size_t)1 << log_coset);
    std::vector<uint8_t> br;
    tree.branch(coset_index, depth, br);
    t.decommit(br.data(), br.size());
  }

  // FRIFoldProver::finish_proof (fri/fold.rs:221-244) and FRIQueryProver (fri/query.rs:51-110)
  void finish_proof(Transcript& t) {
    if (round_words.empty())
      t.decommit_elems(codeword, (size_t)1 << p.log_len());
    else
      t.decommit_elems(round_words.back().data(), round_words.back().size());
    auto depths = p.optimal_depths();
    std::vector<const Tree*> trees{&codeword_tree};
    for (size_t i = 0; i + 1 < round_trees.size(); i++) trees.push_back(&round_trees[i]);
    for (size_t i = 0; i < trees.size() && i < depths.size(); i++)
      t.decommit(trees[i]->layer(depths[i]), 32 * ((size_t)1 << depths[i]));
    for (uint32_t q = 0; q < p.n_queries; q++) {
      size_t index = t.sample_bits(p.rs_log_len());
      coset_opening(t, codeword, codeword_tree, index, p.log_batch, depths[0]);
      for (size_t i = 0; i < round_words.size() && i < p.arities.size() && i + 1 < depths.size();
           i++) {
        index >>= p.arities[i];
        coset_opening(t, round_words[i].data(), round_trees[i], index, p.arities[i], depths[i + 1]);
      }
    }
  }
};

// ---------------------------------------------------------------- ring switching helpers

// fold_1b_rows_for_b128 (ring_switch.rs:197-265): out[k] = sum_i bit_k(mat[i]) * vec[i].
// Rows split over the threads; the partial sums are XORs, combined in any order.
static void fold_1b_rows(const u128* mat, const u128* vec, size_t n, u128 out[128]) {
  for (int k = 0; k < 128; k++) out[k] = 0;
  std::mutex mu;
  parallel_for(n, [&](size_t lo, size_t hi) {
    u128 part[128] = {0};
    for (size_t i = lo; i < hi; i++) {
      const u128 v = vec[i];
      for (uint64_t w = (uint64_t)mat[i]; w; w &= w - 1) part[__builtin_ctzll(w)] ^= v;
      for (uint64_t w = (uint64_t)(mat[i] >> 64); w; w &= w - 1) part[64 + __builtin_ctzll(w)] ^= v;
    }
    std::lock_guard<std::mutex> g(mu);
    for (int k = 0; k < 128; k++) out[k] ^= part[k];
  });
}

// fold_b128_elems_inplace (ring_switch.rs:130-171): x -> sum_k bit_k(x) * vec[k].
static u128 fold_elem(u128 x, const u128 vec[128]) {
  u128 acc = 0;
  for (uint64_t w = (uint64_t)x; w; w &= w - 1) acc ^= vec[__builtin_ctzll(w)];
  for (uint64_t w = (uint64_t)(x >> 64); w; w &= w - 1) acc ^= vec[64 + __builtin_ctzll(w)];
  return acc;
}

// TensorAlgebra<B1, B128>::transpose: the 128 x 128 bit matrix with row k = s[k].
static void transpose128(const u128 in[128], u128 out[128]) {
  for (int j = 0; j < 128; j++) {
    u128 v = 0;
    for (int k = 0; k < 128; k++) v |= (u128)((in[k] >> j) & 1) << k;
    out[j] = v;
  }
}

static u128 inner(const u128* a, const u128* b, size_t n) {
  u128 acc = 0;
  for (size_t i = 0; i < n; i++) acc ^= gf_mul(a[i], b[i]);
  return acc;
}

// ---------------------------------------------------------------- PCS prover

void pcs_prove(const FriParams& p, const u128* tw, const u128* codeword, const Tree& tree,
               const u128* witness, const u128* eval_point, Transcript& t) {
  const uint32_t n = p.log_msg;
  const size_t N = (size_t)1 << n;
  std::vector<u128> suffix_tensor(N);
  eq_ind_partial_eval(eval_point + 7, n, suffix_tensor.data());
  u128 s_hat_v[128];
  fold_1b_rows(witness, suffix_tensor.data(), N, s_hat_v);
  t.message_elems(s_hat_v, 128);
  u128 s_hat_u[128];
  transpose128(s_hat_v, s_hat_u);
  u128 r_dp[7];
  for (int i = 0; i < 7; i++) r_dp[i] = t.sample();
  u128 eq_r[128];
  eq_ind_partial_eval(r_dp, 7, eq_r);
  u128 sum = inner(s_hat_u, eq_r, 128);
  std::vector<u128> a(witness, witness + N), b(N);
  parallel_for(N, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; i++) b[i] = fold_elem(suffix_tensor[i], eq_r);
  });

  // BaseFoldProver::prove: bivariate product sumcheck interleaved with FRI folding.
  FriFolder fri(p, tw, codeword, tree);
  for (uint32_t round = 0; round < n; round++) {
    size_t half = a.size() / 2;
    u128 y1 = 0, yinf = 0;
    std::mutex mu;
    parallel_for(half, [&](size_t lo, size_t hi) {  // XOR sums: any split gives the same value
      u128 s1 = 0, sinf = 0;
      for (size_t i = lo; i < hi; i++) {
        s1 ^= gf_mul(a[half + i], b[half + i]);
        sinf ^= gf_mul(a[i] ^ a[half + i], b[i] ^ b[half + i]);
      }
      std::lock_guard<std::mutex> g(mu);
      y1 ^= s1;
      yinf ^= sinf;
    });
    u128 c0 = sum ^ y1, c2 = yinf, c1 = y1 ^ c0 ^ c2;
    uint8_t root[32];
    bool committed = fri.execute_fold_round(root);
    u128 coeffs[2] = {c0, c1};
    t.message_elems(coeffs, 2);
    if (committed) t.message(root, 32);
    u128 r = t.sample();
    parallel_for(half, [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; i++) {
        a[i] ^= gf_mul(r, a[half + i] ^ a[i]);
        b[i] ^= gf_mul(r, b[half + i] ^ b[i]);
      }
    });
    a.resize(half);
    b.resize(half);
    sum = c0 ^ gf_mul(c1, r) ^ gf_mul(c2, gf_mul(r, r));
    fri.receive_challenge(r);
  }
  uint8_t root[32];
  if (fri.execute_fold_round(root)) t.message(root, 32);
  fri.finish_proof(t);
}

// ---------------------------------------------------------------- PCS verifier

enum VerifyError {
  V_OK = 0,
  V_EVAL_CLAIM = 1,
  V_TAPE = 2,
  V_TERMINAL_ROOT = 3,
  V_TERMINAL_DEGREE = 4,
  V_LAYER_ROOT = 5,
  V_QUERY_PATH = 6,
  V_QUERY_FOLD = 7,
  V_FINAL = 8,
  V_TRAILING = 9,
};

static void leaf_digest(const u128* vals, size_t n, uint8_t out[32]) {
  merkle_leaf_hash((const uint8_t*)vals, 16 * n, out);
}

static void fold_digests(std::vector<uint8_t> d, uint8_t root[32]) {
  size_t len = d.size() / 32;
  while (len > 1) {
    for (size_t i = 0; i < len / 2; i++) {
      uint8_t o[32];
      merkle_node_hash(&d[64 * i], &d[64 * i + 32], o);
      memcpy(&d[32 * i], o, 32);
    }
    len /= 2;
  }
  memcpy(root, d.data(), 32);
}

// BinaryMerkleTreeScheme::verify_opening (merkle_tree/scheme.rs:122-158)
static bool verify_opening(Transcript& t, size_t index, const u128* vals, size_t n_vals,
                           uint32_t layer_depth, uint32_t tree_depth, const uint8_t* layer) {
  uint8_t d[32];
  leaf_digest(vals, n_vals, d);
  for (uint32_t j = 0; j < tree_depth - layer_depth; j++) {
    uint8_t sib[32], o[32];
    if (!t.read_decommit(sib, 32)) return false;
    if ((index & 1) == 0)
      merkle_node_hash(d, sib, o);
    else
      merkle_node_hash(sib, d, o);
    memcpy(d, o, 32);
    index >>= 1;
  }
  return memcmp(d, layer + 32 * index, 32) == 0;
}

int pcs_verify(const FriParams& p, const u128* tw, const u128* eval_point, u128 claim,
               const uint8_t codeword_root[32], Transcript& t) {
  const uint32_t n = p.log_msg;
  u128 s_hat_v[128];
  if (!t.read_message((uint8_t*)s_hat_v, 16 * 128)) return V_TAPE;
  u128 eq_lo[128];
  eq_ind_partial_eval(eval_point, 7, eq_lo);
  if (inner(s_hat_v, eq_lo, 128) != claim) return V_EVAL_CLAIM;
  u128 s_hat_u[128];
  transpose128(s_hat_v, s_hat_u);
  u128 batching[7];
  for (int i = 0; i < 7; i++) batching[i] = t.sample();
  u128 eq_b[128];
  eq_ind_partial_eval(batching, 7, eq_b);
  u128 sum = inner(s_hat_u, eq_b, 128);

  // calculate_fri_commit_rounds (verifier/verifier/src/fri/fold.rs:257-278) with n + 1 rounds.
  std::vector<bool> commit_rounds(n + 1, false);
  {
    uint32_t idx = 0;
    std::vector<uint32_t> steps{p.log_batch};
    steps.insert(steps.end(), p.arities.begin(), p.arities.end());
    for (auto a : steps) {
      idx += a;
      if (idx < n + 1)
        commit_rounds[idx] = true;
      else
        break;
    }
  }
  std::vector<std::vector<uint8_t>> round_roots;
  std::vector<u128> challenges;
  for (uint32_t round = 0; round < n; round++) {
    u128 c[2];
    if (!t.read_message((uint8_t*)c, 32)) return V_TAPE;
    if (commit_rounds[round]) {
      std::vector<uint8_t> r(32);
      if (!t.read_message(r.data(), 32)) return V_TAPE;
      round_roots.push_back(r);
    }
    // RoundProof::recover: c2 = sum - c0 - (c0 + c1)
    u128 c2 = sum ^ c[0] ^ c[0] ^ c[1];
    u128 r = t.sample();
    challenges.push_back(r);
    sum = c[0] ^ gf_mul(c[1], r) ^ gf_mul(c2, gf_mul(r, r));
  }
  if (commit_rounds[n]) {
    std::vector<uint8_t> r(32);
    if (!t.read_message(r.data(), 32)) return V_TAPE;
    round_roots.push_back(r);
  }
  if (round_roots.size() != 1 + p.arities.size()) return V_TAPE;

  // FRIQueryVerifier::verify (verifier/verifier/src/fri/verify.rs:86-200)
  const uint32_t n_final = p.n_final_challenges();
  std::vector<u128> terminal((size_t)1 << (n_final + p.log_inv_rate));
  if (!t.read_decommit((uint8_t*)terminal.data(), 16 * terminal.size())) return V_TAPE;
  {
    std::vector<uint8_t> digests;
    size_t coset = (size_t)1 << n_final;
    for (size_t i = 0; i < terminal.size() / coset; i++) {
      uint8_t d[32];
      leaf_digest(terminal.data() + i * coset, coset, d);
      digests.insert(digests.end(), d, d + 32);
    }
    uint8_t root[32];
    fold_digests(digests, root);
    if (memcmp(root, round_roots.back().data(), 32) != 0) return V_TERMINAL_ROOT;
  }
  const u128* fold_ch = challenges.data() + p.log_batch;
  const size_t n_fold_ch = challenges.size() - p.log_batch;
  u128 final_value = 0;
  {
    size_t coset = (size_t)1 << n_final;
    std::vector<u128> scratch(coset);
    for (size_t i = 0; i < terminal.size() / coset; i++) {
      memcpy(scratch.data(), terminal.data() + i * coset, 16 * coset);
      u128 v = fold_chunk(tw, n_final + p.log_inv_rate, i, scratch.data(),
                          fold_ch + (n_fold_ch - n_final), n_final);
      if (i == 0)
        final_value = v;
      else if (v != final_value)
        return V_TERMINAL_DEGREE;
    }
  }
  auto depths = p.optimal_depths();
  std::vector<std::vector<uint8_t>> layers;
  for (auto d : depths) {
    std::vector<uint8_t> l(32 * ((size_t)1 << d));
    if (!t.read_decommit(l.data(), l.size())) return V_TAPE;
    layers.push_back(l);
  }
  for (size_t i = 0; i < layers.size(); i++) {
    const uint8_t* commitment = i == 0 ? codeword_root : round_roots[i - 1].data();
    uint8_t root[32];
    fold_digests(layers[i], root);
    if (memcmp(root, commitment, 32) != 0) return V_LAYER_ROOT;
  }
  std::vector<u128> interleave_tensor((size_t)1 << p.log_batch);
  eq_ind_partial_eval(challenges.data(), p.log_batch, interleave_tensor.data());
  for (uint32_t q = 0; q < p.n_queries; q++) {
    size_t index = t.sample_bits(p.rs_log_len());
    std::vector<u128> vals((size_t)1 << p.log_batch);
    if (!t.read_decommit((uint8_t*)vals.data(), 16 * vals.size())) return V_TAPE;
    if (!verify_opening(t, index, vals.data(), vals.size(), depths[0], p.rs_log_len(),
                        layers[0].data()))
      return V_QUERY_PATH;
    u128 next = inner(vals.data(), interleave_tensor.data(), vals.size());
    uint32_t fold_round = 0, log_n_cosets = p.rs_log_len();
    for (size_t i = 0; i < p.arities.size() && i + 1 < layers.size(); i++) {
      uint32_t arity = p.arities[i];
      size_t coset_index = index >> arity;
      log_n_cosets -= arity;
      std::vector<u128> cv((size_t)1 << arity);
      if (!t.read_decommit((uint8_t*)cv.data(), 16 * cv.size())) return V_TAPE;
      if (!verify_opening(t, coset_index, cv.data(), cv.size(), depths[i + 1], log_n_cosets,
                          layers[i + 1].data()))
        return V_QUERY_PATH;
      if (next != cv[index % ((size_t)1 << arity)]) return V_QUERY_FOLD;
      next = fold_chunk(tw, p.rs_log_len() - fold_round, coset_index, cv.data(),
                        fold_ch + fold_round, arity);
      index = coset_index;
      fold_round += arity;
    }
    if (next != terminal[index]) return V_QUERY_FOLD;
  }

  // Final consistency (pcs.rs verify): sumcheck value == fri value * rs_eq(z, reversed r, eq_b),
  // with rs_eq evaluated as <rs_eq_ind(batching, z), eq(reversed challenges)>.
  std::vector<u128> rev(challenges.rbegin(), challenges.rend());
  const size_t N = (size_t)1 << n;
  std::vector<u128> z_tensor(N), q_tensor(N);
  eq_ind_partial_eval(eval_point + 7, n, z_tensor.data());
  eq_ind_partial_eval(rev.data(), n, q_tensor.data());
  u128 rs_eq = 0;
  for (size_t i = 0; i < N; i++) rs_eq ^= gf_mul(fold_elem(z_tensor[i], eq_b), q_tensor[i]);
  if (sum != gf_mul(final_value, rs_eq)) return V_FINAL;
  return V_OK;
}

static FriParams make_params(uint32_t log_msg, uint32_t log_batch, uint32_t log_inv_rate,
                             const uint32_t* arities, uint32_t n_arities, uint32_t n_queries) {
  FriParams p;
  p.log_msg = log_msg;
  p.log_batch = log_batch;
  p.log_inv_rate = log_inv_rate;
  p.arities.assign(arities, arities + n_arities);
  p.n_queries = n_queries;
  return p;
}

}  // namespace orc

using namespace orc;

extern "C" {

void* orc_transcript_new(void) { return new Transcript(); }
void orc_transcript_free(void* t) { delete static_cast<Transcript*>(t); }
void orc_transcript_observe(void* t, const uint8_t* p, size_t n) {
  static_cast<Transcript*>(t)->observe(p, n);
}
void orc_transcript_sample(void* t, uint8_t* out, size_t n) {
  static_cast<Transcript*>(t)->sample_bytes(out, n);
}

// Multilinear evaluation of the B1 polynomial whose bit (i << 7) | k is bit k of witness[i].
void orc_eval_1b_mle(const uint64_t* witness, uint32_t log_msg, const uint64_t* point,
                     uint64_t* out) {
  const u128* w = (const u128*)witness;
  const u128* pt = (const u128*)point;
  size_t N = (size_t)1 << log_msg;
  std::vector<u128> hi(N);
  eq_ind_partial_eval(pt + 7, log_msg, hi.data());
  u128 lo[128];
  eq_ind_partial_eval(pt, 7, lo);
  u128 acc = 0;
  for (size_t i = 0; i < N; i++) acc ^= gf_mul(fold_elem(w[i], lo), hi[i]);
  store(out, acc);
}

// Commits the witness (RS encode + Merkle), writes the root as the first transcript message and
// proves the evaluation at eval_point (log_msg + 7 coordinates).  twiddles: the RS code's domain.
int orc_pcs_prove(const uint64_t* twiddles, const uint64_t* witness, uint32_t log_msg,
                  uint32_t log_batch, uint32_t log_inv_rate, const uint32_t* arities,
                  uint32_t n_arities, uint32_t n_queries, const uint64_t* eval_point,
                  uint8_t* proof_out, size_t proof_cap, size_t* proof_len) {
  FriParams p = make_params(log_msg, log_batch, log_inv_rate, arities, n_arities, n_queries);
  const u128* tw = (const u128*)twiddles;
  std::vector<u128> codeword((size_t)1 << p.log_len());
  rs_encode(tw, (const u128*)witness, p.log_dim(), log_inv_rate, log_batch, codeword.data());
  Tree tree = build_tree(codeword.data(), p.rs_log_len(), log_batch);
  Transcript t;
  t.message(tree.root(), 32);
  pcs_prove(p, tw, codeword.data(), tree, (const u128*)witness, (const u128*)eval_point, t);
  *proof_len = t.tape.size();
  if (t.tape.size() > proof_cap) return 1;
  memcpy(proof_out, t.tape.data(), t.tape.size());
  return 0;
}

int orc_pcs_verify(const uint64_t* twiddles, uint32_t log_msg, uint32_t log_batch,
                   uint32_t log_inv_rate, const uint32_t* arities, uint32_t n_arities,
                   uint32_t n_queries, const uint64_t* eval_point, const uint64_t* claim,
                   const uint8_t* proof, size_t proof_len) {
  FriParams p = make_params(log_msg, log_batch, log_inv_rate, arities, n_arities, n_queries);
  Transcript t;
  t.tape.assign(proof, proof + proof_len);
  uint8_t root[32];
  if (!t.read_message(root, 32)) return V_TAPE;
  int rc = pcs_verify(p, (const u128*)twiddles, (const u128*)eval_point, load(claim), root, t);
  if (rc) return rc;
  if (t.overrun) return V_TAPE;
  if (t.pos != t.tape.size()) return V_TRAILING;
  return V_OK;
}

}  // extern "C"
