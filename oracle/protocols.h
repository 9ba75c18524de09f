// CPU oracle (test infrastructure only): the protocol pieces shared by the oracle's reductions
// and its restated Prover::prove / Verifier::verify.
#ifndef BINIUS_ORACLE_PROTOCOLS_H
#define BINIUS_ORACLE_PROTOCOLS_H

#include <stdint.h>

#include <vector>

#include "oracle_internal.h"
#include "transcript.h"

namespace orc {

// ---------------------------------------------------------------- Merkle helpers

struct Tree {
  uint32_t log_leaves = 0;
  std::vector<uint8_t> nodes;
  const uint8_t* root() const { return nodes.data() + nodes.size() - 32; }
  // BinaryMerkleTree::layer (binary_merkle_tree.rs:142-150)
  const uint8_t* layer(uint32_t depth) const {
    size_t total = nodes.size() / 32;
    return nodes.data() + 32 * (total + 1 - ((size_t)1 << (depth + 1)));
  }
  // BinaryMerkleTree::branch (binary_merkle_tree.rs:152-169)
  void branch(size_t index, uint32_t depth, std::vector<uint8_t>& out) const {
    uint32_t L = log_leaves;
    for (uint32_t j = 0; j < L - depth; j++) {
      size_t node = ((((size_t)1 << j) - 1) << (L + 1 - j)) | ((index >> j) ^ 1);
      out.insert(out.end(), nodes.data() + 32 * node, nodes.data() + 32 * node + 32);
    }
  }
};

inline Tree build_tree(const u128* elems, uint32_t log_leaves, uint32_t log_batch) {
  Tree t;
  t.log_leaves = log_leaves;
  t.nodes.resize(32 * (((size_t)2 << log_leaves) - 1));
  merkle_commit(elems, log_leaves, log_batch, t.nodes.data());
  return t;
}

inline uint32_t ceil_log2(uint32_t n) {
  uint32_t r = 0;
  while (((uint64_t)1 << r) < n) r++;
  return r;
}

inline uint32_t log2_exact(size_t n) {
  uint32_t r = 0;
  while (((size_t)1 << r) < n) r++;
  return r;
}

// ---------------------------------------------------------------- FRI parameters

struct FriParams {
  uint32_t log_msg;       // log2 of the interleaved message length (the multilinear's n_vars)
  uint32_t log_batch;
  uint32_t log_inv_rate;
  std::vector<uint32_t> arities;
  uint32_t n_queries;
  uint32_t log_dim() const { return log_msg - log_batch; }
  uint32_t rs_log_len() const { return log_dim() + log_inv_rate; }
  uint32_t log_len() const { return rs_log_len() + log_batch; }
  uint32_t n_final_challenges() const {
    uint32_t s = 0;
    for (auto a : arities) s += a;
    return log_dim() - s;
  }
  // vcs_optimal_layers_depths_iter (verifier/verifier/src/fri/common.rs:154-168)
  std::vector<uint32_t> optimal_depths() const {
    std::vector<uint32_t> d;
    uint32_t cap = ceil_log2(n_queries);
    uint32_t log_n_cosets = log_len();
    std::vector<uint32_t> steps{log_batch};
    steps.insert(steps.end(), arities.begin(), arities.end());
    for (auto a : steps) {
      log_n_cosets -= a;
      d.push_back(cap < log_n_cosets ? cap : log_n_cosets);
    }
    return d;
  }
};

// ---------------------------------------------------------------- 1-bit PCS (pcs.cpp)

void pcs_prove(const FriParams& p, const u128* tw, const u128* codeword, const Tree& tree,
               const u128* witness, const u128* eval_point, Transcript& t);
int pcs_verify(const FriParams& p, const u128* tw, const u128* eval_point, u128 claim,
               const uint8_t root[32], Transcript& t);

// ---------------------------------------------------------------- AND reduction

// eval_shifted_word (verifier/core/src/verify.rs:14-26).
uint64_t shifted_word(uint64_t w, uint32_t variant, uint32_t amount);

struct AndOutput {
  u128 a_eval, b_eval, c_eval, z;
  std::vector<u128> eval_point;
};

AndOutput and_reduction_prove(const uint64_t* a, const uint64_t* b, const uint64_t* c,
                              uint32_t log_n, Transcript& t);
bool and_reduction_verify(uint32_t log_n, Transcript& t, AndOutput& out);

// ---------------------------------------------------------------- IntMul reduction

struct IntMulResult {
  std::vector<u128> eval_point;
  std::vector<u128> a_evals, b_evals, c_lo_evals, c_hi_evals;
};

IntMulResult intmul_prove(const uint64_t* a, const uint64_t* b, const uint64_t* lo,
                          const uint64_t* hi, uint32_t n_vars, Transcript& t);
int intmul_verify(uint32_t n_vars, Transcript& t, IntMulResult& res);

// ---------------------------------------------------------------- shift reduction

struct Ops {
  uint32_t k;                 // operands per constraint
  uint32_t n;                 // constraints (padded)
  const uint32_t* off;        // n * k + 1
  const uint32_t* vi;
  const uint8_t* var;
  const uint32_t* amt;
  const uint32_t* slot_to_operand;  // CSR slot -> KeyCollection operand index
};

struct OpData {
  std::vector<u128> evals;
  u128 r_zhat;
  std::vector<u128> r_x;
  std::vector<u128> eq;       // eq(r_x)
  std::vector<u128> lpow;     // lambda^(i+1)
};

struct ShiftResult {
  std::vector<u128> challenges;  // r_j ++ r_y
  u128 witness_eval;
  u128 initial_sum;              // sum_v <g_v, h_v>
  u128 claim;                    // sum over operators of lambda^(i+1) evals[i]
};

ShiftResult shift_prove(const uint64_t* words, uint32_t log_words, uint32_t log_public,
                        const Ops& and_ops, const Ops& mul_ops, OpData& band, OpData& bmul,
                        Transcript& t);
int shift_verify(const uint64_t* public_words, uint32_t log_words, uint32_t log_public,
                 const Ops& and_ops, const Ops& mul_ops, OpData& band, OpData& bmul,
                 Transcript& t, u128& witness_eval, std::vector<u128>& point);

// Lagrange basis of {phi(t) : t < 64} at z (verifier/math/src/univariate.rs:47-78).
void l_tilde64(u128 z, u128 out[64]);

}  // namespace orc

#endif
