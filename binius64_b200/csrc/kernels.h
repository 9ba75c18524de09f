// Host-side launch helpers shared by the protocol drivers (all asynchronous on `s`).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/binius_gpu.h"
#include "internal.h"

namespace bgpu {

// Up to 32 field elements passed to a kernel by value.
struct Point32 {
  uint4 r[32];
};

// eq_ind_partial_eval of a host point with n <= 32 coordinates into d_out (2^n elements).
int eq_tensor(const uint4* h_point, uint32_t n, uint4* d_out, cudaStream_t s);
// d_out512 (128 elements) = fold_1b_rows_for_b128(mat, vec) over n rows.
int fold_1b_rows(const uint4* d_mat, const uint4* d_vec, uint64_t n, uint32_t* d_out512,
                 cudaStream_t s);
// d_out[i] = sum_k bit_k(d_in[i]) * d_vec128[k]  (d_out may equal d_in).
int fold_b128_elems(const uint4* d_in, uint4* d_out, uint64_t n, const uint4* d_vec128,
                    cudaStream_t s);
// d_out8 = (y_1, y_inf) of the bivariate product round on (a, b) of length 2*half.
int bivariate_eval(const uint4* d_a, const uint4* d_b, uint64_t half, uint32_t* d_out8,
                   cudaStream_t s);
// Fold (a, b) of length size by r, then (y_1, y_inf) of the next round.
int bivariate_fold_eval(uint4* d_a, uint4* d_b, uint64_t size, const uint8_t r[16],
                        uint32_t* d_out8, cudaStream_t s);
// As bivariate_fold_eval with the challenge in device memory (d_r) and no clearing of d_out8.
int bivariate_fold_eval_dev(uint4* d_a, uint4* d_b, uint64_t size, const uint4* d_r,
                            uint32_t* d_out8, cudaStream_t s);
class DeviceTranscript;
// The device Fiat-Shamir step of a plain bivariate product round: reads (y_1, y_inf) at d_ys
// and the claim (d_claim_init if set, else d_claim), writes the message (c_0, c_1) and then the
// 32 bytes at d_commitment if set, samples r into d_r_out and updates d_claim.
int bivariate_round_finish(const DeviceTranscript& dt, const uint4* d_ys, const uint4* d_claim_init,
                           uint4* d_claim, const uint8_t* d_commitment, uint4* d_r_out,
                           cudaStream_t s);
// The last n_rounds rounds of a plain bivariate product sumcheck in one launch (one CTA): each
// round folds (a, b) -- of length len before the first fold -- by the previous challenge
// (d_r_first for the first round, when set) and runs the Fiat-Shamir step of
// bivariate_round_finish; challenges go to d_chal[0 .. n_rounds), the claim stays in d_claim.
int bivariate_tail(const DeviceTranscript& dt, uint4* d_a, uint4* d_b, uint64_t len,
                   uint32_t n_rounds, const uint4* d_r_first, uint4* d_claim, uint4* d_chal,
                   cudaStream_t s);
// Sumcheck rounds whose arrays have at most this many elements before the fold run in the
// single-CTA tail kernels (the calling thread's Tuning::tail_log; 2^11 by default).
inline uint64_t tail_max_len() { return 1ull << tuning().tail_log; }
// Folds of at least this many elements multiply by the fold challenge through its nibble tables
// (gf_mul_nibble, built by every block in shared memory); smaller ones spread each position
// over lanes and use the integer multiply.
constexpr uint64_t kMulTableMinSize = 1ull << 15;

// Lagrange basis of the subspace {phi(t) : t < 2^dim} at x, phi the AES-to-GHASH embedding
// (BinarySubspace::<AESTowerField8b>::with_dim(dim).isomorphic(), lagrange_evals).
void lagrange_phi(uint32_t dim, hu128 x, hu128* out);
hu128 phi_elem(uint32_t b);
// d_out8 = (y_1, y_inf) of the AND reduction's MLE-check round on columns a, b, c of length
// 2 * half with eq of length half: y_1 = sum eq (a_1 b_1 + c_1), y_inf = sum eq a_inf b_inf.
int and_mle_eval(const uint4* d_a, const uint4* d_b, const uint4* d_c, const uint4* d_eq,
                 uint64_t half, uint32_t* d_out8, cudaStream_t s);
// d_out[i] = sum over set bits t of d_words[i] of vec64[t] (fold_words, prover/prover/src/
// fold_word.rs:77-96).
int fold_words64(const uint64_t* d_words, uint64_t n, const hu128* vec64, uint4* d_out,
                 cudaStream_t s);

// FRI folds whose challenges are in device memory (sampled by the device transcript); the same
// results as binius_fri_fold_interleaved / binius_fri_fold_codeword.
int fri_fold_interleaved_dev(const void* d_codeword, uint32_t log_len, uint32_t log_batch,
                             const uint4* d_challenges, void* d_out, cudaStream_t s);
int fri_fold_codeword_dev(const binius_ntt* ntt, const void* d_codeword, uint32_t log_len,
                          const uint4* d_challenges, uint32_t n_challenges, void* d_out,
                          cudaStream_t s);

// From the other translation units.
int rs_encode_batch(const binius_ntt* ntt, const void* d_msg, uint32_t log_dim,
                    uint32_t log_inv_rate, uint32_t log_batch, void* d_codeword,
                    cudaStream_t stream);
int merkle_commit(const void* d_elems, uint32_t log_leaves, uint32_t log_batch, void* d_nodes,
                  cudaStream_t stream);
int vision4_merkle_commit(const void* d_elems, uint32_t log_leaves, uint32_t log_batch,
                          void* d_nodes, cudaStream_t stream);
// The Merkle hash of a commitment scheme: SHA-256 (StdDigest + StdCompression) or Vision-4.
enum MerkleHash : uint32_t { kMerkleSha256 = 0, kMerkleVision4 = 1 };
inline int merkle_commit_with(uint32_t hash, const void* d_elems, uint32_t log_leaves,
                              uint32_t log_batch, void* d_nodes, cudaStream_t stream) {
  return hash == kMerkleVision4
             ? vision4_merkle_commit(d_elems, log_leaves, log_batch, d_nodes, stream)
             : merkle_commit(d_elems, log_leaves, log_batch, d_nodes, stream);
}
int fri_commit_interleaved(const binius_ntt* ntt, const void* d_msg, uint32_t log_dim,
                           uint32_t log_inv_rate, uint32_t log_batch, uint32_t merkle_hash,
                           void* d_codeword, void* d_nodes, void* h_root, cudaStream_t s);
// binius_pcs_commit without the root's read-back: queues the encode and the Merkle commit on s;
// the root is at pcs_committed_root(*out) on the device once they ran, and the caller hands
// the host copy to pcs_committed_set_root before anything reads the committed root.
int pcs_commit_enqueue(const binius_pcs* P, const void* d_witness, binius_pcs_committed** out,
                       cudaStream_t s);
const uint8_t* pcs_committed_root(const binius_pcs_committed* c);
void pcs_committed_set_root(binius_pcs_committed* c, const uint8_t* h_root);

}  // namespace bgpu
