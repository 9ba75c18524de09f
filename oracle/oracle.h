/*
 * CPU oracle for the Binius64 prover hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain C++ restatement of the
 * reference algorithms (IrreducibleOSS/binius64) and exists to check the CUDA
 * library bit-for-bit.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs may load it.  The product path
 * (binius64_b200/) never links, imports or calls anything here.
 *
 * Parity pins: see tests/test_oracle_pins.py (GHASH KATs from
 * verifier/field/src/ghash.rs:798-925, the NTT evaluation semantics of
 * verifier/math/src/ntt/tests_evaluation.rs:244-295, FRI parameter KATs of
 * verifier/verifier/src/fri/common.rs:225-247, SHA-256 against FIPS 180-4 via
 * Python's hashlib, transcript chaining of
 * verifier/transcript/src/fiat_shamir/hasher_challenger.rs:209-280).
 *
 * Field elements are 16-byte little-endian u128 values (the reference's
 * serialization, verifier/field/src/ghash.rs:486-498): two uint64 words, low
 * word first.
 */
#ifndef BINIUS_ORACLE_H
#define BINIUS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- GF(2^128), modulus x^128 + x^7 + x^2 + x + 1 (ghash.rs:3, 68-80) ---- */
void orc_gf_mul(const uint64_t a[2], const uint64_t b[2], uint64_t out[2]);
void orc_gf_mul_portable(const uint64_t a[2], const uint64_t b[2], uint64_t out[2]);
void orc_gf_inv(const uint64_t a[2], uint64_t out[2]);
void orc_gf_mul_x(const uint64_t a[2], uint64_t out[2]);
void orc_gf_mul_inv_x(const uint64_t a[2], uint64_t out[2]);
/* Elementwise products of n pairs (used by tests to cross-check the device). */
void orc_gf_mul_vec(const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n);
/* AES GF(2^8) (aes_field.rs:26-35) and the GF(2^8) -> GF(2^128) embedding. */
uint8_t orc_aes_mul(uint8_t a, uint8_t b);
void orc_aes_to_ghash_table(uint64_t out[512]);

/* ---- SHA-256 (FIPS 180-4) and the Binius node compression (hash/compress.rs:32-57) ---- */
void orc_sha256(const uint8_t* data, size_t len, uint8_t out[32]);
void orc_sha256_compress_node(const uint8_t left[32], const uint8_t right[32], uint8_t out[32]);

/* ---- Domain context: GenericPreExpanded (ntt/domain_context.rs:19-46, 99-159) ----
 * basis: dim elements (NULL = BinarySubspace::with_dim, basis x^i).
 * Writes the flat twiddle table: layer l occupies [2^l - 1, 2^(l+1) - 1). */
int orc_domain_twiddles(const uint64_t* basis, uint32_t dim, uint64_t* twiddles_out);

/* ---- Additive NTT, NeighborsLastReference (ntt/reference.rs:20-76) ---- */
int orc_ntt_forward(const uint64_t* twiddles, uint32_t log_domain, uint64_t* data, uint32_t log_d,
                    uint32_t skip_early, uint32_t skip_late);
int orc_ntt_inverse(const uint64_t* twiddles, uint32_t log_domain, uint64_t* data, uint32_t log_d,
                    uint32_t skip_early, uint32_t skip_late);

/* ---- ReedSolomonCode::encode_batch (reed_solomon.rs:128-201) ---- */
int orc_rs_encode_batch(const uint64_t* twiddles, uint32_t log_domain, const uint64_t* msg,
                        uint32_t log_dim, uint32_t log_inv_rate, uint32_t log_batch,
                        uint64_t* codeword_out);

/* ---- Merkle tree (binary_merkle_tree.rs:65-122), SHA-256 leaves, Binius compression nodes ----
 * nodes_out: (2^(log_leaves+1) - 1) * 32 bytes, leaves first, root last. */
int orc_merkle_commit(const uint64_t* elems, uint32_t log_leaves, uint32_t log_batch,
                      uint8_t* nodes_out);

/* ---- Vision-4 hash (verifier/verifier/src/hash/vision_4) ----
 * state: 4 elements (8 words); digest: incremental updates ending at each of splits[0..n_splits)
 * then at len; compress: 64 input bytes (left || right) -> 32; map: 0 = L, 1 = L^-1, 2 = B,
 * 3 = B^-1; constants: the 17 x 4 round constants and B_INV_COEFFS[0]; merkle_commit: as
 * orc_merkle_commit with Vision-4 leaves (VisionHasherDigest) and nodes (VisionCompression). */
void orc_vision4_permutation(uint64_t* state);
/* Selects the Merkle hash of orc_merkle_commit, the PCS and the whole prove / verify:
 * 0 = SHA-256 (StdDigest + StdCompression, the default), 1 = Vision-4. */
void orc_set_merkle_hash(int kind);
void orc_vision4_digest(const uint8_t* data, size_t len, const size_t* splits, size_t n_splits,
                        uint8_t* out);
void orc_vision4_compress(const uint8_t* in64, uint8_t* out32);
void orc_vision4_map(int which, const uint64_t* x, uint64_t* out);
void orc_vision4_constants(uint64_t* rc, uint64_t* binv0);
int orc_vision4_merkle_commit(const uint64_t* elems, uint32_t log_leaves, uint32_t log_batch,
                              uint8_t* nodes_out);

/* ---- Witness evaluation (verifier/frontend/src/compiler/eval_form/interpreter.rs) ----
 * Runs the bytecode over values[0..n_values) in place.  Returns 0, or -1 unknown opcode, -2 hint
 * call, -3 register out of range, -4 truncated instruction, -5 shift amount >= 64.
 * n_failures / first_error_id: assertion failures and the id of the first one. */
int orc_eval_form_run(const uint8_t* code, size_t len, uint64_t* values, size_t n_values,
                      uint32_t* n_failures, uint32_t* first_error_id);

/* ---- FRI folds (prover/prover/src/fri/fold.rs:260-318; verifier/.../fri/fold.rs:20-130) ---- */
void orc_eq_ind_partial_eval(const uint64_t* point, uint32_t n, uint64_t* out);
int orc_fri_fold_interleaved(const uint64_t* codeword, uint32_t log_len, uint32_t log_batch,
                             const uint64_t* challenges, uint64_t* out);
int orc_fri_fold_codeword(const uint64_t* twiddles, uint32_t log_domain, const uint64_t* codeword,
                          uint32_t log_len, const uint64_t* challenges, uint32_t n_challenges,
                          uint64_t* out);

/* ---- FRI parameters (verifier/verifier/src/fri/common.rs:64-219) ---- */
uint32_t orc_calculate_n_test_queries(uint32_t security_bits, uint32_t log_inv_rate);
uint32_t orc_estimate_optimal_arity(uint32_t log_block_length, uint32_t digest_size,
                                    uint32_t field_size);

/* ---- Fiat-Shamir transcript (HasherChallenger<Sha256>), for known-answer tests ---- */
void* orc_transcript_new(void);
void orc_transcript_free(void* t);
void orc_transcript_observe(void* t, const uint8_t* p, size_t n);
void orc_transcript_sample(void* t, uint8_t* out, size_t n);

/* ---- 1-bit multilinear PCS (ring switching + BaseFold + FRI) ----
 * witness: 2^log_msg packed B128 elements (the B1 multilinear of log_msg + 7 variables);
 * eval_point: log_msg + 7 elements; twiddles: the RS code domain's table. */
void orc_eval_1b_mle(const uint64_t* witness, uint32_t log_msg, const uint64_t* point,
                     uint64_t* out);
int orc_pcs_prove(const uint64_t* twiddles, const uint64_t* witness, uint32_t log_msg,
                  uint32_t log_batch, uint32_t log_inv_rate, const uint32_t* arities,
                  uint32_t n_arities, uint32_t n_queries, const uint64_t* eval_point,
                  uint8_t* proof_out, size_t proof_cap, size_t* proof_len);
/* 0 = accepted; otherwise the failed check (1 evaluation claim, 2 tape, 3 terminal root,
 * 4 terminal degree, 5 layer root, 6 query path, 7 query fold, 8 final consistency, 9 trailing). */
int orc_pcs_verify(const uint64_t* twiddles, uint32_t log_msg, uint32_t log_batch,
                   uint32_t log_inv_rate, const uint32_t* arities, uint32_t n_arities,
                   uint32_t n_queries, const uint64_t* eval_point, const uint64_t* claim,
                   const uint8_t* proof, size_t proof_len);

/* ---- Operands and the AND reduction (prover/prover/src/and_reduction/, prove.rs:329-372) ---- */
uint64_t orc_shifted_word(uint64_t w, uint32_t variant, uint32_t amount);
void orc_and_univariate_round(const uint64_t* a, const uint64_t* b, const uint64_t* c,
                              uint32_t log_n, const uint64_t* big, uint64_t* msg_out);
void orc_and_fold_words(const uint64_t* w, size_t n, const uint64_t* z, uint64_t* out);
int orc_and_reduction_prove(const uint64_t* a, const uint64_t* b, const uint64_t* c,
                            uint32_t log_n, uint8_t* proof_out, size_t cap, size_t* len,
                            uint64_t* out_meta, uint64_t* out_point);
int orc_and_reduction_verify(uint32_t log_n, const uint8_t* proof, size_t len, uint64_t* out_meta,
                             uint64_t* out_point);

/* ---- Shift reduction (prover/prover/src/protocols/shift/, verifier/verifier/src/protocols/shift/verify.rs) ----
 * csr = {offsets, value indices, amounts} (u32 arrays), var = shift variants (u8). */
int orc_shift_prove(const uint64_t* words, uint32_t log_words, uint32_t log_public,
                    const uint32_t* const* and_csr, const uint8_t* and_var, uint32_t n_and,
                    const uint32_t* const* mul_csr, const uint8_t* mul_var, uint32_t n_mul,
                    const uint64_t* and_evals, const uint64_t* and_rz, const uint64_t* and_rx,
                    const uint64_t* mul_evals, const uint64_t* mul_rz, const uint64_t* mul_rx,
                    uint8_t* proof, size_t cap, size_t* len, uint64_t* out_point,
                    uint64_t* out3);
int orc_shift_verify(const uint64_t* public_words, uint32_t log_words, uint32_t log_public,
                     const uint32_t* const* and_csr, const uint8_t* and_var, uint32_t n_and,
                     const uint32_t* const* mul_csr, const uint8_t* mul_var, uint32_t n_mul,
                     const uint64_t* and_evals, const uint64_t* and_rz, const uint64_t* and_rx,
                     const uint64_t* mul_evals, const uint64_t* mul_rz, const uint64_t* mul_rx,
                     const uint8_t* proof, size_t len, uint64_t* out_eval, uint64_t* out_point);
void orc_oblong_eval(const uint64_t* v, uint32_t log_n, const uint64_t* z, const uint64_t* r_x,
                     uint64_t* out);

/* ---- Integer multiplication reduction (prover/prover/src/protocols/intmul/) ----
 * out_point: log_n elements; out_evals: 4 x 64 elements (bit-column evaluations of a, b, lo, hi). */
int orc_intmul_prove(const uint64_t* a, const uint64_t* b, const uint64_t* lo, const uint64_t* hi,
                     uint32_t log_n, uint8_t* proof, size_t cap, size_t* len,
                     uint64_t* out_point, uint64_t* out_evals);
int orc_intmul_verify(uint32_t log_n, const uint8_t* proof, size_t len, uint64_t* out_point,
                      uint64_t* out_evals);

/* ---- Prover::prove / Verifier::verify (prover/prover/src/prove.rs:124-303,
 * verifier/verifier/src/verify.rs:61-282) over a CSR constraint system (as for the shift
 * reduction) and 2^log_words witness words. */
void orc_prove_params(uint32_t log_words, uint32_t log_inv_rate, uint32_t* out4,
                      uint32_t* out_arities);
int orc_prove(const uint64_t* words, uint32_t log_words, uint32_t log_public,
              const uint32_t* const* and_csr, const uint8_t* and_var, uint32_t n_and,
              const uint32_t* const* mul_csr, const uint8_t* mul_var, uint32_t n_mul,
              uint32_t log_inv_rate, uint8_t* proof, size_t cap, size_t* len);
int orc_verify(const uint64_t* public_words, uint32_t log_words, uint32_t log_public,
               const uint32_t* const* and_csr, const uint8_t* and_var, uint32_t n_and,
               const uint32_t* const* mul_csr, const uint8_t* mul_var, uint32_t n_mul,
               uint32_t log_inv_rate, const uint8_t* proof, size_t len);

/* Number of worker threads the oracle may use (1 = scalar). */
void orc_set_threads(int n);

/* ---- Round-by-round sumcheck provers over given challenges (sumcheck.cpp):
 * BivariateProductSumcheckProver (bivariate_product.rs:17-119), QuadraticMleCheckProver with
 * composition a*b - c (quadratic_mle.rs:21-229), InOutCheckProver (inout_check.rs:19-221).
 * coeffs_out: each round's RoundCoeffs (3 or 2 elements); evals_out: finish(). */
int orc_bivariate_rounds(const uint64_t* a, const uint64_t* b, uint32_t n, const uint64_t* sum,
                         const uint64_t* challenges, uint64_t* coeffs_out, uint64_t* evals_out);
int orc_quadratic_mle_rounds(const uint64_t* a, const uint64_t* b, const uint64_t* c, uint32_t n,
                             const uint64_t* point, const uint64_t* claim,
                             const uint64_t* challenges, uint64_t* coeffs_out,
                             uint64_t* evals_out);
int orc_inout_rounds(const uint64_t* w, uint32_t n, const uint64_t* point, uint32_t m,
                     const uint64_t* challenges, uint64_t* coeffs_out, uint64_t* eval_out);

/* The AND univariate round's per-word lookup NTT (ntt_lookup.rs:91-164) and the shift
 * reduction's h multilinears with their Lagrange basis (monster.rs:34-104). */
void orc_and_word_ntt(uint64_t w, uint8_t out[64]);
void orc_shift_h_parts(const uint64_t* r_zhat, uint64_t* h_out, uint64_t* l_tilde_out);

#ifdef __cplusplus
}
#endif
#endif
