/*
 * binius_gpu.h -- C ABI of the B200 (sm_100a) Binius64 prover hot path.
 *
 * Every entry point returns a binius_status; on failure binius_last_error() gives a message
 * (thread-local).  Field elements are BinaryField128bGhash values in their 16-byte little-endian
 * u128 encoding (verifier/field/src/ghash.rs:486-498); digests are 32 raw bytes.  Pointers named
 * d_* are device pointers on the current CUDA device; h_* are host pointers.  `stream` is a
 * cudaStream_t (NULL = legacy default stream).  Device entry points are asynchronous on `stream`
 * unless stated otherwise.  No entry point throws or aborts; argument errors map to BINIUS_E_ARG,
 * mirroring binius_prover::Error::ArgumentError (prover/prover/src/error.rs:9-24).
 */
#ifndef BINIUS_GPU_H
#define BINIUS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum binius_status {
  BINIUS_OK = 0,
  BINIUS_E_ARG = 1,     /* invalid argument / precondition (ArgumentError, assert! in the reference) */
  BINIUS_E_OOM = 2,     /* device allocation refused */
  BINIUS_E_CUDA = 3,    /* CUDA runtime error */
  BINIUS_E_TIMEOUT = 4, /* a bounded device-side wait expired */
  BINIUS_E_UNSUPPORTED = 5
} binius_status;

/* Last error message of the calling thread ("" if none). */
const char* binius_last_error(void);
/* Library version string. */
const char* binius_version(void);
/* Cumulative number of CUDA kernels launched by this library in this process (no reference
 * counterpart: launch accounting for benchmarks and tests). */
uint64_t binius_launch_count(void);
/* Host-side failure injection for tests (no reference counterpart): after n_before_failure more
 * device allocations of the prove path succeed, the next one is refused as the allocator refuses
 * one (BINIUS_E_OOM from the call that made it); a negative value turns injection off.  No
 * kernel is involved: the refusal happens on the host before anything is launched with it. */
void binius_debug_fail_allocs(int64_t n_before_failure);

/* ------------------------------------------------------------------------------------------
 * AdditiveNTT over a GenericPreExpanded domain context.
 * Replaces: trait AdditiveNTT (verifier/math/src/ntt/mod.rs:58-113), DomainContext
 * (ntt/mod.rs:118-179), GenericPreExpanded::generate_from_subspace
 * (ntt/domain_context.rs:114-133), NeighborsLastMultiThread::forward_transform
 * (ntt/neighbors_last.rs:461-520).
 * ------------------------------------------------------------------------------------------ */
typedef struct binius_ntt binius_ntt;

/* Builds the twiddle table (2^log_domain - 1 elements, layer l at offset 2^l - 1) on `device`.
 * h_basis: log_domain field elements, or NULL for BinarySubspace::with_dim (basis x^i). */
int binius_ntt_create(int device, const void* h_basis, uint32_t log_domain, binius_ntt** out);
int binius_ntt_destroy(binius_ntt* ntt);
/* DomainContext::subspace(dim) (ntt/domain_context.rs:142-147) of the domain a binius_ntt_create
 * with the same h_basis / log_domain would build, computed on the host without building the
 * twiddle table: h_out receives dim field elements (the subspace of dimension dim, as the
 * normalized subspace-polynomial evaluations evals[log_domain - dim]).  The Reed-Solomon code of
 * an interleaved commitment of 2^log_batch columns over the standard domain of dimension
 * log_len + log_batch uses subspace(log_len) (verifier/verifier/src/verify.rs:85-97). */
int binius_domain_subspace(const void* h_basis, uint32_t log_domain, uint32_t dim, void* h_out);
/* log2 of the domain size (DomainContext::log_domain_size). */
uint32_t binius_ntt_log_domain(const binius_ntt* ntt);
/* Device pointer of the flat twiddle table (DomainContext::twiddle(layer, block) is entry
 * 2^layer - 1 + block). */
const void* binius_ntt_twiddles(const binius_ntt* ntt);

/* In-place forward / inverse transform of 2^log_len elements, layers
 * [skip_early, log_len - skip_late) (AdditiveNTT::forward_transform / inverse_transform;
 * preconditions of ntt/reference.rs:85-100). */
int binius_ntt_forward(const binius_ntt* ntt, void* d_data, uint32_t log_len, uint32_t skip_early,
                       uint32_t skip_late, void* stream);
int binius_ntt_inverse(const binius_ntt* ntt, void* d_data, uint32_t log_len, uint32_t skip_early,
                       uint32_t skip_late, void* stream);

/* ------------------------------------------------------------------------------------------
 * Reed-Solomon encode.
 * Replaces: ReedSolomonCode::encode_batch (verifier/math/src/reed_solomon.rs:128-201).
 * d_msg: 2^(log_dim + log_batch) elements; d_codeword: 2^(log_dim + log_inv_rate + log_batch)
 * elements (must not alias d_msg).  The code's subspace is the NTT domain's first
 * log_dim + log_inv_rate basis elements.
 * ------------------------------------------------------------------------------------------ */
int binius_rs_encode_batch(const binius_ntt* ntt, const void* d_msg, uint32_t log_dim,
                           uint32_t log_inv_rate, uint32_t log_batch, void* d_codeword,
                           void* stream);

/* ------------------------------------------------------------------------------------------
 * Binary Merkle tree with SHA-256 leaves and the Binius SHA-256 node compression.
 * Replaces: BinaryMerkleTreeProver::commit / commit_iterated
 * (prover/prover/src/merkle_tree/prover.rs:93-118), binary_merkle_tree::build_from_iterator
 * (prover/prover/src/merkle_tree/binary_merkle_tree.rs:65-122), ParallelDigest for Sha256
 * (prover/prover/src/hash/parallel_digest.rs:145-173), Sha256Compression
 * (verifier/verifier/src/hash/compress.rs:32-57).
 * d_elems: 2^(log_leaves + log_batch) elements, leaf i = elements [i*2^log_batch, (i+1)*2^log_batch).
 * d_nodes: (2^(log_leaves+1) - 1) * 32 bytes, layers flat with the leaf digests first and the root
 * last (BinaryMerkleTree::inner_nodes).
 * ------------------------------------------------------------------------------------------ */
int binius_merkle_commit(const void* d_elems, uint32_t log_leaves, uint32_t log_batch,
                         void* d_nodes, void* stream);
/* Copies the Merkle branch of leaf `index` down to layer `layer_depth` (BinaryMerkleTree::branch,
 * binary_merkle_tree.rs:148-169) into h_branch ((log_leaves - layer_depth) * 32 bytes).
 * Synchronous. */
int binius_merkle_branch(const void* d_nodes, uint32_t log_leaves, uint64_t index,
                         uint32_t layer_depth, void* h_branch, void* stream);

/* Copies the 2^layer_depth digests of the tree's layer at depth layer_depth (0 = the root,
 * log_leaves = the leaf digests) into h_out (32 << layer_depth bytes): MerkleTreeProver::layer
 * (prover/prover/src/merkle_tree/mod.rs:50-55), BinaryMerkleTree::layer
 * (binary_merkle_tree.rs:142-150); BINIUS_E_ARG "IncorrectLayerDepth" when layer_depth >
 * log_leaves.  Synchronous. */
int binius_merkle_layer(const void* d_nodes, uint32_t log_leaves, uint32_t layer_depth,
                        void* h_out, void* stream);

/* ------------------------------------------------------------------------------------------
 * Vision-4 hash (the `-c vision4` Merkle hash, prover/examples/src/lib.rs:67-85).
 * binius_vision4_permute replaces the Vision-4 permutation over a batch of states
 * (verifier/verifier/src/hash/vision_4/permutation.rs:104-123; the prover's batch_permutation,
 * prover/prover/src/hash/vision_4/permutation.rs): d_states holds n states of 4 elements, permuted
 * in place.
 * binius_merkle_commit_vision4 is binius_merkle_commit with VisionHasherDigest leaves
 * (verifier/verifier/src/hash/vision_4/digest.rs:37-136; prover/prover/src/hash/vision_4/
 * digest.rs) and VisionCompression nodes (compression.rs:24-52; VisionParallelCompression,
 * prover/prover/src/hash/vision_4/compression.rs:34-145); same layout and arguments.
 * ------------------------------------------------------------------------------------------ */
int binius_vision4_permute(void* d_states, uint64_t n, void* stream);
int binius_merkle_commit_vision4(const void* d_elems, uint32_t log_leaves, uint32_t log_batch,
                                 void* d_nodes, void* stream);

/* ------------------------------------------------------------------------------------------
 * FRI folding.
 * binius_fri_fold_interleaved replaces fold_interleaved (prover/prover/src/fri/fold.rs:260-282):
 *   d_out[i] = <d_codeword[i*2^log_batch ..], eq_ind(h_challenges)>, 2^log_len outputs,
 *   log_batch <= 8 challenges.
 * binius_fri_fold_codeword replaces fold_codeword (prover/prover/src/fri/fold.rs:297-318) with
 *   fold_chunk / fold_pair (verifier/verifier/src/fri/fold.rs:20-99): 2^(log_len - n) outputs,
 *   n <= 8 challenges; the NTT supplies twiddle(log_len - 1 - k, .) for round k.
 * h_challenges are host arrays of 16-byte field elements.
 * ------------------------------------------------------------------------------------------ */
int binius_fri_fold_interleaved(const void* d_codeword, uint32_t log_len, uint32_t log_batch,
                                const void* h_challenges, void* d_out, void* stream);
int binius_fri_fold_codeword(const binius_ntt* ntt, const void* d_codeword, uint32_t log_len,
                             const void* h_challenges, uint32_t n_challenges, void* d_out,
                             void* stream);

/* Allocation-free form of binius_fri_fold_codeword, with no counterpart in the reference.  For
 * callers that may not allocate device memory themselves or let a library do it behind them: a
 * serving loop that admits requests by the free HBM it has budgeted, or a host that owns all device
 * memory in its own arena.  Same arguments and bit-identical output.  A fold over more than 4
 * challenges stages the codeword through a static 4 MiB device array (2^18 elements), so it accepts
 * log_len <= 22 in that case and returns BINIUS_E_ARG beyond; that array is reserved on every GPU
 * that loads the library until exit.  The first call on a device looks up the array's address; make
 * it before any stream capture.  All calls on a device share the array, so calls that overlap on
 * the GPU race.  Makes no cudaMalloc/cudaFree or other allocating call. */
int binius_fri_fold_codeword_noalloc(const binius_ntt* ntt, const void* d_codeword,
                                     uint32_t log_len, const void* h_challenges,
                                     uint32_t n_challenges, void* d_out, void* stream);

/* ------------------------------------------------------------------------------------------
 * FRI commit of an interleaved message: RS encode then Merkle commit with leaves of
 * 2^log_batch consecutive codeword symbols.
 * Replaces: fri::commit_interleaved (prover/prover/src/fri/commit.rs:25-75).
 * Writes the codeword (d_codeword) and tree (d_nodes); if h_root is not NULL the call
 * synchronizes `stream` and copies the 32-byte root there (CommitOutput::commitment).
 * ------------------------------------------------------------------------------------------ */
int binius_fri_commit_interleaved(const binius_ntt* ntt, const void* d_msg, uint32_t log_dim,
                                  uint32_t log_inv_rate, uint32_t log_batch, void* d_codeword,
                                  void* d_nodes, void* h_root, void* stream);

/* ------------------------------------------------------------------------------------------
 * Fiat-Shamir transcript: ProverTranscript<HasherChallenger<Sha256>>.
 * Replaces: ProverTranscript (verifier/transcript/src/transcript.rs:204-327), HasherChallenger
 * (verifier/transcript/src/fiat_shamir/hasher_challenger.rs:14-200), sample_bits_reader
 * (fiat_shamir/sampling.rs:34-50).  Host-side state; the proof is the tape of message() and
 * decommitment() bytes (ProverTranscript::finalize).  As the reference's finalize does, with the
 * environment variable BINIUS_DUMP_PROOF set binius_transcript_finalize also writes the proof
 * bytes to the file it names (BINIUS_E_ARG if that fails).
 * ------------------------------------------------------------------------------------------ */
typedef struct binius_transcript binius_transcript;

int binius_transcript_create(binius_transcript** out);
int binius_transcript_destroy(binius_transcript* t);
/* message(): written to the proof and observed by the challenger. */
int binius_transcript_message(binius_transcript* t, const void* h_bytes, size_t n);
/* decommitment(): written to the proof only. */
int binius_transcript_decommitment(binius_transcript* t, const void* h_bytes, size_t n);
/* observe(): observed only (switches the challenger to observing even when n == 0). */
int binius_transcript_observe(binius_transcript* t, const void* h_bytes, size_t n);
/* n sampled bytes; a B128 challenge is 16 bytes read as a little-endian u128. */
int binius_transcript_sample(binius_transcript* t, void* h_out, size_t n);
uint32_t binius_transcript_sample_bits(binius_transcript* t, uint32_t bits);
size_t binius_transcript_len(const binius_transcript* t);
int binius_transcript_finalize(const binius_transcript* t, void* h_out, size_t cap, size_t* len);

/* ------------------------------------------------------------------------------------------
 * 1-bit multilinear PCS (ring switching + BaseFold + FRI).
 * Replaces: OneBitPCSProver::{new, commit, prove} (prover/prover/src/pcs.rs:58-169) with
 * ring_switch::{fold_1b_rows_for_b128, fold_b128_elems_inplace} (ring_switch.rs:130-265),
 * BaseFoldProver (protocols/basefold.rs:33-166), FRIFoldProver / FRIQueryProver
 * (fri/fold.rs:30-244, fri/query.rs:18-134).
 * FRI parameters as FRIParams::new (verifier/verifier/src/fri/common.rs:35-57): the message is
 * 2^log_msg packed B128 elements (the B1 multilinear has log_msg + 7 variables).  The NTT must be
 * the RS code's domain (dimension >= log_msg - log_batch + log_inv_rate).
 * ------------------------------------------------------------------------------------------ */
typedef struct binius_pcs binius_pcs;
typedef struct binius_pcs_committed binius_pcs_committed;

int binius_pcs_create(const binius_ntt* ntt, uint32_t log_msg, uint32_t log_batch,
                      uint32_t log_inv_rate, const uint32_t* arities, uint32_t n_arities,
                      uint32_t n_queries, binius_pcs** out);
int binius_pcs_destroy(binius_pcs* pcs);
/* The Merkle hash of every commitment the PCS makes (the codeword and each FRI fold round):
 * BINIUS_MERKLE_SHA256 (StdDigest + StdCompression, the default) or BINIUS_MERKLE_VISION4
 * (VisionHasherDigest + VisionCompression, as Prover<_, VisionParallelCompression,
 * VisionHasherDigest> of prover/examples/src/lib.rs:43-46). */
#define BINIUS_MERKLE_SHA256 0u
#define BINIUS_MERKLE_VISION4 1u
int binius_pcs_set_merkle_hash(binius_pcs* pcs, uint32_t merkle_hash);
/* RS encode + Merkle commit of d_witness (2^log_msg elements); the codeword and tree stay on the
 * device in *out; h_root receives the 32-byte commitment.  Synchronous.  The buffers come from
 * the device's stream-ordered pool on `stream` and are released on it by
 * binius_pcs_committed_destroy, so the stream must outlive the committed object. */
int binius_pcs_commit(const binius_pcs* pcs, const void* d_witness, binius_pcs_committed** out,
                      void* h_root, void* stream);
int binius_pcs_committed_destroy(binius_pcs_committed* committed);
const void* binius_pcs_committed_codeword(const binius_pcs_committed* committed);
/* Proves the evaluation of the committed B1 multilinear at h_eval_point (log_msg + 7 field
 * elements), appending the proof to `transcript`.  Synchronous. */
int binius_pcs_prove(const binius_pcs* pcs, const binius_pcs_committed* committed,
                     const void* d_witness, const void* h_eval_point,
                     binius_transcript* transcript, void* stream);

/* ------------------------------------------------------------------------------------------
 * Constraint systems.
 * Replaces: ConstraintSystem::deserialize (verifier/core/src/constraint_system.rs:615-650) with
 * ValueVecLayout::validate / validate_and_prepare (:466-584); eval_operand
 * (verifier/core/src/verify.rs:14-35) used by build_bitand_witness / build_intmul_witness
 * (prover/prover/src/prove.rs:407-465).
 * The CS is parsed from the reference's v2 wire format, padded (AND to a power of two >= 8, MUL
 * to a power of two >= 1) and uploaded to `device` in CSR form.
 * ------------------------------------------------------------------------------------------ */
typedef struct binius_cs binius_cs;

int binius_cs_from_bytes(int device, const void* h_bytes, size_t len, binius_cs** out);
int binius_cs_destroy(binius_cs* cs);
/* h_out12: n_const, n_inout, n_witness, n_internal, offset_inout, offset_witness,
 * committed_total_len, n_scratch, padded AND count, padded MUL count, AND count, MUL count. */
int binius_cs_info(const binius_cs* cs, uint32_t* h_out12);
/* which = 0: AND operands a, b, c -> d_out[3 * n_and] (slot-major); which = 1: MUL operands a, b,
 * hi, lo -> d_out[4 * n_mul].  d_witness: committed_total_len u64 words. */
int binius_eval_operands(const binius_cs* cs, const void* d_witness, int which, void* d_out,
                         void* stream);

/* ------------------------------------------------------------------------------------------
 * AND reduction.
 * Replaces: build_bitand_witness + prove_bitand_reduction (prover/prover/src/prove.rs:329-431),
 * OblongZerocheckProver (prover/prover/src/and_reduction/prover.rs:74-276) with the univariate
 * round (sumcheck_round_messages.rs:62-136), FoldLookup (fold_lookup.rs:18-92) and the quadratic
 * MLE-check (protocols/sumcheck/quadratic_mle.rs, prove.rs:89-121).
 * Samples its challenges from and writes its messages to `transcript`.  h_out_meta receives
 * a_eval, b_eval, c_eval and the univariate challenge z (4 x 16 bytes); h_out_point the output
 * evaluation point (log2(padded AND count) x 16 bytes).  Synchronous.
 * ------------------------------------------------------------------------------------------ */
int binius_and_reduction_prove(const binius_cs* cs, const void* d_witness,
                               binius_transcript* transcript, void* h_out_meta,
                               void* h_out_point, void* stream);

/* ------------------------------------------------------------------------------------------
 * The prove entry.
 * Replaces: Verifier::setup's parameter choice (verifier/verifier/src/verify.rs:61-108: 96-bit
 * security, FRI arity from estimate_optimal_arity(log_code_len, 32, 16),
 * FRIParams::choose_with_constant_fold_arity), Prover::setup (prover/prover/src/prove.rs:95-121)
 * and Prover::prove (prove.rs:124-303): commit, IntMul, AND and shift reductions and the PCS
 * opening on one transcript.
 * binius_prover_setup keeps a reference to `cs`, which must outlive the prover.
 * binius_prover_prove: d_witness holds the committed_total_len witness words (the ValueVec's
 * combined witness) on the CS's device; the proof is appended to `transcript`.  Synchronous.
 * binius_prover_info h_out12: log_witness_elems, log_batch, log_inv_rate, n_queries, n_arities,
 * then up to 7 fold arities.
 * ------------------------------------------------------------------------------------------ */
typedef struct binius_prover binius_prover;

int binius_prover_setup(const binius_cs* cs, uint32_t log_inv_rate, binius_prover** out);
int binius_prover_destroy(binius_prover* prover);
/* setup_vision4 (prover/examples/src/lib.rs:67-85) = binius_prover_setup +
 * binius_prover_set_merkle_hash(prover, BINIUS_MERKLE_VISION4); not while a prove is in flight. */
int binius_prover_set_merkle_hash(binius_prover* prover, uint32_t merkle_hash);
int binius_prover_info(const binius_prover* prover, uint32_t* h_out12);
int binius_prover_prove(const binius_prover* prover, const void* d_witness,
                        binius_transcript* transcript, void* stream);
/* Prover set-up from wire bytes in one call: ConstraintSystem::deserialize (constraint_system.rs:
 * 615-650) on `device`, then Prover::setup, or Prover::setup_with_key_collection when h_kc (a
 * serialized KeyCollection v1, key_collection.rs:400-431) is given (prove.rs:81-121).  The prover
 * owns the constraint system and releases it in binius_prover_destroy. */
int binius_setup(int device, const void* h_cs_bytes, size_t cs_len, uint32_t log_inv_rate,
                 const void* h_kc, size_t kc_len, binius_prover** out);
/* Prover::prove (prove.rs:124-303) over a witness in host memory, returning the proof bytes
 * (ProverTranscript::finalize, verifier/transcript/src/transcript.rs:245-284): h_words holds the
 * ValueVec's committed_total_len words; the proof is appended to `transcript` (NULL = a fresh
 * ProverTranscript of the default challenger) and its whole tape copied to h_proof.  *len is
 * always set; a too-small buffer returns BINIUS_E_ARG.  Synchronous on `stream`; the witness copy
 * and every buffer of the proof are released before it returns. */
int binius_prove(const binius_prover* prover, const uint64_t* h_words, size_t n_words,
                 binius_transcript* transcript, void* h_proof, size_t cap, size_t* len,
                 void* stream);
/* Launch-shape choices of a prover's proofs, none of which changes a result (the arithmetic is
 * exact): h5 = {tail_log: sumcheck rounds on at most 2^tail_log elements run in one single-CTA
 * kernel (8..12, default 11); ntt_pass_layers: NTT layers fused per shared-memory pass (4..8,
 * default 8); merkle_leaf_fuse: a Merkle leaf CTA hashes 2^k leaves and compresses k layers above
 * them (5..8, default 8); merkle_node_fuse: a node CTA reduces 2^k inputs (5..9, default 9);
 * ntt_tile_bits: an NTT pass works on tiles of 2^k elements (9..12, default 12)}.
 * No reference counterpart (the reference's rayon code has no launch shapes).  Not while a prove
 * on the prover is in flight.
 * binius_prover_autotune measures them for the prover's statement shape: coordinate search over
 * the ranges above (tail_log 8..12, tile 10..12, ntt 6..8, leaf 6..8, node 7..9), each candidate
 * scored by the median CUDA-event time of `reps` whole proofs of d_witness on `stream` after a
 * warm-up proof, every candidate's proof checked byte for byte against the first one
 * (BINIUS_E_CUDA if one differs; the prover keeps its choices).  The winner is kept by the
 * prover, written to h_out5 when set, and cached for the process: provers set up later for the
 * same shape (words, AND and MUL counts, log_inv_rate, Merkle hash) start from it.  Synchronous;
 * runs 17 x (reps + 1) proofs at most. */
int binius_prover_get_tuning(const binius_prover* prover, uint32_t* h_out5);
int binius_prover_set_tuning(binius_prover* prover, const uint32_t* h_in5);
int binius_prover_autotune(binius_prover* prover, const void* d_witness, uint32_t reps,
                           void* stream, uint32_t* h_out5);
/* committed_total_len of the prover's constraint system (the witness length in words). */
uint64_t binius_prover_committed_words(const binius_prover* prover);
/* Estimate of the device memory one proof allocates while it runs (admission of concurrent
 * proofs): a static upper bound, or the largest footprint a proof of this prover has measured if
 * that is larger; no reference counterpart. */
uint64_t binius_prover_workspace_bytes(const binius_prover* prover);
/* Host wall-clock milliseconds of the calling thread's last prove's phases (the spans of prove.rs:164-300):
 * witness commit, IntMul, BitAnd, shift reduction, PCS opening.  No counterpart in the reference
 * beyond its tracing spans. */
int binius_prover_phase_ms(const binius_prover* prover, double* h_out5);

/* ------------------------------------------------------------------------------------------
 * Batched / served proving (no reference counterpart: the reference proves one statement per
 * call of Prover::prove, prover/prover/src/prove.rs:124-303, and per process in its CLI,
 * prover/examples/src/cli.rs:455-509).
 * A queue runs n_workers proving threads on `device`, each with its own CUDA stream, and admits
 * requests in FIFO order while the device memory it accounts for fits in hbm_budget_bytes (0 =
 * 90% of the free device memory at creation): the chunks every worker keeps for its next proof,
 * plus each running request's workspace estimate beyond its worker's chunks; idle workers give
 * their chunks back when the head request does not fit.  submit: `witness` holds the prover's
 * committed_total_len words, on the device (witness_on_device = 1) or on the host; it must stay
 * valid until wait returns.  A request whose estimate (binius_prover_workspace_bytes, plus the
 * witness copy for a host witness) exceeds the budget is refused with BINIUS_E_OOM.  A request
 * whose proof fails (a refused allocation: BINIUS_E_OOM) reports the error from wait; the queue
 * and its other requests carry on.  wait blocks until the request is done, copies its proof
 * (the finalized transcript of a fresh ProverTranscript) into h_proof and releases the ticket;
 * with a too-small buffer it sets *len, returns BINIUS_E_ARG and keeps the result.  h_times8
 * (optional): queued, proving and total milliseconds, then the proof's phase milliseconds
 * (commit, IntMul, AND, shift, PCS).  destroy cancels requests not yet admitted and finishes the
 * admitted ones.
 * ------------------------------------------------------------------------------------------ */
typedef struct binius_queue binius_queue;

int binius_queue_create(int device, uint32_t n_workers, uint64_t hbm_budget_bytes,
                        binius_queue** out);
int binius_queue_destroy(binius_queue* queue);
int binius_queue_submit(binius_queue* queue, const binius_prover* prover, const void* witness,
                        int witness_on_device, uint64_t* ticket);
int binius_queue_poll(binius_queue* queue, uint64_t ticket, int* done);
int binius_queue_wait(binius_queue* queue, uint64_t ticket, void* h_proof, size_t cap,
                      size_t* len, double* h_times8);
/* h_out4: budget, accounted bytes now, their peak since creation, finished requests. */
int binius_queue_stats(binius_queue* queue, uint64_t* h_out4);

/* ------------------------------------------------------------------------------------------
 * Wire formats around a prove call (load-prove serving).
 * Replaces: ValuesData::{serialize, deserialize} (verifier/core/src/constraint_system.rs:939-963,
 * version 1), Proof::{serialize, deserialize} (:1066-1098, version 1) and ValueVec::new_from_data
 * (:803-823), as used by the reference's prover binary (prover/examples/src/bin/prover.rs:46-99).
 * Encoders write at most `cap` bytes and always set *len; a too-small buffer returns BINIUS_E_ARG.
 * Decoders reject another version with BINIUS_E_ARG ("InvalidConstruction: Witness::version",
 * "... Proof::version") and truncated input with BINIUS_E_ARG ("NotEnoughBytes: ...").
 * binius_value_vec_from_data requires n_public + n_non_public == committed_total_len
 * ("ValueVecLenMismatch") and writes committed_total_len + n_scratch words, the scratch zeroed.
 * The proof's challenger type for this library's transcript is "HasherChallenger<Sha256>".
 * ------------------------------------------------------------------------------------------ */
int binius_values_data_encode(const uint64_t* h_words, size_t n_words, void* h_out, size_t cap,
                              size_t* len);
int binius_values_data_decode(const void* h_bytes, size_t len, uint64_t* h_words, size_t cap,
                              size_t* n_words);
int binius_proof_encode(const void* h_transcript, size_t n_bytes, const char* challenger,
                        void* h_out, size_t cap, size_t* len);
int binius_proof_decode(const void* h_bytes, size_t len, void* h_transcript, size_t cap,
                        size_t* n_bytes, char* h_challenger, size_t ch_cap);
int binius_value_vec_from_data(const binius_cs* cs, const uint64_t* h_public, size_t n_public,
                               const uint64_t* h_non_public, size_t n_non_public,
                               uint64_t* h_out);

/* ------------------------------------------------------------------------------------------
 * Shift-reduction KeyCollection (setup-time precomputation of the shift reduction's term index).
 * Replaces: build_key_collection + KeyCollection::serialize (prover/prover/src/protocols/shift/
 * key_collection.rs:238-312, 381-398, version 1), Prover::key_collection (prover/prover/src/
 * prove.rs:120-122) and Prover::setup_with_key_collection (:89-115) with
 * KeyCollection::deserialize (key_collection.rs:400-431).
 * binius_key_collection_from_cs_bytes builds the collection of a v2 constraint system on the host
 * alone (no device needed); binius_cs_key_collection builds it for an uploaded one.  Both write
 * the reference's bytes exactly, at most `cap` of them, and always set *len.
 * binius_cs_load_key_collection replaces the constraint system's device term table with the
 * terms a serialized collection describes; it rejects another version ("InvalidConstruction:
 * KeyCollection::version"), truncated or trailing bytes, and a collection that does not describe
 * this constraint system's terms, with BINIUS_E_ARG and the table unchanged.  Not while a prove
 * call on `cs` is in flight.
 * binius_prover_setup_with_key_collection = binius_cs_load_key_collection + binius_prover_setup.
 * ------------------------------------------------------------------------------------------ */
int binius_key_collection_from_cs_bytes(const void* h_cs_bytes, size_t cs_len, void* h_out,
                                        size_t cap, size_t* len);
int binius_cs_key_collection(const binius_cs* cs, void* h_out, size_t cap, size_t* len);
int binius_cs_load_key_collection(binius_cs* cs, const void* h_bytes, size_t len);
int binius_prover_setup_with_key_collection(binius_cs* cs, uint32_t log_inv_rate,
                                            const void* h_kc, size_t kc_len, binius_prover** out);

/* ------------------------------------------------------------------------------------------
 * Witness evaluation (the frontend's evaluation form) on the device.
 * Replaces: EvalForm::evaluate / Interpreter::run (verifier/frontend/src/compiler/eval_form/
 * mod.rs:68-78, interpreter.rs:113-520) with the Word arithmetic of verifier/core/src/word.rs,
 * over a batch of value vectors at once.
 * binius_eval_form_create decodes the bytecode (builder.rs encoding) for value vectors of
 * n_values words and level-schedules it; BINIUS_E_ARG for an unknown opcode, a register >=
 * n_values, a truncated instruction, a shift amount >= 64 or a hint call (0x80: hint handlers
 * are host code and are not run here).  binius_eval_form_info: out5 = instructions, levels,
 * widest level, assertions, register accesses (sources + destinations over the program).
 * binius_eval_form_evaluate runs it over d_values, n_values * batch words laid out register-major
 * (word r of instance i at d_values[r * batch + i]), in place and asynchronously on `stream`.
 * d_fail_count[i] receives instance i's number of failed assertions and d_first_fail[i] its
 * earliest failing assertion in program order as (instruction index << 32 | assertion id), or
 * all ones.
 * binius_values_transpose: d_dst[c * rows + r] = d_src[r * cols + c] for 64-bit words (between
 * instance-major value vectors and the register-major batch).
 * ------------------------------------------------------------------------------------------ */
typedef struct binius_eval_form binius_eval_form;

int binius_eval_form_create(const void* h_bytecode, size_t len, uint64_t n_values,
                            binius_eval_form** out);
int binius_eval_form_info(const binius_eval_form* ef, uint64_t* out5);
int binius_eval_form_evaluate(const binius_eval_form* ef, void* d_values, uint32_t batch,
                              uint32_t* d_fail_count, uint64_t* d_first_fail, void* stream);
int binius_eval_form_destroy(binius_eval_form* ef);
int binius_values_transpose(const void* d_src, uint64_t rows, uint64_t cols, void* d_dst,
                            void* stream);

/* ------------------------------------------------------------------------------------------
 * Integer multiplication reduction.
 * Replaces: build_intmul_witness + prove_intmul_reduction (prover/prover/src/prove.rs:374-391,
 * 432-470), intmul Witness (protocols/intmul/witness.rs:47-270) and IntMulProver::prove
 * (protocols/intmul/prove.rs:93-509).
 * Samples from and writes to `transcript`.  h_out_point receives the output point
 * (log2(padded MUL count) x 16 bytes), h_out_evals the 64 bit-column evaluations of a, b, c_lo and
 * c_hi in that order (4 x 64 x 16 bytes).  Synchronous.
 * ------------------------------------------------------------------------------------------ */
int binius_intmul_reduction_prove(const binius_cs* cs, const void* d_witness,
                                  binius_transcript* transcript, void* h_out_point,
                                  void* h_out_evals, void* stream);

/* ------------------------------------------------------------------------------------------
 * Shift reduction.
 * Replaces: shift::prove (prover/prover/src/protocols/shift/prove.rs:103-153) with
 * build_key_collection (key_collection.rs:246-312), prove_phase_1 (phase_1.rs:43-139),
 * build_h_parts / build_monster_multilinear (monster.rs:34-219) and prove_phase_2
 * (phase_2.rs:56-160) over InOutCheckProver (protocols/inout_check.rs:19-211).
 * h_and_data: AND OperatorData as 16-byte elements a_eval, b_eval, c_eval, r_zhat', then r_x'
 * (log2(padded AND count) elements).  h_mul_data: a_eval, b_eval, lo_eval, hi_eval, r_zhat', then
 * r_x' (log2(padded MUL count) elements).  The public segment is the first offset_witness words.
 * h_out_point receives r_j ++ r_y (6 + log2(committed_total_len) elements), h_out_eval the witness
 * evaluation there.  Samples from and writes to `transcript`.  Synchronous.
 * ------------------------------------------------------------------------------------------ */
int binius_shift_reduction_prove(const binius_cs* cs, const void* d_witness,
                                 binius_transcript* transcript, const void* h_and_data,
                                 const void* h_mul_data, void* h_out_point, void* h_out_eval,
                                 void* stream);

/* ------------------------------------------------------------------------------------------
 * FRI parameters (verifier/verifier/src/fri/common.rs:64-219).
 * ------------------------------------------------------------------------------------------ */
uint32_t binius_fri_n_test_queries(uint32_t security_bits, uint32_t log_inv_rate);
uint32_t binius_fri_estimate_optimal_arity(uint32_t log_block_length, uint32_t digest_size,
                                           uint32_t field_size);

/* ------------------------------------------------------------------------------------------
 * Round-by-round sumcheck provers: the SumcheckProver trait (prover/prover/src/protocols/
 * sumcheck/common.rs:29-101) -- n_vars, execute() -> RoundCoeffs, fold(challenge), finish() ->
 * multilinear evaluations -- and MleCheckProver::eval_point (common.rs:88-101), for
 *   BivariateProductSumcheckProver::new([a, b], sum) (sumcheck/bivariate_product.rs:17-119);
 *   QuadraticMleCheckProver::new([a, b, c], a*b - c, a*b, eval_point, eval_claim)
 *     (sumcheck/quadratic_mle.rs:21-229; the AND reduction's composition, prove.rs:89-121);
 *   InOutCheckProver::new(witness, eval_point) (protocols/inout_check.rs:19-221), the public
 *     segment being the witness's first 2^log_public values.
 * The multilinears (2^n_vars elements each, d_* device buffers) are folded in place by fold
 * (fold_highest_var_inplace), so they must stay valid and untouched until finish; the prover
 * keeps its own eq expansion.  execute writes the round polynomial's coefficients, lowest degree
 * first, to h_coeffs (3 elements for the degree-2 provers, 2 for InOut) and their count to
 * *n_coeffs; finish writes the multilinears' values at the challenge point (2 for the bivariate,
 * 3 for the quadratic MLE-check, 1 for InOut).  Out-of-order calls return BINIUS_E_ARG with
 * "ExpectedFold" / "ExpectedExecute" (sumcheck/error.rs).  All calls synchronize `stream`.
 * ------------------------------------------------------------------------------------------ */
typedef struct binius_sumcheck binius_sumcheck;

int binius_sumcheck_bivariate_create(void* d_a, void* d_b, uint32_t log_len, const void* h_sum,
                                     void* stream, binius_sumcheck** out);
int binius_sumcheck_bivariate_execute(binius_sumcheck* prover, void* h_coeffs,
                                      uint32_t* n_coeffs);
int binius_sumcheck_bivariate_fold(binius_sumcheck* prover, const void* h_challenge);
int binius_sumcheck_bivariate_finish(binius_sumcheck* prover, void* h_evals2);

int binius_sumcheck_quadratic_mle_create(void* d_a, void* d_b, void* d_c, uint32_t n_vars,
                                         const void* h_eval_point, const void* h_eval_claim,
                                         void* stream, binius_sumcheck** out);
int binius_sumcheck_quadratic_mle_execute(binius_sumcheck* prover, void* h_coeffs,
                                          uint32_t* n_coeffs);
int binius_sumcheck_quadratic_mle_fold(binius_sumcheck* prover, const void* h_challenge);
int binius_sumcheck_quadratic_mle_finish(binius_sumcheck* prover, void* h_evals3);
int binius_sumcheck_quadratic_mle_eval_point(const binius_sumcheck* prover, void* h_out);

int binius_sumcheck_inout_create(void* d_witness, uint32_t log_len, const void* h_eval_point,
                                 uint32_t log_public, void* stream, binius_sumcheck** out);
int binius_sumcheck_inout_execute(binius_sumcheck* prover, void* h_coeffs, uint32_t* n_coeffs);
int binius_sumcheck_inout_fold(binius_sumcheck* prover, const void* h_challenge);
int binius_sumcheck_inout_finish(binius_sumcheck* prover, void* h_eval);
int binius_sumcheck_inout_eval_point(const binius_sumcheck* prover, void* h_out);

/* SumcheckProver::n_vars, and the release of any of the three. */
uint32_t binius_sumcheck_n_vars(const binius_sumcheck* prover);
int binius_sumcheck_destroy(binius_sumcheck* prover);

/* The bivariate product round's device kernels on their own (the prove path's fused form of
 * BivariateProductSumcheckProver::execute / fold, bivariate_product.rs:43-95;
 * fold_highest_var_inplace, verifier/math/src/multilinear/fold.rs:14-29).  d_a, d_b: 2^log_len
 * elements each.  round_evals: d_out2 = (y_1, y_inf) = (sum a_hi b_hi, sum (a_lo + a_hi)(b_lo +
 * b_hi)).  fold_round_evals: folds the top variable of both by h_r in place (a[i] += r (a[i + half]
 * - a[i])) and writes the next round's (y_1, y_inf) on the 2^(log_len-1) folded values.  d_out2
 * stays on the device; both are asynchronous on `stream`. */
int binius_bivariate_round_evals(const void* d_a, const void* d_b, uint32_t log_len, void* d_out2,
                                 void* stream);
int binius_bivariate_fold_round_evals(void* d_a, void* d_b, uint32_t log_len, const void* h_r,
                                      void* d_out2, void* stream);

/* Elementwise GF(2^128) products d_out[i] = d_a[i] * d_b[i] (kernel-level check of the field
 * multiplier; BinaryField128bGhash::mul, verifier/field/src/ghash.rs:188-194). */
int binius_gf_mul_batch(const void* d_a, const void* d_b, void* d_out, uint64_t n, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BINIUS_GPU_H */
