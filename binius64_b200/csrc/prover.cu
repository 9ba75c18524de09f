// The top-level prove entry on the device: Verifier::setup's parameter choice
// (verifier/verifier/src/verify.rs:61-108), Prover::setup (prover/prover/src/prove.rs:95-121) and
// Prover::prove (prove.rs:124-303).
//
// The witness stays on the device for the whole proof: its committed words are the packed
// multilinear of the PCS (pack_witness reads word pairs as little-endian 128-bit elements, which
// is their memory layout), the operand columns of the reductions are evaluated from it, and the
// shift reduction and the PCS opening read it in place.  The NTT is the standard-basis domain of
// dim log_code_len; the Reed-Solomon code of the FRI parameters uses its first
// log_dim + log_inv_rate layers.
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <mutex>
#include <vector>

#include "cs.h"
#include "internal.h"
#include "kernels.h"
#include "reductions.h"
#include "transcript.h"

using namespace bgpu;

struct binius_prover {
  const binius_cs* cs = nullptr;
  binius_cs* owned_cs = nullptr;  // binius_setup: the constraint system lives with the prover
  binius_ntt* ntt = nullptr;
  binius_pcs* pcs = nullptr;
  uint32_t log_inv_rate = 0, log_witness_elems = 0, log_batch = 0, n_queries = 0;
  std::vector<uint32_t> arities;
  // largest device footprint (arena chunk bytes) a proof of this prover has taken from an empty
  // arena; raises binius_prover_workspace_bytes when the static estimate is low
  mutable std::atomic<uint64_t> footprint{0};
  // launch-shape choices of its proofs (binius_prover_autotune); not changed while proving
  Tuning tuning;
  uint32_t merkle_hash = 0;
};

namespace {

// Statement shape -> the choices binius_prover_autotune measured for it, so that provers set up
// later for the same shape start from them.
struct ShapeKey {
  uint64_t words, n_and, n_mul;
  uint32_t log_inv_rate, merkle_hash;
  bool operator==(const ShapeKey& o) const {
    return words == o.words && n_and == o.n_and && n_mul == o.n_mul &&
           log_inv_rate == o.log_inv_rate && merkle_hash == o.merkle_hash;
  }
};
std::mutex g_tuned_mu;
std::vector<std::pair<ShapeKey, Tuning>> g_tuned;

ShapeKey shape_of(const binius_prover* P) {
  return ShapeKey{P->cs->committed_total_len, P->cs->and_ops.n_constraints,
                  P->cs->mul_ops.n_constraints, P->log_inv_rate, P->merkle_hash};
}

// The choices measured for P's shape, if any.
void load_tuned(binius_prover* P) {
  std::lock_guard<std::mutex> lock(g_tuned_mu);
  const ShapeKey k = shape_of(P);
  for (const auto& e : g_tuned)
    if (e.first == k) {
      P->tuning = e.second;
      return;
    }
}

void store_tuned(const binius_prover* P) {
  std::lock_guard<std::mutex> lock(g_tuned_mu);
  const ShapeKey k = shape_of(P);
  for (auto& e : g_tuned)
    if (e.first == k) {
      e.second = P->tuning;
      return;
    }
  g_tuned.emplace_back(k, P->tuning);
}

bool valid_tuning(const Tuning& t) {
  return t.tail_log >= 8 && t.tail_log <= 12 && t.ntt_pass_layers >= 4 &&
         t.ntt_pass_layers <= 8 && t.merkle_leaf_fuse >= 5 && t.merkle_leaf_fuse <= 8 &&
         t.merkle_node_fuse >= 5 && t.merkle_node_fuse <= 9 && t.ntt_tile_bits >= 9 &&
         t.ntt_tile_bits <= 12;
}

void tuning_out(const Tuning& t, uint32_t* out5) {
  out5[0] = t.tail_log;
  out5[1] = t.ntt_pass_layers;
  out5[2] = t.merkle_leaf_fuse;
  out5[3] = t.merkle_node_fuse;
  out5[4] = t.ntt_tile_bits;
}

}  // namespace

namespace bgpu {
void prover_note_footprint(const binius_prover* P, uint64_t bytes) {
  uint64_t cur = P->footprint.load(std::memory_order_relaxed);
  while (bytes > cur && !P->footprint.compare_exchange_weak(cur, bytes)) {
  }
}
}  // namespace bgpu

namespace {

// Host wall-clock milliseconds of the calling thread's last prove: commit, IntMul, AND, shift,
// PCS (per thread, so that concurrent proofs on one prover do not share it).
thread_local double t_phase_ms[5] = {0, 0, 0, 0, 0};

constexpr uint32_t kSecurityBits = 96;  // verifier/verifier/src/verify.rs:39
constexpr uint32_t kDigestSize = 32;    // SHA-256
constexpr uint32_t kFieldSize = 16;     // B128

uint32_t log2_ceil(uint64_t n) {
  uint32_t r = 0;
  while ((1ull << r) < n) r++;
  return r;
}

hu128 h128(const void* p) {
  hu128 v;
  memcpy(&v, p, 16);
  return v;
}

// make_final_claim (prove.rs:230-243): sum_i evals[i] l_tilde[i].
hu128 final_claim(const std::vector<hu128>& evals, const hu128* L) {
  hu128 acc = 0;
  for (int i = 0; i < 64; i++) acc ^= host_gf_mul(evals[i], L[i]);
  return acc;
}

}  // namespace

extern "C" {

int binius_prover_setup(const binius_cs* cs, uint32_t log_inv_rate, binius_prover** out) {
  BGPU_ARG(cs && out, "NULL argument");
  *out = nullptr;
  BGPU_ARG(log_inv_rate >= 1 && log_inv_rate <= 4, "log_inv_rate must be in [1, 4]");
  binius_prover* P = new binius_prover();
  P->cs = cs;
  P->log_inv_rate = log_inv_rate;
  uint32_t log_words = log2_ceil(cs->committed_total_len);
  if (log_words < 1) log_words = 1;
  P->log_witness_elems = log_words - 1;
  const uint32_t log_code_len = P->log_witness_elems + log_inv_rate;
  // FRIParams::choose_with_constant_fold_arity (verifier/verifier/src/fri/common.rs:64-115)
  const uint32_t arity = binius_fri_estimate_optimal_arity(log_code_len, kDigestSize, kFieldSize);
  P->log_batch = P->log_witness_elems < arity ? P->log_witness_elems : arity;
  P->n_queries = binius_fri_n_test_queries(kSecurityBits, log_inv_rate);
  const uint32_t rs_log_len = P->log_witness_elems - P->log_batch + log_inv_rate;
  uint32_t term = log2_ceil(P->n_queries);
  if (term < log_inv_rate) term = log_inv_rate;
  if (term > rs_log_len) term = rs_log_len;
  P->arities.assign((rs_log_len - term) / arity, arity);
  if ((rs_log_len - term) % arity) P->arities.push_back((rs_log_len - term) % arity);
  int rc = binius_ntt_create(cs->device, nullptr, log_code_len, &P->ntt);
  if (!rc)
    rc = binius_pcs_create(P->ntt, P->log_witness_elems, P->log_batch, log_inv_rate,
                           P->arities.data(), (uint32_t)P->arities.size(), P->n_queries, &P->pcs);
  if (rc) {
    binius_prover_destroy(P);
    return rc;
  }
  load_tuned(P);
  *out = P;
  return clear_error();
}

int binius_prover_set_merkle_hash(binius_prover* P, uint32_t merkle_hash) {
  BGPU_ARG(P != nullptr, "NULL argument");
  if (int rc = binius_pcs_set_merkle_hash(P->pcs, merkle_hash)) return rc;
  P->merkle_hash = merkle_hash;
  P->tuning = Tuning();
  load_tuned(P);
  return clear_error();
}

int binius_prover_get_tuning(const binius_prover* P, uint32_t* h_out5) {
  BGPU_ARG(P && h_out5, "NULL argument");
  tuning_out(P->tuning, h_out5);
  return clear_error();
}

int binius_prover_set_tuning(binius_prover* P, const uint32_t* h_in5) {
  BGPU_ARG(P && h_in5, "NULL argument");
  Tuning t;
  t.tail_log = h_in5[0];
  t.ntt_pass_layers = h_in5[1];
  t.merkle_leaf_fuse = h_in5[2];
  t.merkle_node_fuse = h_in5[3];
  t.ntt_tile_bits = h_in5[4];
  BGPU_ARG(valid_tuning(t),
           "tuning out of range: tail_log 8..12, ntt_pass_layers 4..8, merkle_leaf_fuse 5..8, "
           "merkle_node_fuse 5..9, ntt_tile_bits 9..12");
  P->tuning = t;
  return clear_error();
}

int binius_prover_destroy(binius_prover* P) {
  if (!P) return BINIUS_OK;
  binius_pcs_destroy(P->pcs);
  binius_ntt_destroy(P->ntt);
  binius_cs_destroy(P->owned_cs);
  delete P;
  return BINIUS_OK;
}

int binius_setup(int device, const void* h_cs_bytes, size_t cs_len, uint32_t log_inv_rate,
                 const void* h_kc, size_t kc_len, binius_prover** out) {
  BGPU_ARG(h_cs_bytes && out, "NULL argument");
  *out = nullptr;
  binius_cs* cs = nullptr;
  if (int rc = binius_cs_from_bytes(device, h_cs_bytes, cs_len, &cs)) return rc;
  binius_prover* P = nullptr;
  int rc = h_kc ? binius_prover_setup_with_key_collection(cs, log_inv_rate, h_kc, kc_len, &P)
                : binius_prover_setup(cs, log_inv_rate, &P);
  if (rc) {
    binius_cs_destroy(cs);
    return rc;
  }
  P->owned_cs = cs;
  *out = P;
  return clear_error();
}

int binius_prover_info(const binius_prover* P, uint32_t* h_out12) {
  BGPU_ARG(P && h_out12, "NULL argument");
  memset(h_out12, 0, 12 * sizeof(uint32_t));
  h_out12[0] = P->log_witness_elems;
  h_out12[1] = P->log_batch;
  h_out12[2] = P->log_inv_rate;
  h_out12[3] = P->n_queries;
  h_out12[4] = (uint32_t)P->arities.size();
  for (size_t i = 0; i < P->arities.size() && i < 7; i++) h_out12[5 + i] = P->arities[i];
  return clear_error();
}

uint64_t binius_prover_committed_words(const binius_prover* P) {
  return P ? P->cs->committed_total_len : 0;
}

uint64_t binius_prover_workspace_bytes(const binius_prover* P) {
  if (!P) return 0;
  const binius_cs* cs = P->cs;
  const uint64_t words = cs->committed_total_len, n_and = cs->and_ops.n_constraints;
  const uint64_t n_mul = cs->mul_ops.n_constraints;
  const uint64_t code = 16ull << (P->log_witness_elems + P->log_inv_rate);
  // codeword + tree, AND columns / folds / eq, shift W / M / g parts, PCS fold buffers, IntMul
  // trees: the stream-ordered allocations of one proof, which its arena never frees before the
  // end, rounded up by one arena chunk; or, if larger, what a proof of this prover took
  const uint64_t est = 2 * code + 96 * n_and + 80 * words + 12288 * n_mul + (72ull << 20);
  const uint64_t seen = P->footprint.load(std::memory_order_relaxed);
  return est > seen ? est : seen;
}

int binius_prover_phase_ms(const binius_prover* P, double* h_out5) {
  BGPU_ARG(P && h_out5, "NULL argument");
  memcpy(h_out5, t_phase_ms, sizeof(t_phase_ms));
  return clear_error();
}

int binius_prover_prove(const binius_prover* P, const void* d_witness,
                        binius_transcript* transcript, void* stream) {
  BGPU_ARG(P && d_witness && transcript, "NULL argument");
  const binius_cs* cs = P->cs;
  cudaStream_t s = as_stream(stream);
  const uint64_t* words = static_cast<const uint64_t*>(d_witness);
  Transcript& t = transcript->t;

  // every device buffer of the proof comes from one arena on s, released at the end
  ArenaScope arena(s, false);
  TuningScope tuned(P->tuning);
  const bool fresh_arena = arena_held_bytes() == 0;
  typedef std::chrono::steady_clock Clock;
  auto t0 = Clock::now();
  auto lap = [&](int phase) {
    const auto now = Clock::now();
    t_phase_ms[phase] = std::chrono::duration<double, std::milli>(now - t0).count();
    t0 = now;
  };
  // The opening host round trip: the commitment's root -- and, with one MUL constraint, that
  // constraint's four operand words, after which the IntMul reduction needs no device work --
  // ride back through the pinned early buffer while the device goes on with the AND reduction's
  // operand evaluation, queued behind the commit (it needs no challenge).
  const bool single_mul = cs->mul_ops.n_constraints == 1;
  uint8_t* early = nullptr;
  if (int rc = early_read_buffer(&early)) return rc;
  if (single_mul) {
    uint64_t* d_cols = nullptr;
    BGPU_CUDA(dev_alloc(&d_cols, 32, s));
    if (int rc = eval_operands(cs->mul_ops, words, d_cols, s)) return rc;
    BGPU_CUDA(cudaMemcpyAsync(early, d_cols, 32, cudaMemcpyDeviceToHost, s));
  }
  // [phase] Witness Commit
  binius_pcs_committed* committed = nullptr;
  int rc = pcs_commit_enqueue(P->pcs, d_witness, &committed, s);
  if (rc) return rc;
  AndPrep ap;
  do {
    cudaError_t e = cudaMemcpyAsync(early + 32, pcs_committed_root(committed), 32,
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = stream_mark(s);
    if (e != cudaSuccess) { rc = cuda_error(e, "commitment root read"); break; }
    if ((rc = and_reduction_begin(cs, words, ap, s))) break;
    if ((e = mark_wait()) != cudaSuccess) { rc = cuda_error(e, "commitment root read"); break; }
    pcs_committed_set_root(committed, early + 32);
    t.message(early + 32, 32);
    lap(0);
    // [phase] IntMul Reduction
    IntMulResult im;
    if (single_mul) {
      uint64_t w[4];  // CSR slots a, b, hi, lo
      memcpy(w, early, 32);
      rc = intmul_single_from_words(w[0], w[1], w[3], w[2], t, im);
    } else {
      rc = intmul_reduction_prove(cs, words, t, im, s);
    }
    if (rc) break;
    lap(1);
    // [phase] BitAnd Reduction
    AndResult ao;
    if ((rc = and_reduction_finish(cs, ap, t, ao, s))) break;
    lap(2);
    // OperatorData of both operations at the AND reduction's r_zhat'
    ShiftOperatorData band, bmul;
    band.evals = {ao.a_eval, ao.b_eval, ao.c_eval};
    band.r_zhat = ao.z;
    band.r_x = ao.eval_point;
    hu128 L[64];
    lagrange_phi(6, ao.z, L);
    bmul.evals = {final_claim(im.a_evals, L), final_claim(im.b_evals, L),
                  final_claim(im.c_lo_evals, L), final_claim(im.c_hi_evals, L)};
    bmul.r_zhat = ao.z;
    bmul.r_x = im.eval_point;
    // [phase] Shift Reduction
    ShiftResult sh;
    if ((rc = shift_reduction_prove(cs, words, t, band, bmul, sh, s))) break;
    lap(3);
    // [phase] PCS Opening at r_j ++ r_y
    rc = binius_pcs_prove(P->pcs, committed, d_witness, sh.point.data(), transcript, stream);
    lap(4);
  } while (0);
  if (ap.words) and_prep_free(ap, s);  // a failure before the AND reduction ran
  binius_pcs_committed_destroy(committed);
  if (!rc && fresh_arena) prover_note_footprint(P, arena_held_bytes());
  return rc ? rc : clear_error();
}

// Coordinate search over the launch-shape choices: each knob in turn takes every value in its range
// with the others at their best so far; a candidate's score is the median CUDA-event time of
// `reps` proofs (after one warm-up proof), the whole proof on the stream as the bench times it.
// Every candidate's proof must equal the proof under the starting choices byte for byte (the
// choices change no arithmetic); a difference is reported as an error and the starting choices
// are kept.
int binius_prover_autotune(binius_prover* P, const void* d_witness, uint32_t reps, void* stream,
                           uint32_t* h_out5) {
  BGPU_ARG(P && d_witness, "NULL argument");
  reps = std::max(1u, std::min(reps, 64u));
  cudaStream_t s = as_stream(stream);
  const Tuning start = P->tuning;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  BGPU_CUDA(cudaEventCreate(&e0));
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    return cuda_error(ce, "cudaEventCreate");
  }
  std::vector<uint8_t> ref;
  auto score = [&](const Tuning& t, double* ms) -> int {
    P->tuning = t;
    std::vector<float> times;
    for (uint32_t r = 0; r <= reps; r++) {
      binius_transcript tr;
      BGPU_CUDA(cudaEventRecord(e0, s));
      if (int rc = binius_prover_prove(P, d_witness, &tr, stream)) return rc;
      BGPU_CUDA(cudaEventRecord(e1, s));
      BGPU_CUDA(cudaEventSynchronize(e1));
      float t_ms = 0;
      BGPU_CUDA(cudaEventElapsedTime(&t_ms, e0, e1));
      if (r > 0) times.push_back(t_ms);
      const std::vector<uint8_t>& tape = tr.t.tape();
      if (ref.empty()) ref = tape;
      else if (tape != ref)
        return set_error(BINIUS_E_CUDA, "autotune: a launch shape changed the proof bytes");
    }
    std::sort(times.begin(), times.end());
    *ms = times[times.size() / 2];
    return BINIUS_OK;
  };
  int rc = BINIUS_OK;
  Tuning best = start;
  double best_ms = 0;
  rc = score(best, &best_ms);
  struct Knob {
    uint32_t Tuning::*field;
    uint32_t lo, hi;
  };
  const Knob knobs[5] = {{&Tuning::tail_log, 8, 12},
                         {&Tuning::ntt_tile_bits, 10, 12},
                         {&Tuning::ntt_pass_layers, 6, 8},
                         {&Tuning::merkle_leaf_fuse, 6, 8},
                         {&Tuning::merkle_node_fuse, 7, 9}};
  for (const Knob& k : knobs) {
    for (uint32_t v = k.lo; v <= k.hi && !rc; v++) {
      if (best.*(k.field) == v) continue;
      Tuning cand = best;
      cand.*(k.field) = v;
      double ms = 0;
      rc = score(cand, &ms);
      if (!rc && ms < best_ms) {
        best = cand;
        best_ms = ms;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    P->tuning = start;
    return rc;
  }
  P->tuning = best;
  store_tuned(P);
  if (h_out5) tuning_out(best, h_out5);
  return clear_error();
}

int binius_prove(const binius_prover* P, const uint64_t* h_words, size_t n_words,
                 binius_transcript* transcript, void* h_proof, size_t cap, size_t* len,
                 void* stream) {
  BGPU_ARG(P && h_words && len, "NULL argument");
  *len = 0;
  BGPU_ARG(n_words == P->cs->committed_total_len,
           "witness length != the constraint system's committed_total_len");
  int prev = 0;
  BGPU_CUDA(cudaGetDevice(&prev));
  if (prev != P->cs->device) BGPU_CUDA(cudaSetDevice(P->cs->device));
  cudaStream_t s = as_stream(stream);
  binius_transcript fresh;
  binius_transcript* t = transcript ? transcript : &fresh;
  int rc = BINIUS_OK;
  {
    // the witness copy and every buffer of the proof come from one arena, released at the end
    ArenaScope arena(s, false);
    void* d_w = nullptr;
    cudaError_t e = dev_alloc(&d_w, 8 * n_words, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_w, h_words, 8 * n_words, cudaMemcpyHostToDevice, s);
    rc = e != cudaSuccess ? cuda_error(e, "witness upload")
                          : binius_prover_prove(P, d_w, t, stream);
    if (!rc) {
      *len = t->t.tape().size();
      if (cap < *len || (!h_proof && *len))
        rc = set_error(BINIUS_E_ARG, "proof buffer too small (len set)");
      else if (*len)
        memcpy(h_proof, t->t.tape().data(), *len);
    }
    stream_wait(s);
  }
  if (prev != P->cs->device) cudaSetDevice(prev);
  return rc ? rc : clear_error();
}

}  // extern "C"
