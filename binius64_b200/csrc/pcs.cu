// FRI-Binius 1-bit multilinear polynomial commitment: commit and the evaluation proof.
//
// Host driver of OneBitPCSProver (prover/prover/src/pcs.rs:58-169): the protocol's sequential
// Fiat-Shamir steps run on the host (transcript.h) while every data-parallel step runs on the GPU
// over device-resident buffers: RS encode + Merkle commit, the eq tensor of the evaluation point's
// suffix, the ring-switch row fold, the ring-switch equality indicator, the BaseFold rounds
// (bivariate product sumcheck, protocols/basefold.rs:130-166) interleaved with FRI folds and
// Merkle commits of the folded codewords (fri/fold.rs:117-175), and the FRI query openings
// (fri/fold.rs:221-244, fri/query.rs:51-134) gathered on the device into one buffer.
#include <string.h>

#include <algorithm>
#include <vector>

#include "dev_transcript.cuh"
#include "internal.h"
#include "kernels.h"
#include "transcript.h"

using namespace bgpu;

struct binius_pcs {
  const binius_ntt* ntt;
  uint32_t log_msg, log_batch, log_inv_rate, n_queries;
  uint32_t merkle_hash = bgpu::kMerkleSha256;
  std::vector<uint32_t> arities;
  uint32_t log_dim() const { return log_msg - log_batch; }
  uint32_t rs_log_len() const { return log_dim() + log_inv_rate; }
  uint32_t log_len() const { return rs_log_len() + log_batch; }
  uint32_t n_final() const {
    uint32_t s = 0;
    for (auto a : arities) s += a;
    return log_dim() - s;
  }
  // vcs_optimal_layers_depths_iter (verifier/verifier/src/fri/common.rs:154-168)
  std::vector<uint32_t> optimal_depths() const {
    uint32_t cap = 0;
    while ((1ull << cap) < n_queries) cap++;
    std::vector<uint32_t> d;
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

struct binius_pcs_committed {
  int device;
  uint32_t log_len;      // codeword log length (rs_log_len + log_batch)
  uint32_t log_leaves;   // rs_log_len
  void* d_codeword;
  void* d_nodes;
  cudaStream_t stream;   // the commit stream: allocation and release are ordered on it
  uint8_t root[32];
};

namespace {

typedef unsigned __int128 u128h;

u128h to_u128(const uint8_t b[16]) {
  u128h v;
  memcpy(&v, b, 16);
  return v;
}
void from_u128(u128h v, uint8_t b[16]) { memcpy(b, &v, 16); }

__host__ __device__ inline uint64_t layer_off(uint32_t L, uint32_t j) {
  return (1ull << (L + 1)) - (1ull << (L + 1 - j));
}

// One opened oracle of a FRI query (FRIQueryProver::prove_at_index, fri/query.rs:51-110): the
// query index is shifted right by `shift` first (the previous fold's arity), then the coset of
// 2^log_coset elements at that index of `data` and the Merkle branch of `nodes` (a tree of 2^L
// leaves whose layers are stored leaves-first) from the leaf up to layer `depth` are opened.
struct QueryLevel {
  const uint8_t* data;
  const uint8_t* nodes;
  uint32_t shift, log_coset, L, depth;
};
constexpr uint32_t kMaxQueryLevels = 16;
struct QueryLayout {
  QueryLevel lv[kMaxQueryLevels];
  uint32_t n_levels;
  uint64_t per_query;  // bytes one query opens
};

// The openings of every query, one warp per query: query q's bytes go to dst[q * per_query ..) in
// the order the proof carries them (per level the coset values, then the branch siblings from
// the leaf layer up), so the host appends the buffer as it is.
__global__ void fri_query_gather_kernel(QueryLayout lay, const uint64_t* __restrict__ idx,
                                        uint32_t n_queries, uint8_t* __restrict__ dst) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= n_queries) return;
  uint4* out = reinterpret_cast<uint4*>(dst + q * lay.per_query);
  uint64_t index = idx[q];
  for (uint32_t l = 0; l < lay.n_levels; l++) {
    const QueryLevel v = lay.lv[l];
    index >>= v.shift;
    const uint32_t n_coset = 1u << v.log_coset;  // 16-byte elements
    const uint4* coset = reinterpret_cast<const uint4*>(v.data) + (index << v.log_coset);
    for (uint32_t i = lane; i < n_coset; i += 32) out[i] = coset[i];
    out += n_coset;
    const uint32_t n_sib = v.L - v.depth;
    const uint4* nodes = reinterpret_cast<const uint4*>(v.nodes);
    for (uint32_t i = lane; i < 2 * n_sib; i += 32) {
      const uint32_t j = i >> 1;
      const uint64_t node = layer_off(v.L, j) | ((index >> j) ^ 1);
      out[i] = nodes[2 * node + (i & 1)];
    }
    out += 2 * n_sib;
  }
}

// Device-side FRIFoldProver state.
struct DevFri {
  const binius_pcs& P;
  const binius_pcs_committed& C;
  cudaStream_t s;
  std::vector<uint4*> words;
  std::vector<uint32_t> word_log_len;
  std::vector<uint8_t*> trees;
  std::vector<uint32_t> tree_log_leaves;
  uint32_t curr_round = 0;
  int64_t next_commit;
  const uint4* d_chal;         // the device transcript's challenges, one per round
  uint32_t n_unprocessed = 0;  // challenges received since the last commit

  DevFri(const binius_pcs& p, const binius_pcs_committed& c, cudaStream_t st, const uint4* chal)
      : P(p), C(c), s(st), next_commit(p.log_batch), d_chal(chal) {}
  ~DevFri() {
    for (auto w : words) dev_free(w, s);
    for (auto t : trees) dev_free(t, s);
  }

  // FRIFoldProver::execute_fold_round (prover/prover/src/fri/fold.rs:117-175): on a commit round,
  // folds by the challenges received since the last commit (device memory) and commits the new
  // codeword; *d_root is then the device address of the new tree's root.
  int execute(bool* committed, const uint8_t** d_root) {
    *committed = false;
    if (next_commit < 0 || (int64_t)curr_round != next_commit) return BINIUS_OK;
    const uint32_t n = n_unprocessed;
    const uint4* ch = d_chal + (curr_round - n);
    uint4* out = nullptr;
    uint32_t log_out;
    if (words.empty()) {
      log_out = P.rs_log_len();
      BGPU_CUDA(dev_alloc(&out, 16ull << log_out, s));
      words.push_back(out);
      word_log_len.push_back(log_out);
      if (int rc = fri_fold_interleaved_dev(C.d_codeword, log_out, P.log_batch, ch, out, s))
        return rc;
    } else {
      const uint32_t log_prev = word_log_len.back();
      log_out = log_prev - n;
      const uint4* prev = words.back();
      BGPU_CUDA(dev_alloc(&out, 16ull << log_out, s));
      words.push_back(out);
      word_log_len.push_back(log_out);
      if (int rc = fri_fold_codeword_dev(P.ntt, prev, log_prev, ch, n, out, s)) return rc;
    }
    n_unprocessed = 0;
    const size_t idx = words.size() - 1;  // number of rounds committed before this one
    const bool has_next = idx < P.arities.size();
    const uint32_t next_arity = has_next ? P.arities[idx] : 0;
    const uint32_t log_coset = has_next ? next_arity : P.n_final();
    const uint32_t log_leaves = log_out - log_coset;
    uint8_t* nodes = nullptr;
    BGPU_CUDA(dev_alloc(&nodes, 32ull * ((2ull << log_leaves) - 1), s));
    trees.push_back(nodes);
    tree_log_leaves.push_back(log_leaves);
    if (int rc = merkle_commit_with(P.merkle_hash, out, log_leaves, log_coset, nodes, s))
      return rc;
    *d_root = nodes + 32 * ((2ull << log_leaves) - 2);
    next_commit = has_next ? next_commit + next_arity : -1;
    *committed = true;
    return BINIUS_OK;
  }

  void receive() {
    n_unprocessed++;
    curr_round++;
  }

  // FRIFoldProver::finish_proof (fri/fold.rs:221-244) with FRIQueryProver (fri/query.rs:51-110).
  // The terminal codeword and the optimal Merkle layers are decommitments (tape only, unseen by
  // the challenger), so the query indices can be sampled first and every opened byte -- terminal
  // codeword, layers, then per query the coset values and branches -- gathered on the device into
  // one buffer (bulk copies, then fri_query_gather_kernel from the uploaded indices) and read back
  // once, then appended in the reference's order.
  int finish(Transcript& t) {
    const auto depths = P.optimal_depths();
    uint8_t* d_dst = nullptr;
    uint64_t* d_idx = nullptr;
    std::vector<std::pair<const uint8_t*, uint64_t>> bulk;
    uint64_t off = 0;
    {
      const uint8_t* term = static_cast<const uint8_t*>(words.empty() ? C.d_codeword : words.back());
      const uint32_t log_term = words.empty() ? C.log_len : word_log_len.back();
      bulk.push_back({term, 16ull << log_term});
    }
    {
      std::vector<const uint8_t*> tr{static_cast<const uint8_t*>(C.d_nodes)};
      std::vector<uint32_t> tl{C.log_leaves};
      for (size_t i = 0; i + 1 < trees.size(); i++) {
        tr.push_back(trees[i]);
        tl.push_back(tree_log_leaves[i]);
      }
      for (size_t i = 0; i < tr.size() && i < depths.size(); i++) {
        const uint32_t d = depths[i], L = tl[i];
        bulk.push_back({tr[i] + 32 * ((2ull << L) - 1 + 1 - (2ull << d)), 32ull << d});
      }
    }
    for (const auto& b : bulk) off += b.second;
    QueryLayout lay;
    memset(&lay, 0, sizeof(lay));
    lay.lv[0] = {static_cast<const uint8_t*>(C.d_codeword), static_cast<const uint8_t*>(C.d_nodes),
                 0, P.log_batch, C.log_leaves, depths[0]};
    lay.n_levels = 1;
    for (size_t i = 0; i < words.size() && i < P.arities.size() && i + 1 < depths.size(); i++) {
      if (lay.n_levels == kMaxQueryLevels) return set_error(BINIUS_E_ARG, "fri: too many folds");
      lay.lv[lay.n_levels++] = {reinterpret_cast<const uint8_t*>(words[i]), trees[i],
                                P.arities[i], P.arities[i], tree_log_leaves[i], depths[i + 1]};
    }
    lay.per_query = 0;
    for (uint32_t l = 0; l < lay.n_levels; l++)
      lay.per_query += (16ull << lay.lv[l].log_coset) + 32ull * (lay.lv[l].L - lay.lv[l].depth);
    std::vector<uint64_t> idx(P.n_queries);
    for (uint32_t q = 0; q < P.n_queries; q++) idx[q] = t.sample_bits(P.rs_log_len());
    const uint64_t total = off + lay.per_query * P.n_queries;
    if (total == 0) return BINIUS_OK;
    BGPU_CUDA(dev_alloc(&d_dst, total, s));
    std::vector<uint8_t> h(total);
    int rc = BINIUS_OK;
    do {
      cudaError_t e = cudaSuccess;
      uint64_t o = 0;
      for (const auto& b : bulk) {
        if (b.second)
          e = cudaMemcpyAsync(d_dst + o, b.first, b.second, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) break;
        o += b.second;
      }
      if (e != cudaSuccess) { rc = cuda_error(e, "fri decommitment copy"); break; }
      if (P.n_queries) {
        if ((e = dev_alloc(&d_idx, 8ull * P.n_queries, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(d_idx, idx.data(), 8ull * P.n_queries, cudaMemcpyHostToDevice,
                                 s)) != cudaSuccess) {
          rc = cuda_error(e, "fri query indices");
          break;
        }
        const unsigned per_block = 4;  // warps (queries) per CTA
        fri_query_gather_kernel<<<(P.n_queries + per_block - 1) / per_block, 32 * per_block, 0,
                                  s>>>(lay, d_idx, P.n_queries, d_dst + off);
        if ((e = cudaGetLastError()) != cudaSuccess) {
          rc = cuda_error(e, "fri_query_gather_kernel");
          break;
        }
        count_launch();
      }
      rc = read_sync(h.data(), d_dst, total, s);
    } while (0);
    dev_free(d_idx, s);
    dev_free(d_dst, s);
    if (rc) return rc;
    t.decommitment(h.data(), h.size());
    return BINIUS_OK;
  }
};

// TensorAlgebra<B1, B128>::transpose of the 128 x 128 bit matrix whose row k is s[k]: out[j] bit
// k = in[k] bit j.  Block swaps of halving size (64, 32, .., 1): at size j, row k < k + j (bit j
// of k clear) trades its columns c + j for row k + j's columns c (bit j of c clear).
void transpose128(const u128h in[128], u128h out[128]) {
  for (int k = 0; k < 128; k++) out[k] = in[k];
  u128h m = ~(u128h)0 >> 64;  // columns with bit j clear, j = 64
  for (int j = 64; j >= 1; j >>= 1, m ^= m << j) {
    for (int k = 0; k < 128; k++) {
      if (k & j) continue;
      const u128h t = ((out[k] >> j) ^ out[k + j]) & m;
      out[k + j] ^= t;
      out[k] ^= t << j;
    }
  }
}

int pcs_prove_impl(const binius_pcs* P, const binius_pcs_committed* C, const void* d_witness,
                   const uint8_t* h_point, Transcript& t, cudaStream_t s) {
  const uint32_t n = P->log_msg;
  const uint64_t N = 1ull << n;
  uint4 *a = nullptr, *b = nullptr, *eq_r = nullptr, *dev = nullptr;
  uint32_t* d_small = nullptr;  // 128 elements (ring switch)
  BGPU_CUDA(dev_alloc(&a, 16 * N, s));
  BGPU_CUDA(dev_alloc(&b, 16 * N, s));
  BGPU_CUDA(dev_alloc(&eq_r, 16 * 128, s));
  BGPU_CUDA(dev_alloc(&d_small, 16 * 128, s));
  // BaseFold round state: sums (2 per round), the claim pair, challenges
  const uint64_t n_dev = 2ull * n + 2 + n;
  BGPU_CUDA(dev_alloc(&dev, 16 * n_dev, s));
  uint4* slots = dev;
  uint4* claim = dev + 2 * n;  // [0] running claim, [1] initial claim
  uint4* chal = claim + 2;
  int rc = BINIUS_OK;
  {
    DevFri fri(*P, *C, s, chal);
    do {
      // suffix tensor of the evaluation point (coordinates 7..) into b
      if ((rc = eq_tensor(reinterpret_cast<const uint4*>(h_point + 16 * 7), n, b, s))) break;
      // s_hat_v = fold_1b_rows_for_b128(witness, suffix_tensor)
      if ((rc = fold_1b_rows(static_cast<const uint4*>(d_witness), b, N, d_small, s))) break;
      // the BaseFold message copy needs no challenge: queued before the host round trip
      cudaError_t e = cudaMemcpyAsync(a, d_witness, 16 * N, cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) { rc = cuda_error(e, "copy witness"); break; }
      uint8_t s_hat_v[128 * 16];
      if ((rc = read_sync(s_hat_v, d_small, sizeof(s_hat_v), s))) break;
      t.message(s_hat_v, sizeof(s_hat_v));
      u128h v[128], u[128];
      for (int k = 0; k < 128; k++) v[k] = to_u128(s_hat_v + 16 * k);
      transpose128(v, u);
      uint8_t r_dp[7 * 16];
      for (int i = 0; i < 7; i++) t.sample_elem(r_dp + 16 * i);
      // eq(r'') (128 entries) on the host; the device copy feeds the element fold
      u128h h_eq[128];
      h_eq[0] = 1;
      for (int i = 0; i < 7; i++) {
        const u128h ri = to_u128(r_dp + 16 * i);
        for (int k = 0; k < (1 << i); k++) {
          const u128h hi = host_gf_mul(h_eq[k], ri);
          h_eq[(1 << i) + k] = hi;
          h_eq[k] ^= hi;
        }
      }
      e = cudaMemcpyAsync(eq_r, h_eq, sizeof(h_eq), cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) { rc = cuda_error(e, "eq(r'') upload"); break; }
      u128h sum = 0;
      for (int j = 0; j < 128; j++) sum ^= host_gf_mul(u[j], h_eq[j]);
      e = cudaMemcpyAsync(claim + 1, &sum, 16, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) { rc = cuda_error(e, "claim upload"); break; }
      e = cudaMemsetAsync(slots, 0, 32ull * n, s);
      if (e != cudaSuccess) { rc = cuda_error(e, "round sums"); break; }
      // rs_eq_ind = fold_b128_elems_inplace(suffix_tensor, eq(r'')) in place in b
      if ((rc = fold_b128_elems(b, b, N, eq_r, s))) break;

      // BaseFold rounds on the device transcript: the round's sums, the FRI fold and commit on a
      // commit round, then the finish kernel (message, root, challenge, next table)
      DeviceTranscript dt;
      if ((rc = dt.begin(t, s))) break;
      uint32_t tape_bytes = 0;
      // the rounds after the last FRI commit inside the loop whose fold starts from at most
      // tail_max_len() elements run in the single-CTA tail
      uint32_t tail0 = 1;
      {
        uint32_t c = P->log_batch;
        if (c < n) tail0 = std::max(tail0, c + 1);
        for (uint32_t a_i : P->arities) {
          c += a_i;
          if (c < n) tail0 = std::max(tail0, c + 1);
        }
        while (tail0 < n && (N >> (tail0 - 1)) > tail_max_len()) tail0++;
      }
      for (uint32_t round = 0; round < tail0 && round < n && rc == BINIUS_OK; round++) {
        const uint64_t size = N >> round;
        uint32_t* ys = reinterpret_cast<uint32_t*>(slots + 2 * round);
        if (round == 0)
          rc = bivariate_eval(a, b, size / 2, ys, s);
        else
          rc = bivariate_fold_eval_dev(a, b, size * 2, chal + round - 1, ys, s);
        if (rc) break;
        bool committed = false;
        const uint8_t* d_root = nullptr;
        if ((rc = fri.execute(&committed, &d_root))) break;
        if ((rc = bivariate_round_finish(dt, slots + 2 * round, round == 0 ? claim + 1 : nullptr,
                                         claim, committed ? d_root : nullptr, chal + round, s)))
          break;
        tape_bytes += committed ? 64 : 32;
        fri.receive();
      }
      if (rc) break;
      if (tail0 < n) {
        if ((rc = bivariate_tail(dt, a, b, N >> (tail0 - 1), n - tail0, chal + tail0 - 1, claim,
                                 chal + tail0, s)))
          break;
        for (uint32_t round = tail0; round < n; round++) fri.receive();
        tape_bytes += 32 * (n - tail0);
      }
      bool committed = false;
      const uint8_t* d_root = nullptr;
      if ((rc = fri.execute(&committed, &d_root))) break;
      if (committed) {
        if ((rc = dt.message_device(d_root, 32, s))) break;
        tape_bytes += 32;
      }
      StagedReads rd(s);
      if ((rc = dt.read(rd, tape_bytes)) || (rc = rd.wait()) || (rc = dt.finish(t))) break;
      rc = fri.finish(t);
    } while (0);
  }
  dev_free(a, s);
  dev_free(b, s);
  dev_free(eq_r, s);
  dev_free(d_small, s);
  dev_free(dev, s);
  cudaError_t e = stream_wait(s);
  if (rc == BINIUS_OK && e != cudaSuccess) rc = cuda_error(e, "pcs prove");
  return rc;
}

}  // namespace

extern "C" {

int binius_pcs_create(const binius_ntt* ntt, uint32_t log_msg, uint32_t log_batch,
                      uint32_t log_inv_rate, const uint32_t* arities, uint32_t n_arities,
                      uint32_t n_queries, binius_pcs** out) {
  BGPU_ARG(out != nullptr && ntt != nullptr, "NULL argument");
  *out = nullptr;
  BGPU_ARG(log_batch <= log_msg && log_batch <= 8, "log_batch must be <= log_msg and <= 8");
  BGPU_ARG(log_msg <= 32, "log_msg too large");
  BGPU_ARG(n_arities == 0 || arities != nullptr, "arities is NULL");
  BGPU_ARG(n_queries >= 1, "n_queries must be positive");
  uint32_t sum = 0;
  for (uint32_t i = 0; i < n_arities; i++) {
    BGPU_ARG(arities[i] >= 1 && arities[i] <= 8, "fold arities must be in [1, 8]");
    sum += arities[i];
  }
  BGPU_ARG(sum <= log_msg - log_batch, "InvalidFoldAritySequence: arities exceed log_dim");
  BGPU_ARG(log_msg - log_batch + log_inv_rate <= ntt->log_domain,
           "NTT domain smaller than the RS code");
  binius_pcs* p = new binius_pcs();
  p->ntt = ntt;
  p->log_msg = log_msg;
  p->log_batch = log_batch;
  p->log_inv_rate = log_inv_rate;
  p->n_queries = n_queries;
  p->arities.assign(arities, arities + n_arities);
  *out = p;
  return clear_error();
}

int binius_pcs_set_merkle_hash(binius_pcs* pcs, uint32_t merkle_hash) {
  BGPU_ARG(pcs != nullptr, "NULL argument");
  BGPU_ARG(merkle_hash <= bgpu::kMerkleVision4, "unknown Merkle hash");
  pcs->merkle_hash = merkle_hash;
  return clear_error();
}

int binius_pcs_destroy(binius_pcs* pcs) {
  delete pcs;
  return BINIUS_OK;
}

int binius_pcs_commit(const binius_pcs* P, const void* d_witness, binius_pcs_committed** out,
                      void* h_root, void* stream) {
  BGPU_ARG(P != nullptr && d_witness != nullptr && out != nullptr, "NULL argument");
  *out = nullptr;
  cudaStream_t s = as_stream(stream);
  binius_pcs_committed* c = nullptr;
  if (int rc = pcs_commit_enqueue(P, d_witness, &c, s)) return rc;
  const uint8_t* d_root = pcs_committed_root(c);
  if (int rc = read_sync(c->root, d_root, 32, s)) {
    binius_pcs_committed_destroy(c);
    return rc;
  }
  if (h_root) memcpy(h_root, c->root, 32);
  *out = c;
  return clear_error();
}

}  // extern "C"

namespace bgpu {

const uint8_t* pcs_committed_root(const binius_pcs_committed* c) {
  return static_cast<const uint8_t*>(c->d_nodes) + 32 * ((2ull << c->log_leaves) - 2);
}

void pcs_committed_set_root(binius_pcs_committed* c, const uint8_t* h_root) {
  memcpy(c->root, h_root, 32);
}

int pcs_commit_enqueue(const binius_pcs* P, const void* d_witness, binius_pcs_committed** out,
                       cudaStream_t s) {
  *out = nullptr;
  binius_pcs_committed* c = new binius_pcs_committed();
  BGPU_CUDA(cudaGetDevice(&c->device));
  c->log_len = P->log_len();
  c->log_leaves = P->rs_log_len();
  c->d_codeword = nullptr;
  c->d_nodes = nullptr;
  c->stream = s;
  int rc = BINIUS_OK;
  do {
    // stream-ordered allocations from the (cached) device pool: no device-wide synchronisation
    cudaError_t e = dev_alloc(&c->d_codeword, 16ull << c->log_len, s);
    if (e != cudaSuccess) { rc = cuda_error(e, "dev_alloc(codeword)"); break; }
    e = dev_alloc(&c->d_nodes, 32ull * ((2ull << c->log_leaves) - 1), s);
    if (e != cudaSuccess) { rc = cuda_error(e, "dev_alloc(tree)"); break; }
    if ((rc = fri_commit_interleaved(P->ntt, d_witness, P->log_dim(), P->log_inv_rate,
                                     P->log_batch, P->merkle_hash, c->d_codeword, c->d_nodes,
                                     nullptr, s)))
      break;
  } while (0);
  if (rc) {
    if (c->d_codeword) dev_free(c->d_codeword, s);
    if (c->d_nodes) dev_free(c->d_nodes, s);
    delete c;
    return rc;
  }
  *out = c;
  return BINIUS_OK;
}

}  // namespace bgpu

extern "C" {

// Releases the buffers in order on the commit stream, which must still exist.
int binius_pcs_committed_destroy(binius_pcs_committed* c) {
  if (!c) return BINIUS_OK;
  dev_free(c->d_codeword, c->stream);
  dev_free(c->d_nodes, c->stream);
  delete c;
  return BINIUS_OK;
}

const void* binius_pcs_committed_codeword(const binius_pcs_committed* c) {
  return c ? c->d_codeword : nullptr;
}

int binius_pcs_prove(const binius_pcs* P, const binius_pcs_committed* C, const void* d_witness,
                     const void* h_eval_point, binius_transcript* transcript, void* stream) {
  BGPU_ARG(P && C && d_witness && h_eval_point && transcript, "NULL argument");
  BGPU_ARG(C->log_len == P->log_len(), "commitment does not match the PCS parameters");
  int rc = pcs_prove_impl(P, C, d_witness, static_cast<const uint8_t*>(h_eval_point),
                          transcript->t, as_stream(stream));
  return rc ? rc : clear_error();
}

}  // extern "C"
