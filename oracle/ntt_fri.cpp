// CPU oracle (test infrastructure only): domain context, additive NTT, Reed-Solomon encode,
// Merkle commit, FRI folds and FRI parameters.
#include <math.h>
#include <string.h>

#include <vector>

#include "oracle.h"
#include "oracle_internal.h"

namespace orc {

// generate_evals_from_subspace (verifier/math/src/ntt/domain_context.rs:19-46):
// evals[0] = basis; evals[i][k-1] = evals[i-1][k] * (evals[i-1][k] + evals[i-1][0]); then each
// row is divided by its first entry (normalized subspace polynomials W^_i(beta_j)).
static std::vector<std::vector<u128>> subspace_evals(const std::vector<u128>& basis) {
  size_t l = basis.size();
  std::vector<std::vector<u128>> evals;
  evals.push_back(basis);
  for (size_t i = 1; i < l; i++) {
    std::vector<u128> row;
    const auto& prev = evals[i - 1];
    for (size_t k = 1; k < prev.size(); k++) row.push_back(gf_mul(prev[k], prev[k] ^ prev[0]));
    evals.push_back(row);
  }
  for (auto& row : evals) {
    u128 inv = gf_inv(row[0]);
    for (auto& v : row) v = gf_mul(v, inv);
  }
  return evals;
}

// GenericPreExpanded::generate_from_subspace (domain_context.rs:114-133): layer `l` holds the
// subset sums of evals[dim-1-l][1..], entry j = XOR of row[k+1] over the set bits k of j.
static void expand_twiddles(const std::vector<std::vector<u128>>& evals, u128* out) {
  size_t dim = evals.size();
  for (size_t layer = 0; layer < dim; layer++) {
    const auto& row = evals[dim - 1 - layer];
    u128* t = out + ((size_t)1 << layer) - 1;
    t[0] = 0;
    size_t len = 1;
    for (size_t i = 1; i < row.size(); i++) {
      for (size_t j = 0; j < len; j++) t[len + j] = t[j] ^ row[i];
      len <<= 1;
    }
  }
}

u128 twiddle(const u128* tw, uint32_t layer, size_t block) {
  return tw[((size_t)1 << layer) - 1 + block];
}

static int ntt_check(uint32_t log_domain, uint32_t log_d, uint32_t skip_early, uint32_t skip_late) {
  // input_check (ntt/reference.rs:85-100)
  if (skip_early + skip_late > log_d) return 1;
  if (log_d - skip_late > log_domain) return 1;
  return 0;
}

// NeighborsLastReference::forward_transform (ntt/reference.rs:20-47).  Each layer's blocks are
// independent, so they are split over threads; the arithmetic per butterfly is unchanged.
void ntt_forward(const u128* tw, u128* data, uint32_t log_d, uint32_t skip_early,
                 uint32_t skip_late) {
  for (uint32_t layer = skip_early; layer < log_d - skip_late; layer++) {
    size_t num_blocks = (size_t)1 << layer;
    size_t half = (size_t)1 << (log_d - layer - 1);
    size_t n_pairs = num_blocks * half;
    parallel_for(n_pairs, [&](size_t lo, size_t hi) {
      for (size_t p = lo; p < hi; p++) {
        size_t block = p / half, off = p % half;
        u128 t = twiddle(tw, layer, block);
        size_t i0 = (block << (log_d - layer)) + off, i1 = i0 | half;
        u128 u = data[i0], v = data[i1];
        u ^= gf_mul(v, t);
        v ^= u;
        data[i0] = u;
        data[i1] = v;
      }
    });
  }
}

void ntt_inverse(const u128* tw, u128* data, uint32_t log_d, uint32_t skip_early,
                 uint32_t skip_late) {
  for (int64_t layer = (int64_t)(log_d - skip_late) - 1; layer >= (int64_t)skip_early; layer--) {
    size_t num_blocks = (size_t)1 << layer;
    size_t half = (size_t)1 << (log_d - layer - 1);
    size_t n_pairs = num_blocks * half;
    parallel_for(n_pairs, [&](size_t lo, size_t hi) {
      for (size_t p = lo; p < hi; p++) {
        size_t block = p / half, off = p % half;
        u128 t = twiddle(tw, (uint32_t)layer, block);
        size_t i0 = (block << (log_d - layer)) + off, i1 = i0 | half;
        u128 u = data[i0], v = data[i1];
        v ^= u;
        u ^= gf_mul(v, t);
        data[i0] = u;
        data[i1] = v;
      }
    });
  }
}

size_t reverse_bits(size_t x, uint32_t bits) {
  size_t r = 0;
  for (uint32_t i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
  return r;
}

// Merkle leaf: SHA-256 over the 16-byte LE encodings of the leaf's elements, nodes compressed
// pairwise (binary_merkle_tree.rs:65-122, 177-205).
void merkle_commit(const u128* elems, uint32_t log_leaves, uint32_t log_batch, uint8_t* nodes) {
  size_t n_leaves = (size_t)1 << log_leaves;
  size_t batch = (size_t)1 << log_batch;
  parallel_for(n_leaves, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; i++)
      merkle_leaf_hash((const uint8_t*)(elems + i * batch), batch * 16, nodes + 32 * i);
  });
  size_t prev = 0, len = n_leaves;
  while (len > 1) {
    size_t next = prev + len;
    size_t half = len / 2;
    parallel_for(half, [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; i++)
        merkle_node_hash(nodes + 32 * (prev + 2 * i), nodes + 32 * (prev + 2 * i + 1),
                         nodes + 32 * (next + i));
    });
    prev = next;
    len = half;
  }
}

// eq_ind_partial_eval (verifier/math/src/multilinear/eq.rs:39-71, 123-131): coordinate i of the
// point selects index bit i; each coordinate doubles the table with lo = v*(1-r), hi = v*r.
void eq_ind_partial_eval(const u128* point, uint32_t n, u128* out) {
  out[0] = 1;
  size_t len = 1;
  for (uint32_t i = 0; i < n; i++) {
    auto expand = [&](size_t lo, size_t hi) {
      for (size_t j = lo; j < hi; j++) {
        u128 prod = gf_mul(out[j], point[i]);
        out[j] ^= prod;
        out[len + j] = prod;
      }
    };
    if (len >= ((size_t)1 << 14))
      parallel_for(len, expand);  // entries of one level are independent
    else
      expand(0, len);
    len <<= 1;
  }
}


// fold_interleaved (prover/prover/src/fri/fold.rs:260-282) -> fold_interleaved_chunk
// (verifier/verifier/src/fri/fold.rs:124-130): out[i] = <codeword[i*2^b .. (i+1)*2^b], eq(r)>.
void fold_interleaved(const u128* cw, uint32_t log_len, uint32_t log_batch, const u128* ch,
                      u128* o) {
  size_t batch = (size_t)1 << log_batch;
  std::vector<u128> tensor(batch);
  eq_ind_partial_eval(ch, log_batch, tensor.data());
  parallel_for((size_t)1 << log_len, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; i++) {
      u128 acc = 0;
      for (size_t j = 0; j < batch; j++) acc ^= gf_mul(cw[i * batch + j], tensor[j]);
      o[i] = acc;
    }
  });
}

// fold_chunk / fold_pair (verifier/verifier/src/fri/fold.rs:20-99): n rounds of the inverse
// butterfly with twiddle(log_len-1, index) followed by the line extrapolation u + (v - u) r.
u128 fold_chunk(const u128* tw, uint32_t log_len, size_t chunk_index, u128* vals, const u128* r,
                uint32_t n) {
  uint32_t cur_log_len = log_len, log_size = n;
  for (uint32_t k = 0; k < n; k++) {
    for (size_t off = 0; off < ((size_t)1 << (log_size - 1)); off++) {
      u128 u = vals[off << 1], v = vals[(off << 1) | 1];
      size_t index = (chunk_index << (log_size - 1)) | off;
      u128 t = twiddle(tw, cur_log_len - 1, index);
      v ^= u;
      u ^= gf_mul(v, t);
      vals[off] = u ^ gf_mul(v ^ u, r[k]);
    }
    cur_log_len--;
    log_size--;
  }
  return vals[0];
}

// fold_codeword (prover/prover/src/fri/fold.rs:297-318): fold_chunk over every coset of 2^n.
void fold_codeword(const u128* tw, const u128* cw, uint32_t log_len, const u128* r, uint32_t n,
                   u128* o) {
  size_t chunk = (size_t)1 << n;
  size_t n_chunks = ((size_t)1 << log_len) / chunk;
  parallel_for(n_chunks, [&](size_t lo, size_t hi) {
    std::vector<u128> vals(chunk);
    for (size_t ci = lo; ci < hi; ci++) {
      memcpy(vals.data(), cw + ci * chunk, chunk * sizeof(u128));
      o[ci] = fold_chunk(tw, log_len, ci, vals.data(), r, n);
    }
  });
}

// ReedSolomonCode::encode_batch (reed_solomon.rs:128-201): bit-reverse the whole message index
// (log_dim + log_batch bits), repeat it 2^log_inv_rate times, then forward-transform with
// skip_early = log_inv_rate and skip_late = log_batch.
void rs_encode(const u128* tw, const u128* m, uint32_t log_dim, uint32_t log_inv_rate,
               uint32_t log_batch, u128* out) {
  uint32_t log_msg = log_dim + log_batch;
  uint32_t log_out = log_msg + log_inv_rate;
  size_t n_msg = (size_t)1 << log_msg;
  for (size_t i = 0; i < n_msg; i++) out[reverse_bits(i, log_msg)] = m[i];
  for (size_t r = 1; r < ((size_t)1 << log_inv_rate); r++)
    memcpy(out + r * n_msg, out, n_msg * sizeof(u128));
  ntt_forward(tw, out, log_out, log_inv_rate, log_batch);
}

}  // namespace orc

using namespace orc;

extern "C" {

int orc_domain_twiddles(const uint64_t* basis, uint32_t dim, uint64_t* twiddles_out) {
  if (dim == 0 || dim > 40) return 1;
  std::vector<u128> b(dim);
  for (uint32_t i = 0; i < dim; i++) b[i] = basis ? load(basis + 2 * i) : ((u128)1 << i);
  auto evals = subspace_evals(b);
  expand_twiddles(evals, (u128*)twiddles_out);
  return 0;
}

int orc_ntt_forward(const uint64_t* twiddles, uint32_t log_domain, uint64_t* data, uint32_t log_d,
                    uint32_t skip_early, uint32_t skip_late) {
  if (ntt_check(log_domain, log_d, skip_early, skip_late)) return 1;
  ntt_forward((const u128*)twiddles, (u128*)data, log_d, skip_early, skip_late);
  return 0;
}

int orc_ntt_inverse(const uint64_t* twiddles, uint32_t log_domain, uint64_t* data, uint32_t log_d,
                    uint32_t skip_early, uint32_t skip_late) {
  if (ntt_check(log_domain, log_d, skip_early, skip_late)) return 1;
  ntt_inverse((const u128*)twiddles, (u128*)data, log_d, skip_early, skip_late);
  return 0;
}

int orc_rs_encode_batch(const uint64_t* twiddles, uint32_t log_domain, const uint64_t* msg,
                        uint32_t log_dim, uint32_t log_inv_rate, uint32_t log_batch,
                        uint64_t* codeword_out) {
  if (log_dim + log_inv_rate > log_domain) return 1;
  rs_encode((const u128*)twiddles, (const u128*)msg, log_dim, log_inv_rate, log_batch,
            (u128*)codeword_out);
  return 0;
}

int orc_merkle_commit(const uint64_t* elems, uint32_t log_leaves, uint32_t log_batch,
                      uint8_t* nodes_out) {
  merkle_commit((const u128*)elems, log_leaves, log_batch, nodes_out);
  return 0;
}

void orc_eq_ind_partial_eval(const uint64_t* point, uint32_t n, uint64_t* out) {
  eq_ind_partial_eval((const u128*)point, n, (u128*)out);
}

int orc_fri_fold_interleaved(const uint64_t* codeword, uint32_t log_len, uint32_t log_batch,
                             const uint64_t* challenges, uint64_t* out) {
  fold_interleaved((const u128*)codeword, log_len, log_batch, (const u128*)challenges, (u128*)out);
  return 0;
}

int orc_fri_fold_codeword(const uint64_t* twiddles, uint32_t log_domain, const uint64_t* codeword,
                          uint32_t log_len, const uint64_t* challenges, uint32_t n_challenges,
                          uint64_t* out) {
  if (n_challenges > log_len || log_len > log_domain) return 1;
  fold_codeword((const u128*)twiddles, (const u128*)codeword, log_len, (const u128*)challenges,
                n_challenges, (u128*)out);
  return 0;
}

// calculate_n_test_queries (verifier/verifier/src/fri/common.rs:182-186).
uint32_t orc_calculate_n_test_queries(uint32_t security_bits, uint32_t log_inv_rate) {
  double rate = pow(2.0, -(double)log_inv_rate);
  double per_query_err = 0.5 * (1.0 + rate);
  return (uint32_t)ceil((double)security_bits / -log2(per_query_err));
}

// estimate_optimal_arity (verifier/verifier/src/fri/common.rs:191-219): scan arities 1.. and stop
// at the first increase of the estimated query proof size.
uint32_t orc_estimate_optimal_arity(uint32_t log_block_length, uint32_t digest_size,
                                    uint32_t field_size) {
  uint32_t best = 1;
  bool have_old = false;
  uint64_t old = 0;
  for (uint32_t arity = 1; arity <= log_block_length; arity++) {
    uint64_t est = ((uint64_t)(log_block_length / 2) * digest_size + ((uint64_t)1 << arity) * field_size) *
                   (log_block_length - arity) / arity;
    if (have_old && est > old) break;
    have_old = true;
    old = est;
    best = arity;
  }
  return best;
}

}  // extern "C"
