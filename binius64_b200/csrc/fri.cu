// FRI folding, the FRI interleaved commit and FRI parameter selection.
//
// fold_interleaved (prover/prover/src/fri/fold.rs:260-282): each output is the inner product of a
// 2^log_batch chunk with eq_ind(challenges).  The 256-bit carry-less products are XOR-accumulated
// unreduced and reduced once per output (reduction is linear, so the bits are identical).
// fold_codeword (prover/prover/src/fri/fold.rs:297-318 -> verifier/verifier/src/fri/fold.rs:20-99):
// one thread folds one coset of 2^n values in registers through all n rounds: the inverse NTT
// butterfly with twiddle(log_len - 1 - round, index) then u + (v - u) * r.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "gf128.cuh"
#include "gf_reduce.cuh"
#include "internal.h"
#include "kernels.h"

using namespace bgpu;

namespace bgpu {
int rs_encode_batch(const binius_ntt* ntt, const void* d_msg, uint32_t log_dim,
                    uint32_t log_inv_rate, uint32_t log_batch, void* d_codeword,
                    cudaStream_t stream);
int merkle_commit(const void* d_elems, uint32_t log_leaves, uint32_t log_batch, void* d_nodes,
                  cudaStream_t stream);
}  // namespace bgpu

namespace {

constexpr uint32_t kMaxChallenges = 8;

struct Challenges {
  uint4 r[kMaxChallenges];
};

unsigned grid_for(uint64_t n, unsigned threads) {
  uint64_t g = (n + threads - 1) / threads;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, 148ull * 64));
}

// Challenges come from ch, or from device memory at dch when that is set (challenges sampled by
// the device transcript).
__global__ void __launch_bounds__(256)
    fold_interleaved_kernel(const uint4* __restrict__ cw, uint32_t log_len, uint32_t log_batch,
                            Challenges ch, const uint4* __restrict__ dch, uint4* __restrict__ out) {
  __shared__ uint4 tensor[1u << kMaxChallenges];
  const uint32_t batch = 1u << log_batch;
  // eq_ind(r)[j] = prod_i (bit_i(j) ? r_i : 1 + r_i)  (multilinear/eq.rs:39-71)
  for (uint32_t j = threadIdx.x; j < batch; j += blockDim.x) {
    uint4 acc = gf_one();
    for (uint32_t i = 0; i < log_batch; i++) {
      uint4 f = dch ? dch[i] : ch.r[i];
      if (!((j >> i) & 1)) f.x ^= 1u;
      acc = gf_mul(acc, f);
    }
    tensor[j] = acc;
  }
  __syncthreads();
  const uint64_t n = 1ull << log_len;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    u256 acc = {0, 0, 0, 0};
    const uint4* row = cw + (i << log_batch);
    for (uint32_t j = 0; j < batch; j++) xor_into(acc, clmul128(__ldg(row + j), tensor[j]));
    out[i] = reduce256(acc);
  }
}

template <int N>
__global__ void __launch_bounds__(256)
    fold_codeword_kernel(const uint4* __restrict__ cw, uint32_t log_len,
                         const uint4* __restrict__ tw, Challenges ch, const uint4* __restrict__ dch,
                         uint4* __restrict__ out) {
  const uint64_t n_chunks = 1ull << (log_len - N);
  uint4 rr[N];
#pragma unroll
  for (int kk = 0; kk < N; kk++) rr[kk] = dch ? dch[kk] : ch.r[kk];
  for (uint64_t ci = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; ci < n_chunks;
       ci += (uint64_t)gridDim.x * blockDim.x) {
    uint4 v[1 << N];
#pragma unroll
    for (int j = 0; j < (1 << N); j++) v[j] = __ldg(cw + (ci << N) + j);
    uint32_t cur = log_len;
#pragma unroll
    for (int kk = 0; kk < N; kk++) {
      const int size = N - kk;
      const uint4 r = rr[kk];
      const uint64_t layer_base = (1ull << (cur - 1)) - 1;
#pragma unroll
      for (int off = 0; off < (1 << (size - 1)); off++) {
        uint4 u = v[off << 1], w = v[(off << 1) | 1];
        const uint64_t index = (ci << (size - 1)) | (uint64_t)off;
        const uint4 t = __ldg(tw + layer_base + index);
        gf_add_into(w, u);
        gf_add_into(u, gf_mul(w, t));
        gf_add_into(w, u);  // w - u
        gf_add_into(u, gf_mul(w, r));
        v[off] = u;
      }
      cur--;
    }
    out[ci] = v[0];
  }
}

// The same fold for launches of less than one wave, where one thread per chunk leaves the SMs
// nearly empty and each thread's 2 (2^N - 1) dependent multiplies are the launch's latency.  Here
// a chunk takes P = 2^(N-1) consecutive lanes: in a round of 2^size values, lane q < 2^(size-1)
// holds values 2q and 2q + 1, runs butterfly q and keeps its output, which lanes 2q' and 2q' + 1
// hand to lane q' by shuffles for the next round.  The chain is N rounds of two multiplies.
template <int N>
__global__ void __launch_bounds__(256)
    fold_codeword_lanes_kernel(const uint4* __restrict__ cw, uint32_t log_len,
                               const uint4* __restrict__ tw, Challenges ch,
                               const uint4* __restrict__ dch, uint4* __restrict__ out) {
  constexpr uint32_t P = 1u << (N - 1);
  const uint64_t n_chunks = 1ull << (log_len - N);
  const uint32_t q = threadIdx.x & (P - 1);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x / P;
  // every lane of a warp runs the same number of iterations (blockDim.x is a multiple of 32)
  const uint64_t first = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / P;
  const uint64_t warp_first = (blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u)) / P;
  for (uint64_t base = warp_first; base < n_chunks; base += stride) {
    const uint64_t ci = base + (first - warp_first);
    const bool live = ci < n_chunks;
    uint4 u = gf_zero(), w = gf_zero();
    if (live) {
      u = __ldg(cw + (ci << N) + 2 * q);
      w = __ldg(cw + (ci << N) + 2 * q + 1);
    }
    uint32_t cur = log_len;
#pragma unroll
    for (int kk = 0; kk < N; kk++) {
      const int size = N - kk;
      if (kk > 0) {  // gather this round's pair from the previous round's outputs
        const uint32_t src = 2 * q < (1u << size) ? 2 * q : 0u;
        const uint4 a = shfl_gf(u, src, P), b = shfl_gf(u, src + 1 < P ? src + 1 : 0u, P);
        w = b;
        u = a;
      }
      if (live && q < (1u << (size - 1))) {
        const uint4 r = dch ? dch[kk] : ch.r[kk];
        const uint64_t layer_base = (1ull << (cur - 1)) - 1;
        const uint64_t index = (ci << (size - 1)) | (uint64_t)q;
        const uint4 t = __ldg(tw + layer_base + index);
        gf_add_into(w, u);
        gf_add_into(u, gf_mul(w, t));
        gf_add_into(w, u);
        gf_add_into(u, gf_mul(w, r));
      }
      cur--;
    }
    if (live && q == 0) out[ci] = u;
  }
}

__global__ void gf_mul_batch_kernel(const uint4* __restrict__ a, const uint4* __restrict__ b,
                                    uint4* __restrict__ out, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = gf_mul(__ldg(a + i), __ldg(b + i));
}

int load_challenges(const void* h, uint32_t n, Challenges& ch) {
  if (n > kMaxChallenges) return set_error(BINIUS_E_ARG, "at most 8 folding challenges per call");
  if (n && !h) return set_error(BINIUS_E_ARG, "challenges is NULL");
  memset(&ch, 0, sizeof(ch));
  if (n) memcpy(ch.r, h, 16 * (size_t)n);
  return BINIUS_OK;
}

// Launches of fewer chunks than this (under one wave of 256-thread blocks on 148 SMs) take the
// lane-parallel kernel.
constexpr uint64_t kCompactFoldChunks = 148ull * 256;

template <int N>
void launch_fold_codeword(const uint4* cw, uint32_t log_len, const uint4* tw, const Challenges& ch,
                          const uint4* dch, uint4* out, cudaStream_t s) {
  uint64_t n_chunks = 1ull << (log_len - N);
  if (n_chunks < kCompactFoldChunks)
    fold_codeword_lanes_kernel<N><<<grid_for(n_chunks << (N - 1), 256), 256, 0, s>>>(
        cw, log_len, tw, ch, dch, out);
  else
    fold_codeword_kernel<N><<<grid_for(n_chunks, 256), 256, 0, s>>>(cw, log_len, tw, ch, dch, out);
}

// ---- Scratch for binius_fri_fold_codeword_noalloc ----
// A fold over more than 4 challenges passes the codeword after its first 4 rounds through an
// intermediate buffer.  The allocation-free entry point keeps that buffer in this file-scope device
// array instead of allocating: 2^18 elements = 4 MiB, reserved on every GPU that loads this
// library until the process exits.
constexpr uint64_t kNoAllocScratchElems = 1ull << 18;
static __device__ __align__(256) uint4 g_fold_scratch[kNoAllocScratchElems];

constexpr int kMaxDevices = 64;
struct ScratchSlot {
  std::once_flag once;
  void* ptr = nullptr;
  cudaError_t err = cudaSuccess;
};
static ScratchSlot g_scratch_slots[kMaxDevices];

// Device address of g_fold_scratch on the current device.  Host code cannot use the symbol's name
// as a device pointer, so the address is looked up once per device (the device being current).
int noalloc_scratch(void** out) {
  int dev = -1;
  BGPU_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return set_error(BINIUS_E_ARG, "device ordinal out of range");
  ScratchSlot& slot = g_scratch_slots[dev];
  std::call_once(slot.once, [&slot] {
    slot.err = cudaGetSymbolAddress(&slot.ptr, g_fold_scratch);
  });
  if (slot.err != cudaSuccess) return cuda_error(slot.err, "cudaGetSymbolAddress(g_fold_scratch)");
  *out = slot.ptr;
  return BINIUS_OK;
}

// The steps of a fold over n_challenges <= 8 rounds: at most 4 rounds per launch (one coset of
// 16 values per thread in registers).  A fold over n challenges equals n successive
// single-challenge folds of the whole codeword, so two steps chain through `tmp`
// (2^(log_len - 4) elements, needed only when n_challenges > 4): codeword -> tmp -> out.
// Challenges come from ch, or from device memory at dch.
int fold_codeword_steps(const binius_ntt* ntt, const void* d_codeword, uint32_t log_len,
                        const Challenges& ch, const uint4* dch, uint32_t n_challenges,
                        void* d_out, uint4* tmp, cudaStream_t s) {
  const uint4* tw = static_cast<const uint4*>(ntt->d_twiddles);
  uint4* out = static_cast<uint4*>(d_out);
  if (n_challenges == 0) {
    BGPU_CUDA(cudaMemcpyAsync(d_out, d_codeword, 16ull << log_len, cudaMemcpyDeviceToDevice, s));
    return BINIUS_OK;
  }
  uint32_t done = 0, cur_len = log_len;
  const uint4* src = static_cast<const uint4*>(d_codeword);
  while (done < n_challenges) {
    uint32_t step = std::min<uint32_t>(4, n_challenges - done);
    Challenges sub;
    memset(&sub, 0, sizeof(sub));
    for (uint32_t i = 0; i < step; i++) sub.r[i] = ch.r[done + i];
    const uint4* dsub = dch ? dch + done : nullptr;
    // the first step writes all of tmp before the second reads it (same stream)
    uint4* dst = (done + step == n_challenges) ? out : tmp;
    switch (step) {
      case 1: launch_fold_codeword<1>(src, cur_len, tw, sub, dsub, dst, s); break;
      case 2: launch_fold_codeword<2>(src, cur_len, tw, sub, dsub, dst, s); break;
      case 3: launch_fold_codeword<3>(src, cur_len, tw, sub, dsub, dst, s); break;
      default: launch_fold_codeword<4>(src, cur_len, tw, sub, dsub, dst, s); break;
    }
    BGPU_LAUNCH_CHECK("fold_codeword_kernel");
    count_launch();
    src = dst;
    cur_len -= step;
    done += step;
  }
  return BINIUS_OK;
}

// The fold behind binius_fri_fold_codeword: the intermediate of a fold over more than 4
// challenges is a stream-ordered allocation.
int fold_codeword_impl(const binius_ntt* ntt, const void* d_codeword, uint32_t log_len,
                       const Challenges& ch, const uint4* dch, uint32_t n_challenges, void* d_out,
                       cudaStream_t s) {
  uint4* tmp = nullptr;
  if (n_challenges > 4) BGPU_CUDA(dev_alloc(&tmp, 16ull << (log_len - 4), s));
  const int rc = fold_codeword_steps(ntt, d_codeword, log_len, ch, dch, n_challenges, d_out, tmp, s);
  if (tmp) {
    cudaError_t e = dev_free(tmp, s);
    if (!rc && e != cudaSuccess) return cuda_error(e, "dev_free(fold intermediate)");
  }
  return rc;
}

}  // namespace

namespace bgpu {

int fri_fold_interleaved_dev(const void* d_codeword, uint32_t log_len, uint32_t log_batch,
                             const uint4* d_challenges, void* d_out, cudaStream_t s) {
  if (log_batch > kMaxChallenges) return set_error(BINIUS_E_ARG, "at most 8 folding challenges");
  Challenges none;
  memset(&none, 0, sizeof(none));
  fold_interleaved_kernel<<<grid_for(1ull << log_len, 256), 256, 0, s>>>(
      static_cast<const uint4*>(d_codeword), log_len, log_batch, none, d_challenges,
      static_cast<uint4*>(d_out));
  BGPU_LAUNCH_CHECK("fold_interleaved_kernel");
  count_launch();
  return BINIUS_OK;
}

int fri_fold_codeword_dev(const binius_ntt* ntt, const void* d_codeword, uint32_t log_len,
                          const uint4* d_challenges, uint32_t n_challenges, void* d_out,
                          cudaStream_t s) {
  if (n_challenges > kMaxChallenges) return set_error(BINIUS_E_ARG, "at most 8 folding challenges");
  Challenges none;
  memset(&none, 0, sizeof(none));
  return fold_codeword_impl(ntt, d_codeword, log_len, none, d_challenges, n_challenges, d_out, s);
}

}  // namespace bgpu

namespace bgpu {

int fri_commit_interleaved(const binius_ntt* ntt, const void* d_msg, uint32_t log_dim,
                           uint32_t log_inv_rate, uint32_t log_batch, uint32_t merkle_hash,
                           void* d_codeword, void* d_nodes, void* h_root, cudaStream_t s) {
  if (int rc = rs_encode_batch(ntt, d_msg, log_dim, log_inv_rate, log_batch, d_codeword, s))
    return rc;
  const uint32_t log_leaves = log_dim + log_inv_rate;
  if (int rc = merkle_commit_with(merkle_hash, d_codeword, log_leaves, log_batch, d_nodes, s))
    return rc;
  if (h_root) {
    const uint8_t* root = static_cast<const uint8_t*>(d_nodes) + 32 * ((2ull << log_leaves) - 2);
    if (int rc = read_sync(h_root, root, 32, s)) return rc;
  }
  return BINIUS_OK;
}

}  // namespace bgpu

extern "C" {

int binius_fri_fold_interleaved(const void* d_codeword, uint32_t log_len, uint32_t log_batch,
                                const void* h_challenges, void* d_out, void* stream) {
  BGPU_ARG(d_codeword != nullptr && d_out != nullptr, "codeword / out is NULL");
  BGPU_ARG(log_len + log_batch <= 40, "codeword too large");
  Challenges ch;
  if (int rc = load_challenges(h_challenges, log_batch, ch)) return rc;
  cudaStream_t s = as_stream(stream);
  fold_interleaved_kernel<<<grid_for(1ull << log_len, 256), 256, 0, s>>>(
      static_cast<const uint4*>(d_codeword), log_len, log_batch, ch, nullptr,
      static_cast<uint4*>(d_out));
  BGPU_LAUNCH_CHECK("fold_interleaved_kernel");
  count_launch();
  return clear_error();
}

int binius_fri_fold_codeword(const binius_ntt* ntt, const void* d_codeword, uint32_t log_len,
                             const void* h_challenges, uint32_t n_challenges, void* d_out,
                             void* stream) {
  BGPU_ARG(ntt != nullptr, "ntt is NULL");
  BGPU_ARG(d_codeword != nullptr && d_out != nullptr, "codeword / out is NULL");
  BGPU_ARG(n_challenges <= log_len, "more challenges than codeword variables");
  BGPU_ARG(log_len <= ntt->log_domain, "codeword longer than the NTT domain");
  Challenges ch;
  if (int rc = load_challenges(h_challenges, n_challenges, ch)) return rc;
  if (int rc = fold_codeword_impl(ntt, d_codeword, log_len, ch, nullptr, n_challenges, d_out,
                                  as_stream(stream)))
    return rc;
  return clear_error();
}

// Same result as binius_fri_fold_codeword, for callers that may not allocate device memory.  For
// n_challenges > 4 the intermediate codeword lives in g_fold_scratch (at most 2^18 elements, so
// log_len - 4 <= 18); larger folds are rejected with BINIUS_E_ARG.  The first call on a device looks
// up the scratch address (cudaGetSymbolAddress); make that first call before any stream capture.
// Every call on a device shares the one scratch array: calls whose kernels overlap on the GPU (for
// example on two streams) race on it.  No cudaMalloc, cudaFree or other allocating call is made.
int binius_fri_fold_codeword_noalloc(const binius_ntt* ntt, const void* d_codeword,
                                     uint32_t log_len, const void* h_challenges,
                                     uint32_t n_challenges, void* d_out, void* stream) {
  BGPU_ARG(ntt != nullptr, "ntt is NULL");
  BGPU_ARG(d_codeword != nullptr && d_out != nullptr, "codeword / out is NULL");
  BGPU_ARG(n_challenges <= log_len, "more challenges than codeword variables");
  BGPU_ARG(log_len <= ntt->log_domain, "codeword longer than the NTT domain");
  Challenges ch;
  if (int rc = load_challenges(h_challenges, n_challenges, ch)) return rc;
  uint4* scratch = nullptr;
  if (n_challenges > 4) {
    if (log_len - 4 > 18)
      return set_error(BINIUS_E_ARG,
                       "binius_fri_fold_codeword_noalloc: a fold of more than 4 challenges needs "
                       "2^(log_len-4) scratch elements and the static scratch holds 2^18 (4 MiB); "
                       "use binius_fri_fold_codeword for log_len > 22");
    void* p = nullptr;
    if (int rc = noalloc_scratch(&p)) return rc;
    scratch = static_cast<uint4*>(p);
  }
  // the same steps as binius_fri_fold_codeword, with the static scratch as the intermediate
  if (int rc = fold_codeword_steps(ntt, d_codeword, log_len, ch, nullptr, n_challenges, d_out,
                                   scratch, as_stream(stream)))
    return rc;
  return clear_error();
}

int binius_fri_commit_interleaved(const binius_ntt* ntt, const void* d_msg, uint32_t log_dim,
                                  uint32_t log_inv_rate, uint32_t log_batch, void* d_codeword,
                                  void* d_nodes, void* h_root, void* stream) {
  if (int rc = bgpu::fri_commit_interleaved(ntt, d_msg, log_dim, log_inv_rate, log_batch,
                                            bgpu::kMerkleSha256, d_codeword, d_nodes, h_root,
                                            as_stream(stream)))
    return rc;
  return clear_error();
}

// calculate_n_test_queries (verifier/verifier/src/fri/common.rs:182-186).
uint32_t binius_fri_n_test_queries(uint32_t security_bits, uint32_t log_inv_rate) {
  double rate = pow(2.0, -(double)log_inv_rate);
  double per_query_err = 0.5 * (1.0 + rate);
  return (uint32_t)ceil((double)security_bits / -log2(per_query_err));
}

// estimate_optimal_arity (verifier/verifier/src/fri/common.rs:191-219).
uint32_t binius_fri_estimate_optimal_arity(uint32_t log_block_length, uint32_t digest_size,
                                           uint32_t field_size) {
  uint32_t best = 1;
  bool have_old = false;
  uint64_t old = 0;
  for (uint32_t arity = 1; arity <= log_block_length; arity++) {
    uint64_t est =
        ((uint64_t)(log_block_length / 2) * digest_size + ((uint64_t)1 << arity) * field_size) *
        (log_block_length - arity) / arity;
    if (have_old && est > old) break;
    have_old = true;
    old = est;
    best = arity;
  }
  return best;
}

int binius_gf_mul_batch(const void* d_a, const void* d_b, void* d_out, uint64_t n, void* stream) {
  BGPU_ARG((d_a && d_b && d_out) || n == 0, "NULL operand");
  if (n == 0) return clear_error();
  gf_mul_batch_kernel<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(
      static_cast<const uint4*>(d_a), static_cast<const uint4*>(d_b), static_cast<uint4*>(d_out),
      n);
  BGPU_LAUNCH_CHECK("gf_mul_batch_kernel");
  count_launch();
  return clear_error();
}

}  // extern "C"
