// Constraint systems on the device: the reference's v2 wire format, validate_and_prepare's padding
// and operand evaluation.
//
// ConstraintSystem::deserialize (verifier/core/src/constraint_system.rs:615-650): u32 version (2),
// the ValueVecLayout as eight u32 (usize fields), constants (u32 count + u64 words), AND
// constraints (u32 count, then per constraint the operands a, b, c) and MUL constraints (a, b, hi,
// lo); an operand is a u32 count of (u32 value index, u8 shift variant, u32 amount) terms.
// validate (:466-530) and validate_and_prepare (:558-584: pad AND to a power of two >= 8 and MUL to
// a power of two >= 1 with empty constraints).
//
// Operands live on the device in CSR form: group g = constraint * k + slot with offsets[g] into a
// term array of (value index, variant << 8 | amount).  eval_operand (verifier/core/src/verify.rs:
// 14-35) runs one thread per group: a gather of the witness words, the shift, and an XOR.
#include <string.h>

#include <algorithm>
#include <vector>

#include "cs.h"
#include "internal.h"

using namespace bgpu;

namespace {

struct Reader {
  const uint8_t* p;
  size_t len, pos = 0;
  bool ok = true;
  uint32_t u32() {
    if (pos + 4 > len) {
      ok = false;
      return 0;
    }
    uint32_t v;
    memcpy(&v, p + pos, 4);
    pos += 4;
    return v;
  }
  uint64_t u64() {
    if (pos + 8 > len) {
      ok = false;
      return 0;
    }
    uint64_t v;
    memcpy(&v, p + pos, 8);
    pos += 8;
    return v;
  }
  uint8_t u8() {
    if (pos + 1 > len) {
      ok = false;
      return 0;
    }
    return p[pos++];
  }
};

__device__ __forceinline__ uint64_t shifted_word(uint64_t w, uint32_t variant, uint32_t n) {
  const uint32_t lo = (uint32_t)w, hi = (uint32_t)(w >> 32), n5 = n & 31;
  switch (variant) {
    case 0: return w << n;                                              // Sll
    case 1: return w >> n;                                              // Slr
    case 2: return (uint64_t)((int64_t)w >> n);                         // Sar
    case 3: return n ? ((w >> n) | (w << (64 - n))) : w;                // Rotr
    case 4: return ((uint64_t)(hi << n5) << 32) | (uint32_t)(lo << n5);  // Sll32
    case 5: return ((uint64_t)(hi >> n5) << 32) | (uint32_t)(lo >> n5);  // Srl32
    case 6:
      return ((uint64_t)(uint32_t)((int32_t)hi >> n5) << 32) | (uint32_t)((int32_t)lo >> n5);
    default:
      return ((uint64_t)__funnelshift_r(hi, hi, n5) << 32) | __funnelshift_r(lo, lo, n5);
  }
}

__global__ void eval_operands_kernel(const uint32_t* __restrict__ offsets,
                                     const uint2* __restrict__ terms,
                                     const uint64_t* __restrict__ witness, uint64_t n_constraints,
                                     uint32_t k, uint64_t* __restrict__ out) {
  const uint64_t groups = n_constraints * k;
  for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < groups;
       g += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t lo = __ldg(offsets + g), hi = __ldg(offsets + g + 1);
    uint64_t acc = 0;
    for (uint32_t t = lo; t < hi; t++) {
      const uint2 term = __ldg(terms + t);
      acc ^= shifted_word(__ldg(witness + term.x), term.y >> 8, term.y & 255);
    }
    const uint64_t c = g / k, slot = g - c * k;
    out[slot * n_constraints + c] = acc;
  }
}

int parse_operands(Reader& r, uint32_t n, uint32_t k, uint32_t total_len, HostOperands& ops) {
  ops.k = k;
  ops.offsets.assign(1, 0);
  ops.terms.clear();
  for (uint32_t i = 0; i < n && r.ok; i++) {
    for (uint32_t s = 0; s < k && r.ok; s++) {
      uint32_t cnt = r.u32();
      if (!r.ok || cnt > (1u << 24)) return set_error(BINIUS_E_ARG, "malformed operand length");
      for (uint32_t t = 0; t < cnt && r.ok; t++) {
        uint32_t vi = r.u32();
        uint32_t variant = r.u8();
        uint32_t amount = r.u32();
        if (!r.ok) break;
        if (variant > 7) return set_error(BINIUS_E_ARG, "unknown ShiftVariant");
        if (amount >= 64) return set_error(BINIUS_E_ARG, "ShiftedValueIndex::amount >= 64");
        if (amount == 0 && variant != 0)
          return set_error(BINIUS_E_ARG, "non-canonical shift (amount 0 with a non-Sll variant)");
        if (vi >= total_len) return set_error(BINIUS_E_ARG, "value index out of range");
        ops.terms.push_back(make_uint2(vi, (variant << 8) | amount));
      }
      ops.offsets.push_back((uint32_t)ops.terms.size());
    }
  }
  if (!r.ok) return set_error(BINIUS_E_ARG, "constraint system bytes truncated");
  return BINIUS_OK;
}

void pad_operands(HostOperands& ops, uint32_t n_target) {
  const uint32_t n = (uint32_t)((ops.offsets.size() - 1) / ops.k);
  for (uint32_t i = n; i < n_target; i++)
    for (uint32_t s = 0; s < ops.k; s++) ops.offsets.push_back((uint32_t)ops.terms.size());
}

uint32_t next_pow2_at_least(uint32_t n, uint32_t min) {
  uint32_t v = n < min ? min : n;
  uint32_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

int upload(const HostOperands& h, DevOperands& d) {
  d.k = h.k;
  d.n_constraints = (uint32_t)((h.offsets.size() - 1) / h.k);
  d.n_terms = h.terms.size();
  BGPU_CUDA(cudaMalloc(&d.offsets, 4 * h.offsets.size()));
  BGPU_CUDA(cudaMemcpy(d.offsets, h.offsets.data(), 4 * h.offsets.size(), cudaMemcpyHostToDevice));
  BGPU_CUDA(cudaMalloc(&d.terms, 8 * (h.terms.empty() ? 1 : h.terms.size())));
  if (!h.terms.empty())
    BGPU_CUDA(cudaMemcpy(d.terms, h.terms.data(), 8 * h.terms.size(), cudaMemcpyHostToDevice));
  return BINIUS_OK;
}

bool is_pow2(uint32_t v) { return v && !(v & (v - 1)); }

// The shift term table (ShiftTerms) built on the device: a counting sort of all operand terms by
// shift key.  Groups (constraint, CSR slot) of both operations form one index space (AND groups
// first); each CTA takes a contiguous range of it, counts its keys in shared memory, and -- after
// one scan of the global counts -- reserves a range per key with one atomic and places its terms
// there.  Terms of one key land in CTA order, in no fixed order within a CTA: every quantity the
// shift reduction takes from the table is a XOR sum over a key's terms.
constexpr uint32_t kSortThreads = 512;
constexpr uint32_t kSortBlocks = 148 * 2;

// Class of CSR slot `slot`: AND (a, b, c) -> 0, 1, 2; MUL slots (a, b, hi, lo) -> 3, 4, 6, 5.
__device__ __forceinline__ uint32_t slot_class(uint32_t k, uint32_t slot) {
  return k == 3 ? slot : (slot == 0 ? 3u : slot == 1 ? 4u : slot == 2 ? 6u : 5u);
}

template <class Fn>
__device__ __forceinline__ void for_each_term(const DevOperands& A, const DevOperands& M,
                                              uint64_t g0, uint64_t g1, Fn&& fn) {
  const uint64_t ga = (uint64_t)A.n_constraints * A.k;
  for (uint64_t g = g0 + threadIdx.x; g < g1; g += blockDim.x) {
    const DevOperands& op = g < ga ? A : M;
    const uint64_t gg = g < ga ? g : g - ga;
    const uint32_t slot = (uint32_t)(gg % op.k), c = (uint32_t)(gg / op.k);
    const uint32_t cls = slot_class(op.k, slot);
    for (uint32_t t = op.offsets[gg]; t < op.offsets[gg + 1]; t++) {
      const uint2 term = op.terms[t];
      fn(term.x, c, ((term.y >> 8) * 64 + (term.y & 255)) * 8 + cls);
    }
  }
}

template <bool SCATTER>
__global__ void __launch_bounds__(kSortThreads)
    shift_terms_kernel(DevOperands A, DevOperands M, uint32_t* __restrict__ counts,
                       uint32_t* __restrict__ vi, uint32_t* __restrict__ cc,
                       uint16_t* __restrict__ keys) {
  __shared__ uint32_t hist[kShiftKeys], base[kShiftKeys];
  const uint64_t G = (uint64_t)A.n_constraints * A.k + (uint64_t)M.n_constraints * M.k;
  const uint64_t per = (G + gridDim.x - 1) / gridDim.x;
  const uint64_t g0 = blockIdx.x * per, g1 = g0 + per < G ? g0 + per : G;
  for (uint32_t k = threadIdx.x; k < kShiftKeys; k += blockDim.x) hist[k] = 0;
  __syncthreads();
  if (g0 < g1) for_each_term(A, M, g0, g1, [&](uint32_t, uint32_t, uint32_t key) {
    atomicAdd(&hist[key], 1u);
  });
  __syncthreads();
  if constexpr (!SCATTER) {
    for (uint32_t k = threadIdx.x; k < kShiftKeys; k += blockDim.x)
      if (hist[k]) atomicAdd(&counts[k], hist[k]);
  } else {
    // counts holds each key's next free position (an exclusive scan of the key totals)
    for (uint32_t k = threadIdx.x; k < kShiftKeys; k += blockDim.x) {
      base[k] = hist[k] ? atomicAdd(&counts[k], hist[k]) : 0u;
      hist[k] = 0;
    }
    __syncthreads();
    if (g0 < g1) for_each_term(A, M, g0, g1, [&](uint32_t v, uint32_t c, uint32_t key) {
      const uint32_t pos = base[key] + atomicAdd(&hist[key], 1u);
      vi[pos] = v;
      cc[pos] = c;
      keys[pos] = (uint16_t)key;
    });
  }
}

// counts[k] <- sum of counts[0..k) over the kShiftKeys keys, in one CTA of 1024 threads.
__global__ void __launch_bounds__(1024) exclusive_scan_keys_kernel(uint32_t* counts) {
  __shared__ uint32_t part[1024];
  constexpr uint32_t per = kShiftKeys / 1024;
  uint32_t v[per], sum = 0;
  for (uint32_t i = 0; i < per; i++) {
    v[i] = counts[threadIdx.x * per + i];
    sum += v[i];
  }
  part[threadIdx.x] = sum;
  __syncthreads();
  for (uint32_t off = 1; off < 1024; off <<= 1) {  // inclusive scan of the per-thread sums
    const uint32_t x = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
    __syncthreads();
    part[threadIdx.x] += x;
    __syncthreads();
  }
  uint32_t run = part[threadIdx.x] - sum;
  for (uint32_t i = 0; i < per; i++) {
    counts[threadIdx.x * per + i] = run;
    run += v[i];
  }
}

__global__ void word_count_kernel(const uint32_t* __restrict__ vi, uint64_t n,
                                  uint32_t* __restrict__ counts) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n;
       t += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(&counts[vi[t]], 1u);
}

// cursor[w] starts at word w's first slot; each term takes the next one (the order of a word's
// terms is immaterial: the monster sums them in GF(2^128)).
__global__ void word_scatter_kernel(const uint32_t* __restrict__ vi, const uint32_t* __restrict__ c,
                                    const uint16_t* __restrict__ key, uint64_t n,
                                    uint32_t* __restrict__ cursor, uint32_t* __restrict__ w_c,
                                    uint16_t* __restrict__ w_key) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t pos = atomicAdd(&cursor[vi[t]], 1u);
    w_c[pos] = c[t];
    w_key[pos] = key[t];
  }
}

// Groups the key-sorted terms by word (a counting sort: per-word counts on the device, their
// exclusive scan on the host, a scatter), for the monster multilinear's per-word sums, and
// records the word each kMonsterChunk-term chunk of that order starts in.
int build_word_order(ShiftTerms& t, uint32_t n_words) {
  const size_t m = t.n ? t.n : 1;
  uint32_t* cursor = nullptr;
  cudaStream_t s = nullptr;
  cudaError_t e;
  std::vector<uint32_t> h((size_t)n_words + 1, 0), chunk_word;
  const unsigned blocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((t.n + 255) / 256, 148 * 16));
  do {
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) break;
    if ((e = cudaMalloc(&t.w_off, 4 * ((size_t)n_words + 1))) != cudaSuccess) break;
    if ((e = cudaMalloc(&t.w_c, 4 * m)) != cudaSuccess) break;
    if ((e = cudaMalloc(&t.w_key, 2 * m)) != cudaSuccess) break;
    if ((e = cudaMalloc(&cursor, 4 * ((size_t)n_words + 1))) != cudaSuccess) break;
    if ((e = cudaMemsetAsync(cursor, 0, 4 * (size_t)n_words, s)) != cudaSuccess) break;
    if (t.n) word_count_kernel<<<blocks, 256, 0, s>>>(t.vi, t.n, cursor);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    if ((e = cudaMemcpyAsync(h.data(), cursor, 4 * (size_t)n_words, cudaMemcpyDeviceToHost, s)) !=
        cudaSuccess)
      break;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) break;
    uint32_t run = 0;
    for (uint32_t w = 0; w <= n_words; w++) {
      const uint32_t c = w < n_words ? h[w] : 0;
      h[w] = run;
      run += c;
    }
    const uint64_t n_chunks = (t.n + kMonsterChunk - 1) / kMonsterChunk;
    chunk_word.assign(n_chunks ? n_chunks : 1, 0);
    for (uint32_t w = 0; w < n_words; w++)  // chunks that start inside word w's terms
      for (uint64_t j = ((uint64_t)h[w] + kMonsterChunk - 1) / kMonsterChunk;
           j * kMonsterChunk < h[w + 1]; j++)
        chunk_word[j] = w;
    if ((e = cudaMalloc(&t.w_chunk, 4 * chunk_word.size())) != cudaSuccess) break;
    if ((e = cudaMemcpyAsync(t.w_chunk, chunk_word.data(), 4 * chunk_word.size(),
                             cudaMemcpyHostToDevice, s)) != cudaSuccess)
      break;
    if ((e = cudaMemcpyAsync(t.w_off, h.data(), 4 * h.size(), cudaMemcpyHostToDevice, s)) !=
        cudaSuccess)
      break;
    if ((e = cudaMemcpyAsync(cursor, t.w_off, 4 * (size_t)n_words, cudaMemcpyDeviceToDevice, s)) !=
        cudaSuccess)
      break;
    if (t.n) word_scatter_kernel<<<blocks, 256, 0, s>>>(t.vi, t.c, t.key, t.n, cursor, t.w_c, t.w_key);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    e = cudaStreamSynchronize(s);
  } while (0);
  if (s) cudaStreamDestroy(s);
  cudaFree(cursor);
  if (e != cudaSuccess) return cuda_error(e, "shift term word order");
  t.n_words = n_words;
  count_launch(t.n ? 2 : 0);
  return BINIUS_OK;
}

int build_shift_terms(const DevOperands& A, const DevOperands& M, uint32_t n_words,
                      ShiftTerms& d) {
  const uint64_t n = A.n_terms + M.n_terms;
  BGPU_ARG(n < 0xffffffffull, "too many operand terms");
  const size_t m = n ? n : 1;
  ShiftTerms t;
  t.n = n;
  uint32_t* counts = nullptr;
  cudaStream_t s = nullptr;  // its own stream: set-up does not wait for other work on the device
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaMalloc(&t.vi, 4 * m)) != cudaSuccess || (e = cudaMalloc(&t.c, 4 * m)) != cudaSuccess ||
      (e = cudaMalloc(&t.key, 2 * m)) != cudaSuccess ||
      (e = cudaMalloc(&counts, 4 * kShiftKeys)) != cudaSuccess ||
      (e = cudaMemsetAsync(counts, 0, 4 * kShiftKeys, s)) != cudaSuccess) {
    cudaFree(t.vi);
    cudaFree(t.c);
    cudaFree(t.key);
    cudaFree(counts);
    if (s) cudaStreamDestroy(s);
    return cuda_error(e, "shift term table");
  }
  shift_terms_kernel<false><<<kSortBlocks, kSortThreads, 0, s>>>(A, M, counts, t.vi, t.c, t.key);
  exclusive_scan_keys_kernel<<<1, 1024, 0, s>>>(counts);
  shift_terms_kernel<true><<<kSortBlocks, kSortThreads, 0, s>>>(A, M, counts, t.vi, t.c, t.key);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  cudaFree(counts);
  if (e != cudaSuccess) {
    cudaFree(t.vi);
    cudaFree(t.c);
    cudaFree(t.key);
    return cuda_error(e, "shift term sort");
  }
  count_launch(3);
  if (int rc = build_word_order(t, n_words)) {
    free_shift_terms(t);
    return rc;
  }
  d = t;
  return BINIUS_OK;
}

}  // namespace

namespace bgpu {

void free_shift_terms(ShiftTerms& t) {
  cudaFree(t.vi);
  cudaFree(t.c);
  cudaFree(t.key);
  cudaFree(t.w_off);
  cudaFree(t.w_c);
  cudaFree(t.w_key);
  cudaFree(t.w_chunk);
  t = ShiftTerms();
}

int upload_shift_terms(const std::vector<uint32_t>& vi, const std::vector<uint32_t>& c,
                       const std::vector<uint16_t>& key, uint64_t n, uint32_t n_words,
                       ShiftTerms& out) {
  const size_t m = n ? n : 1;
  ShiftTerms d;
  d.n = n;
  cudaError_t e;
  if ((e = cudaMalloc(&d.vi, 4 * m)) != cudaSuccess || (e = cudaMalloc(&d.c, 4 * m)) != cudaSuccess ||
      (e = cudaMalloc(&d.key, 2 * m)) != cudaSuccess ||
      (e = cudaMemcpy(d.vi, vi.data(), 4 * m, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(d.c, c.data(), 4 * m, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(d.key, key.data(), 2 * m, cudaMemcpyHostToDevice)) != cudaSuccess) {
    cudaFree(d.vi);
    cudaFree(d.c);
    cudaFree(d.key);
    return cuda_error(e, "shift term table");
  }
  if (int rc = build_word_order(d, n_words)) {
    free_shift_terms(d);
    return rc;
  }
  free_shift_terms(out);
  out = d;
  return BINIUS_OK;
}

// ConstraintSystem::deserialize + ValueVecLayout::validate + validate_and_prepare's padding, on
// the host only (no device state).
int parse_cs(const void* h_bytes, size_t len, binius_cs& cs) {
  Reader r{static_cast<const uint8_t*>(h_bytes), len};
  uint32_t version = r.u32();
  BGPU_ARG(r.ok && version == 2, "ConstraintSystem::version must be 2");
  uint32_t* fields[8] = {&cs.n_const,      &cs.n_inout,         &cs.n_witness,
                         &cs.n_internal,   &cs.offset_inout,    &cs.offset_witness,
                         &cs.committed_total_len, &cs.n_scratch};
  for (auto f : fields) *f = r.u32();
  uint32_t n_constants = r.u32();
  BGPU_ARG(r.ok, "constraint system bytes truncated");
  // ValueVecLayout::validate (constraint_system.rs:686-703)
  BGPU_ARG(is_pow2(cs.committed_total_len), "ValueVecLenNotPowerOfTwo");
  BGPU_ARG(is_pow2(cs.offset_witness), "PublicInputPowerOfTwo");
  BGPU_ARG(cs.offset_witness >= 2, "PublicInputTooShort");
  BGPU_ARG(n_constants == cs.n_const && n_constants <= (1u << 24),
           "ConstraintSystem::constants length != n_const");
  for (uint32_t i = 0; i < n_constants; i++) cs.constants.push_back(r.u64());
  uint32_t n_and = r.u32();
  if (int rc = parse_operands(r, n_and, 3, cs.committed_total_len, cs.h_and)) return rc;
  uint32_t n_mul = r.u32();
  if (int rc = parse_operands(r, n_mul, 4, cs.committed_total_len, cs.h_mul)) return rc;
  cs.n_and_real = n_and;
  cs.n_mul_real = n_mul;
  pad_operands(cs.h_and, next_pow2_at_least(n_and, 8));
  pad_operands(cs.h_mul, next_pow2_at_least(n_mul, 1));
  return BINIUS_OK;
}

int eval_operands(const DevOperands& ops, const uint64_t* d_witness, uint64_t* d_out,
                  cudaStream_t s) {
  const uint64_t groups = (uint64_t)ops.n_constraints * ops.k;
  if (groups == 0) return BINIUS_OK;
  unsigned blocks = (unsigned)std::min<uint64_t>((groups + 255) / 256, 148 * 16);
  eval_operands_kernel<<<blocks, 256, 0, s>>>(ops.offsets, ops.terms, d_witness,
                                              ops.n_constraints, ops.k, d_out);
  BGPU_LAUNCH_CHECK("eval_operands_kernel");
  count_launch();
  return BINIUS_OK;
}

}  // namespace bgpu

extern "C" {

int binius_cs_from_bytes(int device, const void* h_bytes, size_t len, binius_cs** out) {
  BGPU_ARG(out != nullptr && (h_bytes != nullptr || len == 0), "NULL argument");
  *out = nullptr;
  if (int rc = configure_device_pool(device)) return rc;
  binius_cs* cs = new binius_cs();
  cs->device = device;
  int rc = parse_cs(h_bytes, len, *cs);
  if (!rc) {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    rc = upload(cs->h_and, cs->and_ops);
    if (!rc) rc = upload(cs->h_mul, cs->mul_ops);
    if (!rc)
      rc = build_shift_terms(cs->and_ops, cs->mul_ops, cs->committed_total_len, cs->shift_terms);
    cudaSetDevice(prev);
  }
  if (rc) {
    binius_cs_destroy(cs);
    return rc;
  }
  *out = cs;
  return clear_error();
}

int binius_cs_destroy(binius_cs* cs) {
  if (!cs) return BINIUS_OK;
  cudaFree(cs->and_ops.offsets);
  cudaFree(cs->and_ops.terms);
  cudaFree(cs->mul_ops.offsets);
  cudaFree(cs->mul_ops.terms);
  free_shift_terms(cs->shift_terms);
  delete cs;
  return BINIUS_OK;
}

int binius_cs_info(const binius_cs* cs, uint32_t* h_out12) {
  BGPU_ARG(cs && h_out12, "NULL argument");
  uint32_t v[12] = {cs->n_const,      cs->n_inout,         cs->n_witness,     cs->n_internal,
                    cs->offset_inout, cs->offset_witness,  cs->committed_total_len, cs->n_scratch,
                    cs->and_ops.n_constraints, cs->mul_ops.n_constraints, cs->n_and_real,
                    cs->n_mul_real};
  memcpy(h_out12, v, sizeof(v));
  return clear_error();
}

int binius_eval_operands(const binius_cs* cs, const void* d_witness, int which, void* d_out,
                         void* stream) {
  BGPU_ARG(cs && d_witness && d_out, "NULL argument");
  BGPU_ARG(which == 0 || which == 1, "which must be 0 (AND) or 1 (MUL)");
  return eval_operands(which == 0 ? cs->and_ops : cs->mul_ops,
                       static_cast<const uint64_t*>(d_witness), static_cast<uint64_t*>(d_out),
                       as_stream(stream))
             ? BINIUS_E_CUDA
             : clear_error();
}

}  // extern "C"
