// Additive NTT (LCH14 "neighbors-last" form) and Reed-Solomon encode over GF(2^128).
//
// Semantics follow NeighborsLastReference (verifier/math/src/ntt/reference.rs:20-76): layer l acts
// on index bit (log_d - l - 1); block = idx >> (log_d - l) selects twiddle(l, block) =
// expanded[l][block] (GenericPreExpanded, ntt/domain_context.rs:99-159); the forward butterfly is
// u += v*t; v += u.  Field arithmetic is exact, so any evaluation order gives identical bits.
//
// B200 mapping: a pass fuses up to 8 consecutive layers.  One CTA owns a tile of 2^(k+c) elements
// (k butterfly bits plus c contiguous low index bits for coalescing) resident in shared memory
// together with the 2^k - 1 twiddles the tile needs, so each pass reads and writes HBM once with
// 128-bit accesses.  Reed-Solomon encode (reed_solomon.rs:128-201) fuses the message bit reversal
// and the 2^R-fold replication into the first pass's load: for the first pass the butterfly bits
// are exactly the message's low index bits after reversal, so the gather stays coalesced.
#include <algorithm>
#include <vector>

#include "gf128.cuh"
#include "internal.h"

using namespace bgpu;

namespace {

constexpr int kNttThreads = 256;
constexpr uint32_t kTileBits = 12;  // the largest tile: 4096 elements = 64 KiB of shared memory
constexpr uint32_t kMaxPassLayers = 8;

struct NttPass {
  uint32_t log_d;    // index bits of the whole buffer
  uint32_t l0;       // first layer of the pass
  uint32_t k;        // layers in the pass
  uint32_t c;        // contiguous low index bits in a tile
  uint32_t rs_bits;  // RS load: message index bits (bit-reversal width)
};

__device__ __forceinline__ uint32_t rev_bits32(uint32_t x, uint32_t n) {
  return n ? (__brev(x) >> (32 - n)) : 0u;
}
__device__ __forceinline__ uint64_t rev_bits64(uint64_t x, uint32_t n) {
  return n ? (__brevll(x) >> (64 - n)) : 0ull;
}

// twiddle(layer, j) = XOR of row[log_domain-1-layer][k+1] over the set bits k of j.
__global__ void expand_twiddles_kernel(uint4* __restrict__ tw, const uint4* __restrict__ rows,
                                       const uint32_t* __restrict__ row_offsets,
                                       uint32_t log_domain, uint64_t total) {
  for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t layer = 63 - __clzll(idx + 1);
    uint64_t j = idx + 1 - (1ull << layer);
    const uint4* r = rows + row_offsets[log_domain - 1 - layer];
    uint4 acc = gf_zero();
    for (uint32_t k = 0; k < layer; k++)
      if ((j >> k) & 1) gf_add_into(acc, r[k + 1]);
    tw[idx] = acc;
  }
}

template <bool INVERSE, bool RS>
__global__ void __launch_bounds__(kNttThreads)
    ntt_pass_kernel(uint4* __restrict__ data, const uint4* __restrict__ src,
                    const uint4* __restrict__ tw, NttPass p) {
  extern __shared__ uint4 smem[];
  const uint32_t k = p.k, c = p.c;
  const uint32_t tile_elems = 1u << (k + c);
  uint4* tile = smem;
  uint4* twl = smem + tile_elems;
  const uint32_t s = p.log_d - p.l0 - k;  // lowest butterfly index bit
  const uint64_t t = blockIdx.x;
  const uint64_t outer_mid = t & ((1ull << (s - c)) - 1);
  const uint64_t outer_hi = t >> (s - c);
  const uint64_t base = (outer_hi << (s + k)) | (outer_mid << c);

  // Twiddles of this tile: layer l0+m uses blocks (outer_hi << m) + [0, 2^m).
  for (uint32_t i = threadIdx.x; i + 1 < (1u << k); i += blockDim.x) {
    uint32_t m = 31 - __clz(i + 1);
    uint32_t j = i + 1 - (1u << m);
    uint64_t layer = p.l0 + m;
    twl[i] = __ldg(tw + ((1ull << layer) - 1) + (outer_hi << m) + j);
  }
  if (RS) {
    const uint64_t msg_mask = (p.rs_bits == 64) ? ~0ull : ((1ull << p.rs_bits) - 1);
    for (uint32_t e2 = threadIdx.x; e2 < tile_elems; e2 += blockDim.x) {
      uint32_t bfly = rev_bits32(e2 & ((1u << k) - 1), k);
      uint32_t inner = e2 >> k;
      uint64_t g = base | ((uint64_t)bfly << s) | inner;
      uint64_t si = rev_bits64(g & msg_mask, p.rs_bits);
      tile[(bfly << c) | inner] = __ldg(src + si);
    }
  } else {
    for (uint32_t e = threadIdx.x; e < tile_elems; e += blockDim.x) {
      uint64_t g = base | ((uint64_t)(e >> c) << s) | (e & ((1u << c) - 1));
      tile[e] = data[g];
    }
  }
  __syncthreads();

  const uint32_t half = tile_elems >> 1;
  for (uint32_t mm = 0; mm < k; mm++) {
    const uint32_t m = INVERSE ? (k - 1 - mm) : mm;
    const uint32_t h = c + k - 1 - m;
    for (uint32_t q = threadIdx.x; q < half; q += blockDim.x) {
      uint32_t e0 = ((q >> h) << (h + 1)) | (q & ((1u << h) - 1));
      uint32_t e1 = e0 | (1u << h);
      uint4 twd = twl[(1u << m) - 1 + (e0 >> (c + k - m))];
      uint4 u = tile[e0], v = tile[e1];
      if (!INVERSE) {
        gf_add_into(u, gf_mul(v, twd));
        gf_add_into(v, u);
      } else {
        gf_add_into(v, u);
        gf_add_into(u, gf_mul(v, twd));
      }
      tile[e0] = u;
      tile[e1] = v;
    }
    __syncthreads();
  }

  for (uint32_t e = threadIdx.x; e < tile_elems; e += blockDim.x) {
    uint64_t g = base | ((uint64_t)(e >> c) << s) | (e & ((1u << c) - 1));
    data[g] = tile[e];
  }
}

std::vector<NttPass> plan_passes(uint32_t log_d, uint32_t skip_early, uint32_t skip_late,
                                 bool rs, uint32_t rs_bits) {
  // tiles of 2^tile_bits elements: fewer, larger tiles fuse more work per CTA; more, smaller ones
  // spread a small transform evenly over the 148 SMs (a 2^20 codeword is 256 tiles of 2^12)
  const uint32_t tile_bits = std::max(9u, std::min(kTileBits, tuning().ntt_tile_bits));
  std::vector<NttPass> passes;
  uint32_t n_layers = log_d - skip_late - skip_early;
  if (n_layers == 0) {
    if (rs) {
      uint32_t s = log_d - skip_early;
      passes.push_back({log_d, skip_early, 0, std::min(tile_bits, s), rs_bits});
    }
    return passes;
  }
  const uint32_t max_layers =
      std::max(1u, std::min({kMaxPassLayers, tuning().ntt_pass_layers, tile_bits}));
  uint32_t n_passes = (n_layers + max_layers - 1) / max_layers;
  uint32_t base = n_layers / n_passes, extra = n_layers % n_passes;
  uint32_t l0 = skip_early;
  for (uint32_t i = 0; i < n_passes; i++) {
    uint32_t k = base + (i < extra ? 1 : 0);
    uint32_t s = log_d - l0 - k;
    uint32_t c = std::min(tile_bits - k, s);
    passes.push_back({log_d, l0, k, c, i == 0 ? rs_bits : 0u});
    l0 += k;
  }
  return passes;
}

template <bool INVERSE, bool RS>
int launch_pass(const NttPass& p, uint4* data, const uint4* src, const uint4* tw,
                cudaStream_t stream) {
  size_t smem = ((size_t(1) << (p.k + p.c)) + (size_t(1) << p.k) - 1) * sizeof(uint4);
  auto kern = ntt_pass_kernel<INVERSE, RS>;
  // the largest tile of any pass: 2^kTileBits elements plus 2^kMaxPassLayers - 1 twiddles
  constexpr size_t kMaxSmem = ((size_t(1) << kTileBits) + (size_t(1) << kMaxPassLayers) - 1) *
                              sizeof(uint4);
  if (smem > kMaxSmem) return set_error(BINIUS_E_ARG, "ntt: pass tile exceeds the planned maximum");
  if (int rc = ensure_smem_limit(reinterpret_cast<const void*>(kern), kMaxSmem)) return rc;
  uint64_t n_tiles = 1ull << (p.log_d - p.k - p.c);
  if (n_tiles > 0x7fffffffull) return set_error(BINIUS_E_ARG, "ntt: buffer too large");
  kern<<<(unsigned)n_tiles, kNttThreads, smem, stream>>>(data, src, tw, p);
  BGPU_LAUNCH_CHECK("ntt_pass_kernel");
  count_launch();
  return BINIUS_OK;
}

int check_device(const binius_ntt* ntt) {
  int dev = -1;
  BGPU_CUDA(cudaGetDevice(&dev));
  if (dev != ntt->device)
    return set_error(BINIUS_E_ARG, "binius_ntt used on a device other than the one it was built on");
  return BINIUS_OK;
}

int ntt_transform(const binius_ntt* ntt, void* d_data, uint32_t log_len, uint32_t skip_early,
                  uint32_t skip_late, void* stream, bool inverse) {
  BGPU_ARG(ntt != nullptr, "ntt is NULL");
  BGPU_ARG(d_data != nullptr || log_len == 0, "data is NULL");
  BGPU_ARG(log_len <= 40, "log_len too large");
  // input_check (ntt/reference.rs:85-100)
  BGPU_ARG(skip_early + skip_late <= log_len, "skip_early + skip_late must be <= log_len");
  BGPU_ARG(log_len - skip_late <= ntt->log_domain, "domain context too small for the transform");
  if (int rc = check_device(ntt)) return rc;
  auto passes = plan_passes(log_len, skip_early, skip_late, false, 0);
  uint4* data = static_cast<uint4*>(d_data);
  const uint4* tw = static_cast<const uint4*>(ntt->d_twiddles);
  cudaStream_t s = as_stream(stream);
  if (!inverse) {
    for (const auto& p : passes)
      if (int rc = launch_pass<false, false>(p, data, nullptr, tw, s)) return rc;
  } else {
    for (auto it = passes.rbegin(); it != passes.rend(); ++it)
      if (int rc = launch_pass<true, false>(*it, data, nullptr, tw, s)) return rc;
  }
  return clear_error();
}

}  // namespace

namespace bgpu {

int rs_encode_batch(const binius_ntt* ntt, const void* d_msg, uint32_t log_dim,
                    uint32_t log_inv_rate, uint32_t log_batch, void* d_codeword,
                    cudaStream_t stream) {
  BGPU_ARG(ntt != nullptr, "ntt is NULL");
  BGPU_ARG(d_msg != nullptr && d_codeword != nullptr, "msg / codeword is NULL");
  BGPU_ARG(d_msg != d_codeword, "codeword must not alias the message");
  uint32_t log_msg = log_dim + log_batch;
  uint32_t log_out = log_msg + log_inv_rate;
  BGPU_ARG(log_out <= 40, "codeword too large");
  // encode_batch requires the NTT subspace of dimension log_len (reed_solomon.rs:143-145)
  BGPU_ARG(log_dim + log_inv_rate <= ntt->log_domain,
           "NTT domain smaller than the code's evaluation domain");
  if (int rc = check_device(ntt)) return rc;
  auto passes = plan_passes(log_out, log_inv_rate, log_batch, true, log_msg);
  uint4* out = static_cast<uint4*>(d_codeword);
  const uint4* msg = static_cast<const uint4*>(d_msg);
  const uint4* tw = static_cast<const uint4*>(ntt->d_twiddles);
  for (size_t i = 0; i < passes.size(); i++) {
    int rc = (i == 0) ? launch_pass<false, true>(passes[i], out, msg, tw, stream)
                      : launch_pass<false, false>(passes[i], out, nullptr, tw, stream);
    if (rc) return rc;
  }
  return clear_error();
}

}  // namespace bgpu

namespace {

// generate_evals_from_subspace (ntt/domain_context.rs:19-46): row i holds the normalized
// subspace-polynomial evaluations [W_i(b_i), W_i(b_(i+1)), ...] / W_i(b_i) of the domain basis
// (h_basis: l elements, or NULL for BinarySubspace::with_dim's basis x^i).
int subspace_evals(const void* h_basis, uint32_t l, std::vector<std::vector<hu128>>& evals) {
  std::vector<hu128> basis(l);
  for (uint32_t i = 0; i < l; i++) {
    if (h_basis) {
      const uint64_t* b = static_cast<const uint64_t*>(h_basis) + 2 * i;
      basis[i] = ((hu128)b[1] << 64) | b[0];
    } else {
      basis[i] = (hu128)1 << i;
    }
  }
  evals.clear();
  evals.push_back(basis);
  for (uint32_t i = 1; i < l; i++) {
    const auto& prev = evals[i - 1];
    std::vector<hu128> row;
    for (size_t k = 1; k < prev.size(); k++) row.push_back(host_gf_mul(prev[k], prev[k] ^ prev[0]));
    evals.push_back(row);
  }
  for (auto& row : evals) {
    if (row[0] == 0) return set_error(BINIUS_E_ARG, "subspace basis is linearly dependent");
    hu128 inv = host_gf_inv(row[0]);
    for (auto& v : row) v = host_gf_mul(v, inv);
  }
  return BINIUS_OK;
}

}  // namespace

extern "C" {

int binius_domain_subspace(const void* h_basis, uint32_t log_domain, uint32_t dim, void* h_out) {
  BGPU_ARG(h_out != nullptr, "out is NULL");
  BGPU_ARG(log_domain >= 1 && log_domain <= 64, "log_domain must be in [1, 64]");
  BGPU_ARG(dim <= log_domain, "dim must be <= log_domain");
  uint64_t* o = static_cast<uint64_t*>(h_out);
  if (dim == 0) return clear_error();  // BinarySubspace::with_dim(0)
  std::vector<std::vector<hu128>> evals;
  if (int rc = subspace_evals(h_basis, log_domain, evals)) return rc;
  const auto& row = evals[log_domain - dim];
  for (uint32_t i = 0; i < dim; i++) {
    o[2 * i] = (uint64_t)row[i];
    o[2 * i + 1] = (uint64_t)(row[i] >> 64);
  }
  return clear_error();
}

int binius_ntt_create(int device, const void* h_basis, uint32_t log_domain, binius_ntt** out) {
  BGPU_ARG(out != nullptr, "out is NULL");
  *out = nullptr;
  BGPU_ARG(log_domain >= 1 && log_domain <= 32, "log_domain must be in [1, 32]");
  if (int rc = configure_device_pool(device)) return rc;
  const uint32_t l = log_domain;
  std::vector<std::vector<hu128>> evals;
  if (int rc = subspace_evals(h_basis, l, evals)) return rc;
  std::vector<uint32_t> offsets(l);
  std::vector<uint64_t> packed;
  for (uint32_t i = 0; i < l; i++) {
    offsets[i] = (uint32_t)(packed.size() / 2);
    for (hu128 v : evals[i]) {
      packed.push_back((uint64_t)v);
      packed.push_back((uint64_t)(v >> 64));
    }
  }

  int prev_dev = 0;
  BGPU_CUDA(cudaGetDevice(&prev_dev));
  BGPU_CUDA(cudaSetDevice(device));
  uint64_t total = (1ull << l) - 1;
  void* d_tw = nullptr;
  void* d_rows = nullptr;
  void* d_off = nullptr;
  int rc = BINIUS_OK;
  do {
    cudaError_t e = cudaMalloc(&d_tw, total * 16);
    if (e != cudaSuccess) { rc = cuda_error(e, "cudaMalloc(twiddles)"); break; }
    e = cudaMalloc(&d_rows, packed.size() * 8);
    if (e != cudaSuccess) { rc = cuda_error(e, "cudaMalloc(rows)"); break; }
    e = cudaMalloc(&d_off, offsets.size() * 4);
    if (e != cudaSuccess) { rc = cuda_error(e, "cudaMalloc(offsets)"); break; }
    e = cudaMemcpy(d_rows, packed.data(), packed.size() * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { rc = cuda_error(e, "cudaMemcpy(rows)"); break; }
    e = cudaMemcpy(d_off, offsets.data(), offsets.size() * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { rc = cuda_error(e, "cudaMemcpy(offsets)"); break; }
    unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 148ull * 32);
    expand_twiddles_kernel<<<blocks, 256>>>(static_cast<uint4*>(d_tw),
                                            static_cast<const uint4*>(d_rows),
                                            static_cast<const uint32_t*>(d_off), l, total);
    e = cudaGetLastError();
    if (e != cudaSuccess) { rc = cuda_error(e, "expand_twiddles_kernel"); break; }
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { rc = cuda_error(e, "expand_twiddles_kernel sync"); break; }
  } while (0);
  if (d_rows) cudaFree(d_rows);
  if (d_off) cudaFree(d_off);
  if (rc != BINIUS_OK) {
    if (d_tw) cudaFree(d_tw);
    cudaSetDevice(prev_dev);
    return rc;
  }
  binius_ntt* ntt = new binius_ntt;
  ntt->device = device;
  ntt->log_domain = l;
  ntt->d_twiddles = d_tw;
  *out = ntt;
  cudaSetDevice(prev_dev);
  return clear_error();
}

int binius_ntt_destroy(binius_ntt* ntt) {
  if (!ntt) return BINIUS_OK;
  int prev_dev = 0;
  cudaGetDevice(&prev_dev);
  cudaSetDevice(ntt->device);
  cudaFree(ntt->d_twiddles);
  cudaSetDevice(prev_dev);
  delete ntt;
  return BINIUS_OK;
}

uint32_t binius_ntt_log_domain(const binius_ntt* ntt) { return ntt ? ntt->log_domain : 0; }

const void* binius_ntt_twiddles(const binius_ntt* ntt) { return ntt ? ntt->d_twiddles : nullptr; }

int binius_ntt_forward(const binius_ntt* ntt, void* d_data, uint32_t log_len, uint32_t skip_early,
                       uint32_t skip_late, void* stream) {
  return ntt_transform(ntt, d_data, log_len, skip_early, skip_late, stream, false);
}

int binius_ntt_inverse(const binius_ntt* ntt, void* d_data, uint32_t log_len, uint32_t skip_early,
                       uint32_t skip_late, void* stream) {
  return ntt_transform(ntt, d_data, log_len, skip_early, skip_late, stream, true);
}

int binius_rs_encode_batch(const binius_ntt* ntt, const void* d_msg, uint32_t log_dim,
                           uint32_t log_inv_rate, uint32_t log_batch, void* d_codeword,
                           void* stream) {
  return bgpu::rs_encode_batch(ntt, d_msg, log_dim, log_inv_rate, log_batch, d_codeword,
                               as_stream(stream));
}

}  // extern "C"
