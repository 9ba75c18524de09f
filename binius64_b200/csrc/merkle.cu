// Binary Merkle tree commit with SHA-256 leaves and the Binius SHA-256 node compression.
//
// Layout follows BinaryMerkleTree::inner_nodes (prover/prover/src/merkle_tree/binary_merkle_tree.rs
// :65-122): 2^(L+1) - 1 digests of 32 bytes, the 2^L leaf digests first, then each layer, the root
// last; node i of layer k+1 compresses nodes 2i and 2i+1 of layer k (parallel_compression.rs:79-91).
//
// B200 mapping: one thread hashes one leaf (its 2^log_batch elements are read as 128-bit loads);
// the CTA's 256 leaf digests stay in shared memory and the next 8 tree layers are compressed there
// before anything but the layer outputs touches HBM.  Upper layers run in CTAs that fuse 9 layers
// (512 inputs -> 1).  SHA-256 is pure integer work (funnel-shift rotates, three-input logic ops, adds).
#include <string.h>

#include <algorithm>
#include <mutex>

#include "host_sha256.h"
#include "internal.h"
#include "sha256.cuh"

using namespace bgpu;

namespace {

constexpr uint32_t kLeafFuse = 8;  // at most 2^8 leaves per CTA (Tuning::merkle_leaf_fuse)
constexpr uint32_t kNodeFuse = 9;  // at most 2^9 inputs per CTA (Tuning::merkle_node_fuse)

__host__ __device__ __forceinline__ uint64_t layer_offset(uint32_t L, uint32_t k) {
  return (1ull << (L + 1)) - (1ull << (L + 1 - k));
}

__device__ __forceinline__ void store_digest(uint4* nodes, uint64_t i, const uint32_t d[8]) {
  nodes[2 * i] = make_uint4(d[0], d[1], d[2], d[3]);
  nodes[2 * i + 1] = make_uint4(d[4], d[5], d[6], d[7]);
}

__device__ __forceinline__ void load_digest(const uint4* nodes, uint64_t i, uint32_t d[8]) {
  uint4 a = nodes[2 * i], b = nodes[2 * i + 1];
  d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w;
  d[4] = b.x; d[5] = b.y; d[6] = b.z; d[7] = b.w;
}

// Hashes 2^fused leaves per CTA and compresses `fused` layers above them in shared memory.
__global__ void __launch_bounds__(256) merkle_leaves_kernel(const uint4* __restrict__ elems,
                                                            uint32_t log_batch,
                                                            uint4* __restrict__ nodes, uint32_t L,
                                                            uint32_t fused, NodeIV iv) {
  __shared__ uint32_t buf[2][256][9];  // padded rows avoid bank conflicts
  const uint32_t tid = threadIdx.x;
  const uint64_t leaf = (uint64_t)blockIdx.x * blockDim.x + tid;
  uint32_t d[8];
  sha256_elems(elems + (leaf << log_batch), 1u << log_batch, d);
  store_digest(nodes, leaf, d);
#pragma unroll
  for (int i = 0; i < 8; i++) buf[0][tid][i] = d[i];
  for (uint32_t lvl = 1; lvl <= fused; lvl++) {
    __syncthreads();
    const uint32_t n = blockDim.x >> lvl;
    if (tid < n) {
      const uint32_t src = (lvl - 1) & 1, dst = lvl & 1;
      uint32_t l[8], r[8], o[8];
#pragma unroll
      for (int i = 0; i < 8; i++) {
        l[i] = buf[src][2 * tid][i];
        r[i] = buf[src][2 * tid + 1][i];
      }
      compress_node(iv, l, r, o);
#pragma unroll
      for (int i = 0; i < 8; i++) buf[dst][tid][i] = o[i];
      store_digest(nodes, layer_offset(L, lvl) + (uint64_t)blockIdx.x * n + tid, o);
    }
  }
}

// Compresses `fused` layers starting from layer in_level; each CTA reduces 2^fused inputs.
__global__ void __launch_bounds__(256) merkle_nodes_kernel(uint4* __restrict__ nodes, uint32_t L,
                                                           uint32_t in_level, uint32_t fused,
                                                           NodeIV iv) {
  __shared__ uint32_t buf[2][256][9];
  const uint32_t tid = threadIdx.x;
  const uint64_t in_off = layer_offset(L, in_level);
  uint32_t l[8], r[8], o[8];
  {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + tid;
    load_digest(nodes, in_off + 2 * i, l);
    load_digest(nodes, in_off + 2 * i + 1, r);
    compress_node(iv, l, r, o);
    store_digest(nodes, layer_offset(L, in_level + 1) + i, o);
#pragma unroll
    for (int k = 0; k < 8; k++) buf[1][tid][k] = o[k];
  }
  for (uint32_t lvl = 2; lvl <= fused; lvl++) {
    __syncthreads();
    const uint32_t n = (blockDim.x * 2) >> lvl;
    if (tid < n) {
      const uint32_t src = (lvl - 1) & 1, dst = lvl & 1;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        l[k] = buf[src][2 * tid][k];
        r[k] = buf[src][2 * tid + 1][k];
      }
      compress_node(iv, l, r, o);
#pragma unroll
      for (int k = 0; k < 8; k++) buf[dst][tid][k] = o[k];
      store_digest(nodes, layer_offset(L, in_level + lvl) + (uint64_t)blockIdx.x * n + tid, o);
    }
  }
}

}  // namespace

namespace bgpu {

// Sha256Compression::default (hash/compress.rs:37-44): the digest bytes of
// "BINIUS SHA-256 COMPRESS" reinterpreted as native little-endian u32 words.
NodeIV node_iv() {
  static NodeIV iv;
  static std::once_flag once;
  std::call_once(once, [] {
    const char* tag = "BINIUS SHA-256 COMPRESS";
    uint8_t d[32];
    HostSha256::oneshot(reinterpret_cast<const uint8_t*>(tag), strlen(tag), d);
    for (int i = 0; i < 8; i++)
      iv.w[i] = (uint32_t)d[4 * i] | ((uint32_t)d[4 * i + 1] << 8) |
                ((uint32_t)d[4 * i + 2] << 16) | ((uint32_t)d[4 * i + 3] << 24);
  });
  return iv;
}

int merkle_commit(const void* d_elems, uint32_t log_leaves, uint32_t log_batch, void* d_nodes,
                  cudaStream_t stream) {
  BGPU_ARG(d_elems != nullptr && d_nodes != nullptr, "elems / nodes is NULL");
  BGPU_ARG(log_leaves <= 34, "too many leaves");
  BGPU_ARG(log_batch <= 20, "leaf too large");
  const uint32_t L = log_leaves;
  const NodeIV iv = node_iv();
  uint4* nodes = static_cast<uint4*>(d_nodes);
  const uint32_t leaf_fuse = std::max(5u, std::min(kLeafFuse, tuning().merkle_leaf_fuse));
  const uint32_t node_fuse = std::max(5u, std::min(kNodeFuse, tuning().merkle_node_fuse));
  uint32_t fused = std::min(L, leaf_fuse);
  uint64_t grid = 1ull << (L - fused);
  BGPU_ARG(grid <= 0x7fffffffull, "too many leaves");
  merkle_leaves_kernel<<<(unsigned)grid, 1u << fused, 0, stream>>>(
      static_cast<const uint4*>(d_elems), log_batch, nodes, L, fused, iv);
  BGPU_LAUNCH_CHECK("merkle_leaves_kernel");
  count_launch();
  uint32_t level = fused;
  while (level < L) {
    uint32_t f = std::min(L - level, node_fuse);
    uint64_t g = 1ull << (L - level - f);
    merkle_nodes_kernel<<<(unsigned)g, 1u << (f - 1), 0, stream>>>(nodes, L, level, f, iv);
    BGPU_LAUNCH_CHECK("merkle_nodes_kernel");
    count_launch();
    level += f;
  }
  return clear_error();
}

}  // namespace bgpu

extern "C" {

int binius_merkle_commit(const void* d_elems, uint32_t log_leaves, uint32_t log_batch,
                         void* d_nodes, void* stream) {
  return bgpu::merkle_commit(d_elems, log_leaves, log_batch, d_nodes, as_stream(stream));
}

int binius_merkle_branch(const void* d_nodes, uint32_t log_leaves, uint64_t index,
                         uint32_t layer_depth, void* h_branch, void* stream) {
  BGPU_ARG(d_nodes != nullptr && h_branch != nullptr, "nodes / branch is NULL");
  BGPU_ARG(log_leaves <= 40, "log_leaves too large");
  BGPU_ARG(index < (1ull << log_leaves) && layer_depth <= log_leaves, "index out of range");
  cudaStream_t s = as_stream(stream);
  const uint8_t* nodes = static_cast<const uint8_t*>(d_nodes);
  uint8_t* out = static_cast<uint8_t*>(h_branch);
  for (uint32_t j = 0; j < log_leaves - layer_depth; j++) {
    uint64_t node = layer_offset(log_leaves, j) | ((index >> j) ^ 1);
    BGPU_CUDA(cudaMemcpyAsync(out + 32 * j, nodes + 32 * node, 32, cudaMemcpyDeviceToHost, s));
  }
  BGPU_CUDA(stream_wait(s));
  return clear_error();
}

int binius_merkle_layer(const void* d_nodes, uint32_t log_leaves, uint32_t layer_depth,
                        void* h_out, void* stream) {
  BGPU_ARG(d_nodes != nullptr && h_out != nullptr, "nodes / out is NULL");
  BGPU_ARG(log_leaves <= 40, "log_leaves too large");
  BGPU_ARG(layer_depth <= log_leaves, "IncorrectLayerDepth");
  // BinaryMerkleTree::layer: the 2^depth digests that end 2^depth - 1 digests before the end
  const uint64_t total = (2ull << log_leaves) - 1;
  const uint64_t start = total + 1 - (2ull << layer_depth);
  if (int rc = read_sync(h_out, static_cast<const uint8_t*>(d_nodes) + 32 * start,
                         32ull << layer_depth, as_stream(stream)))
    return rc;
  return clear_error();
}

}  // extern "C"
