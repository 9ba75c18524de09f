// Vision-4 over GF(2^128) GHASH (verifier/verifier/src/hash/vision_4, prover/prover/src/hash/
// vision_4): the permutation, the sponge digest of Merkle leaves (VisionHasherDigest,
// digest.rs:37-136) and the MMO node compression (VisionCompression, compression.rs:24-52), as the
// alternative Merkle hash of the `-c vision4` setup (prover/examples/src/lib.rs:67-85).
//
// Permutation (permutation.rs:104-123): add RC[0]; 16 half rounds of sbox -> MDS -> add RC[h+1],
// the sbox alternating B^-1 (even h) and B (odd h) after an elementwise inversion with 0 -> 0.
// B(x) = c0 + c1 x + c2 x^2 + c3 x^4; B^-1(y) = L^-1(y) + L^-1(c0), L the linear part of B.
// The round constants are derived on the host as compute_round_constants does
// (constants.rs:309-338) from INITIAL_CONSTANT, CONSTANTS_MATRIX and CONSTANTS_CONSTANT.
//
// B200 mapping: one thread runs one permutation chain (a leaf's sponge, then the CTA's fused node
// layers).  All the work is GF(2^128) arithmetic on the integer pipes:
//  * the four inversions of an sbox share one (Montgomery: 9 multiplies + 1 inversion);
//  * an inversion is a^(2^128-2) by the chain a^(2^(2k)-1) = (a^(2^k-1))^(2^k) * a^(2^k-1),
//    a^(2^(2k+1)-1) = (a^(2^(2k)-1))^2 * a: 12 multiplies, and the repeated squarings x^(2^k)
//    for k = 7, 15, 31, 63 as GF(2)-linear maps (one table pass each) while k = 1, 3 square
//    directly (bit spread + reduction);
//  * L and L^-1 are table passes too.  A table pass XORs 32 rows picked by the 32 nibbles of
//    x; the tables are stored as four 32-bit planes so a warp's lookups of one nibble position
//    fall into 16 consecutive words of shared memory (no bank conflicts).
// Six maps x 8 KiB of tables + the round constants stay in shared memory for the kernel's life.
// Trees of up to 2^12 leaves (the FRI fold rounds') run one permutation over four lanes instead,
// which shortens the chain of dependent permutations they are made of (see the lane kernels).
#include <string.h>

#include <mutex>
#include <utility>
#include <vector>

#include "gf128.cuh"
#include "internal.h"
#include "kernels.h"

using namespace bgpu;

namespace {

// ------------------------------------------------------------------ constants (host)

constexpr hu128 H(uint64_t hi, uint64_t lo) { return ((hu128)hi << 64) | lo; }

// B_FWD_COEFFS (constants.rs:11-16): c0 + c1 x + c2 x^2 + c3 x^4
const hu128 kBFwd[4] = {
    H(0xb0b849b207a0f1c7, 0x4c29e4d892ca33dd), H(0xf2240891aac3c3a5, 0x855eeb8ce24c9523),
    H(0xb017e96797ef1fbe, 0x9d79908388dd768d), H(0x2bf9f0b94c2b2ceb, 0x00dbb86a2cb472bb)};
// INITIAL_CONSTANT, CONSTANTS_MATRIX (row-major), CONSTANTS_CONSTANT (constants.rs:283-307)
const hu128 kInitial[4] = {
    H(0xd0e015190f5e0795, 0xf4a1d28234ffdf87), H(0x6111731acd9a89f6, 0xb93ec3a23ec7681b),
    H(0x15da8de707ee3f39, 0x18a34a96728b8d29), H(0x2ea920e89fbb13a1, 0xed2a216b1d232bfb)};
const hu128 kMatrix[16] = {
    H(0x1cac9af051191d2c, 0x8ef96344bc8cbd0f), H(0x3ceb350e8c2d2f4d, 0x4750ab0a854c3a4d),
    H(0x09cc78f7eafef94d, 0x8e092e899156946b), H(0x1d1ad17c8c7ee715, 0xa3d58f7eedb30dbb),
    H(0x06bee572113950b3, 0xdd0cdae9dff5dfc5), H(0x4799c3743a356042, 0x8b4bfa1a5cd3d295),
    H(0x516883bf97b07fcf, 0x4cb89ac6bf636d0b), H(0x0b681d1621d6aa1f, 0xdf1a9113b04d755b),
    H(0xe9ba2f01051f6b4b, 0x3ddfe74c125e99e5), H(0x1f58efc5ecf2e1b9, 0x33e31cfb26b916d1),
    H(0x36da671249b5444c, 0xf67efc573241fe19), H(0x056cae18b867d486, 0x615a130556e5eb99),
    H(0x1d8645dd4b1e46b7, 0x8dd9df84956bcf11), H(0x3efa34e48e3b2183, 0x95efe6255339375b),
    H(0x79bf44bae0d23793, 0x97d0812db56c5eff), H(0x7fb3b7fce84776e3, 0x9e538151daddae85)};
const hu128 kConstant[4] = {
    H(0x0d42981a71a7c2e4, 0x93ca17e6bb10203f), H(0x9ceed672ccb7030f, 0xca17ed48e18717b9),
    H(0x0cec5c463024f2ba, 0x95c6ecdb4a349d15), H(0xa46023576301b995, 0x990418f3a23e3c99)};

// Shared-memory image: six nibble tables, then the round constants and the two affine constants.
enum : uint32_t { kMapLinv = 0, kMapLfwd = 1, kMapSq7 = 2, kMapSq15 = 3, kMapSq31 = 4, kMapSq63 = 5 };
constexpr uint32_t kMaps = 6;
constexpr uint32_t kMapWords = 4 * 32 * 16;  // [plane][nibble position][nibble value]
constexpr uint32_t kRcOff = kMaps * kMapWords / 4;  // in uint4 units
constexpr uint32_t kC0Off = kRcOff + 17 * 4, kBinv0Off = kC0Off + 1;
constexpr size_t kImageBytes = 16 * (kBinv0Off + 1);

hu128 l_fwd(hu128 x) {
  const hu128 x2 = host_gf_mul(x, x), x4 = host_gf_mul(x2, x2);
  return host_gf_mul(kBFwd[1], x) ^ host_gf_mul(kBFwd[2], x2) ^ host_gf_mul(kBFwd[3], x4);
}

hu128 apply_cols(const hu128* cols, hu128 x) {
  hu128 r = 0;
  for (int i = 0; i < 128; i++)
    if ((x >> i) & 1) r ^= cols[i];
  return r;
}

struct HostParams {
  hu128 cols[kMaps][128];  // image of each basis vector under each map
  hu128 rc[17][4];
  hu128 binv0;
};

void h_sbox(hu128 s[4], bool inverse, const HostParams& p) {
  for (int i = 0; i < 4; i++) {
    const hu128 v = s[i] ? host_gf_inv(s[i]) : 0;
    s[i] = inverse ? (apply_cols(p.cols[kMapLinv], v) ^ p.binv0) : (l_fwd(v) ^ kBFwd[0]);
  }
}

void h_mds(hu128 a[4]) {
  auto mul_x = [](hu128 v) { return (v << 1) ^ ((v >> 127) ? (hu128)0x87 : 0); };
  const hu128 sum = a[0] ^ a[1] ^ a[2] ^ a[3], a0 = a[0];
  a[0] ^= sum ^ mul_x(a[0] ^ a[1]);
  a[1] ^= sum ^ mul_x(a[1] ^ a[2]);
  a[2] ^= sum ^ mul_x(a[2] ^ a[3]);
  a[3] ^= sum ^ mul_x(a[3] ^ a0);
}

const HostParams& host_params() {
  static HostParams p;
  static std::once_flag once;
  std::call_once(once, [] {
    for (int i = 0; i < 128; i++) p.cols[kMapLfwd][i] = l_fwd((hu128)1 << i);
    // L^-1 by Gauss-Jordan elimination on the pairs (L(e_i), e_i); L is invertible, so every
    // column finds a pivot
    hu128 v[128], u[128];
    for (int i = 0; i < 128; i++) {
      v[i] = p.cols[kMapLfwd][i];
      u[i] = (hu128)1 << i;
    }
    for (int j = 0; j < 128; j++) {
      int piv = j;
      while (piv < 127 && !((v[piv] >> j) & 1)) piv++;
      std::swap(v[j], v[piv]);
      std::swap(u[j], u[piv]);
      for (int k = 0; k < 128; k++)
        if (k != j && ((v[k] >> j) & 1)) {
          v[k] ^= v[j];
          u[k] ^= u[j];
        }
    }
    for (int j = 0; j < 128; j++) p.cols[kMapLinv][j] = u[j];
    p.binv0 = apply_cols(p.cols[kMapLinv], kBFwd[0]);
    const int sq_k[4] = {7, 15, 31, 63};
    for (int m = 0; m < 4; m++)
      for (int i = 0; i < 128; i++) {
        hu128 x = (hu128)1 << i;
        for (int k = 0; k < sq_k[m]; k++) x = host_gf_mul(x, x);
        p.cols[kMapSq7 + m][i] = x;
      }
    // compute_round_constants
    hu128 state[4], inj[4];
    for (int i = 0; i < 4; i++) p.rc[0][i] = state[i] = inj[i] = kInitial[i];
    int idx = 1;
    for (int r = 0; r < 8; r++)
      for (int half = 0; half < 2; half++) {
        hu128 next[4];
        for (int i = 0; i < 4; i++) {
          next[i] = kConstant[i];
          for (int j = 0; j < 4; j++) next[i] ^= host_gf_mul(kMatrix[4 * i + j], inj[j]);
        }
        for (int i = 0; i < 4; i++) inj[i] = next[i];
        h_sbox(state, half == 0, p);
        h_mds(state);
        for (int i = 0; i < 4; i++) p.rc[idx][i] = state[i] ^= inj[i];
        idx++;
      }
  });
  return p;
}

void put_elem(uint32_t* w, hu128 v) {
  for (int i = 0; i < 4; i++) w[i] = (uint32_t)(v >> (32 * i));
}

// The shared-memory image, uploaded once per device.
int device_image(const uint4** out) {
  static std::mutex mu;
  static const uint4* images[64] = {};
  int dev = 0;
  BGPU_CUDA(cudaGetDevice(&dev));
  BGPU_ARG(dev >= 0 && dev < 64, "device ordinal out of range");
  std::lock_guard<std::mutex> g(mu);
  if (!images[dev]) {
    const HostParams& p = host_params();
    std::vector<uint32_t> img(kImageBytes / 4, 0);
    for (uint32_t m = 0; m < kMaps; m++)
      for (uint32_t pos = 0; pos < 32; pos++)
        for (uint32_t nib = 0; nib < 16; nib++) {
          hu128 v = 0;
          for (int b = 0; b < 4; b++)
            if ((nib >> b) & 1) v ^= p.cols[m][4 * pos + b];
          for (int plane = 0; plane < 4; plane++)
            img[m * kMapWords + plane * 512 + pos * 16 + nib] = (uint32_t)(v >> (32 * plane));
        }
    for (int r = 0; r < 17; r++)
      for (int i = 0; i < 4; i++) put_elem(&img[4 * (kRcOff + 4 * r + i)], p.rc[r][i]);
    put_elem(&img[4 * kC0Off], kBFwd[0]);
    put_elem(&img[4 * kBinv0Off], p.binv0);
    void* d = nullptr;
    BGPU_CUDA(cudaMalloc(&d, kImageBytes));
    BGPU_CUDA(cudaMemcpy(d, img.data(), kImageBytes, cudaMemcpyHostToDevice));
    images[dev] = static_cast<const uint4*>(d);
  }
  *out = images[dev];
  return BINIUS_OK;
}

// ------------------------------------------------------------------ device

extern __shared__ uint4 v4_img[];

__device__ __forceinline__ void v4_load_image(const uint4* __restrict__ g) {
  for (uint32_t i = threadIdx.x; i < kImageBytes / 16; i += blockDim.x) v4_img[i] = g[i];
  __syncthreads();
}

// x -> map_m(x): XOR of the rows selected by x's 32 nibbles.
static __device__ __noinline__ uint4 v4_map(uint32_t m, uint4 x) {
  const uint32_t* T = reinterpret_cast<const uint32_t*>(v4_img) + m * kMapWords;
  const uint32_t w[4] = {x.x, x.y, x.z, x.w};
  uint32_t r0 = 0, r1 = 0, r2 = 0, r3 = 0;
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int n = 0; n < 8; n++) {
      const uint32_t idx = (q * 8 + n) * 16 + ((w[q] >> (4 * n)) & 15);
      r0 ^= T[idx];
      r1 ^= T[512 + idx];
      r2 ^= T[1024 + idx];
      r3 ^= T[1536 + idx];
    }
  return make_uint4(r0, r1, r2, r3);
}

__device__ __forceinline__ uint64_t spread32(uint32_t v) {
  uint64_t x = v;
  x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
  x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
  x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}

// x^2: the bits of x spread to the even positions, then reduced.
__device__ __forceinline__ uint4 gf_square(uint4 a) {
  u256 p;
  p.p0 = spread32(a.x);
  p.p1 = spread32(a.y);
  p.p2 = spread32(a.z);
  p.p3 = spread32(a.w);
  return reduce256(p);
}

// a^(2^128 - 2) (0 -> 0): six doublings of the exponent chain a^(2^k - 1), k = 1, 3, 7, ..., 127.
static __device__ __noinline__ uint4 v4_inv(uint4 a) {
  uint4 b = a;  // a^(2^k - 1), k = 1
#pragma unroll 1
  for (uint32_t j = 0; j < 6; j++) {
    uint4 t;  // b^(2^k)
    if (j == 0) {
      t = gf_square(b);
    } else if (j == 1) {
      t = gf_square(gf_square(gf_square(b)));
    } else {
      t = v4_map(kMapSq7 + (j - 2), b);
    }
    b = gf_mul_nl(t, b);             // a^(2^(2k) - 1)
    b = gf_mul_nl(gf_square(b), a);  // a^(2^(2k+1) - 1)
  }
  return gf_square(b);
}

__device__ __forceinline__ uint4 mul_x(uint4 v) {
  const uint32_t m = 0u - (v.w >> 31);
  return make_uint4((v.x << 1) ^ (0x87u & m), (v.y << 1) | (v.x >> 31), (v.z << 1) | (v.y >> 31),
                    (v.w << 1) | (v.z >> 31));
}

// sbox (permutation.rs:69-73): batch inversion (zeros stay zero), then B^-1 or B.
__device__ __forceinline__ void v4_sbox(uint4 s[4], bool inverse) {
  uint4 z[4];
  bool zero[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    zero[i] = gf_is_zero(s[i]);
    z[i] = zero[i] ? gf_one() : s[i];
  }
  const uint4 p01 = gf_mul_nl(z[0], z[1]), p23 = gf_mul_nl(z[2], z[3]);
  const uint4 q = v4_inv(gf_mul_nl(p01, p23));
  const uint4 q01 = gf_mul_nl(q, p23), q23 = gf_mul_nl(q, p01);
  uint4 inv[4];
  inv[0] = gf_mul_nl(q01, z[1]);
  inv[1] = gf_mul_nl(q01, z[0]);
  inv[2] = gf_mul_nl(q23, z[3]);
  inv[3] = gf_mul_nl(q23, z[2]);
  const uint4 k = v4_img[inverse ? kBinv0Off : kC0Off];
  const uint32_t m = inverse ? kMapLinv : kMapLfwd;
#pragma unroll
  for (int i = 0; i < 4; i++) s[i] = gf_add(v4_map(m, zero[i] ? gf_zero() : inv[i]), k);
}

__device__ __forceinline__ void v4_mds(uint4 a[4]) {
  const uint4 sum = gf_add(gf_add(a[0], a[1]), gf_add(a[2], a[3])), a0 = a[0];
  a[0] = gf_add(a[0], gf_add(sum, mul_x(gf_add(a[0], a[1]))));
  a[1] = gf_add(a[1], gf_add(sum, mul_x(gf_add(a[1], a[2]))));
  a[2] = gf_add(a[2], gf_add(sum, mul_x(gf_add(a[2], a[3]))));
  a[3] = gf_add(a[3], gf_add(sum, mul_x(gf_add(a[3], a0))));
}

__device__ __forceinline__ void v4_add_rc(uint4 s[4], uint32_t r) {
#pragma unroll
  for (int i = 0; i < 4; i++) s[i] = gf_add(s[i], v4_img[kRcOff + 4 * r + i]);
}

static __device__ __noinline__ void v4_permute(uint4 s[4]) {
  v4_add_rc(s, 0);
#pragma unroll 1
  for (uint32_t h = 0; h < 16; h++) {
    v4_sbox(s, (h & 1) == 0);
    v4_mds(s);
    v4_add_rc(s, h + 1);
  }
}

// VisionCompression: (p(x) + x)[0..2] for x = left || right.
__device__ __forceinline__ void v4_compress(const uint4 l[2], const uint4 r[2], uint4 o[2]) {
  uint4 s[4] = {l[0], l[1], r[0], r[1]};
  v4_permute(s);
  o[0] = gf_add(s[0], l[0]);
  o[1] = gf_add(s[1], l[1]);
}

__host__ __device__ __forceinline__ uint64_t layer_offset(uint32_t L, uint32_t k) {
  return (1ull << (L + 1)) - (1ull << (L + 1 - k));
}

// 256 threads: two CTAs (2 x 66 KB of shared memory, 2 x 256 x <= 128 registers) and 16 warps per
// SM; the permutation is a long dependent chain, so resident warps are what hides its latency.
constexpr uint32_t kV4Threads = 256;
constexpr uint32_t kV4LeafFuse = 8;  // 2^8 leaves per CTA
constexpr uint32_t kV4NodeFuse = 9;  // 2^9 inputs per CTA
constexpr size_t kV4Smem = kImageBytes + 2 * kV4Threads * 2 * 16;  // image + [2][threads][2] uint4

__global__ void __launch_bounds__(kV4Threads, 2) vision4_permute_kernel(const uint4* __restrict__ img,
                                                                     uint4* __restrict__ states,
                                                                     uint64_t n) {
  v4_load_image(img);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint4 s[4] = {states[4 * i], states[4 * i + 1], states[4 * i + 2], states[4 * i + 3]};
    v4_permute(s);
#pragma unroll
    for (int k = 0; k < 4; k++) states[4 * i + k] = s[k];
  }
}

// Node buffers after the image: [2][kV4Threads][2] uint4.
__device__ __forceinline__ uint4* v4_nodes_buf() { return v4_img + kImageBytes / 16; }

// Hashes 2^fused leaves per CTA (VisionHasherDigest over each leaf's 2^log_batch elements) and
// compresses `fused` layers above them in shared memory.
__global__ void __launch_bounds__(kV4Threads, 2)
    vision4_leaves_kernel(const uint4* __restrict__ img, const uint4* __restrict__ elems,
                          uint32_t log_batch, uint4* __restrict__ nodes, uint32_t L,
                          uint32_t fused) {
  v4_load_image(img);
  uint4* buf = v4_nodes_buf();
  const uint32_t tid = threadIdx.x;
  const uint64_t leaf = (uint64_t)blockIdx.x * blockDim.x + tid;
  const uint4* e = elems + (leaf << log_batch);
  uint4 s[4] = {gf_zero(), gf_zero(), gf_zero(), gf_zero()};
  if (log_batch == 0) {  // 16 bytes: one block with the padding in its second half
    s[0] = e[0];
    s[1] = make_uint4(0x80u, 0u, 0u, 0x01000000u);
    v4_permute(s);
  } else {
    const uint32_t blocks = 1u << (log_batch - 1);
#pragma unroll 1
    for (uint32_t j = 0; j < blocks; j++) {  // absorb: the block overwrites state[0..2]
      s[0] = e[2 * j];
      s[1] = e[2 * j + 1];
      v4_permute(s);
    }
    s[0] = make_uint4(0x80u, 0u, 0u, 0u);  // the padding block 0x80 0 .. 0 0x01
    s[1] = make_uint4(0u, 0u, 0u, 0x01000000u);
    v4_permute(s);
  }
  nodes[2 * leaf] = s[0];
  nodes[2 * leaf + 1] = s[1];
  buf[2 * tid] = s[0];
  buf[2 * tid + 1] = s[1];
  for (uint32_t lvl = 1; lvl <= fused; lvl++) {
    __syncthreads();
    const uint32_t n = blockDim.x >> lvl;
    const uint32_t src = ((lvl - 1) & 1) * 2 * kV4Threads, dst = (lvl & 1) * 2 * kV4Threads;
    if (tid < n) {
      const uint4 l[2] = {buf[src + 4 * tid], buf[src + 4 * tid + 1]};
      const uint4 r[2] = {buf[src + 4 * tid + 2], buf[src + 4 * tid + 3]};
      uint4 o[2];
      v4_compress(l, r, o);
      buf[dst + 2 * tid] = o[0];
      buf[dst + 2 * tid + 1] = o[1];
      const uint64_t at = layer_offset(L, lvl) + (uint64_t)blockIdx.x * n + tid;
      nodes[2 * at] = o[0];
      nodes[2 * at + 1] = o[1];
    }
  }
}

// Compresses `fused` layers starting at layer in_level; each CTA reduces 2^fused inputs.
__global__ void __launch_bounds__(kV4Threads, 2)
    vision4_nodes_kernel(const uint4* __restrict__ img, uint4* __restrict__ nodes, uint32_t L,
                         uint32_t in_level, uint32_t fused) {
  v4_load_image(img);
  uint4* buf = v4_nodes_buf();
  const uint32_t tid = threadIdx.x;
  const uint64_t in_off = layer_offset(L, in_level);
  for (uint32_t lvl = 1; lvl <= fused; lvl++) {
    const uint32_t n = (blockDim.x * 2) >> lvl;
    const uint32_t src = ((lvl - 1) & 1) * 2 * kV4Threads, dst = (lvl & 1) * 2 * kV4Threads;
    if (lvl > 1) __syncthreads();
    if (tid < n) {
      uint4 l[2], r[2], o[2];
      if (lvl == 1) {
        const uint64_t i = in_off + 2 * ((uint64_t)blockIdx.x * n + tid);
        l[0] = nodes[2 * i];
        l[1] = nodes[2 * i + 1];
        r[0] = nodes[2 * i + 2];
        r[1] = nodes[2 * i + 3];
      } else {
        l[0] = buf[src + 4 * tid];
        l[1] = buf[src + 4 * tid + 1];
        r[0] = buf[src + 4 * tid + 2];
        r[1] = buf[src + 4 * tid + 3];
      }
      v4_compress(l, r, o);
      buf[dst + 2 * tid] = o[0];
      buf[dst + 2 * tid + 1] = o[1];
      const uint64_t at = layer_offset(L, in_level + lvl) + (uint64_t)blockIdx.x * n + tid;
      nodes[2 * at] = o[0];
      nodes[2 * at + 1] = o[1];
    }
  }
}

// ---- small trees: one permutation over four lanes
//
// A tree of few leaves cannot fill the GPU, so its time is the chain of dependent permutations
// (a leaf's sponge, then one per layer) on single threads.  Here four consecutive lanes hold one
// state, element e = lane & 3 each: every lane inverts its own element (four inversions instead
// of Montgomery's one, but nothing of the sbox waits for another element) and applies B or B^-1;
// the MDS combines the four elements by shuffles.  About half the instructions of one thread's
// permutation sit on the chain.

__device__ __forceinline__ uint4 shfl_xor_gf(uint4 v, int m) {
  return make_uint4(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m),
                    __shfl_xor_sync(0xffffffffu, v.z, m), __shfl_xor_sync(0xffffffffu, v.w, m));
}

__device__ __forceinline__ uint4 shfl_gf(uint4 v, int src) {
  return make_uint4(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
                    __shfl_sync(0xffffffffu, v.z, src), __shfl_sync(0xffffffffu, v.w, src));
}

// The permutation of the state held by this lane's group of four; returns element e.  Every lane
// of the warp calls it together.
static __device__ __noinline__ uint4 v4_permute_lane(uint4 x, uint32_t e) {
  const uint32_t next = (threadIdx.x & 31u & ~3u) | ((e + 1) & 3u);
  x = gf_add(x, v4_img[kRcOff + e]);
#pragma unroll 1
  for (uint32_t h = 0; h < 16; h++) {
    const bool inverse = (h & 1) == 0;
    x = gf_add(v4_map(inverse ? kMapLinv : kMapLfwd, v4_inv(x)),
               v4_img[inverse ? kBinv0Off : kC0Off]);
    // MDS: x_e += (x_0 + x_1 + x_2 + x_3) + 2 (x_e + x_{e+1 mod 4}), all from the old values
    const uint4 s1 = gf_add(x, shfl_xor_gf(x, 1));
    const uint4 sum = gf_add(s1, shfl_xor_gf(s1, 2));
    const uint4 nx = shfl_gf(x, (int)next);
    x = gf_add(gf_add(x, sum), mul_x(gf_add(x, nx)));
    x = gf_add(x, v4_img[kRcOff + 4 * (h + 1) + e]);
  }
  return x;
}

// Small CTAs (16 leaves = 2 warps; 16 inputs = 1 warp): the trees are too small to fill the GPU,
// so spreading them over many SMs leaves each chain a scheduler of its own.
constexpr uint32_t kLaneLeafFuse = 4;  // 2^4 leaves (64 lanes) per CTA
constexpr uint32_t kLaneNodeFuse = 4;  // 2^4 inputs per CTA
// Trees of up to 2^12 leaves take the four-lane kernels.  Measured: 2^14 leaves on them took
// 9.7 ms against 8.4 ms on the one-thread kernels (four inversions per sbox cost more than the
// SMs the one-thread kernels leave idle).
constexpr uint32_t kLaneMaxLog = 12;

__global__ void __launch_bounds__(256)
    vision4_leaves_lanes_kernel(const uint4* __restrict__ img, const uint4* __restrict__ elems,
                                uint32_t log_batch, uint4* __restrict__ nodes, uint32_t L,
                                uint32_t fused) {
  v4_load_image(img);
  uint4* buf = v4_nodes_buf();
  const uint32_t e = threadIdx.x & 3, item = threadIdx.x >> 2, n0 = 1u << fused;
  const bool valid = item < n0;  // lanes past the CTA's leaves compute along for the shuffles
  const uint64_t leaf = (uint64_t)blockIdx.x * n0 + (valid ? item : 0);
  const uint4* ep = elems + (leaf << log_batch);
  uint4 x = gf_zero();
  if (log_batch == 0) {
    if (e == 0) x = ep[0];
    if (e == 1) x = make_uint4(0x80u, 0u, 0u, 0x01000000u);
    x = v4_permute_lane(x, e);
  } else {
    const uint32_t blocks = 1u << (log_batch - 1);
#pragma unroll 1
    for (uint32_t j = 0; j < blocks; j++) {
      if (e < 2) x = ep[2 * j + e];
      x = v4_permute_lane(x, e);
    }
    if (e == 0) x = make_uint4(0x80u, 0u, 0u, 0u);
    if (e == 1) x = make_uint4(0u, 0u, 0u, 0x01000000u);
    x = v4_permute_lane(x, e);
  }
  if (valid && e < 2) {
    nodes[2 * leaf + e] = x;
    buf[2 * item + e] = x;
  }
  for (uint32_t lvl = 1; lvl <= fused; lvl++) {
    __syncthreads();
    const uint32_t n = n0 >> lvl;
    const uint32_t src = ((lvl - 1) & 1) * 2 * kV4Threads, dst = (lvl & 1) * 2 * kV4Threads;
    const bool act = item < n;
    const uint4 in = act ? buf[src + 4 * item + e] : gf_zero();
    const uint4 y = v4_permute_lane(in, e);
    if (act && e < 2) {
      const uint4 o = gf_add(y, in);
      buf[dst + 2 * item + e] = o;
      nodes[2 * (layer_offset(L, lvl) + (uint64_t)blockIdx.x * n + item) + e] = o;
    }
  }
}

__global__ void __launch_bounds__(256)
    vision4_nodes_lanes_kernel(const uint4* __restrict__ img, uint4* __restrict__ nodes,
                               uint32_t L, uint32_t in_level, uint32_t fused) {
  v4_load_image(img);
  uint4* buf = v4_nodes_buf();
  const uint32_t e = threadIdx.x & 3, item = threadIdx.x >> 2, n_in = 1u << fused;
  const uint64_t in_off = layer_offset(L, in_level) + (uint64_t)blockIdx.x * n_in;
  for (uint32_t lvl = 1; lvl <= fused; lvl++) {
    const uint32_t n = n_in >> lvl;
    const uint32_t src = ((lvl - 1) & 1) * 2 * kV4Threads, dst = (lvl & 1) * 2 * kV4Threads;
    if (lvl > 1) __syncthreads();
    const bool act = item < n;
    uint4 in = gf_zero();
    if (act) in = lvl == 1 ? nodes[2 * in_off + 4 * item + e] : buf[src + 4 * item + e];
    const uint4 y = v4_permute_lane(in, e);
    if (act && e < 2) {
      const uint4 o = gf_add(y, in);
      buf[dst + 2 * item + e] = o;
      nodes[2 * (layer_offset(L, in_level + lvl) + (uint64_t)blockIdx.x * n + item) + e] = o;
    }
  }
}

int vision4_commit_lanes(const uint4* img, const uint4* elems, uint32_t L, uint32_t log_batch,
                         uint4* nodes, cudaStream_t s) {
  if (int rc = ensure_smem_limit((const void*)vision4_leaves_lanes_kernel, kV4Smem)) return rc;
  if (int rc = ensure_smem_limit((const void*)vision4_nodes_lanes_kernel, kV4Smem)) return rc;
  const uint32_t fused = L < kLaneLeafFuse ? L : kLaneLeafFuse;
  const uint32_t threads = (4u << fused) < 32u ? 32u : (4u << fused);
  vision4_leaves_lanes_kernel<<<1u << (L - fused), threads, kV4Smem, s>>>(img, elems, log_batch,
                                                                        nodes, L, fused);
  BGPU_LAUNCH_CHECK("vision4_leaves_lanes_kernel");
  count_launch();
  for (uint32_t level = fused; level < L;) {
    const uint32_t f = (L - level) < kLaneNodeFuse ? (L - level) : kLaneNodeFuse;
    const uint32_t t = (2u << f) < 32u ? 32u : (2u << f);
    vision4_nodes_lanes_kernel<<<1u << (L - level - f), t, kV4Smem, s>>>(img, nodes, L, level, f);
    BGPU_LAUNCH_CHECK("vision4_nodes_lanes_kernel");
    count_launch();
    level += f;
  }
  return BINIUS_OK;
}

}  // namespace

namespace bgpu {

int vision4_merkle_commit(const void* d_elems, uint32_t log_leaves, uint32_t log_batch,
                          void* d_nodes, cudaStream_t s) {
  BGPU_ARG(d_elems != nullptr && d_nodes != nullptr, "elems / nodes is NULL");
  BGPU_ARG(log_leaves <= 34 && log_batch <= 20, "tree too large");
  const uint4* img = nullptr;
  if (int rc = device_image(&img)) return rc;
  if (int rc = ensure_smem_limit((const void*)vision4_leaves_kernel, kV4Smem)) return rc;
  if (int rc = ensure_smem_limit((const void*)vision4_nodes_kernel, kV4Smem)) return rc;
  const uint32_t L = log_leaves;
  uint4* nodes = static_cast<uint4*>(d_nodes);
  if (L <= kLaneMaxLog)
    return vision4_commit_lanes(img, static_cast<const uint4*>(d_elems), L, log_batch, nodes, s);
  // at least 2^8 CTAs: mid-size trees spread over every SM in smaller CTAs
  const uint32_t fused = L - 8 < kV4LeafFuse ? L - 8 : kV4LeafFuse;
  const uint64_t grid = 1ull << (L - fused);
  BGPU_ARG(grid <= 0x7fffffffull, "too many leaves");
  vision4_leaves_kernel<<<(unsigned)grid, 1u << fused, kV4Smem, s>>>(
      img, static_cast<const uint4*>(d_elems), log_batch, nodes, L, fused);
  BGPU_LAUNCH_CHECK("vision4_leaves_kernel");
  count_launch();
  for (uint32_t level = fused; level < L;) {
    const uint32_t f = (L - level) < kV4NodeFuse ? (L - level) : kV4NodeFuse;
    const uint64_t g = 1ull << (L - level - f);
    vision4_nodes_kernel<<<(unsigned)g, 1u << (f - 1), kV4Smem, s>>>(img, nodes, L, level, f);
    BGPU_LAUNCH_CHECK("vision4_nodes_kernel");
    count_launch();
    level += f;
  }
  return BINIUS_OK;
}

}  // namespace bgpu

extern "C" {

int binius_vision4_permute(void* d_states, uint64_t n, void* stream) {
  BGPU_ARG(d_states != nullptr || n == 0, "states is NULL");
  if (n == 0) return clear_error();
  const uint4* img = nullptr;
  if (int rc = device_image(&img)) return rc;
  if (int rc = ensure_smem_limit((const void*)vision4_permute_kernel, kV4Smem)) return rc;
  const uint64_t blocks = (n + kV4Threads - 1) / kV4Threads;
  const unsigned grid = (unsigned)(blocks < 148 * 16 ? blocks : 148 * 16);
  vision4_permute_kernel<<<grid, kV4Threads, kV4Smem, as_stream(stream)>>>(
      img, static_cast<uint4*>(d_states), n);
  BGPU_LAUNCH_CHECK("vision4_permute_kernel");
  count_launch();
  return clear_error();
}

int binius_merkle_commit_vision4(const void* d_elems, uint32_t log_leaves, uint32_t log_batch,
                                 void* d_nodes, void* stream) {
  if (int rc = bgpu::vision4_merkle_commit(d_elems, log_leaves, log_batch, d_nodes,
                                           as_stream(stream)))
    return rc;
  return clear_error();
}

}  // extern "C"
