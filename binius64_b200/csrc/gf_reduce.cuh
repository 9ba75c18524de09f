// CTA-wide XOR (GF(2^128) addition) reductions with atomicXor accumulation into global memory.
#pragma once
#include "gf128.cuh"

namespace bgpu {

__device__ __forceinline__ void atomic_xor_gf(uint32_t* dst, uint4 v) {
  if (v.x) atomicXor(dst + 0, v.x);
  if (v.y) atomicXor(dst + 1, v.y);
  if (v.z) atomicXor(dst + 2, v.z);
  if (v.w) atomicXor(dst + 3, v.w);
}

// v from lane src of the caller's width-lane segment of the (converged) warp.
__device__ __forceinline__ uint4 shfl_gf(uint4 v, uint32_t src, int width) {
  v.x = __shfl_sync(0xffffffffu, v.x, (int)src, width);
  v.y = __shfl_sync(0xffffffffu, v.y, (int)src, width);
  v.z = __shfl_sync(0xffffffffu, v.z, (int)src, width);
  v.w = __shfl_sync(0xffffffffu, v.w, (int)src, width);
  return v;
}

// The XOR of v over the 32 lanes of the (converged) warp, in every lane: one warp reduction (__reduce_xor_sync) per word.
__device__ __forceinline__ uint4 warp_xor_gf(uint4 v) {
  v.x = __reduce_xor_sync(0xffffffffu, v.x);
  v.y = __reduce_xor_sync(0xffffffffu, v.y);
  v.z = __reduce_xor_sync(0xffffffffu, v.z);
  v.w = __reduce_xor_sync(0xffffffffu, v.w);
  return v;
}

// XOR-reduces `NV` field values across the CTA and adds the totals into dst[0..NV) (4 words
// each).  Every thread of the CTA must call it.
template <int NV>
__device__ __forceinline__ void block_xor_reduce(uint4 (&v)[NV], uint32_t* dst) {
  __shared__ uint4 red[NV][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++) {
    v[q] = warp_xor_gf(v[q]);
    if (lane == 0) red[q][warp] = v[q];
  }
  __syncthreads();
  if (warp == 0) {
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++) {
      const uint4 x = warp_xor_gf(lane < nwarps ? red[q][lane] : gf_zero());
      if (lane == 0) atomic_xor_gf(dst + 4 * q, x);
    }
  }
}

// XOR-reduces NV field values across the CTA; the lanes of warp 0 get the totals in v.  Every
// thread must call it; it ends with the CTA synchronised, so it may be called again in a loop.
template <int NV>
__device__ __forceinline__ void block_xor_sum(uint4 (&v)[NV]) {
  __shared__ uint4 red[NV][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++) {
    v[q] = warp_xor_gf(v[q]);
    if (lane == 0) red[q][warp] = v[q];
  }
  __syncthreads();
  if (warp == 0) {
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++) {
      const uint4 x = warp_xor_gf(lane < nwarps ? red[q][lane] : gf_zero());
      v[q] = x;
    }
  }
  __syncthreads();
}

}  // namespace bgpu
