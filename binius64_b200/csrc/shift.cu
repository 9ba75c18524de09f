// Shift reduction (prover/prover/src/protocols/shift/prove.rs:103-153) on the device.
//
// Phase 1 (phase_1.rs:43-276): the g parts g_v[s*64 + j] = sum over operand terms with shift
// (v, s) of lambda^(operand+1) * eq(r_x')[constraint] * bit_j(word), and the h parts
// (monster.rs:34-104) built from the Lagrange basis of {phi(t) : t < 64} at r_zhat'.  The eight
// (g_v, h_v) pairs live interleaved as one array of 8 * 4096 elements, index (s*64 + j)*8 + v, so
// the eight bivariate provers' top-variable folds are the top-variable fold of that one array and
// their summed round sums are its round sums.
//
// g is accumulated from the key-sorted term table (ShiftTerms): terms arrive grouped by
// key = (v*64 + s)*8 + operand class, a CTA stages 256 of them in shared memory (eq value of the
// constraint and the witness word), and each 64-thread group owns the 64 bit positions j of its
// slice, XOR-adding eq into the position's accumulator when bit j of the word is set.  A group
// sees keys in increasing order and flushes its accumulators with atomicXor when the key changes;
// the lambda powers are applied once per (key, j) afterwards.
//
// Phase 2 (phase_2.rs:56-160): r_j_witness = fold_words(words, eq(r_j)), the monster multilinear
// (monster.rs:138-219) M[w] = sum over terms of word w of lambda^(operand+1) eq(r_x')[c]
// h_op[v] eq(r_s)[s] (one multiply per term into a per-key scalar table, atomicXor into M), then
// the batched sumcheck of the bivariate product (r_j_witness, M) with the in/out MLE-check
// (protocols/inout_check.rs:19-211, sumcheck/mle_to_sumcheck.rs:28-77, sumcheck/batch.rs:41-103).
// Both round loops run on the device transcript (dev_transcript.cuh): each round is an
// evaluation kernel and a finish kernel that forms the round polynomial, writes the message and
// samples the challenge; the host waits once per phase.
#include <string.h>

#include <algorithm>
#include <vector>

#include "cs.h"
#include "dev_transcript.cuh"
#include "pdl.cuh"
#include "gf128.cuh"
#include "gf_reduce.cuh"
#include "internal.h"
#include "kernels.h"
#include "reductions.h"
#include "transcript.h"

using namespace bgpu;

namespace {

constexpr uint32_t kLen = 4096;           // 2^(2 * LOG_WORD_SIZE_BITS)
constexpr uint32_t kFlat = 8 * kLen;      // eight shift variants
constexpr uint32_t kNoKey = 0xffffffffu;
constexpr int kTile = 256;

struct Lag64 {
  uint4 l[64];
};

struct ClassPowers {
  uint4 p[8];  // lambda power of each operand class (class 7 unused)
};

unsigned grid_for(uint64_t n, unsigned threads, unsigned cap = 148 * 8) {
  uint64_t g = (n + threads - 1) / threads;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, cap));
}

__device__ __forceinline__ const uint4* eq_of_class(uint32_t key, const uint4* eq_and,
                                                    const uint4* eq_mul) {
  return (key & 7) < 3 ? eq_and : eq_mul;
}

// 8x8 bit-matrix transpose (byte i of x is row i): byte k of the result holds bit k of every
// input byte, bit i from byte i (Hacker's Delight 7-3).
__device__ __forceinline__ uint64_t transpose8x8(uint64_t x) {
  uint64_t t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
  x ^= t ^ (t << 7);
  t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
  x ^= t ^ (t << 14);
  t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
  x ^= t ^ (t << 28);
  return x;
}

// g_raw[key * 64 + j] += sum over terms with that key of eq[c] * bit_j(word).
//
// A tile of 256 key-sorted terms is staged in shared memory as 32 chunks of 8.  For each chunk the
// CTA first builds (a) its 64 bit-column bytes, byte j holding bit j of the chunk's 8 words (one
// 8x8 bit transpose per thread, stored as one 8-byte word), and (b) two 16-entry tables of XOR
// combinations of the chunk's eq values (terms 0-3 and 4-7; four entries per thread from the two
// high eq values' sum), a method-of-four-Russians split of the 0/1 x GF(2^128) product.
// Then each 64-thread group walks its 8 chunks with thread j owning bit position j: a chunk whose
// 8 terms share one key costs one byte load and two table lookups; a chunk that straddles a key
// boundary falls back to per-term masked XORs.  A group flushes its accumulators with atomicXor
// when the key changes.
constexpr uint32_t kChunk = 8, kChunks = kTile / kChunk;
// Staged eq values and words sit at e + e / 8 (one pad slot per chunk), so that the four chunks a
// warp reads at once fall in different shared-memory banks.
__device__ __forceinline__ uint32_t pad8(uint32_t e) { return e + (e >> 3); }

__global__ void __launch_bounds__(kTile)
    shift_g_kernel(const uint32_t* __restrict__ vi, const uint32_t* __restrict__ cidx,
                   const uint16_t* __restrict__ keys, uint64_t n,
                   const uint64_t* __restrict__ words, const uint4* __restrict__ eq_and,
                   const uint4* __restrict__ eq_mul, uint32_t* __restrict__ g_raw) {
  __shared__ uint4 s_eq[kTile + kChunks];
  __shared__ uint64_t s_w[kTile + kChunks];
  __shared__ uint32_t s_key[kTile];
  __shared__ uint64_t s_col[kChunks][8];  // byte j of chunk c's row: bit j of its 8 words
  // nibble tables as 8-byte halves: a 16-entry table of 8-byte words spans the 32 banks once, so
  // the random lookups of a half-warp never conflict (16-byte entries: ~1.7x the wavefronts)
  __shared__ uint2 s_tlo[kChunks][2][16], s_thi[kChunks][2][16];
  const uint32_t tid = threadIdx.x, j = tid & 63, grp = tid >> 6;
  uint32_t cur = kNoKey;
  uint4 acc = gf_zero();
  auto switch_key = [&](uint32_t k) {
    if (k != cur) {
      if (cur != kNoKey) atomic_xor_gf(g_raw + 4 * ((uint64_t)cur * 64 + j), acc);
      cur = k;
      acc = gf_zero();
    }
  };
  // each CTA takes a contiguous range of tiles: the terms are sorted by key, so a group's key
  // (and its flush of 64 accumulators) changes only at key boundaries
  const uint64_t n_tiles_all = (n + kTile - 1) / kTile;
  const uint64_t per = (n_tiles_all + gridDim.x - 1) / gridDim.x;
  const uint64_t tile0 = (uint64_t)blockIdx.x * per;
  const uint64_t n_tiles = tile0 + per < n_tiles_all ? tile0 + per : n_tiles_all;
  // the gathers of a tile (eq value and word of each term) are issued one tile ahead, so their
  // latency overlaps the previous tile's work
  uint32_t nk = kNoKey;
  uint4 ne = gf_zero();
  uint64_t nw = 0;
  auto fetch = [&](uint64_t tile) {
    const uint64_t t = tile * kTile + tid;
    if (tile < n_tiles && t < n) {
      nk = keys[t];
      ne = __ldg(eq_of_class(nk, eq_and, eq_mul) + cidx[t]);
      nw = __ldg(words + vi[t]);
    } else {
      nk = kNoKey;
      ne = gf_zero();
      nw = 0;
    }
  };
  fetch(tile0);
  for (uint64_t tile = tile0; tile < n_tiles; tile++) {
    __syncthreads();
    s_key[tid] = nk;
    s_eq[pad8(tid)] = ne;
    s_w[pad8(tid)] = nw;
    fetch(tile + 1);
    __syncthreads();
    {  // bit columns: thread (chunk c, byte block b)
      const uint32_t c = tid >> 3, b = tid & 7;
      uint64_t x = 0;
#pragma unroll
      for (uint32_t i = 0; i < 8; i++) x |= ((s_w[c * 9 + i] >> (8 * b)) & 0xffull) << (8 * i);
      s_col[c][b] = transpose8x8(x);
    }
    {  // nibble tables: thread (chunk c, half h, quarter q) builds entries 4q .. 4q + 3
      const uint32_t g = tid >> 2, c = g >> 1, h = g & 1, q = tid & 3;
      const uint4* e = s_eq + c * 9 + 4 * h;
      const uint4 e0 = e[0], e1 = e[1];
      uint4 base = gf_zero();
      if (q & 1) gf_add_into(base, e[2]);
      if (q & 2) gf_add_into(base, e[3]);
      const uint4 v[4] = {base, gf_add(base, e0), gf_add(base, e1), gf_add(gf_add(base, e0), e1)};
#pragma unroll
      for (int i = 0; i < 4; i++) {
        s_tlo[c][h][4 * q + i] = make_uint2(v[i].x, v[i].y);
        s_thi[c][h][4 * q + i] = make_uint2(v[i].z, v[i].w);
      }
    }
    __syncthreads();
#pragma unroll 2
    for (uint32_t cc = 0; cc < kChunks / 4; cc++) {
      const uint32_t c = grp * (kChunks / 4) + cc, e0 = c * 8;
      const uint32_t k0 = s_key[e0], k7 = s_key[e0 + 7];
      if (k0 == k7) {
        switch_key(k0);
        if (k0 != kNoKey) {
          const uint32_t byte = reinterpret_cast<const uint8_t*>(s_col[c])[j];
          const uint2 l0 = s_tlo[c][0][byte & 15], h0 = s_thi[c][0][byte & 15];
          const uint2 l1 = s_tlo[c][1][byte >> 4], h1 = s_thi[c][1][byte >> 4];
          acc.x ^= l0.x ^ l1.x;
          acc.y ^= l0.y ^ l1.y;
          acc.z ^= h0.x ^ h1.x;
          acc.w ^= h0.y ^ h1.y;
        }
      } else {
        for (uint32_t i = 0; i < 8; i++) {
          const uint32_t e = e0 + i;
          switch_key(s_key[e]);
          const uint32_t m = 0u - (uint32_t)((s_w[c * 9 + i] >> j) & 1);
          const uint4 x = s_eq[c * 9 + i];
          acc.x ^= x.x & m;
          acc.y ^= x.y & m;
          acc.z ^= x.z & m;
          acc.w ^= x.w & m;
        }
      }
    }
  }
  if (cur != kNoKey) atomic_xor_gf(g_raw + 4 * ((uint64_t)cur * 64 + j), acc);
}

// g[(s*64 + j)*8 + v] = sum over classes of lambda_class * g_raw[((v*64 + s)*8 + class)*64 + j].
__global__ void shift_g_combine_kernel(const uint4* __restrict__ g_raw, ClassPowers pw,
                                       uint4* __restrict__ g) {
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= kFlat) return;
  const uint32_t v = idx & 7, s = (idx >> 3) >> 6, j = (idx >> 3) & 63;
  const uint32_t id = v * 64 + s;
  u256 acc = {0, 0, 0, 0};
#pragma unroll
  for (uint32_t cls = 0; cls < kShiftClasses; cls++) {
    const uint4 x = g_raw[(id * 8 + cls) * 64 + j];
    if (!gf_is_zero(x)) xor_into(acc, clmul128(x, pw.p[cls]));
  }
  g[idx] = reduce256(acc);
}

// build_h_parts (monster.rs:34-104) from l_tilde, interleaved layout.
__global__ void shift_h_kernel(Lag64 L, uint4* __restrict__ h) {
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= kFlat) return;
  const uint32_t v = idx & 7, s = (idx >> 3) >> 6, j = (idx >> 3) & 63;
  uint4 val = gf_zero();
  if (v < 4) {
    switch (v) {
      case 0:  // sll
        if (j + s < 64) val = L.l[s + j];
        break;
      case 1:  // srl
        if (j >= s) val = L.l[j - s];
        break;
      case 2:  // sra
        if (j >= s) val = L.l[j - s];
        if (j == 63)
          for (uint32_t t = 64 - s; t < 64; t++) gf_add_into(val, L.l[t]);
        break;
      default:  // rotr
        val = j < s ? L.l[64 - s + j] : L.l[j - s];
        break;
    }
  } else {
    const uint32_t s32 = s & 31, base = j & 32, jj = j & 31;
    switch (v) {
      case 4:  // sll32
        if (jj + s32 < 32) val = L.l[base + s32 + jj];
        break;
      case 5:  // srl32
        if (jj >= s32) val = L.l[base + jj - s32];
        break;
      case 6:  // sra32
        if (jj >= s32) val = L.l[base + jj - s32];
        if (jj == 31)
          for (uint32_t t = 32 - s32; t < 32; t++) gf_add_into(val, L.l[base + t]);
        break;
      default:  // rotr32
        val = jj < s32 ? L.l[base + 32 - s32 + jj] : L.l[base + jj - s32];
        break;
    }
  }
  h[idx] = val;
}

// out[v] += <h_v, eq(r_j ++ r_s)> for the 8 variants (evaluate_h_op); out zeroed by the caller.
// Each of kHopsBlocks CTAs takes a 4096 / kHopsBlocks slice of the index; a thread owns one
// variant and every 32nd index of the slice.
constexpr int kHopsBlocks = 64;
__global__ void __launch_bounds__(256)
    shift_h_ops_kernel(const uint4* __restrict__ h, const uint4* __restrict__ eq,
                       uint32_t* __restrict__ out) {
  __shared__ uint4 part[256];
  const uint32_t v = threadIdx.x & 7;
  constexpr uint32_t kSlice = kLen / kHopsBlocks;
  u256 acc = {0, 0, 0, 0};
  for (uint32_t i = blockIdx.x * kSlice + (threadIdx.x >> 3); i < (blockIdx.x + 1) * kSlice; i += 32)
    xor_into(acc, clmul128(h[i * 8 + v], eq[i]));
  part[threadIdx.x] = reduce256(acc);
  __syncthreads();
  if (threadIdx.x < 8) {
    uint4 x = gf_zero();
    for (uint32_t q = 0; q < 32; q++) gf_add_into(x, part[q * 8 + threadIdx.x]);
    atomic_xor_gf(out + 4 * threadIdx.x, x);
  }
}

// T[key] = lambda_class * h_op(kind)[v] * eq(r_s)[s] (the monster scalars, monster.rs:168-190).
__global__ void shift_scalars_kernel(ClassPowers pw, Lag64 eq_rs, const uint4* __restrict__ h_ops,
                                     uint32_t mul_offset, uint4* __restrict__ T) {
  const uint32_t key = blockIdx.x * blockDim.x + threadIdx.x;
  if (key >= kShiftKeys) return;
  const uint32_t cls = key & 7, id = key >> 3, v = id >> 6, s = id & 63;
  if (cls >= kShiftClasses) {
    T[key] = gf_zero();
    return;
  }
  const uint4 hop = h_ops[(cls < 3 ? 0 : mul_offset) + v];
  T[key] = gf_mul(gf_mul(pw.p[cls], hop), eq_rs.l[s]);
}

// M[w] = sum over word w's terms of T[key] * eq[c] (build_monster_multilinear, monster.rs:138-219).
// Each thread takes kMonsterChunk consecutive terms of the word-ordered table, so every thread does
// the same number of multiplies whatever the words' term counts.  Products are accumulated
// unreduced while the word stays the same and reduced once per (thread, word); a word whose terms
// all lie in the thread's chunk is stored, one split across chunks is XORed in atomically (M is
// cleared first, which also covers words with no terms).
__global__ void __launch_bounds__(256)
    shift_monster_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ chunk_word,
                         const uint32_t* __restrict__ cidx, const uint16_t* __restrict__ keys,
                         uint64_t n, const uint4* __restrict__ eq_and,
                         const uint4* __restrict__ eq_mul, const uint4* __restrict__ T,
                         uint4* __restrict__ M) {
  const uint64_t n_chunks = (n + kMonsterChunk - 1) / kMonsterChunk;
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n_chunks;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t t0 = j * kMonsterChunk, t1 = min(t0 + kMonsterChunk, n);
    uint32_t w = chunk_word[j];
    uint64_t lo = off[w], hi = off[w + 1];  // word w's terms
    u256 acc = {0, 0, 0, 0};
    auto flush = [&]() {
      const uint4 v = reduce256(acc);
      if (lo >= t0 && hi <= t1)
        M[w] = v;
      else
        atomic_xor_gf(reinterpret_cast<uint32_t*>(M + w), v);
    };
    for (uint64_t t = t0; t < t1; t++) {
      if (t == hi) {  // word w ends here; the next word with terms starts at t (t < n)
        flush();
        acc = {0, 0, 0, 0};
        do {
          w++;
          lo = hi;
          hi = off[w + 1];
        } while (hi == lo);
      }
      const uint32_t k = keys[t];
      const uint4 e = __ldg(eq_of_class(k, eq_and, eq_mul) + cidx[t]);
      xor_into(acc, clmul128(__ldg(T + k), e));
    }
    flush();
  }
}

// out[0] += <x[off0 ..], eq>, out[1] += <x[off1 ..], eq> over len elements.
__global__ void __launch_bounds__(256)
    dot2_kernel(const uint4* __restrict__ x, uint64_t off0, uint64_t off1,
                const uint4* __restrict__ eq, uint64_t len, uint32_t* __restrict__ out) {
  pdl_wait();
  pdl_trigger();
  u256 a0 = {0, 0, 0, 0}, a1 = {0, 0, 0, 0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 e = eq[i];
    xor_into(a0, clmul128(x[off0 + i], e));
    xor_into(a1, clmul128(x[off1 + i], e));
  }
  uint4 v[2] = {reduce256(a0), reduce256(a1)};
  block_xor_reduce<2>(v, out);
}

// Per-round constants of the phase-2 batch, known before the loop: the in/out check's current
// eq coordinate zc = z[gn - 1] and 1 / (1 + zc) (used when the round is past the public
// segment's extra variables), the coordinate alpha_dec the Gruen eq prefix absorbs (0 while the
// round is early), and whether the round is early (p < n_rem).
struct ShiftRoundConst {
  uint4 zc, inv_one_plus_zc, alpha_dec;
  uint32_t early, pad[3];
};

// The Fiat-Shamir step of one phase-2 round on the device.  ys = (y_1, y_inf) of the bivariate
// product (r_j_witness, M) and (lo, hi) of the in/out check's dot products; st3 = (shift claim,
// in/out claim, Gruen eq prefix).  The batch message is the shift round's (s_0, s_1) plus beta
// times the in/out check's Gruen-scaled (d_0, d_1) (MleToSumCheckDecorator + batch_prove); then r
// is sampled and the three running values advance.  When init_lohi is set (the first round) the
// in/out claim is first set to lo + (hi - lo) z0 from it.  One warp runs the step.
__global__ void __launch_bounds__(32)
    shift_round_finish_kernel(TranscriptState* __restrict__ ts, uint8_t* __restrict__ tape,
                              const uint4* __restrict__ ys, const ShiftRoundConst* __restrict__ rc,
                              const uint4* __restrict__ init_lohi, uint4 z0, uint4 beta,
                              uint4* __restrict__ st3, uint4* __restrict__ r_out) {
  pdl_wait();
  pdl_trigger();
  {
    DevTr st;
    st.load(ts);
    const ShiftRoundConst c = *rc;
    uint4 inout = st3[1];
    if (init_lohi)
      inout = gf_add(init_lohi[0], gf_mul_warp(gf_add(init_lohi[1], init_lohi[0]), z0));
    const uint4 y1 = ys[0], yinf = ys[1], lo = ys[2], hi = ys[3];
    const uint4 s0 = gf_add(st3[0], y1), s2 = yinf, s1 = gf_add(gf_add(y1, s0), s2);
    uint4 iy0, iy1;
    if (c.early) {
      iy1 = gf_add(lo, gf_mul_warp(gf_add(hi, lo), c.zc));
      iy0 = inout;
    } else {
      iy1 = lo;
      iy0 = gf_mul_warp(gf_add(inout, gf_mul_warp(iy1, c.zc)), c.inv_one_plus_zc);
    }
    const uint4 q0 = iy0, q1 = gf_add(iy1, iy0);
    uint4 one_a = c.alpha_dec;
    one_a.x ^= 1u;
    const uint4 eqp = st3[2];
    const uint4 d0 = gf_mul_warp(gf_mul_warp(q0, one_a), eqp);
    const uint4 d1 = gf_mul_warp(gf_add(gf_mul_warp(q1, one_a), q0), eqp);
    const uint4 msg[2] = {gf_add(s0, gf_mul_warp(beta, d0)), gf_add(s1, gf_mul_warp(beta, d1))};
    st.message_elems(tape, msg, 2);
    const uint4 r = st.sample_elem();
    *r_out = r;
    st3[0] = gf_add(s0, gf_mul_warp(r, gf_add(s1, gf_mul_warp(s2, r))));
    st3[1] = gf_add(q0, gf_mul_warp(q1, r));
    uint4 f = gf_add(r, c.alpha_dec);
    f.x ^= 1u;
    st3[2] = gf_mul_warp(eqp, f);
    st.store(ts);
  }
}

// The small last rounds of phase 2 in one CTA (see bivariate_tail_kernel).  Round n_rem folds
// (W, M) from 2^(n_rem+1) to 2^n_rem elements by the previous challenge, evaluates the product
// round, takes the in/out check's two dot products with eq_pub and lets warp 0 run
// shift_round_finish_kernel's Fiat-Shamir step.  eq_pub holds eq(z[0 .. m)) with m = p - 1 while
// rounds are early (p < n_rem), then m = n_rem - 1: summing the two halves of eq(z[0 .. m))
// gives eq(z[0 .. m - 1)), so later rounds shrink it in place.  On entry eq_pub is right for
// the first round.
constexpr int kShiftTailThreads = 512;
__global__ void __launch_bounds__(kShiftTailThreads)
    shift_tail_kernel(TranscriptState* __restrict__ ts, uint8_t* __restrict__ tape,
                      uint4* __restrict__ W, uint4* __restrict__ M, uint4* __restrict__ eq_pub,
                      uint32_t n_rem0, uint32_t p, const uint4* __restrict__ r_first,
                      const ShiftRoundConst* __restrict__ rc, uint4 beta, uint4* __restrict__ run,
                      uint4* __restrict__ chal) {
  pdl_wait();
  pdl_trigger();
  __shared__ uint4 r_sh;
  DevTr st;
  uint4 sum = gf_zero(), inout = gf_zero(), eqp = gf_zero();
  if (threadIdx.x < 32) {
    st.load(ts);
    sum = run[0];
    inout = run[1];
    eqp = run[2];
    r_sh = *r_first;
  }
  __syncthreads();
  for (uint32_t k = 0, n_rem = n_rem0; n_rem > 0; k++, n_rem--) {
    const uint4 r = r_sh;
    const uint64_t h = 1ull << n_rem, half = h >> 1;
    for (uint64_t j = threadIdx.x; j < h; j += blockDim.x) {
      const uint4 w0 = W[j], m0 = M[j];
      W[j] = gf_add(w0, gf_mul_nl(r, gf_add(W[h + j], w0)));
      M[j] = gf_add(m0, gf_mul_nl(r, gf_add(M[h + j], m0)));
    }
    const bool early = p < n_rem;
    if (k > 0 && n_rem < p)
      for (uint64_t i = threadIdx.x; i < half; i += blockDim.x)
        eq_pub[i] = gf_add(eq_pub[i], eq_pub[half + i]);
    __syncthreads();
    uint4 v[4] = {gf_zero(), gf_zero(), gf_zero(), gf_zero()};
    for (uint64_t j = threadIdx.x; j < half; j += blockDim.x) {
      const uint4 w0 = W[j], w1 = W[half + j], m0 = M[j], m1 = M[half + j];
      gf_add_into(v[0], gf_mul_nl(w1, m1));
      gf_add_into(v[1], gf_mul_nl(gf_add(w0, w1), gf_add(m0, m1)));
    }
    const uint64_t E = early ? 1ull << (p - 1) : half;
    for (uint64_t i = threadIdx.x; i < E; i += blockDim.x) {
      const uint4 e = eq_pub[i];
      gf_add_into(v[2], gf_mul_nl(W[half + i], e));
      if (early) gf_add_into(v[3], gf_mul_nl(W[half + E + i], e));
    }
    block_xor_sum<4>(v);
    if (threadIdx.x < 32) {
      const ShiftRoundConst c = rc[k];
      const uint4 y1 = v[0], yinf = v[1], lo = v[2], hi = early ? v[3] : v[2];
      const uint4 s0 = gf_add(sum, y1), s2 = yinf, s1 = gf_add(gf_add(y1, s0), s2);
      uint4 iy0, iy1;
      if (c.early) {
        iy1 = gf_add(lo, gf_mul_warp(gf_add(hi, lo), c.zc));
        iy0 = inout;
      } else {
        iy1 = lo;
        iy0 = gf_mul_warp(gf_add(inout, gf_mul_warp(iy1, c.zc)), c.inv_one_plus_zc);
      }
      const uint4 q0 = iy0, q1 = gf_add(iy1, iy0);
      uint4 one_a = c.alpha_dec;
      one_a.x ^= 1u;
      const uint4 d0 = gf_mul_warp(gf_mul_warp(q0, one_a), eqp);
      const uint4 d1 = gf_mul_warp(gf_add(gf_mul_warp(q1, one_a), q0), eqp);
      const uint4 msg[2] = {gf_add(s0, gf_mul_warp(beta, d0)), gf_add(s1, gf_mul_warp(beta, d1))};
      st.message_elems(tape, msg, 2);
      const uint4 rr = st.sample_elem();
      chal[k] = rr;
      sum = gf_add(s0, gf_mul_warp(rr, gf_add(s1, gf_mul_warp(s2, rr))));
      inout = gf_add(q0, gf_mul_warp(q1, rr));
      uint4 f = gf_add(rr, c.alpha_dec);
      f.x ^= 1u;
      eqp = gf_mul_warp(eqp, f);
      r_sh = rr;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    st.store(ts);
    run[0] = sum;
    run[1] = inout;
    run[2] = eqp;
  }
}

// ------------------------------------------------------------------ host helpers

uint4 u4(hu128 v) {
  uint4 r;
  memcpy(&r, &v, 16);
  return r;
}
hu128 h128(const void* p) {
  hu128 v;
  memcpy(&v, p, 16);
  return v;
}
hu128 sample(Transcript& t) {
  uint8_t b[16];
  t.sample_elem(b);
  return h128(b);
}
void eq_host(const hu128* point, uint32_t n, hu128* out) {
  out[0] = 1;
  for (uint32_t i = 0; i < n; i++) {
    const size_t half = (size_t)1 << i;
    for (size_t k = 0; k < half; k++) {
      const hu128 hi = host_gf_mul(out[k], point[i]);
      out[half + k] = hi;
      out[k] ^= hi;
    }
  }
}
std::vector<uint4> to_u4(const std::vector<hu128>& v) {
  std::vector<uint4> r(v.size());
  for (size_t i = 0; i < v.size(); i++) r[i] = u4(v[i]);
  return r;
}
uint32_t log2_ceil(uint64_t n) {
  uint32_t r = 0;
  while ((1ull << r) < n) r++;
  return r;
}

// Device buffers of one shift reduction (freed on every exit path).
struct ShiftBuffers {
  cudaStream_t s;
  std::vector<void*> ptrs;
  explicit ShiftBuffers(cudaStream_t st) : s(st) {}
  ~ShiftBuffers() {
    for (void* p : ptrs) dev_free(p, s);
  }
  template <class T>
  int alloc(T** p, size_t bytes) {
    cudaError_t e = dev_alloc(reinterpret_cast<void**>(p), bytes ? bytes : 16, s);
    if (e != cudaSuccess) return cuda_error(e, "shift reduction buffers");
    ptrs.push_back(*p);
    return BINIUS_OK;
  }
};

#define SHIFT_TRY(expr)                 \
  do {                                  \
    if (int _rc = (expr)) return _rc;   \
  } while (0)

int launched(const char* what, uint64_t n = 1) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, what);
  count_launch(n);
  return BINIUS_OK;
}


}  // namespace

namespace bgpu {

int shift_reduction_prove(const binius_cs* cs, const uint64_t* d_witness, Transcript& t,
                          const ShiftOperatorData& band, const ShiftOperatorData& bmul,
                          ShiftResult& res, cudaStream_t s) {
  const uint64_t n_words = cs->committed_total_len;
  const uint32_t log_words = log2_ceil(n_words);
  const uint32_t log_public = log2_ceil(cs->offset_witness);
  const uint32_t log_and = log2_ceil(cs->and_ops.n_constraints);
  const uint32_t log_mul = log2_ceil(cs->mul_ops.n_constraints);
  if (band.evals.size() != 3 || bmul.evals.size() != 4)
    return set_error(BINIUS_E_ARG, "operator data: 3 AND and 4 MUL evaluations");
  if (band.r_x.size() != log_and || bmul.r_x.size() != log_mul)
    return set_error(BINIUS_E_ARG, "operator data: r_x' length != log2(constraints)");
  if (log_public < 1 || log_public > log_words)
    return set_error(BINIUS_E_ARG, "public segment must hold 2..committed words");
  const ShiftTerms& terms = cs->shift_terms;

  ShiftBuffers B(s);
  uint4 *eq_and, *eq_mul, *g, *h, *h_keep, *eq_rjs, *h_ops, *T, *W, *M, *eq_pub;
  uint32_t *g_raw, *acc;
  SHIFT_TRY(B.alloc(&eq_and, 16ull << log_and));
  SHIFT_TRY(B.alloc(&eq_mul, 16ull << log_mul));
  SHIFT_TRY(B.alloc(&g_raw, 16ull * kShiftKeys * 64));
  SHIFT_TRY(B.alloc(&g, 16ull * kFlat));
  SHIFT_TRY(B.alloc(&h, 16ull * kFlat));
  SHIFT_TRY(B.alloc(&h_keep, 16ull * kFlat * 2));
  SHIFT_TRY(B.alloc(&eq_rjs, 16ull * kLen));
  SHIFT_TRY(B.alloc(&h_ops, 16ull * 16));
  SHIFT_TRY(B.alloc(&T, 16ull * kShiftKeys));
  SHIFT_TRY(B.alloc(&W, 16ull * n_words));
  SHIFT_TRY(B.alloc(&M, 16ull * n_words));
  SHIFT_TRY(B.alloc(&eq_pub, 16ull << (log_public > 0 ? log_public - 1 : 0)));
  SHIFT_TRY(B.alloc(&acc, 64));

  // lambdas and their powers per operand class
  const hu128 lam_and = sample(t), lam_mul = sample(t);
  ClassPowers pw;
  memset(&pw, 0, sizeof(pw));
  {
    hu128 p = lam_and;
    for (int i = 0; i < 3; i++, p = host_gf_mul(p, lam_and)) pw.p[i] = u4(p);
    p = lam_mul;
    for (int i = 0; i < 4; i++, p = host_gf_mul(p, lam_mul)) pw.p[3 + i] = u4(p);
  }
  SHIFT_TRY(eq_tensor(to_u4(band.r_x).data(), log_and, eq_and, s));
  SHIFT_TRY(eq_tensor(to_u4(bmul.r_x).data(), log_mul, eq_mul, s));

  // ---- phase 1: g and h parts
  BGPU_CUDA(cudaMemsetAsync(g_raw, 0, 16ull * kShiftKeys * 64, s));
  if (terms.n) {
    shift_g_kernel<<<grid_for(terms.n, kTile, 148 * 8), kTile, 0, s>>>(
        terms.vi, terms.c, terms.key, terms.n, d_witness, eq_and, eq_mul, g_raw);
    SHIFT_TRY(launched("shift_g_kernel"));
  }
  shift_g_combine_kernel<<<kFlat / 256, 256, 0, s>>>(reinterpret_cast<const uint4*>(g_raw), pw, g);
  SHIFT_TRY(launched("shift_g_combine_kernel"));
  const bool same_z = band.r_zhat == bmul.r_zhat;
  for (int kind = 0; kind < (same_z ? 1 : 2); kind++) {
    hu128 lt[64];
    lagrange_phi(6, kind == 0 ? band.r_zhat : bmul.r_zhat, lt);
    Lag64 L;
    for (int i = 0; i < 64; i++) L.l[i] = u4(lt[i]);
    shift_h_kernel<<<kFlat / 256, 256, 0, s>>>(L, h_keep + kind * kFlat);
    SHIFT_TRY(launched("shift_h_kernel"));
  }
  BGPU_CUDA(cudaMemcpyAsync(h, h_keep, 16ull * kFlat, cudaMemcpyDeviceToDevice, s));

  // device round state: phase-1 sum slots (12 x 2), phase-2 slots (log_words x 4); dstate = the
  // phase-1 claim, the phase-2 running values (shift claim, in/out claim, eq prefix) and the
  // in/out check's first (lo, hi); challenges (12 + log_words)
  uint4 *slots, *dstate, *chal;
  ShiftRoundConst* rconst;
  const uint64_t n_slots = 2 * 12 + 4 * (uint64_t)log_words;
  SHIFT_TRY(B.alloc(&slots, 16 * n_slots));
  SHIFT_TRY(B.alloc(&dstate, 16 * 6));
  SHIFT_TRY(B.alloc(&chal, 16 * (12 + (uint64_t)log_words)));
  SHIFT_TRY(B.alloc(&rconst, sizeof(ShiftRoundConst) * log_words));
  BGPU_CUDA(cudaMemsetAsync(slots, 0, 16 * n_slots, s));
  uint4* slots2 = slots + 24;

  // the provers' claims: sum_v <g_v, h_v> (phase_1.rs:96-101)
  BGPU_CUDA(cudaMemsetAsync(acc + 8, 0, 32, s));
  dot2_kernel<<<grid_for(kFlat, 256, 148), 256, 0, s>>>(g, 0, 0, h, kFlat, acc + 8);
  SHIFT_TRY(launched("dot2_kernel"));
  DeviceTranscript dt;
  SHIFT_TRY(dt.begin(t, s));
  // rounds whose fold starts from at most tail_max_len() elements run in the single-CTA tail
  int tail0 = 1;
  while (((uint64_t)kFlat >> (tail0 - 1)) > tail_max_len()) tail0++;
  for (int round = 0; round < tail0; round++) {
    const uint64_t size = (uint64_t)kFlat >> round;  // before this round's fold
    uint32_t* ys = reinterpret_cast<uint32_t*>(slots + 2 * round);
    if (round == 0) {
      SHIFT_TRY(bivariate_eval(g, h, size / 2, ys, s));
    } else {
      SHIFT_TRY(bivariate_fold_eval_dev(g, h, size * 2, chal + round - 1, ys, s));
    }
    SHIFT_TRY(bivariate_round_finish(dt, slots + 2 * round,
                                     round == 0 ? reinterpret_cast<const uint4*>(acc + 8) : nullptr,
                                     dstate, nullptr, chal + round, s));
  }
  SHIFT_TRY(bivariate_tail(dt, g, h, (uint64_t)kFlat >> (tail0 - 1), 12 - tail0, chal + tail0 - 1,
                           dstate, chal + tail0, s));
  // one read: transcript, challenges and the remaining 16-element g and h
  std::vector<hu128> ch1(12);
  hu128 gamma = 0;
  {
    uint8_t host[2 * 256];
    StagedReads rd(s);
    SHIFT_TRY(dt.read(rd, 12 * 32));
    SHIFT_TRY(rd.add(ch1.data(), chal, 16 * 12));
    SHIFT_TRY(rd.add(host, g, 256));
    SHIFT_TRY(rd.add(host + 256, h, 256));
    SHIFT_TRY(rd.wait());
    SHIFT_TRY(dt.finish(t));
    // fold the remaining 16-element arrays by the last r; gamma = sum_v g_v(r) h_v(r)
    const hu128 r = ch1[11];
    for (int v = 0; v < 8; v++) {
      const hu128 g0 = h128(host + 16 * v), g1 = h128(host + 16 * (8 + v));
      const hu128 h0 = h128(host + 256 + 16 * v), h1 = h128(host + 256 + 16 * (8 + v));
      gamma ^= host_gf_mul(g0 ^ host_gf_mul(r, g1 ^ g0), h0 ^ host_gf_mul(r, h1 ^ h0));
    }
  }
  std::vector<hu128> rev(ch1.rbegin(), ch1.rend());
  std::vector<hu128> r_j(rev.begin(), rev.begin() + 6), r_s(rev.begin() + 6, rev.end());

  // ---- phase 2: fold the words at r_j, build the monster multilinear
  hu128 eq_rj[64], eq_rs[64];
  eq_host(r_j.data(), 6, eq_rj);
  eq_host(r_s.data(), 6, eq_rs);
  SHIFT_TRY(fold_words64(d_witness, n_words, eq_rj, W, s));
  SHIFT_TRY(eq_tensor(to_u4(rev).data(), 12, eq_rjs, s));
  BGPU_CUDA(cudaMemsetAsync(h_ops, 0, 16 * 16, s));
  for (int kind = 0; kind < (same_z ? 1 : 2); kind++) {
    shift_h_ops_kernel<<<kHopsBlocks, 256, 0, s>>>(h_keep + kind * kFlat, eq_rjs,
                                                   reinterpret_cast<uint32_t*>(h_ops + 8 * kind));
    SHIFT_TRY(launched("shift_h_ops_kernel"));
  }
  Lag64 ers;
  for (int i = 0; i < 64; i++) ers.l[i] = u4(eq_rs[i]);
  shift_scalars_kernel<<<kShiftKeys / 256, 256, 0, s>>>(pw, ers, h_ops, same_z ? 0 : 8, T);
  SHIFT_TRY(launched("shift_scalars_kernel"));
  if (terms.n_words != n_words) return set_error(BINIUS_E_ARG, "shift term table of another size");
  BGPU_CUDA(cudaMemsetAsync(M, 0, 16ull * n_words, s));
  if (terms.n) {
    const uint64_t n_chunks = (terms.n + kMonsterChunk - 1) / kMonsterChunk;
    shift_monster_kernel<<<grid_for(n_chunks, 256, 148 * 32), 256, 0, s>>>(
        terms.w_off, terms.w_chunk, terms.w_c, terms.w_key, terms.n, eq_and, eq_mul, T, M);
    SHIFT_TRY(launched("shift_monster_kernel"));
  }

  // in/out check point (InOutCheckProver::new) and the batching coefficient; the public
  // evaluation is taken on the device by the first round's finish kernel
  const uint32_t p = log_public;
  std::vector<hu128> z(p);
  for (auto& v : z) v = sample(t);
  const hu128 beta = sample(t);
  // in the round loop dot2 follows a kernel and is launched programmatically (PDL relaxes only
  // kernel-to-kernel order); the first one follows a memset and is launched plainly
  auto dot2 = [&](uint64_t off0, uint64_t off1, uint64_t len, uint4* out, bool pdl = true) -> int {
    const unsigned grid = grid_for(len, 256, 148 * 2);
    if (pdl)
      BGPU_CUDA(launch_pdl(dot2_kernel, grid, 256, 0, s, (const uint4*)W, off0, off1,
                           (const uint4*)eq_pub, len, reinterpret_cast<uint32_t*>(out)));
    else
      dot2_kernel<<<grid, 256, 0, s>>>(W, off0, off1, eq_pub, len, reinterpret_cast<uint32_t*>(out));
    SHIFT_TRY(launched("dot2_kernel"));
    return BINIUS_OK;
  };
  uint32_t gn = p;  // Gruen32::n_vars_remaining
  SHIFT_TRY(eq_tensor(to_u4(z).data(), gn - 1, eq_pub, s));
  uint4* run = dstate + 1;
  uint4* init_lohi = dstate + 4;
  BGPU_CUDA(cudaMemsetAsync(init_lohi, 0, 32, s));
  SHIFT_TRY(dot2(0, 1ull << (gn - 1), 1ull << (gn - 1), init_lohi, false));
  const uint4 z0 = u4(z[gn - 1]);
  std::vector<ShiftRoundConst> consts(log_words);
  {
    uint32_t g2 = p;
    for (uint32_t n_rem = log_words; n_rem > 0; n_rem--) {
      ShiftRoundConst& c = consts[log_words - n_rem];
      memset(&c, 0, sizeof(c));
      const hu128 zc = z[g2 - 1];
      c.zc = u4(zc);
      c.early = p < n_rem;
      if (!c.early) c.inv_one_plus_zc = u4(host_gf_inv(1 ^ zc));
      c.alpha_dec = u4(n_rem <= p ? z[n_rem - 1] : 0);
      if (n_rem <= p) g2--;
    }
  }
  BGPU_CUDA(cudaMemcpyAsync(rconst, consts.data(), sizeof(ShiftRoundConst) * log_words,
                            cudaMemcpyHostToDevice, s));
  {
    // the in/out claim is set by the first round from init_lohi
    const uint4 init3[3] = {u4(gamma), u4(0), u4(1)};
    BGPU_CUDA(cudaMemcpyAsync(run, init3, sizeof(init3), cudaMemcpyHostToDevice, s));
  }
  SHIFT_TRY(dt.begin(t, s));
  // rounds whose fold starts from at most tail_max_len() elements run in the single-CTA tail
  uint32_t tail_n = 0;  // n_rem of the first tail round (0: no tail)
  for (uint32_t n_rem = log_words - 1; n_rem > 0; n_rem--)
    if ((2ull << n_rem) <= tail_max_len()) {
      tail_n = n_rem;
      break;
    }
  for (uint32_t n_rem = log_words; n_rem > tail_n; n_rem--) {
    const uint32_t k = log_words - n_rem;
    const uint64_t half = 1ull << (n_rem - 1);
    uint4* ys = slots2 + 4 * k;
    if (n_rem == log_words) {
      SHIFT_TRY(bivariate_eval(W, M, half, reinterpret_cast<uint32_t*>(ys), s));
    } else {
      SHIFT_TRY(bivariate_fold_eval_dev(W, M, half * 4, chal + 12 + k - 1,
                                        reinterpret_cast<uint32_t*>(ys), s));
    }
    if (p < n_rem) {
      SHIFT_TRY(dot2(half, half + (1ull << (gn - 1)), 1ull << (gn - 1), ys + 2));
    } else {
      SHIFT_TRY(eq_tensor(to_u4(z).data(), n_rem - 1, eq_pub, s));
      SHIFT_TRY(dot2(half, half, half, ys + 2));
    }
    if (n_rem <= p) gn--;
    BGPU_CUDA(launch_pdl(shift_round_finish_kernel, 1, 32, 0, s, dt.state(), dt.tape(),
                         (const uint4*)ys, (const ShiftRoundConst*)(rconst + k),
                         n_rem == log_words ? (const uint4*)init_lohi : (const uint4*)nullptr, z0,
                         u4(beta), run, chal + 12 + k));
    SHIFT_TRY(launched("shift_round_finish_kernel"));
  }
  if (tail_n) {
    const uint32_t k0 = log_words - tail_n;
    if (tail_n <= p) SHIFT_TRY(eq_tensor(to_u4(z).data(), tail_n - 1, eq_pub, s));
    BGPU_CUDA(launch_pdl(shift_tail_kernel, 1, kShiftTailThreads, 0, s, dt.state(), dt.tape(), W,
                         M, eq_pub, tail_n, p, (const uint4*)(chal + 12 + k0 - 1),
                         (const ShiftRoundConst*)(rconst + k0), u4(beta), run, chal + 12 + k0));
    SHIFT_TRY(launched("shift_tail_kernel"));
  }
  {
    std::vector<hu128> ch2(log_words);
    uint8_t w01[32];
    StagedReads rd(s);
    SHIFT_TRY(dt.read(rd, 32 * log_words));
    SHIFT_TRY(rd.add(ch2.data(), chal + 12, 16ull * log_words));
    SHIFT_TRY(rd.add(w01, W, 32));
    SHIFT_TRY(rd.wait());
    SHIFT_TRY(dt.finish(t));
    const hu128 r = ch2[log_words - 1], w0 = h128(w01), w1 = h128(w01 + 16);
    res.witness_eval = w0 ^ host_gf_mul(r, w1 ^ w0);
    res.point = r_j;
    res.point.insert(res.point.end(), ch2.rbegin(), ch2.rend());
  }
  t.message(&res.witness_eval, 16);
  return BINIUS_OK;
}

}  // namespace bgpu

extern "C" {

int binius_shift_reduction_prove(const binius_cs* cs, const void* d_witness,
                                 binius_transcript* transcript, const void* h_and_data,
                                 const void* h_mul_data, void* h_out_point, void* h_out_eval,
                                 void* stream) {
  BGPU_ARG(cs && d_witness && transcript && h_and_data && h_mul_data, "NULL argument");
  const uint32_t log_and = log2_ceil(cs->and_ops.n_constraints);
  const uint32_t log_mul = log2_ceil(cs->mul_ops.n_constraints);
  auto parse = [](const uint8_t* b, uint32_t n_evals, uint32_t log_n, ShiftOperatorData& d) {
    for (uint32_t i = 0; i < n_evals; i++) d.evals.push_back(h128(b + 16 * i));
    d.r_zhat = h128(b + 16 * n_evals);
    for (uint32_t i = 0; i < log_n; i++) d.r_x.push_back(h128(b + 16 * (n_evals + 1 + i)));
  };
  ShiftOperatorData band, bmul;
  parse(static_cast<const uint8_t*>(h_and_data), 3, log_and, band);
  parse(static_cast<const uint8_t*>(h_mul_data), 4, log_mul, bmul);
  ShiftResult res;
  int rc = shift_reduction_prove(cs, static_cast<const uint64_t*>(d_witness), transcript->t, band,
                                 bmul, res, as_stream(stream));
  if (rc) return rc;
  if (h_out_point) memcpy(h_out_point, res.point.data(), 16 * res.point.size());
  if (h_out_eval) memcpy(h_out_eval, &res.witness_eval, 16);
  return clear_error();
}

}  // extern "C"
