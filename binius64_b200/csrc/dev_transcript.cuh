// The Fiat-Shamir transcript on the device, for stretches of the protocol that run without the
// host: the sumcheck round loops, whose every round is a kernel's sums -> round polynomial ->
// proof message -> challenge -> the next kernel's fold.  Run on the host, each round costs a
// device-to-host round trip; run here, a loop is a chain of launches the host enqueues at once.
//
// The state is the host Transcript's own (TranscriptState): the same HasherChallenger rules
// (verifier/transcript/src/fiat_shamir/hasher_challenger.rs:14-200) over the same SHA-256 stream,
// so a stretch may start and end anywhere in the protocol and the proof bytes do not change.  A
// device stretch is advanced by one warp whose lanes hold the same state (the steps are a strict
// chain; the lanes share the multiplies, see gf_mul_warp); message bytes go to a device tape that
// the host appends to the proof when the stretch ends.
#pragma once
#include <stdint.h>

#include <vector>

#include "gf128.cuh"
#include "internal.h"
#include "sha256.cuh"
#include "transcript.h"

namespace bgpu {

// The scalar protocol steps run on one warp, where every dependent instruction waits out its full
// latency.  Measured on a B200, one warp: the multiply below 0.38 us (the 16 partial products
// combined by shuffle butterflies instead: 0.45 us; nine clmul32 on one thread: 0.63 us); a
// SHA-256 compression fully unrolled on registers 1.5 us, a compact loop (four- or sixteen-round
// body, round constants loaded) 2.2 us.  A Fiat-Shamir step of its own launch (two compressions,
// two multiplies) costs 7.3 us with the unrolled compression against 8.5 us with the loop, so the
// transcript uses the unrolled one everywhere; the tail loops, whose warp 0 alternates between a
// step and the round's folds, also keep their folds on the out-of-line multiply (gf_mul_nl) so
// that the loop's code stays within the instruction cache (measured: the three tails with inlined
// folds and the unrolled compression took 120 us longer per 2^20 proof than with the compact loop;
// with out-of-line folds the unrolled compression is ~30 us faster than the loop).
__device__ __forceinline__ uint4 gf_mul_1t(uint4 a, uint4 b) { return gf_mul_nl(a, b); }

// A product on the critical path of a Fiat-Shamir step, computed by a whole warp: every lane
// passes the same a and b; lane l < 16 forms the 32x32 carry-less product of word l/4 of a and
// word l%4 of b, each of the eight words of the 256-bit product is the XOR of the partial-product
// halves that land on it (one warp reduction, __reduce_xor_sync, per word), and every lane returns the
// reduced product.  One out-of-line copy keeps the code of the launches that call it small.
static __device__ __noinline__ uint4 gf_mul_warp(uint4 a, uint4 b) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t i = (lane >> 2) & 3, j = lane & 3;
  const uint32_t ai = i == 0 ? a.x : i == 1 ? a.y : i == 2 ? a.z : a.w;
  const uint32_t bj = j == 0 ? b.x : j == 1 ? b.y : j == 2 ? b.z : b.w;
  const uint64_t p = lane < 16 ? clmul32(ai, bj) : 0ull;
  const uint32_t lo = (uint32_t)p, hi = (uint32_t)(p >> 32), k = i + j;
  uint32_t w[8];
#pragma unroll
  for (uint32_t q = 0; q < 8; q++)
    w[q] = __reduce_xor_sync(0xffffffffu, (k == q ? lo : 0u) ^ (k + 1 == q ? hi : 0u));
  u256 r;
  r.p0 = ((uint64_t)w[1] << 32) | w[0];
  r.p1 = ((uint64_t)w[3] << 32) | w[2];
  r.p2 = ((uint64_t)w[5] << 32) | w[4];
  r.p3 = ((uint64_t)w[7] << 32) | w[6];
  return reduce256(r);
}

// One compression of blk into st, both held in local memory by the caller: copied to registers,
// compressed by the fully unrolled sha256_compress (round constants as immediates) and written
// back.  One out-of-line copy serves every call site.
static __device__ __noinline__ void sha256_compress_1t(uint32_t* st, const uint32_t* blk) {
  uint32_t s[8], w[16];
#pragma unroll
  for (int i = 0; i < 8; i++) s[i] = st[i];
#pragma unroll
  for (int i = 0; i < 16; i++) w[i] = blk[i];
  sha256_compress(s, w);
#pragma unroll
  for (int i = 0; i < 8; i++) st[i] = s[i];
}

// The challenger held by the warp that advances it.  The partial SHA-256 block is kept as 16
// big-endian words, the sample buffer as 8 little-endian words; absorbing a word is one store at
// a run-time index (the arrays live in local memory, which the out-of-line compression copies to
// registers), so the code around the compression stays small.  The stream is
// absorbed in 4-byte pieces (every message of the protocol is a whole number of words); a piece
// may start at any byte offset.  Words at or past `len` hold no meaning except that a partially
// filled word is zero past its bytes.
struct DevTr {
  uint32_t h[8], w[16], len;  // chaining value, partial block, bytes in it
  uint64_t total;             // bytes absorbed since the last reset
  uint32_t sampling, index;   // mode and bytes of buf consumed
  uint32_t buf[8];            // sample buffer, little-endian words
  uint32_t tape_len, tape_cap, error;

  static __device__ __forceinline__ void compress(uint32_t* st, const uint32_t* blk) {
    sha256_compress_1t(st, blk);
  }

  __device__ __forceinline__ void load(const TranscriptState* g) {
    for (int i = 0; i < 8; i++) h[i] = g->h[i];
    for (int i = 0; i < 16; i++) w[i] = g->w[i];
    len = g->block_len & 63u;
    total = g->total;
    sampling = g->sampling;
    index = g->index;
    for (int i = 0; i < 8; i++) buf[i] = g->buf[i];
    tape_len = g->tape_len;
    tape_cap = g->tape_cap;
    error = g->error;
  }

  __device__ __forceinline__ void store(TranscriptState* g) const {
    for (int i = 0; i < 8; i++) g->h[i] = h[i];
    for (int i = 0; i < 16; i++) g->w[i] = w[i];
    g->block_len = len;
    g->total = total;
    g->sampling = sampling;
    g->index = index;
    for (int i = 0; i < 8; i++) g->buf[i] = buf[i];
    g->tape_len = tape_len;
    g->tape_cap = tape_cap;
    g->error = error;
  }

  // Absorbs 4 stream bytes given as a little-endian word (first byte lowest).
  __device__ __noinline__ void absorb_word(uint32_t le) {
    const uint32_t be = bswap32(le);
    const uint32_t off = len & 3u;
    total += 4;
    if (off == 0) {
      w[len >> 2] = be;
      len += 4;
      if (len == 64) {
        compress(h, w);
        len = 0;
      }
    } else {
      w[len >> 2] |= be >> (8 * off);
      len += 4 - off;
      if (len == 64) {
        compress(h, w);
        len = 0;
      }
      w[len >> 2] = be << (8 * (4 - off));
      len += off;
    }
  }

  // Digest of the stream (FIPS 180-4 padding) as 8 big-endian words; the stream is unchanged.
  __device__ __noinline__ void digest(uint32_t d[8]) const {
    uint32_t st[8], m[16];
    for (int i = 0; i < 8; i++) st[i] = h[i];
    const uint32_t full = len >> 2, part = len & 3u;
    for (uint32_t i = 0; i < 16; i++) m[i] = (i < full || (i == full && part)) ? w[i] : 0u;
    m[full] |= 0x80u << (24 - 8 * part);
    const uint64_t bits = total * 8;
    if (len + 9 > 64) {
      compress(st, m);
      for (int i = 0; i < 16; i++) m[i] = 0;
    }
    m[14] = (uint32_t)(bits >> 32);
    m[15] = (uint32_t)bits;
    compress(st, m);
    for (int i = 0; i < 8; i++) d[i] = st[i];
  }

  __device__ __forceinline__ void to_observer() {
    if (sampling) {
      const uint32_t idx = index;
      absorb_word(idx);
      absorb_word(0u);
      sampling = 0;
    }
  }

  // Appends n whole words (little-endian) to the tape; sets error instead when they do not fit.
  __device__ __forceinline__ void tape_words(uint8_t* tape, const uint32_t* v, uint32_t n) {
    if (tape_len + 4 * n > tape_cap) {
      error = 1;
      return;
    }
    if (threadIdx.x & 31) {  // a warp advancing the transcript together writes from lane 0
    } else if ((tape_len & 3u) == 0) {
      uint32_t* t32 = reinterpret_cast<uint32_t*>(tape + tape_len);
      for (uint32_t i = 0; i < n; i++) t32[i] = v[i];
    } else {
      for (uint32_t i = 0; i < 4 * n; i++)
        tape[tape_len + i] = (uint8_t)(v[i >> 2] >> (8 * (i & 3)));
    }
    tape_len += 4 * n;
  }

  // message(): n words to the tape and the challenger.
  __device__ __forceinline__ void message_words(uint8_t* tape, const uint32_t* v, uint32_t n) {
    tape_words(tape, v, n);
    if (n) {
      to_observer();
      if ((len & 3u) == 0) {  // word-aligned stream (every message of the protocol): inline
        for (uint32_t i = 0; i < n; i++) {
          w[len >> 2] = bswap32(v[i]);
          len += 4;
          if (len == 64) {
            compress(h, w);
            len = 0;
          }
        }
        total += 4ull * n;
      } else {
        for (uint32_t i = 0; i < n; i++) absorb_word(v[i]);
      }
    }
  }
  __device__ __forceinline__ void message_elems(uint8_t* tape, const uint4* e, uint32_t n) {
    message_words(tape, reinterpret_cast<const uint32_t*>(e), 4 * n);
  }
  __device__ __forceinline__ void observe_words(const uint32_t* v, uint32_t n) {
    to_observer();
    for (uint32_t i = 0; i < n; i++) absorb_word(v[i]);
  }

  // Refills the sample buffer from the digest of the stream, which restarts as that digest.
  __device__ __noinline__ void refill() {
    uint32_t d[8];
    digest(d);
    const uint32_t iv[8] = {0x6a09e667u, 0xbb67ae85u, 0x3c6ef372u, 0xa54ff53au,
                            0x510e527fu, 0x9b05688cu, 0x1f83d9abu, 0x5be0cd19u};
    for (int i = 0; i < 8; i++) {
      h[i] = iv[i];
      w[i] = d[i];
      buf[i] = bswap32(d[i]);
    }
    len = 32;
    total = 32;
    index = 0;
  }

  __device__ __forceinline__ void begin_sampling() {
    if (!sampling) {
      sampling = 1;
      index = 32;
    }
  }

  // n bytes as little-endian words out[(n + 3) / 4].
  __device__ __forceinline__ void sample_words(uint32_t* out, uint32_t n) {
    begin_sampling();
    for (uint32_t i = 0; i < (n + 3) / 4; i++) out[i] = 0;
    for (uint32_t i = 0; i < n; i++) {
      if (index == 32) refill();
      out[i >> 2] |= ((buf[index >> 2] >> (8 * (index & 3u))) & 255u) << (8 * (i & 3u));
      index++;
    }
  }

  // A field element: 16 bytes read as a little-endian u128 (transcript.rs:398-407).
  __device__ __forceinline__ uint4 sample_elem() {
    begin_sampling();
    if (index == 32) refill();
    if ((index & 3u) == 0 && index + 16 <= 32) {
      const uint32_t k = index >> 2;
      index += 16;
      return make_uint4(buf[k], buf[k + 1], buf[k + 2], buf[k + 3]);
    }
    uint32_t o[4];
    sample_words(o, 16);
    return make_uint4(o[0], o[1], o[2], o[3]);
  }

  // sample_bits_reader (fiat_shamir/sampling.rs:34-50): a little-endian u32, masked.
  __device__ __forceinline__ uint32_t sample_bits(uint32_t bits) {
    uint32_t v;
    sample_words(&v, 4);
    return bits >= 32 ? v : v & ((1u << bits) - 1);
  }
};


// Host side of one device stretch.  begin() hands the host transcript's state to the device;
// kernels advance state() and write to tape(); read() queues the copy-back of the state and of
// the `tape_bytes` the stretch is known to write, and finish() (after the reads were waited on)
// hands the state back to the host transcript with those bytes appended.
class DeviceTranscript {
 public:
  static constexpr uint32_t kTapeCap = 1u << 16;

  ~DeviceTranscript();
  int begin(const Transcript& t, cudaStream_t s);
  TranscriptState* state() const { return reinterpret_cast<TranscriptState*>(mem_); }
  uint8_t* tape() const { return mem_ + kStateBytes; }
  // message() of n_bytes (a multiple of 4, 4-byte aligned) that are in device memory.
  int message_device(const void* d_bytes, uint32_t n_bytes, cudaStream_t s);
  int read(StagedReads& rd, uint32_t tape_bytes);
  int finish(Transcript& t);

 private:
  static constexpr size_t kStateBytes = 256;
  cudaStream_t s_ = nullptr;
  uint8_t* mem_ = nullptr;
  uint32_t expect_ = 0;
  TranscriptState host_state_;
  std::vector<uint8_t> host_tape_;
};

}  // namespace bgpu
