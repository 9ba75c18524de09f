// Host-side Fiat-Shamir transcript: ProverTranscript<HasherChallenger<Sha256>>.
//
// HasherChallenger (verifier/transcript/src/fiat_shamir/hasher_challenger.rs:14-200) is one
// streaming SHA-256 with two modes.  It starts sampling from SHA-256("") with the hasher holding
// those 32 bytes.  Sampling reads the current 32-byte buffer and, when it is used up, replaces it
// by the digest of the stream, which restarts as that digest.  Switching from sampling to observing
// appends the number of buffer bytes consumed as a little-endian u64; observing appends the bytes;
// switching back to sampling discards the buffer.  ProverTranscript (transcript.rs:204-327) tees
// message() writes into the proof tape and the challenger, decommitment() writes only the tape.
// The protocol is a chain of such dependent steps, so it runs on the host between kernel launches.
#pragma once
#include <stdint.h>
#include <string.h>

#include <vector>

#include "host_sha256.h"

namespace bgpu {

// The challenger's whole state as plain data in the word form the device transcript
// (dev_transcript.cuh) works in: the SHA-256 stream (chaining value, the partial block as
// big-endian words zero past block_len, length), the sampling mode, the sample buffer as
// little-endian words and its read index, plus the device tape's fill level.
struct TranscriptState {
  uint32_t h[8];
  uint32_t w[16];
  uint64_t total;
  uint32_t block_len;
  uint32_t sampling;
  uint32_t index;
  uint32_t tape_len;  // bytes the device appended to its tape
  uint32_t tape_cap;
  uint32_t error;     // set when the device tape overflowed
  uint32_t buf[8];
};

class Transcript {
 public:
  Transcript() {
    uint8_t d0[32];
    HostSha256::oneshot(nullptr, 0, d0);
    hasher_.update(d0, 32);
    memcpy(buffer_, d0, 32);
  }

  // TranscriptWriter for observe(): the challenger switches to observing even for an empty write.
  void observe(const uint8_t* p, size_t n) {
    to_observer();
    hasher_.update(p, n);
  }
  // message(): bytes go to the tape and, if any are written, to the challenger.
  void message(const void* p, size_t n) {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    tape_.insert(tape_.end(), b, b + n);
    if (n) {
      to_observer();
      hasher_.update(b, n);
    }
  }
  void decommitment(const void* p, size_t n) {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    tape_.insert(tape_.end(), b, b + n);
  }
  void sample_bytes(uint8_t* out, size_t n) {
    if (!sampling_) {
      sampling_ = true;
      index_ = 32;
    }
    for (size_t i = 0; i < n; i++) {
      if (index_ == 32) {
        uint8_t d[32];
        hasher_.digest(d);
        hasher_.reset();
        hasher_.update(d, 32);
        memcpy(buffer_, d, 32);
        index_ = 0;
      }
      out[i] = buffer_[index_++];
    }
  }
  // CanSample<B128>: 16 bytes read as a little-endian u128 (transcript.rs:398-407).
  void sample_elem(uint8_t out[16]) { sample_bytes(out, 16); }
  // sample_bits_reader (fiat_shamir/sampling.rs:34-50): a little-endian u32, masked.
  uint32_t sample_bits(uint32_t bits) {
    uint8_t b[4];
    sample_bytes(b, 4);
    uint32_t v = (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) |
                 ((uint32_t)b[3] << 24);
    if (bits >= 32) return v;
    return v & ((1u << bits) - 1);
  }
  const std::vector<uint8_t>& tape() const { return tape_; }

  void save(TranscriptState& st) const {
    memset(&st, 0, sizeof(st));
    uint8_t blk[64];
    hasher_.save(st.h, blk, st.block_len, st.total);
    for (uint32_t i = 0; i < st.block_len; i++)
      st.w[i >> 2] |= (uint32_t)blk[i] << (24 - 8 * (i & 3));
    st.sampling = sampling_ ? 1u : 0u;
    st.index = index_;
    for (int i = 0; i < 32; i++) st.buf[i >> 2] |= (uint32_t)buffer_[i] << (8 * (i & 3));
  }
  // Takes over a state the device advanced and appends the tape bytes it wrote.
  void load(const TranscriptState& st, const uint8_t* tape) {
    uint8_t blk[64];
    for (int i = 0; i < 64; i++) blk[i] = (uint8_t)(st.w[i >> 2] >> (24 - 8 * (i & 3)));
    hasher_.load(st.h, blk, st.block_len, st.total);
    sampling_ = st.sampling != 0;
    index_ = st.index;
    for (int i = 0; i < 32; i++) buffer_[i] = (uint8_t)(st.buf[i >> 2] >> (8 * (i & 3)));
    tape_.insert(tape_.end(), tape, tape + st.tape_len);
  }

 private:
  void to_observer() {
    if (sampling_) {
      uint8_t le[8];
      for (int i = 0; i < 8; i++) le[i] = (uint8_t)((uint64_t)index_ >> (8 * i));
      hasher_.update(le, 8);
      sampling_ = false;
    }
  }

  HostSha256 hasher_;
  bool sampling_ = true;
  uint8_t buffer_[32];
  uint32_t index_ = 0;
  std::vector<uint8_t> tape_;
};

}  // namespace bgpu

struct binius_transcript {
  bgpu::Transcript t;
};
