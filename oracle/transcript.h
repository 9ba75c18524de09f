// CPU oracle (test infrastructure only): Fiat-Shamir transcript shared by the protocol oracles.
//
// HasherChallenger<Sha256> (verifier/transcript/src/fiat_shamir/hasher_challenger.rs:14-200) and
// ProverTranscript / VerifierTranscript (verifier/transcript/src/transcript.rs:36-407).
#ifndef BINIUS_ORACLE_TRANSCRIPT_H
#define BINIUS_ORACLE_TRANSCRIPT_H

#include <string.h>

#include <vector>

#include "oracle_internal.h"

namespace orc {

struct Transcript {
  Sha256Ctx ctx;
  bool sampling = true;
  uint8_t buffer[32];
  uint32_t index = 0;
  std::vector<uint8_t> tape;
  size_t pos = 0;
  bool overrun = false;

  // HasherChallenger::default: the sampler starts on SHA-256("") with the hasher holding it.
  Transcript() {
    uint8_t d0[32];
    sha256(nullptr, 0, d0);
    ctx.update(d0, 32);
    memcpy(buffer, d0, 32);
  }

  void to_observer() {
    if (sampling) {
      uint8_t le[8];
      for (int i = 0; i < 8; i++) le[i] = (uint8_t)((uint64_t)index >> (8 * i));
      ctx.update(le, 8);
      sampling = false;
    }
  }
  void observe(const uint8_t* p, size_t n) {
    if (n == 0) return;  // an empty write never reaches the observer
    to_observer();
    ctx.update(p, n);
  }
  void sample_bytes(uint8_t* out, size_t n) {
    if (!sampling) {
      sampling = true;
      index = 32;
    }
    for (size_t i = 0; i < n; i++) {
      if (index == 32) {
        uint8_t d[32];
        ctx.finalize(d);
        ctx.reset();
        ctx.update(d, 32);
        memcpy(buffer, d, 32);
        index = 0;
      }
      out[i] = buffer[index++];
    }
  }
  u128 sample() {
    uint8_t b[16];
    sample_bytes(b, 16);
    u128 v = 0;
    for (int i = 15; i >= 0; i--) v = (v << 8) | b[i];
    return v;
  }
  uint32_t sample_bits(uint32_t bits) {
    uint8_t b[4];
    sample_bytes(b, 4);
    uint32_t v = (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) |
                 ((uint32_t)b[3] << 24);
    if (bits > 32) bits = 32;
    uint32_t mask = bits == 32 ? 0xffffffffu : ((1u << bits) - 1);
    return v & mask;
  }
  // prover
  void message(const uint8_t* p, size_t n) {
    tape.insert(tape.end(), p, p + n);
    observe(p, n);
  }
  void message_elems(const u128* e, size_t n) { message((const uint8_t*)e, 16 * n); }
  void decommit(const uint8_t* p, size_t n) { tape.insert(tape.end(), p, p + n); }
  void decommit_elems(const u128* e, size_t n) { decommit((const uint8_t*)e, 16 * n); }
  // verifier
  bool read_decommit(uint8_t* p, size_t n) {
    if (pos + n > tape.size()) {
      overrun = true;
      memset(p, 0, n);
      return false;
    }
    memcpy(p, tape.data() + pos, n);
    pos += n;
    return true;
  }
  bool read_message(uint8_t* p, size_t n) {
    bool ok = read_decommit(p, n);
    observe(p, n);
    return ok;
  }
};

}  // namespace orc

#endif
