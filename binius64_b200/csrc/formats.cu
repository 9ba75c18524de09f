// Wire formats around the prove call, for load-prove serving: the witness halves as ValuesData
// (verifier/core/src/constraint_system.rs:889-990, version 1), the proof as Proof (:993-1100,
// version 1) and ValueVec::new_from_data (:803-823), which joins the public and non-public halves.
// The encodings are the reference's SerializeBytes rules (verifier/utils/src/serialization.rs):
// integers little-endian, usize as u32, a Vec or slice as its u32 length then its items, a String
// as its u32 byte length then the UTF-8 bytes, a Word as its u64.
#include <string.h>

#include <string>
#include <vector>

#include "cs.h"
#include "internal.h"

using namespace bgpu;

namespace {

constexpr uint32_t kValuesDataVersion = 1;
constexpr uint32_t kProofVersion = 1;

void put_u32(std::vector<uint8_t>& out, uint32_t v) {
  for (int i = 0; i < 4; i++) out.push_back((uint8_t)(v >> (8 * i)));
}

struct Cursor {
  const uint8_t* p;
  size_t len, pos = 0;
  bool take(size_t n, const uint8_t** at) {
    if (len - pos < n) return false;
    *at = p + pos;
    pos += n;
    return true;
  }
  bool u32(uint32_t* v) {
    const uint8_t* b;
    if (!take(4, &b)) return false;
    memcpy(v, b, 4);
    return true;
  }
};

int copy_out(const std::vector<uint8_t>& bytes, void* h_out, size_t cap, size_t* len) {
  *len = bytes.size();
  BGPU_ARG(cap >= bytes.size() && (h_out != nullptr || bytes.empty()), "output buffer too small");
  if (!bytes.empty()) memcpy(h_out, bytes.data(), bytes.size());
  return clear_error();
}

}  // namespace

extern "C" {

int binius_values_data_encode(const uint64_t* h_words, size_t n_words, void* h_out, size_t cap,
                              size_t* len) {
  BGPU_ARG(len != nullptr && (h_words != nullptr || n_words == 0), "NULL argument");
  BGPU_ARG(n_words <= 0xffffffffull, "UsizeTooLarge: more than 2^32 - 1 words");
  std::vector<uint8_t> out;
  out.reserve(8 + 8 * n_words);
  put_u32(out, kValuesDataVersion);
  put_u32(out, (uint32_t)n_words);
  const size_t at = out.size();
  out.resize(at + 8 * n_words);
  if (n_words) memcpy(out.data() + at, h_words, 8 * n_words);
  return copy_out(out, h_out, cap, len);
}

int binius_values_data_decode(const void* h_bytes, size_t len, uint64_t* h_words, size_t cap,
                              size_t* n_words) {
  BGPU_ARG(n_words != nullptr && (h_bytes != nullptr || len == 0), "NULL argument");
  Cursor c{static_cast<const uint8_t*>(h_bytes), len};
  uint32_t version = 0, n = 0;
  BGPU_ARG(c.u32(&version), "NotEnoughBytes: ValuesData version");
  BGPU_ARG(version == kValuesDataVersion, "InvalidConstruction: Witness::version");
  BGPU_ARG(c.u32(&n), "NotEnoughBytes: ValuesData length");
  const uint8_t* data = nullptr;
  BGPU_ARG(c.take(8ull * n, &data), "NotEnoughBytes: ValuesData words");
  *n_words = n;
  BGPU_ARG(cap >= n && (h_words != nullptr || n == 0), "output buffer too small");
  if (n) memcpy(h_words, data, 8ull * n);
  return clear_error();
}

int binius_proof_encode(const void* h_transcript, size_t n_bytes, const char* challenger,
                        void* h_out, size_t cap, size_t* len) {
  BGPU_ARG(len != nullptr && challenger != nullptr && (h_transcript != nullptr || n_bytes == 0),
           "NULL argument");
  const size_t n_ch = strlen(challenger);
  BGPU_ARG(n_bytes <= 0xffffffffull && n_ch <= 0xffffffffull, "UsizeTooLarge");
  std::vector<uint8_t> out;
  out.reserve(12 + n_ch + n_bytes);
  put_u32(out, kProofVersion);
  put_u32(out, (uint32_t)n_ch);
  out.insert(out.end(), challenger, challenger + n_ch);
  put_u32(out, (uint32_t)n_bytes);
  const uint8_t* t = static_cast<const uint8_t*>(h_transcript);
  if (n_bytes) out.insert(out.end(), t, t + n_bytes);
  return copy_out(out, h_out, cap, len);
}

// h_challenger receives the challenger type NUL-terminated (ch_cap bytes including the NUL).
int binius_proof_decode(const void* h_bytes, size_t len, void* h_transcript, size_t cap,
                        size_t* n_bytes, char* h_challenger, size_t ch_cap) {
  BGPU_ARG(n_bytes != nullptr && (h_bytes != nullptr || len == 0), "NULL argument");
  Cursor c{static_cast<const uint8_t*>(h_bytes), len};
  uint32_t version = 0, n_ch = 0, n = 0;
  BGPU_ARG(c.u32(&version), "NotEnoughBytes: Proof version");
  BGPU_ARG(version == kProofVersion, "InvalidConstruction: Proof::version");
  const uint8_t* ch = nullptr;
  BGPU_ARG(c.u32(&n_ch) && c.take(n_ch, &ch), "NotEnoughBytes: Proof challenger type");
  for (uint32_t i = 0; i < n_ch; i++) BGPU_ARG(ch[i] != 0, "challenger type holds a NUL byte");
  const uint8_t* data = nullptr;
  BGPU_ARG(c.u32(&n) && c.take(n, &data), "NotEnoughBytes: Proof data");
  *n_bytes = n;
  BGPU_ARG(h_challenger == nullptr || ch_cap > n_ch, "challenger buffer too small");
  BGPU_ARG(cap >= n && (h_transcript != nullptr || n == 0), "output buffer too small");
  if (h_challenger) {
    memcpy(h_challenger, ch, n_ch);
    h_challenger[n_ch] = 0;
  }
  if (n) memcpy(h_transcript, data, n);
  return clear_error();
}

// ValueVec::new_from_data: public ++ non_public must fill the committed part exactly; the scratch
// words that follow are zero.  h_out: committed_total_len + n_scratch words.
int binius_value_vec_from_data(const binius_cs* cs, const uint64_t* h_public, size_t n_public,
                               const uint64_t* h_non_public, size_t n_non_public,
                               uint64_t* h_out) {
  BGPU_ARG(cs != nullptr && h_out != nullptr, "NULL argument");
  BGPU_ARG((h_public != nullptr || n_public == 0) && (h_non_public != nullptr || n_non_public == 0),
           "NULL argument");
  BGPU_ARG(n_public + n_non_public == cs->committed_total_len,
           "ValueVecLenMismatch: public + non-public != committed_total_len");
  if (n_public) memcpy(h_out, h_public, 8 * n_public);
  if (n_non_public) memcpy(h_out + n_public, h_non_public, 8 * n_non_public);
  memset(h_out + cs->committed_total_len, 0, 8ull * cs->n_scratch);
  return clear_error();
}

}  // extern "C"
