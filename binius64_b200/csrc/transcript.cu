// C ABI of the host-side Fiat-Shamir transcript (transcript.h).
#include "internal.h"
#include "transcript.h"

using namespace bgpu;

extern "C" {

int binius_transcript_create(binius_transcript** out) {
  BGPU_ARG(out != nullptr, "out is NULL");
  *out = new binius_transcript();
  return clear_error();
}

int binius_transcript_destroy(binius_transcript* t) {
  delete t;
  return BINIUS_OK;
}

int binius_transcript_message(binius_transcript* t, const void* h_bytes, size_t n) {
  BGPU_ARG(t != nullptr && (h_bytes != nullptr || n == 0), "NULL argument");
  t->t.message(h_bytes, n);
  return clear_error();
}

int binius_transcript_decommitment(binius_transcript* t, const void* h_bytes, size_t n) {
  BGPU_ARG(t != nullptr && (h_bytes != nullptr || n == 0), "NULL argument");
  t->t.decommitment(h_bytes, n);
  return clear_error();
}

int binius_transcript_observe(binius_transcript* t, const void* h_bytes, size_t n) {
  BGPU_ARG(t != nullptr && (h_bytes != nullptr || n == 0), "NULL argument");
  t->t.observe(static_cast<const uint8_t*>(h_bytes), n);
  return clear_error();
}

int binius_transcript_sample(binius_transcript* t, void* h_out, size_t n) {
  BGPU_ARG(t != nullptr && (h_out != nullptr || n == 0), "NULL argument");
  t->t.sample_bytes(static_cast<uint8_t*>(h_out), n);
  return clear_error();
}

uint32_t binius_transcript_sample_bits(binius_transcript* t, uint32_t bits) {
  return t ? t->t.sample_bits(bits) : 0;
}

size_t binius_transcript_len(const binius_transcript* t) { return t ? t->t.tape().size() : 0; }

int binius_transcript_finalize(const binius_transcript* t, void* h_out, size_t cap, size_t* len) {
  BGPU_ARG(t != nullptr && len != nullptr, "NULL argument");
  *len = t->t.tape().size();
  BGPU_ARG(cap >= *len && (h_out != nullptr || *len == 0), "proof buffer too small");
  if (*len) memcpy(h_out, t->t.tape().data(), *len);
  return clear_error();
}

}  // extern "C"
