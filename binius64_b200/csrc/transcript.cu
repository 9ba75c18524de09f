// C ABI of the host-side Fiat-Shamir transcript (transcript.h), and the host side of device
// transcript stretches (dev_transcript.cuh).
#include <stdio.h>
#include <stdlib.h>

#include "dev_transcript.cuh"
#include "internal.h"
#include "transcript.h"

using namespace bgpu;

namespace {

__global__ void transcript_load_kernel(TranscriptState st, TranscriptState* dst) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = st;
}

__global__ void transcript_message_kernel(TranscriptState* ts, uint8_t* tape,
                                          const uint32_t* __restrict__ words, uint32_t n) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  DevTr st;
  st.load(ts);
  st.message_words(tape, words, n);
  st.store(ts);
}

}  // namespace

namespace bgpu {

DeviceTranscript::~DeviceTranscript() {
  if (mem_) dev_free(mem_, s_);
}

int DeviceTranscript::begin(const Transcript& t, cudaStream_t s) {
  s_ = s;
  if (!mem_) BGPU_CUDA(dev_alloc(reinterpret_cast<void**>(&mem_), kStateBytes + kTapeCap, s));
  TranscriptState st;
  t.save(st);
  st.tape_cap = kTapeCap;
  transcript_load_kernel<<<1, 32, 0, s>>>(st, state());
  BGPU_LAUNCH_CHECK("transcript_load_kernel");
  count_launch();
  return BINIUS_OK;
}

int DeviceTranscript::message_device(const void* d_bytes, uint32_t n_bytes, cudaStream_t s) {
  if (n_bytes % 4 || reinterpret_cast<uintptr_t>(d_bytes) % 4)
    return set_error(BINIUS_E_ARG, "device message: whole aligned words only");
  transcript_message_kernel<<<1, 32, 0, s>>>(state(), tape(),
                                             static_cast<const uint32_t*>(d_bytes), n_bytes / 4);
  BGPU_LAUNCH_CHECK("transcript_message_kernel");
  count_launch();
  return BINIUS_OK;
}

int DeviceTranscript::read(StagedReads& rd, uint32_t tape_bytes) {
  if (tape_bytes > kTapeCap) return set_error(BINIUS_E_ARG, "device transcript tape too small");
  expect_ = tape_bytes;
  host_tape_.resize(tape_bytes);
  if (int rc = rd.add(&host_state_, state(), sizeof(TranscriptState))) return rc;
  if (tape_bytes)
    if (int rc = rd.add(host_tape_.data(), tape(), tape_bytes)) return rc;
  return BINIUS_OK;
}

int DeviceTranscript::finish(Transcript& t) {
  if (host_state_.error || host_state_.tape_len != expect_)
    return set_error(BINIUS_E_CUDA, "device transcript wrote an unexpected number of bytes");
  t.load(host_state_, host_tape_.data());
  return BINIUS_OK;
}

}  // namespace bgpu

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

// ProverTranscript::finalize (verifier/transcript/src/transcript.rs:245-284), including its proof
// dump: with BINIUS_DUMP_PROOF set, the proof bytes are also written to the file it names.
int binius_transcript_finalize(const binius_transcript* t, void* h_out, size_t cap, size_t* len) {
  BGPU_ARG(t != nullptr && len != nullptr, "NULL argument");
  *len = t->t.tape().size();
  BGPU_ARG(cap >= *len && (h_out != nullptr || *len == 0), "proof buffer too small");
  if (*len) memcpy(h_out, t->t.tape().data(), *len);
  if (const char* path = getenv("BINIUS_DUMP_PROOF")) {
    FILE* f = fopen(path, "wb");
    BGPU_ARG(f != nullptr, "BINIUS_DUMP_PROOF: cannot create the proof dump file");
    const size_t wrote = *len ? fwrite(t->t.tape().data(), 1, *len, f) : 0;
    const int closed = fclose(f);
    BGPU_ARG(wrote == *len && closed == 0, "BINIUS_DUMP_PROOF: cannot write the proof dump file");
  }
  return clear_error();
}

}  // extern "C"
