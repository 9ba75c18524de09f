// Host-side internals shared by the translation units of libbinius_gpu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/binius_gpu.h"

namespace bgpu {

// Records msg as the calling thread's last error and returns code.
int set_error(int code, const std::string& msg);
int clear_error();
int cuda_error(cudaError_t e, const char* what);

#define BGPU_CUDA(expr)                                    \
  do {                                                     \
    cudaError_t _e = (expr);                               \
    if (_e != cudaSuccess) return ::bgpu::cuda_error(_e, #expr); \
  } while (0)

#define BGPU_LAUNCH_CHECK(what)                            \
  do {                                                     \
    cudaError_t _e = cudaGetLastError();                   \
    if (_e != cudaSuccess) return ::bgpu::cuda_error(_e, what); \
  } while (0)

#define BGPU_ARG(cond, msg)                                \
  do {                                                     \
    if (!(cond)) return ::bgpu::set_error(BINIUS_E_ARG, msg); \
  } while (0)

// Waits for the work queued on s: cudaStreamSynchronize, or (threads that called
// set_blocking_waits(true, us)) an event poll that yields the core for up to `us` microseconds,
// then a blocking-sync wait.
cudaError_t stream_wait(cudaStream_t s);
// A point on s that the calling thread waits for later with mark_wait (one outstanding mark per
// thread), while the work queued on s after it runs on; mark_wait waits as stream_wait does.
cudaError_t stream_mark(cudaStream_t s);
cudaError_t mark_wait();
void set_blocking_waits(bool on, double poll_micros = 100.0);

// Device-to-host reads through a per-thread pinned staging buffer: add() queues copies on the
// stream, wait() synchronises once and scatters them to their destinations.  Small reads from
// pinned memory are truly asynchronous, unlike copies into pageable memory.
class StagedReads {
 public:
  explicit StagedReads(cudaStream_t s);
  int add(void* dst, const void* src, size_t bytes);
  int add2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
            size_t height);
  int wait();

 private:
  struct Pending {
    void* dst;
    uint8_t* stage;
    size_t bytes, dpitch, width, height;
  };
  int reserve(size_t bytes, uint8_t** at);
  cudaStream_t s_;
  size_t used_ = 0;
  std::vector<Pending> pending_;
};

// One staged read: copy, synchronise, return.
int read_sync(void* dst, const void* src, size_t bytes, cudaStream_t s);

// A small pinned buffer of the calling thread, apart from the StagedReads stage: a copy queued
// into it before a later synchronising read (of any kind) has landed once that read returns.
constexpr size_t kEarlyReadBytes = 4096;
int early_read_buffer(uint8_t** out);

// Stream-ordered device allocations of the prove path.  Inside an ArenaScope on the calling
// thread (same stream), dev_alloc bump-allocates from a few large chunks the scope took from the
// stream-ordered pool and dev_free of such a buffer does nothing: the scope releases (or, for a
// proving-queue worker, keeps for its next proof) the chunks at its end.  Outside a scope they are
// cudaMallocAsync / cudaFreeAsync.  The pool serialises concurrent threads: measured on B200, 8
// threads that interleave pool calls with their launches issue a fifth of the launches that 8
// threads without them do, so a proof takes a handful of chunks instead of ~100 allocations.
cudaError_t dev_alloc_raw(void** p, size_t bytes, cudaStream_t s);
cudaError_t dev_free(void* p, cudaStream_t s);
template <class T>
cudaError_t dev_alloc(T** p, size_t bytes, cudaStream_t s) {
  return dev_alloc_raw(reinterpret_cast<void**>(p), bytes, s);
}

class ArenaScope {
 public:
  // keep: at the end, keep the chunks with this thread for its next scope on the same stream
  // (a stream that outlives the thread's proofs, as a queue worker's does).
  ArenaScope(cudaStream_t s, bool keep);
  ~ArenaScope();
  ArenaScope(const ArenaScope&) = delete;
  ArenaScope& operator=(const ArenaScope&) = delete;

 private:
  bool owner_ = false;
};

// Returns the calling thread's kept arena chunks to the pool (a queue worker, before it destroys
// its stream, or when the memory it keeps stands in the way of the next request).
void arena_release_thread();
// Device bytes the calling thread's arena holds (its chunks, in use or kept).
uint64_t arena_held_bytes();

// Records that a proof of P took `bytes` of arena chunks from an empty arena (prover.cu).
void prover_note_footprint(const binius_prover* P, uint64_t bytes);

// Launch-shape choices of the prove path that change no result, only speed (exact arithmetic: any
// choice gives identical bytes).  A prover carries its own (binius_prover_autotune measures them
// per statement shape); standalone entry points use the defaults.
struct Tuning {
  uint32_t tail_log = 11;          // sumcheck rounds on <= 2^tail_log elements: single-CTA tail
  uint32_t ntt_pass_layers = 8;    // NTT layers fused per shared-memory pass (<= 8)
  uint32_t merkle_leaf_fuse = 8;   // Merkle leaf CTA: 2^fuse leaves, as many layers above them
  uint32_t merkle_node_fuse = 9;   // Merkle node CTA: 2^fuse inputs (<= 9)
  uint32_t ntt_tile_bits = 12;     // NTT shared-memory tile: 2^bits elements (9..12)
};
// The calling thread's current choices (a prove sets its prover's for its duration).
const Tuning& tuning();
class TuningScope {
 public:
  explicit TuningScope(const Tuning& t);
  ~TuningScope();
  TuningScope(const TuningScope&) = delete;
  TuningScope& operator=(const TuningScope&) = delete;

 private:
  Tuning saved_;
};

// Sets the dynamic shared memory limit of a kernel once per device (see common.cu).
int ensure_smem_limit(const void* func, size_t bytes);

// Keeps the default memory pool of `device` from releasing cached blocks (see common.cu).
int configure_device_pool(int device);

// Cumulative number of kernels this library has launched (all devices, all threads).
void count_launch(uint64_t n = 1);

static inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Host GF(2^128) arithmetic (portable carry-less multiply); used only for domain set-up, which
// the reference also performs on the host (Prover::setup, prover/prover/src/prove.rs:95-121).
typedef unsigned __int128 hu128;
hu128 host_gf_mul(hu128 a, hu128 b);
hu128 host_gf_inv(hu128 a);

}  // namespace bgpu

struct binius_ntt {
  int device;
  uint32_t log_domain;
  void* d_twiddles;  // (2^log_domain - 1) elements of 16 bytes
};
