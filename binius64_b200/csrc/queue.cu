// Served / batched proving: a request queue over the prove entry.
//
// A queue owns `n_workers` host threads on one device, each with its own non-blocking CUDA
// stream.  Requests (a prover, i.e. a constraint system with its parameters, and a witness) are
// admitted in FIFO order while the device memory the queue accounts for stays within its HBM
// budget; an admitted request runs binius_prover_prove on its worker's stream with a fresh
// transcript.  Accounted memory: every worker's arena (the chunks it keeps between proofs so that
// the next proof allocates nothing) plus, for a running request, what its workspace estimate
// (binius_prover_workspace_bytes, plus the witness copy for host witnesses) needs beyond the
// chunks its worker already holds.  When the head request does not fit, idle workers give their
// kept chunks back; a request whose estimate exceeds the whole budget is refused at submission
// with BINIUS_E_OOM.  A proof is a chain of Fiat-Shamir rounds that synchronise with the host, so
// requests proving at the same time fill each other's round trips with kernels, and the device
// keeps every witness, codeword and tree resident until that request's proof is emitted.  Each
// proof is exactly the proof of a lone call: no state is shared between requests.
//
// The reference has no serving layer (its CLI proves one statement per process,
// prover/examples/src/cli.rs:455-509); this is the batching / serving wrapper around
// Prover::prove (prover/prover/src/prove.rs:124-303).
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.h"
#include "pdl.cuh"
#include "transcript.h"

using namespace bgpu;

namespace {

typedef std::chrono::steady_clock Clock;

struct Request {
  uint64_t ticket = 0;
  const binius_prover* prover = nullptr;
  const void* witness = nullptr;
  bool on_device = false;
  uint64_t n_words = 0;
  uint64_t bytes = 0;  // admission estimate
  Clock::time_point submitted, started, finished;
  bool done = false;
  double phase_ms[5] = {0, 0, 0, 0, 0};
  int status = BINIUS_OK;
  std::string error;
  std::vector<uint8_t> proof;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct binius_queue {
  int device = 0;
  // in_use: the accounted bytes (every worker's held chunks, plus each running request's
  // reservation beyond them); peak: its maximum since creation
  uint64_t budget = 0, in_use = 0, peak = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> pending;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> requests;
  std::vector<std::thread> workers;
  std::vector<cudaStream_t> streams;  // one per worker, created before the workers start
  bool stop = false;
  uint64_t next_ticket = 1;
  uint64_t completed = 0;
  uint32_t n_workers = 0;  // set before the workers start

  void worker_loop(uint32_t w);
};

void binius_queue::worker_loop(uint32_t w) {
  cudaSetDevice(device);
  // Workers poll a finished-yet event for a short while before they sleep on it: most waits of a
  // proof end within the poll, and waking from a blocking sync costs more than the poll.  With
  // more workers than host cores, polling workers take the cores from the ones that launch
  // (measured: 32 workers on 16 cores gave half the throughput of 16), so they sleep at once.
  set_blocking_waits(true, n_workers <= std::max(1u, std::thread::hardware_concurrency()) ? 100.0
                                                                                           : 0.0);
  cudaStream_t s = streams[w];
  set_pdl_enabled(true);
  uint64_t held = 0;  // this worker's arena bytes, counted in in_use
  for (;;) {
    std::shared_ptr<Request> r;
    uint64_t reserved = 0;
    {
      std::unique_lock<std::mutex> lock(mu);
      bool give_back = false;
      for (;;) {
        if (pending.empty()) {
          if (stop) break;
        } else {
          // FIFO admission: the head request runs here if the accounted memory with its
          // reservation (the estimate, of which this worker's kept chunks already cover part)
          // fits the budget.  Otherwise an idle worker that keeps chunks gives them back, so
          // that the memory kept by idle workers cannot hold the head request off for good.
          const uint64_t need = std::max(pending.front()->bytes, held);
          if (in_use - held + need <= budget) {
            r = pending.front();
            pending.pop_front();
            reserved = need;
            in_use += need - held;
            peak = std::max(peak, in_use);
            r->started = Clock::now();
            break;
          }
          if (held) {
            give_back = true;
            break;
          }
        }
        cv_work.wait(lock);
      }
      if (!r && !give_back) break;  // stopped
      if (give_back) {
        in_use -= held;
        held = 0;
      }
    }
    if (!r) {  // give the kept chunks back to the pool and let the others re-check
      arena_release_thread();
      stream_wait(s);
      cv_work.notify_all();
      continue;
    }
    int rc = BINIUS_OK;
    std::string err;
    std::vector<uint8_t> proof;
    const void* d_w = r->witness;
    void* owned = nullptr;
    // the proof's device buffers come from this worker's arena, kept for its next proof
    ArenaScope arena(s, true);
    if (!r->on_device) {
      cudaError_t e = dev_alloc(&owned, 8 * r->n_words, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(owned, r->witness, 8 * r->n_words, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) rc = cuda_error(e, "queue witness upload");
      d_w = owned;
    }
    double phases[5] = {0, 0, 0, 0, 0};
    if (!rc) {
      binius_transcript tr;
      rc = binius_prover_prove(r->prover, d_w, &tr, s);
      if (!rc) proof = tr.t.tape();
      binius_prover_phase_ms(r->prover, phases);
    }
    if (rc) err = binius_last_error();
    if (owned) dev_free(owned, s);
    stream_wait(s);
    const uint64_t held_now = arena_held_bytes();
    // a proof that started from an empty arena measured the prover's real footprint
    if (!rc && held == 0 && r->on_device) prover_note_footprint(r->prover, held_now);
    {
      std::lock_guard<std::mutex> lock(mu);
      in_use = in_use - reserved + held_now;
      held = held_now;
      peak = std::max(peak, in_use);
      r->finished = Clock::now();
      r->status = rc;
      r->error = err;
      r->proof.swap(proof);
      memcpy(r->phase_ms, phases, sizeof(phases));
      r->done = true;
      completed++;
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
  arena_release_thread();
  stream_wait(s);
}

extern "C" {

int binius_queue_create(int device, uint32_t n_workers, uint64_t hbm_budget_bytes,
                        binius_queue** out) {
  BGPU_ARG(out != nullptr, "NULL argument");
  *out = nullptr;
  BGPU_ARG(n_workers >= 1 && n_workers <= 256, "n_workers must be in [1, 256]");
  BGPU_CUDA(cudaSetDevice(device));
  if (int rc = configure_device_pool(device)) return rc;
  binius_queue* q = new binius_queue();
  q->device = device;
  if (hbm_budget_bytes == 0) {
    size_t free_b = 0, total_b = 0;
    cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) {
      delete q;
      return cuda_error(e, "cudaMemGetInfo");
    }
    hbm_budget_bytes = (uint64_t)(0.9 * (double)free_b);
  }
  q->budget = hbm_budget_bytes;
  // Reserve pool capacity up front (allocate and release one block; the pool keeps it cached):
  // proofs running side by side then carve their scratch from cached memory instead of growing
  // the pool, which maps memory under the pool's lock while every other proof waits.
  {
    const uint64_t reserve = hbm_budget_bytes / 2 < (8ull << 30) ? hbm_budget_bytes / 2 : (8ull << 30);
    void* p = nullptr;
    if (reserve && cudaMallocAsync(&p, reserve, 0) == cudaSuccess) {
      cudaFreeAsync(p, 0);
      cudaStreamSynchronize(0);
    }
    cudaGetLastError();
  }
  q->n_workers = n_workers;
  for (uint32_t i = 0; i < n_workers; i++) {
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      for (cudaStream_t t : q->streams) cudaStreamDestroy(t);
      delete q;
      return cuda_error(e, "queue worker stream");
    }
    q->streams.push_back(s);
  }
  for (uint32_t i = 0; i < n_workers; i++) q->workers.emplace_back([q, i] { q->worker_loop(i); });
  *out = q;
  return clear_error();
}

int binius_queue_destroy(binius_queue* q) {
  if (!q) return BINIUS_OK;
  {
    // requests not yet admitted are cancelled; admitted ones run to completion
    std::lock_guard<std::mutex> lock(q->mu);
    for (auto& r : q->pending) {
      r->status = BINIUS_E_ARG;
      r->error = "queue destroyed before the request was admitted";
      r->done = true;
    }
    q->pending.clear();
    q->stop = true;
  }
  q->cv_work.notify_all();
  q->cv_done.notify_all();
  for (auto& w : q->workers) w.join();
  for (cudaStream_t s : q->streams) cudaStreamDestroy(s);
  delete q;
  return BINIUS_OK;
}

int binius_queue_submit(binius_queue* q, const binius_prover* prover, const void* witness,
                        int witness_on_device, uint64_t* ticket) {
  BGPU_ARG(q && prover && witness && ticket, "NULL argument");
  auto r = std::make_shared<Request>();
  r->prover = prover;
  r->witness = witness;
  r->on_device = witness_on_device != 0;
  r->n_words = binius_prover_committed_words(prover);
  r->bytes = binius_prover_workspace_bytes(prover) + (r->on_device ? 0 : 8 * r->n_words);
  {
    std::lock_guard<std::mutex> lock(q->mu);
    BGPU_ARG(!q->stop, "queue is shutting down");
    if (r->bytes > q->budget) {
      char buf[160];
      snprintf(buf, sizeof(buf),
               "request needs %llu bytes of device memory, more than the queue's budget of %llu",
               (unsigned long long)r->bytes, (unsigned long long)q->budget);
      return set_error(BINIUS_E_OOM, buf);
    }
    r->ticket = q->next_ticket++;
    r->submitted = Clock::now();
    q->pending.push_back(r);
    q->requests[r->ticket] = r;
    *ticket = r->ticket;
  }
  q->cv_work.notify_all();
  return clear_error();
}

int binius_queue_stats(binius_queue* q, uint64_t* h_out4) {
  BGPU_ARG(q && h_out4, "NULL argument");
  std::lock_guard<std::mutex> lock(q->mu);
  h_out4[0] = q->budget;
  h_out4[1] = q->in_use;
  h_out4[2] = q->peak;
  h_out4[3] = q->completed;
  return clear_error();
}

int binius_queue_poll(binius_queue* q, uint64_t ticket, int* done) {
  BGPU_ARG(q && done, "NULL argument");
  std::lock_guard<std::mutex> lock(q->mu);
  auto it = q->requests.find(ticket);
  BGPU_ARG(it != q->requests.end(), "unknown ticket");
  *done = it->second->done ? 1 : 0;
  return clear_error();
}

int binius_queue_wait(binius_queue* q, uint64_t ticket, void* h_proof, size_t cap, size_t* len,
                      double* h_times8) {
  BGPU_ARG(q && len, "NULL argument");
  std::unique_lock<std::mutex> lock(q->mu);
  auto it = q->requests.find(ticket);
  BGPU_ARG(it != q->requests.end(), "unknown ticket");
  std::shared_ptr<Request> r = it->second;
  q->cv_done.wait(lock, [&] { return r->done; });
  it = q->requests.find(ticket);  // the map may have rehashed while waiting
  if (h_times8) {
    h_times8[0] = ms_between(r->submitted, r->started);  // queued
    h_times8[1] = ms_between(r->started, r->finished);   // proving
    h_times8[2] = ms_between(r->submitted, r->finished); // total latency
    memcpy(h_times8 + 3, r->phase_ms, sizeof(r->phase_ms));
  }
  *len = r->proof.size();
  if (r->status) {
    const int st = r->status;
    const std::string msg = r->error;
    q->requests.erase(it);
    return set_error(st, msg);
  }
  BGPU_ARG(h_proof != nullptr && cap >= r->proof.size(), "proof buffer too small (len set)");
  memcpy(h_proof, r->proof.data(), r->proof.size());
  q->requests.erase(it);
  return clear_error();
}

}  // extern "C"
