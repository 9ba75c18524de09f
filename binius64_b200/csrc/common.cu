// Error reporting, version and host field helpers of libbinius_gpu.
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <chrono>
#include <mutex>
#include <thread>
#include <vector>

#if defined(__PCLMUL__) && defined(__SSE4_1__)
#include <immintrin.h>
#endif

#include "internal.h"
#include "pdl.cuh"

namespace bgpu {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int clear_error() {
  g_last_error.clear();
  return BINIUS_OK;
}

int cuda_error(cudaError_t e, const char* what) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
  return set_error(e == cudaErrorMemoryAllocation ? BINIUS_E_OOM : BINIUS_E_CUDA, buf);
}

static inline void clmul64(uint64_t a, uint64_t b, uint64_t& lo, uint64_t& hi) {
  uint64_t l = 0, h = 0;
  for (int i = 0; i < 64; i++) {
    uint64_t m = (uint64_t)0 - ((b >> i) & 1);
    l ^= (a << i) & m;
    if (i) h ^= (a >> (64 - i)) & m;
  }
  lo = l;
  hi = h;
}

hu128 host_gf_mul(hu128 a, hu128 b) {
  uint64_t a0 = (uint64_t)a, a1 = (uint64_t)(a >> 64), b0 = (uint64_t)b, b1 = (uint64_t)(b >> 64);
  uint64_t l0, l1, h0, h1, m0, m1, x0, x1;
#if defined(__PCLMUL__) && defined(__SSE4_1__)
  // PCLMULQDQ for the host side of the protocol (scalar interpolation and challenges).
  __m128i va = _mm_set_epi64x((long long)a1, (long long)a0);
  __m128i vb = _mm_set_epi64x((long long)b1, (long long)b0);
  __m128i l = _mm_clmulepi64_si128(va, vb, 0x00), h = _mm_clmulepi64_si128(va, vb, 0x11);
  __m128i m = _mm_clmulepi64_si128(va, vb, 0x01), x = _mm_clmulepi64_si128(va, vb, 0x10);
  l0 = (uint64_t)_mm_cvtsi128_si64(l);
  l1 = (uint64_t)_mm_extract_epi64(l, 1);
  h0 = (uint64_t)_mm_cvtsi128_si64(h);
  h1 = (uint64_t)_mm_extract_epi64(h, 1);
  m0 = (uint64_t)_mm_cvtsi128_si64(m);
  m1 = (uint64_t)_mm_extract_epi64(m, 1);
  x0 = (uint64_t)_mm_cvtsi128_si64(x);
  x1 = (uint64_t)_mm_extract_epi64(x, 1);
#else
  clmul64(a0, b0, l0, l1);
  clmul64(a1, b1, h0, h1);
  clmul64(a0, b1, m0, m1);
  clmul64(a1, b0, x0, x1);
#endif
  uint64_t p0 = l0, p1 = l1 ^ m0 ^ x0, p2 = h0 ^ m1 ^ x1, p3 = h1;
  uint64_t t = (p3 >> 63) ^ (p3 >> 62) ^ (p3 >> 57);
  uint64_t lo = p0 ^ p2 ^ (p2 << 1) ^ (p2 << 2) ^ (p2 << 7) ^ t ^ (t << 1) ^ (t << 2) ^ (t << 7);
  uint64_t hi = p1 ^ p3 ^ ((p3 << 1) | (p2 >> 63)) ^ ((p3 << 2) | (p2 >> 62)) ^
                ((p3 << 7) | (p2 >> 57));
  return ((hu128)hi << 64) | lo;
}

// a^(2^128 - 2) by the chain a^(2^k - 1) = (a^(2^(k-1) - 1))^2 * a.
hu128 host_gf_inv(hu128 a) {
  hu128 r = a;
  for (int k = 2; k <= 127; k++) r = host_gf_mul(host_gf_mul(r, r), a);
  return host_gf_mul(r, r);
}

// Raises the dynamic shared memory limit of `func` on the current device to `bytes`, once per
// (device, kernel).  Setting a per-launch value instead races between threads that launch the
// same kernel with different sizes.
int ensure_smem_limit(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::vector<std::pair<int, const void*>> done;
  int dev = 0;
  BGPU_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  for (auto& d : done)
    if (d.first == dev && d.second == func) return BINIUS_OK;
  BGPU_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  done.emplace_back(dev, func);
  return BINIUS_OK;
}

// ---- staged device-to-host reads

namespace {
struct PinnedStage {
  uint8_t* buf = nullptr;
  ~PinnedStage() {
    if (buf) cudaFreeHost(buf);
  }
};
thread_local PinnedStage t_stage;
// The stage is allocated once per thread and never resized: cudaFreeHost and cudaHostAlloc
// synchronise with the device, which would stall every concurrent proof.  Reads that do not fit
// go straight to pageable memory.
constexpr size_t kStageBytes = 4u << 20;
}  // namespace

StagedReads::StagedReads(cudaStream_t s) : s_(s) {}

int StagedReads::reserve(size_t bytes, uint8_t** at) {
  *at = nullptr;
  const size_t need = used_ + ((bytes + 15) & ~size_t(15));
  if (need > kStageBytes) return BINIUS_OK;  // the caller copies directly
  if (!t_stage.buf)
    BGPU_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&t_stage.buf), kStageBytes,
                            cudaHostAllocDefault));
  *at = t_stage.buf + used_;
  used_ = need;
  return BINIUS_OK;
}

int StagedReads::add(void* dst, const void* src, size_t bytes) {
  uint8_t* at = nullptr;
  if (int rc = reserve(bytes, &at)) return rc;
  if (!at) {  // larger than the stage: a pageable copy, complete when the call returns
    BGPU_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s_));
    return BINIUS_OK;
  }
  BGPU_CUDA(cudaMemcpyAsync(at, src, bytes, cudaMemcpyDeviceToHost, s_));
  pending_.push_back({dst, at, bytes, 0, 0, 0});
  return BINIUS_OK;
}

int StagedReads::add2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                       size_t height) {
  uint8_t* at = nullptr;
  if (int rc = reserve(width * height, &at)) return rc;
  if (!at) {
    BGPU_CUDA(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyDeviceToHost,
                                s_));
    return BINIUS_OK;
  }
  BGPU_CUDA(cudaMemcpy2DAsync(at, width, src, spitch, width, height, cudaMemcpyDeviceToHost, s_));
  pending_.push_back({dst, at, width, dpitch, width, height});
  return BINIUS_OK;
}

int StagedReads::wait() {
  BGPU_CUDA(stream_wait(s_));
  for (const auto& p : pending_) {
    if (p.height == 0) {
      memcpy(p.dst, p.stage, p.bytes);
    } else {
      for (size_t r = 0; r < p.height; r++)
        memcpy(static_cast<uint8_t*>(p.dst) + r * p.dpitch, p.stage + r * p.width, p.width);
    }
  }
  pending_.clear();
  used_ = 0;
  return BINIUS_OK;
}

namespace {

struct ArenaChunk {
  uint8_t* base;
  size_t size, used;
};

struct Arena {
  cudaStream_t s = nullptr;
  bool active = false, keep = false;
  std::vector<ArenaChunk> chunks;
  bool owns(const void* p) const {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    for (const auto& c : chunks)
      if (b >= c.base && b < c.base + c.size) return true;
    return false;
  }
  void release() {
    for (const auto& c : chunks) cudaFreeAsync(c.base, s);
    chunks.clear();
  }
};

thread_local Arena t_arena;
constexpr size_t kArenaChunk = 64ull << 20;

// Host-side allocation-failure injection (binius_debug_fail_allocs): the number of device
// allocations that still succeed before the next one is refused, or -1 when off.
std::atomic<int64_t> g_allocs_before_failure{-1};

}  // namespace

cudaError_t dev_alloc_raw(void** p, size_t bytes, cudaStream_t s) {
  int64_t left = g_allocs_before_failure.load(std::memory_order_relaxed);
  while (left >= 0) {
    if (g_allocs_before_failure.compare_exchange_weak(left, left - 1)) {
      if (left == 0) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;  // as the pool reports an allocation it cannot serve
      }
      break;
    }
  }
  Arena& a = t_arena;
  if (!a.active || a.s != s) return cudaMallocAsync(p, bytes ? bytes : 16, s);
  const size_t need = (bytes + 255) & ~size_t(255);
  for (auto& c : a.chunks)  // first fit among the scope's few chunks
    if (c.used + need <= c.size) {
      *p = c.base + c.used;
      c.used += need;
      return cudaSuccess;
    }
  void* base = nullptr;
  const size_t size = need > kArenaChunk ? need : kArenaChunk;
  cudaError_t e = cudaMallocAsync(&base, size, s);
  if (e != cudaSuccess) return e;
  a.chunks.push_back({static_cast<uint8_t*>(base), size, need});
  *p = base;
  return cudaSuccess;
}

cudaError_t dev_free(void* p, cudaStream_t s) {
  if (!p) return cudaSuccess;
  const Arena& a = t_arena;
  if (a.active && a.s == s && a.owns(p)) return cudaSuccess;  // released with the scope
  return cudaFreeAsync(p, s);
}

ArenaScope::ArenaScope(cudaStream_t s, bool keep) {
  Arena& a = t_arena;
  if (a.active) return;  // nested: the outer scope serves the allocations
  if (a.s != s) {        // kept chunks of another stream go back to the pool first
    a.release();
    a.s = s;
  }
  a.active = true;
  a.keep = keep;
  owner_ = true;
}

ArenaScope::~ArenaScope() {
  if (!owner_) return;
  Arena& a = t_arena;
  a.active = false;
  if (a.keep) {
    for (auto& c : a.chunks) c.used = 0;  // the next proof on this stream runs after this one
  } else {
    a.release();
    a.s = nullptr;
  }
}

void arena_release_thread() {
  Arena& a = t_arena;
  if (a.active) return;
  a.release();
  a.s = nullptr;
}

namespace {
thread_local Tuning t_tuning;
thread_local bool t_pdl = true;
}  // namespace

bool pdl_enabled() { return t_pdl; }
void set_pdl_enabled(bool on) { t_pdl = on; }

const Tuning& tuning() { return t_tuning; }
TuningScope::TuningScope(const Tuning& t) : saved_(t_tuning) { t_tuning = t; }
TuningScope::~TuningScope() { t_tuning = saved_; }

uint64_t arena_held_bytes() {
  uint64_t n = 0;
  for (const auto& c : t_arena.chunks) n += c.size;
  return n;
}

namespace {
struct PinnedSmall {
  uint8_t* buf = nullptr;
  ~PinnedSmall() {
    if (buf) cudaFreeHost(buf);
  }
};
thread_local PinnedSmall t_early;
}  // namespace

int early_read_buffer(uint8_t** out) {
  if (!t_early.buf)
    BGPU_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&t_early.buf), kEarlyReadBytes,
                            cudaHostAllocDefault));
  *out = t_early.buf;
  return BINIUS_OK;
}

int read_sync(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  StagedReads r(s);
  if (int rc = r.add(dst, src, bytes)) return rc;
  return r.wait();
}

// Waits for the work queued on `s`.  Threads that enable shared waits (the proving workers of a
// queue, many of which wait at once) poll an event and yield the core between polls for a short
// while -- most round trips of a proof end within it -- and then sleep on the event (blocking
// sync): polling without end from many threads contends for the driver, and sleeping at once
// would add the driver's wake-up latency to each of a proof's ~100 round trips.
namespace {
thread_local bool t_blocking_wait = false;
thread_local cudaEvent_t t_wait_event = nullptr;
thread_local double t_poll_micros = 100.0;
}  // namespace

void set_blocking_waits(bool on, double poll_micros) {
  t_blocking_wait = on;
  t_poll_micros = poll_micros;
}

cudaError_t stream_wait(cudaStream_t s) {
  if (!t_blocking_wait) return cudaStreamSynchronize(s);
  if (!t_wait_event) {
    cudaError_t e = cudaEventCreateWithFlags(&t_wait_event,
                                             cudaEventBlockingSync | cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = cudaEventRecord(t_wait_event, s);
  if (e != cudaSuccess) return e;
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    e = cudaEventQuery(t_wait_event);
    if (e != cudaErrorNotReady) return e;
    if (std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count() >=
        t_poll_micros)
      return cudaEventSynchronize(t_wait_event);
    std::this_thread::yield();
  }
}

namespace {
thread_local cudaEvent_t t_mark_event = nullptr;
}  // namespace

cudaError_t stream_mark(cudaStream_t s) {
  if (!t_mark_event) {
    cudaError_t e = cudaEventCreateWithFlags(&t_mark_event,
                                             cudaEventBlockingSync | cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
  }
  return cudaEventRecord(t_mark_event, s);
}

cudaError_t mark_wait() {
  if (!t_mark_event) return cudaErrorInvalidResourceHandle;
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t e = cudaEventQuery(t_mark_event);
    if (e != cudaErrorNotReady) return e;
    if (t_blocking_wait) {
      if (std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0)
              .count() >= t_poll_micros)
        return cudaEventSynchronize(t_mark_event);
      std::this_thread::yield();
    }
  }
}

// The stream-ordered allocator of `device` keeps freed blocks cached (release threshold = max)
// instead of returning them to the driver at every synchronisation: a proof synchronises once per
// sumcheck round and reallocates its scratch per phase.  The attribute belongs to this process's
// default pool; it changes no setting of the GPU.
int configure_device_pool(int device) {
  static std::mutex mu;
  static std::vector<int> done;
  std::lock_guard<std::mutex> lock(mu);
  for (int d : done)
    if (d == device) return BINIUS_OK;
  cudaMemPool_t pool;
  BGPU_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t threshold = ~0ull;
  BGPU_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
  done.push_back(device);
  return BINIUS_OK;
}

}  // namespace bgpu

extern "C" {

const char* binius_last_error(void) { return bgpu::g_last_error.c_str(); }

const char* binius_version(void) { return "binius64_b200 0.1.0 (sm_100a)"; }

uint64_t binius_launch_count(void) { return bgpu::g_launches.load(std::memory_order_relaxed); }

void binius_debug_fail_allocs(int64_t n_before_failure) {
  bgpu::g_allocs_before_failure.store(n_before_failure < 0 ? -1 : n_before_failure);
}

}  // extern "C"
