// Witness evaluation on the device: the frontend's evaluation-form bytecode
// (verifier/frontend/src/compiler/eval_form/interpreter.rs, Interpreter::run) run over a batch of
// value vectors, with the Word arithmetic of verifier/core/src/word.rs.
//
// The reference interprets the program once per witness, one instruction after another.  Here
// the program is decoded once on the host into fixed-width instructions and level-scheduled: an
// instruction's level is one more than the levels of the instructions it depends on (the last
// writer of each source, and, so that a register written twice keeps the program's order, the
// last reader and writer of its destination).  Instructions of one level are independent; a
// level runs as one launch whose threads are (instruction, instance) pairs, consecutive threads
// the same instruction of consecutive instances.  The batch is laid out register-major
// (values[reg * batch + instance]), so a warp's loads and stores of one register are one 256-byte
// segment and the instruction is a broadcast.  Frontend programs assign each wire once, so a
// level holds every instruction whose inputs are ready: wide circuits run in a few launches,
// while a chain of dependent instructions (a hash's rounds) needs one launch per link and a large
// batch to fill the GPU.
//
// Runs of narrow levels (at most 64 instructions each) go to a kernel whose CTAs each take a group
// of instances through all of them, separated by barriers instead of launches.
//
// Assertions count their failures per instance and keep the earliest failing assertion in
// program order (its instruction index and id); the reference collects up to 100 messages.
// Decoding rejects what the reference would panic on: an unknown opcode, a register outside the
// value vector, a truncated instruction, a shift amount of 64 or more; and hint calls (0x80),
// whose handlers are host code.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "internal.h"

using namespace bgpu;

struct EfInsn {
  uint8_t op, imm;
  uint16_t pad;
  uint32_t r[5];  // per opcode: destinations first, then sources (see decode)
};
static_assert(sizeof(EfInsn) == 24, "instruction layout");

struct binius_eval_form {
  int device = 0;
  uint64_t n_values = 0, n_insn = 0, n_asserts = 0, max_width = 0, n_accesses = 0;
  std::vector<uint64_t> level_start;  // level k holds instructions [start[k], start[k+1])
  EfInsn* d_insn = nullptr;           // level order
  uint32_t* d_prog_index = nullptr;   // program position of each (for assertion order)
  uint32_t* d_side = nullptr;         // bxor_multi source lists
  uint64_t* d_level_start = nullptr;  // level_start on the device (for the segment kernel)
};

namespace {

struct Decoder {
  const uint8_t* p;
  size_t len, pc = 0;
  uint64_t n_values;
  const char* err = nullptr;
  uint8_t u8() {
    if (pc + 1 > len) {
      err = "truncated instruction";
      return 0;
    }
    return p[pc++];
  }
  uint32_t u32() {
    if (pc + 4 > len) {
      err = "truncated instruction";
      return 0;
    }
    uint32_t x;
    memcpy(&x, p + pc, 4);
    pc += 4;
    return x;
  }
  uint32_t reg() {
    const uint32_t r = u32();
    if (!err && r >= n_values) err = "register outside the value vector";
    return r;
  }
  uint8_t shift() {
    const uint8_t s = u8();
    if (!err && s >= 64) err = "shift amount >= 64";
    return s;
  }
};

// Decodes one instruction into `in` (sources that are lists go to `side`); returns its
// destinations and sources through `dst` / `src` for the scheduler.
bool decode_one(Decoder& d, EfInsn& in, std::vector<uint32_t>& side, uint32_t dst[2],
                uint32_t& n_dst, std::vector<uint32_t>& src) {
  memset(&in, 0, sizeof(in));
  src.clear();
  n_dst = 0;
  const uint8_t op = d.u8();
  in.op = op;
  auto regs = [&](int nd, int ns) {
    for (int i = 0; i < nd; i++) in.r[i] = dst[n_dst++] = d.reg();
    for (int i = 0; i < ns; i++) {
      in.r[nd + i] = d.reg();
      src.push_back(in.r[nd + i]);
    }
  };
  switch (op) {
    case 0x01: case 0x02: case 0x03: regs(1, 2); break;            // band, bor, bxor
    case 0x05: regs(1, 3); break;                                   // select(dst, cond, t, f)
    case 0x07: regs(1, 3); break;                                   // fax
    case 0x06: {                                                     // bxor_multi
      in.r[0] = dst[n_dst++] = d.reg();
      const uint32_t cnt = d.u32();
      if (d.err) break;
      if (cnt > (1u << 24)) {
        d.err = "bxor_multi source count too large";
        break;
      }
      in.r[1] = (uint32_t)side.size();
      in.r[2] = cnt;
      for (uint32_t i = 0; i < cnt && !d.err; i++) {
        const uint32_t s = d.reg();
        side.push_back(s);
        src.push_back(s);
      }
      if (side.size() > 0xffffffffull) d.err = "program too large";
      break;
    }
    case 0x10: case 0x11: case 0x12: case 0x42:                      // sll, slr, sar, shr32
      regs(1, 1);
      in.imm = d.shift();
      break;
    case 0x41: case 0x43: case 0x50: case 0x51:                      // rotr32, rotr, masks
      regs(1, 1);
      in.imm = d.u8();
      break;
    case 0x20: case 0x40: regs(2, 2); break;                          // iadd_cout(32)
    case 0x21: case 0x23: regs(2, 3); break;                          // with carry / borrow in
    case 0x30: case 0x31: regs(2, 2); break;                          // imul, smul
    case 0x60: regs(0, 2); in.r[4] = d.u32(); break;                  // assert_eq
    case 0x61: regs(0, 3); in.r[4] = d.u32(); break;                  // assert_eq_cond
    case 0x62: case 0x63: case 0x64: case 0x65: regs(0, 1); in.r[4] = d.u32(); break;
    case 0x80: d.err = "hint calls are evaluated by host handlers (not supported here)"; break;
    default: d.err = "unknown opcode"; break;
  }
  return d.err == nullptr;
}

__device__ __forceinline__ uint64_t ld(const uint64_t* v, uint32_t reg, uint32_t batch,
                                       uint32_t inst) {
  return v[(uint64_t)reg * batch + inst];
}

__device__ __forceinline__ void st(uint64_t* v, uint32_t reg, uint32_t batch, uint32_t inst,
                                   uint64_t x) {
  v[(uint64_t)reg * batch + inst] = x;
}

// Executes instruction k (level order) for instance inst.
__device__ __forceinline__ void exec_insn(const EfInsn* __restrict__ insn,
                                          const uint32_t* __restrict__ prog_index,
                                          const uint32_t* __restrict__ side, uint64_t k,
                                          uint32_t batch, uint32_t inst, uint64_t* __restrict__ v,
                                          uint32_t* __restrict__ fails,
                                          unsigned long long* __restrict__ first) {
  const EfInsn in = insn[k];
  const uint32_t* r = in.r;
  switch (in.op) {
    case 0x01: st(v, r[0], batch, inst, ld(v, r[1], batch, inst) & ld(v, r[2], batch, inst)); break;
    case 0x02: st(v, r[0], batch, inst, ld(v, r[1], batch, inst) | ld(v, r[2], batch, inst)); break;
    case 0x03: st(v, r[0], batch, inst, ld(v, r[1], batch, inst) ^ ld(v, r[2], batch, inst)); break;
    case 0x05: {
      const bool c = (ld(v, r[1], batch, inst) >> 63) != 0;
      st(v, r[0], batch, inst, ld(v, c ? r[2] : r[3], batch, inst));
      break;
    }
    case 0x06: {
      uint64_t x = 0;
      for (uint32_t i = 0; i < r[2]; i++) x ^= ld(v, side[r[1] + i], batch, inst);
      st(v, r[0], batch, inst, x);
      break;
    }
    case 0x07:
      st(v, r[0], batch, inst,
         (ld(v, r[1], batch, inst) & ld(v, r[2], batch, inst)) ^ ld(v, r[3], batch, inst));
      break;
    case 0x10: st(v, r[0], batch, inst, ld(v, r[1], batch, inst) << in.imm); break;
    case 0x11: st(v, r[0], batch, inst, ld(v, r[1], batch, inst) >> in.imm); break;
    case 0x12:
      st(v, r[0], batch, inst, (uint64_t)((int64_t)ld(v, r[1], batch, inst) >> in.imm));
      break;
    case 0x20: case 0x21: case 0x23: {
      const uint64_t x = ld(v, r[2], batch, inst), y = ld(v, r[3], batch, inst);
      const uint64_t c = in.op == 0x20 ? 0 : (ld(v, r[4], batch, inst) >> 63);
      if (in.op == 0x23) {
        const uint64_t diff = x - y - c;
        st(v, r[0], batch, inst, diff);
        st(v, r[1], batch, inst, (~x & y) | (~(x ^ y) & diff));
      } else {
        const uint64_t sum = x + y + c;
        st(v, r[0], batch, inst, sum);
        st(v, r[1], batch, inst, (x & y) | ((x ^ y) & ~sum));
      }
      break;
    }
    case 0x30: case 0x31: {
      const uint64_t x = ld(v, r[2], batch, inst), y = ld(v, r[3], batch, inst);
      const uint64_t lo64 = x * y;
      uint64_t hi64 = __umul64hi(x, y);
      if (in.op == 0x31)  // signed high half from the unsigned one
        hi64 -= ((int64_t)x < 0 ? y : 0) + ((int64_t)y < 0 ? x : 0);
      st(v, r[0], batch, inst, hi64);
      st(v, r[1], batch, inst, lo64);
      break;
    }
    case 0x40: {
      const uint64_t x = ld(v, r[2], batch, inst), y = ld(v, r[3], batch, inst), s = x + y;
      st(v, r[0], batch, inst, s & 0xFFFFFFFFull);
      st(v, r[1], batch, inst, (x & y) | ((x ^ y) & ~s));
      break;
    }
    case 0x41: {
      const uint32_t x = (uint32_t)ld(v, r[1], batch, inst);
      st(v, r[0], batch, inst, (uint64_t)__funnelshift_r(x, x, in.imm & 31));
      break;
    }
    case 0x42: st(v, r[0], batch, inst, (ld(v, r[1], batch, inst) >> in.imm) & 0xFFFFFFFFull); break;
    case 0x43: {
      const uint64_t x = ld(v, r[1], batch, inst);
      const uint32_t s = in.imm & 63;
      st(v, r[0], batch, inst, s ? ((x >> s) | (x << (64 - s))) : x);
      break;
    }
    case 0x50: case 0x51: {
      const uint32_t nb = in.imm;
      uint64_t mask = ~0ull;  // also mask_high(0): the reference's shift by 64 wraps to 0
      if (nb < 64 && !(in.op == 0x51 && nb == 0))
        mask = in.op == 0x50 ? ((1ull << nb) - 1) : ~((1ull << (64 - nb)) - 1);
      st(v, r[0], batch, inst, ld(v, r[1], batch, inst) & mask);
      break;
    }
    default: {  // assertions 0x60..0x65
      bool bad;
      if (in.op == 0x60) {
        bad = ld(v, r[0], batch, inst) != ld(v, r[1], batch, inst);
      } else if (in.op == 0x61) {
        bad = (ld(v, r[0], batch, inst) >> 63) &&
              ld(v, r[1], batch, inst) != ld(v, r[2], batch, inst);
      } else {
        const uint64_t x = ld(v, r[0], batch, inst);
        bad = in.op == 0x62 ? x != 0 : in.op == 0x63 ? x == 0
                                      : in.op == 0x64 ? (x >> 63) != 0 : (x >> 63) == 0;
      }
      if (bad) {
        atomicAdd(fails + inst, 1u);
        atomicMin(first + inst, ((unsigned long long)prog_index[k] << 32) | r[4]);
      }
      break;
    }
  }
}

// POW2: batch = 2^log_batch, so the (instruction, instance) split of a thread index is a shift
// and a mask instead of a 64-bit division.
template <bool POW2>
__device__ __forceinline__ void split(uint64_t t, uint32_t batch, uint32_t log_batch,
                                      uint64_t& k, uint32_t& inst) {
  k = POW2 ? (t >> log_batch) : t / batch;
  inst = (uint32_t)(POW2 ? (t & (batch - 1)) : t % batch);
}

// One wide level: (instruction, instance) pairs over the whole grid.
template <bool POW2>
__global__ void __launch_bounds__(256)
    eval_level_kernel(const EfInsn* __restrict__ insn, const uint32_t* __restrict__ prog_index,
                      const uint32_t* __restrict__ side, uint64_t lo, uint64_t n, uint32_t batch,
                      uint32_t log_batch, uint64_t* __restrict__ v, uint32_t* __restrict__ fails,
                      unsigned long long* __restrict__ first) {
  const uint64_t total = n * batch;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t k;
    uint32_t inst;
    split<POW2>(t, batch, log_batch, k, inst);
    exec_insn(insn, prog_index, side, lo + k, batch, inst, v, fails, first);
  }
}

// A run of narrow levels [k0, k1): each CTA takes kSegInstances instances through all of them,
// a barrier between levels instead of a launch (a deep program, e.g. a hash's rounds, is a long
// chain of levels a few instructions wide).  Instances never depend on one another, so the CTAs
// run independently.  __syncthreads makes a level's global stores visible to the CTA.
constexpr uint32_t kSegThreads = 1024;
constexpr uint32_t kSegWidth = 64;      // levels of at most this many instructions are narrow
constexpr uint32_t kSegInstances = 64;  // instances per CTA: <= 4096 items per level

// WARP: one warp per instance (small batches), the levels separated by __syncwarp, which orders
// the warp's global stores before its next loads at a fraction of a CTA barrier's cost.
template <bool WARP>
__global__ void __launch_bounds__(WARP ? 32 : kSegThreads, 1)
    eval_segment_kernel(const EfInsn* __restrict__ insn, const uint32_t* __restrict__ prog_index,
                        const uint32_t* __restrict__ side, const uint64_t* __restrict__ level_start,
                        uint32_t k0, uint32_t k1, uint32_t batch, uint64_t* __restrict__ v,
                        uint32_t* __restrict__ fails, unsigned long long* __restrict__ first) {
  constexpr uint32_t per = WARP ? 1 : kSegInstances;
  const uint32_t i0 = blockIdx.x * per;
  const uint32_t g = batch - i0 < per ? batch - i0 : per;
  for (uint32_t lv = k0; lv < k1; lv++) {
    const uint64_t lo = level_start[lv];
    const uint32_t total = (uint32_t)(level_start[lv + 1] - lo) * g;
    for (uint32_t t = threadIdx.x; t < total; t += blockDim.x)
      exec_insn(insn, prog_index, side, lo + t / g, batch, i0 + t % g, v, fails, first);
    if (WARP)
      __syncwarp();
    else
      __syncthreads();
  }
}

__global__ void init_fail_kernel(uint32_t* fails, unsigned long long* first, uint32_t batch) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < batch; i += gridDim.x * blockDim.x) {
    fails[i] = 0;
    first[i] = ~0ull;
  }
}

// 32x32 tiles through shared memory: out[c * rows + r] = in[r * cols + c]; block b is tile
// (b / col_tiles, b % col_tiles).
__global__ void __launch_bounds__(256) transpose_words_kernel(const uint64_t* __restrict__ in,
                                                              uint64_t rows, uint64_t cols,
                                                              uint64_t col_tiles,
                                                              uint64_t* __restrict__ out) {
  __shared__ uint64_t tile[32][33];
  const uint64_t r0 = (blockIdx.x / col_tiles) * 32, c0 = (blockIdx.x % col_tiles) * 32;
  for (uint32_t i = threadIdx.y; i < 32; i += 8) {
    const uint64_t r = r0 + i, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[i][threadIdx.x] = in[r * cols + c];
  }
  __syncthreads();
  for (uint32_t i = threadIdx.y; i < 32; i += 8) {
    const uint64_t c = c0 + i, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[c * rows + r] = tile[threadIdx.x][i];
  }
}

}  // namespace

extern "C" {

int binius_eval_form_create(const void* h_bytecode, size_t len, uint64_t n_values,
                            binius_eval_form** out) {
  BGPU_ARG(out != nullptr && (h_bytecode != nullptr || len == 0), "NULL argument");
  *out = nullptr;
  BGPU_ARG(n_values >= 1 && n_values <= 0xffffffffull, "n_values must be in [1, 2^32)");
  Decoder d{static_cast<const uint8_t*>(h_bytecode), len, 0, n_values};
  std::vector<EfInsn> prog;
  std::vector<uint32_t> side, src;
  std::vector<uint32_t> level;                               // per instruction
  std::vector<uint32_t> w_level(n_values, 0), r_level(n_values, 0);  // 0: initial value
  uint64_t n_asserts = 0, n_accesses = 0;
  while (d.pc < d.len) {
    EfInsn in;
    uint32_t dst[2], n_dst = 0;
    if (!decode_one(d, in, side, dst, n_dst, src)) {
      char msg[160];
      snprintf(msg, sizeof msg, "eval form bytecode at byte %zu: %s", d.pc, d.err);
      return set_error(BINIUS_E_ARG, msg);
    }
    uint32_t lv = 1;
    for (uint32_t s : src) lv = std::max(lv, w_level[s] + 1);
    for (uint32_t i = 0; i < n_dst; i++)  // writes after every earlier read and write of dst
      lv = std::max(lv, std::max(w_level[dst[i]], r_level[dst[i]]) + 1);
    for (uint32_t s : src) r_level[s] = std::max(r_level[s], lv);
    for (uint32_t i = 0; i < n_dst; i++) w_level[dst[i]] = lv;
    if (in.op >= 0x60 && in.op <= 0x65) n_asserts++;
    n_accesses += src.size() + n_dst;
    prog.push_back(in);
    level.push_back(lv);
    BGPU_ARG(prog.size() < 0xffffffffull, "program too large");
  }
  uint32_t n_levels = 0;
  for (uint32_t lv : level) n_levels = std::max(n_levels, lv);
  // stable counting sort by level
  std::vector<uint64_t> start(n_levels + 2, 0);
  for (uint32_t lv : level) start[lv]++;
  for (uint32_t k = 1; k <= n_levels + 1; k++) start[k] += start[k - 1];
  // start[k] = number of instructions with level <= k; level k (1-based) = [start[k-1], start[k])
  std::vector<EfInsn> sorted(prog.size());
  std::vector<uint32_t> index(prog.size());
  std::vector<uint64_t> fill(start.begin(), start.end());
  for (size_t i = 0; i < prog.size(); i++) {
    const uint64_t at = fill[level[i] - 1]++;
    sorted[at] = prog[i];
    index[at] = (uint32_t)i;
  }
  binius_eval_form* ef = new binius_eval_form();
  ef->n_values = n_values;
  ef->n_insn = prog.size();
  ef->n_asserts = n_asserts;
  ef->n_accesses = n_accesses;
  ef->level_start.assign(start.begin(), start.begin() + n_levels + 1);
  for (uint32_t k = 0; k < n_levels; k++)
    ef->max_width = std::max<uint64_t>(ef->max_width, start[k + 1] - start[k]);
  cudaGetDevice(&ef->device);
  const size_t m = prog.size() ? prog.size() : 1, ms = side.size() ? side.size() : 1;
  cudaError_t e;
  if ((e = cudaMalloc(&ef->d_level_start, 8 * ef->level_start.size())) != cudaSuccess ||
      (e = cudaMemcpy(ef->d_level_start, ef->level_start.data(), 8 * ef->level_start.size(),
                      cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMalloc(&ef->d_insn, sizeof(EfInsn) * m)) != cudaSuccess ||
      (e = cudaMalloc(&ef->d_prog_index, 4 * m)) != cudaSuccess ||
      (e = cudaMalloc(&ef->d_side, 4 * ms)) != cudaSuccess ||
      (prog.size() &&
       (e = cudaMemcpy(ef->d_insn, sorted.data(), sizeof(EfInsn) * prog.size(),
                       cudaMemcpyHostToDevice)) != cudaSuccess) ||
      (prog.size() && (e = cudaMemcpy(ef->d_prog_index, index.data(), 4 * prog.size(),
                                      cudaMemcpyHostToDevice)) != cudaSuccess) ||
      (side.size() && (e = cudaMemcpy(ef->d_side, side.data(), 4 * side.size(),
                                      cudaMemcpyHostToDevice)) != cudaSuccess)) {
    binius_eval_form_destroy(ef);
    return cuda_error(e, "eval form upload");
  }
  *out = ef;
  return clear_error();
}

// out5: instructions, levels, widest level, assertions, register accesses (sources + destinations).
int binius_eval_form_info(const binius_eval_form* ef, uint64_t* out5) {
  BGPU_ARG(ef != nullptr && out5 != nullptr, "NULL argument");
  out5[0] = ef->n_insn;
  out5[1] = ef->level_start.empty() ? 0 : ef->level_start.size() - 1;
  out5[2] = ef->max_width;
  out5[3] = ef->n_asserts;
  out5[4] = ef->n_accesses;
  return clear_error();
}

int binius_eval_form_evaluate(const binius_eval_form* ef, void* d_values, uint32_t batch,
                              uint32_t* d_fail_count, uint64_t* d_first_fail, void* stream) {
  BGPU_ARG(ef != nullptr && d_values != nullptr && d_fail_count != nullptr &&
               d_first_fail != nullptr, "NULL argument");
  BGPU_ARG(batch >= 1, "batch must be positive");
  cudaStream_t s = as_stream(stream);
  unsigned long long* first = reinterpret_cast<unsigned long long*>(d_first_fail);
  init_fail_kernel<<<(batch + 255) / 256 < 1024 ? (batch + 255) / 256 : 1024, 256, 0, s>>>(
      d_fail_count, first, batch);
  BGPU_LAUNCH_CHECK("init_fail_kernel");
  count_launch();
  uint64_t* v = static_cast<uint64_t*>(d_values);
  const bool pow2 = (batch & (batch - 1)) == 0;
  uint32_t log_batch = 0;
  while ((1u << log_batch) < batch) log_batch++;
  const size_t n_levels = ef->level_start.empty() ? 0 : ef->level_start.size() - 1;
  // Runs of narrow levels (at most kSegWidth instructions) go to the segment kernel; wider
  // levels get a launch each.
  // up to 32 instances: a warp each (on separate SMs); more: CTAs of 64 instances
  const bool seg_warp = batch <= 32;
  const uint32_t seg_grid = seg_warp ? batch : (batch + kSegInstances - 1) / kSegInstances;
  size_t k = 0;
  while (k < n_levels) {
    const uint64_t width = ef->level_start[k + 1] - ef->level_start[k];
    if (width <= kSegWidth) {
      size_t k1 = k + 1;
      while (k1 < n_levels && ef->level_start[k1 + 1] - ef->level_start[k1] <= kSegWidth) k1++;
      if (seg_warp)
        eval_segment_kernel<true><<<seg_grid, 32, 0, s>>>(
            ef->d_insn, ef->d_prog_index, ef->d_side, ef->d_level_start, (uint32_t)k,
            (uint32_t)k1, batch, v, d_fail_count, first);
      else
        eval_segment_kernel<false><<<seg_grid, kSegThreads, 0, s>>>(
            ef->d_insn, ef->d_prog_index, ef->d_side, ef->d_level_start, (uint32_t)k,
            (uint32_t)k1, batch, v, d_fail_count, first);
      BGPU_LAUNCH_CHECK("eval_segment_kernel");
      count_launch();
      k = k1;
      continue;
    }
    const uint64_t lo = ef->level_start[k], n = width;
    const uint64_t threads = n * batch, blocks = (threads + 255) / 256;
    const unsigned grid = (unsigned)std::min<uint64_t>(blocks, 148ull * 64);
    if (pow2)
      eval_level_kernel<true><<<grid, 256, 0, s>>>(ef->d_insn, ef->d_prog_index, ef->d_side, lo,
                                                    n, batch, log_batch, v, d_fail_count, first);
    else
      eval_level_kernel<false><<<grid, 256, 0, s>>>(ef->d_insn, ef->d_prog_index, ef->d_side, lo,
                                                     n, batch, log_batch, v, d_fail_count, first);
    BGPU_LAUNCH_CHECK("eval_level_kernel");
    count_launch();
    k++;
  }
  return clear_error();
}

int binius_eval_form_destroy(binius_eval_form* ef) {
  if (!ef) return BINIUS_OK;
  cudaFree(ef->d_insn);
  cudaFree(ef->d_prog_index);
  cudaFree(ef->d_side);
  cudaFree(ef->d_level_start);
  delete ef;
  return BINIUS_OK;
}

int binius_values_transpose(const void* d_src, uint64_t rows, uint64_t cols, void* d_dst,
                            void* stream) {
  BGPU_ARG(d_src != nullptr && d_dst != nullptr, "NULL argument");
  if (rows == 0 || cols == 0) return clear_error();
  const uint64_t gx = (cols + 31) / 32, gy = (rows + 31) / 32;
  BGPU_ARG(gx * gy <= 0x7fffffffull, "matrix too large for one launch");
  transpose_words_kernel<<<(unsigned)(gx * gy), dim3(32, 8), 0, as_stream(stream)>>>(
      static_cast<const uint64_t*>(d_src), rows, cols, gx, static_cast<uint64_t*>(d_dst));
  BGPU_LAUNCH_CHECK("transpose_words_kernel");
  count_launch();
  return clear_error();
}

}  // extern "C"
