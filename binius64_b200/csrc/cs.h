// Constraint-system handle shared by the reduction drivers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/binius_gpu.h"

namespace bgpu {

struct HostOperands {
  uint32_t k = 0;
  std::vector<uint32_t> offsets;  // n_constraints * k + 1
  std::vector<uint2> terms;       // (value index, variant << 8 | amount)
};

struct DevOperands {
  uint32_t k = 0;
  uint32_t n_constraints = 0;
  uint64_t n_terms = 0;
  uint32_t* offsets = nullptr;
  uint2* terms = nullptr;
};

// Operand terms of both operations in the order the shift reduction consumes them: sorted by
// key = (variant * 64 + amount) * 8 + class, class 0..2 the AND operands (a, b, c) and 3..6 the
// MUL operands in KeyCollection order (a, b, lo, hi).  One entry per term; the reference's
// KeyCollection (prover/prover/src/protocols/shift/key_collection.rs:246-312) groups the same
// terms by word and id, and every quantity the reduction takes from it is a sum over terms.
struct ShiftTerms {
  uint64_t n = 0;
  uint32_t* vi = nullptr;   // value index
  uint32_t* c = nullptr;    // constraint index within its operation
  uint16_t* key = nullptr;
  // the same terms grouped by word: word w's terms are [w_off[w], w_off[w + 1]) of w_c / w_key;
  // w_chunk[j] is the word that holds term j * kMonsterChunk of that order
  uint32_t n_words = 0;
  uint32_t* w_off = nullptr;
  uint32_t* w_c = nullptr;
  uint16_t* w_key = nullptr;
  uint32_t* w_chunk = nullptr;
};
// Frees the device arrays of a term table.
void free_shift_terms(ShiftTerms& t);
// Terms one thread of the monster multilinear takes, consecutive in word order.
constexpr uint32_t kMonsterChunk = 8;
constexpr uint32_t kShiftKeys = 512 * 8;
constexpr uint32_t kShiftClasses = 7;

}  // namespace bgpu
struct binius_cs;
namespace bgpu {
// Parses and validates a v2 constraint system into cs's host fields and pads its operand lists
// (no device state).
int parse_cs(const void* h_bytes, size_t len, binius_cs& cs);

// Uploads a term table (vi, c, key each of n entries, sorted by key) to the current device and
// replaces `out`'s, freeing the old one; on failure `out` is unchanged.
int upload_shift_terms(const std::vector<uint32_t>& vi, const std::vector<uint32_t>& c,
                       const std::vector<uint16_t>& key, uint64_t n, uint32_t n_words,
                       ShiftTerms& out);

// d_out[slot * n_constraints + i] = eval_operand of constraint i's operand `slot`.
int eval_operands(const DevOperands& ops, const uint64_t* d_witness, uint64_t* d_out,
                  cudaStream_t s);

}  // namespace bgpu

struct binius_cs {
  int device = 0;
  uint32_t n_const = 0, n_inout = 0, n_witness = 0, n_internal = 0;
  uint32_t offset_inout = 0, offset_witness = 0, committed_total_len = 0, n_scratch = 0;
  uint32_t n_and_real = 0, n_mul_real = 0;
  std::vector<uint64_t> constants;
  bgpu::HostOperands h_and, h_mul;  // padded (validate_and_prepare)
  bgpu::DevOperands and_ops, mul_ops;
  bgpu::ShiftTerms shift_terms;
};
