// The constraint reductions of Prover::prove (prover/prover/src/prove.rs:124-303) as host drivers
// over device data; each writes its messages into the host transcript.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "cs.h"
#include "internal.h"
#include "transcript.h"

namespace bgpu {

// AndCheckOutput (prover/prover/src/and_reduction/prover.rs): the three operand evaluations at
// (z, eval_point).
struct AndResult {
  hu128 a_eval, b_eval, c_eval, z;
  std::vector<hu128> eval_point;
};

// d_witness: committed_total_len words; writes the AND reduction's transcript messages.
int and_reduction_prove(const binius_cs* cs, const uint64_t* d_witness, Transcript& t,
                        AndResult& res, cudaStream_t s);
// The same in two steps: and_reduction_begin queues what needs no challenge (the device buffers
// and the operand evaluation), so a caller can queue it before a host round trip;
// and_reduction_finish runs the rest and releases the buffers (also on error).
struct AndPrep {
  uint64_t* words = nullptr;
  uint4 *eq_big = nullptr, *fcols = nullptr, *eq = nullptr, *dev = nullptr;
  uint32_t* d_acc = nullptr;
};
int and_reduction_begin(const binius_cs* cs, const uint64_t* d_witness, AndPrep& p,
                        cudaStream_t s);
int and_reduction_finish(const binius_cs* cs, AndPrep& p, Transcript& t, AndResult& res,
                         cudaStream_t s);
void and_prep_free(AndPrep& p, cudaStream_t s);

// IntMulOutput (verifier/verifier/src/protocols/intmul/common.rs:6-13): bit-column evaluations
// of a, b, c_lo and c_hi at eval_point.
struct IntMulResult {
  std::vector<hu128> eval_point;
  std::vector<hu128> a_evals, b_evals, c_lo_evals, c_hi_evals;
};

int intmul_reduction_prove(const binius_cs* cs, const uint64_t* d_witness, Transcript& t,
                           IntMulResult& res, cudaStream_t s);
// The same reduction for a constraint system with one MUL constraint, from its operand words
// (a, b, lo, hi): no device work.
int intmul_single_from_words(uint64_t a, uint64_t b, uint64_t lo, uint64_t hi, Transcript& t,
                             IntMulResult& res);

// OperatorData (prover/prover/src/protocols/shift/prove.rs:20-33): operand evaluations at the
// oblong point (r_zhat', r_x').  AND: (a, b, c); MUL: (a, b, lo, hi).
struct ShiftOperatorData {
  std::vector<hu128> evals;
  hu128 r_zhat = 0;
  std::vector<hu128> r_x;
};

// SumcheckOutput of shift::prove: point r_j ++ r_y and the witness evaluation there.
struct ShiftResult {
  std::vector<hu128> point;
  hu128 witness_eval = 0;
};

int shift_reduction_prove(const binius_cs* cs, const uint64_t* d_witness, Transcript& t,
                          const ShiftOperatorData& bitand_data,
                          const ShiftOperatorData& intmul_data, ShiftResult& res,
                          cudaStream_t s);

}  // namespace bgpu
