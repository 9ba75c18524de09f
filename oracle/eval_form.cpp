// CPU oracle (test infrastructure only): the frontend's witness evaluator, restated from
// verifier/frontend/src/compiler/eval_form/interpreter.rs (Interpreter::run and its exec_*
// handlers) with the Word arithmetic of verifier/core/src/word.rs (iadd_cin_cout :112-120,
// isub_bin_bout :129-137, shr_32 :140-145, sar :150-155, rotr_32 :158-162, rotr :165-168,
// iadd_cout_32 :96-103, imul :252-260, smul :266-278, MSB-bools :305-317).
//
// One program runs over one value vector: each instruction is an opcode byte followed by its
// operands (registers are u32 value-vector indices, shift amounts u8, counts u32, assertion ids
// u32), all little-endian.  Assertion failures are counted; the id of the first is kept.
// Differences from the reference, all on inputs it would panic on: an unknown opcode, a register
// outside the vector, a truncated instruction or a shift amount of 64 or more return an error
// code here; hint calls (0x80) return an error too (their handlers are host code outside this
// path).
#include <string.h>

#include "oracle.h"
#include "oracle_internal.h"

namespace {

struct Vm {
  const uint8_t* code;
  size_t len, pc = 0;
  uint64_t* v;
  size_t n;
  int err = 0;
  uint32_t failures = 0, first_error = 0;

  uint8_t u8() {
    if (pc + 1 > len) {
      err = -4;
      return 0;
    }
    return code[pc++];
  }
  uint32_t u32() {
    if (pc + 4 > len) {
      err = -4;
      return 0;
    }
    uint32_t x;
    memcpy(&x, code + pc, 4);
    pc += 4;
    return x;
  }
  uint32_t reg() {
    const uint32_t r = u32();
    if (!err && r >= n) err = -3;
    return r;
  }
  uint32_t shift() {
    const uint32_t s = u8();
    if (!err && s >= 64) err = -5;
    return s;
  }
  uint64_t ld(uint32_t r) { return err ? 0 : v[r]; }
  void st(uint32_t r, uint64_t x) {
    if (!err) v[r] = x;
  }
  void fail(uint32_t id) {
    if (err) return;
    if (failures == 0) first_error = id;
    failures++;
  }
};

bool msb(uint64_t x) { return (x >> 63) != 0; }

}  // namespace

extern "C" int orc_eval_form_run(const uint8_t* code, size_t len, uint64_t* values,
                                 size_t n_values, uint32_t* n_failures, uint32_t* first_error_id) {
  Vm m{code, len, 0, values, n_values};
  while (m.pc < m.len && !m.err) {
    const uint8_t op = m.u8();
    switch (op) {
      case 0x01: case 0x02: case 0x03: {  // band, bor, bxor
        const uint32_t d = m.reg(), a = m.reg(), b = m.reg();
        const uint64_t x = m.ld(a), y = m.ld(b);
        m.st(d, op == 0x01 ? (x & y) : op == 0x02 ? (x | y) : (x ^ y));
        break;
      }
      case 0x05: {  // select: t if MSB(cond) else f
        const uint32_t d = m.reg(), c = m.reg(), t = m.reg(), f = m.reg();
        m.st(d, msb(m.ld(c)) ? m.ld(t) : m.ld(f));
        break;
      }
      case 0x06: {  // bxor_multi
        const uint32_t d = m.reg(), cnt = m.u32();
        uint64_t x = 0;
        for (uint32_t i = 0; i < cnt && !m.err; i++) x ^= m.ld(m.reg());
        m.st(d, x);
        break;
      }
      case 0x07: {  // fax: (a & b) ^ c
        const uint32_t d = m.reg(), a = m.reg(), b = m.reg(), c = m.reg();
        m.st(d, (m.ld(a) & m.ld(b)) ^ m.ld(c));
        break;
      }
      case 0x10: case 0x11: case 0x12: {  // sll, slr, sar
        const uint32_t d = m.reg(), a = m.reg(), s = m.shift();
        const uint64_t x = m.ld(a);
        m.st(d, op == 0x10 ? (x << s) : op == 0x11 ? (x >> s)
                                                   : (uint64_t)((int64_t)x >> s));
        break;
      }
      case 0x20: case 0x21: case 0x23: {  // iadd_cout, iadd_cin_cout, isub_bin_bout
        const uint32_t ds = m.reg(), dc = m.reg(), a = m.reg(), b = m.reg();
        const uint64_t cin = op == 0x20 ? 0 : (m.ld(m.reg()) >> 63);
        const uint64_t x = m.ld(a), y = m.ld(b);
        if (op == 0x23) {
          const uint64_t diff = x - y - cin;
          m.st(ds, diff);
          m.st(dc, (~x & y) | (~(x ^ y) & diff));
        } else {
          const uint64_t sum = x + y + cin;
          m.st(ds, sum);
          m.st(dc, (x & y) | ((x ^ y) & ~sum));
        }
        break;
      }
      case 0x30: case 0x31: {  // imul, smul: (hi, lo)
        const uint32_t dh = m.reg(), dl = m.reg(), a = m.reg(), b = m.reg();
        const uint64_t x = m.ld(a), y = m.ld(b);
        unsigned __int128 p;
        if (op == 0x30)
          p = (unsigned __int128)x * y;
        else
          p = (unsigned __int128)((__int128)(int64_t)x * (__int128)(int64_t)y);
        m.st(dh, (uint64_t)(p >> 64));
        m.st(dl, (uint64_t)p);
        break;
      }
      case 0x40: {  // iadd_cout32
        const uint32_t ds = m.reg(), dc = m.reg(), a = m.reg(), b = m.reg();
        const uint64_t x = m.ld(a), y = m.ld(b), full = x + y;
        m.st(ds, full & 0xFFFFFFFFull);
        m.st(dc, (x & y) | ((x ^ y) & ~full));
        break;
      }
      case 0x41: {  // rotr32 of the low half
        const uint32_t d = m.reg(), a = m.reg(), s = m.u8();
        const uint32_t x = (uint32_t)m.ld(a), r = s & 31;
        m.st(d, (uint64_t)(r ? ((x >> r) | (x << (32 - r))) : x));
        break;
      }
      case 0x42: {  // shr32
        const uint32_t d = m.reg(), a = m.reg(), s = m.shift();
        m.st(d, (m.ld(a) >> s) & 0xFFFFFFFFull);
        break;
      }
      case 0x43: {  // rotr
        const uint32_t d = m.reg(), a = m.reg(), s = m.u8();
        const uint64_t x = m.ld(a);
        const uint32_t r = s & 63;
        m.st(d, r ? ((x >> r) | (x << (64 - r))) : x);
        break;
      }
      case 0x50: case 0x51: {  // mask_low, mask_high
        const uint32_t d = m.reg(), a = m.reg(), nb = m.u8();
        uint64_t mask;
        // mask_high(0) shifts 1 by 64, which the reference's release build wraps to a shift by
        // 0: the mask is all ones (its debug build panics)
        if (nb >= 64 || (op == 0x51 && nb == 0))
          mask = ~0ull;
        else if (op == 0x50)
          mask = (1ull << nb) - 1;
        else
          mask = ~((1ull << (64 - nb)) - 1);
        m.st(d, m.ld(a) & mask);
        break;
      }
      case 0x60: {  // assert_eq
        const uint32_t a = m.reg(), b = m.reg(), id = m.u32();
        if (m.ld(a) != m.ld(b)) m.fail(id);
        break;
      }
      case 0x61: {  // assert_eq_cond
        const uint32_t c = m.reg(), a = m.reg(), b = m.reg(), id = m.u32();
        if (msb(m.ld(c)) && m.ld(a) != m.ld(b)) m.fail(id);
        break;
      }
      case 0x62: case 0x63: case 0x64: case 0x65: {  // assert_zero / non_zero / false / true
        const uint32_t a = m.reg(), id = m.u32();
        const uint64_t x = m.ld(a);
        const bool bad = op == 0x62 ? x != 0 : op == 0x63 ? x == 0 : op == 0x64 ? msb(x) : !msb(x);
        if (bad) m.fail(id);
        break;
      }
      case 0x80:
        m.err = -2;
        break;
      default:
        m.err = -1;
        break;
    }
  }
  *n_failures = m.failures;
  *first_error_id = m.first_error;
  return m.err;
}
