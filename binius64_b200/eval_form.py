"""The frontend's evaluation form: bytecode that computes every internal wire of a circuit from its
inputs (verifier/frontend/src/compiler/eval_form/{builder,interpreter}.rs), and the device
evaluator that runs it over a batch of value vectors (`EvalForm`, csrc/eval_form.cu).

`BytecodeBuilder` writes the reference's instruction encoding (builder.rs): an opcode byte, then
u32 little-endian registers (value-vector indices), u8 shift amounts, u32 counts and assertion
ids.  `synthetic_program` emits the program that recomputes a `synthetic_circuit`'s internal words
(each AND constraint's new word (A & B) ^ extra, each MUL's (hi, lo)) from its inputs, with the
frontend's register model: committed words first, then one scratch register per temporary.
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

from ._ffi import ArgumentError, check, lib

SLL, SLR, SAR, ROTR, SLL32, SRL32, SRA32, ROTR32 = range(8)


class BytecodeBuilder:
    """builder.rs: one emit_* per instruction, same byte layout."""

    def __init__(self):
        self._b = bytearray()
        self.n_eval_insn = 0

    def _op(self, code: int, *regs: int):
        self.n_eval_insn += 1
        self._b.append(code)
        for r in regs:
            self._b += struct.pack("<I", r)

    def _u8(self, v: int):
        self._b.append(v & 0xFF)

    def _u32(self, v: int):
        self._b += struct.pack("<I", v)

    def band(self, dst, a, b): self._op(0x01, dst, a, b)
    def bor(self, dst, a, b): self._op(0x02, dst, a, b)
    def bxor(self, dst, a, b): self._op(0x03, dst, a, b)
    def select(self, dst, cond, t, f): self._op(0x05, dst, cond, t, f)
    def fax(self, dst, a, b, c): self._op(0x07, dst, a, b, c)

    def bxor_multi(self, dst, srcs):
        self._op(0x06, dst)
        self._u32(len(srcs))
        for s in srcs:
            self._u32(s)

    def _shift(self, code, dst, src, n):
        self._op(code, dst, src)
        self._u8(n)

    def sll(self, dst, src, n): self._shift(0x10, dst, src, n)
    def slr(self, dst, src, n): self._shift(0x11, dst, src, n)
    def sar(self, dst, src, n): self._shift(0x12, dst, src, n)
    def iadd_cout(self, ds, dc, a, b): self._op(0x20, ds, dc, a, b)
    def iadd_cin_cout(self, ds, dc, a, b, cin): self._op(0x21, ds, dc, a, b, cin)
    def isub_bin_bout(self, dd, db, a, b, bin_): self._op(0x23, dd, db, a, b, bin_)
    def imul(self, dhi, dlo, a, b): self._op(0x30, dhi, dlo, a, b)
    def smul(self, dhi, dlo, a, b): self._op(0x31, dhi, dlo, a, b)
    def iadd_cout32(self, ds, dc, a, b): self._op(0x40, ds, dc, a, b)
    def rotr32(self, dst, src, n): self._shift(0x41, dst, src, n)
    def shr32(self, dst, src, n): self._shift(0x42, dst, src, n)
    def rotr(self, dst, src, n): self._shift(0x43, dst, src, n)
    def mask_low(self, dst, src, n): self._shift(0x50, dst, src, n)
    def mask_high(self, dst, src, n): self._shift(0x51, dst, src, n)

    def _assert(self, code, regs, error_id):
        self._op(code, *regs)
        self._u32(error_id)

    def assert_eq(self, a, b, error_id=0): self._assert(0x60, (a, b), error_id)
    def assert_eq_cond(self, c, a, b, error_id=0): self._assert(0x61, (c, a, b), error_id)
    def assert_zero(self, a, error_id=0): self._assert(0x62, (a,), error_id)
    def assert_non_zero(self, a, error_id=0): self._assert(0x63, (a,), error_id)
    def assert_false(self, a, error_id=0): self._assert(0x64, (a,), error_id)
    def assert_true(self, a, error_id=0): self._assert(0x65, (a,), error_id)

    def finalize(self) -> bytes:
        return bytes(self._b)


class _Scratch:
    def __init__(self, base: int):
        self.next = base

    def take(self) -> int:
        r = self.next
        self.next += 1
        return r


def _emit_shifted(bb: BytecodeBuilder, sc: _Scratch, word: int, variant: int, amount: int) -> int:
    """The register holding ShiftedValueIndex(word, variant, amount)'s value (shifted(),
    constraint_system.py; ShiftVariant, verifier/core/src/constraint_system.rs)."""
    if amount == 0:
        return word
    out = sc.take()
    if variant == SLL:
        bb.sll(out, word, amount)
    elif variant == SLR:
        bb.slr(out, word, amount)
    elif variant == SAR:
        bb.sar(out, word, amount)
    elif variant == ROTR:
        bb.rotr(out, word, amount)
    else:  # the 32-bit variants act on both halves; eval_form's 32-bit ops on the low half
        hi_in, lo_in = sc.take(), sc.take()
        bb.mask_high(hi_in, word, 32)          # hi << 32
        bb.mask_low(lo_in, word, 32)           # lo
        hi, lo = sc.take(), sc.take()
        if variant == SLL32:
            bb.sll(hi, hi_in, amount)           # (hi << n) << 32, truncated
            t = sc.take()
            bb.sll(t, lo_in, amount)
            bb.mask_low(lo, t, 32)
        elif variant == SRL32:
            t = sc.take()
            bb.slr(t, hi_in, amount)
            bb.mask_high(hi, t, 32)
            bb.slr(lo, lo_in, amount)
        elif variant == SRA32:
            t = sc.take()
            bb.sar(t, hi_in, amount)
            bb.mask_high(hi, t, 32)
            t2, t3 = sc.take(), sc.take()
            bb.sll(t2, word, 32)                # lo << 32: its sign at bit 63
            bb.sar(t3, t2, amount)
            bb.slr(lo, t3, 32)
        else:  # ROTR32
            t, t2 = sc.take(), sc.take()
            bb.slr(t, word, 32)
            bb.rotr32(t2, t, amount)
            bb.sll(hi, t2, 32)
            bb.rotr32(lo, word, amount)
        bb.bor(out, hi, lo)
    return out


def _emit_operand(bb, sc, terms) -> int:
    regs = [_emit_shifted(bb, sc, w, v, a) for (w, v, a) in terms]
    if len(regs) == 1:
        return regs[0]
    out = sc.take()
    bb.bxor_multi(out, regs)
    return out


def synthetic_program(circ, with_count: bool = False):
    """(bytecode, n_values) recomputing every internal word of a synthetic_circuit from its
    constants, public inputs and witness inputs; n_values = committed words + scratch.  With
    with_count, (bytecode, n_values, number of instructions)."""
    cs = circ.cs
    lay = cs.layout
    total = lay.committed_total_len
    bb, sc = BytecodeBuilder(), _Scratch(total)

    def terms(csr, g):
        lo, hi = int(csr.offsets[g]), int(csr.offsets[g + 1])
        return [(int(csr.value_index[t]), int(csr.variant[t]), int(csr.amount[t]))
                for t in range(lo, hi)]

    and_csr, mul_csr = cs.and_operands(), cs.mul_operands()
    zero = None
    for i in range(cs.n_and()):
        a, b, c = terms(and_csr, 3 * i), terms(and_csr, 3 * i + 1), terms(and_csr, 3 * i + 2)
        new_word, extra = c[0][0], c[1:]
        ra, rb = _emit_operand(bb, sc, a), _emit_operand(bb, sc, b)
        if extra:
            rc = _emit_operand(bb, sc, extra)
        else:
            if zero is None:  # a scratch register that no instruction writes stays zero
                zero = sc.take()
            rc = zero
        bb.fax(new_word, ra, rb, rc)
    for i in range(cs.n_mul()):
        a, b = terms(mul_csr, 4 * i), terms(mul_csr, 4 * i + 1)
        hi, lo = terms(mul_csr, 4 * i + 2)[0][0], terms(mul_csr, 4 * i + 3)[0][0]
        bb.imul(hi, lo, _emit_operand(bb, sc, a), _emit_operand(bb, sc, b))
    if with_count:
        return bb.finalize(), sc.next, bb.n_eval_insn
    return bb.finalize(), sc.next


def chain_program(n_ops: int, seed: int = 0, first_free: int = 8) -> tuple[bytes, int]:
    """(bytecode, n_values) of a deep program: an add-rotate-xor chain in the style of a hash's
    rounds, each instruction writing a fresh register from the last few (registers 0..7 are its
    inputs, fresh ones start at first_free, one or two per instruction), so the levels are a few
    instructions wide and ~n_ops deep."""
    rng = np.random.default_rng(seed)
    bb = BytecodeBuilder()
    live = list(range(8))
    nxt = first_free
    for _ in range(n_ops):
        a, b, c = (live[-1 - int(rng.integers(0, 4))] for _ in range(3))
        op = int(rng.integers(0, 5))
        if op == 0:
            bb.iadd_cout32(nxt, nxt + 1, a, b)
            live += [nxt, nxt + 1]
            nxt += 2
            continue
        if op == 1:
            bb.rotr32(nxt, a, int(rng.integers(1, 32)))
        elif op == 2:
            bb.bxor(nxt, a, b)
        elif op == 3:
            bb.fax(nxt, a, b, c)
        else:
            bb.iadd_cout(nxt, nxt + 1, a, b)
            live += [nxt, nxt + 1]
            nxt += 2
            continue
        live.append(nxt)
        nxt += 1
    return bb.finalize(), nxt


def synthetic_inputs(circ, n_values: int) -> np.ndarray:
    """The value vector before evaluation: constants, public and witness inputs set, internal
    words and scratch zero."""
    lay = circ.cs.layout
    v = np.zeros(n_values, dtype=np.uint64)
    n_in = lay.committed_total_len - lay.n_internal
    v[:n_in] = circ.witness[:n_in]
    return v


class EvalForm:
    """A program decoded, validated and level-scheduled on the host, evaluated on the device over
    a batch of value vectors laid out register-major (`values[reg * batch + instance]`)."""

    def __init__(self, bytecode: bytes, n_values: int):
        self._h = ctypes.c_void_p()
        check(lib().binius_eval_form_create(bytecode, len(bytecode), n_values,
                                            ctypes.byref(self._h)))
        info = (ctypes.c_uint64 * 5)()
        check(lib().binius_eval_form_info(self._h, ctypes.addressof(info)))
        self.n_values = n_values
        (self.n_insn, self.n_levels, self.max_level_width, self.n_asserts,
         self.n_accesses) = list(info)

    def evaluate(self, values, batch: int, stream=None):
        """values: device int64 tensor of n_values * batch words (register-major), updated in
        place.  Returns (failures per instance, first failure per instance: (instruction index
        << 32 | assertion id), or all ones) as device tensors."""
        import torch
        if values.numel() != self.n_values * batch:
            raise ArgumentError(1, "values: n_values * batch words")
        from . import _stream
        fails = torch.empty(batch, dtype=torch.int32, device=values.device)
        first = torch.empty(batch, dtype=torch.int64, device=values.device)
        check(lib().binius_eval_form_evaluate(self._h, values.data_ptr(), batch,
                                              fails.data_ptr(), first.data_ptr(),
                                              _stream(stream)))
        return fails, first

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().binius_eval_form_destroy(h)
            except Exception:
                pass
            self._h = None


def transpose_words(src, rows: int, cols: int, out=None, stream=None):
    """out[c * rows + r] = src[r * cols + c] for 64-bit words on the device (instance-major value
    vectors <-> the register-major batch layout)."""
    import torch
    if src.numel() != rows * cols:
        raise ArgumentError(1, "src: rows * cols words")
    from . import _stream
    if out is None:
        out = torch.empty(rows * cols, dtype=torch.int64, device=src.device)
    check(lib().binius_values_transpose(src.data_ptr(), rows, cols, out.data_ptr(),
                                        _stream(stream)))
    return out
