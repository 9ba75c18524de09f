"""Witness evaluation (verifier/frontend/src/compiler/eval_form): the oracle's interpreter
(Interpreter::run restated) checked opcode by opcode against Word's arithmetic written
independently here with Python integers (verifier/core/src/word.rs), on the value tables of the
reference's own interpreter tests (test_assert_eq_cond, test_select_msb_behavior), on programs
that recompute a synthetic circuit's whole witness, and the device decoder's rejections (host
code, no GPU needed)."""
import ctypes

import numpy as np
import pytest

import oracle as orc
from binius64_b200 import constraint_system as csm
from binius64_b200 import eval_form as ef
from binius64_b200._ffi import ArgumentError, check, lib

M64 = (1 << 64) - 1
MSB = 1 << 63


def run(bb, values):
    rc, out, nf, fe = orc.eval_form_run(bb.finalize(), np.array(values, dtype=np.uint64))
    assert rc == 0
    return [int(x) for x in out], nf, fe


def signed(x):
    return x - (1 << 64) if x >> 63 else x


def rotr(x, n, bits):
    n %= bits
    m = (1 << bits) - 1
    x &= m
    return ((x >> n) | (x << (bits - n))) & m


@pytest.mark.parametrize("seed", range(6))
def test_opcodes_against_word_arithmetic(seed):
    rng = np.random.default_rng(seed)
    specials = [0, 1, M64, MSB, MSB - 1, 0xFFFFFFFF, 1 << 32]
    vals = [int(v) for v in rng.integers(0, 2**63, size=4, dtype=np.uint64) * 2 + 1] + specials
    for x in vals:
        for y in vals[::2]:
            for cin in (0, MSB | 5):
                c = cin >> 63
                bb = ef.BytecodeBuilder()
                bb.band(3, 0, 1); bb.bor(4, 0, 1); bb.bxor(5, 0, 1); bb.fax(6, 0, 1, 2)
                bb.iadd_cout(7, 8, 0, 1); bb.iadd_cin_cout(9, 10, 0, 1, 2)
                bb.isub_bin_bout(11, 12, 0, 1, 2); bb.imul(13, 14, 0, 1); bb.smul(15, 16, 0, 1)
                bb.iadd_cout32(17, 18, 0, 1); bb.select(19, 2, 0, 1); bb.bxor_multi(20, [0, 1, 2, 0])
                v, nf, _ = run(bb, [x, y, cin] + [0] * 18)
                s = (x + y + c) & M64
                d = (x - y - c) & M64
                p = x * y
                sp = (signed(x) * signed(y)) & ((1 << 128) - 1)
                f32 = (x + y) & M64
                assert v[3:7] == [x & y, x | y, x ^ y, (x & y) ^ cin]
                assert v[7:9] == [(x + y) & M64, (x & y) | ((x ^ y) & ~((x + y) & M64) & M64)]
                assert v[9:11] == [s, (x & y) | ((x ^ y) & ~s & M64)]
                assert v[11:13] == [d, (~x & M64 & y) | (~(x ^ y) & M64 & d)]
                assert v[13:17] == [p >> 64, p & M64, sp >> 64, sp & M64]
                assert v[17:19] == [f32 & 0xFFFFFFFF, (x & y) | ((x ^ y) & ~f32 & M64)]
                assert v[19] == (x if cin >> 63 else y) and v[20] == y ^ cin
    for x in vals:
        for n in (0, 1, 7, 31, 32, 33, 63):
            bb = ef.BytecodeBuilder()
            bb.sll(1, 0, n); bb.slr(2, 0, n); bb.sar(3, 0, n); bb.shr32(4, 0, n)
            bb.rotr(5, 0, n); bb.rotr32(6, 0, n); bb.mask_low(7, 0, n); bb.mask_high(8, 0, n)
            bb.rotr(9, 0, n + 64); bb.rotr32(10, 0, n + 32); bb.mask_low(11, 0, 64 + n)
            v, _, _ = run(bb, [x] + [0] * 11)
            assert v[1:5] == [(x << n) & M64, x >> n, (signed(x) >> n) & M64, (x >> n) & 0xFFFFFFFF]
            assert v[5:7] == [rotr(x, n, 64), rotr(x, n, 32)]
            # mask_high(0): the reference shifts 1 by 64, wrapped to 0 in release builds
            high = x if n == 0 else x & ~((1 << (64 - n)) - 1) & M64
            assert v[7:9] == [x & ((1 << n) - 1), high]
            assert v[9:12] == [rotr(x, n, 64), rotr(x, n, 32), x]


def test_assert_eq_cond_and_select_tables():
    """The value tables of the reference's test_assert_eq_cond / test_select_msb_behavior."""
    cases = [((MSB - 1) & M64, 42, 99, 0), (MSB, 100, 100, 0), (M64, 42, 99, 1), (0xFF, 1000, 2000, 0),
             (MSB | 1, 5, 10, 1)]
    for cond, x, y, fails in cases:
        bb = ef.BytecodeBuilder()
        bb.assert_eq_cond(0, 1, 2, error_id=7)
        _, nf, fe = run(bb, [cond, x, y])
        assert nf == fails and fe == (7 if fails else 0)
    for cond, pick in ((0xFF, 1), (MSB, 0), (MSB - 1, 1), (M64, 0)):
        bb = ef.BytecodeBuilder()
        bb.select(3, 2, 0, 1)
        v, _, _ = run(bb, [42, 99, cond, 0])
        assert v[3] == [42, 99][pick]


def test_assertions_count_and_first_id():
    bb = ef.BytecodeBuilder()
    bb.assert_zero(0, 1); bb.assert_non_zero(1, 2); bb.assert_false(2, 3); bb.assert_true(3, 4)
    bb.assert_eq(0, 4, 5)
    _, nf, fe = run(bb, [0, 5, 1, MSB, 0])
    assert (nf, fe) == (0, 0)
    _, nf, fe = run(bb, [1, 0, MSB, 1, 0])
    assert (nf, fe) == (5, 1)
    _, nf, fe = run(bb, [0, 0, MSB, MSB, 0])
    assert (nf, fe) == (2, 2)


@pytest.mark.parametrize("log_words,n_and,n_mul,seed", [(8, 60, 1, 1), (12, 1500, 17, 3)])
def test_synthetic_program_recomputes_witness(log_words, n_and, n_mul, seed):
    circ = csm.synthetic_circuit(log_words, n_and, n_mul, seed=seed)
    code, n_values = ef.synthetic_program(circ)
    v0 = ef.synthetic_inputs(circ, n_values)
    n_in = circ.cs.layout.committed_total_len - circ.cs.layout.n_internal
    assert not v0[n_in:].any()
    rc, out, nf, _ = orc.eval_form_run(code, v0)
    assert rc == 0 and nf == 0
    assert np.array_equal(out[:1 << log_words], circ.witness)
    assert csm.check_satisfied(circ.cs, out[:1 << log_words])


def _create(code: bytes, n_values: int):
    h = ctypes.c_void_p()
    check(lib().binius_eval_form_create(code, len(code), n_values, ctypes.byref(h)))
    return h


@pytest.mark.parametrize("code,n_values,msg,orc_rc", [
    (bytes([0x04]), 4, "unknown opcode", -1),
    (bytes([0x80, 0, 0, 0, 0]), 4, "hint", -2),
    (bytes([0x01]) + (9).to_bytes(4, "little") * 3, 4, "register outside", -3),
    (bytes([0x01, 0, 0]), 4, "truncated", -4),
    (bytes([0x10]) + bytes(8) + bytes([64]), 4, "shift amount", -5),
])
def test_rejections(code, n_values, msg, orc_rc):
    with pytest.raises(ArgumentError, match=msg):
        _create(code, n_values)
    assert orc.eval_form_run(code, np.zeros(n_values, np.uint64))[0] == orc_rc
