"""Pins the oracle's operand evaluation and AND reduction.

* Shift variants: verifier/core/src/word.rs:140-245 semantics restated in Python.
* Univariate round: sumcheck_round_messages.rs:186-274 (test_first_round_message_matches_next_
  round_sum_claim): the 64-point extension message, extended by zeros on the base domain and
  evaluated at a challenge z, equals sum_i (a_i b_i - c_i) eq(point)_i of the words folded at z.
* Round trip: and_reduction/prover.rs:314-402 (test_transcript_prover_verifies) with the verifier
  restated from verifier/verifier/src/and_reduction/verifier.rs, plus the reduction's output claims
  equal the multilinear evaluations of the folded columns at the output point.
"""
import numpy as np
import pytest

import gf_py
import oracle as orc

M64 = (1 << 64) - 1


def py_shift(w, variant, n):
    lo, hi = w & 0xFFFFFFFF, w >> 32

    def s32(x):
        return x - (1 << 32) if x >> 31 else x

    if variant == 0:
        return (w << n) & M64
    if variant == 1:
        return w >> n
    if variant == 2:
        return ((w - (1 << 64) if w >> 63 else w) >> n) & M64
    if variant == 3:
        return ((w >> n) | (w << (64 - n))) & M64 if n else w
    if variant == 4:
        return (((hi << n) & 0xFFFFFFFF) << 32) | ((lo << n) & 0xFFFFFFFF)
    if variant == 5:
        return ((hi >> n) << 32) | (lo >> n)
    if variant == 6:
        return (((s32(hi) >> n) & 0xFFFFFFFF) << 32) | ((s32(lo) >> n) & 0xFFFFFFFF)
    if variant == 7:
        rot = lambda x: ((x >> n) | (x << (32 - n))) & 0xFFFFFFFF if n else x  # noqa: E731
        return (rot(hi) << 32) | rot(lo)


def test_shift_variants():
    rng = np.random.default_rng(0)
    for _ in range(300):
        w = int(rng.integers(0, M64, dtype=np.uint64, endpoint=True))
        v = int(rng.integers(0, 8))
        n = int(rng.integers(0, 32 if v >= 4 else 64))
        assert orc.shifted_word(w, v, n) == py_shift(w, v, n), (hex(w), v, n)


def _words(rng, n):
    return rng.integers(0, np.iinfo(np.uint64).max, size=n, dtype=np.uint64, endpoint=True)


def _phi(b):
    return orc.aes_to_ghash_table()[b]


def _lagrange128(z, dim):
    table = orc.aes_to_ghash_table()
    pts = [table[t] for t in range(1 << dim)]
    out = []
    for t in range(1 << dim):
        num, den = 1, 1
        for s in range(1 << dim):
            if s != t:
                num = gf_py.mul(num, z ^ pts[s])
                den = gf_py.mul(den, pts[t] ^ pts[s])
        out.append(gf_py.mul(num, gf_py.inv(den)))
    return out


@pytest.mark.parametrize("log_n", [3, 4, 7])
def test_first_round_message_matches_folded_sum_claim(log_n):
    rng = np.random.default_rng(log_n)
    a, b = _words(rng, 1 << log_n), _words(rng, 1 << log_n)
    c = a & b
    big = orc.random_elems(rng, log_n - 3)
    msg = orc.and_univariate_round(a, b, c, big)
    z = orc.random_elems(rng, 1)[0]
    lag = _lagrange128(orc.to_int(z), 7)
    expected = 0
    for k in range(64):
        expected ^= gf_py.mul(orc.to_int(msg[k]), lag[64 + k])
    fa, fb, fc = (orc.and_fold_words(x, z) for x in (a, b, c))
    point = orc.from_ints([_phi(2), _phi(4), _phi(16)] + [orc.to_int(x) for x in big])
    eq = orc.eq_ind_partial_eval(point)
    comp = orc.gf_mul_vec(fa, fb) ^ fc
    actual = np.bitwise_xor.reduce(orc.gf_mul_vec(comp, eq), axis=0)
    assert orc.to_int(actual) == expected


def test_fold_words_is_lagrange_combination():
    rng = np.random.default_rng(9)
    w = _words(rng, 4)
    z = orc.random_elems(rng, 1)[0]
    lag = _lagrange128(orc.to_int(z), 6)
    out = orc.and_fold_words(w, z)
    for i in range(4):
        acc = 0
        for t in range(64):
            if (int(w[i]) >> t) & 1:
                acc ^= lag[t]
        assert orc.to_int(out[i]) == acc


@pytest.mark.parametrize("log_n", [3, 5, 10])
def test_and_reduction_round_trip(log_n):
    rng = np.random.default_rng(100 + log_n)
    a, b = _words(rng, 1 << log_n), _words(rng, 1 << log_n)
    c = a & b
    proof, meta, point = orc.and_reduction_prove(a, b, c)
    rc, vmeta, vpoint = orc.and_reduction_verify(log_n, proof)
    assert rc == 0
    assert np.array_equal(meta, vmeta) and np.array_equal(point, vpoint)
    z = meta[3]
    for col, ev in ((a, meta[0]), (b, meta[1]), (c, meta[2])):
        folded = orc.and_fold_words(col, z)
        assert np.array_equal(orc.mle_eval(folded, point), ev)


def test_and_reduction_rejects_unsatisfied_constraint():
    rng = np.random.default_rng(7)
    log_n = 6
    a, b = _words(rng, 1 << log_n), _words(rng, 1 << log_n)
    c = a & b
    c[5] ^= np.uint64(1 << 17)
    proof, _, _ = orc.and_reduction_prove(a, b, c)
    rc, _, _ = orc.and_reduction_verify(log_n, proof)
    assert rc != 0
