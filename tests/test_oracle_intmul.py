"""Pins the oracle's integer multiplication reduction.

* prover/prover/src/protocols/intmul/tests.rs:35-105 (prove_and_verify): the output bit-column
  claims of a, b, c_lo and c_hi equal the multilinear evaluations of those columns at the output
  point, and the restated verifier (verifier/verifier/src/protocols/intmul/verify.rs) accepts the
  proof with the same outputs.
* witness.rs:309-361 (check_consistency): the b tree root (G^a)^b equals the c root
  G^c_lo (G^(2^64))^c_hi, so the two root evaluations written first are equal for true
  statements and differ for a wrong product.
"""
import numpy as np
import pytest

import oracle as orc

M64 = (1 << 64) - 1


def _statements(rng, n, zero_frac=0.0):
    a = rng.integers(1, M64, size=n, dtype=np.uint64, endpoint=True)
    b = rng.integers(1, M64, size=n, dtype=np.uint64, endpoint=True)
    if zero_frac:
        a[rng.random(n) < zero_frac] = 0
        b[rng.random(n) < zero_frac] = 0
    prod = [int(x) * int(y) for x, y in zip(a, b)]
    lo = np.array([p & M64 for p in prod], dtype=np.uint64)
    hi = np.array([p >> 64 for p in prod], dtype=np.uint64)
    return a, b, lo, hi


def _bit_mle(words, k, point):
    col = ((words >> np.uint64(k)) & np.uint64(1)).astype(np.uint64)
    el = np.zeros((len(words), 2), dtype=np.uint64)
    el[:, 0] = col
    return orc.mle_eval(el, point) if len(point) else el[0]


@pytest.mark.parametrize("log_n,zero_frac", [(0, 0.0), (1, 0.0), (3, 0.3), (5, 0.0), (7, 0.1)])
def test_intmul_round_trip(log_n, zero_frac):
    rng = np.random.default_rng(log_n)
    a, b, lo, hi = _statements(rng, 1 << log_n, zero_frac)
    proof, point, evals = orc.intmul_prove(a, b, lo, hi)
    # b and c roots agree (first two messages)
    assert proof[:16] == proof[16:32]
    for col, ev in zip((a, b, lo, hi), evals):
        for k in (0, 1, 17, 63):
            assert np.array_equal(_bit_mle(col, k, point), ev[k]), k
    rc, vpoint, vevals = orc.intmul_verify(log_n, proof)
    assert rc == 0
    assert np.array_equal(vpoint, point)
    assert np.array_equal(vevals, evals)


def test_intmul_rejects_tampering():
    rng = np.random.default_rng(9)
    a, b, lo, hi = _statements(rng, 8)
    proof, _, _ = orc.intmul_prove(a, b, lo, hi)
    for pos in (40, 16 * 20 + 5, len(proof) // 2, len(proof) - 600, len(proof) - 1):
        bad = bytearray(proof)
        bad[pos] ^= 4
        assert orc.intmul_verify(3, bytes(bad))[0] != 0, pos
    assert orc.intmul_verify(3, proof[:-16])[0] != 0


def test_intmul_wrong_product_changes_root():
    rng = np.random.default_rng(11)
    a, b, lo, hi = _statements(rng, 8)
    lo = lo.copy()
    lo[3] ^= np.uint64(1 << 40)
    proof, _, _ = orc.intmul_prove(a, b, lo, hi)
    assert proof[:16] != proof[16:32]


def test_zero_times_zero_is_consistent():
    z = np.zeros(4, dtype=np.uint64)
    proof, point, evals = orc.intmul_prove(z, z, z, z)
    assert proof[:16] == proof[16:32]
    assert orc.intmul_verify(2, proof)[0] == 0
    assert not evals.any()
