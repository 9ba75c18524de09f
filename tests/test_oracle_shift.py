"""Pins the oracle's shift reduction.

* Claim relation: the phase-1 sumcheck starts from sum_v <g_v, h_v> (prover/prover/src/protocols/
  shift/phase_1.rs:86-93); the verifier starts from sum over operators of lambda^(i+1) eval_i
  (verifier/verifier/src/protocols/shift/verify.rs:74-76, 167-170).  They agree only when the
  key-weighted witness bits (g) and the shift-encoding h parts (monster.rs:34-104) are right.
* Round trip: the proof verifies under the restated verifier, whose final check evaluates the
  monster multilinear term by term from the operands (verify.rs:251-306).
* Output claim: the witness evaluation equals the 1-bit multilinear extension of the witness at
  r_j ++ r_y (phase_2.rs:140-148), which is the claim handed to the PCS.
* The operator claims come from the oracle AND reduction (AND) and from direct oblong evaluations
  (MUL); the oblong helper is itself pinned against the AND reduction's output claims.
"""
import numpy as np
import pytest

import oracle as orc
from binius64_b200 import constraint_system as csm


def _setup(log_words, n_and, n_mul, seed):
    circ = csm.synthetic_circuit(log_words, n_and, n_mul, seed=seed)
    cs = circ.cs.prepared()
    words = circ.witness
    and_vals = csm.eval_operands_csr(words, cs.and_csr)
    mul_vals = csm.eval_operands_csr(words, cs.mul_csr)
    a, b, c = (np.ascontiguousarray(and_vals[:, i]) for i in range(3))
    _, meta, r_x = orc.and_reduction_prove(a, b, c)
    z = meta[3]
    and_data = (meta[:3], z, r_x)
    rng = np.random.default_rng(seed + 1)
    log_mul = (mul_vals.shape[0] - 1).bit_length()
    r_x_mul = orc.random_elems(rng, log_mul)
    # CSR slots (a, b, hi, lo) -> operand order (a, b, lo, hi)
    mul_evals = np.stack([orc.oblong_eval(np.ascontiguousarray(mul_vals[:, i]), z, r_x_mul)
                          for i in (0, 1, 3, 2)])
    mul_data = (mul_evals, z, r_x_mul)
    return cs, words, (a, b, c), and_data, mul_data


def _mle_1b(words, point):
    return orc.eval_1b_mle(np.ascontiguousarray(words).view(np.uint64).reshape(-1, 2), point)


def test_oblong_helper_matches_and_reduction():
    cs, words, (a, b, c), and_data, _ = _setup(9, 100, 2, seed=3)
    evals, z, r_x = and_data
    for col, ev in zip((a, b, c), evals):
        assert np.array_equal(orc.oblong_eval(col, z, r_x), ev)


@pytest.mark.parametrize("log_words,log_public,n_and,n_mul,seed", [
    (10, 1, 200, 3, 0),
    (10, 4, 300, 1, 1),
    (9, 8, 120, 5, 2),
    (8, 8, 60, 2, 3),     # public segment covers the whole witness: later rounds only
    (11, 3, 900, 17, 4),
])
def test_shift_round_trip(log_words, log_public, n_and, n_mul, seed):
    cs, words, _, and_data, mul_data = _setup(log_words, n_and, n_mul, seed)
    proof, point, out3 = orc.shift_prove(words, log_public, cs.and_csr, cs.mul_csr, and_data,
                                         mul_data)
    witness_eval, initial_sum, claim = out3
    assert np.array_equal(initial_sum, claim)
    # round messages: 12 + log_words rounds of two elements, then the witness evaluation
    assert len(proof) == 16 * (2 * (12 + log_words) + 1)
    rc, ev, vpoint = orc.shift_verify(words[: 1 << log_public], log_words, log_public, cs.and_csr,
                                      cs.mul_csr, and_data, mul_data, proof)
    assert rc == 0
    assert np.array_equal(ev, witness_eval)
    assert np.array_equal(vpoint, point)
    assert np.array_equal(_mle_1b(words, point), witness_eval)


def test_shift_rejects_tampering():
    cs, words, _, and_data, mul_data = _setup(9, 100, 2, seed=5)
    proof, _, _ = orc.shift_prove(words, 2, cs.and_csr, cs.mul_csr, and_data, mul_data)
    args = (words[:4], 9, 2, cs.and_csr, cs.mul_csr)
    assert orc.shift_verify(*args, and_data, mul_data, proof)[0] == 0
    for pos in (0, 16 * 5 + 3, 16 * 24, len(proof) - 1):
        bad = bytearray(proof)
        bad[pos] ^= 1
        assert orc.shift_verify(*args, and_data, mul_data, bytes(bad))[0] != 0
    # a wrong operator claim
    evals, z, r_x = and_data
    bad_evals = evals.copy()
    bad_evals[1, 0] ^= 1
    assert orc.shift_verify(*args, (bad_evals, z, r_x), mul_data, proof)[0] != 0
    # wrong public input
    pub = words[:4].copy()
    pub[1] ^= np.uint64(1)
    assert orc.shift_verify(pub, *args[1:], and_data, mul_data, proof)[0] != 0
    # truncated proof
    assert orc.shift_verify(*args, and_data, mul_data, proof[:-16])[0] != 0


def test_shift_claims_bind_the_witness():
    cs, words, _, and_data, mul_data = _setup(9, 100, 2, seed=6)
    # a word that some AND operand reads unshifted
    plain = (cs.and_csr.variant == 0) & (cs.and_csr.amount == 0)
    w = int(cs.and_csr.value_index[plain][0])
    bad = words.copy()
    bad[w] ^= np.uint64(1 << 17)
    _, _, out3 = orc.shift_prove(bad, 2, cs.and_csr, cs.mul_csr, and_data, mul_data)
    assert not np.array_equal(out3[1], out3[2])
