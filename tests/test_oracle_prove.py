"""Pins the oracle's whole Prover::prove against its restated Verifier::verify.

The verifier (verifier/verifier/src/verify.rs:143-282) replays the transcript through the IntMul,
AND and shift verifiers, checks the shift reduction's final evaluation against the monster
multilinear computed from the constraint system and the public input, and opens the PCS at the
shift point with the witness evaluation as the claim.  Parameters follow Verifier::setup
(verify.rs:61-108): 96-bit security, arity from estimate_optimal_arity(log_code_len, 32, 16).
"""
import numpy as np
import pytest

import oracle as orc
from binius64_b200 import constraint_system as csm


def _circuit(log_words, n_and, n_mul, seed, log_public=1):
    sc = csm.synthetic_circuit(log_words, n_and, n_mul, seed=seed, log_public=log_public)
    assert csm.check_satisfied(sc.cs, sc.witness)
    return sc, sc.cs.prepared()


def test_setup_params_match_reference_shape():
    # the 2^20-word prove: 2^19 packed elements, batch 16, arities [4, 4], 232 queries
    assert orc.prove_params(20) == (19, 4, 232, [4, 4])
    lwe, lb, nq, ar = orc.prove_params(16)
    assert (lwe, nq) == (15, 232) and lb + sum(ar) <= lwe + 1


@pytest.mark.parametrize("log_words,n_and,n_mul,log_public,seed", [
    (4, 3, 1, 1, 0),
    (8, 60, 1, 1, 1),
    (10, 300, 5, 3, 2),
    (12, 1500, 17, 2, 3),
])
def test_prove_verify_round_trip(log_words, n_and, n_mul, log_public, seed):
    sc, prep = _circuit(log_words, n_and, n_mul, seed, log_public)
    proof = orc.prove(sc.witness, log_public, prep.and_csr, prep.mul_csr)
    pub = sc.witness[: 1 << log_public]
    assert orc.verify(pub, log_words, log_public, prep.and_csr, prep.mul_csr, proof) == 0
    # deterministic
    assert orc.prove(sc.witness, log_public, prep.and_csr, prep.mul_csr) == proof


def test_proof_bytes_do_not_depend_on_host_threads():
    """The oracle splits its sums and folds over the host threads (the bench's CPU baseline uses
    every core, the GPU tests eight); every split must give the same proof bytes.  2^16 words so
    that the large eq tensor levels and the per-thread partial sums all take their threaded
    branches."""
    sc, prep = _circuit(16, 60000, 70, 11, 2)
    proofs = []
    try:
        for threads in (1, 3, 8):
            orc.set_threads(threads)
            proofs.append(orc.prove(sc.witness, 2, prep.and_csr, prep.mul_csr))
    finally:
        orc.set_threads(1)
    assert proofs[0] == proofs[1] == proofs[2]
    pub = sc.witness[:4]
    assert orc.verify(pub, 16, 2, prep.and_csr, prep.mul_csr, proofs[0]) == 0


def test_verify_rejects_tampering_and_wrong_public_input():
    sc, prep = _circuit(9, 100, 3, 4)
    proof = orc.prove(sc.witness, 1, prep.and_csr, prep.mul_csr)
    args = (9, 1, prep.and_csr, prep.mul_csr)
    pub = sc.witness[:2].copy()
    assert orc.verify(pub, *args, proof) == 0
    for pos in (3, 40, len(proof) // 3, len(proof) // 2, len(proof) - 100, len(proof) - 1):
        bad = bytearray(proof)
        bad[pos] ^= 0x10
        assert orc.verify(pub, *args, bytes(bad)) != 0, pos
    pub[1] ^= np.uint64(1)
    assert orc.verify(pub, *args, proof) != 0


def test_unsatisfied_witness_is_rejected():
    sc, prep = _circuit(9, 100, 3, 5)
    bad = sc.witness.copy()
    # an internal word written by an AND constraint: (A & B) ^ C = 0 now fails
    c_col = prep.and_csr.value_index[prep.and_csr.offsets[2]:prep.and_csr.offsets[3]]
    bad[int(c_col[0])] ^= np.uint64(1 << 9)
    assert not csm.check_satisfied(sc.cs, bad)
    proof = orc.prove(bad, 1, prep.and_csr, prep.mul_csr)
    assert orc.verify(bad[:2], 9, 1, prep.and_csr, prep.mul_csr, proof) != 0
