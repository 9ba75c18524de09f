"""Pins the oracle's transcript and PCS (ring switching + BaseFold + FRI).

* Transcript: the known-answer structure of
  verifier/transcript/src/fiat_shamir/hasher_challenger.rs:209-280 (test_starting_sampler,
  test_starting_observer), restated with Python's hashlib as the SHA-256.
* PCS: prove -> verify round trips mirroring prover/prover/src/pcs.rs:288-350
  (run_ring_switched_pcs_prove_and_verify: log_batch 0, arities [2, 2] or [1; n-1], 3 queries,
  R = 1, standard-basis domain) and the parameter choice of Verifier::setup, with the verifier
  restated from verifier/verifier/src/pcs.rs, protocols/basefold.rs and fri/verify.rs; tampered
  proofs and wrong claims must be rejected.
"""
import hashlib

import numpy as np
import pytest

import oracle as orc


def test_transcript_starting_sampler():
    d0 = hashlib.sha256(b"").digest()
    h = hashlib.sha256(d0)
    t = orc.Transcript()
    assert t.sample(8) == d0[:8]
    assert t.sample(24) == d0[8:]
    t.observe(bytes([0x48, 0x55]))
    h.update(bytes([32, 0, 0, 0, 0, 0, 0, 0]))
    h.update(bytes([0x48, 0x55]))
    assert t.sample(2) == h.digest()[:2]


def test_transcript_starting_observer():
    d0 = hashlib.sha256(b"").digest()
    rng = np.random.default_rng(0)
    observable = rng.integers(0, 256, 1019, dtype=np.uint8).tobytes()
    t = orc.Transcript()
    for a, b in [(0, 39), (39, 300), (300, 987), (987, 1019)]:
        t.observe(observable[a:b])
    h = hashlib.sha256(d0 + bytes(8) + observable)
    first = h.digest()
    assert t.sample(7) == first[:7]
    observable2 = rng.integers(0, 256, 1019, dtype=np.uint8).tobytes()
    t.observe(observable2[:128])
    h = hashlib.sha256(first + bytes([7, 0, 0, 0, 0, 0, 0, 0]) + observable2[:128])
    second = h.digest()
    assert t.sample(32) == second
    t.observe(observable2[128:])
    h = hashlib.sha256(second + bytes([32, 0, 0, 0, 0, 0, 0, 0]) + observable2[128:])
    assert t.sample(7) == h.digest()[:7]


def test_transcript_long_sample_chains_digests():
    d0 = hashlib.sha256(b"").digest()
    t = orc.Transcript()
    out = t.sample(100)
    d1 = hashlib.sha256(d0).digest()
    d2 = hashlib.sha256(d1).digest()
    d3 = hashlib.sha256(d2).digest()
    assert out == (d0 + d1 + d2 + d3)[:100]


def _random_point(rng, n):
    return orc.random_elems(rng, n)


def _pcs_case(log_msg, log_batch, log_inv_rate, arities, n_queries, seed, basis_log_batch=None):
    rng = np.random.default_rng(seed)
    rs_log_len = log_msg - log_batch + log_inv_rate
    # The RS domain: row log_batch of the standard domain of dim rs_log_len + log_batch, i.e. its
    # twiddle table truncated (the identity is pinned in test_oracle_pins).
    tw = orc.domain_twiddles(rs_log_len + log_batch)[: (1 << rs_log_len) - 1]
    witness = orc.random_elems(rng, 1 << log_msg)
    point = _random_point(rng, log_msg + 7)
    claim = orc.eval_1b_mle(witness, point)
    proof = orc.pcs_prove(tw, witness, log_batch, log_inv_rate, arities, n_queries, point)
    return tw, witness, point, claim, proof


PCS_CASES = [
    # (log_msg, log_batch, log_inv_rate, arities, n_queries)
    (4, 0, 1, [2, 2], 3),       # pcs.rs test shape, PackedBinaryGhash4x128b
    (6, 0, 1, [1] * 5, 3),      # pcs.rs test shape, arities [1; n-1]
    (8, 2, 1, [2, 2], 5),
    (10, 4, 1, [4], 20),        # Verifier::setup shape at small size (arity 4, batch 16)
    (12, 4, 1, [4, 2], 232),    # full query count
    (9, 3, 2, [3], 30),         # R = 2
]


@pytest.mark.parametrize("case", PCS_CASES)
def test_pcs_round_trip(case):
    log_msg, log_batch, R, arities, nq = case
    tw, w, pt, claim, proof = _pcs_case(log_msg, log_batch, R, arities, nq, seed=log_msg)
    assert orc.pcs_verify(tw, log_msg, log_batch, R, arities, nq, pt, claim, proof) == 0


def test_pcs_rejects_wrong_claim_and_tampering():
    log_msg, log_batch, R, arities, nq = 10, 4, 1, [4], 20
    tw, w, pt, claim, proof = _pcs_case(log_msg, log_batch, R, arities, nq, seed=3)
    bad = claim.copy()
    bad[0] ^= np.uint64(1)
    assert orc.pcs_verify(tw, log_msg, log_batch, R, arities, nq, pt, bad, proof) == 1
    rng = np.random.default_rng(11)
    positions = sorted(set(int(x) for x in rng.integers(32, len(proof), 24))) + [len(proof) - 1]
    for pos in positions:
        tampered = bytearray(proof)
        tampered[pos] ^= 0x5A
        assert orc.pcs_verify(tw, log_msg, log_batch, R, arities, nq, pt, claim,
                              bytes(tampered)) != 0, pos
    assert orc.pcs_verify(tw, log_msg, log_batch, R, arities, nq, pt, claim, proof + b"\0") == 9
    assert orc.pcs_verify(tw, log_msg, log_batch, R, arities, nq, pt, claim, proof[:-1]) == 2
