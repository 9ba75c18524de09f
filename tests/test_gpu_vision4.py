"""Vision-4 on the device against the oracle (itself pinned on the reference's known answers):
the permutation over batches of states (known answers, zero elements entering the sbox, random
states), the Merkle commit with VisionHasherDigest leaves and VisionCompression nodes, byte for
byte over every node for leaves of 1 to 64 elements, and whole proofs whose commitments are all
Vision-4 trees (the `-c vision4` setup)."""
import json
import os

import numpy as np
import pytest

import oracle as orc
from binius64_b200 import constraint_system as csm

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402

KAT = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "vision4_kat.json")))


def test_permutation_known_answers_and_zeros():
    rc, _ = orc.vision4_constants()
    states = [[int(h, 16) for h in c["input"]] for c in KAT["permutation"]]
    states.append(list(rc[0]))                 # every element is zero at the first sbox
    states.append([rc[0][0], 5, rc[0][2], 7])  # two zeros at the first sbox
    rng = np.random.default_rng(11)
    for _ in range(300):
        states.append([int.from_bytes(rng.bytes(16), "little") for _ in range(4)])
    flat = np.concatenate([orc._int_elems(s) for s in states])
    d = bg.to_device(flat)
    bg.vision4_permute(d)
    got = orc._elems_int(bg.to_host(d))
    for i, s in enumerate(states):
        assert got[4 * i:4 * i + 4] == orc.vision4_permutation(s), f"state {i}"
    for i, c in enumerate(KAT["permutation"]):
        assert got[4 * i:4 * i + 4] == [int(h, 16) for h in c["output"]]


@pytest.mark.parametrize("log_leaves,log_batch", [
    (0, 0), (0, 4), (1, 0), (3, 1), (7, 4), (8, 2), (9, 6), (10, 4), (12, 0), (14, 4), (15, 0),
])
def test_vision4_merkle_commit_vs_oracle(log_leaves, log_batch):
    r = np.random.default_rng(700 + 8 * log_leaves + log_batch)
    elems = orc.random_elems(r, 1 << (log_leaves + log_batch))
    orc.set_threads(8)
    try:
        ref = orc.vision4_merkle_commit(elems, log_leaves, log_batch)
    finally:
        orc.set_threads(1)
    root, committed = bg.BinaryMerkleTreeProver("vision4").commit(bg.to_device(elems),
                                                                  1 << log_batch)
    got = committed.nodes.cpu().numpy()
    if not np.array_equal(got, ref):
        bad = np.nonzero((got != ref).any(axis=1))[0]
        pytest.fail(f"{len(bad)} of {len(ref)} nodes differ, first {bad[0]}")
    assert root == bytes(ref[-1])


@pytest.mark.parametrize("log_words,n_and,n_mul,seed", [(10, 300, 5, 1), (14, 6000, 200, 2),
                                                         (16, 60000, 1, 3)])
def test_prove_with_vision4_merkle_matches_oracle(log_words, n_and, n_mul, seed):
    """setup_vision4 (prover/examples/src/lib.rs:67-85): every commitment of the proof is a
    Vision-4 Merkle tree; the proof bytes equal the oracle's and its verifier accepts them."""
    sc = csm.synthetic_circuit(log_words, n_and, n_mul, seed=seed)
    prep = sc.cs.prepared()
    orc.set_threads(8)
    try:
        with orc.merkle_hash("vision4"):
            ref = orc.prove(sc.witness, 1, prep.and_csr, prep.mul_csr, 1)
            ok = orc.verify(sc.witness[:2], log_words, 1, prep.and_csr, prep.mul_csr, ref, 1)
    finally:
        orc.set_threads(1)
    assert ok == 0
    dcs = bg.DeviceConstraintSystem(sc.cs.serialize())
    w = torch.from_numpy(sc.witness.view(np.int64)).cuda()
    got = bg.Prover(dcs, 1, merkle_hash="vision4").prove(w).finalize()
    assert got == ref
    sha = bg.Prover(dcs, 1).prove(w).finalize()
    assert sha != got and len(sha) == len(got)
    # the SHA-256 verifier rejects the Vision-4 proof
    assert orc.verify(sc.witness[:2], log_words, 1, prep.and_csr, prep.mul_csr, got, 1) != 0
