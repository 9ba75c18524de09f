"""The GPU prove entry against the oracle's Prover::prove: byte-identical proofs, accepted by the
restated Verifier::verify."""
import numpy as np
import pytest

import oracle as orc
from binius64_b200 import constraint_system as csm

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402


def _prove_both(log_words, n_and, n_mul, seed, log_public=1, log_inv_rate=1):
    sc = csm.synthetic_circuit(log_words, n_and, n_mul, seed=seed, log_public=log_public)
    prep = sc.cs.prepared()
    orc.set_threads(8)
    try:
        ref = orc.prove(sc.witness, log_public, prep.and_csr, prep.mul_csr, log_inv_rate)
    finally:
        orc.set_threads(1)
    dcs = bg.DeviceConstraintSystem(sc.cs.serialize())
    prover = bg.Prover(dcs, log_inv_rate)
    w = torch.from_numpy(sc.witness.view(np.int64)).cuda()
    got = prover.prove(w).finalize()
    return sc, prep, ref, got, prover


def _assert_same(ref, got):
    assert len(got) == len(ref)
    if got != ref:
        first = next(i for i in range(len(ref)) if got[i] != ref[i])
        pytest.fail(f"proof bytes differ first at offset {first} of {len(ref)}")


@pytest.mark.parametrize("log_words,n_and,n_mul,log_public,log_inv_rate", [
    (4, 3, 1, 1, 1),
    (8, 60, 1, 1, 1),
    (10, 300, 5, 3, 1),
    (12, 1500, 17, 2, 2),
    (16, 60000, 1, 1, 1),
    (17, 100000, 300, 4, 1),
])
def test_prove_matches_oracle(log_words, n_and, n_mul, log_public, log_inv_rate):
    sc, prep, ref, got, prover = _prove_both(log_words, n_and, n_mul, log_words, log_public,
                                             log_inv_rate)
    _assert_same(ref, got)
    assert orc.verify(sc.witness[: 1 << log_public], log_words, log_public, prep.and_csr,
                      prep.mul_csr, got, log_inv_rate) == 0


def test_prove_2_20_words():
    """The 2^20-word shape: about 2^20 AND constraints, one MUL, FRI arities [4, 4]."""
    sc, prep, ref, got, prover = _prove_both(20, (1 << 20) - (1 << 16), 1, 20)
    assert (prover.log_witness_elems, prover.log_batch, prover.fold_arities) == (19, 4, [4, 4])
    _assert_same(ref, got)
    assert orc.verify(sc.witness[:2], 20, 1, prep.and_csr, prep.mul_csr, got) == 0


def test_prover_is_reusable_and_deterministic():
    sc = csm.synthetic_circuit(10, 200, 2, seed=7)
    dcs = bg.DeviceConstraintSystem(sc.cs.serialize())
    prover = bg.Prover(dcs)
    w = torch.from_numpy(sc.witness.view(np.int64)).cuda()
    a = prover.prove(w).finalize()
    b = prover.prove(w).finalize()
    assert a == b
    with pytest.raises(bg.ArgumentError):
        prover.prove(w[:-1])


@pytest.mark.parametrize("with_key_collection", [False, True])
def test_setup_and_prove_from_host_buffers(with_key_collection):
    """binius_setup (ConstraintSystem bytes -> prover) and binius_prove (host witness words ->
    proof bytes): the same bytes as the device-witness path and the oracle."""
    sc = csm.synthetic_circuit(12, 1800, 9, seed=77, log_public=2)
    prep = sc.cs.prepared()
    ref = orc.prove(sc.witness, 2, prep.and_csr, prep.mul_csr, 1)
    cs_bytes = sc.cs.serialize()
    kc = bg.key_collection_from_cs_bytes(cs_bytes) if with_key_collection else None
    p = bg.setup(cs_bytes, 1, key_collection=kc)
    assert p.cs.committed_total_len == len(sc.witness)
    assert p.prove_host(sc.witness) == ref
    assert p.prove_host(sc.witness) == ref  # the prover is reusable
    with pytest.raises(bg.ArgumentError):
        p.prove_host(sc.witness[:-1])
    # appended to a caller's transcript: the tape is the caller's bytes followed by the proof
    t = bg.ProverTranscript()
    t.message(b"\x01" * 16)
    out = p.prove_host(sc.witness, transcript=t)
    assert out[:16] == b"\x01" * 16 and len(out) == 16 + len(ref)


def test_launch_shapes_change_no_bytes_and_autotune():
    """Every launch-shape choice gives the oracle's proof (exact arithmetic); the autotuner picks
    one in range, keeps the bytes and hands it to provers of the same shape set up later."""
    sc = csm.synthetic_circuit(14, 12000, 3, seed=91, log_public=2)
    prep = sc.cs.prepared()
    ref = orc.prove(sc.witness, 2, prep.and_csr, prep.mul_csr, 1)
    p = bg.Prover(bg.DeviceConstraintSystem(sc.cs.serialize()), 1)
    w = torch.from_numpy(sc.witness.view(np.int64)).cuda()
    default = {"tail_log": 11, "ntt_pass_layers": 8, "merkle_leaf_fuse": 8,
               "merkle_node_fuse": 9, "ntt_tile_bits": 12}
    assert p.tuning() == default
    for kw in ({"tail_log": 8}, {"tail_log": 12}, {"ntt_pass_layers": 4}, {"ntt_pass_layers": 6},
               {"merkle_leaf_fuse": 5}, {"merkle_node_fuse": 5}, {"merkle_node_fuse": 7},
               {"ntt_tile_bits": 9}, {"ntt_tile_bits": 10, "ntt_pass_layers": 8},
               {"ntt_tile_bits": 11, "ntt_pass_layers": 5}):
        p.set_tuning(**kw)
        assert p.prove(w).finalize() == ref, kw
        p.set_tuning(**default)
    with pytest.raises(bg.ArgumentError):
        p.set_tuning(tail_log=20)
    with pytest.raises(bg.ArgumentError):
        p.set_tuning(ntt_tile_bits=8)
    best = p.autotune(w, reps=1)
    assert 8 <= best["tail_log"] <= 12 and 6 <= best["ntt_pass_layers"] <= 8
    assert p.tuning() == best
    assert p.prove(w).finalize() == ref
    p2 = bg.Prover(bg.DeviceConstraintSystem(sc.cs.serialize()), 1)
    assert p2.tuning() == best
    assert p2.prove(w).finalize() == ref
