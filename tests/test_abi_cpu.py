"""CPU-only checks of the C ABI: the library loads, exports every declared symbol, and the host-only
entry points (FRI parameters, argument validation) behave like the reference without a GPU."""
import ctypes

import pytest

import oracle as orc
from binius64_b200 import _ffi


def test_library_loads_and_exports_all_declared_symbols():
    L = _ffi.lib()
    declared = _ffi.declared_functions()
    assert len(declared) >= 15
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"
    # every declared function has a ctypes signature in the binding
    assert set(declared) <= set(_ffi._SIGS), set(declared) - set(_ffi._SIGS)


def test_rust_binding_declares_every_entry():
    """The Rust `extern "C"` block a reference maintainer adds declares every
    entry point of the header, so the binding is complete as written."""
    import os
    import re
    with open(os.path.join(_ffi.ROOT, "INTEGRATION.md")) as f:
        text = f.read()
    rust = set(re.findall(r"pub fn (binius_[a-z0-9_]+)\(", text))
    missing = sorted(set(_ffi.declared_functions()) - rust)
    assert not missing, f"declared in the header, not in the Rust binding: {missing}"


def test_version():
    assert b"sm_100a" in _ffi.lib().binius_version()


@pytest.mark.parametrize("bits,rate", [(96, 1), (96, 2), (128, 1), (64, 3)])
def test_n_test_queries_matches_oracle(bits, rate):
    assert _ffi.lib().binius_fri_n_test_queries(bits, rate) == orc.calculate_n_test_queries(bits, rate)


def test_fri_param_kats_through_abi():
    L = _ffi.lib()
    assert L.binius_fri_n_test_queries(96, 1) == 232
    assert L.binius_fri_n_test_queries(96, 2) == 142
    for n in range(22, 35):
        assert L.binius_fri_estimate_optimal_arity(n, 256, 128) == 4
    for n in range(22, 28):
        assert L.binius_fri_estimate_optimal_arity(n, 1024, 128) == 6
    for n in range(1, 30):
        assert L.binius_fri_estimate_optimal_arity(n, 32, 16) == orc.estimate_optimal_arity(n, 32, 16)


def test_argument_errors_without_gpu():
    L = _ffi.lib()
    # NULL handles and impossible shapes are rejected before any CUDA call.
    assert L.binius_rs_encode_batch(None, None, 4, 1, 0, None, None) == _ffi.BINIUS_E_ARG
    assert b"NULL" in L.binius_last_error()
    assert L.binius_ntt_forward(None, None, 4, 0, 0, None) == _ffi.BINIUS_E_ARG
    assert L.binius_merkle_commit(None, 3, 0, None, None) == _ffi.BINIUS_E_ARG
    assert L.binius_fri_fold_interleaved(None, 3, 2, None, None, None) == _ffi.BINIUS_E_ARG
    out = ctypes.c_void_p()
    assert L.binius_ntt_create(0, None, 0, ctypes.byref(out)) == _ffi.BINIUS_E_ARG
    assert L.binius_ntt_create(0, None, 33, ctypes.byref(out)) == _ffi.BINIUS_E_ARG
    assert out.value is None
    # too many folding challenges for one call
    assert L.binius_fri_fold_interleaved(ctypes.c_void_p(16), 3, 9, ctypes.c_void_p(16),
                                         ctypes.c_void_p(16), None) == _ffi.BINIUS_E_ARG


def test_boundary_entries_reject_bad_arguments_without_gpu():
    """The MerkleTreeProver::layer, SumcheckProver, set-up and host-buffer prove entries check
    their arguments before touching the device (the pointers below are never dereferenced)."""
    L = _ffi.lib()
    E = _ffi.BINIUS_E_ARG
    fake = ctypes.c_void_p(256)
    # MerkleTreeProver::layer: NULL buffers; a layer below the leaves is IncorrectLayerDepth
    assert L.binius_merkle_layer(None, 4, 2, fake, None) == E
    assert L.binius_merkle_layer(fake, 4, 5, fake, None) == E
    assert b"IncorrectLayerDepth" in L.binius_last_error()
    out = ctypes.c_void_p()
    assert L.binius_sumcheck_bivariate_create(None, fake, 4, fake, None, ctypes.byref(out)) == E
    assert L.binius_sumcheck_quadratic_mle_create(fake, fake, fake, 34, fake, fake, None,
                                                  ctypes.byref(out)) == E
    assert L.binius_sumcheck_quadratic_mle_create(fake, fake, fake, 3, None, fake, None,
                                                  ctypes.byref(out)) == E
    # InOutCheckProver::new asserts eval_point.len() <= witness.log_len()
    assert L.binius_sumcheck_inout_create(fake, 3, fake, 4, None, ctypes.byref(out)) == E
    assert out.value is None
    # round calls on a NULL prover
    buf = (ctypes.c_uint8 * 64)()
    n = ctypes.c_uint32()
    for name in ("bivariate", "quadratic_mle", "inout"):
        assert getattr(L, f"binius_sumcheck_{name}_execute")(None, buf, ctypes.byref(n)) == E
        assert getattr(L, f"binius_sumcheck_{name}_fold")(None, buf) == E
        assert getattr(L, f"binius_sumcheck_{name}_finish")(None, buf) == E
    assert L.binius_sumcheck_destroy(None) == _ffi.BINIUS_OK
    assert L.binius_sumcheck_n_vars(None) == 0
    # one-call set-up and the host-buffer prove
    assert L.binius_setup(0, None, 0, 1, None, 0, ctypes.byref(out)) == E
    ln = ctypes.c_size_t(7)
    assert L.binius_prove(None, fake, 16, None, fake, 16, ctypes.byref(ln), None) == E
    assert ln.value == 7  # rejected before *len is written


def test_check_maps_argument_error():
    L = _ffi.lib()
    rc = L.binius_merkle_commit(None, 3, 0, None, None)
    with pytest.raises(_ffi.ArgumentError):
        _ffi.check(rc)


def test_fri_params_choice_matches_reference_formula():
    import binius64_b200 as bg
    # C3: 2^19 B128 witness elements, R = 1 -> log_code_len 20, arity 4 (estimate_optimal_arity with
    # 32-byte digests and 16-byte elements), batch 2^4, RS dim 2^15, arities [4, 4], 232 queries.
    arity = bg.estimate_optimal_arity(20, 32, 16)
    assert arity == 4
    p = bg.FRIParams.choose_with_constant_fold_arity(19, 96, 1, arity)
    assert p.log_batch_size == 4
    assert p.rs_code.log_dim == 15
    assert p.fold_arities == [4, 4]
    assert p.n_test_queries == 232
    assert p.log_terminal_dim == 7


def test_library_transcript_known_answers():
    """The library's host transcript against hasher_challenger.rs:209-280's chaining structure."""
    import hashlib

    import numpy as np

    import binius64_b200 as bg
    d0 = hashlib.sha256(b"").digest()
    t = bg.ProverTranscript()
    assert t.sample_bytes(8) == d0[:8]
    assert t.sample_bytes(24) == d0[8:]
    t.observe(bytes([0x48, 0x55]))
    assert t.sample_bytes(2) == hashlib.sha256(d0 + bytes([32] + [0] * 7) + bytes([0x48, 0x55])).digest()[:2]

    rng = np.random.default_rng(0)
    obs = rng.integers(0, 256, 1019, dtype=np.uint8).tobytes()
    t = bg.ProverTranscript()
    t.message(obs[:300])
    t.decommitment(b"not observed")
    t.message(obs[300:])
    first = hashlib.sha256(d0 + bytes(8) + obs).digest()
    assert t.sample_bytes(7) == first[:7]
    assert t.finalize() == obs[:300] + b"not observed" + obs[300:]
    # sample_bits: u32 LE of the next 4 bytes, masked
    v = t.sample_bits(5)
    assert v == int.from_bytes(first[7:11], "little") & 31


def test_library_transcript_matches_oracle_transcript():
    import numpy as np

    import binius64_b200 as bg
    import oracle as orc
    rng = np.random.default_rng(5)
    a, b = bg.ProverTranscript(), orc.Transcript()
    for step in range(40):
        if rng.integers(0, 2):
            data = rng.integers(0, 256, int(rng.integers(1, 200)), dtype=np.uint8).tobytes()
            a.message(data)
            b.observe(data)
        else:
            n = int(rng.integers(1, 80))
            assert a.sample_bytes(n) == b.sample(n), step
