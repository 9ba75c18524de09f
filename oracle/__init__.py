"""CPU oracle for the Binius64 prover hot path -- TEST INFRASTRUCTURE ONLY.

ctypes bindings over ``oracle/liboracle.so`` (a C++ restatement of the reference algorithms, see
``oracle/oracle.h``).  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
legs may import this module; it is the checker, never the thing measured as the GPU product.

Field elements travel as numpy ``uint64`` arrays of shape ``(n, 2)`` (low word, high word), i.e.
the reference's 16-byte little-endian u128 encoding.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def build(force: bool = False) -> str:
    """Compile ``liboracle.so`` with the committed Makefile (make rebuilds it when a source is
    newer; force rebuilds it regardless)."""
    cmd = ["make", "-C", _HERE, "-s"] + (["-B"] if force else [])
    subprocess.run(cmd, check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_gf_mul.argtypes = [_u64p, _u64p, _u64p]
        L.orc_gf_mul_portable.argtypes = [_u64p, _u64p, _u64p]
        L.orc_gf_inv.argtypes = [_u64p, _u64p]
        L.orc_gf_mul_x.argtypes = [_u64p, _u64p]
        L.orc_gf_mul_inv_x.argtypes = [_u64p, _u64p]
        L.orc_gf_mul_vec.argtypes = [_u64p, _u64p, _u64p, ctypes.c_size_t]
        L.orc_aes_mul.argtypes = [ctypes.c_uint8, ctypes.c_uint8]
        L.orc_aes_mul.restype = ctypes.c_uint8
        L.orc_aes_to_ghash_table.argtypes = [_u64p]
        L.orc_sha256.argtypes = [_u8p, ctypes.c_size_t, _u8p]
        L.orc_sha256_compress_node.argtypes = [_u8p, _u8p, _u8p]
        L.orc_domain_twiddles.argtypes = [_u64p, ctypes.c_uint32, _u64p]
        L.orc_domain_twiddles.restype = ctypes.c_int
        for name in ("orc_ntt_forward", "orc_ntt_inverse"):
            f = getattr(L, name)
            f.argtypes = [_u64p, ctypes.c_uint32, _u64p, ctypes.c_uint32, ctypes.c_uint32,
                          ctypes.c_uint32]
            f.restype = ctypes.c_int
        L.orc_rs_encode_batch.argtypes = [_u64p, ctypes.c_uint32, _u64p, ctypes.c_uint32,
                                          ctypes.c_uint32, ctypes.c_uint32, _u64p]
        L.orc_rs_encode_batch.restype = ctypes.c_int
        L.orc_merkle_commit.argtypes = [_u64p, ctypes.c_uint32, ctypes.c_uint32, _u8p]
        L.orc_merkle_commit.restype = ctypes.c_int
        L.orc_set_merkle_hash.argtypes = [ctypes.c_int]
        L.orc_eval_form_run.argtypes = [_u8p, ctypes.c_size_t, _u64p, ctypes.c_size_t,
                                        ctypes.POINTER(ctypes.c_uint32),
                                        ctypes.POINTER(ctypes.c_uint32)]
        L.orc_eval_form_run.restype = ctypes.c_int
        L.orc_vision4_permutation.argtypes = [_u64p]
        L.orc_vision4_digest.argtypes = [_u8p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t),
                                         ctypes.c_size_t, _u8p]
        L.orc_vision4_compress.argtypes = [_u8p, _u8p]
        L.orc_vision4_map.argtypes = [ctypes.c_int, _u64p, _u64p]
        L.orc_vision4_constants.argtypes = [_u64p, _u64p]
        L.orc_vision4_merkle_commit.argtypes = [_u64p, ctypes.c_uint32, ctypes.c_uint32, _u8p]
        L.orc_vision4_merkle_commit.restype = ctypes.c_int
        L.orc_eq_ind_partial_eval.argtypes = [_u64p, ctypes.c_uint32, _u64p]
        L.orc_fri_fold_interleaved.argtypes = [_u64p, ctypes.c_uint32, ctypes.c_uint32, _u64p,
                                               _u64p]
        L.orc_fri_fold_interleaved.restype = ctypes.c_int
        L.orc_fri_fold_codeword.argtypes = [_u64p, ctypes.c_uint32, _u64p, ctypes.c_uint32, _u64p,
                                            ctypes.c_uint32, _u64p]
        L.orc_fri_fold_codeword.restype = ctypes.c_int
        L.orc_calculate_n_test_queries.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.orc_calculate_n_test_queries.restype = ctypes.c_uint32
        L.orc_estimate_optimal_arity.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
        L.orc_estimate_optimal_arity.restype = ctypes.c_uint32
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_transcript_new.restype = ctypes.c_void_p
        L.orc_transcript_free.argtypes = [ctypes.c_void_p]
        L.orc_transcript_observe.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_size_t]
        L.orc_transcript_sample.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_size_t]
        L.orc_eval_1b_mle.argtypes = [_u64p, ctypes.c_uint32, _u64p, _u64p]
        _u32p = ctypes.POINTER(ctypes.c_uint32)
        L.orc_pcs_prove.argtypes = [_u64p, _u64p, ctypes.c_uint32, ctypes.c_uint32,
                                    ctypes.c_uint32, _u32p, ctypes.c_uint32, ctypes.c_uint32,
                                    _u64p, _u8p, ctypes.c_size_t,
                                    ctypes.POINTER(ctypes.c_size_t)]
        L.orc_pcs_prove.restype = ctypes.c_int
        L.orc_pcs_verify.argtypes = [_u64p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                     _u32p, ctypes.c_uint32, ctypes.c_uint32, _u64p, _u64p, _u8p,
                                     ctypes.c_size_t]
        L.orc_pcs_verify.restype = ctypes.c_int
        L.orc_shifted_word.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32]
        L.orc_shifted_word.restype = ctypes.c_uint64
        L.orc_and_univariate_round.argtypes = [_u64p, _u64p, _u64p, ctypes.c_uint32, _u64p, _u64p]
        L.orc_and_fold_words.argtypes = [_u64p, ctypes.c_size_t, _u64p, _u64p]
        L.orc_and_reduction_prove.argtypes = [_u64p, _u64p, _u64p, ctypes.c_uint32, _u8p,
                                              ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t),
                                              _u64p, _u64p]
        L.orc_and_reduction_prove.restype = ctypes.c_int
        L.orc_and_reduction_verify.argtypes = [ctypes.c_uint32, _u8p, ctypes.c_size_t, _u64p, _u64p]
        L.orc_and_reduction_verify.restype = ctypes.c_int
        L.orc_and_word_ntt.argtypes = [ctypes.c_uint64, _u8p]
        L.orc_shift_h_parts.argtypes = [_u64p, _u64p, _u64p]
        L.orc_bivariate_rounds.argtypes = [_u64p, _u64p, ctypes.c_uint32, _u64p, _u64p, _u64p,
                                           _u64p]
        L.orc_quadratic_mle_rounds.argtypes = [_u64p, _u64p, _u64p, ctypes.c_uint32, _u64p,
                                               _u64p, _u64p, _u64p, _u64p]
        L.orc_inout_rounds.argtypes = [_u64p, ctypes.c_uint32, _u64p, ctypes.c_uint32, _u64p,
                                       _u64p, _u64p]
        _lib = L
    return _lib


def _p64(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u64p)


def _p8(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u8p)


def elems(n: int) -> np.ndarray:
    return np.zeros((n, 2), dtype=np.uint64)


def to_int(e) -> int:
    e = np.asarray(e, dtype=np.uint64).reshape(2)
    return int(e[0]) | (int(e[1]) << 64)


def from_int(v: int) -> np.ndarray:
    return np.array([v & ((1 << 64) - 1), v >> 64], dtype=np.uint64)


def from_ints(vs) -> np.ndarray:
    return np.stack([from_int(v) for v in vs]) if len(vs) else elems(0)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def gf_mul(a: int, b: int, portable: bool = False) -> int:
    A, B, O = from_int(a), from_int(b), elems(1)
    f = lib().orc_gf_mul_portable if portable else lib().orc_gf_mul
    f(_p64(A), _p64(B), _p64(O))
    return to_int(O)


def gf_mul_vec(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = elems(a.shape[0])
    lib().orc_gf_mul_vec(_p64(a), _p64(b), _p64(out), a.shape[0])
    return out


def gf_inv(a: int) -> int:
    A, O = from_int(a), elems(1)
    lib().orc_gf_inv(_p64(A), _p64(O))
    return to_int(O)


def gf_mul_x(a: int) -> int:
    A, O = from_int(a), elems(1)
    lib().orc_gf_mul_x(_p64(A), _p64(O))
    return to_int(O)


def gf_mul_inv_x(a: int) -> int:
    A, O = from_int(a), elems(1)
    lib().orc_gf_mul_inv_x(_p64(A), _p64(O))
    return to_int(O)


def aes_mul(a: int, b: int) -> int:
    return int(lib().orc_aes_mul(a, b))


def aes_to_ghash_table() -> list[int]:
    out = elems(256)
    lib().orc_aes_to_ghash_table(_p64(out))
    return [to_int(out[i]) for i in range(256)]


def sha256(data: bytes) -> bytes:
    buf = np.frombuffer(data, dtype=np.uint8).copy() if data else np.zeros(1, dtype=np.uint8)
    out = np.zeros(32, dtype=np.uint8)
    lib().orc_sha256(_p8(buf), len(data), _p8(out))
    return out.tobytes()


def compress_node(left: bytes, right: bytes) -> bytes:
    l = np.frombuffer(left, dtype=np.uint8).copy()
    r = np.frombuffer(right, dtype=np.uint8).copy()
    out = np.zeros(32, dtype=np.uint8)
    lib().orc_sha256_compress_node(_p8(l), _p8(r), _p8(out))
    return out.tobytes()


def domain_twiddles(dim: int, basis=None) -> np.ndarray:
    """Flat GenericPreExpanded twiddle table (layer l at [2^l - 1, 2^(l+1) - 1))."""
    out = elems((1 << dim) - 1)
    bp = None
    if basis is not None:
        b = from_ints(list(basis))
        bp = _p64(b)
    rc = lib().orc_domain_twiddles(bp, dim, _p64(out))
    assert rc == 0
    return out


def ntt_forward(twiddles: np.ndarray, log_domain: int, data: np.ndarray, skip_early: int = 0,
                skip_late: int = 0, inverse: bool = False) -> np.ndarray:
    d = np.ascontiguousarray(data, dtype=np.uint64).copy()
    log_d = int(d.shape[0]).bit_length() - 1
    f = lib().orc_ntt_inverse if inverse else lib().orc_ntt_forward
    rc = f(_p64(twiddles), log_domain, _p64(d), log_d, skip_early, skip_late)
    if rc:
        raise ValueError("ntt precondition violated")
    return d


def rs_encode_batch(twiddles: np.ndarray, log_domain: int, msg: np.ndarray, log_dim: int,
                    log_inv_rate: int, log_batch: int) -> np.ndarray:
    msg = np.ascontiguousarray(msg, dtype=np.uint64)
    assert msg.shape[0] == 1 << (log_dim + log_batch)
    out = elems(1 << (log_dim + log_batch + log_inv_rate))
    rc = lib().orc_rs_encode_batch(_p64(twiddles), log_domain, _p64(msg), log_dim, log_inv_rate,
                                   log_batch, _p64(out))
    if rc:
        raise ValueError("rs encode precondition violated")
    return out


def merkle_commit(elems_: np.ndarray, log_leaves: int, log_batch: int) -> np.ndarray:
    """All tree nodes, (2^(log_leaves+1) - 1, 32) uint8: leaves first, root last."""
    e = np.ascontiguousarray(elems_, dtype=np.uint64)
    assert e.shape[0] == 1 << (log_leaves + log_batch)
    nodes = np.zeros(((1 << (log_leaves + 1)) - 1) * 32, dtype=np.uint8)
    lib().orc_merkle_commit(_p64(e), log_leaves, log_batch, _p8(nodes))
    return nodes.reshape(-1, 32)


def _int_elems(vals) -> np.ndarray:
    out = np.zeros(2 * len(vals), dtype=np.uint64)
    for i, v in enumerate(vals):
        out[2 * i] = v & (2**64 - 1)
        out[2 * i + 1] = v >> 64
    return out


def _elems_int(arr) -> list:
    a = np.asarray(arr, dtype=np.uint64).reshape(-1, 2)
    return [int(lo) | (int(hi) << 64) for lo, hi in a]


def eval_form_run(code: bytes, values: np.ndarray):
    """Interpreter::run over a copy of values (uint64); returns (rc, values, n_failures,
    first_error_id)."""
    v = np.ascontiguousarray(values, dtype=np.uint64).copy()
    buf = np.frombuffer(bytes(code) or b"\0", dtype=np.uint8).copy()
    nf, fe = ctypes.c_uint32(0), ctypes.c_uint32(0)
    rc = lib().orc_eval_form_run(_p8(buf), len(code), _p64(v) if len(v) else None, len(v),
                                 ctypes.byref(nf), ctypes.byref(fe))
    return rc, v, nf.value, fe.value


class merkle_hash:
    """Context manager selecting the oracle's Merkle hash ("sha256" or "vision4") for
    merkle_commit, the PCS and prove / verify inside the block."""

    KINDS = {"sha256": 0, "vision4": 1}

    def __init__(self, name: str):
        self.kind = self.KINDS[name]

    def __enter__(self):
        lib().orc_set_merkle_hash(self.kind)
        return self

    def __exit__(self, *exc):
        lib().orc_set_merkle_hash(0)
        return False


def vision4_permutation(state: list) -> list:
    """Vision-4 permutation of a 4-element state (ints)."""
    s = _int_elems(state)
    lib().orc_vision4_permutation(_p64(s))
    return _elems_int(s)


def vision4_digest(data: bytes, splits=()) -> bytes:
    """VisionHasherDigest over data, updated in pieces ending at each split offset."""
    buf = np.frombuffer(bytes(data) or b"\0", dtype=np.uint8).copy()
    sp = (ctypes.c_size_t * max(1, len(splits)))(*splits)
    out = np.zeros(32, dtype=np.uint8)
    lib().orc_vision4_digest(_p8(buf), len(data), sp, len(splits), _p8(out))
    return out.tobytes()


def vision4_compress(left: bytes, right: bytes) -> bytes:
    buf = np.frombuffer(bytes(left) + bytes(right), dtype=np.uint8).copy()
    out = np.zeros(32, dtype=np.uint8)
    lib().orc_vision4_compress(_p8(buf), _p8(out))
    return out.tobytes()


def vision4_map(which: int, x: int) -> int:
    """0 = L (linear part of B), 1 = L^-1, 2 = B, 3 = B^-1."""
    a, o = _int_elems([x]), np.zeros(2, dtype=np.uint64)
    lib().orc_vision4_map(which, _p64(a), _p64(o))
    return _elems_int(o)[0]


def vision4_constants():
    """(17 x 4 round constants, B_INV_COEFFS[0]) as ints."""
    rc, b0 = np.zeros(17 * 8, dtype=np.uint64), np.zeros(2, dtype=np.uint64)
    lib().orc_vision4_constants(_p64(rc), _p64(b0))
    e = _elems_int(rc)
    return [e[4 * r:4 * r + 4] for r in range(17)], _elems_int(b0)[0]


def vision4_merkle_commit(elems_: np.ndarray, log_leaves: int, log_batch: int) -> np.ndarray:
    """All tree nodes with Vision-4 leaves and nodes, (2^(log_leaves+1) - 1, 32) uint8."""
    e = np.ascontiguousarray(elems_, dtype=np.uint64)
    assert e.shape[0] == 1 << (log_leaves + log_batch)
    nodes = np.zeros(((1 << (log_leaves + 1)) - 1) * 32, dtype=np.uint8)
    lib().orc_vision4_merkle_commit(_p64(e), log_leaves, log_batch, _p8(nodes))
    return nodes.reshape(-1, 32)


def eq_ind_partial_eval(point: np.ndarray) -> np.ndarray:
    p = np.ascontiguousarray(point, dtype=np.uint64).reshape(-1, 2)
    out = elems(1 << p.shape[0])
    lib().orc_eq_ind_partial_eval(_p64(p) if p.shape[0] else None, p.shape[0], _p64(out))
    return out


def fri_fold_interleaved(codeword: np.ndarray, log_len: int, log_batch: int,
                         challenges: np.ndarray) -> np.ndarray:
    cw = np.ascontiguousarray(codeword, dtype=np.uint64)
    ch = np.ascontiguousarray(challenges, dtype=np.uint64).reshape(-1, 2)
    assert ch.shape[0] == log_batch
    out = elems(1 << log_len)
    lib().orc_fri_fold_interleaved(_p64(cw), log_len, log_batch, _p64(ch) if log_batch else None,
                                   _p64(out))
    return out


def fri_fold_codeword(twiddles: np.ndarray, log_domain: int, codeword: np.ndarray, log_len: int,
                      challenges: np.ndarray) -> np.ndarray:
    cw = np.ascontiguousarray(codeword, dtype=np.uint64)
    ch = np.ascontiguousarray(challenges, dtype=np.uint64).reshape(-1, 2)
    n = ch.shape[0]
    out = elems(1 << (log_len - n))
    rc = lib().orc_fri_fold_codeword(_p64(twiddles), log_domain, _p64(cw), log_len,
                                     _p64(ch) if n else None, n, _p64(out))
    if rc:
        raise ValueError("fold precondition violated")
    return out


def calculate_n_test_queries(security_bits: int, log_inv_rate: int) -> int:
    return int(lib().orc_calculate_n_test_queries(security_bits, log_inv_rate))


def estimate_optimal_arity(log_block_length: int, digest_size: int, field_size: int) -> int:
    return int(lib().orc_estimate_optimal_arity(log_block_length, digest_size, field_size))


def random_elems(rng: np.random.Generator, n: int) -> np.ndarray:
    return rng.integers(0, np.iinfo(np.uint64).max, size=(n, 2), dtype=np.uint64, endpoint=True)


class Transcript:
    """HasherChallenger<Sha256> state machine (observe / sample only)."""

    def __init__(self):
        self._h = lib().orc_transcript_new()

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_transcript_free(self._h)
            self._h = None

    def observe(self, data: bytes) -> None:
        buf = np.frombuffer(data, dtype=np.uint8).copy() if data else np.zeros(1, dtype=np.uint8)
        lib().orc_transcript_observe(self._h, _p8(buf), len(data))

    def sample(self, n: int) -> bytes:
        out = np.zeros(max(n, 1), dtype=np.uint8)
        lib().orc_transcript_sample(self._h, _p8(out), n)
        return out.tobytes()[:n]


def eval_1b_mle(witness: np.ndarray, point: np.ndarray) -> np.ndarray:
    w = np.ascontiguousarray(witness, dtype=np.uint64)
    pt = np.ascontiguousarray(point, dtype=np.uint64)
    out = elems(1)
    lib().orc_eval_1b_mle(_p64(w), w.shape[0].bit_length() - 1, _p64(pt), _p64(out))
    return out[0]


def _u32arr(vals):
    a = np.array(list(vals) or [0], dtype=np.uint32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def pcs_prove(twiddles, witness, log_batch, log_inv_rate, arities, n_queries, eval_point) -> bytes:
    w = np.ascontiguousarray(witness, dtype=np.uint64)
    log_msg = w.shape[0].bit_length() - 1
    pt = np.ascontiguousarray(eval_point, dtype=np.uint64)
    ar, arp = _u32arr(arities)
    cap = 1 << 26
    out = np.zeros(cap, dtype=np.uint8)
    n = ctypes.c_size_t(0)
    rc = lib().orc_pcs_prove(_p64(twiddles), _p64(w), log_msg, log_batch, log_inv_rate, arp,
                             len(arities), n_queries, _p64(pt), _p8(out), cap, ctypes.byref(n))
    assert rc == 0, "proof buffer too small"
    return out[: n.value].tobytes()


def pcs_verify(twiddles, log_msg, log_batch, log_inv_rate, arities, n_queries, eval_point, claim,
               proof: bytes) -> int:
    pt = np.ascontiguousarray(eval_point, dtype=np.uint64)
    ar, arp = _u32arr(arities)
    cl = np.ascontiguousarray(claim, dtype=np.uint64).reshape(2)
    pr = np.frombuffer(proof, dtype=np.uint8).copy()
    return int(lib().orc_pcs_verify(_p64(twiddles), log_msg, log_batch, log_inv_rate, arp,
                                    len(arities), n_queries, _p64(pt), _p64(cl), _p8(pr),
                                    len(proof)))


def shifted_word(w: int, variant: int, amount: int) -> int:
    return int(lib().orc_shifted_word(w, variant, amount))


def and_univariate_round(a, b, c, big) -> np.ndarray:
    a, b, c = (np.ascontiguousarray(x, dtype=np.uint64) for x in (a, b, c))
    log_n = a.shape[0].bit_length() - 1
    big = np.ascontiguousarray(big, dtype=np.uint64).reshape(-1, 2)
    out = elems(64)
    lib().orc_and_univariate_round(_p64(a), _p64(b), _p64(c), log_n,
                                   _p64(big) if big.shape[0] else None, _p64(out))
    return out


def and_fold_words(w, z) -> np.ndarray:
    w = np.ascontiguousarray(w, dtype=np.uint64)
    zz = np.ascontiguousarray(z, dtype=np.uint64).reshape(2)
    out = elems(w.shape[0])
    lib().orc_and_fold_words(_p64(w), w.shape[0], _p64(zz), _p64(out))
    return out


def and_reduction_prove(a, b, c):
    """Returns (proof bytes, (a_eval, b_eval, c_eval, z), eval_point) on a fresh transcript."""
    a, b, c = (np.ascontiguousarray(x, dtype=np.uint64) for x in (a, b, c))
    log_n = a.shape[0].bit_length() - 1
    cap = 1 << 20
    out = np.zeros(cap, dtype=np.uint8)
    n = ctypes.c_size_t(0)
    meta = elems(4)
    point = elems(log_n)
    rc = lib().orc_and_reduction_prove(_p64(a), _p64(b), _p64(c), log_n, _p8(out), cap,
                                       ctypes.byref(n), _p64(meta), _p64(point))
    assert rc == 0
    return out[: n.value].tobytes(), meta, point


def and_reduction_verify(log_n: int, proof: bytes):
    pr = np.frombuffer(proof, dtype=np.uint8).copy()
    meta = elems(4)
    point = elems(log_n)
    rc = lib().orc_and_reduction_verify(log_n, _p8(pr), len(proof), _p64(meta), _p64(point))
    return rc, meta, point


def mle_eval(values: np.ndarray, point: np.ndarray) -> np.ndarray:
    """Multilinear evaluation sum_i values[i] eq(point)[i] (point[j] <-> index bit j)."""
    eq = eq_ind_partial_eval(point)
    prods = gf_mul_vec(np.ascontiguousarray(values, dtype=np.uint64), eq)
    return np.bitwise_xor.reduce(prods, axis=0)


# ---- shift reduction ----

_u32pp = ctypes.POINTER(ctypes.POINTER(ctypes.c_uint32))


def _csr_args(csr):
    """(keep-alive arrays, u32 pointer triple, u8 variants, n_constraints) for an OperandCSR."""
    arrs = [np.ascontiguousarray(x, dtype=np.uint32)
            for x in (csr.offsets, csr.value_index, csr.amount)]
    arrs = [a if a.size else np.zeros(1, np.uint32) for a in arrs]
    ptrs = (ctypes.POINTER(ctypes.c_uint32) * 3)(
        *[a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)) for a in arrs])
    var = np.ascontiguousarray(csr.variant, dtype=np.uint8)
    if not var.size:
        var = np.zeros(1, np.uint8)
    n = (len(csr.offsets) - 1) // csr.k
    return (arrs, var), ctypes.cast(ptrs, _u32pp), _p8(var), n


def _op_data(d):
    evals, rz, rx = (np.ascontiguousarray(x, dtype=np.uint64).reshape(-1, 2) for x in d)
    if rx.size == 0:
        rx = elems(1)
    return (evals, rz, rx)


def _shift_lib():
    L = lib()
    if not getattr(L, "_shift_ready", False):
        common = [_u64p, ctypes.c_uint32, ctypes.c_uint32, _u32pp, _u8p, ctypes.c_uint32, _u32pp,
                  _u8p, ctypes.c_uint32, _u64p, _u64p, _u64p, _u64p, _u64p, _u64p]
        L.orc_shift_prove.argtypes = common + [_u8p, ctypes.c_size_t,
                                               ctypes.POINTER(ctypes.c_size_t), _u64p, _u64p]
        L.orc_shift_verify.argtypes = common + [_u8p, ctypes.c_size_t, _u64p, _u64p]
        L.orc_oblong_eval.argtypes = [_u64p, ctypes.c_uint32, _u64p, _u64p, _u64p]
        L._shift_ready = True
    return L


def shift_prove(words, log_public, and_csr, mul_csr, and_data, mul_data):
    """Shift reduction on a fresh transcript.

    and_data / mul_data = (evals, r_zhat', r_x') with AND evals (a, b, c) and MUL evals
    (a, b, lo, hi).  Returns (proof bytes, point r_j ++ r_y, (witness_eval, initial_sum, claim)).
    """
    L = _shift_lib()
    words = np.ascontiguousarray(words, dtype=np.uint64)
    log_words = words.shape[0].bit_length() - 1
    ka, pa, va, na = _csr_args(and_csr)
    km, pm, vm, nm = _csr_args(mul_csr)
    ad, md = _op_data(and_data), _op_data(mul_data)
    cap = 64 * (log_words + 16) + 4096
    out = np.zeros(cap, dtype=np.uint8)
    n = ctypes.c_size_t(0)
    point = elems(6 + log_words)
    out3 = elems(3)
    rc = L.orc_shift_prove(_p64(words), log_words, log_public, pa, va, na, pm, vm, nm,
                           *[_p64(x) for x in ad], *[_p64(x) for x in md], _p8(out), cap,
                           ctypes.byref(n), _p64(point), _p64(out3))
    assert rc == 0
    return out[: n.value].tobytes(), point, out3


def shift_verify(public_words, log_words, log_public, and_csr, mul_csr, and_data, mul_data,
                 proof: bytes):
    """Restated shift verifier; returns (rc, witness_eval, point) with rc 0 = accepted."""
    L = _shift_lib()
    pub = np.ascontiguousarray(public_words, dtype=np.uint64)
    ka, pa, va, na = _csr_args(and_csr)
    km, pm, vm, nm = _csr_args(mul_csr)
    ad, md = _op_data(and_data), _op_data(mul_data)
    pr = np.frombuffer(proof, dtype=np.uint8).copy()
    ev = elems(1)
    point = elems(6 + log_words)
    rc = L.orc_shift_verify(_p64(pub), log_words, log_public, pa, va, na, pm, vm, nm,
                            *[_p64(x) for x in ad], *[_p64(x) for x in md], _p8(pr), len(proof),
                            _p64(ev), _p64(point))
    return rc, ev[0], point


def oblong_eval(values, z, r_x) -> np.ndarray:
    """sum_c eq(r_x)[c] sum_j bit_j(values[c]) L_j(z) over the {phi(t) : t < 64} domain."""
    L = _shift_lib()
    v = np.ascontiguousarray(values, dtype=np.uint64)
    rx = np.ascontiguousarray(r_x, dtype=np.uint64).reshape(-1, 2)
    log_n = rx.shape[0]
    assert v.shape[0] == 1 << log_n
    if rx.size == 0:
        rx = elems(1)
    zz = np.ascontiguousarray(z, dtype=np.uint64).reshape(2)
    out = elems(1)
    L.orc_oblong_eval(_p64(v), log_n, _p64(zz), _p64(rx), _p64(out))
    return out[0]


# ---- integer multiplication reduction ----

def _intmul_lib():
    L = lib()
    if not getattr(L, "_intmul_ready", False):
        L.orc_intmul_prove.argtypes = [_u64p, _u64p, _u64p, _u64p, ctypes.c_uint32, _u8p,
                                       ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), _u64p,
                                       _u64p]
        L.orc_intmul_verify.argtypes = [ctypes.c_uint32, _u8p, ctypes.c_size_t, _u64p, _u64p]
        L._intmul_ready = True
    return L


def intmul_prove(a, b, lo, hi):
    """IntMul reduction on a fresh transcript; returns (proof, eval_point, evals (4, 64, 2)) with
    evals the bit-column evaluations of a, b, lo, hi."""
    L = _intmul_lib()
    cols = [np.ascontiguousarray(x, dtype=np.uint64) for x in (a, b, lo, hi)]
    log_n = cols[0].shape[0].bit_length() - 1
    cap = 1 << 22
    out = np.zeros(cap, dtype=np.uint8)
    n = ctypes.c_size_t(0)
    point = elems(max(log_n, 1))
    evals = elems(256)
    rc = L.orc_intmul_prove(*[_p64(c) for c in cols], log_n, _p8(out), cap, ctypes.byref(n),
                            _p64(point), _p64(evals))
    assert rc == 0
    return out[: n.value].tobytes(), point[:log_n], evals.reshape(4, 64, 2)


def intmul_verify(log_n: int, proof: bytes):
    """Restated IntMul verifier; returns (rc, eval_point, evals) with rc 0 = accepted."""
    L = _intmul_lib()
    pr = np.frombuffer(proof, dtype=np.uint8).copy()
    point = elems(max(log_n, 1))
    evals = elems(256)
    rc = L.orc_intmul_verify(log_n, _p8(pr), len(proof), _p64(point), _p64(evals))
    return rc, point[:log_n], evals.reshape(4, 64, 2)


# ---- whole prove / verify ----

def _prove_lib():
    L = lib()
    if not getattr(L, "_prove_ready", False):
        csr = [_u32pp, _u8p, ctypes.c_uint32]
        L.orc_prove_params.argtypes = [ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.POINTER(ctypes.c_uint32),
                                       ctypes.POINTER(ctypes.c_uint32)]
        L.orc_prove.argtypes = ([_u64p, ctypes.c_uint32, ctypes.c_uint32] + csr + csr +
                                [ctypes.c_uint32, _u8p, ctypes.c_size_t,
                                 ctypes.POINTER(ctypes.c_size_t)])
        L.orc_verify.argtypes = ([_u64p, ctypes.c_uint32, ctypes.c_uint32] + csr + csr +
                                 [ctypes.c_uint32, _u8p, ctypes.c_size_t])
        L._prove_ready = True
    return L


def prove_params(log_words: int, log_inv_rate: int = 1):
    """(log_witness_elems, log_batch, n_queries, arities) chosen by Verifier::setup."""
    L = _prove_lib()
    o4 = (ctypes.c_uint32 * 4)()
    ar = (ctypes.c_uint32 * 8)()
    L.orc_prove_params(log_words, log_inv_rate, o4, ar)
    return o4[0], o4[1], o4[2], list(ar)[: o4[3]]


def prove(words, log_public: int, and_csr, mul_csr, log_inv_rate: int = 1) -> bytes:
    """Prover::prove on a fresh transcript over the prepared (padded) CSR constraint system."""
    L = _prove_lib()
    w = np.ascontiguousarray(words, dtype=np.uint64)
    log_words = w.shape[0].bit_length() - 1
    ka, pa, va, na = _csr_args(and_csr)
    km, pm, vm, nm = _csr_args(mul_csr)
    cap = 1 << 24
    out = np.zeros(cap, dtype=np.uint8)
    n = ctypes.c_size_t(0)
    rc = L.orc_prove(_p64(w), log_words, log_public, pa, va, na, pm, vm, nm, log_inv_rate,
                     _p8(out), cap, ctypes.byref(n))
    assert rc == 0
    return out[: n.value].tobytes()


def verify(public_words, log_words: int, log_public: int, and_csr, mul_csr, proof: bytes,
           log_inv_rate: int = 1) -> int:
    """Restated Verifier::verify; 0 = accepted."""
    L = _prove_lib()
    pub = np.ascontiguousarray(public_words, dtype=np.uint64)
    ka, pa, va, na = _csr_args(and_csr)
    km, pm, vm, nm = _csr_args(mul_csr)
    pr = np.frombuffer(proof, dtype=np.uint8).copy()
    return L.orc_verify(_p64(pub), log_words, log_public, pa, va, na, pm, vm, nm, log_inv_rate,
                        _p8(pr), len(proof))


# ---- shift reduction KeyCollection (prover/prover/src/protocols/shift/key_collection.rs) ----

def key_collection(and_csr, mul_csr, n_words: int) -> bytes:
    """build_key_collection + serialize (v1) over the padded operand lists of a constraint system
    with n_words committed words."""
    L = lib()
    if not getattr(L, "_kc_ready", False):
        csr = [_u32pp, _u8p, ctypes.c_uint32]
        L.orc_key_collection.argtypes = csr + csr + [ctypes.c_uint32, _u8p, ctypes.c_size_t,
                                                     ctypes.POINTER(ctypes.c_size_t)]
        L._kc_ready = True
    ka, pa, va, na = _csr_args(and_csr)
    km, pm, vm, nm = _csr_args(mul_csr)
    n_terms = len(and_csr.value_index) + len(mul_csr.value_index)
    cap = 16 + 8 * n_words + 16 * n_terms
    out = np.zeros(cap, dtype=np.uint8)
    n = ctypes.c_size_t(0)
    rc = L.orc_key_collection(pa, va, na, pm, vm, nm, n_words, _p8(out), cap, ctypes.byref(n))
    assert rc == 0
    return out[: n.value].tobytes()


# ---------------------------------------------------------------- round-by-round sumchecks

def bivariate_rounds(a, b, claimed_sum: int, challenges):
    """BivariateProductSumcheckProver (sumcheck/bivariate_product.rs:17-119) over the given
    challenges: (per-round coefficients (n, 3, 2), final evaluations (2, 2))."""
    n = len(challenges)
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    ch = np.ascontiguousarray(challenges, dtype=np.uint64).reshape(-1, 2)
    s = from_int(claimed_sum)
    co, ev = elems(3 * n), elems(2)
    lib().orc_bivariate_rounds(_p64(a), _p64(b), n, _p64(s), _p64(ch), _p64(co), _p64(ev))
    return co.reshape(n, 3, 2), ev


def quadratic_mle_rounds(a, b, c, point, claim: int, challenges):
    """QuadraticMleCheckProver with composition a*b - c (sumcheck/quadratic_mle.rs:21-229)."""
    n = len(challenges)
    cols = [np.ascontiguousarray(x) for x in (a, b, c)]
    pt = np.ascontiguousarray(point, dtype=np.uint64).reshape(-1, 2)
    ch = np.ascontiguousarray(challenges, dtype=np.uint64).reshape(-1, 2)
    cl = from_int(claim)
    co, ev = elems(3 * n), elems(3)
    lib().orc_quadratic_mle_rounds(_p64(cols[0]), _p64(cols[1]), _p64(cols[2]), n, _p64(pt),
                                   _p64(cl), _p64(ch), _p64(co), _p64(ev))
    return co.reshape(n, 3, 2), ev


def inout_rounds(w, point, challenges):
    """InOutCheckProver (protocols/inout_check.rs:19-221): witness of 2^n values, point of m
    coordinates (the public segment's)."""
    n = len(challenges)
    w = np.ascontiguousarray(w)
    pt = np.ascontiguousarray(point, dtype=np.uint64).reshape(-1, 2)
    m = pt.shape[0]
    ch = np.ascontiguousarray(challenges, dtype=np.uint64).reshape(-1, 2)
    co, ev = elems(2 * n), elems(1)
    lib().orc_inout_rounds(_p64(w), n, _p64(pt if m else elems(1)), m, _p64(ch), _p64(co),
                           _p64(ev))
    return co.reshape(n, 2, 2), ev


def and_word_ntt(w: int) -> list[int]:
    """The AND univariate round's extension evaluations of one 64-bit word (64 GF(2^8) bytes at
    the points 64..127)."""
    out = np.zeros(64, dtype=np.uint8)
    lib().orc_and_word_ntt(int(w), _p8(out))
    return [int(x) for x in out]


def shift_h_parts(r_zhat: int):
    """build_h_parts at r_zhat: ((8, 4096, 2) h multilinears, (64, 2) Lagrange evaluations)."""
    z = from_int(r_zhat)
    h, lt = elems(8 * 4096), elems(64)
    lib().orc_shift_h_parts(_p64(z), _p64(h), _p64(lt))
    return h.reshape(8, 4096, 2), lt
