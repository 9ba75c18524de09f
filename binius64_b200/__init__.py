"""B200-native (sm_100a) Binius64 prover hot path.

Host-side mirror of the reference's plugin surface for this path, over the C ABI in
include/binius_gpu.h (libbinius_gpu.so).  Names, argument meaning and error behaviour follow the
reference:

* ``AdditiveNTT`` -- trait AdditiveNTT / DomainContext (verifier/math/src/ntt/mod.rs:58-179) over a
  GenericPreExpanded domain (ntt/domain_context.rs:99-159).
* ``ReedSolomonCode.encode_batch`` -- verifier/math/src/reed_solomon.rs:128-201.
* ``BinaryMerkleTreeProver`` -- prover/prover/src/merkle_tree/prover.rs:16-119.
* ``FRIParams`` -- verifier/verifier/src/fri/common.rs:14-219.
* ``commit_interleaved`` -- prover/prover/src/fri/commit.rs:25-75.
* ``fold_interleaved`` / ``fold_codeword`` -- prover/prover/src/fri/fold.rs:260-318.

Device buffers are torch tensors (torch is plumbing for device memory and streams only) holding
field elements as int64 pairs of shape (n, 2): the 16-byte little-endian u128 encoding.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from ._ffi import ArgumentError, BiniusError, OutOfMemoryError, check, lib

__all__ = [
    "AdditiveNTT", "ReedSolomonCode", "BinaryMerkleTreeProver", "MerkleCommitted", "FRIParams",
    "CommitOutput", "commit_interleaved", "fold_interleaved", "fold_codeword", "gf_mul_batch",
    "to_device", "to_host", "ArgumentError", "BiniusError", "OutOfMemoryError", "version",
]


def _torch():
    import torch
    return torch


def version() -> str:
    return lib().binius_version().decode()


def _stream(stream=None) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _ptr(t) -> int:
    return t.data_ptr()


def _elems_of(t) -> int:
    assert t.dtype == _torch().int64 and t.is_contiguous(), "field buffers are contiguous int64"
    return t.numel() // 2


def _log2_exact(n: int, what: str) -> int:
    if n <= 0 or n & (n - 1):
        raise ArgumentError(1, f"{what} must be a power of two, got {n}")
    return n.bit_length() - 1


def to_device(arr: np.ndarray, device: str | int = "cuda"):
    """numpy uint64 (n, 2) -> device int64 (n, 2)."""
    torch = _torch()
    a = np.ascontiguousarray(arr, dtype=np.uint64).reshape(-1, 2)
    return torch.from_numpy(a.view(np.int64)).to(device)


def to_host(t) -> np.ndarray:
    """device int64 (n, 2) -> numpy uint64 (n, 2)."""
    return t.detach().cpu().contiguous().numpy().view(np.uint64).reshape(-1, 2)


def empty_elems(n: int, device="cuda"):
    return _torch().empty((n, 2), dtype=_torch().int64, device=device)


class AdditiveNTT:
    """Additive NTT over the GenericPreExpanded domain context of a binary subspace.

    ``basis`` is a list of ``log_domain`` field elements as Python ints (None = the standard basis
    x^i, BinarySubspace::with_dim).
    """

    def __init__(self, log_domain: int, basis=None, device: int | None = None):
        torch = _torch()
        self.device = torch.cuda.current_device() if device is None else int(device)
        self._handle = ctypes.c_void_p()
        buf = None
        if basis is not None:
            basis = list(basis)
            if len(basis) != log_domain:
                raise ArgumentError(1, "basis length must equal log_domain")
            arr = np.array([[b & (2**64 - 1), b >> 64] for b in basis], dtype=np.uint64)
            buf = arr.ctypes.data_as(ctypes.c_void_p)
        check(lib().binius_ntt_create(self.device, buf, log_domain, ctypes.byref(self._handle)))
        self.basis = basis

    @property
    def handle(self):
        return self._handle

    def log_domain_size(self) -> int:
        return int(lib().binius_ntt_log_domain(self._handle))

    def twiddles(self, copy: bool = True):
        """The flat twiddle table (layer l at [2^l - 1, 2^(l+1) - 1)) as a device tensor; with
        copy=False a zero-copy view that is valid while this object is alive."""
        torch = _torch()
        n = (1 << self.log_domain_size()) - 1
        ptr = lib().binius_ntt_twiddles(self._handle)

        class _View:
            __cuda_array_interface__ = {"shape": (n, 2), "typestr": "<i8", "data": (ptr, False),
                                        "version": 3, "strides": None}

        view = torch.as_tensor(_View(), device=f"cuda:{self.device}")
        return view.clone() if copy else view

    def twiddle(self, layer: int, block: int) -> int:
        t = to_host(self.twiddles(copy=False)[(1 << layer) - 1 + block].reshape(1, 2))[0]
        return int(t[0]) | (int(t[1]) << 64)

    def forward_transform(self, data, skip_early: int = 0, skip_late: int = 0, stream=None):
        log_len = _log2_exact(_elems_of(data), "data length")
        check(lib().binius_ntt_forward(self._handle, _ptr(data), log_len, skip_early, skip_late,
                                       _stream(stream)))

    def inverse_transform(self, data, skip_early: int = 0, skip_late: int = 0, stream=None):
        log_len = _log2_exact(_elems_of(data), "data length")
        check(lib().binius_ntt_inverse(self._handle, _ptr(data), log_len, skip_early, skip_late,
                                       _stream(stream)))

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                lib().binius_ntt_destroy(h)
            except Exception:
                pass
            self._handle = None


@dataclass
class ReedSolomonCode:
    log_dim: int
    log_inv_rate: int

    def log_len(self) -> int:
        return self.log_dim + self.log_inv_rate

    def encode_batch(self, ntt: AdditiveNTT, data, log_batch_size: int, out=None, stream=None):
        n = _elems_of(data)
        if n != 1 << (self.log_dim + log_batch_size):
            raise ArgumentError(1, "data.log_len() must equal log_dim + log_batch_size")
        if out is None:
            out = empty_elems(1 << (self.log_len() + log_batch_size), device=data.device)
        check(lib().binius_rs_encode_batch(ntt.handle, _ptr(data), self.log_dim, self.log_inv_rate,
                                           log_batch_size, _ptr(out), _stream(stream)))
        return out


@dataclass
class MerkleCommitted:
    """BinaryMerkleTree: flat digests (2^(L+1) - 1, 32) on the device, root last."""
    log_len: int
    nodes: object  # torch uint8 tensor

    def root(self) -> bytes:
        return bytes(self.nodes[-1].cpu().numpy().tobytes())

    def layer(self, layer_depth: int, stream=None) -> list[bytes]:
        """MerkleTreeProver::layer (prover/prover/src/merkle_tree/mod.rs:50-55): the digests at
        depth layer_depth (0 = the root), copied to the host."""
        buf = (ctypes.c_uint8 * (32 << max(0, min(layer_depth, 40))))()
        check(lib().binius_merkle_layer(_ptr(self.nodes), self.log_len, layer_depth,
                                        ctypes.addressof(buf), _stream(stream)))
        raw = bytes(buf)
        return [raw[32 * i: 32 * (i + 1)] for i in range(1 << layer_depth)]

    def branch(self, index: int, layer_depth: int, stream=None) -> list[bytes]:
        n = self.log_len - layer_depth
        buf = (ctypes.c_uint8 * max(1, 32 * n))()
        check(lib().binius_merkle_branch(_ptr(self.nodes), self.log_len, index, layer_depth,
                                         ctypes.addressof(buf), _stream(stream)))
        raw = bytes(buf)[: 32 * n]
        return [raw[32 * i: 32 * (i + 1)] for i in range(n)]


class BinaryMerkleTreeProver:
    """SHA-256 leaves + Binius SHA-256 compression nodes (StdDigest / StdCompression), or with
    hash="vision4" VisionHasherDigest leaves + VisionCompression nodes (the `-c vision4` setup)."""

    HASHES = ("sha256", "vision4")

    def __init__(self, hash: str = "sha256"):
        if hash not in self.HASHES:
            raise ArgumentError(1, f"unknown Merkle hash {hash!r}")
        self.hash = hash

    def commit(self, elements, batch_size: int, stream=None):
        n = _elems_of(elements)
        log_batch = _log2_exact(batch_size, "batch_size")
        if n % batch_size:
            raise ArgumentError(1, "IncorrectBatchSize")
        log_len = _log2_exact(n // batch_size, "leaf count")
        torch = _torch()
        nodes = torch.empty(((2 << log_len) - 1, 32), dtype=torch.uint8, device=elements.device)
        fn = lib().binius_merkle_commit if self.hash == "sha256" else \
            lib().binius_merkle_commit_vision4
        check(fn(_ptr(elements), log_len, log_batch, _ptr(nodes), _stream(stream)))
        committed = MerkleCommitted(log_len, nodes)
        return committed.root(), committed


def vision4_permute(states, stream=None):
    """The Vision-4 permutation of each 4-element state, in place: states is a device tensor of
    n * 4 field elements (n * 64 bytes)."""
    n = _elems_of(states)
    if n % 4:
        raise ArgumentError(1, "states: a multiple of 4 elements")
    check(lib().binius_vision4_permute(_ptr(states), n // 4, _stream(stream)))
    return states


def n_test_queries(security_bits: int, log_inv_rate: int) -> int:
    return int(lib().binius_fri_n_test_queries(security_bits, log_inv_rate))


def estimate_optimal_arity(log_block_length: int, digest_size: int, field_size: int) -> int:
    return int(lib().binius_fri_estimate_optimal_arity(log_block_length, digest_size, field_size))


def _ceil_log2(n: int) -> int:
    return 0 if n <= 1 else (n - 1).bit_length()


@dataclass
class FRIParams:
    rs_code: ReedSolomonCode
    log_batch_size: int
    fold_arities: list = field(default_factory=list)
    n_test_queries: int = 0

    @property
    def log_terminal_dim(self) -> int:
        return self.rs_code.log_dim - sum(self.fold_arities)

    @classmethod
    def choose_with_constant_fold_arity(cls, log_msg_len: int, security_bits: int,
                                        log_inv_rate: int, arity: int) -> "FRIParams":
        """verifier/verifier/src/fri/common.rs:64-115."""
        assert arity > 0
        log_batch_size = min(log_msg_len, arity)
        log_dim = log_msg_len - log_batch_size
        rs = ReedSolomonCode(log_dim, log_inv_rate)
        nq = n_test_queries(security_bits, log_inv_rate)
        cap_height = _ceil_log2(nq)
        log_terminal_len = min(max(cap_height, log_inv_rate), rs.log_len())
        quotient, remainder = divmod(rs.log_len() - log_terminal_len, arity)
        arities = [arity] * quotient + ([remainder] if remainder else [])
        if sum(arities) > rs.log_dim:
            raise ArgumentError(1, "InvalidFoldAritySequence")
        return cls(rs, log_batch_size, arities, nq)

    def log_len(self) -> int:
        return self.rs_code.log_len() + self.log_batch_size

    def log_msg_len(self) -> int:
        return self.rs_code.log_dim + self.log_batch_size

    def n_fold_rounds(self) -> int:
        return self.log_msg_len()

    def index_bits(self) -> int:
        return self.rs_code.log_len()


def standard_domain_rs_basis(log_code_len: int, log_batch: int, device=None) -> list[int]:
    """Basis of the RS code subspace chosen by Verifier::setup (verify.rs:85-97): row `log_batch` of
    the normalized subspace-polynomial evaluations of the standard domain of dim log_code_len
    (GenericOnTheFly::subspace)."""
    return domain_subspace(log_code_len, log_code_len - log_batch)


def domain_subspace(log_domain: int, dim: int, basis=None) -> list[int]:
    """DomainContext::subspace(dim) (verifier/math/src/ntt/domain_context.rs:142-147) of the domain
    of dimension log_domain over `basis` (default: BinarySubspace::with_dim, basis x^i), computed
    on the host without the twiddle table."""
    out = np.zeros((max(dim, 1), 2), dtype=np.uint64)
    b = None
    if basis is not None:
        b = np.array([[int(v) & ((1 << 64) - 1), int(v) >> 64] for v in basis], dtype=np.uint64)
    check(lib().binius_domain_subspace(None if b is None else b.ctypes.data, log_domain, dim,
                                       out.ctypes.data))
    return [int(t[0]) | (int(t[1]) << 64) for t in out[:dim]]


@dataclass
class CommitOutput:
    commitment: bytes
    committed: MerkleCommitted
    codeword: object


def commit_interleaved(params: FRIParams, ntt: AdditiveNTT, merkle_prover: BinaryMerkleTreeProver,
                       message, stream=None) -> CommitOutput:
    """prover/prover/src/fri/commit.rs:25-75."""
    if _elems_of(message) != 1 << params.log_msg_len():
        raise ArgumentError(1, "interleaved message length does not match code parameters")
    torch = _torch()
    rs = params.rs_code
    codeword = empty_elems(1 << params.log_len(), device=message.device)
    log_leaves = rs.log_len()
    nodes = torch.empty(((2 << log_leaves) - 1, 32), dtype=torch.uint8, device=message.device)
    root = (ctypes.c_uint8 * 32)()
    check(lib().binius_fri_commit_interleaved(ntt.handle, _ptr(message), rs.log_dim,
                                              rs.log_inv_rate, params.log_batch_size,
                                              _ptr(codeword), _ptr(nodes), ctypes.addressof(root),
                                              _stream(stream)))
    return CommitOutput(bytes(root), MerkleCommitted(log_leaves, nodes), codeword)


def _challenges_buf(challenges):
    arr = np.array([[c & (2**64 - 1), c >> 64] for c in challenges], dtype=np.uint64).reshape(-1, 2)
    return arr, (arr.ctypes.data_as(ctypes.c_void_p) if len(challenges) else None)


def fold_interleaved(codeword, challenges, log_len: int, log_batch_size: int, out=None,
                     stream=None):
    """prover/prover/src/fri/fold.rs:260-282."""
    if len(challenges) != log_batch_size:
        raise ArgumentError(1, "challenges.len() must equal log_batch_size")
    if _elems_of(codeword) != 1 << (log_len + log_batch_size):
        raise ArgumentError(1, "codeword length mismatch")
    arr, buf = _challenges_buf(challenges)
    if out is None:
        out = empty_elems(1 << log_len, device=codeword.device)
    check(lib().binius_fri_fold_interleaved(_ptr(codeword), log_len, log_batch_size, buf, _ptr(out),
                                            _stream(stream)))
    return out


def fold_codeword(ntt: AdditiveNTT, codeword, challenges, log_len: int, out=None, stream=None):
    """prover/prover/src/fri/fold.rs:297-318."""
    if _elems_of(codeword) != 1 << log_len:
        raise ArgumentError(1, "codeword length mismatch")
    arr, buf = _challenges_buf(challenges)
    if out is None:
        out = empty_elems(1 << (log_len - len(challenges)), device=codeword.device)
    check(lib().binius_fri_fold_codeword(ntt.handle, _ptr(codeword), log_len, buf, len(challenges),
                                         _ptr(out), _stream(stream)))
    return out


# ------------------------------------------------------------------ round-by-round sumchecks

def _elem_buf(v: int):
    return (ctypes.c_uint8 * 16)(*int(v).to_bytes(16, "little"))


def _elems_from(buf, n: int) -> list[int]:
    raw = bytes(buf)
    return [int.from_bytes(raw[16 * i:16 * (i + 1)], "little") for i in range(n)]


class _SumcheckProver:
    """The SumcheckProver trait (prover/prover/src/protocols/sumcheck/common.rs:29-101) over a
    device prover: execute() -> the round's RoundCoeffs (lowest degree first), fold(challenge),
    finish() -> the multilinears' evaluations.  The multilinears are device tensors folded in
    place; they must stay alive and untouched until finish()."""

    _kind = ""
    _n_evals = 0

    def __init__(self):
        self._h = ctypes.c_void_p()
        self._keep = ()

    def n_vars(self) -> int:
        return int(lib().binius_sumcheck_n_vars(self._h))

    def execute(self) -> list[int]:
        buf = (ctypes.c_uint8 * 48)()
        n = ctypes.c_uint32(0)
        check(getattr(lib(), f"binius_sumcheck_{self._kind}_execute")(self._h, buf,
                                                                      ctypes.byref(n)))
        return _elems_from(buf, n.value)

    def fold(self, challenge: int) -> None:
        check(getattr(lib(), f"binius_sumcheck_{self._kind}_fold")(self._h, _elem_buf(challenge)))

    def finish(self) -> list[int]:
        buf = (ctypes.c_uint8 * (16 * self._n_evals))()
        check(getattr(lib(), f"binius_sumcheck_{self._kind}_finish")(self._h, buf))
        return _elems_from(buf, self._n_evals)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().binius_sumcheck_destroy(h)
            except Exception:
                pass
            self._h = None


def _points_buf(point):
    arr = np.array([[int(c) & (2**64 - 1), int(c) >> 64] for c in point] or [[0, 0]],
                   dtype=np.uint64)
    return arr


class BivariateProductSumcheckProver(_SumcheckProver):
    """BivariateProductSumcheckProver::new([a, b], sum)
    (prover/prover/src/protocols/sumcheck/bivariate_product.rs:17-119)."""

    _kind, _n_evals = "bivariate", 2

    def __init__(self, a, b, sum: int, stream=None):
        super().__init__()
        n = _log2_exact(_elems_of(a), "multilinear length")
        if _elems_of(b) != _elems_of(a):
            raise ArgumentError(1, "MultilinearSizeMismatch")
        check(lib().binius_sumcheck_bivariate_create(_ptr(a), _ptr(b), n, _elem_buf(sum),
                                                     _stream(stream), ctypes.byref(self._h)))
        self._keep = (a, b)


class QuadraticMleCheckProver(_SumcheckProver):
    """QuadraticMleCheckProver::new([a, b, c], a*b - c, a*b, eval_point, eval_claim)
    (prover/prover/src/protocols/sumcheck/quadratic_mle.rs:21-229), the AND reduction's
    MLE-check."""

    _kind, _n_evals = "quadratic_mle", 3

    def __init__(self, a, b, c, eval_point, eval_claim: int, stream=None):
        super().__init__()
        n = len(eval_point)
        for m in (a, b, c):
            if _elems_of(m) != 1 << n:
                raise ArgumentError(1, "MultilinearSizeMismatch")
        pts = _points_buf(eval_point)
        check(lib().binius_sumcheck_quadratic_mle_create(
            _ptr(a), _ptr(b), _ptr(c), n, pts.ctypes.data, _elem_buf(eval_claim), _stream(stream),
            ctypes.byref(self._h)))
        self._keep = (a, b, c)

    def eval_point(self) -> list[int]:
        buf = (ctypes.c_uint8 * (16 * max(1, self.n_vars())))()
        check(lib().binius_sumcheck_quadratic_mle_eval_point(self._h, buf))
        return _elems_from(buf, self.n_vars())


class InOutCheckProver(_SumcheckProver):
    """InOutCheckProver::new(witness, eval_point) (prover/prover/src/protocols/inout_check.rs:
    19-221): eval_point has log_public coordinates, the public segment's."""

    _kind, _n_evals = "inout", 1

    def __init__(self, witness, eval_point, stream=None):
        super().__init__()
        n = _log2_exact(_elems_of(witness), "witness length")
        pts = _points_buf(eval_point)
        check(lib().binius_sumcheck_inout_create(_ptr(witness), n, pts.ctypes.data,
                                                 len(eval_point), _stream(stream),
                                                 ctypes.byref(self._h)))
        self._keep = (witness,)

    def eval_point(self) -> list[int]:
        buf = (ctypes.c_uint8 * (16 * max(1, self.n_vars())))()
        check(lib().binius_sumcheck_inout_eval_point(self._h, buf))
        return _elems_from(buf, self.n_vars())


def gf_mul_batch(a, b, out=None, stream=None):
    n = _elems_of(a)
    if _elems_of(b) != n:
        raise ArgumentError(1, "operand lengths differ")
    if out is None:
        out = empty_elems(n, device=a.device)
    check(lib().binius_gf_mul_batch(_ptr(a), _ptr(b), _ptr(out), n, _stream(stream)))
    return out


class ProverTranscript:
    """ProverTranscript<HasherChallenger<Sha256>> (verifier/transcript/src/transcript.rs:204-407)."""

    def __init__(self):
        self._h = ctypes.c_void_p()
        check(lib().binius_transcript_create(ctypes.byref(self._h)))

    @property
    def handle(self):
        return self._h

    def message(self, data: bytes) -> None:
        check(lib().binius_transcript_message(self._h, data, len(data)))

    def decommitment(self, data: bytes) -> None:
        check(lib().binius_transcript_decommitment(self._h, data, len(data)))

    def observe(self, data: bytes) -> None:
        check(lib().binius_transcript_observe(self._h, data, len(data)))

    def sample_bytes(self, n: int) -> bytes:
        buf = (ctypes.c_uint8 * max(n, 1))()
        check(lib().binius_transcript_sample(self._h, ctypes.addressof(buf), n))
        return bytes(buf)[:n]

    def sample(self) -> int:
        """CanSample<B128>: 16 bytes as a little-endian u128."""
        return int.from_bytes(self.sample_bytes(16), "little")

    def sample_bits(self, bits: int) -> int:
        return int(lib().binius_transcript_sample_bits(self._h, bits))

    def finalize(self) -> bytes:
        n = int(lib().binius_transcript_len(self._h))
        buf = (ctypes.c_uint8 * max(n, 1))()
        out = ctypes.c_size_t(0)
        check(lib().binius_transcript_finalize(self._h, ctypes.addressof(buf), n, ctypes.byref(out)))
        return bytes(buf)[: out.value]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().binius_transcript_destroy(h)
            except Exception:
                pass
            self._h = None


class PcsCommitted:
    """Device-resident codeword + Merkle tree of a PCS commitment."""

    def __init__(self, handle, root: bytes):
        self.handle = handle
        self.root = root

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                lib().binius_pcs_committed_destroy(h)
            except Exception:
                pass
            self.handle = None


MERKLE_HASHES = {"sha256": 0, "vision4": 1}  # BINIUS_MERKLE_SHA256 / BINIUS_MERKLE_VISION4


def _merkle_hash_id(name: str) -> int:
    if name not in MERKLE_HASHES:
        raise ArgumentError(1, f"unknown Merkle hash {name!r}")
    return MERKLE_HASHES[name]


class OneBitPCSProver:
    """OneBitPCSProver (prover/prover/src/pcs.rs:30-169) with SHA-256 Merkle trees, or Vision-4
    ones with merkle_hash="vision4"."""

    def __init__(self, ntt: AdditiveNTT, fri_params: FRIParams, merkle_hash: str = "sha256"):
        self.ntt = ntt
        self.fri_params = fri_params
        self._h = ctypes.c_void_p()
        ar = (ctypes.c_uint32 * max(1, len(fri_params.fold_arities)))(*fri_params.fold_arities)
        check(lib().binius_pcs_create(ntt.handle, fri_params.log_msg_len(),
                                      fri_params.log_batch_size, fri_params.rs_code.log_inv_rate,
                                      ar, len(fri_params.fold_arities), fri_params.n_test_queries,
                                      ctypes.byref(self._h)))
        check(lib().binius_pcs_set_merkle_hash(self._h, _merkle_hash_id(merkle_hash)))

    def commit(self, packed_multilin, stream=None) -> PcsCommitted:
        if _elems_of(packed_multilin) != 1 << self.fri_params.log_msg_len():
            raise ArgumentError(1, "packed multilinear length does not match the FRI parameters")
        out = ctypes.c_void_p()
        root = (ctypes.c_uint8 * 32)()
        check(lib().binius_pcs_commit(self._h, _ptr(packed_multilin), ctypes.byref(out),
                                      ctypes.addressof(root), _stream(stream)))
        return PcsCommitted(out, bytes(root))

    def prove(self, committed: PcsCommitted, packed_multilin, evaluation_point,
              transcript: ProverTranscript, stream=None) -> None:
        n = self.fri_params.log_msg_len() + 7
        if len(evaluation_point) != n:
            raise ArgumentError(1, f"evaluation point must have {n} coordinates")
        pt = np.array([[c & (2**64 - 1), c >> 64] for c in evaluation_point], dtype=np.uint64)
        check(lib().binius_pcs_prove(self._h, committed.handle, _ptr(packed_multilin),
                                     pt.ctypes.data_as(ctypes.c_void_p), transcript.handle,
                                     _stream(stream)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().binius_pcs_destroy(h)
            except Exception:
                pass
            self._h = None


class DeviceConstraintSystem:
    """A constraint system parsed from the reference's v2 wire format and uploaded to the device
    (ConstraintSystem::deserialize + validate_and_prepare)."""

    def __init__(self, cs_bytes: bytes, device: int | None = None,
                 key_collection: bytes | None = None):
        torch = _torch()
        self.device = torch.cuda.current_device() if device is None else int(device)
        self._h = ctypes.c_void_p()
        check(lib().binius_cs_from_bytes(self.device, cs_bytes, len(cs_bytes), ctypes.byref(self._h)))
        info = (ctypes.c_uint32 * 12)()
        check(lib().binius_cs_info(self._h, ctypes.addressof(info)))
        (self.n_const, self.n_inout, self.n_witness, self.n_internal, self.offset_inout,
         self.offset_witness, self.committed_total_len, self.n_scratch, self.n_and, self.n_mul,
         self.n_and_real, self.n_mul_real) = list(info)
        if key_collection is not None:
            self.load_key_collection(key_collection)

    @property
    def handle(self):
        return self._h

    def key_collection(self) -> bytes:
        """build_key_collection(cs) serialized (KeyCollection v1)."""
        return _sized_bytes(lib().binius_cs_key_collection, self._h)

    def load_key_collection(self, data: bytes) -> None:
        """Rebuilds the shift reduction's term table from a serialized KeyCollection, as
        Prover::setup_with_key_collection takes one; a collection that does not describe this
        constraint system raises ArgumentError and leaves the table as it was."""
        check(lib().binius_cs_load_key_collection(self._h, data, len(data)))

    def eval_operands(self, witness_words, which: int = 0, stream=None):
        torch = _torch()
        k, n = (3, self.n_and) if which == 0 else (4, self.n_mul)
        out = torch.empty(k * n, dtype=torch.int64, device=witness_words.device)
        check(lib().binius_eval_operands(self._h, witness_words.data_ptr(), which, out.data_ptr(),
                                         _stream(stream)))
        return out.view(k, n)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().binius_cs_destroy(h)
            except Exception:
                pass
            self._h = None


def _sized_bytes(fn, *args, guess: int = 0) -> bytes:
    """Calls a byte-writing entry point with a buffer of `guess` bytes (an upper bound spares the
    second call), or once to learn the length and again with a buffer that fits."""
    n = ctypes.c_size_t(0)
    buf = ctypes.create_string_buffer(guess) if guess else None
    if fn(*args, buf, guess, ctypes.byref(n)) == 0:
        return buf.raw[:n.value] if buf is not None else b""
    buf = ctypes.create_string_buffer(max(n.value, 1))
    check(fn(*args, buf, len(buf), ctypes.byref(n)))
    return buf.raw[:n.value]


def key_collection_from_cs_bytes(cs_bytes: bytes) -> bytes:
    """build_key_collection + KeyCollection::serialize (prover/prover/src/protocols/shift/
    key_collection.rs:238-312, 381-398) for a v2 constraint system, on the host alone."""
    # bound: a term takes >= 9 bytes of the constraint system and <= 16 of the collection (a key
    # of 11 and an index of 5); 8 bytes of key range per committed word (the u32 at byte 28)
    words = int.from_bytes(cs_bytes[28:32], "little") if len(cs_bytes) >= 32 else 0
    guess = 64 + 16 * (len(cs_bytes) // 9) + 8 * words
    return _sized_bytes(lib().binius_key_collection_from_cs_bytes, cs_bytes, len(cs_bytes),
                        guess=guess)


def and_reduction_prove(cs: DeviceConstraintSystem, witness_words, transcript: ProverTranscript,
                        stream=None):
    """prove_bitand_reduction: returns ((a_eval, b_eval, c_eval, z), eval_point) as ints."""
    log_n = cs.n_and.bit_length() - 1
    meta = (ctypes.c_uint8 * 64)()
    point = (ctypes.c_uint8 * (16 * log_n))()
    check(lib().binius_and_reduction_prove(cs.handle, witness_words.data_ptr(), transcript.handle,
                                           ctypes.addressof(meta), ctypes.addressof(point),
                                           _stream(stream)))
    mb, pb = bytes(meta), bytes(point)
    m = [int.from_bytes(mb[16 * i:16 * i + 16], "little") for i in range(4)]
    p = [int.from_bytes(pb[16 * i:16 * i + 16], "little") for i in range(log_n)]
    return m, p


def _elem_bytes(vals) -> bytes:
    return b"".join(int(v).to_bytes(16, "little") for v in vals)


def shift_reduction_prove(cs: DeviceConstraintSystem, witness_words, transcript: ProverTranscript,
                          bitand_data, intmul_data, stream=None):
    """shift::prove.  bitand_data = ((a, b, c) evals, r_zhat', r_x'), intmul_data = ((a, b, lo, hi)
    evals, r_zhat', r_x'), all as ints.  Returns (r_j ++ r_y, witness_eval) as ints."""
    (ae, az, ax), (me, mz, mx) = bitand_data, intmul_data
    if len(ae) != 3 or len(me) != 4:
        raise ArgumentError(1, "operator data: 3 AND and 4 MUL evaluations")
    if len(ax) != cs.n_and.bit_length() - 1 or len(mx) != cs.n_mul.bit_length() - 1:
        raise ArgumentError(1, "operator data: r_x' length != log2(padded constraint count)")
    band = _elem_bytes([*ae, az, *ax])
    bmul = _elem_bytes([*me, mz, *mx])
    n_point = 6 + cs.committed_total_len.bit_length() - 1
    point = (ctypes.c_uint8 * (16 * n_point))()
    ev = (ctypes.c_uint8 * 16)()
    check(lib().binius_shift_reduction_prove(cs.handle, witness_words.data_ptr(), transcript.handle,
                                             band, bmul, ctypes.addressof(point),
                                             ctypes.addressof(ev), _stream(stream)))
    pb = bytes(point)
    return ([int.from_bytes(pb[16 * i:16 * i + 16], "little") for i in range(n_point)],
            int.from_bytes(bytes(ev), "little"))


def intmul_reduction_prove(cs: DeviceConstraintSystem, witness_words, transcript: ProverTranscript,
                           stream=None):
    """prove_intmul_reduction: returns (eval_point, [a, b, c_lo, c_hi] bit-column evaluations)
    as ints (64 per column)."""
    log_n = cs.n_mul.bit_length() - 1
    point = (ctypes.c_uint8 * max(16, 16 * log_n))()
    evals = (ctypes.c_uint8 * (16 * 256))()
    check(lib().binius_intmul_reduction_prove(cs.handle, witness_words.data_ptr(),
                                              transcript.handle, ctypes.addressof(point),
                                              ctypes.addressof(evals), _stream(stream)))
    pb, eb = bytes(point), bytes(evals)
    p = [int.from_bytes(pb[16 * i:16 * i + 16], "little") for i in range(log_n)]
    e = [int.from_bytes(eb[16 * i:16 * i + 16], "little") for i in range(256)]
    return p, [e[64 * k:64 * (k + 1)] for k in range(4)]


class Prover:
    """Prover::setup + Prover::prove (prover/prover/src/prove.rs:95-303) over a device constraint
    system, with the parameters Verifier::setup chooses (verifier/verifier/src/verify.rs:61-108)."""

    _proof_buf = None  # prove_host's output buffer, kept between calls

    def __init__(self, cs: DeviceConstraintSystem, log_inv_rate: int = 1,
                 key_collection: bytes | None = None, merkle_hash: str = "sha256"):
        self.cs = cs  # the native prover keeps a reference
        self._h = ctypes.c_void_p()
        hash_id = _merkle_hash_id(merkle_hash)
        if key_collection is None:
            check(lib().binius_prover_setup(cs.handle, log_inv_rate, ctypes.byref(self._h)))
        else:  # Prover::setup_with_key_collection (prover/prover/src/prove.rs:89-115)
            check(lib().binius_prover_setup_with_key_collection(
                cs.handle, log_inv_rate, key_collection, len(key_collection),
                ctypes.byref(self._h)))
        # setup_sha256 / setup_vision4 (prover/examples/src/lib.rs:48-85)
        self.merkle_hash = merkle_hash
        check(lib().binius_prover_set_merkle_hash(self._h, hash_id))
        self._load_info()

    def _load_info(self):
        info = (ctypes.c_uint32 * 12)()
        check(lib().binius_prover_info(self._h, ctypes.addressof(info)))
        v = list(info)
        self.log_witness_elems, self.log_batch, self.log_inv_rate, self.n_queries = v[:4]
        self.fold_arities = v[5:5 + v[4]]

    def prove_host(self, words, transcript: ProverTranscript | None = None, stream=None) -> bytes:
        """Prover::prove over a host witness (committed_total_len uint64 words) through
        binius_prove: the witness is copied in and the finalized proof bytes come back."""
        w = np.ascontiguousarray(words, dtype=np.uint64)
        n = ctypes.c_size_t(0)
        t = transcript.handle if transcript is not None else None
        while True:
            # the proof buffer is kept by the prover (sized by the largest proof so far)
            buf = self._proof_buf
            if buf is None:
                buf = self._proof_buf = (ctypes.c_uint8 * (1 << 20))()
            cap = len(buf)
            rc = lib().binius_prove(self._h, w.ctypes.data, len(w), t, buf, cap, ctypes.byref(n),
                                    _stream(stream))
            if rc == 1 and n.value > cap and t is None:  # too small: prove again with room
                self._proof_buf = (ctypes.c_uint8 * n.value)()
                continue
            check(rc)
            return ctypes.string_at(buf, n.value)

    def prove(self, witness_words, transcript: ProverTranscript | None = None,
              stream=None) -> ProverTranscript:
        """witness_words: device int64 tensor of committed_total_len words."""
        if witness_words.numel() != self.cs.committed_total_len:
            raise ArgumentError(1, "witness length != committed_total_len")
        t = transcript if transcript is not None else ProverTranscript()
        check(lib().binius_prover_prove(self._h, witness_words.data_ptr(), t.handle,
                                        _stream(stream)))
        return t

    TUNING_KEYS = ("tail_log", "ntt_pass_layers", "merkle_leaf_fuse", "merkle_node_fuse",
                   "ntt_tile_bits")

    def tuning(self) -> dict:
        """The prover's launch-shape choices (binius_prover_get_tuning)."""
        out = (ctypes.c_uint32 * len(self.TUNING_KEYS))()
        check(lib().binius_prover_get_tuning(self._h, out))
        return dict(zip(self.TUNING_KEYS, list(out)))

    def set_tuning(self, **kw) -> None:
        t = self.tuning()
        t.update(kw)
        buf = (ctypes.c_uint32 * len(self.TUNING_KEYS))(*[t[k] for k in self.TUNING_KEYS])
        check(lib().binius_prover_set_tuning(self._h, buf))

    def autotune(self, witness_words, reps: int = 3, stream=None) -> dict:
        """binius_prover_autotune: measures the launch-shape choices for this statement shape on
        the device witness, keeps the fastest (proof bytes unchanged) and returns them."""
        out = (ctypes.c_uint32 * len(self.TUNING_KEYS))()
        check(lib().binius_prover_autotune(self._h, witness_words.data_ptr(), reps,
                                           _stream(stream), out))
        return dict(zip(self.TUNING_KEYS, list(out)))

    def workspace_bytes(self) -> int:
        """Device memory one proof takes (the queue's admission estimate)."""
        return int(lib().binius_prover_workspace_bytes(self._h))

    def phase_ms(self) -> dict:
        """Host wall-clock milliseconds of the last prove's phases."""
        out = (ctypes.c_double * 5)()
        check(lib().binius_prover_phase_ms(self._h, out))
        return dict(zip(("commit", "intmul", "bitand", "shift", "pcs"), list(out)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().binius_prover_destroy(h)
            except Exception:
                pass
            self._h = None


class _OwnedConstraintSystem:
    """The constraint system a prover from setup() owns: its witness length and device."""

    def __init__(self, committed_total_len: int, device: int):
        self.committed_total_len = committed_total_len
        self.device = device


def setup(cs_bytes: bytes, log_inv_rate: int = 1, key_collection: bytes | None = None,
          device: int | None = None) -> Prover:
    """binius_setup: ConstraintSystem::deserialize then Prover::setup (or
    setup_with_key_collection) in one call (prover/prover/src/prove.rs:81-121); the prover owns
    its constraint system."""
    torch = _torch()
    dev = torch.cuda.current_device() if device is None else int(device)
    p = Prover.__new__(Prover)
    p._h = ctypes.c_void_p()
    kc = key_collection
    check(lib().binius_setup(dev, cs_bytes, len(cs_bytes), log_inv_rate, kc,
                             len(kc) if kc else 0, ctypes.byref(p._h)))
    p.cs = _OwnedConstraintSystem(int(lib().binius_prover_committed_words(p._h)), dev)
    p.merkle_hash = "sha256"
    p._load_info()
    return p


# ---------------------------------------------------------------------------------------- formats

STD_CHALLENGER = "HasherChallenger<Sha256>"  # ChallengerWithName::NAME (verifier/verifier/src/config.rs:19-21)


def _size_out():
    return ctypes.c_size_t(0)


class ValuesData:
    """ValuesData (verifier/core/src/constraint_system.rs:889-990): a run of 64-bit words in the
    version-1 wire format (u32 version, u32 count, u64 words)."""

    SERIALIZATION_VERSION = 1

    def __init__(self, words):
        self.words = np.ascontiguousarray(np.asarray(words, dtype=np.uint64))

    def serialize(self) -> bytes:
        n = _size_out()
        buf = ctypes.create_string_buffer(8 + 8 * len(self.words))
        check(lib().binius_values_data_encode(self.words.ctypes.data, len(self.words), buf,
                                              len(buf), ctypes.byref(n)))
        return buf.raw[:n.value]

    @classmethod
    def deserialize(cls, data: bytes) -> "ValuesData":
        n = _size_out()
        cap = max(0, (len(data) - 8) // 8)
        out = np.zeros(max(cap, 1), dtype=np.uint64)
        check(lib().binius_values_data_decode(data, len(data), out.ctypes.data, cap,
                                              ctypes.byref(n)))
        return cls(out[:n.value].copy())

    def __len__(self):
        return len(self.words)


class Proof:
    """Proof (verifier/core/src/constraint_system.rs:993-1100): the transcript bytes and the
    challenger type, in the version-1 wire format."""

    SERIALIZATION_VERSION = 1

    def __init__(self, data: bytes, challenger_type: str = STD_CHALLENGER):
        self.data = bytes(data)
        self.challenger_type = challenger_type

    def serialize(self) -> bytes:
        n = _size_out()
        ch = self.challenger_type.encode()
        buf = ctypes.create_string_buffer(12 + len(ch) + len(self.data))
        check(lib().binius_proof_encode(self.data, len(self.data), ch, buf, len(buf),
                                        ctypes.byref(n)))
        return buf.raw[:n.value]

    @classmethod
    def deserialize(cls, data: bytes) -> "Proof":
        n = _size_out()
        out = ctypes.create_string_buffer(max(len(data), 1))
        ch = ctypes.create_string_buffer(max(len(data), 1) + 1)
        check(lib().binius_proof_decode(data, len(data), out, len(out), ctypes.byref(n), ch,
                                        len(ch)))
        return cls(out.raw[:n.value], ch.value.decode())


def value_vec_from_data(cs: DeviceConstraintSystem, public, non_public) -> np.ndarray:
    """ValueVec::new_from_data (verifier/core/src/constraint_system.rs:803-823): the committed words
    public ++ non_public (their total must be committed_total_len), then n_scratch zero words."""
    pub = np.ascontiguousarray(np.asarray(public, dtype=np.uint64))
    npub = np.ascontiguousarray(np.asarray(non_public, dtype=np.uint64))
    out = np.zeros(cs.committed_total_len + cs.n_scratch, dtype=np.uint64)
    check(lib().binius_value_vec_from_data(cs.handle, pub.ctypes.data, len(pub), npub.ctypes.data,
                                           len(npub), out.ctypes.data))
    return out


def load_prove(cs_bytes: bytes, public_bytes: bytes, non_public_bytes: bytes,
               log_inv_rate: int = 1, device: int | None = None) -> bytes:
    """The reference prover binary's flow (prover/examples/src/bin/prover.rs:46-99) on the GPU:
    ConstraintSystem v2 + public / non-public ValuesData v1 in, Proof v1 bytes out."""
    torch = _torch()
    cs = DeviceConstraintSystem(cs_bytes, device=device)
    words = value_vec_from_data(cs, ValuesData.deserialize(public_bytes).words,
                                ValuesData.deserialize(non_public_bytes).words)
    w = torch.from_numpy(words[:cs.committed_total_len].view(np.int64)).to(f"cuda:{cs.device}")
    transcript = Prover(cs, log_inv_rate).prove(w)
    return Proof(transcript.finalize(), STD_CHALLENGER).serialize()


class ProveQueue:
    """Batched / served proving over binius_queue_* (see include/binius_gpu.h): n_workers proving
    threads with their own streams, FIFO admission under an HBM budget."""

    def __init__(self, n_workers: int = 8, hbm_budget_bytes: int = 0, device: int | None = None):
        torch = _torch()
        self.device = torch.cuda.current_device() if device is None else int(device)
        self._h = ctypes.c_void_p()
        check(lib().binius_queue_create(self.device, n_workers, hbm_budget_bytes,
                                        ctypes.byref(self._h)))
        self._keep = {}

    def submit(self, prover: Prover, witness) -> int:
        """witness: a device int64 tensor or a host numpy uint64 array of committed_total_len
        words; it is kept alive until wait() returns."""
        t = ctypes.c_uint64(0)
        if isinstance(witness, np.ndarray):
            w = np.ascontiguousarray(witness, dtype=np.uint64)
            if w.shape[0] != prover.cs.committed_total_len:
                raise ArgumentError(1, "witness length != committed_total_len")
            check(lib().binius_queue_submit(self._h, prover._h, w.ctypes.data_as(ctypes.c_void_p),
                                            0, ctypes.byref(t)))
        else:
            w = witness
            if w.numel() != prover.cs.committed_total_len:
                raise ArgumentError(1, "witness length != committed_total_len")
            check(lib().binius_queue_submit(self._h, prover._h, w.data_ptr(), 1, ctypes.byref(t)))
        self._keep[t.value] = (w, prover)
        return t.value

    def stats(self) -> dict:
        """The queue's device-memory accounting: budget, accounted bytes now and at their peak,
        and the number of finished requests."""
        out = (ctypes.c_uint64 * 4)()
        check(lib().binius_queue_stats(self._h, out))
        return {"budget": out[0], "in_use": out[1], "peak": out[2], "completed": out[3]}

    def done(self, ticket: int) -> bool:
        d = ctypes.c_int(0)
        check(lib().binius_queue_poll(self._h, ticket, ctypes.byref(d)))
        return bool(d.value)

    def wait(self, ticket: int):
        """Returns (proof bytes, {"queued_ms", "prove_ms", "latency_ms", "phase_ms"})."""
        n = ctypes.c_size_t(0)
        times = (ctypes.c_double * 8)()
        cap = 1 << 21
        while True:
            buf = (ctypes.c_uint8 * cap)()
            rc = lib().binius_queue_wait(self._h, ticket, buf, cap, ctypes.byref(n), times)
            if rc == 1 and n.value > cap:  # buffer too small: the result is kept
                cap = n.value
                continue
            break
        self._keep.pop(ticket, None)
        check(rc)
        return bytes(buf)[: n.value], {"queued_ms": times[0], "prove_ms": times[1],
                                       "latency_ms": times[2],
                                       "phase_ms": dict(zip(("commit", "intmul", "bitand", "shift",
                                                             "pcs"), list(times)[3:]))}

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().binius_queue_destroy(h)
            self._h = None
        self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
