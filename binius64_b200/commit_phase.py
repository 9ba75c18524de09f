"""The FRI commit phase of an interleaved Reed-Solomon commitment, over preallocated device buffers.

One run is fri::commit_interleaved (ReedSolomonCode::encode_batch, then the Merkle commit whose
leaves are the 2^log_batch interleaved symbols of one codeword position;
prover/prover/src/fri/commit.rs:25-75), followed by `n_folds` fold rounds, each committed as FRI
commits a folded codeword (leaves = cosets of 2^arity consecutive values;
FRIFoldProver::execute_fold_round, prover/prover/src/fri/fold.rs:117-175):

* round 1 folds the interleaved columns with log_batch challenges (fold_interleaved,
  fold.rs:260-282) when log_batch > 0, else `arity` codeword variables;
* later rounds fold `arity` codeword variables (fold_codeword, fold.rs:297-318).

Every kernel runs through the C ABI on one stream; nothing is allocated per run.  The counters
(`algorithmic_bytes`, `gf_mults`, `sha256_compressions`) are the per-run work that the roofline
figures divide: message read, codeword written and read once by the leaf hashing, tree written,
each fold reading its input and writing its output and tree.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import AdditiveNTT, standard_domain_rs_basis
from ._ffi import check, lib


def _ceil_div(a: int, b: int) -> int:
    return -(-a // b)


def leaf_compressions(log_leaves: int, leaf_bytes: int) -> int:
    """SHA-256 compressions of a tree of 2^log_leaves leaves of leaf_bytes each (padding adds 9
    bytes), plus its 2^log_leaves - 1 node compressions."""
    return (1 << log_leaves) * _ceil_div(leaf_bytes + 9, 64) + (1 << log_leaves) - 1


class CommitPhase:
    """RS encode + Merkle commit + FRI fold rounds of a seeded uniform interleaved message.

    log_len: log2 of one column's codeword length; the message has 2^(log_len - log_inv_rate)
    rows of 2^log_batch columns.  The NTT is the Reed-Solomon code's own subspace of the standard
    domain of dimension log_len + log_batch (the subspace Verifier::setup gives the code,
    verifier/verifier/src/verify.rs:85-97)."""

    def __init__(self, log_len: int, log_inv_rate: int, log_batch: int, n_folds: int = 3,
                 arity: int = 4, seed: int = 0, device: int | None = None):
        import torch
        if log_len - log_inv_rate < 1 or log_len < n_folds * arity + (0 if log_batch else arity):
            raise ValueError("code too short for the fold rounds")
        self.torch = torch
        self.device = torch.cuda.current_device() if device is None else int(device)
        d = f"cuda:{self.device}"
        self.log_len, self.log_inv_rate, self.log_batch = log_len, log_inv_rate, log_batch
        self.log_dim = log_len - log_inv_rate
        self.n_folds, self.arity = n_folds, arity
        basis = standard_domain_rs_basis(log_len + log_batch, log_batch)
        self.basis = basis
        self.ntt = AdditiveNTT(log_len, basis=basis, device=self.device)
        gen = torch.Generator(device=d).manual_seed(seed)
        self.message = torch.randint(-2**63, 2**63 - 1, (1 << (self.log_dim + log_batch), 2),
                                     dtype=torch.int64, device=d, generator=gen)
        self.codeword = torch.empty((1 << (log_len + log_batch), 2), dtype=torch.int64, device=d)
        self.nodes = torch.empty(((2 << log_len) - 1, 32), dtype=torch.uint8, device=d)
        # fold rounds: (kind, input log length, challenges, output, tree)
        rng = np.random.default_rng(seed + 1)
        self.rounds = []
        cur = log_len
        for i in range(n_folds):
            interleaved = i == 0 and log_batch > 0
            n_ch = log_batch if interleaved else arity
            ch = np.empty((n_ch, 2), dtype=np.uint64)
            for j in range(n_ch):
                ch[j] = rng.integers(0, 2**64, size=2, dtype=np.uint64)
            out_len = cur if interleaved else cur - arity
            out = torch.empty((1 << out_len, 2), dtype=torch.int64, device=d)
            tree = torch.empty(((2 << (out_len - arity)) - 1, 32), dtype=torch.uint8, device=d)
            self.rounds.append(("interleaved" if interleaved else "codeword", cur, ch, out, tree))
            cur = out_len

    def challenges(self, i: int) -> list[int]:
        return [int(c[0]) | (int(c[1]) << 64) for c in self.rounds[i][2]]

    def run(self, stream=None, marks=None) -> None:
        """One run on `stream`.  With `marks` (a list), CUDA events are recorded on the stream
        after the encode, after its commit and after each fold round (the encode and the commit
        are then issued as their two entry points, which is what commit_interleaved runs)."""
        L = lib()
        st = stream or self.torch.cuda.current_stream()
        s = st.cuda_stream

        def mark():
            if marks is not None:
                e = self.torch.cuda.Event(enable_timing=True)
                e.record(st)
                marks.append(e)

        mark()
        if marks is None:
            check(L.binius_fri_commit_interleaved(self.ntt.handle, self.message.data_ptr(),
                                                  self.log_dim, self.log_inv_rate,
                                                  self.log_batch, self.codeword.data_ptr(),
                                                  self.nodes.data_ptr(), None, s))
        else:
            check(L.binius_rs_encode_batch(self.ntt.handle, self.message.data_ptr(),
                                           self.log_dim, self.log_inv_rate, self.log_batch,
                                           self.codeword.data_ptr(), s))
            mark()
            check(L.binius_merkle_commit(self.codeword.data_ptr(), self.log_len, self.log_batch,
                                         self.nodes.data_ptr(), s))
            mark()
        src = self.codeword
        for kind, cur, ch, out, tree in self.rounds:
            chp = ch.ctypes.data_as(ctypes.c_void_p)
            if kind == "interleaved":
                check(L.binius_fri_fold_interleaved(src.data_ptr(), cur, self.log_batch, chp,
                                                    out.data_ptr(), s))
                out_len = cur
            else:
                check(L.binius_fri_fold_codeword(self.ntt.handle, src.data_ptr(), cur, chp,
                                                 self.arity, out.data_ptr(), s))
                out_len = cur - self.arity
            check(L.binius_merkle_commit(out.data_ptr(), out_len - self.arity, self.arity,
                                         tree.data_ptr(), s))
            mark()
            src = out

    # ---- work counters of one run

    def encode_bytes(self) -> int:
        """Message read, codeword written."""
        return 16 * (1 << (self.log_dim + self.log_batch)) + 16 * (1 << (self.log_len +
                                                                         self.log_batch))

    def merkle_bytes(self) -> int:
        """Codeword read by the leaf hashing, tree written."""
        return 16 * (1 << (self.log_len + self.log_batch)) + 32 * ((2 << self.log_len) - 1)

    def encode_commit_bytes(self) -> int:
        return self.encode_bytes() + self.merkle_bytes()

    def merkle_compressions(self) -> int:
        return leaf_compressions(self.log_len, 16 << self.log_batch)

    def algorithmic_bytes(self) -> int:
        total = self.encode_commit_bytes()
        for kind, cur, ch, out, tree in self.rounds:
            n_in = 1 << (cur + (self.log_batch if kind == "interleaved" else 0))
            n_out = out.shape[0]
            # fold: read input, write output; commit: read output, write tree
            total += 16 * n_in + 32 * n_out + 32 * tree.shape[0]
        return total

    def ntt_gf_mults(self) -> int:
        return (self.log_len - self.log_inv_rate) * (1 << (self.log_len + self.log_batch - 1))

    def gf_mults(self) -> int:
        total = self.ntt_gf_mults()
        for kind, cur, ch, out, tree in self.rounds:
            if kind == "interleaved":
                total += 1 << (cur + self.log_batch)  # one eq-weighted product per input symbol
            else:
                # fold_pair: one twiddle and one challenge product per pair, over `arity` rounds
                total += sum(2 * (1 << (cur - 1 - k)) for k in range(self.arity))
        return total

    def sha256_compressions(self) -> int:
        total = self.merkle_compressions()
        for kind, cur, ch, out, tree in self.rounds:
            total += leaf_compressions(tree.shape[0].bit_length() - 1, 16 << self.arity)
        return total

    def release(self) -> None:
        """Drops the device buffers (the harness of a large point holds tens of GiB)."""
        self.message = self.codeword = self.nodes = None
        self.rounds = []
        self.ntt = None
