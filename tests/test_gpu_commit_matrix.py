"""The kernel-level FRI commit workload at every point of its size matrix, bit-exact against the
oracle: RS encode of seeded uniform GF(2^128) messages (log_len 20 / 22 / 24 per column,
log_inv_rate 1 / 2, 1 / 16 / 64 interleaved columns), the SHA-256 Merkle commit of the codeword
and 3 FRI fold rounds, each with its own commit.

Follows ReedSolomonCode::encode_batch (verifier/math/src/reed_solomon.rs:128-201),
fri::commit_interleaved (prover/prover/src/fri/commit.rs:25-75), fold_interleaved /
fold_codeword (prover/prover/src/fri/fold.rs:260-318).

Codewords of up to 2^24 symbols are compared whole with the oracle's (codeword, every tree node,
every fold output and tree).  Larger ones (up to 2^30 symbols, a 16 GiB codeword) are checked on
samples the oracle computes exactly: whole columns (encode_batch bit-reverses the whole message
index, so codeword column c, the symbols whose low log_batch index bits are c, is the
single-column encoding of the contiguous message block rev(c)), leaf digests (SHA-256 of a codeword row), node compressions of every
tree layer from the GPU's children, the root, and fold outputs of sampled rows; the later fold
rounds are compared whole.
"""
import hashlib

import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402
from binius64_b200.commit_phase import CommitPhase  # noqa: E402

POINTS = [(L, R, b) for L in (20, 22, 24) for R in (1, 2) for b in (0, 4, 6)]
FULL_LIMIT = 24  # log2 of the largest codeword compared whole


def host(t):
    return t.contiguous().cpu().numpy().view(np.uint64).reshape(-1, 2)


def rev_bits(x, n):
    return int(format(x, f"0{n}b")[::-1], 2) if n else 0


def layer_offset(log_leaves, j):
    return (1 << (log_leaves + 1)) - (1 << (log_leaves + 1 - j))


def check_tree_samples(nodes, log_leaves, rng, leaf_rows=None, leaf_digest=None):
    """Leaf digests at sampled leaves (given leaf_digest(idx) -> list of digests) and, at every
    inner layer, node = compress(left child, right child) of the GPU's own children."""
    n_leaves = 1 << log_leaves
    idx = np.unique(np.concatenate([[0, n_leaves - 1], rng.integers(0, n_leaves, 48)]))
    got = nodes[torch.from_numpy(idx).to(nodes.device)].cpu().numpy()
    want = leaf_digest(idx)
    for i, g, w in zip(idx, got, want):
        assert bytes(g) == w, f"leaf {i}"
    for j in range(1, log_leaves + 1):
        size = 1 << (log_leaves - j)
        ks = np.unique(np.concatenate([[0, size - 1], rng.integers(0, size, 8)]))
        off, child = layer_offset(log_leaves, j), layer_offset(log_leaves, j - 1)
        sel = np.concatenate([off + ks, child + 2 * ks, child + 2 * ks + 1])
        v = nodes[torch.from_numpy(sel).to(nodes.device)].cpu().numpy()
        m = len(ks)
        for q in range(m):
            assert bytes(v[q]) == orc.compress_node(bytes(v[m + q]), bytes(v[2 * m + q])), \
                f"layer {j} node {ks[q]}"


@pytest.mark.parametrize("log_len,log_inv_rate,log_batch", POINTS)
def test_commit_matrix_point_vs_oracle(log_len, log_inv_rate, log_batch):
    L, R, b = log_len, log_inv_rate, log_batch
    seed = 7000 + 100 * L + 10 * R + b
    ph = CommitPhase(L, R, b, seed=seed)
    ph.run()
    torch.cuda.synchronize()
    rng = np.random.default_rng(seed)
    tw = orc.domain_twiddles(L, basis=ph.basis)
    log_dim = L - R
    full = L + b <= FULL_LIMIT

    cw_ref = None
    if full:
        cw_ref = orc.rs_encode_batch(tw, L, host(ph.message), log_dim, R, b)
        assert np.array_equal(host(ph.codeword), cw_ref), "codeword"
        nodes_ref = orc.merkle_commit(cw_ref, L, b)
        assert np.array_equal(ph.nodes.cpu().numpy(), nodes_ref), "tree"
    else:
        cw3 = ph.codeword.view(1 << L, 1 << b, 2)
        cols = sorted({0, min(1, (1 << b) - 1), (1 << b) - 1, int(rng.integers(0, 1 << b))})
        for c in cols:
            blk = rev_bits(c, b)
            m = ph.message[blk << log_dim:(blk + 1) << log_dim]
            ref = orc.rs_encode_batch(tw, L, host(m), log_dim, R, 0)
            assert np.array_equal(host(cw3[:, c, :]), ref), f"column {c}"

        def leaf_digest(idx):
            rows = cw3[torch.from_numpy(idx).to(cw3.device)].cpu().numpy()
            return [hashlib.sha256(r.tobytes()).digest() for r in rows]

        check_tree_samples(ph.nodes, L, rng, leaf_digest=leaf_digest)

    src_ref = cw_ref
    for i, (kind, cur, _, out, tree) in enumerate(ph.rounds):
        ch = orc.from_ints(ph.challenges(i))
        if kind == "interleaved":
            if src_ref is not None:
                ref = orc.fri_fold_interleaved(src_ref, cur, b, ch)
                assert np.array_equal(host(out), ref), f"round {i}"
            else:  # sampled rows: a fold output depends on its own row alone
                rows = np.unique(np.concatenate([[0, (1 << cur) - 1],
                                                 rng.integers(0, 1 << cur, 62)]))
                rows = rows[: 1 << int(np.log2(len(rows)))]
                cw3 = ph.codeword.view(1 << cur, 1 << b, 2)
                sub = host(cw3[torch.from_numpy(rows).to(cw3.device)])
                ref = orc.fri_fold_interleaved(sub, int(np.log2(len(rows))), b, ch)
                got = host(out)[rows]
                assert np.array_equal(got, ref), f"round {i} rows"
            out_len = cur
        else:
            src = host(ph.codeword if i == 0 else ph.rounds[i - 1][3]) if src_ref is None \
                else src_ref
            ref = orc.fri_fold_codeword(tw, L, src, cur, ch)
            assert np.array_equal(host(out), ref), f"round {i}"
            out_len = cur - ph.arity
        ref_out = host(out)
        tree_ref = orc.merkle_commit(ref_out, out_len - ph.arity, ph.arity)
        assert np.array_equal(tree.cpu().numpy(), tree_ref), f"round {i} tree"
        src_ref = ref_out
    ph.release()
    torch.cuda.empty_cache()
