"""GPU parity: every CUDA entry point against the CPU oracle, bit-exact, on seeded inputs.

Small and medium sizes are compared element by element; the full kernel-level workload size is
checked through size-independent properties (inverse-after-forward identity, linearity of the
encoder, fold-commutes-with-encode) plus a direct oracle comparison.
"""
import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402


def rng(seed):
    return np.random.default_rng(seed)


def ints(a):
    return [orc.to_int(x) for x in a]


def test_gf_mul_batch_matches_oracle_and_kats():
    r = rng(1)
    n = 1 << 16
    a = orc.random_elems(r, n)
    b = orc.random_elems(r, n)
    # include the reference KAT operands (ghash.rs:798-865)
    kats = [(1, 1), (1, 2), (2, 2), (2, 3), (3, 3), (1 << 127, 2), ((1 << 127) + 1, 2),
            (3 << 126, 2), (1 << 127, 4), (1 << 127, 1 << 122), (0, 5), ((1 << 128) - 1, (1 << 128) - 1)]
    for i, (x, y) in enumerate(kats):
        a[i], b[i] = orc.from_int(x), orc.from_int(y)
    out = bg.to_host(bg.gf_mul_batch(bg.to_device(a), bg.to_device(b)))
    ref = orc.gf_mul_vec(a, b)
    assert np.array_equal(out, ref)
    assert orc.to_int(out[5]) == 0b10000111
    assert orc.to_int(out[6]) == 0b10000101


@pytest.mark.parametrize("log_d,skip_early,skip_late", [
    (1, 0, 0), (4, 0, 0), (6, 1, 2), (10, 0, 0), (12, 3, 4), (13, 0, 13), (13, 13, 0),
    (16, 2, 0), (17, 1, 4), (20, 0, 6),
])
def test_ntt_forward_inverse_vs_oracle(log_d, skip_early, skip_late):
    r = rng(100 + log_d)
    log_domain = log_d + 1
    ntt = bg.AdditiveNTT(log_domain)
    tw = orc.domain_twiddles(log_domain)
    data = orc.random_elems(r, 1 << log_d)
    d = bg.to_device(data)
    ntt.forward_transform(d, skip_early, skip_late)
    ref = orc.ntt_forward(tw, log_domain, data, skip_early, skip_late)
    assert np.array_equal(bg.to_host(d), ref)
    ntt.inverse_transform(d, skip_early, skip_late)
    assert np.array_equal(bg.to_host(d), data)


def test_ntt_nonstandard_basis_and_twiddles():
    r = rng(7)
    basis = [5, 7, 22, 95, 1 << 100 | 3, 0x1234567890abcdef]
    ntt = bg.AdditiveNTT(len(basis), basis=basis)
    tw_ref = orc.domain_twiddles(len(basis), basis=basis)
    assert np.array_equal(bg.to_host(ntt.twiddles()), tw_ref)
    data = orc.random_elems(r, 1 << len(basis))
    d = bg.to_device(data)
    ntt.forward_transform(d)
    assert np.array_equal(bg.to_host(d), orc.ntt_forward(tw_ref, len(basis), data))


def test_ntt_domain_too_small_is_argument_error():
    ntt = bg.AdditiveNTT(4)
    d = bg.to_device(orc.elems(1 << 6))
    with pytest.raises(bg.ArgumentError):
        ntt.forward_transform(d, 0, 0)
    with pytest.raises(bg.ArgumentError):
        ntt.forward_transform(d, 4, 3)


@pytest.mark.parametrize("log_dim,log_inv_rate,log_batch", [
    (0, 1, 0), (1, 2, 0), (4, 2, 0), (6, 2, 1), (8, 3, 2), (3, 0, 2), (10, 1, 4), (12, 2, 6),
    (15, 1, 4), (9, 1, 0),
])
def test_rs_encode_vs_oracle(log_dim, log_inv_rate, log_batch):
    r = rng(200 + log_dim)
    n = log_dim + log_inv_rate
    basis = bg.standard_domain_rs_basis(n + log_batch, log_batch) if n >= 1 else None
    dom = max(n, 1)
    ntt = bg.AdditiveNTT(dom, basis=basis if n >= 1 else None)
    tw = orc.domain_twiddles(dom, basis=basis if n >= 1 else None)
    msg = orc.random_elems(r, 1 << (log_dim + log_batch))
    code = bg.ReedSolomonCode(log_dim, log_inv_rate)
    out = code.encode_batch(ntt, bg.to_device(msg), log_batch)
    ref = orc.rs_encode_batch(tw, dom, msg, log_dim, log_inv_rate, log_batch)
    assert np.array_equal(bg.to_host(out), ref)


@pytest.mark.parametrize("log_leaves,log_batch", [
    (0, 0), (0, 4), (1, 1), (3, 2), (7, 0), (8, 4), (9, 1), (12, 4), (13, 6), (17, 0), (18, 4),
])
def test_merkle_commit_vs_oracle(log_leaves, log_batch):
    r = rng(300 + log_leaves)
    elems = orc.random_elems(r, 1 << (log_leaves + log_batch))
    root, committed = bg.BinaryMerkleTreeProver().commit(bg.to_device(elems), 1 << log_batch)
    ref = orc.merkle_commit(elems, log_leaves, log_batch)
    assert np.array_equal(committed.nodes.cpu().numpy(), ref)
    assert root == bytes(ref[-1])
    # MerkleTreeProver::layer at every depth: the flat node slice of that layer
    for depth in range(log_leaves + 1):
        start = (2 << log_leaves) - (2 << depth)
        assert committed.layer(depth) == [bytes(x) for x in ref[start:start + (1 << depth)]]
    with pytest.raises(bg.ArgumentError, match="IncorrectLayerDepth"):
        committed.layer(log_leaves + 1)
    if log_leaves >= 3:
        idx = (1 << log_leaves) - 3
        br = committed.branch(idx, 1)
        L = log_leaves
        for j, node in enumerate(br):
            off = (1 << (L + 1)) - (1 << (L + 1 - j))
            assert node == bytes(ref[off + ((idx >> j) ^ 1)])


@pytest.mark.parametrize("log_len,log_batch", [(0, 1), (3, 2), (10, 4), (12, 6), (16, 4), (9, 8)])
def test_fold_interleaved_vs_oracle(log_len, log_batch):
    r = rng(400 + log_len)
    cw = orc.random_elems(r, 1 << (log_len + log_batch))
    ch = orc.random_elems(r, log_batch)
    out = bg.fold_interleaved(bg.to_device(cw), ints(ch), log_len, log_batch)
    assert np.array_equal(bg.to_host(out), orc.fri_fold_interleaved(cw, log_len, log_batch, ch))


@pytest.mark.parametrize("log_len,n", [(1, 1), (4, 4), (10, 2), (12, 4), (14, 3), (13, 5), (16, 8),
                                        (9, 0), (17, 4)])
def test_fold_codeword_vs_oracle(log_len, n):
    r = rng(500 + log_len)
    log_domain = log_len + 2
    ntt = bg.AdditiveNTT(log_domain)
    tw = orc.domain_twiddles(log_domain)
    cw = orc.random_elems(r, 1 << log_len)
    ch = orc.random_elems(r, n)
    out = bg.fold_codeword(ntt, bg.to_device(cw), ints(ch), log_len)
    assert np.array_equal(bg.to_host(out), orc.fri_fold_codeword(tw, log_domain, cw, log_len, ch))


def test_commit_interleaved_c3_shape_vs_oracle():
    """The commit phase of the 2^20-word prove: 2^19 elements, R=1, batch 2^4, RS dim 2^15."""
    r = rng(600)
    p = bg.FRIParams.choose_with_constant_fold_arity(19, 96, 1, 4)
    n = p.rs_code.log_len()
    basis = bg.standard_domain_rs_basis(n + p.log_batch_size, p.log_batch_size)
    ntt = bg.AdditiveNTT(n, basis=basis)
    msg = orc.random_elems(r, 1 << p.log_msg_len())
    out = bg.commit_interleaved(p, ntt, bg.BinaryMerkleTreeProver(), bg.to_device(msg))
    tw = orc.domain_twiddles(n, basis=basis)
    cw_ref = orc.rs_encode_batch(tw, n, msg, p.rs_code.log_dim, 1, p.log_batch_size)
    assert np.array_equal(bg.to_host(out.codeword), cw_ref)
    nodes_ref = orc.merkle_commit(cw_ref, n, p.log_batch_size)
    assert out.commitment == bytes(nodes_ref[-1])
    assert np.array_equal(out.committed.nodes.cpu().numpy(), nodes_ref)


def test_full_size_properties():
    """log_len 20 per column, R=1, 16 columns (a 256 MiB codeword): encode linearity, fold∘encode
    commutation through the GPU folds, and NTT inverse∘forward identity."""
    log_dim, R, b = 19, 1, 4
    n = log_dim + R
    ntt = bg.AdditiveNTT(n)
    gen = torch.Generator(device="cuda").manual_seed(5)
    m1 = torch.randint(-2**63, 2**63 - 1, (1 << (log_dim + b), 2), dtype=torch.int64,
                       device="cuda", generator=gen)
    m2 = torch.randint(-2**63, 2**63 - 1, (1 << (log_dim + b), 2), dtype=torch.int64,
                       device="cuda", generator=gen)
    code = bg.ReedSolomonCode(log_dim, R)
    c1 = code.encode_batch(ntt, m1, b)
    c2 = code.encode_batch(ntt, m2, b)
    c12 = code.encode_batch(ntt, m1 ^ m2, b)
    assert torch.equal(c1 ^ c2, c12)
    # fold_interleaved(encode(m)) == encode(fold_rows(m)) where the message rows are combined with
    # the same eq tensor over the bit-reversed batch index.
    ch = [0x1234567 + 99 * i for i in range(b)]
    folded = bg.fold_interleaved(c1, ch, n, b)
    # inverse NTT (skip_early=R) recovers the bit-reversed single-column message in the first half
    tmp = folded.clone()
    ntt.inverse_transform(tmp, R, 0)
    assert torch.equal(tmp[: 1 << log_dim], tmp[1 << log_dim:])
    # NTT identity at full size
    d = m1.clone()
    ntt.forward_transform(d.view(-1, 2)[: 1 << n], 0, 0)
    ntt.inverse_transform(d.view(-1, 2)[: 1 << n], 0, 0)
    assert torch.equal(d, m1)
