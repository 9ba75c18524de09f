"""Pins the CPU oracle against the reference's own known-answer tests and independent restatements.

Every check here runs on the CPU.  Sources of truth:
  * GHASH multiplication KATs: verifier/field/src/ghash.rs:798-865 (test_ghash_mul),
    mul_x / mul_inv_x: ghash.rs:872-925, AES->GHASH homomorphism: ghash.rs:928-935 and the first
    entries of the embedding table, ghash.rs:520-530.
  * SHA-256: FIPS 180-4 through Python's hashlib; the Binius node compression
    (verifier/verifier/src/hash/compress.rs:32-57) through a pure-Python compression function
    that is itself checked against hashlib.
  * NTT: evaluation semantics of verifier/math/src/ntt/tests_evaluation.rs:244-295 (forward
    transform == evaluation of the novel-basis polynomial on the subspace), recomputed in pure
    Python for the standard basis and for the basis [5, 7, 22, 95].
  * RS encode: reed_solomon.rs:229-280 (encode_batch == NTT of the zero-padded, bit-reversed
    message).
  * FRI: fold∘encode commutes (prover/prover/src/fri/fold.rs:334-369) and the parameter KATs of
    verifier/verifier/src/fri/common.rs:225-247.
"""
import hashlib

import numpy as np
import pytest

import gf_py
import oracle as orc


# ---------------------------------------------------------------- field

GHASH_KATS = [
    (1, 1, 1),
    (1, 2, 2),
    (1, 1297182698762987, 1297182698762987),
    (2, 2, 4),
    (2, 3, 6),
    (3, 3, 5),
    (1 << 127, 2, 0b10000111),
    ((1 << 127) + 1, 2, 0b10000101),
    (3 << 126, 2, 0b10000111 + (1 << 127)),
    (1 << 127, 4, 0b10000111 << 1),
    (1 << 127, 1 << 122, (0b00000111 << 121) + 0b10000111),
]


@pytest.mark.parametrize("a,b,c", GHASH_KATS)
def test_ghash_mul_kat(a, b, c):
    assert orc.gf_mul(a, b) == c
    assert orc.gf_mul(a, b, portable=True) == c
    assert gf_py.mul(a, b) == c


def test_ghash_mul_random_three_ways():
    rng = np.random.default_rng(1)
    for _ in range(200):
        a = int(rng.integers(0, 1 << 63)) << 65 | int(rng.integers(0, 1 << 63))
        b = int(rng.integers(0, 1 << 63)) << 64 | int(rng.integers(0, 1 << 63)) << 1
        c = gf_py.mul(a, b)
        assert orc.gf_mul(a, b) == c
        assert orc.gf_mul(a, b, portable=True) == c


MUL_X_CASES = [0x0, 0x1, 0x2, 0x3, 1 << 127, 1 << 126, (1 << 128) - 1, 0x87,
               0x21ac73a21d46a21badd6747bcdfc5d4d]


@pytest.mark.parametrize("v", MUL_X_CASES)
def test_mul_x_and_inverse(v):
    assert orc.gf_mul_x(v) == orc.gf_mul(v, 2)
    assert orc.gf_mul_inv_x(v) == orc.gf_mul(v, orc.gf_inv(2))


def test_inverse():
    rng = np.random.default_rng(2)
    for _ in range(20):
        a = int(rng.integers(1, 1 << 62)) << 66 | int(rng.integers(1, 1 << 62))
        assert orc.gf_mul(a, orc.gf_inv(a)) == 1
    assert orc.gf_inv(0) == 0


def test_multiplicative_generator_order():
    # BinaryField128bGhash::MULTIPLICATIVE_GENERATOR (ghash.rs:502) generates the full group:
    # g^((2^128-1)/p) != 1 for every prime p | 2^128 - 1 (binary_field.rs tests).
    g = 0x494ef99794d5244f9152df59d87a9186
    order = (1 << 128) - 1
    for p in (3, 5, 17, 257, 641, 65537, 274177, 6700417, 67280421310721):
        assert order % p == 0
        assert gf_py.pow_(g, order // p) != 1
    assert gf_py.pow_(g, order) == 1


# First entries of `From<AESTowerField8b> for BinaryField128bGhash` (ghash.rs:520-530).
AES_TABLE_HEAD = [
    0x00000000000000000000000000000000,
    0x00000000000000000000000000000001,
    0x0dcb364640a222fe6b8330483c2e9849,
    0x0dcb364640a222fe6b8330483c2e9848,
    0x3d5bd35c94646a247573da4a5f7710ed,
    0x3d5bd35c94646a247573da4a5f7710ec,
    0x3090e51ad4c648da1ef0ea02635988a4,
    0x3090e51ad4c648da1ef0ea02635988a5,
]


def test_aes_embedding_table():
    table = orc.aes_to_ghash_table()
    assert table[: len(AES_TABLE_HEAD)] == AES_TABLE_HEAD
    rng = np.random.default_rng(3)
    for _ in range(500):
        a, b = (int(x) for x in rng.integers(0, 256, size=2))
        assert table[orc.aes_mul(a, b)] == orc.gf_mul(table[a], table[b])
    # the image of the AES generator is a root of x^8 + x^4 + x^3 + x + 1
    g = table[2]
    acc = gf_py.pow_(g, 8) ^ gf_py.pow_(g, 4) ^ gf_py.pow_(g, 3) ^ g ^ 1
    assert acc == 0


# ---------------------------------------------------------------- hashing

@pytest.mark.parametrize("n", [0, 1, 15, 16, 32, 55, 56, 63, 64, 65, 119, 120, 256, 1000])
def test_sha256_vs_hashlib(n):
    data = bytes((i * 37 + 11) & 0xFF for i in range(n))
    assert orc.sha256(data) == hashlib.sha256(data).digest()


def test_python_compress_matches_hashlib():
    msg = b"abc"
    block = msg + b"\x80" + b"\x00" * (55 - len(msg)) + (8 * len(msg)).to_bytes(8, "big")
    st = gf_py.sha256_compress(list(gf_py.SHA256_H0), block)
    assert b"".join(x.to_bytes(4, "big") for x in st) == hashlib.sha256(msg).digest()


def test_node_compression():
    d = hashlib.sha256(b"BINIUS SHA-256 COMPRESS").digest()
    iv = [int.from_bytes(d[4 * i: 4 * i + 4], "little") for i in range(8)]
    rng = np.random.default_rng(4)
    for _ in range(8):
        left = rng.integers(0, 256, 32, dtype=np.uint8).tobytes()
        right = rng.integers(0, 256, 32, dtype=np.uint8).tobytes()
        st = gf_py.sha256_compress(iv, left + right)
        expect = b"".join(x.to_bytes(4, "little") for x in st)
        assert orc.compress_node(left, right) == expect


def test_merkle_tree_shape():
    rng = np.random.default_rng(5)
    log_leaves, log_batch = 3, 2
    e = orc.random_elems(rng, 1 << (log_leaves + log_batch))
    nodes = orc.merkle_commit(e, log_leaves, log_batch)
    assert nodes.shape == ((1 << (log_leaves + 1)) - 1, 32)
    raw = e.tobytes()
    leaves = [hashlib.sha256(raw[64 * i: 64 * (i + 1)]).digest() for i in range(8)]
    assert [bytes(n) for n in nodes[:8]] == leaves
    l1 = [orc.compress_node(leaves[2 * i], leaves[2 * i + 1]) for i in range(4)]
    assert [bytes(n) for n in nodes[8:12]] == l1
    l2 = [orc.compress_node(l1[2 * i], l1[2 * i + 1]) for i in range(2)]
    assert [bytes(n) for n in nodes[12:14]] == l2
    assert bytes(nodes[14]) == orc.compress_node(l2[0], l2[1])


# ---------------------------------------------------------------- NTT

def _w_hat(domain_basis, i):
    """Normalized subspace polynomial of span(domain_basis[:i]) (tests_evaluation.rs:186-225)."""
    poly = [1]
    for a in gf_py.subspace_iter(domain_basis[:i]):
        poly = gf_py.poly_mul(poly, [a, 1])
    e = gf_py.poly_eval(poly, domain_basis[i])
    s = gf_py.inv(e)
    return [gf_py.mul(c, s) for c in poly]


def _ntt_eval_check(basis, seed):
    log_d = len(basis)
    tw = orc.domain_twiddles(log_d, basis=basis)
    w_hats = [_w_hat(basis, i) for i in range(log_d)]
    novel = [[1]]
    for i in range(log_d):
        novel += [gf_py.poly_mul(p, w_hats[i]) for p in novel]
    rng = np.random.default_rng(seed)
    coeffs = orc.random_elems(rng, 1 << log_d)
    poly = [0] * (1 << log_d)
    for j, b in enumerate(novel):
        c = orc.to_int(coeffs[j])
        for k, bk in enumerate(b):
            poly[k] ^= gf_py.mul(bk, c)
    evals = [gf_py.poly_eval(poly, a) for a in gf_py.subspace_iter(basis)]
    out = orc.ntt_forward(tw, log_d, coeffs)
    assert [orc.to_int(x) for x in out] == evals
    back = orc.ntt_forward(tw, log_d, out, inverse=True)
    assert np.array_equal(back, coeffs)


def test_ntt_evaluation_standard_basis():
    _ntt_eval_check([1 << i for i in range(6)], seed=6)


def test_ntt_evaluation_nonstandard_basis():
    _ntt_eval_check([5, 7, 22, 95], seed=7)


def test_twiddle_table_layout():
    dim = 6
    tw = orc.domain_twiddles(dim)
    assert tw.shape[0] == (1 << dim) - 1
    # layer 0 has a single zero twiddle; each layer's table is a subset-sum expansion
    assert orc.to_int(tw[0]) == 0
    for layer in range(1, dim):
        base = (1 << layer) - 1
        t = [orc.to_int(tw[base + j]) for j in range(1 << layer)]
        for j in range(1 << layer):
            acc = 0
            for k in range(layer):
                if (j >> k) & 1:
                    acc ^= t[1 << k]
            assert t[j] == acc


def rs_basis_from_standard_domain(log_code_len: int, log_batch: int) -> list[int]:
    """Basis of FRIParams' RS subspace: row `log_batch` of the normalized subspace evaluations of
    the standard domain of dim log_code_len (verify.rs:85-97, GenericOnTheFly::subspace)."""
    tw = orc.domain_twiddles(log_code_len)
    n = log_code_len - log_batch
    layer = log_code_len - 1 - log_batch
    base = (1 << layer) - 1
    return [1] + [orc.to_int(tw[base + (1 << k)]) for k in range(n - 1)]


@pytest.mark.parametrize("log_code_len,log_batch", [(6, 0), (8, 2), (10, 4)])
def test_rs_domain_equals_tail_of_standard_domain(log_code_len, log_batch):
    basis = rs_basis_from_standard_domain(log_code_len, log_batch)
    n = len(basis)
    tw_rs = orc.domain_twiddles(n, basis=basis)
    tw_std = orc.domain_twiddles(log_code_len)
    assert np.array_equal(tw_rs, tw_std[: (1 << n) - 1])


def _reverse_bits(x, bits):
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


@pytest.mark.parametrize("log_dim,log_inv_rate,log_batch", [(4, 2, 0), (6, 2, 1), (8, 3, 2), (1, 2, 0)])
def test_rs_encode_matches_padded_ntt(log_dim, log_inv_rate, log_batch):
    rng = np.random.default_rng(8)
    n = log_dim + log_inv_rate
    tw = orc.domain_twiddles(n)
    msg = orc.random_elems(rng, 1 << (log_dim + log_batch))
    cw = orc.rs_encode_batch(tw, n, msg, log_dim, log_inv_rate, log_batch)
    ref = orc.elems(1 << (n + log_batch))
    bits = log_dim + log_batch
    for i in range(msg.shape[0]):
        ref[_reverse_bits(i, bits)] = msg[i]
    ref = orc.ntt_forward(tw, n, ref, 0, log_batch)
    assert np.array_equal(cw, ref)


# ---------------------------------------------------------------- FRI

def _fold_cols(msg, query, log_dim, arity):
    # fold_cols (verifier/math/src/fold.rs:42-66): row-major matrix times vector,
    # out[i] = sum_j msg[i * 2^arity + j] * query[j]
    out = []
    for i in range(1 << log_dim):
        acc = 0
        for j in range(1 << arity):
            acc ^= orc.gf_mul(orc.to_int(msg[(i << arity) + j]), orc.to_int(query[j]))
        out.append(acc)
    return orc.from_ints(out)


@pytest.mark.parametrize("log_dim,arity", [(0, 0), (0, 1), (3, 2), (5, 3), (7, 1)])
def test_fri_fold_commutes_with_encode(log_dim, arity):
    rng = np.random.default_rng(9)
    tw = orc.domain_twiddles(12)
    msg = orc.random_elems(rng, 1 << (log_dim + arity))
    challenges = orc.random_elems(rng, arity)
    query = orc.eq_ind_partial_eval(challenges)
    folded_msg = _fold_cols(msg, query, log_dim, arity)
    codeword = orc.ntt_forward(tw, 12, msg)
    folded_cw = orc.fri_fold_codeword(tw, 12, codeword, log_dim + arity, challenges)
    enc = orc.ntt_forward(tw, 12, folded_msg)
    assert np.array_equal(folded_cw, enc)


def test_eq_tensor_bit_order():
    r = [0x1234, 0xabcdef]
    t = orc.eq_ind_partial_eval(orc.from_ints(r))
    one = 1
    expect = [
        gf_py.mul(one ^ r[0], one ^ r[1]),
        gf_py.mul(r[0], one ^ r[1]),
        gf_py.mul(one ^ r[0], r[1]),
        gf_py.mul(r[0], r[1]),
    ]
    assert [orc.to_int(x) for x in t] == expect


def test_fold_interleaved_is_inner_product():
    rng = np.random.default_rng(10)
    log_len, log_batch = 4, 3
    cw = orc.random_elems(rng, 1 << (log_len + log_batch))
    ch = orc.random_elems(rng, log_batch)
    tensor = orc.eq_ind_partial_eval(ch)
    out = orc.fri_fold_interleaved(cw, log_len, log_batch, ch)
    for i in range(1 << log_len):
        acc = 0
        for j in range(1 << log_batch):
            acc ^= gf_py.mul(orc.to_int(cw[(i << log_batch) + j]), orc.to_int(tensor[j]))
        assert orc.to_int(out[i]) == acc


def test_fri_param_kats():
    assert orc.calculate_n_test_queries(96, 1) == 232
    assert orc.calculate_n_test_queries(96, 2) == 142
    for n in range(22, 35):
        assert orc.estimate_optimal_arity(n, 256, 128) == 4
    for n in range(22, 28):
        assert orc.estimate_optimal_arity(n, 1024, 128) == 6
