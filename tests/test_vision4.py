"""Vision-4 over GF(2^128) (verifier/verifier/src/hash/vision_4): the oracle pinned on the
reference's own known answers (tests/golden/vision4_kat.json, made by make_vision4_fixtures.py):
the permutation outputs of test_permutation, the ROUND_CONSTANTS table that compute_round_constants
must reproduce, and the B_INV_COEFFS linearized polynomial that B^-1 must equal; then the sponge
and MMO structure of the digest and compression, and the Merkle layout.  Host code only."""
import json
import os

import numpy as np
import pytest

import oracle as orc

KAT = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "vision4_kat.json")))
M128 = (1 << 128) - 1


def _ints(hexes):
    return [int(h, 16) for h in hexes]


@pytest.mark.parametrize("case", range(len(KAT["permutation"])))
def test_permutation_known_answers(case):
    c = KAT["permutation"][case]
    assert orc.vision4_permutation(_ints(c["input"])) == _ints(c["output"])


def test_round_constants_match_reference_table():
    rc, b_inv0 = orc.vision4_constants()
    assert rc == [_ints(r) for r in KAT["round_constants"]]
    assert b_inv0 == int(KAT["b_inv_coeffs"][0], 16)


def _square(x):
    return orc.gf_mul(x, x)


def test_b_inverse_is_reference_polynomial():
    """L^-1(x) = sum_i B_INV_COEFFS[i+1] x^(2^i) (constants.rs evaluate_b_inv_linear)."""
    coeffs = _ints(KAT["b_inv_coeffs"])
    rng = np.random.default_rng(4)
    for _ in range(4):
        x = int.from_bytes(rng.bytes(16), "little")
        acc, p = 0, x
        for i in range(128):
            acc ^= orc.gf_mul(coeffs[i + 1], p)
            p = _square(p)
        assert orc.vision4_map(1, x) == acc
        assert orc.vision4_map(3, orc.vision4_map(2, x)) == x  # B^-1(B(x)) = x
        assert orc.vision4_map(1, orc.vision4_map(0, x)) == x


def _state_bytes(s):
    return b"".join(v.to_bytes(16, "little") for v in s)


def test_compression_is_mmo():
    rng = np.random.default_rng(5)
    left, right = rng.bytes(32), rng.bytes(32)
    x = [int.from_bytes((left + right)[16 * i:16 * i + 16], "little") for i in range(4)]
    p = orc.vision4_permutation(x)
    assert orc.vision4_compress(left, right) == _state_bytes([p[0] ^ x[0], p[1] ^ x[1]])


def _sponge(data: bytes) -> bytes:
    """digest.rs: absorb 32-byte blocks by overwriting state[0..2], pad 0x80 .. 0x01."""
    s = [0, 0, 0, 0]
    full, rest = len(data) // 32, len(data) % 32
    blocks = [data[32 * i:32 * i + 32] for i in range(full)]
    last = bytearray(32)
    last[:rest] = data[32 * full:]
    last[rest] |= 0x80
    last[31] |= 0x01
    blocks.append(bytes(last))
    for b in blocks:
        s[0] = int.from_bytes(b[:16], "little")
        s[1] = int.from_bytes(b[16:], "little")
        s = orc.vision4_permutation(s)
    return _state_bytes(s[:2])


@pytest.mark.parametrize("n", [0, 1, 16, 31, 32, 33, 64, 256, 1000])
def test_digest_sponge_and_split_invariance(n):
    data = np.random.default_rng(n).bytes(n)
    d = orc.vision4_digest(data)
    assert d == _sponge(data)
    for splits in ([n // 3, n // 2], [1 % (n + 1)], [n // 2, n // 2, n]):
        assert orc.vision4_digest(data, splits) == d


@pytest.mark.parametrize("log_leaves,log_batch", [(0, 4), (1, 0), (3, 1), (5, 4)])
def test_merkle_layout(log_leaves, log_batch):
    rng = np.random.default_rng(log_leaves * 8 + log_batch)
    el = orc.random_elems(rng, 1 << (log_leaves + log_batch))
    nodes = orc.vision4_merkle_commit(el, log_leaves, log_batch)
    raw = el.tobytes()
    leaf = 16 << log_batch
    for i in range(1 << log_leaves):
        assert nodes[i].tobytes() == orc.vision4_digest(raw[i * leaf:(i + 1) * leaf])
    prev, n = 0, 1 << log_leaves
    while n > 1:
        for i in range(n // 2):
            assert nodes[prev + n + i].tobytes() == orc.vision4_compress(
                nodes[prev + 2 * i].tobytes(), nodes[prev + 2 * i + 1].tobytes())
        prev, n = prev + n, n // 2
