"""The shift reduction's KeyCollection (prover/prover/src/protocols/shift/key_collection.rs):
build_key_collection + KeyCollection::serialize v1 from the library's host builder, byte-identical
to the oracle's literal restatement, and the structure the reference's consumers rely on (one key
range per word tiling the key vector, each key's index range tiling the constraint indices, keys
unique within a word, indices ordered by operand).  Host code only."""
import json
import os
import struct

import pytest

import binius64_b200 as bg
import oracle as orc
from binius64_b200 import constraint_system as csm

FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "formats_v1.json")))


def parse_kc(data: bytes):
    """KeyCollection::deserialize (key_collection.rs:400-431), strict about trailing bytes."""
    pos = 0

    def u32():
        nonlocal pos
        (v,) = struct.unpack_from("<I", data, pos)
        pos += 4
        return v

    assert u32() == 1
    keys = []
    for _ in range(u32()):
        op, kid, start, end = struct.unpack_from("<BHII", data, pos)
        pos += 11
        keys.append((op, kid, start, end))
    ranges = [(u32(), u32()) for _ in range(u32())]
    cis = []
    for _ in range(u32()):
        operand, c = struct.unpack_from("<BI", data, pos)
        pos += 5
        cis.append((operand, c))
    assert pos == len(data)
    return keys, ranges, cis


def _occurrences(prep):
    """(word, operation, id, operand, constraint) for every operand term of the padded system."""
    out = []
    for op, csr, slots in ((0, prep.and_csr, (0, 1, 2)), (1, prep.mul_csr, (0, 1, 3, 2))):
        k = len(slots)
        n = (len(csr.offsets) - 1) // k
        for operand, slot in enumerate(slots):
            for c in range(n):
                g = c * k + slot
                for t in range(csr.offsets[g], csr.offsets[g + 1]):
                    kid = int(csr.variant[t]) * 64 + int(csr.amount[t])
                    out.append((int(csr.value_index[t]), op, kid, operand, c))
    return out


def _check_structure(data, prep, n_words):
    keys, ranges, cis = parse_kc(data)
    assert len(ranges) == n_words
    at = 0
    for w, (k0, k1) in enumerate(ranges):
        assert k0 == at and k1 >= k0
        at = k1
        ids = [(keys[k][0], keys[k][1]) for k in range(k0, k1)]
        assert len(set(ids)) == len(ids), "a key repeats within a word"
    assert at == len(keys)
    at = 0
    for op, kid, s, e in keys:
        assert s == at and e >= s and op in (0, 1) and kid < 512
        ops = [cis[x][0] for x in range(s, e)]
        assert ops == sorted(ops), "indices of a key not ordered by operand"
        at = e
    assert at == len(cis)
    # the multiset of terms is exactly the constraint system's
    got = sorted((w, keys[k][0], keys[k][1], cis[x][0], cis[x][1])
                 for w, (k0, k1) in enumerate(ranges) for k in range(k0, k1)
                 for x in range(keys[k][2], keys[k][3]))
    assert got == sorted(_occurrences(prep))


@pytest.mark.parametrize("log_words,n_and,n_mul,seed", [
    (4, 3, 1, 0),
    (8, 60, 1, 1),
    (10, 300, 5, 2),
    (12, 1500, 17, 3),
    (14, 6000, 200, 4),
])
def test_key_collection_matches_oracle(log_words, n_and, n_mul, seed):
    sc = csm.synthetic_circuit(log_words, n_and, n_mul, seed=seed)
    prep = sc.cs.prepared()
    got = bg.key_collection_from_cs_bytes(sc.cs.serialize())
    ref = orc.key_collection(prep.and_csr, prep.mul_csr, 1 << log_words)
    assert got == ref
    if log_words <= 12:
        _check_structure(got, prep, 1 << log_words)


def test_key_collection_of_reference_fixture():
    """The reference's serialized constraint system fixture (verifier/core/test_data)."""
    data = bytes.fromhex(FIX["constraint_system_v2"])
    cs = csm.ConstraintSystem.deserialize(data)
    prep = cs.prepared()
    n_words = cs.layout.committed_total_len
    got = bg.key_collection_from_cs_bytes(data)
    assert got == orc.key_collection(prep.and_csr, prep.mul_csr, n_words)
    _check_structure(got, prep, n_words)


def test_key_collection_2_20_words():
    """The 2^20-word shape (about 2^20 AND constraints): same bytes as the oracle."""
    sc = csm.synthetic_circuit(20, (1 << 20) - (1 << 16), 1, seed=20)
    prep = sc.cs.prepared()
    got = bg.key_collection_from_cs_bytes(sc.cs.serialize())
    assert got == orc.key_collection(prep.and_csr, prep.mul_csr, 1 << 20)


def test_key_collection_rejects_bad_constraint_system():
    data = bytearray(bytes.fromhex(FIX["constraint_system_v2"]))
    data[0] = 1
    with pytest.raises(bg.ArgumentError, match="version"):
        bg.key_collection_from_cs_bytes(bytes(data))
    with pytest.raises(bg.ArgumentError):
        bg.key_collection_from_cs_bytes(bytes.fromhex(FIX["constraint_system_v2"])[:-3])
