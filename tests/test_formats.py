"""Wire formats around a prove call, pinned on the reference's own serialization fixtures
(verifier/core/test_data, committed as tests/golden/formats_v1.json by make_format_fixtures.py)
and the properties its tests check (verifier/core/src/constraint_system.rs:1465-1880):
ConstraintSystem v2, ValuesData v1 and Proof v1 decode to the asserted contents, re-encode to the
same bytes, round-trip, and reject another version or truncated input.  Host code only."""
import json
import os

import numpy as np
import pytest

import binius64_b200 as bg
from binius64_b200 import constraint_system as csm

FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "formats_v1.json")))


def _b(name):
    return bytes.fromhex(FIX[name])


def test_constraint_system_v2_fixture():
    data = _b("constraint_system_v2")
    exp = FIX["expect"]["constraint_system_v2"]
    cs = csm.ConstraintSystem.deserialize(data)
    assert cs.layout.__dict__ == exp["layout"]
    assert cs.constants == exp["constants"]
    assert (len(cs.and_constraints), len(cs.mul_constraints)) == (exp["n_and"], exp["n_mul"])
    assert data[:4] == (2).to_bytes(4, "little")
    assert cs.serialize_lists() == data and cs.serialize() == data


def test_constraint_system_rejections():
    data = bytearray(_b("constraint_system_v2"))
    data[0] = 1
    with pytest.raises(ValueError, match="version"):
        csm.ConstraintSystem.deserialize(bytes(data))
    with pytest.raises(ValueError, match="NotEnoughBytes"):
        csm.ConstraintSystem.deserialize(_b("constraint_system_v2")[:-3])


def test_values_data_v1_fixture():
    data = _b("witness_v1")
    v = bg.ValuesData.deserialize(data)
    assert [int(x) for x in v.words] == FIX["expect"]["witness_v1"]["words"]
    assert data[:4] == (1).to_bytes(4, "little")
    assert v.serialize() == data


@pytest.mark.parametrize("n", [0, 1, 5, 1000])
def test_values_data_round_trip(n):
    words = np.random.default_rng(n).integers(0, 2**63, size=n, dtype=np.uint64) * np.uint64(2)
    enc = bg.ValuesData(words).serialize()
    assert len(enc) == 8 + 8 * n
    assert np.array_equal(bg.ValuesData.deserialize(enc).words, words)


def test_values_data_rejections():
    bad = bytearray(_b("witness_v1"))
    bad[0] = 2
    with pytest.raises(bg.ArgumentError, match="Witness::version"):
        bg.ValuesData.deserialize(bytes(bad))
    with pytest.raises(bg.ArgumentError, match="NotEnoughBytes"):
        bg.ValuesData.deserialize(_b("witness_v1")[:-1])
    with pytest.raises(bg.ArgumentError, match="NotEnoughBytes"):
        bg.ValuesData.deserialize(b"\x01\x00")


def test_proof_v1_fixture():
    data = _b("proof_v1")
    exp = FIX["expect"]["proof_v1"]
    p = bg.Proof.deserialize(data)
    assert p.challenger_type == exp["challenger"] == bg.STD_CHALLENGER
    assert p.data.hex() == exp["data"] and len(p.data) == 24
    assert data[:4] == (1).to_bytes(4, "little")
    assert p.serialize() == data


@pytest.mark.parametrize("n,ch", [(0, bg.STD_CHALLENGER), (24, "Other"), (300_000, "X" * 70)])
def test_proof_round_trip(n, ch):
    data = np.random.default_rng(n).integers(0, 256, size=n, dtype=np.uint8).tobytes()
    p = bg.Proof.deserialize(bg.Proof(data, ch).serialize())
    assert p.data == data and p.challenger_type == ch


def test_proof_rejections():
    bad = bytearray(_b("proof_v1"))
    bad[0] = 7
    with pytest.raises(bg.ArgumentError, match="Proof::version"):
        bg.Proof.deserialize(bytes(bad))
    for cut in (3, 10, len(bad) - 1):
        with pytest.raises(bg.ArgumentError, match="NotEnoughBytes"):
            bg.Proof.deserialize(_b("proof_v1")[:cut])
