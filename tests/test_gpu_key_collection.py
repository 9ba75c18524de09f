"""Prover::setup_with_key_collection (prover/prover/src/prove.rs:89-115) on the device: a prover
whose shift term table comes from a serialized KeyCollection gives the same proof bytes as one
set up from the constraint system (and as the oracle), also when the collection lists a word's
keys or a key's constraint indices in another order; collections that do not fit the constraint
system are rejected and leave the table as it was."""
import struct

import numpy as np
import pytest

import oracle as orc
from binius64_b200 import constraint_system as csm

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402
from test_key_collection import parse_kc  # noqa: E402


def write_kc(keys, ranges, cis) -> bytes:
    """KeyCollection::serialize (key_collection.rs:381-398)."""
    out = bytearray(struct.pack("<II", 1, len(keys)))
    for op, kid, s, e in keys:
        out += struct.pack("<BHII", op, kid, s, e)
    out += struct.pack("<I", len(ranges))
    for s, e in ranges:
        out += struct.pack("<II", s, e)
    out += struct.pack("<I", len(cis))
    for operand, c in cis:
        out += struct.pack("<BI", operand, c)
    return bytes(out)


def reordered(data: bytes) -> bytes:
    """The same terms with every word's keys and every key's constraint indices reversed."""
    keys, ranges, cis = parse_kc(data)
    nkeys, ncis, nranges = [], [], []
    for k0, k1 in ranges:
        nranges.append((len(nkeys), len(nkeys) + (k1 - k0)))
        for k in reversed(range(k0, k1)):
            op, kid, s, e = keys[k]
            start = len(ncis)
            ncis.extend(reversed(cis[s:e]))
            nkeys.append((op, kid, start, len(ncis)))
    return write_kc(nkeys, nranges, ncis)


def _prove(dcs, witness, log_inv_rate=1, key_collection=None):
    prover = bg.Prover(dcs, log_inv_rate, key_collection=key_collection)
    w = torch.from_numpy(witness.view(np.int64)).cuda()
    return prover.prove(w).finalize()


@pytest.mark.parametrize("log_words,n_and,n_mul,seed", [(10, 300, 5, 1), (14, 6000, 200, 2)])
def test_setup_with_key_collection_same_proof(log_words, n_and, n_mul, seed):
    sc = csm.synthetic_circuit(log_words, n_and, n_mul, seed=seed)
    prep = sc.cs.prepared()
    cs_bytes = sc.cs.serialize()
    kc = bg.key_collection_from_cs_bytes(cs_bytes)
    dcs = bg.DeviceConstraintSystem(cs_bytes)
    assert dcs.key_collection() == kc == orc.key_collection(prep.and_csr, prep.mul_csr,
                                                             1 << log_words)
    ref = orc.prove(sc.witness, 1, prep.and_csr, prep.mul_csr, 1)
    assert _prove(dcs, sc.witness) == ref
    assert _prove(bg.DeviceConstraintSystem(cs_bytes, key_collection=kc), sc.witness) == ref
    assert _prove(bg.DeviceConstraintSystem(cs_bytes), sc.witness, key_collection=kc) == ref
    assert _prove(bg.DeviceConstraintSystem(cs_bytes, key_collection=reordered(kc)),
                  sc.witness) == ref


def test_key_collection_rejections_leave_table():
    sc = csm.synthetic_circuit(10, 300, 5, seed=3)
    cs_bytes = sc.cs.serialize()
    dcs = bg.DeviceConstraintSystem(cs_bytes)
    kc = dcs.key_collection()
    ref = _prove(dcs, sc.witness)
    bad_version = (2).to_bytes(4, "little") + kc[4:]
    other_words = bg.key_collection_from_cs_bytes(
        csm.synthetic_circuit(11, 300, 5, seed=3).cs.serialize())
    more_and = bg.key_collection_from_cs_bytes(
        csm.synthetic_circuit(10, 600, 5, seed=4).cs.serialize())
    keys, ranges, cis = parse_kc(kc)
    dup = list(keys)
    dup[1] = (dup[1][0], dup[1][1], dup[0][2], dup[0][3])  # two keys own the same indices
    bad_op = list(keys)
    bad_op[0] = (2,) + bad_op[0][1:]
    cases = [
        (bad_version, "version"),
        (kc[:-1], "NotEnoughBytes"),
        (kc + b"\0", "trailing"),
        (other_words, "key range"),
        (more_and, "out of range"),
        (write_kc(dup, ranges, cis), "KeyCollection"),
        (write_kc(bad_op, ranges, cis), "UnknownEnumVariant"),
    ]
    for data, msg in cases:
        with pytest.raises(bg.ArgumentError, match=msg):
            dcs.load_key_collection(data)
        assert _prove(dcs, sc.witness) == ref
