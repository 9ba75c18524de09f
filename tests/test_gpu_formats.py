"""Load-prove on the GPU (prover/examples/src/bin/prover.rs:46-99): a ConstraintSystem v2 and the
public / non-public ValuesData v1 halves in, a Proof v1 out whose transcript is the proof
Prover::prove gives for the same witness and which the restated verifier accepts; the reference's
CS fixture loads on the device; ValueVec::new_from_data joins the halves and zero-fills scratch
(constraint_system.rs:803-823, 1822-1880)."""
import json
import os

import numpy as np
import pytest

import oracle as orc
from binius64_b200 import constraint_system as csm

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402

FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "formats_v1.json")))


def test_reference_cs_fixture_loads_on_device():
    dcs = bg.DeviceConstraintSystem(bytes.fromhex(FIX["constraint_system_v2"]))
    exp = FIX["expect"]["constraint_system_v2"]
    assert (dcs.n_const, dcs.n_inout, dcs.n_witness, dcs.n_internal, dcs.offset_inout,
            dcs.offset_witness, dcs.committed_total_len, dcs.n_scratch) == tuple(
                exp["layout"][k] for k in ("n_const", "n_inout", "n_witness", "n_internal",
                                           "offset_inout", "offset_witness",
                                           "committed_total_len", "n_scratch"))
    assert (dcs.n_and_real, dcs.n_mul_real) == (exp["n_and"], exp["n_mul"])
    assert (dcs.n_and, dcs.n_mul) == (8, 1)  # padded by validate_and_prepare


def test_value_vec_from_data_with_scratch():
    layout = csm.ValueVecLayout(2, 3, 4, 3, 4, 8, 16, 5)
    cs = csm.ConstraintSystem(layout, [11, 22], [], [])
    dcs = bg.DeviceConstraintSystem(cs.serialize())
    vals = np.array([0xA5A55A5A ^ (i * 0x9E3779B9) for i in range(21)], dtype=np.uint64)
    pub, non_pub = vals[:8], vals[8:16]
    out = bg.value_vec_from_data(dcs, bg.ValuesData.deserialize(bg.ValuesData(pub).serialize())
                                 .words, non_pub)
    assert np.array_equal(out[:16], vals[:16]) and not out[16:].any() and len(out) == 21
    with pytest.raises(bg.ArgumentError, match="ValueVecLenMismatch"):
        bg.value_vec_from_data(dcs, pub, non_pub[:-1])


@pytest.mark.parametrize("log_words,n_and,n_mul,log_public", [(10, 300, 3, 4), (14, 12000, 9, 6)])
def test_load_prove_matches_prove_and_verifies(log_words, n_and, n_mul, log_public):
    sc = csm.synthetic_circuit(log_words, n_and, n_mul, seed=log_words + 7, log_public=log_public)
    cs_bytes = sc.cs.serialize()
    off = sc.cs.layout.offset_witness
    pub_b = bg.ValuesData(sc.witness[:off]).serialize()
    nonpub_b = bg.ValuesData(sc.witness[off:]).serialize()
    proof = bg.Proof.deserialize(bg.load_prove(cs_bytes, pub_b, nonpub_b, 1))
    assert proof.challenger_type == bg.STD_CHALLENGER
    dcs = bg.DeviceConstraintSystem(cs_bytes)
    w = torch.from_numpy(sc.witness.view(np.int64)).cuda()
    assert proof.data == bg.Prover(dcs, 1).prove(w).finalize()
    prep = sc.cs.prepared()
    assert off == 1 << log_public
    assert orc.verify(sc.witness[:off], log_words, log_public, prep.and_csr, prep.mul_csr,
                      proof.data) == 0
