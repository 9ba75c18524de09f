"""GPU operand evaluation and AND reduction against the oracle: identical transcript bytes."""
import numpy as np
import pytest

import oracle as orc
from binius64_b200 import constraint_system as csm

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402


def _circuit(log_words, n_and, n_mul, seed):
    sc = csm.synthetic_circuit(log_words, n_and, n_mul, seed=seed)
    assert csm.check_satisfied(sc.cs, sc.witness)
    return sc


@pytest.mark.parametrize("log_words,n_and,n_mul", [(8, 5, 1), (10, 300, 3), (14, 9000, 2)])
def test_eval_operands_matches_numpy(log_words, n_and, n_mul):
    sc = _circuit(log_words, n_and, n_mul, seed=log_words)
    dcs = bg.DeviceConstraintSystem(sc.cs.serialize())
    w = torch.from_numpy(sc.witness.view(np.int64)).cuda()
    got = dcs.eval_operands(w, 0).cpu().numpy().view(np.uint64)
    ref = csm.eval_operands_csr(sc.witness, sc.cs.prepared().and_operands()).T
    assert np.array_equal(got, ref)
    gotm = dcs.eval_operands(w, 1).cpu().numpy().view(np.uint64)
    refm = csm.eval_operands_csr(sc.witness, sc.cs.prepared().mul_operands()).T
    assert np.array_equal(gotm, refm)
    assert dcs.n_and >= 8 and dcs.n_and & (dcs.n_and - 1) == 0


@pytest.mark.parametrize("log_words,n_and", [(8, 5), (10, 300), (13, 4000), (16, 60000)])
def test_and_reduction_transcript_matches_oracle(log_words, n_and):
    sc = _circuit(log_words, n_and, 1, seed=100 + log_words)
    prep = sc.cs.prepared()
    abc = csm.eval_operands_csr(sc.witness, prep.and_operands())
    orc.set_threads(8)
    try:
        proof, meta, point = orc.and_reduction_prove(abc[:, 0].copy(), abc[:, 1].copy(),
                                                     abc[:, 2].copy())
    finally:
        orc.set_threads(1)
    dcs = bg.DeviceConstraintSystem(sc.cs.serialize())
    w = torch.from_numpy(sc.witness.view(np.int64)).cuda()
    t = bg.ProverTranscript()
    gmeta, gpoint = bg.and_reduction_prove(dcs, w, t)
    got = t.finalize()
    assert len(got) == len(proof)
    if got != proof:
        first = next(i for i in range(len(proof)) if got[i] != proof[i])
        pytest.fail(f"transcript differs first at byte {first} of {len(proof)}")
    assert gmeta == [orc.to_int(x) for x in meta]
    assert gpoint == [orc.to_int(x) for x in point]
    rc, _, _ = orc.and_reduction_verify(prep.n_and().bit_length() - 1, got)
    assert rc == 0
