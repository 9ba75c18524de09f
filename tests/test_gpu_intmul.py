"""GPU integer multiplication reduction against the oracle: identical transcript bytes."""
import numpy as np
import pytest

import oracle as orc
from binius64_b200 import constraint_system as csm

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402


@pytest.mark.parametrize("log_words,n_and,n_mul", [(8, 5, 1), (9, 20, 2), (10, 50, 7),
                                                    (12, 100, 64), (14, 200, 1000)])
def test_intmul_transcript_matches_oracle(log_words, n_and, n_mul):
    sc = csm.synthetic_circuit(log_words, n_and, n_mul, seed=log_words + n_mul)
    prep = sc.cs.prepared()
    mul = csm.eval_operands_csr(sc.witness, prep.mul_csr)  # slots a, b, hi, lo
    a, b, hi, lo = (np.ascontiguousarray(mul[:, i]) for i in range(4))
    proof, point, evals = orc.intmul_prove(a, b, lo, hi)
    dcs = bg.DeviceConstraintSystem(sc.cs.serialize())
    w = torch.from_numpy(sc.witness.view(np.int64)).cuda()
    t = bg.ProverTranscript()
    gpoint, gevals = bg.intmul_reduction_prove(dcs, w, t)
    got = t.finalize()
    assert len(got) == len(proof)
    if got != proof:
        first = next(i for i in range(len(proof)) if got[i] != proof[i])
        pytest.fail(f"transcript differs first at byte {first} of {len(proof)}")
    assert gpoint == [orc.to_int(x) for x in point]
    for k in range(4):
        assert gevals[k] == [orc.to_int(x) for x in evals[k]]
    log_n = prep.n_mul().bit_length() - 1
    assert orc.intmul_verify(log_n, got)[0] == 0
