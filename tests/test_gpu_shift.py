"""GPU shift reduction against the oracle: identical transcript bytes, point and witness eval."""
import numpy as np
import pytest

import oracle as orc
from binius64_b200 import constraint_system as csm

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402


def _operator_data(sc, seed, distinct_z=False):
    prep = sc.cs.prepared()
    abc = csm.eval_operands_csr(sc.witness, prep.and_csr)
    mul = csm.eval_operands_csr(sc.witness, prep.mul_csr)
    _, meta, r_x = orc.and_reduction_prove(*(np.ascontiguousarray(abc[:, i]) for i in range(3)))
    z = meta[3]
    rng = np.random.default_rng(seed)
    if distinct_z:
        z = orc.random_elems(rng, 1)[0]
    r_x_mul = orc.random_elems(rng, (mul.shape[0] - 1).bit_length())
    mul_evals = np.stack([orc.oblong_eval(np.ascontiguousarray(mul[:, i]), z, r_x_mul)
                          for i in (0, 1, 3, 2)])
    return prep, (meta[:3], meta[3], r_x), (mul_evals, z, r_x_mul)


def _ints(a):
    return [orc.to_int(x) for x in np.asarray(a).reshape(-1, 2)]


@pytest.mark.parametrize("log_words,n_and,n_mul,log_public,distinct_z", [
    (8, 5, 1, 1, False),
    (10, 300, 3, 4, False),
    (12, 2000, 5, 2, True),
    (16, 40000, 7, 5, False),
    (18, 150000, 33, 3, False),
])
def test_shift_transcript_matches_oracle(log_words, n_and, n_mul, log_public, distinct_z):
    sc = csm.synthetic_circuit(log_words, n_and, n_mul, seed=log_words, log_public=log_public)
    prep, band, bmul = _operator_data(sc, seed=log_words, distinct_z=distinct_z)
    orc.set_threads(8)
    try:
        proof, point, out3 = orc.shift_prove(sc.witness, log_public, prep.and_csr, prep.mul_csr,
                                             band, bmul)
    finally:
        orc.set_threads(1)
    dcs = bg.DeviceConstraintSystem(sc.cs.serialize())
    w = torch.from_numpy(sc.witness.view(np.int64)).cuda()
    t = bg.ProverTranscript()
    to_py = lambda d: (_ints(d[0]), orc.to_int(d[1]), _ints(d[2]))  # noqa: E731
    gpoint, geval = bg.shift_reduction_prove(dcs, w, t, to_py(band), to_py(bmul))
    got = t.finalize()
    assert len(got) == len(proof)
    if got != proof:
        first = next(i for i in range(len(proof)) if got[i] != proof[i])
        pytest.fail(f"transcript differs first at byte {first} of {len(proof)}")
    assert gpoint == _ints(point)
    assert geval == orc.to_int(out3[0])
    rc, _, _ = orc.shift_verify(sc.witness[: 1 << log_public], log_words, log_public, prep.and_csr,
                                prep.mul_csr, band, bmul, got)
    # phase 1 builds every h part at the AND r_zhat' (phase_1.rs:59-60), so the verifier accepts
    # only when both operators share it, as Prover::prove arranges (prove.rs:218-243)
    assert rc == (2 if distinct_z else 0)


def test_shift_rejects_bad_operator_data():
    sc = csm.synthetic_circuit(8, 5, 1, seed=1)
    prep, band, bmul = _operator_data(sc, seed=1)
    dcs = bg.DeviceConstraintSystem(sc.cs.serialize())
    w = torch.from_numpy(sc.witness.view(np.int64)).cuda()
    t = bg.ProverTranscript()
    ev, z, rx = _ints(band[0]), orc.to_int(band[1]), _ints(band[2])
    mev, mz, mrx = _ints(bmul[0]), orc.to_int(bmul[1]), _ints(bmul[2])
    with pytest.raises(bg.ArgumentError):
        bg.shift_reduction_prove(dcs, w, t, (ev[:2], z, rx), (mev, mz, mrx))
    with pytest.raises(bg.ArgumentError):
        bg.shift_reduction_prove(dcs, w, t, (ev, z, rx + [1]), (mev, mz, mrx))
