"""GPU 1-bit PCS (ring switching + BaseFold + FRI): proof bytes identical to the oracle's, and
accepted by the oracle's restatement of the reference verifier (verifier/verifier/src/pcs.rs)."""
import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402

CASES = [
    # (log_msg, log_batch, log_inv_rate, arities, n_queries)
    (4, 0, 1, [2, 2], 3),
    (6, 0, 1, [1] * 5, 3),
    (8, 2, 1, [2, 2], 5),
    (10, 4, 1, [4], 20),
    (12, 4, 1, [4, 2], 232),
    (9, 3, 2, [3], 30),
    (14, 4, 1, [4, 4], 232),
]


def _gpu_pcs_proof(log_msg, log_batch, R, arities, nq, witness, point):
    rs_log_len = log_msg - log_batch + R
    basis = bg.standard_domain_rs_basis(rs_log_len + log_batch, log_batch)
    ntt = bg.AdditiveNTT(rs_log_len, basis=basis)
    params = bg.FRIParams(bg.ReedSolomonCode(log_msg - log_batch, R), log_batch, list(arities), nq)
    prover = bg.OneBitPCSProver(ntt, params)
    w = bg.to_device(witness)
    committed = prover.commit(w)
    t = bg.ProverTranscript()
    t.message(committed.root)
    prover.prove(committed, w, [orc.to_int(x) for x in point], t)
    return t.finalize()


@pytest.mark.parametrize("case", CASES)
def test_gpu_pcs_proof_matches_oracle(case):
    log_msg, log_batch, R, arities, nq = case
    rng = np.random.default_rng(1000 + log_msg)
    witness = orc.random_elems(rng, 1 << log_msg)
    point = orc.random_elems(rng, log_msg + 7)
    rs_log_len = log_msg - log_batch + R
    tw = orc.domain_twiddles(rs_log_len + log_batch)[: (1 << rs_log_len) - 1]
    ref = orc.pcs_prove(tw, witness, log_batch, R, arities, nq, point)
    got = _gpu_pcs_proof(log_msg, log_batch, R, arities, nq, witness, point)
    assert len(got) == len(ref)
    if got != ref:
        first = next(i for i in range(len(ref)) if got[i] != ref[i])
        pytest.fail(f"proof bytes differ first at offset {first} of {len(ref)}")
    claim = orc.eval_1b_mle(witness, point)
    assert orc.pcs_verify(tw, log_msg, log_batch, R, arities, nq, point, claim, got) == 0


def test_gpu_pcs_c3_shape():
    """The PCS of the 2^20-word prove: 2^19 packed elements, batch 16, arities [4, 4], 232 queries."""
    log_msg, log_batch, R, arities, nq = 19, 4, 1, [4, 4], 232
    rng = np.random.default_rng(19)
    witness = orc.random_elems(rng, 1 << log_msg)
    point = orc.random_elems(rng, log_msg + 7)
    rs_log_len = log_msg - log_batch + R
    tw = orc.domain_twiddles(rs_log_len + log_batch)[: (1 << rs_log_len) - 1]
    got = _gpu_pcs_proof(log_msg, log_batch, R, arities, nq, witness, point)
    orc.set_threads(8)
    try:
        ref = orc.pcs_prove(tw, witness, log_batch, R, arities, nq, point)
    finally:
        orc.set_threads(1)
    assert got == ref
    claim = orc.eval_1b_mle(witness, point)
    assert orc.pcs_verify(tw, log_msg, log_batch, R, arities, nq, point, claim, got) == 0
