"""Batched / served proving: every proof from the queue equals the lone proof of the same
statement (and the oracle's), whatever else is in flight."""
import numpy as np
import pytest

import oracle as orc
from binius64_b200 import constraint_system as csm

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402

SIZES = [(10, 300, 2), (12, 2000, 1), (13, 3000, 40), (14, 12000, 1), (15, 20000, 5),
         (16, 60000, 1)]


@pytest.fixture(scope="module")
def statements():
    out = []
    for i, (lw, na, nm) in enumerate(SIZES):
        sc = csm.synthetic_circuit(lw, na, nm, seed=500 + i, log_public=1 + i % 3)
        prover = bg.Prover(bg.DeviceConstraintSystem(sc.cs.serialize()))
        w = torch.from_numpy(sc.witness.view(np.int64)).cuda()
        alone = prover.prove(w).finalize()
        out.append((sc, prover, w, alone))
    return out


def test_queue_proofs_equal_lone_proofs(statements):
    q = bg.ProveQueue(n_workers=4)
    tickets = []
    for rep in range(3):
        for i, (sc, prover, w, alone) in enumerate(statements):
            src = w if (rep + i) % 2 == 0 else sc.witness  # device and host witnesses
            tickets.append((i, q.submit(prover, src)))
    for i, t in tickets:
        proof, times = q.wait(t)
        assert proof == statements[i][3], f"statement {i}"
        assert times["latency_ms"] >= times["prove_ms"] > 0
    q.close()
    # the smallest statement against the oracle
    sc, _, _, alone = statements[0]
    prep = sc.cs.prepared()
    assert alone == orc.prove(sc.witness, 1, prep.and_csr, prep.mul_csr)


def test_queue_with_tiny_budget_serialises(statements):
    q = bg.ProveQueue(n_workers=4, hbm_budget_bytes=1)
    tickets = [(i, q.submit(p, w)) for i, (_, p, w, _) in enumerate(statements)]
    for i, t in tickets:
        proof, _ = q.wait(t)
        assert proof == statements[i][3]
    q.close()


def test_queue_rejects_bad_requests(statements):
    q = bg.ProveQueue(n_workers=1)
    sc, prover, w, _ = statements[0]
    with pytest.raises(bg.ArgumentError):
        q.submit(prover, w[:-1])
    with pytest.raises(bg.ArgumentError):
        q.wait(12345)
    q.close()
