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


def test_queue_with_tight_budget_serialises(statements):
    # a budget of the largest request alone: the queue runs one large proof at a time
    budget = max(p.workspace_bytes() for _, p, _, _ in statements)
    q = bg.ProveQueue(n_workers=4, hbm_budget_bytes=budget)
    tickets = [(i, q.submit(p, w)) for i, (_, p, w, _) in enumerate(statements)]
    for i, t in tickets:
        proof, _ = q.wait(t)
        assert proof == statements[i][3]
    st = q.stats()
    assert st["completed"] == len(statements) and st["peak"] <= budget
    q.close()


def test_queue_refuses_a_request_over_its_budget(statements):
    # the refusal is the host's: nothing is launched for it, and the queue keeps serving
    small, large = statements[0], statements[-1]
    budget = small[1].workspace_bytes() + 8 * len(small[0].witness)
    assert large[1].workspace_bytes() > budget
    q = bg.ProveQueue(n_workers=2, hbm_budget_bytes=budget)
    with pytest.raises(bg.OutOfMemoryError):
        q.submit(large[1], large[2])
    for src in (small[2], small[0].witness):
        proof, _ = q.wait(q.submit(small[1], src))
        assert proof == small[3]
    q.close()


@pytest.mark.parametrize("allocs_before_failure", [0, 3, 11])
def test_queue_survives_a_refused_device_allocation(statements, allocs_before_failure):
    # a device allocation refused in the middle of a proof (injected on the host: the allocator
    # call returns the error the pool gives when it has no memory) fails that request alone;
    # the next request on the same queue and worker still gets the lone proof's bytes
    sc, prover, w, alone = statements[2]
    q = bg.ProveQueue(n_workers=1)
    lib = bg.lib()
    try:
        lib.binius_debug_fail_allocs(allocs_before_failure)
        t = q.submit(prover, sc.witness if allocs_before_failure == 0 else w)
        with pytest.raises(bg.OutOfMemoryError):
            q.wait(t)
    finally:
        lib.binius_debug_fail_allocs(-1)
    for src in (w, sc.witness):
        proof, _ = q.wait(q.submit(prover, src))
        assert proof == alone
    assert prover.prove(w).finalize() == alone
    q.close()


def test_queue_holds_device_memory_within_its_budget(statements):
    # workers keep their arena chunks between proofs; the queue counts them, and idle workers
    # give them back when the head request would not fit.  Mixed small and large requests with
    # a budget of about one and a half large proofs: the device pool's used-memory high-water
    # mark during the run stays within the budget.
    drv = pytest.importorskip("cuda.bindings.driver")
    small, large = statements[1], statements[-1]
    for _, p, w, _ in (small, large):
        p.prove(w)  # lone proofs measure each prover's footprint
    budget = int(1.5 * large[1].workspace_bytes())
    q = bg.ProveQueue(n_workers=4, hbm_budget_bytes=budget)
    torch.cuda.synchronize()
    err, pool = drv.cuDeviceGetDefaultMemPool(torch.cuda.current_device())
    assert err == drv.CUresult.CUDA_SUCCESS
    zero = drv.cuuint64_t(0)
    assert drv.cuMemPoolSetAttribute(
        pool, drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH, zero)[0] == \
        drv.CUresult.CUDA_SUCCESS
    tickets = []
    for rep in range(4):
        for st in (large, small, small, large, small):
            tickets.append((st, q.submit(st[1], st[2])))
    for st, t in tickets:
        proof, _ = q.wait(t)
        assert proof == st[3]
    err, high = drv.cuMemPoolGetAttribute(pool, drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH)
    assert err == drv.CUresult.CUDA_SUCCESS
    stats = q.stats()
    q.close()
    assert stats["peak"] <= budget
    assert int(high) <= budget, (int(high), budget, stats)


def test_queue_rejects_bad_requests(statements):
    q = bg.ProveQueue(n_workers=1)
    sc, prover, w, _ = statements[0]
    with pytest.raises(bg.ArgumentError):
        q.submit(prover, w[:-1])
    with pytest.raises(bg.ArgumentError):
        q.wait(12345)
    q.close()
