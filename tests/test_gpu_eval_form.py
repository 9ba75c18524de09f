"""Witness evaluation on the device against the oracle's interpreter: random programs over every
opcode (registers overwritten and read again, so the level schedule must keep the program's
order), with their assertion counts and first failures, over batches of instances; the program
that recomputes a synthetic circuit's witness, for instances with different inputs, followed by
proofs of the generated witnesses identical to the oracle's; deep programs (runs of narrow levels
in one CTA), alone and after wide levels; and the register-major transpose."""
import numpy as np
import pytest

import oracle as orc
from binius64_b200 import constraint_system as csm

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402
from binius64_b200 import eval_form as ef  # noqa: E402


def random_program(rng, n_regs, n_ops):
    bb = ef.BytecodeBuilder()
    R = lambda: int(rng.integers(0, n_regs))  # noqa: E731
    for k in range(n_ops):
        op = int(rng.integers(0, 26))
        n = int(rng.integers(0, 64))
        if op == 0: bb.band(R(), R(), R())
        elif op == 1: bb.bor(R(), R(), R())
        elif op == 2: bb.bxor(R(), R(), R())
        elif op == 3: bb.select(R(), R(), R(), R())
        elif op == 4: bb.bxor_multi(R(), [R() for _ in range(int(rng.integers(0, 6)))])
        elif op == 5: bb.fax(R(), R(), R(), R())
        elif op == 6: bb.sll(R(), R(), n)
        elif op == 7: bb.slr(R(), R(), n)
        elif op == 8: bb.sar(R(), R(), n)
        elif op == 9: bb.iadd_cout(R(), R(), R(), R())
        elif op == 10: bb.iadd_cin_cout(R(), R(), R(), R(), R())
        elif op == 11: bb.isub_bin_bout(R(), R(), R(), R(), R())
        elif op == 12: bb.imul(R(), R(), R(), R())
        elif op == 13: bb.smul(R(), R(), R(), R())
        elif op == 14: bb.iadd_cout32(R(), R(), R(), R())
        elif op == 15: bb.rotr32(R(), R(), int(rng.integers(0, 256)))
        elif op == 16: bb.shr32(R(), R(), n)
        elif op == 17: bb.rotr(R(), R(), int(rng.integers(0, 256)))
        elif op == 18: bb.mask_low(R(), R(), int(rng.integers(0, 80)))
        elif op == 19: bb.mask_high(R(), R(), int(rng.integers(0, 80)))
        elif op == 20: bb.assert_eq(R(), R(), k)
        elif op == 21: bb.assert_eq_cond(R(), R(), R(), k)
        elif op == 22: bb.assert_zero(R(), k)
        elif op == 23: bb.assert_non_zero(R(), k)
        elif op == 24: bb.assert_false(R(), k)
        else: bb.assert_true(R(), k)
    return bb.finalize()


@pytest.mark.parametrize("seed,n_regs,n_ops,batch", [(1, 8, 200, 1), (2, 32, 2000, 7),
                                                      (3, 300, 5000, 64), (4, 16, 3000, 33)])
def test_random_programs_vs_oracle(seed, n_regs, n_ops, batch):
    rng = np.random.default_rng(seed)
    code = random_program(rng, n_regs, n_ops)
    prog = ef.EvalForm(code, n_regs)
    assert prog.n_insn == n_ops
    inst = rng.integers(0, 2**64, size=(batch, n_regs), dtype=np.uint64, endpoint=False)
    inst[:, : n_regs // 4] &= np.uint64(3)  # small values: some assertions pass
    d = torch.from_numpy(np.ascontiguousarray(inst.T).view(np.int64)).cuda().reshape(-1)
    fails, first = prog.evaluate(d, batch)
    got = d.cpu().numpy().view(np.uint64).reshape(n_regs, batch).T
    fails, first = fails.cpu().numpy(), first.cpu().numpy().view(np.uint64)
    for i in range(batch):
        rc, ref, nf, fe = orc.eval_form_run(code, inst[i])
        assert rc == 0
        assert np.array_equal(got[i], ref), f"instance {i}"
        assert int(fails[i]) == nf
        if nf:
            assert int(first[i]) & 0xFFFFFFFF == fe
            assert int(first[i]) >> 32 == fe  # ids here are the instruction indices
        else:
            assert int(first[i]) == 2**64 - 1


def test_transpose_round_trip():
    x = torch.randint(-2**63, 2**63 - 1, (37 * 1000,), dtype=torch.int64, device="cuda")
    y = ef.transpose_words(x, 37, 1000)
    assert torch.equal(y.view(1000, 37), x.view(37, 1000).T)
    assert torch.equal(ef.transpose_words(y, 1000, 37), x)


@pytest.mark.parametrize("log_words,n_and,n_mul,seed,batch", [(10, 300, 5, 1, 5),
                                                               (14, 15000, 3, 2, 4)])
def test_synthetic_witness_generation_then_prove(log_words, n_and, n_mul, seed, batch):
    circ = csm.synthetic_circuit(log_words, n_and, n_mul, seed=seed)
    code, n_values = ef.synthetic_program(circ)
    prog = ef.EvalForm(code, n_values)
    assert prog.n_levels < 100  # a layered circuit: a few launches, not one per instruction
    lay = circ.cs.layout
    n_in = lay.committed_total_len - lay.n_internal
    rng = np.random.default_rng(seed + 100)
    inputs = np.stack([ef.synthetic_inputs(circ, n_values) for _ in range(batch)])
    # instance 0 keeps the circuit's own inputs; the others draw new witness inputs
    inputs[1:, lay.offset_witness:n_in] = rng.integers(
        0, 2**64, size=(batch - 1, n_in - lay.offset_witness), dtype=np.uint64, endpoint=False)
    d = ef.transpose_words(torch.from_numpy(inputs.view(np.int64)).cuda().reshape(-1), batch,
                           n_values)
    fails, _ = prog.evaluate(d, batch)
    assert int(fails.sum()) == 0
    per_inst = ef.transpose_words(d, n_values, batch).view(batch, n_values)
    assert np.array_equal(per_inst[0, :1 << log_words].cpu().numpy().view(np.uint64),
                          circ.witness)
    dcs = bg.DeviceConstraintSystem(circ.cs.serialize())
    prover = bg.Prover(dcs, 1)
    prep = circ.cs.prepared()
    for i in (0, batch - 1):
        rc, ref_vals, nf, _ = orc.eval_form_run(code, inputs[i])
        assert rc == 0 and nf == 0
        w = per_inst[i, :1 << log_words].contiguous()
        assert np.array_equal(w.cpu().numpy().view(np.uint64), ref_vals[:1 << log_words])
        assert csm.check_satisfied(circ.cs, ref_vals[:1 << log_words])
        proof = prover.prove(w).finalize()
        orc.set_threads(8)
        try:
            assert proof == orc.prove(ref_vals[:1 << log_words], 1, prep.and_csr, prep.mul_csr, 1)
        finally:
            orc.set_threads(1)


@pytest.mark.parametrize("n_ops,batch", [(3000, 1), (3000, 32), (3000, 100)])
def test_deep_chain_vs_oracle(n_ops, batch):
    """A deep program (levels a few instructions wide): runs of narrow levels in one CTA."""
    code, n_values = ef.chain_program(n_ops, seed=n_ops + batch)
    prog = ef.EvalForm(code, n_values)
    assert prog.n_levels > n_ops // 4
    rng = np.random.default_rng(batch)
    inst = np.zeros((batch, n_values), dtype=np.uint64)
    inst[:, :8] = rng.integers(0, 2**64, size=(batch, 8), dtype=np.uint64, endpoint=False)
    d = torch.from_numpy(np.ascontiguousarray(inst.T).view(np.int64)).cuda().reshape(-1)
    prog.evaluate(d, batch)
    got = d.cpu().numpy().view(np.uint64).reshape(n_values, batch).T
    for i in (0, batch // 2, batch - 1):
        rc, ref, _, _ = orc.eval_form_run(code, inst[i])
        assert rc == 0 and np.array_equal(got[i], ref), f"instance {i}"


def test_wide_then_deep_program():
    """Wide levels (the synthetic circuit's) and a deep chain after them in one program."""
    circ = csm.synthetic_circuit(10, 300, 5, seed=9)
    code, n_values = ef.synthetic_program(circ)
    chain, total = ef.chain_program(500, seed=3, first_free=n_values)
    full = code + chain
    prog = ef.EvalForm(full, total)
    v0 = np.zeros(total, dtype=np.uint64)
    v0[:n_values] = ef.synthetic_inputs(circ, n_values)
    batch = 3
    inst = np.repeat(v0[None, :], batch, axis=0)
    d = torch.from_numpy(np.ascontiguousarray(inst.T).view(np.int64)).cuda().reshape(-1)
    prog.evaluate(d, batch)
    got = d.cpu().numpy().view(np.uint64).reshape(total, batch).T
    rc, ref, _, _ = orc.eval_form_run(full, v0)
    assert rc == 0
    assert np.array_equal(got[0], ref) and np.array_equal(got[2], ref)
    assert np.array_equal(ref[:1 << 10], circ.witness)
