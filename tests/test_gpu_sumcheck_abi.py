"""The round-by-round sumcheck provers of the C ABI (the SumcheckProver trait's execute / fold /
finish, prover/prover/src/protocols/sumcheck/common.rs:29-101) against the oracle's restatement,
round coefficients and final evaluations bit for bit, and the trait's call-order errors."""
import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402


def ints(a):
    return [orc.to_int(x) for x in a]


def run_rounds(prover, challenges):
    coeffs = []
    for r in challenges:
        coeffs.append(prover.execute())
        prover.fold(r)
    return coeffs, prover.finish()


@pytest.mark.parametrize("n", [1, 3, 8, 14])
def test_bivariate_product_prover_vs_oracle(n):
    r = np.random.default_rng(40 + n)
    a, b = orc.random_elems(r, 1 << n), orc.random_elems(r, 1 << n)
    s = 0
    for x, y in zip(ints(a), ints(b)):
        s ^= orc.gf_mul(x, y)
    ch = orc.random_elems(r, n)
    co_ref, fin_ref = orc.bivariate_rounds(a, b, s, ch)
    p = bg.BivariateProductSumcheckProver(bg.to_device(a), bg.to_device(b), s)
    assert p.n_vars() == n
    co, fin = run_rounds(p, ints(ch))
    assert co == [ints(c) for c in co_ref]
    assert fin == ints(fin_ref)


@pytest.mark.parametrize("n", [1, 2, 7, 12])
def test_quadratic_mle_check_prover_vs_oracle(n):
    r = np.random.default_rng(50 + n)
    a, b, c = (orc.random_elems(r, 1 << n) for _ in range(3))
    z = orc.random_elems(r, n)
    comp = orc.from_ints([orc.gf_mul(x, y) ^ w for x, y, w in zip(ints(a), ints(b), ints(c))])
    claim = orc.to_int(orc.mle_eval(comp, z))
    ch = orc.random_elems(r, n)
    co_ref, fin_ref = orc.quadratic_mle_rounds(a, b, c, z, claim, ch)
    p = bg.QuadraticMleCheckProver(bg.to_device(a), bg.to_device(b), bg.to_device(c), ints(z),
                                   claim)
    assert p.eval_point() == ints(z)
    co = []
    for k, rr in enumerate(ints(ch)):
        co.append(p.execute())
        p.fold(rr)
        assert p.eval_point() == ints(z)[: n - 1 - k]
    assert co == [ints(x) for x in co_ref]
    assert p.finish() == ints(fin_ref)


@pytest.mark.parametrize("n,m", [(1, 0), (1, 1), (5, 2), (10, 4), (7, 7), (12, 0)])
def test_inout_check_prover_vs_oracle(n, m):
    r = np.random.default_rng(60 + 10 * n + m)
    w = orc.random_elems(r, 1 << n)
    z = orc.random_elems(r, m)
    ch = orc.random_elems(r, n)
    co_ref, fin_ref = orc.inout_rounds(w, z, ch)
    p = bg.InOutCheckProver(bg.to_device(w), ints(z))
    assert p.eval_point() == ints(z) + [0] * (n - m)
    co, fin = run_rounds(p, ints(ch))
    assert co == [ints(x) for x in co_ref]
    assert fin == ints(fin_ref)


def test_sumcheck_call_order_errors():
    r = np.random.default_rng(70)
    a, b = orc.random_elems(r, 8), orc.random_elems(r, 8)
    p = bg.BivariateProductSumcheckProver(bg.to_device(a), bg.to_device(b), 0)
    with pytest.raises(bg.ArgumentError, match="ExpectedExecute"):
        p.fold(5)
    with pytest.raises(bg.ArgumentError, match="ExpectedExecute"):
        p.finish()
    p.execute()
    with pytest.raises(bg.ArgumentError, match="ExpectedFold"):
        p.execute()
    with pytest.raises(bg.ArgumentError, match="ExpectedFold"):
        p.finish()
    p.fold(5)
    with pytest.raises(bg.ArgumentError):
        bg.QuadraticMleCheckProver(bg.to_device(a), bg.to_device(b), bg.to_device(b[:4]),
                                   [1, 2, 3], 0)
    with pytest.raises(bg.ArgumentError):
        bg.InOutCheckProver(bg.to_device(a), [1, 2, 3, 4])
