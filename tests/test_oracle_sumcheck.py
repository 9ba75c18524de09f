"""The oracle's round-by-round sumcheck provers against the protocol identities the reference's
verifiers check (CPU only).

* BivariateProductSumcheckProver (prover/prover/src/protocols/sumcheck/bivariate_product.rs):
  each round polynomial R satisfies R(0) + R(1) = the running sum (sumcheck::verify,
  verifier/verifier/src/protocols/sumcheck/verify.rs), and the last sum is the product of the two
  final evaluations, which are the multilinears' values at the challenges (high-to-low binding:
  challenge k binds index bit n - 1 - k).
* QuadraticMleCheckProver with a*b - c (sumcheck/quadratic_mle.rs) and InOutCheckProver
  (protocols/inout_check.rs): each round's prime polynomial R' satisfies
  (1 - alpha) R'(0) + alpha R'(1) = the running claim, alpha the point's coordinate the round binds
  (mlecheck::verify, verifier/verifier/src/protocols/mlecheck.rs:9-50), and the last claim is the
  composition of the final evaluations.  The first claim is the multilinear extension of the
  composite at the evaluation point, computed directly.
"""
import numpy as np
import pytest

import oracle as orc


def gmul(a, b):
    return orc.gf_mul(a, b)


def ev(coeffs, x):
    acc = 0
    for c in reversed(coeffs):
        acc = gmul(acc, x) ^ c
    return acc


def ints(a):
    return [orc.to_int(x) for x in a]


def rev_point(challenges):
    return orc.from_ints(list(reversed(ints(challenges))))


@pytest.mark.parametrize("n", [1, 2, 5, 9])
def test_bivariate_rounds_satisfy_sumcheck(n):
    r = np.random.default_rng(10 + n)
    a, b = orc.random_elems(r, 1 << n), orc.random_elems(r, 1 << n)
    s = 0
    for x, y in zip(ints(a), ints(b)):
        s ^= gmul(x, y)
    ch = orc.random_elems(r, n)
    co, fin = orc.bivariate_rounds(a, b, s, ch)
    last = s
    for k in range(n):
        c = ints(co[k])
        assert ev(c, 0) ^ ev(c, 1) == last, f"round {k}"
        last = ev(c, orc.to_int(ch[k]))
    fa, fb = ints(fin)
    assert last == gmul(fa, fb)
    pt = rev_point(ch)
    assert orc.to_int(orc.mle_eval(a, pt)) == fa
    assert orc.to_int(orc.mle_eval(b, pt)) == fb


@pytest.mark.parametrize("n", [1, 2, 6, 10])
def test_quadratic_mle_rounds_satisfy_mlecheck(n):
    r = np.random.default_rng(20 + n)
    a, b, c = (orc.random_elems(r, 1 << n) for _ in range(3))
    z = orc.random_elems(r, n)
    comp = orc.from_ints([gmul(x, y) ^ w for x, y, w in zip(ints(a), ints(b), ints(c))])
    claim = orc.to_int(orc.mle_eval(comp, z))
    ch = orc.random_elems(r, n)
    co, fin = orc.quadratic_mle_rounds(a, b, c, z, claim, ch)
    last = claim
    zi = ints(z)
    for k in range(n):
        cf = ints(co[k])
        alpha = zi[n - 1 - k]
        assert gmul(1 ^ alpha, ev(cf, 0)) ^ gmul(alpha, ev(cf, 1)) == last, f"round {k}"
        last = ev(cf, orc.to_int(ch[k]))
    fa, fb, fc = ints(fin)
    assert last == gmul(fa, fb) ^ fc
    pt = rev_point(ch)
    assert [orc.to_int(orc.mle_eval(x, pt)) for x in (a, b, c)] == [fa, fb, fc]


@pytest.mark.parametrize("n,m", [(1, 0), (1, 1), (4, 2), (8, 3), (6, 6), (9, 0)])
def test_inout_rounds_satisfy_mlecheck(n, m):
    r = np.random.default_rng(30 + 10 * n + m)
    w = orc.random_elems(r, 1 << n)
    z = orc.random_elems(r, m)
    ch = orc.random_elems(r, n)
    co, fin = orc.inout_rounds(w, z, ch)
    # InOutCheckProver::new's claim: the public segment's MLE at z (the witness at z || 0)
    last = orc.to_int(orc.mle_eval(w[: 1 << m], z)) if m else orc.to_int(w[0])
    full = np.concatenate([z, orc.elems(n - m)]) if m else orc.elems(n)
    assert last == orc.to_int(orc.mle_eval(w, full))
    zi = ints(full)
    for k in range(n):
        cf = ints(co[k])
        alpha = zi[n - 1 - k]
        assert gmul(1 ^ alpha, ev(cf, 0)) ^ gmul(alpha, ev(cf, 1)) == last, f"round {k}"
        last = ev(cf, orc.to_int(ch[k]))
    assert last == orc.to_int(fin[0])
    assert orc.to_int(orc.mle_eval(w, rev_point(ch))) == orc.to_int(fin[0])
