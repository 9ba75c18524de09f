"""Pins of the oracle's protocol layer on the reference's own tests, restated (CPU only).

* prover/prover/src/and_reduction/ntt_lookup.rs:239-267 (assert_accurate_ntt_on_well_known_poly):
  the univariate round's per-word lookup NTT of the word with only bit 0 set, at the output
  point x (64..127), is prod_{b=1..63} (x - b) / b in the AES field.  Extended here to every
  single-bit word (the Lagrange basis polynomial of that domain point) and to linearity.
* prover/prover/src/protocols/shift/monster.rs:232-265 (h_op_consistency): the h multilinears of
  build_h_parts, evaluated directly at r_j ++ r_s, equal the verifier's succinct evaluate_h_op
  (verifier/verifier/src/protocols/shift/monster.rs:31-99 with shift_ind.rs's partial_eval_sigmas,
  partial_eval_sigmas_transpose, partial_eval_phi), restated below in Python.
* verifier/verifier/src/protocols/shift/monster.rs:263-323 (test_evaluate_h_op_hypercube_vertices):
  at the hypercube vertices, with the challenge on a domain point, every h_op value is the
  indicator of its integer shift relation -- for the restated evaluate_h_op and for the oracle's
  build_h_parts on every vertex.
* verifier/verifier/src/and_reduction/univariate/univariate_poly.rs:151-182
  (univariate_po2_sanity_check): Lagrange evaluation over the embedded AES subspace agrees with
  the embedded monomial form, which pins the embedding and the 64-point Lagrange basis together.
* prover/prover/src/fri/fold.rs:334-369 (test_fri_compatible_ntt_domains) with the shrunk cases of
  prover/prover/proptest-regressions/fri/fold.txt (log_dim = 0 with arity 0 and 1) first, then
  the property's whole range (log_dim < 8, arity < 4): over the domain of
  BinarySubspace::with_dim(32) (GenericOnTheFly), FRI-folding the encoded message equals encoding
  the message folded with fold_cols.  The dim-32 domain's twiddles for the first layers come from
  generate_evals_from_subspace (verifier/math/src/ntt/domain_context.rs:19-46), restated below.
"""
import numpy as np
import pytest

import oracle as orc


def gm(a, b):
    """GHASH product; products by 0 or 1 (the hypercube vertices below) without a library call."""
    if a <= 1:
        return b if a else 0
    if b <= 1:
        return a if b else 0
    return orc.gf_mul(a, b)


# ---------------------------------------------------------------- NTT lookup KAT

def aes_inv(a):
    r = 1
    for _ in range(254):
        r = orc.aes_mul(r, a)
    return r


def lagrange_aes(t, x):
    acc = 1
    for b in range(64):
        if b != t:
            acc = orc.aes_mul(acc, orc.aes_mul(x ^ b, aes_inv(t ^ b)))
    return acc


def test_ntt_lookup_well_known_poly():
    got = orc.and_word_ntt(1)
    for k, x in enumerate(range(64, 128)):
        want = 1
        for b in range(1, 64):
            want = orc.aes_mul(want, orc.aes_mul(x ^ b, aes_inv(b)))
        assert got[k] == want, k


def test_ntt_lookup_single_bits_and_linearity():
    for t in (0, 1, 5, 31, 32, 63):
        got = orc.and_word_ntt(1 << t)
        assert got == [lagrange_aes(t, x) for x in range(64, 128)], t
    rng = np.random.default_rng(3)
    for _ in range(20):
        a = int(rng.integers(0, 2**63)) * 2 + int(rng.integers(0, 2))
        b = int(rng.integers(0, 2**63)) * 2 + int(rng.integers(0, 2))
        la, lb, lab = orc.and_word_ntt(a), orc.and_word_ntt(b), orc.and_word_ntt(a ^ b)
        assert lab == [x ^ y for x, y in zip(la, lb)]


# ---------------------------------------------------------------- h_op consistency

def partial_eval_sigmas(r_j, r_s):
    n = len(r_j)
    sigma, sigma_p = [0] * (1 << n), [0] * (1 << n)
    sigma[0] = 1
    for k in range(n):
        j, s = r_j[k], r_s[k]
        both = gm(j, s)
        j_one_s, one_j_s, eq = j ^ both, s ^ both, 1 ^ j ^ s
        for i in range(1 << k):
            sigma[(1 << k) | i] = gm(j_one_s, sigma[i])
            sigma_p[(1 << k) | i] = gm(one_j_s, sigma[i]) ^ gm(eq, sigma_p[i])
            si, spi = sigma[i], sigma_p[i]
            sigma[i] = gm(eq, si) ^ gm(j_one_s, spi)
            sigma_p[i] = gm(spi, one_j_s)
    return sigma, sigma_p


def partial_eval_phi(r_s):
    n = len(r_s)
    phi = [0] * (1 << n)
    for k in range(n):
        s = r_s[k]
        for i in range(1 << k):
            phi[(1 << k) | i] = s ^ gm(1 ^ s, phi[i])
            phi[i] ^= phi[(1 << k) | i] ^ s
    return phi


def partial_eval_sigmas_transpose(r_j, r_s):
    n = len(r_j)
    st, stp = [0] * (1 << n), [0] * (1 << n)
    st[0] = 1
    for k in range(n):
        j, s = r_j[k], r_s[k]
        both, xor = gm(j, s), j ^ s
        eq = 1 ^ xor
        zero = eq ^ both
        for i in range(1 << k):
            st[(1 << k) | i] = gm(xor, st[i]) ^ gm(zero, stp[i])
            stp[(1 << k) | i] = gm(both, stp[i])
            sti = st[i]
            stp[i] = gm(both, sti) ^ gm(xor, stp[i])
            st[i] = gm(zero, sti)
    return st


def ip(a, b):
    acc = 0
    for x, y in zip(a, b):
        acc ^= gm(x, y)
    return acc


def prod(xs):
    acc = 1
    for x in xs:
        acc = gm(acc, x)
    return acc


def eq_tensor(point):
    out = [1]
    for r in point:
        out = [gm(v, 1 ^ r) for v in out] + [gm(v, r) for v in out]
    return out


def evaluate_h_op(lt, r_j, r_s):
    sigma, sigma_p = partial_eval_sigmas(r_j, r_s)
    sigma_t = partial_eval_sigmas_transpose(r_j, r_s)
    phi = partial_eval_phi(r_s)
    s32, s32p = partial_eval_sigmas(r_j[:5], r_s[:5])
    s32t = partial_eval_sigmas_transpose(r_j[:5], r_s[:5])
    phi32 = partial_eval_phi(r_s[:5])
    jp, jp32 = prod(r_j), prod(r_j[:5])
    sll, srl = ip(lt, sigma_t), ip(lt, sigma)
    sra = srl ^ gm(jp, ip(lt, phi))
    rotr = ip(lt, [x ^ y for x, y in zip(sigma, sigma_p)])
    rest = eq_tensor(r_j[5:])
    chunks = [lt[:32], lt[32:]]
    sll32 = ip([ip(c, s32t) for c in chunks], rest)
    srl32 = ip([ip(c, s32) for c in chunks], rest)
    sra32 = srl32 ^ ip([gm(jp32, ip(c, phi32)) for c in chunks], rest)
    rotr32 = ip([ip(c, [x ^ y for x, y in zip(s32, s32p)]) for c in chunks], rest)
    return [sll, srl, sra, rotr, sll32, srl32, sra32, rotr32]


@pytest.mark.parametrize("case", range(4))
def test_h_op_consistency(case):
    rng = np.random.default_rng(100 + case)

    def rnd():
        return int.from_bytes(rng.bytes(16), "little")

    r_zhat = rnd()
    r_j = [rnd() for _ in range(6)]
    r_s = [rnd() for _ in range(6)]
    h, lt = orc.shift_h_parts(r_zhat)
    lt = [orc.to_int(x) for x in lt]
    succinct = evaluate_h_op(lt, r_j, r_s)
    point = orc.from_ints(r_j + r_s)
    direct = [orc.to_int(orc.mle_eval(np.ascontiguousarray(h[v]), point)) for v in range(8)]
    assert succinct == direct


def h_op_indicators(i, j, s):
    """The integer relations a shift variant's h multilinear indicates at a hypercube vertex:
    bit i of the shifted word comes from bit j of the input shifted by s (sll, srl, sra, rotr on
    64 bits, then the same on each 32-bit half)."""
    i_hi, i_lo, j_hi, j_lo, s_lo = i // 32, i % 32, j // 32, j % 32, s % 32
    return [j + s == i, i + s == j, min(i + s, 63) == j, (i + s) % 64 == j,
            i_hi == j_hi and j_lo + s_lo == i_lo, i_hi == j_hi and i_lo + s_lo == j_lo,
            i_hi == j_hi and min(i_lo + s_lo, 31) == j_lo,
            i_hi == j_hi and (i_lo + s_lo) % 32 == j_lo]


def test_h_op_hypercube_vertices():
    """verifier/verifier/src/protocols/shift/monster.rs:263-323
    (test_evaluate_h_op_hypercube_vertices): with the challenge at the i-th point of the
    64-point domain (so the Lagrange evaluations are the indicator of i) and r_j, r_s at the
    hypercube vertices of j and s (index_to_hypercube_point: bit k of the index is coordinate k),
    each of the eight h_op values is 1 exactly when the integer shift relation holds.  Checked on
    1024 random (i, j, s) (the reference test's count) for the restated succinct evaluate_h_op,
    and on every (j, s) of each i for the oracle's build_h_parts, whose domain point i is phi(i),
    the AES byte i embedded in GHASH (the reference test's domain is the GHASH subspace of the
    integers 0..63; the indicator form of the Lagrange evaluations is what both rely on)."""
    phi = orc.aes_to_ghash_table()
    rng = np.random.default_rng(0)
    for _ in range(1024):
        i, j, s = (int(x) for x in rng.integers(0, 64, size=3))
        lt = [1 if t == i else 0 for t in range(64)]
        r_j = [(j >> k) & 1 for k in range(6)]
        r_s = [(s >> k) & 1 for k in range(6)]
        assert evaluate_h_op(lt, r_j, r_s) == [int(b) for b in h_op_indicators(i, j, s)], (i, j, s)
    for i in range(64):
        h, lt = orc.shift_h_parts(phi[i])
        assert [orc.to_int(x) for x in lt] == [1 if t == i else 0 for t in range(64)], i
        want = np.zeros((8, 4096, 2), dtype=np.uint64)  # h[v][s * 64 + j], (lo, hi) words
        for s in range(64):
            for j in range(64):
                want[:, s * 64 + j, 0] = h_op_indicators(i, j, s)
        assert np.array_equal(h, want), i


def test_univariate_po2_sanity_check():
    """verifier/verifier/src/and_reduction/univariate/univariate_poly.rs:151-182
    (univariate_po2_sanity_check): a polynomial of degree < 64 with AES-field coefficients, given
    by its values on the 6-dimensional AES subspace (the integers 0..63), evaluated at a GHASH
    challenge by Lagrange interpolation over the embedded domain equals the polynomial with
    embedded coefficients evaluated there.  The oracle's Lagrange evaluations over
    {phi(t) : t < 64} (the ones build_h_parts and the AND reduction use) stand in for
    GenericPo2UnivariatePoly::evaluate_at_challenge."""
    phi = orc.aes_to_ghash_table()
    rng = np.random.default_rng(5)
    for _ in range(4):
        coeffs = [int(x) for x in rng.integers(0, 256, size=64)]
        values = []
        for t in range(64):
            acc, x = 0, 1
            for c in coeffs:
                acc ^= orc.aes_mul(c, x)
                x = orc.aes_mul(x, t)
            values.append(acc)
        z = int.from_bytes(rng.bytes(16), "little")
        _, lt = orc.shift_h_parts(z)
        lhs = 0
        for t in range(64):
            lhs ^= gm(phi[values[t]], orc.to_int(lt[t]))
        rhs, zp = 0, 1
        for c in coeffs:
            rhs ^= gm(phi[c], zp)
            zp = gm(zp, z)
        assert lhs == rhs


# ---------------------------------------------------------------- FRI fold / encode commutation

def on_the_fly_twiddles(dim, n_layers):
    """Flat twiddle table (layer l at [2^l - 1, 2^(l+1) - 1)) of the first n_layers layers of
    the domain of BinarySubspace::with_dim(dim): twiddle(l, j) = sum over the set bits k of j of
    evals[dim - l - 1][k + 1] (domain_context.rs:84-94)."""
    rows = [[1 << i for i in range(dim)]]
    for i in range(1, dim):
        prev = rows[-1]
        rows.append([gm(prev[k], prev[k] ^ prev[0]) for k in range(1, len(prev))])
    rows = [[gm(v, orc.gf_inv(r[0])) for v in r] for r in rows]
    tw = []
    for layer in range(n_layers):
        row = rows[dim - layer - 1]
        for j in range(1 << layer):
            acc = 0
            for k in range(layer):
                if (j >> k) & 1:
                    acc ^= row[k + 1]
            tw.append(acc)
    return orc.from_ints(tw)


TW32 = None


def fri_commute(log_dim, arity):
    global TW32
    if TW32 is None:
        TW32 = on_the_fly_twiddles(32, 12)
    n = log_dim + arity
    rng = np.random.default_rng(1000 + 10 * log_dim + arity)
    msg = orc.random_elems(rng, 1 << n)
    ch = orc.random_elems(rng, arity)
    folded_msg = orc.fri_fold_interleaved(msg, log_dim, arity, ch)  # fold_cols(msg, eq(ch))
    codeword = orc.ntt_forward(TW32, 12, msg)
    folded_cw = orc.fri_fold_codeword(TW32, 12, codeword, n, ch)
    encoded = orc.ntt_forward(TW32, 12, folded_msg)
    assert np.array_equal(folded_cw, encoded), (log_dim, arity)


@pytest.mark.parametrize("log_dim,arity", [(0, 0), (0, 1)])
def test_fri_fold_regression_seeds(log_dim, arity):
    fri_commute(log_dim, arity)


def test_fri_compatible_ntt_domains_full_range():
    for log_dim in range(8):
        for arity in range(4):
            fri_commute(log_dim, arity)
