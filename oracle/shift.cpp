// CPU oracle (test infrastructure only): the shift reduction, prover side, plus the verifier's
// claim relations used to pin it.
//
// Restates:
//   shift::prove                 prover/prover/src/protocols/shift/prove.rs:53-153
//   KeyCollection / accumulate   protocols/shift/key_collection.rs:95-312 (here per operand term:
//                                a key only groups terms of one word, id and operation, and every
//                                quantity below is a sum over its terms)
//   phase 1                      protocols/shift/phase_1.rs:43-276, monster.rs:34-104 (h parts)
//   phase 2                      protocols/shift/phase_2.rs:56-160, monster.rs:138-219,
//                                fold_word.rs:77-96, protocols/inout_check.rs:19-211,
//                                protocols/sumcheck/{batch.rs:41-103, mle_to_sumcheck.rs:28-77,
//                                gruen32.rs, round_evals.rs:145-156}
//   claim relation               verifier/verifier/src/protocols/shift/verify.rs:74-130
#include <string.h>

#include <mutex>
#include <vector>

#include "oracle.h"
#include "oracle_internal.h"
#include "protocols.h"
#include "transcript.h"

namespace orc {

uint64_t shifted_word(uint64_t w, uint32_t variant, uint32_t amount);

namespace {

u128 phi_of(uint8_t b) {
  static u128 table[256];
  static bool ready = false;
  if (!ready) {
    aes_to_ghash_table(table);
    ready = true;
  }
  return table[b];
}

// lagrange_evals over {phi(t) : t < 64} (verifier/math/src/univariate.rs:47-78).
void l_tilde(u128 z, u128 out[64]) {
  u128 w = 1;
  for (int u = 1; u < 64; u++) w = gf_mul(w, phi_of((uint8_t)u));
  w = gf_inv(w);
  u128 prefix[64], suffix[64];
  prefix[0] = 1;
  for (int i = 1; i < 64; i++) prefix[i] = gf_mul(prefix[i - 1], z ^ phi_of((uint8_t)(i - 1)));
  suffix[63] = 1;
  for (int i = 62; i >= 0; i--) suffix[i] = gf_mul(suffix[i + 1], z ^ phi_of((uint8_t)(i + 1)));
  for (int i = 0; i < 64; i++) out[i] = gf_mul(gf_mul(prefix[i], suffix[i]), w);
}

// build_h_parts (monster.rs:34-104): h[v][s*64 + j].
void build_h_parts(u128 r_zhat, std::vector<u128>& h) {
  u128 L[64];
  l_tilde(r_zhat, L);
  h.assign(8 * 4096, 0);
  auto part = [&](int v, int s) { return h.data() + v * 4096 + s * 64; };
  for (int s = 0; s < 64; s++) {
    u128* p;
    p = part(0, s);  // sll
    for (int j = 0; j < 64 - s; j++) p[j] = L[s + j];
    p = part(1, s);  // srl
    for (int j = s; j < 64; j++) p[j] = L[j - s];
    p = part(2, s);  // sra
    for (int j = s; j < 64; j++) p[j] = L[j - s];
    for (int t = 64 - s; t < 64; t++) p[63] ^= L[t];
    p = part(3, s);  // rotr
    for (int j = 0; j < s; j++) p[j] = L[64 - s + j];
    for (int j = s; j < 64; j++) p[j] = L[j - s];
    const int s32 = s % 32;
    for (int half = 0; half < 2; half++) {
      const u128* Lh = L + 32 * half;
      p = part(4, s) + 32 * half;  // sll32
      for (int j = 0; j < 32 - s32; j++) p[j] = Lh[s32 + j];
      p = part(5, s) + 32 * half;  // srl32
      for (int j = s32; j < 32; j++) p[j] = Lh[j - s32];
      p = part(6, s) + 32 * half;  // sra32
      for (int j = s32; j < 32; j++) p[j] = Lh[j - s32];
      for (int t = 32 - s32; t < 32; t++) p[31] ^= Lh[t];
      p = part(7, s) + 32 * half;  // rotr32
      for (int j = 0; j < s32; j++) p[j] = Lh[32 - s32 + j];
      for (int j = s32; j < 32; j++) p[j] = Lh[j - s32];
    }
  }
}

u128 inner(const u128* a, const u128* b, size_t n) {
  u128 acc = 0;
  for (size_t i = 0; i < n; i++) acc ^= gf_mul(a[i], b[i]);
  return acc;
}

// One round of the bivariate product on (a, b) (halves lo | hi): y1, yinf.  The sums are XORs,
// so the threads' partial sums combine to the same values in any order.
void biv_round(const std::vector<u128>& a, const std::vector<u128>& b, size_t off, size_t len,
               u128& y1, u128& yinf) {
  const size_t half = len / 2;
  std::mutex m;
  parallel_for(half, [&](size_t lo, size_t hi) {
    u128 s1 = 0, sinf = 0;
    for (size_t i = lo; i < hi; i++) {
      const u128 a0 = a[off + i], a1 = a[off + half + i], b0 = b[off + i], b1 = b[off + half + i];
      s1 ^= gf_mul(a1, b1);
      sinf ^= gf_mul(a0 ^ a1, b0 ^ b1);
    }
    std::lock_guard<std::mutex> g(m);
    y1 ^= s1;
    yinf ^= sinf;
  });
}

// out[i] ^= v for each set bit i of w.
inline void xor_at_bits(u128* out, uint64_t w, u128 v) {
  for (; w; w &= w - 1) out[__builtin_ctzll(w)] ^= v;
}

void fold_top(std::vector<u128>& a, size_t off, size_t len, u128 r, std::vector<u128>& out) {
  const size_t half = len / 2;
  for (size_t i = 0; i < half; i++) out.push_back(a[off + i] ^ gf_mul(r, a[off + half + i] ^ a[off + i]));
}

}  // namespace


void l_tilde64(u128 z, u128 out[64]) { l_tilde(z, out); }

ShiftResult shift_prove(const uint64_t* words, uint32_t log_words, uint32_t log_public,
                        const Ops& and_ops, const Ops& mul_ops, OpData& band, OpData& bmul,
                        Transcript& t) {
  ShiftResult res;
  const u128 lam_and = t.sample();
  const u128 lam_mul = t.sample();
  for (OpData* d : {&band, &bmul}) {
    const u128 lam = d == &band ? lam_and : lam_mul;
    d->eq.assign((size_t)1 << d->r_x.size(), 0);
    eq_ind_partial_eval(d->r_x.data(), (uint32_t)d->r_x.size(), d->eq.data());
    d->lpow.clear();
    u128 p = lam;
    for (size_t i = 0; i < d->evals.size(); i++) {
      d->lpow.push_back(p);
      p = gf_mul(p, lam);
    }
  }
  res.claim = inner(band.evals.data(), band.lpow.data(), band.evals.size()) ^
              inner(bmul.evals.data(), bmul.lpow.data(), bmul.evals.size());

  // ---- phase 1: g parts
  std::vector<u128> g(8 * 4096, 0);
  std::mutex g_mu;
  auto add_terms = [&](const Ops& ops, const OpData& d) {
    // constraints split over the threads, each into its own copy of g, XORed together at the end
    parallel_for(ops.n, [&](size_t c_lo, size_t c_hi) {
      std::vector<u128> part(8 * 4096, 0);
      for (size_t c = c_lo; c < c_hi; c++)
        for (uint32_t sl = 0; sl < ops.k; sl++) {
          const uint32_t grp = (uint32_t)c * ops.k + sl;
          const u128 weight = gf_mul(d.lpow[ops.slot_to_operand[sl]], d.eq[c]);
          for (uint32_t e = ops.off[grp]; e < ops.off[grp + 1]; e++)
            xor_at_bits(part.data() + ops.var[e] * 4096 + ops.amt[e] * 64, words[ops.vi[e]],
                        weight);
        }
      std::lock_guard<std::mutex> lk(g_mu);
      for (size_t i = 0; i < part.size(); i++) g[i] ^= part[i];
    });
  };
  add_terms(and_ops, band);
  add_terms(mul_ops, bmul);
  std::vector<u128> h;
  build_h_parts(band.r_zhat, h);
  u128 sum = inner(g.data(), h.data(), g.size());
  res.initial_sum = sum;
  std::vector<u128> ch1;
  size_t len = 4096;
  for (int round = 0; round < 12; round++) {
    u128 y1 = 0, yinf = 0;
    for (int v = 0; v < 8; v++) biv_round(g, h, v * len, len, y1, yinf);
    const u128 c0 = sum ^ y1, c2 = yinf, c1 = y1 ^ c0 ^ c2;
    u128 rp[2] = {c0, c1};
    t.message_elems(rp, 2);
    const u128 r = t.sample();
    ch1.push_back(r);
    std::vector<u128> g2, h2;
    for (int v = 0; v < 8; v++) {
      fold_top(g, v * len, len, r, g2);
      fold_top(h, v * len, len, r, h2);
    }
    g.swap(g2);
    h.swap(h2);
    len /= 2;
    sum = c0 ^ gf_mul(c1, r) ^ gf_mul(c2, gf_mul(r, r));
  }
  u128 gamma = 0;
  for (int v = 0; v < 8; v++) gamma ^= gf_mul(h[v], g[v]);
  std::vector<u128> rev(ch1.rbegin(), ch1.rend());
  std::vector<u128> r_j(rev.begin(), rev.begin() + 6), r_s(rev.begin() + 6, rev.end());

  // ---- phase 2
  const size_t N = (size_t)1 << log_words;
  u128 eq_rj[64];
  eq_ind_partial_eval(r_j.data(), 6, eq_rj);
  std::vector<u128> W(N);
  parallel_for(N, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; i++) {
      u128 acc = 0;
      for (uint64_t w = words[i]; w; w &= w - 1) acc ^= eq_rj[__builtin_ctzll(w)];
      W[i] = acc;
    }
  });
  std::vector<u128> rjs(r_j);
  rjs.insert(rjs.end(), r_s.begin(), r_s.end());
  std::vector<u128> eq_rjs(4096);
  eq_ind_partial_eval(rjs.data(), 12, eq_rjs.data());
  u128 eq_rs[64];
  eq_ind_partial_eval(r_s.data(), 6, eq_rs);
  u128 h_ops[2][8];
  for (int kind = 0; kind < 2; kind++) {
    std::vector<u128> hk;
    build_h_parts(kind == 0 ? band.r_zhat : bmul.r_zhat, hk);
    for (int v = 0; v < 8; v++) h_ops[kind][v] = inner(hk.data() + v * 4096, eq_rjs.data(), 4096);
  }
  std::vector<u128> M(N, 0);
  std::mutex m_mu;
  auto add_monster = [&](const Ops& ops, const OpData& d, int kind) {
    // h_op(variant) * eq(r_s, amount) once per (variant, amount); constraints split over the
    // threads, each into its own copy of M, XORed together at the end (the copies are held to
    // 1 GiB in all; beyond that one thread adds every term)
    std::vector<u128> hs(8 * 64);
    for (int v = 0; v < 8; v++)
      for (int a = 0; a < 64; a++) hs[v * 64 + a] = gf_mul(h_ops[kind][v], eq_rs[a]);
    auto run = [&](size_t c_lo, size_t c_hi) {
      std::vector<u128> part(N, 0);
      for (size_t c = c_lo; c < c_hi; c++)
        for (uint32_t sl = 0; sl < ops.k; sl++) {
          const uint32_t grp = (uint32_t)c * ops.k + sl;
          const u128 weight = gf_mul(d.lpow[ops.slot_to_operand[sl]], d.eq[c]);
          for (uint32_t e = ops.off[grp]; e < ops.off[grp + 1]; e++)
            part[ops.vi[e]] ^= gf_mul(weight, hs[ops.var[e] * 64 + ops.amt[e]]);
        }
      std::lock_guard<std::mutex> lk(m_mu);
      for (size_t i = 0; i < N; i++) M[i] ^= part[i];
    };
    if ((uint64_t)N * sizeof(u128) * (uint64_t)num_threads() <= (1ull << 30))
      parallel_for(ops.n, run);
    else
      run(0, ops.n);
  };
  add_monster(and_ops, band, 0);
  add_monster(mul_ops, bmul, 1);

  const uint32_t p = log_public;
  std::vector<u128> point(p);
  for (auto& v : point) v = t.sample();
  // InOutCheckProver::new: public eval through the Gruen eq expansion
  auto eval_gruen = [&](const u128* m, uint32_t nv, uint32_t gn) -> u128 {
    // gn = gruen n_vars_remaining == nv; eq over point[0 .. gn-1)
    if (nv == 0) return m[0];
    std::vector<u128> eq((size_t)1 << (gn - 1));
    eq_ind_partial_eval(point.data(), gn - 1, eq.data());
    const size_t half = (size_t)1 << (nv - 1);
    const u128 lo = inner(m, eq.data(), half), hi = inner(m + half, eq.data(), half);
    return lo ^ gf_mul(hi ^ lo, point[gn - 1]);
  };
  u128 inout_eval = eval_gruen(W.data(), p, p);
  uint32_t gruen_n = p;
  u128 eq_prefix = 1;
  const u128 beta = t.sample();
  u128 shift_sum = gamma;
  std::vector<u128> ch2;
  for (uint32_t n_rem = log_words; n_rem > 0; n_rem--) {
    const size_t half = (size_t)1 << (n_rem - 1);
    // shift prover
    u128 y1 = 0, yinf = 0;
    biv_round(W, M, 0, (size_t)1 << n_rem, y1, yinf);
    const u128 s0 = shift_sum ^ y1, s2 = yinf, s1 = y1 ^ s0 ^ s2;
    // in/out prover
    u128 iy0, iy1;
    if (p < n_rem) {
      iy1 = eval_gruen(W.data() + half, p, gruen_n);
      iy0 = inout_eval;
    } else {
      std::vector<u128> eq((size_t)1 << (gruen_n - 1));
      eq_ind_partial_eval(point.data(), gruen_n - 1, eq.data());
      iy1 = inner(W.data() + half, eq.data(), half);
      const u128 alpha = point[gruen_n - 1];
      iy0 = gf_mul(inout_eval ^ gf_mul(iy1, alpha), gf_inv(1 ^ alpha));
    }
    const u128 q0 = iy0, q1 = iy1 ^ iy0;
    const u128 alpha_dec = n_rem <= p ? point[n_rem - 1] : 0;
    // round_coeffs_by_eq: prime * (1 + alpha) + X * prime, then * eq_prefix
    const u128 one_a = 1 ^ alpha_dec;
    const u128 d0 = gf_mul(gf_mul(q0, one_a), eq_prefix);
    const u128 d1 = gf_mul(gf_mul(q1, one_a) ^ q0, eq_prefix);
    const u128 d2 = gf_mul(q1, eq_prefix);
    const u128 b0 = s0 ^ gf_mul(beta, d0), b1 = s1 ^ gf_mul(beta, d1);
    u128 rp[2] = {b0, b1};
    t.message_elems(rp, 2);
    (void)d2;
    const u128 r = t.sample();
    ch2.push_back(r);
    shift_sum = s0 ^ gf_mul(s1, r) ^ gf_mul(s2, gf_mul(r, r));
    inout_eval = q0 ^ gf_mul(q1, r);
    parallel_for(half, [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; i++) {
        W[i] ^= gf_mul(r, W[half + i] ^ W[i]);
        M[i] ^= gf_mul(r, M[half + i] ^ M[i]);
      }
    });
    W.resize(half);
    M.resize(half);
    if (n_rem <= p) gruen_n--;
    eq_prefix = gf_mul(eq_prefix, 1 ^ r ^ alpha_dec);
  }
  res.witness_eval = W[0];
  t.message_elems(&W[0], 1);
  res.challenges = r_j;
  res.challenges.insert(res.challenges.end(), ch2.rbegin(), ch2.rend());
  return res;
}


// Restated verifier: shift::verify + check_eval (verifier/verifier/src/protocols/shift/verify.rs:
// 161-306) with evaluate_public_mle (:335-353).  The monster evaluation is taken term by term from
// the operands, independently of the prover's key grouping.  Returns 0 when the proof verifies.
int shift_verify(const uint64_t* public_words, uint32_t log_words, uint32_t log_public,
                 const Ops& and_ops, const Ops& mul_ops, OpData& band, OpData& bmul,
                 Transcript& t, u128& witness_eval, std::vector<u128>& point) {
  const u128 lam_and = t.sample();
  const u128 lam_mul = t.sample();
  for (OpData* d : {&band, &bmul}) {
    const u128 lam = d == &band ? lam_and : lam_mul;
    d->eq.assign((size_t)1 << d->r_x.size(), 0);
    eq_ind_partial_eval(d->r_x.data(), (uint32_t)d->r_x.size(), d->eq.data());
    d->lpow.clear();
    u128 p = lam;
    for (size_t i = 0; i < d->evals.size(); i++) {
      d->lpow.push_back(p);
      p = gf_mul(p, lam);
    }
  }
  u128 sum = inner(band.evals.data(), band.lpow.data(), band.evals.size()) ^
             inner(bmul.evals.data(), bmul.lpow.data(), bmul.evals.size());
  auto run = [&](uint32_t n_vars, std::vector<u128>& ch) {
    for (uint32_t i = 0; i < n_vars; i++) {
      u128 c[2];
      t.read_message((uint8_t*)c, 32);
      const u128 r = t.sample();
      const u128 c2 = sum ^ c[1];
      sum = c[0] ^ gf_mul(c[1], r) ^ gf_mul(c2, gf_mul(r, r));
      ch.push_back(r);
    }
  };
  std::vector<u128> ch1;
  run(12, ch1);
  const u128 gamma = sum;
  std::vector<u128> rev(ch1.rbegin(), ch1.rend());
  std::vector<u128> r_j(rev.begin(), rev.begin() + 6), r_s(rev.begin() + 6, rev.end());
  std::vector<u128> z(log_public);
  for (auto& v : z) v = t.sample();
  u128 eq_rj[64];
  eq_ind_partial_eval(r_j.data(), 6, eq_rj);
  std::vector<u128> eq_z((size_t)1 << log_public);
  eq_ind_partial_eval(z.data(), log_public, eq_z.data());
  u128 public_eval = 0;
  for (size_t i = 0; i < eq_z.size(); i++) {
    u128 f = 0;
    for (int j = 0; j < 64; j++)
      if ((public_words[i] >> j) & 1) f ^= eq_rj[j];
    public_eval ^= gf_mul(f, eq_z[i]);
  }
  const u128 beta = t.sample();
  sum = gamma ^ gf_mul(beta, public_eval);
  std::vector<u128> ch2;
  run(log_words, ch2);
  std::vector<u128> r_y(ch2.rbegin(), ch2.rend());
  t.read_message((uint8_t*)&witness_eval, 16);

  std::vector<u128> eq_ry((size_t)1 << log_words);
  eq_ind_partial_eval(r_y.data(), log_words, eq_ry.data());
  std::vector<u128> rjs(r_j);
  rjs.insert(rjs.end(), r_s.begin(), r_s.end());
  std::vector<u128> eq_rjs(4096);
  eq_ind_partial_eval(rjs.data(), 12, eq_rjs.data());
  u128 eq_rs[64];
  eq_ind_partial_eval(r_s.data(), 6, eq_rs);
  u128 monster = 0;
  for (int kind = 0; kind < 2; kind++) {
    const Ops& ops = kind == 0 ? and_ops : mul_ops;
    const OpData& d = kind == 0 ? band : bmul;
    std::vector<u128> hk;
    build_h_parts(d.r_zhat, hk);
    u128 h_op[8];
    for (int v = 0; v < 8; v++) h_op[v] = inner(hk.data() + v * 4096, eq_rjs.data(), 4096);
    for (uint32_t c = 0; c < ops.n; c++)
      for (uint32_t sl = 0; sl < ops.k; sl++) {
        const uint32_t grp = c * ops.k + sl;
        const u128 weight = gf_mul(d.lpow[ops.slot_to_operand[sl]], d.eq[c]);
        for (uint32_t e = ops.off[grp]; e < ops.off[grp + 1]; e++)
          monster ^= gf_mul(gf_mul(weight, eq_ry[ops.vi[e]]),
                            gf_mul(h_op[ops.var[e]], eq_rs[ops.amt[e]]));
      }
  }
  u128 eq_eval = 1;
  for (uint32_t k = 0; k < log_words; k++)
    eq_eval = gf_mul(eq_eval, 1 ^ r_y[k] ^ (k < log_public ? z[k] : 0));
  point = r_j;
  point.insert(point.end(), r_y.begin(), r_y.end());
  if (t.overrun) return 1;
  if (sum != gf_mul(witness_eval, monster ^ gf_mul(beta, eq_eval))) return 2;
  return 0;
}

// MLE of a word column at the oblong point (univariate z over {phi(t)}, multilinear r_x):
// sum_c eq(r_x)[c] sum_j bit_j(v[c]) L_j(z).
u128 oblong_eval(const uint64_t* v, uint32_t log_n, u128 z, const u128* r_x) {
  u128 L[64];
  l_tilde(z, L);
  std::vector<u128> eq((size_t)1 << log_n);
  eq_ind_partial_eval(r_x, log_n, eq.data());
  u128 acc = 0;
  for (size_t c = 0; c < eq.size(); c++) {
    u128 f = 0;
    for (int j = 0; j < 64; j++)
      if ((v[c] >> j) & 1) f ^= L[j];
    acc ^= gf_mul(f, eq[c]);
  }
  return acc;
}

}  // namespace orc

using namespace orc;

extern "C" {

namespace {

uint32_t log2_ceil(uint32_t n) {
  uint32_t r = 0;
  while ((1u << r) < n) r++;
  return r;
}

void make_ops(const uint32_t* const* csr, const uint8_t* var, uint32_t n, bool is_mul, Ops& o) {
  static const uint32_t and_map[3] = {0, 1, 2};
  static const uint32_t mul_map[4] = {0, 1, 3, 2};  // CSR slots (a, b, hi, lo) -> (a, b, lo, hi)
  o = Ops{is_mul ? 4u : 3u, n, csr[0], csr[1], var, csr[2], is_mul ? mul_map : and_map};
}

void make_data(const uint64_t* evals, uint32_t n_evals, const uint64_t* rz, const uint64_t* rx,
               uint32_t n_constraints, OpData& d) {
  for (uint32_t i = 0; i < n_evals; i++) d.evals.push_back(load(evals + 2 * i));
  d.r_zhat = load(rz);
  for (uint32_t i = 0; i < log2_ceil(n_constraints); i++) d.r_x.push_back(load(rx + 2 * i));
}

}  // namespace

// Shift reduction on a fresh transcript.  CSR operands as in binius64_b200.constraint_system
// (offsets, value indices, amounts as u32; variants as u8; AND slots a, b, c; MUL slots a, b, hi,
// lo).  Operator data: AND evals (a, b, c), MUL evals (a, b, lo, hi), each with its r_zhat' and
// r_x'.  out_point: 6 + log_words elements (r_j ++ r_y); out3: witness eval, the phase-1 initial
// sum and the verifier's batched claim.
// build_h_parts (monster.rs:34-104) at r_zhat: h_out holds 8 x 4096 elements (variant-major,
// index s * 64 + j); l_tilde_out the 64 Lagrange evaluations it is built from.
void orc_shift_h_parts(const uint64_t* r_zhat, uint64_t* h_out, uint64_t* l_tilde_out) {
  std::vector<u128> h;
  build_h_parts(load(r_zhat), h);
  for (size_t i = 0; i < h.size(); i++) store(h_out + 2 * i, h[i]);
  u128 L[64];
  l_tilde64(load(r_zhat), L);
  for (int i = 0; i < 64; i++) store(l_tilde_out + 2 * i, L[i]);
}

int orc_shift_prove(const uint64_t* words, uint32_t log_words, uint32_t log_public,
                    const uint32_t* const* and_csr, const uint8_t* and_var, uint32_t n_and,
                    const uint32_t* const* mul_csr, const uint8_t* mul_var, uint32_t n_mul,
                    const uint64_t* and_evals, const uint64_t* and_rz, const uint64_t* and_rx,
                    const uint64_t* mul_evals, const uint64_t* mul_rz, const uint64_t* mul_rx,
                    uint8_t* proof, size_t cap, size_t* len, uint64_t* out_point,
                    uint64_t* out3) {
  Ops ao, mo;
  make_ops(and_csr, and_var, n_and, false, ao);
  make_ops(mul_csr, mul_var, n_mul, true, mo);
  OpData band, bmul;
  make_data(and_evals, 3, and_rz, and_rx, n_and, band);
  make_data(mul_evals, 4, mul_rz, mul_rx, n_mul, bmul);
  Transcript t;
  ShiftResult r = shift_prove(words, log_words, log_public, ao, mo, band, bmul, t);
  *len = t.tape.size();
  if (t.tape.size() > cap) return 2;
  memcpy(proof, t.tape.data(), t.tape.size());
  for (size_t i = 0; i < r.challenges.size(); i++) store(out_point + 2 * i, r.challenges[i]);
  store(out3 + 0, r.witness_eval);
  store(out3 + 2, r.initial_sum);
  store(out3 + 4, r.claim);
  return 0;
}

// Restated verifier over the proof bytes; 0 = accepted.  out_eval: the witness evaluation read
// from the proof; out_point as for orc_shift_prove.
int orc_shift_verify(const uint64_t* public_words, uint32_t log_words, uint32_t log_public,
                     const uint32_t* const* and_csr, const uint8_t* and_var, uint32_t n_and,
                     const uint32_t* const* mul_csr, const uint8_t* mul_var, uint32_t n_mul,
                     const uint64_t* and_evals, const uint64_t* and_rz, const uint64_t* and_rx,
                     const uint64_t* mul_evals, const uint64_t* mul_rz, const uint64_t* mul_rx,
                     const uint8_t* proof, size_t len, uint64_t* out_eval, uint64_t* out_point) {
  Ops ao, mo;
  make_ops(and_csr, and_var, n_and, false, ao);
  make_ops(mul_csr, mul_var, n_mul, true, mo);
  OpData band, bmul;
  make_data(and_evals, 3, and_rz, and_rx, n_and, band);
  make_data(mul_evals, 4, mul_rz, mul_rx, n_mul, bmul);
  Transcript t;
  t.tape.assign(proof, proof + len);
  u128 w = 0;
  std::vector<u128> point;
  int rc = shift_verify(public_words, log_words, log_public, ao, mo, band, bmul, t, w, point);
  if (rc == 0 && t.pos != t.tape.size()) rc = 3;
  store(out_eval, w);
  for (size_t i = 0; i < point.size(); i++) store(out_point + 2 * i, point[i]);
  return rc;
}

void orc_oblong_eval(const uint64_t* v, uint32_t log_n, const uint64_t* z, const uint64_t* r_x,
                     uint64_t* out) {
  std::vector<u128> rx(log_n);
  for (uint32_t i = 0; i < log_n; i++) rx[i] = load(r_x + 2 * i);
  store(out, oblong_eval(v, log_n, load(z), rx.data()));
}

}  // extern "C"
