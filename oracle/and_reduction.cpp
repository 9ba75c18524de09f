// CPU oracle (test infrastructure only): operand evaluation and the AND reduction (oblong
// zerocheck with a univariate skip round), prover and verifier.
//
// Restates:
//   eval_shifted_word / eval_operand   verifier/core/src/verify.rs:14-35, word.rs:140-245
//   prove_bitand_reduction             prover/prover/src/prove.rs:329-372
//   OblongZerocheckProver              prover/prover/src/and_reduction/prover.rs:74-276
//   univariate round                   and_reduction/sumcheck_round_messages.rs:62-136,
//                                      and_reduction/ntt_lookup.rs:91-164, prover_setup.rs:26-49
//   fold                               and_reduction/fold_lookup.rs:18-92, utils/multivariate.rs:16-57
//   MLE-check                          protocols/sumcheck/quadratic_mle.rs:21-196, gruen32.rs:29-131,
//                                      round_evals.rs:58-142, prove.rs:89-121
//   verifier                           verifier/verifier/src/and_reduction/verifier.rs:26-79,
//                                      protocols/mlecheck.rs:9-50,
//                                      and_reduction/univariate/{univariate_poly,univariate_lagrange}.rs
// The univariate message is the interpolation of each 64-bit word (bit t = value at the domain
// point t of the 6-dimensional subspace of GF(2^8) with basis 1, 2, .., 32) evaluated at the 64
// points 64..127; any exact method gives the same field values, so the oracle evaluates the
// Lagrange basis directly, tabulated per byte of the word.
#include <string.h>

#include <mutex>
#include <vector>

#include "oracle.h"
#include "oracle_internal.h"
#include "protocols.h"
#include "transcript.h"

namespace orc {

// ---------------------------------------------------------------- operands

uint64_t shifted_word(uint64_t w, uint32_t variant, uint32_t amount) {
  uint32_t n = amount;
  uint32_t lo = (uint32_t)w, hi = (uint32_t)(w >> 32), n5 = n & 31;
  switch (variant) {
    case 0: return n >= 64 ? 0 : (w << n);                                  // Sll
    case 1: return n >= 64 ? 0 : (w >> n);                                  // Slr
    case 2: return (uint64_t)((int64_t)w >> (n >= 64 ? 63 : n));            // Sar
    case 3: return n % 64 == 0 ? w : ((w >> (n % 64)) | (w << (64 - n % 64)));  // Rotr
    case 4: return ((uint64_t)(hi << n5) << 32) | (uint32_t)(lo << n5);     // Sll32
    case 5: return ((uint64_t)(hi >> n5) << 32) | (uint32_t)(lo >> n5);     // Srl32
    case 6:
      return ((uint64_t)(uint32_t)((int32_t)hi >> n5) << 32) | (uint32_t)((int32_t)lo >> n5);
    case 7: {
      uint32_t l = n5 ? ((lo >> n5) | (lo << (32 - n5))) : lo;
      uint32_t h = n5 ? ((hi >> n5) | (hi << (32 - n5))) : hi;
      return ((uint64_t)h << 32) | l;
    }
  }
  return 0;
}

// ---------------------------------------------------------------- GF(2^8) / Lagrange helpers

static u128 phi(uint8_t b) {
  static u128 table[256];
  static bool ready = false;
  if (!ready) {
    aes_to_ghash_table(table);
    ready = true;
  }
  return table[b];
}

static uint8_t aes_inv(uint8_t a) {
  if (!a) return 0;
  uint8_t r = 1;
  for (int i = 0; i < 254; i++) r = aes_mul(r, a);
  return r;
}

// Lagrange basis of the subspace {0, .., 2^dim - 1} of GF(2^8) (basis 1, 2, 4, ..) at x.
static void lagrange_aes(uint32_t dim, uint8_t x, uint8_t* out) {
  uint32_t n = 1u << dim;
  uint8_t denom = 1;
  for (uint32_t u = 1; u < n; u++) denom = aes_mul(denom, (uint8_t)u);
  uint8_t dinv = aes_inv(denom);
  for (uint32_t t = 0; t < n; t++) {
    uint8_t num = 1;
    for (uint32_t s = 0; s < n; s++)
      if (s != t) num = aes_mul(num, x ^ (uint8_t)s);
    out[t] = aes_mul(num, dinv);
  }
}

// Lagrange basis of the subspace {phi(t) : t < 2^dim} of GF(2^128) at x (lexicographic order).
static void lagrange_b128(uint32_t dim, u128 x, u128* out) {
  uint32_t n = 1u << dim;
  u128 denom = 1;
  for (uint32_t u = 1; u < n; u++) denom = gf_mul(denom, phi((uint8_t)u));
  u128 dinv = gf_inv(denom);
  std::vector<u128> diff(n);
  for (uint32_t s = 0; s < n; s++) diff[s] = x ^ phi((uint8_t)s);
  // products excluding one element
  std::vector<u128> suffix(n + 1);
  suffix[n] = 1;
  for (int s = (int)n - 1; s >= 0; s--) suffix[s] = gf_mul(suffix[s + 1], diff[s]);
  u128 prefix = 1;
  for (uint32_t t = 0; t < n; t++) {
    out[t] = gf_mul(gf_mul(prefix, suffix[t + 1]), dinv);
    prefix = gf_mul(prefix, diff[t]);
  }
}

static void eq_aes(const uint8_t* r, uint32_t n, uint8_t* out) {
  out[0] = 1;
  uint32_t len = 1;
  for (uint32_t i = 0; i < n; i++) {
    for (uint32_t j = 0; j < len; j++) {
      uint8_t prod = aes_mul(out[j], r[i]);
      out[j] ^= prod;
      out[len + j] = prod;
    }
    len <<= 1;
  }
}

// ---------------------------------------------------------------- AND reduction prover


static const uint8_t kSmallChallenges[3] = {0x2, 0x4, 0x10};  // config.rs:33-37

// Evaluations of each 64-bit word's interpolant at the 64 points 64..127: val[k] = sum over set
// bits t of M[k][t], M[k][t] the Lagrange basis polynomial of domain point t at 64 + k.  The map is
// linear in the word's bits, so it is tabulated per byte of the word (the byte-chunked lookup of
// and_reduction/ntt_lookup.rs:91-164): tab[p][v] holds the 64 values of the word whose byte p is
// v and whose other bytes are zero, and a word's values are the XOR of its eight byte rows.
struct WordNtt {
  uint64_t tab[8][256][8];  // 64 output bytes per row, as eight 8-byte words
  WordNtt() {
    uint8_t M[64][64];
    for (int k = 0; k < 64; k++) lagrange_aes(6, (uint8_t)(64 + k), M[k]);
    for (int p = 0; p < 8; p++)
      for (int v = 0; v < 256; v++) {
        uint8_t row[64] = {0};
        for (int bit = 0; bit < 8; bit++)
          if ((v >> bit) & 1)
            for (int k = 0; k < 64; k++) row[k] ^= M[k][8 * p + bit];
        memcpy(tab[p][v], row, 64);
      }
  }
  void eval(uint64_t w, uint8_t out[64]) const {
    uint64_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int p = 0; p < 8; p++) {
      const uint64_t* r = tab[p][(w >> (8 * p)) & 0xff];
      for (int q = 0; q < 8; q++) acc[q] ^= r[q];
    }
    memcpy(out, acc, 64);
  }
};

// The AES-field product as a 256 x 256 table (the same values as aes_mul).
struct AesMulTable {
  uint8_t t[256][256];
  AesMulTable() {
    for (int a = 0; a < 256; a++)
      for (int b = 0; b < 256; b++) t[a][b] = aes_mul((uint8_t)a, (uint8_t)b);
  }
};

void univariate_round(const uint64_t* a, const uint64_t* b, const uint64_t* c, uint32_t log_n,
                      const u128* big, u128 msg[64]) {
  static const WordNtt ntt;
  static const AesMulTable mul;
  uint8_t eq_small[8];
  eq_aes(kSmallChallenges, 3, eq_small);
  size_t n_chunks = (size_t)1 << (log_n - 3);
  std::vector<u128> eq_big(n_chunks);
  eq_ind_partial_eval(big, log_n - 3, eq_big.data());
  for (int k = 0; k < 64; k++) msg[k] = 0;
  std::vector<u128> partial(64 * (size_t)num_threads());
  parallel_for(n_chunks, [&](size_t lo, size_t hi) {
    u128 acc[64] = {0};
    for (size_t ch = lo; ch < hi; ch++) {
      uint8_t summed[64] = {0};
      for (int j = 0; j < 8; j++) {
        size_t i = ch * 8 + j;
        uint8_t va[64], vb[64], vc[64];
        ntt.eval(a[i], va);
        ntt.eval(b[i], vb);
        ntt.eval(c[i], vc);
        const uint8_t* by_eq = mul.t[eq_small[j]];
        for (int k = 0; k < 64; k++) summed[k] ^= by_eq[mul.t[va[k]][vb[k]] ^ vc[k]];
      }
      for (int k = 0; k < 64; k++) acc[k] ^= gf_mul(eq_big[ch], phi(summed[k]));
    }
    static std::mutex m;
    std::lock_guard<std::mutex> g(m);
    for (int k = 0; k < 64; k++) msg[k] ^= acc[k];
  });
}

// Folds each word into sum_t bit_t(w) L_t(z) over the domain {phi(t) : t < 64}.
// The sum is linear in the word's bits, so it is tabulated per byte: tab[p][v] = sum over the set
// bits b of v of lag[8p + b], and a word's sum is the XOR of its eight byte entries.
void fold_words(const uint64_t* w, size_t n, const u128 lag[64], u128* out) {
  std::vector<u128> tab(8 * 256);
  for (int p = 0; p < 8; p++) {
    u128* tp = tab.data() + 256 * p;
    tp[0] = 0;
    for (int v = 1; v < 256; v++) tp[v] = tp[v & (v - 1)] ^ lag[8 * p + __builtin_ctz(v)];
  }
  parallel_for(n, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; i++) {
      const uint64_t x = w[i];
      u128 acc = 0;
      for (int p = 0; p < 8; p++) acc ^= tab[256 * p + ((x >> (8 * p)) & 0xff)];
      out[i] = acc;
    }
  });
}

AndOutput and_reduction_prove(const uint64_t* a, const uint64_t* b, const uint64_t* c,
                              uint32_t log_n, Transcript& t) {
  AndOutput out;
  std::vector<u128> big(log_n - 3);
  for (auto& v : big) v = t.sample();
  u128 msg[64];
  univariate_round(a, b, c, log_n, big.data(), msg);
  t.message_elems(msg, 64);
  const u128 z = t.sample();
  out.z = z;
  // fold the three columns
  u128 lag64[64];
  lagrange_b128(6, z, lag64);
  const size_t N = (size_t)1 << log_n;
  std::vector<u128> fa(N), fb(N), fc(N);
  fold_words(a, N, lag64, fa.data());
  fold_words(b, N, lag64, fb.data());
  fold_words(c, N, lag64, fc.data());
  // claim = first round message (zero on the base domain) evaluated at z over 128 points
  u128 lag128[128];
  lagrange_b128(7, z, lag128);
  u128 sum = 0;
  for (int k = 0; k < 64; k++) sum ^= gf_mul(msg[k], lag128[64 + k]);
  // MLE-check over eval point [phi(2), phi(4), phi(16)] ++ big
  std::vector<u128> point{phi(2), phi(4), phi(16)};
  point.insert(point.end(), big.begin(), big.end());
  std::vector<u128> challenges;
  for (uint32_t n_rem = log_n; n_rem > 0; n_rem--) {
    const size_t half = (size_t)1 << (n_rem - 1);
    std::vector<u128> eq(half);
    eq_ind_partial_eval(point.data(), n_rem - 1, eq.data());
    u128 y1 = 0, yinf = 0;
    std::mutex m;
    parallel_for(half, [&](size_t lo, size_t hi) {  // XOR sums: any split gives the same value
      u128 s1 = 0, sinf = 0;
      for (size_t i = lo; i < hi; i++) {
        u128 a1 = fa[half + i], b1 = fb[half + i], c1 = fc[half + i];
        u128 ai = fa[i] ^ a1, bi = fb[i] ^ b1;
        s1 ^= gf_mul(eq[i], gf_mul(a1, b1) ^ c1);
        sinf ^= gf_mul(eq[i], gf_mul(ai, bi));
      }
      std::lock_guard<std::mutex> g(m);
      y1 ^= s1;
      yinf ^= sinf;
    });
    const u128 alpha = point[n_rem - 1];
    // RoundEvals2::interpolate_eq: y0 = (sum - y1 alpha) / (1 - alpha)
    const u128 y0 = gf_mul(sum ^ gf_mul(y1, alpha), gf_inv(1 ^ alpha));
    const u128 c0 = y0, c2 = yinf, c1 = y1 ^ c0 ^ c2;
    u128 rp[2] = {c1, c2};  // mlecheck::RoundProof::truncate drops c0
    t.message_elems(rp, 2);
    const u128 r = t.sample();
    challenges.push_back(r);
    sum = c0 ^ gf_mul(c1, r) ^ gf_mul(c2, gf_mul(r, r));
    parallel_for(half, [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; i++) {
        fa[i] ^= gf_mul(r, fa[half + i] ^ fa[i]);
        fb[i] ^= gf_mul(r, fb[half + i] ^ fb[i]);
        fc[i] ^= gf_mul(r, fc[half + i] ^ fc[i]);
      }
    });
  }
  u128 evals[3] = {fa[0], fb[0], fc[0]};
  t.message_elems(evals, 3);
  out.a_eval = fa[0];
  out.b_eval = fb[0];
  out.c_eval = fc[0];
  out.eval_point.assign(challenges.rbegin(), challenges.rend());
  return out;
}

// verify_with_transcript (verifier/verifier/src/and_reduction/verifier.rs:26-79).
bool and_reduction_verify(uint32_t log_n, Transcript& t, AndOutput& out) {
  std::vector<u128> big(log_n - 3);
  for (auto& v : big) v = t.sample();
  u128 msg[64];
  if (!t.read_message((uint8_t*)msg, sizeof(msg))) return false;
  const u128 z = t.sample();
  u128 lag128[128];
  lagrange_b128(7, z, lag128);
  u128 eval = 0;
  for (int k = 0; k < 64; k++) eval ^= gf_mul(msg[k], lag128[64 + k]);
  std::vector<u128> point{phi(2), phi(4), phi(16)};
  point.insert(point.end(), big.begin(), big.end());
  std::vector<u128> challenges;
  for (int i = (int)point.size() - 1; i >= 0; i--) {
    u128 rp[2];
    if (!t.read_message((uint8_t*)rp, 32)) return false;
    const u128 r = t.sample();
    const u128 c0 = eval ^ gf_mul(point[i], rp[0] ^ rp[1]);
    eval = c0 ^ gf_mul(rp[0], r) ^ gf_mul(rp[1], gf_mul(r, r));
    challenges.push_back(r);
  }
  u128 ev[3];
  if (!t.read_message((uint8_t*)ev, 48)) return false;
  if (eval != (gf_mul(ev[0], ev[1]) ^ ev[2])) return false;
  out.a_eval = ev[0];
  out.b_eval = ev[1];
  out.c_eval = ev[2];
  out.z = z;
  out.eval_point.assign(challenges.rbegin(), challenges.rend());
  return true;
}

}  // namespace orc

using namespace orc;

extern "C" {

uint64_t orc_shifted_word(uint64_t w, uint32_t variant, uint32_t amount) {
  return shifted_word(w, variant, amount);
}

// The 64 univariate-round evaluations for explicit big-field challenges (log_n - 3 of them).
void orc_and_univariate_round(const uint64_t* a, const uint64_t* b, const uint64_t* c,
                              uint32_t log_n, const uint64_t* big, uint64_t* msg_out) {
  univariate_round(a, b, c, log_n, (const u128*)big, (u128*)msg_out);
}

// The univariate round's per-word extension evaluations (NTTLookup::ntt, ntt_lookup.rs:91-164):
// out[k] = the word's interpolant over {0..63} in GF(2^8) at the point 64 + k.
void orc_and_word_ntt(uint64_t w, uint8_t out[64]) {
  static const WordNtt ntt;
  ntt.eval(w, out);
}

// Words folded at z: out[i] = sum_t bit_t(w[i]) L_t(z) over {phi(t) : t < 64}.
void orc_and_fold_words(const uint64_t* w, size_t n, const uint64_t* z, uint64_t* out) {
  u128 lag[64];
  lagrange_b128(6, load(z), lag);
  fold_words(w, n, lag, (u128*)out);
}

// Runs the AND reduction on a fresh transcript.  out_meta: a, b, c evals, z (4 elements);
// out_point: log_n elements.
int orc_and_reduction_prove(const uint64_t* a, const uint64_t* b, const uint64_t* c,
                            uint32_t log_n, uint8_t* proof_out, size_t cap, size_t* len,
                            uint64_t* out_meta, uint64_t* out_point) {
  if (log_n < 3) return 1;
  Transcript t;
  AndOutput o = and_reduction_prove(a, b, c, log_n, t);
  *len = t.tape.size();
  if (t.tape.size() > cap) return 2;
  memcpy(proof_out, t.tape.data(), t.tape.size());
  store(out_meta + 0, o.a_eval);
  store(out_meta + 2, o.b_eval);
  store(out_meta + 4, o.c_eval);
  store(out_meta + 6, o.z);
  for (uint32_t i = 0; i < log_n; i++) store(out_point + 2 * i, o.eval_point[i]);
  return 0;
}

int orc_and_reduction_verify(uint32_t log_n, const uint8_t* proof, size_t len, uint64_t* out_meta,
                             uint64_t* out_point) {
  Transcript t;
  t.tape.assign(proof, proof + len);
  AndOutput o;
  if (!and_reduction_verify(log_n, t, o)) return 1;
  if (t.pos != t.tape.size()) return 2;
  store(out_meta + 0, o.a_eval);
  store(out_meta + 2, o.b_eval);
  store(out_meta + 4, o.c_eval);
  store(out_meta + 6, o.z);
  for (uint32_t i = 0; i < log_n; i++) store(out_point + 2 * i, o.eval_point[i]);
  return 0;
}

}  // extern "C"
