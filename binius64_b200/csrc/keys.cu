// The shift reduction's KeyCollection (prover/prover/src/protocols/shift/key_collection.rs) for
// drop-in setup: build_key_collection (:238-312) with its v1 wire format (:314-431), and
// Prover::setup_with_key_collection (prover/prover/src/prove.rs:89-115) -- a constraint system
// whose shift term table is rebuilt from a serialized KeyCollection instead of from its operands.
//
// The reference builds the collection word by word with a linear search per term; the same bytes
// come here from counting sorts: operand terms in the reference's traversal order (AND a, b, c
// then MUL a, b, lo, hi, each over the constraints in order) are grouped by word (stably), each
// word's keys numbered by first appearance through a table indexed by (operation, id), and each
// key's constraint indices ordered stably by operand index.  The device term table
// (ShiftTerms, sorted by shift key) carries the same terms; its order inside a key only changes
// the order of XOR additions.
//
// The reference trusts a loaded collection; here it is also checked against the constraint
// system (one key range per committed word, ranges and index ranges that tile their vectors,
// operand and constraint indices in range, every constraint index owned by exactly one key), so
// a collection built for another constraint system is an argument error, not a wrong proof.
#include <string.h>

#include <algorithm>
#include <memory>
#include <thread>
#include <vector>

#include "cs.h"
#include "internal.h"

using namespace bgpu;

namespace {

constexpr uint32_t kKcVersion = 1;
constexpr uint32_t kKidCount = 2 * 512;  // (operation, id): id = variant * 64 + amount

inline uint8_t* put_u32(uint8_t* p, uint32_t v) {
  memcpy(p, &v, 4);
  return p + 4;
}

// One operand term as a 64-bit record: constraint (bits 0..31), operand index (32..33) and
// kid = operation << 9 | id (34..43).
inline uint64_t record(uint32_t constraint, uint32_t operand, uint32_t kid) {
  return (uint64_t)constraint | ((uint64_t)operand << 32) | ((uint64_t)kid << 34);
}

// The traversal as groups (pass, constraint): the passes are AND operands a, b, c then MUL
// operands a, b, lo, hi, each over the constraints in order; group gi of the flat sequence.
struct Passes {
  const HostOperands* h[7];
  uint32_t operation[7], operand[7], slot[7];
  uint64_t first[8];  // first[p] = flat index of pass p's first group
  explicit Passes(const binius_cs& cs) {
    static const uint32_t mul_slot[4] = {0, 1, 3, 2};  // operands (a, b, lo, hi) in CSR slots
    first[0] = 0;
    for (uint32_t p = 0; p < 7; p++) {
      const bool is_and = p < 3;
      h[p] = is_and ? &cs.h_and : &cs.h_mul;
      operation[p] = is_and ? 0 : 1;
      operand[p] = is_and ? p : p - 3;
      slot[p] = is_and ? p : mul_slot[p - 3];
      first[p + 1] = first[p] + (h[p]->offsets.size() - 1) / h[p]->k;
    }
  }
  uint64_t n_groups() const { return first[7]; }
  // Calls fn(word, record) for every term of groups [g0, g1), in traversal order.
  template <class Fn>
  void visit(uint64_t g0, uint64_t g1, Fn&& fn) const {
    for (uint32_t p = 0; p < 7; p++) {
      const uint64_t lo = g0 > first[p] ? g0 : first[p], hi = g1 < first[p + 1] ? g1 : first[p + 1];
      const HostOperands& H = *h[p];
      for (uint64_t gi = lo; gi < hi; gi++) {
        const uint32_t c = (uint32_t)(gi - first[p]), g = c * H.k + slot[p];
        for (uint32_t t = H.offsets[g]; t < H.offsets[g + 1]; t++) {
          const uint32_t packed = H.terms[t].y;  // variant << 8 | amount
          const uint32_t kid = (operation[p] << 9) | ((packed >> 8) << 6) | (packed & 255);
          fn(H.terms[t].x, record(c, operand[p], kid));
        }
      }
    }
  }
};

template <class Fn>
void parallel(uint32_t T, Fn&& fn) {
  std::vector<std::thread> th;
  for (uint32_t j = 1; j < T; j++) th.emplace_back(fn, j);
  fn(0u);
  for (auto& x : th) x.join();
}

// The collection's bytes.  Threads split the traversal (a stable scatter of the records by word
// through per-thread counts) and then the words (keys numbered per word; a word's constraint
// indices start at its first record, so only the key ranges need the threads' key counts).
int key_collection_bytes(const binius_cs& cs, std::vector<uint8_t>& out) {
  const uint32_t n_words = cs.committed_total_len;
  const size_t n = cs.h_and.terms.size() + cs.h_mul.terms.size();
  const Passes P(cs);
  uint32_t T = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
  // per-thread word counts: T * n_words * 4 bytes of host memory, held to 128 MiB (8 threads up
  // to 2^22 words; a 2^20-word system holds 32 MiB of counts)
  while (T > 1 && (uint64_t)T * n_words > (1ull << 25)) T--;
  if (n < (1u << 16)) T = 1;
  // stable group by word: per-thread counts over contiguous group ranges, then offsets
  const uint64_t NG = P.n_groups();
  std::vector<uint64_t> gcut(T + 1);
  for (uint32_t j = 0; j <= T; j++) gcut[j] = NG * j / T;
  std::vector<std::vector<uint32_t>> cnt(T, std::vector<uint32_t>(n_words, 0));
  parallel(T, [&](uint32_t j) {
    uint32_t* c = cnt[j].data();
    P.visit(gcut[j], gcut[j + 1], [&](uint32_t w, uint64_t) { c[w]++; });
  });
  std::vector<uint32_t> start((size_t)n_words + 1, 0);
  parallel(T, [&](uint32_t j) {  // per word: total, kept in start[w + 1] for the scan below
    const uint32_t w0 = (uint32_t)((uint64_t)n_words * j / T), w1 = (uint32_t)((uint64_t)n_words * (j + 1) / T);
    for (uint32_t w = w0; w < w1; w++) {
      uint32_t s = 0;
      for (uint32_t q = 0; q < T; q++) s += cnt[q][w];
      start[w + 1] = s;
    }
  });
  for (uint32_t w = 0; w < n_words; w++) start[w + 1] += start[w];
  parallel(T, [&](uint32_t j) {  // thread q's first slot of word w: start[w] + counts of q' < q
    const uint32_t w0 = (uint32_t)((uint64_t)n_words * j / T), w1 = (uint32_t)((uint64_t)n_words * (j + 1) / T);
    for (uint32_t w = w0; w < w1; w++) {
      uint32_t run = start[w];
      for (uint32_t q = 0; q < T; q++) {
        const uint32_t c = cnt[q][w];
        cnt[q][w] = run;
        run += c;
      }
    }
  });
  std::unique_ptr<uint64_t[]> rec(new uint64_t[n ? n : 1]);
  parallel(T, [&](uint32_t j) {
    uint32_t* fill = cnt[j].data();
    P.visit(gcut[j], gcut[j + 1], [&](uint32_t w, uint64_t r) { rec[fill[w]++] = r; });
  });
  cnt.clear();
  cnt.shrink_to_fit();
  // per word range: keys in first-appearance order, constraint indices bucketed by (key, operand)
  std::vector<uint32_t> wcut(T + 1);
  for (uint32_t j = 0, w = 0; j <= T; j++) {  // balance the words by records
    const uint64_t target = (uint64_t)n * j / T;
    while (w < n_words && start[w] < target) w++;
    wcut[j] = j == T ? n_words : w;
  }
  std::unique_ptr<uint8_t[]> cis_b(new uint8_t[5 * (n ? n : 1)]);
  std::vector<std::vector<uint8_t>> keys_j(T);
  std::vector<std::vector<uint32_t>> nk_j(T);  // keys per word of the range
  parallel(T, [&](uint32_t j) {
    std::vector<int32_t> local(kKidCount, -1);
    std::vector<uint32_t> word_kids, key_fill;
    std::vector<uint64_t> bucket;
    std::vector<uint8_t>& kb = keys_j[j];
    std::vector<uint32_t>& nkw = nk_j[j];
    nkw.reserve(wcut[j + 1] - wcut[j]);
    kb.reserve(11ull * (start[wcut[j + 1]] - start[wcut[j]]) / 2);
    for (uint32_t w = wcut[j]; w < wcut[j + 1]; w++) {
      const uint64_t* r = rec.get() + start[w];
      const uint32_t m = start[w + 1] - start[w];
      word_kids.clear();
      for (uint32_t q = 0; q < m; q++) {
        const uint32_t kid = (uint32_t)(r[q] >> 34);
        if (local[kid] < 0) {
          local[kid] = (int32_t)word_kids.size();
          word_kids.push_back(kid);
        }
      }
      const uint32_t nk = (uint32_t)word_kids.size();
      key_fill.assign(4 * nk + 1, 0);
      for (uint32_t q = 0; q < m; q++)
        key_fill[4 * local[r[q] >> 34] + ((r[q] >> 32) & 3) + 1]++;
      for (uint32_t x = 0; x < 4 * nk; x++) key_fill[x + 1] += key_fill[x];
      bucket.resize(m);
      for (uint32_t q = 0; q < m; q++)
        bucket[key_fill[4 * local[r[q] >> 34] + ((r[q] >> 32) & 3)]++] = r[q];
      uint8_t* cp = cis_b.get() + 5ull * start[w];
      for (uint32_t k = 0, x = 0; k < nk; k++) {
        const uint32_t kid = word_kids[k], end = key_fill[4 * k + 3];  // bucket ends after the fill
        uint8_t key[11];
        key[0] = (uint8_t)(kid >> 9);  // Operation: BitwiseAnd = 0, IntegerMul = 1
        key[1] = (uint8_t)(kid & 255);
        key[2] = (uint8_t)((kid >> 8) & 1);
        put_u32(key + 3, start[w] + x);
        for (; x < end; x++) {
          *cp++ = (uint8_t)((bucket[x] >> 32) & 3);
          cp = put_u32(cp, (uint32_t)bucket[x]);
        }
        put_u32(key + 7, start[w] + x);
        kb.insert(kb.end(), key, key + 11);
      }
      nkw.push_back(nk);
      for (uint32_t kid : word_kids) local[kid] = -1;
    }
  });
  std::vector<uint64_t> kbase(T + 1, 0);
  for (uint32_t j = 0; j < T; j++) kbase[j + 1] = kbase[j] + keys_j[j].size() / 11;
  const uint64_t n_keys = kbase[T];
  BGPU_ARG(n_keys <= 0xffffffffull, "too many keys");
  const size_t key_off = 8, ranges_off = key_off + 11 * n_keys + 4, cis_off = ranges_off + 8ull * n_words + 4;
  out.resize(cis_off + 5 * n);
  uint8_t* o = out.data();
  put_u32(o, kKcVersion);
  put_u32(o + 4, (uint32_t)n_keys);
  put_u32(o + ranges_off - 4, n_words);
  put_u32(o + cis_off - 4, (uint32_t)n);
  parallel(T, [&](uint32_t j) {
    if (!keys_j[j].empty()) memcpy(o + key_off + 11 * kbase[j], keys_j[j].data(), keys_j[j].size());
    uint32_t k = (uint32_t)kbase[j];
    uint8_t* rp = o + ranges_off + 8ull * wcut[j];
    for (uint32_t nk : nk_j[j]) {
      rp = put_u32(rp, k);
      rp = put_u32(rp, k + nk);
      k += nk;
    }
    const uint64_t c0 = start[wcut[j]], c1 = start[wcut[j + 1]];
    if (c1 > c0) memcpy(o + cis_off + 5 * c0, cis_b.get() + 5 * c0, 5 * (c1 - c0));
  });
  return BINIUS_OK;
}

struct KcReader {
  const uint8_t* p;
  size_t len, pos = 0;
  bool ok = true;
  uint32_t u32() {
    if (len - pos < 4) {
      ok = false;
      return 0;
    }
    uint32_t v;
    memcpy(&v, p + pos, 4);
    pos += 4;
    return v;
  }
  const uint8_t* take(size_t n) {
    if (len - pos < n) {
      ok = false;
      return nullptr;
    }
    const uint8_t* at = p + pos;
    pos += n;
    return at;
  }
};

// KeyCollection::deserialize and the terms it describes, checked against the constraint system's
// layout and constraint counts, uploaded as the device term table sorted by shift key.
int load_key_collection(binius_cs& cs, const uint8_t* kc, size_t len) {
  KcReader r{kc, len};
  BGPU_ARG(r.u32() == kKcVersion && r.ok, "InvalidConstruction: KeyCollection::version");
  const uint32_t n_keys = r.u32();
  const uint8_t* keys = r.take(11ull * n_keys);
  const uint32_t n_ranges = r.u32();
  const uint8_t* ranges = r.take(8ull * n_ranges);
  const uint32_t n_cis = r.u32();
  const uint8_t* cis = r.take(5ull * n_cis);
  BGPU_ARG(r.ok, "NotEnoughBytes: KeyCollection");
  BGPU_ARG(r.pos == len, "KeyCollection: trailing bytes");
  BGPU_ARG(n_ranges == cs.committed_total_len, "KeyCollection: one key range per committed word");
  const uint32_t n_and = (uint32_t)((cs.h_and.offsets.size() - 1) / 3);
  const uint32_t n_mul = (uint32_t)((cs.h_mul.offsets.size() - 1) / 4);
  std::vector<uint32_t> vi(n_cis), cc(n_cis);
  std::vector<uint16_t> key(n_cis);
  std::vector<uint32_t> count(kShiftKeys + 1, 0);
  std::vector<uint8_t> seen(n_cis, 0);
  uint32_t expect_key = 0;
  for (uint32_t w = 0; w < n_ranges; w++) {
    uint32_t k0, k1;
    memcpy(&k0, ranges + 8ull * w, 4);
    memcpy(&k1, ranges + 8ull * w + 4, 4);
    BGPU_ARG(k0 == expect_key && k1 >= k0 && k1 <= n_keys, "KeyCollection: key ranges");
    expect_key = k1;
    for (uint32_t k = k0; k < k1; k++) {
      const uint8_t* kp = keys + 11ull * k;
      const uint32_t operation = kp[0], id = (uint32_t)kp[1] | ((uint32_t)kp[2] << 8);
      uint32_t c0, c1;
      memcpy(&c0, kp + 3, 4);
      memcpy(&c1, kp + 7, 4);
      BGPU_ARG(operation <= 1, "UnknownEnumVariant: Operation");
      BGPU_ARG(id < 512 && c0 <= c1 && c1 <= n_cis, "KeyCollection: key");
      for (uint32_t x = c0; x < c1; x++) {
        const uint8_t* cp = cis + 5ull * x;
        const uint32_t operand = cp[0];
        uint32_t c;
        memcpy(&c, cp + 1, 4);
        BGPU_ARG(!seen[x], "KeyCollection: a constraint index in two keys");
        BGPU_ARG(operation == 0 ? (operand < 3 && c < n_and) : (operand < 4 && c < n_mul),
                 "KeyCollection: constraint index out of range");
        seen[x] = 1;
        // shift key = id * 8 + class; class: AND operands 0..2, MUL operands (a, b, lo, hi) 3..6
        const uint32_t k8 = id * 8 + (operation == 0 ? operand : 3 + operand);
        vi[x] = w;
        cc[x] = c;
        key[x] = (uint16_t)k8;
        count[k8 + 1]++;
      }
    }
  }
  BGPU_ARG(expect_key == n_keys, "KeyCollection: keys outside every word's range");
  for (uint32_t x = 0; x < n_cis; x++) BGPU_ARG(seen[x], "KeyCollection: unowned constraint index");
  for (uint32_t k = 0; k < kShiftKeys; k++) count[k + 1] += count[k];
  const size_t m = n_cis ? n_cis : 1;
  std::vector<uint32_t> svi(m), scc(m);
  std::vector<uint16_t> skey(m);
  for (uint32_t x = 0; x < n_cis; x++) {
    const uint32_t pos = count[key[x]]++;
    svi[pos] = vi[x];
    scc[pos] = cc[x];
    skey[pos] = key[x];
  }
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(cs.device);
  const int rc = upload_shift_terms(svi, scc, skey, n_cis, cs.committed_total_len,
                                  cs.shift_terms);
  cudaSetDevice(prev);
  return rc;
}

int copy_out(const std::vector<uint8_t>& bytes, void* h_out, size_t cap, size_t* len) {
  *len = bytes.size();
  BGPU_ARG(cap >= bytes.size() && (h_out != nullptr || bytes.empty()), "output buffer too small");
  if (!bytes.empty()) memcpy(h_out, bytes.data(), bytes.size());
  return clear_error();
}

}  // namespace

extern "C" {

int binius_key_collection_from_cs_bytes(const void* h_cs_bytes, size_t cs_len, void* h_out,
                                        size_t cap, size_t* len) {
  BGPU_ARG(len != nullptr && (h_cs_bytes != nullptr || cs_len == 0), "NULL argument");
  binius_cs cs;
  if (int rc = parse_cs(h_cs_bytes, cs_len, cs)) return rc;
  std::vector<uint8_t> out;
  if (int rc = key_collection_bytes(cs, out)) return rc;
  return copy_out(out, h_out, cap, len);
}

int binius_cs_key_collection(const binius_cs* cs, void* h_out, size_t cap, size_t* len) {
  BGPU_ARG(cs != nullptr && len != nullptr, "NULL argument");
  std::vector<uint8_t> out;
  if (int rc = key_collection_bytes(*cs, out)) return rc;
  return copy_out(out, h_out, cap, len);
}

int binius_cs_load_key_collection(binius_cs* cs, const void* h_bytes, size_t len) {
  BGPU_ARG(cs != nullptr && (h_bytes != nullptr || len == 0), "NULL argument");
  if (int rc = load_key_collection(*cs, static_cast<const uint8_t*>(h_bytes), len)) return rc;
  return clear_error();
}

int binius_prover_setup_with_key_collection(binius_cs* cs, uint32_t log_inv_rate,
                                            const void* h_kc, size_t kc_len, binius_prover** out) {
  BGPU_ARG(cs != nullptr && out != nullptr, "NULL argument");
  *out = nullptr;
  if (int rc = binius_cs_load_key_collection(cs, h_kc, kc_len)) return rc;
  return binius_prover_setup(cs, log_inv_rate, out);
}

}  // extern "C"
