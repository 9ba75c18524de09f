// CPU oracle (test infrastructure only): the shift reduction's KeyCollection and its v1 wire
// format, restated from prover/prover/src/protocols/shift/key_collection.rs:
//   build_key_collection   :247-312 (update_with_operand :170-245): per word, a list of builder
//                          keys found by linear search on (id, operation) in first-appearance
//                          order over the traversal AND a, b, c then MUL a, b, lo, hi, each over
//                          the constraints in order; a key's constraint indices are then stably
//                          sorted by operand index
//   serialization v1       :320-431 (Operation as u8, Key as u8 + u16 + u32 + u32, key ranges
//                          as u32 pairs, ConstraintIndex as u8 + u32, Vecs with u32 lengths)
#include <string.h>

#include <algorithm>
#include <vector>

#include "oracle.h"
#include "protocols.h"

namespace {

struct CIdx {
  uint8_t operand;
  uint32_t constraint;
};
struct BuilderKey {
  uint16_t id;
  uint8_t operation;
  std::vector<CIdx> cis;
};

void put_u8(std::vector<uint8_t>& o, uint8_t v) { o.push_back(v); }
void put_u16(std::vector<uint8_t>& o, uint16_t v) {
  o.push_back((uint8_t)v);
  o.push_back((uint8_t)(v >> 8));
}
void put_u32(std::vector<uint8_t>& o, uint32_t v) {
  for (int i = 0; i < 4; i++) o.push_back((uint8_t)(v >> (8 * i)));
}

}  // namespace

extern "C" {

// csr slot of operand o: AND (a, b, c) -> (0, 1, 2); MUL operands (a, b, lo, hi) sit in CSR slots
// (0, 1, 3, 2).  Writes the v1 bytes to out (cap bytes) and their length to *len; returns 2 when
// out is too small.
int orc_key_collection(const uint32_t* const* and_csr, const uint8_t* and_var, uint32_t n_and,
                       const uint32_t* const* mul_csr, const uint8_t* mul_var, uint32_t n_mul,
                       uint32_t n_words, uint8_t* out, size_t cap, size_t* len) {
  std::vector<std::vector<BuilderKey>> lists(n_words);
  auto update = [&](uint8_t operation, uint32_t k, uint32_t n, const uint32_t* const* csr,
                    const uint8_t* var, uint32_t operand, uint32_t slot) {
    const uint32_t* off = csr[0];
    const uint32_t* vi = csr[1];
    const uint32_t* amt = csr[2];
    for (uint32_t c = 0; c < n; c++) {
      const uint32_t g = c * k + slot;
      for (uint32_t t = off[g]; t < off[g + 1]; t++) {
        auto& keys = lists[vi[t]];
        const uint16_t id = (uint16_t)(((uint32_t)var[t] << 6) + amt[t]);
        auto it = std::find_if(keys.begin(), keys.end(), [&](const BuilderKey& b) {
          return b.id == id && b.operation == operation;
        });
        if (it != keys.end())
          it->cis.push_back({(uint8_t)operand, c});
        else
          keys.push_back({id, operation, {{(uint8_t)operand, c}}});
      }
    }
  };
  for (uint32_t o = 0; o < 3; o++) update(0, 3, n_and, and_csr, and_var, o, o);
  static const uint32_t mul_slot[4] = {0, 1, 3, 2};
  for (uint32_t o = 0; o < 4; o++) update(1, 4, n_mul, mul_csr, mul_var, o, mul_slot[o]);

  std::vector<uint8_t> keys_b, ranges_b, cis_b;
  uint32_t n_keys = 0, n_cis = 0, key_off = 0;
  for (uint32_t w = 0; w < n_words; w++) {
    put_u32(ranges_b, key_off);
    key_off += (uint32_t)lists[w].size();
    put_u32(ranges_b, key_off);
    for (auto& b : lists[w]) {
      std::stable_sort(b.cis.begin(), b.cis.end(),
                       [](const CIdx& x, const CIdx& y) { return x.operand < y.operand; });
      put_u8(keys_b, b.operation);
      put_u16(keys_b, b.id);
      put_u32(keys_b, n_cis);
      for (const auto& ci : b.cis) {
        put_u8(cis_b, ci.operand);
        put_u32(cis_b, ci.constraint);
      }
      n_cis += (uint32_t)b.cis.size();
      put_u32(keys_b, n_cis);
      n_keys++;
    }
  }
  std::vector<uint8_t> o;
  put_u32(o, 1);
  put_u32(o, n_keys);
  o.insert(o.end(), keys_b.begin(), keys_b.end());
  put_u32(o, n_words);
  o.insert(o.end(), ranges_b.begin(), ranges_b.end());
  put_u32(o, n_cis);
  o.insert(o.end(), cis_b.begin(), cis_b.end());
  *len = o.size();
  if (o.size() > cap) return 2;
  memcpy(out, o.data(), o.size());
  return 0;
}

}  // extern "C"
