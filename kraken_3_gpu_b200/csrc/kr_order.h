// kr_order.h -- the launch order of live slots (host code, no CUDA).
//
// A launch's creatures are grouped by body template and, within a template,
// ordered longest remaining horizon first (LPT: the longest jobs start
// first, so the short ones fill the tail).  Ties keep the order of the slot
// list.  The engine re-orders every live slot before each launch -- every
// slice of a server -- so the order is computed by a stable LSD radix sort
// instead of a comparison sort, on one dense key per slot:
//   key = tpl * (R + 1) + (R - rem),   R = the largest rem of the set,
// which orders as (tpl ascending, rem descending) and needs only
// log2(templates x (R + 1)) bits -- 17 for 25 templates and horizons up to
// 4,096, two passes of 11-bit digits on 32-bit keys (64-bit keys when the
// product exceeds 2^32).  Digits that are the same for every key cost one
// histogram pass and no scatter.
#pragma once

#include <cstdint>
#include <vector>

namespace krb {

namespace detail {
// stable LSD radix sort of keys[0..n) carrying perm, 11-bit digits over the
// low `bits` bits
template <typename K>
inline void radix_by_key(int n, int bits, std::vector<K> &keys, std::vector<K> &keys2, std::vector<int> &perm,
                         std::vector<int> &perm2) {
  constexpr int kBits = 11, kRadix = 1 << kBits;
  const int digits = (bits + kBits - 1) / kBits;
  if (n <= 1 || digits == 0) return;
  keys2.resize(n);
  perm2.resize(n);
  std::vector<int> count((size_t)digits * kRadix, 0);
  for (int i = 0; i < n; i++)
    for (int d = 0; d < digits; d++) count[(size_t)d * kRadix + ((keys[i] >> (d * kBits)) & (kRadix - 1))]++;
  for (int d = 0; d < digits; d++) {
    int *c = count.data() + (size_t)d * kRadix;
    bool constant = false;
    for (int b = 0; b < kRadix; b++)
      if (c[b] == n) { constant = true; break; }
    if (constant) continue;
    int sum = 0;
    for (int b = 0; b < kRadix; b++) {
      const int k = c[b];
      c[b] = sum;
      sum += k;
    }
    for (int i = 0; i < n; i++) {
      const int dst = c[(keys[i] >> (d * kBits)) & (kRadix - 1)]++;
      keys2[dst] = keys[i];
      perm2[dst] = perm[i];
    }
    keys.swap(keys2);
    perm.swap(perm2);
  }
}

inline int bit_length(uint64_t v) {
  int b = 0;
  while (v) { b++; v >>= 1; }
  return b;
}
}  // namespace detail

// perm[0..n) = the positions 0..n-1 ordered by tpl ascending, then rem
// descending, then position ascending.  0 <= tpl[i] < 256, 0 <= rem[i] <
// 2^31.  The scratch vectors are reused between calls.
inline void lpt_order(int n, const int *tpl, const int *rem, std::vector<int> &perm, std::vector<uint64_t> &keys,
                      std::vector<uint64_t> &keys2, std::vector<int> &perm2) {
  perm.resize(n);
  int max_tpl = 0, max_rem = 0;
  for (int i = 0; i < n; i++) {
    perm[i] = i;
    if (tpl[i] > max_tpl) max_tpl = tpl[i];
    if (rem[i] > max_rem) max_rem = rem[i];
  }
  const uint64_t R = (uint64_t)max_rem;
  const uint64_t span = ((uint64_t)max_tpl + 1) * (R + 1);  // keys in [0, span)
  const int bits = detail::bit_length(span - 1);
  if (bits <= 32) {
    // 32-bit keys: half the memory traffic of 64-bit ones
    std::vector<uint32_t> k32(n), k32b;
    for (int i = 0; i < n; i++) k32[i] = (uint32_t)((uint64_t)tpl[i] * (R + 1) + (R - (uint64_t)rem[i]));
    detail::radix_by_key(n, bits, k32, k32b, perm, perm2);
    return;
  }
  keys.resize(n);
  for (int i = 0; i < n; i++) keys[i] = (uint64_t)tpl[i] * (R + 1) + (R - (uint64_t)rem[i]);
  detail::radix_by_key(n, bits, keys, keys2, perm, perm2);
}

}  // namespace krb
