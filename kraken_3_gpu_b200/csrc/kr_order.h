// kr_order.h -- the launch order of live slots (host code, no CUDA).
//
// A launch's creatures are grouped by body template and, within a template,
// ordered longest remaining horizon first (LPT: the longest jobs start
// first, so the short ones fill the tail).  Ties keep the order of the slot
// list.  The engine re-orders every live slot before each launch -- every
// slice of a server -- so the order is computed by a stable LSD radix sort of
// one 39-bit key per slot (template 8 bits, inverted remaining steps 31 bits)
// instead of a comparison sort: digits that are the same for every key (the
// high bits of the remaining steps when horizons are short, the template
// when there is one) cost one histogram pass and no scatter.
#pragma once

#include <cstdint>
#include <vector>

namespace krb {

// perm[0..n) = the positions 0..n-1 ordered by tpl ascending, then rem
// descending, then position ascending.  tpl[i] < 256, 0 <= rem[i] < 2^31.
// scratch vectors are reused between calls.
inline void lpt_order(int n, const int *tpl, const int *rem, std::vector<int> &perm,
                      std::vector<uint64_t> &keys, std::vector<uint64_t> &keys2, std::vector<int> &perm2) {
  constexpr int kBits = 11, kRadix = 1 << kBits, kDigits = 4;  // 44 bits >= 39
  perm.resize(n);
  keys.resize(n);
  keys2.resize(n);
  perm2.resize(n);
  for (int i = 0; i < n; i++) {
    keys[i] = ((uint64_t)(uint32_t)tpl[i] << 31) | (uint64_t)(0x7fffffffu - (uint32_t)rem[i]);
    perm[i] = i;
  }
  std::vector<int> count((size_t)kDigits * kRadix, 0);
  for (int i = 0; i < n; i++)
    for (int d = 0; d < kDigits; d++) count[(size_t)d * kRadix + ((keys[i] >> (d * kBits)) & (kRadix - 1))]++;
  for (int d = 0; d < kDigits; d++) {
    int *c = count.data() + (size_t)d * kRadix;
    bool constant = false;
    for (int b = 0; b < kRadix; b++)
      if (c[b] == n) { constant = true; break; }
    if (constant || n == 0) continue;
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

}  // namespace krb
