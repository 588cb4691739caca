// abstraction.cpp — host-side card-abstraction tables uploaded to the device.
//
//  * Chen-score percentile buckets (the reference's preflop abstraction,
//    poker_cuda/src/abstraction.cpp:10-59, uploaded as a 52x52 LUT by
//    cfr_gpu.cu:1164-1173);
//  * 169 lossless preflop classes;
//  * rank-CDF postflop buckets from exact rank histograms.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/mccfr.h"

namespace mccfr {

static float chen_score(int h0, int h1) {
  int r0 = h0 % 13, r1 = h1 % 13;
  const bool suited = (h0 / 13) == (h1 / 13);
  if (r0 < r1) std::swap(r0, r1);
  float base;
  switch (r0) {
    case 12: base = 10.f; break;
    case 11: base = 8.f; break;
    case 10: base = 7.f; break;
    case 9: base = 6.f; break;
    default: base = std::max(0.5f, r0 / 2.f);
  }
  if (r0 == r1) return std::max(5.f, base * 2.f);
  float score = base + (suited ? 2.f : 0.f);
  const int gap = r0 - r1 - 1;
  static const float gap_penalty[5] = {0.f, 1.f, 2.f, 4.f, 5.f};
  score -= gap_penalty[std::min(gap, 4)];
  if (gap <= 1 && r0 < 12) score += 1.f;
  return score;
}

void build_preflop_lut(int mode, int buckets, uint8_t* lut) {
  if (mode == MCCFR_PREFLOP_CHEN64) {
    std::vector<float> sorted;
    sorted.reserve(1326);
    for (int i = 0; i < 52; ++i)
      for (int j = i + 1; j < 52; ++j) sorted.push_back(chen_score(i, j));
    std::sort(sorted.begin(), sorted.end());
    for (int h0 = 0; h0 < 52; ++h0)
      for (int h1 = 0; h1 < 52; ++h1) {
        uint8_t v = 0;
        if (h0 != h1) {
          const float s = chen_score(h0, h1);
          const long below = std::lower_bound(sorted.begin(), sorted.end(), s) - sorted.begin();
          const float pct = (float)below / (float)sorted.size();
          v = (uint8_t)std::min((int)(pct * (float)buckets), buckets - 1);
        }
        lut[h0 * 52 + h1] = v;
      }
    return;
  }
  for (int h0 = 0; h0 < 52; ++h0)
    for (int h1 = 0; h1 < 52; ++h1) {
      const int a = h0 % 13, b = h1 % 13;
      const int hi = std::max(a, b), lo = std::min(a, b);
      int id;
      if (hi == lo) id = hi * 14;             // pair: diagonal
      else if (h0 / 13 == h1 / 13) id = hi * 13 + lo;  // suited: below the diagonal
      else id = lo * 13 + hi;                 // offsuit: above the diagonal
      lut[h0 * 52 + h1] = (h0 == h1) ? 0 : (uint8_t)id;
    }
}

// counts[r] = number of hands with rank r (0..7462); the bucket of rank r is its
// mid-rank percentile times `buckets`, floored, in exact integer arithmetic.
void build_cdf_lut(const unsigned long long* counts, int buckets, uint8_t* lut) {
  unsigned long long total = 0;
  for (int r = 0; r < 7463; ++r) total += counts[r];
  unsigned long long below = 0;
  for (int r = 0; r < 7463; ++r) {
    unsigned long long b = (2 * below + counts[r]) * (unsigned long long)buckets / (2 * total);
    if (b > (unsigned long long)(buckets - 1)) b = buckets - 1;
    lut[r] = (uint8_t)b;
    below += counts[r];
  }
}

}  // namespace mccfr
