// brute_eval.cpp — independent hand evaluator used to check the rank table.
//
// TEST INFRASTRUCTURE ONLY (part of liboracle.so; see oracle.cpp's header).
//
// Method: a 5-card hand is scored from the hand-ranking rules (rank-group
// pattern, flush, straight); the 7462 classes are numbered by sorting the
// distinct scores of all C(52,5) = 2,598,960 five-card hands; a 6- or 7-card hand
// takes the best of its C(n,5) subsets.  This shares no code with the table
// generator, which classifies 5..7 cards directly.
#include <algorithm>
#include <cstdint>
#include <mutex>
#include <thread>
#include <vector>

namespace {

// cards: 0..51 suit-major (card = suit*13 + rank)
uint64_t score5(const int* c) {
  int r[5], s[5];
  for (int i = 0; i < 5; ++i) {
    r[i] = c[i] % 13;
    s[i] = c[i] / 13;
  }
  bool flush = true;
  for (int i = 1; i < 5; ++i) flush = flush && (s[i] == s[0]);
  int cnt[13] = {0};
  for (int i = 0; i < 5; ++i) cnt[r[i]]++;
  // groups ordered by (size desc, rank desc)
  std::vector<std::pair<int, int>> g;
  for (int x = 12; x >= 0; --x)
    if (cnt[x]) g.push_back({cnt[x], x});
  std::stable_sort(g.begin(), g.end(),
                   [](const std::pair<int, int>& a, const std::pair<int, int>& b) { return a.first > b.first; });
  bool straight = false;
  int high = -1;
  if (g.size() == 5) {
    if (g[0].second - g[4].second == 4) {
      straight = true;
      high = g[0].second;
    } else if (g[0].second == 12 && g[1].second == 3) {  // A-5-4-3-2
      straight = true;
      high = 3;
    }
  }
  int cat;
  if (straight && flush) cat = 8;
  else if (g[0].first == 4) cat = 7;
  else if (g[0].first == 3 && g[1].first == 2) cat = 6;
  else if (flush) cat = 5;
  else if (straight) cat = 4;
  else if (g[0].first == 3) cat = 3;
  else if (g[0].first == 2 && g[1].first == 2) cat = 2;
  else if (g[0].first == 2) cat = 1;
  else cat = 0;
  uint64_t key = (uint64_t)cat << 40;
  if (cat == 8 || cat == 4) return key | ((uint64_t)high << 32);
  for (size_t i = 0; i < g.size(); ++i) key |= (uint64_t)g[i].second << (32 - 8 * i);
  return key;
}

std::vector<uint64_t>& classes() {
  static std::vector<uint64_t> v;
  static std::once_flag once;
  std::call_once(once, [] {
    std::vector<uint64_t> all;
    all.reserve(2598960);
    int c[5];
    for (c[0] = 0; c[0] < 52; ++c[0])
      for (c[1] = c[0] + 1; c[1] < 52; ++c[1])
        for (c[2] = c[1] + 1; c[2] < 52; ++c[2])
          for (c[3] = c[2] + 1; c[3] < 52; ++c[3])
            for (c[4] = c[3] + 1; c[4] < 52; ++c[4]) all.push_back(score5(c));
    std::sort(all.begin(), all.end());
    all.erase(std::unique(all.begin(), all.end()), all.end());
    v.swap(all);
  });
  return v;
}

int index_of(uint64_t key) {
  const auto& v = classes();
  return (int)(std::lower_bound(v.begin(), v.end(), key) - v.begin()) + 1;
}

uint64_t best_score(const int* cards, int n) {
  uint64_t best = 0;
  int sub[5];
  // all 5-subsets of n (n = 5..7) via bit masks
  for (int m = 0; m < (1 << n); ++m) {
    if (__builtin_popcount(m) != 5) continue;
    int k = 0;
    for (int i = 0; i < n; ++i)
      if (m & (1 << i)) sub[k++] = cards[i];
    best = std::max(best, score5(sub));
  }
  return best;
}

}  // namespace

extern "C" {

int brute_class_count(void) { return (int)classes().size(); }

// Best-hand rank 1..7462 of n = 5..7 cards (0..51 suit-major).
int brute_rank(const uint8_t* cards, int n) {
  int c[7];
  for (int i = 0; i < n; ++i) c[i] = cards[i];
  return index_of(best_score(c, n));
}

void brute_rank_batch(const uint8_t* cards, int n, uint16_t* out, size_t count, int nthreads) {
  classes();
  if (nthreads < 1) nthreads = 1;
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t)
    th.emplace_back([=] {
      for (size_t i = t; i < count; i += nthreads) {
        int c[7];
        for (int k = 0; k < n; ++k) c[k] = cards[i * n + k];
        out[i] = (uint16_t)index_of(best_score(c, n));
      }
    });
  for (auto& x : th) x.join();
}

}  // extern "C"
