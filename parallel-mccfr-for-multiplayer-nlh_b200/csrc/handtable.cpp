// Two Plus Two style 7-card hand-rank state machine (32,487,834 int32 entries).
//
// The reference never ships this table: it reads "HandRanks.dat" from disk
// (poker_cuda/src/hand_eval.cpp:88-102, poker_cuda/src/cfr_gpu.cu:1086-1104) and its
// generator is a stub (poker_cuda/tools/gen_lookup_table.cpp:63-97).  This file builds
// the table from the published method (the "2+2 forum" evaluator: a directed state
// machine over canonical partial hands), in this project's own code.
//
// Format (kept identical because the reference's lookups index it directly,
// hand_eval.cpp:47-57 and cfr_gpu.cu:114-150):
//   * a card is c = rank*4 + suit + 1 in 1..52 (rank 0 = deuce, suit 0..3);
//   * the first lookup is T[53 + c]; every later one is T[p + c];
//   * a state for k < 7 cards is s*53 + 53, where s is the position of the
//     state's canonical id in the ascending list of all ids of 0..6 cards;
//   * after the 7th card the entry is the packed rank (category << 12 | ordinal),
//     category 1 = high card .. 9 = straight flush; ordinal counts from 1 within
//     the category, so the decoded rank is 1 (worst) .. 7462 (royal flush);
//   * T[s*53 + 53] of a 5- or 6-card state holds that hand's packed rank;
//   * a card already in the hand leads to state 53 (or 0 after the 7th card).
//
// Canonical id: each card is a byte (rank+1) << 4 | (suit+1); once a hand has
// n >= 4 cards, a card's suit is dropped (low nibble 0) when fewer than n-2 cards
// of the hand share it, since that suit can no longer make a flush by the 7th
// card.  The bytes are sorted descending and packed little-endian into 64 bits.
// There are 612,977 ids (including the empty hand), so the table is exactly
// 612,978 * 53 entries.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "handtable.h"

namespace mccfr {
namespace {

constexpr int kCategoryBase[10] = {0, 0, 1277, 4137, 4995, 5853, 5863, 7140, 7296, 7452};

struct Extended {
  uint64_t id;  // 0 when the new card repeats a card or a rank would appear 5 times
  int n;        // number of cards counted, including the new one
};

// Adds card c (1..52) to the canonical id `id`.
Extended extend_id(uint64_t id, int c) {
  const int newbyte = ((((c - 1) >> 2) + 1) << 4) | (((c - 1) & 3) + 1);
  uint8_t cards[8];
  int n = 0;
  cards[n++] = (uint8_t)newbyte;
  bool repeated = false;
  for (int i = 0; i < 6; ++i) {
    const uint8_t b = (uint8_t)((id >> (8 * i)) & 0xFF);
    if (b == 0) break;
    if (b == newbyte) repeated = true;
    cards[n++] = b;
  }
  if (repeated) return {0, n};
  int suit_count[5] = {0, 0, 0, 0, 0};
  int rank_count[14] = {0};
  for (int i = 0; i < n; ++i) {
    suit_count[cards[i] & 0xF]++;
    rank_count[cards[i] >> 4]++;
  }
  if (n > 4)
    for (int r = 1; r <= 13; ++r)
      if (rank_count[r] > 4) return {0, n};
  const int need = n - 2;
  if (need > 1)
    for (int i = 0; i < n; ++i)
      if (suit_count[cards[i] & 0xF] < need) cards[i] &= 0xF0;
  std::sort(cards, cards + n, [](uint8_t a, uint8_t b) { return a > b; });
  uint64_t out = 0;
  for (int i = 0; i < n; ++i) out |= (uint64_t)cards[i] << (8 * i);
  return {out, n};
}

// ---------------------------------------------------------------------------
// Direct best-hand classifier.  Produces a key that orders hands by strength:
// category (0 = high card .. 8 = straight flush) in bits 20..23 and up to five
// significant ranks (0..12, most significant first) in 4-bit fields below.
// ---------------------------------------------------------------------------
inline int top_bit(uint32_t m) { return 31 - __builtin_clz(m); }

// Highest straight in a 13-bit rank mask: the rank of its top card, or -1.
int straight_high(uint32_t m) {
  const uint32_t wheel = (1u << 12) | 0xFu;  // A-2-3-4-5
  for (int hi = 12; hi >= 4; --hi) {
    const uint32_t run = 0x1Fu << (hi - 4);
    if ((m & run) == run) return hi;
  }
  if ((m & wheel) == wheel) return 3;
  return -1;
}

uint32_t pack_key(int cat, const int* r, int k) {
  uint32_t key = (uint32_t)cat << 20;
  for (int i = 0; i < k; ++i) key |= (uint32_t)r[i] << (16 - 4 * i);
  return key;
}

// Top `k` ranks of a mask, highest first.
int take_top(uint32_t m, int k, int* out) {
  int n = 0;
  while (m && n < k) {
    const int b = top_bit(m);
    out[n++] = b;
    m &= ~(1u << b);
  }
  return n;
}

// ranks[i] in 0..12, suits[i] in 0..4 (0 = suit cannot contribute to a flush).
uint32_t classify(const int* ranks, const int* suits, int n) {
  int count[13] = {0};
  uint32_t all = 0, by_suit[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < n; ++i) {
    count[ranks[i]]++;
    all |= 1u << ranks[i];
    by_suit[suits[i]] |= 1u << ranks[i];
  }
  int r[5];
  for (int s = 1; s <= 4; ++s) {
    if (__builtin_popcount(by_suit[s]) >= 5) {
      const int sh = straight_high(by_suit[s]);
      if (sh >= 0) { r[0] = sh; return pack_key(8, r, 1); }
      take_top(by_suit[s], 5, r);
      // A flush excludes quads and full houses for hands of at most 7 cards.
      return pack_key(5, r, 5);
    }
  }
  int quad = -1, trips[3], nt = 0, pairs[4], np = 0;
  for (int x = 12; x >= 0; --x) {
    if (count[x] == 4 && quad < 0) quad = x;
    else if (count[x] == 3) trips[nt++] = x;
    else if (count[x] == 2) pairs[np++] = x;
  }
  if (quad >= 0) {
    r[0] = quad;
    r[1] = top_bit(all & ~(1u << quad));
    return pack_key(7, r, 2);
  }
  if (nt >= 1 && (nt >= 2 || np >= 1)) {
    r[0] = trips[0];
    int p = -1;
    if (nt >= 2) p = trips[1];
    if (np >= 1 && pairs[0] > p) p = pairs[0];
    r[1] = p;
    return pack_key(6, r, 2);
  }
  const int sh = straight_high(all);
  if (sh >= 0) { r[0] = sh; return pack_key(4, r, 1); }
  if (nt >= 1) {
    r[0] = trips[0];
    take_top(all & ~(1u << trips[0]), 2, r + 1);
    return pack_key(3, r, 3);
  }
  if (np >= 2) {
    r[0] = pairs[0];
    r[1] = pairs[1];
    take_top(all & ~(1u << pairs[0]) & ~(1u << pairs[1]), 1, r + 2);
    return pack_key(2, r, 3);
  }
  if (np == 1) {
    r[0] = pairs[0];
    take_top(all & ~(1u << pairs[0]), 3, r + 1);
    return pack_key(1, r, 4);
  }
  take_top(all, 5, r);
  return pack_key(0, r, 5);
}

// Sorted list of the 7462 distinct five-card hand classes, weakest first.
const std::vector<uint32_t>& class_keys() {
  static const std::vector<uint32_t> keys = [] {
    std::vector<uint32_t> v;
    int rk[5], su[5];
    // Every multiset of five ranks with at most four of a kind, with and without a flush.
    for (int a = 0; a < 13; ++a)
      for (int b = a; b < 13; ++b)
        for (int c = b; c < 13; ++c)
          for (int d = c; d < 13; ++d)
            for (int e = d; e < 13; ++e) {
              if (a == e) continue;  // five of a kind
              rk[0] = a; rk[1] = b; rk[2] = c; rk[3] = d; rk[4] = e;
              // Distinct suits per card of a rank, no flush: cycle through suits 1..4
              // so no suit appears five times.
              for (int i = 0; i < 5; ++i) su[i] = 1 + (i % 4);
              v.push_back(classify(rk, su, 5));
              const bool distinct = a < b && b < c && c < d && d < e;
              if (distinct) {
                for (int i = 0; i < 5; ++i) su[i] = 1;
                v.push_back(classify(rk, su, 5));
              }
            }
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    return v;
  }();
  return keys;
}

int32_t packed_from_key(uint32_t key) {
  const auto& keys = class_keys();
  const auto it = std::lower_bound(keys.begin(), keys.end(), key);
  const int rank = (int)(it - keys.begin()) + 1;  // 1..7462
  const int cat = (int)(key >> 20) + 1;           // 1..9
  return (cat << 12) | (rank - kCategoryBase[cat]);
}

int32_t eval_id(uint64_t id) {
  int ranks[7], suits[7], n = 0;
  for (int i = 0; i < 7; ++i) {
    const int b = (int)((id >> (8 * i)) & 0xFF);
    if (!b) break;
    ranks[n] = (b >> 4) - 1;
    suits[n] = b & 0xF;
    ++n;
  }
  if (n < 5) return 0;
  return packed_from_key(classify(ranks, suits, n));
}

template <class F>
void parallel_for(size_t n, F f) {
  unsigned nt = std::thread::hardware_concurrency();
  if (nt == 0) nt = 1;
  if (nt > 64) nt = 64;
  std::atomic<size_t> next{0};
  const size_t chunk = 4096;
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t)
    th.emplace_back([&] {
      for (;;) {
        const size_t b = next.fetch_add(chunk);
        if (b >= n) break;
        const size_t e = std::min(n, b + chunk);
        for (size_t i = b; i < e; ++i) f(i);
      }
    });
  for (auto& x : th) x.join();
}

}  // namespace

int hand_class_count() { return (int)class_keys().size(); }

int32_t packed_rank_of_cards(const int* cards, int n) {
  // cards in 1..52 (rank*4 + suit + 1)
  int ranks[7], suits[7];
  for (int i = 0; i < n; ++i) {
    ranks[i] = (cards[i] - 1) >> 2;
    suits[i] = ((cards[i] - 1) & 3) + 1;
  }
  return packed_from_key(classify(ranks, suits, n));
}

int decode_packed(int32_t packed) {
  const int cat = (packed >> 12) & 0xF;
  const int ord = packed & 0xFFF;
  if (ord == 0 || cat < 1 || cat > 9) return 0;
  return kCategoryBase[cat] + ord;
}

int64_t generate_hand_table(int32_t* out, size_t n_entries, int* n_states_out) {
  // Level-by-level enumeration of canonical ids.  An id of k cards is numerically
  // smaller than any id of k+1 cards (its top non-zero byte is lower), so the
  // concatenation of the sorted levels is the ascending list of all ids.
  std::vector<uint64_t> ids;
  ids.push_back(0);
  std::vector<uint64_t> level{0};
  for (int k = 0; k < 6; ++k) {
    std::vector<uint64_t> next;
    next.reserve(level.size() * 52);
    for (uint64_t id : level)
      for (int c = 1; c <= 52; ++c) {
        const Extended e = extend_id(id, c);
        if (e.id) next.push_back(e.id);
      }
    std::sort(next.begin(), next.end());
    next.erase(std::unique(next.begin(), next.end()), next.end());
    ids.insert(ids.end(), next.begin(), next.end());
    level.swap(next);
  }
  const size_t n_states = ids.size();
  if (n_states_out) *n_states_out = (int)n_states;
  const size_t needed = n_states * 53 + 53;
  if (n_entries < needed) return -(int64_t)needed;
  std::memset(out, 0, n_entries * sizeof(int32_t));
  class_keys();  // build once before the threads read it

  auto index_of = [&](uint64_t id) -> int64_t {
    const auto it = std::lower_bound(ids.begin(), ids.end(), id);
    return (it != ids.end() && *it == id) ? (int64_t)(it - ids.begin()) : -1;
  };
  std::atomic<int> bad{0};
  parallel_for(n_states, [&](size_t s) {
    const uint64_t id = ids[s];
    int ncards = 0;
    for (int i = 0; i < 7; ++i)
      if ((id >> (8 * i)) & 0xFF) ++ncards;
    for (int c = 1; c <= 52; ++c) {
      const Extended e = extend_id(id, c);
      int32_t v;
      if (e.n < 7) {
        int64_t idx = 0;
        if (e.id) {
          idx = index_of(e.id);
          if (idx < 0) { bad.fetch_add(1); idx = 0; }
        }
        v = (int32_t)(idx * 53 + 53);
      } else {
        v = e.id ? eval_id(e.id) : 0;
      }
      out[s * 53 + 53 + c] = v;
    }
    if (ncards == 5 || ncards == 6) out[s * 53 + 53] = eval_id(id);
  });
  if (bad.load()) return -1;
  return (int64_t)needed;
}

}  // namespace mccfr

extern "C" {

int mccfr_hand_table_generate(int32_t* out, size_t n_entries) {
  if (!out) return 1;
  if (n_entries != (size_t)MCCFR_HAND_TABLE_ENTRIES) return 2;
  int n_states = 0;
  const int64_t r = mccfr::generate_hand_table(out, n_entries, &n_states);
  if (r != (int64_t)n_entries) return 3;
  return 0;
}

int mccfr_hand_table_write(const char* path) {
  if (!path) return 1;
  std::vector<int32_t> t(MCCFR_HAND_TABLE_ENTRIES);
  int rc = mccfr_hand_table_generate(t.data(), t.size());
  if (rc) return rc;
  FILE* f = std::fopen(path, "wb");
  if (!f) return 4;
  const size_t w = std::fwrite(t.data(), sizeof(int32_t), t.size(), f);
  const int cerr = std::fclose(f);
  return (w == t.size() && cerr == 0) ? 0 : 4;
}

int mccfr_hand_class_count(void) { return mccfr::hand_class_count(); }

}  // extern "C"
