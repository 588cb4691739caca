// oracle.cpp — CPU restatement of the reference's MCCFR traversal path.
//
// TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg load this library, and only as the checker.  The product
// (libmccfr.so) never links or calls it.
//
// The reference's traversal exists only as device code (poker_cuda/src/cfr_gpu.cu:
// 644-860 with cuRAND); this file restates it function by function in plain C++,
// with two documented changes that the product shares:
//   * random numbers come from a counter-based Philox4x32-10 keyed by the seed
//     and countered by (traversal, player-update, node path) instead of per-thread
//     cuRAND streams (cfr_gpu.cu:361-368, 465, 523, 963);
//   * regret/strategy-sum deltas of one player-update are summed in fixed point
//     (int64) and applied after the update, with reads during the update seeing
//     the tables as they were at its start.  The reference adds FP32 atomics while
//     other threads read (cfr_gpu.cu:621-623, 788, 1006-1007); a float-mode switch
//     here keeps that FP32 arithmetic (in traversal order) for tolerance checks.
// Every function cites the reference lines it follows.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "../include/mccfr.h"
#include "../parallel-mccfr-for-multiplayer-nlh_b200/csrc/handtable.h"

namespace orc {

// ---------------------------------------------------------------------------
// Philox4x32-10, Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy
// as 1, 2, 3" (SC'11): 10 rounds of two 32x32->64 multiplies with a Weyl key
// schedule.
// ---------------------------------------------------------------------------
struct U4 {
  uint32_t x, y, z, w;
};

static inline U4 philox(U4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
  }
  return c;
}

// (0, 1]: the top 24 bits plus one, times 2^-24.
static inline float uniform01(uint32_t w) {
  return (float)((w >> 8) + 1u) * (1.0f / 16777216.0f);
}

static const uint64_t kPathSeed = 0x243F6A8885A308D3ull;

static inline uint64_t path_step(uint64_t h, int a) {
  h = (h ^ (uint64_t)(a + 1)) * 0x9E3779B97F4A7C15ull;
  return h ^ (h >> 31);
}

static inline uint64_t mix64(uint64_t z) {
  z ^= z >> 33;
  z *= 0xFF51AFD7ED558CCDull;
  z ^= z >> 33;
  z *= 0xC4CEB9FE1A85EC53ull;
  z ^= z >> 33;
  return z;
}

// ---------------------------------------------------------------------------
// Hand ranks through the table (hand_eval.cpp:23-57, cfr_gpu.cu:87-150).
// ---------------------------------------------------------------------------
static inline int to_rm(int c) { return (c % 13) * 4 + c / 13 + 1; }  // cfr_gpu.cu:87-90

static inline uint16_t decode16(uint16_t packed) {  // cfr_gpu.cu:95-112
  const uint16_t cat = packed >> 12;
  const uint16_t ord = packed & 0x0FFFu;
  if (ord == 0) return 0;
  switch (cat) {
    case 1: return ord;
    case 2: return (uint16_t)(1277 + ord);
    case 3: return (uint16_t)(4137 + ord);
    case 4: return (uint16_t)(4995 + ord);
    case 5: return (uint16_t)(5853 + ord);
    case 6: return (uint16_t)(5863 + ord);
    case 7: return (uint16_t)(7140 + ord);
    case 8: return (uint16_t)(7296 + ord);
    case 9: return (uint16_t)(7452 + ord);
    default: return 0;
  }
}

// Chain of lookups in card order; returns the raw value after the last card.
static inline int32_t chain(const int32_t* T, const int* cards, int n) {
  int32_t p = T[53 + to_rm(cards[0])];
  for (int i = 1; i < n; ++i) p = T[p + to_rm(cards[i])];
  return p;
}

// ---------------------------------------------------------------------------
// Preflop buckets.
// ---------------------------------------------------------------------------
static float chen_score(int h0, int h1) {  // abstraction.cpp:10-38
  int r0 = h0 % 13, r1 = h1 % 13;
  const bool suited = (h0 / 13) == (h1 / 13);
  if (r0 < r1) std::swap(r0, r1);
  float base;
  if (r0 == 12) base = 10.f;
  else if (r0 == 11) base = 8.f;
  else if (r0 == 10) base = 7.f;
  else if (r0 == 9) base = 6.f;
  else base = std::max(0.5f, r0 / 2.f);
  float score;
  if (r0 == r1) {
    score = std::max(5.f, base * 2.f);
  } else {
    score = base;
    if (suited) score += 2.f;
    const int gap = r0 - r1 - 1;
    if (gap == 1) score -= 1.f;
    else if (gap == 2) score -= 2.f;
    else if (gap == 3) score -= 4.f;
    else if (gap >= 4) score -= 5.f;
    if (gap <= 1 && r0 < 12) score += 1.f;
  }
  return score;
}

static void preflop_lut(int mode, int buckets, uint8_t* lut) {
  if (mode == MCCFR_PREFLOP_CHEN64) {
    // abstraction.cpp:41-59 and the LUT upload of cfr_gpu.cu:1164-1173.
    std::vector<float> sorted;
    for (int i = 0; i < 52; ++i)
      for (int j = i + 1; j < 52; ++j) sorted.push_back(chen_score(i, j));
    std::sort(sorted.begin(), sorted.end());
    for (int h0 = 0; h0 < 52; ++h0)
      for (int h1 = 0; h1 < 52; ++h1) {
        if (h0 == h1) {
          lut[h0 * 52 + h1] = 0;
          continue;
        }
        const float s = chen_score(h0, h1);
        const auto it = std::lower_bound(sorted.begin(), sorted.end(), s);
        const float pct = (float)(it - sorted.begin()) / (float)sorted.size();
        lut[h0 * 52 + h1] = (uint8_t)std::min((int)(pct * (float)buckets), buckets - 1);
      }
  } else {
    // 169 strategically distinct starting hands on a 13x13 grid: pairs on the
    // diagonal, suited hands at (high, low), offsuit hands at (low, high).
    for (int h0 = 0; h0 < 52; ++h0)
      for (int h1 = 0; h1 < 52; ++h1) {
        const int r0 = h0 % 13, r1 = h1 % 13;
        const int hi = std::max(r0, r1), lo = std::min(r0, r1);
        const bool suited = (h0 / 13) == (h1 / 13);
        int id;
        if (hi == lo) id = hi * 13 + hi;
        else if (suited) id = hi * 13 + lo;
        else id = lo * 13 + hi;
        lut[h0 * 52 + h1] = (h0 == h1) ? 0 : (uint8_t)id;
      }
  }
}

// Rank-CDF buckets: bucket of rank r among all n-card hands (n = 5, 6, 7) by its
// mid-rank percentile, in exact integer arithmetic.
static void rank_hist(const int32_t* T, int ncards, std::vector<uint64_t>& cnt);

static void rank_cdf_lut(const int32_t* T, int ncards, int buckets, uint8_t* lut) {
  std::vector<uint64_t> cnt;
  rank_hist(T, ncards, cnt);
  uint64_t total = 0;
  for (int r = 0; r < 7463; ++r) total += cnt[r];
  uint64_t below = 0;
  for (int r = 0; r < 7463; ++r) {
    const uint64_t num = (2 * below + cnt[r]) * (uint64_t)buckets;
    uint64_t b = num / (2 * total);
    if (b > (uint64_t)(buckets - 1)) b = buckets - 1;
    lut[r] = (uint8_t)b;
    below += cnt[r];
  }
}

// Exact histogram of the best-hand rank over all C(52, ncards) card sets.
static void rank_hist(const int32_t* T, int ncards, std::vector<uint64_t>& cnt) {
  cnt.assign(7463, 0);
  // Enumerate all n-card sets in increasing card order with prefix sharing.
  std::vector<std::vector<uint64_t>> part(52, std::vector<uint64_t>(7463, 0));
  std::vector<std::thread> th;
  for (int t = 0; t < 8; ++t)
    th.emplace_back([&, t] {
      for (int a = t; a < 52; a += 8) {
        auto& c = part[a];
        const int32_t pa = T[53 + to_rm(a)];
        if (ncards == 5) {
          for (int b = a + 1; b < 52; ++b) {
            const int32_t pb = T[pa + to_rm(b)];
            for (int d = b + 1; d < 52; ++d) {
              const int32_t pd = T[pb + to_rm(d)];
              for (int e = d + 1; e < 52; ++e) {
                const int32_t pe = T[pd + to_rm(e)];
                for (int f = e + 1; f < 52; ++f) {
                  const int32_t s5 = T[pe + to_rm(f)];
                  c[decode16((uint16_t)T[s5])]++;
                }
              }
            }
          }
        } else if (ncards == 6) {
          for (int b = a + 1; b < 52; ++b) {
            const int32_t pb = T[pa + to_rm(b)];
            for (int d = b + 1; d < 52; ++d) {
              const int32_t pd = T[pb + to_rm(d)];
              for (int e = d + 1; e < 52; ++e) {
                const int32_t pe = T[pd + to_rm(e)];
                for (int f = e + 1; f < 52; ++f) {
                  const int32_t pf = T[pe + to_rm(f)];
                  for (int g = f + 1; g < 52; ++g) {
                    const int32_t s6 = T[pf + to_rm(g)];
                    c[decode16((uint16_t)T[s6])]++;
                  }
                }
              }
            }
          }
        } else {
          for (int b = a + 1; b < 52; ++b) {
            const int32_t pb = T[pa + to_rm(b)];
            for (int d = b + 1; d < 52; ++d) {
              const int32_t pd = T[pb + to_rm(d)];
              for (int e = d + 1; e < 52; ++e) {
                const int32_t pe = T[pd + to_rm(e)];
                for (int f = e + 1; f < 52; ++f) {
                  const int32_t pf = T[pe + to_rm(f)];
                  for (int g = f + 1; g < 52; ++g) {
                    const int32_t pg = T[pf + to_rm(g)];
                    for (int h = g + 1; h < 52; ++h)
                      c[decode16((uint16_t)T[pg + to_rm(h)])]++;
                  }
                }
              }
            }
          }
        }
      }
    });
  for (auto& x : th) x.join();
  for (int a = 0; a < 52; ++a)
    for (int r = 0; r < 7463; ++r) cnt[r] += part[a][r];
}

// ---------------------------------------------------------------------------
// Game configuration helpers.
// ---------------------------------------------------------------------------
struct Rules {
  mccfr_config c;
  int kind[8];
  int fallback[8];
  int n_fallback;
};

static void make_rules(const mccfr_config& c, Rules& r) {
  r.c = c;
  for (int a = 0; a < 8; ++a) r.kind[a] = (a < c.num_actions) ? c.action_kind[a] : -1;
  // Passive fallback order (cfr_gpu.cu:498-508): check, call, fold, raises in
  // slot order, all-in.
  const int order[] = {MCCFR_ACT_CHECK, MCCFR_ACT_CHECK_CALL, MCCFR_ACT_CALL, MCCFR_ACT_FOLD,
                       -2 /* raises */, MCCFR_ACT_ALL_IN};
  r.n_fallback = 0;
  for (int k : order) {
    for (int a = 0; a < c.num_actions; ++a) {
      const int kd = r.kind[a];
      const bool raise = kd == MCCFR_ACT_RAISE_MIN || kd == MCCFR_ACT_RAISE_POT;
      if ((k == -2 && raise) || kd == k) r.fallback[r.n_fallback++] = a;
    }
  }
}

static inline int min_raise_to(int cb, int lfr, int bb) {  // abstraction.cpp:144-148
  return (cb == 0) ? std::max(1, bb) : cb + std::max(lfr, bb);
}

static inline int raise_target(const Rules& R, int a, int pot, int cb, int mrt) {
  // abstraction.cpp:155-165 / cfr_gpu.cu:208-211,234-237
  if (R.kind[a] == MCCFR_ACT_RAISE_MIN) return mrt;
  const int frac = (R.c.action_num[a] * pot) / R.c.action_den[a];
  return std::max(mrt, cb + std::max(1, frac));
}

// cfr_gpu.cu:186-215 (abstraction.cpp:167-200), with an optional raise cap.
static uint8_t valid_mask(const Rules& R, int pot, int stack, int to_call, int cb, int lfr,
                          int raises) {
  if (pot <= 0) pot = 1;
  const int bb = R.c.big_blind;
  uint32_t m = 0;
  auto set_kind = [&](int k) {
    for (int a = 0; a < R.c.num_actions; ++a)
      if (R.kind[a] == k) m |= 1u << a;
  };
  if (to_call == 0) {
    set_kind(MCCFR_ACT_CHECK);
    set_kind(MCCFR_ACT_CHECK_CALL);
  } else if (to_call >= stack) {
    set_kind(MCCFR_ACT_FOLD);
    set_kind(MCCFR_ACT_ALL_IN);
    return (uint8_t)m;
  } else {
    set_kind(MCCFR_ACT_FOLD);
    set_kind(MCCFR_ACT_CALL);
    set_kind(MCCFR_ACT_CHECK_CALL);
  }
  const int head = stack - to_call;
  if (head <= 0) return (uint8_t)m;
  if (R.c.raise_cap > 0 && raises >= R.c.raise_cap) return (uint8_t)m;
  const int mrt = min_raise_to(cb, lfr, bb);
  const int maxrt = cb + head;
  if (maxrt >= mrt) {
    for (int a = 0; a < R.c.num_actions; ++a) {
      const int kd = R.kind[a];
      if (kd != MCCFR_ACT_RAISE_MIN && kd != MCCFR_ACT_RAISE_POT) continue;
      if (raise_target(R, a, pot, cb, mrt) <= maxrt) m |= 1u << a;
    }
  }
  set_kind(MCCFR_ACT_ALL_IN);
  return (uint8_t)m;
}

// cfr_gpu.cu:217-244 (abstraction.cpp:213-234)
static int chips_for(const Rules& R, int a, int pot, int stack, int to_call, int cb, int lfr) {
  if (pot <= 0) pot = 1;
  const int bb = R.c.big_blind;
  const int mrt = min_raise_to(cb, lfr, bb);
  const int maxrt = cb + std::max(0, stack - to_call);
  switch (R.kind[a]) {
    case MCCFR_ACT_FOLD:
    case MCCFR_ACT_CHECK: return 0;
    case MCCFR_ACT_CALL:
    case MCCFR_ACT_CHECK_CALL: return std::min(to_call, stack);
    case MCCFR_ACT_RAISE_MIN:
    case MCCFR_ACT_RAISE_POT: {
      const int t = std::min(raise_target(R, a, pot, cb, mrt), maxrt);
      return std::min(to_call + std::max(0, t - cb), stack);
    }
    case MCCFR_ACT_ALL_IN: return stack;
    default: return 0;
  }
}

static int passive_fallback(const Rules& R, uint8_t vm) {  // cfr_gpu.cu:498-508
  for (int i = 0; i < R.n_fallback; ++i)
    if (vm & (1u << R.fallback[i])) return R.fallback[i];
  for (int a = 0; a < R.c.num_actions; ++a)
    if (R.kind[a] == MCCFR_ACT_CHECK || R.kind[a] == MCCFR_ACT_CHECK_CALL) return a;
  return 0;
}

// ---------------------------------------------------------------------------
// State of one hand (cfr_gpu.cu:375-418).
// ---------------------------------------------------------------------------
struct Game {
  int N;
  uint32_t combo[6];
  int river_card;
  uint8_t hole[12];
  uint8_t board[5];
  uint8_t hole_b[6];
  uint8_t board_b[6][4];
  uint16_t river_rank[6];
  int dealer;
  // mutable
  int stacks[6], bets[6], inv[6];
  int to_act[6];
  int n_to_act;
  uint32_t folded, all_in;
  int pot, cb, lfr;
  uint32_t abits;
  uint64_t path;
  int street;
  int raises;
};

static inline float bf16_round(float f) {  // __float2bfloat16 (round to nearest even)
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  u &= 0xFFFF0000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

static inline uint32_t fnv_slot(int player, int hb, int bb, int street, uint32_t bits) {
  // cfr_gpu.cu:165-179
  uint32_t h = 2166136261u;
  h = (h ^ (uint8_t)player) * 16777619u;
  h = (h ^ (uint8_t)hb) * 16777619u;
  h = (h ^ (uint8_t)bb) * 16777619u;
  h = (h ^ (uint8_t)street) * 16777619u;
  h = (h ^ (uint8_t)(bits & 0xFF)) * 16777619u;
  h = (h ^ (uint8_t)((bits >> 8) & 0xFF)) * 16777619u;
  h = (h ^ (uint8_t)((bits >> 16) & 0xFF)) * 16777619u;
  h = (h ^ (uint8_t)((bits >> 24) & 0xFF)) * 16777619u;
  return h & ((1u << 26) - 1);
}

struct Row {
  float r[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  uint64_t visits = 0;
};

struct Acc {
  int64_t dr[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int64_t ds[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  uint64_t visits = 0;
  // float mode (reference FP32 order)
  float fr[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  float fs[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

struct Counters {
  int64_t V = 0, U = 0, T = 0, E = 0, X = 0;
};

struct Subgame {
  int street = 0;  // 0 = full game
  int pot = 0;
  uint8_t board[5] = {0, 0, 0, 0, 0};
  std::vector<uint32_t> cdf;  // [N][1326]
};

// Map from nonzero 64-bit keys: an open-addressing slot table (linear probing,
// load at most 1/2) over dense key and value arrays; the oracle's rows and its
// per-thread accumulators.  Iteration order is
// unspecified and never changes a result: sums are integers, rows fold
// independently and exports are sorted by key.
template <class V>
class FlatMap {
 public:
  size_t size() const { return vals_.size(); }
  // A reference stays valid until the next insertion.
  V& operator[](uint64_t key) {
    if (2 * (vals_.size() + 1) > slots_.size()) grow();
    Slot& sl = slots_[slot(key)];
    if (!sl.key) {
      sl = Slot{key, (uint32_t)vals_.size()};
      keys_.push_back(key);
      vals_.emplace_back();
    }
    return vals_[sl.idx];
  }
  const V* find(uint64_t key) const {
    if (slots_.empty()) return nullptr;
    const Slot& sl = slots_[slot(key)];
    return sl.key ? &vals_[sl.idx] : nullptr;
  }
  template <class F>
  void each(F f) const {
    for (size_t j = 0; j < vals_.size(); ++j) f(keys_[j], vals_[j]);
  }

 private:
  struct Slot {
    uint64_t key;  // 0 = empty
    uint32_t idx;  // into keys_ / vals_
  };
  std::vector<Slot> slots_;
  std::vector<uint64_t> keys_;  // insertion order
  std::vector<V> vals_;

  // The key's slot, or the empty slot where it belongs.
  size_t slot(uint64_t key) const {
    const size_t mask = slots_.size() - 1;
    size_t i = (size_t)mix64(key) & mask;
    while (slots_[i].key && slots_[i].key != key) i = (i + 1) & mask;
    return i;
  }
  // Doubles the slot table and re-inserts the keys; values do not move.
  void grow() {
    slots_.assign(slots_.empty() ? 64 : 2 * slots_.size(), Slot{0, 0});
    for (size_t j = 0; j < keys_.size(); ++j) slots_[slot(keys_[j])] = Slot{keys_[j], (uint32_t)j};
  }
};

// Rows sharded by key, so that a player-update's fold runs one shard per host
// thread.  Which shard holds a row changes nothing it computes.
constexpr int kRowShards = 64;
static inline int row_shard(uint64_t key) { return (int)((key * 0x9E3779B97F4A7C15ull) >> 58); }

struct RowTable {
  std::vector<FlatMap<Row>> shard = std::vector<FlatMap<Row>>(kRowShards);
  size_t size() const {
    size_t n = 0;
    for (const auto& m : shard) n += m.size();
    return n;
  }
  Row& operator[](uint64_t key) { return shard[row_shard(key)][key]; }
  const Row* find(uint64_t key) const { return shard[row_shard(key)].find(key); }
  std::vector<uint64_t> sorted_keys() const {
    std::vector<uint64_t> ks;
    ks.reserve(size());
    for (const auto& m : shard) m.each([&](uint64_t k, const Row&) { ks.push_back(k); });
    std::sort(ks.begin(), ks.end());
    return ks;
  }
};

struct Oracle {
  Subgame sg;
  Rules R;
  const int32_t* T = nullptr;
  uint8_t pre_lut[52 * 52];
  uint8_t cdf_lut[3][7463];
  RowTable rows;
  bool float_mode = false;
  int64_t iterations_done = 0;
  Counters total;
  // level-synchronous updates: nodes per depth, summed over traversals
  std::vector<int64_t> wave_hist;
  std::mutex wave_mu;
};

// Fixed-point fraction bits of a player-update's regret deltas: chosen so that
// batch * 64 visits * 20 * N * stack cannot overflow int64.
static int regret_frac_bits(const mccfr_config& c, long long batch) {
  auto bitlen = [](unsigned long long v) {
    int b = 0;
    while (v) { ++b; v >>= 1; }
    return b;
  };
  const unsigned long long span = 20ull * (unsigned long long)c.num_players *
                                  (unsigned long long)std::max(1, c.starting_stack);
  int rb = 61 - bitlen((unsigned long long)batch) - bitlen(span) - 6;
  if (rb > 24) rb = 24;
  if (rb < 8) rb = 8;
  return rb;
}

static inline int64_t fix_r(float x, int rb) { return (int64_t)std::llrint((double)std::ldexp(x, rb)); }
static inline int64_t fix_s(float x) { return (int64_t)std::llrint((double)(x * 4294967296.0f)); }

struct Ctx {
  const Oracle* O;
  int up;           // updating player
  uint32_t t;       // traversal index
  uint32_t launch;  // (iteration-1)*N + player
  int rb;
  FlatMap<Acc>* acc;  // this thread's accumulators, one map per row shard
  Counters* cnt;
  mccfr_trace* trace;
  float w;
  Game* root_out = nullptr;  // set: build the traversal's root game here instead of walking it
};

static inline const Row* find_row(const Oracle& O, uint64_t key) { return O.rows.find(key); }

static uint64_t info_key(const Oracle& O, const Game& g, int player) {
  int hb = g.hole_b[player];
  int bb = g.board_b[player][g.street];
  if (O.sg.street) {  // subgame: exact combo, and the river card on the river
    hb = (int)g.combo[player];
    bb = (g.street == 3 && O.sg.street == 2) ? g.river_card + 1 : 0;
  }
  if (O.R.c.key_mode == MCCFR_KEY_FNV26)
    return (uint64_t)fnv_slot(player, hb, bb, g.street, g.abits) + 1;
  uint64_t k = g.path ^ ((uint64_t)player << 56) ^ ((uint64_t)hb << 44) ^
               ((uint64_t)bb << 32) ^ ((uint64_t)g.street << 28);
  k = mix64(k);
  if (O.R.c.key_bits > 0) return (k & ((1ull << O.R.c.key_bits) - 1)) + 1;
  return k ? k : 1;
}

// BF16 current strategy of cfr_gpu.cu:318-351 and action sampling of
// cfr_gpu.cu:510-537.
static int sample_action(const Rules& R, const float* reg, uint8_t vm, float u) {
  float pos[8], sum = 0.0f;
  for (int a = 0; a < 8; ++a) {
    pos[a] = std::fmax(0.0f, reg[a]);
    sum += pos[a];
  }
  float sig[8];
  for (int a = 0; a < 8; ++a) sig[a] = bf16_round((sum > 1e-7f) ? (pos[a] / sum) : 0.0f);
  float total = 0.0f;
  for (int a = 0; a < 8; ++a)
    if (vm & (1u << a)) total += sig[a];
  if (total < 1e-7f) return passive_fallback(R, vm);
  const float r = u * total;
  float cum = 0.0f;
  int result = -1;
  for (int a = 0; a < 8; ++a) {
    const int valid = (vm >> a) & 1;
    cum += sig[a] * (float)valid;
    if (valid && result < 0 && r <= cum) result = a;
  }
  if (result < 0) result = passive_fallback(R, vm);
  return result;
}

// Regret-matched strategy of the updating player's node (cfr_gpu.cu:784-797).
static void node_strategy(const float* reg, uint8_t vm, float* strat) {
  float r[8], sum_r = 0.0f;
  for (int a = 0; a < 8; ++a) {
    r[a] = (vm & (1u << a)) ? std::fmax(0.0f, reg[a]) : 0.0f;
    sum_r += r[a];
  }
  const float uni = 1.0f / (float)__builtin_popcount(vm);
  for (int a = 0; a < 8; ++a)
    strat[a] = (sum_r > 1e-7f) ? r[a] / sum_r : ((vm & (1u << a)) ? uni : 0.0f);
}

// cfr_gpu.cu:543-573
static bool apply_action(const Rules& R, Game& g, int player, int a) {
  const int to_call = g.cb - g.bets[player];
  const int chips = chips_for(R, a, g.pot, g.stacks[player], to_call, g.cb, g.lfr);
  g.abits = ((g.abits << 3) | (uint32_t)a) & 0x3FFFFFFFu;
  g.path = path_step(g.path, a);
  if (R.kind[a] == MCCFR_ACT_FOLD) {
    g.folded |= 1u << player;
    return false;
  }
  if (R.kind[a] == MCCFR_ACT_CHECK) return false;
  g.stacks[player] -= chips;
  g.bets[player] += chips;
  g.inv[player] += chips;
  g.pot += chips;
  if (g.stacks[player] == 0) g.all_in |= 1u << player;
  if (g.bets[player] > g.cb) {
    const int prev = g.cb;
    const int rs = g.bets[player] - prev;
    if (rs >= g.lfr || prev == 0) g.lfr = rs;
    g.cb = g.bets[player];
    g.raises++;
    return true;
  }
  return false;
}

static void rebuild_queue(Game& g, int raiser) {  // cfr_gpu.cu:575-585
  g.n_to_act = 0;
  for (int i = 1; i < g.N; ++i) {
    const int p = (raiser + i) % g.N;
    if (!(g.folded & (1u << p)) && !(g.all_in & (1u << p))) g.to_act[g.n_to_act++] = p;
  }
}

static float showdown(const Game& g, int up) {  // cfr_gpu.cu:694-753
  uint16_t ranks[6] = {0, 0, 0, 0, 0, 0};
  for (int p = 0; p < g.N; ++p)
    if (!(g.folded & (1u << p))) ranks[p] = g.river_rank[p];
  int levels[6], nL = 0;
  for (int p = 0; p < g.N; ++p) {
    const int v = g.inv[p];
    if (v == 0) continue;
    bool dup = false;
    for (int j = 0; j < nL; ++j)
      if (levels[j] == v) dup = true;
    if (!dup) levels[nL++] = v;
  }
  for (int i = 0; i < nL; ++i)  // ascending, as the reference's bubble sort
    for (int j = i + 1; j < nL; ++j)
      if (levels[j] < levels[i]) std::swap(levels[i], levels[j]);
  float payoff = -(float)g.inv[up];
  int prev = 0;
  for (int li = 0; li < nL; ++li) {
    const int L = levels[li];
    int layer = 0;
    for (int q = 0; q < g.N; ++q) layer += std::max(0, std::min(g.inv[q], L) - prev);
    uint16_t best = 0;
    for (int q = 0; q < g.N; ++q)
      if (!(g.folded & (1u << q)) && g.inv[q] >= L) best = std::max(best, ranks[q]);
    if (best > 0) {
      int nwin = 0;
      for (int q = 0; q < g.N; ++q)
        if (!(g.folded & (1u << q)) && g.inv[q] >= L && ranks[q] == best) nwin++;
      if (!(g.folded & (1u << up)) && g.inv[up] >= L && ranks[up] == best)
        payoff += (float)layer / (float)nwin;
    }
    prev = L;
  }
  return payoff;
}

static void record_node(Ctx& C, uint64_t key, uint8_t vm, const float* rdelta, const float* strat,
                        bool has_r, bool has_s) {
  Acc& A = C.acc[row_shard(key)][key];
  A.visits++;
  for (int a = 0; a < 8; ++a) {
    if (!(vm & (1u << a))) continue;
    if (has_r) {
      A.dr[a] += fix_r(rdelta[a], C.rb);
      A.fr[a] += rdelta[a];
    }
    if (has_s) {
      A.ds[a] += fix_s(strat[a]);
      A.fs[a] += C.w * strat[a];
    }
  }
}

static float traverse(Ctx& C, Game& g, int depth) {  // cfr_gpu.cu:644-860
  const Oracle& O = *C.O;
  const Rules& R = O.R;
  if (depth >= R.c.max_depth) {
    C.cnt->X++;
    return 0.0f;
  }
  int active = 0, winner = -1;
  for (int i = 0; i < g.N; ++i)
    if (!(g.folded & (1u << i))) {
      active++;
      winner = i;
    }
  if (active == 1) {
    C.cnt->X++;
    return (winner == C.up) ? (float)(g.pot - g.inv[C.up]) : (float)(-g.inv[C.up]);
  }
  if (g.n_to_act == 0) {
    if (g.street < 3) {
      g.street++;
      for (int i = 0; i < g.N; ++i) g.bets[i] = 0;
      g.cb = 0;
      g.lfr = R.c.big_blind;
      g.raises = 0;
      g.n_to_act = 0;
      for (int i = 1; i <= g.N; ++i) {
        const int p = (g.dealer + i) % g.N;
        if (!(g.folded & (1u << p)) && !(g.all_in & (1u << p))) g.to_act[g.n_to_act++] = p;
      }
      if (g.n_to_act > 0) return traverse(C, g, depth + 1);
    }
    C.cnt->X++;
    return showdown(g, C.up);
  }

  const int player = g.to_act[0];
  const int to_call = g.cb - g.bets[player];
  const uint8_t vm = valid_mask(R, g.pot, g.stacks[player], to_call, g.cb, g.lfr, g.raises);
  const uint64_t key = info_key(O, g, player);
  const Row* row = find_row(O, key);
  static const float zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const float* reg = row ? row->r : zero;
  C.cnt->V++;

  const U4 draw = philox(U4{C.t, C.launch, (uint32_t)g.path, (uint32_t)(g.path >> 32) | 0x80000000u},
                         (uint32_t)R.c.seed, (uint32_t)(R.c.seed >> 32));
  const float u = uniform01(draw.x);

  auto child_of = [&](int a, Game& ch) {
    ch = g;
    ch.n_to_act--;
    for (int i = 0; i < ch.n_to_act; ++i) ch.to_act[i] = ch.to_act[i + 1];
    if (apply_action(R, ch, player, a)) rebuild_queue(ch, player);
  };

  if (player == C.up) {
    float strat[8];
    node_strategy(reg, vm, strat);
    C.cnt->U++;
    if (R.c.sampling == MCCFR_SAMPLING_REFERENCE) {
      const int s = sample_action(R, reg, vm, u);
      const float q = std::fmax(strat[s], 0.05f);
      if (C.trace) {
        if (C.trace->n_actions < 40) C.trace->actions[C.trace->n_actions] = (uint8_t)s;
        C.trace->n_actions++;
        C.trace->n_traverser_nodes++;
      }
      Game ch;
      child_of(s, ch);
      const float child = traverse(C, ch, depth + 1);
      const float ev = child;
      float rd[8];
      for (int a = 0; a < 8; ++a) {
        const float cf = (a == s) ? (child / q) : 0.0f;
        rd[a] = cf - ev;
      }
      record_node(C, key, vm, rd, strat, true, true);
      return ev;
    }
    // External sampling: every legal action.
    float v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int a = 0; a < 8; ++a) {
      if (!(vm & (1u << a))) continue;
      Game ch;
      child_of(a, ch);
      v[a] = traverse(C, ch, depth + 1);
    }
    float vh = 0.0f;
    for (int a = 0; a < 8; ++a)
      if (vm & (1u << a)) vh = vh + strat[a] * v[a];
    // Regret delta of action a: fix(v[a]) - fix(v_h), exact in fixed point.
    Acc& A = C.acc[row_shard(key)][key];
    A.visits++;
    const int64_t fvh = fix_r(vh, C.rb);
    for (int a = 0; a < 8; ++a) {
      if (!(vm & (1u << a))) continue;
      A.dr[a] += fix_r(v[a], C.rb) - fvh;
      A.fr[a] += v[a] - vh;
    }
    return vh;
  }

  const int s = sample_action(R, reg, vm, u);
  if (C.trace) {
    if (C.trace->n_actions < 40) C.trace->actions[C.trace->n_actions] = (uint8_t)s;
    C.trace->n_actions++;
  }
  if (R.c.sampling == MCCFR_SAMPLING_EXTERNAL) {
    float strat[8];
    node_strategy(reg, vm, strat);
    record_node(C, key, vm, nullptr, strat, false, true);
  }
  Game ch;
  child_of(s, ch);
  return traverse(C, ch, depth + 1);
}

static int combo_of(int a, int b) {
  const int lo = std::min(a, b), hi = std::max(a, b);
  return hi * (hi - 1) / 2 + lo;
}
static void cards_of(int idx, int& lo, int& hi) {
  int h = 1;
  while ((h + 1) * h / 2 <= idx) ++h;
  hi = h;
  lo = idx - h * (h - 1) / 2;
}
static int sample_combo(const uint32_t* cdf, uint32_t w) {
  int lo = 0, hi = 1325;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (w < cdf[mid]) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// Subgame traversal: combos from the ranges with card removal (joint redraws,
// then a player-by-player fallback), the river card uniform among unused cards.
static void run_subgame_traversal(Ctx& C) {
  const Oracle& O = *C.O;
  const Rules& R = O.R;
  const int N = std::min(6, std::max(2, R.c.num_players));
  const uint32_t k0 = (uint32_t)R.c.seed, k1 = (uint32_t)(R.c.seed >> 32);
  const int nb = O.sg.street == 2 ? 4 : 5;
  uint64_t board_mask = 0;
  for (int i = 0; i < nb; ++i) board_mask |= 1ull << O.sg.board[i];
  int combo[6] = {0, 0, 0, 0, 0, 0};
  uint64_t used = board_mask;
  bool ok = false;
  for (int a = 0; a < 16 && !ok; ++a) {
    const U4 w0 = philox(U4{C.t, C.launch, 0x100u + (uint32_t)a, 0u}, k0, k1);
    const U4 w1 = philox(U4{C.t, C.launch, 0x100u + (uint32_t)a, 1u}, k0, k1);
    const uint32_t words[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
    used = board_mask;
    ok = true;
    for (int p = 0; p < N && ok; ++p) {
      combo[p] = sample_combo(O.sg.cdf.data() + 1326 * p, words[p] >> 1);
      int lo, hi;
      cards_of(combo[p], lo, hi);
      const uint64_t m = (1ull << lo) | (1ull << hi);
      if (used & m) ok = false;
      used |= m;
    }
  }
  if (!ok) {
    const U4 w0 = philox(U4{C.t, C.launch, 0x100u, 0u}, k0, k1);
    const U4 w1 = philox(U4{C.t, C.launch, 0x100u, 1u}, k0, k1);
    const uint32_t words[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
    used = board_mask;
    for (int p = 0; p < N; ++p) {
      const uint32_t* cdf = O.sg.cdf.data() + 1326 * p;
      const int start = sample_combo(cdf, words[p] >> 1);
      int pick = -1;
      for (int k = 0; k < 1326 && pick < 0; ++k) {
        const int c = (start + k) % 1326;
        const uint32_t prev = c ? cdf[c - 1] : 0u;
        if (cdf[c] == prev) continue;
        int lo, hi;
        cards_of(c, lo, hi);
        if (!(used & ((1ull << lo) | (1ull << hi)))) pick = c;
      }
      if (pick < 0) pick = start;
      combo[p] = pick;
      int lo, hi;
      cards_of(pick, lo, hi);
      used |= (1ull << lo) | (1ull << hi);
    }
  }
  Game g;
  std::memset(&g, 0, sizeof(g));
  g.N = N;
  for (int i = 0; i < nb; ++i) g.board[i] = O.sg.board[i];
  g.river_card = -1;
  if (nb == 4) {
    const U4 w = philox(U4{C.t, C.launch, 0x200u, 0u}, k0, k1);
    const int free_cards = 52 - __builtin_popcountll(used);
    int k = (int)(((uint64_t)w.x * (uint64_t)free_cards) >> 32);
    for (int c = 0; c < 52; ++c) {
      if ((used >> c) & 1) continue;
      if (k-- == 0) {
        g.river_card = c;
        break;
      }
    }
    g.board[4] = (uint8_t)g.river_card;
  }
  for (int p = 0; p < N; ++p) {
    int lo, hi;
    cards_of(combo[p], lo, hi);
    g.hole[2 * p] = (uint8_t)lo;
    g.hole[2 * p + 1] = (uint8_t)hi;
    g.combo[p] = (uint32_t)combo[p];
    int cards[7] = {lo, hi, g.board[0], g.board[1], g.board[2], g.board[3], g.board[4]};
    g.river_rank[p] = decode16((uint16_t)chain(O.T, cards, 7));
  }
  C.cnt->E += N;
  g.dealer = N - 1;
  for (int i = 0; i < N; ++i) {
    g.stacks[i] = R.c.starting_stack;
    g.bets[i] = 0;
    g.inv[i] = O.sg.pot / N;
  }
  g.pot = O.sg.pot;
  g.cb = 0;
  g.lfr = R.c.big_blind;
  g.abits = 0;
  g.path = kPathSeed;
  g.street = O.sg.street;
  g.raises = 0;
  g.n_to_act = 0;
  for (int i = 1; i <= N; ++i) g.to_act[g.n_to_act++] = (g.dealer + i) % N;
  C.cnt->T++;
  if (C.root_out) {
    *C.root_out = g;
    return;
  }
  traverse(C, g, 0);
}

// One traversal: deal, buckets, blinds, walk (cfr_gpu.cu:916-987).
static void run_traversal(Ctx& C) {
  if (C.O->sg.street) {
    run_subgame_traversal(C);
    return;
  }
  const Oracle& O = *C.O;
  const Rules& R = O.R;
  const int N = std::min(6, std::max(2, R.c.num_players));
  const uint32_t k0 = (uint32_t)R.c.seed, k1 = (uint32_t)(R.c.seed >> 32);
  uint32_t words[24];
  for (int j = 0; j < 6; ++j) {
    const U4 o = philox(U4{C.t, C.launch, 0u, (uint32_t)j}, k0, k1);
    words[4 * j + 0] = o.x;
    words[4 * j + 1] = o.y;
    words[4 * j + 2] = o.z;
    words[4 * j + 3] = o.w;
  }
  // deal_cards, cfr_gpu.cu:460-470
  uint8_t deck[52];
  for (int i = 0; i < 52; ++i) deck[i] = (uint8_t)i;
  const int n_deal = 2 * N + 5;
  for (int i = 0; i < n_deal; ++i) {
    const uint32_t r = words[i];
    const int j = i + (int)(((uint64_t)r * (uint64_t)(52 - i)) >> 32);
    std::swap(deck[i], deck[j]);
  }
  Game g;
  std::memset(&g, 0, sizeof(g));
  g.N = N;
  for (int i = 0; i < 2 * N; ++i) g.hole[i] = deck[i];
  for (int i = 0; i < 5; ++i) g.board[i] = deck[2 * N + i];
  // buckets: cfr_gpu.cu:942-952 and 476-489
  const int32_t* T = O.T;
  for (int p = 0; p < N; ++p) {
    const int h0 = g.hole[2 * p], h1 = g.hole[2 * p + 1];
    g.hole_b[p] = O.pre_lut[h0 * 52 + h1];
    int cards[7] = {h0, h1, g.board[0], g.board[1], g.board[2], g.board[3], g.board[4]};
    const int32_t s5 = chain(T, cards, 5);
    const int32_t s6 = chain(T, cards, 6);
    const int32_t r7 = chain(T, cards, 7);
    g.river_rank[p] = decode16((uint16_t)r7);
    g.board_b[p][0] = 0;
    if (R.c.postflop_mode == MCCFR_POSTFLOP_REF_LINEAR) {
      const uint16_t v[3] = {decode16((uint16_t)s5), decode16((uint16_t)s6), decode16((uint16_t)r7)};
      for (int s = 0; s < 3; ++s)
        g.board_b[p][s + 1] =
            (uint8_t)((uint32_t)(v[s] - 1) * (uint32_t)R.c.postflop_buckets[s] / 7462u);
    } else {
      g.board_b[p][1] = O.cdf_lut[0][decode16((uint16_t)T[s5])];
      g.board_b[p][2] = O.cdf_lut[1][decode16((uint16_t)T[s6])];
      g.board_b[p][3] = O.cdf_lut[2][g.river_rank[p]];
    }
  }
  C.cnt->E += N;
  for (int i = 0; i < N; ++i) {
    g.stacks[i] = R.c.starting_stack;
    g.bets[i] = 0;
    g.inv[i] = 0;
  }
  g.folded = g.all_in = 0;
  g.pot = 0;
  g.cb = 0;
  g.lfr = R.c.big_blind;
  g.abits = 0;
  g.path = kPathSeed;
  g.street = 0;
  g.raises = 0;
  g.dealer = (int)(words[n_deal] % (uint32_t)N);
  const int sbp = (N == 2) ? g.dealer : (g.dealer + 1) % N;
  const int bbp = (N == 2) ? (g.dealer + 1) % N : (g.dealer + 2) % N;
  const int sba = std::min(R.c.small_blind, g.stacks[sbp]);
  const int bba = std::min(R.c.big_blind, g.stacks[bbp]);
  g.stacks[sbp] -= sba;
  g.bets[sbp] = sba;
  g.inv[sbp] = sba;
  g.stacks[bbp] -= bba;
  g.bets[bbp] = bba;
  g.inv[bbp] = bba;
  g.pot = sba + bba;
  g.cb = bba;
  if (g.stacks[sbp] == 0) g.all_in |= 1u << sbp;
  if (g.stacks[bbp] == 0) g.all_in |= 1u << bbp;
  g.n_to_act = 0;
  for (int i = 0; i < N; ++i) {
    const int p = (bbp + 1 + i) % N;
    if (!(g.all_in & (1u << p))) g.to_act[g.n_to_act++] = p;
  }
  if (C.trace) {
    std::memset(C.trace, 0, sizeof(*C.trace));
    std::memcpy(C.trace->hole, g.hole, 12);
    std::memcpy(C.trace->board, g.board, 5);
    C.trace->dealer = (uint8_t)g.dealer;
    for (int p = 0; p < N; ++p) {
      C.trace->hole_bucket[p] = g.hole_b[p];
      for (int s = 0; s < 4; ++s) C.trace->board_bucket[p][s] = g.board_b[p][s];
    }
  }
  C.cnt->T++;
  if (C.root_out) {
    *C.root_out = g;
    return;
  }
  const float v = traverse(C, g, 0);
  if (C.trace) C.trace->payoff = v;
}


// ---------------------------------------------------------------------------
// Level-synchronous form of the same update (a prototype of a breadth-first
// device traversal): the traversals of a chunk are expanded together, one tree
// level at a time, then their values return level by level.  Every node is one
// call of traverse() above, with the same arithmetic in the same order, so the
// rows equal the depth-first walk's bit for bit (deltas are summed in integers,
// draws are keyed by the node's path).
// ---------------------------------------------------------------------------
struct WNode {
  Game g;
  uint32_t t = 0;
  int kind = 0;   // 0 terminal, 1 one child passes its value up, 2 updating player (all
                  // legal actions), 3 updating player (one sampled action)
  int first = 0;  // first child in the next level
  int s = 0;
  uint8_t vm = 0;
  float q = 0.0f, value = 0.0f;
  uint64_t key = 0;
  float strat[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

// traverse() up to the point where it would recurse: the node gets its kind,
// its value if terminal, and its children appended to `next`.
static void wave_expand(Ctx& C, WNode& n, int depth, std::vector<WNode>& next) {
  const Oracle& O = *C.O;
  const Rules& R = O.R;
  Game& g = n.g;
  auto push = [&](const Game& ch) {
    WNode c;
    c.g = ch;
    c.t = n.t;
    next.push_back(c);
  };
  if (depth >= R.c.max_depth) {
    C.cnt->X++;
    n.value = 0.0f;
    return;
  }
  int active = 0, winner = -1;
  for (int i = 0; i < g.N; ++i)
    if (!(g.folded & (1u << i))) {
      active++;
      winner = i;
    }
  if (active == 1) {
    C.cnt->X++;
    n.value = (winner == C.up) ? (float)(g.pot - g.inv[C.up]) : (float)(-g.inv[C.up]);
    return;
  }
  if (g.n_to_act == 0) {
    if (g.street < 3) {
      g.street++;
      for (int i = 0; i < g.N; ++i) g.bets[i] = 0;
      g.cb = 0;
      g.lfr = R.c.big_blind;
      g.raises = 0;
      g.n_to_act = 0;
      for (int i = 1; i <= g.N; ++i) {
        const int p = (g.dealer + i) % g.N;
        if (!(g.folded & (1u << p)) && !(g.all_in & (1u << p))) g.to_act[g.n_to_act++] = p;
      }
      if (g.n_to_act > 0) {
        n.kind = 1;
        n.first = (int)next.size();
        push(g);
        return;
      }
    }
    C.cnt->X++;
    n.value = showdown(g, C.up);
    return;
  }
  const int player = g.to_act[0];
  const int to_call = g.cb - g.bets[player];
  const uint8_t vm = valid_mask(R, g.pot, g.stacks[player], to_call, g.cb, g.lfr, g.raises);
  const uint64_t key = info_key(O, g, player);
  const Row* row = find_row(O, key);
  static const float zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const float* reg = row ? row->r : zero;
  C.cnt->V++;
  const U4 draw = philox(U4{n.t, C.launch, (uint32_t)g.path, (uint32_t)(g.path >> 32) | 0x80000000u},
                         (uint32_t)R.c.seed, (uint32_t)(R.c.seed >> 32));
  const float u = uniform01(draw.x);
  auto child_of = [&](int a, Game& ch) {
    ch = g;
    ch.n_to_act--;
    for (int i = 0; i < ch.n_to_act; ++i) ch.to_act[i] = ch.to_act[i + 1];
    if (apply_action(R, ch, player, a)) rebuild_queue(ch, player);
  };
  n.first = (int)next.size();
  if (player == C.up) {
    node_strategy(reg, vm, n.strat);
    C.cnt->U++;
    n.key = key;
    n.vm = vm;
    if (R.c.sampling == MCCFR_SAMPLING_REFERENCE) {
      n.s = sample_action(R, reg, vm, u);
      n.q = std::fmax(n.strat[n.s], 0.05f);
      Game ch;
      child_of(n.s, ch);
      push(ch);
      n.kind = 3;
      return;
    }
    for (int a = 0; a < 8; ++a) {
      if (!(vm & (1u << a))) continue;
      Game ch;
      child_of(a, ch);
      push(ch);
    }
    n.kind = 2;
    return;
  }
  const int s = sample_action(R, reg, vm, u);
  if (R.c.sampling == MCCFR_SAMPLING_EXTERNAL) {
    float strat[8];
    node_strategy(reg, vm, strat);
    record_node(C, key, vm, nullptr, strat, false, true);
  }
  Game ch;
  child_of(s, ch);
  push(ch);
  n.kind = 1;
}

// Traversals [t0, t1) of one player-update, level by level.
static void run_wave(Ctx& C, uint32_t t0, uint32_t t1, std::vector<int64_t>& hist) {
  std::vector<std::vector<WNode>> level(1);
  for (uint32_t t = t0; t < t1; ++t) {
    WNode n;
    n.t = t;
    C.t = t;
    C.root_out = &n.g;
    run_traversal(C);  // deal, buckets and blinds: the root game
    C.root_out = nullptr;
    level[0].push_back(n);
  }
  for (size_t d = 0; !level[d].empty(); ++d) {
    std::vector<WNode> next;
    for (WNode& n : level[d]) wave_expand(C, n, (int)d, next);
    if (hist.size() <= d) hist.resize(d + 1, 0);
    hist[d] += (int64_t)level[d].size();
    level.push_back(std::move(next));
  }
  for (size_t d = level.size() - 1; d-- > 0;) {
    const std::vector<WNode>& below = level[d + 1];
    for (WNode& n : level[d]) {
      if (n.kind == 1) {
        n.value = below[n.first].value;
      } else if (n.kind == 2) {  // the same sums as traverse()'s external-sampling branch
        float v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int c = n.first;
        for (int a = 0; a < 8; ++a)
          if (n.vm & (1u << a)) v[a] = below[c++].value;
        float vh = 0.0f;
        for (int a = 0; a < 8; ++a)
          if (n.vm & (1u << a)) vh = vh + n.strat[a] * v[a];
        Acc& A = C.acc[row_shard(n.key)][n.key];
        A.visits++;
        const int64_t fvh = fix_r(vh, C.rb);
        for (int a = 0; a < 8; ++a) {
          if (!(n.vm & (1u << a))) continue;
          A.dr[a] += fix_r(v[a], C.rb) - fvh;
          A.fr[a] += v[a] - vh;
        }
        n.value = vh;
      } else if (n.kind == 3) {  // traverse()'s reference-rule branch
        const float child = below[n.first].value;
        float rd[8];
        for (int a = 0; a < 8; ++a) rd[a] = ((a == n.s) ? (child / n.q) : 0.0f) - child;
        record_node(C, n.key, n.vm, rd, n.strat, true, true);
        n.value = child;
      }
    }
  }
}

static int step(Oracle& O, long long iteration, int player, int batch, mccfr_trace* trace,
                int nthreads, bool wave = false) {
  // the level-synchronous form keeps integer sums only (float mode sums FP32 in
  // depth-first order) and writes no per-path traces
  if (wave && (O.float_mode || trace)) return MCCFR_ERR_INVALID_ARG;
  const Rules& R = O.R;
  const int N = R.c.num_players;
  const uint32_t launch = (uint32_t)((iteration - 1) * N + player);
  const int rb = regret_frac_bits(R.c, batch);
  const float w = R.c.use_linear_cfr ? (float)iteration : 1.0f;
  if (nthreads < 1) nthreads = 1;
  if (O.float_mode) nthreads = 1;
  std::vector<std::vector<FlatMap<Acc>>> accs(nthreads, std::vector<FlatMap<Acc>>(kRowShards));
  std::vector<Counters> cnts(nthreads);
  // Float mode keeps per-row FP32 sums in traversal order, so it runs on one thread.
  std::atomic<int> next{0};
  std::vector<std::vector<int64_t>> hists(nthreads);
  auto worker = [&](int tid) {
    for (;;) {
      const int b = next.fetch_add(32);
      if (b >= batch) break;
      const int e = std::min(batch, b + 32);
      if (wave) {
        Ctx C{&O, player, (uint32_t)b, launch, rb, accs[tid].data(), &cnts[tid], nullptr, w};
        run_wave(C, (uint32_t)b, (uint32_t)e, hists[tid]);
        continue;
      }
      for (int t = b; t < e; ++t) {
        Ctx C{&O, player, (uint32_t)t, launch, rb, accs[tid].data(), &cnts[tid],
              trace ? &trace[t] : nullptr, w};
        run_traversal(C);
      }
    }
  };
  if (nthreads == 1) {
    worker(0);
  } else {
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; ++i) th.emplace_back(worker, i);
    for (auto& x : th) x.join();
  }
  if (wave) {
    std::lock_guard<std::mutex> lock(O.wave_mu);
    O.wave_hist.clear();
    for (const auto& h : hists) {
      if (O.wave_hist.size() < h.size()) O.wave_hist.resize(h.size(), 0);
      for (size_t d = 0; d < h.size(); ++d) O.wave_hist[d] += h[d];
    }
  }
  for (auto& c : cnts) {
    O.total.V += c.V;
    O.total.U += c.U;
    O.total.T += c.T;
    O.total.E += c.E;
    O.total.X += c.X;
  }
  // Fold, shard by shard on the same threads: merge the threads' accumulators
  // (integer sums: order-independent), then apply them, the sparse equivalent of
  // the CFR+ clamp sweep (cfr_gpu.cu:1018-1022) over the rows this update touched.
  const double sr = std::ldexp(1.0, -rb);
  const double ss = std::ldexp(1.0, -32);
  auto apply = [&](FlatMap<Row>& rows, const FlatMap<Acc>& all) {
    all.each([&](uint64_t key, const Acc& A) {
      Row& row = rows[key];
      for (int a = 0; a < 8; ++a) {
        float r;
        float s;
        if (O.float_mode) {
          r = row.r[a] + A.fr[a];
          s = row.s[a] + A.fs[a];
        } else {
          r = row.r[a] + (float)((double)A.dr[a] * sr);
          s = row.s[a] + (float)((double)A.ds[a] * ss * (double)w);
        }
        if (R.c.use_cfr_plus) r = (r < 0.0f) ? 0.0f : r;
        row.r[a] = r;
        row.s[a] = s;
      }
      row.visits += A.visits;
    });
  };
  std::atomic<int> next_shard{0};
  auto fold = [&]() {
    for (int sh; (sh = next_shard.fetch_add(1)) < kRowShards;) {
      if (nthreads == 1) {
        apply(O.rows.shard[sh], accs[0][sh]);
        continue;
      }
      FlatMap<Acc> all;
      for (auto& per_thread : accs)
        per_thread[sh].each([&](uint64_t key, const Acc& src) {
          Acc& A = all[key];
          for (int a = 0; a < 8; ++a) {
            A.dr[a] += src.dr[a];
            A.ds[a] += src.ds[a];
            A.fr[a] += src.fr[a];
            A.fs[a] += src.fs[a];
          }
          A.visits += src.visits;
        });
      apply(O.rows.shard[sh], all);
    }
  };
  if (nthreads == 1) {
    fold();
  } else {
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; ++i) th.emplace_back(fold);
    for (auto& x : th) x.join();
  }
  return 0;
}

}  // namespace orc

using namespace orc;

extern "C" {

void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  const U4 o = philox(U4{ctr[0], ctr[1], ctr[2], ctr[3]}, key[0], key[1]);
  out[0] = o.x;
  out[1] = o.y;
  out[2] = o.z;
  out[3] = o.w;
}

float orc_uniform01(uint32_t w) { return uniform01(w); }

void* orc_create(const mccfr_config* cfg, const int32_t* hand_table) {
  Oracle* O = new Oracle();
  make_rules(*cfg, O->R);
  O->T = hand_table;
  preflop_lut(cfg->preflop_mode, cfg->preflop_buckets, O->pre_lut);
  if (cfg->postflop_mode == MCCFR_POSTFLOP_RANK_CDF)
    for (int s = 0; s < 3; ++s) rank_cdf_lut(hand_table, 5 + s, cfg->postflop_buckets[s], O->cdf_lut[s]);
  return O;
}

void orc_destroy(void* h) { delete (Oracle*)h; }

// Subgame oracle; cdf is the [N][1326] range CDF on the 2^31 scale.
void* orc_create_subgame(const mccfr_config* cfg, const int32_t* hand_table, int street, int pot,
                         const uint8_t* board, const uint32_t* cdf) {
  Oracle* O = (Oracle*)orc_create(cfg, hand_table);
  O->sg.street = street;
  O->sg.pot = pot;
  for (int i = 0; i < 5; ++i) O->sg.board[i] = board[i];
  O->sg.cdf.assign(cdf, cdf + 1326 * cfg->num_players);
  return O;
}

// Range CDF on the 2^31 scale (combos using a board card weigh 0; the last
// combo of positive weight ends at 2^31).  Returns 0 when the range is empty.
int orc_range_cdf(const float* w, const uint8_t* board, int nb, uint32_t* out) {
  uint64_t mask = 0;
  for (int i = 0; i < nb; ++i) mask |= 1ull << board[i];
  double total = 0.0;
  for (int c = 0; c < 1326; ++c) {
    int lo, hi;
    cards_of(c, lo, hi);
    const bool blocked = ((mask >> lo) & 1) || ((mask >> hi) & 1);
    total += (!blocked && w[c] > 0.0f) ? (double)w[c] : 0.0;
  }
  if (!(total > 0.0)) return 0;
  double cum = 0.0;
  int last = -1;
  for (int c = 0; c < 1326; ++c) {
    int lo, hi;
    cards_of(c, lo, hi);
    const bool blocked = ((mask >> lo) & 1) || ((mask >> hi) & 1);
    const double x = (!blocked && w[c] > 0.0f) ? (double)w[c] : 0.0;
    cum += x;
    if (x > 0.0) last = c;
    double v = std::floor(cum / total * 2147483648.0);
    if (v > 2147483648.0) v = 2147483648.0;
    out[c] = (uint32_t)v;
  }
  for (int c = last; c < 1326; ++c) out[c] = 2147483648u;
  return 1;
}

void orc_set_float_mode(void* h, int on) { ((Oracle*)h)->float_mode = on != 0; }

int orc_step(void* h, long long iteration, int player, int batch, mccfr_trace* trace, int nthreads) {
  return step(*(Oracle*)h, iteration, player, batch, trace, nthreads);
}

// The same player-update in the level-synchronous form (integer sums, no traces).
int orc_step_wave(void* h, long long iteration, int player, int batch, int nthreads) {
  return step(*(Oracle*)h, iteration, player, batch, nullptr, nthreads, true);
}

// Showdown winners of the deals of traversals 0..n-1 of update (iteration,
// player), the deals training uses (cfr_gpu.cu:460-470, 942-952): bit q of
// masks[t] is set when seat q holds the best 7-card rank (several bits: a
// split).  Every seat is live, as in a checked-down pot.
int orc_showdown_masks(void* h, long long iteration, int player, int n, uint8_t* masks) {
  if (!h || n < 0 || (n > 0 && !masks) || iteration < 1) return MCCFR_ERR_INVALID_ARG;
  Oracle& O = *(Oracle*)h;
  if (O.sg.street) return MCCFR_ERR_INVALID_ARG;
  const int N = O.R.c.num_players;
  if (player < 0 || player >= N) return MCCFR_ERR_INVALID_ARG;
  const uint32_t launch = (uint32_t)((iteration - 1) * N + player);
  FlatMap<Acc> unused[kRowShards];
  Counters cnt;
  for (int t = 0; t < n; ++t) {
    Game g;
    Ctx C{&O, player, (uint32_t)t, launch, 8, unused, &cnt, nullptr, 1.0f};
    C.root_out = &g;
    run_traversal(C);
    uint16_t best = 0;
    for (int q = 0; q < g.N; ++q) best = std::max(best, g.river_rank[q]);
    uint8_t m = 0;
    for (int q = 0; q < g.N; ++q)
      if (g.river_rank[q] == best) m |= (uint8_t)(1u << q);
    masks[t] = m;
  }
  return 0;
}

// Hands i = 0..n-1 of the showdown microbenchmark: 7 distinct cards by partial
// Fisher-Yates (the deal's multiply-shift, cfr_gpu.cu:460-470) from Philox words
// keyed by the seed at counters (i lo, stream, 0x300 | 0x301, i hi), ranked in the
// reference's order (hand_eval.cpp:134-143).
int orc_deal_eval7(const int32_t* T, uint64_t seed, uint32_t stream, size_t n, uint16_t* ranks) {
  if (!T || (n && !ranks)) return MCCFR_ERR_INVALID_ARG;
  for (size_t i = 0; i < n; ++i) {
    const uint32_t lo = (uint32_t)i, hi = (uint32_t)((uint64_t)i >> 32);
    const U4 a = philox(U4{lo, stream, 0x300u, hi}, (uint32_t)seed, (uint32_t)(seed >> 32));
    const U4 b = philox(U4{lo, stream, 0x301u, hi}, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint32_t w[7] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z};
    uint8_t deck[52];
    for (int c = 0; c < 52; ++c) deck[c] = (uint8_t)c;
    int cards[7];
    for (int k = 0; k < 7; ++k) {
      const int j = k + (int)(((uint64_t)w[k] * (uint64_t)(52 - k)) >> 32);
      std::swap(deck[k], deck[j]);
      cards[k] = deck[k];
    }
    ranks[i] = decode16((uint16_t)(chain(T, cards, 7) & 0xFFFF));
  }
  return 0;
}

// Nodes per tree depth in the last level-synchronous update, summed over its
// traversals; returns the number of depths (at most `cap` are written).
int orc_wave_hist(void* h, int64_t* out, int cap) {
  Oracle& O = *(Oracle*)h;
  std::lock_guard<std::mutex> lock(O.wave_mu);
  const int n = (int)O.wave_hist.size();
  for (int d = 0; d < n && d < cap; ++d) out[d] = O.wave_hist[d];
  return n;
}

int orc_train(void* h, long long iters, int batch, int nthreads) {
  Oracle& O = *(Oracle*)h;
  for (long long i = 0; i < iters; ++i) {
    const long long it = O.iterations_done + 1;
    for (int p = 0; p < O.R.c.num_players; ++p) step(O, it, p, batch, nullptr, nthreads);
    O.iterations_done = it;
  }
  return 0;
}

// The three workload presets as plain values (the same games mccfr_config_init
// describes), so that a CPU-only run needs no device library: the reference's
// constructor defaults and 8-slot abstraction (cfr_gpu.cuh:50-55,
// abstraction.h:9-10, 42-53), heads-up 20BB and 6-max 100BB.
// The rank table the reference's evaluator reads from a file, built on the host
// (the generator of this project's product library, compiled into the oracle so
// that CPU-only runs need no device library).
int orc_hand_table_generate(int32_t* out, size_t n) {
  if (!out || n < (size_t)MCCFR_HAND_TABLE_ENTRIES) return MCCFR_ERR_INVALID_ARG;
  int states = 0;
  return mccfr::generate_hand_table(out, n, &states) == (int64_t)MCCFR_HAND_TABLE_ENTRIES ? 0 : MCCFR_ERR_FORMAT;
}

int orc_config_init(mccfr_config* c, int preset) {
  if (!c) return MCCFR_ERR_INVALID_ARG;
  std::memset(c, 0, sizeof(*c));
  c->use_cfr_plus = 1;
  c->use_linear_cfr = 1;
  if (preset == MCCFR_PRESET_REF8) {
    c->num_players = 2;
    c->starting_stack = 1000;
    c->small_blind = 10;
    c->big_blind = 20;
    c->sampling = MCCFR_SAMPLING_REFERENCE;
    c->key_mode = MCCFR_KEY_FNV26;
    c->num_actions = 8;
    const int kinds[8] = {MCCFR_ACT_FOLD, MCCFR_ACT_CHECK, MCCFR_ACT_CALL, MCCFR_ACT_RAISE_MIN,
                          MCCFR_ACT_RAISE_POT, MCCFR_ACT_RAISE_POT, MCCFR_ACT_RAISE_POT, MCCFR_ACT_ALL_IN};
    const int nums[8] = {0, 0, 0, 0, 1, 2, 1, 0}, dens[8] = {1, 1, 1, 1, 2, 3, 1, 1};
    for (int a = 0; a < 8; ++a) {
      c->action_kind[a] = kinds[a];
      c->action_num[a] = nums[a];
      c->action_den[a] = dens[a];
    }
    c->max_depth = 20;
    c->preflop_mode = MCCFR_PREFLOP_CHEN64;
    c->preflop_buckets = 64;
    c->postflop_mode = MCCFR_POSTFLOP_REF_LINEAR;
    c->postflop_buckets[0] = c->postflop_buckets[1] = c->postflop_buckets[2] = 128;
    c->table_log2 = 26;
    c->seed = 42;
    return 0;
  }
  if (preset != MCCFR_PRESET_HU_20BB && preset != MCCFR_PRESET_6MAX_100BB) return MCCFR_ERR_INVALID_ARG;
  const bool hu = preset == MCCFR_PRESET_HU_20BB;
  c->num_players = hu ? 2 : 6;
  c->small_blind = 50;
  c->big_blind = 100;
  c->starting_stack = hu ? 2000 : 10000;
  c->sampling = MCCFR_SAMPLING_EXTERNAL;
  c->key_mode = MCCFR_KEY_ID64;
  if (hu) {
    const int kinds[4] = {MCCFR_ACT_FOLD, MCCFR_ACT_CHECK_CALL, MCCFR_ACT_RAISE_POT, MCCFR_ACT_ALL_IN};
    c->num_actions = 4;
    for (int a = 0; a < 4; ++a) {
      c->action_kind[a] = kinds[a];
      c->action_num[a] = 1;
      c->action_den[a] = 1;
    }
    c->raise_cap = 2;
    c->postflop_buckets[0] = c->postflop_buckets[1] = c->postflop_buckets[2] = 50;
    c->seed = 0;
  } else {
    const int kinds[6] = {MCCFR_ACT_FOLD, MCCFR_ACT_CHECK_CALL, MCCFR_ACT_RAISE_POT,
                          MCCFR_ACT_RAISE_POT, MCCFR_ACT_RAISE_POT, MCCFR_ACT_ALL_IN};
    const int nums[6] = {0, 0, 1, 1, 2, 0}, dens[6] = {1, 1, 2, 1, 1, 1};
    c->num_actions = 6;
    for (int a = 0; a < 6; ++a) {
      c->action_kind[a] = kinds[a];
      c->action_num[a] = nums[a];
      c->action_den[a] = dens[a];
    }
    c->raise_cap = 3;
    c->postflop_buckets[0] = c->postflop_buckets[1] = c->postflop_buckets[2] = 200;
    c->seed = 1;
  }
  c->max_depth = 255;
  c->preflop_mode = MCCFR_PREFLOP_CLASS169;
  c->preflop_buckets = 169;
  c->postflop_mode = MCCFR_POSTFLOP_RANK_CDF;
  c->key_bits = 26;
  c->table_log2 = 27;
  return 0;
}

// Replaces every row with the n given rows (regrets, strategy sums and visit
// counts per key) and sets the completed-iteration count: a table state handed
// over from another trainer, e.g. a device trainer's export, so that the next
// player-update walks exactly the trees that trainer's next update walks.
int orc_import_rows(void* h, const uint64_t* keys, const float* R, const float* S, const uint64_t* visits,
                    size_t n, long long iterations_done) {
  if (!h || (n && (!keys || !R || !S || !visits)) || iterations_done < 0) return MCCFR_ERR_INVALID_ARG;
  Oracle& O = *(Oracle*)h;
  for (size_t i = 0; i < n; ++i)
    if (keys[i] == 0) return MCCFR_ERR_INVALID_ARG;
  O.rows = RowTable();
  // rows grouped by shard, then each shard filled by one host thread
  std::vector<std::vector<uint32_t>> by_shard(kRowShards);
  for (size_t i = 0; i < n; ++i) by_shard[row_shard(keys[i])].push_back((uint32_t)i);
  std::atomic<int> next{0};
  auto fill = [&]() {
    for (int sh; (sh = next.fetch_add(1)) < kRowShards;)
      for (uint32_t i : by_shard[sh]) {
        Row& r = O.rows.shard[sh][keys[i]];
        std::memcpy(r.r, R + 8 * (size_t)i, 32);
        std::memcpy(r.s, S + 8 * (size_t)i, 32);
        r.visits = visits[i];
      }
  };
  const int nt = std::max(1, std::min(kRowShards, (int)std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(fill);
  fill();
  for (auto& x : th) x.join();
  O.iterations_done = iterations_done;
  return 0;
}

// The checksum mccfr_table_digest computes on the device, over the oracle's
// rows: sum (mod 2^64) of a 64-bit mix of each row's key, value bits and update
// count, in this fixed mixing order.
static uint64_t row_digest(uint64_t key, const float* reg, const float* ssum, uint64_t visits) {
  uint64_t h = mix64(key ^ 0x9E3779B97F4A7C15ull);
  for (int a = 0; a < 8; ++a) {
    uint32_t b;
    std::memcpy(&b, reg + a, 4);
    h = mix64(h ^ (uint64_t)b ^ ((uint64_t)a << 32));
  }
  for (int a = 0; a < 8; ++a) {
    uint32_t b;
    std::memcpy(&b, ssum + a, 4);
    h = mix64(h ^ (uint64_t)b ^ ((uint64_t)(a + 8) << 32));
  }
  return mix64(h ^ visits);
}

int orc_table_digest(void* h, uint64_t* digest, uint64_t* rows) {
  if (!h || !digest) return MCCFR_ERR_INVALID_ARG;
  Oracle& O = *(Oracle*)h;
  uint64_t sum = 0, n = 0;
  for (const auto& m : O.rows.shard)
    m.each([&](uint64_t k, const Row& r) {
      sum += row_digest(k, r.r, r.s, r.visits);
      n++;
    });
  *digest = sum;
  if (rows) *rows = n;
  return 0;
}

void orc_counters(void* h, int64_t* out) {
  Oracle& O = *(Oracle*)h;
  out[0] = O.total.T;
  out[1] = O.total.V;
  out[2] = O.total.U;
  out[3] = O.total.E;
  out[4] = O.total.X;
  out[5] = (int64_t)O.rows.size();
}

int orc_export_rows(void* h, uint64_t* keys, float* R, float* S, uint64_t* visits, size_t cap,
                    size_t* count) {
  Oracle& O = *(Oracle*)h;
  const std::vector<uint64_t> ks = O.rows.sorted_keys();
  *count = ks.size();
  if (cap < ks.size()) return MCCFR_ERR_CAPACITY;
  for (size_t i = 0; i < ks.size(); ++i) {
    const Row& r = O.rows[ks[i]];
    keys[i] = ks[i];
    if (R) std::memcpy(R + 8 * i, r.r, 32);
    if (S) std::memcpy(S + 8 * i, r.s, 32);
    if (visits) visits[i] = r.visits;
  }
  return 0;
}

// Normalised average strategy (cfr_gpu.cu:1029-1058 and 1383-1412).
int orc_get_strategy(void* h, uint32_t* keys, uint64_t* keys64, float* probs, size_t cap,
                     size_t* count) {
  Oracle& O = *(Oracle*)h;
  const std::vector<uint64_t> ks = O.rows.sorted_keys();
  std::vector<std::pair<uint64_t, std::array<float, 8>>> out;
  for (uint64_t k : ks) {
    const Row& r = O.rows[k];
    float tot = 0.0f;
    for (int a = 0; a < 8; ++a) tot += r.s[a];
    std::array<float, 8> p;
    for (int a = 0; a < 8; ++a) p[a] = (tot > 1e-7f) ? r.s[a] / tot : 0.0f;
    float t2 = 0.0f;
    for (int a = 0; a < 8; ++a) t2 += p[a];
    if (t2 < 1e-6f) continue;
    out.push_back({k, p});
  }
  *count = out.size();
  if (cap < out.size()) return MCCFR_ERR_CAPACITY;
  for (size_t i = 0; i < out.size(); ++i) {
    const uint64_t k = out[i].first;
    keys[i] = (O.R.c.key_mode == MCCFR_KEY_FNV26) ? (uint32_t)(k - 1) : (uint32_t)k;
    if (keys64) keys64[i] = k;
    std::memcpy(probs + 8 * i, out[i].second.data(), 32);
  }
  return 0;
}

// Reference-order 7-card evaluation (hand_eval.cpp:134-143).
void orc_eval7(const int32_t* T, const uint8_t* cards, uint16_t* ranks, size_t n) {
  for (size_t i = 0; i < n; ++i) {
    int c[7];
    for (int k = 0; k < 7; ++k) c[k] = cards[7 * i + k];
    ranks[i] = decode16((uint16_t)chain(T, c, 7));
  }
}

// The reference's postflop bucket for a street (cfr_gpu.cu:476-489), 0 preflop.
int orc_ref_board_bucket(const int32_t* T, int h0, int h1, const uint8_t* comm, int street,
                         int buckets) {
  if (street == 0) return 0;
  int cards[7] = {h0, h1, comm[0], comm[1], comm[2], comm[3], comm[4]};
  const uint16_t rank = decode16((uint16_t)chain(T, cards, 4 + street));
  return (uint8_t)((uint32_t)(rank - 1) * (uint32_t)buckets / 7462u);
}

void orc_preflop_lut(int mode, int buckets, uint8_t* out) { preflop_lut(mode, buckets, out); }

void orc_rank_hist(const int32_t* T, int ncards, uint64_t* out) {
  std::vector<uint64_t> c;
  rank_hist(T, ncards, c);
  std::memcpy(out, c.data(), 7463 * sizeof(uint64_t));
}

// Order-sensitive digests of the 7-card ranks of all C(52, 7) hands, grouped
// by their two lowest cards (a, b).  Within a group the hands {a < b < c < d <
// e < f < g} run in lexicographic order with i = 0, 1, ...; the digests are
// sum[a*52+b] = sum of ranks and wsum[a*52+b] = sum of (i+1) * rank.  The
// chains share prefixes as in rank_hist (cfr_gpu.cu:114-150).
void orc_rank7_digests(const int32_t* T, uint64_t* sum, uint64_t* wsum) {
  std::memset(sum, 0, 52 * 52 * sizeof(uint64_t));
  std::memset(wsum, 0, 52 * 52 * sizeof(uint64_t));
  std::vector<std::thread> th;
  for (int t = 0; t < 8; ++t)
    th.emplace_back([=] {
      for (int a = t; a < 52; a += 8) {
        const int32_t pa = T[53 + to_rm(a)];
        for (int b = a + 1; b < 52; ++b) {
          const int32_t pb = T[pa + to_rm(b)];
          uint64_t s = 0, w = 0, i = 0;
          for (int c = b + 1; c < 52; ++c) {
            const int32_t pc = T[pb + to_rm(c)];
            for (int d = c + 1; d < 52; ++d) {
              const int32_t pd = T[pc + to_rm(d)];
              for (int e = d + 1; e < 52; ++e) {
                const int32_t pe = T[pd + to_rm(e)];
                for (int f = e + 1; f < 52; ++f) {
                  const int32_t pf = T[pe + to_rm(f)];
                  for (int g = f + 1; g < 52; ++g) {
                    const uint64_t r = decode16((uint16_t)T[pf + to_rm(g)]);
                    s += r;
                    w += ++i * r;
                  }
                }
              }
            }
          }
          sum[a * 52 + b] = s;
          wsum[a * 52 + b] = w;
        }
      }
    });
  for (auto& x : th) x.join();
}

// Rank after chaining n cards (0..51) through the table in the given order; for
// n = 5 or 6 the chain ends on a state, whose card-0 entry holds the hand's rank.
int orc_chain_rank(const int32_t* T, const uint8_t* cards, int n) {
  int c[7];
  for (int i = 0; i < n; ++i) c[i] = cards[i];
  const int32_t p = chain(T, c, n);
  return decode16((uint16_t)(n == 7 ? p : T[p]));
}

void orc_rank_cdf_lut(const int32_t* T, int ncards, int buckets, uint8_t* out) {
  rank_cdf_lut(T, ncards, buckets, out);
}

int orc_valid_mask(const mccfr_config* cfg, int pot, int stack, int to_call, int cb, int lfr,
                   int raises) {
  Rules R;
  make_rules(*cfg, R);
  return valid_mask(R, pot, stack, to_call, cb, lfr, raises);
}

int orc_chips(const mccfr_config* cfg, int a, int pot, int stack, int to_call, int cb, int lfr) {
  Rules R;
  make_rules(*cfg, R);
  return chips_for(R, a, pot, stack, to_call, cb, lfr);
}

int orc_regret_frac_bits(const mccfr_config* cfg, long long batch) {
  return regret_frac_bits(*cfg, batch);
}

}  // extern "C"
