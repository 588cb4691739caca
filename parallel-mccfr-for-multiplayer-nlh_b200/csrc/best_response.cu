// best_response.cu — exact FP64 best response and exploitability of heads-up
// games, on host threads (no device code).
//
// The reference has no exploitability computation (PROPOSAL.md:99 calls it too
// expensive).  This engine evaluates an average strategy, given as info-set
// rows (key, strategy sum), in the game the traversal kernels play:
//   * the public tree is built by the kernels' own rules (valid_mask,
//     chips_for, the raise cap, the action queue and depth cut of es_step in
//     traverse_es.cuh; es_apply's bookkeeping) and keys by info_key, so a node
//     here is an info-set row there;
//   * the walk is vector-valued: at each public state it carries both players'
//     reach for all 1326 hole combos and returns both players' best-response
//     values per combo (counterfactual: weighted by the other's reach).  A
//     best responder maximises per (public state, own combo): it plays the
//     real game, seeing its cards and the board, against the other player's
//     abstract average strategy;
//   * a fold costs O(1326) through per-card reach sums; a showdown O(1326) by
//     a sweep over the combos in rank order with per-card running sums;
//   * chance: hole combos (uniform, or the subgame's range weights), the
//     dealer (uniform, full game), then flop, turn and river cards.  In the
//     full game flops are enumerated up to suit permutation (1,755 classes):
//     with rank-CDF buckets and 169-class or Chen preflop buckets every key is
//     suit-invariant, so a flop's values are a permutation of its class
//     representative's.  Flop classes (full game) are spread over threads.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mccfr.h"
#include "best_response.h"
#include "game.cuh"

namespace mccfr {
void build_cdf_lut(const unsigned long long* counts, int buckets, uint8_t* lut);
void build_preflop_lut(int mode, int buckets, uint8_t* lut);

// Exact histogram of the ranks of all C(52, n) hands (n = 5, 6, 7), in the
// enumeration of the device's k_rank_hist (3-card prefix, then the rest in
// increasing card order).
void host_rank_hist(const int32_t* T, int ncards, unsigned long long* hist, int threads) {
  std::vector<std::vector<unsigned long long>> part(std::max(1, threads), std::vector<unsigned long long>(7463, 0));
  std::atomic<int> next{0};
  auto work = [&](int tid) {
    auto& h = part[tid];
    for (;;) {
      const int a = next.fetch_add(1);
      if (a >= 52) break;
      const int32_t pa = T[53 + to_rm(a)];
      for (int b = a + 1; b < 52; ++b) {
        const int32_t pb = T[pa + to_rm(b)];
        for (int c = b + 1; c < 52; ++c) {
          const int32_t pc = T[pb + to_rm(c)];
          for (int d = c + 1; d < 52; ++d) {
            const int32_t pd = T[pc + to_rm(d)];
            for (int e = d + 1; e < 52; ++e) {
              const int32_t pe = T[pd + to_rm(e)];
              if (ncards == 5) {
                h[decode16((uint32_t)T[pe] & 0xFFFF)]++;
                continue;
              }
              for (int f = e + 1; f < 52; ++f) {
                const int32_t pf = T[pe + to_rm(f)];
                if (ncards == 6) {
                  h[decode16((uint32_t)T[pf] & 0xFFFF)]++;
                  continue;
                }
                for (int g = f + 1; g < 52; ++g) h[decode16((uint32_t)T[pf + to_rm(g)] & 0xFFFF)]++;
              }
            }
          }
        }
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < (int)part.size(); ++t) th.emplace_back(work, t);
  work(0);
  for (auto& t : th) t.join();
  for (int r = 0; r < 7463; ++r) {
    hist[r] = 0;
    for (auto& p : part) hist[r] += p[r];
  }
}

namespace {

constexpr int kC = 1326;

// Hole combos: index hi*(hi-1)/2 + lo for cards lo < hi (card = suit*13 + rank).
struct Combos {
  uint8_t lo[kC], hi[kC];
  uint64_t mask[kC];
  int16_t holding[52][51];  // the 51 combos holding each card
  int16_t index[52][52];
  Combos() {
    int n[52] = {0};
    for (int h = 1; h < 52; ++h)
      for (int l = 0; l < h; ++l) {
        const int c = h * (h - 1) / 2 + l;
        lo[c] = (uint8_t)l;
        hi[c] = (uint8_t)h;
        mask[c] = (1ull << l) | (1ull << h);
        holding[l][n[l]++] = (int16_t)c;
        holding[h][n[h]++] = (int16_t)c;
        index[l][h] = index[h][l] = (int16_t)c;
      }
    for (int c = 0; c < 52; ++c) index[c][c] = -1;
  }
};
const Combos& CB() {
  static const Combos t;
  return t;
}

enum : uint8_t { kDecision, kFold, kShowdown, kCut, kDeal };

struct Node {
  uint8_t type = kCut, player = 0, street = 0, nact = 0;
  uint8_t act[kSlots] = {};
  int child[kSlots] = {};
  int next = -1;      // kDeal: the node after the card(s)
  int inv[2] = {0, 0};
  int pot = 0;
  uint32_t abits = 0;
  uint64_t path = 0;
  long long strat = -1;  // full game: offset of the node's dense strategy table
};

// Betting state of the traversal walk (EsState, traverse_es.cuh), two players.
struct St {
  int stack[2], bet[2], inv[2];
  int pot, cb, lfr;
  uint32_t q;
  int nq;
  uint32_t abits;
  uint64_t path;
  uint32_t folded, allin;
  int street, raises, depth;
};

// es_apply (traverse_es.cuh) on the host.
void apply_action(const GameParams& G, St& s, int player, int a) {
  s.q >>= 4;
  s.nq--;
  const int pstack = s.stack[player], pbet = s.bet[player];
  const int to_call = s.cb - pbet;
  const int chips = chips_for(G, a, s.pot, pstack, to_call, s.cb, s.lfr);
  s.abits = ((s.abits << 3) | (uint32_t)a) & 0x3FFFFFFFu;
  s.path = path_step(s.path, a);
  const int k = G.kind[a];
  if (k == 0) {
    s.folded |= 1u << player;
    return;
  }
  if (k == 1) return;
  const int nstack = pstack - chips, nbet = pbet + chips;
  s.stack[player] = nstack;
  s.bet[player] = nbet;
  s.inv[player] += chips;
  s.pot += chips;
  if (nstack == 0) s.allin |= 1u << player;
  if (nbet > s.cb) {
    const int prev = s.cb;
    const int rs = nbet - prev;
    if (rs >= s.lfr || prev == 0) s.lfr = rs;
    s.cb = nbet;
    s.raises++;
    s.q = 0;
    s.nq = 0;
    const int p = (player + 1) % 2;
    if (!((s.folded >> p) & 1) && !((s.allin >> p) & 1)) s.q |= (uint32_t)p << (4 * s.nq++);
  }
}

// Public tree from state s, in es_step's order of checks: depth cut, one
// player left, end of the street's queue (deal or showdown), decision.
int build_tree(const GameParams& G, std::vector<Node>& T, St s, int dealer) {
  auto push = [&](const Node& n) {
    T.push_back(n);
    return (int)T.size() - 1;
  };
  if (s.depth >= G.max_depth) {
    Node n;
    n.type = kCut;
    n.street = (uint8_t)s.street;
    return push(n);
  }
  const uint32_t live = 3u & ~s.folded;
  if (__builtin_popcount(live) == 1) {
    Node n;
    n.type = kFold;
    n.player = (uint8_t)__builtin_ctz(live);
    n.street = (uint8_t)s.street;
    n.inv[0] = s.inv[0];
    n.inv[1] = s.inv[1];
    n.pot = s.pot;
    return push(n);
  }
  if (s.nq == 0) {
    Node sd;
    sd.type = kShowdown;
    sd.inv[0] = s.inv[0];
    sd.inv[1] = s.inv[1];
    sd.pot = s.pot;
    if (s.street < 3) {
      Node d;
      d.type = kDeal;
      d.street = (uint8_t)(s.street + 1);
      const int id = push(d);
      St t = s;
      t.street++;
      t.bet[0] = t.bet[1] = 0;
      t.cb = 0;
      t.lfr = G.bb;
      t.raises = 0;
      t.q = 0;
      t.nq = 0;
      for (int i = 1; i <= 2; ++i) {
        const int p = (dealer + i) % 2;
        if (!((t.folded >> p) & 1) && !((t.allin >> p) & 1)) t.q |= (uint32_t)p << (4 * t.nq++);
      }
      int nx;
      if (t.nq > 0) {
        t.depth++;
        nx = build_tree(G, T, t, dealer);
      } else {
        sd.street = (uint8_t)t.street;  // everyone all-in: showdown after the runout
        nx = push(sd);
      }
      T[id].next = nx;
      return id;
    }
    sd.street = 3;
    return push(sd);
  }
  const int p = (int)(s.q & 0xF);
  const int to_call = s.cb - s.bet[p];
  const uint32_t vm = valid_mask(G, s.pot, s.stack[p], to_call, s.cb, s.lfr, s.raises);
  Node n;
  n.type = kDecision;
  n.player = (uint8_t)p;
  n.street = (uint8_t)s.street;
  n.abits = s.abits;
  n.path = s.path;
  for (int a = 0; a < kSlots; ++a)
    if ((vm >> a) & 1) n.act[n.nact++] = (uint8_t)a;
  const int id = push(n);
  for (int i = 0; i < n.nact; ++i) {
    St c = s;
    apply_action(G, c, p, n.act[i]);
    c.depth++;
    const int ch = build_tree(G, T, c, dealer);
    T[id].child[i] = ch;
  }
  return id;
}

St full_root(const GameParams& G, int dealer) {
  St s{};
  const int sbp = dealer, bbp = 1 - dealer;
  const int sba = std::min(G.sb, G.stack), bba = std::min(G.bb, G.stack);
  s.stack[0] = s.stack[1] = G.stack;
  s.stack[sbp] -= sba;
  s.bet[sbp] = s.inv[sbp] = sba;
  s.stack[bbp] -= bba;
  s.bet[bbp] = s.inv[bbp] = bba;
  s.pot = sba + bba;
  s.cb = bba;
  s.lfr = G.bb;
  if (G.stack - sba == 0) s.allin |= 1u << sbp;
  if (G.stack - bba == 0) s.allin |= 1u << bbp;
  s.path = kPathSeed;
  for (int i = 0; i < 2; ++i) {
    const int p = (bbp + 1 + i) % 2;
    if (!((s.allin >> p) & 1)) s.q |= (uint32_t)p << (4 * s.nq++);
  }
  return s;
}

St sub_root(const GameParams& G) {
  St s{};
  s.stack[0] = s.stack[1] = G.stack;
  s.inv[0] = s.inv[1] = G.sub_pot / 2;
  s.pot = G.sub_pot;
  s.lfr = G.bb;
  s.street = G.sub_street;
  s.path = kPathSeed;
  const int dealer = 1;  // deal_subgame: the dealer is the last seat
  for (int i = 1; i <= 2; ++i) s.q |= (uint32_t)((dealer + i) % 2) << (4 * s.nq++);
  return s;
}

// key -> row of strategy sums (open addressing).
struct RowMap {
  std::vector<uint64_t> key;
  std::vector<int64_t> row;
  uint64_t mask = 0;
  const float* ssum = nullptr;
  void build(const uint64_t* k, const float* s, size_t n) {
    size_t cap = 1024;
    while (cap < 2 * n) cap <<= 1;
    key.assign(cap, 0);
    row.assign(cap, -1);
    mask = cap - 1;
    ssum = s;
    for (size_t i = 0; i < n; ++i) {
      if (!k[i]) continue;
      uint64_t h = mix64(k[i]) & mask;
      while (row[h] >= 0 && key[h] != k[i]) h = (h + 1) & mask;
      key[h] = k[i];
      row[h] = (int64_t)i;
    }
  }
  const float* find(uint64_t k) const {
    uint64_t h = mix64(k) & mask;
    while (row[h] >= 0) {
      if (key[h] == k) return ssum + 8 * row[h];
      h = (h + 1) & mask;
    }
    return nullptr;
  }
};

// Average strategy of decision node n at `key`: the legal slots' strategy sums
// normalised, uniform when the row is missing or its legal sum is not positive.
void node_probs(const RowMap& M, const Node& n, uint64_t key, double* p) {
  const float* s = M.find(key);
  double sum = 0.0;
  if (s)
    for (int i = 0; i < n.nact; ++i) sum += std::max(0.0, (double)s[n.act[i]]);
  if (s && sum > 0.0) {
    for (int i = 0; i < n.nact; ++i) p[i] = std::max(0.0, (double)s[n.act[i]]) / sum;
  } else {
    for (int i = 0; i < n.nact; ++i) p[i] = 1.0 / n.nact;
  }
}

// ---- suit permutations ------------------------------------------------------
struct SuitPerms {
  int perm[24][4];
  int inv_combo[24][kC];  // combo index of sigma^-1 applied to the combo
  SuitPerms() {
    int p[4] = {0, 1, 2, 3}, n = 0;
    do {
      for (int i = 0; i < 4; ++i) perm[n][i] = p[i];
      ++n;
    } while (std::next_permutation(p, p + 4));
    const Combos& K = CB();
    for (int s = 0; s < 24; ++s) {
      int inv[4];
      for (int i = 0; i < 4; ++i) inv[perm[s][i]] = i;
      for (int c = 0; c < kC; ++c) {
        const int a = inv[K.lo[c] / 13] * 13 + K.lo[c] % 13;
        const int b = inv[K.hi[c] / 13] * 13 + K.hi[c] % 13;
        inv_combo[s][c] = K.index[a][b];
      }
    }
  }
  int apply(int s, int card) const { return perm[s][card / 13] * 13 + card % 13; }
};

// Board state of a walk before the river: known cards and, in the full game,
// the dense-table row of each combo for this street.
struct Ctx {
  int street = 0;  // 0 preflop, 1 flop, 2 turn
  int ncards = 0;
  uint8_t cards[5] = {};
  uint64_t mask = 0;
  const uint16_t* bidx = nullptr;
};

// A complete board: the unblocked combos in ascending rank order.  River
// walks use vectors indexed by position in this order.
struct RiverBoard {
  int n = 0;
  int river = -1;                  // the river card (subgame keys)
  const uint16_t* combo = nullptr;  // [n] combo index
  const uint16_t* bidx = nullptr;   // [n] full game: dense-table row
  const uint8_t* lo = nullptr;      // [n] cards of the combo
  const uint8_t* hi = nullptr;
  const uint16_t* gend = nullptr;   // [n] end of position j's equal-rank group
  const uint16_t* bycard = nullptr; // [52][46] positions of the combos holding each card
  uint64_t mask = 0;                // board cards
};

struct Engine;

struct FlopEntry {
  int node;     // the preflop deal node
  int dealer;
  std::vector<double> r[2];
};

struct Worker {
  const Engine& E;
  std::vector<double> pool;
  size_t top = 0;
  bool overflow = false;
  double prof[2] = {0.0, 0.0};
  long long boards = 0;
  // full game: preflop passes (1 collects flop entries, 2 combines their values)
  int preflop_pass = 0;
  std::vector<FlopEntry>* entries = nullptr;
  std::vector<int>* entry_of = nullptr;          // node -> entry
  std::vector<std::vector<double>>* entry_val = nullptr;  // [entry*2 + player][combo]
  // full game: suit permutations fixing the current flop (identity first);
  // turn cards related by one of them give permuted values
  const SuitPerms* perms = nullptr;
  std::vector<int> stab;
  // board caches of the current flop (full game) or the subgame's board
  uint16_t bidx_flop[kC];
  std::vector<uint16_t> bidx_turn;  // [52][kC]
  std::vector<uint8_t> turn_ready;
  // complete boards, slot = turn card * 52 + river card: combo, bidx, gend
  // (uint16 x n) and lo, hi (uint8 x n), n <= 1081
  std::vector<uint16_t> rb_u16;  // [slot][3][1081]
  std::vector<uint8_t> rb_u8;    // [slot][2][1081]
  std::vector<int> rb_n;         // -1 = not built
  std::vector<uint16_t> rb_card; // [slot][52][46]
  std::vector<uint16_t> rank_count = std::vector<uint16_t>(7464);
  explicit Worker(const Engine& e);
  double* alloc(size_t n) {  // 16-byte aligned (even offsets in an aligned pool)
    n = (n + 1) & ~size_t(1);
    if (top + n > pool.size()) {
      overflow = true;
      top = 0;
    }
    double* p = pool.data() + top;
    top += n;
    return p;
  }
  void reset_flop_caches();
  void flop_ctx(const uint8_t* flop, Ctx& X);
  void turn_ctx(const Ctx& X, int card, Ctx& Y);
  RiverBoard river_board(const uint8_t* cards5, int slot);
  void walk(int ni, const Ctx& X, const double* r0, const double* r1, double* v0, double* v1, double wch);
  void decision(const Node& n, const Ctx& X, const double* r0, const double* r1, double* v0, double* v1,
                double wch);
  void fold(const Node& n, const Ctx& X, const double* r0, const double* r1, double* v0, double* v1, double wch);
  void deal(int next, const Ctx& X, const double* r0, const double* r1, double* v0, double* v1, double wch);
  // river walks on compact vectors
  void rwalk(int ni, const RiverBoard& R, const double* r0, const double* r1, double* v0, double* v1, double wch);
  void rdecision(const Node& n, const RiverBoard& R, const double* r0, const double* r1, double* v0, double* v1,
                 double wch);
  template <class Sink>
  void rfold(const Node& n, const RiverBoard& R, const double* r0, const double* r1, Sink&& sink, double wch);
  template <class Sink>
  void rshowdown(const Node& n, const RiverBoard& R, const double* r0, const double* r1, Sink&& sink, double wch);
};

struct Engine {
  GameParams G;
  bool full = false;
  const int32_t* T = nullptr;
  int H = 1;          // preflop classes
  int B[4] = {1, 1, 1, 1};  // buckets per street
  uint8_t pre[52 * 52];
  uint8_t cdf[3][7463];
  uint16_t hb[kC];
  std::vector<Node> nodes;
  int root[2] = {-1, -1};
  RowMap rows;
  std::vector<double> dense;
  double w[2][kC];
  double Z = 0.0;
  int sub_street = 0;
  uint8_t board[5] = {};
  uint64_t board_mask = 0;

  uint64_t key_of(const Node& n, uint32_t hbv, uint32_t bkt) const {
    return info_key(G, n.player, hbv, bkt, n.street, n.abits, n.path);
  }
};

constexpr int kRiverMax = 1081;  // C(47, 2)

Worker::Worker(const Engine& e) : E(e) {
  pool.assign(size_t(1) << 21, 0.0);
  if (E.full) {
    bidx_turn.assign(52ull * kC, 0);
    turn_ready.assign(52, 0);
  }
  const size_t slots = E.full ? 52 * 52 : 52;
  rb_u16.assign(slots * 3 * kRiverMax, 0);
  rb_u8.assign(slots * 2 * kRiverMax, 0);
  rb_n.assign(slots, -1);
  rb_card.assign(slots * 52 * 46, 0);
}

void Worker::reset_flop_caches() {
  std::fill(rb_n.begin(), rb_n.end(), -1);
  if (E.full) std::fill(turn_ready.begin(), turn_ready.end(), 0);
}

int32_t chain(const int32_t* T, const uint8_t* cards, int n) {
  int32_t p = 53;
  for (int i = 0; i < n; ++i) p = T[p + to_rm(cards[i])];
  return p;
}

void Worker::flop_ctx(const uint8_t* flop, Ctx& X) {
  const Combos& K = CB();
  X = Ctx();
  X.street = 1;
  X.ncards = 3;
  for (int i = 0; i < 3; ++i) {
    X.cards[i] = flop[i];
    X.mask |= 1ull << flop[i];
  }
  const int32_t s3 = chain(E.T, flop, 3);
  for (int c = 0; c < kC; ++c) {
    bidx_flop[c] = 0;
    if (K.mask[c] & X.mask) continue;
    const int32_t s5 = E.T[E.T[s3 + to_rm(K.lo[c])] + to_rm(K.hi[c])];
    const uint32_t r5 = decode16((uint32_t)E.T[s5] & 0xFFFF);
    bidx_flop[c] = (uint16_t)(E.hb[c] * E.B[1] + E.cdf[0][r5]);
  }
  X.bidx = bidx_flop;
}

// Context after dealing the turn `card` to flop context X (full game).
void Worker::turn_ctx(const Ctx& X, int card, Ctx& Y) {
  const Combos& K = CB();
  Y = X;
  Y.street = 2;
  Y.cards[Y.ncards++] = (uint8_t)card;
  Y.mask |= 1ull << card;
  uint16_t* b = bidx_turn.data() + (size_t)card * kC;
  if (!turn_ready[card]) {
    const int32_t s4 = chain(E.T, Y.cards, 4);
    for (int c = 0; c < kC; ++c) {
      b[c] = 0;
      if (K.mask[c] & Y.mask) continue;
      const int32_t s6 = E.T[E.T[s4 + to_rm(K.lo[c])] + to_rm(K.hi[c])];
      const uint32_t r6 = decode16((uint32_t)E.T[s6] & 0xFFFF);
      b[c] = (uint16_t)(E.hb[c] * E.B[2] + E.cdf[1][r6]);
    }
    turn_ready[card] = 1;
  }
  Y.bidx = b;
}

// The complete board `cards5` (cached in `slot`): unblocked combos sorted by
// 7-card rank, with their cards, river buckets and rank groups.
RiverBoard Worker::river_board(const uint8_t* cards5, int slot) {
  const Combos& K = CB();
  uint16_t* combo = rb_u16.data() + (size_t)slot * 3 * kRiverMax;
  uint16_t* bidx = combo + kRiverMax;
  uint16_t* gend = bidx + kRiverMax;
  uint8_t* lo = rb_u8.data() + (size_t)slot * 2 * kRiverMax;
  uint8_t* hi = lo + kRiverMax;
  if (rb_n[slot] < 0) {
    uint64_t mask = 0;
    for (int i = 0; i < 5; ++i) mask |= 1ull << cards5[i];
    const int32_t s5 = chain(E.T, cards5, 5);
    // counting sort by rank, combo index ascending within a rank
    uint16_t rk[kC];
    std::vector<uint16_t>& cnt = rank_count;
    std::fill(cnt.begin(), cnt.end(), 0);
    int n = 0;
    for (int c = 0; c < kC; ++c) {
      if (K.mask[c] & mask) continue;
      rk[c] = (uint16_t)decode16((uint32_t)E.T[E.T[s5 + to_rm(K.lo[c])] + to_rm(K.hi[c])] & 0xFFFF);
      cnt[rk[c] + 1]++;
      ++n;
    }
    for (int r = 1; r < 7464; ++r) cnt[r] += cnt[r - 1];
    for (int c = 0; c < kC; ++c)
      if (!(K.mask[c] & mask)) combo[cnt[rk[c]]++] = (uint16_t)c;
    for (int j = 0; j < n; ++j) {
      const int c = combo[j];
      lo[j] = K.lo[c];
      hi[j] = K.hi[c];
      bidx[j] = E.full ? (uint16_t)(E.hb[c] * E.B[3] + E.cdf[2][rk[c]]) : 0;
    }
    for (int j = n - 1; j >= 0; --j)
      gend[j] = (j + 1 < n && rk[combo[j + 1]] == rk[combo[j]]) ? gend[j + 1] : (uint16_t)(j + 1);
    uint16_t* bc = rb_card.data() + (size_t)slot * 52 * 46;
    int fill[52] = {0};
    for (int j = 0; j < n; ++j) {
      bc[lo[j] * 46 + fill[lo[j]]++] = (uint16_t)j;
      bc[hi[j] * 46 + fill[hi[j]]++] = (uint16_t)j;
    }
    rb_n[slot] = n;
    boards++;
  }
  RiverBoard R;
  R.n = rb_n[slot];
  R.combo = combo;
  R.bidx = bidx;
  R.lo = lo;
  R.hi = hi;
  R.gend = gend;
  R.bycard = rb_card.data() + (size_t)slot * 52 * 46;
  for (int i = 0; i < 5; ++i) R.mask |= 1ull << cards5[i];
  return R;
}

void Worker::walk(int ni, const Ctx& X, const double* r0, const double* r1, double* v0, double* v1, double wch) {
  const Node& n = E.nodes[ni];
  switch (n.type) {
    case kCut:
      std::fill(v0, v0 + kC, 0.0);
      std::fill(v1, v1 + kC, 0.0);
      return;
    case kFold:
      fold(n, X, r0, r1, v0, v1, wch);
      return;
    case kShowdown:  // all-in before the river: run the board out
      deal(ni, X, r0, r1, v0, v1, wch);
      return;
    case kDeal:
      if (X.street == 0) {  // full game, preflop to flop: handled by the flop-class loop
        const int e = (*entry_of)[ni];
        if (preflop_pass == 1) {
          FlopEntry& F = (*entries)[e];
          F.r[0].assign(r0, r0 + kC);
          F.r[1].assign(r1, r1 + kC);
          std::fill(v0, v0 + kC, 0.0);
          std::fill(v1, v1 + kC, 0.0);
        } else {
          std::copy((*entry_val)[2 * e].begin(), (*entry_val)[2 * e].end(), v0);
          std::copy((*entry_val)[2 * e + 1].begin(), (*entry_val)[2 * e + 1].end(), v1);
        }
        return;
      }
      deal(n.next, X, r0, r1, v0, v1, wch);
      return;
    default:
      decision(n, X, r0, r1, v0, v1, wch);
  }
}

// Strategy rows of a decision node: S[j * na + i] for the combos of a walk.
// Full game: rows of the node's dense table, picked by bucket index; subgame:
// looked up by the exact combo (and the river card on the river).
static void subgame_strats(const Engine& E, const Node& n, const uint16_t* combos, int count, int river,
                           double* buf) {
  const uint32_t bkt = (n.street == 3 && E.sub_street == 2) ? (uint32_t)(river + 1) : 0u;
  for (int j = 0; j < count; ++j) {
    const int c = combos ? combos[j] : j;
    node_probs(E.rows, n, E.key_of(n, (uint32_t)c, bkt), buf + (size_t)j * n.nact);
  }
}

void Worker::decision(const Node& n, const Ctx& X, const double* r0, const double* r1, double* v0, double* v1,
                      double wch) {
  const int p = n.player, na = n.nact;
  const size_t mark = top;
  const double* S;
  const uint16_t* rowidx = nullptr;
  if (E.full) {
    S = E.dense.data() + n.strat;
    rowidx = X.bidx;
  } else {
    double* buf = alloc((size_t)kC * na);
    subgame_strats(E, n, nullptr, kC, -1, buf);
    S = buf;
  }
  const double* rp = p ? r1 : r0;
  double* rc = alloc(kC);
  double* c0 = alloc(kC);
  double* c1 = alloc(kC);
  double* vp = p ? v1 : v0;
  double* vo = p ? v0 : v1;
  for (int c = 0; c < kC; ++c) {
    vp[c] = -std::numeric_limits<double>::infinity();
    vo[c] = 0.0;
  }
  for (int i = 0; i < na; ++i) {
    if (rowidx) {
      for (int c = 0; c < kC; ++c) rc[c] = rp[c] * S[(size_t)rowidx[c] * na + i];
    } else {
      for (int c = 0; c < kC; ++c) rc[c] = rp[c] * S[(size_t)c * na + i];
    }
    walk(n.child[i], X, p ? r0 : rc, p ? rc : r1, c0, c1, wch);
    const double* cp = p ? c1 : c0;
    const double* co = p ? c0 : c1;
    for (int c = 0; c < kC; ++c) {
      vp[c] = std::max(vp[c], cp[c]);
      vo[c] += co[c];
    }
  }
  top = mark;
}

// Fold before the river: the winner takes pot - inv; the other loses inv.
void Worker::fold(const Node& n, const Ctx& X, const double* r0, const double* r1, double* v0, double* v1,
                  double wch) {
  const Combos& K = CB();
  for (int i = 0; i < 2; ++i) {
    const double pay = (i == n.player) ? (double)(n.pot - n.inv[i]) : -(double)n.inv[i];
    const double* ro = i ? r0 : r1;
    const double* ri = i ? r1 : r0;
    double* vi = i ? v1 : v0;
    double S = 0.0, Sc[52] = {0.0};
    for (int c = 0; c < kC; ++c) {
      const double x = ro[c];
      if (x != 0.0) {
        S += x;
        Sc[K.lo[c]] += x;
        Sc[K.hi[c]] += x;
      }
    }
    double pv = 0.0;
    for (int c = 0; c < kC; ++c) {
      if (K.mask[c] & X.mask) {
        vi[c] = 0.0;
        continue;
      }
      vi[c] = pay * (S - Sc[K.lo[c]] - Sc[K.hi[c]] + ro[c]);
      pv += ri[c] * vi[c];
    }
    prof[i] += wch * pv;
  }
}

// The next card: every card off the board; given both hands, each of the
// 48 - ncards cards that fits is equally likely.  Turn cards keep full
// vectors (the combos holding the card get reach 0); river cards switch to the
// complete board's compact vectors.
void Worker::deal(int next, const Ctx& X, const double* r0, const double* r1, double* v0, double* v1, double wch) {
  const Combos& K = CB();
  const size_t mark = top;
  const double pw = 1.0 / (double)(48 - X.ncards);
  std::fill(v0, v0 + kC, 0.0);
  std::fill(v1, v1 + kC, 0.0);
  if (X.street == 1) {
    double* f0 = alloc(kC);
    double* f1 = alloc(kC);
    double* c0 = alloc(kC);
    double* c1 = alloc(kC);
    for (int card = 0; card < 52; ++card) {
      if ((X.mask >> card) & 1) continue;
      // With a suit permutation s fixing the flop, the reaches here are
      // s-invariant, so the values after turn s(card) are those after `card`
      // with combos permuted: walk the smallest card of each orbit only.
      int images[24], orbit = 0;
      bool rep = true;
      for (int s : stab) {
        const int im = perms->apply(s, card);
        if (im < card) rep = false;
        bool seen = false;
        for (int q = 0; q < orbit; ++q) seen |= images[2 * q] == im;
        if (!seen && orbit < 12) {
          images[2 * orbit] = im;
          images[2 * orbit + 1] = s;
          ++orbit;
        }
      }
      if (!rep) continue;
      if (orbit == 0) {
        images[0] = card;
        images[1] = 0;
        orbit = 1;
      }
      Ctx Y;
      turn_ctx(X, card, Y);
      std::memcpy(f0, r0, kC * sizeof(double));
      std::memcpy(f1, r1, kC * sizeof(double));
      for (int j = 0; j < 51; ++j) {
        const int c = K.holding[card][j];
        f0[c] = 0.0;
        f1[c] = 0.0;
      }
      walk(next, Y, f0, f1, c0, c1, wch * pw * orbit);
      for (int q = 0; q < orbit; ++q) {
        const int* inv = perms->inv_combo[images[2 * q + 1]];
        if (images[2 * q + 1] == 0) {
          for (int c = 0; c < kC; ++c) {
            v0[c] += pw * c0[c];
            v1[c] += pw * c1[c];
          }
        } else {
          for (int c = 0; c < kC; ++c) {
            v0[c] += pw * c0[inv[c]];
            v1[c] += pw * c1[inv[c]];
          }
        }
      }
    }
  } else {
    double* f0 = alloc(kRiverMax);
    double* f1 = alloc(kRiverMax);
    double* c0 = alloc(kRiverMax);
    double* c1 = alloc(kRiverMax);
    uint8_t cards[5];
    for (int i = 0; i < 4; ++i) cards[i] = X.cards[i];
    for (int card = 0; card < 52; ++card) {
      if ((X.mask >> card) & 1) continue;
      cards[4] = (uint8_t)card;
      RiverBoard R = river_board(cards, E.full ? (int)X.cards[3] * 52 + card : card);
      R.river = card;
      for (int j = 0; j < R.n; ++j) {
        f0[j] = r0[R.combo[j]];
        f1[j] = r1[R.combo[j]];
      }
      rwalk(next, R, f0, f1, c0, c1, wch * pw);
      for (int j = 0; j < R.n; ++j) {
        v0[R.combo[j]] += pw * c0[j];
        v1[R.combo[j]] += pw * c1[j];
      }
    }
  }
  top = mark;
}

// ---- river walks: vectors over R's combos in ascending rank order -----------
// Terminal values go to a sink: stored, or folded straight into the parent
// decision's accumulators (max for the acting player, sum for the other).
struct WriteSink {
  double* v0;
  double* v1;
  void operator()(int j, double a, double b) const {
    v0[j] = a;
    v1[j] = b;
  }
};
struct CombineSink {
  double* vp;  // acting player: max over actions
  double* vo;  // other player: sum over actions
  int p;
  bool first;
  void operator()(int j, double a, double b) const {
    const double x = p ? b : a, y = p ? a : b;
    if (first) {
      vp[j] = x;
      vo[j] = y;
    } else {
      vp[j] = std::max(vp[j], x);
      vo[j] += y;
    }
  }
};

// Both players at once: lane 0 holds player 0's quantities (built from
// player 1's reach), lane 1 player 1's (from player 0's reach).
typedef double v2d __attribute__((vector_size(16)));

template <class Sink>
void Worker::rfold(const Node& n, const RiverBoard& R, const double* r0, const double* r1, Sink&& sink, double wch) {
  const int m = R.n;
  const v2d pay = {(0 == n.player) ? (double)(n.pot - n.inv[0]) : -(double)n.inv[0],
                   (1 == n.player) ? (double)(n.pot - n.inv[1]) : -(double)n.inv[1]};
  // per-card sums by gathering each card's 46 combos (independent chains),
  // the total as half their sum (every combo holds two cards)
  v2d S = {0.0, 0.0}, Sc[52];
  for (int c = 0; c < 52; ++c) {
    v2d a = {0.0, 0.0}, b = {0.0, 0.0};
    if (!((R.mask >> c) & 1)) {
      const uint16_t* pos = R.bycard + c * 46;
      for (int t = 0; t < 46; t += 2) {
        const int j = pos[t], k = pos[t + 1];
        a += v2d{r1[j], r0[j]};
        b += v2d{r1[k], r0[k]};
      }
    }
    Sc[c] = a + b;
    S += Sc[c];
  }
  S *= 0.5;
  v2d pv = {0.0, 0.0};
  for (int j = 0; j < m; ++j) {
    const v2d x = {r1[j], r0[j]};
    const v2d own = {r0[j], r1[j]};
    const v2d val = pay * (S - Sc[R.lo[j]] - Sc[R.hi[j]] + x);
    sink(j, val[0], val[1]);
    pv += own * val;
  }
  prof[0] += wch * pv[0];
  prof[1] += wch * pv[1];
}

// Heads-up showdown: the winner takes min(inv) from the loser (the excess of
// the larger investment comes back, side_pot_payoff in traverse_ref.cuh); a
// tie moves nothing.  One sweep over the rank groups in ascending order keeps
// `below` and cb[card], the other player's reach summed over weaker combos
// (total and per card): before a group is added they give each member's wins,
// after it wins plus ties; at the end they are the totals that give each
// combo's compatible mass.  value = share * (wins - losses).
template <class Sink>
void Worker::rshowdown(const Node& n, const RiverBoard& R, const double* r0, const double* r1, Sink&& sink,
                       double wch) {
  const int m = R.n;
  const size_t mark = top;
  v2d* acc = reinterpret_cast<v2d*>(alloc(2 * (size_t)kRiverMax));
  const double share = (double)std::min(n.inv[0], n.inv[1]);
  v2d below = {0.0, 0.0}, cb[52];
  for (int c = 0; c < 52; ++c) cb[c] = below;
  for (int k = 0; k < m;) {
    const int e = R.gend[k];
    for (int j = k; j < e; ++j) acc[j] = below - cb[R.lo[j]] - cb[R.hi[j]];
    for (int j = k; j < e; ++j) {
      const v2d x = {r1[j], r0[j]};
      below += x;
      cb[R.lo[j]] += x;
      cb[R.hi[j]] += x;
    }
    for (int j = k; j < e; ++j) {
      const v2d x = {r1[j], r0[j]};
      acc[j] += below - cb[R.lo[j]] - cb[R.hi[j]] + x;  // wins + (wins + ties)
    }
    k = e;
  }
  v2d pv = {0.0, 0.0};
  const v2d sh = {share, share};
  for (int j = 0; j < m; ++j) {
    const v2d x = {r1[j], r0[j]};
    const v2d own = {r0[j], r1[j]};
    const v2d compat = below - cb[R.lo[j]] - cb[R.hi[j]] + x;
    const v2d val = sh * (acc[j] - compat);
    sink(j, val[0], val[1]);
    pv += own * val;
  }
  prof[0] += wch * pv[0];
  prof[1] += wch * pv[1];
  top = mark;
}

void Worker::rwalk(int ni, const RiverBoard& R, const double* r0, const double* r1, double* v0, double* v1,
                   double wch) {
  const Node& n = E.nodes[ni];
  switch (n.type) {
    case kDecision:
      rdecision(n, R, r0, r1, v0, v1, wch);
      return;
    case kFold:
      rfold(n, R, r0, r1, WriteSink{v0, v1}, wch);
      return;
    case kShowdown:
      rshowdown(n, R, r0, r1, WriteSink{v0, v1}, wch);
      return;
    default:  // depth cut (no deal follows the river)
      std::fill(v0, v0 + R.n, 0.0);
      std::fill(v1, v1 + R.n, 0.0);
  }
}

void Worker::rdecision(const Node& n, const RiverBoard& R, const double* r0, const double* r1, double* v0,
                       double* v1, double wch) {
  const int p = n.player, na = n.nact, m = R.n;
  const size_t mark = top;
  const double* S;
  const uint16_t* rowidx = nullptr;
  if (E.full) {
    S = E.dense.data() + n.strat;
    rowidx = R.bidx;
  } else {
    double* buf = alloc((size_t)m * na);
    subgame_strats(E, n, R.combo, m, R.river, buf);
    S = buf;
  }
  const double* rp = p ? r1 : r0;
  double* rc = alloc(kRiverMax);
  double* c0 = alloc(kRiverMax);
  double* c1 = alloc(kRiverMax);
  double* vp = p ? v1 : v0;
  double* vo = p ? v0 : v1;
  for (int i = 0; i < na; ++i) {
    if (rowidx) {
      for (int j = 0; j < m; ++j) rc[j] = rp[j] * S[(size_t)rowidx[j] * na + i];
    } else {
      for (int j = 0; j < m; ++j) rc[j] = rp[j] * S[(size_t)j * na + i];
    }
    const Node& ch = E.nodes[n.child[i]];
    const double* a0 = p ? r0 : rc;
    const double* a1 = p ? rc : r1;
    if (ch.type == kFold) {
      rfold(ch, R, a0, a1, CombineSink{vp, vo, p, i == 0}, wch);
      continue;
    }
    if (ch.type == kShowdown) {
      rshowdown(ch, R, a0, a1, CombineSink{vp, vo, p, i == 0}, wch);
      continue;
    }
    rwalk(n.child[i], R, a0, a1, c0, c1, wch);
    const double* cp = p ? c1 : c0;
    const double* co = p ? c0 : c1;
    if (i == 0) {
      std::memcpy(vp, cp, m * sizeof(double));
      std::memcpy(vo, co, m * sizeof(double));
    } else {
      for (int j = 0; j < m; ++j) {
        vp[j] = std::max(vp[j], cp[j]);
        vo[j] += co[j];
      }
    }
  }
  top = mark;
}

struct FlopClass {
  uint8_t cards[3];
  std::vector<int> images;  // one permutation per distinct image of the class
};

std::vector<FlopClass> flop_classes(const SuitPerms& P) {
  auto code = [](int a, int b, int c) {
    int x[3] = {a, b, c};
    std::sort(x, x + 3);
    return (x[0] << 12) | (x[1] << 6) | x[2];
  };
  std::vector<FlopClass> out;
  for (int a = 0; a < 52; ++a)
    for (int b = a + 1; b < 52; ++b)
      for (int c = b + 1; c < 52; ++c) {
        const int self = code(a, b, c);
        int best = self;
        for (int s = 0; s < 24; ++s) best = std::min(best, code(P.apply(s, a), P.apply(s, b), P.apply(s, c)));
        if (best != self) continue;  // not the class representative
        FlopClass F;
        F.cards[0] = (uint8_t)a;
        F.cards[1] = (uint8_t)b;
        F.cards[2] = (uint8_t)c;
        std::vector<int> seen;
        for (int s = 0; s < 24; ++s) {
          const int im = code(P.apply(s, a), P.apply(s, b), P.apply(s, c));
          if (std::find(seen.begin(), seen.end(), im) != seen.end()) continue;
          seen.push_back(im);
          F.images.push_back(s);
        }
        out.push_back(F);
      }
  return out;
}

int hw_threads(int want) {
  if (want > 0) return want;
  const unsigned n = std::thread::hardware_concurrency();
  return n ? (int)n : 1;
}

}  // namespace

int run_best_response(const BrInput& in, const mccfr_br_options& opt, mccfr_exploit* out, std::string& err) {
  const auto t0 = std::chrono::steady_clock::now();
  const mccfr_config& cfg = *in.cfg;
  if (cfg.num_players != 2) return err = "best response is heads-up only", MCCFR_ERR_INVALID_ARG;
  const Combos& K = CB();
  auto Ep = std::make_unique<Engine>();
  Engine& E = *Ep;
  E.G = *in.G;
  E.T = in.T;
  E.full = E.G.sub_street == 0;
  E.sub_street = E.G.sub_street;
  const int threads = hw_threads(opt.threads);
  std::memset(out, 0, sizeof(*out));
  out->threads = threads;
  out->rows = (long long)in.rows;
  out->exact = 1;
  E.rows.build(in.keys, in.ssum, in.rows);

  double br[2] = {0.0, 0.0}, pv[2] = {0.0, 0.0};
  if (E.full) {
    if (cfg.postflop_mode != MCCFR_POSTFLOP_RANK_CDF)
      return err = "full-game best response needs rank-CDF postflop buckets (suit-invariant keys)",
             MCCFR_ERR_INVALID_ARG;
    build_preflop_lut(cfg.preflop_mode, cfg.preflop_buckets, E.pre);
    E.H = cfg.preflop_mode == MCCFR_PREFLOP_CLASS169 ? 169 : cfg.preflop_buckets;
    for (int s = 0; s < 3; ++s) {
      E.B[s + 1] = cfg.postflop_buckets[s];
      unsigned long long hist[7463];
      host_rank_hist(E.T, 5 + s, hist, threads);
      build_cdf_lut(hist, cfg.postflop_buckets[s], E.cdf[s]);
    }
    for (int c = 0; c < kC; ++c) E.hb[c] = E.pre[K.lo[c] * 52 + K.hi[c]];
    for (int d = 0; d < 2; ++d) E.root[d] = build_tree(E.G, E.nodes, full_root(E.G, d), d);
    // dense strategy tables: every (preflop class, street bucket) of every decision node
    long long off = 0;
    for (auto& n : E.nodes)
      if (n.type == kDecision) {
        n.strat = off;
        off += (long long)E.H * E.B[n.street] * n.nact;
      }
    E.dense.assign((size_t)off, 0.0);
    for (auto& n : E.nodes) {
      if (n.type != kDecision) continue;
      for (int h = 0; h < E.H; ++h)
        for (int b = 0; b < E.B[n.street]; ++b)
          node_probs(E.rows, n, E.key_of(n, (uint32_t)h, (uint32_t)b),
                     E.dense.data() + n.strat + ((size_t)h * E.B[n.street] + b) * n.nact);
    }
    for (int c = 0; c < kC; ++c) E.w[0][c] = E.w[1][c] = 1.0;
    E.Z = 1326.0 * 1225.0;
  } else {
    E.root[0] = build_tree(E.G, E.nodes, sub_root(E.G), 1);
    const int nb = E.sub_street == 2 ? 4 : 5;
    for (int i = 0; i < nb; ++i) {
      E.board[i] = E.G.sub_board[i];
      E.board_mask |= 1ull << E.board[i];
    }
    for (int p = 0; p < 2; ++p)
      for (int c = 0; c < kC; ++c) E.w[p][c] = (K.mask[c] & E.board_mask) ? 0.0 : in.weights[p][c];
    E.Z = 0.0;
    for (int c = 0; c < kC; ++c) {
      if (E.w[0][c] == 0.0) continue;
      for (int o = 0; o < kC; ++o)
        if (!(K.mask[o] & K.mask[c])) E.Z += E.w[0][c] * E.w[1][o];
    }
    if (!(E.Z > 0.0)) return err = "the ranges have no disjoint pair of combos", MCCFR_ERR_INVALID_ARG;
  }
  out->nodes = (long long)E.nodes.size();

  if (!E.full) {
    Worker W(E);
    std::vector<double> v0(kC, 0.0), v1(kC, 0.0);
    if (E.sub_street == 2) {
      Ctx X;
      X.street = 2;
      X.ncards = 4;
      for (int i = 0; i < 4; ++i) X.cards[i] = E.board[i];
      X.mask = E.board_mask;
      W.walk(E.root[0], X, E.w[0], E.w[1], v0.data(), v1.data(), 1.0);
    } else {
      RiverBoard R = W.river_board(E.board, 0);
      std::vector<double> a0(R.n), a1(R.n), b0(R.n), b1(R.n);
      for (int j = 0; j < R.n; ++j) {
        a0[j] = E.w[0][R.combo[j]];
        a1[j] = E.w[1][R.combo[j]];
      }
      W.rwalk(E.root[0], R, a0.data(), a1.data(), b0.data(), b1.data(), 1.0);
      for (int j = 0; j < R.n; ++j) {
        v0[R.combo[j]] = b0[j];
        v1[R.combo[j]] = b1[j];
      }
    }
    if (W.overflow) return err = "best-response work space exhausted", MCCFR_ERR_CAPACITY;
    for (int c = 0; c < kC; ++c) {
      br[0] += E.w[0][c] * v0[c];
      br[1] += E.w[1][c] * v1[c];
    }
    pv[0] = W.prof[0];
    pv[1] = W.prof[1];
    out->boards = W.boards;
  } else {
    // Pass 1: each dealer's preflop tree to its flop deals, collecting reaches.
    std::vector<FlopEntry> entries;
    std::vector<int> entry_of(E.nodes.size(), -1);
    for (int d = 0; d < 2; ++d) {
      std::vector<int> stack{E.root[d]};
      while (!stack.empty()) {
        const int ni = stack.back();
        stack.pop_back();
        const Node& n = E.nodes[ni];
        if (n.type == kDecision)
          for (int i = 0; i < n.nact; ++i) stack.push_back(n.child[i]);
        if (n.type == kDeal && n.street == 1) {
          entry_of[ni] = (int)entries.size();
          FlopEntry F;
          F.node = ni;
          F.dealer = d;
          entries.push_back(F);
        }
      }
    }
    std::vector<std::vector<double>> entry_val(2 * entries.size(), std::vector<double>(kC, 0.0));
    {
      Worker W(E);
      W.entries = &entries;
      W.entry_of = &entry_of;
      W.entry_val = &entry_val;
      W.preflop_pass = 1;
      std::vector<double> v0(kC), v1(kC);
      Ctx X;
      X.bidx = E.hb;  // preflop: the class of each combo
      for (int d = 0; d < 2; ++d) W.walk(E.root[d], X, E.w[0], E.w[1], v0.data(), v1.data(), 0.5);
    }
    // Flop classes over threads; each thread sums into its own accumulators.
    const SuitPerms P;
    const std::vector<FlopClass> classes = flop_classes(P);
    const int stride = std::max(1, opt.flop_stride);
    long long weight_total = 0;
    for (size_t f = 0; f < classes.size(); f += stride) weight_total += (long long)classes[f].images.size();
    const double scale = 22100.0 / (double)weight_total;
    if (stride > 1) out->exact = 0;
    std::vector<std::vector<double>> acc(threads, std::vector<double>(2 * entries.size() * kC, 0.0));
    std::vector<double> tprof(2 * threads, 0.0);
    std::vector<long long> tboards(threads, 0);
    std::vector<int> toverflow(threads, 0);
    std::atomic<int> done{0};
    const int nsel = (int)((classes.size() + stride - 1) / stride);
    std::vector<double> iso_part(threads, 0.0);
    auto run = [&](int tid) {
      Worker W(E);
      W.entries = &entries;
      W.entry_of = &entry_of;
      std::vector<double> f0(kC), f1(kC), c0(kC), c1(kC);
      auto one_flop = [&](const uint8_t* flop, const FlopEntry& F, double wprof) {
        Ctx X;
        W.flop_ctx(flop, X);
        std::copy(F.r[0].begin(), F.r[0].end(), f0.begin());
        std::copy(F.r[1].begin(), F.r[1].end(), f1.begin());
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 51; ++j) {
            const int c = K.holding[flop[i]][j];
            f0[c] = f1[c] = 0.0;
          }
        W.walk(E.nodes[F.node].next, X, f0.data(), f1.data(), c0.data(), c1.data(), wprof);
      };
      W.perms = &P;
      for (int k = tid; k < nsel; k += threads) {
        const FlopClass& FC = classes[(size_t)k * stride];
        W.reset_flop_caches();
        W.stab.clear();
        for (int s = 0; s < 24; ++s) {
          int im[3];
          for (int i = 0; i < 3; ++i) im[i] = P.apply(s, FC.cards[i]);
          std::sort(im, im + 3);
          if (im[0] == FC.cards[0] && im[1] == FC.cards[1] && im[2] == FC.cards[2]) W.stab.push_back(s);
        }
        const double pf = scale / 17296.0;
        for (size_t e = 0; e < entries.size(); ++e) {
          one_flop(FC.cards, entries[e], 0.5 * pf * (double)FC.images.size());
          double* a0 = acc[tid].data() + (2 * e) * kC;
          double* a1 = acc[tid].data() + (2 * e + 1) * kC;
          for (int s : FC.images) {
            const int* inv = P.inv_combo[s];
            for (int c = 0; c < kC; ++c) {
              a0[c] += pf * c0[inv[c]];
              a1[c] += pf * c1[inv[c]];
            }
          }
          // Self-check: one permuted image of the class computed directly must
          // equal the permuted values of the representative.
          if ((opt.flags & MCCFR_BR_ISO_CHECK) && k < 3 * threads && FC.images.size() > 1) {
            const int s = FC.images.back();
            const int* inv = P.inv_combo[s];
            uint8_t img[3];
            for (int i = 0; i < 3; ++i) img[i] = (uint8_t)P.apply(s, FC.cards[i]);
            const std::vector<double> p0(c0), p1(c1);
            const double keep0 = W.prof[0], keep1 = W.prof[1];
            const long long keepb = W.boards;
            W.reset_flop_caches();  // the river cache is keyed by (turn, river) of one flop
            const std::vector<int> keep_stab = W.stab;
            W.stab.assign(1, 0);  // every turn card walked: checks the turn symmetry too
            one_flop(img, entries[e], 0.0);
            W.stab = keep_stab;
            W.reset_flop_caches();
            W.prof[0] = keep0;
            W.prof[1] = keep1;
            W.boards = keepb;
            double diff = 0.0, scale = 1e-300;
            for (int c = 0; c < kC; ++c) {
              diff = std::max(diff, std::max(std::fabs(c0[c] - p0[inv[c]]), std::fabs(c1[c] - p1[inv[c]])));
              scale = std::max(scale, std::max(std::fabs(p0[c]), std::fabs(p1[c])));
            }
            iso_part[tid] = std::max(iso_part[tid], diff / scale);
          }
        }
        const int n = ++done;
        if ((opt.flags & MCCFR_BR_VERBOSE) && tid == 0) {
          const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
          fprintf(stderr, "best response: %d/%d flop classes, %.0f s\n", n, nsel, el);
        }
      }
      tprof[2 * tid] = W.prof[0];
      tprof[2 * tid + 1] = W.prof[1];
      tboards[tid] = W.boards;
      toverflow[tid] = W.overflow;
    };
    std::vector<std::thread> th;
    for (int t = 1; t < threads; ++t) th.emplace_back(run, t);
    run(0);
    for (auto& t : th) t.join();
    for (int t = 0; t < threads; ++t)
      if (toverflow[t]) return err = "best-response work space exhausted", MCCFR_ERR_CAPACITY;
    for (size_t e = 0; e < entries.size(); ++e)
      for (int p = 0; p < 2; ++p) {
        std::vector<double>& v = entry_val[2 * e + p];
        for (int t = 0; t < threads; ++t) {
          const double* a = acc[t].data() + (2 * e + p) * kC;
          for (int c = 0; c < kC; ++c) v[c] += a[c];
        }
      }
    for (int t = 0; t < threads; ++t) {
      pv[0] += tprof[2 * t];
      pv[1] += tprof[2 * t + 1];
      out->boards += tboards[t];
    }
    // Pass 2: preflop values from the flop entries' values.
    Worker W(E);
    W.entries = &entries;
    W.entry_of = &entry_of;
    W.entry_val = &entry_val;
    W.preflop_pass = 2;
    std::vector<double> v0(kC), v1(kC);
    Ctx X;
    X.bidx = E.hb;
    for (int d = 0; d < 2; ++d) {
      W.walk(E.root[d], X, E.w[0], E.w[1], v0.data(), v1.data(), 0.5);
      for (int c = 0; c < kC; ++c) {
        br[0] += 0.5 * v0[c];
        br[1] += 0.5 * v1[c];
      }
    }
    pv[0] += W.prof[0];
    pv[1] += W.prof[1];
    for (double x : iso_part) out->iso_check = std::max(out->iso_check, x);
  }
  for (int p = 0; p < 2; ++p) {
    out->br_value[p] = br[p] / E.Z;
    out->profile_value[p] = pv[p] / E.Z;
  }
  out->exploitability = 0.5 * (out->br_value[0] + out->br_value[1]);
  out->mbb_per_game = out->exploitability / (double)E.G.bb * 1000.0;
  out->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return MCCFR_OK;
}

}  // namespace mccfr
