// traverse_ref.cuh — deal kernel and the traversal kernel of the reference's rule.
//
// The reference runs one recursive traversal per thread, dealing and bucketing
// at its start, with its game state in local memory (cfr_gpu.cu:644-1011).  Here:
//   * k_deal deals every traversal of a player-update (counter-based Philox,
//     the reference's partial Fisher-Yates) and computes its buckets and river
//     ranks into a 64-byte record; the rank chains of all players share the
//     3-card board prefix (the table's state depends only on the set of cards,
//     which the tests check);
//   * under the reference's rule every node samples one action, so a traversal
//     is a single root-to-terminal path and every node on it returns the
//     terminal payoff u (cfr_gpu.cu:809-818): k_traverse_ref walks the path
//     iteratively, one thread per traversal, with per-player chip counts and
//     buckets in shared memory (column-major [field][thread], conflict-free,
//     indexable by player without local memory);
//   * each node reads its regret row once (a 32-byte sector) from a snapshot
//     that the update does not modify; the updating player's nodes are recorded
//     in shared memory and, when u is known, folded into the row's fixed-point
//     accumulators with three atomics (visit count, sum of u, sampled-action
//     delta).
// No dynamically indexed per-thread array stays alive across the walk.
#pragma once
#include "game.cuh"
#include "table.cuh"
#include "../../include/mccfr.h"

namespace mccfr {

struct Sched {
  long long iteration;  // 1-based
  int player;
  int pad;
};

struct HandView {
  const int32_t* hr;      // rank table
  const uint8_t* pre;     // preflop LUT [52*52]
  const uint8_t* cdf;     // rank-CDF LUTs [3][7463]
};

// One traversal's deal.  ctx[p] = hole bucket | flop << 8 | turn << 16 | river << 24.
struct DealRec {
  uint32_t ctx[kMaxPlayers];
  uint16_t rank[kMaxPlayers];
  uint8_t hole[2 * kMaxPlayers];
  uint8_t board[5];
  uint8_t dealer;
  uint8_t pad[10];
};
static_assert(sizeof(DealRec) == 64, "deal record is one 64-byte pair of sectors");

struct Counters {
  unsigned long long traversals, visits, updates, terminals, evals;
};

constexpr int kMaxRec = 24;

__device__ __forceinline__ void warp_add_counters(Counters* c, unsigned t, unsigned v, unsigned u,
                                                  unsigned x, unsigned e) {
  const unsigned m = __activemask();
  t = __reduce_add_sync(m, t);
  v = __reduce_add_sync(m, v);
  u = __reduce_add_sync(m, u);
  x = __reduce_add_sync(m, x);
  e = __reduce_add_sync(m, e);
  // only non-zero sums are added: a launch over an empty level adds nothing
  if ((threadIdx.x & 31) == (__ffs(m) - 1)) {
    if (t) atomicAdd(&c->traversals, (unsigned long long)t);
    if (v) atomicAdd(&c->visits, (unsigned long long)v);
    if (u) atomicAdd(&c->updates, (unsigned long long)u);
    if (x) atomicAdd(&c->terminals, (unsigned long long)x);
    if (e) atomicAdd(&c->evals, (unsigned long long)e);
  }
}

__device__ __forceinline__ uint32_t update_id(const Sched* s, int N) {
  return (uint32_t)((s->iteration - 1) * N + s->player);
}

// First combo whose cumulative weight exceeds w (w < 2^31), by bisection.
__device__ __forceinline__ int sample_combo(const uint32_t* __restrict__ cdf, uint32_t w) {
  int lo = 0, hi = 1325;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (w < __ldg(cdf + mid)) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// Subgame deal: every player's hole combo from its range, all combos drawn
// together and redrawn (up to 16 times) until no two share a card; after that,
// player by player, the drawn combo or the next one of positive weight that
// fits.  On the turn the river card is then uniform among the unused cards.
// ctx[p] = combo | (river card + 1) << 16 (the river card enters the river keys).
__device__ __forceinline__ void deal_subgame(const GameParams& G, const int32_t* __restrict__ T, uint32_t t,
                                             uint32_t uid, DealRec* __restrict__ out) {
  const int N = G.N;
  const int nb = G.sub_street == 2 ? 4 : 5;
  uint64_t used_board = 0;
  for (int i = 0; i < nb; ++i) used_board |= 1ull << G.sub_board[i];
  int combo[kMaxPlayers];
  uint64_t used = used_board;
  bool ok = false;
  for (int a = 0; a < 16 && !ok; ++a) {
    const U4 w0 = philox(U4{t, uid, 0x100u + (uint32_t)a, 0u}, G.seed_lo, G.seed_hi);
    const U4 w1 = philox(U4{t, uid, 0x100u + (uint32_t)a, 1u}, G.seed_lo, G.seed_hi);
    const uint32_t words[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
    used = used_board;
    ok = true;
    for (int p = 0; p < N && ok; ++p) {
      combo[p] = sample_combo(G.range_cdf + 1326 * p, words[p] >> 1);
      int lo, hi;
      combo_cards(combo[p], lo, hi);
      const uint64_t m = (1ull << lo) | (1ull << hi);
      if (used & m) ok = false;
      used |= m;
    }
  }
  if (!ok) {
    const U4 w0 = philox(U4{t, uid, 0x100u, 0u}, G.seed_lo, G.seed_hi);
    const U4 w1 = philox(U4{t, uid, 0x100u, 1u}, G.seed_lo, G.seed_hi);
    const uint32_t words[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
    used = used_board;
    for (int p = 0; p < N; ++p) {
      const uint32_t* cdf = G.range_cdf + 1326 * p;
      const int start = sample_combo(cdf, words[p] >> 1);
      int pick = -1;
      for (int k = 0; k < 1326 && pick < 0; ++k) {
        const int c = (start + k) % 1326;
        const uint32_t prev = c ? __ldg(cdf + c - 1) : 0u;
        if (__ldg(cdf + c) == prev) continue;  // zero weight
        int lo, hi;
        combo_cards(c, lo, hi);
        if (!(used & ((1ull << lo) | (1ull << hi)))) pick = c;
      }
      if (pick < 0) pick = start;  // range exhausted by card removal: keep the draw
      combo[p] = pick;
      int lo, hi;
      combo_cards(pick, lo, hi);
      used |= (1ull << lo) | (1ull << hi);
    }
  }
  DealRec r;
  for (int i = 0; i < 10; ++i) r.pad[i] = 0;
  for (int i = 0; i < 5; ++i) r.board[i] = (i < nb) ? G.sub_board[i] : 0;
  int river = -1;
  if (nb == 4) {
    const U4 w = philox(U4{t, uid, 0x200u, 0u}, G.seed_lo, G.seed_hi);
    const int free_cards = 52 - __popcll(used);
    int k = (int)(((unsigned long long)w.x * (unsigned long long)free_cards) >> 32);
    for (int c = 0; c < 52; ++c) {
      if ((used >> c) & 1) continue;
      if (k-- == 0) {
        river = c;
        break;
      }
    }
    r.board[4] = (uint8_t)river;
  }
  r.dealer = (uint8_t)(N - 1);
  int32_t b = __ldg(T + 53 + to_rm(r.board[0]));
  for (int i = 1; i < 5; ++i) b = __ldg(T + b + to_rm(r.board[i]));
  for (int p = 0; p < kMaxPlayers; ++p) {
    r.ctx[p] = 0;
    r.rank[p] = 0;
    r.hole[2 * p] = r.hole[2 * p + 1] = 0;
    if (p >= N) continue;
    int lo, hi;
    combo_cards(combo[p], lo, hi);
    r.hole[2 * p] = (uint8_t)lo;
    r.hole[2 * p + 1] = (uint8_t)hi;
    const int32_t s6 = __ldg(T + b + to_rm(lo));
    r.rank[p] = (uint16_t)decode16((uint32_t)__ldg(T + s6 + to_rm(hi)) & 0xFFFF);
    r.ctx[p] = (uint32_t)combo[p] | ((uint32_t)(river + 1) << 16);
  }
  const uint4* src = reinterpret_cast<const uint4*>(&r);
  uint4* dst = reinterpret_cast<uint4*>(out);
#pragma unroll
  for (int i = 0; i < 4; ++i) dst[i] = src[i];
}

// Deal, buckets and river ranks of traversal t of update `uid`
// (cfr_gpu.cu:460-470, 476-489, 942-952, 963).  `pre` is the 52x52 preflop LUT
// (shared or global memory), `cdf` the rank-CDF LUTs.
__device__ __forceinline__ void deal_one(const GameParams& G, const int32_t* __restrict__ T, const uint8_t* pre,
                                         const uint8_t* __restrict__ cdf, uint32_t t, uint32_t uid,
                                         DealRec* __restrict__ out) {
  if (G.sub_street) {
    deal_subgame(G, T, t, uid, out);
    return;
  }
  const int N = G.N;
  const int n_deal = 2 * N + 5;
  uint32_t words[24];
  const int nblk = (n_deal + 1 + 3) / 4;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    if (j < nblk) {
      const U4 o = philox(U4{t, uid, 0u, (uint32_t)j}, G.seed_lo, G.seed_hi);
      words[4 * j + 0] = o.x;
      words[4 * j + 1] = o.y;
      words[4 * j + 2] = o.z;
      words[4 * j + 3] = o.w;
    }
  }
  uint8_t deck[52];
#pragma unroll
  for (int i = 0; i < 52; ++i) deck[i] = (uint8_t)i;
  for (int i = 0; i < n_deal; ++i) {
    const int j = i + (int)(((unsigned long long)words[i] * (unsigned long long)(52 - i)) >> 32);
    const uint8_t tmp = deck[i];
    deck[i] = deck[j];
    deck[j] = tmp;
  }
  DealRec r;
#pragma unroll
  for (int i = 0; i < 2 * kMaxPlayers; ++i) r.hole[i] = (i < 2 * N) ? deck[i] : 0;
#pragma unroll
  for (int i = 0; i < 5; ++i) r.board[i] = deck[2 * N + i];
  r.dealer = (uint8_t)(words[n_deal] % (uint32_t)N);
#pragma unroll
  for (int i = 0; i < 10; ++i) r.pad[i] = 0;

  int32_t b = __ldg(T + 53 + to_rm(r.board[0]));
  b = __ldg(T + b + to_rm(r.board[1]));
  b = __ldg(T + b + to_rm(r.board[2]));
  int32_t s5[kMaxPlayers], s6[kMaxPlayers], r7[kMaxPlayers], s4[kMaxPlayers];
#pragma unroll
  for (int p = 0; p < kMaxPlayers; ++p)
    if (p < N) s4[p] = __ldg(T + b + to_rm(r.hole[2 * p]));
#pragma unroll
  for (int p = 0; p < kMaxPlayers; ++p)
    if (p < N) s5[p] = __ldg(T + s4[p] + to_rm(r.hole[2 * p + 1]));
  const int rm3 = to_rm(r.board[3]), rm4 = to_rm(r.board[4]);
#pragma unroll
  for (int p = 0; p < kMaxPlayers; ++p)
    if (p < N) s6[p] = __ldg(T + s5[p] + rm3);
#pragma unroll
  for (int p = 0; p < kMaxPlayers; ++p)
    if (p < N) r7[p] = __ldg(T + s6[p] + rm4);
#pragma unroll
  for (int p = 0; p < kMaxPlayers; ++p) {
    r.ctx[p] = 0;
    r.rank[p] = 0;
    if (p >= N) continue;
    const uint32_t hb = pre[r.hole[2 * p] * 52 + r.hole[2 * p + 1]];
    const uint32_t rr = decode16((uint32_t)r7[p] & 0xFFFF);
    uint32_t b1, b2, b3;
    if (G.postflop_mode == 0) {
      // the reference decodes the 5th/6th chain value (a state) as a rank
      b1 = ref_linear_bucket(decode16((uint32_t)s5[p] & 0xFFFF), G.post_b[0]);
      b2 = ref_linear_bucket(decode16((uint32_t)s6[p] & 0xFFFF), G.post_b[1]);
      b3 = ref_linear_bucket(rr, G.post_b[2]);
    } else {
      b1 = __ldg(cdf + decode16((uint32_t)__ldg(T + s5[p]) & 0xFFFF));
      b2 = __ldg(cdf + 7463 + decode16((uint32_t)__ldg(T + s6[p]) & 0xFFFF));
      b3 = __ldg(cdf + 2 * 7463 + rr);
    }
    r.ctx[p] = hb | (b1 << 8) | (b2 << 16) | (b3 << 24);
    r.rank[p] = (uint16_t)rr;
  }
  const uint4* src = reinterpret_cast<const uint4*>(&r);
  uint4* dst = reinterpret_cast<uint4*>(out);
#pragma unroll
  for (int i = 0; i < 4; ++i) dst[i] = src[i];
}

__global__ void __launch_bounds__(128) k_deal(const GameParams G, const HandView hv, const Sched* __restrict__ sched,
                                              int batch, DealRec* __restrict__ out) {
  __shared__ uint8_t s_pre[52 * 52];
  for (int i = threadIdx.x; i < 52 * 52 / 4; i += blockDim.x)
    reinterpret_cast<uint32_t*>(s_pre)[i] = __ldg(reinterpret_cast<const uint32_t*>(hv.pre) + i);
  __syncthreads();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (uint32_t)batch) return;
  deal_one(G, hv.hr, s_pre, hv.cdf, t, update_id(sched, G.N), out + t);
}

// Side-pot showdown for player `up` (cfr_gpu.cu:694-753).  The distinct non-zero
// invested amounts are visited in ascending order as "the smallest amount above
// the previous level", which is the reference's sorted level list without an
// array; invested chips and ranks are read through the caller's accessors.
template <class InvF, class RankF>
__device__ __forceinline__ float side_pot_payoff(int N, int up, uint32_t folded, InvF inv, RankF rank) {
  // The players' amounts and ranks are read once into fixed slots, so the
  // loops below index them with constants.
  int iv[kMaxPlayers];
  uint32_t rk[kMaxPlayers];
#pragma unroll
  for (int q = 0; q < kMaxPlayers; ++q) {
    iv[q] = q < N ? inv(q) : 0;
    rk[q] = q < N ? (uint32_t)rank(q) : 0u;
  }
  int inv_up = 0;
  uint32_t rk_up = 0;
#pragma unroll
  for (int q = 0; q < kMaxPlayers; ++q)
    if (q == up) {
      inv_up = iv[q];
      rk_up = rk[q];
    }
  const bool up_live = !((folded >> up) & 1);
  float payoff = -(float)inv_up;
  int prev = 0;
  for (int guard = 0; guard < kMaxPlayers; ++guard) {
    int L = 0x7FFFFFFF;
#pragma unroll
    for (int q = 0; q < kMaxPlayers; ++q)
      if (q < N && iv[q] > prev && iv[q] < L) L = iv[q];
    if (L == 0x7FFFFFFF) break;
    int layer = 0;
    uint32_t best = 0;
#pragma unroll
    for (int q = 0; q < kMaxPlayers; ++q)
      if (q < N) {
        layer += max(0, min(iv[q], L) - prev);
        if (!((folded >> q) & 1) && iv[q] >= L) best = max(best, rk[q]);
      }
    if (best > 0) {
      int nwin = 0;
#pragma unroll
      for (int q = 0; q < kMaxPlayers; ++q)
        if (q < N && !((folded >> q) & 1) && iv[q] >= L && rk[q] == best) nwin++;
      if (up_live && inv_up >= L && rk_up == best) payoff = __fadd_rn(payoff, __fdiv_rn((float)layer, (float)nwin));
    }
    prev = L;
  }
  return payoff;
}

__device__ __forceinline__ void load_regrets(const TableView& tv, long long slot, float* reg) {
  if (slot >= 0) {
    const float4* p = row_reg(tv, (unsigned long long)slot);
    const float4 r0 = __ldg(p), r1 = __ldg(p + 1);
    reg[0] = r0.x; reg[1] = r0.y; reg[2] = r0.z; reg[3] = r0.w;
    reg[4] = r1.x; reg[5] = r1.y; reg[6] = r1.z; reg[7] = r1.w;
  } else {
#pragma unroll
    for (int a = 0; a < kSlots; ++a) reg[a] = 0.0f;
  }
}

template <int BLOCK, bool TRACE>
__global__ void __launch_bounds__(BLOCK)
k_traverse_ref(const GameParams G, const TableView tv, const DealRec* __restrict__ deals, const Sched* __restrict__ sched,
               int batch, float rscale, Counters* __restrict__ counters, mccfr_trace* __restrict__ trace) {
  __shared__ uint16_t s_stack[kMaxPlayers][BLOCK];
  __shared__ uint16_t s_bet[kMaxPlayers][BLOCK];
  __shared__ uint16_t s_inv[kMaxPlayers][BLOCK];
  __shared__ uint16_t s_rank[kMaxPlayers][BLOCK];
  __shared__ uint32_t s_ctx[kMaxPlayers][BLOCK];
  // updating-player nodes of each thread's path: slot, sampled | mask << 8, q
  __shared__ uint32_t s_rec_slot[kMaxRec][BLOCK];
  __shared__ uint16_t s_rec_sv[kMaxRec][BLOCK];
  __shared__ float s_rec_q[kMaxRec][BLOCK];

  const int tid = threadIdx.x;
  const uint32_t t = blockIdx.x * BLOCK + tid;
  if (t >= (uint32_t)batch) return;
  const int N = G.N;
  const int up = sched->player;
  const uint32_t uid = update_id(sched, N);

  const DealRec& D = deals[t];
  const int dealer = D.dealer;
#pragma unroll
  for (int p = 0; p < kMaxPlayers; ++p)
    if (p < N) {
      s_ctx[p][tid] = D.ctx[p];
      s_rank[p][tid] = D.rank[p];
      s_stack[p][tid] = (uint16_t)G.stack;
      s_bet[p][tid] = 0;
      s_inv[p][tid] = 0;
    }

  // Blinds and preflop queue (cfr_gpu.cu:954-981), or a subgame's start.
  int pot, cb, lfr = G.bb, raises = 0, street = 0;
  uint32_t folded = 0, allin = 0, abits = 0;
  uint64_t path = kPathSeed;
  uint32_t q = 0;  // action queue, 4-bit entries
  int nq = 0;
  if (G.sub_street) {
#pragma unroll
    for (int p = 0; p < kMaxPlayers; ++p)
      if (p < N) s_inv[p][tid] = (uint16_t)(G.sub_pot / N);
    pot = G.sub_pot;
    cb = 0;
    street = G.sub_street;
    for (int i = 1; i <= N; ++i) q |= (uint32_t)seat_after(dealer, i, N) << (4 * nq++);
  } else {
    const int sbp = (N == 2) ? dealer : seat_after(dealer, 1, N);
    const int bbp = (N == 2) ? seat_after(dealer, 1, N) : seat_after(seat_after(dealer, 1, N), 1, N);
    const int sba = min(G.sb, G.stack), bba = min(G.bb, G.stack);
    s_stack[sbp][tid] = (uint16_t)(G.stack - sba);
    s_bet[sbp][tid] = (uint16_t)sba;
    s_inv[sbp][tid] = (uint16_t)sba;
    s_stack[bbp][tid] = (uint16_t)(G.stack - bba);
    s_bet[bbp][tid] = (uint16_t)bba;
    s_inv[bbp][tid] = (uint16_t)bba;
    pot = sba + bba;
    cb = bba;
    if (G.stack - sba == 0) allin |= 1u << sbp;
    if (G.stack - bba == 0) allin |= 1u << bbp;
    for (int i = 0; i < N; ++i) {
      const int p = seat_after(seat_after(bbp, 1, N), i, N);
      if (!((allin >> p) & 1)) q |= (uint32_t)p << (4 * nq++);
    }
  }

  int nrec = 0;
  unsigned n_visits = 0, n_updates = 0;
  int n_act = 0;
  float u = 0.0f;
  int depth = 0;
  const uint32_t all_players = (1u << N) - 1;
  for (;;) {
    if (depth >= G.max_depth) {
      u = 0.0f;
      break;
    }
    const uint32_t live = all_players & ~folded;
    if (__popc(live) == 1) {
      const int winner = __ffs(live) - 1;
      u = (winner == up) ? (float)(pot - (int)s_inv[up][tid]) : (float)(-(int)s_inv[up][tid]);
      break;
    }
    if (nq == 0) {
      bool showdown_now = true;
      if (street < 3) {
        street++;
#pragma unroll
        for (int p = 0; p < kMaxPlayers; ++p)
          if (p < N) s_bet[p][tid] = 0;
        cb = 0;
        lfr = G.bb;
        raises = 0;
        q = 0;
        nq = 0;
        for (int i = 1; i <= N; ++i) {
          const int p = seat_after(dealer, i, N);
          if (!((folded >> p) & 1) && !((allin >> p) & 1)) q |= (uint32_t)p << (4 * nq++);
        }
        if (nq > 0) {
          depth++;
          showdown_now = false;
        }
      }
      if (showdown_now) {
        u = side_pot_payoff(
            N, up, folded, [&](int x) { return (int)s_inv[x][tid]; }, [&](int x) { return (uint32_t)s_rank[x][tid]; });
        break;
      }
      continue;
    }
    // Decision node.
    const int player = (int)(q & 0xF);
    const int pstack = s_stack[player][tid];
    const int pbet = s_bet[player][tid];
    const int to_call = cb - pbet;
    const uint32_t vm = valid_mask(G, pot, pstack, to_call, cb, lfr, raises);
    const uint32_t cw = s_ctx[player][tid];
    uint32_t hb, bkt;
    if (G.sub_street) {  // exact combo; the river card once it is dealt
      hb = cw & 0xFFFF;
      bkt = (street == 3 && G.sub_street == 2) ? (cw >> 16) : 0u;
    } else {
      hb = cw & 0xFF;
      bkt = street ? ((cw >> (8 * street)) & 0xFF) : 0u;
    }
    const unsigned long long key = info_key(G, player, hb, bkt, street, abits, path);
    const bool is_up = (player == up);
    const long long slot = is_up ? table_insert(tv, key) : table_find(tv, key);
    float reg[kSlots];
    load_regrets(tv, slot, reg);
    n_visits++;
    const U4 d = philox(U4{t, uid, (uint32_t)path, (uint32_t)(path >> 32) | 0x80000000u}, G.seed_lo, G.seed_hi);
    const int s = sample_action(G, reg, vm, uniform01(d.x));
    if (is_up) {
      n_updates++;
      if (nrec < kMaxRec && slot >= 0) {
        float strat[kSlots];
        node_strategy(reg, vm, strat);
        s_rec_slot[nrec][tid] = (uint32_t)slot;
        s_rec_sv[nrec][tid] = (uint16_t)((uint32_t)s | (vm << 8));
        s_rec_q[nrec][tid] = fmaxf(strat[s], 0.05f);
        nrec++;
      } else if (slot >= 0) {
        atomicOr(tv.err, kErrRecordOverflow);
      }
    }
    if (TRACE) {
      if (n_act < 40) trace[t].actions[n_act] = (uint8_t)s;
    }
    n_act++;
    // pop the actor, apply (cfr_gpu.cu:803-807, 543-585)
    q >>= 4;
    nq--;
    const int chips = chips_for(G, s, pot, pstack, to_call, cb, lfr);
    abits = ((abits << 3) | (uint32_t)s) & 0x3FFFFFFFu;
    path = path_step(path, s);
    const int k = G.kind[s];
    if (k == 0) {
      folded |= 1u << player;
    } else if (k != 1) {
      const int nstack = pstack - chips, nbet = pbet + chips;
      s_stack[player][tid] = (uint16_t)nstack;
      s_bet[player][tid] = (uint16_t)nbet;
      s_inv[player][tid] = (uint16_t)(s_inv[player][tid] + chips);
      pot += chips;
      if (nstack == 0) allin |= 1u << player;
      if (nbet > cb) {
        const int prev = cb;
        const int rs = nbet - prev;
        if (rs >= lfr || prev == 0) lfr = rs;
        cb = nbet;
        raises++;
        q = 0;
        nq = 0;
        for (int i = 1; i < N; ++i) {
          const int p = seat_after(player, i, N);
          if (!((folded >> p) & 1) && !((allin >> p) & 1)) q |= (uint32_t)p << (4 * nq++);
        }
      }
    }
    depth++;
  }

  // Fold u into the recorded nodes' accumulators.
  const long long fu = fix_r(u, rscale);
  for (int i = 0; i < nrec; ++i) {
    const uint32_t slot = s_rec_slot[i][tid];
    const uint32_t sv = s_rec_sv[i][tid];
    const int s = (int)(sv & 0xFF);
    const uint32_t vm = sv >> 8;
    const long long dsamp = fix_r(__fsub_rn(__fdiv_rn(u, s_rec_q[i][tid]), u), rscale);
    if (touch_row(tv, slot, uid, vm)) {
      atomicAdd(row_cnt(tv, slot), (1ull << 32) | 1ull);
      atomicAdd(row_su(tv, slot), (unsigned long long)fu);
      mark_deltas(tv, slot);
      atomicAdd(row_da(tv, slot) + s, (unsigned long long)(dsamp + fu));
    } else {
      // Mask differs from the row's canonical one (an FNV slot shared by states
      // with different legal actions): add every term directly.
      atomicAdd(row_cnt(tv, slot), 1ull << 32);
      float reg[kSlots], strat[kSlots];
      load_regrets(tv, slot, reg);
      node_strategy(reg, vm, strat);
      long long dr[kSlots], dw[kSlots];
#pragma unroll
      for (int a = 0; a < kSlots; ++a) {
        dr[a] = (a == s) ? dsamp : -fu;
        dw[a] = fix_s(strat[a]);
      }
      add_direct(tv, slot, vm, dr, dw);
    }
  }
  if (TRACE) {
    mccfr_trace& tr = trace[t];
    for (int i = 0; i < 12; ++i) tr.hole[i] = D.hole[i];
    for (int i = 0; i < 5; ++i) tr.board[i] = D.board[i];
    tr.dealer = (uint8_t)dealer;
    tr.n_actions = (uint8_t)n_act;
    tr.n_traverser_nodes = (uint8_t)nrec;
    for (int p = 0; p < 6; ++p) {
      const uint32_t cw = D.ctx[p];
      tr.hole_bucket[p] = (uint8_t)(cw & 0xFF);
      tr.board_bucket[p][0] = 0;
      tr.board_bucket[p][1] = (uint8_t)(cw >> 8);
      tr.board_bucket[p][2] = (uint8_t)(cw >> 16);
      tr.board_bucket[p][3] = (uint8_t)(cw >> 24);
    }
    tr.payoff = u;
    tr.reserved = 0;
  }
  warp_add_counters(counters, 1u, n_visits, n_updates, 1u, (unsigned)N);
}

}  // namespace mccfr
