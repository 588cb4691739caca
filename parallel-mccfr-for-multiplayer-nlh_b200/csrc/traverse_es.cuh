// traverse_es.cuh — external-sampling traversal kernel.
//
// Under external sampling the updating player explores every legal action and
// the other players sample one (the reference samples at both, cfr_gpu.cu:768-859).
// Each traversal is a depth-first walk of the updating player's subtree with an
// explicit frame stack (the reference recurses with a 16 KB per-thread stack,
// cfr_gpu.cu:1253-1258):
//   * a frame is pushed at each updating-player node; children are visited in
//     slot order, and the node value v_h = sum_a strat[a] * v[a] is accumulated
//     in that order as the children return;
//   * each child value v[a] is added to the row's accumulator at once
//     (fix(v[a]) into da[a]); when the node completes, fix(v_h) is subtracted from
//     every legal action (through `su` when the mask is the row's canonical one),
//     so the regret delta of action a is fix(v[a]) - fix(v_h);
//   * sampled opponents' nodes add their regret-matched strategy to the row's
//     strategy sum (a visit count when the mask is canonical).
#pragma once
#include "game.cuh"
#include "table.cuh"
#include "traverse_ref.cuh"

namespace mccfr {

struct EsState {
  uint16_t stack[kMaxPlayers], bet[kMaxPlayers], inv[kMaxPlayers];
  int pot;
  int cb, lfr;
  uint32_t q;        // action queue, 4-bit entries
  uint32_t abits;
  uint64_t path;
  uint8_t folded, allin, street, raises, nq, depth, pad0, pad1;
};

struct EsFrame {
  EsState st;
  float strat[kSlots];
  float vh;
  uint32_t slot;
  uint8_t vm, next_a, player, pad;
};

constexpr int kMaxFrames = 24;

// Applies action a of `player` (cfr_gpu.cu:543-585, 803-807).
__device__ __forceinline__ void es_apply(const GameParams& G, EsState& s, int player, int a) {
  s.q >>= 4;
  s.nq--;
  const int pstack = s.stack[player], pbet = s.bet[player];
  const int to_call = s.cb - pbet;
  const int chips = chips_for(G, a, s.pot, pstack, to_call, s.cb, s.lfr);
  s.abits = ((s.abits << 3) | (uint32_t)a) & 0x3FFFFFFFu;
  s.path = path_step(s.path, a);
  const int k = G.kind[a];
  if (k == 0) {
    s.folded |= (uint8_t)(1u << player);
    return;
  }
  if (k == 1) return;
  const int nstack = pstack - chips, nbet = pbet + chips;
  s.stack[player] = (uint16_t)nstack;
  s.bet[player] = (uint16_t)nbet;
  s.inv[player] = (uint16_t)(s.inv[player] + chips);
  s.pot += chips;
  if (nstack == 0) s.allin |= (uint8_t)(1u << player);
  if (nbet > s.cb) {
    const int prev = s.cb;
    const int rs = nbet - prev;
    if (rs >= s.lfr || prev == 0) s.lfr = rs;
    s.cb = nbet;
    s.raises++;
    s.q = 0;
    s.nq = 0;
    for (int i = 1; i < G.N; ++i) {
      const int p = (player + i) % G.N;
      if (!((s.folded >> p) & 1) && !((s.allin >> p) & 1)) s.q |= (uint32_t)p << (4 * s.nq++);
    }
  }
}

// Frame storage of one thread's walk: frames [0, K) in the caller's shared
// memory (this thread's column, stride `stride` frames), deeper ones in local
// memory.  K is an autotuned shared-memory stack depth.
template <int K>
struct FrameStack {
  EsFrame* smem;
  int stride;
  EsFrame local[kMaxFrames - K];
  __device__ __forceinline__ EsFrame& at(int i) {
    if (K > 0 && i < K) return smem[i * stride];
    return local[i - K];
  }
};

struct EsCounts {
  unsigned visits, updates, terminals;
};

// One external-sampling traversal (deal `D`, traversal index t, update uid of
// player `up`): the updating player's subtree depth-first, opponents sampled.
template <int W, class Frames>
__device__ __forceinline__ void es_walk(const GameParams& G, const TableView& tv, const DealRec& D, uint32_t t,
                                        uint32_t uid, int up, float rscale, Frames& fr, EsCounts& cnt) {
  const int N = G.N;
  const int dealer = D.dealer;
  uint32_t ctx[kMaxPlayers], rank[kMaxPlayers];
#pragma unroll
  for (int p = 0; p < kMaxPlayers; ++p) {
    ctx[p] = D.ctx[p];
    rank[p] = D.rank[p];
  }
  EsState cur;
  if (G.sub_street) {
    // subgame: the dead pot split equally, everyone with the same stack, first
    // to act after the dealer (the last seat)
    for (int p = 0; p < kMaxPlayers; ++p) {
      cur.stack[p] = (uint16_t)G.stack;
      cur.bet[p] = 0;
      cur.inv[p] = (uint16_t)((p < N) ? G.sub_pot / N : 0);
    }
    cur.pot = G.sub_pot;
    cur.cb = 0;
    cur.lfr = G.bb;
    cur.folded = 0;
    cur.allin = 0;
    cur.street = (uint8_t)G.sub_street;
    cur.raises = 0;
    cur.abits = 0;
    cur.path = kPathSeed;
    cur.depth = 0;
    cur.q = 0;
    cur.nq = 0;
    for (int i = 1; i <= N; ++i) cur.q |= (uint32_t)((dealer + i) % N) << (4 * cur.nq++);
  } else {
    for (int p = 0; p < kMaxPlayers; ++p) {
      cur.stack[p] = (uint16_t)G.stack;
      cur.bet[p] = 0;
      cur.inv[p] = 0;
    }
    const int sbp = (N == 2) ? dealer : (dealer + 1) % N;
    const int bbp = (N == 2) ? (dealer + 1) % N : (dealer + 2) % N;
    const int sba = min(G.sb, G.stack), bba = min(G.bb, G.stack);
    cur.stack[sbp] = (uint16_t)(G.stack - sba);
    cur.bet[sbp] = (uint16_t)sba;
    cur.inv[sbp] = (uint16_t)sba;
    cur.stack[bbp] = (uint16_t)(G.stack - bba);
    cur.bet[bbp] = (uint16_t)bba;
    cur.inv[bbp] = (uint16_t)bba;
    cur.pot = sba + bba;
    cur.cb = bba;
    cur.lfr = G.bb;
    cur.folded = 0;
    cur.allin = 0;
    if (G.stack - sba == 0) cur.allin |= (uint8_t)(1u << sbp);
    if (G.stack - bba == 0) cur.allin |= (uint8_t)(1u << bbp);
    cur.street = 0;
    cur.raises = 0;
    cur.abits = 0;
    cur.path = kPathSeed;
    cur.depth = 0;
    cur.q = 0;
    cur.nq = 0;
    for (int i = 0; i < N; ++i) {
      const int p = (bbp + 1 + i) % N;
      if (!((cur.allin >> p) & 1)) cur.q |= (uint32_t)p << (4 * cur.nq++);
    }
  }

  int sp = 0;
  unsigned n_visits = 0, n_updates = 0, n_term = 0;
  const uint32_t all_players = (1u << N) - 1;
  bool aborted = false;

  for (;;) {
    // ---- descend from `cur` to a terminal value or an updating-player node
    float value = 0.0f;
    bool pushed = false;
    for (;;) {
      if (cur.depth >= G.max_depth) {
        value = 0.0f;
        n_term++;
        break;
      }
      const uint32_t live = all_players & ~(uint32_t)cur.folded;
      if (__popc(live) == 1) {
        const int winner = __ffs(live) - 1;
        value = (winner == up) ? (float)(cur.pot - (int)cur.inv[up]) : (float)(-(int)cur.inv[up]);
        n_term++;
        break;
      }
      if (cur.nq == 0) {
        if (cur.street < 3) {
          cur.street++;
          for (int p = 0; p < kMaxPlayers; ++p) cur.bet[p] = 0;
          cur.cb = 0;
          cur.lfr = G.bb;
          cur.raises = 0;
          cur.q = 0;
          cur.nq = 0;
          for (int i = 1; i <= N; ++i) {
            const int p = (dealer + i) % N;
            if (!((cur.folded >> p) & 1) && !((cur.allin >> p) & 1)) cur.q |= (uint32_t)p << (4 * cur.nq++);
          }
          if (cur.nq > 0) {
            cur.depth++;
            continue;
          }
        }
        value = side_pot_payoff(
            N, up, cur.folded, [&](int q) { return (int)cur.inv[q]; }, [&](int q) { return rank[q]; });
        n_term++;
        break;
      }
      const int player = (int)(cur.q & 0xF);
      const int to_call = cur.cb - (int)cur.bet[player];
      const uint32_t vm = valid_mask(G, cur.pot, cur.stack[player], to_call, cur.cb, cur.lfr, cur.raises);
      const uint32_t cw = ctx[player];
      uint32_t hb, bkt;
      if (G.sub_street) {  // exact combo; the river card once it is dealt
        hb = cw & 0xFFFF;
        bkt = (cur.street == 3 && G.sub_street == 2) ? (cw >> 16) : 0u;
      } else {
        hb = cw & 0xFF;
        bkt = cur.street ? ((cw >> (8 * cur.street)) & 0xFF) : 0u;
      }
      const unsigned long long key = info_key(G, player, hb, bkt, cur.street, cur.abits, cur.path);
      const long long slot = table_insert<W>(tv, key);
      float reg[kSlots];
      load_regrets(tv, slot, reg);
      n_visits++;
      if (player == up) {
        if (sp >= kMaxFrames || slot < 0) {
          if (sp >= kMaxFrames) atomicOr(tv.err, kErrStackOverflow);
          aborted = true;
          break;
        }
        EsFrame& F = fr.at(sp++);
        F.st = cur;
        node_strategy(reg, vm, F.strat);
        F.vh = 0.0f;
        F.slot = (uint32_t)slot;
        F.vm = (uint8_t)vm;
        F.player = (uint8_t)player;
        const int a0 = __ffs(vm) - 1;
        F.next_a = (uint8_t)a0;
        es_apply(G, cur, player, a0);
        cur.depth++;
        pushed = true;
        continue;
      }
      // sampled opponent: strategy sum, then one action
      const U4 d = philox(U4{t, uid, (uint32_t)cur.path, (uint32_t)(cur.path >> 32) | 0x80000000u},
                          G.seed_lo, G.seed_hi);
      const int s = sample_action(G, reg, vm, uniform01(d.x));
      if (slot >= 0) {
        if (touch_row(tv, (unsigned long long)slot, uid, vm)) {
          atomicAdd(row_cnt(tv, slot), (1ull << 32) | 1ull);
        } else {
          atomicAdd(row_cnt(tv, slot), 1ull << 32);
          float strat[kSlots];
          node_strategy(reg, vm, strat);
          long long dw[kSlots];
#pragma unroll
          for (int a = 0; a < kSlots; ++a) dw[a] = fix_s(strat[a]);
          add_direct(tv, slot, vm, nullptr, dw);
        }
      }
      es_apply(G, cur, player, s);
      cur.depth++;
    }
    (void)pushed;
    if (aborted) break;
    // ---- return `value` to the frames
    bool resumed = false;
    while (sp > 0) {
      EsFrame& F = fr.at(sp - 1);
      const int a = F.next_a;
      atomicAdd(row_da(tv, F.slot) + a, (unsigned long long)fix_r(value, rscale));
      F.vh = __fadd_rn(F.vh, __fmul_rn(F.strat[a], value));
      const uint32_t rest = (uint32_t)F.vm & ~((2u << a) - 1u);
      if (rest) {
        const int nx = __ffs(rest) - 1;
        F.next_a = (uint8_t)nx;
        cur = F.st;
        es_apply(G, cur, F.player, nx);
        cur.depth++;
        resumed = true;
        break;
      }
      // node complete
      const float vh = F.vh;
      const long long fv = fix_r(vh, rscale);
      atomicAdd(row_cnt(tv, F.slot), 1ull << 32);
      if (touch_row(tv, F.slot, uid, F.vm)) {
        atomicAdd(row_su(tv, F.slot), (unsigned long long)fv);
      } else {
        long long dr[kSlots];
#pragma unroll
        for (int b = 0; b < kSlots; ++b) dr[b] = -fv;
        add_direct(tv, F.slot, F.vm, dr, nullptr);
      }
      n_updates++;
      value = vh;
      sp--;
    }
    if (!resumed) break;
  }
  cnt.visits += n_visits;
  cnt.updates += n_updates;
  cnt.terminals += n_term;
}

template <int BLOCK, int K, int W>
__global__ void __launch_bounds__(BLOCK)
k_traverse_es(const GameParams G, const TableView tv, const DealRec* __restrict__ deals, const Sched* __restrict__ sched,
              int batch, float rscale, Counters* __restrict__ counters) {
  extern __shared__ EsFrame s_frames[];  // [K][BLOCK]
  const uint32_t t = blockIdx.x * BLOCK + threadIdx.x;
  if (t >= (uint32_t)batch) return;
  const int up = sched->player;
  const uint32_t uid = update_id(sched, G.N);
  FrameStack<K> fr;
  fr.smem = s_frames + threadIdx.x;
  fr.stride = BLOCK;
  EsCounts c{0, 0, 0};
  es_walk<W>(G, tv, deals[t], t, uid, up, rscale, fr, c);
  warp_add_counters(counters, 1u, c.visits, c.updates, c.terminals, (unsigned)G.N);
}

inline void launch_traverse_es(const GameParams& G, const TableView& tv, const DealRec* deals, const Sched* sched,
                               int batch, float rscale, Counters* counters, cudaStream_t stream) {
  constexpr int B = 128;
  const int grid = (batch + B - 1) / B;
  static bool carveout_set = false;  // the walk keeps no shared memory: all of it to L1
  if (!carveout_set) {
    cudaFuncSetAttribute(k_traverse_es<B, 0, 1>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    carveout_set = true;
  }
  k_traverse_es<B, 0, 1><<<grid, B, 0, stream>>>(G, tv, deals, sched, batch, rscale, counters);
}

}  // namespace mccfr
