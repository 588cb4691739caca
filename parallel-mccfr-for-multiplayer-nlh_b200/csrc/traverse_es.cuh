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
  // chips put in this street and in the hand; a player's stack is
  // stack_base(G) - inv (es_stack)
  uint16_t bet[kMaxPlayers], inv[kMaxPlayers];
  int pot;
  int cb, lfr;
  uint32_t q;        // action queue, 4-bit entries
  uint32_t abits;
  uint32_t aux;      // traversal index (the level-synchronous form keeps states apart from their lanes)
  uint64_t path;
  uint8_t folded, allin, street, raises, nq, depth, pad0, pad1;
};
static_assert(sizeof(EsState) == 64, "a betting state is one 64-byte record");

// Chips behind of `player`: everyone starts with G.stack behind and, in a
// subgame, an equal share of the dead pot already invested.
__device__ __forceinline__ int es_stack(const GameParams& G, const EsState& s, int player) {
  return G.stack_base - pget(s.inv, player);
}

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
  const int pstack = es_stack(G, s, player), pbet = pget(s.bet, player);
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
  pset(s.bet, player, nbet);
  pset(s.inv, player, pget(s.inv, player) + chips);
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
      const int p = seat_after(player, i, G.N);
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

// One external-sampling traversal in progress on one lane: the betting state,
// the frame-stack depth, and the value being handed back up the frames.
struct EsLane {
  EsState cur;
  const DealRec* deal;
  uint32_t t;
  int dealer;
  int sp;
  float value;
  bool ret;  // returning `value` to the frames
};

// Root state of traversal t (deal `D`): blinds and the preflop queue, or a
// subgame's start (cfr_gpu.cu:954-981).
__device__ __forceinline__ void es_begin(const GameParams& G, const DealRec* D, uint32_t t, EsLane& L) {
  const int N = G.N;
  const int dealer = D->dealer;
  L.deal = D;
  L.t = t;
  L.dealer = dealer;
  L.sp = 0;
  L.value = 0.0f;
  L.ret = false;
  L.cur.aux = t;
  if (G.sub_street) {
    // subgame: the dead pot split equally, everyone with the same stack, first
    // to act after the dealer (the last seat)
    for (int p = 0; p < kMaxPlayers; ++p) {
      L.cur.bet[p] = 0;
      L.cur.inv[p] = (uint16_t)((p < N) ? G.sub_pot / N : 0);
    }
    L.cur.pot = G.sub_pot;
    L.cur.cb = 0;
    L.cur.lfr = G.bb;
    L.cur.folded = 0;
    L.cur.allin = 0;
    L.cur.street = (uint8_t)G.sub_street;
    L.cur.raises = 0;
    L.cur.abits = 0;
    L.cur.path = kPathSeed;
    L.cur.depth = 0;
    L.cur.q = 0;
    L.cur.nq = 0;
    for (int i = 1; i <= N; ++i) L.cur.q |= (uint32_t)seat_after(dealer, i, N) << (4 * L.cur.nq++);
  } else {
    for (int p = 0; p < kMaxPlayers; ++p) {
      L.cur.bet[p] = 0;
      L.cur.inv[p] = 0;
    }
    const int sbp = (N == 2) ? dealer : seat_after(dealer, 1, N);
    const int bbp = (N == 2) ? seat_after(dealer, 1, N) : seat_after(seat_after(dealer, 1, N), 1, N);
    const int sba = min(G.sb, G.stack), bba = min(G.bb, G.stack);
    pset(L.cur.bet, sbp, sba);
    pset(L.cur.inv, sbp, sba);
    pset(L.cur.bet, bbp, bba);
    pset(L.cur.inv, bbp, bba);
    L.cur.pot = sba + bba;
    L.cur.cb = bba;
    L.cur.lfr = G.bb;
    L.cur.folded = 0;
    L.cur.allin = 0;
    if (G.stack - sba == 0) L.cur.allin |= (uint8_t)(1u << sbp);
    if (G.stack - bba == 0) L.cur.allin |= (uint8_t)(1u << bbp);
    L.cur.street = 0;
    L.cur.raises = 0;
    L.cur.abits = 0;
    L.cur.path = kPathSeed;
    L.cur.depth = 0;
    L.cur.q = 0;
    L.cur.nq = 0;
    for (int i = 0; i < N; ++i) {
      const int p = seat_after(seat_after(bbp, 1, N), i, N);
      if (!((L.cur.allin >> p) & 1)) L.cur.q |= (uint32_t)p << (4 * L.cur.nq++);
    }
  }

}

// Kind of a traversal's next event, without doing it: 0 opponent visit, 1
// updating-player visit, 2 return to a frame, 3 showdown, 4 a cheap step
// (depth cut, fold terminal or street change).
__device__ __forceinline__ int es_peek(const GameParams& G, const EsLane& L, int up) {
  if (L.ret) return 2;
  const EsState& cur = L.cur;
  if (cur.depth >= G.max_depth) return 4;
  const uint32_t live = ((1u << G.N) - 1) & ~(uint32_t)cur.folded;
  if (__popc(live) == 1) return 4;
  if (cur.nq == 0) return cur.street < 3 ? 4 : 3;
  return (int)(cur.q & 0xF) == up ? 1 : 0;
}

// One event of a traversal: a descend step (one decision node, a street change
// or a terminal) or a return step (one child value handed to the top frame).
// Returns 0 while the traversal goes on, 1 when it is complete, 2 when it
// stopped on a full table or frame stack (the error flag is set).  The updating
// player's subtree is walked depth-first, opponents sampled.
template <int W, class Frames>
__device__ __forceinline__ int es_step(const GameParams& G, const TableView& tv, uint32_t uid, int up, float rscale,
                                       Frames& fr, EsLane& L, EsCounts& cnt) {
  const int N = G.N;
  const uint32_t all_players = (1u << N) - 1;
  EsState& cur = L.cur;
  const uint32_t t = L.t;
  // the action to apply: every branch that moves to a child ends at one
  // es_apply below, so lanes of a warp in different branches apply together
  int ap = 0, aa = 0;
  if (!L.ret) {
    if (cur.depth >= G.max_depth) {
      L.value = 0.0f;
      cnt.terminals++;
      L.ret = true;
      return 0;
    }
    const uint32_t live = all_players & ~(uint32_t)cur.folded;
    if (__popc(live) == 1) {
      const int winner = __ffs(live) - 1;
      const int inv_up = pget(cur.inv, up);
      L.value = (winner == up) ? (float)(cur.pot - inv_up) : (float)(-inv_up);
      cnt.terminals++;
      L.ret = true;
      return 0;
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
          const int p = seat_after(L.dealer, i, N);
          if (!((cur.folded >> p) & 1) && !((cur.allin >> p) & 1)) cur.q |= (uint32_t)p << (4 * cur.nq++);
        }
        if (cur.nq > 0) {
          cur.depth++;
          return 0;
        }
      }
      const DealRec* D = L.deal;
      L.value = side_pot_payoff(
          N, up, cur.folded, [&](int q) { return pget(cur.inv, q); }, [&](int q) { return (uint32_t)__ldg(D->rank + q); });
      cnt.terminals++;
      L.ret = true;
      return 0;
    }
    const int player = (int)(cur.q & 0xF);
    const int to_call = cur.cb - pget(cur.bet, player);
    const uint32_t vm = valid_mask(G, cur.pot, es_stack(G, cur, player), to_call, cur.cb, cur.lfr, cur.raises);
    const uint32_t cw = __ldg(L.deal->ctx + player);
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
    cnt.visits++;
    if (player == up) {
      if (L.sp >= kMaxFrames || slot < 0) {
        if (L.sp >= kMaxFrames) atomicOr(tv.err, kErrStackOverflow);
        return 2;
      }
      EsFrame& F = fr.at(L.sp++);
      mark_deltas(tv, (unsigned long long)slot);
      F.st = cur;
      node_strategy(reg, vm, F.strat);
      F.vh = 0.0f;
      F.slot = (uint32_t)slot;
      F.vm = (uint8_t)vm;
      F.player = (uint8_t)player;
      const int a0 = __ffs(vm) - 1;
      F.next_a = (uint8_t)a0;
      ap = player;
      aa = a0;
    } else {
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
      ap = player;
      aa = s;
    }
  } else {
    // ---- return step: `value` to the top frame
    if (L.sp == 0) return 1;
    EsFrame& F = fr.at(L.sp - 1);
    const int a = F.next_a;
    const float value = L.value;
    atomicAdd(row_da(tv, F.slot) + a, (unsigned long long)fix_r(value, rscale));
    F.vh = __fadd_rn(F.vh, __fmul_rn(F.strat[a], value));
    const uint32_t rest = (uint32_t)F.vm & ~((2u << a) - 1u);
    if (!rest) {  // node complete
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
      cnt.updates++;
      L.value = vh;
      L.sp--;
      return 0;
    }
    const int nx = __ffs(rest) - 1;
    F.next_a = (uint8_t)nx;
    cur = F.st;
    ap = F.player;
    aa = nx;
    L.ret = false;
  }
  es_apply(G, cur, ap, aa);
  cur.depth++;
  return 0;
}

// Persistent traversal kernel: every lane takes its next traversal from the
// device work counter as soon as its current one is complete (lanes that need
// work together share one atomic), inside the same one-event-per-iteration
// loop.  Tree sizes are heavy-tailed, so with one traversal per thread a warp
// would run as long as its largest tree while the other lanes idle.
template <int BLOCK, int K, int W>
__global__ void __launch_bounds__(BLOCK)
k_traverse_es(const GameParams G, const TableView tv, const DealRec* __restrict__ deals, const Sched* __restrict__ sched,
              int batch, float rscale, Counters* __restrict__ counters, unsigned* __restrict__ work) {
  extern __shared__ EsFrame s_frames[];  // [K][BLOCK]
  const int up = sched->player;
  const uint32_t uid = update_id(sched, G.N);
  FrameStack<K> fr;
  fr.smem = s_frames + threadIdx.x;
  fr.stride = BLOCK;
  EsCounts c{0, 0, 0};
  unsigned trav = 0;
  const int lane = threadIdx.x & 31;
  EsLane L;
  bool have = false, more = true;
  constexpr int kMaxWait = 4;
  int waited = 0;
  // The whole warp stays in the loop until every lane is out of work, and
  // reconverges before each event.
  for (;;) {
    __syncwarp();
    const bool need = !have && more;
    const unsigned needm = __ballot_sync(0xFFFFFFFFu, need);
    if (needm) {
      const int leader = __ffs(needm) - 1;
      unsigned base = 0;
      if (lane == leader) base = atomicAdd(work, (unsigned)__popc(needm));
      base = __shfl_sync(0xFFFFFFFFu, base, leader);
      if (need) {
        const uint32_t t = base + (uint32_t)__popc(needm & ((1u << lane) - 1u));
        if (t < (uint32_t)batch) {
          es_begin(G, deals + t, t, L);
          have = true;
          trav++;
        } else {
          more = false;
        }
      }
    }
    if (!__any_sync(0xFFFFFFFFu, have)) break;
    // Event-kind scheduling: of the expensive kinds, the warp runs the one most
    // lanes wait for (cheap steps run for everyone), so more lanes share each
    // issued instruction; a lane that has waited kMaxWait iterations forces its
    // kind.  Each lane's own sequence of events is unchanged.
    const int ty = have ? es_peek(G, L, up) : -1;
    int pick = 0, best = -1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int n = __popc(__ballot_sync(0xFFFFFFFFu, ty == k));
      if (n > best) {
        best = n;
        pick = k;
      }
    }
    const unsigned forced = __ballot_sync(0xFFFFFFFFu, have && ty < 4 && waited >= kMaxWait);
    if (forced) pick = __shfl_sync(0xFFFFFFFFu, ty, __ffs(forced) - 1);
    if (have && (ty == pick || ty == 4)) {
      waited = 0;
      if (es_step<W>(G, tv, uid, up, rscale, fr, L, c)) have = false;
    } else if (have) {
      waited++;
    }
  }
  warp_add_counters(counters, trav, c.visits, c.updates, c.terminals, trav * (unsigned)G.N);
}

// `work` must be zero when the launch starts; the launch enqueues that reset.
// The two shallowest frames of each walk live in shared memory (measured best
// among 0-4 staged frames and probe widths 1-2 on both presets).
inline void launch_traverse_es(const GameParams& G, const TableView& tv, const DealRec* deals, const Sched* sched,
                               int batch, float rscale, Counters* counters, unsigned* work, cudaStream_t stream,
                               int device) {
  constexpr int B = 128, K = 2;
  constexpr size_t smem = (size_t)K * B * sizeof(EsFrame);
  // resident blocks (blocks per SM at this kernel's register and shared-memory
  // use, times the SMs) of each device, found on its first launch there
  constexpr int kDevices = 64;
  static int resident[kDevices] = {};
  const int d = (device >= 0 && device < kDevices) ? device : 0;
  if (!resident[d]) {
    cudaFuncSetAttribute(k_traverse_es<B, K, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0, sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_traverse_es<B, K, 1>, B, smem);
    resident[d] = std::max(1, per_sm) * std::max(1, sms);
  }
  const int resident_blocks = resident[d];
  const int grid = std::max(1, std::min(resident_blocks, (batch + B - 1) / B));
  cudaMemsetAsync(work, 0, sizeof(unsigned), stream);
  k_traverse_es<B, K, 1><<<grid, B, smem, stream>>>(G, tv, deals, sched, batch, rscale, counters, work);
}

}  // namespace mccfr
