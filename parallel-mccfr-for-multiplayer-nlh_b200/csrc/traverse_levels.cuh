// traverse_levels.cuh — level-synchronous external-sampling traversal.
//
// The same player-update as k_traverse_es (one depth-first walk per lane), with
// the work regrouped so that the lanes of a warp do the same kind of work.  A
// traversal's tree (cfr_gpu.cu:644-860 under external sampling) is cut at the
// updating player's decision nodes: a *seed* is the root of a traversal or a
// child of an updating-player node (the state after one of its legal actions),
// and level L holds the seeds that have L updating-player decisions above them.
//
//   expand(L)  one lane per seed of level L: the lane walks the seed's
//              opponents' nodes (each samples one action and adds its strategy
//              to the row's strategy sum, as in the depth-first walk), street
//              changes and terminals, until it reaches a terminal (the seed's
//              value; a showdown leaves a record for the showdown pass) or an
//              updating-player node.  That node gets a record (its state, row
//              slot, legal mask) and every legal action becomes a seed of level
//              L+1.  Warps take seeds 32 at a time from a per-level counter and
//              hand them to idle lanes as those finish, so a warp keeps its
//              lanes busy whatever the walks' lengths.
//   dfs        seeds that did not fit the buffers (see below) are walked depth
//              first by the frame-stack walk of k_traverse_es, from the seed.
//   showdown   the recorded showdowns' side-pot payoffs, one thread each, so
//              that the walk's loop never runs the side-pot arithmetic for a
//              few of its lanes.
//   back(L)    one thread per updating-player node of level L, deepest level
//              first: it regret-matches the node's row (its regrets are a
//              snapshot the update does not change), reads its children's values,
//              forms v_h = sum_a strat[a] * v[a] in slot order as the depth-first
//              walk does, adds fix(v[a]) - fix(v_h) to every legal action's
//              accumulator and hands v_h to its own seed.  The row is claimed for
//              the update by one atomic maximum on its tag, with no canonical
//              mask (the whole regret term goes to the accumulators), so no
//              thread waits on a compare-and-swap.
//
// Every sum that reaches the table is an integer (fixed point) and every draw
// is keyed by the node's action path, so the rows after an update are
// bit-identical to the depth-first walk's, whatever the order of the lanes.
//
// Buffers.  A level's updating-player nodes and child seeds are appended to
// two bump-allocated arrays (nodes: 64 B state + 16 B record; seeds: 8 B),
// both by one 64-bit add per warp step ((nodes << 32) | seeds).  A
// lane checks, when it picks a seed up, that the arrays still have room for
// the worst case of every lane that may hold a seed meanwhile (one node and
// num_actions seeds each); a seed that fails the check is marked and left to
// the dfs kernel, unwalked.  A showdown past the end of its record list is
// evaluated by the lane that reached it.  So no allocation can overflow, and
// any buffer size gives the same rows.
#pragma once
#include "game.cuh"
#include "table.cuh"
#include "traverse_ref.cuh"
#include "traverse_es.cuh"

namespace mccfr {

constexpr int kMaxLevels = 32;
constexpr uint32_t kSeedDeferred = 0x80000000u;  // walked by the dfs kernel
constexpr uint32_t kSeedInvalid = 0xFFFFFFFFu;   // child of a node that found no row (table full)

// Per-update counters of the level arrays (zeroed before every update), each on
// a 128-byte line of its own: every warp of a level's launch adds to them.
struct LevelCtl {
  // level L: (updating-player nodes reached from level L << 32) | seeds of
  // level L + 1, both bump-allocated by one 64-bit add
  unsigned long long alloc[kMaxLevels][16];
  uint32_t grab[kMaxLevels][32];    // expand work counters
  uint32_t deferred;                // seeds left to the dfs kernel
  uint32_t pad0[31];
  uint32_t show_count;              // showdown records appended by the expand passes
  uint32_t pad2[31];
  uint32_t dfs_grab;
  uint32_t pad1[31];
};
__host__ __device__ __forceinline__ uint32_t level_nodes(const LevelCtl& c, int L) {
  return (uint32_t)(c.alloc[L][0] >> 32);
}
// Seeds of level L >= 1 (level 0 holds the batch's roots).
__host__ __device__ __forceinline__ uint32_t level_seeds(const LevelCtl& c, int L) {
  return (uint32_t)c.alloc[L - 1][0];
}

// Seeds a warp takes from a level's work counter at a time (one atomic per
// chunk instead of one per refill), and the idle lanes a refill waits for.
constexpr uint32_t kGrabChunk = 32;
constexpr int kRefillMin = 8;

// A showdown reached by an expand pass, evaluated by the batched showdown pass:
// the seed whose value it is, the traversal, the folded players and the chips
// each player put in (two per word).
struct __align__(8) ShowRec {
  uint32_t seed, aux, folded, inv01, inv23, inv45;
};

struct LevelBufs {
  EsState* nodes;     // [node_cap] state at the node (aux = traversal index)
  uint4* meta;        // [node_cap] {row slot, own seed, first child seed, legal mask (0: none)}
  uint32_t* child;    // [seed_cap] (node << 3) | action; kSeedDeferred / kSeedInvalid marks
  float* value;       // [seed_cap] the seed's value for the updating player
  ShowRec* show;      // [show_cap] showdowns left to the batched pass
  LevelCtl* ctl;
  uint32_t node_cap, seed_cap, show_cap;
  int nlev;           // seed levels (the last one is left to the dfs kernel)
};

// First seed of level L and first node of level L, from the counts of the
// levels above (final by the time level L runs).
struct LevelBase {
  uint32_t seed, seed_next, node, count;
};
__device__ __forceinline__ LevelBase level_base(const LevelBufs& lb, int L, int batch) {
  LevelBase b;
  uint32_t s = 0, n = 0;
  for (int l = 0; l < L; ++l) {
    s += l == 0 ? (uint32_t)batch : level_seeds(*lb.ctl, l);
    n += level_nodes(*lb.ctl, l);
  }
  b.seed = s;
  b.count = L == 0 ? (uint32_t)batch : level_seeds(*lb.ctl, L);
  b.seed_next = s + b.count;
  b.node = n;
  return b;
}

enum { kLvGoOn = 0, kLvDone = 1, kLvUp = 2, kLvShow = 3 };

// Side-pot showdown payoff of the updating player (side_pot_payoff), kept out
// of line so that the loop the lanes share stays small in the instruction
// cache; the invested chips come packed two per word, by value.
__device__ __noinline__ float lv_showdown(int N, int up, uint32_t folded, uint32_t inv01, uint32_t inv23,
                                          uint32_t inv45, const DealRec* D) {
  const uint32_t w[3] = {inv01, inv23, inv45};
  return side_pot_payoff(
      N, up, folded, [&](int q) { return (int)((w[q >> 1] >> (16 * (q & 1))) & 0xFFFF); },
      [&](int q) { return (uint32_t)__ldg(D->rank + q); });
}

// A sampled opponent's visit whose mask is not the row's canonical one: its
// strategy weights go to the accumulators directly.
__device__ __forceinline__ void lv_off_canonical(const TableView& tv, unsigned long long slot, uint32_t vm,
                                                 const float* reg) {
  atomicAdd(row_cnt(tv, slot), 1ull << 32);
  float strat[kSlots];
  node_strategy(reg, vm, strat);
  long long dw[kSlots];
#pragma unroll
  for (int a = 0; a < kSlots; ++a) dw[a] = fix_s(strat[a]);
  add_direct(tv, slot, vm, nullptr, dw);
}

// An action waiting to be applied to a lane's state: the seed's own action
// (picked up from its parent) or an opponent's sampled one.  Applying it at the
// top of the next step, instead of where it was chosen, leaves one copy of the
// action code in the loop, run by all lanes that have an action together.
struct LvPending {
  int player;  // -1: none
  int action;
};

// One step of a seed's walk (the descend branch of es_step): the pending action,
// the cheap steps (depth cut, fold win, street change), then a showdown (its
// folded players and chips handed back in `sd` for the batched showdown pass)
// or at most one decision node.  An opponent's node is done here (its sampled
// action is left pending); at an updating-player node the walk stops with the
// node's mask and row slot (its regrets are read in back).
template <int W>
__device__ __forceinline__ int lv_step(const GameParams& G, const TableView& tv, uint32_t uid, int up, EsState& cur,
                                       const DealRec* D, LvPending& pend, float& value, uint32_t& vm_out,
                                       long long& slot_out, uint4& sd, EsCounts& cnt) {
  const int N = G.N;
  const uint32_t all_players = (1u << N) - 1;
  if (pend.player >= 0) {
    es_apply(G, cur, pend.player, pend.action);
    cur.depth++;
    pend.player = -1;
  }
  for (int guard = 0; guard < 4; ++guard) {
    if (cur.depth >= G.max_depth) {
      value = 0.0f;
      cnt.terminals++;
      return kLvDone;
    }
    const uint32_t live = all_players & ~(uint32_t)cur.folded;
    if (__popc(live) == 1) {
      const int winner = __ffs(live) - 1;
      const int inv_up = pget(cur.inv, up);
      value = (winner == up) ? (float)(cur.pot - inv_up) : (float)(-inv_up);
      cnt.terminals++;
      return kLvDone;
    }
    if (cur.nq != 0) break;
    if (cur.street < 3) {
      cur.street++;
      for (int p = 0; p < kMaxPlayers; ++p) cur.bet[p] = 0;
      cur.cb = 0;
      cur.lfr = G.bb;
      cur.raises = 0;
      cur.q = 0;
      cur.nq = 0;
      for (int i = 1; i <= N; ++i) {
        const int p = seat_after(D->dealer, i, N);
        if (!((cur.folded >> p) & 1) && !((cur.allin >> p) & 1)) cur.q |= (uint32_t)p << (4 * cur.nq++);
      }
      if (cur.nq > 0) {
        cur.depth++;
        continue;
      }
    }
    sd = make_uint4((uint32_t)cur.folded, (uint32_t)cur.inv[0] | ((uint32_t)cur.inv[1] << 16),
                    (uint32_t)cur.inv[2] | ((uint32_t)cur.inv[3] << 16),
                    (uint32_t)cur.inv[4] | ((uint32_t)cur.inv[5] << 16));
    cnt.terminals++;
    return kLvShow;
  }
  const int player = (int)(cur.q & 0xF);
  const int to_call = cur.cb - pget(cur.bet, player);
  const uint32_t vm = valid_mask(G, cur.pot, es_stack(G, cur, player), to_call, cur.cb, cur.lfr, cur.raises);
  const uint32_t cw = __ldg(D->ctx + player);
  uint32_t hb, bkt;
  if (G.sub_street) {  // exact combo; the river card once it is dealt
    hb = cw & 0xFFFF;
    bkt = (cur.street == 3 && G.sub_street == 2) ? (cw >> 16) : 0u;
  } else {
    hb = cw & 0xFF;
    bkt = cur.street ? ((cw >> (8 * cur.street)) & 0xFF) : 0u;
  }
  const unsigned long long key = info_key(G, player, hb, bkt, cur.street, cur.abits, cur.path);
  cnt.visits++;
  if (tv.direct) {
    // key k owns row k-1: the updating player's row is read (and its key
    // stored) by the back pass; an opponent's key, tag and regrets are loaded
    // together, and its draw is computed while they are in flight
    const unsigned long long rs = key - 1;
    if (player == up) {
      vm_out = vm;
      slot_out = (long long)rs;
      return kLvUp;
    }
    const ulonglong2 kt = __ldcg(reinterpret_cast<const ulonglong2*>(row_ptr(tv, rs)));
    const float4* rp = row_reg(tv, rs);
    const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
    const U4 d = philox(U4{cur.aux, uid, (uint32_t)cur.path, (uint32_t)(cur.path >> 32) | 0x80000000u},
                        G.seed_lo, G.seed_hi);
    if (kt.x != key) __stcg(row_key(tv, rs), key);
    const float reg[kSlots] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
    const int s = sample_action(G, reg, vm, uniform01(d.x));
    if (touch_row_from(tv, rs, uid, vm, kt.y)) {
      atomicAdd(row_cnt(tv, rs), (1ull << 32) | 1ull);
    } else {
      lv_off_canonical(tv, rs, vm, reg);
    }
    pend.player = player;
    pend.action = s;
    return kLvGoOn;
  }
  const long long slot = table_insert<W>(tv, key);
  if (player == up) {
    vm_out = vm;
    slot_out = slot;
    return kLvUp;
  }
  // sampled opponent: strategy sum, then one action (es_step's opponent branch)
  float reg[kSlots];
  load_regrets(tv, slot, reg);
  const U4 d = philox(U4{cur.aux, uid, (uint32_t)cur.path, (uint32_t)(cur.path >> 32) | 0x80000000u}, G.seed_lo,
                      G.seed_hi);
  const int s = sample_action(G, reg, vm, uniform01(d.x));
  if (slot >= 0) {
    if (touch_row(tv, (unsigned long long)slot, uid, vm)) {
      atomicAdd(row_cnt(tv, slot), (1ull << 32) | 1ull);
    } else {
      lv_off_canonical(tv, (unsigned long long)slot, vm, reg);
    }
  }
  pend.player = player;
  pend.action = s;
  return kLvGoOn;
}

// Start of a seed of a level below the root: the parent node's state, with the
// seed's action left pending.
__device__ __forceinline__ void lv_child_start(const LevelBufs& lb, const DealRec* deals, uint32_t w, int up,
                                               EsState& cur, const DealRec*& D, LvPending& pend) {
  const uint32_t node = (w & ~kSeedDeferred) >> 3;
  const uint4* src = reinterpret_cast<const uint4*>(lb.nodes + node);
  uint4* dst = reinterpret_cast<uint4*>(&cur);
#pragma unroll
  for (int i = 0; i < 4; ++i) dst[i] = __ldcg(src + i);
  D = deals + cur.aux;
  pend.player = up;
  pend.action = (int)(w & 7);
}

// Start state of a seed below the root, its action applied (the depth-first
// walk of deferred seeds).
__device__ __forceinline__ void lv_child_state(const GameParams& G, const LevelBufs& lb, const DealRec* deals,
                                               uint32_t w, int up, EsState& cur, const DealRec*& D) {
  LvPending pend;
  lv_child_start(lb, deals, w, up, cur, D, pend);
  es_apply(G, cur, pend.player, pend.action);
  cur.depth++;
}

__device__ __forceinline__ void lv_root_state(const GameParams& G, const DealRec* deals, uint32_t t, EsState& cur,
                                              const DealRec*& D) {
  EsLane tmp;
  es_begin(G, deals + t, t, tmp);
  cur = tmp.cur;
  D = deals + t;
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *(volatile const uint32_t*)p; }

// ROOT: level 0, whose seeds are the traversals' roots (built from the deals);
// deeper levels load their parent's state instead.
// Eight blocks of 128 threads per SM (64 registers): the walk waits on
// dependent table reads, so resident warps matter more than a few spills.
template <int BLOCK, int W, bool ROOT>
__global__ void __launch_bounds__(BLOCK, 8)
k_level_expand(const GameParams G, const TableView tv, const DealRec* __restrict__ deals,
               const Sched* __restrict__ sched, int batch, const LevelBufs lb, int L,
               Counters* __restrict__ counters) {
  __shared__ LevelBase s_base;
  if (threadIdx.x == 0) s_base = level_base(lb, L, batch);
  __syncthreads();
  const LevelBase B = s_base;
  if (B.count == 0) return;
  const int up = sched->player;
  const uint32_t uid = update_id(sched, G.N);
  const bool last = L + 1 >= lb.nlev;
  const int lane = threadIdx.x & 31;
  // room check at pick-up: every lane of the launch may hold a seed meanwhile
  const uint32_t holders = min((uint32_t)(gridDim.x * BLOCK), B.count);
  const unsigned long long need_nodes = (unsigned long long)B.node + holders;
  const unsigned long long need_seeds = (unsigned long long)B.seed_next + (unsigned long long)holders * G.num_actions;
  unsigned long long* alloc = &lb.ctl->alloc[L][0];
  uint32_t* grab = &lb.ctl->grab[L][0];
  EsCounts c{0, 0, 0};
  unsigned trav = 0, deferred = 0;
  EsState cur;
  const DealRec* D = deals;
  LvPending pend{-1, 0};
  uint32_t seed = 0;
  bool have = false, more = true;
  // The warp's seeds not yet handed out, [pool, pool_end): one chunk of
  // kGrabChunk seeds of the level, whose child words were loaded (one per lane,
  // `pw`) when the chunk was taken.  Idle lanes are refilled together, once at
  // least kRefillMin of them wait or none has work: a refill stalls the warp on
  // the new seeds' parent records, so fewer refills stall it less often.
  uint32_t pool = 0, pool_end = 0, pw = 0;
  for (;;) {
    __syncwarp();
    const bool need = !have && more;
    const unsigned needm = __ballot_sync(0xFFFFFFFFu, need);
    const unsigned busym = __ballot_sync(0xFFFFFFFFu, have);
    if (needm && (__popc(needm) >= kRefillMin || !busym)) {
      uint32_t avail = pool_end - pool;
      if (avail == 0) {
        uint32_t chunk = 0;
        if (lane == 0) chunk = atomicAdd(grab, kGrabChunk);
        chunk = __shfl_sync(0xFFFFFFFFu, chunk, 0);
        pool = chunk;
        pool_end = chunk + kGrabChunk;
        avail = kGrabChunk;
        if (!ROOT) pw = chunk + (uint32_t)lane < B.count ? __ldcg(lb.child + B.seed + chunk + lane) : kSeedInvalid;
      }
      const uint32_t k = (uint32_t)__popc(needm);
      const uint32_t take = min(k, avail);
      const uint32_t rank = (uint32_t)__popc(needm & ((1u << lane) - 1u));
      const uint32_t i = pool + rank;
      const uint32_t wl = ROOT ? 0u : __shfl_sync(0xFFFFFFFFu, pw, (int)((i - (pool_end - kGrabChunk)) & 31u));
      if (need && rank < take) {
        if (i >= B.count) {
          more = false;
        } else {
          seed = B.seed + i;
          const uint32_t w = wl;
          bool ok = w != kSeedInvalid && !last;
          if (ok) {
            const unsigned long long a = *(volatile const unsigned long long*)alloc;
            ok = need_nodes + (a >> 32) <= lb.node_cap && need_seeds + (uint32_t)a <= lb.seed_cap;
          }
          if (w == kSeedInvalid) {
            // child of a node that found no row: nothing to walk
          } else if (!ok) {
            lb.child[seed] = w | kSeedDeferred;
            deferred++;
          } else {
            if (ROOT) {
              lb.child[seed] = 0u;
              lv_root_state(G, deals, seed, cur, D);
              trav++;
            } else {
              lv_child_start(lb, deals, w, up, cur, D, pend);
            }
            have = true;
          }
        }
      }
      pool += take;
    }
    if (!__any_sync(0xFFFFFFFFu, have || more)) break;
    int r = -1;
    uint32_t vm = 0;
    long long slot = -1;
    float v = 0.0f;
    uint4 sd = make_uint4(0u, 0u, 0u, 0u);
    if (have) {
      r = lv_step<W>(G, tv, uid, up, cur, D, pend, v, vm, slot, sd, c);
      if (r == kLvDone) {
        lb.value[seed] = v;
        have = false;
      }
    }
    // showdowns of this step: one record each for the batched showdown pass
    // (computed here when the record list is full)
    const bool issd = have && r == kLvShow;
    const unsigned sdm = __ballot_sync(0xFFFFFFFFu, issd);
    if (sdm) {
      uint32_t sb = 0;
      if (lane == 0) sb = atomicAdd(&lb.ctl->show_count, (unsigned)__popc(sdm));
      sb = __shfl_sync(0xFFFFFFFFu, sb, 0);
      if (issd) {
        const uint32_t j = sb + (uint32_t)__popc(sdm & ((1u << lane) - 1u));
        if (j < lb.show_cap) {
          lb.show[j] = ShowRec{seed, cur.aux, sd.x, sd.y, sd.z, sd.w};
        } else {
          lb.value[seed] = lv_showdown(G.N, up, sd.x, sd.y, sd.z, sd.w, D);
        }
        have = false;
      }
    }
    // updating-player nodes of this step: one node record each and one seed per
    // legal action, allocated for the warp by one lane
    const bool isup = have && r == kLvUp;
    const unsigned upm = __ballot_sync(0xFFFFFFFFu, isup);
    if (upm) {
      const int k = isup ? __popc(vm) : 0;
      int incl = k;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      const int total = __shfl_sync(0xFFFFFFFFu, incl, 31);
      unsigned long long j2 = 0;
      if (lane == 0) j2 = atomicAdd(alloc, ((unsigned long long)__popc(upm) << 32) | (unsigned)total);
      j2 = __shfl_sync(0xFFFFFFFFu, j2, 0);
      const uint32_t jn = (uint32_t)(j2 >> 32), jc = (uint32_t)j2;
      if (isup) {
        const uint32_t j = B.node + jn + (uint32_t)__popc(upm & ((1u << lane) - 1u));
        const uint32_t cb = B.seed_next + jc + (uint32_t)(incl - k);
        if (slot < 0) {  // table full (flag raised): the node has no row to update
          lb.meta[j] = make_uint4(0u, seed, cb, 0u);
          for (int q = 0; q < k; ++q) lb.child[cb + q] = kSeedInvalid;
          lb.value[seed] = 0.0f;
        } else {
          const uint4* src = reinterpret_cast<const uint4*>(&cur);
          uint4* dst = reinterpret_cast<uint4*>(lb.nodes + j);
#pragma unroll
          for (int q = 0; q < 4; ++q) dst[q] = src[q];
          lb.meta[j] = make_uint4((uint32_t)slot, seed, cb, vm);
          uint32_t o = cb;
#pragma unroll
          for (int a = 0; a < kSlots; ++a)
            if ((vm >> a) & 1) lb.child[o++] = (j << 3) | (uint32_t)a;
        }
        have = false;
      }
    }
  }
  if (deferred) atomicAdd(&lb.ctl->deferred, deferred);
  warp_add_counters(counters, trav, c.visits, 0u, c.terminals, trav * (unsigned)G.N);
}

// Seeds marked for the depth-first walk, from their start states: persistent
// lanes scan the seed indices through a work counter (most indices are not
// marked) and walk each marked seed's subtree with es_step.
template <int BLOCK, int K, int W>
__global__ void __launch_bounds__(BLOCK)
k_level_dfs(const GameParams G, const TableView tv, const DealRec* __restrict__ deals,
            const Sched* __restrict__ sched, int batch, float rscale, const LevelBufs lb,
            Counters* __restrict__ counters) {
  extern __shared__ EsFrame s_frames[];  // [K][BLOCK]
  if (ld_volatile(&lb.ctl->deferred) == 0) return;
  __shared__ uint32_t s_total;
  if (threadIdx.x == 0) {
    const LevelBase b = level_base(lb, lb.nlev - 1, batch);
    s_total = b.seed_next;
  }
  __syncthreads();
  const uint32_t total = s_total;
  const int up = sched->player;
  const uint32_t uid = update_id(sched, G.N);
  FrameStack<K> fr;
  fr.smem = s_frames + threadIdx.x;
  fr.stride = BLOCK;
  EsCounts c{0, 0, 0};
  unsigned trav = 0;
  const int lane = threadIdx.x & 31;
  EsLane Ln;
  uint32_t seed = 0;
  bool have = false, more = true;
  for (;;) {
    __syncwarp();
    const bool need = !have && more;
    const unsigned needm = __ballot_sync(0xFFFFFFFFu, need);
    if (needm) {
      const int leader = __ffs(needm) - 1;
      unsigned base = 0;
      if (lane == leader) base = atomicAdd(&lb.ctl->dfs_grab, (unsigned)__popc(needm));
      base = __shfl_sync(0xFFFFFFFFu, base, leader);
      if (need) {
        const uint32_t i = base + (uint32_t)__popc(needm & ((1u << lane) - 1u));
        if (i >= total) {
          more = false;
        } else {
          const uint32_t w = __ldcg(lb.child + i);
          if (w != kSeedInvalid && (w & kSeedDeferred)) {
            seed = i;
            const DealRec* D = deals;
            EsState st;
            if (seed < (uint32_t)batch) {
              lv_root_state(G, deals, seed, st, D);
              trav++;
            } else {
              lv_child_state(G, lb, deals, w, up, st, D);
            }
            Ln.cur = st;
            Ln.deal = D;
            Ln.t = st.aux;
            Ln.dealer = D->dealer;
            Ln.sp = 0;
            Ln.value = 0.0f;
            Ln.ret = false;
            have = true;
          }
        }
      }
    }
    if (!__any_sync(0xFFFFFFFFu, have || more)) break;
    if (have) {
      const int r = es_step<W>(G, tv, uid, up, rscale, fr, Ln, c);
      if (r) {
        lb.value[seed] = r == 1 ? Ln.value : 0.0f;
        have = false;
      }
    }
  }
  warp_add_counters(counters, trav, c.visits, c.updates, c.terminals, trav * (unsigned)G.N);
}

// The showdowns the expand passes recorded, one thread each: all lanes of a
// warp run the same side-pot arithmetic (side_pot_payoff) on their own record.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_level_showdown(const GameParams G, const DealRec* __restrict__ deals, const Sched* __restrict__ sched,
                 const LevelBufs lb) {
  const uint32_t n = min(ld_volatile(&lb.ctl->show_count), lb.show_cap);
  const int up = sched->player;
  for (uint32_t i = blockIdx.x * BLOCK + threadIdx.x; i < n; i += gridDim.x * BLOCK) {
    const ShowRec r = lb.show[i];
    lb.value[r.seed] = lv_showdown(G.N, up, r.folded, r.inv01, r.inv23, r.inv45, deals + r.aux);
  }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_level_back(const GameParams G, const TableView tv, const Sched* __restrict__ sched, int batch, float rscale,
             const LevelBufs lb, int L, Counters* __restrict__ counters) {
  const uint32_t n = level_nodes(*lb.ctl, L);
  if (n == 0) return;
  __shared__ LevelBase s_base;
  if (threadIdx.x == 0) s_base = level_base(lb, L, batch);
  __syncthreads();
  const uint32_t nb = s_base.node;
  const uint32_t uid = update_id(sched, G.N);
  unsigned upd = 0;
  for (uint32_t i = blockIdx.x * BLOCK + threadIdx.x; i < n; i += gridDim.x * BLOCK) {
    const uint4 m = __ldcg(lb.meta + nb + i);
    const uint32_t vm = m.w;
    if (!vm) continue;
    const unsigned long long slot = m.x;
    // independent of each other: the claim, the row's regrets, the children's
    // values, and (direct map) the row's key, which the expand pass left to this pass
    if (tv.direct) {
      const unsigned long long k = __ldcg(row_key(tv, slot));
      if (k != slot + 1) __stcg(row_key(tv, slot), slot + 1);
    }
    claim_row(tv, slot, uid);
    float reg[kSlots], strat[kSlots], v[kSlots];
    load_regrets(tv, (long long)slot, reg);
    uint32_t o = m.z;
#pragma unroll
    for (int a = 0; a < kSlots; ++a) v[a] = ((vm >> a) & 1) ? __ldcg(lb.value + o++) : 0.0f;
    node_strategy(reg, vm, strat);
    float vh = 0.0f;
#pragma unroll
    for (int a = 0; a < kSlots; ++a)
      if ((vm >> a) & 1) vh = __fadd_rn(vh, __fmul_rn(strat[a], v[a]));
    const long long fv = fix_r(vh, rscale);
    mark_deltas(tv, slot);
#pragma unroll
    for (int a = 0; a < kSlots; ++a)
      if ((vm >> a) & 1) atomicAdd(row_da(tv, slot) + a, (unsigned long long)(fix_r(v[a], rscale) - fv));
    atomicAdd(row_cnt(tv, slot), 1ull << 32);
    upd++;
    lb.value[m.y] = vh;
  }
  warp_add_counters(counters, 0u, 0u, upd, 0u, 0u);
}

}  // namespace mccfr
