// batched.cuh — many game tables in one persistent traversal kernel.
//
// The plain trainer launches one traversal kernel per (table, player-update),
// with one thread per traversal and blocks scheduled by the hardware.  The
// batched form runs the player-updates of many tables (different player counts,
// stacks, action sets and traversal counts) together:
//   * a phase p groups update (iteration, p) of every table with more than p
//     players; its traversals form one item range, split into per-table ranges
//     by a prefix-offset table;
//   * the persistent kernel (grid = resident blocks only) pulls chunks of items
//     from a device work counter, so warps that finish small trees take more
//     work instead of idling behind the phase's largest traversals;
//   * per-table game parameters are staged in shared memory; tables share one
//     rank table, so their gathers share L2;
//   * every table keeps its own schedule, accumulators and touched list, so the
//     result of each table is bit-identical to training it alone.
#pragma once
#include "traverse_es.cuh"
#include "traverse_ref.cuh"

namespace mccfr {

constexpr int kMaxBatchTables = 64;

// One table of a batch (device array).
struct TableDesc {
  GameParams G;
  TableView tv;
  const uint8_t* pre;
  const uint8_t* cdf;
  Sched* sched;
  Counters* counters;
  float rscale;
  double rinv;
  int batch;  // traversals per player-update
  int pad;
};

// The tables taking part in one phase and their item ranges.
struct PhaseDesc {
  int n;
  int table[kMaxBatchTables];
  unsigned long long off[kMaxBatchTables + 1];  // off[n] = total items
};

__device__ __forceinline__ int phase_table_of(const PhaseDesc& P, unsigned long long g) {
  int lo = 0, hi = P.n - 1;
  while (lo < hi) {  // last j with off[j] <= g
    const int mid = (lo + hi + 1) >> 1;
    if (P.off[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(128) k_deal_batched(const TableDesc* __restrict__ tables,
                                                      const PhaseDesc* __restrict__ phase,
                                                      const int32_t* __restrict__ T, DealRec* __restrict__ out) {
  __shared__ PhaseDesc P;
  for (int i = threadIdx.x; i < (int)(sizeof(PhaseDesc) / 4); i += blockDim.x)
    reinterpret_cast<uint32_t*>(&P)[i] = reinterpret_cast<const uint32_t*>(phase)[i];
  __syncthreads();
  const unsigned long long total = P.off[P.n];
  for (unsigned long long g = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; g < total;
       g += (unsigned long long)gridDim.x * blockDim.x) {
    const int j = phase_table_of(P, g);
    const TableDesc& D = tables[P.table[j]];
    const uint32_t t = (uint32_t)(g - P.off[j]);
    deal_one(D.G, T, D.pre, D.cdf, t, update_id(D.sched, D.G.N), out + g);
  }
}

// A phase's descriptors passed by value: they live in the kernel's parameter
// space and are read through the constant cache, like the plain kernel's game
// parameters (a warp mostly works on one table, so the reads are uniform).
struct PhaseParams {
  unsigned long long off[kMaxBatchTables + 1];
  int n;
  int pad;
  TableDesc T[kMaxBatchTables];  // the phase's tables, in phase order
};

__device__ __forceinline__ int param_table_of(const PhaseParams& P, unsigned long long g) {
  int lo = 0, hi = P.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (P.off[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Persistent external-sampling traversal over a phase's items, in the plain
// kernel's lockstep form: every lane handles one event of its current
// traversal per iteration and the warp reconverges before each event.  A lane
// that finishes a traversal takes its next item from its current run; lanes
// whose runs are used up refill together with one atomic on `work` (lanes x
// grab items, interleaved across the lanes when warp_sync is set, contiguous
// runs of `grab` otherwise).  Counters are summed per lane while it stays on
// one table.
template <int BLOCK, int K, int W>
__global__ void __launch_bounds__(BLOCK)
k_traverse_batched(const __grid_constant__ PhaseParams P, const DealRec* __restrict__ deals,
                   unsigned long long* __restrict__ work, int grab, int warp_sync) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EsFrame* s_frames = reinterpret_cast<EsFrame*>(smem_raw);
  const unsigned long long total = P.off[P.n];
  FrameStack<K> fr;
  fr.smem = s_frames + threadIdx.x;
  fr.stride = BLOCK;
  const int lane = threadIdx.x & 31;
  int cur_j = -1, up = 0;
  uint32_t uid = 0;
  unsigned long long c_trav = 0;
  EsCounts c{0, 0, 0};
  auto flush = [&]() {
    if (cur_j >= 0 && c_trav) {
      Counters* cn = P.T[cur_j].counters;
      atomicAdd(&cn->traversals, c_trav);
      atomicAdd(&cn->visits, (unsigned long long)c.visits);
      atomicAdd(&cn->updates, (unsigned long long)c.updates);
      atomicAdd(&cn->terminals, (unsigned long long)c.terminals);
      atomicAdd(&cn->evals, c_trav * (unsigned long long)P.T[cur_j].G.N);
    }
    c_trav = 0;
    c = EsCounts{0, 0, 0};
  };
  unsigned long long nxt = 0, stop = 0, step = 1;  // this lane's run: nxt, nxt + step, ... < stop
  bool have = false, more = true;
  EsLane L;
  for (;;) {
    __syncwarp();
    const bool need = !have && more;
    const bool refill = need && nxt >= stop;
    const unsigned rm = __ballot_sync(0xFFFFFFFFu, refill);
    if (rm) {
      const int k = __popc(rm);
      const int leader = __ffs(rm) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(work, (unsigned long long)k * grab);
      base = __shfl_sync(0xFFFFFFFFu, base, leader);
      if (refill) {
        const int r = __popc(rm & ((1u << lane) - 1u));
        if (warp_sync) {
          nxt = base + r;
          step = k;
          stop = base + (unsigned long long)k * grab;
        } else {
          nxt = base + (unsigned long long)r * grab;
          step = 1;
          stop = nxt + grab;
        }
        if (stop > total) stop = total;
        if (nxt >= total) more = false;
      }
    }
    if (need && more && nxt < stop) {
      const unsigned long long g = nxt;
      nxt += step;
      const int j = param_table_of(P, g);
      if (j != cur_j) {
        flush();
        cur_j = j;
        uid = update_id(P.T[j].sched, P.T[j].G.N);
        up = P.T[j].sched->player;
      }
      es_begin(P.T[j].G, deals + g, (uint32_t)(g - P.off[j]), L);
      have = true;
      c_trav++;
    }
    if (!__any_sync(0xFFFFFFFFu, have || more)) break;
    if (have) {
      const TableDesc& D = P.T[cur_j];
      if (es_step<W>(D.G, D.tv, uid, up, D.rscale, fr, L, c)) have = false;
    }
  }
  flush();
}

}  // namespace mccfr
