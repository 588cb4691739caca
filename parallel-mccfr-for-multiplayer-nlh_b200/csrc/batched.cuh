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

// Persistent external-sampling traversal over a phase's items.  Each lane takes
// its next `grab` consecutive items from `work` as soon as it is idle (lanes
// that become idle together share one atomic), so no lane waits for the rest of
// its warp.  Counters are summed per lane while it stays on one table.
template <int BLOCK, int K, int W>
__global__ void __launch_bounds__(BLOCK, 2048 / BLOCK / 2)
k_traverse_batched(const __grid_constant__ PhaseParams P, const DealRec* __restrict__ deals,
                   unsigned long long* __restrict__ work, int grab, int warp_sync) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EsFrame* s_frames = reinterpret_cast<EsFrame*>(smem_raw);
  const unsigned long long total = P.off[P.n];
  FrameStack<K> fr;
  fr.smem = s_frames + threadIdx.x;
  fr.stride = BLOCK;
  int cur_j = -1;
  unsigned long long c_trav = 0, c_vis = 0, c_upd = 0, c_term = 0;
  auto flush = [&]() {
    if (cur_j >= 0 && c_trav) {
      Counters* cn = P.T[cur_j].counters;
      atomicAdd(&cn->traversals, c_trav);
      atomicAdd(&cn->visits, c_vis);
      atomicAdd(&cn->updates, c_upd);
      atomicAdd(&cn->terminals, c_term);
      atomicAdd(&cn->evals, c_trav * (unsigned long long)P.T[cur_j].G.N);
    }
    c_trav = c_vis = c_upd = c_term = 0;
  };
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned long long base = 0, stride = 1;
    if (warp_sync) {
      // the whole warp takes 32*grab items and starts them together
      if (lane == 0) base = atomicAdd(work, 32ull * grab);
      base = __shfl_sync(0xFFFFFFFFu, base, 0) + lane;
      stride = 32;
      if (base - lane >= total) break;
    } else {
      // idle lanes that arrive together take consecutive chunks with one atomic
      const unsigned act = __activemask();
      const int leader = __ffs(act) - 1;
      const int rank = __popc(act & ((1u << lane) - 1));
      if (lane == leader) base = atomicAdd(work, (unsigned long long)__popc(act) * grab);
      base = __shfl_sync(act, base, leader) + (unsigned long long)rank * grab;
      if (base >= total) break;
    }
    for (int k = 0; k < grab; ++k) {
      const unsigned long long g = base + k * stride;
      if (g >= total) break;
      const int j = param_table_of(P, g);
      if (j != cur_j) {
        flush();
        cur_j = j;
      }
      const TableDesc& D = P.T[j];
      const uint32_t t = (uint32_t)(g - P.off[j]);
      const Sched* sc = D.sched;
      EsCounts c{0, 0, 0};
      es_walk<W>(D.G, D.tv, deals + g, t, update_id(sc, D.G.N), sc->player, D.rscale, fr, c);
      c_trav++;
      c_vis += c.visits;
      c_upd += c.updates;
      c_term += c.terminals;
    }
    if (warp_sync) __syncwarp();
  }
  flush();
}

}  // namespace mccfr
