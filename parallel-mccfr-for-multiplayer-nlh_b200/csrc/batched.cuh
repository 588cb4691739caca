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

// Bytes of dynamic shared memory before the frame area: the phase descriptor
// and the descriptors of the phase's tables.
constexpr size_t kBatchedHeadBytes =
    ((sizeof(PhaseDesc) + 15) / 16) * 16 + ((kMaxBatchTables * sizeof(TableDesc) + 15) / 16) * 16;

// Persistent external-sampling traversal over a phase's items.  Each warp takes
// `grab` items per lane at a time from `work`.
template <int BLOCK, int K, int W>
__global__ void __launch_bounds__(BLOCK)
k_traverse_batched(const TableDesc* __restrict__ tables, const PhaseDesc* __restrict__ phase,
                   const DealRec* __restrict__ deals, unsigned long long* __restrict__ work, int grab) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PhaseDesc& P = *reinterpret_cast<PhaseDesc*>(smem_raw);
  TableDesc* s_tab = reinterpret_cast<TableDesc*>(smem_raw + ((sizeof(PhaseDesc) + 15) / 16) * 16);
  EsFrame* s_frames = reinterpret_cast<EsFrame*>(smem_raw + kBatchedHeadBytes);
  for (int i = threadIdx.x; i < (int)(sizeof(PhaseDesc) / 4); i += BLOCK)
    reinterpret_cast<uint32_t*>(&P)[i] = reinterpret_cast<const uint32_t*>(phase)[i];
  __syncthreads();
  // descriptors of this phase's tables, in phase order
  for (int i = threadIdx.x; i < P.n * (int)(sizeof(TableDesc) / 4); i += BLOCK) {
    const int j = i / (int)(sizeof(TableDesc) / 4), w = i % (int)(sizeof(TableDesc) / 4);
    reinterpret_cast<uint32_t*>(s_tab + j)[w] = reinterpret_cast<const uint32_t*>(tables + P.table[j])[w];
  }
  __syncthreads();
  const unsigned long long total = P.off[P.n];
  const int lane = threadIdx.x & 31;
  FrameStack<K> fr;
  fr.smem = s_frames + threadIdx.x;
  fr.stride = BLOCK;
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(work, 32ull * (unsigned long long)grab);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (base >= total) break;
    for (int k = 0; k < grab; ++k) {
      const unsigned long long g = base + (unsigned long long)k * 32 + lane;
      if (g >= total) break;
      const int j = phase_table_of(P, g);
      const TableDesc& D = s_tab[j];
      const uint32_t t = (uint32_t)(g - P.off[j]);
      const Sched* sc = D.sched;
      EsCounts c{0, 0, 0};
      es_walk<W>(D.G, D.tv, deals[g], t, update_id(sc, D.G.N), sc->player, D.rscale, fr, c);
      Counters* cn = D.counters;
      atomicAdd(&cn->traversals, 1ull);
      atomicAdd(&cn->visits, (unsigned long long)c.visits);
      atomicAdd(&cn->updates, (unsigned long long)c.updates);
      atomicAdd(&cn->terminals, (unsigned long long)c.terminals);
      atomicAdd(&cn->evals, (unsigned long long)D.G.N);
    }
    __syncwarp();
  }
}

}  // namespace mccfr
