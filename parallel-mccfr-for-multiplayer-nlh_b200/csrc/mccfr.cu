// mccfr.cu — kernels and C ABI of the B200 MCCFR trainer (see include/mccfr.h).
//
// Host side of the reference's GPUCFRTrainer (poker_cuda/src/cfr_gpu.cu:1064-1538)
// restructured for one device-resident table:
//   * the dense regret-matching and clamp sweeps of every player-update
//     (cfr_gpu.cu:318-351, 1018-1022) are replaced by computing the current
//     strategy in the traversal from the row it reads, plus an apply kernel that
//     visits only the rows the update touched;
//   * one iteration (N player-updates x [traverse, apply, advance]) is captured
//     once as a CUDA graph and replayed; the iteration and player are advanced on
//     the device, so replays need no host copies (cfr_gpu.cu:1303-1322 copies
//     two scalars per update);
//   * errors are returned as status codes, never exit() (cfr_gpu.cu:61-69).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../include/mccfr.h"
#include "game.cuh"
#include "handtable.h"
#include "table.cuh"
#include "traverse_ref.cuh"
#include "traverse_es.cuh"
#include "traverse_levels.cuh"
#include "showdown.cuh"
#include "batched.cuh"
#include "best_response.h"

namespace mccfr {
void build_preflop_lut(int mode, int buckets, uint8_t* lut);
void build_cdf_lut(const unsigned long long* counts, int buckets, uint8_t* lut);
}  // namespace mccfr

using namespace mccfr;

// ---------------------------------------------------------------------------
// Small kernels
// ---------------------------------------------------------------------------
namespace {

constexpr int kRefBlock = 128;

// Folds one player-update's accumulators into the rows it touched and zeroes
// them (the sparse equivalent of kernel_clamp_regrets, cfr_gpu.cu:1018-1022).
// Eight lanes per row, lane a owning action slot a: each row field is read and
// written as one coalesced vector, and the row's regret matching gathers the
// eight regrets with shuffles and sums them in slot order, like node_strategy.
// `group`/`ngroups` enumerate the 8-lane groups working on this table.
__device__ __forceinline__ void apply_rows(const GameParams& G, const TableView& tv, const Sched* sched, double rinv,
                                           unsigned group, unsigned ngroups, bool leader) {
  const uint32_t uid = update_id(sched, G.N);
  const size_t per_shard = (tv.mask + 1) / kListShards;
  const double w = G.lcfr ? (double)(float)sched->iteration : 1.0;
  const double s32 = 2.3283064365386962890625e-10;  // 2^-32
  const int a = threadIdx.x & 7;
  const unsigned gmask = 0xFFu << (threadIdx.x & 24);
  unsigned wide_rows = 0;  // rows whose second line was written back (counted by lane 0 of each group)
  for (int sh = 0; sh < kListShards; ++sh) {
  const unsigned n = *list_count(tv, uid & 1, sh);
  const unsigned* list = tv.touched + (size_t)sh * per_shard;
  for (unsigned i = group; i < n; i += ngroups) {
    const unsigned long long slot = list[i];
    // every field of both lines is loaded at once: a row's accumulators are
    // zero unless its flags say they were written, so no load waits on another
    const uint32_t m = (uint32_t)(*row_tag(tv, slot) & 0xFF);
    const unsigned long long cnt = *row_cnt(tv, slot);
    const long long canon = (long long)(cnt & 0xFFFFFFFFull);
    const long long su = (long long)*row_su(tv, slot);
    const unsigned flags = *row_flags(tv, slot);
    float* regp = reinterpret_cast<float*>(row_reg(tv, slot));
    float* ssp = reinterpret_cast<float*>(row_ssum(tv, slot));
    long long* dap = reinterpret_cast<long long*>(row_da(tv, slot));
    long long* dsp = reinterpret_cast<long long*>(row_ds(tv, slot));
    const float r_a = regp[a];
    const float s_a = ssp[a];
    const long long da_a = dap[a];
    const long long ds_a = dsp[a];
    // strategy of the canonical mask from the snapshot regrets (node_strategy)
    float sum_r = 0.0f;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const float rb = __shfl_sync(gmask, r_a, b, 8);
      if ((m >> b) & 1) sum_r = __fadd_rn(sum_r, fmaxf(0.0f, rb));
    }
    const bool in = (m >> a) & 1;
    float strat_a = 0.0f;
    if (in) strat_a = (sum_r > 1e-7f) ? __fdiv_rn(fmaxf(0.0f, r_a), sum_r) : __fdiv_rn(1.0f, (float)__popc(m));
    const long long dr = da_a - (in ? su : 0ll);
    const long long dsv = ds_a + (in ? canon * fix_s(strat_a) : 0ll);
    float r = __fadd_rn(r_a, __double2float_rn(__dmul_rn((double)dr, rinv)));
    if (G.cfr_plus) r = (r < 0.0f) ? 0.0f : r;
    regp[a] = r;
    ssp[a] = __fadd_rn(s_a, __double2float_rn(__dmul_rn(__dmul_rn((double)dsv, s32), w)));
    if (flags & kFlagDa) dap[a] = 0;
    if (flags & kFlagDs) dsp[a] = 0;
    if (a == 0) {
      *row_visits(tv, slot) += cnt >> 32;
      *row_cnt(tv, slot) = 0;
      *row_su(tv, slot) = 0;
      *row_flags(tv, slot) = 0;
      wide_rows += (flags & (kFlagDa | kFlagDs)) ? 1u : 0u;
    }
  }
  }
  wide_rows = __reduce_add_sync(0xFFFFFFFFu, wide_rows);
  if ((threadIdx.x & 31) == 0 && wide_rows) atomicAdd(wide_count(tv, uid & 1), wide_rows);
  if (leader) {
    const uint32_t next = (uid + 1) & 1;
    for (int sh = 0; sh < kListShards; ++sh) *list_count(tv, next, sh) = 0;
    *wide_count(tv, next) = 0;
  }
}

__global__ void __launch_bounds__(256) k_apply(const GameParams G, const TableView tv,
                                               const Sched* __restrict__ sched, double rinv) {
  apply_rows(G, tv, sched, rinv, (blockIdx.x * blockDim.x + threadIdx.x) >> 3, (gridDim.x * blockDim.x) >> 3,
             blockIdx.x == 0 && threadIdx.x == 0);
}

// Apply of every table in a phase: blockIdx.y selects the table.
__global__ void __launch_bounds__(256) k_apply_batched(const TableDesc* __restrict__ tables,
                                                       const PhaseDesc* __restrict__ phase) {
  const TableDesc& D = tables[phase->table[blockIdx.y]];
  apply_rows(D.G, D.tv, D.sched, D.rinv, (blockIdx.x * blockDim.x + threadIdx.x) >> 3,
             (gridDim.x * blockDim.x) >> 3, blockIdx.x == 0 && threadIdx.x == 0);
}

__global__ void k_advance(Sched* s, int N) {
  int p = s->player + 1;
  if (p >= N) {
    p = 0;
    s->iteration += 1;
  }
  s->player = p;
}

__global__ void k_advance_batched(const TableDesc* __restrict__ tables, const PhaseDesc* __restrict__ phase) {
  const int j = threadIdx.x;
  if (j >= phase->n) return;
  const TableDesc& D = tables[phase->table[j]];
  int p = D.sched->player + 1;
  if (p >= D.G.N) {
    p = 0;
    D.sched->iteration += 1;
  }
  D.sched->player = p;
}

// Occupied rows of the table (one atomic per warp).
__global__ void k_count_rows(const TableView tv, unsigned long long cap_slots, unsigned int* __restrict__ on) {
  unsigned c = 0;
  for (unsigned long long s = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; s < cap_slots;
       s += (unsigned long long)gridDim.x * blockDim.x)
    c += *row_key(tv, s) != 0;
  c = __reduce_add_sync(0xFFFFFFFFu, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(on, c);
}

// Order-independent digest of the occupied rows (mccfr_table_digest).
__global__ void k_digest(const TableView tv, unsigned long long cap_slots, unsigned long long* __restrict__ out) {
  unsigned long long sum = 0, rows = 0;
  for (unsigned long long s = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; s < cap_slots;
       s += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long k = *row_key(tv, s);
    if (!k) continue;
    const uint32_t* r = reinterpret_cast<const uint32_t*>(row_reg(tv, s));
    const uint32_t* q = reinterpret_cast<const uint32_t*>(row_ssum(tv, s));
    uint32_t rb[8], qb[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      rb[a] = r[a];
      qb[a] = q[a];
    }
    sum += row_digest(k, rb, qb, *row_visits(tv, s));
    rows++;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_down_sync(0xFFFFFFFFu, sum, o);
    rows += __shfl_down_sync(0xFFFFFFFFu, rows, o);
  }
  if ((threadIdx.x & 31) == 0 && rows) {
    atomicAdd(out, sum);
    atomicAdd(out + 1, rows);
  }
}

// Compacts the occupied rows into arrays of `bound` rows (unordered).
__global__ void k_export(const TableView tv, unsigned long long cap_slots,
                         unsigned long long* __restrict__ okeys, float4* __restrict__ oreg,
                         float4* __restrict__ ossum, unsigned long long* __restrict__ ovis,
                         unsigned int* __restrict__ on, unsigned bound) {
  for (unsigned long long s = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; s < cap_slots;
       s += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long k = *row_key(tv, s);
    if (!k) continue;
    const unsigned i = atomicAdd(on, 1u);
    if (i >= bound) continue;
    okeys[i] = k;
    oreg[2 * i] = row_reg(tv, s)[0];
    oreg[2 * i + 1] = row_reg(tv, s)[1];
    ossum[2 * i] = row_ssum(tv, s)[0];
    ossum[2 * i + 1] = row_ssum(tv, s)[1];
    ovis[i] = *row_visits(tv, s);
  }
}

// Inserts dense reference-layout rows (FNV slot + 1 as key) with any non-zero
// value (load_checkpoint / import_tables).
__global__ void k_import_dense(const TableView tv, const float* __restrict__ dr, const float* __restrict__ ds,
                               unsigned n_slots) {
  for (unsigned s = blockIdx.x * blockDim.x + threadIdx.x; s < n_slots; s += gridDim.x * blockDim.x) {
    float r[8], q[8];
    bool any = false;
    for (int a = 0; a < 8; ++a) {
      r[a] = dr[(size_t)a * n_slots + s];
      q[a] = ds[(size_t)a * n_slots + s];
      any |= (r[a] != 0.0f) || (q[a] != 0.0f);
    }
    if (!any) continue;
    const long long slot = table_insert(tv, (unsigned long long)s + 1);
    if (slot < 0) continue;
    row_reg(tv, slot)[0] = make_float4(r[0], r[1], r[2], r[3]);
    row_reg(tv, slot)[1] = make_float4(r[4], r[5], r[6], r[7]);
    row_ssum(tv, slot)[0] = make_float4(q[0], q[1], q[2], q[3]);
    row_ssum(tv, slot)[1] = make_float4(q[4], q[5], q[6], q[7]);
  }
}

// Rows of a v2 checkpoint into an empty table: each key's row gets its
// regrets, strategy sums and visit count (keys checked on the host first).
__global__ void k_import_rows(const TableView tv, const unsigned long long* __restrict__ keys,
                              const float4* __restrict__ reg, const float4* __restrict__ ssum,
                              const unsigned long long* __restrict__ visits, unsigned long long n) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const long long slot = table_insert(tv, keys[i]);
    if (slot < 0) continue;  // table_insert raised the table-full flag
    row_reg(tv, slot)[0] = reg[2 * i];
    row_reg(tv, slot)[1] = reg[2 * i + 1];
    row_ssum(tv, slot)[0] = ssum[2 * i];
    row_ssum(tv, slot)[1] = ssum[2 * i + 1];
    *row_visits(tv, slot) = visits[i];
  }
}

__global__ void k_export_dense(const TableView tv, unsigned long long cap_slots, float* __restrict__ dr,
                               float* __restrict__ ds, unsigned n_slots) {
  for (unsigned long long s = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; s < cap_slots;
       s += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long k = *row_key(tv, s);
    if (!k || k > n_slots) continue;
    const unsigned d = (unsigned)(k - 1);
    const float* r = reinterpret_cast<const float*>(row_reg(tv, s));
    const float* q = reinterpret_cast<const float*>(row_ssum(tv, s));
    for (int a = 0; a < 8; ++a) {
      dr[(size_t)a * n_slots + d] = r[a];
      ds[(size_t)a * n_slots + d] = q[a];
    }
  }
}

// CFR+ clamp of every row (after importing regrets that may be negative).
__global__ void k_clamp_all(const TableView tv, unsigned long long cap_slots) {
  for (unsigned long long s = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; s < cap_slots;
       s += (unsigned long long)gridDim.x * blockDim.x) {
    float4 a = row_reg(tv, s)[0], b = row_reg(tv, s)[1];
    a.x = a.x < 0.f ? 0.f : a.x; a.y = a.y < 0.f ? 0.f : a.y; a.z = a.z < 0.f ? 0.f : a.z; a.w = a.w < 0.f ? 0.f : a.w;
    b.x = b.x < 0.f ? 0.f : b.x; b.y = b.y < 0.f ? 0.f : b.y; b.z = b.z < 0.f ? 0.f : b.z; b.w = b.w < 0.f ? 0.f : b.w;
    row_reg(tv, s)[0] = a;
    row_reg(tv, s)[1] = b;
  }
}

// One thread per 7-card hand: 7 dependent gathers (hand_eval.cpp:134-143).
__global__ void k_eval7(const int32_t* __restrict__ T, const uint8_t* __restrict__ cards,
                        uint16_t* __restrict__ ranks, unsigned long long n) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint8_t* c = cards + 7 * i;
    int32_t p = __ldg(T + 53 + to_rm(c[0]));
#pragma unroll
    for (int k = 1; k < 7; ++k) p = __ldg(T + p + to_rm(c[k]));
    ranks[i] = (uint16_t)decode16((uint32_t)p & 0xFFFF);
  }
}

// Exact rank histogram of all C(52, n) hands (n = 5, 6, 7), one thread per
// ordered 3-card prefix a<b<c.
__global__ void k_rank_hist(const int32_t* __restrict__ T, int ncards, unsigned long long* __restrict__ hist) {
  __shared__ unsigned int sh[7463];
  for (int i = threadIdx.x; i < 7463; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const unsigned id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id < 52u * 52u * 52u) {
    const int a = id / 2704, b = (id / 52) % 52, c = id % 52;
    if (a < b && b < c) {
      const int32_t pc = __ldg(T + __ldg(T + __ldg(T + 53 + to_rm(a)) + to_rm(b)) + to_rm(c));
      for (int d = c + 1; d < 52; ++d) {
        const int32_t pd = __ldg(T + pc + to_rm(d));
        for (int e = d + 1; e < 52; ++e) {
          const int32_t pe = __ldg(T + pd + to_rm(e));
          if (ncards == 5) {
            atomicAdd(&sh[decode16((uint32_t)__ldg(T + pe) & 0xFFFF)], 1u);
            continue;
          }
          for (int f = e + 1; f < 52; ++f) {
            const int32_t pf = __ldg(T + pe + to_rm(f));
            if (ncards == 6) {
              atomicAdd(&sh[decode16((uint32_t)__ldg(T + pf) & 0xFFFF)], 1u);
              continue;
            }
            for (int g = f + 1; g < 52; ++g)
              atomicAdd(&sh[decode16((uint32_t)__ldg(T + pf + to_rm(g)) & 0xFFFF)], 1u);
          }
        }
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 7463; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], (unsigned long long)sh[i]);
}

}  // namespace

// ---------------------------------------------------------------------------
// Handle
// ---------------------------------------------------------------------------
struct mccfr_handle {
  mccfr_config cfg;
  GameParams gp;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t gev[3 * MCCFR_MAX_PLAYERS] = {};  // per update in the graph: start, after traverse, after apply
  // hand data
  int32_t* d_hr = nullptr;
  uint8_t* d_pre = nullptr;
  uint8_t* d_cdf = nullptr;
  bool has_table = false;
  // info-set table
  unsigned long long cap = 0;
  TableView tv{};
  void* d_block = nullptr;  // one allocation for the table arrays
  size_t block_bytes = 0;
  Sched* d_sched = nullptr;
  DealRec* d_deals = nullptr;  // one record per traversal of an update
  int deals_cap = 0;
  uint32_t* d_ranges = nullptr;  // subgame range CDFs [N][1326]
  bool shared_hr = false;        // d_hr borrowed from another handle
  int round_player = 0;          // next player of round-by-round training
  Sched* h_sched = nullptr;  // pinned
  Counters* d_counters = nullptr;
  unsigned* d_work = nullptr;  // traversal work counter of the persistent kernel
  // level-synchronous form: node and seed buffers of one update
  void* d_level = nullptr;
  size_t level_bytes = 0;
  int level_batch = 0;  // batch the buffers were sized for
  int level_last_batch = 0;  // traversals of the last update enqueued in the level form
  LevelBufs lb{};
  int grid_expand = 0, grid_back = 0, grid_dfs = 0;  // resident blocks on this handle's device
  // graph of one iteration
  cudaGraphExec_t graph = nullptr;
  int graph_batch = -1;
  long long iterations_done = 0;
  long long launches = 0;
  double traverse_ms = 0, apply_ms = 0, last_traverse_ms = 0, last_apply_ms = 0;
  long long touched_last = 0;
  long long wide_last = 0;  // of those, rows whose second line was folded
  int sticky_err = 0;
  std::string last_error;
  size_t persist_prev = 0;
  bool persist_set = false;
};

namespace {

int fail(mccfr_handle* h, int code, const char* fmt, ...) {
  if (h) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    h->last_error = buf;
  }
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(h, e_ == cudaErrorMemoryAllocation ? MCCFR_ERR_OOM : MCCFR_ERR_CUDA,        \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

int regret_frac_bits(const mccfr_config& c, long long batch) {
  auto bitlen = [](unsigned long long v) {
    int b = 0;
    while (v) {
      ++b;
      v >>= 1;
    }
    return b;
  };
  const unsigned long long span =
      20ull * (unsigned long long)c.num_players * (unsigned long long)std::max(1, c.starting_stack);
  int rb = 61 - bitlen((unsigned long long)batch) - bitlen(span) - 6;
  return std::min(24, std::max(8, rb));
}

int validate(const mccfr_config& c, std::string& why) {
  if (c.num_players < 2 || c.num_players > 6) return why = "num_players must be 2..6", 1;
  if (c.starting_stack <= 0 || c.starting_stack > 65535) return why = "starting_stack must be 1..65535", 1;
  if (c.small_blind < 0 || c.big_blind <= 0 || c.small_blind > c.starting_stack || c.big_blind > c.starting_stack)
    return why = "blinds must be positive and at most the stack", 1;
  if (c.num_actions < 1 || c.num_actions > 8) return why = "num_actions must be 1..8", 1;
  bool has_fold = false, has_check = false;
  for (int a = 0; a < c.num_actions; ++a) {
    const int k = c.action_kind[a];
    if (k < 0 || k > 6) return why = "unknown action kind", 1;
    if (k == MCCFR_ACT_RAISE_POT && (c.action_den[a] <= 0 || c.action_num[a] <= 0 || c.action_num[a] > 16))
      return why = "RAISE_POT needs 0 < num <= 16 and den > 0", 1;
    has_fold |= k == MCCFR_ACT_FOLD;
    has_check |= k == MCCFR_ACT_CHECK || k == MCCFR_ACT_CHECK_CALL;
  }
  if (!has_fold || !has_check) return why = "action set needs a fold slot and a check (or check/call) slot", 1;
  if (c.sampling != MCCFR_SAMPLING_REFERENCE && c.sampling != MCCFR_SAMPLING_EXTERNAL)
    return why = "unknown sampling mode", 1;
  if (c.key_mode != MCCFR_KEY_FNV26 && c.key_mode != MCCFR_KEY_ID64) return why = "unknown key mode", 1;
  if (c.max_depth < 1 || c.max_depth > 255) return why = "max_depth must be 1..255", 1;
  if (c.raise_cap < 0 || c.raise_cap > 15) return why = "raise_cap must be 0..15", 1;
  if (c.preflop_mode == MCCFR_PREFLOP_CHEN64) {
    if (c.preflop_buckets < 1 || c.preflop_buckets > 256) return why = "preflop_buckets must be 1..256", 1;
  } else if (c.preflop_mode == MCCFR_PREFLOP_CLASS169) {
    if (c.preflop_buckets != 169) return why = "CLASS169 needs preflop_buckets = 169", 1;
  } else {
    return why = "unknown preflop mode", 1;
  }
  if (c.postflop_mode != MCCFR_POSTFLOP_REF_LINEAR && c.postflop_mode != MCCFR_POSTFLOP_RANK_CDF)
    return why = "unknown postflop mode", 1;
  for (int s = 0; s < 3; ++s)
    if (c.postflop_buckets[s] < 1 || c.postflop_buckets[s] > 256) return why = "postflop buckets must be 1..256", 1;
  if (c.table_log2 < 10 || c.table_log2 > 31) return why = "table_log2 must be 10..31", 1;
  if (c.key_bits < 0 || c.key_bits > 48) return why = "key_bits must be 0..48", 1;
  if (c.traversal_form < MCCFR_FORM_AUTO || c.traversal_form > MCCFR_FORM_LEVELS)
    return why = "unknown traversal form", 1;
  if (c.level_log2 != 0 && (c.level_log2 < 8 || c.level_log2 > 30))
    return why = "level_log2 must be 0 or 8..30", 1;
  // Reference rule walks one path; its records hold the updating player's nodes.
  if (c.sampling == MCCFR_SAMPLING_REFERENCE && c.raise_cap == 0 && c.max_depth > 2 * kMaxRec)
    return why = "reference sampling without a raise cap needs max_depth <= 48", 1;
  if (c.sampling == MCCFR_SAMPLING_REFERENCE && c.raise_cap > 0 && 4 * (c.raise_cap + 1) > kMaxRec)
    return why = "reference sampling needs raise_cap <= 5", 1;
  return 0;
}

// Every key lies in [1, 2^kb]: an FNV26 key is a 26-bit slot plus one, an ID64
// key reduced to key_bits bits is that plus one.  When 2^kb rows fit in the
// table, key k owns row k-1 and the table needs no probing.
int direct_map(const mccfr_config& c) {
  const int kb = c.key_mode == MCCFR_KEY_FNV26 ? 26 : c.key_bits;
  return kb > 0 && kb <= c.table_log2 ? 1 : 0;
}

void make_params(const mccfr_config& c, GameParams& g) {
  std::memset(&g, 0, sizeof(g));
  g.N = c.num_players;
  g.stack = c.starting_stack;
  g.sb = c.small_blind;
  g.bb = c.big_blind;
  g.cfr_plus = c.use_cfr_plus;
  g.lcfr = c.use_linear_cfr;
  g.sampling = c.sampling;
  g.key_mode = c.key_mode;
  g.num_actions = c.num_actions;
  g.raise_cap = c.raise_cap;
  g.max_depth = c.max_depth;
  g.postflop_mode = c.postflop_mode;
  for (int s = 0; s < 3; ++s) g.post_b[s] = c.postflop_buckets[s];
  g.seed_lo = (uint32_t)c.seed;
  g.seed_hi = (uint32_t)(c.seed >> 32);
  g.key_bits = c.key_mode == MCCFR_KEY_ID64 ? c.key_bits : 0;
  g.stack_base = c.starting_stack;
  for (int a = 0; a < 8; ++a) {
    g.kind[a] = (int8_t)(a < c.num_actions ? c.action_kind[a] : -1);
    g.num[a] = (int16_t)(a < c.num_actions ? c.action_num[a] : 0);
    g.den[a] = (int16_t)(a < c.num_actions ? std::max(1, c.action_den[a]) : 1);
    g.den_shift[a] = -1;
    for (int k = 0; k < 15; ++k)
      if (g.den[a] == (1 << k)) g.den_shift[a] = (int8_t)k;
    const int k = g.kind[a];
    if (k == MCCFR_ACT_FOLD) g.m_fold |= 1u << a;
    if (k == MCCFR_ACT_CHECK || k == MCCFR_ACT_CHECK_CALL) g.m_check |= 1u << a;
    if (k == MCCFR_ACT_CALL || k == MCCFR_ACT_CHECK_CALL) g.m_call |= 1u << a;
    if (k == MCCFR_ACT_ALL_IN) g.m_allin |= 1u << a;
    if (k == MCCFR_ACT_RAISE_MIN || k == MCCFR_ACT_RAISE_POT) g.m_raise |= 1u << a;
  }
  // Passive fallback order (cfr_gpu.cu:498-508): check, check/call, call, fold,
  // raises in slot order, all-in.
  const int order[] = {MCCFR_ACT_CHECK, MCCFR_ACT_CHECK_CALL, MCCFR_ACT_CALL, MCCFR_ACT_FOLD, -2,
                       MCCFR_ACT_ALL_IN};
  g.n_fallback = 0;
  for (int k : order)
    for (int a = 0; a < c.num_actions; ++a) {
      const int kd = c.action_kind[a];
      const bool raise = kd == MCCFR_ACT_RAISE_MIN || kd == MCCFR_ACT_RAISE_POT;
      if ((k == -2 && raise) || kd == k) g.fallback[g.n_fallback++] = (uint8_t)a;
    }
  g.default_slot = 0;
  for (int a = 0; a < c.num_actions; ++a)
    if (c.action_kind[a] == MCCFR_ACT_CHECK || c.action_kind[a] == MCCFR_ACT_CHECK_CALL) {
      g.default_slot = (uint8_t)a;
      break;
    }
}

int grid_for(long long work, int block) {
  long long g = (work + block - 1) / block;
  return (int)std::max(1LL, std::min(g, 148LL * 64));
}

int check_device_error(mccfr_handle* h) {
  int e = 0;
  CK(cudaMemcpy(&e, h->tv.err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    h->sticky_err |= e;
    CK(cudaMemset(h->tv.err, 0, sizeof(int)));
    if (e & kErrTableFull)
      return fail(h, MCCFR_ERR_TABLE_FULL, "info-set table full (capacity %llu rows); raise table_log2", h->cap);
    return fail(h, MCCFR_ERR_DEVICE, "kernel error flags 0x%x", e);
  }
  return MCCFR_OK;
}

// Rows the player-update of parity `par` listed (all shards) and folded wide.
int read_touched(mccfr_handle* h, uint32_t par) {
  unsigned c[kCounterBytes / 4];
  CK(cudaMemcpy(c, h->tv.n_touched, sizeof(c), cudaMemcpyDeviceToHost));
  TableView hv = h->tv;
  hv.n_touched = c;
  long long n = 0;
  for (int sh = 0; sh < kListShards; ++sh) n += *list_count(hv, par, sh);
  h->touched_last = n;
  h->wide_last = *wide_count(hv, par);
  return MCCFR_OK;
}

// Records `e` on the handle's stream; inside a stream capture this must be an
// external record so that it becomes an event node of the graph.
int record(mccfr_handle* h, cudaEvent_t e, bool capturing) {
  CK(capturing ? cudaEventRecordWithFlags(e, h->stream, cudaEventRecordExternal) : cudaEventRecord(e, h->stream));
  return MCCFR_OK;
}

bool use_levels(const mccfr_handle* h);
int enqueue_levels(mccfr_handle* h, int batch, float rscale);

// Enqueues one player-update (traverse + apply) reading the device schedule;
// `ev3` (optional) receives event records before, between and after.
int enqueue_update(mccfr_handle* h, int batch, mccfr_trace* d_trace, cudaEvent_t* ev3, bool capturing = false) {
  const int rb = regret_frac_bits(h->cfg, batch);
  const float rscale = std::ldexp(1.0f, rb);
  const double rinv = std::ldexp(1.0, -rb);
  HandView hv{h->d_hr, h->d_pre, h->d_cdf};
  if (batch > h->deals_cap) return fail(h, MCCFR_ERR_INVALID_ARG, "deal buffer smaller than the batch");
  k_deal<<<(batch + 127) / 128, 128, 0, h->stream>>>(h->gp, hv, h->d_sched, batch, h->d_deals);
  CK(cudaGetLastError());
  if (ev3 && record(h, ev3[0], capturing)) return MCCFR_ERR_CUDA;
  if (h->cfg.sampling == MCCFR_SAMPLING_REFERENCE) {
    const int grid = (batch + kRefBlock - 1) / kRefBlock;
    if (d_trace)
      k_traverse_ref<kRefBlock, true><<<grid, kRefBlock, 0, h->stream>>>(h->gp, h->tv, h->d_deals, h->d_sched,
                                                                           batch, rscale, h->d_counters, d_trace);
    else
      k_traverse_ref<kRefBlock, false><<<grid, kRefBlock, 0, h->stream>>>(h->gp, h->tv, h->d_deals, h->d_sched,
                                                                            batch, rscale, h->d_counters, nullptr);
  } else if (use_levels(h)) {
    const int rc = enqueue_levels(h, batch, rscale);
    if (rc) return rc;
  } else {
    launch_traverse_es(h->gp, h->tv, h->d_deals, h->d_sched, batch, rscale, h->d_counters, h->d_work, h->stream,
                       h->device);
  }
  CK(cudaGetLastError());
  if (ev3 && record(h, ev3[1], capturing)) return MCCFR_ERR_CUDA;
  k_apply<<<148 * 8, 256, 0, h->stream>>>(h->gp, h->tv, h->d_sched, rinv);
  CK(cudaGetLastError());
  if (ev3 && record(h, ev3[2], capturing)) return MCCFR_ERR_CUDA;
  return MCCFR_OK;
}

// Traversal form of the update: the level-synchronous kernels for external
// sampling unless the config asks for the depth-first lanes.
bool use_levels(const mccfr_handle* h) {
  return h->cfg.sampling == MCCFR_SAMPLING_EXTERNAL && h->cfg.traversal_form != MCCFR_FORM_LANES;
}

// Seed levels of an update: the updating player acts at most raise_cap + 1
// times per street (once, and once more after each raise of another player),
// and at most once per node of the depth cut; one more level holds the seeds
// below its last possible decision.  Capped at kMaxLevels (the deepest level
// is then walked depth first).
int level_count(const mccfr_handle* h) {
  const mccfr_config& c = h->cfg;
  const int streets = h->gp.sub_street ? 4 - h->gp.sub_street : 4;
  int decisions = c.max_depth;
  if (c.raise_cap > 0) decisions = std::min(decisions, streets * (c.raise_cap + 1));
  return std::min(decisions + 1, kMaxLevels);
}

// Node and seed buffers for updates of `batch` traversals: 2^level_log2 node
// records of 80 B (default: 64 per traversal, 2^18..2^26), 8 seeds of 8 B per
// node (at least the batch and a margin) and one 24-byte showdown record per
// node.  A smaller allocation is tried when the device is short of memory; any
// size gives the same rows.
int ensure_levels(mccfr_handle* h, int batch) {
  const int nlev = level_count(h);
  if (h->d_level && h->level_batch >= batch) {
    if (h->lb.nlev != nlev && h->graph) {  // a subgame re-targeted to another street
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
      h->graph_batch = -1;
    }
    h->lb.nlev = nlev;
    return MCCFR_OK;
  }
  if (h->d_level) {
    CK(cudaStreamSynchronize(h->stream));
    cudaFree(h->d_level);
    h->d_level = nullptr;
    h->level_batch = 0;
  }
  int lg = h->cfg.level_log2;
  if (!lg) {
    lg = 18;
    while (lg < 26 && (1ull << lg) < 64ull * (unsigned long long)batch) ++lg;
  }
  for (;; --lg) {
    const unsigned long long nodes = 1ull << lg;
    const unsigned long long seeds = std::max(8ull * nodes, (unsigned long long)batch + (1ull << 20));
    const unsigned long long shows = nodes;
    const size_t bytes =
        nodes * (sizeof(EsState) + sizeof(uint4)) + seeds * 8 + shows * sizeof(ShowRec) + sizeof(LevelCtl) + 256;
    const cudaError_t e = cudaMalloc(&h->d_level, bytes);
    if (e == cudaSuccess) {
      char* p = static_cast<char*>(h->d_level);
      h->lb.nodes = reinterpret_cast<EsState*>(p);
      p += nodes * sizeof(EsState);
      h->lb.meta = reinterpret_cast<uint4*>(p);
      p += nodes * sizeof(uint4);
      h->lb.child = reinterpret_cast<uint32_t*>(p);
      p += seeds * 4;
      h->lb.value = reinterpret_cast<float*>(p);
      p += seeds * 4;
      h->lb.show = reinterpret_cast<ShowRec*>(p);
      p += shows * sizeof(ShowRec);
      p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(p) + 127) & ~(uintptr_t)127);
      h->lb.ctl = reinterpret_cast<LevelCtl*>(p);
      h->lb.node_cap = (uint32_t)nodes;
      h->lb.seed_cap = (uint32_t)seeds;
      h->lb.show_cap = (uint32_t)shows;
      h->level_bytes = bytes;
      h->level_batch = batch;
      break;
    }
    cudaGetLastError();  // clear the allocation error
    if (e != cudaErrorMemoryAllocation || lg <= 12)
      return fail(h, MCCFR_ERR_OOM, "level buffers: %s", cudaGetErrorString(e));
  }
  h->lb.nlev = nlev;
  if (!h->grid_expand) {
    int sms = 0, per = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_level_expand<128, 1, false>, 128, 0));
    h->grid_expand = std::max(1, per) * sms;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_level_back<256>, 256, 0));
    h->grid_back = std::max(1, per) * sms;
    const size_t smem = 2 * 128 * sizeof(EsFrame);
    CK(cudaFuncSetAttribute(k_level_dfs<128, 2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_level_dfs<128, 2, 1>, 128, smem));
    h->grid_dfs = std::max(1, per) * sms;
  }
  if (h->graph) {  // the graph captured the old buffers
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
    h->graph_batch = -1;
  }
  return MCCFR_OK;
}

// One external-sampling update in the level-synchronous form: the levels
// expanded top down, the seeds that did not fit walked depth first, the
// recorded showdowns evaluated in one pass, the values returned bottom up.
int enqueue_levels(mccfr_handle* h, int batch, float rscale) {
  const LevelBufs& lb = h->lb;
  h->level_last_batch = batch;
  CK(cudaMemsetAsync(lb.ctl, 0, sizeof(LevelCtl), h->stream));
  k_level_expand<128, 1, true><<<h->grid_expand, 128, 0, h->stream>>>(h->gp, h->tv, h->d_deals, h->d_sched, batch,
                                                                      lb, 0, h->d_counters);
  for (int L = 1; L < lb.nlev; ++L)
    k_level_expand<128, 1, false><<<h->grid_expand, 128, 0, h->stream>>>(h->gp, h->tv, h->d_deals, h->d_sched,
                                                                         batch, lb, L, h->d_counters);
  CK(cudaGetLastError());
  k_level_dfs<128, 2, 1><<<h->grid_dfs, 128, 2 * 128 * sizeof(EsFrame), h->stream>>>(
      h->gp, h->tv, h->d_deals, h->d_sched, batch, rscale, lb, h->d_counters);
  CK(cudaGetLastError());
  k_level_showdown<256><<<h->grid_back, 256, 0, h->stream>>>(h->gp, h->d_deals, h->d_sched, lb);
  CK(cudaGetLastError());
  for (int L = lb.nlev - 2; L >= 0; --L)
    k_level_back<256><<<h->grid_back, 256, 0, h->stream>>>(h->gp, h->tv, h->d_sched, batch, rscale, lb, L,
                                                           h->d_counters);
  CK(cudaGetLastError());
  return MCCFR_OK;
}

int ensure_deals(mccfr_handle* h, int batch) {
  if (batch <= h->deals_cap) return MCCFR_OK;
  if (h->d_deals) {
    CK(cudaStreamSynchronize(h->stream));
    cudaFree(h->d_deals);
    h->d_deals = nullptr;
    h->deals_cap = 0;
  }
  CK(cudaMalloc(&h->d_deals, (size_t)batch * sizeof(DealRec)));
  h->deals_cap = batch;
  if (h->graph) {  // the graph captured the old buffer
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
    h->graph_batch = -1;
  }
  return MCCFR_OK;
}

int ensure_graph(mccfr_handle* h, int batch) {
  {
    int rc = ensure_deals(h, batch);
    if (!rc && use_levels(h)) rc = ensure_levels(h, batch);
    if (rc) return rc;
  }
  if (h->graph && h->graph_batch == batch) return MCCFR_OK;
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = MCCFR_OK;
  for (int p = 0; p < h->cfg.num_players && rc == MCCFR_OK; ++p) {
    rc = enqueue_update(h, batch, nullptr, h->gev + 3 * p, true);
    if (rc == MCCFR_OK) {
      k_advance<<<1, 1, 0, h->stream>>>(h->d_sched, h->cfg.num_players);
      if (cudaGetLastError() != cudaSuccess) rc = MCCFR_ERR_CUDA;
    }
  }
  const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (rc != MCCFR_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(h, MCCFR_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  const cudaError_t e2 = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (e2 != cudaSuccess) return fail(h, MCCFR_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e2));
  h->graph_batch = batch;
  return MCCFR_OK;
}

int set_sched(mccfr_handle* h, long long iteration, int player) {
  h->h_sched->iteration = iteration;
  h->h_sched->player = player;
  h->h_sched->pad = 0;
  CK(cudaMemcpyAsync(h->d_sched, h->h_sched, sizeof(Sched), cudaMemcpyHostToDevice, h->stream));
  return MCCFR_OK;
}

struct HostRow {
  unsigned long long key;
  float reg[8], ssum[8];
  unsigned long long visits;
};
static_assert(sizeof(HostRow) == 80, "a v2 checkpoint row is 80 bytes");

// Occupied rows (a counting pass over the table).
int count_rows(mccfr_handle* h, unsigned int* n) {
  CK(cudaStreamSynchronize(h->stream));
  unsigned int* d_n = nullptr;
  CK(cudaMalloc(&d_n, sizeof(unsigned int)));
  cudaError_t e = cudaMemsetAsync(d_n, 0, sizeof(unsigned int), h->stream);
  if (e == cudaSuccess) {
    k_count_rows<<<148 * 16, 256, 0, h->stream>>>(h->tv, h->cap, d_n);
    e = cudaMemcpyAsync(n, d_n, sizeof(unsigned int), cudaMemcpyDeviceToHost, h->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d_n);
  if (e != cudaSuccess) return fail(h, MCCFR_ERR_CUDA, "row count: %s", cudaGetErrorString(e));
  return MCCFR_OK;
}

// Indices of `k` in ascending key order: LSD radix sort, 8 bits per pass,
// skipping the bytes in which all keys agree (keys are distinct).
void order_by_key(const std::vector<unsigned long long>& k, std::vector<unsigned>& order) {
  const size_t n = k.size();
  order.resize(n);
  for (size_t i = 0; i < n; ++i) order[i] = (unsigned)i;
  unsigned long long orv = 0, andv = ~0ull;
  for (unsigned long long x : k) {
    orv |= x;
    andv &= x;
  }
  const unsigned long long vary = orv ^ andv;
  std::vector<unsigned> tmp(n);
  for (int sh = 0; sh < 64; sh += 8) {
    if (((vary >> sh) & 0xFF) == 0) continue;
    size_t cnt[257] = {0};
    for (size_t i = 0; i < n; ++i) cnt[((k[order[i]] >> sh) & 0xFF) + 1]++;
    for (int b = 0; b < 256; ++b) cnt[b + 1] += cnt[b];
    for (size_t i = 0; i < n; ++i) tmp[cnt[(k[order[i]] >> sh) & 0xFF]++] = order[i];
    order.swap(tmp);
  }
}

// Every occupied row, sorted by key: counted first, then compacted into
// buffers of exactly that many rows and copied back.
int read_rows(mccfr_handle* h, std::vector<HostRow>& rows) {
  unsigned int n = 0;
  int rc = count_rows(h, &n);
  if (rc) return rc;
  rows.clear();
  if (n == 0) return MCCFR_OK;
  void* block = nullptr;
  const size_t bytes = (size_t)n * (8 + 8 + 32 + 32) + 256;
  cudaError_t e = cudaMalloc(&block, bytes);
  if (e != cudaSuccess) return fail(h, MCCFR_ERR_OOM, "export buffers: %s", cudaGetErrorString(e));
  char* base = static_cast<char*>(block);
  float4* oreg = reinterpret_cast<float4*>(base);
  float4* ossum = reinterpret_cast<float4*>(base + (size_t)n * 32);
  unsigned long long* okeys = reinterpret_cast<unsigned long long*>(base + (size_t)n * 64);
  unsigned long long* ovis = reinterpret_cast<unsigned long long*>(base + (size_t)n * 72);
  unsigned int* d_n = reinterpret_cast<unsigned int*>(base + (size_t)n * 80);
  std::vector<unsigned long long> k(n), v(n);
  std::vector<float> r(8ull * n), s(8ull * n);
  e = cudaMemsetAsync(d_n, 0, sizeof(unsigned int), h->stream);
  if (e == cudaSuccess) {
    k_export<<<148 * 16, 256, 0, h->stream>>>(h->tv, h->cap, okeys, oreg, ossum, ovis, d_n, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(k.data(), okeys, n * 8ull, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(v.data(), ovis, n * 8ull, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(r.data(), oreg, n * 32ull, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s.data(), ossum, n * 32ull, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(block);
  if (e != cudaSuccess) return fail(h, MCCFR_ERR_CUDA, "export: %s", cudaGetErrorString(e));
  std::vector<unsigned> order;
  order_by_key(k, order);
  rows.resize(n);
  for (unsigned j = 0; j < n; ++j) {
    const unsigned i = order[j];
    rows[j].key = k[i];
    std::memcpy(rows[j].reg, &r[8ull * i], 32);
    std::memcpy(rows[j].ssum, &s[8ull * i], 32);
    rows[j].visits = v[i];
  }
  return MCCFR_OK;
}

void release(mccfr_handle* h) {
  if (!h) return;
  if (h->device >= 0) cudaSetDevice(h->device);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  if (h->persist_set) {
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, h->persist_prev);
  }
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : h->gev)
    if (e) cudaEventDestroy(e);
  if (!h->shared_hr) cudaFree(h->d_hr);
  cudaFree(h->d_ranges);
  cudaFree(h->d_pre);
  cudaFree(h->d_cdf);
  cudaFree(h->d_block);
  cudaFree(h->d_deals);
  cudaFree(h->d_sched);
  cudaFreeHost(h->h_sched);
  cudaFree(h->d_counters);
  cudaFree(h->d_work);
  cudaFree(h->d_level);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* mccfr_strerror(int s) {
  switch (s) {
    case MCCFR_OK: return "ok";
    case MCCFR_ERR_INVALID_ARG: return "invalid argument";
    case MCCFR_ERR_CUDA: return "CUDA error";
    case MCCFR_ERR_OOM: return "out of device memory";
    case MCCFR_ERR_IO: return "file I/O error";
    case MCCFR_ERR_FORMAT: return "bad file format";
    case MCCFR_ERR_NO_HAND_TABLE: return "hand-rank table not loaded";
    case MCCFR_ERR_TABLE_FULL: return "info-set table full";
    case MCCFR_ERR_DEVICE: return "device-side error flag";
    case MCCFR_ERR_OVERFLOW: return "accumulator range exceeded";
    case MCCFR_ERR_CAPACITY: return "output buffer too small";
    case MCCFR_ERR_NO_DEVICE: return "no CUDA device";
    case MCCFR_ERR_TIMEOUT: return "timeout";
    default: return "unknown status";
  }
}

const char* mccfr_last_error(mccfr_handle* h) { return h ? h->last_error.c_str() : ""; }

int mccfr_abi_sizes(size_t* out3) {
  if (!out3) return MCCFR_ERR_INVALID_ARG;
  out3[0] = sizeof(mccfr_config);
  out3[1] = sizeof(mccfr_stats);
  out3[2] = sizeof(mccfr_trace);
  return MCCFR_OK;
}

int mccfr_config_init(mccfr_config* c, int preset) {
  if (!c) return MCCFR_ERR_INVALID_ARG;
  std::memset(c, 0, sizeof(*c));
  c->use_cfr_plus = 1;
  c->use_linear_cfr = 1;
  c->device = 0;
  if (preset == MCCFR_PRESET_REF8) {
    // GPUCFRTrainer defaults (cfr_gpu.cuh:50-55) and the fixed 8-slot
    // abstraction (abstraction.h:9-10, 42-53), FNV keys, depth cut 20.
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
    c->raise_cap = 0;
    c->max_depth = 20;
    c->preflop_mode = MCCFR_PREFLOP_CHEN64;
    c->preflop_buckets = 64;
    c->postflop_mode = MCCFR_POSTFLOP_REF_LINEAR;
    c->postflop_buckets[0] = c->postflop_buckets[1] = c->postflop_buckets[2] = 128;
    // one row per FNV slot, direct-mapped like the reference's [8][2^26] arrays
    // (cfr_gpu.cu:1106-1136): the table never fills
    c->table_log2 = 26;
    c->seed = 42;  // the reference's hard-wired seed (cfr_gpu.cuh:124)
    return MCCFR_OK;
  }
  if (preset == MCCFR_PRESET_HU_20BB || preset == MCCFR_PRESET_6MAX_100BB) {
    const bool hu = preset == MCCFR_PRESET_HU_20BB;
    // chips: 1 BB = 100 chips
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
    // 2^26 hashed info-set keys in a 2^27-row table (load <= 1/2, never full).
    c->key_bits = 26;
    c->table_log2 = 27;
    return MCCFR_OK;
  }
  return MCCFR_ERR_INVALID_ARG;
}

int mccfr_config_validate(const mccfr_config* cfg, char* why, size_t why_len) {
  if (!cfg) return MCCFR_ERR_INVALID_ARG;
  std::string msg;
  const bool bad = validate(*cfg, msg) != 0;
  if (why && why_len) {
    const size_t n = std::min(why_len - 1, bad ? msg.size() : (size_t)0);
    std::memcpy(why, msg.data(), n);
    why[n] = 0;
  }
  return bad ? MCCFR_ERR_INVALID_ARG : MCCFR_OK;
}

int mccfr_create(const mccfr_config* cfg, mccfr_handle** out) {
  if (!cfg || !out) return MCCFR_ERR_INVALID_ARG;
  *out = nullptr;
  std::string why;
  if (validate(*cfg, why)) {
    fprintf(stderr, "mccfr_create: %s\n", why.c_str());
    return MCCFR_ERR_INVALID_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MCCFR_ERR_NO_DEVICE;
  if (cfg->device < 0 || cfg->device >= ndev) return MCCFR_ERR_INVALID_ARG;
  mccfr_handle* h = new mccfr_handle();
  h->cfg = *cfg;
  h->device = cfg->device;
  make_params(*cfg, h->gp);
  auto bail = [&](int rc) {
    fprintf(stderr, "mccfr_create: %s\n", h->last_error.c_str());
    release(h);
    return rc;
  };
#define CKC(call)                                                                         \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return bail(fail(h, e_ == cudaErrorMemoryAllocation ? MCCFR_ERR_OOM : MCCFR_ERR_CUDA, \
                       "%s: %s", #call, cudaGetErrorString(e_)));                         \
  } while (0)
  CKC(cudaSetDevice(h->device));
  CKC(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  for (auto& e : h->ev) CKC(cudaEventCreate(&e));
  for (auto& e : h->gev) CKC(cudaEventCreate(&e));
  uint8_t pre[52 * 52];
  build_preflop_lut(cfg->preflop_mode, cfg->preflop_buckets, pre);
  CKC(cudaMalloc(&h->d_pre, sizeof(pre)));
  CKC(cudaMemcpy(h->d_pre, pre, sizeof(pre), cudaMemcpyHostToDevice));
  CKC(cudaMalloc(&h->d_cdf, 3 * 7463));
  CKC(cudaMemset(h->d_cdf, 0, 3 * 7463));
  CKC(cudaMalloc(&h->d_sched, sizeof(Sched)));
  CKC(cudaMallocHost(&h->h_sched, sizeof(Sched)));
  CKC(cudaMalloc(&h->d_counters, sizeof(Counters)));
  CKC(cudaMemset(h->d_counters, 0, sizeof(Counters)));
  CKC(cudaMalloc(&h->d_work, 256));
  CKC(cudaMemset(h->d_work, 0, 256));
  // Table rows, the touched list and small counters in one allocation.
  h->cap = 1ull << cfg->table_log2;
  const unsigned long long C = h->cap;
  const size_t bytes_rows = C * kRowBytes, bytes_touch = C * 4, bytes_misc = kCounterBytes;
  h->block_bytes = bytes_rows + bytes_touch + bytes_misc;
  CKC(cudaMalloc(&h->d_block, bytes_rows + bytes_touch + bytes_misc));
  CKC(cudaMemset(h->d_block, 0, bytes_rows + bytes_touch + bytes_misc));
  char* base = static_cast<char*>(h->d_block);
  h->tv.rows = reinterpret_cast<unsigned char*>(base);
  h->tv.touched = reinterpret_cast<unsigned int*>(base + bytes_rows);
  char* misc = base + bytes_rows + bytes_touch;
  h->tv.n_touched = reinterpret_cast<unsigned int*>(misc);
  h->tv.err = reinterpret_cast<int*>(misc + kCounterBytes - 128);
  h->tv.mask = C - 1;
  h->tv.log2cap = cfg->table_log2;
  h->tv.direct = direct_map(*cfg);
  *out = h;
  return MCCFR_OK;
#undef CKC
}

void mccfr_destroy(mccfr_handle* h) { release(h); }

int mccfr_get_config(mccfr_handle* h, mccfr_config* out) {
  if (!h || !out) return MCCFR_ERR_INVALID_ARG;
  *out = h->cfg;
  return MCCFR_OK;
}

int mccfr_get_stream(mccfr_handle* h, void** stream) {
  if (!h || !stream) return MCCFR_ERR_INVALID_ARG;
  *stream = (void*)h->stream;
  return MCCFR_OK;
}

int mccfr_set_hand_table(mccfr_handle* h, const int32_t* table, size_t n) {
  if (!h || !table) return MCCFR_ERR_INVALID_ARG;
  if (n != (size_t)MCCFR_HAND_TABLE_ENTRIES)
    return fail(h, MCCFR_ERR_FORMAT, "expected %d int32 entries, found %zu", MCCFR_HAND_TABLE_ENTRIES, n);
  // Known answer of the reference's loader (cfr_gpu.cu:270-299).
  {
    const int seq[7] = {51, 50, 49, 48, 47, 0, 14};
    auto rm = [](int c) { return (c % 13) * 4 + c / 13 + 1; };
    long long p = 53;
    bool ok = true;
    for (int i = 0; i < 7 && ok; ++i) {
      const long long idx = p + rm(seq[i]);
      if (idx < 0 || idx >= (long long)n) ok = false;
      else p = table[idx];
    }
    if (!ok || decode_packed((int32_t)(p & 0xFFFF)) != 7462)
      return fail(h, MCCFR_ERR_FORMAT, "As Ks Qs Js Ts 2c 3d does not decode to 7462");
  }
  CK(cudaSetDevice(h->device));
  const size_t bytes = n * sizeof(int32_t);
  if (!h->d_hr) CK(cudaMalloc(&h->d_hr, bytes));
  CK(cudaMemcpy(h->d_hr, table, bytes, cudaMemcpyHostToDevice));
  // Rank-CDF bucket LUTs from exact histograms.
  if (h->cfg.postflop_mode == MCCFR_POSTFLOP_RANK_CDF) {
    unsigned long long* d_hist = nullptr;
    CK(cudaMalloc(&d_hist, 7463 * sizeof(unsigned long long)));
    uint8_t lut[3][7463];
    for (int s = 0; s < 3; ++s) {
      CK(cudaMemset(d_hist, 0, 7463 * sizeof(unsigned long long)));
      k_rank_hist<<<(52 * 52 * 52 + 127) / 128, 128, 0, h->stream>>>(h->d_hr, 5 + s, d_hist);
      CK(cudaGetLastError());
      unsigned long long hist[7463];
      CK(cudaMemcpyAsync(hist, d_hist, sizeof(hist), cudaMemcpyDeviceToHost, h->stream));
      CK(cudaStreamSynchronize(h->stream));
      build_cdf_lut(hist, h->cfg.postflop_buckets[s], lut[s]);
    }
    cudaFree(d_hist);
    CK(cudaMemcpy(h->d_cdf, lut, sizeof(lut), cudaMemcpyHostToDevice));
  }
  // A persisting L2 access-policy window over the rank table is set only on
  // request (MCCFR_L2_PERSIST=1): the table (130 MB) is larger than the
  // set-aside, so the window marks a random share of its lines persisting and
  // streams the rest, and plain LRU, which keeps the hot upper states of the
  // state machine, hits more (measured on the showdown kernels: 76% vs 70% and
  // 72% vs 60% L2 read hits without and with the window).  Restored in
  // mccfr_destroy when set.
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, h->device));
  const char* env = getenv("MCCFR_L2_PERSIST");
  const bool want = env && env[0] == '1';
  if (want && prop.persistingL2CacheMaxSize > 0 && prop.accessPolicyMaxWindowSize > 0) {
    if (!h->persist_set) {
      size_t prev = 0;
      cudaDeviceGetLimit(&prev, cudaLimitPersistingL2CacheSize);
      h->persist_prev = prev;
      h->persist_set = true;
    }
    const size_t setaside = std::min<size_t>(prop.persistingL2CacheMaxSize, bytes);
    CK(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, setaside));
    cudaStreamAttrValue attr;
    std::memset(&attr, 0, sizeof(attr));
    const size_t win = std::min<size_t>(prop.accessPolicyMaxWindowSize, bytes);
    attr.accessPolicyWindow.base_ptr = h->d_hr;
    attr.accessPolicyWindow.num_bytes = win;
    attr.accessPolicyWindow.hitRatio = std::min(1.0f, (float)setaside / (float)win);
    attr.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    CK(cudaStreamSetAttribute(h->stream, cudaStreamAttributeAccessPolicyWindow, &attr));
    if (h->graph) {  // policies are baked into captured kernel nodes
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
      h->graph_batch = -1;
    }
  }
  h->has_table = true;
  return MCCFR_OK;
}

int mccfr_load_hand_table(mccfr_handle* h, const char* path) {
  if (!h || !path) return MCCFR_ERR_INVALID_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) return fail(h, MCCFR_ERR_IO, "cannot open %s", path);
  fseek(f, 0, SEEK_END);
  const long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  if (sz != (long)MCCFR_HAND_TABLE_ENTRIES * 4) {
    fclose(f);
    return fail(h, MCCFR_ERR_FORMAT, "%s: expected %d int32 entries, found %ld bytes", path,
                MCCFR_HAND_TABLE_ENTRIES, sz);
  }
  std::vector<int32_t> t(MCCFR_HAND_TABLE_ENTRIES);
  const size_t r = fread(t.data(), 4, t.size(), f);
  fclose(f);
  if (r != t.size()) return fail(h, MCCFR_ERR_IO, "%s: short read", path);
  return mccfr_set_hand_table(h, t.data(), t.size());
}

int mccfr_step(mccfr_handle* h, long long iteration, int player, int batch, mccfr_trace* trace) {
  if (!h || iteration < 1 || player < 0 || player >= h->cfg.num_players || batch < 1)
    return MCCFR_ERR_INVALID_ARG;
  if (!h->has_table) return fail(h, MCCFR_ERR_NO_HAND_TABLE, "load a hand-rank table first");
  if (trace && h->cfg.sampling != MCCFR_SAMPLING_REFERENCE)
    return fail(h, MCCFR_ERR_INVALID_ARG, "traces are recorded under reference sampling only");
  CK(cudaSetDevice(h->device));
  mccfr_trace* d_trace = nullptr;
  if (trace) {
    CK(cudaMalloc(&d_trace, (size_t)batch * sizeof(mccfr_trace)));
    CK(cudaMemsetAsync(d_trace, 0, (size_t)batch * sizeof(mccfr_trace), h->stream));
  }
  int rc = ensure_deals(h, batch);
  if (rc == MCCFR_OK && use_levels(h)) rc = ensure_levels(h, batch);
  if (rc == MCCFR_OK) rc = set_sched(h, iteration, player);
  if (rc == MCCFR_OK) rc = enqueue_update(h, batch, d_trace, h->ev);
  if (rc == MCCFR_OK) {
    const cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = fail(h, MCCFR_ERR_CUDA, "step: %s", cudaGetErrorString(e));
  }
  if (rc == MCCFR_OK) {
    float t1 = 0, t2 = 0;
    cudaEventElapsedTime(&t1, h->ev[0], h->ev[1]);
    cudaEventElapsedTime(&t2, h->ev[1], h->ev[2]);
    h->last_traverse_ms = t1;
    h->last_apply_ms = t2;
    h->traverse_ms += t1;
    h->apply_ms += t2;
    h->launches++;
    // the apply kernel resets the other parity's counters, not this one's
    read_touched(h, (uint32_t)((iteration - 1) * h->cfg.num_players + player) & 1);
    rc = check_device_error(h);
  }
  if (rc == MCCFR_OK && trace) {
    const cudaError_t e = cudaMemcpy(trace, d_trace, (size_t)batch * sizeof(mccfr_trace), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = fail(h, MCCFR_ERR_CUDA, "trace copy: %s", cudaGetErrorString(e));
  }
  if (d_trace) cudaFree(d_trace);
  return rc;
}

int mccfr_train(mccfr_handle* h, long long iters, int batch, int verbose, const char* ckpt_path,
                long long ckpt_interval) {
  if (!h || iters < 0 || batch < 1) return MCCFR_ERR_INVALID_ARG;
  if (!h->has_table) return fail(h, MCCFR_ERR_NO_HAND_TABLE, "load a hand-rank table first");
  if (iters == 0) return MCCFR_OK;
  CK(cudaSetDevice(h->device));
  int rc = ensure_graph(h, batch);
  if (rc) return rc;
  const long long base = h->iterations_done;  // iterations before this call
  rc = set_sched(h, base + 1, 0);
  if (rc) return rc;
  const bool timed = (verbose & 2) != 0;
  const auto t0 = std::chrono::steady_clock::now();
  for (long long i = 0; i < iters; ++i) {
    CK(cudaGraphLaunch(h->graph, h->stream));
    if (timed) {
      // event nodes inside the graph bracket every traverse and apply kernel
      const int np = h->cfg.num_players;
      CK(cudaEventSynchronize(h->gev[3 * (np - 1) + 2]));
      for (int p = 0; p < np; ++p) {
        float t1 = 0, t2 = 0;
        cudaEventElapsedTime(&t1, h->gev[3 * p], h->gev[3 * p + 1]);
        cudaEventElapsedTime(&t2, h->gev[3 * p + 1], h->gev[3 * p + 2]);
        h->traverse_ms += t1;
        h->apply_ms += t2;
        h->last_traverse_ms = t1;
        h->last_apply_ms = t2;
      }
      if (i + 1 == iters) {
        // rows touched by this iteration's last player-update (its parity's counter
        // is reset only by the next update's apply)
        if (read_touched(h, (uint32_t)((base + i) * np + np - 1) & 1)) return MCCFR_ERR_CUDA;
      }
    }
    h->launches += h->cfg.num_players;
    const long long it = base + i + 1;
    if ((verbose & 1) && (it % 100 == 0 || i + 1 == iters)) {
      CK(cudaStreamSynchronize(h->stream));
      const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      const double done = (double)(i + 1) * batch * h->cfg.num_players;
      printf("\r  %lld/%lld iters  %.1fM traversals/s  ", i + 1, iters, done / sec / 1e6);
      fflush(stdout);
    }
    if (ckpt_path && ckpt_path[0] && ckpt_interval > 0 && it % ckpt_interval == 0) {
      // the reference's layout for its own keys, v2 (with the iteration) otherwise
      CK(cudaStreamSynchronize(h->stream));
      h->iterations_done = it;
      rc = h->cfg.key_mode == MCCFR_KEY_FNV26 ? mccfr_save_checkpoint(h, ckpt_path)
                                              : mccfr_save_checkpoint_v2(h, ckpt_path);
      if (rc) return rc;
      rc = set_sched(h, it + 1, 0);
      if (rc) return rc;
    }
  }
  CK(cudaStreamSynchronize(h->stream));
  if (verbose & 1) printf("\n");
  h->iterations_done = base + iters;
  return check_device_error(h);
}

int mccfr_get_stats(mccfr_handle* h, mccfr_stats* out) {
  if (!h || !out) return MCCFR_ERR_INVALID_ARG;
  CK(cudaSetDevice(h->device));
  std::memset(out, 0, sizeof(*out));
  Counters c;
  CK(cudaMemcpyAsync(&c, h->d_counters, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  out->iterations_done = h->iterations_done;
  out->launches = h->launches;
  out->traversals = (int64_t)c.traversals;
  out->node_visits = (int64_t)c.visits;
  out->traverser_updates = (int64_t)c.updates;
  out->terminals = (int64_t)c.terminals;
  out->hand_evals = (int64_t)c.evals;
  out->table_capacity = (int64_t)h->cap;
  out->traverse_ms = h->traverse_ms;
  out->apply_ms = h->apply_ms;
  out->last_traverse_ms = h->last_traverse_ms;
  out->last_apply_ms = h->last_apply_ms;
  out->device_error = h->sticky_err;
  out->touched_last = h->touched_last;
  out->wide_rows_last = (int32_t)h->wide_last;
  out->rows_used = -1;  // filled by mccfr_export_rows callers; counting needs a table scan
  return MCCFR_OK;
}

int mccfr_table_digest(mccfr_handle* h, uint64_t* digest, uint64_t* rows) {
  if (!h || !digest) return MCCFR_ERR_INVALID_ARG;
  CK(cudaSetDevice(h->device));
  unsigned long long* d = nullptr;
  CK(cudaMalloc(&d, 2 * sizeof(unsigned long long)));
  unsigned long long out[2] = {0, 0};
  cudaError_t e = cudaMemsetAsync(d, 0, sizeof(out), h->stream);
  if (e == cudaSuccess) {
    k_digest<<<148 * 16, 256, 0, h->stream>>>(h->tv, h->cap, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, sizeof(out), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d);
  if (e != cudaSuccess) return fail(h, MCCFR_ERR_CUDA, "digest: %s", cudaGetErrorString(e));
  *digest = out[0];
  if (rows) *rows = out[1];
  return MCCFR_OK;
}

int mccfr_export_rows(mccfr_handle* h, uint64_t* keys, float* regrets, float* strategy_sum, uint64_t* visits,
                      size_t capacity, size_t* count) {
  if (!h || !count) return MCCFR_ERR_INVALID_ARG;
  CK(cudaSetDevice(h->device));
  if (capacity == 0) {  // size query: a counting pass only
    unsigned int n = 0;
    const int rc = count_rows(h, &n);
    *count = n;
    return rc ? rc : (n ? MCCFR_ERR_CAPACITY : MCCFR_OK);
  }
  std::vector<HostRow> rows;
  const int rc = read_rows(h, rows);
  if (rc) return rc;
  *count = rows.size();
  if (capacity < rows.size()) return MCCFR_ERR_CAPACITY;
  for (size_t i = 0; i < rows.size(); ++i) {
    if (keys) keys[i] = rows[i].key;
    if (regrets) std::memcpy(regrets + 8 * i, rows[i].reg, 32);
    if (strategy_sum) std::memcpy(strategy_sum + 8 * i, rows[i].ssum, 32);
    if (visits) visits[i] = rows[i].visits;
  }
  return MCCFR_OK;
}

// Average strategy (cfr_gpu.cu:1029-1058 normalisation, 1399-1411 host filter).
int mccfr_get_strategy(mccfr_handle* h, uint32_t* keys, uint64_t* keys64, float* probs, size_t capacity,
                       size_t* count) {
  if (!h || !count) return MCCFR_ERR_INVALID_ARG;
  CK(cudaSetDevice(h->device));
  if (capacity == 0) {  // size query: occupied rows, an upper bound of the rows written
    unsigned int n = 0;
    const int rc = count_rows(h, &n);
    *count = n;
    return rc ? rc : (n ? MCCFR_ERR_CAPACITY : MCCFR_OK);
  }
  std::vector<HostRow> rows;
  const int rc = read_rows(h, rows);
  if (rc) return rc;
  size_t n = 0;
  std::vector<std::pair<unsigned long long, std::array<float, 8>>> out;
  out.reserve(rows.size());
  for (const HostRow& r : rows) {
    float tot = 0.0f;
    for (int a = 0; a < 8; ++a) tot += r.ssum[a];
    std::array<float, 8> pr;
    for (int a = 0; a < 8; ++a) pr[a] = (tot > 1e-7f) ? r.ssum[a] / tot : 0.0f;
    float t2 = 0.0f;
    for (int a = 0; a < 8; ++a) t2 += pr[a];
    if (t2 < 1e-6f) continue;
    out.push_back({r.key, pr});
  }
  n = out.size();
  *count = n;
  if (capacity < n) return MCCFR_ERR_CAPACITY;
  for (size_t i = 0; i < n; ++i) {
    const unsigned long long k = out[i].first;
    if (keys) keys[i] = (h->cfg.key_mode == MCCFR_KEY_FNV26) ? (uint32_t)(k - 1) : (uint32_t)k;
    if (keys64) keys64[i] = k;
    if (probs) std::memcpy(probs + 8 * i, out[i].second.data(), 32);
  }
  return MCCFR_OK;
}

int mccfr_num_info_sets_active(mccfr_handle* h, long long* out) {
  if (!h || !out) return MCCFR_ERR_INVALID_ARG;
  std::vector<HostRow> rows;
  const int rc = read_rows(h, rows);
  if (rc) return rc;
  long long n = 0;
  for (const HostRow& r : rows)
    for (int a = 0; a < 8; ++a)
      if (r.ssum[a] > 0.f) {
        ++n;
        break;
      }
  *out = n;
  return MCCFR_OK;
}

int mccfr_export_tables(mccfr_handle* h, float* regrets, float* strategy_sum, size_t n) {
  if (!h || !regrets || !strategy_sum) return MCCFR_ERR_INVALID_ARG;
  if (h->cfg.key_mode != MCCFR_KEY_FNV26)
    return fail(h, MCCFR_ERR_INVALID_ARG, "dense tables exist for FNV26 keys only");
  const size_t need = 8ull * MCCFR_REF_TABLE_SIZE;
  if (n != need) return fail(h, MCCFR_ERR_INVALID_ARG, "expected n = %zu floats per table", need);
  CK(cudaSetDevice(h->device));
  float *dr = nullptr, *ds = nullptr;
  CK(cudaMalloc(&dr, need * 4));
  cudaError_t e = cudaMalloc(&ds, need * 4);
  int rc = MCCFR_OK;
  if (e != cudaSuccess) rc = fail(h, MCCFR_ERR_OOM, "dense export buffers");
  if (!rc) {
    cudaMemsetAsync(dr, 0, need * 4, h->stream);
    cudaMemsetAsync(ds, 0, need * 4, h->stream);
    k_export_dense<<<148 * 16, 256, 0, h->stream>>>(h->tv, h->cap, dr, ds, MCCFR_REF_TABLE_SIZE);
    e = cudaMemcpyAsync(regrets, dr, need * 4, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(strategy_sum, ds, need * 4, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = fail(h, MCCFR_ERR_CUDA, "dense export: %s", cudaGetErrorString(e));
  }
  cudaFree(dr);
  cudaFree(ds);
  return rc;
}

int mccfr_import_tables(mccfr_handle* h, const float* regrets, const float* strategy_sum, size_t n) {
  if (!h || !regrets || !strategy_sum) return MCCFR_ERR_INVALID_ARG;
  if (h->cfg.key_mode != MCCFR_KEY_FNV26)
    return fail(h, MCCFR_ERR_INVALID_ARG, "dense tables exist for FNV26 keys only");
  const size_t need = 8ull * MCCFR_REF_TABLE_SIZE;
  if (n != need) return fail(h, MCCFR_ERR_INVALID_ARG, "expected n = %zu floats per table", need);
  CK(cudaSetDevice(h->device));
  float *dr = nullptr, *ds = nullptr;
  CK(cudaMalloc(&dr, need * 4));
  cudaError_t e = cudaMalloc(&ds, need * 4);
  int rc = MCCFR_OK;
  if (e != cudaSuccess) rc = fail(h, MCCFR_ERR_OOM, "dense import buffers");
  if (!rc) {
    e = cudaMemcpyAsync(dr, regrets, need * 4, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ds, strategy_sum, need * 4, cudaMemcpyHostToDevice, h->stream);
    // The dense tables replace the table's contents, as the reference's load
    // overwrites both arrays (cfr_gpu.cu:1526-1527): rows are cleared first, then
    // every slot with a non-zero value becomes a row (an all-zero slot reads as
    // zeros either way).
    if (e == cudaSuccess) e = cudaMemsetAsync(h->d_block, 0, h->block_bytes, h->stream);
    if (e == cudaSuccess) {
      k_import_dense<<<148 * 16, 256, 0, h->stream>>>(h->tv, dr, ds, MCCFR_REF_TABLE_SIZE);
      e = cudaStreamSynchronize(h->stream);
    }
    if (e != cudaSuccess) rc = fail(h, MCCFR_ERR_CUDA, "dense import: %s", cudaGetErrorString(e));
  }
  cudaFree(dr);
  cudaFree(ds);
  if (!rc) {
    h->touched_last = 0;
    h->wide_last = 0;
    rc = check_device_error(h);
  }
  return rc;
}

int mccfr_save_checkpoint(mccfr_handle* h, const char* path) {
  if (!h || !path) return MCCFR_ERR_INVALID_ARG;
  const size_t n = 8ull * MCCFR_REF_TABLE_SIZE;
  std::vector<float> r(n), s(n);
  int rc = mccfr_export_tables(h, r.data(), s.data(), n);
  if (rc) return rc;
  FILE* f = fopen(path, "wb");
  if (!f) return fail(h, MCCFR_ERR_IO, "cannot open %s", path);
  const uint64_t magic = 0x43465247505500ULL;
  const uint32_t ts = MCCFR_REF_TABLE_SIZE, na = 8;
  bool ok = fwrite(&magic, 8, 1, f) == 1 && fwrite(&ts, 4, 1, f) == 1 && fwrite(&na, 4, 1, f) == 1 &&
            fwrite(r.data(), 4, n, f) == n && fwrite(s.data(), 4, n, f) == n;
  ok = (fclose(f) == 0) && ok;
  return ok ? MCCFR_OK : fail(h, MCCFR_ERR_IO, "write %s failed", path);
}

int mccfr_load_checkpoint(mccfr_handle* h, const char* path) {
  if (!h || !path) return MCCFR_ERR_INVALID_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) return fail(h, MCCFR_ERR_IO, "cannot open %s", path);
  uint64_t magic = 0;
  uint32_t ts = 0, na = 0;
  bool ok = fread(&magic, 8, 1, f) == 1 && fread(&ts, 4, 1, f) == 1 && fread(&na, 4, 1, f) == 1;
  if (!ok || magic != 0x43465247505500ULL || ts != (uint32_t)MCCFR_REF_TABLE_SIZE || na != 8) {
    fclose(f);
    return fail(h, MCCFR_ERR_FORMAT, "%s: not a checkpoint with table_size=2^26 and 8 actions", path);
  }
  const size_t n = 8ull * MCCFR_REF_TABLE_SIZE;
  std::vector<float> r(n), s(n);
  ok = fread(r.data(), 4, n, f) == n && fread(s.data(), 4, n, f) == n;
  fclose(f);
  if (!ok) return fail(h, MCCFR_ERR_FORMAT, "%s: truncated checkpoint", path);
  const int rc = mccfr_import_tables(h, r.data(), s.data(), n);
  if (rc) return rc;
  if (h->cfg.use_cfr_plus) {
    k_clamp_all<<<148 * 16, 256, 0, h->stream>>>(h->tv, h->cap);
    CK(cudaStreamSynchronize(h->stream));
  }
  return MCCFR_OK;
}

// ---- v2 checkpoint (any key mode) -------------------------------------------
// [u64 "MCCFRCK2"][u32 2][u32 sizeof(mccfr_config)][mccfr_config]
// [i64 iterations done][u64 rows] rows x {u64 key, f32 regrets[8],
// f32 strategy_sum[8], u64 visits}, keys ascending.  The reference's checkpoint
// (cfr_gpu.cu:1464-1538) keeps neither the iteration nor the seed, so linear-CFR
// weights restart at t = 1 after its resume; with both kept and counter-based
// draws, training resumed from this file equals uninterrupted training.
namespace {
constexpr uint64_t kCkptV2Magic = 0x324B43524643434DULL;  // "MCCFRCK2" little-endian

// The fields that define the game and its abstraction: all but the device, the
// table capacity and the traversal form (every form gives the same tables).
bool same_game(mccfr_config a, mccfr_config b) {
  a.device = b.device = 0;
  a.table_log2 = b.table_log2 = 0;
  a.traversal_form = b.traversal_form = 0;
  a.level_log2 = b.level_log2 = 0;
  std::memset(a.reserved, 0, sizeof(a.reserved));
  std::memset(b.reserved, 0, sizeof(b.reserved));
  return std::memcmp(&a, &b, sizeof(a)) == 0;
}
}  // namespace

int mccfr_save_checkpoint_v2(mccfr_handle* h, const char* path) {
  if (!h || !path) return MCCFR_ERR_INVALID_ARG;
  CK(cudaSetDevice(h->device));
  std::vector<HostRow> rows;
  const int rc = read_rows(h, rows);
  if (rc) return rc;
  FILE* f = fopen(path, "wb");
  if (!f) return fail(h, MCCFR_ERR_IO, "cannot open %s", path);
  const uint32_t ver = 2, cfg_bytes = sizeof(mccfr_config);
  const int64_t iters = h->iterations_done;
  const uint64_t n = rows.size();
  bool ok = fwrite(&kCkptV2Magic, 8, 1, f) == 1 && fwrite(&ver, 4, 1, f) == 1 && fwrite(&cfg_bytes, 4, 1, f) == 1 &&
            fwrite(&h->cfg, sizeof(mccfr_config), 1, f) == 1 && fwrite(&iters, 8, 1, f) == 1 &&
            fwrite(&n, 8, 1, f) == 1 && (n == 0 || fwrite(rows.data(), sizeof(HostRow), n, f) == n);
  ok = (fclose(f) == 0) && ok;
  return ok ? MCCFR_OK : fail(h, MCCFR_ERR_IO, "write %s failed", path);
}

int mccfr_load_checkpoint_v2(mccfr_handle* h, const char* path) {
  if (!h || !path) return MCCFR_ERR_INVALID_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) return fail(h, MCCFR_ERR_IO, "cannot open %s", path);
  uint64_t magic = 0, n = 0;
  uint32_t ver = 0, cfg_bytes = 0;
  int64_t iters = 0;
  mccfr_config saved{};
  bool ok = fread(&magic, 8, 1, f) == 1 && fread(&ver, 4, 1, f) == 1 && fread(&cfg_bytes, 4, 1, f) == 1 &&
            magic == kCkptV2Magic && ver == 2 && cfg_bytes == sizeof(mccfr_config) &&
            fread(&saved, sizeof(saved), 1, f) == 1 && fread(&iters, 8, 1, f) == 1 && fread(&n, 8, 1, f) == 1;
  if (!ok) {
    fclose(f);
    return fail(h, MCCFR_ERR_FORMAT, "%s: not a v2 checkpoint", path);
  }
  if (!same_game(saved, h->cfg)) {
    fclose(f);
    return fail(h, MCCFR_ERR_INVALID_ARG, "%s: written for a different game or abstraction", path);
  }
  if (iters < 0 || n > h->cap) {
    fclose(f);
    return fail(h, MCCFR_ERR_FORMAT, "%s: %llu rows for a %llu-row table", path, (unsigned long long)n, h->cap);
  }
  std::vector<HostRow> rows(n);
  ok = n == 0 || fread(rows.data(), sizeof(HostRow), n, f) == n;
  fclose(f);
  if (!ok) return fail(h, MCCFR_ERR_FORMAT, "%s: truncated checkpoint", path);
  // Keys must be nonzero, ascending and, in a direct-mapped table, at most the
  // key space (row key-1 must exist): checked here, before any device write.
  const int kb = h->cfg.key_mode == MCCFR_KEY_FNV26 ? 26 : h->cfg.key_bits;
  const unsigned long long kmax = h->tv.direct ? (1ull << kb) : ~0ull;
  for (uint64_t i = 0; i < n; ++i)
    if (rows[i].key == 0 || rows[i].key > kmax || (i && rows[i].key <= rows[i - 1].key))
      return fail(h, MCCFR_ERR_FORMAT, "%s: row %llu has an invalid key", path, (unsigned long long)i);
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaMemsetAsync(h->d_block, 0, h->block_bytes, h->stream));  // rows, touched list, counters
  int rc = MCCFR_OK;
  if (n) {
    std::vector<unsigned long long> keys(n), vis(n);
    std::vector<float> reg(8 * n), ssum(8 * n);
    for (uint64_t i = 0; i < n; ++i) {
      keys[i] = rows[i].key;
      vis[i] = rows[i].visits;
      std::memcpy(&reg[8 * i], rows[i].reg, 32);
      std::memcpy(&ssum[8 * i], rows[i].ssum, 32);
    }
    void* block = nullptr;
    cudaError_t e = cudaMalloc(&block, n * 80);
    if (e != cudaSuccess) return fail(h, MCCFR_ERR_OOM, "checkpoint upload buffers");
    char* base = static_cast<char*>(block);
    float4* d_reg = reinterpret_cast<float4*>(base);
    float4* d_ssum = reinterpret_cast<float4*>(base + n * 32);
    unsigned long long* d_keys = reinterpret_cast<unsigned long long*>(base + n * 64);
    unsigned long long* d_vis = reinterpret_cast<unsigned long long*>(base + n * 72);
    e = cudaMemcpyAsync(d_reg, reg.data(), n * 32, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ssum, ssum.data(), n * 32, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_keys, keys.data(), n * 8, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_vis, vis.data(), n * 8, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
      k_import_rows<<<148 * 16, 256, 0, h->stream>>>(h->tv, d_keys, d_reg, d_ssum, d_vis, n);
      e = cudaStreamSynchronize(h->stream);
    }
    cudaFree(block);
    if (e != cudaSuccess) rc = fail(h, MCCFR_ERR_CUDA, "checkpoint import: %s", cudaGetErrorString(e));
  }
  if (!rc) rc = check_device_error(h);
  if (!rc) {
    h->iterations_done = iters;
    h->touched_last = 0;
    h->wide_last = 0;
  }
  return rc;
}

// Strategy dump v2 (strategy.cpp:6-8, 35-52), rows sorted by key.
int mccfr_save_strategy(mccfr_handle* h, const char* path) {
  if (!h || !path) return MCCFR_ERR_INVALID_ARG;
  size_t n = 0;
  int rc = mccfr_get_strategy(h, nullptr, nullptr, nullptr, 0, &n);
  if (rc && rc != MCCFR_ERR_CAPACITY) return rc;
  std::vector<uint32_t> k(n);
  std::vector<float> p(8 * n);
  rc = mccfr_get_strategy(h, k.data(), nullptr, p.data(), n, &n);
  if (rc) return rc;
  FILE* f = fopen(path, "wb");
  if (!f) return fail(h, MCCFR_ERR_IO, "cannot open %s", path);
  const uint64_t magic = 0x53545241540100ULL;
  const uint32_t ts = MCCFR_REF_TABLE_SIZE, na = 8, cnt = (uint32_t)n;
  bool ok = fwrite(&magic, 8, 1, f) == 1 && fwrite(&ts, 4, 1, f) == 1 && fwrite(&na, 4, 1, f) == 1 &&
            fwrite(&cnt, 4, 1, f) == 1;
  for (size_t i = 0; i < n && ok; ++i) ok = fwrite(&k[i], 4, 1, f) == 1 && fwrite(&p[8 * i], 4, 8, f) == 8;
  ok = (fclose(f) == 0) && ok;
  return ok ? MCCFR_OK : fail(h, MCCFR_ERR_IO, "write %s failed", path);
}

int mccfr_eval7_device(mccfr_handle* h, const uint8_t* dev_cards, uint16_t* dev_ranks, size_t n, float* ms) {
  if (!h || !dev_cards || !dev_ranks) return MCCFR_ERR_INVALID_ARG;
  if (!h->has_table) return fail(h, MCCFR_ERR_NO_HAND_TABLE, "load a hand-rank table first");
  CK(cudaSetDevice(h->device));
  CK(cudaEventRecord(h->ev[0], h->stream));
  if (n) k_eval7<<<grid_for((long long)n, 256), 256, 0, h->stream>>>(h->d_hr, dev_cards, dev_ranks, n);
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ev[1], h->stream));
  CK(cudaEventSynchronize(h->ev[1]));
  if (ms) cudaEventElapsedTime(ms, h->ev[0], h->ev[1]);
  return MCCFR_OK;
}

int mccfr_eval7(mccfr_handle* h, const uint8_t* cards, uint16_t* ranks, size_t n) {
  if (!h || !cards || !ranks) return MCCFR_ERR_INVALID_ARG;
  if (!h->has_table) return fail(h, MCCFR_ERR_NO_HAND_TABLE, "load a hand-rank table first");
  if (n == 0) return MCCFR_OK;
  for (size_t i = 0; i < 7 * n; ++i)
    if (cards[i] > 51) return fail(h, MCCFR_ERR_INVALID_ARG, "card code %d out of range", (int)cards[i]);
  CK(cudaSetDevice(h->device));
  uint8_t* dc = nullptr;
  uint16_t* dr = nullptr;
  CK(cudaMalloc(&dc, 7 * n));
  cudaError_t e = cudaMalloc(&dr, 2 * n);
  int rc = MCCFR_OK;
  if (e == cudaSuccess) e = cudaMemcpyAsync(dc, cards, 7 * n, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) rc = mccfr_eval7_device(h, dc, dr, n, nullptr);
  if (e == cudaSuccess && !rc) e = cudaMemcpy(ranks, dr, 2 * n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) rc = fail(h, MCCFR_ERR_CUDA, "eval7: %s", cudaGetErrorString(e));
  cudaFree(dc);
  cudaFree(dr);
  return rc;
}

int mccfr_level_counts(mccfr_handle* h, uint32_t* seeds, uint32_t* nodes, int cap, int* levels,
                       uint32_t* deferred) {
  if (!h || !levels || cap < 0 || (cap && (!seeds || !nodes))) return MCCFR_ERR_INVALID_ARG;
  *levels = 0;
  if (deferred) *deferred = 0;
  if (!h->d_level) return MCCFR_OK;
  CK(cudaSetDevice(h->device));
  static thread_local LevelCtl c;
  CK(cudaMemcpyAsync(&c, h->lb.ctl, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  *levels = h->lb.nlev;
  for (int L = 0; L < h->lb.nlev && L < cap; ++L) {
    seeds[L] = L == 0 ? (uint32_t)h->level_last_batch : level_seeds(c, L);
    nodes[L] = level_nodes(c, L);
  }
  if (deferred) *deferred = c.deferred;
  return MCCFR_OK;
}

int mccfr_deal_eval7(mccfr_handle* h, uint32_t stream, size_t n, uint16_t* dev_ranks, float* ms) {
  if (!h || (n && !dev_ranks)) return MCCFR_ERR_INVALID_ARG;
  if (!h->has_table) return fail(h, MCCFR_ERR_NO_HAND_TABLE, "load a hand-rank table first");
  CK(cudaSetDevice(h->device));
  CK(cudaEventRecord(h->ev[0], h->stream));
  if (n)
    k_deal_eval7<256><<<grid_for((long long)n, 256), 256, 0, h->stream>>>(h->d_hr, h->gp.seed_lo, h->gp.seed_hi,
                                                                         stream, n, dev_ranks);
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ev[1], h->stream));
  CK(cudaEventSynchronize(h->ev[1]));
  if (ms) cudaEventElapsedTime(ms, h->ev[0], h->ev[1]);
  return MCCFR_OK;
}

int mccfr_showdown_masks(mccfr_handle* h, long long iteration, int player, size_t n, uint8_t* dev_masks,
                         float* ms) {
  if (!h || iteration < 1 || player < 0 || player >= h->cfg.num_players || (n && !dev_masks) ||
      n > 0xFFFFFFFFull)
    return MCCFR_ERR_INVALID_ARG;
  if (h->gp.sub_street) return fail(h, MCCFR_ERR_INVALID_ARG, "showdown masks are defined for the full game");
  if (!h->has_table) return fail(h, MCCFR_ERR_NO_HAND_TABLE, "load a hand-rank table first");
  CK(cudaSetDevice(h->device));
  const uint32_t uid = (uint32_t)((iteration - 1) * h->cfg.num_players + player);
  CK(cudaEventRecord(h->ev[0], h->stream));
  if (n)
    k_showdown_masks<256><<<grid_for((long long)n, 256), 256, 0, h->stream>>>(h->gp, h->d_hr, uid, (unsigned)n,
                                                                             dev_masks);
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ev[1], h->stream));
  CK(cudaEventSynchronize(h->ev[1]));
  if (ms) cudaEventElapsedTime(ms, h->ev[0], h->ev[1]);
  return MCCFR_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched form: many tables in one persistent kernel.
// ---------------------------------------------------------------------------
struct mccfr_batch {
  std::vector<mccfr_handle*> tables;
  std::vector<int> traversals;
  int device = 0;
  int max_players = 0;
  cudaStream_t stream = nullptr;
  TableDesc* d_tables = nullptr;
  PhaseDesc* d_phases = nullptr;
  std::vector<PhaseDesc> phases;
  std::vector<PhaseParams> params;  // by-value descriptors of each phase's traversal launch
  DealRec* d_deals = nullptr;
  unsigned long long* d_work = nullptr;
  unsigned long long max_items = 0;
  mccfr_batch_tuning tuning{128, 2, 0, 1, 1, MCCFR_BATCH_TABLE_GRAPHS, {0, 0}};  // until set or autotuned
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t ev_fork = nullptr;       // table-graph form: fork and joins of the tables' branches
  std::vector<cudaEvent_t> ev_join;
  cudaEvent_t ev_it[2] = {nullptr, nullptr};
  cudaEvent_t ev_ph[2 * MCCFR_MAX_PLAYERS] = {};
  long long iterations = 0;
  double traverse_ms = 0, total_ms = 0;
  std::string last_error;
};

namespace {

int bfail(mccfr_batch* b, int code, const char* msg) {
  if (b) b->last_error = msg;
  fprintf(stderr, "mccfr_batch: %s\n", msg);
  return code;
}

#define BCK(call)                                                                        \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) return bfail(b, e_ == cudaErrorMemoryAllocation ? MCCFR_ERR_OOM : MCCFR_ERR_CUDA, \
                                        cudaGetErrorString(e_));                          \
  } while (0)

using BatchedKernel = void (*)(const PhaseParams, const DealRec*, unsigned long long*, int, int);

template <int B, int K, int W>
BatchedKernel pick3() {
  return k_traverse_batched<B, K, W>;
}
template <int B, int K>
BatchedKernel pick2(int w) {
  return w == 2 ? pick3<B, K, 2>() : pick3<B, K, 1>();
}
template <int B>
BatchedKernel pick1(int k, int w) {
  return k == 4 ? pick2<B, 4>(w) : k == 2 ? pick2<B, 2>(w) : pick2<B, 0>(w);
}
BatchedKernel pick_kernel(const mccfr_batch_tuning& t) {
  return t.block == 64 ? pick1<64>(t.smem_frames, t.probe_width)
         : t.block == 256 ? pick1<256>(t.smem_frames, t.probe_width)
                          : pick1<128>(t.smem_frames, t.probe_width);
}

bool valid_tuning(const mccfr_batch_tuning& t) {
  return (t.block == 64 || t.block == 128 || t.block == 256) && (t.grab == 1 || t.grab == 2 || t.grab == 4 || t.grab == 8) &&
         (t.smem_frames == 0 || t.smem_frames == 2 || t.smem_frames == 4) && (t.probe_width == 1 || t.probe_width == 2) &&
         (t.warp_sync == 0 || t.warp_sync == 1) && (t.form == MCCFR_BATCH_PERSISTENT || t.form == MCCFR_BATCH_TABLE_GRAPHS);
}

size_t batched_smem(const mccfr_batch_tuning& t) {
  return (size_t)t.smem_frames * t.block * sizeof(EsFrame);
}

// Enqueues one iteration: every phase's deal, persistent traversal, apply, advance.
int batch_enqueue_iteration(mccfr_batch* b, bool capturing) {
  const mccfr_batch_tuning& t = b->tuning;
  BatchedKernel kern = pick_kernel(t);
  const size_t smem = batched_smem(t);
  BCK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  BCK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                           t.smem_frames ? (int)cudaSharedmemCarveoutDefault : 0));
  int per_sm = 0;
  BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, t.block, smem));
  cudaDeviceProp prop;
  BCK(cudaGetDeviceProperties(&prop, b->device));
  const int grid = std::max(1, per_sm) * prop.multiProcessorCount;
  const int32_t* T = b->tables[0]->d_hr;
  auto rec = [&](cudaEvent_t e) {
    return capturing ? cudaEventRecordWithFlags(e, b->stream, cudaEventRecordExternal) : cudaEventRecord(e, b->stream);
  };
  BCK(rec(b->ev_it[0]));
  for (int p = 0; p < b->max_players; ++p) {
    const PhaseDesc& P = b->phases[p];
    const unsigned long long items = P.off[P.n];
    BCK(cudaMemsetAsync(b->d_work + p, 0, sizeof(unsigned long long), b->stream));
    const int dgrid = (int)std::min<unsigned long long>((items + 127) / 128, 148ull * 64);
    k_deal_batched<<<std::max(1, dgrid), 128, 0, b->stream>>>(b->d_tables, b->d_phases + p, T, b->d_deals);
    BCK(cudaGetLastError());
    BCK(rec(b->ev_ph[2 * p]));
    kern<<<grid, t.block, smem, b->stream>>>(b->params[p], b->d_deals, b->d_work + p, t.grab, t.warp_sync);
    BCK(cudaGetLastError());
    BCK(rec(b->ev_ph[2 * p + 1]));
    k_apply_batched<<<dim3(148 * 2, P.n), 256, 0, b->stream>>>(b->d_tables, b->d_phases + p);
    BCK(cudaGetLastError());
    k_advance_batched<<<1, 64, 0, b->stream>>>(b->d_tables, b->d_phases + p);
    BCK(cudaGetLastError());
  }
  BCK(rec(b->ev_it[1]));
  return MCCFR_OK;
}

// One iteration of every table, each on its own stream: the batch stream
// forks into one branch per table (its N player-updates, as its own training
// graph holds them) and joins them again, so that a capture of this is one
// graph whose branches the device runs concurrently.  Buffers are sized first:
// nothing may allocate while the stream is captured.
int batch_enqueue_table_graphs(mccfr_batch* b, bool capturing) {
  auto rec = [&](cudaEvent_t e, cudaStream_t s) {
    return capturing ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal) : cudaEventRecord(e, s);
  };
  BCK(rec(b->ev_it[0], b->stream));
  BCK(cudaEventRecord(b->ev_fork, b->stream));
  for (size_t i = 0; i < b->tables.size(); ++i) {
    mccfr_handle* h = b->tables[i];
    BCK(cudaStreamWaitEvent(h->stream, b->ev_fork, 0));
    for (int p = 0; p < h->cfg.num_players; ++p) {
      const int rc = enqueue_update(h, b->traversals[i], nullptr, nullptr, capturing);
      if (rc) return bfail(b, rc, "table update in the batch graph");
      k_advance<<<1, 1, 0, h->stream>>>(h->d_sched, h->cfg.num_players);
      BCK(cudaGetLastError());
    }
    BCK(cudaEventRecord(b->ev_join[i], h->stream));
    BCK(cudaStreamWaitEvent(b->stream, b->ev_join[i], 0));
  }
  BCK(rec(b->ev_it[1], b->stream));
  return MCCFR_OK;
}

int batch_prepare_table_graphs(mccfr_batch* b) {
  if (!b->ev_fork) BCK(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
  while (b->ev_join.size() < b->tables.size()) {
    cudaEvent_t e = nullptr;
    BCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ev_join.push_back(e);
  }
  for (size_t i = 0; i < b->tables.size(); ++i) {
    mccfr_handle* h = b->tables[i];
    int rc = ensure_deals(h, b->traversals[i]);
    if (!rc && use_levels(h)) rc = ensure_levels(h, b->traversals[i]);
    if (rc) return bfail(b, rc, "table buffers for the batch graph");
  }
  return MCCFR_OK;
}

int batch_set_scheds(mccfr_batch* b) {
  for (mccfr_handle* h : b->tables) {
    h->h_sched->iteration = h->iterations_done + 1;
    h->h_sched->player = 0;
    h->h_sched->pad = 0;
    BCK(cudaMemcpyAsync(h->d_sched, h->h_sched, sizeof(Sched), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));  // pinned staging is reused by the next table
  }
  return MCCFR_OK;
}

int batch_after(mccfr_batch* b, long long iters) {
  BCK(cudaStreamSynchronize(b->stream));
  int worst = MCCFR_OK;
  for (mccfr_handle* h : b->tables) {
    h->iterations_done += iters;
    h->launches += iters * h->cfg.num_players;
    const int rc = check_device_error(h);
    if (rc && !worst) worst = rc;
  }
  b->iterations += iters;
  return worst;
}

void batch_time_phases(mccfr_batch* b) {
  float ms = 0;
  for (int p = 0; p < b->max_players; ++p)
    if (cudaEventElapsedTime(&ms, b->ev_ph[2 * p], b->ev_ph[2 * p + 1]) == cudaSuccess) b->traverse_ms += ms;
  if (cudaEventElapsedTime(&ms, b->ev_it[0], b->ev_it[1]) == cudaSuccess) b->total_ms += ms;
}

}  // namespace

extern "C" {

int mccfr_batch_create(mccfr_handle* const* tables, int n, const int* traversals, mccfr_batch** out) {
  if (!tables || !traversals || !out || n < 1 || n > kMaxBatchTables) return MCCFR_ERR_INVALID_ARG;
  *out = nullptr;
  mccfr_batch* b = new mccfr_batch();
  auto bad = [&](int rc, const char* why) {
    bfail(b, rc, why);
    mccfr_batch_destroy(b);
    return rc;
  };
  b->device = tables[0]->device;
  for (int i = 0; i < n; ++i) {
    mccfr_handle* h = tables[i];
    if (!h || traversals[i] < 1) return bad(MCCFR_ERR_INVALID_ARG, "null table or traversal count < 1");
    if (h->device != b->device) return bad(MCCFR_ERR_INVALID_ARG, "tables on different devices");
    if (!h->has_table) return bad(MCCFR_ERR_NO_HAND_TABLE, "a table has no rank table loaded");
    if (h->cfg.sampling != MCCFR_SAMPLING_EXTERNAL) return bad(MCCFR_ERR_INVALID_ARG, "batched tables use external sampling");
    for (mccfr_handle* o : b->tables)
      if (o == h) return bad(MCCFR_ERR_INVALID_ARG, "a table appears twice in the batch");
    b->tables.push_back(h);
    b->traversals.push_back(traversals[i]);
    b->max_players = std::max(b->max_players, h->cfg.num_players);
  }
  if (cudaSetDevice(b->device) != cudaSuccess) return bad(MCCFR_ERR_CUDA, "cudaSetDevice");
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return bad(MCCFR_ERR_CUDA, "stream");
  for (auto& e : b->ev_it)
    if (cudaEventCreate(&e) != cudaSuccess) return bad(MCCFR_ERR_CUDA, "event");
  for (auto& e : b->ev_ph)
    if (cudaEventCreate(&e) != cudaSuccess) return bad(MCCFR_ERR_CUDA, "event");
  std::vector<TableDesc> descs(n);
  for (int i = 0; i < n; ++i) {
    mccfr_handle* h = tables[i];
    TableDesc& d = descs[i];
    std::memset(&d, 0, sizeof(d));
    d.G = h->gp;
    d.tv = h->tv;
    d.pre = h->d_pre;
    d.cdf = h->d_cdf;
    d.sched = h->d_sched;
    d.counters = h->d_counters;
    const int rb = regret_frac_bits(h->cfg, traversals[i]);
    d.rscale = std::ldexp(1.0f, rb);
    d.rinv = std::ldexp(1.0, -rb);
    d.batch = traversals[i];
  }
  b->phases.resize(b->max_players);
  for (int p = 0; p < b->max_players; ++p) {
    PhaseDesc& P = b->phases[p];
    std::memset(&P, 0, sizeof(P));
    unsigned long long off = 0;
    for (int i = 0; i < n; ++i) {
      if (tables[i]->cfg.num_players <= p) continue;
      P.table[P.n] = i;
      P.off[P.n] = off;
      off += (unsigned long long)traversals[i];
      P.n++;
    }
    P.off[P.n] = off;
    b->max_items = std::max(b->max_items, off);
  }
  b->params.resize(b->max_players);
  for (int p = 0; p < b->max_players; ++p) {
    PhaseParams& Q = b->params[p];
    std::memset(&Q, 0, sizeof(Q));
    Q.n = b->phases[p].n;
    for (int j = 0; j <= Q.n; ++j) Q.off[j] = b->phases[p].off[j];
    for (int j = 0; j < Q.n; ++j) Q.T[j] = descs[b->phases[p].table[j]];
  }
  if (cudaMalloc(&b->d_tables, n * sizeof(TableDesc)) != cudaSuccess ||
      cudaMalloc(&b->d_phases, b->max_players * sizeof(PhaseDesc)) != cudaSuccess ||
      cudaMalloc(&b->d_work, b->max_players * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&b->d_deals, b->max_items * sizeof(DealRec)) != cudaSuccess)
    return bad(MCCFR_ERR_OOM, "batch buffers");
  if (cudaMemcpy(b->d_tables, descs.data(), n * sizeof(TableDesc), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->d_phases, b->phases.data(), b->max_players * sizeof(PhaseDesc), cudaMemcpyHostToDevice) !=
          cudaSuccess)
    return bad(MCCFR_ERR_CUDA, "batch upload");
  *out = b;
  return MCCFR_OK;
}

void mccfr_batch_destroy(mccfr_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  for (auto& e : b->ev_join)
    if (e) cudaEventDestroy(e);
  for (auto& e : b->ev_it)
    if (e) cudaEventDestroy(e);
  for (auto& e : b->ev_ph)
    if (e) cudaEventDestroy(e);
  cudaFree(b->d_tables);
  cudaFree(b->d_phases);
  cudaFree(b->d_work);
  cudaFree(b->d_deals);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int mccfr_batch_set_tuning(mccfr_batch* b, const mccfr_batch_tuning* t) {
  if (!b || !t || !valid_tuning(*t)) return MCCFR_ERR_INVALID_ARG;
  b->tuning = *t;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return MCCFR_OK;
}

int mccfr_batch_get_tuning(mccfr_batch* b, mccfr_batch_tuning* t) {
  if (!b || !t) return MCCFR_ERR_INVALID_ARG;
  *t = b->tuning;
  return MCCFR_OK;
}

int mccfr_batch_train(mccfr_batch* b, long long iters, int flags) {
  if (!b || iters < 0) return MCCFR_ERR_INVALID_ARG;
  if (iters == 0) return MCCFR_OK;
  BCK(cudaSetDevice(b->device));
  int rc = batch_set_scheds(b);
  if (rc) return rc;
  const bool tgraphs = b->tuning.form == MCCFR_BATCH_TABLE_GRAPHS;
  if (!b->graph && tgraphs) {
    rc = batch_prepare_table_graphs(b);
    if (rc) return rc;
    BCK(cudaStreamSynchronize(b->stream));
  }
  if (!b->graph) {
    cudaGraph_t g = nullptr;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    rc = tgraphs ? batch_enqueue_table_graphs(b, true) : batch_enqueue_iteration(b, true);
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return bfail(b, MCCFR_ERR_CUDA, "batch graph capture");
    const cudaError_t e2 = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) return bfail(b, MCCFR_ERR_CUDA, "batch graph instantiate");
  }
  const bool timed = (flags & 2) != 0;
  for (long long i = 0; i < iters; ++i) {
    BCK(cudaGraphLaunch(b->graph, b->stream));
    if (timed) {
      BCK(cudaEventSynchronize(b->ev_it[1]));
      if (tgraphs) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, b->ev_it[0], b->ev_it[1]) == cudaSuccess) b->total_ms += ms;
      } else {
        batch_time_phases(b);
      }
    }
  }
  return batch_after(b, iters);
}

int mccfr_batch_autotune(mccfr_batch* b, int max_candidates, mccfr_batch_tuning* best) {
  if (!b) return MCCFR_ERR_INVALID_ARG;
  BCK(cudaSetDevice(b->device));
  std::vector<mccfr_batch_tuning> cands;
  // most informative dimensions first: a prefix of the list is a useful sweep
  for (int blk : {128, 64, 256})
    for (int grab : {1, 2, 4, 8})
      for (int k : {0, 2, 4})
        for (int ws : {1, 0})
          for (int w : {1, 2}) cands.push_back(mccfr_batch_tuning{blk, grab, k, w, ws, MCCFR_BATCH_PERSISTENT, {0, 0}});
  if (max_candidates > 0 && (int)cands.size() > max_candidates) cands.resize(max_candidates);
  // Candidates run on successive real iterations, whose trees change as the
  // strategy sharpens; each is ranked by traversal-kernel time per node visit,
  // summed over a forward and a backward pass through the list so that a
  // steady drift from one iteration to the next weighs on every candidate alike.
  auto visits_now = [&]() {
    unsigned long long v = 0;
    for (mccfr_handle* h : b->tables) {
      Counters c;
      if (cudaMemcpy(&c, h->d_counters, sizeof(c), cudaMemcpyDeviceToHost) == cudaSuccess) v += c.visits;
    }
    return v;
  };
  std::vector<double> cost(cands.size(), 0.0);
  const int nc = (int)cands.size();
  for (int pass = 0; pass < 2 * nc; ++pass) {
    const int ci = pass < nc ? pass : 2 * nc - 1 - pass;
    b->tuning = cands[ci];
    const unsigned long long v0 = visits_now();
    int rc = batch_set_scheds(b);
    if (rc) return rc;
    rc = batch_enqueue_iteration(b, false);
    if (rc) return rc;
    BCK(cudaEventSynchronize(b->ev_it[1]));
    float it_ms = 0;
    double trav = 0;
    for (int p = 0; p < b->max_players; ++p) {
      float ms = 0;
      cudaEventElapsedTime(&ms, b->ev_ph[2 * p], b->ev_ph[2 * p + 1]);
      trav += ms;
    }
    cudaEventElapsedTime(&it_ms, b->ev_it[0], b->ev_it[1]);
    b->traverse_ms += trav;
    b->total_ms += it_ms;
    rc = batch_after(b, 1);
    if (rc) return rc;
    cost[ci] += trav / (double)std::max(1ull, visits_now() - v0);
  }
  mccfr_batch_tuning best_t = cands[0];
  double best_cost = cost[0];
  for (int i = 1; i < nc; ++i)
    if (cost[i] < best_cost) {
      best_cost = cost[i];
      best_t = cands[i];
    }
  b->tuning = best_t;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  if (best) *best = best_t;
  return MCCFR_OK;
}

int mccfr_batch_get_stats(mccfr_batch* b, mccfr_batch_stats* out) {
  if (!b || !out) return MCCFR_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof(*out));
  BCK(cudaSetDevice(b->device));
  BCK(cudaStreamSynchronize(b->stream));
  for (mccfr_handle* h : b->tables) {
    Counters c;
    BCK(cudaMemcpy(&c, h->d_counters, sizeof(c), cudaMemcpyDeviceToHost));
    out->traversals += (int64_t)c.traversals;
    out->node_visits += (int64_t)c.visits;
  }
  out->iterations = b->iterations;
  out->traverse_ms = b->traverse_ms;
  out->total_ms = b->total_ms;
  return MCCFR_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Subgames and continuous batching.
// ---------------------------------------------------------------------------
namespace {

struct RoundCtx {
  int device = -1;
  cudaStream_t stream = nullptr;
  TableDesc* d_tables = nullptr;
  PhaseDesc* d_phase = nullptr;
  DealRec* d_deals = nullptr;
  unsigned long long* d_work = nullptr;
  size_t deals_cap = 0;
  int* h_err = nullptr;  // pinned: the tables' error flags after a round
  PhaseParams params;
};

RoundCtx g_round[64];
std::mutex g_round_mu;

// Range CDF on the 2^31 scale: combos that use a board card weigh 0; the last
// combo of positive weight ends at exactly 2^31.
bool build_range_cdf(const float* w, uint64_t board_mask, uint32_t* out) {
  double total = 0.0;
  for (int c = 0; c < 1326; ++c) {
    int hi = 1;
    while ((hi + 1) * hi / 2 <= c) ++hi;
    const int lo = c - hi * (hi - 1) / 2;
    const bool blocked = ((board_mask >> lo) & 1) || ((board_mask >> hi) & 1);
    const double x = (!blocked && w[c] > 0.0f) ? (double)w[c] : 0.0;
    total += x;
  }
  if (!(total > 0.0)) return false;
  double cum = 0.0;
  int last = -1;
  for (int c = 0; c < 1326; ++c) {
    int hi = 1;
    while ((hi + 1) * hi / 2 <= c) ++hi;
    const int lo = c - hi * (hi - 1) / 2;
    const bool blocked = ((board_mask >> lo) & 1) || ((board_mask >> hi) & 1);
    const double x = (!blocked && w[c] > 0.0f) ? (double)w[c] : 0.0;
    cum += x;
    if (x > 0.0) last = c;
    double v = std::floor(cum / total * 2147483648.0);
    if (v > 2147483648.0) v = 2147483648.0;
    out[c] = (uint32_t)v;
  }
  for (int c = last; c < 1326; ++c) out[c] = 2147483648u;
  return true;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// Checks a subgame against its config and builds each player's range CDF.
int subgame_cdfs(const mccfr_config* cfg, const mccfr_subgame* sg, std::vector<uint32_t>& cdf, int& nb) {
  if (!cfg || !sg || !sg->ranges) return MCCFR_ERR_INVALID_ARG;
  if (cfg->key_mode != MCCFR_KEY_ID64) {
    fprintf(stderr, "subgame: subgames use ID64 keys\n");
    return MCCFR_ERR_INVALID_ARG;
  }
  if (sg->street != 2 && sg->street != 3) return MCCFR_ERR_INVALID_ARG;
  if (cfg->num_players < 2 || cfg->num_players > MCCFR_MAX_PLAYERS) return MCCFR_ERR_INVALID_ARG;
  nb = sg->street == 2 ? 4 : 5;
  uint64_t mask = 0;
  for (int i = 0; i < nb; ++i) {
    if (sg->board[i] > 51 || ((mask >> sg->board[i]) & 1)) return MCCFR_ERR_INVALID_ARG;
    mask |= 1ull << sg->board[i];
  }
  // invested chips are 16-bit: a player's pot share plus its whole stack must fit
  if (sg->pot < 0 || sg->pot % cfg->num_players != 0 || sg->pot / cfg->num_players + cfg->starting_stack > 65535)
    return MCCFR_ERR_INVALID_ARG;
  cdf.assign((size_t)cfg->num_players * 1326, 0);
  for (int p = 0; p < cfg->num_players; ++p)
    if (!build_range_cdf(sg->ranges + 1326 * p, mask, cdf.data() + 1326 * p)) {
      fprintf(stderr, "subgame: player %d's range has no weight off the board\n", p);
      return MCCFR_ERR_INVALID_ARG;
    }
  return MCCFR_OK;
}

void set_subgame_params(mccfr_handle* h, const mccfr_config* cfg, const mccfr_subgame* sg, int nb) {
  h->gp.sub_street = sg->street;
  h->gp.sub_pot = sg->pot;
  h->gp.stack_base = cfg->starting_stack + sg->pot / cfg->num_players;
  for (int i = 0; i < 5; ++i) h->gp.sub_board[i] = (i < nb) ? sg->board[i] : 0;
  h->gp.range_cdf = h->d_ranges;
}

}  // namespace

extern "C" {

int mccfr_create_subgame(const mccfr_config* cfg, const mccfr_subgame* sg, mccfr_handle** out) {
  if (!out) return MCCFR_ERR_INVALID_ARG;
  std::vector<uint32_t> cdf;
  int nb = 0;
  int rc = subgame_cdfs(cfg, sg, cdf, nb);
  if (rc) return rc;
  rc = mccfr_create(cfg, out);
  if (rc) return rc;
  mccfr_handle* h = *out;
  // room for any player count, so a reset can take a different one
  if (cudaMalloc(&h->d_ranges, (size_t)MCCFR_MAX_PLAYERS * 1326 * 4) != cudaSuccess ||
      cudaMemcpy(h->d_ranges, cdf.data(), cdf.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
    mccfr_destroy(h);
    *out = nullptr;
    return MCCFR_ERR_OOM;
  }
  set_subgame_params(h, cfg, sg, nb);
  return MCCFR_OK;
}

int mccfr_subgame_reset(mccfr_handle* h, const mccfr_config* cfg, const mccfr_subgame* sg) {
  if (!h || !cfg || !sg) return MCCFR_ERR_INVALID_ARG;
  if (!h->gp.sub_street || !h->d_ranges) return fail(h, MCCFR_ERR_INVALID_ARG, "not a subgame handle");
  if (cfg->table_log2 != h->cfg.table_log2 || cfg->device != h->cfg.device)
    return fail(h, MCCFR_ERR_INVALID_ARG, "a reset keeps the table capacity and device");
  std::string why;
  if (validate(*cfg, why)) return fail(h, MCCFR_ERR_INVALID_ARG, "%s", why.c_str());
  std::vector<uint32_t> cdf;
  int nb = 0;
  const int rc = subgame_cdfs(cfg, sg, cdf, nb);
  if (rc) return fail(h, rc, "invalid subgame");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  uint8_t pre[52 * 52];
  build_preflop_lut(cfg->preflop_mode, cfg->preflop_buckets, pre);
  CK(cudaMemcpyAsync(h->d_pre, pre, sizeof(pre), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_ranges, cdf.data(), cdf.size() * 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemsetAsync(h->d_block, 0, h->block_bytes, h->stream));  // rows, touched list, counters
  CK(cudaMemsetAsync(h->d_counters, 0, sizeof(Counters), h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->cfg = *cfg;
  h->tv.direct = direct_map(*cfg);
  make_params(*cfg, h->gp);
  set_subgame_params(h, cfg, sg, nb);
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  h->graph_batch = -1;
  h->iterations_done = 0;
  h->launches = 0;
  h->round_player = 0;
  h->traverse_ms = h->apply_ms = h->last_traverse_ms = h->last_apply_ms = 0;
  h->touched_last = 0;
  h->wide_last = 0;
  h->sticky_err = 0;
  h->last_error.clear();
  return MCCFR_OK;
}

int mccfr_share_hand_table(mccfr_handle* h, mccfr_handle* src) {
  if (!h || !src || !src->has_table || h->device != src->device) return MCCFR_ERR_INVALID_ARG;
  if (h->cfg.postflop_mode == MCCFR_POSTFLOP_RANK_CDF && !h->gp.sub_street) {
    if (src->cfg.postflop_mode != MCCFR_POSTFLOP_RANK_CDF ||
        std::memcmp(src->cfg.postflop_buckets, h->cfg.postflop_buckets, sizeof(h->cfg.postflop_buckets)))
      return fail(h, MCCFR_ERR_INVALID_ARG, "rank-CDF buckets differ from the source table's");
    CK(cudaMemcpy(h->d_cdf, src->d_cdf, 3 * 7463, cudaMemcpyDeviceToDevice));
  }
  if (h->d_hr && !h->shared_hr) cudaFree(h->d_hr);
  h->d_hr = src->d_hr;
  h->shared_hr = true;
  h->has_table = true;
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
    h->graph_batch = -1;
  }
  return MCCFR_OK;
}

int mccfr_get_progress(mccfr_handle* h, long long* next_iteration, int* next_player, long long* done) {
  if (!h) return MCCFR_ERR_INVALID_ARG;
  if (next_iteration) *next_iteration = h->iterations_done + 1;
  if (next_player) *next_player = h->round_player;
  if (done) *done = h->iterations_done;
  return MCCFR_OK;
}

int mccfr_batch_round(mccfr_handle* const* tables, int n, const int* traversals, const mccfr_batch_tuning* tuning) {
  if (!tables || !traversals || n < 1 || n > kMaxBatchTables) return MCCFR_ERR_INVALID_ARG;
  mccfr_batch_tuning t{128, 1, 0, 1, 1, MCCFR_BATCH_PERSISTENT, {0, 0}};
  if (tuning) {
    if (!valid_tuning(*tuning)) return MCCFR_ERR_INVALID_ARG;
    t = *tuning;
  }
  const int dev = tables[0]->device;
  for (int i = 0; i < n; ++i) {
    mccfr_handle* h = tables[i];
    if (!h || !h->has_table || h->device != dev || traversals[i] < 1 || h->cfg.sampling != MCCFR_SAMPLING_EXTERNAL)
      return MCCFR_ERR_INVALID_ARG;
  }
  if (dev < 0 || dev >= 64) return MCCFR_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(g_round_mu);
  RoundCtx& R = g_round[dev];
  mccfr_batch* b = nullptr;  // for BCK error reporting
  BCK(cudaSetDevice(dev));
  if (!R.stream) {
    BCK(cudaStreamCreateWithFlags(&R.stream, cudaStreamNonBlocking));
    BCK(cudaMalloc(&R.d_tables, kMaxBatchTables * sizeof(TableDesc)));
    BCK(cudaMalloc(&R.d_phase, sizeof(PhaseDesc)));
    BCK(cudaMalloc(&R.d_work, sizeof(unsigned long long)));
    BCK(cudaMallocHost(&R.h_err, kMaxBatchTables * sizeof(int)));
    R.device = dev;
  }
  unsigned long long total = 0;
  for (int i = 0; i < n; ++i) total += (unsigned long long)traversals[i];
  if (total > R.deals_cap) {
    cudaFree(R.d_deals);
    R.d_deals = nullptr;
    BCK(cudaMalloc(&R.d_deals, total * sizeof(DealRec)));
    R.deals_cap = total;
  }
  std::vector<TableDesc> descs(n);
  PhaseDesc P;
  std::memset(&P, 0, sizeof(P));
  PhaseParams& Q = R.params;
  std::memset(&Q, 0, sizeof(Q));
  unsigned long long off = 0;
  for (int i = 0; i < n; ++i) {
    mccfr_handle* h = tables[i];
    h->h_sched->iteration = h->iterations_done + 1;
    h->h_sched->player = h->round_player;
    h->h_sched->pad = 0;
    BCK(cudaMemcpyAsync(h->d_sched, h->h_sched, sizeof(Sched), cudaMemcpyHostToDevice, R.stream));
    TableDesc& d = descs[i];
    std::memset(&d, 0, sizeof(d));
    d.G = h->gp;
    d.tv = h->tv;
    d.pre = h->d_pre;
    d.cdf = h->d_cdf;
    d.sched = h->d_sched;
    d.counters = h->d_counters;
    const int rb = regret_frac_bits(h->cfg, traversals[i]);
    d.rscale = std::ldexp(1.0f, rb);
    d.rinv = std::ldexp(1.0, -rb);
    d.batch = traversals[i];
    P.table[i] = i;
    P.off[i] = off;
    Q.off[i] = off;
    Q.T[i] = d;
    off += (unsigned long long)traversals[i];
  }
  P.n = n;
  P.off[n] = off;
  Q.n = n;
  Q.off[n] = off;
  BCK(cudaMemcpyAsync(R.d_tables, descs.data(), n * sizeof(TableDesc), cudaMemcpyHostToDevice, R.stream));
  BCK(cudaMemcpyAsync(R.d_phase, &P, sizeof(P), cudaMemcpyHostToDevice, R.stream));
  BCK(cudaMemsetAsync(R.d_work, 0, sizeof(unsigned long long), R.stream));
  const int dgrid = (int)std::min<unsigned long long>((off + 127) / 128, 148ull * 64);
  k_deal_batched<<<std::max(1, dgrid), 128, 0, R.stream>>>(R.d_tables, R.d_phase, tables[0]->d_hr, R.d_deals);
  BCK(cudaGetLastError());
  BatchedKernel kern = pick_kernel(t);
  const size_t smem = batched_smem(t);
  BCK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, t.block, smem));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned long long need_blocks = (off + t.block - 1) / t.block;
  const int grid = (int)std::max<unsigned long long>(1, std::min<unsigned long long>(need_blocks, (unsigned long long)std::max(1, per_sm) * sms));
  kern<<<grid, t.block, smem, R.stream>>>(Q, R.d_deals, R.d_work, t.grab, t.warp_sync);
  BCK(cudaGetLastError());
  k_apply_batched<<<dim3(std::max(1, std::min(148 * 2, (int)((off * 8 + 255) / 256) + 1)), n), 256, 0, R.stream>>>(
      R.d_tables, R.d_phase);
  BCK(cudaGetLastError());
  for (int i = 0; i < n; ++i)  // every table's error flag in one synchronisation
    BCK(cudaMemcpyAsync(R.h_err + i, tables[i]->tv.err, sizeof(int), cudaMemcpyDeviceToHost, R.stream));
  BCK(cudaStreamSynchronize(R.stream));
  int worst = MCCFR_OK;
  for (int i = 0; i < n; ++i) {
    mccfr_handle* h = tables[i];
    h->launches++;
    if (++h->round_player >= h->cfg.num_players) {
      h->round_player = 0;
      h->iterations_done++;
    }
    if (R.h_err[i]) {
      const int rc = check_device_error(h);
      if (rc && !worst) worst = rc;
    }
  }
  return worst;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Heads-up best response (host engine in best_response.cu).
// ---------------------------------------------------------------------------
extern "C" {

void mccfr_br_options_init(mccfr_br_options* opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->flop_stride = 1;
}

int mccfr_rank_cdf_lut(const int32_t* hand_table, size_t table_entries, int ncards, int buckets, uint8_t* out) {
  if (!hand_table || !out || table_entries != (size_t)MCCFR_HAND_TABLE_ENTRIES || ncards < 5 || ncards > 7 ||
      buckets < 1 || buckets > 256)
    return MCCFR_ERR_INVALID_ARG;
  unsigned long long hist[7463];
  host_rank_hist(hand_table, ncards, hist, 0 + (int)std::max(1u, std::thread::hardware_concurrency()));
  build_cdf_lut(hist, buckets, out);
  return MCCFR_OK;
}

int mccfr_best_response(const mccfr_config* cfg, const mccfr_subgame* sg, const int32_t* hand_table,
                        size_t table_entries, const uint64_t* keys, const float* strategy_sum, size_t rows,
                        const mccfr_br_options* opt, mccfr_exploit* out) {
  if (!cfg || !hand_table || !out || (rows && (!keys || !strategy_sum))) return MCCFR_ERR_INVALID_ARG;
  if (table_entries != (size_t)MCCFR_HAND_TABLE_ENTRIES) return MCCFR_ERR_FORMAT;
  std::string why;
  if (validate(*cfg, why)) {
    fprintf(stderr, "mccfr_best_response: %s\n", why.c_str());
    return MCCFR_ERR_INVALID_ARG;
  }
  mccfr_br_options o;
  mccfr_br_options_init(&o);
  if (opt) o = *opt;
  GameParams g;
  make_params(*cfg, g);
  BrInput in;
  in.cfg = cfg;
  in.T = hand_table;
  in.keys = keys;
  in.ssum = strategy_sum;
  in.rows = rows;
  if (sg) {
    if (!sg->ranges || (sg->street != 2 && sg->street != 3) || cfg->num_players != 2) return MCCFR_ERR_INVALID_ARG;
    const int nb = sg->street == 2 ? 4 : 5;
    uint64_t mask = 0;
    for (int i = 0; i < nb; ++i) {
      if (sg->board[i] > 51 || ((mask >> sg->board[i]) & 1)) return MCCFR_ERR_INVALID_ARG;
      mask |= 1ull << sg->board[i];
    }
    if (sg->pot < 0 || sg->pot % 2 != 0) return MCCFR_ERR_INVALID_ARG;
    g.sub_street = sg->street;
    g.sub_pot = sg->pot;
    g.stack_base = cfg->starting_stack + sg->pot / 2;
    for (int i = 0; i < 5; ++i) g.sub_board[i] = (i < nb) ? sg->board[i] : 0;
    for (int p = 0; p < 2; ++p) {
      uint32_t cdf[1326];
      if (!build_range_cdf(sg->ranges + 1326 * p, mask, cdf)) return MCCFR_ERR_INVALID_ARG;
      in.weights[p].resize(1326);
      for (int c = 0; c < 1326; ++c) in.weights[p][c] = (double)cdf[c] - (c ? (double)cdf[c - 1] : 0.0);
    }
  }
  in.G = &g;
  std::string err;
  const int rc = run_best_response(in, o, out, err);
  if (rc) fprintf(stderr, "mccfr_best_response: %s\n", err.c_str());
  return rc;
}

int mccfr_exploitability(mccfr_handle* h, const mccfr_br_options* opt, mccfr_exploit* out) {
  if (!h || !out) return MCCFR_ERR_INVALID_ARG;
  if (!h->has_table) return fail(h, MCCFR_ERR_NO_HAND_TABLE, "no hand table loaded");
  CK(cudaSetDevice(h->device));
  std::vector<HostRow> rows;
  int rc = read_rows(h, rows);
  if (rc) return rc;
  std::vector<uint64_t> keys(rows.size());
  std::vector<float> ssum(rows.size() * 8);
  for (size_t i = 0; i < rows.size(); ++i) {
    keys[i] = rows[i].key;
    std::memcpy(&ssum[8 * i], rows[i].ssum, 32);
  }
  std::vector<int32_t> table(MCCFR_HAND_TABLE_ENTRIES);
  CK(cudaMemcpy(table.data(), h->d_hr, table.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
  mccfr_br_options o;
  mccfr_br_options_init(&o);
  if (opt) o = *opt;
  BrInput in;
  in.cfg = &h->cfg;
  in.G = &h->gp;
  in.T = table.data();
  in.keys = keys.data();
  in.ssum = ssum.data();
  in.rows = rows.size();
  if (h->gp.sub_street) {
    std::vector<uint32_t> cdf(2 * 1326);
    CK(cudaMemcpy(cdf.data(), h->d_ranges, cdf.size() * 4, cudaMemcpyDeviceToHost));
    for (int p = 0; p < 2; ++p) {
      in.weights[p].resize(1326);
      for (int c = 0; c < 1326; ++c)
        in.weights[p][c] = (double)cdf[1326 * p + c] - (c ? (double)cdf[1326 * p + c - 1] : 0.0);
    }
  }
  std::string err;
  rc = run_best_response(in, o, out, err);
  if (rc) return fail(h, rc, "%s", err.c_str());
  return MCCFR_OK;
}

}  // extern "C"
