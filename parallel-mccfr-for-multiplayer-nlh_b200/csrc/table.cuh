// table.cuh — open-addressed info-set table in HBM.
//
// Replaces the reference's direct-mapped SoA tables [8 x 2^26] (cfr_gpu.cu:
// 1106-1136).  Each row is one 256-byte record (two 128-byte lines), so that a
// visit touches two adjacent sectors and folding a row in reads one contiguous
// record instead of a dozen scattered ones:
//     0  key    u64   0 = empty; linear probing from the key's home slot, or row k-1
//                       for key k when every key is at most the capacity (direct map)
//     8  tag    u64   ((update id + 1) << 8) | canonical action mask of that update
//    16  cnt    u64   (all visits << 32) | visits whose mask is the canonical one
//    24  su     i64   sum of fix(u) (reference rule) or fix(v_h) (external sampling)
//    32  reg[8] f32   regrets: read by every visit (snapshot within an update)
//    64  ssum[8] f32  average-strategy sums
//    96  da[8]  i64   per-action regret deltas, 2^-rb units
//   160  ds[8]  i64   strategy weights of non-canonical visits, 2^-32 units
//   224  visits u64   updates received since creation
//   232  flags  u32   bit 0: ds holds values; bit 1: da holds values
// tag/cnt/su/da/ds/flags are per-update accumulators, zeroed by the apply
// kernel.  da and ds are zero unless a flag says they were written (every
// writer sets its flag), so the apply kernel loads the whole record at once and
// writes them back only for flagged rows.
#pragma once
#include <cstdint>

namespace mccfr {

constexpr int kRowBytes = 256;
constexpr int kOffKey = 0, kOffTag = 8, kOffCnt = 16, kOffSu = 24, kOffReg = 32, kOffSsum = 64, kOffDa = 96,
              kOffDs = 160, kOffVisits = 224, kOffFlags = 232;
constexpr unsigned kFlagDs = 1u, kFlagDa = 2u;

// The touched-row list is cut into kListShards shards by the slot's low bits:
// shard s holds slots s, s + S, s + 2S, ..., so it never holds more than cap / S
// rows, and appends spread over S counters instead of queueing on one address.
constexpr int kListShards = 32;
constexpr int kCounterStride = 32;  // counters 128 bytes apart (separate lines)

struct TableView {
  unsigned char* rows;       // [cap][256]
  unsigned int* touched;     // [kListShards][cap / kListShards] rows touched by the update
  // counters, kCounterStride words apart: entries of each shard by update-id
  // parity (index parity * kListShards + shard), then, by parity, rows whose
  // second line the apply kernel folded (index 2 * kListShards + parity)
  unsigned int* n_touched;
  unsigned long long mask;   // cap - 1
  int log2cap;
  int direct;                // every key is at most cap: key k owns row k-1, no probing
  int* err;
};

enum : int {
  kErrTableFull = 1,
  kErrRecordOverflow = 2,
  kErrStackOverflow = 4,
};

constexpr int kProbeLimit = 1 << 14;

__device__ __forceinline__ unsigned char* row_ptr(const TableView& tv, unsigned long long s) {
  return tv.rows + (s << 8);
}
__device__ __forceinline__ unsigned long long* row_key(const TableView& tv, unsigned long long s) {
  return reinterpret_cast<unsigned long long*>(row_ptr(tv, s) + kOffKey);
}
__device__ __forceinline__ unsigned long long* row_tag(const TableView& tv, unsigned long long s) {
  return reinterpret_cast<unsigned long long*>(row_ptr(tv, s) + kOffTag);
}
__device__ __forceinline__ unsigned long long* row_cnt(const TableView& tv, unsigned long long s) {
  return reinterpret_cast<unsigned long long*>(row_ptr(tv, s) + kOffCnt);
}
__device__ __forceinline__ unsigned long long* row_su(const TableView& tv, unsigned long long s) {
  return reinterpret_cast<unsigned long long*>(row_ptr(tv, s) + kOffSu);
}
__device__ __forceinline__ float4* row_reg(const TableView& tv, unsigned long long s) {
  return reinterpret_cast<float4*>(row_ptr(tv, s) + kOffReg);
}
__device__ __forceinline__ float4* row_ssum(const TableView& tv, unsigned long long s) {
  return reinterpret_cast<float4*>(row_ptr(tv, s) + kOffSsum);
}
__device__ __forceinline__ unsigned long long* row_da(const TableView& tv, unsigned long long s) {
  return reinterpret_cast<unsigned long long*>(row_ptr(tv, s) + kOffDa);
}
__device__ __forceinline__ unsigned long long* row_ds(const TableView& tv, unsigned long long s) {
  return reinterpret_cast<unsigned long long*>(row_ptr(tv, s) + kOffDs);
}
__device__ __forceinline__ unsigned long long* row_visits(const TableView& tv, unsigned long long s) {
  return reinterpret_cast<unsigned long long*>(row_ptr(tv, s) + kOffVisits);
}
__device__ __forceinline__ unsigned int* row_flags(const TableView& tv, unsigned long long s) {
  return reinterpret_cast<unsigned int*>(row_ptr(tv, s) + kOffFlags);
}

__device__ __forceinline__ unsigned long long home_slot(const TableView& tv, unsigned long long key) {
  return (key * 0x9E3779B97F4A7C15ull) >> (64 - tv.log2cap);
}

// Read-only lookup; returns the slot or -1.  W keys are loaded per probe step
// (independent loads issued together); W is an autotuned probe width.  A
// direct-mapped table reads the key's own row only.
template <int W = 1>
__device__ __forceinline__ long long table_find(const TableView& tv, unsigned long long key) {
  if (tv.direct) return __ldcg(row_key(tv, key - 1)) == key ? (long long)(key - 1) : -1ll;
  unsigned long long s = home_slot(tv, key);
  for (int step = 0; step < kProbeLimit; step += W) {
    unsigned long long k[W];
#pragma unroll
    for (int i = 0; i < W; ++i) k[i] = __ldcg(row_key(tv, (s + i) & tv.mask));
#pragma unroll
    for (int i = 0; i < W; ++i) {
      if (k[i] == key) return (long long)((s + i) & tv.mask);
      if (k[i] == 0) return -1;
    }
    s = (s + W) & tv.mask;
  }
  return -1;
}

// Find or insert; returns the slot, or -1 when the probe limit is exceeded.
// In a direct-mapped table row k-1 can hold no key but k, so every writer of
// the key stores the same value and no atomic is needed.
template <int W = 1>
__device__ __forceinline__ long long table_insert(const TableView& tv, unsigned long long key) {
  if (tv.direct) {
    unsigned long long* kp = row_key(tv, key - 1);
    if (__ldcg(kp) != key) __stcg(kp, key);
    return (long long)(key - 1);
  }
  unsigned long long s = home_slot(tv, key);
  for (int step = 0; step < kProbeLimit; step += W) {
    unsigned long long k[W];
#pragma unroll
    for (int i = 0; i < W; ++i) k[i] = __ldcg(row_key(tv, (s + i) & tv.mask));
#pragma unroll
    for (int i = 0; i < W; ++i) {
      const unsigned long long slot = (s + i) & tv.mask;
      if (k[i] == key) return (long long)slot;
      if (k[i] == 0) {
        const unsigned long long prev = atomicCAS(row_key(tv, slot), 0ull, key);
        if (prev == 0 || prev == key) return (long long)slot;
      }
    }
    s = (s + W) & tv.mask;
  }
  atomicOr(tv.err, kErrTableFull);
  return -1;
}

__host__ __device__ __forceinline__ unsigned int* list_count(const TableView& tv, uint32_t parity, int shard) {
  return tv.n_touched + (size_t)kCounterStride * (parity * kListShards + shard);
}
__host__ __device__ __forceinline__ unsigned int* wide_count(const TableView& tv, uint32_t parity) {
  return tv.n_touched + (size_t)kCounterStride * (2 * kListShards + parity);
}
// Bytes of the counter block (list counters, wide-row counters, error flag).
constexpr size_t kCounterBytes = (size_t)kCounterStride * 4 * (2 * kListShards + 2) + 128;

__device__ __forceinline__ void list_row(const TableView& tv, unsigned long long slot, uint32_t uid) {
  const int shard = (int)(slot & (kListShards - 1));
  const unsigned int i = atomicAdd(list_count(tv, uid & 1, shard), 1u);
  tv.touched[(size_t)shard * ((tv.mask + 1) / kListShards) + i] = (unsigned int)slot;
}

// Marks the row as touched by update `uid`; returns whether `vm` is the
// update's canonical mask for that row (the first visitor sets it).  `old` is
// the row's tag as the caller read it (any earlier value will do: a stale one
// only makes the compare-and-swap fail and return the current tag).
__device__ __forceinline__ bool touch_row_from(const TableView& tv, unsigned long long slot, uint32_t uid,
                                               uint32_t vm, unsigned long long old) {
  const unsigned long long want = ((unsigned long long)(uid + 1) << 8) | vm;
  unsigned long long* tag = row_tag(tv, slot);
  if ((old >> 8) != (unsigned long long)(uid + 1)) {
    const unsigned long long r = atomicCAS(tag, old, want);
    if (r == old) {
      list_row(tv, slot, uid);
      return true;
    }
    old = r;
  }
  return (uint32_t)(old & 0xFF) == vm;
}
__device__ __forceinline__ bool touch_row(const TableView& tv, unsigned long long slot, uint32_t uid,
                                          uint32_t vm) {
  return touch_row_from(tv, slot, uid, vm, __ldcg(row_tag(tv, slot)));
}

// Marks the row as touched by update `uid` without claiming a canonical mask
// (mask 0: every later visitor takes the direct path), for a visitor that adds
// its whole regret terms to the per-action accumulators; one atomic whose
// result only decides the list entry.  Update ids only grow, so the maximum
// leaves a tag of this update (claimed or not) as it is.
__device__ __forceinline__ void claim_row(const TableView& tv, unsigned long long slot, uint32_t uid) {
  const unsigned long long old = atomicMax(row_tag(tv, slot), (unsigned long long)(uid + 1) << 8);
  if ((old >> 8) < (unsigned long long)(uid + 1)) list_row(tv, slot, uid);
}

// Marks the row's regret accumulators as holding values in this update; every
// writer of da calls it at least once before its first add.
__device__ __forceinline__ void mark_deltas(const TableView& tv, unsigned long long slot) {
  atomicOr(row_flags(tv, slot), kFlagDa);
}

// Adds one visit whose legal mask differs from the row's canonical one: every
// legal action's regret term and strategy weight directly.
__device__ __forceinline__ void add_direct(const TableView& tv, unsigned long long slot, uint32_t vm,
                                           const long long* dr, const long long* dsw) {
  if (dr || dsw) atomicOr(row_flags(tv, slot), (dr ? kFlagDa : 0u) | (dsw ? kFlagDs : 0u));
  for (int a = 0; a < 8; ++a) {
    if (!((vm >> a) & 1)) continue;
    if (dr) atomicAdd(row_da(tv, slot) + a, (unsigned long long)dr[a]);
    if (dsw) atomicAdd(row_ds(tv, slot) + a, (unsigned long long)dsw[a]);
  }
}

}  // namespace mccfr
