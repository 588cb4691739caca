// table.cuh — open-addressed info-set table in HBM.
//
// Replaces the reference's direct-mapped SoA tables [8 x 2^26] (cfr_gpu.cu:
// 1106-1136).  Rows are addressed by linear probing over 64-bit keys (0 = empty)
// in aligned groups of four keys (one 32-byte sector per probe step).  Each row
// has:
//   reg[8]  float  regrets (two float4: one 32-byte sector)
//   ssum[8] float  average-strategy sums
//   visits  u64    updates received since creation
// and per-player-update accumulators, zeroed by the apply kernel:
//   tag     u64    ((update id + 1) << 8) | canonical action mask of that update
//   cnt     u64    (all visits << 32) | visits whose mask equals the canonical one
//   su      i64    sum of fix(u) over canonical visits (reference rule)
//   da[8]   i64    per-action regret deltas (fixed point, 2^-rb units)
//   ds[8]   i64    per-action strategy-sum deltas of non-canonical visits (2^-32)
#pragma once
#include <cstdint>

namespace mccfr {

struct TableView {
  unsigned long long* keys;
  float4* reg;    // [cap][2]
  float4* ssum;   // [cap][2]
  unsigned long long* visits;
  unsigned long long* tag;
  unsigned long long* cnt;
  long long* su;
  long long* da;  // [cap][8]
  long long* ds;  // [cap][8]
  unsigned int* touched;     // [cap]
  unsigned int* n_touched;   // [2], indexed by update-id parity
  unsigned long long mask;   // cap - 1
  int log2cap;
  int* err;
};

enum : int {
  kErrTableFull = 1,
  kErrRecordOverflow = 2,
  kErrStackOverflow = 4,
};

constexpr int kProbeLimit = 1 << 14;

__device__ __forceinline__ unsigned long long home_slot(const TableView& tv, unsigned long long key) {
  return (key * 0x9E3779B97F4A7C15ull) >> (64 - tv.log2cap);
}

// Read-only lookup; returns the slot or -1.
__device__ __forceinline__ long long table_find(const TableView& tv, unsigned long long key) {
  unsigned long long s = home_slot(tv, key) & ~3ull;
  for (int step = 0; step < kProbeLimit; step += 4) {
    const ulonglong2* g = reinterpret_cast<const ulonglong2*>(tv.keys + s);
    const ulonglong2 a = __ldcg(g), b = __ldcg(g + 1);
    if (a.x == key) return (long long)s;
    if (a.y == key) return (long long)(s + 1);
    if (b.x == key) return (long long)(s + 2);
    if (b.y == key) return (long long)(s + 3);
    if (a.x == 0 || a.y == 0 || b.x == 0 || b.y == 0) return -1;
    s = (s + 4) & tv.mask;
  }
  return -1;
}

// Find or insert; returns the slot, or -1 when the probe limit is exceeded.
__device__ __forceinline__ long long table_insert(const TableView& tv, unsigned long long key) {
  unsigned long long s = home_slot(tv, key) & ~3ull;
  for (int step = 0; step < kProbeLimit; step += 4) {
    const ulonglong2* g = reinterpret_cast<const ulonglong2*>(tv.keys + s);
    const ulonglong2 a = __ldcg(g), b = __ldcg(g + 1);
    const unsigned long long v[4] = {a.x, a.y, b.x, b.y};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      unsigned long long cur = v[i];
      if (cur == key) return (long long)(s + i);
      if (cur == 0) {
        cur = atomicCAS(tv.keys + s + i, 0ull, key);
        if (cur == 0 || cur == key) return (long long)(s + i);
      }
    }
    s = (s + 4) & tv.mask;
  }
  atomicOr(tv.err, kErrTableFull);
  return -1;
}

// Marks the row as touched by update `uid`; returns whether `vm` is the
// update's canonical mask for that row (the first visitor sets it).
__device__ __forceinline__ bool touch_row(const TableView& tv, unsigned long long slot, uint32_t uid,
                                          uint32_t vm) {
  const unsigned long long want = ((unsigned long long)(uid + 1) << 8) | vm;
  unsigned long long old = __ldcg(tv.tag + slot);
  if ((old >> 8) != (unsigned long long)(uid + 1)) {
    const unsigned long long r = atomicCAS(tv.tag + slot, old, want);
    if (r == old) {
      const unsigned int i = atomicAdd(tv.n_touched + (uid & 1), 1u);
      tv.touched[i] = (unsigned int)slot;
      return true;
    }
    old = r;
  }
  return (uint32_t)(old & 0xFF) == vm;
}

}  // namespace mccfr
