// game.cuh — device-side game rules, Philox, and info-set keys.
//
// Each function names the reference lines whose semantics it keeps.  All
// arithmetic that decides a sampled action or a table value is IEEE (the library
// is compiled with -fmad=false and without fast-math), so results are bit-exact
// with the CPU oracle.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace mccfr {

constexpr int kMaxPlayers = 6;
constexpr int kSlots = 8;

// Per-launch game description, passed by value to the kernels.
struct GameParams {
  int N, stack, sb, bb;
  int cfr_plus, lcfr, sampling, key_mode;
  int num_actions, raise_cap, max_depth, postflop_mode;
  int post_b[3];
  uint32_t seed_lo, seed_hi;
  int key_bits;
  // subgame re-solve (sub_street 0 = the full game from the blinds)
  int sub_street;               // 2: starts on the turn, 3: on the river
  int sub_pot;                  // chips already in the pot, split equally
  uint8_t sub_board[5];         // known board cards (4 or 5)
  const uint32_t* range_cdf;    // [N][1326] cumulative range weights, 2^31 scale
  // action slots
  int8_t kind[kSlots];
  int16_t num[kSlots], den[kSlots];
  uint8_t m_fold, m_check, m_call, m_allin, m_raise, m_check_kind;
  uint8_t n_fallback;
  uint8_t fallback[kSlots];
  uint8_t default_slot;
  int stack_base;  // chips behind plus chips already in: stack + (subgame) pot share
  int8_t den_shift[kSlots];  // log2(den[a]) when den[a] is a power of two, else -1
};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11).
// ---------------------------------------------------------------------------
struct U4 {
  uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
  }
  return c;
}

// (0, 1]: the top 24 bits plus one, times 2^-24 (exact in FP32).
__device__ __forceinline__ float uniform01(uint32_t w) {
  return __fmul_rn((float)((w >> 8) + 1u), 1.0f / 16777216.0f);
}

constexpr uint64_t kPathSeed = 0x243F6A8885A308D3ull;

__host__ __device__ __forceinline__ uint64_t path_step(uint64_t h, int a) {
  h = (h ^ (uint64_t)(a + 1)) * 0x9E3779B97F4A7C15ull;
  return h ^ (h >> 31);
}

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z ^= z >> 33;
  z *= 0xFF51AFD7ED558CCDull;
  z ^= z >> 33;
  z *= 0xC4CEB9FE1A85EC53ull;
  z ^= z >> 33;
  return z;
}

// Checksum term of one table row (mccfr_table_digest): the row's key, the bits
// of its regrets and strategy sums and its update count, mixed in a fixed order.
__host__ __device__ __forceinline__ uint64_t row_digest(uint64_t key, const uint32_t* reg_bits,
                                                        const uint32_t* ssum_bits, uint64_t visits) {
  uint64_t h = mix64(key ^ 0x9E3779B97F4A7C15ull);
  for (int a = 0; a < 8; ++a) h = mix64(h ^ (uint64_t)reg_bits[a] ^ ((uint64_t)a << 32));
  for (int a = 0; a < 8; ++a) h = mix64(h ^ (uint64_t)ssum_bits[a] ^ ((uint64_t)(a + 8) << 32));
  return mix64(h ^ visits);
}

// ---------------------------------------------------------------------------
// Rank table helpers (cfr_gpu.cu:87-112).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int to_rm(int c) { return (c % 13) * 4 + c / 13 + 1; }

__host__ __device__ __forceinline__ uint32_t decode16(uint32_t packed16) {
  const uint32_t cat = (packed16 >> 12) & 0xF;
  const uint32_t ord = packed16 & 0x0FFFu;
  if (ord == 0 || cat < 1 || cat > 9) return 0;
  // category bases of the 1..7462 scale
  const uint32_t base = (cat == 1) ? 0u : (cat == 2) ? 1277u : (cat == 3) ? 4137u
                      : (cat == 4) ? 4995u : (cat == 5) ? 5853u : (cat == 6) ? 5863u
                      : (cat == 7) ? 7140u : (cat == 8) ? 7296u : 7452u;
  return base + ord;
}

// The reference's postflop bucket value on a decoded chain value
// (cfr_gpu.cu:487-488): unsigned arithmetic, truncated to 8 bits.
__device__ __forceinline__ uint32_t ref_linear_bucket(uint32_t rank16, int buckets) {
  return (uint8_t)(((uint32_t)((int)rank16 - 1) * (uint32_t)buckets) / 7462u);
}

// ---------------------------------------------------------------------------
// Action rules (cfr_gpu.cu:186-244, abstraction.cpp:144-234) with an optional
// per-street raise cap.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }

__host__ __device__ __forceinline__ int min_raise_to(int cb, int lfr, int bb) {
  return (cb == 0) ? imax(1, bb) : cb + imax(lfr, bb);
}

__host__ __device__ __forceinline__ int raise_target(const GameParams& G, int a, int pot, int cb, int mrt) {
  if (G.kind[a] == 4 /*RAISE_MIN*/) return mrt;
  // num * pot >= 0, so a power-of-two denominator is an exact shift
  const int x = G.num[a] * pot, sh = G.den_shift[a];
  const int frac = sh >= 0 ? (x >> sh) : x / G.den[a];
  return imax(mrt, cb + imax(1, frac));
}

__host__ __device__ __forceinline__ uint32_t valid_mask(const GameParams& G, int pot, int stack, int to_call,
                                               int cb, int lfr, int raises) {
  if (pot <= 0) pot = 1;
  uint32_t m;
  if (to_call == 0) {
    m = G.m_check;
  } else if (to_call >= stack) {
    return G.m_fold | G.m_allin;
  } else {
    m = G.m_fold | G.m_call;
  }
  const int head = stack - to_call;
  if (head <= 0) return m;
  if (G.raise_cap > 0 && raises >= G.raise_cap) return m;
  const int mrt = min_raise_to(cb, lfr, G.bb);
  const int maxrt = cb + head;
  if (maxrt >= mrt) {
#pragma unroll
    for (int a = 0; a < kSlots; ++a)
      if ((G.m_raise >> a) & 1)
        if (raise_target(G, a, pot, cb, mrt) <= maxrt) m |= 1u << a;
  }
  return m | G.m_allin;
}

__host__ __device__ __forceinline__ int chips_for(const GameParams& G, int a, int pot, int stack, int to_call,
                                                  int cb, int lfr) {
  if (pot <= 0) pot = 1;
  const int k = G.kind[a];
  if (k == 0 || k == 1) return 0;             // fold, check
  if (k == 2 || k == 3) return imin(to_call, stack);  // call, check/call
  if (k == 6) return stack;                   // all-in
  const int mrt = min_raise_to(cb, lfr, G.bb);
  const int maxrt = cb + imax(0, stack - to_call);
  const int t = imin(raise_target(G, a, pot, cb, mrt), maxrt);
  return imin(to_call + imax(0, t - cb), stack);
}

__device__ __forceinline__ int passive_fallback(const GameParams& G, uint32_t vm) {
  for (int i = 0; i < G.n_fallback; ++i)
    if ((vm >> G.fallback[i]) & 1) return G.fallback[i];
  return G.default_slot;
}

__device__ __forceinline__ float bf16_round(float f) {
  return __bfloat162float(__float2bfloat16_rn(f));
}

// BF16 current strategy (cfr_gpu.cu:318-351) and action sampling
// (cfr_gpu.cu:510-537), both from the same regret row.  The strategy of an
// illegal slot only ever enters the sampling sums multiplied by zero, so only
// legal slots are divided; the result is bit-identical to dividing all eight.
__device__ __forceinline__ int sample_action(const GameParams& G, const float* reg, uint32_t vm,
                                             float u) {
  float sum = 0.0f;
#pragma unroll
  for (int a = 0; a < kSlots; ++a) sum = __fadd_rn(sum, fmaxf(0.0f, reg[a]));
  if (!(sum > 1e-7f)) return passive_fallback(G, vm);  // every BF16 entry is 0
  float sig[kSlots];
  float total = 0.0f;
#pragma unroll
  for (int a = 0; a < kSlots; ++a) {
    sig[a] = 0.0f;
    if ((vm >> a) & 1) {
      // a clamped (non-positive) regret gives +0 exactly: no division needed
      if (reg[a] > 0.0f) sig[a] = bf16_round(__fdiv_rn(reg[a], sum));
      total = __fadd_rn(total, sig[a]);
    }
  }
  if (total < 1e-7f) return passive_fallback(G, vm);
  const float r = __fmul_rn(u, total);
  float cum = 0.0f;
  int result = -1;
#pragma unroll
  for (int a = 0; a < kSlots; ++a) {
    if (!((vm >> a) & 1)) continue;  // adds sig * 0 = +0 in the reference
    cum = __fadd_rn(cum, sig[a]);
    if (result < 0 && r <= cum) result = a;
  }
  if (result < 0) result = passive_fallback(G, vm);
  return result;
}

// Regret-matched strategy of a node (cfr_gpu.cu:784-797); illegal slots are 0.
__device__ __forceinline__ void node_strategy(const float* reg, uint32_t vm, float* strat) {
  float sum_r = 0.0f;
#pragma unroll
  for (int a = 0; a < kSlots; ++a)
    if ((vm >> a) & 1) sum_r = __fadd_rn(sum_r, fmaxf(0.0f, reg[a]));
  if (sum_r > 1e-7f) {
#pragma unroll
    for (int a = 0; a < kSlots; ++a) strat[a] = ((vm >> a) & 1) && reg[a] > 0.0f ? __fdiv_rn(reg[a], sum_r) : 0.0f;
  } else {
    const float uni = __fdiv_rn(1.0f, (float)__popc(vm));
#pragma unroll
    for (int a = 0; a < kSlots; ++a) strat[a] = ((vm >> a) & 1) ? uni : 0.0f;
  }
}

// Seat p + i (0 <= p < N, 0 <= i <= N) around a table of N seats, without a
// division.
__host__ __device__ __forceinline__ int seat_after(int p, int i, int N) {
  const int s = p + i;
  return s >= N ? s - N : s;
}

// Per-player fields indexed by a runtime player: selects over the unrolled
// slots, so that a state held by one thread stays in registers instead of
// being placed in local memory for dynamic indexing.
template <class T>
__device__ __forceinline__ int pget(const T (&a)[kMaxPlayers], int p) {
  int v = a[0];
#pragma unroll
  for (int i = 1; i < kMaxPlayers; ++i)
    if (p == i) v = a[i];
  return v;
}
template <class T>
__device__ __forceinline__ void pset(T (&a)[kMaxPlayers], int p, int v) {
#pragma unroll
  for (int i = 0; i < kMaxPlayers; ++i)
    if (p == i) a[i] = (T)v;
}

// Hole-card combo index of two distinct cards: hi*(hi-1)/2 + lo, 0..1325.
__device__ __forceinline__ int combo_index(int a, int b) {
  const int lo = min(a, b), hi = max(a, b);
  return hi * (hi - 1) / 2 + lo;
}
__device__ __forceinline__ void combo_cards(int idx, int& lo, int& hi) {
  int h = 1;
  while ((h + 1) * h / 2 <= idx) ++h;
  hi = h;
  lo = idx - h * (h - 1) / 2;
}

// Reference info-set slot (cfr_gpu.cu:165-179).
__host__ __device__ __forceinline__ uint32_t fnv_slot(uint32_t player, uint32_t hb, uint32_t bb,
                                             uint32_t street, uint32_t bits) {
  uint32_t h = 2166136261u;
  h = (h ^ (player & 0xFF)) * 16777619u;
  h = (h ^ (hb & 0xFF)) * 16777619u;
  h = (h ^ (bb & 0xFF)) * 16777619u;
  h = (h ^ (street & 0xFF)) * 16777619u;
  h = (h ^ (bits & 0xFF)) * 16777619u;
  h = (h ^ ((bits >> 8) & 0xFF)) * 16777619u;
  h = (h ^ ((bits >> 16) & 0xFF)) * 16777619u;
  h = (h ^ ((bits >> 24) & 0xFF)) * 16777619u;
  return h & ((1u << 26) - 1);
}

__host__ __device__ __forceinline__ uint64_t info_key(const GameParams& G, uint32_t player, uint32_t hb,
                                             uint32_t bb, uint32_t street, uint32_t abits,
                                             uint64_t path) {
  if (G.key_mode == 0) return (uint64_t)fnv_slot(player, hb, bb, street, abits) + 1;
  uint64_t k = path ^ ((uint64_t)player << 56) ^ ((uint64_t)hb << 44) ^ ((uint64_t)bb << 32) ^
               ((uint64_t)street << 28);
  k = mix64(k);
  if (G.key_bits > 0) return (k & ((1ull << G.key_bits) - 1)) + 1;
  return k ? k : 1;
}

// Fixed-point conversions of one delta (bit-exact with the oracle).
__device__ __forceinline__ long long fix_r(float x, float scale) {
  return __float2ll_rn(__fmul_rn(x, scale));
}
__device__ __forceinline__ long long fix_s(float x) {
  return __float2ll_rn(__fmul_rn(x, 4294967296.0f));
}

}  // namespace mccfr
