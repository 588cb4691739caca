// showdown.cuh — showdown-evaluation microbenchmark kernels.
//
// Two forms of the rank-table gathers that training's showdown rests on
// (cfr_gpu.cu:114-150 for the chains, 694-753 for the showdown):
//   * k_deal_eval7: random 7-card hands drawn on the device (counter-based
//     Philox, partial Fisher-Yates over the 52 cards, the deal's multiply-shift)
//     and ranked by 7 dependent gathers each;
//   * k_showdown_masks: the deals of a training update (deal_one's Philox words
//     and Fisher-Yates, so exactly the cards training deals), each seat's 7-card
//     rank with the 5-card board walked once and shared by every seat (5 + 2 per
//     seat gathers: the table's state depends only on the card set), and a mask
//     of the seats holding the best rank (several bits: a split pot).
// The 7-card kernel never materialises a deck: a partial Fisher-Yates touches
// at most two positions per draw, so the swapped positions are kept as a short
// list of (position, card) pairs in registers and every other position holds
// its own card.  The cards drawn are those of the full 52-card shuffle.
#pragma once
#include "game.cuh"
#include "traverse_ref.cuh"

namespace mccfr {

constexpr uint32_t kEval7Stream = 0x300u;  // Philox counter word of the microbenchmark's hands

// Partial Fisher-Yates over 52 cards for the first D draws (D <= 17), with
// only the swapped positions stored: draw k swaps positions k and
// j = k + (w_k * (52 - k)) >> 32 and yields the card now at position k.
template <int D>
struct SparseDeck {
  uint8_t pos[D], card[D];
  int m = 0;
  __device__ __forceinline__ int at(int p) const {
    int c = p;
#pragma unroll
    for (int t = 0; t < D; ++t)
      if (t < m && pos[t] == p) c = card[t];
    return c;
  }
  __device__ __forceinline__ int draw(int k, uint32_t w) {
    const int j = k + (int)(((unsigned long long)w * (unsigned long long)(52 - k)) >> 32);
    const int cj = at(j), ck = at(k);
    if (j != k) {  // position j now holds the card that was at k
      bool found = false;
#pragma unroll
      for (int t = 0; t < D; ++t)
        if (t < m && pos[t] == j) {
          card[t] = (uint8_t)ck;
          found = true;
        }
      if (!found) {
#pragma unroll
        for (int t = 0; t < D; ++t)
          if (t == m) {
            pos[t] = (uint8_t)j;
            card[t] = (uint8_t)ck;
          }
        ++m;
      }
    }
    return cj;
  }
};

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_deal_eval7(const int32_t* __restrict__ T, uint32_t seed_lo, uint32_t seed_hi, uint32_t stream,
             unsigned long long n, uint16_t* __restrict__ ranks) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)BLOCK + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * BLOCK) {
    const U4 w0 = philox(U4{(uint32_t)i, stream, kEval7Stream, (uint32_t)(i >> 32)}, seed_lo, seed_hi);
    const U4 w1 = philox(U4{(uint32_t)i, stream, kEval7Stream + 1u, (uint32_t)(i >> 32)}, seed_lo, seed_hi);
    const uint32_t words[7] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z};
    SparseDeck<7> deck;
    int32_t p = 53;
#pragma unroll
    for (int k = 0; k < 7; ++k) p = __ldg(T + p + to_rm(deck.draw(k, words[k])));
    ranks[i] = (uint16_t)decode16((uint32_t)p & 0xFFFF);
  }
}

// The 6-seat deal draws 17 cards, too many for the register list: its deck is
// a row of 52 bytes per thread in shared memory (13 words, an odd stride, so a
// warp's threads touch 32 different banks), filled with 13 word stores.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_showdown_masks(const GameParams G, const int32_t* __restrict__ T, uint32_t uid, unsigned n,
                 uint8_t* __restrict__ masks) {
  __shared__ uint32_t s_deck[BLOCK * 13];
  uint32_t* row = s_deck + 13 * threadIdx.x;
  uint8_t* deck = reinterpret_cast<uint8_t*>(row);
  const int N = G.N;
  const int n_deal = 2 * N + 5;
  for (unsigned t = blockIdx.x * BLOCK + threadIdx.x; t < n; t += gridDim.x * BLOCK) {
#pragma unroll
    for (int w = 0; w < 13; ++w) row[w] = 0x03020100u + 0x04040404u * (uint32_t)w;  // cards 4w .. 4w+3
    // the deal's Philox blocks (deal_one), four draws per block
    for (int blk = 0; 4 * blk < n_deal; ++blk) {
      const U4 o = philox(U4{t, uid, 0u, (uint32_t)blk}, G.seed_lo, G.seed_hi);
      const uint32_t wv[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int i = 4 * blk + e;
        if (i < n_deal) {
          const int j = i + (int)(((unsigned long long)wv[e] * (unsigned long long)(52 - i)) >> 32);
          const uint8_t tmp = deck[i];
          deck[i] = deck[j];
          deck[j] = tmp;
        }
      }
    }
    // board first (positions 2N .. 2N+4), shared by every seat
    int32_t b = 53;
#pragma unroll
    for (int i = 0; i < 5; ++i) b = __ldg(T + b + to_rm(deck[2 * N + i]));
    uint32_t rk[kMaxPlayers];
#pragma unroll
    for (int q = 0; q < kMaxPlayers; ++q) {
      rk[q] = 0;
      if (q < N) {
        const int32_t s6 = __ldg(T + b + to_rm(deck[2 * q]));
        rk[q] = decode16((uint32_t)__ldg(T + s6 + to_rm(deck[2 * q + 1])) & 0xFFFF);
      }
    }
    uint32_t best = 0;
#pragma unroll
    for (int q = 0; q < kMaxPlayers; ++q) best = max(best, rk[q]);
    uint32_t m = 0;
#pragma unroll
    for (int q = 0; q < kMaxPlayers; ++q)
      if (q < N && rk[q] == best) m |= 1u << q;
    masks[t] = (uint8_t)m;
  }
}

}  // namespace mccfr
