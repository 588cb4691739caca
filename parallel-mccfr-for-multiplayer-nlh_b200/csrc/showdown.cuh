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
// The decks live in shared memory, one byte column per thread.
#pragma once
#include "game.cuh"
#include "traverse_ref.cuh"

namespace mccfr {

constexpr uint32_t kEval7Stream = 0x300u;  // Philox counter word of the microbenchmark's hands

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_deal_eval7(const int32_t* __restrict__ T, uint32_t seed_lo, uint32_t seed_hi, uint32_t stream,
             unsigned long long n, uint16_t* __restrict__ ranks) {
  __shared__ uint8_t deck[52][BLOCK];
  const int tid = threadIdx.x;
  for (unsigned long long i = blockIdx.x * (unsigned long long)BLOCK + tid; i < n;
       i += (unsigned long long)gridDim.x * BLOCK) {
    const U4 w0 = philox(U4{(uint32_t)i, stream, kEval7Stream, (uint32_t)(i >> 32)}, seed_lo, seed_hi);
    const U4 w1 = philox(U4{(uint32_t)i, stream, kEval7Stream + 1u, (uint32_t)(i >> 32)}, seed_lo, seed_hi);
    const uint32_t words[7] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z};
#pragma unroll
    for (int c = 0; c < 52; ++c) deck[c][tid] = (uint8_t)c;
    int32_t p = 53;
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      const int j = k + (int)(((unsigned long long)words[k] * (unsigned long long)(52 - k)) >> 32);
      const uint8_t card = deck[j][tid];
      deck[j][tid] = deck[k][tid];
      deck[k][tid] = card;
      p = __ldg(T + p + to_rm(card));
    }
    ranks[i] = (uint16_t)decode16((uint32_t)p & 0xFFFF);
  }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_showdown_masks(const GameParams G, const int32_t* __restrict__ T, uint32_t uid, unsigned n,
                 uint8_t* __restrict__ masks) {
  __shared__ uint8_t deck[52][BLOCK];
  const int tid = threadIdx.x;
  const int N = G.N;
  const int n_deal = 2 * N + 5;
  const int nblk = (n_deal + 1 + 3) / 4;
  for (unsigned t = blockIdx.x * BLOCK + tid; t < n; t += gridDim.x * BLOCK) {
    uint32_t words[24];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      if (j < nblk) {
        const U4 o = philox(U4{t, uid, 0u, (uint32_t)j}, G.seed_lo, G.seed_hi);
        words[4 * j + 0] = o.x;
        words[4 * j + 1] = o.y;
        words[4 * j + 2] = o.z;
        words[4 * j + 3] = o.w;
      }
    }
#pragma unroll
    for (int c = 0; c < 52; ++c) deck[c][tid] = (uint8_t)c;
    for (int i = 0; i < n_deal; ++i) {
      const int j = i + (int)(((unsigned long long)words[i] * (unsigned long long)(52 - i)) >> 32);
      const uint8_t tmp = deck[i][tid];
      deck[i][tid] = deck[j][tid];
      deck[j][tid] = tmp;
    }
    // board first (positions 2N .. 2N+4), shared by every seat
    int32_t b = 53;
#pragma unroll
    for (int i = 0; i < 5; ++i) b = __ldg(T + b + to_rm(deck[2 * N + i][tid]));
    uint32_t rk[kMaxPlayers];
#pragma unroll
    for (int q = 0; q < kMaxPlayers; ++q) {
      rk[q] = 0;
      if (q < N) {
        const int32_t s6 = __ldg(T + b + to_rm(deck[2 * q][tid]));
        rk[q] = decode16((uint32_t)__ldg(T + s6 + to_rm(deck[2 * q + 1][tid])) & 0xFFFF);
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
