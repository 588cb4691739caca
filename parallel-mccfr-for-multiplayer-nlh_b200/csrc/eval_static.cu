// eval_static.cu — 7-card evaluation that allocates no device memory.
//
// mccfr_eval7 stages the caller's cards and ranks in device buffers it
// allocates per call.  Some callers cannot allocate device memory themselves:
// code that runs inside a framework which owns every device allocation through
// its own allocator, or a process that must not grow its device footprint after
// start-up.  mccfr_eval7_static serves them: the staging lives in a file-scope
// device array (MCCFR_EVAL7_STATIC_MAX_HANDS hands, 9 bytes each, about 2.25 MiB),
// which every GPU that loads this library holds until the process exits.
//
// The array's name, used in host code, is only a host-side stand-in for the
// symbol, not a device address.  The device address is looked up with
// cudaGetSymbolAddress once per device, on the first call made with that device
// current, and passed to the kernel.  That first call must therefore come before
// any stream capture on that device.  Every call on a device shares the one
// array and the array keeps the last call's contents; calls that overlap on the
// GPU (from several host threads) race on it, so callers must serialise them.
// Nothing in the array needs to start at zero: each call writes every card and
// rank slot it reads back.  The looked-up address lives as long as the device's
// context: after cudaDeviceReset the array may sit elsewhere, so a process that
// resets a device must not call this entry point on that device again.
// dev_table must be device memory (or managed memory): a host pointer is
// refused with MCCFR_ERR_INVALID_ARG instead of reaching the kernel.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/mccfr.h"
#include "game.cuh"

namespace {

constexpr size_t kMaxHands = MCCFR_EVAL7_STATIC_MAX_HANDS;
constexpr size_t kCardBytes = 7 * kMaxHands;  // multiple of 256
constexpr size_t kScratchBytes = kCardBytes + 2 * kMaxHands;

static __device__ __align__(256) uint8_t g_eval7_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint8_t* g_scratch_addr[kMaxDevices] = {};

__global__ void k_eval7_static(const int32_t* __restrict__ T, const uint8_t* __restrict__ cards,
                               uint16_t* __restrict__ ranks, unsigned n) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint8_t* c = cards + 7ull * i;
    int32_t p = __ldg(T + 53 + mccfr::to_rm(c[0]));
#pragma unroll
    for (int k = 1; k < 7; ++k) p = __ldg(T + p + mccfr::to_rm(c[k]));
    ranks[i] = (uint16_t)mccfr::decode16((uint32_t)p & 0xFFFF);
  }
}

// Device address of the static array on the current device (looked up once).
int scratch_address(uint8_t** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return MCCFR_ERR_NO_DEVICE;
  if (dev < 0 || dev >= kMaxDevices) return MCCFR_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_eval7_scratch);
    if (e != cudaSuccess || !p) {
      fprintf(stderr, "mccfr_eval7_static: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      return MCCFR_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<uint8_t*>(p);
  }
  *out = g_scratch_addr[dev];
  return MCCFR_OK;
}

}  // namespace

extern "C" int mccfr_eval7_static(const int32_t* dev_table, const uint8_t* cards, uint16_t* ranks, size_t n) {
  if (!dev_table || !cards || !ranks) return MCCFR_ERR_INVALID_ARG;
  if (n > kMaxHands) {
    fprintf(stderr, "mccfr_eval7_static: %zu hands exceed the static maximum of %zu per call\n", n,
            (size_t)kMaxHands);
    return MCCFR_ERR_INVALID_ARG;
  }
  if (n == 0) return MCCFR_OK;
  for (size_t i = 0; i < 7 * n; ++i)
    if (cards[i] > 51) return MCCFR_ERR_INVALID_ARG;
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, dev_table) != cudaSuccess) {
    cudaGetLastError();
    return MCCFR_ERR_INVALID_ARG;
  }
  if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) return MCCFR_ERR_INVALID_ARG;
  uint8_t* base = nullptr;
  const int rc = scratch_address(&base);
  if (rc) return rc;
  uint8_t* d_cards = base;
  uint16_t* d_ranks = reinterpret_cast<uint16_t*>(base + kCardBytes);
  if (cudaMemcpy(d_cards, cards, 7 * n, cudaMemcpyHostToDevice) != cudaSuccess) return MCCFR_ERR_CUDA;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  k_eval7_static<<<blocks, 256>>>(dev_table, d_cards, d_ranks, (unsigned)n);
  if (cudaGetLastError() != cudaSuccess) return MCCFR_ERR_CUDA;
  if (cudaMemcpy(ranks, d_ranks, 2 * n, cudaMemcpyDeviceToHost) != cudaSuccess) return MCCFR_ERR_CUDA;
  return MCCFR_OK;
}
