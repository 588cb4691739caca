// ref_gpu_shim.cu — C entry points over the reference's own GPU trainer.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's poker_cuda/src/cfr_gpu.cu, hand_eval.cpp and abstraction.cpp,
// unmodified and from where they lie, with the reference's release flags
// (-O3 --use_fast_math, poker_cuda/CMakeLists.txt:28) for sm_100a, into
// oracle/_ref/libref_gpu.so.  Tests and bench.py use it as a statistical pin
// of the reference's traversal (its cuRAND streams, fast-math division and
// racy reads make it impossible to match bit for bit) and to time the
// reference's GPU path on the same device.  The product never loads it.
//
// The reference exits the process on any CUDA error (cfr_gpu.cu:38-47, 61-69),
// so callers run it in a process of its own.
#include <cstring>
#include <vector>

#include "cfr_gpu.cuh"

extern "C" {

void* refgpu_create(int players, int stack, int sb, int bb) {
  return new GPUCFRTrainer(players, stack, sb, bb, true, true);
}

void refgpu_destroy(void* h) { delete static_cast<GPUCFRTrainer*>(h); }

int refgpu_load_hand_table(void* h, const char* path) {
  return static_cast<GPUCFRTrainer*>(h)->load_hand_table(path) ? 1 : 0;
}

// GPUCFRTrainer::train (cfr_gpu.cu:1244-1378) without progress output.
void refgpu_train(void* h, long long iters, int batch) {
  static_cast<GPUCFRTrainer*>(h)->train(iters, batch, false, "", 0);
}

// The dense tables [8][2^26] (export_tables, cfr_gpu.cu:1437-1446).
int refgpu_export(void* h, float* regrets, float* strategy_sum, size_t n) {
  std::vector<float> r, s;
  static_cast<GPUCFRTrainer*>(h)->export_tables(r, s);
  if (r.size() != n || s.size() != n) return 0;
  std::memcpy(regrets, r.data(), n * sizeof(float));
  std::memcpy(strategy_sum, s.data(), n * sizeof(float));
  return 1;
}

int refgpu_num_active(void* h) { return static_cast<GPUCFRTrainer*>(h)->num_info_sets_active(); }

}  // extern "C"
