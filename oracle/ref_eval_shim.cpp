// ref_eval_shim.cpp — C entry points over the reference's own strategy-dump
// consumers, for tests only: strategy_load_auto (poker_cuda/src/strategy.cpp:
// 112-138), strategy_load (strategy.cpp:54-110) and evaluate_strategy_np
// (poker_cuda/src/eval.cpp:604-627), compiled unchanged from the reference's
// sources by oracle/Makefile into oracle/_ref/libref_eval.so.
//
// TEST INFRASTRUCTURE ONLY: it plays a strategy dump written by libmccfr.so
// against the reference's scripted opponents, so the dump is shown to be a
// drop-in for the reference's evaluation path.
//
// strategy.cpp's checkpoint branch constructs the reference's trainer class;
// this checker only reads strategy dumps, so the members that branch names are
// defined here as inert stand-ins (no device code is built).
#include <cstdint>
#include <string>

#include "abstraction.h"
#include "cfr_gpu.cuh"
#include "eval.h"
#include "hand_eval.h"
#include "strategy.h"

GPUCFRTrainer::GPUCFRTrainer(int, int, int, int, bool, bool) {}
GPUCFRTrainer::~GPUCFRTrainer() {}
bool GPUCFRTrainer::load_checkpoint(const std::string&) { return false; }
HostStrategyTable GPUCFRTrainer::get_strategy() const { return {}; }

namespace {
HostStrategyTable g_strategy;
}

extern "C" {

// hand_eval_init + abstraction_init (eval.h: both required before play).
int refeval_init(const char* handranks_path) {
  if (!hand_eval_init(handranks_path)) return 0;
  abstraction_init();
  return 1;
}

// Loads a strategy file with the reference's loader; returns its entry count,
// or -1 when the loader rejects it.
long long refeval_load(const char* path) {
  g_strategy.clear();
  if (!strategy_load_auto(g_strategy, path, 2, 1000, 10, 20)) return -1;
  return (long long)g_strategy.size();
}

// One entry of the loaded table: probs[8] for key; returns 0 when absent.
int refeval_entry(uint32_t key, float* probs) {
  const auto it = g_strategy.find(key);
  if (it == g_strategy.end()) return 0;
  for (int a = 0; a < GPU_NUM_ACTIONS; ++a) probs[a] = it->second.probs[a];
  return 1;
}

// evaluate_strategy_np with the loaded table: the bot in seat 0 against
// scripted opponents of one archetype (OpponentType order of eval.h).
int refeval_play(int n_players, int opponent, long long n_hands, int stack, int sb, int bb, unsigned seed,
                 double* bb_per_100, double* net_bb, long long* hands) {
  const EvalResult r = evaluate_strategy_np(g_strategy, n_players, (OpponentType)opponent, n_hands, stack, sb,
                                            bb, seed);
  *bb_per_100 = r.bb_per_100;
  *net_bb = r.net_bb;
  *hands = r.hands_played;
  return 1;
}

}  // extern "C"
