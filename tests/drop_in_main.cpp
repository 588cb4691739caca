// A caller written against the reference's trainer class, with the calls that
// poker_cuda/src/main.cpp:309-397 (train / benchmark) and
// poker_cuda/src/strategy.cpp:132-138 (checkpoint -> strategy) make, compiled
// unchanged against include/mccfr_trainer.hpp and linked to libmccfr.so.
// Prints one JSON line; argv[1] is a scratch directory, argv[2] the iterations.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "mccfr_trainer.hpp"

int main(int argc, char** argv) {
  const std::string dir = argc > 1 ? argv[1] : ".";
  const long long iters = argc > 2 ? std::atoll(argv[2]) : 2;
  try {
    GPUCFRTrainer trainer(2, 1000, 10, 20, true, true);  // the reference's defaults
    if (!trainer.generate_hand_table()) {
      std::printf("{\"error\": \"hand table\"}\n");
      return 1;
    }
    trainer.train(iters, 4096, false);
    const HostStrategyTable strategy = trainer.get_strategy();
    const int active = trainer.num_info_sets_active();
    const std::string ckpt = dir + "/drop_in.ckpt";
    const bool saved = trainer.save_checkpoint(ckpt);

    GPUCFRTrainer restored;  // strategy_load_auto's path: a default trainer, then the checkpoint
    const bool loaded = restored.load_checkpoint(ckpt);
    const HostStrategyTable again = restored.get_strategy();
    bool same = again.size() == strategy.size();
    for (const auto& kv : strategy) {
      const auto it = again.find(kv.first);
      if (it == again.end()) {
        same = false;
        break;
      }
      for (int a = 0; a < GPU_NUM_ACTIONS; ++a)
        if (it->second.probs[a] != kv.second.probs[a]) same = false;
    }
    std::remove(ckpt.c_str());
    std::printf("{\"strategies\": %zu, \"active\": %d, \"saved\": %s, \"loaded\": %s, \"same\": %s}\n",
                strategy.size(), active, saved ? "true" : "false", loaded ? "true" : "false",
                same ? "true" : "false");
  } catch (const std::exception& e) {
    std::printf("{\"exception\": \"%s\"}\n", e.what());
  }
  return 0;
}
