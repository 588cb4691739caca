// cli.cpp — command line with the reference's flag names (poker_cuda/src/main.cpp:29-69,
// 98-139) for the train / benchmark / info modes, on the C++ drop-in class.
// Added flags: --seed, --preset ref8|hu20|6max100, --sampling reference|external,
// --table-log2.  A missing --handranks file is generated instead of failing.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "../../include/mccfr_trainer.hpp"

static void usage(const char* prog) {
  printf(
      "Usage: %s [options]\n"
      "  --mode <train|benchmark|info>   (default: train)\n"
      "  --players <N> (2)  --iters <N> (1000)  --batch <N> (65536)\n"
      "  --stack <N> (1000)  --sb <N> (10)  --bb <N> (20)\n"
      "  --save <file> (strategy.bin)  --load <ckpt>  --handranks <file> (data/handranks.dat)\n"
      "  --no-cfrplus | --cfrplus   --no-lcfr | --lcfr\n"
      "  --seed <N>  --preset <ref8|hu20|6max100>  --sampling <reference|external>  --table-log2 <N>\n",
      prog);
}

int main(int argc, char** argv) {
  std::string mode = "train", save = "strategy.bin", load, hr = "data/handranks.dat", preset = "ref8", sampling;
  int players = 2, batch = 65536, stack = 1000, sb = 10, bb = 20, table_log2 = 0;
  long long iters = 1000, seed = -1;
  bool cfrplus = true, lcfr = true, players_set = false, blinds_set = false;
  for (int i = 1; i < argc; ++i) {
    auto next = [&](void) -> const char* { return (i + 1 < argc) ? argv[++i] : ""; };
    if (!strcmp(argv[i], "--mode")) mode = next();
    else if (!strcmp(argv[i], "--players")) { players = atoi(next()); players_set = true; }
    else if (!strcmp(argv[i], "--iters")) iters = atoll(next());
    else if (!strcmp(argv[i], "--batch")) batch = atoi(next());
    else if (!strcmp(argv[i], "--stack")) { stack = atoi(next()); blinds_set = true; }
    else if (!strcmp(argv[i], "--sb")) { sb = atoi(next()); blinds_set = true; }
    else if (!strcmp(argv[i], "--bb")) { bb = atoi(next()); blinds_set = true; }
    else if (!strcmp(argv[i], "--save")) save = next();
    else if (!strcmp(argv[i], "--load")) load = next();
    else if (!strcmp(argv[i], "--handranks")) hr = next();
    else if (!strcmp(argv[i], "--no-cfrplus")) cfrplus = false;
    else if (!strcmp(argv[i], "--cfrplus")) cfrplus = true;
    else if (!strcmp(argv[i], "--no-lcfr")) lcfr = false;
    else if (!strcmp(argv[i], "--lcfr")) lcfr = true;
    else if (!strcmp(argv[i], "--seed")) seed = atoll(next());
    else if (!strcmp(argv[i], "--preset")) preset = next();
    else if (!strcmp(argv[i], "--sampling")) sampling = next();
    else if (!strcmp(argv[i], "--table-log2")) table_log2 = atoi(next());
    else if (!strcmp(argv[i], "--help")) { usage(argv[0]); return 0; }
  }
  if (mode == "info") {
    int n = 0;
    cudaGetDeviceCount(&n);
    printf("GPUs found: %d\n", n);
    for (int d = 0; d < n; ++d) {
      cudaDeviceProp p;
      cudaGetDeviceProperties(&p, d);
      printf("  [%d] %s  SM=%d  VRAM=%.0fGB  L2=%.0fMB\n", d, p.name, p.multiProcessorCount, p.totalGlobalMem / 1e9,
             p.l2CacheSize / 1e6);
    }
    return 0;
  }
  mccfr_config c;
  const int pid = preset == "hu20" ? MCCFR_PRESET_HU_20BB : preset == "6max100" ? MCCFR_PRESET_6MAX_100BB : MCCFR_PRESET_REF8;
  mccfr_config_init(&c, pid);
  if (pid == MCCFR_PRESET_REF8 || players_set) c.num_players = players;
  if (pid == MCCFR_PRESET_REF8 || blinds_set) {
    c.starting_stack = stack;
    c.small_blind = sb;
    c.big_blind = bb;
  }
  c.use_cfr_plus = cfrplus;
  c.use_linear_cfr = lcfr;
  if (seed >= 0) c.seed = (uint64_t)seed;
  if (sampling == "external") c.sampling = MCCFR_SAMPLING_EXTERNAL;
  if (sampling == "reference") c.sampling = MCCFR_SAMPLING_REFERENCE;
  if (table_log2) c.table_log2 = table_log2;

  auto make = [&]() {
    GPUCFRTrainer* t = new GPUCFRTrainer(c);
    FILE* f = fopen(hr.c_str(), "rb");
    bool ok;
    if (f) {
      fclose(f);
      ok = t->load_hand_table(hr.c_str());
    } else {
      fprintf(stderr, "NOTE: %s not found; generating the rank table in memory\n", hr.c_str());
      ok = t->generate_hand_table();
    }
    if (!ok) {
      fprintf(stderr, "ERROR: could not load a compatible rank table from %s\n", hr.c_str());
      delete t;
      return (GPUCFRTrainer*)nullptr;
    }
    return t;
  };
  try {
    if (mode == "train") {
      GPUCFRTrainer* t = make();
      if (!t) return 1;
      if (!load.empty() && !t->load_checkpoint(load) && mccfr_load_checkpoint_v2(t->handle(), load.c_str()) != MCCFR_OK)
        fprintf(stderr, "WARNING: could not load checkpoint %s\n", load.c_str());
      printf("Training: players=%d iters=%lld batch=%d\n", c.num_players, iters, batch);
      const auto t0 = std::chrono::steady_clock::now();
      t->train(iters, batch, true, save.empty() ? "" : save + ".ckpt", 10000);
      const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      printf("Done: %.0fM traversals in %.2fs (%.1fM traversals/s)\n", iters * (double)batch * c.num_players / 1e6, sec,
             iters * (double)batch * c.num_players / sec / 1e6);
      printf("Info sets active: %d\n", t->num_info_sets_active());
      if (c.key_mode == MCCFR_KEY_FNV26 ? t->save_checkpoint(save + ".ckpt")
                                        : mccfr_save_checkpoint_v2(t->handle(), (save + ".ckpt").c_str()) == MCCFR_OK)
        printf("Checkpoint saved to %s.ckpt\n", save.c_str());
      if (mccfr_save_strategy(t->handle(), save.c_str()) == MCCFR_OK) printf("Strategy saved to %s\n", save.c_str());
      delete t;
    } else if (mode == "benchmark") {
      for (int bs : {4096, 16384, 65536, 262144}) {
        GPUCFRTrainer* t = make();
        if (!t) return 1;
        const auto t0 = std::chrono::steady_clock::now();
        t->train(10, bs, false);
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        const double n = 10.0 * bs * c.num_players;
        printf("  batch=%6d  traversals=%.0fM  time=%.2fs  speed=%.1fM/s\n", bs, n / 1e6, sec, n / sec / 1e6);
        delete t;
      }
    } else {
      fprintf(stderr, "Unknown mode: %s\n", mode.c_str());
      usage(argv[0]);
      return 1;
    }
  } catch (const std::exception& e) {
    fprintf(stderr, "ERROR: %s\n", e.what());
    return 1;
  }
  return 0;
}
