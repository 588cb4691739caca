// cli.cpp — command line with the reference's flag names (poker_cuda/src/main.cpp:29-69,
// 98-139) for the train / benchmark / info modes, on the C++ drop-in class.
// Added flags: --seed, --preset ref8|hu20|6max100, --sampling reference|external,
// --table-log2, --raise-cap, --config <file>, and --mode config (prints the
// resolved game as JSON and checks it, no device needed).  A missing --handranks
// file is generated instead of failing.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

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
      "  --seed <N>  --preset <ref8|hu20|6max100>  --sampling <reference|external>  --table-log2 <N>\n"
      "  --raise-cap <N>  --config <file>  (--mode config: print the resolved game and check it)\n"
      "Config file: 'key = value' lines, '#' comments.  Keys: preset, players, stack, sb, bb,\n"
      "  cfr_plus, lcfr, sampling, keys (fnv26|id64), key_bits, actions (comma list of fold,\n"
      "  check, call, check_call, min_raise, all_in or a pot fraction n/d), raise_cap, max_depth,\n"
      "  preflop (chen64|class169), preflop_buckets, postflop (ref_linear|rank_cdf),\n"
      "  postflop_buckets (flop,turn,river), table_log2, seed.  Flags override the file.\n",
      prog);
}

static std::string trim(const std::string& x) {
  const size_t a = x.find_first_not_of(" \t\r"), b = x.find_last_not_of(" \t\r");
  return a == std::string::npos ? "" : x.substr(a, b - a + 1);
}

static std::vector<std::string> split(const std::string& x, char sep) {
  std::vector<std::string> out;
  std::stringstream ss(x);
  std::string item;
  while (std::getline(ss, item, sep)) out.push_back(trim(item));
  return out;
}

// key = value pairs of a config file, in order; false (with a message) on a
// line that is not a pair.
static bool read_config_file(const std::string& path, std::vector<std::pair<std::string, std::string>>& kv,
                             std::string& err) {
  std::ifstream f(path);
  if (!f) return err = "cannot open " + path, false;
  std::string line;
  for (int n = 1; std::getline(f, line); ++n) {
    line = trim(line.substr(0, line.find('#')));
    if (line.empty()) continue;
    const size_t eq = line.find('=');
    if (eq == std::string::npos) return err = path + ":" + std::to_string(n) + ": expected key = value", false;
    kv.emplace_back(trim(line.substr(0, eq)), trim(line.substr(eq + 1)));
  }
  return true;
}

static bool parse_bool(const std::string& v, int& out) {
  if (v == "1" || v == "true" || v == "yes") return out = 1, true;
  if (v == "0" || v == "false" || v == "no") return out = 0, true;
  return false;
}

// Applies one config-file pair to c; false (with a message) for an unknown key
// or a malformed value.
static bool apply_key(mccfr_config& c, const std::string& k, const std::string& v, std::string& err) {
  auto num = [&](int& dst) {
    char* end = nullptr;
    const long x = strtol(v.c_str(), &end, 10);
    if (v.empty() || *end) return false;
    dst = (int)x;
    return true;
  };
  bool ok = true;
  if (k == "players") ok = num(c.num_players);
  else if (k == "stack") ok = num(c.starting_stack);
  else if (k == "sb") ok = num(c.small_blind);
  else if (k == "bb") ok = num(c.big_blind);
  else if (k == "cfr_plus") ok = parse_bool(v, c.use_cfr_plus);
  else if (k == "lcfr") ok = parse_bool(v, c.use_linear_cfr);
  else if (k == "sampling") {
    if (v == "reference") c.sampling = MCCFR_SAMPLING_REFERENCE;
    else if (v == "external") c.sampling = MCCFR_SAMPLING_EXTERNAL;
    else ok = false;
  } else if (k == "keys") {
    if (v == "fnv26") c.key_mode = MCCFR_KEY_FNV26;
    else if (v == "id64") c.key_mode = MCCFR_KEY_ID64;
    else ok = false;
  } else if (k == "key_bits") ok = num(c.key_bits);
  else if (k == "raise_cap") ok = num(c.raise_cap);
  else if (k == "max_depth") ok = num(c.max_depth);
  else if (k == "preflop_buckets") ok = num(c.preflop_buckets);
  else if (k == "table_log2") ok = num(c.table_log2);
  else if (k == "seed") {
    char* end = nullptr;
    const unsigned long long x = strtoull(v.c_str(), &end, 10);
    ok = !v.empty() && !*end;
    if (ok) c.seed = x;
  } else if (k == "preflop") {
    if (v == "chen64") c.preflop_mode = MCCFR_PREFLOP_CHEN64;
    else if (v == "class169") c.preflop_mode = MCCFR_PREFLOP_CLASS169;
    else ok = false;
  } else if (k == "postflop") {
    if (v == "ref_linear") c.postflop_mode = MCCFR_POSTFLOP_REF_LINEAR;
    else if (v == "rank_cdf") c.postflop_mode = MCCFR_POSTFLOP_RANK_CDF;
    else ok = false;
  } else if (k == "postflop_buckets") {
    const auto p = split(v, ',');
    ok = p.size() == 3;
    for (int i = 0; ok && i < 3; ++i) {
      char* end = nullptr;
      c.postflop_buckets[i] = (int)strtol(p[i].c_str(), &end, 10);
      ok = !p[i].empty() && !*end;
    }
  } else if (k == "actions") {
    const auto p = split(v, ',');
    ok = !p.empty() && p.size() <= MCCFR_MAX_ACTIONS;
    for (size_t a = 0; ok && a < p.size(); ++a) {
      int kind = -1, n = 0, d = 1;
      if (p[a] == "fold") kind = MCCFR_ACT_FOLD;
      else if (p[a] == "check") kind = MCCFR_ACT_CHECK;
      else if (p[a] == "call") kind = MCCFR_ACT_CALL;
      else if (p[a] == "check_call") kind = MCCFR_ACT_CHECK_CALL;
      else if (p[a] == "min_raise") kind = MCCFR_ACT_RAISE_MIN;
      else if (p[a] == "all_in") kind = MCCFR_ACT_ALL_IN;
      else if (sscanf(p[a].c_str(), "%d/%d", &n, &d) == 2) kind = MCCFR_ACT_RAISE_POT;
      ok = kind >= 0;
      c.action_kind[a] = kind;
      c.action_num[a] = kind == MCCFR_ACT_RAISE_POT ? n : 0;
      c.action_den[a] = kind == MCCFR_ACT_RAISE_POT ? d : 1;
    }
    if (ok) c.num_actions = (int)p.size();
  } else {
    return err = "unknown config key '" + k + "'", false;
  }
  if (!ok) err = "bad value '" + v + "' for " + k;
  return ok;
}

static void print_config(const mccfr_config& c, const char* why) {
  printf("{\"players\": %d, \"stack\": %d, \"sb\": %d, \"bb\": %d, \"cfr_plus\": %d, \"lcfr\": %d, ",
         c.num_players, c.starting_stack, c.small_blind, c.big_blind, c.use_cfr_plus, c.use_linear_cfr);
  printf("\"sampling\": \"%s\", \"keys\": \"%s\", \"key_bits\": %d, \"actions\": [",
         c.sampling == MCCFR_SAMPLING_EXTERNAL ? "external" : "reference",
         c.key_mode == MCCFR_KEY_FNV26 ? "fnv26" : "id64", c.key_bits);
  static const char* names[] = {"fold", "check", "call", "check_call", "min_raise", "pot", "all_in"};
  for (int a = 0; a < c.num_actions && a < MCCFR_MAX_ACTIONS; ++a) {
    const int k = c.action_kind[a];
    if (k == MCCFR_ACT_RAISE_POT) printf("%s\"%d/%d\"", a ? ", " : "", c.action_num[a], c.action_den[a]);
    else printf("%s\"%s\"", a ? ", " : "", (k >= 0 && k <= 6) ? names[k] : "?");
  }
  printf("], \"raise_cap\": %d, \"max_depth\": %d, \"preflop\": \"%s\", \"preflop_buckets\": %d, ",
         c.raise_cap, c.max_depth, c.preflop_mode == MCCFR_PREFLOP_CLASS169 ? "class169" : "chen64",
         c.preflop_buckets);
  printf("\"postflop\": \"%s\", \"postflop_buckets\": [%d, %d, %d], \"table_log2\": %d, \"seed\": %llu, ",
         c.postflop_mode == MCCFR_POSTFLOP_RANK_CDF ? "rank_cdf" : "ref_linear", c.postflop_buckets[0],
         c.postflop_buckets[1], c.postflop_buckets[2], c.table_log2, (unsigned long long)c.seed);
  if (why) printf("\"valid\": false, \"why\": \"%s\"}\n", why);
  else printf("\"valid\": true}\n");
}

int main(int argc, char** argv) {
  std::string mode = "train", save = "strategy.bin", load, hr = "data/handranks.dat", preset = "ref8", sampling;
  std::string config_path;
  int players = 2, batch = 65536, stack = 1000, sb = 10, bb = 20, table_log2 = 0, raise_cap = -1;
  long long iters = 1000, seed = -1;
  int cfrplus = -1, lcfr = -1;  // -1: not given
  bool players_set = false, stack_set = false, sb_set = false, bb_set = false;
  for (int i = 1; i < argc; ++i) {
    auto next = [&](void) -> const char* { return (i + 1 < argc) ? argv[++i] : ""; };
    if (!strcmp(argv[i], "--mode")) mode = next();
    else if (!strcmp(argv[i], "--players")) { players = atoi(next()); players_set = true; }
    else if (!strcmp(argv[i], "--iters")) iters = atoll(next());
    else if (!strcmp(argv[i], "--batch")) batch = atoi(next());
    else if (!strcmp(argv[i], "--stack")) { stack = atoi(next()); stack_set = true; }
    else if (!strcmp(argv[i], "--sb")) { sb = atoi(next()); sb_set = true; }
    else if (!strcmp(argv[i], "--bb")) { bb = atoi(next()); bb_set = true; }
    else if (!strcmp(argv[i], "--save")) save = next();
    else if (!strcmp(argv[i], "--load")) load = next();
    else if (!strcmp(argv[i], "--handranks")) hr = next();
    else if (!strcmp(argv[i], "--no-cfrplus")) cfrplus = 0;
    else if (!strcmp(argv[i], "--cfrplus")) cfrplus = 1;
    else if (!strcmp(argv[i], "--no-lcfr")) lcfr = 0;
    else if (!strcmp(argv[i], "--lcfr")) lcfr = 1;
    else if (!strcmp(argv[i], "--seed")) seed = atoll(next());
    else if (!strcmp(argv[i], "--preset")) preset = next();
    else if (!strcmp(argv[i], "--sampling")) sampling = next();
    else if (!strcmp(argv[i], "--table-log2")) table_log2 = atoi(next());
    else if (!strcmp(argv[i], "--raise-cap")) raise_cap = atoi(next());
    else if (!strcmp(argv[i], "--config")) config_path = next();
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
  // preset, then the config file, then the flags
  std::vector<std::pair<std::string, std::string>> file_kv;
  if (!config_path.empty()) {
    std::string err;
    if (!read_config_file(config_path, file_kv, err)) {
      fprintf(stderr, "ERROR: %s\n", err.c_str());
      return 1;
    }
    for (const auto& kv : file_kv)
      if (kv.first == "preset") preset = kv.second;
  }
  if (preset != "ref8" && preset != "hu20" && preset != "6max100") {
    fprintf(stderr, "ERROR: unknown preset '%s'\n", preset.c_str());
    return 1;
  }
  mccfr_config c;
  const int pid = preset == "hu20" ? MCCFR_PRESET_HU_20BB : preset == "6max100" ? MCCFR_PRESET_6MAX_100BB : MCCFR_PRESET_REF8;
  mccfr_config_init(&c, pid);
  for (const auto& kv : file_kv) {
    std::string err;
    if (kv.first != "preset" && !apply_key(c, kv.first, kv.second, err)) {
      fprintf(stderr, "ERROR: %s: %s\n", config_path.c_str(), err.c_str());
      return 1;
    }
  }
  // a flag overrides the preset and the file only when given (the REF8 preset's
  // values are the reference's flag defaults, main.cpp:29-69)
  if (players_set) c.num_players = players;
  if (stack_set) c.starting_stack = stack;
  if (sb_set) c.small_blind = sb;
  if (bb_set) c.big_blind = bb;
  if (cfrplus >= 0) c.use_cfr_plus = cfrplus;
  if (lcfr >= 0) c.use_linear_cfr = lcfr;
  if (seed >= 0) c.seed = (uint64_t)seed;
  if (sampling == "external") c.sampling = MCCFR_SAMPLING_EXTERNAL;
  if (sampling == "reference") c.sampling = MCCFR_SAMPLING_REFERENCE;
  if (table_log2) c.table_log2 = table_log2;
  if (raise_cap >= 0) c.raise_cap = raise_cap;
  if (mode == "config") {
    char why[256];
    const bool ok = mccfr_config_validate(&c, why, sizeof(why)) == MCCFR_OK;
    print_config(c, ok ? nullptr : why);
    return ok ? 0 : 1;
  }

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
