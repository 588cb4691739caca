// mccfr_trainer.hpp — header-only C++ drop-in for the reference's trainer class.
//
// Same class name, constructor defaults, member signatures and return values
// as GPUCFRTrainer in poker_cuda/src/cfr_gpu.cuh:48-132, implemented over the C
// ABI in mccfr.h, so callers such as poker_cuda/src/main.cpp:309-397 and
// strategy_load_auto (poker_cuda/src/strategy.cpp:132-138) compile unchanged
// against it.  Where the reference calls exit(1) on a CUDA error
// (cfr_gpu.cu:61-69) this class throws std::runtime_error.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "mccfr.h"

static constexpr int GPU_NUM_ACTIONS = 8;
static constexpr int GPU_TABLE_SIZE = MCCFR_REF_TABLE_SIZE;

struct StrategyEntry {
  float probs[GPU_NUM_ACTIONS] = {};
};
using HostStrategyTable = std::unordered_map<uint32_t, StrategyEntry>;

class GPUCFRTrainer {
 public:
  GPUCFRTrainer(int num_players = 2, int starting_stack = 1000, int small_blind = 10, int big_blind = 20,
                bool use_cfr_plus = true, bool use_linear_cfr = true) {
    mccfr_config c;
    mccfr_config_init(&c, MCCFR_PRESET_REF8);
    c.num_players = num_players;
    c.starting_stack = starting_stack;
    c.small_blind = small_blind;
    c.big_blind = big_blind;
    c.use_cfr_plus = use_cfr_plus ? 1 : 0;
    c.use_linear_cfr = use_linear_cfr ? 1 : 0;
    create(c);
  }
  // Any preset or custom game (seed, update rule, abstraction).
  explicit GPUCFRTrainer(const mccfr_config& cfg) { create(cfg); }
  ~GPUCFRTrainer() { mccfr_destroy(h_); }
  GPUCFRTrainer(const GPUCFRTrainer&) = delete;
  GPUCFRTrainer& operator=(const GPUCFRTrainer&) = delete;

  bool load_hand_table(const char* path = "data/handranks.dat") {
    return mccfr_load_hand_table(h_, path) == MCCFR_OK;
  }
  // No file needed: builds the 32,487,834-entry table on the host.
  bool generate_hand_table() {
    std::vector<int32_t> t(MCCFR_HAND_TABLE_ENTRIES);
    if (mccfr_hand_table_generate(t.data(), t.size()) != MCCFR_OK) return false;
    return mccfr_set_hand_table(h_, t.data(), t.size()) == MCCFR_OK;
  }

  void train(long long total_iterations, int batch_size = 65536, bool verbose = true,
             const std::string& ckpt_path = "", long long ckpt_interval = 10000) {
    check(mccfr_train(h_, total_iterations, batch_size, verbose ? 1 : 0, ckpt_path.c_str(), ckpt_interval));
  }

  HostStrategyTable get_strategy() const {
    size_t n = 0;
    int rc = mccfr_get_strategy(h_, nullptr, nullptr, nullptr, 0, &n);
    if (rc != MCCFR_OK && rc != MCCFR_ERR_CAPACITY) check(rc);
    std::vector<uint32_t> keys(n);
    std::vector<float> probs(n * GPU_NUM_ACTIONS);
    check(mccfr_get_strategy(h_, keys.data(), nullptr, probs.data(), n, &n));
    HostStrategyTable t;
    t.reserve(n);
    for (size_t i = 0; i < n; ++i) {
      StrategyEntry e;
      for (int a = 0; a < GPU_NUM_ACTIONS; ++a) e.probs[a] = probs[i * GPU_NUM_ACTIONS + a];
      t.emplace(keys[i], e);
    }
    return t;
  }

  bool save_checkpoint(const std::string& path) const { return mccfr_save_checkpoint(h_, path.c_str()) == MCCFR_OK; }
  bool load_checkpoint(const std::string& path) { return mccfr_load_checkpoint(h_, path.c_str()) == MCCFR_OK; }

  int num_info_sets_active() const {
    long long n = 0;
    check(mccfr_num_info_sets_active(h_, &n));
    return (int)n;
  }

  void export_tables(std::vector<float>& regrets, std::vector<float>& strategy_sum) const {
    const size_t n = (size_t)GPU_NUM_ACTIONS * GPU_TABLE_SIZE;
    regrets.resize(n);
    strategy_sum.resize(n);
    check(mccfr_export_tables(h_, regrets.data(), strategy_sum.data(), n));
  }
  void import_tables(const std::vector<float>& regrets, const std::vector<float>& strategy_sum) {
    if (regrets.size() != strategy_sum.size()) throw std::runtime_error("import_tables: size mismatch");
    check(mccfr_import_tables(h_, regrets.data(), strategy_sum.data(), regrets.size()));
  }

  mccfr_handle* handle() const { return h_; }

 private:
  mccfr_handle* h_ = nullptr;

  void create(const mccfr_config& c) {
    const int rc = mccfr_create(&c, &h_);
    if (rc != MCCFR_OK) throw std::runtime_error(std::string("mccfr_create: ") + mccfr_strerror(rc));
  }
  void check(int rc) const {
    if (rc != MCCFR_OK)
      throw std::runtime_error(std::string(mccfr_strerror(rc)) + ": " + mccfr_last_error(h_));
  }
};
