// best_response.h — internal interface of the host best-response engine.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mccfr.h"

namespace mccfr {

struct GameParams;

// One heads-up game and an average strategy to evaluate.
struct BrInput {
  const mccfr_config* cfg = nullptr;
  const GameParams* G = nullptr;   // the trainer's parameters (sub_* fields set for a subgame)
  const int32_t* T = nullptr;      // rank table, MCCFR_HAND_TABLE_ENTRIES entries
  const uint64_t* keys = nullptr;  // info-set rows: key, strategy sum [rows][8]
  const float* ssum = nullptr;
  size_t rows = 0;
  // subgame: each player's combo weights (the quantised range the deal samples)
  std::vector<double> weights[2];
};

// Exact rank histogram of all C(52, n) hands (n = 5, 6, 7).
void host_rank_hist(const int32_t* T, int ncards, unsigned long long* hist, int threads);

int run_best_response(const BrInput& in, const mccfr_br_options& opt, mccfr_exploit* out, std::string& err);

}  // namespace mccfr
