// ref_shim.cpp — C entry points over the reference's own CPU functions.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile together with the
// reference's unmodified poker_cuda/src/hand_eval.cpp and abstraction.cpp (read
// where they lie; never copied) into oracle/_ref/libref.so, so tests can pin the
// oracle's restatements against the reference itself.
#include "abstraction.h"
#include "hand_eval.h"

extern "C" {

int ref_hand_eval_init(const char* path) { return hand_eval_init(path) ? 1 : 0; }

void ref_abstraction_init(void) { abstraction_init(); }

int ref_evaluate_7cards(const unsigned char* c) {
  return evaluate_7cards(c[0], c[1], c[2], c[3], c[4], c[5], c[6]);
}

int ref_evaluate_best(int h0, int h1, const unsigned char* comm, int n_comm) {
  Card cc[5];
  for (int i = 0; i < n_comm && i < 5; ++i) cc[i] = comm[i];
  return evaluate_best((Card)h0, (Card)h1, cc, n_comm);
}

int ref_preflop_bucket(int h0, int h1) { return preflop_bucket((Card)h0, (Card)h1); }

int ref_fast_postflop_bucket(int h0, int h1, const unsigned char* comm, int n_comm) {
  Card cc[5];
  for (int i = 0; i < n_comm && i < 5; ++i) cc[i] = comm[i];
  return fast_postflop_bucket((Card)h0, (Card)h1, cc, n_comm);
}

int ref_valid_actions_mask(int pot, int stack, int to_call, int cb, int lfr, int bb) {
  return valid_actions_mask(pot, stack, to_call, cb, lfr, bb);
}

int ref_action_to_chips(int a, int pot, int stack, int to_call, int cb, int lfr, int bb) {
  return action_to_chips((Action)a, pot, stack, to_call, cb, lfr, bb);
}

}  // extern "C"
