// Host-side builder of the 7-card rank state machine (see handtable.cpp).
#pragma once
#include <cstddef>
#include <cstdint>

#define MCCFR_HAND_TABLE_ENTRIES 32487834

namespace mccfr {
// Fills out[0..n_entries) and returns the number of entries used (612,978*53),
// or a negative value on failure.  *n_states_out receives the number of ids.
int64_t generate_hand_table(int32_t* out, size_t n_entries, int* n_states_out);
// Packed rank (category << 12 | ordinal) of 5..7 cards given as 1..52 codes.
int32_t packed_rank_of_cards(const int* cards, int n);
// Packed rank -> 1..7462 (0 for a value that is not a packed rank).
int decode_packed(int32_t packed);
int hand_class_count();
}  // namespace mccfr
