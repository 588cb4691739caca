/*
 * mccfr.h — C ABI of the B200 MCCFR trainer (libmccfr.so).
 *
 * This is the drop-in boundary for the reference's GPU trainer class
 * `GPUCFRTrainer` (poker_cuda/src/cfr_gpu.cuh:48-132) and the helpers it calls.
 * Every entry point returns an int status (MCCFR_OK = 0); nothing in the
 * library calls exit().  Plain pointers and sizes only: host buffers unless a
 * parameter name says `dev_`.
 *
 * Cards are 0..51 in the reference's suit-major encoding, card = suit*13 + rank
 * (poker_cuda/src/card.h:8-15), except where a comment says "1..52 codes".
 */
#ifndef MCCFR_H
#define MCCFR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MCCFR_MAX_PLAYERS 6
#define MCCFR_MAX_ACTIONS 8
#define MCCFR_HAND_TABLE_ENTRIES 32487834
#define MCCFR_REF_TABLE_SIZE (1 << 26) /* GPU_TABLE_SIZE, cfr_gpu.cuh:18 */

/* Status codes. */
enum {
  MCCFR_OK = 0,
  MCCFR_ERR_INVALID_ARG = 1,
  MCCFR_ERR_CUDA = 2,
  MCCFR_ERR_OOM = 3,
  MCCFR_ERR_IO = 4,
  MCCFR_ERR_FORMAT = 5,
  MCCFR_ERR_NO_HAND_TABLE = 6,
  MCCFR_ERR_TABLE_FULL = 7,
  MCCFR_ERR_DEVICE = 8,   /* a kernel raised its error flag (e.g. stack overflow) */
  MCCFR_ERR_OVERFLOW = 9, /* fixed-point accumulator range would be exceeded */
  MCCFR_ERR_CAPACITY = 10,/* caller buffer too small; *count holds the size needed */
  MCCFR_ERR_NO_DEVICE = 11,
  MCCFR_ERR_TIMEOUT = 12
};

/* Action slot kinds (the reference's fixed 8 slots are abstraction.h:42-53). */
enum {
  MCCFR_ACT_FOLD = 0,
  MCCFR_ACT_CHECK = 1,
  MCCFR_ACT_CALL = 2,
  MCCFR_ACT_CHECK_CALL = 3, /* check when nothing is owed, call otherwise */
  MCCFR_ACT_RAISE_MIN = 4,
  MCCFR_ACT_RAISE_POT = 5,  /* raise by num/den of the pot */
  MCCFR_ACT_ALL_IN = 6
};

/* Update rule at the updating player's nodes. */
enum {
  /* The reference's rule: one action sampled from the BF16 current strategy,
     importance weight 1/max(strat, 0.05), average strategy accumulated at the
     updating player's nodes (cfr_gpu.cu:768-838). */
  MCCFR_SAMPLING_REFERENCE = 0,
  /* External sampling: every legal action of the updating player is explored;
     opponents sample one action; the average strategy is accumulated at the
     sampled opponents' nodes. */
  MCCFR_SAMPLING_EXTERNAL = 1
};

/* Info-set identity. */
enum {
  MCCFR_KEY_FNV26 = 0, /* the reference's FNV-1a slot & (2^26-1), cfr_gpu.cu:165-179 */
  MCCFR_KEY_ID64 = 1   /* 64-bit hash of (player, buckets, street, full action path) */
};

enum { MCCFR_PREFLOP_CHEN64 = 0, MCCFR_PREFLOP_CLASS169 = 1 };
enum {
  /* rank-linear buckets on the reference's raw chain values (cfr_gpu.cu:476-489) */
  MCCFR_POSTFLOP_REF_LINEAR = 0,
  /* percentile of the true 5/6/7-card rank among all hands of that size */
  MCCFR_POSTFLOP_RANK_CDF = 1
};

enum {
  MCCFR_PRESET_REF8 = 0,       /* the reference's own game and abstraction */
  MCCFR_PRESET_HU_20BB = 1,    /* heads-up, 20BB, {fold, check/call, pot, all-in}, cap 2 */
  MCCFR_PRESET_6MAX_100BB = 2  /* 6-max, 100BB, {fold, call, 1/2, pot, 2 pot, all-in}, cap 3 */
};

typedef struct mccfr_config {
  int32_t num_players;      /* 2..6 */
  int32_t starting_stack;   /* chips */
  int32_t small_blind;
  int32_t big_blind;
  int32_t use_cfr_plus;     /* clamp regrets at 0 after each player-update */
  int32_t use_linear_cfr;   /* average-strategy weight = iteration (else 1) */
  int32_t sampling;         /* MCCFR_SAMPLING_* */
  int32_t key_mode;         /* MCCFR_KEY_* */
  int32_t num_actions;      /* action slots used, 1..8 */
  int32_t action_kind[MCCFR_MAX_ACTIONS];
  int32_t action_num[MCCFR_MAX_ACTIONS]; /* pot fraction numerator (RAISE_POT) */
  int32_t action_den[MCCFR_MAX_ACTIONS]; /* pot fraction denominator (RAISE_POT) */
  int32_t raise_cap;        /* raises per street; 0 = unlimited (the reference) */
  int32_t max_depth;        /* depth cut; the reference returns 0 at depth 20 */
  int32_t preflop_mode;     /* MCCFR_PREFLOP_* */
  int32_t preflop_buckets;  /* 64 for CHEN64, 169 for CLASS169 */
  int32_t postflop_mode;    /* MCCFR_POSTFLOP_* */
  int32_t postflop_buckets[3]; /* flop, turn, river */
  int32_t table_log2;       /* info-set table capacity = 2^table_log2 rows */
  int32_t device;           /* CUDA device ordinal */
  uint64_t seed;            /* Philox key */
  /* ID64 keys only: when > 0, keys are reduced to key_bits bits (plus one), so
     at most 2^key_bits rows exist and identities that share the reduced key share
     a row, as the reference's 2^26 direct-mapped slots do.  0 = full 64 bits.
     When every key fits the table (key_bits <= table_log2; for FNV26 keys,
     table_log2 >= 26), key k owns row k-1 and lookups never probe; otherwise
     the table is open-addressed.  Results are the same either way. */
  int32_t key_bits;
  /* External sampling only: how the traversal kernel walks the updating player's
     tree (MCCFR_FORM_*).  Every form gives bit-identical tables, so this field is
     not part of the game (a v2 checkpoint loads into any form). */
  int32_t traversal_form;
  /* MCCFR_FORM_LEVELS only: capacity of the updating-player node buffer as
     log2 of the node records (80 B each; the seed buffer holds eight times as
     many 8 B entries, the showdown buffer one 24 B record per node); 0 = sized
     from the batch.  Subtrees that do not fit are walked depth first inside the
     same update, and showdowns that do not fit are evaluated where they are
     reached, with the same result. */
  int32_t level_log2;
  int32_t reserved[5];
} mccfr_config;

/* Traversal forms (external sampling). */
enum {
  MCCFR_FORM_AUTO = 0,   /* the level-synchronous form */
  /* one lane per traversal, depth first, with an explicit frame stack
     (persistent lanes pulling traversals from a work counter) */
  MCCFR_FORM_LANES = 1,
  /* level-synchronous: all traversals of the update advance together, one
     level of the updating player's decisions per launch (the opponents'
     sampled actions between two of its decisions are walked within the level),
     then the values return level by level */
  MCCFR_FORM_LEVELS = 2
};

/* Counters and timings of one handle. */
typedef struct mccfr_stats {
  int64_t iterations_done;   /* completed iterations t */
  int64_t launches;          /* player-updates launched */
  int64_t traversals;
  int64_t node_visits;       /* decision nodes visited (V) */
  int64_t traverser_updates; /* updating-player nodes updated (U) */
  int64_t terminals;         /* terminal values computed */
  int64_t hand_evals;        /* rank-chain evaluations */
  int64_t rows_used;         /* -1 here: counting takes a table pass; the size query of
                                mccfr_export_rows (capacity 0) returns the occupied rows */
  int64_t table_capacity;
  int64_t touched_last;      /* rows touched by the last player-update */
  double traverse_ms;        /* summed CUDA-event time of traversal kernels */
  double apply_ms;           /* summed CUDA-event time of apply kernels */
  double last_traverse_ms;
  double last_apply_ms;
  int32_t device_error;      /* sticky kernel error bits */
  /* rows of the last player-update whose regret accumulators (or strategy
     weights of visits off the canonical mask) held values and were written back */
  int32_t wide_rows_last;
  int32_t reserved[6];
} mccfr_stats;

/* One traversal's record from mccfr_step_trace (reference sampling mode). */
typedef struct mccfr_trace {
  uint8_t hole[12];           /* [player*2 + i] */
  uint8_t board[5];
  uint8_t dealer;
  uint8_t n_actions;          /* actions taken along the sampled path */
  uint8_t n_traverser_nodes;
  uint8_t hole_bucket[6];
  uint8_t board_bucket[6][4]; /* [player][street] */
  uint8_t actions[40];        /* action slots, in order */
  float payoff;               /* terminal value for the updating player */
  uint32_t reserved;
} mccfr_trace;

typedef struct mccfr_handle mccfr_handle;

/* ---- configuration ---------------------------------------------------- */
/* Fills *cfg with a preset; the REF8 preset reproduces the constructor defaults of
   GPUCFRTrainer (cfr_gpu.cuh:50-55): 2 players, stack 1000, blinds 10/20, CFR+ and
   linear CFR on, the 8 fixed action slots, 64 Chen buckets, 128 rank buckets, and
   one table row per FNV slot (2^26 rows, direct-mapped, 17.2 GB). */
int mccfr_config_init(mccfr_config* cfg, int preset);
/* Checks a config without a device: MCCFR_OK, or MCCFR_ERR_INVALID_ARG with the
   first rule it breaks written to why (NUL-terminated, at most why_len bytes;
   why may be NULL).  mccfr_create applies the same checks. */
int mccfr_config_validate(const mccfr_config* cfg, char* why, size_t why_len);

/* ---- lifetime (replaces GPUCFRTrainer::GPUCFRTrainer / ~GPUCFRTrainer,
        cfr_gpu.cu:1064-1084) ------------------------------------------- */
int mccfr_create(const mccfr_config* cfg, mccfr_handle** out);
void mccfr_destroy(mccfr_handle* h);

/* ---- hand-rank table (replaces GPUCFRTrainer::load_hand_table,
        cfr_gpu.cu:1086-1104, and hand_eval_init, hand_eval.cpp:88-102) -- */
/* Reads a 32,487,834-entry int32 file and validates it like the reference
   (size + As Ks Qs Js Ts 2c 3d decodes to 7462). */
int mccfr_load_hand_table(mccfr_handle* h, const char* path);
/* Uploads a table already in host memory (n must be MCCFR_HAND_TABLE_ENTRIES). */
int mccfr_set_hand_table(mccfr_handle* h, const int32_t* table, size_t n);
/* Builds the table on the host (no reference counterpart: the reference's
   generator, tools/gen_lookup_table.cpp:63-97, is a stub). */
int mccfr_hand_table_generate(int32_t* out, size_t n);
int mccfr_hand_table_write(const char* path);
int mccfr_hand_class_count(void);

/* ---- training (replaces GPUCFRTrainer::train, cfr_gpu.cu:1244-1378) --- */
/* Runs `iters` iterations; each iteration is one player-update of `batch`
   traversals per player.  Checkpoints to ckpt_path every ckpt_interval
   iterations when ckpt_path is non-empty. */
int mccfr_train(mccfr_handle* h, long long iters, int batch, int verbose,
                const char* ckpt_path, long long ckpt_interval);
/* One player-update (iteration t >= 1, player p) of `batch` traversals.  When
   trace != NULL (reference sampling only), one record per traversal is copied
   to trace[0..batch). */
int mccfr_step(mccfr_handle* h, long long iteration, int player, int batch,
               mccfr_trace* trace);

/* ---- results (replaces get_strategy / num_info_sets_active /
        export_tables / import_tables, cfr_gpu.cu:1383-1459) ------------- */
/* Normalised average strategy, one row per info-set key with a non-zero sum,
   sorted by key.  keys[i] is the reference's u32 dump key (the FNV slot) in
   FNV26 mode and the low 32 bits of the 64-bit key otherwise; keys64 (optional)
   receives full keys.  probs is [capacity][8].  capacity 0 is a size query:
   *count receives the number of occupied rows, an upper bound of the rows
   written (MCCFR_ERR_CAPACITY when it is not 0). */
int mccfr_get_strategy(mccfr_handle* h, uint32_t* keys, uint64_t* keys64,
                       float* probs, size_t capacity, size_t* count);
int mccfr_num_info_sets_active(mccfr_handle* h, long long* out);
/* Every occupied row, sorted by key: regrets [8], strategy sums [8] and the
   number of updates the row received.  capacity 0 is a size query (a counting
   pass; MCCFR_ERR_CAPACITY with *count = rows when there are any). */
int mccfr_export_rows(mccfr_handle* h, uint64_t* keys, float* regrets,
                      float* strategy_sum, uint64_t* visits, size_t capacity,
                      size_t* count);
/* Order-independent checksum of every occupied row, computed on the device
   without copying rows out: the sum (mod 2^64) over rows of a 64-bit mix of the
   row's key, the bits of its regrets and strategy sums, and its update count.
   Two tables with the same rows have the same digest; *rows receives the
   occupied-row count.  No reference counterpart (a test and monitoring aid). */
int mccfr_table_digest(mccfr_handle* h, uint64_t* digest, uint64_t* rows);
/* Dense SoA [8][2^26] tables of the reference (FNV26 mode only). */
int mccfr_export_tables(mccfr_handle* h, float* regrets, float* strategy_sum,
                        size_t n);
int mccfr_import_tables(mccfr_handle* h, const float* regrets,
                        const float* strategy_sum, size_t n);

/* ---- files (replaces save/load_checkpoint, cfr_gpu.cu:1464-1538, and
        strategy_save, strategy.cpp:35-52) ------------------------------ */
/* Checkpoint in the reference's layout: [u64 0x43465247505500][u32 2^26]
   [u32 8] regrets[8][2^26] strategy_sum[8][2^26] (FNV26 mode only). */
int mccfr_save_checkpoint(mccfr_handle* h, const char* path);
int mccfr_load_checkpoint(mccfr_handle* h, const char* path);
/* Checkpoint v2, any key mode: [u64 "MCCFRCK2"][u32 2][u32 sizeof(mccfr_config)]
   [mccfr_config][i64 iterations done][u64 rows] then per row {u64 key,
   f32 regrets[8], f32 strategy_sum[8], u64 visits}, keys ascending.  Unlike the
   reference's checkpoint it keeps the iteration count and the seed, so training
   resumed from it equals uninterrupted training bit for bit.  Loading replaces
   the table's contents and the iteration count; it refuses a file written for a
   different game or abstraction (every config field but device and table_log2)
   and keys that cannot belong to this table.  A subgame's board, pot and ranges
   are not in the file: load a subgame checkpoint into a handle created for the
   same subgame. */
int mccfr_save_checkpoint_v2(mccfr_handle* h, const char* path);
int mccfr_load_checkpoint_v2(mccfr_handle* h, const char* path);
/* Strategy dump v2: [u64 0x53545241540100][u32 2^26][u32 8][u32 n]{u32 key, f32[8]}. */
int mccfr_save_strategy(mccfr_handle* h, const char* path);

/* ---- introspection ----------------------------------------------------- */
int mccfr_get_stats(mccfr_handle* h, mccfr_stats* out);
int mccfr_get_config(mccfr_handle* h, mccfr_config* out);
const char* mccfr_strerror(int status);
/* sizeof(mccfr_config), sizeof(mccfr_stats), sizeof(mccfr_trace), for bindings. */
int mccfr_abi_sizes(size_t* out3);
/* The cudaStream_t (as void*) every kernel of the handle is launched on. */
int mccfr_get_stream(mccfr_handle* h, void** stream);
const char* mccfr_last_error(mccfr_handle* h);

/* ---- showdown evaluation (hand-eval microbenchmark) ----------------------- */
/* ranks[i] = 7-card rank (1..7462) of cards[7*i .. 7*i+6] for i < n, computed on
   the device with the handle's table. */
int mccfr_eval7(mccfr_handle* h, const uint8_t* cards, uint16_t* ranks, size_t n);
/* Same on device buffers (dev_cards, dev_ranks), on the handle's stream; the
   call returns after the kernel finished; *ms receives its CUDA-event time. */
int mccfr_eval7_device(mccfr_handle* h, const uint8_t* dev_cards,
                       uint16_t* dev_ranks, size_t n, float* ms);

/* The level-synchronous form's counts of the handle's last external-sampling
   update: seeds[L] (level 0: the update's traversals) and updating-player
   nodes[L] reached from level L, for L < min(cap, *levels), and the seeds left
   to the depth-first walk because the buffers were full.  *levels = 0 before
   the first such update.  No reference counterpart (a tuning aid). */
int mccfr_level_counts(mccfr_handle* h, uint32_t* seeds, uint32_t* nodes, int cap, int* levels,
                       uint32_t* deferred);

/* ---- showdown microbenchmark ---------------------------------------------
   No reference counterpart as entry points; they time the gathers of the
   reference's rank chains and showdown (cfr_gpu.cu:114-150, 694-753) alone.
   mccfr_deal_eval7: hands i = 0..n-1, each 7 distinct cards drawn on the device
   by partial Fisher-Yates over the 52 cards, j = k + (w_k * (52 - k)) >> 32, with
   the words w_0..w_6 of Philox4x32-10 (key = the handle's seed) at counters
   (i mod 2^32, stream, 0x300, i >> 32) and (..., 0x301, ...); dev_ranks[i] is the
   hand's rank (1..7462).
   mccfr_showdown_masks: the deals of traversals 0..n-1 of update (iteration,
   player), the cards training deals; each seat's 7-card rank with the 5-card
   board walked once for all seats (5 + 2 per seat gathers); dev_masks[t] has bit
   q set when seat q holds the best rank (several bits: a split).  Full game only.
   Both run on the handle's stream and return after the kernel; *ms (optional)
   receives its CUDA-event time. */
int mccfr_deal_eval7(mccfr_handle* h, uint32_t stream, size_t n, uint16_t* dev_ranks, float* ms);
int mccfr_showdown_masks(mccfr_handle* h, long long iteration, int player, size_t n,
                         uint8_t* dev_masks, float* ms);

/* ---- batched form: many tables in one persistent kernel ------------------
   No reference counterpart.  A batch groups existing handles
   (tables), each with its own game, table and schedule; one iteration runs
   phase p = 0..max players-1 as ONE persistent traversal launch over the
   player-p updates of every table with more than p players, pulling
   traversals from a device work queue, then one apply launch for those tables.
   Each table's result is bit-identical to training it alone with the same
   traversals per update.  All handles must be distinct, on one device, hold a
   rank table, use external sampling, and not be used elsewhere while batched. */
typedef struct mccfr_batch mccfr_batch;
typedef struct mccfr_batch_tuning {
  int32_t block;          /* threads per block: 64, 128 or 256 */
  int32_t grab;           /* traversals each lane takes per work-queue grab: 1, 2, 4, 8 */
  int32_t smem_frames;    /* frames of each walk's stack staged in shared memory: 0, 2, 4 */
  int32_t probe_width;    /* table keys loaded per probe step: 1 or 2 */
  int32_t warp_sync;      /* lanes that refill together share one grab of lanes x grab
                             traversals; 1: interleaved (neighbouring lanes take neighbouring
                             traversals), 0: each lane a contiguous run of `grab` */
  int32_t form;           /* MCCFR_BATCH_* (mccfr_batch_train only; rounds always run the
                             persistent kernel) */
  int32_t reserved[2];
} mccfr_batch_tuning;
/* Batch forms.  PERSISTENT: per phase one persistent traversal launch over all
   tables (the fields above tune it).  TABLE_GRAPHS: each table's own update
   kernels (for external sampling the level-synchronous form) as independent
   branches of one CUDA graph per iteration, so the tables' launches run
   concurrently; the tuning fields above are then unused.  Both give every
   table the rows of training it alone. */
enum { MCCFR_BATCH_PERSISTENT = 0, MCCFR_BATCH_TABLE_GRAPHS = 1 };
typedef struct mccfr_batch_stats {
  int64_t iterations;
  int64_t traversals;       /* all tables */
  int64_t node_visits;
  double traverse_ms;       /* CUDA-event time of the persistent traversal launches */
  double total_ms;          /* CUDA-event time of whole iterations */
  int32_t reserved[8];
} mccfr_batch_stats;
/* traversals[i] = traversals per player-update of tables[i]. */
int mccfr_batch_create(mccfr_handle* const* tables, int n_tables, const int* traversals,
                       mccfr_batch** out);
void mccfr_batch_destroy(mccfr_batch* b);
int mccfr_batch_set_tuning(mccfr_batch* b, const mccfr_batch_tuning* t);
int mccfr_batch_get_tuning(mccfr_batch* b, mccfr_batch_tuning* t);
/* Runs `iters` iterations of every table (one CUDA graph per iteration), in the
   form of the batch's tuning: a new batch runs MCCFR_BATCH_TABLE_GRAPHS until
   mccfr_batch_set_tuning or mccfr_batch_autotune (which tunes the persistent
   form) changes it.
   flags bit 1: time every iteration with CUDA events (synchronises per iteration). */
int mccfr_batch_train(mccfr_batch* b, long long iters, int flags);
/* Trains two real iterations per candidate tuning, the list forward then
   backward (results do not depend on the tuning), and keeps the candidate with
   the least summed traversal-kernel time per node visit; *best receives it and
   becomes the batch's tuning (persistent form).
   Candidates: block x grab x smem_frames x warp_sync x probe_width from the
   sets above, limited to the first `max_candidates` (0 = all 144). */
int mccfr_batch_autotune(mccfr_batch* b, int max_candidates, mccfr_batch_tuning* best);
int mccfr_batch_get_stats(mccfr_batch* b, mccfr_batch_stats* out);

/* ---- subgame re-solve and continuous batching -----------------------------
   No reference counterpart.  A subgame starts on the turn or the
   river with a known board, a dead pot shared equally by the players, equal
   stacks (cfg->starting_stack), and one 1326-combo range per player (combo of
   cards lo < hi is index hi*(hi-1)/2 + lo; combos that use a board card get
   weight 0).  Hole combos are drawn from the ranges with card removal; info
   sets are keyed by the exact combo (and the river card on the river).  The
   subgame uses 64-bit keys; either update rule.  The batched form and the
   round API run external sampling only. */
typedef struct mccfr_subgame {
  int32_t street;         /* 2 = turn (4 board cards), 3 = river (5) */
  int32_t pot;            /* chips in the pot; must be a multiple of num_players */
  uint8_t board[5];
  uint8_t pad[3];
  const float* ranges;    /* [num_players][1326] non-negative weights */
} mccfr_subgame;
int mccfr_create_subgame(const mccfr_config* cfg, const mccfr_subgame* sg, mccfr_handle** out);
/* Re-targets a subgame handle to a new subgame, as if it had just been created
   with (cfg, sg): same table capacity (cfg->table_log2) and device; everything
   else may differ.  The table is zeroed and the allocations are kept, so a
   server can reuse finished requests' tables without freeing and allocating. */
int mccfr_subgame_reset(mccfr_handle* h, const mccfr_config* cfg, const mccfr_subgame* sg);
/* Makes h use src's device rank table instead of uploading its own (src must
   outlive h).  Valid for subgames and for tables without rank-CDF buckets or
   with the same bucket counts as src. */
int mccfr_share_hand_table(mccfr_handle* h, mccfr_handle* src);
/* One player-update of each listed table, all in one persistent traversal
   launch: the serving step of continuous batching.  Each table advances its
   own (iteration, player) and its iteration count after its last player.
   traversals[i] = traversals of table i's update; tuning may be NULL. */
int mccfr_batch_round(mccfr_handle* const* tables, int n, const int* traversals,
                      const mccfr_batch_tuning* tuning);
/* The (iteration, player) the table's next update will run, and the number of
   completed iterations. */
int mccfr_get_progress(mccfr_handle* h, long long* next_iteration, int* next_player,
                       long long* iterations_done);

/* ---- evaluation without device allocation --------------------------------
   No counterpart in the reference.  For callers that cannot allocate device
   memory (code inside a framework that owns every device allocation, or a
   process that must not grow its device footprint): the same 7-card evaluation
   as mccfr_eval7, with its staging in a static device array of
   MCCFR_EVAL7_STATIC_MAX_HANDS hands (about 2.25 MiB, held by every GPU that
   loads the library until exit).  dev_table is the caller's device copy of the
   32,487,834-entry rank table and must be device (or managed) memory: a host
   pointer returns MCCFR_ERR_INVALID_ARG; cards (7 per hand, 0..51) and ranks
   are host buffers; runs on the current device.  n above the maximum returns
   MCCFR_ERR_INVALID_ARG.  The first call on a device looks up the array's
   address and must come before any stream capture; the address holds for the
   life of the device's context (do not call again on a device after
   cudaDeviceReset).  Calls share the array, so calls that overlap on the GPU
   race: serialise them. */
#define MCCFR_EVAL7_STATIC_MAX_HANDS (1u << 18)
int mccfr_eval7_static(const int32_t* dev_table, const uint8_t* cards, uint16_t* ranks, size_t n);

/* ---- heads-up best response and exploitability -------------------------
   No counterpart in the reference (its PROPOSAL.md:99 calls exploitability too
   expensive; play is measured against scripted bots).  An exact best response
   in double precision on host threads, for heads-up games only: the full game
   from the blinds (rank-CDF postflop buckets, which are suit-invariant, so
   flops are enumerated up to suit permutation), or a turn/river subgame.  The
   evaluated strategy is the rows' strategy sums normalised over each node's
   legal slots; a missing row, or one whose legal sum is 0, plays uniformly.
   The best responder plays the real game: it sees its own cards, the board
   and the action history.  Chance follows the trainer's deal: uniform hole
   cards and a uniform dealer in the full game; in a subgame the hole combos
   drawn with probability proportional to the product of the quantised range
   weights over disjoint pairs (the deal's accepted draw), then a uniform
   river card. */
#define MCCFR_BR_VERBOSE 1   /* progress on stderr */
#define MCCFR_BR_ISO_CHECK 2 /* full game: recompute some suit-permuted flops directly */
typedef struct mccfr_br_options {
  int32_t threads;      /* host threads; 0 = all */
  int32_t flop_stride;  /* full game: 1 = every flop class (exact); k > 1 = every
                           k-th class, reweighted (an estimate, exact = 0) */
  int32_t flags;
  int32_t reserved[5];
} mccfr_br_options;
typedef struct mccfr_exploit {
  double br_value[2];       /* chips per game: player p best-responding to the other */
  double profile_value[2];  /* chips per game: the average-strategy profile, player p */
  double exploitability;    /* (br_value[0] + br_value[1]) / 2, chips per game */
  double mbb_per_game;      /* exploitability in milli-big-blinds per game */
  double seconds;           /* host time of the computation */
  double iso_check;         /* MCCFR_BR_ISO_CHECK: largest difference found, relative to the
                               largest value of the flop compared; else 0 */
  long long boards;         /* river boards evaluated (flop classes count once) */
  long long rows;           /* strategy rows supplied */
  long long nodes;          /* public-tree nodes (all dealer seats) */
  int32_t threads;
  int32_t exact;
  int32_t reserved[4];
} mccfr_exploit;
void mccfr_br_options_init(mccfr_br_options* opt);
/* From host data: cfg (num_players 2), sg NULL for the full game, the rank
   table, and rows as mccfr_export_rows writes them (keys, strategy_sum [rows][8]). */
int mccfr_best_response(const mccfr_config* cfg, const mccfr_subgame* sg, const int32_t* hand_table,
                        size_t table_entries, const uint64_t* keys, const float* strategy_sum, size_t rows,
                        const mccfr_br_options* opt, mccfr_exploit* out);
/* The same for a trainer's current average strategy (its rows and rank table
   are copied from the device). */
int mccfr_exploitability(mccfr_handle* h, const mccfr_br_options* opt, mccfr_exploit* out);
/* Rank-CDF bucket LUT of n-card hands (n = 5, 6, 7) from the exact rank
   histogram, as the trainer builds it: out[rank] for rank 0..7462. */
int mccfr_rank_cdf_lut(const int32_t* hand_table, size_t table_entries, int ncards, int buckets, uint8_t* out);

#ifdef __cplusplus
}
#endif
#endif /* MCCFR_H */
