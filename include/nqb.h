/*
 * nqb.h - C ABI of the B200 N-Queens counter (libnqb.so).
 *
 * The library counts N-Queens solutions with the DoubleSweep-light search of
 * fillpant/GPU-N-Queens: a host-built pool of every valid placement of the first
 * `depth` rows (row 0 restricted to the left half of the board, counts of
 * left-half states doubled), then one depth-first search per pool state with
 * unit-row propagation, summed into a uint64 count.
 *
 * Every entry point returns an NQB_* status code and never exits the process
 * (the reference's FAIL_IF / CHECK_CUDA_ERROR exit; deffinitions.cuh:148-156).
 * Plain pointers and sizes only; no C++ or torch types cross this boundary.
 * Calls are re-entrant: each call owns its own stream and device buffers.
 */
#ifndef NQB_H
#define NQB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NQB_VERSION 10200 /* 1.2.0 */

/* Board sizes.  The reference accepts 7 < N < 32 (deffinitions.cuh:116-118);
 * this library accepts 4..31.  Counts are exact in uint64 up to N = 28. */
#define NQB_MIN_N 4
#define NQB_MAX_N 31

/* ---- status codes ------------------------------------------------------ */
#define NQB_OK 0
#define NQB_E_INVALID 1  /* bad argument: n, depth, null pointer, bad state      */
#define NQB_E_NOMEM 2    /* host allocation failed (reference: errno ENOMEM)      */
#define NQB_E_CUDA 3     /* CUDA runtime error (reference: CHECK_CUDA_ERROR exit) */
#define NQB_E_NODEVICE 4 /* no usable sm_100 device (reference: check_gpu_compatibility) */
#define NQB_E_RANGE 5    /* size beyond a supported limit (reference: errno ERANGE) */
#define NQB_E_STALL 6    /* a device-side bounded wait ran out                    */
#define NQB_E_DEVICE 7   /* a device-side bounds check failed                     */
#define NQB_E_MODEL 8    /* learned cost model missing or not trained            */
#define NQB_E_IO 9       /* a file could not be opened, read or written          */
#define NQB_E_FORMAT 10  /* a state file is malformed, or of another version or
                            generation flags (reference reader: -3 / -4)          */

/* ---- search state ------------------------------------------------------ */
/*
 * One search state: rows [0, row) hold queens, the search continues at `row`.
 * 16 bytes, the unit of the pool in host memory and in HBM.
 *
 *   cols   bit c set <=> a queen stands in column c
 *   ldiag  bit c set <=> column c of row `row` is attacked along a diagonal
 *          whose column grows with the row (each row down shifts it left 1)
 *   rdiag  same for diagonals whose column shrinks with the row (shift right 1)
 *   weight multiplier applied to this state's completion count: 2 for a row-0
 *          queen in the left half (column < n/2), 1 for the middle column of an
 *          odd board, 1 for arbitrary boards solved without mirror weighting
 *
 * Relation to the reference's nq_state_t (n_queens.cuh:100-113; diagonals.cuh:8-34)
 * at curr_row = r:  cols = queens_in_columns,
 *   rdiag = (uint32)(diagonal >> r),  ldiag = (uint32)(antidiagonal >> (N - r)).
 */
typedef struct nqb_state {
    uint32_t cols;
    uint32_t ldiag;
    uint32_t rdiag;
    uint8_t row;
    uint8_t n;
    uint8_t weight;
    uint8_t flags; /* reserved, must be 0 */
} nqb_state;

/* ---- options and statistics ------------------------------------------- */
#define NQB_FORM_PLAIN 0   /* one thread per state, static assignment            */
#define NQB_FORM_BATCHED 1 /* persistent kernel, device work queue, re-splitting */

struct nqb_model; /* learned cost model, see nqb_model_create */

typedef struct nqb_opts {
    int device;           /* CUDA device ordinal (default 0)                           */
    int form;             /* NQB_FORM_PLAIN or NQB_FORM_BATCHED                        */
    int block_size;       /* threads per block; 0 = library default                    */
    int count_unit_nodes; /* 1: also count unit-propagation placements (slower kernel) */
    int max_split_rounds; /* batched form with a model: rounds of splitting the items
                             predicted larger than the split threshold into their
                             children; -1 = library default (3), 0 = no splitting       */
    int split_factor;     /* batched form with a model: split threshold = predicted total
                             nodes / (resident lanes x split_factor); 0 = default (4)   */
    const struct nqb_model* model; /* batched form: learned cost model; the queue is
                             ordered largest predicted first and large items are split.
                             NULL = FIFO: items in the given order, no splitting        */
    int host_pool;        /* nqb_count_ex: 1 = build the pool on the host and copy it to
                             the GPU (the reference's way); 0 = build it on the GPU    */
    int autotune;         /* nqb_count_ex: 1 = pick form, block size and split factor with
                             nqb_tune_count on a 1/64 sample of the pool first          */
    int count_lane_steps; /* 1: run the instrumented search kernel that also counts its
                             lane-steps (nqb_stats.placed_lane_steps, lane_step_slots)  */
    int sched_cost;       /* batched form without a model: 0 = FIFO; a model-free cost drives
                             the learned schedule's split-and-order steps instead of the
                             network (its ablation): 1 = log2(1 + free columns x rows
                             left), 2 = sum over the rows below of log2(1 + cells left
                             free there by the queens above)                           */
    int reserved[4];
} nqb_opts;

typedef struct nqb_stats {
    uint64_t states;     /* pool states (or boards) solved                         */
    uint64_t nodes;      /* queen placements at rows >= each state's start row     */
    uint64_t unit_nodes; /* of which unit-row propagations; UINT64_MAX if not counted */
    double gen_ms;       /* host pool generation                                   */
    double h2d_ms;       /* host->device copy of the pool                          */
    double kernel_ms;    /* device time of the search kernels (CUDA events)        */
    double wall_ms;      /* whole call                                             */
    uint32_t pregen_depth;
    uint32_t kernel_launches;
    uint64_t items;      /* items the search kernel was given (after learned splitting) */
    double sched_ms;     /* learned scheduling: prediction, splitting, ordering        */
    uint32_t block_size; /* threads per block of the search launch                        */
    int32_t form;        /* search form used (NQB_FORM_*)                                  */
    /* With nqb_opts.count_lane_steps (else 0): lane-steps of the search loop that placed a
     * queen, and lane-step slots issued (32 per warp step).  Their ratio is the search's
     * warp execution efficiency in active lanes. */
    uint64_t placed_lane_steps;
    uint64_t lane_step_slots;
} nqb_stats;

/* Fills `opts` with the defaults (device 0, plain form, library block size). */
void nqb_default_opts(nqb_opts* opts);

/* Human-readable text for a status code (static storage). */
const char* nqb_strerror(int status);

int nqb_version(void);

/* Checks that `device` is an sm_100 GPU this library can run on.
 * Replaces check_gpu_compatibility (GPU_NQueens.cu:23-54). */
int nqb_device_check(int device);

/* Device buffers of a call (the pool, its level buffers, scratch) come from the library's
 * own stream-ordered memory pool on that device and stay cached for the next call instead
 * of being unmapped; this returns the cached memory of `device` to the driver. */
int nqb_trim_device_memory(int device);

/* Test hook for the error paths: makes one allocation of the library fail as if memory had
 * run out.  after >= 0: the library's next `after` allocations succeed and the one after
 * them fails (once; the hook is then off); after < 0 turns the hook off.  Counted are the
 * library's own device buffers, pinned host buffers and host arrays (pools, state-file
 * placements), from every thread; allocations inside the C++ standard library are not.
 * Returns the countdown it replaces: -1 when the hook was off or has fired, else the number
 * of allocations that were still to succeed.  A call whose allocation fails returns
 * NQB_E_NOMEM, releases what it had allocated and leaves the library usable; no entry point
 * lets a C++ exception escape (one from the standard library is NQB_E_NOMEM too). */
long long nqb_debug_fail_allocation(long long after);

/* Measures the integer lane-ops per second `device` sustains (the search kernels'
 * roofline denominator): every SM at full occupancy running independent chains of one
 * integer instruction kind.  per_kind (optional, 4 entries): LOP3, add, IMAD, and LOP3 and
 * IMAD alternated; *best = the largest.  Takes about 0.1 s. */
int nqb_measure_int32_peak(int device, double* best, double* per_kind);

/* Number of CUDA devices visible to the process (NQB_E_NODEVICE when none). */
int nqb_device_count(int* count);

/* ---- the drop-in count -------------------------------------------------- */
/*
 * Counts all solutions of the n-queens puzzle: builds the pool of every valid
 * `pregen_depth`-row prefix (row-0 queen in columns < ceil(n/2), prefixes whose
 * next row has no free column dropped), solves it on the GPU and returns the
 * mirror-weighted uint64 total.  1 <= pregen_depth <= n-1.
 * Replaces nq_generate_states_rowlock (n_queens.cuh:119) followed by
 * solve() / gpu_solver_driver (NQ_solver.cu:192-209, GPU_NQueens.cuh:13).
 */
int nqb_count(unsigned n, unsigned pregen_depth, uint64_t* count);

/* nqb_count with options (NULL = defaults) and statistics (may be NULL). */
int nqb_count_ex(unsigned n, unsigned pregen_depth, const nqb_opts* opts, uint64_t* count,
                 nqb_stats* stats);

/* ---- the pool ----------------------------------------------------------- */
/*
 * Builds the pool on the host: the same prefixes, in the same order, as the
 * reference's gen_states_threaded_rowlock (n_queens.cu:235-315): row-0 columns
 * 0..ceil(n/2)-1 in turn, each followed by its prefixes in depth-first order,
 * lowest column first.  *states is allocated by the library (16-byte aligned);
 * release it with nqb_free.  Replaces nq_generate_states_rowlock (n_queens.cuh:119).
 */
int nqb_generate_pool(unsigned n, unsigned depth, nqb_state** states, uint64_t* count);

/* Same, into a caller buffer of `capacity` states.  With buf == NULL only the
 * size is computed.  Returns NQB_E_RANGE if the pool does not fit. */
int nqb_generate_pool_into(unsigned n, unsigned depth, nqb_state* buf, uint64_t capacity,
                           uint64_t* count);

/* Same pool built on the GPU (level-by-level expansion, same order), in a device buffer
 * allocated by the library on `stream` (a cudaStream_t; stream-ordered allocation):
 * release it with nqb_free_device.  *count may be 0.  Asynchronous apart from the level
 * sizes it reads back. */
int nqb_generate_pool_device(unsigned n, unsigned depth, nqb_state** d_states, uint64_t* count, void* stream);
void nqb_free_device(void* d_ptr, void* stream);
/* Same, copied into a caller device buffer of `capacity` states (NQB_E_RANGE, with *count
 * set, when it does not fit). */
int nqb_generate_pool_device_into(unsigned n, unsigned depth, nqb_state* d_buf, uint64_t capacity, uint64_t* count,
                                  void* stream);

/* ---- placements, state files and count-target sizing ----------------- */
/*
 * A partial board as the reference's state files hold it: the column of the queen in
 * each row [0, row) (nq_state_t.queen_at_index / curr_row, n_queens.cuh:100-113);
 * col[r] for r >= row is 0xFF (the reference's UNSET_QUEEN_INDEX).  32 bytes.
 */
typedef struct nqb_placement {
    uint8_t n;
    uint8_t row;
    uint8_t col[30];
} nqb_placement;

/* The pool of nqb_generate_pool as placements, same states in the same order;
 * release with nqb_free. */
int nqb_generate_pool_placements(unsigned n, unsigned depth, nqb_placement** placements, uint64_t* count);

/* Rebuilds search states from placements by placing each queen in turn (the state-file
 * reader's place_queen_at loop, nq_utils.cu:232-240).  mirror_weight != 0: weight 2 when
 * the row-0 queen is left of centre, else 1 (GPU_NQueens.cu:354-357); 0: weight 1.
 * NQB_E_INVALID for n out of range, row >= n or row > 30, or a column >= n. */
int nqb_states_from_placements(const nqb_placement* placements, uint64_t count, int mirror_weight, nqb_state* out);

/* State files (.nqsf; nq_utils.cu:127-259).  Layout, little-endian:
 *   [u32 version = 1, u64 flags]   generation-flags header (COMPILATION_PARAMETER_FLAGS_
 *                                  IN_STATE_FILES, on in the reference's default build)
 *   u8 n, u8 locked_row, u64 total
 *   per distinct row r, ascending: u8 r, u64 cnt, then cnt x r column bytes, the states
 *   of that row in input order.
 * flags: bit 0 experimental optimisations, bit 1 mirror elimination; the reference's
 * default build, and this library, write NQB_STATE_FILE_FLAGS. */
#define NQB_STATE_FILE_VERSION 1
#define NQB_STATE_FILE_FLAGS 3ull

typedef struct nqb_state_file {
    uint32_t version;    /* 0 when the file has no header                          */
    uint64_t flags;
    unsigned n;
    unsigned locked_row;
    uint64_t count;
} nqb_state_file;

/* Writes `count` placements (all of board size n) with the given locked row.  count == 0
 * is NQB_E_INVALID, as the reference writer refuses an empty buffer.  header != 0 writes
 * the version/flags header. */
int nqb_write_state_file(const char* path, const nqb_placement* placements, uint64_t count, unsigned n,
                         unsigned locked_row, int header);

/* Reads a state file.  expect_n != 0 requires that board size (the reference asserts
 * it).  With a header, version != 1 or flags != NQB_STATE_FILE_FLAGS is NQB_E_FORMAT
 * (the reference returns -3 / -4); so is a truncated file, a segment row >= n, a column
 * >= n, or segment counts that do not add up to the total.  *placements is allocated by
 * the library (release with nqb_free) and *info filled. */
int nqb_read_state_file(const char* path, int header, unsigned expect_n, nqb_state_file* info,
                        nqb_placement** placements);

/*
 * Count-target pool sizing (nq_generate_states -> gen_states_threaded, n_queens.cu:128-219,
 * :397-406; deffinitions.cuh:57,61): the lock row the reference picks for a requested
 * pool size `how_many`.  Hard limit = (uint64)(how_many * 1.2); the first row tried is
 * floor(log(how_many) / log(n)), at most n - 1 (NQB_E_INVALID when it is 0, i.e.
 * how_many < n).  Ever deeper rows are tried while a row's pool is no smaller than the
 * previous one, the row is at most n and the pool is within the hard limit; the answer
 * is the row tried before the last.  NQB_E_RANGE when the first row already exceeds the
 * limit.  If one row-0 column's pool reaches the limit the search ends there with the
 * previous row (limit_hit = 1; the reference's own error path, n_queens.cu:176-180).
 * Lock row 1 stands for the reference's row-1 pool, whose states hold two queens:
 * pool_depth is then 2.
 */
typedef struct nqb_target {
    unsigned lock_row;        /* the locked row the reference reports and writes           */
    unsigned pool_depth;      /* queens per pool state: lock_row, or 2 when lock_row == 1   */
    uint64_t count;           /* pool states                                               */
    uint64_t hard_limit;
    unsigned first_row;       /* rows first_row .. first_row + tried - 1 were tried          */
    unsigned tried;
    int limit_hit;
    unsigned reserved;
    uint64_t tried_count[32]; /* pool states of each tried row                             */
} nqb_target;

int nqb_pool_for_target(unsigned n, uint64_t how_many, nqb_target* target);

/* ---- launch autotuner ------------------------------------------------------------ */
/*
 * Picks the launch of a full count by timing: for each depth in `depths` the pool is built
 * on the GPU and every `sample_div`-th state taken (an unbiased 1/sample_div sample of the
 * count's work, in pool order); on it every candidate runs twice and the faster time
 * counts.  Candidates: both forms x block sizes 64, 128, 256, and with opts->model the
 * batched form's split factors 1, 4, 16.  All candidates of a depth must agree on the
 * sample's count (else NQB_E_DEVICE).  The fastest is reported with the candidates tried
 * (the first 64 of them listed).
 */
typedef struct nqb_tune_entry {
    unsigned depth;
    int form;
    int block_size;
    int split_factor;
    double ms;
} nqb_tune_entry;

typedef struct nqb_tune_result {
    unsigned depth;          /* the fastest candidate                                  */
    int form;
    int block_size;
    int split_factor;
    double best_ms;          /* its time on the sample                                  */
    uint64_t sample_states;  /* states in its depth's sample                            */
    unsigned sample_div;
    unsigned n_tried;
    nqb_tune_entry tried[64];
} nqb_tune_result;

int nqb_tune_count(unsigned n, const unsigned* depths, unsigned n_depths, const nqb_opts* opts,
                   unsigned sample_div, nqb_tune_result* out);

/* Sum of the pool's weights: the number of full-board prefixes it stands for. */
int nqb_pool_weighted_size(unsigned n, unsigned depth, uint64_t* weighted);

void nqb_free(void* p);

/*
 * Seeded random valid partial boards (no counterpart in the reference, which has no
 * batch mode): board i draws n uniformly from [n_min, n_max] and a depth uniformly
 * from [d_min, d_max], then fills rows 0..depth-1 in order, each with a column drawn
 * uniformly among the row's free columns, restarting the board when a row before the
 * depth has no free column.  Row `depth` may be dead (the board then has 0
 * completions).  Weight 1.  Random stream: splitmix64 from `seed`; a draw in [0, k)
 * is ((next >> 32) * k) >> 32.
 */
int nqb_sample_boards(uint64_t seed, uint64_t count, unsigned n_min, unsigned n_max, unsigned d_min,
                      unsigned d_max, nqb_state* out);

/* ---- solving states ---------------------------------------------------- */
/*
 * Solves `count` states held in host memory on the GPU and returns the sum of
 * weight x completions.  States may mix board sizes and start rows.
 * Replaces gpu_solver_driver (GPU_NQueens.cuh:13) for the library's state layout.
 */
int nqb_solve_states(const nqb_state* states, uint64_t count, const nqb_opts* opts,
                     uint64_t* total, nqb_stats* stats);

/* nqb_solve_states over several GPUs (the reference driver's configs list, GPU_NQueens.cu:
 * 56-175): device k of `devices` gets a contiguous slice of floor(count / ndev) states, the
 * last also the remainder (:84-90), each solved by its own host thread; the counts are
 * summed on the host (:164-171).  Devices may repeat; opts->device is ignored.  stats: sums
 * of states, nodes, launches and items, and the slowest device's h2d and kernel times. */
int nqb_solve_states_multi(const nqb_state* states, uint64_t count, const int* devices, unsigned ndev,
                           const nqb_opts* opts, uint64_t* total, nqb_stats* stats);

/*
 * Per-board completion counts: out[i] = weight_i x completions of boards[i]
 * (pass weight 1 for plain counts; no mirror weighting is implied).
 * Boards may mix n (4..31) and row.  Used for batches of uneven partial boards.
 */
int nqb_solve_batch(const nqb_state* boards, uint64_t count, const nqb_opts* opts,
                    uint64_t* out, nqb_stats* stats);

/* Size in bytes of the reference's nq_state_t for board size n
 * ({u64 diagonal, u64 antidiagonal, u32 cols, char curr_row, u8 queen_at_index[n]},
 * 8-byte aligned; n_queens.cuh:100-113). */
size_t nqb_ref_state_size(unsigned n);

/*
 * Converts `count` reference nq_state_t records (stride nqb_ref_state_size(n)) to
 * library states.  With mirror_weight != 0 the weight is 2 when queen_at_index[0]
 * < n/2, else 1 (GPU_NQueens.cu:354-357,437-439); otherwise 1.
 */
int nqb_states_from_ref(unsigned n, const void* ref_states, uint64_t count, int mirror_weight,
                        nqb_state* out);

/*
 * Direct replacement for gpu_solver_driver (GPU_NQueens.cu:56-175) on a buffer of
 * reference nq_state_t records generated for lock row `locked_row` (every state
 * has curr_row == locked_row): mirror-weighted total in *total.
 */
int nqb_solve_ref_states(unsigned n, const void* ref_states, uint64_t count, unsigned locked_row,
                         const nqb_opts* opts, uint64_t* total);

/* ---- device-resident launches (inputs already in HBM) ------------------- */
/*
 * Plain form on states already in device memory: one thread per state.
 * d_out points to 4 device uint64 words {weighted count, nodes, unit nodes, error
 * flags}; the kernel adds into them, so zero them first.  Unit nodes are counted
 * only with count_unit_nodes != 0.  stack_depth bounds the pending rows one search
 * can hold: the largest number of free columns of any state minus one (0 = 30);
 * a search that needs more sets error flag 1 in d_out[3].  `stream` is a
 * cudaStream_t (NULL = legacy default stream).  Asynchronous: returns after the
 * launch.  The kernel launch of gpu_solver_driver (GPU_NQueens.cu:128-138).
 */
int nqb_plain_launch(const nqb_state* d_states, uint64_t count, uint64_t* d_out, int block_size,
                     int count_unit_nodes, unsigned stack_depth, void* stream);

/*
 * Batched form on items already in device memory: a persistent kernel (one wave of
 * blocks over all SMs of the current device) that hands items to idle lanes from a
 * queue and, once the queue is empty, splits the pending rows of busy lanes onto
 * idle ones.  d_order (optional) gives the queue order as item indices; d_head is a
 * device uint32 queue head (scratch) that must be zero at launch; d_out as for
 * nqb_plain_launch (unit nodes are not counted).  count <= 2^31.  Asynchronous.
 */
int nqb_batched_launch(const nqb_state* d_items, uint64_t count, const uint32_t* d_order, uint32_t* d_head,
                       uint64_t* d_out, int block_size, unsigned stack_depth, void* stream);

/* Scratch of nqb_batched_launch_ex with the library's own steal ring (65,536 slots). */
#define NQB_BATCHED_SCRATCH_BYTES (64ull + 32ull * 65536ull)

/*
 * The batched form with work stealing across warps.  d_scratch (16-byte aligned, zeroed
 * before every launch) holds 64 bytes of control words and a ring of 32-byte slots:
 * warps that run out of work take rows from the ring, and while such warps exist the
 * other warps publish their lanes' shallowest pending rows into it, so a long subtree
 * spreads over the whole GPU.  The ring uses the largest power of two of slots that fits
 * (NQB_BATCHED_SCRATCH_BYTES: 65,536); scratch_bytes below 64 + 2 x 32 launches without
 * the ring, exactly as nqb_batched_launch.  d_lane_stats (optional): two device uint64
 * words, zeroed first, that the instrumented kernel adds {lane-steps that placed a queen,
 * lane-step slots} into.  wait_limit: polls without progress after which a waiting warp
 * gives up (0 = the library default, about 2 s); a launch in which one gave up sets error
 * flag 4 in d_out[3] (NQB_E_STALL from the calls that read it) and its counts are not to
 * be used.  count <= 2^31.  Asynchronous.  Extends the kernel launch of gpu_solver_driver
 * (GPU_NQueens.cu:128-138), which has no work sharing.
 */
int nqb_batched_launch_ex(const nqb_state* d_items, uint64_t count, const uint32_t* d_order, void* d_scratch,
                          uint64_t scratch_bytes, uint64_t* d_out, uint64_t* d_lane_stats, int block_size,
                          unsigned stack_depth, unsigned wait_limit, void* stream);

/* ---- learned cost model ------------------------------------------------ */
/*
 * An MLP (NQB_MODEL_INPUTS -> 128 -> 128 -> 1, GELU) predicting log2(1 + nodes) of the
 * search below a state, from the state's masks (free columns, both diagonals: 3 x 32
 * bits), n/32, row/32, free columns/32 and next-row candidates/32.  Trained on the GPU by
 * the library's own kernels (FP16 operands, FP32 accumulation, Adam) on node counts the
 * solver records (nqb_record_nodes).  It only orders and splits the batched form's queue;
 * counts never depend on it.  No counterpart in the reference.
 */
#define NQB_MODEL_INPUTS 112
#define NQB_MODEL_PARAMS 31105 /* W1 112x128 | b1 | W2 128x128 | b2 | w3 128 | b3, row-major [in][out] */

typedef struct nqb_model nqb_model;

typedef struct nqb_train_opts {
    int epochs;    /* passes over the data (default 8)  */
    int batch;     /* rows per Adam step (default 4096)  */
    float lr;      /* Adam learning rate (default 1e-3)  */
    int reserved0;
    uint64_t seed; /* shuffling seed (default 1)         */
    int reserved[8];
} nqb_train_opts;

/* Creates a model on `device` with seeded Glorot-uniform weights. */
int nqb_model_create(int device, uint64_t seed, nqb_model** model);
void nqb_model_destroy(nqb_model* model);
int nqb_model_get_params(const nqb_model* model, float* params /* NQB_MODEL_PARAMS */);
int nqb_model_set_params(nqb_model* model, const float* params /* NQB_MODEL_PARAMS */);
/* Host computation of the input features (count x NQB_MODEL_INPUTS floats). */
int nqb_model_features(const nqb_state* states, uint64_t count, float* features);
/* Predicted log2(1 + nodes) per state (fused tensor-core inference kernel). */
int nqb_model_predict(const nqb_model* model, const nqb_state* states, uint64_t count, float* log2_nodes);
/* Same, with an explicit bound on the wait for each tensor-core product: `wait_limit`
 * non-blocking probes of its completion barrier (0 = the library's default bounded wait).
 * A wait that runs out drains the products in flight (a second bounded wait), frees the
 * block's tensor memory and makes the call return NQB_E_STALL with `log2_nodes` undefined;
 * the model and the device stay usable.  If the drain runs out as well, products may still
 * have been writing the tensor memory when it was freed: the call returns NQB_E_DEVICE, and
 * later results on that device are not to be trusted.  A bound of 1 forces the first path
 * (tests); the default drain bound is seconds. */
int nqb_model_predict_ex(const nqb_model* model, const nqb_state* states, uint64_t count, float* log2_nodes,
                         uint32_t wait_limit);
/* One forward and backward pass over all `count` rows (count <= 2^20): mean squared
 * error and its gradient (NQB_MODEL_PARAMS floats), without updating the weights. */
int nqb_model_loss_grad(nqb_model* model, const nqb_state* states, const float* targets, uint64_t count,
                        float* loss, float* grad);
/* Trains on (state, target) pairs; epoch_loss (optional) receives each epoch's mean loss. */
int nqb_model_train(nqb_model* model, const nqb_state* states, const float* targets, uint64_t count,
                    const nqb_train_opts* opts, float* epoch_loss);
/* Per-state search nodes and (weighted) completions, recorded by the batched kernel: the
 * training labels of the cost model. */
int nqb_record_nodes(const nqb_state* states, uint64_t count, const nqb_opts* opts, uint64_t* nodes,
                     uint64_t* counts);

/* ---- batch plans: one board set solved repeatedly through a CUDA graph --- */
/*
 * A plan uploads `count` boards once, builds the batched form's schedule (with
 * opts->model, or a model-free opts->sched_cost: splitting and largest-first order) and
 * captures the solve (zeroing of the outputs and the launch scratch, one persistent-kernel
 * launch with work stealing, read-back) into a CUDA graph.  With autotune != 0 every
 * candidate (block size 64/128/256 x split factor 1/4/16 when a cost is given) is first
 * timed once on a stride sample of about 4,096 boards, and the fastest is captured for
 * the whole batch.  The model is only read during creation.  No counterpart in the
 * reference.
 */
typedef struct nqb_batch_plan nqb_batch_plan;
int nqb_batch_plan_create(const nqb_state* boards, uint64_t count, const nqb_opts* opts, int autotune,
                          nqb_batch_plan** plan);
/* Replays the graph; out[i] = weight_i x completions of board i (as nqb_solve_batch). */
int nqb_batch_plan_run(nqb_batch_plan* plan, uint64_t* out, nqb_stats* stats);
/* The configuration the plan runs with. */
int nqb_batch_plan_config(const nqb_batch_plan* plan, int* block_size, int* split_factor, uint64_t* items);
void nqb_batch_plan_destroy(nqb_batch_plan* plan);

/* Scratch held by nqb_batched_launch_static on every GPU that loads the library. */
#define NQB_STATIC_SCRATCH_BYTES 256
/* Largest item count nqb_batched_launch_static accepts (its 32-bit queue head). */
#define NQB_STATIC_MAX_ITEMS (1ull << 31)

/*
 * nqb_batched_launch for callers that cannot allocate device memory.  It has no
 * counterpart in the reference.
 *
 * Some callers may not call cudaMalloc or cudaFree at all: code whose framework hands
 * out all device memory through its own caching allocator (a raw cudaMalloc beside it
 * fragments or oversubscribes what the framework budgets), and code that must not stall
 * the GPU (cudaFree synchronises the whole device).  This entry point needs no scratch
 * buffer from them: the queue head lives in a 256-byte array of this library's device
 * memory (NQB_STATIC_SCRATCH_BYTES), which every GPU that loads the library holds until
 * the process exits.  The caller still passes the items, the optional order and the four
 * result words, exactly as for nqb_batched_launch; this call allocates nothing and calls
 * no allocating library routine.  It launches without the steal ring of
 * nqb_batched_launch_ex (warps share work only inside themselves).
 *
 * - The first call on a device looks the array's device address up
 *   (cudaGetSymbolAddress) with that device current, which loads the library's module on
 *   the device if nothing has yet.  The address is kept per device and context: after a
 *   device reset (cudaDeviceReset) the next call looks it up again, so that call is a
 *   first call too.
 * - Each call clears the queue head on `stream` before launching (the array keeps
 *   whatever the previous call left).  All calls on a device share the one array, so
 *   calls whose work overlaps on the GPU race: serialise them, e.g. on one stream.
 * - count > NQB_STATIC_MAX_ITEMS returns NQB_E_RANGE without launching.
 */
int nqb_batched_launch_static(const nqb_state* d_items, uint64_t count, const uint32_t* d_order,
                              uint64_t* d_out, int block_size, unsigned stack_depth, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NQB_H */
