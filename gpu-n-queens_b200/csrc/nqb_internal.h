// Internal declarations shared by the translation units of libnqb.so.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "nqb.h"

// Returns from the enclosing function with the status of `expr` unless it is NQB_OK.
#define NQB_TRY(expr)                \
    do {                             \
        const int s_ = (expr);       \
        if (s_ != NQB_OK) return s_; \
    } while (0)

// Handler of the C ABI entry points, each written as a function-try-block
// (`int nqb_f(...) try { ... } NQB_ABI_CATCH`), so that no C++ exception crosses the C ABI.
// The library throws none of its own.  The standard library's containers, `new` and
// std::thread throw when host memory or threads run out (std::bad_alloc, std::length_error,
// std::system_error); the entry point then returns NQB_E_NOMEM.  The body's objects are
// destroyed on the way out, so the device buffers, streams and events they own are released.
#define NQB_ABI_CATCH       \
    catch (...) {           \
        return NQB_E_NOMEM; \
    }

namespace nqb {

inline uint32_t board_mask(unsigned n) { return n >= 32 ? 0xFFFFFFFFu : ((1u << n) - 1u); }

// A state the kernels accept: 1 <= n <= 31, flags 0, no column outside the board.
bool state_valid(const nqb_state& s);

// Host pool generator (pool.cpp).  With buf == nullptr only count/weighted are computed.
// Returns NQB_E_RANGE when the pool holds more than `capacity` states.
// Host generator with optional outputs: states (buf), placements (pbuf), the pool size
// of each row-0 column (per_first_col, ceil(n/2) entries).  With buf and pbuf both null
// only the sizes are computed.
int generate_pool_ex(unsigned n, unsigned depth, nqb_state* buf, nqb_placement* pbuf, uint64_t capacity,
                     uint64_t* count, uint64_t* weighted, uint64_t* per_first_col);
int generate_pool(unsigned n, unsigned depth, nqb_state* buf, uint64_t capacity, uint64_t* count,
                  uint64_t* weighted);

// The same pool built on the device (pool_gpu.cu), stream-ordered buffer in *d_out.
int generate_pool_device(unsigned n, unsigned depth, cudaStream_t s, nqb_state** d_out, uint64_t* count);

// Worker threads used by host-side passes (NQB_THREADS overrides the core count).
unsigned host_threads();

// Largest number of free columns minus one over `count` states: the deepest stack of
// pending alternatives one search can hold.
unsigned max_stack_depth(const nqb_state* states, uint64_t count);

// Plain search kernel (plain.cu).  d_out: {weighted count, nodes, unit nodes, error flags}.
// d_per_state (optional): weight x completions per state.  d_lane_stats (optional): the
// instrumented kernel adds {lane-steps that placed a queen, lane-step slots} into it.
int launch_plain(const nqb_state* d_states, uint64_t count, unsigned long long* d_out,
                 unsigned long long* d_per_state, int block_size, bool count_unit, unsigned stack_depth,
                 cudaStream_t stream, unsigned* launches, unsigned long long* d_lane_stats = nullptr);

// Scratch of one batched launch (zeroed before it): 64 bytes of control words (word 0 is
// the item queue head), then the steal ring, 32 bytes a slot.  Scratch of 4 bytes (the
// head alone) launches without stealing across warps.
constexpr size_t kBatchedCtlBytes = 64;
constexpr size_t kBatchedSlotBytes = 32;
constexpr uint32_t kBatchedRingSlots = 1u << 16;  // the library's own launches: 2 MB
constexpr size_t kBatchedScratchBytes = kBatchedCtlBytes + kBatchedRingSlots * kBatchedSlotBytes;
constexpr uint32_t kBatchedWaitLimit = 1u << 18;  // polls without progress (about 2 s of backoff)
// Ring slots a scratch buffer of `scratch_bytes` holds (a power of two; 0 = no ring).
uint32_t batched_ring_slots(size_t scratch_bytes);

// Batched (persistent, work-queue) search kernel (batched.cu).  d_scratch as above.
// d_order (optional): queue position -> item; d_board_of (optional): item -> output slot.
// d_out: {weighted count, nodes, 0, error flags}.  d_lane_stats as for launch_plain.
// wait_limit: polls without progress before a wait of the work stealing gives up (0 =
// kBatchedWaitLimit).
int launch_batched(const nqb_state* d_items, uint32_t n_items, const uint32_t* d_order, const uint32_t* d_board_of,
                   void* d_scratch, size_t scratch_bytes, unsigned long long* d_out,
                   unsigned long long* d_per_board, unsigned long long* d_per_board_nodes, int block_size,
                   unsigned stack_depth, int device, cudaStream_t stream, unsigned* launches,
                   unsigned long long* d_lane_stats = nullptr, uint32_t wait_limit = 0);

// Items after learned scheduling: the caller's arrays, or split / ordered device copies
// owned by the schedule until release() (stream-ordered frees).
struct Schedule {
    const uint4* items = nullptr;
    const uint32_t* board = nullptr;  // item -> output slot (nullptr: identity)
    const uint32_t* order = nullptr;  // queue order (nullptr: as stored)
    uint32_t n = 0;
    double sched_ms = 0.0;
    uint4* owned_items = nullptr;
    uint32_t* owned_board = nullptr;
    uint32_t* owned_order = nullptr;
    cudaStream_t stream = nullptr;
    void release();
};
// Predicts, splits and orders `n` device items with o.model (no-op without a model or
// for queues longer than 64 items per resident lane).  Split placements are added into
// *d_split_nodes (and d_per_board_nodes[board]).
int schedule_items(const nqb_state* d_items, uint32_t n, const uint32_t* d_board, const nqb_opts& o, int device,
                   cudaStream_t s, unsigned long long* d_split_nodes, unsigned long long* d_per_board_nodes,
                   Schedule* out);

// Batched form with optional learned scheduling (schedule.cu): with o.model, items are
// split and ordered by predicted cost before the launch; otherwise launched as given.
struct SchedInfo {
    uint64_t items = 0;     // items given to the search kernel
    double sched_ms = 0.0;  // prediction + splitting + ordering (device time)
};
int launch_batched_scheduled(const nqb_state* d_items, uint32_t n, const uint32_t* d_board, void* d_scratch,
                             size_t scratch_bytes, unsigned long long* d_out, unsigned long long* d_per_board,
                             unsigned long long* d_per_board_nodes, const nqb_opts& o, unsigned stack_depth,
                             int device, cudaStream_t s, unsigned* launches, SchedInfo* info,
                             unsigned long long* d_lane_stats = nullptr);

// Stream-ordered device allocation from the library's pool on the current device
// (devmem.cu); release with dev_free on a stream.  Freed memory stays cached for later
// calls until nqb_trim_device_memory.
int dev_alloc_bytes(void** p, size_t bytes, cudaStream_t s);
template <class T>
int dev_alloc(T** p, size_t bytes, cudaStream_t s) {
    void* v = nullptr;
    const int st = dev_alloc_bytes(&v, bytes, s);
    *p = static_cast<T*>(v);
    return st;
}
void dev_free(void* p, cudaStream_t s);

int cuda_status(cudaError_t e);

// The allocation-failure test hook (nqb_debug_fail_allocation, devmem.cu): true when the
// allocation being made now is the one chosen to fail.  Every allocation of the library's own
// code asks it first: device buffers (dev_alloc_bytes, cuda_malloc), pinned host buffers
// (cuda_malloc_host) and host buffers (the pool and state-file arrays).
bool alloc_fault();

// cudaMalloc and cudaMallocHost behind the test hook; *p is nullptr unless NQB_OK.
template <class T>
int cuda_malloc(T** p, size_t bytes) {
    *p = nullptr;
    if (alloc_fault()) return NQB_E_NOMEM;
    void* v = nullptr;
    const int s = cuda_status(cudaMalloc(&v, bytes ? bytes : 16));
    if (s == NQB_OK) *p = static_cast<T*>(v);
    return s;
}
template <class T>
int cuda_malloc_host(T** p, size_t bytes) {
    *p = nullptr;
    if (alloc_fault()) return NQB_E_NOMEM;
    void* v = nullptr;
    const int s = cuda_status(cudaMallocHost(&v, bytes ? bytes : 16));
    if (s == NQB_OK) *p = static_cast<T*>(v);
    return s;
}

// Unique id of the calling thread's current CUDA context, 0 when none (devmem.cu).
unsigned long long current_context_id();

// Learned cost model (mlp.cu): predicted log2(1 + nodes) of `count` device states.
int model_predict_device(const nqb_model* m, const nqb_state* d_states, uint32_t count, float* d_out, cudaStream_t s,
                         uint32_t wait_limit = 0);
int model_device(const nqb_model* m);

}  // namespace nqb
