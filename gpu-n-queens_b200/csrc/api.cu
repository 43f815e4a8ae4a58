// C ABI of libnqb.so (include/nqb.h): argument checks, device buffers, streams and timing
// around the pool generator and the search kernels.  Replaces the reference's solve()
// (NQ_solver.cu:192-209) and gpu_solver_driver (GPU_NQueens.cu:56-175); unlike those it
// never exits the process and frees everything it allocated on every path.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "nqb_internal.h"

namespace nqb {

bool state_valid(const nqb_state& s) {
    if (s.n < 1 || s.n > NQB_MAX_N || s.flags != 0) return false;
    return (s.cols & ~board_mask(s.n)) == 0;
}

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return NQB_OK;
    if (e == cudaErrorMemoryAllocation) return NQB_E_NOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice || e == cudaErrorInsufficientDriver)
        return NQB_E_NODEVICE;
    return NQB_E_CUDA;
}

namespace {

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Device-call scope: selects the device, owns a stream, timing events and buffers,
// and restores the caller's device on exit.
class Scope {
   public:
    int status = NQB_OK;
    int device = 0;
    cudaStream_t stream = nullptr;

    explicit Scope(int dev) : device(dev) {
        cudaGetDevice(&prev_);
        status = nqb_device_check(dev);
        if (status != NQB_OK) return;
        if ((status = cuda_status(cudaSetDevice(dev))) != NQB_OK) return;
        status = cuda_status(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    }
    ~Scope() {
        for (void* p : bufs_) dev_free(p, stream);
        if (stream) cudaStreamSynchronize(stream);
        for (cudaEvent_t e : events_) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
        cudaSetDevice(prev_);
    }
    // The slot is added before the buffer or event is made: a push_back that throws then
    // leaves nothing behind.
    template <class T>
    int alloc(T** p, size_t bytes) {
        bufs_.push_back(nullptr);
        const int s = dev_alloc_bytes(&bufs_.back(), bytes, stream);
        if (s != NQB_OK) {
            bufs_.pop_back();
            return s;
        }
        *p = static_cast<T*>(bufs_.back());
        return NQB_OK;
    }
    int event(cudaEvent_t* e) {
        events_.push_back(nullptr);
        const int s = cuda_status(cudaEventCreate(&events_.back()));
        if (s != NQB_OK) {
            events_.pop_back();
            return s;
        }
        *e = events_.back();
        return s;
    }
    Scope(const Scope&) = delete;
    Scope& operator=(const Scope&) = delete;

   private:
    int prev_ = 0;
    std::vector<void*> bufs_;
    std::vector<cudaEvent_t> events_;
};

nqb_opts resolve(const nqb_opts* o) {
    nqb_opts r;
    nqb_default_opts(&r);
    if (o) r = *o;
    return r;
}


// Solves `count` states already on the device (d_states, stack bound `depth`) with the form
// o.form; fills totals {count, nodes, unit, err} and optional per-state results.  e_start is
// recorded before any H2D copy so that h2d_ms covers it.
int solve_device_states(Scope& sc, const nqb_state* d_states, uint64_t count, unsigned depth, const nqb_opts& o,
                        unsigned long long totals[4], uint64_t* per_state, nqb_stats* st,
                        uint64_t* per_state_nodes, cudaEvent_t e_start) {
    const bool batched = o.form == NQB_FORM_BATCHED;
    if (o.form != NQB_FORM_PLAIN && !batched) return NQB_E_INVALID;
    if (batched && count > (1ull << 31)) return NQB_E_RANGE;
    // 4 result words, 2 lane-step counters, 2 spare, then the batched launch's scratch
    unsigned long long* d_out = nullptr;
    unsigned long long* d_per = nullptr;
    const size_t out_bytes = 8 * sizeof(unsigned long long) + (batched ? kBatchedScratchBytes : 0);
    NQB_TRY(sc.alloc(&d_out, out_bytes));
    if (per_state) NQB_TRY(sc.alloc(&d_per, count * sizeof(unsigned long long)));
    unsigned long long* d_per_nodes = nullptr;
    if (per_state_nodes) {
        if (!batched) return NQB_E_INVALID;
        NQB_TRY(sc.alloc(&d_per_nodes, count * sizeof(unsigned long long)));
        NQB_TRY(cuda_status(cudaMemsetAsync(d_per_nodes, 0, count * sizeof(unsigned long long), sc.stream)));
    }
    unsigned long long* d_lanes = o.count_lane_steps ? d_out + 4 : nullptr;
    cudaEvent_t e1, e2;
    NQB_TRY(sc.event(&e1));
    NQB_TRY(sc.event(&e2));
    NQB_TRY(cuda_status(cudaMemsetAsync(d_out, 0, out_bytes, sc.stream)));
    if (d_per) NQB_TRY(cuda_status(cudaMemsetAsync(d_per, 0, count * sizeof(unsigned long long), sc.stream)));
    NQB_TRY(cuda_status(cudaEventRecord(e1, sc.stream)));
    unsigned launches = 0;
    SchedInfo sched;
    sched.items = count;
    if (count) {
        if (batched) {
            NQB_TRY(launch_batched_scheduled(d_states, (uint32_t)count, nullptr, d_out + 8, kBatchedScratchBytes, d_out,
                                             d_per, d_per_nodes, o, depth, sc.device, sc.stream, &launches, &sched,
                                             d_lanes));
        } else {
            NQB_TRY(launch_plain(d_states, count, d_out, d_per, o.block_size, o.count_unit_nodes != 0, depth,
                                 sc.stream, &launches, d_lanes));
        }
    }
    NQB_TRY(cuda_status(cudaEventRecord(e2, sc.stream)));
    unsigned long long lanes[2] = {0, 0};
    NQB_TRY(cuda_status(cudaMemcpyAsync(totals, d_out, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                        sc.stream)));
    if (d_lanes)
        NQB_TRY(cuda_status(cudaMemcpyAsync(lanes, d_lanes, sizeof(lanes), cudaMemcpyDeviceToHost, sc.stream)));
    if (per_state)
        NQB_TRY(cuda_status(cudaMemcpyAsync(per_state, d_per, count * sizeof(unsigned long long),
                                            cudaMemcpyDeviceToHost, sc.stream)));
    if (per_state_nodes)
        NQB_TRY(cuda_status(cudaMemcpyAsync(per_state_nodes, d_per_nodes, count * sizeof(unsigned long long),
                                            cudaMemcpyDeviceToHost, sc.stream)));
    NQB_TRY(cuda_status(cudaStreamSynchronize(sc.stream)));
    if (totals[3] & 4) return NQB_E_STALL;
    if (totals[3]) return NQB_E_DEVICE;
    if (st) {
        float h2d = 0, ker = 0;
        if (e_start) cudaEventElapsedTime(&h2d, e_start, e1);
        cudaEventElapsedTime(&ker, e1, e2);
        st->states = count;
        st->nodes = totals[1];
        st->unit_nodes = (o.count_unit_nodes && !batched) ? totals[2] : UINT64_MAX;
        st->h2d_ms = h2d;
        st->kernel_ms = ker;
        st->kernel_launches = launches;
        st->items = sched.items;
        st->sched_ms = sched.sched_ms;
        st->block_size = (uint32_t)(o.block_size ? o.block_size : 128);
        st->form = o.form;
        st->placed_lane_steps = lanes[0];
        st->lane_step_slots = lanes[1];
    }
    return NQB_OK;
}

// Solves `count` host states on the device with the form o.form; fills totals
// {count, nodes, unit, err} and, if per_state != nullptr, per-state weighted counts.
// `known_depth` != 0: the states come from the library's own generator, so the
// per-state validation and the stack-depth scan are skipped.
int solve_host_states(Scope& sc, const nqb_state* states, uint64_t count, const nqb_opts& o,
                      unsigned long long totals[4], uint64_t* per_state, nqb_stats* st,
                      uint64_t* per_state_nodes = nullptr, unsigned known_depth = 0) {
    if (!known_depth)
        for (uint64_t i = 0; i < count; ++i)
            if (!state_valid(states[i])) return NQB_E_INVALID;
    const unsigned depth = known_depth ? known_depth : max_stack_depth(states, count);
    nqb_state* d_states = nullptr;
    NQB_TRY(sc.alloc(&d_states, count * sizeof(nqb_state)));
    cudaEvent_t e0;
    NQB_TRY(sc.event(&e0));
    NQB_TRY(cuda_status(cudaEventRecord(e0, sc.stream)));
    NQB_TRY(cuda_status(
        cudaMemcpyAsync(d_states, states, count * sizeof(nqb_state), cudaMemcpyHostToDevice, sc.stream)));
    return solve_device_states(sc, d_states, count, depth, o, totals, per_state, st, per_state_nodes, e0);
}

void* aligned_host_alloc(size_t bytes) {
    void* p = nullptr;
    if (alloc_fault()) return nullptr;
    if (posix_memalign(&p, 64, bytes ? bytes : 64)) return nullptr;
    return p;
}

}  // namespace
}  // namespace nqb

using namespace nqb;

extern "C" {

void nqb_default_opts(nqb_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->device = 0;
    o->form = NQB_FORM_PLAIN;
    o->block_size = 0;
    o->max_split_rounds = -1;
    o->split_factor = 0;
    o->model = nullptr;
}

const char* nqb_strerror(int s) {
    switch (s) {
        case NQB_OK: return "ok";
        case NQB_E_INVALID: return "invalid argument";
        case NQB_E_NOMEM: return "out of memory";
        case NQB_E_CUDA: return "CUDA runtime error";
        case NQB_E_NODEVICE: return "no usable sm_100 CUDA device";
        case NQB_E_RANGE: return "size beyond a supported limit";
        case NQB_E_STALL: return "device-side bounded wait ran out";
        case NQB_E_DEVICE: return "device-side check failed";
        case NQB_E_MODEL: return "learned cost model missing or not trained";
        case NQB_E_IO: return "file could not be opened, read or written";
        case NQB_E_FORMAT: return "malformed state file, or another version or generation flags";
        default: return "unknown status";
    }
}

int nqb_version(void) { return NQB_VERSION; }

int nqb_device_count(int* count) {
    if (!count) return NQB_E_INVALID;
    *count = 0;
    const int s = cuda_status(cudaGetDeviceCount(count));
    if (s) *count = 0;
    return s ? s : (*count > 0 ? NQB_OK : NQB_E_NODEVICE);
}

int nqb_device_check(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return NQB_E_NODEVICE;
    }
    if (device < 0 || device >= n) return NQB_E_NODEVICE;
    int major = 0, warp = 0, mode = 0;  // single attributes: cheaper than the whole cudaDeviceProp
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&warp, cudaDevAttrWarpSize, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&mode, cudaDevAttrComputeMode, device) != cudaSuccess)
        return NQB_E_NODEVICE;
    if (major != 10 || warp != 32 || mode == cudaComputeModeProhibited) return NQB_E_NODEVICE;
    return NQB_OK;
}

void nqb_free(void* p) { std::free(p); }

int nqb_generate_pool_into(unsigned n, unsigned depth, nqb_state* buf, uint64_t capacity, uint64_t* count) try {
    if (!count) return NQB_E_INVALID;
    return generate_pool(n, depth, buf, buf ? capacity : 0, count, nullptr);
} NQB_ABI_CATCH

int nqb_pool_weighted_size(unsigned n, unsigned depth, uint64_t* weighted) try {
    if (!weighted) return NQB_E_INVALID;
    uint64_t c = 0;
    return generate_pool(n, depth, nullptr, 0, &c, weighted);
} NQB_ABI_CATCH

int nqb_generate_pool(unsigned n, unsigned depth, nqb_state** states, uint64_t* count) try {
    if (!states || !count) return NQB_E_INVALID;
    *states = nullptr;
    uint64_t c = 0;
    NQB_TRY(generate_pool(n, depth, nullptr, 0, &c, nullptr));
    std::unique_ptr<nqb_state, void (*)(void*)> p(static_cast<nqb_state*>(aligned_host_alloc(c * sizeof(nqb_state))),
                                                  std::free);
    if (!p) return NQB_E_NOMEM;
    NQB_TRY(generate_pool(n, depth, p.get(), c, count, nullptr));
    *states = p.release();
    return NQB_OK;
} NQB_ABI_CATCH

int nqb_count_ex(unsigned n, unsigned depth, const nqb_opts* opts, uint64_t* count, nqb_stats* stats) try {
    const double t0 = now_ms();
    if (!count || n < NQB_MIN_N || n > NQB_MAX_N || depth < 1 || depth >= n) return NQB_E_INVALID;
    nqb_opts o = resolve(opts);
    if (o.autotune) {  // pick the launch on a sample of this pool first
        nqb_tune_result t;
        NQB_TRY(nqb_tune_count(n, &depth, 1, &o, 64, &t));
        o.form = t.form;
        o.block_size = t.block_size;
        o.split_factor = t.split_factor;
    }
    if (stats) std::memset(stats, 0, sizeof(*stats));
    Scope sc(o.device);
    NQB_TRY(sc.status);
    unsigned long long totals[4] = {0, 0, 0, 0};
    double gen_ms = 0.0;
    if (o.host_pool) {  // the reference's way: build the pool on the host, copy it over
        nqb_state* pool = nullptr;
        uint64_t cnt = 0;
        const double tg = now_ms();
        NQB_TRY(nqb_generate_pool(n, depth, &pool, &cnt));
        std::unique_ptr<nqb_state, void (*)(void*)> own(pool, std::free);
        gen_ms = now_ms() - tg;
        NQB_TRY(solve_host_states(sc, pool, cnt, o, totals, nullptr, stats, nullptr,
                                  n - depth - 1 > 0 ? n - depth - 1 : 1));
    } else {  // build the pool on the GPU: nothing crosses PCIe but the result
        cudaEvent_t g0, g1;
        NQB_TRY(sc.event(&g0));
        NQB_TRY(sc.event(&g1));
        NQB_TRY(cuda_status(cudaEventRecord(g0, sc.stream)));
        nqb_state* d_pool = nullptr;
        uint64_t cnt = 0;
        NQB_TRY(generate_pool_device(n, depth, sc.stream, &d_pool, &cnt));
        cudaEventRecord(g1, sc.stream);
        const int s = solve_device_states(sc, d_pool, cnt, n - depth - 1 > 0 ? n - depth - 1 : 1, o, totals, nullptr,
                                          stats, nullptr, nullptr);
        dev_free(d_pool, sc.stream);
        NQB_TRY(s);
        float g = 0.0f;
        cudaEventElapsedTime(&g, g0, g1);
        gen_ms = g;
    }
    *count = totals[0];
    if (stats) {
        stats->gen_ms = gen_ms;
        stats->pregen_depth = depth;
        stats->wall_ms = now_ms() - t0;
    }
    return NQB_OK;
} NQB_ABI_CATCH

int nqb_count(unsigned n, unsigned depth, uint64_t* count) { return nqb_count_ex(n, depth, nullptr, count, nullptr); }

int nqb_solve_states(const nqb_state* states, uint64_t count, const nqb_opts* opts, uint64_t* total,
                     nqb_stats* stats) try {
    const double t0 = now_ms();
    if (!total || (count && !states)) return NQB_E_INVALID;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    *total = 0;
    if (count == 0) return NQB_OK;
    const nqb_opts o = resolve(opts);
    Scope sc(o.device);
    NQB_TRY(sc.status);
    unsigned long long totals[4] = {0, 0, 0, 0};
    NQB_TRY(solve_host_states(sc, states, count, o, totals, nullptr, stats));
    *total = totals[0];
    if (stats) stats->wall_ms = now_ms() - t0;
    return NQB_OK;
} NQB_ABI_CATCH

int nqb_solve_states_multi(const nqb_state* states, uint64_t count, const int* devices, unsigned ndev,
                           const nqb_opts* opts, uint64_t* total, nqb_stats* stats) try {
    const double t0 = now_ms();
    if (!total || (count && !states) || !devices || ndev == 0) return NQB_E_INVALID;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    *total = 0;
    const nqb_opts base = resolve(opts);
    std::vector<uint64_t> part(ndev, 0);
    std::vector<nqb_stats> pst(ndev);
    std::vector<int> status(ndev, NQB_OK);
    std::vector<std::thread> workers;
    const uint64_t per = count / ndev;  // contiguous slices, the last one takes the remainder
    auto work = [&](unsigned k) {
        const uint64_t first = per * k, len = per + (k == ndev - 1 ? count % ndev : 0);
        nqb_opts o = base;
        o.device = devices[k];
        status[k] = nqb_solve_states(states + first, len, &o, &part[k], &pst[k]);
    };
    for (unsigned k = 0; k < ndev; ++k) {
        try {  // no exception may cross the C ABI: without a thread, solve the slice here
            workers.emplace_back(work, k);
        } catch (...) {
            work(k);
        }
    }
    for (auto& w : workers) w.join();
    for (unsigned k = 0; k < ndev; ++k) NQB_TRY(status[k]);
    for (unsigned k = 0; k < ndev; ++k) {
        *total += part[k];
        if (!stats) continue;
        stats->states += pst[k].states;
        stats->nodes += pst[k].nodes;
        stats->h2d_ms = std::max(stats->h2d_ms, pst[k].h2d_ms);
        stats->kernel_ms = std::max(stats->kernel_ms, pst[k].kernel_ms);
        stats->kernel_launches += pst[k].kernel_launches;
        stats->items += pst[k].items;
    }
    if (stats) {
        stats->unit_nodes = UINT64_MAX;
        stats->wall_ms = now_ms() - t0;
    }
    return NQB_OK;
} NQB_ABI_CATCH

int nqb_solve_batch(const nqb_state* boards, uint64_t count, const nqb_opts* opts, uint64_t* out,
                    nqb_stats* stats) try {
    const double t0 = now_ms();
    if (!out || (count && !boards)) return NQB_E_INVALID;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (count == 0) return NQB_OK;
    const nqb_opts o = resolve(opts);
    Scope sc(o.device);
    NQB_TRY(sc.status);
    unsigned long long totals[4] = {0, 0, 0, 0};
    NQB_TRY(solve_host_states(sc, boards, count, o, totals, out, stats));
    if (stats) stats->wall_ms = now_ms() - t0;
    return NQB_OK;
} NQB_ABI_CATCH

int nqb_record_nodes(const nqb_state* states, uint64_t count, const nqb_opts* opts, uint64_t* nodes,
                     uint64_t* counts) try {
    if (!nodes || !counts || (count && !states)) return NQB_E_INVALID;
    if (count == 0) return NQB_OK;
    nqb_opts o = resolve(opts);
    o.form = NQB_FORM_BATCHED;
    o.model = nullptr;
    Scope sc(o.device);
    NQB_TRY(sc.status);
    unsigned long long totals[4] = {0, 0, 0, 0};
    return solve_host_states(sc, states, count, o, totals, counts, nullptr, nodes);
} NQB_ABI_CATCH

size_t nqb_ref_state_size(unsigned n) {
    if (n < 1 || n > NQB_MAX_N) return 0;
    return ((16u + 4u + 1u + n) + 7u) & ~(size_t)7u;
}

int nqb_states_from_ref(unsigned n, const void* ref_states, uint64_t count, int mirror_weight, nqb_state* out) {
    if (n < NQB_MIN_N || n > NQB_MAX_N || (count && (!ref_states || !out))) return NQB_E_INVALID;
    const size_t sz = nqb_ref_state_size(n);
    const uint8_t* p = static_cast<const uint8_t*>(ref_states);
    const uint32_t mask = board_mask(n);
    for (uint64_t i = 0; i < count; ++i, p += sz) {
        uint64_t diag, anti;
        uint32_t cols;
        std::memcpy(&diag, p, 8);
        std::memcpy(&anti, p + 8, 8);
        std::memcpy(&cols, p + 16, 4);
        const int row = (int8_t)p[20];
        if (row < 0 || row > (int)n || (cols & ~mask)) return NQB_E_INVALID;
        nqb_state& s = out[i];
        s.cols = cols;
        s.rdiag = (uint32_t)(diag >> row);                 // diagonals.cuh:17-20
        s.ldiag = (uint32_t)(anti >> (n - (unsigned)row));
        s.row = (uint8_t)row;
        s.n = (uint8_t)n;
        s.weight = (uint8_t)(mirror_weight ? (p[21] < (n >> 1) ? 2 : 1) : 1);  // GPU_NQueens.cu:356
        s.flags = 0;
    }
    return NQB_OK;
}

int nqb_solve_ref_states(unsigned n, const void* ref_states, uint64_t count, unsigned locked_row,
                         const nqb_opts* opts, uint64_t* total) try {
    if (!total || n < NQB_MIN_N || n > NQB_MAX_N || locked_row < 1 || locked_row >= n) return NQB_E_INVALID;
    if (count && !ref_states) return NQB_E_INVALID;
    *total = 0;
    if (count == 0) return NQB_OK;
    nqb_state* st = static_cast<nqb_state*>(aligned_host_alloc(count * sizeof(nqb_state)));
    if (!st) return NQB_E_NOMEM;
    int s = nqb_states_from_ref(n, ref_states, count, 1, st);
    for (uint64_t i = 0; s == NQB_OK && i < count; ++i)
        if (st[i].row != locked_row) s = NQB_E_INVALID;  // the reference solves one lock row per call
    if (s == NQB_OK) s = nqb_solve_states(st, count, opts, total, nullptr);
    std::free(st);
    return s;
} NQB_ABI_CATCH

int nqb_plain_launch(const nqb_state* d_states, uint64_t count, uint64_t* d_out, int block_size,
                     int count_unit_nodes, unsigned stack_depth, void* stream) try {
    return launch_plain(d_states, count, reinterpret_cast<unsigned long long*>(d_out), nullptr, block_size,
                        count_unit_nodes != 0, stack_depth, static_cast<cudaStream_t>(stream), nullptr);
} NQB_ABI_CATCH

int nqb_batched_launch(const nqb_state* d_items, uint64_t count, const uint32_t* d_order, uint32_t* d_head,
                       uint64_t* d_out, int block_size, unsigned stack_depth, void* stream) try {
    if (count > (1ull << 31)) return NQB_E_RANGE;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NQB_E_NODEVICE;
    return launch_batched(d_items, (uint32_t)count, d_order, nullptr, d_head, sizeof(uint32_t),
                          reinterpret_cast<unsigned long long*>(d_out), nullptr, nullptr, block_size, stack_depth, dev,
                          static_cast<cudaStream_t>(stream), nullptr);
} NQB_ABI_CATCH

int nqb_batched_launch_ex(const nqb_state* d_items, uint64_t count, const uint32_t* d_order, void* d_scratch,
                          uint64_t scratch_bytes, uint64_t* d_out, uint64_t* d_lane_stats, int block_size,
                          unsigned stack_depth, unsigned wait_limit, void* stream) try {
    if (count > (1ull << 31)) return NQB_E_RANGE;
    if (!d_out || !d_scratch || scratch_bytes < sizeof(uint32_t) || (count && !d_items)) return NQB_E_INVALID;
    if (batched_ring_slots((size_t)scratch_bytes) && (reinterpret_cast<uintptr_t>(d_scratch) & 15) != 0)
        return NQB_E_INVALID;  // the ring's words need 16-byte alignment
    if (stack_depth > NQB_MAX_N) return NQB_E_INVALID;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NQB_E_NODEVICE;
    return launch_batched(d_items, (uint32_t)count, d_order, nullptr, d_scratch, (size_t)scratch_bytes,
                          reinterpret_cast<unsigned long long*>(d_out), nullptr, nullptr, block_size, stack_depth, dev,
                          static_cast<cudaStream_t>(stream), nullptr,
                          reinterpret_cast<unsigned long long*>(d_lane_stats), wait_limit);
} NQB_ABI_CATCH

int nqb_generate_pool_device(unsigned n, unsigned depth, nqb_state** d_states, uint64_t* count, void* stream) try {
    if (!d_states || !count) return NQB_E_INVALID;
    return generate_pool_device(n, depth, static_cast<cudaStream_t>(stream), d_states, count);
} NQB_ABI_CATCH

int nqb_generate_pool_device_into(unsigned n, unsigned depth, nqb_state* d_buf, uint64_t capacity, uint64_t* count,
                                  void* stream) try {
    if (!count || (capacity && !d_buf)) return NQB_E_INVALID;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    nqb_state* d_pool = nullptr;
    int s = generate_pool_device(n, depth, st, &d_pool, count);
    if (s) return s;
    if (*count > capacity) s = NQB_E_RANGE;
    else if (*count) s = cuda_status(cudaMemcpyAsync(d_buf, d_pool, *count * sizeof(nqb_state), cudaMemcpyDeviceToDevice, st));
    dev_free(d_pool, st);
    return s;
} NQB_ABI_CATCH

void nqb_free_device(void* p, void* stream) {
    dev_free(p, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
