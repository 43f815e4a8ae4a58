// Batch plans: a batch of uneven partial boards solved repeatedly through one captured CUDA
// graph, with the launch configuration chosen by timing (the autotuner).
//
// Creation uploads the boards once.  With autotuning every (block size, split factor)
// candidate is first timed with CUDA events on a stride sample of the boards (at most about
// 4,096 of them, each with the sample's own learned schedule), which costs a fraction of one
// solve of the batch.  The learned schedule (split + order, schedule.cu) of the batch is then
// built for the winning split factor, and the whole solve (zero the per-board counts and the
// launch scratch, one batched-kernel launch, read the results back into pinned host memory)
// is captured into a CUDA graph.  A run is then a single cudaGraphLaunch.
#include <algorithm>
#include <cstring>
#include <vector>

#include "nqb_internal.h"

struct nqb_batch_plan {
    int device = 0;
    int prev_device = 0;
    cudaStream_t s = nullptr;
    uint64_t count = 0;
    unsigned stack_depth = 0;
    nqb_state* d_boards = nullptr;
    unsigned long long* d_per = nullptr;  // per-board weighted counts
    unsigned long long* d_out = nullptr;  // {count, nodes, unit, error flags}, 4 spare words, batched scratch
    unsigned long long* d_split = nullptr;
    unsigned long long* h_per = nullptr;  // pinned
    unsigned long long* h_out = nullptr;  // pinned
    nqb::Schedule sch;
    uint64_t split_nodes = 0;
    cudaGraphExec_t exec = nullptr;
    int block = 128;
    int factor = 0;
    double sched_ms = 0.0;
};

namespace {

using nqb::cuda_status;

// Zero the outputs and the launch scratch, launch, read back: the sequence a run replays.
int solve_sequence(nqb_batch_plan* p, int block) {
    cudaStream_t s = p->s;
    int st = cuda_status(cudaMemsetAsync(p->d_per, 0, p->count * sizeof(unsigned long long), s));
    if (!st)
        st = cuda_status(
            cudaMemsetAsync(p->d_out, 0, 8 * sizeof(unsigned long long) + nqb::kBatchedScratchBytes, s));
    if (!st)
        st = nqb::launch_batched(reinterpret_cast<const nqb_state*>(p->sch.items), p->sch.n, p->sch.order,
                                 p->sch.board, p->d_out + 8, nqb::kBatchedScratchBytes, p->d_out, p->d_per, nullptr,
                                 block, p->stack_depth, p->device, s,
                                 nullptr);
    if (!st)
        st = cuda_status(
            cudaMemcpyAsync(p->h_per, p->d_per, p->count * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    if (!st)
        st = cuda_status(
            cudaMemcpyAsync(p->h_out, p->d_out, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    return st;
}

int capture(nqb_batch_plan* p, int block, cudaGraphExec_t* exec) {
    // one uncaptured pass first: sets the kernel's attributes and checks the launch
    int st = solve_sequence(p, block);
    if (!st) st = cuda_status(cudaStreamSynchronize(p->s));
    if (st) return st;
    cudaGraph_t g = nullptr;
    if ((st = cuda_status(cudaStreamBeginCapture(p->s, cudaStreamCaptureModeRelaxed)))) return st;
    const int st_body = solve_sequence(p, block);
    st = cuda_status(cudaStreamEndCapture(p->s, &g));
    if (st_body) st = st_body;
    if (!st) st = cuda_status(cudaGraphInstantiate(exec, g, 0));
    if (g) cudaGraphDestroy(g);
    return st;
}

int time_graph(nqb_batch_plan* p, cudaGraphExec_t exec, float* ms) {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, p->s);
    int st = cuda_status(cudaGraphLaunch(exec, p->s));
    cudaEventRecord(b, p->s);
    if (!st) st = cuda_status(cudaEventSynchronize(b));
    if (!st) cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return st;
}

int build_schedule(nqb_batch_plan* p, const nqb_opts& o, int factor) {
    p->sch.release();
    p->sch = nqb::Schedule();
    nqb_opts oo = o;
    oo.split_factor = factor;
    cudaMemsetAsync(p->d_split, 0, sizeof(unsigned long long), p->s);
    int st = nqb::schedule_items(p->d_boards, (uint32_t)p->count, nullptr, oo, p->device, p->s, p->d_split, nullptr,
                                 &p->sch);
    unsigned long long split = 0;
    if (!st) st = cuda_status(cudaMemcpyAsync(&split, p->d_split, sizeof(split), cudaMemcpyDeviceToHost, p->s));
    if (!st) st = cuda_status(cudaStreamSynchronize(p->s));
    p->split_nodes = split;
    p->factor = factor;
    p->sched_ms = p->sch.sched_ms;
    return st;
}

__global__ void stride_gather(const uint4* __restrict__ in, uint64_t count, uint64_t stride, uint4* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = in[i * stride];
}

// Boards in the tuning sample: every board of small batches, every k-th of large ones.
constexpr uint64_t kTuneSample = 4096;

// Times every (block, split factor) candidate once on a stride sample of the boards: the
// sample's own schedule and one launch each, timed with CUDA events.  Each board stands for
// its subtree, so the sample keeps the batch's spread of sizes at 1/stride of its work.
int tune_on_sample(nqb_batch_plan* p, const nqb_opts& o, const std::vector<int>& blocks,
                   const std::vector<int>& factors, int* best_block, int* best_factor) {
    const uint64_t stride = std::max<uint64_t>(1, p->count / kTuneSample);
    const uint64_t n = (p->count + stride - 1) / stride;
    nqb_state* d_sample = nullptr;
    unsigned long long* d_split = nullptr;
    int st = nqb::dev_alloc(&d_sample, n * sizeof(nqb_state), p->s);
    if (!st) st = nqb::dev_alloc(&d_split, sizeof(unsigned long long), p->s);
    if (!st) {
        stride_gather<<<(unsigned)((n + 255) / 256), 256, 0, p->s>>>(reinterpret_cast<const uint4*>(p->d_boards), n,
                                                                      stride, reinterpret_cast<uint4*>(d_sample));
        st = cuda_status(cudaGetLastError());
    }
    cudaEvent_t a = nullptr, b = nullptr;
    if (!st) st = cuda_status(cudaEventCreate(&a));
    if (!st) st = cuda_status(cudaEventCreate(&b));
    float best = -1.0f;
    for (size_t fi = 0; fi < factors.size() && !st; ++fi) {
        nqb_opts oo = o;
        oo.split_factor = factors[fi];
        nqb::Schedule sch;
        st = nqb::schedule_items(d_sample, (uint32_t)n, nullptr, oo, p->device, p->s, d_split, nullptr, &sch);
        for (size_t bi = 0; bi < blocks.size() && !st; ++bi) {
            st = cuda_status(
                cudaMemsetAsync(p->d_out, 0, 8 * sizeof(unsigned long long) + nqb::kBatchedScratchBytes, p->s));
            if (!st) st = cuda_status(cudaEventRecord(a, p->s));
            if (!st)
                st = nqb::launch_batched(reinterpret_cast<const nqb_state*>(sch.items), sch.n, sch.order, sch.board,
                                         p->d_out + 8, nqb::kBatchedScratchBytes, p->d_out, nullptr, nullptr,
                                         blocks[bi], p->stack_depth, p->device, p->s, nullptr);
            if (!st) st = cuda_status(cudaEventRecord(b, p->s));
            if (!st) st = cuda_status(cudaEventSynchronize(b));
            float ms = 0.0f;
            if (!st) st = cuda_status(cudaEventElapsedTime(&ms, a, b));
            if (!st && (best < 0.0f || ms < best)) {
                best = ms;
                *best_block = blocks[bi];
                *best_factor = factors[fi];
            }
        }
        sch.release();
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    nqb::dev_free(d_sample, p->s);
    nqb::dev_free(d_split, p->s);
    if (!st) st = cuda_status(cudaStreamSynchronize(p->s));
    return st;
}

}  // namespace

extern "C" {

void nqb_batch_plan_destroy(nqb_batch_plan* p) {
    if (!p) return;
    cudaSetDevice(p->device);
    if (p->s) cudaStreamSynchronize(p->s);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    p->sch.release();
    if (p->s) cudaStreamSynchronize(p->s);
    cudaFree(p->d_boards);
    cudaFree(p->d_per);
    cudaFree(p->d_out);
    cudaFree(p->d_split);
    cudaFreeHost(p->h_per);
    cudaFreeHost(p->h_out);
    if (p->s) cudaStreamDestroy(p->s);
    cudaSetDevice(p->prev_device);
    delete p;
}

int nqb_batch_plan_create(const nqb_state* boards, uint64_t count, const nqb_opts* opts, int autotune,
                          nqb_batch_plan** out) try {
    if (!out || !boards || count == 0) return NQB_E_INVALID;
    *out = nullptr;
    if (count > (1ull << 31)) return NQB_E_RANGE;
    nqb_opts o;
    nqb_default_opts(&o);
    if (opts) o = *opts;
    for (uint64_t i = 0; i < count; ++i)
        if (!nqb::state_valid(boards[i])) return NQB_E_INVALID;
    std::vector<int> blocks, factors;  // built before anything that needs releasing
    if (autotune) {
        blocks = {64, 128, 256};
        factors = (o.model || o.sched_cost) ? std::vector<int>{1, 4, 16} : std::vector<int>{o.split_factor};
    } else {
        blocks = {o.block_size ? o.block_size : 128};
        factors = {o.split_factor};
    }
    int st = nqb_device_check(o.device);
    if (st) return st;
    nqb_batch_plan* p = new nqb_batch_plan();
    cudaGetDevice(&p->prev_device);
    p->device = o.device;
    p->count = count;
    p->stack_depth = nqb::max_stack_depth(boards, count);
    auto fail = [&](int code) {
        nqb_batch_plan_destroy(p);
        return code;
    };
    if ((st = cuda_status(cudaSetDevice(p->device)))) return fail(st);
    if ((st = cuda_status(cudaStreamCreateWithFlags(&p->s, cudaStreamNonBlocking)))) return fail(st);
    if ((st = nqb::cuda_malloc(&p->d_boards, count * sizeof(nqb_state)))) return fail(st);
    if ((st = nqb::cuda_malloc(&p->d_per, count * sizeof(unsigned long long)))) return fail(st);
    if ((st = nqb::cuda_malloc(&p->d_out, 8 * sizeof(unsigned long long) + nqb::kBatchedScratchBytes)))
        return fail(st);
    if ((st = nqb::cuda_malloc(&p->d_split, sizeof(unsigned long long)))) return fail(st);
    if ((st = nqb::cuda_malloc_host(&p->h_per, count * sizeof(unsigned long long)))) return fail(st);
    if ((st = nqb::cuda_malloc_host(&p->h_out, 4 * sizeof(unsigned long long)))) return fail(st);
    if ((st = cuda_status(cudaMemcpyAsync(p->d_boards, boards, count * sizeof(nqb_state), cudaMemcpyHostToDevice,
                                          p->s))))
        return fail(st);

    int best_block = blocks[0], best_factor = factors[0];
    if (blocks.size() * factors.size() > 1 &&
        (st = tune_on_sample(p, o, blocks, factors, &best_block, &best_factor)))
        return fail(st);
    if ((st = build_schedule(p, o, best_factor))) return fail(st);
    if ((st = capture(p, best_block, &p->exec))) return fail(st);
    p->block = best_block;
    *out = p;
    cudaSetDevice(p->prev_device);
    return NQB_OK;
} NQB_ABI_CATCH

int nqb_batch_plan_run(nqb_batch_plan* p, uint64_t* out, nqb_stats* stats) {
    if (!p || !out) return NQB_E_INVALID;
    int prev = 0;
    cudaGetDevice(&prev);
    int st = cuda_status(cudaSetDevice(p->device));
    float ms = 0.0f;
    if (!st) st = time_graph(p, p->exec, &ms);
    if (!st) {
        std::memcpy(out, p->h_per, p->count * sizeof(uint64_t));
        if (p->h_out[3]) st = (p->h_out[3] & 4) ? NQB_E_STALL : NQB_E_DEVICE;
    }
    if (!st && stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->states = p->count;
        stats->nodes = p->h_out[1] + p->split_nodes;
        stats->unit_nodes = UINT64_MAX;
        stats->kernel_ms = ms;
        stats->wall_ms = ms;
        stats->kernel_launches = 1;
        stats->items = p->sch.n;
        stats->sched_ms = p->sched_ms;
    }
    cudaSetDevice(prev);
    return st;
}

int nqb_batch_plan_config(const nqb_batch_plan* p, int* block_size, int* split_factor, uint64_t* items) {
    if (!p) return NQB_E_INVALID;
    if (block_size) *block_size = p->block;
    if (split_factor) *split_factor = p->factor;
    if (items) *items = p->sch.n;
    return NQB_OK;
}

}  // extern "C"
