// Learned scheduling of the batched form: the cost model orders the work queue and decides
// which items are split before the persistent search kernel runs.  The search arithmetic is
// untouched: an item is split into its children (one per candidate of its next row, in column
// order), the placements that create the children are counted as nodes here, and the
// children are searched like any other item, so counts and nodes are exactly those of the
// unsplit search.
//
// Pipeline on the device (all on the caller's stream):
//   1. predict log2(1 + nodes) of every item (fused MLP kernel, mlp.cu);
//   2. split round: threshold = predicted total / (resident lanes x split_factor); items
//      predicted above it (and with >= 2 candidates and >= 3 free columns) are replaced
//      by their children: mark -> exclusive scan (CUB) -> scatter; re-predict; repeat for up
//      to max_split_rounds rounds or until nothing is split;
//   3. order the queue by predicted cost, largest first (CUB radix sort of (cost, index));
//   4. one launch of the batched kernel with that order.
// Without a model the items go to the kernel unchanged, in their given order (FIFO), unless
// a model-free cost is asked for (nqb_opts.sched_cost: the ablation arms of the learned
// schedule), which then drives the same split-and-order steps in place of the prediction.
#include <algorithm>
#include <cmath>
#include <vector>

#include <cub/cub.cuh>

#include "nqb_internal.h"

namespace nqb {
namespace {

// Stream-ordered device buffer (from the library's device memory pool): no
// device-wide synchronisation on allocation or release, and pool memory is reused across
// calls.
template <class T>
struct Buf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    explicit Buf(cudaStream_t st) : s(st) {}
    int alloc(size_t count) {
        if (p) dev_free(p, s);
        p = nullptr;
        n = count;
        return dev_alloc(&p, count * sizeof(T), s);
    }
    T* take() {
        T* q = p;
        p = nullptr;
        return q;
    }
    ~Buf() {
        if (p) dev_free(p, s);
    }
};

__global__ void iota_kernel(uint32_t* v, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

__global__ void work_sum_kernel(const float* __restrict__ cost, uint32_t n, double* __restrict__ out) {
    double s = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        s += exp2((double)cost[i]);
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

__device__ __forceinline__ uint32_t item_avail(const uint4 s, uint32_t* nc_out) {
    const uint32_t n = (s.w >> 8) & 0xFFu;
    const uint32_t mask = n >= 32 ? 0xFFFFFFFFu : ((1u << n) - 1u);
    const uint32_t nc = mask & ~s.x;
    *nc_out = nc;
    return nc & ~(s.y | s.z);
}

// k[i] = number of items item i becomes: its candidates when split, else 1.
__global__ void mark_kernel(const uint4* __restrict__ items, const float* __restrict__ cost, uint32_t n,
                            const double* __restrict__ work, double lanes_x_factor, uint32_t* __restrict__ k) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float thr = (float)log2(fmax(work[0] / lanes_x_factor, 1.0));
    uint32_t nc;
    const uint32_t avail = item_avail(items[i], &nc);
    const uint32_t c = __popc(avail);
    k[i] = (cost[i] > thr && c >= 2 && __popc(nc) >= 3) ? c : 1u;
}

// Writes item i (or its children) at offset[i]; counts the split placements as nodes.
__global__ void split_kernel(const uint4* __restrict__ items, const uint32_t* __restrict__ board,
                             const uint32_t* __restrict__ k, const uint32_t* __restrict__ offset, uint32_t n,
                             uint4* __restrict__ out, uint32_t* __restrict__ out_board,
                             unsigned long long* __restrict__ nodes, unsigned long long* __restrict__ board_nodes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 s = items[i];
    const uint32_t b_id = board ? board[i] : i;
    uint32_t o = offset[i];
    if (k[i] == 1u) {
        out[o] = s;
        out_board[o] = b_id;
        return;
    }
    uint32_t nc;
    uint32_t avail = item_avail(s, &nc);
    const uint32_t placed = __popc(avail);
    const uint32_t meta = s.w + 1u;  // row + 1 (row is the low byte; n <= 31 keeps it in range)
    while (avail) {
        const uint32_t b = avail & (0u - avail);
        avail ^= b;
        out[o] = make_uint4(s.x | b, (s.y | b) << 1, (s.z | b) >> 1, meta);
        out_board[o] = b_id;
        ++o;
    }
    atomicAdd(nodes, (unsigned long long)placed);
    if (board_nodes) atomicAdd(board_nodes + b_id, (unsigned long long)placed);
}

// Model-free costs (log2 of an estimate of the nodes below each item), the ablation arms of
// the learned schedule: kind 1 = free columns x rows left; kind 2 = the product over the rows
// below of (1 + the cells the queens above leave free in that row).
__global__ void heuristic_cost_kernel(const uint4* __restrict__ items, uint32_t n, int kind, float* __restrict__ cost) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 s = items[i];
    uint32_t nc;
    item_avail(s, &nc);
    const uint32_t rows_left = ((s.w >> 8) & 0xFFu) - (s.w & 0xFFu);
    if (kind == 1) {
        cost[i] = log2f(1.0f + (float)__popc(nc) * (float)rows_left);
        return;
    }
    float c = 0.0f;
    for (uint32_t k = 0; k < rows_left && k < 32; ++k) c += log2f(1.0f + (float)__popc(nc & ~((s.y << k) | (s.z >> k))));
    cost[i] = c;
}

}  // namespace

int schedule_items(const nqb_state* d_items, uint32_t n, const uint32_t* d_board, const nqb_opts& o, int device,
                   cudaStream_t s, unsigned long long* d_split_nodes, unsigned long long* d_per_board_nodes,
                   Schedule* out) {
    out->items = reinterpret_cast<const uint4*>(d_items);
    out->board = d_board;
    out->order = nullptr;
    out->n = n;
    out->sched_ms = 0.0;
    const int heuristic = o.model ? 0 : o.sched_cost;  // a model takes precedence
    if (!o.model && heuristic == 0) return NQB_OK;
    if (heuristic < 0 || heuristic > 2) return NQB_E_INVALID;
    if (o.model && model_device(o.model) != device) return NQB_E_INVALID;
    const int rounds = o.max_split_rounds < 0 ? 3 : o.max_split_rounds;
    const int factor = o.split_factor > 0 ? o.split_factor : 4;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const double lanes = (double)sms * 1024.0;  // resident lanes, order of magnitude
    // With more than 64 items per resident lane the end-of-queue tail is already a tiny
    // fraction of the run (measured: N=21 d=7, 39M items, ordering changes nothing), so
    // the queue goes to the kernel as given; splitting likewise stops at that size.
    const uint64_t kMaxItems = (uint64_t)(64.0 * lanes);
    if (n > kMaxItems) return NQB_OK;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventRecord(ev0, s);
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
        }
    } ev_guard{ev0, ev1};

    Buf<uint4> items[2] = {Buf<uint4>(s), Buf<uint4>(s)};
    Buf<uint32_t> board[2] = {Buf<uint32_t>(s), Buf<uint32_t>(s)};
    Buf<float> cost(s);
    Buf<uint32_t> k(s), offs(s);
    Buf<double> work(s);
    Buf<unsigned char> tmp(s);
    int cur = -1;  // -1: the caller's arrays
    const uint4* cur_items = reinterpret_cast<const uint4*>(d_items);
    const uint32_t* cur_board = d_board;
    int st = work.alloc(1);
    if (st) return st;
    for (int r = 0;; ++r) {
        if ((st = cost.alloc(n))) return st;
        if (heuristic) {
            heuristic_cost_kernel<<<(n + 255) / 256, 256, 0, s>>>(cur_items, n, heuristic, cost.p);
            if ((st = cuda_status(cudaGetLastError()))) return st;
        } else if ((st = model_predict_device(o.model, reinterpret_cast<const nqb_state*>(cur_items), n, cost.p,
                                              s))) {
            return st;
        }
        if (r >= rounds) break;
        cudaMemsetAsync(work.p, 0, sizeof(double), s);
        work_sum_kernel<<<std::max(1u, std::min((n + 255) / 256, 1024u)), 256, 0, s>>>(cost.p, n, work.p);
        if ((st = k.alloc(n)) || (st = offs.alloc(n))) return st;
        mark_kernel<<<(n + 255) / 256, 256, 0, s>>>(cur_items, cost.p, n, work.p, lanes * factor, k.p);
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, k.p, offs.p, n, s);
        if (tmp.n < tb && (st = tmp.alloc(tb))) return st;
        if ((st = cuda_status(cub::DeviceScan::ExclusiveSum(tmp.p, tb, k.p, offs.p, n, s)))) return st;
        uint32_t last_k = 0, last_off = 0;
        cudaMemcpyAsync(&last_k, k.p + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&last_off, offs.p + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
        const uint64_t total = (uint64_t)last_off + last_k;
        if (total == n || total > kMaxItems) break;  // nothing split, or too many items
        const int nxt = cur == 0 ? 1 : 0;
        if ((st = items[nxt].alloc(total)) || (st = board[nxt].alloc(total))) return st;
        split_kernel<<<(n + 255) / 256, 256, 0, s>>>(cur_items, cur_board, k.p, offs.p, n, items[nxt].p,
                                                     board[nxt].p, d_split_nodes, d_per_board_nodes);
        if ((st = cuda_status(cudaGetLastError()))) return st;
        cur = nxt;
        cur_items = items[cur].p;
        cur_board = board[cur].p;
        n = (uint32_t)total;
    }
    // order: largest predicted cost first
    Buf<float> keys_out(s);
    Buf<uint32_t> idx(s), order(s);
    if ((st = keys_out.alloc(n)) || (st = idx.alloc(n)) || (st = order.alloc(n))) return st;
    iota_kernel<<<(n + 255) / 256, 256, 0, s>>>(idx.p, n);
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, cost.p, keys_out.p, idx.p, order.p, (int)n, 0, 32, s);
    if (tmp.n < tb && (st = tmp.alloc(tb))) return st;
    if ((st = cuda_status(cub::DeviceRadixSort::SortPairsDescending(tmp.p, tb, cost.p, keys_out.p, idx.p, order.p,
                                                                    (int)n, 0, 32, s))))
        return st;
    cudaEventRecord(ev1, s);
    float ms = 0.0f;
    cudaEventSynchronize(ev1);
    cudaEventElapsedTime(&ms, ev0, ev1);
    out->sched_ms = ms;
    out->n = n;
    out->stream = s;
    out->owned_order = order.take();
    out->order = out->owned_order;
    if (cur >= 0) {
        out->owned_items = items[cur].take();
        out->owned_board = board[cur].take();
        out->items = out->owned_items;
        out->board = out->owned_board;
    }
    return NQB_OK;
}

void Schedule::release() {
    if (owned_items) dev_free(owned_items, stream);
    if (owned_board) dev_free(owned_board, stream);
    if (owned_order) dev_free(owned_order, stream);
    owned_items = nullptr;
    owned_board = nullptr;
    owned_order = nullptr;
}

// Runs the batched form on `n` device items.  `d_board` (optional) maps items to output
// slots.  Extra nodes made by splitting are added into d_out[1] (and d_per_board_nodes).
int launch_batched_scheduled(const nqb_state* d_items, uint32_t n, const uint32_t* d_board, void* d_scratch,
                             size_t scratch_bytes, unsigned long long* d_out, unsigned long long* d_per_board,
                             unsigned long long* d_per_board_nodes, const nqb_opts& o, unsigned stack_depth,
                             int device, cudaStream_t s, unsigned* launches, SchedInfo* info,
                             unsigned long long* d_lane_stats) {
    Schedule sch;
    int st = schedule_items(d_items, n, d_board, o, device, s, d_out + 1, d_per_board_nodes, &sch);
    if (!st)
        st = launch_batched(reinterpret_cast<const nqb_state*>(sch.items), sch.n, sch.order, sch.board, d_scratch,
                            scratch_bytes, d_out, d_per_board, d_per_board_nodes, o.block_size, stack_depth, device,
                            s, launches, d_lane_stats);
    sch.release();  // stream-ordered after the kernel that reads the arrays
    if (info) {
        info->items = sch.n;
        info->sched_ms = sch.sched_ms;
    }
    return st;
}

}  // namespace nqb
