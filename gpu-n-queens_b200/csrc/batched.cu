// Batched form: a persistent search kernel fed by a device work queue.
//
// The plain form (plain.cu) binds one pool state to one thread for the whole launch,
// so a warp runs as long as its largest subtree while lanes whose subtree ended sit
// idle (the loss the reference's README describes for kern_doitall_v2_regld).  Here
// the grid is one wave of blocks over all SMs and each warp keeps its lanes busy:
//   - refill: when lanes are idle and the queue still has items, the warp claims one
//     item per idle lane with a single atomicAdd on the queue head; items are taken
//     in the order of an optional permutation (e.g. largest predicted cost first);
//   - re-split: once the queue is empty, a lane with pending rows hands its shallowest
//     pending row (the largest piece of its remaining subtree) to an idle lane of the
//     same warp, which searches it as a new piece of the same item.  Nothing is waited
//     on: no spin, barrier or flag crosses warps.
// The search step is search_step.cuh.  A lane's stack holds the sentinel entry at
// `base` and its pending rows above it; giving away the bottom row turns that row's
// slot into the new sentinel, so base moves up one slot.  Because pending rows are
// strictly deeper towards the top, sentinel and rows never pass base0 + f - 1 slots
// for a piece that started with f free columns.
//
// Lane counters are 32-bit; every kEpoch rounds they are folded into 64-bit per-piece
// totals.  When a lane finishes its piece of an item, the piece's weighted count and
// nodes go to the warp's totals and, optionally, to per-board slots (64-bit atomics).
#include <algorithm>
#include <mutex>

#include "nqb_internal.h"
#include "search_step.cuh"

namespace nqb {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint32_t kNoItem = 0xFFFFFFFFu;
#ifndef NQB_BATCHED_UNROLL
#define NQB_BATCHED_UNROLL 16
#endif
constexpr int kUnroll = NQB_BATCHED_UNROLL;  // search steps between idle-lane checks
constexpr uint32_t kEpoch = 1u << 26;        // rounds between folds: kUnroll x kEpoch < 2^32

struct BatchArgs {
    const uint4* items;        // search states (nqb_state layout)
    const uint32_t* order;     // optional: queue position -> item index
    const uint32_t* board_of;  // optional: item index -> output slot (default: item index)
    uint32_t n_items;
    uint32_t stack_depth;
    uint32_t* head;                       // queue head, zero at launch
    unsigned long long* out;              // {weighted count, nodes, 0, error flags}
    unsigned long long* per_board;        // optional: weighted count per board
    unsigned long long* per_board_nodes;  // optional: nodes per board
};

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) batched_search_kernel(const BatchArgs a) {
    extern __shared__ uint4 stack[];  // [stack_depth + 1][BLOCK]
    constexpr int kStride = BLOCK * 16;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t base0 = (uint32_t)__cvta_generic_to_shared(stack) + tid * 16;

    const uint32_t top = base0 + a.stack_depth * kStride;  // the lane's last slot
    uint32_t base = base0;
    write_sentinel(base0);
    Lane s;
    lane_park(s, base);
    s.sols = 0;
    s.nodes = 0;
    s.err = 0;
    uint32_t weight = 0, item = kNoItem;
    unsigned long long piece_sols = 0, piece_nodes = 0;  // folded lane counters of the current piece
    unsigned long long total = 0, total_nodes = 0;
    bool bad = false, qempty = false;
    uint32_t epoch = kEpoch;

    for (;;) {
        const bool me_idle = s.avail == 0 && s.sp == base;
        const uint32_t idle = __ballot_sync(kFull, me_idle);
        if (idle) {
            if (me_idle && item != kNoItem) {  // the lane's piece of work is complete
                piece_sols += s.sols;
                piece_nodes += s.nodes;
                const unsigned long long c = piece_sols * weight;
                total += c;
                total_nodes += piece_nodes;
                const uint32_t slot = a.board_of ? __ldg(a.board_of + item) : item;
                if (a.per_board && c) atomicAdd(a.per_board + slot, c);
                if (a.per_board_nodes && piece_nodes) atomicAdd(a.per_board_nodes + slot, piece_nodes);
                item = kNoItem;
                s.sols = s.nodes = 0;
                piece_sols = piece_nodes = 0;
            }
            if (!qempty) {
                const uint32_t k = __popc(idle);
                uint32_t start = 0;
                if (lane == 0) start = atomicAdd(a.head, k);
                start = __shfl_sync(kFull, start, 0);
                if (start + k >= a.n_items) qempty = true;
                const uint32_t q = start + __popc(idle & lt_mask);
                if (me_idle && q < a.n_items) {
                    const uint32_t it = a.order ? __ldg(a.order + q) : q;
                    const uint4 st = __ldg(a.items + it);
                    base = base0;
                    write_sentinel(base0);
                    if (lane_load(s, st, base) > a.stack_depth) {
                        bad = true;  // skip the item: its search could overrun the stack
                        lane_park(s, base);
                        s.sols = 0;
                    } else {
                        weight = (st.w >> 16) & 0xFFu;
                        item = it;
                    }
                }
            } else {
                const uint32_t donors = __ballot_sync(kFull, !me_idle && s.sp != base);
                if (!donors) {
                    if (idle == kFull) break;  // the warp's work is done
                } else {
                    const uint32_t k = min(__popc(idle), __popc(donors));
                    const uint32_t ri = __popc(idle & lt_mask);    // rank among idle lanes
                    const uint32_t rd = __popc(donors & lt_mask);  // rank among donors
                    const bool recv = me_idle && ri < k;
                    const bool give = ((donors >> lane) & 1u) && rd < k;
                    uint32_t src = lane;
                    if (recv) {  // lane of the ri-th donor
                        uint32_t m = donors;
                        for (uint32_t j = 0; j < ri; ++j) m &= m - 1u;
                        src = __ffs(m) - 1;
                    }
                    const uint32_t slot = __shfl_sync(kFull, base + kStride, src);  // donor's bottom row
                    const uint32_t dw = __shfl_sync(kFull, weight, src);
                    const uint32_t ditem = __shfl_sync(kFull, item, src);
                    __syncwarp();
                    if (recv) {
                        const uint4 e = lds128(slot);
                        base = base0;
                        write_sentinel(base0);
                        s.avail = e.x;
                        s.nc = e.y;
                        s.l = e.z;
                        s.r = e.w;
                        s.sp = base;
                        weight = dw;
                        item = ditem;
                    }
                    __syncwarp();
                    if (give) {  // the handed-over row's slot becomes the new sentinel
                        base += kStride;
                        write_sentinel(base);
                    }
                }
            }
        }
        if (--epoch == 0) {  // fold lane counters before they can wrap
            piece_sols += s.sols;
            piece_nodes += s.nodes;
            s.sols = s.nodes = 0;
            epoch = kEpoch;
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) search_step<kStride>(s, base, top);
    }

    total = warp_sum_u64(total);
    total_nodes = warp_sum_u64(total_nodes);
    const unsigned any_bad = __any_sync(kFull, bad);
    const unsigned any_bound = __any_sync(kFull, s.err != 0);  // checked builds only
    if (lane == 0) {
        if (total) atomicAdd(a.out + 0, total);
        if (total_nodes) atomicAdd(a.out + 1, total_nodes);
        if (any_bad) atomicOr(a.out + 3, 1ull);
        if (any_bound) atomicOr(a.out + 3, 2ull);
    }
}

template <int BLOCK>
int launch_batched_t(const BatchArgs& a, int device, cudaStream_t stream, unsigned* launches) {
    auto kern = batched_search_kernel<BLOCK>;
    const size_t smem = (size_t)(a.stack_depth + 1) * BLOCK * sizeof(uint4);
    if (smem > 227 * 1024) return NQB_E_RANGE;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e);
    int sms = 0, per_sm = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return cuda_status(e);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BLOCK, smem)) != cudaSuccess)
        return cuda_status(e);
    if (per_sm < 1) return NQB_E_RANGE;
    const uint64_t need = ((uint64_t)a.n_items + BLOCK - 1) / BLOCK;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sms * per_sm, need));
    kern<<<grid, BLOCK, smem, stream>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
    if (launches) (*launches)++;
    return NQB_OK;
}

}  // namespace

int launch_batched(const nqb_state* d_items, uint32_t n_items, const uint32_t* d_order, const uint32_t* d_board_of,
                   uint32_t* d_head, unsigned long long* d_out, unsigned long long* d_per_board,
                   unsigned long long* d_per_board_nodes, int block_size, unsigned stack_depth, int device,
                   cudaStream_t stream, unsigned* launches) {
    if (!d_out || !d_head || (n_items && !d_items)) return NQB_E_INVALID;
    if (n_items == 0) return NQB_OK;
    if (n_items > (1u << 31)) return NQB_E_RANGE;
    if (stack_depth == 0) stack_depth = NQB_MAX_N - 1;
    if (stack_depth > NQB_MAX_N) return NQB_E_INVALID;
    BatchArgs a;
    a.items = reinterpret_cast<const uint4*>(d_items);
    a.order = d_order;
    a.board_of = d_board_of;
    a.n_items = n_items;
    a.stack_depth = stack_depth;
    a.head = d_head;
    a.out = d_out;
    a.per_board = d_per_board;
    a.per_board_nodes = d_per_board_nodes;
    if (block_size == 0) block_size = 128;
    switch (block_size) {
        case 64: return launch_batched_t<64>(a, device, stream, launches);
        case 128: return launch_batched_t<128>(a, device, stream, launches);
        case 256: return launch_batched_t<256>(a, device, stream, launches);
        default: return NQB_E_INVALID;
    }
}

}  // namespace nqb

// ---- Batched launch that allocates nothing -------------------------------------
//
// Scratch of nqb_batched_launch_static: the batched kernel's queue head lives in this
// file-scope device array instead of a buffer the caller allocates.  Every GPU that
// loads the library holds these 256 bytes until the process exits; word 0 is the queue
// head, the rest is unused headroom.  In host code `g_static_scratch` only names the
// symbol: its device address is looked up with cudaGetSymbolAddress, once per device,
// and that address is what the kernel receives.
static __device__ __align__(256) uint32_t g_static_scratch[NQB_STATIC_SCRATCH_BYTES / 4];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
uint32_t* g_static_addr[kMaxDevices] = {};

// Device address of g_static_scratch on the current device (set up on first use).
int static_scratch_address(int dev, uint32_t** out) {
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return nqb::cuda_status(e);
        g_static_addr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_static_addr[dev];
    return NQB_OK;
}

}  // namespace

extern "C" int nqb_batched_launch_static(const nqb_state* d_items, uint64_t count, const uint32_t* d_order,
                                         uint64_t* d_out, int block_size, unsigned stack_depth, void* stream) {
    if (count > NQB_STATIC_MAX_ITEMS) return NQB_E_RANGE;
    if (!d_out || (count && !d_items)) return NQB_E_INVALID;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NQB_E_NODEVICE;
    if (dev < 0 || dev >= kMaxDevices) return NQB_E_RANGE;
    uint32_t* head = nullptr;
    const int s = static_scratch_address(dev, &head);
    if (s != NQB_OK) return s;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The array keeps the previous call's head; the queue must start empty.
    const cudaError_t e = cudaMemsetAsync(head, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return nqb::cuda_status(e);
    return nqb::launch_batched(d_items, (uint32_t)count, d_order, nullptr, head,
                               reinterpret_cast<unsigned long long*>(d_out), nullptr, nullptr, block_size,
                               stack_depth, dev, st, nullptr);
}
