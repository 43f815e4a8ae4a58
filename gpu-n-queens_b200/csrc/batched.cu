// Batched form: a persistent search kernel fed by a device work queue, with work
// stealing across warps.
//
// The plain form (plain.cu) binds one pool state to one thread for the whole launch,
// so a warp runs as long as its largest subtree while lanes whose subtree ended sit
// idle (the loss the reference's README describes for kern_doitall_v2_regld).  Here
// the grid is one wave of blocks over all SMs and each warp keeps its lanes busy:
//   - refill: when lanes are idle and the queue still has items, the warp claims one
//     item per idle lane with a single atomicAdd on the queue head; items are taken
//     in the order of an optional permutation (e.g. largest predicted cost first).  With
//     fewer items than the grid has lanes (the SPREAD instance) a warp claims only its
//     share, so the items reach every warp before any splitting starts;
//   - re-split inside the warp: once the queue is empty, a lane with pending rows hands
//     its shallowest pending row (the largest piece of its remaining subtree) to an idle
//     lane of the same warp, which searches it as a new piece of the same item;
//   - stealing across warps (when the launch has a steal ring): a warp with no work left
//     registers as hungry and takes rows from a device ring; while hungry warps exist,
//     busy warps publish the shallowest pending rows of their lanes into it, so a long
//     subtree spreads over every warp of the GPU instead of ending on one.
// The search step is search_step.cuh.  A lane's stack holds the sentinel entry at
// `base` and its pending rows above it; giving away the bottom row turns that row's
// slot into the new sentinel, so base moves up one slot.  Because pending rows are
// strictly deeper towards the top, sentinel and rows never pass base0 + f - 1 slots
// for a piece that started with f free columns.
//
// Steal ring: `ring_cap` slots (a power of two) of 32 bytes, {avail, nc, l, r} then
// {item, weight, turn, 0}; monotonic 32-bit head and tail in the control words; slot
// idx % cap is written by the producer of idx when turn == 2 x lap (lap = idx / cap) and
// released with turn = 2 x lap + 1, and read by the consumer of idx, which hands it back
// with turn = 2 x lap + 2 (the bounded queue of D. Vyukov).  Producers move the tail only
// by a compare-and-swap against the snapshot that found the ring under half full, so they
// never wait a lap.  A warp may leave the kernel when every warp that has started is
// hungry and the ring is empty: no warp then holds work (a warp that has just claimed rows
// stays counted until it has them, and searches them itself; a warp that starts later
// finds the item queue empty).  Counting started warps rather than the grid keeps this
// right even when not every block is resident.  Every wait -- a hungry warp's polls, a
// slot's turn -- is bounded by `wait_limit` polls without progress; a warp that gives up
// sets error bit 4 (NQB_E_STALL on the host) and leaves, and the launch's result is not
// to be used.
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
#define NQB_BATCHED_UNROLL 48
#endif
// Search steps between idle-lane checks.  Measured at N=19..21 (depth 7): 32 is 7% faster
// than 16 (the per-round checks cost more than the idle lanes they save), 48 another 0.75%,
// and 64 is slower again.
constexpr int kUnroll = NQB_BATCHED_UNROLL;
constexpr uint32_t kEpoch = (1u << 27) / kUnroll;  // rounds between folds: 31 nodes x kUnroll x kEpoch < 2^32
constexpr uint32_t kDonateEvery = 16;        // rounds between a busy warp's looks at the hungry count
// The spread instance (launches with fewer items than lanes) looks 8x less often.  Measured on
// coarse pools against every 16 and 64 rounds: N=19 d=4 215 / 205 / 196 ms, N=20 d=4 1400 /
// 1385 / 1373 ms, the 65,536 uneven boards 1836 ms at 64 and 1824 ms at 128; only the smallest
// launch (N=17 d=3, 9 ms) is faster at 64, by 0.5 ms.  256 is no better than 128.
constexpr uint32_t kDonateEverySpread = 8 * kDonateEvery;

// Error flags written to out[3].
constexpr unsigned long long kErrStack = 1ull;  // an item needed a deeper stack than provided
constexpr unsigned long long kErrBound = 2ull;  // checked builds: a push would have passed a lane's last slot
constexpr unsigned long long kErrStall = 4ull;  // a bounded wait of the work stealing ran out

struct BatchArgs {
    const uint4* items;        // search states (nqb_state layout)
    const uint32_t* order;     // optional: queue position -> item index
    const uint32_t* board_of;  // optional: item index -> output slot (default: item index)
    uint32_t n_items;
    uint32_t stack_depth;
    uint32_t* ctl;                        // zero at launch: item head, hungry warps, ring head, ring tail,
                                          // started warps
    uint4* ring;                          // steal ring (2 x uint4 per slot), turn words zero at launch
    uint32_t ring_cap;                    // slots, a power of two; 0 = no stealing across warps
    uint32_t ring_shift;                  // log2(ring_cap)
    uint32_t wait_limit;                  // polls without progress before a wait gives up
    unsigned long long* out;              // {weighted count, nodes, 0, error flags}
    unsigned long long* per_board;        // optional: weighted count per board
    unsigned long long* per_board_nodes;  // optional: nodes per board
    unsigned long long* lane_stats;       // LANES builds: {lane-steps that placed, lane-step slots}
};

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Waits (bounded) until a ring slot's turn word reads `want`.
__device__ __forceinline__ bool wait_turn(const uint32_t* turn, uint32_t want, uint32_t limit) {
    for (uint32_t i = 0;; ++i) {
        if (ld_acquire(turn) == want) return true;
        if (i >= limit) return false;
        __nanosleep(64);
    }
}

template <int BLOCK, bool LANES, bool SPREAD>
__global__ void __launch_bounds__(BLOCK) batched_search_kernel(const BatchArgs a) {
    extern __shared__ uint4 stack[];  // [stack_depth + 1][BLOCK]
    constexpr int kStride = BLOCK * 16;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t base0 = (uint32_t)__cvta_generic_to_shared(stack) + tid * 16;
    uint32_t* const hungry_warps = a.ctl + 1;
    uint32_t* const ring_head = a.ctl + 2;  // ring head and tail: one 8-byte word
    uint32_t* const ring_tail = a.ctl + 3;
    uint32_t* const started_warps = a.ctl + 4;
    if (a.ring_cap && lane == 0) atomicAdd(started_warps, 1u);

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
    unsigned long long placed64 = 0, rounds64 = 0;       // LANES builds
    uint32_t placed = 0;
    bool bad = false, qempty = false, stalled = false;
    uint32_t epoch = kEpoch, rounds = 0;

    // An idle lane of rank `rank` < k takes ring row start + rank (bounded wait for its turn).
    auto take_row = [&](uint32_t start, uint32_t k, bool mine, uint32_t rank) {
        if (!mine || rank >= k) return;
        const uint32_t idx = start + rank;
        uint4* slot = a.ring + 2ull * (idx & (a.ring_cap - 1u));
        uint32_t* turn = reinterpret_cast<uint32_t*>(slot + 1) + 2;
        const uint32_t lap = idx >> a.ring_shift;
        if (wait_turn(turn, 2u * lap + 1u, a.wait_limit)) {
            const uint4 row = __ldcg(slot);
            const uint4 meta = __ldcg(slot + 1);
            st_release(turn, 2u * lap + 2u);
            base = base0;
            write_sentinel(base0);
            s.avail = row.x;
            s.nc = row.y;
            s.l = row.z;
            s.r = row.w;
            s.sp = base;
            item = meta.x;
            weight = meta.y;
        } else {
            stalled = true;  // the row is lost: the launch reports a stall
        }
    };

    // SPREAD (launches with fewer items than lanes): a refill claims only the warp's share of
    // the items, so they spread over every warp before any splitting starts.  A separate
    // instance: the same few instructions cost the large launches 2.5% (measured at N=21).
    const uint32_t claim_cap =
        SPREAD ? max(1u, (a.n_items + gridDim.x * (BLOCK / 32) - 1) / (gridDim.x * (BLOCK / 32))) : 0u;

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
                const uint32_t k = SPREAD ? min((uint32_t)__popc(idle), claim_cap) : (uint32_t)__popc(idle);
                uint32_t start = 0;
                if (lane == 0) start = atomicAdd(a.ctl, k);
                start = __shfl_sync(kFull, start, 0);
                if (start + k >= a.n_items) qempty = true;
                const uint32_t ri = __popc(idle & lt_mask);
                const uint32_t q = start + ri;
                if (me_idle && (!SPREAD || ri < k) && q < a.n_items) {
                    const uint32_t it = a.order ? __ldg(a.order + q) : q;
                    const uint4 st = __ldg(a.items + it);
                    base = base0;
                    write_sentinel(base0);
                    if (lane_load(s, st, base) > a.stack_depth) {
                        bad = true;  // skip the item: its search could overrun the stack
                        lane_park(s, base);
                        s.sols = 0;
                        s.nodes = 0;
                    } else {
                        weight = (st.w >> 16) & 0xFFu;
                        item = it;
                    }
                }
            } else {
                const uint32_t donors = __ballot_sync(kFull, !me_idle && s.sp != base);
                if (!donors) {
                    if (idle == kFull) {  // the warp has no work left
                        if (!a.ring_cap) break;
                        // Register as hungry, then poll the ring: claim up to 32 rows, or
                        // leave once every started warp is hungry and the ring is empty.
                        if (lane == 0) atomicAdd(hungry_warps, 1u);
                        uint32_t k = 0, start = 0, done = 0;
                        if (lane == 0) {
                            unsigned long long last_ht = ~0ull;
                            uint32_t last_g = ~0u, polls = 0, nap = 128;
                            for (;;) {
                                const unsigned long long ht =
                                    ld_relaxed64(reinterpret_cast<const unsigned long long*>(ring_head));
                                const uint32_t h = (uint32_t)ht, t = (uint32_t)(ht >> 32);
                                if (t != h) {
                                    const uint32_t want = min(t - h, 32u);
                                    if (atomicCAS(ring_head, h, h + want) == h) {
                                        k = want;
                                        start = h;
                                        break;
                                    }
                                    polls = 0;  // another warp took rows: retry at once
                                    nap = 128;
                                    continue;
                                }
                                const uint32_t g = ld_relaxed(hungry_warps);
                                if (g == ld_relaxed(started_warps)) {
                                    done = 1;
                                    break;
                                }
                                if (ht != last_ht || g != last_g) {
                                    last_ht = ht;
                                    last_g = g;
                                    polls = 0;
                                    nap = 128;
                                } else if (++polls >= a.wait_limit) {
                                    done = 2;
                                    break;
                                }
                                __nanosleep(nap);
                                if (nap < 16384) nap <<= 1;
                            }
                        }
                        k = __shfl_sync(kFull, k, 0);
                        start = __shfl_sync(kFull, start, 0);
                        done = __shfl_sync(kFull, done, 0);
                        if (done) {
                            stalled |= done == 2;
                            break;
                        }
                        take_row(start, k, true, lane);
                        __syncwarp();
                        if (lane == 0) atomicSub(hungry_warps, 1u);
                        rounds = 0;
                    }
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
        // Publish rows for hungry warps: while the ring holds fewer than 32 rows per hungry
        // warp (and at most half its slots), lanes with pending rows give their bottom row.
        // A warp whose lanes are all busy looks at the hungry count too: it need not have
        // seen the item queue run dry itself (hungry warps exist only once it has).  The tail
        // only moves by a compare-and-swap against the snapshot the room was computed from,
        // so the ring never holds more than half its slots and a producer never waits a lap.
        if (a.ring_cap && ++rounds == (SPREAD ? kDonateEverySpread : kDonateEvery)) {
            rounds = 0;
            const uint32_t donors = __ballot_sync(kFull, s.sp != base);
            if (donors) {
                uint32_t k = 0, t0 = 0;
                if (lane == 0) {
                    const uint32_t g = ld_relaxed(hungry_warps);
                    if (g) {
                        const unsigned long long ht =
                            ld_relaxed64(reinterpret_cast<const unsigned long long*>(ring_head));
                        const uint32_t h = (uint32_t)ht, t = (uint32_t)(ht >> 32);
                        const uint32_t need = min(32u * g, a.ring_cap >> 1);
                        if (t - h < need) {
                            k = min((uint32_t)__popc(donors), need - (t - h));
                            if (atomicCAS(ring_tail, t, t + k) == t) t0 = t;
                            else k = 0;  // another warp published first: look again next time
                        }
                    }
                }
                k = __shfl_sync(kFull, k, 0);
                t0 = __shfl_sync(kFull, t0, 0);
                const uint32_t rd = __popc(donors & lt_mask);
                if (((donors >> lane) & 1u) && rd < k) {
                    const uint32_t idx = t0 + rd;
                    uint4* slot = a.ring + 2ull * (idx & (a.ring_cap - 1u));
                    uint32_t* turn = reinterpret_cast<uint32_t*>(slot + 1) + 2;
                    const uint32_t lap = idx >> a.ring_shift;
                    if (wait_turn(turn, 2u * lap, a.wait_limit)) {
                        __stcg(slot, lds128(base + kStride));
                        __stcg(reinterpret_cast<uint2*>(slot + 1), make_uint2(item, weight));
                        st_release(turn, 2u * lap + 1u);
                        base += kStride;  // the row is given away: its slot becomes the sentinel
                        write_sentinel(base);
                    } else {
                        stalled = true;  // the claimed slot stays empty: its consumer reports it too
                    }
                }
            }
        }
        if (--epoch == 0) {  // fold lane counters before they can wrap
            piece_sols += s.sols;
            piece_nodes += s.nodes;
            s.sols = s.nodes = 0;
            placed64 += placed;
            placed = 0;
            epoch = kEpoch;
        }
        if (LANES) ++rounds64;
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const StepInfo si = search_step<kStride>(s, base, top);
            if (LANES) placed += (si.placed != 0u);
        }
    }

    total = warp_sum_u64(total);
    total_nodes = warp_sum_u64(total_nodes);
    const unsigned any_bad = __any_sync(kFull, bad);
    const unsigned any_bound = __any_sync(kFull, s.err != 0);  // checked builds only
    const unsigned any_stall = __any_sync(kFull, stalled);
    if (LANES) {
        placed64 = warp_sum_u64(placed64 + placed);
        if (lane == 0) {
            atomicAdd(a.lane_stats + 0, placed64);
            atomicAdd(a.lane_stats + 1, 32ull * kUnroll * rounds64);
        }
    }
    if (lane == 0) {
        if (total) atomicAdd(a.out + 0, total);
        if (total_nodes) atomicAdd(a.out + 1, total_nodes);
        if (any_bad) atomicOr(a.out + 3, kErrStack);
        if (any_bound) atomicOr(a.out + 3, kErrBound);
        if (any_stall) atomicOr(a.out + 3, kErrStall);
    }
}

template <int BLOCK, bool LANES>
int launch_batched_t(const BatchArgs& a, int device, cudaStream_t stream, unsigned* launches) {
    const size_t smem = (size_t)(a.stack_depth + 1) * BLOCK * sizeof(uint4);
    if (smem > 227 * 1024) return NQB_E_RANGE;
    auto kern = batched_search_kernel<BLOCK, LANES, false>;
    auto spread = batched_search_kernel<BLOCK, LANES, true>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(spread, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e);
    int sms = 0, per_sm = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return cuda_status(e);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BLOCK, smem)) != cudaSuccess)
        return cuda_status(e);
    if (per_sm < 1) return NQB_E_RANGE;
    const uint64_t need = ((uint64_t)a.n_items + BLOCK - 1) / BLOCK;
    // One wave of blocks; with stealing, fewer items than lanes still fill the whole GPU.
    const uint64_t wave = (uint64_t)sms * per_sm;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, a.ring_cap ? wave : std::min<uint64_t>(wave, need));
    if (a.ring_cap && (uint64_t)a.n_items < (uint64_t)grid * BLOCK)
        spread<<<grid, BLOCK, smem, stream>>>(a);
    else
        kern<<<grid, BLOCK, smem, stream>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
    if (launches) (*launches)++;
    return NQB_OK;
}

}  // namespace

uint32_t batched_ring_slots(size_t scratch_bytes) {
    if (scratch_bytes < kBatchedCtlBytes + 2 * kBatchedSlotBytes) return 0;
    const uint64_t slots = (scratch_bytes - kBatchedCtlBytes) / kBatchedSlotBytes;
    uint32_t cap = 1;
    while ((uint64_t)cap * 2 <= slots && cap < (1u << 30)) cap *= 2;
    return cap;
}

int launch_batched(const nqb_state* d_items, uint32_t n_items, const uint32_t* d_order, const uint32_t* d_board_of,
                   void* d_scratch, size_t scratch_bytes, unsigned long long* d_out,
                   unsigned long long* d_per_board, unsigned long long* d_per_board_nodes, int block_size,
                   unsigned stack_depth, int device, cudaStream_t stream, unsigned* launches,
                   unsigned long long* d_lane_stats, uint32_t wait_limit) {
    if (!d_out || !d_scratch || scratch_bytes < sizeof(uint32_t) || (n_items && !d_items)) return NQB_E_INVALID;
    if (n_items == 0) return NQB_OK;
    if (n_items > (1u << 31)) return NQB_E_RANGE;
    if (stack_depth == 0) stack_depth = NQB_MAX_N - 1;
    if (stack_depth > NQB_MAX_N) return NQB_E_INVALID;
    // a steal ring needs the control words and its slots 16-byte aligned
    if (batched_ring_slots(scratch_bytes) && (reinterpret_cast<uintptr_t>(d_scratch) & 15) != 0)
        return NQB_E_INVALID;
    BatchArgs a;
    a.items = reinterpret_cast<const uint4*>(d_items);
    a.order = d_order;
    a.board_of = d_board_of;
    a.n_items = n_items;
    a.stack_depth = stack_depth;
    a.ctl = static_cast<uint32_t*>(d_scratch);
    a.ring_cap = batched_ring_slots(scratch_bytes);
    a.ring_shift = 0;
    while ((1u << a.ring_shift) < a.ring_cap) ++a.ring_shift;
    a.ring = a.ring_cap ? reinterpret_cast<uint4*>(static_cast<char*>(d_scratch) + kBatchedCtlBytes) : nullptr;
    a.wait_limit = wait_limit ? wait_limit : kBatchedWaitLimit;
    a.out = d_out;
    a.per_board = d_per_board;
    a.per_board_nodes = d_per_board_nodes;
    a.lane_stats = d_lane_stats;
    if (block_size == 0) block_size = 128;
    const bool lanes = d_lane_stats != nullptr;
    switch (block_size) {
        case 64:
            return lanes ? launch_batched_t<64, true>(a, device, stream, launches)
                         : launch_batched_t<64, false>(a, device, stream, launches);
        case 128:
            return lanes ? launch_batched_t<128, true>(a, device, stream, launches)
                         : launch_batched_t<128, false>(a, device, stream, launches);
        case 256:
            return lanes ? launch_batched_t<256, true>(a, device, stream, launches)
                         : launch_batched_t<256, false>(a, device, stream, launches);
        default:
            return NQB_E_INVALID;
    }
}

}  // namespace nqb

// ---- Batched launch that allocates nothing -------------------------------------
//
// Scratch of nqb_batched_launch_static: the batched kernel's queue head lives in this
// file-scope device array instead of a buffer the caller allocates.  Every GPU that
// loads the library holds these 256 bytes until the process exits; word 0 is the queue
// head, the rest is unused headroom.  In host code `g_static_scratch` only names the
// symbol: its device address is looked up with cudaGetSymbolAddress, once per device
// and context, and that address is what the kernel receives.
static __device__ __align__(256) uint32_t g_static_scratch[NQB_STATIC_SCRATCH_BYTES / 4];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
uint32_t* g_static_addr[kMaxDevices] = {};
unsigned long long g_static_ctx[kMaxDevices] = {};  // context the address belongs to

// Device address of g_static_scratch on the current device (set up on first use, and again
// after a device reset: the new context loads the module, and the array, anew).
int static_scratch_address(int dev, uint32_t** out) {
    std::lock_guard<std::mutex> lock(g_static_mu);
    const unsigned long long ctx = nqb::current_context_id();
    if (!g_static_addr[dev] || ctx == 0 || ctx != g_static_ctx[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return nqb::cuda_status(e);
        g_static_addr[dev] = static_cast<uint32_t*>(p);
        g_static_ctx[dev] = nqb::current_context_id();  // set up by the lookup if it was not yet
    }
    *out = g_static_addr[dev];
    return NQB_OK;
}

}  // namespace

extern "C" int nqb_batched_launch_static(const nqb_state* d_items, uint64_t count, const uint32_t* d_order,
                                         uint64_t* d_out, int block_size, unsigned stack_depth, void* stream) try {
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
    return nqb::launch_batched(d_items, (uint32_t)count, d_order, nullptr, head, sizeof(uint32_t),
                               reinterpret_cast<unsigned long long*>(d_out), nullptr, nullptr, block_size,
                               stack_depth, dev, st, nullptr);
} NQB_ABI_CATCH
