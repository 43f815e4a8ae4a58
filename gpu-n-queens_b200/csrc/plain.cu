// Plain form: one thread per pool state, the drop-in for kern_doitall_v2_regld
// (GPU_NQueens.cu:338-452) and its launch in gpu_solver_driver (GPU_NQueens.cu:128-138).
//
// Each thread runs the depth-first search of search_step.cuh from its state; the
// warp leaves the loop by a __all_sync vote once every lane is parked
// (GPU_NQueens.cu:358-360).  kUnroll steps run between votes; a lane that finishes in
// between stays parked.  Counters are 32-bit per lane and are folded into 64-bit
// totals every kEpoch votes, so no lane counter can wrap.  Counts are reduced per warp
// with shuffles and per block through shared memory, then added with one uint64
// atomic per block (the reference adds one atomic per thread, GPU_NQueens.cu:441-443).
#include <algorithm>

#include "nqb_internal.h"
#include "search_step.cuh"

namespace nqb {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kUnroll = 64;  // steps between done-votes (16 and 32 measured 0.6% slower)
constexpr uint32_t kEpoch = (1u << 27) / kUnroll;  // votes between folds: 31 nodes x kUnroll x kEpoch < 2^32

// Error flags written to out[3].
constexpr unsigned kErrStack = 1u;  // a state needed a deeper stack than provided
constexpr unsigned kErrBound = 2u;  // checked builds: a push would have passed a lane's last slot

// per_state (optional): weight x completions of each state, for per-board results.
// UNIT: also count placements made by unit-row propagation (the reference's split of
// nodes: the candidate of a row entered with exactly one candidate, other than the start
// row).  lane_stats (optional, LANES builds): {lane-steps that placed a queen, lane-step
// slots issued (32 per warp step)}: their ratio is the search loop's warp execution
// efficiency in active lanes.
template <int BLOCK, bool UNIT, bool LANES>
__global__ void __launch_bounds__(BLOCK) plain_search_kernel(const uint4* __restrict__ states, uint32_t count,
                                                             unsigned long long* __restrict__ out,
                                                             unsigned long long* __restrict__ per_state,
                                                             unsigned long long* __restrict__ lane_stats,
                                                             uint32_t stack_depth) {
    extern __shared__ uint4 stack[];  // [stack_depth + 1][BLOCK]; row 0 holds the sentinels
    constexpr int kStride = BLOCK * 16;
    const uint32_t tid = threadIdx.x;
    const uint32_t gi = blockIdx.x * BLOCK + tid;
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(stack) + tid * 16;
    const uint32_t top = base + stack_depth * kStride;  // the lane's last slot
    write_sentinel(base);

    Lane s;
    lane_park(s, base);
    s.sols = 0;
    s.nodes = 0;
    s.err = 0;
    uint32_t weight = 0;
    bool bad = false;
    if (gi < count) {
        const uint4 st = __ldg(states + gi);
        weight = (st.w >> 16) & 0xFFu;
        if (lane_load(s, st, base) > stack_depth) {
            bad = true;
            lane_park(s, base);
            s.sols = 0;
            s.nodes = 0;
        }
    }
    unsigned long long sols = 0, nodes = 0, unit64 = 0, placed64 = 0, votes = 0;
    uint32_t unit = 0, placed = 0;
    uint32_t epoch = kEpoch;
    while (!__all_sync(kFull, s.avail == 0 && s.sp == base)) {
        if (--epoch == 0) {  // fold lane counters before they can wrap
            sols += s.sols;
            nodes += s.nodes;
            s.sols = s.nodes = 0;
            unit64 += unit;
            placed64 += placed;
            unit = placed = 0;
            epoch = kEpoch;
        }
        if (LANES) ++votes;
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const StepInfo si = search_step<kStride>(s, base, top);
            if (UNIT) unit += (si.cand == 1u);
            if (LANES) placed += (si.placed != 0u);
        }
    }
    sols += s.sols;
    nodes += s.nodes;
    unit64 += unit;
    placed64 += placed;
    if (LANES) {
        const unsigned long long pw = warp_sum_u64(placed64);
        if ((tid & 31) == 0) {
            atomicAdd(lane_stats + 0, pw);
            atomicAdd(lane_stats + 1, 32ull * kUnroll * votes);
        }
    }

    unsigned long long c = sols * weight;
    if (per_state && gi < count) per_state[gi] = c;
    unsigned long long un = unit64;
    c = warp_sum_u64(c);
    nodes = warp_sum_u64(nodes);
    if (UNIT) un = warp_sum_u64(un);
    const unsigned flags = (__any_sync(kFull, bad) ? kErrStack : 0u) | (__any_sync(kFull, s.err != 0) ? kErrBound : 0u);

    __syncthreads();  // the stack area is reused for the block reduction
    unsigned long long* red = reinterpret_cast<unsigned long long*>(stack);
    const uint32_t warp = tid >> 5, lane = tid & 31;
    constexpr int kWarps = BLOCK / 32;
    if (lane == 0) {
        red[warp] = c;
        red[kWarps + warp] = nodes;
        red[2 * kWarps + warp] = un;
        red[3 * kWarps + warp] = flags;
    }
    __syncthreads();
    if (warp == 0) {
        c = lane < kWarps ? red[lane] : 0;
        nodes = lane < kWarps ? red[kWarps + lane] : 0;
        un = lane < kWarps ? red[2 * kWarps + lane] : 0;
        const unsigned of = warp_or(lane < kWarps ? (unsigned)red[3 * kWarps + lane] : 0u);
        c = warp_sum_u64(c);
        nodes = warp_sum_u64(nodes);
        un = warp_sum_u64(un);
        if (lane == 0) {
            if (c) atomicAdd(out + 0, c);
            atomicAdd(out + 1, nodes);
            if (UNIT && un) atomicAdd(out + 2, un);
            if (of) atomicOr(out + 3, (unsigned long long)of);
        }
    }
}

template <int BLOCK, bool UNIT, bool LANES>
int launch_t(const nqb_state* d_states, uint64_t count, unsigned long long* d_out,
             unsigned long long* d_per_state, unsigned long long* d_lanes, unsigned stack_depth,
             cudaStream_t stream, unsigned* launches) {
    auto kern = plain_search_kernel<BLOCK, UNIT, LANES>;
    // Room for the stack (with its sentinel row), and for 4 x (BLOCK/32) reduction words.
    const size_t smem = std::max<size_t>((size_t)(stack_depth + 1) * BLOCK * sizeof(uint4),
                                         4 * (BLOCK / 32) * sizeof(unsigned long long));
    if (smem > 227 * 1024) return NQB_E_RANGE;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e);
    const uint64_t kChunk = 1ull << 30;  // states per launch (grid.x stays < 2^31)
    const uint4* base = reinterpret_cast<const uint4*>(d_states);
    for (uint64_t off = 0; off < count; off += kChunk) {
        const uint32_t c = (uint32_t)std::min<uint64_t>(kChunk, count - off);
        const unsigned grid = (c + BLOCK - 1) / BLOCK;
        kern<<<grid, BLOCK, smem, stream>>>(base + off, c, d_out, d_per_state ? d_per_state + off : nullptr,
                                            d_lanes, stack_depth);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_status(e);
        if (launches) (*launches)++;
    }
    return NQB_OK;
}

template <int BLOCK>
int launch_block(const nqb_state* d_states, uint64_t count, unsigned long long* d_out,
                 unsigned long long* d_per_state, unsigned long long* d_lanes, bool count_unit, unsigned stack_depth,
                 cudaStream_t stream, unsigned* launches) {
    if (d_lanes)
        return count_unit ? launch_t<BLOCK, true, true>(d_states, count, d_out, d_per_state, d_lanes, stack_depth,
                                                        stream, launches)
                          : launch_t<BLOCK, false, true>(d_states, count, d_out, d_per_state, d_lanes, stack_depth,
                                                         stream, launches);
    return count_unit ? launch_t<BLOCK, true, false>(d_states, count, d_out, d_per_state, nullptr, stack_depth,
                                                     stream, launches)
                      : launch_t<BLOCK, false, false>(d_states, count, d_out, d_per_state, nullptr, stack_depth,
                                                      stream, launches);
}

}  // namespace

int launch_plain(const nqb_state* d_states, uint64_t count, unsigned long long* d_out,
                 unsigned long long* d_per_state, int block_size, bool count_unit, unsigned stack_depth,
                 cudaStream_t stream, unsigned* launches, unsigned long long* d_lane_stats) {
    if (!d_out || (count && !d_states)) return NQB_E_INVALID;
    if (count == 0) return NQB_OK;
    if (stack_depth == 0) stack_depth = NQB_MAX_N - 1;
    if (stack_depth > NQB_MAX_N) return NQB_E_INVALID;
    if (block_size == 0) block_size = 128;
    switch (block_size) {
        case 64:
            return launch_block<64>(d_states, count, d_out, d_per_state, d_lane_stats, count_unit, stack_depth,
                                    stream, launches);
        case 128:
            return launch_block<128>(d_states, count, d_out, d_per_state, d_lane_stats, count_unit, stack_depth,
                                     stream, launches);
        case 256:
            return launch_block<256>(d_states, count, d_out, d_per_state, d_lane_stats, count_unit, stack_depth,
                                     stream, launches);
        default:
            return NQB_E_INVALID;
    }
}

}  // namespace nqb
