// Plain form: one thread per pool state, the drop-in for kern_doitall_v2_regld
// (GPU_NQueens.cu:338-452) and its launch in gpu_solver_driver (GPU_NQueens.cu:128-138).
//
// Each thread runs a depth-first search from its state.  Per row the thread keeps
// four 32-bit words in registers:
//   avail  candidate columns of the current row not tried yet
//   nc     columns still without a queen
//   l, r   columns of the current row attacked along the two diagonals
// One loop iteration places exactly one queen (one search node):
//   - when avail is empty it pops the deepest row that still has candidates from a
//     per-thread stack in shared memory (16 bytes per entry, one LDS.128),
//   - it takes the lowest candidate b, and pushes the row back (one STS.128) only if
//     candidates remain,
//   - it steps to the next row: nc ^= b, l = (l|b) << 1, r = (r|b) >> 1,
//     avail = nc & ~(l|r).
// A row that is left with no candidate is never pushed, so a row with exactly one
// free column is filled and passed through without a branch point: that is the
// reference's DoubleSweep-light unit-row propagation (GPU_NQueens.cu:392-408), and
// the set of placements (nodes) equals the reference's.  nc == 0 marks a solution
// (the reference tests cols == N_MASK, GPU_NQueens.cu:420-424).
// The warp leaves the loop by a __any_sync vote when every lane is done
// (GPU_NQueens.cu:358-360).  Counts are reduced per warp with shuffles and per
// block through shared memory, then added with one uint64 atomic per block.
#include <algorithm>

#include "nqb_internal.h"

namespace nqb {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    return v;
}

// Error flags written to out[3].
constexpr unsigned long long kErrStack = 1ull;  // a search needed more stack than provided

// per_state (optional): weight x completions of each state, for per-board results.
template <int BLOCK, bool UNIT>
__global__ void __launch_bounds__(BLOCK) plain_search_kernel(const uint4* __restrict__ states, uint32_t count,
                                                             unsigned long long* __restrict__ out,
                                                             unsigned long long* __restrict__ per_state,
                                                             uint32_t stack_depth) {
    extern __shared__ uint4 stack[];  // [stack_depth][BLOCK]
    const uint32_t tid = threadIdx.x;
    const uint32_t gi = blockIdx.x * BLOCK + tid;

    uint32_t avail = 0, nc = 0, l = 0, r = 0, weight = 0;
    unsigned long long sols = 0, nodes = 0;
    uint32_t unit = 0;
    bool first = true;
    if (gi < count) {
        const uint4 s = __ldg(states + gi);
        const uint32_t n = (s.w >> 8) & 0xFFu;
        const uint32_t mask = n >= 32 ? kFull : ((1u << n) - 1u);
        nc = mask & ~s.x;
        l = s.y;
        r = s.z;
        weight = (s.w >> 16) & 0xFFu;
        avail = nc & ~(l | r);
        sols = (nc == 0);  // a complete board handed in as a state
    }
    uint32_t sp = tid;  // next free stack slot; the stack base is tid
    const uint32_t sp_lim = tid + stack_depth * BLOCK;
    bool overflow = false;

    for (;;) {
        const bool active = (avail != 0) | (sp != tid);
        if (!__any_sync(kFull, active)) break;
        if (active) {
            bool fresh = !first;
            if (avail == 0) {  // backtrack to the deepest row with candidates left
                sp -= BLOCK;
                const uint4 e = stack[sp];
                avail = e.x;
                nc = e.y;
                l = e.z;
                r = e.w;
                fresh = false;
            }
            const uint32_t b = avail & (0u - avail);
            if (UNIT) unit += (fresh && avail == b);  // row entered with one free column
            first = false;
            avail ^= b;
            if (avail) {
                if (sp < sp_lim) {
                    stack[sp] = make_uint4(avail, nc, l, r);
                    sp += BLOCK;
                } else {  // cannot happen when stack_depth covers the states; flag it
                    overflow = true;
                    avail = 0;
                    sp = tid;
                }
            }
            nc ^= b;
            l = (l | b) << 1;
            r = (r | b) >> 1;
            avail = nc & ~(l | r);
            sols += (nc == 0);
            nodes++;
        }
    }

    unsigned long long c = sols * weight;
    if (per_state && gi < count) per_state[gi] = c;
    unsigned long long nd = nodes;
    unsigned long long un = unit;
    c = warp_sum_u64(c);
    nd = warp_sum_u64(nd);
    if (UNIT) un = warp_sum_u64(un);
    const unsigned any_overflow = __any_sync(kFull, overflow);

    __syncthreads();  // the stack area is reused for the block reduction
    unsigned long long* red = reinterpret_cast<unsigned long long*>(stack);
    const uint32_t warp = tid >> 5, lane = tid & 31;
    constexpr int kWarps = BLOCK / 32;
    if (lane == 0) {
        red[warp] = c;
        red[kWarps + warp] = nd;
        red[2 * kWarps + warp] = un;
        red[3 * kWarps + warp] = any_overflow;
    }
    __syncthreads();
    if (warp == 0) {
        c = lane < kWarps ? red[lane] : 0;
        nd = lane < kWarps ? red[kWarps + lane] : 0;
        un = lane < kWarps ? red[2 * kWarps + lane] : 0;
        unsigned long long of = lane < kWarps ? red[3 * kWarps + lane] : 0;
        c = warp_sum_u64(c);
        nd = warp_sum_u64(nd);
        un = warp_sum_u64(un);
        of = warp_sum_u64(of);
        if (lane == 0) {
            if (c) atomicAdd(out + 0, c);
            atomicAdd(out + 1, nd);
            if (UNIT && un) atomicAdd(out + 2, un);
            if (of) atomicOr(out + 3, kErrStack);
        }
    }
}

template <int BLOCK, bool UNIT>
int launch_t(const nqb_state* d_states, uint64_t count, unsigned long long* d_out,
             unsigned long long* d_per_state, unsigned stack_depth, cudaStream_t stream, unsigned* launches) {
    auto kern = plain_search_kernel<BLOCK, UNIT>;
    // Room for the stack, and for 4 x (BLOCK/32) reduction words.
    const size_t smem = std::max<size_t>((size_t)stack_depth * BLOCK * sizeof(uint4),
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
                                            stack_depth);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_status(e);
        if (launches) (*launches)++;
    }
    return NQB_OK;
}

}  // namespace

int launch_plain(const nqb_state* d_states, uint64_t count, unsigned long long* d_out,
                 unsigned long long* d_per_state, int block_size, bool count_unit, unsigned stack_depth,
                 cudaStream_t stream, unsigned* launches) {
    if (!d_out || (count && !d_states)) return NQB_E_INVALID;
    if (count == 0) return NQB_OK;
    if (stack_depth == 0) stack_depth = NQB_MAX_N - 1;
    if (stack_depth > NQB_MAX_N) return NQB_E_INVALID;
    if (block_size == 0) block_size = 128;
    switch (block_size) {
        case 64:
            return count_unit ? launch_t<64, true>(d_states, count, d_out, d_per_state, stack_depth, stream, launches)
                              : launch_t<64, false>(d_states, count, d_out, d_per_state, stack_depth, stream, launches);
        case 128:
            return count_unit ? launch_t<128, true>(d_states, count, d_out, d_per_state, stack_depth, stream, launches)
                              : launch_t<128, false>(d_states, count, d_out, d_per_state, stack_depth, stream, launches);
        case 256:
            return count_unit ? launch_t<256, true>(d_states, count, d_out, d_per_state, stack_depth, stream, launches)
                              : launch_t<256, false>(d_states, count, d_out, d_per_state, stack_depth, stream, launches);
        default:
            return NQB_E_INVALID;
    }
}

}  // namespace nqb
