// Pool generation on the GPU: the same prefixes, in the same order, as the host generator
// (pool.cpp) and the reference's gen_states_threaded_rowlock (n_queens.cu:235-315), built level
// by level so the pool never crosses PCIe.
//
// Level r holds every valid placement of rows [0, r) in lexicographic order of their
// columns (row 0 restricted to columns < ceil(n/2), the mirror elimination).  Expanding a
// level writes each state's children (one per free column of row r, lowest column first)
// contiguously at the state's offset from an exclusive scan of the child counts, so level
// r + 1 is again in lexicographic order, which is the reference's depth-first order.  The
// last expansion writes only the children whose next row still has a free column
// (n_queens.cu:46-49), so the pool is written once, at its final size.
#include <vector>

#include <cub/cub.cuh>

#include "nqb_internal.h"

namespace nqb {
namespace {

__device__ __forceinline__ uint32_t free_cols(const uint4 s) {
    const uint32_t n = (s.w >> 8) & 0xFFu;
    const uint32_t mask = n >= 32 ? 0xFFFFFFFFu : ((1u << n) - 1u);
    return mask & ~(s.x | s.y | s.z);
}

// The child of state s for column bit b: one more row placed.
__device__ __forceinline__ uint4 child_of(const uint4 s, uint32_t b) {
    return make_uint4(s.x | b, (s.y | b) << 1, (s.z | b) >> 1, s.w + 1u);  // row + 1
}

// last != 0: only children whose next row has a free column count (and are written).
__device__ __forceinline__ uint32_t children(const uint4 s, int last) {
    uint32_t f = free_cols(s);
    if (!last) return f;
    uint32_t kept = 0;
    for (uint32_t g = f; g;) {
        const uint32_t b = g & (0u - g);
        g ^= b;
        if (free_cols(child_of(s, b))) kept |= b;
    }
    return kept;
}

__global__ void child_count_kernel(const uint4* __restrict__ st, uint32_t m, int last, uint32_t* __restrict__ k) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    k[i] = (uint32_t)__popc(children(st[i], last));
}

// Position of the k-th (0-based) set bit of x, k < popc(x): the largest position with at
// most k set bits below it, found by binary search on popcounts.
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t x, uint32_t k) {
    uint32_t pos = 0;
#pragma unroll
    for (uint32_t step = 16; step; step >>= 1)
        if ((uint32_t)__popc(x & ((1u << (pos + step)) - 1u)) <= k) pos += step;
    return pos;
}

// Writes the children of 32 parents per warp as one contiguous run: output j of the run
// comes from the last lane whose child prefix is <= j (a shuffle search over the warp's
// prefix sums), as that lane's (j - prefix)-th child in column order.  Consecutive lanes
// store consecutive 16-byte states, so every warp store covers 512 contiguous bytes.
__global__ void expand_kernel(const uint4* __restrict__ st, uint32_t m, const uint32_t* __restrict__ offs, int last,
                              uint4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31;
    if ((i & ~31u) >= m) return;  // the whole warp is past the end
    const bool valid = i < m;
    const uint4 s = valid ? st[i] : make_uint4(0, 0, 0, 0);
    const uint32_t f = valid ? children(s, last) : 0u;
    const uint32_t c = __popc(f);
    uint32_t p = c;  // inclusive prefix over the warp
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, p, d);
        if (lane >= (uint32_t)d) p += v;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, p, 31);
    p -= c;  // exclusive
    const uint32_t base = __shfl_sync(0xFFFFFFFFu, valid ? offs[i] - p : 0u, 0);
    for (uint32_t j0 = 0; j0 < total; j0 += 32) {
        const uint32_t j = j0 + lane;
        uint32_t src = 0;
#pragma unroll
        for (uint32_t step = 16; step; step >>= 1) {  // last lane with prefix <= j
            const uint32_t q = __shfl_sync(0xFFFFFFFFu, p, src + step);
            if (q <= j) src += step;
        }
        const uint32_t sf = __shfl_sync(0xFFFFFFFFu, f, src);
        const uint32_t sp = __shfl_sync(0xFFFFFFFFu, p, src);
        uint4 ps;
        ps.x = __shfl_sync(0xFFFFFFFFu, s.x, src);
        ps.y = __shfl_sync(0xFFFFFFFFu, s.y, src);
        ps.z = __shfl_sync(0xFFFFFFFFu, s.z, src);
        ps.w = __shfl_sync(0xFFFFFFFFu, s.w, src);
        if (j < total) out[base + j] = child_of(ps, 1u << nth_set_bit(sf, j - sp));
    }
}

// Exclusive scan of k[0..m) into offs; returns the total.
int scan_total(const uint32_t* k, uint32_t* offs, uint32_t m, cudaStream_t s, uint64_t* total) {
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, k, offs, m, s);
    void* tmp = nullptr;
    int st = dev_alloc_bytes(&tmp, tb, s);
    if (!st) st = cuda_status(cub::DeviceScan::ExclusiveSum(tmp, tb, k, offs, m, s));
    uint32_t last_k = 0, last_o = 0;
    if (!st) st = cuda_status(cudaMemcpyAsync(&last_k, k + (m - 1), 4, cudaMemcpyDeviceToHost, s));
    if (!st) st = cuda_status(cudaMemcpyAsync(&last_o, offs + (m - 1), 4, cudaMemcpyDeviceToHost, s));
    if (tmp) dev_free(tmp, s);
    if (!st) st = cuda_status(cudaStreamSynchronize(s));
    *total = (uint64_t)last_o + last_k;
    return st;
}

}  // namespace

int generate_pool_device(unsigned n, unsigned depth, cudaStream_t s, nqb_state** d_out, uint64_t* count) {
    *d_out = nullptr;
    *count = 0;
    if (n < NQB_MIN_N || n > NQB_MAX_N || depth < 1 || depth >= n) return NQB_E_INVALID;
    // level 1: the row-0 placements of the left half (weight 2 left of centre, 1 for the
    // middle column of an odd board; GPU_NQueens.cu:354-357)
    std::vector<nqb_state> seed;
    const uint32_t mask = n >= 32 ? 0xFFFFFFFFu : ((1u << n) - 1u);
    for (unsigned c0 = 0; c0 < (n + 1) / 2; ++c0) {
        const uint32_t b = 1u << c0;
        if (depth == 1 && !(mask & ~(b | (b << 1) | (b >> 1)))) continue;  // the keep test, for a 1-row pool
        seed.push_back(nqb_state{b, b << 1, b >> 1, 1, (uint8_t)n, (uint8_t)(c0 < (n >> 1) ? 2 : 1), 0});
    }
    uint4* cur = nullptr;
    uint64_t m = seed.size();
    int st = dev_alloc(&cur, m * sizeof(uint4), s);
    if (!st && m) st = cuda_status(cudaMemcpyAsync(cur, seed.data(), m * sizeof(uint4), cudaMemcpyHostToDevice, s));
    uint32_t *k = nullptr, *offs = nullptr;
    for (unsigned row = 1; !st && row < depth; ++row) {  // level row -> row + 1
        const int last = row + 1 == depth;
        if ((st = dev_alloc(&k, m * sizeof(uint32_t), s))) break;
        if ((st = dev_alloc(&offs, m * sizeof(uint32_t), s))) break;
        const unsigned grid = (unsigned)((m + 255) / 256);
        child_count_kernel<<<grid, 256, 0, s>>>(cur, (uint32_t)m, last, k);
        uint64_t total = 0;
        if ((st = scan_total(k, offs, (uint32_t)m, s, &total))) break;
        if (total > 0xFFFFFFFFull) {
            st = NQB_E_RANGE;
            break;
        }
        uint4* next = nullptr;
        if ((st = dev_alloc(&next, total * sizeof(uint4), s))) break;
        expand_kernel<<<grid, 256, 0, s>>>(cur, (uint32_t)m, offs, last, next);
        if ((st = cuda_status(cudaGetLastError()))) {
            dev_free(next, s);
            break;
        }
        dev_free(cur, s);
        dev_free(k, s);
        dev_free(offs, s);
        k = offs = nullptr;
        cur = next;
        m = total;
        if (m == 0) break;  // no prefix reaches the depth: an empty pool
    }
    if (k) dev_free(k, s);
    if (offs) dev_free(offs, s);
    if (st) {
        if (cur) dev_free(cur, s);
        return st;
    }
    *d_out = reinterpret_cast<nqb_state*>(cur);
    *count = m;
    return NQB_OK;
}

}  // namespace nqb
