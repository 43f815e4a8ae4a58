// Pool generation on the GPU: the same prefixes, in the same order, as the host generator
// (pool.cpp) and the reference's gen_states_threaded_rowlock (n_queens.cu:235-315), built level
// by level so the pool never crosses PCIe.
//
// Level r holds every valid placement of rows [0, r) in lexicographic order of their
// columns (row 0 restricted to columns < ceil(n/2), the mirror elimination).  Expanding a
// level writes each state's children (one per free column of row r, lowest column first)
// contiguously at the state's offset from an exclusive scan of the child counts, so level
// r + 1 is again in lexicographic order, which is the reference's depth-first order.  The
// last step keeps the depth-`depth` prefixes whose next row still has a free column
// (n_queens.cu:46-49), by a scan of 0/1 flags and a scatter.
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

// keep_only != 0: k[i] = (state i has a free column); else k[i] = its number of children.
__global__ void child_count_kernel(const uint4* __restrict__ st, uint32_t m, int keep_only, uint32_t* __restrict__ k) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t f = free_cols(st[i]);
    k[i] = keep_only ? (f != 0u) : (uint32_t)__popc(f);
}

__global__ void expand_kernel(const uint4* __restrict__ st, uint32_t m, const uint32_t* __restrict__ offs,
                              uint4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint4 s = st[i];
    uint32_t f = free_cols(s);
    uint32_t o = offs[i];
    while (f) {
        const uint32_t b = f & (0u - f);
        f ^= b;
        out[o++] = make_uint4(s.x | b, (s.y | b) << 1, (s.z | b) >> 1, s.w + 1u);  // row + 1
    }
}

__global__ void keep_kernel(const uint4* __restrict__ st, uint32_t m, const uint32_t* __restrict__ k,
                            const uint32_t* __restrict__ offs, uint4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m && k[i]) out[offs[i]] = st[i];
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
    for (unsigned c0 = 0; c0 < (n + 1) / 2; ++c0) {
        const uint32_t b = 1u << c0;
        seed.push_back(nqb_state{b, b << 1, b >> 1, 1, (uint8_t)n, (uint8_t)(c0 < (n >> 1) ? 2 : 1), 0});
    }
    uint4* cur = nullptr;
    uint64_t m = seed.size();
    int st = dev_alloc(&cur, m * sizeof(uint4), s);
    if (!st) st = cuda_status(cudaMemcpyAsync(cur, seed.data(), m * sizeof(uint4), cudaMemcpyHostToDevice, s));
    uint32_t *k = nullptr, *offs = nullptr;
    for (unsigned row = 1; !st; ++row) {
        const bool last = row == depth;
        if ((st = dev_alloc(&k, m * sizeof(uint32_t), s))) break;
        if ((st = dev_alloc(&offs, m * sizeof(uint32_t), s))) break;
        const unsigned grid = (unsigned)((m + 255) / 256);
        child_count_kernel<<<grid, 256, 0, s>>>(cur, (uint32_t)m, last ? 1 : 0, k);
        uint64_t total = 0;
        if ((st = scan_total(k, offs, (uint32_t)m, s, &total))) break;
        if (total > 0xFFFFFFFFull) {
            st = NQB_E_RANGE;
            break;
        }
        uint4* next = nullptr;
        if ((st = dev_alloc(&next, total * sizeof(uint4), s)))
            break;
        if (last) keep_kernel<<<grid, 256, 0, s>>>(cur, (uint32_t)m, k, offs, next);
        else expand_kernel<<<grid, 256, 0, s>>>(cur, (uint32_t)m, offs, next);
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
        if (last) break;
        if (m == 0) {  // no prefix reaches the depth: an empty pool
            st = NQB_OK;
            break;
        }
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
