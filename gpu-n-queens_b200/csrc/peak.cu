// INT32 issue-rate microbenchmark: the measured denominator of the search kernels'
// roofline (integer lane-ops per second this GPU sustains).
//
// Every thread runs 8 independent dependency chains of one integer instruction kind, so
// the issue rate, not latency, bounds it; the grid fills every SM at full occupancy.
// Kinds: LOP3 (logic), integer add, IMAD (multiply-add, on the FMA pipe) and an
// alternation of LOP3 and IMAD, the mix the search step is written to use.  Every op is
// one PTX instruction with no operand that needs another instruction: one lane-op.
#include "nqb_internal.h"

namespace nqb {
namespace {

constexpr int kChains = 8;
constexpr int kInner = 16;  // instructions per chain per loop iteration

template <int KIND>
__device__ __forceinline__ uint32_t op(uint32_t a, uint32_t b, uint32_t c, int j) {
    uint32_t d;
    if (KIND == 0 || (KIND == 3 && (j & 1) == 0)) {
        asm volatile("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    } else if (KIND == 1) {
        asm volatile("add.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(c));
    } else {
        asm volatile("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    }
    return d;
}

template <int KIND>
__global__ void __launch_bounds__(256) int32_peak_kernel(uint32_t iters, uint32_t seed, uint32_t* out) {
    uint32_t v[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = seed * (threadIdx.x + 1) + c * 0x9E3779B9u;
    const uint32_t k = seed | 1u;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < kInner; ++j) {
#pragma unroll
            for (int c = 0; c < kChains; ++c) v[c] = op<KIND>(v[c], k, v[(c + 1) & (kChains - 1)], j);
        }
    }
    uint32_t x = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) x ^= v[c];
    if (x == 0x12345678u) out[blockIdx.x] = x;  // keeps the chains live; practically never taken
}

template <int KIND>
int time_kind(int sms, uint32_t iters, uint32_t* d_out, cudaStream_t s, double* ops_per_s) {
    const int blocks_per_sm = 8, threads = 256;  // 2048 threads per SM
    const int grid = sms * blocks_per_sm;
    cudaEvent_t e0, e1;
    NQB_TRY(cuda_status(cudaEventCreate(&e0)));
    int st = cuda_status(cudaEventCreate(&e1));
    if (!st) {
        int32_peak_kernel<KIND><<<grid, threads, 0, s>>>(iters / 8 + 1, 7u, d_out);  // warm-up
        cudaEventRecord(e0, s);
        int32_peak_kernel<KIND><<<grid, threads, 0, s>>>(iters, 7u, d_out);
        cudaEventRecord(e1, s);
        st = cuda_status(cudaGetLastError());
        if (!st) st = cuda_status(cudaEventSynchronize(e1));
        float ms = 0.0f;
        if (!st) st = cuda_status(cudaEventElapsedTime(&ms, e0, e1));
        const double per_thread = (double)iters * kInner * kChains;
        *ops_per_s = ms > 0 ? per_thread * grid * threads / (ms * 1e-3) : 0.0;
        cudaEventDestroy(e1);
    }
    cudaEventDestroy(e0);
    return st;
}

}  // namespace
}  // namespace nqb

extern "C" int nqb_measure_int32_peak(int device, double* best, double* per_kind) try {
    using namespace nqb;
    if (!best) return NQB_E_INVALID;
    *best = 0;
    NQB_TRY(nqb_device_check(device));
    int prev = 0;
    cudaGetDevice(&prev);
    int st = cuda_status(cudaSetDevice(device));
    int sms = 0;
    if (!st) st = cuda_status(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    cudaStream_t s = nullptr;
    if (!st) st = cuda_status(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    uint32_t* d_out = nullptr;
    if (!st) st = dev_alloc(&d_out, (size_t)sms * 8 * sizeof(uint32_t), s);
    double r[4] = {0, 0, 0, 0};
    const uint32_t iters = 16384;  // 2.1 M lane-ops per thread, 0.64 T per kind: ~20 ms each
    if (!st) st = time_kind<0>(sms, iters, d_out, s, &r[0]);
    if (!st) st = time_kind<1>(sms, iters, d_out, s, &r[1]);
    if (!st) st = time_kind<2>(sms, iters, d_out, s, &r[2]);
    if (!st) st = time_kind<3>(sms, iters, d_out, s, &r[3]);
    if (d_out) dev_free(d_out, s);
    if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    cudaSetDevice(prev);
    if (st) return st;
    for (int k = 0; k < 4; ++k) {
        if (per_kind) per_kind[k] = r[k];
        if (r[k] > *best) *best = r[k];
    }
    return NQB_OK;
} NQB_ABI_CATCH
