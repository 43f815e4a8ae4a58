// Learned cost model: an MLP 112 -> 128 -> 128 -> 1 (GELU) that predicts log2 of the number
// of search nodes below a state.  Trained on the GPU by the kernels in this file (FP16
// operands, FP32 accumulation on the tensor cores; FP32 master weights, Adam), on node
// counts the batched search kernel records per item; inference (predict_kernel) runs on
// tcgen05 with the accumulator in tensor memory.  Used only to order and split the batched
// form's queue (schedule.cu); counts never depend on it.
//
// Training step on a batch of B rows (X: B x 112 fp16):
//   Z1 = X W1           H1 = gelu(Z1 + b1)      (fp16 copy of H1 feeds the next GEMM)
//   Z2 = H1 W2          H2 = gelu(Z2 + b2)
//   y  = H2 w3 + b3     loss = mean (y - t)^2
//   dy = 2 (y - t)      dZ2 = dy w3^T * gelu'(Z2 + b2)      dH1 = dZ2 W2^T
//   dZ1 = dH1 * gelu'(Z1 + b1)
//   dW2 = H1^T dZ2 / B  dW1 = X^T dZ1 / B  dw3 = H2^T dy / B  (bias grads: column sums / B)
// All GEMMs go through one tcgen05 kernel with arbitrary operand strides (gemm_tc).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "mlp.cuh"
#include "nqb_internal.h"

namespace nqb {
namespace mlp {
namespace {

// ---- tcgen05 building blocks -----------------------------------------------------------
// Operand tiles are 128 rows x K fp16 in the 128-byte-swizzled K-major layout: 16-byte
// chunk j (8 K-elements) of row r sits at (j / 8) x 16 KB + r x 128 + ((j % 8) ^ (r % 8)) x 16
// from a 1024-byte-aligned base.  One thread issues the MMAs; the accumulator lives in
// tensor memory and each warp reads its 32 lanes back with tcgen05.ld.
constexpr int kTileRows = 128;
constexpr uint32_t kOpBytes = kTileRows * 128 * 2;  // one 128 x 128 fp16 operand tile: 32 KB
constexpr uint32_t kAtomBytes = kTileRows * 128;    // 64 K-elements (128 B) of all 128 rows: 16 KB
constexpr uint32_t kTmemCols = 128;
constexpr uint32_t kSpinLimit = 1u << 22;  // waits: far above the ~1 us a product takes
// instruction descriptor, kind::f16: D fp32 (bits 4-5 = 1), A and B fp16 and K-major,
// N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t kIdesc = (1u << 4) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
constexpr size_t kPredictSmem = 1024 /* alignment slack */ + 3 * kOpBytes + (3 * kH + 4) * sizeof(float) + 16;

__device__ __forceinline__ uint32_t sw128_chunk(uint32_t r, uint32_t j) {
    return (j >> 3) * kAtomBytes + r * 128u + (((j & 7u) ^ (r & 7u)) << 4);
}

// Shared-memory matrix descriptor of a 128-byte-swizzled K-major tile starting at `addr`
// (1024-byte aligned atom, or an offset of 32 bytes times the K step inside it).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu)  // start address, 16-byte units
           | ((uint64_t)1u << 16)             // leading byte offset (not used with swizzling)
           | ((uint64_t)(1024u >> 4) << 32)   // stride byte offset: 8 rows x 128 B
           | ((uint64_t)1u << 46)             // descriptor version of sm_100
           | ((uint64_t)2u << 61);            // 128-byte swizzle
}

// Byte offset of K step k (16 elements) inside an operand tile.
__device__ __forceinline__ uint32_t kstep_offset(int k) { return (uint32_t)(k >> 2) * kAtomBytes + (uint32_t)(k & 3) * 32u; }

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %3, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %4, {%5, %5, %5, %5}, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(accumulate), "r"(kIdesc), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// Bounded wait for a phase of the completion barrier.  By default mbarrier.try_wait, which
// may suspend the thread until the phase completes (no issue slots burnt while the tensor
// cores work); with probe_only, `limit` non-blocking mbarrier.test_wait probes, an exact
// count whatever the hardware's suspend time (a caller-chosen bound).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t limit = kSpinLimit,
                                          bool probe_only = false) {
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        if (probe_only)
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(bar), "r"(parity)
                : "memory");
        else
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(bar), "r"(parity)
                : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_half2(float a, float b) {
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// ---- GEMM: C (M x N, fp32, row-major ldc) = alpha * A x B, on tcgen05 ----------------------
// A(i, k) = A[i * sai + k * sak], B(k, j) = B[k * sbk + j * sbj], fp16; N <= 128.  A block
// owns 128 rows of C and a range of K; every 64-element K step is loaded into swizzled
// shared memory (a 16-byte vector per chunk when K is contiguous and aligned, else 8
// element loads that are coalesced across the block's rows) and multiplied as four K=16
// MMAs into a 128 x 128 fp32 tensor-memory accumulator.  With several K ranges (the weight
// gradients, K = batch rows) each block adds its partial product with fp32 atomics into a
// zeroed C.  The shared-memory request caps residency at 3 blocks (384 tensor-memory
// columns) per SM.
constexpr uint32_t kGemmSmem = 72 * 1024;
constexpr int kGemmK = 64;

__device__ __forceinline__ void load_chunk(const __half* __restrict__ p, long stride_k, int valid, bool vec,
                                           uint32_t q[4]) {
    if (vec && valid == 8) {
        const uint4 v = *reinterpret_cast<const uint4*>(p);
        q[0] = v.x, q[1] = v.y, q[2] = v.z, q[3] = v.w;
        return;
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const __half a = 2 * e < valid ? p[(long)(2 * e) * stride_k] : __float2half(0.0f);
        const __half b = 2 * e + 1 < valid ? p[(long)(2 * e + 1) * stride_k] : __float2half(0.0f);
        __half2 h = __halves2half2(a, b);
        q[e] = *reinterpret_cast<const uint32_t*>(&h);
    }
}

__global__ void __launch_bounds__(128) gemm_tc(const __half* __restrict__ A, long sai, long sak, bool a_vec,
                                               const __half* __restrict__ B, long sbk, long sbj, bool b_vec,
                                               float* __restrict__ C, long ldc, int M, int N, int K, int k_per_block,
                                               float alpha, bool atomic, unsigned* __restrict__ err) {
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    const uint32_t as = base, bs = base + kAtomBytes, bar = base + 2 * kAtomBytes, tmem_slot = bar + 8;
    const uint32_t t = threadIdx.x, warp = t >> 5;
    const int m0 = blockIdx.x * kTileRows;
    const int kb = blockIdx.y * k_per_block, ke = min(K, kb + k_per_block);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tmem_slot),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    uint32_t tmem = 0;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(tmem) : "r"(tmem_slot) : "memory");
    uint32_t phase = 0;
    bool failed = false, undrained = false;
    const int i = m0 + (int)t;  // this thread's row of A and of C
    const int j = (int)t;       // this thread's row of B (column of C)
    for (int k0 = kb; k0 < ke && !failed; k0 += kGemmK) {
#pragma unroll
        for (uint32_t c = 0; c < kGemmK / 8; ++c) {
            const int k = k0 + (int)c * 8;
            const int valid = max(0, min(8, ke - k));
            uint32_t q[4] = {0u, 0u, 0u, 0u};
            if (i < M) load_chunk(A + (long)i * sai + (long)k * sak, sak, valid, a_vec, q);
            asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(as + sw128_chunk(t, c)), "r"(q[0]),
                         "r"(q[1]), "r"(q[2]), "r"(q[3])
                         : "memory");
            q[0] = q[1] = q[2] = q[3] = 0u;
            if (j < N) load_chunk(B + (long)k * sbk + (long)j * sbj, sbk, valid, b_vec, q);
            asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(bs + sw128_chunk(t, c)), "r"(q[0]),
                         "r"(q[1]), "r"(q[2]), "r"(q[3])
                         : "memory");
        }
        proxy_fence();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
#pragma unroll
            for (int ks = 0; ks < 4; ++ks)
                umma_f16(tmem, sw128_desc(as + ks * 32u), sw128_desc(bs + ks * 32u), (k0 > kb || ks > 0) ? 1u : 0u);
            umma_commit(bar);
        }
        const bool ok = mbar_wait(bar, phase);
        if (__syncthreads_or(!ok)) {  // timed out: drain the MMAs in flight (bounded), then leave
            undrained = !__syncthreads_and(mbar_wait(bar, phase));
            failed = true;
            break;
        }
        phase ^= 1u;  // the shared tiles are free again once the MMAs are done
    }
    if (!failed && kb < ke) {
        // Epilogue: 32 accumulator columns at a time go through shared memory (the operand
        // tiles are free now), [128 rows][33 floats], so that a warp then writes 32
        // consecutive floats of one row of C per store.
        tc_fence_after();
        const uint32_t my_lanes = tmem + ((warp * 32u) << 16);
        float* stage = reinterpret_cast<float*>(smem_raw + (base - raw));
        constexpr int kLd = 33;  // padded row: column reads of the staging tile avoid bank conflicts
        for (int c0 = 0; c0 < 128; c0 += 32) {
            float v[32];
            tmem_ld16(my_lanes + (uint32_t)c0, v);
            tmem_ld16(my_lanes + (uint32_t)c0 + 16u, v + 16);
#pragma unroll
            for (int e = 0; e < 32; ++e) stage[t * kLd + e] = v[e];
            __syncthreads();
            const int lane = (int)(t & 31u), col = c0 + lane;
            for (int r = (int)warp; r < kTileRows; r += 4) {
                const int row = m0 + r;
                if (row < M && col < N) {
                    float* p = C + (long)row * ldc + col;
                    const float x = alpha * stage[r * kLd + lane];
                    if (atomic) atomicAdd(p, x);
                    else *p = x;
                }
            }
            __syncthreads();
        }
    }
    // bit 0: a completion wait timed out; bit 1: the drain timed out too, so products may still
    // have been in flight when the tensor memory was freed
    if (failed && t == 0) atomicOr(err, undrained ? 3u : 1u);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

// C = alpha * A x B (the only form training uses; beta must be 0).  `err`: device word the
// kernel sets when an MMA completion wait times out.
int gemm(const __half* A, long sai, long sak, const __half* B, long sbk, long sbj, float* C, long ldc, int M, int N,
         int K, float alpha, float beta, unsigned* err, cudaStream_t s) {
    if (M <= 0 || N <= 0 || K <= 0) return NQB_OK;
    if (beta != 0.0f || N > 128) return NQB_E_INVALID;
    NQB_TRY(cuda_status(cudaFuncSetAttribute(gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem)));
    auto vec_ok = [](const __half* p, long s_row, long s_k) {
        return s_k == 1 && ((uintptr_t)p & 15u) == 0 && (s_row * (long)sizeof(__half)) % 16 == 0;
    };
    const bool a_vec = vec_ok(A, sai, sak), b_vec = vec_ok(B, sbj, sbk);
    const int m_tiles = (M + kTileRows - 1) / kTileRows;
    // split K when it is long (the weight gradients): at least 256 K per block
    int splits = 1;
    if (K > 256) splits = std::min((K + 255) / 256, std::max(1, 148 * 3 / m_tiles));
    const int per = ((K + splits - 1) / splits + kGemmK - 1) / kGemmK * kGemmK;
    splits = (K + per - 1) / per;
    if (splits > 1)  // partial products are added into a zeroed C
        NQB_TRY(cuda_status(
            cudaMemset2DAsync(C, (size_t)ldc * sizeof(float), 0, (size_t)N * sizeof(float), (size_t)M, s)));
    const dim3 grid(m_tiles, splits);
    gemm_tc<<<grid, kTileRows, kGemmSmem, s>>>(A, sai, sak, a_vec, B, sbk, sbj, b_vec, C, ldc, M, N, K, per, alpha,
                                              splits > 1, err);
    return cuda_status(cudaGetLastError());
}

// ---- elementwise and reduction kernels -------------------------------------------------
__global__ void features_kernel(const uint4* __restrict__ st, const uint32_t* __restrict__ rows, uint32_t n_rows,
                                __half* __restrict__ X) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)n_rows * kIn) return;
    const uint32_t i = (uint32_t)(e / kIn), j = (uint32_t)(e % kIn);
    const uint4 s = st[rows ? rows[i] : i];
    X[e] = __float2half(feature(s, (int)j));
}

// H = gelu(Z + b) (fp16), Zb = Z + b kept for the backward pass.
__global__ void bias_gelu_kernel(const float* __restrict__ Z, const float* __restrict__ b, uint32_t rows,
                                 float* __restrict__ Zb, __half* __restrict__ H) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)rows * kH) return;
    const float z = Z[e] + b[e % kH];
    Zb[e] = z;
    H[e] = __float2half(gelu(z));
}

// y_i = H2_i . w3 + b3 (one warp per row).
__global__ void head_kernel(const __half* __restrict__ H2, const float* __restrict__ w3, const float* __restrict__ b3,
                            uint32_t rows, float* __restrict__ y) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= rows) return;
    float s = 0.0f;
    for (int j = lane; j < kH; j += 32) s += __half2float(H2[(uint64_t)row * kH + j]) * w3[j];
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if (lane == 0) y[row] = s + b3[0];
}

// dy = 2 (y - t); the squared error is summed into loss[0].
__global__ void loss_kernel(const float* __restrict__ y, const float* __restrict__ t, uint32_t rows,
                            float* __restrict__ dy, float* __restrict__ loss) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float e2 = 0.0f;
    if (i < rows) {
        const float d = y[i] - t[i];
        dy[i] = 2.0f * d;
        e2 = d * d;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) e2 += __shfl_xor_sync(0xFFFFFFFFu, e2, o);
    if ((threadIdx.x & 31) == 0 && e2 != 0.0f) atomicAdd(loss, e2);
}

// dZ2 = dy_i * w3_j * gelu'(Zb2_ij), fp16.
__global__ void dz2_kernel(const float* __restrict__ dy, const float* __restrict__ w3, const float* __restrict__ Zb2,
                           uint32_t rows, __half* __restrict__ dZ2) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)rows * kH) return;
    dZ2[e] = __float2half(dy[e / kH] * w3[e % kH] * gelu_grad(Zb2[e]));
}

// dZ1 = dH1 * gelu'(Zb1), fp16.
__global__ void dz1_kernel(const float* __restrict__ dH1, const float* __restrict__ Zb1, uint32_t rows,
                           __half* __restrict__ dZ1) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)rows * kH) return;
    dZ1[e] = __float2half(dH1[e] * gelu_grad(Zb1[e]));
}

// out[j] = scale * sum_i D[i][j] (D fp16 rows x 128); with dy != null: scale * sum_i dy_i D[i][j].
__global__ void colsum_kernel(const __half* __restrict__ D, const float* __restrict__ dy, uint32_t rows, float scale,
                              float* __restrict__ out) {
    const int j = threadIdx.x;  // blockDim = 128
    float s = 0.0f;
    for (uint32_t i = blockIdx.x; i < rows; i += gridDim.x) {
        const float v = __half2float(D[(uint64_t)i * kH + j]);
        s += dy ? v * dy[i] : v;
    }
    atomicAdd(out + j, s * scale);
}

__global__ void sum_kernel(const float* __restrict__ v, uint32_t n, float scale, float* __restrict__ out) {
    float s = 0.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += v[i];
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s * scale);
}

__global__ void gather_f16_rows(const __half* __restrict__ X, const uint32_t* __restrict__ rows, uint32_t n_rows,
                                __half* __restrict__ out) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)n_rows * kIn) return;
    out[e] = X[(uint64_t)rows[e / kIn] * kIn + e % kIn];
}

__global__ void gather_f32(const float* __restrict__ v, const uint32_t* __restrict__ rows, uint32_t n,
                           float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = v[rows[i]];
}

// Adam (Kingma & Ba 2015) on the flat fp32 parameters; refreshes the fp16 copies of W1, W2.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ grad, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2,
                            __half* __restrict__ w1h, __half* __restrict__ w2h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = grad[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float w = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = w;
    if (i < kW1Size) w1h[i] = __float2half(w);
    else if (i >= kW2 && i < kB2) w2h[i - kW2] = __float2half(w);
}

__global__ void to_half_kernel(const float* __restrict__ p, __half* __restrict__ w1h, __half* __restrict__ w2h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kW1Size) w1h[i] = __float2half(p[kW1 + i]);
    if (i < kH * kH) w2h[i] = __float2half(p[kW2 + i]);
}

// ---- fused inference on the 5th-generation tensor cores (tcgen05) ----------------------
// One CTA of 4 warps runs 128-row tiles: features -> layer 1 -> GELU -> layer 2 -> GELU ->
// head.  Both layers are M=128, N=128, K=128 products (the 112 inputs zero-padded) issued as
// eight K=16 tcgen05.mma by one thread, with FP16 operands in shared memory and the FP32
// accumulator in tensor memory (128 lanes x 128 columns).  Thread t owns tile row t: it
// builds that row's features, and after each layer reads the row's 128 accumulators with
// tcgen05.ld (warp w may read lanes 32w..32w+31), so GELU and the head's dot product need
// no shuffles.  Operand tiles use the 128-byte-swizzled K-major layout: 16-byte chunk j of
// row r of a 128-row tile sits at (j / 8) x 16 KB + r x 128 + ((j % 8) ^ (r % 8)) x 16.
// Every wait on the MMA completion barrier is bounded; on a timeout the block sets the
// error word and leaves, freeing its tensor memory on the way out.
// Writes W (math layout [in][out], fp16, `in_rows` real inputs) as the B operand: tile row n
// = output n, K = input, zero beyond in_rows.  Thread t writes row t.
__device__ __forceinline__ void stage_weights(uint32_t tile, const __half* __restrict__ w, int in_rows, uint32_t t) {
    for (uint32_t j = 0; j < 16; ++j) {
        uint32_t q[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int k0 = (int)j * 8 + 2 * e;
            const float a = k0 < in_rows ? __half2float(w[(size_t)k0 * kH + t]) : 0.0f;
            const float b = k0 + 1 < in_rows ? __half2float(w[(size_t)(k0 + 1) * kH + t]) : 0.0f;
            q[e] = pack_half2(a, b);
        }
        asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(tile + sw128_chunk(t, j)), "r"(q[0]), "r"(q[1]),
                     "r"(q[2]), "r"(q[3])
                     : "memory");
    }
}

__global__ void __launch_bounds__(128) predict_kernel(const uint4* __restrict__ st, uint32_t count,
                                                      const __half* __restrict__ w1h, const __half* __restrict__ w2h,
                                                      const float* __restrict__ params, float* __restrict__ out,
                                                      uint32_t wait_limit, unsigned* __restrict__ err) {
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;  // swizzle atoms need 1024-byte alignment
    const uint32_t w1s = base, w2s = base + kOpBytes, xs = base + 2 * kOpBytes;
    float* vec = reinterpret_cast<float*>(smem_raw + (base - raw) + 3 * kOpBytes);  // b1 | b2 | w3 | b3
    const uint32_t bar = base + 3 * kOpBytes + (3 * kH + 4) * sizeof(float);
    const uint32_t tmem_slot = bar + 8;
    const uint32_t t = threadIdx.x, warp = t >> 5;

    stage_weights(w1s, w1h, kIn, t);
    stage_weights(w2s, w2h, kH, t);
    for (uint32_t e = t; e < (uint32_t)kH; e += blockDim.x) {
        vec[e] = params[kB1 + e];
        vec[kH + e] = params[kB2 + e];
        vec[2 * kH + e] = params[kW3 + e];
    }
    if (t == 0) {
        vec[3 * kH] = params[kB3];
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tmem_slot),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    uint32_t tmem = 0;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(tmem) : "r"(tmem_slot) : "memory");
    const uint32_t my_lanes = tmem + ((warp * 32u) << 16);
    uint32_t phase = 0;
    bool failed = false, undrained = false;

    for (uint32_t tile = blockIdx.x; (uint64_t)tile * kTileRows < count && !failed; tile += gridDim.x) {
        const uint64_t i = (uint64_t)tile * kTileRows + t;
        const uint4 s = i < count ? st[i] : make_uint4(0, 0, 0, 0);
        for (uint32_t j = 0; j < 16; ++j) {  // the row's 128 features (zero for rows past the end)
            uint32_t q[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int k0 = (int)j * 8 + 2 * e;
                q[e] = i < count ? pack_half2(feature(s, k0), feature(s, k0 + 1)) : 0u;
            }
            asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(xs + sw128_chunk(t, j)), "r"(q[0]),
                         "r"(q[1]), "r"(q[2]), "r"(q[3])
                         : "memory");
        }
        float sum = 0.0f;
        for (int layer = 0; layer < 2 && !failed; ++layer) {
            proxy_fence();  // make the operand tile visible to the tensor cores
            tc_fence_before();
            __syncthreads();
            if (t == 0) {
                tc_fence_after();
                const uint32_t wt = layer == 0 ? w1s : w2s;
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    umma_f16(tmem, sw128_desc(xs + kstep_offset(k)), sw128_desc(wt + kstep_offset(k)), k > 0 ? 1u : 0u);
                umma_commit(bar);
            }
            const bool ok = wait_limit ? mbar_wait(bar, phase, wait_limit, true) : mbar_wait(bar, phase);
            if (__syncthreads_or(!ok)) {  // timed out: drain the MMAs in flight (bounded), then leave
                undrained = !__syncthreads_and(mbar_wait(bar, phase));
                failed = true;
                break;
            }
            phase ^= 1u;
            tc_fence_after();
            const float* bias = vec + layer * kH;
            for (uint32_t c = 0; c < (uint32_t)kH; c += 16) {
                float v[16];
                tmem_ld16(my_lanes + c, v);
                if (layer == 0) {  // H1 = gelu(Z1 + b1), fp16, becomes the A operand of layer 2
                    uint32_t q[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        q[e] = pack_half2(gelu(v[2 * e] + bias[c + 2 * e]), gelu(v[2 * e + 1] + bias[c + 2 * e + 1]));
                    asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(xs + sw128_chunk(t, c / 8)),
                                 "r"(q[0]), "r"(q[1]), "r"(q[2]), "r"(q[3])
                                 : "memory");
                    asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(xs + sw128_chunk(t, c / 8 + 1)),
                                 "r"(q[4]), "r"(q[5]), "r"(q[6]), "r"(q[7])
                                 : "memory");
                } else {  // head: H2 rounded to fp16 as in the training forward pass
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        sum += __half2float(__float2half(gelu(v[e] + bias[c + e]))) * vec[2 * kH + c + e];
                }
            }
            tc_fence_before();
        }
        if (!failed && i < count) out[i] = sum + vec[3 * kH];
        __syncthreads();  // the operand tile and the accumulator are free for the next tile
    }
    // bit 0: a completion wait timed out; bit 1: the drain timed out too, so products may still
    // have been in flight when the tensor memory was freed
    if (failed && t == 0) atomicOr(err, undrained ? 3u : 1u);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

// Device buffers of one training or gradient pass over batches of up to `cap` rows.
struct Work {
    __half *X = nullptr, *H1 = nullptr, *H2 = nullptr, *dZ2 = nullptr, *dZ1 = nullptr;
    float *t = nullptr, *Z = nullptr, *Zb1 = nullptr, *Zb2 = nullptr, *y = nullptr, *dy = nullptr, *dH1 = nullptr,
          *loss = nullptr;
    unsigned* err = nullptr;  // set by a GEMM whose tensor-core completion wait timed out
    uint32_t cap = 0;
    std::vector<void*> owned;

    int init(uint32_t rows) {
        cap = rows;
        const size_t r = rows;
        owned.reserve(16);  // may throw, but before anything is allocated; push_back then does not
        auto get = [&](auto** p, size_t bytes) {
            void* v = nullptr;
            const int s = cuda_malloc(&v, bytes);
            if (s == NQB_OK) {
                owned.push_back(v);
                *p = static_cast<std::remove_pointer_t<decltype(p)>>(v);
            }
            return s;
        };
        int s = NQB_OK;
        if (!s) s = get(&X, r * kIn * sizeof(__half));
        if (!s) s = get(&H1, r * kH * sizeof(__half));
        if (!s) s = get(&H2, r * kH * sizeof(__half));
        if (!s) s = get(&dZ2, r * kH * sizeof(__half));
        if (!s) s = get(&dZ1, r * kH * sizeof(__half));
        if (!s) s = get(&t, r * sizeof(float));
        if (!s) s = get(&Z, r * kH * sizeof(float));
        if (!s) s = get(&Zb1, r * kH * sizeof(float));
        if (!s) s = get(&Zb2, r * kH * sizeof(float));
        if (!s) s = get(&y, r * sizeof(float));
        if (!s) s = get(&dy, r * sizeof(float));
        if (!s) s = get(&dH1, r * kH * sizeof(float));
        if (!s) s = get(&loss, sizeof(float));
        if (!s) s = get(&err, sizeof(unsigned));
        if (!s) s = cuda_status(cudaMemset(err, 0, sizeof(unsigned)));
        return s;
    }
    // NQB_E_STALL if a GEMM of the passes so far timed out (synchronises the stream).
    int check(cudaStream_t s) const {
        unsigned h = 0;
        int st = cuda_status(cudaMemcpyAsync(&h, err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        if (!st) st = cuda_status(cudaStreamSynchronize(s));
        return st ? st : (h & 2u) ? NQB_E_DEVICE : (h ? NQB_E_STALL : NQB_OK);
    }
    ~Work() {
        for (void* p : owned) cudaFree(p);
    }
};

unsigned blocks_for(uint64_t n, unsigned per = 256) { return (unsigned)((n + per - 1) / per); }

}  // namespace
}  // namespace mlp
}  // namespace nqb

// ---- the model object ---------------------------------------------------------------------
struct nqb_model {
    int device = 0;
    float* params = nullptr;  // fp32 master weights (kParams)
    float* grad = nullptr;
    float* m = nullptr;  // Adam moments
    float* v = nullptr;
    __half* w1h = nullptr;  // fp16 copies fed to the tensor cores
    __half* w2h = nullptr;
    long adam_step = 0;
};

namespace nqb {
namespace mlp {
namespace {

// Forward and backward over `rows` rows already in w.X / w.t; accumulates the mean
// squared error into w.loss and writes the mean gradient into m->grad.
int pass(nqb_model* m, Work& w, uint32_t rows, cudaStream_t s) {
    const float* P = m->params;
    float* G = m->grad;
    int st;
    cudaMemsetAsync(G, 0, kParams * sizeof(float), s);
    // forward
    if ((st = gemm(w.X, kIn, 1, m->w1h, kH, 1, w.Z, kH, rows, kH, kIn, 1.0f, 0.0f, w.err, s))) return st;
    bias_gelu_kernel<<<blocks_for((uint64_t)rows * kH), 256, 0, s>>>(w.Z, P + kB1, rows, w.Zb1, w.H1);
    if ((st = gemm(w.H1, kH, 1, m->w2h, kH, 1, w.Z, kH, rows, kH, kH, 1.0f, 0.0f, w.err, s))) return st;
    bias_gelu_kernel<<<blocks_for((uint64_t)rows * kH), 256, 0, s>>>(w.Z, P + kB2, rows, w.Zb2, w.H2);
    head_kernel<<<blocks_for((uint64_t)rows * 32), 256, 0, s>>>(w.H2, P + kW3, P + kB3, rows, w.y);
    loss_kernel<<<blocks_for(rows), 256, 0, s>>>(w.y, w.t, rows, w.dy, w.loss);
    // backward (mean over the rows)
    const float inv = 1.0f / (float)rows;
    colsum_kernel<<<std::min<unsigned>(rows, 512), kH, 0, s>>>(w.H2, w.dy, rows, inv, G + kW3);  // dw3
    sum_kernel<<<std::min<unsigned>(blocks_for(rows), 256), 256, 0, s>>>(w.dy, rows, inv, G + kB3);
    dz2_kernel<<<blocks_for((uint64_t)rows * kH), 256, 0, s>>>(w.dy, P + kW3, w.Zb2, rows, w.dZ2);
    colsum_kernel<<<std::min<unsigned>(rows, 512), kH, 0, s>>>(w.dZ2, nullptr, rows, inv, G + kB2);
    // dW2 = H1^T dZ2: A(i, k) = H1[k][i], B(k, j) = dZ2[k][j]
    if ((st = gemm(w.H1, 1, kH, w.dZ2, kH, 1, G + kW2, kH, kH, kH, rows, inv, 0.0f, w.err, s))) return st;
    // dH1 = dZ2 W2^T: B(k, j) = W2[j][k]
    if ((st = gemm(w.dZ2, kH, 1, m->w2h, 1, kH, w.dH1, kH, rows, kH, kH, 1.0f, 0.0f, w.err, s))) return st;
    dz1_kernel<<<blocks_for((uint64_t)rows * kH), 256, 0, s>>>(w.dH1, w.Zb1, rows, w.dZ1);
    colsum_kernel<<<std::min<unsigned>(rows, 512), kH, 0, s>>>(w.dZ1, nullptr, rows, inv, G + kB1);
    // dW1 = X^T dZ1
    if ((st = gemm(w.X, 1, kIn, w.dZ1, kH, 1, G + kW1, kH, kIn, kH, rows, inv, 0.0f, w.err, s))) return st;
    return cuda_status(cudaGetLastError());
}

// Seeded uniform initialisation: W ~ U(-sqrt(6/(fan_in+fan_out)), +) (Glorot), biases 0,
// b3 = the mean target so the first steps start near the data.
void init_params(std::vector<float>& p, uint64_t seed) {
    p.assign(kParams, 0.0f);
    uint64_t st = seed ? seed : 0x9E3779B97F4A7C15ull;
    auto next = [&]() {
        uint64_t z = (st += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int n, int fin, int fout) {
        const double a = std::sqrt(6.0 / (fin + fout));
        for (int i = 0; i < n; ++i) p[off + i] = (float)((2.0 * next() - 1.0) * a);
    };
    fill(kW1, kIn * kH, 100, kH);  // 100 live inputs of the 112
    fill(kW2, kH * kH, kH, kH);
    fill(kW3, kH, kH, 1);
}

}  // namespace
}  // namespace mlp
}  // namespace nqb

using namespace nqb;
using namespace nqb::mlp;

namespace {

struct CallScope {  // current device for the call, restored afterwards; one stream
    int prev = 0;
    cudaStream_t s = nullptr;
    int status = NQB_OK;
    explicit CallScope(int dev) {
        cudaGetDevice(&prev);
        if ((status = cuda_status(cudaSetDevice(dev)))) return;
        status = cuda_status(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    }
    ~CallScope() {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
        cudaSetDevice(prev);
    }
};

template <class T>
struct DevBuf {
    T* p = nullptr;
    int alloc(size_t n) { return cuda_malloc(&p, (n ? n : 1) * sizeof(T)); }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

int refresh_half(nqb_model* m, cudaStream_t s) {
    to_half_kernel<<<blocks_for(kH * kH), 256, 0, s>>>(m->params, m->w1h, m->w2h);
    return cuda_status(cudaGetLastError());
}

}  // namespace

extern "C" {

int nqb_model_create(int device, uint64_t seed, nqb_model** out) try {
    if (!out) return NQB_E_INVALID;
    *out = nullptr;
    int st = nqb_device_check(device);
    if (st) return st;
    CallScope cs(device);
    if (cs.status) return cs.status;
    std::vector<float> p;  // before the model object: nothing to release if this throws
    init_params(p, seed);
    nqb_model* m = new nqb_model();
    m->device = device;
    st = cuda_malloc(&m->params, kParams * sizeof(float));
    if (!st) st = cuda_malloc(&m->grad, kParams * sizeof(float));
    if (!st) st = cuda_malloc(&m->m, kParams * sizeof(float));
    if (!st) st = cuda_malloc(&m->v, kParams * sizeof(float));
    if (!st) st = cuda_malloc(&m->w1h, kW1Size * sizeof(__half));
    if (!st) st = cuda_malloc(&m->w2h, kH * kH * sizeof(__half));
    if (!st) st = cuda_status(cudaMemcpyAsync(m->params, p.data(), kParams * sizeof(float), cudaMemcpyHostToDevice, cs.s));
    if (!st) st = cuda_status(cudaMemsetAsync(m->m, 0, kParams * sizeof(float), cs.s));
    if (!st) st = cuda_status(cudaMemsetAsync(m->v, 0, kParams * sizeof(float), cs.s));
    if (!st) st = refresh_half(m, cs.s);
    if (!st) st = cuda_status(cudaStreamSynchronize(cs.s));
    if (st) {
        nqb_model_destroy(m);
        return st;
    }
    *out = m;
    return NQB_OK;
} NQB_ABI_CATCH

void nqb_model_destroy(nqb_model* m) {
    if (!m) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(m->device);
    cudaFree(m->params);
    cudaFree(m->grad);
    cudaFree(m->m);
    cudaFree(m->v);
    cudaFree(m->w1h);
    cudaFree(m->w2h);
    cudaSetDevice(prev);
    delete m;
}

int nqb_model_get_params(const nqb_model* m, float* out) {
    if (!m || !out) return NQB_E_INVALID;
    CallScope cs(m->device);
    if (cs.status) return cs.status;
    int st = cuda_status(cudaMemcpyAsync(out, m->params, kParams * sizeof(float), cudaMemcpyDeviceToHost, cs.s));
    if (!st) st = cuda_status(cudaStreamSynchronize(cs.s));
    return st;
}

int nqb_model_set_params(nqb_model* m, const float* in) {
    if (!m || !in) return NQB_E_INVALID;
    CallScope cs(m->device);
    if (cs.status) return cs.status;
    int st = cuda_status(cudaMemcpyAsync(m->params, in, kParams * sizeof(float), cudaMemcpyHostToDevice, cs.s));
    if (!st) st = cuda_status(cudaMemsetAsync(m->m, 0, kParams * sizeof(float), cs.s));
    if (!st) st = cuda_status(cudaMemsetAsync(m->v, 0, kParams * sizeof(float), cs.s));
    if (!st) st = refresh_half(m, cs.s);
    if (!st) st = cuda_status(cudaStreamSynchronize(cs.s));
    m->adam_step = 0;
    return st;
}

int nqb_model_features(const nqb_state* states, uint64_t count, float* out) try {
    if (count && (!states || !out)) return NQB_E_INVALID;
    for (uint64_t i = 0; i < count; ++i) {
        uint4 st;
        std::memcpy(&st, &states[i], sizeof(st));
        for (int j = 0; j < kIn; ++j) out[i * kIn + j] = feature(st, j);
    }
    return NQB_OK;
} NQB_ABI_CATCH

int nqb_model_predict(const nqb_model* m, const nqb_state* states, uint64_t count, float* out) try {
    return nqb_model_predict_ex(m, states, count, out, 0);
} NQB_ABI_CATCH

int nqb_model_predict_ex(const nqb_model* m, const nqb_state* states, uint64_t count, float* out,
                         uint32_t wait_limit) try {
    if (!m || (count && (!states || !out))) return NQB_E_INVALID;
    if (count == 0) return NQB_OK;
    if (count > 0xFFFFFFFFull) return NQB_E_RANGE;
    CallScope cs(m->device);
    if (cs.status) return cs.status;
    DevBuf<nqb_state> d_st;
    DevBuf<float> d_out;
    int st = d_st.alloc(count);
    if (!st) st = d_out.alloc(count);
    if (!st) st = cuda_status(cudaMemcpyAsync(d_st.p, states, count * sizeof(nqb_state), cudaMemcpyHostToDevice, cs.s));
    if (!st) st = nqb::model_predict_device(m, d_st.p, (uint32_t)count, d_out.p, cs.s, wait_limit);
    if (!st) st = cuda_status(cudaMemcpyAsync(out, d_out.p, count * sizeof(float), cudaMemcpyDeviceToHost, cs.s));
    if (!st) st = cuda_status(cudaStreamSynchronize(cs.s));
    return st;
} NQB_ABI_CATCH

int nqb_model_loss_grad(nqb_model* m, const nqb_state* states, const float* targets, uint64_t count, float* loss,
                        float* grad) try {
    if (!m || !states || !targets || !loss || !grad || count == 0) return NQB_E_INVALID;
    if (count > (1u << 20)) return NQB_E_RANGE;
    CallScope cs(m->device);
    if (cs.status) return cs.status;
    Work w;
    DevBuf<nqb_state> d_st;
    int st = w.init((uint32_t)count);
    if (!st) st = d_st.alloc(count);
    if (!st) st = cuda_status(cudaMemcpyAsync(d_st.p, states, count * sizeof(nqb_state), cudaMemcpyHostToDevice, cs.s));
    if (!st) st = cuda_status(cudaMemcpyAsync(w.t, targets, count * sizeof(float), cudaMemcpyHostToDevice, cs.s));
    if (st) return st;
    features_kernel<<<blocks_for(count * kIn), 256, 0, cs.s>>>(reinterpret_cast<const uint4*>(d_st.p), nullptr,
                                                                 (uint32_t)count, w.X);
    cudaMemsetAsync(w.loss, 0, sizeof(float), cs.s);
    if ((st = pass(m, w, (uint32_t)count, cs.s))) return st;
    float l = 0;
    st = cuda_status(cudaMemcpyAsync(&l, w.loss, sizeof(float), cudaMemcpyDeviceToHost, cs.s));
    if (!st) st = cuda_status(cudaMemcpyAsync(grad, m->grad, kParams * sizeof(float), cudaMemcpyDeviceToHost, cs.s));
    if (!st) st = w.check(cs.s);
    *loss = l / (float)count;
    return st;
} NQB_ABI_CATCH

int nqb_model_train(nqb_model* m, const nqb_state* states, const float* targets, uint64_t count,
                    const nqb_train_opts* opts, float* epoch_loss) try {
    if (!m || !states || !targets || count == 0) return NQB_E_INVALID;
    if (count > 0xFFFFFFFFull) return NQB_E_RANGE;
    nqb_train_opts o;
    std::memset(&o, 0, sizeof(o));
    o.epochs = 8;
    o.batch = 4096;
    o.lr = 1e-3f;
    o.seed = 1;
    if (opts) o = *opts;
    if (o.epochs <= 0 || o.batch <= 0 || o.batch > (1 << 20) || !(o.lr > 0.0f)) return NQB_E_INVALID;
    CallScope cs(m->device);
    if (cs.status) return cs.status;
    const uint32_t B = (uint32_t)std::min<uint64_t>(o.batch, count);
    Work w;
    DevBuf<nqb_state> d_st;
    DevBuf<__half> d_X;
    DevBuf<float> d_t;
    DevBuf<uint32_t> d_perm;
    int st = w.init(B);
    if (!st) st = d_st.alloc(count);
    if (!st) st = d_X.alloc(count * kIn);
    if (!st) st = d_t.alloc(count);
    if (!st) st = d_perm.alloc(count);
    if (!st) st = cuda_status(cudaMemcpyAsync(d_st.p, states, count * sizeof(nqb_state), cudaMemcpyHostToDevice, cs.s));
    if (!st) st = cuda_status(cudaMemcpyAsync(d_t.p, targets, count * sizeof(float), cudaMemcpyHostToDevice, cs.s));
    if (st) return st;
    features_kernel<<<blocks_for(count * kIn), 256, 0, cs.s>>>(reinterpret_cast<const uint4*>(d_st.p), nullptr,
                                                                 (uint32_t)count, d_X.p);
    std::vector<uint32_t> perm(count);
    for (uint64_t i = 0; i < count; ++i) perm[i] = (uint32_t)i;
    uint64_t rng = o.seed * 0x9E3779B97F4A7C15ull + 1;
    auto next = [&]() {
        uint64_t z = (rng += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < o.epochs; ++ep) {
        for (uint64_t i = count - 1; i > 0; --i) std::swap(perm[i], perm[next() % (i + 1)]);  // Fisher-Yates
        st = cuda_status(cudaMemcpyAsync(d_perm.p, perm.data(), count * sizeof(uint32_t), cudaMemcpyHostToDevice, cs.s));
        if (st) return st;
        cudaMemsetAsync(w.loss, 0, sizeof(float), cs.s);
        for (uint64_t off = 0; off < count; off += B) {
            const uint32_t rows = (uint32_t)std::min<uint64_t>(B, count - off);
            gather_f16_rows<<<blocks_for((uint64_t)rows * kIn), 256, 0, cs.s>>>(d_X.p, d_perm.p + off, rows, w.X);
            gather_f32<<<blocks_for(rows), 256, 0, cs.s>>>(d_t.p, d_perm.p + off, rows, w.t);
            if ((st = pass(m, w, rows, cs.s))) return st;
            m->adam_step++;
            const float c1 = 1.0f - std::pow(b1, (float)m->adam_step), c2 = 1.0f - std::pow(b2, (float)m->adam_step);
            adam_kernel<<<blocks_for(kParams), 256, 0, cs.s>>>(m->params, m->grad, m->m, m->v, kParams, o.lr, b1, b2,
                                                                eps, c1, c2, m->w1h, m->w2h);
        }
        float l = 0;
        st = cuda_status(cudaMemcpyAsync(&l, w.loss, sizeof(float), cudaMemcpyDeviceToHost, cs.s));
        if (!st) st = w.check(cs.s);
        if (st) return st;
        if (epoch_loss) epoch_loss[ep] = l / (float)count;
    }
    return cuda_status(cudaStreamSynchronize(cs.s));
} NQB_ABI_CATCH

}  // extern "C"

namespace nqb {

int model_predict_device(const nqb_model* m, const nqb_state* d_states, uint32_t count, float* d_out, cudaStream_t s,
                         uint32_t wait_limit) {
    if (count == 0) return NQB_OK;  // wait_limit 0: the default (suspending) bounded wait
    cudaError_t e = cudaFuncSetAttribute(predict_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPredictSmem);
    if (e != cudaSuccess) return cuda_status(e);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device);
    const uint64_t tiles = (count + kTileRows - 1) / kTileRows;
    // at most 2 blocks per SM (shared memory), so their tensor memory (2 x 128 columns) fits
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(tiles, (uint64_t)sms * 2));
    unsigned* d_err = nullptr;
    NQB_TRY(dev_alloc(&d_err, sizeof(unsigned), s));
    unsigned h_err = 0;
    int st = cuda_status(cudaMemsetAsync(d_err, 0, sizeof(unsigned), s));
    if (!st) {
        predict_kernel<<<grid, kTileRows, kPredictSmem, s>>>(reinterpret_cast<const uint4*>(d_states), count, m->w1h,
                                                             m->w2h, m->params, d_out, wait_limit, d_err);
        st = cuda_status(cudaGetLastError());
    }
    if (!st) st = cuda_status(cudaMemcpyAsync(&h_err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    if (!st) st = cuda_status(cudaStreamSynchronize(s));
    dev_free(d_err, s);
    if (!st && h_err) st = (h_err & 2u) ? NQB_E_DEVICE : NQB_E_STALL;
    return st;
}

int model_device(const nqb_model* m) { return m->device; }

}  // namespace nqb
