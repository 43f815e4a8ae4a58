// Learned cost model: shapes, the feature encoding and the activation shared by the training
// kernels (mlp.cu), the fused inference kernel and the host.  Device and host.
#pragma once

#include <cstdint>

#include <cuda_fp16.h>

namespace nqb {
namespace mlp {

// Network 112 -> 128 -> 128 -> 1, GELU after both hidden layers.
constexpr int kIn = 112;  // 3 x 32 mask bits + 4 scalars, zero-padded to a multiple of 16
constexpr int kH = 128;
constexpr int kW1Size = kIn * kH;
constexpr int kW1 = 0;  // offsets of the parameters in the flat fp32 vector
constexpr int kB1 = kW1 + kW1Size;
constexpr int kW2 = kB1 + kH;
constexpr int kB2 = kW2 + kH * kH;
constexpr int kW3 = kB2 + kH;
constexpr int kB3 = kW3 + kH;
constexpr int kParams = kB3 + 1;

// GELU, tanh form (Hendrycks & Gimpel 2016): 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).
constexpr float kGeluC = 0.7978845608028654f;
constexpr float kGeluA = 0.044715f;

__device__ __forceinline__ float gelu(float x) {
    return 0.5f * x * (1.0f + tanhf(kGeluC * (x + kGeluA * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float th = tanhf(kGeluC * (x + kGeluA * x * x * x));
    return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * kGeluC * (1.0f + 3.0f * kGeluA * x * x);
}

// Feature j of a state {cols, ldiag, rdiag, meta}: bits 0..31 of the free-column mask,
// bits 0..31 of the ldiag mask restricted to the board, bits 0..31 of rdiag, then n/32,
// row/32, free columns/32 and candidates of the next row/32; zero beyond.
__host__ __device__ __forceinline__ float feature(const uint4 st, int j) {
    const uint32_t n = (st.w >> 8) & 0xFFu;
    const uint32_t row = st.w & 0xFFu;
    const uint32_t mask = n >= 32 ? 0xFFFFFFFFu : ((1u << n) - 1u);
    const uint32_t nc = mask & ~st.x;
    if (j < 32) return (float)((nc >> j) & 1u);
    if (j < 64) return (float)(((st.y & mask) >> (j - 32)) & 1u);
    if (j < 96) return (float)(((st.z & mask) >> (j - 64)) & 1u);
    const uint32_t avail = nc & ~(st.y | st.z);
    switch (j) {
        case 96: return n / 32.0f;
        case 97: return row / 32.0f;
#ifdef __CUDA_ARCH__
        case 98: return __popc(nc) / 32.0f;
        case 99: return __popc(avail) / 32.0f;
#else
        case 98: return __builtin_popcount(nc) / 32.0f;
        case 99: return __builtin_popcount(avail) / 32.0f;
#endif
        default: return 0.0f;
    }
}

__device__ __forceinline__ uint32_t pack_half2(__half lo, __half hi) {
    return (uint32_t)__half_as_ushort(lo) | ((uint32_t)__half_as_ushort(hi) << 16);
}

}  // namespace mlp
}  // namespace nqb
