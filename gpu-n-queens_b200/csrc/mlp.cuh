// Learned cost model: shapes, the feature encoding and the activation shared by the training
// kernels (mlp.cu), the fused inference kernel and the host.  Device and host.
#pragma once

#include <cstdint>

#include <cuda_fp16.h>

namespace nqb {
namespace mlp {

// Network 112 -> 128 -> 128 -> 1, GELU after both hidden layers.
constexpr int kIn = 112;  // 96 + 6 board-relative features (see feature()), zero-padded to a multiple of 16
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

__host__ __device__ __forceinline__ uint32_t popc32(uint32_t v) {
#ifdef __CUDA_ARCH__
    return __popc(v);
#else
    return (uint32_t)__builtin_popcount(v);
#endif
}

// Cells of row `row + k` that the queens above leave free (k = 0: the next row's candidates).
__host__ __device__ __forceinline__ uint32_t free_cells_below(uint32_t nc, uint32_t ld, uint32_t rd, uint32_t k) {
    return popc32(nc & ~((ld << k) | (rd >> k)));
}

// Feature j of a state {cols, ldiag, rdiag, meta}.  Every feature is relative to the board, so
// one network ranks states of different board sizes:
//   0..31   free cells of each of the next 32 rows under the queens already placed
//           (row + k for feature k; 0 beyond the last row), / 32
//   32..63  the free-column mask, centred on the board (bit i at 16 - n/2 + i)
//   64..95  the next row's candidate mask, centred the same way
//   96      rows left / 32        97  free columns / 32      98  next-row candidates / 32
//   99      n / 32                100 row / 32               101 sum of features 0..31 x 32 / 256
// then zero.  All are small integers over powers of two, exact in fp16.
__host__ __device__ __forceinline__ float feature(const uint4 st, int j) {
    const uint32_t n = (st.w >> 8) & 0xFFu;
    const uint32_t row = st.w & 0xFFu;
    const uint32_t mask = n >= 32 ? 0xFFFFFFFFu : ((1u << n) - 1u);
    const uint32_t nc = mask & ~st.x;
    const uint32_t left = n > row ? n - row : 0u;
    const uint32_t shift = 16u - (n >> 1);
    if (j < 32) return (uint32_t)j < left ? free_cells_below(nc, st.y, st.z, (uint32_t)j) / 32.0f : 0.0f;
    if (j < 64) return (float)(((nc << shift) >> (j - 32)) & 1u);
    const uint32_t avail = nc & ~(st.y | st.z);
    if (j < 96) return (float)(((avail << shift) >> (j - 64)) & 1u);
    switch (j) {
        case 96: return left / 32.0f;
        case 97: return popc32(nc) / 32.0f;
        case 98: return popc32(avail) / 32.0f;
        case 99: return n / 32.0f;
        case 100: return row / 32.0f;
        case 101: {
            uint32_t sum = 0;
            for (uint32_t k = 0; k < left && k < 32; ++k) sum += free_cells_below(nc, st.y, st.z, k);
            return sum / 256.0f;
        }
        default: return 0.0f;
    }
}

__device__ __forceinline__ uint32_t pack_half2(__half lo, __half hi) {
    return (uint32_t)__half_as_ushort(lo) | ((uint32_t)__half_as_ushort(hi) << 16);
}

}  // namespace mlp
}  // namespace nqb
