// One search step of the DoubleSweep-light depth-first search, shared by the plain and
// batched kernels.  Device-only.
//
// A lane's search state is four 32-bit words kept in registers:
//   avail  candidate columns of the current row not tried yet
//   nc     columns without a queen
//   l, r   columns of the current row attacked along the two diagonals
// plus `sp`, the shared-memory byte address of the top entry of the lane's stack of
// pending rows.  The entry at `base` is a sentinel: popping an empty stack loads it,
// and a step leaves the sentinel state {avail 0, nc 1<<31, l 1<<30, r 0} unchanged
// (l shifts onto nc's bit 31, so no candidate appears, and nc != 0, so no solution is
// counted; bit 31 is never a column since n <= 31).  A lane whose search is over
// therefore parks without a branch.  Entries of a lane sit BLOCK x 16 bytes apart
// ([level][BLOCK] layout), so the 32 lanes of a warp touch 32 consecutive 16-byte
// slots and an LDS.128 / STS.128 needs no bank replays.
//
// Per step: if the row has no candidate left, pop the deepest pending row; place the
// lowest candidate b; push the row back only if candidates remain; step to the next
// row.  A row left without candidates is not pushed, so a row with one free column is
// filled without creating a branch point: the reference's unit-row propagation
// (GPU_NQueens.cu:392-408, n_queens.cuh:145-163).  A step places at most one queen and
// every placement is one node; nc == 0 right after a placement is a solution.
// b is a free column, so it is in nc and in neither diagonal mask, and the updates
// nc ^= b, l = (l|b) << 1, r = (r|b) >> 1 are written as subtractions and additions,
// which lets the compiler spread them over the integer ALU and the IMAD pipe.
//
// Stack bound: a row is pushed only while another free column remains, and pushed
// rows are strictly deeper towards the top, so a search from a state with f free
// columns holds at most f - 1 entries.  Kernels check that bound once per item, so the
// step itself carries no bounds check.  Built with NQB_CHECKS (the checked library), every
// push is also compared with `top`, the lane's last slot: a push past it is dropped and
// sets bit 0 of the lane's `err`, which the kernels report as a device error.
#pragma once

#include <cstdint>

namespace nqb {

constexpr uint32_t kSentinelNc = 0x80000000u;
constexpr uint32_t kSentinelL = 0x40000000u;

struct Lane {
    uint32_t avail, nc, l, r;
    uint32_t sp;     // shared byte address of the top entry; == base when the stack is empty
    uint32_t sols;   // solutions since the last fold
    uint32_t nodes;  // placements since the last fold
    uint32_t err;    // NQB_CHECKS builds: bit 0 = a push would have passed the lane's last slot
};

__device__ __forceinline__ uint4 lds128(uint32_t addr) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(addr)
                 : "memory");
    return v;
}

__device__ __forceinline__ void sts128(uint32_t addr, uint4 v) {
    asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                 : "memory");
}

__device__ __forceinline__ void write_sentinel(uint32_t addr) {
    sts128(addr, make_uint4(0u, kSentinelNc, kSentinelL, 0u));
}

// One step; STRIDE is the byte distance between a lane's stack entries (BLOCK x 16);
// `top` is the byte address of the lane's last stack slot (checked builds only).
template <int STRIDE>
__device__ __forceinline__ void search_step(Lane& s, uint32_t base, uint32_t top) {
#ifndef NQB_CHECKS
    (void)top;
    asm volatile(
        "{\n\t.reg .pred p, q, t;\n\t.reg .u32 b, nb;\n\t"
        "setp.eq.u32 p, %0, 0;\n\t"                        // no candidate left: pop
        "@p ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n\t"
        "setp.ne.and.u32 q, %4, %7, p;\n\t"
        "@q sub.u32 %4, %4, %8;\n\t"
        "neg.s32 nb, %0;\n\t"                              // b = lowest candidate
        "and.b32 b, %0, nb;\n\t"
        "sub.u32 %0, %0, b;\n\t"
        "setp.ne.u32 t, %0, 0;\n\t"                        // candidates remain: push the row
        "@t add.u32 %4, %4, %8;\n\t"
        "@t st.shared.v4.u32 [%4], {%0, %1, %2, %3};\n\t"
        "sub.u32 %1, %1, b;\n\t"                           // next row
        "add.u32 %2, %2, b;\n\t"
        "shl.b32 %2, %2, 1;\n\t"
        "add.u32 %3, %3, b;\n\t"
        "shr.u32 %3, %3, 1;\n\t"
        "or.b32 nb, %2, %3;\n\t"
        "not.b32 nb, nb;\n\t"
        "and.b32 %0, %1, nb;\n\t"
        "setp.ne.u32 t, b, 0;\n\t"                         // one node per placement
        "@t add.u32 %5, %5, 1;\n\t"
        "setp.eq.u32 t, %1, 0;\n\t"                        // all columns used: a solution
        "@t add.u32 %6, %6, 1;\n\t}"
        : "+r"(s.avail), "+r"(s.nc), "+r"(s.l), "+r"(s.r), "+r"(s.sp), "+r"(s.nodes), "+r"(s.sols)
        : "r"(base), "n"(STRIDE)
        : "memory");
#else
    asm volatile(
        "{\n\t.reg .pred p, q, t, ov, ok;\n\t.reg .u32 b, nb, nsp;\n\t"
        "setp.eq.u32 p, %0, 0;\n\t"
        "@p ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n\t"
        "setp.ne.and.u32 q, %4, %8, p;\n\t"
        "@q sub.u32 %4, %4, %9;\n\t"
        "neg.s32 nb, %0;\n\t"
        "and.b32 b, %0, nb;\n\t"
        "sub.u32 %0, %0, b;\n\t"
        "setp.ne.u32 t, %0, 0;\n\t"
        "add.u32 nsp, %4, %9;\n\t"                         // the push's slot must not pass top
        "setp.gt.u32 ov, nsp, %10;\n\t"
        "and.pred ok, t, !ov;\n\t"
        "@ok mov.u32 %4, nsp;\n\t"
        "@ok st.shared.v4.u32 [%4], {%0, %1, %2, %3};\n\t"
        "and.pred ov, t, ov;\n\t"
        "@ov or.b32 %7, %7, 1;\n\t"
        "sub.u32 %1, %1, b;\n\t"
        "add.u32 %2, %2, b;\n\t"
        "shl.b32 %2, %2, 1;\n\t"
        "add.u32 %3, %3, b;\n\t"
        "shr.u32 %3, %3, 1;\n\t"
        "or.b32 nb, %2, %3;\n\t"
        "not.b32 nb, nb;\n\t"
        "and.b32 %0, %1, nb;\n\t"
        "setp.ne.u32 t, b, 0;\n\t"
        "@t add.u32 %5, %5, 1;\n\t"
        "setp.eq.u32 t, %1, 0;\n\t"
        "@t add.u32 %6, %6, 1;\n\t}"
        : "+r"(s.avail), "+r"(s.nc), "+r"(s.l), "+r"(s.r), "+r"(s.sp), "+r"(s.nodes), "+r"(s.sols), "+r"(s.err)
        : "r"(base), "n"(STRIDE), "r"(top)
        : "memory");
#endif
}

// Loads a state {cols, ldiag, rdiag, meta} into a lane with an empty stack.  Returns
// the stack depth the search needs (free columns - 1).
__device__ __forceinline__ uint32_t lane_load(Lane& s, const uint4 st, uint32_t base) {
    const uint32_t n = (st.w >> 8) & 0xFFu;
    const uint32_t mask = n >= 32 ? 0xFFFFFFFFu : ((1u << n) - 1u);
    s.nc = mask & ~st.x;
    s.l = st.y;
    s.r = st.z;
    s.avail = s.nc & ~(s.l | s.r);
    s.sp = base;
    s.sols = (s.nc == 0);  // a complete board handed in as a state
    const uint32_t f = __popc(s.nc);
    return f ? f - 1 : 0;
}

// Empties a lane: the next step pops the sentinel.
__device__ __forceinline__ void lane_park(Lane& s, uint32_t base) {
    s.avail = 0;
    s.nc = kSentinelNc;
    s.l = kSentinelL;
    s.r = 0;
    s.sp = base;
}

__device__ __forceinline__ unsigned warp_or(unsigned v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v |= __shfl_down_sync(0xFFFFFFFFu, v, o);
    return v;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    return v;
}

}  // namespace nqb
