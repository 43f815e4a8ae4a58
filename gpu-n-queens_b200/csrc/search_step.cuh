// One search step of the DoubleSweep-light depth-first search, shared by the plain and
// batched kernels.  Device-only.
//
// A lane's search state is four 32-bit words kept in registers:
//   avail  candidate columns of the current row still to be searched below
//   nc     columns without a queen
//   l, r   columns of the current row attacked along the two diagonals
// plus `sp`, the shared-memory byte address of the top entry of the lane's stack of
// pending rows.  The entry at `base` is a sentinel: popping an empty stack loads it,
// and a step leaves the sentinel state {avail 0, nc 1<<31, l 1<<30, r 0} unchanged
// (no candidate appears and nothing is counted; bit 31 is never a column since
// n <= 31), so a lane whose search is over parks without a branch.  Entries of a lane
// sit BLOCK x 16 bytes apart ([level][BLOCK] layout), so the 32 lanes of a warp touch 32
// consecutive 16-byte slots and an LDS.128 / STS.128 needs no bank replays.
//
// Per step: if the row has no candidate left, pop the deepest pending row; place the
// lowest candidate b (avail & (avail - 1) is the row without it, and their XOR is b); push
// the row back only if candidates remain; step to the next
// row and "enter" it.  A row left without candidates is not pushed, so a row with one
// free column is filled without creating a branch point: the reference's unit-row
// propagation (GPU_NQueens.cu:392-408, n_queens.cuh:145-163).  b is a free column, so it
// is in nc and in neither diagonal mask, and the updates nc ^= b, l = (l|b) << 1,
// r = (r|b) >> 1 are written as subtractions and additions, which spreads them over the
// integer ALU and the IMAD pipe.
//
// Entering a row counts every candidate of the row as a node at once: the search places
// each of them exactly once, so nodes = the sum of the candidate counts of the rows
// entered (the same placements the reference's kernel loop makes, unit and branch alike).
// A row entered with one free column is the last row: its candidate, if any, completes a
// board (a solution).
//
// Dead ends are then counted without being visited.  Placing candidate c leaves the next
// row with the candidates G & ~{c-1, c, c+1}, where G = nc & ~((l << 1) | (r >> 1)) are the
// columns free two rows down from the queens above (c's own column and diagonals aside).
// So c leads to an empty row -- a leaf, whose node was just counted -- exactly when G lies
// inside {c-1, c, c+1}.  When G is empty every candidate is a leaf; when G is one column g
// the leaves are the candidates in {g-1, g, g+1}.  Both cases are removed from `avail`
// before the row is searched (G of two or three adjacent columns also makes leaves; those
// are few and are searched normally, which costs a step but counts them the same way).  At
// N=17..21 this removes 34% of the placements from the step loop and a third of the stack
// pushes and pops.  The last row is always removed this way, so no step ever places a queen
// there.
//
// Stack bound: a row is pushed only while another candidate remains, and pushed rows are
// strictly deeper towards the top, so a search from a state with f free columns holds at
// most f - 1 entries.  Kernels check that bound once per item, so the step itself carries
// no bounds check.  Built with NQB_CHECKS (the checked library), every push is also
// compared with `top`, the lane's last slot: a push past it is dropped and sets bit 0 of the
// lane's `err`, which the kernels report as a device error.
//
// Lane counters are 32-bit: one step adds at most 31 nodes, so kernels fold them into
// 64-bit totals at least every 2^27 / 31 steps.
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

// What one step did, for the optional counters of the kernels.
struct StepInfo {
    uint32_t placed;  // the column placed (0: the lane is parked)
    uint32_t cand;    // candidates of the row entered (before dead ends are dropped)
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

// Candidates `a` of a row minus those whose placement leaves the next row empty, when
// G (see the file comment) has at most one column.  Same arithmetic as the step's.
__device__ __forceinline__ uint32_t drop_leaves(uint32_t a, uint32_t nc, uint32_t l, uint32_t r) {
    const uint32_t g = nc & ~((l << 1) | (r >> 1));
    if ((g & (0u - g)) != g) return a;
    return g ? a & ~((g * 7u) >> 1) : 0u;
}

// PTX of the row entry (candidates, node and solution counts, dead ends dropped), shared
// by both builds of the step: %0 avail, %1 nc, %2 l, %3 r, %5 nodes, %6 sols, %8 cand.
#define NQB_ENTER_ROW                                                   \
    "or.b32 x, %2, %3;\n\t"                                             \
    "not.b32 x, x;\n\t"                                                 \
    "and.b32 %0, %1, x;\n\t"         /* candidates of the entered row */ \
    "popc.b32 %8, %0;\n\t"                                              \
    "add.u32 %5, %5, %8;\n\t"        /* each is placed once: nodes */    \
    "sub.u32 x, %1, 1;\n\t"                                             \
    "and.b32 x, x, %1;\n\t"                                             \
    "setp.eq.u32 u, x, 0;\n\t"       /* one free column: the last row */ \
    "@u add.u32 %6, %6, %8;\n\t"     /* its candidate is a solution */   \
    "shl.b32 g, %2, 1;\n\t"                                             \
    "shr.u32 x, %3, 1;\n\t"                                             \
    "or.b32 g, g, x;\n\t"                                               \
    "not.b32 g, g;\n\t"                                                 \
    "and.b32 g, g, %1;\n\t"          /* G */                             \
    "neg.s32 x, g;\n\t"                                                 \
    "not.b32 w, x;\n\t"                                                 \
    "and.b32 w, w, g;\n\t"                                              \
    "setp.eq.u32 u, w, 0;\n\t"       /* G has at most one column */      \
    "shr.s32 x, x, 31;\n\t"          /* all ones iff G != 0 */           \
    "mul.lo.u32 w, g, 7;\n\t"                                           \
    "shr.u32 w, w, 1;\n\t"           /* {g-1, g, g+1} */                 \
    "not.b32 w, w;\n\t"                                                 \
    "and.b32 w, w, x;\n\t"                                              \
    "@u and.b32 %0, %0, w;\n\t"      /* drop the leaves */

// One step; STRIDE is the byte distance between a lane's stack entries (BLOCK x 16);
// `top` is the byte address of the lane's last stack slot (checked builds only).
template <int STRIDE>
__device__ __forceinline__ StepInfo search_step(Lane& s, uint32_t base, uint32_t top) {
    StepInfo o;
#ifndef NQB_CHECKS
    (void)top;
    asm volatile(
        "{\n\t.reg .pred p, q, t, u;\n\t.reg .u32 x, g, w;\n\t"
        "setp.eq.u32 p, %0, 0;\n\t"                        // no candidate left: pop
        "@p ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n\t"
        "setp.ne.and.u32 q, %4, %9, p;\n\t"
        "@q sub.u32 %4, %4, %10;\n\t"
        "sub.u32 x, %0, 1;\n\t"                            // the row without its lowest candidate b
        "and.b32 x, x, %0;\n\t"
        "setp.ne.u32 t, x, 0;\n\t"                         // candidates remain: push the row
        "xor.b32 %7, %0, x;\n\t"
        "mov.u32 %0, x;\n\t"
        "@t add.u32 %4, %4, %10;\n\t"
        "@t st.shared.v4.u32 [%4], {%0, %1, %2, %3};\n\t"
        "sub.u32 %1, %1, %7;\n\t"                          // next row
        "add.u32 %2, %2, %7;\n\t"
        "shl.b32 %2, %2, 1;\n\t"
        "add.u32 %3, %3, %7;\n\t"
        "shr.u32 %3, %3, 1;\n\t"
        NQB_ENTER_ROW
        "}"
        : "+r"(s.avail), "+r"(s.nc), "+r"(s.l), "+r"(s.r), "+r"(s.sp), "+r"(s.nodes), "+r"(s.sols),
          "=r"(o.placed), "=r"(o.cand)
        : "r"(base), "n"(STRIDE)
        : "memory");
#else
    asm volatile(
        "{\n\t.reg .pred p, q, t, u, ov, ok;\n\t.reg .u32 x, g, w, nsp;\n\t"
        "setp.eq.u32 p, %0, 0;\n\t"
        "@p ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n\t"
        "setp.ne.and.u32 q, %4, %10, p;\n\t"
        "@q sub.u32 %4, %4, %11;\n\t"
        "sub.u32 x, %0, 1;\n\t"
        "and.b32 x, x, %0;\n\t"
        "setp.ne.u32 t, x, 0;\n\t"
        "xor.b32 %7, %0, x;\n\t"
        "mov.u32 %0, x;\n\t"
        "add.u32 nsp, %4, %11;\n\t"                        // the push's slot must not pass top
        "setp.gt.u32 ov, nsp, %12;\n\t"
        "and.pred ok, t, !ov;\n\t"
        "@ok mov.u32 %4, nsp;\n\t"
        "@ok st.shared.v4.u32 [%4], {%0, %1, %2, %3};\n\t"
        "and.pred ov, t, ov;\n\t"
        "@ov or.b32 %9, %9, 1;\n\t"
        "sub.u32 %1, %1, %7;\n\t"
        "add.u32 %2, %2, %7;\n\t"
        "shl.b32 %2, %2, 1;\n\t"
        "add.u32 %3, %3, %7;\n\t"
        "shr.u32 %3, %3, 1;\n\t"
        NQB_ENTER_ROW
        "}"
        : "+r"(s.avail), "+r"(s.nc), "+r"(s.l), "+r"(s.r), "+r"(s.sp), "+r"(s.nodes), "+r"(s.sols),
          "=r"(o.placed), "=r"(o.cand), "+r"(s.err)
        : "r"(base), "n"(STRIDE), "r"(top)
        : "memory");
#endif
    return o;
}

// Loads a state {cols, ldiag, rdiag, meta} into a lane with an empty stack and enters its
// row: the lane's node and solution counters are set to that row's (a complete board handed
// in counts one solution).  Returns the stack depth the search needs (free columns - 1).
__device__ __forceinline__ uint32_t lane_load(Lane& s, const uint4 st, uint32_t base) {
    const uint32_t n = (st.w >> 8) & 0xFFu;
    const uint32_t mask = n >= 32 ? 0xFFFFFFFFu : ((1u << n) - 1u);
    s.nc = mask & ~st.x;
    s.l = st.y;
    s.r = st.z;
    s.sp = base;
    const uint32_t a = s.nc & ~(s.l | s.r);
    const uint32_t pc = __popc(a);
    s.nodes = pc;
    s.sols = (s.nc & (s.nc - 1u)) == 0 ? pc + (s.nc == 0) : 0u;
    s.avail = drop_leaves(a, s.nc, s.l, s.r);
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
