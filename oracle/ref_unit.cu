// Compiles one source file of fillpant/GPU-N-Queens, read in place, for a board size
// chosen at build time.  TEST INFRASTRUCTURE ONLY (oracle/_ref).
// The reference fixes N with `#define N 17` (deffinitions.cuh:38) behind an include
// guard; including that header first and redefining N makes every later use of N,
// N_MASK and the block-size formula see NQO_REF_N without editing the sources.
#include "deffinitions.cuh"
#undef N
#define N NQO_REF_N
#include NQO_REF_SRC
