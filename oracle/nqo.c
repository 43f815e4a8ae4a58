/*
 * nqo.c - CPU oracle for the N-Queens counter.  TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of fillpant/GPU-N-Queens' host generator and device search,
 * used by tests/, the smoke check and the bench's CPU-baseline leg as the checker.
 * It is never linked into libnqb.so and never measured as the product.
 *
 * Parity pins: the reference's known-answer table (test.cu:18), its weighted pool
 * sizes (test.cu:88-104), and outputs of the reference's own host code built from
 * its sources by oracle/Makefile (`make -C oracle ref`; tests/golden/ holds the
 * captured vectors).
 *
 * Reference state model restated here (n_queens.cuh:100-113, diagonals.cuh:8-34):
 *   diag bit (c + i) and anti bit (c + N - i) mark the queen at row i, column c;
 *   the attacked set of row r is (diag >> r) | (anti >> (N - r)), truncated to 32
 *   bits (diagonals.cuh:17-20).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NQO_UNSET 0xFFu
#define NQO_MAXN 31

typedef struct nqo_ref_state {
    uint64_t diag, anti;
    uint32_t cols;
    int curr_row;
    uint8_t q[32];
} nqo_ref_state;

/* Same 16-byte layout as nqb_state in include/nqb.h. */
typedef struct nqo_state {
    uint32_t cols, ldiag, rdiag;
    uint8_t row, n, weight, flags;
} nqo_state;

static uint32_t nq_mask(unsigned n) { return n >= 32 ? 0xFFFFFFFFu : ((1u << n) - 1u); }

/* diagonals.cuh:17-20 */
static uint32_t ref_extract(const nqo_ref_state* s, unsigned n, int row) {
    return (uint32_t)((s->diag >> row) | (s->anti >> (n - (unsigned)row)));
}
/* n_queens.cuh:14 NQ_FREE_COLS_AT */
static uint32_t ref_free_at(const nqo_ref_state* s, unsigned n, int row) {
    return ~(s->cols | ref_extract(s, n, row)) & nq_mask(n);
}
/* n_queens.cuh:125-132 place_queen_at; diagonals.cuh:26-29 dad_add */
static void ref_place(nqo_ref_state* s, unsigned n, int row, unsigned col) {
    s->cols |= 1u << col;
    s->q[row] = (uint8_t)col;
    s->diag |= ((uint64_t)(1u << col)) << row;
    s->anti |= ((uint64_t)(1u << col)) << (n - (unsigned)row);
}
/* n_queens.cuh:134-141 remove_queen_at; diagonals.cuh:31-34 dad_remove */
static void ref_remove(nqo_ref_state* s, unsigned n, int row, unsigned col) {
    s->cols &= ~(1u << col);
    s->q[row] = NQO_UNSET;
    s->diag &= ~(((uint64_t)(1u << col)) << row);
    s->anti &= ~(((uint64_t)(1u << col)) << (n - (unsigned)row));
}
static unsigned lowest_bit_index(uint32_t x) { return (unsigned)__builtin_ctz(x); }

static void ref_init(nqo_ref_state* s) {
    memset(s, 0, sizeof(*s));
    memset(s->q, NQO_UNSET, sizeof(s->q));
}

/*
 * One DFS step restricted to rows [top, lock] (n_queens.cu:423-445,
 * locked_advance_nq_state): take the next free column of the current row (above
 * the queen already there, if any), or backtrack.  Returns 1 when a queen was placed.
 */
static int ref_locked_advance(nqo_ref_state* s, unsigned n, int top, int lock) {
    while (s->curr_row >= top) {
        const unsigned qi = s->q[s->curr_row];
        uint32_t fr = ref_free_at(s, n, s->curr_row);
        if (qi != NQO_UNSET) {
            fr &= (nq_mask(n) << (qi + 1u));
            ref_remove(s, n, s->curr_row, qi);
        }
        if (fr == 0) {
            --s->curr_row;
        } else {
            ref_place(s, n, s->curr_row, lowest_bit_index(fr));
            if (s->curr_row < lock) s->curr_row++;
            return 1;
        }
    }
    return 0;
}

static void ref_to_state(const nqo_ref_state* s, unsigned n, int weight, nqo_state* o) {
    const int r = s->curr_row;
    o->cols = s->cols;
    o->rdiag = (uint32_t)(s->diag >> r);
    o->ldiag = (uint32_t)(s->anti >> (n - (unsigned)r));
    o->row = (uint8_t)r;
    o->n = (uint8_t)n;
    o->weight = (uint8_t)weight;
    o->flags = 0;
}

/* GPU_NQueens.cu:354-357 / :437-439: doubled when the row-0 queen is left of centre. */
static int ref_mirror_weight(unsigned n, unsigned q0) { return q0 < (n >> 1) ? 2 : 1; }

/*
 * Pool generation in the reference's order (n_queens.cu:27-83 gen_states_rowlock,
 * :111-124 one worker per row-0 column, :235-315 concatenation in column order).
 * Emits every state to `emit`; with `keep_ref` the reference record is passed too.
 * A state is kept when rows [0, d) are placed and row d has a free column
 * (n_queens.cu:46-49); its curr_row is d (n_queens.cu:52).  For d == 1 the
 * reference's lock row d-1 = 0 lies above the first searched row, so it places
 * row 1 as well and emits 2-row prefixes with curr_row = 2; this restatement
 * keeps that behaviour.
 */
typedef void (*nqo_emit_fn)(void* ctx, const nqo_ref_state* s, unsigned q0);

static void gen_rowlock(unsigned n, unsigned d, nqo_emit_fn emit, void* ctx) {
    const unsigned half = (n + 1) / 2; /* CEILING(N,2), n_queens.cu:237 */
    for (unsigned c0 = 0; c0 < half; ++c0) {
        nqo_ref_state m;
        ref_init(&m);
        ref_place(&m, n, 0, c0);
        m.curr_row = 1;
        const int top = 1, lock = (int)d - 1;
        for (;;) {
            int adv;
            do {
                adv = ref_locked_advance(&m, n, top, lock);
            } while (adv && (ref_free_at(&m, n, m.curr_row + 1) == 0 || m.q[m.curr_row] == NQO_UNSET));
            if (!adv) break;
            nqo_ref_state out = m;
            out.curr_row++;
            emit(ctx, &out, c0);
        }
    }
}

typedef struct pool_ctx {
    nqo_state* out;
    uint8_t* queens; /* optional: cnt x 32 bytes of queen_at_index */
    uint64_t cap, cnt, weighted;
    unsigned n;
} pool_ctx;

static void pool_emit(void* vctx, const nqo_ref_state* s, unsigned q0) {
    pool_ctx* c = (pool_ctx*)vctx;
    const int w = ref_mirror_weight(c->n, q0);
    if (c->out && c->cnt < c->cap) {
        ref_to_state(s, c->n, w, &c->out[c->cnt]);
        if (c->queens) memcpy(c->queens + 32 * c->cnt, s->q, 32);
    }
    c->cnt++;
    c->weighted += (uint64_t)w;
}

/* Number of pool states and their summed weights. */
int nqo_pool_size(unsigned n, unsigned d, uint64_t* cnt, uint64_t* weighted) {
    if (n < 2 || n > NQO_MAXN || d < 1 || d >= n) return 1;
    pool_ctx c = {0};
    c.n = n;
    gen_rowlock(n, d, pool_emit, &c);
    *cnt = c.cnt;
    *weighted = c.weighted;
    return 0;
}

/* Fills up to cap states (and, if queens != NULL, 32-byte queen rows per state). */
int nqo_pool_fill(unsigned n, unsigned d, nqo_state* out, uint8_t* queens, uint64_t cap,
                  uint64_t* cnt) {
    if (n < 2 || n > NQO_MAXN || d < 1 || d >= n) return 1;
    pool_ctx c = {0};
    c.n = n;
    c.out = out;
    c.queens = queens;
    c.cap = cap;
    gen_rowlock(n, d, pool_emit, &c);
    *cnt = c.cnt;
    return c.cnt > cap ? 2 : 0;
}

/*
 * Replay of one thread of kern_doitall_v2_regld (GPU_NQueens.cu:338-452) on the CPU:
 * the advance sub-step (:363-389), DoubleSweep-light unit-row propagation
 * (:392-408) and the solution test (:410-435), until the state backtracks above
 * `lock`.  Returns the unweighted count; nodes = all placements, unit = those made
 * by propagation.
 */
static void replay_ref(nqo_ref_state* s, unsigned n, int lock, uint64_t* count, uint64_t* nodes,
                       uint64_t* unit) {
    const uint32_t mask = nq_mask(n);
    uint64_t c = 0, nd = 0, un = 0;
    for (;;) {
        if (!(s->curr_row >= lock)) break;
        while (s->curr_row >= lock) { /* advance */
            const unsigned qi = s->q[s->curr_row];
            uint32_t fr = ref_free_at(s, n, s->curr_row);
            if (qi != NQO_UNSET) {
                fr &= (mask << (qi + 1u));
                ref_remove(s, n, s->curr_row, qi);
            }
            if (!fr) {
                --s->curr_row;
            } else {
                ref_place(s, n, s->curr_row, lowest_bit_index(fr));
                nd++;
                if (s->curr_row < (int)n - 1) ++s->curr_row;
                break;
            }
        }
        while (s->q[s->curr_row] == NQO_UNSET) { /* propagate */
            const uint32_t fr = ref_free_at(s, n, s->curr_row);
            if (__builtin_popcount(fr) == 1) {
                ref_place(s, n, s->curr_row, 31u - (unsigned)__builtin_clz(fr));
                nd++;
                un++;
                if (s->curr_row < (int)n - 1) ++s->curr_row;
            } else {
                break;
            }
        }
        c += (s->cols == mask);
    }
    *count = c;
    *nodes = nd;
    *unit = un;
}

/* Builds the reference record of a library state (inverse of ref_to_state). */
static void state_to_ref(const nqo_state* st, const uint8_t* queens, nqo_ref_state* s) {
    ref_init(s);
    const unsigned n = st->n;
    for (int r = 0; r < st->row; ++r) ref_place(s, n, r, queens[r]);
    s->curr_row = st->row;
}

/*
 * Replays every state of the (n, d) pool: mirror-weighted count, nodes and unit
 * nodes summed over the pool (GPU_NQueens.cu:437-443 weighting and summation).
 * stride/offset select a deterministic sample: states i with i % stride == offset.
 */
int nqo_replay_pool(unsigned n, unsigned d, uint64_t stride, uint64_t offset, uint64_t* wcount,
                    uint64_t* nodes, uint64_t* unit, uint64_t* sampled) {
    uint64_t cnt, weighted;
    if (nqo_pool_size(n, d, &cnt, &weighted)) return 1;
    if (stride == 0) stride = 1;
    nqo_state* st = (nqo_state*)malloc(sizeof(nqo_state) * (cnt ? cnt : 1));
    uint8_t* qs = (uint8_t*)malloc(32 * (cnt ? cnt : 1));
    if (!st || !qs) { free(st); free(qs); return 2; }
    uint64_t got;
    nqo_pool_fill(n, d, st, qs, cnt, &got);
    const int lock = (d == 1) ? 1 : (int)d; /* the reference solves with locked_row_end = d */
    uint64_t wc = 0, nd = 0, un = 0, sm = 0;
    for (uint64_t i = offset; i < got; i += stride) {
        nqo_ref_state s;
        state_to_ref(&st[i], qs + 32 * i, &s);
        uint64_t c, a, b;
        replay_ref(&s, n, lock, &c, &a, &b);
        wc += c * st[i].weight;
        nd += a;
        un += b;
        sm++;
    }
    free(st);
    free(qs);
    *wcount = wc;
    *nodes = nd;
    *unit = un;
    *sampled = sm;
    return 0;
}

/*
 * Independent plain backtracker (own design, not the reference's method): classic
 * shifted-bitmask recursion.  Counts completions of a library state and the
 * placements made below its start row.
 */
static void bt(uint32_t avail_cols, uint32_t ld, uint32_t rd, uint64_t* count, uint64_t* nodes) {
    if (avail_cols == 0) { (*count)++; return; }
    uint32_t f = avail_cols & ~(ld | rd);
    while (f) {
        const uint32_t b = f & (0u - f);
        f ^= b;
        (*nodes)++;
        bt(avail_cols ^ b, (ld | b) << 1, (rd | b) >> 1, count, nodes);
    }
}

/* Completions (unweighted) and nodes of one library state. */
void nqo_solve_state(const nqo_state* s, uint64_t* count, uint64_t* nodes) {
    uint64_t c = 0, nd = 0;
    bt(nq_mask(s->n) & ~s->cols, s->ldiag, s->rdiag, &c, &nd);
    *count = c;
    *nodes = nd;
}

/* Solves an array of library states: out[i] = weight x completions. */
void nqo_solve_states(const nqo_state* s, uint64_t cnt, uint64_t* out, uint64_t* total_nodes) {
    uint64_t tn = 0;
    for (uint64_t i = 0; i < cnt; ++i) {
        uint64_t c, nd;
        nqo_solve_state(&s[i], &c, &nd);
        out[i] = c * s[i].weight;
        tn += nd;
    }
    *total_nodes = tn;
}

/* Full count of the n-board by the independent backtracker (no pool, no mirror). */
void nqo_backtrack_count(unsigned n, uint64_t* count, uint64_t* nodes) {
    uint64_t c = 0, nd = 0;
    bt(nq_mask(n), 0, 0, &c, &nd);
    *count = c;
    *nodes = nd;
}

/* Reference nq_state_t size for board n: 8-byte aligned {u64,u64,u32,char,u8[n]}. */
uint64_t nqo_ref_state_size(unsigned n) { return ((16u + 4u + 1u + n) + 7u) & ~7ull; }

/* Writes the pool as reference nq_state_t records (stride nqo_ref_state_size(n)). */
int nqo_pool_fill_ref(unsigned n, unsigned d, uint8_t* out, uint64_t cap, uint64_t* cnt) {
    uint64_t c, w;
    if (nqo_pool_size(n, d, &c, &w)) return 1;
    nqo_state* st = (nqo_state*)malloc(sizeof(nqo_state) * (c ? c : 1));
    uint8_t* qs = (uint8_t*)malloc(32 * (c ? c : 1));
    if (!st || !qs) { free(st); free(qs); return 2; }
    uint64_t got;
    nqo_pool_fill(n, d, st, qs, c, &got);
    const uint64_t sz = nqo_ref_state_size(n);
    for (uint64_t i = 0; i < got && i < cap; ++i) {
        nqo_ref_state s;
        state_to_ref(&st[i], qs + 32 * i, &s);
        uint8_t* p = out + sz * i;
        memset(p, 0, sz);
        memcpy(p, &s.diag, 8);
        memcpy(p + 8, &s.anti, 8);
        memcpy(p + 16, &s.cols, 4);
        p[20] = (uint8_t)(int8_t)s.curr_row;
        memcpy(p + 21, s.q, n);
    }
    free(st);
    free(qs);
    *cnt = got;
    return got > cap ? 2 : 0;
}
