// Host pool generator: every valid placement of the first `depth` rows, in the order of
// the reference's gen_states_threaded_rowlock (n_queens.cu:235-315).
//
// The reference runs one pthread per row-0 column (n_queens.cu:111-124), walks rows
// [1, depth) with locked_advance_nq_state (n_queens.cu:423-445, lowest free column
// first) and keeps a prefix when row `depth` still has a free column
// (n_queens.cu:46-49), then concatenates the per-column buffers in column order.
// Here the walk is a recursion over shifted 32-bit masks, split into tasks of
// (row-0, row-1) column pairs for load balance; a counting pass sizes every task, a
// prefix sum gives each task its offset, and a second pass writes the states in
// place, so the concatenated order equals the reference's.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <cstdlib>
#include <thread>
#include <vector>

#include "nqb_internal.h"

namespace nqb {

unsigned host_threads() {
    if (const char* e = std::getenv("NQB_THREADS")) {
        const long v = std::strtol(e, nullptr, 10);
        if (v > 0 && v < 4096) return (unsigned)v;
    }
    const unsigned h = std::thread::hardware_concurrency();
    return h ? h : 1;
}

namespace {

struct Walker {
    unsigned n, depth;
    uint32_t mask;
    uint8_t weight;
    nqb_state* out;      // nullptr: no states written
    nqb_placement* pout; // nullptr: no placements written
    uint64_t cnt = 0;
    uint8_t path[32];    // column of the queen in each row placed so far

    void walk(unsigned row, uint32_t cols, uint32_t ld, uint32_t rd) {
        if (row == depth) {
            if (mask & ~(cols | ld | rd)) {
                if (pout) {
                    nqb_placement& p = pout[cnt];
                    std::memset(&p, 0xFF, sizeof(p));  // rows >= depth: no queen (UNSET)
                    p.n = (uint8_t)n;
                    p.row = (uint8_t)row;
                    std::memcpy(p.col, path, row);
                }
                if (out) {
                    nqb_state& s = out[cnt];
                    s.cols = cols;
                    s.ldiag = ld;
                    s.rdiag = rd;
                    s.row = (uint8_t)row;
                    s.n = (uint8_t)n;
                    s.weight = weight;
                    s.flags = 0;
                }
                cnt++;
            }
            return;
        }
        uint32_t f = mask & ~(cols | ld | rd);
        while (f) {
            const uint32_t b = f & (0u - f);
            f ^= b;
            path[row] = (uint8_t)__builtin_ctz(b);
            walk(row + 1, cols | b, (ld | b) << 1, (rd | b) >> 1);
        }
    }
};

struct Task {
    unsigned c0;
    int c1;  // -1: task covers only the row-0 placement (depth == 1)
};

}  // namespace

int generate_pool_ex(unsigned n, unsigned depth, nqb_state* buf, nqb_placement* pbuf, uint64_t capacity,
                     uint64_t* count, uint64_t* weighted, uint64_t* per_first_col) {
    if (n < NQB_MIN_N || n > NQB_MAX_N || depth < 1 || depth >= n || !count) return NQB_E_INVALID;
    const uint32_t mask = board_mask(n);
    const unsigned half = (n + 1) / 2;  // row-0 columns searched (mirror elimination)

    std::vector<Task> tasks;
    for (unsigned c0 = 0; c0 < half; ++c0) {
        if (depth == 1) {
            tasks.push_back({c0, -1});
            continue;
        }
        const uint32_t b0 = 1u << c0;
        uint32_t f1 = mask & ~(b0 | (b0 << 1) | (b0 >> 1));
        while (f1) {
            const uint32_t b1 = f1 & (0u - f1);
            f1 ^= b1;
            tasks.push_back({c0, __builtin_ctz(b1)});
        }
    }
    auto run_task = [&](const Task& t, nqb_state* out, nqb_placement* pout) -> uint64_t {
        Walker w;
        w.n = n;
        w.depth = depth;
        w.mask = mask;
        w.weight = (uint8_t)(t.c0 < (n >> 1) ? 2 : 1);  // GPU_NQueens.cu:354-357
        w.out = out;
        w.pout = pout;
        w.path[0] = (uint8_t)t.c0;
        const uint32_t b0 = 1u << t.c0;
        if (t.c1 < 0) {
            w.walk(1, b0, b0 << 1, b0 >> 1);
        } else {
            w.path[1] = (uint8_t)t.c1;
            const uint32_t b1 = 1u << t.c1;
            const uint32_t ld = ((b0 << 1) | b1) << 1, rd = ((b0 >> 1) | b1) >> 1;
            w.walk(2, b0 | b1, ld, rd);
        }
        return w.cnt;
    };

    const unsigned nt = std::max(1u, std::min<unsigned>(host_threads(), (unsigned)tasks.size()));
    std::vector<uint64_t> sizes(tasks.size(), 0);
    auto parallel = [&](auto&& fn) {
        std::atomic<size_t> next(0);
        auto body = [&]() {
            for (;;) {
                const size_t k = next.fetch_add(1);
                if (k >= tasks.size()) break;
                fn(k);
            }
        };
        if (nt == 1) {
            body();
            return;
        }
        std::vector<std::thread> ts;
        try {  // tasks are claimed from a shared counter, so fewer threads only take longer
            ts.reserve(nt);
            for (unsigned i = 0; i < nt; ++i) ts.emplace_back(body);
        } catch (...) {
        }
        body();
        for (auto& t : ts) t.join();
    };
    parallel([&](size_t k) { sizes[k] = run_task(tasks[k], nullptr, nullptr); });

    std::vector<uint64_t> offs(tasks.size() + 1, 0);
    uint64_t w_total = 0;
    for (size_t k = 0; k < tasks.size(); ++k) {
        offs[k + 1] = offs[k] + sizes[k];
        w_total += sizes[k] * (tasks[k].c0 < (n >> 1) ? 2u : 1u);
    }
    *count = offs.back();
    if (weighted) *weighted = w_total;
    if (per_first_col) {
        std::fill(per_first_col, per_first_col + half, 0ull);
        for (size_t k = 0; k < tasks.size(); ++k) per_first_col[tasks[k].c0] += sizes[k];
    }
    if (!buf && !pbuf) return NQB_OK;
    if (offs.back() > capacity) return NQB_E_RANGE;
    parallel([&](size_t k) { run_task(tasks[k], buf ? buf + offs[k] : nullptr, pbuf ? pbuf + offs[k] : nullptr); });
    return NQB_OK;
}

int generate_pool(unsigned n, unsigned depth, nqb_state* buf, uint64_t capacity, uint64_t* count,
                  uint64_t* weighted) {
    return generate_pool_ex(n, depth, buf, nullptr, capacity, count, weighted, nullptr);
}

unsigned max_stack_depth(const nqb_state* states, uint64_t count) {
    unsigned best = 0;
    for (uint64_t i = 0; i < count; ++i) {
        const unsigned n = states[i].n;
        const unsigned f = (unsigned)__builtin_popcount(board_mask(n > 32 ? 32 : n) & ~states[i].cols);
        if (f > best) best = f;
    }
    return best > 1 ? best - 1 : 1;
}

}  // namespace nqb

namespace {

struct SplitMix64 {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    uint32_t below(uint32_t k) { return (uint32_t)(((next() >> 32) * (uint64_t)k) >> 32); }
};

}  // namespace

extern "C" int nqb_sample_boards(uint64_t seed, uint64_t count, unsigned n_min, unsigned n_max, unsigned d_min,
                                 unsigned d_max, nqb_state* out) try {
    if ((count && !out) || n_min < NQB_MIN_N || n_max > NQB_MAX_N || n_min > n_max || d_min < 1 || d_min > d_max ||
        d_max >= n_min)
        return NQB_E_INVALID;
    SplitMix64 rng{seed};
    for (uint64_t i = 0; i < count; ++i) {
        const unsigned n = n_min + rng.below(n_max - n_min + 1);
        const unsigned d = d_min + rng.below(d_max - d_min + 1);
        const uint32_t mask = nqb::board_mask(n);
        uint32_t cols, ld, rd;
        for (;;) {
            cols = ld = rd = 0;
            unsigned r = 0;
            for (; r < d; ++r) {
                uint32_t f = mask & ~(cols | ld | rd);
                if (!f) break;
                for (uint32_t k = rng.below((uint32_t)__builtin_popcount(f)); k; --k) f &= f - 1;
                const uint32_t b = f & (0u - f);
                cols |= b;
                ld = (ld | b) << 1;
                rd = (rd | b) >> 1;
            }
            if (r == d) break;
        }
        nqb_state& s = out[i];
        s.cols = cols;
        s.ldiag = ld;
        s.rdiag = rd;
        s.row = (uint8_t)d;
        s.n = (uint8_t)n;
        s.weight = 1;
        s.flags = 0;
    }
    return NQB_OK;
} NQB_ABI_CATCH
