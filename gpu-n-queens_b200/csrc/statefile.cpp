// Placements, .nqsf state files and count-target pool sizing: the host-side formats and
// rules of the reference's CLI path (nq_utils.cu:127-259, n_queens.cu:128-219 and :397-406),
// over the same pool as the search (pool.cpp).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "nqb_internal.h"

namespace nqb {
namespace {

constexpr unsigned kMaxRow = sizeof(((nqb_placement*)nullptr)->col);  // 30
// Largest number of row-0 boards one file may hold (their segment has no bytes to bound it).
constexpr uint64_t kMaxRow0Boards = 1ull << 32;
// Largest number of boards whose placements fit one allocation.
constexpr uint64_t kMaxPlacements = SIZE_MAX / sizeof(nqb_placement);

bool placement_ok(const nqb_placement& p) {
    if (p.n < NQB_MIN_N || p.n > NQB_MAX_N || p.row >= p.n || p.row > kMaxRow) return false;
    for (unsigned r = 0; r < p.row; ++r)
        if (p.col[r] >= p.n) return false;
    return true;
}

// Buffered little-endian writer; remembers the first failure.
struct Out {
    FILE* f;
    std::vector<uint8_t> buf;
    bool bad = false;
    // The buffer is sized once (it may throw then) and a flush empties it before it
    // would grow, so writing never allocates.
    explicit Out(FILE* fp) : f(fp) { buf.reserve((1 << 20) + 64); }
    void flush() {
        if (!buf.empty() && std::fwrite(buf.data(), 1, buf.size(), f) != buf.size()) bad = true;
        buf.clear();
    }
    void bytes(const void* p, size_t k) {
        const uint8_t* b = static_cast<const uint8_t*>(p);
        buf.insert(buf.end(), b, b + k);
        if (buf.size() >= (1u << 20)) flush();
    }
    template <class T>
    void put(T v) {
        uint8_t b[sizeof(T)];
        for (size_t i = 0; i < sizeof(T); ++i) b[i] = (uint8_t)((uint64_t)v >> (8 * i));
        bytes(b, sizeof(T));
    }
};

template <class T>
bool get(FILE* f, T* v) {
    uint8_t b[sizeof(T)];
    if (std::fread(b, 1, sizeof(T), f) != sizeof(T)) return false;
    uint64_t x = 0;
    for (size_t i = 0; i < sizeof(T); ++i) x |= (uint64_t)b[i] << (8 * i);
    *v = (T)x;
    return true;
}

// Pool size of each row-0 column for the reference's lock row L: row 1 stands for the
// 2-row prefixes (its generator places row 1 too), row >= n is empty.
int sizes_for_lock(unsigned n, unsigned lock, uint64_t* per_c0, uint64_t* total) {
    const unsigned half = (n + 1) / 2;
    if (lock >= n) {
        std::fill(per_c0, per_c0 + half, 0ull);
        *total = 0;
        return NQB_OK;
    }
    return generate_pool_ex(n, lock == 1 ? 2 : lock, nullptr, nullptr, 0, total, nullptr, per_c0);
}

}  // namespace
}  // namespace nqb

using namespace nqb;

extern "C" {

int nqb_generate_pool_placements(unsigned n, unsigned depth, nqb_placement** placements, uint64_t* count) try {
    if (!placements || !count) return NQB_E_INVALID;
    *placements = nullptr;
    uint64_t cnt = 0;
    NQB_TRY(generate_pool_ex(n, depth, nullptr, nullptr, 0, &cnt, nullptr, nullptr));
    nqb_placement* p =
        alloc_fault() ? nullptr : static_cast<nqb_placement*>(std::malloc((cnt ? cnt : 1) * sizeof(nqb_placement)));
    if (!p) return NQB_E_NOMEM;
    uint64_t got = 0;
    const int s = generate_pool_ex(n, depth, nullptr, p, cnt, &got, nullptr, nullptr);
    if (s != NQB_OK) {
        std::free(p);
        return s;
    }
    *placements = p;
    *count = got;
    return NQB_OK;
} NQB_ABI_CATCH

int nqb_states_from_placements(const nqb_placement* placements, uint64_t count, int mirror_weight, nqb_state* out) {
    if (count && (!placements || !out)) return NQB_E_INVALID;
    for (uint64_t i = 0; i < count; ++i) {
        const nqb_placement& p = placements[i];
        if (!placement_ok(p)) return NQB_E_INVALID;
        uint32_t cols = 0, ld = 0, rd = 0;
        for (unsigned r = 0; r < p.row; ++r) {  // place_queen_at, row by row
            const uint32_t b = 1u << p.col[r];
            cols |= b;
            ld = (ld | b) << 1;
            rd = (rd | b) >> 1;
        }
        nqb_state& s = out[i];
        s.cols = cols;
        s.ldiag = ld;
        s.rdiag = rd;
        s.row = p.row;
        s.n = p.n;
        s.weight = (uint8_t)(mirror_weight && p.row >= 1 && p.col[0] < (p.n >> 1) ? 2 : 1);
        s.flags = 0;
    }
    return NQB_OK;
}

int nqb_write_state_file(const char* path, const nqb_placement* placements, uint64_t count, unsigned n,
                         unsigned locked_row, int header) try {
    if (!path || !placements || count == 0 || n < NQB_MIN_N || n > NQB_MAX_N || locked_row > 255)
        return NQB_E_INVALID;
    uint64_t per_row[kMaxRow + 1] = {};
    for (uint64_t i = 0; i < count; ++i) {
        if (placements[i].n != n || !placement_ok(placements[i])) return NQB_E_INVALID;
        per_row[placements[i].row]++;
    }
    Out o(nullptr);
    FILE* f = std::fopen(path, "wb");
    if (!f) return NQB_E_IO;
    o.f = f;
    if (header) {
        o.put<uint32_t>(NQB_STATE_FILE_VERSION);
        o.put<uint64_t>(NQB_STATE_FILE_FLAGS);
    }
    o.put<uint8_t>((uint8_t)n);
    o.put<uint8_t>((uint8_t)locked_row);
    o.put<uint64_t>(count);
    for (unsigned r = 0; r <= kMaxRow; ++r) {  // one segment per row present, rows ascending
        if (!per_row[r]) continue;
        o.put<uint8_t>((uint8_t)r);
        o.put<uint64_t>(per_row[r]);
        for (uint64_t i = 0; i < count; ++i)
            if (placements[i].row == r) o.bytes(placements[i].col, r);
    }
    o.flush();
    const bool bad = o.bad || std::ferror(f);
    if (std::fclose(f) != 0 || bad) return NQB_E_IO;
    return NQB_OK;
} NQB_ABI_CATCH

int nqb_read_state_file(const char* path, int header, unsigned expect_n, nqb_state_file* info,
                        nqb_placement** placements) try {
    if (!path || !info || !placements) return NQB_E_INVALID;
    std::memset(info, 0, sizeof(*info));
    *placements = nullptr;
    const uint64_t chunk = 1u << 16;  // boards per read
    std::vector<uint8_t> cols;
    cols.reserve(chunk * kMaxRow);  // before the file is open: nothing below throws
    FILE* f = std::fopen(path, "rb");
    if (!f) return NQB_E_IO;
    std::fseek(f, 0, SEEK_END);
    const long fsize = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    nqb_placement* p = nullptr;
    auto fail = [&](int code) {
        std::free(p);
        std::fclose(f);
        return code;
    };
    if (header) {
        if (!get(f, &info->version) || !get(f, &info->flags)) return fail(NQB_E_FORMAT);
        if (info->version != NQB_STATE_FILE_VERSION || info->flags != NQB_STATE_FILE_FLAGS) return fail(NQB_E_FORMAT);
    }
    uint8_t n8 = 0, lock8 = 0;
    uint64_t total = 0;
    if (!get(f, &n8) || !get(f, &lock8) || !get(f, &total)) return fail(NQB_E_FORMAT);
    info->n = n8;
    info->locked_row = lock8;
    info->count = total;
    if (n8 < NQB_MIN_N || n8 > NQB_MAX_N) return fail(NQB_E_FORMAT);
    if (expect_n && n8 != expect_n) return fail(NQB_E_INVALID);
    uint64_t filled = 0, cap = 0;
    for (;;) {
        uint8_t r = 0;
        if (std::fread(&r, 1, 1, f) != 1) break;  // end of file between segments
        uint64_t cnt = 0;
        if (!get(f, &cnt)) return fail(NQB_E_FORMAT);
        if (r >= n8 || r > kMaxRow || cnt > total - filled) return fail(NQB_E_FORMAT);
        const uint64_t left = (uint64_t)(fsize - std::ftell(f));
        // A segment of row r > 0 carries r bytes a board, so the file size bounds its count;
        // boards of row 0 carry none, so their count has a fixed bound instead.
        if (r ? cnt > left / r : cnt > kMaxRow0Boards) return fail(NQB_E_FORMAT);
        if (cnt > kMaxPlacements - filled) return fail(NQB_E_FORMAT);
        for (uint64_t done = 0; done < cnt;) {
            const uint64_t k = cnt - done < chunk ? cnt - done : chunk;
            if (filled + done + k > cap) {  // grow as boards arrive, at most to the segment's end
                uint64_t want = cap * 2 > filled + cnt ? filled + cnt : cap * 2;
                if (want < filled + done + k) want = filled + done + k;
                nqb_placement* q = alloc_fault() ? nullptr
                                                 : static_cast<nqb_placement*>(std::realloc(p, want * sizeof(nqb_placement)));
                if (!q) return fail(NQB_E_NOMEM);
                p = q;
                cap = want;
            }
            cols.resize(k * r);
            if (r && std::fread(cols.data(), 1, k * r, f) != k * r) return fail(NQB_E_FORMAT);
            for (uint64_t j = 0; j < k; ++j) {
                nqb_placement& q = p[filled + done + j];
                std::memset(&q, 0xFF, sizeof(q));
                q.n = n8;
                q.row = r;
                for (unsigned c = 0; c < r; ++c) {
                    const uint8_t v = cols[j * r + c];
                    if (v >= n8) return fail(NQB_E_FORMAT);
                    q.col[c] = v;
                }
            }
            done += k;
        }
        filled += cnt;
    }
    if (std::ferror(f)) return fail(NQB_E_IO);
    if (filled != total) return fail(NQB_E_FORMAT);
    std::fclose(f);
    if (!p && !alloc_fault()) p = static_cast<nqb_placement*>(std::malloc(sizeof(nqb_placement)));
    if (!p) return NQB_E_NOMEM;
    *placements = p;
    return NQB_OK;
} NQB_ABI_CATCH

int nqb_pool_for_target(unsigned n, uint64_t how_many, nqb_target* t) try {
    if (!t || n < NQB_MIN_N || n > NQB_MAX_N || how_many == 0) return NQB_E_INVALID;
    std::memset(t, 0, sizeof(*t));
    // the reference's arithmetic, in double as it does it (n_queens.cu:135-139)
    t->hard_limit = (uint64_t)((double)how_many * (1 + 0.2));
    unsigned lock = (unsigned)(std::log((double)how_many) / std::log((double)n));
    lock = lock >= n ? n - 1 : lock;
    if (!lock) return NQB_E_INVALID;
    t->first_row = lock;
    const unsigned half = (n + 1) / 2;
    bool have = false;  // `actual` holds a generated row
    unsigned a_lock = 0;
    uint64_t a_total = 0, tmp_total = 0;
    bool go = true;
    while (go) {
        if (t->tried) {  // actual = tmp
            have = true;
            a_lock = lock - 1;
            a_total = tmp_total;
        }
        uint64_t per_c0[16] = {};
        uint64_t total = 0;
        NQB_TRY(sizes_for_lock(n, lock, per_c0, &total));
        t->tried_count[t->tried++] = total;
        bool thread_full = false;  // gen_states_rowlock stops at the limit (n_queens.cu:40-74)
        for (unsigned c = 0; c < half; ++c) thread_full |= per_c0[c] >= t->hard_limit;
        if (thread_full) {
            t->limit_hit = 1;
            break;
        }
        tmp_total = total;
        lock++;
        go = tmp_total >= a_total && lock <= n && tmp_total <= t->hard_limit;  // n_queens.cu:189-192
    }
    if (!have) return NQB_E_RANGE;
    t->lock_row = a_lock;
    t->pool_depth = a_lock == 1 ? 2 : a_lock;
    t->count = a_total;
    return NQB_OK;
} NQB_ABI_CATCH

}  // extern "C"
