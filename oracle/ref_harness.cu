// Harness around the reference's own code (fillpant/GPU-N-Queens), built per board size
// by oracle/Makefile into oracle/_ref/N<n>/ref_harness.  TEST INFRASTRUCTURE ONLY:
// it produces golden vectors, the reference CPU baseline and the reference CUDA
// comparator.  Every result line starts with "NQO_JSON ".
//
//   ref_harness pool   <d>                      pool size, weighted size, content hash
//   ref_harness dump   <d> <file>               pool as nq_state_t records
//   ref_harness replay <d> [stride offset]      kernel-loop replay (GPU_NQueens.cu:338-452)
//   ref_harness cpu    <d> <threads> [stride offset]  host DFS count (n_queens.cu:423-445)
//   ref_harness gpu    <d> [reps]                gpu_solver_driver on the pool (GPU_NQueens.cu:56)
//   ref_harness writemix <d1> <d2> <file>        the d1 and d2 pools interleaved state by state,
//                                                written by util_write_nq_states_to_stream
//   ref_harness readfile <file>                  util_read_nq_states_from_stream: count, lock, hash
//   ref_harness boards <file> <threads>          partial boards of this N, one per line "d c0 .. c(d-1)":
//                                                each built with init_nq_state + place_queen_at and
//                                                streamed with locked_advance_nq_state(d, N-1)
//                                                (n_queens.cu:423-445), no mirror weight: the
//                                                completions and placements below row d of each
#include "deffinitions.cuh"
#undef N
#define N NQO_REF_N
#include "GPU_NQueens.cuh"
#include "n_queens.cuh"
#include "nq_utils.cuh"

#include <atomic>
#include <chrono>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static nq_state_t* make_pool(unsigned d, uint64_t* cnt, nq_mem_handle_t** h) {
    *h = nq_generate_states_rowlock(d, cnt);
    if (!*h || !(*h)->mem_ptr) {
        fprintf(stderr, "pool generation failed\n");
        exit(2);
    }
    return (nq_state_t*)(*h)->mem_ptr;
}

static uint64_t weight_of(const nq_state_t* s) { return s->queen_at_index[0] < (N >> 1) ? 2 : 1; }

// FNV-1a over (curr_row, queen_at_index[0..curr_row)) of every state, in order.
static uint64_t pool_hash(const nq_state_t* p, uint64_t cnt) {
    uint64_t h = 1469598103934665603ull;
    for (uint64_t i = 0; i < cnt; ++i) {
        const unsigned r = (unsigned)p[i].curr_row;
        h = (h ^ r) * 1099511628211ull;
        for (unsigned k = 0; k < r; ++k) h = (h ^ p[i].queen_at_index[k]) * 1099511628211ull;
    }
    return h;
}

static int cmd_pool(unsigned d) {
    uint64_t cnt;
    nq_mem_handle_t* h;
    nq_state_t* p = make_pool(d, &cnt, &h);
    uint64_t w = 0;
    for (uint64_t i = 0; i < cnt; ++i) w += weight_of(&p[i]);
    printf("NQO_JSON {\"n\": %u, \"d\": %u, \"states\": %" PRIu64 ", \"weighted\": %" PRIu64
           ", \"hash\": \"%016" PRIx64 "\", \"state_size\": %zu}\n",
           (unsigned)N, d, cnt, w, pool_hash(p, cnt), sizeof(nq_state_t));
    nq_mem_free(h);
    return 0;
}

static int cmd_dump(unsigned d, const char* path) {
    uint64_t cnt;
    nq_mem_handle_t* h;
    nq_state_t* p = make_pool(d, &cnt, &h);
    FILE* f = fopen(path, "wb");
    if (!f) return 3;
    fwrite(p, sizeof(nq_state_t), cnt, f);
    fclose(f);
    printf("NQO_JSON {\"n\": %u, \"d\": %u, \"states\": %" PRIu64 ", \"state_size\": %zu}\n",
           (unsigned)N, d, cnt, sizeof(nq_state_t));
    nq_mem_free(h);
    return 0;
}

// One thread of kern_doitall_v2_regld replayed with the reference's host functions:
// advance == locked_advance_nq_state(s, lock, N-1), propagation ==
// host_doublesweep_light_nq_state, solution test == cols == N_MASK.
static void replay_one(nq_state_t s, unsigned lock, uint64_t* c, uint64_t* nodes, uint64_t* unit) {
    while (s.curr_row >= (int)lock) {
        if (locked_advance_nq_state(&s, lock, N - 1)) (*nodes)++;
        const int before = __builtin_popcount(s.queens_in_columns);
        host_doublesweep_light_nq_state(&s);
        const int placed = __builtin_popcount(s.queens_in_columns) - before;
        *nodes += (uint64_t)placed;
        *unit += (uint64_t)placed;
        *c += (s.queens_in_columns == N_MASK);
    }
}

static int cmd_replay(unsigned d, uint64_t stride, uint64_t offset) {
    uint64_t cnt;
    nq_mem_handle_t* h;
    nq_state_t* p = make_pool(d, &cnt, &h);
    uint64_t wc = 0, nodes = 0, unit = 0, sampled = 0;
    for (uint64_t i = offset; i < cnt; i += stride) {
        uint64_t c = 0;
        replay_one(p[i], d, &c, &nodes, &unit);
        wc += c * weight_of(&p[i]);
        sampled++;
    }
    printf("NQO_JSON {\"n\": %u, \"d\": %u, \"states\": %" PRIu64 ", \"sampled\": %" PRIu64
           ", \"count\": %" PRIu64 ", \"nodes\": %" PRIu64 ", \"unit\": %" PRIu64 "}\n",
           (unsigned)N, d, cnt, sampled, wc, nodes, unit);
    nq_mem_free(h);
    return 0;
}

// The reference's host DFS (locked_advance_nq_state to row N-1) over the pool, one
// worker thread per host core pulling states from an atomic index.
static int cmd_cpu(unsigned d, unsigned threads, uint64_t stride, uint64_t offset) {
    uint64_t cnt;
    nq_mem_handle_t* h;
    const double tg = now_s();
    nq_state_t* p = make_pool(d, &cnt, &h);
    const double gen_s = now_s() - tg;
    std::vector<uint64_t> idx;
    for (uint64_t i = offset; i < cnt; i += stride) idx.push_back(i);
    std::atomic<uint64_t> next(0), total(0), nodes(0);
    auto work = [&]() {
        uint64_t lc = 0, ln = 0;
        for (;;) {
            const uint64_t k = next.fetch_add(1);
            if (k >= idx.size()) break;
            nq_state_t s = p[idx[k]];
            const uint64_t w = weight_of(&s);
            uint64_t c = 0;
            while (locked_advance_nq_state(&s, d, N - 1)) {
                ln++;
                c += (s.queens_in_columns == N_MASK);
            }
            lc += c * w;
        }
        total += lc;
        nodes += ln;
    };
    const double t0 = now_s();
    std::vector<std::thread> ts;
    for (unsigned t = 0; t < threads; ++t) ts.emplace_back(work);
    for (auto& t : ts) t.join();
    const double secs = now_s() - t0;
    printf("NQO_JSON {\"n\": %u, \"d\": %u, \"states\": %" PRIu64 ", \"sampled\": %zu"
           ", \"count\": %" PRIu64 ", \"nodes\": %" PRIu64 ", \"seconds\": %.6f, \"gen_seconds\": %.6f"
           ", \"threads\": %u}\n",
           (unsigned)N, d, cnt, idx.size(), total.load(), nodes.load(), secs, gen_s, threads);
    nq_mem_free(h);
    return 0;
}

static int cmd_gpu(unsigned d, unsigned reps) {
    uint64_t cnt;
    nq_mem_handle_t* h;
    const double tg = now_s();
    nq_state_t* p = make_pool(d, &cnt, &h);
    const double gen_s = now_s() - tg;
    gpu_config_t cfg;
    cfg.device_id = 0;
    cfg.async = false;
    for (unsigned r = 0; r < reps; ++r) {
        const double t0 = now_s();
        const uint64_t res = gpu_solver_driver(p, (uint_least32_t)cnt, d, &cfg, 1);
        const double secs = now_s() - t0;
        printf("NQO_JSON {\"n\": %u, \"d\": %u, \"states\": %" PRIu64 ", \"count\": %" PRIu64
               ", \"driver_seconds\": %.6f, \"gen_seconds\": %.6f, \"rep\": %u}\n",
               (unsigned)N, d, cnt, res, secs, gen_s, r);
        fflush(stdout);
    }
    nq_mem_free(h);
    return 0;
}

static int cmd_writemix(unsigned d1, unsigned d2, const char* path) {
    uint64_t c1, c2;
    nq_mem_handle_t *h1, *h2;
    nq_state_t* p1 = make_pool(d1, &c1, &h1);
    nq_state_t* p2 = make_pool(d2, &c2, &h2);
    std::vector<nq_state_t> mix;
    mix.reserve(c1 + c2);
    for (uint64_t i = 0; i < c1 || i < c2; ++i) {
        if (i < c1) mix.push_back(p1[i]);
        if (i < c2) mix.push_back(p2[i]);
    }
    FILE* f = fopen(path, "wb");
    if (!f) return 3;
    const int w = util_write_nq_states_to_stream(f, mix.data(), mix.size(), (unsigned char)d1);
    fclose(f);
    printf("NQO_JSON {\"d1\": %u, \"d2\": %u, \"states\": %zu, \"hash\": \"%016" PRIx64 "\", \"status\": %d}\n", d1, d2,
           mix.size(), pool_hash(mix.data(), mix.size()), w);
    nq_mem_free(h1);
    nq_mem_free(h2);
    return w ? 4 : 0;
}

static int cmd_readfile(const char* path) {
    FILE* f = fopen(path, "rb");
    if (!f) return 3;
    nq_mem_handle_t h;
    uint64_t len = 0;
    unsigned char lock = 0;
    const int r = util_read_nq_states_from_stream(f, &h, &len, &lock, false);
    fclose(f);
    if (r) return 4;
    const nq_state_t* p = (const nq_state_t*)h.mem_ptr;
    uint64_t w = 0;
    for (uint64_t i = 0; i < len; ++i) w += weight_of(&p[i]);
    printf("NQO_JSON {\"states\": %" PRIu64 ", \"lock\": %u, \"weighted\": %" PRIu64 ", \"hash\": \"%016" PRIx64 "\"}\n",
           len, (unsigned)lock, w, pool_hash(p, len));
    nq_mem_free(&h);
    return 0;
}

static int cmd_boards(const char* path, unsigned threads) {
    FILE* f = fopen(path, "r");
    if (!f) return 3;
    std::vector<nq_state_t> boards;
    std::vector<unsigned> depth;
    char line[512];
    while (fgets(line, sizeof line, f)) {
        char* p = line;
        char* e = nullptr;
        const unsigned d = (unsigned)strtoul(p, &e, 10);
        if (e == p) continue;
        p = e;
        nq_state_t s = init_nq_state();
        for (unsigned r = 0; r < d; ++r) {
            const unsigned c = (unsigned)strtoul(p, &e, 10);
            p = e;
            place_queen_at(&s, (unsigned char)r, (unsigned char)c);
        }
        s.curr_row = (char)d;
        boards.push_back(s);
        depth.push_back(d);
    }
    fclose(f);
    std::vector<uint64_t> count(boards.size()), nodes(boards.size());
    std::atomic<uint64_t> next(0);
    auto work = [&]() {
        for (;;) {
            const uint64_t k = next.fetch_add(1);
            if (k >= boards.size()) break;
            nq_state_t s = boards[k];
            uint64_t c = 0, ln = 0;
            while (locked_advance_nq_state(&s, depth[k], N - 1)) {
                ln++;
                c += (s.queens_in_columns == N_MASK);
            }
            count[k] = c;
            nodes[k] = ln;
        }
    };
    std::vector<std::thread> ts;
    for (unsigned t = 0; t < (threads ? threads : 1); ++t) ts.emplace_back(work);
    for (auto& t : ts) t.join();
    printf("NQO_JSON {\"n\": %u, \"boards\": %zu, \"count\": [", (unsigned)N, boards.size());
    for (size_t i = 0; i < boards.size(); ++i) printf("%s%" PRIu64, i ? ", " : "", count[i]);
    printf("], \"nodes\": [");
    for (size_t i = 0; i < boards.size(); ++i) printf("%s%" PRIu64, i ? ", " : "", nodes[i]);
    printf("]}\n");
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s pool|dump|replay|cpu|gpu <d> ...\n", argv[0]);
        return 1;
    }
    const unsigned d = (unsigned)strtoul(argv[2], nullptr, 10);
    if (!strcmp(argv[1], "pool")) return cmd_pool(d);
    if (!strcmp(argv[1], "dump") && argc > 3) return cmd_dump(d, argv[3]);
    if (!strcmp(argv[1], "replay")) {
        const uint64_t stride = argc > 3 ? strtoull(argv[3], nullptr, 10) : 1;
        const uint64_t offset = argc > 4 ? strtoull(argv[4], nullptr, 10) : 0;
        return cmd_replay(d, stride ? stride : 1, offset);
    }
    if (!strcmp(argv[1], "cpu") && argc > 3) {
        const unsigned th = (unsigned)strtoul(argv[3], nullptr, 10);
        const uint64_t stride = argc > 4 ? strtoull(argv[4], nullptr, 10) : 1;
        const uint64_t offset = argc > 5 ? strtoull(argv[5], nullptr, 10) : 0;
        return cmd_cpu(d, th ? th : 1, stride ? stride : 1, offset);
    }
    if (!strcmp(argv[1], "writemix") && argc > 4)
        return cmd_writemix(d, (unsigned)strtoul(argv[3], nullptr, 10), argv[4]);
    if (!strcmp(argv[1], "readfile")) return cmd_readfile(argv[2]);
    if (!strcmp(argv[1], "boards"))
        return cmd_boards(argv[2], argc > 3 ? (unsigned)strtoul(argv[3], nullptr, 10) : 1);
    if (!strcmp(argv[1], "gpu")) return cmd_gpu(d, argc > 3 ? (unsigned)strtoul(argv[3], nullptr, 10) : 1);
    fprintf(stderr, "unknown command\n");
    return 1;
}
