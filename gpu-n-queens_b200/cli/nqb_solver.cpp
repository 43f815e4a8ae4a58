// nqb_solver: the reference's command line (NQ_solver.cu:16-448) over the nqb C ABI.
//
// Same options, meanings and files as the reference's NQ_solver:
//   -t/--try-solve <n>        count-target pool of about n states, solved (default 80M)
//   -g/--gen-states <n>       count-target pool written to -w (no search)
//   -R/--gen-rowlock <row>    pool locked at `row` written to -w (no search)
//   -w/--write-states <path>  output file, or directory with -s
//   -s/--split-states <k>     k chunk files chunk_<i>_for_n<N>_cnt_<c>.nqsf
//   -m/--mix-states           shuffle the pool (generated or loaded)
//   -r/--random-seed <seed>   srand(seed) for the shuffle
//   -l/--load-states <file>   solve the pool of a state file
//   -d/--devices <a,b,...>    GPUs to split the pool across (default: all)
//   -h/--help
// The reference fixes N at compile time (deffinitions.cuh:38, 17); here it is a run-time
// option, -n/--board (default 17), or taken from the file with -l.  -f/--form picks the
// search form (batched by default, or plain).
#include <cerrno>
#include <cinttypes>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>
#include <utility>
#include <vector>

#include "nqb.h"

namespace {

// A library-allocated array (released with nqb_free), used in place.
template <class T>
struct LibArray {
    T* p = nullptr;
    uint64_t n = 0;
    LibArray() = default;
    LibArray(const LibArray&) = delete;
    LibArray& operator=(const LibArray&) = delete;
    ~LibArray() { nqb_free(p); }
    T* data() const { return p; }
    uint64_t size() const { return n; }
    T& operator[](uint64_t i) const { return p[i]; }
};

struct Opt {
    char key;
    const char* shorts;  // accepted short letters
    const char* name;
    const char* value;   // value name, nullptr for a flag
    const char* help;
};

const Opt kOpts[] = {
    {'t', "tT", "try-solve", "limit", "Generate about `limit` states by count-target sizing and solve them"},
    {'g', "gG", "gen-states", "limit", "Generate about `limit` states (soft limit) and write them with -w; no search"},
    {'R', "R", "gen-rowlock", "row", "Generate the pool locked at `row` and write it with -w; no search"},
    {'w', "wW", "write-states", "file/dir", "File for the generated states; a directory when -s is given"},
    {'s', "sS", "split-states", "count", "Split the generated states into `count` chunk files"},
    {'m', "mM", "mix-states", nullptr, "Shuffle the states (generated or loaded)"},
    {'r', "r", "random-seed", "seed", "Seed of the shuffle"},
    {'l', "lL", "load-states", "file", "Load and solve the states of a state file"},
    {'h', "?hH", "help", nullptr, "Show help options"},
    {'d', "dD", "devices", "gpu1,gpu2,...", "Comma-separated CUDA device ids to use (default: all)"},
    {'n', "n", "board", "N", "Board size (default 17; with -l, the file's)"},
    {'f', "f", "form", "plain|batched", "Search form (default batched)"},
};

void usage(const char* argv0) {
    std::printf("Usage: %s <option 1> <option 2> ...\n", argv0);
    for (const Opt& o : kOpts) {
        std::string left = std::string("-") + o.shorts[0] + ", --" + o.name;
        if (o.value) left += std::string("=") + o.value;
        std::printf("  %-32s %s\n", left.c_str(), o.help);
    }
}

// util_large_integer_string_decimal_sep (nq_utils.cu:100-116): thousands separators.
std::string with_commas(uint64_t v) {
    std::string s = std::to_string(v), out;
    for (size_t i = 0; i < s.size(); ++i) {
        if (i && (s.size() - i) % 3 == 0) out += ',';
        out += s[i];
    }
    return out;
}

// shuffle_states (NQ_solver.cu:40-55): for i in [0, len - 2) swap i with
// ((r mod len) + i) mod len, r = four rand() values as the 16-bit lanes of a uint64.
// Below 3 states nothing moves (the reference's bound len - 2 wraps there).
template <class A>
void shuffle(A& v) {
    const uint64_t len = v.size();
    if (len < 3) return;
    for (uint64_t i = 0; i < len - 2; ++i) {
        uint64_t r = 0;
        for (int k = 0; k < 4; ++k) r |= (uint64_t)(uint16_t)std::rand() << (16 * k);
        r = ((r % len) + i) % len;
        if (r != i) std::swap(v[i], v[r]);
    }
}

int fail(const char* fmt, const char* arg = nullptr) {
    std::fprintf(stderr, fmt, arg);
    std::fprintf(stderr, "\n");
    return EXIT_FAILURE;
}

int nqb_fail(const char* what, int status) {
    std::fprintf(stderr, "%s: %s (status %d)\n", what, nqb_strerror(status), status);
    return EXIT_FAILURE;
}

// write_gen_states_to_file (NQ_solver.cu:57-108): one file, or `chunks` files of
// ceil(count / chunks) states, one fewer after the first count % chunks files.
int write_states(const LibArray<nqb_placement>& pl, unsigned n, unsigned lock, int chunks, const char* out) {
    const uint64_t cnt = pl.size();
    if (!chunks) {
        std::printf("Writing generated states to file...");
        const int s = nqb_write_state_file(out, pl.data(), cnt, n, lock, 1);
        if (s) return nqb_fail("Failed to write states to file", s);
        return EXIT_SUCCESS;
    }
    uint64_t per = (uint64_t)std::ceil(cnt / (double)chunks);
    const int left = (int)(cnt % chunks);
    if (!per) return fail("Cannot divide state pool across requested number of chunks! More chunks than states!");
    std::printf("Writing approx. %" PRIu64 " states per file across %d chunk files in %s...\n", per, chunks, out);
    uint64_t written = 0;
    for (int i = 0; i < chunks; ++i) {
        char path[PATH_MAX + 1];
        const int len = std::snprintf(path, sizeof(path), "%s/chunk_%d_for_n%u_cnt_%" PRIu64 ".nqsf", out, i, n, per);
        if (len < 0 || len >= (int)sizeof(path))
            return fail("Failed to construct chunk file path. Max file path length exceeded!");
        std::printf("\tWriting %" PRIu64 " states for chunk %d in file [%s]...", per, i, path);
        const int s = per ? nqb_write_state_file(path, pl.data() + written, per, n, lock, 1) : NQB_E_INVALID;
        if (s) return nqb_fail("\nFailed to write chunk", s);
        written += per;
        if (i == left - 1) --per;
        std::printf("Done\n");
    }
    return written == cnt ? EXIT_SUCCESS : fail("chunk sizes do not add up");
}

// parse_gpu_configs (NQ_solver.cu:143-178): non-empty comma-separated integers.
bool parse_devices(const char* s, std::vector<int>* out) {
    out->clear();
    std::string cur;
    for (const char* p = s;; ++p) {
        if (*p == ',' || !*p) {
            if (cur.empty() || cur.size() >= 20) return false;
            errno = 0;
            char* end = nullptr;
            const long long id = std::strtoll(cur.c_str(), &end, 10);
            if (errno || id < 0 || id > INT_MAX) return false;
            out->push_back((int)id);
            cur.clear();
            if (!*p) break;
        } else {
            cur += *p;
        }
    }
    return !out->empty();
}

struct Args {
    const char* gen_file = nullptr;
    long long state_count = 0, try_count = 0;
    unsigned lock_gen = 0;
    const char* in_file = nullptr;
    int split = 0;
    std::vector<int> devices;
    bool shuffle = false;
    unsigned n = 17;
    bool n_given = false;
    int form = NQB_FORM_BATCHED;
};

const Opt* find_short(char c) {
    for (const Opt& o : kOpts)
        if (std::strchr(o.shorts, c)) return &o;
    return nullptr;
}

const Opt* find_long(const std::string& name) {
    for (const Opt& o : kOpts)
        if (name == o.name) return &o;
    return nullptr;
}

// Returns -1 to go on, else the exit code.
int parse(int argc, char** argv, Args* a) {
    for (int i = 1; i < argc; ++i) {
        const char* arg = argv[i];
        const Opt* o = nullptr;
        const char* val = nullptr;
        if (arg[0] == '-' && arg[1] == '-') {
            std::string name = arg + 2;
            const size_t eq = name.find('=');
            if (eq != std::string::npos) {
                val = arg + 2 + eq + 1;
                name = name.substr(0, eq);
            }
            o = find_long(name);
        } else if (arg[0] == '-' && arg[1]) {
            o = find_short(arg[1]);
            if (o && arg[2]) val = arg[2] == '=' ? arg + 3 : arg + 2;
        }
        if (!o) {
            std::fprintf(stderr, "Unsupported argument '%s'!\n", arg);  // the reference goes on
            continue;
        }
        if (o->value && !val) {
            if (i + 1 >= argc) return fail("Option '%s' needs a value.", arg);
            val = argv[++i];
        }
        long long res = 0;
        errno = 0;
        switch (o->key) {
            case 'r':
                res = std::strtol(val, nullptr, 10);
                if (res > UINT_MAX || res < 0) return fail("Seed '%s' is out of range.", val);
                std::srand((unsigned)res);
                break;
            case 'R':
                res = std::strtoll(val, nullptr, 10);
                if (errno || res <= 0 || res > 255) return fail("Cannot lock at row '%s'!", val);
                a->lock_gen = (unsigned)res;
                break;
            case 'g':
                res = std::strtoll(val, nullptr, 10);
                if (errno || res <= 0) return fail("Cannot generate '%s' many states!", val);
                a->state_count = res;
                break;
            case 'w': a->gen_file = val; break;
            case 's':
                res = std::strtol(val, nullptr, 10);
                if (errno || res <= 0 || res > INT_MAX) return fail("Count value '%s' is invalid.", val);
                a->split = (int)res;
                break;
            case 'l': a->in_file = val; break;
            case 'm': a->shuffle = true; break;
            case 'h': usage(argv[0]); return EXIT_SUCCESS;
            case 'd':
                if (!parse_devices(val, &a->devices)) return fail("Failed to parse GPU list!");
                break;
            case 't':
                res = std::strtoll(val, nullptr, 10);
                if (errno || res <= 0) return fail("Cannot try with '%s' many states!", val);
                a->try_count = res;
                break;
            case 'n':
                res = std::strtoll(val, nullptr, 10);
                if (errno || res < NQB_MIN_N || res > NQB_MAX_N) return fail("Board size '%s' is not supported.", val);
                a->n = (unsigned)res;
                a->n_given = true;
                break;
            case 'f':
                if (!std::strcmp(val, "plain")) a->form = NQB_FORM_PLAIN;
                else if (!std::strcmp(val, "batched")) a->form = NQB_FORM_BATCHED;
                else return fail("Unknown form '%s' (plain or batched).", val);
                break;
        }
    }
    return -1;
}

int print_target(unsigned n, uint64_t how_many, nqb_target* t) {
    const int s = nqb_pool_for_target(n, how_many, t);
    if (s == NQB_OK || s == NQB_E_RANGE)
        for (unsigned k = 0; k < t->tried; ++k)
            std::printf("Lock at row %u... %" PRIu64 " states generated\n", t->first_row + k, t->tried_count[k]);
    if (t->limit_hit)
        std::printf("A first-row column reached the hard limit of %" PRIu64 " states; keeping lock row %u.\n",
                    t->hard_limit, t->lock_row);
    return s;
}

int solve_and_print(const nqb_state* states, uint64_t count, unsigned n, const Args& a) {
    nqb_opts o;
    nqb_default_opts(&o);
    o.form = a.form;
    std::vector<int> devs = a.devices;
    if (devs.empty()) {
        int cnt = 0;
        if (nqb_device_count(&cnt) != NQB_OK || cnt <= 0) return fail("No CUDA device found.");
        for (int d = 0; d < cnt; ++d) devs.push_back(d);
    }
    for (int d : devs) {
        const int s = nqb_device_check(d);
        if (s) return nqb_fail("Device check failed", s);
    }
    std::printf("Solving...\n");
    uint64_t total = 0;
    nqb_stats st;
    const int s = nqb_solve_states_multi(states, count, devs.data(), (unsigned)devs.size(), &o, &total, &st);
    if (s) return nqb_fail("Solving failed", s);
    std::printf("solution_count(%u) = %" PRIu64 " (%s)\n", n, total, with_commas(total).c_str());
    std::printf("\t%" PRIu64 " states on %zu device(s), %" PRIu64 " nodes, kernel %.3f ms, wall %.3f ms\n", st.states,
                devs.size(), st.nodes, st.kernel_ms, st.wall_ms);
    return EXIT_SUCCESS;
}

std::vector<nqb_state> to_states(const LibArray<nqb_placement>& pl, int* status) {
    std::vector<nqb_state> st(pl.size());
    *status = nqb_states_from_placements(pl.data(), pl.size(), 1, st.data());
    return st;
}

int run(int argc, char** argv) {
    Args a;
    const int pr = parse(argc, argv, &a);
    if (pr >= 0) return pr;

    std::printf("\nnqb_solver (libnqb %d), N=%u%s, %s form\n", nqb_version(), a.n, a.n_given ? "" : " (default)",
                a.form == NQB_FORM_PLAIN ? "plain" : "batched");

    if (a.state_count || a.lock_gen) {  // generation to files, no search
        if (a.state_count && a.lock_gen) return fail("The flags -R and -g must not be combined!");
        if (!a.gen_file) return fail("State generation selected, but no output file supplied!");
        if (a.try_count) std::printf("Ignoring solving state count flag -- This is not applicable here.\n");
        unsigned lock = a.lock_gen;
        if (lock) {
            if (lock >= a.n) return fail("Cannot lock at row %s: it must be below N.", std::to_string(lock).c_str());
            std::printf("Starting state generation, locked at row %u. Writing to: %s.\n", lock, a.gen_file);
        } else {
            std::printf("Starting state generation for up to %lld states. Writing to: %s.\n", a.state_count, a.gen_file);
            nqb_target t;
            const int s = print_target(a.n, (uint64_t)a.state_count, &t);
            if (s) return nqb_fail("State generation failed", s);
            lock = t.lock_row;
        }
        LibArray<nqb_placement> pl;
        const int s = nqb_generate_pool_placements(a.n, lock == 1 ? 2 : lock, &pl.p, &pl.n);  // lock row 1: 2-row states
        if (s) return nqb_fail("State generation failed", s);
        if (a.shuffle) shuffle(pl);
        const int w = write_states(pl, a.n, lock, a.split, a.gen_file);
        if (w) return w;
        std::printf("Generation completed.\n");
        return EXIT_SUCCESS;
    }

    if (a.in_file) {  // load a state file and solve it
        if (a.try_count) std::printf("Ignoring solving state count flag -- This is not applicable here.\n");
        std::printf("Loading states from file...\n");
        nqb_state_file info;
        LibArray<nqb_placement> pl;
        int s = nqb_read_state_file(a.in_file, 1, a.n_given ? a.n : 0, &info, &pl.p);
        if (s) return nqb_fail("Failed to read states from file", s);
        pl.n = info.count;
        std::printf("Loaded %" PRIu64 " states\n", info.count);
        if (a.shuffle) {
            std::printf("Shuffling loaded states...\n");
            shuffle(pl);
        }
        bool other_rows = false;
        for (uint64_t i = 0; i < pl.size(); ++i) other_rows |= pl[i].row != info.locked_row;
        if (other_rows)
            std::printf("Note: states start below the file's locked row %u; each is solved from its own row "
                        "(the reference's kernel would also search rows above them).\n", info.locked_row);
        const std::vector<nqb_state> st = to_states(pl, &s);
        if (s) return nqb_fail("Invalid states in file", s);
        return solve_and_print(st.data(), st.size(), info.n, a);
    }

    // count-target pool, solved
    if (!a.try_count) {
        std::printf("WARN: Test-solve run without set number of states. Defaulting to 80M\n");
        a.try_count = 80000000;
    }
    nqb_target t;
    int s = print_target(a.n, (uint64_t)a.try_count, &t);
    if (s) return nqb_fail("Failed to generate states", s);
    LibArray<nqb_state> st;
    s = nqb_generate_pool(a.n, t.pool_depth, &st.p, &st.n);
    if (s) return nqb_fail("Failed to generate states", s);
    std::printf("%" PRIu64 " states generated.\n", st.size());
    return solve_and_print(st.data(), st.size(), a.n, a);
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const std::exception& e) {  // the standard library ran out of host memory or threads
        std::fprintf(stderr, "nqb_solver: %s\n", e.what());
        return EXIT_FAILURE;
    }
}
