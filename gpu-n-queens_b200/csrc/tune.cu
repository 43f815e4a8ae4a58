// Launch autotuner for full counts: picks the pool depth, form, block size and split
// factor by timing candidates on a stride sample of each candidate depth's pool.
//
// Every state of a pool stands for one subtree, so every k-th state is an unbiased sample
// of 1/k of the count's work; the sample keeps the pool's order and spread of subtree
// sizes.  Each candidate runs twice on the sample (the first run also warms it up) and
// the faster time counts.  All candidates of one depth must agree on the sample's count.
#include <cstring>
#include <vector>

#include "nqb_internal.h"

namespace nqb {
namespace {

__global__ void stride_gather_kernel(const uint4* __restrict__ in, uint64_t count, uint64_t stride,
                                     uint4* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = in[i * stride];
}

struct Candidate {
    int form, block, factor;
};

// Times one candidate on the sample: the faster of two runs (ms) and the sample's count.
int time_candidate(const nqb_state* d_sample, uint32_t count, unsigned depth, const nqb_opts& base,
                   const Candidate& c, int device, cudaStream_t s, unsigned long long* d_out, double* ms,
                   unsigned long long* sample_count) {
    nqb_opts o = base;
    o.form = c.form;
    o.block_size = c.block;
    o.split_factor = c.factor;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    NQB_TRY(cuda_status(cudaEventCreate(&e0)));
    int st = cuda_status(cudaEventCreate(&e1));
    double best = -1.0;
    for (int rep = 0; rep < 2 && !st; ++rep) {
        st = cuda_status(cudaMemsetAsync(d_out, 0, 8 * sizeof(unsigned long long) + kBatchedScratchBytes, s));
        if (!st) st = cuda_status(cudaEventRecord(e0, s));
        unsigned launches = 0;
        if (!st) {
            if (c.form == NQB_FORM_BATCHED) {
                SchedInfo info;
                st = launch_batched_scheduled(d_sample, count, nullptr, d_out + 8, kBatchedScratchBytes, d_out,
                                              nullptr, nullptr, o, depth, device, s, &launches, &info);
            } else {
                st = launch_plain(d_sample, count, d_out, nullptr, c.block, false, depth, s, &launches);
            }
        }
        if (!st) st = cuda_status(cudaEventRecord(e1, s));
        unsigned long long h[4] = {0, 0, 0, 0};
        if (!st) st = cuda_status(cudaMemcpyAsync(h, d_out, sizeof(h), cudaMemcpyDeviceToHost, s));
        if (!st) st = cuda_status(cudaStreamSynchronize(s));
        float t = 0.0f;
        if (!st) st = cuda_status(cudaEventElapsedTime(&t, e0, e1));
        if (!st && h[3]) st = (h[3] & 4) ? NQB_E_STALL : NQB_E_DEVICE;
        if (!st) {
            if (best < 0 || t < best) best = t;
            *sample_count = h[0];
        }
    }
    cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    *ms = best;
    return st;
}

}  // namespace
}  // namespace nqb

using namespace nqb;

extern "C" int nqb_tune_count(unsigned n, const unsigned* depths, unsigned n_depths, const nqb_opts* opts,
                              unsigned sample_div, nqb_tune_result* out) try {
    if (!out || !depths || n_depths == 0 || sample_div == 0) return NQB_E_INVALID;
    std::memset(out, 0, sizeof(*out));
    nqb_opts base;
    nqb_default_opts(&base);
    if (opts) base = *opts;
    for (unsigned k = 0; k < n_depths; ++k)
        if (n < NQB_MIN_N || n > NQB_MAX_N || depths[k] < 1 || depths[k] >= n) return NQB_E_INVALID;
    std::vector<Candidate> cands;
    for (int form : {NQB_FORM_PLAIN, NQB_FORM_BATCHED})
        for (int block : {64, 128, 256}) {
            if (form == NQB_FORM_BATCHED && (base.model || base.sched_cost)) {
                for (int factor : {1, 4, 16}) cands.push_back({form, block, factor});
            } else {
                cands.push_back({form, block, 0});
            }
        }
    NQB_TRY(nqb_device_check(base.device));
    struct Held {  // released on every way out, an exception included
        int prev = 0;
        cudaStream_t s = nullptr;
        unsigned long long* d_out = nullptr;
        ~Held() {
            if (d_out) dev_free(d_out, s);
            if (s) {
                cudaStreamSynchronize(s);
                cudaStreamDestroy(s);
            }
            cudaSetDevice(prev);
        }
    } held;
    cudaGetDevice(&held.prev);
    int st = cuda_status(cudaSetDevice(base.device));
    if (!st) st = cuda_status(cudaStreamCreateWithFlags(&held.s, cudaStreamNonBlocking));
    const cudaStream_t s = held.s;
    if (!st) st = dev_alloc(&held.d_out, 8 * sizeof(unsigned long long) + kBatchedScratchBytes, s);  // results, scratch
    unsigned long long* const d_out = held.d_out;

    out->sample_div = sample_div;
    out->best_ms = -1.0;
    for (unsigned k = 0; k < n_depths && !st; ++k) {
        const unsigned depth = depths[k];
        const unsigned stack_depth = n - depth - 1 > 0 ? n - depth - 1 : 1;
        nqb_state* d_pool = nullptr;
        uint64_t cnt = 0;
        st = generate_pool_device(n, depth, s, &d_pool, &cnt);
        if (st) break;
        const uint64_t m = (cnt + sample_div - 1) / sample_div;
        nqb_state* d_sample = nullptr;
        if (m > (1ull << 31)) st = NQB_E_RANGE;
        if (!st && m) st = dev_alloc(&d_sample, m * sizeof(nqb_state), s);
        if (!st && m) {
            stride_gather_kernel<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(
                reinterpret_cast<const uint4*>(d_pool), m, sample_div, reinterpret_cast<uint4*>(d_sample));
            st = cuda_status(cudaGetLastError());
        }
        dev_free(d_pool, s);
        unsigned long long first = 0;
        for (size_t c = 0; c < cands.size() && !st && m; ++c) {
            double ms = 0.0;
            unsigned long long cnt_c = 0;
            st = time_candidate(d_sample, (uint32_t)m, stack_depth, base, cands[c], base.device, s, d_out, &ms, &cnt_c);
            if (st) break;
            if (c == 0) first = cnt_c;
            else if (cnt_c != first) st = NQB_E_DEVICE;  // candidates must agree on the count
            if (out->n_tried < sizeof(out->tried) / sizeof(out->tried[0])) {
                nqb_tune_entry& e = out->tried[out->n_tried++];
                e.depth = depth;
                e.form = cands[c].form;
                e.block_size = cands[c].block;
                e.split_factor = cands[c].factor;
                e.ms = ms;
            }
            if (out->best_ms < 0 || ms < out->best_ms) {
                out->best_ms = ms;
                out->depth = depth;
                out->form = cands[c].form;
                out->block_size = cands[c].block;
                out->split_factor = cands[c].factor;
                out->sample_states = m;
            }
        }
        if (d_sample) dev_free(d_sample, s);
    }
    return st;
} NQB_ABI_CATCH
