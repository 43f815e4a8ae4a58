// Stream-ordered device memory from the library's own pool, one per device.  Buffers
// freed back to the pool stay mapped (release threshold: no limit), so a call does not
// map and unmap its pool and level buffers again each time; nqb_trim_device_memory
// returns what is cached.
#include <cuda.h>

#include <atomic>
#include <mutex>

#include "nqb_internal.h"

namespace nqb {

// The unique id of the calling thread's current CUDA context (0 when none is current), from
// the driver's cuCtxGetCurrent / cuCtxGetId, reached through the runtime's entry-point
// lookup so the library needs no link against the driver library.  A device reset or a
// torn-down primary context gives the device a new context with a new id, so objects
// cached per device (a memory pool, a symbol's address) are keyed on it.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    return get_id(ctx, &id) == CUDA_SUCCESS ? id : 0;
}

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_pools_mu;
cudaMemPool_t g_pools[kMaxDevices] = {};
unsigned long long g_pool_ctx[kMaxDevices] = {};  // context the pool was created in

int device_pool(int dev, cudaMemPool_t* out) {
    if (dev < 0 || dev >= kMaxDevices) return NQB_E_NODEVICE;
    std::lock_guard<std::mutex> g(g_pools_mu);
    const unsigned long long ctx = current_context_id();
    if (g_pools[dev] && ctx != g_pool_ctx[dev]) g_pools[dev] = nullptr;  // the device was reset: the pool is gone
    if (!g_pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        NQB_TRY(cuda_status(cudaMemPoolCreate(&p, &props)));
        uint64_t keep = UINT64_MAX;
        const int s = cuda_status(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep));
        if (s) {
            cudaMemPoolDestroy(p);
            return s;
        }
        g_pools[dev] = p;
        g_pool_ctx[dev] = current_context_id();
    }
    *out = g_pools[dev];
    return NQB_OK;
}

}  // namespace

// Allocations left before the one that fails; -1: the hook is off (nqb_debug_fail_allocation).
std::atomic<long long> g_fail_countdown{-1};

bool alloc_fault() {
    long long v = g_fail_countdown.load(std::memory_order_relaxed);
    while (v >= 0) {  // count this allocation down; the one that takes the countdown to -1 fails
        if (g_fail_countdown.compare_exchange_weak(v, v - 1, std::memory_order_relaxed)) return v == 0;
    }
    return false;
}

int dev_alloc_bytes(void** p, size_t bytes, cudaStream_t s) {
    *p = nullptr;
    if (alloc_fault()) return NQB_E_NOMEM;
    int dev = 0;
    NQB_TRY(cuda_status(cudaGetDevice(&dev)));
    cudaMemPool_t pool = nullptr;
    NQB_TRY(device_pool(dev, &pool));
    return cuda_status(cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, s));
}

void dev_free(void* p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

}  // namespace nqb

extern "C" long long nqb_debug_fail_allocation(long long after) {
    return nqb::g_fail_countdown.exchange(after < 0 ? -1 : after);
}

extern "C" int nqb_trim_device_memory(int device) {
    if (device < 0 || device >= nqb::kMaxDevices) return NQB_E_NODEVICE;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return NQB_E_NODEVICE;
    NQB_TRY(nqb::cuda_status(cudaSetDevice(device)));
    const unsigned long long ctx = nqb::current_context_id();
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> g(nqb::g_pools_mu);
        if (nqb::g_pools[device] && nqb::g_pool_ctx[device] == ctx) pool = nqb::g_pools[device];
    }
    const int s = pool ? nqb::cuda_status(cudaMemPoolTrimTo(pool, 0)) : NQB_OK;
    cudaSetDevice(prev);
    return s;
}
