// Stream-ordered device memory from the library's own pool, one per device.  Buffers
// freed back to the pool stay mapped (release threshold: no limit), so a call does not
// map and unmap its pool and level buffers again each time; nqb_trim_device_memory
// returns what is cached.
#include <mutex>

#include "nqb_internal.h"

namespace nqb {
namespace {

constexpr int kMaxDevices = 64;
std::mutex g_pools_mu;
cudaMemPool_t g_pools[kMaxDevices] = {};

int device_pool(int dev, cudaMemPool_t* out) {
    if (dev < 0 || dev >= kMaxDevices) return NQB_E_NODEVICE;
    std::lock_guard<std::mutex> g(g_pools_mu);
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
    }
    *out = g_pools[dev];
    return NQB_OK;
}

}  // namespace

int dev_alloc_bytes(void** p, size_t bytes, cudaStream_t s) {
    *p = nullptr;
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

extern "C" int nqb_trim_device_memory(int device) {
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> g(nqb::g_pools_mu);
        if (device < 0 || device >= nqb::kMaxDevices) return NQB_E_NODEVICE;
        pool = nqb::g_pools[device];
    }
    if (!pool) return NQB_OK;
    return nqb::cuda_status(cudaMemPoolTrimTo(pool, 0));
}
