#include "devmem.hpp"

#include <cstdint>
#include <mutex>

namespace tycho {

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxDevices] = {};

// The pool of the current device, made on first use.  Freed memory stays in
// the pool for the next allocation (release threshold: no limit), like a
// caching allocator: returning tens of GB to the system and mapping them
// again for the next problem took hundreds of milliseconds per problem.
// dev_trim hands the unused part back.
cudaError_t pool_of_current(cudaMemPool_t *out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pool[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        e = cudaMemPoolCreate(&g_pool[dev], &props);
        if (e != cudaSuccess) {
            g_pool[dev] = nullptr;
            return e;
        }
        uint64_t keep = ~0ull;
        e = cudaMemPoolSetAttribute(g_pool[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
    }
    *out = g_pool[dev];
    return cudaSuccess;
}

}  // namespace

cudaError_t dev_malloc(void **p, size_t bytes, cudaStream_t s)
{
    *p = nullptr;
    cudaMemPool_t pool;
    cudaError_t e = pool_of_current(&pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, s);
}

void dev_free(void *p, cudaStream_t s)
{
    if (p) cudaFreeAsync(p, s);
}

cudaError_t dev_trim(int device)
{
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        pool = g_pool[device];
    }
    if (!pool) return cudaSuccess;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();  // frees still in flight land first
    if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, 0);
    return e;
}

cudaError_t dev_pool_usage(int device, uint64_t *reserved, uint64_t *used)
{
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        pool = g_pool[device];
    }
    uint64_t r = 0, u = 0;
    cudaError_t e = cudaSuccess;
    if (pool) {
        e = cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r);
        if (e == cudaSuccess) e = cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u);
    }
    if (reserved) *reserved = r;
    if (used) *used = u;
    return e;
}

}  // namespace tycho
