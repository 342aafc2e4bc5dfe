// Device memory of sweepers and batches: one stream-ordered pool per device
// (cudaMallocFromPoolAsync / cudaFreeAsync).  Unlike cudaFree, freeing into
// the pool never waits for the whole device, so a solve service can build
// and retire problems while the sweeps of other problems keep running.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace tycho {

// Allocates `bytes` (at least 1) on the current device, ordered on stream s;
// the memory may be used on other streams once s has passed the allocation.
cudaError_t dev_malloc(void **p, size_t bytes, cudaStream_t s);
template <typename T>
cudaError_t dev_malloc(T **p, size_t bytes, cudaStream_t s)
{
    return dev_malloc(reinterpret_cast<void **>(p), bytes, s);
}
// Returns p (may be null) to the pool once stream s reaches this point; no
// other stream may still use it.
void dev_free(void *p, cudaStream_t s);
template <typename T>
void dev_release(T *&p, cudaStream_t s)
{
    dev_free(p, s);
    p = nullptr;
}

// Returns the pool's unused memory on `device` to the system (waits for the
// device first).
cudaError_t dev_trim(int device);

// Bytes the pool of `device` holds from the system and bytes of it in use
// (both 0 before its first allocation).
cudaError_t dev_pool_usage(int device, uint64_t *reserved, uint64_t *used);

}  // namespace tycho
