// The sweep entry point that allocates nothing (tycho_sweeper_sweep_noalloc).
//
// Some callers cannot allocate device memory at the moment they need a sweep:
// a host framework that owns all device memory through its own pool and
// budget (a serving loop admitting work by its HBM footprint cannot tolerate
// hidden allocations), a plugin that may only use the buffers its host hands
// it, or a time-critical loop where cudaMalloc's implicit synchronization
// would stall every stream.  For them the persistent dataflow sweep runs on
// the caller's own source and psi buffers, and its scratch -- the per-item
// completion flags and the control words -- lives in one file-scope device
// array of fixed size instead of memory the sweeper allocates.
//
// Limits and sharing, as documented in include/tycho_cuda.h:
//   * at most kNoAllocMaxItems (cells x angles) items; larger problems are
//     rejected with TYCHO_ERR_ARG;
//   * every GPU that loads the library holds the array until the process
//     exits; its device address is looked up when a sweeper is created on
//     that device (Sweeper::init), which also loads the module that holds
//     it, so the sweep calls themselves map and load nothing;
//   * all calls share the array; calls that overlap on the GPU race;
//   * a call reads its error words back and synchronizes its stream.
#include <cstring>
#include <mutex>

#include "status.hpp"
#include "sweeper.hpp"

namespace tycho {

constexpr uint64_t kNoAllocMaxItems = 1ull << 24;   // 16,777,216 (cell, angle) items
constexpr uint64_t kNoAllocCtlWords = 64;           // control block after the flags
constexpr int kNoAllocMaxDevices = 64;

// Completion flags for kNoAllocMaxItems items, then the control block
// ([0..2] error, [3] abort, [4] epoch).  64 MiB + 256 B per device.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocMaxItems + kNoAllocCtlWords];

namespace {

std::mutex g_scratch_mu;
uint32_t *g_scratch_addr[kNoAllocMaxDevices] = {};

// The device address of the scratch array on the current device, looked up
// once per device.  In host code the array's name is only a host-side
// stand-in, so kernels must be given this address instead.
int scratch_address(int device, uint32_t **out, std::string &err)
{
    if (device < 0 || device >= kNoAllocMaxDevices) {
        err = "device ordinal out of range for the no-alloc scratch table";
        return kErrArg;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            err = std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e);
            return kErrCuda;
        }
        g_scratch_addr[device] = static_cast<uint32_t *>(p);
    }
    *out = g_scratch_addr[device];
    return kOk;
}

// Clears the error and abort words left by the previous call and advances
// the shared epoch, so flags from any earlier call (of any sweeper) never
// match this one.
__global__ void noalloc_begin_kernel(uint32_t *ctl)
{
    ctl[0] = 0u;
    ctl[1] = 0u;
    ctl[2] = 0u;
    ctl[3] = 0u;
    const uint32_t v = ctl[4] + 1u;
    ctl[4] = v == 0u ? 1u : v;
}

}  // namespace

int noalloc_scratch_prepare(int device, std::string &err)
{
    uint32_t *base = nullptr;
    return scratch_address(device, &base, err);
}

int Sweeper::sweep_external(int prec, const void *iso, void *psi, uint32_t *done, uint32_t *ctl,
                            cudaStream_t s, std::string &err)
{
    if (prec == 1 && !fp32_) { err = "sweeper was created without the FP32 sweep"; return kErrArg; }
    if (!have_xs_) { err = "cross sections not set"; return kErrMissing; }
    if (!psi) { err = "psi buffer is required"; return kErrArg; }
    if (n_bound_sides()) { err = "faces toward other partitions: no no-alloc sweep"; return kErrArg; }
    if (solver_ != kSolveNoPivot) {
        err = "the no-alloc sweep runs the NoPivot solver only (GaussElim NoPivot)";
        return kErrArg;
    }
    if ((reinterpret_cast<uintptr_t>(psi) | reinterpret_cast<uintptr_t>(iso)) % 16u != 0) {
        err = "psi and iso must be 16-byte aligned (the sweep moves groups as vectors)";
        return kErrArg;
    }
    const LevelArgs p = level_args(prec, iso, nullptr, psi);
    DataflowArgs df;
    df.done = done;
    df.err = ctl;
    df.abort = ctl + 3;
    df.epoch = ctl + 4;
    df.n_items = sched_.n_padded;
    df.spin_limit = spin_limit_;
    cudaError_t e = cudaSetDevice(device_);
    if (e == cudaSuccess) {
        noalloc_begin_kernel<<<1, 1, 0, s>>>(ctl);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        err = std::string("no-alloc sweep: ") + cudaGetErrorString(e);
        return kErrCuda;
    }
    // The record and direct-record shapes sweep with the per-item records,
    // which tycho_sweeper_configure allocated; this call never allocates them.
    // Stale ones (new cross sections) are recomputed in place on `s`.
    const LaunchShape &sh = shape_[prec ? 1 : 0];
    if (sh.variant == 2 || sh.variant == 3) {
        const int k = prec ? 1 : 0;
        if (!d_rec_[k]) {
            err = "no-alloc sweep: the launch shape's per-item records were never allocated";
            return kErrMissing;
        }
        if (!rec_valid_[k]) {
            const LevelArgs rp = level_args(prec, nullptr, nullptr, d_psi_);
            e = prec ? launch_item_records<float>(rp, sched_.n_padded, d_rec_[1], s)
                     : launch_item_records<double>(rp, sched_.n_padded, d_rec_[0], s);
            if (e != cudaSuccess) {
                err = std::string("no-alloc sweep (records): ") + cudaGetErrorString(e);
                return kErrCuda;
            }
            rec_valid_[k] = true;
        }
    }
    const int st = launch_dataflow_shape(prec, p, df, s, err);
    if (st != kOk) return st;
    uint32_t word[3] = {0, 0, 0};
    e = cudaMemcpyAsync(word, ctl, sizeof word, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        err = std::string("no-alloc sweep: ") + cudaGetErrorString(e);
        return kErrCuda;
    }
    if (word[0] != 0) {
        err = "sweep wait timed out at item " + std::to_string(word[1]) + " face " + std::to_string(word[2]);
        return kErrTimeout;
    }
    return kOk;
}

}  // namespace tycho

namespace tycho {

int sweep_noalloc(Sweeper &sw, int precision, const void *iso, void *psi, void *stream, std::string &err)
{
    const uint64_t items = sw.n_cells() * (uint64_t)sw.n_angles();
    if (precision != 0 && precision != 1) {
        err = "precision must be 0 (FP64) or 1 (FP32)";
        return kErrArg;
    }
    if (items > kNoAllocMaxItems) {
        err = "no-alloc sweep takes at most " + std::to_string(kNoAllocMaxItems) +
              " cells x angles; this sweeper has " + std::to_string(items);
        return kErrArg;
    }
    cudaError_t e = cudaSetDevice(sw.device());
    if (e != cudaSuccess) {
        err = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
        return kErrCuda;
    }
    uint32_t *base = nullptr;
    int st = scratch_address(sw.device(), &base, err);
    if (st != kOk) return st;
    return sw.sweep_external(precision, iso, psi, base, base + kNoAllocMaxItems,
                             static_cast<cudaStream_t>(stream), err);
}

}  // namespace tycho
