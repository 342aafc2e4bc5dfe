// Device-side levelling of every (cell, angle) item: the GPU form of
// build_schedule (schedule.cpp), with the same result -- t-levels, the
// (level, octant, cell*A + angle) item order with each (level, octant)
// segment padded to a multiple of 32, and the incoming-face count.
//
// Per direction the reference walks the cell graph with priority queues
// (src/GraphTraverser.cc:467-759); here all directions advance together one
// frontier per level (Kahn's algorithm): an item enters level L + 1 when the
// last of its upwind neighbours leaves level L, which makes its level the
// longest upwind chain ending at it.  Compiled with -fmad=false: omega.n is
// formed exactly as on the host (src/TychoMesh.cc:212-223).
#include <cub/device/device_radix_sort.cuh>

#include "devmem.hpp"
#include "schedule.hpp"
#include "status.hpp"
#include "trace.hpp"

namespace tycho {

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kMaxLevels = 1u << 16;    // frontier counters kept on the device
constexpr uint32_t kLevelBatch = 32;         // level steps launched between host checks
constexpr unsigned kStepGrid = 148 * 8;      // blocks of the grid-stride level step

// Appends v where pred holds to buf, with one atomic per warp for the slots
// (lanes active at the call take part; pred false appends nothing).
__device__ __forceinline__ void warp_append(bool pred, uint32_t v, uint32_t *buf, uint32_t *count)
{
    const unsigned active = __activemask();
    const unsigned ballot = __ballot_sync(active, pred);
    if (!ballot) return;
    const int leader = __ffs(ballot) - 1;
    const unsigned lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(count, (uint32_t)__popc(ballot));
    base = __shfl_sync(active, base, leader);
    if (pred) buf[base + __popc(ballot & ((1u << lane) - 1u))] = v;
}

// Per item (angle-major index a*nc + c): upwind mask (bits 0-3), downwind
// mask (bits 4-7), count of upwind interior faces; level-0 items seed the
// frontier.  Faces with omega.n == 0 carry no flux and order nothing (see
// flux_mask in schedule.cpp).
__global__ void level_init_kernel(const double *__restrict__ normal, const int4 *__restrict__ adj,
                                  const double *__restrict__ omega, uint32_t A, uint64_t nc,
                                  uint8_t *__restrict__ mask, uint32_t *__restrict__ cnt,
                                  uint32_t *__restrict__ tlevel, uint32_t *__restrict__ frontier,
                                  uint32_t *__restrict__ n_frontier, unsigned long long *__restrict__ incoming)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)A * nc) return;  // whole warps past the end, or a tail the intrinsics below mask out
    const uint32_t a = (uint32_t)(i / nc);
    const uint64_t c = i - (uint64_t)a * nc;
    const double xi = omega[a], eta = omega[A + a], mu = omega[2 * A + a];
    const int4 nb = adj[c];
    const int nbs[4] = {nb.x, nb.y, nb.z, nb.w};
    unsigned m = 0;
    uint32_t d = 0;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const double *n = normal + (c * 4 + f) * 3;
        const double odn = xi * n[0] + eta * n[1] + mu * n[2];
        if (odn < 0) {
            m |= 1u << f;
            if (nbs[f] >= 0) ++d;
        }
        if (odn > 0) m |= 16u << f;
    }
    mask[i] = (uint8_t)m;
    cnt[i] = d;
    if (!d) tlevel[i] = 0;
    // one atomic per warp for the incoming-face total and the frontier slots
    const unsigned active = __activemask();
    const unsigned wsum = __reduce_add_sync(active, d);
    if ((threadIdx.x & 31u) == (unsigned)(__ffs(active) - 1)) atomicAdd(incoming, (unsigned long long)wsum);
    warp_append(d == 0, (uint32_t)i, frontier, n_frontier);
}

// One level: every frontier item releases its downwind neighbours; the last
// release of a neighbour puts it on the next frontier one level higher.  The
// frontier's size is read on the device (level_count[level]), so the host
// launches many levels without waiting for each; a level past the last
// non-empty one has nothing to do.
__global__ void level_step_kernel(const uint32_t *__restrict__ frontier, uint32_t level,
                                  const int4 *__restrict__ adj, const uint8_t *__restrict__ mask, uint64_t nc,
                                  uint32_t *__restrict__ cnt, uint32_t *__restrict__ tlevel,
                                  uint32_t *__restrict__ next, uint32_t *__restrict__ level_count)
{
    const uint32_t n = level_count[level];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t i = frontier[k];
        const uint64_t a = i / nc, c = i - a * nc;
        const int4 nb = adj[c];
        const int nbs[4] = {nb.x, nb.y, nb.z, nb.w};
        const unsigned m = mask[i];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const bool down = (m >> (f + 4) & 1u) && nbs[f] >= 0;
            const uint64_t j = a * nc + (uint64_t)(down ? nbs[f] : 0);
            const bool ready = down && atomicSub(&cnt[j], 1u) == 1u;
            if (ready) tlevel[j] = level + 1;
            warp_append(ready, (uint32_t)j, next, level_count + level + 1);
        }
    }
}

// Sort keys in (cell*A + angle) order: level * 8 + octant.
__global__ void level_keys_kernel(const uint32_t *__restrict__ tlevel, const uint8_t *__restrict__ oct, uint32_t A,
                                  uint64_t nc, uint32_t *__restrict__ keys, uint32_t *__restrict__ vals)
{
    const uint64_t ca = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ca >= (uint64_t)A * nc) return;
    const uint64_t c = ca / A, a = ca - c * A;
    keys[ca] = tlevel[a * nc + c] * (uint32_t)kOctants + oct[a];
    vals[ca] = (uint32_t)ca;
}

// Sorted item j (key k) goes to padded[k] + (j - unpadded[k]).
__global__ void level_scatter_kernel(const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals,
                                     uint64_t n, const uint64_t *__restrict__ unpadded,
                                     const uint64_t *__restrict__ padded, uint32_t *__restrict__ items)
{
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t k = keys[j];
    items[padded[k] + (j - unpadded[k])] = vals[j];
}

// Segment starts of sorted keys: start[s] = the first j with keys[j] >= s,
// for s in [0, nseg]; each s is written by exactly one j (no atomics: sorted
// keys would put every lane of a warp on the same counter).
__global__ void seg_starts_kernel(const uint32_t *__restrict__ keys, uint64_t n, uint32_t nseg,
                                  uint64_t *__restrict__ start)
{
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t k = keys[j];
    const uint32_t prev_end = j == 0 ? 0u : keys[j - 1] + 1u;  // s in [prev_end, k] starts at j
    for (uint32_t s = prev_end; s <= k && s <= nseg; ++s) start[s] = j;
    if (j == n - 1)
        for (uint32_t s = k + 1; s <= nseg; ++s) start[s] = n;
}

// Key of schedule position i for the angle-chunked sweep: chunk(angle) *
// n_levels + level(i), or the trailing bucket K * n_levels for padding.  The
// level of position i is found by bisection of the level offsets.
__global__ void chunk_keys_kernel(const uint32_t *__restrict__ items, uint64_t n_padded,
                                  const uint64_t *__restrict__ level_off, uint32_t n_levels, uint32_t A,
                                  uint32_t K, uint32_t *__restrict__ keys, uint32_t *__restrict__ vals)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_padded) return;
    const uint32_t ca = items[i];
    uint32_t key = K * n_levels;
    if (ca != 0xFFFFFFFFu) {
        uint32_t lo = 0, hi = n_levels;  // level_off[lo] <= i < level_off[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (level_off[mid] <= i) lo = mid;
            else hi = mid;
        }
        const uint32_t a = ca % A;
        key = (uint32_t)(((uint64_t)a * K) / A) * n_levels + lo;
    }
    keys[i] = key;
    vals[i] = (uint32_t)i;
}

unsigned blocks_for(uint64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// A temporary from the stream-ordered pool, returned on scope exit.
struct DevBuf {
    void *p = nullptr;
    cudaStream_t s = nullptr;
    ~DevBuf() { dev_free(p, s); }
};

cudaError_t take(DevBuf &b, size_t bytes, cudaStream_t st)
{
    b.s = st;
    return dev_malloc(&b.p, bytes, st);
}

}  // namespace

#define TS_CUDA(expr)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (expr);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            err = std::string(#expr) + ": " + cudaGetErrorString(e_);                  \
            return e_ == cudaErrorMemoryAllocation ? kErrOom : kErrCuda;               \
        }                                                                              \
    } while (0)

#define TS_CHECK_HOST(expr)                                                            \
    do {                                                                               \
        const int st_ = (expr);                                                        \
        if (st_ != kOk) return st_;                                                    \
    } while (0)

int build_schedule_device(const MeshTables &t, const Quadrature &q, Schedule &s, uint32_t **d_items_out,
                          cudaStream_t st, std::string &err)
{
    const uint64_t nc = t.n_cells;
    const uint32_t A = (uint32_t)q.n_angles;
    const uint64_t n = (uint64_t)A * nc;
    if (n >= (1ull << 32) || nc >= (1ull << 31)) {
        err = "cells x angles exceeds 2^32 items";
        return kErrArg;
    }
    if (n == 0) {
        TS_CHECK_HOST(build_schedule(t, q, s, err));
        if (d_items_out) {
            *d_items_out = nullptr;
            s.items.clear();
            s.tlevel.clear();
        }
        return kOk;
    }
    s = Schedule();
    std::vector<int4> adj(nc);
    for (uint64_t c = 0; c < nc; ++c) {
        int v[4];
        for (int f = 0; f < 4; ++f) {
            const uint64_t nb = t.adj_cell[c * 4 + f];
            v[f] = nb == kNone ? -1 : (int)nb;
        }
        adj[c] = make_int4(v[0], v[1], v[2], v[3]);
    }
    std::vector<double> omega(3 * (size_t)A);
    std::vector<uint8_t> oct(A);
    TraceScope trace_prep("levelling.upload_init");
    for (uint32_t a = 0; a < A; ++a) {
        omega[a] = q.xi[a];
        omega[A + a] = q.eta[a];
        omega[2 * A + a] = q.mu[a];
        oct[a] = (uint8_t)octant(q, (int)a);
    }
    DevBuf d_normal, d_adj, d_omega, d_oct, d_mask, d_cnt, d_tlevel, d_front[2], d_ctr, d_inc;
    TS_CUDA(take(d_normal, sizeof(double) * t.normal.size(), st));
    TS_CUDA(take(d_adj, sizeof(int4) * nc, st));
    TS_CUDA(take(d_omega, sizeof(double) * omega.size(), st));
    TS_CUDA(take(d_oct, A, st));
    TS_CUDA(take(d_mask, n, st));
    TS_CUDA(take(d_cnt, sizeof(uint32_t) * n, st));
    TS_CUDA(take(d_tlevel, sizeof(uint32_t) * n, st));
    TS_CUDA(take(d_front[0], sizeof(uint32_t) * n, st));
    TS_CUDA(take(d_front[1], sizeof(uint32_t) * n, st));
    TS_CUDA(take(d_ctr, sizeof(uint32_t) * (kMaxLevels + 1), st));  // frontier size per level
    TS_CUDA(take(d_inc, sizeof(unsigned long long), st));
    TS_CUDA(cudaMemcpyAsync(d_normal.p, t.normal.data(), sizeof(double) * t.normal.size(), cudaMemcpyHostToDevice, st));
    TS_CUDA(cudaMemcpyAsync(d_adj.p, adj.data(), sizeof(int4) * nc, cudaMemcpyHostToDevice, st));
    TS_CUDA(cudaMemcpyAsync(d_omega.p, omega.data(), sizeof(double) * omega.size(), cudaMemcpyHostToDevice, st));
    TS_CUDA(cudaMemcpyAsync(d_oct.p, oct.data(), A, cudaMemcpyHostToDevice, st));
    TS_CUDA(cudaMemsetAsync(d_ctr.p, 0, sizeof(uint32_t) * (kMaxLevels + 1), st));
    TS_CUDA(cudaMemsetAsync(d_inc.p, 0, sizeof(unsigned long long), st));
    uint32_t *ctr = (uint32_t *)d_ctr.p;
    level_init_kernel<<<blocks_for(n), kThreads, 0, st>>>(
        (const double *)d_normal.p, (const int4 *)d_adj.p, (const double *)d_omega.p, A, nc, (uint8_t *)d_mask.p,
        (uint32_t *)d_cnt.p, (uint32_t *)d_tlevel.p, (uint32_t *)d_front[0].p, ctr,
        (unsigned long long *)d_inc.p);
    TS_CUDA(cudaGetLastError());
    trace_prep.next("levelling.frontiers");
    // Levels in batches of kLevelBatch launches, each reading its frontier's
    // size on the device; between batches the host reads the batch's sizes
    // and stops at the first empty level.
    uint64_t done = 0;
    uint32_t level = 0;  // number of non-empty levels found so far
    std::vector<uint32_t> h_cnt(kLevelBatch);
    for (bool more = true; more;) {
        if (level + kLevelBatch > kMaxLevels) {
            err = "more than 65536 wavefront levels";
            return kErrArg;
        }
        for (uint32_t b = 0; b < kLevelBatch; ++b) {
            const uint32_t l = level + b;
            level_step_kernel<<<kStepGrid, kThreads, 0, st>>>(
                (const uint32_t *)d_front[l & 1u].p, l, (const int4 *)d_adj.p, (const uint8_t *)d_mask.p, nc,
                (uint32_t *)d_cnt.p, (uint32_t *)d_tlevel.p, (uint32_t *)d_front[(l + 1) & 1u].p, ctr);
        }
        TS_CUDA(cudaGetLastError());
        TS_CUDA(cudaMemcpyAsync(h_cnt.data(), ctr + level, sizeof(uint32_t) * kLevelBatch, cudaMemcpyDeviceToHost,
                                st));
        TS_CUDA(cudaStreamSynchronize(st));
        for (uint32_t b = 0; b < kLevelBatch; ++b) {
            if (h_cnt[b] == 0) {
                more = false;
                break;
            }
            done += h_cnt[b];
            ++level;
        }
    }
    if (done != n) {
        err = "a direction's cell dependency graph has a cycle";
        return kErrCycle;
    }
    trace_prep.next("levelling.sort_scatter");
    s.n_levels = level;
    s.n_items = n;
    unsigned long long inc = 0;
    TS_CUDA(cudaMemcpyAsync(&inc, d_inc.p, sizeof inc, cudaMemcpyDeviceToHost, st));
    // (level, octant, cell*A + angle) order: a stable radix sort of the keys
    // of the items taken in cell*A + angle order
    DevBuf d_keys[2], d_vals[2], d_temp, d_hist, d_unpad, d_pad, d_items;
    for (int k = 0; k < 2; ++k) {
        TS_CUDA(take(d_keys[k], sizeof(uint32_t) * n, st));
        TS_CUDA(take(d_vals[k], sizeof(uint32_t) * n, st));
    }
    level_keys_kernel<<<blocks_for(n), kThreads, 0, st>>>((const uint32_t *)d_tlevel.p, (const uint8_t *)d_oct.p, A,
                                                          nc, (uint32_t *)d_keys[0].p, (uint32_t *)d_vals[0].p);
    TS_CUDA(cudaGetLastError());
    const uint64_t nseg = (uint64_t)s.n_levels * kOctants;
    int end_bit = 1;
    while (end_bit < 32 && (1ull << end_bit) < nseg) ++end_bit;
    cub::DoubleBuffer<uint32_t> kb((uint32_t *)d_keys[0].p, (uint32_t *)d_keys[1].p);
    cub::DoubleBuffer<uint32_t> vb((uint32_t *)d_vals[0].p, (uint32_t *)d_vals[1].p);
    size_t temp = 0;
    TS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, kb, vb, (int64_t)n, 0, end_bit, st));
    TS_CUDA(take(d_temp, temp, st));
    TS_CUDA(cub::DeviceRadixSort::SortPairs(d_temp.p, temp, kb, vb, (int64_t)n, 0, end_bit, st));
    // segment starts (unpadded offsets), then padded offsets
    TS_CUDA(take(d_hist, sizeof(uint64_t) * (nseg + 1), st));
    seg_starts_kernel<<<blocks_for(n), kThreads, 0, st>>>(kb.Current(), n, (uint32_t)nseg, (uint64_t *)d_hist.p);
    TS_CUDA(cudaGetLastError());
    std::vector<uint64_t> unpadded(nseg + 1);
    TS_CUDA(cudaMemcpyAsync(unpadded.data(), d_hist.p, sizeof(uint64_t) * (nseg + 1), cudaMemcpyDeviceToHost, st));
    TS_CUDA(cudaStreamSynchronize(st));
    s.octant_offset.resize(nseg + 1);
    s.octant_offset[0] = 0;
    for (uint64_t k = 0; k < nseg; ++k) {
        const uint64_t cnt = unpadded[k + 1] - unpadded[k];
        s.octant_offset[k + 1] = s.octant_offset[k] + (cnt + kLevelPad - 1) / kLevelPad * kLevelPad;
    }
    s.level_offset.resize(s.n_levels + 1);
    for (uint32_t l = 0; l <= s.n_levels; ++l) s.level_offset[l] = s.octant_offset[(size_t)l * kOctants];
    const uint64_t total = s.level_offset[s.n_levels];
    TS_CUDA(take(d_unpad, sizeof(uint64_t) * (nseg + 1), st));
    TS_CUDA(take(d_pad, sizeof(uint64_t) * (nseg + 1), st));
    TS_CUDA(take(d_items, sizeof(uint32_t) * total, st));
    TS_CUDA(cudaMemcpyAsync(d_unpad.p, unpadded.data(), sizeof(uint64_t) * (nseg + 1), cudaMemcpyHostToDevice, st));
    TS_CUDA(cudaMemcpyAsync(d_pad.p, s.octant_offset.data(), sizeof(uint64_t) * (nseg + 1), cudaMemcpyHostToDevice,
                            st));
    TS_CUDA(cudaMemsetAsync(d_items.p, 0xFF, sizeof(uint32_t) * total, st));  // kSentinelItem
    level_scatter_kernel<<<blocks_for(n), kThreads, 0, st>>>(kb.Current(), vb.Current(), n,
                                                             (const uint64_t *)d_unpad.p, (const uint64_t *)d_pad.p,
                                                             (uint32_t *)d_items.p);
    TS_CUDA(cudaGetLastError());
    s.n_padded = total;
    s.n_incoming_interior = inc;
    if (d_items_out) {
        TS_CUDA(cudaStreamSynchronize(st));
        *d_items_out = (uint32_t *)d_items.p;
        d_items.p = nullptr;
        return kOk;
    }
    s.items.resize(total);
    s.tlevel.resize(n);
    TS_CUDA(cudaMemcpyAsync(s.items.data(), d_items.p, sizeof(uint32_t) * total, cudaMemcpyDeviceToHost, st));
    TS_CUDA(cudaMemcpyAsync(s.tlevel.data(), d_tlevel.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st));
    TS_CUDA(cudaStreamSynchronize(st));
    return kOk;
}

int angle_chunks_device(const uint32_t *d_items, uint64_t n_padded, const uint64_t *d_level_off, uint32_t n_levels,
                        uint32_t A, uint32_t K, uint32_t **d_pos_out, std::vector<uint64_t> &off, cudaStream_t st,
                        std::string &err)
{
    *d_pos_out = nullptr;
    const uint64_t nseg = (uint64_t)K * n_levels;
    off.assign(nseg + 1, 0);
    if (n_padded == 0 || K == 0 || K > A) {
        err = "angle chunks: empty schedule or more chunks than angles";
        return kErrArg;
    }
    DevBuf d_keys[2], d_vals[2], d_temp, d_hist;
    for (int k = 0; k < 2; ++k) {
        TS_CUDA(take(d_keys[k], sizeof(uint32_t) * n_padded, st));
        TS_CUDA(take(d_vals[k], sizeof(uint32_t) * n_padded, st));
    }
    chunk_keys_kernel<<<blocks_for(n_padded), kThreads, 0, st>>>(d_items, n_padded, d_level_off, n_levels, A, K,
                                                                (uint32_t *)d_keys[0].p, (uint32_t *)d_vals[0].p);
    TS_CUDA(cudaGetLastError());
    int end_bit = 1;
    while (end_bit < 32 && (1ull << end_bit) <= nseg) ++end_bit;
    cub::DoubleBuffer<uint32_t> kb((uint32_t *)d_keys[0].p, (uint32_t *)d_keys[1].p);
    cub::DoubleBuffer<uint32_t> vb((uint32_t *)d_vals[0].p, (uint32_t *)d_vals[1].p);
    size_t temp = 0;
    TS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, kb, vb, (int64_t)n_padded, 0, end_bit, st));
    TS_CUDA(take(d_temp, temp, st));
    TS_CUDA(cub::DeviceRadixSort::SortPairs(d_temp.p, temp, kb, vb, (int64_t)n_padded, 0, end_bit, st));
    // starts of the nseg chunk-level segments (keys nseg: the padding, last)
    TS_CUDA(take(d_hist, sizeof(uint64_t) * (nseg + 1), st));
    seg_starts_kernel<<<blocks_for(n_padded), kThreads, 0, st>>>(kb.Current(), n_padded, (uint32_t)nseg,
                                                                 (uint64_t *)d_hist.p);
    TS_CUDA(cudaGetLastError());
    TS_CUDA(cudaMemcpyAsync(off.data(), d_hist.p, sizeof(uint64_t) * (nseg + 1), cudaMemcpyDeviceToHost, st));
    TS_CUDA(cudaStreamSynchronize(st));
    // the sorted positions (the padding bucket sorts last and is not used)
    DevBuf &cur = vb.Current() == (uint32_t *)d_vals[0].p ? d_vals[0] : d_vals[1];
    *d_pos_out = (uint32_t *)cur.p;
    cur.p = nullptr;
    return kOk;
}

}  // namespace tycho
