// Batched sweep of many independent instances (uneven mesh size, group
// count and SN order) in one set of launches.  There is no counterpart in
// the reference, which sweeps one problem per process.
//
// Each pass (one operator application of every active member, in one
// precision) is one CUDA graph:
//   plan        device work list over (member, wavefront level): per level,
//               the active members' record ranges as segments with chunk
//               prefixes; per member, its phi chunks
//   accept      phi += delta for members that finished an inner solve
//   scatter     iso = [Q] + M S phi_in                   (per phi element)
//   level L     one launch per global level L = 0..max levels - 1: every
//               warp takes IPW-item chunks of the level's work list, finds
//               its member by binary search over the segments, and runs the
//               record kernel's per-(item, group) arithmetic for that member
//   psi->phi    phi_out = sum_a w_a psi
//   post        per member operation (SI change, residual, inner update)
//               with per-chunk partial L1 sums
//   finish      per member: its partials in chunk order -> two norms
// Chunks are member-local (kChunk phi elements of one member), so every
// member's arithmetic and reductions are the same alone and in any mix.
#pragma once

#include "batch_types.hpp"
#include "sweep_records.cuh"
#include "stream_ops.cuh"

namespace tycho {

constexpr int kBatchPlanThreads = 256;

__host__ __device__ __forceinline__ uint32_t batch_class(uint32_t vg) { return vg == 4 ? 2u : vg == 2 ? 1u : 0u; }

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *total)
{
    __shared__ uint32_t warp_tot[kBatchPlanThreads / 32];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    uint32_t base = 0, all = 0;
    for (uint32_t k = 0; k < kBatchPlanThreads / 32; ++k) {
        if (k < w) base += warp_tot[k];
        all += warp_tot[k];
    }
    __syncthreads();
    *total = all;
    return base + x - v;
}

// Grid: max levels + 1 blocks of kBatchPlanThreads.  Block L < max levels
// builds level L's segments, one list per vector-width class (members of a
// class run the same kernel body); the last block lists the active members
// and their phi chunk prefix.
template <int IPW>
__global__ void __launch_bounds__(kBatchPlanThreads)
batch_plan_kernel(const BatchSlot *__restrict__ slots, uint32_t n_slots, uint32_t max_levels, uint32_t rec_bytes,
                  BatchPlan pl)
{
    const uint32_t L = blockIdx.x;
    if (L < max_levels) {
        for (uint32_t cls = 0; cls < kBatchClasses; ++cls) {
            uint32_t chunk_run = 0, seg_run = 0;
            BatchSeg *segs = pl.segs + ((size_t)L * kBatchClasses + cls) * pl.seg_stride;
            for (uint32_t base = 0; base < n_slots; base += kBatchPlanThreads) {
                const uint32_t j = base + threadIdx.x;
                uint32_t nch = 0;
                uint64_t lo = 0;
                const uint32_t sh = j < n_slots ? slots[j].level_shift : 0u;
                if (j < n_slots && slots[j].active && L >= sh && L - sh < slots[j].n_levels &&
                    batch_class(slots[j].vg) == cls) {
                    lo = slots[j].level_off[L - sh];
                    const uint64_t items = slots[j].level_off[L - sh + 1] - lo;
                    // IPW items per chunk; IPW == 0 (direct kernel): 32 (item, group vector) tasks
                    nch = IPW ? (uint32_t)(items / IPW) : (uint32_t)(items / 32 * (slots[j].G / slots[j].vg));
                }
                uint32_t tot_c, tot_s;
                const uint32_t ex_c = block_exclusive_scan(nch, &tot_c);
                const uint32_t ex_s = block_exclusive_scan(nch ? 1u : 0u, &tot_s);
                if (nch) {
                    const BatchSlot &sl = slots[j];
                    BatchSeg sg;
                    sg.rec = (const char *)sl.rec + lo * rec_bytes;
                    sg.psi = sl.psi;
                    sg.iso = sl.iso32 ? (const void *)sl.iso32 : (const void *)sl.iso;
                    sg.item_begin = lo;
                    sg.slot = j;
                    sg.chunk_begin = chunk_run + ex_c;
                    sg.G = sl.G;
                    sg.vmagic = sl.vmagic;
                    sg.solver = sl.solver;
                    segs[seg_run + ex_s] = sg;
                }
                chunk_run += tot_c;
                seg_run += tot_s;
            }
            if (threadIdx.x == 0) {
                pl.level_nchunk[L * kBatchClasses + cls] = chunk_run;
                pl.level_nseg[L * kBatchClasses + cls] = seg_run;
            }
        }
        return;
    }
    uint32_t chunk_run = 0, act_run = 0;
    for (uint32_t base = 0; base < n_slots; base += kBatchPlanThreads) {
        const uint32_t j = base + threadIdx.x;
        uint32_t nch = 0, on = 0;
        if (j < n_slots && slots[j].active) {
            on = 1;
            const uint64_t n = slots[j].nc * 4 * slots[j].G;
            nch = (uint32_t)((n + kBatchChunk - 1) / kBatchChunk);
        }
        uint32_t tot_c, tot_a;
        const uint32_t ex_c = block_exclusive_scan(nch, &tot_c);
        const uint32_t ex_a = block_exclusive_scan(on, &tot_a);
        if (on) {
            pl.act[act_run + ex_a] = j;
            pl.chunk_prefix[act_run + ex_a] = chunk_run + ex_c;
        }
        chunk_run += tot_c;
        act_run += tot_a;
    }
    if (threadIdx.x == 0) {
        pl.chunk_prefix[act_run] = chunk_run;
        *pl.n_act = act_run;
    }
}

// Largest k in [0, n) with key(k) <= x (key(0) <= x is given).
template <typename KeyFn>
__device__ __forceinline__ uint32_t upper_index(uint32_t n, uint32_t x, KeyFn key)
{
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (key(mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <typename Real>
__device__ __forceinline__ LevelArgs slot_args(const BatchSlot &s)
{
    LevelArgs p = {};
    p.iso = s.iso32 ? (const void *)s.iso32 : (const void *)s.iso;
    p.qang = nullptr;
    p.psi = s.psi;
    p.G = s.G;
    p.vg = s.vg;
    p.vmagic = s.vmagic;
    p.solver = s.solver;
    return p;
}

// The chunks of one class at one level, taken by this block's warps with a
// stride of the class's block count.  The first chunk's records are staged
// before waiting on the previous level (programmatic dependent launch).
template <typename Real, int IPW, int VG>
__device__ __forceinline__ void batch_class_body(const BatchSlot *__restrict__ slots, const BatchPlan &pl,
                                                 uint32_t L, uint32_t cls, uint32_t blk, uint32_t nblk,
                                                 RecordTile<Real, IPW> &T, bool &waited)
{
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint32_t nchunk = pl.level_nchunk[L * kBatchClasses + cls];
    const uint32_t nseg = pl.level_nseg[L * kBatchClasses + cls];
    const BatchSeg *__restrict__ segs = pl.segs + ((size_t)L * kBatchClasses + cls) * pl.seg_stride;
    for (uint32_t ch = blk * 4u + w; ch < nchunk; ch += nblk * 4u) {
        const uint32_t k = upper_index(nseg, ch, [&](uint32_t m) { return segs[m].chunk_begin; });
        const BatchSeg sg = segs[k];
        const BatchSlot &s = slots[sg.slot];
        const ItemRecord<Real> *rec = (const ItemRecord<Real> *)s.rec;
        tile_fill<Real, IPW>(T, rec + sg.item_begin + (uint64_t)(ch - sg.chunk_begin) * IPW + lane, lane, true);
        if (!waited) {
            pdl_wait_prerequisites();
            waited = true;
        }
        __syncwarp();
        record_pairs<Real, IPW, VG, false>(slot_args<Real>(s), T, lane);
        __syncwarp();
    }
}

// Direct form (compact records rebuilt into registers): chunk = 32 (item,
// group vector) tasks of one member at one level (a level's item count is a
// multiple of 32, so chunks never straddle members), one task per lane.  The
// block stages its class's segments of the level in shared memory before the
// wait on the previous level (up to kBatchSegSmem of them; more are searched
// in global memory), so a warp's member lookup is a shared-memory search.
constexpr uint32_t kBatchSegSmem = 256;

// One chunk (32 tasks of one member at one level) of the direct form: the
// member's segment found by binary search, its compact record rebuilt in
// registers, the source loaded, then (after `wait`, which the caller uses to
// wait for the previous level) the upwind rows and the solve.  L2_ONLY: the
// upwind rows are read around L1 (they were written by other SMs during the
// same launch).
template <typename Real, int VG, bool ANY, bool L2_ONLY, typename Wait>
__device__ __forceinline__ void batch_direct_chunk(const BatchSeg *segs, uint32_t nseg, uint32_t ch, uint32_t lane,
                                                   Wait wait)
{
    const uint32_t k = upper_index(nseg, ch, [&](uint32_t m) { return segs[m].chunk_begin; });
    const BatchSeg &sg = segs[k];
    LevelArgs p = {};
    p.psi = sg.psi;
    p.iso = sg.iso;
    p.G = sg.G;
    p.vg = VG;
    p.vmagic = sg.vmagic;
    p.solver = sg.solver;
    const uint32_t gpv = p.G / VG;
    const uint32_t task = (ch - sg.chunk_begin) * 32u + lane;
    const uint32_t itl = gpv == 1u ? task : __umulhi(task, p.vmagic);
    const uint32_t g = (task - itl * gpv) * VG;
    RegRecord<Real> R;
    // FP64 NoPivot: the LU is rebuilt after the upwind loads are issued, in
    // their latency (at 128 registers this also removes the kernel's spills;
    // the FP32 body measured the same either way and keeps it before).
    constexpr bool kLate = !ANY && sizeof(Real) == 8;
    if constexpr (kLate) load_compact_raw((const CompactRecord<Real> *)sg.rec + itl, R);
    else load_record((const CompactRecord<Real> *)sg.rec + itl, R, ANY ? p.solver : (uint32_t)kSolveNoPivot);
    const bool live = R.u(0) != kSentinel;
    PairIn<Real, VG> in;
    if (live) pair_load_source<Real, VG>(p, R, g, in);
    wait();
    if (live) {
        pair_load_upwind<Real, VG, L2_ONLY>(p, R, g, in);
        if constexpr (kLate) compact_factor_nopivot(R);
        pair_solve_store_any<Real, VG, RegRecord<Real>, ANY>(p, R, g, in);
    }
}

// Stages a (level, class) list of segments in shared memory when it fits
// (block-wide); returns the list to search.
__device__ __forceinline__ const BatchSeg *batch_stage_segs(const BatchPlan &pl, uint32_t L, uint32_t cls,
                                                            BatchSeg *sseg, uint32_t &nseg)
{
    nseg = pl.level_nseg[L * kBatchClasses + cls];
    const BatchSeg *gsegs = pl.segs + ((size_t)L * kBatchClasses + cls) * pl.seg_stride;
    const bool staged = nseg <= kBatchSegSmem;
    if (staged)
        for (uint32_t i = threadIdx.x; i < nseg; i += blockDim.x) sseg[i] = gsegs[i];
    __syncthreads();
    return staged ? sseg : gsegs;
}

template <typename Real, int VG, bool ANY>
__device__ __forceinline__ void batch_direct_body(const BatchPlan &pl, uint32_t L, uint32_t cls, uint32_t blk,
                                                  uint32_t nblk, BatchSeg *sseg, bool &waited)
{
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint32_t nchunk = pl.level_nchunk[L * kBatchClasses + cls];
    uint32_t nseg;
    const BatchSeg *segs = batch_stage_segs(pl, L, cls, sseg, nseg);
    for (uint32_t ch = blk * 4u + w; ch < nchunk; ch += nblk * 4u)
        batch_direct_chunk<Real, VG, ANY, false>(segs, nseg, ch, lane, [&] {
            if (!waited) {
                pdl_wait_prerequisites();
                waited = true;
            }
        });
}

// ANY: some member solves with Original or a Cramer solver (each member's
// own p.solver); otherwise every member uses NoPivot.
// MINB: blocks per SM the register allocation must allow (FP64 NoPivot: 4,
// i.e. at most 128 registers, measured 13% faster than its natural 146).
template <typename Real, bool ANY, int MINB = 1>
__global__ void __launch_bounds__(128, MINB)
batch_direct_level_kernel(const BatchSlot *__restrict__ slots, BatchPlan pl, uint32_t L, BatchCuts cut)
{
    __shared__ BatchSeg sseg[kBatchSegSmem];
    pdl_launch_dependents();
    bool waited = false;
    const uint32_t b = blockIdx.x;
    if (b < cut.c[1]) {
        batch_direct_body<Real, 1, ANY>(pl, L, 0, b, cut.c[1], sseg, waited);
    } else if (b < cut.c[2]) {
        batch_direct_body<Real, 2, ANY>(pl, L, 1, b - cut.c[1], cut.c[2] - cut.c[1], sseg, waited);
    } else if constexpr (sizeof(Real) == 4) {
        batch_direct_body<Real, 4, ANY>(pl, L, 2, b - cut.c[2], cut.c[3] - cut.c[2], sseg, waited);
    }
    if (!waited) pdl_wait_prerequisites();
    (void)slots;
}

// Persistent form of a pass's wavefront: one cooperative launch walks every
// global level.  Within a level, for each vector-width class, the warps take
// chunks from a device work queue (one counter per level and class, zeroed
// before the launch) until the level's chunks run out; then every block
// meets at a bounded grid barrier before the next level.  The per-chunk
// arithmetic is the level kernels' (bit-identical results); upwind rows are
// read around L1, since other SMs wrote them during this launch.
template <typename Real, int VG, bool ANY>
__device__ __noinline__ void batch_persist_class(const BatchPlan &pl, const BatchPersistArgs &a, uint32_t L,
                                                    uint32_t cls, BatchSeg *sseg)
{
    const uint32_t nchunk = pl.level_nchunk[L * kBatchClasses + cls];
    if (nchunk == 0) return;  // the same for every thread of the block
    uint32_t nseg;
    const BatchSeg *segs = batch_stage_segs(pl, L, cls, sseg, nseg);
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t *q = a.queue + L * kBatchClasses + cls;
    for (;;) {
        uint32_t ch = 0;
        if (lane == 0) ch = atomicAdd(q, 1u);
        ch = __shfl_sync(0xffffffffu, ch, 0);
        if (ch >= nchunk) break;
        batch_direct_chunk<Real, VG, ANY, true>(segs, nseg, ch, lane, [] {});
    }
    __syncthreads();  // the segment list is restaged for the next class
}

template <typename Real, bool ANY, int MINB = 1>
__global__ void __launch_bounds__(128, MINB)
batch_persist_kernel(const BatchSlot *__restrict__ slots, BatchPlan pl, BatchPersistArgs a)
{
    __shared__ BatchSeg sseg[kBatchSegSmem];
    for (uint32_t L = 0; L < a.max_levels; ++L) {
        batch_persist_class<Real, 1, ANY>(pl, a, L, 0, sseg);
        batch_persist_class<Real, 2, ANY>(pl, a, L, 1, sseg);
        if constexpr (sizeof(Real) == 4) batch_persist_class<Real, 4, ANY>(pl, a, L, 2, sseg);
        if (L + 1 < a.max_levels &&
            !grid_barrier(a.barrier, (unsigned long long)(L + 1) * gridDim.x, a.df, L))
            return;
    }
    (void)slots;
}

// One global level of the batched sweep, 4 warps per block, IPW items per
// chunk.  Blocks [cut[c], cut[c+1]) serve vector-width class c (1, 2, 4
// groups per access), so each block runs one kernel body.  The work list was
// built by the plan kernel, which completed before the first level started.
template <typename Real, int IPW>
__global__ void __launch_bounds__(128)
batch_level_kernel(const BatchSlot *__restrict__ slots, BatchPlan pl, uint32_t L, BatchCuts cut)
{
    __shared__ RecordTile<Real, IPW> tiles[4];
    pdl_launch_dependents();
    RecordTile<Real, IPW> &T = tiles[threadIdx.x >> 5];
    bool waited = false;
    const uint32_t b = blockIdx.x;
    if (b < cut.c[1]) {
        batch_class_body<Real, IPW, 1>(slots, pl, L, 0, b, cut.c[1], T, waited);
    } else if (b < cut.c[2]) {
        batch_class_body<Real, IPW, 2>(slots, pl, L, 1, b - cut.c[1], cut.c[2] - cut.c[1], T, waited);
    } else if constexpr (sizeof(Real) == 4) {
        batch_class_body<Real, IPW, 4>(slots, pl, L, 2, b - cut.c[2], cut.c[3] - cut.c[2], T, waited);
    }
    if (!waited) pdl_wait_prerequisites();
}

}  // namespace tycho

namespace tycho {

// Cooperative launch of the persistent form with as many blocks as can be
// resident at once.
template <typename Real, bool ANY, int MINB>
cudaError_t batch_persist_launch(const BatchSlot *slots, const BatchPlan &pl, const BatchPersistArgs &a,
                                 cudaStream_t s)
{
    const void *fn = (const void *)batch_persist_kernel<Real, ANY, MINB>;
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 128, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(per_sm * sms));
    cfg.blockDim = dim3(128);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    BatchPlan plc = pl;
    BatchPersistArgs ac = a;
    void *args[] = {(void *)&slots, (void *)&plc, (void *)&ac};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace tycho
