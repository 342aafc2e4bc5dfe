// Device-resident sweep instance and its outer solvers.
//
// Reference call structure mirrored here:
//   SweeperTraverse::sweep            -> Sweeper::apply / Sweeper::sweep_host
//   SourceIteration::fixedPoint       -> Sweeper::solve, method 0
//   SourceIteration::krylov (+PETSc)  -> Sweeper::solve, method 1 (own GMRES)
//   FP32-sweep GMRES in FP64 iterative refinement -> method 2
// (src/SweeperTraverse.cc:65-89, src/SourceIteration.cc:76-285).
#include "sweeper.hpp"

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <mutex>
#include <thread>

#include <omp.h>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "devmem.hpp"
#include "rng.hpp"
#include "status.hpp"
#include "trace.hpp"

namespace tycho {

#define TY_CUDA(expr)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (expr);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            err = std::string(#expr) + ": " + cudaGetErrorString(e_);                  \
            return e_ == cudaErrorMemoryAllocation ? kErrOom : kErrCuda;               \
        }                                                                              \
    } while (0)

#define TY_CHECK(expr)                  \
    do {                                \
        int s_ = (expr);                \
        if (s_ != kOk) return s_;       \
    } while (0)

namespace {

template <typename T>
cudaError_t upload(T *&dst, const T *src, size_t n, cudaStream_t s)
{
    cudaError_t e = dev_malloc(&dst, sizeof(T) * std::max<size_t>(n, 1), s);
    if (e != cudaSuccess) return e;
    if (n) e = cudaMemcpyAsync(dst, src, sizeof(T) * n, cudaMemcpyHostToDevice, s);
    return e;
}

uint32_t group_magic(uint32_t G)
{
    return G == 1 ? 0u : (uint32_t)(((1ull << 32) + G - 1) / G);
}

}  // namespace

Sweeper::~Sweeper()
{
    TraceScope trace("sweeper.destroy");
    if (device_ >= 0) cudaSetDevice(device_);
    for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second.exec);
    for (auto &kv : step_graphs_) cudaGraphExecDestroy(kv.second);
    for (auto &g : chunk_graphs_)
        if (g) cudaGraphExecDestroy(g);
    dev_free(d_chunk_pos_, stream_);
    for (cudaEvent_t ev : {ev_start_})
        if (ev) cudaEventDestroy(ev);
    for (int j = 0; j < kMaxHostChunks; ++j) {
        if (ev_h2d_[j]) cudaEventDestroy(ev_h2d_[j]);
        if (ev_swept_[j]) cudaEventDestroy(ev_swept_[j]);
    }
    for (void *b : h_stage_)
        if (b) cudaFreeHost(b);
    for (auto &e : ev_stage_)
        if (e) cudaEventDestroy(e);
    if (h2d_stream_) cudaStreamDestroy(h2d_stream_);
    if (d2h_stream_) cudaStreamDestroy(d2h_stream_);
    void *bufs[] = {d_items_, d_abar64_, d_abar32_, d_adj_, d_nbrmap_, d_cellk64_, d_cellk32_,
                    d_w_, d_sigs_, d_scat_, d_qiso_, d_qang_, d_src_, d_iso_, d_iso32_, d_psi_,
                    d_phi_, d_r_, d_tmp_, d_V_, d_h_, d_flush_, d_done_, d_ctl_, d_rec_[0], d_rec_[1],
                    d_level_off_, d_barrier_, d_crec_[0], d_crec_[1], d_flags_, d_adj32_, d_psi_prev_};
    for (void *b : bufs) dev_free(b, stream_);
    for (auto &kv : links_) {
        dev_free(kv.second.d_send_row, stream_);
        dev_free(kv.second.d_send_vtx, stream_);
        dev_free(kv.second.d_recv_ghost, stream_);
    }
    reducer_free(red_, stream_);
    for (auto &st : aux_)
        if (st) cudaStreamDestroy(st);
    for (auto &ev : join_)
        if (ev) cudaEventDestroy(ev);
    if (fork_) cudaEventDestroy(fork_);
    if (stream_) cudaStreamDestroy(stream_);
}

// A_f = area * omega.n of every item position (the schedule's order).
int Sweeper::compute_item_abar(std::string &err)
{
    const MeshTables &t = *tables_;
    std::vector<double> omega(3 * (size_t)A_);
    std::copy(quad_.xi.begin(), quad_.xi.end(), omega.begin());
    std::copy(quad_.eta.begin(), quad_.eta.end(), omega.begin() + A_);
    std::copy(quad_.mu.begin(), quad_.mu.end(), omega.begin() + 2 * A_);
    double *d_omega = nullptr, *d_normal = nullptr, *d_area = nullptr;
    cudaError_t e = upload(d_omega, omega.data(), omega.size(), stream_);
    if (e == cudaSuccess) e = upload(d_normal, t.normal.data(), t.normal.size(), stream_);
    if (e == cudaSuccess) e = upload(d_area, t.area.data(), t.area.size(), stream_);
    if (e == cudaSuccess)
        e = launch_item_abar(d_items_, sched_.n_padded, A_, d_normal, d_area, d_omega, d_abar64_, d_abar32_, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    dev_free(d_omega, stream_);
    dev_free(d_normal, stream_);
    dev_free(d_area, stream_);
    TY_CUDA(e);
    return kOk;
}

int Sweeper::set_work_order(int order, std::string &err)
{
    if (order < 0 || order > 2) { err = "work order must be 0 (cell), 1 (b-level) or 2 (random)"; return kErrArg; }
    if (order == work_order_) return kOk;
    TY_CUDA(cudaSetDevice(device_));
    TY_CUDA(cudaStreamSynchronize(stream_));
    schedule_host();  // the item list on the host
    std::vector<uint32_t> blev;
    if (order == 1) b_levels(*tables_, quad_, sched_, blev);
    const uint64_t nc = nc_;
    const uint32_t A = (uint32_t)A_;
    const size_t nseg = sched_.octant_offset.size() - 1;
    #pragma omp parallel for schedule(dynamic, 64)
    for (size_t k = 0; k < nseg; ++k) {
        const uint64_t b = sched_.octant_offset[k], e = sched_.octant_offset[k + 1];
        uint64_t n = b;
        while (n < e && sched_.items[n] != kSentinelItem) ++n;  // padding sits at the segment's end
        uint32_t *it = sched_.items.data();
        std::sort(it + b, it + n);  // the cell order: increasing cell * A + angle
        if (order == 1) {
            // Priorities' b-levels (src/Priorities.cc:59-164, intraAngleP 1):
            // the longest downwind chain first
            std::stable_sort(it + b, it + n, [&](uint32_t x, uint32_t y) {
                return blev[(size_t)(x % A) * nc + x / A] > blev[(size_t)(y % A) * nc + y / A];
            });
        } else if (order == 2) {
            // a seeded random order (intraAngleP 0), the same on every run
            Rng rng(0x5eedull + k);
            for (uint64_t i = n - b; i > 1; --i) std::swap(it[b + i - 1], it[b + rng.range(0, (int64_t)i - 1)]);
        }
    }
    TY_CUDA(cudaMemcpyAsync(d_items_, sched_.items.data(), sizeof(uint32_t) * sched_.n_padded,
                            cudaMemcpyHostToDevice, stream_));
    TY_CHECK(compute_item_abar(err));
    // everything kept per item position is stale
    rec_valid_[0] = rec_valid_[1] = false;
    crec_valid_[0] = crec_valid_[1] = false;
    for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second.exec);
    graphs_.clear();
    drop_step_graphs();
    for (auto &g : chunk_graphs_)
        if (g) cudaGraphExecDestroy(g);
    chunk_graphs_.clear();
    dev_free(d_chunk_pos_, stream_);
    d_chunk_pos_ = nullptr;
    chunk_k_ = 0;
    work_order_ = order;
    return kOk;
}

const Schedule &Sweeper::schedule_host() const
{
    if (sched_.items.size() != sched_.n_padded) {
        sched_.items.resize(sched_.n_padded);
        if (cudaSetDevice(device_) != cudaSuccess ||
            cudaMemcpy(sched_.items.data(), d_items_, sizeof(uint32_t) * sched_.n_padded,
                       cudaMemcpyDeviceToHost) != cudaSuccess) {
            sched_.items.clear();
            throw std::runtime_error("copying the schedule back from the device failed");
        }
        tlevel_from_items(sched_, nc_, A_);
    }
    return sched_;
}

int Sweeper::init(std::shared_ptr<const MeshTables> tp, const SweeperOptions &o, std::string &err)
{
    if (!tp) { err = "no mesh tables"; return kErrArg; }
    const MeshTables &t = *tp;
    if (o.n_groups < 1 || o.n_groups > 64) { err = "nGroups must be in 1..64"; return kErrArg; }
    if (o.gauss_elim < 0 || o.gauss_elim > 3) { err = "GaussElim must be 0..3"; return kErrArg; }
    solver_ = o.gauss_elim;
    TraceScope trace_init("sweeper.init");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        err = "no CUDA device: the B200 sweep has no CPU fallback";
        return kErrCuda;
    }
    if (o.device < 0 || o.device >= ndev) { err = "bad device ordinal"; return kErrArg; }
    device_ = o.device;
    TY_CUDA(cudaSetDevice(device_));
    // the no-alloc sweep's fixed scratch array: resolved here, once per
    // device, so that tycho_sweeper_sweep_noalloc itself loads nothing
    TY_CHECK(noalloc_scratch_prepare(device_, err));
    TY_CHECK(make_quadrature(o.sn_order, quad_, err));
    n_angles_full_ = quad_.n_angles;
    angle_begin_ = o.angle_begin;
    if (o.angle_begin != 0 || o.angle_end != 0) {
        // an angle shard: the directions [begin, end) with their weights, so
        // that phi is the partial sum over them (src/Util.cc:85-97 split by
        // angle range); every direction sweeps independently
        if (o.angle_begin < 0 || o.angle_end > quad_.n_angles || o.angle_begin >= o.angle_end) {
            err = "angle range must satisfy 0 <= begin < end <= " + std::to_string(quad_.n_angles);
            return kErrArg;
        }
        auto cut = [&](std::vector<double> &v) {
            v = std::vector<double>(v.begin() + o.angle_begin, v.begin() + o.angle_end);
        };
        cut(quad_.xi);
        cut(quad_.eta);
        cut(quad_.mu);
        cut(quad_.wt);
        quad_.n_angles = o.angle_end - o.angle_begin;
    }
    tables_ = std::move(tp);
    nc_ = t.n_cells;
    A_ = quad_.n_angles;
    G_ = o.n_groups;
    fp32_ = o.fp32;
    TY_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    if (o.levelling < 0 || o.levelling > 2) { err = "levelling must be 0, 1 or 2"; return kErrArg; }
    const bool on_device = o.levelling == 2 || (o.levelling == 0 && nc_ * (uint64_t)A_ >= (1ull << 20));
    // Levelled on the device, the item list stays there; the host copy is
    // made only for the diagnostics that ask for it (schedule_host).
    {
        TraceScope ts(on_device ? "sweeper.init.levelling_device" : "sweeper.init.levelling_host");
        if (on_device) TY_CHECK(build_schedule_device(t, quad_, sched_, &d_items_, stream_, err));
        else TY_CHECK(build_schedule(t, quad_, sched_, err));
    }
    TraceScope trace_rest("sweeper.init.topology_uploads_buffers");
    for (auto &st : aux_) TY_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    TY_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
    for (auto &ev : join_) TY_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));

    // Faces toward another partition (one partition of a multi-partition
    // mesh; src/TychoMeshIO.cc:250-262): bound sides b = 0.. in side order.
    bound_side_.clear();
    side_bound_.assign(t.n_sides, -1);
    if (!t.adj_rank.empty())
        for (uint64_t c = 0; c < nc_; ++c)
            for (int f = 0; f < 4; ++f) {
                const uint64_t r = t.adj_rank[c * 4 + f];
                if (t.adj_cell[c * 4 + f] != kNone || r == kNone || r == t.partition) continue;
                side_bound_[t.side[c * 4 + f]] = (int64_t)bound_side_.size();
                bound_side_.push_back(t.side[c * 4 + f]);
            }
    n_bound_ = bound_side_.size();
    if (n_bound_ && (2 * (nc_ + n_bound_) + n_bound_) * (uint64_t)A_ >= (1ull << 31)) {
        err = "too many cells and partition sides";
        return kErrArg;
    }

    // Per-cell topology: neighbours and, per (face, local vertex), the
    // neighbour's vertex index (neighborVrtx o cellToFaceVrtx).  A face
    // toward another partition names its ghost row instead, whose vertex fv
    // = cellToFaceVrtx(c, f, j) holds psiBound(g, fv, a, side): the kernels
    // read it as an upwind row, and the schedule orders nothing by it.
    std::vector<int4> adj(nc_), adj32;
    std::vector<uint32_t> nmap(nc_, 0);
    for (uint64_t c = 0; c < nc_; ++c) {
        int a4[4];
        for (int f = 0; f < 4; ++f) {
            uint64_t n = t.adj_cell[c * 4 + f];
            const int64_t b = n == kNone && n_bound_ ? side_bound_[t.side[c * 4 + f]] : -1;
            a4[f] = n != kNone ? (int)n : b >= 0 ? (int)(nc_ + (uint64_t)b) : -1;
            if (n == kNone && b < 0) continue;
            for (int j = 0; j < 4; ++j) {
                if (j == f) continue;
                uint64_t fv = t.cell_to_face[(c * 4 + f) * 4 + j];
                uint64_t nv = n == kNone ? fv : t.neighbor_vrtx[(c * 4 + f) * 3 + fv];
                nmap[c] |= (uint32_t)(nv & 3u) << ((f * 4 + j) * 2);
            }
        }
        adj[c] = make_int4(a4[0], a4[1], a4[2], a4[3]);
    }
    if (n_bound_ && o.fp32) {
        adj32 = adj;
        const int shift = (int)(nc_ + 2 * n_bound_);  // 2 (nc + B) + b = (nc + b) + (nc + 2B)
        for (auto &a : adj32) {
            int *v = &a.x;
            for (int f = 0; f < 4; ++f)
                if (v[f] >= (int)nc_) v[f] += shift;
        }
    }
    if (nc_ >= (1ull << 31)) { err = "too many cells"; return kErrArg; }
    const uint64_t nitems = sched_.n_padded;
    if (!on_device || !d_items_) TY_CUDA(upload(d_items_, sched_.items.data(), nitems, stream_));
    TY_CUDA(upload(d_adj_, adj.data(), nc_, stream_));
    if (!adj32.empty()) TY_CUDA(upload(d_adj32_, adj32.data(), nc_, stream_));
    TY_CUDA(upload(d_nbrmap_, nmap.data(), nc_, stream_));
    TY_CUDA(upload(d_w_, quad_.wt.data(), (size_t)A_, stream_));
    TY_CUDA(dev_malloc(&d_abar64_, sizeof(double4) * std::max<uint64_t>(nitems, 1), stream_));
    if (fp32_) TY_CUDA(dev_malloc(&d_abar32_, sizeof(float4) * std::max<uint64_t>(nitems, 1), stream_));
    TY_CHECK(compute_item_abar(err));
    const size_t nphi = phi_size(), npsi = psi_size();
    // psi rows, then the partition boundary's ghost rows (FP64, then FP32)
    const size_t ghost = n_bound_ * (size_t)A_ * 4 * G_;
    const size_t psi_bytes = sizeof(double) * (npsi + ghost) + (fp32_ ? sizeof(float) * ghost : 0);
    TY_CUDA(dev_malloc(&d_psi_, std::max<size_t>(psi_bytes, 8), stream_));
    TY_CUDA(cudaMemsetAsync(d_psi_, 0, psi_bytes, stream_));
    TY_CUDA(dev_malloc(&d_iso_, sizeof(double) * nphi, stream_));
    if (fp32_) TY_CUDA(dev_malloc(&d_iso32_, sizeof(float) * nphi, stream_));
    TY_CUDA(dev_malloc(&d_phi_, sizeof(double) * nphi, stream_));
    TY_CUDA(dev_malloc(&d_r_, sizeof(double) * nphi, stream_));
    TY_CUDA(dev_malloc(&d_tmp_, sizeof(double) * nphi, stream_));
    TY_CUDA(cudaMemsetAsync(d_phi_, 0, sizeof(double) * nphi, stream_));
    TY_CUDA(dev_malloc(&d_cellk64_, sizeof(double) * 3 * nc_, stream_));
    if (fp32_) TY_CUDA(dev_malloc(&d_cellk32_, sizeof(float) * 3 * nc_, stream_));
    TY_CUDA(dev_malloc(&d_sigs_, sizeof(double) * nc_, stream_));
    TY_CUDA(reducer_init(red_, stream_));

    // Dataflow schedule: completion epochs per item and a control block;
    // grid = every block that can be co-resident (cooperative launch).
    TY_CUDA(dev_malloc(&d_done_, sizeof(uint32_t) * (size_t)nc_ * A_, stream_));
    TY_CUDA(cudaMemsetAsync(d_done_, 0, sizeof(uint32_t) * (size_t)nc_ * A_, stream_));
    TY_CUDA(dev_malloc(&d_ctl_, sizeof(uint32_t) * 8, stream_));
    TY_CUDA(cudaMemsetAsync(d_ctl_, 0, sizeof(uint32_t) * 8, stream_));
    TY_CUDA(upload(d_level_off_, sched_.level_offset.data(), sched_.level_offset.size(), stream_));
    TY_CUDA(dev_malloc(&d_barrier_, sizeof(unsigned long long), stream_));
    // Default launch shape: compact records in registers, one launch per
    // level (64-thread blocks); schedule 2 asks for the persistent dataflow
    // kernel (warp tiles); explicit threads-per-item selects the
    // item-parallel variant.  The autotuner can replace any of them.
    // Original and the Cramer solvers run in the direct kernels (128 threads)
    const bool nopivot = solver_ == kSolveNoPivot;
    for (int prec = 0; prec < (fp32_ ? 2 : 1); ++prec) {
        const int tpi = prec ? o.tpi32 : o.tpi64;
        if (!nopivot && (tpi || o.schedule == 2)) {
            err = "GaussElim Original / CramerGlu / CramerIntel run on the level schedule with compact records";
            return kErrArg;
        }
        if (tpi) TY_CHECK(configure(prec, o.schedule == 1 ? 1 : 2, 0, tpi, err));
        else if (o.schedule == 2) TY_CHECK(configure(prec, 2, 1, 4, err));
        // compact records in 64-thread blocks on 2 octant streams: FP32 with
        // slotted upwind rows at most 85 registers, FP64 at most 102 (the
        // fastest measured shapes on the 32^3 S8 workload)
        else {
            const bool slots = prec == 1 && nopivot && record_vg(true, (uint32_t)G_) >= 2;
            TY_CHECK(configure(prec, 1, 4, nopivot ? (slots ? -180 : -96) : 128, err, 0, nopivot ? 2 : 1));
        }
    }
    TY_CUDA(cudaStreamSynchronize(stream_));
    return kOk;
}

int Sweeper::configure(int prec, int schedule, int variant, int knob, std::string &err, int vg, int streams)
{
    if (prec == 1 && !fp32_) { err = "sweeper was created without the FP32 sweep"; return kErrArg; }
    if (streams != 1 && streams != 2 && streams != 4 && streams != 8) {
        err = "streams must be 1, 2, 4 or 8";
        return kErrArg;
    }
    if (streams > 1 && schedule != 1) { err = "several streams: level schedule only"; return kErrArg; }
    if (n_bound_ && schedule != 1) {
        // the dataflow flags cover the cells' rows only
        err = "faces toward other partitions: the level schedule only";
        return kErrArg;
    }
    if (vg == 0) vg = (int)record_vg(prec != 0, (uint32_t)G_);
    // one access moves up to 16 bytes (4 FP32 / 2 FP64 groups); the direct
    // variants on levels also take two such vectors per task (8 / 4)
    const bool halves = (prec == 1 && vg == 8) || (prec == 0 && vg == 4);
    if (solver_ != kSolveNoPivot && (variant < 3 || schedule != 1 || knob != 128 || halves)) {
        err = "GaussElim Original / CramerGlu / CramerIntel: direct record variants on the level schedule, "
              "128 threads per block, one group vector per task";
        return kErrArg;
    }
    if (vg != 1 && vg != 2 && !(vg == 4 && prec == 1) && !halves) {
        err = "group vector width must be 1, 2 (FP64: or 4) or 1, 2, 4 (FP32: or 8)";
        return kErrArg;
    }
    if (halves && (variant < 3 || schedule != 1 || knob < 0)) {
        err = "two group vectors per task: direct variants on the level schedule only";
        return kErrArg;
    }
    if (G_ % vg != 0) { err = "group vector width must divide the number of groups"; return kErrArg; }
    if (schedule < 1 || schedule > 3) {
        err = "schedule must be 1 (levels), 2 (dataflow) or 3 (persistent levels)";
        return kErrArg;
    }
    if (schedule == 3 && variant != 2) {
        err = "the persistent-levels schedule runs the record variant only";
        return kErrArg;
    }
    if (variant == 0 && knob != 1 && knob != 2 && knob != 4 && knob != 8 && knob != 16) {
        err = "item-parallel variant: threads per item must be 1, 2, 4, 8 or 16";
        return kErrArg;
    }
    if (variant == 1 && knob != 1 && knob != 2 && knob != 4) {
        err = "warp-tile variant: warps per block must be 1, 2 or 4";
        return kErrArg;
    }
    if (variant == 2 && knob != 8 && knob != 16 && knob != 32) {
        err = "record variant: items per warp must be 8, 16 or 32";
        return kErrArg;
    }
    if (schedule == 3 && prec == 0 && knob == 32) {
        err = "persistent levels in FP64: items per warp must be 8 or 16";
        return kErrArg;
    }
    if (variant >= 3 && schedule == 1 && knob != 64 && knob != 128 && knob != 256 && knob != -64 &&
        knob != -128 && knob != -96 && knob != -80 && knob != -196 && knob != -180 && knob != -172) {
        err = "direct record variants on levels: 64, 128 or 256 threads per block (-64, -128: 64 registers; "
              "-96 / -80: 64 threads, at most 102 / 85 registers; FP32 slotted upwind rows -196 / -180 / -172: "
              "64 threads, at most 102 / 85 / 73 registers)";
        return kErrArg;
    }
    if (knob <= -172 && (prec != 1 || (vg != 2 && vg != 4))) {
        err = "slotted upwind rows (knobs -196, -180, -172): the FP32 sweep with 2 or 4 groups per vector";
        return kErrArg;
    }
    if (variant >= 3 && schedule == 2) {
        const int gv = vg ? vg : (int)record_vg(prec != 0, (uint32_t)G_);
        const int gpv = G_ % gv == 0 ? G_ / gv : 0;
        if (knob != 128 || gpv == 0 || gpv > 32 || (gpv & (gpv - 1)) != 0) {
            err = "direct record variants on dataflow: 128 threads per block, nGroups / vector a power of two <= 32";
            return kErrArg;
        }
    }
    if (variant >= 3 && schedule == 3) {
        err = "the persistent-levels schedule runs the record variant only";
        return kErrArg;
    }
    if (variant < 0 || variant > 4) {
        err = "variant must be 0 (item-parallel), 1 (warp tiles), 2 (records), 3 (direct records) or 4 "
              "(direct compact records)";
        return kErrArg;
    }
    if (variant >= 2) TY_CHECK(ensure_records(prec, false, err, variant == 4));
    int sms = 0, per_sm = 0;
    TY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
    if (variant == 0)
        TY_CUDA(prec ? dataflow_blocks_per_sm<float>(knob, &per_sm) : dataflow_blocks_per_sm<double>(knob, &per_sm));
    else if (variant == 1 || variant == 4)  // compact: the no-alloc sweep runs the 4-warp tile kernel
        TY_CUDA(prec ? tile_dataflow_blocks_per_sm<float>(variant == 4 ? 4 : knob, &per_sm)
                     : tile_dataflow_blocks_per_sm<double>(variant == 4 ? 4 : knob, &per_sm));
    else  // records; the direct variant's no-alloc sweep runs the 16-item record dataflow kernel
        TY_CUDA(prec ? record_dataflow_blocks_per_sm<float>(variant == 3 ? 16 : knob, halves ? vg / 2 : vg, &per_sm)
                     : record_dataflow_blocks_per_sm<double>(variant == 3 ? 16 : knob, halves ? vg / 2 : vg, &per_sm));
    if (per_sm < 1) { err = "dataflow kernel does not fit on an SM"; return kErrCuda; }
    int persist_per_sm = 0;
    if (schedule == 3) {
        TY_CUDA(prec ? record_persist_blocks_per_sm<float>(knob, vg, &persist_per_sm)
                     : record_persist_blocks_per_sm<double>(knob, vg, &persist_per_sm));
        if (persist_per_sm < 1) { err = "persistent-levels kernel does not fit on an SM"; return kErrCuda; }
    }
    LaunchShape &sh = shape_[prec ? 1 : 0];
    sh.schedule = schedule;
    sh.variant = variant;
    sh.knob = knob;
    sh.vg = variant >= 2 ? vg : 1;
    sh.streams = streams;
    sh.grid = (unsigned)(sms * per_sm);
    sh.persist_grid = (unsigned)(sms * persist_per_sm);
    sh.direct_grid = 0;
    if (variant >= 3 && schedule == 2) {
        int direct_per_sm = 0;
        TY_CUDA(prec ? direct_dataflow_blocks_per_sm<float>(vg, variant == 4, &direct_per_sm)
                     : direct_dataflow_blocks_per_sm<double>(vg, variant == 4, &direct_per_sm));
        if (direct_per_sm < 1) { err = "direct dataflow kernel does not fit on an SM"; return kErrCuda; }
        sh.direct_grid = (unsigned)(sms * direct_per_sm);
        const size_t flags = (size_t)nc_ * A_ * (G_ / vg);
        if (flags > flags_cap_) {
            if (d_flags_) dev_free(d_flags_, stream_);
            d_flags_ = nullptr;
            flags_cap_ = 0;
            TY_CUDA(dev_malloc(&d_flags_, sizeof(uint32_t) * flags, stream_));
            TY_CUDA(cudaMemsetAsync(d_flags_, 0, sizeof(uint32_t) * flags, stream_));
            flags_cap_ = flags;
        }
    }
    // cached level graphs were captured for the previous launch shape
    for (auto it = graphs_.begin(); it != graphs_.end();) {
        if (std::get<0>(it->first) == prec) {
            cudaGraphExecDestroy(it->second.exec);
            it = graphs_.erase(it);
        } else {
            ++it;
        }
    }
    drop_step_graphs();
    return kOk;
}

void Sweeper::drop_step_graphs()
{
    for (auto &kv : step_graphs_) cudaGraphExecDestroy(kv.second);
    step_graphs_.clear();
}

// Times every launch shape -- schedule x variant x (threads per item or warps
// per block) -- on this instance's own problem and keeps the fastest.
int Sweeper::autotune(int prec, int reps, LaunchShape *best_shape, double *best_ms, std::string &err)
{
    if (prec == 1 && !fp32_) { err = "sweeper was created without the FP32 sweep"; return kErrArg; }
    if (!have_xs_) { err = "cross sections not set"; return kErrMissing; }
    double best = 1e300;
    LaunchShape keep = shape_[prec ? 1 : 0];
    for (int sched = 1; sched <= (n_bound_ ? 1 : 3); ++sched)
        for (int variant = 0; variant <= 4; ++variant)
            for (int knob : {1, 2, 4, 8, 16, 32, 64, 128, 256, -64, -80, -96, -128, -196, -180, -172}) {
                if (knob < 0 && (variant < 3 || sched != 1)) continue;
                if (solver_ != kSolveNoPivot && (variant < 3 || sched != 1 || knob != 128)) continue;
                if (variant == 0 && ((knob > 2 * G_ && knob > 1) || knob > 16)) continue;  // idle lanes
                if (variant == 1 && knob > 4) continue;
                if (variant == 2 && (knob < 8 || knob > 32)) continue;
                if (variant >= 3 && ((knob > 0 && knob < 64) || sched == 3 || (sched == 2 && knob != 128)))
                    continue;
                if (sched == 3 && (variant != 2 || (prec == 0 && knob == 32))) continue;
                for (int vg : {1, 2, 4, 8}) {
                    if (vg > 1 && (variant < 2 || G_ % vg != 0)) continue;
                    const bool halves = (prec == 1 && vg == 8) || (prec == 0 && vg == 4);
                    if (prec == 0 && vg == 8) continue;
                    if (halves && (variant < 3 || sched != 1 || knob < 0 || solver_ != kSolveNoPivot)) continue;
                    if (knob <= -172 && (prec != 1 || (vg != 2 && vg != 4))) continue;  // FP32 slots only
                    if (variant >= 3 && sched == 2) {
                        const int gpv = G_ / vg;
                        if (gpv > 32 || (gpv & (gpv - 1)) != 0) continue;
                    }
                    for (int streams : {1, 2, 4, 8}) {
                        if (streams > 1 && (sched != 1 || variant < 3)) continue;
                        const int cs = configure(prec, sched, variant, knob, err, vg, streams);
                        if (cs == kErrOom) continue;  // records do not fit next to psi
                        TY_CHECK(cs);
                        double ms[2];
                        TY_CHECK(time_sweeps(prec, 1, false, ms, err));  // warm-up (and graph capture)
                        TY_CHECK(time_sweeps(prec, reps, true, ms, err));   // L2 flushed, as in use
                        if (ms[0] < best) { best = ms[0]; keep = shape_[prec ? 1 : 0]; }
                    }
                }
            }
    TY_CHECK(configure(prec, keep.schedule, keep.variant, keep.knob, err, keep.vg, keep.streams));
    if (best_shape) *best_shape = shape_[prec ? 1 : 0];
    if (best_ms) *best_ms = best;
    return kOk;
}

int Sweeper::launch_dataflow_shape(int prec, const LevelArgs &p, const DataflowArgs &df, cudaStream_t s,
                                   std::string &err)
{
    const LaunchShape &sh = shape_[prec ? 1 : 0];
    cudaError_t e;
    if (sh.variant == 0)
        e = prec ? launch_dataflow<float>(sh.knob, p, df, sh.grid, s)
                 : launch_dataflow<double>(sh.knob, p, df, sh.grid, s);
    else if (sh.variant == 1 || sh.variant == 4)
        e = prec ? launch_dataflow_tile<float>(sh.variant == 4 ? 4 : sh.knob, p, df, sh.grid, s)
                 : launch_dataflow_tile<double>(sh.variant == 4 ? 4 : sh.knob, p, df, sh.grid, s);
    else {
        TY_CHECK(ensure_records(prec, true, err));
        const int ipw = sh.variant == 3 ? 16 : sh.knob;
        LevelArgs q = p;
        if (q.vg > (prec ? 4u : 2u)) {  // two vectors per task: the record kernels take one
            q.vg /= 2;
            q.vmagic = group_magic(q.G / q.vg);
        }
        e = prec ? launch_dataflow_record<float>(ipw, q, d_rec_[1], df, sh.grid, s)
                 : launch_dataflow_record<double>(ipw, q, d_rec_[0], df, sh.grid, s);
    }
    TY_CUDA(e);
    return kOk;
}

LevelArgs Sweeper::level_args(int prec, const void *iso, const double *qang, void *psi) const
{
    LevelArgs p;
    p.items = d_items_;
    p.abar = prec ? (const void *)d_abar32_ : (const void *)d_abar64_;
    p.adj = prec && d_adj32_ ? d_adj32_ : d_adj_;
    p.nbrmap = d_nbrmap_;
    p.cellk = prec ? (const void *)d_cellk32_ : (const void *)d_cellk64_;
    p.iso = iso;
    p.qang = qang;
    p.psi = psi;
    p.A = (uint32_t)A_;
    p.G = (uint32_t)G_;
    p.gmagic = group_magic((uint32_t)G_);
    p.vg = (uint32_t)shape_[prec ? 1 : 0].vg;
    p.vmagic = group_magic((uint32_t)G_ / p.vg);
    p.solver = (uint32_t)solver_;
    return p;
}

int Sweeper::device_view(int prec, DeviceView &v, std::string &err, bool compact)
{
    if (prec == 1 && !fp32_) { err = "sweeper was created without the FP32 sweep"; return kErrArg; }
    if (n_bound_) { err = "faces toward other partitions: not in a batch"; return kErrArg; }
    if (!have_xs_) { err = "cross sections not set"; return kErrMissing; }
    TY_CUDA(cudaSetDevice(device_));
    TY_CHECK(ensure_records(prec, true, err, compact));
    TY_CUDA(cudaStreamSynchronize(stream_));
    v.rec = compact ? d_crec_[prec ? 1 : 0] : d_rec_[prec ? 1 : 0];
    v.psi = d_psi_;
    v.iso = d_iso_;
    v.iso32 = d_iso32_;
    v.qiso = d_qiso_;
    v.sigs = d_sigs_;
    v.scat = d_scat_;
    v.w = d_w_;
    v.phi = d_phi_;
    v.tmp = d_tmp_;
    v.level_off = d_level_off_;
    v.n_levels = sched_.n_levels;
    v.vg = record_vg(prec != 0, (uint32_t)G_);
    return kOk;
}

// Allocates (once) and fills (once per cross-section set) the per-item
// records of the record variant for one precision.
int Sweeper::ensure_records(int prec, bool need_filled, std::string &err, bool compact)
{
    const int k = prec ? 1 : 0;
    void *&buf = compact ? d_crec_[k] : d_rec_[k];
    bool &valid = compact ? crec_valid_[k] : rec_valid_[k];
    if (!buf) {
        const size_t bytes =
            (compact ? compact_record_bytes(prec == 1) : record_bytes(prec == 1)) * sched_.n_padded;
        cudaError_t e = dev_malloc(&buf, bytes, stream_);
        if (e != cudaSuccess) {
            cudaGetLastError();
            buf = nullptr;
            err = std::string(compact ? "compact records (" : "records (") + std::to_string(bytes >> 20) +
                  " MiB) do not fit: " + cudaGetErrorString(e);
            return e == cudaErrorMemoryAllocation ? kErrOom : kErrCuda;
        }
        valid = false;
    }
    if (!valid && have_xs_) {
        const LevelArgs p = level_args(prec, nullptr, nullptr, d_psi_);
        const uint64_t n = sched_.n_padded;
        if (compact)
            TY_CUDA(prec ? launch_compact_records<float>(p, n, buf, stream_)
                         : launch_compact_records<double>(p, n, buf, stream_));
        else
            TY_CUDA(prec ? launch_item_records<float>(p, n, buf, stream_)
                         : launch_item_records<double>(p, n, buf, stream_));
        valid = true;
        // the records are read on other streams too (octant chains, batches)
        TY_CUDA(cudaStreamSynchronize(stream_));
    }
    if (need_filled && !valid) { err = "cross sections not set"; return kErrMissing; }
    return kOk;
}

int Sweeper::check_device_error(std::string &err)
{
    if (!d_ctl_) return kOk;
    uint32_t ctl[4];
    TY_CUDA(cudaMemcpyAsync(ctl, d_ctl_, sizeof ctl, cudaMemcpyDeviceToHost, stream_));
    TY_CUDA(cudaStreamSynchronize(stream_));
    if (ctl[0] == 0) return kOk;
    err = "sweep wait timed out at item " + std::to_string(ctl[1]) + " face " + std::to_string(ctl[2]) +
          " (upwind item never completed)";
    TY_CUDA(cudaMemsetAsync(d_ctl_, 0, sizeof(uint32_t) * 4, stream_));
    TY_CUDA(cudaStreamSynchronize(stream_));
    return kErrTimeout;
}

int Sweeper::set_cross_sections(const double *sigma_t, const double *sigma_s, const double *scatter,
                                std::string &err)
{
    if (!sigma_t || !sigma_s) { err = "sigma_t and sigma_s are required"; return kErrArg; }
    TY_CUDA(cudaSetDevice(device_));
    std::vector<double> k64(3 * nc_);
    std::vector<float> k32(3 * nc_);
    for (uint64_t c = 0; c < nc_; ++c) {
        const double volume = tables_->volume[c], sigma = sigma_t[c];
        if (!(sigma >= 0.0) || !std::isfinite(sigma)) { err = "sigma_t must be finite and >= 0"; return kErrArg; }
        // Transport.cc:66-69 and :84-102 with the reference's grouping.
        k64[3 * c + 0] = volume / 20.0;
        k64[3 * c + 1] = 1.0 * sigma * volume / 20.0;
        k64[3 * c + 2] = 2.0 * sigma * volume / 20.0;
        for (int i = 0; i < 3; ++i) k32[3 * c + i] = (float)k64[3 * c + i];
    }
    TY_CUDA(cudaMemcpyAsync(d_cellk64_, k64.data(), sizeof(double) * k64.size(), cudaMemcpyHostToDevice, stream_));
    if (d_cellk32_)
        TY_CUDA(cudaMemcpyAsync(d_cellk32_, k32.data(), sizeof(float) * k32.size(), cudaMemcpyHostToDevice, stream_));
    TY_CUDA(cudaMemcpyAsync(d_sigs_, sigma_s, sizeof(double) * nc_, cudaMemcpyHostToDevice, stream_));
    if (scatter) {
        if (!d_scat_) TY_CUDA(dev_malloc(&d_scat_, sizeof(double) * G_ * G_, stream_));
        TY_CUDA(cudaMemcpyAsync(d_scat_, scatter, sizeof(double) * G_ * G_, cudaMemcpyHostToDevice, stream_));
    } else if (d_scat_) {
        dev_free(d_scat_, stream_);
        d_scat_ = nullptr;
    }
    TY_CUDA(cudaStreamSynchronize(stream_));
    drop_step_graphs();  // they hold the source and scattering buffers' addresses
    have_xs_ = true;
    rec_valid_[0] = rec_valid_[1] = false;
    crec_valid_[0] = crec_valid_[1] = false;
    for (int k = 0; k < 2; ++k)
        if (shape_[k].variant == 2 && (k == 0 || fp32_)) TY_CHECK(ensure_records(k, true, err));
    return kOk;
}

int Sweeper::set_source(int kind, const double *q, std::string &err)
{
    TY_CUDA(cudaSetDevice(device_));
    if (kind != 0 && kind != 1) { err = "source kind must be 0 (angular) or 1 (isotropic)"; return kErrArg; }
    drop_step_graphs();
    double *&dst = kind == 0 ? d_qang_ : d_qiso_;
    const size_t n = kind == 0 ? psi_size() : phi_size();
    if (!q) {
        if (dst) dev_free(dst, stream_);
        dst = nullptr;
        return kOk;
    }
    if (!dst) TY_CUDA(dev_malloc(&dst, sizeof(double) * n, stream_));
    TY_CUDA(cudaMemcpyAsync(dst, q, sizeof(double) * n, cudaMemcpyHostToDevice, stream_));
    TY_CUDA(cudaStreamSynchronize(stream_));
    return kOk;
}

int Sweeper::levels(int prec, bool has_iso, const double *qang, cudaEvent_t beg, cudaEvent_t end,
                    std::string &err)
{
    const void *iso = has_iso ? (prec ? (const void *)d_iso32_ : (const void *)d_iso_) : nullptr;
    const LaunchShape &sh = shape_[prec ? 1 : 0];
    if (sh.schedule == 3) {
        TY_CHECK(ensure_records(prec, true, err));
        const LevelArgs p = level_args(prec, iso, qang, d_psi_);
        DataflowArgs df;
        df.done = d_done_;
        df.err = d_ctl_;
        df.abort = d_ctl_ + 3;
        df.epoch = d_ctl_ + 4;
        df.n_items = sched_.n_padded;
        df.spin_limit = spin_limit_;
        if (beg) TY_CUDA(cudaEventRecord(beg, stream_));
        TY_CUDA(prec ? launch_persist_record<float>(sh.knob, p, d_rec_[1], d_level_off_, sched_.n_levels,
                                                    d_barrier_, df, sh.persist_grid, stream_)
                     : launch_persist_record<double>(sh.knob, p, d_rec_[0], d_level_off_, sched_.n_levels,
                                                     d_barrier_, df, sh.persist_grid, stream_));
        if (end) TY_CUDA(cudaEventRecord(end, stream_));
        return kOk;
    }
    if (sh.schedule == 2 && sh.variant >= 3) {
        TY_CHECK(ensure_records(prec, true, err, sh.variant == 4));
        const LevelArgs p = level_args(prec, iso, qang, d_psi_);
        DataflowArgs df;
        df.done = d_flags_;
        df.err = d_ctl_;
        df.abort = d_ctl_ + 3;
        df.epoch = d_ctl_ + 4;
        df.n_items = sched_.n_padded;
        df.spin_limit = spin_limit_;
        TY_CUDA(launch_bump_epoch(d_ctl_ + 4, stream_));
        if (beg) TY_CUDA(cudaEventRecord(beg, stream_));
        const void *rec = sh.variant == 4 ? d_crec_[prec ? 1 : 0] : d_rec_[prec ? 1 : 0];
        TY_CUDA(prec ? launch_direct_dataflow<float>(p, rec, sh.variant == 4, df, sh.direct_grid, stream_)
                     : launch_direct_dataflow<double>(p, rec, sh.variant == 4, df, sh.direct_grid, stream_));
        if (end) TY_CUDA(cudaEventRecord(end, stream_));
        return kOk;
    }
    if (sh.schedule == 2) {
        const LevelArgs p = level_args(prec, iso, qang, d_psi_);
        DataflowArgs df;
        df.done = d_done_;
        df.err = d_ctl_;
        df.abort = d_ctl_ + 3;
        df.epoch = d_ctl_ + 4;
        df.n_items = sched_.n_padded;
        df.spin_limit = spin_limit_;
        TY_CUDA(launch_bump_epoch(d_ctl_ + 4, stream_));
        if (beg) TY_CUDA(cudaEventRecord(beg, stream_));
        TY_CHECK(launch_dataflow_shape(prec, p, df, stream_, err));
        if (end) TY_CUDA(cudaEventRecord(end, stream_));
        return kOk;
    }
    LevelGraph *lg = nullptr;
    TY_CHECK(level_graph(prec, has_iso, qang, lg, err));
    if (beg) TY_CUDA(cudaEventRecord(beg, stream_));
    TY_CUDA(cudaGraphLaunch(lg->exec, stream_));
    if (end) TY_CUDA(cudaEventRecord(end, stream_));
    return kOk;
}

// The level schedule's launches on stream_ (into a capture): one chain of
// level launches per octant group, each on its own stream, forked from and
// joined into stream_; consecutive levels of a chain use programmatic
// dependent launch.
cudaError_t Sweeper::enqueue_levels(int prec, bool has_iso, const double *qang)
{
    const void *iso = has_iso ? (prec ? (const void *)d_iso32_ : (const void *)d_iso_) : nullptr;
    const LaunchShape &sh = shape_[prec ? 1 : 0];
    const LevelArgs p = level_args(prec, iso, qang, d_psi_);
    cudaError_t le = cudaSuccess;
    const int S = sh.streams;
    if (S > 1) le = cudaEventRecord(fork_, stream_);
    for (int g = 0; g < S && le == cudaSuccess; ++g) {
        cudaStream_t st = S > 1 ? aux_[g] : stream_;
        if (S > 1) le = cudaStreamWaitEvent(st, fork_, 0);
        for (uint32_t l = 0; l < sched_.n_levels && le == cudaSuccess; ++l) {
            const uint64_t b = sched_.octant_offset[(size_t)l * kOctants + g * kOctants / S];
            const uint64_t e = sched_.octant_offset[(size_t)l * kOctants + (g + 1) * kOctants / S];
            if (e <= b) continue;
            if (sh.variant == 0)
                le = prec ? launch_level<float>(sh.knob, p, b, e, st)
                          : launch_level<double>(sh.knob, p, b, e, st);
            else if (sh.variant == 1)
                le = prec ? launch_level_tile<float>(sh.knob, p, b, e, st)
                          : launch_level_tile<double>(sh.knob, p, b, e, st);
            else if (sh.variant == 2)
                le = prec ? launch_level_record<float>(sh.knob, p, d_rec_[1], b, e, st)
                          : launch_level_record<double>(sh.knob, p, d_rec_[0], b, e, st);
            else if (sh.variant == 3)
                le = prec ? launch_direct_level<float>(sh.knob, p, d_rec_[1], b, e, st, false)
                          : launch_direct_level<double>(sh.knob, p, d_rec_[0], b, e, st, false);
            else
                le = prec ? launch_direct_level<float>(sh.knob, p, d_crec_[1], b, e, st, true)
                          : launch_direct_level<double>(sh.knob, p, d_crec_[0], b, e, st, true);
        }
        if (S > 1 && le == cudaSuccess) le = cudaEventRecord(join_[g], st);
        if (S > 1 && le == cudaSuccess) le = cudaStreamWaitEvent(stream_, join_[g], 0);
    }
    return le;
}

int Sweeper::level_graph(int prec, bool has_iso, const double *qang, LevelGraph *&lg, std::string &err)
{
    const LaunchShape &sh = shape_[prec ? 1 : 0];
    if (sh.schedule != 1) { err = "no level graph for this schedule"; return kErrArg; }
    if (sh.variant >= 2) TY_CHECK(ensure_records(prec, true, err, sh.variant == 4));
    auto key = std::make_tuple(prec, has_iso, qang);
    auto it = graphs_.find(key);
    if (it == graphs_.end()) {
        cudaGraph_t graph;
        TY_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        const cudaError_t le = enqueue_levels(prec, has_iso, qang);
        cudaError_t ce = cudaStreamEndCapture(stream_, &graph);
        TY_CUDA(le);
        TY_CUDA(ce);
        cudaGraphExec_t exec;
        cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        TY_CUDA(ie);
        LevelGraph g;
        g.exec = exec;
        it = graphs_.emplace(key, g).first;
    }
    lg = &it->second;
    return kOk;
}

int Sweeper::capture_apply(int prec, const double *phi_in, bool with_fixed, double *phi_out, std::string &err)
{
    const double *qang = with_fixed ? d_qang_ : nullptr;
    const double *qfix = with_fixed ? d_qiso_ : nullptr;
    const bool has_iso = phi_in != nullptr || qfix != nullptr;
    LevelGraph *lg = nullptr;
    TY_CHECK(level_graph(prec, has_iso, qang, lg, err));  // cached: nothing is captured here
    if (has_iso)
        TY_CUDA(launch_scatter_source(phi_in, qfix, d_sigs_, d_scat_, d_iso_, prec ? d_iso32_ : nullptr, nc_,
                                      (uint32_t)G_, stream_));
    // the level launches themselves (not the level graph as a child node:
    // a child graph loses the programmatic edges between its levels)
    TY_CUDA(enqueue_levels(prec, has_iso, qang));
    if (phi_out)
        TY_CUDA(launch_psi_to_phi(d_psi_, prec == 1, d_w_, phi_out, nc_, (uint32_t)A_, (uint32_t)G_, stream_));
    return kOk;
}

int Sweeper::si_step_graph(cudaGraphExec_t &exec, std::string &err)
{
    exec = nullptr;
    if (shape_[0].schedule != 1) return kOk;
    auto key = std::make_tuple(0, 0, 0);
    auto it = step_graphs_.find(key);
    if (it != step_graphs_.end()) { exec = it->second; return kOk; }
    LevelGraph *lg = nullptr;
    TY_CHECK(level_graph(0, true, d_qang_, lg, err));
    const uint64_t n = phi_size();
    // phi_old = phi; phi = T(phi_old); the L1 change and norm to the host
    cudaGraph_t graph;
    TY_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    int st = kOk;
    cudaError_t e = cudaMemcpyAsync(d_tmp_, d_phi_, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_);
    if (e == cudaSuccess) st = capture_apply(0, d_tmp_, true, d_phi_, err);
    if (e == cudaSuccess && st == kOk) e = l1_pair_dev(d_phi_, d_tmp_, n, red_, red_.result, stream_);
    if (e == cudaSuccess && st == kOk)
        e = cudaMemcpyAsync(red_.host, red_.result, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream_);
    cudaError_t ce = cudaStreamEndCapture(stream_, &graph);
    TY_CHECK(st);
    TY_CUDA(e);
    TY_CUDA(ce);
    cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    TY_CUDA(ie);
    step_graphs_.emplace(key, exec);
    TY_CUDA(cudaGraphUpload(exec, stream_));  // its first launch then pays no upload
    return kOk;
}

// Arnoldi step k of GMRES(m) with the precision-prec operator: w = V_{k+1} =
// (I - K) V_k, classical Gram-Schmidt twice against V_0..V_k (coefficients
// to result[0..k] and result[64..64+k]), ||w||^2 to result[128], w
// normalized, its norm to result[129]; result[0..130) to the host.
int Sweeper::arnoldi_step_graph(int prec, int k, cudaGraphExec_t &exec, std::string &err)
{
    exec = nullptr;
    if (shape_[prec ? 1 : 0].schedule != 1 || k + 1 > 64) return kOk;
    auto key = std::make_tuple(1, prec, k);
    auto it = step_graphs_.find(key);
    if (it != step_graphs_.end()) { exec = it->second; return kOk; }
    LevelGraph *lg = nullptr;
    TY_CHECK(level_graph(prec, true, nullptr, lg, err));
    const uint64_t n = phi_size();
    double *V = d_V_, *vk = V + (size_t)k * n, *w = V + (size_t)(k + 1) * n, *res = red_.result;
    cudaGraph_t graph;
    TY_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    int st = capture_apply(prec, vk, false, w, err);
    cudaError_t e = cudaSuccess;
    if (st == kOk) e = sub_from(vk, w, n, stream_);
    for (int pass = 0; pass < 2 && st == kOk && e == cudaSuccess; ++pass) {
        e = multi_dot_dev(w, V, n, k + 1, n, red_, res + 64 * pass, stream_);
        if (e == cudaSuccess) e = multi_axpy(w, V, n, res + 64 * pass, k + 1, n, stream_);
    }
    if (st == kOk && e == cudaSuccess) e = multi_dot_dev(w, w, n, 1, n, red_, res + 128, stream_);
    if (st == kOk && e == cudaSuccess) e = scale_by_norm(w, n, res + 128, res + 129, stream_);
    if (st == kOk && e == cudaSuccess)
        e = cudaMemcpyAsync(red_.host, res, sizeof(double) * 130, cudaMemcpyDeviceToHost, stream_);
    cudaError_t ce = cudaStreamEndCapture(stream_, &graph);
    TY_CHECK(st);
    TY_CUDA(e);
    TY_CUDA(ce);
    cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    TY_CUDA(ie);
    step_graphs_.emplace(key, exec);
    TY_CUDA(cudaGraphUpload(exec, stream_));  // its first launch then pays no upload
    return kOk;
}

static thread_local cudaEvent_t tl_level_beg = nullptr, tl_level_end = nullptr;

int Sweeper::apply(int prec, const double *phi_in, bool with_fixed, double *phi_out,
                   const double *qang_override, std::string &err)
{
    if (!have_xs_) { err = "cross sections not set"; return kErrMissing; }
    if (prec == 1 && !fp32_) { err = "sweeper was created without the FP32 sweep"; return kErrArg; }
    const double *qang = qang_override ? qang_override : (with_fixed ? d_qang_ : nullptr);
    if (prec == 1 && qang) { err = "the FP32 sweep takes isotropic sources only"; return kErrArg; }
    const double *qfix = with_fixed ? d_qiso_ : nullptr;
    const bool has_iso = phi_in != nullptr || qfix != nullptr;
    if (has_iso)
        TY_CUDA(launch_scatter_source(phi_in, qfix, d_sigs_, d_scat_, d_iso_, prec ? d_iso32_ : nullptr,
                                      nc_, (uint32_t)G_, stream_));
    TY_CHECK(levels(prec, has_iso, qang, tl_level_beg, tl_level_end, err));
    if (phi_out) TY_CUDA(launch_psi_to_phi(d_psi_, prec == 1, d_w_, phi_out, nc_, (uint32_t)A_, (uint32_t)G_, stream_));
    last_psi_prec_ = prec;
    return kOk;
}

int Sweeper::apply_external(int prec, const double *phi_in, bool with_fixed, double *phi_out, cudaStream_t s,
                            std::string &err)
{
    TY_CUDA(cudaSetDevice(device_));
    if (prec == 1 && !fp32_) { err = "sweeper was created without the FP32 sweep"; return kErrArg; }
    cudaEvent_t ev;
    TY_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ev, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream_, ev, 0);
    cudaEventDestroy(ev);
    TY_CUDA(e);
    TY_CHECK(apply(prec, phi_in, with_fixed, phi_out, nullptr, err));
    TY_CUDA(cudaStreamSynchronize(stream_));
    return check_device_error(err);
}

// Chunks of the drop-in sweep: large psi (copies of ~0.1 s and more over
// PCIe) is moved and swept in K contiguous angle ranges, so that uploading
// chunk j+1 and downloading chunk j-1 overlap the sweep of chunk j and each
// other; small problems keep one copy each way (a chunk's level launches
// would cost more than the overlap saves).
int Sweeper::host_chunks() const
{
    if (solver_ != kSolveNoPivot || !have_xs_) return 1;
    const uint64_t bytes = psi_size() * sizeof(double);
    const int K = bytes >= (1ull << 30) ? kMaxHostChunks : bytes >= (64ull << 20) ? 4 : 1;
    return std::min(K, A_);
}

// Each angle is swept independently (the upwind values of an item come from
// the same angle), so chunk j's sweep needs only chunk j's source and
// writes only chunk j's psi.  Chunk j's angles are contiguous in every
// cell's row of the reference layout: one strided (2D) copy per chunk and
// direction.  Chunk j sweeps its items level by level in schedule order
// (the same per-item arithmetic and results as the whole sweep).
namespace {

// Page-locked (or registered) host memory: copies from and to it run
// asynchronously, so chunks in the two directions can overlap.  Pageable
// memory is staged through page-locked buffers (sweep_host_chunked).
bool page_locked(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// One row of a staged copy.  The staging copies stream gigabytes through
// host memory while both DMA directions use it too; with 16-byte aligned
// destinations they store around the caches (non-temporal stores: no read
// of the destination lines before they are written), else plain memcpy.
// The caller fences (stream_fence) before the data is handed on.
inline void copy_row(char *dst, const char *src, size_t n)
{
#if defined(__SSE2__)
    if ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0 && (n & 15u) == 0) {
        __m128i *d = reinterpret_cast<__m128i *>(dst);
        const __m128i *s = reinterpret_cast<const __m128i *>(src);
        const size_t k = n / 16;
        size_t i = 0;
        for (; i + 4 <= k; i += 4) {
            const __m128i a = _mm_loadu_si128(s + i), b = _mm_loadu_si128(s + i + 1);
            const __m128i c = _mm_loadu_si128(s + i + 2), e = _mm_loadu_si128(s + i + 3);
            _mm_stream_si128(d + i, a);
            _mm_stream_si128(d + i + 1, b);
            _mm_stream_si128(d + i + 2, c);
            _mm_stream_si128(d + i + 3, e);
        }
        for (; i < k; ++i) _mm_stream_si128(d + i, _mm_loadu_si128(s + i));
        return;
    }
#endif
    std::memcpy(dst, src, n);
}

inline void stream_fence()
{
#if defined(__SSE2__)
    _mm_sfence();
#endif
}

}  // namespace

int Sweeper::sweep_host_chunked(const double *source, double *psi, int K, std::string &err)
{
    TY_CHECK(ensure_records(0, true, err, true));  // kErrOom before any copy
    if (chunk_k_ != K) {
        for (auto &g : chunk_graphs_)
            if (g) cudaGraphExecDestroy(g);
        chunk_graphs_.clear();
        dev_free(d_chunk_pos_, stream_);
        d_chunk_pos_ = nullptr;
        chunk_k_ = 0;
        TY_CHECK(angle_chunks_device(d_items_, sched_.n_padded, d_level_off_, sched_.n_levels, (uint32_t)A_,
                                     (uint32_t)K, &d_chunk_pos_, chunk_off_, stream_, err));
        chunk_graphs_.assign(K, nullptr);
        chunk_k_ = K;
    }
    if (!h2d_stream_) TY_CUDA(cudaStreamCreateWithFlags(&h2d_stream_, cudaStreamNonBlocking));
    if (!d2h_stream_) TY_CUDA(cudaStreamCreateWithFlags(&d2h_stream_, cudaStreamNonBlocking));
    if (!ev_start_) TY_CUDA(cudaEventCreateWithFlags(&ev_start_, cudaEventDisableTiming));
    for (int j = 0; j < K; ++j) {
        if (!ev_h2d_[j]) TY_CUDA(cudaEventCreateWithFlags(&ev_h2d_[j], cudaEventDisableTiming));
        if (!ev_swept_[j]) TY_CUDA(cudaEventCreateWithFlags(&ev_swept_[j], cudaEventDisableTiming));
    }
    const uint32_t n_levels = sched_.n_levels;
    for (int j = 0; j < K; ++j) {
        if (chunk_graphs_[j]) continue;
        LevelArgs p = level_args(0, nullptr, d_src_, d_psi_);
        p.vg = G_ % 2 == 0 ? 2u : 1u;
        p.vmagic = group_magic((uint32_t)G_ / p.vg);
        cudaGraph_t graph;
        TY_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        cudaError_t le = cudaSuccess;
        for (uint32_t l = 0; l < n_levels && le == cudaSuccess; ++l)
            le = launch_direct_subset<double>(p, d_crec_[0], d_chunk_pos_, chunk_off_[(size_t)j * n_levels + l],
                                              chunk_off_[(size_t)j * n_levels + l + 1], stream_);
        cudaError_t ce = cudaStreamEndCapture(stream_, &graph);
        TY_CUDA(le);
        TY_CUDA(ce);
        cudaError_t ie = cudaGraphInstantiate(&chunk_graphs_[j], graph, 0);
        cudaGraphDestroy(graph);
        TY_CUDA(ie);
    }
    // Pageable host buffers go through two page-locked staging buffers per
    // direction, in pieces of at most kStageBytes: the calling thread gathers
    // a piece of the source (OpenMP threads over the rows) while the previous
    // piece uploads; a second host thread scatters downloaded pieces of psi
    // while the next one downloads.  Page-locked buffers are copied directly.
    const bool stage_in = !page_locked(source), stage_out = !page_locked(psi);
    if ((stage_in || stage_out) && !h_stage_[0]) {
        cudaError_t ae = cudaSuccess;
        for (auto &b : h_stage_)
            if (ae == cudaSuccess) ae = cudaHostAlloc(&b, kStageBytes, cudaHostAllocPortable);
        if (ae != cudaSuccess) {  // no page-locked memory to spare: the one-copy form
            cudaGetLastError();
            for (auto &b : h_stage_) {
                if (b) cudaFreeHost(b);
                b = nullptr;
            }
            err = "no page-locked staging memory";
            return kErrOom;
        }
        for (auto &e : ev_stage_) TY_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    // after whatever ran on the sweeper's stream before
    TY_CUDA(cudaEventRecord(ev_start_, stream_));
    TY_CUDA(cudaStreamWaitEvent(h2d_stream_, ev_start_, 0));
    TY_CUDA(cudaStreamWaitEvent(d2h_stream_, ev_start_, 0));
    const size_t per_angle = (size_t)4 * G_ * sizeof(double), row = per_angle * A_;
    auto span = [&](int j, size_t &off, size_t &width) {
        const size_t a0 = (size_t)j * A_ / K, a1 = (size_t)(j + 1) * A_ / K;
        off = a0 * per_angle;
        width = (a1 - a0) * per_angle;
    };
    const int nt = std::max(1, omp_get_max_threads() / (stage_in && stage_out ? 2 : 1));
    // rows [r0, r1) of the chunk's columns [off, off + width) to or from a
    // packed staging buffer
    auto pack = [&](char *dst, const char *src, size_t off, size_t width, uint64_t r0, uint64_t r1) {
#pragma omp parallel num_threads(nt)
        {
#pragma omp for schedule(static)
            for (int64_t r = (int64_t)r0; r < (int64_t)r1; ++r)
                copy_row(dst + (size_t)(r - r0) * width, src + (size_t)r * row + off, width);
            stream_fence();
        }
    };
    auto unpack = [&](char *dst, const char *src, size_t off, size_t width, uint64_t r0, uint64_t r1) {
#pragma omp parallel num_threads(nt)
        {
#pragma omp for schedule(static)
            for (int64_t r = (int64_t)r0; r < (int64_t)r1; ++r)
                copy_row(dst + (size_t)r * row + off, src + (size_t)(r - r0) * width, width);
            stream_fence();
        }
    };
    // the downloading side: in this thread when psi is page-locked (plain
    // asynchronous copies), else on a helper thread that scatters the pieces
    std::mutex mu;
    std::condition_variable cv;
    int swept = 0;  // chunks whose sweep has been enqueued
    cudaError_t out_err = cudaSuccess;
    auto download = [&]() {
        char *dst = reinterpret_cast<char *>(psi);
        const char *dev = reinterpret_cast<const char *>(d_psi_);
        uint64_t q = 0;  // pieces enqueued so far
        struct Pending { size_t off, width; uint64_t r0, r1; } last[2];
        cudaError_t e = cudaSuccess;
        for (int j = 0; j < K && e == cudaSuccess; ++j) {
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return swept > j || out_err != cudaSuccess; });
                if (out_err != cudaSuccess) return;
            }
            size_t off, width;
            span(j, off, width);
            e = cudaStreamWaitEvent(d2h_stream_, ev_swept_[j], 0);
            const uint64_t rows = std::max<uint64_t>(1, kStageBytes / width);
            for (uint64_t r0 = 0; r0 < nc_ && e == cudaSuccess; r0 += rows, ++q) {
                const uint64_t r1 = std::min<uint64_t>(nc_, r0 + rows);
                char *buf = reinterpret_cast<char *>(h_stage_[2 + q % 2]);
                e = cudaMemcpy2DAsync(buf, width, dev + r0 * row + off, row, width, r1 - r0, cudaMemcpyDeviceToHost,
                                      d2h_stream_);
                if (e == cudaSuccess) e = cudaEventRecord(ev_stage_[2 + q % 2], d2h_stream_);
                last[q % 2] = {off, width, r0, r1};
                if (q >= 1 && e == cudaSuccess) {  // the previous piece has landed: scatter it
                    const Pending &pp = last[(q - 1) % 2];
                    e = cudaEventSynchronize(ev_stage_[2 + (q - 1) % 2]);
                    if (e == cudaSuccess)
                        unpack(dst, reinterpret_cast<const char *>(h_stage_[2 + (q - 1) % 2]), pp.off, pp.width, pp.r0,
                               pp.r1);
                }
            }
        }
        if (q >= 1 && e == cudaSuccess) {
            const Pending &pp = last[(q - 1) % 2];
            e = cudaEventSynchronize(ev_stage_[2 + (q - 1) % 2]);
            if (e == cudaSuccess)
                unpack(dst, reinterpret_cast<const char *>(h_stage_[2 + (q - 1) % 2]), pp.off, pp.width, pp.r0, pp.r1);
        }
        std::lock_guard<std::mutex> lk(mu);
        if (out_err == cudaSuccess) out_err = e;
    };
    std::thread helper;
    if (stage_out) helper = std::thread(download);
    cudaError_t e = cudaSuccess;
    uint64_t p = 0;  // source pieces enqueued so far
    for (int j = 0; j < K && e == cudaSuccess; ++j) {
        size_t off, width;
        span(j, off, width);
        if (!stage_in) {
            e = cudaMemcpy2DAsync(reinterpret_cast<char *>(d_src_) + off, row,
                                  reinterpret_cast<const char *>(source) + off, row, width, nc_,
                                  cudaMemcpyHostToDevice, h2d_stream_);
        } else {
            const uint64_t rows = std::max<uint64_t>(1, kStageBytes / width);
            for (uint64_t r0 = 0; r0 < nc_ && e == cudaSuccess; r0 += rows, ++p) {
                const uint64_t r1 = std::min<uint64_t>(nc_, r0 + rows);
                if (p >= 2) e = cudaEventSynchronize(ev_stage_[p % 2]);  // its last upload is done
                if (e != cudaSuccess) break;
                char *buf = reinterpret_cast<char *>(h_stage_[p % 2]);
                pack(buf, reinterpret_cast<const char *>(source), off, width, r0, r1);
                e = cudaMemcpy2DAsync(reinterpret_cast<char *>(d_src_) + r0 * row + off, row, buf, width, width,
                                      r1 - r0, cudaMemcpyHostToDevice, h2d_stream_);
                if (e == cudaSuccess) e = cudaEventRecord(ev_stage_[p % 2], h2d_stream_);
            }
        }
        if (e == cudaSuccess) e = cudaEventRecord(ev_h2d_[j], h2d_stream_);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(stream_, ev_h2d_[j], 0);
        if (e == cudaSuccess) e = cudaGraphLaunch(chunk_graphs_[j], stream_);
        if (e == cudaSuccess) e = cudaEventRecord(ev_swept_[j], stream_);
        if (e == cudaSuccess && !stage_out) {
            e = cudaStreamWaitEvent(d2h_stream_, ev_swept_[j], 0);
            if (e == cudaSuccess)
                e = cudaMemcpy2DAsync(reinterpret_cast<char *>(psi) + off, row,
                                      reinterpret_cast<const char *>(d_psi_) + off, row, width, nc_,
                                      cudaMemcpyDeviceToHost, d2h_stream_);
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            if (e == cudaSuccess) swept = j + 1;
            else if (out_err == cudaSuccess) out_err = e;
        }
        cv.notify_all();
    }
    if (helper.joinable()) helper.join();
    TY_CUDA(e);
    TY_CUDA(out_err);
    TY_CUDA(cudaStreamSynchronize(d2h_stream_));
    TY_CUDA(cudaStreamSynchronize(h2d_stream_));
    TY_CUDA(cudaStreamSynchronize(stream_));
    last_psi_prec_ = 0;
    return check_device_error(err);
}



int Sweeper::sweep_host(const double *source, double *psi, std::string &err)
{
    if (!source || !psi) { err = "source and psi are required"; return kErrArg; }
    TY_CUDA(cudaSetDevice(device_));
    const size_t n = psi_size();
    if (!d_src_) TY_CUDA(dev_malloc(&d_src_, sizeof(double) * n, stream_));
    // page-locked buffers are copied directly, pageable ones through the
    // staging buffers of the chunked form
    const int K = host_chunks();
    if (K > 1) {
        // no room for the chunk plan or the compact FP64 records: one copy
        // each way instead (nothing was copied yet)
        const int st = sweep_host_chunked(source, psi, K, err);
        if (st != kErrOom) return st;
        err.clear();
    }
    TY_CUDA(cudaMemcpyAsync(d_src_, source, sizeof(double) * n, cudaMemcpyHostToDevice, stream_));
    TY_CHECK(apply(0, nullptr, false, nullptr, d_src_, err));
    TY_CUDA(cudaMemcpyAsync(psi, d_psi_, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_));
    TY_CUDA(cudaStreamSynchronize(stream_));
    return check_device_error(err);
}

int Sweeper::ensure_krylov(int m, std::string &err)
{
    if (m < 1 || m > 60) { err = "GMRES restart must be in 1..60"; return kErrArg; }
    if (krylov_m_ >= m) return kOk;
    drop_step_graphs();  // they hold the basis's addresses
    if (d_V_) dev_free(d_V_, stream_);
    d_V_ = nullptr;
    TY_CUDA(dev_malloc(&d_V_, sizeof(double) * phi_size() * (m + 1), stream_));
    if (!d_h_) TY_CUDA(dev_malloc(&d_h_, sizeof(double) * 64, stream_));
    krylov_m_ = m;
    return kOk;
}

// Restarted GMRES(m) on (I - K) x = b, K = D L^{-1} M S swept in `prec`,
// x starting at 0.  Classical Gram-Schmidt applied twice, Givens rotations
// on the host, stop when the residual estimate <= rtol ||b||; the true
// residual is recomputed at each restart.
int Sweeper::gmres(int prec, const double *b, double *x, int m, double rtol, int iter_max, int &its,
                   double &rnorm, SolveStats &st, std::string &err, double *r_out)
{
    TY_CHECK(ensure_krylov(m, err));
    const uint64_t n = phi_size();
    double *V = d_V_;
    its = 0;
    TY_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, stream_));
    TY_CUDA(multi_dot(b, b, n, 1, n, red_, stream_));
    const double bnorm = std::sqrt(red_.host[0]);
    rnorm = bnorm;
    if (bnorm == 0.0) {
        if (r_out) TY_CUDA(cudaMemsetAsync(r_out, 0, sizeof(double) * n, stream_));
        return kOk;
    }
    TY_CUDA(cudaMemcpyAsync(V, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_));
    double beta = bnorm;
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    for (;;) {
        if (beta <= rtol * bnorm || its >= iter_max) {
            rnorm = beta;
            if (r_out) TY_CUDA(cudaMemcpyAsync(r_out, V, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_));
            break;
        }
        TY_CUDA(axpby(1.0 / beta, V, 0.0, V, n, stream_));
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int k = 0;
        bool converged = false;
        double est = beta;
        for (; k < m && its < iter_max;) {
            double *vk = V + (size_t)k * n, *w = V + (size_t)(k + 1) * n;
            // the whole Arnoldi step as one captured graph with the level
            // schedule (one host synchronization for its coefficients)
            cudaGraphExec_t step = nullptr;
            TY_CHECK(arnoldi_step_graph(prec, k, step, err));
            double hn = 0.0;
            for (int j = 0; j <= k; ++j) H[(size_t)j * m + k] = 0.0;
            if (step) {
                TY_CUDA(cudaGraphLaunch(step, stream_));
                TY_CUDA(cudaStreamSynchronize(stream_));
                last_psi_prec_ = prec;
                for (int pass = 0; pass < 2; ++pass)
                    for (int j = 0; j <= k; ++j) H[(size_t)j * m + k] += red_.host[64 * pass + j];
                hn = red_.host[129];
            } else {
                TY_CHECK(apply(prec, vk, false, w, nullptr, err));
                TY_CUDA(sub_from(vk, w, n, stream_));
                for (int pass = 0; pass < 2; ++pass) {
                    TY_CUDA(multi_dot(w, V, n, k + 1, n, red_, stream_));
                    for (int j = 0; j <= k; ++j) H[(size_t)j * m + k] += red_.host[j];
                    TY_CUDA(multi_axpy(w, V, n, red_.result, k + 1, n, stream_));
                }
                TY_CUDA(multi_dot(w, w, n, 1, n, red_, stream_));
                hn = std::sqrt(red_.host[0]);
                if (hn > 0.0) TY_CUDA(axpby(1.0 / hn, w, 0.0, w, n, stream_));
            }
            (prec ? st.sweeps_fp32 : st.sweeps_fp64)++;
            H[(size_t)(k + 1) * m + k] = hn;
            for (int j = 0; j < k; ++j) {
                const double h0 = H[(size_t)j * m + k], h1 = H[(size_t)(j + 1) * m + k];
                H[(size_t)j * m + k] = cs[j] * h0 + sn[j] * h1;
                H[(size_t)(j + 1) * m + k] = -sn[j] * h0 + cs[j] * h1;
            }
            const double hk = H[(size_t)k * m + k];
            const double den = std::hypot(hk, hn);
            cs[k] = den > 0 ? hk / den : 1.0;
            sn[k] = den > 0 ? hn / den : 0.0;
            H[(size_t)k * m + k] = den;
            g[k + 1] = -sn[k] * g[k];
            g[k] = cs[k] * g[k];
            est = std::fabs(g[k + 1]);
            ++its;
            ++k;
            if (est <= rtol * bnorm || hn == 0.0) { converged = true; break; }
        }
        for (int i = k - 1; i >= 0; --i) {
            double s = g[i];
            for (int j = i + 1; j < k; ++j) s -= H[(size_t)i * m + j] * y[j];
            y[i] = s / H[(size_t)i * m + i];
        }
        std::vector<double> negy(k);
        for (int j = 0; j < k; ++j) negy[j] = -y[j];
        TY_CUDA(cudaMemcpyAsync(d_h_, negy.data(), sizeof(double) * k, cudaMemcpyHostToDevice, stream_));
        TY_CUDA(multi_axpy(x, V, n, d_h_, k, n, stream_));
        if (converged || its >= iter_max) {
            rnorm = est;
            if (r_out) {
                // beta e1 - H y = Omega^T (0, ..., 0, g_k): the rotations
                // undone in reverse order; r = V_{0..k} z
                std::vector<double> negz(k + 1, 0.0);
                double zj1 = g[k];
                for (int j = k - 1; j >= 0; --j) {
                    negz[j + 1] = -(cs[j] * zj1);
                    zj1 = -sn[j] * zj1;
                }
                negz[0] = -zj1;
                if (k == 0) negz[0] = -g[0];
                TY_CUDA(cudaMemsetAsync(r_out, 0, sizeof(double) * n, stream_));
                TY_CUDA(cudaMemcpyAsync(d_h_, negz.data(), sizeof(double) * (k + 1), cudaMemcpyHostToDevice, stream_));
                TY_CUDA(multi_axpy(r_out, V, n, d_h_, k + 1, n, stream_));
            }
            TY_CUDA(cudaStreamSynchronize(stream_));
            break;
        }
        // True residual r = b - (x - K x) into V_0.
        TY_CHECK(apply(prec, x, false, V, nullptr, err));
        (prec ? st.sweeps_fp32 : st.sweeps_fp64)++;
        TY_CUDA(sub_from(x, V, n, stream_));
        TY_CUDA(sub_from(b, V, n, stream_));
        TY_CUDA(multi_dot(V, V, n, 1, n, red_, stream_));
        beta = std::sqrt(red_.host[0]);
    }
    return kOk;
}

int Sweeper::solve(const SolveOptions &o, double *phi_out, double *psi_out, SolveStats &st,
                   std::string &err)
{
    TY_CUDA(cudaSetDevice(device_));
    st = SolveStats();
    const uint64_t n = phi_size();
    // the Krylov basis and the captured step graphs are set-up, not solve
    // time: made before the timed region
    if (o.method == 1 || o.method == 2) {
        TY_CHECK(ensure_krylov(o.restart, err));
        const int prec = o.method == 2 ? 1 : 0;
        cudaGraphExec_t g = nullptr;
        for (int k = 0; k < o.restart; ++k) TY_CHECK(arnoldi_step_graph(prec, k, g, err));
    } else if (o.method == 0) {
        cudaGraphExec_t g = nullptr;
        TY_CHECK(si_step_graph(g, err));
    }
    cudaEvent_t e0, e1;
    TY_CUDA(cudaEventCreate(&e0));
    TY_CUDA(cudaEventCreate(&e1));
    TY_CUDA(cudaEventRecord(e0, stream_));
    double *result = nullptr;  // phi consistent with the resident psi
    int status = kOk;
    if (o.method == 0) {
        // SourceIteration::fixedPoint: L1 relative change of phi.
        // each step one captured graph (copy, scattering source, the level
        // graph, psi -> phi, the L1 pair to the host) with the level schedule
        TY_CUDA(cudaMemsetAsync(d_phi_, 0, sizeof(double) * n, stream_));
        cudaGraphExec_t step = nullptr;
        TY_CHECK(si_step_graph(step, err));
        int iter = 0;
        double error = 1.0;
        while (iter < o.iter_max && error > o.err_max) {
            if (step) {
                TY_CUDA(cudaGraphLaunch(step, stream_));
                TY_CUDA(cudaStreamSynchronize(stream_));
                last_psi_prec_ = 0;
            } else {
                TY_CUDA(cudaMemcpyAsync(d_tmp_, d_phi_, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_));
                TY_CHECK(apply(0, d_tmp_, true, d_phi_, nullptr, err));
                TY_CUDA(l1_pair(d_phi_, d_tmp_, n, red_, stream_));
            }
            st.sweeps_fp64++;
            error = red_.host[0] / red_.host[1];
            ++iter;
        }
        st.iterations = iter;
        st.final_error = error;
        result = d_phi_;
    } else if (o.method == 1) {
        // SourceIteration::krylov: b = D L^{-1} Q, GMRES, psi = L^{-1}(MS phi + Q)
        // (the last sweep only when psi is asked for; phi is then that psi's).
        TY_CHECK(apply(0, nullptr, true, d_r_, nullptr, err));
        st.sweeps_fp64++;
        int its = 0;
        double rn = 0;
        TY_CHECK(gmres(0, d_r_, d_phi_, o.restart, o.err_max, o.iter_max, its, rn, st, err));
        TY_CUDA(multi_dot(d_r_, d_r_, n, 1, n, red_, stream_));
        const double bnorm = std::sqrt(red_.host[0]);
        st.iterations = its;
        st.final_error = bnorm > 0 ? rn / bnorm : 0.0;
        result = d_phi_;
        if (psi_out) {  // psi = L^{-1}(M S phi + Q), src/SourceIteration.cc:254-260
            TY_CHECK(apply(0, d_phi_, true, d_tmp_, nullptr, err));
            st.sweeps_fp64++;
            result = d_tmp_;
        }
    } else if (o.method == 2) {
        // FP64 iterative refinement around FP32-sweep GMRES, with as few FP64
        // sweeps as the FP32 sweep's accuracy allows:
        //  1. x = 0 refined against the FP32 sweep of the fixed source
        //     b32 = D L32^{-1} Q: (I - K32) x = b32 to min(inner_tol, 1e-6);
        //  2. r = T64(x) - x, one FP64 sweep (T = D L^{-1} (Q + M S .));
        //  3. (I - K32) d = r by GMRES, x += d; the new residual r - (I - K32) d
        //     comes from the GMRES Arnoldi relation, without a sweep, when the
        //     FP32 operator's error on d (at most kFp32OpErr ||d||) is below a
        //     tenth of the tolerance; otherwise back to 2.
        // Stop when ||r|| <= errMax ||b32||.  psi_out: one more FP64 sweep at
        // the final x unless the last step was one.
        if (!fp32_) { err = "mixed precision needs a sweeper created with fp32"; return kErrArg; }
        if (d_qang_) { err = "mixed precision takes an isotropic fixed source"; return kErrArg; }
        // relative error of one FP32 operator application (measured 3-7e-8
        // in phi, 2-3e-7 in psi; a margin of 30)
        constexpr double kFp32OpErr = 2e-6;
        TY_CUDA(cudaMemsetAsync(d_phi_, 0, sizeof(double) * n, stream_));
        TY_CHECK(apply(1, nullptr, true, d_r_, nullptr, err));
        st.sweeps_fp32++;
        TY_CUDA(multi_dot(d_r_, d_r_, n, 1, n, red_, stream_));
        const double bnorm = std::sqrt(red_.host[0]);
        double rnorm = bnorm;
        int ref = 0;
        bool at_t64 = false;  // d_tmp_ holds T64(x) and psi is its FP64 sweep
        if (bnorm > 0.0) {
            int its = 0;
            double rn = 0;
            TY_CHECK(gmres(1, d_r_, d_phi_, o.restart, std::min(o.inner_tol, 1e-6), o.iter_max, its, rn, st, err));
            st.iterations += its;
            bool need_true = true;
            for (;;) {
                if (need_true) {
                    TY_CHECK(apply(0, d_phi_, true, d_tmp_, nullptr, err));
                    st.sweeps_fp64++;
                    at_t64 = true;
                    TY_CUDA(cudaMemcpyAsync(d_r_, d_tmp_, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_));
                    TY_CUDA(axpby(-1.0, d_phi_, 1.0, d_r_, n, stream_));
                    TY_CUDA(multi_dot(d_r_, d_r_, n, 1, n, red_, stream_));
                    rnorm = std::sqrt(red_.host[0]);
                }
                if (rnorm <= o.err_max * bnorm || ref >= o.refine_max || st.iterations >= o.iter_max) break;
                const double rtol = std::max(0.5 * o.err_max * bnorm / rnorm, 1e-8);
                its = 0;
                TY_CHECK(gmres(1, d_r_, d_tmp_, o.restart, rtol, o.iter_max - st.iterations, its, rn, st, err,
                               d_r_));
                at_t64 = false;
                st.iterations += its;
                TY_CUDA(axpby(1.0, d_tmp_, 1.0, d_phi_, n, stream_));
                ++ref;
                TY_CUDA(multi_dot(d_tmp_, d_tmp_, n, 1, n, red_, stream_));
                const double dnorm = std::sqrt(red_.host[0]);
                need_true = kFp32OpErr * dnorm > 0.1 * o.err_max * bnorm;
                if (!need_true) {
                    TY_CUDA(multi_dot(d_r_, d_r_, n, 1, n, red_, stream_));
                    rnorm = std::sqrt(red_.host[0]);
                }
            }
        }
        if (!at_t64 && psi_out) {
            TY_CHECK(apply(0, d_phi_, true, d_tmp_, nullptr, err));
            st.sweeps_fp64++;
            at_t64 = true;
        }
        st.refinements = ref;
        st.final_error = bnorm > 0 ? rnorm / bnorm : 0.0;
        result = at_t64 ? d_tmp_ : d_phi_;
    } else {
        err = "unknown method";
        return kErrArg;
    }
    TY_CUDA(cudaEventRecord(e1, stream_));
    TY_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    st.seconds = ms * 1e-3;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (result != d_phi_) TY_CUDA(cudaMemcpyAsync(d_phi_, result, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_));
    if (phi_out) TY_CUDA(cudaMemcpyAsync(phi_out, d_phi_, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_));
    if (psi_out) TY_CUDA(cudaMemcpyAsync(psi_out, d_psi_, sizeof(double) * psi_size(), cudaMemcpyDeviceToHost, stream_));
    TY_CUDA(cudaStreamSynchronize(stream_));
    if (status == kOk) status = check_device_error(err);
    return status;
}

int Sweeper::read_psi(double *psi, std::string &err)
{
    if (!psi) { err = "psi is required"; return kErrArg; }
    if (last_psi_prec_ != 0) { err = "no FP64 psi resident (run a solve or an FP64 sweep first)"; return kErrMissing; }
    TY_CUDA(cudaSetDevice(device_));
    TY_CUDA(cudaMemcpyAsync(psi, d_psi_, sizeof(double) * psi_size(), cudaMemcpyDeviceToHost, stream_));
    TY_CUDA(cudaStreamSynchronize(stream_));
    return kOk;
}

int Sweeper::write_psi(const std::string &path, std::string &err)
{
    if (last_psi_prec_ != 0) { err = "no FP64 psi resident (run a solve or an FP64 sweep first)"; return kErrMissing; }
    TY_CUDA(cudaSetDevice(device_));
    std::vector<double> psi(psi_size());
    TY_CUDA(cudaMemcpyAsync(psi.data(), d_psi_, sizeof(double) * psi.size(), cudaMemcpyDeviceToHost, stream_));
    TY_CUDA(cudaStreamSynchronize(stream_));
    FILE *fp = std::fopen(path.c_str(), "wb");
    if (!fp) { err = "cannot open " + path; return kErrIO; }
    // PsiData::writeToFile (src/PsiData.cc:62-106): 32-byte name, version 1,
    // cells, angles, groups, then psi cell by cell at global offsets.
    char name[32] = "Tycho 2 Psi Output";
    uint64_t hdr[4] = {1, nc_, (uint64_t)A_, (uint64_t)G_};
    bool ok = std::fwrite(name, 1, 32, fp) == 32 && std::fwrite(hdr, 8, 4, fp) == 4;
    const size_t per = (size_t)A_ * 4 * G_;
    for (uint64_t c = 0; c < nc_ && ok; ++c) {
        ok = std::fseek(fp, (long)(64 + tables_->cell_gid[c] * per * 8), SEEK_SET) == 0 &&
             std::fwrite(&psi[c * per], 8, per, fp) == per;
    }
    std::fclose(fp);
    if (!ok) { err = "write failed: " + path; return kErrIO; }
    return kOk;
}

uint64_t Sweeper::launches_per_apply(int prec) const
{
    const LaunchShape &sh = shape_[prec ? 1 : 0];
    uint64_t sweep = 0;
    if (sh.schedule == 1) {
        const int S = sh.streams;
        for (uint32_t l = 0; l < sched_.n_levels; ++l)
            for (int g = 0; g < S; ++g) {
                const uint64_t b = sched_.octant_offset[(size_t)l * kOctants + g * kOctants / S];
                const uint64_t e = sched_.octant_offset[(size_t)l * kOctants + (g + 1) * kOctants / S];
                sweep += e > b;
            }
    } else {
        sweep = sh.schedule == 2 ? 2 : 1;  // dataflow: epoch bump + the sweep
    }
    return sweep + 2;  // the scattering source before, psi -> phi after
}

int Sweeper::time_sweeps(int prec, int n, bool flush_l2, double *ms, std::string &err)
{
    TY_CUDA(cudaSetDevice(device_));
    if (n < 1) { err = "n must be >= 1"; return kErrArg; }
    const size_t flush_bytes = 256ull << 20;  // > 126 MB L2
    if (flush_l2 && !d_flush_) TY_CUDA(dev_malloc(&d_flush_, flush_bytes, stream_));
    cudaEvent_t e0, e1, l0, l1;
    TY_CUDA(cudaEventCreate(&e0));
    TY_CUDA(cudaEventCreate(&e1));
    TY_CUDA(cudaEventCreate(&l0));
    TY_CUDA(cudaEventCreate(&l1));
    double tot = 0, lvl = 0;
    int status = kOk;
    for (int i = 0; i < n && status == kOk; ++i) {
        if (flush_l2) TY_CUDA(cudaMemsetAsync(d_flush_, i & 0xff, flush_bytes, stream_));
        TY_CUDA(cudaEventRecord(e0, stream_));
        tl_level_beg = l0;
        tl_level_end = l1;
        status = apply(prec, d_phi_, true, d_r_, nullptr, err);
        tl_level_beg = tl_level_end = nullptr;
        TY_CUDA(cudaEventRecord(e1, stream_));
        TY_CUDA(cudaEventSynchronize(e1));
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, e0, e1);
        cudaEventElapsedTime(&b, l0, l1);
        tot += a;
        lvl += b;
    }
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(l0); cudaEventDestroy(l1);
    if (status == kOk) status = check_device_error(err);
    ms[0] = tot / n;
    ms[1] = lvl / n;
    return status;
}

}  // namespace tycho
