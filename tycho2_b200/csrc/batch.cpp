// Batched solves: host side (member state machines, slot tables, pass graphs).
#include "batch.hpp"

#include <algorithm>
#include <cmath>

#include "device_ops.hpp"
#include "devmem.hpp"
#include "status.hpp"

namespace tycho {

#define TB_CUDA(expr)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (expr);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            err = std::string(#expr) + ": " + cudaGetErrorString(e_);                  \
            return e_ == cudaErrorMemoryAllocation ? kErrOom : kErrCuda;               \
        }                                                                              \
    } while (0)

#define TB_CHECK(expr)            \
    do {                          \
        int s_ = (expr);          \
        if (s_ != kOk) return s_; \
    } while (0)

namespace {

constexpr unsigned kStreamGrid = 148 * 8;     // blocks of the grid-stride streaming kernels
constexpr unsigned kLevelGridCap = 148 * 16;  // level kernels loop beyond this
// Relative error of one FP32 operator application, used to decide when a
// correction is small enough to be accepted without an FP64 residual sweep
// (measured on B200: 2-3e-7 relative L1 / L2 in psi, 3-7e-8 in phi, over
// S4-S8, G = 1..8, 4^3-24^3 meshes; the bound keeps a margin of 30).
constexpr double kFp32OpErr = 2e-6;

uint32_t magic(uint32_t d) { return d == 1 ? 0u : (uint32_t)(((1ull << 32) + d - 1) / d); }


}  // namespace

Batch::~Batch()
{
    cudaSetDevice(device_);
    for (auto &g : graph_)
        if (g) cudaGraphExecDestroy(g);
    for (auto &m : members_) {
        dev_release(m.r, stream_);
        dev_release(m.d, stream_);
        dev_release(m.k, stream_);
    }
    for (int p = 0; p < 2; ++p) {
        dev_release(d_slots_[p], stream_);
        if (h_slots_[p]) cudaFreeHost(h_slots_[p]);
    }
    if (h_norms_) cudaFreeHost(h_norms_);
    for (auto &pl : plan_) {
        dev_release(pl.segs, stream_);
        dev_release(pl.level_nseg, stream_);
        dev_release(pl.level_nchunk, stream_);
        dev_release(pl.act, stream_);
        dev_release(pl.chunk_prefix, stream_);
        dev_release(pl.n_act, stream_);
        dev_release(pl.partials, stream_);
    }
    dev_release(norms_, stream_);
    for (int p = 0; p < 2; ++p) {
        dev_release(d_barrier_[p], stream_);
        dev_release(d_queue_[p], stream_);
    }
    dev_release(d_ctl_, stream_);
    for (auto &e : ev_)
        if (e) cudaEventDestroy(e);
    if (join_) cudaEventDestroy(join_);
    if (stream32_) cudaStreamDestroy(stream32_);
    if (stream_) cudaStreamDestroy(stream_);
}

int Batch::init(int device, int ipw32, int ipw64, std::string &err)
{
    for (int ipw : {ipw32, ipw64})
        if (ipw != 0 && ipw != 8 && ipw != 16 && ipw != 32) {
            err = "items per warp must be 8, 16 or 32 (0: direct kernel)";
            return kErrArg;
        }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        err = "no CUDA device: the batched sweep has no CPU fallback";
        return kErrCuda;
    }
    if (device < 0 || device >= ndev) { err = "bad device ordinal"; return kErrArg; }
    device_ = device;
    ipw_[0] = ipw64;
    ipw_[1] = ipw32;
    TB_CUDA(cudaSetDevice(device_));
    TB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    TB_CUDA(cudaStreamCreateWithFlags(&stream32_, cudaStreamNonBlocking));
    for (auto &e : ev_) TB_CUDA(cudaEventCreate(&e));
    TB_CUDA(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming));
    return kOk;
}

void Batch::invalidate()
{
    for (auto &g : graph_)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

int Batch::add(Sweeper *sw, const BatchOptions &o, int &id, std::string &err)
{
    if (!sw) { err = "null sweeper"; return kErrArg; }
    if (sw->device() != device_) { err = "sweeper lives on another device than the batch"; return kErrArg; }
    if (o.method != 0 && o.method != 2) { err = "batch method must be 0 (source iteration) or 2 (mixed)"; return kErrArg; }
    if (o.iter_max < 1 || o.err_max < 0 || o.inner_tol <= 0 || o.inner_max < 1 || o.refine_max < 0) {
        err = "bad batch solve options";
        return kErrArg;
    }
    for (const auto &m : members_)
        if (m.sw == sw) { err = "sweeper is already in the batch"; return kErrArg; }
    if (sw->solver() != kSolveNoPivot && (ipw_[0] != 0 || (o.method == 2 && ipw_[1] != 0))) {
        err = "GaussElim Original / Cramer members need the direct batch kernels (items per warp 0)";
        return kErrArg;
    }
    TB_CUDA(cudaSetDevice(device_));
    Member m;
    m.sw = sw;
    m.o = o;
    TB_CHECK(sw->device_view(0, m.v[0], err, ipw_[0] == 0));
    if (o.method == 2) {
        TB_CHECK(sw->device_view(1, m.v[1], err, ipw_[1] == 0));
        const size_t n = sw->phi_size();
        TB_CUDA(dev_malloc(&m.r, sizeof(double) * n, stream_));
        TB_CUDA(dev_malloc(&m.d, sizeof(double) * n, stream_));
        TB_CUDA(dev_malloc(&m.k, sizeof(double) * n, stream_));
        m.state = kRunFirst;
    } else {
        m.v[1] = m.v[0];
        m.state = kRunSI;
    }
    m.cur = m.v[0].phi;
    m.nxt = m.v[0].tmp;
    TB_CUDA(cudaMemsetAsync(m.v[0].phi, 0, sizeof(double) * sw->phi_size(), stream_));
    m.updates = sw->n_cells() * (uint64_t)sw->n_angles() * (uint64_t)sw->n_groups();
    m.id = next_id_++;
    id = m.id;
    members_.push_back(m);
    invalidate();
    return kOk;
}

int Batch::remove(int id, std::string &err)
{
    for (size_t i = 0; i < members_.size(); ++i)
        if (members_[i].id == id) {
            TB_CUDA(cudaSetDevice(device_));
            TB_CUDA(cudaStreamSynchronize(stream_));
            dev_release(members_[i].r, stream_);
            dev_release(members_[i].d, stream_);
            dev_release(members_[i].k, stream_);
            members_.erase(members_.begin() + (long)i);
            invalidate();
            return kOk;
        }
    err = "no batch member with that id";
    return kErrArg;
}

int Batch::ensure_capacity(std::string &err)
{
    const size_t n = members_.size();
    uint32_t lv = 0;
    size_t chunks = 0;
    for (const auto &m : members_) {
        lv = std::max(lv, m.v[0].n_levels);
        chunks += (m.sw->phi_size() + kBatchChunk - 1) / kBatchChunk;
    }
    max_levels_ = lv;
    if (n > cap_slots_ || lv > cap_levels_) {
        const size_t cs = std::max(n, cap_slots_ * 2 > 16 ? cap_slots_ * 2 : (size_t)16);
        const size_t cl = std::max((size_t)lv, cap_levels_);
        for (int p = 0; p < 2; ++p) {
            dev_release(d_slots_[p], stream_);
            if (h_slots_[p]) cudaFreeHost(h_slots_[p]);
            h_slots_[p] = nullptr;
            TB_CUDA(dev_malloc(&d_slots_[p], sizeof(BatchSlot) * cs, stream_));
            TB_CUDA(cudaMallocHost(&h_slots_[p], sizeof(BatchSlot) * cs));
        }
        if (h_norms_) cudaFreeHost(h_norms_);
        h_norms_ = nullptr;
        TB_CUDA(cudaMallocHost(&h_norms_, sizeof(double) * 2 * cs));
        dev_release(norms_, stream_);
        TB_CUDA(dev_malloc(&norms_, sizeof(double) * 2 * cs, stream_));
        TB_CUDA(cudaMemsetAsync(norms_, 0, sizeof(double) * 2 * cs, stream_));
        const size_t lc = std::max<size_t>(cl, 1) * kBatchClasses;
        for (int p = 0; p < 2; ++p) {  // the persistent form's counters, per pass
            dev_release(d_barrier_[p], stream_);
            dev_release(d_queue_[p], stream_);
            TB_CUDA(dev_malloc(&d_barrier_[p], sizeof(unsigned long long), stream_));
            TB_CUDA(dev_malloc(&d_queue_[p], sizeof(uint32_t) * lc, stream_));
        }
        if (!d_ctl_) {
            TB_CUDA(dev_malloc(&d_ctl_, sizeof(uint32_t) * 4, stream_));
            TB_CUDA(cudaMemsetAsync(d_ctl_, 0, sizeof(uint32_t) * 4, stream_));
        }
        for (auto &pl : plan_) {  // one work list per pass: the two passes run at once
            dev_release(pl.segs, stream_);
            dev_release(pl.level_nseg, stream_);
            dev_release(pl.level_nchunk, stream_);
            dev_release(pl.act, stream_);
            dev_release(pl.chunk_prefix, stream_);
            dev_release(pl.n_act, stream_);
            TB_CUDA(dev_malloc(&pl.segs, sizeof(BatchSeg) * cs * lc, stream_));
            TB_CUDA(dev_malloc(&pl.level_nseg, sizeof(uint32_t) * lc, stream_));
            TB_CUDA(dev_malloc(&pl.level_nchunk, sizeof(uint32_t) * lc, stream_));
            TB_CUDA(dev_malloc(&pl.act, sizeof(uint32_t) * cs, stream_));
            TB_CUDA(dev_malloc(&pl.chunk_prefix, sizeof(uint32_t) * (cs + 1), stream_));
            TB_CUDA(dev_malloc(&pl.n_act, sizeof(uint32_t), stream_));
            pl.norms = norms_;  // members of the two passes are disjoint
            pl.seg_stride = (uint32_t)cs;
        }
        cap_slots_ = cs;
        cap_levels_ = cl;
        invalidate();  // the graphs hold the old buffers
    }
    if (chunks > cap_chunks_) {
        const size_t cc = std::max(chunks, cap_chunks_ * 2);
        for (auto &pl : plan_) {
            dev_release(pl.partials, stream_);
            TB_CUDA(dev_malloc(&pl.partials, sizeof(double) * 2 * cc, stream_));
        }
        cap_chunks_ = cc;
        invalidate();
    }
    return kOk;
}

void Batch::assign_shifts()
{
    std::vector<double> work(max_levels_, 0.0);
    std::vector<size_t> order(members_.size());
    std::vector<double> total(members_.size(), 0.0);
    for (size_t i = 0; i < members_.size(); ++i) {
        order[i] = i;
        const auto &lo = members_[i].sw->schedule().level_offset;
        total[i] = (double)(lo.back() - lo.front()) * members_[i].sw->n_groups();
    }
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return total[a] > total[b]; });
    for (size_t i : order) {
        Member &m = members_[i];
        const auto &lo = m.sw->schedule().level_offset;
        const uint32_t n = m.v[0].n_levels;
        const double G = (double)m.sw->n_groups();
        uint32_t best_o = 0;
        double best = 1e300;
        for (uint32_t o = 0; o + n <= max_levels_; ++o) {
            double peak = 0.0;
            for (uint32_t l = 0; l < n && peak < best; ++l)
                peak = std::max(peak, work[o + l] + (double)(lo[l + 1] - lo[l]) * G);
            if (peak < best) {
                best = peak;
                best_o = o;
            }
        }
        m.shift = best_o;
        for (uint32_t l = 0; l < n; ++l) work[best_o + l] += (double)(lo[l + 1] - lo[l]) * G;
    }
}

void Batch::fill_slot(int prec, const Member &m, BatchSlot &s) const
{
    const Sweeper::DeviceView &v = m.v[prec];
    s = BatchSlot();
    s.rec = v.rec;
    s.psi = v.psi;
    s.iso = m.v[0].iso;
    s.iso32 = prec ? v.iso32 : nullptr;
    s.sigma_s = v.sigs;
    s.scat = v.scat;
    s.w = v.w;
    s.level_off = v.level_off;
    s.nc = m.sw->n_cells();
    s.A = (uint32_t)m.sw->n_angles();
    s.G = (uint32_t)m.sw->n_groups();
    s.vg = v.vg;
    s.vmagic = magic(s.G / s.vg);
    s.n_levels = v.n_levels;
    s.level_shift = m.shift;
    s.solver = (uint32_t)m.sw->solver();
    s.active = 0;
    if (prec == 0 && m.state == kRunSI) {
        s.active = 1;
        s.op = kOpSI;
        s.phi_in = m.cur;
        s.q_fixed = v.qiso;
        s.phi_out = m.nxt;
    } else if (prec == 1 && m.state == kRunFirst) {
        // FP32 source iteration on the whole problem: phi <- T32(phi)
        s.active = 1;
        s.op = kOpSI;
        s.phi_in = m.cur;
        s.q_fixed = m.v[0].qiso;
        s.phi_out = m.nxt;
    } else if (prec == 0 && m.state == kRunOuter) {
        s.active = 1;
        s.op = kOpOuter;
        s.phi = m.cur;
        s.phi_in = m.cur;
        s.q_fixed = v.qiso;
        s.phi_out = m.nxt;
        s.vec_r = m.r;
        s.vec_d = m.d;
        s.accept = m.accept ? 1u : 0u;
    } else if (prec == 1 && m.state == kRunInner) {
        s.active = 1;
        s.op = kOpInner;
        s.phi_in = m.d;
        s.q_fixed = nullptr;
        s.phi_out = m.k;
        s.vec_r = m.r;
        s.vec_d = m.d;
    }
}

int Batch::build_graph(int prec, std::string &err)
{
    if (!graph_[0] && !graph_[1]) assign_shifts();  // the member set changed
    const int ipw = ipw_[prec];
    const uint32_t n = (uint32_t)members_.size();
    // Blocks per level and class: enough for every member's chunks at once
    // (fewer when some are idle; the kernel's warps then exit at once).
    std::vector<BatchCuts> cuts(max_levels_);
    for (uint32_t L = 0; L < max_levels_; ++L) {
        uint64_t chunks[kBatchClasses] = {0, 0, 0};
        for (const auto &m : members_) {
            const auto &lo = m.sw->schedule().level_offset;
            if (L < m.shift || L - m.shift >= m.v[0].n_levels) continue;
            const uint64_t items = lo[L - m.shift + 1] - lo[L - m.shift];
            const uint32_t vg = m.v[prec].vg;
            chunks[vg == 4 ? 2 : vg == 2 ? 1 : 0] +=
                ipw ? items / ipw : items / 32 * ((uint64_t)m.sw->n_groups() / vg);
        }
        cuts[L].c[0] = 0;
        for (uint32_t c = 0; c < kBatchClasses; ++c)
            cuts[L].c[c + 1] = cuts[L].c[c] + (unsigned)std::min<uint64_t>((chunks[c] + 3) / 4, kLevelGridCap);
    }
    bool any_solver = false;
    for (const auto &m : members_) any_solver = any_solver || m.sw->solver() != kSolveNoPivot;
    cudaGraph_t g;
    cudaStream_t st = prec ? stream32_ : stream_;
    const BatchPlan &plan = plan_[prec];
    TB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const uint32_t rec_bytes =
        (uint32_t)(ipw ? record_bytes(prec == 1) : compact_record_bytes(prec == 1));
    cudaError_t e = launch_batch_plan(ipw, d_slots_[prec], n, max_levels_, rec_bytes, plan, st);
    if (e == cudaSuccess && prec == 0) e = launch_batch_accept(d_slots_[prec], plan, kStreamGrid, st);
    if (e == cudaSuccess) e = launch_batch_scatter(d_slots_[prec], plan, kStreamGrid, st);
    if (persist_) {
        const size_t lc = (size_t)std::max<uint32_t>(max_levels_, 1) * kBatchClasses;
        if (e == cudaSuccess) e = cudaMemsetAsync(d_barrier_[prec], 0, sizeof(unsigned long long), st);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_queue_[prec], 0, sizeof(uint32_t) * lc, st);
        BatchPersistArgs a = {};
        a.barrier = d_barrier_[prec];
        a.queue = d_queue_[prec];
        a.max_levels = max_levels_;
        a.df.err = d_ctl_;
        a.df.abort = d_ctl_ + 3;
        a.df.spin_limit = spin_limit_;
        if (e == cudaSuccess)
            e = prec ? launch_batch_persist<float>(d_slots_[prec], plan, a, any_solver, st)
                     : launch_batch_persist<double>(d_slots_[prec], plan, a, any_solver, st);
    } else {
        for (uint32_t L = 0; L < max_levels_ && e == cudaSuccess; ++L)
            e = prec ? launch_batch_level<float>(ipw, d_slots_[prec], plan, L, cuts[L], any_solver, st)
                     : launch_batch_level<double>(ipw, d_slots_[prec], plan, L, cuts[L], any_solver, st);
    }
    if (e == cudaSuccess) e = launch_batch_psi_to_phi(prec == 1, d_slots_[prec], plan, kStreamGrid, st);
    if (e == cudaSuccess) e = launch_batch_post(d_slots_[prec], plan, kStreamGrid, st);
    if (e == cudaSuccess) e = launch_batch_finish(d_slots_[prec], plan, 64, st);
    cudaError_t ce = cudaStreamEndCapture(st, &g);
    TB_CUDA(e);
    TB_CUDA(ce);
    cudaError_t ie = cudaGraphInstantiate(&graph_[prec], g, 0);
    cudaGraphDestroy(g);
    TB_CUDA(ie);
    return kOk;
}

int Batch::set_persistent(bool on, std::string &err)
{
    if (on && (ipw_[0] != 0 || ipw_[1] != 0)) {
        err = "the persistent batched form runs the direct kernels (items per warp 0)";
        return kErrArg;
    }
    if (persist_ != on) {
        persist_ = on;
        invalidate();
    }
    return kOk;
}

// The persistent form's error words: a grid barrier that gave up.
int Batch::check_ctl(std::string &err)
{
    if (!persist_ || !d_ctl_) return kOk;
    uint32_t ctl[4] = {0, 0, 0, 0};
    TB_CUDA(cudaMemcpyAsync(ctl, d_ctl_, sizeof ctl, cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    if (ctl[0] == 0) return kOk;
    TB_CUDA(cudaMemsetAsync(d_ctl_, 0, sizeof ctl, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    err = "batched persistent pass: grid barrier timed out at level " + std::to_string(ctl[1]);
    return kErrTimeout;
}

int Batch::pass(int prec, std::string &err)
{
    const size_t n = members_.size();
    bool any = false;
    for (const auto &m : members_)
        any = any || (prec == 0 ? m.state == kRunSI || m.state == kRunOuter
                                : m.state == kRunInner || m.state == kRunFirst);
    if (!any) return kOk;
    // the graph (and with it the members' level shifts) before the slot table
    if (!graph_[prec]) TB_CHECK(build_graph(prec, err));
    for (size_t j = 0; j < n; ++j) fill_slot(prec, members_[j], h_slots_[prec][j]);
    cudaStream_t st = prec ? stream32_ : stream_;
    TB_CUDA(cudaMemcpyAsync(d_slots_[prec], h_slots_[prec], sizeof(BatchSlot) * n, cudaMemcpyHostToDevice, st));
    TB_CUDA(cudaEventRecord(ev_[2 * prec], st));
    TB_CUDA(cudaGraphLaunch(graph_[prec], st));
    TB_CUDA(cudaEventRecord(ev_[2 * prec + 1], st));
    passes_[prec]++;
    for (size_t j = 0; j < n; ++j)
        if (h_slots_[prec][j].active) updates_[prec] += (double)members_[j].updates;
    return kOk;
}

int Batch::step(int &n_running, std::string &err)
{
    TB_CHECK(step_launch(err));
    return step_finish(n_running, err);
}

int Batch::step_launch(std::string &err)
{
    launched_ = false;
    int running = 0;
    for (const auto &m : members_) running += m.state != kDone;
    if (running == 0) return kOk;
    TB_CUDA(cudaSetDevice(device_));
    TB_CHECK(ensure_capacity(err));
    before_[0] = passes_[0];
    before_[1] = passes_[1];
    // the FP32 pass waits for the previous step's end on the main stream;
    // both passes then run concurrently (their members are disjoint) and
    // the main stream joins the FP32 one before reading the norms
    TB_CUDA(cudaEventRecord(join_, stream_));
    TB_CUDA(cudaStreamWaitEvent(stream32_, join_, 0));
    TB_CHECK(pass(0, err));
    TB_CHECK(pass(1, err));
    TB_CUDA(cudaEventRecord(join_, stream32_));
    TB_CUDA(cudaStreamWaitEvent(stream_, join_, 0));
    TB_CUDA(cudaMemcpyAsync(h_norms_, norms_, sizeof(double) * 2 * members_.size(), cudaMemcpyDeviceToHost,
                            stream_));
    launched_ = true;
    return kOk;
}

int Batch::step_finish(int &n_running, std::string &err)
{
    n_running = 0;
    if (!launched_) return kOk;
    launched_ = false;
    TB_CUDA(cudaSetDevice(device_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    TB_CHECK(check_ctl(err));  // before any member advances on this step's norms
    const size_t n = members_.size();
    const int *before = before_;
    for (int p = 0; p < 2; ++p)
        if (passes_[p] > before[p]) {
            float ms = 0;
            cudaEventElapsedTime(&ms, ev_[2 * p], ev_[2 * p + 1]);
            ms_[p] += ms;
        }
    n_running = 0;
    for (size_t j = 0; j < n; ++j) {
        Member &m = members_[j];
        if (m.state == kDone) continue;
        const double d = h_norms_[2 * j], mm = h_norms_[2 * j + 1];
        const double e = mm > 0 ? d / mm : 0.0;
        m.st.steps++;
        if (m.state == kRunSI) {
            std::swap(m.cur, m.nxt);
            m.st.sweeps_fp64++;
            m.st.iterations++;
            m.st.final_error = e;
            if (e <= m.o.err_max || m.st.iterations >= m.o.iter_max) {
                m.state = kDone;
                m.sw->note_psi_precision(0);
            }
        } else if (m.state == kRunFirst) {
            // FP32 source iteration from phi = 0 to min(inner_tol, 1e-6)
            std::swap(m.cur, m.nxt);
            m.st.sweeps_fp32++;
            m.st.iterations++;
            if (e <= std::min(m.o.inner_tol, 1e-6) || m.st.iterations >= m.o.iter_max) m.state = kRunOuter;
        } else if (m.state == kRunOuter) {
            // r = T64(phi) - phi (after phi += d when accept was set)
            m.accept = false;
            m.st.sweeps_fp64++;
            m.st.final_error = e;
            m.phi_l1 = mm;
            if (e <= m.o.err_max || m.st.refinements >= m.o.refine_max || m.st.iterations >= m.o.iter_max) {
                m.state = kDone;
                m.res = m.nxt;  // T64(phi), and psi is its FP64 sweep
                m.sw->note_psi_precision(0);
            } else {
                m.state = kRunInner;
                m.inner_its = 0;
            }
        } else {
            // d <- r + K32 d; accepting phi + d leaves the residual
            // K64 (d - d_prev) + (K64 - K32) d_prev: at most the last change
            // plus the FP32 operator's error on d.  When both are below the
            // tolerance the solve ends without another FP64 sweep.
            m.st.sweeps_fp32++;
            m.st.iterations++;
            m.inner_its++;
            const double tol_abs = m.o.err_max * m.phi_l1;
            const bool small = kFp32OpErr * mm <= 0.1 * tol_abs;
            if (small && d <= 0.5 * tol_abs) {
                m.state = kDone;
                m.st.refinements++;
                m.st.final_error = m.phi_l1 > 0 ? (d + kFp32OpErr * mm) / m.phi_l1 : 0.0;
                m.accept_at_result = true;
                m.res = m.cur;
                m.sw->note_psi_precision(-1);  // psi holds the last correction's FP32 sweep
            } else if (e <= m.o.inner_tol || m.inner_its >= m.o.inner_max || m.st.iterations >= m.o.iter_max) {
                m.state = kRunOuter;
                m.accept = true;
                m.st.refinements++;
            }
        }
        if (m.state == kDone) {
            m.st.done = 1;
        } else {
            ++n_running;
        }
    }
    return kOk;
}

int Batch::running() const
{
    int n = 0;
    for (const auto &m : members_) n += m.state != kDone;
    return n;
}

int Batch::run(std::string &err)
{
    int running = 1;
    while (running > 0) TB_CHECK(step(running, err));
    return kOk;
}

int Batch::result(int id, double *phi_host, BatchMemberStats &st, std::string &err)
{
    for (auto &m : members_)
        if (m.id == id) {
            st = m.st;
            if (phi_host) {
                const double *src = m.o.method == 0 ? m.cur : m.res;
                TB_CUDA(cudaSetDevice(device_));
                if (!src) { err = "the member's solve has not finished"; return kErrArg; }
                if (m.accept_at_result) {
                    TB_CUDA(axpby(1.0, m.d, 1.0, m.cur, m.sw->phi_size(), stream_));
                    m.accept_at_result = false;
                }
                TB_CUDA(cudaMemcpyAsync(phi_host, src, sizeof(double) * m.sw->phi_size(), cudaMemcpyDeviceToHost,
                                        stream_));
                TB_CUDA(cudaStreamSynchronize(stream_));
            }
            return kOk;
        }
    err = "no batch member with that id";
    return kErrArg;
}

void Batch::timing(double ms[2], int passes[2]) const
{
    ms[0] = ms_[0];
    ms[1] = ms_[1];
    passes[0] = passes_[0];
    passes[1] = passes_[1];
}

}  // namespace tycho
