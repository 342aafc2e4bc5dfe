// Solve service: admission by footprint, host-side builds, continuous batching.
#include "server.hpp"

#include <algorithm>
#include <chrono>
#include <exception>
#include <new>
#include <thread>

#include "devmem.hpp"
#include "status.hpp"

namespace tycho {

constexpr int kSoloRestart = 20;  // GMRES restart of the large requests' mixed solve

uint64_t footprint_bytes(uint64_t n_cells, int sn_order, int n_groups, bool fp32, bool compact)
{
    const uint64_t A = 2ull * sn_order * sn_order;
    // level padding adds at most 31 items per level; levels stay below 16 n
    // for Kuhn cubes, far below 5% of the items
    const uint64_t items = n_cells * A + n_cells * A / 20 + 4096;
    const uint64_t G = (uint64_t)n_groups, phi = n_cells * 4 * G * 8;
    uint64_t b = items * 4 * G * 8;                 // psi (FP64-sized; the FP32 sweep shares it)
    b += items * (32 + (fp32 ? 16 : 0));            // per-item face terms
    b += items * (4 + 4);                           // item list, completion epochs
    b += items * (compact ? 112 + (fp32 ? 64 : 0) : 256 + (fp32 ? 128 : 0));  // records
    b += n_cells * (16 + 4 + 24 + 12 + 8 + 8 + 8);  // adjacency, maps, cell terms, sigma, levels
    b += phi * (7 + (fp32 ? 4 : 0));                // phi, iso, r, tmp, (FP32 iso, batch r/d/k)
    return b + (b >> 5) + (8ull << 20);             // allocator rounding
}

Server::~Server()
{
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_work_.notify_all();
    cv_solo_.notify_all();
    if (solo_thread_.joinable()) solo_thread_.join();
    for (auto &t : workers_) t.join();
}

// Large requests, one at a time, each with the single-instance solver on its
// sweeper's own streams (concurrently with the batch of small requests).
// A request's result does not depend on what else is being served.
void Server::solo()
{
    for (;;) {
        Request *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_solo_.wait(lk, [&] { return stop_ || !solo_q_.empty(); });
            if (solo_q_.empty()) return;
            r = solo_q_.front();
            solo_q_.pop_front();
        }
        SolveOptions so;
        so.method = o_.solve.method == 2 ? 2 : 0;
        so.iter_max = o_.solve.iter_max;
        so.err_max = o_.solve.err_max;
        so.restart = kSoloRestart;
        so.inner_tol = o_.solve.inner_tol;
        so.refine_max = o_.solve.refine_max;
        SolveStats st;
        std::string err;
        int s = kOk;
        try {
            s = r->sw->solve(so, r->phi_out, nullptr, st, err);
        } catch (const std::bad_alloc &) {
            s = kErrOom;
            err = "host memory exhausted while solving the request";
        } catch (const std::exception &e) {
            s = kErrArg;
            err = std::string("solving the request: ") + e.what();
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            r->status = s;
            r->error = err;
            r->stats.iterations = st.iterations;
            r->stats.sweeps_fp64 = st.sweeps_fp64;
            r->stats.sweeps_fp32 = st.sweeps_fp32;
            r->stats.refinements = st.refinements;
            r->stats.final_error = st.final_error;
            r->stats.done = s == kOk;
            r->stats.steps = 0;
            solo_done_.push_back(r);
        }
        cv_built_.notify_all();
    }
}

int Server::init(const ServerOptions &o, std::string &err)
{
    if (o.budget_bytes <= 0 || o.setup_threads < 1 || o.setup_threads > 64) {
        err = "bad server options (budget > 0, 1..64 setup threads)";
        return kErrArg;
    }
    if (o.solve.method != 0 && o.solve.method != 2) { err = "server method must be 0 or 2"; return kErrArg; }
    o_ = o;
    for (auto &b : lanes_) {
        const int s = b.init(o.device, o.ipw32, o.ipw64, err);
        if (s != kOk) return s;
    }
    reserve_pool();
    return kOk;
}

// Maps the budget (at most 90% of the free device memory) into the device
// pool once, so that no request's build waits for fresh device memory to be
// mapped (a 48^3 S8 G=8 request holds ~40 GB: mapping it took ~0.4 s).  A
// failed reservation only costs that time later.
void Server::reserve_pool()
{
    size_t free_b = 0, total_b = 0;
    if (cudaSetDevice(o_.device) != cudaSuccess || cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    const size_t want = (size_t)std::min(o_.budget_bytes, 0.9 * (double)free_b);
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    void *p = nullptr;
    if (dev_malloc(&p, want, s) == cudaSuccess) dev_free(p, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    cudaGetLastError();
}

double Server::now() const
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count() - t0_;
}

int Server::submit(std::shared_ptr<const MeshTables> tp, int sn, int G, const double *sigma_t, const double *sigma_s,
                   const double *scatter, const double *q_iso, double arrival, double *phi_out, int &id,
                   std::string &err)
{
    if (!tp || !sigma_t || !sigma_s || !phi_out || G < 1 || G > 64 || arrival < 0) {
        err = "bad request (cross sections, phi buffer, 1..64 groups, arrival >= 0)";
        return kErrArg;
    }
    auto r = std::make_unique<Request>();
    r->id = (int)reqs_.size() + 1;
    const MeshTables &t = *tp;
    r->tables = tp;
    r->sn = sn;
    r->G = G;
    const size_t nc = t.n_cells;
    r->sigma_t.assign(sigma_t, sigma_t + nc);
    r->sigma_s.assign(sigma_s, sigma_s + nc);
    if (scatter) r->scatter.assign(scatter, scatter + (size_t)G * G);
    if (q_iso) r->q.assign(q_iso, q_iso + nc * 4 * (size_t)G);
    r->arrival = arrival;
    r->phi_out = phi_out;
    r->footprint = footprint_bytes(nc, sn, G, o_.solve.method == 2, o_.ipw32 == 0 && o_.ipw64 == 0);
    r->lane = (double)nc * 2.0 * sn * sn >= o_.large_items ? 1 : 0;
    if (r->lane == 1 && o_.large_solo && o_.solve.method == 2)  // the GMRES basis and Hessenberg
        r->footprint += (uint64_t)(kSoloRestart + 1) * nc * 4 * G * 8 + 4096;
    id = r->id;
    reqs_.push_back(std::move(r));
    return kOk;
}

const Server::Request *Server::request(int id) const
{
    if (id < 1 || id > (int)reqs_.size()) return nullptr;
    return reqs_[id - 1].get();
}

void Server::stats(double &peak_bytes, int &peak_active, int &steps, double &makespan) const
{
    peak_bytes = peak_bytes_;
    peak_active = peak_active_;
    steps = steps_;
    makespan = makespan_;
}

// Builds a request's sweeper: schedule, uploads, cross sections, source and
// the records of every precision the solve sweeps in.
void Server::worker()
{
    for (;;) {
        Request *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_work_.wait(lk, [&] { return stop_ || !build_q_.empty() || !retire_q_.empty(); });
            if (!retire_q_.empty()) {
                auto job = std::move(retire_q_.front());
                retire_q_.pop_front();
                lk.unlock();
                job.first.reset();
                lk.lock();
                freed_bytes_ += job.second;
                continue;
            }
            if (stop_ && build_q_.empty()) return;
            r = build_q_.front();
            build_q_.pop_front();
        }
        std::string err;
        auto sw = std::make_unique<Sweeper>();
        SweeperOptions so;
        so.sn_order = r->sn;
        so.n_groups = r->G;
        so.device = o_.device;
        so.fp32 = o_.solve.method == 2;
        int s = kOk;
        try {  // a failed build fails its request, never the service
            s = sw->init(r->tables, so, err);
            if (s == kOk)
                s = sw->set_cross_sections(r->sigma_t.data(), r->sigma_s.data(),
                                           r->scatter.empty() ? nullptr : r->scatter.data(), err);
            if (s == kOk && !r->q.empty()) s = sw->set_source(1, r->q.data(), err);
            Sweeper::DeviceView v;
            if (s == kOk) s = sw->device_view(0, v, err, o_.ipw64 == 0);
            if (s == kOk && so.fp32) s = sw->device_view(1, v, err, o_.ipw32 == 0);
        } catch (const std::bad_alloc &) {
            s = kErrOom;
            err = "host memory exhausted while building the request";
        } catch (const std::exception &e) {
            s = kErrArg;
            err = std::string("building the request: ") + e.what();
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            r->status = s;
            r->error = err;
            if (s == kOk) r->sw = std::move(sw);
            r->t_built = now();
            built_.push_back(r);
        }
        cv_built_.notify_all();
    }
}

int Server::run(std::string &err)
{
    using namespace std::chrono;
    t0_ = 0;
    t0_ = now();
    if (workers_.empty())
        for (int i = 0; i < o_.setup_threads; ++i) workers_.emplace_back([this] { worker(); });
    if (o_.large_solo && !solo_thread_.joinable()) solo_thread_ = std::thread([this] { solo(); });
    std::vector<Request *> order;
    for (auto &r : reqs_)
        if (r->state == 0) order.push_back(r.get());
    std::stable_sort(order.begin(), order.end(), [](Request *a, Request *b) { return a->arrival < b->arrival; });
    size_t next = 0;  // next request to admit, in arrival order
    double reserved = 0;
    int pending = (int)order.size(), building = 0;
    int in_lane[kLanes] = {0, 0};
    int in_solo = 0;  // large requests with the solo thread
    bool inflight[kLanes] = {false, false};
    std::vector<Request *> waiting[kLanes];  // built, joining at the lane's next step boundary
    while (pending > 0) {
        // admission in arrival order: first come, first served, no overtaking
        const double t = now();
        while (next < order.size() && order[next]->arrival <= t) {
            Request *r = order[next];
            if ((double)r->footprint > o_.budget_bytes) {
                r->state = 5;
                r->status = kErrOom;
                r->error = "request footprint exceeds the server budget";
                r->t_done = t;
                --pending;
                ++next;
                continue;
            }
            if (reserved + (double)r->footprint > o_.budget_bytes) break;
            reserved += (double)r->footprint;
            peak_bytes_ = std::max(peak_bytes_, reserved);
            r->state = 1;
            r->t_admit = t;
            ++building;
            {
                std::lock_guard<std::mutex> lk(mu_);
                build_q_.push_back(r);
            }
            cv_work_.notify_one();
            ++next;
        }
        // built requests wait for their lane's next step boundary
        std::vector<Request *> ready;
        {
            std::unique_lock<std::mutex> lk(mu_);
            reserved -= freed_bytes_;  // retired sweepers the workers have destroyed
            freed_bytes_ = 0;
            const bool idle = !inflight[0] && !inflight[1] && in_lane[0] + in_lane[1] == 0 &&
                              waiting[0].empty() && waiting[1].empty();
            if (idle && built_.empty() && solo_done_.empty()) {
                // no batch step to drive: wait for a build, a solo solve or
                // the next arrival
                const double wait = next < order.size() && order[next]->arrival > t ? order[next]->arrival - t : 0.05;
                cv_built_.wait_for(lk, duration<double>(std::min(std::max(wait, 1e-4), 0.05)),
                                   [&] { return !built_.empty() || !solo_done_.empty(); });
            }
            ready.swap(built_);
            for (Request *r : solo_done_) {
                r->state = r->status == kOk ? 4 : 5;
                r->t_done = now();
                retire_q_.emplace_back(std::move(r->sw), (double)r->footprint);
                --in_solo;
                --pending;
            }
            if (!solo_done_.empty()) cv_work_.notify_one();
            solo_done_.clear();
        }
        for (Request *r : ready) {
            --building;
            if (r->status != kOk) {
                r->state = 5;
                r->t_done = now();
                reserved -= (double)r->footprint;
                --pending;
                continue;
            }
            r->state = 2;
            if (r->lane == 1 && o_.large_solo) {
                r->state = 3;
                ++in_solo;
                {
                    std::lock_guard<std::mutex> lk(mu_);
                    solo_q_.push_back(r);
                }
                cv_solo_.notify_one();
                peak_active_ = std::max(peak_active_, in_lane[0] + in_lane[1] + in_solo);
                continue;
            }
            waiting[r->lane].push_back(r);
        }
        // each lane steps on its own stream: finish a step when its stream is
        // done, retire finished members, admit waiting ones, launch the next
        bool progressed = false;
        for (int L = 0; L < kLanes; ++L) {
            Batch &b = lanes_[L];
            if (inflight[L]) {
                if (!b.step_done()) continue;
                int running = 0;
                int s = b.step_finish(running, err);
                if (s != kOk) return s;
                inflight[L] = false;
                progressed = true;
                for (auto &rp : reqs_) {
                    Request *r = rp.get();
                    if (r->state != 3 || r->lane != L) continue;
                    BatchMemberStats st;
                    s = b.result(r->member, nullptr, st, err);
                    if (s != kOk) return s;
                    if (!st.done) continue;
                    s = b.result(r->member, r->phi_out, st, err);
                    if (s != kOk) return s;
                    r->stats = st;
                    s = b.remove(r->member, err);
                    if (s != kOk) return s;
                    {
                        std::lock_guard<std::mutex> lk(mu_);
                        retire_q_.emplace_back(std::move(r->sw), (double)r->footprint);
                    }
                    cv_work_.notify_one();
                    r->state = 4;
                    r->t_done = now();
                    --in_lane[L];
                    --pending;
                }
            }
            for (Request *r : waiting[L]) {
                int s = b.add(r->sw.get(), o_.solve, r->member, err);
                if (s != kOk) return s;
                r->state = 3;
                ++in_lane[L];
            }
            waiting[L].clear();
            peak_active_ = std::max(peak_active_, in_lane[0] + in_lane[1] + in_solo);
            if (in_lane[L] > 0 && b.running() > 0) {
                int s = b.step_launch(err);
                if (s != kOk) return s;
                inflight[L] = true;
                ++steps_;
                progressed = true;
            }
        }
        if (!progressed && (inflight[0] || inflight[1])) std::this_thread::sleep_for(microseconds(20));
    }
    makespan_ = now();
    return kOk;
}

}  // namespace tycho
