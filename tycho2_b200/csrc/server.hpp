// Solve service on one GPU: requests arrive over time, are admitted by their
// device-memory footprint against a budget, built into device-resident
// sweepers by host worker threads, and solved by continuous batching -- a
// request that arrives while others are on the GPU joins the batch at the
// next step, and a finished one leaves it and frees its memory.  No
// counterpart in the reference (one solve per process run).
#pragma once

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "batch.hpp"
#include "mesh.hpp"
#include "sweeper.hpp"

namespace tycho {

struct ServerOptions {
    int device = 0;
    double budget_bytes = 150e9;  // device memory the resident requests may hold
    int setup_threads = 2;        // host threads building sweepers
    int ipw32 = 0, ipw64 = 0;     // batch level kernels: items per warp (0 = direct, compact records)
    BatchOptions solve;           // method 0 FP64 source iteration, 2 mixed
    double large_items = 32e6;    // cells x angles from which a request runs in the large lane
    // Large requests: solved one at a time by the single-instance solver on
    // their sweeper's own streams (true: FP64 source iteration, or for the
    // mixed service FP32-sweep GMRES(20) in FP64 refinement), or as members
    // of a second batch (false).
    bool large_solo = true;
};

// Device bytes one resident request holds (sweeper + batch vectors), an
// upper estimate made before anything is allocated; compact: the batch runs
// the direct kernels on compact records.
uint64_t footprint_bytes(uint64_t n_cells, int sn_order, int n_groups, bool fp32, bool compact);

class Server {
public:
    struct Request {
        int id = 0;
        std::shared_ptr<const MeshTables> tables;
        int sn = 4, G = 1;
        std::vector<double> sigma_t, sigma_s, scatter, q;
        double arrival = 0;     // seconds after run() starts
        double *phi_out = nullptr;
        uint64_t footprint = 0;
        // progress (times in seconds after run() starts)
        int state = 0;          // 0 queued, 1 building, 2 built, 3 in batch, 4 done, 5 failed
        double t_admit = -1, t_built = -1, t_done = -1;
        int member = -1, status = 0;
        int lane = 0;           // 0 small, 1 large (its own batch and stream)
        std::string error;
        BatchMemberStats stats;
        std::unique_ptr<Sweeper> sw;
    };

    ~Server();
    int init(const ServerOptions &o, std::string &err);
    int submit(std::shared_ptr<const MeshTables> t, int sn, int G, const double *sigma_t, const double *sigma_s,
               const double *scatter, const double *q_iso, double arrival, double *phi_out, int &id,
               std::string &err);
    // Serves every submitted request (arrivals relative to the call).
    int run(std::string &err);
    const Request *request(int id) const;
    // peak device bytes reserved, peak requests in the batch, batch steps
    void stats(double &peak_bytes, int &peak_active, int &steps, double &makespan) const;

private:
    void worker();
    void solo();  // the large requests' single-instance solves, in order
    double now() const;

    ServerOptions o_;
    std::vector<std::unique_ptr<Request>> reqs_;
    // Two lanes, each a batch on its own stream: requests of at least
    // large_items cells x angles sweep in lane 1, so a deep mesh does not set
    // the step time of the small ones; both lanes run on the GPU at once.
    void reserve_pool();
    static constexpr int kLanes = 2;
    Batch lanes_[kLanes];
    // build queue shared with the workers
    std::mutex mu_;
    std::condition_variable cv_work_, cv_built_;
    std::deque<Request *> build_q_;
    std::vector<Request *> built_;
    // finished requests' sweepers, destroyed by the workers (not on the loop
    // thread); their footprints go back to the budget once destroyed
    std::deque<std::pair<std::unique_ptr<Sweeper>, double>> retire_q_;
    double freed_bytes_ = 0;
    // large requests for the solo thread, and those it has finished
    std::condition_variable cv_solo_;
    std::deque<Request *> solo_q_;
    std::vector<Request *> solo_done_;
    std::thread solo_thread_;
    bool stop_ = false;
    std::vector<std::thread> workers_;
    double t0_ = 0;
    double peak_bytes_ = 0, makespan_ = 0;
    int peak_active_ = 0, steps_ = 0;
};

}  // namespace tycho
