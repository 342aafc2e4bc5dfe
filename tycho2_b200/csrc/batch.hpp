// Batched solves of many independent sweep instances on one GPU (no
// counterpart in the reference, which solves one problem per process).
//
// Members are device-resident Sweepers (mesh tables, wavefront schedule,
// per-item records, psi).  Each step runs at most two passes, each one CUDA
// graph over every member that needs it:
//   FP64 pass  members in source iteration (reference fixed point) or at an
//              outer refinement step (FP64 residual sweep)
//   FP32 pass  members inside their inner FP32 solve of the correction
// then reads every member's two norms in one copy and advances each member's
// solver on the host.  A member's arithmetic never depends on the others, so
// its result is bit-identical alone and in any mix.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "batch_types.hpp"
#include "sweeper.hpp"

namespace tycho {

struct BatchOptions {
    int method = 2;           // 0 FP64 source iteration, 2 mixed (FP32 inner SI, FP64 refinement)
    int iter_max = 1000;      // sweeps of the solve (inner FP32 sweeps count for mixed)
    double err_max = 1e-10;   // L1 relative change of phi (SourceIteration.cc:167-175)
    double inner_tol = 1e-5;  // inner FP32 iteration: L1 relative change of the correction
    int inner_max = 200;
    int refine_max = 30;
};

struct BatchMemberStats {
    int iterations = 0, sweeps_fp64 = 0, sweeps_fp32 = 0, refinements = 0;
    double final_error = 1.0;
    int done = 0;
    int steps = 0;  // batch steps the member took part in
};

class Batch {
public:
    ~Batch();
    int init(int device, int ipw32, int ipw64, std::string &err);
    // Adds a sweeper (cross sections and fixed source set, same device);
    // the solve starts from phi = 0 at the next step.
    int add(Sweeper *sw, const BatchOptions &o, int &id, std::string &err);
    int remove(int id, std::string &err);
    // One step of every running member; n_running receives how many still run.
    int step(int &n_running, std::string &err);
    // The same in two halves: enqueue the step's passes on the batch's own
    // stream, then wait for them and advance the members (so that several
    // batches can run on the GPU at once).
    int step_launch(std::string &err);
    int step_finish(int &n_running, std::string &err);
    int running() const;
    // The launched step has finished on the GPU, failed (step_finish reports
    // it), or nothing is in flight.
    bool step_done() const { return !launched_ || cudaStreamQuery(stream_) != cudaErrorNotReady; }
    int run(std::string &err);
    int result(int id, double *phi_host, BatchMemberStats &st, std::string &err);
    // Device time of the passes so far: [0] FP64, [1] FP32 (ms), and counts.
    void timing(double ms[2], int passes[2]) const;
    // Updates (cell x angle x group) swept so far, per precision.
    void updates(double out[2]) const { out[0] = updates_[0]; out[1] = updates_[1]; }
    int size() const { return (int)members_.size(); }
    // Wavefront of each pass: false (default) one launch per global level;
    // true one persistent cooperative launch with a device work queue and a
    // bounded grid barrier between levels (direct kernels only).
    int set_persistent(bool on, std::string &err);
    // Polls of the persistent form's grid barrier before it gives up
    // (the step then fails with a timeout and the batch stays usable).
    void set_wait_limit(uint32_t polls) { spin_limit_ = polls; }

private:
    enum State { kRunSI = 0, kRunOuter = 1, kRunInner = 2, kDone = 3, kRunFirst = 4 };
    struct Member {
        int id = 0;
        Sweeper *sw = nullptr;
        BatchOptions o;
        State state = kRunSI;
        BatchMemberStats st;
        Sweeper::DeviceView v[2];
        double *r = nullptr, *d = nullptr, *k = nullptr;  // residual, correction, K delta
        double *cur = nullptr, *nxt = nullptr;            // SI: phi and the next iterate
        bool accept = false;
        bool accept_at_result = false;  // mixed, finished after an inner solve: phi += d on read
        double phi_l1 = 0.0;            // mixed: ||T64(phi)||_1 of the last FP64 pass
        const double *res = nullptr;    // mixed: where the result lives once done
        int inner_its = 0;
        uint64_t updates = 0;                             // per sweep
        uint32_t shift = 0;                               // global level of the member's level 0
    };
    // Staggers the members' level ranges over the global levels so that the
    // work per global level is even (small members fill the levels where
    // only the deepest ones have work).
    void assign_shifts();
    int pass(int prec, std::string &err);
    int build_graph(int prec, std::string &err);
    void fill_slot(int prec, const Member &m, BatchSlot &s) const;
    int ensure_capacity(std::string &err);
    void invalidate();

    int device_ = 0, ipw_[2] = {16, 16};
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
    std::vector<Member> members_;
    int next_id_ = 1;
    // device tables: [prec] slot tables, shared plan buffers
    BatchSlot *d_slots_[2] = {nullptr, nullptr};
    BatchSlot *h_slots_[2] = {nullptr, nullptr};  // pinned staging
    double *h_norms_ = nullptr;                    // pinned
    BatchPlan plan_[2] = {};        // [0] FP64 pass, [1] FP32 pass
    double *norms_ = nullptr;        // per member: the two norms of its last pass
    cudaStream_t stream32_ = nullptr;  // the FP32 pass runs here, beside the FP64 one
    cudaEvent_t join_ = nullptr;
    size_t cap_slots_ = 0, cap_levels_ = 0, cap_chunks_ = 0;
    cudaGraphExec_t graph_[2] = {nullptr, nullptr};
    uint32_t max_levels_ = 0;
    double ms_[2] = {0, 0};
    int passes_[2] = {0, 0};
    double updates_[2] = {0, 0};
    bool launched_ = false;
    int before_[2] = {0, 0};
    // persistent form: per pass a barrier counter and a work-queue counter
    // per (level, class); control words [0..2] error, [3] abort
    bool persist_ = false;
    uint32_t spin_limit_ = 1u << 22;
    unsigned long long *d_barrier_[2] = {nullptr, nullptr};
    uint32_t *d_queue_[2] = {nullptr, nullptr};
    uint32_t *d_ctl_ = nullptr;
    int check_ctl(std::string &err);
};

}  // namespace tycho
