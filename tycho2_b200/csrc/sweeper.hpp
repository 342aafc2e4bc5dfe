// Device-resident sweep instance: mesh tables, wavefront schedule, psi and
// the outer solvers (source iteration, GMRES, mixed-precision refinement).
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "device_ops.hpp"
#include "mesh.hpp"
#include "schedule.hpp"

namespace tycho {

struct SweeperOptions {
    int sn_order = 4;
    int n_groups = 1;
    int device = 0;
    bool fp32 = false;
    int tpi64 = 0;  // 0 = auto
    int tpi32 = 0;
    int schedule = 0;  // 0 auto (levels, compact records), 1 level-synchronous, 2 dataflow
    int gauss_elim = 1;  // 4x4 solver, numbered as tycho_gauss_elim (deck key GaussElim)
    int levelling = 0;   // 0 auto, 1 host, 2 device
    // directions [angle_begin, angle_end) of the quadrature only (both 0:
    // all): an angle shard whose phi is the partial sum over its directions
    int angle_begin = 0, angle_end = 0;
};

// Launch shape of one precision's sweep.
struct LaunchShape {
    int schedule = 2;   // 1 one launch per wavefront level, 2 persistent dataflow,
                        // 3 persistent levels (record variant only)
    int variant = 1;    // 0 item-parallel (knob = threads per item),
                        // 1 warp tiles (knob = warps per block),
                        // 2 precomputed per-item records (knob = items per warp),
                        // 3 records in registers, 4 compact records in registers
                        //   (knob = threads per block; level schedule)
    int knob = 4;
    int vg = 1;                 // records: groups per vector access of a psi row
    int streams = 1;            // level schedule: octant groups swept on this many streams
    unsigned grid = 0;          // dataflow kernel of this variant: co-resident blocks
    unsigned persist_grid = 0;  // persistent-levels kernel: co-resident blocks
    unsigned direct_grid = 0;   // direct variants on the dataflow schedule: co-resident blocks
};

struct SolveOptions {
    int method = 0;  // 0 SI, 1 GMRES, 2 mixed
    int iter_max = 100;
    double err_max = 1e-10;
    int restart = 20;
    double inner_tol = 1e-5;
    int refine_max = 10;
};

struct SolveStats {
    int iterations = 0, sweeps_fp64 = 0, sweeps_fp32 = 0, refinements = 0;
    double final_error = 0.0, seconds = 0.0;
};

class Sweeper {
public:
    ~Sweeper();
    // The sweeper keeps a reference to the tables (no copy).
    int init(std::shared_ptr<const MeshTables> t, const SweeperOptions &o, std::string &err);

    int set_cross_sections(const double *sigma_t, const double *sigma_s, const double *scatter,
                           std::string &err);
    int set_source(int kind, const double *q, std::string &err);
    int sweep_host(const double *source, double *psi, std::string &err);
    int solve(const SolveOptions &o, double *phi_out, double *psi_out, SolveStats &st,
              std::string &err);
    int write_psi(const std::string &path, std::string &err);
    // The resident FP64 psi (the last FP64 sweep's) into host memory, PsiData layout.
    int read_psi(double *psi, std::string &err);
    int time_sweeps(int precision, int n, bool flush_l2, double *ms, std::string &err);
    // vg: record variant's groups per vector access (0 = widest dividing G).
    int configure(int prec, int schedule, int variant, int knob, std::string &err, int vg = 0, int streams = 1);
    int autotune(int prec, int reps, LaunchShape *best, double *best_ms, std::string &err);
    const LaunchShape &shape(int prec) const { return shape_[prec ? 1 : 0]; }
    // Kernel launches of one operator application with the current shape
    // (source, the sweep's launches, psi -> phi).
    uint64_t launches_per_apply(int prec) const;

    // One operator application, on the device:
    //   phi_out = D L^{-1} ( [Q] + M S phi_in )     (phi_in / phi_out nullable)
    // prec 0 = FP64, 1 = FP32.  qang overrides the angular fixed source.
    int apply(int prec, const double *phi_in, bool with_fixed, double *phi_out,
              const double *qang_override, std::string &err);
    // apply() on caller-owned device vectors, ordered after the work already
    // queued on `s` (nullable: the legacy default stream); returns once
    // phi_out is written.
    int apply_external(int prec, const double *phi_in, bool with_fixed, double *phi_out, cudaStream_t s,
                       std::string &err);

    // One persistent-dataflow sweep psi = L^{-1} iso on caller-owned device
    // buffers (iso: phi layout, may be null; psi: psi layout; both in the
    // sweep precision), with caller-provided completion flags (n_items words)
    // and control words (ctl[0..2] error, [3] abort, [4] epoch).  Allocates
    // nothing; synchronizes `s` and reports a timed-out wait.
    int sweep_external(int prec, const void *iso, void *psi, uint32_t *done, uint32_t *ctl,
                       cudaStream_t s, std::string &err);

    // Device state read by the batch driver (batch.cpp); computes the
    // records of `prec` (compact or full) when stale and waits for the
    // instance's stream.
    struct DeviceView {
        const void *rec;  // CompactRecord<Real> (compact) or ItemRecord<Real>
        void *psi;
        double *iso;
        float *iso32;
        const double *qiso, *sigs, *scat, *w;
        double *phi, *tmp;
        const uint64_t *level_off;
        uint32_t n_levels, vg;
    };
    int device_view(int prec, DeviceView &v, std::string &err, bool compact);
    // The resident psi was written by a sweep of this precision elsewhere.
    void note_psi_precision(int prec) { last_psi_prec_ = prec; }
    uint64_t n_items() const { return sched_.n_padded; }
    // Polls of one flag or barrier before a persistent kernel's bounded wait
    // gives up (dataflow, persistent levels and the no-alloc sweep).
    void set_wait_limit(uint32_t polls) { spin_limit_ = polls; }
    // Order of the items within each (level, octant) segment of the schedule
    // (results are the same in any order): 0 increasing cell * A + angle, 1
    // Priorities' b-levels, longest downwind chain first, 2 seeded random.
    int set_work_order(int order, std::string &err);
    int work_order() const { return work_order_; }
    uint32_t wait_limit() const { return spin_limit_; }
    int solver() const { return solver_; }

    // One partition of a multi-partition mesh (the sweep of Util::sweepLocal,
    // src/Util.cc:138-145): faces whose neighbour is another partition take
    // their incoming psi from psiBound (src/Transport.cc:766-773), kept on
    // the device in both precisions.  Level schedule only.
    uint64_t n_bound_sides() const { return n_bound_; }
    // psi_bound: host memory in PsiBoundData layout ((side * A + a) * 3 + fv)
    // * G + g over all sides and the whole quadrature (src/PsiData.hh:253-262);
    // sides toward no other partition are not read.
    int set_psi_bound(const double *psi_bound, std::string &err);
    // The values held, in the same layout (other sides and, for an angle
    // shard, other directions zero).
    int get_psi_bound(double *psi_bound, std::string &err);
    // CommSides (src/CommSides.cc:48-240) on the device: toward partition q,
    // every (side, direction) whose face is outgoing here, in the reference's
    // (cell, face, direction) order, carries psi at the face's three vertices
    // (fv order) for every group.
    int side_counts(uint64_t q, uint64_t &n_send, uint64_t &n_recv, std::string &err);
    // (global side id, direction) of each packet sent to q.
    int side_send_list(uint64_t q, uint64_t *gside, uint32_t *angle, std::string &err);
    // packets to q from the resident psi into dst (device, FP64, [n][3][G]).
    int side_pack(uint64_t q, double *dst, cudaStream_t s, bool sync, std::string &err);
    // q's send list (its side_send_list), once: where each packet from q lands.
    int side_link(uint64_t q, uint64_t n, const uint64_t *gside, const uint32_t *angle, std::string &err);
    // packets from q (device, FP64, [n][3][G]) into the boundary values.
    int side_unpack(uint64_t q, const double *src, cudaStream_t s, bool sync, std::string &err);
    // L1 norms of psi - psi_prev and of psi over this sweeper's psi (FP64
    // sweep), then psi_prev = psi: SweeperPBJ's convergence test
    // (src/SweeperPBJ.cc:181-195).
    int psi_change(double &diff, double &norm, std::string &err);

    const MeshTables &tables() const { return *tables_; }
    const Quadrature &quadrature() const { return quad_; }
    // Levels, offsets and counts; items and tlevel are empty when the
    // schedule was levelled on the device (schedule_host fills them).
    const Schedule &schedule() const { return sched_; }
    // The schedule with its item list and t-levels on the host, copied back
    // from the device on first use.  Not safe to call concurrently with
    // other calls on the same sweeper.
    const Schedule &schedule_host() const;
    uint64_t n_cells() const { return nc_; }
    int n_angles() const { return A_; }
    int n_groups() const { return G_; }
    uint64_t phi_size() const { return nc_ * 4 * (uint64_t)G_; }
    uint64_t psi_size() const { return nc_ * (uint64_t)A_ * 4 * G_; }
    cudaStream_t stream() const { return stream_; }
    int device() const { return device_; }

private:
    struct LevelGraph {
        cudaGraphExec_t exec = nullptr;
    };
    int levels(int prec, bool has_iso, const double *qang, cudaEvent_t beg, cudaEvent_t end,
               std::string &err);
    int compute_item_abar(std::string &err);
    cudaError_t enqueue_levels(int prec, bool has_iso, const double *qang);
    // The level graph of the level schedule (built and cached on first use).
    int level_graph(int prec, bool has_iso, const double *qang, LevelGraph *&lg, std::string &err);
    // One operator application appended to the graph being captured on
    // stream_ (level schedule only; its level graph must exist already).
    int capture_apply(int prec, const double *phi_in, bool with_fixed, double *phi_out, std::string &err);
    // Captures (once) and returns the step graph of a source-iteration step
    // or of Arnoldi step k; nullptr when the shape has no level graph.
    int si_step_graph(cudaGraphExec_t &exec, std::string &err);
    int arnoldi_step_graph(int prec, int k, cudaGraphExec_t &exec, std::string &err);
    // Reads (and clears) the dataflow schedule's device error word.
    int check_device_error(std::string &err);
    LevelArgs level_args(int prec, const void *iso, const double *qang, void *psi) const;
    int launch_dataflow_shape(int prec, const LevelArgs &p, const DataflowArgs &df, cudaStream_t s,
                              std::string &err);
    // r_out (nullable): on return b - (I - K) x from the last cycle's Arnoldi
    // relation, without another sweep.
    int gmres(int prec, const double *b, double *x, int restart, double rtol, int iter_max,
              int &its, double &rnorm, SolveStats &st, std::string &err, double *r_out = nullptr);
    int ensure_krylov(int restart, std::string &err);
    // The drop-in sweep with its host copies overlapped: angle chunks (0 or 1:
    // one copy in, one sweep, one copy out) and the pipelined form.
    int host_chunks() const;
    int sweep_host_chunked(const double *source, double *psi, int K, std::string &err);
    // Allocates the record array of one precision; need_filled also requires
    // (and computes, when stale) its contents for the current cross sections.
    int ensure_records(int prec, bool need_filled, std::string &err, bool compact = false);

    std::shared_ptr<const MeshTables> tables_;
    Quadrature quad_;
    mutable Schedule sched_;
    uint64_t nc_ = 0;
    int A_ = 0, G_ = 0, device_ = 0;
    bool fp32_ = false, have_xs_ = false;
    int solver_ = 1;  // SolveKind
    int last_psi_prec_ = -1;
    uint32_t spin_limit_ = 1u << 22;  // about 2-4 s of polling
    int work_order_ = 0;

    cudaStream_t stream_ = nullptr;
    // level schedule on several streams: one per octant group, forked from
    // and joined into stream_ inside the captured graph
    cudaStream_t aux_[8] = {};
    cudaEvent_t fork_ = nullptr, join_[8] = {};
    uint32_t *d_items_ = nullptr;
    double4 *d_abar64_ = nullptr;
    float4 *d_abar32_ = nullptr;
    int4 *d_adj_ = nullptr;
    uint32_t *d_nbrmap_ = nullptr;
    double *d_cellk64_ = nullptr;
    float *d_cellk32_ = nullptr;
    double *d_w_ = nullptr;
    double *d_sigs_ = nullptr;
    double *d_scat_ = nullptr;
    double *d_qiso_ = nullptr;
    double *d_qang_ = nullptr;
    double *d_src_ = nullptr;     // staging for sweep_host's source
    double *d_iso_ = nullptr;
    float *d_iso32_ = nullptr;
    void *d_psi_ = nullptr;
    double *d_phi_ = nullptr, *d_r_ = nullptr, *d_tmp_ = nullptr;
    double *d_V_ = nullptr, *d_h_ = nullptr;
    int krylov_m_ = 0;
    void *d_flush_ = nullptr;
    Reducer red_;
    // level graphs by (precision, with an isotropic source, angular source)
    std::map<std::tuple<int, bool, const double *>, LevelGraph> graphs_;
    // whole solver steps as graphs: (kind 0 = source iteration step, 1 =
    // Arnoldi step k; precision; k); rebuilt when buffers or shapes change
    std::map<std::tuple<int, int, int>, cudaGraphExec_t> step_graphs_;
    void drop_step_graphs();
    // dataflow schedule
    LaunchShape shape_[2];  // [0] FP64, [1] FP32
    uint32_t *d_done_ = nullptr;   // per item: epoch of completion
    uint32_t *d_ctl_ = nullptr;    // [0..2] error, [3] abort, [4] epoch
    // record variant: per-item factors, [0] FP64, [1] FP32
    void *d_rec_[2] = {nullptr, nullptr};
    bool rec_valid_[2] = {false, false};
    // compact records (direct compact variant and the batch driver)
    void *d_crec_[2] = {nullptr, nullptr};
    bool crec_valid_[2] = {false, false};
    // direct dataflow: a completion epoch per (item, group vector)
    uint32_t *d_flags_ = nullptr;
    size_t flags_cap_ = 0;
    // persistent-levels schedule: level offsets and the grid barrier counter
    uint64_t *d_level_off_ = nullptr;
    // drop-in sweep in angle chunks: schedule positions grouped by chunk then
    // level, one level graph per chunk, copy streams and their events
    int chunk_k_ = 0;
    uint32_t *d_chunk_pos_ = nullptr;
    std::vector<uint64_t> chunk_off_;
    std::vector<cudaGraphExec_t> chunk_graphs_;
    cudaStream_t h2d_stream_ = nullptr, d2h_stream_ = nullptr;
    static constexpr int kMaxHostChunks = 16;
    cudaEvent_t ev_start_ = nullptr, ev_h2d_[kMaxHostChunks] = {}, ev_swept_[kMaxHostChunks] = {};
    // page-locked staging for pageable host buffers: [0, 1] source pieces,
    // [2, 3] psi pieces, each with the event of its last copy
    static constexpr size_t kStageBytes = 64ull << 20;
    void *h_stage_[4] = {};
    cudaEvent_t ev_stage_[4] = {};
    unsigned long long *d_barrier_ = nullptr;
    // partition boundary: bound side b <-> side; FP64 ghost rows (nc + b) * A
    // + a follow the cells' psi rows, FP32 ghost rows (2 (nc + B) + b) * A + a
    // follow the FP64 ghost rows (the FP32 neighbour table names those)
    uint64_t n_bound_ = 0;
    std::vector<uint64_t> bound_side_;
    std::vector<int64_t> side_bound_;
    int4 *d_adj32_ = nullptr;
    int angle_begin_ = 0, n_angles_full_ = 0;
    double *ghost64() const;
    float *ghost32() const;
    struct SideLink {
        bool built = false;
        std::vector<uint64_t> send_gside;
        std::vector<uint32_t> send_angle;
        uint64_t n_recv = 0;
        uint64_t *d_send_row = nullptr;   // per packet: psi row c * A + a
        uint32_t *d_send_vtx = nullptr;   // per packet: the face's cell vertices, 2 bits each
        uint64_t n_link = 0;
        uint64_t *d_recv_ghost = nullptr;  // per packet from q: ghost row b * A + a, or ~0
    };
    std::map<uint64_t, SideLink> links_;
    int side_link_build(uint64_t q, SideLink *&l, std::string &err);
    double *d_psi_prev_ = nullptr;
};

// The no-alloc sweep (tycho_sweeper_sweep_noalloc, sweep_noalloc.cu): scratch
// in a fixed file-scope device array instead of allocated memory.
int sweep_noalloc(Sweeper &sw, int precision, const void *iso, void *psi, void *stream,
                  std::string &err);
// Looks up the no-alloc scratch array's address on `device` (the current
// device) once per process; the first lookup loads the module holding it.
int noalloc_scratch_prepare(int device, std::string &err);

}  // namespace tycho
