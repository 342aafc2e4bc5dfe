// Host-safe types of the batched sweep (batch_kernels.cuh): the per-member
// slot table the host fills before each pass, the device work list the plan
// kernel builds, and the launchers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "launch.hpp"

namespace tycho {

constexpr uint32_t kBatchChunk = 4096;  // phi elements per reduction chunk

// Post-pass operation of a member (see batch_post_kernel).
enum BatchOp : uint32_t { kOpSI = 0, kOpOuter = 1, kOpInner = 2 };

struct alignas(16) BatchSlot {
    const void *rec;            // ItemRecord<Real> of the pass precision
    void *psi;                  // Real, psi layout
    double *iso;                // FP64 total source, phi layout
    float *iso32;               // FP32 copy (FP32 pass), else null
    const double *phi_in;       // scatter input (nullable)
    const double *q_fixed;      // fixed isotropic source (nullable)
    const double *sigma_s;      // per cell
    const double *scat;         // G x G, nullable = within-group
    const double *w;            // quadrature weights
    double *phi_out;            // psi -> phi output
    double *phi;                // solution (accept target)
    double *vec_r;              // residual r
    double *vec_d;              // correction delta
    const uint64_t *level_off;  // member's level offsets (n_levels + 1)
    uint64_t nc;
    uint32_t A, G, vg, vmagic, n_levels, op, active, accept;
    uint32_t level_shift;  // the member's level l runs at global level level_shift + l
    uint32_t solver;       // 4x4 solver (GaussElim), numbered as tycho_gauss_elim
};

// One member's items at one level, with what a warp needs to sweep them
// (resolved by the plan kernel, so a warp reads one segment and nothing else).
struct alignas(16) BatchSeg {
    const void *rec;       // the member's record of the level's first item
    void *psi;             // the member's psi (pass precision)
    const void *iso;       // the member's total source (pass precision)
    uint64_t item_begin;   // first item of the member's level
    uint32_t slot;
    uint32_t chunk_begin;  // first chunk of this segment within the level
    uint32_t G;
    uint32_t vmagic;
    uint32_t solver;       // the member's 4x4 solver (GaussElim)
};

// Members are split by vector width (groups per psi-row access): class 0
// = 1, class 1 = 2, class 2 = 4.
constexpr uint32_t kBatchClasses = 3;

// Block ranges of one level launch: class c owns blocks [c[c], c[c+1]).
struct BatchCuts {
    uint32_t c[kBatchClasses + 1];
};

struct BatchPlan {
    BatchSeg *segs;          // [level][class][seg_stride]
    uint32_t *level_nseg;    // [level][class]
    uint32_t *level_nchunk;  // [level][class]
    uint32_t *act;           // active slots in order
    uint32_t *chunk_prefix;  // [n_act + 1]: phi chunks of the active members
    uint32_t *n_act;         // [1]
    double *partials;        // [2 * total chunks]
    double *norms;           // [2 * n_slots]
    uint32_t seg_stride;     // = n_slots
};

// Launchers (batch_ops.cu: double and the streaming kernels, compiled with
// -fmad=false; batch_f32.cu: the float level kernel).  `grid` is the block
// count of the grid-stride kernels.
// rec_bytes: size of one record of the pass's kernel (full or compact).
cudaError_t launch_batch_plan(int ipw, const BatchSlot *slots, uint32_t n_slots, uint32_t max_levels,
                              uint32_t rec_bytes, const BatchPlan &pl, cudaStream_t s);
cudaError_t launch_batch_accept(const BatchSlot *slots, const BatchPlan &pl, unsigned grid, cudaStream_t s);
cudaError_t launch_batch_scatter(const BatchSlot *slots, const BatchPlan &pl, unsigned grid, cudaStream_t s);
cudaError_t launch_batch_psi_to_phi(bool fp32, const BatchSlot *slots, const BatchPlan &pl, unsigned grid,
                                    cudaStream_t s);
cudaError_t launch_batch_post(const BatchSlot *slots, const BatchPlan &pl, unsigned grid, cudaStream_t s);
cudaError_t launch_batch_finish(const BatchSlot *slots, const BatchPlan &pl, unsigned grid, cudaStream_t s);
// One global level: cut.c[3] blocks of 4 warps (programmatic dependent launch);
// any_solver: some member solves with Original or a Cramer solver (direct
// kernel only; the shared-memory record kernels take NoPivot).
template <typename Real>
cudaError_t launch_batch_level(int ipw, const BatchSlot *slots, const BatchPlan &pl, uint32_t level,
                               const BatchCuts &cut, bool any_solver, cudaStream_t s);
// The whole wavefront of a pass in one cooperative launch (as many blocks as
// can be resident; direct kernels only): barrier and queue counters zeroed
// before the launch, the bounded barrier's control words in df.
struct BatchPersistArgs {
    unsigned long long *barrier;  // arrivals
    uint32_t *queue;              // [level][class] chunks taken
    uint32_t max_levels;
    DataflowArgs df;              // err / abort / spin_limit of the barrier
};
template <typename Real>
cudaError_t launch_batch_persist(const BatchSlot *slots, const BatchPlan &pl, const BatchPersistArgs &a,
                                 bool any_solver, cudaStream_t s);
template <>
cudaError_t launch_batch_level<double>(int ipw, const BatchSlot *slots, const BatchPlan &pl, uint32_t level,
                                       const BatchCuts &cut, bool any_solver, cudaStream_t s);
template <>
cudaError_t launch_batch_level<float>(int ipw, const BatchSlot *slots, const BatchPlan &pl, uint32_t level,
                                      const BatchCuts &cut, bool any_solver, cudaStream_t s);

}  // namespace tycho
