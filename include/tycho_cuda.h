/*
 * tycho_cuda.h -- C ABI of the B200-native DG SN sweep.
 *
 * A drop-in for the transport sweep of lanl/tycho2: the reference's
 * SweeperAbstract (src/SweeperAbstract.hh:47-70) is implemented on top of
 * these calls (tycho2_b200/csrc/SweeperCuda.hh), so SourceIteration and the
 * Krylov driver call the GPU sweep unchanged.  Plain pointers and sizes only;
 * host arrays use the reference's layouts:
 *
 *   psi / angular source   ((cell*A + angle)*4 + vertex)*G + group
 *                          (PsiData, src/PsiData.hh:155-163)
 *   phi / isotropic source (cell*4 + vertex)*G + group
 *                          (PhiData, src/PsiData.hh:363-370)
 *   per-face tables        [cell][face][...] row-major, face k opposite
 *                          cell vertex k (src/TychoMeshIO.cc:128-145)
 *   psiBound               ((side*A + angle)*3 + face vertex)*G + group
 *                          (PsiBoundData, src/PsiData.hh:253-262): the
 *                          incoming psi of one partition's faces toward
 *                          other partitions
 *
 * Every entry point returns a tycho_status; tycho_last_error() gives the
 * message of the calling thread's last failure.  The reference aborts on
 * the same conditions through Insist (src/Assert.hh:62); the C++ adapter
 * maps a nonzero status back onto Insist.  There is no CPU fallback: without
 * a usable CUDA device the sweeper entry points fail with TYCHO_ERR_CUDA.
 *
 * Threading: a handle is used from one host thread at a time; distinct
 * handles are independent.
 */
#ifndef TYCHO_CUDA_H
#define TYCHO_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tycho_status {
    TYCHO_OK = 0,
    TYCHO_ERR_ARG = 1,
    TYCHO_ERR_IO = 2,
    TYCHO_ERR_FORMAT = 3,
    TYCHO_ERR_CUDA = 4,
    TYCHO_ERR_OOM = 5,
    TYCHO_ERR_CYCLE = 6,
    TYCHO_ERR_NOT_CONVERGED = 7,
    TYCHO_ERR_TIMEOUT = 8,
    TYCHO_ERR_BUSY = 9,
    TYCHO_ERR_MISSING = 10
} tycho_status;

/* Arithmetic of the sweep (psi, face fluxes, 4x4 solves). */
typedef enum tycho_precision { TYCHO_FP64 = 0, TYCHO_FP32 = 1 } tycho_precision;

/* Outer solver of tycho_sweeper_solve. */
typedef enum tycho_method {
    TYCHO_SOURCE_ITERATION = 0, /* SourceIteration::fixedPoint (src/SourceIteration.cc:127-207) */
    TYCHO_GMRES = 1,            /* SourceIteration::krylov (src/SourceIteration.cc:216-285) */
    TYCHO_MIXED_GMRES = 2       /* FP32-sweep GMRES inside FP64 iterative refinement */
} tycho_method;

/* Local 4x4 solve (deck key GaussElim, src/Global.hh:99-105; the four cases
   of gaussElim4, src/Transport.cc:277-677).  NoPivot runs in every kernel;
   Original and the Cramer solvers in the direct record kernels on the level
   schedule (128 threads per block), which a sweeper with one of them
   configures by default. */
typedef enum tycho_gauss_elim {
    TYCHO_GAUSS_ORIGINAL = 0,
    TYCHO_GAUSS_NOPIVOT = 1,
    TYCHO_GAUSS_CRAMER_GLU = 2,
    TYCHO_GAUSS_CRAMER_INTEL = 3
} tycho_gauss_elim;

typedef struct tycho_mesh tycho_mesh;       /* host-side mesh (ingest + tables) */
typedef struct tycho_sweeper tycho_sweeper; /* device-resident sweep instance */

const char *tycho_status_string(int status);
/* Copies the calling thread's last error message; returns its length. */
size_t tycho_last_error(char *buf, size_t len);
int tycho_version(void);

/* ---- mesh ingest: replaces TychoMesh::TychoMesh (src/TychoMesh.cc:193-260)
        and TychoMesh::readTychoMesh (src/TychoMeshIO.cc:153-333) ---------- */

/* Reads a one-partition .pmesh (src/ParallelMesh.hh:43-81). */
int tycho_mesh_read_pmesh(const char *path, tycho_mesh **out);
/* Reads one partition of a multi-partition .pmesh: what MPI rank
   `partition` reads (ParallelMesh::readInParallel, src/ParallelMesh.cc:
   581-690) with the tables TychoMesh builds from it, including the sides
   (faces on the mesh or partition boundary, numbered in (cell, face)
   order), their global face ids and the partition across each face
   (src/TychoMeshIO.cc:196-262).  Such a mesh cannot be written back. */
int tycho_mesh_read_pmesh_partition(const char *path, uint64_t partition, tycho_mesh **out);
/* partition, number of partitions, and the number of faces toward another
   partition (any pointer may be NULL). */
int tycho_mesh_partition_info(const tycho_mesh *mesh, uint64_t *partition, uint64_t *n_partitions,
                              uint64_t *n_bound_sides);
/* Material index of each cell [n] (TychoMesh::getCellMaterial; 1 for meshes
   made from arrays). */
int tycho_mesh_cell_material(const tycho_mesh *mesh, uint64_t *material);
/* For a mesh made from a reference TychoMesh's arrays (tycho_mesh_from_arrays)
   on one MPI rank of a multi-partition run: the rank, the number of ranks,
   adj_rank [n*4] (getAdjRank, UINT64_MAX = BAD_RANK on the mesh boundary)
   and side_gid [n_sides] (getLGSide, sides numbered in (cell, face) order as
   TychoMesh numbers them).  Call before making sweepers from the mesh. */
int tycho_mesh_set_partition(tycho_mesh *mesh, uint64_t partition, uint64_t n_partitions,
                             const uint64_t *adj_rank, const uint64_t *side_gid);
/* side [n*4] (TychoMesh::getSide, UINT64_MAX on interior faces), adj_rank
   [n*4] (getAdjRank: the partition across the face, this one for interior
   faces, UINT64_MAX on the mesh boundary), side_gid [n_sides] (getLGSide);
   any pointer may be NULL. */
int tycho_mesh_side_tables(const tycho_mesh *mesh, uint64_t *side, uint64_t *adj_rank, uint64_t *side_gid);
/* Reads a .smesh (src/SerialMesh.hh:43-68) as one partition, as the
   reference's util/PartitionColumns 1 1 would convert it. */
int tycho_mesh_read_smesh(const char *path, tycho_mesh **out);
/* Kuhn-split cube: n^3 hexes x 6 tets on [0,length]^3, interior vertices
   jittered by U(-jitter*h, jitter*h) per coordinate (seeded). */
int tycho_mesh_kuhn_cube(uint32_t n, double jitter, uint64_t seed, double length,
                         tycho_mesh **out);
/* From an already-loaded reference TychoMesh, through its getters
   (src/TychoMesh.hh:70-116): cell_nodes [n*4] (getCellNode), coords
   [n_nodes*3] (getNodeCoord), adj_cell [n*4] (getAdjCell, UINT64_MAX on the
   boundary), face_to_cell [n*12] (getFaceToCellVrtx), cell_gid [n]
   (getLGCell, may be NULL).  Volumes, areas, normals, cellToFaceVrtx and
   neighborVrtx are derived as TychoMesh derives them.  Such a mesh has no
   face records, so it cannot be written back as .smesh/.pmesh. */
int tycho_mesh_from_arrays(uint64_t n_cells, uint64_t n_nodes, const uint64_t *cell_nodes,
                           const double *coords, const uint64_t *adj_cell,
                           const uint64_t *face_to_cell, const uint64_t *cell_gid,
                           tycho_mesh **out);
int tycho_mesh_write_smesh(const tycho_mesh *mesh, const char *path);
int tycho_mesh_write_pmesh(const tycho_mesh *mesh, const char *path);
int tycho_mesh_info(const tycho_mesh *mesh, uint64_t *n_cells, uint64_t *n_nodes,
                    uint64_t *n_sides);
/* Copies TychoMesh tables out; any pointer may be NULL.  Sizes: adj_cell,
   cell_nodes [n*4]; neighbor_vrtx, face_to_cell [n*12]; cell_to_face [n*16]
   (UINT64_MAX at [c][f][f]); volume [n]; area [n*4]; normal [n*12];
   cell_gid [n]; coords [n_nodes*3].  Boundary = UINT64_MAX. */
int tycho_mesh_tables(const tycho_mesh *mesh, uint64_t *adj_cell, uint64_t *neighbor_vrtx,
                      uint64_t *face_to_cell, uint64_t *cell_to_face, uint64_t *cell_nodes,
                      double *volume, double *area, double *normal, uint64_t *cell_gid,
                      double *coords);
void tycho_mesh_free(tycho_mesh *mesh);

/* Host-side levelling of a mesh for one quadrature, no device needed.
   (angle, cell) order, any output may be NULL: t-levels of the wavefront
   schedule, dependency counts as the GraphTraverser constructor sets them
   (src/GraphTraverser.cc:442-458) and b-levels as Priorities' BLevelData
   computes them (src/Priorities.cc:59-164).  n_levels receives the number
   of wavefront levels.  TYCHO_ERR_CYCLE if some direction is cyclic. */
int tycho_mesh_levels(const tycho_mesh *mesh, int sn_order, uint32_t *tlevel, uint32_t *deps,
                      uint32_t *blevel, uint32_t *n_levels);

/* b-levels of SweepSchedule's constructor (calcDependencies and calcLevels,
   src/SweepSchedule.cc:107-125, :472-508), no device needed: a face is a
   child face of (cell, angle) when omega.n > 1e-10, a parent face when
   omega.n < -1e-10 (interior faces only), and a pair's level is the longest
   chain of child faces below it.  Unlike the GraphTraverser rule, faces with
   |omega.n| <= 1e-10 order nothing, so S6's exact ties form no cycle.
   levels [A * n_cells] in (angle, cell) order (may be NULL); n_levels
   receives the largest level, as calcLevels returns it. */
int tycho_mesh_sweep_schedule_levels(const tycho_mesh *mesh, int sn_order, uint32_t *levels,
                                     uint32_t *n_levels);

/* ---- quadrature: Quadrature::Quadrature (src/Quadrature.cc:150-244) ----- */

/* Fills the 2*sn^2 directions and weights; returns the count or -1. */
int tycho_quadrature(int sn_order, double *xi, double *eta, double *mu, double *wt);

/* ---- sweeper: SweeperAbstract (src/SweeperAbstract.hh:47-70) ----------- */

typedef struct tycho_sweeper_opts {
    int sn_order;   /* deck key snOrder */
    int n_groups;   /* deck key nGroups */
    int gauss_elim; /* tycho_gauss_elim, deck key GaussElim */
    int device;     /* CUDA device ordinal */
    int fp32;       /* nonzero: also prepare the FP32 sweep (mixed precision) */
    int tpi64;      /* threads per (cell,angle) item of the FP64 sweep, 0 = auto */
    int tpi32;      /* same for the FP32 sweep, 0 = auto */
    int schedule;   /* 0 = auto (one launch per level, compact records in
                       registers), 1 = one launch per wavefront level,
                       2 = one persistent dataflow launch per sweep */
    int levelling;  /* where the wavefront levels are computed: 0 = auto (on
                       the device from 1M cells x angles), 1 = host threads,
                       2 = device; the result is the same either way */
} tycho_sweeper_opts;

/* Builds the device-resident instance: uploads the mesh tables, levels every
   (cell, angle) pair into wavefronts (replaces the GraphTraverser constructor
   and Priorities, src/GraphTraverser.cc:416-459, src/Priorities.cc:396-435)
   and allocates psi.  Fails with TYCHO_ERR_CYCLE on a cyclic direction. */
int tycho_sweeper_create(const tycho_mesh *mesh, const tycho_sweeper_opts *opts,
                         tycho_sweeper **out);

/* The same for the directions [angle_begin, angle_end) of the quadrature
   only: an angle shard.  Each direction sweeps independently of the others,
   so the shards of one problem on several GPUs (one process each) sweep in
   parallel and the sum of their phi (tycho_sweeper_apply) over the shards
   is the whole problem's psiToPhi (src/Util.cc:85-97; the reference
   parallelises over spatial partitions instead, src/GraphTraverser.cc:659-731).
   Both 0: every direction, as tycho_sweeper_create. */
int tycho_sweeper_create_angles(const tycho_mesh *mesh, const tycho_sweeper_opts *opts, int angle_begin,
                                int angle_end, tycho_sweeper **sw);
void tycho_sweeper_destroy(tycho_sweeper *sw);

/* Cross sections (Problem::createCrossSections, src/Problem.cc:149-172):
   sigma_t[c], sigma_s[c] per cell.  scatter == NULL: within-group
   scattering sigma_s[c]/(4 pi) phi_g (src/Util.cc:118-130); otherwise the
   G x G matrix scatter[g*G + g'] scales sigma_s[c] for g' -> g. */
int tycho_sweeper_set_cross_sections(tycho_sweeper *sw, const double *sigma_t,
                                     const double *sigma_s, const double *scatter);

/* Fixed source Q (Problem::getSource, src/Problem.cc:140-143).
   kind 0: angular, psi layout (as the reference's PsiData source);
   kind 1: isotropic, phi layout.  q == NULL clears it. */
int tycho_sweeper_set_source(tycho_sweeper *sw, int kind, const double *q);

/* The drop-in SweeperAbstract::sweep(psi, source): psi = L^{-1} source for
   an angular source in psi layout, vacuum boundaries.  Host buffers; the
   copies in and out are part of the call.  From 64 MiB of psi (NoPivot),
   when at least one of the two buffers is page-locked (pinned, or
   registered with tycho_host_register), the copies and the sweep run in
   angle chunks on three streams so that uploads, downloads and the sweep
   overlap; a pageable buffer's copies are staged by the calling thread
   while the rest runs beside them. */
int tycho_sweeper_sweep(tycho_sweeper *sw, const double *source, double *psi);

/* Page-locks (cudaHostRegister, portable) / releases a host buffer that the
   caller keeps for many sweeps, such as the PsiData arrays a sweeper owns
   (SweeperAbstract's c_psi and c_source, src/SweeperAbstract.hh:68-69, host
   `new double[]`, src/PsiData.hh:94-103).  The buffer must be unregistered
   before it is freed.  No counterpart in the reference, which never copies
   to a device. */
int tycho_host_register(void *p, size_t bytes);
int tycho_host_unregister(void *p);

typedef struct tycho_solve_opts {
    int method;        /* tycho_method */
    int iter_max;      /* SI steps / Krylov iterations (deck key iterMax) */
    double err_max;    /* SI: L1 relative change; Krylov: relative residual (errMax) */
    int restart;       /* GMRES restart length */
    double inner_tol;  /* mixed: relative tolerance of the first FP32 solve (at most 1e-6) */
    int refine_max;    /* mixed: maximum correction solves */
} tycho_solve_opts;

typedef struct tycho_solve_stats {
    int iterations;        /* SI steps or total Krylov iterations */
    int sweeps_fp64;       /* FP64 sweeps performed */
    int sweeps_fp32;       /* FP32 sweeps performed */
    int refinements;       /* mixed: correction solves */
    double final_error;    /* SI: last L1 relative change; Krylov: relative residual */
    double seconds;        /* device time of the solve */
} tycho_solve_stats;

/* SweeperAbstract::solve (src/SweeperTraverse.cc:65-74): psi starts at 0 and
   the chosen outer iteration runs on the device.  phi_out / psi_out (host,
   may be NULL) receive the result; psi stays resident on the device.
   GMRES ends with the FP64 sweep psi = L^{-1}(M S phi + Q) of the reference's
   krylov (src/SourceIteration.cc:254-260) when psi_out is given; without it
   phi is the GMRES iterate and that sweep is skipped.
   TYCHO_MIXED_GMRES: x solves (I - K32) x = D L32^{-1} Q by FP32-sweep
   GMRES (FP64 vectors) to min(inner_tol, 1e-6); then r = T64(x) - x with one
   FP64 sweep (T = D L^{-1}(Q + M S .)), (I - K32) d = r by FP32-sweep GMRES,
   x += d.  The residual after a correction comes from the GMRES Arnoldi
   relation, without a sweep, when d is small enough that the FP32
   operator's error on it stays below a tenth of err_max; otherwise from
   another FP64 sweep.  Stops at ||r|| <= err_max ||D L32^{-1} Q||; with
   psi_out one FP64 sweep at the final phi supplies psi (unless the last
   residual sweep was at it). */
int tycho_sweeper_solve(tycho_sweeper *sw, const tycho_solve_opts *opts, double *phi_out,
                        double *psi_out, tycho_solve_stats *stats);

/* Writes the resident psi in the reference's .psi format
   (PsiData::writeToFile, src/PsiData.cc:62-106). */
int tycho_sweeper_write_psi(tycho_sweeper *sw, const char *path);
/* The resident psi of the last FP64 sweep, solve or operator application
   into host memory (PsiData layout, this sweeper's cells and directions). */
int tycho_sweeper_read_psi(tycho_sweeper *sw, double *psi);

/* Schedule facts: levels (max over angles), items (cells x angles) and the
   number of incoming interior faces summed over items. */
int tycho_sweeper_schedule_info(const tycho_sweeper *sw, uint32_t *n_levels, uint64_t *n_items,
                                uint64_t *n_incoming_interior);
/* The wavefront schedule itself (any pointer may be NULL): the item list
   (cell*A + angle, UINT32_MAX for padding) in level, then octant order, its
   length, and the n_levels * 8 + 1 offsets of its (level, octant) segments. */
int tycho_sweeper_schedule_arrays(const tycho_sweeper *sw, uint64_t *n_padded, uint32_t *items,
                                  uint64_t *octant_offset);
/* Kernel launches of one operator application of the given precision with
   its current launch shape (source, the sweep's launches, psi -> phi). */
int tycho_sweeper_launches(const tycho_sweeper *sw, int precision, uint64_t *launches);
/* Integer tables for parity, (angle, cell) order, any pointer may be NULL:
   t-levels of the wavefront schedule, the GraphTraverser constructor's
   dependency counts and Priorities' b-levels. */
int tycho_sweeper_levels(const tycho_sweeper *sw, uint32_t *tlevel, uint32_t *deps,
                         uint32_t *blevel);

/* Launch shape of one precision's sweep:
     schedule 1 = one launch per wavefront level, 2 = persistent dataflow,
              3 = persistent levels: one cooperative launch walking the
                  levels with a bounded grid barrier between them (variant 2
                  only; FP64 knob 8 or 16);
     variant  0 = item-parallel: knob lanes per (cell, angle) item, each lane
                  a strided subset of the groups (group tiling; 1..16),
              1 = warp tiles: 32 items per warp, factors in shared memory,
                  knob warps per block (1, 2, 4),
              2 = records: the per-item factors precomputed once per
                  cross-section set (128 B per item in FP32, 256 B in FP64),
                  pairs loaded several at a time; knob items per warp (8, 16, 32),
              3 = direct records: the same records loaded straight into
                  registers, one thread per (item, group vector), the source
                  read before the wait on the previous level; level schedule
                  only, knob threads per block (64, 128, 256; -64 / -128:
                  the same capped at 64 registers; -96 / -80: 64 threads
                  capped at 102 / 85 registers; FP32 with 2 or 4 groups per
                  vector also -196 / -180 / -172: the upwind faces (at most
                  three per cell and direction) in three slots instead of
                  four face positions, 64 threads capped at 102 / 85 / 73
                  registers),
              4 = direct compact records: 64 B (FP32) / 96 B (FP64) per item
                  holding the matrix inputs (face terms, sigma_t V/20, V/20)
                  and topology; the factors are rebuilt in registers with the
                  same arithmetic; level schedule, knob as for 3;
     vector   records (2, 3): groups per vector access of a psi row (1, 2, or
              4 in FP32; must divide nGroups); 0 = the widest that divides
              nGroups (4 or 2 in FP32, 2 in FP64). */
typedef struct tycho_launch_shape {
    int schedule;
    int variant;
    int knob;
    int vector;
    int streams;  /* level schedule: the octant groups of every level sweep
                     on this many concurrent streams (1, 2, 4, 8) inside one
                     captured graph; directions of different octants never
                     depend on each other */
} tycho_launch_shape;

/* Autotuner: times every launch shape of the given precision's sweep with
   `reps` operator applications each on this instance's own problem, keeps
   the fastest and reports it.  Cross sections must be set. */
int tycho_sweeper_autotune(tycho_sweeper *sw, int precision, int reps, tycho_launch_shape *best,
                           double *best_ms);
/* Sets the launch shape explicitly. */
int tycho_sweeper_configure(tycho_sweeper *sw, int precision, const tycho_launch_shape *shape);
/* Reads the current launch shape. */
int tycho_sweeper_get_shape(const tycho_sweeper *sw, int precision, tycho_launch_shape *shape);

/* A sweep that allocates nothing.  No counterpart in the reference.
   For callers that cannot allocate device memory when they sweep: a host
   framework that owns all device memory through its own pool and budget (an
   allocation behind its back breaks its accounting), a plugin that may only
   use the buffers its host hands it, or a time-critical loop that cannot
   afford cudaMalloc's implicit synchronization.  psi = L^{-1} iso for an isotropic source on the caller's
   own device buffers, in the sweep precision (0: double, 1: float):
     iso  phi layout (cell*4 + vertex)*G + group, may be NULL (zero source);
     psi  psi layout, written.
   The persistent dataflow kernel's scratch (per-item completion flags and
   control words) lives in one file-scope device array of 64 MiB + 256 B,
   which every GPU that loads this library holds until the process exits, so
   at most 16,777,216 cells x angles are accepted (larger: TYCHO_ERR_ARG).
   tycho_sweeper_create looks up that array's device address (once per
   device and process; the first lookup loads the module holding it), so the
   call itself maps and loads nothing.  All calls share the array and each
   leaves its flags behind (a per-call epoch makes them stale; the error and
   abort words are cleared at the start of every call), so calls that
   overlap on the GPU race.  The call runs on `stream` (a cudaStream_t, NULL
   = legacy default stream), reads the error words back and synchronizes
   `stream` before it returns.  It returns TYCHO_ERR_TIMEOUT if a bounded wait gave up
   (tycho_sweeper_set_wait_limit).  The sweeper's psi and results are not
   touched; with a records or direct-records launch shape whose records are
   stale (new cross sections), it recomputes them in place on `stream`. */
int tycho_sweeper_sweep_noalloc(tycho_sweeper *sw, int precision, const void *iso, void *psi,
                                void *stream);

/* The order in which each wavefront's (cell, direction) items are taken
   within a (level, octant) segment: the reference's traversal priorities
   (Priorities::calcPriorities, src/Priorities.cc:396-435, and the
   schedules of src/Sweeper.cc:373-515) as work orders of the level
   schedule.  0: increasing cell * A + angle (default); 1: b-levels, the
   longest downwind chain first (intraAngleP 1); 2: a seeded random order
   (intraAngleP 0).  psi is the same in every order (each item's arithmetic
   does not depend on it); only the dataflow and persistent schedules, which
   take items in this order, can run faster or slower. */
int tycho_sweeper_set_work_order(tycho_sweeper *sw, int order);

/* Bounded waits of the persistent kernels (dataflow schedule, persistent
   levels, tycho_sweeper_sweep_noalloc): polls of one completion flag or
   level barrier before a wait gives up, records the item and face it waited
   for, makes every warp drain, and the call returns TYCHO_ERR_TIMEOUT with
   the sweeper still usable.  Default 4,194,304 (seconds of polling).  The
   reference spins without a bound on the same waits
   (src/GraphTraverser.cc:518).  0 gives up at the first wait that is not
   already satisfied: the failure path can be exercised without a hang. */
int tycho_sweeper_set_wait_limit(tycho_sweeper *sw, uint32_t polls);

/* One operator application on caller-owned device vectors (phi layout,
   FP64): phi_out = D L^{-1} ([Q] + M S phi_in) in the given precision
   (lhsOperator's sweep with calcTotalSource and psiToPhi around it,
   src/SourceIteration.cc:76-114; phi_in NULL: no scattering source;
   with_fixed: add the fixed source).  For an angle shard phi_out is its
   directions' part of the sum.  Ordered after the work queued on `stream`
   (a cudaStream_t, NULL = legacy default stream); returns once phi_out is
   written. */
int tycho_sweeper_apply(tycho_sweeper *sw, int precision, const double *phi_in, int with_fixed, double *phi_out,
                        void *stream);

/* ---- one partition of a multi-partition mesh: Util::sweepLocal(psi,
        source, psiBound) and CommSides (src/Util.cc:138-145,
        src/CommSides.cc:48-240), the local sweep of the reference's PBJ and
        Schur sweepers (src/SweeperPBJ.cc, src/SweeperSchur.cc) -------------
   A sweeper made from a partition (tycho_mesh_read_pmesh_partition) reads
   the incoming psi on faces toward other partitions from psiBound
   (src/Transport.cc:766-773) instead of vacuum; every sweep, apply and
   solve uses the values last set.  Level schedule only; not in a batch,
   the service or the no-alloc sweep. */

/* Number of faces toward other partitions (0: an ordinary sweeper). */
int tycho_sweeper_bound_sides(const tycho_sweeper *sw, uint64_t *n_bound_sides);
/* psiBound in the reference's PsiBoundData layout, host memory:
   ((side * nAngles + angle) * 3 + fv) * nGroups + group over every side and
   direction of the quadrature (src/PsiData.hh:253-262); only faces toward
   another partition are read. */
int tycho_sweeper_set_psi_bound(tycho_sweeper *sw, const double *psi_bound);
/* The values held, in the same layout (zeros elsewhere). */
int tycho_sweeper_get_psi_bound(tycho_sweeper *sw, double *psi_bound);

/* CommSides on the device.  Toward partition q this partition sends, for
   every (cell, face toward q, direction) with the face outgoing, in that
   order (src/CommSides.cc:68-95), psi at the face's vertices fv = 0, 1, 2
   for every group: a packet of 3 * nGroups doubles.  n_send / n_recv: the
   reference's packet counts (any pointer may be NULL). */
int tycho_sweeper_side_counts(tycho_sweeper *sw, uint64_t q, uint64_t *n_send, uint64_t *n_recv);
/* (global side id, direction) of each packet sent to q, [n_send] each. */
int tycho_sweeper_side_send_list(tycho_sweeper *sw, uint64_t q, uint64_t *gside, uint32_t *angle);
/* The packets to q from the resident psi (the last sweep's) into dst, a
   device buffer of n_send * 3 * nGroups doubles.  Ordered after the work on
   `stream` and the sweeper's own; stream NULL: returns when done. */
int tycho_sweeper_side_pack(tycho_sweeper *sw, uint64_t q, double *dst, void *stream);
/* Once per neighbour: q's send list (from q's tycho_sweeper_side_send_list),
   so that each packet from q lands at psiBound(g, fv, angle, this
   partition's side with that global id) -- CommSides' receive
   (src/CommSides.cc:209-234).  A packet for a direction outside an angle
   shard is dropped. */
int tycho_sweeper_side_link(tycho_sweeper *sw, uint64_t q, uint64_t n, const uint64_t *gside,
                            const uint32_t *angle);
/* Packets from q (device, n * 3 * nGroups doubles, in q's send order) into
   psiBound.  Stream as for tycho_sweeper_side_pack. */
int tycho_sweeper_side_unpack(tycho_sweeper *sw, uint64_t q, const double *src, void *stream);
/* SweeperPBJ's convergence measure (src/SweeperPBJ.cc:181-195): L1 norms of
   psi - psi_prev and of psi over the resident FP64 psi, then psi_prev = psi
   (psi_prev starts at zero: a psi-sized FP64 copy on the device, allocated
   by the first call). */
int tycho_sweeper_psi_change(tycho_sweeper *sw, double *diff, double *norm);

/* Device timing of n back-to-back operator applications
   phi_out = D L^{-1} (M S phi_in + Q) in the given precision, on the
   sweeper's stream with CUDA events (inputs resident).  ms[0] = mean time
   of one application, ms[1] = mean time of its wavefront kernels alone. */
int tycho_sweeper_time_sweeps(tycho_sweeper *sw, int precision, int n, int flush_l2,
                              double *ms);

/* ---- batched solves: many independent instances on one GPU ------------
   No counterpart in the reference, which solves one problem per process.
   Members are sweepers (cross sections and isotropic fixed source set) on
   the batch's device, of any size, group count and SN order.  Every step
   runs one FP64 pass over the members in source iteration or at an outer
   refinement step and one FP32 pass over the members in their inner
   correction solve; each pass is one CUDA graph whose wavefront launches
   take their work from a device list over (member, level) built by the
   pass's first kernel.  A member's arithmetic and reductions do not depend
   on the other members: its result is bit-identical alone and in any mix. */

typedef struct tycho_batch tycho_batch;

typedef struct tycho_batch_opts {
    int method;       /* TYCHO_SOURCE_ITERATION (FP64 throughout) or
                         TYCHO_MIXED_GMRES's batched form: FP32-sweep source
                         iteration on phi from 0 to min(inner_tol, 1e-6),
                         then FP64 residuals r = T64(phi) - phi with FP32
                         source iteration on the correction; a correction
                         small enough that the FP32 operator's error on it
                         is below a tenth of err_max ends the solve without
                         another FP64 sweep (phi += d when the result is
                         read; psi is then not an FP64 sweep of phi) */
    int iter_max;     /* sweeps of the solve (FP32 inner sweeps included) */
    double err_max;   /* stop: L1 relative change of phi over one FP64 sweep
                         (SourceIteration.cc:167-175), or the same bound on
                         the residual after the last correction */
    double inner_tol; /* mixed: inner stop, L1 relative change of the correction */
    int inner_max;    /* mixed: inner sweeps per correction */
    int refine_max;   /* mixed: corrections */
} tycho_batch_opts;

/* ipw32 / ipw64: items per warp of the FP32 / FP64 wavefront kernels (8, 16,
   32: records staged in shared memory), or 0: records loaded straight into
   registers, one thread per (item, group vector). */
int tycho_batch_create(int device, int ipw32, int ipw64, tycho_batch **out);
void tycho_batch_destroy(tycho_batch *b);
/* The form of each pass's wavefront.  0 (default): one launch per global
   level (captured in the pass's graph, consecutive levels overlapped by
   programmatic dependent launch).  1: one persistent cooperative kernel per
   pass that walks every global level, its warps taking (member, level)
   chunks from a device work queue (one counter per level and vector-width
   class), with a bounded grid barrier between levels; the per-chunk
   arithmetic is the same, so results are bit-identical.  Direct kernels
   only (ipw32 = ipw64 = 0).  The reference has no batched form
   (src/GraphTraverser.cc:467-759 is its per-problem task queue). */
int tycho_batch_set_persistent(tycho_batch *b, int on);
/* Polls of the persistent form's grid barrier before it gives up: the step
   then returns TYCHO_ERR_TIMEOUT and the batch stays usable.  Default
   4,194,304; 0 gives up at the first barrier that is not already met. */
int tycho_batch_set_wait_limit(tycho_batch *b, uint32_t polls);
/* Adds a member (the sweeper must outlive its membership); its solve starts
   from phi = 0 at the next step.  *id identifies it. */
int tycho_batch_add(tycho_batch *b, tycho_sweeper *sw, const tycho_batch_opts *opts, int *id);
int tycho_batch_remove(tycho_batch *b, int id);
/* One step of every running member; *n_running = members still running. */
int tycho_batch_step(tycho_batch *b, int *n_running);
/* Steps until every member is done. */
int tycho_batch_run(tycho_batch *b);
/* A member's statistics and (phi != NULL) its phi, phi layout.  *done is 1
   once it has converged or hit a limit.  The member's sweeper keeps the FP64
   psi of its last sweep (tycho_sweeper_write_psi), except for a mixed
   member that finished on a correction without a final FP64 sweep. */
int tycho_batch_result(tycho_batch *b, int id, double *phi, tycho_solve_stats *stats, int *done);
/* Device time of all passes so far (ms) and pass counts, [0] FP64, [1] FP32,
   and the cell x angle x group updates swept in each. */
int tycho_batch_timing(const tycho_batch *b, double *ms, int *passes, double *updates);

/* ---- solve service: continuous batching under a device-memory budget -----
   Requests (mesh, SN order, groups, cross sections, isotropic source) are
   submitted with an arrival time; tycho_server_run serves them in arrival
   order: a request is admitted when its footprint (tycho_footprint_bytes)
   fits the budget next to the requests already resident, host threads build
   its device-resident sweeper (schedule, records, psi), and it joins the
   running batch at the next step; when its solve finishes, phi is copied to
   the caller's buffer, the request leaves the batch and its memory is freed.
   A request's result is bit-identical to the same request served alone. */

/* Device bytes a resident request holds (upper estimate, before building).
   mixed != 0: the mixed-precision service (FP32 sweep state as well);
   compact != 0: the service's batch runs the direct kernels (ipw 0) on
   compact records. */
uint64_t tycho_footprint_bytes(uint64_t n_cells, int sn_order, int n_groups, int mixed, int compact);

/* Sweepers, batches and servers take device memory from one stream-ordered
   pool per device, which keeps freed memory for the next allocation (freeing
   never waits for the device, and the next problem of the same size maps no
   new memory).  This hands the pool's unused memory back to the system;
   it waits for the device first. */
int tycho_release_cached_memory(int device);
/* Bytes that pool holds from the system on `device` and bytes of it in use
   (0 and 0 before the library's first allocation there). */
int tycho_device_memory(int device, uint64_t *pool_reserved, uint64_t *pool_used);

typedef struct tycho_server tycho_server;

typedef struct tycho_server_opts {
    int device;
    double budget_bytes;    /* device memory the resident requests may hold */
    int setup_threads;      /* host threads building sweepers */
    int ipw32, ipw64;       /* batched level kernels: items per warp (8, 16, 32; 0 = direct) */
    tycho_batch_opts solve; /* method TYCHO_SOURCE_ITERATION or TYCHO_MIXED_GMRES */
    double large_items;     /* cells x angles from which a request is large; 0 =
                               32e6.  Large requests do not join the batch of
                               small ones (a deep mesh would set its step
                               time): they run beside it on their own
                               streams */
    int large_batched;      /* 0: large requests are solved one at a time by
                               the single-instance solver (source iteration;
                               for the mixed service FP32-sweep GMRES(20) in
                               FP64 refinement to err_max in the residual
                               2-norm); 1: as members of a second batch */
} tycho_server_opts;

typedef struct tycho_request_info {
    int state;        /* 0 queued, 1 building, 2 built, 3 in the batch, 4 done, 5 failed */
    int status;       /* tycho_status of a failed request */
    double arrival;   /* seconds after tycho_server_run started */
    double admitted;  /* -1 if never */
    double built;
    double finished;
    uint64_t footprint;
    tycho_solve_stats stats;
} tycho_request_info;

int tycho_server_create(const tycho_server_opts *opts, tycho_server **out);
void tycho_server_destroy(tycho_server *s);
/* Copies the request's inputs; phi_out (phi layout) must stay valid until
   tycho_server_run returns.  scatter and q_iso may be NULL. */
int tycho_server_submit(tycho_server *s, const tycho_mesh *mesh, int sn_order, int n_groups,
                        const double *sigma_t, const double *sigma_s, const double *scatter,
                        const double *q_iso, double arrival, double *phi_out, int *id);
/* Serves every submitted request; returns when all are done or failed. */
int tycho_server_run(tycho_server *s);
int tycho_server_request(const tycho_server *s, int id, tycho_request_info *info);
int tycho_server_stats(const tycho_server *s, double *peak_bytes, int *peak_active, int *steps,
                       double *makespan);

#ifdef __cplusplus
}
#endif

#endif
