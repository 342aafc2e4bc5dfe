// Host-safe declarations of the wavefront launch (no device code): the
// per-level argument block and the launcher, instantiated for double (in
// device_ops.cu, FMA contraction off) and float (sweep_f32.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tycho {

// The 4x4 solvers of gaussElim4 (deck key GaussElim, src/Global.hh:99-105),
// numbered as tycho_gauss_elim.  Each one factors the group-independent
// matrix once per item into 16 numbers (and, for Original, a row order) and
// applies them to every group's right-hand side in the reference's order.
enum SolveKind : uint32_t { kSolveOriginal = 0, kSolveNoPivot = 1, kSolveCramerGlu = 2, kSolveCramerIntel = 3 };

struct LevelArgs {
    const uint32_t *items;   // cell*A + angle, level-sorted
    const void *abar;        // Real4 per item: face area * omega.n, faces 0..3
    const int4 *adj;         // per cell: neighbour across face f, -1 on the boundary
    const uint32_t *nbrmap;  // per cell: 2 bits per (face f, vertex j): neighbour's vertex at j
    const void *cellk;       // Real[3] per cell: V/20, sigma_t V/20, 2 sigma_t V/20
    const void *iso;         // Real, phi layout: isotropic total source (nullable)
    const double *qang;      // angular source, psi layout, FP64 only (nullable)
    void *psi;               // Real, psi layout
    uint32_t A, G;
    uint32_t gmagic;         // ceil(2^32 / G): pair -> item in the warp-tile variant (0 when G == 1)
    uint32_t vg;             // record variant: groups per vector access (divides G)
    uint32_t vmagic;         // ceil(2^32 / (G / vg)): task -> item (0 when G == vg)
    uint32_t solver;         // 4x4 solver (deck key GaussElim), numbered as tycho_gauss_elim
};

// Record variant's group vector width: 16-byte accesses where G allows.
constexpr uint32_t record_vg(bool fp32, uint32_t G)
{
    return fp32 ? (G % 4 == 0 ? 4 : (G % 2 == 0 ? 2 : 1)) : (G % 2 == 0 ? 2 : 1);
}

// Per-sweep state of the persistent (dataflow) schedule.
struct DataflowArgs {
    uint32_t *done;       // per cell*A + angle: epoch of the sweep that finished it
    uint32_t *err;        // [0] error code (0 = none), [1] item, [2] face
    uint32_t *abort;      // raised on the first failure; every warp drains
    const uint32_t *epoch;  // device word: this sweep's epoch (never 0)
    uint64_t n_items;     // padded item count, a multiple of 32
    uint32_t spin_limit;  // polls of one upwind flag before giving up
};
constexpr uint32_t kErrTimeoutCode = 1;

// Launches the wavefront kernel over items [begin, end) with `tpi` threads
// per item (1, 2, 4, 8 or 16).
template <typename Real>
cudaError_t launch_level(int tpi, const LevelArgs &p, uint64_t begin, uint64_t end, cudaStream_t s);

// The whole sweep as one cooperative launch of `grid` 256-thread blocks
// (at most the co-resident count from dataflow_blocks_per_sm).
template <typename Real>
cudaError_t launch_dataflow(int tpi, const LevelArgs &p, const DataflowArgs &df, unsigned grid,
                            cudaStream_t s);
template <typename Real>
cudaError_t dataflow_blocks_per_sm(int tpi, int *blocks);

// Warp-tile variant (sweep_tiles.cuh): 32 items per warp, `wpb` warps per
// block (1, 2 or 4); same contracts as the launchers above.
template <typename Real>
cudaError_t launch_level_tile(int wpb, const LevelArgs &p, uint64_t begin, uint64_t end, cudaStream_t s);
template <typename Real>
cudaError_t launch_dataflow_tile(int wpb, const LevelArgs &p, const DataflowArgs &df, unsigned grid,
                                 cudaStream_t s);
template <typename Real>
cudaError_t tile_dataflow_blocks_per_sm(int wpb, int *blocks);

// Record variant (sweep_records.cuh): per-item factors precomputed once per
// cross-section set into `rec` (128 B per item for float, 256 B for double).
constexpr size_t record_bytes(bool fp32) { return fp32 ? 128 : 256; }
template <typename Real>
cudaError_t launch_item_records(const LevelArgs &p, uint64_t n, void *rec, cudaStream_t s);
template <typename Real>
cudaError_t launch_level_record(int wpb, const LevelArgs &p, const void *rec, uint64_t begin, uint64_t end,
                                cudaStream_t s);
template <typename Real>
cudaError_t launch_dataflow_record(int wpb, const LevelArgs &p, const void *rec, const DataflowArgs &df,
                                   unsigned grid, cudaStream_t s);
template <typename Real>
cudaError_t record_dataflow_blocks_per_sm(int ipw, int vg, int *blocks);
// Direct record variant (level schedule only): one thread per (item, group
// vector), `bs` threads per block (64, 128 or 256).
template <typename Real>
cudaError_t launch_direct_level(int bs, const LevelArgs &p, const void *rec, uint64_t begin, uint64_t end,
                                cudaStream_t s, bool compact);
// Direct variants on the dataflow schedule: one cooperative launch, a
// completion flag per (item, group vector) in df.done (n_cells * A * G/vg
// words, G/vg a power of two <= 32).
template <typename Real>
cudaError_t launch_direct_dataflow(const LevelArgs &p, const void *rec, bool compact, const DataflowArgs &df,
                                   unsigned grid, cudaStream_t s);
template <typename Real>
cudaError_t direct_dataflow_blocks_per_sm(int vg, bool compact, int *blocks);
// Direct kernel (compact records, NoPivot, p.vg 1 or 2) over the schedule
// positions pos[begin, end).
template <typename Real>
cudaError_t launch_direct_subset(const LevelArgs &p, const void *rec, const uint32_t *pos, uint64_t begin,
                                 uint64_t end, cudaStream_t s);
// Compact records (64 B per item for float, 96 B for double): the inputs of
// each item's matrix, from which the direct kernels rebuild its factors.
constexpr size_t compact_record_bytes(bool fp32) { return fp32 ? 64 : 112; }
template <typename Real>
cudaError_t launch_compact_records(const LevelArgs &p, uint64_t n, void *rec, cudaStream_t s);
// Persistent levels: one cooperative launch, a bounded grid barrier between
// levels (level_off: device copy of the n_levels + 1 level offsets).
template <typename Real>
cudaError_t launch_persist_record(int ipw, const LevelArgs &p, const void *rec, const uint64_t *level_off,
                                  uint32_t n_levels, unsigned long long *barrier, const DataflowArgs &df,
                                  unsigned grid, cudaStream_t s);
template <typename Real>
cudaError_t record_persist_blocks_per_sm(int ipw, int vg, int *blocks);

}  // namespace tycho
