// Quadrature and the wavefront schedule of the sweep.
//
// The reference walks each direction's cell dependency graph dynamically with
// per-thread priority queues (src/GraphTraverser.cc:467-759).  Here every
// (cell, angle) pair is levelled once: its t-level is the length of the
// longest upwind chain that ends at it, so all pairs of one level depend only
// on pairs of lower levels and can be updated together.  Items of a level are
// stored contiguously, grouped by the octant of their direction (directions
// of different octants never depend on each other, so the octant groups of a
// level can sweep on different streams) and within an octant in increasing
// (cell*A + angle) order, the psi row order.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "mesh.hpp"

namespace tycho {

struct Quadrature {
    int sn_order = 0;
    int n_angles = 0;
    std::vector<double> xi, eta, mu, wt;
};

// Product Gauss-Legendre x Chebyshev set (src/Quadrature.cc:150-244).
int make_quadrature(int sn_order, Quadrature &q, std::string &err);

constexpr uint32_t kSentinelItem = 0xFFFFFFFFu;  // level padding
constexpr uint64_t kLevelPad = 32;
constexpr int kOctants = 8;

// Octant of a direction: bit 2 xi < 0, bit 1 eta < 0, bit 0 mu < 0.
inline int octant(const Quadrature &q, int a)
{
    return (q.xi[a] < 0 ? 4 : 0) | (q.eta[a] < 0 ? 2 : 0) | (q.mu[a] < 0 ? 1 : 0);
}

struct Schedule {
    uint32_t n_levels = 0;
    uint64_t n_items = 0;                // cells x angles (without padding)
    uint64_t n_padded = 0;               // length of items (with padding)
    std::vector<uint64_t> level_offset;  // n_levels + 1 offsets into items
    std::vector<uint64_t> octant_offset; // n_levels * kOctants + 1: level l, octant o
                                         // starts at [l * kOctants + o]
    std::vector<uint32_t> items;         // cell*A + angle, grouped by level,
                                         // then octant, each (level, octant)
                                         // padded to kLevelPad
    std::vector<uint32_t> tlevel;        // (angle, cell)
    uint64_t n_incoming_interior = 0;    // sum over items of incoming interior faces
};

// omega.n with the reference's operation order (src/TychoMesh.cc:212-223).
inline double omega_dot_n(const Quadrature &q, int a, const double *n)
{
    return q.xi[a] * n[0] + q.eta[a] * n[1] + q.mu[a] * n[2];
}

// Levels every (cell, angle) pair.  Fails with kErrCycle if some direction's
// graph has a cycle (the reference would spin forever on such a mesh).
int build_schedule(const MeshTables &t, const Quadrature &q, Schedule &s, std::string &err);
// The same on the current CUDA device (schedule_gpu.cu), on stream `st`:
// level-by-level frontiers for all directions at once and a stable radix
// sort into (level, octant, cell*A + angle) order.  Identical result.  With
// d_items non-null the item list stays on the device: *d_items receives it
// (cudaMalloc'd, owned by the caller) and s.items and s.tlevel stay empty;
// tlevel_from_items derives s.tlevel once s.items has been copied back.
int build_schedule_device(const MeshTables &t, const Quadrature &q, Schedule &s, uint32_t **d_items,
                          cudaStream_t st, std::string &err);
// The schedule's positions grouped by angle chunk, then level (stable in
// schedule order), on the device: chunk j holds the angles [j*A/K,
// (j+1)*A/K).  *d_pos receives the positions (from the device pool, owned by
// the caller); positions off[j*n_levels + l] .. off[j*n_levels + l + 1] are
// chunk j's items of level l.  Padding items are left out.
int angle_chunks_device(const uint32_t *d_items, uint64_t n_padded, const uint64_t *d_level_off, uint32_t n_levels,
                        uint32_t A, uint32_t K, uint32_t **d_pos, std::vector<uint64_t> &off, cudaStream_t st,
                        std::string &err);
// s.tlevel from s.items and s.level_offset (every item of segment l has level l).
void tlevel_from_items(Schedule &s, uint64_t n_cells, int n_angles);

// Dependency counts as the GraphTraverser constructor sets them
// (src/GraphTraverser.cc:442-458) and b-levels as Priorities' BLevelData
// computes them (src/Priorities.cc:59-164); (angle, cell) order.
void dependency_counts(const MeshTables &t, const Quadrature &q, std::vector<uint32_t> &deps);
void b_levels(const MeshTables &t, const Quadrature &q, const Schedule &s, std::vector<uint32_t> &blev);

// b-levels as SweepSchedule's constructor computes them (calcDependencies and
// calcLevels, src/SweepSchedule.cc:107-125, :472-508): face f is a child face
// of (cell, angle) when omega.n > 1e-10 and a parent face when omega.n <
// -1e-10, interior faces only; a cell's level is the longest chain of child
// faces below it (0 when it has none).  (angle, cell) order; n_levels gets
// the largest level, as calcLevels returns it.  A cycle cannot stall it: as
// in the reference, a pair that a cycle keeps waiting is never passed on to
// its parents.
void sweep_schedule_levels(const MeshTables &t, const Quadrature &q, std::vector<uint32_t> &lev,
                           uint32_t &n_levels);

}  // namespace tycho
