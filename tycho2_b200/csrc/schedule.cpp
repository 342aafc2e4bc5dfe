// Quadrature and host-side levelling of the sweep's dependency graphs.
#include "schedule.hpp"

#include <algorithm>
#include <cmath>

#include "gauss_legendre_tables.h"
#include "status.hpp"

namespace tycho {

int make_quadrature(int sn, Quadrature &q, std::string &err)
{
    const double *gn = nullptr, *gw = nullptr;
    if (tycho_gl_table(sn, &gn, &gw) != 0) {
        err = "Quadrature order not supported: " + std::to_string(sn);
        return kErrArg;
    }
    const double pi = M_PI;
    q.sn_order = sn;
    q.n_angles = 2 * sn * sn;
    q.xi.resize(q.n_angles); q.eta.resize(q.n_angles);
    q.mu.resize(q.n_angles); q.wt.resize(q.n_angles);
    for (int i = 0; i < sn; ++i)
        for (int k = 0; k < 2 * sn; ++k) {
            double phi = (2.0 * pi) / (2 * sn) * (k + 0.5);
            int idx = i * 2 * sn + k;
            q.xi[idx] = std::sqrt(1.0 - gn[i] * gn[i]) * std::cos(phi);
            q.eta[idx] = std::sqrt(1.0 - gn[i] * gn[i]) * std::sin(phi);
            q.mu[idx] = gn[i];
            q.wt[idx] = gw[i] * (2.0 * pi) / (2 * sn);
        }
    return kOk;
}

namespace {

// Bit k of the mask is set when face k is incoming, i.e. !(omega.n > 0)
// (src/TychoMesh.hh:107-110); ties count as incoming, as in the reference.
inline unsigned incoming_mask(const MeshTables &t, const Quadrature &q, uint64_t c, int a)
{
    unsigned m = 0;
    for (int f = 0; f < 4; ++f)
        if (!(omega_dot_n(q, a, &t.normal[(c * 4 + f) * 3]) > 0)) m |= 1u << f;
    return m;
}

// Faces that carry flux: bits 0-3 upwind (omega.n < 0), bits 4-7 downwind
// (omega.n > 0).  A face with omega.n == 0 exactly contributes nothing to the
// cell solve (Transport.cc:113 and :184 test area > 0 / area < 0) yet the
// reference counts it as incoming on both sides, a two-cycle on which its
// traversal never finishes (it happens on Kuhn meshes with S6, whose 45 degree
// azimuth makes xi == eta).  The wavefront schedule orders on flux-carrying
// faces only; the result is the same psi the reference would compute.
inline unsigned flux_mask(const MeshTables &t, const Quadrature &q, uint64_t c, int a)
{
    unsigned m = 0;
    for (int f = 0; f < 4; ++f) {
        const double odn = omega_dot_n(q, a, &t.normal[(c * 4 + f) * 3]);
        if (odn < 0) m |= 1u << f;
        if (odn > 0) m |= 16u << f;
    }
    return m;
}

}  // namespace

void dependency_counts(const MeshTables &t, const Quadrature &q, std::vector<uint32_t> &deps)
{
    const uint64_t nc = t.n_cells;
    const int A = q.n_angles;
    deps.assign((size_t)A * nc, 0);
    #pragma omp parallel for schedule(static)
    for (int a = 0; a < A; ++a)
        for (uint64_t c = 0; c < nc; ++c) {
            unsigned m = incoming_mask(t, q, c, a);
            uint32_t d = 0;
            for (int f = 0; f < 4; ++f)
                if ((m >> f & 1u) && t.adj_cell[c * 4 + f] != kNone) ++d;
            deps[(size_t)a * nc + c] = d;
        }
}

int build_schedule(const MeshTables &t, const Quadrature &q, Schedule &s, std::string &err)
{
    const uint64_t nc = t.n_cells;
    const int A = q.n_angles;
    if ((uint64_t)A * nc >= (1ull << 32)) {
        err = "cells x angles exceeds 2^32 items";
        return kErrArg;
    }
    s = Schedule();
    s.tlevel.assign((size_t)A * nc, 0);
    std::vector<uint32_t> level_count_per_angle((size_t)A, 0);
    int cyclic = 0;
    uint64_t incoming_total = 0;
    #pragma omp parallel for schedule(dynamic) reduction(| : cyclic) reduction(+ : incoming_total)
    for (int a = 0; a < A; ++a) {
        std::vector<uint32_t> cnt(nc), queue(nc);
        std::vector<unsigned char> mask(nc);
        uint32_t *lev = &s.tlevel[(size_t)a * nc];
        size_t tail = 0;
        for (uint64_t c = 0; c < nc; ++c) {
            unsigned m = flux_mask(t, q, c, a);
            mask[c] = (unsigned char)m;
            uint32_t d = 0;
            for (int f = 0; f < 4; ++f)
                if ((m >> f & 1u) && t.adj_cell[c * 4 + f] != kNone) ++d;
            cnt[c] = d;
            incoming_total += d;
            if (d == 0) queue[tail++] = (uint32_t)c;
        }
        size_t head = 0;
        uint32_t maxlev = 0;
        while (head < tail) {
            uint32_t c = queue[head++];
            for (int f = 0; f < 4; ++f) {
                uint64_t adj = t.adj_cell[(uint64_t)c * 4 + f];
                if (adj == kNone || !(mask[c] >> (f + 4) & 1u)) continue;
                if (lev[adj] < lev[c] + 1) lev[adj] = lev[c] + 1;
                if (--cnt[adj] == 0) queue[tail++] = (uint32_t)adj;
            }
            maxlev = std::max(maxlev, lev[c]);
        }
        if (tail != nc) cyclic |= 1;
        level_count_per_angle[a] = maxlev + 1;
    }
    if (cyclic) {
        err = "a direction's cell dependency graph has a cycle";
        return kErrCycle;
    }
    s.n_incoming_interior = incoming_total;
    s.n_levels = *std::max_element(level_count_per_angle.begin(), level_count_per_angle.end());
    // Items per (level, octant); each such segment is padded to a multiple
    // of kLevelPad with sentinel items, so that a warp's chunk never spans
    // two levels (or two octants).
    std::vector<int> oct(A);
    for (int a = 0; a < A; ++a) oct[a] = octant(q, a);
    const size_t nseg = (size_t)s.n_levels * kOctants;
    std::vector<uint64_t> count(nseg, 0);
    for (uint64_t c = 0; c < nc; ++c)
        for (int a = 0; a < A; ++a) count[(size_t)s.tlevel[(size_t)a * nc + c] * kOctants + oct[a]]++;
    s.octant_offset.resize(nseg + 1);
    s.octant_offset[0] = 0;
    for (size_t k = 0; k < nseg; ++k)
        s.octant_offset[k + 1] = s.octant_offset[k] + (count[k] + kLevelPad - 1) / kLevelPad * kLevelPad;
    s.level_offset.resize(s.n_levels + 1);
    for (uint32_t l = 0; l <= s.n_levels; ++l) s.level_offset[l] = s.octant_offset[(size_t)l * kOctants];
    s.n_items = (uint64_t)A * nc;
    s.n_padded = s.level_offset[s.n_levels];
    std::vector<uint64_t> pos(s.octant_offset.begin(), s.octant_offset.end() - 1);
    s.items.assign(s.level_offset[s.n_levels], kSentinelItem);
    for (uint64_t c = 0; c < nc; ++c)
        for (int a = 0; a < A; ++a) {
            const size_t k = (size_t)s.tlevel[(size_t)a * nc + c] * kOctants + oct[a];
            s.items[pos[k]++] = (uint32_t)(c * A + a);
        }
    return kOk;
}

void tlevel_from_items(Schedule &s, uint64_t n_cells, int n_angles)
{
    s.tlevel.assign((size_t)n_angles * n_cells, 0);
    #pragma omp parallel for schedule(dynamic, 1)
    for (int64_t l = 0; l < (int64_t)s.n_levels; ++l)
        for (uint64_t i = s.level_offset[l]; i < s.level_offset[l + 1]; ++i) {
            const uint32_t ca = s.items[i];
            if (ca == kSentinelItem) continue;
            const uint64_t c = ca / (uint32_t)n_angles, a = ca % (uint32_t)n_angles;
            s.tlevel[a * n_cells + c] = (uint32_t)l;
        }
}

void b_levels(const MeshTables &t, const Quadrature &q, const Schedule &s, std::vector<uint32_t> &blev)
{
    const uint64_t nc = t.n_cells;
    const int A = q.n_angles;
    blev.assign((size_t)A * nc, 0);
    // Visit items from the highest level down: every downwind neighbour of a
    // level-L pair sits at a level > L, so it is final when L is visited.
    for (uint32_t l = s.n_levels; l-- > 0;) {
        const uint64_t b = s.level_offset[l], e = s.level_offset[l + 1];
        #pragma omp parallel for schedule(static)
        for (uint64_t i = b; i < e; ++i) {
            uint32_t ca = s.items[i];
            if (ca == kSentinelItem) continue;
            uint64_t c = ca / A;
            int a = (int)(ca - c * A);
            unsigned m = incoming_mask(t, q, c, a);
            uint32_t best = 0;
            for (int f = 0; f < 4; ++f) {
                uint64_t adj = t.adj_cell[c * 4 + f];
                if (adj == kNone || (m >> f & 1u)) continue;
                best = std::max(best, blev[(size_t)a * nc + adj] + 1);
            }
            blev[(size_t)a * nc + c] = best;
        }
    }
}

void sweep_schedule_levels(const MeshTables &t, const Quadrature &q, std::vector<uint32_t> &lev,
                           uint32_t &n_levels)
{
    constexpr double kTol = 1.e-10;  // src/SweepSchedule.cc:56
    const uint64_t nc = t.n_cells;
    const int A = q.n_angles;
    lev.assign((size_t)A * nc, 0);
    uint32_t top = 0;
    #pragma omp parallel for schedule(dynamic) reduction(max : top)
    for (int a = 0; a < A; ++a) {
        // bits 0-3 child faces, 4-7 parent faces (interior only)
        std::vector<unsigned char> rel(nc);
        std::vector<uint32_t> need(nc), queue;
        queue.reserve(nc);
        uint32_t *L = &lev[(size_t)a * nc];
        for (uint64_t c = 0; c < nc; ++c) {
            unsigned m = 0, kids = 0;
            for (int f = 0; f < 4; ++f) {
                if (t.adj_cell[c * 4 + f] == kNone) continue;
                const double odn = omega_dot_n(q, a, &t.normal[(c * 4 + f) * 3]);
                if (odn > kTol) { m |= 1u << f; ++kids; }
                else if (odn < -kTol) m |= 16u << f;
            }
            rel[c] = (unsigned char)m;
            need[c] = kids;
            if (kids == 0) queue.push_back((uint32_t)c);
        }
        // Leaves first; a cell is visited once its last child is, so its
        // level is final when it passes it on to its parents.
        for (size_t h = 0; h < queue.size(); ++h) {
            const uint32_t c = queue[h];
            for (int f = 0; f < 4; ++f) {
                if (!(rel[c] >> (f + 4) & 1u)) continue;
                const uint64_t p = t.adj_cell[(uint64_t)c * 4 + f];
                if (L[p] < L[c] + 1) L[p] = L[c] + 1;
                if (--need[p] == 0) queue.push_back((uint32_t)p);
            }
            top = std::max(top, L[c]);
        }
    }
    n_levels = top;
}

}  // namespace tycho
