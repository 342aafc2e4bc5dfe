// extern "C" entry points declared in include/tycho_cuda.h.
#include "../../include/tycho_cuda.h"

#include <cstring>
#include <memory>
#include <exception>
#include <new>
#include <string>

#include "mesh.hpp"
#include "schedule.hpp"
#include "status.hpp"
#include "batch.hpp"
#include "devmem.hpp"
#include "server.hpp"
#include "sweeper.hpp"

struct tycho_mesh {
    tycho::MeshRecords rec;
    // shared with the sweepers and served requests made from this mesh, so
    // that they hold the tables without copying them
    std::shared_ptr<tycho::MeshTables> tabp = std::make_shared<tycho::MeshTables>();
    tycho::MeshTables &tab = *tabp;
};

struct tycho_sweeper {
    tycho::Sweeper sw;
};

struct tycho_batch {
    tycho::Batch b;
};

struct tycho_server {
    tycho::Server s;
};

namespace tycho {

static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }
const std::string &last_error() { return g_last_error; }

}  // namespace tycho

namespace {

int finish(int status, const std::string &err)
{
    if (status != tycho::kOk) tycho::set_last_error(err.empty() ? tycho_status_string(status) : err);
    return status;
}

template <typename F>
int guarded(F &&f)
{
    try {
        return f();
    } catch (const std::bad_alloc &) {
        tycho::set_last_error("host allocation failed");
        return tycho::kErrOom;
    } catch (const std::exception &e) {
        tycho::set_last_error(e.what());
        return tycho::kErrArg;
    }
}

int mesh_from_records(tycho_mesh *m, tycho_mesh **out)
{
    std::string err;
    int st = tycho::build_tables(m->rec, m->tab, err);
    if (st != tycho::kOk) {
        delete m;
        return finish(st, err);
    }
    *out = m;
    return tycho::kOk;
}

}  // namespace

extern "C" {

const char *tycho_status_string(int s)
{
    switch (s) {
    case TYCHO_OK: return "ok";
    case TYCHO_ERR_ARG: return "invalid argument";
    case TYCHO_ERR_IO: return "I/O error";
    case TYCHO_ERR_FORMAT: return "malformed input";
    case TYCHO_ERR_CUDA: return "CUDA error";
    case TYCHO_ERR_OOM: return "out of memory";
    case TYCHO_ERR_CYCLE: return "cyclic sweep dependency";
    case TYCHO_ERR_NOT_CONVERGED: return "not converged";
    case TYCHO_ERR_TIMEOUT: return "device wait timed out";
    case TYCHO_ERR_BUSY: return "admission refused";
    case TYCHO_ERR_MISSING: return "required input not set";
    default: return "unknown status";
    }
}

size_t tycho_last_error(char *buf, size_t len)
{
    const std::string &e = tycho::last_error();
    if (buf && len) {
        size_t n = e.size() < len - 1 ? e.size() : len - 1;
        std::memcpy(buf, e.data(), n);
        buf[n] = 0;
    }
    return e.size();
}

int tycho_version(void) { return 1; }

int tycho_mesh_read_pmesh(const char *path, tycho_mesh **out)
{
    if (!path || !out) return finish(TYCHO_ERR_ARG, "null argument");
    return guarded([&] {
        auto *m = new tycho_mesh;
        std::string err;
        int st = tycho::read_pmesh(path, m->rec, err);
        if (st != tycho::kOk) { delete m; return finish(st, err); }
        return mesh_from_records(m, out);
    });
}

int tycho_mesh_read_pmesh_partition(const char *path, uint64_t partition, tycho_mesh **out)
{
    if (!path || !out) return finish(TYCHO_ERR_ARG, "null argument");
    if (partition > (uint64_t)INT64_MAX) return finish(TYCHO_ERR_ARG, "bad partition");
    return guarded([&] {
        auto *m = new tycho_mesh;
        std::string err;
        int st = tycho::read_pmesh(path, m->rec, err, (int64_t)partition);
        if (st != tycho::kOk) { delete m; return finish(st, err); }
        return mesh_from_records(m, out);
    });
}

int tycho_mesh_partition_info(const tycho_mesh *m, uint64_t *partition, uint64_t *n_partitions,
                              uint64_t *n_bound_sides)
{
    if (!m) return finish(TYCHO_ERR_ARG, "null mesh");
    const auto &t = m->tab;
    if (partition) *partition = t.partition;
    if (n_partitions) *n_partitions = t.n_partitions;
    if (n_bound_sides) {
        uint64_t n = 0;
        if (!t.adj_rank.empty())
            for (uint64_t i = 0; i < t.n_cells * 4; ++i)
                n += t.adj_cell[i] == tycho::kNone && t.adj_rank[i] != tycho::kNone && t.adj_rank[i] != t.partition;
        *n_bound_sides = n;
    }
    return TYCHO_OK;
}

int tycho_mesh_cell_material(const tycho_mesh *m, uint64_t *material)
{
    if (!m || !material) return finish(TYCHO_ERR_ARG, "null argument");
    const auto &t = m->tab;
    if (t.cell_material.size() != t.n_cells) return finish(TYCHO_ERR_MISSING, "mesh has no material indices");
    std::memcpy(material, t.cell_material.data(), sizeof(uint64_t) * t.n_cells);
    return TYCHO_OK;
}

int tycho_mesh_set_partition(tycho_mesh *m, uint64_t partition, uint64_t n_partitions, const uint64_t *adj_rank,
                             const uint64_t *side_gid)
{
    if (!m || !adj_rank || !side_gid) return finish(TYCHO_ERR_ARG, "null argument");
    auto &t = m->tab;
    if (n_partitions == 0 || partition >= n_partitions) return finish(TYCHO_ERR_ARG, "bad partition");
    for (uint64_t i = 0; i < t.n_cells * 4; ++i)
        if (t.adj_cell[i] == tycho::kNone && adj_rank[i] != tycho::kNone && adj_rank[i] >= n_partitions)
            return finish(TYCHO_ERR_ARG, "adjacent partition out of range");
    t.partition = partition;
    t.n_partitions = n_partitions;
    t.adj_rank.assign(adj_rank, adj_rank + t.n_cells * 4);
    t.side_gid.assign(side_gid, side_gid + t.n_sides);
    return TYCHO_OK;
}

int tycho_mesh_side_tables(const tycho_mesh *m, uint64_t *side, uint64_t *adj_rank, uint64_t *side_gid)
{
    if (!m) return finish(TYCHO_ERR_ARG, "null mesh");
    const auto &t = m->tab;
    if (side) std::memcpy(side, t.side.data(), sizeof(uint64_t) * t.side.size());
    if (adj_rank) {
        if (t.adj_rank.empty()) {
            // tables from arrays: one partition, no partition boundary
            for (uint64_t i = 0; i < t.n_cells * 4; ++i) adj_rank[i] = t.adj_cell[i] == tycho::kNone ? tycho::kNone : 0;
        } else {
            std::memcpy(adj_rank, t.adj_rank.data(), sizeof(uint64_t) * t.adj_rank.size());
        }
    }
    if (side_gid) {
        if (t.side_gid.size() == t.n_sides) std::memcpy(side_gid, t.side_gid.data(), sizeof(uint64_t) * t.n_sides);
        else for (uint64_t i = 0; i < t.n_sides; ++i) side_gid[i] = i;
    }
    return TYCHO_OK;
}

int tycho_mesh_read_smesh(const char *path, tycho_mesh **out)
{
    if (!path || !out) return finish(TYCHO_ERR_ARG, "null argument");
    return guarded([&] {
        auto *m = new tycho_mesh;
        std::string err;
        int st = tycho::read_smesh(path, m->rec, err);
        if (st != tycho::kOk) { delete m; return finish(st, err); }
        return mesh_from_records(m, out);
    });
}

int tycho_mesh_kuhn_cube(uint32_t n, double jitter, uint64_t seed, double length, tycho_mesh **out)
{
    if (!out || n == 0 || !(jitter >= 0.0 && jitter < 0.25) || !(length > 0.0))
        return finish(TYCHO_ERR_ARG, "kuhn cube: need n >= 1, 0 <= jitter < 0.25, length > 0");
    return guarded([&] {
        auto *m = new tycho_mesh;
        tycho::kuhn_cube(n, jitter, seed, length, m->rec);
        return mesh_from_records(m, out);
    });
}

int tycho_mesh_from_arrays(uint64_t n_cells, uint64_t n_nodes, const uint64_t *cell_nodes,
                           const double *coords, const uint64_t *adj_cell,
                           const uint64_t *face_to_cell, const uint64_t *cell_gid, tycho_mesh **out)
{
    if (!out || !cell_nodes || !coords || !adj_cell || !face_to_cell || n_cells == 0)
        return finish(TYCHO_ERR_ARG, "null argument");
    return guarded([&] {
        auto *m = new tycho_mesh;
        std::string err;
        int st = tycho::tables_from_arrays(n_cells, n_nodes, cell_nodes, coords, adj_cell,
                                           face_to_cell, cell_gid, m->tab, err);
        if (st != tycho::kOk) { delete m; return finish(st, err); }
        *out = m;
        return (int)TYCHO_OK;
    });
}

int tycho_mesh_write_smesh(const tycho_mesh *m, const char *path)
{
    if (!m || !path) return finish(TYCHO_ERR_ARG, "null argument");
    if (m->rec.n_cells == 0) return finish(TYCHO_ERR_ARG, "mesh has no face records to write");
    std::string err;
    return finish(tycho::write_smesh(path, m->rec, err), err);
}

int tycho_mesh_write_pmesh(const tycho_mesh *m, const char *path)
{
    if (!m || !path) return finish(TYCHO_ERR_ARG, "null argument");
    if (m->rec.n_cells == 0) return finish(TYCHO_ERR_ARG, "mesh has no face records to write");
    std::string err;
    return finish(tycho::write_pmesh(path, m->rec, err), err);
}

int tycho_mesh_info(const tycho_mesh *m, uint64_t *nc, uint64_t *nn, uint64_t *ns)
{
    if (!m) return finish(TYCHO_ERR_ARG, "null mesh");
    if (nc) *nc = m->tab.n_cells;
    if (nn) *nn = m->tab.n_nodes;
    if (ns) *ns = m->tab.n_sides;
    return TYCHO_OK;
}

int tycho_mesh_tables(const tycho_mesh *m, uint64_t *adj_cell, uint64_t *neighbor_vrtx,
                      uint64_t *face_to_cell, uint64_t *cell_to_face, uint64_t *cell_nodes,
                      double *volume, double *area, double *normal, uint64_t *cell_gid,
                      double *coords)
{
    if (!m) return finish(TYCHO_ERR_ARG, "null mesh");
    const auto &t = m->tab;
    auto cp = [](auto *dst, const auto &v) {
        if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(adj_cell, t.adj_cell);
    cp(neighbor_vrtx, t.neighbor_vrtx);
    cp(face_to_cell, t.face_to_cell);
    cp(cell_to_face, t.cell_to_face);
    cp(cell_nodes, t.cell_nodes);
    cp(volume, t.volume);
    cp(area, t.area);
    cp(normal, t.normal);
    cp(cell_gid, t.cell_gid);
    cp(coords, t.coords);
    return TYCHO_OK;
}

void tycho_mesh_free(tycho_mesh *m) { delete m; }

int tycho_mesh_levels(const tycho_mesh *m, int sn, uint32_t *tlevel, uint32_t *deps, uint32_t *blevel,
                      uint32_t *n_levels)
{
    if (!m) return finish(TYCHO_ERR_ARG, "null mesh");
    return guarded([&] {
        tycho::Quadrature q;
        tycho::Schedule s;
        std::string err;
        int st = tycho::make_quadrature(sn, q, err);
        if (st == tycho::kOk) st = tycho::build_schedule(m->tab, q, s, err);
        if (st != tycho::kOk) return finish(st, err);
        if (n_levels) *n_levels = s.n_levels;
        if (tlevel) std::memcpy(tlevel, s.tlevel.data(), s.tlevel.size() * 4);
        if (deps) {
            std::vector<uint32_t> d;
            tycho::dependency_counts(m->tab, q, d);
            std::memcpy(deps, d.data(), d.size() * 4);
        }
        if (blevel) {
            std::vector<uint32_t> b;
            tycho::b_levels(m->tab, q, s, b);
            std::memcpy(blevel, b.data(), b.size() * 4);
        }
        return (int)TYCHO_OK;
    });
}

int tycho_mesh_sweep_schedule_levels(const tycho_mesh *m, int sn, uint32_t *levels, uint32_t *n_levels)
{
    if (!m) return finish(TYCHO_ERR_ARG, "null mesh");
    return guarded([&] {
        tycho::Quadrature q;
        std::string err;
        const int st = tycho::make_quadrature(sn, q, err);
        if (st != tycho::kOk) return finish(st, err);
        std::vector<uint32_t> lev;
        uint32_t top = 0;
        tycho::sweep_schedule_levels(m->tab, q, lev, top);
        if (levels) std::memcpy(levels, lev.data(), lev.size() * 4);
        if (n_levels) *n_levels = top;
        return (int)TYCHO_OK;
    });
}

int tycho_quadrature(int sn, double *xi, double *eta, double *mu, double *wt)
{
    tycho::Quadrature q;
    std::string err;
    if (tycho::make_quadrature(sn, q, err) != tycho::kOk) {
        tycho::set_last_error(err);
        return -1;
    }
    size_t b = sizeof(double) * q.n_angles;
    if (xi) std::memcpy(xi, q.xi.data(), b);
    if (eta) std::memcpy(eta, q.eta.data(), b);
    if (mu) std::memcpy(mu, q.mu.data(), b);
    if (wt) std::memcpy(wt, q.wt.data(), b);
    return q.n_angles;
}

int tycho_sweeper_create(const tycho_mesh *mesh, const tycho_sweeper_opts *opts, tycho_sweeper **out)
{
    return tycho_sweeper_create_angles(mesh, opts, 0, 0, out);
}

int tycho_sweeper_create_angles(const tycho_mesh *mesh, const tycho_sweeper_opts *opts, int angle_begin,
                                int angle_end, tycho_sweeper **out)
{
    if (!mesh || !opts || !out) return finish(TYCHO_ERR_ARG, "null argument");
    return guarded([&] {
        auto *h = new tycho_sweeper;
        tycho::SweeperOptions o;
        o.sn_order = opts->sn_order;
        o.n_groups = opts->n_groups;
        o.device = opts->device;
        o.fp32 = opts->fp32 != 0;
        o.tpi64 = opts->tpi64;
        o.tpi32 = opts->tpi32;
        o.schedule = opts->schedule;
        o.levelling = opts->levelling;
        if (o.schedule < 0 || o.schedule > 2) {
            delete h;
            return finish(TYCHO_ERR_ARG, "schedule must be 0, 1 or 2");
        }
        std::string err;
        if (opts->gauss_elim < TYCHO_GAUSS_ORIGINAL || opts->gauss_elim > TYCHO_GAUSS_CRAMER_INTEL) {
            delete h;
            return finish(TYCHO_ERR_ARG, "GaussElim must be Original, NoPivot, CramerGlu or CramerIntel");
        }
        o.gauss_elim = opts->gauss_elim;
        o.angle_begin = angle_begin;
        o.angle_end = angle_end;
        int st = h->sw.init(mesh->tabp, o, err);
        if (st != tycho::kOk) { delete h; return finish(st, err); }
        *out = h;
        return (int)TYCHO_OK;
    });
}

void tycho_sweeper_destroy(tycho_sweeper *h) { delete h; }

int tycho_sweeper_set_cross_sections(tycho_sweeper *h, const double *sigma_t, const double *sigma_s,
                                     const double *scatter)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    std::string err;
    return finish(h->sw.set_cross_sections(sigma_t, sigma_s, scatter, err), err);
}

int tycho_sweeper_set_source(tycho_sweeper *h, int kind, const double *q)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    std::string err;
    return finish(h->sw.set_source(kind, q, err), err);
}

int tycho_sweeper_sweep(tycho_sweeper *h, const double *source, double *psi)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    std::string err;
    return guarded([&] { return finish(h->sw.sweep_host(source, psi, err), err); });
}

int tycho_sweeper_solve(tycho_sweeper *h, const tycho_solve_opts *opts, double *phi_out,
                        double *psi_out, tycho_solve_stats *stats)
{
    if (!h || !opts) return finish(TYCHO_ERR_ARG, "null argument");
    return guarded([&] {
        tycho::SolveOptions o;
        o.method = opts->method;
        o.iter_max = opts->iter_max;
        o.err_max = opts->err_max;
        o.restart = opts->restart > 0 ? opts->restart : 20;
        o.inner_tol = opts->inner_tol > 0 ? opts->inner_tol : 1e-5;
        o.refine_max = opts->refine_max > 0 ? opts->refine_max : 10;
        tycho::SolveStats st;
        std::string err;
        int s = h->sw.solve(o, phi_out, psi_out, st, err);
        if (stats) {
            stats->iterations = st.iterations;
            stats->sweeps_fp64 = st.sweeps_fp64;
            stats->sweeps_fp32 = st.sweeps_fp32;
            stats->refinements = st.refinements;
            stats->final_error = st.final_error;
            stats->seconds = st.seconds;
        }
        return finish(s, err);
    });
}

int tycho_sweeper_read_psi(tycho_sweeper *h, double *psi)
{
    if (!h || !psi) return finish(TYCHO_ERR_ARG, "null argument");
    std::string err;
    return guarded([&] { return finish(h->sw.read_psi(psi, err), err); });
}

int tycho_sweeper_write_psi(tycho_sweeper *h, const char *path)
{
    if (!h || !path) return finish(TYCHO_ERR_ARG, "null argument");
    std::string err;
    return guarded([&] { return finish(h->sw.write_psi(path, err), err); });
}

int tycho_sweeper_schedule_info(const tycho_sweeper *h, uint32_t *n_levels, uint64_t *n_items,
                                uint64_t *n_incoming)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    const auto &s = h->sw.schedule();
    if (n_levels) *n_levels = s.n_levels;
    if (n_items) *n_items = s.n_items;
    if (n_incoming) *n_incoming = s.n_incoming_interior;
    return TYCHO_OK;
}

int tycho_sweeper_schedule_arrays(const tycho_sweeper *h, uint64_t *n_padded, uint32_t *items,
                                  uint64_t *octant_offset)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    return guarded([&] {
        const auto &s = items ? h->sw.schedule_host() : h->sw.schedule();
        if (n_padded) *n_padded = s.n_padded;
        if (items) std::memcpy(items, s.items.data(), sizeof(uint32_t) * s.items.size());
        if (octant_offset)
            std::memcpy(octant_offset, s.octant_offset.data(), sizeof(uint64_t) * s.octant_offset.size());
        return (int)TYCHO_OK;
    });
}

int tycho_sweeper_launches(const tycho_sweeper *h, int precision, uint64_t *launches)
{
    if (!h || !launches || (precision != 0 && precision != 1)) return finish(TYCHO_ERR_ARG, "bad argument");
    *launches = h->sw.launches_per_apply(precision);
    return TYCHO_OK;
}

int tycho_sweeper_levels(const tycho_sweeper *h, uint32_t *tlevel, uint32_t *deps, uint32_t *blevel)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    return guarded([&] {
        const auto &sw = h->sw;
        if (tlevel) std::memcpy(tlevel, sw.schedule_host().tlevel.data(), sw.schedule_host().tlevel.size() * 4);
        if (deps) {
            std::vector<uint32_t> d;
            tycho::dependency_counts(sw.tables(), sw.quadrature(), d);
            std::memcpy(deps, d.data(), d.size() * 4);
        }
        if (blevel) {
            std::vector<uint32_t> b;
            tycho::b_levels(sw.tables(), sw.quadrature(), sw.schedule_host(), b);
            std::memcpy(blevel, b.data(), b.size() * 4);
        }
        return (int)TYCHO_OK;
    });
}

int tycho_sweeper_autotune(tycho_sweeper *h, int precision, int reps, tycho_launch_shape *best,
                           double *best_ms)
{
    if (!h || reps < 1 || (precision != 0 && precision != 1))
        return finish(TYCHO_ERR_ARG, "null sweeper, reps < 1 or bad precision");
    std::string err;
    return guarded([&] {
        tycho::LaunchShape sh;
        int s = h->sw.autotune(precision, reps, &sh, best_ms, err);
        if (s == tycho::kOk && best) {
            best->schedule = sh.schedule;
            best->variant = sh.variant;
            best->knob = sh.knob;
            best->vector = sh.vg;
            best->streams = sh.streams;
        }
        return finish(s, err);
    });
}

int tycho_sweeper_configure(tycho_sweeper *h, int precision, const tycho_launch_shape *shape)
{
    if (!h || !shape || (precision != 0 && precision != 1))
        return finish(TYCHO_ERR_ARG, "bad sweeper, precision or shape");
    std::string err;
    return finish(h->sw.configure(precision, shape->schedule, shape->variant, shape->knob, err, shape->vector,
                                  shape->streams ? shape->streams : 1),
                  err);
}

int tycho_sweeper_get_shape(const tycho_sweeper *h, int precision, tycho_launch_shape *shape)
{
    if (!h || !shape || (precision != 0 && precision != 1))
        return finish(TYCHO_ERR_ARG, "bad sweeper, precision or shape");
    const tycho::LaunchShape &sh = h->sw.shape(precision);
    shape->schedule = sh.schedule;
    shape->variant = sh.variant;
    shape->knob = sh.knob;
    shape->vector = sh.vg;
    shape->streams = sh.streams;
    return TYCHO_OK;
}

int tycho_sweeper_sweep_noalloc(tycho_sweeper *h, int precision, const void *iso, void *psi, void *stream)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    std::string err;
    return finish(tycho::sweep_noalloc(h->sw, precision, iso, psi, stream, err), err);
}

int tycho_sweeper_apply(tycho_sweeper *h, int precision, const double *phi_in, int with_fixed, double *phi_out,
                        void *stream)
{
    if (!h || !phi_out) return finish(TYCHO_ERR_ARG, "null argument");
    if (precision != 0 && precision != 1) return finish(TYCHO_ERR_ARG, "precision must be 0 (FP64) or 1 (FP32)");
    std::string err;
    return guarded([&] {
        return finish(h->sw.apply_external(precision, phi_in, with_fixed != 0, phi_out, (cudaStream_t)stream, err),
                      err);
    });
}

int tycho_sweeper_bound_sides(const tycho_sweeper *h, uint64_t *n_bound_sides)
{
    if (!h || !n_bound_sides) return finish(TYCHO_ERR_ARG, "null argument");
    *n_bound_sides = h->sw.n_bound_sides();
    return TYCHO_OK;
}

int tycho_sweeper_set_psi_bound(tycho_sweeper *h, const double *psi_bound)
{
    if (!h || !psi_bound) return finish(TYCHO_ERR_ARG, "null argument");
    std::string err;
    return guarded([&] { return finish(h->sw.set_psi_bound(psi_bound, err), err); });
}

int tycho_sweeper_get_psi_bound(tycho_sweeper *h, double *psi_bound)
{
    if (!h || !psi_bound) return finish(TYCHO_ERR_ARG, "null argument");
    std::string err;
    return guarded([&] { return finish(h->sw.get_psi_bound(psi_bound, err), err); });
}

int tycho_sweeper_side_counts(tycho_sweeper *h, uint64_t partition, uint64_t *n_send, uint64_t *n_recv)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    std::string err;
    return guarded([&] {
        uint64_t a = 0, b = 0;
        int st = h->sw.side_counts(partition, a, b, err);
        if (st == TYCHO_OK) {
            if (n_send) *n_send = a;
            if (n_recv) *n_recv = b;
        }
        return finish(st, err);
    });
}

int tycho_sweeper_side_send_list(tycho_sweeper *h, uint64_t partition, uint64_t *gside, uint32_t *angle)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    std::string err;
    return guarded([&] { return finish(h->sw.side_send_list(partition, gside, angle, err), err); });
}

int tycho_sweeper_side_pack(tycho_sweeper *h, uint64_t partition, double *dst, void *stream)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    std::string err;
    return guarded([&] {
        return finish(h->sw.side_pack(partition, dst, (cudaStream_t)stream, stream == nullptr, err), err);
    });
}

int tycho_sweeper_side_link(tycho_sweeper *h, uint64_t partition, uint64_t n, const uint64_t *gside,
                            const uint32_t *angle)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    std::string err;
    return guarded([&] { return finish(h->sw.side_link(partition, n, gside, angle, err), err); });
}

int tycho_sweeper_side_unpack(tycho_sweeper *h, uint64_t partition, const double *src, void *stream)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    std::string err;
    return guarded([&] {
        return finish(h->sw.side_unpack(partition, src, (cudaStream_t)stream, stream == nullptr, err), err);
    });
}

int tycho_sweeper_psi_change(tycho_sweeper *h, double *diff, double *norm)
{
    if (!h || !diff || !norm) return finish(TYCHO_ERR_ARG, "null argument");
    std::string err;
    return guarded([&] { return finish(h->sw.psi_change(*diff, *norm, err), err); });
}

int tycho_sweeper_set_work_order(tycho_sweeper *h, int order)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    std::string err;
    return guarded([&] { return finish(h->sw.set_work_order(order, err), err); });
}

int tycho_sweeper_set_wait_limit(tycho_sweeper *h, uint32_t polls)
{
    if (!h) return finish(TYCHO_ERR_ARG, "null sweeper");
    h->sw.set_wait_limit(polls);
    return TYCHO_OK;
}

int tycho_sweeper_time_sweeps(tycho_sweeper *h, int precision, int n, int flush_l2, double *ms)
{
    if (!h || !ms) return finish(TYCHO_ERR_ARG, "null argument");
    std::string err;
    return guarded([&] { return finish(h->sw.time_sweeps(precision, n, flush_l2 != 0, ms, err), err); });
}

int tycho_batch_create(int device, int ipw32, int ipw64, tycho_batch **out)
{
    if (!out) return finish(TYCHO_ERR_ARG, "null output");
    *out = nullptr;
    std::string err;
    return guarded([&] {
        auto *b = new tycho_batch();
        int s = b->b.init(device, ipw32, ipw64, err);
        if (s != tycho::kOk) {
            delete b;
            return finish(s, err);
        }
        *out = b;
        return (int)TYCHO_OK;
    });
}

void tycho_batch_destroy(tycho_batch *b) { delete b; }

int tycho_batch_set_persistent(tycho_batch *b, int on)
{
    if (!b) return finish(TYCHO_ERR_ARG, "null batch");
    std::string err;
    return guarded([&] { return finish(b->b.set_persistent(on != 0, err), err); });
}

int tycho_batch_set_wait_limit(tycho_batch *b, uint32_t polls)
{
    if (!b) return finish(TYCHO_ERR_ARG, "null batch");
    b->b.set_wait_limit(polls);
    return TYCHO_OK;
}

int tycho_batch_add(tycho_batch *b, tycho_sweeper *sw, const tycho_batch_opts *o, int *id)
{
    if (!b || !sw || !o || !id) return finish(TYCHO_ERR_ARG, "null argument");
    tycho::BatchOptions bo;
    bo.method = o->method;
    bo.iter_max = o->iter_max;
    bo.err_max = o->err_max;
    bo.inner_tol = o->inner_tol;
    bo.inner_max = o->inner_max;
    bo.refine_max = o->refine_max;
    std::string err;
    return guarded([&] { return finish(b->b.add(&sw->sw, bo, *id, err), err); });
}

int tycho_batch_remove(tycho_batch *b, int id)
{
    if (!b) return finish(TYCHO_ERR_ARG, "null batch");
    std::string err;
    return guarded([&] { return finish(b->b.remove(id, err), err); });
}

int tycho_batch_step(tycho_batch *b, int *n_running)
{
    if (!b || !n_running) return finish(TYCHO_ERR_ARG, "null argument");
    std::string err;
    return guarded([&] { return finish(b->b.step(*n_running, err), err); });
}

int tycho_batch_run(tycho_batch *b)
{
    if (!b) return finish(TYCHO_ERR_ARG, "null batch");
    std::string err;
    return guarded([&] { return finish(b->b.run(err), err); });
}

int tycho_batch_result(tycho_batch *b, int id, double *phi, tycho_solve_stats *stats, int *done)
{
    if (!b) return finish(TYCHO_ERR_ARG, "null batch");
    std::string err;
    return guarded([&] {
        tycho::BatchMemberStats st;
        int s = b->b.result(id, phi, st, err);
        if (s == tycho::kOk) {
            if (stats) {
                stats->iterations = st.iterations;
                stats->sweeps_fp64 = st.sweeps_fp64;
                stats->sweeps_fp32 = st.sweeps_fp32;
                stats->refinements = st.refinements;
                stats->final_error = st.final_error;
                stats->seconds = 0.0;
            }
            if (done) *done = st.done;
        }
        return finish(s, err);
    });
}

int tycho_batch_timing(const tycho_batch *b, double *ms, int *passes, double *updates)
{
    if (!b) return finish(TYCHO_ERR_ARG, "null batch");
    double m[2], u[2];
    int p[2];
    b->b.timing(m, p);
    b->b.updates(u);
    for (int i = 0; i < 2; ++i) {
        if (ms) ms[i] = m[i];
        if (passes) passes[i] = p[i];
        if (updates) updates[i] = u[i];
    }
    return TYCHO_OK;
}

uint64_t tycho_footprint_bytes(uint64_t n_cells, int sn_order, int n_groups, int mixed, int compact)
{
    return tycho::footprint_bytes(n_cells, sn_order, n_groups, mixed != 0, compact != 0);
}

int tycho_host_register(void *p, size_t bytes)
{
    if (!p || !bytes) return finish(TYCHO_ERR_ARG, "null pointer or zero size");
    const cudaError_t e = cudaHostRegister(p, bytes, cudaHostRegisterPortable);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return finish(TYCHO_ERR_CUDA, std::string("page-locking host memory: ") + cudaGetErrorString(e));
    }
    return TYCHO_OK;
}

int tycho_host_unregister(void *p)
{
    if (!p) return finish(TYCHO_ERR_ARG, "null pointer");
    const cudaError_t e = cudaHostUnregister(p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return finish(TYCHO_ERR_CUDA, std::string("unlocking host memory: ") + cudaGetErrorString(e));
    }
    return TYCHO_OK;
}

int tycho_release_cached_memory(int device)
{
    const cudaError_t e = tycho::dev_trim(device);
    if (e != cudaSuccess) return finish(TYCHO_ERR_CUDA, std::string("releasing cached memory: ") + cudaGetErrorString(e));
    return TYCHO_OK;
}

int tycho_device_memory(int device, uint64_t *pool_reserved, uint64_t *pool_used)
{
    const cudaError_t e = tycho::dev_pool_usage(device, pool_reserved, pool_used);
    if (e != cudaSuccess) return finish(TYCHO_ERR_CUDA, std::string("reading the memory pool: ") + cudaGetErrorString(e));
    return TYCHO_OK;
}

int tycho_server_create(const tycho_server_opts *o, tycho_server **out)
{
    if (!o || !out) return finish(TYCHO_ERR_ARG, "null argument");
    *out = nullptr;
    std::string err;
    return guarded([&] {
        tycho::ServerOptions so;
        so.device = o->device;
        so.budget_bytes = o->budget_bytes;
        so.setup_threads = o->setup_threads;
        so.ipw32 = o->ipw32;
        so.ipw64 = o->ipw64;
        so.solve.method = o->solve.method;
        so.solve.iter_max = o->solve.iter_max;
        so.solve.err_max = o->solve.err_max;
        so.solve.inner_tol = o->solve.inner_tol;
        so.solve.inner_max = o->solve.inner_max;
        so.solve.refine_max = o->solve.refine_max;
        if (o->large_items > 0) so.large_items = o->large_items;
        so.large_solo = o->large_batched == 0;
        auto *h = new tycho_server();
        int s = h->s.init(so, err);
        if (s != tycho::kOk) {
            delete h;
            return finish(s, err);
        }
        *out = h;
        return (int)TYCHO_OK;
    });
}

void tycho_server_destroy(tycho_server *s) { delete s; }

int tycho_server_submit(tycho_server *s, const tycho_mesh *mesh, int sn_order, int n_groups,
                        const double *sigma_t, const double *sigma_s, const double *scatter,
                        const double *q_iso, double arrival, double *phi_out, int *id)
{
    if (!s || !mesh || !id) return finish(TYCHO_ERR_ARG, "null argument");
    if (sn_order < 2 || sn_order > 32 || sn_order % 2) return finish(TYCHO_ERR_ARG, "bad SN order");
    std::string err;
    return guarded([&] {
        return finish(s->s.submit(mesh->tabp, sn_order, n_groups, sigma_t, sigma_s, scatter, q_iso, arrival,
                                  phi_out, *id, err),
                      err);
    });
}

int tycho_server_run(tycho_server *s)
{
    if (!s) return finish(TYCHO_ERR_ARG, "null server");
    std::string err;
    return guarded([&] { return finish(s->s.run(err), err); });
}

int tycho_server_request(const tycho_server *s, int id, tycho_request_info *info)
{
    if (!s || !info) return finish(TYCHO_ERR_ARG, "null argument");
    const tycho::Server::Request *r = s->s.request(id);
    if (!r) return finish(TYCHO_ERR_ARG, "no request with that id");
    info->state = r->state;
    info->status = r->status;
    info->arrival = r->arrival;
    info->admitted = r->t_admit;
    info->built = r->t_built;
    info->finished = r->t_done;
    info->footprint = r->footprint;
    info->stats.iterations = r->stats.iterations;
    info->stats.sweeps_fp64 = r->stats.sweeps_fp64;
    info->stats.sweeps_fp32 = r->stats.sweeps_fp32;
    info->stats.refinements = r->stats.refinements;
    info->stats.final_error = r->stats.final_error;
    info->stats.seconds = r->t_done >= 0 ? r->t_done - r->arrival : -1.0;
    return TYCHO_OK;
}

int tycho_server_stats(const tycho_server *s, double *peak_bytes, int *peak_active, int *steps, double *makespan)
{
    if (!s) return finish(TYCHO_ERR_ARG, "null server");
    double pb, ms;
    int pa, st;
    s->s.stats(pb, pa, st, ms);
    if (peak_bytes) *peak_bytes = pb;
    if (peak_active) *peak_active = pa;
    if (steps) *steps = st;
    if (makespan) *makespan = ms;
    return TYCHO_OK;
}

}  // extern "C"
