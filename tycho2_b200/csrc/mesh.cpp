// Host mesh ingest: .smesh/.pmesh I/O, Kuhn-cube generator and the TychoMesh
// tables (reference: src/SerialMesh.cc, src/ParallelMesh.cc,
// src/TychoMeshIO.cc:153-333, src/TychoMesh.cc:67-260).
#include "mesh.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <unordered_map>

#include "rng.hpp"
#include "status.hpp"

namespace tycho {

namespace {

const char kSerialName[32] = "Tycho 2 Serial Mesh";
const char kParallelName[32] = "Tycho 2 Parallel Mesh";

struct File {
    FILE *fp = nullptr;
    explicit File(const std::string &p, const char *mode) { fp = std::fopen(p.c_str(), mode); }
    ~File() { if (fp) std::fclose(fp); }
};

bool rd(FILE *fp, void *dst, size_t bytes) { return std::fread(dst, 1, bytes, fp) == bytes; }
bool wr(FILE *fp, const void *src, size_t bytes) { return std::fwrite(src, 1, bytes, fp) == bytes; }

// Face k of a cell is opposite cell vertex k (src/TychoMeshIO.cc:128-145).
uint64_t lface_index(const uint64_t *cn, const uint64_t *fn)
{
    for (uint64_t v = 0; v < 4; ++v)
        if (cn[v] != fn[0] && cn[v] != fn[1] && cn[v] != fn[2]) return v;
    return kNone;
}

}  // namespace

int read_smesh(const std::string &path, MeshRecords &m, std::string &err)
{
    File f(path, "rb");
    if (!f.fp) { err = "cannot open " + path; return kErrIO; }
    char name[32];
    uint64_t hdr[4];
    if (!rd(f.fp, name, 32) || std::memcmp(name, kSerialName, 32) != 0) {
        err = path + ": not a Tycho 2 serial mesh"; return kErrFormat;
    }
    if (!rd(f.fp, hdr, sizeof hdr) || hdr[0] != 2) { err = path + ": bad header"; return kErrFormat; }
    m = MeshRecords();
    m.n_cells = hdr[1]; m.n_faces = hdr[2]; m.n_nodes = hdr[3];
    std::vector<uint64_t> cb(m.n_cells * 9), fb(m.n_faces * 5);
    m.coords.resize(m.n_nodes * 3);
    if (!rd(f.fp, cb.data(), cb.size() * 8) || !rd(f.fp, fb.data(), fb.size() * 8) ||
        !rd(f.fp, m.coords.data(), m.coords.size() * 8)) {
        err = path + ": truncated"; return kErrFormat;
    }
    m.cell_faces.resize(m.n_cells * 4); m.cell_nodes.resize(m.n_cells * 4);
    m.cell_material.resize(m.n_cells); m.cell_gid.resize(m.n_cells);
    for (uint64_t c = 0; c < m.n_cells; ++c) {
        for (int k = 0; k < 4; ++k) {
            m.cell_faces[c * 4 + k] = cb[c * 9 + k];
            m.cell_nodes[c * 4 + k] = cb[c * 9 + 4 + k];
        }
        m.cell_material[c] = cb[c * 9 + 8];
        m.cell_gid[c] = c;
    }
    m.face_cells.resize(m.n_faces * 2); m.face_nodes.resize(m.n_faces * 3);
    m.face_btype.assign(m.n_faces, 2);
    for (uint64_t fc = 0; fc < m.n_faces; ++fc) {
        m.face_cells[fc * 2] = fb[fc * 5];
        m.face_cells[fc * 2 + 1] = fb[fc * 5 + 1];
        for (int k = 0; k < 3; ++k) m.face_nodes[fc * 3 + k] = fb[fc * 5 + 2 + k];
    }
    make_single_partition(m);
    return kOk;
}

int write_smesh(const std::string &path, const MeshRecords &m, std::string &err)
{
    File f(path, "wb");
    if (!f.fp) { err = "cannot open " + path; return kErrIO; }
    std::vector<uint64_t> u = {2, m.n_cells, m.n_faces, m.n_nodes};
    u.reserve(4 + m.n_cells * 9 + m.n_faces * 5);
    for (uint64_t c = 0; c < m.n_cells; ++c) {
        for (int k = 0; k < 4; ++k) u.push_back(m.cell_faces[c * 4 + k]);
        for (int k = 0; k < 4; ++k) u.push_back(m.cell_nodes[c * 4 + k]);
        u.push_back(m.cell_material[c]);
    }
    for (uint64_t fc = 0; fc < m.n_faces; ++fc) {
        u.push_back(m.face_cells[fc * 2]);
        u.push_back(m.face_cells[fc * 2 + 1]);
        for (int k = 0; k < 3; ++k) u.push_back(m.face_nodes[fc * 3 + k]);
    }
    if (!wr(f.fp, kSerialName, 32) || !wr(f.fp, u.data(), u.size() * 8) ||
        !wr(f.fp, m.coords.data(), m.coords.size() * 8)) {
        err = "write failed: " + path; return kErrIO;
    }
    return kOk;
}

void make_single_partition(MeshRecords &m)
{
    // One partition keeps every index (src/ParallelMesh.cc:397-562 with a
    // single part maps each ordered set onto itself).
    m.cell_gid.resize(m.n_cells);
    for (uint64_t c = 0; c < m.n_cells; ++c) m.cell_gid[c] = c;
    m.face_btype.assign(m.n_faces, 2);
    m.face_gid.resize(m.n_faces);
    m.face_part.assign(m.n_faces * 2, 0);
    for (uint64_t fc = 0; fc < m.n_faces; ++fc) {
        m.face_gid[fc] = fc;
        if (m.face_cells[fc * 2] == kNone || m.face_cells[fc * 2 + 1] == kNone) {
            m.face_btype[fc] = 0;
            m.face_part[fc * 2 + (m.face_cells[fc * 2] == kNone ? 0 : 1)] = kNone;
        }
    }
    m.partition = 0;
    m.n_partitions = 1;
}

int read_pmesh(const std::string &path, MeshRecords &m, std::string &err, int64_t partition)
{
    File f(path, "rb");
    if (!f.fp) { err = "cannot open " + path; return kErrIO; }
    char name[32];
    uint64_t vp[2];
    if (!rd(f.fp, name, 32) || std::memcmp(name, kParallelName, 32) != 0) {
        err = path + ": not a Tycho 2 parallel mesh"; return kErrFormat;
    }
    if (!rd(f.fp, vp, sizeof vp) || vp[0] != 2) { err = path + ": bad header"; return kErrFormat; }
    const uint64_t np = vp[1];
    if (np == 0 || np > (1u << 24)) { err = path + ": bad partition count"; return kErrFormat; }
    if (partition < 0 && np != 1) {
        err = path + ": has " + std::to_string(np) + " partitions; name the partition to read";
        return kErrArg;
    }
    const uint64_t part = partition < 0 ? 0 : (uint64_t)partition;
    if (part >= np) {
        err = path + ": partition " + std::to_string(part) + " of " + std::to_string(np);
        return kErrArg;
    }
    // offsets[np + 1] follow the header; this partition's is offsets[part]
    uint64_t off = 0, cnt[3];
    if (std::fseek(f.fp, (long)(32 + (2 + part) * 8), SEEK_SET) != 0 || !rd(f.fp, &off, sizeof off) ||
        std::fseek(f.fp, (long)off, SEEK_SET) != 0 || !rd(f.fp, cnt, sizeof cnt)) {
        err = path + ": truncated header"; return kErrFormat;
    }
    m = MeshRecords();
    m.partition = part;
    m.n_partitions = np;
    m.n_cells = cnt[0]; m.n_faces = cnt[1]; m.n_nodes = cnt[2];
    std::vector<uint64_t> cb(m.n_cells * 10), fb(m.n_faces * 9), nb(m.n_nodes * 4);
    if (!rd(f.fp, cb.data(), cb.size() * 8) || !rd(f.fp, fb.data(), fb.size() * 8) ||
        !rd(f.fp, nb.data(), nb.size() * 8)) {
        err = path + ": truncated"; return kErrFormat;
    }
    m.cell_faces.resize(m.n_cells * 4); m.cell_nodes.resize(m.n_cells * 4);
    m.cell_material.resize(m.n_cells); m.cell_gid.resize(m.n_cells);
    for (uint64_t c = 0; c < m.n_cells; ++c) {
        for (int k = 0; k < 4; ++k) {
            m.cell_faces[c * 4 + k] = cb[c * 10 + k];
            m.cell_nodes[c * 4 + k] = cb[c * 10 + 4 + k];
        }
        m.cell_gid[c] = cb[c * 10 + 8];
        m.cell_material[c] = cb[c * 10 + 9];
    }
    m.face_cells.resize(m.n_faces * 2); m.face_nodes.resize(m.n_faces * 3);
    m.face_btype.resize(m.n_faces); m.face_gid.resize(m.n_faces); m.face_part.resize(m.n_faces * 2);
    for (uint64_t fc = 0; fc < m.n_faces; ++fc) {
        m.face_cells[fc * 2] = fb[fc * 9];
        m.face_cells[fc * 2 + 1] = fb[fc * 9 + 1];
        for (int k = 0; k < 3; ++k) m.face_nodes[fc * 3 + k] = fb[fc * 9 + 2 + k];
        m.face_gid[fc] = fb[fc * 9 + 5];
        m.face_part[fc * 2] = fb[fc * 9 + 6];
        m.face_part[fc * 2 + 1] = fb[fc * 9 + 7];
        m.face_btype[fc] = fb[fc * 9 + 8];
        if (m.face_btype[fc] > 2) { err = path + ": bad boundary type"; return kErrFormat; }
        // every face of a partition's records touches that partition
        // (src/TychoMeshIO.cc:254-256)
        if (m.face_part[fc * 2] != part && m.face_part[fc * 2 + 1] != part) {
            err = path + ": a face of partition " + std::to_string(part) + " does not touch it";
            return kErrFormat;
        }
    }
    m.coords.resize(m.n_nodes * 3);
    for (uint64_t n = 0; n < m.n_nodes; ++n) std::memcpy(&m.coords[n * 3], &nb[n * 4], 24);
    return kOk;
}

int write_pmesh(const std::string &path, const MeshRecords &m, std::string &err)
{
    if (m.n_partitions != 1) {
        err = "one partition of a multi-partition mesh cannot be written as a one-partition .pmesh";
        return kErrArg;
    }
    File f(path, "wb");
    if (!f.fp) { err = "cannot open " + path; return kErrIO; }
    // Header, then partition 0 (src/ParallelMesh.hh:43-81, offsets as in
    // src/ParallelMesh.cc:539-561).
    uint64_t off0 = 32 + (3 + 1) * 8;
    uint64_t size = 3 * 8 + m.n_cells * 80 + m.n_faces * 72 + m.n_nodes * 32;
    std::vector<uint64_t> u = {2, 1, off0, off0 + size, m.n_cells, m.n_faces, m.n_nodes};
    u.reserve(u.size() + m.n_cells * 10 + m.n_faces * 9 + m.n_nodes * 4);
    for (uint64_t c = 0; c < m.n_cells; ++c) {
        for (int k = 0; k < 4; ++k) u.push_back(m.cell_faces[c * 4 + k]);
        for (int k = 0; k < 4; ++k) u.push_back(m.cell_nodes[c * 4 + k]);
        u.push_back(m.cell_gid[c]);
        u.push_back(m.cell_material[c]);
    }
    for (uint64_t fc = 0; fc < m.n_faces; ++fc) {
        uint64_t c0 = m.face_cells[fc * 2], c1 = m.face_cells[fc * 2 + 1];
        u.push_back(c0);
        u.push_back(c1);
        for (int k = 0; k < 3; ++k) u.push_back(m.face_nodes[fc * 3 + k]);
        u.push_back(fc);
        u.push_back(c0 == kNone ? kNone : 0);
        u.push_back(c1 == kNone ? kNone : 0);
        u.push_back(m.face_btype[fc]);
    }
    for (uint64_t n = 0; n < m.n_nodes; ++n) {
        uint64_t xyz[3];
        std::memcpy(xyz, &m.coords[n * 3], 24);
        u.push_back(xyz[0]); u.push_back(xyz[1]); u.push_back(xyz[2]);
        u.push_back(n);
    }
    if (!wr(f.fp, kParallelName, 32) || !wr(f.fp, u.data(), u.size() * 8)) {
        err = "write failed: " + path; return kErrIO;
    }
    return kOk;
}

void kuhn_cube(uint32_t n, double jitter, uint64_t seed, double length, MeshRecords &m)
{
    m = MeshRecords();
    const uint64_t np = n + 1;
    const double h = length / n;
    m.n_nodes = np * np * np;
    m.coords.resize(m.n_nodes * 3);
    Rng rng(seed);
    for (uint64_t k = 0; k < np; ++k)
        for (uint64_t j = 0; j < np; ++j)
            for (uint64_t i = 0; i < np; ++i) {
                uint64_t node = i + np * (j + np * k);
                double p[3] = {i * h, j * h, k * h};
                bool interior = i > 0 && i < n && j > 0 && j < n && k > 0 && k < n;
                for (int d = 0; d < 3; ++d) {
                    double u = rng.uniform();  // drawn for every node: stable streams
                    if (interior && jitter > 0) p[d] += (2.0 * u - 1.0) * jitter * h;
                    m.coords[node * 3 + d] = p[d];
                }
            }
    // Six tets per hex: path (0,0,0) -> +e_p0 -> +e_p1 -> (1,1,1) for each
    // permutation p of the axes (Kuhn / Freudenthal split; conforming).
    static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    m.n_cells = 6ull * n * n * n;
    m.cell_nodes.resize(m.n_cells * 4);
    m.cell_material.assign(m.n_cells, 1);
    for (uint64_t hz = 0; hz < n; ++hz)
        for (uint64_t hy = 0; hy < n; ++hy)
            for (uint64_t hx = 0; hx < n; ++hx) {
                uint64_t hex = hx + n * (hy + n * hz);
                for (int t = 0; t < 6; ++t) {
                    uint64_t ijk[3] = {hx, hy, hz};
                    uint64_t *cn = &m.cell_nodes[(hex * 6 + t) * 4];
                    cn[0] = ijk[0] + np * (ijk[1] + np * ijk[2]);
                    for (int s = 0; s < 3; ++s) {
                        ijk[perms[t][s]] += 1;
                        cn[s + 1] = ijk[0] + np * (ijk[1] + np * ijk[2]);
                    }
                }
            }
    // Unique faces keyed by their sorted node triple.
    std::unordered_map<uint64_t, uint64_t> seen;  // packed key -> face
    seen.reserve(m.n_cells * 3);
    m.cell_faces.resize(m.n_cells * 4);
    const uint64_t nn = m.n_nodes;
    for (uint64_t c = 0; c < m.n_cells; ++c) {
        const uint64_t *cn = &m.cell_nodes[c * 4];
        for (int f = 0; f < 4; ++f) {
            std::array<uint64_t, 3> tri;
            int k = 0;
            for (int v = 0; v < 4; ++v)
                if (v != f) tri[k++] = cn[v];
            std::sort(tri.begin(), tri.end());
            uint64_t key = (tri[0] * nn + tri[1]) * nn + tri[2];
            auto it = seen.find(key);
            if (it == seen.end()) {
                uint64_t face = m.n_faces++;
                seen.emplace(key, face);
                m.face_cells.push_back(c);
                m.face_cells.push_back(kNone);
                m.face_nodes.insert(m.face_nodes.end(), tri.begin(), tri.end());
                m.cell_faces[c * 4 + f] = face;
            } else {
                m.face_cells[it->second * 2 + 1] = c;
                m.cell_faces[c * 4 + f] = it->second;
            }
        }
    }
    make_single_partition(m);
}

namespace {

void cross(const double a[3], const double b[3], double c[3])
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

}  // namespace

int build_tables(const MeshRecords &m, MeshTables &t, std::string &err)
{
    const uint64_t nc = m.n_cells;
    t = MeshTables();
    t.n_cells = nc; t.n_nodes = m.n_nodes;
    t.cell_nodes = m.cell_nodes; t.cell_gid = m.cell_gid; t.cell_material = m.cell_material;
    t.coords = m.coords;
    t.adj_cell.resize(nc * 4); t.adj_face.resize(nc * 4); t.side.resize(nc * 4);
    std::vector<uint64_t> handle(nc * 4);
    for (uint64_t c = 0; c < nc; ++c) {
        const uint64_t *cn = &m.cell_nodes[c * 4];
        for (uint64_t v = 0; v < 4; ++v)
            if (cn[v] >= m.n_nodes) { err = "cell node out of range"; return kErrFormat; }
        for (uint64_t fi = 0; fi < 4; ++fi) {
            uint64_t face = m.cell_faces[c * 4 + fi];
            if (face >= m.n_faces) { err = "cell face out of range"; return kErrFormat; }
            uint64_t lf = lface_index(cn, &m.face_nodes[face * 3]);
            if (lf == kNone) { err = "face does not belong to its cell"; return kErrFormat; }
            handle[c * 4 + lf] = fi;
            if (m.face_btype[face] != 2) {
                t.adj_cell[c * 4 + lf] = kNone;
                t.adj_face[c * 4 + lf] = kNone;
                t.n_sides++;
            } else {
                uint64_t c0 = m.face_cells[face * 2], c1 = m.face_cells[face * 2 + 1];
                uint64_t adj = (c0 == c) ? c1 : c0;
                if (adj >= nc) { err = "interior face with a bad neighbour"; return kErrFormat; }
                t.adj_cell[c * 4 + lf] = adj;
                t.adj_face[c * 4 + lf] = lface_index(&m.cell_nodes[adj * 4], &m.face_nodes[face * 3]);
            }
        }
    }
    uint64_t s = 0;
    for (uint64_t c = 0; c < nc; ++c)
        for (int f = 0; f < 4; ++f) t.side[c * 4 + f] = (t.adj_cell[c * 4 + f] == kNone) ? s++ : kNone;

    // sides in (cell, face) order with their global face ids, and the
    // partition across each face (src/TychoMeshIO.cc:228-262)
    t.partition = m.partition;
    t.n_partitions = m.n_partitions;
    t.side_gid.resize(t.n_sides);
    t.adj_rank.resize(nc * 4);
    for (uint64_t c = 0; c < nc; ++c)
        for (int f = 0; f < 4; ++f) {
            const uint64_t face = m.cell_faces[c * 4 + handle[c * 4 + f]];
            if (t.side[c * 4 + f] != kNone) t.side_gid[t.side[c * 4 + f]] = m.face_gid[face];
            const uint64_t p0 = m.face_part[face * 2], p1 = m.face_part[face * 2 + 1];
            t.adj_rank[c * 4 + f] = p0 == m.partition ? p1 : p0;
            if (m.face_btype[face] == 1 && (t.adj_rank[c * 4 + f] == kNone ||
                                            t.adj_rank[c * 4 + f] >= m.n_partitions)) {
                err = "partition boundary face without a valid neighbouring partition";
                return kErrFormat;
            }
        }

    // The face-vertex index of a node is its slot in the face record
    // (src/TychoMeshIO.cc:273-296).
    t.face_to_cell.resize(nc * 12);
    t.cell_to_face.assign(nc * 16, kNone);
    for (uint64_t c = 0; c < nc; ++c)
        for (int f = 0; f < 4; ++f) {
            const uint64_t face = m.cell_faces[c * 4 + handle[c * 4 + f]];
            for (int k = 0; k < 3; ++k)
                for (int v = 0; v < 4; ++v)
                    if (m.face_nodes[face * 3 + k] == m.cell_nodes[c * 4 + v]) {
                        t.face_to_cell[(c * 4 + f) * 3 + k] = v;
                        t.cell_to_face[(c * 4 + f) * 4 + v] = k;
                    }
        }

    return finish_tables(t, err);
}

int finish_tables(MeshTables &t, std::string &err)
{
    const uint64_t nc = t.n_cells;
    // cellToFaceVrtx and faceToCellVrtx invert each other on every face
    // (the reference's check, src/TychoMesh.cc:225-240)
    for (uint64_t c = 0; c < nc; ++c)
        for (int f = 0; f < 4; ++f) {
            for (int cv = 0; cv < 4; ++cv) {
                if (cv == f) continue;
                const uint64_t fv = t.cell_to_face[(c * 4 + f) * 4 + cv];
                if (fv >= 3 || t.face_to_cell[(c * 4 + f) * 3 + fv] != (uint64_t)cv) {
                    err = "face-vertex numbering of cell " + std::to_string(c) + " does not round-trip";
                    return kErrFormat;
                }
            }
            for (int fv = 0; fv < 3; ++fv) {
                const uint64_t cv = t.face_to_cell[(c * 4 + f) * 3 + fv];
                if (cv >= 4 || t.cell_to_face[(c * 4 + f) * 4 + cv] != (uint64_t)fv) {
                    err = "face-vertex numbering of cell " + std::to_string(c) + " does not round-trip";
                    return kErrFormat;
                }
            }
        }
    // Geometry with the reference's operation order (src/TychoMesh.cc:67-187).
    t.volume.resize(nc); t.area.resize(nc * 4); t.normal.resize(nc * 12);
    for (uint64_t c = 0; c < nc; ++c) {
        double cp[4][3];
        for (int v = 0; v < 4; ++v)
            for (int d = 0; d < 3; ++d) cp[v][d] = t.coords[t.cell_nodes[c * 4 + v] * 3 + d];
        {
            double a[3], b[3], cc[3], x[3];
            for (int d = 0; d < 3; ++d) {
                a[d] = cp[1][d] - cp[0][d]; b[d] = cp[2][d] - cp[0][d]; cc[d] = cp[3][d] - cp[0][d];
            }
            cross(a, b, x);
            t.volume[c] = 1.0 / 6.0 * std::fabs(x[0] * cc[0] + x[1] * cc[1] + x[2] * cc[2]);
        }
        for (int f = 0; f < 4; ++f) {
            double fp[3][3];
            for (int k = 0; k < 3; ++k)
                for (int d = 0; d < 3; ++d) fp[k][d] = cp[t.face_to_cell[(c * 4 + f) * 3 + k]][d];
            double a[3], b[3], x[3];
            for (int d = 0; d < 3; ++d) { a[d] = fp[1][d] - fp[0][d]; b[d] = fp[2][d] - fp[0][d]; }
            cross(a, b, x);
            double len = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
            t.area[c * 4 + f] = 0.5 * len;
            double *nrm = &t.normal[(c * 4 + f) * 3];
            nrm[0] = x[0] / len; nrm[1] = x[1] / len; nrm[2] = x[2] / len;
            int vi = 0;
            for (; vi < 4; ++vi) {
                bool eq = false;
                for (int k = 0; k < 3; ++k)
                    if (cp[vi][0] == fp[k][0] && cp[vi][1] == fp[k][1] && cp[vi][2] == fp[k][2]) eq = true;
                if (!eq) break;
            }
            if (vi == 4) { err = "degenerate cell (repeated vertex)"; return kErrFormat; }
            double dot = nrm[0] * (cp[vi][0] - fp[0][0]) + nrm[1] * (cp[vi][1] - fp[0][1]) +
                         nrm[2] * (cp[vi][2] - fp[0][2]);
            if (dot > 0) { nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2]; }
        }
        if (!(t.volume[c] > 0)) { err = "zero-volume cell " + std::to_string(c); return kErrFormat; }
    }

    t.neighbor_vrtx.resize(nc * 12);
    for (uint64_t c = 0; c < nc; ++c)
        for (int f = 0; f < 4; ++f)
            for (int k = 0; k < 3; ++k) {
                uint64_t adj = t.adj_cell[c * 4 + f];
                if (adj == kNone) { t.neighbor_vrtx[(c * 4 + f) * 3 + k] = kNone; continue; }
                uint64_t node = t.cell_nodes[c * 4 + t.face_to_cell[(c * 4 + f) * 3 + k]];
                uint64_t nv = kNone;
                for (uint64_t v = 0; v < 4; ++v)
                    if (t.cell_nodes[adj * 4 + v] == node) { nv = v; break; }
                if (nv == kNone) { err = "neighbour does not share a face node"; return kErrFormat; }
                t.neighbor_vrtx[(c * 4 + f) * 3 + k] = nv;
            }
    return kOk;
}

int tables_from_arrays(uint64_t n_cells, uint64_t n_nodes, const uint64_t *cell_nodes,
                       const double *coords, const uint64_t *adj_cell,
                       const uint64_t *face_to_cell, const uint64_t *cell_gid, MeshTables &t,
                       std::string &err)
{
    t = MeshTables();
    t.n_cells = n_cells;
    t.n_nodes = n_nodes;
    t.cell_nodes.assign(cell_nodes, cell_nodes + n_cells * 4);
    t.coords.assign(coords, coords + n_nodes * 3);
    t.adj_cell.assign(adj_cell, adj_cell + n_cells * 4);
    t.face_to_cell.assign(face_to_cell, face_to_cell + n_cells * 12);
    t.cell_material.assign(n_cells, 1);
    if (cell_gid) t.cell_gid.assign(cell_gid, cell_gid + n_cells);
    else { t.cell_gid.resize(n_cells); for (uint64_t c = 0; c < n_cells; ++c) t.cell_gid[c] = c; }
    t.adj_face.assign(n_cells * 4, kNone);
    t.side.resize(n_cells * 4);
    t.cell_to_face.assign(n_cells * 16, kNone);
    for (uint64_t c = 0; c < n_cells; ++c) {
        for (int v = 0; v < 4; ++v)
            if (t.cell_nodes[c * 4 + v] >= n_nodes) { err = "cell node out of range"; return kErrFormat; }
        for (int f = 0; f < 4; ++f) {
            const uint64_t adj = t.adj_cell[c * 4 + f];
            if (adj != kNone && adj >= n_cells) { err = "neighbour out of range"; return kErrFormat; }
            t.side[c * 4 + f] = adj == kNone ? t.n_sides++ : kNone;
            for (int k = 0; k < 3; ++k) {
                const uint64_t v = t.face_to_cell[(c * 4 + f) * 3 + k];
                if (v > 3 || (int)v == f) { err = "bad face-to-cell vertex"; return kErrFormat; }
                t.cell_to_face[(c * 4 + f) * 4 + v] = k;
            }
        }
    }
    return finish_tables(t, err);
}

}  // namespace tycho
