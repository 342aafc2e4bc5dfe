// Host-side mesh ingest for the B200 sweep.
//
// Reads tycho2's one-partition .pmesh files (format: src/ParallelMesh.hh:43-81
// in the reference) and derives the same per-cell tables that the reference's
// TychoMesh builds (src/TychoMeshIO.cc:153-333, src/TychoMesh.cc:193-260),
// bit for bit.  Also writes .smesh/.pmesh and generates the Kuhn-split cube
// meshes used by the benchmark problems.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace tycho {

constexpr uint64_t kNone = UINT64_MAX;  // boundary marker (TychoMesh::BOUNDARY_FACE)

// Raw mesh records, shared by the .smesh and .pmesh formats.
struct MeshRecords {
    uint64_t n_cells = 0, n_faces = 0, n_nodes = 0;
    std::vector<uint64_t> cell_faces;   // (c,4) bounding faces, file order
    std::vector<uint64_t> cell_nodes;   // (c,4)
    std::vector<uint64_t> cell_material;
    std::vector<uint64_t> cell_gid;     // global id (identity for one partition)
    std::vector<uint64_t> face_cells;   // (f,2), second = kNone on the boundary
    std::vector<uint64_t> face_nodes;   // (f,3)
    std::vector<uint64_t> face_btype;   // 0 mesh boundary, 1 partition boundary, 2 interior
    std::vector<uint64_t> face_gid;     // global face id (identity for one partition)
    std::vector<uint64_t> face_part;    // (f,2) partitions of the two sides, kNone on the mesh boundary
    std::vector<double> coords;         // (node,3)
    uint64_t partition = 0, n_partitions = 1;  // which partition of how many the records hold
};

// The TychoMesh tables the sweep needs, all row-major [cell][face][...].
struct MeshTables {
    uint64_t n_cells = 0, n_nodes = 0, n_sides = 0;
    uint64_t partition = 0, n_partitions = 1;
    std::vector<uint64_t> adj_cell;        // (c,4)    kNone on the boundary
    std::vector<uint64_t> adj_face;        // (c,4)
    std::vector<uint64_t> side;            // (c,4)    kNone when interior
    // (c,4) partition across each face (TychoMesh::getAdjRank): this
    // partition for interior faces, kNone on the mesh boundary; empty for
    // tables made from arrays (one partition, no partition boundary)
    std::vector<uint64_t> adj_rank;
    std::vector<uint64_t> side_gid;        // (n_sides) global face id of each side (getLGSide)
    std::vector<uint64_t> face_to_cell;    // (c,4,3)  faceToCellVrtx
    std::vector<uint64_t> cell_to_face;    // (c,4,4)  cellToFaceVrtx, kNone at [c][f][f]
    std::vector<uint64_t> neighbor_vrtx;   // (c,4,3)
    std::vector<uint64_t> cell_nodes;      // (c,4)
    std::vector<uint64_t> cell_gid;        // c -> global cell id (.psi order)
    std::vector<uint64_t> cell_material;
    std::vector<double> coords;            // (node,3)
    std::vector<double> volume;            // c
    std::vector<double> area;              // (c,4)
    std::vector<double> normal;            // (c,4,3) outward unit normals
};

// Status codes shared with the C ABI (see include/tycho_cuda.h).
int read_smesh(const std::string &path, MeshRecords &out, std::string &err);
int write_smesh(const std::string &path, const MeshRecords &m, std::string &err);
// partition < 0: the file must hold one partition; otherwise the records of
// that partition of a multi-partition file (one MPI rank's view,
// src/ParallelMesh.cc:581-690).
int read_pmesh(const std::string &path, MeshRecords &out, std::string &err, int64_t partition = -1);
int write_pmesh(const std::string &path, const MeshRecords &m, std::string &err);

// Adds the partition-0 fields (global ids, boundary types) that a one-partition
// .pmesh carries, as the reference's PartitionColumns 1 1 would.
void make_single_partition(MeshRecords &m);

// Unit-cube-like mesh: n^3 hexes of side length/n, each split into 6 Kuhn tets
// around its (0,0,0)-(1,1,1) diagonal; interior vertices moved by
// U(-jitter*h, +jitter*h) per coordinate from a seeded generator.
void kuhn_cube(uint32_t n, double jitter, uint64_t seed, double length, MeshRecords &out);

int build_tables(const MeshRecords &m, MeshTables &t, std::string &err);

// Geometry (volumes, areas, outward normals) and neighbour vertices from
// cell_nodes, coords, face_to_cell and adj_cell already in `t`.
int finish_tables(MeshTables &t, std::string &err);

// The tables from what a reference TychoMesh exposes through its getters
// (getCellNode, getNodeCoord, getAdjCell, getFaceToCellVrtx, getLGCell).
int tables_from_arrays(uint64_t n_cells, uint64_t n_nodes, const uint64_t *cell_nodes,
                       const double *coords, const uint64_t *adj_cell,
                       const uint64_t *face_to_cell, const uint64_t *cell_gid, MeshTables &t,
                       std::string &err);

}  // namespace tycho
