"""The benchmark workloads written without the product library.  TEST
INFRASTRUCTURE: used by bench.py's reference arm and by tests, so that the
reference's own CPU sweep runs on a mesh and inputs that no product code
produced.

Restates, in numpy, the Kuhn-cube generator of the product (n^3 hexes split
into six tets each around the (0,0,0)-(1,1,1) diagonal, interior nodes
jittered by U(-jitter*h, +jitter*h) per coordinate from a xoshiro256** stream
seeded through splitmix64, one draw per node and coordinate) and writes the
reference's serial mesh format (src/SerialMesh.cc: a 32-byte name, then
u64 version 2, cells, faces, nodes; per cell 4 faces, 4 nodes, material; per
face 2 cells, 3 sorted nodes; then the f64 coordinates).  Faces are numbered
in the order a cell-major, face-minor walk first meets them, face k of a cell
being the one opposite its node k.  The reference's PartitionColumns turns the
file into the .pmesh its TychoMesh reads (src/TychoMeshIO.cc:153-333).

The cross sections and source follow the workload definitions: sigma_t per
cell from numpy's default_rng(seed + 1) (lognormal) or uniform, and q = 1 in
every cell or in the cells whose centroid lies in [1/4, 3/4]^3.
"""
import os
import subprocess

import numpy as np

NONE = np.uint64(0xFFFFFFFFFFFFFFFF)
_M64 = (1 << 64) - 1
SERIAL_NAME = b"Tycho 2 Serial Mesh".ljust(32, b"\0")

# the workloads the reference arm and the parity checks run, defined as the
# product defines them
WORKLOADS = {
    "kuhn8_s4_g1": dict(n=8, jitter=0.0, sn=4, groups=1, sigma="uniform", sigma_t=1.0, ratio=0.5,
                        scatter="within", source="all"),
    "kuhn24_s8_g8": dict(n=24, jitter=0.05, sn=8, groups=8, sigma="lognormal", lognormal_s=0.5, ratio=0.6,
                         scatter="down", source="box"),
    "kuhn32_s8_g8": dict(n=32, jitter=0.05, sn=8, groups=8, sigma="lognormal", lognormal_s=0.5, ratio=0.6,
                         scatter="down", source="box"),
}


def _splitmix(state):
    state = (state + 0x9E3779B97F4A7C15) & _M64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return state, z ^ (z >> 31)


def _rotl(x, k):
    return ((x << k) | (x >> (64 - k))) & _M64


def uniform_stream(seed, count):
    """`count` doubles in [0, 1) (53 high bits of xoshiro256**)."""
    s, st = [0] * 4, seed & _M64
    for i in range(4):
        st, s[i] = _splitmix(st)
    out = np.empty(count)
    for i in range(count):
        r = (_rotl((s[1] * 5) & _M64, 7) * 9) & _M64
        t = (s[1] << 17) & _M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = _rotl(s[3], 45)
        out[i] = (r >> 11) * 2.0 ** -53
    return out


def kuhn_cube(n, jitter=0.0, seed=0, length=1.0):
    """(cell_nodes [nc,4], coords [nn,3], cell_faces [nc,4], face_cells [nf,2],
    face_nodes [nf,3]) of the jittered Kuhn cube."""
    np1 = n + 1
    h = length / n
    k, j, i = np.meshgrid(np.arange(np1), np.arange(np1), np.arange(np1), indexing="ij")
    base = np.stack([i * h, j * h, k * h], axis=-1).reshape(-1, 3)  # node = i + np1*(j + np1*k)
    u = uniform_stream(seed, base.size).reshape(-1, 3)
    interior = ((i > 0) & (i < n) & (j > 0) & (j < n) & (k > 0) & (k < n)).reshape(-1)
    coords = base.copy()
    if jitter > 0:
        coords[interior] = base[interior] + (2.0 * u[interior] - 1.0) * jitter * h
    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    hz, hy, hx = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    hexes = np.stack([hx.ravel(), hy.ravel(), hz.ravel()], axis=1)  # hex = hx + n*(hy + n*hz)
    nodes = np.empty((hexes.shape[0], 6, 4), np.int64)
    for t, p in enumerate(perms):
        ijk = hexes.copy()
        nodes[:, t, 0] = ijk[:, 0] + np1 * (ijk[:, 1] + np1 * ijk[:, 2])
        for s in range(3):
            ijk[:, p[s]] += 1
            nodes[:, t, s + 1] = ijk[:, 0] + np1 * (ijk[:, 1] + np1 * ijk[:, 2])
    cell_nodes = nodes.reshape(-1, 4)
    nc = cell_nodes.shape[0]
    # face f of a cell: its nodes other than node f, sorted
    tri = np.stack([np.delete(cell_nodes, f, axis=1) for f in range(4)], axis=1)  # [nc, 4, 3]
    tri = np.sort(tri, axis=2).reshape(-1, 3)
    nn = np1 ** 3
    key = (tri[:, 0] * nn + tri[:, 1]) * nn + tri[:, 2]
    uniq, first, inv = np.unique(key, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")  # faces in order of first appearance
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    cell_faces = rank[inv].reshape(nc, 4)
    nf = uniq.size
    face_cells = np.full((nf, 2), NONE, np.uint64)
    occ = np.arange(nc * 4)
    face_of = cell_faces.reshape(-1)
    is_first = occ == first[inv]
    face_cells[face_of[is_first], 0] = (occ[is_first] // 4).astype(np.uint64)
    face_cells[face_of[~is_first], 1] = (occ[~is_first] // 4).astype(np.uint64)
    face_nodes = tri[first[order]]
    return cell_nodes, coords, cell_faces, face_cells, face_nodes


def write_smesh(path, mesh):
    cell_nodes, coords, cell_faces, face_cells, face_nodes = mesh
    nc, nf, nn = cell_nodes.shape[0], face_cells.shape[0], coords.shape[0]
    cells = np.concatenate([cell_faces.astype(np.uint64), cell_nodes.astype(np.uint64),
                            np.ones((nc, 1), np.uint64)], axis=1)
    faces = np.concatenate([face_cells, face_nodes.astype(np.uint64)], axis=1)
    with open(path, "wb") as f:
        f.write(SERIAL_NAME)
        np.array([2, nc, nf, nn], np.uint64).tofile(f)
        cells.tofile(f)
        faces.tofile(f)
        np.ascontiguousarray(coords, np.float64).tofile(f)


def workload_inputs(mesh, groups, sigma="uniform", sigma_t=1.0, lognormal_s=0.5, source="all", seed=1234,
                    length=1.0, **_):
    """(sigma_t [nc], q [nc, 4, groups]) of a workload on this mesh."""
    cell_nodes, coords = mesh[0], mesh[1]
    nc = cell_nodes.shape[0]
    rng = np.random.default_rng(seed + 1)
    st = np.full(nc, float(sigma_t)) if sigma == "uniform" else np.exp(rng.normal(0.0, lognormal_s, nc))
    q = np.zeros((nc, 4, groups))
    if source == "all":
        q[:] = 1.0
    else:
        cen = coords[cell_nodes].mean(axis=1) / length
        q[np.all((cen >= 0.25) & (cen <= 0.75), axis=1)] = 1.0
    return st, q


def downscatter_matrix(n_groups, ratio):
    """Lower-triangular g' -> g scattering matrix, row g split equally over
    g' <= g, each row summing to `ratio`."""
    m = np.zeros((n_groups, n_groups))
    for g in range(n_groups):
        m[g, : g + 1] = ratio / (g + 1)
    return m


def make_problem(n, jitter, sn, groups, ratio=0.5, scatter="within", seed=1234, length=1.0, **kw):
    """(mesh arrays, sigma_t, sigma_s, scatter matrix or None, q) of one
    problem: within-group scattering sigma_s = ratio * sigma_t, or the
    downscatter matrix with sigma_s = sigma_t."""
    mesh = kuhn_cube(n, jitter, seed, length)
    st, q = workload_inputs(mesh, groups, seed=seed, length=length, **kw)
    if scatter == "within":
        return mesh, st, ratio * st, None, q
    return mesh, st, st.copy(), downscatter_matrix(groups, ratio), q


def partition(mesh, d, name, partition_columns):
    """Writes `name`.smesh and runs the reference's PartitionColumns (one
    partition) on it; returns the .pmesh path."""
    smesh, pmesh = os.path.join(d, name + ".smesh"), os.path.join(d, name + ".pmesh")
    write_smesh(smesh, mesh)
    r = subprocess.run([partition_columns, "1", "1", smesh, pmesh], capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError("PartitionColumns failed: %s" % r.stderr[-300:])
    return pmesh


def make_workload(name, seed=1234):
    """(mesh arrays, sigma_t, q, definition) of a named workload."""
    w = dict(WORKLOADS[name])
    mesh = kuhn_cube(w["n"], w["jitter"], seed, w.get("length", 1.0))
    st, q = workload_inputs(mesh, seed=seed, **w)
    return mesh, st, q, w
