"""Host side of the product (C++ ingest behind the C ABI, no GPU needed):
mesh files, TychoMesh tables, quadrature and the wavefront levelling, checked
bit for bit against the reference's fixture and the oracle, plus the error
behaviour of the ingest."""
import hashlib
import os
import struct

import numpy as np
import pytest

from conftest import bits_equal


def test_pmesh_bytes_match_partition_columns(built, workdir, kuhn3_ref):
    import tycho2_b200 as ty
    mesh = ty.TychoMesh.kuhn_cube(3, 0.05, 2024, 100.0)
    path = os.path.join(str(workdir), "k3_product.pmesh")
    mesh.write_pmesh(path)
    digest = hashlib.sha256(open(path, "rb").read()).digest()
    assert digest == kuhn3_ref["pmesh_sha256"].tobytes()


def test_tables_match_reference(built, kuhn3_ref):
    import tycho2_b200 as ty
    t = ty.TychoMesh.kuhn_cube(3, 0.05, 2024, 100.0).tables()
    r = kuhn3_ref
    assert np.array_equal(t["adj_cell"].ravel(), r["s4_adj"])
    assert np.array_equal(t["neighbor_vrtx"].ravel(), r["s4_nbr"])
    assert np.array_equal(t["face_to_cell"].ravel(), r["s4_f2c"])
    assert np.array_equal(t["cell_to_face"].ravel(), r["s4_c2f"])
    assert bits_equal(t["volume"], r["s4_vol"])
    assert bits_equal(t["area"].ravel(), r["s4_area"])


@pytest.mark.parametrize("sn", [4, 8])
def test_levels_match_reference(built, kuhn3_ref, sn):
    import tycho2_b200 as ty
    mesh = ty.TychoMesh.kuhn_cube(3, 0.05, 2024, 100.0)
    tl, deps, blev, nl = mesh.levels(sn)
    assert np.array_equal(deps.ravel().astype(np.uint64), kuhn3_ref["s%d_deps" % sn])
    assert np.array_equal(blev.ravel().astype(np.uint64), kuhn3_ref["s%d_blev" % sn])
    assert nl == tl.max() + 1


@pytest.mark.parametrize("n,jitter,sn", [(4, 0.0, 4), (5, 0.05, 8), (3, 0.05, 2), (4, 0.03, 6)])
def test_tables_and_levels_match_oracle(built, workdir, n, jitter, sn):
    from helpers import kuhn
    from oracle.oracle import Oracle
    mesh, om = kuhn(workdir, n, jitter, seed=11)
    t, ot = mesh.tables(), om.tables()
    for k in ("adj_cell", "neighbor_vrtx", "face_to_cell", "cell_to_face", "cell_nodes", "cell_gid"):
        assert np.array_equal(t[k], ot[k]), k
    for k in ("volume", "area", "normal"):
        assert bits_equal(t[k], ot[k]), k
    o = Oracle(om, sn, 1)
    tl, deps, blev, nl = mesh.levels(sn)
    otl, odeps, oblev = o.levels()
    assert np.array_equal(tl, otl)
    assert np.array_equal(deps, odeps)
    assert np.array_equal(blev, oblev)


def test_mesh_from_reference_getters(built):
    """tycho_mesh_from_arrays (the SweeperCuda adapter's entry) rebuilds the
    same tables from what TychoMesh's getters expose."""
    import tycho2_b200 as ty
    mesh = ty.TychoMesh.kuhn_cube(4, 0.06, 9, 3.0)
    t = mesh.tables()
    m2 = ty.TychoMesh.from_arrays(t["cell_nodes"], t["coords"], t["adj_cell"], t["face_to_cell"],
                                  t["cell_gid"])
    t2 = m2.tables()
    for k in t:
        assert bits_equal(t[k], t2[k]) if t[k].dtype == np.float64 else np.array_equal(t[k], t2[k]), k
    assert m2.n_sides == mesh.n_sides
    assert np.array_equal(m2.levels(8)[0], mesh.levels(8)[0])
    with pytest.raises(ty.TychoError):
        m2.write_pmesh("/nonexistent/never_written.pmesh")
    bad = t["face_to_cell"].copy()
    bad[0, 0, 0] = 0  # face 0 cannot contain vertex 0
    with pytest.raises(ty.TychoError):
        ty.TychoMesh.from_arrays(t["cell_nodes"], t["coords"], t["adj_cell"], bad)


def test_s6_ties_are_not_dependencies(built):
    """S6 has a 45-degree azimuth, so xi == eta and faces of normal (1,-1,0)/sqrt2
    between unjittered nodes have omega.n == 0 exactly.  The reference counts
    such a face as incoming on both sides (its traversal would never finish);
    the wavefront schedule orders on flux-carrying faces only."""
    import tycho2_b200 as ty
    mesh = ty.TychoMesh.kuhn_cube(4, 0.0, 0, 1.0)
    tl, deps, blev, nl = mesh.levels(6)
    q = ty.Quadrature(6)
    t = mesh.tables()
    odn = np.einsum("cfk,ka->acf", t["normal"], np.stack([q.xi, q.eta, q.mu]))
    ties = (odn == 0) & (t["adj_cell"][None] != np.uint64(2**64 - 1))
    assert ties.any()
    # deps follow the reference's rule (ties count as incoming)
    interior = t["adj_cell"][None] != np.uint64(2**64 - 1)
    assert np.array_equal(deps, (~(odn > 0) & interior).sum(axis=2))
    # levels respect every flux-carrying dependency
    up = (odn < 0) & interior
    a_idx, c_idx, f_idx = np.nonzero(up)
    nb = t["adj_cell"][c_idx, f_idx].astype(np.int64)
    assert np.all(tl[a_idx, c_idx] > tl[a_idx, nb])


def test_quadrature_matches_oracle(built):
    import tycho2_b200 as ty
    from oracle.oracle import lib, _p
    for sn in range(2, 31, 2):
        q = ty.Quadrature(sn)
        ref = [np.empty(2 * sn * sn) for _ in range(4)]
        assert lib().oq_quadrature(sn, *(_p(x) for x in ref)) == 2 * sn * sn
        for mine, theirs in zip((q.xi, q.eta, q.mu, q.wt), ref):
            assert bits_equal(mine, theirs)
        assert abs(q.wt.sum() - 4 * np.pi) < 1e-12
    with pytest.raises(ty.TychoError):
        ty.Quadrature(5)


@pytest.mark.parametrize("n", [1, 2, 5])
def test_kuhn_cube_is_a_valid_mesh(built, n):
    import tycho2_b200 as ty
    mesh = ty.TychoMesh.kuhn_cube(n, 0.08, 3, 2.0)
    t = mesh.tables()
    assert mesh.n_cells == 6 * n ** 3
    assert mesh.n_sides == 12 * n * n  # two triangles per boundary square
    assert abs(t["volume"].sum() - 8.0) < 1e-12
    adj = t["adj_cell"].astype(np.int64)
    inner = t["adj_cell"] != np.uint64(2**64 - 1)
    c, f = np.nonzero(inner)
    # adjacency is symmetric and opposite normals are exact negatives
    back = (adj[adj[c, f]] == c[:, None])
    assert np.all(back.sum(axis=1) == 1)
    fb = np.argmax(back, axis=1)
    assert bits_equal(t["normal"][c, f], -t["normal"][adj[c, f], fb])
    # closed cells: sum of area-weighted outward normals vanishes
    s = (t["normal"] * t["area"][..., None]).sum(axis=1)
    assert np.abs(s).max() < 1e-12


def test_ingest_errors(built, workdir):
    import tycho2_b200 as ty
    from tycho2_b200._capi import TychoError
    d = str(workdir)
    with pytest.raises(TychoError) as e:
        ty.TychoMesh.read_pmesh(os.path.join(d, "missing.pmesh"))
    assert e.value.status == 2
    bad = os.path.join(d, "bad.pmesh")
    open(bad, "wb").write(b"not a mesh" * 10)
    with pytest.raises(TychoError) as e:
        ty.TychoMesh.read_pmesh(bad)
    assert e.value.status == 3
    good = os.path.join(d, "k2.pmesh")
    ty.TychoMesh.kuhn_cube(2).write_pmesh(good)
    raw = open(good, "rb").read()
    trunc = os.path.join(d, "trunc.pmesh")
    open(trunc, "wb").write(raw[: len(raw) // 2])
    with pytest.raises(TychoError) as e:
        ty.TychoMesh.read_pmesh(trunc)
    assert e.value.status == 3
    # two partitions: the caller names the one to read
    two = bytearray(raw)
    two[40:48] = struct.pack("<Q", 2)
    p2 = os.path.join(d, "two.pmesh")
    open(p2, "wb").write(bytes(two))
    with pytest.raises(TychoError) as e:
        ty.TychoMesh.read_pmesh(p2)
    assert e.value.status == 1 and "name the partition" in str(e.value)
    with pytest.raises(TychoError):
        ty.TychoMesh.kuhn_cube(0)


def test_zero_volume_cell_is_rejected(built, workdir):
    """A degenerate tet (all four nodes in one plane) is a format error, not a
    division by zero later in the sweep."""
    import tycho2_b200 as ty
    from tycho2_b200._capi import TychoError
    mesh = ty.TychoMesh.kuhn_cube(1)
    path = os.path.join(str(workdir), "flat.smesh")
    mesh.write_smesh(path)
    raw = bytearray(open(path, "rb").read())
    nc, nf, nn = struct.unpack("<QQQ", raw[40:64])
    coords_off = 64 + nc * 9 * 8 + nf * 5 * 8
    xyz = np.frombuffer(bytes(raw[coords_off:]), np.float64).reshape(nn, 3).copy()
    xyz[:, 2] = 0.0  # flatten the cube
    raw[coords_off:] = xyz.tobytes()
    open(path, "wb").write(bytes(raw))
    with pytest.raises(TychoError) as e:
        ty.TychoMesh.read_smesh(path)
    assert e.value.status == 3


def test_face_vertex_numbering_must_round_trip(built):
    """TychoMesh's constructor insists that cellToFaceVrtx and
    faceToCellVrtx invert each other (src/TychoMesh.cc:225-240); a mesh whose
    face 0 lists one vertex twice is rejected."""
    import tycho2_b200 as ty
    m = ty.TychoMesh.kuhn_cube(1, 0.0, 0, 1.0)
    t = m.tables()
    f2c = t["face_to_cell"].copy()
    f2c[0, 0] = [1, 1, 3]  # vertex 2 of face 0 missing
    with pytest.raises(ty.TychoError, match="round-trip"):
        ty.TychoMesh.from_arrays(t["cell_nodes"], t["coords"], t["adj_cell"], f2c)
    ok = ty.TychoMesh.from_arrays(t["cell_nodes"], t["coords"], t["adj_cell"], t["face_to_cell"])
    assert ok.n_cells == m.n_cells
