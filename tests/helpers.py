"""Shared helpers for the parity tests: meshes written once per test session
and loaded by both the product (C++ ingest) and the oracle."""
import os

import numpy as np

from conftest import GOLDEN


def kuhn(workdir, n, jitter=0.05, seed=2024, length=1.0):
    import tycho2_b200 as ty
    from oracle.oracle import OracleMesh
    mesh = ty.TychoMesh.kuhn_cube(n, jitter, seed, length)
    path = os.path.join(str(workdir), "kuhn_%d_%g_%d_%g.pmesh" % (n, jitter, seed, length))
    if not os.path.exists(path):
        mesh.write_pmesh(path)
    return mesh, OracleMesh(path)


def cube208(workdir):
    import tycho2_b200 as ty
    from oracle.oracle import OracleMesh
    mesh = ty.TychoMesh.read_smesh(os.path.join(GOLDEN, "cube-208.smesh"))
    path = os.path.join(str(workdir), "cube-208.pmesh")
    if not os.path.exists(path):
        mesh.write_pmesh(path)
    return mesh, OracleMesh(path)


def gold_psi():
    raw = np.fromfile(os.path.join(GOLDEN, "gold.psi"), np.float64)
    return raw[8:].reshape(208, 128, 4, 2)


def frac_inputs(n, mult, salt):
    """n deterministic values in [0, 1): ((i * mult + salt) mod 1000003) /
    1000003 for i = 0..n-1 (integer arithmetic, one correctly rounded
    division): the same bits on every machine, no generator involved."""
    i = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        k = (i * np.uint64(mult) + np.uint64(salt)) % np.uint64(1000003)
    return k.astype(np.float64) / 1000003.0


def partition_inputs(n_cells, n_angles, n_groups, n_sides, salt):
    """sigma_t, angular source (psi layout) and psiBound (PsiBoundData
    layout) of a partition-local sweep test."""
    st = 0.5 + 2.5 * frac_inputs(n_cells, 7919, salt)
    src = frac_inputs(n_cells * n_angles * 4 * n_groups, 2654435761, salt).reshape(n_cells, n_angles, 4, n_groups)
    pb = 0.2 + frac_inputs(n_sides * n_angles * 3 * n_groups, 40503, salt).reshape(n_sides, n_angles, 3, n_groups)
    return st, src, pb


def psi_hash(psi):
    """64-bit words x_i of an array summed as x_i * (2i + 1) mod 2^64."""
    w = np.ascontiguousarray(psi).reshape(-1).view(np.uint64)
    idx = np.arange(w.size, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return int(np.sum(w * (idx * np.uint64(2) + np.uint64(1)), dtype=np.uint64))


def partitions_fixture(workdir, P):
    """(path of the P-partition Kuhn mesh written from the fixture, fixture)."""
    ref = np.load(os.path.join(GOLDEN, "partitions_ref.npz"))
    path = os.path.join(str(workdir), "kuhn4_p%d.pmesh" % P)
    if not os.path.exists(path):
        ref["p%d_pmesh" % P].tofile(path)
    return path, ref


class OraclePartition:
    """One partition of a PBJ solve on the oracle (host, numpy): the same
    operations as tycho2_b200.partitions.GpuPartition, with CommSides
    restated from src/CommSides.cc:48-240 (packets to q: every (cell, face
    toward q, direction) with omega.n > 0, in that order, psi at the face's
    vertices in face-vertex order; received packets go to psiBound(g, fv,
    angle, the side with that global id))."""

    def __init__(self, path, p, sn, G, sigma_t, sigma_s, scatter, q_iso):
        import torch
        from oracle.oracle import Oracle, OracleMesh
        self.om = OracleMesh(path, p)
        self.o = Oracle(self.om, sn, G)
        self.partition, self.n_groups = p, G
        t = self.om.tables()
        self.t = t
        gid = t["cell_gid"].astype(np.int64)
        self.gid = gid
        self.st = np.ascontiguousarray(sigma_t[gid])
        self.ss = np.ascontiguousarray(sigma_s[gid])
        self.mat = scatter
        self.q = np.ascontiguousarray(q_iso[gid])
        self.rank, self.side_gid = self.om.partition_tables()
        none = np.uint64(0xFFFFFFFFFFFFFFFF)
        bound = (t["adj_cell"] == none) & (self.rank != none) & (self.rank != np.uint64(p))
        self.neighbours = sorted(int(r) for r in np.unique(self.rank[bound]))
        self.odn = self.o.omega_dot_n()  # (f, c, a)
        self.pb = np.zeros((self.om.n_sides, self.o.A, 3, G))
        self.psi = np.zeros(self.o.psi_shape)
        self.prev = np.zeros(self.o.psi_shape)
        self.recv = {}
        self.torch = torch

    def send_entries(self, q):
        ent = []
        for c in range(self.om.n_cells):
            for f in range(4):
                if self.t["adj_cell"][c, f] != np.uint64(0xFFFFFFFFFFFFFFFF) or int(self.rank[c, f]) != q:
                    continue
                for a in range(self.o.A):
                    if self.odn[f, c, a] > 0:
                        ent.append((c, f, a))
        return ent

    def send_list(self, q):
        ent = self.send_entries(q)
        gs = np.array([self.side_gid[self.t["side"][c, f]] for c, f, _ in ent], np.uint64)
        an = np.array([a for _, _, a in ent], np.uint32)
        return gs, an

    def link(self, q, gside, angle):
        gl = {int(self.side_gid[s]): s for s in range(self.om.n_sides)}
        self.recv[q] = [(gl[int(g)], int(a)) for g, a in zip(gside, angle)]

    def pack(self, q):
        ent = self.send_entries(q)
        out = np.empty((len(ent), 3, self.n_groups))
        for k, (c, f, a) in enumerate(ent):
            for v in range(3):
                out[k, v] = self.psi[c, a, int(self.t["face_to_cell"][c, f, v])]
        return self.torch.from_numpy(out.reshape(-1))

    def unpack(self, q, data):
        d = data.numpy().reshape(-1, 3, self.n_groups)
        for k, (s, a) in enumerate(self.recv[q]):
            self.pb[s, a] = d[k]

    def phi_zeros(self):
        return self.torch.zeros(self.o.phi_shape, dtype=self.torch.float64)

    def apply(self, phi_in, phi_out, with_fixed):
        phi = np.ascontiguousarray(phi_in.numpy()) if phi_in is not None else np.zeros(self.o.phi_shape)
        iso = self.o.scatter(self.ss, self.mat, phi)
        if with_fixed:
            iso = self.q + iso
        self.psi = self.o.sweep_local(self.st, self.pb, src_iso=np.ascontiguousarray(iso))
        phi_out.copy_(self.torch.from_numpy(self.o.psi_to_phi(self.psi)))

    def psi_change(self):
        d = float(np.abs(self.psi - self.prev).sum())
        n = float(np.abs(self.psi).sum())
        self.prev = self.psi.copy()
        return d, n

    def get_bound(self):
        return self.pb.copy()

    def set_bound(self, pb):
        self.pb = np.ascontiguousarray(pb, np.float64).reshape(self.pb.shape).copy()
