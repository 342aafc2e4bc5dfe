"""ctypes binding of the CPU oracle (tycho_oracle.c).  TEST INFRASTRUCTURE:
imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, as the checker; the product never calls it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libtycho_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        sig = {
            "om_load_pmesh": (P, [C.c_char_p]), "om_load_pmesh_part": (P, [C.c_char_p, C.c_int64]),
            "om_free": (None, [P]), "om_partition": (None, [P] * 5),
            "om_ncells": (C.c_uint64, [P]), "om_nnodes": (C.c_uint64, [P]),
            "om_nsides": (C.c_uint64, [P]), "om_tables": (None, [P] * 11),
            "oq_quadrature": (C.c_int, [C.c_int, P, P, P, P]),
            "oc_create": (P, [P, C.c_int, C.c_int]), "oc_free": (None, [P]),
            "oc_num_angles": (C.c_int, [P]), "oc_cyclic": (C.c_int, [P]),
            "oc_set_gauss_elim": (None, [P, C.c_int]),
            "oc_quadrature": (None, [P] * 5), "oc_omega_dot_n": (None, [P, P]),
            "oc_levels": (None, [P, P, P]), "oc_blevels": (None, [P, P]),
            "oc_sweep": (C.c_int, [P] * 5), "oc_sweep_local": (C.c_int, [P] * 6),
            "oc_psi_to_phi": (None, [P] * 3),
            "oc_scatter": (None, [P] * 5),
            "oc_source_iteration": (C.c_int, [P] * 6 + [C.c_int, C.c_double, P, P, P]),
            "oc_krylov": (C.c_int, [P] * 6 + [C.c_int, C.c_int, C.c_double, P, P, P]),
            "oc_hat_source": (None, [P] * 4), "oc_write_psi": (C.c_int, [P, P, C.c_char_p]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype, f.argtypes = r, a
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


class OracleMesh:
    """One partition of a .pmesh (partition None: the file must hold one)."""

    def __init__(self, path, partition=None):
        self.h = lib().om_load_pmesh_part(str(path).encode(), -1 if partition is None else int(partition))
        if not self.h:
            raise ValueError("oracle could not read %s" % path)
        self.n_cells = lib().om_ncells(self.h)
        self.n_sides = lib().om_nsides(self.h)
        part, nparts = C.c_uint64(), C.c_uint64()
        lib().om_partition(self.h, C.byref(part), C.byref(nparts), None, None)
        self.partition, self.n_partitions = part.value, nparts.value

    def partition_tables(self):
        """adj_rank (c,4): the partition across each face (UINT64_MAX on the
        mesh boundary); side_gid (n_sides): each side's global face id."""
        ar = np.empty((self.n_cells, 4), np.uint64)
        sg = np.empty(max(self.n_sides, 1), np.uint64)
        lib().om_partition(self.h, None, None, _p(ar), _p(sg))
        return ar, sg[:self.n_sides]

    def tables(self):
        n = self.n_cells
        t = dict(adj_cell=np.empty((n, 4), np.uint64), neighbor_vrtx=np.empty((n, 4, 3), np.uint64),
                 face_to_cell=np.empty((n, 4, 3), np.uint64), cell_to_face=np.empty((n, 4, 4), np.uint64),
                 cell_nodes=np.empty((n, 4), np.uint64), volume=np.empty(n), area=np.empty((n, 4)),
                 normal=np.empty((n, 4, 3)), side=np.empty((n, 4), np.uint64),
                 cell_gid=np.empty(n, np.uint64))
        lib().om_tables(self.h, *(_p(t[k]) for k in ("adj_cell", "neighbor_vrtx", "face_to_cell",
                                                     "cell_to_face", "cell_nodes", "volume", "area",
                                                     "normal", "side", "cell_gid")))
        return t

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.om_free(self.h)
            self.h = None


class Oracle:
    """The reference's sweep path on the CPU for one mesh, quadrature, G."""

    def __init__(self, mesh, sn, groups, gauss_elim="NoPivot"):
        self.mesh = mesh
        self.h = lib().oc_create(mesh.h, sn, groups)
        if not self.h:
            raise ValueError("bad quadrature order")
        self.A = lib().oc_num_angles(self.h)
        self.G = groups
        self.nc = mesh.n_cells
        lib().oc_set_gauss_elim(self.h, {"Original": 0, "NoPivot": 1, "CramerGlu": 2,
                                         "CramerIntel": 3}[gauss_elim])
        if lib().oc_cyclic(self.h):
            raise ValueError("cyclic sweep graph")

    @property
    def psi_shape(self):
        return (self.nc, self.A, 4, self.G)

    @property
    def phi_shape(self):
        return (self.nc, 4, self.G)

    def quadrature(self):
        q = [np.empty(self.A) for _ in range(4)]
        lib().oc_quadrature(self.h, *(_p(x) for x in q))
        return q

    def omega_dot_n(self):
        out = np.empty((4, self.nc, self.A))
        lib().oc_omega_dot_n(self.h, _p(out))
        return out

    def levels(self):
        t = np.empty((self.A, self.nc), np.uint32)
        d = np.empty((self.A, self.nc), np.uint32)
        b = np.empty((self.A, self.nc), np.uint32)
        lib().oc_levels(self.h, _p(t), _p(d))
        lib().oc_blevels(self.h, _p(b))
        return t, d, b

    def sweep(self, sigma_t, src_ang=None, src_iso=None):
        psi = np.zeros(self.psi_shape)
        st = np.ascontiguousarray(sigma_t, np.float64)
        r = lib().oc_sweep(self.h, _p(src_ang), _p(src_iso), _p(st), _p(psi))
        assert r == 0
        return psi

    def sweep_local(self, sigma_t, psi_bound, src_ang=None, src_iso=None):
        """Util::sweepLocal of this partition: psi_bound in PsiBoundData
        layout (n_sides, A, 3, G), read on faces whose neighbour is another
        partition."""
        psi = np.zeros(self.psi_shape)
        st = np.ascontiguousarray(sigma_t, np.float64)
        pb = np.ascontiguousarray(psi_bound, np.float64)
        assert pb.size == self.mesh.n_sides * self.A * 3 * self.G
        r = lib().oc_sweep_local(self.h, _p(src_ang), _p(src_iso), _p(st), _p(pb), _p(psi))
        assert r == 0
        return psi

    def psi_to_phi(self, psi):
        phi = np.empty(self.phi_shape)
        lib().oc_psi_to_phi(self.h, _p(psi), _p(phi))
        return phi

    def scatter(self, sigma_s, scatter, phi):
        iso = np.empty(self.phi_shape)
        lib().oc_scatter(self.h, _p(np.ascontiguousarray(sigma_s, np.float64)),
                         _p(None if scatter is None else np.ascontiguousarray(scatter, np.float64)),
                         _p(phi), _p(iso))
        return iso

    def hat_source(self, sigma_t, sigma_s):
        src = np.empty(self.psi_shape)
        lib().oc_hat_source(self.h, _p(np.ascontiguousarray(sigma_t)), _p(np.ascontiguousarray(sigma_s)), _p(src))
        return src

    def source_iteration(self, sigma_t, sigma_s, scatter=None, q_ang=None, q_iso=None,
                         iter_max=100, err_max=1e-10):
        psi = np.empty(self.psi_shape)
        phi = np.empty(self.phi_shape)
        err = np.zeros(1)
        it = lib().oc_source_iteration(
            self.h, _p(np.ascontiguousarray(sigma_t, np.float64)),
            _p(np.ascontiguousarray(sigma_s, np.float64)),
            _p(None if scatter is None else np.ascontiguousarray(scatter, np.float64)),
            _p(q_ang), _p(q_iso), iter_max, err_max, _p(psi), _p(phi), _p(err))
        return psi, phi, it, float(err[0])

    def krylov(self, sigma_t, sigma_s, scatter=None, q_ang=None, q_iso=None, restart=20,
               iter_max=200, rtol=1e-10):
        psi = np.empty(self.psi_shape)
        phi = np.empty(self.phi_shape)
        rn = np.zeros(1)
        it = lib().oc_krylov(
            self.h, _p(np.ascontiguousarray(sigma_t, np.float64)),
            _p(np.ascontiguousarray(sigma_s, np.float64)),
            _p(None if scatter is None else np.ascontiguousarray(scatter, np.float64)),
            _p(q_ang), _p(q_iso), restart, iter_max, rtol, _p(psi), _p(phi), _p(rn))
        return psi, self.psi_to_phi(psi), it, float(rn[0])

    def write_psi(self, psi, path):
        return lib().oc_write_psi(self.h, _p(psi), str(path).encode())

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.oc_free(self.h)
            self.h = None
