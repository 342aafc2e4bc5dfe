"""Host-side mirror of tycho2's sweeper interface over the C ABI.

Names follow the reference so that callers read the same:
  TychoMesh        src/TychoMesh.hh      (tables from .pmesh/.smesh or a Kuhn cube)
  Quadrature       src/Quadrature.hh     (getXi/getEta/getMu/getWt)
  SweeperCuda      src/SweeperAbstract.hh (sweep, solve, getPsi, writePsiToFile)
Every call goes to libtycho_b200.so; errors raise TychoError with the
library's status and message (the reference aborts through Insist).
"""
import ctypes as C

import numpy as np

from . import _capi
from ._capi import check, lib, ptr

NONE = np.uint64(0xFFFFFFFFFFFFFFFF)  # TychoMesh::BOUNDARY_FACE

GAUSS_ELIM = {"Original": 0, "NoPivot": 1, "CramerGlu": 2, "CramerIntel": 3}
METHODS = {"si": 0, "gmres": 1, "mixed": 2}


class TychoMesh:
    """TychoMesh (src/TychoMesh.hh:52-159) built by the C++ host ingest."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)
        nc, nn, ns = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(lib().tycho_mesh_info(self._h, C.byref(nc), C.byref(nn), C.byref(ns)))
        self.n_cells, self.n_nodes, self.n_sides = nc.value, nn.value, ns.value
        p, np_, nb = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(lib().tycho_mesh_partition_info(self._h, C.byref(p), C.byref(np_), C.byref(nb)))
        self.partition, self.n_partitions, self.n_bound_sides = p.value, np_.value, nb.value
        self._tables = None

    @classmethod
    def read_pmesh(cls, path, partition=None):
        """A .pmesh; partition: which partition of a multi-partition file
        (the one MPI rank `partition` reads); None: the file must hold one."""
        h = C.c_void_p()
        if partition is None:
            check(lib().tycho_mesh_read_pmesh(str(path).encode(), C.byref(h)))
        else:
            check(lib().tycho_mesh_read_pmesh_partition(str(path).encode(), int(partition), C.byref(h)))
        return cls(h.value)

    def cell_material(self):
        """TychoMesh::getCellMaterial of every cell."""
        m = np.empty(self.n_cells, np.uint64)
        check(lib().tycho_mesh_cell_material(self._h, ptr(m)))
        return m

    def side_tables(self):
        """(side (c,4), adj_rank (c,4), side_gid (n_sides)): TychoMesh::getSide,
        getAdjRank and getLGSide; UINT64_MAX where the reference has
        NOT_BOUNDARY_FACE / BAD_RANK."""
        side = np.empty((self.n_cells, 4), np.uint64)
        rank = np.empty((self.n_cells, 4), np.uint64)
        gid = np.empty(max(self.n_sides, 1), np.uint64)
        check(lib().tycho_mesh_side_tables(self._h, ptr(side), ptr(rank), ptr(gid)))
        return side, rank, gid[:self.n_sides]

    @classmethod
    def read_smesh(cls, path):
        h = C.c_void_p()
        check(lib().tycho_mesh_read_smesh(str(path).encode(), C.byref(h)))
        return cls(h.value)

    @classmethod
    def kuhn_cube(cls, n, jitter=0.0, seed=0, length=1.0):
        h = C.c_void_p()
        check(lib().tycho_mesh_kuhn_cube(n, jitter, seed, length, C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_arrays(cls, cell_nodes, coords, adj_cell, face_to_cell, cell_gid=None):
        """From the arrays a reference TychoMesh exposes through its getters."""
        cn = np.ascontiguousarray(cell_nodes, np.uint64)
        xyz = np.ascontiguousarray(coords, np.float64)
        adj = np.ascontiguousarray(adj_cell, np.uint64)
        f2c = np.ascontiguousarray(face_to_cell, np.uint64)
        gid = None if cell_gid is None else np.ascontiguousarray(cell_gid, np.uint64)
        h = C.c_void_p()
        check(lib().tycho_mesh_from_arrays(cn.shape[0], xyz.shape[0], ptr(cn), ptr(xyz), ptr(adj),
                                           ptr(f2c), ptr(gid), C.byref(h)))
        return cls(h.value)

    def write_smesh(self, path):
        check(lib().tycho_mesh_write_smesh(self._h, str(path).encode()))

    def write_pmesh(self, path):
        check(lib().tycho_mesh_write_pmesh(self._h, str(path).encode()))

    def tables(self):
        """dict of the TychoMesh tables as numpy arrays, [cell][face][...]."""
        if self._tables is None:
            n, nn = self.n_cells, self.n_nodes
            t = {
                "adj_cell": np.empty((n, 4), np.uint64),
                "neighbor_vrtx": np.empty((n, 4, 3), np.uint64),
                "face_to_cell": np.empty((n, 4, 3), np.uint64),
                "cell_to_face": np.empty((n, 4, 4), np.uint64),
                "cell_nodes": np.empty((n, 4), np.uint64),
                "volume": np.empty(n, np.float64),
                "area": np.empty((n, 4), np.float64),
                "normal": np.empty((n, 4, 3), np.float64),
                "cell_gid": np.empty(n, np.uint64),
                "coords": np.empty((nn, 3), np.float64),
            }
            check(lib().tycho_mesh_tables(
                self._h, *(ptr(t[k]) for k in ("adj_cell", "neighbor_vrtx", "face_to_cell",
                                               "cell_to_face", "cell_nodes", "volume", "area",
                                               "normal", "cell_gid", "coords"))))
            self._tables = t
        return self._tables

    def levels(self, sn_order):
        """(tlevel, deps, blevel) in (angle, cell) order and the level count."""
        A = 2 * sn_order * sn_order
        t = np.empty((A, self.n_cells), np.uint32)
        d = np.empty((A, self.n_cells), np.uint32)
        b = np.empty((A, self.n_cells), np.uint32)
        nl = C.c_uint32()
        check(lib().tycho_mesh_levels(self._h, sn_order, ptr(t), ptr(d), ptr(b), C.byref(nl)))
        return t, d, b, nl.value

    def sweep_schedule_levels(self, sn_order):
        """SweepSchedule's b-levels (calcLevels, +-1e-10 omega.n rule) in
        (angle, cell) order and their maximum."""
        A = 2 * sn_order * sn_order
        lev = np.empty((A, self.n_cells), np.uint32)
        nl = C.c_uint32()
        check(lib().tycho_mesh_sweep_schedule_levels(self._h, sn_order, ptr(lev), C.byref(nl)))
        return lev, nl.value

    def centroids(self):
        t = self.tables()
        return t["coords"][t["cell_nodes"].astype(np.int64)].mean(axis=1)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _capi._lib is not None:
            _capi._lib.tycho_mesh_free(h)
            self._h = None


class Quadrature:
    """Quadrature (src/Quadrature.hh:45-64): 2 N^2 directions."""

    def __init__(self, sn_order):
        A = 2 * sn_order * sn_order
        self.xi, self.eta, self.mu, self.wt = (np.empty(A) for _ in range(4))
        n = lib().tycho_quadrature(sn_order, ptr(self.xi), ptr(self.eta), ptr(self.mu), ptr(self.wt))
        if n != A:
            raise _capi.TychoError(1, "Quadrature order not supported: %d" % sn_order)
        self.sn_order, self.n_angles = sn_order, A

    def getXi(self, a):
        return self.xi[a]

    def getEta(self, a):
        return self.eta[a]

    def getMu(self, a):
        return self.mu[a]

    def getWt(self, a):
        return self.wt[a]


class SweeperCuda:
    """SweeperAbstract (src/SweeperAbstract.hh:47-70) on the B200 sweep.

    sweep(psi, source) fills psi = L^-1 source in place (host arrays in the
    PsiData layout); solve() runs SourceIteration / Krylov / mixed-precision
    refinement on the device and keeps psi resident.
    """

    SCHEDULES = {"auto": 0, "levels": 1, "dataflow": 2, "persist": 3}

    LEVELLING = {"auto": 0, "host": 1, "device": 2}

    def __init__(self, mesh, sn_order, n_groups, gauss_elim="NoPivot", fp32=False, device=0,
                 tpi64=0, tpi32=0, schedule="auto", levelling="auto", angles=None):
        """angles=(begin, end): the directions [begin, end) of the quadrature
        only (an angle shard, tycho_sweeper_create_angles)."""
        if gauss_elim not in GAUSS_ELIM:
            raise ValueError("GaussElim must be one of %s" % sorted(GAUSS_ELIM))
        self.mesh = mesh
        self.n_groups = n_groups
        self.device = device
        self.quadrature = Quadrature(sn_order)
        a0, a1 = angles if angles is not None else (0, self.quadrature.n_angles)
        self.angles = (a0, a1)
        self.n_angles = a1 - a0
        opts = _capi.SweeperOpts(sn_order, n_groups, GAUSS_ELIM[gauss_elim], device, int(fp32),
                                 tpi64, tpi32, self.SCHEDULES[schedule], self.LEVELLING[levelling])
        h = C.c_void_p()
        if angles is None:
            check(lib().tycho_sweeper_create(mesh._h, C.byref(opts), C.byref(h)))
        else:
            check(lib().tycho_sweeper_create_angles(mesh._h, C.byref(opts), int(a0), int(a1), C.byref(h)))
        self._h = h
        self.stats = None

    # sizes of the reference containers
    @property
    def psi_shape(self):
        return (self.mesh.n_cells, self.n_angles, 4, self.n_groups)

    @property
    def phi_shape(self):
        return (self.mesh.n_cells, 4, self.n_groups)

    def set_cross_sections(self, sigma_t, sigma_s, scatter=None):
        st = np.ascontiguousarray(sigma_t, np.float64)
        ss = np.ascontiguousarray(sigma_s, np.float64)
        sc = None if scatter is None else np.ascontiguousarray(scatter, np.float64)
        assert st.shape == (self.mesh.n_cells,) and ss.shape == (self.mesh.n_cells,)
        if sc is not None:
            assert sc.shape == (self.n_groups, self.n_groups)
        check(lib().tycho_sweeper_set_cross_sections(self._h, ptr(st), ptr(ss), ptr(sc)))
        self._xs = (st, ss, sc)

    def set_source(self, q, kind="angular"):
        """Fixed source Q: 'angular' in the psi layout, 'isotropic' in phi's."""
        k = {"angular": 0, "isotropic": 1}[kind]
        if q is None:
            check(lib().tycho_sweeper_set_source(self._h, k, None))
            return
        arr = np.ascontiguousarray(q, np.float64)
        assert arr.size == np.prod(self.psi_shape if k == 0 else self.phi_shape)
        check(lib().tycho_sweeper_set_source(self._h, k, ptr(arr)))

    def sweep(self, psi, source, zeroPsiBound=False):
        """SweeperAbstract::sweep: psi = L^-1 source; vacuum on the mesh
        boundary and, on faces toward other partitions, the psiBound last
        set (zeroPsiBound: zeros instead, for this sweep only, as
        SweeperPBJOuter::sweep takes c_zeroPsiBound, src/SweeperPBJ.cc:129-138)."""
        src = np.ascontiguousarray(source, np.float64)
        assert psi.dtype == np.float64 and psi.flags["C_CONTIGUOUS"] and psi.size == src.size
        keep = self.get_psi_bound() if zeroPsiBound and self.n_bound_sides else None
        if keep is not None:
            self.set_psi_bound(np.zeros_like(keep))
        try:
            check(lib().tycho_sweeper_sweep(self._h, ptr(src), ptr(psi)))
        finally:
            if keep is not None:
                self.set_psi_bound(keep)
        return psi

    def solve(self, method="si", iter_max=100, err_max=1e-10, restart=20, inner_tol=1e-5,
              refine_max=10, want_psi=True):
        """SweeperAbstract::solve; returns (phi, psi or None, stats dict)."""
        o = _capi.SolveOpts(METHODS[method], iter_max, err_max, restart, inner_tol, refine_max)
        phi = np.empty(self.phi_shape)
        psi = np.empty(self.psi_shape) if want_psi else None
        st = _capi.SolveStats()
        status = lib().tycho_sweeper_solve(self._h, C.byref(o), ptr(phi), ptr(psi), C.byref(st))
        self.stats = {k: getattr(st, k) for k, _ in _capi.SolveStats._fields_}
        check(status)
        return phi, psi, self.stats

    def writePsiToFile(self, filename):
        check(lib().tycho_sweeper_write_psi(self._h, str(filename).encode()))

    def schedule_info(self):
        nl, ni, nin = C.c_uint32(), C.c_uint64(), C.c_uint64()
        check(lib().tycho_sweeper_schedule_info(self._h, C.byref(nl), C.byref(ni), C.byref(nin)))
        return {"n_levels": nl.value, "n_items": ni.value, "n_incoming_interior": nin.value}

    def schedule_arrays(self):
        """(items in level/octant order with padding, (level, octant) segment offsets)."""
        n = C.c_uint64()
        check(lib().tycho_sweeper_schedule_arrays(self._h, C.byref(n), None, None))
        items = np.empty(n.value, np.uint32)
        offs = np.empty(self.schedule_info()["n_levels"] * 8 + 1, np.uint64)
        check(lib().tycho_sweeper_schedule_arrays(self._h, None, ptr(items), ptr(offs)))
        return items, offs

    def launches(self, precision):
        """Kernel launches of one operator application with the current shape."""
        n = C.c_uint64()
        check(lib().tycho_sweeper_launches(self._h, precision, C.byref(n)))
        return n.value

    def time_sweeps(self, precision, n, flush_l2=True):
        ms = np.zeros(2)
        check(lib().tycho_sweeper_time_sweeps(self._h, precision, n, int(flush_l2), ptr(ms)))
        return float(ms[0]), float(ms[1])

    VARIANTS = {"items": 0, "tiles": 1, "records": 2, "direct": 3, "compact": 4}

    @staticmethod
    def _shape_dict(sh):
        return {"schedule": {1: "levels", 2: "dataflow", 3: "persist"}[sh.schedule],
                "variant": {0: "items", 1: "tiles", 2: "records", 3: "direct", 4: "compact"}[sh.variant],
                "knob": sh.knob,
                "vector": sh.vector, "streams": sh.streams}

    def autotune(self, precision, reps=3):
        """Picks the fastest launch shape (schedule, variant, knob) for one precision."""
        sh, ms = _capi.LaunchShape(), C.c_double()
        check(lib().tycho_sweeper_autotune(self._h, precision, reps, C.byref(sh), C.byref(ms)))
        d = self._shape_dict(sh)
        d["ms"] = ms.value
        return d

    def configure(self, precision, schedule, variant, knob, vector=0, streams=1):
        """schedule 'levels'|'dataflow'|'persist' (records only); variant 'items' (knob = lanes per item),
        'tiles' (knob = warps per block), 'records' (knob = items per warp) or 'direct' (records
        in registers, level schedule, knob = threads per block); vector = records' groups per
        psi-row access, 0 = widest dividing nGroups; streams: level schedule on 1, 2, 4 or 8 concurrent
        streams (octant groups)."""
        sh = _capi.LaunchShape(self.SCHEDULES[schedule], self.VARIANTS[variant], knob, vector, streams)
        check(lib().tycho_sweeper_configure(self._h, precision, C.byref(sh)))

    def apply(self, phi_in, phi_out, precision=0, with_fixed=True):
        """phi_out = D L^-1 ([Q] + M S phi_in) on device tensors (torch, FP64,
        phi layout; phi_in may be None), ordered after the current torch
        stream's work (tycho_sweeper_apply).  For an angle shard phi_out is
        its directions' part of phi."""
        import torch
        for t in (phi_in, phi_out):
            if t is not None:
                assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
                assert tuple(t.shape) == self.phi_shape or t.numel() == int(np.prod(self.phi_shape))
        stream = torch.cuda.current_stream(phi_out.device)
        check(lib().tycho_sweeper_apply(self._h, int(precision),
                                        C.c_void_p(phi_in.data_ptr()) if phi_in is not None else None,
                                        int(bool(with_fixed)), C.c_void_p(phi_out.data_ptr()),
                                        C.c_void_p(stream.cuda_stream)))

    # ---- one partition of a multi-partition mesh (Util::sweepLocal with
    #      psiBound, CommSides on the device) ------------------------------

    @property
    def n_bound_sides(self):
        """Faces toward other partitions (0: an ordinary sweeper)."""
        n = C.c_uint64()
        check(lib().tycho_sweeper_bound_sides(self._h, C.byref(n)))
        return n.value

    @property
    def psi_bound_shape(self):
        """PsiBoundData (src/PsiData.hh:168-263): (sides, angles, 3, groups)."""
        return (self.mesh.n_sides, self.quadrature.n_angles, 3, self.n_groups)

    def set_psi_bound(self, psi_bound):
        """Incoming psi on faces toward other partitions, PsiBoundData layout
        (host array of psi_bound_shape); every later sweep reads it."""
        pb = np.ascontiguousarray(psi_bound, np.float64)
        assert pb.size == int(np.prod(self.psi_bound_shape))
        check(lib().tycho_sweeper_set_psi_bound(self._h, ptr(pb)))

    def get_psi_bound(self):
        pb = np.empty(self.psi_bound_shape)
        check(lib().tycho_sweeper_get_psi_bound(self._h, ptr(pb)))
        return pb

    def side_counts(self, q):
        """(packets sent to partition q, packets q sends here), as CommSides
        counts them (src/CommSides.cc:68-95)."""
        a, b = C.c_uint64(), C.c_uint64()
        check(lib().tycho_sweeper_side_counts(self._h, int(q), C.byref(a), C.byref(b)))
        return a.value, b.value

    def side_send_list(self, q):
        """(global side id, direction) of each packet sent to partition q."""
        n, _ = self.side_counts(q)
        gs = np.empty(max(n, 1), np.uint64)
        an = np.empty(max(n, 1), np.uint32)
        check(lib().tycho_sweeper_side_send_list(self._h, int(q), ptr(gs), ptr(an)))
        return gs[:n], an[:n]

    def side_link(self, q, gside, angle):
        """q's send list, once: where q's packets land here."""
        gs = np.ascontiguousarray(gside, np.uint64)
        an = np.ascontiguousarray(angle, np.uint32)
        assert gs.shape == an.shape
        check(lib().tycho_sweeper_side_link(self._h, int(q), gs.size, ptr(gs), ptr(an)))

    def side_pack(self, q, dst):
        """Packets to q from the resident psi into dst (torch FP64 device
        tensor of side_counts(q)[0] * 3 * G), on the current torch stream."""
        import torch
        assert dst.is_cuda and dst.dtype == torch.float64 and dst.is_contiguous()
        stream = torch.cuda.current_stream(dst.device)
        check(lib().tycho_sweeper_side_pack(self._h, int(q), C.c_void_p(dst.data_ptr()),
                                            C.c_void_p(stream.cuda_stream)))

    def side_unpack(self, q, src):
        """Packets from q (torch FP64 device tensor, q's send order) into
        psiBound, on the current torch stream."""
        import torch
        assert src.is_cuda and src.dtype == torch.float64 and src.is_contiguous()
        stream = torch.cuda.current_stream(src.device)
        check(lib().tycho_sweeper_side_unpack(self._h, int(q), C.c_void_p(src.data_ptr()),
                                              C.c_void_p(stream.cuda_stream)))

    def read_psi(self):
        """The resident FP64 psi (PsiData layout) on the host."""
        psi = np.empty(self.psi_shape)
        check(lib().tycho_sweeper_read_psi(self._h, ptr(psi)))
        return psi

    def psi_change(self):
        """(L1 of psi - psi_prev, L1 of psi) over the resident FP64 psi, then
        psi_prev = psi (SweeperPBJ's test, src/SweeperPBJ.cc:181-195)."""
        d, n = C.c_double(), C.c_double()
        check(lib().tycho_sweeper_psi_change(self._h, C.byref(d), C.byref(n)))
        return d.value, n.value

    WORK_ORDERS = {"cell": 0, "blevel": 1, "random": 2}

    def set_work_order(self, order):
        """Order of the items within each wavefront segment: 'cell'
        (default), 'blevel' (the reference's b-level priorities, longest
        downwind chain first) or 'random' (seeded); psi is the same."""
        check(lib().tycho_sweeper_set_work_order(self._h, self.WORK_ORDERS[order]))

    def set_wait_limit(self, polls):
        """Polls of one flag or level barrier before a persistent kernel's
        bounded wait gives up (TYCHO_ERR_TIMEOUT); 0 gives up at the first
        wait that is not already satisfied."""
        check(lib().tycho_sweeper_set_wait_limit(self._h, int(polls)))

    def shape(self, precision):
        sh = _capi.LaunchShape()
        check(lib().tycho_sweeper_get_shape(self._h, precision, C.byref(sh)))
        return self._shape_dict(sh)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value and _capi._lib is not None:
            _capi._lib.tycho_sweeper_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()


class BatchSolver:
    """Many independent sweepers solved together on one GPU (tycho_batch_*).

    method "si": FP64 source iteration (the reference's fixed point);
    "mixed": FP32-sweep source iteration on the correction inside FP64
    refinement.  Each member's result is bit-identical alone and in any mix.
    """

    BATCH_METHODS = {"si": 0, "mixed": 2}

    def __init__(self, device=0, ipw32=0, ipw64=0, persistent=False):
        """persistent: each pass's wavefront in one persistent kernel with a
        device work queue over (member, level) instead of one launch per
        level (tycho_batch_set_persistent)."""
        h = C.c_void_p()
        check(lib().tycho_batch_create(device, ipw32, ipw64, C.byref(h)))
        self._h = h
        self._members = {}
        if persistent:
            check(lib().tycho_batch_set_persistent(h, 1))

    def set_wait_limit(self, polls):
        """Polls of the persistent form's grid barrier before a step fails
        with TYCHO_ERR_TIMEOUT."""
        check(lib().tycho_batch_set_wait_limit(self._h, int(polls)))

    def add(self, sweeper, method="mixed", iter_max=1000, err_max=1e-10, inner_tol=1e-5,
            inner_max=200, refine_max=30):
        o = _capi.BatchOpts(self.BATCH_METHODS[method], iter_max, err_max, inner_tol, inner_max,
                            refine_max)
        mid = C.c_int()
        check(lib().tycho_batch_add(self._h, sweeper._h, C.byref(o), C.byref(mid)))
        self._members[mid.value] = sweeper
        return mid.value

    def remove(self, mid):
        check(lib().tycho_batch_remove(self._h, mid))
        self._members.pop(mid, None)

    def step(self):
        n = C.c_int()
        check(lib().tycho_batch_step(self._h, C.byref(n)))
        return n.value

    def run(self):
        check(lib().tycho_batch_run(self._h))

    def result(self, mid, want_phi=True):
        """(phi or None, stats dict, done)."""
        sw = self._members[mid]
        phi = np.empty(sw.phi_shape) if want_phi else None
        st, done = _capi.SolveStats(), C.c_int()
        check(lib().tycho_batch_result(self._h, mid, ptr(phi), C.byref(st), C.byref(done)))
        stats = {k: getattr(st, k) for k, _ in _capi.SolveStats._fields_ if k != "seconds"}
        return phi, stats, bool(done.value)

    # the shapes `autotune` tries: (items per warp, persistent)
    TUNE_SHAPES = ((0, False), (0, True), (16, False), (8, False))

    @classmethod
    def autotune(cls, sweepers, device=0, steps=3, shapes=None):
        """Picks the batch's kernel shapes for these members by timing them:
        for each shape (items per warp 0 = compact records in registers, 8 /
        16 = records staged in shared memory; one launch per level or the
        persistent kernel), `steps` steps of FP64 source iteration (FP64
        passes) and of the mixed solve's first FP32 passes, all members
        active, pass time from CUDA events.  Shapes that do not fit in device
        memory (full records for every member) are skipped.  Returns
        (dict(ipw32, ipw64, persistent) of the fastest, the table)."""
        table = []
        items = sum(sw.mesh.n_cells * sw.n_angles for sw in sweepers)
        try:
            import torch
            free = torch.cuda.mem_get_info(device)[0]
        except Exception:
            free = 0
        for ipw, persistent in (shapes or cls.TUNE_SHAPES):
            row = {"ipw": ipw, "persistent": persistent}
            if ipw and items * (256 + 128) > 0.5 * free:
                # full FP64 + FP32 records for every member would not fit
                row.update(fp64_ms_per_pass=None, fp32_ms_per_pass=None, skipped="records do not fit")
                table.append(row)
                continue
            for method, key in (("si", "fp64_ms_per_pass"), ("mixed", "fp32_ms_per_pass")):
                b = None
                try:
                    b = cls(device=device, ipw32=ipw, ipw64=ipw, persistent=persistent)
                    for sw in sweepers:
                        b.add(sw, method, iter_max=10 * steps)
                    for _ in range(steps):
                        b.step()
                    t = b.timing()
                    p = "fp64" if method == "si" else "fp32"
                    row[key] = t[p + "_ms"] / max(1, t[p + "_passes"])
                except _capi.TychoError as e:
                    row[key] = None
                    row["skipped"] = str(e)[:120]
                finally:
                    if b is not None:
                        b.close()
            table.append(row)

        def best(key, ok):
            rows = [r for r in table if r.get(key) is not None and ok(r)]
            return min(rows, key=lambda r: r[key]) if rows else None

        # the form is shared by both passes: pick it on their sum, then each
        # precision's items per warp within that form
        forms = {}
        for persistent in (False, True):
            r64 = best("fp64_ms_per_pass", lambda r: r["persistent"] == persistent)
            r32 = best("fp32_ms_per_pass", lambda r: r["persistent"] == persistent)
            if r64 and r32:
                forms[persistent] = (r64["fp64_ms_per_pass"] + r32["fp32_ms_per_pass"], r64["ipw"], r32["ipw"])
        persistent = min(forms, key=lambda k: forms[k][0])
        _, ipw64, ipw32 = forms[persistent]
        return {"ipw32": ipw32, "ipw64": ipw64, "persistent": persistent}, table

    def timing(self):
        ms, passes, upd = np.zeros(2), np.zeros(2, np.int32), np.zeros(2)
        check(lib().tycho_batch_timing(self._h, ptr(ms), ptr(passes), ptr(upd)))
        return {"fp64_ms": float(ms[0]), "fp32_ms": float(ms[1]), "fp64_passes": int(passes[0]),
                "fp32_passes": int(passes[1]), "fp64_updates": float(upd[0]),
                "fp32_updates": float(upd[1])}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value and _capi._lib is not None:
            _capi._lib.tycho_batch_destroy(self._h)
        self._h = None
        self._members = {}

    def __del__(self):
        self.close()


def release_cached_memory(device=0):
    """Hands the device memory pool's unused memory back to the system (the
    pool keeps what sweepers free for reuse, like a caching allocator)."""
    check(lib().tycho_release_cached_memory(device))


def device_memory(device=0):
    """(bytes the library's memory pool holds on `device`, bytes in use)."""
    r, u = C.c_uint64(), C.c_uint64()
    check(lib().tycho_device_memory(device, C.byref(r), C.byref(u)))
    return r.value, u.value


def footprint_bytes(n_cells, sn_order, n_groups, mixed=True, compact=True):
    """Device bytes one resident solve request holds (tycho_footprint_bytes)."""
    return int(lib().tycho_footprint_bytes(n_cells, sn_order, n_groups, int(mixed), int(compact)))


class SolveServer:
    """Solve service on one GPU (tycho_server_*): requests with arrival times
    are admitted by device-memory footprint against `budget_bytes`, built by
    host threads and solved by continuous batching; requests of at least
    `large_items` cells x angles are solved one at a time beside the batch by
    the single-instance solver (or, large_batched, in a second batch)."""

    STATES = {0: "queued", 1: "building", 2: "built", 3: "in batch", 4: "done", 5: "failed"}

    def __init__(self, method="mixed", budget_bytes=150e9, device=0, setup_threads=2, ipw32=0,
                 ipw64=0, iter_max=3000, err_max=1e-10, inner_tol=1e-5, inner_max=200, refine_max=30,
                 large_items=0.0, large_batched=False):
        solve = _capi.BatchOpts(BatchSolver.BATCH_METHODS[method], iter_max, err_max, inner_tol,
                                inner_max, refine_max)
        o = _capi.ServerOpts(device, float(budget_bytes), setup_threads, ipw32, ipw64, solve,
                             float(large_items), int(bool(large_batched)))
        h = C.c_void_p()
        check(lib().tycho_server_create(C.byref(o), C.byref(h)))
        self._h = h
        self.method = method
        self._out = {}
        self._keep = []

    def submit(self, mesh, sn_order, n_groups, sigma_t, sigma_s, scatter=None, q_iso=None, arrival=0.0):
        """Queues a request; returns its id.  phi is available after run()."""
        phi = np.empty((mesh.n_cells, 4, n_groups))
        arrs = [np.ascontiguousarray(a, np.float64) if a is not None else None
                for a in (sigma_t, sigma_s, scatter, q_iso)]
        rid = C.c_int()
        check(lib().tycho_server_submit(self._h, mesh._h, sn_order, n_groups, *(ptr(a) for a in arrs),
                                        float(arrival), ptr(phi), C.byref(rid)))
        self._out[rid.value] = phi
        self._keep.append(mesh)
        return rid.value

    def run(self):
        check(lib().tycho_server_run(self._h))

    def phi(self, rid):
        return self._out[rid]

    def info(self, rid):
        i = _capi.RequestInfo()
        check(lib().tycho_server_request(self._h, rid, C.byref(i)))
        d = {k: getattr(i, k) for k, _ in _capi.RequestInfo._fields_ if k != "stats"}
        d["state"] = self.STATES.get(d["state"], d["state"])
        d["stats"] = {k: getattr(i.stats, k) for k, _ in _capi.SolveStats._fields_}
        d["latency"] = d["finished"] - d["arrival"] if d["finished"] >= 0 else None
        return d

    def stats(self):
        pb, ms = C.c_double(), C.c_double()
        pa, st = C.c_int(), C.c_int()
        check(lib().tycho_server_stats(self._h, C.byref(pb), C.byref(pa), C.byref(st), C.byref(ms)))
        return {"peak_bytes": pb.value, "peak_active": pa.value, "steps": st.value, "makespan": ms.value}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value and _capi._lib is not None:
            _capi._lib.tycho_server_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()
