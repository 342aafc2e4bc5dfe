"""Multi-partition sweeps: the reference's parallel block Jacobi (PBJ)
sweepers over partition-local B200 sweeps.

The reference splits a mesh into spatial partitions, one per MPI rank
(util/PartitionColumns, src/ParallelMesh.cc).  Its PBJ sweepers sweep each
partition on its own -- Util::sweepLocal(psi, source, psiBound), where the
incoming psi on faces toward other partitions is psiBound, the values those
partitions sent at the last exchange -- and then exchange boundary psi
(CommSides::commSides), iterating until the partitions agree
(src/SweeperPBJ.cc, src/CommSides.cc, src/Util.cc:138-145).

Here a partition is a SweeperCuda made from one partition of the .pmesh
(TychoMesh.read_pmesh(path, partition)); the exchange runs on the device
(tycho_sweeper_side_pack / side_unpack).  The partitions of one problem
live either in one process (PartitionSet: any devices, packets moved by
device copies) or one per process (DistributedPartitions: packets moved by
torch.distributed point-to-point sends, NCCL between GPUs).  Both present
the same operations to the solvers below:

  pbj_si     SweeperPBJSI::solve    src/SweeperPBJ.cc:218-280
  pbj        SweeperPBJ::solve      src/SweeperPBJ.cc:147-211 (source
             iteration whose every sweep iterates sweepLocal + commSides
             until psi changes by at most ddErrMax)
  pbj_outer  SweeperPBJOuter::solve src/SweeperPBJ.cc:59-141 (source
             iteration to errMax with the boundary values fixed, then
             commSides, until psi changes by at most ddErrMax)
  schur      SweeperSchur::solve    src/SweeperSchur.cc:196-326 (source
             iteration whose every sweep solves for the boundary values
             by GMRES)
  schur_outer SweeperSchurOuter::solve src/SweeperSchur.cc:326-470 (GMRES
             on the boundary values, a whole source iteration in every
             operator application)
  schur_krylov SweeperSchurKrylov::solve src/SweeperSchur.cc:487-604 (one
             GMRES over the boundary values and phi together)
  source_krylov SourceIteration::krylov over the PBJ, PBJOuter or Schur
             sweep (the solvers' deck key SourceIteration false)

Iteration counts and convergence follow the reference's tests; the L1 sums
run on the device, in another order than the reference's loops, so a
change that lands within rounding of a tolerance may take one iteration
more or less.  The converged phi is the single-partition solution's.
"""
import numpy as np

from .sweeper import NONE, SweeperCuda, TychoMesh


def neighbours_of(mesh):
    """Partitions across this partition's faces toward other partitions,
    in increasing order (CommSides::CommSides lists them by first
    appearance; the order of exchanges does not change any value)."""
    side, rank, _ = mesh.side_tables()
    adj = mesh.tables()["adj_cell"]
    sel = (adj == NONE) & (rank != NONE) & (rank != np.uint64(mesh.partition))
    return sorted(int(r) for r in np.unique(rank[sel]))


class GpuPartition:
    """One partition's sweeper and its packet buffers."""

    def __init__(self, sweeper):
        import torch
        self.sw = sweeper
        self.mesh = sweeper.mesh
        self.partition = self.mesh.partition
        self.device = torch.device("cuda", sweeper.device)
        self.neighbours = neighbours_of(self.mesh)
        self.gid = self.mesh.tables()["cell_gid"].astype(np.int64)  # global cell of each cell
        self._send = {}

    def send_list(self, q):
        return self.sw.side_send_list(q)

    def link(self, q, gside, angle):
        self.sw.side_link(q, gside, angle)

    def pack(self, q):
        import torch
        n, _ = self.sw.side_counts(q)
        buf = self._send.get(q)
        if buf is None:
            buf = self._send[q] = torch.empty(max(n, 1) * 3 * self.sw.n_groups, dtype=torch.float64,
                                              device=self.device)
        with torch.cuda.device(self.device):
            if n:
                self.sw.side_pack(q, buf)
        return buf[:n * 3 * self.sw.n_groups]

    def unpack(self, q, data):
        import torch
        with torch.cuda.device(self.device):
            if data.numel():
                self.sw.side_unpack(q, data)

    def phi_zeros(self):
        import torch
        return torch.zeros(self.sw.phi_shape, dtype=torch.float64, device=self.device)

    def apply(self, phi_in, phi_out, with_fixed):
        import torch
        with torch.cuda.device(self.device):
            self.sw.apply(phi_in, phi_out, with_fixed=with_fixed)

    def psi_change(self):
        return self.sw.psi_change()

    def get_bound(self):
        """psiBound (PsiBoundData layout, host)."""
        return self.sw.get_psi_bound()

    def set_bound(self, pb):
        self.sw.set_psi_bound(pb)


class PartitionSet:
    """Every partition of one problem in this process (emulated ranks).

    `parts`: one GpuPartition (or any object with the same methods) per
    partition, in partition order.  The exchange packs each partition's
    packets for every neighbour and unpacks them at the neighbour, on that
    neighbour's device."""

    def __init__(self, parts):
        self.parts = list(parts)
        for p, part in enumerate(self.parts):
            assert part.partition == p, "partitions must be given in order"
        for part in self.parts:
            for q in part.neighbours:
                gs, an = part.send_list(q)
                self.parts[q].link(part.partition, gs, an)

    @classmethod
    def from_pmesh(cls, path, sn_order, n_groups, devices=(0,), **kw):
        """Sweepers on every partition of a .pmesh, placed round-robin on
        `devices`; keyword arguments go to SweeperCuda."""
        m0 = TychoMesh.read_pmesh(path, 0)
        parts = []
        for p in range(m0.n_partitions):
            mesh = m0 if p == 0 else TychoMesh.read_pmesh(path, p)
            sw = SweeperCuda(mesh, sn_order, n_groups, device=devices[p % len(devices)], **kw)
            parts.append(GpuPartition(sw))
        return cls(parts)

    @property
    def local(self):
        return self.parts

    def exchange(self):
        """CommSides::commSides for every partition (src/CommSides.cc:119-240)."""
        moved = []
        for part in self.parts:
            for q in part.neighbours:
                moved.append((q, part.partition, part.pack(q)))
        for q, src, data in moved:
            dst = self.parts[q]
            dev = getattr(dst, "device", None)
            dst.unpack(src, data.to(dev) if dev is not None else data)

    def allsum(self, values):
        return list(values)

    def close(self):
        for part in self.parts:
            sw = getattr(part, "sw", None)
            if sw is not None:
                sw.close()


class DistributedPartitions:
    """This process's partition of a problem spread over a torch.distributed
    group, one partition per rank (rank r holds partition r).  Packets go by
    point-to-point sends (isend / irecv) to each neighbour; sums by
    all_reduce.  With the gloo backend the packets travel through host
    memory."""

    def __init__(self, part, group=None):
        import torch
        import torch.distributed as dist
        self.part = part
        self.group = group
        self.rank = dist.get_rank(group)
        assert part.partition == self.rank, "rank r holds partition r"
        self.host = dist.get_backend(group) != "nccl"
        self.sizes = {}
        # send lists to the neighbours, received lists link the packets
        for q in part.neighbours:
            gs, an = part.send_list(q)
            pairs = np.stack([gs.astype(np.int64), an.astype(np.int64)], axis=1).reshape(-1)
            out = self._wire(torch.from_numpy(pairs.copy()))
            n_out = self._wire(torch.tensor([pairs.size], dtype=torch.int64))
            n_in = self._wire(torch.zeros(1, dtype=torch.int64))
            self._swap(q, n_out, n_in)
            got = self._wire(torch.zeros(int(n_in.item()), dtype=torch.int64))
            self._swap(q, out, got)
            got = got.cpu().numpy().reshape(-1, 2)
            part.link(q, got[:, 0].astype(np.uint64), got[:, 1].astype(np.uint32))
            self.sizes[q] = got.shape[0] * 3 * self._groups()

    def _groups(self):
        sw = getattr(self.part, "sw", None)
        return sw.n_groups if sw is not None else self.part.n_groups

    def _wire(self, t):
        import torch
        return t if self.host else t.to(torch.device("cuda", torch.cuda.current_device()))

    def _swap(self, q, send, recv):
        import torch.distributed as dist
        ops = [dist.P2POp(dist.isend, send, q, self.group), dist.P2POp(dist.irecv, recv, q, self.group)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()

    @property
    def local(self):
        return [self.part]

    def exchange(self):
        import torch
        for q in self.part.neighbours:
            data = self.part.pack(q)
            send = data.cpu() if self.host and data.is_cuda else data
            recv = torch.empty(self.sizes[q], dtype=torch.float64, device=send.device)
            self._swap(q, send.contiguous(), recv)
            dev = getattr(self.part, "device", None)
            self.part.unpack(q, recv.to(dev) if dev is not None else recv)

    def allsum(self, values):
        import torch
        import torch.distributed as dist
        t = self._wire(torch.tensor(values, dtype=torch.float64))
        dist.all_reduce(t, group=self.group)
        return t.cpu().tolist()


def _l1(parts, a, b):
    """(sum |a - b|, sum |a|) over this process's partitions (b may be None)."""
    d = m = 0.0
    for x, y in zip(a, b if b is not None else [None] * len(a)):
        m += float(x.abs().sum())
        if y is not None:
            d += float((x - y).abs().sum())
    return d, m


def pbj_si(ps, dd_iter_max=100, dd_err_max=1e-10):
    """SweeperPBJSI::solve: phi1 = T(phi0) on every partition with the last
    exchanged boundary values, exchange, stop when the L1 relative change of
    phi is below dd_err_max (the exchange comes before the test, as in the
    reference).  Returns (phi per local partition, iterations, change)."""
    phi0 = [p.phi_zeros() for p in ps.local]
    phi1 = [p.phi_zeros() for p in ps.local]
    it, err = 1, 1.0
    while it < dd_iter_max:
        for p, a, b in zip(ps.local, phi0, phi1):
            p.apply(a, b, True)
        ps.exchange()
        d, m = ps.allsum(_l1(ps.local, phi1, phi0))
        err = d / m if m > 0 else 0.0
        phi0, phi1 = phi1, phi0
        if err < dd_err_max:
            break
        it += 1
    return phi0, it, err


def _pbj_sweep(ps, phi_old, phi_out, dd_iter_max, dd_err_max, with_fixed=True):
    """SweeperPBJ::sweep: sweepLocal until psi changes by less than
    dd_err_max (L1, relative), exchanging after every sweep that has not
    converged.  Returns the number of local sweeps."""
    it = 1
    while it < dd_iter_max:
        for p, a, b in zip(ps.local, phi_old, phi_out):
            p.apply(a, b, with_fixed)
        d, m = ps.allsum([sum(v) for v in zip(*[p.psi_change() for p in ps.local])])
        if m > 0 and d / m < dd_err_max:
            break
        ps.exchange()
        it += 1
    return it


def pbj(ps, iter_max=100, err_max=1e-10, dd_iter_max=100, dd_err_max=1e-10, method="si"):
    """SweeperPBJ::solve with source iteration (SourceIteration::fixedPoint,
    src/SourceIteration.cc:127-207, over SweeperPBJ::sweep), or with
    method "krylov" SourceIteration::krylov over the same sweep
    (source_krylov).  Returns (phi per local partition, source iterations
    or Krylov iterations, last change or residual norm, local sweeps)."""
    if method == "krylov":
        counter = _SweepCounter(ps)
        phi, its, rn = source_krylov(counter, "pbj", iter_max, err_max, dd_iter_max=dd_iter_max,
                                     dd_err_max=dd_err_max)
        return phi, its, rn, counter.sweeps
    phi_new = [p.phi_zeros() for p in ps.local]
    phi_old = [p.phi_zeros() for p in ps.local]
    it, err, sweeps = 0, 1.0, 0
    while it < iter_max and err > err_max:
        for a, b in zip(phi_old, phi_new):
            a.copy_(b)
        sweeps += _pbj_sweep(ps, phi_old, phi_new, dd_iter_max, dd_err_max)
        d, m = ps.allsum(_l1(ps.local, phi_new, phi_old))
        err = d / m if m > 0 else 0.0
        it += 1
    return phi_new, it, err, sweeps


def pbj_outer(ps, iter_max=100, err_max=1e-10, dd_iter_max=100, dd_err_max=1e-10, method="si"):
    """SweeperPBJOuter::solve: each outer iteration solves the partitions'
    problems with the boundary values fixed -- SourceIteration::fixedPoint
    to err_max from the current psi, or with method "krylov"
    SourceIteration::krylov (source_krylov, "pbj_outer") -- then tests the
    L1 change of psi against dd_err_max and exchanges.  Returns (phi per
    local partition, outer iterations, inner iterations per outer
    iteration)."""
    phi_new = [p.phi_zeros() for p in ps.local]
    phi_old = [p.phi_zeros() for p in ps.local]
    its = []
    outer = 1
    while outer < dd_iter_max:
        if method == "krylov":
            phi, k, _ = source_krylov(ps, "pbj_outer", iter_max, err_max)
            for a, b in zip(phi_new, phi):
                a.copy_(b)
            its.append(k)
            d, m = ps.allsum([sum(v) for v in zip(*[p.psi_change() for p in ps.local])])
            if m > 0 and d / m < dd_err_max:
                break
            ps.exchange()
            outer += 1
            continue
        it, err = 0, 1.0
        while it < iter_max and err > err_max:
            for a, b in zip(phi_old, phi_new):
                a.copy_(b)
            for p, a, b in zip(ps.local, phi_old, phi_new):
                p.apply(a, b, True)
            d, m = ps.allsum(_l1(ps.local, phi_new, phi_old))
            err = d / m if m > 0 else 0.0
            it += 1
        its.append(it)
        d, m = ps.allsum([sum(v) for v in zip(*[p.psi_change() for p in ps.local])])
        if m > 0 and d / m < dd_err_max:
            break
        ps.exchange()
        outer += 1
    return phi_new, outer, its


def _dot(ps, u, v):
    """Inner product of two distributed vectors (lists of arrays -- numpy on
    the host or torch tensors -- one per local partition) over every
    partition."""
    return ps.allsum([sum(float((a.reshape(-1) * b.reshape(-1)).sum()) for a, b in zip(u, v))])[0]


def _copy(a):
    return a.clone() if hasattr(a, "clone") else a.copy()


def _gmres(ps, op, b, x, rtol, iter_max, restart=30):
    """Restarted GMRES on distributed vectors (lists of arrays, one per
    local partition): op(x) -> A x, b the right-hand side, x the initial
    guess (updated in place); classical Gram-Schmidt twice, Givens
    rotations, the true residual at each restart, stop when ||r|| <= rtol
    ||b||.  The reference's KrylovSolver is PETSc's KSPGMRES with these
    tolerances (src/KrylovSolver.cc:97-101); PETSc is absent, so the
    iterates are this method's.  Returns (iterations, residual norm)."""
    bnorm = np.sqrt(_dot(ps, b, b))
    its = 0

    def residual():
        ax = op(x)
        return [bi - ai for bi, ai in zip(b, ax)]

    # a zero initial guess needs no operator application (as KSPSolve)
    zero = ps.allsum([float(sum(float(abs(xi).sum()) for xi in x))])[0] == 0.0
    r = [_copy(bi) for bi in b] if zero else residual()
    beta = np.sqrt(_dot(ps, r, r))
    while its < iter_max and beta > rtol * bnorm:
        V = [[ri / beta for ri in r]]
        H = np.zeros((restart + 1, restart))
        cs, sn, g = np.zeros(restart), np.zeros(restart), np.zeros(restart + 1)
        g[0] = beta
        k = 0
        while k < restart and its < iter_max:
            w = op(V[k])
            for _ in range(2):
                h = [_dot(ps, w, V[j]) for j in range(k + 1)]
                for j in range(k + 1):
                    H[j, k] += h[j]
                    w = [wi - h[j] * vj for wi, vj in zip(w, V[j])]
            hn = np.sqrt(_dot(ps, w, w))
            H[k + 1, k] = hn
            for j in range(k):
                h0, h1 = H[j, k], H[j + 1, k]
                H[j, k], H[j + 1, k] = cs[j] * h0 + sn[j] * h1, -sn[j] * h0 + cs[j] * h1
            den = np.hypot(H[k, k], hn)
            cs[k], sn[k] = (H[k, k] / den, hn / den) if den > 0 else (1.0, 0.0)
            H[k, k] = den
            g[k + 1], g[k] = -sn[k] * g[k], cs[k] * g[k]
            its += 1
            k += 1
            V.append([wi / hn for wi in w] if hn > 0 else w)
            if abs(g[k]) <= rtol * bnorm or hn == 0:
                break
        y = np.linalg.solve(np.triu(H[:k, :k]), g[:k]) if k else np.zeros(0)
        for j in range(k):
            for xi, vj in zip(x, V[j]):
                xi += y[j] * vj
        r = residual()
        beta = np.sqrt(_dot(ps, r, r))
    return its, beta


def _sweep_exchange(ps, bounds, phi_in, with_fixed, phi_out):
    """Util::sweepLocal on every partition with the given psiBound, then
    CommSides: returns the boundary values after the exchange."""
    for part, pb in zip(ps.local, bounds):
        part.set_bound(pb)
    for part, a, o in zip(ps.local, phi_in, phi_out):
        part.apply(a, o, with_fixed)
    ps.exchange()
    return [part.get_bound() for part in ps.local]


def schur(ps, iter_max=100, err_max=1e-10, dd_iter_max=100, dd_err_max=1e-10, method="si"):
    """SweeperSchur::solve with source iteration (src/SweeperSchur.cc:
    196-326): every sweep of SourceIteration::fixedPoint solves for the
    incoming partition-boundary psi by Krylov,
      (I - W L_I^-1 L_B) psi_B = W L_I^-1 q,
    with the last sweep's psi_B as initial guess (the right-hand side: one
    local sweep of the total source with zero boundary values, then the
    exchange), then sweeps each partition with the solved values.  The
    Krylov vectors are the partitions' psiBound arrays on the host.
    Returns (phi per local partition, source iterations, last change,
    local sweeps); with method "krylov" SourceIteration::krylov over the
    same sweep (source_krylov): (phi, Krylov iterations, residual norm,
    local sweeps)."""
    if method == "krylov":
        counter = _SweepCounter(ps)
        phi, its, rn = source_krylov(counter, "schur", iter_max, err_max, dd_iter_max=dd_iter_max,
                                     dd_err_max=dd_err_max)
        return phi, its, rn, counter.sweeps
    phi_new = [p.phi_zeros() for p in ps.local]
    phi_old = [p.phi_zeros() for p in ps.local]
    state = _SchurState(ps)
    it, err = 0, 1.0
    while it < iter_max and err > err_max:
        for a, b in zip(phi_old, phi_new):
            a.copy_(b)
        state.sweep(phi_old, True, phi_new, dd_iter_max, dd_err_max)
        d, m = ps.allsum(_l1(ps.local, phi_new, phi_old))
        err = d / m if m > 0 else 0.0
        it += 1
    return phi_new, it, err, state.sweeps


class _SchurState:
    """SweeperSchur::sweep (src/SweeperSchur.cc:246-323) with its
    c_psiBoundPrev: the Krylov solve for the incoming boundary values from
    the last solve's values, then one local sweep with them."""

    def __init__(self, ps):
        self.ps = ps
        self.prev = [np.zeros_like(p.get_bound()) for p in ps.local]
        self.tmp = [p.phi_zeros() for p in ps.local]
        self.sweeps = 0

    def sweep(self, phi_in, with_fixed, phi_out, dd_iter_max, dd_err_max):
        ps, tmp = self.ps, self.tmp

        def op(x):
            y = _sweep_exchange(ps, x, [None] * len(x), False, tmp)
            return [xi - yi for xi, yi in zip(x, y)]

        rhs = _sweep_exchange(ps, [np.zeros_like(x) for x in self.prev], phi_in, with_fixed, tmp)
        x = [pv.copy() for pv in self.prev]
        its, _ = _gmres(ps, op, rhs, x, dd_err_max, dd_iter_max)
        for part, xi in zip(ps.local, x):
            part.set_bound(xi)
        for part, a, o in zip(ps.local, phi_in, phi_out):
            part.apply(a, o, with_fixed)
        self.prev = x
        self.sweeps += 2 + its


def schur_outer(ps, iter_max=100, err_max=1e-10, dd_iter_max=100, dd_err_max=1e-10):
    """SweeperSchurOuter::solve with source iteration (src/SweeperSchur.cc:
    326-470): GMRES from zero on the incoming boundary values,
      (I - W (L_I - M S D)^-1 L_B) psi_B = W (L_I - M S D)^-1 Q,
    where every operator application is a whole source iteration
    (SourceIteration::fixedPoint from the current psi, zero source, the
    given boundary values) followed by the exchange; the right-hand side is
    the source iteration of Q with zero boundary values, the answer the
    source iteration of Q with the solved ones.  Returns (phi per local
    partition, Krylov iterations, residual norm, source iterations: the
    right-hand side's, each operator application's, the last one's)."""
    phi = [p.phi_zeros() for p in ps.local]

    def fixed_point(with_fixed):
        # from phi = psiToPhi(psi) of the last sweep, as fixedPoint starts
        it, err = 0, 1.0
        while it < iter_max and err > err_max:
            old = [t.clone() for t in phi]
            for part, a, o in zip(ps.local, old, phi):
                part.apply(a, o, with_fixed)
            d, m = ps.allsum(_l1(ps.local, phi, old))
            err = d / m if m > 0 else 0.0
            it += 1
        return it

    for part in ps.local:
        part.set_bound(np.zeros_like(part.get_bound()))
    its_rhs = fixed_point(True)
    ps.exchange()
    rhs = [part.get_bound() for part in ps.local]
    for t in phi:  # psi = 0
        t.zero_()
    its_op = []

    def op(x):
        for part, xi in zip(ps.local, x):
            part.set_bound(xi)
        its_op.append(fixed_point(False))
        ps.exchange()
        return [xi - part.get_bound() for part, xi in zip(ps.local, x)]

    x = [np.zeros_like(b) for b in rhs]
    its, rn = _gmres(ps, op, rhs, x, dd_err_max, dd_iter_max)
    for part, xi in zip(ps.local, x):
        part.set_bound(xi)
    its_end = fixed_point(True)
    return phi, its, rn, (its_rhs, its_op, its_end)


def schur_krylov(ps, dd_iter_max=100, dd_err_max=1e-10):
    """SweeperSchurKrylov::solve (src/SweeperSchur.cc:487-604): one Krylov
    solve for the incoming partition-boundary psi and phi together,
      (I - W L_I^-1 L_B) psi_B - W L_I^-1 M S phi  = W L_I^-1 Q
      -D L_I^-1 L_B psi_B + (I - D L_I^-1 M S) phi = D L_I^-1 Q,
    from zero, then one local sweep of Q + M S phi with the solved boundary
    values.  Returns (phi per local partition, Krylov iterations, residual
    norm)."""
    import torch
    n = len(ps.local)
    tmp = [p.phi_zeros() for p in ps.local]

    def to_dev(a, like):
        return torch.from_numpy(np.ascontiguousarray(a)).to(like.device).reshape(like.shape)

    def op(x):
        xb, xp = x[:n], x[n:]
        yb = _sweep_exchange(ps, xb, [to_dev(a, t) for a, t in zip(xp, tmp)], False, tmp)
        yp = [t.cpu().numpy().copy() for t in tmp]
        return [a - b for a, b in zip(x, yb + yp)]

    rb = _sweep_exchange(ps, [np.zeros_like(p.get_bound()) for p in ps.local], [None] * n, True, tmp)
    rhs = rb + [t.cpu().numpy().copy() for t in tmp]
    x = [np.zeros_like(a) for a in rhs]
    its, rn = _gmres(ps, op, rhs, x, dd_err_max, dd_iter_max)
    phi = [p.phi_zeros() for p in ps.local]
    for part, b in zip(ps.local, x[:n]):
        part.set_bound(b)
    for part, a, o in zip(ps.local, x[n:], phi):
        part.apply(to_dev(a, o), o, True)
    return phi, its, rn


class _SweepCounter:
    """The same partitions, counting local sweeps (one per apply of every
    partition)."""

    def __init__(self, ps):
        self._ps = ps
        self.sweeps = 0
        self.local = [_CountingPart(p, self) for p in ps.local]

    def exchange(self):
        self._ps.exchange()

    def allsum(self, values):
        return self._ps.allsum(values)


class _CountingPart:
    def __init__(self, part, counter):
        self._p, self._c = part, counter

    def apply(self, a, b, with_fixed):
        if self._p is self._c.local[0]._p:
            self._c.sweeps += 1
        self._p.apply(a, b, with_fixed)

    def __getattr__(self, name):
        return getattr(self._p, name)


def source_krylov(ps, sweeper="pbj", iter_max=100, err_max=1e-10, restart=30, dd_iter_max=100,
                  dd_err_max=1e-10):
    """SourceIteration::krylov (src/SourceIteration.cc:216-285) over the
    partitions: GMRES on (I - D L^-1 M S) phi = D L^-1 Q, where L^-1 is the
    named sweeper's sweep (src/SweeperPBJ.cc, src/SweeperSchur.cc):
      "pbj"        SweeperPBJ::sweep -- sweepLocal and exchange until psi
                   settles (the boundary values carry over between sweeps)
      "pbj_outer"  SweeperPBJOuter::sweep -- one sweepLocal; the operator's
                   sweeps take zero boundary values (lhsOperator passes
                   zeroPsiBound, src/SourceIteration.cc:81-103), the others
                   the values held, which this solver never exchanges
      "schur"      SweeperSchur::sweep -- the Krylov solve for the boundary
                   values, then sweepLocal
    then psi = L^-1 (M S phi + Q).  Returns (phi per local partition,
    iterations, residual norm)."""
    n = len(ps.local)
    state = _SchurState(ps) if sweeper == "schur" else None
    if sweeper not in ("pbj", "pbj_outer", "schur"):
        raise ValueError("sweeper must be 'pbj', 'pbj_outer' or 'schur'")

    def sweep(phi_in, with_fixed, zero_bound, phi_out):
        if sweeper == "pbj":
            _pbj_sweep(ps, phi_in, phi_out, dd_iter_max, dd_err_max, with_fixed)
        elif sweeper == "schur":
            state.sweep(phi_in, with_fixed, phi_out, dd_iter_max, dd_err_max)
        else:
            keep = [p.get_bound() for p in ps.local] if zero_bound else None
            if keep is not None:
                for p, k in zip(ps.local, keep):
                    p.set_bound(np.zeros_like(k))
            for p, a, o in zip(ps.local, phi_in, phi_out):
                p.apply(a, o, with_fixed)
            if keep is not None:
                for p, k in zip(ps.local, keep):
                    p.set_bound(k)

    tmp = [p.phi_zeros() for p in ps.local]
    b = [p.phi_zeros() for p in ps.local]
    sweep([None] * n, True, False, b)

    def op(x):
        sweep(x, False, True, tmp)
        return [xi - ti for xi, ti in zip(x, tmp)]

    x = [p.phi_zeros() for p in ps.local]
    its, rn = _gmres(ps, op, b, x, err_max, iter_max, restart)
    phi = [p.phi_zeros() for p in ps.local]
    sweep(x, True, False, phi)
    return phi, its, rn


def gather_phi(parts, phis):
    """phi of every partition into one array in global cell order (each
    part's `gid`: its cells' global ids)."""
    n = 1 + max(int(p.gid.max()) for p in parts)
    out = None
    for part, phi in zip(parts, phis):
        a = phi.cpu().numpy() if hasattr(phi, "cpu") else np.asarray(phi)
        if out is None:
            out = np.zeros((n,) + a.shape[1:])
        out[part.gid] = a
    return out
