"""Angle-sharded solves: one problem's directions split over several GPUs.

The reference parallelises a sweep over spatial partitions, with boundary
psi exchanged between MPI ranks as the wavefront crosses them
(src/GraphTraverser.cc:659-731, src/SweeperPBJ.cc, src/SweeperSchur.cc).
Directions, however, never depend on each other within one sweep: only the
scalar flux phi = sum_a w_a psi_a (src/Util.cc:85-97) couples them.  Here
each process (one per GPU) holds the whole mesh and sweeps a contiguous
range of directions (tycho_sweeper_create_angles); one operator
application is its shard's partial phi followed by one all-reduce (sum) of
phi, Nc * 4 * G doubles, over NCCL.  The outer iterations (source
iteration, GMRES) then run identically on every rank.

The sum over shards adds the shards' partial sums, not the directions one
by one in angle order as psiToPhi does, so phi agrees with the one-GPU
result to rounding (not bit for bit).
"""
import numpy as np

from .sweeper import SweeperCuda


def angle_ranges(n_angles, world):
    """Contiguous, balanced direction ranges [begin, end), one per shard."""
    if not 1 <= world <= n_angles:
        raise ValueError("need 1 <= shards <= directions (%d)" % n_angles)
    return [(n_angles * r // world, n_angles * (r + 1) // world) for r in range(world)]


class ShardedOperator:
    """phi_out = sum over shards of D L^-1 ([Q] + M S phi_in) restricted to
    each shard's directions.

    `apply_local(phi_in, phi_out, with_fixed)` writes this process's partial
    sum (one shard, or the sum of several shards held by this process);
    `reduce(t)` sums t over processes in place (torch.distributed.all_reduce
    when a process group is given; nothing for one process)."""

    def __init__(self, apply_local, group=None, distributed=None):
        import torch.distributed as dist
        self.apply_local = apply_local
        self.group = group
        self.distributed = dist.is_available() and dist.is_initialized() if distributed is None else distributed

    def reduce(self, t):
        if self.distributed:
            import torch.distributed as dist
            dist.all_reduce(t, group=self.group)

    def agree(self, values):
        """The same small vector of scalars on every process (rank 0's):
        every rank then takes the same branches of the outer iteration."""
        if self.distributed:
            import torch
            import torch.distributed as dist
            t = torch.tensor(values, dtype=torch.float64)
            if dist.get_backend(self.group) == "nccl":
                t = t.cuda()
            dist.broadcast(t, src=dist.get_global_rank(self.group, 0) if self.group else 0, group=self.group)
            return t.cpu().tolist()
        return list(values)

    def __call__(self, phi_in, phi_out, with_fixed):
        self.apply_local(phi_in, phi_out, with_fixed)
        self.reduce(phi_out)


def source_iteration(op, like, iter_max=100, err_max=1e-10):
    """SourceIteration::fixedPoint (src/SourceIteration.cc:127-207) over a
    sharded operator: phi <- T(phi) until the L1 relative change is at most
    err_max.  `like`: a tensor of phi's shape, dtype and device.  Returns
    (phi, iterations, last change)."""
    import torch
    phi = torch.zeros_like(like)
    nxt = torch.empty_like(like)
    err, it = 1.0, 0
    while it < iter_max and err > err_max:
        op(phi, nxt, True)
        d = float((nxt - phi).abs().sum())
        m = float(nxt.abs().sum())
        d, m = op.agree([d, m])
        err = d / m if m > 0 else 0.0
        phi, nxt = nxt, phi
        it += 1
    return phi, it, err


def gmres(op, like, restart=20, rtol=1e-10, iter_max=200):
    """SourceIteration::krylov (src/SourceIteration.cc:216-285) over a
    sharded operator: restarted GMRES on (I - D L^-1 M S) phi = D L^-1 Q
    (classical Gram-Schmidt twice, Givens rotations, true residual at each
    restart), inner products on every rank with rank 0's values broadcast.
    Returns (phi, iterations, relative residual)."""
    import torch
    b = torch.empty_like(like)
    op(None, b, True)
    x = torch.zeros_like(like)
    bnorm = op.agree([float(torch.linalg.vector_norm(b))])[0]
    if bnorm == 0.0:
        return x, 0, 0.0
    m = restart
    V = [torch.empty_like(like) for _ in range(m + 1)]
    w = torch.empty_like(like)
    r = b.clone()
    beta = bnorm
    its = 0
    while its < iter_max and beta > rtol * bnorm:
        V[0].copy_(r / beta)
        H = np.zeros((m + 1, m))
        cs, sn = np.zeros(m), np.zeros(m)
        g = np.zeros(m + 1)
        g[0] = beta
        k = 0
        while k < m and its < iter_max:
            op(V[k], w, False)
            w.neg_().add_(V[k])  # w = (I - K) v_k
            h = np.zeros(k + 1)
            for _ in range(2):
                c = op.agree([float(torch.dot(w.reshape(-1), V[j].reshape(-1))) for j in range(k + 1)])
                for j in range(k + 1):
                    w.add_(V[j], alpha=-c[j])
                h += np.array(c)
            hn = op.agree([float(torch.linalg.vector_norm(w))])[0]
            H[: k + 1, k] = h
            H[k + 1, k] = hn
            if hn > 0:
                V[k + 1].copy_(w / hn)
            for j in range(k):
                h0, h1 = H[j, k], H[j + 1, k]
                H[j, k], H[j + 1, k] = cs[j] * h0 + sn[j] * h1, -sn[j] * h0 + cs[j] * h1
            den = np.hypot(H[k, k], hn)
            cs[k], sn[k] = (H[k, k] / den, hn / den) if den > 0 else (1.0, 0.0)
            H[k, k], H[k + 1, k] = den, 0.0
            g[k + 1] = -sn[k] * g[k]
            g[k] = cs[k] * g[k]
            its += 1
            k += 1
            if abs(g[k]) <= rtol * bnorm or hn == 0.0:
                break
        y = np.linalg.solve(np.triu(H[:k, :k]), g[:k])
        for j in range(k):
            x.add_(V[j], alpha=float(y[j]))
        op(x, w, False)  # true residual r = b - (I - K) x
        r = b - x + w
        beta = op.agree([float(torch.linalg.vector_norm(r))])[0]
    return x, its, beta / bnorm


class AngleShardedSolver:
    """One process's shard of an angle-sharded problem on its GPU.

    With torch.distributed initialised (NCCL, one process per GPU), rank r
    of W sweeps directions angle_ranges(2 sn^2, W)[r]; without it, one
    process sweeps them all.  `solve` runs source iteration or GMRES over
    the sharded operator; every rank returns the same phi."""

    def __init__(self, mesh, sn_order, n_groups, device=0, group=None, fp32=False, **kw):
        import torch.distributed as dist
        dist_on = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if dist_on else 0
        self.world = dist.get_world_size(group) if dist_on else 1
        self.device = device
        self.range = angle_ranges(2 * sn_order * sn_order, self.world)[self.rank]
        self.sweeper = SweeperCuda(mesh, sn_order, n_groups, fp32=fp32, device=device, angles=self.range, **kw)
        self.op = ShardedOperator(self._local, group=group, distributed=dist_on)

    def _local(self, phi_in, phi_out, with_fixed):
        self.sweeper.apply(phi_in, phi_out, 0, with_fixed)

    def set_cross_sections(self, sigma_t, sigma_s, scatter=None):
        self.sweeper.set_cross_sections(sigma_t, sigma_s, scatter)

    def set_source(self, q_iso):
        """Isotropic fixed source, phi layout (the same on every rank)."""
        self.sweeper.set_source(q_iso, "isotropic")

    def solve(self, method="si", iter_max=200, err_max=1e-10, restart=20):
        import torch
        like = torch.empty(self.sweeper.phi_shape, dtype=torch.float64, device="cuda:%d" % self.device)
        if method == "si":
            return source_iteration(self.op, like, iter_max, err_max)
        if method == "gmres":
            return gmres(self.op, like, restart, err_max, iter_max)
        raise ValueError("method must be 'si' or 'gmres'")

    def close(self):
        self.sweeper.close()
