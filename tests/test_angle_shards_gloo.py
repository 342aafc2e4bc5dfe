"""Angle-sharded solves at world_size 2 over gloo on the host (no GPU).

Each rank's shard operator is the oracle's: the whole sweep restricted to
the rank's directions (phi_part = sum over its angles of w_a psi_a), summed
over the ranks by the all-reduce of tycho2_b200.angles.ShardedOperator.
Source iteration and GMRES over the two shards reach the oracle's
single-process source iteration and GMRES, and both ranks hold the same
phi.  The GPU form (tycho_sweeper_create_angles shards on one device) is
checked in tests/test_gpu_angle_shards.py.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(d):
    import tycho2_b200 as ty
    from oracle.oracle import Oracle, OracleMesh
    from tycho2_b200 import problems
    mesh = ty.TychoMesh.kuhn_cube(4, 0.05, 17, 1.0)
    path = os.path.join(d, "k4.pmesh")
    mesh.write_pmesh(path)
    sn, G = 4, 3
    o = Oracle(OracleMesh(path), sn, G)
    rng = np.random.default_rng(5)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    mat = problems.downscatter_matrix(G, 0.7)
    q = rng.uniform(0.0, 1.0, o.phi_shape)
    return o, st, st.copy(), mat, q


def _shard_apply(o, st, ss, mat, q, a0, a1):
    import torch
    wts = o.quadrature()[3]

    def apply(phi_in, phi_out, with_fixed):
        iso = o.scatter(ss, mat, np.ascontiguousarray(phi_in.numpy())) if phi_in is not None else np.zeros(o.phi_shape)
        if with_fixed:
            iso = q + iso
        psi = o.sweep(st, src_iso=np.ascontiguousarray(iso))
        part = np.einsum("cavg,a->cvg", psi[:, a0:a1], wts[a0:a1])
        phi_out.copy_(torch.from_numpy(np.ascontiguousarray(part)).reshape(phi_out.shape))

    return apply


def _worker(rank, world, port, d, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import torch
    import torch.distributed as dist
    from tycho2_b200.angles import ShardedOperator, angle_ranges, gmres, source_iteration
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        o, st, ss, mat, q = _problem(d)
        a0, a1 = angle_ranges(o.A, world)[rank]
        op = ShardedOperator(_shard_apply(o, st, ss, mat, q, a0, a1))
        like = torch.empty(o.phi_shape, dtype=torch.float64)
        phi_si, it, err = source_iteration(op, like, iter_max=300, err_max=1e-12)
        phi_k, its, rn = gmres(op, like, restart=10, rtol=1e-12, iter_max=200)
        out.put((rank, (a0, a1), phi_si.numpy().copy(), it, err, phi_k.numpy().copy(), its, rn))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_angle_shards_over_gloo(tmp_path):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path), q)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(world):
        r = q.get(timeout=150)
        got[r[0]] = r[1:]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    (r0, phi0, it0, e0, k0, its0, rn0), (r1, phi1, it1, e1, k1, its1, rn1) = got[0], got[1]
    assert r0[0] == 0 and r0[1] == r1[0] and r1[1] == 2 * 4 * 4
    # both ranks hold the same phi and took the same steps
    assert np.array_equal(phi0, phi1) and it0 == it1 and np.array_equal(k0, k1) and its0 == its1
    assert e0 <= 1e-12 and rn0 <= 1e-12
    o, st, ss, mat, qq = _problem(str(tmp_path))
    _, phi_ref, it_ref, _ = o.source_iteration(st, ss, scatter=mat, q_iso=qq, iter_max=300, err_max=1e-12)
    assert abs(it0 - it_ref) <= 1
    assert np.abs(phi0 - phi_ref).sum() / np.abs(phi_ref).sum() <= 1e-12
    _, phi_kref, _, _ = o.krylov(st, ss, mat, q_iso=qq, restart=10, iter_max=200, rtol=1e-12)
    assert np.abs(k0 - phi_kref).sum() / np.abs(phi_kref).sum() <= 1e-11


def test_angle_ranges_cover_every_direction_once():
    import sys
    sys.path.insert(0, ROOT)
    from tycho2_b200.angles import angle_ranges
    for A in (8, 32, 72, 128):
        for W in (1, 2, 3, 8):
            rs = angle_ranges(A, W)
            assert rs[0][0] == 0 and rs[-1][1] == A
            assert all(rs[i][1] == rs[i + 1][0] for i in range(W - 1))
            sizes = [b - a for a, b in rs]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        angle_ranges(8, 9)
