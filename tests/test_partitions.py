"""Multi-partition meshes and the PBJ drivers on the host (no GPU).

Pins, against the reference (tests/golden/partitions_ref.npz, written by
tests/golden/make_golden.py from the reference's PartitionColumns and
ref_dump's sweep_local mode, which runs Util::sweepLocal on one rank's
partition):
  - the product's partition ingest (TychoMesh.read_pmesh(path, p)) and the
    oracle's: adjCell, adjRank, side and lGSides of every partition of a
    2- and a 4-partition Kuhn cube;
  - the oracle's partition-local sweep with psiBound: the hash of its psi
    equals the reference's, bit for bit.
Then the PBJ and Schur drivers (tycho2_b200.partitions) over oracle
partitions reach the single-partition solution, and for PBJ one process
holding both partitions and two gloo ranks holding one each take the same
iterations to the same phi.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT, bits_equal, rel_l1
from helpers import OraclePartition, partition_inputs, partitions_fixture, psi_hash

NONE = np.uint64(0xFFFFFFFFFFFFFFFF)


@pytest.mark.parametrize("P", [2, 4])
def test_partition_tables_match_reference(built, workdir, P):
    import tycho2_b200 as ty
    from oracle.oracle import OracleMesh
    path, ref = partitions_fixture(workdir, P)
    gids = []
    for p in range(P):
        mesh = ty.TychoMesh.read_pmesh(path, p)
        assert mesh.partition == p and mesh.n_partitions == P
        side, rank, sgid = mesh.side_tables()
        adj = mesh.tables()["adj_cell"]
        assert np.array_equal(adj.reshape(-1), ref["p%d_%d_adj" % (P, p)])
        assert np.array_equal(rank.reshape(-1), ref["p%d_%d_rank" % (P, p)])
        assert np.array_equal(side.reshape(-1), ref["p%d_%d_side" % (P, p)])
        assert np.array_equal(sgid, ref["p%d_%d_lgside" % (P, p)])
        om = OracleMesh(path, p)
        ot = om.tables()
        orank, ogid = om.partition_tables()
        assert np.array_equal(ot["adj_cell"], adj) and np.array_equal(orank, rank)
        assert np.array_equal(ot["side"], side) and np.array_equal(ogid, sgid)
        for k in ("neighbor_vrtx", "face_to_cell", "cell_to_face", "volume", "area", "normal", "cell_gid"):
            assert bits_equal(ot[k], mesh.tables()[k]) if ot[k].dtype == np.float64 else \
                np.array_equal(ot[k], mesh.tables()[k]), k
        bound = (adj == NONE) & (rank != NONE) & (rank != np.uint64(p))
        assert mesh.n_bound_sides == int(bound.sum()) > 0
        gids.append(mesh.tables()["cell_gid"])
    # the partitions cover the serial mesh once
    allg = np.sort(np.concatenate(gids))
    assert np.array_equal(allg, np.arange(allg.size, dtype=np.uint64))


@pytest.mark.parametrize("P", [2, 4])
def test_oracle_sweep_local_matches_reference(built, workdir, P):
    from oracle.oracle import Oracle, OracleMesh
    path, ref = partitions_fixture(workdir, P)
    for p in range(P):
        om = OracleMesh(path, p)
        o = Oracle(om, 4, 3)
        st, src, pb = partition_inputs(om.n_cells, o.A, 3, om.n_sides, 10 * P + p)
        psi = o.sweep_local(st, pb, src_ang=src)
        assert psi_hash(psi) == int(ref["p%d_%d_psi_hash" % (P, p)][0]), (P, p)
        # psiBound is read: zero boundary values give another psi
        assert psi_hash(o.sweep_local(st, np.zeros_like(pb), src_ang=src)) != psi_hash(psi)


def test_partition_read_errors(built, workdir):
    import tycho2_b200 as ty
    path, _ = partitions_fixture(workdir, 4)
    with pytest.raises(ty.TychoError, match="name the partition"):
        ty.TychoMesh.read_pmesh(path)
    with pytest.raises(ty.TychoError, match="partition 4 of 4"):
        ty.TychoMesh.read_pmesh(path, 4)
    m = ty.TychoMesh.read_pmesh(path, 1)
    with pytest.raises(ty.TychoError, match="cannot be written"):
        m.write_pmesh(os.path.join(str(workdir), "x.pmesh"))
    # an ordinary mesh: one partition, no faces toward another
    k = ty.TychoMesh.kuhn_cube(2, 0.0, 0, 1.0)
    assert (k.partition, k.n_partitions, k.n_bound_sides) == (0, 1, 0)


def _problem(P, G=2):
    """Global cross sections and isotropic source of the 4^3 Kuhn cube."""
    from tycho2_b200 import problems
    nc = 384
    i = np.arange(nc)
    st = 1.0 + (i % 7) / 4.0
    ss = st * (0.3 + (i % 5) / 10.0)
    mat = problems.downscatter_matrix(G, 0.7)
    q = 0.5 + ((np.arange(nc * 4 * G) * 37) % 11).reshape(nc, 4, G) / 10.0
    return st, ss, mat, q


def _oracle_parts(path, P, sn=4, G=2):
    st, ss, mat, q = _problem(P, G)
    return [OraclePartition(path, p, sn, G, st, ss, mat, q) for p in range(P)]


def _single_partition_si(workdir, sn=4, G=2):
    import tycho2_b200 as ty
    from oracle.oracle import Oracle, OracleMesh
    path = os.path.join(str(workdir), "kuhn4_single.pmesh")
    if not os.path.exists(path):
        ty.TychoMesh.kuhn_cube(4, 0.05, 7, 1.0).write_pmesh(path)
    st, ss, mat, q = _problem(1, G)
    o = Oracle(OracleMesh(path), sn, G)
    _, phi, it, _ = o.source_iteration(st, ss, scatter=mat, q_iso=q, iter_max=400, err_max=1e-12)
    return phi, it


def _gather(parts, phis):
    out = np.zeros((384,) + tuple(phis[0].shape[1:]))
    for part, phi in zip(parts, phis):
        out[part.gid] = phi.numpy()
    return out


@pytest.mark.timeout(300)
def test_pbj_solvers_in_one_process_reach_the_single_partition_solution(built, workdir):
    from tycho2_b200.partitions import PartitionSet, pbj, pbj_outer, pbj_si
    path, _ = partitions_fixture(workdir, 2)
    ref, it_ref = _single_partition_si(workdir)
    ps = PartitionSet(_oracle_parts(path, 2))
    phi, it, err = pbj_si(ps, dd_iter_max=400, dd_err_max=1e-12)
    assert err < 1e-12 and it > it_ref  # the lagged boundary costs iterations
    assert rel_l1(_gather(ps.parts, phi), ref) <= 1e-10
    ps = PartitionSet(_oracle_parts(path, 2))
    phi, it, err, sweeps = pbj(ps, iter_max=400, err_max=1e-12, dd_iter_max=100, dd_err_max=1e-13)
    assert abs(it - it_ref) <= 1 and sweeps > it
    assert rel_l1(_gather(ps.parts, phi), ref) <= 1e-10
    ps = PartitionSet(_oracle_parts(path, 2))
    phi, outer, its = pbj_outer(ps, iter_max=400, err_max=1e-13, dd_iter_max=100, dd_err_max=1e-12)
    assert outer > 1 and len(its) == outer
    assert rel_l1(_gather(ps.parts, phi), ref) <= 1e-10


@pytest.mark.timeout(300)
def test_schur_solvers_reach_the_single_partition_solution(built, workdir):
    from tycho2_b200.partitions import PartitionSet, schur, schur_krylov, schur_outer
    path, _ = partitions_fixture(workdir, 2)
    ref, it_ref = _single_partition_si(workdir)
    ps = PartitionSet(_oracle_parts(path, 2))
    phi, it, err, sweeps = schur(ps, iter_max=400, err_max=1e-12, dd_iter_max=200, dd_err_max=1e-13)
    # each sweep is the whole mesh's sweep to the Krylov tolerance
    assert abs(it - it_ref) <= 1 and sweeps > 2 * it
    assert rel_l1(_gather(ps.parts, phi), ref) <= 1e-10
    ps = PartitionSet(_oracle_parts(path, 2))
    phi, its, rn = schur_krylov(ps, dd_iter_max=400, dd_err_max=1e-13)
    assert its < it_ref  # one Krylov solve of the whole problem
    assert rel_l1(_gather(ps.parts, phi), ref) <= 1e-10
    ps = PartitionSet(_oracle_parts(path, 2))
    phi, its, rn, (i1, iop, i3) = schur_outer(ps, iter_max=400, err_max=1e-13, dd_iter_max=100, dd_err_max=1e-12)
    assert len(iop) >= its and i1 > 1 and i3 >= 1
    assert rel_l1(_gather(ps.parts, phi), ref) <= 1e-10


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, path, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime
    import torch.distributed as dist
    from tycho2_b200.partitions import DistributedPartitions, pbj, pbj_si
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        st, ss, mat, q = _problem(world)
        part = OraclePartition(path, rank, 4, 2, st, ss, mat, q)
        ds = DistributedPartitions(part)
        phi, it, err = pbj_si(ds, dd_iter_max=400, dd_err_max=1e-12)
        part2 = OraclePartition(path, rank, 4, 2, st, ss, mat, q)
        ds2 = DistributedPartitions(part2)
        phi2, it2, err2, sweeps2 = pbj(ds2, iter_max=400, err_max=1e-12, dd_iter_max=100, dd_err_max=1e-13)
        out.put((rank, part.gid, phi[0].numpy().copy(), it, err, phi2[0].numpy().copy(), it2, sweeps2))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("world", [2, 4])
def test_pbj_over_gloo_ranks_matches_one_process(built, workdir, world):
    """One partition per gloo rank (2 ranks: one neighbour each; 4: two
    each, exchanged in increasing neighbour order, which no pair of ranks
    can deadlock).  With two ranks the all-reduced sums are the one
    process's, bit for bit; with four, gloo may add the ranks' partial sums
    in another order, so a change within rounding of the tolerance may end
    one iteration apart (then phi agrees to the tolerance)."""
    from tycho2_b200.partitions import PartitionSet, pbj, pbj_si
    path, _ = partitions_fixture(workdir, world)
    port = _free_port()
    ctx = mp.get_context("spawn")
    qu = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, path, qu)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = {}
    for _ in range(world):
        r = qu.get(timeout=240)
        got[r[0]] = r[1:]
    for pr in procs:
        pr.join(timeout=30)
        assert pr.exitcode == 0
    ps = PartitionSet(_oracle_parts(path, world))
    phi, it, err = pbj_si(ps, dd_iter_max=400, dd_err_max=1e-12)
    ps2 = PartitionSet(_oracle_parts(path, world))
    phi2, it2, err2, sweeps2 = pbj(ps2, iter_max=400, err_max=1e-12, dd_iter_max=100, dd_err_max=1e-13)
    for r in range(world):
        gid, p_si, it_si, err_si, p_pbj, it_pbj, sw_pbj = got[r]
        assert np.array_equal(gid, ps.parts[r].gid)
        if world == 2 or it_si == it:
            assert it_si == it and bits_equal(p_si, phi[r].numpy())
        else:
            assert abs(it_si - it) <= 1 and rel_l1(p_si, phi[r].numpy()) <= 1e-11
        if world == 2 or (it_pbj, sw_pbj) == (it2, sweeps2):
            assert it_pbj == it2 and sw_pbj == sweeps2 and bits_equal(p_pbj, phi2[r].numpy())
        else:
            assert abs(it_pbj - it2) <= 1 and rel_l1(p_pbj, phi2[r].numpy()) <= 1e-11


@pytest.mark.timeout(300)
def test_krylov_forms_reach_the_single_partition_solution(built, workdir):
    """SourceIteration::krylov over the PBJ, PBJOuter and Schur sweeps
    (deck key SourceIteration false)."""
    from tycho2_b200.partitions import PartitionSet, pbj, pbj_outer, schur, source_krylov
    path, _ = partitions_fixture(workdir, 2)
    ref, it_ref = _single_partition_si(workdir)
    ps = PartitionSet(_oracle_parts(path, 2))
    phi, its, rn, sweeps = pbj(ps, iter_max=200, err_max=1e-12, dd_iter_max=200, dd_err_max=1e-13,
                               method="krylov")
    assert its < it_ref and sweeps > its
    assert rel_l1(_gather(ps.parts, phi), ref) <= 1e-10
    ps = PartitionSet(_oracle_parts(path, 2))
    phi, its, rn, sweeps = schur(ps, iter_max=200, err_max=1e-12, dd_iter_max=200, dd_err_max=1e-13,
                                 method="krylov")
    assert its < it_ref
    assert rel_l1(_gather(ps.parts, phi), ref) <= 1e-10
    ps = PartitionSet(_oracle_parts(path, 2))
    phi, outer, its = pbj_outer(ps, iter_max=200, err_max=1e-13, dd_iter_max=200, dd_err_max=1e-12,
                                method="krylov")
    assert outer > 1 and all(k > 0 for k in its)
    assert rel_l1(_gather(ps.parts, phi), ref) <= 1e-10
    with pytest.raises(ValueError):
        source_krylov(ps, "traverse")
