"""Multi-partition sweeps on the GPU.

A sweeper made from one partition of a 2- or 4-partition .pmesh reads the
incoming psi on faces toward other partitions from psiBound
(tycho_sweeper_set_psi_bound):
  - its FP64 sweep is bit-identical to the reference's Util::sweepLocal on
    that rank's partition (the psi hash recorded from ref_dump's sweep_local
    in tests/golden/partitions_ref.npz) and to the oracle, in every launch
    shape that the level schedule offers;
  - its FP32 sweep (slotted kernel, FP32 ghost rows) agrees with the oracle
    to FP32 rounding; an angle shard of a partition sweeps its directions
    bit for bit;
  - the device CommSides (side_pack / side_unpack) leaves psiBound
    bit-identical to the host restatement (tests/helpers.OraclePartition);
  - the PBJ and Schur drivers over the GPU partitions take the oracle
    partitions' iterations to the same phi, which is the single-partition
    solution;
  - the schedules and paths that cannot read ghost rows refuse such a
    sweeper.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, bits_equal, rel_l1
from helpers import OraclePartition, partition_inputs, partitions_fixture, psi_hash

pytestmark = pytest.mark.gpu

SHAPES = [
    None,                                   # default: compact records in registers, 2 octant chains
    ("levels", "records", 16, 0, 1),
    ("levels", "direct", 128, 0, 1),
    ("levels", "items", 2, 0, 1),
    ("levels", "tiles", 2, 0, 1),
    ("levels", "compact", -96, 0, 2),
]


@pytest.mark.parametrize("P", [2, 4])
def test_partition_sweep_bit_identical_to_reference(built, workdir, P):
    import tycho2_b200 as ty
    from oracle.oracle import Oracle, OracleMesh
    path, ref = partitions_fixture(workdir, P)
    for p in range(P):
        mesh = ty.TychoMesh.read_pmesh(path, p)
        o = Oracle(OracleMesh(path, p), 4, 3)
        st, src, pb = partition_inputs(mesh.n_cells, o.A, 3, mesh.n_sides, 10 * P + p)
        want = o.sweep_local(st, pb, src_ang=src)
        assert psi_hash(want) == int(ref["p%d_%d_psi_hash" % (P, p)][0])
        sw = ty.SweeperCuda(mesh, 4, 3)
        assert sw.n_bound_sides == mesh.n_bound_sides > 0
        sw.set_cross_sections(st, np.zeros_like(st))
        sw.set_psi_bound(pb)
        for shape in SHAPES:
            if shape is not None:
                sw.configure(0, *shape)
            psi = np.empty(o.psi_shape)
            sw.sweep(psi, src)
            assert bits_equal(psi, want), (P, p, shape)
        # the values held, and vacuum when asked for
        got = sw.get_psi_bound()
        side, rank, _ = mesh.side_tables()
        adj = mesh.tables()["adj_cell"]
        none = np.uint64(0xFFFFFFFFFFFFFFFF)
        bsides = side[(adj == none) & (rank != none) & (rank != np.uint64(p))].astype(np.int64)
        assert bits_equal(got[bsides], pb[bsides])
        others = np.setdiff1d(np.arange(mesh.n_sides), bsides)
        assert not got[others].any()
        psi0 = np.empty(o.psi_shape)
        sw.sweep(psi0, src, zeroPsiBound=True)
        assert bits_equal(psi0, o.sweep_local(st, np.zeros_like(pb), src_ang=src))
        sw.sweep(psi, src)
        assert bits_equal(psi, want)
        sw.close()


def test_partition_fp32_sweep_and_angle_shard(built, workdir):
    import torch
    import tycho2_b200 as ty
    from oracle.oracle import Oracle, OracleMesh
    path, _ = partitions_fixture(workdir, 4)
    for p in range(4):
        mesh = ty.TychoMesh.read_pmesh(path, p)
        G = 4
        o = Oracle(OracleMesh(path, p), 4, G)
        st, _, pb = partition_inputs(mesh.n_cells, o.A, G, mesh.n_sides, 70 + p)
        q = 0.5 + np.arange(mesh.n_cells * 4 * G).reshape(mesh.n_cells, 4, G) % 13 / 10.0
        want = o.sweep_local(st, pb, src_iso=np.ascontiguousarray(q))
        phi_want = o.psi_to_phi(want)
        sw = ty.SweeperCuda(mesh, 4, G, fp32=True)
        sw.set_cross_sections(st, np.zeros_like(st))
        sw.set_source(q, "isotropic")
        sw.set_psi_bound(pb)
        out = torch.empty(sw.phi_shape, dtype=torch.float64, device="cuda")
        sw.apply(None, out, precision=0)
        assert bits_equal(out.cpu().numpy(), phi_want)
        sw.apply(None, out, precision=1)  # FP32 slotted kernel, FP32 ghost rows
        assert rel_l1(out.cpu().numpy(), phi_want) <= 2e-6
        sw.configure(1, "levels", "compact", -172, 4, 2)
        sw.apply(None, out, precision=1)
        assert rel_l1(out.cpu().numpy(), phi_want) <= 2e-6
        sw.close()
        # directions 8..24 of the same partition
        sh = ty.SweeperCuda(mesh, 4, G, angles=(8, 24))
        sh.set_cross_sections(st, np.zeros_like(st))
        sh.set_psi_bound(pb)
        src = np.ascontiguousarray(np.broadcast_to(q[:, None], (mesh.n_cells, 16, 4, G)))
        psi = np.empty(src.shape)
        sh.sweep(psi, src)
        assert bits_equal(psi, want[:, 8:24])
        sh.close()


def _parts(path, P, kind, sn=4, G=2):
    import tycho2_b200 as ty
    from tycho2_b200.partitions import GpuPartition
    from test_partitions import _problem
    st, ss, mat, q = _problem(P, G)
    parts = []
    for p in range(P):
        if kind == "oracle":
            parts.append(OraclePartition(path, p, sn, G, st, ss, mat, q))
            continue
        mesh = ty.TychoMesh.read_pmesh(path, p)
        gid = mesh.tables()["cell_gid"].astype(np.int64)
        sw = ty.SweeperCuda(mesh, sn, G)
        sw.set_cross_sections(st[gid], ss[gid], mat)
        sw.set_source(np.ascontiguousarray(q[gid]), "isotropic")
        parts.append(GpuPartition(sw))
    return parts


@pytest.mark.parametrize("P", [2, 4])
def test_device_exchange_matches_commsides(built, workdir, P):
    import torch
    from tycho2_b200.partitions import PartitionSet
    path, _ = partitions_fixture(workdir, P)
    gpu = PartitionSet(_parts(path, P, "gpu"))
    ora = PartitionSet(_parts(path, P, "oracle"))
    for g, o in zip(gpu.parts, ora.parts):
        assert g.neighbours == o.neighbours
        for q in g.neighbours:
            n_send, n_recv = g.sw.side_counts(q)
            gs, an = g.send_list(q)
            ogs, oan = o.send_list(q)
            assert np.array_equal(gs, ogs) and np.array_equal(an, oan) and n_send == gs.size
            # what q receives from here is what q counts as its receives
            assert gpu.parts[q].sw.side_counts(g.partition)[1] == n_send
    phis = [torch.zeros(p.sw.phi_shape, dtype=torch.float64, device="cuda") for p in gpu.parts]
    ophis = [p.phi_zeros() for p in ora.parts]
    for step in range(3):
        for part, a in zip(gpu.parts, phis):
            part.apply(a.clone(), a, True)
        for part, a in zip(ora.parts, ophis):
            part.apply(a.clone(), a, True)
        gpu.exchange()
        ora.exchange()
        for g, o, a, b in zip(gpu.parts, ora.parts, phis, ophis):
            assert bits_equal(a.cpu().numpy(), b.numpy()), step
            assert bits_equal(g.sw.get_psi_bound(), o.pb), step
    gpu.close()


@pytest.mark.timeout(600)
def test_pbj_solvers_on_the_gpu_match_the_oracle(built, workdir):
    from tycho2_b200.partitions import PartitionSet, pbj, pbj_outer, pbj_si, schur, schur_krylov, schur_outer

    def pbj_krylov(ps, **kw):
        return pbj(ps, method="krylov", **kw)

    from test_partitions import _gather, _single_partition_si
    path, _ = partitions_fixture(workdir, 4)
    ref, it_ref = _single_partition_si(workdir)
    for solver, kw in ((pbj_si, dict(dd_iter_max=400, dd_err_max=1e-12)),
                       (pbj, dict(iter_max=400, err_max=1e-12, dd_iter_max=100, dd_err_max=1e-13)),
                       (pbj_outer, dict(iter_max=400, err_max=1e-13, dd_iter_max=100, dd_err_max=1e-12)),
                       (schur, dict(iter_max=400, err_max=1e-12, dd_iter_max=200, dd_err_max=1e-13)),
                       (schur_krylov, dict(dd_iter_max=400, dd_err_max=1e-13)),
                       (schur_outer, dict(iter_max=400, err_max=1e-13, dd_iter_max=100, dd_err_max=1e-12)),
                       (pbj_krylov, dict(iter_max=200, err_max=1e-12, dd_iter_max=200, dd_err_max=1e-13))):
        gpu = PartitionSet(_parts(path, 4, "gpu"))
        ora = PartitionSet(_parts(path, 4, "oracle"))
        rg = solver(gpu, **kw)
        ro = solver(ora, **kw)
        phi_g = _gather(gpu.parts, [x.cpu() for x in rg[0]])
        phi_o = _gather(ora.parts, ro[0])
        # iteration counts (pbj_si: iterations; pbj: source iterations and
        # local sweeps; pbj_outer: outer iterations and source iterations of
        # each); the L1 sums run in another order on the device, so a change
        # within rounding of a tolerance may end one iteration apart
        counts = {pbj_si: lambda r: (r[1],), pbj: lambda r: (r[1], r[3]), pbj_outer: lambda r: (r[1], r[2]),
                  schur: lambda r: (r[1], r[3]), schur_krylov: lambda r: (r[1],),
                  schur_outer: lambda r: (r[1], r[3][0], tuple(r[3][1]), r[3][2]),
                  pbj_krylov: lambda r: (r[1], r[3])}[solver]
        if solver is pbj_krylov:
            # GMRES on phi: its inner products are summed on the device for
            # GPU partitions and on the host for the oracle's, so the iterates
            # agree to rounding, not bit for bit
            assert abs(rg[1] - ro[1]) <= 1 and rel_l1(phi_g, phi_o) <= 1e-11, solver.__name__
        elif counts(rg) == counts(ro):
            assert bits_equal(phi_g, phi_o), solver.__name__
        else:
            assert abs(rg[1] - ro[1]) <= 1, (solver.__name__, counts(rg), counts(ro))
        assert rel_l1(phi_g, ref) <= 1e-10, solver.__name__
        gpu.close()


def test_partition_sweeper_refusals(built, workdir):
    import tycho2_b200 as ty
    path, _ = partitions_fixture(workdir, 2)
    mesh = ty.TychoMesh.read_pmesh(path, 0)
    sw = ty.SweeperCuda(mesh, 4, 2)
    st = np.ones(mesh.n_cells)
    sw.set_cross_sections(st, 0.5 * st)
    with pytest.raises(ty.TychoError, match="level schedule"):
        sw.configure(0, "dataflow", "tiles", 4)
    with pytest.raises(ty.TychoError, match="level schedule"):
        sw.configure(0, "persist", "records", 16)
    b = ty.BatchSolver(0)
    with pytest.raises(ty.TychoError, match="not in a batch"):
        b.add(sw, method="si")
    b.close()
    with pytest.raises(ty.TychoError):
        ty.SweeperCuda(mesh, 4, 2, schedule="dataflow")
    # the autotuner keeps to the level schedule
    sw.autotune(0, reps=1)
    assert sw.shape(0)["schedule"] == "levels"
    sw.close()


BIN = os.path.join(ROOT, "oracle", "_ref")


@pytest.mark.skipif(not os.path.exists(os.path.join(BIN, "sweep_cuda.x")),
                    reason="reference-side binding not built (needs the tycho2 tree at build time)")
def test_reference_adapter_sweep_local(built, workdir):
    """SweeperCuda.hh's sweepLocal inside the reference's own process
    (sweep_cuda.x sweep-local: its TychoMesh of one rank's partition, its
    PsiData and PsiBoundData): the psi of Util::sweepLocal, bit for bit."""
    from oracle.oracle import OracleMesh
    P = 4
    path, ref = partitions_fixture(workdir, P)
    d = os.path.join(str(workdir), "adapter_local")
    os.makedirs(d, exist_ok=True)
    deck = os.path.join(d, "local.deck")
    with open(deck, "w") as f:
        f.write("snOrder 4\niterMax 10\nerrMax 1e-10\nmaxCellsPerStep 100\nintraAngleP 3\ninterAngleP 1\n"
                "nGroups 3\nsigmaT1 1\nsigmaS1 0\nsigmaT2 1\nsigmaS2 0\nOutputFile false\n"
                "OutputFilename out.psi\nSourceIteration true\nMPIType TychoTwoSided\nDD_IterMax 100\n"
                "DD_ErrMax 1e-10\nSweepType Cuda\nGaussElim NoPivot\n")
    for p in range(P):
        om = OracleMesh(path, p)
        st, src, pb = partition_inputs(om.n_cells, 32, 3, om.n_sides, 10 * P + p)
        files = [os.path.join(d, n) for n in ("st.f64", "src.f64", "pb.f64", "psi.f64")]
        for arr, fn in zip((st, src, pb), files):
            arr.tofile(fn)
        env = dict(os.environ, TYCHO_SHIM_RANK=str(p), TYCHO_SHIM_SIZE=str(P))
        r = subprocess.run([os.path.join(BIN, "sweep_cuda.x"), path, deck, "sweep-local", *files], cwd=d,
                           env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        psi = np.fromfile(files[3])
        assert psi_hash(psi) == int(ref["p%d_%d_psi_hash" % (P, p)][0]), p


def _dist_worker(rank, world, port, path, out):
    import datetime
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    from tycho2_b200.partitions import DistributedPartitions, pbj_si
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        part = _parts(path, world, "gpu")[rank]
        phi, it, err = pbj_si(DistributedPartitions(part), dd_iter_max=400, dd_err_max=1e-12)
        out.put((rank, phi[0].cpu().numpy().copy(), it))
        part.sw.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(600)
def test_distributed_partitions_two_processes(built, workdir):
    """Two processes, one partition each, on the one GPU: their device
    sweeps never wait on each other (the packets go through gloo on the
    host between sweeps); they take the one-process GPU partition set's
    iterations to the same phi, bit for bit."""
    import socket
    import torch.multiprocessing as mp
    from tycho2_b200.partitions import PartitionSet, pbj_si
    path, _ = partitions_fixture(workdir, 2)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_dist_worker, args=(r, 2, port, path, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        r = q.get(timeout=500)
        got[r[0]] = r[1:]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ps = PartitionSet(_parts(path, 2, "gpu"))
    phi, it, err = pbj_si(ps, dd_iter_max=400, dd_err_max=1e-12)
    for r in range(2):
        assert got[r][1] == it and bits_equal(got[r][0], phi[r].cpu().numpy()), r
    ps.close()
