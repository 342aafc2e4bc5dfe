"""Parity of the B200 sweep (through the C ABI) with the oracle and the
reference's fixtures.  FP64: bit-identical psi.  FP32: relative error within
the tolerance stated in each test."""
import os

import numpy as np
import pytest

from conftest import bits_equal, rel_l1, rel_linf
from helpers import cube208, gold_psi, kuhn

pytestmark = pytest.mark.gpu


def make(mesh, sn, G, **kw):
    import tycho2_b200 as ty
    return ty.SweeperCuda(mesh, sn, G, **kw)


def test_fp64_sweep_bit_exact_vs_reference_fixture(built, kuhn3_ref):
    """One SweeperTraverse::sweep of the reference (S4, G=3, angular source)."""
    import tycho2_b200 as ty
    r = kuhn3_ref
    mesh = ty.TychoMesh.kuhn_cube(3, 0.05, 2024, 100.0)
    for shape in (("levels", "items", 1), ("levels", "items", 2), ("dataflow", "items", 4),
                  ("levels", "tiles", 4), ("dataflow", "tiles", 1), ("dataflow", "tiles", 2),
                  ("levels", "records", 8), ("dataflow", "records", 16), ("dataflow", "records", 32),
                  ("persist", "records", 8), ("persist", "records", 16), ("levels", "direct", 256),
                  ("levels", "compact", 128)):
        sw = make(mesh, 4, 3)
        sw.configure(0, *shape)
        sw.set_cross_sections(r["sweep_sigma_t"], np.zeros(mesh.n_cells))
        psi = np.empty(sw.psi_shape)
        sw.sweep(psi, r["sweep_source"])
        assert bits_equal(psi, r["sweep_psi"]), shape


@pytest.mark.parametrize("schedule,variant,vector", [
    ("levels", "items", 0), ("levels", "tiles", 0), ("levels", "records", 0), ("levels", "records", 1),
    ("dataflow", "items", 0), ("dataflow", "tiles", 0), ("dataflow", "records", 0),
    ("persist", "records", 0), ("persist", "records", 1), ("levels", "direct", 0), ("levels", "direct", 1),
    ("levels", "compact", 0), ("levels", "compact", 1), ("dataflow", "compact", 0), ("dataflow", "direct", 1),
    ("levels", "compact", 4)])
@pytest.mark.parametrize("n,jitter,sn,G,tpi", [
    (4, 0.05, 4, 1, 1), (5, 0.05, 8, 2, 2), (3, 0.0, 2, 3, 1), (6, 0.05, 6, 4, 4),
    (4, 0.07, 8, 8, 8), (2, 0.05, 4, 16, 16), (7, 0.05, 4, 5, 2), (1, 0.0, 4, 1, 1),
    (3, 0.05, 4, 64, 4), (2, 0.05, 4, 33, 1)])
def test_fp64_sweep_bit_exact_vs_oracle(built, workdir, n, jitter, sn, G, tpi, variant, schedule, vector):
    from oracle.oracle import Oracle
    mesh, om = kuhn(workdir, n, jitter, seed=5)
    o = Oracle(om, sn, G)
    rng = np.random.default_rng(n * 100 + G)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    src = rng.uniform(-0.2, 1.0, o.psi_shape)
    sw = make(mesh, sn, G)
    knob = {"items": tpi, "tiles": min(tpi, 4), "records": 8 if tpi <= 2 else (16 if tpi <= 4 else 32),
            "direct": 64 * min(tpi, 4) if tpi != 4 else 128}
    # compact: also the register-capped blocks (64 threads; at most 102, 85, 64 registers)
    knob["compact"] = {1: 64, 2: -96, 4: -80, 8: 256, 16: -64}[tpi]
    if vector == 4 and G % 4:
        pytest.skip("two 2-group vectors per task need nGroups divisible by 4")
    if vector == 4:
        knob["compact"] = 128  # two vectors per task: no register cap
    if schedule == "dataflow" and variant in ("direct", "compact"):
        vg = vector or (2 if G % 2 == 0 else 1)
        if (G // vg) & (G // vg - 1) or G // vg > 32:
            pytest.skip("direct dataflow needs nGroups / vector a power of two <= 32")
        knob[variant] = 128
    if schedule == "persist":
        knob["records"] = min(knob["records"], 16)  # two 32-item FP64 tiles exceed shared memory
    sw.configure(0, schedule, variant, knob[variant], vector)
    sw.set_cross_sections(st, np.zeros(mesh.n_cells))
    psi = np.empty(sw.psi_shape)
    sw.sweep(psi, src)
    assert bits_equal(psi, o.sweep(st, src_ang=src))
    sw.sweep(psi, src)  # a second sweep (next completion epoch) is identical
    assert bits_equal(psi, o.sweep(st, src_ang=src))


@pytest.mark.parametrize("streams", [2, 4, 8])
@pytest.mark.parametrize("variant,knob", [("compact", 64), ("direct", 128), ("records", 16), ("tiles", 4)])
def test_fp64_sweep_on_several_streams_bit_exact(built, workdir, streams, variant, knob):
    """Octant groups of every level on concurrent streams: the same psi."""
    from oracle.oracle import Oracle
    for n, sn, G in [(5, 8, 4), (3, 6, 2), (2, 4, 1)]:
        mesh, om = kuhn(workdir, n, 0.05, seed=31)
        o = Oracle(om, sn, G)
        rng = np.random.default_rng(n + G)
        st = rng.lognormal(0.0, 0.5, mesh.n_cells)
        src = rng.uniform(-0.2, 1.0, o.psi_shape)
        sw = make(mesh, sn, G)
        sw.configure(0, "levels", variant, knob, 0, streams)
        assert sw.shape(0)["streams"] == streams
        sw.set_cross_sections(st, np.zeros(mesh.n_cells))
        psi = np.empty(sw.psi_shape)
        sw.sweep(psi, src)
        assert bits_equal(psi, o.sweep(st, src_ang=src)), (n, sn, G)
        sw.close()


def test_fp64_operator_bit_exact_vs_oracle_downscatter(built, workdir):
    """phi_out = D L^-1 (Q_iso + M S phi_in) with a group-to-group matrix."""
    from oracle.oracle import Oracle
    from tycho2_b200 import problems
    mesh, om = kuhn(workdir, 5, 0.05, seed=8)
    G = 4
    o = Oracle(om, 4, G)
    rng = np.random.default_rng(3)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    mat = problems.downscatter_matrix(G, 0.6)
    q = rng.uniform(0.0, 1.0, o.phi_shape)
    sw = make(mesh, 4, G)
    sw.set_cross_sections(st, st, mat)
    sw.set_source(q, "isotropic")
    # Source iteration for 3 steps on both sides, bit for bit at every step.
    phi_o = np.zeros(o.phi_shape)
    for it in range(1, 4):
        iso = q + o.scatter(st, mat, phi_o)
        psi_o = o.sweep(st, src_iso=np.ascontiguousarray(iso))
        phi_o = o.psi_to_phi(psi_o)
        phi, psi, stats = sw.solve("si", iter_max=it, err_max=-1.0)
        assert stats["iterations"] == it
        assert bits_equal(psi, psi_o) and bits_equal(phi, phi_o), "step %d" % it


def test_gold_psi_source_iteration_on_gpu(built, workdir):
    """input-gold.deck end to end: SI to 1e-10 on cube-208, S8, G=2."""
    from oracle.oracle import Oracle
    mesh, om = cube208(workdir)
    o = Oracle(om, 8, 2)
    st = np.full(mesh.n_cells, 10.0)
    ss = np.full(mesh.n_cells, 5.0)
    src = o.hat_source(st, ss)
    sw = make(mesh, 8, 2)
    sw.set_cross_sections(st, ss)
    sw.set_source(src, "angular")
    phi, psi, stats = sw.solve("si", iter_max=100, err_max=1e-10)
    gold = gold_psi()
    assert stats["iterations"] == 34
    assert rel_l1(psi, gold) < 1e-10 and rel_linf(psi, gold) < 1e-10
    psi_o, phi_o, it_o, _ = o.source_iteration(st, ss, q_ang=src, err_max=1e-10)
    assert it_o == 34
    assert rel_l1(psi, psi_o) <= 1e-12
    path = os.path.join(str(workdir), "gpu.psi")
    sw.writePsiToFile(path)
    v = np.fromfile(path)[8:]
    assert rel_l1(v, gold.ravel()) < 1e-10 and rel_linf(v, gold.ravel()) < 1e-10


def test_gold_psi_krylov_on_gpu(built, workdir):
    """input-gold-krylov.deck: the Krylov path reproduces gold.psi at 1e-10."""
    from oracle.oracle import Oracle
    mesh, om = cube208(workdir)
    o = Oracle(om, 8, 2)
    st = np.full(mesh.n_cells, 10.0)
    ss = np.full(mesh.n_cells, 5.0)
    sw = make(mesh, 8, 2)
    sw.set_cross_sections(st, ss)
    sw.set_source(o.hat_source(st, ss), "angular")
    phi, psi, stats = sw.solve("gmres", iter_max=100, err_max=1e-10, restart=30)
    gold = gold_psi()
    assert rel_l1(psi, gold) < 1e-10 and rel_linf(psi, gold) < 1e-10


def test_si_matches_reference_fixture(built, kuhn3_ref):
    """SourceIteration::fixedPoint of the reference (hat source, per-cell sigma)."""
    import tycho2_b200 as ty
    from tycho2_b200 import problems
    r = kuhn3_ref
    mesh = ty.TychoMesh.kuhn_cube(3, 0.05, 2024, 100.0)
    sw = make(mesh, 4, 2)
    sw.set_cross_sections(r["si_sigma_t"], r["si_sigma_s"])
    sw.set_source(problems.hat_source(mesh, sw.quadrature, r["si_sigma_t"], r["si_sigma_s"], 2), "angular")
    phi, psi, stats = sw.solve("si", iter_max=100, err_max=1e-12)
    assert rel_l1(psi, r["si_psi"]) <= 1e-12


def test_kuhn8_s4_workload_matches_oracle(built, workdir):
    """The 3,072-tet S4 G=1 workload: SI to 1e-10 on GPU and oracle."""
    from oracle.oracle import Oracle
    from tycho2_b200 import problems
    w = problems.WORKLOADS["kuhn8_s4_g1"]
    mesh, st, ss, mat, q = problems.make_problem(**w)
    path = os.path.join(str(workdir), "k8.pmesh")
    mesh.write_pmesh(path)
    from oracle.oracle import OracleMesh
    o = Oracle(OracleMesh(path), 4, 1)
    psi_o, phi_o, it_o, _ = o.source_iteration(st, ss, q_iso=q, err_max=1e-10)
    sw = make(mesh, 4, 1)
    sw.set_cross_sections(st, ss, mat)
    sw.set_source(q, "isotropic")
    phi, psi, stats = sw.solve("si", iter_max=100, err_max=1e-10)
    assert abs(stats["iterations"] - it_o) <= 1
    assert rel_l1(phi, phi_o) <= 1e-12 and rel_l1(psi, psi_o) <= 1e-12


def test_fp32_sweep_within_tolerance(built, workdir):
    """FP32 sweep vs FP64 oracle: relative L1 error of psi <= 1e-6."""
    from oracle.oracle import Oracle
    from tycho2_b200 import problems
    mesh, om = kuhn(workdir, 6, 0.05, seed=9)
    G = 8
    o = Oracle(om, 8, G)
    rng = np.random.default_rng(4)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    mat = problems.downscatter_matrix(G, 0.6)
    q = rng.uniform(0.0, 1.0, o.phi_shape)
    psi_ref, phi_ref, _, _ = o.krylov(st, st, mat, q_iso=q, restart=20, iter_max=200, rtol=1e-11)
    for shape in (("levels", "items", 1), ("levels", "items", 8), ("dataflow", "items", 4),
                  ("levels", "tiles", 2), ("dataflow", "tiles", 4), ("levels", "records", 16),
                  ("dataflow", "records", 32), ("persist", "records", 8), ("persist", "records", 32),
                  ("levels", "records", 16, 1), ("levels", "records", 16, 2), ("levels", "direct", 128),
                  ("levels", "direct", 64, 1), ("levels", "compact", 64), ("levels", "compact", 128, 2),
                  ("dataflow", "compact", 128), ("dataflow", "direct", 128, 2), ("levels", "compact", 64, 8),
                  ("levels", "direct", 128, 8), ("levels", "compact", 64, 4, 8), ("levels", "compact", 64, 2, 2),
                  ("levels", "compact", -96, 4, 2), ("levels", "direct", -96, 4), ("levels", "compact", -80, 4),
                  ("levels", "direct", -64, 2, 2), ("levels", "compact", -180, 4, 2), ("levels", "direct", -196, 2),
                  ("levels", "compact", -196, 4), ("levels", "compact", -172, 4, 2), ("levels", "direct", -180, 4)):
        sw = make(mesh, 8, G, fp32=True)
        sw.configure(1, *shape)
        sw.set_cross_sections(st, st, mat)
        sw.set_source(q, "isotropic")
        # The FP32 operator inside FP64 refinement: converged phi within 1e-8.
        phi, psi, stats = sw.solve("mixed", iter_max=200, err_max=1e-11, restart=20)
        assert rel_l1(phi, phi_ref) <= 1e-8, shape
        assert stats["sweeps_fp32"] > stats["sweeps_fp64"]
        sw.close()


def test_mixed_vs_fp64_gmres_and_si(built, workdir):
    from oracle.oracle import Oracle
    from tycho2_b200 import problems
    mesh, om = kuhn(workdir, 6, 0.05, seed=10)
    G = 4
    rng = np.random.default_rng(5)
    st = rng.lognormal(0.0, 1.0, mesh.n_cells)
    mat = problems.downscatter_matrix(G, 0.95)
    q = np.ones((mesh.n_cells, 4, G))
    sw = make(mesh, 4, G, fp32=True)
    sw.set_cross_sections(st, st, mat)
    sw.set_source(q, "isotropic")
    phi64, psi64, s64 = sw.solve("gmres", iter_max=300, err_max=1e-12, restart=30)
    phim, psim, sm = sw.solve("mixed", iter_max=300, err_max=1e-11, restart=30)
    assert rel_l1(phim, phi64) <= 1e-8
    assert sm["refinements"] >= 1 and sm["sweeps_fp32"] > 0
    o = Oracle(om, 4, G)
    psi_o, phi_o, its, _ = o.krylov(st, st, mat, q_iso=q, restart=30, iter_max=300, rtol=1e-12)
    assert rel_l1(phi64, phi_o) <= 1e-10


def test_zero_source_gives_zero_psi(built, workdir):
    mesh, _ = kuhn(workdir, 3, 0.05, seed=1)
    sw = make(mesh, 4, 2)
    sw.set_cross_sections(np.ones(mesh.n_cells), np.zeros(mesh.n_cells))
    psi = np.full(sw.psi_shape, 7.0)
    sw.sweep(psi, np.zeros(sw.psi_shape))
    assert np.all(psi == 0.0)


def test_pure_streaming_void(built, workdir):
    """sigma_t = 0 everywhere: psi stays finite and matches the oracle."""
    from oracle.oracle import Oracle
    mesh, om = kuhn(workdir, 4, 0.05, seed=2)
    o = Oracle(om, 4, 1)
    st = np.zeros(mesh.n_cells)
    src = np.ones(o.psi_shape)
    sw = make(mesh, 4, 1)
    sw.set_cross_sections(st, st)
    psi = np.empty(sw.psi_shape)
    sw.sweep(psi, src)
    assert np.all(np.isfinite(psi))
    assert bits_equal(psi, o.sweep(st, src_ang=src))


def test_missing_inputs_are_errors(built, workdir):
    import tycho2_b200 as ty
    mesh, _ = kuhn(workdir, 2, 0.0, seed=1)
    sw = make(mesh, 4, 1)
    with pytest.raises(ty.TychoError) as e:
        sw.solve("si")
    assert e.value.status == 10
    sw.set_cross_sections(np.ones(mesh.n_cells), np.full(mesh.n_cells, 0.5))
    with pytest.raises(ty.TychoError) as e:
        sw.solve("mixed")  # created without the FP32 sweep
    assert e.value.status == 1
    # Like SourceIteration::fixedPoint, hitting iterMax is not an error: the
    # caller reads the last relative change.
    sw.set_source(np.ones(sw.phi_shape), "isotropic")
    phi, psi, stats = sw.solve("si", iter_max=2, err_max=1e-30)
    assert stats["iterations"] == 2 and stats["final_error"] > 1e-30


def test_autotune_keeps_results_bit_exact(built, workdir):
    """Whatever launch shape the autotuner picks, the FP64 sweep is unchanged."""
    from oracle.oracle import Oracle
    mesh, om = kuhn(workdir, 6, 0.05, seed=12)
    G = 4
    o = Oracle(om, 8, G)
    rng = np.random.default_rng(12)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    src = rng.uniform(0.0, 1.0, o.psi_shape)
    sw = make(mesh, 8, G, fp32=True)
    sw.set_cross_sections(st, np.zeros(mesh.n_cells))
    best64 = sw.autotune(0, reps=2)
    best32 = sw.autotune(1, reps=2)
    assert best64["variant"] in ("items", "tiles", "records", "direct", "compact") and best32["schedule"] in ("levels", "dataflow", "persist")
    assert sw.shape(0) == {k: best64[k] for k in ("schedule", "variant", "knob", "vector", "streams")}
    psi = np.empty(sw.psi_shape)
    sw.sweep(psi, src)
    assert bits_equal(psi, o.sweep(st, src_ang=src))


@pytest.mark.parametrize("kind", ["Original", "CramerGlu", "CramerIntel"])
def test_fp64_sweep_other_solvers_bit_exact(built, workdir, kuhn3_ref, kind):
    """GaussElim Original / CramerGlu / CramerIntel: the reference's own sweep
    (fixture) and the oracle, bit for bit, in both direct record forms."""
    import tycho2_b200 as ty
    from oracle.oracle import Oracle
    r = kuhn3_ref
    mesh = ty.TychoMesh.kuhn_cube(3, 0.05, 2024, 100.0)
    src1 = np.ascontiguousarray(r["sweep_source"][..., :1])
    for variant, streams in (("compact", 1), ("direct", 2)):
        sw = ty.SweeperCuda(mesh, 4, 1, gauss_elim=kind)
        assert sw.shape(0)["variant"] == "compact"  # the default for these solvers
        sw.configure(0, "levels", variant, 128, 0, streams)
        sw.set_cross_sections(r["sweep_sigma_t"], np.zeros(mesh.n_cells))
        psi = np.empty(sw.psi_shape)
        sw.sweep(psi, src1)
        assert bits_equal(psi, r["sweep_psi_" + kind]), (kind, variant)
        sw.close()
    for n, sn, G in [(4, 8, 4), (3, 6, 3)]:
        mesh, om = kuhn(workdir, n, 0.05, seed=77)
        o = Oracle(om, sn, G, gauss_elim=kind)
        rng = np.random.default_rng(n * G)
        st = rng.lognormal(0.0, 0.5, mesh.n_cells)
        src = rng.uniform(-0.2, 1.0, o.psi_shape)
        for variant in ("compact", "direct"):
            sw = ty.SweeperCuda(mesh, sn, G, gauss_elim=kind)
            sw.configure(0, "levels", variant, 128)
            sw.set_cross_sections(st, np.zeros(mesh.n_cells))
            psi = np.empty(sw.psi_shape)
            sw.sweep(psi, src)
            assert bits_equal(psi, o.sweep(st, src_ang=src)), (kind, variant, n, sn, G)
            sw.close()


def test_other_solvers_reject_unsupported_shapes(built, workdir):
    import tycho2_b200 as ty
    mesh, _ = kuhn(workdir, 2, 0.05, seed=1)
    sw = ty.SweeperCuda(mesh, 4, 2, gauss_elim="Original")
    for shape in (("levels", "tiles", 4), ("dataflow", "compact", 128), ("levels", "compact", 64),
                  ("levels", "records", 16)):
        with pytest.raises(ty.TychoError):
            sw.configure(0, *shape)
    with pytest.raises(ty.TychoError):
        ty.SweeperCuda(mesh, 4, 2, gauss_elim="CramerGlu", schedule="dataflow")
    sw.close()


@pytest.mark.parametrize("kind", ["Original", "CramerIntel"])
def test_fp32_other_solvers_within_tolerance(built, workdir, kind):
    from oracle.oracle import Oracle
    import tycho2_b200 as ty
    mesh, om = kuhn(workdir, 5, 0.05, seed=9)
    G = 4
    o = Oracle(om, 8, G, gauss_elim=kind)
    rng = np.random.default_rng(5)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    src = rng.uniform(0.0, 1.0, (mesh.n_cells, 4, G))
    sw = ty.SweeperCuda(mesh, 8, G, fp32=True, gauss_elim=kind)
    sw.set_cross_sections(st, 0.5 * st)
    sw.set_source(src, "isotropic")
    phi, _, stats = sw.solve("mixed", iter_max=200, err_max=1e-12)
    assert stats["sweeps_fp32"] > 0
    _, phi_ref, _, _ = o.source_iteration(st, 0.5 * st, q_iso=src, iter_max=400, err_max=1e-13)
    assert rel_l1(phi, phi_ref) <= 1e-8
    sw.close()


@pytest.mark.parametrize("n,jitter,sn", [(3, 0.05, 4), (6, 0.05, 8), (4, 0.0, 6), (9, 0.05, 8), (1, 0.0, 2)])
def test_device_levelling_equals_host(built, workdir, n, jitter, sn):
    """The wavefront schedule levelled on the device: the same t-levels, item
    order, segment offsets and incoming-face count as the host levelling."""
    import tycho2_b200 as ty
    mesh, _ = kuhn(workdir, n, jitter, seed=41)
    host = ty.SweeperCuda(mesh, sn, 1, levelling="host")
    dev = ty.SweeperCuda(mesh, sn, 1, levelling="device")
    assert host.schedule_info() == dev.schedule_info()
    ih, oh = host.schedule_arrays()
    idv, odv = dev.schedule_arrays()
    assert np.array_equal(ih, idv) and np.array_equal(oh, odv)
    assert host.launches(0) == dev.launches(0)
    host.close()
    dev.close()


def test_pool_memory_reused_and_released(built, workdir):
    """Sweepers take device memory from the library's pool: a second sweeper
    reuses what the first freed, the pool can be trimmed, and results do not
    depend on either."""
    import tycho2_b200 as ty
    mesh, _ = kuhn(workdir, 5, 0.05, seed=3)
    rng = np.random.default_rng(8)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    psis = []
    for trim in (False, True, False):
        sw = make(mesh, 8, 4)
        sw.set_cross_sections(st, np.zeros(mesh.n_cells))
        src = np.random.default_rng(1).uniform(0.0, 1.0, sw.psi_shape)
        psi = np.empty(sw.psi_shape)
        sw.sweep(psi, src)
        psis.append(psi)
        sw.close()
        if trim:
            ty.release_cached_memory(0)
    assert bits_equal(psis[0], psis[1]) and bits_equal(psis[0], psis[2])


@pytest.mark.parametrize("n,G,chunks,locked", [(8, 8, 4, "both"), (12, 3, 4, "both"), (16, 16, 16, "both"),
                                               (8, 8, 4, "none"), (12, 3, 4, "psi"), (16, 16, 16, "source"),
                                               (16, 16, 16, "none")])
def test_dropin_sweep_in_angle_chunks_bit_exact(built, workdir, n, G, chunks, locked):
    """The drop-in sweep of a large psi (64 MiB and up) moves and sweeps K
    contiguous angle ranges so that its host copies overlap the sweep;
    page-locked host buffers are copied directly, pageable ones through
    page-locked staging pieces of 64 MiB (two pieces per chunk at 16^3 G=16):
    psi bit-identical to the oracle's, on two calls in a row and after a
    solve on the same sweeper."""
    import torch
    from oracle.oracle import Oracle
    mesh, om = kuhn(workdir, n, 0.05, seed=23)
    o = Oracle(om, 8, G)
    rng = np.random.default_rng(n * G)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    sw = make(mesh, 8, G)
    assert mesh.n_cells * 128 * 4 * G * 8 >= (64 << 20) * (16 if chunks == 16 else 1)
    sw.set_cross_sections(st, np.zeros(mesh.n_cells))
    src0 = rng.uniform(-0.2, 1.0, o.psi_shape)
    ref = o.sweep(st, src_ang=src0)
    def buffer(lock):
        if lock:
            return torch.empty(o.psi_shape, dtype=torch.float64, pin_memory=True).numpy()
        return np.empty(o.psi_shape)
    src = buffer(locked in ("both", "source"))
    psi = buffer(locked in ("both", "psi"))
    src[...] = src0
    for _ in range(2):
        psi[...] = np.nan
        sw.sweep(psi, src)
        assert bits_equal(psi, ref)
    sw.set_source(np.ones(sw.phi_shape), "isotropic")
    sw.solve("si", iter_max=2, err_max=-1.0, want_psi=False)
    psi[...] = np.nan
    sw.sweep(psi, src)
    assert bits_equal(psi, ref)
    sw.close()


def test_invalid_arguments_are_errors(built, workdir):
    """Bad sizes and launch shapes come back as TYCHO_ERR_ARG (status 1),
    never as a fault: 0 or 65 groups, an SN order without a quadrature table,
    a knob, vector width or stream count the kernels do not have."""
    import tycho2_b200 as ty
    mesh, _ = kuhn(workdir, 2, 0.05, seed=3)
    for sn, G in ((4, 0), (4, 65), (3, 1), (0, 1)):
        with pytest.raises(ty.TychoError) as e:
            make(mesh, sn, G)
        assert e.value.status == 1, (sn, G)
    sw = make(mesh, 4, 4, fp32=True)
    for args in (("levels", "compact", 96), ("levels", "direct", -72), ("levels", "compact", 64, 3),
                 ("levels", "compact", 64, 2, 3), ("dataflow", "tiles", 4, 0, 2), ("persist", "direct", 64),
                 ("levels", "compact", -180, 1)):
        for prec in (0, 1):
            with pytest.raises(ty.TychoError) as e:
                sw.configure(prec, *args)
            assert e.value.status == 1, (prec, args)
    sw.configure(1, "levels", "compact", -96, 4, 2)  # still usable after the refusals
    sw.set_cross_sections(np.ones(mesh.n_cells), np.full(mesh.n_cells, 0.5))
    sw.set_source(np.ones(sw.phi_shape), "isotropic")
    phi, _, _ = sw.solve("mixed", iter_max=50, err_max=1e-10, want_psi=False)
    assert np.all(np.isfinite(phi))
    sw.close()


def test_fp64_refuses_slotted_rows(built, workdir):
    """The slotted upwind rows change the summation order, so they exist for
    the FP32 sweep only; the FP64 sweep keeps the reference's order."""
    import tycho2_b200 as ty
    mesh, _ = kuhn(workdir, 2, 0.05, seed=3)
    sw = make(mesh, 4, 4, fp32=True)
    for knob in (-196, -180, -172):
        with pytest.raises(ty.TychoError) as e:
            sw.configure(0, "levels", "compact", knob, 2)
        assert e.value.status == 1
        sw.configure(1, "levels", "compact", knob, 4)
    assert sw.shape(1)["knob"] == -172
    sw.close()


@pytest.mark.parametrize("order", ["blevel", "random", "cell"])
def test_work_orders_permute_each_segment_and_keep_psi(built, workdir, order):
    """The reference's traversal priorities as work orders of the level
    schedule (tycho_sweeper_set_work_order): each (level, octant) segment
    holds the same items in another order -- for 'blevel' in non-increasing
    b-level, the reference's Priorities -- and the FP64 psi stays
    bit-identical to the oracle's under every schedule that takes items in
    that order."""
    from oracle.oracle import Oracle
    mesh, om = kuhn(workdir, 5, 0.05, seed=37)
    sn, G = 8, 4
    o = Oracle(om, sn, G)
    rng = np.random.default_rng(77)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    src = rng.uniform(-0.2, 1.0, o.psi_shape)
    ref = o.sweep(st, src_ang=src)
    sw = make(mesh, sn, G, levelling="host")
    sw.set_cross_sections(st, np.zeros(mesh.n_cells))
    items0, off0 = sw.schedule_arrays()
    sw.set_work_order(order)
    items1, off1 = sw.schedule_arrays()
    assert np.array_equal(off0, off1)
    for b, e in zip(off0[:-1], off0[1:]):
        assert np.array_equal(np.sort(items0[b:e]), np.sort(items1[b:e]))
    if order == "blevel":
        _, _, blev, _ = mesh.levels(sn)
        A = 2 * sn * sn
        for b, e in zip(off1[:-1], off1[1:]):
            seg = items1[b:e]
            seg = seg[seg != 0xFFFFFFFF]
            key = blev[seg % A, seg // A]
            # within each octant group of the level: non-increasing b-level
            octs = np.array([int(o.quadrature()[0][a] < 0) * 4 + int(o.quadrature()[1][a] < 0) * 2
                             + int(o.quadrature()[2][a] < 0) for a in seg % A])
            for oc in np.unique(octs):
                k = key[octs == oc]
                assert np.all(np.diff(k.astype(np.int64)) <= 0)
    for shape in (("levels", "compact", 128), ("levels", "direct", 256), ("dataflow", "records", 16),
                  ("persist", "records", 16), ("dataflow", "tiles", 2)):
        sw.configure(0, *shape)
        psi = np.full(sw.psi_shape, np.nan)
        sw.sweep(psi, src)
        assert bits_equal(psi, ref), (order, shape)
    sw.close()
