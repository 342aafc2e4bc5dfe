"""Pins the CPU oracle (oracle/tycho_oracle.c) to the reference before it is
trusted as the checker of the B200 sweep:
  - the reference's own regression vector test/regression/gold.psi, with its
    own criterion (L1 and Linf relative error < 1e-10, test/diff.py:42-56);
  - what the reference computes on a jittered Kuhn mesh (fixture made by
    tests/golden/make_golden.py from the reference built from source):
    tables, one sweep and a source iteration, bit for bit;
  - the reference build itself, when oracle/_ref is present (this container).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, bits_equal, rel_l1, rel_linf
from helpers import cube208, gold_psi


def test_gold_psi_source_iteration(built, workdir):
    from oracle.oracle import Oracle
    _, om = cube208(workdir)
    o = Oracle(om, 8, 2)
    st = np.full(om.n_cells, 10.0)
    ss = np.full(om.n_cells, 5.0)
    src = o.hat_source(st, ss)
    psi, phi, iters, err = o.source_iteration(st, ss, q_ang=src, iter_max=100, err_max=1e-10)
    gold = gold_psi()
    assert iters == 34  # what the reference prints for input-gold.deck
    assert rel_l1(psi, gold) < 1e-10 and rel_linf(psi, gold) < 1e-10
    # The gold file came from another compiler; the restatement is within a
    # few ulps of it.
    assert rel_l1(psi, gold) < 1e-14


def test_gold_psi_krylov(built, workdir):
    """input-gold-krylov.deck reproduces the same gold.psi at 1e-10."""
    from oracle.oracle import Oracle
    _, om = cube208(workdir)
    o = Oracle(om, 8, 2)
    st = np.full(om.n_cells, 10.0)
    ss = np.full(om.n_cells, 5.0)
    src = o.hat_source(st, ss)
    psi, phi, its, rn = o.krylov(st, ss, q_ang=src, restart=30, iter_max=100, rtol=1e-10)
    gold = gold_psi()
    assert rel_l1(psi, gold) < 1e-10 and rel_linf(psi, gold) < 1e-10


def test_oracle_tables_match_reference(built, workdir, kuhn3_ref):
    from oracle.oracle import Oracle, OracleMesh
    import tycho2_b200 as ty
    mesh = ty.TychoMesh.kuhn_cube(3, 0.05, 2024, 100.0)
    path = os.path.join(str(workdir), "k3.pmesh")
    mesh.write_pmesh(path)
    om = OracleMesh(path)
    t = om.tables()
    r = kuhn3_ref
    assert np.array_equal(t["adj_cell"].ravel(), r["s4_adj"])
    assert np.array_equal(t["neighbor_vrtx"].ravel(), r["s4_nbr"])
    assert np.array_equal(t["face_to_cell"].ravel(), r["s4_f2c"])
    assert np.array_equal(t["cell_to_face"].ravel(), r["s4_c2f"])
    assert bits_equal(t["volume"], r["s4_vol"])
    assert bits_equal(t["area"].ravel(), r["s4_area"])
    for sn in (4, 8):
        o = Oracle(om, sn, 1)
        tl, deps, blev = o.levels()
        assert np.array_equal(deps.ravel().astype(np.uint64), r["s%d_deps" % sn])
        assert np.array_equal(blev.ravel().astype(np.uint64), r["s%d_blev" % sn])
        if sn == 4:
            assert bits_equal(o.omega_dot_n().ravel(), r["s4_odn"])


def test_oracle_sweep_and_si_match_reference(built, workdir, kuhn3_ref):
    from oracle.oracle import Oracle, OracleMesh
    import tycho2_b200 as ty
    mesh = ty.TychoMesh.kuhn_cube(3, 0.05, 2024, 100.0)
    path = os.path.join(str(workdir), "k3.pmesh")
    mesh.write_pmesh(path)
    om = OracleMesh(path)
    r = kuhn3_ref
    o = Oracle(om, 4, 3)
    psi = o.sweep(r["sweep_sigma_t"], src_ang=np.ascontiguousarray(r["sweep_source"]))
    assert bits_equal(psi, r["sweep_psi"])
    # the other 4x4 solvers of gaussElim4 (deck key GaussElim), bit for bit
    src1 = np.ascontiguousarray(r["sweep_source"][..., :1])
    for kind in ("Original", "CramerGlu", "CramerIntel"):
        psi = Oracle(om, 4, 1, gauss_elim=kind).sweep(r["sweep_sigma_t"], src_ang=src1)
        assert bits_equal(psi, r["sweep_psi_" + kind]), kind
    o = Oracle(om, 4, 2)
    src = o.hat_source(r["si_sigma_t"], r["si_sigma_s"])
    psi, phi, iters, err = o.source_iteration(r["si_sigma_t"], r["si_sigma_s"], q_ang=src,
                                              iter_max=100, err_max=1e-12)
    assert bits_equal(psi, r["si_psi"])


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "sweep.x")),
                    reason="reference build not present")
def test_oracle_bit_identical_to_reference_build(built, workdir):
    """The reference's own sweep.x on gold's deck vs the restatement."""
    from oracle.oracle import Oracle
    _, om = cube208(workdir)
    deck = os.path.join(str(workdir), "gold.deck")
    with open(deck, "w") as f:
        f.write("snOrder 8\niterMax 100\nerrMax 1e-10\nmaxCellsPerStep 100\nintraAngleP 3\n"
                "interAngleP 1\nnGroups 2\nsigmaT1 10\nsigmaS1 5\nsigmaT2 10\nsigmaS2 5\n"
                "OutputFile true\nOutputFilename out.psi\nSourceIteration true\n"
                "MPIType TychoTwoSided\nDD_IterMax 100\nDD_ErrMax 1e-10\n"
                "SweepType TraverseGraph\nGaussElim NoPivot\n")
    env = dict(os.environ, OMP_NUM_THREADS="2")
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", "sweep.x"),
                    os.path.join(str(workdir), "cube-208.pmesh"), deck],
                   cwd=str(workdir), env=env, check=True, stdout=subprocess.DEVNULL)
    ref = np.fromfile(os.path.join(str(workdir), "out.psi"))[8:].reshape(208, 128, 4, 2)
    o = Oracle(om, 8, 2)
    st = np.full(om.n_cells, 10.0)
    ss = np.full(om.n_cells, 5.0)
    psi, _, _, _ = o.source_iteration(st, ss, q_ang=o.hat_source(st, ss), err_max=1e-10)
    assert bits_equal(psi, ref)


def test_oracle_psi_writer_format(built, workdir):
    from oracle.oracle import Oracle
    _, om = cube208(workdir)
    o = Oracle(om, 4, 1)
    psi = np.arange(np.prod(o.psi_shape), dtype=np.float64).reshape(o.psi_shape)
    path = os.path.join(str(workdir), "w.psi")
    assert o.write_psi(psi, path) == 0
    raw = open(path, "rb").read()
    assert raw[:18] == b"Tycho 2 Psi Output" and raw[18:32] == bytes(14)
    hdr = np.frombuffer(raw[32:64], np.uint64)
    assert list(hdr) == [1, 208, 32, 1]
    assert np.array_equal(np.frombuffer(raw[64:], np.float64), psi.ravel())


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "sweep.x")),
                    reason="reference build not present")
def test_problem_checks_match_the_reference_printout(built, workdir):
    """Problem::hatL2Error and Util::diffBetweenGroups as the reference's
    main prints them after gold's solve (src/Main.cc:340-344), against
    tycho2_b200.problems.hat_l2_error / diff_between_groups of that psi."""
    import re
    import tycho2_b200 as ty
    from tycho2_b200 import problems
    mesh, _ = cube208(workdir)
    d = os.path.join(str(workdir), "checks")
    os.makedirs(d, exist_ok=True)
    deck = os.path.join(d, "gold.deck")
    with open(deck, "w") as f:
        f.write("snOrder 8\niterMax 100\nerrMax 1e-10\nmaxCellsPerStep 100\nintraAngleP 3\n"
                "interAngleP 1\nnGroups 2\nsigmaT1 10\nsigmaS1 5\nsigmaT2 10\nsigmaS2 5\n"
                "OutputFile true\nOutputFilename out.psi\nSourceIteration true\n"
                "MPIType TychoTwoSided\nDD_IterMax 100\nDD_ErrMax 1e-10\n"
                "SweepType TraverseGraph\nGaussElim NoPivot\n")
    r = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "sweep.x"),
                        os.path.join(str(workdir), "cube-208.pmesh"), deck],
                       cwd=d, env=dict(os.environ, OMP_NUM_THREADS="2"), check=True,
                       capture_output=True, text=True)
    l2 = float(re.search(r"L2 Relative Error: (\S+)", r.stdout).group(1))
    dg = float(re.search(r"Diff between groups: (\S+)", r.stdout).group(1))
    psi = np.fromfile(os.path.join(d, "out.psi"))[8:].reshape(208, 128, 4, 2)
    assert abs(problems.hat_l2_error(mesh, psi) - l2) <= 1e-6 * l2
    assert abs(problems.diff_between_groups(psi) - dg) <= 1e-6 * max(dg, 1e-300)
    # groups with equal cross sections and sources: identical psi
    assert problems.diff_between_groups(psi) == 0.0 and dg == 0.0
    # a psi whose groups differ
    psi2 = psi.copy()
    psi2[..., 1] *= 1.5
    assert problems.diff_between_groups(psi2) > 0.0
