"""Regenerates the golden fixtures in this directory from the reference.

Needs the tycho2 source tree ($TYCHO2_REF, default: a tree named reference
beside this repository) and the
reference built from it by `make -C oracle ref` (oracle/_ref).  Writes:

  gold.psi, cube-208.smesh   the reference's own regression vector and mesh
                             (test/regression/gold.psi, util/cube-208.smesh),
                             copied byte for byte
  kuhn3_ref.npz              what the reference computes on a jittered Kuhn
                             cube (3^3 hexes x 6 tets on [0,100]^3, written by
                             this project's generator and converted by the
                             reference's PartitionColumns 1 1):
                               pmesh_sha256       the converted mesh file
                               s{4,8}_{adj,nbr,f2c,c2f,deps,blev}  integer tables
                               s4_vol, s4_area, s4_odn             geometry (f64)
                               sweep_* : one SweeperTraverse::sweep of a seeded
                                         angular source, S4, G=3 (GaussElim
                                         NoPivot); sweep_psi_<kind>: its first
                                         group with GaussElim Original,
                                         CramerGlu, CramerIntel
                               si_*    : SourceIteration::fixedPoint with the
                                         hat source, per-cell sigma, S4, G=2
  partitions_ref.npz         one partition's local sweep: a jittered Kuhn cube
                             (4^3 hexes x 6 tets on [0,1]^3, oracle/kuhn_problem)
                             split by the reference's PartitionColumns 2 1 and
                             2 2:
                               p{2,4}_pmesh          the partitioned mesh files
                               p{P}_{p}_{adj,rank,side,lgside}  each partition's
                                          adjCell, adjRank, side, lGSides
                               p{P}_{p}_psi_hash     hash of Util::sweepLocal's
                                          psi (S4, G=3) for the inputs of
                                          tests/helpers.partition_inputs with
                                          salt 10 P + p
  sweep_schedule_levels.npz  SweepSchedule's b-levels (calcDependencies and
                             calcLevels with their +-1e-10 omega.n rule) on the
                             jittered cube above and on an unjittered one
                             (3^3 hexes on [0,1]^3, where S6 has exact
                             omega.n ties), S4, S6 and S8:
                               {jit,flat}_s{4,6,8}  (angle, cell) levels, then
                                                    their maximum

Run:  python tests/golden/make_golden.py [--levels-only | --partitions-only]
"""
import hashlib
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

REF = os.environ.get("TYCHO2_REF", os.path.join(os.path.dirname(ROOT), "reference"))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")


def run(*args, cwd=None, env=None):
    subprocess.run(list(args), check=True, cwd=cwd, stdout=subprocess.DEVNULL,
                   env=None if env is None else dict(os.environ, **env))


def kuhn3_fixture(tmp):
    import tycho2_b200 as ty
    from tycho2_b200 import problems

    mesh = ty.TychoMesh.kuhn_cube(3, 0.05, 2024, 100.0)
    smesh = os.path.join(tmp, "k3.smesh")
    pmesh = os.path.join(tmp, "k3.pmesh")
    mesh.write_smesh(smesh)
    run(os.path.join(REF_BIN, "PartitionColumns.x"), "1", "1", smesh, pmesh)
    out = {"pmesh_sha256": np.frombuffer(hashlib.sha256(open(pmesh, "rb").read()).digest(), np.uint8)}
    nc = mesh.n_cells
    for sn in (4, 8):
        pre = os.path.join(tmp, "s%d_" % sn)
        run(os.path.join(REF_BIN, "ref_dump.x"), "tables", pmesh, str(sn), pre)
        for k in ("adj", "nbr", "f2c", "c2f", "deps", "blev"):
            out["s%d_%s" % (sn, k)] = np.fromfile(pre + k + ".u64", np.uint64)
        if sn == 4:
            for k in ("vol", "area", "odn"):
                out["s4_" + k] = np.fromfile(pre + k + ".f64", np.float64)
    # One sweep of a seeded angular source.
    rng = np.random.default_rng(7)
    A, G = 32, 3
    sig_t = rng.uniform(0.5, 3.0, nc)
    src = rng.uniform(0.0, 1.0, (nc, A, 4, G))
    f_st, f_src, f_psi = (os.path.join(tmp, n) for n in ("st.f64", "src.f64", "psi.f64"))
    sig_t.tofile(f_st)
    src.tofile(f_src)
    run(os.path.join(REF_BIN, "ref_dump.x"), "sweep", pmesh, "4", str(G), f_st, f_src, f_psi)
    out["sweep_sigma_t"] = sig_t
    out["sweep_source"] = src
    out["sweep_psi"] = np.fromfile(f_psi, np.float64).reshape(nc, A, 4, G)
    # The same sweep, first group only, with each other GaussElim solver.
    src1 = np.ascontiguousarray(src[..., :1])
    src1.tofile(f_src)
    for kind in ("Original", "CramerGlu", "CramerIntel"):
        run(os.path.join(REF_BIN, "ref_dump.x"), "sweep", pmesh, "4", "1", f_st, f_src, f_psi,
            env={"TYCHO_GAUSS_ELIM": kind})
        out["sweep_psi_" + kind] = np.fromfile(f_psi, np.float64).reshape(nc, A, 4, 1)
    # Source iteration with the hat source and per-cell cross sections.
    G = 2
    sig_t = rng.uniform(1.0, 4.0, nc)
    sig_s = sig_t * rng.uniform(0.2, 0.8, nc)
    quad = ty.Quadrature(4)
    hat = problems.hat_source(mesh, quad, sig_t, sig_s, G)
    f_ss = os.path.join(tmp, "ss.f64")
    sig_t.tofile(f_st)
    sig_s.tofile(f_ss)
    hat.tofile(f_src)
    run(os.path.join(REF_BIN, "ref_dump.x"), "si", pmesh, "4", str(G), f_st, f_ss, f_src, "100",
        "1e-12", f_psi)
    out["si_sigma_t"] = sig_t
    out["si_sigma_s"] = sig_s
    out["si_psi"] = np.fromfile(f_psi, np.float64).reshape(nc, A, 4, G)
    np.savez_compressed(os.path.join(HERE, "kuhn3_ref.npz"), **out)


def levels_fixture(tmp):
    import tycho2_b200 as ty

    out = {}
    meshes = {"jit": ty.TychoMesh.kuhn_cube(3, 0.05, 2024, 100.0), "flat": ty.TychoMesh.kuhn_cube(3, 0.0, 0, 1.0)}
    for name, mesh in meshes.items():
        smesh, pmesh = os.path.join(tmp, name + ".smesh"), os.path.join(tmp, name + ".pmesh")
        mesh.write_smesh(smesh)
        run(os.path.join(REF_BIN, "PartitionColumns.x"), "1", "1", smesh, pmesh)
        for sn in (4, 6, 8):
            f = os.path.join(tmp, "%s_s%d.u64" % (name, sn))
            run(os.path.join(REF_BIN, "ref_dump.x"), "levels", pmesh, str(sn), f)
            out["%s_s%d" % (name, sn)] = np.fromfile(f, np.uint64)
    np.savez_compressed(os.path.join(HERE, "sweep_schedule_levels.npz"), **out)


def partitions_fixture(tmp):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import partition_inputs, psi_hash
    from oracle import kuhn_problem

    mesh = kuhn_problem.kuhn_cube(4, 0.05, 7, 1.0)
    smesh = os.path.join(tmp, "k4.smesh")
    kuhn_problem.write_smesh(smesh, mesh)
    out = {}
    sn, G, A = 4, 3, 32
    for px, py in ((2, 1), (2, 2)):
        P = px * py
        pmesh = os.path.join(tmp, "k4_%d.pmesh" % P)
        run(os.path.join(REF_BIN, "PartitionColumns.x"), str(px), str(py), smesh, pmesh)
        out["p%d_pmesh" % P] = np.fromfile(pmesh, np.uint8)
        for p in range(P):
            env = {"TYCHO_SHIM_RANK": str(p), "TYCHO_SHIM_SIZE": str(P), "OMP_NUM_THREADS": "2"}
            pre = os.path.join(tmp, "t%d_%d_" % (P, p))
            from oracle.oracle import OracleMesh
            om = OracleMesh(pmesh, p)
            st, src, pb = partition_inputs(om.n_cells, A, G, om.n_sides, 10 * P + p)
            f_st, f_src, f_pb, f_psi = (os.path.join(tmp, n) for n in ("st.f64", "src.f64", "pb.f64", "psi.f64"))
            st.tofile(f_st)
            src.tofile(f_src)
            pb.tofile(f_pb)
            run(os.path.join(REF_BIN, "ref_dump.x"), "sweep_local", pmesh, str(sn), str(G), f_st, f_src, f_pb,
                f_psi, pre, env=env)
            for k in ("adj", "rank", "side", "lgside"):
                out["p%d_%d_%s" % (P, p, k)] = np.fromfile(pre + k + ".u64", np.uint64)
            psi = np.fromfile(f_psi, np.float64)
            assert psi.size == om.n_cells * A * 4 * G
            out["p%d_%d_psi_hash" % (P, p)] = np.array([psi_hash(psi)], np.uint64)
    np.savez_compressed(os.path.join(HERE, "partitions_ref.npz"), **out)


def main():
    if not os.path.isdir(REF):
        sys.exit("reference tree not found: %s" % REF)
    run("make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", "oracle", "REF=" + REF)
    shutil.copyfile(os.path.join(REF, "test", "regression", "gold.psi"), os.path.join(HERE, "gold.psi"))
    shutil.copyfile(os.path.join(REF, "util", "cube-208.smesh"), os.path.join(HERE, "cube-208.smesh"))
    with tempfile.TemporaryDirectory() as tmp:
        if "--partitions-only" in sys.argv:
            partitions_fixture(tmp)
            return
        if "--levels-only" not in sys.argv:
            kuhn3_fixture(tmp)
        levels_fixture(tmp)
        partitions_fixture(tmp)


if __name__ == "__main__":
    main()
