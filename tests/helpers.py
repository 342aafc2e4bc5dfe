"""Shared helpers for the parity tests: meshes written once per test session
and loaded by both the product (C++ ingest) and the oracle."""
import os

import numpy as np

from conftest import GOLDEN


def kuhn(workdir, n, jitter=0.05, seed=2024, length=1.0):
    import tycho2_b200 as ty
    from oracle.oracle import OracleMesh
    mesh = ty.TychoMesh.kuhn_cube(n, jitter, seed, length)
    path = os.path.join(str(workdir), "kuhn_%d_%g_%d_%g.pmesh" % (n, jitter, seed, length))
    if not os.path.exists(path):
        mesh.write_pmesh(path)
    return mesh, OracleMesh(path)


def cube208(workdir):
    import tycho2_b200 as ty
    from oracle.oracle import OracleMesh
    mesh = ty.TychoMesh.read_smesh(os.path.join(GOLDEN, "cube-208.smesh"))
    path = os.path.join(str(workdir), "cube-208.pmesh")
    if not os.path.exists(path):
        mesh.write_pmesh(path)
    return mesh, OracleMesh(path)


def gold_psi():
    raw = np.fromfile(os.path.join(GOLDEN, "gold.psi"), np.float64)
    return raw[8:].reshape(208, 128, 4, 2)
