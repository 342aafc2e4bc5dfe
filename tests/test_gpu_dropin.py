"""The drop-in itself: the reference's driver flow with SweeperCuda plugged in
(oracle/_ref/sweep_cuda.x: the reference's deck reader, TychoMesh, Problem
and .psi writer, built from the reference sources, calling the GPU sweep
through the C ABI) reproduces test/regression/gold.psi with the reference's
own criterion, test/diff.py (L1 and Linf relative error < 1e-10)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, rel_l1, rel_linf
from helpers import gold_psi

pytestmark = pytest.mark.gpu
BIN = os.path.join(ROOT, "oracle", "_ref")

DECK = """snOrder 8
iterMax 100
errMax 1e-10
maxCellsPerStep 100
intraAngleP 3
interAngleP 1
nGroups 2
sigmaT1 10
sigmaS1 5
sigmaT2 10
sigmaS2 5
OutputFile true
OutputFilename out.psi
SourceIteration {si}
MPIType TychoTwoSided
DD_IterMax 100
DD_ErrMax 1e-10
SweepType Cuda
GaussElim NoPivot
"""


def _run_driver(workdir, name, si, gauss="NoPivot", extra=()):
    d = os.path.join(str(workdir), name)
    os.makedirs(d, exist_ok=True)
    subprocess.run([os.path.join(BIN, "PartitionColumns.x"), "1", "1",
                    os.path.join(GOLDEN, "cube-208.smesh"), os.path.join(d, "c.pmesh")],
                   check=True, stdout=subprocess.DEVNULL)
    with open(os.path.join(d, "gold.deck"), "w") as f:
        f.write(DECK.format(si=si).replace("GaussElim NoPivot", "GaussElim " + gauss))
    r = subprocess.run([os.path.join(BIN, "sweep_cuda.x"), "c.pmesh", "gold.deck", *extra], cwd=d,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return np.fromfile(os.path.join(d, "out.psi"))[8:], r.stdout


NOT_BUILT = "reference-side binding not built (needs the tycho2 tree at build time)"


@pytest.mark.skipif(not os.path.exists(os.path.join(BIN, "sweep_cuda.x")), reason=NOT_BUILT)
@pytest.mark.parametrize("si", ["true", "false"])
def test_reference_driver_with_gpu_sweeper_reproduces_gold(workdir, si):
    psi, _ = _run_driver(workdir, "dropin_" + si, si)
    gold = gold_psi().ravel()
    assert rel_l1(psi, gold) < 1e-10 and rel_linf(psi, gold) < 1e-10


@pytest.mark.skipif(not os.path.exists(os.path.join(BIN, "sweep_cuda.x")), reason=NOT_BUILT)
@pytest.mark.parametrize("gauss", ["NoPivot", "Original", "CramerGlu", "CramerIntel"])
def test_reference_fixed_point_over_gpu_sweep_reproduces_gold(workdir, gauss):
    """The reference's own SourceIteration::fixedPoint (its psiToPhi,
    calcTotalSource and L1 stopping rule on the host) calls
    SweeperCuda::sweep with the reference's PsiData buffers, as
    SweeperTraverse::solve calls SweeperTraverse::sweep; every deck value of
    GaussElim is parsed and reaches the GPU solver.  gold.psi within
    test/diff.py's 1e-10, in the gold run's 34 iterations."""
    psi, out = _run_driver(workdir, "fixedpoint_" + gauss, "true", gauss, ("reference-loop",))
    gold = gold_psi().ravel()
    assert rel_l1(psi, gold) < 1e-10 and rel_linf(psi, gold) < 1e-10
    assert "fixedPoint over SweeperCuda::sweep: 34 iterations" in out
