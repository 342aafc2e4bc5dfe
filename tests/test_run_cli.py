"""The reference's command line on the B200 sweep (tycho2_b200.run): the
host-side pieces without a GPU -- the deck reader on the reference's deck
format, the material cross sections, the .psi writer's format."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

GOLD_DECK = """# Sample input deck
# Copy this to input.deck (or any other name you choose)

snOrder         8
iterMax         100
errMax          1e-10
maxCellsPerStep 100
intraAngleP     3
interAngleP     1
nGroups         2
sigmaT1         10
sigmaS1         5
sigmaT2         10
sigmaS2         5
OutputFile      true
OutputFilename  out.psi
SourceIteration true
MPIType         TychoTwoSided

DD_IterMax      100
DD_ErrMax       1e-10

# Types: OriginalTycho1, OriginalTycho2, TraverseGraph
SweepType TraverseGraph
GaussElim NoPivot
"""


def test_deck_reader(tmp_path):
    from tycho2_b200.run import _get, read_deck
    p = tmp_path / "in.deck"
    p.write_text(GOLD_DECK)
    d = read_deck(str(p))
    assert _get(d, "snOrder", int) == 8 and _get(d, "SNORDER", int) == 8
    assert _get(d, "errMax", float) == 1e-10 and _get(d, "SourceIteration", bool) is True
    assert _get(d, "SweepType", str) == "TraverseGraph" and _get(d, "OutputFilename", str) == "out.psi"
    assert _get(d, "GaussElim", str, "NoPivot") == "NoPivot"
    assert _get(d, "missingKey", int, "7") == 7
    with pytest.raises(KeyError):
        _get(d, "missingKey", int)
    p.write_text("SourceIteration maybe\n")
    with pytest.raises(ValueError):
        _get(read_deck(str(p)), "SourceIteration", bool)


def test_cross_sections_by_material(built):
    import tycho2_b200 as ty
    from tycho2_b200.run import cross_sections
    mesh = ty.TychoMesh.read_smesh(os.path.join(GOLDEN, "cube-208.smesh"))
    mat = mesh.cell_material()
    assert set(np.unique(mat).tolist()) <= {1, 2}
    st, ss = cross_sections(mesh, 10.0, 5.0, 3.0, 1.0)
    assert np.array_equal(st, np.where(mat == 1, 10.0, 3.0)) and np.array_equal(ss, np.where(mat == 1, 5.0, 1.0))


def test_psi_writer_format(tmp_path):
    from tycho2_b200.run import write_psi
    psi0 = np.arange(2 * 3 * 4 * 2, dtype=np.float64).reshape(2, 3, 4, 2)
    psi1 = -np.arange(1 * 3 * 4 * 2, dtype=np.float64).reshape(1, 3, 4, 2)
    path = str(tmp_path / "o.psi")
    write_psi(path, [(np.array([2, 0], np.uint64), psi0), (np.array([1], np.uint64), psi1)], 3, 3, 2)
    raw = open(path, "rb").read()
    assert raw[:18] == b"Tycho 2 Psi Output" and raw[18:32] == bytes(14)
    assert list(np.frombuffer(raw[32:64], np.uint64)) == [1, 3, 3, 2]
    data = np.frombuffer(raw[64:], np.float64).reshape(3, 3, 4, 2)
    assert np.array_equal(data[2], psi0[0]) and np.array_equal(data[0], psi0[1]) and np.array_equal(data[1], psi1[0])
