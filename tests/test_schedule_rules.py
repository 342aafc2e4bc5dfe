"""The reference's two dependency rules on the host (no GPU needed).

* SweepSchedule's b-levels (calcDependencies + calcLevels,
  src/SweepSchedule.cc:107-125, :472-508: omega.n beyond +-1e-10 orders a
  face) against the reference's own functions, dumped by oracle/ref_dump.cc
  into tests/golden/sweep_schedule_levels.npz, on a jittered cube and on an
  unjittered one whose S6 directions have exact omega.n ties.
* A cyclic dependency graph built on the host: two tets on the same side of
  their shared face, so that for every direction with mu > 0 each is upwind
  of the other.  The reference's GraphTraverser spins on such a graph
  (src/GraphTraverser.cc:518); the wavefront levelling rejects it with
  TYCHO_ERR_CYCLE, the host levelling here and both levelling builders of
  the sweeper in a GPU test.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

TYCHO_ERR_CYCLE = 6


@pytest.fixture(scope="module")
def schedule_levels_ref():
    return dict(np.load(os.path.join(GOLDEN, "sweep_schedule_levels.npz")))


def _mesh(name):
    import tycho2_b200 as ty
    if name == "jit":
        return ty.TychoMesh.kuhn_cube(3, 0.05, 2024, 100.0)
    return ty.TychoMesh.kuhn_cube(3, 0.0, 0, 1.0)


@pytest.mark.parametrize("name", ["jit", "flat"])
@pytest.mark.parametrize("sn", [4, 6, 8])
def test_sweep_schedule_levels_match_reference(built, schedule_levels_ref, name, sn):
    mesh = _mesh(name)
    lev, top = mesh.sweep_schedule_levels(sn)
    ref = schedule_levels_ref["%s_s%d" % (name, sn)]
    assert np.array_equal(lev.ravel().astype(np.uint64), ref[:-1])
    assert top == int(ref[-1])


@pytest.mark.parametrize("sn", [4, 8])
def test_sweep_schedule_levels_equal_priorities_without_ties(built, sn):
    """Away from |omega.n| <= 1e-10 both reference rules order the same faces,
    so SweepSchedule's levels equal Priorities' b-levels."""
    mesh = _mesh("jit")
    t = mesh.tables()
    import tycho2_b200 as ty
    q = ty.Quadrature(sn)
    omega = np.stack([q.xi, q.eta, q.mu], axis=1)
    odn = np.einsum("ad,cfd->acf", omega, t["normal"])
    assert np.abs(odn).min() > 1e-10
    _, _, blev, _ = mesh.levels(sn)
    lev, top = mesh.sweep_schedule_levels(sn)
    assert np.array_equal(lev, blev)
    assert top == blev.max()


def _cyclic_pair():
    """Two tets sharing face {0, 1, 2} (z = 0) with both apexes above it: both
    outward normals of the shared face are (0, 0, -1)."""
    import tycho2_b200 as ty
    none = ty.sweeper.NONE
    cell_nodes = np.array([[0, 1, 2, 3], [0, 1, 2, 4]], np.uint64)
    coords = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.2, 0.2, 1.0], [0.3, 0.25, 0.5]], float)
    adj = np.array([[none, none, none, 1], [none, none, none, 0]], np.uint64)
    f2c = np.array([[[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]]] * 2, np.uint64)
    return ty.TychoMesh.from_arrays(cell_nodes, coords, adj, f2c)


def test_cyclic_graph_is_rejected_by_the_host_levelling(built):
    from tycho2_b200._capi import TychoError
    mesh = _cyclic_pair()
    normal = mesh.tables()["normal"]
    assert np.array_equal(normal[:, 3], [[0, 0, -1], [0, 0, -1]])
    with pytest.raises(TychoError) as e:
        mesh.levels(4)
    assert e.value.status == TYCHO_ERR_CYCLE and "cycle" in str(e.value)
    # SweepSchedule's rule never stalls: it returns, the pair being each
    # other's parent for mu > 0 and each other's child for mu < 0
    lev, top = mesh.sweep_schedule_levels(4)
    assert lev.shape == (32, 2) and np.all(lev[:16] == 0) and top >= 1


@pytest.mark.gpu
@pytest.mark.parametrize("levelling", ["host", "device"])
def test_cyclic_graph_is_rejected_by_the_sweeper(built, levelling):
    """Creating a sweeper on the cyclic pair fails with TYCHO_ERR_CYCLE for
    both levelling builders, and the device stays usable."""
    import tycho2_b200 as ty
    from tycho2_b200._capi import TychoError
    with pytest.raises(TychoError) as e:
        ty.SweeperCuda(_cyclic_pair(), 4, 1, levelling=levelling)
    assert e.value.status == TYCHO_ERR_CYCLE and "cycle" in str(e.value)
    sw = ty.SweeperCuda(_mesh("jit"), 4, 1, levelling=levelling)
    sw.set_cross_sections(np.ones(sw.mesh.n_cells), np.zeros(sw.mesh.n_cells))
    psi = np.empty(sw.psi_shape)
    sw.sweep(psi, np.ones(sw.psi_shape))
    assert np.all(np.isfinite(psi)) and psi.max() > 0
    sw.close()
