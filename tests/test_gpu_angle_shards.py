"""Angle shards on the GPU (tycho_sweeper_create_angles, tycho_sweeper_apply).

Two shards of one problem, emulated in one process on one GPU (no collective:
the process sums its two shards' partial phi itself, which is what the
all-reduce does across GPUs): the partial phi of each shard sum to the
whole problem's operator application within rounding (the sum adds two
partial sums instead of every direction in angle order), and source
iteration and GMRES over the shards reach the one-sweeper solves and the
oracle.  The multi-process form over torch.distributed is covered by
tests/test_angle_shards_gloo.py on the host.
"""
import numpy as np
import pytest

from conftest import rel_l1
from helpers import kuhn

pytestmark = pytest.mark.gpu


def _setup(workdir, G=4, sn=6):
    import tycho2_b200 as ty
    from tycho2_b200 import problems
    mesh, om = kuhn(workdir, 6, 0.05, seed=29)
    rng = np.random.default_rng(11)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    mat = problems.downscatter_matrix(G, 0.8)
    q = rng.uniform(0.0, 1.0, (mesh.n_cells, 4, G))
    A = 2 * sn * sn
    from tycho2_b200.angles import angle_ranges
    shards = []
    for a0, a1 in angle_ranges(A, 2):
        sw = ty.SweeperCuda(mesh, sn, G, angles=(a0, a1))
        sw.set_cross_sections(st, st.copy(), mat)
        sw.set_source(q, "isotropic")
        shards.append(sw)
    full = ty.SweeperCuda(mesh, sn, G)
    full.set_cross_sections(st, st.copy(), mat)
    full.set_source(q, "isotropic")
    return mesh, om, st, mat, q, shards, full


def test_shard_partials_sum_to_the_whole_application(built, workdir):
    import torch
    mesh, om, st, mat, q, shards, full = _setup(workdir)
    shape = full.phi_shape
    phi_in = torch.tensor(np.random.default_rng(3).uniform(0, 1, shape), dtype=torch.float64, device="cuda")
    whole = torch.empty(shape, dtype=torch.float64, device="cuda")
    full.apply(phi_in, whole)
    parts = []
    for sw in shards:
        assert sw.n_angles == full.n_angles // 2
        out = torch.empty(shape, dtype=torch.float64, device="cuda")
        sw.apply(phi_in, out)
        parts.append(out)
    total = (parts[0] + parts[1]).cpu().numpy()
    ref = whole.cpu().numpy()
    assert rel_l1(total, ref) <= 1e-14
    # and without the fixed source, without scattering
    for w_fixed, pin in ((False, phi_in), (True, None)):
        full.apply(pin, whole, with_fixed=w_fixed)
        for sw, out in zip(shards, parts):
            sw.apply(pin, out, with_fixed=w_fixed)
        assert rel_l1((parts[0] + parts[1]).cpu().numpy(), whole.cpu().numpy()) <= 1e-14
    for sw in shards + [full]:
        sw.close()


def test_sharded_source_iteration_and_gmres_match_one_sweeper(built, workdir):
    import torch
    from oracle.oracle import Oracle
    from tycho2_b200.angles import ShardedOperator, gmres, source_iteration
    mesh, om, st, mat, q, shards, full = _setup(workdir)
    tmp = [torch.empty(full.phi_shape, dtype=torch.float64, device="cuda") for _ in shards]

    def apply_local(phi_in, phi_out, with_fixed):
        for sw, t in zip(shards, tmp):
            sw.apply(phi_in, t, with_fixed=with_fixed)
        torch.add(tmp[0], tmp[1], out=phi_out)

    op = ShardedOperator(apply_local, distributed=False)
    like = torch.empty(full.phi_shape, dtype=torch.float64, device="cuda")
    phi_si, it, err = source_iteration(op, like, iter_max=400, err_max=1e-11)
    phi_k, its, rn = gmres(op, like, restart=20, rtol=1e-12, iter_max=200)
    ref_si, _, s_si = full.solve("si", iter_max=400, err_max=1e-11, want_psi=False)
    ref_k, _, s_k = full.solve("gmres", iter_max=200, err_max=1e-12, want_psi=False)
    assert abs(it - s_si["iterations"]) <= 1
    assert rel_l1(phi_si.cpu().numpy(), ref_si) <= 1e-11
    assert rel_l1(phi_k.cpu().numpy(), ref_k) <= 1e-10 and rn <= 1e-12
    o = Oracle(om, 6, 4)
    _, phi_o, _, _ = o.krylov(st, st.copy(), mat, q_iso=q, restart=20, iter_max=200, rtol=1e-12)
    assert rel_l1(phi_k.cpu().numpy(), phi_o) <= 1e-10
    for sw in shards + [full]:
        sw.close()


def test_one_process_angle_sharded_solver_is_the_whole_problem(built, workdir):
    """Without a process group the solver holds every direction."""
    from tycho2_b200.angles import AngleShardedSolver
    mesh, om, st, mat, q, shards, full = _setup(workdir)
    s = AngleShardedSolver(mesh, 6, 4)
    assert s.world == 1 and s.range == (0, 72)
    s.set_cross_sections(st, st.copy(), mat)
    s.set_source(q)
    phi, it, err = s.solve("gmres", err_max=1e-12)
    ref, _, _ = full.solve("gmres", iter_max=200, err_max=1e-12, want_psi=False)
    assert rel_l1(phi.cpu().numpy(), ref) <= 1e-10
    s.close()
    for sw in shards + [full]:
        sw.close()
