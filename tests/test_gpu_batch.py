"""Batched solves of uneven instances (mesh size, group count, SN order).

Parity: a member's FP64 source iteration reproduces the oracle's
SourceIteration::fixedPoint restatement; the mixed-precision solve lands
within 1e-8 (relative L1) of it; and every member's result is bit-identical
alone and inside the mix (its arithmetic and reductions never touch another
member's data).
"""
import numpy as np
import pytest

from conftest import bits_equal, rel_l1
from helpers import kuhn

pytestmark = pytest.mark.gpu

# (n, jitter, sn, G, scattering ratio, downscatter)
CASES = [(3, 0.05, 4, 1, 0.5, False), (4, 0.05, 6, 2, 0.8, True), (2, 0.05, 8, 4, 0.3, True),
         (5, 0.05, 4, 8, 0.9, True), (3, 0.05, 8, 3, 0.6, False)]


def _problem(workdir, case, seed):
    import tycho2_b200 as ty
    from tycho2_b200 import problems
    n, jitter, sn, G, ratio, down = case
    mesh, om = kuhn(workdir, n, jitter, seed=seed)
    rng = np.random.default_rng(seed)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    if down:  # sigma_s(g' -> g) = sigma_t * matrix, rows summing to the ratio
        ss, mat = st, problems.downscatter_matrix(G, ratio)
    else:
        ss, mat = ratio * st, None
    q = np.ones((mesh.n_cells, 4, G))
    sw = ty.SweeperCuda(mesh, sn, G, fp32=True)
    sw.set_cross_sections(st, ss, mat)
    sw.set_source(q, "isotropic")
    return sw, om, (st, ss, mat, q)


def _solve(sws, method, ipw=16, persistent=False, **kw):
    import tycho2_b200 as ty
    b = ty.BatchSolver(ipw32=ipw, ipw64=ipw, persistent=persistent)
    ids = [b.add(sw, method, **kw) for sw in sws]
    b.run()
    out = [b.result(i) for i in ids]
    for i in ids:
        b.remove(i)
    b.close()
    return out


@pytest.mark.parametrize("ipw", [16, 0])
def test_batch_si_matches_oracle_source_iteration(built, workdir, ipw):
    from oracle.oracle import Oracle
    probs = [_problem(workdir, c, 40 + k) for k, c in enumerate(CASES)]
    res = _solve([p[0] for p in probs], "si", ipw=ipw, err_max=1e-10, iter_max=400)
    for (sw, om, (st, ss, mat, q)), case, (phi, stats, done) in zip(probs, CASES, res):
        o = Oracle(om, case[2], case[3])
        _, phi_ref, it_ref, _ = o.source_iteration(st, ss, mat, q_iso=q, iter_max=400, err_max=1e-10)
        assert done and stats["sweeps_fp32"] == 0
        if stats["iterations"] == it_ref:
            # same sweeps, same scatter and psi->phi arithmetic: the same bits
            assert bits_equal(phi, phi_ref), case
        else:  # the stopping test sits on the threshold; one extra iteration apart
            assert abs(stats["iterations"] - it_ref) == 1 and rel_l1(phi, phi_ref) <= 1e-9, case


@pytest.mark.parametrize("ipw", [16, 0])
def test_batch_mixed_within_1e8_of_fp64(built, workdir, ipw):
    probs = [_problem(workdir, c, 60 + k) for k, c in enumerate(CASES)]
    sws = [p[0] for p in probs]
    si = _solve(sws, "si", ipw=ipw, err_max=1e-12, iter_max=2000)
    mixed = _solve(sws, "mixed", ipw=ipw, err_max=1e-12, iter_max=4000)
    for case, (phi64, s64, _), (phim, sm, done) in zip(CASES, si, mixed):
        assert done
        assert rel_l1(phim, phi64) <= 1e-8, (case, rel_l1(phim, phi64))
        assert sm["sweeps_fp32"] > sm["sweeps_fp64"] and sm["refinements"] >= 1


@pytest.mark.parametrize("method,ipw", [("si", 16), ("mixed", 16), ("si", 0), ("mixed", 0)])
def test_batch_member_bit_identical_alone_and_in_mix(built, workdir, method, ipw):
    probs = [_problem(workdir, c, 80 + k) for k, c in enumerate(CASES)]
    sws = [p[0] for p in probs]
    alone = [_solve([sw], method, ipw=ipw, err_max=1e-10)[0] for sw in sws]
    mixed = _solve(sws, method, ipw=ipw, err_max=1e-10)
    for case, (pa, sa, _), (pm, smx, _) in zip(CASES, alone, mixed):
        assert bits_equal(pa, pm), case
        assert sa == smx, case
    # and again in another order, with a repeated solve of the same members
    rev = _solve(sws[::-1], method, ipw=ipw, err_max=1e-10)[::-1]
    for case, (pa, _, _), (pr, _, _) in zip(CASES, alone, rev):
        assert bits_equal(pa, pr), case


def test_batch_psi_is_the_last_fp64_sweep(built, workdir):
    """After a batched solve the member's resident psi is its last FP64
    sweep, consistent with the returned phi for source iteration."""
    import tycho2_b200 as ty
    sw, om, (st, ss, mat, q) = _problem(workdir, CASES[1], 99)
    (phi, stats, done), = _solve([sw], "si", err_max=1e-10)
    path = str(workdir / "batch.psi")
    sw.writePsiToFile(path)
    raw = np.fromfile(path, np.float64)
    psi = raw[raw.size - np.prod(sw.psi_shape):].reshape(sw.psi_shape)
    w = ty.Quadrature(CASES[1][2]).wt
    phi_from_psi = np.einsum("cavg,a->cvg", psi, w)
    assert rel_l1(phi_from_psi, phi) <= 1e-13


def test_batch_errors(built, workdir):
    import tycho2_b200 as ty
    sw, _, _ = _problem(workdir, CASES[0], 7)
    b = ty.BatchSolver()
    b.add(sw, "si")
    with pytest.raises(ty.TychoError):
        b.add(sw, "si")  # already a member
    with pytest.raises(ty.TychoError):
        b.remove(12345)
    mesh, _ = kuhn(workdir, 2, 0.0, seed=3)
    plain = ty.SweeperCuda(mesh, 4, 1)  # no FP32 sweep
    plain.set_cross_sections(np.ones(mesh.n_cells), np.zeros(mesh.n_cells))
    with pytest.raises(ty.TychoError):
        b.add(plain, "mixed")
    b.close()


def test_batch_members_with_other_solvers(built, workdir):
    """Members with GaussElim Original / CramerGlu / CramerIntel next to
    NoPivot ones: each bit-identical alone and in the mix, and each member's
    FP64 source iteration equal to the oracle's with its own solver."""
    import tycho2_b200 as ty
    from oracle.oracle import Oracle
    kinds = ["Original", "NoPivot", "CramerGlu", "CramerIntel"]
    sws, refs = [], []
    for k, (kind, case) in enumerate(zip(kinds, CASES)):
        n, jitter, sn, G, ratio, down = case
        mesh, om = kuhn(workdir, n, jitter, seed=200 + k)
        rng = np.random.default_rng(200 + k)
        st = rng.lognormal(0.0, 0.5, mesh.n_cells)
        ss = ratio * st
        q = np.ones((mesh.n_cells, 4, G))
        sw = ty.SweeperCuda(mesh, sn, G, fp32=True, gauss_elim=kind)
        sw.set_cross_sections(st, ss)
        sw.set_source(q, "isotropic")
        sws.append(sw)
        _, phi_ref, it_ref, _ = Oracle(om, sn, G, gauss_elim=kind).source_iteration(
            st, ss, q_iso=q, iter_max=400, err_max=1e-10)
        refs.append((phi_ref, it_ref))
    alone = [_solve([sw], "si", ipw=0, err_max=1e-10, iter_max=400)[0] for sw in sws]
    mixed = _solve(sws, "si", ipw=0, err_max=1e-10, iter_max=400)
    for kind, (pa, sa, _), (pm, _, _), (phi_ref, it_ref) in zip(kinds, alone, mixed, refs):
        assert bits_equal(pa, pm), kind
        if sa["iterations"] == it_ref:
            assert bits_equal(pa, phi_ref), kind
        else:
            assert rel_l1(pa, phi_ref) <= 1e-9, kind
    mixed32 = _solve(sws, "mixed", ipw=0, err_max=1e-11)
    for kind, (pm, _, done), (phi_ref, _) in zip(kinds, mixed32, refs):
        assert done and rel_l1(pm, phi_ref) <= 1e-8, kind
    with pytest.raises(ty.TychoError):  # the shared-memory batch kernels take NoPivot only
        ty.BatchSolver(ipw32=16, ipw64=16).add(sws[0], "si")


@pytest.mark.parametrize("method", ["si", "mixed"])
def test_persistent_batch_is_bit_identical_to_level_launches(built, workdir, method):
    """One persistent kernel per pass (device work queue over (member, level),
    bounded grid barrier between levels) gives the same bits as one launch
    per level, alone and in the mix; its FP64 source iteration is the
    oracle's."""
    probs = [_problem(workdir, c, 120 + k) for k, c in enumerate(CASES)]
    sws = [p[0] for p in probs]
    levels = _solve(sws, method, ipw=0, err_max=1e-10)
    persist = _solve(sws, method, ipw=0, persistent=True, err_max=1e-10)
    alone = [_solve([sw], method, ipw=0, persistent=True, err_max=1e-10)[0] for sw in sws[:2]]
    for case, (pl, sl, _), (pp, sp, done) in zip(CASES, levels, persist):
        assert done and bits_equal(pl, pp), case
        assert sl == sp, case
    for (pa, _, _), (pp, _, _) in zip(alone, persist[:2]):
        assert bits_equal(pa, pp)
    if method == "si":
        from oracle.oracle import Oracle
        (sw, om, (st, ss, mat, q)), case = probs[0], CASES[0]
        o = Oracle(om, case[2], case[3])
        _, phi_ref, it_ref, _ = o.source_iteration(st, ss, mat, q_iso=q, iter_max=400, err_max=1e-10)
        if persist[0][1]["iterations"] == it_ref:
            assert bits_equal(persist[0][0], phi_ref)


def test_persistent_batch_barrier_timeout_is_an_error(built, workdir):
    """A wait limit of 0 makes the grid barrier give up at its first level
    that is not already met: the step fails with TYCHO_ERR_TIMEOUT (status
    8), no fault, and a new batch on the same device then solves normally."""
    import tycho2_b200 as ty
    from tycho2_b200._capi import TychoError
    probs = [_problem(workdir, c, 140 + k) for k, c in enumerate(CASES[:2])]
    sws = [p[0] for p in probs]
    b = ty.BatchSolver(ipw32=0, ipw64=0, persistent=True)
    b.set_wait_limit(0)
    for sw in sws:
        b.add(sw, "si", err_max=1e-10)
    with pytest.raises(TychoError) as e:
        b.run()
    assert e.value.status == 8 and "timed out" in str(e.value)
    b.close()
    ref = _solve(sws, "si", ipw=0, err_max=1e-10)
    again = _solve(sws, "si", ipw=0, persistent=True, err_max=1e-10)
    for (pr, _, _), (pa, _, done) in zip(ref, again):
        assert done and bits_equal(pr, pa)


def test_batch_autotuner_picks_a_measured_shape(built, workdir):
    """BatchSolver.autotune times each candidate shape on the members and
    returns the fastest; the batch built with its pick solves as the default
    one does (bit-identical: the shapes share the per-chunk arithmetic)."""
    import tycho2_b200 as ty
    probs = [_problem(workdir, c, 160 + k) for k, c in enumerate(CASES)]
    sws = [p[0] for p in probs]
    pick, table = ty.BatchSolver.autotune(sws, steps=2)
    assert {"ipw32", "ipw64", "persistent"} <= set(pick)
    assert len(table) == len(ty.BatchSolver.TUNE_SHAPES)
    timed = [r for r in table if r.get("fp64_ms_per_pass") is not None]
    assert timed and all(r["fp64_ms_per_pass"] > 0 and r["fp32_ms_per_pass"] > 0 for r in timed)
    fastest64 = min(r["fp64_ms_per_pass"] for r in timed if r["persistent"] == pick["persistent"])
    assert any(r["ipw"] == pick["ipw64"] and r["fp64_ms_per_pass"] == fastest64 for r in timed)
    ref = _solve(sws, "si", ipw=0, err_max=1e-10)
    b = ty.BatchSolver(**pick)
    ids = [b.add(sw, "si", err_max=1e-10) for sw in sws]
    b.run()
    got = [b.result(i) for i in ids]
    b.close()
    for (pr, _, _), (pg, _, done) in zip(ref, got):
        assert done and bits_equal(pr, pg)
