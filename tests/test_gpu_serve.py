"""Solve service: admission by footprint, continuous batching, and the same
result for a request served alone and in a mix of overlapping arrivals."""
import numpy as np
import pytest

from conftest import bits_equal, rel_l1

pytestmark = pytest.mark.gpu


def _requests(count, seed):
    from tycho2_b200 import problems
    params = problems.batch_instances(count, seed=seed, n_range=(2, 6))
    out = []
    for p in params:
        mesh, st, ss, mat, q = problems.make_problem(**p)
        out.append((p, mesh, st, ss, mat, q))
    return out


def _serve(reqs, method, arrivals, budget=150e9, threads=2, large_items=0.0, large_batched=False):
    import tycho2_b200 as ty
    srv = ty.SolveServer(method=method, budget_bytes=budget, setup_threads=threads, err_max=1e-10,
                         large_items=large_items, large_batched=large_batched)
    ids = [srv.submit(mesh, p["sn"], p["groups"], st, ss, mat, q, arrival=t)
           for (p, mesh, st, ss, mat, q), t in zip(reqs, arrivals)]
    srv.run()
    res = [(srv.phi(i).copy(), srv.info(i)) for i in ids]
    stats = srv.stats()
    srv.close()
    return res, stats


@pytest.mark.parametrize("method,large_items,batched", [("mixed", 0.0, False), ("si", 0.0, False),
                                                       ("mixed", 20000.0, False), ("si", 20000.0, False),
                                                       ("mixed", 20000.0, True)])
def test_served_result_same_alone_and_in_mix(built, method, large_items, batched):
    """large_items 20000: the bigger requests run beside the batch of small
    ones, solved one at a time by the single-instance solver (or in a second
    batch with its own stream)."""
    reqs = _requests(6, seed=11)
    alone = [_serve([r], method, [0.0], large_items=large_items, large_batched=batched)[0][0] for r in reqs]
    rng = np.random.default_rng(3)
    arrivals = np.cumsum(rng.exponential(0.01, len(reqs)))  # overlapping arrivals
    mixed, stats = _serve(reqs, method, arrivals, large_items=large_items, large_batched=batched)
    if large_items:
        sizes = [r[1].n_cells * 2 * r[0]["sn"] ** 2 for r in reqs]
        assert min(sizes) < large_items <= max(sizes)  # both lanes in use
    assert stats["peak_active"] >= 2  # the requests did share the GPU
    for (pa, ia), (pm, im) in zip(alone, mixed):
        assert ia["state"] == "done" and im["state"] == "done"
        assert bits_equal(pa, pm)
        assert im["arrival"] <= im["admitted"] <= im["built"] <= im["finished"]


def test_served_solution_matches_fp64_solve(built):
    """The mixed service's phi is within 1e-8 of the FP64 service's."""
    reqs = _requests(4, seed=5)
    a = [0.0, 0.0, 0.005, 0.01]
    mixed, _ = _serve(reqs, "mixed", a)
    fp64, _ = _serve(reqs, "si", a)
    for (pm, im), (p64, i64) in zip(mixed, fp64):
        assert rel_l1(pm, p64) <= 1e-8
        assert im["stats"]["sweeps_fp32"] > 0 and i64["stats"]["sweeps_fp32"] == 0


def test_admission_respects_the_budget(built):
    import tycho2_b200 as ty
    reqs = _requests(5, seed=21)
    fps = [ty.footprint_bytes(r[1].n_cells, r[0]["sn"], r[0]["groups"], True) for r in reqs]
    budget = max(fps) * 1.2  # one request at a time for the largest, a few small ones together
    res, stats = _serve(reqs, "mixed", [0.0] * len(reqs), budget=budget)
    assert stats["peak_bytes"] <= budget
    assert all(i["state"] == "done" for _, i in res)
    # a request larger than the whole budget fails; the others are served
    res2, _ = _serve(reqs[:2], "mixed", [0.0, 0.0], budget=min(fps[:2]) * 1.01)
    states = sorted(i["state"] for _, i in res2)
    big = int(np.argmax(fps[:2]))
    if fps[0] != fps[1]:
        assert res2[big][1]["state"] == "failed" and res2[1 - big][1]["state"] == "done"
    else:
        assert states == ["done", "done"]


@pytest.mark.parametrize("method", ["si", "mixed"])
def test_large_requests_solo_match_batched(built, method):
    """Large requests solved by the single-instance solver: the FP64 source
    iteration bit-identical to the batched one; the mixed service's GMRES-
    based refinement within 1e-8 of its batched source-iteration form."""
    reqs = _requests(6, seed=17)
    arrivals = [0.0, 0.0, 0.004, 0.008, 0.012, 0.02]
    sizes = [r[1].n_cells * 2 * r[0]["sn"] ** 2 for r in reqs]
    large = float(sorted(sizes)[-2])  # the two largest run beside the batch
    solo, _ = _serve(reqs, method, arrivals, large_items=large, large_batched=False)
    batched, _ = _serve(reqs, method, arrivals, large_items=large, large_batched=True)
    for (ps, i_s), (pb, ib), size in zip(solo, batched, sizes):
        assert i_s["state"] == "done" and ib["state"] == "done"
        if method == "si" or size < large:
            assert bits_equal(ps, pb)
        else:
            assert rel_l1(ps, pb) <= 1e-8
            assert i_s["stats"]["sweeps_fp32"] > 0
