"""tycho_sweeper_sweep_noalloc: the sweep for callers that cannot allocate
device memory when they sweep (hosts that own all device memory through their
own pool and budget, plugins limited to the buffers they are given,
time-critical loops).  The caller owns the source and psi buffers; the
sweep's scratch is a fixed file-scope device array.

Checked through the C ABI against the existing entry point
(tycho_sweeper_sweep) on two calls in a row, for the default launch shape and
for the record and direct-record shapes (whose per-item records the call must
not allocate): FP64 bit for bit, FP32 within the FP32 tolerance used
elsewhere (relative L1 <= 1e-5 of the FP64 psi).  The second call must leave
the device's free memory and the library's memory pool unchanged.  The
bounded-wait failure path runs too: with a wait limit of 0 the call returns
TYCHO_ERR_TIMEOUT, and the next call succeeds and matches again."""
import ctypes as C

import numpy as np
import pytest

from conftest import bits_equal, rel_l1

pytestmark = pytest.mark.gpu

TYCHO_ERR_TIMEOUT = 8

# launch shapes (schedule, variant, knob) per precision; None = the default
SHAPES = {
    "default": None,
    "records": {0: ("levels", "records", 16), 1: ("levels", "records", 16)},
    "direct": {0: ("levels", "direct", 64), 1: ("levels", "direct", 64)},
}


def _problem():
    import tycho2_b200 as ty
    mesh = ty.TychoMesh.kuhn_cube(5, 0.05, 31, 1.0)
    G, sn = 4, 8
    sw = ty.SweeperCuda(mesh, sn, G, fp32=True)
    rng = np.random.default_rng(31)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    sw.set_cross_sections(st, np.zeros(mesh.n_cells))
    q = rng.uniform(0.0, 1.0, sw.phi_shape)
    # existing entry point: the same isotropic source given as an angular one
    src = np.ascontiguousarray(np.broadcast_to(q[:, None, :, :], sw.psi_shape))
    psi_ref = np.empty(sw.psi_shape)
    sw.sweep(psi_ref, src)
    return sw, q, psi_ref


def _noalloc(sw, precision, iso, psi, stream):
    from tycho2_b200._capi import lib
    return lib().tycho_sweeper_sweep_noalloc(sw._h, precision, C.c_void_p(iso.data_ptr()),
                                             C.c_void_p(psi.data_ptr()), C.c_void_p(stream.cuda_stream))


def _check(out, psi_ref, precision, what):
    if precision == 0:
        assert bits_equal(out, psi_ref), what
    else:
        assert np.all(np.isfinite(out)) and rel_l1(out, psi_ref) <= 1e-5, what


@pytest.mark.parametrize("shape", sorted(SHAPES))
def test_noalloc_sweep_matches_existing_entry_point(built, shape):
    import torch
    import tycho2_b200 as ty
    from tycho2_b200._capi import check

    sw, q, psi_ref = _problem()
    if SHAPES[shape]:
        for prec, (sched, variant, knob) in SHAPES[shape].items():
            sw.configure(prec, sched, variant, knob)
        # new cross sections make the configured records stale: the no-alloc
        # call recomputes them in place, allocating nothing
        sw.set_cross_sections(*sw._xs)
    stream = torch.cuda.current_stream()
    for precision, dtype in ((0, torch.float64), (1, torch.float32)):
        iso = torch.tensor(q, dtype=dtype, device="cuda").contiguous()
        bufs = [torch.full(sw.psi_shape, float("nan"), dtype=dtype, device="cuda") for _ in range(2)]
        stream.synchronize()
        mem = []
        for call, psi in enumerate(bufs):
            check(_noalloc(sw, precision, iso, psi, stream))
            stream.synchronize()
            mem.append((torch.cuda.mem_get_info()[0], ty.device_memory(0)))
            _check(psi.cpu().numpy().astype(np.float64), psi_ref, precision,
                   "%s, precision %d, call %d" % (shape, precision, call))
        assert mem[1] == mem[0], "the second call changed device memory: %s" % (mem,)
    sw.close()


def test_noalloc_sweep_times_out_and_recovers(built):
    import torch
    from tycho2_b200._capi import TychoError, check

    sw, q, psi_ref = _problem()
    stream = torch.cuda.current_stream()
    iso = torch.tensor(q, dtype=torch.float64, device="cuda").contiguous()
    psi = torch.empty(sw.psi_shape, dtype=torch.float64, device="cuda")
    stream.synchronize()
    sw.set_wait_limit(0)  # every wait that is not already satisfied gives up
    with pytest.raises(TychoError) as e:
        check(_noalloc(sw, 0, iso, psi, stream))
    assert e.value.status == TYCHO_ERR_TIMEOUT and "timed out" in str(e.value)
    sw.set_wait_limit(1 << 22)
    for call in range(2):
        psi.fill_(float("nan"))
        check(_noalloc(sw, 0, iso, psi, stream))
        _check(psi.cpu().numpy(), psi_ref, 0, "after the timeout, call %d" % call)
    sw.close()


def test_noalloc_sweep_rejects_problems_beyond_its_scratch(built):
    import torch
    import tycho2_b200 as ty
    from tycho2_b200._capi import TychoError, check, lib

    # 28^3 hexes x 6 = 131,712 tets x 128 directions = 16.9M items > 2^24.
    mesh = ty.TychoMesh.kuhn_cube(28, 0.0, 0, 1.0)
    sw = ty.SweeperCuda(mesh, 8, 1)
    sw.set_cross_sections(np.ones(mesh.n_cells), np.zeros(mesh.n_cells))
    psi = torch.empty(8, dtype=torch.float64, device="cuda")
    with pytest.raises(TychoError) as e:
        check(lib().tycho_sweeper_sweep_noalloc(sw._h, 0, None, C.c_void_p(psi.data_ptr()), None))
    assert e.value.status == 1 and "at most 16777216" in str(e.value)
    sw.close()
