"""tycho_sweeper_sweep_noalloc: the sweep for callers that cannot allocate
device memory when they sweep (hosts that own all device memory through their
own pool and budget, plugins limited to the buffers they are given,
time-critical loops).  The caller owns the source and psi buffers; the
sweep's scratch is a fixed file-scope device array.  Checked through the C ABI against the existing entry point
(tycho_sweeper_sweep) on two calls in a row: FP64 bit for bit, FP32 within
the FP32 tolerance used elsewhere (relative L1 <= 1e-5 of the FP64 psi)."""
import ctypes as C

import numpy as np
import pytest

from conftest import bits_equal, rel_l1

pytestmark = pytest.mark.gpu


def test_noalloc_sweep_matches_existing_entry_point(built):
    import torch
    import tycho2_b200 as ty
    from tycho2_b200._capi import check, lib

    mesh = ty.TychoMesh.kuhn_cube(5, 0.05, 31, 1.0)
    G, sn = 4, 8
    sw = ty.SweeperCuda(mesh, sn, G, fp32=True)
    rng = np.random.default_rng(31)
    st = rng.lognormal(0.0, 0.5, mesh.n_cells)
    sw.set_cross_sections(st, np.zeros(mesh.n_cells))
    q = rng.uniform(0.0, 1.0, sw.phi_shape)

    # Existing entry point: the same isotropic source given as an angular one.
    src = np.ascontiguousarray(np.broadcast_to(q[:, None, :, :], sw.psi_shape))
    psi_ref = np.empty(sw.psi_shape)
    sw.sweep(psi_ref, src)

    stream = torch.cuda.current_stream()
    for precision, dtype in ((0, torch.float64), (1, torch.float32)):
        iso = torch.tensor(q, dtype=dtype, device="cuda").contiguous()
        for call in range(2):
            psi = torch.full(sw.psi_shape, float("nan"), dtype=dtype, device="cuda")
            stream.synchronize()
            check(lib().tycho_sweeper_sweep_noalloc(sw._h, precision, C.c_void_p(iso.data_ptr()),
                                                    C.c_void_p(psi.data_ptr()),
                                                    C.c_void_p(stream.cuda_stream)))
            out = psi.cpu().numpy().astype(np.float64)
            if precision == 0:
                assert bits_equal(out, psi_ref), "FP64 call %d" % call
            else:
                assert np.all(np.isfinite(out)) and rel_l1(out, psi_ref) <= 1e-5, "FP32 call %d" % call
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
