"""tycho2_b200: a B200-native drop-in for lanl/tycho2's DG SN transport sweep.

The sweep, the scalar-flux reduction and the outer solvers run as sm_100a
CUDA kernels in libtycho_b200.so (C ABI: include/tycho_cuda.h); this package
is the host-side mirror of the reference's interface over that ABI.
"""
from ._capi import TychoError, lib  # noqa: F401
from .sweeper import (BatchSolver, Quadrature, SolveServer, SweeperCuda, TychoMesh, device_memory,  # noqa: F401
                      footprint_bytes, release_cached_memory)
from . import angles, partitions, problems  # noqa: F401

__all__ = ["TychoError", "TychoMesh", "Quadrature", "SweeperCuda", "BatchSolver", "SolveServer",
           "device_memory", "footprint_bytes", "release_cached_memory", "problems", "angles", "partitions", "lib"]
