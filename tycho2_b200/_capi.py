"""ctypes binding of the C ABI in include/tycho_cuda.h (libtycho_b200.so).

The library is built in-tree by tycho2_b200/csrc/Makefile (see
__graft_entry__.build()).  Loading fails loudly when it is missing: there is
no CPU fallback for the sweep.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libtycho_b200.so")

TYCHO_OK = 0
STATUS_NAMES = {
    0: "TYCHO_OK", 1: "TYCHO_ERR_ARG", 2: "TYCHO_ERR_IO", 3: "TYCHO_ERR_FORMAT",
    4: "TYCHO_ERR_CUDA", 5: "TYCHO_ERR_OOM", 6: "TYCHO_ERR_CYCLE",
    7: "TYCHO_ERR_NOT_CONVERGED", 8: "TYCHO_ERR_TIMEOUT", 9: "TYCHO_ERR_BUSY",
    10: "TYCHO_ERR_MISSING",
}

# Every function the header declares, with (restype, argtypes).
_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
_U64P = C.POINTER(C.c_uint64)
_U32P = C.POINTER(C.c_uint32)


class SweeperOpts(C.Structure):
    _fields_ = [("sn_order", C.c_int), ("n_groups", C.c_int), ("gauss_elim", C.c_int),
                ("device", C.c_int), ("fp32", C.c_int), ("tpi64", C.c_int), ("tpi32", C.c_int),
                ("schedule", C.c_int), ("levelling", C.c_int)]


class SolveOpts(C.Structure):
    _fields_ = [("method", C.c_int), ("iter_max", C.c_int), ("err_max", C.c_double),
                ("restart", C.c_int), ("inner_tol", C.c_double), ("refine_max", C.c_int)]


class LaunchShape(C.Structure):
    _fields_ = [("schedule", C.c_int), ("variant", C.c_int), ("knob", C.c_int), ("vector", C.c_int),
                ("streams", C.c_int)]


class BatchOpts(C.Structure):
    _fields_ = [("method", C.c_int), ("iter_max", C.c_int), ("err_max", C.c_double),
                ("inner_tol", C.c_double), ("inner_max", C.c_int), ("refine_max", C.c_int)]


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("budget_bytes", C.c_double), ("setup_threads", C.c_int),
                ("ipw32", C.c_int), ("ipw64", C.c_int), ("solve", BatchOpts), ("large_items", C.c_double),
                ("large_batched", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("sweeps_fp64", C.c_int), ("sweeps_fp32", C.c_int),
                ("refinements", C.c_int), ("final_error", C.c_double), ("seconds", C.c_double)]


SIGNATURES = {
    "tycho_status_string": (C.c_char_p, [C.c_int]),
    "tycho_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "tycho_version": (C.c_int, []),
    "tycho_mesh_read_pmesh": (C.c_int, [C.c_char_p, _PP]),
    "tycho_mesh_read_smesh": (C.c_int, [C.c_char_p, _PP]),
    "tycho_mesh_read_pmesh_partition": (C.c_int, [C.c_char_p, C.c_uint64, _PP]),
    "tycho_mesh_partition_info": (C.c_int, [_P, _U64P, _U64P, _U64P]),
    "tycho_mesh_side_tables": (C.c_int, [_P, _P, _P, _P]),
    "tycho_mesh_set_partition": (C.c_int, [_P, C.c_uint64, C.c_uint64, _P, _P]),
    "tycho_mesh_cell_material": (C.c_int, [_P, _P]),
    "tycho_sweeper_read_psi": (C.c_int, [_P, _P]),
    "tycho_mesh_kuhn_cube": (C.c_int, [C.c_uint32, C.c_double, C.c_uint64, C.c_double, _PP]),
    "tycho_mesh_from_arrays": (C.c_int, [C.c_uint64, C.c_uint64, _P, _P, _P, _P, _P, _PP]),
    "tycho_mesh_write_smesh": (C.c_int, [_P, C.c_char_p]),
    "tycho_mesh_write_pmesh": (C.c_int, [_P, C.c_char_p]),
    "tycho_mesh_info": (C.c_int, [_P, _U64P, _U64P, _U64P]),
    "tycho_mesh_tables": (C.c_int, [_P] + [_P] * 10),
    "tycho_mesh_free": (None, [_P]),
    "tycho_mesh_levels": (C.c_int, [_P, C.c_int, _P, _P, _P, _U32P]),
    "tycho_mesh_sweep_schedule_levels": (C.c_int, [_P, C.c_int, _P, _U32P]),
    "tycho_quadrature": (C.c_int, [C.c_int, _P, _P, _P, _P]),
    "tycho_sweeper_create": (C.c_int, [_P, C.POINTER(SweeperOpts), _PP]),
    "tycho_sweeper_create_angles": (C.c_int, [_P, C.POINTER(SweeperOpts), C.c_int, C.c_int, _PP]),
    "tycho_sweeper_apply": (C.c_int, [_P, C.c_int, _P, C.c_int, _P, _P]),
    "tycho_sweeper_destroy": (None, [_P]),
    "tycho_sweeper_set_cross_sections": (C.c_int, [_P, _P, _P, _P]),
    "tycho_sweeper_set_source": (C.c_int, [_P, C.c_int, _P]),
    "tycho_sweeper_sweep": (C.c_int, [_P, _P, _P]),
    "tycho_sweeper_solve": (C.c_int, [_P, C.POINTER(SolveOpts), _P, _P, C.POINTER(SolveStats)]),
    "tycho_sweeper_write_psi": (C.c_int, [_P, C.c_char_p]),
    "tycho_sweeper_schedule_info": (C.c_int, [_P, _U32P, _U64P, _U64P]),
    "tycho_sweeper_levels": (C.c_int, [_P, _P, _P, _P]),
    "tycho_sweeper_launches": (C.c_int, [_P, C.c_int, _U64P]),
    "tycho_release_cached_memory": (C.c_int, [C.c_int]),
    "tycho_device_memory": (C.c_int, [C.c_int, _U64P, _U64P]),
    "tycho_host_register": (C.c_int, [_P, C.c_size_t]),
    "tycho_host_unregister": (C.c_int, [_P]),
    "tycho_sweeper_schedule_arrays": (C.c_int, [_P, _U64P, _P, _P]),
    "tycho_sweeper_time_sweeps": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, _P]),
    "tycho_sweeper_autotune": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(LaunchShape),
                                         C.POINTER(C.c_double)]),
    "tycho_sweeper_configure": (C.c_int, [_P, C.c_int, C.POINTER(LaunchShape)]),
    "tycho_sweeper_get_shape": (C.c_int, [_P, C.c_int, C.POINTER(LaunchShape)]),
    "tycho_sweeper_sweep_noalloc": (C.c_int, [_P, C.c_int, _P, _P, _P]),
    "tycho_sweeper_set_wait_limit": (C.c_int, [_P, C.c_uint32]),
    "tycho_sweeper_set_work_order": (C.c_int, [_P, C.c_int]),
    "tycho_sweeper_bound_sides": (C.c_int, [_P, _U64P]),
    "tycho_sweeper_set_psi_bound": (C.c_int, [_P, _P]),
    "tycho_sweeper_get_psi_bound": (C.c_int, [_P, _P]),
    "tycho_sweeper_side_counts": (C.c_int, [_P, C.c_uint64, _U64P, _U64P]),
    "tycho_sweeper_side_send_list": (C.c_int, [_P, C.c_uint64, _P, _P]),
    "tycho_sweeper_side_pack": (C.c_int, [_P, C.c_uint64, _P, _P]),
    "tycho_sweeper_side_link": (C.c_int, [_P, C.c_uint64, C.c_uint64, _P, _P]),
    "tycho_sweeper_side_unpack": (C.c_int, [_P, C.c_uint64, _P, _P]),
    "tycho_sweeper_psi_change": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "tycho_batch_create": (C.c_int, [C.c_int, C.c_int, C.c_int, _PP]),
    "tycho_batch_destroy": (None, [_P]),
    "tycho_batch_set_persistent": (C.c_int, [_P, C.c_int]),
    "tycho_batch_set_wait_limit": (C.c_int, [_P, C.c_uint32]),
    "tycho_batch_add": (C.c_int, [_P, _P, C.POINTER(BatchOpts), C.POINTER(C.c_int)]),
    "tycho_batch_remove": (C.c_int, [_P, C.c_int]),
    "tycho_batch_step": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "tycho_batch_run": (C.c_int, [_P]),
    "tycho_batch_result": (C.c_int, [_P, C.c_int, _P, C.POINTER(SolveStats), C.POINTER(C.c_int)]),
    "tycho_batch_timing": (C.c_int, [_P, _P, _P, _P]),
}

class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("status", C.c_int), ("arrival", C.c_double),
                ("admitted", C.c_double), ("built", C.c_double), ("finished", C.c_double),
                ("footprint", C.c_uint64), ("stats", SolveStats)]


SIGNATURES.update({
    "tycho_footprint_bytes": (C.c_uint64, [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int]),
    "tycho_server_create": (C.c_int, [C.POINTER(ServerOpts), _PP]),
    "tycho_server_destroy": (None, [_P]),
    "tycho_server_submit": (C.c_int, [_P, _P, C.c_int, C.c_int, _P, _P, _P, _P, C.c_double, _P,
                                      C.POINTER(C.c_int)]),
    "tycho_server_run": (C.c_int, [_P]),
    "tycho_server_request": (C.c_int, [_P, C.c_int, C.POINTER(RequestInfo)]),
    "tycho_server_stats": (C.c_int, [_P, _P, C.POINTER(C.c_int), C.POINTER(C.c_int), _P]),
})

_lib = None


class TychoError(RuntimeError):
    """A nonzero tycho_status, with the library's message."""

    def __init__(self, status, message):
        self.status = status
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))


def lib():
    """Loads libtycho_b200.so once; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libtycho_b200.so is not built (%s); run __graft_entry__.build()" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != TYCHO_OK:
        buf = C.create_string_buffer(1024)
        lib().tycho_last_error(buf, 1024)
        raise TychoError(status, buf.value.decode(errors="replace"))


def ptr(a):
    """Raw pointer of a C-contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)
