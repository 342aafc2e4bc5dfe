"""The C ABI library loads, exports every function include/tycho_cuda.h
declares, and refuses to sweep without a GPU (there is no CPU fallback)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT, gpu_available


def declared_functions():
    text = open(os.path.join(ROOT, "include", "tycho_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tycho_\w+)\s*\(", text)))


def test_header_declares_the_abi():
    names = declared_functions()
    for required in ("tycho_sweeper_create", "tycho_sweeper_sweep", "tycho_sweeper_solve",
                     "tycho_mesh_read_pmesh", "tycho_quadrature"):
        assert required in names


def test_library_exports_every_declared_symbol(built):
    from tycho2_b200._capi import LIB_PATH, SIGNATURES
    lib = ctypes.CDLL(LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name
        assert name in SIGNATURES, "binding missing for %s" % name


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU failure mode")
def test_sweeper_fails_loudly_without_gpu(built):
    import tycho2_b200 as ty
    mesh = ty.TychoMesh.kuhn_cube(2)
    with pytest.raises(ty.TychoError) as e:
        ty.SweeperCuda(mesh, 4, 1)
    assert e.value.status == 4 and "no CPU fallback" in str(e.value)


def test_footprint_estimate_covers_psi_and_records():
    """Admission estimate (no device needed): at least psi (FP64) plus the
    per-item records of both precisions, growing with cells, groups, order."""
    import tycho2_b200 as ty
    for nc, sn, G in [(384, 4, 1), (82944, 8, 8), (663552, 8, 8)]:
        A = 2 * sn * sn
        b = ty.footprint_bytes(nc, sn, G, True, False)
        assert b >= nc * A * (4 * G * 8 + 256 + 128)
        assert ty.footprint_bytes(nc, sn, G, True, True) >= nc * A * (4 * G * 8 + 96 + 64)
        assert ty.footprint_bytes(nc, sn, G, True, True) < b
        assert ty.footprint_bytes(nc, sn, G, False, False) < b
        assert ty.footprint_bytes(2 * nc, sn, G, True, False) > b
        assert ty.footprint_bytes(nc, sn, 2 * G, True, False) > b


def test_header_is_plain_c(tmp_path):
    """The boundary is a C ABI: the header compiles as strict C99 (a cgo,
    JNI or ctypes binding sees no C++), and every struct zero-initialises."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "abi.c"
    src.write_text('#include "tycho_cuda.h"\n'
                   "int main(void) {\n"
                   "    tycho_sweeper_opts o = {0}; tycho_launch_shape s = {0};\n"
                   "    tycho_solve_opts so = {0}; tycho_batch_opts b = {0}; tycho_server_opts sv = {0};\n"
                   "    (void)o; (void)s; (void)so; (void)b; (void)sv; return 0;\n"
                   "}\n")
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                        "-I" + os.path.join(ROOT, "include"), "-c", str(src), "-o", str(tmp_path / "abi.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
