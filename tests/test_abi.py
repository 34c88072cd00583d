"""C-ABI checks that need no GPU: the library loads, exports every entry point
include/efvm.h declares, and the ctypes mirror matches the header's layouts."""
import ctypes as C
import os
import re
import subprocess

import pytest

from dev_field_efvm_b200 import abi, device

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "efvm.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(efvm_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from dev_field_efvm_b200 import build
    build.build()
    return device.load()


def test_library_exports_every_declared_symbol(lib):
    decl = declared_functions()
    assert len(decl) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", device.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (efvm_[a-z_0-9]+)", out))
    missing = [d for d in decl if d not in exported]
    assert not missing, missing
    assert sorted(decl) == sorted(device.EXPORTS)
    for name in decl:
        assert hasattr(lib, name)
    assert lib.efvm_abi_version() == abi.ABI_VERSION


def test_struct_layouts_match_the_header(tmp_path):
    probe = tmp_path / "probe.c"
    probe.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "efvm.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n\","
        "sizeof(efvm_bc),sizeof(efvm_grid),sizeof(efvm_params),sizeof(efvm_solver_state),"
        "sizeof(efvm_cylinder),sizeof(efvm_vortex),sizeof(efvm_step_info),"
        "offsetof(efvm_params,body_force_x),offsetof(efvm_grid,bc),"
        "sizeof(efvm_batch_case_result),offsetof(efvm_batch_case_result,finished));return 0;}\n")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(probe), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    want = [C.sizeof(abi.EfvmBC), C.sizeof(abi.EfvmGrid), C.sizeof(abi.EfvmParams), C.sizeof(abi.EfvmSolverState),
            C.sizeof(abi.EfvmCylinder), C.sizeof(abi.EfvmVortex), C.sizeof(abi.EfvmStepInfo),
            abi.EfvmParams.body_force_x.offset, abi.EfvmGrid.bc.offset,
            C.sizeof(abi.EfvmBatchCaseResult), abi.EfvmBatchCaseResult.finished.offset]
    assert got == want


def test_create_without_a_gpu_fails_loudly_or_rejects_bad_config(lib):
    # A half-periodic axis is rejected before any device work.
    g = abi.make_grid(8, 8, bcs={abi.XLO: abi.BC_PERIODIC})
    h = C.c_void_p()
    rc = lib.efvm_create(C.byref(g), C.byref(abi.make_params()), C.byref(h))
    assert rc == abi.ERR_INVALID_ARG
    assert b"periodic" in lib.efvm_last_error(None)
    # 3-D meshes run in FP64 without the 2-D case systems: those options are
    # rejected before any device work.
    g3 = abi.make_grid(8, 8, nz=4)
    p32 = abi.make_params(precision=abi.PREC_FP32_FLUX)
    assert lib.efvm_create(C.byref(g3), C.byref(p32), C.byref(h)) == abi.ERR_UNSUPPORTED
    assert b"FP64" in lib.efvm_last_error(None)
    pi = abi.make_params(parabolic_inflow=1, inflow_u_max=1.0, inflow_height=1.0, inflow_rho=1.0)
    assert lib.efvm_create(C.byref(g3), C.byref(pi), C.byref(h)) == abi.ERR_UNSUPPORTED
    assert b"parabolic" in lib.efvm_last_error(None)
    g0 = abi.make_grid(8, 8, nz=0)
    assert lib.efvm_create(C.byref(g0), C.byref(abi.make_params()), C.byref(h)) == abi.ERR_INVALID_ARG
