"""efvm_cfl_dt_noalloc against efvm_cfl.

The no-allocation entry point serves callers whose device memory belongs to
another allocator, so they pass every buffer themselves: here the test owns the
conserved planes (torch tensors with a row pitch wider than the grid) and the
one-double output.  Two calls in a row on different cases must give the same dt
as the context path's efvm_cfl within the parity tolerance of the GPU tests
(1e-12 relative); the second call also checks that the shared static scratch
left over from the first does not leak into it.  This file is collected last so
that a run stopping at the first failure has run every other test already; it
also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from dev_field_efvm_b200 import abi, device
from dev_field_efvm_b200.device import Context
from dev_field_efvm_b200 import cases

pytestmark = pytest.mark.gpu
TOL = 1e-12


def noalloc_dt(grid, params, u, pitch_pad=5):
    import torch
    ny, nx = u.shape[0], u.shape[1]
    pitch = nx + pitch_pad
    planes = []
    for v in (0, 1, 2, 4):  # rho, rho_u, rho_v, rho_e
        t = torch.zeros((ny, pitch), dtype=torch.float64, device="cuda")
        t[:, :nx] = torch.from_numpy(np.ascontiguousarray(u[..., v]))
        planes.append(t)
    dt = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    L = device.load()
    rc = L.efvm_cfl_dt_noalloc(*[C.c_void_p(t.data_ptr()) for t in planes], pitch, C.byref(grid), C.byref(params),
                               C.c_void_p(dt.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert rc == abi.OK, L.efvm_last_error(None).decode()
    stream.synchronize()
    return float(dt.item())


def context_dt(grid, params, u):
    with Context(grid, params) as ctx:
        ctx.upload(u)
        return ctx.cfl()


def test_noalloc_cfl_matches_context_cfl_on_two_calls():
    import torch
    torch.cuda.init()
    # call 1: the periodic vortex, inviscid, 256 x 192
    g1, p1, u1, _ = cases.vortex_case(256, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4, ny=192)
    a1 = noalloc_dt(g1, p1, u1)
    b1 = context_dt(g1, p1, u1)
    assert abs(a1 - b1) <= TOL * b1, (a1, b1)
    # call 2: the viscous cylinder channel, fewer rows than call 1 (stale scratch rows beyond ny)
    g2, p2, u2, _ = cases.cylinder_case(220, 41, muscl=True)
    a2 = noalloc_dt(g2, p2, u2, pitch_pad=11)
    b2 = context_dt(g2, p2, u2)
    assert abs(a2 - b2) <= TOL * b2, (a2, b2)
    assert abs(a1 - a2) > 1e-6 * a1  # the two cases really differ


def test_noalloc_rejects_grids_beyond_its_scratch():
    L = device.load()
    g = abi.make_grid(8, 16385)
    p = abi.make_params()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.efvm_cfl_dt_noalloc(dummy, dummy, dummy, dummy, 8, C.byref(g), C.byref(p), dummy, None)
    assert rc == abi.ERR_INVALID_ARG
    assert b"16384-row scratch" in L.efvm_last_error(None)
