"""efvm_cfl_dt_noalloc against efvm_cfl.

The no-allocation entry point serves callers whose device memory belongs to
another allocator, so they pass every buffer themselves: here the test owns the
conserved planes (torch tensors with a row pitch wider than the grid) and the
one-double output.  Calls in a row on different cases must give exactly the dt
of the context path's efvm_cfl: both evaluate the same wave speed with every
operation rounded explicitly, and a maximum does not depend on the order of
the reduction.  The cases cover an inviscid vortex, a viscous channel with
constant viscosity, the same channel with Sutherland's law, and a fixed dt;
each call after the first also checks that the shared static scratch left over
from the call before does not leak into it.  The argument checks (rows beyond
the scratch, 3-D meshes, non-positive extents) run without a GPU.

This file is collected last so that a run stopping at the first failure has run
every other test already; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from dev_field_efvm_b200 import abi, device
from dev_field_efvm_b200.device import Context
from dev_field_efvm_b200 import cases


def with_params(params, **changes):
    p = abi.make_params(**{f: getattr(params, f) for f, _ in abi.EfvmParams._fields_})
    for k, v in changes.items():
        setattr(p, k, type(getattr(p, k))(v))
    return p


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


@pytest.mark.gpu
def test_noalloc_cfl_equals_context_cfl_on_calls_in_a_row():
    import torch
    torch.cuda.init()
    got = []
    # call 1: the periodic vortex, inviscid, 256 x 192
    g1, p1, u1, _ = cases.vortex_case(256, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4, ny=192)
    a1 = noalloc_dt(g1, p1, u1)
    assert a1 == context_dt(g1, p1, u1)
    got.append(a1)
    # call 2: the viscous cylinder channel (constant viscosity), fewer rows than
    # call 1, so rows of the scratch beyond ny hold stale maxima
    g2, p2, u2, _ = cases.cylinder_case(220, 41, muscl=True)
    a2 = noalloc_dt(g2, p2, u2, pitch_pad=11)
    assert a2 == context_dt(g2, p2, u2)
    got.append(a2)
    # call 3: the same channel with Sutherland's law (T about 348 K)
    p3 = with_params(p2, viscosity_model=abi.VISC_SUTHERLAND)
    a3 = noalloc_dt(g2, p3, u2, pitch_pad=3)
    assert a3 == context_dt(g2, p3, u2)
    got.append(a3)
    # call 4: a fixed dt overrides the wave speed
    p4 = with_params(p1, fixed_dt=1.25e-3)
    a4 = noalloc_dt(g1, p4, u1)
    assert a4 == 1.25e-3 == context_dt(g1, p4, u1)
    # call 5: call 1 again after the others, with a different pitch
    assert noalloc_dt(g1, p1, u1, pitch_pad=17) == a1
    # the cases really differ, so a leaked maximum would show
    assert len({round(x, 15) for x in got}) == 3, got


def test_noalloc_rejects_grids_beyond_its_scratch():
    L = device.load()
    g = abi.make_grid(8, abi.CFL_NOALLOC_MAX_ROWS + 1)
    p = abi.make_params()
    dummy = C.c_void_p(16)  # never dereferenced: the argument checks come first
    rc = L.efvm_cfl_dt_noalloc(dummy, dummy, dummy, dummy, 8, C.byref(g), C.byref(p), dummy, None)
    assert rc == abi.ERR_INVALID_ARG
    assert b"16384-row scratch" in L.efvm_last_error(None)


def test_noalloc_rejects_3d_meshes_and_empty_extents():
    L = device.load()
    p = abi.make_params()
    dummy = C.c_void_p(16)  # never dereferenced: the argument checks come first
    g3 = abi.make_grid(8, 8, nz=4)
    rc = L.efvm_cfl_dt_noalloc(dummy, dummy, dummy, dummy, 8, C.byref(g3), C.byref(p), dummy, None)
    assert rc == abi.ERR_UNSUPPORTED
    assert b"2-D meshes" in L.efvm_last_error(None)
    for axis in range(3):
        g = abi.make_grid(8, 8)
        g.hi[axis] = g.lo[axis]  # zero extent: dx = 0
        rc = L.efvm_cfl_dt_noalloc(dummy, dummy, dummy, dummy, 8, C.byref(g), C.byref(p), dummy, None)
        assert rc == abi.ERR_INVALID_ARG
        assert b"extent" in L.efvm_last_error(None)
    g = abi.make_grid(8, 8, lo=(1.0, 0.0, 0.0), hi=(0.0, 1.0, 1.0))  # reversed bounds: dx < 0
    rc = L.efvm_cfl_dt_noalloc(dummy, dummy, dummy, dummy, 8, C.byref(g), C.byref(p), dummy, None)
    assert rc == abi.ERR_INVALID_ARG
