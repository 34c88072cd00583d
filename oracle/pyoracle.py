"""ctypes binding of the CPU ORACLE (test infrastructure only).

Loaded by tests/, by ``__graft_entry__.smoke()`` as the checker, and by the
bench's CPU-baseline leg.  Never imported by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REPO = os.path.dirname(_HERE)
if _REPO not in sys.path:
    sys.path.insert(0, _REPO)

from dev_field_efvm_b200 import abi  # noqa: E402  (structs only)

_LIBS: dict = {}


def build() -> None:
    """Compile the oracle libraries (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib(parallel: bool = False) -> C.CDLL:
    name = "liboracle_omp.so" if parallel else "liboracle.so"
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(_HERE, "_build", name)
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    vp, dp, i64, i32 = C.c_void_p, C.POINTER(C.c_double), C.c_int64, C.c_int32
    L.oracle_create.restype = vp
    L.oracle_create.argtypes = [C.POINTER(abi.EfvmGrid), C.POINTER(abi.EfvmParams)]
    L.oracle_create_error.restype = C.c_char_p
    L.oracle_destroy.argtypes = [vp]
    L.oracle_set_option.argtypes = [vp, C.c_char_p, C.c_double]
    for fn in ("oracle_upload_state", "oracle_download_state"):
        getattr(L, fn).argtypes = [vp, dp, i64, i64, i64]
    for fn in ("oracle_upload_state3", "oracle_download_state3"):
        getattr(L, fn).argtypes = [vp, dp, i64, i64, i64, i64]
    L.oracle_raw_size.restype = i64
    L.oracle_raw_size.argtypes = [vp]
    L.oracle_get_raw_state.argtypes = [vp, dp]
    L.oracle_set_raw_state.argtypes = [vp, dp]
    L.oracle_init_vortex.argtypes = [vp, C.POINTER(abi.EfvmVortex)]
    L.oracle_vortex_state.argtypes = [C.POINTER(abi.EfvmVortex), C.c_double, dp, dp]
    L.oracle_density_error.argtypes = [vp, C.POINTER(abi.EfvmVortex), dp]
    L.oracle_total_mass.argtypes = [vp, dp]
    L.oracle_substep.argtypes = [vp]
    L.oracle_step.argtypes = [vp, i64, i32, C.c_double, dp, C.POINTER(abi.EfvmStepInfo)]
    L.oracle_cfl.argtypes = [vp, dp]
    L.oracle_get_solver_state.argtypes = [vp, C.POINTER(abi.EfvmSolverState)]
    L.oracle_set_solver_state.argtypes = [vp, C.POINTER(abi.EfvmSolverState)]
    L.oracle_set_cylinders.argtypes = [vp, C.POINTER(abi.EfvmCylinder), i32, dp]
    L.oracle_set_spheres.argtypes = [vp, C.POINTER(abi.EfvmSphere), i32, i32, dp]
    L.oracle_set_discs.argtypes = [vp, C.POINTER(abi.EfvmDisc), i32, i32, dp]
    L.oracle_sphere_markers.argtypes = [C.POINTER(abi.EfvmSphere), i32, dp]
    L.oracle_marker_force.argtypes = [vp, dp]
    L.oracle_wall_force.argtypes = [vp, dp]
    L.oracle_ibm_counts.argtypes = [vp, C.POINTER(i64), C.POINTER(i64)]
    L.oracle_apply_geometry.argtypes = [vp]
    L.oracle_body_loads.argtypes = [vp, i32, dp]
    L.oracle_get_mask.argtypes = [vp, C.POINTER(C.c_uint8)]
    L.oracle_flux.argtypes = [C.c_int, C.c_double, C.c_double, dp, dp, C.c_int, dp]
    L.oracle_flux_normal.argtypes = [C.c_int, C.c_double, C.c_double, dp, dp, dp, dp]
    L.oracle_physical_flux.argtypes = [C.c_double, C.c_double, dp, C.c_int, dp]
    L.oracle_cons_to_prim.argtypes = [C.c_double, C.c_double, dp, dp]
    L.oracle_prim_to_cons.argtypes = [C.c_double, C.c_double, dp, dp]
    for fn in ("oracle_sound_speed", "oracle_pressure"):
        getattr(L, fn).restype = C.c_double
        getattr(L, fn).argtypes = [C.c_double, C.c_double, dp]
    L.oracle_sutherland.restype = C.c_double
    L.oracle_sutherland.argtypes = [C.c_double]
    L.oracle_thermal_conductivity.restype = C.c_double
    L.oracle_thermal_conductivity.argtypes = [C.c_double, C.c_double, C.c_double]
    L.oracle_limiter.restype = C.c_double
    L.oracle_limiter.argtypes = [C.c_int, C.c_double, C.c_double]
    L.oracle_bc_ghost.argtypes = [C.POINTER(abi.EfvmBC), C.c_int, C.c_double, C.c_double, dp, dp]
    L.oracle_integrator_substep.restype = C.c_int
    L.oracle_integrator_substep.argtypes = [C.c_int, dp, dp, dp, i64, C.c_double, C.c_int, C.POINTER(C.c_int)]
    L.oracle_num_threads.restype = C.c_int
    L.oracle_is_parallel.restype = C.c_int
    _LIBS[name] = L
    return L


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def arr(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def sphere_markers(sphere: abi.EfvmSphere, n_markers: int) -> np.ndarray:
    """[n, 10]: position, normal, area, wall velocity of the Fibonacci markers."""
    L = lib()
    out = np.zeros((max(n_markers, 12), 10))
    n = L.oracle_sphere_markers(C.byref(sphere), int(n_markers), _dp(out))
    return out[:n]


class OracleCase:
    """One case on the CPU oracle: the App of the reference, substage by substage."""

    def __init__(self, grid: abi.EfvmGrid, params: abi.EfvmParams, parallel: bool = False):
        self.L = lib(parallel)
        self.grid, self.params = grid, params
        self.h = self.L.oracle_create(C.byref(grid), C.byref(params))
        if not self.h:
            raise ValueError(self.L.oracle_create_error().decode())
        self.nx, self.ny, self.nz = grid.nx, grid.ny, grid.nz

    def close(self):
        if self.h:
            self.L.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, name: str, value: float) -> None:
        assert self.L.oracle_set_option(self.h, name.encode(), float(value)) == 0

    # state as an (ny, nx, 5) array (2-D) or an (nz, ny, nx, 5) array (3-D):
    # rho, rho_u, rho_v, rho_w, rho_e
    def upload(self, u: np.ndarray) -> None:
        u = arr(u)
        if self.nz > 1:
            assert u.shape == (self.nz, self.ny, self.nx, 5)
            self.L.oracle_upload_state3(self.h, _dp(u), 5, 5 * self.nx, 5 * self.nx * self.ny, 1)
            return
        assert u.shape == (self.ny, self.nx, 5)
        self.L.oracle_upload_state(self.h, _dp(u), 5, 5 * self.nx, 1)

    def download(self) -> np.ndarray:
        if self.nz > 1:
            out = np.zeros((self.nz, self.ny, self.nx, 5))
            self.L.oracle_download_state3(self.h, _dp(out), 5, 5 * self.nx, 5 * self.nx * self.ny, 1)
            return out
        out = np.zeros((self.ny, self.nx, 5))
        self.L.oracle_download_state(self.h, _dp(out), 5, 5 * self.nx, 1)
        return out

    def init_vortex(self, v: abi.EfvmVortex) -> None:
        self.L.oracle_init_vortex(self.h, C.byref(v))

    def substep(self) -> None:
        self.L.oracle_substep(self.h)

    def step(self, n_steps: int, t_stop: float | None = None, history: bool = False):
        info = abi.EfvmStepInfo()
        hist = np.zeros((3 * n_steps, 6)) if history else None
        self.L.oracle_step(self.h, int(n_steps), 1 if t_stop is not None else 0,
                           float(t_stop if t_stop is not None else 0.0),
                           _dp(hist) if history else None, C.byref(info))
        if history:
            return info, hist[: info.substeps_done]
        return info

    def run_until(self, t_final: float, chunk: int = 1 << 30):
        """The case drivers' loop: whole RK3 steps until time >= t_final."""
        return self.step(chunk, t_stop=t_final)

    def cfl(self) -> float:
        d = C.c_double()
        self.L.oracle_cfl(self.h, C.byref(d))
        return d.value

    def solver_state(self) -> abi.EfvmSolverState:
        s = abi.EfvmSolverState()
        self.L.oracle_get_solver_state(self.h, C.byref(s))
        return s

    def set_solver_state(self, s: abi.EfvmSolverState) -> None:
        self.L.oracle_set_solver_state(self.h, C.byref(s))

    def set_cylinders(self, cyls, freestream) -> None:
        arr_t = abi.EfvmCylinder * len(cyls)
        ca = arr_t(*[abi.EfvmCylinder(*c) for c in cyls])
        fs = arr(freestream)
        self.L.oracle_set_cylinders(self.h, ca, len(cyls), _dp(fs))

    def set_discs(self, discs, freestream, n_theta: int = 64) -> None:
        """discs: abi.EfvmDisc values (moving 2-D bodies)."""
        arr_t = abi.EfvmDisc * max(len(discs), 1)
        da = arr_t(*discs)
        fs = arr(freestream)
        self.L.oracle_set_discs(self.h, da, len(discs), int(n_theta), _dp(fs))

    def set_spheres(self, spheres, freestream, n_markers: int = 2000) -> None:
        """spheres: abi.EfvmSphere values (abi.make_sphere)."""
        arr_t = abi.EfvmSphere * max(len(spheres), 1)
        sa = arr_t(*spheres)
        fs = arr(freestream)
        self.L.oracle_set_spheres(self.h, sa, len(spheres), int(n_markers), _dp(fs))

    def marker_force(self) -> np.ndarray:
        out = np.zeros(6)
        self.L.oracle_marker_force(self.h, _dp(out))
        return out

    def wall_force(self) -> np.ndarray:
        out = np.zeros(6)
        self.L.oracle_wall_force(self.h, _dp(out))
        return out

    def body_loads(self, n_bodies: int) -> np.ndarray:
        out = np.zeros((n_bodies, 9))
        self.L.oracle_body_loads(self.h, n_bodies, _dp(out))
        return out

    def apply_geometry(self) -> None:
        self.L.oracle_apply_geometry(self.h)

    def ibm_counts(self):
        a, b = C.c_int64(), C.c_int64()
        self.L.oracle_ibm_counts(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def mask(self) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), dtype=np.uint8)
        self.L.oracle_get_mask(self.h, out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out

    def density_error(self, v: abi.EfvmVortex):
        out = np.zeros(2)
        self.L.oracle_density_error(self.h, C.byref(v), _dp(out))
        return float(out[0]), float(out[1])

    def total_mass(self) -> float:
        d = C.c_double()
        self.L.oracle_total_mass(self.h, C.byref(d))
        return d.value

    def raw_state(self) -> np.ndarray:
        n = self.L.oracle_raw_size(self.h)
        out = np.zeros((n, 5))
        self.L.oracle_get_raw_state(self.h, _dp(out))
        return out


# ---- single-function helpers (known-answer tests) ---------------------------

def flux(scheme, left, right, dir, gamma=1.4, r_gas=287.058):
    out = np.zeros(5)
    lib().oracle_flux(scheme, gamma, r_gas, _dp(arr(left)), _dp(arr(right)), dir, _dp(out))
    return out


def flux_normal(scheme, owner, other, normal, gamma=1.4, r_gas=287.058):
    out = np.zeros(5)
    lib().oracle_flux_normal(scheme, gamma, r_gas, _dp(arr(owner)), _dp(arr(other)), _dp(arr(normal)), _dp(out))
    return out


def physical_flux(u, dir, gamma=1.4, r_gas=287.058):
    out = np.zeros(5)
    lib().oracle_physical_flux(gamma, r_gas, _dp(arr(u)), dir, _dp(out))
    return out


def cons_to_prim(u, gamma=1.4, r_gas=287.058):
    out = np.zeros(6)
    lib().oracle_cons_to_prim(gamma, r_gas, _dp(arr(u)), _dp(out))
    return out


def prim_to_cons(p, gamma=1.4, r_gas=287.058):
    out = np.zeros(5)
    lib().oracle_prim_to_cons(gamma, r_gas, _dp(arr(p)), _dp(out))
    return out


def sound_speed(u, gamma=1.4, r_gas=287.058):
    return lib().oracle_sound_speed(gamma, r_gas, _dp(arr(u)))


def pressure(u, gamma=1.4, r_gas=287.058):
    return lib().oracle_pressure(gamma, r_gas, _dp(arr(u)))


def sutherland(t):
    return lib().oracle_sutherland(t)


def thermal_conductivity(mu, gamma=1.4, r_gas=287.058):
    return lib().oracle_thermal_conductivity(mu, gamma, r_gas)


def limiter(kind, a, b):
    return lib().oracle_limiter(kind, a, b)


def bc_ghost(bc: abi.EfvmBC, side: int, interior, gamma=1.4, r_gas=287.058):
    out = np.zeros(5)
    lib().oracle_bc_ghost(C.byref(bc), side, gamma, r_gas, _dp(arr(interior)), _dp(out))
    return out


def integrator_substep(integrator, u, u0, rhs, dt, stage):
    u, u0, rhs = arr(u).copy(), arr(u0).copy(), arr(rhs)
    done = C.c_int()
    nxt = lib().oracle_integrator_substep(integrator, _dp(u), _dp(u0), _dp(rhs), u.shape[0], dt, stage, C.byref(done))
    return u, u0, nxt, bool(done.value)


def vortex_state(v: abi.EfvmVortex, t: float, x) -> np.ndarray:
    out = np.zeros(5)
    lib().oracle_vortex_state(C.byref(v), t, _dp(arr(list(x) + [0.0] * (3 - len(x)))), _dp(out))
    return out
