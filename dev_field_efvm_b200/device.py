"""ctypes binding of libefvm_b200.so (the C-ABI of include/efvm.h).

This is the product path: every call goes to the CUDA library.  There is no
CPU fallback; importing a context without the built library or without a CUDA
device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libefvm_b200.so")
_LIB = None

# every entry point of include/efvm.h
EXPORTS = (
    "efvm_abi_version", "efvm_create", "efvm_destroy", "efvm_last_error", "efvm_upload_state",
    "efvm_download_state", "efvm_upload_state_3d", "efvm_download_state_3d", "efvm_set_spheres", "efvm_set_discs", "efvm_get_solver_state", "efvm_set_solver_state", "efvm_substep", "efvm_step",
    "efvm_cfl", "efvm_set_cylinders", "efvm_marker_force", "efvm_wall_force", "efvm_ibm_counts", "efvm_get_solid_mask",
    "efvm_density_error", "efvm_init_vortex", "efvm_total_mass", "efvm_get_stream", "efvm_launch_count",
    "efvm_profile_steps", "efvm_set_stage_tiling", "efvm_get_stage_tiling", "efvm_autotune_stage", "efvm_set_stage_wait_limit", "efvm_inject_stage_stall", "efvm_create_slab", "efvm_prepare", "efvm_halo_pack", "efvm_halo_unpack",
    "efvm_wave_speed_slot", "efvm_get_state_buffers", "efvm_set_halo_peer", "efvm_get_state_ipc", "efvm_set_halo_peer_ipc", "efvm_batch_create", "efvm_batch_destroy", "efvm_batch_last_error",
    "efvm_batch_upload_state", "efvm_batch_download_state", "efvm_batch_get_solver_state", "efvm_batch_run",
    "efvm_batch_launch_count", "efvm_batch_get_stream", "efvm_batch_set_autotune", "efvm_batch_get_rows",
    "efvm_batch_set_persistent", "efvm_batch_set_wait_limit", "efvm_batch_inject_stall", "efvm_batch_get_blocks_per_sm",
    "efvm_nn_gemm_bf16", "efvm_body_loads", "efvm_output_fields", "efvm_synchronize", "efvm_write_vtk", "efvm_nn_param_count", "efvm_nn_create",
    "efvm_nn_destroy", "efvm_nn_get_params", "efvm_nn_set_params", "efvm_nn_get_scale", "efvm_nn_forward",
    "efvm_nn_loss_grad", "efvm_nn_adam", "efvm_set_flux_correction", "efvm_correction_stats", "efvm_cfl_dt_noalloc",
)


class EfvmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"efvm error {abi.STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def load(path: str | None = None) -> C.CDLL:
    """Load the library (build it first with ``python -m dev_field_efvm_b200.build``)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(f"{p} is missing: build it with `python -m dev_field_efvm_b200.build`")
    L = C.CDLL(p)
    vp, dp, i64, i32 = C.c_void_p, C.POINTER(C.c_double), C.c_int64, C.c_int32
    L.efvm_abi_version.restype = C.c_int
    L.efvm_create.argtypes = [C.POINTER(abi.EfvmGrid), C.POINTER(abi.EfvmParams), C.POINTER(vp)]
    L.efvm_destroy.argtypes = [vp]
    L.efvm_last_error.restype = C.c_char_p
    L.efvm_last_error.argtypes = [vp]
    L.efvm_upload_state.argtypes = [vp, dp, i64, i64, i64]
    L.efvm_download_state.argtypes = [vp, dp, i64, i64, i64]
    L.efvm_upload_state_3d.argtypes = [vp, dp, i64, i64, i64, i64]
    L.efvm_set_spheres.argtypes = [vp, C.POINTER(abi.EfvmSphere), i32, i32, dp]
    L.efvm_set_discs.argtypes = [vp, C.POINTER(abi.EfvmDisc), i32, i32, dp]
    L.efvm_download_state_3d.argtypes = [vp, dp, i64, i64, i64, i64]
    L.efvm_get_solver_state.argtypes = [vp, C.POINTER(abi.EfvmSolverState)]
    L.efvm_set_solver_state.argtypes = [vp, C.POINTER(abi.EfvmSolverState)]
    L.efvm_substep.argtypes = [vp]
    L.efvm_step.argtypes = [vp, i64, i32, C.c_double, dp, C.POINTER(abi.EfvmStepInfo)]
    L.efvm_cfl.argtypes = [vp, dp]
    L.efvm_set_cylinders.argtypes = [vp, C.POINTER(abi.EfvmCylinder), i32, dp]
    L.efvm_marker_force.argtypes = [vp, dp]
    L.efvm_wall_force.argtypes = [vp, dp]
    L.efvm_ibm_counts.argtypes = [vp, C.POINTER(i64), C.POINTER(i64)]
    L.efvm_get_solid_mask.argtypes = [vp, C.POINTER(C.c_uint8)]
    L.efvm_density_error.argtypes = [vp, C.POINTER(abi.EfvmVortex), dp]
    L.efvm_init_vortex.argtypes = [vp, C.POINTER(abi.EfvmVortex)]
    L.efvm_total_mass.argtypes = [vp, dp]
    L.efvm_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.efvm_launch_count.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.efvm_profile_steps.argtypes = [vp, i64, dp]
    L.efvm_set_stage_tiling.argtypes = [vp, i32, i32, i32]
    L.efvm_get_stage_tiling.argtypes = [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
    L.efvm_autotune_stage.argtypes = [vp, i32, dp]
    L.efvm_set_stage_wait_limit.argtypes = [vp, C.c_double]
    L.efvm_inject_stage_stall.argtypes = [vp, i32]
    L.efvm_create_slab.argtypes = [C.POINTER(abi.EfvmGrid), C.POINTER(abi.EfvmParams), i32, i32, C.POINTER(vp)]
    L.efvm_prepare.argtypes = [vp]
    L.efvm_halo_pack.argtypes = [vp, i32, vp]
    L.efvm_halo_unpack.argtypes = [vp, i32, vp]
    L.efvm_wave_speed_slot.argtypes = [vp, C.POINTER(vp)]
    L.efvm_get_state_buffers.argtypes = [vp, C.POINTER(vp), C.POINTER(i64), C.POINTER(i32)]
    L.efvm_set_halo_peer.argtypes = [vp, i32, C.POINTER(vp), i64, i32]
    L.efvm_get_state_ipc.argtypes = [vp, C.c_char_p]
    L.efvm_set_halo_peer_ipc.argtypes = [vp, i32, C.c_char_p, i64, i32]
    L.efvm_batch_create.argtypes = [C.POINTER(abi.EfvmGrid), i32, C.POINTER(abi.EfvmParams), C.POINTER(vp)]
    L.efvm_batch_destroy.argtypes = [vp]
    L.efvm_batch_last_error.restype = C.c_char_p
    L.efvm_batch_last_error.argtypes = [vp]
    L.efvm_batch_upload_state.argtypes = [vp, i32, dp, i64, i64, i64]
    L.efvm_batch_download_state.argtypes = [vp, i32, dp, i64, i64, i64]
    L.efvm_batch_get_solver_state.argtypes = [vp, i32, C.POINTER(abi.EfvmSolverState)]
    L.efvm_batch_run.argtypes = [vp, dp, i64, i64, C.POINTER(abi.EfvmBatchCaseResult)]
    L.efvm_batch_launch_count.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.efvm_batch_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.efvm_batch_set_autotune.argtypes = [vp, i32]
    L.efvm_batch_get_rows.argtypes = [vp, C.POINTER(C.c_int32)]
    L.efvm_batch_set_persistent.argtypes = [vp, i32]
    L.efvm_batch_set_wait_limit.argtypes = [vp, C.c_double]
    L.efvm_batch_inject_stall.argtypes = [vp, i32]
    L.efvm_batch_get_blocks_per_sm.argtypes = [vp, C.POINTER(C.c_int32)]
    L.efvm_nn_gemm_bf16.argtypes = [vp, vp, vp, i32, i32, i32, vp]
    L.efvm_body_loads.argtypes = [vp, i32, dp]
    L.efvm_output_fields.argtypes = [vp, dp, i32]
    L.efvm_synchronize.argtypes = [vp]
    L.efvm_write_vtk.argtypes = [vp, C.c_char_p]
    L.efvm_nn_param_count.restype = C.c_int
    L.efvm_nn_create.argtypes = [C.c_float, C.c_float, C.c_uint64, C.POINTER(vp)]
    L.efvm_nn_destroy.argtypes = [vp]
    L.efvm_nn_get_params.argtypes = [vp, C.POINTER(C.c_float)]
    L.efvm_nn_set_params.argtypes = [vp, C.POINTER(C.c_float)]
    L.efvm_nn_get_scale.argtypes = [vp, C.POINTER(C.c_float)]
    L.efvm_nn_forward.argtypes = [vp, vp, i32, i32, i32, vp, vp]
    L.efvm_nn_loss_grad.argtypes = [vp, vp, vp, i32, i32, i32, C.c_double, C.c_double, C.POINTER(C.c_float), vp,
                                    C.POINTER(C.c_double), vp]
    L.efvm_nn_adam.argtypes = [vp, C.c_float, vp]
    L.efvm_set_flux_correction.argtypes = [vp, vp, C.c_float]
    L.efvm_correction_stats.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.efvm_cfl_dt_noalloc.argtypes = [vp, vp, vp, vp, i64, C.POINTER(abi.EfvmGrid), C.POINTER(abi.EfvmParams), vp, vp]
    if L.efvm_abi_version() != abi.ABI_VERSION:
        raise ImportError("libefvm_b200.so ABI version mismatch")
    if path is None:
        _LIB = L
    return L


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Context:
    """One case on the GPU: an efvm_ctx and its device state."""

    def __init__(self, grid: abi.EfvmGrid, params: abi.EfvmParams, rows: tuple[int, int] | None = None):
        """rows = (row0, n): a slab of global rows [row0, row0 + n) (efvm_create_slab)."""
        self.L = load()
        self.grid, self.params = grid, params
        self.nx, self.nz = grid.nx, grid.nz
        self.row0, self.ny = (0, grid.ny) if rows is None else (int(rows[0]), int(rows[1]))
        h = C.c_void_p()
        if rows is None:
            rc = self.L.efvm_create(C.byref(grid), C.byref(params), C.byref(h))
        else:
            rc = self.L.efvm_create_slab(C.byref(grid), C.byref(params), self.row0, self.ny, C.byref(h))
        if rc != abi.OK:
            raise EfvmError(rc, self.L.efvm_last_error(None).decode())
        self.h = h

    def _check(self, rc: int) -> None:
        if rc != abi.OK:
            raise EfvmError(rc, self.L.efvm_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.efvm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # conserved state as an (ny, nx, 5) array: rho, rho_u, rho_v, rho_w, rho_e
    def upload(self, u: np.ndarray) -> None:
        """u: [ny, nx, 5] (2-D) or [nz, ny, nx, 5] (3-D) conserved states."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        if self.nz > 1:
            assert u.shape == (self.nz, self.ny, self.nx, 5), u.shape
            self._check(self.L.efvm_upload_state_3d(self.h, _dp(u), 5, 5 * self.nx, 5 * self.nx * self.ny, 1))
            return
        assert u.shape == (self.ny, self.nx, 5), u.shape
        self._check(self.L.efvm_upload_state(self.h, _dp(u), 5, 5 * self.nx, 1))

    def upload_ptr(self, ptr: int, si: int, sj: int, sv: int) -> None:
        self._check(self.L.efvm_upload_state(self.h, C.cast(ptr, C.POINTER(C.c_double)), si, sj, sv))

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        if self.nz > 1:
            if out is None:
                out = np.zeros((self.nz, self.ny, self.nx, 5))
            self._check(self.L.efvm_download_state_3d(self.h, _dp(out), 5, 5 * self.nx, 5 * self.nx * self.ny, 1))
            return out
        if out is None:
            out = np.zeros((self.ny, self.nx, 5))
        self._check(self.L.efvm_download_state(self.h, _dp(out), 5, 5 * self.nx, 1))
        return out

    def download_ptr(self, ptr: int, si: int, sj: int, sv: int) -> None:
        self._check(self.L.efvm_download_state(self.h, C.cast(ptr, C.POINTER(C.c_double)), si, sj, sv))

    def upload_ptr3(self, ptr: int, si: int, sj: int, sk: int, sv: int) -> None:
        self._check(self.L.efvm_upload_state_3d(self.h, C.cast(ptr, C.POINTER(C.c_double)), si, sj, sk, sv))

    def download_ptr3(self, ptr: int, si: int, sj: int, sk: int, sv: int) -> None:
        self._check(self.L.efvm_download_state_3d(self.h, C.cast(ptr, C.POINTER(C.c_double)), si, sj, sk, sv))

    def substep(self) -> None:
        self._check(self.L.efvm_substep(self.h))

    # ---- learned flux correction ----
    def set_flux_correction(self, net, sensor: float = 0.2) -> None:
        self._check(self.L.efvm_set_flux_correction(self.h, net.h if net is not None else None, sensor))
        self._net = net  # keep the network alive while attached

    def correction_stats(self):
        a, b = C.c_uint64(), C.c_uint64()
        self._check(self.L.efvm_correction_stats(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    # ---- slabs (efvm_create_slab) ----
    def prepare(self) -> None:
        self._check(self.L.efvm_prepare(self.h))

    def halo_pack(self, side: int, dev_ptr: int) -> None:
        self._check(self.L.efvm_halo_pack(self.h, side, C.c_void_p(dev_ptr)))

    def halo_unpack(self, side: int, dev_ptr: int) -> None:
        self._check(self.L.efvm_halo_unpack(self.h, side, C.c_void_p(dev_ptr)))

    def state_buffers(self) -> tuple[list[int], int, int]:
        """Device addresses of the three state buffers, their plane (doubles) and the rows."""
        bufs = (C.c_void_p * 3)()
        plane, rows = C.c_int64(), C.c_int32()
        self._check(self.L.efvm_get_state_buffers(self.h, bufs, C.byref(plane), C.byref(rows)))
        return [int(b) for b in bufs], plane.value, rows.value

    def set_halo_peer(self, side: int, bufs: list[int] | None, plane: int = 0, rows: int = 0) -> None:
        """Store this slab's edge rows of `side` into the neighbour's buffers (None: pack / unpack)."""
        arr = None if bufs is None else (C.c_void_p * 3)(*bufs)
        self._check(self.L.efvm_set_halo_peer(self.h, int(side), arr, int(plane), int(rows)))

    def state_ipc(self) -> bytes:
        """CUDA IPC handles of the three state buffers (3 x 64 bytes)."""
        buf = C.create_string_buffer(3 * 64)
        self._check(self.L.efvm_get_state_ipc(self.h, buf))
        return buf.raw

    def set_halo_peer_ipc(self, side: int, handles: bytes, plane: int, rows: int) -> None:
        """Map another process's state buffers (efvm_get_state_ipc) as the side's halo peer."""
        self._check(self.L.efvm_set_halo_peer_ipc(self.h, int(side), bytes(handles), int(plane), int(rows)))

    def wave_speed_slot(self) -> int:
        """Device address of the external wave-speed slot (a uint64)."""
        p = C.c_void_p()
        self._check(self.L.efvm_wave_speed_slot(self.h, C.byref(p)))
        return int(p.value)

    def step_async(self, n_steps: int) -> None:
        """Enqueue whole steps on the context's stream without waiting."""
        self._check(self.L.efvm_step(self.h, int(n_steps), 0, 0.0, None, None))

    def profile_steps(self, n_steps: int) -> np.ndarray:
        """Device ms of [stage kernels, IBM kernels, step set-up, whole steps]."""
        out = np.zeros(4)
        self._check(self.L.efvm_profile_steps(self.h, int(n_steps), _dp(out)))
        return out

    def set_stage_tiling(self, form: int = abi.STAGE_AUTO, rows_per_warp: int = 0, blocks_per_sm: int = 0) -> None:
        """Stage-kernel form (abi.STAGE_*), rows per warp and blocks per SM (0: built-in)."""
        self._check(self.L.efvm_set_stage_tiling(self.h, int(form), int(rows_per_warp), int(blocks_per_sm)))

    def stage_tiling(self) -> tuple[int, int, int]:
        """(form the next stage runs, its rows per warp, its blocks per SM)."""
        f, r, b = C.c_int32(), C.c_int32(), C.c_int32()
        self._check(self.L.efvm_get_stage_tiling(self.h, C.byref(f), C.byref(r), C.byref(b)))
        return f.value, r.value, b.value

    def set_stage_wait_limit(self, seconds: float) -> None:
        self._check(self.L.efvm_set_stage_wait_limit(self.h, float(seconds)))

    def inject_stage_stall(self, enable: bool) -> None:
        """Test hook: the TMA-fed stage's first block stops refilling its ring."""
        self._check(self.L.efvm_inject_stage_stall(self.h, 1 if enable else 0))

    def autotune_stage(self, n_steps: int = 3) -> float:
        """Keep the fastest stage tiling (state restored); device ms per step."""
        ms = C.c_double()
        self._check(self.L.efvm_autotune_stage(self.h, int(n_steps), C.byref(ms)))
        return ms.value

    def step(self, n_steps: int, t_stop: float | None = None, history: bool = False):
        info = abi.EfvmStepInfo()
        hist = np.zeros((3 * max(n_steps, 1), 6)) if history else None
        rc = self.L.efvm_step(self.h, int(n_steps), 1 if t_stop is not None else 0,
                              float(t_stop if t_stop is not None else 0.0),
                              _dp(hist) if history else None, C.byref(info))
        self._check(rc)
        if history:
            return info, hist[: info.substeps_done]
        return info

    def run_until(self, t_final: float, max_steps: int = 10_000_000):
        return self.step(max_steps, t_stop=t_final)

    def cfl(self) -> float:
        d = C.c_double()
        self._check(self.L.efvm_cfl(self.h, C.byref(d)))
        return d.value

    def solver_state(self) -> abi.EfvmSolverState:
        s = abi.EfvmSolverState()
        self._check(self.L.efvm_get_solver_state(self.h, C.byref(s)))
        return s

    def set_solver_state(self, s: abi.EfvmSolverState) -> None:
        self._check(self.L.efvm_set_solver_state(self.h, C.byref(s)))

    def set_cylinders(self, cyls, freestream) -> None:
        arr_t = abi.EfvmCylinder * max(len(cyls), 1)
        ca = arr_t(*[abi.EfvmCylinder(*c) for c in cyls])
        fs = np.ascontiguousarray(freestream, dtype=np.float64)
        self._check(self.L.efvm_set_cylinders(self.h, ca, len(cyls), _dp(fs)))

    def set_discs(self, discs, freestream, n_theta: int = 64) -> None:
        """Moving 2-D discs (abi.EfvmDisc values); call again between steps to move them."""
        arr_t = abi.EfvmDisc * max(len(discs), 1)
        da = arr_t(*discs)
        fs = np.ascontiguousarray(freestream, dtype=np.float64)
        self._check(self.L.efvm_set_discs(self.h, da, len(discs), int(n_theta), _dp(fs)))

    def set_spheres(self, spheres, freestream, n_markers: int = 2000) -> None:
        """Immersed spheres (abi.make_sphere values) on a 3-D context; call again
        between steps to move them."""
        arr_t = abi.EfvmSphere * max(len(spheres), 1)
        sa = arr_t(*spheres)
        fs = np.ascontiguousarray(freestream, dtype=np.float64)
        self._check(self.L.efvm_set_spheres(self.h, sa, len(spheres), int(n_markers), _dp(fs)))

    def marker_force(self) -> np.ndarray:
        out = np.zeros(6)
        self._check(self.L.efvm_marker_force(self.h, _dp(out)))
        return out

    def output_fields(self, out: np.ndarray | None = None, wait: bool = True) -> np.ndarray:
        """(7, ny, nx): density, pressure, temperature, u, v, w, Mach.  With
        wait=False the copy is only enqueued (call synchronize() before use)."""
        if out is None:
            out = np.zeros((7, self.ny, self.nx))
        self._check(self.L.efvm_output_fields(self.h, _dp(out), 0 if wait else 1))
        return out

    def synchronize(self) -> None:
        self._check(self.L.efvm_synchronize(self.h))

    def write_vtk(self, path: str) -> None:
        self._check(self.L.efvm_write_vtk(self.h, path.encode()))

    def body_loads(self, n_bodies: int) -> np.ndarray:
        """[n_bodies, 9]: pressure force, viscous force, torque about the centre."""
        out = np.zeros((n_bodies, 9))
        self._check(self.L.efvm_body_loads(self.h, n_bodies, _dp(out)))
        return out

    def wall_force(self) -> np.ndarray:
        out = np.zeros(6)
        self._check(self.L.efvm_wall_force(self.h, _dp(out)))
        return out

    def apply_geometry(self) -> None:
        """Apply cylinders set since the last step to the current state now: the
        solid mask, the stagnant re-seed of cells that turn solid and the IBM
        lists (the Setup phase of the next substage would do the same).  A
        restore calls it before loading its fields, so that they are not
        re-seeded afterwards."""
        self.ibm_counts()

    def ibm_counts(self):
        a, b = C.c_int64(), C.c_int64()
        self._check(self.L.efvm_ibm_counts(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def solid_mask(self) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), dtype=np.uint8)
        self._check(self.L.efvm_get_solid_mask(self.h, out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out

    def density_error(self, v: abi.EfvmVortex):
        out = np.zeros(2)
        self._check(self.L.efvm_density_error(self.h, C.byref(v), _dp(out)))
        return float(out[0]), float(out[1])

    def init_vortex(self, v: abi.EfvmVortex) -> None:
        self._check(self.L.efvm_init_vortex(self.h, C.byref(v)))

    def total_mass(self) -> float:
        d = C.c_double()
        self._check(self.L.efvm_total_mass(self.h, C.byref(d)))
        return d.value

    def stream(self) -> int:
        p = C.c_void_p()
        self._check(self.L.efvm_get_stream(self.h, C.byref(p)))
        return p.value or 0

    def launch_count(self) -> int:
        n = C.c_uint64()
        self._check(self.L.efvm_launch_count(self.h, C.byref(n)))
        return n.value


class Batch:
    """Many independent cases advanced together (efvm_batch_*)."""

    def __init__(self, grids, params: abi.EfvmParams):
        self.L = load()
        self.n = len(grids)
        self.shapes = [(g.ny, g.nx) for g in grids]
        arr = (abi.EfvmGrid * self.n)(*grids)
        h = C.c_void_p()
        rc = self.L.efvm_batch_create(arr, self.n, C.byref(params), C.byref(h))
        if rc != abi.OK:
            raise EfvmError(rc, self.L.efvm_batch_last_error(None).decode())
        self.h = h

    def _check(self, rc: int) -> None:
        if rc != abi.OK:
            raise EfvmError(rc, self.L.efvm_batch_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.efvm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, k: int, u: np.ndarray) -> None:
        ny, nx = self.shapes[k]
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.shape == (ny, nx, 5), u.shape
        self._check(self.L.efvm_batch_upload_state(self.h, k, _dp(u), 5, 5 * nx, 1))

    def download(self, k: int) -> np.ndarray:
        ny, nx = self.shapes[k]
        out = np.zeros((ny, nx, 5))
        self._check(self.L.efvm_batch_download_state(self.h, k, _dp(out), 5, 5 * nx, 1))
        return out

    def solver_state(self, k: int) -> abi.EfvmSolverState:
        s = abi.EfvmSolverState()
        self._check(self.L.efvm_batch_get_solver_state(self.h, k, C.byref(s)))
        return s

    def run(self, t_stop, max_steps: int = 10_000_000, chunk: int = 16):
        """Advance every case to its t_stop; returns per-case results."""
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(t_stop, dtype=np.float64), (self.n,)))
        res = (abi.EfvmBatchCaseResult * self.n)()
        self._check(self.L.efvm_batch_run(self.h, _dp(t), max_steps, chunk, res))
        return list(res)

    def launch_count(self) -> int:
        v = C.c_uint64()
        self._check(self.L.efvm_batch_launch_count(self.h, C.byref(v)))
        return v.value

    def stream(self) -> int:
        p = C.c_void_p()
        self._check(self.L.efvm_batch_get_stream(self.h, C.byref(p)))
        return int(p.value or 0)

    def set_autotune(self, enable: bool) -> None:
        self._check(self.L.efvm_batch_set_autotune(self.h, int(enable)))

    def rows(self):
        r = (C.c_int32 * 4)()
        self._check(self.L.efvm_batch_get_rows(self.h, r))
        return list(r)

    def set_persistent(self, enable: bool) -> None:
        self._check(self.L.efvm_batch_set_persistent(self.h, int(enable)))

    def set_wait_limit(self, seconds: float) -> None:
        self._check(self.L.efvm_batch_set_wait_limit(self.h, float(seconds)))

    def inject_stall(self, k: int) -> None:
        self._check(self.L.efvm_batch_inject_stall(self.h, int(k)))

    def blocks_per_sm(self) -> int:
        v = C.c_int32()
        self._check(self.L.efvm_batch_get_blocks_per_sm(self.h, C.byref(v)))
        return v.value


class FluxNet:
    """The learned face-flux correction network (efvm_nn_*).  States and
    residuals are device tensors (torch, float64, [batch, 4, ny, nx])."""

    def __init__(self, out_scale: float, gamma: float = 1.4, seed: int = 0):
        self.L = load()
        self.P = self.L.efvm_nn_param_count()
        h = C.c_void_p()
        rc = self.L.efvm_nn_create(out_scale, gamma, seed, C.byref(h))
        if rc != abi.OK:
            raise EfvmError(rc, self.L.efvm_last_error(None).decode())
        self.h = h

    def _check(self, rc: int) -> None:
        if rc != abi.OK:
            raise EfvmError(rc, self.L.efvm_last_error(None).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.efvm_nn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.zeros(self.P, dtype=np.float32)
        self._check(self.L.efvm_nn_get_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.P
        self._check(self.L.efvm_nn_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))))

    def out_scale(self) -> float:
        v = C.c_float()
        self._check(self.L.efvm_nn_get_scale(self.h, C.byref(v)))
        return float(v.value)

    def forward(self, states, corr) -> None:
        b, _, ny, nx = states.shape
        self._check(self.L.efvm_nn_forward(self.h, C.c_void_p(states.data_ptr()), b, nx, ny,
                                           C.c_void_p(corr.data_ptr()), None))

    def loss_grad(self, states, resid, dx: float, dy: float, w, grad=None) -> float:
        b, _, ny, nx = states.shape
        wv = (C.c_float * 4)(*[float(x) for x in w])
        loss = C.c_double()
        gp = C.c_void_p(grad.data_ptr()) if grad is not None else None
        self._check(self.L.efvm_nn_loss_grad(self.h, C.c_void_p(states.data_ptr()), C.c_void_p(resid.data_ptr()), b,
                                             nx, ny, dx, dy, wv, gp, C.byref(loss), None))
        return loss.value

    def adam(self, lr: float) -> None:
        self._check(self.L.efvm_nn_adam(self.h, lr, None))

