"""ctypes mirror of ``include/efvm.h`` (structs and enums only, no library load).

The field order and types here must match the C header exactly; the
``tests/test_abi.py`` check compares the struct sizes with the ones the built
library reports.
"""
from __future__ import annotations

import ctypes as C

ABI_VERSION = 1

# efvm_status
OK, ERR_INVALID_ARG, ERR_CUDA, ERR_NONPHYSICAL, ERR_TIMEOUT, ERR_OOM, ERR_UNSUPPORTED = range(7)
STATUS_NAMES = {
    OK: "OK",
    ERR_INVALID_ARG: "INVALID_ARG",
    ERR_CUDA: "CUDA",
    ERR_NONPHYSICAL: "NONPHYSICAL",
    ERR_TIMEOUT: "TIMEOUT",
    ERR_OOM: "OOM",
    ERR_UNSUPPORTED: "UNSUPPORTED",
}

# boundary sides (FIELD BoundarySide order)
XLO, XHI, YLO, YHI, ZLO, ZHI = range(6)

# efvm_bc_kind (crates/cfd_boundary/src/lib.rs:172-362)
BC_SUPERSONIC_OUTFLOW = 0
BC_PERIODIC = 1
BC_SLIP_WALL = 2
BC_NO_SLIP_WALL = 3
BC_SYMMETRY = 4
BC_SUPERSONIC_INFLOW = 5
BC_SUBSONIC_INFLOW = 6
BC_PRESSURE_OUTLET = 7

FLUX_RUSANOV, FLUX_HLLC, FLUX_HLLC_TEXTBOOK = 0, 1, 2
RECON_FIRST_ORDER, RECON_MUSCL = 0, 1
LIMITER_MINMOD, LIMITER_MC = 0, 1
INTEGRATOR_RK3, INTEGRATOR_EULER = 0, 1
VISC_SUTHERLAND, VISC_CONSTANT = 0, 1
PREC_FP64, PREC_FP32_FLUX = 0, 1
# efvm_stage_form: the stage kernel's form (efvm_set_stage_tiling)
STAGE_AUTO, STAGE_STRIP, STAGE_TMA = 0, 1, 2
SEAM_REFERENCE, SEAM_TRUE_PERIODIC = 0, 1
# rows of static scratch behind efvm_cfl_dt_noalloc (EFVM_CFL_NOALLOC_MAX_ROWS)
CFL_NOALLOC_MAX_ROWS = 16384


class EfvmBC(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("reserved", C.c_int32),
        ("rho", C.c_double),
        ("u", C.c_double),
        ("v", C.c_double),
        ("w", C.c_double),
        ("p", C.c_double),
        ("t", C.c_double),
    ]


class EfvmGrid(C.Structure):
    _fields_ = [
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("nz", C.c_int32),
        ("ng", C.c_int32),
        ("lo", C.c_double * 3),
        ("hi", C.c_double * 3),
        ("bc", EfvmBC * 6),
    ]


class EfvmParams(C.Structure):
    _fields_ = [
        ("gamma", C.c_double),
        ("r_gas", C.c_double),
        ("cfl", C.c_double),
        ("fixed_dt", C.c_double),
        ("flux_scheme", C.c_int32),
        ("reconstruction", C.c_int32),
        ("limiter", C.c_int32),
        ("integrator", C.c_int32),
        ("viscous", C.c_int32),
        ("viscosity_model", C.c_int32),
        ("mu", C.c_double),
        ("precision", C.c_int32),
        ("periodic_seam", C.c_int32),
        ("parabolic_inflow", C.c_int32),
        ("reserved0", C.c_int32),
        ("inflow_u_max", C.c_double),
        ("inflow_height", C.c_double),
        ("inflow_rho", C.c_double),
        ("sponge", C.c_int32),
        ("reserved1", C.c_int32),
        ("sponge_x_start", C.c_double),
        ("sponge_x_end", C.c_double),
        ("sponge_sigma", C.c_double),
        ("sponge_u_max", C.c_double),
        ("sponge_height", C.c_double),
        ("sponge_rho", C.c_double),
        ("sponge_p", C.c_double),
        ("body_force_x", C.c_double),
    ]


class EfvmBatchCaseResult(C.Structure):
    _fields_ = [
        ("steps", C.c_int64),
        ("time", C.c_double),
        ("completion_ms", C.c_double),
        ("nonphysical", C.c_int32),
        ("finished", C.c_int32),
    ]


class EfvmSolverState(C.Structure):
    _fields_ = [
        ("dt", C.c_double),
        ("time", C.c_double),
        ("step", C.c_uint64),
        ("rk_stage", C.c_int32),
        ("completed_full_step", C.c_int32),
    ]


class EfvmCylinder(C.Structure):
    _fields_ = [("cx", C.c_double), ("cy", C.c_double), ("radius", C.c_double)]


class EfvmDisc(C.Structure):
    """A moving 2-D disc: centre, radius, velocity, spin (efvm_disc)."""
    _fields_ = [(n, C.c_double) for n in ("cx", "cy", "radius", "vx", "vy", "omega")]


class EfvmSphere(C.Structure):
    """centre, radius, translational velocity, angular velocity (efvm_sphere)."""
    _fields_ = [(n, C.c_double) for n in ("cx", "cy", "cz", "radius", "vx", "vy", "vz", "wx", "wy", "wz")]


def make_sphere(centre, radius, velocity=(0.0, 0.0, 0.0), omega=(0.0, 0.0, 0.0)) -> EfvmSphere:
    return EfvmSphere(*(float(x) for x in (*centre, radius, *velocity, *omega)))


class EfvmVortex(C.Structure):
    _fields_ = [
        ("gamma", C.c_double),
        ("beta", C.c_double),
        ("cx0", C.c_double),
        ("cy0", C.c_double),
        ("mean_u", C.c_double),
        ("mean_v", C.c_double),
        ("lo_x", C.c_double),
        ("lo_y", C.c_double),
        ("len_x", C.c_double),
        ("len_y", C.c_double),
        ("min_image", C.c_int32),
        ("reserved", C.c_int32),
    ]


class EfvmStepInfo(C.Structure):
    _fields_ = [
        ("steps_done", C.c_int64),
        ("substeps_done", C.c_int64),
        ("time", C.c_double),
        ("dt", C.c_double),
        ("stopped_at_t_stop", C.c_int32),
        ("reserved", C.c_int32),
    ]


def make_bc(kind: int = BC_SUPERSONIC_OUTFLOW, **kw) -> EfvmBC:
    b = EfvmBC()
    b.kind = kind
    for k, v in kw.items():
        setattr(b, k, float(v))
    return b


def make_grid(nx: int, ny: int, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), bcs=None, nz: int = 1, ng: int = 2) -> EfvmGrid:
    """A UniformMeshConfig plus a BoundaryRegistry (default: zero-gradient on every side)."""
    g = EfvmGrid()
    g.nx, g.ny, g.nz, g.ng = int(nx), int(ny), int(nz), int(ng)
    for a in range(3):
        g.lo[a] = float(lo[a])
        g.hi[a] = float(hi[a])
    bcs = bcs or {}
    for side in range(6):
        b = bcs.get(side, make_bc(BC_SUPERSONIC_OUTFLOW))
        g.bc[side] = b if isinstance(b, EfvmBC) else make_bc(int(b))
    return g


def make_params(**kw) -> EfvmParams:
    """Solver settings; defaults are the reference's (SolverConfig cfl=0.4, air,
    HLLC with Thornber, first order, RK3, Sutherland viscosity off)."""
    p = EfvmParams()
    p.gamma = 1.4
    p.r_gas = 287.058
    p.cfl = 0.4
    p.fixed_dt = 0.0
    p.flux_scheme = FLUX_HLLC
    p.reconstruction = RECON_FIRST_ORDER
    p.limiter = LIMITER_MINMOD
    p.integrator = INTEGRATOR_RK3
    p.viscous = 0
    p.viscosity_model = VISC_SUTHERLAND
    p.mu = 0.0
    p.precision = PREC_FP64
    p.periodic_seam = SEAM_REFERENCE
    for k, v in kw.items():
        cur = getattr(p, k)
        setattr(p, k, type(cur)(v))
    return p


def make_vortex(gamma=1.4, beta=5.0, cx0=5.0, cy0=5.0, mean_u=0.5, mean_v=0.5, lo=(0.0, 0.0), length=(10.0, 10.0),
                min_image=False) -> EfvmVortex:
    v = EfvmVortex()
    v.gamma, v.beta, v.cx0, v.cy0, v.mean_u, v.mean_v = gamma, beta, cx0, cy0, mean_u, mean_v
    v.lo_x, v.lo_y = lo
    v.len_x, v.len_y = length
    v.min_image = 1 if min_image else 0
    return v
