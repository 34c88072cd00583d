/*
 * efvm.h — C-ABI of the B200 explicit finite-volume step (MUSCL/HLLC fluxes,
 * viscous terms, SSP-RK3 stage update, CFL dt reduction, ghost-cell IBM fill and
 * marker-load sum) of dev_field_efvm.
 *
 * Every entry point is a plain `extern "C"` function over plain pointers and
 * sizes.  Every call returns an `int` status (efvm_status); `efvm_last_error`
 * gives the message of the last failure on a context.  No C++ exception and no
 * device trap crosses this boundary.
 *
 * Ownership: a context owns all of its device memory and one CUDA stream on the
 * device that was current when it was created.  Host pointers are borrowed only
 * for the duration of a call.  A context is not thread-safe (use one per
 * thread); distinct contexts are independent.
 *
 * The reference interfaces each entry point replaces are cited as
 * `path:line` inside the dev_field_efvm source tree (the Rust crates under
 * `crates/` and the case drivers under `examples/`).
 */
#ifndef EFVM_H
#define EFVM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define EFVM_ABI_VERSION 1

/* Status codes.  The reference panics or returns Option; the C-ABI returns a
 * code instead (crates/cfd_boundary/src/lib.rs:516-518 panics on a half-periodic
 * axis -> EFVM_ERR_INVALID_ARG here). */
typedef enum {
    EFVM_OK = 0,
    EFVM_ERR_INVALID_ARG = 1,
    EFVM_ERR_CUDA = 2,
    EFVM_ERR_NONPHYSICAL = 3, /* rho<=0, p<=0 or a NaN appeared in the state */
    EFVM_ERR_TIMEOUT = 4,     /* a bounded device-side wait ran out */
    EFVM_ERR_OOM = 5,
    EFVM_ERR_UNSUPPORTED = 6
} efvm_status;

/* Boundary sides in FIELD's BoundarySide / PatchId order (XLo..ZHi = 0..5). */
enum { EFVM_XLO = 0, EFVM_XHI = 1, EFVM_YLO = 2, EFVM_YHI = 3, EFVM_ZLO = 4, EFVM_ZHI = 5 };

/* Stock boundary conditions, crates/cfd_boundary/src/lib.rs:172-362. */
typedef enum {
    EFVM_BC_SUPERSONIC_OUTFLOW = 0, /* zero-gradient copy (:173-189), registry default (:375-381) */
    EFVM_BC_PERIODIC = 1,           /* halo wrap from the opposite slab (:197-216) */
    EFVM_BC_SLIP_WALL = 2,          /* flip wall-normal momentum (:246-272) */
    EFVM_BC_NO_SLIP_WALL = 3,       /* flip all momentum (:276-296) */
    EFVM_BC_SYMMETRY = 4,           /* == slip wall (:299-310) */
    EFVM_BC_SUPERSONIC_INFLOW = 5,  /* prescribed rho,u,v,w,p; T = p/(rho*287.058) (:220-243) */
    EFVM_BC_SUBSONIC_INFLOW = 6,    /* prescribed rho,u,v,w,t; p from the interior (:314-337) */
    EFVM_BC_PRESSURE_OUTLET = 7     /* prescribed p; rho,u from the interior (:341-362) */
} efvm_bc_kind;

typedef struct {
    int32_t kind; /* efvm_bc_kind */
    int32_t reserved;
    double rho, u, v, w, p, t; /* parameters of the inflow/outlet kinds */
} efvm_bc;

/* A uniform mesh (FIELD UniformMeshConfig{nx,ny,nz,ng,bounds_lo,bounds_hi}
 * with ng == 2) plus one boundary condition per side (BoundaryRegistry,
 * crates/cfd_boundary/src/lib.rs:370-449).  nz == 1 is the 2-D form of the
 * benchmark cases: the z extent enters the CFL (crates/cfd_solver/src/lib.rs:
 * 659-661) and the marker area.  nz > 1 is a 3-D mesh with z faces (FP64; no
 * IBM, slabs, batches, flux correction or output fields; state through
 * efvm_upload_state_3d / efvm_download_state_3d). */
typedef struct {
    int32_t nx, ny, nz, ng;
    double lo[3], hi[3];
    efvm_bc bc[6];
} efvm_grid;

typedef enum { EFVM_FLUX_RUSANOV = 0, EFVM_FLUX_HLLC = 1, EFVM_FLUX_HLLC_TEXTBOOK = 2 } efvm_flux_scheme;
typedef enum { EFVM_RECON_FIRST_ORDER = 0, EFVM_RECON_MUSCL = 1 } efvm_reconstruction;
typedef enum { EFVM_LIMITER_MINMOD = 0, EFVM_LIMITER_MC = 1 } efvm_limiter;
typedef enum { EFVM_INTEGRATOR_RK3 = 0, EFVM_INTEGRATOR_EULER = 1 } efvm_integrator;
typedef enum { EFVM_VISC_SUTHERLAND = 0, EFVM_VISC_CONSTANT = 1 } efvm_viscosity;
/* FP64: everything in double.  FP32_FLUX: reconstruction and face fluxes in
 * float, stage accumulation, RK combination and marker integral in double. */
typedef enum { EFVM_PREC_FP64 = 0, EFVM_PREC_FP32_FLUX = 1 } efvm_precision;
/* How MUSCL treats the periodic seam.  REFERENCE: the halo-ghost side of a seam
 * face is not reconstructed and has zero slope (crates/cfd_solver/src/lib.rs:
 * 250-253,323-331), so each side computes its own seam flux.  TRUE_PERIODIC:
 * the wrapped ghost is reconstructed like an interior cell (conservative). */
typedef enum { EFVM_SEAM_REFERENCE = 0, EFVM_SEAM_TRUE_PERIODIC = 1 } efvm_seam;

/* Solver, gas, transport and case-system settings.  Mirrors SolverConfig
 * (crates/cfd_solver/src/lib.rs:39-58), IdealGas (crates/cfd_eos/src/lib.rs:
 * 27-41), Viscosity (:99-117), the flux/limiter plugins (crates/cfd_solver/src/
 * lib.rs:764-842), IntegratorPlugin (:877-902) and the case-local systems of the
 * cylinder and channel drivers. */
typedef struct {
    double gamma, r_gas;
    double cfl;
    double fixed_dt; /* > 0 overrides the CFL dt (SolverConfig.fixed_dt) */
    int32_t flux_scheme;    /* efvm_flux_scheme */
    int32_t reconstruction; /* efvm_reconstruction */
    int32_t limiter;        /* efvm_limiter */
    int32_t integrator;     /* efvm_integrator */
    int32_t viscous;        /* SolverConfig.viscous */
    int32_t viscosity_model;/* efvm_viscosity */
    double mu;              /* Viscosity::Constant(mu) */
    int32_t precision;      /* efvm_precision */
    int32_t periodic_seam;  /* efvm_seam */
    /* parabolic velocity inlet overriding the x-lo ghosts,
     * examples/cylinder_drag_validation/main.rs:151-177 */
    int32_t parabolic_inflow;
    int32_t reserved0;
    double inflow_u_max, inflow_height, inflow_rho;
    /* downstream sponge after each completed step, main.rs:186-229: toward the
     * parabolic profile of height sponge_height on a 2-D mesh; toward the uniform
     * freestream (sponge_rho, sponge_u_max, 0, 0, sponge_p) on a 3-D mesh, the
     * sphere case's sponge (examples/sphere_drag_validation/main.rs:119-160) */
    int32_t sponge;
    int32_t reserved1;
    double sponge_x_start, sponge_x_end, sponge_sigma;
    double sponge_u_max, sponge_height, sponge_rho, sponge_p;
    /* uniform streamwise body force added in PostFlux,
     * crates/cfd_solver/tests/poiseuille_channel_validation.rs:100-118 */
    double body_force_x;
} efvm_params;

/* SolverState{dt,time,step,rk_stage} (crates/cfd_solver/src/lib.rs:61-73) and
 * StepBoundary.completed_full_step (:607-621).  rk_stage: 0,1,2 = First..Third. */
typedef struct {
    double dt;
    double time;
    uint64_t step;
    int32_t rk_stage;
    int32_t completed_full_step;
} efvm_solver_state;

/* A z-aligned analytic cylinder, crates/cfd_ibm/src/lib.rs:61-87. */
typedef struct {
    double cx, cy, radius;
} efvm_cylinder;

/* A moving disc (the 2-D rigid body of examples/dkt_sedimentation/main.rs:66-103):
 * a z-aligned cylinder with translational velocity (vx, vy) and spin omega about
 * z; the wall moves at (vx - omega ry, vy + omega rx). */
typedef struct {
    double cx, cy, radius;
    double vx, vy, omega;
} efvm_disc;

/* A rigid sphere with its kinematic state (SphereBody, crates/cfd_ibm/src/
 * sphere.rs:26-72): centre, radius, translational velocity (vx, vy, vz) and
 * angular velocity (wx, wy, wz); the wall moves at v + w x (p - centre). */
typedef struct {
    double cx, cy, cz, radius;
    double vx, vy, vz;
    double wx, wy, wz;
} efvm_sphere;

/* The Shu isentropic vortex used as exact solution (crates/cfd_solver/tests/
 * isentropic_vortex_muscl_convergence.rs:48-64): centre (cx0,cy0) at t=0,
 * translated by (mean_u,mean_v).  min_image != 0 measures the displacement
 * with the minimum image on a periodic box of size (len_x,len_y) from lo. */
typedef struct {
    double gamma, beta;
    double cx0, cy0, mean_u, mean_v;
    double lo_x, lo_y, len_x, len_y;
    int32_t min_image;
    int32_t reserved;
} efvm_vortex;

/* Counters of one efvm_step call. */
typedef struct {
    int64_t steps_done;
    int64_t substeps_done;
    double time;
    double dt;
    int32_t stopped_at_t_stop;
    int32_t reserved;
} efvm_step_info;

typedef struct efvm_ctx efvm_ctx;

/* ---- lifecycle ---------------------------------------------------------- */

/* Replaces App::new + FieldDefaultPlugins + CfdStatePlugin + IdealGasPlugin/
 * GasPlugin + BoundaryPlugin/StructuredBoundaryPlugin + FluxPlugin/MusclPlugin
 * + IntegratorPlugin + SolverPlugin + app.prepare()
 * (crates/cfd_solver/src/lib.rs:691-940, crates/cfd_boundary/src/lib.rs:
 * 457-533).  Validates the configuration (half-periodic axes, ng != 2 and, on
 * 3-D meshes, the 2-D-only options are rejected) and allocates the device state.  The state must then be
 * uploaded (the reference's init_state_system, crates/cfd_solver/src/lib.rs:
 * 681-686, is a host closure). */
int efvm_create(const efvm_grid* grid, const efvm_params* params, efvm_ctx** out);
int efvm_destroy(efvm_ctx* ctx);
/* Message of the last failed call on ctx (never NULL). */
const char* efvm_last_error(const efvm_ctx* ctx);
int efvm_abi_version(void);

/* ---- state -------------------------------------------------------------- */

/* Copy the interior conserved state in (CfdState.u, crates/cfd_state/src/
 * lib.rs:180-195).  Element (i,j) component v (0..4 = rho, rho_u, rho_v, rho_w,
 * rho_e) is read at base[i*stride_i + j*stride_j + v*stride_var], i < nx,
 * j < ny (strides in doubles).  rho_w is ignored (2-D).  The ghost bands are
 * filled from the interior before the next substage, as the Halo/Boundary
 * phases do.  Marks the CFL dt as stale. */
int efvm_upload_state(efvm_ctx* ctx, const double* base, int64_t stride_i, int64_t stride_j,
                      int64_t stride_var);
/* The inverse of efvm_upload_state; writes rho_w = 0. */
int efvm_download_state(efvm_ctx* ctx, double* base, int64_t stride_i, int64_t stride_j,
                        int64_t stride_var);
/* The state of a 3-D context (nz > 1), as CfdState.u over all layers: element
 * (i,j,k) component v (0..4 = rho, rho_u, rho_v, rho_w, rho_e) at
 * base[i*stride_i + j*stride_j + k*stride_k + v*stride_var].  On a 2-D context
 * they act as efvm_upload_state / efvm_download_state (stride_k unused).  The
 * 2-D calls above refuse a 3-D context. */
int efvm_upload_state_3d(efvm_ctx* ctx, const double* base, int64_t stride_i, int64_t stride_j, int64_t stride_k,
                         int64_t stride_var);
int efvm_download_state_3d(efvm_ctx* ctx, double* base, int64_t stride_i, int64_t stride_j, int64_t stride_k,
                           int64_t stride_var);

int efvm_get_solver_state(efvm_ctx* ctx, efvm_solver_state* out);
/* Restores dt/time/step/rk_stage (checkpoint resume, crates/cfd_solver/src/
 * lib.rs:895-897). */
int efvm_set_solver_state(efvm_ctx* ctx, const efvm_solver_state* in);

/* ---- stepping ----------------------------------------------------------- */

/* Exactly one app.run(): one RK substage through every phase the reference
 * runs (Setup: CFL on the first stage + IBM geometry; Halo; Boundary; PreFlux:
 * IBM mirror; Flux: inviscid + viscous; PostFlux; Update; PostUpdate: sponge;
 * Output: marker and wall forces).  crates/cfd_solver/src/lib.rs:607-677. */
int efvm_substep(efvm_ctx* ctx);

/* Run up to n_steps whole RK3 steps from a step boundary on the device,
 * stopping at the first step boundary where time >= t_stop when stop_at_t is
 * non-zero (the case drivers' `loop { if t >= T break; 3x app.run() }`,
 * crates/cfd_solver/tests/isentropic_vortex_muscl_convergence.rs:109-117).
 * When force_history is not NULL it receives the MarkerForce after every
 * substage (6 doubles each: pressure xyz, viscous xyz), capacity
 * 3*n_steps*6 doubles, as examples/cylinder_drag_validation/main.rs:334-340
 * reads it.  Returns EFVM_ERR_NONPHYSICAL if the state went non-physical.
 * With stop_at_t == 0, force_history == NULL and info == NULL the call only
 * enqueues the work on the context's stream and returns without waiting; a
 * non-physical state is then reported by the next synchronising call
 * (efvm_get_solver_state, efvm_step with info, a download). */
int efvm_step(efvm_ctx* ctx, int64_t n_steps, int32_t stop_at_t, double t_stop,
              double* force_history, efvm_step_info* info);

/* CFL dt of the current state without stepping (cfl_system,
 * crates/cfd_solver/src/lib.rs:626-677). */
int efvm_cfl(efvm_ctx* ctx, double* dt_out);

/* ---- immersed boundary -------------------------------------------------- */

/* CylinderIbmPlugin::with_cylinders + GhostCellIbmPlugin
 * (crates/cfd_ibm/src/lib.rs:621-680).  freestream = ConsVar (5 doubles) that
 * seeds the cells that flip solid/fluid. */
int efvm_set_cylinders(efvm_ctx* ctx, const efvm_cylinder* cylinders, int32_t n,
                       const double freestream[5]);
/* The moving-disc geometry of examples/dkt_sedimentation/main.rs:143-287 with
 * GhostCellIbmPlugin on a 2-D context: the cylinder mask, ghosts and markers
 * (n_theta per disc) with each disc's wall velocity in the ghost mirror and the
 * marker traction.  An FSI driver calls it between steps with the new centres
 * and velocities; efvm_body_loads then gives each disc's load and torque.
 * efvm_set_cylinders is the same with bodies at rest and 64 markers. */
int efvm_set_discs(efvm_ctx* ctx, const efvm_disc* discs, int32_t n, int32_t n_theta, const double freestream[5]);
/* SphereIbmPlugin::new(..).with_markers(n_markers) + GhostCellIbmPlugin
 * (crates/cfd_ibm/src/sphere.rs:77-292) on a 3-D context: the solid mask
 * (cell centres inside any sphere, flipped cells seeded as with cylinders), the
 * ghost list (solid cells with a fluid face neighbour, image point mirrored
 * across the nearest sphere, wall velocity of that body at the ghost's wall
 * footprint) and max(n_markers, 12) Fibonacci markers per sphere of area
 * 4 pi R^2 / n.  A moving body: call again between steps with the new centres
 * and velocities; the lists are rebuilt before the next substep, as the
 * reference's Setup systems do every substep.  Marker and staircase wall forces
 * are then read with efvm_marker_force / efvm_wall_force. */
int efvm_set_spheres(efvm_ctx* ctx, const efvm_sphere* spheres, int32_t n, int32_t n_markers,
                     const double freestream[5]);
/* MarkerForce{pressure,viscous} of the last Output phase
 * (crates/cfd_ibm/src/lib.rs:442-480,601-615).  On a 2-D mesh, efvm_step
 * computes the forces of a step's last substage in the next step's first
 * launch; this call (and every call that replaces the state or the bodies, or
 * steps with a history or a stop time) first runs them if they are still
 * pending, so it always returns the last substage's forces. */
int efvm_marker_force(efvm_ctx* ctx, double out[6]);
/* WallForce{pressure,viscous}, the staircase estimate (crates/cfd_ibm/src/
 * lib.rs:309-395); pending forces are run first, as for efvm_marker_force. */
int efvm_wall_force(efvm_ctx* ctx, double out[6]);
/* ---- output -------------------------------------------------------------- */
/* The fields write_vtk_to writes (crates/cfd_output/src/lib.rs:36-125) for the
 * current state, computed on the device: 7 planes of nx*ny doubles, x fastest:
 * density, pressure, temperature, velocity u, v, w (= 0), Mach.  With async != 0
 * the copy into host_out (pinned memory for a truly asynchronous copy) is only
 * enqueued on the context's stream, so a solver can keep stepping; wait with
 * efvm_synchronize before reading host_out. */
int efvm_output_fields(efvm_ctx* ctx, double* host_out, int32_t async);
/* Wait for everything enqueued on the context's stream. */
int efvm_synchronize(efvm_ctx* ctx);
/* write_vtk (crates/cfd_output/src/lib.rs:110-125): the current state as a VTK
 * legacy ASCII RECTILINEAR_GRID file (nz = 1 cell layer), same fields, order and
 * number format as the reference writer. */
int efvm_write_vtk(efvm_ctx* ctx, const char* path);

/* compute_marker_loadings_per_body (crates/cfd_ibm/src/lib.rs:509-562) on the
 * current state: for each of the first n_bodies cylinders, out[9 b ..] =
 * pressure force[3], viscous force[3] and the torque[3] about its centre (the
 * centre taken at the z of its markers), from its own 64 markers. */
int efvm_body_loads(efvm_ctx* ctx, int32_t n_bodies, double* out);
/* Number of solid cells and of IBM ghost cells (IbmGhostCells.cells.len()). */
int efvm_ibm_counts(efvm_ctx* ctx, int64_t* n_solid, int64_t* n_ghost);
/* The interior SolidMask (crates/cfd_state/src/lib.rs:202-206) as nx*ny bytes,
 * x fastest (1 = solid). */
int efvm_get_solid_mask(efvm_ctx* ctx, uint8_t* out);

/* ---- diagnostics -------------------------------------------------------- */

/* Volume-weighted L1 and the max-norm of (rho - rho_exact) over the interior at
 * the context's current time (crates/cfd_solver/tests/
 * isentropic_vortex_muscl_convergence.rs:119-138). */
int efvm_density_error(efvm_ctx* ctx, const efvm_vortex* exact, double out[2]);
/* Fill the interior with the vortex at t=0 on the device (synthetic inputs). */
int efvm_init_vortex(efvm_ctx* ctx, const efvm_vortex* v);
/* Sum of rho*volume over the interior (total mass). */
int efvm_total_mass(efvm_ctx* ctx, double* out);

/* The CUDA stream the context launches on (a cudaStream_t), so a caller can
 * time it with its own events. */
int efvm_get_stream(efvm_ctx* ctx, void** stream);
/* Number of kernels this context has launched since creation. */
int efvm_launch_count(efvm_ctx* ctx, uint64_t* out);

/* Run n_steps whole steps with individually launched kernels and CUDA events
 * around each kernel class on the context's stream; out_ms[0..3] receives the
 * summed device time of the stage kernels, the IBM mirror/force kernels, the
 * per-step set-up kernel, and the whole steps.  Instrumentation for the bench
 * (the reference has no timers). */
int efvm_profile_steps(efvm_ctx* ctx, int64_t n_steps, double out_ms[4]);

/* ---- stage-kernel form and tiling ------------------------------------------ */

/* The stage kernel of a 2-D context comes in two forms with the same
 * arithmetic.  EFVM_STAGE_STRIP: each warp marches a strip of 31 columns and
 * reads its rows, halo cells and U^n through L1/L2.  EFVM_STAGE_TMA: a block's
 * four warps march the same rows of four adjacent strips, fed by TMA
 * (cp.async.bulk.tensor) into a shared-memory ring of rows one iteration ahead
 * of their use; it runs for cases without viscous terms, immersed bodies, a
 * body force, an outlet sponge or a flux correction, and the other cases run
 * the strip form whatever is set.
 * EFVM_STAGE_AUTO is the built-in choice: the TMA-fed form wherever the case
 * allows it (the faster of the two at 4096^2 in both precisions), else the
 * strip form.  Both give the reference's results
 * (the forms, and the strip form's builds for different block counts, differ
 * from each other by a few ulps at most; a form gives the same bits for any
 * rows per warp). */
typedef enum { EFVM_STAGE_AUTO = 0, EFVM_STAGE_STRIP = 1, EFVM_STAGE_TMA = 2 } efvm_stage_form;
/* Select the form, the rows each warp marches and the strip form's resident
 * blocks per SM (0 = built-in choice for each; the FP64 inviscid strip form is
 * built for 6 and 7 blocks, every other form for one count; a count the
 * selected form is not built for returns EFVM_ERR_INVALID_ARG).  The reference
 * runs its systems on the CPU and has no counterpart; this replaces no call.
 * EFVM_ERR_UNSUPPORTED for EFVM_STAGE_TMA on a 3-D context. */
int efvm_set_stage_tiling(efvm_ctx* ctx, int32_t form, int32_t rows_per_warp, int32_t blocks_per_sm);
/* The form the context's next stage runs, its rows per warp and blocks per SM. */
int efvm_get_stage_tiling(efvm_ctx* ctx, int32_t* form, int32_t* rows_per_warp, int32_t* blocks_per_sm);
/* Time n_steps whole steps (default 3) of every candidate tiling on the live
 * state -- each form the case allows (the strip form at each block count it is
 * built for), with 4, 8, 16 and 32 rows per warp and with the rows that put the
 * whole grid in one wave of resident blocks -- and
 * keep the fastest.  The state, the clock and the force outputs are restored
 * after every candidate, so tuning changes no result; the call holds a
 * temporary device copy of the state (4 planes) while it runs.  2-D RK3 contexts at a
 * step boundary without slabs or a flux correction; *best_ms_per_step (may be
 * NULL) receives the winner's device time per step.  No counterpart in the
 * reference. */
int efvm_autotune_stage(efvm_ctx* ctx, int32_t n_steps, double* best_ms_per_step);
/* Limit of one wait of the TMA-fed stage kernel for a row of its ring (default
 * 4 s, far above any real wait).  A wait that runs out ends the stage's march
 * in that block and the next status read returns EFVM_ERR_TIMEOUT; the GPU and
 * other contexts stay usable.  No counterpart in the reference. */
int efvm_set_stage_wait_limit(efvm_ctx* ctx, double seconds);
/* Failure injection for tests: enable != 0 makes the first block of the
 * TMA-fed stage stop refilling its ring after the first rows, so its waits run
 * out (EFVM_ERR_TIMEOUT).  The state is then meaningless.  No counterpart in
 * the reference. */
int efvm_inject_stage_stall(efvm_ctx* ctx, int32_t enable);

/* ---- slabs of one grid on several GPUs ------------------------------------ */

/* A grid split into row slabs runs one context per slab (one process per GPU).
 * field_core decomposes a mesh over MPI ranks and fills rank-edge ghosts with
 * halo_exchange_forward_all, and the solver min-reduces dt over ranks
 * (all_reduce_min_f64); a slab does the same with two calls per neighbour per
 * RK stage and one reduction per step, which the caller carries over its own
 * transport (NCCL, or copies between contexts on one GPU):
 *
 *   efvm_prepare(ctx);  max-reduce *slot over slabs;
 *   for s in 0..2 { efvm_halo_pack(ctx, YLO/YHI, send); exchange with the two
 *                   neighbours; efvm_halo_unpack(ctx, YLO/YHI, recv);
 *                   efvm_substep(ctx); }
 *   (efvm_prepare does work only after an upload or a solver-state change)
 *
 * Faces between slabs are interior faces, so results do not depend on the
 * split (field_core leaves the halo side of a rank edge unreconstructed under
 * MUSCL, crates/cfd_solver/src/lib.rs:323-331; here only the global periodic
 * seam keeps the efvm_seam rule).  IBM cylinders and efvm_step are not
 * supported on slabs (EFVM_ERR_UNSUPPORTED). */

/* A context for global rows [row0, row0 + rows) of `grid` (rows >= 2).  Cell
 * coordinates, spacing and boundary conditions are the global grid's; a y side
 * that faces another slab, or the periodic wrap of a periodic y axis, takes its
 * two ghost rows from efvm_halo_unpack.  Upload/download cover the slab's rows. */
int efvm_create_slab(const efvm_grid* grid, const efvm_params* params, int32_t row0, int32_t rows,
                     efvm_ctx** out);
/* Run now what the next substep would run first: the stand-alone CFL pass after
 * an upload (into the wave speed slot when one is enabled), pending cylinder
 * geometry, and the boundary-ghost fill of non-HALO sides. */
int efvm_prepare(efvm_ctx* ctx);
/* Copy the two interior rows next to y side `side` (EFVM_YLO: rows 0,1;
 * EFVM_YHI: rows ny-2, ny-1) of the next substep's input into dev_buf, a device
 * buffer of 8*nx doubles laid out [variable rho, rho_u, rho_v, rho_e][row, in
 * increasing j][i].  Asynchronous on the context's stream. */
int efvm_halo_pack(efvm_ctx* ctx, int32_t side, double* dev_buf);
/* Write such a buffer, packed by the neighbour on that side, into the two ghost
 * rows of side `side` (EFVM_YLO: rows -2,-1; EFVM_YHI: rows ny, ny+1) of the next
 * substep's input.  The side must take its ghosts from a neighbour.  Asynchronous. */
int efvm_halo_unpack(efvm_ctx* ctx, int32_t side, const double* dev_buf);
/* Switch the context to an external wave-speed slot and return its device
 * address: an unsigned 64-bit word holding the bits of the largest wave speed
 * (a non-negative double, so its bits order like the value).  The last stage of
 * each step (and the CFL pass after an upload) max-accumulates into it; the
 * next step's set-up reads it, takes dt = cfl / slot, and clears it.  Between
 * the two the caller max-reduces the word across slabs (an integer max). */
int efvm_wave_speed_slot(efvm_ctx* ctx, uint64_t** dev_slot);

/* Halo peers: the exchange fused into the stage kernel.  Instead of
 * efvm_halo_pack -> transport -> efvm_halo_unpack between stages (the
 * reference's halo_exchange_forward_all, crates/cfd_solver/src/lib.rs:79-81),
 * a slab's stage kernel can store its two rows next to a y side straight into
 * the ghost rows of the neighbouring slab's output buffer of the same stage:
 * another slab's buffer on the same GPU, or a peer GPU's buffer mapped into
 * this process (peer access or CUDA IPC).  All slabs must share nx and run the
 * same integrator in lockstep; the caller orders stage t of a slab after stage
 * t - 1 of both neighbours (stream events on one GPU) and still max-reduces the
 * wave-speed slot once per step.  Ghost rows of a freshly uploaded state come
 * from one pack / unpack exchange before the first substep.
 *
 * efvm_get_state_buffers: the context's three state buffers (U^n and the two
 * stage buffers, each 4 planes of `plane` doubles) and its rows. */
int efvm_get_state_buffers(efvm_ctx* ctx, double* bufs[3], int64_t* plane, int32_t* rows);
/* Write side `side`'s edge rows into the neighbour's buffers peer_bufs[0..2]
 * (as that neighbour's efvm_get_state_buffers returns them, in its order) of
 * peer_plane doubles per plane and peer_rows rows; NULL peer_bufs returns the
 * side to the pack / unpack exchange.  The side must face another slab. */
int efvm_set_halo_peer(efvm_ctx* ctx, int32_t side, double* const peer_bufs[3], int64_t peer_plane,
                       int32_t peer_rows);
/* The same across processes (one process per GPU): efvm_get_state_ipc writes
 * the CUDA IPC handles of the three state buffers (3 x 64 bytes) for the
 * neighbours to map; efvm_set_halo_peer_ipc maps a neighbour's handles into
 * this process (with peer access) and sets them as the side's peer.  The
 * mapping is released when the side is reset or the context is destroyed.
 * A process cannot map its own handles: slabs in one process use
 * efvm_get_state_buffers. */
#define EFVM_IPC_HANDLE_BYTES 64
int efvm_get_state_ipc(efvm_ctx* ctx, void* handles);
int efvm_set_halo_peer_ipc(efvm_ctx* ctx, int32_t side, const void* handles, int64_t peer_plane,
                           int32_t peer_rows);

/* ---- batches of independent cases ---------------------------------------- */

/* A batch advances many independent cases (an ensemble or a parameter sweep;
 * the reference runs one App per case) together, each case with its own grid,
 * boundary conditions, CFL dt, clock and stop time.  By default one persistent
 * kernel launch runs a whole chunk of RK3 steps of every running case: its
 * warps take the tiles of all cases from one packed queue, a tile waits only
 * for its own case's previous stage, and the last tile of a case's step runs
 * that case's next set-up, so small cases run ahead of large ones.  The waits
 * are bounded (efvm_batch_set_wait_limit); a wait that runs out ends the run
 * with EFVM_ERR_TIMEOUT.  The other form (efvm_batch_set_persistent(b, 0))
 * launches one set-up per step and one kernel per stage over the table.  Each
 * chunk is a captured CUDA graph.  All cases share one efvm_params (RK3 only);
 * IBM cylinders are not supported in a batch. */
typedef struct efvm_batch efvm_batch;

typedef struct {
    int64_t steps;         /* whole steps this run took */
    double time;           /* the case's clock at the end */
    double completion_ms;  /* device time from the start of the run to the set-up that stopped the case;
                              -1 if it did not stop */
    int32_t nonphysical;   /* non-physical state flags (as efvm_get_solver_state reports) */
    int32_t finished;      /* 1 if the case reached its stop time */
} efvm_batch_case_result;

/* n_cases grids (each as for efvm_create) sharing `params`. */
int efvm_batch_create(const efvm_grid* grids, int32_t n_cases, const efvm_params* params, efvm_batch** out);
int efvm_batch_destroy(efvm_batch* batch);
/* Message of the last failed batch call (batch may be NULL). */
const char* efvm_batch_last_error(const efvm_batch* batch);
/* State of case `k`, strided as for efvm_upload_state / efvm_download_state. */
int efvm_batch_upload_state(efvm_batch* batch, int32_t k, const double* base, int64_t stride_i, int64_t stride_j,
                            int64_t stride_var);
int efvm_batch_download_state(efvm_batch* batch, int32_t k, double* base, int64_t stride_i, int64_t stride_j,
                              int64_t stride_var);
int efvm_batch_get_solver_state(efvm_batch* batch, int32_t k, efvm_solver_state* out);
/* Advance every case by whole RK3 steps until its clock reaches t_stop[k] (the
 * time loop of the example drivers: while t < t_final, three app.run() per step) or
 * max_steps steps have run.  Finished cases leave the launch table every
 * `chunk` steps (<= 0: 16).  results (may be NULL) receives one entry per case.
 * Returns EFVM_ERR_NONPHYSICAL if any case went non-physical. */
int efvm_batch_run(efvm_batch* batch, const double* t_stop, int64_t max_steps, int64_t chunk,
                   efvm_batch_case_result* results);
int efvm_batch_launch_count(efvm_batch* batch, uint64_t* out);
/* The CUDA stream the batch launches on (a cudaStream_t). */
int efvm_batch_get_stream(efvm_batch* batch, void** stream);
/* Autotuning (on by default): on the first efvm_batch_run the batch times one
 * step with tiles of 2, 4, 8 and 16 rows per warp for each case-size bucket
 * present (cells < 64^2, < 128^2, < 256^2, larger) and then, for the persistent
 * kernel, its grid at the form's maximum resident blocks per SM and up to three
 * fewer, on a copy of the states; it keeps the fastest and caches the choice per
 * process for the device, the method, the kernel and the buckets.  Tuning
 * changes no result.  enable = 0 returns to the built-in heuristic. */
int efvm_batch_set_autotune(efvm_batch* batch, int32_t enable);
/* Rows per warp chosen for the four buckets (0 = heuristic / not tuned yet). */
int efvm_batch_get_rows(efvm_batch* batch, int32_t rows[4]);
/* Resident blocks per SM of the persistent kernel's grid (tuned or default). */
int efvm_batch_get_blocks_per_sm(efvm_batch* batch, int32_t* out);
/* enable != 0: one persistent launch per chunk of steps (the default); 0: one
 * launch per stage.  Both give the same results bit for bit. */
int efvm_batch_set_persistent(efvm_batch* batch, int32_t enable);
/* Limit of one wait of the persistent kernel for a case's previous stage, in
 * seconds (default 2, at most 60). */
int efvm_batch_set_wait_limit(efvm_batch* batch, double seconds);
/* Fault injection for the bounded waits (host side, no device fault): the next
 * efvm_batch_run counts one tile more for case k than its table holds, so that
 * case's first stage never completes, its next stage's waits run out and the
 * run returns EFVM_ERR_TIMEOUT with the states partly advanced.  No counterpart
 * in the reference. */
int efvm_batch_inject_stall(efvm_batch* batch, int32_t k);

/* ---- learned flux correction: BF16 tensor-core kernels -------------------- */

/* D[m x n] = A[m x k] * B[n x k]^T with BF16 A and B (device pointers, row-major,
 * k contiguous) and FP32 D, on the tensor cores (tcgen05, FP32 accumulation in
 * tensor memory): the GEMM tile the correction network is built from, exposed
 * so that it can be checked against a CPU product.  m a multiple of 128; n and
 * k multiples of 16 in [16, 256].  Synchronous.  No counterpart in the
 * reference (the learned correction is this library's addition). */
int efvm_nn_gemm_bf16(const uint16_t* a, const uint16_t* b, float* d, int32_t m, int32_t n, int32_t k, void* stream);

/* The correction network (no counterpart in the reference).  Per face, the
 * 5 x 5 stencil of primitive variables (rho - 1, normal and tangential
 * velocity, p - 1) in the face's frame feeds three layers (100 -> 32 -> 32 -> 4,
 * relu) whose output times out_scale is added to that face's flux, so the
 * correction is conservative.  BF16 weights on the tensor cores, FP32 biases
 * and accumulation.  Parameters are FP32, flat:
 * W1[32][112] (columns >= 100 unused), W2[32][32], W3[4][32], b1[32], b2[32], b3[4]. */
typedef struct efvm_nn efvm_nn;

int efvm_nn_param_count(void);
/* Seeded initial weights (He normal, a near-zero output layer, zero biases). */
int efvm_nn_create(float out_scale, float gamma, uint64_t seed, efvm_nn** out);
int efvm_nn_destroy(efvm_nn* nn);
int efvm_nn_get_params(efvm_nn* nn, float* host_params);
int efvm_nn_set_params(efvm_nn* nn, const float* host_params);
int efvm_nn_get_scale(efvm_nn* nn, float* out_scale);
/* Corrections of every face of `batch` periodic states (device, conserved FP64,
 * [batch][4][ny][nx], rho, rho_u, rho_v, rho_e) into corr (device FP32,
 * [batch][2][4][ny][nx]: x face on the left of a cell, then y face below it;
 * grid-frame components).  nx*ny a multiple of 64.  Synchronous. */
int efvm_nn_forward(efvm_nn* nn, const double* states, int32_t batch, int32_t nx, int32_t ny, float* corr,
                    void* stream);
/* Loss and gradient on a batch: per cell e = resid + div(corr), the loss is
 * sum_v w[v] * mean(e_v^2), and resid (device FP64, [batch][4][ny][nx]) is the
 * coarse-step residual (target - plain step) / dt.  The gradient (P floats)
 * goes to grad_out (device, may be NULL) and to the network's own buffer for
 * efvm_nn_adam; the loss to *loss (host, may be NULL).  Synchronous. */
int efvm_nn_loss_grad(efvm_nn* nn, const double* states, const double* resid, int32_t batch, int32_t nx, int32_t ny,
                      double dx, double dy, const float w[4], float* grad_out, double* loss, void* stream);
/* One Adam step (beta 0.9 / 0.999) with the gradient of the last efvm_nn_loss_grad. */
int efvm_nn_adam(efvm_nn* nn, float lr, void* stream);
/* Attach a network to a context (periodic in x and y, MUSCL + HLLC, no IBM,
 * nx*ny a multiple of 64): every stage then adds its corrections to the face
 * fluxes.  A face keeps the plain flux where the sensor fires: the pressures of
 * its two cells differ by more than sensor * min(p), or rho or p is not
 * positive.  NULL detaches.  The network must outlive its use. */
int efvm_set_flux_correction(efvm_ctx* ctx, efvm_nn* nn, float sensor);
/* Faces evaluated and faces that fell back to the plain flux since attach. */
int efvm_correction_stats(efvm_ctx* ctx, uint64_t* faces, uint64_t* fallbacks);

/* ---- CFL time step without any allocation -------------------------------- */

/* Rows of scratch that efvm_cfl_dt_noalloc keeps in static device memory. */
#define EFVM_CFL_NOALLOC_MAX_ROWS 16384

/* The CFL time step (cfl / max wave speed, or fixed_dt) of a state that the
 * caller keeps in its own device memory, computed without allocating anything.
 * It has no counterpart in the reference; it evaluates the same wave speed as
 * efvm_cfl.
 *
 * It is for callers that cannot call cudaMalloc or let a library do it: a host
 * whose device memory is handed out by its own allocator (a framework's memory
 * pool or a fixed per-process budget) has to supply every buffer itself.  Here
 * the caller passes the four conserved planes (device pointers to interior cell
 * (0,0); cell (i,j) at plane[j*pitch + i], pitch in doubles), the grid and
 * params that define spacing, gas and viscosity, a device pointer that
 * receives dt, and the stream to run on (NULL = default stream).  The call is
 * asynchronous on that stream.
 *
 * Its only scratch is file-scope device memory of the library: one double per
 * grid row (EFVM_CFL_NOALLOC_MAX_ROWS rows, 128 KB) and a counter, held on
 * every GPU that loads the library until the process exits.  Grids with more
 * rows are rejected with EFVM_ERR_INVALID_ARG (use efvm_cfl), and so are
 * non-positive extents (hi <= lo on an axis).  Only 2-D meshes are accepted:
 * nz > 1 returns EFVM_ERR_UNSUPPORTED, since a 3-D wave speed needs rho_w and
 * every layer.  The result equals efvm_cfl's bit for bit.  All calls on a
 * device share that scratch and it keeps the last call's contents; calls whose
 * kernels overlap on the GPU race and may return a wrong dt, so order them on
 * one stream.  The first call on a device looks up the scratch's device
 * address (once per device, with that device current); make that first call
 * before any stream capture.  Errors are reported by efvm_last_error(NULL). */
int efvm_cfl_dt_noalloc(const double* rho, const double* rho_u, const double* rho_v, const double* rho_e,
                        int64_t pitch, const efvm_grid* grid, const efvm_params* params, double* dt_out,
                        void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif

#endif /* EFVM_H */
