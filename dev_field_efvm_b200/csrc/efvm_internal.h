// efvm_internal.h — device data layout and kernel parameters shared by the
// CUDA kernels (efvm_kernels.cu) and the C-ABI host code (efvm_api.cu).
//
// HBM layout of one conserved state (structure of arrays, FP64):
//   4 planes (rho, rho_u, rho_v, rho_e), each (ny + 2*YO) rows x `pitch`
//   doubles; interior cell (i, j) sits at row YO + j, column XO + i.  Columns
//   XO-2, XO-1 and XO+nx, XO+nx+1 are the two ghost layers of FIELD's ng = 2
//   (rows likewise).  XO = 4 makes every interior row start on a 32-byte
//   sector; the pitch is a multiple of 8 doubles.  rho_w is identically zero in
//   2-D and is not stored.
// A 3-D state (nz > 1) has 5 planes (rho, rho_u, rho_v, rho_w, rho_e), each
// (nz + 4) layers of `layer` doubles; interior cell (i, j, k) sits in layer 2 + k
// (efvm_kernels3d.cuh).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/efvm.h"

namespace efvm {

constexpr int XO = 4;  // column of interior cell i = 0
constexpr int YO = 2;  // row of interior cell j = 0
constexpr int NG = 2;  // FIELD ghost layers

// Per-step device solver state (SolverState + the CFL reduction buffers).
struct DevState {
    double dt;
    double time;
    unsigned long long step;
    int rk_stage;            // 0,1,2
    int completed;           // StepBoundary.completed_full_step
    unsigned long long lam[2];  // max wave speed (bits of a non-negative double)
    int lam_idx;             // lam[lam_idx] is being accumulated / is current
    int active;              // 0 once t_stop was reached (kernels become no-ops)
    int stop_at_t;
    int nonphysical;         // bit 0: rho<=0, bit 1: p<=0, bit 2: NaN, bit 3: a TMA row wait ran out
    double t_stop;
    long long hist_pos;      // next MarkerForce history slot
    long long hist_cap;
    unsigned long long lam_ext;  // external wave-speed slot (slabs), see efvm_wave_speed_slot
    int ext_lam;             // 1: accumulate into / read from lam_ext
    int forces_pending;      // the last stage's IBM forces are still to run (step graph)
    unsigned long long done_ns;  // device global timer when the set-up stopped the run
    int step_par;            // parity of the step in progress (step & 1 at its set-up): the z-ghost
                             // buffer that the forces of its first two stages read
    int pad_par_;
};

// Boundary side description resolved for the device.
struct DevBC {
    int kind;
    int pad;
    double rho, u, v, w, p, t;
};

struct Geometry {
    int nx, ny;
    int pitch;            // doubles per row
    long long plane;      // doubles per plane
    int nz;               // 1 for the 2-D layout
    int pad3_;
    long long layer;      // doubles per z layer (3-D)
    double inv_z;         // face area / cell volume for z faces
    double lo[3], hi[3];
    double h[3];          // spacing dx, dy, dz
    double inv_x, inv_y;  // face area / cell volume for x and y faces
    double cell_volume;
    int j_off;            // global index of row 0 (slabs; 0 otherwise)
    int pad_;
    double inv_h[3];      // 1 / dx, 1 / dy, 1 / dz (the CFL wave speed)
};

struct Physics {
    double gamma, r_gas;
    double cfl, fixed_dt;
    int flux_scheme, reconstruction, limiter, integrator;
    int viscous, viscosity_model;
    double mu;
    int precision, periodic_seam;
    int periodic_x, periodic_y, periodic_z, pad_z;
    // Slabs (efvm_create_slab): a y side whose ghosts come from a neighbouring
    // slab, and whether that side is the global periodic seam.
    int halo_ylo, halo_yhi;
    int seam_ylo, seam_yhi;
    DevBC bc[6];  // XLO, XHI, YLO, YHI, ZLO, ZHI
    int parabolic_inflow;
    double inflow_u_max, inflow_height, inflow_rho;
    int sponge;
    double sponge_x_start, sponge_x_end, sponge_sigma, sponge_u_max, sponge_height, sponge_rho, sponge_p;
    double body_force_x;
    double dx_inv2;       // 1/(dx*dx), viscous x weight
    double cp;            // gamma*R/(gamma-1)
    double cp_pr;         // cp / 0.72 (Pr), for kappa = mu*cp/Pr
    double cfl_visc_sum;  // 1/dx^2 + 1/dy^2 + 1/dz^2
    double inv_r_gas;     // 1 / R (the CFL wave speed's temperature)
    // Sponge constants, formed once on the host with the device's operations:
    // 1 / (x_end - x_start), p / (gamma - 1), and the 3-D uniform target state.
    double sponge_inv_w, sponge_e0;
    double sponge_t[5];
};

// Bits of IbmGhostDev::fluid / MarkerDev::fluid.  The solid mask changes only
// with the geometry, so which neighbours and bilinear corners are fluid is
// fixed when the lists are built.
constexpr unsigned FLUID_NB_SHIFT = 0;      // +x, -x, +y, -y face neighbour (ghosts only)
constexpr unsigned FLUID_CORNER_SHIFT = 4;  // bilinear corner k = 2*di + dj
// Set on the solid cells the mirror rewrites.  With cylinders that is every solid
// cell (the 2-D mesh's z neighbours are fluid ghost layers); with the moving
// discs only those with a fluid in-plane neighbour (compute_disc_ghosts,
// examples/dkt_sedimentation/main.rs:175-249).  The list holds every solid cell
// either way, for the staircase wall force.
constexpr unsigned GHOST_MIRROR_BIT = 1u << 12;
constexpr int IBM_THREADS = 128;            // threads per block of the IBM kernel

// One solid cell that the IBM mirror refills every substage (IbmGhostCells).
struct IbmGhostDev {
    int i, j;                // interior cell
    int lo_i, lo_j;          // low corner of the bilinear block (interior indices, may be -1 / n)
    double tx, ty;           // bilinear fractions
    int valid;               // locate() succeeded
    unsigned fluid;          // FLUID_* bits
    double uw[2];            // wall velocity at the cell's wall footprint (moving discs)
};

// One surface marker (IbmMarker) with its sample point already located.
struct MarkerDev {
    double normal[3];
    double area;
    double wall_velocity[3];
    int lo_i, lo_j;
    double tx, ty;
    int valid;
    unsigned fluid;          // FLUID_CORNER bits
    double pos[2];           // marker position (its z is the z-cell centre)
    int body;                // cylinder index
    int pad;
};

// 3-D immersed spheres: one solid cell of the ghost list, and one surface
// marker, with their trilinear sample located when the lists are built.
// fluid bits: 0..5 the +x, -x, +y, -y, +z, -z face neighbour; 8 + 4 di + 2 dj + dk
// the trilinear corner (di, dj, dk).
constexpr unsigned FLUID3_CORNER_SHIFT = 8;
struct IbmGhost3Dev {
    int i, j, k, valid;
    int lo[3];
    unsigned fluid;
    double t[3];
    double uw[3];           // wall velocity at the ghost's wall footprint
};
struct Marker3Dev {
    double normal[3];
    double area;
    double uw[3];           // wall velocity at the marker
    double t[3];
    int lo[3];
    int valid;
    unsigned fluid;
    int body;
};

struct Ibm {
    int enabled;
    int n_ghost;
    int n_markers;
    int pad;
    const IbmGhostDev* ghosts;
    const MarkerDev* markers;
    double sample_offset;   // dx
    // emulated z-ghost states of the solid cells (the 2-D mesh's z layers),
    // used only by the staircase wall force: zg0 (saved at stage 1, one buffer
    // per step parity, so that the last stage's forces of one step can run
    // beside the next step's first mirror) and the pre-mirror fill of each RK
    // stage (one buffer per stage)
    double* zg0;            // 2 x n_ghost x 4
    double* zfill;          // 3 x n_ghost x 4
    double* force_out;      // 12 doubles: marker force (6) then wall force (6)
    double* history;        // hist_cap x 6 (may be null)
    double* partials;       // 6 doubles per force block (deterministic reduction)
    unsigned int* counter;  // blocks finished in the current force launch
    const IbmGhost3Dev* ghosts3;  // 3-D lists (spheres)
    const Marker3Dev* markers3;
};

// Everything a stage kernel needs.
struct StageArgs {
    Geometry g;
    Physics ph;
    const double* __restrict__ uin;   // stage input (stencil)
    const double* u0;                 // U^n (RK stages 2 and 3); may alias uout on stage 3
    double* uout;
    const uint8_t* __restrict__ mask; // solid mask (same layout as one plane, bytes) or null
    const double* __restrict__ yw;    // 3*ny viscous y weights: y_im, y_ip, y_is
    const double* __restrict__ zw;    // 3*nz viscous z weights (3-D) or null
    DevState* st;
    int stage;                        // 0,1,2 for RK3; 3 = Euler
    int completes_step;               // sponge + CFL + clock in the epilogue
    int want_cfl;
    const float* corr;                // learned face-flux corrections [2][4][ny][nx] or null
    int defer_forces;                 // stage 2 of the step graph: its IBM forces run in the next launch
    // The TMA-fed stage kernel (2-D, inviscid, no bodies, no correction): host
    // copies of the tensor maps (CUtensorMap, 128 bytes) of the stage input and
    // of U^n, copied into the launch's parameters; null selects the strip kernel.
    const void* tmap_in;
    const void* tmap_u0;
    int rows;                         // rows per warp; 0 = the built-in choice
    int blocks;                       // resident blocks per SM of the strip form; 0 = the built-in choice
    unsigned long long wait_ns;       // limit of one wait of the TMA-fed kernel for a row (ns)
    int stall;                        // failure injection: the first block's ring stops being refilled
    // Slabs with halo peers (efvm_set_halo_peer): the output buffer of this
    // stage of the neighbouring slab below (0) and above (1), its plane and
    // rows; the stage stores its two edge rows straight into that slab's
    // ghost rows.  Null: the side is filled by efvm_halo_unpack instead.
    double* peer_out[2];
    long long peer_plane[2];
    int peer_ny[2];
};

// ---- batches of independent cases (efvm_batch.cu) --------------------------
// One case of a batch, as the batch kernels read it.
struct BatchCase {
    Geometry g;
    Physics ph;             // the shared settings with this case's boundaries and spacing
    int rows;               // rows per warp of this case's tiles
    int pad;
    double* U[3];
    const double* yw;
    DevState* st;
};

// One stage over the tiles of every active case: tile (case, strip, row block)
// is one warp's share of that case's stage.
struct BatchStageArgs {
    Physics ph;             // the shared settings (scheme, precision, gas, CFL)
    const BatchCase* __restrict__ cases;
    const int4* tiles;
    int stage, completes_step, want_cfl;
    int in_buf, out_buf;    // U[in_buf] -> U[out_buf]; U[0] is u^n
};

// One launch of the persistent batch kernel: every warp takes work tickets in
// order; ticket t is RK stage r = t / n_tiles (3 per step) of table tile
// t % n_tiles.  A tile of stage r > 0 waits until its case's stage r - 1 is
// complete (ready[k] >= r; no wait on any other case), the last tile of a
// case's stage publishes it, and the last tile of a step's third stage runs
// that case's next set-up first.  A case that stops publishes ~0u, so its later
// tiles pass at once and skip.  Waits are bounded by wait_ns: a wait that runs
// out sets status bit 0 and the launch winds down (EFVM_ERR_TIMEOUT).
struct PersistArgs {
    Physics ph;                      // the shared settings (scheme, precision, gas, CFL)
    const BatchCase* __restrict__ cases;
    const int4* tiles;               // (case, strip, row block, 0) of every case in the table
    const int* case_tiles;           // per case: its tiles in the table
    unsigned int* ready;             // per case: stages of this launch complete
    unsigned int* done;              // per case: tiles completed in this launch
    unsigned long long* ticket;      // the next work ticket
    int* status;
    long long n_tiles;
    int rounds;                      // RK stages this launch runs (3 per step)
    int want_cfl;
    unsigned long long wait_ns;
};
int launch_batch_persistent(const PersistArgs& p, int blocks_per_sm, int n_sms, void* stream);
// Resident blocks per SM of the batch stage forms (their register budget).
int batch_form_blocks(bool fp32, bool viscous);

// Stage-kernel tiling of one case: strips of columns, and rows per warp for a
// case that runs alone (fp32: the FP32-flux form; viscous: with viscous terms).
int stage_strips(int nx);
int stage_rows(int nx, int ny, bool fp32, bool viscous, bool tma = false);
// Resident blocks per SM of the stage-kernel form (tma: the TMA-fed kernel), and
// the strip form's second choice for the autotuner (0: none).
int stage_blocks_per_sm(bool fp32, bool viscous, bool tma);
int stage_alt_blocks(bool fp32, bool viscous);
// Whether a stage of this case can run the TMA-fed kernel (2-D, inviscid, no
// immersed bodies, no learned correction), and the tensor map of a state
// buffer of the case's layout as a 3-D tensor (columns, rows, planes) with the
// box of the stage input (u0 = false) or of U^n (u0 = true); 0 on success.
bool stage_tma_eligible(const Geometry& g, const Physics& ph, bool ibm, bool corr);
int encode_state_map(const Geometry& g, const double* buf, bool u0, void* map_out);
int launch_batch_stage(const BatchStageArgs& b, int n_tiles, bool pdl, void* stream);
// Per-step set-up of every case (one thread each).
int launch_batch_setup(const Physics& ph, const BatchCase* cases, int n_cases, bool pdl, void* stream);
// Write the device global timer (ns) to *out.
int launch_clock(unsigned long long* out, void* stream);

// The learned correction (efvm_nn.cu): corrections of every face of one
// periodic context state, and the kernel attributes its launches need.
int nn_forward_padded(const efvm_nn* h, const double* q, long long plane, int pitch, int nx, int ny, float* corr,
                      float4* prims, float sensor, unsigned long long* fallbacks, void* stream);
int nn_prepare_launches();

// Validation and the device description of one case (efvm_api.cu): global rows
// [row0, row0 + rows) of `gr`, halo sides when `slab`.  Returns a status and
// sets `err` on failure.
int setup_case(const efvm_grid& gr, const efvm_params& p, int row0, int rows, bool slab, Geometry& g, Physics& ph,
               std::string& err);
std::vector<double> viscous_y_weights(const Geometry& g);
std::vector<double> viscous_z_weights(const Geometry& g);

// Sets the message efvm_last_error(NULL) returns (efvm_api.cu).
void set_global_error(const std::string& msg);

// Host-side launch wrappers (efvm_kernels.cu); each returns the number of
// kernels it launched.
// `pdl`: launch with programmatic stream serialization (the kernels of a step).
int launch_stage(const StageArgs& a, bool pdl, void* stream);
int launch_fill_ghosts(const Geometry& g, const Physics& ph, double* q, void* stream);
int launch_cfl(const Geometry& g, const Physics& ph, const double* q, DevState* st, void* stream);
int launch_step_setup(const Physics& ph, DevState* st, bool pdl, void* stream);
int launch_geometry(const Geometry& g, const double* cyl, int ncyl, const double* stagnant, const double* ambient,
                     double* q, uint8_t* mask, void* stream);
// IBM work between stage kernels, one launch: the forces of the state q after
// stage force_stage (-1: none), the ghost mirror of q for stage mirror_stage
// (-1: none) and, with setup, the per-step set-up before the mirror.  With
// deferred, the forces are those of the last stage of the previous step, run
// only while DevState::forces_pending is set (and cleared by them).
int launch_ibm(const Geometry& g, const Physics& ph, const Ibm& ibm, double* q, DevState* st,
               int force_stage, int mirror_stage, int setup, bool pdl, void* stream, int deferred = 0);
int launch_pack(const Geometry& g, const double* host_like, int64_t si, int64_t sj, int64_t sv, double* q,
                 int to_device, void* stream);
// 3-D spheres: the solid mask with the stagnant/ambient re-seed of flipped
// cells (spheres: n x 10 doubles as efvm_sphere), the ghost mirror of q before
// a stage, and the marker and staircase forces of q after one (one block,
// fixed-order sums, the marker force appended to the history when it is set).
int launch_geometry3(const Geometry& g, const Physics& ph, const double* spheres, int n, const double* stagnant,
                     const double* ambient, double* q, uint8_t* mask, void* stream);
int launch_mirror3(const Geometry& g, const Physics& ph, const Ibm& ib, double* q, bool pdl, void* stream);
int launch_forces3(const Geometry& g, const Physics& ph, const Ibm& ib, const double* q, DevState* st, bool pdl,
                   void* stream);
// The same for a 3-D state: element (i, j, k, v) at i si + j sj + k sk + v sv.
int launch_pack3(const Geometry& g, double* host_like, int64_t si, int64_t sj, int64_t sk, int64_t sv, double* q,
                 int to_device, void* stream);
int launch_init_vortex(const Geometry& g, const efvm_vortex& v, double* q, void* stream);
int launch_density_error(const Geometry& g, const efvm_vortex& v, const double* q, const DevState* st,
                          double* partial, int nblocks, void* stream);
int launch_total_mass(const Geometry& g, const double* q, double* partial, int nblocks, void* stream);
// Rows j0, j0+1 (all four variables, interior columns) to buf (unpack = 0) or
// from buf (unpack = 1); buf is [variable][row][i], 8*nx doubles.
int launch_halo_rows(const Geometry& g, double* q, double* buf, int j0, int unpack, void* stream);
// Per-body marker loads and torque (compute_marker_loadings_per_body): one warp
// per body over its n_theta consecutive markers; out[9 b ..] = pressure[3],
// viscous[3], torque[3] about (centres[2 b], centres[2 b + 1]).
int launch_body_loads(const Geometry& g, const Physics& ph, const Ibm& ib, const double* q, const double* centres,
                      int n_bodies, int markers_per_body, double* out, void* stream);
// The VTK output fields (7 planes of nx*ny doubles) of a state.
int launch_output_fields(const Geometry& g, const Physics& ph, const double* q, double* out, void* stream);
int launch_set_control(DevState* st, int active, int stop_at_t, double t_stop, long long hist_cap, void* stream);

}  // namespace efvm
