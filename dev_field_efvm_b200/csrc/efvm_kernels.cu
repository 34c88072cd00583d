// efvm_kernels.cu — sm_100a kernels of the explicit finite-volume step.
//
//   stage_kernel   one RK substage over strips of 31 columns: MUSCL slopes, L/R face
//                  states, one numerical flux per face (HLLC-Thornber /
//                  textbook HLLC / Rusanov), flux divergence, viscous terms,
//                  solid-cell zeroing, body force, SSP-RK3 (or Euler)
//                  combination, and on the step's last stage the sponge, the
//                  boundary-ghost refill of the output and the CFL wave-speed
//                  max (one atomic per warp).
//   fill_ghosts    Halo + Boundary phases for a freshly uploaded state.
//   step_setup     per-step dt = cfl / max wave speed, clock/stop bookkeeping.
//   ibm_kernel     ghost-cell IBM mirror (bilinear image sample) and, after a
//                  stage, the marker-integrated and staircase wall forces.
//   geometry       cylinder solid mask and the stagnant/ambient re-seed.
//   utilities      strided pack/unpack, vortex init, error and mass partials.
//   efvm_kernels3d.cuh  the 3-D forms: stage3 (x, y and z faces, warps stacked
//                  in z), ghost fill, CFL, transfers, mass, and the sphere
//                  geometry, mirror and force kernels.
//
// The stencil kernels are bound by instruction issue and FP64 dependency
// latency: HBM runs at 10-25 % of its copy bandwidth and the FP64 units at
// 15-25 % of their peak.  No tensor cores are involved.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstdio>

#include "efvm_internal.h"
#include "efvm_math.cuh"
#include "efvm_tma.cuh"

namespace efvm {

namespace {

__device__ __forceinline__ long long cidx(const Geometry& g, int i, int j) {
    return (long long)(YO + j) * g.pitch + (XO + i);
}

// Programmatic dependent launch.  The kernels of a step are launched with
// programmatic stream serialization, so a kernel's blocks may be scheduled while
// its predecessor is still draining.  Each such kernel waits for the predecessor
// to complete (and its writes to become visible) before it reads anything, then
// lets its own successor launch.  Without the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_wait_then_release() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Cell centre lo + (i + 0.5) h with one rounding per operation, as the host
// computes it (no FMA), so geometry tests agree bit for bit.
__device__ __forceinline__ double centre(double lo, double h, int i) {
    return __dadd_rn(lo, __dmul_rn((double)i + 0.5, h));
}

// ---- 2-D conserved state in the grid frame ---------------------------------
struct U4 {
    double r, mx, my, E;
};

__device__ __forceinline__ U4 load4(const double* q, long long plane, long long o) {
    return U4{q[o], q[plane + o], q[2 * plane + o], q[3 * plane + o]};
}
// Loads of a stage's inputs.  CG: through L2 only (ld.global.cg), for the
// persistent batch kernel, whose inputs were written earlier in the same launch
// by other blocks (an L1 line of this SM could still hold an older value).
template <bool CG>
__device__ __forceinline__ double gld(const double* p) {
    if constexpr (CG) return __ldcg(p);
    else return *p;
}
template <bool CG>
__device__ __forceinline__ U4 load4g(const double* q, long long plane, long long o) {
    return U4{gld<CG>(q + o), gld<CG>(q + plane + o), gld<CG>(q + 2 * plane + o), gld<CG>(q + 3 * plane + o)};
}
__device__ __forceinline__ void store4(double* q, long long plane, long long o, const U4& u) {
    q[o] = u.r;
    q[plane + o] = u.mx;
    q[2 * plane + o] = u.my;
    q[3 * plane + o] = u.E;
}

// The helpers below (pressure, prim_to_cons, the boundary ghosts, the wave
// speed) are evaluated in more than one kernel on the same state: the stage
// epilogue refills ghosts and takes the CFL maximum, and the stand-alone ghost
// fill and CFL pass do the same after an upload.  A restart must see identical
// values from both, so these round every operation explicitly (no FMA
// contraction, whose choice may differ between inlined copies).
__device__ __forceinline__ double mul_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_(double a, double b) { return __dsub_rn(a, b); }

// IdealGas::pressure, crates/cfd_eos/src/lib.rs:61-64 (w = 0)
__device__ __forceinline__ double pressure_d(const U4& u, double gm1) {
    return mul_(gm1, sub_(u.E, mul_(0.5, add_(mul_(u.mx, u.mx), mul_(u.my, u.my))) / u.r));
}

// IdealGas::prim_to_cons (2-D, w = 0), crates/cfd_eos/src/lib.rs:55-59
__device__ __forceinline__ U4 prim_to_cons(double rho, double u, double v, double p, double gm1) {
    const double ke = mul_(mul_(0.5, rho), add_(mul_(u, u), mul_(v, v)));
    return U4{rho, mul_(rho, u), mul_(rho, v), add_(p / gm1, ke)};
}

// Viscosity::mu, crates/cfd_eos/src/lib.rs:108-117 (Sutherland :75-80)
__device__ __forceinline__ double viscosity(const Physics& ph, double t) {
    if (ph.viscosity_model == EFVM_VISC_CONSTANT) return ph.mu;
    const double MU_REF = 1.827e-5, T_REF = 291.15, S = 120.0;
    return MU_REF * pow(t / T_REF, 1.5) * (T_REF + S) / (t + S);
}

// One boundary ghost from its interior neighbour (BoundaryCondition::ghost_at),
// crates/cfd_boundary/src/lib.rs:172-362.  side = 0..3 (XLO, XHI, YLO, YHI).
__device__ __forceinline__ U4 bc_ghost(const DevBC& bc, int side, const U4& in, double gm1) {
    switch (bc.kind) {
        case EFVM_BC_SLIP_WALL:
        case EFVM_BC_SYMMETRY: {
            const double n0 = side < 2 ? (side == 1 ? 1.0 : -1.0) : 0.0;
            const double n1 = side >= 2 ? (side == 3 ? 1.0 : -1.0) : 0.0;
            const double mn = add_(mul_(in.mx, n0), mul_(in.my, n1));
            U4 g = in;
            g.mx = sub_(in.mx, mul_(mul_(2.0, mn), n0));
            g.my = sub_(in.my, mul_(mul_(2.0, mn), n1));
            return g;
        }
        case EFVM_BC_NO_SLIP_WALL:
            return U4{in.r, -in.mx, -in.my, in.E};
        case EFVM_BC_SUPERSONIC_INFLOW: {
            const double ke = mul_(mul_(0.5, bc.rho), add_(add_(mul_(bc.u, bc.u), mul_(bc.v, bc.v)), mul_(bc.w, bc.w)));
            return U4{bc.rho, mul_(bc.rho, bc.u), mul_(bc.rho, bc.v), add_(bc.p / gm1, ke)};
        }
        case EFVM_BC_SUBSONIC_INFLOW: {
            const double p_in = pressure_d(in, gm1);
            const double ke = mul_(mul_(0.5, bc.rho), add_(add_(mul_(bc.u, bc.u), mul_(bc.v, bc.v)), mul_(bc.w, bc.w)));
            return U4{bc.rho, mul_(bc.rho, bc.u), mul_(bc.rho, bc.v), add_(p_in / gm1, ke)};
        }
        case EFVM_BC_PRESSURE_OUTLET: {
            const double inv = 1.0 / in.r;
            const double u = mul_(in.mx, inv), v = mul_(in.my, inv);
            return prim_to_cons(in.r, u, v, bc.p, gm1);
        }
        default:
            return in;
    }
}

// Boundary-ghost refill for the cell (i, j) whose new value is `u`: the Halo
// (periodic wrap) and Boundary phases of the next substage, done by the thread
// that owns the interior source cell (each ghost has exactly one writer).
// PXY: both axes are known to be periodic at compile time (the TMA-fed form
// of fully periodic cases), so the boundary-condition paths are not compiled.
template <bool PXY = false>
__device__ __forceinline__ void write_ghosts(const Geometry& g, const Physics& ph, double* q, int i, int j,
                                             const U4& u) {
    const long long P = g.plane;
    const double gm1 = ph.gamma - 1.0;
    if (PXY || ph.periodic_x) {
        if (i >= g.nx - NG) store4(q, P, cidx(g, i - g.nx, j), u);
        if (i < NG) store4(q, P, cidx(g, i + g.nx, j), u);
    } else {
        if (i == 0) {
            store4(q, P, cidx(g, -1, j), bc_ghost(ph.bc[0], 0, u, gm1));
            if (ph.parabolic_inflow) {
                // parabolic_inflow_system, examples/cylinder_drag_validation/main.rs:151-177
                const double y = centre(g.lo[1], g.h[1], j + g.j_off);
                const double um = ph.inflow_u_max, hh = ph.inflow_height, rho = ph.inflow_rho;
                const double uy = mul_(mul_(mul_(4.0, um), y), sub_(hh, y)) / mul_(hh, hh);
                const double p_in = pressure_d(u, gm1);
                const U4 c = prim_to_cons(rho, uy, 0.0, p_in, gm1);
                store4(q, P, cidx(g, -1, j), c);
                store4(q, P, cidx(g, -2, j), c);
            }
        }
        if (i == g.nx - 1) store4(q, P, cidx(g, g.nx, j), bc_ghost(ph.bc[1], 1, u, gm1));
    }
    if (PXY || ph.periodic_y) {
        if (j >= g.ny - NG) store4(q, P, cidx(g, i, j - g.ny), u);
        if (j < NG) store4(q, P, cidx(g, i, j + g.ny), u);
    } else {
        // a side that faces another slab is filled by the caller's halo exchange
        if (j == 0 && !ph.halo_ylo) store4(q, P, cidx(g, i, -1), bc_ghost(ph.bc[2], 2, u, gm1));
        if (j == g.ny - 1 && !ph.halo_yhi) store4(q, P, cidx(g, i, g.ny), bc_ghost(ph.bc[3], 3, u, gm1));
    }
}

// A slab's two rows next to a side with a halo peer go straight into the
// peer's ghost rows of the same stage's output: rows 0, 1 become the lower
// slab's rows ny_lo, ny_lo + 1, and rows ny - 2, ny - 1 the upper slab's rows
// -2, -1 (the peers share this slab's nx, hence its pitch).  The exchange that
// halo_exchange_forward_all does between stages then happens as the stage
// writes, on this GPU's peer memory path (another slab's buffer on the same
// GPU, or a peer GPU's buffer over NVLink).  Batch cases have no peers.
__device__ __forceinline__ void peer_rows(const StageArgs& a, const Geometry& g, int i, int j, const U4& u) {
    if (a.peer_out[0] && j < NG)
        store4(a.peer_out[0], a.peer_plane[0], (long long)(YO + a.peer_ny[0] + j) * g.pitch + (XO + i), u);
    if (a.peer_out[1] && j >= g.ny - NG)
        store4(a.peer_out[1], a.peer_plane[1], (long long)(YO + j - g.ny) * g.pitch + (XO + i), u);
    // a peer on another GPU reads these rows after the stage: make them visible system-wide
    if ((a.peer_out[0] && j < NG) || (a.peer_out[1] && j >= g.ny - NG)) __threadfence_system();
}
template <class A>
__device__ __forceinline__ void peer_rows(const A&, const Geometry&, int, int, const U4&) {}

// The wave-speed accumulator of the current step: the context's own double
// buffer, or the external slot that slabs max-reduce across GPUs.
__device__ __forceinline__ unsigned long long* lam_slot(DevState* st) {
    return st->ext_lam ? &st->lam_ext : &st->lam[st->lam_idx];
}
// The same slot, its selectors read coherently (the persistent batch kernel).
__device__ __forceinline__ unsigned long long* lam_slot_v(DevState* st) {
    const volatile DevState* v = st;
    return v->ext_lam ? &st->lam_ext : &st->lam[v->lam_idx];
}

// Local max wave speed of cfl_system, crates/cfd_solver/src/lib.rs:647-669.
// The divisions of the reference's formula (by rho, by dx/dy/dz, by R) are taken
// as products with reciprocals (1 / rho once per cell, the others once per
// mesh): the wave speed differs from the reference's by a few ulps, and so
// does dt, far below the step's own error.  The stage epilogue and the
// stand-alone CFL pass both call this function, so they agree bit for bit.
__device__ __forceinline__ double wave_speed(const Geometry& g, const Physics& ph, const U4& u) {
    if (!(u.r > 0.0)) return 0.0;
    const double gm1 = ph.gamma - 1.0;
    const double inv = 1.0 / u.r;
    const double vx = mul_(u.mx, inv), vy = mul_(u.my, inv);
    const double ke = mul_(mul_(0.5, u.r), add_(mul_(vx, vx), mul_(vy, vy)));
    const double p = mul_(gm1, sub_(u.E, ke));
    const double a = sqrt(mul_(mul_(ph.gamma, p), inv));
    double lam = add_(add_(mul_(add_(fabs(vx), a), g.inv_h[0]), mul_(add_(fabs(vy), a), g.inv_h[1])),
                      mul_(add_(0.0, a), g.inv_h[2]));
    if (ph.viscous) {
        const double t = mul_(mul_(p, inv), ph.inv_r_gas);
        const double nu = mul_(viscosity(ph, t), inv);
        lam = add_(lam, mul_(mul_(2.0, nu), ph.cfl_visc_sum));
    }
    return lam;
}

__device__ __forceinline__ void block_max_atomic(double v, unsigned long long* target) {
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nw = (blockDim.x * blockDim.y + 31) / 32;
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid < 32) {
        double w = tid < nw ? red[tid] : 0.0;
        for (int o = 16; o > 0; o >>= 1) w = fmax(w, __shfl_xor_sync(0xffffffffu, w, o));
        if (tid == 0 && w > 0.0 && w == w) atomicMax(target, (unsigned long long)__double_as_longlong(w));
    }
}

// A conserved state in the reconstruction precision R, grid frame.
template <class R>
struct V4 {
    R r, mx, my, E;
};
template <class R>
__device__ __forceinline__ V4<R> toR(const U4& u) {
    return V4<R>{R(u.r), R(u.mx), R(u.my), R(u.E)};
}
__device__ __forceinline__ U4 toU4(const V4<double>& u) { return U4{u.r, u.mx, u.my, u.E}; }
__device__ __forceinline__ U4 toU4(const V4<float>& u) { return U4{u.r, u.mx, u.my, u.E}; }
// The state in the frame of an x-face (normal x) or a y-face (normal y).
template <class R>
__device__ __forceinline__ Q4<R> xq(const V4<R>& u) {
    return Q4<R>{u.r, u.mx, u.my, u.E};
}
template <class R>
__device__ __forceinline__ Q4<R> yq(const V4<R>& u) {
    return Q4<R>{u.r, u.my, u.mx, u.E};
}

// The two face states c + s/2 (toward the next cell) and c - s/2 (toward the
// previous one) of a cell, s = lim(p - c, c - m) per conserved variable
// (limited_slope_cons and reconstruct_to_face, crates/cfd_solver/src/lib.rs:199-211,273-286);
// m/c/p are the previous/own/next cells along the face normal.  The FP32 path
// takes the differences in FP32.
//
// fp and fm scale the slope of the two states: 0.5 where the face on that side
// reconstructs this cell, 0 where it takes the cell value itself (a first-order
// side on the domain edge), so the edge faces need no select of whole states.
// c + s fp and c - s fm are each one multiply-add; with fp = fm = 0.5 the
// product is exact, so they are the bits of c + (s/2) and c - (s/2), and with 0
// they are c.
template <class R>
__device__ __forceinline__ R half_slope(int limiter, R m, R c, R p) {
    return limit<R>(limiter, p - c, c - m) * R(0.5);
}
__device__ __forceinline__ double fma_(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fma_(float a, float b, float c) { return fmaf(a, b, c); }
template <class R>
__device__ __forceinline__ void slope_faces(int limiter, const V4<R>& m, const V4<R>& c, const V4<R>& p, R fp, R fm,
                                            V4<R>& plus, V4<R>& minus) {
    const R sr = limit<R>(limiter, p.r - c.r, c.r - m.r), sx = limit<R>(limiter, p.mx - c.mx, c.mx - m.mx);
    const R sy = limit<R>(limiter, p.my - c.my, c.my - m.my), se = limit<R>(limiter, p.E - c.E, c.E - m.E);
    plus = V4<R>{fma_(sr, fp, c.r), fma_(sx, fp, c.mx), fma_(sy, fp, c.my), fma_(se, fp, c.E)};
    minus = V4<R>{fma_(-sr, fm, c.r), fma_(-sx, fm, c.mx), fma_(-sy, fm, c.my), fma_(-se, fm, c.E)};
}
// The same two states with both factors 0.5, as c + h and c - h of one half
// slope h = s/2: the same bits as the factor form.  The FP32-flux forms and
// the batch kernels use this one (the factor form raised their spills).
template <class R>
__device__ __forceinline__ void slope_faces_half(int limiter, const V4<R>& m, const V4<R>& c, const V4<R>& p,
                                                 V4<R>& plus, V4<R>& minus) {
    const R hr = half_slope(limiter, m.r, c.r, p.r), hx = half_slope(limiter, m.mx, c.mx, p.mx);
    const R hy = half_slope(limiter, m.my, c.my, p.my), he = half_slope(limiter, m.E, c.E, p.E);
    plus = V4<R>{c.r + hr, c.mx + hx, c.my + hy, c.E + he};
    minus = V4<R>{c.r - hr, c.mx - hx, c.my - hy, c.E - he};
}
// The slope factor of a side that a face does (0.5) or does not (0) reconstruct.
template <class R>
__device__ __forceinline__ R rec_factor(bool rec) {
    return rec ? R(0.5) : R(0);
}

template <class R>
__device__ __forceinline__ V4<R> shfl_up_v(const V4<R>& u, int d) {
    return V4<R>{__shfl_up_sync(0xffffffffu, u.r, d), __shfl_up_sync(0xffffffffu, u.mx, d),
                 __shfl_up_sync(0xffffffffu, u.my, d), __shfl_up_sync(0xffffffffu, u.E, d)};
}
template <class R>
__device__ __forceinline__ V4<R> shfl_down_v(const V4<R>& u, int d) {
    return V4<R>{__shfl_down_sync(0xffffffffu, u.r, d), __shfl_down_sync(0xffffffffu, u.mx, d),
                 __shfl_down_sync(0xffffffffu, u.my, d), __shfl_down_sync(0xffffffffu, u.E, d)};
}

template <class R>
__device__ __forceinline__ Q4<R> shfl_up_q(const Q4<R>& u, int d) {
    return Q4<R>{__shfl_up_sync(0xffffffffu, u.r, d), __shfl_up_sync(0xffffffffu, u.mn, d),
                 __shfl_up_sync(0xffffffffu, u.mt, d), __shfl_up_sync(0xffffffffu, u.E, d)};
}
template <class R>
__device__ __forceinline__ Q4<R> shfl_down_q(const Q4<R>& u, int d) {
    return Q4<R>{__shfl_down_sync(0xffffffffu, u.r, d), __shfl_down_sync(0xffffffffu, u.mn, d),
                 __shfl_down_sync(0xffffffffu, u.mt, d), __shfl_down_sync(0xffffffffu, u.E, d)};
}

// Primitive (u, v, T) of a state given 1/rho (cons_to_prim, crates/cfd_eos/src/lib.rs:44-53).
__device__ __forceinline__ void prim_uvt(const U4& u, double inv, double gm1, double inv_r_gas, double& vu, double& vv,
                                         double& t) {
    vu = u.mx * inv;
    vv = u.my * inv;
    const double ke = 0.5 * u.r * (vu * vu + vv * vv);
    t = gm1 * (u.E - ke) * inv * inv_r_gas;  // T = p / (rho R), the division by R as a product
}

constexpr int STRIP = 31;  // cells a warp owns per row (lane 31 supplies the right face)
constexpr int WPB = 4;     // warps per block

// Where a stage reads its rows, the halo cells of a row and U^n.
//
// GlobalSrc reads them from the state buffers in global memory (through L1 and
// L2); its hooks around each row are empty.
template <bool CG>
struct GlobalSrc {
    const double* uin;
    const double* u0;
    const double* colp = nullptr;  // this lane's column at row 0
    long long P = 0;
    int pitch = 0;
    __device__ __forceinline__ void bind(const Geometry& g, int /*i*/, int ic) {
        P = g.plane;
        pitch = g.pitch;
        colp = uin + cidx(g, ic, 0);
    }
    __device__ __forceinline__ U4 col(int jj) const { return load4g<CG>(colp, P, (long long)jj * pitch); }
    __device__ __forceinline__ U4 at(const Geometry& g, int ii, int jj) const {
        return load4g<CG>(uin, P, cidx(g, ii, jj));
    }
    __device__ __forceinline__ double u0v(int v, long long o, int /*i*/, int /*j*/) const {
        return gld<CG>(u0 + v * P + o);
    }
    __device__ __forceinline__ bool wait_row(int) { return true; }
    __device__ __forceinline__ void refill(int) {}
    __device__ __forceinline__ void release(int) {}
};

// TmaSrc reads them from the block's shared-memory row ring (efvm_tma.cuh),
// which TMA fills ahead of use: before the first read of row r the warp
// waits for its slot (wait_row), at the start of iteration j thread 0 loads row
// j - 1 + RING into the slot that row j - 1 held (refill), and at the end of iteration
// j every warp releases row j (release).
struct TmaSrc {
    double* ring;
    uint64_t* full;
    uint64_t* empty;
    const CUtensorMap* map_in;
    const CUtensorMap* map_u0;  // null: this stage reads no U^n
    DevState* st;
    int first, last;            // the block's row stream
    int u0_lo, u0_hi;           // rows [u0_lo, u0_hi) carry a U^n copy
    int x_in, x_u0;             // tensor-map x of slot column 0 (input, U^n)
    int col0;                   // interior column of input slot column 0
    int scol;                   // this lane's input slot column
    int issued;                 // producer: the last row issued
    unsigned long long wait_ns; // limit of one wait
    bool producer;
    bool stall;                 // failure injection: the producer issues no row after the first RING
    bool ok;

    static constexpr int SLOT_D = tma::SLOT_BYTES / 8;
    __device__ __forceinline__ int slot(int r) const { return (r - first) & (tma::RING - 1); }
    __device__ __forceinline__ uint32_t parity(int r) const { return (uint32_t)((r - first) / tma::RING) & 1u; }
    __device__ __forceinline__ const double* row(int r) const { return ring + slot(r) * SLOT_D; }
    __device__ __forceinline__ void issue(int r) {
        const int s = slot(r);
        double* base = ring + s * SLOT_D;
        const bool with_u0 = tma::U0_IN_RING && map_u0 != nullptr && r >= u0_lo && r < u0_hi;
        tma::arrive_expect(&full[s], tma::IN_BYTES + (with_u0 ? tma::U0_BYTES : 0));
        tma::load_3d(base, map_in, x_in, r + YO, 0, &full[s]);
        if (with_u0) tma::load_3d(base + tma::IN_BYTES / 8, map_u0, x_u0, r + YO, 0, &full[s]);
        issued = r;
    }
    __device__ __forceinline__ void fail() {
        ok = false;
        atomicOr(&st->nonphysical, tma::TIMEOUT_BIT);
    }
    __device__ __forceinline__ void bind(const Geometry&, int i, int /*ic*/) { scol = i - col0; }
    __device__ __forceinline__ U4 col(int jj) const {
        const double* p = row(jj) + scol;
        return U4{p[0], p[tma::IN_COLS], p[2 * tma::IN_COLS], p[3 * tma::IN_COLS]};
    }
    __device__ __forceinline__ U4 at(const Geometry&, int ii, int jj) const {
        const double* p = row(jj) + (ii - col0);
        return U4{p[0], p[tma::IN_COLS], p[2 * tma::IN_COLS], p[3 * tma::IN_COLS]};
    }
    const double* u0;           // U^n in global memory (when the ring holds no U^n rows)
    long long plane;
    __device__ __forceinline__ double u0v(int v, long long o, int i, int j) const {
        if constexpr (tma::U0_IN_RING) return row(j)[tma::IN_BYTES / 8 + v * tma::U0_COLS + (i - col0 - 2)];
        else return u0[v * plane + o];
    }
    // Every lane waits; the warp goes on only if all of them saw the row land.
    __device__ __forceinline__ bool wait_row(int r) {
        const bool got = ok && tma::wait(&full[slot(r)], parity(r), wait_ns);
        if (__all_sync(0xffffffffu, got)) return true;
        if (ok) fail();
        return false;
    }
    __device__ __forceinline__ void refill(int j) {
        if (!producer || !ok || stall) return;
        const int r = j - 1 + tma::RING;  // into the slot that row j - 1 held
        if (r > last) return;
        if (j - 1 >= first && !tma::wait(&empty[slot(j - 1)], parity(j - 1), wait_ns)) {
            fail();
            return;
        }
        issue(r);
    }
    __device__ __forceinline__ void release(int r) {
        __syncwarp();
        if ((threadIdx.x & 31) == 0) tma::arrive(&empty[slot(r)]);
    }
    // Thread 0 before the block exits after a wait ran out: wait (bounded) for
    // every copy it issued, so that none lands after the block is gone.
    __device__ __forceinline__ void drain() {
        for (int r = max(first, issued - (tma::RING - 1)); r <= issued; ++r)
            if (!tma::wait(&full[slot(r)], parity(r), wait_ns)) return;
    }
};

}  // namespace

// ---------------------------------------------------------------------------
// The fused stage kernel.
//
// Each warp owns a strip of 31 columns and marches up `rows` rows of it.  Lane
// l holds column i0+l and, per row, computes the x-face flux on the left of its
// column and the y-face flux above it; the x neighbours come from warp
// shuffles and the y-face flux below a row is carried from the previous row,
// so every face is evaluated once per strip and no block barrier is needed.
// Each lane then forms the flux divergence of its own cell (lanes 0..30),
// adds the viscous terms, zeroes solid cells, applies the RK combination and,
// on a step's last stage, the sponge, refills the boundary ghosts of the output
// and takes the wave-speed max for the next step's CFL dt.
// ---------------------------------------------------------------------------
// LIM >= 0 fixes the limiter at compile time and PXY a fully periodic grid
// (the TMA-fed form is built per limiter and for that case); -1 and false read
// them from the physics at run time.
template <int SCHEME, int RECON, class R, bool VISC, class A, bool CORR, bool XFIRST, bool CG, class SRC,
          int LIM = -1, bool PXY = false>
__device__ __forceinline__ void stage_strip_src(const A& a, int rows, int strip, int by, SRC& src) {
    if (!(CG ? *(volatile const int*)&a.st->active : a.st->active)) return;
    const Geometry& g = a.g;
    const Physics& ph = a.ph;
    const long long P = g.plane;
    const int lane = threadIdx.x & 31;
    if (strip == 0 && by == 0 && lane == 0) {
        // RK state machine and clock of update_system, crates/cfd_solver/src/lib.rs:607-621
        // (no other thread reads time/step/rk_stage during this stage)
        auto machine = [&](auto* st) {
            if (a.stage >= 2) {
                st->rk_stage = 0;
                st->completed = 1;
                st->step += 1;
                st->time += st->dt;
                if (a.defer_forces) st->forces_pending = 1;
            } else {
                st->rk_stage = a.stage + 1;
                st->completed = 0;
            }
        };
        // the persistent batch kernel's set-up writes the state from other blocks
        // during the launch: coherent (volatile) accesses there
        if constexpr (CG) machine((volatile DevState*)a.st);
        else machine(a.st);
    }
    const int i0 = strip * STRIP;
    const int jb = by * rows;
    double lam = 0.0;
    if (i0 < g.nx && jb < g.ny) {  // uniform across the warp
        constexpr bool MUSCL = RECON == EFVM_RECON_MUSCL;
        constexpr bool FP64 = sizeof(R) == sizeof(double);
        const int je = min(jb + rows, g.ny);
        const int i = i0 + lane;
        const int ic = min(i, g.nx + NG - 1);  // clamped load column (lanes past the grid)
        const bool owner = lane < STRIP && i < g.nx;
        const bool true_seam = ph.periodic_seam == EFVM_SEAM_TRUE_PERIODIC;
        const double gm1 = ph.gamma - 1.0;
        const R rg = R(ph.gamma), rgm1 = R(gm1);
        const int limiter = LIM >= 0 ? LIM : ph.limiter;
        const double* __restrict__ uin = a.uin;  // the viscous neighbours
        src.bind(g, i, ic);
        auto ld = [&](int ii, int jj) { return src.at(g, ii, jj); };
        auto ldrow = [&](int jj) { return toR<R>(src.col(jj)); };

        // What a lane carries from one row to the next (the flux of the y face
        // below the row, in the face frame, and the row's +y face state) and,
        // within a row, the x part of the flux divergence while the y face is
        // formed.  The FP32-flux forms keep them in registers.  The FP64 forms
        // keep them in shared memory, one slot per thread (12 doubles, 12 KB per
        // block): that frees 24 registers through both flux evaluations, halves
        // the FP64 inviscid form's spills, and took the 4096^2 FP64 strip step
        // from 2.73 to 2.58 ms (FP32 fluxes, TMA form: 1.73 -> 1.90 ms, so not
        // there).
        constexpr bool CARRY_GB = FP64, CARRY_PC = FP64, CARRY_PART = FP64;
        constexpr int SLOT_GB = 0, SLOT_PC = SLOT_GB + (CARRY_GB ? 4 : 0), SLOT_PART = SLOT_PC + (CARRY_PC ? 4 : 0);
        constexpr int CARRY_SLOTS = SLOT_PART + (CARRY_PART ? 4 : 0);
        __shared__ double carry_s[CARRY_SLOTS > 0 ? CARRY_SLOTS : 1][32 * WPB];
        const int tq = threadIdx.x;

        // Which sides of the faces on the domain edge are reconstructed; every
        // interior face reconstructs both sides under MUSCL.  x: this lane's face,
        // between columns i-1 and i, takes column i-1's +x state (rec_l) and
        // column i's -x state (rec_r), or the cell values where they are false.
        // y: the faces below row 0 and above row ny-1 (rec_below, rec_above).
        bool rec_l = true, rec_r = true;  // face i: column i-1's +x state, column i's -x state
        if (i == 0) {
            rec_l = ph.periodic_x && true_seam;
            rec_r = ph.periodic_x;
        } else if (i == g.nx) {
            rec_l = ph.periodic_x;
            rec_r = ph.periodic_x && true_seam;
        }
        const bool y_periodic = ph.periodic_y || ph.seam_ylo || ph.seam_yhi;
        const bool seam_rec = y_periodic && true_seam;  // the side across the periodic seam
        const bool edge_rec = y_periodic;               // the side inside the domain
        // y face above row jj: whether its lower side (row jj's +y state) and
        // its upper side (row jj+1's -y state) are reconstructed; an edge between
        // slabs is an interior face.  Warp-uniform.  (The edge conditions are
        // read where they are used: hoisted out of the loop they made the batch
        // kernels, whose physics is read from the case table, 6 % slower.)
        auto rec_below = [&](int jj) {
            const bool lo_edge_rows = !ph.halo_ylo || ph.seam_ylo, hi_edge_rows = !ph.halo_yhi || ph.seam_yhi;
            const bool lo = jj == -1 && lo_edge_rows, hi = jj + 1 == g.ny && hi_edge_rows;
            return lo ? seam_rec : (hi ? edge_rec : true);
        };
        auto rec_above = [&](int jj) {
            const bool lo_edge_rows = !ph.halo_ylo || ph.seam_ylo, hi_edge_rows = !ph.halo_yhi || ph.seam_yhi;
            const bool lo = jj == -1 && lo_edge_rows, hi = jj + 1 == g.ny && hi_edge_rows;
            return lo ? edge_rec : (hi ? seam_rec : true);
        };
        // The FP64 single-case forms take the y-edge flags as slope factors; the
        // FP32-flux forms and the persistent batch kernel (CG) keep the select
        // of whole states, which measured faster for them (FP32 strip form
        // 37.5 against 36.6 ms per 20 steps at 4096^2).
        constexpr bool Y_FACTORS = FP64 && !CG;
        auto fy_below = [&](int jj) { return rec_factor<R>(rec_below(jj)); };
        auto fy_above = [&](int jj) { return rec_factor<R>(rec_above(jj)); };

        // Row window of this lane's column: uc = U(j), un = U(j+1); pc = +y face
        // state of row j; gb = flux of the y-face below row j (face frame).  Each
        // row is loaded once and its y-slope limited once.  The loop starts one
        // row early, where it only forms the face below the first row, so that
        // every y-face flux comes from the same code: a face on the edge of two
        // warps' row ranges is computed by both and must agree bit for bit.
        const bool rows_ok = src.wait_row(jb - 2) && src.wait_row(jb - 1) && src.wait_row(jb);
        V4<R> uc = ldrow(jb - 1), un = ldrow(jb), pc = uc;
        if (MUSCL) {
            V4<R> unused;
            if constexpr (Y_FACTORS) slope_faces(limiter, ldrow(jb - 2), uc, un, fy_below(jb - 1), R(0), pc, unused);
            else slope_faces_half(limiter, ldrow(jb - 2), uc, un, pc, unused);
        }
        src.release(jb - 2);
        const double dt = gld<CG>(&a.st->dt);  // set by the step's set-up, constant during the stage
        Q4<R> gb{R(0), R(0), R(0), R(0)};
        // carry slots: gb (r, mn, mt, E), pc (r, mx, my, E), the x part (4 planes)
        auto put_gb = [&](const Q4<R>& q) {
            if constexpr (CARRY_GB) {
                carry_s[SLOT_GB][tq] = q.r; carry_s[SLOT_GB + 1][tq] = q.mn;
                carry_s[SLOT_GB + 2][tq] = q.mt; carry_s[SLOT_GB + 3][tq] = q.E;
            } else {
                gb = q;
            }
        };
        auto get_gb = [&]() {
            if constexpr (CARRY_GB)
                return Q4<R>{carry_s[SLOT_GB][tq], carry_s[SLOT_GB + 1][tq], carry_s[SLOT_GB + 2][tq],
                             carry_s[SLOT_GB + 3][tq]};
            else return gb;
        };
        auto put_pc = [&](const V4<R>& u) {
            if constexpr (CARRY_PC) {
                carry_s[SLOT_PC][tq] = u.r; carry_s[SLOT_PC + 1][tq] = u.mx;
                carry_s[SLOT_PC + 2][tq] = u.my; carry_s[SLOT_PC + 3][tq] = u.E;
            } else {
                pc = u;
            }
        };
        auto get_pc = [&]() {
            if constexpr (CARRY_PC)
                return V4<R>{carry_s[SLOT_PC][tq], carry_s[SLOT_PC + 1][tq], carry_s[SLOT_PC + 2][tq],
                             carry_s[SLOT_PC + 3][tq]};
            else return pc;
        };
        put_gb(gb);
        if (MUSCL) put_pc(pc);
        for (int j = jb - 1; rows_ok && j < je; ++j) {
            src.refill(j);
            if (!src.wait_row(j + 2)) break;
            // Rows j, j+1 and j+2 of the window.  The FP64 TMA-fed form reads
            // them from the ring at each use instead of holding them through the
            // row: with the carry in shared memory that left it no spills at 80
            // registers, and took the 4096^2 vortex from 2.64 (strip form) to
            // 2.26 ms per step.  The other forms hold them in registers.
            constexpr bool REREAD = FP64 && std::is_same<SRC, TmaSrc>::value;
            const V4<R> un2 = REREAD ? V4<R>{} : ldrow(j + 2);
            auto row_c = [&]() { if constexpr (REREAD) return ldrow(j); else return uc; };
            auto row_n = [&]() { if constexpr (REREAD) return ldrow(j + 1); else return un; };
            auto row_n2 = [&]() { if constexpr (REREAD) return ldrow(j + 2); else return un2; };
            const bool row = j >= jb;  // warp-uniform: the first pass only forms the face below row jb

            // ---- x-face on the left of column i, row j, and the divergence of
            // the faces below, left and right of the cell ----
            // Flux divergence, (F_left - F_right) / dx + (G_below - G_above) / dy
            // per conserved variable: the sum of the four face terms that
            // muscl_flux_system scatters into the cell (crates/cfd_solver/src/lib.rs:
            // 333-337), formed as two differences (exact for the nearly equal
            // fluxes of neighbouring faces) and one multiply-add, a few ulps from
            // the reference's sequential sum.  Only the x part stays live through
            // the y-face flux below.
            double part_r[4];
            auto put_part = [&](int v, double x) {
                if constexpr (CARRY_PART) carry_s[SLOT_PART + v][tq] = x;
                else part_r[v] = x;
            };
            auto get_part = [&](int v) {
                if constexpr (CARRY_PART) return carry_s[SLOT_PART + v][tq];
                else return part_r[v];
            };
            auto x_face = [&]() {
                V4<R> ul = shfl_up_v(row_c(), 1), ur = shfl_down_v(row_c(), 1);
                V4<R> ull = ul;  // column i-2 (lane 0 only)
                if (lane == 0) {
                    ul = toR<R>(ld(i0 - 1, j));
                    if (MUSCL) ull = toR<R>(ld(i0 - 2, j));
                }
                if (MUSCL && lane == 31) ur = toR<R>(ld(min(i0 + 32, g.nx + NG - 1), j));
                Q4<R> fx;
                if (MUSCL) {
                    V4<R> pp, mm;  // this column's +x and -x face states
                    if constexpr (FP64) slope_faces(limiter, ul, row_c(), ur, R(0.5), R(0.5), pp, mm);
                    else slope_faces_half(limiter, ul, row_c(), ur, pp, mm);
                    V4<R> lp = shfl_up_v(pp, 1);  // +x state of column i-1
                    if (lane == 0) {
                        V4<R> unused;
                        if constexpr (FP64) slope_faces(limiter, ull, ul, row_c(), R(0.5), R(0), lp, unused);
                        else slope_faces_half(limiter, ull, ul, row_c(), lp, unused);
                    }
                    fx = face_flux<SCHEME, R>(xq(rec_l ? lp : ul), xq(rec_r ? mm : row_c()), rg, rgm1);
                } else {
                    fx = face_flux<SCHEME, R>(xq(ul), xq(row_c()), rg, rgm1);
                }
                const Q4<R> fxr = shfl_down_q(fx, 1);  // face on the right of column i
                const double fl[4] = {(double)fx.r, (double)fx.mn, (double)fx.mt, (double)fx.E};
                const double fr[4] = {(double)fxr.r, (double)fxr.mn, (double)fxr.mt, (double)fxr.E};
#pragma unroll
                for (int v = 0; v < 4; ++v) put_part(v, (fl[v] - fr[v]) * g.inv_x);
            };
            Q4<R> gt;
            V4<R> pn = row_n();  // +y face state of row j+1
            if (XFIRST && row) x_face();
            // ---- y-face above row j ----
            if (MUSCL) {
                V4<R> mn;
                const V4<R> pcr = get_pc();
                if constexpr (Y_FACTORS) slope_faces(limiter, row_c(), row_n(), row_n2(), fy_below(j + 1), fy_above(j), pn, mn);
                else slope_faces_half(limiter, row_c(), row_n(), row_n2(), pn, mn);
                put_pc(pn);
                if constexpr (Y_FACTORS) {
                    gt = face_flux<SCHEME, R>(yq(pcr), yq(mn), rg, rgm1);
                } else {
                    const bool rb = rec_below(j), rt = rec_above(j);
                    gt = face_flux<SCHEME, R>(yq(rb ? pcr : row_c()), yq(rt ? mn : row_n()), rg, rgm1);
                }
            } else {
                gt = face_flux<SCHEME, R>(yq(row_c()), yq(row_n()), rg, rgm1);
            }
            if (!XFIRST && row) x_face();

            if (row && owner) {
                const long long o = cidx(g, i, j);
                // the cell's state in FP64 (the FP32 path reads it again)
                const U4 ucd = FP64 ? toU4(row_c()) : ld(i, j);
                const double gtv[4] = {(double)gt.r, (double)gt.mt, (double)gt.mn, (double)gt.E};
                const Q4<R> gbq = get_gb();
                const double gbd[4] = {(double)gbq.r, (double)gbq.mt, (double)gbq.mn, (double)gbq.E};
                double rhs[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) rhs[v] = fma(gbd[v] - gtv[v], g.inv_y, get_part(v));
                if constexpr (CORR) {
                    // learned corrections of the four faces (periodic grid): the
                    // x face on the left of a cell, the y face below it
                    const long long n = (long long)g.nx * g.ny, c = (long long)j * g.nx + i;
                    const long long cr = (long long)j * g.nx + (i + 1 == g.nx ? 0 : i + 1);
                    const long long ct = (long long)(j + 1 == g.ny ? 0 : j + 1) * g.nx + i;
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        const float* cx = a.corr + v * n;
                        const float* cy = a.corr + (4 + v) * n;
                        rhs[v] += ((double)cx[c] - (double)cx[cr]) * g.inv_x + ((double)cy[c] - (double)cy[ct]) * g.inv_y;
                    }
                }
                // the TMA-fed form runs only cases without bodies, a body force or
                // a sponge: those paths are not compiled into it
                constexpr bool LEAN = std::is_same<SRC, TmaSrc>::value;
                const bool ibm = !LEAN && a.mask != nullptr;
                const bool solid = ibm && a.mask[o];
                if (VISC && !solid) {
                    // viscous_system, crates/cfd_solver/src/lib.rs:514-557 (z terms vanish in 2-D).
                    // Neighbours +x, -x, +y, -y; a solid one takes (0, 0, T of the cell).  The
                    // densities come first: the five reciprocals from one reciprocal of their
                    // product (running products forward, then peeled off backward).  The other
                    // components are loaded one axis pair at a time, which keeps the live
                    // state small.
                    const long long no[4] = {o + 1, o - 1, o + g.pitch, o - g.pitch};
                    bool sn[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) sn[k] = ibm && a.mask[no[k]];
                    const double r0 = ucd.r, r1 = sn[0] ? 1.0 : gld<CG>(uin + no[0]),
                                 r2 = sn[1] ? 1.0 : gld<CG>(uin + no[1]);
                    const double r3 = sn[2] ? 1.0 : (FP64 ? (double)row_n().r : gld<CG>(uin + no[2]));
                    const double r4 = sn[3] ? 1.0 : gld<CG>(uin + no[3]);
                    const double p1 = r0 * r1, p2 = p1 * r2, p3 = p2 * r3;
                    double w = rcp_(p3 * r4);
                    const double i4 = p3 * w;
                    w = w * r4;
                    const double i3 = p2 * w;
                    w = w * r3;
                    const double i2 = p1 * w;
                    w = w * r2;
                    const double ninv[4] = {r0 * w, i2, i3, i4};
                    const double rn[4] = {r1, r2, r3, r4};
                    const double i0 = r1 * w;
                    double us, vs, ts;
                    prim_uvt(ucd, i0, gm1, ph.inv_r_gas, us, vs, ts);
                    auto nb = [&](int k, double& vu, double& vv, double& t) {
                        if (sn[k]) {
                            vu = 0.0; vv = 0.0; t = ts;
                            return;
                        }
                        U4 q;
                        if (FP64 && k == 2) {
                            q = toU4(row_n());
                        } else {
                            q.r = rn[k];
                            q.mx = gld<CG>(uin + P + no[k]);
                            q.my = gld<CG>(uin + 2 * P + no[k]);
                            q.E = gld<CG>(uin + 3 * P + no[k]);
                        }
                        prim_uvt(q, ninv[k], gm1, ph.inv_r_gas, vu, vv, t);
                    };
                    const double y_im = a.yw[j], y_ip = a.yw[g.ny + j], y_is = a.yw[2 * g.ny + j];
                    const double dxi2 = ph.dx_inv2;
                    auto d2x = [&](double m, double p, double c) { return (p - 2.0 * c + m) * dxi2; };
                    auto d2y = [&](double m, double p, double c) { return ((p - c) * y_ip - (c - m) * y_im) * y_is; };
                    double lu, lv, lt;  // d2x + d2y of u, v, T
                    {
                        double pu, pv, pt, mu_, mv, mt;
                        nb(0, pu, pv, pt);
                        nb(1, mu_, mv, mt);
                        lu = d2x(mu_, pu, us);
                        lv = d2x(mv, pv, vs);
                        lt = d2x(mt, pt, ts);
                    }
                    {
                        double pu, pv, pt, mu_, mv, mt;
                        nb(2, pu, pv, pt);
                        nb(3, mu_, mv, mt);
                        lu = lu + d2y(mu_, pu, us);
                        lv = lv + d2y(mv, pv, vs);
                        lt = lt + d2y(mt, pt, ts);
                    }
                    const double mu = viscosity(ph, ts);
                    const double kappa = mu * ph.cp_pr;  // thermal_conductivity mu cp / Pr, crates/cfd_eos/src/lib.rs:83-87
                    const double fxv = mu * lu;
                    const double fyv = mu * lv;
                    rhs[1] += fxv;
                    rhs[2] += fyv;
                    rhs[3] += us * fxv + vs * fyv + kappa * lt;
                }
                if (solid) rhs[0] = rhs[1] = rhs[2] = rhs[3] = 0.0;  // zero_solid_rhs, crates/cfd_ibm/src/lib.rs:293-301
                if (!LEAN && ph.body_force_x != 0.0) {  // crates/cfd_solver/tests/poiseuille_channel_validation.rs:100-118
                    rhs[1] += ucd.r * ph.body_force_x;
                    rhs[3] += ph.body_force_x * ucd.mx;
                }

                // Rk3Integrator / EulerIntegrator::substep, crates/cfd_solver/src/integrate.rs:48-101,
                // with multiply-adds: u + dt r, then w0 u0 + w1 (u + dt r)
                const double ucv[4] = {ucd.r, ucd.mx, ucd.my, ucd.E};
                double un_[4];
                if (a.stage == 1 || a.stage == 2) {
                    const double w0 = a.stage == 1 ? 0.75 : (1.0 / 3.0);
                    const double w1 = a.stage == 1 ? 0.25 : (2.0 / 3.0);
#pragma unroll
                    for (int v = 0; v < 4; ++v) un_[v] = fma(w1, fma(rhs[v], dt, ucv[v]), w0 * src.u0v(v, o, i, j));
                } else {
#pragma unroll
                    for (int v = 0; v < 4; ++v) un_[v] = fma(rhs[v], dt, ucv[v]);
                }
                U4 nw{un_[0], un_[1], un_[2], un_[3]};

                if (!LEAN && a.completes_step && ph.sponge) {
                    // outlet_sponge_system, examples/cylinder_drag_validation/main.rs:186-229
                    const double cx = centre(g.lo[0], g.h[0], i);
                    if (cx >= ph.sponge_x_start) {
                        const double cy = centre(g.lo[1], g.h[1], j + g.j_off);
                        const double s = fmin(fmax((cx - ph.sponge_x_start) * ph.sponge_inv_w, 0.0), 1.0);
                        const double f = fmin(ph.sponge_sigma * s * s * dt, 1.0);
                        const double hh = ph.sponge_height;
                        const double uy = 4.0 * ph.sponge_u_max * cy * (hh - cy) / (hh * hh);
                        // prim_to_cons(rho, uy, 0, p) with p / (gamma - 1) formed on the host
                        const double rho_s = ph.sponge_rho;
                        const double ke = mul_(mul_(0.5, rho_s), add_(mul_(uy, uy), mul_(0.0, 0.0)));
                        const U4 tg{rho_s, mul_(rho_s, uy), mul_(rho_s, 0.0), add_(ph.sponge_e0, ke)};
                        nw.r += f * (tg.r - nw.r);
                        nw.mx += f * (tg.mx - nw.mx);
                        nw.my += f * (tg.my - nw.my);
                        nw.E += f * (tg.E - nw.E);
                    }
                }

                store4(a.uout, P, o, nw);
                write_ghosts<PXY>(g, ph, a.uout, i, j, nw);
                peer_rows(a, g, i, j, nw);

                // non-physical state flag (rho<=0, p<=0, NaN)
                // p > 0 with rho > 0 is 2 E rho > m^2 (no division)
                // (a NaN in any component fails one of the two tests, so the NaN
                // bit is only looked at once a test has failed)
                int bad = 0;
                if (!(nw.r > 0.0)) bad |= 1;
                if (!(2.0 * nw.E * nw.r > nw.mx * nw.mx + nw.my * nw.my)) bad |= 2;
                if (bad) {
                    if (nw.r != nw.r || nw.mx != nw.mx || nw.my != nw.my || nw.E != nw.E) bad |= 4;
                    atomicOr(&a.st->nonphysical, bad);
                }

                if (a.completes_step && a.want_cfl) lam = fmax(lam, wave_speed(g, ph, nw));
            }
            src.release(j);
            put_gb(gt);
            uc = un;
            un = un2;
        }
    }
    // wave-speed max for the next step's CFL dt: one atomic per warp
    if (a.completes_step && a.want_cfl) {
        for (int o = 16; o > 0; o >>= 1) lam = fmax(lam, __shfl_xor_sync(0xffffffffu, lam, o));
        if (lane == 0 && lam > 0.0 && lam == lam)
            atomicMax(CG ? lam_slot_v(a.st) : lam_slot(a.st), (unsigned long long)__double_as_longlong(lam));
    }
}

// The strip code reading its rows from global memory.
template <int SCHEME, int RECON, class R, bool VISC, class A, bool CORR = false, bool XFIRST = true, bool CG = false,
          int LIM = -1>
__device__ __forceinline__ void stage_strip(const A& a, int rows, int strip, int by) {
    GlobalSrc<CG> src{a.uin, a.u0};
    stage_strip_src<SCHEME, RECON, R, VISC, A, CORR, XFIRST, CG, GlobalSrc<CG>, LIM>(a, rows, strip, by, src);
}

template <int SCHEME, int RECON, class R, int MINB, bool VISC, bool CORR = false, bool XFIRST = true, int LIM = -1>
__global__ void __launch_bounds__(32 * WPB, MINB) stage_kernel(StageArgs a, int rows) {
    pdl_wait_then_release();
    stage_strip<SCHEME, RECON, R, VISC, StageArgs, CORR, XFIRST, false, LIM>(a, rows, blockIdx.x * WPB + (threadIdx.x >> 5),
                                                                            blockIdx.y);
}

// The same stage with its rows fed by TMA (2-D meshes without viscous terms,
// immersed bodies or the learned correction).  A block's four warps march the
// same rows of four adjacent strips (124 columns); each row of the stage input
// with two halo columns on each side, and the block's row of U^n, reach the
// shared-memory ring (efvm_tma.cuh) one iteration before they are read, so the
// strip code's halo cells and U^n no longer wait on L2 and its rows come from
// shared memory.  The arithmetic is the strip code's.
template <int SCHEME, int RECON, class R, int MINB, bool XFIRST, int LIM, bool PXY>
__global__ void __launch_bounds__(32 * WPB, MINB)
    stage_tma_kernel(StageArgs a, int rows, const __grid_constant__ CUtensorMap map_in,
                     const __grid_constant__ CUtensorMap map_u0) {
    extern __shared__ __align__(128) unsigned char smem[];
    pdl_wait_then_release();
    if (!a.st->active) return;  // the whole grid, before any barrier
    const int strips = (a.g.nx + STRIP - 1) / STRIP;
    const int n_active = min(WPB, strips - (int)blockIdx.x * WPB);  // warps with columns
    const int jb = blockIdx.y * rows, je = min(jb + rows, a.g.ny);
    const bool with_u0 = a.stage == 1 || a.stage == 2;
    const int i0b = blockIdx.x * WPB * STRIP;
    TmaSrc src;
    src.ring = reinterpret_cast<double*>(smem);
    src.full = reinterpret_cast<uint64_t*>(smem + tma::RING * tma::SLOT_BYTES);
    src.empty = src.full + tma::RING;
    src.map_in = &map_in;
    src.map_u0 = with_u0 ? &map_u0 : nullptr;
    src.u0 = a.u0;
    src.plane = a.g.plane;
    src.st = a.st;
    src.first = jb - 2;
    src.last = je + 1;
    src.u0_lo = jb;
    src.u0_hi = je;
    src.x_in = XO + i0b - 2;  // even: a 16-byte boundary
    src.x_u0 = XO + i0b;
    src.col0 = i0b - 2;
    src.scol = 0;
    src.issued = src.first - 1;
    src.producer = threadIdx.x == 0;
    src.wait_ns = a.wait_ns;
    src.stall = a.stall && blockIdx.x == 0 && blockIdx.y == 0;
    src.ok = true;
    if (threadIdx.x == 0) {
        tma::prefetch_map(&map_in);
        if (with_u0) tma::prefetch_map(&map_u0);
        for (int s = 0; s < tma::RING; ++s) {
            tma::bar_init(&src.full[s], 1);
            tma::bar_init(&src.empty[s], (uint32_t)n_active);
        }
        tma::fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int r = src.first; r < src.first + tma::RING && r <= src.last; ++r) src.issue(r);
    const int warp = threadIdx.x >> 5;
    if (warp < n_active)
        stage_strip_src<SCHEME, RECON, R, false, StageArgs, false, XFIRST, false, TmaSrc, LIM, PXY>(a, rows, blockIdx.x * WPB + warp,
                                                                                  blockIdx.y, src);
    if (threadIdx.x == 0 && !src.ok) src.drain();
}

// The stage arguments of one batch case, with its geometry and physics in the
// case table in global memory.
struct BatchView {
    const Geometry& g;
    const Physics& ph;
    const double* __restrict__ uin;
    const double* u0;
    double* uout;
    const uint8_t* __restrict__ mask;
    const double* __restrict__ yw;
    DevState* st;
    int stage, completes_step, want_cfl;
    const float* corr;
    int defer_forces;  // batches have no IBM: always 0
};

// The same stage over a batch of independent cases, one warp per tile: warp w
// of block b runs tiles[b * WPB + w] = (case, strip, row block) of that case,
// with the case's geometry, boundary conditions, buffers and clock.  Warps are
// the unit so that small cases waste no lanes of a block.
template <int SCHEME, int RECON, class R, int MINB, bool VISC, bool XFIRST>
__global__ void __launch_bounds__(32 * WPB, MINB) batch_stage_kernel(BatchStageArgs b, int n_tiles) {
    pdl_wait_then_release();
    const int tile = blockIdx.x * WPB + (threadIdx.x >> 5);
    if (tile >= n_tiles) return;  // uniform per warp; the kernel has no block barrier
    const int4 t = b.tiles[tile];
    const BatchCase& c = b.cases[t.x];
    // the case's geometry and physics are read in place from the case table
    const BatchView v{c.g, c.ph, c.U[b.in_buf], c.U[0], c.U[b.out_buf], nullptr, c.yw, c.st,
                      b.stage, b.completes_step, b.want_cfl, nullptr};
    stage_strip<SCHEME, RECON, R, VISC, BatchView, false, XFIRST>(v, c.rows, t.y, t.z);
}


// ---------------------------------------------------------------------------
// CFL wave-speed max over the interior of one state (standalone pass)
// ---------------------------------------------------------------------------
__global__ void cfl_kernel(Geometry g, Physics ph, const double* __restrict__ q, DevState* st) {
    double lam = 0.0;
    const long long n = (long long)g.nx * g.ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t / g.nx), i = (int)(t - (long long)j * g.nx);
        const U4 u = load4(q, g.plane, cidx(g, i, j));
        lam = fmax(lam, wave_speed(g, ph, u));
    }
    block_max_atomic(lam, lam_slot(st));
}

__global__ void reset_lam_kernel(DevState* st) {
    *lam_slot(st) = 0ull;
}

// Per-step Setup: dt from the wave-speed max (cfl_system's final lines,
// crates/cfd_solver/src/lib.rs:671-676) or fixed_dt, and the stop test of the
// case drivers' `if t >= T_FINAL break`.
// The stop rule of step_setup: a non-physical state or t >= t_stop ends the run.
template <class S>
__device__ __forceinline__ bool step_stops(S* st) {
    return st->nonphysical || (st->stop_at_t && st->time >= st->t_stop);
}

// Per-step set-up (one thread): stop check, dt = cfl / max wave speed (cfl_system,
// crates/cfd_solver/src/lib.rs:647-669) and the switch of the wave-speed buffer
// that the step's last stage accumulates into.
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// S = DevState, or volatile DevState where other blocks of the same launch
// write the state (the persistent batch kernel).
template <class S>
__device__ __forceinline__ void step_setup(const Physics& ph, S* st) {
    if (step_stops(st)) {
        st->active = 0;
        st->done_ns = global_ns();
        return;
    }
    double dt;
    if (ph.fixed_dt > 0.0) {
        dt = ph.fixed_dt;
    } else {
        const unsigned long long bits = st->ext_lam ? st->lam_ext : st->lam[st->lam_idx];
        const double lam = __longlong_as_double((long long)bits);
        dt = lam > 0.0 ? ph.cfl / lam : INFINITY;
    }
    st->dt = dt;
    st->step_par = (int)(st->step & 1ull);
    if (st->ext_lam) {  // the slot starts this step's accumulation from zero
        st->lam_ext = 0ull;
        return;
    }
    const int nxt = st->lam_idx ^ 1;
    st->lam[nxt] = 0ull;
    st->lam_idx = nxt;
}

__global__ void step_setup_kernel(Physics ph, DevState* st) {
    pdl_wait_then_release();
    if (!st->active) return;
    step_setup(ph, st);
}

__global__ void batch_setup_kernel(Physics ph, const BatchCase* cases, int n) {
    pdl_wait_then_release();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    DevState* st = cases[k].st;
    if (st->active) step_setup(ph, st);
}

__global__ void clock_kernel(unsigned long long* out) { *out = global_ns(); }


// ---- the persistent batch kernel -------------------------------------------
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Spin (one lane) until *flag >= target.  Bounded: the device global timer
// limits the wait to limit_ns, and a wait that sees another warp's give-up in
// *status stops too.  Returns false when it gave up.
__device__ __forceinline__ bool wait_at_least(const unsigned* flag, unsigned target, unsigned long long limit_ns,
                                              int* status) {
    if (ld_acquire_u32(flag) >= target) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned n = 1;; ++n) {
        __nanosleep(64);
        if (ld_acquire_u32(flag) >= target) return true;
        if ((n & 15u) == 0u) {
            if (*(volatile int*)status) return false;
            if (global_ns() - t0 > limit_ns || n > (1u << 30)) {
                atomicOr(status, 1);
                return false;
            }
        }
    }
}

// Every warp runs tiles of the table in ticket order until the launch's stages
// are used up (PersistArgs).  Tickets are taken only by running warps and a
// tile waits only for tiles of lower tickets (its case's previous stage), so
// the waits end whatever the number of resident blocks; the kernel has no block
// barrier.  The stage inputs were written earlier in the same launch by other
// blocks, so they are loaded through L2 (stage_strip with CG).
template <int SCHEME, int RECON, class R, int MINB, bool VISC, bool XFIRST>
__global__ void __launch_bounds__(32 * WPB, MINB) batch_persistent_kernel(PersistArgs p) {
    const int lane = threadIdx.x & 31;
    const unsigned long long total = (unsigned long long)p.rounds * (unsigned long long)p.n_tiles;
    for (;;) {
        unsigned long long t = total;
        if (lane == 0 && !*(volatile int*)p.status) t = atomicAdd(p.ticket, 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= total) return;
        const int r = (int)(t / (unsigned long long)p.n_tiles);
        const int4 tile = p.tiles[t - (unsigned long long)r * (unsigned long long)p.n_tiles];
        const int k = tile.x;
        if (r > 0) {
            int ok = 1;
            if (lane == 0) ok = wait_at_least(p.ready + k, (unsigned)r, p.wait_ns, p.status);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) return;
            (void)ld_acquire_u32(p.ready + k);  // each lane orders its own loads after the publication
        }
        const BatchCase& c = p.cases[k];
        const int stage = r % 3;
        const BatchView v{c.g, c.ph, c.U[stage], c.U[0], c.U[stage == 2 ? 0 : stage + 1], nullptr, c.yw, c.st,
                          stage, stage == 2, stage == 2 && p.want_cfl, nullptr, 0};
        stage_strip<SCHEME, RECON, R, VISC, BatchView, false, XFIRST, true>(v, c.rows, tile.y, tile.z);
        __threadfence();  // this lane's results before the count below
        __syncwarp();
        int last = 0;
        if (lane == 0) last = atomicAdd(p.done + k, 1u) + 1u == (unsigned)(r + 1) * (unsigned)p.case_tiles[k];
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last && lane == 0) {
            __threadfence();
            unsigned next = (unsigned)(r + 1);
            // the case's next step: its set-up, or its end (the set-up of the step
            // after the launch's last stage is the next launch's first work)
            if (stage == 2 && r + 1 < p.rounds) {
                volatile DevState* st = c.st;
                if (st->active) step_setup(c.ph, st);
                if (!st->active) next = ~0u;
                __threadfence();
            }
            atomicMax(p.ready + k, next);
        }
    }
}

// ---------------------------------------------------------------------------
// Halo + Boundary for a whole state (after upload / geometry changes)
// ---------------------------------------------------------------------------
__global__ void fill_ghosts_y_kernel(Geometry g, Physics ph, double* q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nx) return;
    const long long P = g.plane;
    const double gm1 = ph.gamma - 1.0;
    if (ph.periodic_y) {
        for (int k = 0; k < NG; ++k) {
            store4(q, P, cidx(g, i, -NG + k), load4(q, P, cidx(g, i, g.ny - NG + k)));
            store4(q, P, cidx(g, i, g.ny + k), load4(q, P, cidx(g, i, k)));
        }
    } else {
        if (!ph.halo_ylo) store4(q, P, cidx(g, i, -1), bc_ghost(ph.bc[2], 2, load4(q, P, cidx(g, i, 0)), gm1));
        if (!ph.halo_yhi)
            store4(q, P, cidx(g, i, g.ny), bc_ghost(ph.bc[3], 3, load4(q, P, cidx(g, i, g.ny - 1)), gm1));
    }
}
__global__ void fill_ghosts_x_kernel(Geometry g, Physics ph, double* q) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= g.ny) return;
    const long long P = g.plane;
    const double gm1 = ph.gamma - 1.0;
    if (ph.periodic_x) {
        for (int k = 0; k < NG; ++k) {
            store4(q, P, cidx(g, -NG + k, j), load4(q, P, cidx(g, g.nx - NG + k, j)));
            store4(q, P, cidx(g, g.nx + k, j), load4(q, P, cidx(g, k, j)));
        }
    } else {
        const U4 u0 = load4(q, P, cidx(g, 0, j));
        store4(q, P, cidx(g, -1, j), bc_ghost(ph.bc[0], 0, u0, gm1));
        if (ph.parabolic_inflow) {
            const double y = centre(g.lo[1], g.h[1], j + g.j_off);
            const double um = ph.inflow_u_max, hh = ph.inflow_height, rho = ph.inflow_rho;
            const double uy = mul_(mul_(mul_(4.0, um), y), sub_(hh, y)) / mul_(hh, hh);
            const U4 c = prim_to_cons(rho, uy, 0.0, pressure_d(u0, gm1), gm1);
            store4(q, P, cidx(g, -1, j), c);
            store4(q, P, cidx(g, -2, j), c);
        }
        store4(q, P, cidx(g, g.nx, j), bc_ghost(ph.bc[1], 1, load4(q, P, cidx(g, g.nx - 1, j)), gm1));
    }
}

// ---------------------------------------------------------------------------
// IBM
// ---------------------------------------------------------------------------

// refresh_cylinder_mask, crates/cfd_ibm/src/lib.rs:155-183 (static bodies: the
// flip happens on the first call only).
__global__ void geometry_kernel(Geometry g, const double* __restrict__ cyl, int ncyl, U4 stagnant, U4 ambient,
                                double* q, uint8_t* mask) {
    const long long n = (long long)g.nx * g.ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t / g.nx), i = (int)(t - (long long)j * g.nx);
        const double cx = centre(g.lo[0], g.h[0], i), cy = centre(g.lo[1], g.h[1], j + g.j_off);
        bool inside = false;
        for (int b = 0; b < ncyl && !inside; ++b) {
            const double dx = __dsub_rn(cx, cyl[3 * b]), dy = __dsub_rn(cy, cyl[3 * b + 1]);
            const double sd = __dsub_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy))), cyl[3 * b + 2]);
            inside = sd < 0.0;
        }
        const long long o = cidx(g, i, j);
        const bool was = mask[o] != 0;
        if (inside && !was) {
            mask[o] = 1;
            store4(q, g.plane, o, stagnant);
        } else if (!inside && was) {
            mask[o] = 0;
            store4(q, g.plane, o, ambient);
        }
    }
}

// sample_trilinear restricted to the z = centre plane (the z weight is exactly
// 1 on the cell layer and 0 on the ghost layers), crates/cfd_ibm/src/lib.rs:106-149.
// Solid corners (clear FLUID_CORNER bits) are skipped.  The four corner states
// are loaded before any of them is used so that the loads overlap.
__device__ __forceinline__ bool sample_bilinear(const Geometry& g, const Physics& ph, const double* q,
                                                unsigned fluid, int lo_i, int lo_j, double tx, double ty,
                                                double out[5]) {
    const double gm1 = ph.gamma - 1.0;
    U4 cu[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) cu[k] = load4(q, g.plane, cidx(g, lo_i + (k >> 1), lo_j + (k & 1)));
    double acc[5] = {0, 0, 0, 0, 0};  // rho, u, v, p, t
    double total = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {  // (di, dj) = (0,0), (0,1), (1,0), (1,1)
        const double wx = (k >> 1) == 0 ? 1.0 - tx : tx;
        const double wy = (k & 1) == 0 ? 1.0 - ty : ty;
        const U4 u = cu[k];
        if (!((fluid >> (FLUID_CORNER_SHIFT + k)) & 1u)) continue;
        if (!isfinite(u.r) || u.r <= 0.0) continue;
        const double w = wx * wy;
        const double inv = 1.0 / u.r;
        const double vu = u.mx * inv, vv = u.my * inv;
        const double ke = 0.5 * u.r * (vu * vu + vv * vv);
        const double p = gm1 * (u.E - ke);
        const double t = p * inv * ph.inv_r_gas;
        acc[0] += w * u.r;
        acc[1] += w * vu;
        acc[2] += w * vv;
        acc[3] += w * p;
        acc[4] += w * t;
        total += w;
    }
    if (total < 1e-12) return false;
    const double inv = 1.0 / total;
    for (int k = 0; k < 5; ++k) out[k] = acc[k] * inv;
    return true;
}

// Mirror (apply_ibm_ghost_bc, crates/cfd_ibm/src/lib.rs:258-289) of every solid
// ghost cell, recording its pre-mirror value for the emulated z-ghost of the
// staircase wall force.  One thread per ghost cell.
__device__ __forceinline__ void mirror_ghost(const Geometry& g, const Physics& ph, const Ibm& ib, double* q,
                                             int stage, int k, int par) {
    const IbmGhostDev gh = ib.ghosts[k];
    const long long o = cidx(g, gh.i, gh.j);
    const U4 pre = load4(q, g.plane, o);
    double img[5];
    const bool ok = gh.valid && (gh.fluid & GHOST_MIRROR_BIT) &&
                    sample_bilinear(g, ph, q, gh.fluid, gh.lo_i, gh.lo_j, gh.tx, gh.ty, img);
    double* zf = ib.zfill + ((long long)stage % 3) * ib.n_ghost * 4 + 4LL * k;
    zf[0] = pre.r; zf[1] = pre.mx; zf[2] = pre.my; zf[3] = pre.E;
    if (stage == 0 || stage == 3) {
        double* z0 = ib.zg0 + 4LL * ((long long)par * ib.n_ghost + k);
        z0[0] = pre.r; z0[1] = pre.mx; z0[2] = pre.my; z0[3] = pre.E;
    }
    if (!ok || !(gh.fluid & GHOST_MIRROR_BIT)) return;
    // u_ghost = 2 u_wall - u_image; rho, p, T from the image
    const U4 m = prim_to_cons(img[0], 2.0 * gh.uw[0] - img[1], 2.0 * gh.uw[1] - img[2], img[3], ph.gamma - 1.0);
    store4(q, g.plane, o, m);
}

// Output phase: MarkerForce (compute_marker_loadings, crates/cfd_ibm/src/
// lib.rs:442-480) in block 0 and WallForce (compute_wall_forces, :309-362) over
// blocks 1..: each block reduces its share in a fixed order (warp shuffle
// trees, then the warps in order) and writes 6 partial sums; the last block to
// finish adds the wall partials in a fixed order (deterministic), publishes
// both forces and appends the marker force to the substage history.
__device__ __forceinline__ void forces_block(const Geometry& g, const Physics& ph, const Ibm& ib,
                                             const double* __restrict__ q, DevState* st, int stage, int blk,
                                             int nblk, int deferred) {
    __shared__ double red[IBM_THREADS / 32][6];
    __shared__ bool last;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double gm1 = ph.gamma - 1.0;
    double f[6] = {0, 0, 0, 0, 0, 0};
    if (blk == 0) {
        const double inv_off = 1.0 / ib.sample_offset;  // traction = mu * u_t / offset
        for (int m = tid; m < ib.n_markers; m += blockDim.x) {
            const MarkerDev mk = ib.markers[m];
            if (!mk.valid) continue;
            double img[5];
            if (!sample_bilinear(g, ph, q, mk.fluid, mk.lo_i, mk.lo_j, mk.tx, mk.ty, img)) continue;
            if (!(isfinite(img[3]) && isfinite(img[4]) && isfinite(img[1]) && isfinite(img[2]))) continue;
            const double usd[3] = {img[1] - mk.wall_velocity[0], img[2] - mk.wall_velocity[1], 0.0 - mk.wall_velocity[2]};
            const double udotn = usd[0] * mk.normal[0] + usd[1] * mk.normal[1] + usd[2] * mk.normal[2];
            const double mu = viscosity(ph, img[4]);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double ut = usd[d] - udotn * mk.normal[d];
                f[d] += -img[3] * mk.normal[d] * mk.area;
                f[3 + d] += mu * ut * inv_off * mk.area;
            }
        }
    } else {
        const int k = (blk - 1) * blockDim.x + tid;
        if (k < ib.n_ghost) {
            const IbmGhostDev gh = ib.ghosts[k];
            const int i = gh.i, j = gh.j;
            const double dx = g.h[0], dy = g.h[1], dz = g.h[2];
            const double face_area[3] = {dy * dz, dx * dz, dx * dy};
            const double* zf = ib.zfill + ((long long)stage % 3) * ib.n_ghost * 4 + 4LL * k;
            // the step's saved z-ghost state.  Stage 3's forces run after its stage
            // kernel has counted the step, and the step counter is stable while they
            // run (the next step's first launch, or the substep call).  The forces of
            // stages 1 and 2 may run on a side branch while the next stage kernel
            // counts the step, so they take the parity that the step's set-up recorded.
            const int par = stage == 2 ? (int)((st->step - 1ull) & 1ull) : st->step_par;
            const double* z0 = ib.zg0 + 4LL * ((long long)par * ib.n_ghost + k);
            // all neighbour states first (in bounds: the ring of boundary ghosts)
            U4 nbu[6];
            nbu[0] = load4(q, g.plane, cidx(g, i + 1, j));
            nbu[1] = load4(q, g.plane, cidx(g, i - 1, j));
            nbu[2] = load4(q, g.plane, cidx(g, i, j + 1));
            nbu[3] = load4(q, g.plane, cidx(g, i, j - 1));
            {
                // the two z-ghost layers of the 2-D mesh (never solid; their state is
                // the slip-wall copy of this cell, RK-advanced with a zero rhs)
                double zv[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    if (stage == 1) zv[c] = 0.75 * z0[c] + 0.25 * (zf[c] + 0.0);
                    else if (stage == 2) zv[c] = (1.0 / 3.0) * z0[c] + (2.0 / 3.0) * (zf[c] + 0.0);
                    else zv[c] = zf[c] + 0.0;
                }
                nbu[4] = nbu[5] = U4{zv[0], zv[1], zv[2], zv[3]};
            }
            // the six face neighbours of compute_wall_forces: +x, -x, +y, -y, +z, -z
#pragma unroll
            for (int nb = 0; nb < 6; ++nb) {
                if (nb < 4 && !((gh.fluid >> (FLUID_NB_SHIFT + nb)) & 1u)) continue;
                const U4 u = nbu[nb];
                const int dim = nb >> 1;
                const double sign = (nb & 1) ? -1.0 : 1.0;
                // one division per neighbour (1/rho); p, T and the wall-distance
                // quotient u / (dn / 2) as products, a few ulps from the
                // reference's divisions
                const double inv = 1.0 / u.r;
                const double vel0 = u.mx * inv, vel1 = u.my * inv;
                const double ke = 0.5 * u.r * (vel0 * vel0 + vel1 * vel1);
                const double p = gm1 * (u.E - ke);
                f[dim] -= p * sign * face_area[dim];
                const double t = p * inv * ph.inv_r_gas;
                const double mu = viscosity(ph, t);
                const double vel[3] = {vel0, vel1, 0.0};
                const double inv_half_dn = 2.0 * g.inv_h[dim];
#pragma unroll
                for (int td = 0; td < 3; ++td)
                    if (td != dim) f[3 + td] += mu * vel[td] * inv_half_dn * face_area[dim];
            }
        }
    }
#pragma unroll
    for (int d = 0; d < 6; ++d)
        for (int o = 16; o > 0; o >>= 1) f[d] += __shfl_down_sync(0xffffffffu, f[d], o);
    if (lane == 0)
#pragma unroll
        for (int d = 0; d < 6; ++d) red[warp][d] = f[d];
    __syncthreads();
    if (tid == 0) {
        double* part = ib.partials + 6LL * blk;
#pragma unroll
        for (int d = 0; d < 6; ++d) {
            double v = red[0][d];
            for (int w = 1; w < IBM_THREADS / 32; ++w) v += red[w][d];
            part[d] = v;
        }
        __threadfence();
        const unsigned int done = atomicAdd(ib.counter, 1u);
        last = done == (unsigned)nblk - 1;
    }
    __syncthreads();
    if (last && warp == 0) {
        __threadfence();
        const volatile double* part = ib.partials;
        double wall[6] = {0, 0, 0, 0, 0, 0};
        for (int b = 1 + lane; b < nblk; b += 32)
#pragma unroll
            for (int d = 0; d < 6; ++d) wall[d] += part[6 * b + d];
#pragma unroll
        for (int d = 0; d < 6; ++d)
            for (int o = 16; o > 0; o >>= 1) wall[d] += __shfl_down_sync(0xffffffffu, wall[d], o);
        if (lane == 0) {
            for (int d = 0; d < 6; ++d) {
                ib.force_out[d] = part[d];
                ib.force_out[6 + d] = wall[d];
            }
            if (ib.history && st->hist_pos < st->hist_cap) {
                for (int d = 0; d < 6; ++d) ib.history[6 * st->hist_pos + d] = part[d];
                st->hist_pos += 1;
            }
            *ib.counter = 0u;  // ready for the next launch
            // only the deferred launch clears the flag: the stage that sets it starts
            // while the previous stage's forces may still run on the side branch
            if (deferred) st->forces_pending = 0;
        }
    }
}

// One launch of the IBM work between two stage kernels: `n_force_blocks`
// blocks integrate the marker and wall forces of the state q that stage
// `force_stage` wrote, and the remaining blocks mirror the ghost cells of the
// same q for stage `mirror_stage` (-1: none).  The two parts touch disjoint
// data: the forces read fluid cells and the stage's z-fill, the mirror reads
// fluid cells and writes solid cells and the next stage's z-fill.  With
// `setup`, thread 0 of the first mirror block also does the per-step set-up,
// and every mirror thread applies its stop rule itself, so a step that ends
// there leaves the state untouched.
__global__ void __launch_bounds__(IBM_THREADS) ibm_kernel(Geometry g, Physics ph, Ibm ib, double* q, DevState* st,
                                                          int force_stage, int n_force_blocks, int mirror_stage,
                                                          int setup, int deferred) {
    pdl_wait_then_release();
    const int b = blockIdx.x;
    if (b < n_force_blocks) {  // uniform per block
        // Deferred forces belong to a step that ran; they go ahead whatever this
        // launch's set-up decides, and only while they are pending.  Every block
        // reads the flag before it counts itself in, and only the last one clears it.
        if (deferred ? !st->forces_pending : !st->active) return;
        forces_block(g, ph, ib, q, st, force_stage, b, n_force_blocks, deferred);
        return;
    }
    if (!st->active) return;
    if (setup) {
        if (b == n_force_blocks && threadIdx.x == 0) step_setup(ph, st);
        if (step_stops(st)) return;
    }
    const int k = (b - n_force_blocks) * blockDim.x + threadIdx.x;
    if (mirror_stage >= 0 && k < ib.n_ghost) mirror_ghost(g, ph, ib, q, mirror_stage, k, (int)(st->step & 1ull));
}

// ---------------------------------------------------------------------------
// Utilities
// ---------------------------------------------------------------------------

// Strided AoS (5 doubles per cell: rho, rho_u, rho_v, rho_w, rho_e) <-> SoA.
__global__ void pack_kernel(Geometry g, const double* src, int64_t si, int64_t sj, int64_t sv, double* q,
                            double* dst, int to_device) {
    const long long n = (long long)g.nx * g.ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t / g.nx), i = (int)(t - (long long)j * g.nx);
        const long long h = (long long)i * si + (long long)j * sj;
        const long long o = cidx(g, i, j);
        if (to_device) {
            q[o] = src[h];
            q[g.plane + o] = src[h + sv];
            q[2 * g.plane + o] = src[h + 2 * sv];
            q[3 * g.plane + o] = src[h + 4 * sv];
        } else {
            dst[h] = q[o];
            dst[h + sv] = q[g.plane + o];
            dst[h + 2 * sv] = q[2 * g.plane + o];
            dst[h + 3 * sv] = 0.0;
            dst[h + 4 * sv] = q[3 * g.plane + o];
        }
    }
}

__device__ __forceinline__ double vortex_rho(const efvm_vortex& v, double t, double x, double y, U4* cons) {
    const double PI = 3.141592653589793;
    const double cx = v.cx0 + v.mean_u * t, cy = v.cy0 + v.mean_v * t;
    double dx = x - cx, dy = y - cy;
    if (v.min_image) {
        dx = dx - v.len_x * rint(dx / v.len_x);
        dy = dy - v.len_y * rint(dy / v.len_y);
    }
    const double r2 = dx * dx + dy * dy;
    const double f = exp(0.5 * (1.0 - r2));
    const double du = -v.beta / (2.0 * PI) * dy * f;
    const double dv = v.beta / (2.0 * PI) * dx * f;
    const double dtemp = -(v.gamma - 1.0) * v.beta * v.beta / (8.0 * v.gamma * PI * PI) * exp(1.0 - r2);
    const double temp = 1.0 + dtemp;
    const double rho = pow(temp, 1.0 / (v.gamma - 1.0));
    if (cons) {
        const double p = pow(rho, v.gamma);
        *cons = prim_to_cons(rho, v.mean_u + du, v.mean_v + dv, p, v.gamma - 1.0);
    }
    return rho;
}

__global__ void init_vortex_kernel(Geometry g, efvm_vortex v, double* q) {
    const long long n = (long long)g.nx * g.ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t / g.nx), i = (int)(t - (long long)j * g.nx);
        U4 c;
        vortex_rho(v, 0.0, centre(g.lo[0], g.h[0], i), centre(g.lo[1], g.h[1], j + g.j_off), &c);
        store4(q, g.plane, cidx(g, i, j), c);
    }
}

// Per-block partials of sum |rho - rho_exact| and max |rho - rho_exact|.
__global__ void density_error_kernel(Geometry g, efvm_vortex v, const double* __restrict__ q,
                                     const DevState* st, double* partial) {
    __shared__ double s1[256], s2[256];
    const double t = st->time;
    double a = 0.0, m = 0.0;
    const long long n = (long long)g.nx * g.ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(k / g.nx), i = (int)(k - (long long)j * g.nx);
        const double ex = vortex_rho(v, t, centre(g.lo[0], g.h[0], i), centre(g.lo[1], g.h[1], j + g.j_off), nullptr);
        const double e = fabs(q[cidx(g, i, j)] - ex);
        a += e;
        m = fmax(m, e);
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            s1[threadIdx.x] += s1[threadIdx.x + s];
            s2[threadIdx.x] = fmax(s2[threadIdx.x], s2[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = s1[0];
        partial[2 * blockIdx.x + 1] = s2[0];
    }
}

__global__ void total_mass_kernel(Geometry g, const double* __restrict__ q, double* partial) {
    __shared__ double s1[256];
    double a = 0.0;
    const long long n = (long long)g.nx * g.ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(k / g.nx), i = (int)(k - (long long)j * g.nx);
        a += q[cidx(g, i, j)] * g.cell_volume;
    }
    s1[threadIdx.x] = a;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) s1[threadIdx.x] += s1[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s1[0];
}

// ---------------------------------------------------------------------------
// Host launch wrappers
// ---------------------------------------------------------------------------
// Launch with programmatic stream serialization when `pdl` is set (the kernel
// must begin with pdl_wait_then_release).
template <typename... KArgs, typename... Args>
static void launch_ks(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, bool pdl,
                      Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}
template <typename... KArgs, typename... Args>
static void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, bool pdl, Args... args) {
    launch_ks(kernel, grid, block, 0, s, pdl, args...);
}

static int grid_for(long long n, int block) {
    long long b = (n + block - 1) / block;
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    return (int)b;
}

// Resident blocks per SM (the register budget: 65536 / (MINB x 128 threads))
// and the loop order of each stage-kernel form, from a sweep of MINB 4..8, both
// orders and 2..8 rows per warp, timed as whole steps:
//  * FP64 inviscid (4096^2 vortex): 6 blocks (80 registers), x-face first --
//    2.674 ms per step against 2.747 at 5 blocks with the y-face first;
//  * FP64 viscous (1100x205 cylinder): 5 blocks (96), x-face first; the
//    cylinder is latency-bound and within 0.2 % for every choice;
//  * FP32-flux inviscid: 8 blocks (64), y-face first (x-face first costs 20 %);
//  * FP32-flux viscous: 5 blocks (96), y-face first: 92.2 us per cylinder step
//    against 96.3 at 8 blocks, where the FP64 viscous terms spill.
template <class R, bool VISC>
struct StageForm {
    static constexpr bool FP64 = sizeof(R) == sizeof(double);
    static constexpr int MINB = FP64 ? (VISC ? 5 : 6) : (VISC ? 5 : 8);
    // a second resident-block count the stage autotuner may pick (0: none): the FP64
    // inviscid form at 7 blocks (72 registers) measured from 4 % faster to 0.6 %
    // slower than at 6 on different boxes and run lengths
    static constexpr int ALT = FP64 && !VISC ? 7 : 0;
    static constexpr bool XFIRST = FP64;
};

static int form_minb(bool fp32, bool viscous) {
    return fp32 ? (viscous ? StageForm<float, true>::MINB : StageForm<float, false>::MINB)
                : (viscous ? StageForm<double, true>::MINB : StageForm<double, false>::MINB);
}

// Rows each warp marches.  Small grids take the fewest rows that still fill the
// resident slots in one wave (the warp's first row also pays for the face below
// it); large grids take 16, measured fastest at 4096^2 (ms per step, FP64 strip
// / FP32-flux TMA form: 8 rows 2.589 / 1.737, 16 rows 2.575 / 1.671, 32 rows
// 2.599 / 1.689, 64 rows 2.874 / 1.779, one wave of 158 rows 2.681 / 1.813).
static int rows_per_warp(int nx, int ny, int blocks_per_sm) {
    const long long strips = (nx + STRIP - 1) / STRIP;
    const long long slots = 148LL * blocks_per_sm * WPB;
    long long rows = (strips * ny + slots - 1) / slots;
    if (rows < 2) rows = 2;
    if (rows > 16) rows = 16;
    return (int)rows;
}

template <int SCHEME, int RECON, class R, bool VISC>
static void launch_stage_t(const StageArgs& a, bool pdl, cudaStream_t s) {
    using F = StageForm<R, VISC>;
    const bool alt = F::ALT > 0 && a.blocks == F::ALT;
    const int rows = a.rows > 0 ? a.rows : rows_per_warp(a.g.nx, a.g.ny, alt ? F::ALT : F::MINB);
    const int strips = (a.g.nx + STRIP - 1) / STRIP;
    dim3 block(32 * WPB);
    dim3 grid((strips + WPB - 1) / WPB, (a.g.ny + rows - 1) / rows);
    if constexpr (F::ALT > 0) {
        if (alt) {
            launch_k(stage_kernel<SCHEME, RECON, R, F::ALT, VISC, false, F::XFIRST>, grid, block, s, pdl, a, rows);
            return;
        }
    }
    // the viscous MUSCL forms (the strip kernel is the only form of their cases)
    // are built per limiter, as the TMA-fed form is
    if constexpr (VISC && RECON == EFVM_RECON_MUSCL) {
        if (a.ph.limiter == EFVM_LIMITER_MC)
            launch_k(stage_kernel<SCHEME, RECON, R, F::MINB, VISC, false, F::XFIRST, EFVM_LIMITER_MC>, grid, block, s,
                     pdl, a, rows);
        else
            launch_k(stage_kernel<SCHEME, RECON, R, F::MINB, VISC, false, F::XFIRST, EFVM_LIMITER_MINMOD>, grid, block,
                     s, pdl, a, rows);
        return;
    }
    launch_k(stage_kernel<SCHEME, RECON, R, F::MINB, VISC, false, F::XFIRST>, grid, block, s, pdl, a, rows);
}

template <class R, bool VISC>
static void launch_stage_v(const StageArgs& a, bool pdl, cudaStream_t s) {
    const bool muscl = a.ph.reconstruction == EFVM_RECON_MUSCL;
    switch (a.ph.flux_scheme) {
        case EFVM_FLUX_RUSANOV:
            muscl ? launch_stage_t<EFVM_FLUX_RUSANOV, EFVM_RECON_MUSCL, R, VISC>(a, pdl, s)
                  : launch_stage_t<EFVM_FLUX_RUSANOV, EFVM_RECON_FIRST_ORDER, R, VISC>(a, pdl, s);
            break;
        case EFVM_FLUX_HLLC_TEXTBOOK:
            muscl ? launch_stage_t<EFVM_FLUX_HLLC_TEXTBOOK, EFVM_RECON_MUSCL, R, VISC>(a, pdl, s)
                  : launch_stage_t<EFVM_FLUX_HLLC_TEXTBOOK, EFVM_RECON_FIRST_ORDER, R, VISC>(a, pdl, s);
            break;
        default:
            muscl ? launch_stage_t<EFVM_FLUX_HLLC, EFVM_RECON_MUSCL, R, VISC>(a, pdl, s)
                  : launch_stage_t<EFVM_FLUX_HLLC, EFVM_RECON_FIRST_ORDER, R, VISC>(a, pdl, s);
    }
}

// The viscous terms are a compile-time branch: the inviscid kernels carry none
// of their registers.
template <class R>
static void launch_stage_r(const StageArgs& a, bool pdl, cudaStream_t s) {
    if (a.ph.viscous) launch_stage_v<R, true>(a, pdl, s);
    else launch_stage_v<R, false>(a, pdl, s);
}

// ---- the TMA-fed stage kernel ----------------------------------------------
// Resident blocks per SM.  The FP32-flux form's shared memory is the ring
// (32.3 KB per block), so six fit in the SM's 228 KB, and it is built for six
// (80 registers).  The FP64 form adds its 12 KB row carry, so five fit, and it
// is built for five (up to 102 registers; it uses 92, 1 % faster at 4096^2
// than the same form held to 80).
constexpr int TMA_MINB = 6;
constexpr int tma_resident(bool fp32) { return fp32 ? TMA_MINB : 5; }

bool stage_tma_eligible(const Geometry& g, const Physics& ph, bool ibm, bool corr) {
    return g.nz <= 1 && !ph.viscous && !ibm && !corr && !ph.sponge && ph.body_force_x == 0.0;
}

template <int SCHEME, int RECON, class R, int LIM, bool PXY>
static void launch_stage_tma_k(const StageArgs& a, bool pdl, cudaStream_t s) {
    constexpr bool XFIRST = StageForm<R, false>::XFIRST;
    auto kernel = stage_tma_kernel<SCHEME, RECON, R, tma_resident(sizeof(R) == sizeof(float)), XFIRST, LIM, PXY>;
    // the largest shared-memory carve-out, once per device
    static unsigned long long carveout_set = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !(carveout_set & (1ull << dev))) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
        carveout_set |= 1ull << dev;
    }
    const int rows = a.rows > 0 ? a.rows : rows_per_warp(a.g.nx, a.g.ny, tma_resident(sizeof(R) == sizeof(float)));
    const int strips = (a.g.nx + STRIP - 1) / STRIP;
    const dim3 grid((strips + WPB - 1) / WPB, (a.g.ny + rows - 1) / rows);
    const CUtensorMap* m_in = static_cast<const CUtensorMap*>(a.tmap_in);
    const CUtensorMap* m_u0 = static_cast<const CUtensorMap*>(a.tmap_u0 ? a.tmap_u0 : a.tmap_in);
    launch_ks(kernel, grid, dim3(32 * WPB), (size_t)tma::SMEM_BYTES, s, pdl, a, rows, *m_in, *m_u0);
}

// The TMA-fed form is built per limiter (MUSCL) and for fully periodic grids,
// so that those branches are decided at compile time: with the sponge, body
// force and solid mask compiled out as well, the FP64 form's no_instruction and
// branch_resolving stalls were the largest after the FP64 dependency chains.
template <int SCHEME, int RECON, class R>
static void launch_stage_tma_t(const StageArgs& a, bool pdl, cudaStream_t s) {
    const bool pxy = a.ph.periodic_x && a.ph.periodic_y;
    if constexpr (RECON == EFVM_RECON_MUSCL) {
        if (a.ph.limiter == EFVM_LIMITER_MC)
            pxy ? launch_stage_tma_k<SCHEME, RECON, R, EFVM_LIMITER_MC, true>(a, pdl, s)
                : launch_stage_tma_k<SCHEME, RECON, R, EFVM_LIMITER_MC, false>(a, pdl, s);
        else
            pxy ? launch_stage_tma_k<SCHEME, RECON, R, EFVM_LIMITER_MINMOD, true>(a, pdl, s)
                : launch_stage_tma_k<SCHEME, RECON, R, EFVM_LIMITER_MINMOD, false>(a, pdl, s);
    } else {
        pxy ? launch_stage_tma_k<SCHEME, RECON, R, -1, true>(a, pdl, s)
            : launch_stage_tma_k<SCHEME, RECON, R, -1, false>(a, pdl, s);
    }
}

template <class R>
static void launch_stage_tma_r(const StageArgs& a, bool pdl, cudaStream_t s) {
    const bool muscl = a.ph.reconstruction == EFVM_RECON_MUSCL;
    switch (a.ph.flux_scheme) {
        case EFVM_FLUX_RUSANOV:
            muscl ? launch_stage_tma_t<EFVM_FLUX_RUSANOV, EFVM_RECON_MUSCL, R>(a, pdl, s)
                  : launch_stage_tma_t<EFVM_FLUX_RUSANOV, EFVM_RECON_FIRST_ORDER, R>(a, pdl, s);
            break;
        case EFVM_FLUX_HLLC_TEXTBOOK:
            muscl ? launch_stage_tma_t<EFVM_FLUX_HLLC_TEXTBOOK, EFVM_RECON_MUSCL, R>(a, pdl, s)
                  : launch_stage_tma_t<EFVM_FLUX_HLLC_TEXTBOOK, EFVM_RECON_FIRST_ORDER, R>(a, pdl, s);
            break;
        default:
            muscl ? launch_stage_tma_t<EFVM_FLUX_HLLC, EFVM_RECON_MUSCL, R>(a, pdl, s)
                  : launch_stage_tma_t<EFVM_FLUX_HLLC, EFVM_RECON_FIRST_ORDER, R>(a, pdl, s);
    }
}

// A state buffer (4 planes of ny + 4 rows x pitch doubles) as a 3-D tensor
// (columns, rows, planes); the box is one row of the 4 planes, 128 columns for
// the stage input and 124 for U^n.  cuTensorMapEncodeTiled comes from the
// driver through the runtime's entry-point query, so the library links no
// driver library.
int encode_state_map(const Geometry& g, const double* buf, bool u0, void* map_out) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return 1;
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[3] = {(cuuint64_t)g.pitch, (cuuint64_t)(g.ny + 2 * YO), 4};
    const cuuint64_t strides[2] = {(cuuint64_t)g.pitch * sizeof(double), (cuuint64_t)g.plane * sizeof(double)};
    const cuuint32_t box[3] = {(cuuint32_t)(u0 ? tma::U0_COLS : tma::IN_COLS), 1, 4};
    const cuuint32_t elem[3] = {1, 1, 1};
    const CUresult r = encode(static_cast<CUtensorMap*>(map_out), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                              const_cast<double*>(buf), dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : 2;
}

#include "efvm_kernels3d.cuh"

int launch_stage(const StageArgs& a, bool pdl, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (a.g.nz > 1) return launch_stage3(a, pdl, s);
    if (a.tmap_in && stage_tma_eligible(a.g, a.ph, a.mask != nullptr, a.corr != nullptr)) {
        if (a.ph.precision == EFVM_PREC_FP32_FLUX) launch_stage_tma_r<float>(a, pdl, s);
        else launch_stage_tma_r<double>(a, pdl, s);
        return 1;
    }
    if (a.corr) {  // the learned correction runs with MUSCL + HLLC (checked when it is attached)
        using F32 = StageForm<float, false>;
        using F64 = StageForm<double, false>;
        const bool fp32 = a.ph.precision == EFVM_PREC_FP32_FLUX;
        const int rows = rows_per_warp(a.g.nx, a.g.ny, form_minb(fp32, false));
        dim3 grid((stage_strips(a.g.nx) + WPB - 1) / WPB, (a.g.ny + rows - 1) / rows);
        if (fp32)
            launch_k(stage_kernel<EFVM_FLUX_HLLC, EFVM_RECON_MUSCL, float, F32::MINB, false, true, F32::XFIRST>, grid,
                     dim3(32 * WPB), s, pdl, a, rows);
        else
            launch_k(stage_kernel<EFVM_FLUX_HLLC, EFVM_RECON_MUSCL, double, F64::MINB, false, true, F64::XFIRST>, grid,
                     dim3(32 * WPB), s, pdl, a, rows);
        return 1;
    }
    if (a.ph.precision == EFVM_PREC_FP32_FLUX) launch_stage_r<float>(a, pdl, s);
    else launch_stage_r<double>(a, pdl, s);
    return 1;
}

int stage_strips(int nx) { return (nx + STRIP - 1) / STRIP; }

int stage_rows(int nx, int ny, bool fp32, bool viscous, bool tma) {
    return rows_per_warp(nx, ny, tma ? tma_resident(fp32) : form_minb(fp32, viscous));
}
int stage_blocks_per_sm(bool fp32, bool viscous, bool tma) { return tma ? tma_resident(fp32) : form_minb(fp32, viscous); }

int stage_alt_blocks(bool fp32, bool viscous) {
    return fp32 ? (viscous ? StageForm<float, true>::ALT : StageForm<float, false>::ALT)
                : (viscous ? StageForm<double, true>::ALT : StageForm<double, false>::ALT);
}

template <int SCHEME, int RECON, class R, bool VISC>
static void launch_batch_f(const BatchStageArgs& b, int n_tiles, bool pdl, cudaStream_t s) {
    using F = StageForm<R, VISC>;
    launch_k(batch_stage_kernel<SCHEME, RECON, R, F::MINB, VISC, F::XFIRST>, dim3((n_tiles + WPB - 1) / WPB),
             dim3(32 * WPB), s, pdl, b, n_tiles);
}

template <int SCHEME, int RECON, class R>
static void launch_batch_t(const BatchStageArgs& b, int n_tiles, bool pdl, cudaStream_t s) {
    // every case of a batch shares the viscous setting
    if (b.ph.viscous) launch_batch_f<SCHEME, RECON, R, true>(b, n_tiles, pdl, s);
    else launch_batch_f<SCHEME, RECON, R, false>(b, n_tiles, pdl, s);
}

template <class R>
static void launch_batch_r(const BatchStageArgs& b, int n_tiles, bool pdl, cudaStream_t s) {
    const bool muscl = b.ph.reconstruction == EFVM_RECON_MUSCL;
    switch (b.ph.flux_scheme) {
        case EFVM_FLUX_RUSANOV:
            muscl ? launch_batch_t<EFVM_FLUX_RUSANOV, EFVM_RECON_MUSCL, R>(b, n_tiles, pdl, s)
                  : launch_batch_t<EFVM_FLUX_RUSANOV, EFVM_RECON_FIRST_ORDER, R>(b, n_tiles, pdl, s);
            break;
        case EFVM_FLUX_HLLC_TEXTBOOK:
            muscl ? launch_batch_t<EFVM_FLUX_HLLC_TEXTBOOK, EFVM_RECON_MUSCL, R>(b, n_tiles, pdl, s)
                  : launch_batch_t<EFVM_FLUX_HLLC_TEXTBOOK, EFVM_RECON_FIRST_ORDER, R>(b, n_tiles, pdl, s);
            break;
        default:
            muscl ? launch_batch_t<EFVM_FLUX_HLLC, EFVM_RECON_MUSCL, R>(b, n_tiles, pdl, s)
                  : launch_batch_t<EFVM_FLUX_HLLC, EFVM_RECON_FIRST_ORDER, R>(b, n_tiles, pdl, s);
    }
}

int launch_batch_stage(const BatchStageArgs& b, int n_tiles, bool pdl, void* stream) {
    if (n_tiles <= 0) return 0;
    cudaStream_t s = (cudaStream_t)stream;
    if (b.ph.precision == EFVM_PREC_FP32_FLUX) launch_batch_r<float>(b, n_tiles, pdl, s);
    else launch_batch_r<double>(b, n_tiles, pdl, s);
    return 1;
}

template <int SCHEME, int RECON, class R, bool VISC>
static void launch_persist_f(const PersistArgs& p, int blocks, cudaStream_t s) {
    using F = StageForm<R, VISC>;
    launch_k(batch_persistent_kernel<SCHEME, RECON, R, F::MINB, VISC, F::XFIRST>, dim3(blocks), dim3(32 * WPB), s,
             false, p);
}

template <class R>
static void launch_persist_r(const PersistArgs& p, int blocks, cudaStream_t s) {
    const bool muscl = p.ph.reconstruction == EFVM_RECON_MUSCL;
    const bool visc = p.ph.viscous != 0;
#define EFVM_PERSIST_V(S, RC)                                                   \
    (visc ? launch_persist_f<S, RC, R, true>(p, blocks, s) : launch_persist_f<S, RC, R, false>(p, blocks, s))
    switch (p.ph.flux_scheme) {
        case EFVM_FLUX_RUSANOV:
            muscl ? EFVM_PERSIST_V(EFVM_FLUX_RUSANOV, EFVM_RECON_MUSCL) : EFVM_PERSIST_V(EFVM_FLUX_RUSANOV, EFVM_RECON_FIRST_ORDER);
            break;
        case EFVM_FLUX_HLLC_TEXTBOOK:
            muscl ? EFVM_PERSIST_V(EFVM_FLUX_HLLC_TEXTBOOK, EFVM_RECON_MUSCL)
                  : EFVM_PERSIST_V(EFVM_FLUX_HLLC_TEXTBOOK, EFVM_RECON_FIRST_ORDER);
            break;
        default:
            muscl ? EFVM_PERSIST_V(EFVM_FLUX_HLLC, EFVM_RECON_MUSCL) : EFVM_PERSIST_V(EFVM_FLUX_HLLC, EFVM_RECON_FIRST_ORDER);
    }
#undef EFVM_PERSIST_V
}

int batch_form_blocks(bool fp32, bool viscous) { return form_minb(fp32, viscous); }

// One block per resident slot (blocks_per_sm on every SM): the warps take their
// work from the ticket counter, so the grid does not depend on the table.
int launch_batch_persistent(const PersistArgs& p, int blocks_per_sm, int n_sms, void* stream) {
    if (p.n_tiles <= 0 || p.rounds <= 0) return 0;
    const int blocks = std::max(1, blocks_per_sm) * std::max(1, n_sms);
    cudaStream_t s = (cudaStream_t)stream;
    if (p.ph.precision == EFVM_PREC_FP32_FLUX) launch_persist_r<float>(p, blocks, s);
    else launch_persist_r<double>(p, blocks, s);
    return 1;
}

int launch_batch_setup(const Physics& ph, const BatchCase* cases, int n_cases, bool pdl, void* stream) {
    launch_k(batch_setup_kernel, dim3((n_cases + 127) / 128), dim3(128), (cudaStream_t)stream, pdl, ph, cases,
             n_cases);
    return 1;
}

int launch_clock(unsigned long long* out, void* stream) {
    clock_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(out);
    return 1;
}

int launch_fill_ghosts(const Geometry& g, const Physics& ph, double* q, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (g.nz > 1) {
        fill_ghosts3_kernel<<<grid_for((long long)g.nx * g.ny * g.nz, 256), 256, 0, s>>>(g, ph, q);
        return 1;
    }
    fill_ghosts_x_kernel<<<(g.ny + 127) / 128, 128, 0, s>>>(g, ph, q);
    fill_ghosts_y_kernel<<<(g.nx + 127) / 128, 128, 0, s>>>(g, ph, q);
    return 2;
}

int launch_cfl(const Geometry& g, const Physics& ph, const double* q, DevState* st, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    reset_lam_kernel<<<1, 1, 0, s>>>(st);
    if (g.nz > 1) {
        cfl3_kernel<<<grid_for((long long)g.nx * g.ny * g.nz, 256), 256, 0, s>>>(g, ph, q, st);
        return 2;
    }
    cfl_kernel<<<grid_for((long long)g.nx * g.ny, 256), 256, 0, s>>>(g, ph, q, st);
    return 2;
}

int launch_step_setup(const Physics& ph, DevState* st, bool pdl, void* stream) {
    launch_k(step_setup_kernel, dim3(1), dim3(1), (cudaStream_t)stream, pdl, ph, st);
    return 1;
}

// The output fields of write_vtk_to (crates/cfd_output/src/lib.rs:36-125) per
// interior cell, x fastest: density, pressure, temperature, velocity (u, v, w)
// and Mach, as 7 planes of nx*ny doubles.
__global__ void output_fields_kernel(Geometry g, Physics ph, const double* __restrict__ q, double* __restrict__ out) {
    const long long n = (long long)g.nx * g.ny;
    const double gm1 = ph.gamma - 1.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t / g.nx), i = (int)(t - (long long)j * g.nx);
        const U4 u = load4(q, g.plane, cidx(g, i, j));
        const double p = pressure_d(u, gm1);                     // IdealGas::pressure
        const double vu = u.mx / u.r, vv = u.my / u.r;
        const double ke = 0.5 * u.r * (vu * vu + vv * vv);
        const double t_ = gm1 * (u.E - ke) / u.r / ph.r_gas;     // cons_to_prim(u).t
        const double a = sqrt(ph.gamma * p / u.r);               // sound_speed
        out[t] = u.r;
        out[n + t] = p;
        out[2 * n + t] = t_;
        out[3 * n + t] = vu;
        out[4 * n + t] = vv;
        out[5 * n + t] = 0.0;
        out[6 * n + t] = sqrt(vu * vu + vv * vv) / a;
    }
}

int launch_output_fields(const Geometry& g, const Physics& ph, const double* q, double* out, void* stream) {
    output_fields_kernel<<<grid_for((long long)g.nx * g.ny, 256), 256, 0, (cudaStream_t)stream>>>(g, ph, q, out);
    return 1;
}

// compute_marker_loadings_per_body, crates/cfd_ibm/src/lib.rs:509-562: warp b
// sums the traction of body b's markers (lane l takes markers l, l + 32, ...),
// then a shuffle tree (fixed order) gives the body's loads and torque.
__global__ void body_loads_kernel(Geometry g, Physics ph, Ibm ib, const double* __restrict__ q,
                                  const double* __restrict__ centres, int n_bodies, int per_body,
                                  double* __restrict__ out) {
    const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= n_bodies) return;  // uniform per warp
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int m = b * per_body + lane; m < (b + 1) * per_body; m += 32) {
        const MarkerDev mk = ib.markers[m];
        if (!mk.valid) continue;
        double img[5];
        if (!sample_bilinear(g, ph, q, mk.fluid, mk.lo_i, mk.lo_j, mk.tx, mk.ty, img)) continue;
        if (!(isfinite(img[3]) && isfinite(img[4]) && isfinite(img[1]) && isfinite(img[2]))) continue;
        const double us[3] = {img[1] - mk.wall_velocity[0], img[2] - mk.wall_velocity[1], 0.0 - mk.wall_velocity[2]};
        const double udotn = us[0] * mk.normal[0] + us[1] * mk.normal[1] + us[2] * mk.normal[2];
        const double mu = viscosity(ph, img[4]);
        double df[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double ut = us[d] - udotn * mk.normal[d];
            const double fp = -img[3] * mk.normal[d] * mk.area;
            const double fv = mu * ut / ib.sample_offset * mk.area;
            acc[d] += fp;
            acc[3 + d] += fv;
            df[d] = fp + fv;
        }
        const double r[3] = {mk.pos[0] - centres[2 * b], mk.pos[1] - centres[2 * b + 1], 0.0};
        acc[6] += r[1] * df[2] - r[2] * df[1];
        acc[7] += r[2] * df[0] - r[0] * df[2];
        acc[8] += r[0] * df[1] - r[1] * df[0];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k)
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], o);
    if (lane == 0)
        for (int k = 0; k < 9; ++k) out[9 * b + k] = acc[k];
}

int launch_body_loads(const Geometry& g, const Physics& ph, const Ibm& ib, const double* q, const double* centres,
                      int n_bodies, int markers_per_body, double* out, void* stream) {
    if (n_bodies <= 0) return 0;
    body_loads_kernel<<<(n_bodies + 3) / 4, 128, 0, (cudaStream_t)stream>>>(g, ph, ib, q, centres, n_bodies,
                                                                           markers_per_body, out);
    return 1;
}

// Two rows of one y side to/from a contiguous buffer [variable][row][i].
// unpack == 0: interior rows j0, j0+1 -> buf; unpack == 1: buf -> rows j0, j0+1.
__global__ void halo_rows_kernel(Geometry g, double* q, double* buf, int j0, int unpack) {
    const int n = 4 * 2 * g.nx;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int v = t / (2 * g.nx), r = (t / g.nx) % 2, i = t % g.nx;
        const long long o = (long long)v * g.plane + cidx(g, i, j0 + r);
        if (unpack) q[o] = buf[t];
        else buf[t] = q[o];
    }
}

int launch_halo_rows(const Geometry& g, double* q, double* buf, int j0, int unpack, void* stream) {
    const int n = 4 * 2 * g.nx;
    halo_rows_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(g, q, buf, j0, unpack);
    return 1;
}

__global__ void set_control_kernel(DevState* st, int active, int stop_at_t, double t_stop, long long hist_cap) {
    st->active = active;
    st->stop_at_t = stop_at_t;
    st->t_stop = t_stop;
    st->hist_pos = 0;
    st->hist_cap = hist_cap;
}

int launch_set_control(DevState* st, int active, int stop_at_t, double t_stop, long long hist_cap, void* stream) {
    set_control_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(st, active, stop_at_t, t_stop, hist_cap);
    return 1;
}

int launch_geometry(const Geometry& g, const double* cyl, int ncyl, const double* stagnant, const double* ambient,
                    double* q, uint8_t* mask, void* stream) {
    const U4 sg{stagnant[0], stagnant[1], stagnant[2], stagnant[4]};
    const U4 am{ambient[0], ambient[1], ambient[2], ambient[4]};
    geometry_kernel<<<grid_for((long long)g.nx * g.ny, 256), 256, 0, (cudaStream_t)stream>>>(g, cyl, ncyl, sg, am, q,
                                                                                               mask);
    return 1;
}

int launch_ibm(const Geometry& g, const Physics& ph, const Ibm& ib, double* q, DevState* st,
               int force_stage, int mirror_stage, int setup, bool pdl, void* stream, int deferred) {
    const int nf = force_stage >= 0 ? 1 + (ib.n_ghost + IBM_THREADS - 1) / IBM_THREADS : 0;
    int nm = mirror_stage >= 0 ? (ib.n_ghost + IBM_THREADS - 1) / IBM_THREADS : 0;
    if (setup && nm < 1) nm = 1;
    if (nf + nm == 0) return 0;
    launch_k(ibm_kernel, dim3(nf + nm), dim3(IBM_THREADS), (cudaStream_t)stream, pdl, g, ph, ib, q, st, force_stage,
             nf, mirror_stage, setup, deferred);
    return 1;
}

int launch_pack(const Geometry& g, const double* src, int64_t si, int64_t sj, int64_t sv, double* q, int to_device,
                void* stream) {
    pack_kernel<<<grid_for((long long)g.nx * g.ny, 256), 256, 0, (cudaStream_t)stream>>>(
        g, src, si, sj, sv, q, const_cast<double*>(src), to_device);
    return 1;
}

int launch_init_vortex(const Geometry& g, const efvm_vortex& v, double* q, void* stream) {
    init_vortex_kernel<<<grid_for((long long)g.nx * g.ny, 256), 256, 0, (cudaStream_t)stream>>>(g, v, q);
    return 1;
}

int launch_density_error(const Geometry& g, const efvm_vortex& v, const double* q, const DevState* st,
                         double* partial, int nblocks, void* stream) {
    density_error_kernel<<<nblocks, 256, 0, (cudaStream_t)stream>>>(g, v, q, st, partial);
    return 1;
}

int launch_total_mass(const Geometry& g, const double* q, double* partial, int nblocks, void* stream) {
    if (g.nz > 1) {
        total_mass3_kernel<<<nblocks, 256, 0, (cudaStream_t)stream>>>(g, q, partial);
        return 1;
    }
    total_mass_kernel<<<nblocks, 256, 0, (cudaStream_t)stream>>>(g, q, partial);
    return 1;
}


int launch_pack3(const Geometry& g, double* host_like, int64_t si, int64_t sj, int64_t sk, int64_t sv, double* q,
                 int to_device, void* stream) {
    pack3_kernel<<<grid_for((long long)g.nx * g.ny * g.nz, 256), 256, 0, (cudaStream_t)stream>>>(
        g, host_like, si, sj, sk, sv, q, to_device);
    return 1;
}

int launch_geometry3(const Geometry& g, const Physics& ph, const double* spheres, int n, const double* stagnant,
                     const double* ambient, double* q, uint8_t* mask, void* stream) {
    const U5 sg{stagnant[0], stagnant[1], stagnant[2], stagnant[3], stagnant[4]};
    const U5 am{ambient[0], ambient[1], ambient[2], ambient[3], ambient[4]};
    geometry3_kernel<<<grid_for((long long)g.nx * g.ny * g.nz, 256), 256, 0, (cudaStream_t)stream>>>(
        g, ph, spheres, n, sg, am, q, mask);
    return 1;
}

int launch_mirror3(const Geometry& g, const Physics& ph, const Ibm& ib, double* q, bool pdl, void* stream) {
    const int nb = ib.n_ghost > 0 ? (ib.n_ghost + 127) / 128 : 1;
    launch_k(mirror3_kernel, dim3(nb), dim3(128), (cudaStream_t)stream, pdl, g, ph, ib, q);
    return 1;
}

int launch_forces3(const Geometry& g, const Physics& ph, const Ibm& ib, const double* q, DevState* st, bool pdl,
                   void* stream) {
    launch_k(forces3_kernel, dim3(1), dim3(FORCE3_THREADS), (cudaStream_t)stream, pdl, g, ph, ib, q, st);
    return 1;
}

}  // namespace efvm
