// efvm_oracle.cpp — CPU ORACLE (test infrastructure only; see efvm_oracle.hpp).
//
// Serial FP64 restatement of dev_field_efvm's explicit finite-volume step plus a
// C API (oracle_*) that tests and the bench's CPU-baseline leg load with ctypes.
// Citations are file:line inside the dev_field_efvm source tree.
#include "efvm_oracle.hpp"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

static const double PI = 3.141592653589793;  // std::f64::consts::PI
static const double R_GAS_AIR = 287.058;     // examples/cylinder_drag_validation/main.rs:69

// ---------------------------------------------------------------------------
// cfd_riemann (crates/cfd_riemann/src/lib.rs)
// ---------------------------------------------------------------------------

// physical_flux_inline, :21-43
ConsVar physical_flux(const ConsVar& u, const IdealGas& eos, int dir) {
    const double p = eos.pressure(u);
    double vel[3];
    u.velocity(vel);
    const double v_n = vel[dir];
    ConsVar f(u.rho * v_n, u.rho_u * v_n, u.rho_v * v_n, u.rho_w * v_n, (u.rho_e + p) * v_n);
    f.comp(dir) += p;
    return f;
}

// Rusanov::flux_inline, :222-240
ConsVar rusanov_flux(const ConsVar& left, const ConsVar& right, const IdealGas& eos, int dir) {
    const ConsVar f_l = physical_flux(left, eos, dir);
    const ConsVar f_r = physical_flux(right, eos, dir);
    double vel_l[3], vel_r[3];
    left.velocity(vel_l);
    right.velocity(vel_r);
    const double a_l = eos.sound_speed(left);
    const double a_r = eos.sound_speed(right);
    const double lambda = std::fmax(std::fabs(vel_l[dir]) + a_l, std::fabs(vel_r[dir]) + a_r);
    return 0.5 * (f_l + f_r) - (0.5 * lambda) * (right - left);
}

// thornber_reconstruct, :456-506
static void thornber_reconstruct(const ConsVar& left, const ConsVar& right, const IdealGas& eos,
                                 ConsVar& left_c, ConsVar& right_c, double& a_l, double& a_r) {
    double vel_l[3], vel_r[3];
    left.velocity(vel_l);
    right.velocity(vel_r);
    const double v_l_sq = vel_l[0] * vel_l[0] + vel_l[1] * vel_l[1] + vel_l[2] * vel_l[2];
    const double v_r_sq = vel_r[0] * vel_r[0] + vel_r[1] * vel_r[1] + vel_r[2] * vel_r[2];
    a_l = eos.sound_speed(left);
    a_r = eos.sound_speed(right);
    const double v_max_sq = std::fmax(v_l_sq, v_r_sq);
    const double a_max = std::fmax(a_l, a_r);
    const double z = (v_max_sq >= a_max * a_max) ? 1.0 : std::sqrt(v_max_sq) / a_max;
    const double half = 0.5;
    const double avg0 = half * (vel_l[0] + vel_r[0]);
    const double avg1 = half * (vel_l[1] + vel_r[1]);
    const double avg2 = half * (vel_l[2] + vel_r[2]);
    const double dvel0 = half * z * (vel_l[0] - vel_r[0]);
    const double dvel1 = half * z * (vel_l[1] - vel_r[1]);
    const double dvel2 = half * z * (vel_l[2] - vel_r[2]);
    const double vel_lc[3] = {avg0 + dvel0, avg1 + dvel1, avg2 + dvel2};
    const double vel_rc[3] = {avg0 - dvel0, avg1 - dvel1, avg2 - dvel2};
    const double v_lc_sq = vel_lc[0] * vel_lc[0] + vel_lc[1] * vel_lc[1] + vel_lc[2] * vel_lc[2];
    const double v_rc_sq = vel_rc[0] * vel_rc[0] + vel_rc[1] * vel_rc[1] + vel_rc[2] * vel_rc[2];
    left_c = ConsVar(left.rho, left.rho * vel_lc[0], left.rho * vel_lc[1], left.rho * vel_lc[2],
                     left.rho_e + 0.5 * left.rho * (v_lc_sq - v_l_sq));
    right_c = ConsVar(right.rho, right.rho * vel_rc[0], right.rho * vel_rc[1], right.rho * vel_rc[2],
                      right.rho_e + 0.5 * right.rho * (v_rc_sq - v_r_sq));
}

// star_state, :619-644
static ConsVar star_state(const ConsVar& u, const double vel[3], double p, double un, double s,
                          double s_star, int dir) {
    const double rho_star = u.rho * (s - un) / (s - s_star);
    const double energy_per_mass = u.rho_e / u.rho;
    const double e_star = energy_per_mass + (s_star - un) * (s_star + p / (u.rho * (s - un)));
    const double rho_u = dir == 0 ? rho_star * s_star : rho_star * vel[0];
    const double rho_v = dir == 1 ? rho_star * s_star : rho_star * vel[1];
    const double rho_w = dir == 2 ? rho_star * s_star : rho_star * vel[2];
    return ConsVar(rho_star, rho_u, rho_v, rho_w, rho_star * e_star);
}

// Hllc::flux_with_thornber, :395-440
ConsVar hllc_flux(const ConsVar& left, const ConsVar& right, const IdealGas& eos, int dir, bool thornber) {
    ConsVar left_c, right_c;
    double a_l, a_r;
    if (thornber) {
        thornber_reconstruct(left, right, eos, left_c, right_c, a_l, a_r);
    } else {
        a_l = eos.sound_speed(left);
        a_r = eos.sound_speed(right);
        left_c = left;
        right_c = right;
    }
    double vel_l[3], vel_r[3];
    left_c.velocity(vel_l);
    right_c.velocity(vel_r);
    const double p_l = eos.pressure(left_c);
    const double p_r = eos.pressure(right_c);
    const double un_l = vel_l[dir];
    const double un_r = vel_r[dir];
    const double s_l = std::fmin(un_l - a_l, un_r - a_r);
    const double s_r = std::fmax(un_l + a_l, un_r + a_r);
    const double factor_l = left_c.rho * (s_l - un_l);
    const double factor_r = right_c.rho * (s_r - un_r);
    const double s_star = ((p_r - p_l) + factor_l * un_l - factor_r * un_r) / (factor_l - factor_r);
    if (s_l >= 0.0) {
        return physical_flux(left_c, eos, dir);
    } else if (s_star >= 0.0) {
        const ConsVar u_star_l = star_state(left_c, vel_l, p_l, un_l, s_l, s_star, dir);
        return physical_flux(left_c, eos, dir) + s_l * (u_star_l - left_c);
    } else if (s_r >= 0.0) {
        const ConsVar u_star_r = star_state(right_c, vel_r, p_r, un_r, s_r, s_star, dir);
        return physical_flux(right_c, eos, dir) + s_r * (u_star_r - right_c);
    } else {
        return physical_flux(right_c, eos, dir);
    }
}

ConsVar scheme_flux(int scheme, const ConsVar& l, const ConsVar& r, const IdealGas& eos, int dir) {
    switch (scheme) {
        case EFVM_FLUX_RUSANOV: return rusanov_flux(l, r, eos, dir);
        case EFVM_FLUX_HLLC_TEXTBOOK: return hllc_flux(l, r, eos, dir, false);
        default: return hllc_flux(l, r, eos, dir, true);
    }
}

// axis_and_sign, :147-167
static void axis_and_sign(const double n[3], int& dir, double& sign) {
    dir = 0;
    double maxabs = std::fabs(n[0]);
    if (std::fabs(n[1]) > maxabs) { dir = 1; maxabs = std::fabs(n[1]); }
    if (std::fabs(n[2]) > maxabs) { dir = 2; }
    sign = n[dir] >= 0.0 ? 1.0 : -1.0;
}

// axis_aligned, :100-109
static bool axis_aligned(const double n[3], int& dir, double& sign) {
    const double a = std::fabs(n[0]), b = std::fabs(n[1]), c = std::fabs(n[2]);
    const double mx = std::fmax(std::fmax(a, b), c);
    if (mx > 0.0 && (a + b + c - mx) <= 1e-12 * mx) {
        axis_and_sign(n, dir, sign);
        return true;
    }
    return false;
}

static void cross3(const double u[3], const double v[3], double o[3]) {
    o[0] = u[1] * v[2] - u[2] * v[1];
    o[1] = u[2] * v[0] - u[0] * v[2];
    o[2] = u[0] * v[1] - u[1] * v[0];
}

// face_frame / to_frame / from_frame, :113-143
static void face_frame(const double n[3], double fr[3][3]) {
    double a[3];
    if (std::fabs(n[0]) <= std::fabs(n[1]) && std::fabs(n[0]) <= std::fabs(n[2])) { a[0] = 1; a[1] = 0; a[2] = 0; }
    else if (std::fabs(n[1]) <= std::fabs(n[2])) { a[0] = 0; a[1] = 1; a[2] = 0; }
    else { a[0] = 0; a[1] = 0; a[2] = 1; }
    double t1[3];
    cross3(n, a, t1);
    const double l = std::sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
    t1[0] /= l; t1[1] /= l; t1[2] /= l;
    double t2[3];
    cross3(n, t1, t2);
    for (int d = 0; d < 3; ++d) { fr[0][d] = n[d]; fr[1][d] = t1[d]; fr[2][d] = t2[d]; }
}
static ConsVar to_frame(const ConsVar& u, const double fr[3][3]) {
    const double m[3] = {u.rho_u, u.rho_v, u.rho_w};
    double r[3];
    for (int e = 0; e < 3; ++e) r[e] = fr[e][0] * m[0] + fr[e][1] * m[1] + fr[e][2] * m[2];
    return ConsVar(u.rho, r[0], r[1], r[2], u.rho_e);
}
static ConsVar from_frame(const ConsVar& f, const double fr[3][3]) {
    const double m[3] = {f.rho_u, f.rho_v, f.rho_w};
    double b[3];
    for (int d = 0; d < 3; ++d) b[d] = fr[0][d] * m[0] + fr[1][d] * m[1] + fr[2][d] * m[2];
    return ConsVar(f.rho, b[0], b[1], b[2], f.rho_e);
}

// RiemannFlux::flux_normal, :76-93
ConsVar flux_normal(int scheme, const ConsVar& owner, const ConsVar& other, const IdealGas& eos, const double n[3]) {
    int dir;
    double sign;
    if (axis_aligned(n, dir, sign)) {
        if (sign >= 0.0) return scheme_flux(scheme, owner, other, eos, dir);
        return scheme_flux(scheme, other, owner, eos, dir) * -1.0;
    }
    double fr[3][3];
    face_frame(n, fr);
    const ConsVar f = scheme_flux(scheme, to_frame(owner, fr), to_frame(other, fr), eos, 0);
    return from_frame(f, fr);
}

// ---------------------------------------------------------------------------
// Limiters, crates/cfd_solver/src/lib.rs:170-211
// ---------------------------------------------------------------------------
double minmod(double a, double b) {
    if (a * b <= 0.0) return 0.0;
    if (std::fabs(a) < std::fabs(b)) return a;
    return b;
}
double monotonized_central(double a, double b) {
    if (a * b <= 0.0) return 0.0;
    const double s = a > 0.0 ? 1.0 : -1.0;
    return s * std::fmin(std::fmin(2.0 * std::fabs(a), 2.0 * std::fabs(b)), 0.5 * std::fabs(a + b));
}
ConsVar limited_slope_cons(const ConsVar& fwd, const ConsVar& bwd, int limiter) {
    double (*lim)(double, double) = limiter == EFVM_LIMITER_MC ? monotonized_central : minmod;
    return ConsVar(lim(fwd.rho, bwd.rho), lim(fwd.rho_u, bwd.rho_u), lim(fwd.rho_v, bwd.rho_v),
                   lim(fwd.rho_w, bwd.rho_w), lim(fwd.rho_e, bwd.rho_e));
}

// ---------------------------------------------------------------------------
// Boundary conditions, crates/cfd_boundary/src/lib.rs:172-362
// ---------------------------------------------------------------------------
ConsVar bc_ghost(const efvm_bc& bc, int side, const ConsVar& interior, const IdealGas& eos) {
    switch (bc.kind) {
        case EFVM_BC_SLIP_WALL:
        case EFVM_BC_SYMMETRY: {
            // SlipWall::ghost_at, :258-268: m' = m - 2 (m.n) n with the unit outward normal.
            ConsVar s = interior;
            double n[3] = {0, 0, 0};
            n[side / 2] = (side % 2 == 1) ? 1.0 : -1.0;
            const double mn = s.rho_u * n[0] + s.rho_v * n[1] + s.rho_w * n[2];
            s.rho_u -= 2.0 * mn * n[0];
            s.rho_v -= 2.0 * mn * n[1];
            s.rho_w -= 2.0 * mn * n[2];
            return s;
        }
        case EFVM_BC_NO_SLIP_WALL: {  // :278-284
            ConsVar s = interior;
            s.rho_u = -s.rho_u;
            s.rho_v = -s.rho_v;
            s.rho_w = -s.rho_w;
            return s;
        }
        case EFVM_BC_SUPERSONIC_INFLOW: {  // :228-231
            const double t = bc.p / (bc.rho * R_GAS_AIR);
            return eos.prim_to_cons(PrimVar{bc.rho, bc.u, bc.v, bc.w, bc.p, t});
        }
        case EFVM_BC_SUBSONIC_INFLOW: {  // :322-325
            const double p_interior = eos.pressure(interior);
            return eos.prim_to_cons(PrimVar{bc.rho, bc.u, bc.v, bc.w, p_interior, bc.t});
        }
        case EFVM_BC_PRESSURE_OUTLET: {  // :345-350
            PrimVar prim = eos.cons_to_prim(interior);
            prim.p = bc.p;
            prim.t = bc.p / (prim.rho * R_GAS_AIR);
            return eos.prim_to_cons(prim);
        }
        case EFVM_BC_PERIODIC:            // :199-201 (never called by the fill)
        case EFVM_BC_SUPERSONIC_OUTFLOW:  // :175-177
        default:
            return interior;
    }
}

// ---------------------------------------------------------------------------
// Mesh (inferred FIELD UniformMesh semantics; see the header)
// ---------------------------------------------------------------------------
void Mesh::init(const efvm_grid& g) {
    n[0] = g.nx; n[1] = g.ny; n[2] = g.nz;
    ng = g.ng;
    for (int a = 0; a < 3; ++a) {
        N[a] = n[a] + 2 * ng;
        lo[a] = g.lo[a];
        hi[a] = g.hi[a];
        h[a] = (hi[a] - lo[a]) / (double)n[a];
        periodic[a] = g.bc[2 * a].kind == EFVM_BC_PERIODIC && g.bc[2 * a + 1].kind == EFVM_BC_PERIODIC;
    }
}

bool Mesh::locate(const double p[3], size_t& lo_idx, int lo_raw[3], double t[3]) const {
    for (int a = 0; a < 3; ++a) {
        const double f = (p[a] - lo[a]) / h[a] - 0.5;
        const double fl = std::floor(f);
        const int i0 = (int)fl + ng;
        if (!(i0 >= 0 && i0 + 1 < N[a])) return false;
        lo_raw[a] = i0;
        t[a] = f - fl;
    }
    lo_idx = idx_raw(lo_raw[0], lo_raw[1], lo_raw[2]);
    return true;
}

// ---------------------------------------------------------------------------
// Case: the systems of one App, in MeshScheduleSet order
// ---------------------------------------------------------------------------
bool Case::setup(const efvm_grid& g, const efvm_params& p, const char** err) {
    static std::string msg;
    if (g.nx < 1 || g.ny < 1 || g.nz < 1 || g.ng < 1) { msg = "grid dimensions must be >= 1"; *err = msg.c_str(); return false; }
    for (int a = 0; a < 3; ++a) {
        const bool lo_p = g.bc[2 * a].kind == EFVM_BC_PERIODIC, hi_p = g.bc[2 * a + 1].kind == EFVM_BC_PERIODIC;
        if (lo_p != hi_p) {  // BoundaryRegistry::validate_periodic_pairs, crates/cfd_boundary/src/lib.rs:437-448
            msg = "invalid periodic boundary configuration: periodic boundary on axis " + std::to_string(a) +
                  " requires both sides";
            *err = msg.c_str();
            return false;
        }
        if (!(g.hi[a] > g.lo[a])) { msg = "bounds_hi must exceed bounds_lo"; *err = msg.c_str(); return false; }
    }
    grid = g;
    prm = p;
    mesh.init(g);
    eos.gamma = p.gamma;
    eos.r_gas = p.r_gas;
    visc.model = p.viscosity_model;
    visc.mu_const = p.mu;
    const size_t n = mesh.n_raw();
    u.assign(n, ConsVar());
    rhs.assign(n, ConsVar());
    u0.assign(n, ConsVar());
    solid.assign(n, 0);
    slopes.assign(3 * n, ConsVar());
    ss = SolverState();
    return true;
}

// cfl_system, crates/cfd_solver/src/lib.rs:626-677 (the loop; the gate is in substep)
double Case::cfl_dt() const {
    const double dx = mesh.h[0], dy = mesh.h[1], dz = mesh.h[2];
    double lambda_max = 0.0;
    for (int i = 0; i < mesh.n[0]; ++i)
        for (int j = 0; j < mesh.n[1]; ++j)
            for (int k = 0; k < mesh.n[2]; ++k) {
                const ConsVar& uc = u[mesh.idx(i, j, k)];
                if (uc.rho <= 0.0) continue;
                double vel[3];
                uc.velocity(vel);
                const double a = eos.sound_speed(uc);
                double lambda = (std::fabs(vel[0]) + a) / dx + (std::fabs(vel[1]) + a) / dy + (std::fabs(vel[2]) + a) / dz;
                if (prm.viscous) {
                    const double nu = visc.mu(eos.cons_to_prim(uc).t) / uc.rho;
                    lambda += 2.0 * nu * (1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz));
                }
                lambda_max = std::fmax(lambda_max, lambda);
            }
    return lambda_max > 0.0 ? prm.cfl / lambda_max : std::numeric_limits<double>::infinity();
}

void Case::cfl_system() {
    if (ss.rk_stage != 0) return;
    if (prm.fixed_dt > 0.0) { ss.dt = prm.fixed_dt; return; }
    ss.dt = cfl_dt();  // serial comm: all_reduce_min_f64 is the identity
}

// halo_system + FIELD's serial periodic wrap (crates/cfd_boundary/src/lib.rs:805-828)
void Case::halo_system() {
    const int ng = mesh.ng;
    for (int a = 0; a < 3; ++a) {
        if (!mesh.periodic[a]) continue;
        const int b = (a + 1) % 3, c = (a + 2) % 3;
        for (int ib = ng; ib < mesh.n[b] + ng; ++ib)
            for (int ic = ng; ic < mesh.n[c] + ng; ++ic)
                for (int g = 0; g < ng; ++g) {
                    int r_lo[3], s_lo[3], r_hi[3], s_hi[3];
                    r_lo[b] = s_lo[b] = r_hi[b] = s_hi[b] = ib;
                    r_lo[c] = s_lo[c] = r_hi[c] = s_hi[c] = ic;
                    r_lo[a] = g;                       // low ghost g  <- interior n-ng+g
                    s_lo[a] = mesh.n[a] + g;
                    r_hi[a] = mesh.n[a] + ng + g;      // high ghost    <- interior g
                    s_hi[a] = ng + g;
                    const size_t dl = mesh.idx_raw(r_lo[0], r_lo[1], r_lo[2]), sl = mesh.idx_raw(s_lo[0], s_lo[1], s_lo[2]);
                    const size_t dh = mesh.idx_raw(r_hi[0], r_hi[1], r_hi[2]), sh = mesh.idx_raw(s_hi[0], s_hi[1], s_hi[2]);
                    u[dl] = u[sl];
                    u[dh] = u[sh];
                    if (ibm) { solid[dl] = solid[sl]; solid[dh] = solid[sh]; }
                }
    }
}

// boundary_system, crates/cfd_boundary/src/lib.rs:574-601
void Case::boundary_system() {
    mesh.for_each_face([&](const Face& f) {
        if (f.patch < 0) return;
        const efvm_bc& bc = grid.bc[f.patch];
        if (bc.kind == EFVM_BC_PERIODIC) return;
        u[f.other] = bc_ghost(bc, f.patch, u[f.owner], eos);
    });
}

// parabolic_inflow_system, examples/cylinder_drag_validation/main.rs:151-177
void Case::parabolic_inflow_system() {
    const int ng = mesh.ng;
    const double um = prm.inflow_u_max, h = prm.inflow_height, rho = prm.inflow_rho;
    for (int k = 0; k < mesh.n[2]; ++k) {
        const int kr = k + ng;
        for (int j = 0; j < mesh.n[1]; ++j) {
            const int jr = j + ng;
            const size_t first = mesh.idx_raw(ng, jr, kr);
            const double y = mesh.centroid_axis(1, jr);
            const double uy = 4.0 * um * y * (h - y) / (h * h);
            const double p_in = eos.pressure(u[first]);
            const double t = p_in / (rho * R_GAS_AIR);
            const ConsVar cons = eos.prim_to_cons(PrimVar{rho, uy, 0.0, 0.0, p_in, t});
            for (int gi = 0; gi < ng; ++gi) u[mesh.idx_raw(gi, jr, kr)] = cons;
        }
    }
}

// zero_rhs_system, crates/cfd_solver/src/lib.rs:86-88
void Case::zero_rhs_system() { std::fill(rhs.begin(), rhs.end(), ConsVar()); }

bool Case::reconstructs(size_t c) const {
    int r[3];
    mesh.raw_coords(c, r);
    if (mesh.is_local_raw(r)) return true;
    if (prm.periodic_seam != EFVM_SEAM_TRUE_PERIODIC) return false;
    int ghost_axes = 0, seam_axis = -1;
    for (int a = 0; a < 3; ++a) {
        if (r[a] >= mesh.ng && r[a] < mesh.n[a] + mesh.ng) continue;
        ++ghost_axes;
        seam_axis = a;
        if (!(r[a] == mesh.ng - 1 || r[a] == mesh.n[a] + mesh.ng)) return false;  // first ghost layer only
    }
    return ghost_axes == 1 && mesh.periodic[seam_axis];
}

// compute_slopes_system, crates/cfd_solver/src/lib.rs:233-268
void Case::compute_slopes_system() {
    const size_t n = mesh.n_raw();
    const size_t off[3] = {1, (size_t)mesh.N[0], (size_t)mesh.N[0] * mesh.N[1]};
#pragma omp parallel for schedule(static) if (colored)
    for (long long cc = 0; cc < (long long)n; ++cc) {
        const size_t c = (size_t)cc;
        if (!reconstructs(c)) {
            for (int a = 0; a < 3; ++a) slopes[3 * c + a] = ConsVar();
            continue;
        }
        const ConsVar u_self = u[c];
        for (int a = 0; a < 3; ++a) {
            // neighbor_mean of one neighbour, :217-226
            const ConsVar up = (ConsVar() + u[c + off[a]]) * (1.0 / 1.0);
            const ConsVar un = (ConsVar() + u[c - off[a]]) * (1.0 / 1.0);
            slopes[3 * c + a] = limited_slope_cons(up - u_self, u_self - un, prm.limiter);
        }
    }
}

// reconstruct_to_face, crates/cfd_solver/src/lib.rs:273-286
static inline ConsVar reconstruct_to_face(const ConsVar& u_self, const ConsVar* slope, const double fc[3],
                                          const double cc[3]) {
    ConsVar uu = u_self;
    for (int a = 0; a < 3; ++a) {
        const double frac = fc[a] > cc[a] ? 0.5 : (fc[a] < cc[a] ? -0.5 : 0.0);
        uu += slope[a] * frac;
    }
    return uu;
}

// Visit every face; the OpenMP build colours the faces so no two faces of one
// parallel sweep share a cell (same faces and arithmetic, other order).
template <class F>
static void visit_faces(const Case& cs, F&& f) {
    if (!cs.colored) {
        cs.mesh.for_each_face(f);
        return;
    }
    const Mesh& m = cs.mesh;
    for (int a = 0; a < 3; ++a) {
        const int b = (a + 1) % 3, c = (a + 2) % 3;
        for (int parity = 0; parity < 2; ++parity) {
            const long long lines = (long long)m.n[b] * m.n[c];
#pragma omp parallel for schedule(static)
            for (long long l = 0; l < lines; ++l) {
                int coord[3];
                coord[b] = (int)(l % m.n[b]);
                coord[c] = (int)(l / m.n[b]);
                for (int ia = parity; ia < m.n[a]; ia += 2) {
                    coord[a] = ia;
                    int r[3] = {coord[0] + m.ng, coord[1] + m.ng, coord[2] + m.ng};
                    const size_t cell = m.idx_raw(r[0], r[1], r[2]);
                    double cc[3] = {m.centroid_axis(0, r[0]), m.centroid_axis(1, r[1]), m.centroid_axis(2, r[2])};
                    int off[3] = {0, 0, 0};
                    off[a] = 1;
                    const double area = m.face_area(a);
                    if (ia == 0) {
                        Face fc;
                        fc.owner = cell; fc.other = m.idx_raw(r[0] - off[0], r[1] - off[1], r[2] - off[2]);
                        fc.axis = a; fc.sign = -1.0; fc.area = area;
                        for (int d = 0; d < 3; ++d) fc.centroid[d] = cc[d];
                        fc.centroid[a] = cc[a] - 0.5 * m.h[a];
                        fc.patch = m.periodic[a] ? -1 : 2 * a;
                        f(fc);
                    }
                    Face fc;
                    fc.owner = cell; fc.other = m.idx_raw(r[0] + off[0], r[1] + off[1], r[2] + off[2]);
                    fc.axis = a; fc.sign = 1.0; fc.area = area;
                    for (int d = 0; d < 3; ++d) fc.centroid[d] = cc[d];
                    fc.centroid[a] = cc[a] + 0.5 * m.h[a];
                    fc.patch = (ia + 1 < m.n[a]) ? -1 : (m.periodic[a] ? -1 : 2 * a + 1);
                    f(fc);
                }
            }
        }
    }
}

// flux_system, crates/cfd_solver/src/lib.rs:93-122
void Case::flux_system() {
    const double vol = mesh.cell_volume();
    visit_faces(*this, [&](const Face& f) {
        const double area = f.area;
        if (area == 0.0) return;
        double nhat[3] = {0.0, 0.0, 0.0};
        nhat[f.axis] = f.sign * area / area;
        const ConsVar fn = flux_normal(prm.flux_scheme, u[f.owner], u[f.other], eos, nhat);
        rhs[f.owner] -= fn * (area / vol);
        if (f.patch < 0 && mesh.is_local_cell(f.other)) rhs[f.other] += fn * (area / vol);
    });
}

// muscl_flux_system, crates/cfd_solver/src/lib.rs:293-339
void Case::muscl_flux_system() {
    const double vol = mesh.cell_volume();
    visit_faces(*this, [&](const Face& f) {
        const double area = f.area;
        if (area == 0.0) return;
        double nhat[3] = {0.0, 0.0, 0.0};
        nhat[f.axis] = f.sign * area / area;
        const bool interior = f.patch < 0;
        double cc[3];
        ConsVar u_l, u_r;
        if (interior) {
            mesh.cell_centroid(f.owner, cc);
            u_l = reconstruct_to_face(u[f.owner], &slopes[3 * f.owner], f.centroid, cc);
        } else {
            u_l = u[f.owner];
        }
        const bool other_local = mesh.is_local_cell(f.other);
        if (interior && reconstructs(f.other)) {
            mesh.cell_centroid(f.other, cc);
            u_r = reconstruct_to_face(u[f.other], &slopes[3 * f.other], f.centroid, cc);
        } else {
            u_r = u[f.other];
        }
        const ConsVar fn = flux_normal(prm.flux_scheme, u_l, u_r, eos, nhat);
        rhs[f.owner] -= fn * (area / vol);
        if (interior && other_local) rhs[f.other] += fn * (area / vol);
    });
}

// d2_pre, crates/cfd_solver/src/lib.rs:451-453
static inline double d2_pre(double um, double uc, double up, double inv_hm, double inv_hp, double inv_hs2) {
    return ((up - uc) * inv_hp - (uc - um) * inv_hm) * inv_hs2;
}

// viscous_system, crates/cfd_solver/src/lib.rs:463-560
void Case::viscous_system() {
    const size_t n = mesh.n_raw();
    std::vector<PrimVar> prim(n);
    for (size_t c = 0; c < n; ++c) prim[c] = eos.cons_to_prim(u[c]);
    const int ni = mesh.n[0], nj = mesh.n[1], nk = mesh.n[2], ng = mesh.ng;
    const double dx = mesh.h[0];
    const double dx_inv2 = 1.0 / (dx * dx);
    std::vector<double> y_im(nj), y_ip(nj), y_is(nj), z_im(nk), z_ip(nk), z_is(nk);
    for (int j = 0; j < nj; ++j) {
        const int jr = j + ng;
        const double hm = mesh.centroid_axis(1, jr) - mesh.centroid_axis(1, jr - 1);
        const double hp = mesh.centroid_axis(1, jr + 1) - mesh.centroid_axis(1, jr);
        y_im[j] = 1.0 / hm; y_ip[j] = 1.0 / hp; y_is[j] = 2.0 / (hm + hp);
    }
    for (int k = 0; k < nk; ++k) {
        const int kr = k + ng;
        const double hm = mesh.centroid_axis(2, kr) - mesh.centroid_axis(2, kr - 1);
        const double hp = mesh.centroid_axis(2, kr + 1) - mesh.centroid_axis(2, kr);
        z_im[k] = 1.0 / hm; z_ip[k] = 1.0 / hp; z_is[k] = 2.0 / (hm + hp);
    }
    const bool have_mask = ibm;
    auto is_solid = [&](size_t c) { return have_mask && solid[c]; };
    struct Nb { double u, v, w, t; };
    auto nb = [&](size_t c, double self_t) -> Nb {
        if (is_solid(c)) return {0.0, 0.0, 0.0, self_t};
        const PrimVar& p = prim[c];
        return {p.u, p.v, p.w, p.t};
    };
    const size_t sx = 1, sy = (size_t)mesh.N[0], sz = (size_t)mesh.N[0] * mesh.N[1];
#pragma omp parallel for schedule(static) if (colored)
    for (int kj = 0; kj < nk * nj; ++kj) {
        const int k = kj / nj, j = kj % nj;
        const int kr = k + ng, jr = j + ng;
        for (int i = 0; i < ni; ++i) {
            const int ir = i + ng;
            const size_t c = mesh.idx_raw(ir, jr, kr);
            if (is_solid(c)) continue;
            const PrimVar ps = prim[c];
            const double mu = visc.mu(ps.t);
            const double kappa = thermal_conductivity(mu, eos.gamma, eos.r_gas);
            const Nb xp = nb(c + sx, ps.t), xm = nb(c - sx, ps.t);
            const Nb yp = nb(c + sy, ps.t), ym = nb(c - sy, ps.t);
            const Nb zp = nb(c + sz, ps.t), zm = nb(c - sz, ps.t);
            const double vel[3] = {ps.u, ps.v, ps.w};
            auto d2_x = [&](double xm_c, double xp_c, double vc) { return (xp_c - 2.0 * vc + xm_c) * dx_inv2; };
            auto d2_y = [&](double ym_c, double yp_c, double vc) { return d2_pre(ym_c, vc, yp_c, y_im[j], y_ip[j], y_is[j]); };
            auto d2_z = [&](double zm_c, double zp_c, double vc) { return d2_pre(zm_c, vc, zp_c, z_im[k], z_ip[k], z_is[k]); };
            const double visc_fx = mu * (d2_x(xm.u, xp.u, vel[0]) + d2_y(ym.u, yp.u, vel[0]) + d2_z(zm.u, zp.u, vel[0]));
            const double visc_fy = mu * (d2_x(xm.v, xp.v, vel[1]) + d2_y(ym.v, yp.v, vel[1]) + d2_z(zm.v, zp.v, vel[1]));
            const double visc_fz = mu * (d2_x(xm.w, xp.w, vel[2]) + d2_y(ym.w, yp.w, vel[2]) + d2_z(zm.w, zp.w, vel[2]));
            const double d2t = d2_x(xm.t, xp.t, ps.t) + d2_y(ym.t, yp.t, ps.t) + d2_z(zm.t, zp.t, ps.t);
            const double visc_energy = vel[0] * visc_fx + vel[1] * visc_fy + vel[2] * visc_fz + kappa * d2t;
            rhs[c] += ConsVar(0.0, visc_fx, visc_fy, visc_fz, visc_energy);
        }
    }
}

// update_system + Rk3Integrator/EulerIntegrator::substep,
// crates/cfd_solver/src/lib.rs:607-621, crates/cfd_solver/src/integrate.rs:48-101
void Case::update_system() {
    const double dt = ss.dt;
    const long long n = (long long)u.size();
    int next = 0;
    bool completed = true;
    if (prm.integrator == EFVM_INTEGRATOR_EULER) {
#pragma omp parallel for schedule(static) if (colored)
        for (long long c = 0; c < n; ++c) u[c] += rhs[c] * dt;
    } else if (ss.rk_stage == 0) {
        u0 = u;  // CfdState::save_state, crates/cfd_state/src/lib.rs:192-194
#pragma omp parallel for schedule(static) if (colored)
        for (long long c = 0; c < n; ++c) u[c] += rhs[c] * dt;
        next = 1;
        completed = false;
    } else if (ss.rk_stage == 1) {
#pragma omp parallel for schedule(static) if (colored)
        for (long long c = 0; c < n; ++c) u[c] = 0.75 * u0[c] + 0.25 * (u[c] + rhs[c] * dt);
        next = 2;
        completed = false;
    } else {
#pragma omp parallel for schedule(static) if (colored)
        for (long long c = 0; c < n; ++c) u[c] = (1.0 / 3.0) * u0[c] + (2.0 / 3.0) * (u[c] + rhs[c] * dt);
        next = 0;
        completed = true;
    }
    ss.rk_stage = next;
    ss.completed_full_step = completed;
    if (completed) {
        ss.step += 1;
        ss.time += ss.dt;
    }
}

// outlet_sponge_system, examples/cylinder_drag_validation/main.rs:186-229
void Case::outlet_sponge_system() {
    if (ss.rk_stage != 0) return;
    const int ng = mesh.ng;
    const double dt = ss.dt;
    const double x0 = prm.sponge_x_start, x1 = prm.sponge_x_end, sig = prm.sponge_sigma;
    const double um = prm.sponge_u_max, h = prm.sponge_height, rho = prm.sponge_rho, p = prm.sponge_p;
    const double inv_w = 1.0 / (x1 - x0);
    for (int k = 0; k < mesh.n[2]; ++k)
        for (int j = 0; j < mesh.n[1]; ++j)
            for (int i = 0; i < mesh.n[0]; ++i) {
                const int ir = i + ng, jr = j + ng, kr = k + ng;
                const size_t idx = mesh.idx_raw(ir, jr, kr);
                const double cx = mesh.centroid_axis(0, ir), cy = mesh.centroid_axis(1, jr);
                if (cx < x0) continue;
                const double s = std::min(std::max((cx - x0) * inv_w, 0.0), 1.0);
                const double f = std::fmin(sig * s * s * dt, 1.0);
                // a 3-D mesh relaxes toward the uniform freestream (rho, u_max, 0, 0, p),
                // examples/sphere_drag_validation/main.rs:119-160; 2-D toward the parabolic
                // inlet profile, examples/cylinder_drag_validation/main.rs:186-229
                const double uy = mesh.n[2] > 1 ? um : 4.0 * um * cy * (h - cy) / (h * h);
                const ConsVar target = eos.prim_to_cons(PrimVar{rho, uy, 0.0, 0.0, p, p / (rho * R_GAS_AIR)});
                ConsVar& uu = u[idx];
                uu.rho += f * (target.rho - uu.rho);
                uu.rho_u += f * (target.rho_u - uu.rho_u);
                uu.rho_v += f * (target.rho_v - uu.rho_v);
                uu.rho_w += f * (target.rho_w - uu.rho_w);
                uu.rho_e += f * (target.rho_e - uu.rho_e);
            }
}

// body_force_system, crates/cfd_solver/tests/poiseuille_channel_validation.rs:100-118
void Case::body_force_system() {
    const double gx = prm.body_force_x;
    for (int k = 0; k < mesh.n[2]; ++k)
        for (int j = 0; j < mesh.n[1]; ++j)
            for (int i = 0; i < mesh.n[0]; ++i) {
                const size_t c = mesh.idx(i, j, k);
                const double rho = u[c].rho, rho_u = u[c].rho_u;
                rhs[c].rho_u += rho * gx;
                rhs[c].rho_e += gx * rho_u;
            }
}

// ---- IBM (crates/cfd_ibm/src/lib.rs) --------------------------------------

// refresh_cylinder_mask, :155-183
void Case::refresh_cylinder_mask() {
    for (int k = 0; k < mesh.n[2]; ++k)
        for (int j = 0; j < mesh.n[1]; ++j)
            for (int i = 0; i < mesh.n[0]; ++i) {
                const size_t c = mesh.idx(i, j, k);
                double cc[3];
                mesh.cell_centroid(c, cc);
                bool inside = false;
                for (const Cylinder& cy : cyls)
                    if (cy.signed_distance(cc) < 0.0) { inside = true; break; }
                const bool was = solid[c] != 0;
                if (inside && !was) {
                    solid[c] = 1;
                    u[c] = stagnant;
                    rhs[c] = ConsVar();
                } else if (!inside && was) {
                    solid[c] = 0;
                    u[c] = ambient;
                    rhs[c] = ConsVar();
                }
            }
}

// compute_cylinder_ghosts, :187-254
void Case::compute_cylinder_ghosts() {
    ghosts.clear();
    if (cyls.empty()) return;
    const int ng = mesh.ng;
    const size_t sx = 1, sy = (size_t)mesh.N[0], sz = (size_t)mesh.N[0] * mesh.N[1];
    for (int k = 0; k < mesh.n[2]; ++k)
        for (int j = 0; j < mesh.n[1]; ++j)
            for (int i = 0; i < mesh.n[0]; ++i) {
                const size_t c = mesh.idx_raw(i + ng, j + ng, k + ng);
                if (!solid[c]) continue;
                // CylinderIbmPlugin: the six face neighbours; the moving discs'
                // compute_disc_ghosts (examples/dkt_sedimentation/main.rs:175-249): the
                // four in-plane ones
                const size_t nbrs[6] = {c + sx, c - sx, c + sy, c - sy, c + sz, c - sz};
                bool any_fluid = false;
                for (int q = 0; q < (disc_ghost_rule ? 4 : 6); ++q) any_fluid = any_fluid || !solid[nbrs[q]];
                if (!any_fluid) continue;
                IbmGhost gh;
                gh.idx = c;
                mesh.cell_centroid(c, gh.cell_center);
                double best_abs = std::numeric_limits<double>::max(), best_signed = 0.0;
                double best_normal[3] = {1.0, 0.0, 0.0}, best_wall[3] = {0.0, 0.0, 0.0};
                uint32_t best_body = 0;
                for (size_t bid = 0; bid < cyls.size(); ++bid) {
                    const double s = cyls[bid].signed_distance(gh.cell_center);
                    if (std::fabs(s) < best_abs) {
                        best_abs = std::fabs(s);
                        best_signed = s;
                        cyls[bid].normal(gh.cell_center, best_normal);
                        best_body = (uint32_t)bid;
                        // the wall velocity at the cell's wall footprint (compute_disc_ghosts,
                        // examples/dkt_sedimentation/main.rs:175-249; zero for a body at rest)
                        const double foot[3] = {gh.cell_center[0] - s * best_normal[0],
                                                gh.cell_center[1] - s * best_normal[1], gh.cell_center[2]};
                        cyls[bid].wall_velocity(foot, best_wall);
                    }
                }
                const double push = 2.0 * (-best_signed);
                for (int d = 0; d < 3; ++d) {
                    gh.image_point[d] = gh.cell_center[d] + push * best_normal[d];
                    gh.normal[d] = best_normal[d];
                    gh.wall_velocity[d] = best_wall[d];
                }
                gh.body_id = best_body;
                ghosts.push_back(gh);
            }
}

// compute_cylinder_markers, :566-598
void Case::compute_cylinder_markers() {
    markers.clear();
    if (cyls.empty()) return;
    const int nk = mesh.n[2], ng = mesh.ng;
    const double z_lo = mesh.centroid_axis(2, ng) - 0.5 * mesh.h[2];
    const double z_hi = mesh.centroid_axis(2, ng + nk - 1) + 0.5 * mesh.h[2];
    const double lz = z_hi - z_lo;
    const int n_theta = cylinder_markers_n, n_z = std::max(nk, 1);
    for (size_t bid = 0; bid < cyls.size(); ++bid) {
        const Cylinder& cy = cyls[bid];
        const double area = 2.0 * PI * cy.r * lz / (double)(n_theta * n_z);
        for (int it = 0; it < n_theta; ++it) {
            const double theta = 2.0 * PI * ((double)it + 0.5) / (double)n_theta;
            const double nx = std::cos(theta), ny = std::sin(theta);
            for (int iz = 0; iz < n_z; ++iz) {
                const double z = z_lo + ((double)iz + 0.5) * lz / (double)n_z;
                IbmMarker m;
                m.body_id = (uint32_t)bid;
                m.position[0] = cy.cx + cy.r * nx;
                m.position[1] = cy.cy + cy.r * ny;
                m.position[2] = z;
                m.normal[0] = nx; m.normal[1] = ny; m.normal[2] = 0.0;
                m.area = area;
                cy.wall_velocity(m.position, m.wall_velocity);
                markers.push_back(m);
            }
        }
    }
}

// refresh_sphere_mask, crates/cfd_ibm/src/sphere.rs:81-111
void Case::refresh_sphere_mask() {
    for (int k = 0; k < mesh.n[2]; ++k)
        for (int j = 0; j < mesh.n[1]; ++j)
            for (int i = 0; i < mesh.n[0]; ++i) {
                const size_t c = mesh.idx(i, j, k);
                double cc[3];
                mesh.cell_centroid(c, cc);
                bool inside = false;
                for (const Sphere& b : spheres)
                    if (b.signed_distance(cc) < 0.0) { inside = true; break; }
                const bool was = solid[c] != 0;
                if (inside && !was) {
                    solid[c] = 1;
                    u[c] = stagnant;
                    rhs[c] = ConsVar();
                } else if (!inside && was) {
                    solid[c] = 0;
                    u[c] = ambient;
                    rhs[c] = ConsVar();
                }
            }
}

// compute_sphere_ghosts, crates/cfd_ibm/src/sphere.rs:116-195
void Case::compute_sphere_ghosts() {
    ghosts.clear();
    if (spheres.empty()) return;
    const int ng = mesh.ng;
    const size_t sx = 1, sy = (size_t)mesh.N[0], sz = (size_t)mesh.N[0] * mesh.N[1];
    for (int k = 0; k < mesh.n[2]; ++k)
        for (int j = 0; j < mesh.n[1]; ++j)
            for (int i = 0; i < mesh.n[0]; ++i) {
                const size_t c = mesh.idx_raw(i + ng, j + ng, k + ng);
                if (!solid[c]) continue;
                const size_t nbrs[6] = {c + sx, c - sx, c + sy, c - sy, c + sz, c - sz};
                bool any_fluid = false;
                for (size_t nbi : nbrs) any_fluid = any_fluid || !solid[nbi];
                if (!any_fluid) continue;
                IbmGhost gh;
                gh.idx = c;
                mesh.cell_centroid(c, gh.cell_center);
                double best_abs = std::numeric_limits<double>::max(), best_signed = 0.0;
                double best_normal[3] = {1.0, 0.0, 0.0}, best_wall[3] = {0.0, 0.0, 0.0};
                uint32_t best_body = 0;
                for (size_t bid = 0; bid < spheres.size(); ++bid) {
                    const double sd = spheres[bid].signed_distance(gh.cell_center);
                    if (std::fabs(sd) < best_abs) {
                        best_abs = std::fabs(sd);
                        best_signed = sd;
                        spheres[bid].normal(gh.cell_center, best_normal);
                        best_body = (uint32_t)bid;
                        // the body's surface velocity at the cell's wall footprint
                        const double foot[3] = {gh.cell_center[0] - sd * best_normal[0],
                                                gh.cell_center[1] - sd * best_normal[1],
                                                gh.cell_center[2] - sd * best_normal[2]};
                        spheres[bid].wall_velocity(foot, best_wall);
                    }
                }
                const double push = 2.0 * (-best_signed);
                for (int d = 0; d < 3; ++d) {
                    gh.image_point[d] = gh.cell_center[d] + push * best_normal[d];
                    gh.normal[d] = best_normal[d];
                    gh.wall_velocity[d] = best_wall[d];
                }
                gh.body_id = best_body;
                ghosts.push_back(gh);
            }
}

// compute_sphere_markers + sphere_markers, crates/cfd_ibm/src/sphere.rs:201-245:
// the golden-angle spherical Fibonacci lattice, area 4 pi R^2 / n per marker.
void Case::compute_sphere_markers() {
    markers.clear();
    if (spheres.empty()) return;
    const int n = std::max(sphere_markers_n, 12);
    const double golden = PI * (3.0 - std::sqrt(5.0));
    for (size_t bid = 0; bid < spheres.size(); ++bid) {
        const Sphere& b = spheres[bid];
        const double area = 4.0 * PI * b.r * b.r / (double)n;
        for (int m = 0; m < n; ++m) {
            const double zr = 1.0 - 2.0 * ((double)m + 0.5) / (double)n;
            const double rr = std::sqrt(std::max(1.0 - zr * zr, 0.0));
            const double phi = golden * (double)m;
            const double dir[3] = {rr * std::cos(phi), rr * std::sin(phi), zr};
            IbmMarker mk;
            mk.body_id = (uint32_t)bid;
            for (int d = 0; d < 3; ++d) {
                mk.position[d] = b.c[d] + b.r * dir[d];
                mk.normal[d] = dir[d];
            }
            mk.area = area;
            b.wall_velocity(mk.position, mk.wall_velocity);
            markers.push_back(mk);
        }
    }
}

void Case::geometry_systems() {
    if (!spheres.empty()) {
        refresh_sphere_mask();
        compute_sphere_ghosts();
        compute_sphere_markers();
    } else {
        refresh_cylinder_mask();
        compute_cylinder_ghosts();
        compute_cylinder_markers();
    }
}

// sample_trilinear, :106-149
bool Case::sample_trilinear(const double point[3], PrimVar& out) const {
    size_t lo_idx;
    int lo[3];
    double t[3];
    if (!mesh.locate(point, lo_idx, lo, t)) return false;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    double total_w = 0.0;
    for (int di = 0; di < 2; ++di) {
        const double wx = di == 0 ? 1.0 - t[0] : t[0];
        for (int dj = 0; dj < 2; ++dj) {
            const double wy = dj == 0 ? 1.0 - t[1] : t[1];
            for (int dk = 0; dk < 2; ++dk) {
                const double wz = dk == 0 ? 1.0 - t[2] : t[2];
                const size_t c = mesh.idx_raw(lo[0] + di, lo[1] + dj, lo[2] + dk);
                if (solid[c]) continue;
                const ConsVar& uc = u[c];
                if (!std::isfinite(uc.rho) || uc.rho <= 0.0) continue;
                const double w = wx * wy * wz;
                const PrimVar p = eos.cons_to_prim(uc);
                acc[0] += w * p.rho;
                acc[1] += w * p.u;
                acc[2] += w * p.v;
                acc[3] += w * p.w;
                acc[4] += w * p.p;
                acc[5] += w * p.t;
                total_w += w;
            }
        }
    }
    if (total_w < 1e-12) return false;
    const double inv = 1.0 / total_w;
    out = PrimVar{acc[0] * inv, acc[1] * inv, acc[2] * inv, acc[3] * inv, acc[4] * inv, acc[5] * inv};
    return true;
}

// apply_ibm_ghost_bc, :258-289
void Case::apply_ibm_ghost_bc() {
    if (ghosts.empty()) return;
    for (const IbmGhost& g : ghosts) {
        PrimVar image;
        if (!sample_trilinear(g.image_point, image)) continue;
        const double* uw = g.wall_velocity;
        const PrimVar mirrored{image.rho, 2.0 * uw[0] - image.u, 2.0 * uw[1] - image.v, 2.0 * uw[2] - image.w,
                               image.p, image.t};
        u[g.idx] = eos.prim_to_cons(mirrored);
    }
}

// zero_solid_rhs, :293-301
void Case::zero_solid_rhs() {
    for (size_t c = 0; c < solid.size(); ++c)
        if (solid[c]) rhs[c] = ConsVar();
}

// marker_force_system + compute_marker_loadings, :442-480,601-615
void Case::marker_force_system() {
    const double sample_offset = mesh.h[0];
    double fp[3] = {0, 0, 0}, fv[3] = {0, 0, 0};
    for (const IbmMarker& m : markers) {
        const double sp[3] = {m.position[0] + sample_offset * m.normal[0], m.position[1] + sample_offset * m.normal[1],
                              m.position[2] + sample_offset * m.normal[2]};
        PrimVar img;
        if (!sample_trilinear(sp, img)) continue;
        if (!(std::isfinite(img.p) && std::isfinite(img.t) && std::isfinite(img.u) && std::isfinite(img.v) &&
              std::isfinite(img.w)))
            continue;
        const double us[3] = {img.u - m.wall_velocity[0], img.v - m.wall_velocity[1], img.w - m.wall_velocity[2]};
        const double udotn = us[0] * m.normal[0] + us[1] * m.normal[1] + us[2] * m.normal[2];
        const double mu = visc.mu(img.t);
        for (int d = 0; d < 3; ++d) {
            const double ut = us[d] - udotn * m.normal[d];
            fp[d] += -img.p * m.normal[d] * m.area;
            fv[d] += mu * ut / sample_offset * m.area;
        }
    }
    for (int d = 0; d < 3; ++d) { marker_force[d] = fp[d]; marker_force[3 + d] = fv[d]; }
}

// wall_force_system + compute_wall_forces, :309-395
void Case::wall_force_system() {
    double f_p[3] = {0, 0, 0}, f_v[3] = {0, 0, 0};
    const int ng = mesh.ng;
    const size_t sx = 1, sy = (size_t)mesh.N[0], sz = (size_t)mesh.N[0] * mesh.N[1];
    const double dx = mesh.h[0], dy = mesh.h[1], dz = mesh.h[2];
    const double face_area[3] = {dy * dz, dx * dz, dx * dy};
    const double dn[3] = {dx, dy, dz};
    for (int k = 0; k < mesh.n[2]; ++k)
        for (int j = 0; j < mesh.n[1]; ++j)
            for (int i = 0; i < mesh.n[0]; ++i) {
                const size_t c = mesh.idx_raw(i + ng, j + ng, k + ng);
                if (!solid[c]) continue;
                const struct { size_t nbr; int dim; double sign; } nbrs[6] = {
                    {c + sx, 0, 1.0}, {c - sx, 0, -1.0}, {c + sy, 1, 1.0},
                    {c - sy, 1, -1.0}, {c + sz, 2, 1.0}, {c - sz, 2, -1.0}};
                for (const auto& nb : nbrs) {
                    if (solid[nb.nbr]) continue;
                    const ConsVar& uc = u[nb.nbr];
                    f_p[nb.dim] -= eos.pressure(uc) * nb.sign * face_area[nb.dim];
                    const PrimVar prim = eos.cons_to_prim(uc);
                    const double mu = visc.mu(prim.t);
                    const double vel[3] = {prim.u, prim.v, prim.w};
                    for (int td = 0; td < 3; ++td)
                        if (td != nb.dim) f_v[td] += mu * vel[td] / (0.5 * dn[nb.dim]) * face_area[nb.dim];
                }
            }
    for (int d = 0; d < 3; ++d) { wall_force[d] = f_p[d]; wall_force[3 + d] = f_v[d]; }
}

// One app.run(): every phase of MeshScheduleSet in order (crates/cfd_solver/src/
// lib.rs:919-940, crates/cfd_ibm/src/lib.rs:623-673, and the case-local systems
// of examples/cylinder_drag_validation/main.rs:304-315).
void Case::substep() {
    // Setup: cfl_system (SolverPlugin) then the cylinder geometry (CylinderIbmPlugin)
    cfl_system();
    if (ibm) geometry_systems();
    // Halo
    halo_system();
    // Boundary: the stock fill, then the case's parabolic inlet
    boundary_system();
    if (prm.parabolic_inflow) parabolic_inflow_system();
    // PreFlux: zero rhs; the IBM mirror and the MUSCL slope pass
    zero_rhs_system();
    const bool muscl = prm.reconstruction == EFVM_RECON_MUSCL;
    if (muscl && slopes_before_ibm) compute_slopes_system();
    if (ibm) apply_ibm_ghost_bc();
    if (muscl && !slopes_before_ibm) compute_slopes_system();
    // Flux: inviscid sweep, then viscous terms
    if (muscl) muscl_flux_system();
    else flux_system();
    if (prm.viscous) viscous_system();
    // PostFlux
    if (ibm) zero_solid_rhs();
    if (prm.body_force_x != 0.0) body_force_system();
    // Update
    update_system();
    // PostUpdate
    if (prm.sponge) outlet_sponge_system();
    // Output
    if (ibm) {
        marker_force_system();
        wall_force_system();
    }
}

}  // namespace oracle

// ===========================================================================
// C API for ctypes (tests and the CPU baseline only)
// ===========================================================================
using namespace oracle;

struct OracleHandle {
    Case cs;
    std::string err;
};

static thread_local std::string g_create_error;

extern "C" {

const char* oracle_create_error(void) { return g_create_error.c_str(); }

void* oracle_create(const efvm_grid* g, const efvm_params* p) {
    if (!g || !p) { g_create_error = "null argument"; return nullptr; }
    OracleHandle* h = new OracleHandle();
    const char* err = nullptr;
    if (!h->cs.setup(*g, *p, &err)) {
        g_create_error = err ? err : "invalid configuration";
        delete h;
        return nullptr;
    }
#ifdef _OPENMP
    h->cs.colored = true;
#endif
    return h;
}

void oracle_destroy(void* hp) { delete (OracleHandle*)hp; }

int oracle_is_parallel(void) {
#ifdef _OPENMP
    return 1;
#else
    return 0;
#endif
}

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int oracle_set_option(void* hp, const char* name, double value) {
    OracleHandle* h = (OracleHandle*)hp;
    const std::string n(name);
    if (n == "slopes_before_ibm") h->cs.slopes_before_ibm = value != 0.0;
    else if (n == "colored") h->cs.colored = value != 0.0;
    else return EFVM_ERR_INVALID_ARG;
    return EFVM_OK;
}

// Interior upload; ghosts get the nearest interior value so nothing is unset.
int oracle_upload_state(void* hp, const double* base, int64_t si, int64_t sj, int64_t sv) {
    Case& cs = ((OracleHandle*)hp)->cs;
    const Mesh& m = cs.mesh;
    for (int k = 0; k < m.N[2]; ++k)
        for (int j = 0; j < m.N[1]; ++j)
            for (int i = 0; i < m.N[0]; ++i) {
                const int ii = std::min(std::max(i - m.ng, 0), m.n[0] - 1);
                const int jj = std::min(std::max(j - m.ng, 0), m.n[1] - 1);
                const double* e = base + ii * si + jj * sj;
                cs.u[m.idx_raw(i, j, k)] = ConsVar(e[0], e[sv], e[2 * sv], e[3 * sv], e[4 * sv]);
            }
    return EFVM_OK;
}

int oracle_download_state(void* hp, double* base, int64_t si, int64_t sj, int64_t sv) {
    Case& cs = ((OracleHandle*)hp)->cs;
    const Mesh& m = cs.mesh;
    for (int j = 0; j < m.n[1]; ++j)
        for (int i = 0; i < m.n[0]; ++i) {
            const ConsVar& c = cs.u[m.idx(i, j, 0)];
            double* e = base + i * si + j * sj;
            e[0] = c.rho; e[sv] = c.rho_u; e[2 * sv] = c.rho_v; e[3 * sv] = c.rho_w; e[4 * sv] = c.rho_e;
        }
    return EFVM_OK;
}

// 3-D forms: element (i, j, k, v) at i si + j sj + k sk + v sv over all layers.
int oracle_upload_state3(void* hp, const double* base, int64_t si, int64_t sj, int64_t sk, int64_t sv) {
    Case& cs = ((OracleHandle*)hp)->cs;
    const Mesh& m = cs.mesh;
    for (int k = 0; k < m.N[2]; ++k)
        for (int j = 0; j < m.N[1]; ++j)
            for (int i = 0; i < m.N[0]; ++i) {
                const int ii = std::min(std::max(i - m.ng, 0), m.n[0] - 1);
                const int jj = std::min(std::max(j - m.ng, 0), m.n[1] - 1);
                const int kk = std::min(std::max(k - m.ng, 0), m.n[2] - 1);
                const double* e = base + ii * si + jj * sj + kk * sk;
                cs.u[m.idx_raw(i, j, k)] = ConsVar(e[0], e[sv], e[2 * sv], e[3 * sv], e[4 * sv]);
            }
    return EFVM_OK;
}

int oracle_download_state3(void* hp, double* base, int64_t si, int64_t sj, int64_t sk, int64_t sv) {
    Case& cs = ((OracleHandle*)hp)->cs;
    const Mesh& m = cs.mesh;
    for (int k = 0; k < m.n[2]; ++k)
        for (int j = 0; j < m.n[1]; ++j)
            for (int i = 0; i < m.n[0]; ++i) {
                const ConsVar& c = cs.u[m.idx(i, j, k)];
                double* e = base + i * si + j * sj + k * sk;
                e[0] = c.rho; e[sv] = c.rho_u; e[2 * sv] = c.rho_v; e[3 * sv] = c.rho_w; e[4 * sv] = c.rho_e;
            }
    return EFVM_OK;
}

// Full raw array (all layers, 5 doubles per cell, FIELD raw order).
int64_t oracle_raw_size(void* hp) { return (int64_t)((OracleHandle*)hp)->cs.mesh.n_raw(); }
int oracle_get_raw_state(void* hp, double* out) {
    Case& cs = ((OracleHandle*)hp)->cs;
    for (size_t c = 0; c < cs.u.size(); ++c) {
        const ConsVar& v = cs.u[c];
        out[5 * c] = v.rho; out[5 * c + 1] = v.rho_u; out[5 * c + 2] = v.rho_v; out[5 * c + 3] = v.rho_w; out[5 * c + 4] = v.rho_e;
    }
    return EFVM_OK;
}
int oracle_set_raw_state(void* hp, const double* in) {
    Case& cs = ((OracleHandle*)hp)->cs;
    for (size_t c = 0; c < cs.u.size(); ++c)
        cs.u[c] = ConsVar(in[5 * c], in[5 * c + 1], in[5 * c + 2], in[5 * c + 3], in[5 * c + 4]);
    return EFVM_OK;
}

// The reference's vortex_state closure (crates/cfd_solver/tests/
// isentropic_vortex_muscl_convergence.rs:48-64) with a minimum-image option.
static double vortex_rho(const efvm_vortex& v, double t, const double x[3], ConsVar* out_cons) {
    const IdealGas eos{v.gamma, 1.0};
    double cx = v.cx0 + v.mean_u * t;
    double cy = v.cy0 + v.mean_v * t;
    double dx = x[0] - cx, dy = x[1] - cy;
    if (v.min_image) {
        dx = dx - v.len_x * std::round(dx / v.len_x);
        dy = dy - v.len_y * std::round(dy / v.len_y);
    }
    const double r2 = dx * dx + dy * dy;
    const double f = std::exp(0.5 * (1.0 - r2));
    const double du = -v.beta / (2.0 * PI) * dy * f;
    const double dv = v.beta / (2.0 * PI) * dx * f;
    const double dtemp = -(v.gamma - 1.0) * v.beta * v.beta / (8.0 * v.gamma * std::pow(PI, 2)) * std::exp(1.0 - r2);
    const double temp = 1.0 + dtemp;
    const double rho = std::pow(temp, 1.0 / (v.gamma - 1.0));
    const double p = std::pow(rho, v.gamma);
    if (out_cons) *out_cons = eos.prim_to_cons(PrimVar{rho, v.mean_u + du, v.mean_v + dv, 0.0, p, temp});
    return rho;
}

// init_state_system semantics: every raw cell from its centroid.
int oracle_init_vortex(void* hp, const efvm_vortex* v) {
    Case& cs = ((OracleHandle*)hp)->cs;
    for (size_t c = 0; c < cs.u.size(); ++c) {
        double x[3];
        cs.mesh.cell_centroid(c, x);
        vortex_rho(*v, 0.0, x, &cs.u[c]);
    }
    return EFVM_OK;
}

int oracle_vortex_state(const efvm_vortex* v, double t, const double x[3], double out[5]) {
    ConsVar c;
    vortex_rho(*v, t, x, &c);
    out[0] = c.rho; out[1] = c.rho_u; out[2] = c.rho_v; out[3] = c.rho_w; out[4] = c.rho_e;
    return EFVM_OK;
}

int oracle_density_error(void* hp, const efvm_vortex* v, double out[2]) {
    Case& cs = ((OracleHandle*)hp)->cs;
    const Mesh& m = cs.mesh;
    const double t = cs.ss.time;
    double num = 0.0, vol = 0.0, linf = 0.0;
    for (int j = 0; j < m.n[1]; ++j)
        for (int i = 0; i < m.n[0]; ++i) {
            const size_t c = m.idx(i, j, 0);
            double x[3];
            m.cell_centroid(c, x);
            const double ex = vortex_rho(*v, t, x, nullptr);
            const double cv = m.cell_volume();
            const double e = std::fabs(cs.u[c].rho - ex);
            num += e * cv;
            vol += cv;
            linf = std::fmax(linf, e);
        }
    out[0] = num / vol;
    out[1] = linf;
    return EFVM_OK;
}

int oracle_total_mass(void* hp, double* out) {
    Case& cs = ((OracleHandle*)hp)->cs;
    const Mesh& m = cs.mesh;
    double s = 0.0;
    for (size_t c = 0; c < cs.u.size(); ++c)
        if (m.is_local_cell(c)) s += cs.u[c].rho * m.cell_volume();
    *out = s;
    return EFVM_OK;
}

int oracle_substep(void* hp) {
    ((OracleHandle*)hp)->cs.substep();
    return EFVM_OK;
}

int oracle_step(void* hp, int64_t n_steps, int32_t stop_at_t, double t_stop, double* force_history,
                efvm_step_info* info) {
    Case& cs = ((OracleHandle*)hp)->cs;
    if (cs.ss.rk_stage != 0) return EFVM_ERR_INVALID_ARG;
    const int subs = cs.prm.integrator == EFVM_INTEGRATOR_EULER ? 1 : 3;
    int64_t done = 0, sub_done = 0;
    int stopped = 0;
    for (int64_t s = 0; s < n_steps; ++s) {
        if (stop_at_t && cs.ss.time >= t_stop) { stopped = 1; break; }
        for (int k = 0; k < subs; ++k) {
            cs.substep();
            if (force_history) for (int d = 0; d < 6; ++d) force_history[6 * sub_done + d] = cs.marker_force[d];
            ++sub_done;
        }
        ++done;
    }
    if (stop_at_t && !stopped && cs.ss.time >= t_stop) stopped = 1;
    if (info) {
        info->steps_done = done;
        info->substeps_done = sub_done;
        info->time = cs.ss.time;
        info->dt = cs.ss.dt;
        info->stopped_at_t_stop = stopped;
    }
    return EFVM_OK;
}

int oracle_cfl(void* hp, double* dt) {
    Case& cs = ((OracleHandle*)hp)->cs;
    *dt = cs.prm.fixed_dt > 0.0 ? cs.prm.fixed_dt : cs.cfl_dt();
    return EFVM_OK;
}

int oracle_get_solver_state(void* hp, efvm_solver_state* out) {
    Case& cs = ((OracleHandle*)hp)->cs;
    out->dt = cs.ss.dt;
    out->time = cs.ss.time;
    out->step = cs.ss.step;
    out->rk_stage = cs.ss.rk_stage;
    out->completed_full_step = cs.ss.completed_full_step ? 1 : 0;
    return EFVM_OK;
}

int oracle_set_solver_state(void* hp, const efvm_solver_state* in) {
    Case& cs = ((OracleHandle*)hp)->cs;
    cs.ss.dt = in->dt;
    cs.ss.time = in->time;
    cs.ss.step = in->step;
    cs.ss.rk_stage = in->rk_stage;
    cs.ss.completed_full_step = in->completed_full_step != 0;
    return EFVM_OK;
}

int oracle_set_cylinders(void* hp, const efvm_cylinder* c, int32_t n, const double fs[5]);

// The moving discs of examples/dkt_sedimentation/main.rs (n_theta markers per disc).
int oracle_set_discs(void* hp, const efvm_disc* d, int32_t n, int32_t n_theta, const double fs[5]) {
    std::vector<efvm_cylinder> c((size_t)n);
    for (int i = 0; i < n; ++i) c[i] = efvm_cylinder{d[i].cx, d[i].cy, d[i].radius};
    const int rc = oracle_set_cylinders(hp, c.data(), n, fs);
    Case& cs = ((OracleHandle*)hp)->cs;
    for (int i = 0; i < n; ++i) {
        cs.cyls[i].vx = d[i].vx;
        cs.cyls[i].vy = d[i].vy;
        cs.cyls[i].omega = d[i].omega;
    }
    cs.cylinder_markers_n = n_theta;
    cs.disc_ghost_rule = true;
    return rc;
}

int oracle_set_cylinders(void* hp, const efvm_cylinder* c, int32_t n, const double fs[5]) {
    Case& cs = ((OracleHandle*)hp)->cs;
    cs.cyls.clear();
    cs.cylinder_markers_n = 64;
    cs.disc_ghost_rule = false;
    for (int i = 0; i < n; ++i) cs.cyls.push_back(Cylinder{c[i].cx, c[i].cy, c[i].radius});
    const ConsVar f(fs[0], fs[1], fs[2], fs[3], fs[4]);
    // CylinderIbmPlugin::build, crates/cfd_ibm/src/lib.rs:665-669
    cs.stagnant = ConsVar(f.rho, 0.0, 0.0, 0.0, f.rho_e - f.kinetic_energy());
    cs.ambient = f;
    cs.ibm = true;
    return EFVM_OK;
}

// SphereIbmPlugin::new(bodies, freestream).with_markers(n_markers),
// crates/cfd_ibm/src/sphere.rs:262-286: the bodies replace any earlier ones
// (an FSI driver moves them between steps this way).
int oracle_set_spheres(void* hp, const efvm_sphere* s, int32_t n, int32_t n_markers, const double fs[5]) {
    Case& cs = ((OracleHandle*)hp)->cs;
    cs.spheres.clear();
    for (int i = 0; i < n; ++i)
        cs.spheres.push_back(Sphere{{s[i].cx, s[i].cy, s[i].cz}, s[i].radius, {s[i].vx, s[i].vy, s[i].vz},
                                    {s[i].wx, s[i].wy, s[i].wz}});
    cs.sphere_markers_n = n_markers;
    const ConsVar f(fs[0], fs[1], fs[2], fs[3], fs[4]);
    cs.stagnant = ConsVar(f.rho, 0.0, 0.0, 0.0, f.rho_e - f.kinetic_energy());
    cs.ambient = f;
    cs.ibm = true;
    return EFVM_OK;
}

// The markers compute_sphere_markers places for one sphere (test access to the
// lattice): per marker position[3], normal[3], area, wall_velocity[3] (10 doubles).
int oracle_sphere_markers(const efvm_sphere* s, int32_t n_markers, double* out) {
    Case cs;
    cs.spheres.push_back(Sphere{{s->cx, s->cy, s->cz}, s->radius, {s->vx, s->vy, s->vz}, {s->wx, s->wy, s->wz}});
    cs.sphere_markers_n = n_markers;
    cs.compute_sphere_markers();
    for (size_t m = 0; m < cs.markers.size(); ++m) {
        double* o = out + 10 * m;
        for (int d = 0; d < 3; ++d) {
            o[d] = cs.markers[m].position[d];
            o[3 + d] = cs.markers[m].normal[d];
            o[7 + d] = cs.markers[m].wall_velocity[d];
        }
        o[6] = cs.markers[m].area;
    }
    return (int)cs.markers.size();
}

// The Setup-phase geometry systems alone (refresh_cylinder_mask,
// compute_cylinder_ghosts, compute_cylinder_markers; crates/cfd_ibm/src/lib.rs:155-254,566-598),
// as a freshly prepared App runs them before a restore overwrites its fields.
int oracle_apply_geometry(void* hp) {
    Case& cs = ((OracleHandle*)hp)->cs;
    if (cs.ibm) cs.geometry_systems();
    return EFVM_OK;
}

// compute_marker_loadings_per_body, crates/cfd_ibm/src/lib.rs:509-562: per body
// pressure and viscous force and the torque about the body centre, from the
// current state; out[9 b ..] = pressure[3], viscous[3], torque[3].  The centre of
// a cylinder is (cx, cy) at the z of its markers (the z-cell centre).
int oracle_body_loads(void* hp, int32_t n_bodies, double* out) {
    Case& cs = ((OracleHandle*)hp)->cs;
    for (int q = 0; q < 9 * n_bodies; ++q) out[q] = 0.0;
    const double sample_offset = cs.mesh.h[0];
    for (const IbmMarker& m : cs.markers) {
        const int b = (int)m.body_id;
        if (b >= n_bodies || b >= (int)cs.cyls.size()) continue;
        const double sp[3] = {m.position[0] + sample_offset * m.normal[0], m.position[1] + sample_offset * m.normal[1],
                              m.position[2] + sample_offset * m.normal[2]};
        PrimVar img;
        if (!cs.sample_trilinear(sp, img)) continue;
        if (!(std::isfinite(img.p) && std::isfinite(img.t) && std::isfinite(img.u) && std::isfinite(img.v) &&
              std::isfinite(img.w)))
            continue;
        const double us[3] = {img.u - m.wall_velocity[0], img.v - m.wall_velocity[1], img.w - m.wall_velocity[2]};
        const double udotn = us[0] * m.normal[0] + us[1] * m.normal[1] + us[2] * m.normal[2];
        const double mu = cs.visc.mu(img.t);
        double df[3];
        for (int d = 0; d < 3; ++d) {
            const double ut = us[d] - udotn * m.normal[d];
            const double fp = -img.p * m.normal[d] * m.area;
            const double fv = mu * ut / sample_offset * m.area;
            out[9 * b + d] += fp;
            out[9 * b + 3 + d] += fv;
            df[d] = fp + fv;
        }
        const double c[3] = {cs.cyls[b].cx, cs.cyls[b].cy, m.position[2]};
        const double r[3] = {m.position[0] - c[0], m.position[1] - c[1], m.position[2] - c[2]};
        out[9 * b + 6] += r[1] * df[2] - r[2] * df[1];
        out[9 * b + 7] += r[2] * df[0] - r[0] * df[2];
        out[9 * b + 8] += r[0] * df[1] - r[1] * df[0];
    }
    return EFVM_OK;
}

int oracle_marker_force(void* hp, double out[6]) {
    Case& cs = ((OracleHandle*)hp)->cs;
    for (int d = 0; d < 6; ++d) out[d] = cs.marker_force[d];
    return EFVM_OK;
}

int oracle_wall_force(void* hp, double out[6]) {
    Case& cs = ((OracleHandle*)hp)->cs;
    for (int d = 0; d < 6; ++d) out[d] = cs.wall_force[d];
    return EFVM_OK;
}

int oracle_ibm_counts(void* hp, int64_t* n_solid, int64_t* n_ghost) {
    Case& cs = ((OracleHandle*)hp)->cs;
    int64_t s = 0;
    for (uint8_t b : cs.solid) s += b ? 1 : 0;
    *n_solid = s;
    *n_ghost = (int64_t)cs.ghosts.size();
    return EFVM_OK;
}

// Interior solid mask (nx*ny bytes, x fastest) for comparison with the device.
int oracle_get_mask(void* hp, uint8_t* out) {
    Case& cs = ((OracleHandle*)hp)->cs;
    const Mesh& m = cs.mesh;
    for (int j = 0; j < m.n[1]; ++j)
        for (int i = 0; i < m.n[0]; ++i) out[(size_t)j * m.n[0] + i] = cs.solid[m.idx(i, j, 0)];
    return EFVM_OK;
}

// ---- known-answer helpers (single-function restatements) ------------------

int oracle_flux(int scheme, double gamma, double r_gas, const double* l, const double* r, int dir, double* out) {
    const IdealGas eos{gamma, r_gas};
    const ConsVar f = scheme_flux(scheme, ConsVar(l[0], l[1], l[2], l[3], l[4]), ConsVar(r[0], r[1], r[2], r[3], r[4]), eos, dir);
    out[0] = f.rho; out[1] = f.rho_u; out[2] = f.rho_v; out[3] = f.rho_w; out[4] = f.rho_e;
    return EFVM_OK;
}

int oracle_flux_normal(int scheme, double gamma, double r_gas, const double* l, const double* r, const double* n,
                       double* out) {
    const IdealGas eos{gamma, r_gas};
    const ConsVar f = flux_normal(scheme, ConsVar(l[0], l[1], l[2], l[3], l[4]), ConsVar(r[0], r[1], r[2], r[3], r[4]), eos, n);
    out[0] = f.rho; out[1] = f.rho_u; out[2] = f.rho_v; out[3] = f.rho_w; out[4] = f.rho_e;
    return EFVM_OK;
}

int oracle_physical_flux(double gamma, double r_gas, const double* u, int dir, double* out) {
    const IdealGas eos{gamma, r_gas};
    const ConsVar f = physical_flux(ConsVar(u[0], u[1], u[2], u[3], u[4]), eos, dir);
    out[0] = f.rho; out[1] = f.rho_u; out[2] = f.rho_v; out[3] = f.rho_w; out[4] = f.rho_e;
    return EFVM_OK;
}

int oracle_cons_to_prim(double gamma, double r_gas, const double* u, double* out) {
    const IdealGas eos{gamma, r_gas};
    const PrimVar p = eos.cons_to_prim(ConsVar(u[0], u[1], u[2], u[3], u[4]));
    out[0] = p.rho; out[1] = p.u; out[2] = p.v; out[3] = p.w; out[4] = p.p; out[5] = p.t;
    return EFVM_OK;
}

int oracle_prim_to_cons(double gamma, double r_gas, const double* p, double* out) {
    const IdealGas eos{gamma, r_gas};
    const ConsVar c = eos.prim_to_cons(PrimVar{p[0], p[1], p[2], p[3], p[4], p[5]});
    out[0] = c.rho; out[1] = c.rho_u; out[2] = c.rho_v; out[3] = c.rho_w; out[4] = c.rho_e;
    return EFVM_OK;
}

double oracle_sound_speed(double gamma, double r_gas, const double* u) {
    const IdealGas eos{gamma, r_gas};
    return eos.sound_speed(ConsVar(u[0], u[1], u[2], u[3], u[4]));
}

double oracle_pressure(double gamma, double r_gas, const double* u) {
    const IdealGas eos{gamma, r_gas};
    return eos.pressure(ConsVar(u[0], u[1], u[2], u[3], u[4]));
}

double oracle_sutherland(double t) { return sutherland_viscosity(t); }
double oracle_thermal_conductivity(double mu, double gamma, double r_gas) { return thermal_conductivity(mu, gamma, r_gas); }
double oracle_limiter(int limiter, double a, double b) {
    return limiter == EFVM_LIMITER_MC ? monotonized_central(a, b) : minmod(a, b);
}

int oracle_bc_ghost(const efvm_bc* bc, int side, double gamma, double r_gas, const double* interior, double* out) {
    const IdealGas eos{gamma, r_gas};
    const ConsVar g = bc_ghost(*bc, side, ConsVar(interior[0], interior[1], interior[2], interior[3], interior[4]), eos);
    out[0] = g.rho; out[1] = g.rho_u; out[2] = g.rho_v; out[3] = g.rho_w; out[4] = g.rho_e;
    return EFVM_OK;
}

// One integrator substep on n cells (crates/cfd_solver/src/integrate.rs:48-101);
// u, u0, rhs are n x 5 doubles; returns the next stage (completed flag in *completed).
int oracle_integrator_substep(int integrator, double* u, double* u0, const double* rhs, int64_t n, double dt,
                              int stage, int* completed) {
    Case cs;
    cs.prm = efvm_params{};
    cs.prm.integrator = integrator;
    cs.u.resize((size_t)n);
    cs.u0.resize((size_t)n);
    cs.rhs.resize((size_t)n);
    for (int64_t c = 0; c < n; ++c) {
        cs.u[c] = ConsVar(u[5 * c], u[5 * c + 1], u[5 * c + 2], u[5 * c + 3], u[5 * c + 4]);
        cs.u0[c] = ConsVar(u0[5 * c], u0[5 * c + 1], u0[5 * c + 2], u0[5 * c + 3], u0[5 * c + 4]);
        cs.rhs[c] = ConsVar(rhs[5 * c], rhs[5 * c + 1], rhs[5 * c + 2], rhs[5 * c + 3], rhs[5 * c + 4]);
    }
    cs.ss.dt = dt;
    cs.ss.rk_stage = stage;
    cs.update_system();
    for (int64_t c = 0; c < n; ++c) {
        const ConsVar& a = cs.u[c];
        const ConsVar& b = cs.u0[c];
        u[5 * c] = a.rho; u[5 * c + 1] = a.rho_u; u[5 * c + 2] = a.rho_v; u[5 * c + 3] = a.rho_w; u[5 * c + 4] = a.rho_e;
        u0[5 * c] = b.rho; u0[5 * c + 1] = b.rho_u; u0[5 * c + 2] = b.rho_v; u0[5 * c + 3] = b.rho_w; u0[5 * c + 4] = b.rho_e;
    }
    *completed = cs.ss.completed_full_step ? 1 : 0;
    return cs.ss.rk_stage;
}

}  // extern "C"
