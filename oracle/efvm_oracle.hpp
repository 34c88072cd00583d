// efvm_oracle.hpp — CPU ORACLE (test infrastructure only).
//
// A serial FP64 C++17 restatement of dev_field_efvm's explicit finite-volume
// step.  It is the checker for the CUDA path and the timed CPU baseline; it is
// never linked into the product library.  Only tests/, the smoke check and the
// bench's CPU-baseline leg may load it.
//
// Every function cites the reference file:line it restates (paths inside the
// dev_field_efvm source tree).  The reference's mesh substrate (field_core at
// git 28c532a8) is not vendored, so its semantics are inferred and stated once
// in `Mesh` below; the inferences are pinned against the reference's published
// per-run numbers (examples/make_validation_plots.py:83-141) by tests/.
//
// Built with -O2 -ffp-contract=off so each operation rounds once, in the order
// the Rust source writes it.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "../include/efvm.h"

namespace oracle {

// ---- cfd_state: crates/cfd_state/src/lib.rs ------------------------------

// ConsVar, crates/cfd_state/src/lib.rs:17-50 (5 x f64, AoS).
struct ConsVar {
    double rho = 0, rho_u = 0, rho_v = 0, rho_w = 0, rho_e = 0;
    ConsVar() = default;
    ConsVar(double a, double b, double c, double d, double e) : rho(a), rho_u(b), rho_v(c), rho_w(d), rho_e(e) {}
    // velocity(), :40-44
    void velocity(double v[3]) const {
        const double inv_rho = 1.0 / rho;
        v[0] = rho_u * inv_rho;
        v[1] = rho_v * inv_rho;
        v[2] = rho_w * inv_rho;
    }
    // kinetic_energy(), :46-50
    double kinetic_energy() const {
        return 0.5 * (rho_u * rho_u + rho_v * rho_v + rho_w * rho_w) / rho;
    }
    double& comp(int d) { return d == 0 ? rho_u : (d == 1 ? rho_v : rho_w); }
    double comp(int d) const { return d == 0 ? rho_u : (d == 1 ? rho_v : rho_w); }
};
// Algebra, :78-148 (component-wise, one rounding each).
inline ConsVar operator+(const ConsVar& a, const ConsVar& b) {
    return {a.rho + b.rho, a.rho_u + b.rho_u, a.rho_v + b.rho_v, a.rho_w + b.rho_w, a.rho_e + b.rho_e};
}
inline ConsVar operator-(const ConsVar& a, const ConsVar& b) {
    return {a.rho - b.rho, a.rho_u - b.rho_u, a.rho_v - b.rho_v, a.rho_w - b.rho_w, a.rho_e - b.rho_e};
}
inline ConsVar operator*(const ConsVar& a, double s) {
    return {a.rho * s, a.rho_u * s, a.rho_v * s, a.rho_w * s, a.rho_e * s};
}
inline ConsVar operator*(double s, const ConsVar& a) { return a * s; }
inline ConsVar& operator+=(ConsVar& a, const ConsVar& b) {
    a.rho += b.rho; a.rho_u += b.rho_u; a.rho_v += b.rho_v; a.rho_w += b.rho_w; a.rho_e += b.rho_e;
    return a;
}
inline ConsVar& operator-=(ConsVar& a, const ConsVar& b) {
    a.rho -= b.rho; a.rho_u -= b.rho_u; a.rho_v -= b.rho_v; a.rho_w -= b.rho_w; a.rho_e -= b.rho_e;
    return a;
}

// PrimVar, :151-169.
struct PrimVar {
    double rho = 0, u = 0, v = 0, w = 0, p = 0, t = 0;
};

// ---- cfd_eos: crates/cfd_eos/src/lib.rs ----------------------------------

// IdealGas, :27-69.
struct IdealGas {
    double gamma = 1.4, r_gas = 287.058;
    // cons_to_prim, :44-53
    PrimVar cons_to_prim(const ConsVar& u) const {
        const double inv_rho = 1.0 / u.rho;
        const double vu = u.rho_u * inv_rho, vv = u.rho_v * inv_rho, vw = u.rho_w * inv_rho;
        const double ke = 0.5 * u.rho * (vu * vu + vv * vv + vw * vw);
        const double p = (gamma - 1.0) * (u.rho_e - ke);
        const double t = p * inv_rho / r_gas;
        return {u.rho, vu, vv, vw, p, t};
    }
    // prim_to_cons, :55-59
    ConsVar prim_to_cons(const PrimVar& p) const {
        const double ke = 0.5 * p.rho * (p.u * p.u + p.v * p.v + p.w * p.w);
        const double rho_e = p.p / (gamma - 1.0) + ke;
        return {p.rho, p.rho * p.u, p.rho * p.v, p.rho * p.w, rho_e};
    }
    // pressure, :61-63 (kinetic energy through the division form of :46-50)
    double pressure(const ConsVar& u) const { return (gamma - 1.0) * (u.rho_e - u.kinetic_energy()); }
    // sound_speed, :65-68
    double sound_speed(const ConsVar& u) const {
        const double p = pressure(u);
        return std::sqrt(gamma * p / u.rho);
    }
};

// sutherland_viscosity, :75-80
inline double sutherland_viscosity(double t) {
    const double MU_REF = 1.827e-5, T_REF = 291.15, S = 120.0;
    return MU_REF * std::pow(t / T_REF, 1.5) * (T_REF + S) / (t + S);
}
// thermal_conductivity, :83-87
inline double thermal_conductivity(double mu, double gamma, double r_gas) {
    const double cp = gamma * r_gas / (gamma - 1.0);
    const double PR = 0.72;
    return mu * cp / PR;
}
// Viscosity::mu, :108-117
struct Viscosity {
    int model = EFVM_VISC_SUTHERLAND;
    double mu_const = 0.0;
    double mu(double t) const { return model == EFVM_VISC_CONSTANT ? mu_const : sutherland_viscosity(t); }
};

// ---- cfd_riemann: crates/cfd_riemann/src/lib.rs --------------------------

ConsVar physical_flux(const ConsVar& u, const IdealGas& eos, int dir);               // :21-43
ConsVar rusanov_flux(const ConsVar& l, const ConsVar& r, const IdealGas& eos, int dir); // :222-240
ConsVar hllc_flux(const ConsVar& l, const ConsVar& r, const IdealGas& eos, int dir, bool thornber); // :395-440
ConsVar scheme_flux(int scheme, const ConsVar& l, const ConsVar& r, const IdealGas& eos, int dir);
// RiemannFlux::flux_normal default method, :76-93 (axis-aligned and rotated).
ConsVar flux_normal(int scheme, const ConsVar& owner, const ConsVar& other, const IdealGas& eos,
                    const double n[3]);

// ---- cfd_solver limiters: crates/cfd_solver/src/lib.rs:170-211 -----------
double minmod(double a, double b);
double monotonized_central(double a, double b);
ConsVar limited_slope_cons(const ConsVar& fwd, const ConsVar& bwd, int limiter);

// ---- cfd_boundary: one ghost state, crates/cfd_boundary/src/lib.rs:172-362
ConsVar bc_ghost(const efvm_bc& bc, int side, const ConsVar& interior, const IdealGas& eos);

// ---- the inferred FIELD UniformMesh ---------------------------------------
//
// field_core is not vendored; these are the semantics this oracle assumes:
//  * raw array over (nx+2g)(ny+2g)(nz+2g) cells, x fastest:
//    idx_raw(i,j,k) = i + NX*(j + NY*k); idx(i,j,k) = idx_raw(i+g,j+g,k+g);
//  * spacing h = (hi-lo)/n per axis; cell_centroid = lo + ((i_raw-g) + 0.5)*h;
//    cell_volume = (hx*hy)*hz; an axis-a face has area = product of the other
//    two spacings and centroid = owner centroid +- h/2 on axis a;
//  * for_each_face walks the interior cells k,j,i (x fastest) and for each axis
//    emits the low-side face when the cell is on the low edge, then its +axis
//    face.  A +axis face to an interior cell is an interior face (patch None)
//    emitted once.  At a domain edge the face's `other` is the adjacent ghost:
//    a patch face (patch = side) on a physical side, a halo face (patch None)
//    on a periodic side, emitted from both sides of the seam;
//  * axis_neighbors(c,a,+-) is the single face neighbour, ghosts included;
//  * locate(p) returns the raw low corner of the 2x2x2 block of cell centres
//    bracketing p with fractions t in [0,1]^3, None when the block leaves the
//    raw array;
//  * the periodic halo copies both ghost layers from the opposite interior
//    slab over the interior range of the other axes
//    (crates/cfd_boundary/src/lib.rs:805-828).
struct Face {
    size_t owner, other;
    int axis;
    double sign;      // +1 / -1: the outward normal of owner
    double area;
    double centroid[3];
    int patch;        // -1 = None, else the BoundarySide index
};

struct Mesh {
    int n[3] = {1, 1, 1};
    int ng = 2;
    int N[3] = {5, 5, 5};
    double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1}, h[3] = {1, 1, 1};
    bool periodic[3] = {false, false, false};

    void init(const efvm_grid& g);
    size_t n_raw() const { return (size_t)N[0] * N[1] * N[2]; }
    size_t idx_raw(int i, int j, int k) const { return (size_t)i + (size_t)N[0] * ((size_t)j + (size_t)N[1] * k); }
    size_t idx(int i, int j, int k) const { return idx_raw(i + ng, j + ng, k + ng); }
    void raw_coords(size_t c, int r[3]) const {
        r[0] = (int)(c % N[0]);
        r[1] = (int)((c / N[0]) % N[1]);
        r[2] = (int)(c / ((size_t)N[0] * N[1]));
    }
    double centroid_axis(int a, int raw) const { return lo[a] + ((double)(raw - ng) + 0.5) * h[a]; }
    void cell_centroid(size_t c, double out[3]) const {
        int r[3];
        raw_coords(c, r);
        for (int a = 0; a < 3; ++a) out[a] = centroid_axis(a, r[a]);
    }
    double cell_volume() const { return h[0] * h[1] * h[2]; }
    double face_area(int a) const { return a == 0 ? h[1] * h[2] : (a == 1 ? h[0] * h[2] : h[0] * h[1]); }
    bool is_local_raw(const int r[3]) const {
        for (int a = 0; a < 3; ++a)
            if (r[a] < ng || r[a] >= n[a] + ng) return false;
        return true;
    }
    bool is_local_cell(size_t c) const {
        int r[3];
        raw_coords(c, r);
        return is_local_raw(r);
    }
    bool locate(const double p[3], size_t& lo_idx, int lo_raw[3], double t[3]) const;

    template <class F>
    void for_each_face(F&& f) const;
};

template <class F>
void Mesh::for_each_face(F&& f) const {
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const int ir = i + ng, jr = j + ng, kr = k + ng;
                const size_t c = idx_raw(ir, jr, kr);
                const int coord[3] = {i, j, k};
                double cc[3] = {centroid_axis(0, ir), centroid_axis(1, jr), centroid_axis(2, kr)};
                for (int a = 0; a < 3; ++a) {
                    int off[3] = {0, 0, 0};
                    off[a] = 1;
                    const size_t hi_nb = idx_raw(ir + off[0], jr + off[1], kr + off[2]);
                    const size_t lo_nb = idx_raw(ir - off[0], jr - off[1], kr - off[2]);
                    const double area = face_area(a);
                    if (coord[a] == 0) {
                        Face fc;
                        fc.owner = c; fc.other = lo_nb; fc.axis = a; fc.sign = -1.0; fc.area = area;
                        for (int d = 0; d < 3; ++d) fc.centroid[d] = cc[d];
                        fc.centroid[a] = cc[a] - 0.5 * h[a];
                        fc.patch = periodic[a] ? -1 : 2 * a;
                        f(fc);
                    }
                    Face fc;
                    fc.owner = c; fc.other = hi_nb; fc.axis = a; fc.sign = 1.0; fc.area = area;
                    for (int d = 0; d < 3; ++d) fc.centroid[d] = cc[d];
                    fc.centroid[a] = cc[a] + 0.5 * h[a];
                    if (coord[a] + 1 < n[a]) fc.patch = -1;
                    else fc.patch = periodic[a] ? -1 : 2 * a + 1;
                    f(fc);
                }
            }
}

// ---- IBM: crates/cfd_ibm/src/lib.rs ---------------------------------------
struct Cylinder {
    double cx, cy, r;
    double vx = 0.0, vy = 0.0, omega = 0.0;  // a moving disc (examples/dkt_sedimentation/main.rs:66-103)
    // Disc::wall_velocity, :94-102: v + omega z x (p - c)
    void wall_velocity(const double p[3], double out[3]) const {
        const double rx = p[0] - cx, ry = p[1] - cy;
        out[0] = vx - omega * ry;
        out[1] = vy + omega * rx;
        out[2] = 0.0;
    }
    double signed_distance(const double p[3]) const {   // :70-74
        const double dx = p[0] - cx, dy = p[1] - cy;
        return std::sqrt(dx * dx + dy * dy) - r;
    }
    void normal(const double p[3], double n[3]) const {  // :77-86
        const double dx = p[0] - cx, dy = p[1] - cy;
        const double rr = std::sqrt(dx * dx + dy * dy);
        if (rr < 1e-12) { n[0] = 1.0; n[1] = 0.0; n[2] = 0.0; }
        else { n[0] = dx / rr; n[1] = dy / rr; n[2] = 0.0; }
    }
};
// SphereBody, crates/cfd_ibm/src/sphere.rs:26-72
struct Sphere {
    double c[3], r, v[3], w[3];
    double signed_distance(const double p[3]) const {
        const double d0 = p[0] - c[0], d1 = p[1] - c[1], d2 = p[2] - c[2];
        return std::sqrt(d0 * d0 + d1 * d1 + d2 * d2) - r;
    }
    void normal(const double p[3], double n[3]) const {
        const double d0 = p[0] - c[0], d1 = p[1] - c[1], d2 = p[2] - c[2];
        const double rr = std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        if (rr < 1e-12) { n[0] = 1.0; n[1] = 0.0; n[2] = 0.0; }
        else { n[0] = d0 / rr; n[1] = d1 / rr; n[2] = d2 / rr; }
    }
    void wall_velocity(const double p[3], double out[3]) const {
        const double r0 = p[0] - c[0], r1 = p[1] - c[1], r2 = p[2] - c[2];
        out[0] = v[0] + w[1] * r2 - w[2] * r1;
        out[1] = v[1] + w[2] * r0 - w[0] * r2;
        out[2] = v[2] + w[0] * r1 - w[1] * r0;
    }
};
struct IbmGhost {
    size_t idx;
    double cell_center[3], image_point[3], normal[3];
    uint32_t body_id;
    double wall_velocity[3];
};
struct IbmMarker {
    uint32_t body_id;
    double position[3], normal[3], area, wall_velocity[3];
};

// ---- the App: one case, substage by substage ------------------------------
struct SolverState {
    double dt = 0.0, time = 0.0;
    uint64_t step = 0;
    int rk_stage = 0;  // 0 First, 1 Second, 2 Third
    bool completed_full_step = false;
};

struct Case {
    Mesh mesh;
    IdealGas eos;
    Viscosity visc;
    efvm_grid grid{};
    efvm_params prm{};
    std::vector<ConsVar> u, rhs, u0;
    std::vector<uint8_t> solid;                 // SolidMask
    std::vector<ConsVar> slopes;                // MusclSlopes, 3 per raw cell
    SolverState ss;
    bool ibm = false;
    std::vector<Cylinder> cyls;
    std::vector<Sphere> spheres;                 // SphereBodies (3-D)
    int sphere_markers_n = 2000;                 // SphereMarkerCfg
    int cylinder_markers_n = 64;                 // n_theta of the cylinder / disc markers
    bool disc_ghost_rule = false;                // compute_disc_ghosts: in-plane neighbours only
    ConsVar stagnant, ambient;                   // MaskConsts
    std::vector<IbmGhost> ghosts;
    std::vector<IbmMarker> markers;
    double marker_force[6] = {0, 0, 0, 0, 0, 0}; // pressure xyz, viscous xyz
    double wall_force[6] = {0, 0, 0, 0, 0, 0};
    bool slopes_before_ibm = false;              // plugin registration order variant
    bool colored = false;                        // OpenMP face colouring (same faces, other order)
    // Whether a cell gets MUSCL slopes and face reconstruction: every local cell,
    // plus (EFVM_SEAM_TRUE_PERIODIC only) the first ghost layer across a periodic
    // seam, so both sides of a seam face see the same reconstructed states.
    bool reconstructs(size_t c) const;

    bool setup(const efvm_grid& g, const efvm_params& p, const char** err);
    void substep();
    // systems
    void cfl_system();
    void halo_system();
    void boundary_system();
    void parabolic_inflow_system();
    void zero_rhs_system();
    void compute_slopes_system();
    void flux_system();
    void muscl_flux_system();
    void viscous_system();
    void update_system();
    void outlet_sponge_system();
    void body_force_system();
    void refresh_cylinder_mask();
    void compute_cylinder_ghosts();
    void compute_cylinder_markers();
    void refresh_sphere_mask();
    void compute_sphere_ghosts();
    void compute_sphere_markers();
    void geometry_systems();  // the Setup-phase geometry of whichever bodies are set
    void apply_ibm_ghost_bc();
    void zero_solid_rhs();
    void marker_force_system();
    void wall_force_system();
    bool sample_trilinear(const double point[3], PrimVar& out) const;
    double cfl_dt() const;
};

}  // namespace oracle
