// efvm_api.cu — the C-ABI of include/efvm.h: context lifecycle, device
// memory, the per-substage phase order of one app.run(), CUDA-graph captured
// RK3 steps, strided state upload/download and the IBM geometry set-up.
//
// The IBM geometry that the reference rebuilds every substage (ghost list,
// image points, markers; crates/cfd_ibm/src/lib.rs:155-254,566-598) is static
// for a fixed body, so it is built once per efvm_set_cylinders: the solid mask
// on the device, the ghost list and marker sample points on the host with the
// same one-rounding-per-operation arithmetic as the reference's Rust.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "efvm_internal.h"

using namespace efvm;

struct efvm_ctx {
    efvm_grid grid;
    efvm_params params;
    Geometry g;
    Physics ph;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;      // IBM forces, forked from the step graph
    cudaEvent_t ev_fork[3] = {nullptr, nullptr, nullptr}, ev_join = nullptr;
    double* U[3] = {nullptr, nullptr, nullptr};  // U0 (= u^n), U1, U2
    uint8_t* mask = nullptr;
    double* yw = nullptr;                          // viscous y weights
    double* zw = nullptr;                          // viscous z weights (3-D)
    DevState* st = nullptr;                        // device
    double* partial = nullptr;                     // reduction partials
    int n_partial = 0;
    double* staging = nullptr;
    size_t staging_bytes = 0;
    // host mirror of the RK state machine (the device holds the authoritative clock)
    int rk_stage = 0;
    int euler_cur = 0;  // Euler ping-pong buffer index
    bool lam_stale = true;
    bool ghosts_stale = true;
    bool control_dirty = true;
    // IBM
    bool ibm = false;
    bool geom_dirty = false;
    std::vector<double> cyl_host;  // cx, cy, r per body
    std::vector<double> disc_motion;  // vx, vy, omega per body (moving discs; zero for cylinders)
    int cyl_markers = 64;             // markers per cylinder / disc
    bool disc_rule = false;           // moving discs: mirror only cells with a fluid in-plane neighbour
    int64_t n_mirror = 0;             // solid cells the mirror rewrites
    std::vector<double> sph_host;  // 3-D spheres: efvm_sphere's 10 doubles per body
    double* sph_dev = nullptr;
    int sphere_markers = 2000;     // Fibonacci markers per sphere
    IbmGhost3Dev* ghosts3_dev = nullptr;
    Marker3Dev* markers3_dev = nullptr;
    double stagnant[5] = {0, 0, 0, 0, 0};  // MaskConsts.stagnant
    // learned face-flux correction (efvm_set_flux_correction)
    efvm_nn* nn = nullptr;
    float* corr = nullptr;               // [2][4][ny][nx]
    float4* prims = nullptr;             // the network's per-cell inputs
    unsigned long long* fallbacks = nullptr;
    float sensor = 0.f;
    uint64_t corr_faces = 0;
    double* out_fields = nullptr;        // efvm_output_fields
    double ambient[5] = {0, 0, 0, 0, 0};   // MaskConsts.ambient
    double* cyl_dev = nullptr;
    IbmGhostDev* ghosts_dev = nullptr;
    MarkerDev* markers_dev = nullptr;
    double* zg0 = nullptr;
    double* zfill = nullptr;
    double* force_out = nullptr;
    double* force_partials = nullptr;
    unsigned int* force_counter = nullptr;
    double* history = nullptr;
    long long history_cap = 0;
    Ibm ibm_desc{};
    int64_t n_solid = 0;
    // CUDA graph of one RK3 step
    cudaGraphExec_t graph_exec = nullptr;
    bool graph_valid = false;
    bool graph_with_history = false;
    int graph_kernels = 0;
    uint64_t launches = 0;
    // The TMA-fed stage kernel (2-D contexts): tensor maps of U0, U1, U2 as the
    // stage input and of U0 as U^n, and the stage tiling (efvm_set_stage_tiling)
    CUtensorMap tmap[3];
    CUtensorMap tmap_u0;
    bool tmaps = false;
    int stage_form = EFVM_STAGE_AUTO;
    int stage_rows = 0;
    int stage_blocks = 0;
    unsigned long long stage_wait_ns = 4000000000ull;  // one TMA ring wait (efvm_set_stage_wait_limit)
    int stage_stall = 0;                               // efvm_inject_stage_stall
    // halo peers of a slab (efvm_set_halo_peer): per y side the neighbour's
    // three state buffers, their plane and the neighbour's rows
    double* peer_bufs[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    long long peer_plane[2] = {0, 0};
    int peer_rows[2] = {0, 0};
    void* peer_ipc[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};  // mapped by this context
    std::string err;
};

namespace {

thread_local std::string g_last_error;

int fail(efvm_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    g_last_error = msg;
    return code;
}

#define CUDA_TRY(ctx, call)                                                                     \
    do {                                                                                        \
        cudaError_t e__ = (call);                                                               \
        if (e__ != cudaSuccess)                                                                 \
            return fail(ctx, e__ == cudaErrorMemoryAllocation ? EFVM_ERR_OOM : EFVM_ERR_CUDA,   \
                        std::string(#call) + ": " + cudaGetErrorString(e__));                   \
    } while (0)

// Host arithmetic with one rounding per operation (built with -ffp-contract=off).
double centre_h(double lo, double h, int i) { return lo + ((double)i + 0.5) * h; }

// FIELD locate() restricted to x/y (see the oracle header for the inferred rule):
// f = (p - lo)/h - 0.5, low corner floor(f), fraction f - floor(f); valid when
// the 2x2 block stays inside the raw array (ghosts included).
bool locate_h(const Geometry& g, double px, double py, int& li, int& lj, double& tx, double& ty) {
    const double fx = (px - g.lo[0]) / g.h[0] - 0.5;
    const double fy = (py - g.lo[1]) / g.h[1] - 0.5;
    const double flx = std::floor(fx), fly = std::floor(fy);
    li = (int)flx;
    lj = (int)fly;
    tx = fx - flx;
    ty = fy - fly;
    const bool okx = li + NG >= 0 && li + NG + 1 < g.nx + 2 * NG;
    const bool oky = lj + NG >= 0 && lj + NG + 1 < g.ny + 2 * NG;
    return okx && oky;
}

cudaStream_t S(efvm_ctx* c) { return c->stream; }

double* cur_buf(efvm_ctx* c) {
    if (c->params.integrator == EFVM_INTEGRATOR_EULER) return c->U[c->euler_cur];
    return c->U[c->rk_stage];
}

// Entry points built for the 2-D layout answer a 3-D context (nz > 1) with this.
int refuse_3d(efvm_ctx* c, const char* what) {
    return fail(c, EFVM_ERR_UNSUPPORTED, std::string(what) + " is built for 2-D meshes (nz == 1)");
}
bool is_3d(const efvm_ctx* c) { return c && c->g.nz > 1; }

int ensure_staging(efvm_ctx* c, size_t bytes) {
    if (c->staging_bytes >= bytes) return EFVM_OK;
    if (c->staging) cudaFree(c->staging);
    c->staging = nullptr;
    c->staging_bytes = 0;
    CUDA_TRY(c, cudaMalloc(&c->staging, bytes));
    c->staging_bytes = bytes;
    return EFVM_OK;
}

int sync_control(efvm_ctx* c, int stop_at_t, double t_stop, long long hist_cap) {
    c->launches += launch_set_control(c->st, 1, stop_at_t, t_stop, hist_cap, S(c));
    c->control_dirty = stop_at_t != 0 || hist_cap != 0;
    return EFVM_OK;
}

// Build the IBM ghost list and marker sample points after the device mask flip.
// Rigid surface velocity v + omega z x (p - c) of disc b (Disc::wall_velocity,
// examples/dkt_sedimentation/main.rs:94-102); zero for a cylinder at rest.
void disc_wall_velocity(const efvm_ctx* c, int b, const double p[2], double out[2]) {
    if (c->disc_motion.empty()) {
        out[0] = out[1] = 0.0;
        return;
    }
    const double rx = p[0] - c->cyl_host[3 * b], ry = p[1] - c->cyl_host[3 * b + 1];
    const double* m = &c->disc_motion[3 * b];
    out[0] = m[0] - m[2] * ry;
    out[1] = m[1] + m[2] * rx;
}

int build_ibm_lists(efvm_ctx* c) {
    const Geometry& g = c->g;
    std::vector<uint8_t> m((size_t)g.nx * g.ny);
    CUDA_TRY(c, cudaMemcpy2DAsync(m.data(), g.nx, c->mask + (size_t)YO * g.pitch + XO, g.pitch, g.nx, g.ny,
                                  cudaMemcpyDeviceToHost, S(c)));
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    const int ncyl = (int)(c->cyl_host.size() / 3);
    // the mask is zero outside the interior
    auto solid = [&](int i, int j) {
        return i >= 0 && i < g.nx && j >= 0 && j < g.ny && m[(size_t)j * g.nx + i] != 0;
    };
    auto corner_bits = [&](int lo_i, int lo_j) {
        unsigned b = 0;
        for (int k = 0; k < 4; ++k)
            if (!solid(lo_i + (k >> 1), lo_j + (k & 1))) b |= 1u << (FLUID_CORNER_SHIFT + k);
        return b;
    };
    std::vector<IbmGhostDev> ghosts;
    c->n_solid = 0;
    c->n_mirror = 0;
    for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i < g.nx; ++i) {
            if (!m[(size_t)j * g.nx + i]) continue;
            ++c->n_solid;
            // compute_cylinder_ghosts, crates/cfd_ibm/src/lib.rs:187-254: a solid cell
            // with >= 1 non-solid face neighbour.  The 2-D mesh's two z neighbours are
            // ghost layers, which are never solid, so every solid cell qualifies.
            const double cc[2] = {centre_h(g.lo[0], g.h[0], i), centre_h(g.lo[1], g.h[1], j)};
            double best_abs = std::numeric_limits<double>::max(), best_signed = 0.0;
            double nrm[2] = {1.0, 0.0};
            int best_b = 0;
            for (int b = 0; b < ncyl; ++b) {
                const double dx = cc[0] - c->cyl_host[3 * b], dy = cc[1] - c->cyl_host[3 * b + 1];
                const double r = std::sqrt(dx * dx + dy * dy);
                const double s = r - c->cyl_host[3 * b + 2];
                if (std::fabs(s) < best_abs) {
                    best_abs = std::fabs(s);
                    best_signed = s;
                    best_b = b;
                    if (r < 1e-12) { nrm[0] = 1.0; nrm[1] = 0.0; }
                    else { nrm[0] = dx / r; nrm[1] = dy / r; }
                }
            }
            const double push = 2.0 * (-best_signed);
            const double ip[2] = {cc[0] + push * nrm[0], cc[1] + push * nrm[1]};
            IbmGhostDev gh{};
            gh.i = i;
            gh.j = j;
            // the nearest body's wall velocity at the cell's wall footprint
            // (compute_disc_ghosts, examples/dkt_sedimentation/main.rs:175-249)
            const double foot[2] = {cc[0] - best_signed * nrm[0], cc[1] - best_signed * nrm[1]};
            disc_wall_velocity(c, best_b, foot, gh.uw);
            gh.valid = locate_h(g, ip[0], ip[1], gh.lo_i, gh.lo_j, gh.tx, gh.ty) ? 1 : 0;
            const int nbi[4] = {i + 1, i - 1, i, i}, nbj[4] = {j, j, j + 1, j - 1};
            for (int k = 0; k < 4; ++k)
                if (!solid(nbi[k], nbj[k])) gh.fluid |= 1u << (FLUID_NB_SHIFT + k);
            if (!c->disc_rule || (gh.fluid & (0xFu << FLUID_NB_SHIFT))) {
                gh.fluid |= GHOST_MIRROR_BIT;
                ++c->n_mirror;
            }
            if (gh.valid) gh.fluid |= corner_bits(gh.lo_i, gh.lo_j);
            ghosts.push_back(gh);
        }
    // compute_cylinder_markers, crates/cfd_ibm/src/lib.rs:566-598 (n_theta = 64, n_z = 1)
    std::vector<MarkerDev> markers;
    const double PI = 3.141592653589793;
    const double z_lo = centre_h(g.lo[2], g.h[2], 0) - 0.5 * g.h[2];
    const double z_hi = centre_h(g.lo[2], g.h[2], 0) + 0.5 * g.h[2];
    const double lz = z_hi - z_lo;
    const int n_theta = c->cyl_markers, n_z = 1;
    const double offset = g.h[0];  // marker_force_system: sample offset = spacing(0, 0)
    for (int b = 0; b < ncyl; ++b) {
        const double cx = c->cyl_host[3 * b], cy = c->cyl_host[3 * b + 1], r = c->cyl_host[3 * b + 2];
        const double area = 2.0 * PI * r * lz / (double)(n_theta * n_z);
        for (int it = 0; it < n_theta; ++it) {
            const double theta = 2.0 * PI * ((double)it + 0.5) / (double)n_theta;
            const double nx = std::cos(theta), ny = std::sin(theta);
            MarkerDev mk{};
            mk.normal[0] = nx;
            mk.normal[1] = ny;
            mk.normal[2] = 0.0;
            mk.area = area;
            const double px = cx + r * nx, py = cy + r * ny;
            const double sx = px + offset * nx, sy = py + offset * ny;
            mk.valid = locate_h(g, sx, sy, mk.lo_i, mk.lo_j, mk.tx, mk.ty) ? 1 : 0;
            if (mk.valid) mk.fluid = corner_bits(mk.lo_i, mk.lo_j);
            mk.pos[0] = px;
            mk.pos[1] = py;
            mk.body = b;
            const double pp[2] = {px, py};
            double uw2[2];
            disc_wall_velocity(c, b, pp, uw2);
            mk.wall_velocity[0] = uw2[0];
            mk.wall_velocity[1] = uw2[1];
            mk.wall_velocity[2] = 0.0;
            markers.push_back(mk);
        }
    }
    if (c->ghosts_dev) cudaFree(c->ghosts_dev);
    if (c->markers_dev) cudaFree(c->markers_dev);
    if (c->zg0) cudaFree(c->zg0);
    if (c->zfill) cudaFree(c->zfill);
    c->ghosts_dev = nullptr;
    c->markers_dev = nullptr;
    c->zg0 = c->zfill = nullptr;
    const size_t ng = std::max<size_t>(ghosts.size(), 1), nm = std::max<size_t>(markers.size(), 1);
    CUDA_TRY(c, cudaMalloc(&c->ghosts_dev, ng * sizeof(IbmGhostDev)));
    CUDA_TRY(c, cudaMalloc(&c->markers_dev, nm * sizeof(MarkerDev)));
    if (c->force_partials) cudaFree(c->force_partials);
    c->force_partials = nullptr;
    const size_t nblocks = 1 + (ghosts.size() + IBM_THREADS - 1) / IBM_THREADS;
    CUDA_TRY(c, cudaMalloc(&c->force_partials, nblocks * 6 * sizeof(double)));
    CUDA_TRY(c, cudaMalloc(&c->zg0, 2 * ng * 4 * sizeof(double)));
    CUDA_TRY(c, cudaMalloc(&c->zfill, 3 * ng * 4 * sizeof(double)));
    CUDA_TRY(c, cudaMemsetAsync(c->zg0, 0, 2 * ng * 4 * sizeof(double), S(c)));
    CUDA_TRY(c, cudaMemsetAsync(c->zfill, 0, 3 * ng * 4 * sizeof(double), S(c)));
    if (!ghosts.empty())
        CUDA_TRY(c, cudaMemcpyAsync(c->ghosts_dev, ghosts.data(), ghosts.size() * sizeof(IbmGhostDev),
                                    cudaMemcpyHostToDevice, S(c)));
    if (!markers.empty())
        CUDA_TRY(c, cudaMemcpyAsync(c->markers_dev, markers.data(), markers.size() * sizeof(MarkerDev),
                                    cudaMemcpyHostToDevice, S(c)));
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    Ibm& d = c->ibm_desc;
    d.enabled = 1;
    d.n_ghost = (int)ghosts.size();
    d.n_markers = (int)markers.size();
    d.ghosts = c->ghosts_dev;
    d.markers = c->markers_dev;
    d.sample_offset = offset;
    d.zg0 = c->zg0;
    d.zfill = c->zfill;
    d.force_out = c->force_out;
    d.partials = c->force_partials;
    d.counter = c->force_counter;
    return EFVM_OK;
}

// The 3-D lists after the mask changed (compute_sphere_ghosts and
// compute_sphere_markers, crates/cfd_ibm/src/sphere.rs:116-245), built on the host
// from the device mask with the reference's arithmetic, then uploaded.  The mask
// of a ghost layer is the interior's image on a periodic axis (the reference's
// halo copies it with the state) and fluid elsewhere.
int build_ibm_lists3(efvm_ctx* c) {
    const Geometry& g = c->g;
    std::vector<uint8_t> m((size_t)g.plane);
    CUDA_TRY(c, cudaMemcpyAsync(m.data(), c->mask, (size_t)g.plane, cudaMemcpyDeviceToHost, S(c)));
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    const int n[3] = {g.nx, g.ny, g.nz};
    const bool per[3] = {c->ph.periodic_x != 0, c->ph.periodic_y != 0, c->ph.periodic_z != 0};
    auto at = [&](int i, int j, int k) {
        return (size_t)(2 + k) * (size_t)g.layer + (size_t)(YO + j) * g.pitch + (size_t)(XO + i);
    };
    // solid at interior coordinates, ghost layers included (-2 .. n+1)
    auto solid = [&](int i, int j, int k) {
        int q[3] = {i, j, k};
        for (int a = 0; a < 3; ++a) {
            if (q[a] >= 0 && q[a] < n[a]) continue;
            if (!per[a]) return false;
            q[a] = q[a] < 0 ? q[a] + n[a] : q[a] - n[a];
        }
        return m[at(q[0], q[1], q[2])] != 0;
    };
    // FIELD locate(): low corner floor(f) of the 2x2x2 block of cell centres
    // around p, f = (p - lo)/h - 0.5; valid when the block stays inside the raw array
    auto locate3 = [&](const double p[3], int lo[3], double t[3]) {
        bool ok = true;
        for (int a = 0; a < 3; ++a) {
            const double f = (p[a] - g.lo[a]) / g.h[a] - 0.5;
            const double fl = std::floor(f);
            lo[a] = (int)fl;
            t[a] = f - fl;
            ok = ok && lo[a] + NG >= 0 && lo[a] + NG + 1 < n[a] + 2 * NG;
        }
        return ok;
    };
    auto corner_bits = [&](const int lo[3]) {
        unsigned b = 0;
        for (int di = 0; di < 2; ++di)
            for (int dj = 0; dj < 2; ++dj)
                for (int dk = 0; dk < 2; ++dk)
                    if (!solid(lo[0] + di, lo[1] + dj, lo[2] + dk))
                        b |= 1u << (FLUID3_CORNER_SHIFT + 4 * di + 2 * dj + dk);
        return b;
    };
    const int nb = (int)(c->sph_host.size() / 10);
    auto sd_of = [&](int b, const double p[3], double nrm[3]) {
        const double* s = &c->sph_host[10 * b];
        const double d0 = p[0] - s[0], d1 = p[1] - s[1], d2 = p[2] - s[2];
        const double rr = std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        if (rr < 1e-12) { nrm[0] = 1.0; nrm[1] = 0.0; nrm[2] = 0.0; }
        else { nrm[0] = d0 / rr; nrm[1] = d1 / rr; nrm[2] = d2 / rr; }
        return rr - s[3];
    };
    auto wall_velocity = [&](int b, const double p[3], double out[3]) {
        const double* s = &c->sph_host[10 * b];
        const double r0 = p[0] - s[0], r1 = p[1] - s[1], r2 = p[2] - s[2];
        out[0] = s[4] + s[8] * r2 - s[9] * r1;
        out[1] = s[5] + s[9] * r0 - s[7] * r2;
        out[2] = s[6] + s[7] * r1 - s[8] * r0;
    };
    std::vector<IbmGhost3Dev> ghosts;
    c->n_solid = 0;
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                if (!m[at(i, j, k)]) continue;
                ++c->n_solid;
                const int nbd[6][3] = {{i + 1, j, k}, {i - 1, j, k}, {i, j + 1, k}, {i, j - 1, k}, {i, j, k + 1}, {i, j, k - 1}};
                unsigned fl = 0;
                for (int q = 0; q < 6; ++q)
                    if (!solid(nbd[q][0], nbd[q][1], nbd[q][2])) fl |= 1u << q;
                if (!fl) continue;  // fully buried
                const double cc[3] = {centre_h(g.lo[0], g.h[0], i), centre_h(g.lo[1], g.h[1], j),
                                      centre_h(g.lo[2], g.h[2], k)};
                double best_abs = std::numeric_limits<double>::max(), best_signed = 0.0;
                double best_n[3] = {1.0, 0.0, 0.0}, best_w[3] = {0.0, 0.0, 0.0};
                for (int b = 0; b < nb; ++b) {
                    double nrm[3];
                    const double sd = sd_of(b, cc, nrm);
                    if (std::fabs(sd) < best_abs) {
                        best_abs = std::fabs(sd);
                        best_signed = sd;
                        for (int d = 0; d < 3; ++d) best_n[d] = nrm[d];
                        const double foot[3] = {cc[0] - sd * best_n[0], cc[1] - sd * best_n[1], cc[2] - sd * best_n[2]};
                        wall_velocity(b, foot, best_w);
                    }
                }
                const double push = 2.0 * (-best_signed);
                const double ip[3] = {cc[0] + push * best_n[0], cc[1] + push * best_n[1], cc[2] + push * best_n[2]};
                IbmGhost3Dev gh{};
                gh.i = i;
                gh.j = j;
                gh.k = k;
                gh.fluid = fl;
                gh.valid = locate3(ip, gh.lo, gh.t) ? 1 : 0;
                if (gh.valid) gh.fluid |= corner_bits(gh.lo);
                for (int d = 0; d < 3; ++d) gh.uw[d] = best_w[d];
                ghosts.push_back(gh);
            }
    // sphere_markers: the golden-angle Fibonacci lattice, area 4 pi R^2 / n
    std::vector<Marker3Dev> markers;
    const double PI = 3.141592653589793;
    const int nm = std::max(c->sphere_markers, 12);
    const double golden = PI * (3.0 - std::sqrt(5.0));
    const double offset = g.h[0];  // marker_force_system: sample offset = spacing(0, 0)
    for (int b = 0; b < nb; ++b) {
        const double* s = &c->sph_host[10 * b];
        const double area = 4.0 * PI * s[3] * s[3] / (double)nm;
        for (int q = 0; q < nm; ++q) {
            const double zr = 1.0 - 2.0 * ((double)q + 0.5) / (double)nm;
            const double rr = std::sqrt(std::max(1.0 - zr * zr, 0.0));
            const double phi = golden * (double)q;
            const double dir[3] = {rr * std::cos(phi), rr * std::sin(phi), zr};
            const double pos[3] = {s[0] + s[3] * dir[0], s[1] + s[3] * dir[1], s[2] + s[3] * dir[2]};
            Marker3Dev mk{};
            for (int d = 0; d < 3; ++d) mk.normal[d] = dir[d];
            mk.area = area;
            wall_velocity(b, pos, mk.uw);
            const double sp[3] = {pos[0] + offset * dir[0], pos[1] + offset * dir[1], pos[2] + offset * dir[2]};
            mk.valid = locate3(sp, mk.lo, mk.t) ? 1 : 0;
            if (mk.valid) mk.fluid = corner_bits(mk.lo);
            mk.body = b;
            markers.push_back(mk);
        }
    }
    cudaFree(c->ghosts3_dev);
    cudaFree(c->markers3_dev);
    c->ghosts3_dev = nullptr;
    c->markers3_dev = nullptr;
    CUDA_TRY(c, cudaMalloc(&c->ghosts3_dev, std::max<size_t>(ghosts.size(), 1) * sizeof(IbmGhost3Dev)));
    CUDA_TRY(c, cudaMalloc(&c->markers3_dev, std::max<size_t>(markers.size(), 1) * sizeof(Marker3Dev)));
    if (!ghosts.empty())
        CUDA_TRY(c, cudaMemcpyAsync(c->ghosts3_dev, ghosts.data(), ghosts.size() * sizeof(IbmGhost3Dev),
                                    cudaMemcpyHostToDevice, S(c)));
    if (!markers.empty())
        CUDA_TRY(c, cudaMemcpyAsync(c->markers3_dev, markers.data(), markers.size() * sizeof(Marker3Dev),
                                    cudaMemcpyHostToDevice, S(c)));
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    Ibm& d = c->ibm_desc;
    d.enabled = 1;
    d.n_ghost = (int)ghosts.size();
    d.n_markers = (int)markers.size();
    d.ghosts3 = c->ghosts3_dev;
    d.markers3 = c->markers3_dev;
    d.sample_offset = offset;
    d.force_out = c->force_out;
    return EFVM_OK;
}

// Setup-phase work that precedes a step boundary's first stage, in the
// reference's Setup order: CFL (SolverPlugin) before the geometry refresh
// (CylinderIbmPlugin), then Halo/Boundary for a state that changed on the host.
int prologue(efvm_ctx* c) {
    if (c->rk_stage == 0 && c->lam_stale && c->ph.fixed_dt <= 0.0) {
        c->launches += launch_cfl(c->g, c->ph, cur_buf(c), c->st, S(c));
        c->lam_stale = false;
    }
    if (c->ibm && c->geom_dirty) {
        int rc;
        if (is_3d(c)) {
            c->launches += launch_geometry3(c->g, c->ph, c->sph_dev, (int)(c->sph_host.size() / 10), c->stagnant,
                                            c->ambient, cur_buf(c), c->mask, S(c));
            rc = build_ibm_lists3(c);
        } else {
            c->launches += launch_geometry(c->g, c->cyl_dev, (int)(c->cyl_host.size() / 3), c->stagnant, c->ambient,
                                           cur_buf(c), c->mask, S(c));
            rc = build_ibm_lists(c);
        }
        if (rc) return rc;
        c->geom_dirty = false;
        c->ghosts_stale = true;
        c->graph_valid = false;
    }
    if (c->ghosts_stale) {
        c->launches += launch_fill_ghosts(c->g, c->ph, cur_buf(c), S(c));
        c->ghosts_stale = false;
    }
    return EFVM_OK;
}

// The stage-kernel form a context runs.  The TMA-fed kernel runs where it is
// selected and the case allows it (2-D, inviscid, no bodies, no learned
// correction); EFVM_STAGE_AUTO selects it in both precisions: at 4096^2 it
// measured 1.70 against 1.85 ms per step (FP32 fluxes) and 2.26 against 2.47
// (FP64) for the strip kernel.
int resolved_form(const efvm_ctx* c) {
    const bool want = c->stage_form == EFVM_STAGE_TMA || c->stage_form == EFVM_STAGE_AUTO;
    if (want && c->tmaps && stage_tma_eligible(c->g, c->ph, c->ibm, c->nn != nullptr)) return EFVM_STAGE_TMA;
    return EFVM_STAGE_STRIP;
}

void enqueue_stage_kernel(efvm_ctx* c, int stage, double* uin, double* uout, bool pdl = true, bool defer = false) {
    if (c->nn)  // the learned corrections of this stage's input
        c->launches += nn_forward_padded(c->nn, uin, c->g.plane, c->g.pitch, c->g.nx, c->g.ny, c->corr, c->prims,
                                         c->sensor, c->fallbacks, S(c));
    StageArgs a{};
    a.corr = c->nn ? c->corr : nullptr;
    a.g = c->g;
    a.ph = c->ph;
    a.uin = uin;
    a.u0 = c->U[0];
    a.uout = uout;
    a.mask = c->ibm ? c->mask : nullptr;
    a.yw = c->yw;
    a.zw = c->zw;
    a.st = c->st;
    a.stage = stage;
    a.completes_step = (stage == 2 || stage == 3) ? 1 : 0;
    a.want_cfl = a.completes_step && c->ph.fixed_dt <= 0.0;
    a.defer_forces = defer ? 1 : 0;
    if (c->tmaps && resolved_form(c) == EFVM_STAGE_TMA) {
        for (int k = 0; k < 3; ++k)
            if (uin == c->U[k]) a.tmap_in = &c->tmap[k];
        a.tmap_u0 = &c->tmap_u0;
    }
    a.rows = c->stage_rows;
    a.blocks = c->stage_blocks;
    a.wait_ns = c->stage_wait_ns;
    a.stall = c->stage_stall;
    for (int side = 0; side < 2; ++side) {
        if (!c->peer_bufs[side][0]) continue;
        for (int k = 0; k < 3; ++k)
            if (uout == c->U[k]) a.peer_out[side] = c->peer_bufs[side][k];
        a.peer_plane[side] = c->peer_plane[side];
        a.peer_ny[side] = c->peer_rows[side];
    }
    c->launches += launch_stage(a, pdl, S(c));
}

// The IBM forces of the step graph's last stage run in the next step's first
// launch (beside its set-up and mirror), so that the step ends with its last
// stage.  Anything that reads the forces, or changes what they read (the state,
// the bodies, the force history's control), first runs them here if a step
// left them pending: the kernel does nothing otherwise.
static int finish_forces(efvm_ctx* c) {
    if (!c->ibm || is_3d(c)) return EFVM_OK;
    c->launches += launch_ibm(c->g, c->ph, c->ibm_desc, c->U[0], c->st, 2, -1, 0, false, S(c), 1);
    return EFVM_OK;
}

// Launch the kernels of one substage at RK stage `stage` (0..2, or 3 = Euler):
// [step set-up +] IBM mirror of uin, the stage, the IBM forces of uout.
void enqueue_substage(efvm_ctx* c, int stage, double* uin, double* uout, bool with_setup) {
    if (c->ibm && is_3d(c)) {  // spheres: [set-up], mirror, stage, forces, all on the main stream
        if (with_setup) c->launches += launch_step_setup(c->ph, c->st, true, S(c));
        c->launches += launch_mirror3(c->g, c->ph, c->ibm_desc, uin, true, S(c));
        enqueue_stage_kernel(c, stage, uin, uout);
        c->launches += launch_forces3(c->g, c->ph, c->ibm_desc, uout, c->st, true, S(c));
        return;
    }
    if (c->ibm) c->launches += launch_ibm(c->g, c->ph, c->ibm_desc, uin, c->st, -1, stage, with_setup, true, S(c));
    else if (with_setup) c->launches += launch_step_setup(c->ph, c->st, true, S(c));
    enqueue_stage_kernel(c, stage, uin, uout);
    if (c->ibm) c->launches += launch_ibm(c->g, c->ph, c->ibm_desc, uout, c->st, stage, -1, 0, true, S(c));
}

// One whole SSP-RK3 step, as captured into the step graph.  With IBM the
// forces of stages 1 and 2 run on a side branch that forks after the stage, in
// parallel with the mirror and the next stage (they read only fluid cells of
// the stage's output and the stage's z-fill, which the next stage leaves
// alone); the branch joins at the end of the step.  The forces of stage 3 run
// in the next step's first launch (finish_forces runs them before anything
// reads them): they read fluid cells of U0, which that launch's mirror leaves
// alone, stage 3's z-fill, and this step's saved z-ghost state, which the next
// step saves into the other parity's buffer.
int enqueue_rk3_step(efvm_ctx* c) {
    double* bufs[4] = {c->U[0], c->U[1], c->U[2], c->U[0]};
    if (c->ibm && is_3d(c)) {
        for (int s = 0; s < 3; ++s) enqueue_substage(c, s, bufs[s], bufs[s + 1], s == 0);
        return EFVM_OK;
    }
    // the first launch: the forces of the previous step's last stage (when pending),
    // the set-up and the mirror of stage 1; bufs[0] is both their state and its input
    if (c->ibm) c->launches += launch_ibm(c->g, c->ph, c->ibm_desc, bufs[0], c->st, 2, 0, 1, true, S(c), 1);
    else c->launches += launch_step_setup(c->ph, c->st, true, S(c));
    for (int s = 0; s < 3; ++s) {
        enqueue_stage_kernel(c, s, bufs[s], bufs[s + 1], true, c->ibm && s == 2);
        if (c->ibm && s < 2) {
            CUDA_TRY(c, cudaEventRecord(c->ev_fork[s], S(c)));
            CUDA_TRY(c, cudaStreamWaitEvent(c->side, c->ev_fork[s], 0));
            c->launches += launch_ibm(c->g, c->ph, c->ibm_desc, bufs[s + 1], c->st, s, -1, 0, false, c->side);
            c->launches += launch_ibm(c->g, c->ph, c->ibm_desc, bufs[s + 1], c->st, -1, s + 1, 0, true, S(c));
        }
    }
    if (c->ibm) {
        CUDA_TRY(c, cudaEventRecord(c->ev_join, c->side));
        CUDA_TRY(c, cudaStreamWaitEvent(S(c), c->ev_join, 0));
    }
    return EFVM_OK;
}

int capture_step_graph(efvm_ctx* c) {
    if (c->graph_exec) {
        cudaGraphExecDestroy(c->graph_exec);
        c->graph_exec = nullptr;
    }
    if (c->ibm && !is_3d(c) && !c->side) {
        CUDA_TRY(c, cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
        for (auto& ev : c->ev_fork) CUDA_TRY(c, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CUDA_TRY(c, cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    }
    const uint64_t before = c->launches;
    cudaGraph_t graph;
    CUDA_TRY(c, cudaStreamBeginCapture(S(c), cudaStreamCaptureModeThreadLocal));
    const int rc_enq = enqueue_rk3_step(c);
    cudaError_t e = cudaStreamEndCapture(S(c), &graph);
    c->graph_kernels = (int)(c->launches - before);
    c->launches = before;
    if (rc_enq) {
        if (e == cudaSuccess) cudaGraphDestroy(graph);
        return rc_enq;
    }
    if (e != cudaSuccess) return fail(c, EFVM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&c->graph_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(c, EFVM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    c->graph_valid = true;
    return EFVM_OK;
}

int read_state(efvm_ctx* c, DevState& s) {
    CUDA_TRY(c, cudaMemcpyAsync(&s, c->st, sizeof(DevState), cudaMemcpyDeviceToHost, S(c)));
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    return EFVM_OK;
}

bool bc_supported(int k) { return k >= EFVM_BC_SUPERSONIC_OUTFLOW && k <= EFVM_BC_PRESSURE_OUTLET; }
bool has_halo(const efvm_ctx* c) { return c->ph.halo_ylo || c->ph.halo_yhi; }

}  // namespace

namespace efvm {
void set_global_error(const std::string& msg) { g_last_error = msg; }
}  // namespace efvm

namespace efvm {

int setup_case(const efvm_grid& gr, const efvm_params& p, int row0, int rows, bool slab, Geometry& g, Physics& ph,
               std::string& err) {
    auto bad = [&](int code, const std::string& m) {
        err = m;
        return code;
    };
    if (gr.nz < 1) return bad(EFVM_ERR_INVALID_ARG, "nz must be >= 1");
    if (gr.ng != 2) return bad(EFVM_ERR_UNSUPPORTED, "only ng == 2 ghost layers are supported");
    const bool d3 = gr.nz > 1;  // a 3-D mesh: 5 conserved planes, z faces (efvm_kernels3d.cuh)
    if (d3) {
        if (slab) return bad(EFVM_ERR_UNSUPPORTED, "slabs are built for 2-D meshes (nz == 1)");
        if (p.precision != EFVM_PREC_FP64) return bad(EFVM_ERR_UNSUPPORTED, "3-D meshes run in FP64");
        if (p.parabolic_inflow) return bad(EFVM_ERR_UNSUPPORTED, "the parabolic inlet is a 2-D case system");
    }
    if (gr.nx < 2 || gr.ny < 1) return bad(EFVM_ERR_INVALID_ARG, "nx must be >= 2 and ny >= 1");
    for (int a = 0; a < 3; ++a)
        if (!(gr.hi[a] > gr.lo[a])) return bad(EFVM_ERR_INVALID_ARG, "bounds_hi must exceed bounds_lo");
    for (int a = 0; a < 3; ++a) {
        const bool lo_p = gr.bc[2 * a].kind == EFVM_BC_PERIODIC, hi_p = gr.bc[2 * a + 1].kind == EFVM_BC_PERIODIC;
        if (lo_p != hi_p)
            return bad(EFVM_ERR_INVALID_ARG,
                        "invalid periodic boundary configuration: periodic boundary on axis " + std::to_string(a) +
                            " requires both sides");
    }
    for (int s = 0; s < 6; ++s)
        if (!bc_supported(gr.bc[s].kind)) return bad(EFVM_ERR_INVALID_ARG, "unknown boundary kind");
    if ((gr.bc[EFVM_XLO].kind == EFVM_BC_PERIODIC && gr.nx < 2) || (gr.bc[EFVM_YLO].kind == EFVM_BC_PERIODIC && gr.ny < 2))
        return bad(EFVM_ERR_INVALID_ARG, "a periodic axis needs at least 2 cells (two ghost layers wrap)");
    if (!d3 && gr.bc[EFVM_ZLO].kind == EFVM_BC_PERIODIC)
        return bad(EFVM_ERR_UNSUPPORTED, "a periodic z axis has no meaning on a 2-D mesh");
    if (!(p.gamma > 1.0) || !(p.r_gas > 0.0)) return bad(EFVM_ERR_INVALID_ARG, "gamma must exceed 1, r_gas > 0");
    if (!(p.cfl > 0.0) && !(p.fixed_dt > 0.0)) return bad(EFVM_ERR_INVALID_ARG, "cfl or fixed_dt must be > 0");
    if (p.flux_scheme < 0 || p.flux_scheme > 2 || p.reconstruction < 0 || p.reconstruction > 1 || p.limiter < 0 ||
        p.limiter > 1 || p.integrator < 0 || p.integrator > 1 || p.precision < 0 || p.precision > 1 ||
        p.periodic_seam < 0 || p.periodic_seam > 1 || p.viscosity_model < 0 || p.viscosity_model > 1)
        return bad(EFVM_ERR_INVALID_ARG, "enum field out of range");
    if (p.sponge && !(p.sponge_x_end > p.sponge_x_start))
        return bad(EFVM_ERR_INVALID_ARG, "sponge_x_end must exceed sponge_x_start");
    if (slab && (row0 < 0 || rows < 2 || (int64_t)row0 + rows > gr.ny))
        return bad(EFVM_ERR_INVALID_ARG, "a slab needs rows >= 2 inside the grid: 0 <= row0, row0 + rows <= ny");

    g = Geometry{};
    ph = Physics{};
    g.nx = gr.nx;
    g.ny = rows;
    g.j_off = row0;
    g.pitch = ((XO + gr.nx + NG) + 7) / 8 * 8;
    g.plane = ((long long)(rows + 2 * YO) * g.pitch + 31) / 32 * 32;
    g.nz = gr.nz;
    g.layer = (long long)(rows + 2 * YO) * g.pitch;
    if (d3) g.plane = ((long long)(gr.nz + 4) * g.layer + 31) / 32 * 32;
    const int n[3] = {gr.nx, gr.ny, gr.nz};
    for (int a = 0; a < 3; ++a) {
        g.lo[a] = gr.lo[a];
        g.hi[a] = gr.hi[a];
        g.h[a] = (gr.hi[a] - gr.lo[a]) / (double)n[a];
    }
    g.cell_volume = g.h[0] * g.h[1] * g.h[2];
    g.inv_x = (g.h[1] * g.h[2]) / g.cell_volume;
    g.inv_y = (g.h[0] * g.h[2]) / g.cell_volume;
    g.inv_z = (g.h[0] * g.h[1]) / g.cell_volume;
    for (int a = 0; a < 3; ++a) g.inv_h[a] = 1.0 / g.h[a];
    ph.gamma = p.gamma;
    ph.r_gas = p.r_gas;
    ph.cfl = p.cfl;
    ph.fixed_dt = p.fixed_dt;
    ph.flux_scheme = p.flux_scheme;
    ph.reconstruction = p.reconstruction;
    ph.limiter = p.limiter;
    ph.integrator = p.integrator;
    ph.viscous = p.viscous;
    ph.viscosity_model = p.viscosity_model;
    ph.mu = p.mu;
    ph.precision = p.precision;
    ph.periodic_seam = p.periodic_seam;
    ph.periodic_x = gr.bc[EFVM_XLO].kind == EFVM_BC_PERIODIC;
    ph.periodic_y = gr.bc[EFVM_YLO].kind == EFVM_BC_PERIODIC;
    ph.periodic_z = d3 && gr.bc[EFVM_ZLO].kind == EFVM_BC_PERIODIC;
    if (slab) {
        // the periodic wrap of y, like the edges between slabs, goes through halos
        const bool per_y = ph.periodic_y != 0;
        ph.halo_ylo = row0 > 0 || per_y;
        ph.halo_yhi = row0 + rows < gr.ny || per_y;
        ph.seam_ylo = per_y && row0 == 0;
        ph.seam_yhi = per_y && row0 + rows == gr.ny;
        ph.periodic_y = 0;
    }
    for (int s = 0; s < 6; ++s) {
        ph.bc[s].kind = gr.bc[s].kind;
        ph.bc[s].rho = gr.bc[s].rho;
        ph.bc[s].u = gr.bc[s].u;
        ph.bc[s].v = gr.bc[s].v;
        ph.bc[s].w = gr.bc[s].w;
        ph.bc[s].p = gr.bc[s].p;
        ph.bc[s].t = gr.bc[s].t;
    }
    ph.parabolic_inflow = p.parabolic_inflow;
    ph.inflow_u_max = p.inflow_u_max;
    ph.inflow_height = p.inflow_height;
    ph.inflow_rho = p.inflow_rho;
    ph.sponge = p.sponge;
    ph.sponge_x_start = p.sponge_x_start;
    ph.sponge_x_end = p.sponge_x_end;
    ph.sponge_sigma = p.sponge_sigma;
    ph.sponge_u_max = p.sponge_u_max;
    ph.sponge_height = p.sponge_height;
    ph.sponge_rho = p.sponge_rho;
    ph.sponge_p = p.sponge_p;
    ph.body_force_x = p.body_force_x;
    ph.dx_inv2 = 1.0 / (g.h[0] * g.h[0]);
    ph.cp = p.gamma * p.r_gas / (p.gamma - 1.0);
    ph.cp_pr = ph.cp / 0.72;
    ph.cfl_visc_sum = 1.0 / (g.h[0] * g.h[0]) + 1.0 / (g.h[1] * g.h[1]) + 1.0 / (g.h[2] * g.h[2]);
    ph.inv_r_gas = 1.0 / p.r_gas;
    // the sponge's constants with the operations the device would apply (this file
    // is compiled without floating-point contraction): inv_w as in the 2-D and 3-D
    // sponges, p / (gamma - 1) as in prim_to_cons, and the 3-D uniform target
    // (rho, rho u_max, 0, 0, E) as prim_to_cons5 forms it
    const double gm1 = p.gamma - 1.0;
    ph.sponge_inv_w = 1.0 / (p.sponge_x_end - p.sponge_x_start);
    ph.sponge_e0 = p.sponge_p / gm1;
    {
        const double rho = p.sponge_rho, u = p.sponge_u_max, v = 0.0, w = 0.0;
        const double ke = (0.5 * rho) * ((u * u + v * v) + w * w);
        ph.sponge_t[0] = rho;
        ph.sponge_t[1] = rho * u;
        ph.sponge_t[2] = rho * v;
        ph.sponge_t[3] = rho * w;
        ph.sponge_t[4] = p.sponge_p / gm1 + ke;
    }
    return EFVM_OK;
}

// viscous_system's pre-inverted y weights from centroid distances (global row
// indices), crates/cfd_solver/src/lib.rs:484-493: y_im, y_ip, y_is per row.
std::vector<double> viscous_y_weights(const Geometry& g) {
    std::vector<double> yw(3 * (size_t)g.ny);
    for (int j = 0; j < g.ny; ++j) {
        const int jg = j + g.j_off;
        const double hm = centre_h(g.lo[1], g.h[1], jg) - centre_h(g.lo[1], g.h[1], jg - 1);
        const double hp = centre_h(g.lo[1], g.h[1], jg + 1) - centre_h(g.lo[1], g.h[1], jg);
        yw[j] = 1.0 / hm;
        yw[g.ny + j] = 1.0 / hp;
        yw[2 * g.ny + j] = 2.0 / (hm + hp);
    }
    return yw;
}

// The same weights along z (z_im, z_ip, z_is per layer) for a 3-D mesh.
std::vector<double> viscous_z_weights(const Geometry& g) {
    std::vector<double> zw(3 * (size_t)g.nz);
    for (int k = 0; k < g.nz; ++k) {
        const double hm = centre_h(g.lo[2], g.h[2], k) - centre_h(g.lo[2], g.h[2], k - 1);
        const double hp = centre_h(g.lo[2], g.h[2], k + 1) - centre_h(g.lo[2], g.h[2], k);
        zw[k] = 1.0 / hm;
        zw[g.nz + k] = 1.0 / hp;
        zw[2 * g.nz + k] = 2.0 / (hm + hp);
    }
    return zw;
}

}  // namespace efvm

extern "C" {

int efvm_abi_version(void) { return EFVM_ABI_VERSION; }

const char* efvm_last_error(const efvm_ctx* ctx) {
    if (ctx) return ctx->err.c_str();
    return g_last_error.c_str();
}

// efvm_create / efvm_create_slab: a context for global rows [row0, row0 + rows)
// of `grid`; `slab` marks the y sides that face another slab or the periodic
// wrap as halo sides.
static int create_impl(const efvm_grid* grid, const efvm_params* params, int32_t row0, int32_t rows, bool slab,
                       efvm_ctx** out) {
    if (!grid || !params || !out) return fail(nullptr, EFVM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    Geometry g;
    Physics ph;
    std::string err;
    const int rc = setup_case(*grid, *params, row0, rows, slab, g, ph, err);
    if (rc) return fail(nullptr, rc, err);
    efvm_ctx* c = new efvm_ctx();
    c->grid = *grid;
    c->params = *params;
    cudaGetDevice(&c->device);
    c->g = g;
    c->ph = ph;
    auto cleanup_fail = [&](int code) {
        efvm_destroy(c);
        return code;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        fail(nullptr, EFVM_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
        delete c;
        return EFVM_ERR_CUDA;
    }
    const size_t state_bytes = (size_t)(g.nz > 1 ? 5 : 4) * g.plane * sizeof(double);
    for (int k = 0; k < 3; ++k) {
        e = cudaMalloc(&c->U[k], state_bytes);
        if (e != cudaSuccess) {
            fail(nullptr, EFVM_ERR_OOM, std::string("cudaMalloc state: ") + cudaGetErrorString(e));
            return cleanup_fail(EFVM_ERR_OOM);
        }
        cudaMemsetAsync(c->U[k], 0, state_bytes, c->stream);
    }
    if (g.nz <= 1) {  // tensor maps of the TMA-fed stage kernel (none: the strip kernel only)
        bool ok = true;
        for (int k = 0; k < 3 && ok; ++k) ok = encode_state_map(g, c->U[k], false, &c->tmap[k]) == 0;
        ok = ok && encode_state_map(g, c->U[0], true, &c->tmap_u0) == 0;
        c->tmaps = ok;
    }
    e = cudaMalloc(&c->mask, (size_t)g.plane);
    if (e != cudaSuccess) return cleanup_fail(fail(nullptr, EFVM_ERR_OOM, "cudaMalloc mask"));
    cudaMemsetAsync(c->mask, 0, (size_t)g.plane, c->stream);
    const std::vector<double> yw = viscous_y_weights(g);
    if (cudaMalloc(&c->yw, yw.size() * sizeof(double)) != cudaSuccess) return cleanup_fail(fail(nullptr, EFVM_ERR_OOM, "cudaMalloc"));
    cudaMemcpyAsync(c->yw, yw.data(), yw.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (g.nz > 1) {
        const std::vector<double> zw = viscous_z_weights(g);
        if (cudaMalloc(&c->zw, zw.size() * sizeof(double)) != cudaSuccess)
            return cleanup_fail(fail(nullptr, EFVM_ERR_OOM, "cudaMalloc"));
        cudaMemcpyAsync(c->zw, zw.data(), zw.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    }
    if (cudaMalloc(&c->st, sizeof(DevState)) != cudaSuccess) return cleanup_fail(fail(nullptr, EFVM_ERR_OOM, "cudaMalloc"));
    DevState s0{};
    s0.active = 1;
    cudaMemcpyAsync(c->st, &s0, sizeof(DevState), cudaMemcpyHostToDevice, c->stream);
    c->n_partial = 296;
    if (cudaMalloc(&c->partial, 2 * c->n_partial * sizeof(double)) != cudaSuccess)
        return cleanup_fail(fail(nullptr, EFVM_ERR_OOM, "cudaMalloc"));
    if (cudaMalloc(&c->force_out, 12 * sizeof(double)) != cudaSuccess)
        return cleanup_fail(fail(nullptr, EFVM_ERR_OOM, "cudaMalloc"));
    if (cudaMalloc(&c->force_counter, sizeof(unsigned int)) != cudaSuccess)
        return cleanup_fail(fail(nullptr, EFVM_ERR_OOM, "cudaMalloc"));
    cudaMemsetAsync(c->force_counter, 0, sizeof(unsigned int), c->stream);
    cudaMemsetAsync(c->force_out, 0, 12 * sizeof(double), c->stream);
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cleanup_fail(fail(nullptr, EFVM_ERR_CUDA, std::string("create: ") + cudaGetErrorString(e)));
    *out = c;
    return EFVM_OK;
}

int efvm_create(const efvm_grid* grid, const efvm_params* params, efvm_ctx** out) {
    return create_impl(grid, params, 0, grid ? grid->ny : 0, false, out);
}

int efvm_create_slab(const efvm_grid* grid, const efvm_params* params, int32_t row0, int32_t rows,
                     efvm_ctx** out) {
    return create_impl(grid, params, row0, rows, true, out);
}

int efvm_destroy(efvm_ctx* c) {
    if (!c) return EFVM_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    for (auto& side : c->peer_ipc)
        for (void* p : side)
            if (p) cudaIpcCloseMemHandle(p);
    for (int k = 0; k < 3; ++k) cudaFree(c->U[k]);
    cudaFree(c->mask);
    cudaFree(c->yw);
    cudaFree(c->zw);
    cudaFree(c->st);
    cudaFree(c->partial);
    cudaFree(c->staging);
    cudaFree(c->cyl_dev);
    cudaFree(c->sph_dev);
    cudaFree(c->ghosts3_dev);
    cudaFree(c->markers3_dev);
    cudaFree(c->ghosts_dev);
    cudaFree(c->markers_dev);
    cudaFree(c->zg0);
    cudaFree(c->zfill);
    cudaFree(c->force_out);
    cudaFree(c->force_partials);
    cudaFree(c->force_counter);
    cudaFree(c->history);
    cudaFree(c->corr);
    cudaFree(c->fallbacks);
    cudaFree(c->out_fields);
    cudaFree(c->prims);
    for (auto& ev : c->ev_fork)
        if (ev) cudaEventDestroy(ev);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return EFVM_OK;
}

static int transfer_state(efvm_ctx* c, double* base, int64_t si, int64_t sj, int64_t sv, bool upload) {
    if (!c || !base) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (upload) {  // pending forces read the state this replaces
        const int rcf = finish_forces(c);
        if (rcf) return rcf;
    }
    const Geometry& g = c->g;
    // the host span the strides address, [min offset, max offset]
    int64_t lo = 0, hi = 0;
    const int64_t corners[3] = {(int64_t)(g.nx - 1) * si, (int64_t)(g.ny - 1) * sj, 4 * sv};
    for (int k = 0; k < 3; ++k) {
        lo += std::min<int64_t>(0, corners[k]);
        hi += std::max<int64_t>(0, corners[k]);
    }
    const int64_t span = hi - lo + 1;
    const bool dense = span == (int64_t)g.nx * g.ny * 5;
    int rc = ensure_staging(c, (size_t)span * sizeof(double));
    if (rc) return rc;
    double* host0 = base + lo;
    double* dev0 = c->staging - lo;  // device pointer of element offset 0
    double* q = cur_buf(c);
    if (upload) {
        CUDA_TRY(c, cudaMemcpyAsync(c->staging, host0, (size_t)span * sizeof(double), cudaMemcpyHostToDevice, S(c)));
        c->launches += launch_pack(g, dev0, si, sj, sv, q, 1, S(c));
        c->lam_stale = true;
        c->ghosts_stale = true;
    } else {
        if (!dense)  // keep the caller's values in the gaps of a sparse layout
            CUDA_TRY(c, cudaMemcpyAsync(c->staging, host0, (size_t)span * sizeof(double), cudaMemcpyHostToDevice, S(c)));
        c->launches += launch_pack(g, dev0, si, sj, sv, q, 0, S(c));
        CUDA_TRY(c, cudaMemcpyAsync(host0, c->staging, (size_t)span * sizeof(double), cudaMemcpyDeviceToHost, S(c)));
    }
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    CUDA_TRY(c, cudaGetLastError());
    return EFVM_OK;
}

int efvm_upload_state(efvm_ctx* c, const double* base, int64_t si, int64_t sj, int64_t sv) {
    if (is_3d(c)) return refuse_3d(c, "efvm_upload_state (use efvm_upload_state_3d)");
    return transfer_state(c, const_cast<double*>(base), si, sj, sv, true);
}

int efvm_download_state(efvm_ctx* c, double* base, int64_t si, int64_t sj, int64_t sv) {
    if (is_3d(c)) return refuse_3d(c, "efvm_download_state (use efvm_download_state_3d)");
    return transfer_state(c, base, si, sj, sv, false);
}

// The 3-D form of transfer_state: element (i, j, k, v) at i si + j sj + k sk + v sv.
static int transfer_state3(efvm_ctx* c, double* base, int64_t si, int64_t sj, int64_t sk, int64_t sv, bool upload) {
    if (!c || !base) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (!is_3d(c)) return transfer_state(c, base, si, sj, sv, upload);
    const Geometry& g = c->g;
    int64_t lo = 0, hi = 0;
    const int64_t corners[4] = {(int64_t)(g.nx - 1) * si, (int64_t)(g.ny - 1) * sj, (int64_t)(g.nz - 1) * sk, 4 * sv};
    for (int k = 0; k < 4; ++k) {
        lo += std::min<int64_t>(0, corners[k]);
        hi += std::max<int64_t>(0, corners[k]);
    }
    const int64_t span = hi - lo + 1;
    const bool dense = span == (int64_t)g.nx * g.ny * g.nz * 5;
    int rc = ensure_staging(c, (size_t)span * sizeof(double));
    if (rc) return rc;
    double* host0 = base + lo;
    double* dev0 = c->staging - lo;
    double* q = cur_buf(c);
    if (upload) {
        CUDA_TRY(c, cudaMemcpyAsync(c->staging, host0, (size_t)span * sizeof(double), cudaMemcpyHostToDevice, S(c)));
        c->launches += launch_pack3(g, dev0, si, sj, sk, sv, q, 1, S(c));
        c->lam_stale = true;
        c->ghosts_stale = true;
    } else {
        if (!dense)
            CUDA_TRY(c, cudaMemcpyAsync(c->staging, host0, (size_t)span * sizeof(double), cudaMemcpyHostToDevice, S(c)));
        c->launches += launch_pack3(g, dev0, si, sj, sk, sv, q, 0, S(c));
        CUDA_TRY(c, cudaMemcpyAsync(host0, c->staging, (size_t)span * sizeof(double), cudaMemcpyDeviceToHost, S(c)));
    }
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    CUDA_TRY(c, cudaGetLastError());
    return EFVM_OK;
}

int efvm_upload_state_3d(efvm_ctx* c, const double* base, int64_t si, int64_t sj, int64_t sk, int64_t sv) {
    return transfer_state3(c, const_cast<double*>(base), si, sj, sk, sv, true);
}

int efvm_download_state_3d(efvm_ctx* c, double* base, int64_t si, int64_t sj, int64_t sk, int64_t sv) {
    return transfer_state3(c, base, si, sj, sk, sv, false);
}

int efvm_get_solver_state(efvm_ctx* c, efvm_solver_state* out) {
    if (!c || !out) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    DevState s;
    int rc = read_state(c, s);
    if (rc) return rc;
    out->dt = s.dt;
    out->time = s.time;
    out->step = s.step;
    out->rk_stage = c->rk_stage;
    out->completed_full_step = s.completed;
    if (s.nonphysical & 8)
        return fail(c, EFVM_ERR_TIMEOUT, "a stage kernel's wait for a row of its shared-memory ring ran out");
    if (s.nonphysical) return fail(c, EFVM_ERR_NONPHYSICAL, "the state went non-physical (rho<=0, p<=0 or NaN)");
    return EFVM_OK;
}

int efvm_set_solver_state(efvm_ctx* c, const efvm_solver_state* in) {
    if (!c || !in) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    {
        const int rcf = finish_forces(c);
        if (rcf) return rcf;
    }
    if (in->rk_stage < 0 || in->rk_stage > 2) return fail(c, EFVM_ERR_INVALID_ARG, "rk_stage must be 0..2");
    DevState s;
    int rc = read_state(c, s);
    if (rc) return rc;
    s.dt = in->dt;
    s.time = in->time;
    s.step = in->step;
    s.step_par = (int)(in->step & 1ull);
    s.rk_stage = in->rk_stage;
    s.completed = in->completed_full_step;
    CUDA_TRY(c, cudaMemcpyAsync(c->st, &s, sizeof(DevState), cudaMemcpyHostToDevice, S(c)));
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    c->rk_stage = in->rk_stage;
    c->lam_stale = true;
    return EFVM_OK;
}

int efvm_set_flux_correction(efvm_ctx* c, efvm_nn* nn, float sensor) {
    if (!c) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (!nn) {
        c->nn = nullptr;
        c->graph_valid = false;
        return EFVM_OK;
    }
    if (is_3d(c)) return refuse_3d(c, "the flux correction");
    if (!c->ph.periodic_x || !c->ph.periodic_y || has_halo(c) || c->ibm)
        return fail(c, EFVM_ERR_UNSUPPORTED, "the flux correction needs a periodic grid without IBM or slabs");
    if (c->params.reconstruction != EFVM_RECON_MUSCL || c->params.flux_scheme != EFVM_FLUX_HLLC || c->ph.viscous)
        return fail(c, EFVM_ERR_UNSUPPORTED, "the flux correction runs inviscid with MUSCL + HLLC");
    if (((long long)c->g.nx * c->g.ny) % 64 || c->g.nx < 5 || c->g.ny < 5)
        return fail(c, EFVM_ERR_UNSUPPORTED, "the flux correction needs nx*ny a multiple of 64 and nx, ny >= 5");
    if (!c->corr) {
        CUDA_TRY(c, cudaMalloc(&c->corr, 8ull * c->g.nx * c->g.ny * sizeof(float)));
        CUDA_TRY(c, cudaMalloc(&c->fallbacks, sizeof(unsigned long long)));
        CUDA_TRY(c, cudaMalloc(&c->prims, (size_t)c->g.nx * c->g.ny * sizeof(float4)));
    }
    CUDA_TRY(c, cudaMemsetAsync(c->fallbacks, 0, sizeof(unsigned long long), S(c)));
    if (nn_prepare_launches()) return fail(c, EFVM_ERR_CUDA, "flux correction: kernel attributes");
    c->nn = nn;
    c->sensor = sensor;
    c->corr_faces = 0;
    c->graph_valid = false;
    return EFVM_OK;
}

int efvm_output_fields(efvm_ctx* c, double* host_out, int32_t async) {
    if (is_3d(c)) return refuse_3d(c, "efvm_output_fields");
    if (!c || !host_out) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    const size_t bytes = (size_t)7 * c->g.nx * c->g.ny * sizeof(double);
    if (!c->out_fields) CUDA_TRY(c, cudaMalloc(&c->out_fields, bytes));
    c->launches += launch_output_fields(c->g, c->ph, cur_buf(c), c->out_fields, S(c));
    CUDA_TRY(c, cudaMemcpyAsync(host_out, c->out_fields, bytes, cudaMemcpyDeviceToHost, S(c)));
    if (!async) CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    return EFVM_OK;
}

int efvm_synchronize(efvm_ctx* c) {
    if (!c) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    return EFVM_OK;
}

int efvm_write_vtk(efvm_ctx* c, const char* path) {
    if (is_3d(c)) return refuse_3d(c, "efvm_write_vtk");
    if (!c || !path) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    const int nx = c->g.nx, ny = c->g.ny;
    const long long n = (long long)nx * ny;
    std::vector<double> f(7 * (size_t)n);
    int rc = efvm_output_fields(c, f.data(), 0);
    if (rc) return rc;
    FILE* fp = std::fopen(path, "w");
    if (!fp) return fail(c, EFVM_ERR_INVALID_ARG, std::string("efvm_write_vtk: cannot open ") + path);
    // fmt_e: %.10e (two or more exponent digits), non-finite values as zero
    auto e = [&](double x) { std::fprintf(fp, "%.10e", std::isfinite(x) ? x : 0.0); };
    std::fprintf(fp, "# vtk DataFile Version 3.0\ndev_field_efvm output\nASCII\nDATASET RECTILINEAR_GRID\n");
    std::fprintf(fp, "DIMENSIONS %d %d %d\n", nx + 1, ny + 1, 2);
    const int ns[3] = {nx, ny, 1};
    const char* lab[3] = {"X", "Y", "Z"};
    for (int a = 0; a < 3; ++a) {
        std::fprintf(fp, "%s_COORDINATES %d double\n", lab[a], ns[a] + 1);
        const int off = a == 1 ? c->g.j_off : 0;
        for (int m = 0; m <= ns[a]; ++m) {
            // face = centroid - half spacing, then the last centroid + half spacing
            const int mm = m < ns[a] ? m : ns[a] - 1;
            const double cc = centre_h(c->g.lo[a], c->g.h[a], mm + off);
            e(m < ns[a] ? cc - 0.5 * c->g.h[a] : cc + 0.5 * c->g.h[a]);
            std::fputc('\n', fp);
        }
    }
    std::fprintf(fp, "CELL_DATA %lld\n", n);
    const char* names[3] = {"density", "pressure", "temperature"};
    for (int k = 0; k < 3; ++k) {
        std::fprintf(fp, "SCALARS %s double 1\nLOOKUP_TABLE default\n", names[k]);
        for (long long t = 0; t < n; ++t) {
            e(f[k * n + t]);
            std::fputc('\n', fp);
        }
    }
    std::fprintf(fp, "VECTORS velocity double\n");
    for (long long t = 0; t < n; ++t) {
        e(f[3 * n + t]);
        std::fputc(' ', fp);
        e(f[4 * n + t]);
        std::fputc(' ', fp);
        e(f[5 * n + t]);
        std::fputc('\n', fp);
    }
    std::fprintf(fp, "SCALARS mach double 1\nLOOKUP_TABLE default\n");
    for (long long t = 0; t < n; ++t) {
        e(f[6 * n + t]);
        std::fputc('\n', fp);
    }
    const bool ok = std::fclose(fp) == 0;
    if (!ok) return fail(c, EFVM_ERR_INVALID_ARG, std::string("efvm_write_vtk: write failed for ") + path);
    return EFVM_OK;
}

int efvm_body_loads(efvm_ctx* c, int32_t n_bodies, double* out) {
    if (is_3d(c)) return refuse_3d(c, "efvm_body_loads");
    if (!c || !out || n_bodies < 0) return fail(c, EFVM_ERR_INVALID_ARG, "invalid argument");
    if (!c->ibm) return fail(c, EFVM_ERR_INVALID_ARG, "efvm_body_loads: no cylinders are set");
    const int nb = (int)(c->cyl_host.size() / 3);
    if (n_bodies > nb) return fail(c, EFVM_ERR_INVALID_ARG, "efvm_body_loads: more bodies asked than cylinders set");
    if (c->geom_dirty) {
        int rc = prologue(c);
        if (rc) return rc;
    }
    const size_t bytes = (size_t)9 * nb * sizeof(double);
    int rc = ensure_staging(c, bytes);
    if (rc) return rc;
    // centres (cx, cy) after the loads in the staging buffer
    rc = ensure_staging(c, bytes + (size_t)2 * nb * sizeof(double));
    if (rc) return rc;
    std::vector<double> centres(2 * nb);
    for (int b = 0; b < nb; ++b) {
        centres[2 * b] = c->cyl_host[3 * b];
        centres[2 * b + 1] = c->cyl_host[3 * b + 1];
    }
    double* d_out = c->staging;
    double* d_cen = c->staging + 9 * nb;
    CUDA_TRY(c, cudaMemcpyAsync(d_cen, centres.data(), centres.size() * sizeof(double), cudaMemcpyHostToDevice, S(c)));
    c->launches += launch_body_loads(c->g, c->ph, c->ibm_desc, cur_buf(c), d_cen, nb, c->ibm_desc.n_markers / nb,
                                     d_out, S(c));
    std::vector<double> all(9 * nb);
    CUDA_TRY(c, cudaMemcpyAsync(all.data(), d_out, bytes, cudaMemcpyDeviceToHost, S(c)));
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    std::copy(all.begin(), all.begin() + 9 * n_bodies, out);
    return EFVM_OK;
}

int efvm_correction_stats(efvm_ctx* c, uint64_t* faces, uint64_t* fallbacks) {
    if (!c || !faces || !fallbacks) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    unsigned long long fb = 0;
    if (c->fallbacks) {
        CUDA_TRY(c, cudaMemcpyAsync(&fb, c->fallbacks, sizeof(fb), cudaMemcpyDeviceToHost, S(c)));
        CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    }
    *faces = c->corr_faces;
    *fallbacks = fb;
    return EFVM_OK;
}

int efvm_prepare(efvm_ctx* c) {
    if (!c) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (c->control_dirty) sync_control(c, 0, 0.0, 0);
    int rc = prologue(c);
    if (rc) return rc;
    CUDA_TRY(c, cudaGetLastError());
    return EFVM_OK;
}

static int halo_rows(efvm_ctx* c, int32_t side, double* buf, int unpack) {
    if (is_3d(c)) return refuse_3d(c, "the slab halo exchange");
    if (!c || !buf) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (side != EFVM_YLO && side != EFVM_YHI) return fail(c, EFVM_ERR_INVALID_ARG, "side must be EFVM_YLO or EFVM_YHI");
    if (c->g.ny < 2) return fail(c, EFVM_ERR_INVALID_ARG, "halo rows need ny >= 2");
    if (unpack && !(side == EFVM_YLO ? c->ph.halo_ylo : c->ph.halo_yhi))
        return fail(c, EFVM_ERR_INVALID_ARG, "efvm_halo_unpack: that side does not face another slab");
    int j0;
    if (unpack) j0 = side == EFVM_YLO ? -2 : c->g.ny;
    else j0 = side == EFVM_YLO ? 0 : c->g.ny - 2;
    c->launches += launch_halo_rows(c->g, cur_buf(c), buf, j0, unpack, S(c));
    CUDA_TRY(c, cudaGetLastError());
    return EFVM_OK;
}

int efvm_halo_pack(efvm_ctx* c, int32_t side, double* dev_buf) { return halo_rows(c, side, dev_buf, 0); }

int efvm_halo_unpack(efvm_ctx* c, int32_t side, const double* dev_buf) {
    return halo_rows(c, side, const_cast<double*>(dev_buf), 1);
}

int efvm_get_state_buffers(efvm_ctx* c, double* bufs[3], int64_t* plane, int32_t* rows) {
    if (!c || !bufs || !plane || !rows) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (is_3d(c)) return refuse_3d(c, "efvm_get_state_buffers");
    for (int k = 0; k < 3; ++k) bufs[k] = c->U[k];
    *plane = c->g.plane;
    *rows = c->g.ny;
    return EFVM_OK;
}

int efvm_set_halo_peer(efvm_ctx* c, int32_t side, double* const peer_bufs[3], int64_t peer_plane,
                       int32_t peer_rows) {
    if (!c) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (is_3d(c)) return refuse_3d(c, "efvm_set_halo_peer");
    if (side != EFVM_YLO && side != EFVM_YHI) return fail(c, EFVM_ERR_INVALID_ARG, "side must be EFVM_YLO or EFVM_YHI");
    if (!(side == EFVM_YLO ? c->ph.halo_ylo : c->ph.halo_yhi))
        return fail(c, EFVM_ERR_INVALID_ARG, "efvm_set_halo_peer: that side does not face another slab");
    const int s = side == EFVM_YLO ? 0 : 1;
    if (!peer_bufs) {  // back to the pack / unpack exchange (and unmap a neighbour's IPC buffers)
        for (int k = 0; k < 3; ++k) {
            if (c->peer_ipc[s][k]) cudaIpcCloseMemHandle(c->peer_ipc[s][k]);
            c->peer_ipc[s][k] = nullptr;
            c->peer_bufs[s][k] = nullptr;
        }
        c->peer_plane[s] = 0;
        c->peer_rows[s] = 0;
        c->graph_valid = false;
        return EFVM_OK;
    }
    for (int k = 0; k < 3; ++k)
        if (!peer_bufs[k]) return fail(c, EFVM_ERR_INVALID_ARG, "efvm_set_halo_peer: null peer buffer");
    if (peer_rows < 2 || peer_plane < (int64_t)(peer_rows + 2 * YO) * c->g.pitch)
        return fail(c, EFVM_ERR_INVALID_ARG, "efvm_set_halo_peer: the peer needs >= 2 rows and a plane of "
                                             "(rows + 4) x pitch doubles");
    for (int k = 0; k < 3; ++k) c->peer_bufs[s][k] = peer_bufs[k];
    c->peer_plane[s] = peer_plane;
    c->peer_rows[s] = peer_rows;
    c->graph_valid = false;
    return EFVM_OK;
}

int efvm_get_state_ipc(efvm_ctx* c, void* handles) {
    if (!c || !handles) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (is_3d(c)) return refuse_3d(c, "efvm_get_state_ipc");
    auto* h = static_cast<cudaIpcMemHandle_t*>(handles);
    for (int k = 0; k < 3; ++k) CUDA_TRY(c, cudaIpcGetMemHandle(&h[k], c->U[k]));
    return EFVM_OK;
}

static void close_peer_ipc(efvm_ctx* c, int s) {
    for (int k = 0; k < 3; ++k) {
        if (c->peer_ipc[s][k]) cudaIpcCloseMemHandle(c->peer_ipc[s][k]);
        c->peer_ipc[s][k] = nullptr;
    }
}

int efvm_set_halo_peer_ipc(efvm_ctx* c, int32_t side, const void* handles, int64_t peer_plane, int32_t peer_rows) {
    if (!c || !handles) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (side != EFVM_YLO && side != EFVM_YHI) return fail(c, EFVM_ERR_INVALID_ARG, "side must be EFVM_YLO or EFVM_YHI");
    const int s = side == EFVM_YLO ? 0 : 1;
    const auto* h = static_cast<const cudaIpcMemHandle_t*>(handles);
    void* opened[3] = {nullptr, nullptr, nullptr};
    for (int k = 0; k < 3; ++k) {
        const cudaError_t e = cudaIpcOpenMemHandle(&opened[k], h[k], cudaIpcMemLazyEnablePeerAccess);
        if (e != cudaSuccess) {
            for (int q = 0; q < k; ++q) cudaIpcCloseMemHandle(opened[q]);
            return fail(c, EFVM_ERR_CUDA, std::string("efvm_set_halo_peer_ipc: cudaIpcOpenMemHandle: ") +
                                              cudaGetErrorString(e));
        }
    }
    double* bufs[3] = {static_cast<double*>(opened[0]), static_cast<double*>(opened[1]),
                       static_cast<double*>(opened[2])};
    const int rc = efvm_set_halo_peer(c, side, bufs, peer_plane, peer_rows);
    if (rc) {
        for (auto* p : opened) cudaIpcCloseMemHandle(p);
        return rc;
    }
    close_peer_ipc(c, s);  // a mapping this one replaces
    for (int k = 0; k < 3; ++k) c->peer_ipc[s][k] = opened[k];
    return EFVM_OK;
}

int efvm_wave_speed_slot(efvm_ctx* c, uint64_t** dev_slot) {
    if (is_3d(c)) return refuse_3d(c, "efvm_wave_speed_slot");
    if (!c || !dev_slot) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    DevState s;
    int rc = read_state(c, s);
    if (rc) return rc;
    if (!s.ext_lam) {
        s.ext_lam = 1;
        s.lam_ext = 0ull;
        CUDA_TRY(c, cudaMemcpyAsync(c->st, &s, sizeof(DevState), cudaMemcpyHostToDevice, S(c)));
        CUDA_TRY(c, cudaStreamSynchronize(S(c)));
        c->lam_stale = true;  // the next prologue measures the current state into the slot
    }
    *dev_slot = reinterpret_cast<uint64_t*>(&c->st->lam_ext);
    return EFVM_OK;
}

int efvm_substep(efvm_ctx* c) {
    if (!c) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    int rc0 = finish_forces(c);
    if (rc0) return rc0;
    if (c->control_dirty) sync_control(c, 0, 0.0, 0);
    int rc = prologue(c);
    if (rc) return rc;
    if (c->params.integrator == EFVM_INTEGRATOR_EULER) {
        double* in = c->U[c->euler_cur];
        double* outb = c->U[c->euler_cur ^ 1];
        enqueue_substage(c, 3, in, outb, true);
        c->euler_cur ^= 1;
    } else {
        const int s = c->rk_stage;
        double* in = c->U[s];
        double* outb = c->U[(s + 1) % 3];
        enqueue_substage(c, s, in, outb, s == 0);
        if (c->nn) c->corr_faces += 2ull * c->g.nx * c->g.ny;
        c->rk_stage = (s + 1) % 3;
    }
    CUDA_TRY(c, cudaGetLastError());
    return EFVM_OK;
}

int efvm_step(efvm_ctx* c, int64_t n_steps, int32_t stop_at_t, double t_stop, double* force_history,
              efvm_step_info* info) {
    if (!c) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (n_steps < 0) return fail(c, EFVM_ERR_INVALID_ARG, "n_steps must be >= 0");
    if (has_halo(c))
        return fail(c, EFVM_ERR_UNSUPPORTED, "a slab advances by efvm_substep with a halo exchange per stage");
    if (c->params.integrator != EFVM_INTEGRATOR_EULER && c->rk_stage != 0)
        return fail(c, EFVM_ERR_INVALID_ARG, "efvm_step must start at a step boundary (rk_stage == 0)");
    const bool async = !stop_at_t && !force_history && !info;
    DevState s_before{};
    int rc = EFVM_OK;
    if (!async) {
        rc = read_state(c, s_before);
        if (rc) return rc;
    }
    const int subs = c->params.integrator == EFVM_INTEGRATOR_EULER ? 1 : 3;
    const long long cap = force_history && c->ibm ? (long long)subs * n_steps : 0;
    if (cap > c->history_cap) {
        cudaFree(c->history);
        c->history = nullptr;
        c->history_cap = 0;
        CUDA_TRY(c, cudaMalloc(&c->history, (size_t)cap * 6 * sizeof(double)));
        c->history_cap = cap;
        c->graph_valid = false;
    }
    if (c->graph_with_history != (cap != 0)) c->graph_valid = false;
    c->graph_with_history = cap != 0;
    if (!async || c->control_dirty) {
        // forces a previous call left pending go into that call's history, not this one's
        rc = finish_forces(c);
        if (rc) return rc;
        sync_control(c, stop_at_t, t_stop, cap);
    }
    rc = prologue(c);  // may rebuild the IBM descriptor (first step after set_cylinders)
    if (rc) return rc;
    c->ibm_desc.history = cap ? c->history : nullptr;
    if (c->params.integrator == EFVM_INTEGRATOR_EULER) {
        for (int64_t k = 0; k < n_steps; ++k) {
            double* in = c->U[c->euler_cur];
            double* outb = c->U[c->euler_cur ^ 1];
            enqueue_substage(c, 3, in, outb, true);
            c->euler_cur ^= 1;
        }
    } else {
        if (!c->graph_valid) {
            rc = capture_step_graph(c);
            if (rc) return rc;
        }
        const int64_t chunk = 64;
        for (int64_t k = 0; k < n_steps; ++k) {
            CUDA_TRY(c, cudaGraphLaunch(c->graph_exec, S(c)));
            c->launches += c->graph_kernels;
            if (c->nn) c->corr_faces += 6ull * c->g.nx * c->g.ny;
            if (stop_at_t && (k + 1) % chunk == 0 && k + 1 < n_steps) {
                DevState s;
                rc = read_state(c, s);
                if (rc) return rc;
                if (!s.active) break;
            }
        }
    }
    CUDA_TRY(c, cudaGetLastError());
    if (async) return EFVM_OK;
    rc = finish_forces(c);  // the last step's stage-3 forces, for the history and later reads
    if (rc) return rc;
    DevState s;
    rc = read_state(c, s);
    if (rc) return rc;
    if (cap && s.hist_pos > 0)
        CUDA_TRY(c, cudaMemcpy(force_history, c->history, (size_t)s.hist_pos * 6 * sizeof(double),
                               cudaMemcpyDeviceToHost));
    else if (force_history && !c->ibm)
        std::memset(force_history, 0, (size_t)subs * n_steps * 6 * sizeof(double));
    if (info) {
        info->steps_done = (int64_t)(s.step - s_before.step);
        info->substeps_done = info->steps_done * subs;
        info->time = s.time;
        info->dt = s.dt;
        info->stopped_at_t_stop = (stop_at_t && s.time >= t_stop) ? 1 : 0;
    }
    c->control_dirty = stop_at_t != 0 || cap != 0;
    if (s.nonphysical & 8)
        return fail(c, EFVM_ERR_TIMEOUT, "a stage kernel's wait for a row of its shared-memory ring ran out");
    if (s.nonphysical) return fail(c, EFVM_ERR_NONPHYSICAL, "the state went non-physical (rho<=0, p<=0 or NaN)");
    return EFVM_OK;
}

int efvm_cfl(efvm_ctx* c, double* dt_out) {
    if (!c || !dt_out) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (c->ph.fixed_dt > 0.0) {
        *dt_out = c->ph.fixed_dt;
        return EFVM_OK;
    }
    c->launches += launch_cfl(c->g, c->ph, cur_buf(c), c->st, S(c));
    DevState s;
    int rc = read_state(c, s);
    if (rc) return rc;
    double lam;
    std::memcpy(&lam, s.ext_lam ? &s.lam_ext : &s.lam[s.lam_idx], sizeof(double));
    *dt_out = lam > 0.0 ? c->ph.cfl / lam : std::numeric_limits<double>::infinity();
    if (c->rk_stage == 0) c->lam_stale = false;
    else c->lam_stale = true;
    return EFVM_OK;
}

int efvm_set_cylinders(efvm_ctx* c, const efvm_cylinder* cyl, int32_t n, const double fs[5]) {
    if (is_3d(c)) return refuse_3d(c, "efvm_set_cylinders");
    if (!c || (n > 0 && (!cyl || !fs)) || n < 0) return fail(c, EFVM_ERR_INVALID_ARG, "invalid cylinder arguments");
    {  // pending forces belong to the bodies being replaced
        const int rcf = finish_forces(c);
        if (rcf) return rcf;
    }
    if (n == 0) {
        c->ibm = false;
        c->graph_valid = false;
        return EFVM_OK;
    }
    if (has_halo(c)) return fail(c, EFVM_ERR_UNSUPPORTED, "IBM cylinders are not supported on a slab");
    c->cyl_host.clear();
    c->disc_motion.clear();
    c->cyl_markers = 64;
    c->disc_rule = false;
    for (int b = 0; b < n; ++b) {
        if (!(cyl[b].radius > 0.0)) return fail(c, EFVM_ERR_INVALID_ARG, "cylinder radius must be > 0");
        c->cyl_host.push_back(cyl[b].cx);
        c->cyl_host.push_back(cyl[b].cy);
        c->cyl_host.push_back(cyl[b].radius);
    }
    // MaskConsts of CylinderIbmPlugin::build, crates/cfd_ibm/src/lib.rs:665-669:
    // stagnant = freestream at rest (same rho and internal energy), ambient = freestream
    const double ke = 0.5 * (fs[1] * fs[1] + fs[2] * fs[2] + fs[3] * fs[3]) / fs[0];
    const double st5[5] = {fs[0], 0.0, 0.0, 0.0, fs[4] - ke};
    std::memcpy(c->stagnant, st5, sizeof(st5));
    std::memcpy(c->ambient, fs, 5 * sizeof(double));
    if (c->cyl_dev) cudaFree(c->cyl_dev);
    c->cyl_dev = nullptr;
    CUDA_TRY(c, cudaMalloc(&c->cyl_dev, c->cyl_host.size() * sizeof(double)));
    CUDA_TRY(c, cudaMemcpy(c->cyl_dev, c->cyl_host.data(), c->cyl_host.size() * sizeof(double), cudaMemcpyHostToDevice));
    c->ibm = true;
    c->geom_dirty = true;
    c->graph_valid = false;
    return EFVM_OK;
}

int efvm_set_discs(efvm_ctx* c, const efvm_disc* d, int32_t n, int32_t n_theta, const double fs[5]) {
    if (is_3d(c)) return refuse_3d(c, "efvm_set_discs");
    if (!c || n < 0 || n_theta < 1 || (n > 0 && (!d || !fs))) return fail(c, EFVM_ERR_INVALID_ARG, "invalid disc arguments");
    std::vector<efvm_cylinder> cyl((size_t)n);
    for (int b = 0; b < n; ++b) cyl[b] = efvm_cylinder{d[b].cx, d[b].cy, d[b].radius};
    const int rc = efvm_set_cylinders(c, n ? cyl.data() : nullptr, n, fs);
    if (rc || n == 0) return rc;
    c->disc_motion.clear();
    for (int b = 0; b < n; ++b) {
        c->disc_motion.push_back(d[b].vx);
        c->disc_motion.push_back(d[b].vy);
        c->disc_motion.push_back(d[b].omega);
    }
    c->cyl_markers = n_theta;
    c->disc_rule = true;
    return EFVM_OK;
}

int efvm_set_spheres(efvm_ctx* c, const efvm_sphere* sph, int32_t n, int32_t n_markers, const double fs[5]) {
    if (!c || n < 0 || n_markers < 0 || (n > 0 && (!sph || !fs)))
        return fail(c, EFVM_ERR_INVALID_ARG, "invalid sphere arguments");
    if (!is_3d(c))
        return fail(c, EFVM_ERR_UNSUPPORTED,
                    "spheres are 3-D bodies: efvm_set_spheres needs nz > 1 (efvm_set_cylinders is the 2-D form)");
    if (n == 0) {
        c->ibm = false;
        c->graph_valid = false;
        return EFVM_OK;
    }
    std::vector<double> h;
    for (int b = 0; b < n; ++b) {
        if (!(sph[b].radius > 0.0)) return fail(c, EFVM_ERR_INVALID_ARG, "sphere radius must be > 0");
        const double v[10] = {sph[b].cx, sph[b].cy, sph[b].cz, sph[b].radius, sph[b].vx,
                              sph[b].vy, sph[b].vz, sph[b].wx, sph[b].wy, sph[b].wz};
        h.insert(h.end(), v, v + 10);
    }
    // MaskConsts of SphereIbmPlugin::build, crates/cfd_ibm/src/sphere.rs:277-279
    const double ke = 0.5 * (fs[1] * fs[1] + fs[2] * fs[2] + fs[3] * fs[3]) / fs[0];
    const double st5[5] = {fs[0], 0.0, 0.0, 0.0, fs[4] - ke};
    std::memcpy(c->stagnant, st5, sizeof(st5));
    std::memcpy(c->ambient, fs, 5 * sizeof(double));
    if (c->sph_dev && c->sph_host.size() != h.size()) {
        cudaFree(c->sph_dev);
        c->sph_dev = nullptr;
    }
    if (!c->sph_dev) CUDA_TRY(c, cudaMalloc(&c->sph_dev, h.size() * sizeof(double)));
    CUDA_TRY(c, cudaMemcpyAsync(c->sph_dev, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, S(c)));
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    c->sph_host = h;
    c->sphere_markers = n_markers;
    c->ibm = true;
    c->geom_dirty = true;
    c->graph_valid = false;
    return EFVM_OK;
}

static int read_forces(efvm_ctx* c, double* out, int offset) {
    if (!c || !out) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (!c->ibm) {
        for (int d = 0; d < 6; ++d) out[d] = 0.0;
        return EFVM_OK;
    }
    const int rc = finish_forces(c);
    if (rc) return rc;
    CUDA_TRY(c, cudaMemcpyAsync(out, c->force_out + offset, 6 * sizeof(double), cudaMemcpyDeviceToHost, S(c)));
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    return EFVM_OK;
}

int efvm_marker_force(efvm_ctx* c, double out[6]) { return read_forces(c, out, 0); }
int efvm_wall_force(efvm_ctx* c, double out[6]) { return read_forces(c, out, 6); }

int efvm_ibm_counts(efvm_ctx* c, int64_t* n_solid, int64_t* n_ghost) {
    if (!c || !n_solid || !n_ghost) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (c->ibm && c->geom_dirty) {
        int rc = prologue(c);
        if (rc) return rc;
    }
    *n_solid = c->ibm ? c->n_solid : 0;
    *n_ghost = c->ibm ? (is_3d(c) ? c->ibm_desc.n_ghost : c->n_mirror) : 0;
    return EFVM_OK;
}

int efvm_get_solid_mask(efvm_ctx* c, uint8_t* out) {
    if (is_3d(c)) return refuse_3d(c, "efvm_get_solid_mask");
    if (!c || !out) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (c->ibm && c->geom_dirty) {
        int rc = prologue(c);
        if (rc) return rc;
    }
    const Geometry& g = c->g;
    CUDA_TRY(c, cudaMemcpy2DAsync(out, g.nx, c->mask + (size_t)YO * g.pitch + XO, g.pitch, g.nx, g.ny,
                                  cudaMemcpyDeviceToHost, S(c)));
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    return EFVM_OK;
}

int efvm_density_error(efvm_ctx* c, const efvm_vortex* v, double out[2]) {
    if (is_3d(c)) return refuse_3d(c, "efvm_density_error");
    if (!c || !v || !out) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    c->launches += launch_density_error(c->g, *v, cur_buf(c), c->st, c->partial, c->n_partial, S(c));
    std::vector<double> part(2 * (size_t)c->n_partial);
    CUDA_TRY(c, cudaMemcpyAsync(part.data(), c->partial, part.size() * sizeof(double), cudaMemcpyDeviceToHost, S(c)));
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    double sum = 0.0, mx = 0.0;
    for (int b = 0; b < c->n_partial; ++b) {
        sum += part[2 * b];
        mx = std::max(mx, part[2 * b + 1]);
    }
    // volume-weighted mean over uniform cells
    out[0] = sum / ((double)c->g.nx * (double)c->g.ny);
    out[1] = mx;
    return EFVM_OK;
}

int efvm_init_vortex(efvm_ctx* c, const efvm_vortex* v) {
    if (is_3d(c)) return refuse_3d(c, "efvm_init_vortex");
    if (!c || !v) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    {
        const int rcf = finish_forces(c);
        if (rcf) return rcf;
    }
    c->launches += launch_init_vortex(c->g, *v, cur_buf(c), S(c));
    c->lam_stale = true;
    c->ghosts_stale = true;
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    return EFVM_OK;
}

int efvm_total_mass(efvm_ctx* c, double* out) {
    if (!c || !out) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    c->launches += launch_total_mass(c->g, cur_buf(c), c->partial, c->n_partial, S(c));
    std::vector<double> part((size_t)c->n_partial);
    CUDA_TRY(c, cudaMemcpyAsync(part.data(), c->partial, part.size() * sizeof(double), cudaMemcpyDeviceToHost, S(c)));
    CUDA_TRY(c, cudaStreamSynchronize(S(c)));
    double sum = 0.0;
    for (double x : part) sum += x;
    *out = sum;
    return EFVM_OK;
}

int efvm_get_stream(efvm_ctx* c, void** stream) {
    if (!c || !stream) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    *stream = (void*)c->stream;
    return EFVM_OK;
}

int efvm_profile_steps(efvm_ctx* c, int64_t n_steps, double out_ms[4]) {
    if (!c || !out_ms || n_steps < 0) return fail(c, EFVM_ERR_INVALID_ARG, "invalid argument");
    if (c->params.integrator == EFVM_INTEGRATOR_EULER || c->rk_stage != 0)
        return fail(c, EFVM_ERR_INVALID_ARG, "efvm_profile_steps needs an RK3 context at a step boundary");
    {
        const int rcf = finish_forces(c);
        if (rcf) return rcf;
    }
    if (c->control_dirty) sync_control(c, 0, 0.0, 0);
    int rc = prologue(c);
    if (rc) return rc;
    cudaEvent_t ev[8];
    for (auto& e : ev) CUDA_TRY(c, cudaEventCreate(&e));
    double acc[4] = {0, 0, 0, 0};
    Ibm ib = c->ibm_desc;
    ib.history = nullptr;
    double* bufs[4] = {c->U[0], c->U[1], c->U[2], c->U[0]};
    for (int64_t k = 0; k < n_steps; ++k) {
        CUDA_TRY(c, cudaEventRecord(ev[0], S(c)));
        c->launches += launch_step_setup(c->ph, c->st, false, S(c));
        CUDA_TRY(c, cudaEventRecord(ev[1], S(c)));
        float ms_stage = 0.f, ms_ibm = 0.f;
        for (int s = 0; s < 3; ++s) {
            if (c->ibm)
                c->launches += is_3d(c) ? launch_mirror3(c->g, c->ph, ib, bufs[s], false, S(c))
                                        : launch_ibm(c->g, c->ph, ib, bufs[s], c->st, -1, s, 0, false, S(c));
            CUDA_TRY(c, cudaEventRecord(ev[2], S(c)));
            enqueue_stage_kernel(c, s, bufs[s], bufs[s + 1], false);
            CUDA_TRY(c, cudaEventRecord(ev[3], S(c)));
            if (c->ibm)
                c->launches += is_3d(c) ? launch_forces3(c->g, c->ph, ib, bufs[s + 1], c->st, false, S(c))
                                        : launch_ibm(c->g, c->ph, ib, bufs[s + 1], c->st, s, -1, 0, false, S(c));
            CUDA_TRY(c, cudaEventRecord(ev[4], S(c)));
            CUDA_TRY(c, cudaEventSynchronize(ev[4]));
            float t_stage = 0.f, t_after = 0.f;
            cudaEventElapsedTime(&t_stage, ev[2], ev[3]);
            cudaEventElapsedTime(&t_after, ev[3], ev[4]);
            float t_before = 0.f;
            cudaEventElapsedTime(&t_before, s == 0 ? ev[1] : ev[5], ev[2]);
            ms_stage += t_stage;
            ms_ibm += t_after + t_before;
            CUDA_TRY(c, cudaEventRecord(ev[5], S(c)));
        }
        CUDA_TRY(c, cudaEventSynchronize(ev[5]));
        float t_setup = 0.f, t_step = 0.f;
        cudaEventElapsedTime(&t_setup, ev[0], ev[1]);
        cudaEventElapsedTime(&t_step, ev[0], ev[5]);
        acc[0] += ms_stage;
        acc[1] += ms_ibm;
        acc[2] += t_setup;
        acc[3] += t_step;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    for (int k = 0; k < 4; ++k) out_ms[k] = acc[k];
    CUDA_TRY(c, cudaGetLastError());
    return EFVM_OK;
}

int efvm_set_stage_tiling(efvm_ctx* c, int32_t form, int32_t rows_per_warp, int32_t blocks_per_sm) {
    if (!c) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    const bool fp32 = c->ph.precision == EFVM_PREC_FP32_FLUX, visc = c->ph.viscous != 0;
    // a count the selected form is built for (the strip form: its built-in and
    // alternate counts; the TMA-fed form: its own; AUTO: any of them)
    const bool strip_count = blocks_per_sm == stage_blocks_per_sm(fp32, visc, false) ||
                             blocks_per_sm == stage_alt_blocks(fp32, visc);
    const bool tma_count = blocks_per_sm == stage_blocks_per_sm(fp32, visc, true);
    const bool count_ok = blocks_per_sm == 0 || (form == EFVM_STAGE_STRIP && strip_count) ||
                          (form == EFVM_STAGE_TMA && tma_count) ||
                          (form == EFVM_STAGE_AUTO && (strip_count || tma_count));
    if (!count_ok)
        return fail(c, EFVM_ERR_INVALID_ARG, "blocks_per_sm must be 0 or a count the selected stage form is built for");
    if (form < EFVM_STAGE_AUTO || form > EFVM_STAGE_TMA)
        return fail(c, EFVM_ERR_INVALID_ARG, "form must be EFVM_STAGE_AUTO, EFVM_STAGE_STRIP or EFVM_STAGE_TMA");
    if (rows_per_warp < 0 || rows_per_warp > 65536)
        return fail(c, EFVM_ERR_INVALID_ARG, "rows_per_warp must be in [0, 65536]");
    if (form == EFVM_STAGE_TMA && !c->tmaps)
        return fail(c, EFVM_ERR_UNSUPPORTED, "the TMA-fed stage kernel needs a 2-D context with tensor maps");
    c->stage_form = form;
    c->stage_rows = rows_per_warp;
    c->stage_blocks = blocks_per_sm;
    c->graph_valid = false;
    return EFVM_OK;
}

// The blocks per SM a stage of this context runs with: the strip form's
// alternate count when it was selected, else the form's built-in count.
static int resolved_blocks(const efvm_ctx* c, int form) {
    const bool fp32 = c->ph.precision == EFVM_PREC_FP32_FLUX, visc = c->ph.viscous != 0;
    const int alt = stage_alt_blocks(fp32, visc);
    if (form == EFVM_STAGE_STRIP && alt > 0 && c->stage_blocks == alt) return alt;
    return stage_blocks_per_sm(fp32, visc, form == EFVM_STAGE_TMA);
}

int efvm_get_stage_tiling(efvm_ctx* c, int32_t* form, int32_t* rows_per_warp, int32_t* blocks_per_sm) {
    if (!c || !form || !rows_per_warp || !blocks_per_sm) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    *form = resolved_form(c);
    *blocks_per_sm = resolved_blocks(c, *form);
    *rows_per_warp = c->stage_rows > 0 ? c->stage_rows
                                       : stage_rows(c->g.nx, c->g.ny, c->ph.precision == EFVM_PREC_FP32_FLUX,
                                                    c->ph.viscous != 0, *form == EFVM_STAGE_TMA);
    if (c->stage_rows <= 0 && *blocks_per_sm != stage_blocks_per_sm(c->ph.precision == EFVM_PREC_FP32_FLUX,
                                                                     c->ph.viscous != 0, *form == EFVM_STAGE_TMA)) {
        // the built-in rows follow the resident slots of the count in use
        const long long strips = stage_strips(c->g.nx), slots = 148LL * *blocks_per_sm * 4;
        *rows_per_warp = (int)std::min<long long>(16, std::max<long long>(2, (strips * c->g.ny + slots - 1) / slots));
    }
    return EFVM_OK;
}

// Times whole steps of every candidate tiling on the live state and keeps the
// fastest: the strip kernel at its built-in and its alternate resident-block
// count and (where the case allows it) the TMA-fed kernel, each with 4, 8, 16
// and 32 rows per warp and with the rows that fit the whole grid into one wave
// of resident blocks.  The state, the clock and the force
// outputs are saved first and restored after every candidate, so tuning
// changes no result.
int efvm_autotune_stage(efvm_ctx* c, int32_t n_steps, double* best_ms_per_step) {
    if (!c) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (is_3d(c) || has_halo(c) || c->nn || c->params.integrator == EFVM_INTEGRATOR_EULER)
        return fail(c, EFVM_ERR_UNSUPPORTED, "stage tuning covers 2-D RK3 contexts without slabs or a flux correction");
    if (c->rk_stage != 0) return fail(c, EFVM_ERR_INVALID_ARG, "efvm_autotune_stage needs a step boundary");
    if (n_steps <= 0) n_steps = 3;
    int rc = finish_forces(c);
    if (rc) return rc;
    if (c->control_dirty) sync_control(c, 0, 0.0, 0);
    rc = prologue(c);
    if (rc) return rc;
    DevState s0;
    rc = read_state(c, s0);
    if (rc) return rc;
    const size_t state_bytes = (size_t)4 * c->g.plane * sizeof(double);
    double* backup = nullptr;
    CUDA_TRY(c, cudaMalloc(&backup, state_bytes));
    double f0[12] = {0};
    if (c->ibm) CUDA_TRY(c, cudaMemcpy(f0, c->force_out, sizeof(f0), cudaMemcpyDeviceToHost));
    CUDA_TRY(c, cudaMemcpyAsync(backup, c->U[0], state_bytes, cudaMemcpyDeviceToDevice, S(c)));
    auto restore = [&]() -> int {
        CUDA_TRY(c, cudaMemcpyAsync(c->U[0], backup, state_bytes, cudaMemcpyDeviceToDevice, S(c)));
        CUDA_TRY(c, cudaMemcpyAsync(c->st, &s0, sizeof(DevState), cudaMemcpyHostToDevice, S(c)));
        if (c->ibm) CUDA_TRY(c, cudaMemcpyAsync(c->force_out, f0, sizeof(f0), cudaMemcpyHostToDevice, S(c)));
        CUDA_TRY(c, cudaStreamSynchronize(S(c)));
        return EFVM_OK;
    };
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const bool fp32 = c->ph.precision == EFVM_PREC_FP32_FLUX;
    std::vector<int> forms{EFVM_STAGE_STRIP};
    if (c->tmaps && stage_tma_eligible(c->g, c->ph, c->ibm, false)) forms.push_back(EFVM_STAGE_TMA);
    cudaEvent_t e0, e1;
    CUDA_TRY(c, cudaEventCreate(&e0));
    CUDA_TRY(c, cudaEventCreate(&e1));
    const int saved_form = c->stage_form, saved_rows = c->stage_rows, saved_blocks = c->stage_blocks;
    float best = 1e30f;
    int best_form = saved_form, best_rows = saved_rows, best_blocks = saved_blocks;
    // (form, resident blocks per SM) pairs: the strip form at its built-in count
    // and at its alternate one, the TMA form at its own
    std::vector<std::pair<int, int>> shapes{{EFVM_STAGE_STRIP, 0}};
    const int alt = stage_alt_blocks(fp32, c->ph.viscous != 0);
    if (alt > 0) shapes.push_back({EFVM_STAGE_STRIP, alt});
    for (int form : forms)
        if (form == EFVM_STAGE_TMA) shapes.push_back({EFVM_STAGE_TMA, 0});
    for (const auto& shape : shapes) {
        const int form = shape.first, blocks = shape.second;
        // one wave: the rows that spread the grid's strips over every resident block once
        const int minb = blocks > 0 ? blocks : stage_blocks_per_sm(fp32, c->ph.viscous != 0, form == EFVM_STAGE_TMA);
        const int bx = (stage_strips(c->g.nx) + 3) / 4;
        const int by = std::max(1, sms * minb / std::max(bx, 1));
        std::vector<int> rows{4, 8, 16, 32, (c->g.ny + by - 1) / by};
        std::sort(rows.begin(), rows.end());
        rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
        for (int r : rows) {
            if (r > c->g.ny && r != rows.front()) continue;
            c->stage_form = form;
            c->stage_rows = r;
            c->stage_blocks = blocks;
            rc = capture_step_graph(c);
            if (rc) break;
            CUDA_TRY(c, cudaGraphLaunch(c->graph_exec, S(c)));  // warm-up
            CUDA_TRY(c, cudaEventRecord(e0, S(c)));
            for (int k = 0; k < n_steps; ++k) CUDA_TRY(c, cudaGraphLaunch(c->graph_exec, S(c)));
            CUDA_TRY(c, cudaEventRecord(e1, S(c)));
            CUDA_TRY(c, cudaEventSynchronize(e1));
            c->launches += (uint64_t)(n_steps + 1) * c->graph_kernels;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            DevState s;
            rc = read_state(c, s);
            if (!rc && (s.nonphysical & 8))
                rc = fail(c, EFVM_ERR_TIMEOUT, "a stage kernel's wait for a row of its shared-memory ring ran out");
            if (!rc) rc = restore();
            if (rc) break;
            if (ms < best) {
                best = ms;
                best_form = form;
                best_rows = r;
                best_blocks = blocks;
            }
        }
        if (rc) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int rc2 = restore();
    cudaFree(backup);
    c->stage_form = rc ? saved_form : best_form;
    c->stage_rows = rc ? saved_rows : best_rows;
    c->stage_blocks = rc ? saved_blocks : best_blocks;
    c->graph_valid = false;
    if (rc) return rc;
    if (rc2) return rc2;
    if (best_ms_per_step) *best_ms_per_step = best / n_steps;
    return EFVM_OK;
}

int efvm_set_stage_wait_limit(efvm_ctx* c, double seconds) {
    if (!c) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    if (!(seconds > 0.0) || seconds > 600.0) return fail(c, EFVM_ERR_INVALID_ARG, "the limit must be in (0, 600] s");
    c->stage_wait_ns = (unsigned long long)(seconds * 1e9);
    c->graph_valid = false;
    return EFVM_OK;
}

int efvm_inject_stage_stall(efvm_ctx* c, int32_t enable) {
    if (!c) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    c->stage_stall = enable != 0;
    c->graph_valid = false;
    return EFVM_OK;
}

int efvm_launch_count(efvm_ctx* c, uint64_t* out) {
    if (!c || !out) return fail(c, EFVM_ERR_INVALID_ARG, "null argument");
    *out = c->launches;
    return EFVM_OK;
}

}  // extern "C"
