// efvm_kernels3d.cuh — the 3-D (nz > 1) forms of the stage, ghost-fill, CFL,
// transfer and mass kernels.  Included by efvm_kernels.cu inside namespace
// efvm after its 2-D helpers (the rounding wrappers, the gas model, the launch
// helper), which these kernels share.
//
// HBM layout of one 3-D state: 5 FP64 planes (rho, rho_u, rho_v, rho_w,
// rho_e), each (nz + 2 ZO) layers of (ny + 2 YO) rows x `pitch` doubles; cell
// (i, j, k) sits at layer ZO + k, row YO + j, column XO + i.  Layers ZO-2,
// ZO-1 and ZO+nz, ZO+nz+1 are the two z ghost layers of FIELD's ng = 2.
//
// The stage kernel keeps the 2-D kernel's organisation: a warp owns a strip of
// 31 columns of one layer k and marches `rows` rows with the carried y window,
// and the x faces come from warp shuffles.  The warps of a block stack in z
// over the same strip and rows and share the z direction through shared
// memory: each limits the z slope of its own cell once and forms the z face
// above its layer once.  A z face on the edge of two blocks is formed by both
// through the same (non-unrolled) loop bodies, so the two results agree bit
// for bit and the scheme stays conservative across layers.

namespace {

constexpr int ZO = 2;  // layer of interior cell k = 0

__device__ __forceinline__ long long cidx3(const Geometry& g, int i, int j, int k) {
    return (long long)(ZO + k) * g.layer + (long long)(YO + j) * g.pitch + (XO + i);
}

struct U5 {
    double r, mx, my, mz, E;
};
__device__ __forceinline__ U5 load5(const double* q, long long P, long long o) {
    return U5{q[o], q[P + o], q[2 * P + o], q[3 * P + o], q[4 * P + o]};
}
__device__ __forceinline__ void store5(double* q, long long P, long long o, const U5& u) {
    q[o] = u.r;
    q[P + o] = u.mx;
    q[2 * P + o] = u.my;
    q[3 * P + o] = u.mz;
    q[4 * P + o] = u.E;
}

// IdealGas::pressure (crates/cfd_eos/src/lib.rs:61-64) and prim_to_cons (:55-59),
// every operation rounded explicitly (evaluated by the stage epilogue and the
// stand-alone ghost fill / CFL pass alike).
__device__ __forceinline__ double pressure5(const U5& u, double gm1) {
    const double mm = add_(add_(mul_(u.mx, u.mx), mul_(u.my, u.my)), mul_(u.mz, u.mz));
    return mul_(gm1, sub_(u.E, mul_(0.5, mm) / u.r));
}
__device__ __forceinline__ U5 prim_to_cons5(double rho, double u, double v, double w, double p, double gm1) {
    const double ke = mul_(mul_(0.5, rho), add_(add_(mul_(u, u), mul_(v, v)), mul_(w, w)));
    return U5{rho, mul_(rho, u), mul_(rho, v), mul_(rho, w), add_(p / gm1, ke)};
}

// BoundaryCondition::ghost_at, crates/cfd_boundary/src/lib.rs:172-362, for
// side 0..5 (XLO, XHI, YLO, YHI, ZLO, ZHI).
__device__ __forceinline__ U5 bc_ghost5(const DevBC& bc, int side, const U5& in, double gm1) {
    switch (bc.kind) {
        case EFVM_BC_SLIP_WALL:
        case EFVM_BC_SYMMETRY: {
            double n[3] = {0.0, 0.0, 0.0};
            n[side / 2] = (side % 2 == 1) ? 1.0 : -1.0;
            const double mn = add_(add_(mul_(in.mx, n[0]), mul_(in.my, n[1])), mul_(in.mz, n[2]));
            U5 g = in;
            g.mx = sub_(in.mx, mul_(mul_(2.0, mn), n[0]));
            g.my = sub_(in.my, mul_(mul_(2.0, mn), n[1]));
            g.mz = sub_(in.mz, mul_(mul_(2.0, mn), n[2]));
            return g;
        }
        case EFVM_BC_NO_SLIP_WALL:
            return U5{in.r, -in.mx, -in.my, -in.mz, in.E};
        case EFVM_BC_SUPERSONIC_INFLOW:
            return prim_to_cons5(bc.rho, bc.u, bc.v, bc.w, bc.p, gm1);
        case EFVM_BC_SUBSONIC_INFLOW:
            return prim_to_cons5(bc.rho, bc.u, bc.v, bc.w, pressure5(in, gm1), gm1);
        case EFVM_BC_PRESSURE_OUTLET: {
            const double inv = 1.0 / in.r;
            return prim_to_cons5(in.r, mul_(in.mx, inv), mul_(in.my, inv), mul_(in.mz, inv), bc.p, gm1);
        }
        default:
            return in;
    }
}

// The Halo (periodic wrap of both ghost layers) and Boundary (first ghost
// layer) phases for the ghosts whose source is interior cell (i, j, k) with
// value u, written by the thread that owns that cell.  PXYZ: all three axes
// are known to be periodic at compile time (the boundary-condition paths are
// not compiled).
template <bool PXYZ = false>
__device__ __forceinline__ void write_ghosts3(const Geometry& g, const Physics& ph, double* q, int i, int j, int k,
                                              const U5& u) {
    const long long P = g.plane;
    const double gm1 = ph.gamma - 1.0;
    if (PXYZ || ph.periodic_x) {
        if (i >= g.nx - NG) store5(q, P, cidx3(g, i - g.nx, j, k), u);
        if (i < NG) store5(q, P, cidx3(g, i + g.nx, j, k), u);
    } else {
        if (i == 0) store5(q, P, cidx3(g, -1, j, k), bc_ghost5(ph.bc[0], 0, u, gm1));
        if (i == g.nx - 1) store5(q, P, cidx3(g, g.nx, j, k), bc_ghost5(ph.bc[1], 1, u, gm1));
    }
    if (PXYZ || ph.periodic_y) {
        if (j >= g.ny - NG) store5(q, P, cidx3(g, i, j - g.ny, k), u);
        if (j < NG) store5(q, P, cidx3(g, i, j + g.ny, k), u);
    } else {
        if (j == 0) store5(q, P, cidx3(g, i, -1, k), bc_ghost5(ph.bc[2], 2, u, gm1));
        if (j == g.ny - 1) store5(q, P, cidx3(g, i, g.ny, k), bc_ghost5(ph.bc[3], 3, u, gm1));
    }
    if (PXYZ || ph.periodic_z) {
        if (k >= g.nz - NG) store5(q, P, cidx3(g, i, j, k - g.nz), u);
        if (k < NG) store5(q, P, cidx3(g, i, j, k + g.nz), u);
    } else {
        if (k == 0) store5(q, P, cidx3(g, i, j, -1), bc_ghost5(ph.bc[4], 4, u, gm1));
        if (k == g.nz - 1) store5(q, P, cidx3(g, i, j, g.nz), bc_ghost5(ph.bc[5], 5, u, gm1));
    }
}

// Local max wave speed of cfl_system, crates/cfd_solver/src/lib.rs:647-669.
// As the 2-D wave_speed: the reference's divisions taken as products with
// reciprocals (a few ulps from its value), one code for the stage epilogue and
// the stand-alone CFL pass.
__device__ __forceinline__ double wave_speed3(const Geometry& g, const Physics& ph, const U5& u) {
    if (!(u.r > 0.0)) return 0.0;
    const double gm1 = ph.gamma - 1.0;
    const double inv = 1.0 / u.r;
    const double vx = mul_(u.mx, inv), vy = mul_(u.my, inv), vz = mul_(u.mz, inv);
    const double ke = mul_(mul_(0.5, u.r), add_(add_(mul_(vx, vx), mul_(vy, vy)), mul_(vz, vz)));
    const double p = mul_(gm1, sub_(u.E, ke));
    const double a = sqrt(mul_(mul_(ph.gamma, p), inv));
    double lam = add_(add_(mul_(add_(fabs(vx), a), g.inv_h[0]), mul_(add_(fabs(vy), a), g.inv_h[1])),
                      mul_(add_(fabs(vz), a), g.inv_h[2]));
    if (ph.viscous) {
        const double t = mul_(mul_(p, inv), ph.inv_r_gas);
        const double nu = mul_(viscosity(ph, t), inv);
        lam = add_(lam, mul_(mul_(2.0, nu), ph.cfl_visc_sum));
    }
    return lam;
}

// A conserved state in the grid frame and its face-frame views.
struct V5 {
    double r, mx, my, mz, E;
};
__device__ __forceinline__ V5 toV5(const U5& u) { return V5{u.r, u.mx, u.my, u.mz, u.E}; }
__device__ __forceinline__ U5 toU5(const V5& u) { return U5{u.r, u.mx, u.my, u.mz, u.E}; }
__device__ __forceinline__ Q5<double> xq5(const V5& u) { return Q5<double>{u.r, u.mx, u.my, u.mz, u.E}; }
__device__ __forceinline__ Q5<double> yq5(const V5& u) { return Q5<double>{u.r, u.my, u.mx, u.mz, u.E}; }
__device__ __forceinline__ Q5<double> zq5(const V5& u) { return Q5<double>{u.r, u.mz, u.mx, u.my, u.E}; }
// A face flux back in the grid frame (x, y, z faces).
__device__ __forceinline__ V5 xg5(const Q5<double>& f) { return V5{f.r, f.mn, f.mt, f.ms, f.E}; }
__device__ __forceinline__ V5 yg5(const Q5<double>& f) { return V5{f.r, f.mt, f.mn, f.ms, f.E}; }
__device__ __forceinline__ V5 zg5(const Q5<double>& f) { return V5{f.r, f.mt, f.ms, f.mn, f.E}; }

// The +face and -face states c +- s/2 of a cell, s = lim(p - c, c - m)
// (limited_slope_cons and reconstruct_to_face, crates/cfd_solver/src/lib.rs:199-211,273-286).
__device__ __forceinline__ void slope_faces5(int limiter, const V5& m, const V5& c, const V5& p, V5& plus, V5& minus) {
    const double hr = half_slope(limiter, m.r, c.r, p.r), hx = half_slope(limiter, m.mx, c.mx, p.mx);
    const double hy = half_slope(limiter, m.my, c.my, p.my), hz = half_slope(limiter, m.mz, c.mz, p.mz);
    const double he = half_slope(limiter, m.E, c.E, p.E);
    plus = V5{c.r + hr, c.mx + hx, c.my + hy, c.mz + hz, c.E + he};
    minus = V5{c.r - hr, c.mx - hx, c.my - hy, c.mz - hz, c.E - he};
}

__device__ __forceinline__ V5 shfl_up5(const V5& u, int d) {
    return V5{__shfl_up_sync(0xffffffffu, u.r, d), __shfl_up_sync(0xffffffffu, u.mx, d),
              __shfl_up_sync(0xffffffffu, u.my, d), __shfl_up_sync(0xffffffffu, u.mz, d),
              __shfl_up_sync(0xffffffffu, u.E, d)};
}
__device__ __forceinline__ V5 shfl_down5(const V5& u, int d) {
    return V5{__shfl_down_sync(0xffffffffu, u.r, d), __shfl_down_sync(0xffffffffu, u.mx, d),
              __shfl_down_sync(0xffffffffu, u.my, d), __shfl_down_sync(0xffffffffu, u.mz, d),
              __shfl_down_sync(0xffffffffu, u.E, d)};
}

// Primitive (u, v, w, T) of a state given 1/rho (cons_to_prim, crates/cfd_eos/src/lib.rs:44-53).
__device__ __forceinline__ void prim5(const U5& u, double inv, double gm1, double inv_r_gas, double& vu, double& vv,
                                      double& vw, double& t) {
    vu = u.mx * inv;
    vv = u.my * inv;
    vw = u.mz * inv;
    const double ke = 0.5 * u.r * (vu * vu + vv * vv + vw * vw);
    t = gm1 * (u.E - ke) * inv * inv_r_gas;
}

constexpr int WPB3 = 4;   // warps per block of the 3-D stage kernel, stacked in z
constexpr int MINB3 = 4;  // resident blocks per SM of the 3-D stage kernel (128 registers)

}  // namespace

// ---------------------------------------------------------------------------
// The 3-D stage kernel: one RK substage.  Block (b, by) covers strip b mod
// strips and the WPB3 consecutive layers starting at WPB3 (b div strips); warp
// w takes layer WPB3 (b div strips) + w, so the block's warps stack in z over
// the same columns and rows.  Per row, each warp limits the z slope of its own
// cell (warp 0 also that of the cell below, the top warp that of the cell
// above), hands the right state of the face below its cell to the warp under
// it, forms the z face above its layer and hands that flux to the warp above;
// only warp 0 also forms the face below its layer.  Slopes and faces each go
// through one non-unrolled loop body, so a face formed at the top of one block
// and again at the bottom of the next is bit-identical.  Every warp adds the
// face below and then the face above, in the same order, so the step commutes
// with shifts in z.  A warp past the last layer computes on the last layer
// (its loads stay in bounds) and stores nothing; it only keeps the block's
// barriers.
// ---------------------------------------------------------------------------
// LIM >= 0 fixes the limiter and PXYZ a fully periodic mesh at compile time
// (the inviscid forms are built so); -1 and false read them at run time.
template <int SCHEME, int RECON, bool VISC, int LIM, bool PXYZ>
__global__ void __launch_bounds__(32 * WPB3, MINB3) stage3_kernel(StageArgs a, int rows) {
    pdl_wait_then_release();
    if (!a.st->active) return;
    const Geometry& g = a.g;
    const Physics& ph = a.ph;
    const int limiter = LIM >= 0 ? LIM : ph.limiter;
    const long long P = g.plane;
    const int lane = threadIdx.x & 31;
    const int strips = (g.nx + STRIP - 1) / STRIP;
    const int warp = threadIdx.x >> 5;
    const int kgroup = blockIdx.x / strips, strip = blockIdx.x - kgroup * strips;
    const int k_raw = kgroup * WPB3 + warp;
    const bool act = k_raw < g.nz;       // warp-uniform
    const int k = act ? k_raw : g.nz - 1;
    const int by = blockIdx.y;
    __shared__ double zup[WPB3][5][32];     // the flux of the face above each warp's layer, per lane
    // z face states of the block's column, face f lying below layer WPB3 (b div strips) + f
    __shared__ double zst[2][WPB3 + 1][5][32];  // [left/right state][face][variable][lane]
    if (strip == 0 && by == 0 && k_raw == 0 && lane == 0) {
        // RK state machine and clock of update_system, crates/cfd_solver/src/lib.rs:607-621
        DevState* st = a.st;
        if (a.stage >= 2) {
            st->rk_stage = 0;
            st->completed = 1;
            st->step += 1;
            st->time += st->dt;
        } else {
            st->rk_stage = a.stage + 1;
            st->completed = 0;
        }
    }
    const int i0 = strip * STRIP;
    const int jb = by * rows;
    double lam = 0.0;
    if (jb < g.ny) {  // uniform across the block (its barriers sit inside)
        constexpr bool MUSCL = RECON == EFVM_RECON_MUSCL;
        const int je = min(jb + rows, g.ny);
        const int i = i0 + lane;
        const int ic = min(i, g.nx + NG - 1);
        const bool owner = lane < STRIP && i < g.nx;
        const bool true_seam = ph.periodic_seam == EFVM_SEAM_TRUE_PERIODIC;
        const double gm1 = ph.gamma - 1.0;
        const double rg = ph.gamma;
        const double* __restrict__ uin = a.uin;
        auto ld = [&](int ii, int jj, int kk) { return load5(uin, P, cidx3(g, ii, jj, kk)); };
        const double* __restrict__ colp = uin + cidx3(g, ic, 0, k);
        auto ldrow = [&](int jj) { return toV5(load5(colp, P, (long long)jj * g.pitch)); };
        auto ldz = [&](int jj, int dk) { return toV5(load5(colp, P, (long long)jj * g.pitch + (long long)dk * g.layer)); };

        // reconstruction flags of the faces on the domain edges (as the 2-D kernel)
        bool rec_l = MUSCL, rec_r = MUSCL;
        if (i == 0) {
            rec_l = MUSCL && ph.periodic_x && true_seam;
            rec_r = MUSCL && ph.periodic_x;
        } else if (i == g.nx) {
            rec_l = MUSCL && ph.periodic_x;
            rec_r = MUSCL && ph.periodic_x && true_seam;
        }
        const bool seam_rec_y = MUSCL && ph.periodic_y && true_seam;
        const bool edge_rec_y = MUSCL && ph.periodic_y;
        // z faces: below (k - 1/2) and above (k + 1/2); side A is the lower cell
        bool zrA[2] = {MUSCL, MUSCL}, zrB[2] = {MUSCL, MUSCL};
        if (k == 0) {
            zrA[0] = MUSCL && ph.periodic_z && true_seam;
            zrB[0] = MUSCL && ph.periodic_z;
        }
        if (k == g.nz - 1) {
            zrA[1] = MUSCL && ph.periodic_z;
            zrB[1] = MUSCL && ph.periodic_z && true_seam;
        }
        const double dt = a.st->dt;

        V5 uc = ldrow(jb - 1), un = ldrow(jb), pc = uc;
        if (MUSCL) {
            V5 unused;
            slope_faces5(limiter, ldrow(jb - 2), uc, un, pc, unused);
        }
        V5 gb;  // flux of the y face below row j, grid frame
        for (int j = jb - 1; j < je; ++j) {
            const bool row = j >= jb;  // warp-uniform: the first pass only forms the face below row jb

            // Flux divergence, accumulated as each face is formed: the y face below
            // (carried), the x faces left and right, the z faces below and above,
            // then the y face above.  The reference sums an interior cell's faces in
            // for_each_face order (z below, y below, x left, +x, +y, +z;
            // crates/cfd_solver/src/lib.rs:333-337); the order here keeps at most
            // one face flux live at a time and differs from it only in rounding.
            double acc[5];
            if (row) {
                // ---- x faces on the left and right of column i ----
                V5 ul = shfl_up5(uc, 1), ur = shfl_down5(uc, 1);
                V5 ull = ul;
                if (lane == 0) {
                    ul = toV5(ld(i0 - 1, j, k));
                    if (MUSCL) ull = toV5(ld(i0 - 2, j, k));
                }
                if (MUSCL && lane == 31) ur = toV5(ld(min(i0 + 32, g.nx + NG - 1), j, k));
                Q5<double> xl = xq5(ul), xr = xq5(uc);
                if (MUSCL) {
                    V5 pp, mm;
                    slope_faces5(limiter, ul, uc, ur, pp, mm);
                    V5 lp = shfl_up5(pp, 1);
                    if (lane == 0) {
                        V5 unused;
                        slope_faces5(limiter, ull, ul, uc, lp, unused);
                    }
                    xl = xq5(rec_l ? lp : ul);
                    xr = xq5(rec_r ? mm : uc);
                }
                const V5 fx = xg5(face_flux5<SCHEME, double>(xl, xr, rg, gm1));
                const V5 fxr = shfl_down5(fx, 1);
                const double yb[5] = {gb.r, gb.mx, gb.my, gb.mz, gb.E};
                const double fl[5] = {fx.r, fx.mx, fx.my, fx.mz, fx.E};
                const double fr[5] = {fxr.r, fxr.mx, fxr.my, fxr.mz, fxr.E};
#pragma unroll
                for (int v = 0; v < 5; ++v) {
                    double t = __dmul_rn(yb[v], g.inv_y);
                    t = __dadd_rn(t, __dmul_rn(fl[v], g.inv_x));
                    acc[v] = __dsub_rn(t, __dmul_rn(fr[v], g.inv_x));
                }

                // ---- z faces.  One non-unrolled loop marches the column up through
                // the cells whose z slope this warp limits: its own, and for warp 0
                // the one below, for the top warp (the last of the block, or of the
                // mesh) the one above; so every slope comes from one code path.  Each
                // slope gives the right state of the face below its cell and the left
                // state of the face above; they meet in shared memory, every face
                // state with one writer.  A second non-unrolled loop forms the face
                // above the warp's layer (warp 0 also the one below), whose flux goes
                // to the warp above.  A face on the edge of two blocks is formed from
                // the same states through the same code by both. ----
                const bool top = warp == WPB3 - 1 || k_raw + 1 >= g.nz;
                const int lo = warp == 0 ? -1 : 0, hi = top ? 1 : 0;
                auto put = [&](int side, int f, const V5& q) {
                    zst[side][f][0][lane] = q.r;
                    zst[side][f][1][lane] = q.mx;
                    zst[side][f][2][lane] = q.my;
                    zst[side][f][3][lane] = q.mz;
                    zst[side][f][4][lane] = q.E;
                };
                auto get = [&](int side, int f) {
                    return V5{zst[side][f][0][lane], zst[side][f][1][lane], zst[side][f][2][lane],
                              zst[side][f][3][lane], zst[side][f][4][lane]};
                };
                {
                    V5 m = ldz(j, lo - 1), c = ldz(j, lo);
#pragma unroll 1
                    for (int dk = lo; dk <= hi; ++dk) {
                        const V5 p = ldz(j, dk + 1);
                        V5 pl = c, mi = c;
                        if (MUSCL) {
                            V5 sp, sm;
                            slope_faces5(limiter, m, c, p, sp, sm);
                            if (dk < 0 ? zrA[0] : zrA[1]) pl = sp;
                            if (dk > 0 ? zrB[1] : zrB[0]) mi = sm;
                        }
                        // a warp past the last layer writes nothing: its faces belong to the top warp
                        if (act && dk < 1) put(0, warp + dk + 1, pl);  // left state of the face above cell k + dk
                        if (act && dk > -1) put(1, warp + dk, mi);     // right state of the face below it
                        m = c;
                        c = p;
                    }
                }
                __syncthreads();
                V5 fzb, fza;
#pragma unroll 1
                for (int s = warp == 0 ? 0 : 1; s < 2; ++s) {
                    const V5 L = get(0, warp + s), Rv = get(1, warp + s);
                    const V5 f = zg5(face_flux5<SCHEME, double>(zq5(L), zq5(Rv), rg, gm1));
                    if (s) fza = f;
                    else fzb = f;
                }
                zup[warp][0][lane] = fza.r;
                zup[warp][1][lane] = fza.mx;
                zup[warp][2][lane] = fza.my;
                zup[warp][3][lane] = fza.mz;
                zup[warp][4][lane] = fza.E;
                __syncthreads();  // zst is rewritten on the next row only after this barrier
                if (warp > 0)
                    fzb = V5{zup[warp - 1][0][lane], zup[warp - 1][1][lane], zup[warp - 1][2][lane],
                             zup[warp - 1][3][lane], zup[warp - 1][4][lane]};
                const double zb[5] = {fzb.r, fzb.mx, fzb.my, fzb.mz, fzb.E};
                const double za[5] = {fza.r, fza.mx, fza.my, fza.mz, fza.E};
#pragma unroll
                for (int v = 0; v < 5; ++v) {  // in through the face below, out through the one above
                    acc[v] = __dadd_rn(acc[v], __dmul_rn(zb[v], g.inv_z));
                    acc[v] = __dsub_rn(acc[v], __dmul_rn(za[v], g.inv_z));
                }
            }

            // ---- y face above row j ----
            const V5 un2 = ldrow(j + 2);
            V5 pn = un;
            Q5<double> yb_, yt_;
            if (MUSCL) {
                V5 mn;
                slope_faces5(limiter, uc, un, un2, pn, mn);
                const bool lo_edge = j == -1, hi_edge = j + 1 == g.ny;
                const bool rb = lo_edge ? seam_rec_y : (hi_edge ? edge_rec_y : true);
                const bool rt = lo_edge ? edge_rec_y : (hi_edge ? seam_rec_y : true);
                yb_ = yq5(rb ? pc : uc);
                yt_ = yq5(rt ? mn : un);
            } else {
                yb_ = yq5(uc);
                yt_ = yq5(un);
            }
            const V5 gt = yg5(face_flux5<SCHEME, double>(yb_, yt_, rg, gm1));

            if (row && owner && act) {
                const long long o = cidx3(g, i, j, k);
                const U5 ucd = toU5(uc);
                const double yt[5] = {gt.r, gt.mx, gt.my, gt.mz, gt.E};
                double rhs[5];
#pragma unroll
                for (int v = 0; v < 5; ++v) rhs[v] = __dsub_rn(acc[v], __dmul_rn(yt[v], g.inv_y));
                const bool ibm = a.mask != nullptr;
                const bool solid = ibm && a.mask[o];
                if (VISC && !solid) {
                    // viscous_system, crates/cfd_solver/src/lib.rs:514-557 (7-point stencil),
                    // one axis pair of neighbours at a time; a solid neighbour enters as
                    // (0, 0, 0, T of the cell).  The seven reciprocal densities come from
                    // one reciprocal of their product.
                    const long long nbo[6] = {cidx3(g, i + 1, j, k), cidx3(g, i - 1, j, k), cidx3(g, i, j + 1, k),
                                              cidx3(g, i, j - 1, k), cidx3(g, i, j, k + 1), cidx3(g, i, j, k - 1)};
                    bool sn[6];
                    double rn[6];
#pragma unroll
                    for (int n = 0; n < 6; ++n) {
                        sn[n] = ibm && a.mask[nbo[n]];
                        rn[n] = sn[n] ? 1.0 : uin[nbo[n]];
                    }
                    double pr[7];
                    pr[0] = ucd.r;
#pragma unroll
                    for (int n = 0; n < 6; ++n) pr[n + 1] = pr[n] * rn[n];
                    double w = rcp_(pr[6]);
                    double inv[7];
#pragma unroll
                    for (int n = 6; n >= 1; --n) {
                        inv[n] = pr[n - 1] * w;
                        w = w * rn[n - 1];  // now 1 / pr[n - 1]
                    }
                    inv[0] = w;
                    double us, vs, ws, ts;
                    prim5(ucd, inv[0], gm1, ph.inv_r_gas, us, vs, ws, ts);
                    const double mu = viscosity(ph, ts);
                    const double kappa = mu * ph.cp_pr;  // thermal_conductivity mu cp / Pr, crates/cfd_eos/src/lib.rs:83-87
                    double lu = 0.0, lv = 0.0, lw = 0.0, lt = 0.0;  // d2x + d2y + d2z of u, v, w, T
#pragma unroll
                    for (int ax = 0; ax < 3; ++ax) {
                        double pu = 0.0, pv = 0.0, pw = 0.0, pt = ts, mu_ = 0.0, mv = 0.0, mw = 0.0, mt = ts;
                        if (!sn[2 * ax])
                            prim5(load5(uin, P, nbo[2 * ax]), inv[2 * ax + 1], gm1, ph.inv_r_gas, pu, pv, pw, pt);
                        if (!sn[2 * ax + 1])
                            prim5(load5(uin, P, nbo[2 * ax + 1]), inv[2 * ax + 2], gm1, ph.inv_r_gas, mu_, mv, mw, mt);
                        double im = 0.0, ip = 0.0, is = 0.0;
                        if (ax == 1) {
                            im = a.yw[j];
                            ip = a.yw[g.ny + j];
                            is = a.yw[2 * g.ny + j];
                        } else if (ax == 2) {
                            im = a.zw[k];
                            ip = a.zw[g.nz + k];
                            is = a.zw[2 * g.nz + k];
                        }
                        auto d2 = [&](double m, double p, double c) {
                            return ax == 0 ? (p - 2.0 * c + m) * ph.dx_inv2 : ((p - c) * ip - (c - m) * im) * is;
                        };
                        const double du = d2(mu_, pu, us), dv = d2(mv, pv, vs), dw = d2(mw, pw, ws), dt_ = d2(mt, pt, ts);
                        lu = ax == 0 ? du : lu + du;
                        lv = ax == 0 ? dv : lv + dv;
                        lw = ax == 0 ? dw : lw + dw;
                        lt = ax == 0 ? dt_ : lt + dt_;
                    }
                    const double fxv = mu * lu, fyv = mu * lv, fzv = mu * lw;
                    rhs[1] += fxv;
                    rhs[2] += fyv;
                    rhs[3] += fzv;
                    rhs[4] += us * fxv + vs * fyv + ws * fzv + kappa * lt;
                }
                if (solid)  // zero_solid_rhs, crates/cfd_ibm/src/lib.rs:293-301
#pragma unroll
                    for (int v = 0; v < 5; ++v) rhs[v] = 0.0;
                if (ph.body_force_x != 0.0) {  // crates/cfd_solver/tests/poiseuille_channel_validation.rs:100-118
                    rhs[1] += ucd.r * ph.body_force_x;
                    rhs[4] += ph.body_force_x * ucd.mx;
                }
                // Rk3Integrator / EulerIntegrator::substep, crates/cfd_solver/src/integrate.rs:48-101
                const double ucv[5] = {ucd.r, ucd.mx, ucd.my, ucd.mz, ucd.E};
                double nwv[5];
                if (a.stage == 1 || a.stage == 2) {
                    const double w0 = a.stage == 1 ? 0.75 : (1.0 / 3.0);
                    const double w1 = a.stage == 1 ? 0.25 : (2.0 / 3.0);
#pragma unroll
                    for (int v = 0; v < 5; ++v)
                        nwv[v] = __dadd_rn(__dmul_rn(w0, a.u0[v * P + o]),
                                           __dmul_rn(w1, __dadd_rn(ucv[v], __dmul_rn(rhs[v], dt))));
                } else {
#pragma unroll
                    for (int v = 0; v < 5; ++v) nwv[v] = __dadd_rn(ucv[v], __dmul_rn(rhs[v], dt));
                }
                U5 nwu{nwv[0], nwv[1], nwv[2], nwv[3], nwv[4]};
                if (a.completes_step && ph.sponge) {
                    // the sphere case's outlet sponge toward the uniform freestream
                    // (rho, u_max, 0, 0, p), examples/sphere_drag_validation/main.rs:119-160
                    const double cx = centre(g.lo[0], g.h[0], i);
                    if (cx >= ph.sponge_x_start) {
                        const double s = fmin(fmax((cx - ph.sponge_x_start) * ph.sponge_inv_w, 0.0), 1.0);
                        const double f = fmin(ph.sponge_sigma * s * s * dt, 1.0);
                        // prim_to_cons5(rho, u_max, 0, 0, p), formed on the host
                        const U5 tg{ph.sponge_t[0], ph.sponge_t[1], ph.sponge_t[2], ph.sponge_t[3], ph.sponge_t[4]};
                        nwu.r += f * (tg.r - nwu.r);
                        nwu.mx += f * (tg.mx - nwu.mx);
                        nwu.my += f * (tg.my - nwu.my);
                        nwu.mz += f * (tg.mz - nwu.mz);
                        nwu.E += f * (tg.E - nwu.E);
                    }
                }
                store5(a.uout, P, o, nwu);
                write_ghosts3<PXYZ>(g, ph, a.uout, i, j, k, nwu);
                int bad = 0;
                if (!(nwu.r > 0.0)) bad |= 1;
                if (!(2.0 * nwu.E * nwu.r > nwu.mx * nwu.mx + nwu.my * nwu.my + nwu.mz * nwu.mz)) bad |= 2;
                if (nwu.r != nwu.r || nwu.mx != nwu.mx || nwu.my != nwu.my || nwu.mz != nwu.mz || nwu.E != nwu.E)
                    bad |= 4;
                if (bad) atomicOr(&a.st->nonphysical, bad);
                if (a.completes_step && a.want_cfl) lam = fmax(lam, wave_speed3(g, ph, nwu));
            }
            gb = gt;
            uc = un;
            un = un2;
            pc = pn;
        }
    }
    if (a.completes_step && a.want_cfl) {
        for (int o = 16; o > 0; o >>= 1) lam = fmax(lam, __shfl_xor_sync(0xffffffffu, lam, o));
        if (lane == 0 && lam > 0.0 && lam == lam)
            atomicMax(lam_slot(a.st), (unsigned long long)__double_as_longlong(lam));
    }
}

// Halo + Boundary of a whole 3-D state (after an upload): every interior cell
// writes the ghosts it is the source of, as the stage epilogue does.
__global__ void fill_ghosts3_kernel(Geometry g, Physics ph, double* q) {
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t / ((long long)g.nx * g.ny));
        const long long r = t - (long long)k * g.nx * g.ny;
        const int j = (int)(r / g.nx), i = (int)(r - (long long)j * g.nx);
        write_ghosts3(g, ph, q, i, j, k, load5(q, g.plane, cidx3(g, i, j, k)));
    }
}

__global__ void cfl3_kernel(Geometry g, Physics ph, const double* __restrict__ q, DevState* st) {
    double lam = 0.0;
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t / ((long long)g.nx * g.ny));
        const long long r = t - (long long)k * g.nx * g.ny;
        const int j = (int)(r / g.nx), i = (int)(r - (long long)j * g.nx);
        lam = fmax(lam, wave_speed3(g, ph, load5(q, g.plane, cidx3(g, i, j, k))));
    }
    block_max_atomic(lam, lam_slot(st));
}

// Strided host-like buffer (element (i, j, k, v) at i si + j sj + k sk + v sv)
// to or from the device layout.
__global__ void pack3_kernel(Geometry g, double* h, int64_t si, int64_t sj, int64_t sk, int64_t sv, double* q,
                             int to_device) {
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t / ((long long)g.nx * g.ny));
        const long long r = t - (long long)k * g.nx * g.ny;
        const int j = (int)(r / g.nx), i = (int)(r - (long long)j * g.nx);
        const long long o = cidx3(g, i, j, k);
        double* e = h + i * si + j * sj + k * sk;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            if (to_device) q[v * g.plane + o] = e[v * sv];
            else e[v * sv] = q[v * g.plane + o];
        }
    }
}

__global__ void total_mass3_kernel(Geometry g, const double* __restrict__ q, double* partial) {
    __shared__ double s1[256];
    double a = 0.0;
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t / ((long long)g.nx * g.ny));
        const long long r = t - (long long)k * g.nx * g.ny;
        const int j = (int)(r / g.nx), i = (int)(r - (long long)j * g.nx);
        a += q[cidx3(g, i, j, k)] * g.cell_volume;
    }
    s1[threadIdx.x] = a;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) s1[threadIdx.x] += s1[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s1[0];
}

// ---- immersed spheres (3-D) -------------------------------------------------
// refresh_sphere_mask, crates/cfd_ibm/src/sphere.rs:81-111: a cell whose centre
// is inside any sphere is solid; a cell that flips is seeded with the stagnant
// (fluid -> solid) or ambient (solid -> fluid) state.  The mask's ghost layers on
// a periodic axis hold the images of the interior (the reference's halo copies
// the mask with the state).  Every operation is rounded explicitly, as on the
// host, so the mask and the host-built lists agree.
__global__ void geometry3_kernel(Geometry g, Physics ph, const double* __restrict__ sph, int nb, U5 stagnant,
                                 U5 ambient, double* q, uint8_t* mask) {
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t / ((long long)g.nx * g.ny));
        const long long r = t - (long long)k * g.nx * g.ny;
        const int j = (int)(r / g.nx), i = (int)(r - (long long)j * g.nx);
        const double cc[3] = {centre(g.lo[0], g.h[0], i), centre(g.lo[1], g.h[1], j), centre(g.lo[2], g.h[2], k)};
        bool inside = false;
        for (int b = 0; b < nb && !inside; ++b) {
            const double* s = sph + 10 * b;
            const double d0 = __dsub_rn(cc[0], s[0]), d1 = __dsub_rn(cc[1], s[1]), d2 = __dsub_rn(cc[2], s[2]);
            const double rr = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2)));
            inside = __dsub_rn(rr, s[3]) < 0.0;
        }
        const long long o = cidx3(g, i, j, k);
        const bool was = mask[o] != 0;
        if (inside && !was) store5(q, g.plane, o, stagnant);
        else if (!inside && was) store5(q, g.plane, o, ambient);
        const uint8_t m = inside ? 1 : 0;
        mask[o] = m;
        if (ph.periodic_x) {
            if (i >= g.nx - NG) mask[cidx3(g, i - g.nx, j, k)] = m;
            if (i < NG) mask[cidx3(g, i + g.nx, j, k)] = m;
        }
        if (ph.periodic_y) {
            if (j >= g.ny - NG) mask[cidx3(g, i, j - g.ny, k)] = m;
            if (j < NG) mask[cidx3(g, i, j + g.ny, k)] = m;
        }
        if (ph.periodic_z) {
            if (k >= g.nz - NG) mask[cidx3(g, i, j, k - g.nz)] = m;
            if (k < NG) mask[cidx3(g, i, j, k + g.nz)] = m;
        }
    }
}

// sample_trilinear, crates/cfd_ibm/src/lib.rs:106-149: primitive (rho, u, v, w,
// p, T) at a located point from the fluid corners of its 2x2x2 block (clear
// corner bits are solid), skipping non-positive or non-finite densities, the
// weights renormalised; false when they sum below 1e-12.
__device__ __forceinline__ bool sample_trilinear3(const Geometry& g, const Physics& ph, const double* q,
                                                  unsigned fluid, const int lo[3], const double t[3], double out[6]) {
    const double gm1 = ph.gamma - 1.0;
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double total = 0.0;
#pragma unroll
    for (int di = 0; di < 2; ++di) {
        const double wx = di == 0 ? 1.0 - t[0] : t[0];
#pragma unroll
        for (int dj = 0; dj < 2; ++dj) {
            const double wy = dj == 0 ? 1.0 - t[1] : t[1];
#pragma unroll
            for (int dk = 0; dk < 2; ++dk) {
                const double wz = dk == 0 ? 1.0 - t[2] : t[2];
                if (!(fluid & (1u << (FLUID3_CORNER_SHIFT + 4 * di + 2 * dj + dk)))) continue;
                const U5 u = load5(q, g.plane, cidx3(g, lo[0] + di, lo[1] + dj, lo[2] + dk));
                if (!isfinite(u.r) || u.r <= 0.0) continue;
                const double w = wx * wy * wz;
                const double inv = 1.0 / u.r;
                const double vu = u.mx * inv, vv = u.my * inv, vw = u.mz * inv;
                const double ke = 0.5 * u.r * (vu * vu + vv * vv + vw * vw);
                const double p = gm1 * (u.E - ke);
                const double tt = p * inv / ph.r_gas;
                acc[0] += w * u.r;
                acc[1] += w * vu;
                acc[2] += w * vv;
                acc[3] += w * vw;
                acc[4] += w * p;
                acc[5] += w * tt;
                total += w;
            }
        }
    }
    if (total < 1e-12) return false;
    const double inv = 1.0 / total;
#pragma unroll
    for (int v = 0; v < 6; ++v) out[v] = acc[v] * inv;
    return true;
}

// apply_ibm_ghost_bc, crates/cfd_ibm/src/lib.rs:258-289: every ghost takes its
// image point's density, pressure and temperature and the velocity mirrored
// about the wall velocity, 2 u_w - u_image; a ghost whose sample fails keeps its
// value.
__global__ void mirror3_kernel(Geometry g, Physics ph, Ibm ib, double* q) {
    pdl_wait_then_release();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ib.n_ghost) return;
    const IbmGhost3Dev gh = ib.ghosts3[t];
    if (!gh.valid) return;
    double im[6];
    if (!sample_trilinear3(g, ph, q, gh.fluid, gh.lo, gh.t, im)) return;
    const double u = 2.0 * gh.uw[0] - im[1], v = 2.0 * gh.uw[1] - im[2], w = 2.0 * gh.uw[2] - im[3];
    const double ke = 0.5 * im[0] * (u * u + v * v + w * w);
    const U5 c{im[0], im[0] * u, im[0] * v, im[0] * w, im[4] / (ph.gamma - 1.0) + ke};
    store5(q, g.plane, cidx3(g, gh.i, gh.j, gh.k), c);
}

// marker_force_system + compute_marker_loadings (crates/cfd_ibm/src/lib.rs:442-480,
// 601-615) and wall_force_system (:309-395) over the state after a stage: one
// block, each thread summing a strided share of the markers and of the solid
// cells with fluid neighbours (the ghost list), then a fixed-order tree sum.
constexpr int FORCE3_THREADS = 256;
__global__ void __launch_bounds__(FORCE3_THREADS) forces3_kernel(Geometry g, Physics ph, Ibm ib, const double* q,
                                                                  DevState* st) {
    pdl_wait_then_release();
    __shared__ double red[12][FORCE3_THREADS];
    double f[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // marker p, v; wall p, v
    const double gm1 = ph.gamma - 1.0;
    for (int m = threadIdx.x; m < ib.n_markers; m += FORCE3_THREADS) {
        const Marker3Dev mk = ib.markers3[m];
        if (!mk.valid) continue;
        double img[6];
        if (!sample_trilinear3(g, ph, q, mk.fluid, mk.lo, mk.t, img)) continue;
        if (!(isfinite(img[4]) && isfinite(img[5]) && isfinite(img[1]) && isfinite(img[2]) && isfinite(img[3])))
            continue;
        const double us[3] = {img[1] - mk.uw[0], img[2] - mk.uw[1], img[3] - mk.uw[2]};
        const double udotn = us[0] * mk.normal[0] + us[1] * mk.normal[1] + us[2] * mk.normal[2];
        const double mu = viscosity(ph, img[5]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double ut = us[d] - udotn * mk.normal[d];
            f[d] += -img[4] * mk.normal[d] * mk.area;
            f[3 + d] += mu * ut / ib.sample_offset * mk.area;
        }
    }
    const double face_area[3] = {g.h[1] * g.h[2], g.h[0] * g.h[2], g.h[0] * g.h[1]};
    for (int t = threadIdx.x; t < ib.n_ghost; t += FORCE3_THREADS) {
        const IbmGhost3Dev gh = ib.ghosts3[t];
#pragma unroll
        for (int nbk = 0; nbk < 6; ++nbk) {
            if (!(gh.fluid & (1u << nbk))) continue;
            const int dim = nbk >> 1;
            const double sign = (nbk & 1) ? -1.0 : 1.0;
            const int di = dim == 0 ? (nbk & 1 ? -1 : 1) : 0, dj = dim == 1 ? (nbk & 1 ? -1 : 1) : 0,
                      dk = dim == 2 ? (nbk & 1 ? -1 : 1) : 0;
            const U5 uc = load5(q, g.plane, cidx3(g, gh.i + di, gh.j + dj, gh.k + dk));
            f[6 + dim] -= pressure5(uc, gm1) * sign * face_area[dim];
            const double inv = 1.0 / uc.r;
            const double vel[3] = {uc.mx * inv, uc.my * inv, uc.mz * inv};
            const double ke = 0.5 * uc.r * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
            const double tt = gm1 * (uc.E - ke) * inv / ph.r_gas;
            const double mu = viscosity(ph, tt);
#pragma unroll
            for (int td = 0; td < 3; ++td)
                if (td != dim) f[9 + td] += mu * vel[td] / (0.5 * g.h[dim]) * face_area[dim];
        }
    }
#pragma unroll
    for (int v = 0; v < 12; ++v) red[v][threadIdx.x] = f[v];
    __syncthreads();
    for (int s = FORCE3_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
#pragma unroll
            for (int v = 0; v < 12; ++v) red[v][threadIdx.x] += red[v][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int v = 0; v < 12; ++v) ib.force_out[v] = red[v][0];
        if (ib.history && st->hist_pos < st->hist_cap) {
            for (int d = 0; d < 6; ++d) ib.history[6 * st->hist_pos + d] = red[d][0];
            st->hist_pos += 1;
        }
    }
}

// ---- launches ---------------------------------------------------------------
// Rows per warp of the 3-D stage: the fewest that fill the resident slots in one
// wave, clamped to [2, 12].  A sweep at 256^3 over 4-16 rows and 3-5 resident
// blocks per SM measured 12 rows and 4 blocks fastest (6.53 ms per inviscid step
// against 6.65 at 8 rows; 3 and 5 blocks 15 % and 10 % slower).
static int rows_per_warp3(int nx, int ny, int nz) {
    const long long strips = (nx + STRIP - 1) / STRIP;
    const long long slots = 148LL * MINB3 * WPB3;
    long long rows = (strips * ny * nz + slots - 1) / slots;
    if (rows < 2) rows = 2;
    if (rows > 12) rows = 12;
    return (int)rows;
}

template <int SCHEME, int RECON, bool VISC, int LIM, bool PXYZ>
static void launch_stage3_k(const StageArgs& a, bool pdl, cudaStream_t s) {
    const int rows = rows_per_warp3(a.g.nx, a.g.ny, a.g.nz);
    const long long blocks = (long long)((a.g.nx + STRIP - 1) / STRIP) * ((a.g.nz + WPB3 - 1) / WPB3);
    dim3 grid((unsigned)blocks, (a.g.ny + rows - 1) / rows);
    launch_k(stage3_kernel<SCHEME, RECON, VISC, LIM, PXYZ>, grid, dim3(32 * WPB3), s, pdl, a, rows);
}

// The inviscid forms are built per limiter (MUSCL) and for fully periodic
// meshes, so those branches are decided at compile time (as the 2-D TMA-fed
// form is); the viscous forms read them at run time.
template <int SCHEME, int RECON, bool VISC>
static void launch_stage3_t(const StageArgs& a, bool pdl, cudaStream_t s) {
    if constexpr (VISC) {
        launch_stage3_k<SCHEME, RECON, VISC, -1, false>(a, pdl, s);
    } else {
        const bool pxyz = a.ph.periodic_x && a.ph.periodic_y && a.ph.periodic_z;
        if constexpr (RECON == EFVM_RECON_MUSCL) {
            if (a.ph.limiter == EFVM_LIMITER_MC)
                pxyz ? launch_stage3_k<SCHEME, RECON, VISC, EFVM_LIMITER_MC, true>(a, pdl, s)
                     : launch_stage3_k<SCHEME, RECON, VISC, EFVM_LIMITER_MC, false>(a, pdl, s);
            else
                pxyz ? launch_stage3_k<SCHEME, RECON, VISC, EFVM_LIMITER_MINMOD, true>(a, pdl, s)
                     : launch_stage3_k<SCHEME, RECON, VISC, EFVM_LIMITER_MINMOD, false>(a, pdl, s);
        } else {
            pxyz ? launch_stage3_k<SCHEME, RECON, VISC, -1, true>(a, pdl, s)
                 : launch_stage3_k<SCHEME, RECON, VISC, -1, false>(a, pdl, s);
        }
    }
}

template <bool VISC>
static void launch_stage3_v(const StageArgs& a, bool pdl, cudaStream_t s) {
    const bool muscl = a.ph.reconstruction == EFVM_RECON_MUSCL;
    switch (a.ph.flux_scheme) {
        case EFVM_FLUX_RUSANOV:
            muscl ? launch_stage3_t<EFVM_FLUX_RUSANOV, EFVM_RECON_MUSCL, VISC>(a, pdl, s)
                  : launch_stage3_t<EFVM_FLUX_RUSANOV, EFVM_RECON_FIRST_ORDER, VISC>(a, pdl, s);
            break;
        case EFVM_FLUX_HLLC_TEXTBOOK:
            muscl ? launch_stage3_t<EFVM_FLUX_HLLC_TEXTBOOK, EFVM_RECON_MUSCL, VISC>(a, pdl, s)
                  : launch_stage3_t<EFVM_FLUX_HLLC_TEXTBOOK, EFVM_RECON_FIRST_ORDER, VISC>(a, pdl, s);
            break;
        default:
            muscl ? launch_stage3_t<EFVM_FLUX_HLLC, EFVM_RECON_MUSCL, VISC>(a, pdl, s)
                  : launch_stage3_t<EFVM_FLUX_HLLC, EFVM_RECON_FIRST_ORDER, VISC>(a, pdl, s);
    }
}

static int launch_stage3(const StageArgs& a, bool pdl, cudaStream_t s) {
    if (a.ph.viscous) launch_stage3_v<true>(a, pdl, s);
    else launch_stage3_v<false>(a, pdl, s);
    return 1;
}
