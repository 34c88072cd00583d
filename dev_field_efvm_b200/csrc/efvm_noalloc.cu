// efvm_noalloc.cu — the CFL time step of a caller-owned device state, computed
// without allocating any memory.
//
// Some callers cannot let a library call cudaMalloc: their device memory is
// owned by another allocator (a host framework's pool or a fixed per-process
// budget), so every byte has to come from them or already exist.  This entry
// point takes the state and the output from the caller and keeps its only
// scratch — one wave-speed maximum per grid row plus a completion counter — in
// file-scope __device__ storage that exists on every GPU that loads the
// library, from load until process exit.
//
// The scratch is shared by all calls on a device and keeps the previous call's
// contents.  The row maxima are fully rewritten by every call; the counter is
// cleared at the start of every call.  Two calls whose kernels overlap on the
// GPU (different streams, no ordering between them) race on the scratch and
// may return wrong values: order such calls on one stream or with events.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "efvm_internal.h"

namespace {

constexpr int NOALLOC_THREADS = 256;

// The scratch.  In host code these names are host-side stand-ins, not device
// addresses; the host looks the device addresses up with
// cudaGetSymbolAddress and passes them to the kernel.
static __device__ __align__(256) double g_cfl_row_max[EFVM_CFL_NOALLOC_MAX_ROWS];
static __device__ __align__(256) unsigned int g_cfl_rows_done;

struct ScratchAddr {
    double* row_max = nullptr;
    unsigned int* done = nullptr;
};

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
ScratchAddr g_addr[MAX_DEVICES];

// One-time look-up of the scratch's device addresses on the current device.
int scratch_for_current_device(ScratchAddr& out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        efvm::set_global_error(std::string("efvm_cfl_dt_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
        return EFVM_ERR_CUDA;
    }
    if (dev < 0 || dev >= MAX_DEVICES) {
        efvm::set_global_error("efvm_cfl_dt_noalloc: device ordinal out of range");
        return EFVM_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev].row_max) {
        ScratchAddr a;
        e = cudaGetSymbolAddress((void**)&a.row_max, g_cfl_row_max);
        if (e != cudaSuccess) {
            efvm::set_global_error(std::string("efvm_cfl_dt_noalloc: cudaGetSymbolAddress(row maxima): ") + cudaGetErrorString(e));
            return EFVM_ERR_CUDA;
        }
        e = cudaGetSymbolAddress((void**)&a.done, g_cfl_rows_done);
        if (e != cudaSuccess) {
            efvm::set_global_error(std::string("efvm_cfl_dt_noalloc: cudaGetSymbolAddress(counter): ") + cudaGetErrorString(e));
            return EFVM_ERR_CUDA;
        }
        g_addr[dev] = a;
    }
    out = g_addr[dev];
    return EFVM_OK;
}

struct CflArgs {
    const double *rho, *mx, *my, *E;
    long long pitch;
    int nx, ny;
    double dx, dy, dz;
    double idx, idy, idz, inv_r_gas;  // 1 / dx, 1 / dy, 1 / dz, 1 / R
    double gamma, r_gas, cfl, fixed_dt;
    int viscous, visc_model;
    double mu, visc_sum;
};

// Same wave speed as the context path's CFL (cfl_system's per-cell lambda with
// the z term of the 2-D mesh and the optional viscous spectral radius), in the
// context path's form: the reference's divisions by rho, dx, dy, dz and R taken
// as products with reciprocals.  Every operation is rounded explicitly (no FMA
// contraction), as in the context path, so the two agree bit for bit.
__device__ double cell_lambda(const CflArgs& a, double r, double mx, double my, double E) {
    if (!(r > 0.0)) return 0.0;
    const double gm1 = a.gamma - 1.0;
    const double inv = 1.0 / r;
    const double vx = __dmul_rn(mx, inv), vy = __dmul_rn(my, inv);
    const double ke = __dmul_rn(__dmul_rn(0.5, r), __dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)));
    const double p = __dmul_rn(gm1, __dsub_rn(E, ke));
    const double c = sqrt(__dmul_rn(__dmul_rn(a.gamma, p), inv));
    double lam = __dadd_rn(__dadd_rn(__dmul_rn(__dadd_rn(fabs(vx), c), a.idx), __dmul_rn(__dadd_rn(fabs(vy), c), a.idy)),
                           __dmul_rn(__dadd_rn(0.0, c), a.idz));
    if (a.viscous) {
        const double t = __dmul_rn(__dmul_rn(p, inv), a.inv_r_gas);
        double mu = a.mu;
        if (a.visc_model == EFVM_VISC_SUTHERLAND) {
            const double MU_REF = 1.827e-5, T_REF = 291.15, S = 120.0;
            mu = MU_REF * pow(t / T_REF, 1.5) * (T_REF + S) / (t + S);
        }
        lam = __dadd_rn(lam, __dmul_rn(__dmul_rn(2.0, __dmul_rn(mu, inv)), a.visc_sum));
    }
    return lam;
}

// One block per grid row writes that row's maximum into the scratch; the last
// block to finish takes the maximum over the rows and writes dt.
__global__ void __launch_bounds__(NOALLOC_THREADS) cfl_noalloc_kernel(CflArgs a, double* row_max, unsigned int* done,
                                                                     double* dt_out) {
    __shared__ double red[NOALLOC_THREADS / 32];
    __shared__ bool last;
    const int j = blockIdx.x;
    double lam = 0.0;
    for (int i = threadIdx.x; i < a.nx; i += blockDim.x) {
        const long long o = (long long)j * a.pitch + i;
        lam = fmax(lam, cell_lambda(a, a.rho[o], a.mx[o], a.my[o], a.E[o]));
    }
    for (int s = 16; s > 0; s >>= 1) lam = fmax(lam, __shfl_xor_sync(0xffffffffu, lam, s));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lam;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < NOALLOC_THREADS / 32; ++w) m = fmax(m, red[w]);
        row_max[j] = m;
        __threadfence();
        last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        const volatile double* rm = row_max;
        double m = 0.0;
        for (int r = 0; r < (int)gridDim.x; ++r) m = fmax(m, rm[r]);
        *dt_out = a.fixed_dt > 0.0 ? a.fixed_dt : (m > 0.0 ? a.cfl / m : INFINITY);
        *done = 0u;
    }
}

}  // namespace

extern "C" int efvm_cfl_dt_noalloc(const double* rho, const double* rho_u, const double* rho_v, const double* rho_e,
                                   int64_t pitch, const efvm_grid* grid, const efvm_params* params, double* dt_out,
                                   void* stream) {
    if (!rho || !rho_u || !rho_v || !rho_e || !grid || !params || !dt_out) {
        efvm::set_global_error("efvm_cfl_dt_noalloc: null argument");
        return EFVM_ERR_INVALID_ARG;
    }
    if (grid->nx < 1 || grid->ny < 1 || pitch < grid->nx) {
        efvm::set_global_error("efvm_cfl_dt_noalloc: need nx >= 1, ny >= 1 and pitch >= nx");
        return EFVM_ERR_INVALID_ARG;
    }
    if (grid->nz > 1) {
        // the entry point takes no rho_w plane and reads one layer: a 3-D mesh's
        // wave speed needs |w| and every layer (efvm_cfl handles 3-D contexts)
        efvm::set_global_error("efvm_cfl_dt_noalloc: nz = " + std::to_string(grid->nz) +
                               ": only 2-D meshes (nz <= 1) are supported; use efvm_cfl");
        return EFVM_ERR_UNSUPPORTED;
    }
    for (int a = 0; a < 3; ++a) {
        if (!(grid->hi[a] > grid->lo[a])) {  // also rejects NaN bounds
            efvm::set_global_error("efvm_cfl_dt_noalloc: the mesh extent hi - lo must be positive on every axis");
            return EFVM_ERR_INVALID_ARG;
        }
    }
    if (grid->ny > EFVM_CFL_NOALLOC_MAX_ROWS) {
        efvm::set_global_error("efvm_cfl_dt_noalloc: ny = " + std::to_string(grid->ny) + " exceeds the " +
                std::to_string(EFVM_CFL_NOALLOC_MAX_ROWS) + "-row scratch of this entry point; use efvm_cfl");
        return EFVM_ERR_INVALID_ARG;
    }
    if (!(params->gamma > 1.0) || (!(params->cfl > 0.0) && !(params->fixed_dt > 0.0))) {
        efvm::set_global_error("efvm_cfl_dt_noalloc: gamma must exceed 1 and cfl or fixed_dt must be > 0");
        return EFVM_ERR_INVALID_ARG;
    }
    ScratchAddr s;
    int rc = scratch_for_current_device(s);
    if (rc) return rc;
    CflArgs a;
    a.rho = rho;
    a.mx = rho_u;
    a.my = rho_v;
    a.E = rho_e;
    a.pitch = pitch;
    a.nx = grid->nx;
    a.ny = grid->ny;
    a.dx = (grid->hi[0] - grid->lo[0]) / (double)grid->nx;
    a.dy = (grid->hi[1] - grid->lo[1]) / (double)grid->ny;
    a.dz = (grid->hi[2] - grid->lo[2]) / (double)(grid->nz > 0 ? grid->nz : 1);
    a.idx = 1.0 / a.dx;
    a.idy = 1.0 / a.dy;
    a.idz = 1.0 / a.dz;
    a.inv_r_gas = 1.0 / params->r_gas;
    a.gamma = params->gamma;
    a.r_gas = params->r_gas;
    a.cfl = params->cfl;
    a.fixed_dt = params->fixed_dt;
    a.viscous = params->viscous;
    a.visc_model = params->viscosity_model;
    a.mu = params->mu;
    a.visc_sum = 1.0 / (a.dx * a.dx) + 1.0 / (a.dy * a.dy) + 1.0 / (a.dz * a.dz);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(s.done, 0, sizeof(unsigned int), st);  // counter starts at zero
    if (e != cudaSuccess) {
        efvm::set_global_error(std::string("efvm_cfl_dt_noalloc: clearing the counter: ") + cudaGetErrorString(e));
        return EFVM_ERR_CUDA;
    }
    cfl_noalloc_kernel<<<grid->ny, NOALLOC_THREADS, 0, st>>>(a, s.row_max, s.done, dt_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        efvm::set_global_error(std::string("efvm_cfl_dt_noalloc: launch: ") + cudaGetErrorString(e));
        return EFVM_ERR_CUDA;
    }
    return EFVM_OK;
}
