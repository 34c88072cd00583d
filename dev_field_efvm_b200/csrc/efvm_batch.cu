// efvm_batch.cu — many independent cases advanced together.
//
// A parameter sweep or an ensemble runs hundreds of small grids; one context
// per case would launch a handful of kernels per case per step, and a 32^2 case
// fills a fraction of one SM.  A batch keeps every case's state in one pool and
// advances all of them with four launches per RK3 step: one set-up thread per
// case (its own dt from its own CFL maximum, its own clock and stop time) and
// one launch per stage over a table of tiles, each tile one warp's strip of one
// case.  Cases that reach their stop time drop out of the table, which the host
// rebuilds between chunks of steps (the step is a CUDA graph, re-captured when
// the table changes).  Per-case completion is stamped on the device global
// timer by the set-up that stops the case.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "efvm_internal.h"

using namespace efvm;

struct efvm_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    efvm_params params{};
    Physics ph{};                    // shared settings (from case 0)
    int n = 0;
    std::vector<Geometry> g;
    std::vector<Physics> phc;        // per case
    std::vector<BatchCase> cases;    // host copy of the case table
    BatchCase* cases_d = nullptr;
    DevState* st_d = nullptr;
    double* pool = nullptr;          // U[3] of every case
    double* yw_pool = nullptr;
    double* staging = nullptr;
    size_t staging_bytes = 0;
    int4* tiles_d = nullptr;
    int tiles_cap = 0;
    int n_tiles = 0;
    std::vector<char> fresh;         // state uploaded since the last run: CFL pass and ghost fill due
    std::vector<char> active;
    bool autotune = true;              // tune rows per warp per size bucket on the first run
    bool tuned = false;
    std::array<int, 4> bucket_rows{{0, 0, 0, 0}};  // 0 = the default heuristic
    cudaGraphExec_t graph = nullptr;
    unsigned long long* clock_d = nullptr;
    uint64_t launches = 0;
    std::string err;
};

namespace {

thread_local std::string g_batch_error;

int bfail(efvm_batch* b, int code, const std::string& msg) {
    if (b) b->err = msg;
    g_batch_error = msg;
    set_global_error(msg);
    return code;
}

#define BATCH_TRY(b, call)                                                                          \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return bfail(b, EFVM_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

int read_states(efvm_batch* b, std::vector<DevState>& s) {
    s.resize(b->n);
    BATCH_TRY(b, cudaMemcpyAsync(s.data(), b->st_d, b->n * sizeof(DevState), cudaMemcpyDeviceToHost, b->stream));
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    return EFVM_OK;
}

int write_states(efvm_batch* b, const std::vector<DevState>& s) {
    BATCH_TRY(b, cudaMemcpyAsync(b->st_d, s.data(), b->n * sizeof(DevState), cudaMemcpyHostToDevice, b->stream));
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    return EFVM_OK;
}

// Tiles of the active cases, case by case: (case, strip, row block).
int build_tiles(efvm_batch* b) {
    std::vector<int4> t;
    for (int k = 0; k < b->n; ++k) {
        if (!b->active[k]) continue;
        const int strips = stage_strips(b->g[k].nx);
        const int rows = b->cases[k].rows;
        const int blocks_y = (b->g[k].ny + rows - 1) / rows;
        for (int by = 0; by < blocks_y; ++by)
            for (int sx = 0; sx < strips; ++sx) t.push_back(make_int4(k, sx, by, 0));
    }
    if ((int)t.size() > b->tiles_cap) {
        if (b->tiles_d) cudaFree(b->tiles_d);
        b->tiles_d = nullptr;
        b->tiles_cap = 0;
        BATCH_TRY(b, cudaMalloc(&b->tiles_d, t.size() * sizeof(int4)));
        b->tiles_cap = (int)t.size();
    }
    if (!t.empty())
        BATCH_TRY(b, cudaMemcpyAsync(b->tiles_d, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice, b->stream));
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    b->n_tiles = (int)t.size();
    return EFVM_OK;
}

// ---- the autotuner -----------------------------------------------------------
// Rows per warp is the one tiling choice of the stage kernel that depends on the
// case size: more rows amortise each strip's first y face, fewer rows give more
// warps.  Cases are grouped in size buckets (cells < 64^2, < 128^2, < 256^2,
// larger); for each bucket present the tuner times one batch step with 2, 4 and
// 8 rows and keeps the fastest, on a copy of the states (restored afterwards, so
// tuning changes no result).  Choices are cached per process for the device, its
// SM count, the numerical method and the set of buckets present.
constexpr int N_BUCKETS = 4;
constexpr int ROW_CHOICES[3] = {2, 4, 8};

int size_bucket(const Geometry& g) {
    const long long c = (long long)g.nx * g.ny;
    return c < 64 * 64 ? 0 : c < 128 * 128 ? 1 : c < 256 * 256 ? 2 : 3;
}

using TuneKey = std::tuple<int, int, int, int, int, int>;
std::mutex g_tune_mu;
std::map<TuneKey, std::array<int, 4>> g_tune_cache;

// One RK3 step of every active case: set-up, then the three stages.
void enqueue_step(efvm_batch* b) {
    b->launches += launch_batch_setup(b->ph, b->cases_d, b->n, true, b->stream);
    const int in_buf[3] = {0, 1, 2}, out_buf[3] = {1, 2, 0};
    for (int s = 0; s < 3; ++s) {
        BatchStageArgs a{};
        a.ph = b->ph;
        a.cases = b->cases_d;
        a.tiles = b->tiles_d;
        a.stage = s;
        a.completes_step = s == 2;
        a.want_cfl = s == 2 && b->ph.fixed_dt <= 0.0;
        a.in_buf = in_buf[s];
        a.out_buf = out_buf[s];
        b->launches += launch_batch_stage(a, b->n_tiles, true, b->stream);
    }
}

int capture(efvm_batch* b) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    const uint64_t before = b->launches;
    cudaGraph_t graph;
    BATCH_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_step(b);
    cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    b->launches = before;
    if (e != cudaSuccess) return bfail(b, EFVM_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return bfail(b, EFVM_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(e));
    return EFVM_OK;
}

// Rows of every case from the per-bucket choice (0 = default), uploaded.
int apply_rows(efvm_batch* b) {
    const bool fp32 = b->params.precision == EFVM_PREC_FP32_FLUX;
    for (int k = 0; k < b->n; ++k) {
        const int r = b->bucket_rows[size_bucket(b->g[k])];
        b->cases[k].rows = r > 0 ? r : std::min(stage_rows(b->g[k].nx, b->g[k].ny, fp32, b->ph.viscous), 8);
    }
    BATCH_TRY(b, cudaMemcpyAsync(b->cases_d, b->cases.data(), b->n * sizeof(BatchCase), cudaMemcpyHostToDevice,
                                 b->stream));
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    return EFVM_OK;
}

int tune(efvm_batch* b) {
    int present = 0;
    for (int k = 0; k < b->n; ++k) present |= 1 << size_bucket(b->g[k]);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    const TuneKey key{b->device, sms, b->params.precision, b->params.flux_scheme * 2 + b->params.reconstruction,
                      b->params.limiter, present};
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            b->bucket_rows = it->second;
            return apply_rows(b);
        }
    }
    // work on the live buffers, then put states and clocks back
    size_t pool_bytes = 0;
    for (int k = 0; k < b->n; ++k) pool_bytes += 3 * (((size_t)4 * b->g[k].plane + 31) / 32 * 32) * sizeof(double);
    double* backup = nullptr;
    BATCH_TRY(b, cudaMalloc(&backup, pool_bytes));
    std::vector<DevState> saved;
    int rc = read_states(b, saved);
    if (rc) return rc;
    BATCH_TRY(b, cudaMemcpyAsync(backup, b->pool, pool_bytes, cudaMemcpyDeviceToDevice, b->stream));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int bucket = 0; bucket < N_BUCKETS && rc == EFVM_OK; ++bucket) {
        if (!(present & (1 << bucket))) continue;
        float best_ms = 1e30f;
        int best = ROW_CHOICES[0];
        for (int r : ROW_CHOICES) {
            b->bucket_rows[bucket] = r;
            if ((rc = apply_rows(b)) || (rc = build_tiles(b)) || (rc = capture(b))) break;
            cudaGraphLaunch(b->graph, b->stream);  // warm-up
            cudaEventRecord(e0, b->stream);
            for (int i = 0; i < 2; ++i) cudaGraphLaunch(b->graph, b->stream);
            cudaEventRecord(e1, b->stream);
            cudaError_t e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) {
                rc = bfail(b, EFVM_ERR_CUDA, std::string("batch autotune: ") + cudaGetErrorString(e));
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best_ms) {
                best_ms = ms;
                best = r;
            }
        }
        b->bucket_rows[bucket] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaMemcpyAsync(b->pool, backup, pool_bytes, cudaMemcpyDeviceToDevice, b->stream);
    const int rc2 = write_states(b, saved);
    cudaFree(backup);
    if (rc) return rc;
    if (rc2) return rc2;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache[key] = b->bucket_rows;
    }
    return apply_rows(b);
}

}  // namespace

extern "C" {

int efvm_batch_create(const efvm_grid* grids, int32_t n_cases, const efvm_params* params, efvm_batch** out) {
    if (!grids || !params || !out || n_cases < 1) return bfail(nullptr, EFVM_ERR_INVALID_ARG, "efvm_batch_create: null argument or n_cases < 1");
    *out = nullptr;
    if (params->integrator != EFVM_INTEGRATOR_RK3)
        return bfail(nullptr, EFVM_ERR_UNSUPPORTED, "efvm_batch_create: batches run SSP-RK3 only");
    efvm_batch* b = new efvm_batch();
    b->n = n_cases;
    b->params = *params;
    cudaGetDevice(&b->device);
    b->g.resize(n_cases);
    b->phc.resize(n_cases);
    for (int k = 0; k < n_cases; ++k) {
        std::string err;
        if (grids[k].nz != 1) {
            delete b;
            return bfail(nullptr, EFVM_ERR_UNSUPPORTED, "efvm_batch_create: case " + std::to_string(k) +
                                                            ": batches hold 2-D cases (nz == 1)");
        }
        const int rc = setup_case(grids[k], *params, 0, grids[k].ny, false, b->g[k], b->phc[k], err);
        if (rc) {
            delete b;
            return bfail(nullptr, rc, "efvm_batch_create: case " + std::to_string(k) + ": " + err);
        }
    }
    b->ph = b->phc[0];
    auto cleanup = [&](int code) {
        efvm_batch_destroy(b);
        return code;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete b;
        return bfail(nullptr, EFVM_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    // one pool for every case's three states; each state starts on a 256-byte boundary
    std::vector<size_t> off(n_cases);
    size_t total = 0, yw_total = 0;
    for (int k = 0; k < n_cases; ++k) {
        off[k] = total;
        const size_t state = ((size_t)4 * b->g[k].plane + 31) / 32 * 32;
        total += 3 * state;
        yw_total += 3 * (size_t)b->g[k].ny;
    }
    if (cudaMalloc(&b->pool, total * sizeof(double)) != cudaSuccess)
        return cleanup(bfail(nullptr, EFVM_ERR_OOM, "efvm_batch_create: cudaMalloc state pool"));
    cudaMemsetAsync(b->pool, 0, total * sizeof(double), b->stream);
    if (cudaMalloc(&b->yw_pool, yw_total * sizeof(double)) != cudaSuccess)
        return cleanup(bfail(nullptr, EFVM_ERR_OOM, "efvm_batch_create: cudaMalloc"));
    if (cudaMalloc(&b->st_d, n_cases * sizeof(DevState)) != cudaSuccess)
        return cleanup(bfail(nullptr, EFVM_ERR_OOM, "efvm_batch_create: cudaMalloc"));
    if (cudaMalloc(&b->cases_d, n_cases * sizeof(BatchCase)) != cudaSuccess)
        return cleanup(bfail(nullptr, EFVM_ERR_OOM, "efvm_batch_create: cudaMalloc"));
    if (cudaMalloc(&b->clock_d, sizeof(unsigned long long)) != cudaSuccess)
        return cleanup(bfail(nullptr, EFVM_ERR_OOM, "efvm_batch_create: cudaMalloc"));
    std::vector<double> yw_all;
    yw_all.reserve(yw_total);
    b->cases.resize(n_cases);
    const bool fp32 = params->precision == EFVM_PREC_FP32_FLUX;
    for (int k = 0; k < n_cases; ++k) {
        BatchCase& c = b->cases[k];
        c.g = b->g[k];
        c.ph = b->phc[k];
        // rows per warp: a batch fills the GPU with many cases, so each case takes
        // the rows it would take alone, at most 8
        c.rows = std::min(stage_rows(c.g.nx, c.g.ny, fp32, c.ph.viscous), 8);
        const size_t state = ((size_t)4 * c.g.plane + 31) / 32 * 32;
        for (int s = 0; s < 3; ++s) c.U[s] = b->pool + off[k] + s * state;
        c.yw = b->yw_pool + yw_all.size();
        const std::vector<double> yw = viscous_y_weights(c.g);
        yw_all.insert(yw_all.end(), yw.begin(), yw.end());
        c.st = b->st_d + k;
    }
    std::vector<DevState> s0(n_cases);
    for (auto& s : s0) {
        s = DevState{};
        s.active = 1;
    }
    cudaMemcpyAsync(b->yw_pool, yw_all.data(), yw_total * sizeof(double), cudaMemcpyHostToDevice, b->stream);
    cudaMemcpyAsync(b->st_d, s0.data(), n_cases * sizeof(DevState), cudaMemcpyHostToDevice, b->stream);
    cudaMemcpyAsync(b->cases_d, b->cases.data(), n_cases * sizeof(BatchCase), cudaMemcpyHostToDevice, b->stream);
    e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return cleanup(bfail(nullptr, EFVM_ERR_CUDA, std::string("efvm_batch_create: ") + cudaGetErrorString(e)));
    b->fresh.assign(n_cases, 1);
    b->active.assign(n_cases, 1);
    *out = b;
    return EFVM_OK;
}

int efvm_batch_destroy(efvm_batch* b) {
    if (!b) return EFVM_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    cudaFree(b->pool);
    cudaFree(b->yw_pool);
    cudaFree(b->st_d);
    cudaFree(b->cases_d);
    cudaFree(b->tiles_d);
    cudaFree(b->staging);
    cudaFree(b->clock_d);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return EFVM_OK;
}

const char* efvm_batch_last_error(const efvm_batch* b) { return b ? b->err.c_str() : g_batch_error.c_str(); }

static int batch_transfer(efvm_batch* b, int32_t k, double* base, int64_t si, int64_t sj, int64_t sv, bool upload) {
    if (!b || !base) return bfail(b, EFVM_ERR_INVALID_ARG, "null argument");
    if (k < 0 || k >= b->n) return bfail(b, EFVM_ERR_INVALID_ARG, "case index out of range");
    const Geometry& g = b->g[k];
    int64_t lo = 0, hi = 0;
    const int64_t corners[3] = {(int64_t)(g.nx - 1) * si, (int64_t)(g.ny - 1) * sj, 4 * sv};
    for (int d = 0; d < 3; ++d) {
        lo += std::min<int64_t>(0, corners[d]);
        hi += std::max<int64_t>(0, corners[d]);
    }
    const int64_t span = hi - lo + 1;
    const bool dense = span == (int64_t)g.nx * g.ny * 5;
    if ((size_t)span * sizeof(double) > b->staging_bytes) {
        cudaFree(b->staging);
        b->staging = nullptr;
        b->staging_bytes = 0;
        BATCH_TRY(b, cudaMalloc(&b->staging, (size_t)span * sizeof(double)));
        b->staging_bytes = (size_t)span * sizeof(double);
    }
    double* host0 = base + lo;
    double* dev0 = b->staging - lo;
    double* q = b->cases[k].U[0];
    if (upload) {
        BATCH_TRY(b, cudaMemcpyAsync(b->staging, host0, (size_t)span * sizeof(double), cudaMemcpyHostToDevice, b->stream));
        b->launches += launch_pack(g, dev0, si, sj, sv, q, 1, b->stream);
        b->fresh[k] = 1;
    } else {
        if (!dense)
            BATCH_TRY(b, cudaMemcpyAsync(b->staging, host0, (size_t)span * sizeof(double), cudaMemcpyHostToDevice, b->stream));
        b->launches += launch_pack(g, dev0, si, sj, sv, q, 0, b->stream);
        BATCH_TRY(b, cudaMemcpyAsync(host0, b->staging, (size_t)span * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    }
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    BATCH_TRY(b, cudaGetLastError());
    return EFVM_OK;
}

int efvm_batch_upload_state(efvm_batch* b, int32_t k, const double* base, int64_t si, int64_t sj, int64_t sv) {
    return batch_transfer(b, k, const_cast<double*>(base), si, sj, sv, true);
}

int efvm_batch_download_state(efvm_batch* b, int32_t k, double* base, int64_t si, int64_t sj, int64_t sv) {
    return batch_transfer(b, k, base, si, sj, sv, false);
}

int efvm_batch_get_solver_state(efvm_batch* b, int32_t k, efvm_solver_state* out) {
    if (!b || !out) return bfail(b, EFVM_ERR_INVALID_ARG, "null argument");
    if (k < 0 || k >= b->n) return bfail(b, EFVM_ERR_INVALID_ARG, "case index out of range");
    DevState s;
    BATCH_TRY(b, cudaMemcpyAsync(&s, b->st_d + k, sizeof(DevState), cudaMemcpyDeviceToHost, b->stream));
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    out->dt = s.dt;
    out->time = s.time;
    out->step = s.step;
    out->rk_stage = s.rk_stage;
    out->completed_full_step = s.completed;
    return EFVM_OK;
}

int efvm_batch_run(efvm_batch* b, const double* t_stop, int64_t max_steps, int64_t chunk,
                   efvm_batch_case_result* results) {
    if (!b || !t_stop) return bfail(b, EFVM_ERR_INVALID_ARG, "null argument");
    if (max_steps < 0) return bfail(b, EFVM_ERR_INVALID_ARG, "max_steps must be >= 0");
    if (chunk < 1) chunk = 16;
    // a freshly uploaded case: CFL maximum of its state and its boundary ghosts
    for (int k = 0; k < b->n; ++k) {
        if (!b->fresh[k]) continue;
        if (b->ph.fixed_dt <= 0.0) b->launches += launch_cfl(b->g[k], b->phc[k], b->cases[k].U[0], b->st_d + k, b->stream);
        b->launches += launch_fill_ghosts(b->g[k], b->phc[k], b->cases[k].U[0], b->stream);
        b->fresh[k] = 0;
    }
    std::vector<DevState> s;
    int rc = read_states(b, s);
    if (rc) return rc;
    std::vector<unsigned long long> step0(b->n);
    for (int k = 0; k < b->n; ++k) {
        s[k].active = 1;
        s[k].stop_at_t = 1;
        s[k].t_stop = t_stop[k];
        s[k].nonphysical = 0;
        s[k].done_ns = 0;
        step0[k] = s[k].step;
        b->active[k] = 1;
    }
    rc = write_states(b, s);
    if (rc) return rc;
    if (b->autotune && !b->tuned) {
        rc = tune(b);
        if (rc) return rc;
        b->tuned = true;
    }
    b->launches += launch_clock(b->clock_d, b->stream);
    rc = build_tiles(b);
    if (rc) return rc;
    rc = capture(b);
    if (rc) return rc;
    int64_t done = 0;
    while (done < max_steps) {
        const int64_t m = std::min<int64_t>(chunk, max_steps - done);
        for (int64_t i = 0; i < m; ++i) {
            BATCH_TRY(b, cudaGraphLaunch(b->graph, b->stream));
            b->launches += 4;
        }
        done += m;
        rc = read_states(b, s);
        if (rc) return rc;
        bool changed = false, any = false;
        for (int k = 0; k < b->n; ++k) {
            const char a = s[k].active ? 1 : 0;
            if (a != b->active[k]) changed = true;
            b->active[k] = a;
            any |= a != 0;
        }
        if (!any) break;
        if (changed) {
            rc = build_tiles(b);
            if (rc) return rc;
            rc = capture(b);
            if (rc) return rc;
        }
    }
    unsigned long long start = 0;
    BATCH_TRY(b, cudaMemcpyAsync(&start, b->clock_d, sizeof(start), cudaMemcpyDeviceToHost, b->stream));
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    int status = EFVM_OK;
    for (int k = 0; k < b->n; ++k) {
        if (results) {
            efvm_batch_case_result& r = results[k];
            r.steps = (int64_t)(s[k].step - step0[k]);
            r.time = s[k].time;
            r.completion_ms = s[k].done_ns ? (double)(s[k].done_ns - start) * 1e-6 : -1.0;
            r.nonphysical = s[k].nonphysical;
            r.finished = s[k].active ? 0 : 1;
        }
        if (s[k].nonphysical) status = EFVM_ERR_NONPHYSICAL;
    }
    if (status) return bfail(b, status, "a case of the batch went non-physical (rho<=0, p<=0 or NaN)");
    return EFVM_OK;
}

int efvm_batch_launch_count(efvm_batch* b, uint64_t* out) {
    if (!b || !out) return bfail(b, EFVM_ERR_INVALID_ARG, "null argument");
    *out = b->launches;
    return EFVM_OK;
}

int efvm_batch_set_autotune(efvm_batch* b, int32_t enable) {
    if (!b) return bfail(b, EFVM_ERR_INVALID_ARG, "null argument");
    b->autotune = enable != 0;
    if (!b->autotune) {
        b->bucket_rows = {{0, 0, 0, 0}};
        b->tuned = false;
        return apply_rows(b);
    }
    return EFVM_OK;
}

int efvm_batch_get_rows(efvm_batch* b, int32_t rows[4]) {
    if (!b || !rows) return bfail(b, EFVM_ERR_INVALID_ARG, "null argument");
    for (int i = 0; i < 4; ++i) rows[i] = b->bucket_rows[i];
    return EFVM_OK;
}

int efvm_batch_get_stream(efvm_batch* b, void** stream) {
    if (!b || !stream) return bfail(b, EFVM_ERR_INVALID_ARG, "null argument");
    *stream = (void*)b->stream;
    return EFVM_OK;
}

}  // extern "C"
