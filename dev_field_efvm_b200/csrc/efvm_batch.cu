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
    int graph_steps = 0;               // steps one replay of `graph` runs
    unsigned long long* clock_d = nullptr;
    uint64_t launches = 0;
    std::string err;
    // the persistent kernel (on by default): one launch per chunk of steps
    bool persistent = true;
    int n_sms = 0;
    int blocks_per_sm = 0;             // resident blocks per SM of its grid (0 = the form's maximum)
    unsigned int* ready_d = nullptr;   // per case (PersistArgs)
    unsigned int* done_d = nullptr;
    int* case_tiles_d = nullptr;
    unsigned long long* ticket_d = nullptr;
    int* status_d = nullptr;
    double wait_s = 2.0;               // limit of one wait in the persistent kernel
    int stall_case = -1;               // test hook: the next run's table claims one tile too many for this case
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

// Tiles of the active cases, case by case: (case, strip, row block), and the
// number of tiles of each case (the persistent kernel's completion counts).
int build_tiles(efvm_batch* b) {
    std::vector<int4> t;
    std::vector<int> per_case(b->n, 0);
    for (int k = 0; k < b->n; ++k) {
        if (!b->active[k]) continue;
        const int strips = stage_strips(b->g[k].nx);
        const int rows = b->cases[k].rows;
        const int blocks_y = (b->g[k].ny + rows - 1) / rows;
        for (int by = 0; by < blocks_y; ++by)
            for (int sx = 0; sx < strips; ++sx) t.push_back(make_int4(k, sx, by, 0));
        per_case[k] = strips * blocks_y;
    }
    // fault injection for the bounded waits: the case's stages can never complete
    if (b->stall_case >= 0 && b->stall_case < b->n && per_case[b->stall_case] > 0) per_case[b->stall_case] += 1;
    BATCH_TRY(b, cudaMemcpyAsync(b->case_tiles_d, per_case.data(), b->n * sizeof(int), cudaMemcpyHostToDevice,
                                 b->stream));
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

int resident_blocks(const efvm_batch* b) {
    const int form = batch_form_blocks(b->params.precision == EFVM_PREC_FP32_FLUX, b->ph.viscous != 0);
    return b->blocks_per_sm > 0 ? std::min(b->blocks_per_sm, form) : form;
}

// `steps` RK3 steps of every active case.  Persistent: the first step's set-up,
// then one launch for all 3 x steps stages (the later set-ups run inside it).
// Otherwise per step a set-up launch and one launch per stage over the table.
void enqueue_steps(efvm_batch* b, int steps) {
    if (b->persistent) {
        b->launches += launch_batch_setup(b->ph, b->cases_d, b->n, false, b->stream);
        cudaMemsetAsync(b->ready_d, 0, b->n * sizeof(unsigned int), b->stream);
        cudaMemsetAsync(b->done_d, 0, b->n * sizeof(unsigned int), b->stream);
        cudaMemsetAsync(b->ticket_d, 0, sizeof(unsigned long long), b->stream);
        PersistArgs p{};
        p.ph = b->ph;
        p.cases = b->cases_d;
        p.tiles = b->tiles_d;
        p.case_tiles = b->case_tiles_d;
        p.ready = b->ready_d;
        p.done = b->done_d;
        p.ticket = b->ticket_d;
        p.status = b->status_d;
        p.n_tiles = b->n_tiles;
        p.rounds = 3 * steps;
        p.want_cfl = b->ph.fixed_dt <= 0.0;
        p.wait_ns = (unsigned long long)(b->wait_s * 1e9);
        b->launches += launch_batch_persistent(p, resident_blocks(b), b->n_sms, b->stream);
        return;
    }
    for (int step = 0; step < steps; ++step) {
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
}

// Launches per replay of the captured steps.
uint64_t launches_per_replay(const efvm_batch* b, int steps) { return b->persistent ? 2 : 4ull * steps; }

int capture(efvm_batch* b, int steps) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    const uint64_t before = b->launches;
    cudaGraph_t graph;
    BATCH_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_steps(b, steps);
    cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    b->launches = before;
    if (e != cudaSuccess) return bfail(b, EFVM_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return bfail(b, EFVM_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(e));
    b->graph_steps = steps;
    return EFVM_OK;
}

// ---- the autotuner -----------------------------------------------------------
// Two tiling choices of the batch depend on the case sizes and the device: the
// tile height (rows per warp; more rows amortise each strip's first y face,
// fewer give more tiles) per case-size bucket (cells < 64^2, < 128^2, < 256^2,
// larger), and, for the persistent kernel, its resident blocks per SM.  The
// tuner times one batch step for each height per bucket present (greedily,
// bucket by bucket), then each block count, on the live states (restored
// afterwards, so tuning changes no result), and keeps the fastest.  Choices are
// cached per process for the device, its SM count, the numerical method, the
// kernel and the set of buckets present.
constexpr int N_BUCKETS = 4;
constexpr int ROW_CHOICES[4] = {2, 4, 8, 16};

int size_bucket(const Geometry& g) {
    const long long c = (long long)g.nx * g.ny;
    return c < 64 * 64 ? 0 : c < 128 * 128 ? 1 : c < 256 * 256 ? 2 : 3;
}

using TuneKey = std::tuple<int, int, int, int, int, int, int>;
struct TuneChoice {
    std::array<int, 4> rows;
    int blocks_per_sm;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneChoice> g_tune_cache;

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
    const TuneKey key{b->device, b->n_sms, b->params.precision, b->params.flux_scheme * 2 + b->params.reconstruction,
                      b->params.limiter, present, b->persistent ? 1 : 0};
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            b->bucket_rows = it->second.rows;
            b->blocks_per_sm = it->second.blocks_per_sm;
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
    if (rc) {
        cudaFree(backup);
        return rc;
    }
    BATCH_TRY(b, cudaMemcpyAsync(backup, b->pool, pool_bytes, cudaMemcpyDeviceToDevice, b->stream));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // one step with the current choices: warm-up replay, then two timed replays
    auto trial = [&](float& ms) -> int {
        int r = apply_rows(b);
        if (!r) r = build_tiles(b);
        if (!r) r = capture(b, 1);
        if (r) return r;
        cudaGraphLaunch(b->graph, b->stream);
        cudaEventRecord(e0, b->stream);
        for (int i = 0; i < 2; ++i) cudaGraphLaunch(b->graph, b->stream);
        cudaEventRecord(e1, b->stream);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) return bfail(b, EFVM_ERR_CUDA, std::string("batch autotune: ") + cudaGetErrorString(e));
        cudaEventElapsedTime(&ms, e0, e1);
        return EFVM_OK;
    };
    for (int bucket = 0; bucket < N_BUCKETS && rc == EFVM_OK; ++bucket) {
        if (!(present & (1 << bucket))) continue;
        float best_ms = 1e30f;
        int best = ROW_CHOICES[0];
        for (int r : ROW_CHOICES) {
            b->bucket_rows[bucket] = r;
            float ms = 0.f;
            if ((rc = trial(ms))) break;
            if (ms < best_ms) {
                best_ms = ms;
                best = r;
            }
        }
        b->bucket_rows[bucket] = best;
    }
    if (b->persistent && rc == EFVM_OK) {
        const int form = batch_form_blocks(b->params.precision == EFVM_PREC_FP32_FLUX, b->ph.viscous != 0);
        float best_ms = 1e30f;
        int best = form;
        for (int blocks = form; blocks >= std::max(2, form - 3); --blocks) {
            b->blocks_per_sm = blocks;
            float ms = 0.f;
            if ((rc = trial(ms))) break;
            if (ms < best_ms) {
                best_ms = ms;
                best = blocks;
            }
        }
        b->blocks_per_sm = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaMemcpyAsync(b->pool, backup, pool_bytes, cudaMemcpyDeviceToDevice, b->stream);
    const int rc2 = write_states(b, saved);
    cudaFree(backup);
    if (rc) return rc;
    if (rc2) return rc2;
    int status = 0;
    BATCH_TRY(b, cudaMemcpy(&status, b->status_d, sizeof(int), cudaMemcpyDeviceToHost));
    if (status) return bfail(b, EFVM_ERR_TIMEOUT, "batch autotune: a wait of the persistent kernel ran out");
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache[key] = TuneChoice{b->bucket_rows, b->blocks_per_sm};
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
    if (cudaMalloc(&b->ready_d, n_cases * sizeof(unsigned int)) != cudaSuccess ||
        cudaMalloc(&b->done_d, n_cases * sizeof(unsigned int)) != cudaSuccess ||
        cudaMalloc(&b->case_tiles_d, n_cases * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->ticket_d, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&b->status_d, sizeof(int)) != cudaSuccess)
        return cleanup(bfail(nullptr, EFVM_ERR_OOM, "efvm_batch_create: cudaMalloc"));
    cudaMemsetAsync(b->status_d, 0, sizeof(int), b->stream);
    cudaDeviceGetAttribute(&b->n_sms, cudaDevAttrMultiProcessorCount, b->device);
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
    cudaFree(b->ready_d);
    cudaFree(b->done_d);
    cudaFree(b->case_tiles_d);
    cudaFree(b->ticket_d);
    cudaFree(b->status_d);
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
        const int stall = b->stall_case;  // an injected stall is for the run, not the tuning steps
        b->stall_case = -1;
        rc = tune(b);
        b->stall_case = stall;
        if (rc) return rc;
        b->tuned = true;
    }
    b->launches += launch_clock(b->clock_d, b->stream);
    rc = build_tiles(b);
    if (rc) return rc;
    // the persistent kernel runs a chunk of steps per replay; otherwise one step
    const int64_t per_replay_max = b->persistent ? chunk : 1;
    int64_t done = 0;
    bool recapture = true;
    while (done < max_steps) {
        const int64_t m = std::min<int64_t>(chunk, max_steps - done);
        const int steps = (int)std::min<int64_t>(m, per_replay_max);
        if (recapture || b->graph_steps != steps) {
            rc = capture(b, steps);
            if (rc) return rc;
            recapture = false;
        }
        for (int64_t i = 0; i < m / steps; ++i) {
            BATCH_TRY(b, cudaGraphLaunch(b->graph, b->stream));
            b->launches += launches_per_replay(b, steps);
        }
        done += (m / steps) * steps;
        rc = read_states(b, s);
        if (rc) return rc;
        if (b->persistent) {
            int status = 0;
            BATCH_TRY(b, cudaMemcpyAsync(&status, b->status_d, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
            BATCH_TRY(b, cudaStreamSynchronize(b->stream));
            if (status) {
                b->stall_case = -1;
                cudaMemsetAsync(b->status_d, 0, sizeof(int), b->stream);
                cudaStreamSynchronize(b->stream);
                return bfail(b, EFVM_ERR_TIMEOUT,
                             "a wait of the persistent batch kernel ran out; the cases' states are partly advanced");
            }
        }
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
            recapture = true;
        }
    }
    b->stall_case = -1;
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
        b->blocks_per_sm = 0;
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

int efvm_batch_set_persistent(efvm_batch* b, int32_t enable) {
    if (!b) return bfail(b, EFVM_ERR_INVALID_ARG, "null argument");
    b->persistent = enable != 0;
    b->tuned = false;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return EFVM_OK;
}

int efvm_batch_set_wait_limit(efvm_batch* b, double seconds) {
    if (!b || !(seconds > 0.0) || seconds > 60.0)
        return bfail(b, EFVM_ERR_INVALID_ARG, "efvm_batch_set_wait_limit: need 0 < seconds <= 60");
    b->wait_s = seconds;
    if (b->graph) {  // the limit is a kernel argument of the captured launch
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return EFVM_OK;
}

int efvm_batch_inject_stall(efvm_batch* b, int32_t k) {
    if (!b) return bfail(b, EFVM_ERR_INVALID_ARG, "null argument");
    if (k < 0 || k >= b->n) return bfail(b, EFVM_ERR_INVALID_ARG, "case index out of range");
    b->stall_case = k;
    return EFVM_OK;
}

int efvm_batch_get_blocks_per_sm(efvm_batch* b, int32_t* out) {
    if (!b || !out) return bfail(b, EFVM_ERR_INVALID_ARG, "null argument");
    *out = resident_blocks(b);
    return EFVM_OK;
}

int efvm_batch_get_stream(efvm_batch* b, void** stream) {
    if (!b || !stream) return bfail(b, EFVM_ERR_INVALID_ARG, "null argument");
    *stream = (void*)b->stream;
    return EFVM_OK;
}

}  // extern "C"
