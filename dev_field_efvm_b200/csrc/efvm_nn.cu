// efvm_nn.cu — BF16 tensor-core (tcgen05) kernels of the learned flux correction.
//
// This file holds the tensor-core GEMM tile that the correction network's
// forward and backward kernels are built from, and a stand-alone entry point
// that runs it on caller matrices (used to check the tile against a CPU
// product).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "efvm_internal.h"
#include "efvm_tc.cuh"

namespace efvm {
namespace {

__device__ int g_nn_error;  // set by a kernel whose tensor-core wait ran out

__host__ __device__ constexpr int tmem_cols_for(int n) { return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : 256; }

// D[M x N] = A[M x K] * B[N x K]^T, row-major BF16 inputs (K contiguous), FP32
// output; one CTA of 128 threads per 128 rows of A.
__global__ void __launch_bounds__(128) nn_gemm_kernel(const __nv_bfloat16* __restrict__ A,
                                                      const __nv_bfloat16* __restrict__ B, float* __restrict__ D,
                                                      int N, int K) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    unsigned char* sa = smem;
    unsigned char* sb = smem + 128 * K * 2;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long m0 = (long long)blockIdx.x * 128;
    for (int idx = tid; idx < 128 * K; idx += 128) {
        const int r = idx / K, k = idx - r * K;
        *reinterpret_cast<__nv_bfloat16*>(sa + tc::canon_offset(r, k, 128)) = A[(m0 + r) * K + k];
    }
    for (int idx = tid; idx < N * K; idx += 128) {
        const int r = idx / K, k = idx - r * K;
        *reinterpret_cast<__nv_bfloat16*>(sb + tc::canon_offset(r, k, N)) = B[(long long)r * K + k];
    }
    const uint32_t ncols = (uint32_t)tmem_cols_for(N);
    if (warp == 0) tc::tmem_alloc(&tslot, ncols);
    if (tid == 0) tc::mbar_init(&bar, 1);
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tslot;
    tc::gemm_issue(tmem, sa, sb, N, K, &bar);
    bool ok = tc::mbar_wait(&bar, 0);
    ok = __syncthreads_and(ok);
    if (!ok) {
        if (tid == 0) atomicExch(&g_nn_error, 1);
        tc::mbar_wait(&bar, 0);  // give the MMA a second bounded chance to retire before TMEM is released
    } else {
        tc::fence_after_sync();
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tmem, c0, v);
            float* out = D + (m0 + 32 * warp + lane) * N + c0;
#pragma unroll
            for (int i = 0; i < 16; ++i) out[i] = v[i];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tmem, ncols);
}


// ===========================================================================
// The correction network.  Per face, the 5 x 5 stencil of primitive variables
// (rho - 1, normal velocity, tangential velocity, p - 1) in the face's own
// frame (x faces as they are; y faces transposed with u and v swapped, so one
// network serves both orientations) feeds
//     h1 = relu(W1 x + b1)   (100 -> 32, K padded to 112)
//     h2 = relu(W2 h1 + b2)  (32 -> 32)
//     y  = W3 h2 + b3        (32 -> 4, N padded to 16)
// and out_scale * y is the correction (rho, m_n, m_t, E) added to that face's
// flux.  Weights are BF16 on the tensor cores, biases and accumulation FP32.
// One CTA of 128 threads handles 128 faces; thread r owns face r of the tile.
// ===========================================================================
namespace nn {

constexpr int IN = 100, K1 = 112, H = 32, NOUT = 4, N3 = 16;
constexpr int P_W1 = 0, P_W2 = P_W1 + H * K1, P_W3 = P_W2 + H * H, P_B1 = P_W3 + NOUT * H, P_B2 = P_B1 + H,
              P_B3 = P_B2 + H, P_COUNT = P_B3 + NOUT;

struct Net {
    const __nv_bfloat16* w1;  // [H][K1], columns >= IN zero
    const __nv_bfloat16* w2;  // [H][H]
    const __nv_bfloat16* w3;  // [N3][H], rows >= NOUT zero
    const float* p;           // FP32 parameters (the biases are read here)
    float out_scale;
    float gamma;
};

// Periodic index for -n <= i < 2n.  Every caller is within 3 cells of the
// grid (the 5x5 stencil, the residual's neighbours) and every entry point
// requires nx, ny >= 5, so one conditional wrap replaces an integer modulo
// (whose division sequence would run per stencil cell).
__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// Conserved states [B][4][n][n] (FP64, periodic), as the training batches hold them.
struct PackedStates {
    const double* q;
    int nx, ny;
    __device__ double get(int b, int v, int i, int j) const {
        i = wrap(i, nx);
        j = wrap(j, ny);
        return q[(((long long)b * 4 + v) * ny + j) * nx + i];
    }
};
// One context state buffer (periodic in x and y), read by interior index.
struct PaddedState {
    const double* q;
    long long plane;
    int pitch, nx, ny;
    __device__ double get(int, int v, int i, int j) const {
        i = wrap(i, nx);
        j = wrap(j, ny);
        return q[(long long)v * plane + (long long)(YO + j) * pitch + XO + i];
    }
};

// Shared-memory plan of one tile (byte offsets; every operand 128-byte aligned).
constexpr int SM_X = 0;                       // [128][K1]   A of layer 1
constexpr int SM_XT = SM_X + 128 * K1 * 2;    // [K1][128]   B of dW1
constexpr int SM_W1 = SM_XT + K1 * 128 * 2;   // [H][K1]
constexpr int SM_W2 = SM_W1 + H * K1 * 2;     // [H][H]
constexpr int SM_W3 = SM_W2 + H * H * 2;      // [N3][H]
constexpr int SM_W2T = SM_W3 + N3 * H * 2;    // [H][H]      W2 transposed
constexpr int SM_W3T = SM_W2T + H * H * 2;    // [H][N3]     W3 transposed
constexpr int SM_H1 = SM_W3T + H * N3 * 2;    // [128][H]
constexpr int SM_H2 = SM_H1 + 128 * H * 2;    // [128][H]
constexpr int SM_H1T = SM_H2 + 128 * H * 2;   // [H][128]
constexpr int SM_H2T = SM_H1T + H * 128 * 2;  // [H][128]
constexpr int SM_DY = SM_H2T + H * 128 * 2;   // [128][N3]   output gradient
constexpr int SM_DZ = SM_DY + 128 * N3 * 2;   // [128][H]    dZ2, A of dH1
constexpr int SM_AT = SM_DZ + 128 * H * 2;    // [128][128]  transposed gradient, A of the weight gradients
constexpr int SM_RED = SM_AT + 128 * 128 * 2; // [4][K1] floats: per-warp column sums
constexpr int SM_TOTAL = SM_RED + 4 * K1 * 4;
constexpr int SM_FWD = SM_H2 + 128 * H * 2;   // the forward pass needs the buffers up to H2

__device__ __forceinline__ void put(unsigned char* base, int r, int k, int rows, float v) {
    *reinterpret_cast<__nv_bfloat16*>(base + tc::canon_offset(r, k, rows)) = __float2bfloat16_rn(v);
}
__device__ __forceinline__ float get_bf(const unsigned char* base, int r, int k, int rows) {
    return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(base + tc::canon_offset(r, k, rows)));
}

struct FaceId {
    int b, orient, i, j;
};
__device__ __forceinline__ FaceId face_of(long long f, int nx, int ny) {
    const long long per = 2LL * nx * ny;
    FaceId id;
    if (f < 0x7fffffffLL && per < 0x7fffffffLL) {  // the same quotients in 32-bit arithmetic
        const unsigned uf = (unsigned)f, up = (unsigned)per, un = (unsigned)nx * (unsigned)ny;
        id.b = (int)(uf / up);
        unsigned rem = uf - (unsigned)id.b * up;
        id.orient = (int)(rem / un);
        rem -= (unsigned)id.orient * un;
        id.j = (int)(rem / (unsigned)nx);
        id.i = (int)(rem - (unsigned)id.j * (unsigned)nx);
        return id;
    }
    id.b = (int)(f / per);
    long long rem = f - (long long)id.b * per;
    id.orient = (int)(rem / ((long long)nx * ny));
    rem -= (long long)id.orient * nx * ny;
    id.j = (int)(rem / nx);
    id.i = (int)(rem - (long long)id.j * nx);
    return id;
}

// Primitive (rho, u, v, p) of a stencil cell.
template <class SV>
__device__ __forceinline__ void prim_at(const SV& sv, int b, int i, int j, float gamma, float (&w)[4]) {
    const double r = sv.get(b, 0, i, j), mx = sv.get(b, 1, i, j), my = sv.get(b, 2, i, j), E = sv.get(b, 3, i, j);
    const double u = mx / r, v = my / r;
    const double p = (gamma - 1.0) * (E - 0.5 * r * (u * u + v * v));
    w[0] = (float)r;
    w[1] = (float)u;
    w[2] = (float)v;
    w[3] = (float)p;
}

// The network's per-cell inputs (rho - 1, u, v, p - 1) in FP32, computed once
// per cell by nn_prims_kernel; each cell feeds 50 face stencils.
struct PrimView {
    const float4* p;
    int nx, ny;
    __device__ float4 get(int b, int i, int j) const {
        i = wrap(i, nx);
        j = wrap(j, ny);
        return p[((long long)b * ny + j) * nx + i];
    }
};

template <class SV>
__global__ void nn_prims_kernel(SV sv, int batch, float gamma, float4* __restrict__ out) {
    const long long n = (long long)sv.nx * sv.ny, total = (long long)batch * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / n);
        const long long c = t - (long long)b * n;
        const int j = (int)(c / sv.nx), i = (int)(c - (long long)j * sv.nx);
        float w[4];
        prim_at(sv, b, i, j, gamma, w);
        out[t] = make_float4(w[0] - 1.0f, w[1], w[2], w[3] - 1.0f);
    }
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// The stencil features of face `id`, written as row r of X with one 16-byte
// store per two stencil cells (8 consecutive K in the canonical layout), and
// into X^T (element by element) when xt != null.  Feature 4q + v is variable v
// (rho - 1, normal velocity, tangential velocity, p - 1) of stencil cell
// q = (c + 2) * 5 + (a + 3), a the offset along the face normal (-3..1), c across.
__device__ void gather_face(const PrimView& pv, const FaceId& id, unsigned char* x, unsigned char* xt, int r) {
#pragma unroll 7
    for (int m = 0; m < K1 / 8; ++m) {
        float f[8];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int q = 2 * m + h;
            if (q < 25) {
                const int c = q / 5 - 2, a = q % 5 - 3;
                const int ci = id.orient == 0 ? id.i + a : id.i + c;
                const int cj = id.orient == 0 ? id.j + c : id.j + a;
                const float4 w = pv.get(id.b, ci, cj);
                f[4 * h + 0] = w.x;
                f[4 * h + 1] = id.orient == 0 ? w.y : w.z;
                f[4 * h + 2] = id.orient == 0 ? w.z : w.y;
                f[4 * h + 3] = w.w;
            } else {
                f[4 * h + 0] = f[4 * h + 1] = f[4 * h + 2] = f[4 * h + 3] = 0.f;
            }
        }
        const uint4 v = make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]),
                                   pack_bf16x2(f[6], f[7]));
        *reinterpret_cast<uint4*>(x + tc::canon_offset(r, 8 * m, 128)) = v;
        if (xt)
#pragma unroll
            for (int e = 0; e < 8; ++e) put(xt, 8 * m + e, r, K1, f[e]);
    }
}

// Weights into shared memory, 16 bytes (8 consecutive K of one row) per copy,
// and their transposes for the backward pass element by element.
__device__ void load_weights(const Net& net, unsigned char* sm, bool transposed) {
    const uint4* w1 = reinterpret_cast<const uint4*>(net.w1);
    for (int t = threadIdx.x; t < H * K1 / 8; t += blockDim.x) {
        const int o = t / (K1 / 8), g = t - o * (K1 / 8);
        *reinterpret_cast<uint4*>(sm + SM_W1 + tc::canon_offset(o, 8 * g, H)) = w1[t];
    }
    const uint4* w2 = reinterpret_cast<const uint4*>(net.w2);
    for (int t = threadIdx.x; t < H * H / 8; t += blockDim.x) {
        const int o = t / (H / 8), g = t - o * (H / 8);
        *reinterpret_cast<uint4*>(sm + SM_W2 + tc::canon_offset(o, 8 * g, H)) = w2[t];
    }
    const uint4* w3 = reinterpret_cast<const uint4*>(net.w3);
    for (int t = threadIdx.x; t < N3 * H / 8; t += blockDim.x) {
        const int o = t / (H / 8), g = t - o * (H / 8);
        *reinterpret_cast<uint4*>(sm + SM_W3 + tc::canon_offset(o, 8 * g, N3)) = w3[t];
    }
    if (transposed) {
        for (int t = threadIdx.x; t < H * H; t += blockDim.x) {
            const int o = t / H, k = t - o * H;
            *reinterpret_cast<__nv_bfloat16*>(sm + SM_W2T + tc::canon_offset(k, o, H)) = net.w2[t];
        }
        for (int t = threadIdx.x; t < N3 * H; t += blockDim.x) {
            const int o = t / H, k = t - o * H;
            *reinterpret_cast<__nv_bfloat16*>(sm + SM_W3T + tc::canon_offset(k, o, H)) = net.w3[t];
        }
    }
}

// Tensor-core state of a tile: TMEM columns, the mbarrier and its phase.
struct TC {
    uint64_t* bar;
    uint32_t tmem;
    uint32_t phase;
    bool ok;
};

// Issue D = A B^T, wait for it (bounded) and make TMEM readable; false if the
// wait ran out anywhere in the CTA.
__device__ bool run_gemm(TC& t, const unsigned char* a, const unsigned char* b, int n, int k) {
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::gemm_issue(t.tmem, a, b, n, k, t.bar);
    bool ok = tc::mbar_wait(t.bar, t.phase);
    ok = __syncthreads_and(ok);
    t.phase ^= 1u;
    if (!ok) {
        if (threadIdx.x == 0) atomicExch(&g_nn_error, 1);
        tc::mbar_wait(t.bar, t.phase ^ 1u);  // a second bounded chance to retire before TMEM is released
        t.ok = false;
        return false;
    }
    tc::fence_after_sync();
    return true;
}

// Row r's 32 accumulator columns + bias, through relu, into A (row r) and, if
// given, its transpose.  Returns nothing; the caller barriers before reuse.
__device__ void relu_epilogue(uint32_t tmem, const float* bias, unsigned char* out, unsigned char* out_t, int r) {
#pragma unroll
    for (int c0 = 0; c0 < H; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tmem, c0, v);
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = fmaxf(v[c] + bias[c0 + c], 0.f);
#pragma unroll
        for (int g = 0; g < 2; ++g)
            *reinterpret_cast<uint4*>(out + tc::canon_offset(r, c0 + 8 * g, 128)) =
                make_uint4(pack_bf16x2(v[8 * g], v[8 * g + 1]), pack_bf16x2(v[8 * g + 2], v[8 * g + 3]),
                           pack_bf16x2(v[8 * g + 4], v[8 * g + 5]), pack_bf16x2(v[8 * g + 6], v[8 * g + 7]));
        if (out_t)
#pragma unroll
            for (int c = 0; c < 16; ++c) put(out_t, c0 + c, r, H, v[c]);
    }
}

// Forward pass of one tile through layer 2 (H1, H2 in shared memory).
__device__ bool forward_hidden(const PrimView& pv, const Net& net, unsigned char* sm, TC& t, long long f0,
                               bool keep_transposes) {
    const int r = threadIdx.x;
    const FaceId id = face_of(f0 + r, pv.nx, pv.ny);
    gather_face(pv, id, sm + SM_X, keep_transposes ? sm + SM_XT : nullptr, r);
    load_weights(net, sm, keep_transposes);
    if (!run_gemm(t, sm + SM_X, sm + SM_W1, H, K1)) return false;
    relu_epilogue(t.tmem, net.p + P_B1, sm + SM_H1, keep_transposes ? sm + SM_H1T : nullptr, r);
    if (!run_gemm(t, sm + SM_H1, sm + SM_W2, H, H)) return false;
    relu_epilogue(t.tmem, net.p + P_B2, sm + SM_H2, keep_transposes ? sm + SM_H2T : nullptr, r);
    return true;
}

__device__ void tile_setup(TC& t, uint64_t* bar, uint32_t* slot) {
    if ((threadIdx.x >> 5) == 0) tc::tmem_alloc(slot, 128);
    if (threadIdx.x == 0) tc::mbar_init(bar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    t.bar = bar;
    t.tmem = *slot;
    t.phase = 0;
    t.ok = true;
}
__device__ void tile_teardown(const TC& t) {
    tc::fence_before_sync();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) tc::tmem_free(t.tmem, 128);
}

// Forward: the correction of every face, grid frame, corr[((b*2+orient)*4+v)*ny*nx + j*nx + i].
// sensor > 0 (inference): a face whose two cells differ in pressure by more than
// sensor * min(p), or where rho or p is not positive, keeps the plain flux.
__global__ void __launch_bounds__(128) nn_forward_kernel(PrimView pv, Net net, float* __restrict__ corr, float sensor,
                                                         unsigned long long* fallbacks) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t slot;
    TC t;
    tile_setup(t, &bar, &slot);
    const long long f0 = (long long)blockIdx.x * 128;
    const int r = threadIdx.x;
    if (forward_hidden(pv, net, sm, t, f0, false) && run_gemm(t, sm + SM_H2, sm + SM_W3, N3, H)) {
        float v[16];
        tc::tmem_ld16(t.tmem, 0, v);
        const FaceId id = face_of(f0 + r, pv.nx, pv.ny);
        float y[4];
#pragma unroll
        for (int o = 0; o < 4; ++o) y[o] = (v[o] + net.p[P_B3 + o]) * net.out_scale;
        if (sensor > 0.f) {
            const int il = id.orient == 0 ? id.i - 1 : id.i, jl = id.orient == 0 ? id.j : id.j - 1;
            const float4 ql = pv.get(id.b, il, jl), qr = pv.get(id.b, id.i, id.j);
            const float rl = ql.x + 1.0f, rr = qr.x + 1.0f, pl = ql.w + 1.0f, pr = qr.w + 1.0f;
            const bool fire = !(rl > 0.f && rr > 0.f && pl > 0.f && pr > 0.f) ||
                              fabsf(pr - pl) > sensor * fminf(pl, pr);
            if (fire) {
                y[0] = y[1] = y[2] = y[3] = 0.f;
                atomicAdd(fallbacks, 1ull);
            }
        }
        // face frame (rho, m_n, m_t, E) -> grid frame (rho, m_x, m_y, E)
        const float g[4] = {y[0], id.orient == 0 ? y[1] : y[2], id.orient == 0 ? y[2] : y[1], y[3]};
        const long long cell = (long long)id.j * pv.nx + id.i, nn = (long long)pv.nx * pv.ny;
#pragma unroll
        for (int q = 0; q < 4; ++q) corr[((long long)(id.b * 2 + id.orient) * 4 + q) * nn + cell] = g[q];
    }
    tile_teardown(t);
}

// Column sums of per-thread rows: each warp reduces its 32 rows by shuffles,
// then thread c adds the four warp sums in order (deterministic).
__device__ void column_sums(const float* vals, int ncols, float* red, float* out) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = 0; c < ncols; ++c) {
        float s = vals[c];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[w * K1 + c] = s;
    }
    __syncthreads();
    if ((int)threadIdx.x < ncols) out[threadIdx.x] = red[threadIdx.x] + red[K1 + threadIdx.x] + red[2 * K1 + threadIdx.x] + red[3 * K1 + threadIdx.x];
    __syncthreads();
}

// Rows 0..rows-1 of the accumulator (warp 0's lanes), ncols columns, to out[row * ncols + col].
__device__ void store_weight_grad(uint32_t tmem, int rows, int ncols, float* out) {
    if ((threadIdx.x >> 5) != 0) return;  // warp-uniform: rows < 32 live in warp 0's lanes
    const int lane = threadIdx.x & 31;
    for (int c0 = 0; c0 < ncols; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tmem, c0, v);
        if (lane < rows)
#pragma unroll
            for (int c = 0; c < 16; ++c)
                if (c0 + c < ncols) out[lane * ncols + c0 + c] = v[c];
    }
}

// Backward: given dL/dcorr (grid frame, the layout of corr), the gradient of the
// loss with respect to every parameter, summed over this tile's 128 faces, into
// partials[tile][P_COUNT].
__global__ void __launch_bounds__(128) nn_backward_kernel(PrimView sv, Net net, const float* __restrict__ dcorr,
                                                          float* __restrict__ partials) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t slot;
    TC t;
    tile_setup(t, &bar, &slot);
    const long long f0 = (long long)blockIdx.x * 128;
    const int r = threadIdx.x;
    float* part = partials + (long long)blockIdx.x * P_COUNT;
    float* red = reinterpret_cast<float*>(sm + SM_RED);
    // the transposed-gradient operand: rows beyond the layer width stay zero
    for (int q = threadIdx.x; q < 128 * 128 * 2 / 16; q += blockDim.x)
        reinterpret_cast<uint4*>(sm + SM_AT)[q] = make_uint4(0, 0, 0, 0);
    do {
        if (!forward_hidden(sv, net, sm, t, f0, true)) break;
        // output gradient of this face in its own frame, times out_scale
        const FaceId id = face_of(f0 + r, sv.nx, sv.ny);
        const long long cell = (long long)id.j * sv.nx + id.i, nn = (long long)sv.nx * sv.ny;
        float g[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) g[q] = dcorr[((long long)(id.b * 2 + id.orient) * 4 + q) * nn + cell];
        const float dy[4] = {g[0] * net.out_scale, (id.orient == 0 ? g[1] : g[2]) * net.out_scale,
                             (id.orient == 0 ? g[2] : g[1]) * net.out_scale, g[3] * net.out_scale};
        float dyrow[N3];
#pragma unroll
        for (int o = 0; o < N3; ++o) dyrow[o] = o < NOUT ? __bfloat162float(__float2bfloat16_rn(dy[o])) : 0.f;
#pragma unroll
        for (int g = 0; g < 2; ++g)
            *reinterpret_cast<uint4*>(sm + SM_DY + tc::canon_offset(r, 8 * g, 128)) =
                make_uint4(pack_bf16x2(dyrow[8 * g], dyrow[8 * g + 1]), pack_bf16x2(dyrow[8 * g + 2], dyrow[8 * g + 3]),
                           pack_bf16x2(dyrow[8 * g + 4], dyrow[8 * g + 5]), pack_bf16x2(dyrow[8 * g + 6], dyrow[8 * g + 7]));
#pragma unroll
        for (int o = 0; o < NOUT; ++o) put(sm + SM_AT, o, r, 128, dyrow[o]);
        column_sums(dyrow, NOUT, red, part + P_B3);
        // dW3 = dY^T H2
        if (!run_gemm(t, sm + SM_AT, sm + SM_H2T, H, 128)) break;
        store_weight_grad(t.tmem, NOUT, H, part + P_W3);
        // dH2 = dY W3, dZ2 = dH2 * relu'(h2)
        if (!run_gemm(t, sm + SM_DY, sm + SM_W3T, H, N3)) break;
        {
            float dz[H];
#pragma unroll
            for (int c0 = 0; c0 < H; c0 += 16) {
                float v[16];
                tc::tmem_ld16(t.tmem, c0, v);
#pragma unroll
                for (int c = 0; c < 16; ++c) {
                    const float z = get_bf(sm + SM_H2, r, c0 + c, 128) > 0.f ? v[c] : 0.f;
                    dz[c0 + c] = __bfloat162float(__float2bfloat16_rn(z));
                }
            }
#pragma unroll
            for (int g = 0; g < H / 8; ++g)
                *reinterpret_cast<uint4*>(sm + SM_DZ + tc::canon_offset(r, 8 * g, 128)) =
                    make_uint4(pack_bf16x2(dz[8 * g], dz[8 * g + 1]), pack_bf16x2(dz[8 * g + 2], dz[8 * g + 3]),
                               pack_bf16x2(dz[8 * g + 4], dz[8 * g + 5]), pack_bf16x2(dz[8 * g + 6], dz[8 * g + 7]));
#pragma unroll
            for (int c = 0; c < H; ++c) put(sm + SM_AT, c, r, 128, dz[c]);
            column_sums(dz, H, red, part + P_B2);
        }
        // dW2 = dZ2^T H1
        if (!run_gemm(t, sm + SM_AT, sm + SM_H1T, H, 128)) break;
        store_weight_grad(t.tmem, H, H, part + P_W2);
        // dH1 = dZ2 W2, dZ1 = dH1 * relu'(h1)
        if (!run_gemm(t, sm + SM_DZ, sm + SM_W2T, H, H)) break;
        {
            float dz[H];
#pragma unroll
            for (int c0 = 0; c0 < H; c0 += 16) {
                float v[16];
                tc::tmem_ld16(t.tmem, c0, v);
#pragma unroll
                for (int c = 0; c < 16; ++c) {
                    const float z = get_bf(sm + SM_H1, r, c0 + c, 128) > 0.f ? v[c] : 0.f;
                    dz[c0 + c] = __bfloat162float(__float2bfloat16_rn(z));
                }
            }
            __syncthreads();  // the previous GEMM has read A^T; now overwrite it
#pragma unroll
            for (int c = 0; c < H; ++c) put(sm + SM_AT, c, r, 128, dz[c]);
            column_sums(dz, H, red, part + P_B1);
        }
        // dW1 = dZ1^T X
        if (!run_gemm(t, sm + SM_AT, sm + SM_XT, K1, 128)) break;
        store_weight_grad(t.tmem, H, K1, part + P_W1);
    } while (0);
    tile_teardown(t);
}

// grad[p] = sum over tiles of partials[tile][p], in tile order.
__global__ void nn_reduce_kernel(const float* __restrict__ partials, int tiles, float* __restrict__ grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P_COUNT) return;
    float s = 0.f;
    for (int t = 0; t < tiles; ++t) s += partials[(long long)t * P_COUNT + p];
    grad[p] = s;
}

// Residual loss of a batch: e = R + div(corr) per cell and variable,
// L = sum_v w_v * mean(e_v^2); dcorr = dL/dcorr.  One thread per cell.
__global__ void nn_residual_kernel(const float* __restrict__ corr, const double* __restrict__ resid, int batch, int nx,
                                   int ny, double inv_dx, double inv_dy, float w0, float w1, float w2, float w3,
                                   float* __restrict__ dcorr, double* loss) {
    const long long n = (long long)nx * ny, total = (long long)batch * n;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (t < total) {
        const int b = (int)(t / n);
        const long long cell = t - (long long)b * n;
        const int j = (int)(cell / nx), i = (int)(cell - (long long)j * nx);
        auto cx = [&](int v, int ii, int jj) {  // x-face correction on the left of cell (ii, jj)
            ii = wrap(ii, nx);
            jj = wrap(jj, ny);
            return (double)corr[((long long)(b * 2 + 0) * 4 + v) * n + (long long)jj * nx + ii];
        };
        auto cy = [&](int v, int ii, int jj) {
            ii = wrap(ii, nx);
            jj = wrap(jj, ny);
            return (double)corr[((long long)(b * 2 + 1) * 4 + v) * n + (long long)jj * nx + ii];
        };
        auto err = [&](int v, int ii, int jj) {
            const int i2 = wrap(ii, nx), j2 = wrap(jj, ny);
            const double div = (cx(v, ii + 1, jj) - cx(v, ii, jj)) * inv_dx + (cy(v, ii, jj + 1) - cy(v, ii, jj)) * inv_dy;
            return resid[((long long)b * 4 + v) * n + (long long)j2 * nx + i2] + div;
        };
        const float w[4] = {w0, w1, w2, w3};
        const double scale = 2.0 / (double)total;
        for (int v = 0; v < 4; ++v) {
            const double e = err(v, i, j);
            l += w[v] * e * e;
            // x face on the left of (i, j): +1/dx in cell (i-1, j), -1/dx in cell (i, j)
            const double gx = scale * w[v] * (err(v, i - 1, j) - e) * inv_dx;
            const double gy = scale * w[v] * (err(v, i, j - 1) - e) * inv_dy;
            dcorr[((long long)(b * 2 + 0) * 4 + v) * n + cell] = (float)gx;
            dcorr[((long long)(b * 2 + 1) * 4 + v) * n + cell] = (float)gy;
        }
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.0) atomicAdd(loss, l / (double)total);
}

// Adam on the FP32 parameters, then the BF16 copies the tensor cores read.
__global__ void nn_adam_kernel(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                               const float* __restrict__ g, float lr, float b1t, float b2t,
                               __nv_bfloat16* w1, __nv_bfloat16* w2, __nv_bfloat16* w3) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P_COUNT) return;
    const bool pad = q < P_W2 && (q - P_W1) % K1 >= IN;  // W1 columns beyond the 100 inputs stay zero
    if (!pad) {
        const float gq = g[q];
        const float mq = 0.9f * m[q] + 0.1f * gq;
        const float vq = 0.999f * v[q] + 0.001f * gq * gq;
        m[q] = mq;
        v[q] = vq;
        const float mh = mq / (1.f - b1t), vh = vq / (1.f - b2t);
        p[q] -= lr * mh / (sqrtf(vh) + 1e-8f);
    }
    if (q < P_W2) w1[q - P_W1] = __float2bfloat16_rn(pad ? 0.f : p[q]);
    else if (q < P_W3) w2[q - P_W2] = __float2bfloat16_rn(p[q]);
    else if (q < P_B1) w3[q - P_W3] = __float2bfloat16_rn(p[q]);  // rows 0..NOUT-1 of [N3][H]
}

}  // namespace nn
}  // namespace
}  // namespace efvm

using namespace efvm;

// ---- the network object ------------------------------------------------------
struct efvm_nn {
    float *p = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr;
    __nv_bfloat16 *w1 = nullptr, *w2 = nullptr, *w3 = nullptr;
    float out_scale = 1e-3f, gamma = 1.4f;
    int64_t steps = 0;
    float* partials = nullptr;
    size_t partials_cap = 0;
    float *corr = nullptr, *dcorr = nullptr;
    size_t corr_cap = 0;
    float4* prims = nullptr;
    size_t prims_cap = 0;
    double* loss_d = nullptr;
    std::string err;
};

namespace efvm {
nn::Net nn_net(const efvm_nn* h) {
    nn::Net n;
    n.w1 = h->w1;
    n.w2 = h->w2;
    n.w3 = h->w3;
    n.p = h->p;
    n.out_scale = h->out_scale;
    n.gamma = h->gamma;
    return n;
}

int nn_forward_padded(const efvm_nn* h, const double* q, long long plane, int pitch, int nx, int ny, float* corr,
                      float4* prims, float sensor, unsigned long long* fallbacks, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    nn::PaddedState sv{q, plane, pitch, nx, ny};
    nn::nn_prims_kernel<nn::PaddedState><<<(nx * ny + 255) / 256, 256, 0, s>>>(sv, 1, h->gamma, prims);
    const int tiles = (int)(2LL * nx * ny / 128);
    nn::nn_forward_kernel<<<tiles, 128, nn::SM_FWD, s>>>(nn::PrimView{prims, nx, ny}, nn_net(h), corr, sensor,
                                                          fallbacks);
    return 2;
}

int nn_prepare_launches() {
    cudaError_t e = cudaFuncSetAttribute(nn::nn_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, nn::SM_FWD);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(nn::nn_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, nn::SM_TOTAL);
    return e == cudaSuccess ? EFVM_OK : EFVM_ERR_CUDA;
}
}  // namespace efvm

namespace {

int nfail(efvm_nn* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    set_global_error(msg);
    return code;
}

#define NN_TRY(h, call)                                                                                     \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) return nfail(h, EFVM_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

// splitmix64 and a Box-Muller normal, for the seeded initial weights
uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double normal(uint64_t& s) {
    const double u1 = ((splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    const double u2 = ((splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

// Upload FP32 parameters and refresh the BF16 copies (an Adam step with lr = 0
// and a zero gradient leaves p unchanged and rewrites the copies).
int upload_params(efvm_nn* h, const float* host, cudaStream_t s) {
    NN_TRY(h, cudaMemcpyAsync(h->p, host, nn::P_COUNT * sizeof(float), cudaMemcpyHostToDevice, s));
    NN_TRY(h, cudaMemsetAsync(h->grad, 0, nn::P_COUNT * sizeof(float), s));
    nn::nn_adam_kernel<<<(nn::P_COUNT + 255) / 256, 256, 0, s>>>(h->p, h->m, h->v, h->grad, 0.f, 0.5f, 0.5f, h->w1,
                                                                 h->w2, h->w3);
    NN_TRY(h, cudaGetLastError());
    NN_TRY(h, cudaStreamSynchronize(s));
    return EFVM_OK;
}

int check_shape(efvm_nn* h, int batch, int nx, int ny) {
    if (batch < 1 || nx < 5 || ny < 5 || ((long long)nx * ny) % 64)
        return nfail(h, EFVM_ERR_INVALID_ARG, "the network needs batch >= 1, nx, ny >= 5 and nx*ny a multiple of 64");
    return EFVM_OK;
}

int ensure_buffers(efvm_nn* h, int batch, int nx, int ny) {
    const size_t faces = 2ull * batch * nx * ny, tiles = faces / 128;
    if (tiles * nn::P_COUNT > h->partials_cap) {
        cudaFree(h->partials);
        h->partials = nullptr;
        h->partials_cap = 0;
        NN_TRY(h, cudaMalloc(&h->partials, tiles * nn::P_COUNT * sizeof(float)));
        h->partials_cap = tiles * nn::P_COUNT;
    }
    if ((size_t)batch * nx * ny > h->prims_cap) {
        cudaFree(h->prims);
        h->prims = nullptr;
        h->prims_cap = 0;
        NN_TRY(h, cudaMalloc(&h->prims, (size_t)batch * nx * ny * sizeof(float4)));
        h->prims_cap = (size_t)batch * nx * ny;
    }
    if (faces * 4 > h->corr_cap) {
        cudaFree(h->corr);
        cudaFree(h->dcorr);
        h->corr = h->dcorr = nullptr;
        h->corr_cap = 0;
        NN_TRY(h, cudaMalloc(&h->corr, faces * 4 * sizeof(float)));
        NN_TRY(h, cudaMalloc(&h->dcorr, faces * 4 * sizeof(float)));
        h->corr_cap = faces * 4;
    }
    return EFVM_OK;
}

int tc_status(efvm_nn* h) {
    int err = 0;
    NN_TRY(h, cudaMemcpyFromSymbol(&err, g_nn_error, sizeof(int)));
    if (err) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_nn_error, &zero, sizeof(int));
        return nfail(h, EFVM_ERR_TIMEOUT, "a tensor-core completion wait ran out");
    }
    return EFVM_OK;
}

}  // namespace

extern "C" {

int efvm_nn_param_count(void) { return nn::P_COUNT; }

int efvm_nn_create(float out_scale, float gamma, uint64_t seed, efvm_nn** out) {
    if (!out || !(out_scale > 0.f) || !(gamma > 1.f)) return nfail(nullptr, EFVM_ERR_INVALID_ARG, "efvm_nn_create: invalid argument");
    *out = nullptr;
    efvm_nn* h = new efvm_nn();
    h->out_scale = out_scale;
    h->gamma = gamma;
    auto bad = [&](int code) {
        efvm_nn_destroy(h);
        return code;
    };
    const size_t pb = nn::P_COUNT * sizeof(float);
    if (cudaMalloc(&h->p, pb) || cudaMalloc(&h->m, pb) || cudaMalloc(&h->v, pb) || cudaMalloc(&h->grad, pb) ||
        cudaMalloc(&h->w1, nn::H * nn::K1 * 2) || cudaMalloc(&h->w2, nn::H * nn::H * 2) ||
        cudaMalloc(&h->w3, nn::N3 * nn::H * 2) || cudaMalloc(&h->loss_d, sizeof(double)))
        return bad(nfail(nullptr, EFVM_ERR_OOM, "efvm_nn_create: cudaMalloc"));
    cudaMemset(h->m, 0, pb);
    cudaMemset(h->v, 0, pb);
    cudaMemset(h->w3, 0, nn::N3 * nn::H * 2);  // rows >= NOUT stay zero
    if (nn_prepare_launches()) return bad(nfail(nullptr, EFVM_ERR_CUDA, "efvm_nn_create: kernel attributes"));
    // He-normal hidden layers, a small output layer (the initial correction is near zero), zero biases
    std::vector<float> p(nn::P_COUNT, 0.f);
    uint64_t s = seed;
    for (int o = 0; o < nn::H; ++o)
        for (int k = 0; k < nn::IN; ++k) p[nn::P_W1 + o * nn::K1 + k] = (float)(normal(s) * std::sqrt(2.0 / nn::IN));
    for (int q = 0; q < nn::H * nn::H; ++q) p[nn::P_W2 + q] = (float)(normal(s) * std::sqrt(2.0 / nn::H));
    for (int q = 0; q < nn::NOUT * nn::H; ++q) p[nn::P_W3 + q] = (float)(normal(s) * 0.01);
    const int rc = upload_params(h, p.data(), 0);
    if (rc) return bad(rc);
    *out = h;
    return EFVM_OK;
}

int efvm_nn_destroy(efvm_nn* h) {
    if (!h) return EFVM_OK;
    cudaFree(h->p);
    cudaFree(h->m);
    cudaFree(h->v);
    cudaFree(h->grad);
    cudaFree(h->w1);
    cudaFree(h->w2);
    cudaFree(h->w3);
    cudaFree(h->partials);
    cudaFree(h->corr);
    cudaFree(h->dcorr);
    cudaFree(h->prims);
    cudaFree(h->loss_d);
    delete h;
    return EFVM_OK;
}

int efvm_nn_get_params(efvm_nn* h, float* host) {
    if (!h || !host) return nfail(h, EFVM_ERR_INVALID_ARG, "null argument");
    NN_TRY(h, cudaMemcpy(host, h->p, nn::P_COUNT * sizeof(float), cudaMemcpyDeviceToHost));
    return EFVM_OK;
}

int efvm_nn_set_params(efvm_nn* h, const float* host) {
    if (!h || !host) return nfail(h, EFVM_ERR_INVALID_ARG, "null argument");
    return upload_params(h, host, 0);
}

int efvm_nn_get_scale(efvm_nn* h, float* out_scale) {
    if (!h || !out_scale) return nfail(h, EFVM_ERR_INVALID_ARG, "null argument");
    *out_scale = h->out_scale;
    return EFVM_OK;
}

int efvm_nn_forward(efvm_nn* h, const double* states, int32_t batch, int32_t nx, int32_t ny, float* corr,
                    void* stream) {
    if (!h || !states || !corr) return nfail(h, EFVM_ERR_INVALID_ARG, "null argument");
    int rc = check_shape(h, batch, nx, ny);
    if (rc) return rc;
    rc = ensure_buffers(h, batch, nx, ny);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    nn::PackedStates sv{states, nx, ny};
    const long long cells = (long long)batch * nx * ny;
    nn::nn_prims_kernel<nn::PackedStates><<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(sv, batch, h->gamma, h->prims);
    const int tiles = (int)(2LL * batch * nx * ny / 128);
    nn::nn_forward_kernel<<<tiles, 128, nn::SM_FWD, s>>>(nn::PrimView{h->prims, nx, ny}, nn_net(h), corr, 0.f, nullptr);
    NN_TRY(h, cudaGetLastError());
    NN_TRY(h, cudaStreamSynchronize(s));
    return tc_status(h);
}

int efvm_nn_loss_grad(efvm_nn* h, const double* states, const double* resid, int32_t batch, int32_t nx, int32_t ny,
                      double dx, double dy, const float w[4], float* grad_out, double* loss, void* stream) {
    if (!h || !states || !resid || !w) return nfail(h, EFVM_ERR_INVALID_ARG, "null argument");
    int rc = check_shape(h, batch, nx, ny);
    if (rc) return rc;
    rc = ensure_buffers(h, batch, nx, ny);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    nn::PackedStates sv{states, nx, ny};
    const long long cells = (long long)batch * nx * ny;
    const int tiles = (int)(2 * cells / 128);
    nn::nn_prims_kernel<nn::PackedStates><<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(sv, batch, h->gamma, h->prims);
    const nn::PrimView pv{h->prims, nx, ny};
    nn::nn_forward_kernel<<<tiles, 128, nn::SM_FWD, s>>>(pv, nn_net(h), h->corr, 0.f, nullptr);
    NN_TRY(h, cudaMemsetAsync(h->loss_d, 0, sizeof(double), s));
    nn::nn_residual_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(h->corr, resid, batch, nx, ny, 1.0 / dx,
                                                                         1.0 / dy, w[0], w[1], w[2], w[3], h->dcorr,
                                                                         h->loss_d);
    nn::nn_backward_kernel<<<tiles, 128, nn::SM_TOTAL, s>>>(pv, nn_net(h), h->dcorr, h->partials);
    nn::nn_reduce_kernel<<<(nn::P_COUNT + 255) / 256, 256, 0, s>>>(h->partials, tiles, h->grad);
    if (grad_out) NN_TRY(h, cudaMemcpyAsync(grad_out, h->grad, nn::P_COUNT * sizeof(float), cudaMemcpyDeviceToDevice, s));
    NN_TRY(h, cudaGetLastError());
    if (loss) NN_TRY(h, cudaMemcpyAsync(loss, h->loss_d, sizeof(double), cudaMemcpyDeviceToHost, s));
    NN_TRY(h, cudaStreamSynchronize(s));
    return tc_status(h);
}

int efvm_nn_adam(efvm_nn* h, float lr, void* stream) {
    if (!h) return nfail(h, EFVM_ERR_INVALID_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    h->steps += 1;
    const float b1t = (float)std::pow(0.9, (double)h->steps), b2t = (float)std::pow(0.999, (double)h->steps);
    nn::nn_adam_kernel<<<(nn::P_COUNT + 255) / 256, 256, 0, s>>>(h->p, h->m, h->v, h->grad, lr, b1t, b2t, h->w1, h->w2,
                                                                 h->w3);
    NN_TRY(h, cudaGetLastError());
    return EFVM_OK;
}

}  // extern "C"


extern "C" int efvm_nn_gemm_bf16(const uint16_t* a, const uint16_t* b, float* d, int32_t m, int32_t n, int32_t k,
                                 void* stream) {
    if (!a || !b || !d) {
        set_global_error("efvm_nn_gemm_bf16: null argument");
        return EFVM_ERR_INVALID_ARG;
    }
    if (m <= 0 || m % 128 || n < 16 || n > 256 || n % 16 || k < 16 || k > 256 || k % 16) {
        set_global_error("efvm_nn_gemm_bf16: need m a multiple of 128, n and k multiples of 16 in [16, 256]");
        return EFVM_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int zero = 0;
    cudaError_t e = cudaMemcpyToSymbolAsync(g_nn_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s);
    // The operands need (128 + n) * k * 2 bytes; the launch takes 200 KB so that
    // every descriptor stride stays inside the CTA's shared memory whatever the
    // operand shape.
    const size_t smem = 200 * 1024;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(nn_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
        set_global_error(std::string("efvm_nn_gemm_bf16: ") + cudaGetErrorString(e));
        return EFVM_ERR_CUDA;
    }
    nn_gemm_kernel<<<m / 128, 128, smem, s>>>(reinterpret_cast<const __nv_bfloat16*>(a),
                                              reinterpret_cast<const __nv_bfloat16*>(b), d, n, k);
    int err = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyFromSymbolAsync(&err, g_nn_error, sizeof(int), 0, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_global_error(std::string("efvm_nn_gemm_bf16: ") + cudaGetErrorString(e));
        return EFVM_ERR_CUDA;
    }
    if (err) {
        set_global_error("efvm_nn_gemm_bf16: a tensor-core completion wait ran out");
        return EFVM_ERR_TIMEOUT;
    }
    return EFVM_OK;
}
