// efvm_nn.cu — BF16 tensor-core (tcgen05) kernels of the learned flux correction.
//
// This file holds the tensor-core GEMM tile that the correction network's
// forward and backward kernels are built from, and a stand-alone entry point
// that runs it on caller matrices (used to check the tile against a CPU
// product).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>

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

}  // namespace
}  // namespace efvm

using namespace efvm;

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
