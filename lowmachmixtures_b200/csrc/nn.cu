// nn.cu - tensor-core (tcgen05) kernels of the learned preconditioner stage.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/lmm_learned.h"
#include "../../include/lmm_stokes.h"
#include "kernels.h"
#include "tc.cuh"

namespace lmm {
namespace {

// plain row-major GEMM operands: A[M x K], B[N x K] (BF16), K % 8 == 0
struct GatherRowMajor {
    const __nv_bfloat16* A;
    const __nv_bfloat16* B;
    int M, N, K;
    __device__ void a(int m0, int k0, uint8_t* sA) const {
        for (int u = threadIdx.x; u < tc::kM * (tc::kKC / 8); u += blockDim.x) {
            const int r = u / (tc::kKC / 8), g = u % (tc::kKC / 8);
            const int row = m0 + r, k = k0 + 8 * g;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (row < M && k < K) v = *reinterpret_cast<const uint4*>(A + (int64_t)row * K + k);
            *reinterpret_cast<uint4*>(sA + tc::chunk_off(tc::kM, r, 8 * g)) = v;
        }
    }
    __device__ void b(int k0, uint8_t* sB) const {
        for (int u = threadIdx.x; u < N * (tc::kKC / 8); u += blockDim.x) {
            const int r = u / (tc::kKC / 8), g = u % (tc::kKC / 8);
            const int k = k0 + 8 * g;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (k < K) v = *reinterpret_cast<const uint4*>(B + (int64_t)r * K + k);
            *reinterpret_cast<uint4*>(sB + tc::chunk_off(N, r, 8 * g)) = v;
        }
    }
};

struct EpiStore {
    float* D;
    int M, N;
    __device__ void operator()(int row, int c0, const float (&v)[16]) const {
        if (row >= M) return;
#pragma unroll
        for (int i = 0; i < 16; ++i)
            if (c0 + i < N) D[(int64_t)row * N + c0 + i] = v[i];
    }
};

__global__ void __launch_bounds__(tc::kThreadsTC) k_gemm_bf16(GatherRowMajor G, EpiStore E, int* err) {
    extern __shared__ __align__(1024) uint8_t tc_smem[];
    tc::gemm_tile(G, E, blockIdx.x * tc::kM, G.N, G.K, tc_smem, err);
}

}  // namespace
}  // namespace lmm

extern "C" int lmm_nn_gemm_bf16(const void* A, const void* B, float* D, int M, int N, int K, int* err_dev, void* stream) {
    using namespace lmm;
    if (!A || !B || !D || !err_dev || M < 1 || K < 8 || (K % 8) || N < 16 || N > 256 || (N % 16)) return LMM_ERR_INVALID;
    const size_t smem = tc::smem_bytes(N);
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
            return LMM_ERR_CUDA;
        attr = true;
    }
    GatherRowMajor G{static_cast<const __nv_bfloat16*>(A), static_cast<const __nv_bfloat16*>(B), M, N, K};
    EpiStore E{D, M, N};
    k_gemm_bf16<<<(M + tc::kM - 1) / tc::kM, tc::kThreadsTC, smem, static_cast<cudaStream_t>(stream)>>>(G, E, err_dev);
    if (cudaGetLastError() != cudaSuccess) return LMM_ERR_CUDA;
    count_launch();
    return LMM_OK;
}
