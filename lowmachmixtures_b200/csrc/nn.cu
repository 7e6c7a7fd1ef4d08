// nn.cu - tensor-core (tcgen05) kernels of the learned preconditioner stage.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/lmm_learned.h"
#include "../../include/lmm_stokes.h"
#include "kernels.h"
#include "conv_tile.cuh"
#include "nn_layers.cuh"
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
    if (raise_smem_limit((const void*)k_gemm_bf16, smem) != cudaSuccess) return LMM_ERR_CUDA;
    GatherRowMajor G{static_cast<const __nv_bfloat16*>(A), static_cast<const __nv_bfloat16*>(B), M, N, K};
    EpiStore E{D, M, N};
    k_gemm_bf16<<<(M + tc::kM - 1) / tc::kM, tc::kThreadsTC, smem, static_cast<cudaStream_t>(stream)>>>(G, E, err_dev);
    if (cudaGetLastError() != cudaSuccess) return LMM_ERR_CUDA;
    count_launch();
    return LMM_OK;
}

// ------------------------------------------------------------ layer launchers
namespace lmm {
namespace nn {

static inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

int conv3d(const bf16* x, const bf16* w, const float* bias, const bf16* skip, const bf16* mask, bf16* out, float* out32, int B,
           int nx, int ny, int nz, int up, int Cin, int Cout, int Cs, int relu, int* err, cudaStream_t s) {
    if (!x || !w || !err || (!out && !out32) || B < 1 || nx < 1 || ny < 1 || nz < 1 || Cin < 8 || (Cin % 8) || Cout < 1 ||
        Cout > 256 || Cs < Cout || (out && (Cs % 8)) || (up && ((nx | ny | nz) & 1)))
        return LMM_ERR_INVALID;
    ConvGather G;
    G.x = x;
    G.w = w;
    G.g = Grid3{nx, ny, nz, nx * ny * nz};
    G.up = up;
    G.Cin = Cin;
    G.Mtot = B * nx * ny * nz;
    G.N = round_up(Cout, 16);
    G.K = 27 * Cin;
    ConvEpi E{bias, skip, mask, out, out32, G.Mtot, Cout, Cs, relu};
    // the shifted-view tile kernel where the grid tiles by 8 x 16 and the
    // weights and three halo planes fit in shared memory
    const int cinp = round_up(Cin, 16);
    if (nx % kTX == 0 && ny % kTY == 0 && G.N <= 64 && (cinp == 16 || cinp == 32 || cinp == 64) &&
        tile_smem_bytes(cinp, G.N) <= 227 * 1024) {
        TileConvArgs A{x, w, nx, ny, nz, up, Cin, G.N, B, 1, nx / kTX, ny / kTY, 1};
        const int tiles = A.tiles_x * A.tiles_y * B;
        int zch = (148 * 4 + tiles - 1) / tiles;
        zch = zch < 1 ? 1 : (zch > nz ? nz : zch);
        A.KZ = (nz + zch - 1) / zch;
        A.zchunks = (nz + A.KZ - 1) / A.KZ;
        const size_t smem = tile_smem_bytes(cinp, G.N);
        const unsigned blocks = (unsigned)(tiles * A.zchunks);
        cudaError_t e = cudaSuccess;
        if (cinp == 16) {
            e = raise_smem_limit((const void*)k_conv3d_tile<16>, smem);
            if (e == cudaSuccess) k_conv3d_tile<16><<<blocks, tc::kThreadsTC, smem, s>>>(A, E, err);
        } else if (cinp == 32) {
            e = raise_smem_limit((const void*)k_conv3d_tile<32>, smem);
            if (e == cudaSuccess) k_conv3d_tile<32><<<blocks, tc::kThreadsTC, smem, s>>>(A, E, err);
        } else {
            e = raise_smem_limit((const void*)k_conv3d_tile<64>, smem);
            if (e == cudaSuccess) k_conv3d_tile<64><<<blocks, tc::kThreadsTC, smem, s>>>(A, E, err);
        }
        if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return LMM_ERR_CUDA;
        count_launch();
        return LMM_OK;
    }
    if (raise_smem_limit((const void*)k_conv3d, tc::smem_bytes(G.N)) != cudaSuccess) return LMM_ERR_CUDA;
    k_conv3d<<<(G.Mtot + tc::kM - 1) / tc::kM, tc::kThreadsTC, tc::smem_bytes(G.N), s>>>(G, E, err);
    if (cudaGetLastError() != cudaSuccess) return LMM_ERR_CUDA;
    count_launch();
    return LMM_OK;
}

int conv3d_wgrad(const bf16* x, const bf16* g, float* dw, int B, int nx, int ny, int nz, int up, int Cin, int Cg, int Cout, int* err,
                 cudaStream_t s) {
    if (!x || !g || !dw || !err || B < 1 || Cin < 8 || (Cin % 8) || Cg < Cout || (Cg % 8) || Cout < 1 || Cout > 256 ||
        (up && ((nx | ny | nz) & 1)))
        return LMM_ERR_INVALID;
    WgradGather G;
    G.x = x;
    G.gr = g;
    G.g = Grid3{nx, ny, nz, nx * ny * nz};
    G.up = up;
    G.Cin = Cin;
    G.Cg = Cg;
    G.Mtot = B * nx * ny * nz;
    G.N = round_up(Cout, 16);
    G.kbeg = 0;
    const int rows = 27 * Cin;
    WgradEpi E{dw, rows, Cout};
    // split the voxels so that about 4 CTAs per SM run
    const int mt = (rows + tc::kM - 1) / tc::kM;
    int splits = (148 * 4 + mt - 1) / mt;
    int kspan = round_up((G.Mtot + splits - 1) / splits, tc::kKC);
    if (kspan < 8 * tc::kKC) kspan = 8 * tc::kKC;
    splits = (G.Mtot + kspan - 1) / kspan;
    if (raise_smem_limit((const void*)k_conv3d_wgrad, tc::smem_bytes(G.N)) != cudaSuccess) return LMM_ERR_CUDA;
    k_conv3d_wgrad<<<dim3(mt, splits), tc::kThreadsTC, tc::smem_bytes(G.N), s>>>(G, E, kspan, err);
    if (cudaGetLastError() != cudaSuccess) return LMM_ERR_CUDA;
    count_launch();
    return LMM_OK;
}

int pack_weights(const float* w, bf16* wf, bf16* wt, int Cout, int Cin, cudaStream_t s) {
    if (!w || !wf || Cin < 1 || Cout < 1) return LMM_ERR_INVALID;
    const int Npad = round_up(Cout, 16), Coutp = round_up(Cout, 8), Cinpad = round_up(Cin, 16);
    const int n = Npad * 27 * Cin + (wt ? Cinpad * 27 * Coutp : 0);
    k_pack_weights<<<(n + 255) / 256, 256, 0, s>>>(w, wf, wt, Cout, Cin, Npad, Coutp, Cinpad);
    if (cudaGetLastError() != cudaSuccess) return LMM_ERR_CUDA;
    count_launch();
    return LMM_OK;
}

}  // namespace nn
}  // namespace lmm

extern "C" int lmm_nn_conv3d(const void* x, const void* w, const float* bias, const void* skip, const void* mask, void* out,
                             float* out32, int B, int nx, int ny, int nz, int up, int Cin, int Cout, int Cs, int relu, int* err_dev,
                             void* stream) {
    using lmm::nn::bf16;
    return lmm::nn::conv3d(static_cast<const bf16*>(x), static_cast<const bf16*>(w), bias, static_cast<const bf16*>(skip),
                           static_cast<const bf16*>(mask), static_cast<bf16*>(out), out32, B, nx, ny, nz, up, Cin, Cout, Cs, relu,
                           err_dev, static_cast<cudaStream_t>(stream));
}

extern "C" int lmm_nn_conv3d_wgrad(const void* x, const void* g, float* dw, int B, int nx, int ny, int nz, int up, int Cin, int Cg,
                                   int Cout, int* err_dev, void* stream) {
    using lmm::nn::bf16;
    return lmm::nn::conv3d_wgrad(static_cast<const bf16*>(x), static_cast<const bf16*>(g), dw, B, nx, ny, nz, up, Cin, Cg, Cout,
                                 err_dev, static_cast<cudaStream_t>(stream));
}

extern "C" int lmm_nn_pack_weights(const float* w, void* wf, void* wt, int Cout, int Cin, void* stream) {
    using lmm::nn::bf16;
    return lmm::nn::pack_weights(w, static_cast<bf16*>(wf), static_cast<bf16*>(wt), Cout, Cin, static_cast<cudaStream_t>(stream));
}
