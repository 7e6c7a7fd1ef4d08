// nn.cu - tensor-core (tcgen05) kernels of the learned preconditioner stage.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/lmm_learned.h"
#include "../../include/lmm_stokes.h"
#include "kernels.h"
#include "conv_tile_ws.cuh"
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

// persistent launch of a tile kernel (ZN: the warp-specialised kernel with
// the z taps in N, else 27 taps):
// as many CTAs as are resident at once (shared memory, registers and TMEM
// columns permitting), split evenly over the output-channel slices, each
// taking an equal run of its slice's (tile, plane) sequence
template <bool ZN, int CINP, int NS>
static int launch_tile_n(TileConvArgs A, const ConvEpi& E, int* err, cudaStream_t s) {
    constexpr int smem_c = ZN ? ws_smem_bytes(CINP, NS) : tile_smem_bytes(CINP, NS);
    constexpr int threads = ZN ? kThreadsWS : tc::kThreadsTC;
    if constexpr (smem_c > 227 * 1024 || (ZN && (CINP > 32 || NS != 16))) {
        return LMM_ERR_INVALID;
    } else {
        const void* kern;
        if constexpr (ZN)
            kern = (const void*)k_conv3d_ws<CINP, NS>;
        else
            kern = (const void*)k_conv3d_tile<CINP, NS>;
        const size_t smem = smem_c;
        if (raise_smem_limit(kern, smem) != cudaSuccess) return LMM_ERR_CUDA;
        // resident CTAs per SM, from the SM's shared memory (the carveout is
        // set to its maximum), its register file and its 512 TMEM columns
        static int per_sm_cached[16] = {};
        int dev = 0, sms = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return LMM_ERR_CUDA;
        int per_sm = dev < 16 ? per_sm_cached[dev] : 0;
        if (per_sm == 0) {
            int smem_sm = 0, smem_rsv = 0, regs_sm = 0;
            cudaFuncAttributes fa;
            if (cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess ||
                cudaFuncGetAttributes(&fa, kern) != cudaSuccess ||
                cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess)
                return LMM_ERR_CUDA;
            const int by_smem = smem_sm / (int)(smem + fa.sharedSizeBytes + smem_rsv);
            const int regs_warp = ((fa.numRegs + 7) / 8 * 8) * 32;
            const int by_regs = regs_sm / (regs_warp * (threads / 32));
            const int by_tmem = 512 / (int)(ZN ? ws_tmem_cols(NS) : tile_tmem_cols(NS));
            per_sm = by_smem < by_regs ? by_smem : by_regs;
            per_sm = per_sm < by_tmem ? per_sm : by_tmem;
            per_sm = per_sm < 16 ? per_sm : 16;
            if (per_sm < 1) per_sm = 1;
            if (dev < 16) per_sm_cached[dev] = per_sm;
        }
        int64_t cps = (int64_t)sms * per_sm / A.slices;
        cps = cps < 1 ? 1 : (cps > A.total ? A.total : cps);
        A.ctas_per_slice = (int)cps;
        const unsigned blocks = (unsigned)(A.slices * cps);
        if constexpr (ZN)
            k_conv3d_ws<CINP, NS><<<blocks, threads, smem, s>>>(A, E, err);
        else
            k_conv3d_tile<CINP, NS><<<blocks, tc::kThreadsTC, smem, s>>>(A, E, err);
        if (cudaGetLastError() != cudaSuccess) return LMM_ERR_CUDA;
        count_launch();
        return LMM_OK;
    }
}
template <bool ZN, int CINP>
static int launch_tile_c(int ns, const TileConvArgs& A, const ConvEpi& E, int* err, cudaStream_t s) {
    switch (ns) {
        case 16: return launch_tile_n<ZN, CINP, 16>(A, E, err, s);
        case 32: return launch_tile_n<ZN, CINP, 32>(A, E, err, s);
        case 48: return launch_tile_n<ZN, CINP, 48>(A, E, err, s);
        case 64: return launch_tile_n<ZN, CINP, 64>(A, E, err, s);
        default: return LMM_ERR_INVALID;
    }
}
// LMM_ERR_INVALID: no tile instantiation for (zn, cinp, ns); the caller gathers
static int launch_tile(bool zn, int cinp, int ns, const TileConvArgs& A, const ConvEpi& E, int* err, cudaStream_t s) {
    switch (cinp) {
        case 16: return zn ? launch_tile_c<true, 16>(ns, A, E, err, s) : launch_tile_c<false, 16>(ns, A, E, err, s);
        case 32: return zn ? launch_tile_c<true, 32>(ns, A, E, err, s) : launch_tile_c<false, 32>(ns, A, E, err, s);
        case 64: return launch_tile_c<false, 64>(ns, A, E, err, s);
        default: return LMM_ERR_INVALID;
    }
}
// the output-channel slice (a multiple of 16 dividing n) of a tile kernel:
// 16 with the warp-specialised z-taps-in-N kernel (*zn) for 16 or 32 input
// channels; else the 27-tap kernel's widest slice that fits in shared
// memory; 0 when none does
static int tile_slice(int cinp, int n, bool* zn) {
    *zn = cinp <= 32 && n % 16 == 0;
    if (*zn) return 16;
    for (int ns = 64; ns >= 16; ns -= 16)
        if (ns <= n && n % ns == 0 && tile_smem_bytes(cinp, ns) <= 227 * 1024) return ns;
    return 0;
}

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
    // the shifted-view tile kernel where the grid tiles by 8 x 16, a slice
    // of the weights and the halo ring fit in shared memory, and skip / mask
    // rows can be read as 16-byte vectors
    const int cinp = round_up(Cin, 16);
    bool zn = false;
    const int ns = (cinp == 16 || cinp == 32 || cinp == 64) && G.N <= 64 ? tile_slice(cinp, G.N, &zn) : 0;
    if (nx % kTX == 0 && ny % kTY == 0 && ns > 0 && ((!skip && !mask) || Cs % 8 == 0)) {
        TileConvArgs A{x, w, nx, ny, nz, up, Cin, B, nx / kTX, ny / kTY, 0, G.N / ns, 1};
        A.total = (int64_t)A.tiles_x * A.tiles_y * B * nz;
        const int rc = launch_tile(zn, cinp, ns, A, E, err, s);
        if (rc != LMM_ERR_INVALID) return rc;
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

// the bounds-check table and record of this translation unit (empty
// unless built with -DLMM_BOUNDS_CHECK)
LMM_BC_UNIT(nn)
