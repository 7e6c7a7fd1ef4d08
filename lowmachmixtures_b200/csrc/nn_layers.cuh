// nn_layers.cuh - layers of the learned preconditioner network on the
// tcgen05 tile of tc.cuh: 3x3x3 periodic convolutions as implicit GEMMs
// (forward and data gradient: voxels x output channels, K = 27 taps x input
// channels, K-major operands gathered straight from channels-last
// activations), the weight gradient (rows = taps x input channels, columns =
// output channels, K = voxels, MN-major operands) and the elementwise pieces
// (pooling, upsampling adjoint, ReLU masks, bias gradient, Adam).
//
// Activations are channels-last BF16, [batch][z][y][x][C], C a multiple of 8.
// Weights are [Cout][27][Cin] (tap t = (dz+1)*9 + (dy+1)*3 + (dx+1)), stored
// for the GEMM as BF16 rows padded to a multiple of 16.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "tc.cuh"

namespace lmm {
namespace nn {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ int wrapn(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// voxel m of the batch (row of the implicit GEMM) -> (b, i, j, k)
struct Grid3 {
    int nx, ny, nz, V;
    __device__ __forceinline__ void decode(int m, int& b, int& i, int& j, int& k) const {
        b = m / V;
        int v = m - b * V;
        i = v % nx;
        v /= nx;
        j = v % ny;
        k = v / ny;
    }
};

// index of the input voxel read by tap t of output voxel (b, i, j, k); with
// up = 1 the input lives on the half grid (nearest-neighbour upsampling)
__device__ __forceinline__ int64_t tap_src(const Grid3& g, int up, int b, int i, int j, int k, int t) {
    const int ii = wrapn(i + (t % 3) - 1, g.nx);
    const int jj = wrapn(j + (t / 3) % 3 - 1, g.ny);
    const int kk = wrapn(k + t / 9 - 1, g.nz);
    const int nxi = g.nx >> up, nyi = g.ny >> up, nzi = g.nz >> up;
    return (((int64_t)b * nzi + (kk >> up)) * nyi + (jj >> up)) * nxi + (ii >> up);
}

// ------------------------------------------------------------ convolution
struct ConvGather {
    const bf16* x;   // input activations, Cin channels
    const bf16* w;   // [N][K] BF16, K = 27 * Cin
    Grid3 g;         // output grid
    int up, Cin, Mtot, N, K;
    __device__ void a(int m0, int k0, uint8_t* sA) const {
        // thread r owns row r: decode its voxel once per chunk
        for (int r = threadIdx.x; r < tc::kM; r += blockDim.x) {
            const int m = m0 + r;
            int b = 0, i = 0, j = 0, k = 0;
            const bool row_ok = m < Mtot;
            if (row_ok) g.decode(m, b, i, j, k);
#pragma unroll
            for (int q = 0; q < tc::kKC / 8; ++q) {
                const int kq = k0 + 8 * q;
                uint4 v = make_uint4(0, 0, 0, 0);
                if (row_ok && kq < K) {
                    const int t = kq / Cin, c0 = kq - t * Cin;
                    v = *reinterpret_cast<const uint4*>(x + tap_src(g, up, b, i, j, k, t) * Cin + c0);
                }
                *reinterpret_cast<uint4*>(sA + tc::chunk_off(tc::kM, r, 8 * q)) = v;
            }
        }
    }
    __device__ void b(int k0, uint8_t* sB) const {
        for (int u = threadIdx.x; u < N * (tc::kKC / 8); u += blockDim.x) {
            const int r = u / (tc::kKC / 8), q = u % (tc::kKC / 8);
            const int kq = k0 + 8 * q;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (kq < K) v = *reinterpret_cast<const uint4*>(w + (int64_t)r * K + kq);
            *reinterpret_cast<uint4*>(sB + tc::chunk_off(N, r, 8 * q)) = v;
        }
    }
};

// out = act(acc + bias + skip) [* (mask > 0)], channels 0..Cout-1 of a
// row of Cs channels (the padding channels Cout..Cs-1 are written 0)
struct ConvEpi {
    const float* bias;   // [Cout] or null
    const bf16* skip;    // [Mtot][Cs] or null
    const bf16* mask;    // [Mtot][Cs] or null
    bf16* out;           // [Mtot][Cs] or null
    float* out32;        // [Mtot][Cs] or null
    int Mtot, Cout, Cs, relu;
    __device__ void operator()(int row, int c0, const float (&v)[16]) const {
        if (row >= Mtot || c0 >= Cs) return;
        float o[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int c = c0 + q;
            float val = 0.f;
            if (c < Cout) {
                val = v[q];
                if (bias) val += bias[c];
                if (skip) val += __bfloat162float(skip[(int64_t)row * Cs + c]);
                if (relu) val = fmaxf(val, 0.f);
                if (mask && !(__bfloat162float(mask[(int64_t)row * Cs + c]) > 0.f)) val = 0.f;
            }
            o[q] = val;
        }
        const int nc = (Cs - c0) < 16 ? (Cs - c0) : 16;   // 8 or 16 (Cs % 8 == 0)
        if (out) {
            __align__(16) bf16 h[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) h[q] = __float2bfloat16(o[q]);
            uint4* dst = reinterpret_cast<uint4*>(out + (int64_t)row * Cs + c0);
            dst[0] = reinterpret_cast<const uint4*>(h)[0];
            if (nc > 8) dst[1] = reinterpret_cast<const uint4*>(h)[1];
        }
        if (out32) {
            float* dst = out32 + (int64_t)row * Cs + c0;
            for (int q = 0; q < nc; ++q) dst[q] = o[q];
        }
    }
};

static __global__ void __launch_bounds__(tc::kThreadsTC) k_conv3d(ConvGather G, ConvEpi E, int* err) {
    extern __shared__ __align__(1024) uint8_t conv_smem[];
    tc::gemm_tile(G, E, blockIdx.x * tc::kM, G.N, G.K, conv_smem, err);
}

// ------------------------------------------------------------ weight gradient
// dW[co][t][ci] += sum over this CTA's voxels of g[v][co] * x_tap_t(v)[ci];
// rows of the GEMM are (t, ci), columns co, K the voxels.
struct WgradGather {
    const bf16* x;   // input activations, Cin channels
    const bf16* gr;  // output gradient [Mtot][Cg]
    Grid3 g;
    int up, Cin, Cg, Mtot, N, kbeg;
    __device__ void a(int m0, int k0, uint8_t* sA) const {
        const int rows = 27 * Cin;
        for (int u = threadIdx.x; u < (tc::kM / 8) * tc::kKC; u += blockDim.x) {
            const int q = u % (tc::kM / 8), kk = u / (tc::kM / 8);
            const int mrow = m0 + 8 * q, vox = kbeg + k0 + kk;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (mrow < rows && vox < Mtot) {
                const int t = mrow / Cin, c0 = mrow - t * Cin;
                int b, i, j, k;
                g.decode(vox, b, i, j, k);
                v = *reinterpret_cast<const uint4*>(x + tap_src(g, up, b, i, j, k, t) * Cin + c0);
            }
            *reinterpret_cast<uint4*>(sA + tc::chunk_off_mn(tc::kM, 8 * q, kk)) = v;
        }
    }
    __device__ void b(int k0, uint8_t* sB) const {
        const int ng = N / 8;
        for (int u = threadIdx.x; u < ng * tc::kKC; u += blockDim.x) {
            const int q = u % ng, kk = u / ng;
            const int vox = kbeg + k0 + kk;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (vox < Mtot && 8 * q < Cg) v = *reinterpret_cast<const uint4*>(gr + (int64_t)vox * Cg + 8 * q);
            *reinterpret_cast<uint4*>(sB + tc::chunk_off_mn(N, 8 * q, kk)) = v;
        }
    }
};

struct WgradEpi {
    float* dw;   // [Cout][27 * Cin]
    int rows, Cout;
    __device__ void operator()(int row, int c0, const float (&v)[16]) const {
        if (row >= rows) return;
#pragma unroll
        for (int q = 0; q < 16; ++q)
            if (c0 + q < Cout) atomicAdd(dw + (int64_t)(c0 + q) * rows + row, v[q]);
    }
};

static __global__ void __launch_bounds__(tc::kThreadsTC) k_conv3d_wgrad(WgradGather G, WgradEpi E, int kspan, int* err) {
    extern __shared__ __align__(1024) uint8_t wg_smem[];
    WgradGather g = G;
    g.kbeg = blockIdx.y * kspan;
    int K = G.Mtot - g.kbeg;
    if (K > kspan) K = kspan;
    tc::gemm_tile<WgradGather, WgradEpi, 1, 1>(g, E, blockIdx.x * tc::kM, G.N, K, wg_smem, err);
}

// ------------------------------------------------------------ elementwise
// the sum over the 8 fine children of coarse voxel (b, i, j, k), channels
// 8g .. 8g+7, children in the order d = 0..7 (x fastest), in FP32; C % 8 == 0
__device__ __forceinline__ void sum_children8(const bf16* __restrict__ f, int64_t b, int i, int j, int k, int g, int nx,
                                              int ny, int nz, int C, float (&s)[8]) {
#pragma unroll
    for (int q = 0; q < 8; ++q) s[q] = 0.f;
#pragma unroll
    for (int d = 0; d < 8; ++d) {
        const int fi = 2 * i + (d & 1), fj = 2 * j + ((d >> 1) & 1), fk = 2 * k + (d >> 2);
        const uint4 u = *reinterpret_cast<const uint4*>(f + (((b * 2 * nz + fk) * 2 * ny + fj) * 2 * nx + fi) * C + 8 * g);
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            s[2 * q] += __uint_as_float(w[q] << 16);
            s[2 * q + 1] += __uint_as_float(w[q] & 0xFFFF0000u);
        }
    }
}
__device__ __forceinline__ uint4 pack8_bf16(const float (&s)[8], float scale) {
    uint32_t w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(s[2 * q] * scale, s[2 * q + 1] * scale);
        w[q] = *reinterpret_cast<const uint32_t*>(&h);
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

// 2x2x2 average pooling, [B][nz][ny][nx][C] from the fine grid of twice the
// extents; one thread per (coarse voxel, group of 8 channels)
static __global__ void k_pool2(const bf16* __restrict__ f, bf16* __restrict__ c, int B, int nx, int ny, int nz, int C) {
    const int G = C / 8;
    const int64_t n = (int64_t)B * nx * ny * nz * G;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int g = (int)(e % G);
        int64_t v = e / G;
        const int i = (int)(v % nx);
        v /= nx;
        const int j = (int)(v % ny);
        v /= ny;
        const int k = (int)(v % nz);
        const int64_t b = v / nz;
        float s[8];
        sum_children8(f, b, i, j, k, g, nx, ny, nz, C, s);
        *reinterpret_cast<uint4*>(c + e * 8) = pack8_bf16(s, 0.125f);
    }
}

// adjoint of nearest upsampling: coarse[v][c] = sum of the 8 fine children
static __global__ void k_downsum(const bf16* __restrict__ f, bf16* __restrict__ c, int B, int nx, int ny, int nz, int C) {
    const int G = C / 8;
    const int64_t n = (int64_t)B * nx * ny * nz * G;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int g = (int)(e % G);
        int64_t v = e / G;
        const int i = (int)(v % nx);
        v /= nx;
        const int j = (int)(v % ny);
        v /= ny;
        const int k = (int)(v % nz);
        const int64_t b = v / nz;
        float s[8];
        sum_children8(f, b, i, j, k, g, nx, ny, nz, C, s);
        *reinterpret_cast<uint4*>(c + e * 8) = pack8_bf16(s, 1.f);
    }
}

// g = (a + pool_adjoint(p)) * (act > 0) on the fine grid [B][nz][ny][nx][C];
// p (coarse, may be null) contributes p[parent] / 8
static __global__ void k_grad_combine(const bf16* __restrict__ a, const bf16* __restrict__ p, const bf16* __restrict__ act,
                               bf16* __restrict__ g, int B, int nx, int ny, int nz, int C) {
    const int64_t n = (int64_t)B * nx * ny * nz * C;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        float s = a ? __bfloat162float(a[e]) : 0.f;
        if (p) {
            const int ch = (int)(e % C);
            int64_t v = e / C;
            const int i = (int)(v % nx);
            v /= nx;
            const int j = (int)(v % ny);
            v /= ny;
            const int k = (int)(v % nz);
            const int b = (int)(v / nz);
            const int64_t pc = ((((int64_t)b * (nz / 2) + k / 2) * (ny / 2) + j / 2) * (nx / 2) + i / 2) * C + ch;
            s += __bfloat162float(p[pc]) * 0.125f;
        }
        if (!(__bfloat162float(act[e]) > 0.f)) s = 0.f;
        g[e] = __float2bfloat16(s);
    }
}

// db[c] += sum_m g[m][c]  (Cs channels per row, the first C summed)
static __global__ void k_bias_grad(const bf16* __restrict__ g, float* __restrict__ db, int64_t M, int C, int Cs) {
    __shared__ float acc[64];
    for (int c = threadIdx.x; c < 64; c += blockDim.x) acc[c] = 0.f;
    __syncthreads();
    const int c = threadIdx.x % C;
    const int lanes = blockDim.x / C;
    float s = 0.f;
    if ((int)threadIdx.x < lanes * C)
        for (int64_t m = blockIdx.x * (int64_t)lanes + threadIdx.x / C; m < M; m += (int64_t)gridDim.x * lanes)
            s += __bfloat162float(g[m * Cs + c]);
    atomicAdd(&acc[c], s);
    __syncthreads();
    for (int q = threadIdx.x; q < C; q += blockDim.x) atomicAdd(&db[q], acc[q]);
}

// Adam on FP32 master parameters
static __global__ void k_adam(float* __restrict__ w, float* __restrict__ m1, float* __restrict__ m2, const float* __restrict__ gr,
                       int64_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const float g = gr[e];
        const float a = b1 * m1[e] + (1.f - b1) * g;
        const float b = b2 * m2[e] + (1.f - b2) * g * g;
        m1[e] = a;
        m2[e] = b;
        w[e] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
    }
}

// FP32 master [Cout][27][Cin] -> forward GEMM rows wf[Npad][27*Cin] and the
// data-gradient rows wt[Cinpad][27*Coutp]: wt[ci][s][co] = w[co][26-s][ci]
static __global__ void k_pack_weights(const float* __restrict__ w, bf16* __restrict__ wf, bf16* __restrict__ wt, int Cout, int Cin,
                               int Npad, int Coutp, int Cinpad) {
    const int K = 27 * Cin, Kt = 27 * Coutp;
    const int nf = Npad * K, nt = wt ? Cinpad * Kt : 0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nf + nt; e += gridDim.x * blockDim.x) {
        if (e < nf) {
            const int co = e / K, r = e % K;
            wf[e] = __float2bfloat16(co < Cout ? w[(int64_t)co * K + r] : 0.f);
        } else {
            const int f = e - nf;
            const int ci = f / Kt, r = f % Kt, s = r / Coutp, co = r % Coutp;
            float v = 0.f;
            if (ci < Cin && co < Cout) v = w[((int64_t)co * 27 + (26 - s)) * Cin + ci];
            wt[f] = __float2bfloat16(v);
        }
    }
}

}  // namespace nn
}  // namespace lmm
