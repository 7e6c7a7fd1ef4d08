// learned.cu - the Stokes-side kernels of the learned preconditioner stage
// (3D): network inputs from a residual, training targets from an error,
// the correction from the network output, and the accept/fallback step.
//
// Scales: with s the RMS of the velocity residual, the network sees
// r_u / s (velocity residual averaged to cells), r_p / (s dx) (divergence
// residual) and log beta, and predicts beta e_u / (s dx^2) and e_p / (s dx)
// at cells, so its inputs and outputs are O(1) whatever the grid spacing,
// the viscosity contrast and the residual's size.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "learned.cuh"

namespace lmm {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void k_randn(double* out, int64_t n, uint64_t seed) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t h = mix64(seed ^ mix64((uint64_t)e * 2 + 1));
        const double u1 = ((double)(h >> 11) + 1.0) / 9007199254740993.0;
        const uint64_t h2 = mix64(h);
        const double u2 = (double)(h2 >> 11) / 9007199254740992.0;
        out[e] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    }
}

__global__ void k_lin(double* out, const double* a, double alpha, const double* b, int64_t n) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        out[e] = a[e] + alpha * b[e];
}

__device__ __forceinline__ double vel_scale(const double* sums, int64_t n) {
    const double s2 = (sums[0] + sums[1] + sums[2]) / (3.0 * (double)n);
    return s2 > 0.0 ? sqrt(s2) : 1.0;
}

__device__ __forceinline__ void cell_of(const Dims& D, int64_t s, int& i, int& j, int& k) {
    i = (int)(s % D.nx);
    const int64_t t = s / D.nx;
    j = (int)(t % D.ny);
    k = (int)(t / D.ny);
}

__global__ void k_features(Dims D, const double* __restrict__ r, const double* __restrict__ beta, const double* __restrict__ sums,
                           double dx, __nv_bfloat16* __restrict__ x) {
    const int64_t n = (int64_t)D.nx * D.ny * D.nz;
    const double s = vel_scale(sums, n);
    const double iu = 1.0 / s, ip = 1.0 / (s * dx);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(D, e, i, j, k);
        const int64_t ex = (i == D.nx - 1) ? e - (D.nx - 1) : e + 1;
        const int64_t ey = (j == D.ny - 1) ? e - (int64_t)(D.ny - 1) * D.nx : e + D.nx;
        const int64_t ez = (k == D.nz - 1) ? e - (int64_t)(D.nz - 1) * D.nx * D.ny : e + (int64_t)D.nx * D.ny;
        __align__(16) __nv_bfloat16 h[8];
        h[0] = __float2bfloat16((float)(0.5 * (r[e] + r[ex]) * iu));
        h[1] = __float2bfloat16((float)(0.5 * (r[n + e] + r[n + ey]) * iu));
        h[2] = __float2bfloat16((float)(0.5 * (r[2 * n + e] + r[2 * n + ez]) * iu));
        h[3] = __float2bfloat16((float)(r[3 * n + e] * ip));
        h[4] = __float2bfloat16((float)log(beta[e]));
        h[5] = h[6] = h[7] = __float2bfloat16(0.f);
        *reinterpret_cast<uint4*>(x + e * 8) = *reinterpret_cast<const uint4*>(h);
    }
}

// psum[3]: sum of e_p (its mean is removed: the pressure is defined up to a constant)
__global__ void k_target(Dims D, const double* __restrict__ ev, const double* __restrict__ beta, const double* __restrict__ sums,
                         const double* __restrict__ psum, double dx, float* __restrict__ t) {
    const int64_t n = (int64_t)D.nx * D.ny * D.nz;
    const double s = vel_scale(sums, n);
    const double iu = 1.0 / (s * dx * dx), ip = 1.0 / (s * dx);
    const double pmean = psum[3] / (double)n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(D, e, i, j, k);
        const int64_t ex = (i == D.nx - 1) ? e - (D.nx - 1) : e + 1;
        const int64_t ey = (j == D.ny - 1) ? e - (int64_t)(D.ny - 1) * D.nx : e + D.nx;
        const int64_t ez = (k == D.nz - 1) ? e - (int64_t)(D.nz - 1) * D.nx * D.ny : e + (int64_t)D.nx * D.ny;
        const double bu = beta[e] * iu;
        t[e * 4 + 0] = (float)(0.5 * (ev[e] + ev[ex]) * bu);
        t[e * 4 + 1] = (float)(0.5 * (ev[n + e] + ev[n + ey]) * bu);
        t[e * 4 + 2] = (float)(0.5 * (ev[2 * n + e] + ev[2 * n + ez]) * bu);
        t[e * 4 + 3] = (float)((ev[3 * n + e] - pmean) * ip);
    }
}

// c_u(face i) = (y_u/beta (cell i-1) + y_u/beta (cell i)) / 2 * s dx^2, c_p = y_p s dx
__global__ void k_correction(Dims D, const float* __restrict__ y, const double* __restrict__ beta, const double* __restrict__ sums,
                             double dx, double* __restrict__ c) {
    const int64_t n = (int64_t)D.nx * D.ny * D.nz;
    const double s = vel_scale(sums, n);
    const double su = s * dx * dx, sp = s * dx;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(D, e, i, j, k);
        const int64_t mx = (i == 0) ? e + (D.nx - 1) : e - 1;
        const int64_t my = (j == 0) ? e + (int64_t)(D.ny - 1) * D.nx : e - D.nx;
        const int64_t mz = (k == 0) ? e + (int64_t)(D.nz - 1) * D.nx * D.ny : e - (int64_t)D.nx * D.ny;
        const double ib = 1.0 / beta[e];
        c[e] = 0.5 * ((double)y[mx * 4 + 0] / beta[mx] + (double)y[e * 4 + 0] * ib) * su;
        c[n + e] = 0.5 * ((double)y[my * 4 + 1] / beta[my] + (double)y[e * 4 + 1] * ib) * su;
        c[2 * n + e] = 0.5 * ((double)y[mz * 4 + 2] / beta[mz] + (double)y[e * 4 + 2] * ib) * su;
        c[3 * n + e] = (double)y[e * 4 + 3] * sp;
    }
}

// accept the correction c when it reduced the residual (w += A c), else
// c = 0 (n1 = Stokes norm of r1, n2 = of r1 - A c, in reduction slots)
__global__ void k_accept(double* __restrict__ c, double* __restrict__ w, const double* __restrict__ Ac, const double* __restrict__ n1,
                         const double* __restrict__ n2, double factor, int* __restrict__ uses, int64_t len) {
    const bool use = *n2 < factor * *n1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        uses[0] += use ? 1 : 0;
        uses[1] += 1;
    }
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < len; e += (int64_t)gridDim.x * blockDim.x) {
        if (use)
            w[e] = w[e] + Ac[e];
        else
            c[e] = 0.0;
    }
}

int grid_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (int)(b > 8192 ? 8192 : (b < 1 ? 1 : b));
}

}  // namespace

void launch_randn(double* out, int64_t n, uint64_t seed, cudaStream_t s) { k_randn<<<grid_for(n), 256, 0, s>>>(out, n, seed); }
void launch_lin(double* out, const double* a, double alpha, const double* b, int64_t n, cudaStream_t s) {
    k_lin<<<grid_for(n), 256, 0, s>>>(out, a, alpha, b, n);
}
void launch_features(const Dims& D, const double* r, const double* beta, const double* sums, double dx, __nv_bfloat16* x,
                     cudaStream_t s) {
    k_features<<<grid_for((int64_t)D.nx * D.ny * D.nz), 256, 0, s>>>(D, r, beta, sums, dx, x);
}
void launch_target(const Dims& D, const double* e, const double* beta, const double* sums, const double* psum, double dx, float* t,
                   cudaStream_t s) {
    k_target<<<grid_for((int64_t)D.nx * D.ny * D.nz), 256, 0, s>>>(D, e, beta, sums, psum, dx, t);
}
void launch_correction(const Dims& D, const float* y, const double* beta, const double* sums, double dx, double* c, cudaStream_t s) {
    k_correction<<<grid_for((int64_t)D.nx * D.ny * D.nz), 256, 0, s>>>(D, y, beta, sums, dx, c);
}
void launch_accept(double* c, double* w, const double* Ac, const double* n1, const double* n2, double factor, int* uses, int64_t len,
                   cudaStream_t s) {
    k_accept<<<grid_for(len), 256, 0, s>>>(c, w, Ac, n1, n2, factor, uses, len);
}

}  // namespace lmm

// the bounds-check table and record of this translation unit (empty
// unless built with -DLMM_BOUNDS_CHECK)
LMM_BC_UNIT(learned)
