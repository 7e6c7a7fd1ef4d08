// tail.cuh - the coarse end of the V-cycles in one thread block.
//
// Every multigrid level below a size threshold (its smooths, residual
// restrictions, bottom smooths and prolongations: stag_mg_solver.f90:338-760
// for the velocity, and this library's cell-centred pressure V-cycle) runs
// inside ONE kernel of a single thread block.  phi and rhs of all those
// levels live in shared memory for the whole tail; coefficients are read
// through the read-only cache; steps are separated by __syncthreads()
// instead of kernel boundaries, so the ~30 launches per coarse level
// collapse into one.  Only the first tail level's phi goes back to global
// memory.  The arithmetic is the same device code as the per-level kernels,
// so results are bit-identical.
//
// 2D batches (Dims::nz instances stacked along the third index): one block
// per instance, blockIdx.x = the instance; its views see one instance
// (nz = 1, every array offset by instance x nx*ny of that level).
#pragma once
#include <cstring>

#include "kernels.cuh"

namespace lmm {

constexpr int kTailThreads = 512;
constexpr int kMaxTail = 12;

template <class T>
struct TailLevel {
    Dims D;
    T dxsqinv;
    Coef<T> C;
    const T* pa[3];
};

template <class T>
struct TailArgs {
    int nl;
    int nu1, nu2, nub, smoother;
    T omega;
    T* g_phi[3];       // first tail level, global memory (in/out)
    const T* g_rhs[3]; // first tail level, global memory (in)
    T* g_pphi;         // pressure: first level phi (in/out)
    const T* g_prhs;   // pressure: first level rhs (in)
    TailLevel<T> L[kMaxTail];
};

// shared-memory views of one level
template <class T>
struct TailView {
    Dims D;
    T dxsqinv;
    Coef<T> C;
    T* phi[3];
    T* rhs[3];
    T* tmp[3];
    const T* pa[3];
    T* pphi;
    T* prhs;
    T* ptmp;   // odd levels: the pressure colour's new values
};

__device__ __forceinline__ int ncells(const Dims& D) { return D.nx * D.ny * D.nz; }

__device__ __forceinline__ void unflat3d(const Dims& D, int w, int& i, int& j, int& k) {
    i = w % D.nx;
    int r = w / D.nx;
    j = r % D.ny;
    k = r / D.ny;
}

// W: a grid with walls (wall faces keep their zero; the stencils and ghost
// rules of the per-level wall kernels)
// faces of one colour of an even level
__device__ __forceinline__ int colour_count(const Dims& D) { return (D.nx >> 1) * D.ny * D.nz; }

// threads t0, t0 + stride, ... of the block take the colour's faces
template <class T, int DM, int VISC, int COMP, bool W>
__device__ __forceinline__ void tail_colour(const TailView<T>& L, int parity, T omega, int t0, int stride) {
    const T b = ld(L.C.beta, 0), c = ld(L.C.gamma, 0);
    const int half = L.D.nx >> 1;
    const int count = half * L.D.ny * L.D.nz;
    const T* phi[3] = {L.phi[0], L.phi[1], L.phi[2]};
    T* p = L.phi[COMP];
    const T* r = L.rhs[COMP];
    for (int w = t0; w < count; w += stride) {
        const int ih = w % half;
        const int q = w / half;
        const int j = q % L.D.ny, k = q / L.D.ny;
        const int i = 2 * ih + ((j + k + parity) & 1);
        Nb nb = W ? make_nbw(L.D, i, j, k) : make_nb(L.D, i, j, k);
        if (W && wall_face(nb, COMP)) continue;
        T Lp = face_L<T, DM, VISC, COMP, 1, T, W>(phi, L.C, nb, L.dxsqinv, b, c);
        T fac = face_diag<T, DM, VISC, COMP, W>(L.C, nb, L.dxsqinv, b, c);
        T cur = p[nb.s];
        p[nb.s] = cur + omega * (r[nb.s] - Lp) / fac;
    }
}

// a colour on an odd level (as k_colour_update): every new value from the
// values before the colour's pass, staged in L.tmp[COMP]
template <class T, int DM, int VISC, int COMP, bool W>
__device__ __forceinline__ void tail_colour_odd(const TailView<T>& L, int parity, T omega) {
    const T b = ld(L.C.beta, 0), c = ld(L.C.gamma, 0);
    const int n = ncells(L.D);
    const T* phi[3] = {L.phi[0], L.phi[1], L.phi[2]};
    T* p = L.phi[COMP];
    const T* r = L.rhs[COMP];
    for (int w = threadIdx.x; w < n; w += blockDim.x) {
        int i, j, k;
        unflat3d(L.D, w, i, j, k);
        if (((i + j + k) & 1) != parity) continue;
        Nb nb = W ? make_nbw(L.D, i, j, k) : make_nb(L.D, i, j, k);
        if (W && wall_face(nb, COMP)) {
            L.tmp[COMP][w] = p[nb.s];  // stays zero
            continue;
        }
        T Lp = face_L<T, DM, VISC, COMP, 1, T, W>(phi, L.C, nb, L.dxsqinv, b, c);
        T fac = face_diag<T, DM, VISC, COMP, W>(L.C, nb, L.dxsqinv, b, c);
        T cur = p[nb.s];
        L.tmp[COMP][w] = cur + omega * (r[nb.s] - Lp) / fac;
    }
    __syncthreads();
    for (int w = threadIdx.x; w < n; w += blockDim.x) {
        int i, j, k;
        unflat3d(L.D, w, i, j, k);
        if (((i + j + k) & 1) == parity) p[w] = L.tmp[COMP][w];
    }
}

template <class T, int DM, int VISC, bool W>
__device__ void tail_smooth(const TailView<T>& L, int nsm, int smoother, T omega) {
    const T b = ld(L.C.beta, 0), c = ld(L.C.gamma, 0);
    const int n = ncells(L.D);
    // Gauss-Seidel on an even level whose colours have at most 32 faces (4^3,
    // 2^3; 4^2, 2^2): warp 0 takes every sweep, a __syncwarp between colours
    // instead of the block's barrier (the same faces, the same arithmetic)
    if (smoother != 0 && !odd_level(L.D) && colour_count(L.D) <= 32) {
        if (threadIdx.x < 32) {
            for (int s = 0; s < nsm; ++s)
                for (int color = 1; color <= 2 * DM; ++color) {
                    const int comp = (color - 1) / 2;
                    const int parity = (color % 2 == 1) ? 0 : 1;
                    if (comp == 0)
                        tail_colour<T, DM, VISC, 0, W>(L, parity, omega, threadIdx.x, 32);
                    else if (comp == 1)
                        tail_colour<T, DM, VISC, 1, W>(L, parity, omega, threadIdx.x, 32);
                    else if constexpr (DM == 3)
                        tail_colour<T, DM, VISC, 2, W>(L, parity, omega, threadIdx.x, 32);
                    __syncwarp();
                }
        }
        __syncthreads();
        return;
    }
    for (int s = 0; s < nsm; ++s) {
        if (smoother == 0) {
            const T* phi[3] = {L.phi[0], L.phi[1], L.phi[2]};
            for (int w = threadIdx.x; w < n; w += blockDim.x) {
                int i, j, k;
                unflat3d(L.D, w, i, j, k);
                Nb nb = W ? make_nbw(L.D, i, j, k) : make_nb(L.D, i, j, k);
                if (W && wall_face(nb, 0)) {
                    L.tmp[0][w] = T(0);
                } else {
                    T Lp = face_L<T, DM, VISC, 0, 1, T, W>(phi, L.C, nb, L.dxsqinv, b, c);
                    T fac = face_diag<T, DM, VISC, 0, W>(L.C, nb, L.dxsqinv, b, c);
                    L.tmp[0][w] = L.phi[0][w] + omega * (L.rhs[0][w] - Lp) / fac;
                }
                if (W && wall_face(nb, 1)) {
                    L.tmp[1][w] = T(0);
                } else {
                    T Lp = face_L<T, DM, VISC, 1, 1, T, W>(phi, L.C, nb, L.dxsqinv, b, c);
                    T fac = face_diag<T, DM, VISC, 1, W>(L.C, nb, L.dxsqinv, b, c);
                    L.tmp[1][w] = L.phi[1][w] + omega * (L.rhs[1][w] - Lp) / fac;
                }
                if constexpr (DM == 3) {
                    if (W && wall_face(nb, 2)) {
                        L.tmp[2][w] = T(0);
                    } else {
                        T Lp = face_L<T, DM, VISC, 2, 1, T, W>(phi, L.C, nb, L.dxsqinv, b, c);
                        T fac = face_diag<T, DM, VISC, 2, W>(L.C, nb, L.dxsqinv, b, c);
                        L.tmp[2][w] = L.phi[2][w] + omega * (L.rhs[2][w] - Lp) / fac;
                    }
                }
            }
            __syncthreads();
            for (int w = threadIdx.x; w < n; w += blockDim.x)
                for (int d = 0; d < DM; ++d) L.phi[d][w] = L.tmp[d][w];
            __syncthreads();
        } else {
            for (int color = 1; color <= 2 * DM; ++color) {
                const int comp = (color - 1) / 2;
                const int parity = (color % 2 == 1) ? 0 : 1;
                if (odd_level(L.D)) {
                    if (comp == 0)
                        tail_colour_odd<T, DM, VISC, 0, W>(L, parity, omega);
                    else if (comp == 1)
                        tail_colour_odd<T, DM, VISC, 1, W>(L, parity, omega);
                    else if constexpr (DM == 3)
                        tail_colour_odd<T, DM, VISC, 2, W>(L, parity, omega);
                } else {
                    if (comp == 0)
                        tail_colour<T, DM, VISC, 0, W>(L, parity, omega, threadIdx.x, blockDim.x);
                    else if (comp == 1)
                        tail_colour<T, DM, VISC, 1, W>(L, parity, omega, threadIdx.x, blockDim.x);
                    else if constexpr (DM == 3)
                        tail_colour<T, DM, VISC, 2, W>(L, parity, omega, threadIdx.x, blockDim.x);
                }
                __syncthreads();
            }
        }
    }
}

// this block's offset into a level's arrays: 2D, instance blockIdx.x of
// the batch; 3D, none
template <int DM>
__device__ __forceinline__ int64_t inst_offset(const Dims& D) {
    return DM == 2 ? (int64_t)blockIdx.x * D.nx * D.ny : 0;
}
template <class T>
__device__ __forceinline__ const T* shift(const T* p, int64_t o) {
    return p ? p + o : p;
}

// carve the dynamic shared memory into per-level phi / rhs / (tmp) arrays
template <class T, int DM>
__device__ void tail_views(const TailArgs<T>& A, T* sm, TailView<T>* V, bool stag, bool jacobi) {
    const bool wall = A.L[0].D.wall != 0;  // wall levels hold the residual in tmp
    size_t off = 0;
    for (int l = 0; l < A.nl; ++l) {
        TailView<T>& v = V[l];
        v.D = A.L[l].D;
        v.dxsqinv = A.L[l].dxsqinv;
        v.C = A.L[l].C;
        const int64_t io = inst_offset<DM>(v.D);
        // an instance's edge array: n+1 nodes along a nodal wall-bounded direction
        const int64_t ie = DM == 2 ? (int64_t)blockIdx.x * edge_ext(v.D, 0, 0) * edge_ext(v.D, 0, 1) : 0;
        if (DM == 2) v.D.nz = 1;
        for (int d = 0; d < 3; ++d) {
            v.C.alpha[d] = shift(v.C.alpha[d], io);
            v.C.bed[d] = shift(v.C.bed[d], ie);
        }
        v.C.beta = shift(v.C.beta, io);
        v.C.gamma = shift(v.C.gamma, io);
        const int n = ncells(v.D);
        for (int d = 0; d < 3; ++d) {
            v.pa[d] = shift(A.L[l].pa[d], io);
            v.phi[d] = v.rhs[d] = v.tmp[d] = nullptr;
        }
        v.pphi = v.prhs = v.ptmp = nullptr;
        const bool odd = odd_level(v.D);
        if (stag) {
            for (int d = 0; d < DM; ++d) { v.phi[d] = sm + off; off += n; }
            for (int d = 0; d < DM; ++d) { v.rhs[d] = sm + off; off += n; }
            if (jacobi || odd || wall)
                for (int d = 0; d < DM; ++d) { v.tmp[d] = sm + off; off += n; }
        } else {
            v.pphi = sm + off; off += n;
            v.prhs = sm + off; off += n;
            if (odd) { v.ptmp = sm + off; off += n; }
        }
    }
}

// The coarse end of a staggered V-cycle.  In: the first tail level's rhs and
// phi (global); out: its phi (global).  Levels below are zeroed in shared
// memory.
template <class T, int DM, int VISC, bool W = false>
__global__ void __launch_bounds__(kTailThreads, 1) k_vcycle_tail(const __grid_constant__ TailArgs<T> A) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char tail_smem[];
    T* sm = reinterpret_cast<T*>(tail_smem);
    __shared__ TailView<T> V[kMaxTail];
    if (threadIdx.x == 0) tail_views<T, DM>(A, sm, V, true, A.smoother == 0);
    __syncthreads();
    const int64_t g0 = inst_offset<DM>(A.L[0].D);
    {
        const int n0 = ncells(V[0].D);
        for (int w = threadIdx.x; w < n0; w += blockDim.x)
            for (int d = 0; d < DM; ++d) {
                V[0].phi[d][w] = A.g_phi[d][g0 + w];
                V[0].rhs[d][w] = A.g_rhs[d][g0 + w];
            }
        for (int l = 1; l < A.nl; ++l) {
            const int n = ncells(V[l].D);
            for (int w = threadIdx.x; w < n; w += blockDim.x)
                for (int d = 0; d < DM; ++d) V[l].phi[d][w] = T(0);
        }
    }
    __syncthreads();
    for (int l = 0; l < A.nl - 1; ++l) {
        tail_smooth<T, DM, VISC, W>(V[l], A.nu1, A.smoother, A.omega);
        const TailView<T>& F = V[l];
        const TailView<T>& Cc = V[l + 1];
        const int nc = ncells(Cc.D);
        const T* rf[3] = {F.rhs[0], F.rhs[1], F.rhs[2]};
        const T* pf[3] = {F.phi[0], F.phi[1], F.phi[2]};
        if constexpr (W) {
            // the wall levels' residual_restrict: residual on every fine face
            // (zero on wall faces) into F.tmp, then the restriction
            const int nf = ncells(F.D);
            for (int w2 = threadIdx.x; w2 < nf * DM; w2 += blockDim.x) {
                const int comp = w2 / nf, w = w2 - comp * nf;
                int i, j, k;
                unflat3d(F.D, w, i, j, k);
                const Nb nb = make_nbw(F.D, i, j, k);
                const T b = ld(F.C.beta, 0), c = ld(F.C.gamma, 0);
                T v = T(0);
                if (comp == 0) {
                    if (!wall_face(nb, 0)) v = (face_L<T, DM, VISC, 0, 1, T, true>(pf, F.C, nb, F.dxsqinv, b, c) - rf[0][w]) * T(-1);
                } else if (comp == 1) {
                    if (!wall_face(nb, 1)) v = (face_L<T, DM, VISC, 1, 1, T, true>(pf, F.C, nb, F.dxsqinv, b, c) - rf[1][w]) * T(-1);
                } else if constexpr (DM == 3) {
                    if (!wall_face(nb, 2)) v = (face_L<T, DM, VISC, 2, 1, T, true>(pf, F.C, nb, F.dxsqinv, b, c) - rf[2][w]) * T(-1);
                }
                F.tmp[comp][w] = v;
            }
            __syncthreads();
            for (int w = threadIdx.x; w < nc; w += blockDim.x) {
                int i, j, k;
                unflat3d(Cc.D, w, i, j, k);
                restrict_cell<T, DM, true, 1>(F.D, F.tmp[0], F.tmp[1], F.tmp[2], Cc.D, Cc.rhs[0], Cc.rhs[1], Cc.rhs[2], i, j, k, w);
            }
        } else {
            for (int w2 = threadIdx.x; w2 < nc * DM; w2 += blockDim.x) {
                const int comp = w2 / nc, w = w2 - comp * nc;
                int i, j, k;
                unflat3d(Cc.D, w, i, j, k);
                restrict_comp<T, DM, VISC, 1>(comp, F.D, F.C, rf, pf, Cc.rhs, w, i, j, k, F.dxsqinv);
            }
        }
        __syncthreads();
    }
    tail_smooth<T, DM, VISC, W>(V[A.nl - 1], A.nub, A.smoother, A.omega);
    for (int l = A.nl - 2; l >= 0; --l) {
        const TailView<T>& F = V[l];
        const TailView<T>& Cc = V[l + 1];
        const int nf = ncells(F.D);
        for (int w = threadIdx.x; w < nf; w += blockDim.x) {
            int i, j, k;
            unflat3d(F.D, w, i, j, k);
            prolong_cell<T, DM, 1, W>(Cc.D, Cc.phi[0], Cc.phi[1], Cc.phi[2], F.phi[0], F.phi[1], F.phi[2], w, i, j, k);
        }
        __syncthreads();
        tail_smooth<T, DM, VISC, W>(F, A.nu2, A.smoother, A.omega);
    }
    const int n0 = ncells(V[0].D);
    for (int w = threadIdx.x; w < n0; w += blockDim.x)
        for (int d = 0; d < DM; ++d) A.g_phi[d][g0 + w] = V[0].phi[d][w];
}

// ------------------------------------------------------------------ pressure
template <class T, int DM>
__device__ void tail_cc_smooth(const TailView<T>& L, int nsweeps) {
    const int half = L.D.nx >> 1;
    const int count = half * L.D.ny * L.D.nz;
    if (odd_level(L.D)) {
        // odd level: each colour from the values before its pass
        const int n = ncells(L.D);
        for (int s = 0; s < nsweeps; ++s)
            for (int parity = 0; parity < 2; ++parity) {
                for (int w = threadIdx.x; w < n; w += blockDim.x) {
                    int i, j, k;
                    unflat3d(L.D, w, i, j, k);
                    if (((i + j + k) & 1) != parity) continue;
                    Nb nb = make_nb(L.D, i, j, k);
                    T res = L.prhs[nb.s] - cc_lap<T, DM, 1>(L.pa, L.pphi, nb, L.dxsqinv);
                    T cur = L.pphi[nb.s];
                    L.ptmp[w] = cur + res / cc_diag<T, DM>(L.pa, nb, L.dxsqinv);
                }
                __syncthreads();
                for (int w = threadIdx.x; w < n; w += blockDim.x) {
                    int i, j, k;
                    unflat3d(L.D, w, i, j, k);
                    if (((i + j + k) & 1) == parity) L.pphi[w] = L.ptmp[w];
                }
                __syncthreads();
            }
        return;
    }
    // at most 32 cells per colour: warp 0 takes every sweep, a __syncwarp
    // between colours instead of the block's barrier
    const bool narrow = count <= 32;
    if (narrow && threadIdx.x >= 32) {
        __syncthreads();
        return;
    }
    const int t0 = threadIdx.x, stride = narrow ? 32 : blockDim.x;
    for (int s = 0; s < nsweeps; ++s)
        for (int parity = 0; parity < 2; ++parity) {
            for (int w = t0; w < count; w += stride) {
                const int ih = w % half;
                const int q = w / half;
                const int j = q % L.D.ny, k = q / L.D.ny;
                const int i = 2 * ih + ((j + k + parity) & 1);
                Nb nb = make_nb(L.D, i, j, k);
                T res = L.prhs[nb.s] - cc_lap<T, DM, 1>(L.pa, L.pphi, nb, L.dxsqinv);
                T cur = L.pphi[nb.s];
                L.pphi[nb.s] = cur + res / cc_diag<T, DM>(L.pa, nb, L.dxsqinv);
            }
            if (narrow)
                __syncwarp();
            else
                __syncthreads();
        }
    if (narrow) __syncthreads();
}

template <class T, int DM>
__global__ void __launch_bounds__(kTailThreads, 1) k_ccmg_tail(const __grid_constant__ TailArgs<T> A) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char tail_smem[];
    T* sm = reinterpret_cast<T*>(tail_smem);
    __shared__ TailView<T> V[kMaxTail];
    if (threadIdx.x == 0) tail_views<T, DM>(A, sm, V, false, false);
    __syncthreads();
    const int64_t g0 = inst_offset<DM>(A.L[0].D);
    {
        const int n0 = ncells(V[0].D);
        for (int w = threadIdx.x; w < n0; w += blockDim.x) {
            V[0].pphi[w] = A.g_pphi[g0 + w];
            V[0].prhs[w] = A.g_prhs[g0 + w];
        }
        for (int l = 1; l < A.nl; ++l) {
            const int n = ncells(V[l].D);
            for (int w = threadIdx.x; w < n; w += blockDim.x) V[l].pphi[w] = T(0);
        }
    }
    __syncthreads();
    for (int l = 0; l < A.nl - 1; ++l) {
        tail_cc_smooth<T, DM>(V[l], A.nu1);
        const TailView<T>& F = V[l];
        const TailView<T>& Cc = V[l + 1];
        const int nc = ncells(Cc.D);
        for (int w = threadIdx.x; w < nc; w += blockDim.x) {
            int i, j, k;
            unflat3d(Cc.D, w, i, j, k);
            const int I = 2 * i, J = 2 * j, K = 2 * k;
#define R(ii, jj, kk) cc_res_at<T, DM, 1>(F.D, F.pa, F.pphi, F.prhs, ii, jj, kk, F.dxsqinv)
            if constexpr (DM == 2)
                Cc.prhs[w] = T(0.25) * (R(I, J, 0) + R(I + 1, J, 0) + R(I, J + 1, 0) + R(I + 1, J + 1, 0));
            else
                Cc.prhs[w] = T(0.125) * (R(I, J, K) + R(I + 1, J, K) + R(I, J + 1, K) + R(I + 1, J + 1, K) + R(I, J, K + 1) +
                                         R(I + 1, J, K + 1) + R(I, J + 1, K + 1) + R(I + 1, J + 1, K + 1));
#undef R
        }
        __syncthreads();
    }
    tail_cc_smooth<T, DM>(V[A.nl - 1], A.nub);
    for (int l = A.nl - 2; l >= 0; --l) {
        const TailView<T>& F = V[l];
        const TailView<T>& Cc = V[l + 1];
        const int nf = ncells(F.D);
        for (int w = threadIdx.x; w < nf; w += blockDim.x) {
            int i, j, k;
            unflat3d(F.D, w, i, j, k);
            F.pphi[w] = F.pphi[w] + Cc.pphi[(i >> 1) + Cc.D.nx * ((j >> 1) + Cc.D.ny * (k >> 1))];
        }
        __syncthreads();
        tail_cc_smooth<T, DM>(F, A.nu2);
    }
    const int n0 = ncells(V[0].D);
    for (int w = threadIdx.x; w < n0; w += blockDim.x) A.g_pphi[g0 + w] = V[0].pphi[w];
}

// ------------------------------------------------------------------ launchers
template <class T>
static TailArgs<T> tail_args(const LevelDev<T>* L, int nl, int nu1, int nu2, int nub, int smoother, double omega) {
    TailArgs<T> a;
    memset(&a, 0, sizeof(a));
    a.nl = nl;
    a.nu1 = nu1;
    a.nu2 = nu2;
    a.nub = nub;
    a.smoother = smoother;
    a.omega = (T)omega;
    for (int d = 0; d < 3; ++d) {
        a.g_phi[d] = L[0].phi[d];
        a.g_rhs[d] = L[0].rhs[d];
    }
    a.g_pphi = L[0].pphi;
    a.g_prhs = L[0].prhs;
    for (int l = 0; l < nl; ++l) {
        TailLevel<T>& t = a.L[l];
        t.D = L[l].D;
        t.dxsqinv = (T)(1.0 / (L[l].dx * L[l].dx));
        t.C = L[l].coef();
        for (int d = 0; d < 3; ++d) t.pa[d] = L[l].pa[d];
    }
    return a;
}

// shared memory of a tail over levels L[0..nl-1]
template <class T>
size_t tail_smem_bytes(const LevelDev<T>* L, int nl, bool stag, bool jacobi) {
    size_t e = 0;
    jacobi = jacobi || L[0].D.wall != 0;  // wall levels hold the residual in tmp as well
    for (int l = 0; l < nl; ++l) {
        const bool odd = odd_level(L[l].D);
        const size_t n = (size_t)L[l].n / (L[l].D.dm == 2 ? L[l].D.nz : 1);  // one instance
        e += n * (stag ? (size_t)L[l].D.dm * ((jacobi || odd) ? 3 : 2) : (odd ? 3 : 2));
    }
    return e * sizeof(T);
}

// the dynamic shared-memory limit is raised once per kernel (never while a
// stream is being captured into a graph: the first call always runs eagerly)
template <class K, class A>
static cudaError_t launch_tail(K kernel, const A& args, size_t smem, cudaStream_t s) {
    cudaError_t e = raise_smem_limit((const void*)kernel, smem);
    if (e != cudaSuccess) return e;
    // one block per instance of a 2D batch (nz instances), else one block
    const int blocks = args.L[0].D.dm == 2 ? args.L[0].D.nz : 1;
    launch_pdl(kernel, dim3(blocks), dim3(kTailThreads), smem, s, args);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_vcycle_tail(const LevelDev<T>* L, int nl, int visc, int nu1, int nu2, int nub, int smoother, double omega,
                               cudaStream_t s) {
    if (nl < 1 || nl > kMaxTail) return cudaErrorInvalidValue;
    TailArgs<T> a = tail_args<T>(L, nl, nu1, nu2, nub, smoother, omega);
    const size_t smem = tail_smem_bytes<T>(L, nl, true, smoother == 0);
    cudaError_t e = cudaErrorInvalidValue;
    const bool wall = L[0].D.wall != 0;
    if (L[0].D.dm == 2) {
        if (wall) {
            LMM_VISC_DISPATCH(visc, (e = launch_tail(k_vcycle_tail<T, 2, V, true>, a, smem, s)))
        } else {
            LMM_VISC_DISPATCH(visc, (e = launch_tail(k_vcycle_tail<T, 2, V>, a, smem, s)))
        }
    } else {
        if (wall) {
            LMM_VISC_DISPATCH(visc, (e = launch_tail(k_vcycle_tail<T, 3, V, true>, a, smem, s)))
        } else {
            LMM_VISC_DISPATCH(visc, (e = launch_tail(k_vcycle_tail<T, 3, V>, a, smem, s)))
        }
    }
    return e;
}

template <class T>
cudaError_t launch_ccmg_tail(const LevelDev<T>* L, int nl, int nu1, int nu2, int nub, cudaStream_t s) {
    if (nl < 1 || nl > kMaxTail) return cudaErrorInvalidValue;
    TailArgs<T> a = tail_args<T>(L, nl, nu1, nu2, nub, 1, 1.0);
    const size_t smem = tail_smem_bytes<T>(L, nl, false, false);
    if (L[0].D.dm == 2) return launch_tail(k_ccmg_tail<T, 2>, a, smem, s);
    return launch_tail(k_ccmg_tail<T, 3>, a, smem, s);
}

#define LMM_INSTANTIATE_TAIL(T)                                                                                       \
    template cudaError_t launch_vcycle_tail<T>(const LevelDev<T>*, int, int, int, int, int, int, double, cudaStream_t); \
    template cudaError_t launch_ccmg_tail<T>(const LevelDev<T>*, int, int, int, int, cudaStream_t);                   \
    template size_t tail_smem_bytes<T>(const LevelDev<T>*, int, bool, bool);

}  // namespace lmm
