// tail.cuh - the coarse end of the V-cycles in one launch.
//
// Every multigrid level below a size threshold (its smooths, residual
// restrictions, bottom smooths and prolongations: stag_mg_solver.f90:338-760
// for the velocity, and this library's cell-centred pressure V-cycle) runs
// inside ONE kernel made of a single thread-block cluster.  The steps are
// separated by hardware cluster barriers instead of kernel boundaries, so
// the ~30 launches per coarse level collapse into one.  Arrays the kernel
// writes (phi, rhs, Jacobi scratch) are read through L2 (ld.global.cg): the
// blocks of the cluster sit on different SMs whose L1 caches are not
// coherent.  Arithmetic is the same device code as the per-level kernels,
// so results are bit-identical.
#pragma once
#include <cooperative_groups.h>

#include <cstring>

#include "kernels.cuh"

namespace lmm {

namespace cg = cooperative_groups;

constexpr int kTailThreads = 512;
constexpr int kMaxTail = 12;

template <class T>
struct TailLevel {
    Dims D;
    T dxsqinv;
    Coef<T> C;
    T* phi[3];
    T* rhs[3];
    T* tmp[3];
    const T* pa[3];
    T* pphi;
    T* prhs;
};

template <class T>
struct TailArgs {
    int nl;
    int nu1, nu2, nub, smoother;
    T omega;
    TailLevel<T> L[kMaxTail];
};

struct Team {
    int rank, size;
};

__device__ __forceinline__ Team team() {
    cg::cluster_group cl = cg::this_cluster();
    Team t;
    t.rank = (int)(cl.block_rank() * blockDim.x + threadIdx.x);
    t.size = (int)(cl.num_blocks() * blockDim.x);
    return t;
}
__device__ __forceinline__ void tsync() { cg::this_cluster().sync(); }

__device__ __forceinline__ void unflat3d(const Dims& D, int w, int& i, int& j, int& k) {
    i = w % D.nx;
    int r = w / D.nx;
    j = r % D.ny;
    k = r / D.ny;
}

template <class T, int DM, int VISC, int COMP>
__device__ __forceinline__ void tail_colour(const TailLevel<T>& L, int parity, T omega, const Team& tm) {
    const T b = ld(L.C.beta, 0), c = ld(L.C.gamma, 0);
    const int half = L.D.nx >> 1;
    const int count = half * L.D.ny * L.D.nz;
    const T* phi[3] = {L.phi[0], L.phi[1], L.phi[2]};
    T* p = L.phi[COMP];
    const T* r = L.rhs[COMP];
    for (int w = tm.rank; w < count; w += tm.size) {
        const int ih = w % half;
        const int q = w / half;
        const int j = q % L.D.ny, k = q / L.D.ny;
        const int i = 2 * ih + ((j + k + parity) & 1);
        Nb nb = make_nb(L.D, i, j, k);
        T Lp = face_L<T, DM, VISC, COMP, 2>(phi, L.C, nb, L.dxsqinv, b, c);
        T fac = face_diag<T, DM, VISC, COMP>(L.C, nb, L.dxsqinv, b, c);
        T cur = __ldcg(p + nb.s);
        p[nb.s] = cur + omega * (__ldcg(r + nb.s) - Lp) / fac;
    }
}

template <class T, int DM, int VISC>
__device__ void tail_smooth(const TailLevel<T>& L, int nsm, int smoother, T omega, const Team& tm) {
    const T b = ld(L.C.beta, 0), c = ld(L.C.gamma, 0);
    const int n = L.D.nx * L.D.ny * L.D.nz;
    for (int s = 0; s < nsm; ++s) {
        if (smoother == 0) {
            const T* phi[3] = {L.phi[0], L.phi[1], L.phi[2]};
            for (int w = tm.rank; w < n; w += tm.size) {
                int i, j, k;
                unflat3d(L.D, w, i, j, k);
                Nb nb = make_nb(L.D, i, j, k);
                {
                    T Lp = face_L<T, DM, VISC, 0, 2>(phi, L.C, nb, L.dxsqinv, b, c);
                    T fac = face_diag<T, DM, VISC, 0>(L.C, nb, L.dxsqinv, b, c);
                    L.tmp[0][w] = __ldcg(L.phi[0] + w) + omega * (__ldcg(L.rhs[0] + w) - Lp) / fac;
                }
                {
                    T Lp = face_L<T, DM, VISC, 1, 2>(phi, L.C, nb, L.dxsqinv, b, c);
                    T fac = face_diag<T, DM, VISC, 1>(L.C, nb, L.dxsqinv, b, c);
                    L.tmp[1][w] = __ldcg(L.phi[1] + w) + omega * (__ldcg(L.rhs[1] + w) - Lp) / fac;
                }
                if constexpr (DM == 3) {
                    T Lp = face_L<T, DM, VISC, 2, 2>(phi, L.C, nb, L.dxsqinv, b, c);
                    T fac = face_diag<T, DM, VISC, 2>(L.C, nb, L.dxsqinv, b, c);
                    L.tmp[2][w] = __ldcg(L.phi[2] + w) + omega * (__ldcg(L.rhs[2] + w) - Lp) / fac;
                }
            }
            tsync();
            for (int w = tm.rank; w < n; w += tm.size)
                for (int d = 0; d < DM; ++d) L.phi[d][w] = __ldcg(L.tmp[d] + w);
            tsync();
        } else {
            for (int color = 1; color <= 2 * DM; ++color) {
                const int comp = (color - 1) / 2;
                const int parity = (color % 2 == 1) ? 0 : 1;
                if (comp == 0)
                    tail_colour<T, DM, VISC, 0>(L, parity, omega, tm);
                else if (comp == 1)
                    tail_colour<T, DM, VISC, 1>(L, parity, omega, tm);
                else if constexpr (DM == 3)
                    tail_colour<T, DM, VISC, 2>(L, parity, omega, tm);
                tsync();
            }
        }
    }
}

// The coarse end of a staggered V-cycle: A.L[0] holds rhs (and the current
// phi of its level); levels 1.. are zeroed here.
template <class T, int DM, int VISC>
__global__ void __launch_bounds__(kTailThreads) k_vcycle_tail(const __grid_constant__ TailArgs<T> A) {
    const Team tm = team();
    for (int l = 1; l < A.nl; ++l) {
        const int n = A.L[l].D.nx * A.L[l].D.ny * A.L[l].D.nz;
        for (int w = tm.rank; w < n; w += tm.size)
            for (int d = 0; d < DM; ++d) A.L[l].phi[d][w] = T(0);
    }
    tsync();
    for (int l = 0; l < A.nl - 1; ++l) {
        tail_smooth<T, DM, VISC>(A.L[l], A.nu1, A.smoother, A.omega, tm);
        const TailLevel<T>& F = A.L[l];
        const TailLevel<T>& Cc = A.L[l + 1];
        const int nc = Cc.D.nx * Cc.D.ny * Cc.D.nz;
        const T* rf[3] = {F.rhs[0], F.rhs[1], F.rhs[2]};
        const T* pf[3] = {F.phi[0], F.phi[1], F.phi[2]};
        for (int w2 = tm.rank; w2 < nc * DM; w2 += tm.size) {
            const int comp = w2 / nc, w = w2 - comp * nc;
            int i, j, k;
            unflat3d(Cc.D, w, i, j, k);
            restrict_comp<T, DM, VISC, 2>(comp, F.D, F.C, rf, pf, Cc.rhs, w, i, j, k, F.dxsqinv);
        }
        tsync();
    }
    tail_smooth<T, DM, VISC>(A.L[A.nl - 1], A.nub, A.smoother, A.omega, tm);
    for (int l = A.nl - 2; l >= 0; --l) {
        const TailLevel<T>& F = A.L[l];
        const TailLevel<T>& Cc = A.L[l + 1];
        const int nf = F.D.nx * F.D.ny * F.D.nz;
        for (int w = tm.rank; w < nf; w += tm.size) {
            int i, j, k;
            unflat3d(F.D, w, i, j, k);
            prolong_cell<T, DM, 2>(Cc.D, Cc.phi[0], Cc.phi[1], Cc.phi[2], F.phi[0], F.phi[1], F.phi[2], w, i, j, k);
        }
        tsync();
        tail_smooth<T, DM, VISC>(F, A.nu2, A.smoother, A.omega, tm);
    }
}

// ------------------------------------------------------------------ pressure
template <class T, int DM>
__device__ void tail_cc_smooth(const TailLevel<T>& L, int nsweeps, const Team& tm) {
    const int half = L.D.nx >> 1;
    const int count = half * L.D.ny * L.D.nz;
    for (int s = 0; s < nsweeps; ++s)
        for (int parity = 0; parity < 2; ++parity) {
            for (int w = tm.rank; w < count; w += tm.size) {
                const int ih = w % half;
                const int q = w / half;
                const int j = q % L.D.ny, k = q / L.D.ny;
                const int i = 2 * ih + ((j + k + parity) & 1);
                Nb nb = make_nb(L.D, i, j, k);
                T res = __ldcg(L.prhs + nb.s) - cc_lap<T, DM, 2>(L.pa, L.pphi, nb, L.dxsqinv);
                T cur = __ldcg(L.pphi + nb.s);
                L.pphi[nb.s] = cur + res / cc_diag<T, DM>(L.pa, nb, L.dxsqinv);
            }
            tsync();
        }
}

template <class T, int DM>
__global__ void __launch_bounds__(kTailThreads) k_ccmg_tail(const __grid_constant__ TailArgs<T> A) {
    const Team tm = team();
    for (int l = 1; l < A.nl; ++l) {
        const int n = A.L[l].D.nx * A.L[l].D.ny * A.L[l].D.nz;
        for (int w = tm.rank; w < n; w += tm.size) A.L[l].pphi[w] = T(0);
    }
    tsync();
    for (int l = 0; l < A.nl - 1; ++l) {
        tail_cc_smooth<T, DM>(A.L[l], A.nu1, tm);
        const TailLevel<T>& F = A.L[l];
        const TailLevel<T>& Cc = A.L[l + 1];
        const int nc = Cc.D.nx * Cc.D.ny * Cc.D.nz;
        for (int w = tm.rank; w < nc; w += tm.size) {
            int i, j, k;
            unflat3d(Cc.D, w, i, j, k);
            const int I = 2 * i, J = 2 * j, K = 2 * k;
#define R(ii, jj, kk) cc_res_at<T, DM, 2>(F.D, F.pa, F.pphi, F.prhs, ii, jj, kk, F.dxsqinv)
            if constexpr (DM == 2)
                Cc.prhs[w] = T(0.25) * (R(I, J, 0) + R(I + 1, J, 0) + R(I, J + 1, 0) + R(I + 1, J + 1, 0));
            else
                Cc.prhs[w] = T(0.125) * (R(I, J, K) + R(I + 1, J, K) + R(I, J + 1, K) + R(I + 1, J + 1, K) + R(I, J, K + 1) +
                                         R(I + 1, J, K + 1) + R(I, J + 1, K + 1) + R(I + 1, J + 1, K + 1));
#undef R
        }
        tsync();
    }
    tail_cc_smooth<T, DM>(A.L[A.nl - 1], A.nub, tm);
    for (int l = A.nl - 2; l >= 0; --l) {
        const TailLevel<T>& F = A.L[l];
        const TailLevel<T>& Cc = A.L[l + 1];
        const int nf = F.D.nx * F.D.ny * F.D.nz;
        for (int w = tm.rank; w < nf; w += tm.size) {
            int i, j, k;
            unflat3d(F.D, w, i, j, k);
            F.pphi[w] = __ldcg(F.pphi + w) + __ldcg(Cc.pphi + ((i >> 1) + Cc.D.nx * ((j >> 1) + Cc.D.ny * (k >> 1))));
        }
        tsync();
        tail_cc_smooth<T, DM>(F, A.nu2, tm);
    }
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
    for (int l = 0; l < nl; ++l) {
        TailLevel<T>& t = a.L[l];
        t.D = L[l].D;
        t.dxsqinv = (T)(1.0 / (L[l].dx * L[l].dx));
        t.C = L[l].coef();
        for (int d = 0; d < 3; ++d) {
            t.phi[d] = L[l].phi[d];
            t.rhs[d] = L[l].rhs[d];
            t.tmp[d] = L[l].tmp[d];
            t.pa[d] = L[l].pa[d];
        }
        t.pphi = L[l].pphi;
        t.prhs = L[l].prhs;
    }
    return a;
}

template <class K, class A>
static cudaError_t launch_cluster(K kernel, const A& args, int csize, cudaStream_t s) {
    if (csize > 8) {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(csize, 1, 1);
    cfg.blockDim = dim3(kTailThreads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args);
}

template <class T>
cudaError_t launch_vcycle_tail(const LevelDev<T>* L, int nl, int visc, int nu1, int nu2, int nub, int smoother, double omega,
                               int csize, cudaStream_t s) {
    if (nl < 1 || nl > kMaxTail) return cudaErrorInvalidValue;
    TailArgs<T> a = tail_args<T>(L, nl, nu1, nu2, nub, smoother, omega);
    cudaError_t e = cudaErrorInvalidValue;
    if (L[0].D.dm == 2) {
        LMM_VISC_DISPATCH(visc, (e = launch_cluster(k_vcycle_tail<T, 2, V>, a, csize, s)))
    } else {
        LMM_VISC_DISPATCH(visc, (e = launch_cluster(k_vcycle_tail<T, 3, V>, a, csize, s)))
    }
    return e;
}

template <class T>
cudaError_t launch_ccmg_tail(const LevelDev<T>* L, int nl, int nu1, int nu2, int nub, int csize, cudaStream_t s) {
    if (nl < 1 || nl > kMaxTail) return cudaErrorInvalidValue;
    TailArgs<T> a = tail_args<T>(L, nl, nu1, nu2, nub, 1, 1.0);
    if (L[0].D.dm == 2) return launch_cluster(k_ccmg_tail<T, 2>, a, csize, s);
    return launch_cluster(k_ccmg_tail<T, 3>, a, csize, s);
}

#define LMM_INSTANTIATE_TAIL(T)                                                                                       \
    template cudaError_t launch_vcycle_tail<T>(const LevelDev<T>*, int, int, int, int, int, int, double, int,          \
                                               cudaStream_t);                                                          \
    template cudaError_t launch_ccmg_tail<T>(const LevelDev<T>*, int, int, int, int, int, cudaStream_t);

}  // namespace lmm
