// kernels.cuh - implementations of the staggered Stokes kernels (templated on
// the arithmetic type).  Included once per precision by kernels_fp64.cu and
// kernels_fp32.cu, which instantiate the launchers of kernels.h.
//
// Reference loops restated (compact periodic layout, no ghost cells):
//   stag_applyop_2d/_3d        src_common/stag_applyop.f90:204-1067
//   stag_mg_update (+colours)  src_gmres/stag_mg_solver.f90:1637-2463
//   residual + stag_restriction src_gmres/stag_mg_solver.f90:406-437, 1033-1175
//   stag_prolongation          src_gmres/stag_mg_solver.f90:1424-1633
//   coefficient coarsening     src_gmres/stag_mg_solver.f90:214-230, 873-968,
//                              1229-1244, 1326-1367
//   compute_div / compute_grad src_common/div_and_grad.f90:16-455
//   subtract_weighted_gradp    src_gmres/macproject.f90:320-364
//   norms / sum_umac_press     src_gmres/norm_inner_product.f90:16-794
// The pressure multigrid kernels (cc_*) are this library's own cell-centred
// V-cycle (the reference delegates to BoxLib F_MG, which it does not ship).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "kernels.h"
#include "pdl.cuh"
#include "stencil.cuh"

namespace lmm {

constexpr int kThreads = 256;


static inline int nblocks_for(int64_t n, int threads = kThreads) {
    int64_t b = (n + threads - 1) / threads;
    return (int)(b < 1 ? 1 : b);
}

// 3D launch: x spans nx (i, or i/2 for a colour), y spans ny, z spans nz
struct G3 {
    dim3 grid, block;
};
static inline G3 geom3(int nx, int ny, int nz) {
    int bx = nx < 64 ? nx : 64;
    if (bx < 1) bx = 1;
    int by = kThreads / bx;
    if (by > ny) by = ny;
    if (by < 1) by = 1;
    G3 g;
    g.block = dim3(bx, by, 1);
    g.grid = dim3((nx + bx - 1) / bx, (ny + by - 1) / by, nz);
    return g;
}

// the geometry of a tuned kernel: a shape forced by the autotuner while it
// times candidates, else the shape it chose for this grid, else geom3's
static inline G3 geom3_shape(int nx, int ny, int nz, Shape s) {
    G3 g;
    const int bx = std::max(1, std::min(s.bx, nx)), by = std::max(1, std::min(s.by, ny));
    g.block = dim3(bx, by, 1);
    g.grid = dim3((nx + bx - 1) / bx, (ny + by - 1) / by, nz);
    return g;
}
static inline G3 geom3_tuned(int kernel, int wbytes, int visc, const Dims& D, int nx, int ny, int nz) {
    Shape s = forced_shape();
    if (!s.bx) s = tuned_shape(kernel, wbytes, visc, D);
    return s.bx ? geom3_shape(nx, ny, nz, s) : geom3(nx, ny, nz);
}

// --------------------------------------------------------------- applyop
// W: a grid with walls; L phi is zero on the wall faces (stag_applyop.f90:197-201)
template <class T, int DM, int VISC, bool W = false>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 5 : 0) k_applyop(Dims D, Coef<T> C, const T* __restrict__ p0, const T* __restrict__ p1,
                                                      const T* __restrict__ p2, T* __restrict__ o0, T* __restrict__ o1,
                                                      T* __restrict__ o2, T dxsqinv, int color) {
    pdl_enter();
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok) return;
    const int i = q.i, j = q.j, k = q.k;
    Nb nb = W ? make_nbw(D, i, j, k) : make_nb(D, i, j, k);
    const int t = nb.s;
    const T* phi[3] = {p0, p1, p2};
    const T b = ld(C.beta, 0), c = ld(C.gamma, 0);
    // colour c >= 1 covers component (c-1)/2, faces with (i+j+k) even for odd c
    const int ccomp = (color - 1) / 2;
    const bool on = (color == 0) || ((((i + j + ck<DM>(k)) & 1) == ((color % 2 == 1) ? 0 : 1)));
    if (color == 0 || (ccomp == 0 && on)) o0[t] = (W && wall_face(nb, 0)) ? T(0) : face_L<T, DM, VISC, 0, 0, T, W>(phi, C, nb, dxsqinv, b, c);
    if (color == 0 || (ccomp == 1 && on)) o1[t] = (W && wall_face(nb, 1)) ? T(0) : face_L<T, DM, VISC, 1, 0, T, W>(phi, C, nb, dxsqinv, b, c);
    if constexpr (DM == 3)
        if (color == 0 || (ccomp == 2 && on)) o2[t] = (W && wall_face(nb, 2)) ? T(0) : face_L<T, DM, VISC, 2, 0, T, W>(phi, C, nb, dxsqinv, b, c);
}

// --------------------------------------------------------------- one component per thread
// The same face values as k_applyop (colour 0) and k_residual with one face
// component per thread: grid.z covers nz * DM, component = blockIdx.z % DM
// (uniform per block), so a thread keeps one stencil live instead of DM.
struct PosC {
    int i, j, k, comp;
    bool ok;
};
template <int DM>
__device__ __forceinline__ PosC posc(int nx, int ny) {
    PosC p;
    p.i = blockIdx.x * blockDim.x + threadIdx.x;
    p.j = blockIdx.y * blockDim.y + threadIdx.y;
    p.k = blockIdx.z / DM;
    p.comp = blockIdx.z - p.k * DM;
    p.ok = (p.i < nx) && (p.j < ny);
    return p;
}

template <class T, int DM, int VISC, bool W = false>
__global__ void __launch_bounds__(kThreads) k_applyop_c(Dims D, Coef<T> C, const T* __restrict__ p0, const T* __restrict__ p1,
                                                        const T* __restrict__ p2, T* __restrict__ o0, T* __restrict__ o1,
                                                        T* __restrict__ o2, T dxsqinv) {
    pdl_enter();
    const PosC q = posc<DM>(D.nx, D.ny);
    if (!q.ok) return;
    Nb nb = W ? make_nbw(D, q.i, q.j, q.k) : make_nb(D, q.i, q.j, q.k);
    const int t = nb.s;
    const T* phi[3] = {p0, p1, p2};
    const T b = ld(C.beta, 0), c = ld(C.gamma, 0);
    if (q.comp == 0) {
        o0[t] = (W && wall_face(nb, 0)) ? T(0) : face_L<T, DM, VISC, 0, 0, T, W>(phi, C, nb, dxsqinv, b, c);
    } else if (q.comp == 1) {
        o1[t] = (W && wall_face(nb, 1)) ? T(0) : face_L<T, DM, VISC, 1, 0, T, W>(phi, C, nb, dxsqinv, b, c);
    } else if constexpr (DM == 3) {
        o2[t] = (W && wall_face(nb, 2)) ? T(0) : face_L<T, DM, VISC, 2, 0, T, W>(phi, C, nb, dxsqinv, b, c);
    }
}

template <class T, int DM, int VISC, bool W = false>
__global__ void __launch_bounds__(kThreads) k_residual_c(Dims D, Coef<T> C, const T* __restrict__ r0, const T* __restrict__ r1,
                                                         const T* __restrict__ r2, const T* __restrict__ p0, const T* __restrict__ p1,
                                                         const T* __restrict__ p2, T* __restrict__ o0, T* __restrict__ o1,
                                                         T* __restrict__ o2, T dxsqinv) {
    pdl_enter();
    const PosC q = posc<DM>(D.nx, D.ny);
    if (!q.ok) return;
    Nb nb = W ? make_nbw(D, q.i, q.j, q.k) : make_nb(D, q.i, q.j, q.k);
    const int t = nb.s;
    const T* phi[3] = {p0, p1, p2};
    const T b = ld(C.beta, 0), c = ld(C.gamma, 0);
    if (q.comp == 0) {
        if (W && wall_face(nb, 0)) {
            o0[t] = T(0);
        } else {
            T v = face_L<T, DM, VISC, 0, 0, T, W>(phi, C, nb, dxsqinv, b, c) - ld(r0, t);
            o0[t] = v * T(-1);
        }
    } else if (q.comp == 1) {
        if (W && wall_face(nb, 1)) {
            o1[t] = T(0);
        } else {
            T v = face_L<T, DM, VISC, 1, 0, T, W>(phi, C, nb, dxsqinv, b, c) - ld(r1, t);
            o1[t] = v * T(-1);
        }
    } else if constexpr (DM == 3) {
        if (W && wall_face(nb, 2)) {
            o2[t] = T(0);
        } else {
            T v = face_L<T, DM, VISC, 2, 0, T, W>(phi, C, nb, dxsqinv, b, c) - ld(r2, t);
            o2[t] = v * T(-1);
        }
    }
}

// --------------------------------------------------------------- GS colour
// One colour of stag_applyop_level(color) + stag_mg_update(color): faces of
// component COMP with (i+j+k) % 2 == parity are updated in place.  Faces of
// one colour never read each other (even cell counts), so the in-place
// update equals the reference's compute-all-then-update order.
// W: wall faces keep their zero (physbc_domainvel after every colour)
// reverse: the blocks take the planes (the instances of a 2D batch) in
// decreasing order, so a launch that follows one in increasing order starts
// on the planes whose operands that launch left in L2 (the faces of one
// colour are independent: the order changes no value)
template <class T, int DM, int VISC, int COMP, bool W = false>
__global__ void __launch_bounds__(kThreads) k_gs_colour(Dims D, Coef<T> C, const T* __restrict__ rhs, T* p0, T* p1, T* p2,
                                                        int parity, T omega, T dxsqinv, int reverse) {
    pdl_enter();
    const Pos q = pos3(D.nx >> 1, D.ny);
    if (!q.ok) return;
    const int j = q.j, k = reverse ? (int)gridDim.z - 1 - q.k : q.k;
    const int i = 2 * q.i + ((j + ck<DM>(k) + parity) & 1);
    Nb nb = W ? make_nbw(D, i, j, k) : make_nb(D, i, j, k);
    if (W && wall_face(nb, COMP)) return;
    const T* phi[3] = {p0, p1, p2};
    const T b = ld(C.beta, 0), c = ld(C.gamma, 0);
    T* p = (COMP == 0) ? p0 : (COMP == 1 ? p1 : p2);
    if constexpr (DM == 3 && !W) {
        p[nb.s] = face_update3<T, VISC, COMP>(phi, C, rhs, nb, dxsqinv, b, c, omega);
    } else {
        T Lp = face_L<T, DM, VISC, COMP, 0, T, W>(phi, C, nb, dxsqinv, b, c);
        T fac = face_diag<T, DM, VISC, COMP, W>(C, nb, dxsqinv, b, c);
        T cur = p[nb.s];
        p[nb.s] = cur + omega * (ld(rhs, nb.s) - Lp) / fac;
    }
}

// --------------------------------------------------------------- odd levels
// A level with an odd cell count (only a coarsest level can have one) lets
// two faces of the same colour be periodic neighbours, so a colour is
// applied as the reference writes it: L phi of the colour's faces first
// (stag_applyop_level with the colour), then every update from those values
// (stag_mg_update).
__host__ __device__ __forceinline__ bool odd_level(const Dims& D) {
    return (D.nx & 1) || (D.ny & 1) || (D.dm == 3 && (D.nz & 1));
}

template <class T, int DM, int VISC, int COMP, bool W = false>
__global__ void __launch_bounds__(kThreads) k_colour_update(Dims D, Coef<T> C, const T* __restrict__ rhs, const T* __restrict__ Lp,
                                                            T* p, int parity, T omega, T dxsqinv) {
    pdl_enter();
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok || ((q.i + q.j + ck<DM>(q.k)) & 1) != parity) return;
    Nb nb = W ? make_nbw(D, q.i, q.j, q.k) : make_nb(D, q.i, q.j, q.k);
    if (W && wall_face(nb, COMP)) return;
    const T b = ld(C.beta, 0), c = ld(C.gamma, 0);
    T fac = face_diag<T, DM, VISC, COMP, W>(C, nb, dxsqinv, b, c);
    T cur = p[nb.s];
    p[nb.s] = cur + omega * (ld(rhs, nb.s) - ld(Lp, nb.s)) / fac;
}

// --------------------------------------------------------------- GS red/black pair (3D)
// Both colours of one component in one launch (colours 2*COMP+1 and
// 2*COMP+2 of the sweep above, same arithmetic).  The block owns a
// TX x TY x TZ tile.  Phase 1 updates the faces of parity par0 ("red") on the
// tile, on the one-face rings around each of its planes and on the planes
// just below and above it, into shared memory; phase 2, after one barrier,
// updates the other parity ("black"), whose six same-component neighbours are
// all red and all in shared memory.  Red values depend only on the input
// buffers, so a face computed by two blocks has the same bits in both.
//
// The update is out of place: every input (p0, p1, p2) is read-only and the
// new values of component COMP (both parities) go to `out`, so one pair
// reads each array once instead of once per colour.
template <class T, int VISC, int COMP>
__global__ void __launch_bounds__(kThreads) k_gs_pair(Dims D, Coef<T> C, const T* __restrict__ rhs, const T* __restrict__ p0,
                                                      const T* __restrict__ p1, const T* __restrict__ p2, T* __restrict__ out,
                                                      int TX, int TY, int TZ, int par0, T omega, T dxsqinv) {
    extern __shared__ __align__(16) unsigned char pair_smem[];
    T* red = reinterpret_cast<T*>(pair_smem);   // (TZ+2) planes of (TY+2) x (TX+2)
    const int W = TX + 2, PL = (TY + 2) * W;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * blockDim.x + tx;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY, k0 = blockIdx.z * TZ;
    const T* phi[3] = {p0, p1, p2};
    const T* pc = phi[COMP];
    const T b = ld(C.beta, 0), c = ld(C.gamma, 0);
    const int j = j0 + ty;
    // phase 1: red faces (two planes in flight per thread)
#pragma unroll 2
    for (int kk = 0; kk < TZ + 2; ++kk) {
        const int k = wrapi(k0 - 1 + kk, D.nz);
        T* slot = red + kk * PL;
        {
            const int x = 2 * tx + ((par0 + j + k) & 1);
            const Nb nb = make_nb(D, i0 + x, j, k);
            const T Lp = face_L3<T, VISC, COMP>(phi, C, nb, dxsqinv, b, c);
            const T fac = face_diag3<T, VISC, COMP>(C, nb, dxsqinv, b, c);
            const T v = ld(pc, nb.s) + omega * (ld(rhs, nb.s) - Lp) / fac;
            slot[(ty + 1) * W + x + 1] = v;
            if (kk >= 1 && kk <= TZ) out[nb.s] = v;
        }
        if (kk >= 1 && kk <= TZ && tid < TX + TY) {   // rings y = -1, y = TY, x = -1, x = TX
            int x, y;
            if (tid < TX) {
                const bool lo = tid < TX / 2;
                y = lo ? -1 : TY;
                x = 2 * (lo ? tid : tid - TX / 2) + ((par0 + j0 + y + k) & 1);
            } else {
                const int r = tid - TX;
                const bool lo = r < TY / 2;
                x = lo ? -1 : TX;
                y = 2 * (lo ? r : r - TY / 2) + ((par0 + i0 + x + j0 + k) & 1);
            }
            const Nb nb = make_nb(D, wrapi(i0 + x, D.nx), wrapi(j0 + y, D.ny), k);
            const T Lp = face_L3<T, VISC, COMP>(phi, C, nb, dxsqinv, b, c);
            const T fac = face_diag3<T, VISC, COMP>(C, nb, dxsqinv, b, c);
            slot[(y + 1) * W + x + 1] = ld(pc, nb.s) + omega * (ld(rhs, nb.s) - Lp) / fac;
        }
    }
    __syncthreads();
    // phase 2: black faces of the TZ planes
#pragma unroll 2
    for (int kk = 1; kk <= TZ; ++kk) {
        const int k = wrapi(k0 - 1 + kk, D.nz);
        const int x = 2 * tx + ((par0 + 1 + j + k) & 1);
        const T* sc = red + kk * PL;
        const int o = (ty + 1) * W + x + 1;
        const Nb nb = make_nb(D, i0 + x, j, k);
        const T nbv[6] = {sc[o + 1], sc[o - 1], sc[o + W], sc[o - W], sc[o + PL], sc[o - PL]};
        const T cur = ld(pc, nb.s);
        const T Lp = face_L3_own<T, VISC, COMP>(cur, nbv, phi, C, nb, dxsqinv, b, c);
        const T fac = face_diag3<T, VISC, COMP>(C, nb, dxsqinv, b, c);
        out[nb.s] = cur + omega * (ld(rhs, nb.s) - Lp) / fac;
    }
}

// --------------------------------------------------------------- Jacobi
template <class T, int DM, int VISC, bool W = false>
__global__ void __launch_bounds__(kThreads) k_jacobi(Dims D, Coef<T> C, const T* __restrict__ r0, const T* __restrict__ r1,
                                                     const T* __restrict__ r2, const T* __restrict__ p0, const T* __restrict__ p1,
                                                     const T* __restrict__ p2, T* __restrict__ o0, T* __restrict__ o1,
                                                     T* __restrict__ o2, T omega, T dxsqinv) {
    pdl_enter();
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok) return;
    Nb nb = W ? make_nbw(D, q.i, q.j, q.k) : make_nb(D, q.i, q.j, q.k);
    const int t = nb.s;
    const T* phi[3] = {p0, p1, p2};
    const T b = ld(C.beta, 0), c = ld(C.gamma, 0);
    if (W && wall_face(nb, 0)) {
        o0[t] = T(0);
    } else {
        T Lp = face_L<T, DM, VISC, 0, 0, T, W>(phi, C, nb, dxsqinv, b, c);
        T fac = face_diag<T, DM, VISC, 0, W>(C, nb, dxsqinv, b, c);
        o0[t] = ld(p0, t) + omega * (ld(r0, t) - Lp) / fac;
    }
    if (W && wall_face(nb, 1)) {
        o1[t] = T(0);
    } else {
        T Lp = face_L<T, DM, VISC, 1, 0, T, W>(phi, C, nb, dxsqinv, b, c);
        T fac = face_diag<T, DM, VISC, 1, W>(C, nb, dxsqinv, b, c);
        o1[t] = ld(p1, t) + omega * (ld(r1, t) - Lp) / fac;
    }
    if constexpr (DM == 3) {
        if (W && wall_face(nb, 2)) {
            o2[t] = T(0);
        } else {
            T Lp = face_L<T, DM, VISC, 2, 0, T, W>(phi, C, nb, dxsqinv, b, c);
            T fac = face_diag<T, DM, VISC, 2, W>(C, nb, dxsqinv, b, c);
            o2[t] = ld(p2, t) + omega * (ld(r2, t) - Lp) / fac;
        }
    }
}

// --------------------------------------------------------------- residual + restriction
// residual of one fine face: (L phi - rhs) * -1  (stag_mg_solver.f90:414-415)
template <class T, int DM, int VISC, int D_, int LD = 0>
__device__ __forceinline__ T fine_resid(const Dims& F, const Coef<T>& C, const T* const phi[3], const T* rhs, int i, int j, int k,
                                        T dxsqinv, T b, T c) {
    i = wrapi(i, F.nx);
    j = wrapi(j, F.ny);
    k = (DM == 3) ? wrapi(k, F.nz) : k;
    Nb nb = make_nb(F, i, j, k);
    T v = face_L<T, DM, VISC, D_, LD>(phi, C, nb, dxsqinv, b, c) - ldp<LD>(rhs, nb.s);
    return v * T(-1);
}

// coarse face of component COMP at coarse index (i, j, k): the fine-level
// residual restricted with the 6-point (2D) / 12-point (3D) stencil.  The 12
// (6) fine residuals are evaluated one at a time (keeps registers low) and
// summed in the reference's order:
//   3D: 1/8 (r0+r1+r2+r3) + 1/16 (r4+r5+r6+r7) + 1/16 (r8+r9+r10+r11)
//   2D: 1/4 (r0+r1) + 1/8 (r2+r3+r4+r5)
// with normal offsets 0, +1, -1 and the transverse offsets of
// stag_mg_solver.f90:1063-1078, 1133-1171.
template <class T, int DM, int VISC, int COMP, int LD = 0>
__device__ __forceinline__ T restrict_face(const Dims& F, const Coef<T>& C, const T* const rhs[3], const T* const phi[3], int i,
                                           int j, int k, T dxsqinv) {
    const T b = ld(C.beta, 0), cc = ld(C.gamma, 0);
    constexpr int NQ = (DM == 2) ? 2 : 4;
    // transverse offsets (di, dj, dk) per component
    int qi[4], qj[4], qk[4];
    if constexpr (DM == 2) {
        if (COMP == 0) { qi[0] = 0; qj[0] = 0; qi[1] = 0; qj[1] = 1; }
        else { qi[0] = 0; qj[0] = 0; qi[1] = 1; qj[1] = 0; }
        qk[0] = qk[1] = 0;
    } else {
        if (COMP == 0) { int a_[4] = {0, 0, 0, 0}, b_[4] = {0, 1, 0, 1}, c_[4] = {0, 0, 1, 1};
            for (int q = 0; q < 4; ++q) { qi[q] = a_[q]; qj[q] = b_[q]; qk[q] = c_[q]; } }
        else if (COMP == 1) { int a_[4] = {0, 1, 0, 1}, b_[4] = {0, 0, 0, 0}, c_[4] = {0, 0, 1, 1};
            for (int q = 0; q < 4; ++q) { qi[q] = a_[q]; qj[q] = b_[q]; qk[q] = c_[q]; } }
        else { int a_[4] = {0, 1, 0, 1}, b_[4] = {0, 0, 1, 1}, c_[4] = {0, 0, 0, 0};
            for (int q = 0; q < 4; ++q) { qi[q] = a_[q]; qj[q] = b_[q]; qk[q] = c_[q]; } }
    }
    T r[3 * NQ];
    const int I = 2 * i, J = 2 * j, K = (DM == 3) ? 2 * k : k;
#pragma unroll 1
    for (int m = 0; m < 3 * NQ; ++m) {
        const int nrm = (m < NQ) ? 0 : (m < 2 * NQ ? 1 : -1);
        const int q = m % NQ;
        int ii = I + qi[q], jj = J + qj[q], kk = K + qk[q];
        if (COMP == 0) ii += nrm;
        else if (COMP == 1) jj += nrm;
        else kk += nrm;
        r[m] = fine_resid<T, DM, VISC, COMP, LD>(F, C, phi, rhs[COMP], ii, jj, kk, dxsqinv, b, cc);
    }
    if constexpr (DM == 2)
        return T(0.25) * (r[0] + r[1]) + T(0.125) * (r[2] + r[3] + r[4] + r[5]);
    else
        return T(0.125) * (r[0] + r[1] + r[2] + r[3]) + T(0.0625) * (r[4] + r[5] + r[6] + r[7]) +
               T(0.0625) * (r[8] + r[9] + r[10] + r[11]);
}

template <class T, int DM, int VISC, int LD = 0>
__device__ __forceinline__ void restrict_comp(int comp, const Dims& F, const Coef<T>& C, const T* const rhs[3],
                                              const T* const phi[3], T* const out[3], int t, int i, int j, int k, T dxsqinv) {
    if (comp == 0)
        out[0][t] = restrict_face<T, DM, VISC, 0, LD>(F, C, rhs, phi, i, j, k, dxsqinv);
    else if (comp == 1)
        out[1][t] = restrict_face<T, DM, VISC, 1, LD>(F, C, rhs, phi, i, j, k, dxsqinv);
    else if constexpr (DM == 3)
        out[2][t] = restrict_face<T, DM, VISC, 2, LD>(F, C, rhs, phi, i, j, k, dxsqinv);
}

// r = (L phi - rhs) * -1 on every face of one level (stag_mg_solver.f90:406-415)
// W: the residual is zero on wall faces (physbc_domainvel, stag_mg_solver.f90:424-425)
template <class T, int DM, int VISC, bool W = false>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 5 : 0) k_residual(Dims D, Coef<T> C, const T* __restrict__ r0, const T* __restrict__ r1,
                                                       const T* __restrict__ r2, const T* __restrict__ p0, const T* __restrict__ p1,
                                                       const T* __restrict__ p2, T* __restrict__ o0, T* __restrict__ o1,
                                                       T* __restrict__ o2, T dxsqinv) {
    pdl_enter();
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok) return;
    Nb nb = W ? make_nbw(D, q.i, q.j, q.k) : make_nb(D, q.i, q.j, q.k);
    const int t = nb.s;
    const T* phi[3] = {p0, p1, p2};
    const T b = ld(C.beta, 0), c = ld(C.gamma, 0);
    if (W && wall_face(nb, 0)) {
        o0[t] = T(0);
    } else {
        T v = face_L<T, DM, VISC, 0, 0, T, W>(phi, C, nb, dxsqinv, b, c) - ld(r0, t);
        o0[t] = v * T(-1);
    }
    if (W && wall_face(nb, 1)) {
        o1[t] = T(0);
    } else {
        T v = face_L<T, DM, VISC, 1, 0, T, W>(phi, C, nb, dxsqinv, b, c) - ld(r1, t);
        o1[t] = v * T(-1);
    }
    if constexpr (DM == 3) {
        if (W && wall_face(nb, 2)) {
            o2[t] = T(0);
        } else {
            T v = face_L<T, DM, VISC, 2, 0, T, W>(phi, C, nb, dxsqinv, b, c) - ld(r2, t);
            o2[t] = v * T(-1);
        }
    }
}

// 6-point (2D) / 12-point (3D) restriction of precomputed fine residuals,
// same summation order as restrict_face, for the coarse cell (i, j, k) at
// coarse index t.  W: coarse wall faces are zero (physbc_domainvel on the
// restricted residual, stag_mg_solver.f90:439-443); every other coarse face
// reads fine faces inside the box.  LD: load mode of the fine arrays (ldp).
template <class T, int DM, bool W = false, int LD = 0>
__device__ __forceinline__ void restrict_cell(const Dims& F, const T* f0, const T* f1, const T* f2, const Dims& Dc, T* c0, T* c1,
                                              T* c2, int i, int j, int k, int t) {
    const int I = 2 * i, J = 2 * j, K = 2 * k;
    if constexpr (W) {
        // wall faces first; the others fall through to the periodic formula
        const int x[3] = {i, j, k};
        bool wf[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) wf[d] = d < DM && ((Dc.wall >> d) & 1) && x[d] == 0;
        if (wf[0]) c0[t] = T(0);
        if (wf[1]) c1[t] = T(0);
        if (DM == 3 && wf[2]) c2[t] = T(0);
        if (wf[0]) c0 = nullptr;
        if (wf[1]) c1 = nullptr;
        if (wf[2]) c2 = nullptr;
    }
    auto R = [&](const T* f, int ii, int jj, int kk) {
        ii = wrapi(ii, F.nx);
        jj = wrapi(jj, F.ny);
        kk = (DM == 3) ? wrapi(kk, F.nz) : kk;
        return ldp<LD>(f, ii + F.nx * (jj + F.ny * kk));
    };
    if constexpr (DM == 2) {
        if (!W || c0)
        c0[t] = T(0.25) * (R(f0, I, J, k) + R(f0, I, J + 1, k)) +
                T(0.125) * (R(f0, I + 1, J, k) + R(f0, I + 1, J + 1, k) + R(f0, I - 1, J, k) + R(f0, I - 1, J + 1, k));
        if (!W || c1)
        c1[t] = T(0.25) * (R(f1, I, J, k) + R(f1, I + 1, J, k)) +
                T(0.125) * (R(f1, I, J + 1, k) + R(f1, I + 1, J + 1, k) + R(f1, I, J - 1, k) + R(f1, I + 1, J - 1, k));
    } else {
        if (!W || c0)
        c0[t] = T(0.125) * (R(f0, I, J, K) + R(f0, I, J + 1, K) + R(f0, I, J, K + 1) + R(f0, I, J + 1, K + 1)) +
                T(0.0625) * (R(f0, I + 1, J, K) + R(f0, I + 1, J + 1, K) + R(f0, I + 1, J, K + 1) + R(f0, I + 1, J + 1, K + 1)) +
                T(0.0625) * (R(f0, I - 1, J, K) + R(f0, I - 1, J + 1, K) + R(f0, I - 1, J, K + 1) + R(f0, I - 1, J + 1, K + 1));
        if (!W || c1)
        c1[t] = T(0.125) * (R(f1, I, J, K) + R(f1, I + 1, J, K) + R(f1, I, J, K + 1) + R(f1, I + 1, J, K + 1)) +
                T(0.0625) * (R(f1, I, J + 1, K) + R(f1, I + 1, J + 1, K) + R(f1, I, J + 1, K + 1) + R(f1, I + 1, J + 1, K + 1)) +
                T(0.0625) * (R(f1, I, J - 1, K) + R(f1, I + 1, J - 1, K) + R(f1, I, J - 1, K + 1) + R(f1, I + 1, J - 1, K + 1));
        if (!W || c2)
        c2[t] = T(0.125) * (R(f2, I, J, K) + R(f2, I + 1, J, K) + R(f2, I, J + 1, K) + R(f2, I + 1, J + 1, K)) +
                T(0.0625) * (R(f2, I, J, K + 1) + R(f2, I + 1, J, K + 1) + R(f2, I, J + 1, K + 1) + R(f2, I + 1, J + 1, K + 1)) +
                T(0.0625) * (R(f2, I, J, K - 1) + R(f2, I + 1, J, K - 1) + R(f2, I, J + 1, K - 1) + R(f2, I + 1, J + 1, K - 1));
    }
}

template <class T, int DM, bool W = false>
__global__ void __launch_bounds__(kThreads) k_restrict(Dims F, const T* __restrict__ f0, const T* __restrict__ f1,
                                                       const T* __restrict__ f2, Dims Dc, T* __restrict__ c0, T* __restrict__ c1,
                                                       T* __restrict__ c2) {
    pdl_enter();
    const Pos q = pos3(Dc.nx, Dc.ny);
    if (!q.ok) return;
    const int t = q.i + Dc.nx * (q.j + Dc.ny * q.k);
    restrict_cell<T, DM, W, 0>(F, f0, f1, f2, Dc, c0, c1, c2, q.i, q.j, q.k, t);
}

// Residual and restriction of one 3D periodic level in one pass
// (stag_mg_solver.f90:406-437 then stag_restriction, :1133-1171), opt-in
// (knobs.residual_fusion = 1): it saves writing and re-reading the fine
// residual but evaluates the face layer each block shares with its
// neighbour twice and launches few blocks on coarse levels, and measured
// slower than the split pair below on every level of the benchmark.  A block
// owns RCX x RCY x RCZ coarse cells; it evaluates into shared memory every
// fine residual r = (L phi - rhs) * -1 that their 12-point restrictions read
// (the fine faces of the tile plus one face layer on the low and high side
// normal to each component), then forms the coarse faces from shared memory
// in restrict_cell's order.  The fine residual never goes to global memory,
// and each one is evaluated once per block (the 2 x 2 x 2-to-1 stencil
// overlaps only across the block boundary).
constexpr int RCX = 8, RCY = 4, RCZ = 4;
template <int COMP>
struct RTile {  // fine residuals of one component held by the block
    static constexpr int NX = 2 * RCX + (COMP == 0 ? 1 : 0);
    static constexpr int NY = 2 * RCY + (COMP == 1 ? 1 : 0);
    static constexpr int NZ = 2 * RCZ + (COMP == 2 ? 1 : 0);
    static constexpr int N = NX * NY * NZ;
};

template <class T, int VISC>
__global__ void __launch_bounds__(kThreads) k_resid_restrict3(Dims F, Coef<T> C, const T* __restrict__ r0, const T* __restrict__ r1,
                                                              const T* __restrict__ r2, const T* __restrict__ p0,
                                                              const T* __restrict__ p1, const T* __restrict__ p2, Dims Dc,
                                                              T* __restrict__ c0, T* __restrict__ c1, T* __restrict__ c2,
                                                              T dxsqinv) {
    pdl_enter();
    using X = RTile<0>;
    using Y = RTile<1>;
    using Z = RTile<2>;
    __shared__ T rs[X::N + Y::N + Z::N];
    const int ci0 = blockIdx.x * RCX, cj0 = blockIdx.y * RCY, ck0 = blockIdx.z * RCZ;
    const T* phi[3] = {p0, p1, p2};
    const T b = ld(C.beta, 0), c = ld(C.gamma, 0);
    // fine residuals: component x from fine i = 2 ci0 - 1, y from j = 2 cj0 - 1,
    // z from k = 2 ck0 - 1 (one layer below the tile in its own direction)
    for (int t = threadIdx.x; t < X::N + Y::N + Z::N; t += kThreads) {
        if (t < X::N) {
            const int a = t % X::NX, bb = (t / X::NX) % X::NY, cc = t / (X::NX * X::NY);
            rs[t] = fine_resid<T, 3, VISC, 0>(F, C, phi, r0, 2 * ci0 - 1 + a, 2 * cj0 + bb, 2 * ck0 + cc, dxsqinv, b, c);
        } else if (t < X::N + Y::N) {
            const int u = t - X::N;
            const int a = u % Y::NX, bb = (u / Y::NX) % Y::NY, cc = u / (Y::NX * Y::NY);
            rs[t] = fine_resid<T, 3, VISC, 1>(F, C, phi, r1, 2 * ci0 + a, 2 * cj0 - 1 + bb, 2 * ck0 + cc, dxsqinv, b, c);
        } else {
            const int u = t - X::N - Y::N;
            const int a = u % Z::NX, bb = (u / Z::NX) % Z::NY, cc = u / (Z::NX * Z::NY);
            rs[t] = fine_resid<T, 3, VISC, 2>(F, C, phi, r2, 2 * ci0 + a, 2 * cj0 + bb, 2 * ck0 - 1 + cc, dxsqinv, b, c);
        }
    }
    __syncthreads();
    constexpr int NC = RCX * RCY * RCZ;
    for (int t = threadIdx.x; t < 3 * NC; t += kThreads) {
        const int comp = t / NC, u = t - comp * NC;
        const int i = u % RCX, j = (u / RCX) % RCY, k = u / (RCX * RCY);
        // fine index of the coarse face's first fine face inside the block's arrays
        const int I = 2 * i + (comp == 0 ? 1 : 0), J = 2 * j + (comp == 1 ? 1 : 0), K = 2 * k + (comp == 2 ? 1 : 0);
        const int out = (ci0 + i) + Dc.nx * ((cj0 + j) + Dc.ny * (ck0 + k));
        if (comp == 0) {
            auto R = [&](int ii, int jj, int kk) { return rs[ii + X::NX * (jj + X::NY * kk)]; };
            c0[out] = T(0.125) * (R(I, J, K) + R(I, J + 1, K) + R(I, J, K + 1) + R(I, J + 1, K + 1)) +
                      T(0.0625) * (R(I + 1, J, K) + R(I + 1, J + 1, K) + R(I + 1, J, K + 1) + R(I + 1, J + 1, K + 1)) +
                      T(0.0625) * (R(I - 1, J, K) + R(I - 1, J + 1, K) + R(I - 1, J, K + 1) + R(I - 1, J + 1, K + 1));
        } else if (comp == 1) {
            auto R = [&](int ii, int jj, int kk) { return rs[X::N + ii + Y::NX * (jj + Y::NY * kk)]; };
            c1[out] = T(0.125) * (R(I, J, K) + R(I + 1, J, K) + R(I, J, K + 1) + R(I + 1, J, K + 1)) +
                      T(0.0625) * (R(I, J + 1, K) + R(I + 1, J + 1, K) + R(I, J + 1, K + 1) + R(I + 1, J + 1, K + 1)) +
                      T(0.0625) * (R(I, J - 1, K) + R(I + 1, J - 1, K) + R(I, J - 1, K + 1) + R(I + 1, J - 1, K + 1));
        } else {
            auto R = [&](int ii, int jj, int kk) { return rs[X::N + Y::N + ii + Z::NX * (jj + Z::NY * kk)]; };
            c2[out] = T(0.125) * (R(I, J, K) + R(I + 1, J, K) + R(I, J + 1, K) + R(I + 1, J + 1, K)) +
                      T(0.0625) * (R(I, J, K + 1) + R(I + 1, J, K + 1) + R(I, J + 1, K + 1) + R(I + 1, J + 1, K + 1)) +
                      T(0.0625) * (R(I, J, K - 1) + R(I + 1, J, K - 1) + R(I, J + 1, K - 1) + R(I + 1, J + 1, K - 1));
        }
    }
}

// --------------------------------------------------------------- prolongation
template <class T, int LD = 0>
__device__ __forceinline__ T cat(const T* a, const Dims& Dc, int i, int j, int k) {
    i = wrapi(i, Dc.nx);
    j = wrapi(j, Dc.ny);
    k = (Dc.dm == 3) ? wrapi(k, Dc.nz) : k;
    return ldp<LD>(a, i + Dc.nx * (j + Dc.ny * k));
}

// coarse value of component COMP at (i, j, k) on a grid with walls (the
// coarse level's ghost fills): periodic directions wrap; across its own
// walls the component is zero; across another direction's wall the ghost
// mirrors the face, negated at a no-slip wall
template <class T, int LD, int COMP>
__device__ __forceinline__ T catw(const T* a, const Dims& Dc, int i, int j, int k) {
    int x[3] = {i, j, k};
    const int n[3] = {Dc.nx, Dc.ny, Dc.nz};
    bool neg = false;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d >= Dc.dm) continue;
        if (!((Dc.wall >> d) & 1)) {
            x[d] = wrapi(x[d], n[d]);
            continue;
        }
        if (d == COMP) {
            if (x[d] < 0 || x[d] >= n[d]) return T(0);
            continue;
        }
        if (x[d] < 0) {
            x[d] = 0;
            if (!((Dc.slip_lo >> d) & 1)) neg = !neg;
        } else if (x[d] >= n[d]) {
            x[d] = n[d] - 1;
            if (!((Dc.slip_hi >> d) & 1)) neg = !neg;
        }
    }
    const T v = ldp<LD>(a, x[0] + Dc.nx * (x[1] + Dc.ny * x[2]));
    return neg ? -v : v;
}
template <class T, int LD, bool W, int COMP>
__device__ __forceinline__ T pcat(const T* a, const Dims& Dc, int i, int j, int k) {
    if constexpr (W)
        return catw<T, LD, COMP>(a, Dc, i, j, k);
    else
        return cat<T, LD>(a, Dc, i, j, k);
}

// add the interpolated coarse correction to the DM fine faces at (i, j, k);
// W: fine wall faces keep their zero (physbc_domainvel after the
// prolongation, stag_mg_solver.f90:681-690)
template <class T, int DM, int LD = 0, bool W = false>
__device__ __forceinline__ void prolong_cell(const Dims& Dc, const T* q0, const T* q1, const T* q2, T* f0, T* f1, T* f2, int t,
                                             int i, int j, int k) {
    if constexpr (W) {
        // the fine grid's wall bits are the coarse grid's
        const int x[3] = {i, j, k};
        if ((Dc.wall & 1) && x[0] == 0) f0 = nullptr;
        if (((Dc.wall >> 1) & 1) && x[1] == 0) f1 = nullptr;
        if constexpr (DM == 3)
            if (((Dc.wall >> 2) & 1) && x[2] == 0) f2 = nullptr;
    }
    const int i2 = i >> 1, j2 = j >> 1, k2 = k >> 1;
    if constexpr (DM == 2) {
        if (!W || f0) {
            int joff = ((j & 1) == 0) ? -1 : 1;
            T v = (LD == 2) ? __ldcg(f0 + t) : f0[t];
            if ((i & 1) == 0)
                v = v + T(0.75) * pcat<T, LD, W, 0>(q0, Dc, i2, j2, k) + T(0.25) * pcat<T, LD, W, 0>(q0, Dc, i2, j2 + joff, k);
            else
                v = v + T(0.375) * pcat<T, LD, W, 0>(q0, Dc, i2, j2, k) + T(0.125) * pcat<T, LD, W, 0>(q0, Dc, i2, j2 + joff, k) + T(0.375) * pcat<T, LD, W, 0>(q0, Dc, i2 + 1, j2, k) +
                    T(0.125) * pcat<T, LD, W, 0>(q0, Dc, i2 + 1, j2 + joff, k);
            f0[t] = v;
        }
        if (!W || f1) {
            int ioff = ((i & 1) == 0) ? -1 : 1;
            T v = (LD == 2) ? __ldcg(f1 + t) : f1[t];
            if ((j & 1) == 0)
                v = v + T(0.75) * pcat<T, LD, W, 1>(q1, Dc, i2, j2, k) + T(0.25) * pcat<T, LD, W, 1>(q1, Dc, i2 + ioff, j2, k);
            else
                v = v + T(0.375) * pcat<T, LD, W, 1>(q1, Dc, i2, j2, k) + T(0.125) * pcat<T, LD, W, 1>(q1, Dc, i2 + ioff, j2, k) + T(0.375) * pcat<T, LD, W, 1>(q1, Dc, i2, j2 + 1, k) +
                    T(0.125) * pcat<T, LD, W, 1>(q1, Dc, i2 + ioff, j2 + 1, k);
            f1[t] = v;
        }
    } else {
        const T n16 = T(9.0 / 16.0), t16 = T(3.0 / 16.0), o16 = T(1.0 / 16.0);
        const T n32 = T(9.0 / 32.0), t32 = T(3.0 / 32.0), o32 = T(1.0 / 32.0);
        const int ioff = ((i & 1) == 0) ? -1 : 1, joff = ((j & 1) == 0) ? -1 : 1, koff = ((k & 1) == 0) ? -1 : 1;
        if (!W || f0) {
            T v = (LD == 2) ? __ldcg(f0 + t) : f0[t];
            if ((i & 1) == 0)
                v = v + n16 * pcat<T, LD, W, 0>(q0, Dc, i2, j2, k2) + t16 * pcat<T, LD, W, 0>(q0, Dc, i2, j2 + joff, k2) + t16 * pcat<T, LD, W, 0>(q0, Dc, i2, j2, k2 + koff) +
                    o16 * pcat<T, LD, W, 0>(q0, Dc, i2, j2 + joff, k2 + koff);
            else
                v = v + n32 * pcat<T, LD, W, 0>(q0, Dc, i2, j2, k2) + t32 * pcat<T, LD, W, 0>(q0, Dc, i2, j2 + joff, k2) + t32 * pcat<T, LD, W, 0>(q0, Dc, i2, j2, k2 + koff) +
                    o32 * pcat<T, LD, W, 0>(q0, Dc, i2, j2 + joff, k2 + koff) + n32 * pcat<T, LD, W, 0>(q0, Dc, i2 + 1, j2, k2) +
                    t32 * pcat<T, LD, W, 0>(q0, Dc, i2 + 1, j2 + joff, k2) + t32 * pcat<T, LD, W, 0>(q0, Dc, i2 + 1, j2, k2 + koff) +
                    o32 * pcat<T, LD, W, 0>(q0, Dc, i2 + 1, j2 + joff, k2 + koff);
            f0[t] = v;
        }
        if (!W || f1) {
            T v = (LD == 2) ? __ldcg(f1 + t) : f1[t];
            if ((j & 1) == 0)
                v = v + n16 * pcat<T, LD, W, 1>(q1, Dc, i2, j2, k2) + t16 * pcat<T, LD, W, 1>(q1, Dc, i2 + ioff, j2, k2) + t16 * pcat<T, LD, W, 1>(q1, Dc, i2, j2, k2 + koff) +
                    o16 * pcat<T, LD, W, 1>(q1, Dc, i2 + ioff, j2, k2 + koff);
            else
                v = v + n32 * pcat<T, LD, W, 1>(q1, Dc, i2, j2, k2) + t32 * pcat<T, LD, W, 1>(q1, Dc, i2 + ioff, j2, k2) + t32 * pcat<T, LD, W, 1>(q1, Dc, i2, j2, k2 + koff) +
                    o32 * pcat<T, LD, W, 1>(q1, Dc, i2 + ioff, j2, k2 + koff) + n32 * pcat<T, LD, W, 1>(q1, Dc, i2, j2 + 1, k2) +
                    t32 * pcat<T, LD, W, 1>(q1, Dc, i2 + ioff, j2 + 1, k2) + t32 * pcat<T, LD, W, 1>(q1, Dc, i2, j2 + 1, k2 + koff) +
                    o32 * pcat<T, LD, W, 1>(q1, Dc, i2 + ioff, j2 + 1, k2 + koff);
            f1[t] = v;
        }
        if (!W || f2) {
            T v = (LD == 2) ? __ldcg(f2 + t) : f2[t];
            if ((k & 1) == 0)
                v = v + n16 * pcat<T, LD, W, 2>(q2, Dc, i2, j2, k2) + t16 * pcat<T, LD, W, 2>(q2, Dc, i2 + ioff, j2, k2) + t16 * pcat<T, LD, W, 2>(q2, Dc, i2, j2 + joff, k2) +
                    o16 * pcat<T, LD, W, 2>(q2, Dc, i2 + ioff, j2 + joff, k2);
            else
                v = v + n32 * pcat<T, LD, W, 2>(q2, Dc, i2, j2, k2) + t32 * pcat<T, LD, W, 2>(q2, Dc, i2 + ioff, j2, k2) + t32 * pcat<T, LD, W, 2>(q2, Dc, i2, j2 + joff, k2) +
                    o32 * pcat<T, LD, W, 2>(q2, Dc, i2 + ioff, j2 + joff, k2) + n32 * pcat<T, LD, W, 2>(q2, Dc, i2, j2, k2 + 1) +
                    t32 * pcat<T, LD, W, 2>(q2, Dc, i2 + ioff, j2, k2 + 1) + t32 * pcat<T, LD, W, 2>(q2, Dc, i2, j2 + joff, k2 + 1) +
                    o32 * pcat<T, LD, W, 2>(q2, Dc, i2 + ioff, j2 + joff, k2 + 1);
            f2[t] = v;
        }
    }
}

template <class T, int DM, bool W = false>
__global__ void __launch_bounds__(kThreads) k_prolong_add(Dims F, Dims Dc, const T* __restrict__ q0, const T* __restrict__ q1,
                                                          const T* __restrict__ q2, T* __restrict__ f0, T* __restrict__ f1,
                                                          T* __restrict__ f2) {
    pdl_enter();
    const Pos q = pos3(F.nx, F.ny);
    if (!q.ok) return;
    const int t = q.i + F.nx * (q.j + F.ny * q.k);
    prolong_cell<T, DM, 0, W>(Dc, q0, q1, q2, f0, f1, f2, t, q.i, q.j, q.k);
}

// --------------------------------------------------------------- coefficient coarsening
// fine-grid value at (i, j, k), all indices inside the fine box
template <class T>
__device__ __forceinline__ T fat(const T* a, const Dims& F, int i, int j, int k) {
    return ld(a, i + F.nx * (j + F.ny * k));
}

// do_visc: 0 faces only, 1 faces + cells + edges, 2 faces + cells (the edges
// of a grid with walls go through k_coarsen_edges_w)
template <class T, int DM>
__global__ void __launch_bounds__(kThreads) k_coarsen(Dims F, Dims Dc, Coef<T> Cf, T* a0, T* a1, T* a2, T* beta, T* gamma,
                                                      T* e0, T* e1, T* e2, int do_visc) {
    const Pos q = pos3(Dc.nx, Dc.ny);
    if (!q.ok) return;
    const int i = q.i, j = q.j, k = q.k;
    const int t = i + Dc.nx * (j + Dc.ny * k);
    const int I = 2 * i, J = 2 * j, K = 2 * k;
    if constexpr (DM == 2) {
        a0[t] = T(0.5) * (fat(Cf.alpha[0], F, I, J, k) + fat(Cf.alpha[0], F, I, J + 1, k));
        a1[t] = T(0.5) * (fat(Cf.alpha[1], F, I, J, k) + fat(Cf.alpha[1], F, I + 1, J, k));
        if (do_visc) {
            const T* b = Cf.beta;
            beta[t] = T(0.25) * (fat(b, F, I, J, k) + fat(b, F, I + 1, J, k) + fat(b, F, I, J + 1, k) + fat(b, F, I + 1, J + 1, k));
            const T* g = Cf.gamma;
            gamma[t] = T(0.25) * (fat(g, F, I, J, k) + fat(g, F, I + 1, J, k) + fat(g, F, I, J + 1, k) + fat(g, F, I + 1, J + 1, k));
            if (do_visc == 1) e0[t] = fat(Cf.bed[0], F, I, J, k);  // nodal injection
        }
    } else {
        const T* A0 = Cf.alpha[0];
        const T* A1 = Cf.alpha[1];
        const T* A2 = Cf.alpha[2];
        a0[t] = T(0.25) * (fat(A0, F, I, J, K) + fat(A0, F, I, J + 1, K) + fat(A0, F, I, J, K + 1) + fat(A0, F, I, J + 1, K + 1));
        a1[t] = T(0.25) * (fat(A1, F, I, J, K) + fat(A1, F, I + 1, J, K) + fat(A1, F, I, J, K + 1) + fat(A1, F, I + 1, J, K + 1));
        a2[t] = T(0.25) * (fat(A2, F, I, J, K) + fat(A2, F, I + 1, J, K) + fat(A2, F, I, J + 1, K) + fat(A2, F, I + 1, J + 1, K));
        if (do_visc) {
            const T* b = Cf.beta;
            beta[t] = T(0.125) * (fat(b, F, I, J, K) + fat(b, F, I + 1, J, K) + fat(b, F, I, J + 1, K) + fat(b, F, I + 1, J + 1, K) +
                                  fat(b, F, I, J, K + 1) + fat(b, F, I + 1, J, K + 1) + fat(b, F, I, J + 1, K + 1) +
                                  fat(b, F, I + 1, J + 1, K + 1));
            const T* g = Cf.gamma;
            gamma[t] = T(0.125) * (fat(g, F, I, J, K) + fat(g, F, I + 1, J, K) + fat(g, F, I, J + 1, K) + fat(g, F, I + 1, J + 1, K) +
                                   fat(g, F, I, J, K + 1) + fat(g, F, I + 1, J, K + 1) + fat(g, F, I, J + 1, K + 1) +
                                   fat(g, F, I + 1, J + 1, K + 1));
            if (do_visc == 1) {
                e0[t] = T(0.5) * (fat(Cf.bed[0], F, I, J, K) + fat(Cf.bed[0], F, I, J, K + 1));
                e1[t] = T(0.5) * (fat(Cf.bed[1], F, I, J, K) + fat(Cf.bed[1], F, I, J + 1, K));
                e2[t] = T(0.5) * (fat(Cf.bed[2], F, I, J, K) + fat(Cf.bed[2], F, I + 1, J, K));
            }
        }
    }
}

// edge coefficients of a grid with walls (n+1 nodes along a nodal
// wall-bounded direction): nodal injection in 2D (nodal_restriction,
// stag_mg_solver.f90:1229-1244), two-point average along the edge in 3D
// (edge_restriction, :1326-1367); the launch covers (nx+1, ny+1, nz+1)
template <class T, int DM>
__global__ void __launch_bounds__(kThreads) k_coarsen_edges_w(Dims F, Dims Dc, const T* f0, const T* f1, const T* f2, T* e0, T* e1,
                                                              T* e2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    const int I = 2 * i, J = 2 * j, K = 2 * k;
    const T* f[3] = {f0, f1, f2};
    T* e[3] = {e0, e1, e2};
#pragma unroll
    for (int q = 0; q < (DM == 2 ? 1 : 3); ++q) {
        // 2D: the third index is the instance (a batch stacks nz of them)
        const int cx = edge_ext(Dc, q, 0), cy = edge_ext(Dc, q, 1), cz = (DM == 3) ? edge_ext(Dc, q, 2) : Dc.nz;
        if (i >= cx || j >= cy || k >= cz) continue;
        const int fx = edge_ext(F, q, 0), fy = edge_ext(F, q, 1);
        auto at = [&](int a, int b, int c) { return ld(f[q], a + fx * (b + fy * c)); };
        T v;
        if (DM == 2) v = at(I, J, k);
        else if (q == 0) v = T(0.5) * (at(I, J, K) + at(I, J, K + 1));
        else if (q == 1) v = T(0.5) * (at(I, J, K) + at(I, J + 1, K));
        else v = T(0.5) * (at(I, J, K) + at(I + 1, J, K));
        e[q][i + cx * (j + cy * k)] = v;
    }
}

// --------------------------------------------------------------- pressure multigrid
template <class T, int DM, int LD = 0>
__device__ __forceinline__ T cc_lap(const T* const a[3], const T* phi, const Nb& n, T dxsqinv) {
    const int s = n.s;
    const T p = ldp<LD>(phi, s);
    T v = (ld(a[0], s + n.op[0]) * (ldp<LD>(phi, s + n.op[0]) - p) - ld(a[0], s) * (p - ldp<LD>(phi, s + n.om[0]))) +
          (ld(a[1], s + n.op[1]) * (ldp<LD>(phi, s + n.op[1]) - p) - ld(a[1], s) * (p - ldp<LD>(phi, s + n.om[1])));
    if constexpr (DM == 3)
        v = v + (ld(a[2], s + n.op[2]) * (ldp<LD>(phi, s + n.op[2]) - p) - ld(a[2], s) * (p - ldp<LD>(phi, s + n.om[2])));
    return v * dxsqinv;
}
template <class T, int DM>
__device__ __forceinline__ T cc_diag(const T* const a[3], const Nb& n, T dxsqinv) {
    const int s = n.s;
    T sum = ld(a[0], s) + ld(a[0], s + n.op[0]) + ld(a[1], s) + ld(a[1], s + n.op[1]);
    if constexpr (DM == 3) sum = sum + ld(a[2], s) + ld(a[2], s + n.op[2]);
    return -(sum * dxsqinv);
}

// flag = 1 when an entry of a0, a1 or a2 (a1, a2 may be null) differs from
// a0[0] in its bits
template <class T>
__global__ void k_uniform_check(const T* __restrict__ a0, const T* __restrict__ a1, const T* __restrict__ a2, int64_t n,
                                int* __restrict__ flag) {
    auto bits = [](T x) -> unsigned long long {
        if constexpr (sizeof(T) == 8)
            return (unsigned long long)__double_as_longlong((double)x);
        else
            return (unsigned long long)(unsigned)__float_as_int((float)x);
    };
    const unsigned long long v = bits(a0[0]);
    bool diff = false;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n && !diff; t += (int64_t)gridDim.x * blockDim.x)
        diff = bits(a0[t]) != v || (a1 && bits(a1[t]) != v) || (a2 && bits(a2[t]) != v);
    if (diff) atomicOr(flag, 1);
}

// the same two expressions with every face coefficient equal to c (the
// value each load would return: the same operations, the same bits)
template <class T, int DM, int LD = 0>
__device__ __forceinline__ T cc_lap_u(T c, const T* phi, const Nb& n, T dxsqinv) {
    const int s = n.s;
    const T p = ldp<LD>(phi, s);
    T v = (c * (ldp<LD>(phi, s + n.op[0]) - p) - c * (p - ldp<LD>(phi, s + n.om[0]))) +
          (c * (ldp<LD>(phi, s + n.op[1]) - p) - c * (p - ldp<LD>(phi, s + n.om[1])));
    if constexpr (DM == 3) v = v + (c * (ldp<LD>(phi, s + n.op[2]) - p) - c * (p - ldp<LD>(phi, s + n.om[2])));
    return v * dxsqinv;
}
template <class T, int DM>
__device__ __forceinline__ T cc_diag_u(T c, T dxsqinv) {
    T sum = c + c + c + c;
    if constexpr (DM == 3) sum = sum + c + c;
    return -(sum * dxsqinv);
}

// U: every face coefficient equals cu (the arrays a0..a2 are not read);
// reverse: the blocks take the planes in decreasing order (see k_gs_colour)
template <class T, int DM, bool U = false>
__global__ void __launch_bounds__(kThreads) k_cc_smooth(Dims D, const T* a0, const T* a1, const T* a2, const T* __restrict__ rhs,
                                                        T* phi, int parity, T dxsqinv, T cu, int reverse) {
    pdl_enter();
    const Pos q = pos3(D.nx >> 1, D.ny);
    if (!q.ok) return;
    const int j = q.j, k = reverse ? (int)gridDim.z - 1 - q.k : q.k;
    const int i = 2 * q.i + ((j + ck<DM>(k) + parity) & 1);
    Nb nb = make_nb(D, i, j, k);
    if constexpr (U) {
        T res = ld(rhs, nb.s) - cc_lap_u<T, DM>(cu, phi, nb, dxsqinv);
        T cur = phi[nb.s];
        phi[nb.s] = cur + res / cc_diag_u<T, DM>(cu, dxsqinv);
    } else {
        const T* a[3] = {a0, a1, a2};
        T res = ld(rhs, nb.s) - cc_lap<T, DM>(a, phi, nb, dxsqinv);
        T cur = phi[nb.s];
        phi[nb.s] = cur + res / cc_diag<T, DM>(a, nb, dxsqinv);
    }
}

// one colour of the pressure smoother on an odd level: new values from the
// values before the colour's pass (out), then copied back
template <class T, int DM>
__global__ void __launch_bounds__(kThreads) k_cc_smooth_odd(Dims D, const T* a0, const T* a1, const T* a2, const T* __restrict__ rhs,
                                                            const T* __restrict__ phi, T* __restrict__ out, int parity, T dxsqinv) {
    pdl_enter();
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok || ((q.i + q.j + ck<DM>(q.k)) & 1) != parity) return;
    Nb nb = make_nb(D, q.i, q.j, q.k);
    const T* a[3] = {a0, a1, a2};
    T res = ld(rhs, nb.s) - cc_lap<T, DM>(a, phi, nb, dxsqinv);
    T cur = phi[nb.s];
    out[nb.s] = cur + res / cc_diag<T, DM>(a, nb, dxsqinv);
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_copy_parity(Dims D, const T* __restrict__ in, T* __restrict__ out, int parity) {
    pdl_enter();
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok || ((q.i + q.j + (D.dm == 3 ? q.k : 0)) & 1) != parity) return;
    const int s = q.i + D.nx * (q.j + D.ny * q.k);
    out[s] = in[s];
}

template <class T, int DM, int LD = 0>
__device__ __forceinline__ T cc_res_at(const Dims& F, const T* const a[3], const T* phi, const T* rhs, int i, int j, int k,
                                       T dxsqinv) {
    Nb nb = make_nb(F, i, j, k);
    return ldp<LD>(rhs, nb.s) - cc_lap<T, DM, LD>(a, phi, nb, dxsqinv);
}

template <class T, int DM, bool U = false>
__global__ void __launch_bounds__(kThreads) k_cc_residual_restrict(Dims F, const T* a0, const T* a1, const T* a2,
                                                                   const T* __restrict__ rhs, const T* __restrict__ phi, Dims Dc,
                                                                   T* __restrict__ rc, T dxsqinv, T cu) {
    pdl_enter();
    const Pos q = pos3(Dc.nx, Dc.ny);
    if (!q.ok) return;
    const int i = q.i, j = q.j, k = q.k;
    const int t = i + Dc.nx * (j + Dc.ny * k);
    const T* a[3] = {a0, a1, a2};
    const int I = 2 * i, J = 2 * j, K = 2 * k;
    auto res_at = [&](int ii, int jj, int kk) -> T {
        if constexpr (U) {
            Nb nb = make_nb(F, ii, jj, kk);
            return ld(rhs, nb.s) - cc_lap_u<T, DM>(cu, phi, nb, dxsqinv);
        } else {
            return cc_res_at<T, DM>(F, a, phi, rhs, ii, jj, kk, dxsqinv);
        }
    };
#define R(ii, jj, kk) res_at(ii, jj, kk)
    if constexpr (DM == 2)
        rc[t] = T(0.25) * (R(I, J, k) + R(I + 1, J, k) + R(I, J + 1, k) + R(I + 1, J + 1, k));
    else
        rc[t] = T(0.125) * (R(I, J, K) + R(I + 1, J, K) + R(I, J + 1, K) + R(I + 1, J + 1, K) + R(I, J, K + 1) + R(I + 1, J, K + 1) +
                            R(I, J + 1, K + 1) + R(I + 1, J + 1, K + 1));
#undef R
}

template <class T, int DM>
__global__ void __launch_bounds__(kThreads) k_cc_prolong_add(Dims F, Dims Dc, const T* __restrict__ pc, T* __restrict__ pf) {
    pdl_enter();
    const Pos q = pos3(F.nx, F.ny);
    if (!q.ok) return;
    const int t = q.i + F.nx * (q.j + F.ny * q.k);
    pf[t] = pf[t] + ld(pc, (q.i >> 1) + Dc.nx * ((q.j >> 1) + Dc.ny * ((DM == 3) ? (q.k >> 1) : q.k)));
}

template <class T, int DM>
__global__ void __launch_bounds__(kThreads) k_neg_cc_lap(Dims D, const T* a0, const T* a1, const T* a2, const T* __restrict__ phi,
                                                         T* __restrict__ out, T dxsqinv) {
    pdl_enter();
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok) return;
    Nb nb = make_nb(D, q.i, q.j, q.k);
    const T* a[3] = {a0, a1, a2};
    out[nb.s] = -cc_lap<T, DM>(a, phi, nb, dxsqinv);
}

// --------------------------------------------------------------- div / grad pieces
// W: the hi+1 wall face of a wall-normal component is zero
template <class T, int DM, bool W = false>
__global__ void __launch_bounds__(kThreads) k_div_plus(Dims D, const T* __restrict__ u0, const T* __restrict__ u1,
                                                       const T* __restrict__ u2, const T* __restrict__ bp, T* __restrict__ out,
                                                       T dxinv) {
    pdl_enter();
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok) return;
    Nb nb = W ? make_nbw(D, q.i, q.j, q.k) : make_nb(D, q.i, q.j, q.k);
    const int t = nb.s;
    auto up = [&](const T* u, int d) {
        const T v = ld(u, t + nb.op[d]);
        return W ? wapply(wall_mul(nb, d, d, true), v) : v;
    };
    T v = (up(u0, 0) - ld(u0, t)) * dxinv + (up(u1, 1) - ld(u1, t)) * dxinv;
    if constexpr (DM == 3) v = v + (up(u2, 2) - ld(u2, t)) * dxinv;
    out[t] = v + ld(bp, t);
}

// W: wall faces are left alone (the wall gradient of a FOEXTRAP pressure
// is zero, div_and_grad.f90:139-182)
template <class T, int DM, bool W = false>
__global__ void __launch_bounds__(kThreads) k_sub_weighted_grad(Dims D, const T* c0, const T* c1, const T* c2,
                                                                const T* __restrict__ phi, T* u0, T* u1, T* u2, T dxinv) {
    pdl_enter();
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok) return;
    Nb nb = W ? make_nbw(D, q.i, q.j, q.k) : make_nb(D, q.i, q.j, q.k);
    const int t = nb.s;
    const T p = ld(phi, t);
    T* u[3] = {u0, u1, u2};
    const T* c[3] = {c0, c1, c2};
#pragma unroll
    for (int d = 0; d < DM; ++d) {
        if (W && wall_face(nb, d)) continue;
        T g = (p - ld(phi, t + nb.om[d])) * dxinv;
        if (c[d]) g = g * ld(c[d], t);
        u[d][t] = u[d][t] + T(-1) * g;
    }
}

// --------------------------------------------------------------- small vector ops
template <class Tin, class Tout>
__global__ void k_convert(const Tin* __restrict__ in, Tout* __restrict__ out, int64_t n) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) out[t] = (Tout)in[t];
}
template <class T>
__global__ void k_scale_copy(const T* __restrict__ in, T* __restrict__ out, T s, int64_t n) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) out[t] = in[t] * s;
}
template <class T>
__global__ void k_add_to(T* __restrict__ x, const T* __restrict__ y, int64_t n) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) x[t] = x[t] + y[t];
}
template <class T>
__global__ void k_recip(const T* __restrict__ in, T* __restrict__ out, int64_t n) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) out[t] = T(1) / in[t];
}
template <class T>
__global__ void k_fill(T* __restrict__ out, T v, int64_t n) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) out[t] = v;
}

// --------------------------------------------------------------- deterministic reductions
// Each block accumulates a fixed grid-stride subset in double, reduces it in
// a fixed tree, writes its partials; the last block to finish sums all
// partials in block order.  The result depends only on n and the launch
// shape, never on scheduling.
//
// MODE 0: weighted dot, MODE 1: weighted sum, MODE 2: max |a - b| (inf norm).
// Seam weights: the main loop gives every face weight 1; a second loop over
// the periodic seam plane of face component c (index_c == 0) adds
// (w_c - 1) a b, so the seam face ends with weight w_c.
// out[0..dm] per component; out[4] = sum_d out[d] + pw^2 out[dm] (the
// Hessenberg entry of gmres.f90:344), out[5] = sqrt(|u|^2 + (pw |p|)^2)
// (the Stokes norm of gmres.f90:127-130).
//
// 2D batches (D.nz instances of nx*ny cells): blockIdx.y is the instance,
// with its own partials, counter and 8-double output slot out + 8 * b; the
// grid's x extent and every summation order are those of one instance
// reduced alone, so each instance's result has the same bits.
// k_reduce may take entries in pairs: rows of even length and every array
// aligned to a pair (the same choice in the bounds-check build, whose pair
// loads are checked as one access each, so both builds sum alike)
static inline int reduce_pairs(const Dims& D, size_t elem, const void* const a[4], const void* const b[4]) {
    if (D.nx % 2) return 0;
    for (int q = 0; q < 4; ++q) {
        if (q == 2 && D.dm == 2) continue;  // a 2D reduction reads no third face array
        if ((a[q] && (uintptr_t)a[q] % (2 * elem)) || (b[q] && (uintptr_t)b[q] % (2 * elem))) return 0;
    }
    return 1;
}

template <class T>
struct Pair2;
template <>
struct Pair2<double> {
    using type = double2;
};
template <>
struct Pair2<float> {
    using type = float2;
};

// vec = 1 (reduce_pairs): entries in pairs by one 16- (FP64) or 8-byte
// (FP32) load per array; the sums change order within a thread's pair only
template <class T, int DM, int MODE>
__global__ void __launch_bounds__(kThreads) k_reduce(Dims D, const T* a0, const T* a1, const T* a2, const T* a3, const T* b0,
                                                     const T* b1, const T* b2, const T* b3, double w0, double w1, double w2,
                                                     double pw, double* partials, unsigned* counter, double* out, int vec) {
    pdl_enter();
    constexpr int NC = DM + 1;
    const int nzi = (DM == 3) ? D.nz : 1;  // third extent of one instance
    const int n = D.nx * D.ny * nzi;
    {
        const int64_t off = (int64_t)blockIdx.y * n;
        a0 = a0 ? a0 + off : a0;
        a1 = a1 ? a1 + off : a1;
        a2 = a2 ? a2 + off : a2;
        a3 = a3 ? a3 + off : a3;
        b0 = b0 ? b0 + off : b0;
        b1 = b1 ? b1 + off : b1;
        b2 = b2 ? b2 + off : b2;
        b3 = b3 ? b3 + off : b3;
        partials += (int64_t)blockIdx.y * gridDim.x * NC;
        counter += blockIdx.y;
        out += (int64_t)blockIdx.y * 8;
    }
    const T* A[4] = {a0, a1, a2, a3};
    const T* B[4] = {b0, b1, b2, b3};
    const double W[3] = {w0, w1, w2};
    double acc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = 0.0;
    const int stride = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const T* AA[NC];
    const T* BB[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        AA[c] = (c < DM) ? A[c] : A[3];
        BB[c] = (c < DM) ? B[c] : B[3];
    }
    if (vec) {
        using V2 = typename Pair2<T>::type;
        const int n2 = n >> 1;
        for (int p = tid; p < n2; p += stride) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if (!AA[c]) continue;
                const V2 xa = ld2(reinterpret_cast<const V2*>(AA[c]), p);
                double x0 = (double)xa.x, x1 = (double)xa.y;
                if (MODE == 2) {
                    double y0 = 0.0, y1 = 0.0;
                    if (BB[c]) {
                        const V2 xb = ld2(reinterpret_cast<const V2*>(BB[c]), p);
                        y0 = (double)xb.x;
                        y1 = (double)xb.y;
                    }
                    acc[c] = fmax(acc[c], fabs(x0 - y0));
                    acc[c] = fmax(acc[c], fabs(x1 - y1));
                } else {
                    if (MODE == 0) {
                        const V2 xb = ld2(reinterpret_cast<const V2*>(BB[c]), p);
                        x0 = x0 * (double)xb.x;
                        x1 = x1 * (double)xb.y;
                    }
                    acc[c] += x0;
                    acc[c] += x1;
                }
            }
        }
    } else {
        for (int t = tid; t < n; t += stride) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if (!AA[c]) continue;
                double x = (double)ld(AA[c], t);
                if (MODE == 2) {
                    acc[c] = fmax(acc[c], fabs(x - (BB[c] ? (double)ld(BB[c], t) : 0.0)));
                } else {
                    if (MODE == 0) x = x * (double)ld(BB[c], t);
                    acc[c] += x;
                }
            }
        }
    }
    if (MODE != 2) {
        // seam planes: x faces i == 0 (ny*nz of them), y faces j == 0 (nx*nz),
        // z faces k == 0 (nx*ny)
#pragma unroll
        for (int c = 0; c < DM; ++c) {
            const T* a = A[c];
            const T* b = B[c];
            if (!a || W[c] == 1.0) continue;
            const int m = (c == 0) ? D.ny * nzi : (c == 1 ? D.nx * nzi : D.nx * D.ny);
            double v = 0.0;
            for (int q = tid; q < m; q += stride) {
                int t;
                if (c == 0) t = D.nx * q;                                     // (0, j, k)
                else if (c == 1) t = (q % D.nx) + D.nx * D.ny * (q / D.nx);   // (i, 0, k)
                else t = q;                                                   // (i, j, 0)
                double x = (double)ld(a, t);
                if (MODE == 0) x = x * (double)ld(b, t);
                v += x;
            }
            acc[c] += (W[c] - 1.0) * v;
        }
    }
    __shared__ double sh[NC][kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) {
            double u = __shfl_down_sync(0xffffffffu, v, o);
            v = (MODE == 2) ? fmax(v, u) : v + u;
        }
        if (lane == 0) sh[c][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int c = 0; c < NC; ++c) {
            double v = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) v = (MODE == 2) ? fmax(v, sh[c][w]) : v + sh[c][w];
            partials[blockIdx.x * NC + c] = v;
        }
        __threadfence();
    }
    __shared__ bool last;
    if (threadIdx.x == 0) {
        unsigned prev = atomicAdd(counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // final sum in a fixed order: thread t adds partials t, t + 256, ... of
    // each component, then the same fixed warp/block tree as above
    __shared__ double fin[4];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        double v = 0.0;
        for (unsigned bidx = threadIdx.x; bidx < gridDim.x; bidx += blockDim.x) {
            double q = ((volatile double*)partials)[bidx * NC + c];
            v = (MODE == 2) ? fmax(v, q) : v + q;
        }
        for (int o = 16; o > 0; o >>= 1) {
            double u = __shfl_down_sync(0xffffffffu, v, o);
            v = (MODE == 2) ? fmax(v, u) : v + u;
        }
        __syncthreads();
        if (lane == 0) sh[c][warp] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double r = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) r = (MODE == 2) ? fmax(r, sh[c][w]) : r + sh[c][w];
            fin[c] = r;
            out[c] = r;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double su = 0.0;
        for (int c = 0; c < DM; ++c) su = su + fin[c];
        out[4] = su + (pw * pw) * fin[DM];
        double nu = sqrt(su);
        double np = pw * sqrt(fin[DM]);
        out[5] = sqrt(nu * nu + np * np);
        *counter = 0u;
    }
}

// --------------------------------------------------------------- BFBt Schur approximation pieces
// inverse_diag_lap (src_gmres/inverse_diag_lap.f90:17-250): per face the
// reciprocal of the viscous operator's diagonal without theta*alpha and dx^2
template <class T, int DM, int VISC>
__global__ void __launch_bounds__(kThreads) k_inverse_diag_lap(Dims D, Coef<T> C, T* m0, T* m1, T* m2) {
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok) return;
    Nb nb = make_nb(D, q.i, q.j, q.k);
    const int s = nb.s;
    T* m[3] = {m0, m1, m2};
    const T b = ld(C.beta, 0);
#pragma unroll
    for (int d = 0; d < DM; ++d) {
        T v;
        if (VISC == 1) {
            v = T(1) / ((DM == 3 ? T(6) : T(4)) * b);
        } else if (VISC == 2) {
            v = T(1) / ((DM == 3 ? T(8) : T(6)) * b);
        } else if constexpr (DM == 2) {
            const int t = 1 - d;
            const T be = ld(C.beta, s), bm = ld(C.beta, s + nb.om[d]);
            const T E = ld(C.bed[0], s), Ep = ld(C.bed[0], s + nb.op[t]);
            v = (VISC == -1) ? T(1) / (be + bm + Ep + E) : T(1) / (T(2) * be + T(2) * bm + Ep + E);
        } else {
            // (e1, t1), (e2, t2) of the face component as in Perm3
            const int e1 = d == 2 ? 1 : 0, t1 = d == 0 ? 1 : 0;
            const int e2 = d == 0 ? 1 : 2, t2 = d == 2 ? 1 : 2;
            const T be = ld(C.beta, s), bm = ld(C.beta, s + nb.om[d]);
            const T A = ld(C.bed[e1], s), Ap = ld(C.bed[e1], s + nb.op[t1]);
            const T B = ld(C.bed[e2], s), Bp = ld(C.bed[e2], s + nb.op[t2]);
            v = (VISC == -1) ? T(1) / (be + bm + A + Ap + B + Bp) : T(1) / (T(2) * be + T(2) * bm + A + Ap + B + Bp);
        }
        m[d][s] = v;
    }
}

// g_d = ((phi - phi(-e_d)) / dx) * m_d   (compute_grad, then multifab_mult_mult_c)
template <class T, int DM>
__global__ void __launch_bounds__(kThreads) k_grad_mul(Dims D, const T* __restrict__ phi, const T* m0, const T* m1, const T* m2, T* g0,
                                                      T* g1, T* g2, T dxinv) {
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok) return;
    Nb nb = make_nb(D, q.i, q.j, q.k);
    const int t = nb.s;
    const T p = ld(phi, t);
    const T* m[3] = {m0, m1, m2};
    T* g[3] = {g0, g1, g2};
#pragma unroll
    for (int d = 0; d < DM; ++d) g[d][t] = ((p - ld(phi, t + nb.om[d])) * dxinv) * ld(m[d], t);
}

// out = div(m * L): each face product first (multifab_mult_mult_c), then
// compute_div's differences in its order
template <class T, int DM>
__global__ void __launch_bounds__(kThreads) k_div_mul(Dims D, const T* l0, const T* l1, const T* l2, const T* m0, const T* m1,
                                                     const T* m2, T* __restrict__ out, T dxinv) {
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok) return;
    Nb nb = make_nb(D, q.i, q.j, q.k);
    const int t = nb.s;
    const T x1 = ld(l0, t + nb.op[0]) * ld(m0, t + nb.op[0]), x0 = ld(l0, t) * ld(m0, t);
    const T y1 = ld(l1, t + nb.op[1]) * ld(m1, t + nb.op[1]), y0 = ld(l1, t) * ld(m1, t);
    T v = (x1 - x0) * dxinv + (y1 - y0) * dxinv;
    if constexpr (DM == 3) {
        const T z1 = ld(l2, t + nb.op[2]) * ld(m2, t + nb.op[2]), z0 = ld(l2, t) * ld(m2, t);
        v = v + (z1 - z0) * dxinv;
    }
    out[t] = v;
}

// =============================================================== launchers
#define LMM_VISC_DISPATCH(VISC, ...)                      \
    switch (VISC) {                                       \
    case -1: { constexpr int V = -1; __VA_ARGS__; } break; \
    case 1: { constexpr int V = 1; __VA_ARGS__; } break;   \
    case -2: { constexpr int V = -2; __VA_ARGS__; } break; \
    case 2: { constexpr int V = 2; __VA_ARGS__; } break;   \
    case -3: { constexpr int V = -3; __VA_ARGS__; } break; \
    case 3: { constexpr int V = 3; __VA_ARGS__; } break;   \
    default: break;                                       \
    }

template <class T>
void launch_applyop(const LevelDev<T>& L, int visc, const T* const phi[3], T* const out[3], cudaStream_t s, int color) {
    if (L.D.wall) return wl_applyop<T>(L, visc, phi, out, s, color);
    const T dxsqinv = T(1.0 / (L.dx * L.dx));
    if (color == 0) {
        const G3 gc = geom3_tuned(TK_APPLYOP, sizeof(T), visc, L.D, L.D.nx, L.D.ny, L.D.nz * L.D.dm);
        if (L.D.dm == 2) {
            LMM_VISC_DISPATCH(visc, launch_pdl(k_applyop_c<T, 2, V>, gc.grid, gc.block, 0, s, L.D, L.coef(), phi[0], phi[1], phi[2], out[0], out[1], out[2], dxsqinv))
        } else {
            LMM_VISC_DISPATCH(visc, launch_pdl(k_applyop_c<T, 3, V>, gc.grid, gc.block, 0, s, L.D, L.coef(), phi[0], phi[1], phi[2], out[0], out[1], out[2], dxsqinv))
        }
        return;
    }
    const G3 g = geom3(L.D.nx, L.D.ny, L.D.nz);
    if (L.D.dm == 2) {
        LMM_VISC_DISPATCH(visc, (launch_pdl(k_applyop<T, 2, V>, g.grid, g.block, 0, s, L.D, L.coef(), phi[0], phi[1], phi[2], out[0], out[1], out[2], dxsqinv, color)))
    } else {
        LMM_VISC_DISPATCH(visc, (launch_pdl(k_applyop<T, 3, V>, g.grid, g.block, 0, s, L.D, L.coef(), phi[0], phi[1], phi[2], out[0], out[1], out[2], dxsqinv, color)))
    }
}

template <class T>
void launch_gs_colour(const LevelDev<T>& L, int visc, int color, const T* const rhs[3], T* const phi[3], double omega,
                      cudaStream_t s, int reverse) {
    if (L.D.wall) return wl_gs_colour<T>(L, visc, color, rhs, phi, omega, s, reverse);
    const T dxsqinv = T(1.0 / (L.dx * L.dx));
    const int comp = (color - 1) / 2;
    const int parity = (color % 2 == 1) ? 0 : 1;
    const T om = (T)omega;
    if (odd_level(L.D)) {
        const T* pin[3] = {phi[0], phi[1], phi[2]};
        T* lp[3] = {L.tmp[0], L.tmp[1], L.tmp[2]};
        launch_applyop<T>(L, visc, pin, lp, s, color);
        count_launch();
        const G3 go = geom3(L.D.nx, L.D.ny, L.D.nz);
#define CU(DM_, COMP_) launch_pdl(k_colour_update<T, DM_, V, COMP_>, go.grid, go.block, 0, s, L.D, L.coef(), rhs[COMP_], L.tmp[COMP_], phi[COMP_], parity, om, dxsqinv)
        if (L.D.dm == 2) {
            if (comp == 0) { LMM_VISC_DISPATCH(visc, CU(2, 0)) }
            else { LMM_VISC_DISPATCH(visc, CU(2, 1)) }
        } else {
            if (comp == 0) { LMM_VISC_DISPATCH(visc, CU(3, 0)) }
            else if (comp == 1) { LMM_VISC_DISPATCH(visc, CU(3, 1)) }
            else { LMM_VISC_DISPATCH(visc, CU(3, 2)) }
        }
#undef CU
        return;
    }
    const G3 g = geom3_tuned(TK_GS_COLOUR, sizeof(T), visc, L.D, L.D.nx / 2, L.D.ny, L.D.nz);
#define GS(DM_, COMP_) launch_pdl(k_gs_colour<T, DM_, V, COMP_>, g.grid, g.block, 0, s, L.D, L.coef(), rhs[COMP_], phi[0], phi[1], phi[2], parity, om, dxsqinv, reverse)
    if (L.D.dm == 2) {
        if (comp == 0) { LMM_VISC_DISPATCH(visc, GS(2, 0)) }
        else { LMM_VISC_DISPATCH(visc, GS(2, 1)) }
    } else {
        if (comp == 0) { LMM_VISC_DISPATCH(visc, GS(3, 0)) }
        else if (comp == 1) { LMM_VISC_DISPATCH(visc, GS(3, 1)) }
        else { LMM_VISC_DISPATCH(visc, GS(3, 2)) }
    }
#undef GS
}

// tile of the fused pair on one level (ok == false: use the per-colour
// kernels); tz_req > 1 forces the planes per block
struct PairGeom {
    bool ok = false;
    int TX = 0, TY = 0, TZ = 0;
};
static inline PairGeom pair_geom(const Dims& D, int tz_req) {
    PairGeom g;
    if (D.dm != 3) return g;
    if ((D.nx & 1) || (D.ny & 1) || (D.nz & 1) || D.nx < 8 || D.ny < 4 || D.nz < 2) return g;
    g.TX = D.nx < 64 ? D.nx : 64;
    if (D.nx % g.TX) return g;
    auto blocks = [&](int ty, int tz) { return (int64_t)(D.nx / g.TX) * (D.ny / ty) * (D.nz / tz); };
    g.TY = (D.ny % 8 == 0 && D.nz % 8 == 0 && blocks(8, 8) >= 444) ? 8 : 4;
    if (D.ny % g.TY) return g;
    if (tz_req > 1) {
        if (D.nz % tz_req) return g;
        g.TZ = tz_req;
    } else {
        g.TZ = (D.nz % 8 == 0 && blocks(g.TY, 8) >= 444) ? 8 : (D.nz % 4 == 0 ? 4 : 2);
    }
    g.ok = (g.TX / 2) * g.TY >= g.TX + g.TY;
    return g;
}

template <class T>
bool gs_pair_supported(const LevelDev<T>& L, int tz) {
    return !L.D.wall && pair_geom(L.D, tz).ok;
}

template <class T>
void launch_gs_pair(const LevelDev<T>& L, int visc, int comp, const T* const rhs[3], const T* const cur[3], T* out, double omega,
                    int tz, cudaStream_t s) {
    const PairGeom pg = pair_geom(L.D, tz);
    const T dxsqinv = T(1.0 / (L.dx * L.dx));
    const T om = (T)omega;
    const dim3 grid(L.D.nx / pg.TX, L.D.ny / pg.TY, L.D.nz / pg.TZ), block(pg.TX / 2, pg.TY, 1);
    const size_t smem = (size_t)(pg.TZ + 2) * (pg.TY + 2) * (pg.TX + 2) * sizeof(T);
#define GSP(COMP_)                                                                                                       \
    {                                                                                                                    \
        raise_smem_limit((const void*)k_gs_pair<T, V, COMP_>, smem);                                                     \
        k_gs_pair<T, V, COMP_><<<grid, block, smem, s>>>(L.D, L.coef(), rhs[COMP_], cur[0], cur[1], cur[2], out, pg.TX, \
                                                          pg.TY, pg.TZ, 0, om, dxsqinv);                                 \
    }
    if (comp == 0) { LMM_VISC_DISPATCH(visc, GSP(0)) }
    else if (comp == 1) { LMM_VISC_DISPATCH(visc, GSP(1)) }
    else { LMM_VISC_DISPATCH(visc, GSP(2)) }
#undef GSP
}

template <class T>
void launch_jacobi(const LevelDev<T>& L, int visc, const T* const rhs[3], const T* const pin[3], T* const pout[3],
                   double omega, cudaStream_t s) {
    if (L.D.wall) return wl_jacobi<T>(L, visc, rhs, pin, pout, omega, s);
    const T dxsqinv = T(1.0 / (L.dx * L.dx));
    const G3 g = geom3(L.D.nx, L.D.ny, L.D.nz);
    const T om = (T)omega;
    if (L.D.dm == 2) {
        LMM_VISC_DISPATCH(visc, (launch_pdl(k_jacobi<T, 2, V>, g.grid, g.block, 0, s, L.D, L.coef(), rhs[0], rhs[1], rhs[2], pin[0], pin[1], pin[2], pout[0], pout[1], pout[2], om, dxsqinv)))
    } else {
        LMM_VISC_DISPATCH(visc, (launch_pdl(k_jacobi<T, 3, V>, g.grid, g.block, 0, s, L.D, L.coef(), rhs[0], rhs[1], rhs[2], pin[0], pin[1], pin[2], pout[0], pout[1], pout[2], om, dxsqinv)))
    }
}

template <class T>
void launch_residual_restrict(const LevelDev<T>& F, const LevelDev<T>& Cc, int visc, const T* const rhs_f[3],
                              const T* const phi_f[3], T* const rhs_c[3], cudaStream_t s, int fused) {
    if (F.D.wall) return wl_residual_restrict<T>(F, Cc, visc, rhs_f, phi_f, rhs_c, s);
    const T dxsqinv = T(1.0 / (F.dx * F.dx));
    if (fused && F.D.dm == 3 && Cc.D.nx % RCX == 0 && Cc.D.ny % RCY == 0 && Cc.D.nz % RCZ == 0 && !odd_level(F.D)) {
        // residual and restriction in one pass, the residual kept in shared memory
        const dim3 grid(Cc.D.nx / RCX, Cc.D.ny / RCY, Cc.D.nz / RCZ);
        LMM_VISC_DISPATCH(visc, launch_pdl(k_resid_restrict3<T, V>, grid, dim3(kThreads), 0, s, F.D, F.coef(), rhs_f[0], rhs_f[1], rhs_f[2], phi_f[0], phi_f[1], phi_f[2], Cc.D, rhs_c[0], rhs_c[1], rhs_c[2], dxsqinv))
        return;
    }
    // residual on every fine face into F.tmp, then the pure restriction
    const G3 g = geom3_tuned(TK_RESIDUAL, sizeof(T), visc, F.D, F.D.nx, F.D.ny, F.D.nz * F.D.dm);
    if (F.D.dm == 2) {
        LMM_VISC_DISPATCH(visc, launch_pdl(k_residual_c<T, 2, V>, g.grid, g.block, 0, s, F.D, F.coef(), rhs_f[0], rhs_f[1], rhs_f[2], phi_f[0], phi_f[1], phi_f[2], F.tmp[0], F.tmp[1], F.tmp[2], dxsqinv))
    } else {
        LMM_VISC_DISPATCH(visc, launch_pdl(k_residual_c<T, 3, V>, g.grid, g.block, 0, s, F.D, F.coef(), rhs_f[0], rhs_f[1], rhs_f[2], phi_f[0], phi_f[1], phi_f[2], F.tmp[0], F.tmp[1], F.tmp[2], dxsqinv))
    }
    count_launch();
    const G3 gc = geom3(Cc.D.nx, Cc.D.ny, Cc.D.nz);
    if (F.D.dm == 2)
        launch_pdl(k_restrict<T, 2>, gc.grid, gc.block, 0, s, F.D, F.tmp[0], F.tmp[1], F.tmp[2], Cc.D, rhs_c[0], rhs_c[1], rhs_c[2]);
    else
        launch_pdl(k_restrict<T, 3>, gc.grid, gc.block, 0, s, F.D, F.tmp[0], F.tmp[1], F.tmp[2], Cc.D, rhs_c[0], rhs_c[1], rhs_c[2]);
}

template <class T>
void launch_prolong_add(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* const phi_c[3], T* const phi_f[3],
                        cudaStream_t s) {
    if (F.D.wall) return wl_prolong_add<T>(F, Cc, phi_c, phi_f, s);
    const G3 g = geom3_tuned(TK_PROLONG, sizeof(T), 0, F.D, F.D.nx, F.D.ny, F.D.nz);
    if (F.D.dm == 2)
        launch_pdl(k_prolong_add<T, 2>, g.grid, g.block, 0, s, F.D, Cc.D, phi_c[0], phi_c[1], phi_c[2], phi_f[0], phi_f[1], phi_f[2]);
    else
        launch_pdl(k_prolong_add<T, 3>, g.grid, g.block, 0, s, F.D, Cc.D, phi_c[0], phi_c[1], phi_c[2], phi_f[0], phi_f[1], phi_f[2]);
}

template <class T>
void launch_coarsen_coeffs(const LevelDev<T>& F, const LevelDev<T>& Cc, bool pressure_faces, cudaStream_t s) {
    const G3 g = geom3(Cc.D.nx, Cc.D.ny, Cc.D.nz);
    Coef<T> cf = F.coef();
    cf.alpha_uniform = 0;  // the arrays are read (and may be others below)
    if (pressure_faces) {
        for (int d = 0; d < 3; ++d) cf.alpha[d] = F.pa[d];
        if (F.D.dm == 2)
            k_coarsen<T, 2><<<g.grid, g.block, 0, s>>>(F.D, Cc.D, cf, Cc.pa[0], Cc.pa[1], Cc.pa[2], nullptr, nullptr, nullptr, nullptr, nullptr, 0);
        else
            k_coarsen<T, 3><<<g.grid, g.block, 0, s>>>(F.D, Cc.D, cf, Cc.pa[0], Cc.pa[1], Cc.pa[2], nullptr, nullptr, nullptr, nullptr, nullptr, 0);
        return;
    }
    const int dv = F.D.wall ? 2 : 1;
    if (F.D.dm == 2)
        k_coarsen<T, 2><<<g.grid, g.block, 0, s>>>(F.D, Cc.D, cf, Cc.alpha[0], Cc.alpha[1], Cc.alpha[2], Cc.beta, Cc.gamma, Cc.bed[0], Cc.bed[1], Cc.bed[2], dv);
    else
        k_coarsen<T, 3><<<g.grid, g.block, 0, s>>>(F.D, Cc.D, cf, Cc.alpha[0], Cc.alpha[1], Cc.alpha[2], Cc.beta, Cc.gamma, Cc.bed[0], Cc.bed[1], Cc.bed[2], dv);
    if (F.D.wall) {
        count_launch();
        const G3 ge = geom3(Cc.D.nx + 1, Cc.D.ny + 1, Cc.D.dm == 3 ? Cc.D.nz + 1 : Cc.D.nz);
        if (F.D.dm == 2)
            k_coarsen_edges_w<T, 2><<<ge.grid, ge.block, 0, s>>>(F.D, Cc.D, F.bed[0], F.bed[1], F.bed[2], Cc.bed[0], Cc.bed[1], Cc.bed[2]);
        else
            k_coarsen_edges_w<T, 3><<<ge.grid, ge.block, 0, s>>>(F.D, Cc.D, F.bed[0], F.bed[1], F.bed[2], Cc.bed[0], Cc.bed[1], Cc.bed[2]);
    }
}

template <class T>
void launch_cc_smooth(const LevelDev<T>& L, int parity, cudaStream_t s, int reverse) {
    const T dxsqinv = T(1.0 / (L.dx * L.dx));
    if (odd_level(L.D)) {
        const G3 go = geom3(L.D.nx, L.D.ny, L.D.nz);
        if (L.D.dm == 2)
            launch_pdl(k_cc_smooth_odd<T, 2>, go.grid, go.block, 0, s, L.D, L.pa[0], L.pa[1], L.pa[2], L.prhs, L.pphi, L.ptmp, parity, dxsqinv);
        else
            launch_pdl(k_cc_smooth_odd<T, 3>, go.grid, go.block, 0, s, L.D, L.pa[0], L.pa[1], L.pa[2], L.prhs, L.pphi, L.ptmp, parity, dxsqinv);
        count_launch();
        launch_pdl(k_copy_parity<T>, go.grid, go.block, 0, s, L.D, L.ptmp, L.pphi, parity);
        return;
    }
    const G3 g = geom3(L.D.nx / 2, L.D.ny, L.D.nz);
    const int rev = reverse ? 1 : 0;
    if (L.pa_uniform) {
        if (L.D.dm == 2)
            launch_pdl(k_cc_smooth<T, 2, true>, g.grid, g.block, 0, s, L.D, L.pa[0], L.pa[1], L.pa[2], L.prhs, L.pphi, parity, dxsqinv, L.pa_value, rev);
        else
            launch_pdl(k_cc_smooth<T, 3, true>, g.grid, g.block, 0, s, L.D, L.pa[0], L.pa[1], L.pa[2], L.prhs, L.pphi, parity, dxsqinv, L.pa_value, rev);
        return;
    }
    if (L.D.dm == 2)
        launch_pdl(k_cc_smooth<T, 2>, g.grid, g.block, 0, s, L.D, L.pa[0], L.pa[1], L.pa[2], L.prhs, L.pphi, parity, dxsqinv, T(0), rev);
    else
        launch_pdl(k_cc_smooth<T, 3>, g.grid, g.block, 0, s, L.D, L.pa[0], L.pa[1], L.pa[2], L.prhs, L.pphi, parity, dxsqinv, T(0), rev);
}

template <class T>
void launch_uniform_check(const LevelDev<T>& L, int* flag, cudaStream_t s, bool velocity) {
    const int64_t n = L.n;
    const int blocks = (int)std::min<int64_t>((n + kThreads - 1) / kThreads, 1184);
    T* const* a = velocity ? L.alpha : L.pa;
    k_uniform_check<T><<<blocks, kThreads, 0, s>>>(a[0], a[1], L.D.dm == 3 ? a[2] : nullptr, n, flag);
}

template <class T>
void launch_cc_residual_restrict(const LevelDev<T>& F, const LevelDev<T>& Cc, cudaStream_t s) {
    const T dxsqinv = T(1.0 / (F.dx * F.dx));
    const G3 g = geom3(Cc.D.nx, Cc.D.ny, Cc.D.nz);
    if (F.pa_uniform) {
        if (F.D.dm == 2)
            launch_pdl(k_cc_residual_restrict<T, 2, true>, g.grid, g.block, 0, s, F.D, F.pa[0], F.pa[1], F.pa[2], F.prhs, F.pphi, Cc.D, Cc.prhs, dxsqinv, F.pa_value);
        else
            launch_pdl(k_cc_residual_restrict<T, 3, true>, g.grid, g.block, 0, s, F.D, F.pa[0], F.pa[1], F.pa[2], F.prhs, F.pphi, Cc.D, Cc.prhs, dxsqinv, F.pa_value);
        return;
    }
    if (F.D.dm == 2)
        launch_pdl(k_cc_residual_restrict<T, 2>, g.grid, g.block, 0, s, F.D, F.pa[0], F.pa[1], F.pa[2], F.prhs, F.pphi, Cc.D, Cc.prhs, dxsqinv, T(0));
    else
        launch_pdl(k_cc_residual_restrict<T, 3>, g.grid, g.block, 0, s, F.D, F.pa[0], F.pa[1], F.pa[2], F.prhs, F.pphi, Cc.D, Cc.prhs, dxsqinv, T(0));
}

template <class T>
void launch_cc_prolong_add(const LevelDev<T>& F, const LevelDev<T>& Cc, cudaStream_t s) {
    const G3 g = geom3(F.D.nx, F.D.ny, F.D.nz);
    if (F.D.dm == 2)
        launch_pdl(k_cc_prolong_add<T, 2>, g.grid, g.block, 0, s, F.D, Cc.D, Cc.pphi, F.pphi);
    else
        launch_pdl(k_cc_prolong_add<T, 3>, g.grid, g.block, 0, s, F.D, Cc.D, Cc.pphi, F.pphi);
}

template <class T>
void launch_neg_cc_lap(const LevelDev<T>& L, const T* phi, T* out, cudaStream_t s) {
    const T dxsqinv = T(1.0 / (L.dx * L.dx));
    const G3 g = geom3(L.D.nx, L.D.ny, L.D.nz);
    if (L.D.dm == 2)
        launch_pdl(k_neg_cc_lap<T, 2>, g.grid, g.block, 0, s, L.D, L.pa[0], L.pa[1], L.pa[2], phi, out, dxsqinv);
    else
        launch_pdl(k_neg_cc_lap<T, 3>, g.grid, g.block, 0, s, L.D, L.pa[0], L.pa[1], L.pa[2], phi, out, dxsqinv);
}

template <class T>
void launch_div_plus(const LevelDev<T>& L, const T* const u[3], const T* bp, T* out, cudaStream_t s) {
    const T dxinv = T(1.0 / L.dx);
    const G3 g = geom3(L.D.nx, L.D.ny, L.D.nz);
    if (L.D.wall) {
        if (L.D.dm == 2)
            launch_pdl(k_div_plus<T, 2, true>, g.grid, g.block, 0, s, L.D, u[0], u[1], u[2], bp, out, dxinv);
        else
            launch_pdl(k_div_plus<T, 3, true>, g.grid, g.block, 0, s, L.D, u[0], u[1], u[2], bp, out, dxinv);
        return;
    }
    if (L.D.dm == 2)
        launch_pdl(k_div_plus<T, 2>, g.grid, g.block, 0, s, L.D, u[0], u[1], u[2], bp, out, dxinv);
    else
        launch_pdl(k_div_plus<T, 3>, g.grid, g.block, 0, s, L.D, u[0], u[1], u[2], bp, out, dxinv);
}

template <class T>
void launch_sub_weighted_grad(const LevelDev<T>& L, const T* const coef[3], const T* phi, T* const u[3], cudaStream_t s) {
    const T dxinv = T(1.0 / L.dx);
    const G3 g = geom3(L.D.nx, L.D.ny, L.D.nz);
    const T* c0 = coef ? coef[0] : nullptr;
    const T* c1 = coef ? coef[1] : nullptr;
    const T* c2 = coef ? coef[2] : nullptr;
    if (L.D.wall) {
        if (L.D.dm == 2)
            launch_pdl(k_sub_weighted_grad<T, 2, true>, g.grid, g.block, 0, s, L.D, c0, c1, c2, phi, u[0], u[1], u[2], dxinv);
        else
            launch_pdl(k_sub_weighted_grad<T, 3, true>, g.grid, g.block, 0, s, L.D, c0, c1, c2, phi, u[0], u[1], u[2], dxinv);
        return;
    }
    if (L.D.dm == 2)
        launch_pdl(k_sub_weighted_grad<T, 2>, g.grid, g.block, 0, s, L.D, c0, c1, c2, phi, u[0], u[1], u[2], dxinv);
    else
        launch_pdl(k_sub_weighted_grad<T, 3>, g.grid, g.block, 0, s, L.D, c0, c1, c2, phi, u[0], u[1], u[2], dxinv);
}

template <class Tin, class Tout>
void launch_convert(const Tin* in, Tout* out, int64_t n, cudaStream_t s) {
    launch_pdl(k_convert<Tin, Tout>, nblocks_for(n), kThreads, 0, s, in, out, n);
}
template <class T>
void launch_add_to(T* x, const T* y, int64_t n, cudaStream_t s) {
    launch_pdl(k_add_to<T>, nblocks_for(n), kThreads, 0, s, x, y, n);
}

template <class T>
void launch_scale_copy(const T* in, T* out, double scale, int64_t n, cudaStream_t s) {
    launch_pdl(k_scale_copy<T>, nblocks_for(n), kThreads, 0, s, in, out, (T)scale, n);
}
template <class T>
void launch_recip(const T* in, T* out, int64_t n, cudaStream_t s) {
    launch_pdl(k_recip<T>, nblocks_for(n), kThreads, 0, s, in, out, n);
}
template <class T>
void launch_fill(T* out, double v, int64_t n, cudaStream_t s) {
    launch_pdl(k_fill<T>, nblocks_for(n), kThreads, 0, s, out, (T)v, n);
}

template <class T>
void launch_reduce(const Dims& D, int mode, const T* const a[4], const T* const b[4], const double wseam[3], double pw,
                   double* partials, unsigned* counter, double* out, int nblocks, cudaStream_t s, int ninst) {
    const dim3 grid(nblocks, ninst);
    const void* pa[4] = {a[0], a[1], a[2], a[3]};
    const void* pb[4] = {b[0], b[1], b[2], b[3]};
    const int vec = reduce_pairs(D, sizeof(T), pa, pb);
#define RED(DM_, M_) launch_pdl(k_reduce<T, DM_, M_>, grid, dim3(kThreads), 0, s, D, a[0], a[1], a[2], a[3], b[0], b[1], b[2], b[3], wseam[0], wseam[1], wseam[2], pw, partials, counter, out, vec)
    if (D.dm == 2) {
        if (mode == 0) RED(2, 0); else if (mode == 1) RED(2, 1); else RED(2, 2);
    } else {
        if (mode == 0) RED(3, 0); else if (mode == 1) RED(3, 1); else RED(3, 2);
    }
#undef RED
}

template <class T>
void launch_inverse_diag_lap(const LevelDev<T>& L, int visc, T* const m[3], cudaStream_t s) {
    const G3 g = geom3(L.D.nx, L.D.ny, L.D.nz);
#define IDL(DM_, V_) k_inverse_diag_lap<T, DM_, V_><<<g.grid, g.block, 0, s>>>(L.D, L.coef(), m[0], m[1], m[2])
    if (L.D.dm == 2) {
        if (visc == -1) IDL(2, -1); else if (visc == 1) IDL(2, 1); else if (visc == -2) IDL(2, -2); else IDL(2, 2);
    } else {
        if (visc == -1) IDL(3, -1); else if (visc == 1) IDL(3, 1); else if (visc == -2) IDL(3, -2); else IDL(3, 2);
    }
#undef IDL
}

template <class T>
void launch_grad_mul(const LevelDev<T>& L, const T* phi, const T* const m[3], T* const g[3], cudaStream_t s) {
    const T dxinv = T(1.0 / L.dx);
    const G3 gg = geom3(L.D.nx, L.D.ny, L.D.nz);
    if (L.D.dm == 2)
        k_grad_mul<T, 2><<<gg.grid, gg.block, 0, s>>>(L.D, phi, m[0], m[1], m[2], g[0], g[1], g[2], dxinv);
    else
        k_grad_mul<T, 3><<<gg.grid, gg.block, 0, s>>>(L.D, phi, m[0], m[1], m[2], g[0], g[1], g[2], dxinv);
}

template <class T>
void launch_div_mul(const LevelDev<T>& L, const T* const l[3], const T* const m[3], T* out, cudaStream_t s) {
    const T dxinv = T(1.0 / L.dx);
    const G3 gg = geom3(L.D.nx, L.D.ny, L.D.nz);
    if (L.D.dm == 2)
        k_div_mul<T, 2><<<gg.grid, gg.block, 0, s>>>(L.D, l[0], l[1], l[2], m[0], m[1], m[2], out, dxinv);
    else
        k_div_mul<T, 3><<<gg.grid, gg.block, 0, s>>>(L.D, l[0], l[1], l[2], m[0], m[1], m[2], out, dxinv);
}

}  // namespace lmm
#include "gs_tma.cuh"
namespace lmm {

#define LMM_INSTANTIATE(T)                                                                                                     \
    template void launch_applyop<T>(const LevelDev<T>&, int, const T* const[3], T* const[3], cudaStream_t, int);              \
    template void launch_gs_colour<T>(const LevelDev<T>&, int, int, const T* const[3], T* const[3], double, cudaStream_t, int); \
    template void launch_jacobi<T>(const LevelDev<T>&, int, const T* const[3], const T* const[3], T* const[3], double,         \
                                   cudaStream_t);                                                                              \
    template bool gs_pair_supported<T>(const LevelDev<T>&, int);                                                               \
    template void launch_inverse_diag_lap<T>(const LevelDev<T>&, int, T* const[3], cudaStream_t);                                \
    template void launch_grad_mul<T>(const LevelDev<T>&, const T*, const T* const[3], T* const[3], cudaStream_t);                \
    template void launch_div_mul<T>(const LevelDev<T>&, const T* const[3], const T* const[3], T*, cudaStream_t);                 \
    template void launch_gs_pair<T>(const LevelDev<T>&, int, int, const T* const[3], const T* const[3], T*, double, int,        \
                                    cudaStream_t);                                                                             \
    template void launch_residual_restrict<T>(const LevelDev<T>&, const LevelDev<T>&, int, const T* const[3],                  \
                                              const T* const[3], T* const[3], cudaStream_t, int);                              \
    template void launch_prolong_add<T>(const LevelDev<T>&, const LevelDev<T>&, const T* const[3], T* const[3], cudaStream_t); \
    template void launch_coarsen_coeffs<T>(const LevelDev<T>&, const LevelDev<T>&, bool, cudaStream_t);                        \
    template void launch_cc_smooth<T>(const LevelDev<T>&, int, cudaStream_t, int);                                              \
    template void launch_cc_residual_restrict<T>(const LevelDev<T>&, const LevelDev<T>&, cudaStream_t);                        \
    template void launch_cc_prolong_add<T>(const LevelDev<T>&, const LevelDev<T>&, cudaStream_t);                              \
    template void launch_uniform_check<T>(const LevelDev<T>&, int*, cudaStream_t, bool);                                            \
    template void launch_neg_cc_lap<T>(const LevelDev<T>&, const T*, T*, cudaStream_t);                                        \
    template void launch_div_plus<T>(const LevelDev<T>&, const T* const[3], const T*, T*, cudaStream_t);                        \
    template void launch_sub_weighted_grad<T>(const LevelDev<T>&, const T* const[3], const T*, T* const[3], cudaStream_t);     \
    template void launch_scale_copy<T>(const T*, T*, double, int64_t, cudaStream_t);                                           \
    template void launch_add_to<T>(T*, const T*, int64_t, cudaStream_t);                                                      \
    template void launch_recip<T>(const T*, T*, int64_t, cudaStream_t);                                                        \
    template void launch_fill<T>(T*, double, int64_t, cudaStream_t);                                                           \
    template void launch_reduce<T>(const Dims&, int, const T* const[4], const T* const[4], const double[3], double,            \
                                   double*, unsigned*, double*, int, cudaStream_t, int);                                      \
    template bool gs_tma_supported<T>(const LevelDev<T>&, int, int, int);                                                     \
    template cudaError_t launch_gs_pair_tma<T>(const LevelDev<T>&, int, int, const T* const[3], const T* const[3], T*, double, \
                                               int, int, int*, cudaStream_t);

}  // namespace lmm
