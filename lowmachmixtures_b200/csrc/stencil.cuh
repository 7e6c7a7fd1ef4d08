// stencil.cuh - per-face staggered viscous operator on the compact periodic
// layout (device side).
//
// One face value of  L phi = theta*alpha phi - div(beta grad phi [+ grad^T]) ...
// exactly as src_common/stag_applyop.f90:204-1067 writes it, and the diagonal
// of src_gmres/stag_mg_solver.f90:1637-2463 (stag_mg_update).  Operand order
// follows the Fortran expression by expression; the FP64 build is compiled
// without FMA contraction, so every face is the reference's rounding
// sequence.  Face component d is stored compactly: n periodic faces per
// direction, (i + nx*(j + ny*k)), the seam face hi+1 implied equal to face 0.
//
// Directions: a face of component d at index (i,j,k) sits between cells
// idx-e_d and idx.  The two transverse directions t1 < t2 and the edge arrays
// follow the Fortran: x faces use (xy, xz), y faces (xy, yz), z faces
// (xz, yz); 2D uses the single nodal beta_ed.
#pragma once
#include <cstdint>

namespace lmm {

// neighbour offsets (with periodic wrap) of one index; 32-bit indices
// (a field holds at most 2^31 - 1 entries)
struct Nb {
    int s;       // linear index
    int op[3];   // offset to +1 in direction d
    int om[3];   // offset to -1 in direction d
};

struct Dims {
    int nx, ny, nz;  // nz == 1 in 2D
    int dm;
};

__device__ __forceinline__ Nb make_nb(const Dims& D, int i, int j, int k) {
    Nb b;
    const int sx = 1, sy = D.nx, sz = D.nx * D.ny;
    b.s = i + sy * j + sz * k;
    b.op[0] = (i == D.nx - 1) ? -(D.nx - 1) * sx : sx;
    b.om[0] = (i == 0) ? (D.nx - 1) * sx : -sx;
    b.op[1] = (j == D.ny - 1) ? -(D.ny - 1) * sy : sy;
    b.om[1] = (j == 0) ? (D.ny - 1) * sy : -sy;
    if (D.dm == 3) {
        b.op[2] = (k == D.nz - 1) ? -(D.nz - 1) * sz : sz;
        b.om[2] = (k == 0) ? (D.nz - 1) * sz : -sz;
    } else {
        b.op[2] = 0;
        b.om[2] = 0;
    }
    return b;
}

template <class T>
struct Coef {
    const T* alpha[3];   // theta * alpha_fc on faces
    const T* beta;       // cells
    const T* bed[3];     // 2D: [0] nodal; 3D: xy, xz, yz edges
    const T* gamma;      // cells
};

template <class T>
__device__ __forceinline__ T ld(const T* p, int i) {
    return __ldg(p + i);
}

// loads of arrays a kernel may also write (phi, rhs):
//   LD 0  read-only path (__ldg): the array is not written by this kernel;
//   LD 1  plain load: written by other threads of the same block between
//         __syncthreads();
//   LD 2  L2 load (ld.global.cg): written by other blocks of the same
//         thread-block cluster between cluster barriers.
template <int LD, class T>
__device__ __forceinline__ T ldp(const T* p, int i) {
    if constexpr (LD == 0)
        return __ldg(p + i);
    else if constexpr (LD == 1)
        return p[i];
    else
        return __ldcg(p + i);
}

// periodic wrap of an index known to lie in [-n, 2n)
__device__ __forceinline__ int wrapi(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// 3D launch geometry: x covers i (or i/2 for one colour), y covers j, z covers k
struct Pos {
    int i, j, k;
    bool ok;
};
__device__ __forceinline__ Pos pos3(int nx, int ny) {
    Pos p;
    p.i = blockIdx.x * blockDim.x + threadIdx.x;
    p.j = blockIdx.y * blockDim.y + threadIdx.y;
    p.k = blockIdx.z;
    p.ok = (p.i < nx) && (p.j < ny);
    return p;
}

// compile-time direction bookkeeping of a 3D face component
template <int COMP> struct Perm3;
template <> struct Perm3<0> { static constexpr int t1 = 1, t2 = 2, e1 = 0, e2 = 1; };
template <> struct Perm3<1> { static constexpr int t1 = 0, t2 = 2, e1 = 0, e2 = 2; };
template <> struct Perm3<2> { static constexpr int t1 = 0, t2 = 1, e1 = 1, e2 = 2; };

// ------------------------------------------------------------------ 3D
// The face value with the own component's centre p0 and its six neighbours
// nb = {+x, -x, +y, -y, +z, -z} supplied by the caller (global memory for the
// plain kernels, shared memory for the fused red/black pair); the other two
// components and the coefficients are read through phi / C.
template <class T, int VISC, int D, int LD = 0, class TP = T>
__device__ __forceinline__ T face_L3_own(const T p0, const T (&nb)[6], const TP* const phi[3], const Coef<T>& C, const Nb& n,
                                         T dxsqinv, T b, T c) {
    constexpr int t1 = Perm3<D>::t1, t2 = Perm3<D>::t2, e1 = Perm3<D>::e1, e2 = Perm3<D>::e2;
    const T onethird = T(1) / T(3), twothirds = T(2) / T(3), fourthirds = T(4) / T(3);
    const int s = n.s;
    const T a = ld(C.alpha[D], s);
    if (VISC == 1) {
        T nbs = nb[0] + nb[1] + nb[2] + nb[3] + nb[4] + nb[5];
        return p0 * (a + T(6) * b * dxsqinv) - nbs * b * dxsqinv;
    }
    const TP* q1 = phi[t1];
    const TP* q2 = phi[t2];
    const T ppd = nb[2 * D], pmd = nb[2 * D + 1];
    const T pp1 = nb[2 * t1], pm1 = nb[2 * t1 + 1];
    const T pp2 = nb[2 * t2], pm2 = nb[2 * t2 + 1];
    // cross terms q(i,+t) , q(i) , q(i-d,+t) , q(i-d)
    const T c10 = (T)ldp<LD>(q1, s + n.op[t1]), c11 = (T)ldp<LD>(q1, s), c12 = (T)ldp<LD>(q1, s + n.om[D] + n.op[t1]), c13 = (T)ldp<LD>(q1, s + n.om[D]);
    const T c20 = (T)ldp<LD>(q2, s + n.op[t2]), c21 = (T)ldp<LD>(q2, s), c22 = (T)ldp<LD>(q2, s + n.om[D] + n.op[t2]), c23 = (T)ldp<LD>(q2, s + n.om[D]);
    if (VISC == 2) {
        return p0 * (a + T(8) * b * dxsqinv) -
               (T(2) * ppd + T(2) * pmd + pp1 + pm1 + pp2 + pm2 + c10 - c11 - c12 + c13 + c20 - c21 - c22 + c23) * b * dxsqinv;
    }
    if (VISC == 3) {
        T nbt;
        if (D == 0) nbt = pp1 + pm1 + pp2 + pm2;              // j+1, j-1, k+1, k-1
        else if (D == 1) nbt = pp1 + pm1 + pp2 + pm2;         // i+1, i-1, k+1, k-1
        else nbt = pp1 + pm1 + pp2 + pm2;                     // i+1, i-1, j+1, j-1
        return p0 * (a + (T(20) * b * onethird + T(2) * c) * dxsqinv) -
               ((ppd + pmd) * (fourthirds * b + c) + nbt * b +
                (c10 - c11 - c12 + c13 + c20 - c21 - c22 + c23) * (onethird * b + c)) * dxsqinv;
    }
    const T be = ld(C.beta, s), bm = ld(C.beta, s + n.om[D]);
    const T E1 = ld(C.bed[e1], s), E1p = ld(C.bed[e1], s + n.op[t1]);
    const T E2 = ld(C.bed[e2], s), E2p = ld(C.bed[e2], s + n.op[t2]);
    if (VISC == -1) {
        return p0 * (a + (be + bm + E1 + E1p + E2 + E2p) * dxsqinv) -
               (ppd * be + pmd * bm + pp1 * E1p + pm1 * E1 + pp2 * E2p + pm2 * E2) * dxsqinv;
    }
    if (VISC == -2) {
        return p0 * (a + (T(2) * be + T(2) * bm + E1 + E1p + E2 + E2p) * dxsqinv) -
               (T(2) * ppd * be + T(2) * pmd * bm + pp1 * E1p + pm1 * E1 + pp2 * E2p + pm2 * E2 + c10 * E1p - c11 * E1 - c12 * E1p +
                c13 * E1 + c20 * E2p - c21 * E2 - c22 * E2p + c23 * E2) * dxsqinv;
    }
    // VISC == -3
    const T g = ld(C.gamma, s), gm = ld(C.gamma, s + n.om[D]);
    return p0 * (a + (fourthirds * be + g + fourthirds * bm + gm + E1 + E1p + E2 + E2p) * dxsqinv) -
           (ppd * (fourthirds * be + g) + pmd * (fourthirds * bm + gm) + pp1 * E1p + pm1 * E1 + pp2 * E2p + pm2 * E2 +
            c10 * (E1p - twothirds * be + g) - c11 * (E1 - twothirds * be + g) - c12 * (E1p - twothirds * bm + gm) +
            c13 * (E1 - twothirds * bm + gm) + c20 * (E2p - twothirds * be + g) - c21 * (E2 - twothirds * be + g) -
            c22 * (E2p - twothirds * bm + gm) + c23 * (E2 - twothirds * bm + gm)) * dxsqinv;
}

template <class T, int VISC, int D, int LD = 0, class TP = T>
__device__ __forceinline__ T face_L3(const TP* const phi[3], const Coef<T>& C, const Nb& n, T dxsqinv, T b, T c) {
    const TP* p = phi[D];
    const int s = n.s;
    const T p0 = (T)ldp<LD>(p, s);
    const T nb[6] = {(T)ldp<LD>(p, s + n.op[0]), (T)ldp<LD>(p, s + n.om[0]), (T)ldp<LD>(p, s + n.op[1]),
                     (T)ldp<LD>(p, s + n.om[1]), (T)ldp<LD>(p, s + n.op[2]), (T)ldp<LD>(p, s + n.om[2])};
    return face_L3_own<T, VISC, D, LD, TP>(p0, nb, phi, C, n, dxsqinv, b, c);
}

template <class T, int VISC, int D>
__device__ __forceinline__ T face_diag3(const Coef<T>& C, const Nb& n, T dxsqinv, T b, T c) {
    constexpr int t1 = Perm3<D>::t1, t2 = Perm3<D>::t2, e1 = Perm3<D>::e1, e2 = Perm3<D>::e2;
    const int s = n.s;
    const T a = ld(C.alpha[D], s);
    if (VISC == 1) return a + T(6) * b * dxsqinv;
    if (VISC == 2) return a + T(8) * b * dxsqinv;
    if (VISC == 3) return a + (T(20) / T(3) * b + T(2) * c) * dxsqinv;
    const T be = ld(C.beta, s), bm = ld(C.beta, s + n.om[D]);
    const T E1 = ld(C.bed[e1], s), E1p = ld(C.bed[e1], s + n.op[t1]);
    const T E2 = ld(C.bed[e2], s), E2p = ld(C.bed[e2], s + n.op[t2]);
    if (VISC == -1) return a + (be + bm + E1 + E1p + E2 + E2p) * dxsqinv;
    if (VISC == -2) return a + (T(2) * be + T(2) * bm + E1 + E1p + E2 + E2p) * dxsqinv;
    const T fourthirds = T(4) / T(3);
    const T g = ld(C.gamma, s), gm = ld(C.gamma, s + n.om[D]);
    return a + (fourthirds * be + g + fourthirds * bm + gm + E1 + E1p + E2 + E2p) * dxsqinv;
}

// ------------------------------------------------------------------ 2D
template <class T, int VISC, int D, int LD = 0, class TP = T>
__device__ __forceinline__ T face_L2(const TP* const phi[3], const Coef<T>& C, const Nb& n, T dxsqinv, T b, T c) {
    constexpr int t = 1 - D;
    const T onethird = T(1) / T(3), twothirds = T(2) / T(3), fourthirds = T(4) / T(3);
    const TP* p = phi[D];
    const TP* q = phi[t];
    const int s = n.s;
    const T p0 = (T)ldp<LD>(p, s);
    const T a = ld(C.alpha[D], s);
    const T ppd = (T)ldp<LD>(p, s + n.op[D]), pmd = (T)ldp<LD>(p, s + n.om[D]);
    const T ppt = (T)ldp<LD>(p, s + n.op[t]), pmt = (T)ldp<LD>(p, s + n.om[t]);
    if (VISC == 1) {
        // x: i+1, i-1, j+1, j-1 ; y: j+1, j-1, i+1, i-1  (own direction first)
        return p0 * (a + T(4) * b * dxsqinv) - (ppd + pmd + ppt + pmt) * b * dxsqinv;
    }
    const T c0 = (T)ldp<LD>(q, s + n.op[t]), c1 = (T)ldp<LD>(q, s), c2 = (T)ldp<LD>(q, s + n.om[D] + n.op[t]), c3 = (T)ldp<LD>(q, s + n.om[D]);
    if (VISC == 2) {
        return p0 * (a + T(6) * b * dxsqinv) - (T(2) * ppd + T(2) * pmd + ppt + pmt + c0 - c1 - c2 + c3) * b * dxsqinv;
    }
    if (VISC == 3) {
        return p0 * (a + (T(14) * b * onethird + T(2) * c) * dxsqinv) -
               ((ppd + pmd) * (fourthirds * b + c) + (ppt + pmt) * b + (c0 - c1 - c2 + c3) * (onethird * b + c)) * dxsqinv;
    }
    const T be = ld(C.beta, s), bm = ld(C.beta, s + n.om[D]);
    const T E = ld(C.bed[0], s), Ep = ld(C.bed[0], s + n.op[t]);
    if (VISC == -1) {
        return p0 * (a + (be + bm + Ep + E) * dxsqinv) - (ppd * be + pmd * bm + ppt * Ep + pmt * E) * dxsqinv;
    }
    if (VISC == -2) {
        return p0 * (a + (T(2) * be + T(2) * bm + Ep + E) * dxsqinv) -
               (T(2) * ppd * be + T(2) * pmd * bm + ppt * Ep + pmt * E + c0 * Ep - c1 * E - c2 * Ep + c3 * E) * dxsqinv;
    }
    const T g = ld(C.gamma, s), gm = ld(C.gamma, s + n.om[D]);
    return p0 * (a + (fourthirds * be + g + fourthirds * bm + gm + Ep + E) * dxsqinv) -
           (ppd * (fourthirds * be + g) + pmd * (fourthirds * bm + gm) + ppt * Ep + pmt * E + c0 * (Ep - twothirds * be + g) -
            c1 * (E - twothirds * be + g) - c2 * (Ep - twothirds * bm + gm) + c3 * (E - twothirds * bm + gm)) * dxsqinv;
}

template <class T, int VISC, int D>
__device__ __forceinline__ T face_diag2(const Coef<T>& C, const Nb& n, T dxsqinv, T b, T c) {
    constexpr int t = 1 - D;
    const int s = n.s;
    const T a = ld(C.alpha[D], s);
    if (VISC == 1) return a + T(4) * b * dxsqinv;
    if (VISC == 2) return a + T(6) * b * dxsqinv;
    if (VISC == 3) return a + (T(14) / T(3) * b + T(2) * c) * dxsqinv;
    const T be = ld(C.beta, s), bm = ld(C.beta, s + n.om[D]);
    const T E = ld(C.bed[0], s), Ep = ld(C.bed[0], s + n.op[t]);
    if (VISC == -1) return a + (be + bm + E + Ep) * dxsqinv;
    if (VISC == -2) return a + (T(2) * be + T(2) * bm + E + Ep) * dxsqinv;
    const T fourthirds = T(4) / T(3);
    const T g = ld(C.gamma, s), gm = ld(C.gamma, s + n.om[D]);
    return a + (fourthirds * be + g + fourthirds * bm + gm + E + Ep) * dxsqinv;
}

template <class T, int DM, int VISC, int D, int LD = 0, class TP = T>
__device__ __forceinline__ T face_L(const TP* const phi[3], const Coef<T>& C, const Nb& n, T dxsqinv, T b, T c) {
    if constexpr (DM == 2)
        return face_L2<T, VISC, D, LD, TP>(phi, C, n, dxsqinv, b, c);
    else
        return face_L3<T, VISC, D, LD, TP>(phi, C, n, dxsqinv, b, c);
}
template <class T, int DM, int VISC, int D>
__device__ __forceinline__ T face_diag(const Coef<T>& C, const Nb& n, T dxsqinv, T b, T c) {
    if constexpr (DM == 2)
        return face_diag2<T, VISC, D>(C, n, dxsqinv, b, c);
    else
        return face_diag3<T, VISC, D>(C, n, dxsqinv, b, c);
}

}  // namespace lmm
