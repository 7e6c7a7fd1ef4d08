// stencil.cuh - per-face staggered viscous operator on the compact layout
// (device side), periodic or with walls.
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
//
// Walls (template flag W): along a wall-bounded direction d the face array of
// component d stores faces lo..hi, face lo being the wall (kept zero) and the
// wall face hi+1 implied zero; every other array stores its n cells; an edge
// array nodal in d stores n+1 nodes.  Neighbour values across a wall follow
// the reference's ghost fills (multifab_physbc_stag.f90): the wall-normal
// component is zero on and behind the wall (physbc_domainvel), a transverse
// component's ghost is -interior at a no-slip wall and +interior at a slip
// wall (physbc_macvel).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace lmm {

// ------------------------------------------------------------ bounds checks
// A build with -DLMM_BOUNDS_CHECK tests every load through ld / ldp: a
// global address must lie in one of the registered device allocations (the
// arenas and learned-stage blocks of the live handles, and the caller's
// arrays of an entry point that reads them in place), a shared-memory one
// (the single-CTA coarse tails) within the CTA's shared memory.  A load outside them is skipped
// (it reads zero), counted, and the first such address kept; the host reads
// and clears the record after each solve and reports LMM_ERR_BOUNDS.  Device
// globals are per translation unit (no relocatable device code), so each
// unit that includes this header owns a table and a record, reached through
// the host functions LMM_BC_UNIT(name) defines in it.
namespace bc {
constexpr int kRanges = 64;
struct Table {
    unsigned long long lo[kRanges], hi[kRanges];
    int n;
};
struct Record {
    unsigned long long count, first;
};
}  // namespace bc
#ifdef LMM_BOUNDS_CHECK
static __device__ bc::Table g_bc_table;
static __device__ bc::Record g_bc_record;
// a load of `bytes` at p: in shared memory it must lie within this CTA's
// shared memory (static + dynamic), in global memory within a registered
// allocation; other windows (local) are not tracked
__device__ __forceinline__ bool bc_ok(const void* p, unsigned bytes) {
    const unsigned long long a = reinterpret_cast<unsigned long long>(p);
    bool ok;
    if (__isShared(p)) {
        // the CTA's own shared memory (static, then dynamic) follows the
        // reserved region: offsets [cap, cap + total)
        unsigned total, cap;
        asm("mov.u32 %0, %%total_smem_size;" : "=r"(total));
        asm("mov.u32 %0, %%reserved_smem_offset_cap;" : "=r"(cap));
        const unsigned long long off = __cvta_generic_to_shared(p);
        ok = off >= cap && off + bytes <= (unsigned long long)cap + total;
    } else if (__isGlobal(p)) {
        ok = false;
        const int n = g_bc_table.n;
        for (int r = 0; r < n && !ok; ++r) ok = a >= g_bc_table.lo[r] && a + bytes <= g_bc_table.hi[r];
    } else {
        ok = true;
    }
    if (!ok && atomicAdd(&g_bc_record.count, 1ull) == 0ull) g_bc_record.first = a;
    return ok;
}
#define LMM_BC_UNIT(name)                                                                             \
    cudaError_t lmm_bc_sync_##name(const lmm::bc::Table& t) {                                         \
        return cudaMemcpyToSymbol(lmm::g_bc_table, &t, sizeof(t));                                    \
    }                                                                                                 \
    cudaError_t lmm_bc_take_##name(lmm::bc::Record* r) {                                              \
        const lmm::bc::Record z{0ull, 0ull};                                                          \
        cudaError_t e = cudaMemcpyFromSymbol(r, lmm::g_bc_record, sizeof(*r));                        \
        return e == cudaSuccess ? cudaMemcpyToSymbol(lmm::g_bc_record, &z, sizeof(z)) : e;            \
    }
#else
#define LMM_BC_UNIT(name)
#endif
// the translation units that include this header, each ending in
// LMM_BC_UNIT(its name)
#define LMM_BC_UNITS(X) \
    X(autotune) X(kernels_fp32) X(kernels_fp64) X(krylov) X(learned) X(net) X(nn) X(noalloc) X(solver) X(stochastic) X(walls_fp32) X(walls_fp64)

// neighbour offsets (with periodic wrap) of one index; 32-bit indices
// (a field holds at most 2^31 - 1 entries)
struct Dims {
    // 2D: nz is the number of independent instances stacked along the third
    // index (1 for one grid; a batch of B problems of one grid has nz = B).
    // The third index of a 2D array is then the instance: never wrapped,
    // coarsened or part of a colour.
    int nx, ny, nz;
    int dm;
    // bit d of wall: direction d is bounded by walls (else periodic); bit d
    // of slip_lo / slip_hi: that wall is a slip wall (else no-slip).  Plain
    // members (Dims sits in shared-memory structs): every Dims built sets
    // them, all zero for a periodic box.
    int wall, slip_lo, slip_hi;
};

struct Nb {
    int s;       // linear index
    int op[3];   // offset to +1 in direction d
    int om[3];   // offset to -1 in direction d
    // walls (make_nbw only): the position, the grid, and bit masks of the
    // wall-bounded directions in which it is the first (lo) / last (hi) index
    int i, j, k, lo, hi;
    Dims D;
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

// Neighbours on a grid with walls: as make_nb, except that an offset does
// not wrap across a wall (it is 0 at the wall-adjacent index; the value
// read there is then scaled by wall_mul).
__device__ __forceinline__ Nb make_nbw(const Dims& D, int i, int j, int k) {
    Nb b = make_nb(D, i, j, k);
    b.i = i;
    b.j = j;
    b.k = k;
    b.lo = 0;
    b.hi = 0;
    b.D = D;
    const int x[3] = {i, j, k}, n[3] = {D.nx, D.ny, D.nz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d >= D.dm || !((D.wall >> d) & 1)) continue;
        if (x[d] == 0) {
            b.lo |= 1 << d;
            b.om[d] = 0;
        }
        if (x[d] == n[d] - 1) {
            b.hi |= 1 << d;
            b.op[d] = 0;
        }
    }
    return b;
}

// multiplier of the value of component c read at the +1 (plus) / -1
// neighbour in direction d: 1 inside, 0 for the wall-normal component
// across its wall, -1 / +1 for a transverse component at a no-slip / slip
// wall (the neighbour offset is then 0: the ghost mirrors the face itself)
__device__ __forceinline__ int wall_mul(const Nb& n, int c, int d, bool plus) {
    const int bit = 1 << d;
    if (!((plus ? n.hi : n.lo) & bit)) return 1;
    if (d == c) return 0;
    return ((plus ? n.D.slip_hi : n.D.slip_lo) & bit) ? 1 : -1;
}
template <class T>
__device__ __forceinline__ T wapply(int m, T v) {
    return m > 0 ? v : (m < 0 ? -v : T(0));
}
// true when the face of component c at this position is a wall face
__device__ __forceinline__ bool wall_face(const Nb& n, int c) { return (n.lo >> c) & 1; }

// edge array e (2D: the nodal array; 3D: 0 xy, 1 xz, 2 yz) is nodal in d
__host__ __device__ __forceinline__ bool edge_nodal(int dm, int e, int d) {
    if (dm == 2) return d < 2;
    return (e == 0) ? (d != 2) : (e == 1 ? (d != 1) : (d != 0));
}
// entries of edge array e along direction d (n+1 along a nodal wall-bounded d)
__host__ __device__ __forceinline__ int edge_ext(const Dims& D, int e, int d) {
    const int n = (d == 0) ? D.nx : (d == 1 ? D.ny : D.nz);
    return n + ((d < D.dm && ((D.wall >> d) & 1) && edge_nodal(D.dm, e, d)) ? 1 : 0);
}
__host__ __device__ __forceinline__ int64_t edge_count(const Dims& D, int e) {
    return (int64_t)edge_ext(D, e, 0) * edge_ext(D, e, 1) * (D.dm == 3 ? edge_ext(D, e, 2) : D.nz);
}
// index of edge e at the face position of n, moved +1 along direction t
// (t < 0: no move); a periodic direction wraps
__device__ __forceinline__ int edge_at(const Nb& n, int e, int t) {
    int x[3] = {n.i, n.j, n.k};
    const int nn[3] = {n.D.nx, n.D.ny, n.D.nz};
    if (t >= 0) {
        x[t] += 1;
        if (x[t] == nn[t] && !((n.D.wall >> t) & 1)) x[t] = 0;
    }
    const int ex = edge_ext(n.D, e, 0), ey = edge_ext(n.D, e, 1);
    return x[0] + ex * (x[1] + ey * x[2]);
}

// the third index's share of a colour: (i + j + k) % 2 in 3D, (i + j) % 2
// in 2D (k is the instance)
template <int DM>
__host__ __device__ __forceinline__ int ck(int k) {
    return DM == 3 ? k : 0;
}

template <class T>
struct Coef {
    const T* alpha[3];   // theta * alpha_fc on faces
    const T* beta;       // cells
    const T* bed[3];     // 2D: [0] nodal; 3D: xy, xz, yz edges
    const T* gamma;      // cells
    // every face of every alpha array holds alpha_u (checked on the device
    // at each coefficient load): the operator takes it as a scalar instead
    // of reading the arrays -- the value each load would return, so the
    // same bits.  Set by LevelDev::coef(), the only place a Coef is made.
    int alpha_uniform;
    T alpha_u;
};

template <class T>
__device__ __forceinline__ T ld(const T* p, int i) {
#ifdef LMM_BOUNDS_CHECK
    if (!bc_ok(p + i, sizeof(T))) return T(0);
#endif
    return __ldg(p + i);
}

// a pair of entries (double2 / float2) by one load, checked as one access
template <class V>
__device__ __forceinline__ V ld2(const V* p, int i) {
#ifdef LMM_BOUNDS_CHECK
    if (!bc_ok(p + i, sizeof(V))) return V{};
#endif
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
#ifdef LMM_BOUNDS_CHECK
    if (!bc_ok(p + i, sizeof(T))) return T(0);
#endif
    if constexpr (LD == 0)
        return __ldg(p + i);
    else if constexpr (LD == 1)
        return p[i];
    else
        return __ldcg(p + i);
}

// theta*alpha of face s of component d
template <class T>
__device__ __forceinline__ T alpha_at(const Coef<T>& C, int d, int s) {
    return C.alpha_uniform ? C.alpha_u : ld(C.alpha[d], s);
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
template <class T, int VISC, int D, int LD = 0, class TP = T, bool W = false>
__device__ __forceinline__ T face_L3_own(const T p0, const T (&nb)[6], const TP* const phi[3], const Coef<T>& C, const Nb& n,
                                         T dxsqinv, T b, T c) {
    constexpr int t1 = Perm3<D>::t1, t2 = Perm3<D>::t2, e1 = Perm3<D>::e1, e2 = Perm3<D>::e2;
    const T onethird = T(1) / T(3), twothirds = T(2) / T(3), fourthirds = T(4) / T(3);
    const int s = n.s;
    const T a = alpha_at(C, D, s);
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
    T c10 = (T)ldp<LD>(q1, s + n.op[t1]), c11 = (T)ldp<LD>(q1, s), c12 = (T)ldp<LD>(q1, s + n.om[D] + n.op[t1]), c13 = (T)ldp<LD>(q1, s + n.om[D]);
    T c20 = (T)ldp<LD>(q2, s + n.op[t2]), c21 = (T)ldp<LD>(q2, s), c22 = (T)ldp<LD>(q2, s + n.om[D] + n.op[t2]), c23 = (T)ldp<LD>(q2, s + n.om[D]);
    if constexpr (W) {
        // component t across its own wall at +t is zero (the face is not a wall face, so -d stays inside)
        const int m1 = wall_mul(n, t1, t1, true), m2 = wall_mul(n, t2, t2, true);
        c10 = wapply(m1, c10);
        c12 = wapply(m1, c12);
        c20 = wapply(m2, c20);
        c22 = wapply(m2, c22);
    }
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
    const T E1 = ld(C.bed[e1], W ? edge_at(n, e1, -1) : s), E1p = ld(C.bed[e1], W ? edge_at(n, e1, t1) : s + n.op[t1]);
    const T E2 = ld(C.bed[e2], W ? edge_at(n, e2, -1) : s), E2p = ld(C.bed[e2], W ? edge_at(n, e2, t2) : s + n.op[t2]);
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

template <class T, int VISC, int D, int LD = 0, class TP = T, bool W = false>
__device__ __forceinline__ T face_L3(const TP* const phi[3], const Coef<T>& C, const Nb& n, T dxsqinv, T b, T c) {
    const TP* p = phi[D];
    const int s = n.s;
    const T p0 = (T)ldp<LD>(p, s);
    T nb[6] = {(T)ldp<LD>(p, s + n.op[0]), (T)ldp<LD>(p, s + n.om[0]), (T)ldp<LD>(p, s + n.op[1]),
               (T)ldp<LD>(p, s + n.om[1]), (T)ldp<LD>(p, s + n.op[2]), (T)ldp<LD>(p, s + n.om[2])};
    if constexpr (W) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            nb[2 * d] = wapply(wall_mul(n, D, d, true), nb[2 * d]);
            nb[2 * d + 1] = wapply(wall_mul(n, D, d, false), nb[2 * d + 1]);
        }
    }
    return face_L3_own<T, VISC, D, LD, TP, W>(p0, nb, phi, C, n, dxsqinv, b, c);
}

template <class T, int VISC, int D, bool W = false>
__device__ __forceinline__ T face_diag3(const Coef<T>& C, const Nb& n, T dxsqinv, T b, T c) {
    constexpr int t1 = Perm3<D>::t1, t2 = Perm3<D>::t2, e1 = Perm3<D>::e1, e2 = Perm3<D>::e2;
    const int s = n.s;
    const T a = alpha_at(C, D, s);
    if (VISC == 1) return a + T(6) * b * dxsqinv;
    if (VISC == 2) return a + T(8) * b * dxsqinv;
    if (VISC == 3) return a + (T(20) / T(3) * b + T(2) * c) * dxsqinv;
    const T be = ld(C.beta, s), bm = ld(C.beta, s + n.om[D]);
    const T E1 = ld(C.bed[e1], W ? edge_at(n, e1, -1) : s), E1p = ld(C.bed[e1], W ? edge_at(n, e1, t1) : s + n.op[t1]);
    const T E2 = ld(C.bed[e2], W ? edge_at(n, e2, -1) : s), E2p = ld(C.bed[e2], W ? edge_at(n, e2, t2) : s + n.op[t2]);
    if (VISC == -1) return a + (be + bm + E1 + E1p + E2 + E2p) * dxsqinv;
    if (VISC == -2) return a + (T(2) * be + T(2) * bm + E1 + E1p + E2 + E2p) * dxsqinv;
    const T fourthirds = T(4) / T(3);
    const T g = ld(C.gamma, s), gm = ld(C.gamma, s + n.om[D]);
    return a + (fourthirds * be + g + fourthirds * bm + gm + E1 + E1p + E2 + E2p) * dxsqinv;
}

// ------------------------------------------------------------ face arithmetic on values
// L phi of one 3D face of component D from its loaded operands: p0 and nb =
// {+x, -x, +y, -y, +z, -z} of the own component, q1/q2 the cross terms
// {q(s+t), q(s), q(s-d+t), q(s-d)} of components t1, t2, a = theta alpha,
// be/bm = beta at s and s-d, E1/E1p and E2/E2p the two edge arrays at s and
// s+t, g/gm = gamma at s and s-d; b, c the constant beta, gamma of |visc|
// 1..3.  Same expressions, same order as face_L3_own.
template <class T, int VISC>
__device__ __forceinline__ T face_L3_vals(T p0, const T (&nb)[6], int D, const T (&q1)[4], const T (&q2)[4], T a, T be, T bm,
                                          T E1, T E1p, T E2, T E2p, T g, T gm, T dxsqinv, T b, T c) {
    const T onethird = T(1) / T(3), twothirds = T(2) / T(3), fourthirds = T(4) / T(3);
    if (VISC == 1) {
        T nbs = nb[0] + nb[1] + nb[2] + nb[3] + nb[4] + nb[5];
        return p0 * (a + T(6) * b * dxsqinv) - nbs * b * dxsqinv;
    }
    const int t1 = (D == 0) ? 1 : 0, t2 = (D == 2) ? 1 : 2;
    const T ppd = nb[2 * D], pmd = nb[2 * D + 1];
    const T pp1 = nb[2 * t1], pm1 = nb[2 * t1 + 1];
    const T pp2 = nb[2 * t2], pm2 = nb[2 * t2 + 1];
    const T c10 = q1[0], c11 = q1[1], c12 = q1[2], c13 = q1[3];
    const T c20 = q2[0], c21 = q2[1], c22 = q2[2], c23 = q2[3];
    if (VISC == 2) {
        return p0 * (a + T(8) * b * dxsqinv) -
               (T(2) * ppd + T(2) * pmd + pp1 + pm1 + pp2 + pm2 + c10 - c11 - c12 + c13 + c20 - c21 - c22 + c23) * b * dxsqinv;
    }
    if (VISC == 3) {
        const T nbt = pp1 + pm1 + pp2 + pm2;
        return p0 * (a + (T(20) * b * onethird + T(2) * c) * dxsqinv) -
               ((ppd + pmd) * (fourthirds * b + c) + nbt * b +
                (c10 - c11 - c12 + c13 + c20 - c21 - c22 + c23) * (onethird * b + c)) * dxsqinv;
    }
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
    return p0 * (a + (fourthirds * be + g + fourthirds * bm + gm + E1 + E1p + E2 + E2p) * dxsqinv) -
           (ppd * (fourthirds * be + g) + pmd * (fourthirds * bm + gm) + pp1 * E1p + pm1 * E1 + pp2 * E2p + pm2 * E2 +
            c10 * (E1p - twothirds * be + g) - c11 * (E1 - twothirds * be + g) - c12 * (E1p - twothirds * bm + gm) +
            c13 * (E1 - twothirds * bm + gm) + c20 * (E2p - twothirds * be + g) - c21 * (E2 - twothirds * be + g) -
            c22 * (E2p - twothirds * bm + gm) + c23 * (E2 - twothirds * bm + gm)) * dxsqinv;
}

// the diagonal of the same face (face_diag3's expressions)
template <class T, int VISC>
__device__ __forceinline__ T face_diag3_vals(T a, T be, T bm, T E1, T E1p, T E2, T E2p, T g, T gm, T dxsqinv, T b, T c) {
    if (VISC == 1) return a + T(6) * b * dxsqinv;
    if (VISC == 2) return a + T(8) * b * dxsqinv;
    if (VISC == 3) return a + (T(20) / T(3) * b + T(2) * c) * dxsqinv;
    if (VISC == -1) return a + (be + bm + E1 + E1p + E2 + E2p) * dxsqinv;
    if (VISC == -2) return a + (T(2) * be + T(2) * bm + E1 + E1p + E2 + E2p) * dxsqinv;
    const T fourthirds = T(4) / T(3);
    return a + (fourthirds * be + g + fourthirds * bm + gm + E1 + E1p + E2 + E2p) * dxsqinv;
}

// One Gauss-Seidel update of a 3D face of component D on a periodic grid,
// phi + omega (rhs - L phi) / diag, with every operand read once from
// global memory and L phi and the diagonal formed from the same values
// (face_L3_vals, face_diag3_vals: face_L3 / face_diag3's expressions, so
// the same bits).
template <class T, int VISC, int D>
__device__ __forceinline__ T face_update3(const T* const phi[3], const Coef<T>& C, const T* rhs, const Nb& n, T dxsqinv, T b,
                                          T c, T omega) {
    constexpr int t1 = Perm3<D>::t1, t2 = Perm3<D>::t2, e1 = Perm3<D>::e1, e2 = Perm3<D>::e2;
    const int s = n.s;
    const T* p = phi[D];
    const T p0 = ld(p, s);
    const T nb[6] = {ld(p, s + n.op[0]), ld(p, s + n.om[0]), ld(p, s + n.op[1]),
                     ld(p, s + n.om[1]), ld(p, s + n.op[2]), ld(p, s + n.om[2])};
    T q1[4] = {T(0), T(0), T(0), T(0)}, q2[4] = {T(0), T(0), T(0), T(0)};
    if constexpr (VISC == 2 || VISC == 3 || VISC == -2 || VISC == -3) {
        const T* a1 = phi[t1];
        const T* a2 = phi[t2];
        q1[0] = ld(a1, s + n.op[t1]);
        q1[1] = ld(a1, s);
        q1[2] = ld(a1, s + n.om[D] + n.op[t1]);
        q1[3] = ld(a1, s + n.om[D]);
        q2[0] = ld(a2, s + n.op[t2]);
        q2[1] = ld(a2, s);
        q2[2] = ld(a2, s + n.om[D] + n.op[t2]);
        q2[3] = ld(a2, s + n.om[D]);
    }
    const T a = alpha_at(C, D, s);
    T be = T(0), bm = T(0), E1 = T(0), E1p = T(0), E2 = T(0), E2p = T(0), g = T(0), gm = T(0);
    if constexpr (VISC < 0) {
        be = ld(C.beta, s);
        bm = ld(C.beta, s + n.om[D]);
        E1 = ld(C.bed[e1], s);
        E1p = ld(C.bed[e1], s + n.op[t1]);
        E2 = ld(C.bed[e2], s);
        E2p = ld(C.bed[e2], s + n.op[t2]);
    }
    if constexpr (VISC == -3) {
        g = ld(C.gamma, s);
        gm = ld(C.gamma, s + n.om[D]);
    }
    const T Lp = face_L3_vals<T, VISC>(p0, nb, D, q1, q2, a, be, bm, E1, E1p, E2, E2p, g, gm, dxsqinv, b, c);
    const T fac = face_diag3_vals<T, VISC>(a, be, bm, E1, E1p, E2, E2p, g, gm, dxsqinv, b, c);
    return p0 + omega * (ld(rhs, s) - Lp) / fac;
}

// ------------------------------------------------------------------ 2D
template <class T, int VISC, int D, int LD = 0, class TP = T, bool W = false>
__device__ __forceinline__ T face_L2(const TP* const phi[3], const Coef<T>& C, const Nb& n, T dxsqinv, T b, T c) {
    constexpr int t = 1 - D;
    const T onethird = T(1) / T(3), twothirds = T(2) / T(3), fourthirds = T(4) / T(3);
    const TP* p = phi[D];
    const TP* q = phi[t];
    const int s = n.s;
    const T p0 = (T)ldp<LD>(p, s);
    const T a = alpha_at(C, D, s);
    T ppd = (T)ldp<LD>(p, s + n.op[D]), pmd = (T)ldp<LD>(p, s + n.om[D]);
    T ppt = (T)ldp<LD>(p, s + n.op[t]), pmt = (T)ldp<LD>(p, s + n.om[t]);
    if constexpr (W) {
        ppd = wapply(wall_mul(n, D, D, true), ppd);
        pmd = wapply(wall_mul(n, D, D, false), pmd);
        ppt = wapply(wall_mul(n, D, t, true), ppt);
        pmt = wapply(wall_mul(n, D, t, false), pmt);
    }
    if (VISC == 1) {
        // x: i+1, i-1, j+1, j-1 ; y: j+1, j-1, i+1, i-1  (own direction first)
        return p0 * (a + T(4) * b * dxsqinv) - (ppd + pmd + ppt + pmt) * b * dxsqinv;
    }
    T c0 = (T)ldp<LD>(q, s + n.op[t]), c1 = (T)ldp<LD>(q, s), c2 = (T)ldp<LD>(q, s + n.om[D] + n.op[t]), c3 = (T)ldp<LD>(q, s + n.om[D]);
    if constexpr (W) {
        const int m = wall_mul(n, t, t, true);
        c0 = wapply(m, c0);
        c2 = wapply(m, c2);
    }
    if (VISC == 2) {
        return p0 * (a + T(6) * b * dxsqinv) - (T(2) * ppd + T(2) * pmd + ppt + pmt + c0 - c1 - c2 + c3) * b * dxsqinv;
    }
    if (VISC == 3) {
        return p0 * (a + (T(14) * b * onethird + T(2) * c) * dxsqinv) -
               ((ppd + pmd) * (fourthirds * b + c) + (ppt + pmt) * b + (c0 - c1 - c2 + c3) * (onethird * b + c)) * dxsqinv;
    }
    const T be = ld(C.beta, s), bm = ld(C.beta, s + n.om[D]);
    const T E = ld(C.bed[0], W ? edge_at(n, 0, -1) : s), Ep = ld(C.bed[0], W ? edge_at(n, 0, t) : s + n.op[t]);
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

template <class T, int VISC, int D, bool W = false>
__device__ __forceinline__ T face_diag2(const Coef<T>& C, const Nb& n, T dxsqinv, T b, T c) {
    constexpr int t = 1 - D;
    const int s = n.s;
    const T a = alpha_at(C, D, s);
    if (VISC == 1) return a + T(4) * b * dxsqinv;
    if (VISC == 2) return a + T(6) * b * dxsqinv;
    if (VISC == 3) return a + (T(14) / T(3) * b + T(2) * c) * dxsqinv;
    const T be = ld(C.beta, s), bm = ld(C.beta, s + n.om[D]);
    const T E = ld(C.bed[0], W ? edge_at(n, 0, -1) : s), Ep = ld(C.bed[0], W ? edge_at(n, 0, t) : s + n.op[t]);
    if (VISC == -1) return a + (be + bm + E + Ep) * dxsqinv;
    if (VISC == -2) return a + (T(2) * be + T(2) * bm + E + Ep) * dxsqinv;
    const T fourthirds = T(4) / T(3);
    const T g = ld(C.gamma, s), gm = ld(C.gamma, s + n.om[D]);
    return a + (fourthirds * be + g + fourthirds * bm + gm + E + Ep) * dxsqinv;
}

template <class T, int DM, int VISC, int D, int LD = 0, class TP = T, bool W = false>
__device__ __forceinline__ T face_L(const TP* const phi[3], const Coef<T>& C, const Nb& n, T dxsqinv, T b, T c) {
    if constexpr (DM == 2)
        return face_L2<T, VISC, D, LD, TP, W>(phi, C, n, dxsqinv, b, c);
    else
        return face_L3<T, VISC, D, LD, TP, W>(phi, C, n, dxsqinv, b, c);
}
template <class T, int DM, int VISC, int D, bool W = false>
__device__ __forceinline__ T face_diag(const Coef<T>& C, const Nb& n, T dxsqinv, T b, T c) {
    if constexpr (DM == 2)
        return face_diag2<T, VISC, D, W>(C, n, dxsqinv, b, c);
    else
        return face_diag3<T, VISC, D, W>(C, n, dxsqinv, b, c);
}

}  // namespace lmm
