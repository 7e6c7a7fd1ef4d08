// gs_tma.cuh - both Gauss-Seidel colours of one velocity component in one
// launch, with every operand staged in shared memory by the tensor-memory
// accelerator (TMA).
//
// Reference loop: the colour loop of stag_mg_solver.f90:363-401
// (stag_applyop_level with the colour, then stag_mg_update), i.e. colours
// 2*COMP+1 ("red", faces with i+j+k even) then 2*COMP+2 ("black") of the
// 3D smoother, stag_applyop.f90:707-815 and stag_mg_solver.f90:2036-2463.
//
// Design (3D, periodic, even sizes, variable viscosity visc_type -1/-2/-3,
// instantiated row lengths 32/64/128/256; other levels use the per-colour
// kernels):
//  - A CTA owns a tile of TY full rows (all i) of one k-slab of KZ planes.
//    It marches through the slab plane by plane: at step s it updates the
//    red faces of plane r (the TY tile rows plus one ring row below and
//    above) into a shared-memory ring of red planes, then the black faces
//    of the plane behind r, whose six same-component neighbours are all red
//    and all in shared memory.  The red planes just outside the slab are
//    computed too (never written): red values depend only on the input
//    arrays, so a face computed by two CTAs has the same bits in both.
//  - Component x and y march in +k, component z in -k: then every step
//    reads the input planes r-1, r, r+1 only (z faces read x, y, beta and
//    gamma one plane below; y and x faces read z one plane above).
//  - Inputs: a ring of four plane sets (every staged array's rows of one
//    plane), filled by 3D-box cp.async.bulk.tensor copies (box: all i x the
//    rows the stencil needs x one plane), one mbarrier per set with the copy
//    bytes as transaction count; the plane two steps ahead is requested at
//    the start of a step, so one plane is always in flight while the CTA
//    computes.  A tile whose rows wrap around the periodic y boundary
//    fetches each run of consecutive rows with one contiguous bulk copy
//    (cp.async.bulk), two or three per array instead of one per row: every
//    TMA operation has a fixed cost, and one copy per row made those CTAs
//    the stragglers of the launch.
//  - Row length and tile rows are compile-time, so every shared-memory
//    operand is a per-step register plus an immediate offset (see the
//    thread layout at the kernel).
//  - Out of place: the inputs are never written; the new values of
//    component COMP (red and black) go to `out` as aligned pairs (i, i+1).
//  - Arithmetic: face_L3_vals / face_diag3_vals restate the expressions of
//    face_L3_own / face_diag3 operand for operand, so the FP64 build (no
//    contraction) gives the bits of the per-colour kernels and the oracle.
//  - Every mbarrier wait is bounded; on a timeout the CTA records an error,
//    waits (bounded again) for its own copies in flight and returns.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "kernels.h"
#include "pdl.cuh"
#include "stencil.cuh"

namespace lmm {

namespace gst {

constexpr int kNS = 4;    // plane sets of the ring (5 where one CTA per SM has the room: Geo::NS)
constexpr int kRNS = 3;   // red-value plane slots
constexpr unsigned kSpinLimit = 1u << 22;

// staged arrays
enum { A_P = 0, A_Q1, A_Q2, A_RHS, A_AL, A_BE, A_E1, A_E2, A_GA, A_N };

__host__ __device__ constexpr bool staged(int visc, int a) {
    return a == A_P || a == A_RHS || a == A_AL ||
           ((a == A_Q1 || a == A_Q2) && (visc == 2 || visc == 3 || visc == -2 || visc == -3)) ||
           ((a == A_BE || a == A_E1 || a == A_E2) && visc < 0) || (a == A_GA && visc == -3);
}
// rows of array a below the tile's first row / above its last row that the
// red faces of the tile and its two ring rows read (component comp)
__host__ __device__ constexpr int rows_lo(int comp, int a) {
    return a == A_P ? 2 : (comp == 1 && (a == A_Q1 || a == A_Q2 || a == A_BE || a == A_GA)) ? 2 : 1;
}
__host__ __device__ constexpr int rows_hi(int comp, int a) {
    return a == A_P ? 2
                    : ((comp == 0 && (a == A_Q1 || a == A_E1)) || (comp == 2 && (a == A_Q2 || a == A_E2))) ? 2 : 1;
}

// kernel arguments (the tensor maps travel separately as a grid constant)
template <class T>
struct Args {
    Dims D;
    int TY;        // tile rows (divides ny)
    int slabs;     // k-slabs (grid = ny / TY * slabs)
    int dir;       // +1: march in +k (components x, y); -1: in -k (z)
    T omega, dxsqinv;
    T* out;
    int* err;
    const T* src[A_N];   // the staged arrays (rows that wrap in y are fetched by bulk copies)
};

struct Maps {
    CUtensorMap tile[A_N];   // box: nx x (TY + lo + hi) rows x 1 plane
};

__device__ __forceinline__ uint32_t su32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void bar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count));
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
// true once the phase with this parity has completed; false after kSpinLimit polls
__device__ __forceinline__ bool bar_wait(uint64_t* b, unsigned parity) {
    const uint32_t a = su32(b);
    for (unsigned it = 0; it < kSpinLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (it > 32) __nanosleep(32);
    }
    return false;
}
// contiguous bulk load (16-byte aligned addresses, size a multiple of 16)
// completing on mbarrier b
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(su32(dst)),
                 "l"(src), "r"(bytes), "r"(su32(b))
                 : "memory");
}
// 3D tile load (x, y, z coordinates in elements) completing on mbarrier b
__device__ __forceinline__ void tma_load3(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* b) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            su32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(su32(b))
        : "memory");
}

template <class T>
struct Vec2;
template <>
struct Vec2<float> {
    using type = float2;
};
template <>
struct Vec2<double> {
    using type = double2;
};

// compile-time geometry of one instantiation: row length NX, tile rows TY
template <class T, int VISC, int COMP, int NX, int TY>
struct Geo {
    static constexpr int HALF = NX / 2;
    static constexpr int rows(int a) { return staged(VISC, a) ? TY + rows_lo(COMP, a) + rows_hi(COMP, a) : 0; }
    // element offset of array a inside one plane set (all staged arrays of one plane)
    static constexpr int off(int a) {
        int o = 0;
        for (int b = 0; b < a; ++b) o += rows(b) * NX;
        return o;
    }
    static constexpr int SS = off(A_N);            // elements of one plane set
    static constexpr int RS = HALF + 1;            // red-value row stride (padded: no bank conflicts)
    static constexpr int RP = (TY + 2) * RS;       // red-value plane
    static constexpr int THREADS = TY * HALF;      // one thread per face pair of the tile
    static constexpr size_t BAR_BYTES = 128;
    static constexpr size_t SET_BYTES = (size_t)SS * sizeof(T);
    static constexpr size_t smem_for(int ns) { return BAR_BYTES + ns * SET_BYTES + (size_t)kRNS * RP * sizeof(T); }
    // plane sets: a fifth (two planes requested ahead instead of one) when
    // four already leave room for a single CTA per SM and five still fit
    static constexpr int NS = (smem_for(4) > 113 * 1024 && smem_for(5) <= 227 * 1024) ? 5 : 4;
    static constexpr size_t SMEM = smem_for(NS);
};

// Thread layout: one thread per face pair (i = 2q, 2q + 1) of the tile:
// thread t takes x-pair q = (t / 2) % (NX / 2) in tile row
// lj = 2 ((t / 2) / (NX / 2)) + (t & 1).  It updates the black face of its
// pair in each plane and the red face of its pair; the two ring rows' red
// faces (rows -1 and TY) go to the threads of rows 0 and 1 as a second
// item.  In one plane a thread's faces sit in one column (i = 2q + the
// parity of j + k), so a step computes the column and its two periodic
// neighbours once, and every shared-memory operand is a per-step register
// plus a compile-time offset.  Adjacent lanes take the two rows of a pair,
// whose faces lie in different columns: no bank conflicts.
template <class T, int VISC, int COMP, int NX, int TY>
__global__ void __launch_bounds__(TY * NX / 2, 1) k_gs_pair_tma(const Args<T> A, const __grid_constant__ Maps M) {
    using G = Geo<T, VISC, COMP, NX, TY>;
    constexpr int HALF = G::HALF, SS = G::SS, RS = G::RS, RP = G::RP, NS = G::NS;
    constexpr int D = COMP;
    constexpr int t1 = (D == 0) ? 1 : 0, t2 = (D == 2) ? 1 : 2;
    constexpr int ex[3] = {1, 0, 0}, ey[3] = {0, 1, 0}, ez[3] = {0, 0, 1};
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
    T* set = reinterpret_cast<T*>(smem + G::BAR_BYTES);               // NS plane sets
    T* red = reinterpret_cast<T*>(smem + G::BAR_BYTES + NS * G::SET_BYTES);  // kRNS red planes
    pdl_enter();
    const int ny = A.D.ny, nz = A.D.nz;
    const int tiles_y = ny / TY;
    const int ty = blockIdx.x % tiles_y, slab = blockIdx.x / tiles_y;
    const int j0 = ty * TY;
    const int kb = nz / A.slabs, krem = nz % A.slabs;
    const int KZ = kb + (slab < krem ? 1 : 0);
    const int k0 = slab * kb + (slab < krem ? slab : krem);
    const int dir = A.dir;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q = (tid >> 1) % HALF;
    const int g = 2 * ((tid >> 1) / HALF) + (tid & 1);   // this thread's tile row
    const bool ring = g < 2;                              // also a ring row's red face (row -1 + TY + 1 + g)
    const int qp = (q == HALF - 1) ? 0 : q + 1, qm = (q == 0) ? HALF - 1 : q - 1;
    auto plane_of = [&](int L) {
        const int p = (dir > 0) ? (k0 - 2 + L) : (k0 + KZ + 1 - L);
        return p < 0 ? p + nz : (p >= nz ? p - nz : p);
    };
    const bool wraps = (j0 - 2 < 0) || (j0 + TY + 2 > ny);

    if (tid == 0) {
        for (int b = 0; b < NS; ++b) bar_init(&bars[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // warp 0 requests plane L of every staged array into plane set L % NS
    auto issue = [&](int L) {
        const int p = plane_of(L);
        T* dst0 = set + (L % NS) * SS;
        uint64_t* b = &bars[L % NS];
        if (lane == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            bar_expect_tx(b, (uint32_t)(SS * sizeof(T)));
        }
        __syncwarp();
        if (!wraps) {
            for (int a = lane; a < A_N; a += 32)
                if (staged(VISC, a)) tma_load3(dst0 + G::off(a), &M.tile[a], 0, j0 - rows_lo(COMP, a), p, b);
        } else {
            // rows that wrap around the periodic y boundary: each run of
            // consecutive rows of one plane is contiguous in memory, one bulk
            // copy per run (two, or three when the tile spans every row)
            for (int a = lane; a < A_N; a += 32) {
                if (!staged(VISC, a)) continue;
                const int H = G::rows(a);
                int jg = j0 - rows_lo(COMP, a);
                while (jg < 0) jg += ny;
                for (int r = 0; r < H;) {
                    const int run = min(H - r, ny - jg);
                    bulk_load(dst0 + G::off(a) + r * NX, A.src[a] + ((int64_t)p * ny + jg) * NX, (uint32_t)(run * NX * sizeof(T)), b);
                    r += run;
                    jg = 0;
                }
            }
        }
    };
    if (warp == 0)
        for (int L = 0; L < NS && L <= KZ + 3; ++L) issue(L);
    int issued = NS < KZ + 4 ? NS : KZ + 4;

    const T om = A.omega, dxsqinv = A.dxsqinv;
    bool failed = false;

    // one face of the strip: `col` = its column and the two neighbours,
    // `sb` = the plane-set bases of planes -1, 0, +1 (march direction
    // applied), m0 = the element offset of the face's row (relative to the
    // row the array's row 0 corresponds to, before rows_lo)
    struct Cols {
        int c, p, m;
    };
    auto op = [&](const T* base, int a, int dzo, int dyo, int dxo, const int (&sb)[3], const Cols& cl, int rowoff) -> T {
        const int col = dxo > 0 ? cl.p : (dxo < 0 ? cl.m : cl.c);
        return base[sb[1 + dzo] + G::off(a) + (rowoff + rows_lo(COMP, a) + dyo) * NX + col];
    };
    auto face = [&](T p0, const T (&nb)[6], const int (&sb)[3], const Cols& cl, int rowoff) -> T {
        T q1[4] = {T(0), T(0), T(0), T(0)}, q2[4] = {T(0), T(0), T(0), T(0)};
        T be = T(0), bm = T(0), E1 = T(0), E1p = T(0), E2 = T(0), E2p = T(0), gg = T(0), gm = T(0);
        const T a = op(set, A_AL, 0, 0, 0, sb, cl, rowoff);
        const T rhs = op(set, A_RHS, 0, 0, 0, sb, cl, rowoff);
        if constexpr (VISC == -2 || VISC == -3) {
            q1[0] = op(set, A_Q1, ez[t1], ey[t1], ex[t1], sb, cl, rowoff);
            q1[1] = op(set, A_Q1, 0, 0, 0, sb, cl, rowoff);
            q1[2] = op(set, A_Q1, ez[t1] - ez[D], ey[t1] - ey[D], ex[t1] - ex[D], sb, cl, rowoff);
            q1[3] = op(set, A_Q1, -ez[D], -ey[D], -ex[D], sb, cl, rowoff);
            q2[0] = op(set, A_Q2, ez[t2], ey[t2], ex[t2], sb, cl, rowoff);
            q2[1] = op(set, A_Q2, 0, 0, 0, sb, cl, rowoff);
            q2[2] = op(set, A_Q2, ez[t2] - ez[D], ey[t2] - ey[D], ex[t2] - ex[D], sb, cl, rowoff);
            q2[3] = op(set, A_Q2, -ez[D], -ey[D], -ex[D], sb, cl, rowoff);
        }
        be = op(set, A_BE, 0, 0, 0, sb, cl, rowoff);
        bm = op(set, A_BE, -ez[D], -ey[D], -ex[D], sb, cl, rowoff);
        E1 = op(set, A_E1, 0, 0, 0, sb, cl, rowoff);
        E1p = op(set, A_E1, ez[t1], ey[t1], ex[t1], sb, cl, rowoff);
        E2 = op(set, A_E2, 0, 0, 0, sb, cl, rowoff);
        E2p = op(set, A_E2, ez[t2], ey[t2], ex[t2], sb, cl, rowoff);
        if constexpr (VISC == -3) {
            gg = op(set, A_GA, 0, 0, 0, sb, cl, rowoff);
            gm = op(set, A_GA, -ez[D], -ey[D], -ex[D], sb, cl, rowoff);
        }
        const T Lp = face_L3_vals<T, VISC>(p0, nb, D, q1, q2, a, be, bm, E1, E1p, E2, E2p, gg, gm, dxsqinv, T(0), T(0));
        const T fac = face_diag3_vals<T, VISC>(a, be, bm, E1, E1p, E2, E2p, gg, gm, dxsqinv, T(0), T(0));
        return p0 + om * (rhs - Lp) / fac;
    };
    using V2 = typename Vec2<T>::type;

#pragma unroll 1
    for (int s = 0; s <= KZ + 1; ++s) {
        // request the plane NS - 2 steps ahead into the set freed by step s - 1
        if (s >= 1 && s + NS - 1 <= KZ + 3) {
            if (warp == 0) issue(s + NS - 1);
            issued = s + NS;
        }
        {
            bool ok = true;
            for (int L = (s == 0 ? 0 : s + 2); L <= s + 2; ++L) ok = ok && bar_wait(&bars[L % NS], (L / NS) & 1);
            failed = __syncthreads_or(!ok);
            if (failed) break;
        }
        // red faces of plane L = s + 1: red row rr = g (tile row g - 1), and
        // for the threads of rows 0 and 1 also rr = TY + g (tile row TY + g - 1)
        {
            const int L = s + 1;
            const int r = plane_of(L);
            const int sb[3] = {((L - dir) % NS) * SS, (L % NS) * SS, ((L + dir) % NS) * SS};
            const int par = (j0 + g + 1 + r) & 1;   // red: i + j + k even, j = j0 - 1 + g (+ TY, even)
            Cols cl;
            cl.c = 2 * q + par;
            cl.p = (cl.c == NX - 1) ? 0 : cl.c + 1;
            cl.m = (cl.c == 0) ? NX - 1 : cl.c - 1;
            T* rs = red + (L % kRNS) * RP + g * RS + q;
#pragma unroll
            for (int m = 0; m < 2; ++m) {
                if (m == 1 && !ring) break;
                const int rowoff = g - 1 + m * TY;   // tile row lj of this face
                const T p0 = op(set, A_P, 0, 0, 0, sb, cl, rowoff);
                const T nb[6] = {op(set, A_P, 0, 0, 1, sb, cl, rowoff), op(set, A_P, 0, 0, -1, sb, cl, rowoff),
                                 op(set, A_P, 0, 1, 0, sb, cl, rowoff), op(set, A_P, 0, -1, 0, sb, cl, rowoff),
                                 op(set, A_P, 1, 0, 0, sb, cl, rowoff), op(set, A_P, -1, 0, 0, sb, cl, rowoff)};
                rs[m * TY * RS] = face(p0, nb, sb, cl, rowoff);
            }
        }
        __syncthreads();
        // black face of plane L = s in tile row g, stored with its red partner
        if (s >= 2) {
            const int L = s;
            const int bpl = plane_of(L);
            const int sb[3] = {((L - dir) % NS) * SS, (L % NS) * SS, ((L + dir) % NS) * SS};
            const int par = (j0 + g + bpl) & 1;     // the pair's red face is i = 2q + par
            Cols cl;
            cl.c = 2 * q + 1 - par;
            cl.p = (cl.c == NX - 1) ? 0 : cl.c + 1;
            cl.m = (cl.c == 0) ? NX - 1 : cl.c - 1;
            const T* r0 = red + (L % kRNS) * RP + g * RS;
            const T* rup = red + ((L + dir) % kRNS) * RP + g * RS;
            const T* rdn = red + ((L - dir) % kRNS) * RP + g * RS;
            const int xp = par == 0 ? qp : q, xm = par == 0 ? q : qm;   // red neighbours in x
            T* orow = A.out + ((int64_t)bpl * ny + j0 + g) * NX + 2 * q;
            {
                const int rowoff = g;                  // tile row lj
                constexpr int rr = 1;                  // red row of lj (relative to g)
                const T nb[6] = {r0[rr * RS + xp], r0[rr * RS + xm], r0[(rr + 1) * RS + q], r0[(rr - 1) * RS + q],
                                 rup[rr * RS + q], rdn[rr * RS + q]};
                const T p0 = op(set, A_P, 0, 0, 0, sb, cl, rowoff);
                const T vb = face(p0, nb, sb, cl, rowoff);
                const T vr = r0[rr * RS + q];
                V2 pr;
                pr.x = par == 0 ? vr : vb;
                pr.y = par == 0 ? vb : vr;
                *reinterpret_cast<V2*>(orow) = pr;
            }
        }
        __syncthreads();
    }
    if (failed) {
        if (tid == 0) atomicExch(A.err, 1);
        // the copies in flight must land before the CTA's shared memory is
        // released: the last plane requested into each set (earlier ones in
        // a set were waited for before it was reused), bounded again
        for (int L = (issued > NS ? issued - NS : 0); L < issued; ++L) bar_wait(&bars[L % NS], (L / NS) & 1);
        __syncthreads();
    }
}

}  // namespace gst
}  // namespace lmm

// ============================================================ host side
namespace lmm {
namespace gst {

// the driver's tensor-map encoder, fetched through the runtime (the
// library does not link libcuda)
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                                 const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline EncodeTiled encoder() {
    static EncodeTiled fn = []() -> EncodeTiled {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<EncodeTiled>(p);
    }();
    return fn;
}

// A 3D tensor map over one compact array (nx, ny, nz) with box nx x rows x 1,
// cached per (array, grid, rows): encoding is a host-only call, but the
// maps of one level are the same on every launch.
template <class T>
cudaError_t make_map(CUtensorMap* m, const T* base, const Dims& D, int rows) {
    using Key = std::tuple<const void*, int, int, int, int, int>;
    static std::mutex mu;
    static std::map<Key, CUtensorMap> cache;
    const Key key(base, D.nx, D.ny, D.nz, rows, (int)sizeof(T));
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            *m = it->second;
            return cudaSuccess;
        }
    }
    EncodeTiled enc = encoder();
    if (!enc) return cudaErrorNotSupported;
    const cuuint64_t dims[3] = {(cuuint64_t)D.nx, (cuuint64_t)D.ny, (cuuint64_t)D.nz};
    const cuuint64_t strides[2] = {(cuuint64_t)D.nx * sizeof(T), (cuuint64_t)D.nx * D.ny * sizeof(T)};
    const cuuint32_t box[3] = {(cuuint32_t)D.nx, (cuuint32_t)rows, 1u};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    CUtensorMap t;
    std::memset(&t, 0, sizeof(t));
    const CUresult r = enc(&t, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                           const_cast<T*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = t;
    *m = t;
    return cudaSuccess;
}

// shared-memory bytes of one instantiation (the same sums as Geo)
inline size_t smem_bytes(size_t w, int visc, int comp, int NX, int TY) {
    size_t rows = 0;
    for (int a = 0; a < A_N; ++a)
        if (staged(visc, a)) rows += (size_t)TY + rows_lo(comp, a) + rows_hi(comp, a);
    auto with = [&](size_t ns) { return 128 + ns * rows * NX * w + (size_t)kRNS * (TY + 2) * (NX / 2 + 1) * w; };
    return (with(4) > 113 * 1024 && with(5) <= 227 * 1024) ? with(5) : with(4);
}
constexpr size_t kMaxSmem = 227 * 1024;   // dynamic shared memory one CTA may use

// instantiated (element bytes, row length NX, tile rows TY), the preferred
// tile first for each (w, NX)
struct GeoKey {
    int w, nx, ty;
};
constexpr GeoKey kGeos[] = {{4, 128, 8}, {4, 128, 4}, {4, 256, 4}, {4, 64, 8}, {4, 64, 16}, {4, 32, 8}, {4, 32, 16},
                            {8, 128, 4}, {8, 64, 8}, {8, 64, 4}, {8, 32, 8}, {8, 32, 16}};

// the launch geometry of one level and component
struct Plan {
    bool ok = false;
    int TY = 0, slabs = 0;
    size_t smem = 0;
};

// Whether a level runs the TMA pair kernel, and its geometry.  ty_req > 0
// forces the rows per tile, slabs_req > 0 the k-slabs; sms = the device's
// SM count (the grid is sized to about one wave of resident CTAs).
inline Plan plan(const Dims& D, int visc, int comp, size_t w, int ty_req, int slabs_req, int sms) {
    Plan none;
    if (D.dm != 3 || D.wall || visc >= 0) return none;
    if ((D.nx & 1) || (D.ny & 1) || (D.nz & 1) || D.nz < 2) return none;
    Plan p;
    for (const GeoKey& g : kGeos) {
        if (g.w != (int)w || g.nx != D.nx) continue;
        if (ty_req > 0 && g.ty != ty_req) continue;
        if (D.ny % g.ty) continue;
        const size_t sm = smem_bytes(w, visc, comp, g.nx, g.ty);
        if (sm > kMaxSmem) continue;
        p.TY = g.ty;
        p.smem = sm;
        break;
    }
    if (p.TY == 0) return none;
    const int tiles = D.ny / p.TY;
    const int per_sm = std::max<int>(1, (int)((228 * 1024) / (p.smem + 1024)));
    int slabs = slabs_req > 0 ? slabs_req : std::max(1, sms * per_sm / tiles);
    slabs = std::min(slabs, slabs_req > 0 ? D.nz : std::max(1, D.nz / 2));
    p.slabs = slabs;
    p.ok = true;
    return p;
}

template <class T, int VISC, int COMP, int NX, int TY>
cudaError_t launch_geo(const Args<T>& a, const Maps& m, unsigned blocks, cudaStream_t s) {
    using G = Geo<T, VISC, COMP, NX, TY>;
    if constexpr (G::SMEM > kMaxSmem) {
        return cudaErrorInvalidValue;
    } else {
        auto kern = k_gs_pair_tma<T, VISC, COMP, NX, TY>;
        const cudaError_t e = raise_smem_limit((const void*)kern, G::SMEM);
        if (e != cudaSuccess) return e;
        launch_pdl(kern, dim3(blocks), dim3(G::THREADS), G::SMEM, s, a, m);
        return cudaSuccess;
    }
}

template <class T, int VISC, int COMP>
cudaError_t launch_comp(const Args<T>& a, const Maps& m, unsigned blocks, int nx, int ty, cudaStream_t s) {
    if constexpr (sizeof(T) == 4) {
        if (nx == 128 && ty == 8) return launch_geo<T, VISC, COMP, 128, 8>(a, m, blocks, s);
        if (nx == 128 && ty == 4) return launch_geo<T, VISC, COMP, 128, 4>(a, m, blocks, s);
        if (nx == 256 && ty == 4) return launch_geo<T, VISC, COMP, 256, 4>(a, m, blocks, s);
        if (nx == 64 && ty == 8) return launch_geo<T, VISC, COMP, 64, 8>(a, m, blocks, s);
        if (nx == 64 && ty == 16) return launch_geo<T, VISC, COMP, 64, 16>(a, m, blocks, s);
        if (nx == 32 && ty == 8) return launch_geo<T, VISC, COMP, 32, 8>(a, m, blocks, s);
        if (nx == 32 && ty == 16) return launch_geo<T, VISC, COMP, 32, 16>(a, m, blocks, s);
    } else {
        if (nx == 128 && ty == 4) return launch_geo<T, VISC, COMP, 128, 4>(a, m, blocks, s);
        if (nx == 64 && ty == 8) return launch_geo<T, VISC, COMP, 64, 8>(a, m, blocks, s);
        if (nx == 64 && ty == 4) return launch_geo<T, VISC, COMP, 64, 4>(a, m, blocks, s);
        if (nx == 32 && ty == 8) return launch_geo<T, VISC, COMP, 32, 8>(a, m, blocks, s);
        if (nx == 32 && ty == 16) return launch_geo<T, VISC, COMP, 32, 16>(a, m, blocks, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace gst
}  // namespace lmm

namespace lmm {

inline int device_sms() {
    static int sms[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (sms[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        sms[dev] = v;
    }
    return sms[dev];
}

template <class T>
bool gs_tma_supported(const LevelDev<T>& L, int visc, int ty_req, int slabs_req) {
    for (int c = 0; c < 3; ++c)
        if (!gst::plan(L.D, visc, c, sizeof(T), ty_req, slabs_req, device_sms()).ok) return false;
    return gst::encoder() != nullptr;
}

template <class T>
cudaError_t launch_gs_pair_tma(const LevelDev<T>& L, int visc, int comp, const T* const rhs[3], const T* const cur[3], T* out,
                               double omega, int ty_req, int slabs_req, int* err, cudaStream_t s) {
    using namespace gst;
    const Plan p = plan(L.D, visc, comp, sizeof(T), ty_req, slabs_req, device_sms());
    if (!p.ok) return cudaErrorInvalidValue;
    Args<T> a;
    std::memset(&a, 0, sizeof(a));
    a.D = L.D;
    a.TY = p.TY;
    a.slabs = p.slabs;
    a.dir = (comp == 2) ? -1 : 1;
    a.omega = (T)omega;
    a.dxsqinv = T(1.0 / (L.dx * L.dx));
    a.out = out;
    a.err = err;
    const int t1 = (comp == 0) ? 1 : 0, t2 = (comp == 2) ? 1 : 2;
    const int e1 = (comp == 2) ? 1 : 0, e2 = (comp == 0) ? 1 : 2;
    const T* arr[A_N] = {cur[comp], cur[t1], cur[t2], rhs[comp], L.alpha[comp], L.beta, L.bed[e1], L.bed[e2], L.gamma};
    Maps m;
    std::memset(&m, 0, sizeof(m));
    for (int q = 0; q < A_N; ++q) {
        a.src[q] = arr[q];
        if (!staged(visc, q)) continue;
        const int rows = p.TY + rows_lo(comp, q) + rows_hi(comp, q);
        const cudaError_t e = make_map<T>(&m.tile[q], arr[q], L.D, rows);
        if (e != cudaSuccess) return e;
    }
    const unsigned blocks = (unsigned)((L.D.ny / p.TY) * p.slabs);
    const int nx = L.D.nx, ty = p.TY;
    switch (visc * 4 + comp) {
    case -4: return launch_comp<T, -1, 0>(a, m, blocks, nx, ty, s);
    case -3: return launch_comp<T, -1, 1>(a, m, blocks, nx, ty, s);
    case -2: return launch_comp<T, -1, 2>(a, m, blocks, nx, ty, s);
    case -8: return launch_comp<T, -2, 0>(a, m, blocks, nx, ty, s);
    case -7: return launch_comp<T, -2, 1>(a, m, blocks, nx, ty, s);
    case -6: return launch_comp<T, -2, 2>(a, m, blocks, nx, ty, s);
    case -12: return launch_comp<T, -3, 0>(a, m, blocks, nx, ty, s);
    case -11: return launch_comp<T, -3, 1>(a, m, blocks, nx, ty, s);
    case -10: return launch_comp<T, -3, 2>(a, m, blocks, nx, ty, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace lmm
