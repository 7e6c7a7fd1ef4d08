// tc.cuh - the 5th-generation tensor-core (tcgen05) building block of the
// learned preconditioner stage: D[128 x N] (FP32, in TMEM) = sum_k A[128 x k]
// B[N x k], with BF16 operands that the CTA's threads gather into shared
// memory in the K-major, non-swizzled core-matrix layout, one 64-wide K chunk
// per stage, two stages in flight.  One elected thread issues the MMAs and
// commits each stage to an mbarrier; every wait is bounded and reports
// through an error flag instead of hanging.
//
// Shared-memory operand layout of one chunk (R rows x 64 k, BF16):
//   4 slices of 16 k (one MMA each), slice kk at kk * R * 32 bytes;
//   inside a slice, row r and k-half h (8 elements = 16 bytes) at
//   (r / 8) * 256 + h * 128 + (r % 8) * 16,
// i.e. core matrices of 8 rows x 16 bytes, stride 128 bytes along k (LBO)
// and 256 bytes along rows (SBO).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace lmm {
namespace tc {

constexpr int kM = 128;         // rows of the tile (TMEM lanes)
constexpr int kKC = 64;         // k per stage
constexpr int kThreadsTC = 128; // 4 warps: warp w owns TMEM lanes 32w..32w+31
constexpr unsigned kSpinLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of (row r, k) inside one chunk of R rows
__device__ __forceinline__ uint32_t chunk_off(int R, int r, int k) {
    return (uint32_t)((k >> 4) * R * 32 + (r >> 3) * 256 + ((k >> 3) & 1) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFF) >> 4);       // start address
    d |= (uint64_t)(128 >> 4) << 16;              // leading (k) byte offset
    d |= (uint64_t)(256 >> 4) << 32;              // stride (row) byte offset
    d |= (uint64_t)1 << 46;                       // descriptor version (sm_100)
    return d;                                     // base offset 0, no swizzle
}

// byte offset of the 16-byte unit holding rows mn0..mn0+7 (mn0 % 8 == 0) at
// one k, for an MN-major operand chunk of R rows (same core-matrix grid as
// chunk_off: the 8 contiguous elements run along MN instead of k)
__device__ __forceinline__ uint32_t chunk_off_mn(int R, int mn0, int k) {
    return (uint32_t)((k >> 4) * R * 32 + (mn0 >> 3) * 256 + ((k >> 3) & 1) * 128 + (k & 7) * 16);
}

// kind::f16 instruction descriptor: D FP32, A and B BF16; amn / bmn select
// the MN-major operand layout (0 = K-major)
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int amn = 0, int bmn = 0) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)amn << 15) | ((uint32_t)bmn << 16) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// true once the phase with this parity has completed; false after kSpinLimit polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    const uint32_t a = smem_u32(bar);
    for (unsigned it = 0; it < kSpinLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// whole warp
__device__ __forceinline__ void tmem_alloc(uint32_t* holder, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(holder)), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 16 FP32 columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 FP32 columns into this warp's 32 lanes; tmem_wait_st before the
// columns are read by an MMA
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};\n" ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
        "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
        "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 16 FP32 columns of this warp's 32 lanes without the wait: several loads
// may be in flight before one tmem_wait_ld
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__host__ __device__ constexpr uint32_t tmem_cols(int N) {
    return N <= 32 ? 32u : (N <= 64 ? 64u : (N <= 128 ? 128u : 256u));
}

// shared-memory bytes of the pipeline for N columns
__host__ __device__ constexpr size_t smem_bytes(int N) {
    return 2 * ((size_t)kM * kKC * 2 + (size_t)N * kKC * 2) + 64;
}

// The tile loop.  Gather: struct with
//   __device__ void a(int m0, int k0, uint8_t* sA)   fills rows 0..127, k0..k0+63
//   __device__ void b(int k0, uint8_t* sB)           fills rows 0..N-1
// (each called by all kThreadsTC threads; zero-fill past the ends);
// Epi: __device__ void operator()(int row, int col0, const float (&v)[16])
// for row = m0 + 32*warp + lane, columns col0..col0+15.
// Returns false (and sets *err) when a bounded wait gave up.
template <class Gather, class Epi, int AMN = 0, int BMN = 0>
__device__ bool gemm_tile(const Gather& G, const Epi& E, int m0, int N, int K, uint8_t* smem, int* err) {
    uint8_t* sA[2];
    uint8_t* sB[2];
    sA[0] = smem;
    sA[1] = smem + kM * kKC * 2;
    sB[0] = smem + 2 * kM * kKC * 2;
    sB[1] = sB[0] + N * kKC * 2;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sB[1] + N * kKC * 2);  // 2 mbarriers
    uint32_t* holder = reinterpret_cast<uint32_t*>(bars + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t ncols = tmem_cols(N);
    if (warp == 0) tmem_alloc(holder, ncols);
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *holder;
    const uint32_t idesc = idesc_bf16(kM, N, AMN, BMN);
    const int nchunks = (K + kKC - 1) / kKC;
    bool ok = true;
    int issued = 0;  // chunks whose MMAs were committed
    for (int c = 0; c < nchunks; ++c) {
        const int st = c & 1;
        if (c >= 2) {
            // every thread takes the same decision: stop the tile if the
            // stage did not come free within the bound
            ok = __syncthreads_and(mbar_wait(&bars[st], ((c - 2) >> 1) & 1));
            if (!ok) break;
        }
        G.a(m0, c * kKC, sA[st]);
        G.b(c * kKC, sB[st]);
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA[st]), b0 = smem_u32(sB[st]);
#pragma unroll
            for (int kk = 0; kk < kKC / 16; ++kk)
                mma_bf16(tmem, smem_desc(a0 + kk * kM * 32), smem_desc(b0 + kk * N * 32), idesc, (c > 0 || kk > 0) ? 1u : 0u);
            mma_commit(&bars[st]);
        }
        issued = c + 1;
    }
    // Every MMA of this tile is complete once the last commit has arrived
    // (MMAs complete in issue order and a commit tracks all earlier ones).
    // It is waited for also when the loop stopped early; a wait that gives
    // up is followed by one more bounded wait, so TMEM is freed below only
    // after the tile's MMAs have drained or two full bounds have passed.
    // Freeing it even then is deliberate: a CTA that exits holding TMEM
    // leaves the next CTA on its SM blocked in tcgen05.alloc, and the error
    // flag makes the host discard every result of this launch.
    bool drained = true;
    if (issued > 0) {
        const unsigned par = ((issued - 1) >> 1) & 1;
        drained = mbar_wait(&bars[(issued - 1) & 1], par);
        if (!drained) drained = mbar_wait(&bars[(issued - 1) & 1], par);
    }
    ok = __syncthreads_and(ok && drained);
    if (ok) {
        tc_fence_after();
        const int row = m0 + 32 * warp + lane;
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
            E(row, c0, v);
        }
    } else if (tid == 0) {
        atomicExch(err, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
    return ok;
}

}  // namespace tc
}  // namespace lmm
