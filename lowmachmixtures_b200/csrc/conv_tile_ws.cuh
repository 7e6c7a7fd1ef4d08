// conv_tile_ws.cuh - the learned stage's 3x3x3 periodic convolution for 16
// or 32 input channels: the three z taps in the MMA's N dimension, and a
// warp-specialised pipeline.
//
// Same output tile (8 x 16 voxels = 128 MMA rows), halo-plane layout and
// fused epilogue as conv_tile.cuh.  Each input halo plane p is read by ONE
// MMA of N = 3 NS per (dy, dx, K-step): its product P_p holds, in three
// NS-column blocks, the plane's contributions to out[p-1] (tap dz = +1),
// out[p] (dz = 0) and out[p+1] (dz = -1).  Small-N tcgen05 MMAs are bound by
// reading their operands from shared memory; against 27 taps of N = NS this
// reads the 4 KB A tile 9 instead of 27 times per output plane.
//
// Roles (5 warps, no CTA-wide barrier while a CTA works):
//   - warp 4's lane 0 issues plane g's MMAs into TMEM buffer g % 2 once the
//     plane's copies have landed (mbarrier full, one per ring slot) and the
//     buffer is free (mbarrier tempty), and commits them to mbarrier tfull;
//   - warps 0..3 (TMEM lanes 32w .. 32w+31), once P_g is in: copy input
//     plane g+3 (cp.async, arriving on its full barrier) into the slot of
//     plane g-1, whose MMAs the commit just seen has completed; read P_g's
//     three blocks and release the buffer; keep the two unfinished output
//     planes as running sums in registers: out[p-1] = sum + P_p(+1) is
//     complete and goes through bias / skip / ReLU / mask to memory.
// The copies, the MMAs of the next plane and this plane's epilogue overlap;
// the MMA issue, bound by the tensor core's operand reads, runs back to back.
// Every wait is bounded; a role that gives up sets the error word and a
// shared abort flag the other roles poll, and the CTA leaves after waiting
// (bounded) for its last commit and its copies.
#pragma once
#include "conv_tile.cuh"

namespace lmm {
namespace nn {

constexpr int kRingW = 4;                              // input halo planes held
constexpr int kThreadsWS = 160;                        // 4 epilogue / copy warps + the MMA warp
constexpr int kBarsWS = kRingW + 4;                    // full per slot; tfull, tempty per buffer

__host__ __device__ constexpr int ws_weight_bytes(int cinp, int ns) { return 9 * (cinp / 16) * 3 * ns * 32; }
__host__ __device__ constexpr int ws_smem_bytes(int cinp, int ns) {
    return ws_weight_bytes(cinp, ns) + kRingW * tile_plane_bytes(cinp) + 4 * ns + kBarsWS * 8 + 16;
}
// TMEM columns of one product buffer (3 NS used) and of both
__host__ __device__ constexpr uint32_t ws_buf_cols(int ns) { return tc::tmem_cols(3 * ns); }
__host__ __device__ constexpr uint32_t ws_tmem_cols(int ns) { return tc::tmem_cols(2 * (int)ws_buf_cols(ns)); }
// the register budget ptxas is held to: 3 resident CTAs per SM (TMEM
// admits 4 at NS = 16, shared memory more)
constexpr int kMinBlocksWS = 3;

// a CTA's position in its plane sequence: the run of output planes
// z0 .. z0+K-1 of tile (b, x0, y0) starting at `pos`, and the local index i
// (0 .. K+1) of the input plane z0-1+i being processed
struct RunCursor {
    int64_t pos;
    int z0, K, i, b, x0, y0;
};
__device__ __forceinline__ RunCursor run_open(int64_t pos, int64_t end, const TileConvArgs& A) {
    RunCursor c;
    c.pos = pos;
    int64_t tile = pos / A.nz;
    c.z0 = (int)(pos - tile * A.nz);
    c.K = (int)((end - pos) < (int64_t)(A.nz - c.z0) ? (end - pos) : (int64_t)(A.nz - c.z0));
    c.i = 0;
    c.x0 = (int)(tile % A.tiles_x) * kTX;
    tile /= A.tiles_x;
    c.y0 = (int)(tile % A.tiles_y) * kTY;
    c.b = (int)(tile / A.tiles_y);
    return c;
}
__device__ __forceinline__ RunCursor run_next(RunCursor c, int64_t end, const TileConvArgs& A) {
    if (++c.i > c.K + 1) {
        c.pos += c.K;
        if (c.pos < end) c = run_open(c.pos, end, A);
    }
    return c;
}

// one CTA computes output channels [slice * NS, slice * NS + NS) of its
// planes (instantiated for NS = 16: wider slices need more registers for the
// running sums than three CTAs per SM leave)
template <int CINP, int NS>
__global__ void __launch_bounds__(kThreadsWS, kMinBlocksWS) k_conv3d_ws(TileConvArgs A, ConvEpi E, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int KS = CINP / 16;                       // K=16 steps per (dy, dx)
    constexpr int NCH = NS / 16;                        // 16-column epilogue chunks
    constexpr int PLANE = tile_plane_bytes(CINP);
    constexpr int NGR = CINP / 8;                       // 8-channel groups
    constexpr int UNITS = NGR * kHalo;                  // 16-byte units of one halo plane
    constexpr int PER = (UNITS + 127) / 128;            // units per epilogue thread
    constexpr uint32_t BUFC = ws_buf_cols(NS);
    constexpr uint32_t NCOLS = ws_tmem_cols(NS);
    constexpr int WBLK = 3 * NS * 32;                   // bytes of one (dy, dx, K-step) weight block
    uint8_t* sw = smem;                                        // weights
    uint8_t* ring = smem + ws_weight_bytes(CINP, NS);          // kRingW halo planes
    float* sbias = reinterpret_cast<float*>(ring + kRingW * PLANE);
    uint64_t* full = reinterpret_cast<uint64_t*>(sbias + NS);  // [kRingW]
    uint64_t* tfull = full + kRingW;                           // [2]
    uint64_t* tempty = tfull + 2;                              // [2]
    uint32_t* holder = reinterpret_cast<uint32_t*>(tempty + 2);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(holder + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nxi = A.nx >> A.up, nyi = A.ny >> A.up, nzi = A.nz >> A.up;
    const int64_t in_plane = (int64_t)nyi * nxi * A.Cin;
    const int slice = blockIdx.x / A.ctas_per_slice, cta = blockIdx.x - slice * A.ctas_per_slice;
    const int n0 = slice * NS;  // first output channel of this CTA

    if (warp == 0) tc::tmem_alloc(holder, NCOLS);
    if (tid == 0) {
        for (int r = 0; r < kRingW; ++r) tc::mbar_init(full + r, 128);
        for (int q = 0; q < 2; ++q) {
            tc::mbar_init(tfull + q, 1);
            tc::mbar_init(tempty + q, 4);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // weights: block (q, p) = ((dy, dx), K-step), row g * NS + n of group g
    // holds output channel n0 + n of tap (dz = 1 - g, dy, dx), input
    // channels 16p .. 16p+15
    for (int u = tid; u < 9 * KS * 3 * NS * 2; u += kThreadsWS) {
        const int blk = u / (3 * NS * 2), v = u - blk * (3 * NS * 2);
        const int nw = v >> 1, h = v & 1;
        const int g = nw / NS, n = nw - g * NS;
        const int q = blk / KS, p = blk - q * KS;
        const int t = (2 - g) * 9 + q;
        const int c0 = 16 * p + 8 * h;
        uint4 val = make_uint4(0, 0, 0, 0);
        if (c0 < A.Cin) val = *reinterpret_cast<const uint4*>(A.w + (int64_t)(n0 + n) * 27 * A.Cin + t * A.Cin + c0);
        *reinterpret_cast<uint4*>(sw + blk * WBLK + (nw >> 3) * 256 + h * 128 + (nw & 7) * 16) = val;
    }
    for (int c = tid; c < NS; c += kThreadsWS) sbias[c] = (E.bias && n0 + c < E.Cout) ? E.bias[n0 + c] : 0.f;
    // units of channel groups past Cin stay zero; the copies never touch them
    for (int u = tid; u < kRingW * UNITS; u += kThreadsWS) *reinterpret_cast<uint4*>(ring + u * 16) = make_uint4(0, 0, 0, 0);
    tc::fence_async_smem();
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *holder;

    // this CTA's planes: runs of output planes z0 .. z0+K-1 of one tile, each
    // needing input planes z0-1 .. z0+K (local index i = 0 .. K+1)
    const int64_t start = A.total * cta / A.ctas_per_slice, end = A.total * (cta + 1) / A.ctas_per_slice;
    int64_t G = 0;  // input planes this CTA processes
    for (int64_t pos = start; pos < end;) {
        const int z0 = (int)(pos % A.nz);
        const int64_t K = (end - pos) < (int64_t)(A.nz - z0) ? (end - pos) : (int64_t)(A.nz - z0);
        G += K + 2;
        pos += K;
    }
    // bounded wait on an mbarrier phase by one lane; false on time-out or abort
    auto wait_bar = [&](uint64_t* bar, unsigned parity) -> bool {
        const uint32_t a = tc::smem_u32(bar);
        for (unsigned it = 0; it < tc::kSpinLimit; ++it) {
            uint32_t done;
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                : "=r"(done)
                : "r"(a), "r"(parity)
                : "memory");
            if (done) return true;
            if ((it & 63) == 63) {
                if (*abort_flag) return false;
                __nanosleep(64);
            }
        }
        return false;
    };
    auto give_up = [&]() {
        *abort_flag = 1;
        atomicExch(err, 1);
    };

    if (warp == 4) {
        // ------------------------------------------------------------- MMA
        const uint32_t idesc = tc::idesc_bf16(tc::kM, 3 * NS);
        const uint32_t a_lo = (tc::smem_u32(ring) >> 4) | ((uint32_t)(kGStride >> 4) << 16);
        const uint32_t a_hi = (uint32_t)((kHX * 16) >> 4) | (1u << 14);
        const uint32_t b_lo = (tc::smem_u32(sw) >> 4) | ((uint32_t)(128 >> 4) << 16);
        const uint32_t b_hi = (uint32_t)(256 >> 4) | (1u << 14);
        if (lane == 0) {
            int64_t last = -1;  // plane of the last MMA commit
            for (int64_t gm = 0; gm < G; ++gm) {
                const int slot = (int)(gm % kRingW), buf = (int)(gm & 1);
                if (!wait_bar(full + slot, (unsigned)((gm / kRingW) & 1)) ||
                    !wait_bar(tempty + buf, (unsigned)(((gm >> 1) & 1) ^ 1))) {
                    give_up();
                    break;
                }
                tc::fence_async_smem();  // the copies (generic proxy) before the MMAs read them
                tc::tc_fence_after();
                const uint32_t d = tmem + (uint32_t)buf * BUFC;
                const uint32_t alo = a_lo + (uint32_t)(slot * (PLANE >> 4));
#pragma unroll
                for (int q = 0; q < 9; ++q) {
                    const int dy = q / 3, dx = q % 3;
#pragma unroll
                    for (int p = 0; p < KS; ++p) {
                        const uint64_t ad = ((uint64_t)a_hi << 32) | (uint64_t)(alo + (uint32_t)(dy * kHX + dx + 2 * p * kHalo));
                        const uint64_t bd = ((uint64_t)b_hi << 32) | (uint64_t)(b_lo + (uint32_t)((q * KS + p) * (WBLK >> 4)));
                        tc::mma_bf16(d, ad, bd, idesc, (q | p) ? 1u : 0u);
                    }
                }
                tc::mma_commit(tfull + buf);
                last = gm;
            }
            // TMEM is released below: the last commit (already consumed on
            // the normal path) must have completed
            if (last >= 0) tc::mbar_wait(tfull + (last & 1), (unsigned)((last >> 1) & 1));
        }
        __syncwarp();
    } else {
        // --------------------------------------- epilogue and halo copies
        const int m = 32 * warp + lane;  // this thread's accumulator row
        const uint32_t lane_base = tmem + ((uint32_t)(32 * warp) << 16);
        float pend1[NCH][16] = {}, pend2[NCH][16] = {};  // out[p] and out[p+1] so far
        uint4 sk[NCH][2], mk[NCH][2];                    // skip / mask rows of the next output plane
        // unit u = tid + 128 k of a plane is channel group u % NGR of halo
        // voxel u / NGR (groups fastest: a warp's copies cover whole 32-byte
        // sectors); off: its element offset in an input plane, -1 = none;
        // sdst: its byte offset in a ring slot
        int off[PER];
        uint32_t sdst[PER];
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int u = tid + 128 * k, v = u / NGR, g = u - v * NGR;
            sdst[k] = tc::smem_u32(ring) + (uint32_t)(g * kGStride + v * 16);
        }
        RunCursor ce = run_open(start, end, A), cc = ce;  // epilogue and copy positions
        // copy input plane gc (cursor cc) into slot gc % 4 and arrive on its
        // full barrier once the copies have landed
        auto copy_plane = [&](int64_t gc) {
            if (cc.i == 0) {
#pragma unroll
                for (int k = 0; k < PER; ++k) {
                    const int u = tid + 128 * k, v = u / NGR, g = u - v * NGR;
                    off[k] = -1;
                    if (u < UNITS) {
                        const int hy = v / kHX, hx = v - hy * kHX;
                        int xx = cc.x0 - 1 + hx, yy = cc.y0 - 1 + hy;
                        xx = xx < 0 ? xx + A.nx : (xx >= A.nx ? xx - A.nx : xx);
                        yy = yy < 0 ? yy + A.ny : (yy >= A.ny ? yy - A.ny : yy);
                        if (8 * g < A.Cin) off[k] = ((yy >> A.up) * nxi + (xx >> A.up)) * A.Cin + 8 * g;
                    }
                }
            }
            const int slot = (int)(gc % kRingW);
            int z = cc.z0 - 1 + cc.i;
            z = z < 0 ? z + A.nz : (z >= A.nz ? z - A.nz : z);
            const bf16* base = A.x + ((int64_t)cc.b * nzi + (z >> A.up)) * in_plane;
#pragma unroll
            for (int k = 0; k < PER; ++k)
                if (off[k] >= 0)
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sdst[k] + (uint32_t)(slot * PLANE)), "l"(base + off[k])
                                 : "memory");
            asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(tc::smem_u32(full + slot)) : "memory");
            cc = run_next(cc, end, A);
        };
        auto out_row = [&](int z) { return (((int64_t)ce.b * A.nz + z) * A.ny + ce.y0 + (m >> 3)) * A.nx + ce.x0 + (m & 7); };
        auto fetch_rows = [&](int z) {
            const int64_t r = out_row(z) * E.Cs + n0;
#pragma unroll
            for (int c = 0; c < NCH; ++c)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const bool in = n0 + 16 * c + 8 * h < E.Cs;
                    sk[c][h] = (E.skip && in) ? *reinterpret_cast<const uint4*>(E.skip + r + 16 * c + 8 * h) : make_uint4(0, 0, 0, 0);
                    mk[c][h] = (E.mask && in) ? *reinterpret_cast<const uint4*>(E.mask + r + 16 * c + 8 * h) : make_uint4(0, 0, 0, 0);
                }
        };
        // planes 0, 1, 2 (the ring is fresh)
        int64_t gc = 0;
        for (; gc < G && gc < kRingW - 1; ++gc) copy_plane(gc);
        for (int64_t ge = 0; ge < G; ++ge) {
            const int buf = (int)(ge & 1), i = ce.i;
            int w = 1;
            if (lane == 0) w = wait_bar(tfull + buf, (unsigned)((ge >> 1) & 1)) ? 1 : 0;
            if (!__shfl_sync(0xffffffffu, w, 0)) {
                if (lane == 0) give_up();
                break;
            }
            tc::tc_fence_after();
            // plane ge+3 into the slot of plane ge-1, whose MMAs completed
            // before the commit just seen
            if (gc < G) copy_plane(gc++);
            if (i == 0) fetch_rows(ce.z0);
            const int64_t row = out_row(ce.z0 + i - 2);
#pragma unroll
            for (int c = 0; c < NCH; ++c) {
                // blocks dz = +1, 0, -1 of this chunk: three loads, one wait
                uint32_t ra[16], rb[16], rc[16];
                const uint32_t col = lane_base + (uint32_t)buf * BUFC + (uint32_t)(16 * c);
                tc::tmem_ld16_async(col, ra);
                tc::tmem_ld16_async(col + (uint32_t)NS, rb);
                tc::tmem_ld16_async(col + (uint32_t)(2 * NS), rc);
                tc::tmem_wait_ld();
                float o[16];
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    o[q] = pend1[c][q] + __uint_as_float(ra[q]);
                    pend1[c][q] = (i == 0 ? 0.f : pend2[c][q]) + __uint_as_float(rb[q]);
                }
                const float4* b4 = reinterpret_cast<const float4*>(sbias + 16 * c);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float4 bb = b4[q];
                    pend2[c][4 * q] = bb.x + __uint_as_float(rc[4 * q]);
                    pend2[c][4 * q + 1] = bb.y + __uint_as_float(rc[4 * q + 1]);
                    pend2[c][4 * q + 2] = bb.z + __uint_as_float(rc[4 * q + 2]);
                    pend2[c][4 * q + 3] = bb.w + __uint_as_float(rc[4 * q + 3]);
                }
                // this warp's reads of the buffer are complete: release it
                if (c == NCH - 1) {
                    tc::tc_fence_before();
                    __syncwarp();
                    if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(tempty + buf)) : "memory");
                }
                const int c0 = n0 + 16 * c;
                if (i >= 2 && c0 < E.Cs) tile_store(E, row, c0, o, sk[c], mk[c]);
            }
            if (i >= 2 && i <= ce.K) fetch_rows(ce.z0 + i - 1);
            ce = run_next(ce, end, A);
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    if (warp == 0) tc::tmem_dealloc(tmem, NCOLS);
}

}  // namespace nn
}  // namespace lmm
