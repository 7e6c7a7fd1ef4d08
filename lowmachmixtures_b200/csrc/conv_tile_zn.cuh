// conv_tile_zn.cuh - the learned stage's 3x3x3 periodic convolution with the
// three z taps in the MMA's N dimension.
//
// Same output tile (8 x 16 voxels = 128 MMA rows), halo-plane layout,
// copies and epilogue as conv_tile.cuh, but each input halo plane p is read
// by ONE MMA of N = 3 NS per (dy, dx, K-step), which adds its contribution
// to all three output planes it feeds: out[p-1] (tap dz = +1), out[p]
// (dz = 0) and out[p+1] (dz = -1).  The accumulator of output plane o lives
// in TMEM column block o mod 3, so every MMA writes the same 3 NS columns;
// what rotates with p is which dz-weights land in which block.  The weights
// of each (dy, dx, K-step) are stored as five NS-row groups
// [dz=+1, 0, -1, +1, 0] and the MMA of input plane p reads the three groups
// starting at group (1 - p) mod 3.  Small-N tcgen05 MMAs are bound by
// reading their operands from shared memory; against 27 taps of N = NS into
// one accumulator this reads the 4 KB A tile 9 instead of 27 times per
// output plane.
//
// Per input plane i of a run (i = 0 .. K+1 are planes z0-1 .. z0+K):
//   - one elected thread issues plane i's 9 x CINP/16 MMAs and commits them;
//   - all threads wait for that commit; output plane z0+i-2 is then complete
//     in its block, its fused epilogue reads it, and the bias is written into
//     the same block as the start value of output plane z0+i+1;
//   - input plane i+3 is copied (cp.async) into the ring slot plane i has
//     released (three slots: planes i+1 and i+2 are in flight meanwhile).
// Waits are bounded; a wait that gives up sets the error word, waits once
// more (bounded) for the last commit, frees TMEM and leaves.
#pragma once
#include "conv_tile.cuh"

namespace lmm {
namespace nn {

constexpr int kRingZ = 3;  // input halo planes held

__host__ __device__ constexpr int zn_weight_bytes(int cinp, int ns) { return 9 * (cinp / 16) * 5 * ns * 32; }
__host__ __device__ constexpr int zn_smem_bytes(int cinp, int ns) {
    return zn_weight_bytes(cinp, ns) + kRingZ * tile_plane_bytes(cinp) + 4 * ns + 64;
}
__host__ __device__ constexpr uint32_t zn_tmem_cols(int ns) { return tc::tmem_cols(3 * ns); }
// CTAs per SM that the shared memory admits, capped at 5 (the register
// budget ptxas is held to)
__host__ __device__ constexpr int zn_min_blocks(int cinp, int ns) {
    return (233472 / (zn_smem_bytes(cinp, ns) + 1024)) < 1 ? 1
           : (233472 / (zn_smem_bytes(cinp, ns) + 1024)) > 5 ? 5
                                                              : (233472 / (zn_smem_bytes(cinp, ns) + 1024));
}

// one CTA computes output channels [slice * NS, slice * NS + NS) of its run
template <int CINP, int NS>
__global__ void __launch_bounds__(tc::kThreadsTC, zn_min_blocks(CINP, NS)) k_conv3d_tile_zn(TileConvArgs A, ConvEpi E, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int KS = CINP / 16;                       // K=16 steps per (dy, dx)
    constexpr int NCH = NS / 16;                        // 16-column epilogue chunks
    constexpr int PLANE = tile_plane_bytes(CINP);
    constexpr int UNITS = (CINP / 8) * kHalo;           // 16-byte units of one halo plane
    constexpr int PER = (UNITS + tc::kThreadsTC - 1) / tc::kThreadsTC;
    constexpr uint32_t NCOLS = zn_tmem_cols(NS);
    constexpr int WBLK = 5 * NS * 32;                   // bytes of one (dy, dx, K-step) weight block
    uint8_t* sw = smem;                                        // weights
    uint8_t* ring = smem + zn_weight_bytes(CINP, NS);          // kRingZ halo planes
    float* sbias = reinterpret_cast<float*>(ring + kRingZ * PLANE);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sbias + NS);
    uint32_t* holder = reinterpret_cast<uint32_t*>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nxi = A.nx >> A.up, nyi = A.ny >> A.up, nzi = A.nz >> A.up;
    const int64_t in_plane = (int64_t)nyi * nxi * A.Cin;
    const int slice = blockIdx.x / A.ctas_per_slice, cta = blockIdx.x - slice * A.ctas_per_slice;
    const int n0 = slice * NS;  // first output channel of this CTA

    if (warp == 0) tc::tmem_alloc(holder, NCOLS);
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // weights: block (q, p) = ((dy, dx), K-step), row g * NS + n of group g
    // holds output channel n0 + n of tap (dz = 1 - g % 3, dy, dx), input
    // channels 16p .. 16p+15
    for (int u = tid; u < 9 * KS * 5 * NS * 2; u += tc::kThreadsTC) {
        const int blk = u / (5 * NS * 2), v = u - blk * (5 * NS * 2);
        const int nw = v >> 1, h = v & 1;
        const int g = nw / NS, n = nw - g * NS;
        const int q = blk / KS, p = blk - q * KS;
        const int t = (2 - g % 3) * 9 + q;
        const int c0 = 16 * p + 8 * h;
        uint4 val = make_uint4(0, 0, 0, 0);
        if (c0 < A.Cin) val = *reinterpret_cast<const uint4*>(A.w + (int64_t)(n0 + n) * 27 * A.Cin + t * A.Cin + c0);
        *reinterpret_cast<uint4*>(sw + blk * WBLK + (nw >> 3) * 256 + h * 128 + (nw & 7) * 16) = val;
    }
    for (int c = tid; c < NS; c += tc::kThreadsTC) sbias[c] = (E.bias && n0 + c < E.Cout) ? E.bias[n0 + c] : 0.f;
    for (int u = tid; u < kRingZ * UNITS; u += tc::kThreadsTC) *reinterpret_cast<uint4*>(ring + u * 16) = make_uint4(0, 0, 0, 0);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *holder;
    const uint32_t idesc = tc::idesc_bf16(tc::kM, 3 * NS);
    // descriptor words: only the start-address field (bits 0..13, address /
    // 16) differs between the views, by the slot, the shift and the window
    const uint32_t a_lo = (tc::smem_u32(ring) >> 4) | ((uint32_t)(kGStride >> 4) << 16);
    const uint32_t a_hi = (uint32_t)((kHX * 16) >> 4) | (1u << 14);
    const uint32_t b_lo = (tc::smem_u32(sw) >> 4) | ((uint32_t)(128 >> 4) << 16);
    const uint32_t b_hi = (uint32_t)(256 >> 4) | (1u << 14);
    const int m = 32 * warp + lane;  // this thread's accumulator row
    const uint32_t lane_base = tmem + ((uint32_t)(32 * warp) << 16);

    // state of the current run
    int b = 0, x0 = 0, y0 = 0;
    int off[PER];                  // per unit: element offset of its 8 channels in an input plane, -1 = zero
    uint4 sk[NCH][2], mk[NCH][2];  // skip / mask rows of the output plane whose epilogue is next

    auto wrapz = [&](int z) { return z < 0 ? z + A.nz : (z >= A.nz ? z - A.nz : z); };
    const uint32_t ring_s = tc::smem_u32(ring) + (uint32_t)tid * 16;
    auto fetch = [&](int z, int slot) {
        const bf16* base = A.x + ((int64_t)b * nzi + (wrapz(z) >> A.up)) * in_plane;
        const uint32_t dst = ring_s + (uint32_t)(slot * PLANE);
#pragma unroll
        for (int i = 0; i < PER; ++i)
            if (off[i] >= 0)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + (uint32_t)(i * tc::kThreadsTC * 16)),
                             "l"(base + off[i])
                             : "memory");
    };
    auto commit = [] { asm volatile("cp.async.commit_group;" ::: "memory"); };
    auto out_row = [&](int z) { return (((int64_t)b * A.nz + z) * A.ny + y0 + (m >> 3)) * A.nx + x0 + (m & 7); };
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
    // the bias as the start value of the output plane held in block blk
    auto bias_init = [&](int blk) {
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            float v[16];
            const float4* b4 = reinterpret_cast<const float4*>(sbias + 16 * c);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 bb = b4[q];
                v[4 * q] = bb.x;
                v[4 * q + 1] = bb.y;
                v[4 * q + 2] = bb.z;
                v[4 * q + 3] = bb.w;
            }
            tc::tmem_st16(lane_base + (uint32_t)(blk * NS + 16 * c), v);
        }
        tc::tmem_wait_st();
    };
    auto epilogue = [&](int z, int blk) {
        const int64_t row = out_row(z);
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            const int c0 = n0 + 16 * c;  // first output channel of the chunk
            if (c0 >= E.Cs) break;       // uniform over the CTA
            float o[16];
            tc::tmem_ld16(lane_base + (uint32_t)(blk * NS + 16 * c), o);
            tile_store(E, row, c0, o, sk[c], mk[c]);
        }
    };
    // bounded wait for commit number s: lane 0 of each warp polls, the warp
    // learns the outcome from it
    auto wait_commit = [&](int64_t s) {
        int w = 1;
        if (lane == 0) w = tc::mbar_wait(bar, (unsigned)(s & 1)) ? 1 : 0;
        return __shfl_sync(0xffffffffu, w, 0) != 0;
    };

    const int64_t start = A.total * cta / A.ctas_per_slice, end = A.total * (cta + 1) / A.ctas_per_slice;
    int64_t seq = 0;  // MMA commits issued by this CTA
    bool ok = true;
    for (int64_t pos = start; pos < end && ok;) {
        int64_t tile = pos / A.nz;
        const int z0 = (int)(pos - tile * A.nz);
        const int K = (int)((end - pos) < (int64_t)(A.nz - z0) ? (end - pos) : (int64_t)(A.nz - z0));
        pos += K;
        const int tx = (int)(tile % A.tiles_x);
        tile /= A.tiles_x;
        const int ty = (int)(tile % A.tiles_y);
        b = (int)(tile / A.tiles_y);
        x0 = tx * kTX;
        y0 = ty * kTY;
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int u = tid + tc::kThreadsTC * i;
            off[i] = -1;
            if (u < UNITS) {
                const int g = u / kHalo, v = u - g * kHalo;
                const int hy = v / kHX, hx = v - hy * kHX;
                int xx = x0 - 1 + hx, yy = y0 - 1 + hy;
                xx = xx < 0 ? xx + A.nx : (xx >= A.nx ? xx - A.nx : xx);
                yy = yy < 0 ? yy + A.ny : (yy >= A.ny ? yy - A.ny : yy);
                if (8 * g < A.Cin) off[i] = ((yy >> A.up) * nxi + (xx >> A.up)) * A.Cin + 8 * g;
            }
        }
        // input planes 0, 1, 2 (z0-1, z0, z0+1) into slots 0, 1, 2; output
        // plane z0 (block 1) starts from the bias.  The ring and TMEM are
        // free: every earlier commit and copy has been waited for.
        fetch(z0 - 1, 0);
        commit();
        fetch(z0, 1);
        commit();
        fetch(z0 + 1, 2);
        commit();
        fetch_rows(z0);
        bias_init(1);
        asm volatile("cp.async.wait_group 2;" ::: "memory");
        tc::fence_async_smem();
        tc::tc_fence_before();
        __syncthreads();
        for (int i = 0; i <= K + 1; ++i) {
            const int64_t s = seq + i;
            if (tid == 0) {
                tc::tc_fence_after();
                const uint32_t alo = a_lo + (uint32_t)((i % kRingZ) * (PLANE >> 4));
                const uint32_t blo = b_lo + (uint32_t)((((1 - i) % 3 + 3) % 3) * NS * 2);
#pragma unroll
                for (int q = 0; q < 9; ++q) {
                    const int dy = q / 3, dx = q % 3;
#pragma unroll
                    for (int p = 0; p < KS; ++p) {
                        const uint64_t ad = ((uint64_t)a_hi << 32) | (uint64_t)(alo + (uint32_t)(dy * kHX + dx + 2 * p * kHalo));
                        const uint64_t bd = ((uint64_t)b_hi << 32) | (uint64_t)(blo + (uint32_t)((q * KS + p) * (WBLK >> 4)));
                        tc::mma_bf16(tmem, ad, bd, idesc, 1u);
                    }
                }
                tc::mma_commit(bar);
            }
            const bool w = wait_commit(s);
            ok = ok && w;
            if (w) {
                tc::tc_fence_after();
                if (i >= 2) epilogue(z0 + i - 2, (i - 1) % 3);  // output plane z0+i-2 is complete
                if (i + 2 <= K) bias_init((i + 2) % 3);         // start of output plane z0+i+1
            }
            if (i >= 2 && i <= K) fetch_rows(z0 + i - 1);
            // input plane i+3 into the slot plane i has released; then input
            // plane i+1 must have landed before the barrier
            if (i + 3 <= K + 1) fetch(z0 + i + 2, i % kRingZ);
            commit();
            asm volatile("cp.async.wait_group 2;" ::: "memory");
            tc::fence_async_smem();
            tc::tc_fence_before();
            if (!__syncthreads_and(ok)) {
                ok = false;
                seq = s + 1;
                break;
            }
        }
        if (!ok) break;
        seq += K + 2;
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();
    }
    if (!ok) {
        // the last commit may still be outstanding: one more bounded wait
        // before TMEM and the shared tile are released
        if (tid == 0) atomicExch(err, 1);
        if (seq > 0) wait_commit(seq - 1);
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        tc::tc_fence_before();
        __syncthreads();
    }
    tc::tc_fence_after();
    if (warp == 0) tc::tmem_dealloc(tmem, NCOLS);
}

}  // namespace nn
}  // namespace lmm
