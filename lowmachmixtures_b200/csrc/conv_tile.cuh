// conv_tile.cuh - the 3x3x3 periodic convolution of the learned stage as 27
// shifted tensor-core views of one shared-memory halo tile.
//
// A CTA owns an 8 (x) x 16 (y) tile of output voxels (the 128 rows of one
// tcgen05 MMA: row m = 8 g + r is voxel (x0 + r, y0 + g)) and marches through
// a run of output planes.  It keeps:
//   - every tap's weights resident in shared memory (27 x CINP/16 blocks of
//     N x 16 BF16 in the K-major no-swizzle core-matrix layout of tc.cuh);
//   - a ring of five input halo planes (10 x 18 voxels), laid out
//     channel-group-major: [group of 8 channels][y][x][8 channels], 16 bytes
//     per (voxel, group).
// In that layout the A operand of tap (dx, dy, dz) is the halo plane of z+dz
// read from voxel (1+dx, 1+dy) on: eight consecutive voxels of one halo row
// form one core matrix (8 rows x 16 bytes), consecutive row groups are one
// halo row apart (SBO = 10 x 16 bytes), the two 8-channel halves of a K=16
// step are one channel group apart (LBO).  So the 27 x CINP/16 MMAs of a
// plane read shifted descriptors of the same tile: no data moves per tap,
// where a gather reads every input voxel 27 times.  Only the 14-bit start
// address field of a descriptor changes between views, by a compile-time
// offset, so the issuing thread forms each one with one add.
//
// The grid is persistent (as many CTAs as fit on the device).  Output
// channels are computed in slices of NS (all of them when the weights fit
// in shared memory); per slice, the (tile, plane) sequence, planes fastest,
// is split into equal contiguous ranges, one per CTA, so every CTA computes
// the same number of planes to within one.  Per plane j of a run the CTA
// overlaps three things:
//   - one elected thread issues plane j's MMAs into TMEM accumulator j % 2
//     and commits them to mbarrier j % 2;
//   - meanwhile all threads wait for plane j-1's commit and run its fused
//     bias / skip / ReLU / mask epilogue from the other accumulator (skip and
//     mask rows were fetched one plane earlier);
//   - the halo plane z+3 is copied (cp.async) into the ring slot plane j-1's
//     MMAs have released, while plane z+2, copied one plane earlier, lands.
// Waits are bounded; a wait that gives up sets the error word, waits once
// more (bounded) for the last commit, frees TMEM and leaves.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "nn_layers.cuh"
#include "tc.cuh"

namespace lmm {
namespace nn {

constexpr int kTX = 8, kTY = 16;                 // output tile (x, y); 128 rows
constexpr int kHX = kTX + 2, kHY = kTY + 2;      // halo plane
constexpr int kHalo = kHX * kHY;                 // voxels of one halo plane
constexpr int kGStride = kHalo * 16;             // bytes between 8-channel groups of one plane
constexpr int kRing = 5;                         // halo planes held: 3 read by the MMAs, 2 in flight

__host__ __device__ constexpr int tile_plane_bytes(int cinp) { return (cinp / 8) * kGStride; }
__host__ __device__ constexpr int tile_weight_bytes(int cinp, int n) { return 27 * cinp * n * 2; }
__host__ __device__ constexpr int tile_smem_bytes(int cinp, int n) {
    return tile_weight_bytes(cinp, n) + kRing * tile_plane_bytes(cinp) + 4 * n + 64;
}
// CTAs per SM that the shared memory admits (228 KB per SM, 1 KB reserved
// per CTA), capped at 5: the register budget ptxas is held to
__host__ __device__ constexpr int tile_min_blocks(int cinp, int n) {
    return (233472 / (tile_smem_bytes(cinp, n) + 1024)) < 1 ? 1
           : (233472 / (tile_smem_bytes(cinp, n) + 1024)) > 5 ? 5
                                                                : (233472 / (tile_smem_bytes(cinp, n) + 1024));
}
// TMEM columns of the two accumulators
__host__ __device__ constexpr uint32_t tile_tmem_cols(int n) { return tc::tmem_cols(2 * n); }

struct TileConvArgs {
    const bf16* x;   // input activations, Cin channels per voxel (on the half grid when up)
    const bf16* w;   // weight rows [N][27 * Cin], tap-major
    int nx, ny, nz;  // output grid
    int up, Cin, B;
    int tiles_x, tiles_y;
    int64_t total;   // tiles x nz planes to compute per output-channel slice
    int slices;      // output channels are computed in slices of the kernel's NS
    int ctas_per_slice;
};

// BF16 element k (0..7) of 8 packed in a uint4, as FP32
__device__ __forceinline__ float bf16_lane(const uint4& u, int k) {
    const uint32_t w = (k >> 1) == 0 ? u.x : ((k >> 1) == 1 ? u.y : ((k >> 1) == 2 ? u.z : u.w));
    return __uint_as_float((k & 1) ? (w & 0xFFFF0000u) : (w << 16));
}
__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// one CTA computes output channels [slice * NS, slice * NS + NS) of its run
// the fused epilogue of one 16-column chunk of output row `row` whose first
// output channel is c0, given the accumulator values with the bias added:
// skip add, ReLU, mask, zero at and past Cout, BF16 or FP32 store
__device__ __forceinline__ void tile_store(const ConvEpi& E, int64_t row, int c0, float (&o)[16], const uint4 (&sk)[2],
                                           const uint4 (&mk)[2]) {
    if (E.skip) {
#pragma unroll
        for (int q = 0; q < 16; ++q) o[q] += bf16_lane(sk[q >> 3], q & 7);
    }
    if (E.relu) {
#pragma unroll
        for (int q = 0; q < 16; ++q) o[q] = fmaxf(o[q], 0.f);
    }
    if (E.mask) {
#pragma unroll
        for (int q = 0; q < 16; ++q)
            if (!(bf16_lane(mk[q >> 3], q & 7) > 0.f)) o[q] = 0.f;
    }
    const int lim = E.Cout - c0;
    if (lim < 16) {
#pragma unroll
        for (int q = 0; q < 16; ++q)
            if (q >= lim) o[q] = 0.f;
    }
    const int nc = (E.Cs - c0) < 16 ? (E.Cs - c0) : 16;
    if (E.out) {
        uint4* dst = reinterpret_cast<uint4*>(E.out + row * E.Cs + c0);
        dst[0] = make_uint4(pack_bf16x2(o[0], o[1]), pack_bf16x2(o[2], o[3]), pack_bf16x2(o[4], o[5]), pack_bf16x2(o[6], o[7]));
        if (nc > 8)
            dst[1] = make_uint4(pack_bf16x2(o[8], o[9]), pack_bf16x2(o[10], o[11]), pack_bf16x2(o[12], o[13]), pack_bf16x2(o[14], o[15]));
    }
    if (E.out32) {
        float* dst = E.out32 + row * E.Cs + c0;
        if ((E.Cs & 3) == 0) {
#pragma unroll
            for (int q = 0; q < 16; q += 4)
                if (q < nc) *reinterpret_cast<float4*>(dst + q) = make_float4(o[q], o[q + 1], o[q + 2], o[q + 3]);
        } else {
#pragma unroll
            for (int q = 0; q < 16; ++q)
                if (q < nc) dst[q] = o[q];
        }
    }
}

template <int CINP, int NS>
__global__ void __launch_bounds__(tc::kThreadsTC, tile_min_blocks(CINP, NS)) k_conv3d_tile(TileConvArgs A, ConvEpi E, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int KS = CINP / 16;                       // K=16 steps per tap
    constexpr int NCH = NS / 16;                        // 16-column epilogue chunks
    constexpr int PLANE = tile_plane_bytes(CINP);
    constexpr int NGR = CINP / 8;                       // 8-channel groups
    constexpr int UNITS = NGR * kHalo;                  // 16-byte units of one halo plane
    constexpr int PER = (UNITS + tc::kThreadsTC - 1) / tc::kThreadsTC;
    constexpr uint32_t NCOLS = tile_tmem_cols(NS);
    constexpr uint32_t ACC = NCOLS / 2;                 // column offset of accumulator 1
    uint8_t* sw = smem;                                        // weights
    uint8_t* ring = smem + tile_weight_bytes(CINP, NS);        // kRing halo planes
    float* sbias = reinterpret_cast<float*>(ring + kRing * PLANE);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sbias + NS);   // two mbarriers
    uint32_t* holder = reinterpret_cast<uint32_t*>(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nxi = A.nx >> A.up, nyi = A.ny >> A.up, nzi = A.nz >> A.up;
    const int64_t in_plane = (int64_t)nyi * nxi * A.Cin;
    const int slice = blockIdx.x / A.ctas_per_slice, cta = blockIdx.x - slice * A.ctas_per_slice;
    const int n0 = slice * NS;  // first output channel of this CTA

    if (warp == 0) tc::tmem_alloc(holder, NCOLS);
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::mbar_init(bar + 1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // weights: block (t, p) holds rows n of channels 16p .. 16p+15 of tap t
    for (int u = tid; u < 27 * KS * NS * 2; u += tc::kThreadsTC) {
        const int blk = u / (NS * 2), v = u - blk * (NS * 2);
        const int n = v >> 1, h = v & 1;
        const int t = blk / KS, p = blk - t * KS;
        const int c0 = 16 * p + 8 * h;
        uint4 val = make_uint4(0, 0, 0, 0);
        if (c0 < A.Cin) val = *reinterpret_cast<const uint4*>(A.w + (int64_t)(n0 + n) * 27 * A.Cin + t * A.Cin + c0);
        *reinterpret_cast<uint4*>(sw + blk * NS * 32 + (n >> 3) * 256 + h * 128 + (n & 7) * 16) = val;
    }
    for (int c = tid; c < NS; c += tc::kThreadsTC) sbias[c] = (E.bias && n0 + c < E.Cout) ? E.bias[n0 + c] : 0.f;
    for (int u = tid; u < kRing * UNITS; u += tc::kThreadsTC) *reinterpret_cast<uint4*>(ring + u * 16) = make_uint4(0, 0, 0, 0);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *holder;
    const uint32_t idesc = tc::idesc_bf16(tc::kM, NS);
    // descriptor words: the start-address field (bits 0..13, address / 16)
    // of a shifted view is the slot's base plus a compile-time offset
    const uint32_t a_lo = (tc::smem_u32(ring) >> 4) | ((uint32_t)(kGStride >> 4) << 16);
    const uint32_t a_hi = (uint32_t)((kHX * 16) >> 4) | (1u << 14);
    const uint32_t b_lo = (tc::smem_u32(sw) >> 4) | ((uint32_t)(128 >> 4) << 16);
    const uint32_t b_hi = (uint32_t)(256 >> 4) | (1u << 14);
    const int m = 32 * warp + lane;  // this thread's accumulator row
    const uint32_t lane_base = tmem + ((uint32_t)(32 * warp) << 16);

    // state of the current run
    int b = 0, x0 = 0, y0 = 0;
    int off[PER];            // per unit: element offset of its 8 channels inside an input plane, -1 = zero
    uint4 sk[NCH][2], mk[NCH][2];  // skip / mask rows of the plane whose epilogue is next

    auto wrapz = [&](int z) { return z < 0 ? z + A.nz : (z >= A.nz ? z - A.nz : z); };
    // asynchronous 16-byte copies of halo plane z into ring slot q (units
    // of channel groups past Cin stay the zeros written at the start).  Unit
    // u = tid + 128 i is channel group u % NGR of halo voxel u / NGR (groups
    // fastest: a warp's copies cover whole sectors); sdst is its byte offset
    // in a slot
    uint32_t sdst[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int u = tid + tc::kThreadsTC * i, v = u / NGR, g = u - v * NGR;
        sdst[i] = tc::smem_u32(ring) + (uint32_t)(g * kGStride + v * 16);
    }
    auto fetch = [&](int z, int q) {
        const bf16* base = A.x + ((int64_t)b * nzi + (wrapz(z) >> A.up)) * in_plane;
#pragma unroll
        for (int i = 0; i < PER; ++i)
            if (off[i] >= 0)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sdst[i] + (uint32_t)(q * PLANE)), "l"(base + off[i])
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
    auto epilogue = [&](int z, uint32_t acc) {
        const int64_t row = out_row(z);
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            const int c0 = n0 + 16 * c;  // first output channel of the chunk
            if (c0 >= E.Cs) break;       // uniform over the CTA
            float o[16];
            tc::tmem_ld16(lane_base + acc + (uint32_t)(16 * c), o);
            const float4* b4 = reinterpret_cast<const float4*>(sbias + 16 * c);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 bb = b4[q];
                o[4 * q] += bb.x;
                o[4 * q + 1] += bb.y;
                o[4 * q + 2] += bb.z;
                o[4 * q + 3] += bb.w;
            }
            tile_store(E, row, c0, o, sk[c], mk[c]);
        }
    };
    // bounded wait for commit number s: lane 0 of each warp polls, the
    // warp learns the outcome from it
    auto wait_commit = [&](int64_t s) {
        int w = 1;
        if (lane == 0) w = tc::mbar_wait(bar + (s & 1), (unsigned)((s >> 1) & 1)) ? 1 : 0;
        return __shfl_sync(0xffffffffu, w, 0) != 0;
    };

    const int64_t start = A.total * cta / A.ctas_per_slice, end = A.total * (cta + 1) / A.ctas_per_slice;
    int64_t seq = 0;        // MMA commits issued by this CTA
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
            const int u = tid + tc::kThreadsTC * i, v = u / NGR, g = u - v * NGR;
            off[i] = -1;
            if (u < UNITS) {
                const int hy = v / kHX, hx = v - hy * kHX;
                int xx = x0 - 1 + hx, yy = y0 - 1 + hy;
                xx = xx < 0 ? xx + A.nx : (xx >= A.nx ? xx - A.nx : xx);
                yy = yy < 0 ? yy + A.ny : (yy >= A.ny ? yy - A.ny : yy);
                if (8 * g < A.Cin) off[i] = ((yy >> A.up) * nxi + (xx >> A.up)) * A.Cin + 8 * g;
            }
        }
        // planes z0-1, z0, z0+1 into slots 0, 1, 2 and z0+2 into slot 3 (the
        // ring is free: every earlier commit and copy has been waited for)
        fetch(z0 - 1, 0);
        fetch(z0, 1);
        fetch(z0 + 1, 2);
        commit();
        if (K > 1) fetch(z0 + 2, 3);
        commit();
        fetch_rows(z0);
        asm volatile("cp.async.wait_group 1;" ::: "memory");
        tc::fence_async_smem();
        tc::tc_fence_before();
        __syncthreads();
        for (int j = 0; j < K; ++j) {
            const int z = z0 + j;
            const int64_t s = seq + j;
            // planes z-1, z, z+1 sit in slots j, j+1, j+2 (mod 5), z+2 in j+3
            if (tid == 0) {
                tc::tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(s & 1) * ACC;
                uint32_t blo = b_lo;
#pragma unroll 1
                for (int dz = 0; dz < 3; ++dz) {
                    const uint32_t alo = a_lo + (uint32_t)(((j + dz) % kRing) * (PLANE >> 4));
#pragma unroll
                    for (int q = 0; q < 9; ++q) {
                        const int dy = q / 3, dx = q % 3;
#pragma unroll
                        for (int p = 0; p < KS; ++p) {
                            const uint64_t ad = ((uint64_t)a_hi << 32) | (uint64_t)(alo + (uint32_t)(dy * kHX + dx + 2 * p * kHalo));
                            const uint64_t bd = ((uint64_t)b_hi << 32) | (uint64_t)(blo + (uint32_t)((q * KS + p) * NS * 2));
                            tc::mma_bf16(d, ad, bd, idesc, (dz | q | p) ? 1u : 0u);
                        }
                    }
                    blo += (uint32_t)(9 * KS * NS * 2);
                }
                tc::mma_commit(bar + (s & 1));
            }
            if (j > 0) {
                const bool w = wait_commit(s - 1);
                ok = ok && w;
                if (w) {
                    tc::tc_fence_after();
                    epilogue(z - 1, (uint32_t)((s - 1) & 1) * ACC);
                }
                fetch_rows(z);
            }
            // plane z+3 (read from plane j+2 on) into the slot plane j-1's
            // MMAs have released; then plane z+2, fetched one plane ago, must
            // have landed before the barrier
            if (j + 2 < K) fetch(z + 3, (j + 4) % kRing);
            commit();
            asm volatile("cp.async.wait_group 1;" ::: "memory");
            tc::fence_async_smem();
            tc::tc_fence_before();
            if (!__syncthreads_and(ok)) {
                ok = false;
                seq = s + 1;
                break;
            }
        }
        if (!ok) break;
        seq += K;
        // the run's last plane
        const bool w = wait_commit(seq - 1);
        if (w) {
            tc::tc_fence_after();
            epilogue(z0 + K - 1, (uint32_t)((seq - 1) & 1) * ACC);
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        tc::tc_fence_before();
        ok = __syncthreads_and(w);
        if (!ok) break;
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
