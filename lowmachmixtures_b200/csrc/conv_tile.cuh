// conv_tile.cuh - the 3x3x3 periodic convolution of the learned stage as 27
// shifted tensor-core views of one shared-memory halo tile.
//
// A CTA owns an 8 (x) x 16 (y) tile of output voxels (the 128 rows of one
// tcgen05 MMA: row m = 8 g + r is voxel (x0 + r, y0 + g)) and marches through
// a run of output planes.  It keeps:
//   - every tap's weights resident in shared memory (27 x CINP/16 blocks of
//     N x 16 BF16 in the K-major no-swizzle core-matrix layout of tc.cuh);
//   - a ring of three input halo planes (10 x 18 voxels), laid out
//     channel-group-major: [group of 8 channels][y][x][8 channels], 16 bytes
//     per (voxel, group).
// In that layout the A operand of tap (dx, dy, dz) is the halo plane of z+dz
// read from voxel (1+dx, 1+dy) on: eight consecutive voxels of one halo row
// form one core matrix (8 rows x 16 bytes), consecutive row groups are one
// halo row apart (SBO = 10 x 16 bytes), the two 8-channel halves of a K=16
// step are one channel group apart (LBO).  So the 27 x CINP/16 MMAs of a
// plane read shifted descriptors of the same tile: no data moves per tap,
// where a gather reads every input voxel 27 times.
//
// Per plane: the threads load the next halo plane (plain 16-byte loads with
// periodic wrap; nearest upsampling read from the half grid), one elected
// thread issues the MMAs into a TMEM accumulator and commits them to an
// mbarrier, and the four warps read their 32 TMEM lanes back for the fused
// bias / skip / ReLU / mask epilogue of ConvEpi.  Waits are bounded; a wait
// that gives up sets the error word, waits once more (bounded), frees TMEM
// and leaves.
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
constexpr int kGStride = kHX * kHY * 16;         // bytes between 8-channel groups of one plane

__host__ __device__ constexpr int tile_plane_bytes(int cinp) { return (cinp / 8) * kGStride; }
__host__ __device__ constexpr int tile_weight_bytes(int cinp, int n) { return 27 * cinp * n * 2; }
__host__ __device__ constexpr int tile_smem_bytes(int cinp, int n) {
    return tile_weight_bytes(cinp, n) + 3 * tile_plane_bytes(cinp) + 64;
}

// a K-major, no-swizzle shared-memory matrix descriptor with explicit
// leading (K) and stride (row-group) byte offsets
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFF) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version (sm_100)
    return d;
}

struct TileConvArgs {
    const bf16* x;   // input activations, Cin channels per voxel (on the half grid when up)
    const bf16* w;   // weight rows [N][27 * Cin], tap-major
    int nx, ny, nz;  // output grid
    int up, Cin, N, B, KZ;
    int tiles_x, tiles_y, zchunks;
};

template <int CINP>
__global__ void __launch_bounds__(tc::kThreadsTC) k_conv3d_tile(TileConvArgs A, ConvEpi E, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int NGR = CINP / 8;
    constexpr int PLANE = tile_plane_bytes(CINP);
    const int N = A.N;
    uint8_t* sw = smem;                                        // weights
    uint8_t* ring = smem + tile_weight_bytes(CINP, N);         // 3 halo planes
    uint64_t* bar = reinterpret_cast<uint64_t*>(ring + 3 * PLANE);
    uint32_t* holder = reinterpret_cast<uint32_t*>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    int bid = blockIdx.x;
    const int tx = bid % A.tiles_x;
    bid /= A.tiles_x;
    const int ty = bid % A.tiles_y;
    bid /= A.tiles_y;
    const int zc = bid % A.zchunks;
    const int b = bid / A.zchunks;
    const int x0 = tx * kTX, y0 = ty * kTY, z0 = zc * A.KZ;
    const int z1 = min(z0 + A.KZ, A.nz);
    const int nxi = A.nx >> A.up, nyi = A.ny >> A.up, nzi = A.nz >> A.up;

    const uint32_t ncols = tc::tmem_cols(N);
    if (warp == 0) tc::tmem_alloc(holder, ncols);
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // weights: block (t, p) holds rows n of channels 16p .. 16p+15 of tap t
    {
        const int nblk = 27 * (CINP / 16);
        const int per = N * 2;  // 16-byte units per block
        for (int u = tid; u < nblk * per; u += blockDim.x) {
            const int blk = u / per, v = u - blk * per;
            const int n = v >> 1, h = v & 1;
            const int t = blk / (CINP / 16), p = blk - t * (CINP / 16);
            const int c0 = 16 * p + 8 * h;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (c0 < A.Cin) val = *reinterpret_cast<const uint4*>(A.w + (int64_t)n * 27 * A.Cin + t * A.Cin + c0);
            *reinterpret_cast<uint4*>(sw + blk * N * 32 + (n >> 3) * 256 + h * 128 + (n & 7) * 16) = val;
        }
    }
    // halo plane of output plane z (any integer: wrapped) into ring slot q
    auto load_plane = [&](int z, int q) {
        const int zz = ((z % A.nz) + A.nz) % A.nz;
        uint8_t* dst = ring + q * PLANE;
        for (int u = tid; u < NGR * kHX * kHY; u += blockDim.x) {
            const int g = u / (kHX * kHY), v = u - g * (kHX * kHY);
            const int hy = v / kHX, hx = v - hy * kHX;
            int xx = x0 - 1 + hx, yy = y0 - 1 + hy;
            xx = xx < 0 ? xx + A.nx : (xx >= A.nx ? xx - A.nx : xx);
            yy = yy < 0 ? yy + A.ny : (yy >= A.ny ? yy - A.ny : yy);
            uint4 val = make_uint4(0, 0, 0, 0);
            if (8 * g < A.Cin) {
                const int64_t src = (((int64_t)b * nzi + (zz >> A.up)) * nyi + (yy >> A.up)) * nxi + (xx >> A.up);
                val = *reinterpret_cast<const uint4*>(A.x + src * A.Cin + 8 * g);
            }
            *reinterpret_cast<uint4*>(dst + g * kGStride + v * 16) = val;
        }
    };
    load_plane(z0 - 1, 0);
    load_plane(z0, 1);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *holder;
    const uint32_t idesc = tc::idesc_bf16(tc::kM, N);
    const uint32_t sw0 = tc::smem_u32(sw), ring0 = tc::smem_u32(ring);
    bool ok = true;
    int committed = 0;
    for (int z = z0; z < z1; ++z) {
        const int j = z - z0;  // planes z-1, z, z+1 sit in slots j % 3, (j+1) % 3, (j+2) % 3
        load_plane(z + 1, (j + 2) % 3);
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::tc_fence_after();
#pragma unroll 1
            for (int t = 0; t < 27; ++t) {
                const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
                const uint32_t abase = ring0 + ((j + 1 + dz) % 3) * PLANE + ((1 + dy) * kHX + (1 + dx)) * 16;
#pragma unroll
                for (int p = 0; p < CINP / 16; ++p) {
                    const uint64_t ad = desc_kmajor(abase + 2 * p * kGStride, kGStride, kHX * 16);
                    const uint64_t bd = tc::smem_desc(sw0 + (t * (CINP / 16) + p) * N * 32);
                    tc::mma_bf16(tmem, ad, bd, idesc, (t > 0 || p > 0) ? 1u : 0u);
                }
            }
            tc::mma_commit(bar);
        }
        committed = j + 1;
        ok = __syncthreads_and(tc::mbar_wait(bar, j & 1));
        if (!ok) break;
        tc::tc_fence_after();
        {
            const int m = 32 * warp + lane;
            const int xx = x0 + (m & 7), yy = y0 + (m >> 3);
            const int row = (int)((((int64_t)b * A.nz + z) * A.ny + yy) * A.nx + xx);
            for (int c0 = 0; c0 < N; c0 += 16) {
                float v[16];
                tc::tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
                E(row, c0, v);
            }
        }
        tc::tc_fence_before();
        __syncthreads();
    }
    if (!ok) {
        // the last commit may still be outstanding: one more bounded wait
        // before TMEM and the shared tile are released
        if (tid == 0) atomicExch(err, 1);
        tc::mbar_wait(bar, (committed - 1) & 1);
        tc::tc_fence_before();
        __syncthreads();
    }
    if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

}  // namespace nn
}  // namespace lmm
