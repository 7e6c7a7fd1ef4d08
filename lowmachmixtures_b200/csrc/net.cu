// net.cu - the learned preconditioner network: a 3-level convolutional
// encoder-decoder on periodic grids (3x3x3 convolutions, 16/32/64 channels,
// BF16 weights and activations, FP32 accumulation on the tensor cores),
// with its forward pass, backward pass and Adam step written as explicit
// launches of the layer kernels (nn_layers.cuh).
//
//   a0 = relu(E0a x)            s0 = relu(E0b a0)             n^3, 16 ch
//   a1 = relu(E1a pool s0)      s1 = relu(E1b a1)             (n/2)^3, 32 ch
//   a2 = relu(E2a pool s1)      b2 = relu(E2b a2)             (n/4)^3, 64 ch
//   c1 = relu(D1a up b2 + s1)   d1 = relu(D1b c1)             (n/2)^3, 32 ch
//   c0 = relu(D0a up d1 + s0)   d0 = relu(D0b c0)             n^3, 16 ch
//   y  = Out d0                                               n^3, 4 ch FP32
// x has 8 channels (5 used: the velocity residual averaged to cells, the
// divergence residual, log beta).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lmm_learned.h"
#include "../../include/lmm_stokes.h"
#include "kernels.h"
#include "nn_layers.cuh"

namespace lmm {
namespace nn {

int conv3d(const bf16* x, const bf16* w, const float* bias, const bf16* skip, const bf16* mask, bf16* out, float* out32, int B,
           int nx, int ny, int nz, int up, int Cin, int Cout, int Cs, int relu, int* err, cudaStream_t s);
int conv3d_wgrad(const bf16* x, const bf16* g, float* dw, int B, int nx, int ny, int nz, int up, int Cin, int Cg, int Cout, int* err,
                 cudaStream_t s);
int pack_weights(const float* w, bf16* wf, bf16* wt, int Cout, int Cin, cudaStream_t s);

namespace {

struct LayerSpec {
    int cin, cout, level, up, relu;
};
// E0a E0b E1a E1b E2a E2b D1a D1b D0a D0b Out
constexpr int kLayers = 11;
constexpr LayerSpec kSpec[kLayers] = {{8, 16, 0, 0, 1},  {16, 16, 0, 0, 1}, {16, 32, 1, 0, 1}, {32, 32, 1, 0, 1},
                                      {32, 64, 2, 0, 1}, {64, 64, 2, 0, 1}, {64, 32, 1, 1, 1}, {32, 32, 1, 0, 1},
                                      {32, 16, 0, 1, 1}, {16, 16, 0, 0, 1}, {16, 4, 0, 0, 0}};

inline int r8(int v) { return (v + 7) / 8 * 8; }
inline int r16(int v) { return (v + 15) / 16 * 16; }

// counter-based normal numbers for the weight initialisation (splitmix64
// hash of (seed, index), Box-Muller)
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__global__ void k_init_normal(float* w, int64_t n, float stdv, uint64_t seed) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t h = mix64(seed ^ mix64((uint64_t)e));
        const float u1 = ((float)((h >> 40) & 0xFFFFFF) + 1.f) / 16777217.f;
        const float u2 = (float)((h >> 8) & 0xFFFFFF) / 16777216.f;
        w[e] = stdv * sqrtf(-2.f * logf(u1)) * cospif(2.f * u2);
    }
}

// loss = sum (y - t)^2 / count ; gy = 2 (y - t) in BF16 rows of 8 channels
__global__ void k_loss_grad(const float* __restrict__ y, const float* __restrict__ t, bf16* __restrict__ gy, float* __restrict__ loss,
                            int64_t M, float inv_count) {
    float s = 0.f;
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < M; m += (int64_t)gridDim.x * blockDim.x) {
        __align__(16) bf16 h[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float d = 0.f;
            if (c < 4) {
                d = y[m * 4 + c] - t[m * 4 + c];
                s += d * d;
            }
            h[c] = __float2bfloat16(2.f * d);
        }
        *reinterpret_cast<uint4*>(gy + m * 8) = *reinterpret_cast<const uint4*>(h);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * inv_count);
}

// dL/dy given in FP32 [M][4] -> BF16 rows of 8 channels
__global__ void k_gy_pack(const float* __restrict__ gy, bf16* __restrict__ out, int64_t M) {
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < M; m += (int64_t)gridDim.x * blockDim.x) {
        __align__(16) bf16 h[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) h[c] = __float2bfloat16(c < 4 ? gy[m * 4 + c] : 0.f);
        *reinterpret_cast<uint4*>(out + m * 8) = *reinterpret_cast<const uint4*>(h);
    }
}

int blocks_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (int)(b > 4096 ? 4096 : (b < 1 ? 1 : b));
}

}  // namespace

struct Net {
    int nx[3], ny[3], nz[3], V[3];  // per level
    int B;
    cudaStream_t s = nullptr;
    int* err = nullptr;
    float* loss = nullptr;
    // parameters: per layer w [cout][27][cin] then b [cout], concatenated
    int64_t off_w[kLayers], off_b[kLayers], nparams = 0;
    float *p = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    bf16* wf[kLayers] = {};
    bf16* wt[kLayers] = {};
    int64_t step = 0;
    // activations (BF16 channels-last) and gradients
    bf16 *x = nullptr, *a0, *s0, *p0, *a1, *s1, *p1, *a2, *b2, *c1, *d1, *c0, *d0;
    float* y = nullptr;
    bf16 *gy, *g_d0, *g_c0, *gup0, *g_d1, *g_c1, *gup1, *g_b2, *g_a2, *g_p1, *g_s1, *g_a1, *g_p0, *g_s0, *g_a0, *tmp1;
    std::vector<void*> allocs;

    template <class T>
    T* alloc(int64_t count) {
        void* q = nullptr;
        if (cudaMalloc(&q, (size_t)count * sizeof(T)) != cudaSuccess) throw LMM_ERR_CUDA;
        allocs.push_back(q);
        cudaMemsetAsync(q, 0, (size_t)count * sizeof(T), s);
        return static_cast<T*>(q);
    }
    ~Net() {
        for (void* q : allocs) cudaFree(q);
        if (s) cudaStreamDestroy(s);
    }
    int64_t M(int level) const { return (int64_t)B * V[level]; }

    int conv(int l, const bf16* in, const bf16* skip, const bf16* mask, bf16* out, float* out32, int Cs) {
        const LayerSpec& L = kSpec[l];
        const int lv = L.level;
        return conv3d(in, wf[l], p + off_b[l], skip, mask, out, out32, B, nx[lv], ny[lv], nz[lv], L.up, L.cin, L.cout, Cs, L.relu, err,
                      s);
    }
    // weight + bias gradient of layer l given its output gradient gout (Cg channels)
    int wgrad(int l, const bf16* in, const bf16* gout, int Cg) {
        const LayerSpec& L = kSpec[l];
        const int lv = L.level;
        int rc = conv3d_wgrad(in, gout, g + off_w[l], B, nx[lv], ny[lv], nz[lv], L.up, L.cin, Cg, L.cout, err, s);
        if (rc) return rc;
        k_bias_grad<<<256, 256, 0, s>>>(gout, g + off_b[l], M(lv), L.cout, Cg);
        count_launch();
        return cudaGetLastError() == cudaSuccess ? LMM_OK : LMM_ERR_CUDA;
    }
    // data gradient through layer l (flipped weights), optional ReLU mask of the input activation
    int dgrad(int l, const bf16* gout, const bf16* mask, bf16* gin) {
        const LayerSpec& L = kSpec[l];
        const int lv = L.level;
        return conv3d(gout, wt[l], nullptr, nullptr, mask, gin, nullptr, B, nx[lv], ny[lv], nz[lv], 0, r8(L.cout), L.cin, L.cin, 0, err,
                      s);
    }
    void pack() {
        for (int l = 0; l < kLayers; ++l) pack_weights(p + off_w[l], wf[l], wt[l], kSpec[l].cout, kSpec[l].cin, s);
    }

    int forward(const bf16* xin) {
        int rc = 0;
        const bf16* in = xin ? xin : x;
        rc |= conv(0, in, nullptr, nullptr, a0, nullptr, 16);
        rc |= conv(1, a0, nullptr, nullptr, s0, nullptr, 16);
        k_pool2<<<blocks_for(M(1) * 2), 256, 0, s>>>(s0, p0, B, nx[1], ny[1], nz[1], 16);
        rc |= conv(2, p0, nullptr, nullptr, a1, nullptr, 32);
        rc |= conv(3, a1, nullptr, nullptr, s1, nullptr, 32);
        k_pool2<<<blocks_for(M(2) * 4), 256, 0, s>>>(s1, p1, B, nx[2], ny[2], nz[2], 32);
        rc |= conv(4, p1, nullptr, nullptr, a2, nullptr, 64);
        rc |= conv(5, a2, nullptr, nullptr, b2, nullptr, 64);
        rc |= conv(6, b2, s1, nullptr, c1, nullptr, 32);
        rc |= conv(7, c1, nullptr, nullptr, d1, nullptr, 32);
        rc |= conv(8, d1, s0, nullptr, c0, nullptr, 16);
        rc |= conv(9, c0, nullptr, nullptr, d0, nullptr, 16);
        rc |= conv(10, d0, nullptr, nullptr, nullptr, y, 4);
        count_launch();
        count_launch();
        if (cudaGetLastError() != cudaSuccess) return LMM_ERR_CUDA;
        return rc ? LMM_ERR_INVALID : LMM_OK;
    }

    // gradients of sum(gy . y) into g (zeroed first); gy BF16 [M0][8]
    int backward(const bf16* xin) {
        const bf16* in = xin ? xin : x;
        int rc = 0;
        cudaMemsetAsync(g, 0, (size_t)nparams * sizeof(float), s);
        rc |= wgrad(10, d0, gy, 8);
        rc |= dgrad(10, gy, d0, g_d0);
        rc |= wgrad(9, c0, g_d0, 16);
        rc |= dgrad(9, g_d0, c0, g_c0);
        rc |= wgrad(8, d1, g_c0, 16);
        rc |= dgrad(8, g_c0, nullptr, gup0);  // fine grid, 32 ch
        k_downsum<<<blocks_for(M(1) * 4), 256, 0, s>>>(gup0, tmp1, B, nx[1], ny[1], nz[1], 32);
        k_grad_combine<<<blocks_for(M(1) * 32), 256, 0, s>>>(tmp1, nullptr, d1, g_d1, B, nx[1], ny[1], nz[1], 32);
        rc |= wgrad(7, c1, g_d1, 32);
        rc |= dgrad(7, g_d1, c1, g_c1);
        rc |= wgrad(6, b2, g_c1, 32);
        rc |= dgrad(6, g_c1, nullptr, gup1);  // level-1 grid, 64 ch
        k_downsum<<<blocks_for(M(2) * 8), 256, 0, s>>>(gup1, g_b2, B, nx[2], ny[2], nz[2], 64);
        k_grad_combine<<<blocks_for(M(2) * 64), 256, 0, s>>>(g_b2, nullptr, b2, g_b2, B, nx[2], ny[2], nz[2], 64);
        rc |= wgrad(5, a2, g_b2, 64);
        rc |= dgrad(5, g_b2, a2, g_a2);
        rc |= wgrad(4, p1, g_a2, 64);
        rc |= dgrad(4, g_a2, nullptr, g_p1);  // level-2 grid, 32 ch
        k_grad_combine<<<blocks_for(M(1) * 32), 256, 0, s>>>(g_c1, g_p1, s1, g_s1, B, nx[1], ny[1], nz[1], 32);
        rc |= wgrad(3, a1, g_s1, 32);
        rc |= dgrad(3, g_s1, a1, g_a1);
        rc |= wgrad(2, p0, g_a1, 32);
        rc |= dgrad(2, g_a1, nullptr, g_p0);  // level-1 grid, 16 ch
        k_grad_combine<<<blocks_for(M(0) * 16), 256, 0, s>>>(g_c0, g_p0, s0, g_s0, B, nx[0], ny[0], nz[0], 16);
        rc |= wgrad(1, a0, g_s0, 16);
        rc |= dgrad(1, g_s0, a0, g_a0);
        rc |= wgrad(0, in, g_a0, 16);
        for (int q = 0; q < 5; ++q) count_launch();
        if (cudaGetLastError() != cudaSuccess) return LMM_ERR_CUDA;
        return rc ? LMM_ERR_INVALID : LMM_OK;
    }

    int adam(float lr) {
        ++step;
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
        k_adam<<<blocks_for(nparams), 256, 0, s>>>(p, m1, m2, g, nparams, lr, b1, b2, eps, c1, c2);
        count_launch();
        pack();
        return cudaGetLastError() == cudaSuccess ? LMM_OK : LMM_ERR_CUDA;
    }
};

}  // namespace nn
}  // namespace lmm

using lmm::nn::Net;

extern "C" int lmm_net_create(int nx, int ny, int nz, int batch, unsigned long long seed, lmm_net** out) {
    using namespace lmm::nn;
    if (!out || batch < 1 || nx < 8 || ny < 8 || nz < 8 || (nx % 4) || (ny % 4) || (nz % 4)) return LMM_ERR_INVALID;
    *out = nullptr;
    Net* n = new Net();
    try {
        if (cudaStreamCreateWithFlags(&n->s, cudaStreamNonBlocking) != cudaSuccess) throw LMM_ERR_CUDA;
        n->B = batch;
        for (int l = 0; l < 3; ++l) {
            n->nx[l] = nx >> l;
            n->ny[l] = ny >> l;
            n->nz[l] = nz >> l;
            n->V[l] = n->nx[l] * n->ny[l] * n->nz[l];
        }
        for (int l = 0; l < kLayers; ++l) {
            n->off_w[l] = n->nparams;
            n->nparams += (int64_t)27 * kSpec[l].cin * kSpec[l].cout;
            n->off_b[l] = n->nparams;
            n->nparams += kSpec[l].cout;
        }
        n->p = n->alloc<float>(n->nparams);
        n->g = n->alloc<float>(n->nparams);
        n->m1 = n->alloc<float>(n->nparams);
        n->m2 = n->alloc<float>(n->nparams);
        for (int l = 0; l < kLayers; ++l) {
            n->wf[l] = n->alloc<bf16>((int64_t)r16(kSpec[l].cout) * 27 * kSpec[l].cin);
            n->wt[l] = n->alloc<bf16>((int64_t)r16(kSpec[l].cin) * 27 * r8(kSpec[l].cout));
            const float stdv = (l == kLayers - 1 ? 0.1f : 1.f) * sqrtf(2.f / (27.f * kSpec[l].cin));
            k_init_normal<<<256, 256, 0, n->s>>>(n->p + n->off_w[l], (int64_t)27 * kSpec[l].cin * kSpec[l].cout, stdv,
                                                 seed * 1000003ull + (uint64_t)l);
        }
        n->err = n->alloc<int>(1);
        n->loss = n->alloc<float>(1);
        const int64_t M0 = n->M(0), M1 = n->M(1), M2 = n->M(2);
        n->x = n->alloc<bf16>(M0 * 8);
        n->a0 = n->alloc<bf16>(M0 * 16);
        n->s0 = n->alloc<bf16>(M0 * 16);
        n->p0 = n->alloc<bf16>(M1 * 16);
        n->a1 = n->alloc<bf16>(M1 * 32);
        n->s1 = n->alloc<bf16>(M1 * 32);
        n->p1 = n->alloc<bf16>(M2 * 32);
        n->a2 = n->alloc<bf16>(M2 * 64);
        n->b2 = n->alloc<bf16>(M2 * 64);
        n->c1 = n->alloc<bf16>(M1 * 32);
        n->d1 = n->alloc<bf16>(M1 * 32);
        n->c0 = n->alloc<bf16>(M0 * 16);
        n->d0 = n->alloc<bf16>(M0 * 16);
        n->y = n->alloc<float>(M0 * 4);
        n->gy = n->alloc<bf16>(M0 * 8);
        n->g_d0 = n->alloc<bf16>(M0 * 16);
        n->g_c0 = n->alloc<bf16>(M0 * 16);
        n->gup0 = n->alloc<bf16>(M0 * 32);
        n->tmp1 = n->alloc<bf16>(M1 * 32);
        n->g_d1 = n->alloc<bf16>(M1 * 32);
        n->g_c1 = n->alloc<bf16>(M1 * 32);
        n->gup1 = n->alloc<bf16>(M1 * 64);
        n->g_b2 = n->alloc<bf16>(M2 * 64);
        n->g_a2 = n->alloc<bf16>(M2 * 64);
        n->g_p1 = n->alloc<bf16>(M2 * 32);
        n->g_s1 = n->alloc<bf16>(M1 * 32);
        n->g_a1 = n->alloc<bf16>(M1 * 32);
        n->g_p0 = n->alloc<bf16>(M1 * 16);
        n->g_s0 = n->alloc<bf16>(M0 * 16);
        n->g_a0 = n->alloc<bf16>(M0 * 16);
        n->pack();
        if (cudaStreamSynchronize(n->s) != cudaSuccess || cudaGetLastError() != cudaSuccess) throw LMM_ERR_CUDA;
    } catch (int code) {
        delete n;
        return code;
    }
    *out = reinterpret_cast<lmm_net*>(n);
    return LMM_OK;
}

extern "C" int lmm_net_destroy(lmm_net* h) {
    delete reinterpret_cast<Net*>(h);
    return LMM_OK;
}

extern "C" int64_t lmm_net_num_params(lmm_net* h) { return h ? reinterpret_cast<Net*>(h)->nparams : -1; }

extern "C" int lmm_net_stream(lmm_net* h, void** stream) {
    if (!h || !stream) return LMM_ERR_INVALID;
    *stream = reinterpret_cast<Net*>(h)->s;
    return LMM_OK;
}

static int finish(Net* n) {
    if (cudaStreamSynchronize(n->s) != cudaSuccess) return LMM_ERR_CUDA;
    int e = 0;
    if (cudaMemcpy(&e, n->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return LMM_ERR_CUDA;
    return e ? LMM_ERR_WATCHDOG : LMM_OK;
}

extern "C" int lmm_net_params(lmm_net* h, float* host, int set) {
    if (!h || !host) return LMM_ERR_INVALID;
    Net* n = reinterpret_cast<Net*>(h);
    const size_t bytes = (size_t)n->nparams * sizeof(float);
    if (set) {
        if (cudaMemcpyAsync(n->p, host, bytes, cudaMemcpyHostToDevice, n->s) != cudaSuccess) return LMM_ERR_CUDA;
        n->pack();
    } else if (cudaMemcpyAsync(host, n->p, bytes, cudaMemcpyDeviceToHost, n->s) != cudaSuccess) {
        return LMM_ERR_CUDA;
    }
    return finish(n);
}

// ------------------------------------------------------------ weight files
namespace lmm {
void set_last_error(const std::string& what);  // solver.cu
}
namespace {
constexpr char kMagic[8] = {'L', 'M', 'M', 'N', 'E', 'T', '0', '1'};
constexpr uint32_t kFormat = 1;
// FNV-1a, 64-bit (offset basis 14695981039346656037, prime 1099511628211)
uint64_t fnv1a64(const unsigned char* p, size_t n) {
    uint64_t h = 14695981039346656037ull;
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}
int file_error(const std::string& what, const char* path) {
    lmm::set_last_error(what + ": " + path);
    return LMM_ERR_INVALID;
}
}  // namespace

extern "C" int lmm_net_save(lmm_net* h, const char* path) {
    using namespace lmm::nn;
    if (!h || !path) return LMM_ERR_INVALID;
    Net* n = reinterpret_cast<Net*>(h);
    std::vector<float> p((size_t)n->nparams);
    const int rc = lmm_net_params(h, p.data(), 0);
    if (rc) return rc;
    std::vector<uint32_t> table;
    for (int l = 0; l < kLayers; ++l) {
        table.push_back((uint32_t)kSpec[l].cin);
        table.push_back((uint32_t)kSpec[l].cout);
    }
    const uint32_t head[2] = {kFormat, (uint32_t)kLayers};
    const uint64_t count = (uint64_t)n->nparams;
    const uint64_t hash = fnv1a64(reinterpret_cast<const unsigned char*>(p.data()), p.size() * sizeof(float));
    FILE* f = std::fopen(path, "wb");
    if (!f) return file_error("cannot open for writing", path);
    bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(head, 4, 2, f) == 2 &&
              std::fwrite(table.data(), 4, table.size(), f) == table.size() && std::fwrite(&count, 8, 1, f) == 1 &&
              std::fwrite(&hash, 8, 1, f) == 1 && std::fwrite(p.data(), sizeof(float), p.size(), f) == p.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? LMM_OK : file_error("write failed", path);
}

extern "C" int lmm_net_load(lmm_net* h, const char* path) {
    using namespace lmm::nn;
    if (!h || !path) return LMM_ERR_INVALID;
    Net* n = reinterpret_cast<Net*>(h);
    FILE* f = std::fopen(path, "rb");
    if (!f) return file_error("cannot open", path);
    char magic[8];
    uint32_t head[2] = {0, 0};
    std::vector<uint32_t> table(2 * kLayers);
    uint64_t count = 0, hash = 0;
    std::vector<float> p;
    std::string err;
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kMagic, 8) != 0) {
        err = "not a weight file (magic)";
    } else if (std::fread(head, 4, 2, f) != 2 || head[0] != kFormat) {
        err = "unsupported weight-file version";
    } else if (head[1] != (uint32_t)kLayers || std::fread(table.data(), 4, table.size(), f) != table.size()) {
        err = "weight file for another architecture (layer count)";
    } else {
        for (int l = 0; l < kLayers && err.empty(); ++l)
            if (table[2 * l] != (uint32_t)kSpec[l].cin || table[2 * l + 1] != (uint32_t)kSpec[l].cout)
                err = "weight file for another architecture (layer " + std::to_string(l) + " channels)";
        if (err.empty() && (std::fread(&count, 8, 1, f) != 1 || std::fread(&hash, 8, 1, f) != 1))
            err = "truncated weight file (header)";
        else if (err.empty() && count != (uint64_t)n->nparams)
            err = "weight file holds " + std::to_string(count) + " parameters, the network " + std::to_string(n->nparams);
        if (err.empty()) {
            p.resize((size_t)count);
            if (std::fread(p.data(), sizeof(float), p.size(), f) != p.size())
                err = "truncated weight file (parameters)";
            else if (std::fgetc(f) != EOF)
                err = "weight file longer than its header says";
            else if (fnv1a64(reinterpret_cast<const unsigned char*>(p.data()), p.size() * sizeof(float)) != hash)
                err = "weight-file checksum mismatch";
        }
    }
    std::fclose(f);
    if (!err.empty()) return file_error(err, path);
    return lmm_net_params(h, p.data(), 1);
}

extern "C" int lmm_net_forward(lmm_net* h, const void* x, float* y) {
    if (!h || !x) return LMM_ERR_INVALID;
    Net* n = reinterpret_cast<Net*>(h);
    int rc = n->forward(static_cast<const lmm::nn::bf16*>(x));
    if (rc) return rc;
    if (y && cudaMemcpyAsync(y, n->y, (size_t)n->M(0) * 4 * sizeof(float), cudaMemcpyDeviceToDevice, n->s) != cudaSuccess)
        return LMM_ERR_CUDA;
    return finish(n);
}

extern "C" int lmm_net_gradients(lmm_net* h, const void* x, const float* gy, float* grads_host) {
    using lmm::nn::bf16;
    if (!h || !x || !gy) return LMM_ERR_INVALID;
    Net* n = reinterpret_cast<Net*>(h);
    int rc = n->forward(static_cast<const bf16*>(x));
    if (rc) return rc;
    lmm::nn::k_gy_pack<<<lmm::nn::blocks_for(n->M(0)), 256, 0, n->s>>>(gy, n->gy, n->M(0));
    lmm::count_launch();
    rc = n->backward(static_cast<const bf16*>(x));
    if (rc) return rc;
    if (grads_host && cudaMemcpyAsync(grads_host, n->g, (size_t)n->nparams * sizeof(float), cudaMemcpyDeviceToHost, n->s) != cudaSuccess)
        return LMM_ERR_CUDA;
    return finish(n);
}

extern "C" int lmm_net_train_step(lmm_net* h, const void* x, const float* target, float lr, float* loss_host) {
    using lmm::nn::bf16;
    if (!h || !x || !target) return LMM_ERR_INVALID;
    Net* n = reinterpret_cast<Net*>(h);
    int rc = n->forward(static_cast<const bf16*>(x));
    if (rc) return rc;
    cudaMemsetAsync(n->loss, 0, sizeof(float), n->s);
    lmm::nn::k_loss_grad<<<lmm::nn::blocks_for(n->M(0)), 256, 0, n->s>>>(n->y, target, n->gy, n->loss, n->M(0),
                                                                          1.f / (float)(n->M(0) * 4));
    lmm::count_launch();
    rc = n->backward(static_cast<const bf16*>(x));
    if (rc) return rc;
    rc = n->adam(lr);
    if (rc) return rc;
    if (loss_host && cudaMemcpyAsync(loss_host, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->s) != cudaSuccess)
        return LMM_ERR_CUDA;
    return finish(n);
}

namespace lmm {
namespace nn {
__nv_bfloat16* net_input(lmm_net* h) { return reinterpret_cast<Net*>(h)->x; }
float* net_output(lmm_net* h) { return reinterpret_cast<Net*>(h)->y; }
void net_dims(lmm_net* h, int* nx, int* ny, int* nz, int* batch) {
    Net* n = reinterpret_cast<Net*>(h);
    *nx = n->nx[0];
    *ny = n->ny[0];
    *nz = n->nz[0];
    *batch = n->B;
}
// forward of the batch in net->x on the caller's stream (the network's own
// stream is swapped out for the duration)
int net_forward_on(lmm_net* h, cudaStream_t s) {
    Net* n = reinterpret_cast<Net*>(h);
    cudaStream_t own = n->s;
    n->s = s;
    const int rc = n->forward(nullptr);
    n->s = own;
    return rc;
}
}  // namespace nn
}  // namespace lmm

// the bounds-check table and record of this translation unit (empty
// unless built with -DLMM_BOUNDS_CHECK)
LMM_BC_UNIT(net)
