// noalloc.cu - lmm_inner_prod_noalloc: the weighted Stokes inner product with
// its reduction scratch in a static __device__ array (include/lmm_noalloc.h).
//
// Callers that cannot allocate device memory at the point where they need an
// inner product (their device memory is held by their own pool, or they have
// no solver handle and creating one would allocate a full solve workspace)
// get the same deterministic reduction as lmm_op_inner_prod, with the block
// partials, the last-block counter and the result in a fixed 19 KB array.
// Built with -fmad=false like the FP64 kernels, so both entry points return
// the same bits.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "kernels.cuh"
#include "../../include/lmm_noalloc.h"

namespace lmm {
void set_last_error(const std::string& what);  // solver.cu
}

namespace {

struct NoallocScratch {
    double partials[LMM_NOALLOC_MAX_BLOCKS * 4];  // block partial sums, 4 components
    double out[8];                                // result slot (6 used)
    unsigned counter;                             // finished blocks; must be 0 at launch
};

static __device__ __align__(256) NoallocScratch g_scratch;

constexpr int kMaxDevices = 64;
std::mutex g_mu;
NoallocScratch* g_addr[kMaxDevices] = {};

// a failed CUDA call: its text becomes the calling thread's lmm_strerror message
int cuda_failed(const char* call, cudaError_t e) {
    lmm::set_last_error(std::string("lmm_inner_prod_noalloc: ") + call + ": " + cudaGetErrorString(e));
    return LMM_ERR_CUDA;
}

// Set-up, once per device with that device current: the address of the
// static scratch in this device's copy of the module.  The address is kept
// for the life of the process; a device reset (cudaDeviceReset) unloads the
// module and invalidates it, so a process that resets a device must not call
// this entry point on that device again.
int scratch_address(NoallocScratch** out) {
    int dev = -1;
    const cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        lmm::set_last_error(std::string("lmm_inner_prod_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
        return LMM_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        lmm::set_last_error("lmm_inner_prod_noalloc: device ordinal above 63");
        return LMM_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t es = cudaGetSymbolAddress(&p, g_scratch);
        if (es != cudaSuccess) return cuda_failed("cudaGetSymbolAddress", es);
        if (!p) {
            lmm::set_last_error("lmm_inner_prod_noalloc: cudaGetSymbolAddress returned no address");
            return LMM_ERR_CUDA;
        }
        g_addr[dev] = static_cast<NoallocScratch*>(p);
    }
    *out = g_addr[dev];
    return LMM_OK;
}

}  // namespace

extern "C" int lmm_inner_prod_noalloc(int dm, const int n[3], const double* const a_u[3], const double* a_p,
                                      const double* const b_u[3], const double* b_p, double p_norm_weight, void* stream,
                                      double* out_host) {
    using namespace lmm;
    if ((dm != 2 && dm != 3) || !n || !a_u || !b_u || !a_p || !b_p || !out_host) {
        lmm::set_last_error("lmm_inner_prod_noalloc: dm must be 2 or 3 and every pointer non-null");
        return LMM_ERR_INVALID;
    }
    int64_t cells = 1;
    for (int d = 0; d < dm; ++d) {
        if (n[d] < 1) {
            lmm::set_last_error("lmm_inner_prod_noalloc: every n[d] must be at least 1");
            return LMM_ERR_INVALID;
        }
        cells *= n[d];
        if (cells > LMM_NOALLOC_MAX_CELLS) return LMM_ERR_TOO_LARGE;
    }
    for (int d = 0; d < dm; ++d)
        if (!a_u[d] || !b_u[d]) {
            lmm::set_last_error("lmm_inner_prod_noalloc: a face-array pointer is null");
            return LMM_ERR_INVALID;
        }
    // reduce_blocks never returns more than LMM_NOALLOC_MAX_BLOCKS today; the
    // check keeps the fixed scratch safe should that clamp ever change
    const int nblocks = reduce_blocks(cells);
    if (nblocks > LMM_NOALLOC_MAX_BLOCKS) return LMM_ERR_TOO_LARGE;

    NoallocScratch* scr = nullptr;
    const int rc = scratch_address(&scr);
    if (rc != LMM_OK) return rc;

    // bounds-check builds: the caller's arrays are read in place
    lmm::BcScope scope_a({a_u[0], a_u[1], dm == 3 ? a_u[2] : nullptr, a_p}, (size_t)cells * sizeof(double));
    lmm::BcScope scope_b({b_u[0], b_u[1], dm == 3 ? b_u[2] : nullptr, b_p}, (size_t)cells * sizeof(double));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Dims D;
    D.nx = n[0];
    D.ny = n[1];
    D.nz = dm == 3 ? n[2] : 1;
    D.dm = dm;
    D.wall = D.slip_lo = D.slip_hi = 0;
    // each periodic seam face is stored once and weighed 1.5 per stored copy
    // in the reference's two copies (as lmm_op_inner_prod)
    const double w = 3.0;
    cudaError_t e = cudaMemsetAsync(&scr->counter, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return cuda_failed("cudaMemsetAsync", e);
    // the same load layout as lmm_op_inner_prod, so both give the same bits
    const void* pa[4] = {a_u[0], a_u[1], dm == 3 ? a_u[2] : nullptr, a_p};
    const void* pb[4] = {b_u[0], b_u[1], dm == 3 ? b_u[2] : nullptr, b_p};
    const int vec = reduce_pairs(D, sizeof(double), pa, pb);
    if (dm == 2)
        k_reduce<double, 2, 0><<<nblocks, kThreads, 0, s>>>(D, a_u[0], a_u[1], nullptr, a_p, b_u[0], b_u[1], nullptr, b_p, w, w, w,
                                                             p_norm_weight, scr->partials, &scr->counter, scr->out, vec);
    else
        k_reduce<double, 3, 0><<<nblocks, kThreads, 0, s>>>(D, a_u[0], a_u[1], a_u[2], a_p, b_u[0], b_u[1], b_u[2], b_p, w, w, w,
                                                             p_norm_weight, scr->partials, &scr->counter, scr->out, vec);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_failed("k_reduce launch", e);
    count_launch();
    if ((e = cudaMemcpyAsync(out_host, scr->out, 6 * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_failed("cudaMemcpyAsync", e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_failed("cudaStreamSynchronize", e);
    return lmm::bc_status();
}

// the bounds-check table and record of this translation unit (empty
// unless built with -DLMM_BOUNDS_CHECK)
LMM_BC_UNIT(noalloc)
