/* lmm_noalloc.h - an entry point of liblmmstokes that allocates no device
 * memory.
 *
 * lmm_inner_prod_noalloc has no counterpart in the reference.  It computes
 * the same weighted staggered + cell inner products as lmm_op_inner_prod
 * (stag_inner_prod / cc_inner_prod, src_gmres/norm_inner_product.f90:16-375)
 * on caller-owned device arrays in the compact periodic layout, without a
 * solver handle.  Its reduction scratch (block partial sums, the
 * last-block counter and the result) lives in one fixed, statically sized
 * __device__ array of the library instead of memory allocated per handle.
 *
 * Who needs it: code that must evaluate an inner product where it cannot
 * allocate, e.g. a diagnostic inside a time step of an application whose
 * device memory is fully reserved by its own pool, or a caller that holds
 * no solver handle and must not create one (creation allocates the whole
 * workspace of a solve).
 *
 * Limits and rules:
 *  - dm is 2 or 3, every n[d] >= 1 for d < dm, and the cell count
 *    n[0]*n[1](*n[2]) is at most LMM_NOALLOC_MAX_CELLS; larger grids are
 *    rejected with LMM_ERR_TOO_LARGE before anything is launched.  The
 *    limit is 2^31 - 1 less one grid-stride (LMM_NOALLOC_MAX_BLOCKS x 256
 *    threads), so the reduction's 32-bit element index cannot wrap.  The
 *    static scratch holds LMM_NOALLOC_MAX_BLOCKS partial sums of 4
 *    components (about 19 KB), which every accepted size fits.
 *  - The scratch address of a device is looked up once and kept for the
 *    life of the process; do not call this entry point on a device after
 *    resetting it (cudaDeviceReset), which unloads the module.
 *  - The first call on a device does that device's set-up (the library's
 *    device module is loaded if it is not yet, and the scratch address is
 *    looked up); make that first call before any stream capture.
 *  - The scratch is shared by every call on the same device: calls that
 *    overlap in time (other host threads, or other streams still running
 *    an earlier call) race on it and must be serialised by the caller.
 *    One call returns only after its result has reached out_host.
 *  - stream: a cudaStream_t (NULL = the legacy default stream) on the
 *    current device, where every array must live.
 *  - out_host[0..dm-1] = per-component face sums, out_host[dm] = cell sum,
 *    exactly as lmm_op_inner_prod; out_host[4] = sum of the face sums +
 *    p_norm_weight^2 * cell sum; out_host[5] = sqrt of that for a == b.
 *    out_host must hold 6 doubles.
 * Returns LMM_OK, LMM_ERR_INVALID (bad dm, n or pointer), LMM_ERR_TOO_LARGE,
 * LMM_ERR_NO_DEVICE or LMM_ERR_CUDA; on an error lmm_strerror names the
 * failing check or CUDA call. */
#ifndef LMM_NOALLOC_H
#define LMM_NOALLOC_H

#include "lmm_stokes.h"

#ifdef __cplusplus
extern "C" {
#endif

#define LMM_ERR_TOO_LARGE      -7  /* grid larger than a fixed-size entry point accepts */
#define LMM_NOALLOC_MAX_BLOCKS 592
#define LMM_NOALLOC_MAX_CELLS  (2147483647LL - LMM_NOALLOC_MAX_BLOCKS * 256LL)  /* 2147332095 */

int lmm_inner_prod_noalloc(int dm, const int n[3], const double* const a_u[3], const double* a_p,
                           const double* const b_u[3], const double* b_p, double p_norm_weight,
                           void* stream, double* out_host);

#ifdef __cplusplus
}
#endif

#endif /* LMM_NOALLOC_H */
