// solver.cu - the gmres(...) replacement: persistent device workspace, the
// staggered V-cycle driver, the pressure V-cycle, apply_precon for every
// precon_type, the reference GMRES and the flexible GMRES, and the C ABI.
//
// Reference control flow restated here:
//   gmres             src_gmres/gmres.f90:30-605
//   apply_precon      src_gmres/apply_precon.f90:29-536
//   stag_mg_solver    src_gmres/stag_mg_solver.f90:37-868 (V-cycle order,
//                     colour order 1..2*dm, bottom smooths, coefficient
//                     coarsening hoisted to once per solve)
//   macproject        src_gmres/macproject.f90:34-318 (front end; the
//                     V-cycle is this library's own design)
// Scalars of the Arnoldi process (H, norms) stay on the device; the host
// reads one Hessenberg column per inner iteration to run the Givens
// rotations and the stopping tests exactly as the reference does.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/lmm_ensemble.h"
#include "../../include/lmm_noalloc.h"
#include "../../include/lmm_stokes.h"
#include "kernels.h"
#include "krylov.cuh"
#include "learned.cuh"

using namespace lmm;

#ifdef LMM_BOUNDS_CHECK
#define LMM_BC_DECLARE(name)                                  \
    cudaError_t lmm_bc_sync_##name(const lmm::bc::Table& t); \
    cudaError_t lmm_bc_take_##name(lmm::bc::Record* r);
LMM_BC_UNITS(LMM_BC_DECLARE)
#undef LMM_BC_DECLARE
#endif

namespace {

thread_local std::string g_last_error;

}  // namespace

namespace lmm {
void set_last_error(const std::string& what);
// bounds-check builds: the device allocations loads may touch, copied into
// every translation unit's table whenever they change
#ifdef LMM_BOUNDS_CHECK
std::mutex g_bc_mu;
std::map<const void*, size_t> g_bc_ranges;
cudaError_t bc_sync_locked() {
    lmm::bc::Table t{};
    for (const auto& kv : g_bc_ranges) {
        if (t.n == lmm::bc::kRanges) break;
        t.lo[t.n] = reinterpret_cast<unsigned long long>(kv.first);
        t.hi[t.n] = t.lo[t.n] + kv.second;
        ++t.n;
    }
    cudaError_t e = cudaSuccess, f;
#define LMM_BC_SYNC(name) \
    if ((f = lmm_bc_sync_##name(t)) != cudaSuccess) e = f;
    LMM_BC_UNITS(LMM_BC_SYNC)
#undef LMM_BC_SYNC
    return e;
}
#endif
void bc_add(const void* p, size_t bytes) {
#ifdef LMM_BOUNDS_CHECK
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_bc_mu);
    g_bc_ranges[p] = bytes;
    bc_sync_locked();
#else
    (void)p;
    (void)bytes;
#endif
}
void bc_remove(const void* p) {
#ifdef LMM_BOUNDS_CHECK
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_bc_mu);
    g_bc_ranges.erase(p);
    bc_sync_locked();
#else
    (void)p;
#endif
}
// LMM_OK, or LMM_ERR_BOUNDS (message: count and first address) when a load
// since the last call fell outside the registered allocations
int bc_status() {
#ifdef LMM_BOUNDS_CHECK
    std::lock_guard<std::mutex> lock(g_bc_mu);
    unsigned long long count = 0, first = 0;
    lmm::bc::Record r;
#define LMM_BC_TAKE(name)                                        \
    if (lmm_bc_take_##name(&r) == cudaSuccess && r.count) {      \
        if (!count) first = r.first;                             \
        count += r.count;                                        \
    }
    LMM_BC_UNITS(LMM_BC_TAKE)
#undef LMM_BC_TAKE
    if (count) {
        // where the first one lies against the nearest registered allocation
        long long best = 0;
        unsigned long long blo = 0, bhi = 0;
        bool any = false;
        for (const auto& kv : g_bc_ranges) {
            const unsigned long long lo = reinterpret_cast<unsigned long long>(kv.first), hi = lo + kv.second;
            const long long d = first < lo ? (long long)(first - lo) : (long long)(first - hi);
            if (!any || std::llabs(d) < std::llabs(best)) {
                best = d;
                blo = lo;
                bhi = hi;
                any = true;
            }
        }
        char buf[256];
        std::snprintf(buf, sizeof(buf),
                      "bounds check: %llu loads outside the registered allocations, the first at 0x%llx (%lld bytes %s the "
                      "allocation [0x%llx, 0x%llx))",
                      count, first, std::llabs(best), best < 0 ? "before" : "past", blo, bhi);
        lmm::set_last_error(buf);
        return LMM_ERR_BOUNDS;
    }
#endif
    return LMM_OK;
}
}  // namespace lmm

namespace {
using lmm::bc_add;
using lmm::bc_remove;
using lmm::bc_status;

// NVTX range over one phase of a solve (solve, Krylov cycle, Arnoldi column,
// preconditioner, V-cycle, pressure solve, learned stage); a profiler shows
// them on the host timeline, and they cost one call each when none is
// attached
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// LMM_DEBUG set in the environment: every launch is followed by a
// synchronisation of the solving thread's stream (outside graph capture),
// so a failing kernel is reported at its own launch; errors go to stderr
const bool g_debug = std::getenv("LMM_DEBUG") != nullptr;
thread_local cudaStream_t g_debug_stream = nullptr;
thread_local int g_debug_dims[3] = {0, 0, 0};  // the solving handle's nx, ny, nz

// the handle whose stream LMM_DEBUG checks while a solve runs on this thread
struct DebugScope {
    explicit DebugScope(const lmm_handle* h);
    ~DebugScope() { g_debug_stream = nullptr; }
};

// a failed CUDA call or launch: its text and source line in the calling
// thread's last error
void note_error(const std::string& what, const char* fn, int line) {
    g_last_error = what + " (" + fn + ":" + std::to_string(line) + ")";
    if (g_debug)
        std::fprintf(stderr, "lmm: %s [handle %d x %d x %d]\n", g_last_error.c_str(), g_debug_dims[0], g_debug_dims[1],
                     g_debug_dims[2]);
}

#define LMM_CK(call)                                                                     \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            note_error(std::string(#call) + ": " + cudaGetErrorString(e_), __func__, __LINE__); \
            throw LmmError(LMM_ERR_CUDA);                                                \
        }                                                                                \
    } while (0)

struct LmmError {
    int code;
    explicit LmmError(int c) : code(c) {}
};

inline void check_launch(const char* fn = __builtin_FUNCTION(), int line = __builtin_LINE()) {
    lmm::count_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && g_debug && g_debug_stream) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(g_debug_stream, &cs);
        if (cs == cudaStreamCaptureStatusNone) e = cudaStreamSynchronize(g_debug_stream);
    }
    if (e != cudaSuccess) {
        note_error(std::string("kernel launch: ") + cudaGetErrorString(e), fn, line);
        throw LmmError(LMM_ERR_CUDA);
    }
}

int compute_nlevs(const int n[3], int dm, int minwidth) {
    int nl = -1;
    for (int d = 0; d < dm; ++d) {
        int temp = n[d], rdir = 1;
        while (temp % 2 == 0 && temp / minwidth != 1) {
            temp /= 2;
            ++rdir;
        }
        nl = (nl == -1) ? rdir : std::min(nl, rdir);
    }
    return nl;
}

}  // namespace

namespace lmm {
// the calling thread's message for lmm_strerror, for entry points defined
// outside this file
void set_last_error(const std::string& what) { g_last_error = what; }
}  // namespace lmm

// ============================================================ handle
struct lmm_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    lmm_grid grid{};
    lmm_knobs knobs{};
    int dm = 0;
    int64_t n = 0;
    Dims D0{};
    int nlev = 0;      // staggered levels
    int nlev_p = 0;    // pressure levels
    std::vector<LevelDev<double>> L64;
    std::vector<LevelDev<float>> L32;
    // arena
    char* arena = nullptr;
    size_t arena_bytes = 0, arena_used = 0;
    // level-0 unscaled inputs (compact)
    double* alpha_fc[3] = {nullptr, nullptr, nullptr};
    double* alphainv[3] = {nullptr, nullptr, nullptr};
    float* alphainv32[3] = {nullptr, nullptr, nullptr};
    // Krylov storage
    int m = 0;
    std::vector<SVec> V;
    std::vector<SVec> Z64;
    std::vector<float*> Z32;  // (dm+1)*n floats each
    SVec b, x, r, w, tmp, zt;
    // apply_precon scratch (FP64 and FP32)
    double *mac64 = nullptr, *src64 = nullptr, *xptmp64 = nullptr, *butmp64[3] = {nullptr, nullptr, nullptr};
    float *mac32 = nullptr, *src32 = nullptr, *xptmp32 = nullptr, *butmp32[3] = {nullptr, nullptr, nullptr};
    // BFBt scratch per precision: [0] zero, [1] kept phi, [2..4] m grad phi, [5..7] L(m grad phi)
    double* bf64[8] = {};
    float* bf32[8] = {};
    float* pin32 = nullptr;   // FP32 copy of a Stokes vector (precon input)
    float* pout32 = nullptr;  // FP32 precon output
    // reductions
    double* partials = nullptr;
    unsigned* counter = nullptr;
    double* scal = nullptr;       // device scalar slots (8 doubles per slot)
    double* hscal = nullptr;      // pinned host mirror
    double* hmisc = nullptr;      // pinned: per-level pressure coefficients and flags (64 doubles)
    int red_blocks = 0;
    static constexpr int kSlots = 256;
    // BoxLib staging
    double* stage = nullptr;
    int64_t stage_elems = 0;
    // statistics
    int vcycles = 0, pvcycles = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t wait_ev = nullptr;  // knobs.host_wait = 1: host waits block instead of spinning
    cudaEvent_t col_ev = nullptr;   // FGMRES: the Hessenberg column has reached the host
    bool coeffs_loaded = false;
    double theta_loaded = 0.0;
    // captured preconditioner applications: (input, output, theta, precision)
    struct Graph {
        int seen = 0;
        cudaGraphExec_t exec = nullptr;
        int64_t launches = 0;
        int vcycles = 0, pvcycles = 0;
    };
    std::map<std::tuple<const void*, const void*, double, int>, Graph> graphs;
    // learned stage (3D, FGMRES with the FP32 preconditioner): network and
    // its buffers, allocated by lmm_stokes_set_net outside the arena
    lmm_net* net = nullptr;
    void* lrn_block = nullptr;
    SVec lr1, lc, lAc, le;
    std::vector<SVec> Zc;  // FP64 corrections added to the FP32 Z basis
    float* lz32 = nullptr;
    int* luses = nullptr;  // [accepted, tried] of the current solve
    static constexpr int kLrnSlot = 250;
    // error word of the kernels with bounded waits (the TMA smoother): set
    // on the device when a wait gave up, read and cleared after each solve
    int* dev_err = nullptr;
    bool tma_smoother = false;  // a level of this handle runs the TMA smoother
    // a batch of 2D problems (lmm_stokes_create_batch): `batch` instances of
    // one grid stacked along the third index of every array (D0.nz = batch);
    // per-instance scalars in slot arrays of batch x 8 doubles
    int batch = 1;
    bool batched = false;
    static constexpr int kBSlots = 48;
    static constexpr int kGatherFields = 11;  // b_u(2), b_p, alpha_fc(2), beta, beta_ed, gamma, x_u(2), x_p
    double* bslots = nullptr;                 // kBSlots slot arrays (device)
    double* bhost = nullptr;                  // pinned mirror
    double* ys = nullptr;                     // (m + 1) x batch update coefficients (device)
    double* ys_host = nullptr;                // pinned
    void** ztab = nullptr;                    // device table of the m Z vectors
    const double** gtab = nullptr;            // device table: kGatherFields x batch array pointers
    const double** gtab_host = nullptr;       // pinned
    double* bslot(int k) { return bslots + (int64_t)k * batch * 8; }

    template <class T>
    T* alloc(int64_t count) {
        size_t bytes = ((size_t)count * sizeof(T) + 255) & ~(size_t)255;
        if (arena_used + bytes > arena_bytes) throw LmmError(LMM_ERR_CUDA);
        T* p = reinterpret_cast<T*>(arena + arena_used);
        arena_used += bytes;
        return p;
    }
    double* slot(int k) { return scal + 8 * k; }
};

DebugScope::DebugScope(const lmm_handle* h) {
    g_debug_stream = h->stream;
    g_debug_dims[0] = h->D0.nx;
    g_debug_dims[1] = h->D0.ny;
    g_debug_dims[2] = h->D0.nz;
}

namespace {

// wait for the handle's stream: spin (default, lowest latency) or block the
// thread (knobs.host_wait = 1; many host threads driving solvers at once)
cudaError_t host_wait(lmm_handle* h) {
    if (!h->wait_ev) return cudaStreamSynchronize(h->stream);
    cudaError_t e = cudaEventRecord(h->wait_ev, h->stream);
    if (e != cudaSuccess) return e;
    return cudaEventSynchronize(h->wait_ev);
}

bool bc_wall(int c) { return (c >= 100 && c <= 103) || (c >= 200 && c <= 203); }  // bc.f90:23-35
bool bc_noslip(int c) { return c >= 100 && c <= 103; }

// the grid's wall bits (Dims::wall / slip_lo / slip_hi)
void set_walls(Dims& D, const lmm_grid& g) {
    D.wall = D.slip_lo = D.slip_hi = 0;
    for (int d = 0; d < g.dm; ++d) {
        if (g.bc_lo[d] == LMM_BC_PERIODIC) continue;
        D.wall |= 1 << d;
        if (!bc_noslip(g.bc_lo[d])) D.slip_lo |= 1 << d;
        if (!bc_noslip(g.bc_hi[d])) D.slip_hi |= 1 << d;
    }
}

// velocity components whose mean apply_precon removes
// (apply_precon.f90:439-458): with theta alpha = 0 and no no-slip wall, the
// periodic directions
int mean_mask(const lmm_handle* h, double theta) {
    if (theta != 0.0) return 0;
    for (int d = 0; d < h->dm; ++d)
        if (bc_noslip(h->grid.bc_lo[d]) || bc_noslip(h->grid.bc_hi[d])) return 0;
    return ((1 << h->dm) - 1) & ~h->D0.wall;
}

// reduction partials: k_mdot's 592 blocks x 8 vectors x 4 components, or
// per instance of a batch k_reduce's blocks x 3 components
int64_t partials_count(const lmm_grid& g, int batch) {
    const int64_t one = 4096 * 8;
    if (g.dm != 2 || batch <= 1) return one;
    const int64_t ni = (int64_t)g.n[0] * g.n[1];
    // per instance: k_reduce's blocks x 3 components, k_mdot's x 8 vectors x 3
    return std::max<int64_t>(one, (int64_t)batch * std::max<int64_t>(reduce_blocks(ni) * 3, (int64_t)mdot_blocks(ni) * 8 * 3));
}

int64_t level_cells(const int n[3], int dm, int lev) {
    int64_t c = 1;
    for (int d = 0; d < dm; ++d) c *= (n[d] >> lev);
    return c;
}

// batch: 2D instances stacked along the third index (1 for one problem);
// batched: a batch handle (its slot arrays, tables and pinned mirrors)
size_t plan_bytes(const lmm_grid& g, const lmm_knobs& k, int nlev, int nlev_p, int batch = 1, bool batched = false) {
    const int dm = g.dm;
    const int64_t nb = (dm == 2) ? batch : 1;
    const int ne = (dm == 2) ? 1 : 3;
    size_t tot = 0;
    auto add = [&](int64_t count, size_t sz) { tot += ((size_t)count * sz + 255) & ~(size_t)255; };
    for (int l = 0; l < std::max(nlev, nlev_p); ++l) {
        int64_t c = level_cells(g.n, dm, l) * nb;
        Dims Dl;
        Dl.dm = dm;
        Dl.nx = g.n[0] >> l;
        Dl.ny = g.n[1] >> l;
        Dl.nz = (dm == 3) ? (g.n[2] >> l) : batch;
        set_walls(Dl, g);
        for (int prec = 0; prec < 2; ++prec) {
            size_t sz = prec ? sizeof(float) : sizeof(double);
            if (l < nlev) {
                for (int q = 0; q < 4 * dm + 2; ++q) add(c, sz);     // alpha, phi, rhs, tmp, beta, gamma
                for (int e = 0; e < ne; ++e) add(edge_count(Dl, e), sz);  // bed (n+1 nodes along walls)
            }
            if (l < nlev_p) {
                for (int q = 0; q < dm + 3; ++q) add(c, sz);
                if (k.visc_schur_approx == 1)
                    for (int q = 0; q < dm; ++q) add(c, sz);  // pmu
            }
        }
    }
    int64_t n = level_cells(g.n, dm, 0) * nb;
    int64_t vec = (int64_t)(dm + 1) * n;
    add(n, sizeof(double) * 2 * dm);                    // alpha_fc, alphainv
    add(n, sizeof(float) * dm);                         // alphainv32
    add(vec * (k.gmres_max_inner + 1), sizeof(double)); // V
    if (k.method == LMM_METHOD_FGMRES) {
        if (k.precision == LMM_PRECISION_FP32)
            add(vec * k.gmres_max_inner, sizeof(float));
        else
            add(vec * k.gmres_max_inner, sizeof(double));
    }
    for (int q = 0; q < 6; ++q) add(vec, sizeof(double));  // b x r w tmp zt
    for (int q = 0; q < 3 + dm; ++q) add(n, sizeof(double));
    for (int q = 0; q < 3 + dm; ++q) add(n, sizeof(float));
    add(vec, sizeof(float));
    add(vec, sizeof(float));
    add(partials_count(g, batch), sizeof(double));  // reduction partials
    add(std::max(64, batch), sizeof(unsigned));
    add(64, sizeof(int));  // error word of the kernels with bounded waits
    add(8 * lmm_handle::kSlots, sizeof(double));
    // BoxLib staging: the largest field with up to 4 ghost layers
    int64_t st = 1;
    for (int d = 0; d < dm; ++d) st *= (g.n[d] + 1 + 8);
    add(st, sizeof(double));
    if (k.visc_schur_approx == 1)
        for (int prec = 0; prec < 2; ++prec)
            for (int q = 0; q < 8; ++q) add(n, prec ? sizeof(float) : sizeof(double));  // BFBt scratch
    if (batched) {
        add((int64_t)lmm_handle::kBSlots * batch * 8, sizeof(double));  // slot arrays
        add((int64_t)(k.gmres_max_inner + 1) * batch, sizeof(double));  // ys
        add(k.gmres_max_inner + 1, sizeof(void*));                     // ztab
        add((int64_t)lmm_handle::kGatherFields * batch, sizeof(void*));  // gtab
    }
    return tot + (1 << 20);
}

template <class T>
std::vector<LevelDev<T>>& levels(lmm_handle* h);
template <>
std::vector<LevelDev<double>>& levels<double>(lmm_handle* h) { return h->L64; }
template <>
std::vector<LevelDev<float>>& levels<float>(lmm_handle* h) { return h->L32; }

template <class T>
void build_levels(lmm_handle* h) {
    auto& L = levels<T>(h);
    const int dm = h->dm;
    const int nl = std::max(h->nlev, h->nlev_p);
    L.resize(nl);
    for (int l = 0; l < nl; ++l) {
        LevelDev<T>& v = L[l];
        std::memset(&v, 0, sizeof(v));
        v.D.dm = dm;
        v.D.nx = h->grid.n[0] >> l;
        v.D.ny = h->grid.n[1] >> l;
        v.D.nz = (dm == 3) ? (h->grid.n[2] >> l) : h->batch;
        set_walls(v.D, h->grid);
        v.dx = h->grid.dx * (double)(1 << l);
        v.n = (int64_t)v.D.nx * v.D.ny * v.D.nz;
        if (l < h->nlev) {
            // the coefficients first and contiguous (one L2 persistence window
            // can cover them), then the fields
            for (int d = 0; d < dm; ++d) v.alpha[d] = h->alloc<T>(v.n);
            for (int e = 0; e < (dm == 2 ? 1 : 3); ++e) v.bed[e] = h->alloc<T>(edge_count(v.D, e));
            v.beta = h->alloc<T>(v.n);
            v.gamma = h->alloc<T>(v.n);
            for (int d = 0; d < dm; ++d) {
                v.phi[d] = h->alloc<T>(v.n);
                v.rhs[d] = h->alloc<T>(v.n);
                v.tmp[d] = h->alloc<T>(v.n);
            }
        }
        if (l < h->nlev_p) {
            for (int d = 0; d < dm; ++d) v.pa[d] = h->alloc<T>(v.n);
            if (h->knobs.visc_schur_approx == 1)
                for (int d = 0; d < dm; ++d) v.pmu[d] = h->alloc<T>(v.n);
            v.pphi = h->alloc<T>(v.n);
            v.prhs = h->alloc<T>(v.n);
            v.ptmp = h->alloc<T>(v.n);
        }
    }
}

// Keep the finest FP32 level's coefficients (theta alpha, beta_ed, beta,
// gamma: read by every colour pass, residual and operator application of
// the V-cycle) resident in L2 for kernels on the handle's stream: an access
// policy window marks them persisting.  The persisting carve-out is a
// limit of this process's context (it ends with the context).  Skipped
// when the arrays do not fit the device's window or carve-out.
void set_l2_window(lmm_handle* h) {
    const LevelDev<float>& v = h->L32[0];
    const int ne = (h->dm == 2) ? 1 : 3;
    const size_t bytes = (size_t)(h->dm + ne + 2) * (((size_t)v.n * sizeof(float) + 255) & ~(size_t)255);
    int max_window = 0, max_persist = 0;
    if (cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, h->device) != cudaSuccess) return;
    if (cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, h->device) != cudaSuccess) return;
    if (max_window <= 0 || max_persist <= 0 || bytes > (size_t)max_window) return;
    size_t cur = 0;
    cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize);
    const size_t want = std::min(bytes, (size_t)max_persist);
    if (cur < want && cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) return;
    cudaStreamAttrValue a{};
    a.accessPolicyWindow.base_ptr = v.alpha[0];
    a.accessPolicyWindow.num_bytes = bytes;
    a.accessPolicyWindow.hitRatio = (float)std::min(1.0, (double)want / (double)bytes);
    a.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    a.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    cudaStreamSetAttribute(h->stream, cudaStreamAttributeAccessPolicyWindow, &a);
    cudaGetLastError();
}

SVec make_svec(lmm_handle* h) {
    SVec s;
    s.n = h->n;
    s.dm = h->dm;
    s.base = h->alloc<double>(s.size());
    return s;
}

// ------------------------------------------------------------ reductions
// a reduction's output slot and instance count: one slot for one problem;
// on a batch handle a slot array (instance b at + 8b), one result each
double* rslot(lmm_handle* h, int k) { return h->batched ? h->bslot(k) : h->slot(k); }
int ninst(const lmm_handle* h) { return h->batched ? h->batch : 1; }

void stokes_reduce(lmm_handle* h, int mode, const double* const a[4], const double* const b[4], int slot) {
    double w[3];
    if (mode == 0) {
        w[0] = w[1] = w[2] = 3.0;  // each seam face is stored twice and weighed 1.5 per copy
    } else {
        // sum_umac_press: the x tiles span the box (weight 3 at the seam);
        // y/z tiles of 8 cells span it only when n < 16 (else weight 2).
        const int tile[3] = {1024000, 8, 8};
        for (int d = 0; d < 3; ++d) {
            int nd = (d < h->dm) ? h->grid.n[d] : 1;
            w[d] = (nd / tile[d] < 2) ? 3.0 : 2.0;
        }
    }
    launch_reduce<double>(h->D0, mode, a, b, w, h->knobs.p_norm_weight, h->partials, h->counter, rslot(h, slot),
                          h->red_blocks, h->stream, ninst(h));
    check_launch();
}

void svec_ptrs(const SVec& v, const double* p[4]) {
    for (int c = 0; c < 3; ++c) p[c] = (c < v.dm) ? v.c(c) : nullptr;
    p[3] = v.p();
}

// slot[4] = Hessenberg dot, slot[5] = Stokes norm
void stokes_dot(lmm_handle* h, const SVec& a, const SVec& b, int slot) {
    const double* pa[4];
    const double* pb[4];
    svec_ptrs(a, pa);
    svec_ptrs(b, pb);
    stokes_reduce(h, 0, pa, pb, slot);
}
void stokes_norm(lmm_handle* h, const SVec& a, int slot) { stokes_dot(h, a, a, slot); }

double read_slot(lmm_handle* h, int slot, int idx) {
    LMM_CK(cudaMemcpyAsync(h->hscal, h->slot(slot), 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    LMM_CK(host_wait(h));
    return h->hscal[idx];
}

// ------------------------------------------------------------ coefficients
// Level-0 coefficients in FP64 (theta*alpha, beta, beta_ed, gamma), the
// hierarchy by coarsening (stag_mg_solver.f90:200-230, hoisted out of the
// V-cycle), 1/alpha for the pressure solve and the FP32 copies.
void load_coeffs(lmm_handle* h, const double* const alpha_dev[3], const double* beta, const double* const bed[3],
                 const double* gamma, double theta) {
    const int dm = h->dm;
    LevelDev<double>& L0 = h->L64[0];
    const int64_t n = h->n;
    for (int d = 0; d < dm; ++d) {
        if (alpha_dev[d] != h->alpha_fc[d])
            LMM_CK(cudaMemcpyAsync(h->alpha_fc[d], alpha_dev[d], n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        launch_scale_copy<double>(h->alpha_fc[d], L0.alpha[d], theta, n, h->stream);
        launch_recip<double>(h->alpha_fc[d], h->alphainv[d], n, h->stream);
        check_launch();
    }
    if (beta != L0.beta) LMM_CK(cudaMemcpyAsync(L0.beta, beta, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    if (gamma) {
        if (gamma != L0.gamma) LMM_CK(cudaMemcpyAsync(L0.gamma, gamma, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    } else {
        LMM_CK(cudaMemsetAsync(L0.gamma, 0, n * sizeof(double), h->stream));
    }
    for (int e = 0; e < (dm == 2 ? 1 : 3); ++e)
        if (bed[e] != L0.bed[e])
            LMM_CK(cudaMemcpyAsync(L0.bed[e], bed[e], edge_count(L0.D, e) * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    for (int l = 1; l < h->nlev; ++l) {
        launch_coarsen_coeffs<double>(h->L64[l - 1], h->L64[l], false, h->stream);
        check_launch();
    }
    // pressure face coefficients 1/alpha_fc, coarsened by face averaging
    if (h->nlev_p > 0) {
        for (int d = 0; d < dm; ++d)
            LMM_CK(cudaMemcpyAsync(h->L64[0].pa[d], h->alphainv[d], n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        if (h->D0.wall) {
            // homogeneous Neumann pressure at walls: no flux crosses a wall
            // face on any level (coarsening averages the zeros)
            launch_zero_wall_faces(h->D0, h->L64[0].pa, h->stream);
            check_launch();
        }
        for (int l = 1; l < h->nlev_p; ++l) {
            launch_coarsen_coeffs<double>(h->L64[l - 1], h->L64[l], true, h->stream);
            check_launch();
        }
    }
    // BFBt: 1/diag(viscous operator) on faces, coarsened like 1/alpha
    if (h->knobs.visc_schur_approx == 1 && h->nlev_p > 0) {
        launch_inverse_diag_lap<double>(h->L64[0], h->knobs.visc_type, h->L64[0].pmu, h->stream);
        check_launch();
        for (int l = 1; l < h->nlev_p; ++l) {
            LevelDev<double> F = h->L64[l - 1], C = h->L64[l];
            for (int d = 0; d < 3; ++d) {
                F.pa[d] = F.pmu[d];
                C.pa[d] = C.pmu[d];
            }
            launch_coarsen_coeffs<double>(F, C, true, h->stream);
            check_launch();
        }
    }
    if (h->knobs.precision == LMM_PRECISION_FP32) {
        for (int l = 0; l < (int)h->L64.size(); ++l) {
            LevelDev<double>& a = h->L64[l];
            LevelDev<float>& b = h->L32[l];
            if (l < h->nlev) {
                for (int d = 0; d < dm; ++d) launch_convert<double, float>(a.alpha[d], b.alpha[d], a.n, h->stream);
                for (int e = 0; e < (dm == 2 ? 1 : 3); ++e)
                    launch_convert<double, float>(a.bed[e], b.bed[e], edge_count(a.D, e), h->stream);
                launch_convert<double, float>(a.beta, b.beta, a.n, h->stream);
                launch_convert<double, float>(a.gamma, b.gamma, a.n, h->stream);
            }
            if (l < h->nlev_p)
                for (int d = 0; d < dm; ++d) launch_convert<double, float>(a.pa[d], b.pa[d], a.n, h->stream);
            if (l < h->nlev_p && h->knobs.visc_schur_approx == 1)
                for (int d = 0; d < dm; ++d) launch_convert<double, float>(a.pmu[d], b.pmu[d], a.n, h->stream);
            check_launch();
        }
        for (int d = 0; d < dm; ++d) launch_convert<double, float>(h->alphainv[d], h->alphainv32[d], n, h->stream);
        check_launch();
    }
    // levels whose face coefficients are one value (constant density):
    // the pressure smoother and residual take 1/alpha as a scalar, the
    // velocity operator theta*alpha (up to 16 levels of each; the flags
    // and values share the handle's error word block and misc buffer)
    {
        const int np = std::min(h->nlev_p, 16), nv = std::min(h->nlev, 16);
        int* flags = h->dev_err + 32;
        LMM_CK(cudaMemsetAsync(flags, 0, 32 * sizeof(int), h->stream));
        for (int l = 0; l < np; ++l) {
            launch_uniform_check<double>(h->L64[l], flags + l, h->stream);
            check_launch();
            LMM_CK(cudaMemcpyAsync(h->hmisc + l, h->L64[l].pa[0], sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        }
        for (int l = 0; l < nv; ++l) {
            launch_uniform_check<double>(h->L64[l], flags + 16 + l, h->stream, true);
            check_launch();
            LMM_CK(cudaMemcpyAsync(h->hmisc + 16 + l, h->L64[l].alpha[0], sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        }
        int* hflags = reinterpret_cast<int*>(h->hmisc + 32);
        LMM_CK(cudaMemcpyAsync(hflags, flags, 32 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        LMM_CK(host_wait(h));
        for (int l = 0; l < (int)h->L64.size(); ++l) {
            const bool u = l < np && hflags[l] == 0 && !h->D0.wall;
            h->L64[l].pa_uniform = u ? 1 : 0;
            h->L64[l].pa_value = u ? h->hmisc[l] : 0.0;
            const bool ua = l < nv && hflags[16 + l] == 0 && h->knobs.uniform_alpha >= 0;
            h->L64[l].a_uniform = ua ? 1 : 0;
            h->L64[l].a_value = ua ? h->hmisc[16 + l] : 0.0;
            if (l < (int)h->L32.size()) {
                h->L32[l].pa_uniform = h->L64[l].pa_uniform;
                h->L32[l].pa_value = (float)h->L64[l].pa_value;
                h->L32[l].a_uniform = h->L64[l].a_uniform;
                h->L32[l].a_value = (float)h->L64[l].a_value;
            }
        }
    }
    h->coeffs_loaded = true;
    h->theta_loaded = theta;
}

// ------------------------------------------------------------ staggered V-cycle
// rows per tile the knobs ask of the TMA smoother (0: the level's default)
int tma_rows(const lmm_knobs& K) { return K.smoother_tma >= 2 ? K.smoother_tma : 0; }

// the level runs both colours of each component in one TMA-staged launch
template <class T>
bool use_tma_smoother(const lmm_handle* h, const LevelDev<T>& L) {
    const lmm_knobs& K = h->knobs;
    const int64_t min_cells = K.smoother_tma_cells > 0 ? K.smoother_tma_cells : 32768;
    return K.stag_mg_smoother != 0 && K.smoother_fusion == 0 && K.smoother_tma > 0 && h->dm == 3 && !h->batched &&
           L.n >= min_cells && gs_tma_supported<T>(L, K.visc_type, tma_rows(K), K.smoother_tma_slabs);
}

template <class T>
void smooth(lmm_handle* h, LevelDev<T>& L, int nsm) {
    const lmm_knobs& K = h->knobs;
    if (nsm > 0 && use_tma_smoother<T>(h, L)) {
        h->tma_smoother = true;
        // TMA-staged colour pairs, ping-ponging each component between phi and tmp
        T* cur[3] = {L.phi[0], L.phi[1], L.phi[2]};
        T* alt[3] = {L.tmp[0], L.tmp[1], L.tmp[2]};
        for (int m = 0; m < nsm; ++m)
            for (int d = 0; d < 3; ++d) {
                LMM_CK(launch_gs_pair_tma<T>(L, K.visc_type, d, L.rhs, cur, alt[d], K.stag_mg_omega, tma_rows(K),
                                             K.smoother_tma_slabs, h->dev_err, h->stream));
                check_launch();
                std::swap(cur[d], alt[d]);
            }
        if (cur[0] != L.phi[0])
            for (int d = 0; d < 3; ++d)
                LMM_CK(cudaMemcpyAsync(L.phi[d], cur[d], L.n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
        return;
    }
    if (K.stag_mg_smoother != 0 && K.smoother_fusion > 0 && nsm > 0 && gs_pair_supported<T>(L, K.smoother_fusion) &&
        (K.smoother_fusion_cells <= 0 || L.n <= K.smoother_fusion_cells)) {
        // fused colour pairs, ping-ponging each component between phi and tmp
        T* cur[3] = {L.phi[0], L.phi[1], L.phi[2]};
        T* alt[3] = {L.tmp[0], L.tmp[1], L.tmp[2]};
        for (int m = 0; m < nsm; ++m)
            for (int d = 0; d < h->dm; ++d) {
                launch_gs_pair<T>(L, K.visc_type, d, L.rhs, cur, alt[d], K.stag_mg_omega, K.smoother_fusion, h->stream);
                check_launch();
                std::swap(cur[d], alt[d]);
            }
        if (cur[0] != L.phi[0])
            for (int d = 0; d < h->dm; ++d)
                LMM_CK(cudaMemcpyAsync(L.phi[d], cur[d], L.n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
        return;
    }
    for (int m = 0; m < nsm; ++m) {
        if (K.stag_mg_smoother == 0) {
            launch_jacobi<T>(L, K.visc_type, L.rhs, L.phi, L.tmp, K.stag_mg_omega, h->stream);
            check_launch();
            for (int d = 0; d < h->dm; ++d)
                LMM_CK(cudaMemcpyAsync(L.phi[d], L.tmp[d], L.n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
        } else {
            // consecutive colour launches take the planes in alternating order
            // (smoother_order = 0): each starts where the last left its operands in L2
            for (int color = 1; color <= 2 * h->dm; ++color) {
                launch_gs_colour<T>(L, K.visc_type, color, L.rhs, L.phi, K.stag_mg_omega, h->stream,
                                    (K.smoother_order == 0 && color % 2 == 0) ? 1 : 0);
                check_launch();
            }
        }
    }
}

// Block-shape autotuner.  On the first handle of a grid size (per
// precision and visc_type; the table is the process's), time the candidate
// block shapes of the Gauss-Seidel colour, operator, residual and
// prolongation kernels on every periodic level with at least 4096 cells,
// and of apply_matrix on the finest (one problem, not a batch) -- one warm-up
// and five timed repetitions each, CUDA events on the handle's stream; the
// colour kernel as one whole sweep (its 2 dm colours in the smoother's
// plane order, so a shape is judged with the L2 reuse between consecutive
// colours) -- and keep the fastest, but the default geometry unless the
// fastest beats it by 2% (closer than that is timing noise, and a flip on
// noise has cost a whole sweep more than it saved).  It runs at creation,
// on the fresh arena's zeros; the colour
// kernel divides by the zero diagonal there, so phi and tmp of a tuned
// level are zeroed again afterwards.  Shapes change no value.
template <class T>
void autotune_levels(lmm_handle* h, std::vector<LevelDev<T>>& Ls) {
    static const Shape cands[] = {{0, 0}, {64, 4}, {32, 8}, {128, 2}, {16, 16}, {32, 4}, {64, 2}, {128, 1}, {256, 1}};
    const int visc = h->knobs.visc_type;
    for (int l = 0; l < h->nlev && l < (int)Ls.size(); ++l) {
        LevelDev<T>& L = Ls[l];
        if (L.n < 4096 || L.D.wall || (L.D.nx & 1) || (L.D.ny & 1) || (L.D.dm == 3 && (L.D.nz & 1))) continue;
        bool touched = false;
        for (int kid = 0; kid < TK_N; ++kid) {
            if ((kid == TK_PROLONG || kid == TK_RESIDUAL) && l + 1 >= h->nlev) continue;  // needs a coarser level
            // apply_matrix: the finest level only, on the vector type this precision feeds it
            if (kid == TK_APPLY_MATRIX && (l != 0 || h->batched || (sizeof(T) == 4 && h->Z32.empty()))) continue;
            const int kv = (kid == TK_PROLONG) ? 0 : visc;
            if (is_tuned(kid, sizeof(T), kv, L.D)) continue;
            const int nxe = (kid == TK_GS_COLOUR) ? L.D.nx / 2 : L.D.nx;
            auto launch = [&]() {
                if (kid == TK_GS_COLOUR) {
                    for (int color = 1; color <= 2 * h->dm; ++color) {
                        launch_gs_colour<T>(L, visc, color, L.rhs, L.phi, 1.0, h->stream,
                                            (h->knobs.smoother_order == 0 && color % 2 == 0) ? 1 : 0);
                        if (color < 2 * h->dm) check_launch();
                    }
                } else if (kid == TK_APPLYOP)
                    launch_applyop<T>(L, visc, L.phi, L.tmp, h->stream, 0);
                else if (kid == TK_RESIDUAL)  // the split residual (its restriction is timed with it)
                    launch_residual_restrict<T>(L, Ls[l + 1], visc, L.rhs, L.phi, Ls[l + 1].rhs, h->stream, 0);
                else if (kid == TK_APPLY_MATRIX) {
                    if constexpr (sizeof(T) == 4)
                        launch_apply_matrix_f32(h->L64[0], visc, h->Z32[0], h->n, h->dm, h->tmp, h->stream);
                    else
                        launch_apply_matrix(h->L64[0], visc, h->x, h->tmp, h->stream);
                } else
                    launch_prolong_add<T>(L, Ls[l + 1], Ls[l + 1].phi, L.phi, h->stream);
                check_launch();
            };
            double best = 1e300, def = 0.0;
            Shape bs{};
            for (const Shape& c : cands) {
                if (c.bx > std::max(nxe, 32)) continue;
                force_shape(c);
                launch();
                constexpr int kReps = 5;
                LMM_CK(cudaEventRecord(h->ev0, h->stream));
                for (int r = 0; r < kReps; ++r) launch();
                LMM_CK(cudaEventRecord(h->ev1, h->stream));
                LMM_CK(cudaEventSynchronize(h->ev1));
                float ms = 0.f;
                LMM_CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
                // per launch (a colour sweep is 2 dm launches)
                const double per = ms / kReps / (kid == TK_GS_COLOUR ? 2 * h->dm : 1);
                if (c.bx == 0) def = per;
                if (per < best) {
                    best = per;
                    bs = c;
                }
            }
            if (bs.bx != 0 && best > 0.98 * def) {
                bs = Shape{};
                best = def;
            }
            force_shape(Shape{});
            set_tuned_shape(kid, sizeof(T), kv, L.D, bs, def, best);
            touched = true;
        }
        if (touched)
            for (int d = 0; d < h->dm; ++d) {
                LMM_CK(cudaMemsetAsync(L.phi[d], 0, L.n * sizeof(T), h->stream));
                LMM_CK(cudaMemsetAsync(L.tmp[d], 0, L.n * sizeof(T), h->stream));
            }
    }
}

// first level handled by the shared-memory tail kernel (nl: no tail): the
// largest run of coarse levels with at most tail_cells cells each whose
// phi/rhs fit the shared-memory budget
template <class T>
int tail_start(lmm_handle* h, const std::vector<LevelDev<T>>& L, int nl, bool stag) {
    // default: the velocity tail from 8^3 cells down (a 16^3 level runs
    // faster as per-level launches over many SMs than as ~50 barrier phases
    // on one) -- one 2D problem from 32^2 down (64^2 solve 2.71 -> 2.58 ms;
    // a batch's per-problem tails were slower from 32^2) -- and the
    // pressure tail from 16^3 down
    const int vel_cells = (h->dm == 2 && !h->batched) ? 1024 : 512;
    const int cells = h->knobs.tail_cells == 0 ? (stag ? vel_cells : 4096) : h->knobs.tail_cells;
    if (cells < 0) return nl;
    const size_t budget = (size_t)(h->knobs.tail_smem_kb > 0 ? h->knobs.tail_smem_kb : 200) * 1024;
    const bool jacobi = stag && h->knobs.stag_mg_smoother == 0;
    const int64_t inst = (h->dm == 2) ? h->batch : 1;  // a 2D batch: one tail block per instance
    int lc = nl;
    while (lc > 0 && nl - (lc - 1) <= 12 && L[lc - 1].n / inst <= cells &&
           tail_smem_bytes<T>(&L[lc - 1], nl - (lc - 1), stag, jacobi) <= budget)
        --lc;
    return lc;
}

template <class T>
void vcycle(lmm_handle* h, std::vector<LevelDev<T>>& L) {
    NvtxRange nvtx_("stag_mg V-cycle");
    const lmm_knobs& K = h->knobs;
    const int nl = h->nlev;
    const int lc = tail_start<T>(h, L, nl, true);
    // coarse-level initial guesses are zero; the tail zeroes the levels below its first
    for (int l = 1; l <= std::min(lc, nl - 1); ++l)
        for (int d = 0; d < h->dm; ++d) LMM_CK(cudaMemsetAsync(L[l].phi[d], 0, L[l].n * sizeof(T), h->stream));
    for (int l = 0; l < lc && l < nl - 1; ++l) {
        smooth<T>(h, L[l], K.stag_mg_nsmooths_down);
        launch_residual_restrict<T>(L[l], L[l + 1], K.visc_type, L[l].rhs, L[l].phi, L[l + 1].rhs, h->stream,
                                    K.residual_fusion > 0 ? 1 : 0);
        check_launch();
    }
    if (lc < nl) {
        LMM_CK(launch_vcycle_tail<T>(&L[lc], nl - lc, K.visc_type, K.stag_mg_nsmooths_down, K.stag_mg_nsmooths_up,
                                     K.stag_mg_nsmooths_bottom, K.stag_mg_smoother, K.stag_mg_omega, h->stream));
        check_launch();
    } else {
        smooth<T>(h, L[nl - 1], K.stag_mg_nsmooths_bottom);
    }
    for (int l = std::min(lc, nl - 1) - 1; l >= 0; --l) {
        launch_prolong_add<T>(L[l], L[l + 1], L[l + 1].phi, L[l].phi, h->stream);
        check_launch();
        smooth<T>(h, L[l], K.stag_mg_nsmooths_up);
    }
}

// inf-norm of (L phi - rhs) per component at level 0 (stag_mg_solver.f90:259-270, 766-786)
template <class T>
void mg_resid_inf(lmm_handle* h, LevelDev<T>& L0, int slot);

template <>
void mg_resid_inf<double>(lmm_handle* h, LevelDev<double>& L0, int slot) {
    launch_applyop<double>(L0, h->knobs.visc_type, L0.phi, L0.tmp, h->stream, 0);
    check_launch();
    const double* a[4] = {L0.tmp[0], L0.tmp[1], h->dm == 3 ? L0.tmp[2] : nullptr, nullptr};
    const double* b[4] = {L0.rhs[0], L0.rhs[1], h->dm == 3 ? L0.rhs[2] : nullptr, nullptr};
    const double w[3] = {1, 1, 1};
    launch_reduce<double>(h->D0, 2, a, b, w, 0.0, h->partials, h->counter, h->slot(slot), h->red_blocks, h->stream);
    check_launch();
}
template <>
void mg_resid_inf<float>(lmm_handle* h, LevelDev<float>& L0, int slot) {
    launch_applyop<float>(L0, h->knobs.visc_type, L0.phi, L0.tmp, h->stream, 0);
    check_launch();
    const float* a[4] = {L0.tmp[0], L0.tmp[1], h->dm == 3 ? L0.tmp[2] : nullptr, nullptr};
    const float* b[4] = {L0.rhs[0], L0.rhs[1], h->dm == 3 ? L0.rhs[2] : nullptr, nullptr};
    const double w[3] = {1, 1, 1};
    launch_reduce<float>(h->D0, 2, a, b, w, 0.0, h->partials, h->counter, h->slot(slot), h->red_blocks, h->stream);
    check_launch();
}

// stag_mg_solver: phi (initial guess) and rhs live in L[0].phi / L[0].rhs
template <class T>
void stag_mg_solver(lmm_handle* h) {
    auto& L = levels<T>(h);
    const lmm_knobs& K = h->knobs;
    const int dm = h->dm;
    if (K.stag_mg_max_vcycles <= 1) {
        vcycle<T>(h, L);
    } else {
        const int s0 = h->kSlots - 2, s1 = h->kSlots - 1;
        mg_resid_inf<T>(h, L[0], s0);
        double r0[3] = {0, 0, 0};
        LMM_CK(cudaMemcpyAsync(h->hscal, h->slot(s0), 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        LMM_CK(host_wait(h));
        bool all_zero = true, any_zero = false;
        for (int d = 0; d < dm; ++d) {
            r0[d] = h->hscal[d];
            all_zero = all_zero && r0[d] == 0.0;
            any_zero = any_zero || r0[d] == 0.0;
        }
        if (!all_zero) {
            if (any_zero) {
                double mx = 0;
                for (int d = 0; d < dm; ++d) mx = std::max(mx, r0[d]);
                for (int d = 0; d < dm; ++d) r0[d] = mx;
            }
            for (int vc = 1; vc <= K.stag_mg_max_vcycles; ++vc) {
                vcycle<T>(h, L);
                mg_resid_inf<T>(h, L[0], s1);
                LMM_CK(cudaMemcpyAsync(h->hscal, h->slot(s1), 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
                LMM_CK(host_wait(h));
                bool done = true;
                for (int d = 0; d < dm; ++d) done = done && (h->hscal[d] / r0[d] < K.stag_mg_rel_tol);
                if (done) break;
            }
        }
    }
    h->vcycles += dm * K.stag_mg_max_vcycles;
}

// ------------------------------------------------------------ pressure V-cycle
template <class T>
void cc_smooth(lmm_handle* h, LevelDev<T>& L, int nsweeps) {
    for (int s = 0; s < nsweeps; ++s)
        for (int parity = 0; parity < 2; ++parity) {
            launch_cc_smooth<T>(L, parity, h->stream, (h->knobs.smoother_order == 0 && parity == 1) ? 1 : 0);
            check_launch();
        }
}

// phi (L[0].pphi) <- mg_max_vcycles V-cycles of div(a grad phi) = L[0].prhs
template <class T>
void macproject(lmm_handle* h) {
    NvtxRange nvtx_("macproject (pressure V-cycle)");
    auto& L = levels<T>(h);
    const lmm_knobs& K = h->knobs;
    const int nl = h->nlev_p;
    const int lc = tail_start<T>(h, L, nl, false);
    LMM_CK(cudaMemsetAsync(L[0].pphi, 0, L[0].n * sizeof(T), h->stream));
    for (int vc = 0; vc < K.mg_max_vcycles; ++vc) {
        for (int l = 1; l <= std::min(lc, nl - 1); ++l) LMM_CK(cudaMemsetAsync(L[l].pphi, 0, L[l].n * sizeof(T), h->stream));
        for (int l = 0; l < lc && l < nl - 1; ++l) {
            cc_smooth<T>(h, L[l], K.mg_nsmooths_down);
            launch_cc_residual_restrict<T>(L[l], L[l + 1], h->stream);
            check_launch();
        }
        if (lc < nl) {
            LMM_CK(launch_ccmg_tail<T>(&L[lc], nl - lc, K.mg_nsmooths_down, K.mg_nsmooths_up, K.mg_nsmooths_bottom,
                                       h->stream));
            check_launch();
        } else {
            cc_smooth<T>(h, L[nl - 1], K.mg_nsmooths_bottom);
        }
        for (int l = std::min(lc, nl - 1) - 1; l >= 0; --l) {
            launch_cc_prolong_add<T>(L[l], L[l + 1], h->stream);
            check_launch();
            cc_smooth<T>(h, L[l], K.mg_nsmooths_up);
        }
    }
    h->pvcycles += K.mg_max_vcycles;
}

// ------------------------------------------------------------ apply_precon
template <class T>
struct PrecScratch {
    T* mac;
    T* src;
    T* xptmp;
    T* butmp[3];
    T* alphainv[3];
    T* bf[8];
};
template <class T>
PrecScratch<T> prec_scratch(lmm_handle* h);
template <>
PrecScratch<double> prec_scratch<double>(lmm_handle* h) {
    return {h->mac64, h->src64, h->xptmp64, {h->butmp64[0], h->butmp64[1], h->butmp64[2]},
            {h->alphainv[0], h->alphainv[1], h->alphainv[2]},
            {h->bf64[0], h->bf64[1], h->bf64[2], h->bf64[3], h->bf64[4], h->bf64[5], h->bf64[6], h->bf64[7]}};
}
template <>
PrecScratch<float> prec_scratch<float>(lmm_handle* h) {
    return {h->mac32, h->src32, h->xptmp32, {h->butmp32[0], h->butmp32[1], h->butmp32[2]},
            {h->alphainv32[0], h->alphainv32[1], h->alphainv32[2]},
            {h->bf32[0], h->bf32[1], h->bf32[2], h->bf32[3], h->bf32[4], h->bf32[5], h->bf32[6], h->bf32[7]}};
}

// sums of p and of the velocity components d in umask (bit d); the others
// are not read
template <class T>
void reduce_means(lmm_handle* h, T* const u[3], const T* p, int slot, int umask = 7);
template <>
void reduce_means<double>(lmm_handle* h, double* const u[3], const double* p, int slot, int umask) {
    const double* a[4] = {(umask & 1) ? u[0] : nullptr, (umask & 2) ? u[1] : nullptr,
                          (h->dm == 3 && (umask & 4)) ? u[2] : nullptr, p};
    const double* b[4] = {nullptr, nullptr, nullptr, nullptr};
    stokes_reduce(h, 1, a, b, slot);
}
template <>
void reduce_means<float>(lmm_handle* h, float* const u[3], const float* p, int slot, int umask) {
    const float* a[4] = {(umask & 1) ? u[0] : nullptr, (umask & 2) ? u[1] : nullptr,
                         (h->dm == 3 && (umask & 4)) ? u[2] : nullptr, p};
    const float* b[4] = {nullptr, nullptr, nullptr, nullptr};
    const int tile[3] = {1024000, 8, 8};
    double w[3];
    for (int d = 0; d < 3; ++d) {
        int nd = (d < h->dm) ? h->grid.n[d] : 1;
        w[d] = (nd / tile[d] < 2) ? 3.0 : 2.0;
    }
    launch_reduce<float>(h->D0, 1, a, b, w, 0.0, h->partials, h->counter, rslot(h, slot), h->red_blocks, h->stream, ninst(h));
    check_launch();
}

// visc_schur_complement (apply_precon.f90:538-685), the BFBt Schur
// approximation: with M = 1/diag(viscous operator) on faces,
//   x_p = (D M G)^-1 D M L M G (D M G)^-1 rhs  [+ theta alpha phi]
// where phi is the 1/alpha pressure solution already in L0.pphi; both
// Poisson solves use this library's pressure V-cycle with face coefficient
// M.  rhs (mac) is overwritten as in the reference.
template <class T>
void visc_schur(lmm_handle* h, T* mac, T* x_p) {
    auto& L = levels<T>(h);
    LevelDev<T>& L0 = L[0];
    const int dm = h->dm;
    const int64_t n = h->n;
    const double theta = h->theta_loaded;
    PrecScratch<T> S = prec_scratch<T>(h);
    T* zero = S.bf[0];
    T* keep = S.bf[1];
    T* g[3] = {S.bf[2], S.bf[3], S.bf[4]};
    T* lg[3] = {S.bf[5], S.bf[6], S.bf[7]};
    const T* m[3] = {L0.pmu[0], L0.pmu[1], L0.pmu[2]};
    if (std::fabs(theta) > 0.0) LMM_CK(cudaMemcpyAsync(keep, L0.pphi, n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
    // the pressure solves of BFBt use 1/diag(viscous operator) as face
    // coefficient: swapped into pa, with the uniform-coefficient path off
    std::vector<int> uni(h->nlev_p, 0);
    bool swapped = false;
    auto swap_coefficients = [&]() {
        swapped = !swapped;
        for (int l = 0; l < h->nlev_p; ++l) {
            for (int d = 0; d < dm; ++d) std::swap(L[l].pa[d], L[l].pmu[d]);
            if (swapped) {
                uni[l] = L[l].pa_uniform;
                L[l].pa_uniform = 0;
            } else {
                L[l].pa_uniform = uni[l];
            }
        }
    };
    swap_coefficients();
    // STEP 1: phi_mu = (D M G)^-1 rhs
    LMM_CK(cudaMemcpyAsync(L0.prhs, mac, n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
    macproject<T>(h);
    // STEP 2: rhs = D M L (M G phi_mu), L the viscous operator without theta alpha and gamma
    launch_grad_mul<T>(L0, L0.pphi, m, g, h->stream);
    check_launch();
    LMM_CK(cudaMemsetAsync(zero, 0, n * sizeof(T), h->stream));
    {
        LevelDev<T> Lv = L0;
        for (int d = 0; d < 3; ++d) Lv.alpha[d] = zero;
        Lv.a_uniform = 0;  // read the zero arrays
        Lv.gamma = zero;
        const T* gc[3] = {g[0], g[1], g[2]};
        launch_applyop<T>(Lv, h->knobs.visc_type, gc, lg, h->stream, 0);
        check_launch();
    }
    const T* lgc[3] = {lg[0], lg[1], lg[2]};
    launch_div_mul<T>(L0, lgc, m, mac, h->stream);
    check_launch();
    // STEP 3: x_p = (D M G)^-1 rhs
    LMM_CK(cudaMemcpyAsync(L0.prhs, mac, n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
    macproject<T>(h);
    swap_coefficients();
    LMM_CK(cudaMemcpyAsync(x_p, L0.pphi, n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
    // STEP 4: x_p += theta alpha phi
    if (std::fabs(theta) > 0.0) {
        launch_scale_copy<T>(keep, keep, theta, n, h->stream);
        check_launch();
        launch_add_to<T>(x_p, keep, n, h->stream);
        check_launch();
    }
}

// x = M^-1 b.  b_u / b_p and x_u / x_p are level-0 arrays of type T (they
// may alias the level-0 rhs / phi arrays of the hierarchy).
template <class T>
void apply_precon(lmm_handle* h, const T* const b_u[3], const T* b_p, T* const x_u[3], T* x_p) {
    NvtxRange nvtx_("apply_precon");
    const lmm_knobs& K = h->knobs;
    const int dm = h->dm;
    const int64_t n = h->n;
    const int pt = K.precon_type;
    const int av = std::abs(K.visc_type);
    const double theta = h->theta_loaded;
    auto& L = levels<T>(h);
    LevelDev<T>& L0 = L[0];
    PrecScratch<T> S = prec_scratch<T>(h);
    const int mean_slot = h->batched ? lmm_handle::kBSlots - 1 : h->kSlots - 3;

    // the staggered solve reads its rhs from L0.rhs and iterates on L0.phi
    auto vel_solve = [&](const T* const rhs[3], bool zero_guess) {
        for (int d = 0; d < dm; ++d) {
            if (rhs[d] != L0.rhs[d]) LMM_CK(cudaMemcpyAsync(L0.rhs[d], rhs[d], n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
            if (zero_guess) LMM_CK(cudaMemsetAsync(L0.phi[d], 0, n * sizeof(T), h->stream));
        }
        stag_mg_solver<T>(h);
        for (int d = 0; d < dm; ++d)
            if (x_u[d] != L0.phi[d]) LMM_CK(cudaMemcpyAsync(x_u[d], L0.phi[d], n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
    };
    auto pres_solve = [&](const T* rhs) {
        if (rhs != L0.prhs) LMM_CK(cudaMemcpyAsync(L0.prhs, rhs, n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
        macproject<T>(h);
    };
    const T* xu_c[3] = {x_u[0], x_u[1], x_u[2]};
    switch (std::abs(pt)) {
    case 1: {
        vel_solve(b_u, true);
        launch_div_plus<T>(L0, xu_c, b_p, S.mac, h->stream);
        check_launch();
        pres_solve(S.mac);
        const T* ai[3] = {S.alphainv[0], S.alphainv[1], S.alphainv[2]};
        launch_sub_weighted_grad<T>(L0, ai, L0.pphi, x_u, h->stream);
        check_launch();
        if (!(pt == 1 || theta == 0.0)) {
            launch_neg_cc_lap<T>(L0, L0.pphi, S.src, h->stream);
            check_launch();
        }
        if (K.visc_schur_approx == 1) {
            visc_schur<T>(h, S.mac, x_p);
        } else {
            launch_schur<T>(1, pt, av, theta, S.mac, S.src, L0.beta, L0.gamma, L0.pphi, b_p, x_p, n, h->stream);
            check_launch();
        }
        break;
    }
    case 2:
    case 5: {
        vel_solve(b_u, true);
        launch_div_plus<T>(L0, xu_c, b_p, S.mac, h->stream);
        check_launch();
        if (std::fabs(theta) > 0.0)
            pres_solve(S.mac);
        else
            LMM_CK(cudaMemsetAsync(L0.pphi, 0, n * sizeof(T), h->stream));
        if (K.visc_schur_approx == 1) {
            visc_schur<T>(h, S.mac, x_p);
            if (pt == -2 || pt == -5) {
                launch_scale_copy<T>(x_p, x_p, -1.0, n, h->stream);
                check_launch();
            }
        } else {
            launch_schur<T>(0, pt, av, theta, S.mac, nullptr, L0.beta, L0.gamma, L0.pphi, b_p, x_p, n, h->stream);
            check_launch();
        }
        if (std::abs(pt) == 5) {
            for (int d = 0; d < dm; ++d)
                LMM_CK(cudaMemcpyAsync(S.butmp[d], b_u[d], n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
            launch_sub_weighted_grad<T>(L0, nullptr, x_p, S.butmp, h->stream);
            check_launch();
            const T* bt[3] = {S.butmp[0], S.butmp[1], S.butmp[2]};
            // second viscous solve starts from the current x_u (apply_precon.f90:276)
            for (int d = 0; d < dm; ++d)
                if (x_u[d] != L0.phi[d])
                    LMM_CK(cudaMemcpyAsync(L0.phi[d], x_u[d], n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
            vel_solve(bt, false);
        }
        break;
    }
    case 3: {
        LMM_CK(cudaMemcpyAsync(S.mac, b_p, n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
        if (pt == -3) {
            launch_scale_copy<T>(S.mac, S.mac, -1.0, n, h->stream);
            check_launch();
        }
        if (std::fabs(theta) > 0.0)
            pres_solve(S.mac);
        else
            LMM_CK(cudaMemsetAsync(L0.pphi, 0, n * sizeof(T), h->stream));
        if (K.visc_schur_approx == 1) {
            visc_schur<T>(h, S.mac, x_p);
        } else {
            launch_schur<T>(0, 3, av, theta, S.mac, nullptr, L0.beta, L0.gamma, L0.pphi, b_p, x_p, n, h->stream);
            check_launch();
        }
        for (int d = 0; d < dm; ++d) LMM_CK(cudaMemcpyAsync(S.butmp[d], b_u[d], n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
        launch_sub_weighted_grad<T>(L0, nullptr, x_p, S.butmp, h->stream);
        check_launch();
        const T* bt[3] = {S.butmp[0], S.butmp[1], S.butmp[2]};
        vel_solve(bt, true);
        break;
    }
    case 4: {
        vel_solve(b_u, true);
        if (std::fabs(theta) > 0.0)
            pres_solve(b_p);
        else
            LMM_CK(cudaMemsetAsync(L0.pphi, 0, n * sizeof(T), h->stream));
        if (K.visc_schur_approx == 1) {
            // the reference leaves mac_rhs unset here when theta = 0; b_p is
            // what it holds whenever it is set (apply_precon.f90:362-366)
            LMM_CK(cudaMemcpyAsync(S.mac, b_p, n * sizeof(T), cudaMemcpyDeviceToDevice, h->stream));
            visc_schur<T>(h, S.mac, x_p);
        } else {
            launch_schur<T>(2, pt, av, theta, nullptr, nullptr, L0.beta, L0.gamma, L0.pphi, b_p, x_p, n, h->stream);
            check_launch();
        }
        break;
    }
    default:
        throw LmmError(LMM_ERR_INVALID);
    }
    // mean removal (apply_precon.f90:433-460)
    // only the sums the subtraction uses: p, and the velocity components of the mask
    reduce_means<T>(h, x_u, x_p, mean_slot, mean_mask(h, theta));
    double tv = 1.0;
    for (int d = 0; d < dm; ++d) tv *= (double)h->grid.n[d];
    launch_sub_means<T>(h->D0, x_u, x_p, rslot(h, mean_slot), tv, mean_mask(h, theta), h->stream);
    check_launch();
}

// Run `body` (a fixed sequence of launches on h->stream) through a CUDA graph
// keyed by (in, out, theta, precision): the first call runs eagerly (kernel
// attributes get set), the second captures and instantiates, later calls
// replay.  Launch and V-cycle counters advance as if launched eagerly.
template <class F>
void run_graphed(lmm_handle* h, const void* in, const void* out, int prec, F body) {
    // stag_mg_max_vcycles > 1 reads residual norms on the host between cycles
    if (h->knobs.use_graphs < 0 || h->knobs.stag_mg_max_vcycles > 1) {
        body();
        return;
    }
    auto key = std::make_tuple(in, out, h->theta_loaded, prec);
    lmm_handle::Graph& g = h->graphs[key];
    if (g.exec) {
        LMM_CK(cudaGraphLaunch(g.exec, h->stream));
        if (g_debug) LMM_CK(cudaStreamSynchronize(h->stream));
        for (int64_t q = 0; q < g.launches; ++q) count_launch();
        h->vcycles += g.vcycles;
        h->pvcycles += g.pvcycles;
        return;
    }
    if (g.seen++ == 0) {
        body();
        return;
    }
    const int64_t l0 = launches_total();
    const int v0 = h->vcycles, p0 = h->pvcycles;
    cudaGraph_t graph = nullptr;
    LMM_CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    try {
        body();
    } catch (...) {
        cudaStreamEndCapture(h->stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    LMM_CK(cudaStreamEndCapture(h->stream, &graph));
    cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        g_last_error = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e);
        throw LmmError(LMM_ERR_CUDA);
    }
    g.launches = launches_total() - l0;
    g.vcycles = h->vcycles - v0;
    g.pvcycles = h->pvcycles - p0;
    LMM_CK(cudaGraphLaunch(g.exec, h->stream));
    if (g_debug) LMM_CK(cudaStreamSynchronize(h->stream));
}

// FP64 Stokes vector in, FP64 Stokes vector out
void precon64(lmm_handle* h, const SVec& bin, const SVec& xout) {
    const double* bu[3] = {bin.c(0), bin.c(1), h->dm == 3 ? bin.c(2) : nullptr};
    double* xu[3] = {xout.c(0), xout.c(1), h->dm == 3 ? xout.c(2) : nullptr};
    run_graphed(h, bin.base, xout.base, 0, [&]() { apply_precon<double>(h, bu, bin.p(), xu, xout.p()); });
}

// FP64 Stokes vector in, FP32 Stokes vector out (Z storage).  converted:
// h->pin32 already holds bin in FP32 (written with bin by launch_div_by_f32)
void precon32(lmm_handle* h, const SVec& bin, float* zout, bool converted = false) {
    const int dm = h->dm;
    const int64_t n = h->n;
    run_graphed(h, bin.base, zout, converted ? 2 : 1, [&]() {
        if (!converted) {
            launch_convert<double, float>(bin.base, h->pin32, (int64_t)(dm + 1) * n, h->stream);
            check_launch();
        }
        const float* bu[3] = {h->pin32, h->pin32 + n, dm == 3 ? h->pin32 + 2 * n : nullptr};
        float* xu[3] = {zout, zout + n, dm == 3 ? zout + 2 * n : nullptr};
        apply_precon<float>(h, bu, h->pin32 + (int64_t)dm * n, xu, zout + (int64_t)dm * n);
    });
}

// ------------------------------------------------------------ Givens (host, gmres.f90:517-605)
void rotmat(double a, double b, double& cs, double& sn) {
    if (b == 0.0) {
        cs = 1.0;
        sn = 0.0;
    } else if (std::fabs(b) > std::fabs(a)) {
        double temp = a / b;
        sn = 1.0 / std::sqrt(1.0 + temp * temp);
        cs = temp * sn;
    } else {
        double temp = b / a;
        cs = 1.0 / std::sqrt(1.0 + temp * temp);
        sn = temp * cs;
    }
}

struct Hess {
    int ld;
    std::vector<double> v;
    double& operator()(int r, int c) { return v[(size_t)(r - 1) + (size_t)ld * (c - 1)]; }
};

void least_squares(int i, Hess& H, std::vector<double>& cs, std::vector<double>& sn, std::vector<double>& s) {
    for (int k = 1; k <= i - 1; ++k) {
        double temp = cs[k] * H(k, i) + sn[k] * H(k + 1, i);
        H(k + 1, i) = -sn[k] * H(k, i) + cs[k] * H(k + 1, i);
        H(k, i) = temp;
    }
    rotmat(H(i, i), H(i + 1, i), cs[i], sn[i]);
    double temp = cs[i] * s[i];
    s[i + 1] = -sn[i] * s[i];
    s[i] = temp;
    H(i, i) = cs[i] * H(i, i) + sn[i] * H(i + 1, i);
    H(i + 1, i) = 0.0;
}

void solve_utri(int k, Hess& H, std::vector<double>& s, std::vector<double>& y) {
    y[k + 1] = s[k + 1] / H(k + 1, k + 1);
    for (int i = k; i >= 1; --i) {
        double dot = 0.0;
        for (int q = i + 1; q <= k + 1; ++q) dot = dot + H(i, q) * y[q];
        y[i] = (s[i] - dot) / H(i, i);
    }
}

void push_hist(lmm_stats* st, double v) {
    if (st && st->n_history < LMM_HISTORY_MAX) st->history[st->n_history++] = v;
}

// MGS of w against V_0..V_{i-1} with H(k,i) kept on the device, then
// H(i+1,i) = |w|; returns the Hessenberg column on the host.
// Arnoldi column i in two halves: enqueue the projections of w and its norm
// (slots 1..i+1) and the copy of those slots to the host, then -- after the
// caller has enqueued whatever may run meanwhile -- wait for the copy only.
void arnoldi_column_enqueue(lmm_handle* h, int i) {
    NvtxRange nvtx_("arnoldi column (MGS)");
    const int64_t len = h->w.size();
    for (int k = 1; k <= i; ++k) {
        stokes_dot(h, h->w, h->V[k - 1], k);
        launch_sub_scaled(h->w.base, h->V[k - 1].base, h->slot(k) + 4, len, h->stream);
        check_launch();
    }
    stokes_norm(h, h->w, i + 1);
    LMM_CK(cudaMemcpyAsync(h->hscal, h->scal, 8 * sizeof(double) * (i + 2), cudaMemcpyDeviceToHost, h->stream));
    LMM_CK(cudaEventRecord(h->col_ev, h->stream));
}
void arnoldi_column_collect(lmm_handle* h, int i, std::vector<double>& col) {
    LMM_CK(cudaEventSynchronize(h->col_ev));
    col.assign(i + 2, 0.0);
    for (int k = 1; k <= i; ++k) col[k] = h->hscal[8 * k + 4];
    col[i + 1] = h->hscal[8 * (i + 1) + 5];
}

// The same column by classical Gram-Schmidt (FGMRES option): every
// <w, V_k> from the unmodified w in one pass, then one pass subtracting
// all projections, then the norm.  Same H entries up to rounding; three
// launches and about 2i+5 vector passes instead of 2i+1 launches and 5i+3.
void arnoldi_column(lmm_handle* h, int i, std::vector<double>& col) {
    arnoldi_column_enqueue(h, i);
    arnoldi_column_collect(h, i, col);
}

// The classical Gram-Schmidt column, launches only: H(k,i) into slots 1..i
// (entry 4), |w| into slot i+1 (entry 5); on a batch handle one of each per
// problem (slot arrays, stride batch * 8 between slots).
void cgs_column(lmm_handle* h, int i) {
    NvtxRange nvtx_("arnoldi column (CGS)");
    const int64_t len = h->w.size();
    const int64_t ss = h->batched ? (int64_t)h->batch * 8 : 8;
    const int64_t N = h->batched ? h->n : 0, ni = h->batched ? (int64_t)h->D0.nx * h->D0.ny : 0;
    for (int k0 = 0; k0 < i; k0 += 8) {
        MVecs V{};
        const int J = std::min(8, i - k0);
        for (int j = 0; j < J; ++j) V.p[j] = h->V[k0 + j].base;
        launch_mdot(h->D0, h->w.base, V, J, 3.0, h->knobs.p_norm_weight, h->partials, h->counter, rslot(h, k0 + 1), h->stream,
                    ninst(h), ss);
        check_launch();
    }
    for (int k0 = 0; k0 < i; k0 += 8) {
        MVecs V{};
        const int J = std::min(8, i - k0);
        for (int j = 0; j < J; ++j) V.p[j] = h->V[k0 + j].base;
        if (k0 + J < i) {
            launch_maxpy(h->w.base, V, J, rslot(h, k0 + 1), len, h->stream, N, ni, ss);
        } else {
            // the last projections and |w| in one pass over w
            launch_maxpy_norm(h->D0, h->w.base, V, J, rslot(h, k0 + 1), 3.0, h->knobs.p_norm_weight, h->partials, h->counter,
                              rslot(h, i + 1), h->stream, ninst(h), ss);
        }
        check_launch();
    }
}

void arnoldi_column_cgs_enqueue(lmm_handle* h, int i) {
    cgs_column(h, i);
    LMM_CK(cudaMemcpyAsync(h->hscal, h->scal, 8 * sizeof(double) * (i + 2), cudaMemcpyDeviceToHost, h->stream));
    LMM_CK(cudaEventRecord(h->col_ev, h->stream));
}

// ------------------------------------------------------------ the reference GMRES
int run_gmres(lmm_handle* h, double* theta_alpha, double* norm_pre_rhs, lmm_stats* st) {
    NvtxRange nvtx_("gmres");
    const lmm_knobs& K = h->knobs;
    const int m = K.gmres_max_inner;
    const int64_t len = h->b.size();
    std::vector<double> cs(m + 2), sn(m + 2), y(m + 2), s(m + 3), col;
    Hess H{m + 1, std::vector<double>((size_t)(m + 1) * m, 0.0)};

    h->vcycles = 0;
    precon64(h, h->b, h->tmp);
    stokes_norm(h, h->tmp, 0);
    const double norm_pre_b = read_slot(h, 0, 5);
    if (norm_pre_rhs) *norm_pre_rhs = norm_pre_b;
    stokes_norm(h, h->b, 0);
    const double norm_b = read_slot(h, 0, 5);
    if (st) {
        st->norm_b = norm_b;
        st->norm_pre_b = norm_pre_b;
    }
    if (!std::isfinite(norm_b) || !std::isfinite(norm_pre_b)) return LMM_ERR_NONFINITE;
    if (norm_b <= 0.0) {
        LMM_CK(cudaMemsetAsync(h->x.base, 0, len * sizeof(double), h->stream));
        return LMM_OK;
    }
    int status = LMM_OK;
    int total_iter = 0, iter = 0, i_copy = 0;
    double norm_init_resid = 0, norm_init_Stokes = 0;
    h->vcycles = 0;
    for (;;) {
        launch_apply_matrix(h->L64[0], K.visc_type, h->x, h->tmp, h->stream);
        check_launch();
        launch_neg_resid(h->tmp.base, h->b.base, len, h->stream);
        check_launch();
        stokes_norm(h, h->tmp, 0);
        int vtemp = h->vcycles;
        precon64(h, h->tmp, h->r);
        h->vcycles = vtemp;
        stokes_norm(h, h->r, 1);
        LMM_CK(cudaMemcpyAsync(h->hscal, h->scal, 16 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        LMM_CK(host_wait(h));
        const double norm_resid_Stokes = h->hscal[5];
        const double norm_resid = h->hscal[8 + 5];
        if (!std::isfinite(norm_resid) || !std::isfinite(norm_resid_Stokes)) return LMM_ERR_NONFINITE;
        if (iter == 0) {
            norm_init_Stokes = norm_resid_Stokes;
            norm_init_resid = norm_resid;
        }
        if (st) {
            st->norm_resid = norm_resid;
            st->norm_init_resid = norm_init_resid;
            st->norm_resid_true = norm_resid_Stokes;
            st->norm_init_true = norm_init_Stokes;
        }
        if (total_iter >= K.gmres_max_iter) {
            status = LMM_WARN_MAX_ITER;
            break;
        }
        if (total_iter >= K.gmres_min_iter) {
            if (norm_resid <= K.gmres_rel_tol * std::min(norm_pre_b, norm_init_resid)) {
                if (norm_resid_Stokes >= 10 * K.gmres_rel_tol * std::min(norm_b, norm_init_Stokes)) status = LMM_WARN_RESID_MISMATCH;
                break;
            } else if (norm_resid <= K.gmres_abs_tol) {
                break;
            }
        }
        if (iter >= K.gmres_max_outer) {
            status = LMM_WARN_MAX_OUTER;
            break;
        }
        iter = iter + 1;
        launch_div_by(h->r.base, h->V[0].base, h->slot(1) + 5, len, h->stream);
        check_launch();
        std::fill(s.begin(), s.end(), 0.0);
        s[1] = norm_resid;
        int i;
        for (i = 1; i <= m; ++i) {
            total_iter = total_iter + 1;
            i_copy = i;
            launch_apply_matrix(h->L64[0], K.visc_type, h->V[i - 1], h->tmp, h->stream);
            check_launch();
            precon64(h, h->tmp, h->w);
            arnoldi_column(h, i, col);
            for (int k = 1; k <= i + 1; ++k) H(k, i) = col[k];
            for (int k = 1; k <= i + 1; ++k)
                if (!std::isfinite(col[k])) return LMM_ERR_NONFINITE;
            if (H(i + 1, i) != 0.0) {
                launch_div_by(h->w.base, h->V[i].base, h->slot(i + 1) + 5, len, h->stream);
                check_launch();
            } else {
                g_last_error = "gmres: error in orthogonalization (H(i+1,i) == 0)";
                return LMM_ERR_BREAKDOWN;
            }
            least_squares(i, H, cs, sn, s);
            const double est = std::fabs(s[i + 1]);
            push_hist(st, est);
            if (total_iter >= K.gmres_max_iter) break;
            if (total_iter >= K.gmres_min_iter) {
                if (est <= K.gmres_rel_tol * std::min(norm_pre_b, norm_init_resid) || est <= K.gmres_abs_tol) break;
            }
        }
        solve_utri(i_copy - 1, H, s, y);
        for (int it = 1; it <= i_copy; ++it) {
            launch_add_scaled(h->x.base, h->V[it - 1].base, y[it], len, h->stream);
            check_launch();
        }
    }
    if (st) {
        st->total_iter = total_iter;
        st->outer_iter = iter;
        st->vcycles = h->vcycles;
    }
    (void)theta_alpha;
    return status;
}

// ------------------------------------------------------------ flexible GMRES
// ------------------------------------------------------------ learned stage
// After z1 = M v (FP32 V-cycles) and w = A z1: r1 = v - w, c = network(r1)
// with its means removed (the constant modes of the periodic operator, as
// apply_precon.f90:433-460 removes them from z1), and, when
// |r1 - A c| < |r1| (decided on the device, no host synchronisation),
// z = z1 + c (c kept in FP64 beside the FP32 basis) and w = A z1 + A c;
// otherwise c = 0 and the plain V-cycle result stands.  Mode 2 computes the
// correction but never accepts it (the stage's cost without its effect).
void learned_stage(lmm_handle* h, const SVec& c, const SVec& v, int mode) {
    NvtxRange nvtx_("learned stage");
    const int64_t len = v.size();
    const int S1 = lmm_handle::kLrnSlot, S2 = S1 + 1, S3 = S1 + 2;
    launch_lin(h->lr1.base, v.base, -1.0, h->w.base, len, h->stream);
    check_launch();
    stokes_norm(h, h->lr1, S1);
    launch_features(h->D0, h->lr1.base, h->L64[0].beta, h->slot(S1), h->grid.dx, nn::net_input(h->net), h->stream);
    check_launch();
    if (nn::net_forward_on(h->net, h->stream) != LMM_OK) throw LmmError(LMM_ERR_CUDA);
    launch_correction(h->D0, nn::net_output(h->net), h->L64[0].beta, h->slot(S1), h->grid.dx, c.base, h->stream);
    check_launch();
    {
        double* cu[3] = {c.c(0), c.c(1), c.c(2)};
        reduce_means<double>(h, cu, c.p(), S3);
        double tv = 1.0;
        for (int d = 0; d < h->dm; ++d) tv *= (double)h->grid.n[d];
        launch_sub_means<double>(h->D0, cu, c.p(), h->slot(S3), tv, mean_mask(h, h->theta_loaded), h->stream);
        check_launch();
    }
    launch_apply_matrix(h->L64[0], h->knobs.visc_type, c, h->lAc, h->stream);
    check_launch();
    launch_lin(h->le.base, h->lr1.base, -1.0, h->lAc.base, len, h->stream);
    check_launch();
    stokes_norm(h, h->le, S2);
    launch_accept(c.base, h->w.base, h->lAc.base, h->slot(S1) + 5, h->slot(S2) + 5, mode == 2 ? 0.0 : 1.0, h->luses, len,
                  h->stream);
    check_launch();
}

// The network's estimate of the error left by one preconditioner
// application: with w = A z1 for z1 = M v, the residual r1 = v - w goes
// through the network, whose output (scaled back) becomes c, with its
// constant modes removed like every preconditioner output.
void network_correction(lmm_handle* h, const SVec& c, const SVec& v) {
    const int64_t len = v.size();
    const int S1 = lmm_handle::kLrnSlot, S3 = S1 + 2;
    launch_lin(h->lr1.base, v.base, -1.0, h->w.base, len, h->stream);
    check_launch();
    stokes_norm(h, h->lr1, S1);
    launch_features(h->D0, h->lr1.base, h->L64[0].beta, h->slot(S1), h->grid.dx, nn::net_input(h->net), h->stream);
    check_launch();
    if (nn::net_forward_on(h->net, h->stream) != LMM_OK) throw LmmError(LMM_ERR_CUDA);
    launch_correction(h->D0, nn::net_output(h->net), h->L64[0].beta, h->slot(S1), h->grid.dx, c.base, h->stream);
    check_launch();
    double* cu[3] = {c.c(0), c.c(1), c.c(2)};
    reduce_means<double>(h, cu, c.p(), S3);
    double tv = 1.0;
    for (int d = 0; d < h->dm; ++d) tv *= (double)h->grid.n[d];
    launch_sub_means<double>(h->D0, cu, c.p(), h->slot(S3), tv, mean_mask(h, h->theta_loaded), h->stream);
    check_launch();
}

// Where a solve hands over to the plain restarted FGMRES (run_fgmres) at a
// restart: the counters so far and the first true residual.
struct FgmresResume {
    int total_iter, iter;
    double norm_init;
};
int run_fgmres(lmm_handle* h, double* norm_pre_rhs, lmm_stats* st, const FgmresResume* resume = nullptr);

// FGMRES with the learned stage as an extra direction (learned_stage = 1):
// every step adds two columns to the flexible Krylov basis, the FP32
// V-cycle's z1 = M v and the network's correction c of the residual
// v - A z1, and the least-squares problem minimises over both.  A cycle
// holds m V-cycle columns (up to 2m columns in all); a network column
// whose image lies in the span of the basis already (|w| after
// orthogonalisation below 1e-8 of |A c|) is dropped, so it can neither
// end a cycle as a false breakdown nor make the Hessenberg matrix
// singular.  Iterations count V-cycle applications, as without the stage.
// learned_stage = 2 computes every correction and adds none (the cost of
// the stage without its effect: bitwise the stage-free solve).
// learned_stage = 4 lets the GMRES residual judge the network: a network
// column that lowers the residual estimate |s_{i+1}| by less than 10%
// (or is dropped) is a miss, and after two misses the solve goes on with
// the plain V-cycle alone -- no further forward passes; at the next
// restart it hands the iterate over to the plain restarted FGMRES (the same
// V-cycle columns and arithmetic, with its look-ahead).  Each solve judges
// afresh.
int run_fgmres_augmented(lmm_handle* h, double* norm_pre_rhs, lmm_stats* st) {
    NvtxRange nvtx_("fgmres (learned columns)");
    const lmm_knobs& K = h->knobs;
    const int m = K.gmres_max_inner;
    const int mc = 2 * m;  // columns per cycle
    const int64_t len = h->b.size();
    const bool judged = (K.learned_stage == 4);
    const bool add = (K.learned_stage == 1 || judged);
    LMM_CK(cudaMemsetAsync(h->luses, 0, 2 * sizeof(int), h->stream));
    int net_tried = 0, net_kept = 0, net_misses = 0;
    bool net_on = true;  // judged: false once the network has missed twice
    std::vector<double> cs(mc + 2), sn(mc + 2), y(mc + 2), s(mc + 3), col;
    Hess H{mc + 1, std::vector<double>((size_t)(mc + 1) * mc, 0.0)};
    std::vector<const void*> zcol(mc + 1);
    std::vector<int> zkind(mc + 1);  // 0: FP32 V-cycle column, 1: FP64 network column
    h->vcycles = 0;
    if (norm_pre_rhs) *norm_pre_rhs = 0.0;
    stokes_norm(h, h->b, 0);
    const double norm_b = read_slot(h, 0, 5);
    if (st) st->norm_b = norm_b;
    if (!std::isfinite(norm_b)) return LMM_ERR_NONFINITE;
    if (norm_b <= 0.0) {
        LMM_CK(cudaMemsetAsync(h->x.base, 0, len * sizeof(double), h->stream));
        return LMM_OK;
    }
    int status = LMM_OK, total_iter = 0, iter = 0;
    double norm_init = 0.0;
    auto col_norms_ok = [](const std::vector<double>& c, int i) {
        for (int k = 1; k <= i + 1; ++k)
            if (!std::isfinite(c[k])) return false;
        return true;
    };
    for (;;) {
        if (judged && !net_on) {
            // the network is out for this solve: the plain FGMRES takes over
            int u[2] = {net_kept, net_tried};
            LMM_CK(cudaMemcpyAsync(h->luses, u, sizeof(u), cudaMemcpyHostToDevice, h->stream));
            LMM_CK(host_wait(h));
            const FgmresResume r{total_iter, iter, norm_init};
            return run_fgmres(h, norm_pre_rhs, st, &r);
        }
        launch_apply_matrix(h->L64[0], K.visc_type, h->x, h->tmp, h->stream);
        check_launch();
        launch_neg_resid(h->tmp.base, h->b.base, len, h->stream);
        check_launch();
        stokes_norm(h, h->tmp, 0);
        const double norm_r = read_slot(h, 0, 5);
        if (!std::isfinite(norm_r)) return LMM_ERR_NONFINITE;
        if (iter == 0) norm_init = norm_r;
        if (st) {
            st->norm_resid_true = norm_r;
            st->norm_init_true = norm_init;
            st->norm_resid = norm_r;
        }
        if (total_iter >= K.gmres_min_iter && (norm_r <= K.gmres_rel_tol * norm_b || norm_r <= K.gmres_abs_tol)) break;
        if (total_iter >= K.gmres_max_iter) {
            status = LMM_WARN_MAX_ITER;
            break;
        }
        if (iter >= K.gmres_max_outer) {
            status = LMM_WARN_MAX_OUTER;
            break;
        }
        iter = iter + 1;
        launch_div_by_f32(h->tmp.base, h->V[0].base, h->pin32, h->slot(0) + 5, len, h->stream);
        check_launch();
        std::fill(s.begin(), s.end(), 0.0);
        s[1] = norm_r;
        int i = 0;      // columns of this cycle
        bool stop = false;
        // one column: Arnoldi of w against V_0..V_{i-1}, V_i = w / H(i+1,i),
        // the Hessenberg column to the host; false when the column is dropped
        // (a network column is orthogonalised by modified Gram-Schmidt whatever
        // the knob: it is often close to the span of the basis, where one
        // classical pass loses orthogonality)
        auto arnoldi = [&](int i1, bool droppable) -> bool {
            if (K.orthogonalization == 1 && !droppable)
                arnoldi_column_cgs_enqueue(h, i1);
            else
                arnoldi_column_enqueue(h, i1);
            launch_div_by_f32(h->w.base, h->V[i1].base, h->pin32, h->slot(i1 + 1) + 5, len, h->stream);
            check_launch();
            arnoldi_column_collect(h, i1, col);
            if (!col_norms_ok(col, i1)) throw LmmError(LMM_ERR_NONFINITE);
            if (droppable) {
                double proj = 0.0;
                for (int k = 1; k <= i1; ++k) proj += col[k] * col[k];
                const double full = std::sqrt(proj + col[i1 + 1] * col[i1 + 1]);
                if (!(col[i1 + 1] > 1e-8 * full)) return false;
            }
            for (int k = 1; k <= i1 + 1; ++k) H(k, i1) = col[k];
            return true;
        };
        auto after_column = [&](int i1) {
            const bool happy = (H(i1 + 1, i1) == 0.0);
            least_squares(i1, H, cs, sn, s);
            const double est = std::fabs(s[i1 + 1]);
            push_hist(st, est);
            if (happy || (total_iter >= K.gmres_min_iter && (est <= K.gmres_rel_tol * norm_b || est <= K.gmres_abs_tol)))
                stop = true;
        };
        // The V-cycle is applied to the basis vector its own previous column
        // produced (vin), never to one a network column produced: without
        // network columns this is plain FGMRES step for step, and the network
        // only adds directions to the space the least-squares step minimises
        // over.
        int vin = 0;
        bool pin_ok = true;  // h->pin32 holds V[vin] in FP32 (written with it)
        for (int k = 0; k < m && !stop; ++k) {
            // V-cycle column: z = M v (FP32), w = A z
            total_iter = total_iter + 1;
            precon32(h, h->V[vin], h->Z32[k], pin_ok);
            launch_apply_matrix_f32(h->L64[0], K.visc_type, h->Z32[k], h->n, h->dm, h->w, h->stream);
            check_launch();
            // the network's correction of what this application leaves (before
            // the Arnoldi step overwrites w)
            if (net_on) {
                network_correction(h, h->Zc[k], h->V[vin]);
                ++net_tried;
            }
            i = i + 1;
            zcol[i] = h->Z32[k];
            zkind[i] = 0;
            arnoldi(i, false);
            vin = i;
            pin_ok = true;
            after_column(i);
            if (stop || total_iter >= K.gmres_max_iter) {
                stop = true;
                break;
            }
            if (!add || !net_on || i + 1 > mc) continue;
            // network column: z = c, w = A c
            const double est_before = std::fabs(s[i + 1]);
            launch_apply_matrix(h->L64[0], K.visc_type, h->Zc[k], h->w, h->stream);
            check_launch();
            pin_ok = false;  // the network column's V overwrote the FP32 copy of V[vin]
            bool helped = false;
            if (arnoldi(i + 1, true)) {
                i = i + 1;
                zcol[i] = h->Zc[k].base;
                zkind[i] = 1;
                ++net_kept;
                after_column(i);
                helped = std::fabs(s[i + 1]) < 0.9 * est_before;
            }
            if (judged && !helped && ++net_misses >= 2) net_on = false;
        }
        solve_utri(i - 1, H, s, y);
        // update_sol: runs of consecutive V-cycle columns as in run_fgmres
        // (up to 8 FP32 basis vectors per pass), network columns one by one
        for (int it = 1; it <= i;) {
            if (zkind[it] == 1) {
                launch_add_scaled(h->x.base, static_cast<const double*>(zcol[it]), y[it], len, h->stream);
                check_launch();
                ++it;
                continue;
            }
            MZ32 Z{};
            YS ys{};
            int J = 0;
            while (J < 8 && it + J <= i && zkind[it + J] == 0) {
                Z.p[J] = static_cast<const float*>(zcol[it + J]);
                ys.y[J] = y[it + J];
                ++J;
            }
            launch_add_scaled_multi_f32(h->x.base, Z, ys, J, len, h->stream);
            check_launch();
            it += J;
        }
    }
    int u[2] = {net_kept, net_tried};
    LMM_CK(cudaMemcpyAsync(h->luses, u, sizeof(u), cudaMemcpyHostToDevice, h->stream));
    LMM_CK(host_wait(h));
    if (st) {
        st->total_iter = total_iter;
        st->outer_iter = iter;
        st->vcycles = h->vcycles;
    }
    return status;
}

// resume: continue a solve that run_fgmres_augmented hands over at a
// restart (its counters kept, the learned stage off from there on).
int run_fgmres(lmm_handle* h, double* norm_pre_rhs, lmm_stats* st, const FgmresResume* resume) {
    NvtxRange nvtx_("fgmres");
    const lmm_knobs& K = h->knobs;
    const int m = K.gmres_max_inner;
    const int64_t len = h->b.size();
    const bool fp32 = (K.precision == LMM_PRECISION_FP32);
    const bool learned = fp32 && K.learned_stage > 0 && h->net != nullptr && !resume;
    if (learned && (K.learned_stage == 1 || K.learned_stage == 2 || K.learned_stage == 4))
        return run_fgmres_augmented(h, norm_pre_rhs, st);
    if (learned) LMM_CK(cudaMemsetAsync(h->luses, 0, 2 * sizeof(int), h->stream));
    std::vector<double> cs(m + 2), sn(m + 2), y(m + 2), s(m + 3), col;
    Hess H{m + 1, std::vector<double>((size_t)(m + 1) * m, 0.0)};
    if (!resume) {
        h->vcycles = 0;
        if (norm_pre_rhs) *norm_pre_rhs = 0.0;
    }
    stokes_norm(h, h->b, 0);
    const double norm_b = read_slot(h, 0, 5);
    if (st) st->norm_b = norm_b;
    if (!std::isfinite(norm_b)) return LMM_ERR_NONFINITE;
    if (norm_b <= 0.0) {
        LMM_CK(cudaMemsetAsync(h->x.base, 0, len * sizeof(double), h->stream));
        return LMM_OK;
    }
    int status = LMM_OK, total_iter = resume ? resume->total_iter : 0, iter = resume ? resume->iter : 0;
    double norm_init = resume ? resume->norm_init : 0.0;
    for (;;) {
        launch_apply_matrix(h->L64[0], K.visc_type, h->x, h->tmp, h->stream);
        check_launch();
        launch_neg_resid(h->tmp.base, h->b.base, len, h->stream);
        check_launch();
        stokes_norm(h, h->tmp, 0);
        const double norm_r = read_slot(h, 0, 5);
        if (!std::isfinite(norm_r)) return LMM_ERR_NONFINITE;
        if (iter == 0) norm_init = norm_r;
        if (st) {
            st->norm_resid_true = norm_r;
            st->norm_init_true = norm_init;
            st->norm_resid = norm_r;
        }
        if (total_iter >= K.gmres_min_iter && (norm_r <= K.gmres_rel_tol * norm_b || norm_r <= K.gmres_abs_tol)) break;
        if (total_iter >= K.gmres_max_iter) {
            status = LMM_WARN_MAX_ITER;
            break;
        }
        if (iter >= K.gmres_max_outer) {
            status = LMM_WARN_MAX_OUTER;
            break;
        }
        iter = iter + 1;
        if (fp32)
            launch_div_by_f32(h->tmp.base, h->V[0].base, h->pin32, h->slot(0) + 5, len, h->stream);
        else
            launch_div_by(h->tmp.base, h->V[0].base, h->slot(0) + 5, len, h->stream);
        check_launch();
        std::fill(s.begin(), s.end(), 0.0);
        s[1] = norm_r;
        int i, i_copy = 0;
        bool happy = false;
        // While the host reads column i of H and applies its Givens rotation,
        // the device may already run the next column's preconditioner and
        // operator application (V_i = w / H(i+1,i) is formed on the device):
        // done when the last residual estimate is far (50x) above the
        // stopping threshold, so a column computed ahead is almost never
        // thrown away.
        const bool can_ahead = !learned && K.stag_mg_max_vcycles <= 1;
        const double thr = std::max(K.gmres_rel_tol * norm_b, K.gmres_abs_tol);
        double est_prev = norm_r;
        bool ahead = false;
        int ahead_v = 0, ahead_p = 0;
        auto column_work = [&](int c) {  // Z_c = M^-1 V_c, w = A Z_c (c 0-based)
            if (fp32) {
                precon32(h, h->V[c], h->Z32[c], true);
                launch_apply_matrix_f32(h->L64[0], K.visc_type, h->Z32[c], h->n, h->dm, h->w, h->stream);
                if (learned) learned_stage(h, h->Zc[c], h->V[c], 1);
            } else {
                precon64(h, h->V[c], h->Z64[c]);
                launch_apply_matrix(h->L64[0], K.visc_type, h->Z64[c], h->w, h->stream);
            }
            check_launch();
        };
        for (i = 1; i <= m; ++i) {
            total_iter = total_iter + 1;
            i_copy = i;
            if (!ahead) column_work(i - 1);
            ahead = false;
            if (K.orthogonalization == 1)
                arnoldi_column_cgs_enqueue(h, i);
            else
                arnoldi_column_enqueue(h, i);
            // V_i = w / H(i+1,i) (a zero H(i+1,i) ends the cycle below, V_i unused)
            if (fp32)
                launch_div_by_f32(h->w.base, h->V[i].base, h->pin32, h->slot(i + 1) + 5, len, h->stream);
            else
                launch_div_by(h->w.base, h->V[i].base, h->slot(i + 1) + 5, len, h->stream);
            check_launch();
            if (can_ahead && i < m && total_iter < K.gmres_max_iter &&
                (total_iter < K.gmres_min_iter || est_prev > 50.0 * thr)) {
                ahead_v = h->vcycles;
                ahead_p = h->pvcycles;
                column_work(i);
                ahead_v = h->vcycles - ahead_v;
                ahead_p = h->pvcycles - ahead_p;
                ahead = true;
            }
            arnoldi_column_collect(h, i, col);
            for (int k = 1; k <= i + 1; ++k) H(k, i) = col[k];
            for (int k = 1; k <= i + 1; ++k)
                if (!std::isfinite(col[k])) return LMM_ERR_NONFINITE;
            if (H(i + 1, i) == 0.0) happy = true;
            least_squares(i, H, cs, sn, s);
            const double est = std::fabs(s[i + 1]);
            push_hist(st, est);
            est_prev = est;
            if (happy || total_iter >= K.gmres_max_iter) break;
            if (total_iter >= K.gmres_min_iter && (est <= K.gmres_rel_tol * norm_b || est <= K.gmres_abs_tol)) break;
        }
        if (ahead) {
            // a column computed ahead of a converged cycle: not part of the solve
            h->vcycles -= ahead_v;
            h->pvcycles -= ahead_p;
        }
        solve_utri(i_copy - 1, H, s, y);
        if (fp32 && !learned) {
            // update_sol: x += sum y_k Z_k, up to 8 basis vectors per pass
            for (int k0 = 1; k0 <= i_copy; k0 += 8) {
                const int J = std::min(8, i_copy - k0 + 1);
                MZ32 Z{};
                YS ys{};
                for (int j = 0; j < J; ++j) {
                    Z.p[j] = h->Z32[k0 + j - 1];
                    ys.y[j] = y[k0 + j];
                }
                launch_add_scaled_multi_f32(h->x.base, Z, ys, J, len, h->stream);
                check_launch();
            }
        } else {
            for (int it = 1; it <= i_copy; ++it) {
                if (fp32) {
                    launch_add_scaled_f32(h->x.base, h->Z32[it - 1], y[it], len, h->stream);
                    check_launch();
                    launch_add_scaled(h->x.base, h->Zc[it - 1].base, y[it], len, h->stream);
                } else
                    launch_add_scaled(h->x.base, h->Z64[it - 1].base, y[it], len, h->stream);
                check_launch();
            }
        }
    }
    if (st) {
        st->total_iter = total_iter;
        st->outer_iter = iter;
        st->vcycles = h->vcycles;
    }
    return status;
}

// ------------------------------------------------------------ batches of 2D problems
// FGMRES (modified or classical Gram-Schmidt, knobs.orthogonalization) on
// the instances of a batch handle at once:
// every vector operation, preconditioner application and reduction covers
// the whole batch in one launch, while the host keeps per instance the
// Hessenberg matrix, Givens sequence, stopping decisions and statistics of
// run_fgmres.  Per instance the arithmetic is run_fgmres's (the reductions
// partition and sum each instance as they would one problem).  An instance that has stopped rides along: its
// columns are computed and not used, its update coefficients are zero.
int run_fgmres_batch(lmm_handle* h, int count, lmm_stats* stats, int* status) {
    NvtxRange nvtx_("fgmres batch");
    const lmm_knobs& K = h->knobs;
    const int m = K.gmres_max_inner, B = h->batch, ni = h->D0.nx * h->D0.ny;
    const int64_t n = h->n, len = h->b.size();
    const bool fp32 = (K.precision == LMM_PRECISION_FP32);
    // slots s0 .. s0+ns-1 to the host: bhost[(k - s0) * B * 8 + b * 8 + c]
    auto fetch = [&](int s0, int ns) {
        LMM_CK(cudaMemcpyAsync(h->bhost, h->bslot(s0), sizeof(double) * ns * B * 8, cudaMemcpyDeviceToHost, h->stream));
        LMM_CK(host_wait(h));
    };
    auto at = [&](int k, int s0, int b, int c) { return h->bhost[(int64_t)(k - s0) * B * 8 + b * 8 + c]; };
    struct Inst {
        Hess H;
        std::vector<double> cs, sn, s, y;
        double norm_b = 0.0, norm_init = 0.0, norm_r = 0.0;
        bool done = false, stop = false;
        int ib = 0, total = 0, outer = 0, status = LMM_OK;
    };
    std::vector<Inst> P(B);
    int64_t apps = 0;  // preconditioner applications (each covers the batch)
    for (auto& p : P) {
        p.H = Hess{m + 1, std::vector<double>((size_t)(m + 1) * m, 0.0)};
        p.cs.assign(m + 2, 0.0);
        p.sn.assign(m + 2, 0.0);
        p.s.assign(m + 3, 0.0);
        p.y.assign(m + 2, 0.0);
    }
    h->vcycles = 0;
    stokes_norm(h, h->b, 0);
    fetch(0, 1);
    for (int b = 0; b < B; ++b) {
        Inst& p = P[b];
        p.norm_b = at(0, 0, b, 5);
        if (b < count) stats[b].norm_b = p.norm_b;
        if (!std::isfinite(p.norm_b)) {
            p.status = LMM_ERR_NONFINITE;
            p.done = true;
        } else if (p.norm_b <= 0.0) {
            p.done = true;  // x = 0 (gmres.f90:142-150)
            for (int c = 0; c <= h->dm; ++c)
                LMM_CK(cudaMemsetAsync(h->x.c(c) + (int64_t)b * ni, 0, sizeof(double) * ni, h->stream));
        }
    }
    auto column_work = [&](int c) {  // Z_c = M^-1 V_c, w = A Z_c
        if (fp32) {
            precon32(h, h->V[c], h->Z32[c], true);
            launch_apply_matrix_f32(h->L64[0], K.visc_type, h->Z32[c], h->n, h->dm, h->w, h->stream);
        } else {
            precon64(h, h->V[c], h->Z64[c]);
            launch_apply_matrix(h->L64[0], K.visc_type, h->Z64[c], h->w, h->stream);
        }
        check_launch();
        ++apps;
    };
    int iter = 0;
    bool first = true;
    for (;;) {
        launch_apply_matrix(h->L64[0], K.visc_type, h->x, h->tmp, h->stream);
        check_launch();
        launch_neg_resid(h->tmp.base, h->b.base, len, h->stream);
        check_launch();
        stokes_norm(h, h->tmp, 0);
        fetch(0, 1);
        bool any = false;
        for (int b = 0; b < B; ++b) {
            Inst& p = P[b];
            if (p.done) continue;
            p.norm_r = at(0, 0, b, 5);
            if (!std::isfinite(p.norm_r)) {
                p.status = LMM_ERR_NONFINITE;
                p.done = true;
                continue;
            }
            if (first) p.norm_init = p.norm_r;
            if (p.total >= K.gmres_min_iter && (p.norm_r <= K.gmres_rel_tol * p.norm_b || p.norm_r <= K.gmres_abs_tol)) {
                p.done = true;
            } else if (p.total >= K.gmres_max_iter) {
                p.status = LMM_WARN_MAX_ITER;
                p.done = true;
            } else if (iter >= K.gmres_max_outer) {
                p.status = LMM_WARN_MAX_OUTER;
                p.done = true;
            } else {
                any = true;
            }
        }
        first = false;
        if (!any) break;
        iter = iter + 1;
        launch_div_by_batch(h->tmp.base, h->V[0].base, fp32 ? h->pin32 : nullptr, h->bslot(0), n, ni, len, h->stream);
        check_launch();
        for (auto& p : P) {
            if (!p.done) p.outer = iter;
            p.stop = p.done;
            p.ib = 0;
            std::fill(p.s.begin(), p.s.end(), 0.0);
            p.s[1] = p.norm_r;
        }
        for (int i = 1; i <= m; ++i) {
            column_work(i - 1);
            if (K.orthogonalization == 1) {
                cgs_column(h, i);
            } else {
                for (int k = 1; k <= i; ++k) {
                    stokes_dot(h, h->w, h->V[k - 1], k);
                    launch_sub_scaled_batch(h->w.base, h->V[k - 1].base, h->bslot(k), n, ni, len, h->stream);
                    check_launch();
                }
                stokes_norm(h, h->w, i + 1);
            }
            launch_div_by_batch(h->w.base, h->V[i].base, fp32 ? h->pin32 : nullptr, h->bslot(i + 1), n, ni, len, h->stream);
            check_launch();
            fetch(1, i + 1);
            bool cont = false;
            for (int b = 0; b < B; ++b) {
                Inst& p = P[b];
                if (p.stop) continue;
                p.total = p.total + 1;
                bool bad = false;
                for (int k = 1; k <= i; ++k) p.H(k, i) = at(k, 1, b, 4);
                p.H(i + 1, i) = at(i + 1, 1, b, 5);
                for (int k = 1; k <= i + 1; ++k) bad = bad || !std::isfinite(p.H(k, i));
                if (bad) {
                    p.status = LMM_ERR_NONFINITE;
                    p.done = p.stop = true;
                    p.ib = 0;
                    continue;
                }
                // a zero H(i+1,i) (happy breakdown) is read before the
                // Givens rotation of least_squares overwrites it
                const bool happy = (p.H(i + 1, i) == 0.0);
                least_squares(i, p.H, p.cs, p.sn, p.s);
                p.ib = i;
                const double est = std::fabs(p.s[i + 1]);
                if (b < count) push_hist(&stats[b], est);
                if (happy || p.total >= K.gmres_max_iter)
                    p.stop = true;
                else if (p.total >= K.gmres_min_iter && (est <= K.gmres_rel_tol * p.norm_b || est <= K.gmres_abs_tol))
                    p.stop = true;
                else
                    cont = true;
            }
            if (!cont) break;
        }
        // x += sum_k y_k Z_k per instance (update_sol)
        int J = 0;
        for (auto& p : P) {
            if (p.done || p.ib == 0) continue;
            solve_utri(p.ib - 1, p.H, p.s, p.y);
            J = std::max(J, p.ib);
        }
        if (J > 0) {
            for (int k = 0; k < J; ++k)
                for (int b = 0; b < B; ++b) {
                    const Inst& p = P[b];
                    h->ys_host[(int64_t)k * B + b] = (!p.done && k < p.ib) ? p.y[k + 1] : 0.0;
                }
            LMM_CK(cudaMemcpyAsync(h->ys, h->ys_host, sizeof(double) * J * B, cudaMemcpyHostToDevice, h->stream));
            if (fp32)
                launch_add_scaled_multi_batch<float>(h->x.base, reinterpret_cast<const float* const*>(h->ztab), h->ys, J, B, n, ni,
                                                     len, h->stream);
            else
                launch_add_scaled_multi_batch<double>(h->x.base, reinterpret_cast<const double* const*>(h->ztab), h->ys, J, B, n,
                                                      ni, len, h->stream);
            check_launch();
        }
    }
    // per instance as one solve reports them: V-cycles of its own columns
    const int64_t v_per = apps > 0 ? h->vcycles / apps : 0, p_per = apps > 0 ? h->pvcycles / apps : 0;
    int worst = LMM_OK;
    for (int b = 0; b < count; ++b) {
        const Inst& p = P[b];
        lmm_stats& st = stats[b];
        st.total_iter = p.total;
        st.outer_iter = p.outer;
        st.vcycles = (int)(v_per * p.total);
        st.pressure_vcycles = (int)(p_per * p.total);
        st.norm_resid_true = p.norm_r;
        st.norm_init_true = p.norm_init;
        st.norm_resid = p.norm_r;
        status[b] = p.status;
        if (p.status < 0)
            worst = std::min(worst, p.status);
        else if (worst >= 0)
            worst = std::max(worst, p.status);
    }
    return worst;
}

int validate(const lmm_grid* g, const lmm_knobs* k) {
    if (!g || !k) return LMM_ERR_INVALID;
    if (g->dm != 2 && g->dm != 3) return LMM_ERR_INVALID;
    if (!(g->dx > 0.0)) return LMM_ERR_INVALID;
    bool walls = false;
    for (int d = 0; d < g->dm; ++d) {
        if (g->n[d] < 2) return LMM_ERR_INVALID;
        const bool per = g->bc_lo[d] == LMM_BC_PERIODIC && g->bc_hi[d] == LMM_BC_PERIODIC;
        if (!per && !(bc_wall(g->bc_lo[d]) && bc_wall(g->bc_hi[d]))) {
            g_last_error = "a direction is periodic on both sides or bounded by walls (100-103 no-slip, 200-203 slip) on both";
            return LMM_ERR_INVALID;
        }
        walls = walls || !per;
    }
    const int av = std::abs(k->visc_type);
    if (av < 1 || av > 3) return LMM_ERR_INVALID;
    const int ap = std::abs(k->precon_type);
    if (ap < 1 || ap > 5) {
        g_last_error = "unsupported precon_type";
        return LMM_ERR_INVALID;
    }
    if (k->visc_schur_approx != 0 && k->visc_schur_approx != 1) return LMM_ERR_INVALID;
    if (k->visc_schur_approx == 1 && av == 3) {
        // inverse_diag_lap.f90:135,246
        g_last_error = "inverse_diag_lap does not support abs(visc_type) = 3";
        return LMM_ERR_INVALID;
    }
    if (k->gmres_max_inner < 1 || k->gmres_max_inner > 120) return LMM_ERR_INVALID;
    if (k->method != LMM_METHOD_GMRES && k->method != LMM_METHOD_FGMRES) return LMM_ERR_INVALID;
    if (k->precision == LMM_PRECISION_FP32 && k->method != LMM_METHOD_FGMRES) {
        g_last_error = "the FP32 preconditioner needs LMM_METHOD_FGMRES";
        return LMM_ERR_INVALID;
    }
    if (k->stag_mg_smoother != 0 && k->stag_mg_smoother != 1) return LMM_ERR_INVALID;
    if (k->orthogonalization != 0 && !(k->orthogonalization == 1 && k->method == LMM_METHOD_FGMRES)) {
        g_last_error = "classical Gram-Schmidt (orthogonalization = 1) is an FGMRES option";
        return LMM_ERR_INVALID;
    }
    // levels halve exactly down to the coarsest (which may have an odd cell
    // count: its colours are then applied in the reference's two steps)
    int nl = compute_nlevs(g->n, g->dm, k->stag_mg_minwidth);
    for (int d = 0; d < g->dm; ++d)
        if ((g->n[d] >> (nl - 1)) << (nl - 1) != g->n[d]) return LMM_ERR_INVALID;
    if (walls) {
        if (k->visc_schur_approx == 1) {
            g_last_error = "the BFBt Schur approximation (visc_schur_approx = 1) needs a periodic box";
            return LMM_ERR_INVALID;
        }
        if (k->learned_stage > 0) {
            g_last_error = "the learned stage needs a periodic box";
            return LMM_ERR_INVALID;
        }
        const int nlp = compute_nlevs(g->n, g->dm, k->mg_minwidth);
        for (int d = 0; d < g->dm; ++d)
            if ((g->n[d] >> (nl - 1)) < 2 || (g->n[d] >> (nlp - 1)) < 2) {
                g_last_error = "with walls every multigrid level needs at least 2 cells per direction";
                return LMM_ERR_INVALID;
            }
    }
    return LMM_OK;
}

}  // namespace

// ============================================================ C ABI
extern "C" {

int lmm_version(void) { return 100; }

const char* lmm_strerror(int code) {
    switch (code) {
    case LMM_OK: return "converged";
    case LMM_WARN_MAX_ITER: return "GMRES did not converge in max number of total inner iterations";
    case LMM_WARN_MAX_OUTER: return "GMRES did not converge in max number of outer iterations";
    case LMM_WARN_RESID_MISMATCH: return "gmres may not have converged: true residual disagrees with preconditioned residual";
    case LMM_ERR_INVALID: return g_last_error.empty() ? "invalid argument" : g_last_error.c_str();
    case LMM_ERR_BREAKDOWN: return "gmres: error in orthogonalization";
    case LMM_ERR_NONFINITE: return "non-finite value in an input or a residual";
    case LMM_ERR_CUDA: return g_last_error.empty() ? "CUDA error" : g_last_error.c_str();
    case LMM_ERR_WATCHDOG: return "a bounded device wait gave up";
    case LMM_ERR_NO_DEVICE: return "no CUDA device";
    case LMM_ERR_BOUNDS: return g_last_error.empty() ? "a load outside the registered allocations was skipped" : g_last_error.c_str();
    case LMM_ERR_TOO_LARGE: return "grid larger than this fixed-size entry point accepts";
    default: return "unknown status";
    }
}

void lmm_default_knobs(lmm_knobs* k) {
    std::memset(k, 0, sizeof(*k));
    k->precon_type = 1;
    k->visc_schur_approx = 0;
    k->p_norm_weight = 1.0;
    k->scale_factor = 1.0;
    k->mg_max_vcycles = 1;
    k->mg_minwidth = 2;
    k->mg_bottom_solver = 4;
    k->mg_nsmooths_down = 2;
    k->mg_nsmooths_up = 2;
    k->mg_nsmooths_bottom = 8;
    k->mg_max_bottom_nlevels = 10;
    k->mg_rel_tol = 1e-9;
    k->stag_mg_max_vcycles = 1;
    k->stag_mg_minwidth = 2;
    k->stag_mg_bottom_solver = 4;
    k->stag_mg_nsmooths_down = 2;
    k->stag_mg_nsmooths_up = 2;
    k->stag_mg_nsmooths_bottom = 8;
    k->stag_mg_max_bottom_nlevels = 10;
    k->stag_mg_omega = 1.0;
    k->stag_mg_smoother = 1;
    k->stag_mg_rel_tol = 1e-9;
    k->gmres_rel_tol = 1e-9;
    k->gmres_abs_tol = 0.0;
    k->gmres_verbose = 1;
    k->gmres_max_outer = 20;
    k->gmres_max_inner = 5;
    k->gmres_max_iter = 100;
    k->gmres_min_iter = 1;
    k->visc_type = 1;
    k->method = LMM_METHOD_GMRES;
    k->precision = LMM_PRECISION_FP64;
    k->learned_stage = 0;
}

// one problem (batch 1, batched false) or a batch handle of `batch` 2D instances
static int create_impl(const lmm_grid* g, const lmm_knobs* k, int device, int batch, bool batched, lmm_handle** out) {
    if (!out) return LMM_ERR_INVALID;
    *out = nullptr;
    g_last_error.clear();
    int rc = validate(g, k);
    if (rc != LMM_OK) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        g_last_error = "no CUDA device";
        return LMM_ERR_NO_DEVICE;
    }
    lmm_handle* h = new lmm_handle();
    try {
        h->device = device;
        LMM_CK(cudaSetDevice(device));
        h->grid = *g;
        h->knobs = *k;
        h->dm = g->dm;
        h->D0.dm = g->dm;
        h->D0.nx = g->n[0];
        h->D0.ny = g->n[1];
        h->batch = batch;
        h->batched = batched;
        h->D0.nz = (g->dm == 3) ? g->n[2] : batch;
        set_walls(h->D0, *g);
        h->n = (int64_t)h->D0.nx * h->D0.ny * h->D0.nz;
        h->nlev = compute_nlevs(g->n, g->dm, k->stag_mg_minwidth);
        const int ap = std::abs(k->precon_type);
        h->nlev_p = compute_nlevs(g->n, g->dm, k->mg_minwidth);
        (void)ap;
        h->m = k->gmres_max_inner;
        LMM_CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        LMM_CK(cudaEventCreate(&h->ev0));
        LMM_CK(cudaEventCreate(&h->ev1));
        if (k->host_wait == 1) LMM_CK(cudaEventCreateWithFlags(&h->wait_ev, cudaEventBlockingSync | cudaEventDisableTiming));
        LMM_CK(cudaEventCreateWithFlags(&h->col_ev, cudaEventDisableTiming | (k->host_wait == 1 ? cudaEventBlockingSync : 0)));
        h->arena_bytes = plan_bytes(*g, *k, h->nlev, h->nlev_p, batch, batched);
        LMM_CK(cudaMalloc(&h->arena, h->arena_bytes));
        bc_add(h->arena, h->arena_bytes);
        // zeroed on the handle's own (non-blocking) stream: a cudaMemset on
        // the legacy stream may still run when later copies on h->stream
        // (the batch pointer tables) have landed, and would wipe them
        LMM_CK(cudaMemsetAsync(h->arena, 0, h->arena_bytes, h->stream));
        build_levels<double>(h);
        if (k->precision == LMM_PRECISION_FP32) {
            build_levels<float>(h);
            if (k->l2_persist > 0 && !h->D0.wall) set_l2_window(h);
        }
        const int dm = h->dm;
        for (int d = 0; d < dm; ++d) {
            h->alpha_fc[d] = h->alloc<double>(h->n);
            h->alphainv[d] = h->alloc<double>(h->n);
            h->alphainv32[d] = h->alloc<float>(h->n);
        }
        for (int q = 0; q <= h->m; ++q) h->V.push_back(make_svec(h));
        if (k->method == LMM_METHOD_FGMRES) {
            for (int q = 0; q < h->m; ++q) {
                if (k->precision == LMM_PRECISION_FP32)
                    h->Z32.push_back(h->alloc<float>((int64_t)(dm + 1) * h->n));
                else
                    h->Z64.push_back(make_svec(h));
            }
        }
        h->b = make_svec(h);
        h->x = make_svec(h);
        h->r = make_svec(h);
        h->w = make_svec(h);
        h->tmp = make_svec(h);
        h->zt = make_svec(h);
        h->mac64 = h->alloc<double>(h->n);
        h->src64 = h->alloc<double>(h->n);
        h->xptmp64 = h->alloc<double>(h->n);
        for (int d = 0; d < dm; ++d) h->butmp64[d] = h->alloc<double>(h->n);
        h->mac32 = h->alloc<float>(h->n);
        h->src32 = h->alloc<float>(h->n);
        h->xptmp32 = h->alloc<float>(h->n);
        if (k->visc_schur_approx == 1)
            for (int q = 0; q < 8; ++q) {
                h->bf64[q] = h->alloc<double>(h->n);
                h->bf32[q] = h->alloc<float>(h->n);
            }
        for (int d = 0; d < dm; ++d) h->butmp32[d] = h->alloc<float>(h->n);
        h->pin32 = h->alloc<float>((int64_t)(dm + 1) * h->n);
        h->pout32 = h->alloc<float>((int64_t)(dm + 1) * h->n);
        // a batch reduces each instance with one problem's block count
        h->red_blocks = reduce_blocks(batched ? (int64_t)g->n[0] * g->n[1] : h->n);
        h->partials = h->alloc<double>(partials_count(*g, batch));
        h->counter = h->alloc<unsigned>(std::max(64, batch));
        h->dev_err = h->alloc<int>(64);
        h->scal = h->alloc<double>(8 * lmm_handle::kSlots);
        int64_t st = 1;
        for (int d = 0; d < dm; ++d) st *= (g->n[d] + 1 + 8);
        h->stage_elems = st;
        h->stage = h->alloc<double>(st);
        LMM_CK(cudaMallocHost(&h->hscal, 8 * sizeof(double) * lmm_handle::kSlots));
        LMM_CK(cudaMallocHost(&h->hmisc, 64 * sizeof(double)));
        if (batched) {
            h->bslots = h->alloc<double>((int64_t)lmm_handle::kBSlots * batch * 8);
            h->ys = h->alloc<double>((int64_t)(h->m + 1) * batch);
            h->ztab = h->alloc<void*>(h->m + 1);
            h->gtab = h->alloc<const double*>((int64_t)lmm_handle::kGatherFields * batch);
            LMM_CK(cudaMallocHost(&h->bhost, sizeof(double) * lmm_handle::kBSlots * batch * 8));
            LMM_CK(cudaMallocHost(&h->ys_host, sizeof(double) * (h->m + 1) * batch));
            LMM_CK(cudaMallocHost(&h->gtab_host, sizeof(const double*) * lmm_handle::kGatherFields * batch));
            // the Z basis table never changes
            std::vector<void*> zt(h->m + 1, nullptr);
            for (int q = 0; q < h->m; ++q)
                zt[q] = (k->precision == LMM_PRECISION_FP32) ? (void*)h->Z32[q] : (void*)h->Z64[q].base;
            LMM_CK(cudaMemcpyAsync(h->ztab, zt.data(), sizeof(void*) * (h->m + 1), cudaMemcpyHostToDevice, h->stream));
        }
        if (k->autotune >= 0 && k->stag_mg_smoother != 0) {
            if (k->precision == LMM_PRECISION_FP32)
                autotune_levels<float>(h, h->L32);
            else
                autotune_levels<double>(h, h->L64);
        }
        LMM_CK(host_wait(h));
    } catch (const LmmError& e) {
        force_shape(Shape{});
        lmm_stokes_destroy(h);
        return e.code;
    }
    *out = h;
    return LMM_OK;
}

int lmm_stokes_create(const lmm_grid* g, const lmm_knobs* k, int device, lmm_handle** out) {
    return create_impl(g, k, device, 1, false, out);
}

int lmm_stokes_create_batch(const lmm_grid* g, const lmm_knobs* k, int batch, int device, lmm_handle** out) {
    if (!out) return LMM_ERR_INVALID;
    *out = nullptr;
    g_last_error.clear();
    if (!g || !k || batch < 1 || batch > 4096) return LMM_ERR_INVALID;
    if (g->dm != 2 || k->method != LMM_METHOD_FGMRES || k->visc_type >= 0 || k->learned_stage != 0 || k->visc_schur_approx != 0 ||
        k->stag_mg_max_vcycles > 1 || k->scale_factor != 1.0 || k->gmres_max_inner > lmm_handle::kBSlots - 3) {
        g_last_error =
            "batches: 2D, FGMRES, visc_type < 0, one V-cycle per application, scale_factor 1, gmres_max_inner <= 45, no BFBt or "
            "learned stage";
        return LMM_ERR_INVALID;
    }
    if ((int64_t)g->n[0] * g->n[1] * batch > (int64_t)INT32_MAX / 4) {
        g_last_error = "batches: at most 2^29 cells per batch";
        return LMM_ERR_INVALID;
    }
    return create_impl(g, k, device, batch, true, out);
}

int lmm_stokes_update_knobs(lmm_handle* h, const lmm_knobs* k) {
    if (!h || !k) return LMM_ERR_INVALID;
    g_last_error.clear();
    const lmm_knobs& a = h->knobs;
#define SAME(f) (a.f == k->f)
    const bool same = SAME(precon_type) && SAME(visc_schur_approx) && SAME(p_norm_weight) && SAME(scale_factor) &&
                      SAME(mg_max_vcycles) && SAME(mg_minwidth) && SAME(mg_bottom_solver) && SAME(mg_nsmooths_down) &&
                      SAME(mg_nsmooths_up) && SAME(mg_nsmooths_bottom) && SAME(mg_max_bottom_nlevels) &&
                      SAME(stag_mg_max_vcycles) && SAME(stag_mg_minwidth) && SAME(stag_mg_bottom_solver) &&
                      SAME(stag_mg_nsmooths_down) && SAME(stag_mg_nsmooths_up) && SAME(stag_mg_nsmooths_bottom) &&
                      SAME(stag_mg_max_bottom_nlevels) && SAME(stag_mg_omega) && SAME(stag_mg_smoother) &&
                      SAME(gmres_max_inner) && SAME(visc_type) && SAME(method) && SAME(precision) &&
                      SAME(learned_stage) && SAME(tail_cells) && SAME(tail_smem_kb) && SAME(use_graphs) &&
                      SAME(smoother_fusion) && SAME(l2_persist) && SAME(orthogonalization) && SAME(host_wait) &&
                      SAME(smoother_tma) && SAME(smoother_tma_slabs) && SAME(smoother_tma_cells) && SAME(smoother_order) &&
                      SAME(autotune) && SAME(residual_fusion) && SAME(uniform_alpha) && SAME(smoother_fusion_cells);
#undef SAME
    if (!same) {
        g_last_error = "lmm_stokes_update_knobs changes only the stopping rules; create a new handle for the rest";
        return LMM_ERR_INVALID;
    }
    if (!(k->gmres_rel_tol >= 0.0) || !(k->gmres_abs_tol >= 0.0) || k->gmres_max_iter < 0 || k->gmres_max_outer < 0 ||
        k->gmres_min_iter < 0 || !(k->stag_mg_rel_tol >= 0.0) || !(k->mg_rel_tol >= 0.0))
        return LMM_ERR_INVALID;
    h->knobs.gmres_rel_tol = k->gmres_rel_tol;
    h->knobs.gmres_abs_tol = k->gmres_abs_tol;
    h->knobs.gmres_max_outer = k->gmres_max_outer;
    h->knobs.gmres_max_iter = k->gmres_max_iter;
    h->knobs.gmres_min_iter = k->gmres_min_iter;
    h->knobs.stag_mg_rel_tol = k->stag_mg_rel_tol;
    h->knobs.mg_rel_tol = k->mg_rel_tol;
    h->knobs.gmres_verbose = k->gmres_verbose;
    h->knobs.mg_verbose = k->mg_verbose;
    h->knobs.cg_verbose = k->cg_verbose;
    h->knobs.stag_mg_verbosity = k->stag_mg_verbosity;
    return LMM_OK;
}

int lmm_stokes_destroy(lmm_handle* h) {
    if (!h) return LMM_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto& kv : h->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    bc_remove(h->arena);
    bc_remove(h->lrn_block);
    if (h->arena) cudaFree(h->arena);
    if (h->lrn_block) cudaFree(h->lrn_block);
    if (h->hscal) cudaFreeHost(h->hscal);
    if (h->hmisc) cudaFreeHost(h->hmisc);
    if (h->bhost) cudaFreeHost(h->bhost);
    if (h->ys_host) cudaFreeHost(h->ys_host);
    if (h->gtab_host) cudaFreeHost(h->gtab_host);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->wait_ev) cudaEventDestroy(h->wait_ev);
    if (h->col_ev) cudaEventDestroy(h->col_ev);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return LMM_OK;
}

void* lmm_stream(lmm_handle* h) { return h ? (void*)h->stream : nullptr; }

int lmm_op_num_levels(lmm_handle* h) { return h ? h->nlev : -1; }

}  // extern "C"

// ------------------------------------------------------------ solve entry points
namespace {

// device inputs (compact) -> handle buffers, the solve, solution -> x (device)
int solve_core(lmm_handle* h, const lmm_fields_in* in, const double* x0_u[3], const double* x0_p, double* theta_alpha,
               double* norm_pre_rhs, lmm_stats* st) {
    const lmm_knobs& K = h->knobs;
    const int dm = h->dm;
    const int64_t n = h->n;
    double theta = *theta_alpha;
    const double sf = K.scale_factor;
    DebugScope dbg(h);  // LMM_DEBUG: launch checks on this solve's stream
    // scale_factor (gmres.f90:106-122): applied to device copies only
    if (sf != 1.0) theta = theta * sf;
    LevelDev<double>& L0 = h->L64[0];
    // b = (scaled) rhs, x = (scaled) initial guess
    for (int d = 0; d < dm; ++d) {
        if (sf != 1.0)
            launch_scale_copy<double>(in->b_u[d], h->b.c(d), sf, n, h->stream);
        else
            LMM_CK(cudaMemcpyAsync(h->b.c(d), in->b_u[d], n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        LMM_CK(cudaMemcpyAsync(h->x.c(d), x0_u[d], n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    }
    LMM_CK(cudaMemcpyAsync(h->b.p(), in->b_p, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    if (sf != 1.0)
        launch_scale_copy<double>(x0_p, h->x.p(), sf, n, h->stream);
    else
        LMM_CK(cudaMemcpyAsync(h->x.p(), x0_p, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    check_launch();
    if (h->D0.wall) {
        // wall-normal velocities on the walls are not unknowns: zero in x
        // (apply_matrix's physbc_domainvel) and in b (the reference's
        // preconditioner zeroes them in every correction)
        double* bu[3] = {h->b.c(0), h->b.c(1), dm == 3 ? h->b.c(2) : h->b.c(0)};
        double* xu[3] = {h->x.c(0), h->x.c(1), dm == 3 ? h->x.c(2) : h->x.c(0)};
        launch_zero_wall_faces(h->D0, bu, h->stream);
        check_launch();
        launch_zero_wall_faces(h->D0, xu, h->stream);
        check_launch();
    }
    // coefficients (beta, beta_ed, gamma scaled by scale_factor)
    const double* beta = in->beta;
    const double* bed[3] = {in->beta_ed[0], in->beta_ed[1], in->beta_ed[2]};
    const double* gamma = in->gamma;
    if (sf != 1.0) {
        launch_scale_copy<double>(in->beta, L0.beta, sf, n, h->stream);
        beta = L0.beta;
        for (int e = 0; e < (dm == 2 ? 1 : 3); ++e) {
            launch_scale_copy<double>(in->beta_ed[e], L0.bed[e], sf, edge_count(L0.D, e), h->stream);
            bed[e] = L0.bed[e];
        }
        if (gamma) {
            launch_scale_copy<double>(in->gamma, L0.gamma, sf, n, h->stream);
            gamma = L0.gamma;
        }
        check_launch();
    }
    const double* al[3] = {in->alpha_fc[0], in->alpha_fc[1], in->alpha_fc[2]};
    load_coeffs(h, al, beta, bed, gamma, theta);
    h->pvcycles = 0;
    int rc = (K.method == LMM_METHOD_FGMRES) ? run_fgmres(h, norm_pre_rhs, st) : run_gmres(h, theta_alpha, norm_pre_rhs, st);
    if (h->tma_smoother && rc != LMM_ERR_WATCHDOG) {
        // a bounded wait of the TMA smoother that gave up makes the solve an error
        int* herr = reinterpret_cast<int*>(h->hscal + 8 * (lmm_handle::kSlots - 1));
        LMM_CK(cudaMemcpyAsync(herr, h->dev_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        LMM_CK(host_wait(h));
        if (*herr != 0) {
            LMM_CK(cudaMemsetAsync(h->dev_err, 0, sizeof(int), h->stream));
            g_last_error = "a bounded wait of the TMA Gauss-Seidel smoother gave up";
            return LMM_ERR_WATCHDOG;
        }
    }
    if (sf != 1.0) {
        theta = theta / sf;
        launch_scale_copy<double>(h->x.p(), h->x.p(), 1.0 / sf, n, h->stream);
        check_launch();
    }
    *theta_alpha = theta;
    if (st) st->pressure_vcycles = h->pvcycles;
    const int bc = bc_status();
    return bc != LMM_OK ? bc : rc;
}

}  // namespace

extern "C" int lmm_stokes_solve_device(lmm_handle* h, const lmm_fields_in* in, lmm_fields_out* out, double* theta_alpha,
                                       double* norm_pre_rhs, lmm_stats* st) {
    if (!h || h->batched || !in || !out || !theta_alpha) return LMM_ERR_INVALID;
    if (in->layout != LMM_LAYOUT_COMPACT || out->layout != LMM_LAYOUT_COMPACT) return LMM_ERR_INVALID;
    g_last_error.clear();
    NvtxRange nvtx_("lmm_stokes_solve_device");
    try {
        LMM_CK(cudaSetDevice(h->device));
        if (st) std::memset(st, 0, sizeof(*st));
        LMM_CK(cudaEventRecord(h->ev0, h->stream));
        const double* x0u[3] = {out->x_u[0], out->x_u[1], out->x_u[2]};
        int rc = solve_core(h, in, x0u, out->x_p, theta_alpha, norm_pre_rhs, st);
        if (rc >= 0 || rc == LMM_ERR_BREAKDOWN || rc == LMM_ERR_NONFINITE) {
            for (int d = 0; d < h->dm; ++d)
                LMM_CK(cudaMemcpyAsync(out->x_u[d], h->x.c(d), h->n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
            LMM_CK(cudaMemcpyAsync(out->x_p, h->x.p(), h->n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        }
        LMM_CK(cudaEventRecord(h->ev1, h->stream));
        LMM_CK(host_wait(h));
        if (st) {
            float ms = 0;
            cudaEventElapsedTime(&ms, h->ev0, h->ev1);
            st->solve_ms = ms;
        }
        return rc;
    } catch (const LmmError& e) {
        return e.code;
    }
}

extern "C" int lmm_stokes_solve(lmm_handle* h, const lmm_fields_in* in, lmm_fields_out* out, double* theta_alpha,
                                double* norm_pre_rhs, lmm_stats* st) {
    if (!h || h->batched || !in || !out || !theta_alpha) return LMM_ERR_INVALID;
    g_last_error.clear();
    NvtxRange nvtx_("lmm_stokes_solve");
    const int dm = h->dm;
    const int64_t n = h->n;
    const Dims& D = h->D0;
    try {
        LMM_CK(cudaSetDevice(h->device));
        if (st) std::memset(st, 0, sizeof(*st));
        auto t0 = std::chrono::steady_clock::now();
        // host -> device: inputs land in the level-0 / Krylov buffers
        LevelDev<double>& L0 = h->L64[0];
        // staging targets: b -> r, x0 -> w, coefficients -> their level-0 homes
        // cext: compact extents (an edge array of a grid with walls keeps
        // n+1 nodes along a nodal wall-bounded direction)
        auto upload = [&](const double* src, double* dst, int layout, int ng, const int nodal[3], const int* cext = nullptr) {
            const int64_t cn = cext ? (int64_t)cext[0] * cext[1] * (dm == 3 ? cext[2] : 1) : n;
            if (layout == LMM_LAYOUT_COMPACT) {
                LMM_CK(cudaMemcpyAsync(dst, src, cn * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            } else {
                int64_t sz = boxlib_size(D, nodal, ng);
                if (sz > h->stage_elems || ng > 4) {
                    g_last_error = "ghost width above 4 is not supported";
                    throw LmmError(LMM_ERR_INVALID);
                }
                LMM_CK(cudaMemcpyAsync(h->stage, src, sz * sizeof(double), cudaMemcpyHostToDevice, h->stream));
                if (cext)
                    launch_gather_boxlib_ext(D, cext, nodal, ng, h->stage, dst, h->stream);
                else
                    launch_gather_boxlib(D, nodal, ng, h->stage, dst, h->stream);
                check_launch();
            }
        };
        int nod_face[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        int nod_cell[3] = {0, 0, 0};
        int nod_edge[3][3] = {{1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
        if (dm == 2) nod_edge[0][2] = 0;
        const int lay = in->layout;
        for (int d = 0; d < dm; ++d) {
            upload(in->b_u[d], h->r.c(d), lay, in->ng_b_u, nod_face[d]);
            upload(in->alpha_fc[d], h->alpha_fc[d], lay, in->ng_alpha, nod_face[d]);
            upload(out->x_u[d], h->w.c(d), out->layout, out->ng_x_u, nod_face[d]);
        }
        upload(in->b_p, h->r.p(), lay, in->ng_b_p, nod_cell);
        upload(out->x_p, h->w.p(), out->layout, out->ng_x_p, nod_cell);
        upload(in->beta, L0.beta, lay, in->ng_beta, nod_cell);
        for (int e = 0; e < (dm == 2 ? 1 : 3); ++e) {
            const int cext[3] = {edge_ext(D, e, 0), edge_ext(D, e, 1), edge_ext(D, e, 2)};
            upload(in->beta_ed[e], L0.bed[e], lay, in->ng_beta_ed, nod_edge[e], D.wall ? cext : nullptr);
        }
        // gamma enters only the visc_type +-3 operator (stag_applyop.f90): not
        // copied otherwise (solve_core then zeroes the device copy)
        const bool use_gamma = in->gamma && std::abs(h->knobs.visc_type) == 3;
        if (use_gamma) upload(in->gamma, L0.gamma, lay, in->ng_gamma, nod_cell);
        LMM_CK(host_wait(h));
        auto t1 = std::chrono::steady_clock::now();
        lmm_fields_in din{};
        for (int d = 0; d < 3; ++d) {
            din.b_u[d] = (d < dm) ? h->r.c(d) : nullptr;
            din.alpha_fc[d] = (d < dm) ? h->alpha_fc[d] : nullptr;
            din.beta_ed[d] = L0.bed[d];
        }
        din.b_p = h->r.p();
        din.beta = L0.beta;
        din.gamma = use_gamma ? L0.gamma : nullptr;
        din.layout = LMM_LAYOUT_COMPACT;
        const double* x0u[3] = {h->w.c(0), h->w.c(1), dm == 3 ? h->w.c(2) : nullptr};
        LMM_CK(cudaEventRecord(h->ev0, h->stream));
        int rc = solve_core(h, &din, x0u, h->w.p(), theta_alpha, norm_pre_rhs, st);
        LMM_CK(cudaEventRecord(h->ev1, h->stream));
        // device -> host
        if (rc >= 0 || rc == LMM_ERR_BREAKDOWN || rc == LMM_ERR_NONFINITE) {
            auto download = [&](const double* src, double* dst, int layout, int ng, const int nodal[3], int kind) {
                if (layout == LMM_LAYOUT_COMPACT) {
                    LMM_CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
                } else {
                    int64_t sz = boxlib_size(D, nodal, ng);
                    if (sz > h->stage_elems || ng > 4) throw LmmError(LMM_ERR_INVALID);
                    if (D.wall)
                        launch_scatter_boxlib_w(D, kind, nodal, ng, src, h->stage, h->stream);
                    else
                        launch_scatter_boxlib(D, nodal, ng, src, h->stage, h->stream);
                    check_launch();
                    LMM_CK(cudaMemcpyAsync(dst, h->stage, sz * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
                    LMM_CK(host_wait(h));
                }
            };
            for (int d = 0; d < dm; ++d) download(h->x.c(d), out->x_u[d], out->layout, out->ng_x_u, nod_face[d], d);
            download(h->x.p(), out->x_p, out->layout, out->ng_x_p, nod_cell, -1);
        }
        LMM_CK(host_wait(h));
        auto t2 = std::chrono::steady_clock::now();
        if (st) {
            float ms = 0;
            cudaEventElapsedTime(&ms, h->ev0, h->ev1);
            st->solve_ms = ms;
            st->h2d_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
            st->d2h_ms = std::chrono::duration<double, std::milli>(t2 - t1).count() - ms;
        }
        return rc;
    } catch (const LmmError& e) {
        return e.code;
    }
}

// ------------------------------------------------------------ batches of 2D problems
extern "C" int lmm_stokes_solve_batch(lmm_handle* h, lmm_ensemble_item* items, int count) {
    if (!h || !h->batched || !items || count < 1 || count > h->batch) return LMM_ERR_INVALID;
    g_last_error.clear();
    const int B = h->batch, ni = h->D0.nx * h->D0.ny;
    const double theta = items[0].theta_alpha;
    const bool has_gamma = items[0].gamma != nullptr;
    for (int q = 0; q < count; ++q) {
        const lmm_ensemble_item& it = items[q];
        if (it.n[0] != h->grid.n[0] || it.n[1] != h->grid.n[1] || it.dx != h->grid.dx || it.theta_alpha != theta) {
            g_last_error = "a batch holds problems of one grid, spacing and theta_alpha";
            return LMM_ERR_INVALID;
        }
        if (!it.b_u[0] || !it.b_u[1] || !it.b_p || !it.alpha_fc[0] || !it.alpha_fc[1] || !it.beta || !it.beta_ed[0] ||
            !it.x_u[0] || !it.x_u[1] || !it.x_p || (it.gamma != nullptr) != has_gamma) {
            g_last_error = "a batch item lacks an array (gamma: all or none)";
            return LMM_ERR_INVALID;
        }
    }
    try {
        LMM_CK(cudaSetDevice(h->device));
        DebugScope dbg(h);
        LevelDev<double>& L0 = h->L64[0];
        std::vector<lmm_stats> st(count);
        std::vector<int> status(count, LMM_OK);
        for (auto& x : st) std::memset(&x, 0, sizeof(x));
        LMM_CK(cudaEventRecord(h->ev0, h->stream));
        // gather: table entry f*B + b is field f of instance b; instances
        // past count are zero problems (rhs and initial guess zeroed below)
        // on the first instance's coefficients
        double* dst[lmm_handle::kGatherFields] = {h->b.c(0), h->b.c(1), h->b.p(),   h->alpha_fc[0], h->alpha_fc[1], L0.beta,
                                                  L0.bed[0], L0.gamma,  h->x.c(0), h->x.c(1),      h->x.p()};
        auto field = [&](const lmm_ensemble_item& it, int f) -> const double* {
            switch (f) {
            case 0: return it.b_u[0];
            case 1: return it.b_u[1];
            case 2: return it.b_p;
            case 3: return it.alpha_fc[0];
            case 4: return it.alpha_fc[1];
            case 5: return it.beta;
            case 6: return it.beta_ed[0];
            case 7: return it.gamma;
            case 8: return it.x_u[0];
            case 9: return it.x_u[1];
            default: return it.x_p;
            }
        };
        // the pinned table may still be read by the previous call's copy
        LMM_CK(host_wait(h));
        for (int f = 0; f < lmm_handle::kGatherFields; ++f)
            for (int b = 0; b < B; ++b) h->gtab_host[(int64_t)f * B + b] = field(items[b < count ? b : 0], f);
        LMM_CK(cudaMemcpyAsync(h->gtab, h->gtab_host, sizeof(const double*) * lmm_handle::kGatherFields * B, cudaMemcpyHostToDevice,
                               h->stream));
        for (int f = 0; f < lmm_handle::kGatherFields; ++f) {
            if (f == 7 && !has_gamma) {
                LMM_CK(cudaMemsetAsync(L0.gamma, 0, sizeof(double) * h->n, h->stream));
                continue;
            }
            // an edge array (field 6) keeps n+1 nodes along a nodal wall-bounded direction
            const int nf = (f == 6) ? edge_ext(h->D0, 0, 0) * edge_ext(h->D0, 0, 1) : ni;
            launch_gather_ptrs(h->gtab + (int64_t)f * B, dst[f], nf, B, h->stream);
            check_launch();
        }
        if (count < B) {
            const size_t rest = sizeof(double) * (size_t)(B - count) * ni;
            for (int c = 0; c < 3; ++c) {
                LMM_CK(cudaMemsetAsync(h->b.c(c) + (int64_t)count * ni, 0, rest, h->stream));
                LMM_CK(cudaMemsetAsync(h->x.c(c) + (int64_t)count * ni, 0, rest, h->stream));
            }
        }
        if (h->D0.wall) {
            // wall-normal velocities on the walls are not unknowns (as solve_core)
            double* bu[3] = {h->b.c(0), h->b.c(1), h->b.c(0)};
            double* xu[3] = {h->x.c(0), h->x.c(1), h->x.c(0)};
            launch_zero_wall_faces(h->D0, bu, h->stream);
            check_launch();
            launch_zero_wall_faces(h->D0, xu, h->stream);
            check_launch();
        }
        const double* al[3] = {h->alpha_fc[0], h->alpha_fc[1], nullptr};
        const double* bed[3] = {L0.bed[0], nullptr, nullptr};
        load_coeffs(h, al, L0.beta, bed, L0.gamma, theta);
        h->pvcycles = 0;
        const int rc = run_fgmres_batch(h, count, st.data(), status.data());
        // scatter x_u, x_p to the instances' arrays (table entries (f-8)*B + b)
        LMM_CK(host_wait(h));
        for (int f = 8; f < lmm_handle::kGatherFields; ++f)
            for (int b = 0; b < count; ++b) h->gtab_host[(int64_t)(f - 8) * B + b] = field(items[b], f);
        LMM_CK(cudaMemcpyAsync(h->gtab, h->gtab_host, sizeof(const double*) * 3 * B, cudaMemcpyHostToDevice, h->stream));
        for (int f = 8; f < lmm_handle::kGatherFields; ++f) {
            launch_scatter_ptrs(dst[f], const_cast<double* const*>(h->gtab + (int64_t)(f - 8) * B), ni, count, h->stream);
            check_launch();
        }
        LMM_CK(cudaEventRecord(h->ev1, h->stream));
        LMM_CK(host_wait(h));
        float ms = 0;
        cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        for (int q = 0; q < count; ++q) {
            st[q].solve_ms = ms;
            items[q].stats = st[q];
            items[q].status = status[q];
        }
        const int bc = bc_status();
        return bc != LMM_OK ? bc : rc;
    } catch (const LmmError& e) {
        return e.code;
    }
}

// ------------------------------------------------------------ operator-level entry points
extern "C" int64_t lmm_kernel_launches(void) { return lmm::launches_total(); }

extern "C" int lmm_time_op(lmm_handle* h, int which, int reps, double* ms_per_rep) {
    if (!h || !h->coeffs_loaded || reps < 1 || !ms_per_rep) return LMM_ERR_INVALID;
    if ((which == 1 || which == 5) && h->knobs.precision != LMM_PRECISION_FP32) return LMM_ERR_INVALID;
    NvtxRange nvtx_("lmm_time_op");  // a profiler can select these launches (not the autotuner's)
    try {
        LevelDev<double>& L = h->L64[0];
        auto once = [&]() {
            switch (which) {
            // sweeps are timed in pairs, so the fused smoother's buffers end
            // where they started (no copy-back inside the timed region)
            case 0: smooth<double>(h, L, 2); break;
            case 1: smooth<float>(h, h->L32[0], 2); break;
            case 2:
                launch_applyop<double>(L, h->knobs.visc_type, L.phi, L.tmp, h->stream, 0);
                check_launch();
                break;
            case 3:
                launch_apply_matrix(L, h->knobs.visc_type, h->x, h->tmp, h->stream);
                check_launch();
                break;
            case 4: vcycle<double>(h, h->L64); break;
            case 5: vcycle<float>(h, h->L32); break;
            case 6: macproject<double>(h); break;
            case 7:
                // one restart cycle's Gram-Schmidt passes (columns 1..m)
                for (int i = 1; i <= h->knobs.gmres_max_inner; ++i) cgs_column(h, i);
                break;
            case 8:
                if (h->knobs.precision == LMM_PRECISION_FP32)
                    launch_div_by_f32(h->w.base, h->V[1].base, h->pin32, h->slot(2) + 5, h->w.size(), h->stream);
                else
                    launch_div_by(h->w.base, h->V[1].base, h->slot(2) + 5, h->w.size(), h->stream);
                check_launch();
                break;
            default: throw LmmError(LMM_ERR_INVALID);
            }
        };
        once();  // warm
        LMM_CK(cudaEventRecord(h->ev0, h->stream));
        for (int r = 0; r < reps; ++r) once();
        LMM_CK(cudaEventRecord(h->ev1, h->stream));
        LMM_CK(cudaEventSynchronize(h->ev1));
        float ms = 0;
        LMM_CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
        *ms_per_rep = (double)ms / reps / ((which == 0 || which == 1) ? 2 : 1);
        return LMM_OK;
    } catch (const LmmError& e) {
        return e.code;
    }
}

extern "C" int lmm_op_load_coeffs(lmm_handle* h, const lmm_fields_in* c, double theta_alpha) {
    if (!h || h->batched || !c) return LMM_ERR_INVALID;
    try {
        const double* al[3] = {c->alpha_fc[0], c->alpha_fc[1], c->alpha_fc[2]};
        const double* bed[3] = {c->beta_ed[0], c->beta_ed[1], c->beta_ed[2]};
        load_coeffs(h, al, c->beta, bed, c->gamma, theta_alpha);
        LMM_CK(host_wait(h));
        return bc_status();
    } catch (const LmmError& e) {
        return e.code;
    }
}

extern "C" int lmm_op_stag_applyop(lmm_handle* h, const double* const phi[3], double* const Lphi[3], int color) {
    if (!h || h->batched || !h->coeffs_loaded) return LMM_ERR_INVALID;
    try {
        if (color < 0 || color > 2 * h->dm) return LMM_ERR_INVALID;
        const bool d3 = h->dm == 3;
        lmm::BcScope scope({phi[0], phi[1], d3 ? phi[2] : nullptr, Lphi[0], Lphi[1], d3 ? Lphi[2] : nullptr},
                           (size_t)h->L64[0].n * sizeof(double));
        launch_applyop<double>(h->L64[0], h->knobs.visc_type, phi, Lphi, h->stream, color);
        check_launch();
        LMM_CK(host_wait(h));
        return bc_status();
    } catch (const LmmError& e) {
        return e.code;
    }
}

extern "C" int lmm_op_apply_matrix(lmm_handle* h, const double* const x_u[3], const double* x_p, double* const b_u[3],
                                   double* b_p) {
    if (!h || h->batched || !h->coeffs_loaded) return LMM_ERR_INVALID;
    try {
        const int dm = h->dm;
        const int64_t n = h->n;
        for (int d = 0; d < dm; ++d)
            LMM_CK(cudaMemcpyAsync(h->r.c(d), x_u[d], n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        LMM_CK(cudaMemcpyAsync(h->r.p(), x_p, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        launch_apply_matrix(h->L64[0], h->knobs.visc_type, h->r, h->tmp, h->stream);
        check_launch();
        for (int d = 0; d < dm; ++d)
            LMM_CK(cudaMemcpyAsync(b_u[d], h->tmp.c(d), n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        LMM_CK(cudaMemcpyAsync(b_p, h->tmp.p(), n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        LMM_CK(host_wait(h));
        return bc_status();
    } catch (const LmmError& e) {
        return e.code;
    }
}

extern "C" int lmm_op_apply_precon(lmm_handle* h, const double* const b_u[3], const double* b_p, double* const x_u[3],
                                   double* x_p) {
    if (!h || h->batched || !h->coeffs_loaded) return LMM_ERR_INVALID;
    try {
        const int dm = h->dm;
        const int64_t n = h->n;
        for (int d = 0; d < dm; ++d)
            LMM_CK(cudaMemcpyAsync(h->r.c(d), b_u[d], n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        LMM_CK(cudaMemcpyAsync(h->r.p(), b_p, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        if (h->knobs.precision == LMM_PRECISION_FP32) {
            precon32(h, h->r, h->pout32);
            launch_convert<float, double>(h->pout32, h->w.base, h->w.size(), h->stream);
            check_launch();
        } else {
            precon64(h, h->r, h->w);
        }
        for (int d = 0; d < dm; ++d)
            LMM_CK(cudaMemcpyAsync(x_u[d], h->w.c(d), n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        LMM_CK(cudaMemcpyAsync(x_p, h->w.p(), n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        LMM_CK(host_wait(h));
        return bc_status();
    } catch (const LmmError& e) {
        return e.code;
    }
}

extern "C" int lmm_op_stag_mg_solver(lmm_handle* h, const double* const rhs[3], double* const phi[3]) {
    if (!h || h->batched || !h->coeffs_loaded) return LMM_ERR_INVALID;
    try {
        LevelDev<double>& L0 = h->L64[0];
        for (int d = 0; d < h->dm; ++d) {
            LMM_CK(cudaMemcpyAsync(L0.rhs[d], rhs[d], h->n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
            LMM_CK(cudaMemcpyAsync(L0.phi[d], phi[d], h->n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        }
        stag_mg_solver<double>(h);
        for (int d = 0; d < h->dm; ++d)
            LMM_CK(cudaMemcpyAsync(phi[d], L0.phi[d], h->n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        LMM_CK(host_wait(h));
        return bc_status();
    } catch (const LmmError& e) {
        return e.code;
    }
}

extern "C" int lmm_op_smooth(lmm_handle* h, int lev, const double* const rhs[3], double* const phi[3], int color) {
    if (!h || h->batched || !h->coeffs_loaded || lev < 0 || lev >= h->nlev) return LMM_ERR_INVALID;
    try {
        LevelDev<double>& L = h->L64[lev];
        for (int d = 0; d < h->dm; ++d) {
            LMM_CK(cudaMemcpyAsync(L.rhs[d], rhs[d], L.n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
            LMM_CK(cudaMemcpyAsync(L.phi[d], phi[d], L.n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        }
        if (color == 0) {
            launch_jacobi<double>(L, h->knobs.visc_type, L.rhs, L.phi, L.tmp, h->knobs.stag_mg_omega, h->stream);
            check_launch();
            for (int d = 0; d < h->dm; ++d)
                LMM_CK(cudaMemcpyAsync(phi[d], L.tmp[d], L.n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        } else {
            launch_gs_colour<double>(L, h->knobs.visc_type, color, L.rhs, L.phi, h->knobs.stag_mg_omega, h->stream);
            check_launch();
            for (int d = 0; d < h->dm; ++d)
                LMM_CK(cudaMemcpyAsync(phi[d], L.phi[d], L.n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        }
        LMM_CK(host_wait(h));
        return bc_status();
    } catch (const LmmError& e) {
        return e.code;
    }
}

extern "C" int lmm_op_residual_restrict(lmm_handle* h, int lev, const double* const rhs[3], const double* const phi[3],
                                        double* const rhs_coarse[3]) {
    if (!h || h->batched || !h->coeffs_loaded || lev < 0 || lev + 1 >= h->nlev) return LMM_ERR_INVALID;
    try {
        const bool d3 = h->dm == 3;
        lmm::BcScope fine({rhs[0], rhs[1], d3 ? rhs[2] : nullptr, phi[0], phi[1], d3 ? phi[2] : nullptr},
                          (size_t)h->L64[lev].n * sizeof(double));
        lmm::BcScope coarse({rhs_coarse[0], rhs_coarse[1], d3 ? rhs_coarse[2] : nullptr}, (size_t)h->L64[lev + 1].n * sizeof(double));
        launch_residual_restrict<double>(h->L64[lev], h->L64[lev + 1], h->knobs.visc_type, rhs, phi, rhs_coarse, h->stream,
                                         h->knobs.residual_fusion > 0 ? 1 : 0);
        check_launch();
        LMM_CK(host_wait(h));
        return bc_status();
    } catch (const LmmError& e) {
        return e.code;
    }
}

extern "C" int lmm_op_prolong_add(lmm_handle* h, int lev, const double* const phi_coarse[3], double* const phi_fine[3]) {
    if (!h || h->batched || lev < 0 || lev + 1 >= h->nlev) return LMM_ERR_INVALID;
    try {
        const bool d3 = h->dm == 3;
        lmm::BcScope fine({phi_fine[0], phi_fine[1], d3 ? phi_fine[2] : nullptr}, (size_t)h->L64[lev].n * sizeof(double));
        lmm::BcScope coarse({phi_coarse[0], phi_coarse[1], d3 ? phi_coarse[2] : nullptr}, (size_t)h->L64[lev + 1].n * sizeof(double));
        launch_prolong_add<double>(h->L64[lev], h->L64[lev + 1], phi_coarse, phi_fine, h->stream);
        check_launch();
        LMM_CK(host_wait(h));
        return bc_status();
    } catch (const LmmError& e) {
        return e.code;
    }
}

extern "C" int lmm_op_inner_prod(lmm_handle* h, const double* const a_u[3], const double* a_p, const double* const b_u[3],
                                 const double* b_p, double* out_host) {
    if (!h || h->batched) return LMM_ERR_INVALID;
    try {
        const double* a[4] = {a_u[0], a_u[1], h->dm == 3 ? a_u[2] : nullptr, a_p};
        const double* b[4] = {b_u[0], b_u[1], h->dm == 3 ? b_u[2] : nullptr, b_p};
        const size_t bytes = (size_t)h->n * sizeof(double);
        lmm::BcScope scope({a[0], a[1], a[2], a[3], b[0], b[1], b[2], b[3]}, bytes);
        stokes_reduce(h, 0, a, b, 2);
        LMM_CK(cudaMemcpyAsync(h->hscal, h->slot(2), 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        LMM_CK(host_wait(h));
        for (int c = 0; c <= h->dm; ++c) out_host[c] = h->hscal[c];
        return bc_status();
    } catch (const LmmError& e) {
        return e.code;
    }
}

extern "C" int lmm_op_sum_umac_press(lmm_handle* h, const double* const u[3], const double* p, double* out_host) {
    if (!h || h->batched) return LMM_ERR_INVALID;
    try {
        const double* a[4] = {u[0], u[1], h->dm == 3 ? u[2] : nullptr, p};
        const double* b[4] = {nullptr, nullptr, nullptr, nullptr};
        lmm::BcScope scope({a[0], a[1], a[2], a[3]}, (size_t)h->n * sizeof(double));
        stokes_reduce(h, 1, a, b, 2);
        LMM_CK(cudaMemcpyAsync(h->hscal, h->slot(2), 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        LMM_CK(host_wait(h));
        double tv = 1.0;
        for (int d = 0; d < h->dm; ++d) tv *= (double)h->grid.n[d];
        out_host[0] = h->hscal[h->dm] / tv;
        for (int d = 0; d < h->dm; ++d) out_host[1 + d] = h->hscal[d] / tv;
        return bc_status();
    } catch (const LmmError& e) {
        return e.code;
    }
}

namespace lmm {
namespace {
std::atomic<int64_t> g_launches{0};
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
cudaError_t raise_smem_limit(const void* kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> raised;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = raised[{dev, kernel}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}
int64_t launches_total() { return g_launches.load(std::memory_order_relaxed); }
int reduce_blocks(int64_t n) {
    int64_t b = (n + 2047) / 2048;  // at least 8 elements per thread
    if (b > 592) b = 592;           // 4 blocks per SM on 148 SMs
    if (b < 1) b = 1;
    return (int)b;
}
}  // namespace lmm

// ------------------------------------------------------------ learned stage entry points
extern "C" int lmm_stokes_set_net(lmm_handle* h, lmm_net* net) {
    if (!h || h->batched) return LMM_ERR_INVALID;
    try {
        if (net) {
            int nx, ny, nz, B;
            nn::net_dims(net, &nx, &ny, &nz, &B);
            if (h->D0.wall) {
                g_last_error = "the learned stage needs a periodic box";
                return LMM_ERR_INVALID;
            }
            if (h->dm != 3 || nx != h->grid.n[0] || ny != h->grid.n[1] || nz != h->grid.n[2]) {
                g_last_error = "the network's grid differs from the solver's (3D only)";
                return LMM_ERR_INVALID;
            }
            if (!h->lrn_block) {
                const int64_t len = (int64_t)(h->dm + 1) * h->n;
                // 4 work vectors, m network corrections and m more Krylov
                // vectors (a cycle with the stage holds up to 2m columns)
                const int nv = 4 + 2 * h->m;
                const size_t bytes = (size_t)nv * len * sizeof(double) + (size_t)len * sizeof(float) + 256;
                LMM_CK(cudaMalloc(&h->lrn_block, bytes));
                bc_add(h->lrn_block, bytes);
                double* p = static_cast<double*>(h->lrn_block);
                h->Zc.assign(h->m, SVec());
                const size_t v0 = h->V.size();
                h->V.resize(v0 + h->m);
                SVec* v[4] = {&h->lr1, &h->lc, &h->lAc, &h->le};
                for (int q = 0; q < nv; ++q) {
                    SVec& t = q < 4 ? *v[q] : (q < 4 + h->m ? h->Zc[q - 4] : h->V[v0 + (q - 4 - h->m)]);
                    t.base = p + (int64_t)q * len;
                    t.n = h->n;
                    t.dm = h->dm;
                }
                h->lz32 = reinterpret_cast<float*>(p + (int64_t)nv * len);
                h->luses = reinterpret_cast<int*>(h->lz32 + len);
                LMM_CK(cudaMemsetAsync(h->luses, 0, 2 * sizeof(int), h->stream));
            }
        }
        h->net = net;
        return LMM_OK;
    } catch (const LmmError& e) {
        return e.code;
    }
}

// Training pairs from the solver's own operators on the loaded coefficients:
// e0 ~ N(0,1) on every face and cell, r0 = A e0, z1 = M r0 (the configured
// preconditioner), e1 = e0 - z1, r1 = A e1; pair q gets the network input
// rows of r1 and the target rows of e1.
extern "C" int lmm_learned_make_pairs(lmm_handle* h, unsigned long long seed, int count, void* x_out, float* t_out) {
    if (!h || h->batched || !h->coeffs_loaded || !h->lrn_block || count < 1 || !x_out || !t_out) return LMM_ERR_INVALID;
    try {
        const int64_t len = (int64_t)(h->dm + 1) * h->n;
        const int S1 = lmm_handle::kLrnSlot, S3 = S1 + 2;
        for (int q = 0; q < count; ++q) {
            launch_randn(h->le.base, len, seed * 7919ull + (unsigned long long)q, h->stream);
            check_launch();
            launch_apply_matrix(h->L64[0], h->knobs.visc_type, h->le, h->lAc, h->stream);
            check_launch();
            if (h->knobs.precision == LMM_PRECISION_FP32) {
                precon32(h, h->lAc, h->lz32);
                launch_convert<float, double>(h->lz32, h->lc.base, len, h->stream);
                check_launch();
            } else {
                precon64(h, h->lAc, h->lc);
            }
            launch_lin(h->le.base, h->le.base, -1.0, h->lc.base, len, h->stream);
            check_launch();
            launch_apply_matrix(h->L64[0], h->knobs.visc_type, h->le, h->lr1, h->stream);
            check_launch();
            stokes_norm(h, h->lr1, S1);
            const double* a[4] = {h->le.c(0), h->le.c(1), h->le.c(2), h->le.p()};
            const double* b[4] = {nullptr, nullptr, nullptr, nullptr};
            stokes_reduce(h, 1, a, b, S3);
            launch_features(h->D0, h->lr1.base, h->L64[0].beta, h->slot(S1), h->grid.dx,
                            static_cast<__nv_bfloat16*>(x_out) + (int64_t)q * h->n * 8, h->stream);
            check_launch();
            launch_target(h->D0, h->le.base, h->L64[0].beta, h->slot(S1), h->slot(S3), h->grid.dx, t_out + (int64_t)q * h->n * 4, h->stream);
            check_launch();
        }
        LMM_CK(host_wait(h));
        return LMM_OK;
    } catch (const LmmError& e) {
        return e.code;
    }
}

// One fresh pair through the attached network: ratios[0] = |r1| / |r0|
// (what the preconditioner alone leaves), ratios[1] = |r1 - A c| / |r1|
// (what the network's correction leaves of that).
extern "C" int lmm_learned_eval(lmm_handle* h, unsigned long long seed, double* ratios) {
    if (!h || h->batched || !h->net || !h->coeffs_loaded || !ratios) return LMM_ERR_INVALID;
    try {
        const int64_t len = (int64_t)(h->dm + 1) * h->n;
        const int S1 = lmm_handle::kLrnSlot, S2 = S1 + 1, S3 = S1 + 2;
        launch_randn(h->le.base, len, seed * 7919ull, h->stream);
        check_launch();
        launch_apply_matrix(h->L64[0], h->knobs.visc_type, h->le, h->lAc, h->stream);
        check_launch();
        stokes_norm(h, h->lAc, S3);
        if (h->knobs.precision == LMM_PRECISION_FP32) {
            precon32(h, h->lAc, h->lz32);
            launch_convert<float, double>(h->lz32, h->lc.base, len, h->stream);
            check_launch();
        } else {
            precon64(h, h->lAc, h->lc);
        }
        launch_lin(h->le.base, h->le.base, -1.0, h->lc.base, len, h->stream);
        check_launch();
        launch_apply_matrix(h->L64[0], h->knobs.visc_type, h->le, h->lr1, h->stream);
        check_launch();
        stokes_norm(h, h->lr1, S1);
        launch_features(h->D0, h->lr1.base, h->L64[0].beta, h->slot(S1), h->grid.dx, nn::net_input(h->net), h->stream);
        check_launch();
        if (nn::net_forward_on(h->net, h->stream) != LMM_OK) throw LmmError(LMM_ERR_CUDA);
        launch_correction(h->D0, nn::net_output(h->net), h->L64[0].beta, h->slot(S1), h->grid.dx, h->lc.base, h->stream);
        check_launch();
        launch_apply_matrix(h->L64[0], h->knobs.visc_type, h->lc, h->lAc, h->stream);
        check_launch();
        launch_lin(h->le.base, h->lr1.base, -1.0, h->lAc.base, len, h->stream);
        check_launch();
        stokes_norm(h, h->le, S2);
        const double n0 = read_slot(h, S3, 5), n1 = read_slot(h, S1, 5), n2 = read_slot(h, S2, 5);
        ratios[0] = n0 > 0 ? n1 / n0 : 0.0;
        ratios[1] = n1 > 0 ? n2 / n1 : 0.0;
        return LMM_OK;
    } catch (const LmmError& e) {
        return e.code;
    }
}

// accepted / tried corrections of the last solve
extern "C" int lmm_learned_stats(lmm_handle* h, int* accepted, int* tried) {
    if (!h || !accepted || !tried) return LMM_ERR_INVALID;
    if (!h->luses) {
        *accepted = *tried = 0;
        return LMM_OK;
    }
    int u[2] = {0, 0};
    if (cudaMemcpyAsync(u, h->luses, sizeof(u), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess) return LMM_ERR_CUDA;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return LMM_ERR_CUDA;
    *accepted = u[0];
    *tried = u[1];
    return LMM_OK;
}

// the bounds-check table and record of this translation unit (empty
// unless built with -DLMM_BOUNDS_CHECK)
LMM_BC_UNIT(solver)
