// ensemble.cu - lmm_ensemble_solve: many independent Stokes problems of
// uneven sizes (different grids, seeds and viscosity fields) solved
// concurrently on one GPU.
//
// Worker threads pull instances from a shared queue, largest first; each
// worker owns one solver handle per grid shape of the ensemble (its own CUDA
// stream, device workspaces and captured preconditioner graphs; all created
// before the first solve and destroyed after the last), so small 2D solves
// from different workers overlap on the GPU instead of running one after
// another.  Results are the same bits as one lmm_stokes_solve_device call
// per instance.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <numeric>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/lmm_ensemble.h"
#include "../../include/lmm_stokes.h"

namespace {

using Shape = std::tuple<int, int, int, double>;

Shape shape_of(const lmm_ensemble_item& it, int dm) { return std::make_tuple(it.n[0], it.n[1], dm == 3 ? it.n[2] : 1, it.dx); }

}  // namespace

// the worker pool's handles: one per (worker, grid shape)
struct lmm_ensemble {
    int dm = 2, device = 0, workers = 1;
    lmm_knobs knobs{};
    std::vector<std::map<Shape, lmm_handle*>> handles;
    ~lmm_ensemble() {
        for (auto& m : handles)
            for (auto& kv : m) lmm_stokes_destroy(kv.second);
    }
};

extern "C" int lmm_ensemble_create(int dm, const lmm_knobs* knobs, int device, const lmm_ensemble_item* shapes, int nshapes,
                                   int workers, lmm_ensemble** out) {
    if ((dm != 2 && dm != 3) || !knobs || !shapes || nshapes < 1 || workers < 1 || !out) return LMM_ERR_INVALID;
    *out = nullptr;
    lmm_ensemble* E = new lmm_ensemble();
    E->dm = dm;
    E->device = device;
    E->workers = workers;
    E->knobs = *knobs;
    E->handles.resize(workers);
    std::vector<Shape> list;
    for (int i = 0; i < nshapes; ++i) {
        const Shape sh = shape_of(shapes[i], dm);
        if (std::find(list.begin(), list.end(), sh) == list.end()) list.push_back(sh);
    }
    for (int w = 0; w < workers; ++w)
        for (const Shape& sh : list) {
            lmm_grid g{};
            g.dm = dm;
            g.n[0] = std::get<0>(sh);
            g.n[1] = std::get<1>(sh);
            g.n[2] = std::get<2>(sh);
            for (int d = 0; d < 3; ++d) g.bc_lo[d] = g.bc_hi[d] = LMM_BC_PERIODIC;
            g.dx = std::get<3>(sh);
            lmm_handle* h = nullptr;
            const int rc = lmm_stokes_create(&g, knobs, device, &h);
            if (rc < 0) {
                delete E;
                return rc;
            }
            E->handles[w][sh] = h;
        }
    *out = E;
    return LMM_OK;
}

extern "C" int lmm_ensemble_destroy(lmm_ensemble* E) {
    delete E;
    return LMM_OK;
}

extern "C" int lmm_ensemble_run(lmm_ensemble* E, lmm_ensemble_item* items, int count) {
    if (!E || !items || count < 0) return LMM_ERR_INVALID;
    const int dm = E->dm;
    for (int i = 0; i < count; ++i) {
        items[i].status = LMM_ERR_INVALID;  // until a worker solves it
        if (E->handles[0].find(shape_of(items[i], dm)) == E->handles[0].end()) return LMM_ERR_INVALID;
    }
    if (count == 0) return LMM_OK;
    // largest instances first, so the queue ends with short jobs
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    auto cells = [&](int i) {
        int64_t c = 1;
        for (int d = 0; d < dm; ++d) c *= items[i].n[d];
        return c;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cells(a) > cells(b); });
    const int nw = std::min(E->workers, count);
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    pool.reserve(nw);
    for (int w = 0; w < nw; ++w) {
        pool.emplace_back([&, w]() {
            if (cudaSetDevice(E->device) != cudaSuccess) return;
            for (;;) {
                const int q = next.fetch_add(1);
                if (q >= count) break;
                lmm_ensemble_item& it = items[order[q]];
                lmm_handle* h = E->handles[w][shape_of(it, dm)];
                double th = it.theta_alpha, npr = 0.0;
                lmm_fields_in fin{};
                lmm_fields_out fout{};
                for (int d = 0; d < 3; ++d) {
                    fin.b_u[d] = it.b_u[d];
                    fin.alpha_fc[d] = it.alpha_fc[d];
                    fin.beta_ed[d] = it.beta_ed[d];
                    fout.x_u[d] = it.x_u[d];
                }
                fin.b_p = it.b_p;
                fin.beta = it.beta;
                fin.gamma = it.gamma;
                fin.layout = LMM_LAYOUT_COMPACT;
                fout.x_p = it.x_p;
                fout.layout = LMM_LAYOUT_COMPACT;
                it.status = lmm_stokes_solve_device(h, &fin, &fout, &th, &npr, &it.stats);
            }
        });
    }
    for (auto& t : pool) t.join();
    int worst = LMM_OK;
    for (int i = 0; i < count; ++i)
        if (items[i].status < 0) worst = items[i].status;
    return worst;
}

extern "C" int lmm_ensemble_solve(int dm, const lmm_knobs* knobs, int device, lmm_ensemble_item* items, int count, int workers) {
    if ((dm != 2 && dm != 3) || !knobs || !items || count < 0 || workers < 1) return LMM_ERR_INVALID;
    if (count == 0) return LMM_OK;
    lmm_ensemble* E = nullptr;
    const int rc = lmm_ensemble_create(dm, knobs, device, items, count, std::min(workers, count), &E);
    if (rc < 0) return rc;
    const int r = lmm_ensemble_run(E, items, count);
    lmm_ensemble_destroy(E);
    return r;
}
