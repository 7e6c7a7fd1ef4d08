// ensemble.cu - lmm_ensemble_solve: many independent Stokes problems of
// uneven sizes (different grids, seeds and viscosity fields) solved
// concurrently on one GPU.
//
// Worker threads pull instances from a shared queue, largest first; each
// worker owns one solver handle per grid shape it meets (its own CUDA
// stream, device workspaces and captured preconditioner graphs), so small
// 2D solves from different workers overlap on the GPU instead of running
// one after another.  Results are the same bits as one lmm_stokes_solve_device
// call per instance.
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

struct Worker {
    int device = 0;
    lmm_knobs knobs{};
    int dm = 2;
    std::map<std::tuple<int, int, int, double>, lmm_handle*> handles;
    ~Worker() {
        for (auto& kv : handles) lmm_stokes_destroy(kv.second);
    }
    lmm_handle* handle_for(const lmm_ensemble_item& it, int* rc) {
        const auto key = std::make_tuple(it.n[0], it.n[1], dm == 3 ? it.n[2] : 1, it.dx);
        auto f = handles.find(key);
        if (f != handles.end()) return f->second;
        lmm_grid g{};
        g.dm = dm;
        for (int d = 0; d < 3; ++d) {
            g.n[d] = d < dm ? it.n[d] : 1;
            g.bc_lo[d] = g.bc_hi[d] = LMM_BC_PERIODIC;
        }
        g.dx = it.dx;
        lmm_handle* h = nullptr;
        *rc = lmm_stokes_create(&g, &knobs, device, &h);
        if (*rc < 0) return nullptr;
        handles[key] = h;
        return h;
    }
};

}  // namespace

extern "C" int lmm_ensemble_solve(int dm, const lmm_knobs* knobs, int device, lmm_ensemble_item* items, int count, int workers) {
    if ((dm != 2 && dm != 3) || !knobs || !items || count < 0 || workers < 1) return LMM_ERR_INVALID;
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
    std::atomic<int> next{0};
    const int nw = std::min(workers, count);
    std::vector<std::thread> pool;
    pool.reserve(nw);
    for (int w = 0; w < nw; ++w) {
        pool.emplace_back([&, w]() {
            Worker W;
            W.device = device;
            W.knobs = *knobs;
            W.dm = dm;
            if (cudaSetDevice(device) != cudaSuccess) return;
            for (;;) {
                const int q = next.fetch_add(1);
                if (q >= count) break;
                lmm_ensemble_item& it = items[order[q]];
                int rc = LMM_OK;
                lmm_handle* h = W.handle_for(it, &rc);
                if (!h) {
                    it.status = rc;
                    continue;
                }
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
