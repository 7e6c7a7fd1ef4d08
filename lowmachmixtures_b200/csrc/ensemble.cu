// ensemble.cu - lmm_ensemble_solve: many independent Stokes problems of
// uneven sizes (different grids, seeds and viscosity fields) solved
// concurrently on one GPU.
//
// 2D problems whose knobs batch (lmm_stokes_create_batch; knobs
// ensemble_batch = 0) are solved in batches: the problems of one (grid, dx,
// theta_alpha) group share a batch handle holding up to kMaxBatch of them,
// so each kernel launch and captured graph covers the group; groups run
// concurrently, one host thread and stream each.
//
// Otherwise worker threads pull instances from a shared queue, largest
// first; each worker owns one solver handle per grid shape of the ensemble
// (its own CUDA stream, device workspaces and captured preconditioner
// graphs; all created before the first solve and destroyed after the last),
// so small solves from different workers overlap on the GPU instead of
// running one after another.
//
// Either way each result is the same bits as one lmm_stokes_solve_device
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

using Shape = std::tuple<int, int, int, double>;
using BatchKey = std::tuple<int, int, double, double>;  // nx, ny, dx, theta_alpha

// problems per batch handle: 128 instances of 256^2 take about 4 GB
constexpr int kMaxBatch = 128;

Shape shape_of(const lmm_ensemble_item& it, int dm) { return std::make_tuple(it.n[0], it.n[1], dm == 3 ? it.n[2] : 1, it.dx); }
BatchKey batch_key(const lmm_ensemble_item& it) { return std::make_tuple(it.n[0], it.n[1], it.dx, it.theta_alpha); }

// the knobs lmm_stokes_create_batch accepts
bool batchable(int dm, const lmm_knobs& k) {
    return k.ensemble_batch == 0 && dm == 2 && k.method == LMM_METHOD_FGMRES && k.visc_type < 0 && k.learned_stage == 0 &&
           k.visc_schur_approx == 0 && k.stag_mg_max_vcycles <= 1 && k.scale_factor == 1.0 && k.gmres_max_inner <= 45;
}

}  // namespace

// batch handles per (grid, dx, theta_alpha), or the worker pool's handles:
// one per (worker, grid shape)
struct lmm_ensemble {
    int dm = 2, device = 0, workers = 1;
    lmm_knobs knobs{};
    bool batched = false;
    std::map<BatchKey, lmm_handle*> batches;
    std::map<BatchKey, int> batch_size;
    std::vector<std::map<Shape, lmm_handle*>> handles;
    ~lmm_ensemble() {
        for (auto& kv : batches) lmm_stokes_destroy(kv.second);
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
    if (batchable(dm, *knobs)) {
        E->batched = true;
        std::map<BatchKey, int> counts;
        for (int i = 0; i < nshapes; ++i) counts[batch_key(shapes[i])] += 1;
        for (const auto& kv : counts) {
            lmm_grid g{};
            g.dm = 2;
            g.n[0] = std::get<0>(kv.first);
            g.n[1] = std::get<1>(kv.first);
            g.n[2] = 1;
            for (int d = 0; d < 3; ++d) g.bc_lo[d] = g.bc_hi[d] = LMM_BC_PERIODIC;
            g.dx = std::get<2>(kv.first);
            const int bs = std::min(kv.second, kMaxBatch);
            lmm_handle* h = nullptr;
            const int rc = lmm_stokes_create_batch(&g, knobs, bs, device, &h);
            if (rc < 0) {
                delete E;
                return rc;
            }
            E->batches[kv.first] = h;
            E->batch_size[kv.first] = bs;
        }
        *out = E;
        return LMM_OK;
    }
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

namespace {

// the items of each (grid, dx, theta_alpha) group in chunks of its handle's
// batch size; groups concurrently, one host thread each
int run_batched(lmm_ensemble* E, lmm_ensemble_item* items, int count) {
    std::map<BatchKey, std::vector<int>> groups;
    for (int i = 0; i < count; ++i) {
        items[i].status = LMM_ERR_INVALID;  // until its batch is solved
        const BatchKey key = batch_key(items[i]);
        if (E->batches.find(key) == E->batches.end()) return LMM_ERR_INVALID;
        groups[key].push_back(i);
    }
    std::vector<int> rcs(groups.size(), LMM_OK);
    std::vector<std::thread> pool;
    int gi = 0;
    for (auto& kv : groups) {
        lmm_handle* h = E->batches[kv.first];
        const size_t bs = (size_t)E->batch_size[kv.first];
        const std::vector<int>* idx = &kv.second;
        int* rc = &rcs[gi++];
        pool.emplace_back([=]() {
            if (cudaSetDevice(E->device) != cudaSuccess) {
                *rc = LMM_ERR_CUDA;
                return;
            }
            std::vector<lmm_ensemble_item> chunk;
            for (size_t s = 0; s < idx->size();) {
                const size_t e = std::min(idx->size(), s + bs);
                chunk.clear();
                for (size_t q = s; q < e; ++q) chunk.push_back(items[(*idx)[q]]);
                const int r = lmm_stokes_solve_batch(h, chunk.data(), (int)chunk.size());
                for (size_t q = s; q < e; ++q) items[(*idx)[q]] = chunk[q - s];
                if (r < 0 && r != LMM_ERR_NONFINITE) *rc = r;  // per-item statuses carry the rest
                s = e;
            }
        });
    }
    for (auto& t : pool) t.join();
    int worst = LMM_OK;
    for (int i = 0; i < count; ++i)
        if (items[i].status < 0) worst = items[i].status;
    for (int r : rcs)
        if (r < 0) worst = r;
    return worst;
}

}  // namespace

extern "C" int lmm_ensemble_run(lmm_ensemble* E, lmm_ensemble_item* items, int count) {
    if (!E || !items || count < 0) return LMM_ERR_INVALID;
    if (E->batched) return count == 0 ? LMM_OK : run_batched(E, items, count);
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
