// autotune.cu - the table of the block-shape autotuner (kernels.h).
//
// The autotuner itself (solver.cu, autotune_level) times candidate block
// shapes of the stencil kernels of one level on the first handle of that
// grid size and stores the fastest here; every later launch of the same
// kernel on the same grid, precision and visc_type, by any handle of the
// process (the one-problem handles and the batch handles of an ensemble),
// reads it.  The choice changes only the launch geometry, never a value.
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "kernels.h"

namespace lmm {
namespace {

using Key = std::tuple<int, int, int, int, int, int, int>;  // kernel, bytes, visc, dm, nx, ny, nz
struct Entry {
    Shape s;
    double ms_default, ms_best;
};
std::mutex g_mu;
std::map<Key, Entry> g_table;
thread_local Shape g_forced;

Key key_of(int kernel, int wbytes, int visc, const Dims& D) { return Key(kernel, wbytes, visc, D.dm, D.nx, D.ny, D.nz); }

const char* kernel_name(int k) {
    switch (k) {
    case TK_GS_COLOUR: return "gs_colour";
    case TK_APPLYOP: return "applyop";
    case TK_PROLONG: return "prolong_add";
    case TK_RESIDUAL: return "residual";
    case TK_APPLY_MATRIX: return "apply_matrix";
    default: return "?";
    }
}

}  // namespace

Shape tuned_shape(int kernel, int wbytes, int visc, const Dims& D) {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_table.find(key_of(kernel, wbytes, visc, D));
    return it == g_table.end() ? Shape{} : it->second.s;
}

bool is_tuned(int kernel, int wbytes, int visc, const Dims& D) {
    std::lock_guard<std::mutex> lock(g_mu);
    return g_table.count(key_of(kernel, wbytes, visc, D)) != 0;
}

void set_tuned_shape(int kernel, int wbytes, int visc, const Dims& D, Shape s, double ms_default, double ms_best) {
    std::lock_guard<std::mutex> lock(g_mu);
    g_table[key_of(kernel, wbytes, visc, D)] = Entry{s, ms_default, ms_best};
}

void force_shape(Shape s) { g_forced = s; }
Shape forced_shape() { return g_forced; }

}  // namespace lmm

// One line per tuned (kernel, precision, visc_type, grid): the chosen block
// (0 x 0 = the library's default geometry) and the measured ms of one
// launch with the default and with the choice.  Returns the bytes the full
// report needs (excluding the terminating zero); writes at most cap - 1 of
// them and a terminating zero when cap > 0.
extern "C" int lmm_autotune_report(char* buf, int cap) {
    using namespace lmm;
    std::string out;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        for (const auto& kv : g_table) {
            int kid, w, visc, dm, nx, ny, nz;
            std::tie(kid, w, visc, dm, nx, ny, nz) = kv.first;
            char line[256];
            std::snprintf(line, sizeof(line), "%s fp%d visc %d %dD %dx%dx%d: block %dx%d (%.4f ms default, %.4f ms chosen)\n",
                          kernel_name(kid), 8 * w, visc, dm, nx, ny, nz, kv.second.s.bx, kv.second.s.by, kv.second.ms_default,
                          kv.second.ms_best);
            out += line;
        }
    }
    if (buf && cap > 0) {
        const size_t n = std::min(out.size(), (size_t)cap - 1);
        std::memcpy(buf, out.data(), n);
        buf[n] = 0;
    }
    return (int)out.size();
}

// the bounds-check table and record of this translation unit (empty
// unless built with -DLMM_BOUNDS_CHECK)
LMM_BC_UNIT(autotune)
