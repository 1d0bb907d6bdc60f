// batch.cpp — many independent forging cases stepped together, and the tuner that picks their factorisation's
// launch parameters.
//
// The reference runs independent cases (the levels of a mesh-convergence study) with Parallel.For
// (ThreeD/MeshConvergence.cs:117), one solver per case. Here each case keeps its own context, hence its own CUDA
// streams and captured graphs, and a pool of host threads steps the cases: the GPU receives the kernels of many
// cases at once and runs them side by side, so small cases that leave most SMs idle on their own fill the device
// together. A case that fails stops; the others go on.
//
// The tuner times the single-precision factorisation and one solve of a case's current matrix for each candidate
// of the two launch parameters that shape its kernels: the row count from which the trailing update runs on the
// tensor cores, and the front height from which the solves use the multi-CTA path. The best pair is cached by
// problem size (the equation count rounded to a power of two), so that one case of each size class is measured
// and the others of its class reuse the choice.
#include <atomic>
#include <chrono>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ifea_gpu.h"

namespace {

struct Batch {
    std::vector<ifea3d *> c3;
    std::vector<ifea2d *> c2;
    int threads = 1;
};

std::mutex g_tune_mutex;
std::map<int, std::pair<double, double>> g_tune_cache;  // size class -> (tc_rows, wide_front_rows)

}  // namespace

struct ifea_batch {
    Batch b;
};

extern "C" {

ifea_status ifea_batch_create(int32_t n3, ifea3d *const *ctx3, int32_t n2, ifea2d *const *ctx2, int32_t threads,
                              ifea_batch **out)
{
    if (!out || n3 < 0 || n2 < 0 || (n3 && !ctx3) || (n2 && !ctx2) || n3 + n2 == 0) return IFEA_INPUT_INVALID;
    auto *b = new ifea_batch;
    b->b.c3.assign(ctx3, ctx3 + n3);
    b->b.c2.assign(ctx2, ctx2 + n2);
    int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    b->b.threads = threads > 0 ? threads : std::min(n3 + n2, hw);
    *out = b;
    return IFEA_OK;
}

void ifea_batch_destroy(ifea_batch *b) { delete b; }

ifea_status ifea_batch_step(ifea_batch *bh, int32_t increments, ifea_step_info *infos, int32_t *status)
{
    if (!bh || increments <= 0 || !infos || !status) return IFEA_INPUT_INVALID;
    Batch &b = bh->b;
    int n3 = (int)b.c3.size(), n = n3 + (int)b.c2.size();
    for (int c = 0; c < n; c++) status[c] = IFEA_OK;
    // one case per task, each task all of that case's increments: the cases' contexts are independent and a
    // context is only ever driven by one thread at a time
    std::atomic<int> next{0};
    auto worker = [&] {
        for (;;) {
            int c = next.fetch_add(1);
            if (c >= n) return;
            for (int k = 0; k < increments; k++) {
                ifea_step_info *info = infos + (size_t)c * increments + k;
                ifea_status st = c < n3 ? ifea3d_step(b.c3[c], info, nullptr) : ifea2d_step(b.c2[c - n3], info, nullptr);
                if (st != IFEA_OK) {
                    status[c] = st;
                    break;
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < std::min(b.threads, n); t++) pool.emplace_back(worker);
    for (auto &t : pool) t.join();
    for (int c = 0; c < n; c++)
        if (status[c] != IFEA_OK) return (ifea_status)status[c];
    return IFEA_OK;
}

ifea_status ifea3d_autotune(ifea3d *ctx, int32_t use_cache, double *tc_rows, double *wide_rows, double *best_ms)
{
    if (!ctx) return IFEA_INPUT_INVALID;
    double nd = 0;
    ifea_status st = ifea3d_get_scalar(ctx, "ndof", &nd);
    if (st != IFEA_OK) return st;
    int cls = (int)std::lround(std::log2(std::max(nd, 1.0)));
    if (use_cache) {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cache.find(cls);
        if (it != g_tune_cache.end()) {
            ifea3d_set_scalar(ctx, "tc_rows", it->second.first);
            ifea3d_set_scalar(ctx, "wide_front_rows", it->second.second);
            if (tc_rows) *tc_rows = it->second.first;
            if (wide_rows) *wide_rows = it->second.second;
            if (best_ms) *best_ms = -1;
            return IFEA_OK;
        }
    }
    // the matrix of the next increment's first Newton iteration, then each candidate's factorisation + solve
    if ((st = ifea3d_prepare_step(ctx)) != IFEA_OK) return st;
    double e = 0, p = 0, md = 0;
    if ((st = ifea3d_assemble(ctx, 1, 1, nullptr, &e, &p)) != IFEA_OK) return st;
    if ((st = ifea3d_apply_bc(ctx, &md)) != IFEA_OK) return st;
    const double tc_cand[4] = {512, 1024, 2048, 1e9};
    const double wide_cand[3] = {96, 192, 384};
    double best = INFINITY, bt = 1024, bw = 192;
    for (double w : wide_cand) {
        if ((st = ifea3d_set_scalar(ctx, "wide_front_rows", w)) != IFEA_OK) return st;
        for (double tcr : tc_cand) {
            if ((st = ifea3d_set_scalar(ctx, "tc_rows", tcr)) != IFEA_OK) return st;
            double ms = 0;
            for (int rep = 0; rep < 2; rep++)  // the first run after a change captures the graphs
                if ((st = ifea3d_time_factor_solve(ctx, &ms)) != IFEA_OK) return st;
            if (ms < best) {
                best = ms;
                bt = tcr;
                bw = w;
            }
        }
    }
    ifea3d_set_scalar(ctx, "wide_front_rows", bw);
    ifea3d_set_scalar(ctx, "tc_rows", bt);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tune_cache[cls] = {bt, bw};
    }
    if (tc_rows) *tc_rows = bt;
    if (wide_rows) *wide_rows = bw;
    if (best_ms) *best_ms = best;
    return IFEA_OK;
}

}  // extern "C"
