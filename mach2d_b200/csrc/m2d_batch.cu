// m2d_batch.cu -- many nozzle instances advanced together on one GPU.
//
// No counterpart in the reference (one instance per process there).  Each
// instance is a full context (own arena and non-blocking stream), so
// instances never share device state.  A single instance keeps at most the
// two MSI9 clusters busy (ny/32 SMs each), leaving most of the 148 SMs idle.
// A batch runs W host worker threads, each advancing its share of the
// instances.  Instances whose iterations run as captured CUDA graphs
// (m2d_ctx_set_graph) are advanced in two passes per iteration: every
// instance's graph is launched on its own stream first, then each stream is
// waited for and its iteration closed, so all of them are in flight at once
// and the GPU schedules their kernels together.  Other instances are advanced
// one call of m2d_iterate at a time.  Results of every instance are bitwise
// identical to running it alone.
#include <chrono>
#include <string>
#include <thread>
#include <vector>
#include "../../include/mach2d_b200.h"

extern void m2d_set_last_error_msg(const char *);
bool ctx_graph_on(const m2d_ctx *x);
int ctx_iterate_launch(m2d_ctx *x);
int ctx_iterate_complete(m2d_ctx *x, m2d_report *rep);

struct m2d_batch {
    std::vector<m2d_ctx *> ctx;
    std::vector<int> status;   // first non-zero status of each instance (it stops there)
    int workers = 1;
};

extern "C" int m2d_batch_create(const m2d_case *cases, int n, int device, int workers, m2d_batch **out)
{
    if (!cases || n < 1 || !out) {
        m2d_set_last_error_msg("m2d_batch_create: bad arguments");
        return M2D_ERR_ARG;
    }
    *out = nullptr;
    m2d_batch *b = new m2d_batch;
    b->workers = workers > 0 ? workers : (n < 16 ? n : 16);
    if (b->workers > n) b->workers = n;
    b->ctx.assign(n, nullptr);
    b->status.assign(n, M2D_OK);
    // the instances are set up by the worker threads (the host part of each
    // set-up, grid nodes and quasi-1D strips, runs in parallel; each device
    // part runs on its instance's own stream)
    std::vector<int> rc(n, M2D_OK);
    std::vector<std::string> msg(n);
    auto work = [&](int w) {
        for (int k = w; k < n; k += b->workers) {
            rc[k] = m2d_create(&cases[k], device, &b->ctx[k]);
            if (rc[k] != M2D_OK) msg[k] = m2d_last_error();
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < b->workers; w++) pool.emplace_back(work, w);
    work(0);
    for (auto &t : pool) t.join();
    for (int k = 0; k < n; k++) {
        if (rc[k] != M2D_OK) {
            const std::string m = std::string("m2d_batch_create: instance ") + std::to_string(k) + ": " + msg[k];
            for (m2d_ctx *c : b->ctx) if (c) m2d_destroy(c);
            delete b;
            m2d_set_last_error_msg(m.c_str());
            return rc[k];
        }
    }
    *out = b;
    return M2D_OK;
}

extern "C" int m2d_batch_size(const m2d_batch *b, int *n)
{
    if (!b || !n) return M2D_ERR_ARG;
    *n = (int)b->ctx.size();
    return M2D_OK;
}

extern "C" int m2d_batch_ctx(m2d_batch *b, int k, m2d_ctx **ctx)
{
    if (!b || !ctx || k < 0 || k >= (int)b->ctx.size()) return M2D_ERR_ARG;
    *ctx = b->ctx[k];
    return M2D_OK;
}

extern "C" int m2d_batch_iterate(m2d_batch *b, int iters, m2d_report *reps)
{
    if (!b || iters < 0) {
        m2d_set_last_error_msg("m2d_batch_iterate: bad arguments");
        return M2D_ERR_ARG;
    }
    const int n = (int)b->ctx.size(), W = b->workers;
    std::vector<std::string> msg(n);
    auto fail = [&](int k, int rc) {
        b->status[k] = rc;
        msg[k] = m2d_last_error();
    };
    auto work = [&](int w) {
        std::vector<char> launched(n, 0);
        for (int it = 0; it < iters; it++) {
            // captured iterations: every graph in flight before any wait
            for (int k = w; k < n; k += W) {
                launched[k] = 0;
                if (b->status[k] != M2D_OK || !ctx_graph_on(b->ctx[k])) continue;
                const int rc = ctx_iterate_launch(b->ctx[k]);
                if (rc != M2D_OK) fail(k, rc);
                else launched[k] = 1;
            }
            for (int k = w; k < n; k += W) {
                if (b->status[k] != M2D_OK) continue;
                m2d_report r;
                const int rc = launched[k] ? ctx_iterate_complete(b->ctx[k], &r) : m2d_iterate(b->ctx[k], &r);
                if (reps) reps[k] = r;
                if (rc != M2D_OK) fail(k, rc);
            }
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < W; w++) pool.emplace_back(work, w);
    work(0);
    for (auto &t : pool) t.join();
    for (int k = 0; k < n; k++) {
        if (b->status[k] != M2D_OK) {
            const std::string m = std::string("instance ") + std::to_string(k) + ": " + msg[k];
            m2d_set_last_error_msg(m.c_str());
            return b->status[k];
        }
    }
    return M2D_OK;
}

extern "C" int m2d_batch_set_msi_schedule(m2d_batch *b, int variant)
{
    if (!b || variant < 0 || variant > 3) {
        m2d_set_last_error_msg("m2d_batch_set_msi_schedule: bad arguments");
        return M2D_ERR_ARG;
    }
    for (m2d_ctx *c : b->ctx) {
        const int rc = m2d_ctx_set_msi_schedule(c, variant);
        if (rc != M2D_OK) return rc;
    }
    return M2D_OK;
}

// The schedule autotuner: the batch's own next iterations, `iters` of them
// (after one untimed iteration that captures the graphs) with each candidate
// schedule of every instance's MSI solves, timed on the host clock; the
// fastest is kept.  All schedules give the same iterates, so tuning on live
// iterations changes no result.
extern "C" int m2d_batch_autotune(m2d_batch *b, int iters, int *chosen, double *ms_per_iter)
{
    if (!b || iters < 1) {
        m2d_set_last_error_msg("m2d_batch_autotune: bad arguments");
        return M2D_ERR_ARG;
    }
    // the one-CTA kernel computes in FP64 only: a candidate only where every
    // instance solves in FP64
    bool fp64 = true;
    for (m2d_ctx *c : b->ctx) {
        double solver = 0;
        m2d_get_scalar(c, "solver", &solver);
        if (solver >= 2) fp64 = false;
    }
    const int cands[3] = {1, 2, 3};
    const int ncand = fp64 ? 3 : 2;
    int best = 1;
    double best_ms = 0;
    for (int q = 0; q < 4; q++)
        if (ms_per_iter) ms_per_iter[q] = -1.0;
    for (int q = 0; q < ncand; q++) {
        int rc = m2d_batch_set_msi_schedule(b, cands[q]);
        if (rc == M2D_OK) rc = m2d_batch_iterate(b, 1, nullptr);
        if (rc != M2D_OK) return rc;
        const auto t0 = std::chrono::steady_clock::now();
        rc = m2d_batch_iterate(b, iters, nullptr);
        if (rc != M2D_OK) return rc;
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / iters;
        if (ms_per_iter) ms_per_iter[cands[q]] = ms;
        if (q == 0 || ms < best_ms) { best = cands[q]; best_ms = ms; }
    }
    if (chosen) *chosen = best;
    return m2d_batch_set_msi_schedule(b, best);
}

extern "C" int m2d_batch_status(const m2d_batch *b, int k, int *status)
{
    if (!b || !status || k < 0 || k >= (int)b->ctx.size()) return M2D_ERR_ARG;
    *status = b->status[k];
    return M2D_OK;
}

extern "C" int m2d_batch_destroy(m2d_batch *b)
{
    if (!b) return M2D_OK;
    for (m2d_ctx *c : b->ctx) m2d_destroy(c);
    delete b;
    return M2D_OK;
}
