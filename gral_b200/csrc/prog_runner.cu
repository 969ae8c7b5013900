// prog_runner.cu -- gral_prog_solve_instances: independent weather situations on grids of
// different sizes, solved several at once.
//
// GRAL solves its situations one after the other (Program.cs:403-742); a single situation keeps
// only part of a B200 busy (its wavefronts are a few hundred warps wide), so independent
// instances run side by side, each in its own context on its own non-blocking stream.  The
// wavefront kernels claim their tasks in dependency order from an atomic counter, so they need no
// co-residency and make progress next to each other's launches.
//
// The instances go in waves of K (largest first, so a wave holds instances of similar size): the
// calling thread loads the wave's instances one after the other while nothing else runs on the
// device, then K threads iterate and store them at the same time.  Loading in between running
// solves would not overlap with them: a device allocation (DevBuf growth at load) and the memsets
// of the set-up wait for all work already in flight on the device.  Loads of later waves mostly
// reuse the buffers of the first, larger ones.
#include <algorithm>
#include <numeric>
#include <thread>
#include <vector>

#include "prog_ctx.cuh"

namespace {

// The part of gral_prog_solve_batch after the load, for one situation: iterate, store, timings.
int finish_one(gral_ctx *ctx, gral_fields *f, gral_stats *st) {
    cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1];
    cudaEventRecord(e0, ctx->stream);
    int rc = gral_prog_iterate(ctx);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float ms_it = 0.f;
    cudaEventElapsedTime(&ms_it, e0, e1);
    if (rc != GRAL_OK) return rc;
    rc = gral_prog_store(ctx, f, st);
    if (st) {
        st->ms_iterate = ms_it;
        st->ms_total = st->ms_upload + ms_it + st->ms_download;
    }
    return rc;
}

// A failed instance other than for non-finite results may leave its context unusable: it is
// released, and a new one is created for the slot's next instance.
void drop_if_failed(gral_ctx *&ctx, int rc) {
    if (rc == GRAL_OK || rc == GRAL_ENONFINITE || !ctx) return;
    gral_prog_destroy(ctx);
    ctx = nullptr;
}

}  // namespace

extern "C" int gral_prog_solve_instances(int32_t n, const gral_params *p, const gral_static *s, gral_fields *f,
                                         gral_stats *stats, int32_t *status, int32_t max_concurrent,
                                         uint64_t hbm_bytes) {
    if (n < 1 || !p || !s || !f || !status || max_concurrent < 1) return GRAL_EINVAL;
    int dims[4] = {4, 4, 3, 2};   // capacity of every context: the largest of each dimension
    for (int b = 0; b < n; ++b) {
        dims[0] = std::max(dims[0], p[b].nii);
        dims[1] = std::max(dims[1], p[b].njj);
        dims[2] = std::max(dims[2], p[b].nkk);
        dims[3] = std::max(dims[3], p[b].kadvmax);
        status[b] = GRAL_EINVAL;
    }
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    auto cells = [&](int b) { return (long long)(p[b].nii + 2) * (p[b].njj + 2) * (p[b].nkk + 2); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cells(a) > cells(b); });

    size_t free0 = 0, total = 0, free1 = 0;
    if (cudaMemGetInfo(&free0, &total) != cudaSuccess) {
        cudaGetLastError();
        return GRAL_ENODEV;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    std::vector<gral_ctx *> slot(1, nullptr);
    int rc = gral_prog_create(dims[0], dims[1], dims[2], dims[3], 1, &slot[0]);
    if (rc != GRAL_OK) return rc;
    // the largest instance is loaded first: its footprint decides the wave size K
    int first_rc = gral_prog_load(slot[0], 1, p + order[0], s + order[0], f + order[0]);
    cudaMemGetInfo(&free1, &total);
    const size_t footprint = std::max<size_t>(free0 > free1 ? free0 - free1 : 0, 64u << 20) * 11 / 10;
    const uint64_t budget = hbm_bytes ? hbm_bytes : (uint64_t)(0.9 * (double)free0);
    int K = (int)std::min<uint64_t>((uint64_t)max_concurrent, std::max<uint64_t>(1, budget / footprint));
    K = std::min(K, n);
    slot.resize(K, nullptr);

    std::vector<int> rcs(K);
    for (int w0 = 0; w0 < n; w0 += K) {
        const int m = std::min(K, n - w0);
        // loads of the wave, nothing else on the device
        for (int t = 0; t < m; ++t) {
            const int b = order[w0 + t];
            if (w0 == 0 && t == 0) {
                rcs[t] = first_rc;
                continue;
            }
            rcs[t] = GRAL_OK;
            if (!slot[t]) rcs[t] = gral_prog_create(dims[0], dims[1], dims[2], dims[3], 1, &slot[t]);
            if (rcs[t] == GRAL_OK) rcs[t] = gral_prog_load(slot[t], 1, p + b, s + b, f + b);
        }
        // iterations and stores of the wave, side by side
        std::vector<std::thread> pool;
        pool.reserve(m);
        for (int t = 0; t < m; ++t) {
            if (rcs[t] != GRAL_OK) continue;
            const int b = order[w0 + t];
            pool.emplace_back([&, t, b]() {
                cudaSetDevice(dev);
                rcs[t] = finish_one(slot[t], f + b, stats ? stats + b : nullptr);
            });
        }
        for (auto &th : pool) th.join();
        for (int t = 0; t < m; ++t) {
            status[order[w0 + t]] = rcs[t];
            drop_if_failed(slot[t], rcs[t]);
        }
    }
    for (auto *c : slot)
        if (c) gral_prog_destroy(c);
    for (int b = 0; b < n; ++b)
        if (status[b] != GRAL_OK) return status[b];
    return GRAL_OK;
}
