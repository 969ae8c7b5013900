// prog_runner.cu -- gral_prog_solve_instances: independent weather situations on grids of
// different sizes, solved several at once.
//
// GRAL solves its situations one after the other (Program.cs:403-742); a single situation keeps
// only part of a B200 busy (its wavefronts are a few hundred warps wide), so independent
// instances run side by side, each in its own context on its own non-blocking stream.  The
// wavefront kernels claim their tasks in dependency order from an atomic counter, so they need no
// co-residency and make progress next to each other's launches.
//
// Admission and packing: the instances are ordered by their device footprint, largest first.
// The largest is loaded and its footprint measured; the others' are scaled from it by their field
// sizes, and K slots are opened for the largest K instances whose footprints fit the HBM budget
// together.  Those K loads run one after the other before any solve starts, so every device
// allocation happens while nothing else runs (an allocation can wait for work in flight on the
// device).  Then each slot's thread solves its instance and takes the next largest one left from a
// shared queue as soon as it is done, loading it into the buffers of its first (larger) instance:
// no slot waits for another, and the memory in use never exceeds what was admitted.
#include <algorithm>
#include <atomic>
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

// Device bytes of one instance's load, up to a common factor: the solver fields and row carry
// ([col][KS] floats, ten fields), the staging copies ([col][NKK+2], three fields) and the
// per-column tables.
double footprint_units(const gral_params &q) {
    const double ncols = (double)(q.nii + 2) * (q.njj + 2);
    const double ks = (double)(((q.kadvmax + 2) + 7) / 8 * 8);
    return ncols * (10.0 * ks + 3.0 * (q.nkk + 2) + 16.0);
}

}  // namespace

extern "C" int gral_prog_solve_instances(int32_t n, const gral_params *p, const gral_static *s, gral_fields *f,
                                         gral_stats *stats, int32_t *status, int32_t max_concurrent,
                                         uint64_t hbm_bytes) {
    if (n < 1 || !p || !s || !f || !status || max_concurrent < 1) return GRAL_EINVAL;
    int dims[4] = {4, 4, 3, 2};   // capacity bounds of every context: the largest of each dimension
    for (int b = 0; b < n; ++b) {
        dims[0] = std::max(dims[0], p[b].nii);
        dims[1] = std::max(dims[1], p[b].njj);
        dims[2] = std::max(dims[2], p[b].nkk);
        dims[3] = std::max(dims[3], p[b].kadvmax);
        status[b] = GRAL_EINVAL;
    }
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return footprint_units(p[a]) > footprint_units(p[b]); });

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
    // the largest instance is loaded first; its measured footprint scales the others'
    const int first_rc = gral_prog_load(slot[0], 1, p + order[0], s + order[0], f + order[0]);
    cudaMemGetInfo(&free1, &total);
    const double bytes0 = (double)std::max<size_t>(free0 > free1 ? free0 - free1 : 0, 64u << 20) * 1.1;
    const double per_unit = bytes0 / footprint_units(p[order[0]]);
    const double budget = hbm_bytes ? (double)hbm_bytes : 0.9 * (double)free0;
    int K = 1;
    double used = bytes0;
    while (K < std::min(n, max_concurrent)) {
        const double next = per_unit * footprint_units(p[order[K]]);
        if (used + next > budget) break;
        used += next;
        ++K;
    }
    slot.resize(K, nullptr);

    // the first K loads, one after the other, before any solve
    std::vector<int> rcs(K, GRAL_OK);
    rcs[0] = first_rc;
    for (int t = 1; t < K; ++t) {
        const int b = order[t];
        rcs[t] = gral_prog_create(dims[0], dims[1], dims[2], dims[3], 1, &slot[t]);
        if (rcs[t] == GRAL_OK) rcs[t] = gral_prog_load(slot[t], 1, p + b, s + b, f + b);
    }
    // each slot solves its instance, then takes the next largest one left
    std::atomic<int> next{K};
    std::vector<std::thread> pool;
    pool.reserve(K);
    for (int t = 0; t < K; ++t) {
        pool.emplace_back([&, t]() {
            cudaSetDevice(dev);
            int q = t;
            int lrc = rcs[t];
            for (;;) {
                const int b = order[q];
                if (lrc == GRAL_OK) lrc = finish_one(slot[t], f + b, stats ? stats + b : nullptr);
                status[b] = lrc;
                drop_if_failed(slot[t], lrc);
                q = next.fetch_add(1);
                if (q >= n) break;
                const int nb = order[q];
                lrc = GRAL_OK;
                if (!slot[t]) lrc = gral_prog_create(dims[0], dims[1], dims[2], dims[3], 1, &slot[t]);
                if (lrc == GRAL_OK) lrc = gral_prog_load(slot[t], 1, p + nb, s + nb, f + nb);
            }
        });
    }
    for (auto &th : pool) th.join();
    for (auto *c : slot)
        if (c) gral_prog_destroy(c);
    for (int b = 0; b < n; ++b)
        if (status[b] != GRAL_OK) return status[b];
    return GRAL_OK;
}

extern "C" int gral_prog_solve_batch_devices(int32_t ndev, const int32_t *devices, int32_t n, const gral_params *p,
                                             const gral_static *s, gral_fields *f, gral_stats *stats) {
    if (ndev < 1 || !devices || n < ndev || !p || !s || !f) return GRAL_EINVAL;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) {
        cudaGetLastError();
        return GRAL_ENODEV;
    }
    for (int d = 0; d < ndev; ++d)
        if (devices[d] < 0 || devices[d] >= count) return GRAL_EINVAL;
    std::vector<int> rcs(ndev, GRAL_OK);
    std::vector<std::thread> pool;
    pool.reserve(ndev);
    for (int d = 0; d < ndev; ++d) {
        pool.emplace_back([&, d]() {
            const int b0 = (int)((long long)d * n / ndev), b1 = (int)((long long)(d + 1) * n / ndev);
            if (cudaSetDevice(devices[d]) != cudaSuccess) {
                rcs[d] = GRAL_ENODEV;
                return;
            }
            gral_ctx *ctx = nullptr;
            int rc = gral_prog_create(p[b0].nii, p[b0].njj, p[b0].nkk, p[b0].kadvmax, b1 - b0, &ctx);
            if (rc == GRAL_OK) rc = gral_prog_solve_batch(ctx, b1 - b0, p + b0, s, f + b0, stats ? stats + b0 : nullptr);
            if (ctx) gral_prog_destroy(ctx);
            rcs[d] = rc;
        });
    }
    for (auto &th : pool) th.join();
    for (int d = 0; d < ndev; ++d)
        if (rcs[d] != GRAL_OK) return rcs[d];
    return GRAL_OK;
}
