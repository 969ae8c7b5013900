// prog_host.cu -- C ABI of the B200 prognostic solver (include/gral_prog.h).
//
// A context owns the device memory of a batch of situations on one grid.  load() copies the host
// fields into full-height staging buffers, runs the per-situation set-up of
// PrognosticFlowfield.Calculate (PrognosticFlowfield.cs:45-579) and extracts the level slab the
// SIMPLE loop works on; iterate() replays a CUDA graph of one SIMPLE iteration (:584-1182) until
// every situation has converged or reached its iteration limit, deciding only at the iterations
// where the reference tests convergence; store() runs the post-checks (:1187-1245) and copies the
// fields back.  Per-column constants (VerticalIndex, KSTART, the friction-velocity help terms,
// the SIMD-chunk positions of the reference's Vector<float> loops) are computed here on the host
// in float, with the same expressions as the reference, once per load.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <utility>
#include <string>
#include <vector>

#include "gral_prog.h"
#include "prog_common.cuh"
#include "prog_ctx.cuh"
#include "prog_gff.cuh"
#include "prog_kernels.cuh"
#include "prog_prep.cuh"

using namespace gral;


namespace {

inline float f32(float x) { return x; }

// Math.Max/Math.Min(float, float) of .NET 8 (IEEE 754:2019 maximum/minimum)
inline float net_max(float a, float b) {
    if (a != b) { if (!std::isnan(a)) return (b < a) ? a : b; return a; }
    return std::signbit(b) ? a : b;
}
inline float net_min(float a, float b) {
    if (a != b) { if (!std::isnan(a)) return (a < b) ? a : b; return a; }
    return std::signbit(a) ? a : b;
}

// ---- per-column constants (host) ----------------------------------------------------------

// Levels of the reference's Vector<float> chunk loop (U-prognostic-microscale_1.cs:194-202):
// chunk bases KSTART, KSTART+W, ..., the last one pulled back to KEND-W.  kad is the first level
// processed by a chunk whose base lies above KKART+1 (extra eddy-viscosity terms, :453); wc_lo..
// wc_hi are the levels processed by chunks that contain KKART+1 (masked wall term, :419).
void chunk_levels(int K0, int KEND, int KK, int W, int &kad, int &wlo, int &whi) {
    kad = KEND;
    wlo = 1;
    whi = 0;
    for (int s = K0; s < KEND; s += W) {
        int base = s;
        if (s > KEND - W) base = KEND - W;
        const int hi = std::min(s + W - 1, KEND - 1);
        if (base > KK + 1) kad = std::min(kad, s);
        if (base <= KK + 1 && KK + 1 < base + W) {
            if (whi < wlo) { wlo = s; whi = hi; }
            else { wlo = std::min(wlo, s); whi = std::max(whi, hi); }
        }
    }
}

int build_meta(gral_ctx *ctx, const gral_params &p, const gral_static &s, std::vector<ColMeta> &meta,
               std::vector<uint32_t> &cfl, std::vector<ColF> &colf, std::vector<ColKE> &colke, int &vi_min,
               int &vi_max) {
    const int NII = p.nii, NJJ = p.njj, NKK = p.nkk, nj2 = NJJ + 2;
    const int ncols = (NII + 2) * nj2;
    meta.assign(ncols, ColMeta{});
    cfl.assign(ncols, 0u);
    colf.assign(ncols, ColF{});
    colke.assign(ncols, ColKE{0.0, -1, -1, -1, -1});
    auto adv = [&](int i, int j) { return (i >= 0 && i <= NII + 1 && j >= 0 && j <= NJJ + 1) ? s.advdom[i * nj2 + j] : 0; };
    auto kk = [&](int i, int j) { return (int)s.kkart[i * nj2 + j]; };
    const float *DZK = s.dzk;
    vi_min = 1 << 20;
    vi_max = 0;
    for (int i = 0; i <= NII + 1; ++i) {
        for (int j = 0; j <= NJJ + 1; ++j) {
            const int c = i * nj2 + j;
            ColMeta &m = meta[c];
            const int KK = kk(i, j);
            const float cutk = s.cutk[c];
            const bool inner = (i >= 1 && i <= NII && j >= 1 && j <= NJJ);
            const int VI = inner ? std::min(NKK - 1, KK + p.vert_cells_ff) : 0;   // :339
            const int K0 = (cutk == 0) ? KK + 1 : 1;
            m.kkart = (int16_t)KK;
            m.vi = (int16_t)VI;
            m.kstart = (int16_t)K0;
            m.kkm_u = (int16_t)std::max(KK, i >= 1 ? kk(i - 1, j) : KK);
            m.kkm_v = (int16_t)std::max(KK, j >= 1 ? kk(i, j - 1) : KK);
            int kad = VI + 1, wlo = 1, whi = 0;
            if (p.turbulence_model == 1 && inner) chunk_levels(K0, VI + 1, KK, p.simd_width, kad, wlo, whi);
            m.kad = (int16_t)kad;
            m.wc_lo = (int16_t)wlo;
            m.wc_hi = (int16_t)whi;
            uint32_t f = 0;
            if (adv(i, j) == 1) f |= F_ADV;
            if (inner) {
                const int ip = std::min(i + 1, NII + 1), jp = std::min(j + 1, NJJ + 1);
                if (adv(i, j) == 1 || adv(i - 1, j) == 1 || adv(ip, j) == 1 || adv(i, j - 1) == 1 ||
                    adv(i - 1, j - 1) == 1 || adv(ip, j - 1) == 1 || adv(i, jp) == 1 || adv(i - 1, jp) == 1 ||
                    adv(ip, jp) == 1)
                    f |= F_ALLOC3;
            }
            if (s.veg && s.veg_mask && s.veg_mask[c]) f |= F_VEG;
            if (cutk == 0) f |= F_CUTK0;
            if (cutk < 1) f |= F_CUTKLT1;
            if (cutk > 0) f |= F_CUTKGT0;
            if (i >= 1 && j >= 1 && (adv(i, j) == 1 || adv(i - 1, j) == 1 || adv(i, j - 1) == 1)) f |= F_VC;
            if (adv(i, j - 1) < 1 || j == 2) f |= F_BS;
            if (adv(i, j + 1) < 1 || j == NJJ - 1) f |= F_BN;
            if (adv(i - 1, j) < 1 || i == 2) f |= F_BW;
            if (adv(i + 1, j) < 1 || i == NII - 1) f |= F_BE;
            const float z0 = s.z0[c];
            ColF &cf = colf[c];
            cf.cov = s.cov ? s.cov[c] : 0.0f;
            cf.z0 = z0;
            if (inner && KK + 1 <= NKK) {
                const int k = KK + 1;
                if (z0 >= f32(DZK[k] * 0.1f)) f |= F_Z0GE;
                if ((double)z0 >= (double)DZK[k] * 0.1) f |= F_Z0GED;
                if (K0 <= k && k <= VI) {                                         // :347-403
                    if (cutk < 1) {
                        if ((double)z0 >= (double)DZK[k] * 0.1)
                            cf.help_t = 0.4f / logf((DZK[k] + DZK[k + 1] * 0.5f) / DZK[k] * 0.1f);
                        else
                            cf.help_t = 0.4f / logf(DZK[k] * 0.5f / z0);
                    } else {
                        cf.help_o = 0.4f / logf(DZK[k] * 0.5f / p.building_z0);
                    }
                }
            }
            // k-eps wall functions of the TKE back-substitution (TKE-prognostic-microscale.cs:278-338)
            if (p.turbulence_model == 2 && inner) {
                ColKE &ke = colke[c];
                const int k = KK + 1;
                if (k + 1 <= NKK + 1) {
                    if ((double)z0 >= (double)DZK[k] * 0.5) {
                        f |= F_GMODE1;
                        ke.gfac = 0.4 / std::log(((double)DZK[k] + (double)DZK[k + 1] * 0.5) / (double)z0);
                    } else {
                        ke.gfac = 0.4 / std::log((double)DZK[k] * 0.5 / (double)z0);
                    }
                }
                auto kwn = [&](int ii, int jj) { return s.cutk[ii * nj2 + jj] > 0 ? (int16_t)(kk(ii, jj) + 1) : (int16_t)-1; };
                ke.kw_e = kwn(i + 1, j); ke.kw_w = kwn(i - 1, j); ke.kw_n = kwn(i, j + 1); ke.kw_s = kwn(i, j - 1);
            }
            cfl[c] = f;
            vi_max = std::max(vi_max, VI);
            if ((f & F_ADV) && i >= 2 && i <= NII - 1 && j >= 2 && j <= NJJ - 1) {
                vi_min = std::min(vi_min, VI);
                if (p.turbulence_model == 1 && VI + 1 - p.simd_width < 1)
                    return fail(ctx, GRAL_EINVAL, "VerticalIndex below the SIMD width of the model-1 parity path");
            }
        }
    }
    if (vi_min == (1 << 20)) vi_min = 0;
    return GRAL_OK;
}

Geom make_geom(int ia, int ni, int ja, int nj) {
    Geom G;
    G.g.ia = ia; G.g.ni = std::max(ni, 0); G.g.ja = ja; G.g.nj = std::max(nj, 0);
    const int nd = (G.g.ni > 0 && G.g.nj > 0) ? G.g.ni + G.g.nj - 1 : 0;
    G.g.ndiag = nd;
    G.ds.assign(nd + 1, 0);
    for (int d = 0; d < nd; ++d) {
        const int lo = std::max(0, d - (G.g.nj - 1)), hi = std::min(d, G.g.ni - 1);
        G.ds[d + 1] = G.ds[d] + (hi - lo + 1);
    }
    return G;
}

int validate(gral_ctx *ctx, int n, const gral_params *p, const gral_static *s, const gral_fields *f) {
    if (!ctx) return GRAL_EINVAL;
    if (n < 1 || n > ctx->cap_batch) return fail(ctx, GRAL_EINVAL, "batch size outside 1..max_batch");
    if (!p || !s || !f) return fail(ctx, GRAL_EINVAL, "null argument");
    if (!s->kkart || !s->advdom || !s->cutk || !s->z0 || !s->dzk || !s->hokart)
        return fail(ctx, GRAL_EINVAL, "missing static array");
    const gral_params &p0 = p[0];
    if (p0.nii < 4 || p0.njj < 4 || p0.nkk < 3) return fail(ctx, GRAL_EINVAL, "grid too small");
    if (p0.nii > ctx->cap_nii || p0.njj > ctx->cap_njj || p0.nkk > ctx->cap_nkk || p0.kadvmax > ctx->cap_kadv)
        return fail(ctx, GRAL_EINVAL, "grid larger than the context capacity");
    if (p0.nii > 0xffff || p0.njj > 0xffff) return fail(ctx, GRAL_EINVAL, "grid dimension above 65535");
    if (p0.kadvmax < 2 || p0.kadvmax + 2 > KMAX_LEVELS || p0.kadvmax > p0.nkk)
        return fail(ctx, GRAL_EINVAL, "KADVMAX outside 2..62 or above NKK");
    if (p0.turbulence_model < 0 || p0.turbulence_model > 2) return fail(ctx, GRAL_EINVAL, "turbulence_model must be 0, 1 or 2");
    if (p0.turbulence_model == 1 && p0.simd_width != 8 && p0.simd_width != 16)
        return fail(ctx, GRAL_EINVAL, "simd_width must be 8 (Vector<float> path) or 16 (Vector512 path)");
    for (int b = 0; b < n; ++b) {
        const gral_params &q = p[b];
        if (q.nii != p0.nii || q.njj != p0.njj || q.nkk != p0.nkk || q.kadvmax != p0.kadvmax ||
            q.vert_cells_ff != p0.vert_cells_ff || q.turbulence_model != p0.turbulence_model ||
            q.simd_width != p0.simd_width || q.dxk != p0.dxk || q.dyk != p0.dyk ||
            q.iteration_steps_min != p0.iteration_steps_min || q.iteration_steps_max != p0.iteration_steps_max ||
            q.conv_cadence != p0.conv_cadence || q.relax != p0.relax || q.relaxp != p0.relaxp ||
            q.building_z0 != p0.building_z0 || q.coriolis != p0.coriolis)
            return fail(ctx, GRAL_EINVAL, "situations of a batch must share grid and solver controls");
        if (q.post_diagnostic != p0.post_diagnostic)
            return fail(ctx, GRAL_EINVAL, "post_diagnostic must be the same for every situation of a batch");
        if (q.conv_cadence < 1 || q.iteration_steps_max < 1) return fail(ctx, GRAL_EINVAL, "bad iteration controls");
        if (q.ref_i < 1 || q.ref_i > q.nii || q.ref_j < 1 || q.ref_j > q.njj)
            return fail(ctx, GRAL_EINVAL, "reference point outside the grid");
        if (!f[b].uk || !f[b].vk || !f[b].wk) return fail(ctx, GRAL_EINVAL, "null field");
        if (q.turbulence_model != 1 && (!f[b].turb || !f[b].tdiss))
            return fail(ctx, GRAL_EINVAL, "TURB/TDISS fields are required for turbulence_model 0 and 2");
        if (q.turbulence_model != 1 && q.turb_init == 0 && (!s->z0_init || !s->ob_init || !s->ust_init))
            return fail(ctx, GRAL_EINVAL, "z0_init/ob_init/ust_init are required to initialise TURB");
    }
    return GRAL_OK;
}

// The slab family's model-1 sweeps run on the strip schedule (pmode 1+v) rather than the
// diagonal-claim wavefront (pmode 0).
bool use_strips(const gral_ctx *ctx) { return !ctx->il && ctx->model == 1 && ctx->pmode > 0; }

}  // namespace

int gral::strip_variant_of(const gral_ctx *ctx) {
    return (ctx->pmode - 1 < strip_num_variants()) ? ctx->pmode - 1 : 0;
}

bool gral::fused_strips(const gral_ctx *ctx) {
    return use_strips(ctx) && ctx->pmode == 1 + strip_num_variants();
}

namespace {

// One SIMPLE iteration (PrognosticFlowfield.cs:584-1182), enqueued on st.
void launch_iteration(gral_ctx *ctx, cudaStream_t st) {
    const KArgs &a = ctx->ka;
    cudaMemsetAsync(ctx->counters.p, 0, 8 * kCounterSlots * sizeof(unsigned int), st);
    launch_bc(a, ctx->bc, st);
    if (use_strips(ctx)) {
        const int v = strip_variant_of(ctx);
        if (fused_strips(ctx)) {
            launch_fused_strip(a, ctx->fgeo, ctx->fstrip_grid, st);
        } else {
            launch_strip(PH_PRESSURE, a, ctx->geo_p.g, v, ctx->strip_grid[PH_PRESSURE], st);
            launch_velcorr(a, st);
            launch_average(a, st);
            launch_strip(PH_U, a, ctx->geo_u.g, v, ctx->strip_grid[PH_U], st);
        }
        launch_strip(PH_V, a, ctx->geo_v.g, v, ctx->strip_grid[PH_V], st);
        launch_strip(PH_W, a, ctx->geo_p.g, v, ctx->strip_grid[PH_W], st);
        launch_bookkeeping(a, st);
        return;
    }
    if (ctx->fused) {
        launch_fused_pvau(a, ctx->fgeo, ctx->fused_grid, st);
    } else {
        launch_gs(PH_PRESSURE, a, ctx->geo_p.g, ctx->grid_gs[PH_PRESSURE], st);
        launch_velcorr(a, st);
        launch_average(a, st);
        launch_gs(PH_U, a, ctx->geo_u.g, ctx->grid_gs[PH_U], st);
    }
    launch_gs(PH_V, a, ctx->geo_v.g, ctx->grid_gs[PH_V], st);
    launch_gs(PH_W, a, ctx->geo_p.g, ctx->grid_gs[PH_W], st);
    if (ctx->model == 2) launch_gs(PH_TKE, a, ctx->geo_p.g, ctx->grid_gs[PH_TKE], st);
    launch_bookkeeping(a, st);
}

// Grid sizes of the wavefront kernels for the current family and variant: every resident block
// slot of the GPU (the kernels are persistent and claim tasks).
// kernel launches of one SIMPLE iteration: 3 boundary kernels, one per Gauss-Seidel phase and
// group set, velocity correction, averages and bookkeeping
int launches_per_iteration(const gral_ctx *ctx) {
    const int gs = ctx->ka.group_set <= 0 ? ctx->ngroups : ctx->ka.group_set;
    const int sets = ctx->il ? (ctx->ngroups + gs - 1) / gs : 1;
    if (fused_strips(ctx)) return 3 + 3 + 1;
    if (use_strips(ctx)) return 3 + 4 + 3;
    if (ctx->fused) return 3 + 1 + 2 + 1;
    const int phases = (ctx->model == 2) ? 5 : 4;
    return 3 + phases * sets + 3;
}

int size_grids(gral_ctx *ctx) {
    const int kinds[5] = {PH_PRESSURE, PH_U, PH_V, PH_W, PH_TKE};
    const bool il = ctx->il;
    const int nkv = gs_num_variants();
    const int vv = il ? std::max(ctx->variant, 0) : 0;
    const int v = vv % nkv;                     // kernel variant
    const int gm = vv / nkv;                    // group-set mode: 0 all groups, 1 two, 2 one
    ctx->ka.group_set = (gm == 0) ? 0 : (gm == 1 ? 2 : 1);
    ctx->ka.group_lo = 0;
    ctx->ka.group_n = ctx->ngroups;
    ctx->ka.ctr_slot = 0;
    if (il && (ctx->ngroups + std::max(ctx->ka.group_set, 1) - 1) / std::max(ctx->ka.group_set, 1) > kCounterSlots)
        ctx->ka.group_set = 0;
    // Plain family: enough warps for `lookahead` diagonals of the average wavefront width, so a
    // warp's pre-wait work runs a few diagonals ahead of the front without thousands of warps
    // polling far-future flags (0 = as many as fit).
    const double diag_width = (double)ctx->nb * (double)(ctx->nii - 3) * (double)(ctx->njj - 3) /
                              (double)std::max(1, ctx->nii + ctx->njj - 7);
    const int warps_per_block = gs_block_threads(false, 0) / 32;
    for (int q = 0; q < 5; ++q) {
        int bps = 0;
        CK(gs_occupancy(il, kinds[q], ctx->model, ctx->ka.simd, ctx->ks, v, &bps));
        long long blocks = (long long)std::max(1, bps) * ctx->num_sms;
        const int la = (kinds[q] == PH_PRESSURE) ? ctx->lookahead_p : ctx->lookahead;
        const long long want_blocks = (long long)std::ceil(la * diag_width / (double)warps_per_block);
        if (!il && la > 0) blocks = std::max<long long>(ctx->num_sms, std::min(blocks, want_blocks));
        ctx->grid_gs[kinds[q]] = (int)blocks;
    }
    if (use_strips(ctx)) {
        // one block per strip at most: the strip kernels are persistent and claim strips in order
        const int sv = strip_variant_of(ctx);
        const Geom *gk[4] = {&ctx->geo_p, &ctx->geo_u, &ctx->geo_v, &ctx->geo_p};
        for (int q = 0; q < 4; ++q) {
            int bps = 0;
            CK(strip_occupancy(kinds[q], sv, &bps));
            const int sr = strip_rows(sv);
            const long long strips = (long long)((gk[q]->g.ni + sr - 1) / sr) * ctx->nb;
            ctx->strip_grid[kinds[q]] =
                (int)std::max<long long>(1, std::min<long long>((long long)std::max(1, bps) * ctx->num_sms, strips));
        }
        if (fused_strips(ctx)) {
            int bps = 0;
            CK(fused_strip_occupancy(&bps));
            const long long claims = (long long)fused_strip_claims(ctx->geo_p.g) * ctx->nb;
            ctx->fstrip_grid = (int)std::max<long long>(1, std::min<long long>((long long)std::max(1, bps) * ctx->num_sms, claims));
        }
    }
    const int warps = ctx->grid_gs[PH_PRESSURE] * gs_block_threads(il, v) / 32;
    const long long per_diag = (long long)(il ? ctx->ngroups : ctx->nb) * std::min(ctx->nii, ctx->njj);
    ctx->ka.chunk = il ? 1 : (int)std::max(1LL, std::min(16LL, per_diag / (2LL * warps)));
    ctx->ka.variant = v;
    return GRAL_OK;
}

int build_graph(gral_ctx *ctx) {
    if (ctx->graph) { cudaGraphExecDestroy(ctx->graph); ctx->graph = nullptr; }
    cudaGraph_t g = nullptr;
    cudaStream_t st = ctx->stream;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    launch_iteration(ctx, st);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (e != cudaSuccess) return fail(ctx, GRAL_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&ctx->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(ctx, GRAL_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return GRAL_OK;
}

// Autotuner of the batched family: every launch variant gives bit-identical results, so the first
// iterations of the solve each run one variant, timed with CUDA events, and the fastest is kept
// and captured into the iteration graph.  Runs only when enough iterations remain before the
// first convergence test; otherwise variant 0 is used.
int tune_plain(gral_ctx *ctx);

int tune_variants(gral_ctx *ctx) {
    if (!ctx->il) return tune_plain(ctx);
    if (ctx->variant >= 0) return GRAL_OK;
    const int nv = gs_num_variants() * (ctx->ngroups > 2 ? 3 : (ctx->ngroups > 1 ? 2 : 1));
    const int first_stop = std::min(((ctx->it_host + ctx->cadence - 1) / ctx->cadence) * ctx->cadence, ctx->it_max);
    if (ctx->forced_variant >= 0 && ctx->forced_variant < nv) {
        ctx->variant = ctx->forced_variant;
    } else if (first_stop - ctx->it_host + 1 > nv) {
        cudaStream_t st = ctx->stream;
        float best = 1e30f;
        int best_v = 0;
        for (int v = 0; v < nv; ++v) {
            ctx->variant = v;
            int rc = size_grids(ctx);
            if (rc != GRAL_OK) return rc;
            CK(cudaEventRecord(ctx->ev[2], st));
            launch_iteration(ctx, st);
            CK(cudaEventRecord(ctx->ev[3], st));
            CK(cudaEventSynchronize(ctx->ev[3]));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
            if (v < 64) ctx->tune_ms[v] = ms;
            if (ms < best) { best = ms; best_v = v; }
            ctx->it_host++;
        }
        ctx->variant = best_v;
    } else {
        ctx->variant = 0;
    }
    int rc = size_grids(ctx);
    if (rc != GRAL_OK) return rc;
    return build_graph(ctx);
}

// Autotuner of the slab family (model 1): the diagonal-claim wavefront and every strip variant
// give bit-identical results, so before the first convergence test each mode runs two live
// iterations (the first warms the kernels up), the second timed with CUDA events, and the fastest
// mode is kept and captured into the iteration graph.  Without room for the trials the default
// mode is kept.
constexpr int kDefaultPlainMode = 1;   // strips of 4 rows, 4 warps per row (fastest on the 400x400 grid)

}  // namespace

int gral::plain_schedule_default(gral_ctx *ctx) {
    const int nv = 2 + strip_num_variants();
    ctx->pmode = (ctx->model != 1) ? 0 : ((ctx->forced_pmode >= 0 && ctx->forced_pmode < nv) ? ctx->forced_pmode : kDefaultPlainMode);
    return size_grids(ctx);
}

namespace {

int tune_plain(gral_ctx *ctx) {
    if (ctx->pmode >= 0) return GRAL_OK;
    const int nv = 2 + strip_num_variants();
    const int first_stop = std::min(((ctx->it_host + ctx->cadence - 1) / ctx->cadence) * ctx->cadence, ctx->it_max);
    if (ctx->model != 1) {
        ctx->pmode = 0;
    } else if (ctx->forced_pmode >= 0 && ctx->forced_pmode < nv) {
        ctx->pmode = ctx->forced_pmode;
    } else if (first_stop - ctx->it_host + 1 > 2 * nv) {
        cudaStream_t st = ctx->stream;
        float best = 1e30f;
        int best_v = 0;
        for (int v = 0; v < nv; ++v) {
            ctx->pmode = v;
            int rc = size_grids(ctx);
            if (rc != GRAL_OK) return rc;
            launch_iteration(ctx, st);
            ctx->it_host++;
            CK(cudaEventRecord(ctx->ev[2], st));
            launch_iteration(ctx, st);
            CK(cudaEventRecord(ctx->ev[3], st));
            CK(cudaEventSynchronize(ctx->ev[3]));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
            if (v < 16) ctx->ptune_ms[v] = ms;
            if (ms < best) { best = ms; best_v = v; }
            ctx->it_host++;
        }
        ctx->pmode = best_v;
    } else {
        ctx->pmode = kDefaultPlainMode;
    }
    int rc = size_grids(ctx);
    if (rc != GRAL_OK) return rc;
    return build_graph(ctx);
}

}  // namespace

// DiagnosticFlowfield.Calculate and the final vertical velocity (MicroscaleFlat.cs:383-462) on the
// full-height staging fields of every situation, after the scatter of the prognostic result.
int run_diagnostic(gral_ctx *ctx) {
    cudaStream_t st = ctx->stream;
    const int nk2 = ctx->nkk + 2;
    KArgs kd = ctx->ka;
    kd.il = 0;
    kd.ks = nk2;
    kd.uk = ctx->sg.uk; kd.vk = ctx->sg.vk; kd.wk = ctx->sg.wk;
    kd.dpm = ctx->ddpm.p;
    kd.flags = ctx->dflags.p;
    kd.chunk = 1;
    DiagTabs t;
    t.dzk = ctx->dtab.p; t.app = ctx->dtab.p + nk2; t.atp = ctx->dtab.p + 2 * nk2;
    t.abp0 = ctx->dtab.p + 3 * nk2; t.abp1 = ctx->dtab.p + 4 * nk2;
    t.dtime = ctx->ddt.p;
    launch_diag_dtime(kd, ctx->params[0].kadvmax, ctx->ddt.p, st);
    CK(cudaMemsetAsync(ctx->ddpm.p, 0, (size_t)ctx->nb * ctx->ncols * nk2 * sizeof(float), st));
    CK(cudaMemsetAsync(ctx->dflags.p, 0, (size_t)ctx->nb * ctx->ncols * sizeof(int), st));
    for (int d = 1; d <= 10; ++d) {                    // Iterations = 10 after a prognostic solve (:33-37)
        kd.diag_iter = d;
        CK(cudaMemsetAsync(ctx->counters.p, 0, 8 * sizeof(unsigned int), st));
        launch_diag_pressure(kd, ctx->geo_p.g, t, ctx->diag_grid, st);
        launch_diag_velcorr(kd, t, st);
    }
    launch_diag_wfinal(kd, t, st);
    CK(cudaGetLastError());
    return GRAL_OK;
}

extern "C" {

int gral_prog_version(void) { return GRAL_PROG_ABI_VERSION; }

int gral_prog_create(int32_t nii, int32_t njj, int32_t nkk, int32_t kadvmax, int32_t max_batch, gral_ctx **out) {
    if (!out || nii < 4 || njj < 4 || nkk < 3 || kadvmax < 2 || max_batch < 1) return GRAL_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return GRAL_ENODEV;
    gral_ctx *ctx = new gral_ctx();
    ctx->cap_nii = nii; ctx->cap_njj = njj; ctx->cap_nkk = nkk; ctx->cap_kadv = kadvmax; ctx->cap_batch = max_batch;
    cudaGetDevice(&ctx->device);
    // GRAL_PROG_LAYOUT=interleaved|slab forces the kernel family regardless of the batch size.
    if (const char *lay = std::getenv("GRAL_PROG_LAYOUT")) {
        if (std::strcmp(lay, "interleaved") == 0) ctx->il_min_batch = 1;
        else if (std::strcmp(lay, "slab") == 0) ctx->il_min_batch = 1 << 30;
    }
    if (const char *v = std::getenv("GRAL_PROG_BATCH_VARIANT")) ctx->forced_variant = std::atoi(v);
    if (const char *v = std::getenv("GRAL_PROG_PLAIN_MODE")) ctx->forced_pmode = std::atoi(v);
    if (const char *v = std::getenv("GRAL_PROG_LOOKAHEAD")) ctx->lookahead = std::max(0, std::atoi(v));
    if (const char *v = std::getenv("GRAL_PROG_LOOKAHEAD_P")) ctx->lookahead_p = std::max(0, std::atoi(v));
    if (const char *v = std::getenv("GRAL_PROG_LOOKAHEAD_F")) ctx->lookahead_f = std::max(0, std::atoi(v));
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device);
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) { delete ctx; return GRAL_ECUDA; }
    for (auto &e : ctx->ev)
        if (cudaEventCreate(&e) != cudaSuccess) { delete ctx; return GRAL_ECUDA; }
    *out = ctx;
    return GRAL_OK;
}

const char *gral_prog_last_error(gral_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void gral_prog_destroy(gral_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete ctx;
}

int gral_prog_load(gral_ctx *ctx, int32_t n, const gral_params *p, const gral_static *s, gral_fields *f) {
    int rc = validate(ctx, n, p, s, f);
    if (rc != GRAL_OK) return rc;
    CK(cudaSetDevice(ctx->device));
    const gral_params &p0 = p[0];
    const int NII = p0.nii, NJJ = p0.njj, NKK = p0.nkk, nj2 = NJJ + 2, ncols = (NII + 2) * nj2;
    const int nk2 = NKK + 2;
    const int ks = ((p0.kadvmax + 2) + 7) / 8 * 8;
    // Layout: batches of at least il_min_batch situations use the interleaved layout and the
    // lane-per-situation kernels; smaller ones the slab layout and the warp-per-column kernels.
    const bool il = n >= ctx->il_min_batch;
    const int ngroups = (n + 31) / 32;
    ctx->il = il;
    ctx->ngroups = ngroups;
    ctx->loaded = false;
    ctx->stored = false;
    ctx->h_kkart.assign(s->kkart, s->kkart + (size_t)ncols);
    ctx->nii = NII; ctx->njj = NJJ; ctx->nkk = NKK; ctx->ks = ks; ctx->nb = n; ctx->ncols = ncols; ctx->nj2 = nj2;
    ctx->model = p0.turbulence_model;
    ctx->params.assign(p, p + n);
    ctx->fields.assign(f, f + n);
    ctx->it_min = p0.iteration_steps_min; ctx->it_max = p0.iteration_steps_max; ctx->cadence = p0.conv_cadence;

    // ---- per-column constants ----
    std::vector<ColMeta> meta;
    std::vector<uint32_t> cfl;
    std::vector<ColF> colf;
    std::vector<ColKE> colke;
    int vi_min = 0, vi_max = 0;
    rc = build_meta(ctx, p0, *s, meta, cfl, colf, colke, vi_min, vi_max);
    if (rc != GRAL_OK) return rc;
    if (vi_max + 1 >= ks) return fail(ctx, GRAL_EINVAL, "VerticalIndex above KADVMAX");

    // ---- row-carry writers of the pressure sweep ----
    // A column of the pressure sweep row j writes the carry at levels max(KKART, vi_min) < k <= VI
    // (PrognosticFlowfield.cs:865-880); the column reading level VI+1 gets it from the last such
    // writer before it in sweep order, or the zeroed buffer when there is none.
    std::vector<short2> rcw(ncols, make_short2(-1, -1));
    {
        std::vector<int> last(ks + 1);
        for (int dir = 0; dir < 2; ++dir)
            for (int j = 2; j <= NJJ - 1; ++j) {
                std::fill(last.begin(), last.end(), -1);
                for (int q = 2; q <= NII - 1; ++q) {
                    const int i = (dir == 0) ? q : NII + 1 - q;
                    const int c = i * nj2 + j;
                    const int VI = meta[c].vi, KK = meta[c].kkart;
                    const short w = (short)((VI + 1 <= ks) ? last[VI + 1] : -1);
                    if (dir == 0) rcw[c].x = w; else rcw[c].y = w;
                    if (cfl[c] & F_ADV)
                        for (int k = std::max(KK, vi_min) + 1; k <= VI && k <= ks; ++k) last[k] = i;
                }
            }
    }

    // ---- level tables (float, reference expressions) ----
    const float DXK = p0.dxk, DYK = p0.dyk, AREA = DXK * DYK;
    std::vector<float> tab(5 * ks, 0.0f);   // dzk, hokart, app, abp, atp
    for (int k = 0; k < ks; ++k) {
        tab[k] = (k < nk2) ? s->dzk[k] : 0.0f;
        tab[ks + k] = (k < nk2) ? s->hokart[k] : 0.0f;
    }
    for (int k = 1; k < ks - 1 && k + 1 < nk2; ++k) {                    // PrognosticFlowfield.cs:857-866
        const float *DZ = s->dzk;
        tab[2 * ks + k] = 2.0f * (DYK * DZ[k] / DXK + DXK * DZ[k] / DYK + AREA / DZ[k]);
        tab[3 * ks + k] = (k > 1) ? AREA / (0.5f * (DZ[k - 1] + DZ[k])) : AREA / DZ[k];
        tab[4 * ks + k] = AREA / (0.5f * (DZ[k + 1] + DZ[k]));
    }

    // ---- initial fields built on the device (gral_prog_load_flat) ----
    // The staging of every situation is filled by the flat-terrain set-up kernels; the six values
    // of the reference column that the scalars below need come back to the host.
    if (ctx->flat_met) {
        const size_t ssz0 = (size_t)ncols * nk2;
        CK(ctx->stage.ensure(ssz0 * ((ctx->model != 1) ? 5 : 3) * n));
        cudaStream_t st0 = ctx->stream;
        PrepBufs &pb = ctx->prep;
        CK(pb.cutk.ensure(ncols));
        CK(cudaMemcpyAsync(pb.cutk.p, s->cutk, ncols * sizeof(float), cudaMemcpyHostToDevice, st0));
        if (ctx->flat_grid->near_wall == 1) {
            CK(pb.adv.ensure(ncols));
            CK(cudaMemcpyAsync(pb.adv.p, s->advdom, ncols, cudaMemcpyHostToDevice, st0));
        }
        float *u0 = ctx->stage.p, *v0 = u0 + ssz0 * n, *w0 = v0 + ssz0 * n;
        ctx->h_ref.assign(6 * (size_t)n, 0.0f);
        for (int b = 0; b < n; ++b) {
            int *dk = nullptr;
            const int frc = flat_fill(ctx, ctx->flat_grid, pb.cutk.p, pb.adv.p, s->dzk, s->hokart, &ctx->flat_met[b],
                                      u0 + ssz0 * b, v0 + ssz0 * b, w0 + ssz0 * b, &dk, false);
            if (frc != GRAL_OK) return frc;
            const int rx = p[b].ref_i, ry = p[b].ref_j;
            auto at = [&](int i, int j, int k) { return ((size_t)i * nj2 + j) * nk2 + k; };
            const float *src[6] = {u0 + ssz0 * b + at(rx, ry, NKK - 1), v0 + ssz0 * b + at(rx, ry, NKK - 1),
                                   u0 + ssz0 * b + at(rx, ry, p[b].kadvmax), v0 + ssz0 * b + at(rx, ry, p[b].kadvmax),
                                   u0 + ssz0 * b + at(rx + 1, ry, NKK - 1), v0 + ssz0 * b + at(rx, ry + 1, NKK - 1)};
            for (int q = 0; q < 6; ++q)
                CK(cudaMemcpyAsync(&ctx->h_ref[6 * (size_t)b + q], src[q], sizeof(float), cudaMemcpyDeviceToHost, st0));
        }
        CK(cudaStreamSynchronize(st0));
    }

    // ---- per-situation scalars (:146-163, 231-240, 406-407) ----
    ctx->h_sit.assign(n, SitDev{});
    std::vector<float> ap0((size_t)n * ks, 0.0f);
    for (int b = 0; b < n; ++b) {
        const gral_params &q = p[b];
        const int rx = q.ref_i, ry = q.ref_j;
        auto I3 = [&](int i, int j, int k) { return ((size_t)i * nj2 + j) * nk2 + k; };
        // U, V of the reference column at NKK-1 and KADVMAX, U east and V north of it at NKK-1
        float rv[6];
        if (ctx->flat_met) {
            for (int r = 0; r < 6; ++r) rv[r] = ctx->h_ref[6 * (size_t)b + r];
        } else {
            const float *UK = f[b].uk, *VK = f[b].vk;
            rv[0] = UK[I3(rx, ry, NKK - 1)];
            rv[1] = VK[I3(rx, ry, NKK - 1)];
            rv[2] = UK[I3(rx, ry, q.kadvmax)];
            rv[3] = VK[I3(rx, ry, q.kadvmax)];
            rv[4] = UK[I3(rx + 1, ry, NKK - 1)];
            rv[5] = VK[I3(rx, ry + 1, NKK - 1)];
        }
        const float u1 = rv[0], v1 = rv[1];
        float topwind = (float)std::sqrt((double)(u1 * u1 + v1 * v1));
        topwind = net_max(topwind, 0.01f);
        const float u2 = rv[2], v2 = rv[3];
        float DT = 0.5f * net_min(DXK, s->dzk[1]) / net_max(0.01f, sqrtf(u2 * u2 + v2 * v2));
        DT = net_min(DT, 5.0f);
        for (int k = 1; k <= q.kadvmax; ++k) ap0[(size_t)b * ks + k] = AREA * s->dzk[k] / DT;
        SitDev &S = ctx->h_sit[b];
        S.frund = (double)((q.turbulence_model == 2 ? 10000 : 8000) / topwind);
        S.rfrund = 1.0 / S.frund;
        S.rcp_ok = 0;                 // set on the device by the check after the upload
        S.conv_threshold = q.conv_threshold;
        S.dtime = DT;
        S.topwind = topwind;
        const bool alloc = (cfl[rx * nj2 + ry] & F_ALLOC3) != 0;
        S.ug = alloc ? 0.5f * (rv[0] + rv[4]) : 0.0f;
        S.vg = alloc ? 0.5f * (rv[1] + rv[5]) : 0.0f;
        S.it = 1;
        S.active = 1;
        S.it_min = q.iteration_steps_min;
        S.it_max = q.iteration_steps_max;
        S.cadence = q.conv_cadence;
        S.quantise = q.quantise;
        S.potdtdz = q.potdtdz;
        S.std_dev_v = q.std_dev_v;
        S.v0_1 = q.v0_1;
        S.turb_init = q.turb_init;
    }
    // vertical-variance term of the TURB initialisation per situation and column
    // (PrognosticFlowfield.cs:488-495), float arithmetic with libm powf as the reference
    std::vector<float> varw;
    if (ctx->model != 1) {
        varw.assign((size_t)n * ncols, 0.0f);
        for (int b = 0; b < n; ++b) {
            const gral_params &q = p[b];
            if (q.turb_init) continue;
            std::map<std::pair<float, float>, float> memo;
            for (int i = 1; i <= NII; ++i)
                for (int j = 1; j <= NJJ; ++j) {
                    const int c = i * nj2 + j;
                    const float ObLength = s->ob_init[c], ust = s->ust_init[c];
                    auto key = std::make_pair(ObLength, ust);
                    auto it = memo.find(key);
                    float vw;
                    if (it != memo.end()) {
                        vw = it->second;
                    } else {
                        if (ObLength < 0) {
                            const float t = 1.15f + 0.1f * powf(q.bd_lay_height / (-ObLength), 0.67f);
                            vw = (ust * ust) * (t * t) * (q.std_dev_w * q.std_dev_w);
                        } else {
                            const float t = ust * q.std_dev_w * 1.25f;
                            vw = t * t;
                        }
                        memo.emplace(key, vw);
                    }
                    varw[(size_t)b * ncols + c] = vw;
                }
        }
    }

    // ---- boundary-condition event lists ----
    std::vector<int> wptr(nj2 + 1, 0), wev, sptr(NII + 3, 0), sev;
    auto adv = [&](int i, int j) { return s->advdom[i * nj2 + j]; };
    for (int j = 0; j <= NJJ + 1; ++j) {
        wptr[j] = (int)wev.size();
        if (j >= 2 && j <= NJJ)
            for (int i = 3; i <= NII - 1; ++i) {
                if (adv(i, j) != 1) continue;
                const bool iM = (adv(i - 1, j) < 1) || (i == 3), iP = (adv(i + 1, j) < 1) || (i == NII - 1);
                if (iM || iP) wev.push_back(i | (iM << 16) | (iP << 17));
            }
    }
    wptr[nj2] = (int)wev.size();
    for (int i = 0; i <= NII + 1; ++i) {
        sptr[i] = (int)sev.size();
        if (i >= 2 && i <= NII)
            for (int j = 3; j <= NJJ - 1; ++j) {
                if (adv(i, j) != 1) continue;
                const bool jM = (adv(i, j - 1) < 1) || (j == 3), jP = (adv(i, j + 1) < 1) || (j == NJJ - 1);
                if (jM || jP) sev.push_back(j | (jM << 16) | (jP << 17));
            }
    }
    sptr[NII + 2] = (int)sev.size();

    // ---- sweeps ----
    ctx->geo_p = make_geom(2, NII - 2, 2, NJJ - 2);
    ctx->geo_u = make_geom(3, NII - 3, 2, NJJ - 2);
    ctx->geo_v = make_geom(2, NII - 2, 3, NJJ - 3);

    // ---- device memory ----
    const size_t units = il ? (size_t)ngroups * 32 : (size_t)n;     // situation slots
    const size_t fsz = units * ncols * ks;
    const int nfields = 10;
    const size_t ssz = (size_t)ncols * nk2;
    const int nstage = (ctx->model != 1) ? 5 : 3;
    const int tcap = ctx->it_max;
    CK(ctx->slab.ensure(fsz * nfields));
    CK(ctx->stage.ensure(ssz * nstage * n));
    CK(ctx->meta.ensure(ncols));
    CK(ctx->cflags.ensure(ncols));
    CK(ctx->colf.ensure(ncols));
    CK(ctx->rcw.ensure(ncols));
    if (ctx->model != 1) {
        CK(ctx->colke.ensure(ncols));
        CK(ctx->varw.ensure((size_t)n * ncols));
        CK(ctx->z0i.ensure(ncols));
    }
    CK(ctx->tables.ensure(5 * ks));
    CK(ctx->ap0.ensure((size_t)n * ks));
    CK(ctx->sit.ensure(n));
    const size_t flag_units = il ? (size_t)ngroups : (size_t)n;
    CK(ctx->flags.ensure(flag_units * ncols));
    CK(ctx->rowcarry.ensure(units * nj2 * 2 * ks));
    CK(ctx->trace.ensure((size_t)n * tcap));
    CK(ctx->misc.ensure(3 + n));                      // err, nact, it, act[n]
    CK(ctx->counters.ensure(8 * kCounterSlots));
    CK(ctx->counts.ensure(4 * (size_t)n));
    const size_t dsz = ctx->geo_p.ds.size() + ctx->geo_u.ds.size() + ctx->geo_v.ds.size();
    CK(ctx->diag.ensure(dsz));
    CK(ctx->bcl.ensure(wptr.size() + wev.size() + sptr.size() + sev.size() + 4));
    const bool has_veg = s->veg && s->veg_mask;
    if (has_veg) CK(ctx->veg.ensure((size_t)ncols * ks));

    cudaStream_t st = ctx->stream;
    CK(cudaEventRecord(ctx->ev[0], st));
    float *slab = ctx->slab.p;
    KArgs &a = ctx->ka;
    a = KArgs{};
    a.nii = NII; a.njj = NJJ; a.nkk = NKK; a.ks = ks; a.nj2 = nj2; a.ncols = ncols; a.nb = n;
    a.il = il ? 1 : 0;
    a.ngroups = ngroups;
    a.dxk = DXK; a.dyk = DYK; a.areaxy = AREA;
    a.relax = p0.relax; a.relaxp = p0.relaxp; a.coriolis = p0.coriolis;
    a.vishmin = (p0.turbulence_model == 2) ? 0.01f : 0.0f;
    a.simd = p0.simd_width;
    a.model = p0.turbulence_model;
    a.colke = (ctx->model == 2) ? ctx->colke.p : nullptr;
    a.building_z0 = p0.building_z0;
    a.ustern_fx = (float)(0.4 / std::log((double)DXK * 0.5 / (double)p0.building_z0));   // :515
    a.meta = ctx->meta.p; a.cflags = ctx->cflags.p; a.colf = ctx->colf.p;
    a.dzk = ctx->tables.p; a.hokart = ctx->tables.p + ks;
    a.app = ctx->tables.p + 2 * ks; a.abp = ctx->tables.p + 3 * ks; a.atp = ctx->tables.p + 4 * ks;
    a.veg = has_veg ? ctx->veg.p : nullptr;
    a.sit = ctx->sit.p;
    a.ap0 = ctx->ap0.p;
    float **fp[10] = {&a.uk, &a.vk, &a.wk, &a.dpm, &a.dpmnew, &a.uks, &a.vks, &a.wks, &a.turb, &a.tdiss};
    for (int q = 0; q < nfields; ++q) *fp[q] = slab + fsz * q;
    a.flags = ctx->flags.p;
    a.counters = ctx->counters.p;
    a.rowcarry = ctx->rowcarry.p;
    a.rcw = ctx->rcw.p;
    a.err = ctx->misc.p;
    a.nact = ctx->misc.p + 1;
    a.it_global = ctx->misc.p + 2;
    a.act = ctx->misc.p + 3;
    // bound of every device-side spin wait (GRAL_PROG_WAIT_NS overrides it, e.g. to exercise the
    // timeout path: the waiting kernel sets the error word and returns, the context stays usable)
    a.wait_limit_ns = 2000000000ull;
    if (const char *v = std::getenv("GRAL_PROG_WAIT_NS")) a.wait_limit_ns = std::strtoull(v, nullptr, 10);
    a.trace = ctx->trace.p;
    a.trace_cap = tcap;
    a.vi_min = vi_min;

    Staging &sg = ctx->sg;
    sg.stride = ssz;
    sg.uk = ctx->stage.p;
    sg.vk = sg.uk + ssz * n;
    sg.wk = sg.vk + ssz * n;
    sg.turb = (nstage == 5) ? sg.wk + ssz * n : nullptr;
    sg.tdiss = (nstage == 5) ? sg.turb + ssz * n : nullptr;
    sg.stride = ssz;
    // situation b's staging block is at sg.X + b*ssz: fields are grouped per field, per situation.

    // geometry tables
    int *dp = ctx->diag.p;
    auto put_geom = [&](Geom &G) {
        G.g.diag_start = dp;
        cudaMemcpyAsync(dp, G.ds.data(), G.ds.size() * sizeof(int), cudaMemcpyHostToDevice, st);
        dp += G.ds.size();
    };
    put_geom(ctx->geo_p);
    put_geom(ctx->geo_u);
    put_geom(ctx->geo_v);

    ctx->fgeo.gp = ctx->geo_p.g;     // also read by the fused strip launch
    ctx->fgeo.gu = ctx->geo_u.g;
    // task list of the fused pressure/velcorr/average/U wavefront: step s holds pressure diagonal
    // s, velocity-correction diagonal s-1, averages s-2 and U-diagonal s-5 (P-diagonal s-4)
    {
        const char *fz = std::getenv("GRAL_PROG_FUSE");
        ctx->fused = !il && ctx->model == 1 && !(fz && std::atoi(fz) == 0);
        if (ctx->fused) {
            const Geom &gp = ctx->geo_p, &gu = ctx->geo_u;
            const int DP = gp.g.ndiag, DU = gu.g.ndiag;
            std::vector<int> start(1, 0), code;
            auto add = [&](int kind, const Geom &G, int d) {
                code.push_back(kind | (d << 3));
                start.push_back(start.back() + (G.ds[d + 1] - G.ds[d]));
            };
            // U trails the pressure by lag_u >= 4 P-diagonals (its averages' neighbourhood must be
            // complete); more lag lets its pre-wait work start before its U predecessors finish
            int lag_u = 16;
            if (const char *v = std::getenv("GRAL_PROG_FUSE_LAG")) lag_u = std::max(4, std::atoi(v));
            const int steps = std::max(DP + 2, DU + lag_u + 1);
            for (int q = 0; q < steps; ++q) {
                if (q < DP) add(PH_PRESSURE, gp, q);
                if (q - 1 >= 0 && q - 1 < DP) add(PH_VC, gp, q - 1);
                if (q - 2 >= 0 && q - 2 < DP) add(PH_AV, gp, q - 2);
                const int du = q - lag_u - 1;               // U-diagonal du is P-diagonal du + 1
                if (du >= 0 && du < DU) add(PH_U, gu, du);
            }
            CK(ctx->fseg.ensure(start.size() + code.size()));
            CK(cudaMemcpyAsync(ctx->fseg.p, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(ctx->fseg.p + start.size(), code.data(), code.size() * sizeof(int),
                               cudaMemcpyHostToDevice, st));
            ctx->fgeo.seg_start = ctx->fseg.p;
            ctx->fgeo.seg_code = ctx->fseg.p + start.size();
            ctx->fgeo.nseg = (int)code.size();
            ctx->fgeo.gp = gp.g;
            ctx->fgeo.gu = gu.g;
            int bps = 0;
            CK(fused_occupancy(&bps));
            const double width = (double)n * (NII - 3) * (NJJ - 3) / std::max(1, NII + NJJ - 7);
            const long long want = (long long)std::ceil(ctx->lookahead_f * 2.0 * width / 4.0);
            ctx->fused_grid = (int)std::max<long long>(ctx->num_sms,
                                                       std::min<long long>((long long)std::max(1, bps) * ctx->num_sms, want));
        }
    }
    int *bp = ctx->bcl.p;
    auto put_ints = [&](const std::vector<int> &v) {
        int *dst = bp;
        if (!v.empty()) cudaMemcpyAsync(bp, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice, st);
        bp += v.size() + 1;
        return (const int *)dst;
    };
    ctx->bc.we_ptr = put_ints(wptr);
    ctx->bc.we_ev = put_ints(wev);
    ctx->bc.sn_ptr = put_ints(sptr);
    ctx->bc.sn_ev = put_ints(sev);

    CK(cudaMemcpyAsync(ctx->meta.p, meta.data(), ncols * sizeof(ColMeta), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->cflags.p, cfl.data(), ncols * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->colf.p, colf.data(), ncols * sizeof(ColF), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->rcw.p, rcw.data(), ncols * sizeof(short2), cudaMemcpyHostToDevice, st));
    ctx->post_diag = p0.post_diagnostic != 0;
    if (ctx->post_diag) {
        // full-height level tables of DiagnosticFlowfield.cs:124-138 (float, the reference's
        // expressions): dzk, app, atp, abp0 (k = KKART+1), abp1 (k > KKART+1)
        const float *DZK = s->dzk;
        std::vector<float> dt(5 * (size_t)nk2, 0.0f);
        for (int k = 0; k < nk2; ++k) dt[k] = DZK[k];
        for (int k = 1; k <= NKK - 1; ++k) {
            dt[nk2 + k] = 2 * (DYK * DZK[k] / DXK + DXK * DZK[k] / DYK + DXK * DYK / DZK[k]);
            dt[2 * nk2 + k] = (DXK * DYK) / (0.5F * (DZK[k + 1] + DZK[k]));
            dt[3 * nk2 + k] = DXK * DYK / DZK[k];
            dt[4 * nk2 + k] = DXK * DYK / (0.5F * (DZK[k - 1] + DZK[k]));
        }
        CK(ctx->dtab.ensure(dt.size()));
        CK(ctx->ddpm.ensure((size_t)n * ncols * nk2));
        CK(ctx->dflags.ensure((size_t)n * ncols));
        CK(ctx->ddt.ensure(n));
        CK(cudaMemcpyAsync(ctx->dtab.p, dt.data(), dt.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        CK(diag_prepare(nk2));
        int bps = 0;
        CK(diag_occupancy(nk2, &bps));
        const double width = (double)n * (NII - 3) * (NJJ - 3) / std::max(1, NII + NJJ - 7);
        ctx->diag_grid = (int)std::max<long long>(ctx->num_sms, std::min<long long>((long long)std::max(1, bps) * ctx->num_sms,
                                                  (long long)std::ceil(8 * width / 4)));
    }
    if (ctx->model != 1) {
        CK(cudaMemcpyAsync(ctx->colke.p, colke.data(), ncols * sizeof(ColKE), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->varw.p, varw.data(), varw.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        if (s->z0_init) CK(cudaMemcpyAsync(ctx->z0i.p, s->z0_init, ncols * sizeof(float), cudaMemcpyHostToDevice, st));
        else CK(cudaMemsetAsync(ctx->z0i.p, 0, ncols * sizeof(float), st));
    }
    CK(cudaMemcpyAsync(ctx->tables.p, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->ap0.p, ap0.data(), ap0.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->sit.p, ctx->h_sit.data(), n * sizeof(SitDev), cudaMemcpyHostToDevice, st));
    bool any_quant = false;
    for (int b = 0; b < n; ++b) any_quant |= ctx->h_sit[b].quantise != 0;
    if (any_quant) {
        CK(cudaMemsetAsync(ctx->counts.p, 0, n * sizeof(int), st));
        launch_rcp_check(ctx->ka, ctx->counts.p, st);
    }
    ctx->h_act.resize(3 + n);
    ctx->h_act[0] = 0;
    ctx->h_act[1] = n;
    ctx->h_act[2] = 1;
    for (int b = 0; b < n; ++b) ctx->h_act[3 + b] = b;
    CK(cudaMemcpyAsync(ctx->misc.p, ctx->h_act.data(), (3 + n) * sizeof(int), cudaMemcpyHostToDevice, st));
    if (has_veg) {
        std::vector<float> vs((size_t)ncols * ks, 0.0f);
        for (int c = 0; c < ncols; ++c)
            for (int k = 0; k < ks && k < nk2; ++k) vs[(size_t)c * ks + k] = s->veg[(size_t)c * nk2 + k];
        CK(cudaMemcpyAsync(ctx->veg.p, vs.data(), vs.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
    CK(cudaMemsetAsync(slab, 0, fsz * nfields * sizeof(float), st));
    CK(cudaMemsetAsync(ctx->flags.p, 0, flag_units * ncols * sizeof(int), st));
    CK(cudaMemsetAsync(ctx->rowcarry.p, 0, units * nj2 * 2 * ks * sizeof(float), st));
    CK(cudaMemsetAsync(ctx->trace.p, 0, (size_t)n * tcap * sizeof(float), st));
    // host fields -> staging (one contiguous copy per field and situation)
    for (int b = 0; b < n; ++b) {
        if (!ctx->flat_met) {   // else already built on the device
            CK(cudaMemcpyAsync(sg.uk + ssz * b, f[b].uk, ssz * sizeof(float), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(sg.vk + ssz * b, f[b].vk, ssz * sizeof(float), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(sg.wk + ssz * b, f[b].wk, ssz * sizeof(float), cudaMemcpyHostToDevice, st));
        }
        if (ctx->model != 1) {
            CK(cudaMemcpyAsync(sg.turb + ssz * b, f[b].turb, ssz * sizeof(float), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(sg.tdiss + ssz * b, f[b].tdiss, ssz * sizeof(float), cudaMemcpyHostToDevice, st));
        }
    }
    launch_setup(a, sg, ctx->model, ctx->model != 1 ? ctx->varw.p : nullptr, ctx->model != 1 ? ctx->z0i.p : nullptr, st);
    launch_gather(a, sg, ctx->model, st);
    CK(cudaGetLastError());

    // ---- launch shapes of the wavefront kernels ----
    CK(gs_prepare(il, ks, ctx->model));
    ctx->it_host = 1;
    ctx->variant = -1;
    ctx->pmode = -1;
    int brc = size_grids(ctx);
    if (brc != GRAL_OK) return brc;
    CK(cudaEventRecord(ctx->ev[1], st));
    CK(cudaStreamSynchronize(st));
    CK(cudaEventElapsedTime(&ctx->ms_upload, ctx->ev[0], ctx->ev[1]));
    ctx->loaded = true;
    return GRAL_OK;
}

int gral_prog_iterate(gral_ctx *ctx) {
    if (!ctx) return GRAL_EINVAL;
    if (!ctx->loaded) return fail(ctx, GRAL_ESTATE, "iterate before load");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int trc = tune_variants(ctx);
    if (trc != GRAL_OK) return trc;
    int nact = ctx->h_act[1];
    while (nact > 0 && ctx->it_host <= ctx->it_max) {
        // run up to the next iteration where the reference can stop (a convergence test or the limit)
        const int c = ctx->cadence;
        int stop = ((ctx->it_host + c - 1) / c) * c;
        if (stop < ctx->it_host) stop = ctx->it_host;
        stop = std::min(stop, ctx->it_max);
        for (int it = ctx->it_host; it <= stop; ++it) CK(cudaGraphLaunch(ctx->graph, st));
        ctx->it_host = stop + 1;
        int herr = 0;
        CK(cudaMemcpyAsync(&herr, ctx->misc.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(ctx->h_sit.data(), ctx->sit.p, ctx->nb * sizeof(SitDev), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (herr == ERR_TIMEOUT) return fail(ctx, GRAL_ETIMEDOUT, "a wavefront wait exceeded its time limit");
        std::vector<int> act;
        for (int b = 0; b < ctx->nb; ++b)
            if (ctx->h_sit[b].active) act.push_back(b);
        if ((int)act.size() != nact) {
            nact = (int)act.size();
            ctx->h_act[1] = nact;
            for (int q = 0; q < nact; ++q) ctx->h_act[3 + q] = act[q];
            CK(cudaMemcpyAsync(ctx->misc.p + 1, ctx->h_act.data() + 1, sizeof(int), cudaMemcpyHostToDevice, st));
            if (nact > 0)
                CK(cudaMemcpyAsync(ctx->misc.p + 3, ctx->h_act.data() + 3, nact * sizeof(int), cudaMemcpyHostToDevice, st));
        }
    }
    return GRAL_OK;
}

int gral_prog_iterate_timed(gral_ctx *ctx, int32_t iterations, double *phase_ms, double *total_ms) {
    if (!ctx) return GRAL_EINVAL;
    if (!ctx->loaded) return fail(ctx, GRAL_ESTATE, "iterate before load");
    if (iterations < 1) return fail(ctx, GRAL_EINVAL, "iterations must be >= 1");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int trc = tune_variants(ctx);
    if (trc != GRAL_OK) return trc;
    const KArgs &a = ctx->ka;
    // the iteration's launches in order, each tagged with the phase it is timed under
    std::vector<std::pair<int, std::function<void()>>> seq;
    seq.push_back({GRAL_PHASE_BC, [&] {
        cudaMemsetAsync(ctx->counters.p, 0, 8 * kCounterSlots * sizeof(unsigned int), st);
        launch_bc(a, ctx->bc, st);
    }});
    const int sv = strip_variant_of(ctx);
    if (use_strips(ctx)) {
        if (fused_strips(ctx)) {
            seq.push_back({GRAL_PHASE_FUSED, [&] { launch_fused_strip(a, ctx->fgeo, ctx->fstrip_grid, st); }});
        } else {
            seq.push_back({GRAL_PHASE_PRESSURE, [&] { launch_strip(PH_PRESSURE, a, ctx->geo_p.g, sv, ctx->strip_grid[PH_PRESSURE], st); }});
            seq.push_back({GRAL_PHASE_VELCORR, [&] { launch_velcorr(a, st); }});
            seq.push_back({GRAL_PHASE_AVERAGE, [&] { launch_average(a, st); }});
            seq.push_back({GRAL_PHASE_U, [&] { launch_strip(PH_U, a, ctx->geo_u.g, sv, ctx->strip_grid[PH_U], st); }});
        }
        seq.push_back({GRAL_PHASE_V, [&] { launch_strip(PH_V, a, ctx->geo_v.g, sv, ctx->strip_grid[PH_V], st); }});
        seq.push_back({GRAL_PHASE_W, [&] { launch_strip(PH_W, a, ctx->geo_p.g, sv, ctx->strip_grid[PH_W], st); }});
    } else if (ctx->fused) {
        seq.push_back({GRAL_PHASE_FUSED, [&] { launch_fused_pvau(a, ctx->fgeo, ctx->fused_grid, st); }});
    } else {
        seq.push_back({GRAL_PHASE_PRESSURE, [&] { launch_gs(PH_PRESSURE, a, ctx->geo_p.g, ctx->grid_gs[PH_PRESSURE], st); }});
        seq.push_back({GRAL_PHASE_VELCORR, [&] { launch_velcorr(a, st); }});
        seq.push_back({GRAL_PHASE_AVERAGE, [&] { launch_average(a, st); }});
        seq.push_back({GRAL_PHASE_U, [&] { launch_gs(PH_U, a, ctx->geo_u.g, ctx->grid_gs[PH_U], st); }});
    }
    if (!use_strips(ctx)) {
        seq.push_back({GRAL_PHASE_V, [&] { launch_gs(PH_V, a, ctx->geo_v.g, ctx->grid_gs[PH_V], st); }});
        seq.push_back({GRAL_PHASE_W, [&] { launch_gs(PH_W, a, ctx->geo_p.g, ctx->grid_gs[PH_W], st); }});
    }
    if (ctx->model == 2)
        seq.push_back({GRAL_PHASE_TKE, [&] { launch_gs(PH_TKE, a, ctx->geo_p.g, ctx->grid_gs[PH_TKE], st); }});
    seq.push_back({GRAL_PHASE_BOOKKEEPING, [&] { launch_bookkeeping(a, st); }});
    const int marks = (int)seq.size() + 1;
    std::vector<cudaEvent_t> ev((size_t)iterations * marks, nullptr);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    for (int it = 0; it < iterations; ++it) {
        cudaEvent_t *E = ev.data() + (size_t)it * marks;
        for (size_t q = 0; q < seq.size(); ++q) {
            CK(cudaEventRecord(E[q], st));
            seq[q].second();
        }
        CK(cudaEventRecord(E[seq.size()], st));
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    int herr = 0;
    CK(cudaMemcpy(&herr, ctx->misc.p, sizeof(int), cudaMemcpyDeviceToHost));
    double ph[GRAL_NUM_PHASES] = {0};
    for (int it = 0; it < iterations; ++it) {
        cudaEvent_t *E = ev.data() + (size_t)it * marks;
        for (size_t q = 0; q < seq.size(); ++q) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, E[q], E[q + 1]));
            ph[seq[q].first] += ms;
        }
    }
    float tot = 0.f;
    CK(cudaEventElapsedTime(&tot, ev.front(), ev.back()));
    for (auto &e : ev) cudaEventDestroy(e);
    ctx->it_host += iterations;
    if (phase_ms) for (int q = 0; q < GRAL_NUM_PHASES; ++q) phase_ms[q] = ph[q];
    if (total_ms) *total_ms = tot;
    if (herr == ERR_TIMEOUT) return fail(ctx, GRAL_ETIMEDOUT, "a wavefront wait exceeded its time limit");
    return GRAL_OK;
}

int gral_prog_store(gral_ctx *ctx, gral_fields *f, gral_stats *stats) {
    if (!ctx) return GRAL_EINVAL;
    if (!ctx->loaded) return fail(ctx, GRAL_ESTATE, "store before load");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int n = ctx->nb;
    if (!f) f = ctx->fields.data();
    // post-checks run on every situation regardless of its loop state
    for (int b = 0; b < n; ++b) ctx->h_act[3 + b] = b;
    ctx->h_act[1] = n;
    std::vector<SitDev> hs(n);
    CK(cudaMemcpyAsync(hs.data(), ctx->sit.p, n * sizeof(SitDev), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<SitDev> tmp = hs;
    for (auto &x : tmp) x.active = 1;
    CK(cudaMemcpyAsync(ctx->sit.p, tmp.data(), n * sizeof(SitDev), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->misc.p + 1, ctx->h_act.data() + 1, sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->misc.p + 3, ctx->h_act.data() + 3, n * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(ctx->counts.p, 0, 4 * n * sizeof(int), st));
    CK(cudaEventRecord(ctx->ev[2], st));
    launch_postcheck(ctx->ka, ctx->counts.p, st);
    launch_scatter(ctx->ka, ctx->sg, ctx->model, st);
    CK(cudaGetLastError());
    if (ctx->post_diag) CK_RC(run_diagnostic(ctx));
    ctx->stored = true;
    const size_t ssz = ctx->sg.stride;
    for (int b = 0; b < n; ++b) {
        CK(cudaMemcpyAsync(f[b].uk, ctx->sg.uk + ssz * b, ssz * sizeof(float), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(f[b].vk, ctx->sg.vk + ssz * b, ssz * sizeof(float), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(f[b].wk, ctx->sg.wk + ssz * b, ssz * sizeof(float), cudaMemcpyDeviceToHost, st));
        if (ctx->model != 1) {
            CK(cudaMemcpyAsync(f[b].turb, ctx->sg.turb + ssz * b, ssz * sizeof(float), cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(f[b].tdiss, ctx->sg.tdiss + ssz * b, ssz * sizeof(float), cudaMemcpyDeviceToHost, st));
        }
    }
    std::vector<int> counts(4 * n);
    int herr = 0;
    CK(cudaMemcpyAsync(counts.data(), ctx->counts.p, 4 * n * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&herr, ctx->misc.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(ctx->sit.p, hs.data(), n * sizeof(SitDev), cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(ctx->ev[3], st));
    CK(cudaStreamSynchronize(st));
    if (herr == ERR_TIMEOUT) return fail(ctx, GRAL_ETIMEDOUT, "a wavefront wait exceeded its time limit");
    float ms_down = 0.f;
    cudaEventElapsedTime(&ms_down, ctx->ev[2], ctx->ev[3]);
    int rc = GRAL_OK;
    for (int b = 0; b < n; ++b) {
        const SitDev &S = hs[b];
        if (counts[4 * b + 3] > 0) rc = GRAL_ENONFINITE;
        if (!stats) continue;
        gral_stats &o = stats[b];
        o.iterations = S.iters_done;
        o.iteration_loops = S.it;
        o.converged = S.converged;
        o.delta_first = S.delta_first;
        o.delta_finish = S.delta_finish;
        o.convergence_problem = (S.delta_finish > S.delta_first) ? 1 : 0;
        o.n_history = std::min(S.n_hist, GRAL_MAX_HISTORY);
        for (int q = 0; q < o.n_history; ++q) o.delta_history[q] = S.hist[q];
        o.uk_unrealistic = counts[4 * b + 0];
        o.vk_unrealistic = counts[4 * b + 1];
        o.wk_unrealistic = counts[4 * b + 2];
        double g;
        std::memcpy(&g, &S.geschw_bits, sizeof(double));
        o.geschw_max = g;
        o.topwind = S.topwind;
        o.dtime = S.dtime;
        o.frund = S.frund;
        o.last_delta_umax = S.last_dumax;
        if (o.trace_delta_umax && o.trace_capacity > 0) {
            const int m = std::min(o.trace_capacity, ctx->it_max);
            CK(cudaMemcpy(o.trace_delta_umax, ctx->trace.p + (size_t)b * ctx->it_max, m * sizeof(float),
                          cudaMemcpyDeviceToHost));
        }
        o.ms_upload = ctx->ms_upload;
        o.ms_download = ms_down;
        o.layout = ctx->il ? 1 : 0;
        o.launch_variant = ctx->il ? ctx->variant : ctx->pmode;
        o.launches_per_iteration = launches_per_iteration(ctx);
    }
    if (rc != GRAL_OK) fail(ctx, rc, "non-finite values in the solved fields");
    return rc;
}

int gral_prog_solve_batch(gral_ctx *ctx, int32_t n, const gral_params *p, const gral_static *s, gral_fields *f,
                          gral_stats *stats) {
    int rc = gral_prog_load(ctx, n, p, s, f);
    if (rc != GRAL_OK) return rc;
    cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1];
    cudaEventRecord(e0, ctx->stream);
    rc = gral_prog_iterate(ctx);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float ms_it = 0.f;
    cudaEventElapsedTime(&ms_it, e0, e1);
    if (rc != GRAL_OK) return rc;
    rc = gral_prog_store(ctx, f, stats);
    if (stats)
        for (int b = 0; b < n; ++b) {
            stats[b].ms_iterate = ms_it;
            stats[b].ms_total = stats[b].ms_upload + ms_it + stats[b].ms_download;
        }
    return rc;
}

int gral_prog_load_flat(gral_ctx *ctx, int32_t n, const gral_params *p, const gral_static *s, const gral_met *met,
                        const gral_flat_grid *g, gral_fields *f) {
    if (!ctx) return GRAL_EINVAL;
    if (n < 1 || !p || !s || !met || !g || !s->cutk || !s->dzk || !s->hokart)
        return fail(ctx, GRAL_EINVAL, "null pointer or empty batch");
    if (g->nii != p[0].nii || g->njj != p[0].njj || g->nkk != p[0].nkk || g->vert_cells_ff != p[0].vert_cells_ff ||
        g->dxk != p[0].dxk || g->dyk != p[0].dyk)
        return fail(ctx, GRAL_EINVAL, "set-up grid differs from the parameters");
    for (int b = 0; b < n; ++b) {
        const int rc = flat_check(ctx, g, s->hokart, &met[b], s->advdom != nullptr);
        if (rc != GRAL_OK) return rc;
    }
    ctx->flat_met = met;
    ctx->flat_grid = g;
    const int rc = gral_prog_load(ctx, n, p, s, f);
    ctx->flat_met = nullptr;
    ctx->flat_grid = nullptr;
    return rc;
}

int gral_prog_solve(gral_ctx *ctx, const gral_params *p, const gral_static *s, gral_fields *f, gral_stats *stats) {
    return gral_prog_solve_batch(ctx, 1, p, s, f, stats);
}

}  // extern "C"
