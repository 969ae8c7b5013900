// prog_prep.cu -- the flow-field set-up that GRAL runs on the host before each prognostic solve,
// on the device: the prognostic sub-domains (ReadGeometryAndDomains.cs:321-347), the flat-terrain
// initial field with KKART/AHK/KADVMAX (MicroscaleFlat.cs:29-197) and its near-wall damping
// (:201-357), and the vegetation rasterisation (ReadVegetation.cs:83-118).
//
// The transcendental values of these routines (MathF.Pow of the wind profile, MathF.Log of the
// wall damping, Math.Pow of the vegetation cover) depend only on the level, the Obukhov length,
// a distance of a few cells or one vegetation line, so they are evaluated on the host with the C
// library -- which is what .NET calls for them -- into small tables; the kernels do the per-cell
// work with the reference's float/double expressions.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

#include "prog_ctx.cuh"
#include "prog_prep.cuh"

namespace gral {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// ---- host helpers ----

// MathF.Max(float, float): IEEE 754:2019 maximum (NaN propagates)
inline float host_net_max(float a, float b) {
    if (a != b) { if (!std::isnan(a)) return (b < a) ? a : b; return a; }
    return std::signbit(b) ? a : b;
}

// C-library calls kept as calls (MathF.Pow/Log and Math.Pow map onto them)
float (*volatile c_powf)(float, float) = ::powf;
float (*volatile c_logf)(float) = ::logf;
double (*volatile c_pow)(double, double) = ::pow;

// (int)(factor * CUTK / DXK) of ReadGeometryAndDomains.cs:331-332: int * float in float, / in float
__host__ __device__ inline int reach_cells(int factor, float cutk, float d) {
    const float x = (float)factor * cutk;
    return (int)(x / d);
}

// ---- prognostic sub-domains ----
// The union of rectangles |i1-i| <= ip(i,j), |j1-j| <= jp(i,j) over building cells (i,j) is found
// in two passes: R(i, j1) = max ip(i,j) over the cells of row i whose j-range covers j1 (-1 if
// none), then ADVDOM(i1, j1) = 1 iff some row i has R(i, j1) >= |i1 - i|.
__global__ void __launch_bounds__(kThreads) k_sub_reach(int nii, int njj, float dxk, float dyk, int factor,
                                                        int jmax, const float *__restrict__ cutk, int *__restrict__ reach) {
    const int j1 = blockIdx.x * blockDim.x + threadIdx.x + 1, i = blockIdx.y + 1;
    if (j1 > njj) return;
    const int nj2 = njj + 2;
    int r = -1;
    const int lo = max(1, j1 - jmax), hi = min(njj, j1 + jmax);
    for (int j = lo; j <= hi; ++j) {
        const float c = cutk[i * nj2 + j];
        if (c > 0 && abs(j1 - j) <= reach_cells(factor, c, dyk)) r = max(r, reach_cells(factor, c, dxk));
    }
    reach[i * nj2 + j1] = r;
}

__global__ void __launch_bounds__(kThreads) k_sub_mark(int nii, int njj, int imax, const int *__restrict__ reach,
                                                       uint8_t *__restrict__ advdom) {
    const int j1 = blockIdx.x * blockDim.x + threadIdx.x + 1, i1 = blockIdx.y + 1;
    if (j1 > njj) return;
    const int nj2 = njj + 2;
    const int lo = max(1, i1 - imax), hi = min(nii, i1 + imax);
    uint8_t a = 0;
    for (int i = lo; i <= hi && !a; ++i)
        if (reach[i * nj2 + j1] >= abs(i1 - i)) a = 1;
    advdom[i1 * nj2 + j1] = a;
}

// ---- flat-terrain initial field (MicroscaleFlat.cs:56-197) ----
// One warp per column (i = 1..NII, j = 1..NJJ), lanes over the levels.  The reference's loop also
// zeroes U of the east neighbour and V of the north neighbour of an obstacle cell; in its
// sequential order that neighbour column comes later and sets the same zero by its own
// west/south test, so those writes are left to it.  The east edge U[NII+1] and the north edge
// V[NJJ+1] receive the final U[NII] / V[NJJ] of the level, which is what the reference's
// in-loop copies leave in sequential order.
struct FlatTabs {
    const float *vertk;   // [nkk+1]: HOKART[k-1] + DZK[k]*0.5
    const float *hok;     // HOKART
    const float *pu, *pv; // [nprof][nkk+1] initial U, V of a column outside obstacles
    const int *col_prof;  // profile per column, or nullptr (profile 0)
};

__global__ void __launch_bounds__(kThreads) k_flat_columns(int nii, int njj, int nkk, FlatTabs t,
                                                           const float *__restrict__ cutk,
                                                           float *__restrict__ uk, float *__restrict__ vk,
                                                           int16_t *__restrict__ kkart, float *__restrict__ ahk,
                                                           int *kadv) {
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.y + 1, j = blockIdx.x * kWarps + (threadIdx.x >> 5) + 1;   // grid (j tiles, rows)
    if (j > njj) return;
    const int nj2 = njj + 2, nk2 = nkk + 2;
    const int c = i * nj2 + j;
    const float cut = cutk[c];
    const float cut_w = (i > 1) ? cutk[c - nj2] : 0.f, cut_s = (j > 1) ? cutk[c - 1] : 0.f;
    const int prof = t.col_prof ? t.col_prof[c] : 0;
    const float *pu = t.pu + prof * (nkk + 1), *pv = t.pv + prof * (nkk + 1);
    float *ucol = uk + (size_t)c * nk2, *vcol = vk + (size_t)c * nk2;
    float *ueast = (i == nii) ? ucol + (size_t)nj2 * nk2 : nullptr;   // U[NII+1][j]
    float *vnorth = (j == njj) ? vcol + nk2 : nullptr;                 // V[i][NJJ+1]
    int kk = 0;
    float ah = 0.f;
    for (int k = 1 + lane; k <= nkk; k += 32) {
        const float vz = t.vertk[k];
        float u = 0.f, v = 0.f;
        if (vz > cut) {
            u = pu[k];
            v = pv[k];
            if (i > 1 && vz <= cut_w) u = 0.f;
            if (j > 1 && vz <= cut_s) v = 0.f;
        } else {
            ah = fmaxf(t.hok[k], ah);
            kk = k;
        }
        ucol[k] = u;
        vcol[k] = v;
        if (ueast) ueast[k] = u;
        if (vnorth) vnorth[k] = v;
    }
    // AHK is a maximum of heights >= 0 (the host checks HOKART), which orders like their bits
    kk = __reduce_max_sync(0xffffffffu, kk);
    const int ahb = __reduce_max_sync(0xffffffffu, __float_as_int(ah));
    if (lane == 0) {
        kkart[c] = (int16_t)kk;
        ahk[c] = __int_as_float(ahb);
        if (cut > 0) atomicMax(kadv, kk);
    }
}

// Near-wall damping (MicroscaleFlat.cs:201-357) on columns i = 1+IGEB..NII-IGEB, j = 1+IGEB..NJJ-IGEB,
// levels KKART < k < NKK: in each of eight directions the nearest cell within IGEB with CUTK > 1
// whose AHK reaches the level multiplies the factor 0.19*ln((d+0.5)*10) of its distance d (if
// d <= 20 m; the table holds 1 otherwise).  fac: [3][igeb+1] for x, y and diagonal steps.
__global__ void __launch_bounds__(kThreads) k_flat_near_wall(int nii, int njj, int nkk, int igeb, int mode,
                                                             const uint8_t *__restrict__ advdom,
                                                             const float *__restrict__ cutk,
                                                             const float *__restrict__ ahk,
                                                             const int16_t *__restrict__ kkart,
                                                             const float *__restrict__ vertk,
                                                             const float *__restrict__ fac, float *__restrict__ uk,
                                                             float *__restrict__ vk) {
    const int lane = threadIdx.x & 31;
    const int ni = nii - 2 * igeb, nj = njj - 2 * igeb;
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (ni <= 0 || nj <= 0 || w >= (long long)ni * nj) return;
    const int i = (int)(w / nj) + 1 + igeb, j = (int)(w % nj) + 1 + igeb;
    const int nj2 = njj + 2, nk2 = nkk + 2;
    const size_t c = (size_t)i * nj2 + j;
    if (mode == 1 && advdom[c] != 0) return;
    const int kk = kkart[c];
    const float *fx = fac, *fy = fac + (igeb + 1), *fd = fac + 2 * (igeb + 1);
    // direction steps in the reference's order: W, E, N, S, (+,+), (-,-), (+,-), (-,+)
    const int di[8] = {-1, 1, 0, 0, 1, -1, 1, -1};
    const int dj[8] = {0, 0, 1, -1, 1, -1, -1, 1};
    for (int k = max(kk + 1, 1) + lane; k < nkk; k += 32) {
        const float vz = vertk[k];
        float ab = 1.f;
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            const float *f = (d < 2) ? fx : (d < 4) ? fy : fd;
            for (int n = 1; n <= igeb; ++n) {
                const size_t g = (size_t)(i + n * di[d]) * nj2 + (j + n * dj[d]);
                if (cutk[g] > 1 && vz <= ahk[g]) {
                    ab = ab * f[n];
                    break;
                }
            }
        }
        uk[c * nk2 + k] = uk[c * nk2 + k] * ab;
        vk[c * nk2 + k] = vk[c * nk2 + k] * ab;
    }
}

// ---- vegetation (ReadVegetation.cs:83-118) ----
struct VegRec {            // one in-bounds line of vegetation.dat, file order kept per cell
    double crown, trunk;   // crown_height, trunk_height
    float v_trunk, v_crown; // (float)(0.3 * Math.Pow(COV, 3) * LAD)
    float cov;
    int drag;
};

// One warp per cell that has lines: lanes over k = 0..NKK-1, lines applied in order.
__global__ void __launch_bounds__(kThreads) k_vegetation(int njj, int nkk, int ncells,
                                                         const int *__restrict__ cells,
                                                         const int *__restrict__ first,
                                                         const VegRec *__restrict__ rec,
                                                         const int16_t *__restrict__ kkart,
                                                         const float *__restrict__ dzk,
                                                         const float *__restrict__ hok, float *__restrict__ veg,
                                                         uint8_t *__restrict__ mask, float *__restrict__ cov) {
    const int lane = threadIdx.x & 31;
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= ncells) return;
    const int c = cells[w];
    const int kk = kkart[c];
    const int r0 = first[w], r1 = first[w + 1];
    const size_t base = (size_t)c * (nkk + 2);
    for (int k = lane; k < nkk; k += 32) {
        float v = 0.f;
        if (k >= kk - 1) {
            const float mch = hok[k] - hok[kk] + dzk[k] * 0.5f;
            for (int r = r0; r < r1; ++r) {
                const VegRec &p = rec[r];
                if (!p.drag) continue;
                if ((double)mch < p.crown) {
                    if (mch >= 0 && (double)mch < p.trunk) v = p.v_trunk;
                    else if (mch >= 0 && (double)mch >= p.trunk) v = p.v_crown;
                }
            }
        }
        veg[base + k] = v;
    }
    if (lane == 0) {
        int any = 0;
        for (int r = r0; r < r1; ++r) any |= rec[r].drag;
        mask[c] = (uint8_t)(any ? 1 : 0);
        cov[c] = rec[r1 - 1].cov;
    }
}

int grid_warps(long long warps) { return (int)((warps + kWarps - 1) / kWarps); }

}  // namespace

int flat_check(gral_ctx *ctx, const gral_flat_grid *g, const float *hokart, const gral_met *met, bool have_advdom) {
    const int NII = g->nii, NJJ = g->njj, NKK = g->nkk;
    if (NII < 1 || NJJ < 1 || NKK < 2 || NII > ctx->cap_nii || NJJ > ctx->cap_njj || NKK > ctx->cap_nkk)
        return fail(ctx, GRAL_EINVAL, "grid outside the context's capacity");
    if (g->vert_cells_ff < 0) return fail(ctx, GRAL_EINVAL, "negative vert_cells_ff");
    if ((long long)(NII + 2) * (NJJ + 2) >= (1LL << 31)) return fail(ctx, GRAL_ETOOLARGE, "more than 2^31 columns");
    if (g->near_wall < 0 || g->near_wall > 2) return fail(ctx, GRAL_EINVAL, "near_wall must be 0, 1 or 2");
    if (g->near_wall == 1 && !have_advdom) return fail(ctx, GRAL_EINVAL, "near_wall 1 needs ADVDOM");
    if (g->near_wall && g->igeb < 1) return fail(ctx, GRAL_EINVAL, "igeb must be at least 1");
    for (int k = 0; k < NKK + 2; ++k)
        if (!(hokart[k] >= 0)) return fail(ctx, GRAL_EINVAL, "HOKART must be non-negative");
    if (NII > 65535) return fail(ctx, GRAL_ETOOLARGE, "more than 65535 rows");
    const int nh = met->n_heights;
    if (nh < 1 || !met->measurement_height || !met->obs_u || !met->obs_v)
        return fail(ctx, GRAL_EINVAL, "met profile needs at least one height");
    return GRAL_OK;
}

int flat_fill(gral_ctx *ctx, const gral_flat_grid *g, const float *d_cutk, const uint8_t *d_adv, const float *dzk,
              const float *hokart, const gral_met *met, float *du, float *dv, float *dw, int **d_kadv_out,
              bool timed) {
    const int NII = g->nii, NJJ = g->njj, NKK = g->nkk;
    const int nh = met->n_heights;
    const float *MH = met->measurement_height, *OU = met->obs_u, *OV = met->obs_v;
    const int nj2 = NJJ + 2, nk2 = NKK + 2;
    const size_t ncols = (size_t)(NII + 2) * nj2, cells = ncols * nk2;

    // ---- host tables ----
    std::vector<float> vertk(NKK + 1, 0.f);
    for (int k = 1; k <= NKK; ++k) vertk[k] = hokart[k - 1] + dzk[k] * 0.5f;
    // profile per Obukhov length (MicroscaleFlat.cs:84-140)
    auto profile = [&](float ob, float *pu, float *pv) {
        auto exponent = [&]() {
            if (ob <= 0) return host_net_max(0.35f - 0.4f * c_powf(std::fabs(ob), -0.15f), 0.05f);
            return 0.56f * c_powf(ob, -0.15f);
        };
        for (int k = 1; k <= NKK; ++k) {
            const float vz = vertk[k];
            float u, v;
            if (vz <= MH[1]) {
                const float dumfac = c_powf(vz / MH[1], exponent());
                u = OU[1] * dumfac;
                v = OV[1] * dumfac;
            } else if (vz > MH[nh]) {
                if (nh == 1) {
                    const float dumfac = c_powf(vz / MH[nh], exponent());
                    u = OU[nh] * dumfac;
                    v = OV[nh] * dumfac;
                } else {
                    u = OU[nh];
                    v = OV[nh];
                }
            } else {
                int ipo = 1;
                for (int q = 1; q <= nh; ++q)
                    if (vz > MH[q]) ipo = q + 1;
                u = OU[ipo - 1] + (OU[ipo] - OU[ipo - 1]) / (MH[ipo] - MH[ipo - 1]) * (vz - MH[ipo - 1]);
                v = OV[ipo - 1] + (OV[ipo] - OV[ipo - 1]) / (MH[ipo] - MH[ipo - 1]) * (vz - MH[ipo - 1]);
            }
            pu[k] = u;
            pv[k] = v;
        }
    };
    std::vector<float> pu, pv;
    std::vector<int> col_prof;
    if (met->ol_column) {
        std::map<uint32_t, int> index;   // distinct Obukhov lengths, keyed by their bits
        col_prof.assign(ncols, 0);
        for (int i = 1; i <= NII; ++i)
            for (int j = 1; j <= NJJ; ++j) {
                const size_t c = (size_t)i * nj2 + j;
                uint32_t key;
                std::memcpy(&key, &met->ol_column[c], 4);
                auto it = index.find(key);
                int q;
                if (it == index.end()) {
                    q = (int)index.size();
                    index.emplace(key, q);
                    pu.resize((size_t)(q + 1) * (NKK + 1), 0.f);
                    pv.resize((size_t)(q + 1) * (NKK + 1), 0.f);
                    profile(met->ol_column[c], pu.data() + (size_t)q * (NKK + 1), pv.data() + (size_t)q * (NKK + 1));
                } else {
                    q = it->second;
                }
                col_prof[c] = q;
            }
        if (pu.empty()) { pu.assign(NKK + 1, 0.f); pv.assign(NKK + 1, 0.f); }
    } else {
        pu.assign(NKK + 1, 0.f);
        pv.assign(NKK + 1, 0.f);
        profile(met->ob_length, pu.data(), pv.data());
    }
    // wall-damping factors (MicroscaleFlat.cs:223-340): x, y and diagonal distances of n cells
    const int igeb = g->near_wall ? g->igeb : 0;
    std::vector<float> fac(3 * (igeb + 1), 1.f);
    for (int n = 1; n <= igeb; ++n) {
        const float ex = std::fabs((float)n * g->dxk), ey = std::fabs((float)n * g->dyk);
        const float px = (float)n * g->dxk, py = (float)n * g->dyk;
        const float ed = std::sqrt(px * px + py * py);
        const float e[3] = {ex, ey, ed};
        for (int q = 0; q < 3; ++q)
            fac[q * (igeb + 1) + n] = (e[q] <= 20) ? 0.19f * c_logf((e[q] + 0.5f) * 10) : 1.f;
    }

    // ---- device ----
    cudaStream_t st = ctx->stream;
    PrepBufs &b = ctx->prep;
    const size_t ntab = (NKK + 1) + nk2 + pu.size() + pv.size() + fac.size();
    CK(b.ahk.ensure(ncols));
    CK(b.kkart.ensure(ncols));
    CK(b.tab.ensure(ntab));
    CK(b.ints.ensure(col_prof.size() + 1));
    float *d_vertk = b.tab.p, *d_hok = d_vertk + (NKK + 1), *d_pu = d_hok + nk2, *d_pv = d_pu + pu.size(),
          *d_fac = d_pv + pv.size();
    CK(cudaMemcpyAsync(d_vertk, vertk.data(), vertk.size() * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_hok, hokart, nk2 * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_pu, pu.data(), pu.size() * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_pv, pv.data(), pv.size() * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_fac, fac.data(), fac.size() * 4, cudaMemcpyHostToDevice, st));
    int *d_kadv = b.ints.p + col_prof.size();
    if (!col_prof.empty())
        CK(cudaMemcpyAsync(b.ints.p, col_prof.data(), col_prof.size() * 4, cudaMemcpyHostToDevice, st));
    const int one = 1;
    CK(cudaMemcpyAsync(d_kadv, &one, 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(du, 0, cells * sizeof(float), st));
    CK(cudaMemsetAsync(dv, 0, cells * sizeof(float), st));
    CK(cudaMemsetAsync(dw, 0, cells * sizeof(float), st));
    CK(cudaMemsetAsync(b.kkart.p, 0, ncols * sizeof(int16_t), st));
    CK(cudaMemsetAsync(b.ahk.p, 0, ncols * sizeof(float), st));
    FlatTabs t{d_vertk, d_hok, d_pu, d_pv, col_prof.empty() ? nullptr : b.ints.p};
    if (timed) CK(cudaEventRecord(ctx->ev[0], st));
    k_flat_columns<<<dim3((NJJ + kWarps - 1) / kWarps, NII), kThreads, 0, st>>>(NII, NJJ, NKK, t, d_cutk, du, dv,
                                                                                b.kkart.p, b.ahk.p, d_kadv);
    if (g->near_wall && NII > 2 * igeb && NJJ > 2 * igeb)
        k_flat_near_wall<<<grid_warps((long long)(NII - 2 * igeb) * (NJJ - 2 * igeb)), kThreads, 0, st>>>(
            NII, NJJ, NKK, igeb, g->near_wall, d_adv, d_cutk, b.ahk.p, b.kkart.p, d_vertk, d_fac, du, dv);
    CK(cudaGetLastError());
    if (timed) CK(cudaEventRecord(ctx->ev[1], st));
    *d_kadv_out = d_kadv;
    return GRAL_OK;
}

}  // namespace gral

using namespace gral;

namespace {

// device time between ev[0] and ev[1] of a completed set-up call
int record_ms(gral_ctx *ctx) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    ctx->prep_ms = ms;
    return GRAL_OK;
}

}  // namespace

extern "C" {

int gral_prog_subdomains(gral_ctx *ctx, int32_t nii, int32_t njj, float dxk, float dyk, int32_t factor,
                         const float *cutk, uint8_t *advdom) {
    if (!ctx) return GRAL_EINVAL;
    if (!cutk || !advdom) return fail(ctx, GRAL_EINVAL, "null pointer");
    if (nii < 1 || njj < 1 || nii > ctx->cap_nii || njj > ctx->cap_njj)
        return fail(ctx, GRAL_EINVAL, "grid outside the context's capacity");
    if (!(dxk > 0) || !(dyk > 0) || factor < 0) return fail(ctx, GRAL_EINVAL, "bad cell size or factor");
    const int nj2 = njj + 2;
    const size_t ncols = (size_t)(nii + 2) * nj2;
    // the largest reach bounds both passes' search ranges (reach grows with CUTK)
    float cmax = 0.f;
    for (int i = 1; i <= nii; ++i)
        for (int j = 1; j <= njj; ++j) cmax = std::max(cmax, cutk[(size_t)i * nj2 + j]);
    const int imax = reach_cells(factor, cmax, dxk), jmax = reach_cells(factor, cmax, dyk);
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    PrepBufs &b = ctx->prep;
    CK(b.cutk.ensure(ncols));
    CK(b.ints.ensure(ncols));
    CK(b.adv.ensure(ncols));
    CK(cudaMemcpyAsync(b.cutk.p, cutk, ncols * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(b.adv.p, 0, ncols, st));
    const dim3 grid((njj + kThreads - 1) / kThreads, nii);
    CK(cudaEventRecord(ctx->ev[0], st));
    k_sub_reach<<<grid, kThreads, 0, st>>>(nii, njj, dxk, dyk, factor, jmax, b.cutk.p, b.ints.p);
    k_sub_mark<<<grid, kThreads, 0, st>>>(nii, njj, imax, b.ints.p, b.adv.p);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[1], st));
    CK(cudaMemcpyAsync(advdom, b.adv.p, ncols, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return record_ms(ctx);
}

int gral_prog_flat_init(gral_ctx *ctx, const gral_flat_grid *g, const float *cutk, const float *dzk,
                        const float *hokart, const uint8_t *advdom, const gral_met *met, int16_t *kkart,
                        float *ahk, int32_t *kadvmax, gral_fields *f) {
    if (!ctx) return GRAL_EINVAL;
    if (!g || !cutk || !dzk || !hokart || !met || !kkart || !ahk || !kadvmax || !f || !f->uk || !f->vk || !f->wk)
        return fail(ctx, GRAL_EINVAL, "null pointer");
    int rc = flat_check(ctx, g, hokart, met, advdom != nullptr);
    if (rc != GRAL_OK) return rc;
    const int NII = g->nii, NJJ = g->njj, NKK = g->nkk;
    const int nj2 = NJJ + 2, nk2 = NKK + 2;
    const size_t ncols = (size_t)(NII + 2) * nj2, cells = ncols * nk2;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    PrepBufs &b = ctx->prep;
    CK(b.cutk.ensure(ncols));
    CK(b.fields.ensure(3 * cells));
    if (g->near_wall == 1) CK(b.adv.ensure(ncols));
    CK(cudaMemcpyAsync(b.cutk.p, cutk, ncols * 4, cudaMemcpyHostToDevice, st));
    if (g->near_wall == 1) CK(cudaMemcpyAsync(b.adv.p, advdom, ncols, cudaMemcpyHostToDevice, st));
    float *du = b.fields.p, *dv = du + cells, *dw = dv + cells;
    int *d_kadv = nullptr;
    rc = flat_fill(ctx, g, b.cutk.p, b.adv.p, dzk, hokart, met, du, dv, dw, &d_kadv, true);
    if (rc != GRAL_OK) return rc;
    int kadv1 = 1;
    CK(cudaMemcpyAsync(&kadv1, d_kadv, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(kkart, b.kkart.p, ncols * sizeof(int16_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(ahk, b.ahk.p, ncols * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(f->uk, du, cells * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(f->vk, dv, cells * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(f->wk, dw, cells * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // KADVMAX = 1, then the largest KKART of a building column, then + VertCellsFF capped at NKK
    *kadvmax = std::min(NKK, std::max(1, kadv1) + g->vert_cells_ff);
    return record_ms(ctx);
}

int gral_prog_vegetation(gral_ctx *ctx, int32_t nii, int32_t njj, int32_t nkk, const int16_t *kkart,
                         const float *dzk, const float *hokart, int32_t n_points, const gral_veg_point *points,
                         float *veg, uint8_t *veg_mask, float *cov) {
    if (!ctx) return GRAL_EINVAL;
    if (!kkart || !dzk || !hokart || !veg || !veg_mask || !cov || (n_points > 0 && !points))
        return fail(ctx, GRAL_EINVAL, "null pointer");
    if (nii < 1 || njj < 1 || nkk < 2 || nii > ctx->cap_nii || njj > ctx->cap_njj || nkk > ctx->cap_nkk)
        return fail(ctx, GRAL_EINVAL, "grid outside the context's capacity");
    if (n_points < 0) return fail(ctx, GRAL_EINVAL, "negative point count");
    const int nj2 = njj + 2, nk2 = nkk + 2;
    const size_t ncols = (size_t)(nii + 2) * nj2, cells = ncols * nk2;
    for (size_t c = 0; c < ncols; ++c)
        if (kkart[c] < 0 || kkart[c] > nkk) return fail(ctx, GRAL_EINVAL, "KKART outside 0..NKK");
    // lines grouped by cell in file order (ReadVegetation.cs:85-87 skips lines outside the grid)
    std::vector<std::vector<int>> per;
    std::map<size_t, int> slot;
    std::vector<int> cell_of;
    for (int q = 0; q < n_points; ++q) {
        const gral_veg_point &p = points[q];
        if (!(p.i <= nii && p.i >= 1 && p.j <= njj && p.j >= 1)) continue;
        const size_t c = (size_t)p.i * nj2 + p.j;
        auto it = slot.find(c);
        if (it == slot.end()) {
            it = slot.emplace(c, (int)per.size()).first;
            per.emplace_back();
            cell_of.push_back((int)c);
        }
        per[it->second].push_back(q);
    }
    const int ncell = (int)per.size();
    std::vector<int> first(ncell + 1, 0);
    std::vector<VegRec> rec;
    rec.reserve(n_points);
    for (int s = 0; s < ncell; ++s) {
        first[s] = (int)rec.size();
        for (int q : per[s]) {
            const gral_veg_point &p = points[q];
            const double c3 = c_pow(p.cov, 3.0);
            rec.push_back(VegRec{p.crown_height, p.trunk_height, (float)(0.3 * c3 * p.trunk_lad),
                                 (float)(0.3 * c3 * p.crown_lad), (float)p.cov, p.drag ? 1 : 0});
        }
    }
    first[ncell] = (int)rec.size();
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    PrepBufs &b = ctx->prep;
    CK(b.veg.ensure(cells));
    CK(b.mask.ensure(ncols));
    CK(b.cov.ensure(ncols));
    CK(b.kkart.ensure(ncols));
    CK(b.tab.ensure(2 * (size_t)nk2));
    CK(b.ints.ensure(2 * (size_t)ncell + 1));
    CK(b.points.ensure(std::max<size_t>(rec.size(), 1) * sizeof(VegRec)));
    float *d_dzk = b.tab.p, *d_hok = d_dzk + nk2;
    int *d_cells = b.ints.p, *d_first = d_cells + ncell;
    CK(cudaMemcpyAsync(d_dzk, dzk, nk2 * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_hok, hokart, nk2 * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(b.kkart.p, kkart, ncols * sizeof(int16_t), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(b.cov.p, cov, ncols * sizeof(float), cudaMemcpyHostToDevice, st));
    if (ncell) {
        CK(cudaMemcpyAsync(d_cells, cell_of.data(), ncell * sizeof(int), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_first, first.data(), (ncell + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(b.points.p, rec.data(), rec.size() * sizeof(VegRec), cudaMemcpyHostToDevice, st));
    }
    CK(cudaMemsetAsync(b.veg.p, 0, cells * sizeof(float), st));
    CK(cudaMemsetAsync(b.mask.p, 0, ncols, st));
    CK(cudaEventRecord(ctx->ev[0], st));
    if (ncell)
        k_vegetation<<<grid_warps(ncell), kThreads, 0, st>>>(njj, nkk, ncell, d_cells, d_first,
                                                             reinterpret_cast<const VegRec *>(b.points.p),
                                                             b.kkart.p, d_dzk, d_hok, b.veg.p, b.mask.p, b.cov.p);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[1], st));
    CK(cudaMemcpyAsync(veg, b.veg.p, cells * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(veg_mask, b.mask.p, ncols, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(cov, b.cov.p, ncols * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return record_ms(ctx);
}

int gral_prog_prep_last_ms(gral_ctx *ctx, double *kernel_ms) {
    if (!ctx || !kernel_ms) return GRAL_EINVAL;
    *kernel_ms = ctx->prep_ms;
    return GRAL_OK;
}

}  // extern "C"
