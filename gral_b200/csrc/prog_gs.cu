// prog_gs.cu -- Gauss-Seidel wavefront kernels: pressure correction and the mixing-length
// (TurbulenceModel 1) U, V, W momentum equations.
//
// The reference sweeps every (i,j) column lexicographically and updates it in place
// (PrognosticFlowfield.cs:804-901; U-prognostic-microscale_1.cs:96-529; V-...1.cs:94-524;
// W-...1.cs:93-453), so a column reads the already-updated neighbours that precede it in sweep
// order and the old values of those that follow.  With a 5-point horizontal stencil this order is
// reproduced exactly by a wavefront over the anti-diagonals of the sweep coordinates: a column may
// run as soon as its two sweep predecessors (i1-1, j1) and (i1, j1-1) have finished.  Each warp
// claims column tasks in diagonal order from an atomic counter (so every claimed task's
// predecessors were claimed earlier by running warps: no deadlock, no co-residency assumption),
// waits with a bounded spin on the predecessors' stamps, solves, and publishes its own stamp.
// Values another warp may write inside the same kernel (the swept field, the pressure row carry)
// are read with ld.global.cg so no stale L1 line is used.
//
// Two families share the per-level arithmetic of prog_level.cuh:
//   plain   (slab layout)        one warp per (situation, column), lane = level; lane 0 runs the
//                                serial Thomas sweep on the warp's shared rows;
//   batched (interleaved layout) one warp per (group of 32 situations, column), lane =
//                                situation; every lane runs its own k loop and Thomas sweep, the
//                                P/Q rows live in shared memory [k][thread].
#include <algorithm>

#include "prog_common.cuh"
#include "prog_kernels.cuh"
#include "prog_level.cuh"

namespace gral {

namespace {

constexpr int GS_WARPS = 4;      // warps per block, plain family
constexpr int SM_ROWS = 5;       // shared rows per warp of the plain family: A, B, C, D, phi

__device__ __forceinline__ void sweep_dir(int it, int &IS, int &JS) {
    // PrognosticFlowfield.cs:770-802
    const int m = it % 4;
    if (m == 0) { IS = -1; JS = 1; }
    else if (m == 1) { IS = -1; JS = -1; }
    else if (m == 2) { IS = 1; JS = -1; }
    else { IS = 1; JS = 1; }
}

// Task t -> (unit index, i1, j1): diagonal-major, then unit (situation or group), then position.
__device__ __forceinline__ void decode_task(unsigned t, const SweepGeom &g, unsigned units, int &u, int &i1,
                                            int &j1) {
    int lo = 0, hi = g.ndiag;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if ((unsigned)g.diag_start[mid] * units <= t) lo = mid; else hi = mid;
    }
    const int d = lo;
    const unsigned r = t - (unsigned)g.diag_start[d] * units;
    const unsigned len = (unsigned)(g.diag_start[d + 1] - g.diag_start[d]);
    u = (int)(r / len);
    const int pos = (int)(r % len);
    const int ioff = max(0, d - (g.nj - 1)) + pos;
    i1 = g.ia + ioff;
    j1 = g.ja + d - ioff;
}

// The wavefront task loop shared by every Gauss-Seidel phase.  A unit is a situation (plain) or a
// group of 32 situations (batched); flags are stamped per (unit, column).
// body(u, i, j, IS, JS, first) solves one column with the whole warp; `first` marks the first
// column of a sweep row.
template <int PHASE, bool REVERSE, bool IL, class Body>
__device__ __forceinline__ void gs_tasks(const KArgs &a, const SweepGeom &g, Body &&body) {
    const int lane = threadIdx.x & 31;
    const unsigned units = IL ? (unsigned)a.ngroups : (unsigned)*a.nact;
    const unsigned total = (unsigned)g.diag_start[g.ndiag] * units;
    unsigned int *ctr = a.counters + PHASE;
    const int it = *a.it_global;
    int IS, JS;
    sweep_dir(it, IS, JS);
    if (REVERSE) { IS = -IS; JS = -JS; }
    const int stamp = it * 8 + PHASE;
    for (;;) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(ctr, (unsigned)a.chunk);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) break;
        if (*(volatile int *)a.err != ERR_NONE) break;
        const unsigned end = min(total, base + (unsigned)a.chunk);
        for (unsigned t = base; t < end; ++t) {
            int u, i1, j1;
            decode_task(t, g, units, u, i1, j1);
            if (!IL) u = a.act[u];
            const int i = (IS == 1) ? i1 : a.nii - i1 + 1;
            const int j = (JS == 1) ? j1 : a.njj - j1 + 1;
            int *fl = a.flags + (size_t)u * a.ncols;
            int ok = 1;
            if (lane == 0) {
                if (i1 > g.ia) ok = wait_stamp(fl + (i - IS) * a.nj2 + j, stamp, a.err, a.wait_limit_ns);
                if (ok && j1 > g.ja) ok = wait_stamp(fl + i * a.nj2 + (j - JS), stamp, a.err, a.wait_limit_ns);
            }
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (ok) body(u, i, j, IS, JS, i1 == g.ia);
            __syncwarp();
            if (lane == 0) {
                __threadfence();
                st_release(fl + i * a.nj2 + j, stamp);
            }
        }
    }
}

// Serial vertical Thomas recurrence and relaxed back-substitution of one column, run by lane 0
// on the warp's shared rows (U-prognostic-microscale_1.cs:485-524): rows A, B, C, D, phi.
__device__ __forceinline__ void thomas_relax(float (*S)[KMAX_LEVELS], int K0, int KK, int VI, int kkm,
                                             float relax) {
    float P = 0.0f, Q = 0.0f;
    for (int k = K0; k <= VI; ++k) {
        const float A = S[0][k], B = S[1][k], C = S[2][k], D = S[3][k];
        if (k > KK + 1) {
            const float T = 1.0f / (A - C * P);
            P = B * T;
            Q = (D + C * Q) * T;
        } else {
            const float T = 1.0f / A;
            P = B * T;
            Q = D * T;
        }
        S[1][k] = P;
        S[3][k] = Q;
    }
    float up = S[4][VI + 1];
    for (int k = VI; k >= K0; --k) {
        float u = S[4][k];
        if (kkm < k) {
            u += relax * (S[1][k] * up + S[3][k] - u);
            S[4][k] = u;
        }
        up = u;
    }
}

enum { COMP_U = 0, COMP_V = 1, COMP_W = 2 };

template <int COMP, bool IL>
__device__ __forceinline__ Coef ml_level(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc, int k) {
    if (COMP == COMP_U) return u1_level<IL>(a, x, c, sc, k);
    if (COMP == COMP_V) return v1_level<IL>(a, x, c, sc, k);
    return w1_level<IL>(a, x, c, sc, k);
}

template <int COMP>
__device__ __forceinline__ int back_limit(const ColCtx &c) {
    // U back-substitution skips levels at or below max(KKART, KKART[i-1][j]) (:513-524), V the
    // same with j-1; W updates every level from KSTART (W-...1.cs:444-448).
    return COMP == COMP_U ? c.kkm_u : (COMP == COMP_V ? c.kkm_v : -32768);
}

template <int COMP>
__device__ __forceinline__ float *comp_field(const KArgs &a) {
    return COMP == COMP_U ? a.uk : (COMP == COMP_V ? a.vk : a.wk);
}

// ---------------------------- plain family -------------------------------------------------

template <int COMP>
__device__ void plain_ml_column(const KArgs &a, int s, int i, int j, float (*S)[KMAX_LEVELS]) {
    const int lane = threadIdx.x & 31;
    const ColCtx c = make_col(a, i, j);
    if (!(c.fl & F_ADV) || !a.sit[s].active) return;
    const SitCtx sc = make_sit(a, s);
    const Acc<false> x = make_acc<false>(a, s, c.col);
    float *F = comp_field<COMP>(a);
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k < c.K0 || k > c.VI) continue;
        const Coef q = ml_level<COMP, false>(a, x, c, sc, k);
        S[0][k] = q.A; S[1][k] = q.B; S[2][k] = q.C; S[3][k] = q.D; S[4][k] = q.phi;
    }
    if (lane == 0) S[4][c.VI + 1] = __ldcg(F + x.at(0, c.VI + 1));
    __syncwarp();
    const int kkm = back_limit<COMP>(c);
    if (lane == 0) thomas_relax(S, c.K0, c.KK, c.VI, kkm, a.relax);
    __syncwarp();
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k >= c.K0 && k <= c.VI && kkm < k) __stcg(F + x.at(0, k), S[4][k]);
    }
}

// Pressure correction (PrognosticFlowfield.cs:804-901).  The reference's PIMP/QIMP buffer lives
// per sweep row and is not cleared between columns, so the top level reads P/Q at
// VerticalIndex+1 left by an earlier column of the same row (:865-868); the row carry buffer
// reproduces that.  Row carry of the plain family: [s][j][2][KS].
__device__ void plain_pressure_column(const KArgs &a, int s, int i, int j, int IS, int JS, bool first,
                                      float (*S)[KMAX_LEVELS]) {
    const int lane = threadIdx.x & 31;
    const int ks = a.ks;
    float *rc = a.rowcarry + ((size_t)s * a.nj2 + j) * 2 * ks;
    if (first) {
        for (int k = lane; k < 2 * ks; k += 32) __stcg(rc + k, 0.0f);
        __threadfence_block();
        __syncwarp();
    }
    const ColCtx c = make_col(a, i, j);
    if (!(c.fl & F_ADV) || !a.sit[s].active) return;
    const SitCtx sc = make_sit(a, s);
    const Acc<false> x = make_acc<false>(a, s, c.col);
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k <= c.KK || k > c.VI) continue;
        S[3][k] = pressure_dim<false>(a, x, c, sc, k, IS, JS);
    }
    __syncwarp();
    if (lane == 0) {
        float P = __ldcg(rc + c.VI + 1), Q = __ldcg(rc + ks + c.VI + 1);
        for (int k = c.VI; k > c.KK; --k) {
            const float T = 1.0f / (a.app[k] - a.atp[k] * P);
            P = a.abp[k] * T;
            Q = (a.atp[k] * Q + S[3][k]) * T;
            S[1][k] = P;
            S[2][k] = Q;
        }
        float prev = 0.0f;                                         // DPM[KKART] is always 0
        for (int k = c.KK + 1; k <= c.VI; ++k) {
            prev = S[1][k] * prev + S[2][k];
            S[4][k] = prev;
        }
    }
    __syncwarp();
    unsigned dmax = 0;
    const int klo = max(c.KK, a.vi_min);
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k <= c.KK || k > c.VI) continue;
        const float temp = S[4][k];
        dmax = max(dmax, residual_key(temp, sc));
        __stcg(a.dpm + x.at(0, k), temp);
        a.dpmnew[x.at(0, k)] += a.relaxp * temp;
        if (k > klo) {
            __stcg(rc + k, S[1][k]);
            __stcg(rc + ks + k, S[2][k]);
        }
    }
    for (int d = 16; d > 0; d >>= 1) dmax = max(dmax, __shfl_xor_sync(0xffffffffu, dmax, d));
    if (lane == 0 && dmax > 0) atomicMax(&a.sit[s].dumax_bits, dmax);
}

__global__ void __launch_bounds__(GS_WARPS * 32) k_pressure(KArgs a, SweepGeom g) {
    __shared__ float sm[GS_WARPS][SM_ROWS][KMAX_LEVELS];
    float (*S)[KMAX_LEVELS] = sm[threadIdx.x >> 5];
    gs_tasks<PH_PRESSURE, false, false>(a, g, [&](int s, int i, int j, int IS, int JS, bool first) {
        plain_pressure_column(a, s, i, j, IS, JS, first, S);
    });
}

template <int COMP>
__global__ void __launch_bounds__(GS_WARPS * 32) k_mom_ml(KArgs a, SweepGeom g) {
    __shared__ float sm[GS_WARPS][SM_ROWS][KMAX_LEVELS];
    float (*S)[KMAX_LEVELS] = sm[threadIdx.x >> 5];
    constexpr int PH = COMP == COMP_U ? PH_U : (COMP == COMP_V ? PH_V : PH_W);
    gs_tasks<PH, COMP == COMP_V, false>(a, g, [&](int s, int i, int j, int, int, bool) {
        plain_ml_column<COMP>(a, s, i, j, S);
    });
}

// ---------------------------- batched family -----------------------------------------------
// One block per task = (group of 32 situations, column).  The block's warps split the levels for
// the coefficient assembly (lane = situation, contiguous 128-byte loads in the interleaved layout)
// and write A, B, C, D, phi rows [k][32] to shared memory; warp 0 then runs the 32 situations'
// Thomas recurrences and back-substitutions side by side.

// Shared rows of one task, [k][32] each, carved from dynamic shared memory sized by KS.
struct BRows {
    float *A, *B, *C, *D, *phi;
    __device__ __forceinline__ float &a(int k, int l) { return A[k * 32 + l]; }
    __device__ __forceinline__ float &b(int k, int l) { return B[k * 32 + l]; }
    __device__ __forceinline__ float &c(int k, int l) { return C[k * 32 + l]; }
    __device__ __forceinline__ float &d(int k, int l) { return D[k * 32 + l]; }
    __device__ __forceinline__ float &p(int k, int l) { return phi[k * 32 + l]; }
};

__device__ __forceinline__ BRows carve_rows(float *smem, int ks) {
    BRows R;
    R.A = smem; R.B = R.A + ks * 32; R.C = R.B + ks * 32; R.D = R.C + ks * 32; R.phi = R.D + ks * 32;
    return R;
}

// Block-wide variant of gs_tasks: thread 0 claims and waits, the block works, thread 0 publishes.
template <int PHASE, bool REVERSE, class Body>
__device__ __forceinline__ void gs_tasks_block(const KArgs &a, const SweepGeom &g, Body &&body) {
    __shared__ unsigned s_base;
    __shared__ int s_ok;
    const unsigned units = (unsigned)a.group_n;
    const unsigned total = (unsigned)g.diag_start[g.ndiag] * units;
    unsigned int *ctr = a.counters + 8 * a.ctr_slot + PHASE;
    const int it = *a.it_global;
    int IS, JS;
    sweep_dir(it, IS, JS);
    if (REVERSE) { IS = -IS; JS = -JS; }
    const int stamp = it * 8 + PHASE;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0)
            s_base = (*(volatile int *)a.err != ERR_NONE) ? 0xffffffffu : atomicAdd(ctr, (unsigned)a.chunk);
        __syncthreads();
        const unsigned base = s_base;
        if (base >= total) break;
        const unsigned end = min(total, base + (unsigned)a.chunk);
        for (unsigned t = base; t < end; ++t) {
            int grp, i1, j1;
            decode_task(t, g, units, grp, i1, j1);
            grp += a.group_lo;
            const int i = (IS == 1) ? i1 : a.nii - i1 + 1;
            const int j = (JS == 1) ? j1 : a.njj - j1 + 1;
            int *fl = a.flags + (size_t)grp * a.ncols;
            if (threadIdx.x == 0) {
                int ok = 1;
                if (i1 > g.ia) ok = wait_stamp(fl + (i - IS) * a.nj2 + j, stamp, a.err, a.wait_limit_ns);
                if (ok && j1 > g.ja) ok = wait_stamp(fl + i * a.nj2 + (j - JS), stamp, a.err, a.wait_limit_ns);
                s_ok = ok;
            }
            __syncthreads();
            if (s_ok) body(grp, i, j, IS, JS, i1 == g.ia);
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                st_release(fl + i * a.nj2 + j, stamp);
            }
        }
    }
}

template <int COMP, int NW>
__device__ void batch_ml_column(const KArgs &a, int grp, int i, int j, BRows R) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = grp * 32 + lane;
    const ColCtx c = make_col(a, i, j);
    if (!(c.fl & F_ADV)) return;
    const bool act = (s < a.nb) && a.sit[s].active;
    const Acc<true> x = make_acc<true>(a, act ? s : grp * 32, c.col);
    if (act) {
        const SitCtx sc = make_sit(a, s);
#pragma unroll 2
        for (int k = c.K0 + warp; k <= c.VI; k += NW) {
            const Coef q = ml_level<COMP, true>(a, x, c, sc, k);
            R.a(k, lane) = q.A; R.b(k, lane) = q.B; R.c(k, lane) = q.C; R.d(k, lane) = q.D; R.p(k, lane) = q.phi;
        }
    }
    __syncthreads();
    if (warp != 0 || !act) return;
    float *F = comp_field<COMP>(a);
    float P = 0.0f, Q = 0.0f;
    for (int k = c.K0; k <= c.VI; ++k) {
        const float A = R.a(k, lane), B = R.b(k, lane), C = R.c(k, lane), D = R.d(k, lane);
        if (k > c.KK + 1) {
            const float T = 1.0f / (A - C * P);
            P = B * T;
            Q = (D + C * Q) * T;
        } else {
            const float T = 1.0f / A;
            P = B * T;
            Q = D * T;
        }
        R.b(k, lane) = P;
        R.d(k, lane) = Q;
    }
    const int kkm = back_limit<COMP>(c);
    const float relax = a.relax;
    float up = __ldcg(F + x.at(0, c.VI + 1));
    for (int k = c.VI; k >= c.K0; --k) {
        float u = R.p(k, lane);
        if (kkm < k) {
            u += relax * (R.b(k, lane) * up + R.d(k, lane) - u);
            __stcg(F + x.at(0, k), u);
        }
        up = u;
    }
}

// Row carry of the batched family: [group][j][2][KS][32].
template <int NW>
__device__ void batch_pressure_column(const KArgs &a, int grp, int i, int j, int IS, int JS, bool first, BRows R,
                                      unsigned &nmax_acc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = grp * 32 + lane;
    const int ks = a.ks;
    float *rc = a.rowcarry + (((size_t)grp * a.nj2 + j) * 2 * ks) * 32 + lane;
    if (first && warp == 0)
        for (int k = 0; k < 2 * ks; ++k) __stcg(rc + (size_t)k * 32, 0.0f);
    const ColCtx c = make_col(a, i, j);
    if (!(c.fl & F_ADV)) return;
    const bool act = (s < a.nb) && a.sit[s].active;
    const Acc<true> x = make_acc<true>(a, act ? s : grp * 32, c.col);
    const SitCtx sc = make_sit(a, act ? s : grp * 32);
    if (act)
        for (int k = c.KK + 1 + warp; k <= c.VI; k += NW) R.d(k, lane) = pressure_dim<true>(a, x, c, sc, k, IS, JS);
    __syncthreads();
    if (warp == 0 && act) {
        float P = __ldcg(rc + (size_t)(c.VI + 1) * 32), Q = __ldcg(rc + (size_t)(ks + c.VI + 1) * 32);
        for (int k = c.VI; k > c.KK; --k) {
            const float T = 1.0f / (a.app[k] - a.atp[k] * P);
            P = a.abp[k] * T;
            Q = (a.atp[k] * Q + R.d(k, lane)) * T;
            R.b(k, lane) = P;
            R.c(k, lane) = Q;
        }
        float prev = 0.0f;                                         // DPM[KKART] is always 0
        for (int k = c.KK + 1; k <= c.VI; ++k) {
            prev = R.b(k, lane) * prev + R.c(k, lane);
            R.p(k, lane) = prev;
        }
    }
    __syncthreads();
    if (!act) return;
    const int klo = max(c.KK, a.vi_min);
    unsigned nmax = 0;
    for (int k = c.KK + 1 + warp; k <= c.VI; k += NW) {
        const float temp = R.p(k, lane);
        nmax = max(nmax, residual_key(temp, sc));
        __stcg(a.dpm + x.at(0, k), temp);
        a.dpmnew[x.at(0, k)] += a.relaxp * temp;
        if (k > klo) {
            __stcg(rc + (size_t)k * 32, R.b(k, lane));
            __stcg(rc + (size_t)(ks + k) * 32, R.c(k, lane));
        }
    }
    nmax_acc = max(nmax_acc, nmax);
}

template <int NW, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB) k_pressure_b(KArgs a, SweepGeom g) {
    extern __shared__ float smem[];
    BRows R = carve_rows(smem, a.ks);
    __shared__ unsigned red[NW][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned nmax = 0;
    int cur = -1;
    auto flush = [&]() {
        // block-reduce the residual keys of the current group and publish one atomic per situation
        red[warp][lane] = nmax;
        __syncthreads();
        if (warp == 0 && cur >= 0) {
            unsigned m = 0;
            for (int w = 0; w < NW; ++w) m = max(m, red[w][lane]);
            const int s = cur * 32 + lane;
            if (m > 0 && s < a.nb) atomicMax(&a.sit[s].dumax_bits, m);
        }
        __syncthreads();
        nmax = 0;
    };
    gs_tasks_block<PH_PRESSURE, false>(a, g, [&](int grp, int i, int j, int IS, int JS, bool first) {
        if (grp != cur) { flush(); cur = grp; }
        batch_pressure_column<NW>(a, grp, i, j, IS, JS, first, R, nmax);
    });
    flush();
}

template <int COMP, int NW, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB) k_mom_ml_b(KArgs a, SweepGeom g) {
    extern __shared__ float smem[];
    BRows R = carve_rows(smem, a.ks);
    constexpr int PH = COMP == COMP_U ? PH_U : (COMP == COMP_V ? PH_V : PH_W);
    gs_tasks_block<PH, COMP == COMP_V>(a, g, [&](int grp, int i, int j, int, int, bool) {
        batch_ml_column<COMP, NW>(a, grp, i, j, R);
    });
}

// Launch variants of the batched family: (warps per block, minimum resident blocks per SM).
// The host times them once per context and keeps the fastest (GRAL_PROG_BATCH_VARIANT forces one).
struct BVariant {
    int nw, minb;
    void (*pressure)(KArgs, SweepGeom);
    void (*mom[3])(KArgs, SweepGeom);
};

#define GRAL_BV(NW, MB)                                                                          \
    BVariant{NW, MB, k_pressure_b<NW, MB>,                                                       \
             {k_mom_ml_b<COMP_U, NW, MB>, k_mom_ml_b<COMP_V, NW, MB>, k_mom_ml_b<COMP_W, NW, MB>}}

const BVariant kVariants[] = {GRAL_BV(8, 2), GRAL_BV(4, 4), GRAL_BV(4, 6)};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

}  // namespace

int gs_num_variants() { return kNumVariants; }

int gs_block_threads(bool il, int variant) { return il ? kVariants[variant].nw * 32 : GS_WARPS * 32; }

size_t gs_smem_bytes(bool il, int ks, int variant) {
    (void)variant;
    return il ? (size_t)5 * ks * 32 * sizeof(float) : 0;
}

cudaError_t gs_prepare(bool il, int ks) {
    if (!il) return cudaSuccess;
    const int bytes = (int)gs_smem_bytes(true, ks, 0);
    for (int v = 0; v < kNumVariants; ++v) {
        const BVariant &V = kVariants[v];
        cudaError_t e = cudaFuncSetAttribute(V.pressure, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        for (int q = 0; q < 3 && e == cudaSuccess; ++q)
            e = cudaFuncSetAttribute(V.mom[q], cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t gs_occupancy(bool il, int kind, int ks, int variant, int *blocks_per_sm) {
    const int th = gs_block_threads(il, variant);
    if (!il) {
        switch (kind) {
            case PH_PRESSURE: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_pressure, th, 0);
            case PH_U: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_mom_ml<COMP_U>, th, 0);
            case PH_V: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_mom_ml<COMP_V>, th, 0);
            default: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_mom_ml<COMP_W>, th, 0);
        }
    }
    const BVariant &V = kVariants[variant];
    const size_t sm = gs_smem_bytes(true, ks, variant);
    void (*f)(KArgs, SweepGeom) = (kind == PH_PRESSURE) ? V.pressure : V.mom[kind == PH_U ? 0 : (kind == PH_V ? 1 : 2)];
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, f, th, sm);
}

// Group sets of the batched family: a launch sweeps group_set groups at a time (0 = all groups),
// each launch with its own task counter.
template <class F>
void for_group_sets(const KArgs &a, F &&f) {
    const int gs = (a.group_set <= 0) ? a.ngroups : a.group_set;
    int slot = 0;
    for (int lo = 0; lo < a.ngroups; lo += gs, ++slot) {
        KArgs b = a;
        b.group_lo = lo;
        b.group_n = std::min(gs, a.ngroups - lo);
        b.ctr_slot = slot;
        f(b);
    }
}

void launch_pressure(const KArgs &a, const SweepGeom &g, int grid, cudaStream_t st) {
    if (a.il) {
        const BVariant &V = kVariants[a.variant];
        for_group_sets(a, [&](const KArgs &b) {
            V.pressure<<<grid, V.nw * 32, gs_smem_bytes(true, a.ks, a.variant), st>>>(b, g);
        });
    } else {
        k_pressure<<<grid, GS_WARPS * 32, 0, st>>>(a, g);
    }
}

void launch_mom_ml(int comp, const KArgs &a, const SweepGeom &g, int grid, cudaStream_t st) {
    if (a.il) {
        const BVariant &V = kVariants[a.variant];
        for_group_sets(a, [&](const KArgs &b) {
            V.mom[comp]<<<grid, V.nw * 32, gs_smem_bytes(true, a.ks, a.variant), st>>>(b, g);
        });
    } else {
        if (comp == 0) k_mom_ml<COMP_U><<<grid, GS_WARPS * 32, 0, st>>>(a, g);
        else if (comp == 1) k_mom_ml<COMP_V><<<grid, GS_WARPS * 32, 0, st>>>(a, g);
        else k_mom_ml<COMP_W><<<grid, GS_WARPS * 32, 0, st>>>(a, g);
    }
}

}  // namespace gral
