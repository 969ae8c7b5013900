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
constexpr int SM_ROWS = 5;       // shared rows per warp of the plain family: A, B, C, D, phi (model 1: rows 0-3 hold 16-byte level records)

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
            if (lane == 0)
                ok = wait_stamps((i1 > g.ia) ? fl + (i - IS) * a.nj2 + j : nullptr,
                                 (j1 > g.ja) ? fl + i * a.nj2 + (j - JS) : nullptr, stamp, a.err, a.wait_limit_ns);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            __syncwarp();
            if (ok) body(u, i, j, IS, JS, i1 == g.ia);
            __syncwarp();
            if (lane == 0) st_release(fl + i * a.nj2 + j, stamp);
        }
    }
}

enum { COMP_U = 0, COMP_V = 1, COMP_W = 2 };

template <int COMP, bool IL, int SW = 0>
__device__ __forceinline__ Coef ml_level(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc, int k) {
    if (COMP == COMP_U) return u1_level<IL, SW>(a, x, c, sc, k);
    if (COMP == COMP_V) return v1_level<IL, SW>(a, x, c, sc, k);
    return w1_level<IL, SW>(a, x, c, sc, k);
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

// Coefficients of one level for model MODEL (0 no diffusion, 1 mixing length, 2 k-eps); SW as
// for the model-1 routines.
template <int MODEL, int COMP, bool IL, int SW = 0>
__device__ __forceinline__ Coef mom_level(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc, int k) {
    if (MODEL == 1) return ml_level<COMP, IL, SW>(a, x, c, sc, k);
    if (COMP == COMP_W) return w_scalar_level<MODEL == 2, IL>(a, x, c, sc, k);
    return uv_scalar_level<MODEL == 2, COMP, IL>(a, x, c, sc, k);
}

// Vertical Thomas recurrence and relaxed back-substitution of one situation's column on rows
// R.a/b/c/d/p (A, B, C, D, phi): model 1 multiplies by 1/(A - C*P) (U-prognostic-microscale_1.cs:
// 485-504), models 2 and 0 divide twice (U-prognostic-microscale_2.cs:247-256), and the model-0
// W routine keeps P and Q in double (W-prognostic-microscale_0.cs:35-36, 124-139).  phi is
// replaced by the new values on the levels the reference updates.
template <int MODEL, int COMP, class Rows>
__device__ __forceinline__ void mom_sweep(Rows &R, int K0, int KK, int VI, int kkm, float relax, float top) {
    if (MODEL == 0 && COMP == COMP_W) {
        double P = 0.0, Q = 0.0;
        for (int k = K0; k <= VI; ++k) {
            const float A = R.a(k), B = R.b(k), C = R.c(k), D = R.d(k);
            if (k > KK + 1) {
                const double den = (double)A - (double)C * P;
                const double Pn = (double)B / den;
                Q = ((double)D + (double)C * Q) / den;
                P = Pn;
            } else {
                P = (double)(B / A);
                Q = (double)(D / A);
            }
            R.pd(k) = P;
            R.qd(k) = Q;
        }
        float up = top;
        for (int k = VI; k >= K0; --k) {
            float u = R.p(k);
            u += (float)((double)relax * (R.pd(k) * (double)up + R.qd(k) - (double)u));
            R.p(k) = u;
            up = u;
        }
        return;
    }
    // float recurrences, eight levels per step (operands loaded together, arithmetic chain serial)
    constexpr int CH = 8;
    auto level = [&](int k, float A, float B, float C, float D, float &P, float &Q) {
        if (k > KK + 1) {
            if (MODEL == 1) {
                const float T = 1.0f / (A - C * P);
                P = B * T;
                Q = (D + C * Q) * T;
            } else {
                const float Pn = B / (A - C * P);
                Q = (D + C * Q) / (A - C * P);
                P = Pn;
            }
        } else {
            if (MODEL == 1) {
                const float T = 1.0f / A;
                P = B * T;
                Q = D * T;
            } else {
                P = B / A;
                Q = D / A;
            }
        }
    };
    float P = 0.0f, Q = 0.0f;
    int k = K0;
    for (; k + CH - 1 <= VI; k += CH) {
        float A[CH], B[CH], C[CH], D[CH];
#pragma unroll
        for (int q = 0; q < CH; ++q) { A[q] = R.a(k + q); B[q] = R.b(k + q); C[q] = R.c(k + q); D[q] = R.d(k + q); }
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            level(k + q, A[q], B[q], C[q], D[q], P, Q);
            B[q] = P;
            D[q] = Q;
        }
#pragma unroll
        for (int q = 0; q < CH; ++q) { R.b(k + q) = B[q]; R.d(k + q) = D[q]; }
    }
    for (; k <= VI; ++k) {
        level(k, R.a(k), R.b(k), R.c(k), R.d(k), P, Q);
        R.b(k) = P;
        R.d(k) = Q;
    }
    float up = top;
    k = VI;
    for (; k - (CH - 1) >= K0; k -= CH) {
        float Pv[CH], Qv[CH], U[CH];
#pragma unroll
        for (int q = 0; q < CH; ++q) { Pv[q] = R.b(k - q); Qv[q] = R.d(k - q); U[q] = R.p(k - q); }
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            float u = U[q];
            if (kkm < k - q) u += relax * (Pv[q] * up + Qv[q] - u);
            U[q] = u;
            up = u;
        }
#pragma unroll
        for (int q = 0; q < CH; ++q) R.p(k - q) = U[q];
    }
    for (; k >= K0; --k) {
        float u = R.p(k);
        if (kkm < k) {
            u += relax * (R.b(k) * up + R.d(k) - u);
            R.p(k) = u;
        }
        up = u;
    }
}

// k and eps: two recurrences with divisions sharing A, then the back-substitution with the wall
// functions of ground, roof and the four neighbour walls, and the clamps
// (TKE-prognostic-microscale.cs:255-347).  Rows: a, b1, c1, d1, b2, c2, d2, k1 (TURB), e1 (TDISS);
// vel(field, dc, k) loads UK/VK/WK of the column (dc = 0) or its east/north neighbour.
template <class Rows, class Vel>
__device__ __forceinline__ void tke_sweep(Rows &R, const KArgs &a, const ColCtx &c, const ColKE &ke, float ktop,
                                          float etop, Vel &&vel) {
    const int K0 = c.K0, KK = c.KK, VI = c.VI;
    float PT = 0.0f, QT = 0.0f, PE = 0.0f, QE = 0.0f;
    for (int k = K0; k <= VI; ++k) {
        const float A = R.a(k), B1 = R.b1(k), C1 = R.c1(k), D1 = R.d1(k);
        const float B2 = R.b2(k), C2 = R.c2(k), D2 = R.d2(k);
        if (k > KK + 1) {
            const float PTn = B1 / (A - C1 * PT);
            QT = (D1 + C1 * QT) / (A - C1 * PT);
            PT = PTn;
            const float PEn = B2 / (A - C2 * PE);
            QE = (D2 + C2 * QE) / (A - C2 * PE);
            PE = PEn;
        } else {
            PT = B1 / A; QT = D1 / A; PE = B2 / A; QE = D2 / A;
        }
        R.b1(k) = PT; R.d1(k) = QT; R.b2(k) = PE; R.d2(k) = QE;
    }
    const long long E = c.nj2, N = 1;
    auto hyp = [](double p, double q) { return sqrt(p * p + q * q); };
    float kup = ktop, eup = etop;
    for (int k = VI; k >= K0; --k) {
        float kn = R.k1(k), en = R.e1(k);
        if (KK < k) {
            float U;
            bool wall = true;
            double div;   // TDISS divisor
            if (k == KK + 1 && (c.fl & F_CUTK0)) {
                if (c.fl & F_GMODE1) {
                    U = (float)(ke.gfac * hyp(0.5 * (double)(vel(0, 0, k + 1) + vel(0, E, k + 1)),
                                              0.5 * (double)(vel(1, 0, k + 1) + vel(1, N, k + 1))));
                    div = ((double)a.dzk[k] + (double)a.dzk[k + 1] * 0.5) * 0.4;
                } else {
                    U = (float)(ke.gfac * hyp(0.5 * (double)((vel(0, 0, k + 1)) + vel(0, E, k)),
                                              0.5 * (double)((vel(1, 0, k)) + vel(1, N, k))));
                    div = (double)a.dzk[k] * 0.5 * 0.4;
                }
            } else if (k == KK + 1 && (c.fl & F_CUTKGT0)) {
                U = c.cf.help_o * (float)hyp(0.5 * (double)(vel(0, 0, k) + vel(0, E, k)),
                                             0.5 * (double)(vel(1, 0, k) + vel(1, N, k)));
                div = (double)a.dzk[k] * 0.5 * 0.4;
            } else if (k == ke.kw_e || k == ke.kw_w) {
                U = (float)((double)a.ustern_fx * hyp(0.5 * (double)(vel(2, 0, k) + vel(2, 0, k + 1)),
                                                      0.5 * (double)(vel(1, 0, k) + vel(1, N, k))));
                div = (double)a.building_z0 * 0.4;
            } else if (k == ke.kw_n || k == ke.kw_s) {
                U = (float)((double)a.ustern_fx * hyp(0.5 * (double)(vel(2, 0, k) + vel(2, 0, k + 1)),
                                                      0.5 * (double)(vel(0, 0, k) + vel(0, E, k))));
                div = (double)a.building_z0 * 0.4;
            } else {
                wall = false;
                kn = R.b1(k) * kup + R.d1(k);
                en = R.b2(k) * eup + R.d2(k);
            }
            if (wall) {
                kn = (float)(3.33 * (double)(U * U));
                en = (float)((double)(U * U * U) / div);
            }
            kn = (float)net_maxd((double)kn, 0.001);
            en = (float)net_maxd((double)en, 0.0000001);
            R.k1(k) = kn;
            R.e1(k) = en;
        }
        kup = kn;
        eup = en;
    }
}

// ---------------------------- plain family -------------------------------------------------

struct PlainRows {
    float (*S)[KMAX_LEVELS];
    double (*SD)[KMAX_LEVELS];
    __device__ __forceinline__ float &a(int k) { return S[0][k]; }
    __device__ __forceinline__ float &b(int k) { return S[1][k]; }
    __device__ __forceinline__ float &c(int k) { return S[2][k]; }
    __device__ __forceinline__ float &d(int k) { return S[3][k]; }
    __device__ __forceinline__ float &p(int k) { return S[4][k]; }
    __device__ __forceinline__ double &pd(int k) { return SD[0][k]; }
    __device__ __forceinline__ double &qd(int k) { return SD[1][k]; }
    // TKE rows
    __device__ __forceinline__ float &b1(int k) { return S[1][k]; }
    __device__ __forceinline__ float &c1(int k) { return S[2][k]; }
    __device__ __forceinline__ float &d1(int k) { return S[3][k]; }
    __device__ __forceinline__ float &k1(int k) { return S[4][k]; }
    __device__ __forceinline__ float &b2(int k) { return S[5][k]; }
    __device__ __forceinline__ float &c2(int k) { return S[6][k]; }
    __device__ __forceinline__ float &d2(int k) { return S[7][k]; }
    __device__ __forceinline__ float &e1(int k) { return S[8][k]; }
};

template <int MODEL, int COMP>
__device__ void plain_mom_column(const KArgs &a, int s, int i, int j, float (*S)[KMAX_LEVELS],
                                 double (*SD)[KMAX_LEVELS]) {
    const int lane = threadIdx.x & 31;
    const ColCtx c = make_col(a, i, j);
    if (!(c.fl & F_ADV) || !a.sit[s].active) return;
    const SitCtx sc = make_sit(a, s);
    const Acc<false> x = make_acc<false>(a, s, c.col);
    float *F = comp_field<COMP>(a);
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k < c.K0 || k > c.VI) continue;
        const Coef q = mom_level<MODEL, COMP, false>(a, x, c, sc, k);
        S[0][k] = q.A; S[1][k] = q.B; S[2][k] = q.C; S[3][k] = q.D; S[4][k] = q.phi;
    }
    __syncwarp();
    const int kkm = back_limit<COMP>(c);
    if (lane == 0) {
        PlainRows R{S, SD};
        mom_sweep<MODEL, COMP>(R, c.K0, c.KK, c.VI, kkm, a.relax, __ldcg(F + x.at(0, c.VI + 1)));
    }
    __syncwarp();
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k >= c.K0 && k <= c.VI && kkm < k) __stcg(F + x.at(0, k), S[4][k]);
    }
}

__device__ void plain_tke_column(const KArgs &a, int s, int i, int j, float (*S)[KMAX_LEVELS]) {
    const int lane = threadIdx.x & 31;
    const ColCtx c = make_col(a, i, j);
    if (!(c.fl & F_ADV) || !a.sit[s].active) return;
    const SitCtx sc = make_sit(a, s);
    const Acc<false> x = make_acc<false>(a, s, c.col);
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k < c.K0 || k > c.VI) continue;
        const CoefKE q = tke_level<false>(a, x, c, sc, k);
        S[0][k] = q.A; S[1][k] = q.B1; S[2][k] = q.C1; S[3][k] = q.D1; S[4][k] = q.k1;
        S[5][k] = q.B2; S[6][k] = q.C2; S[7][k] = q.D2; S[8][k] = q.e1;
    }
    __syncwarp();
    if (lane == 0) {
        PlainRows R{S, nullptr};
        const ColKE ke = a.colke[c.col];
        const float *vf[3] = {a.uk, a.vk, a.wk};
        tke_sweep(R, a, c, ke, __ldcg(a.turb + x.at(0, c.VI + 1)), __ldcg(a.tdiss + x.at(0, c.VI + 1)),
                  [&](int f, long long dc, int k) { return vf[f][x.at(dc, k)]; });
    }
    __syncwarp();
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k >= c.K0 && k <= c.VI && c.KK < k) {
            __stcg(a.turb + x.at(0, k), S[4][k]);
            __stcg(a.tdiss + x.at(0, k), S[8][k]);
        }
    }
}

template <int MODEL, int COMP>
__global__ void __launch_bounds__(GS_WARPS * 32) k_mom(KArgs a, SweepGeom g) {
    __shared__ __align__(16) float sm[GS_WARPS][SM_ROWS][KMAX_LEVELS];
    __shared__ double smd[(MODEL == 0 && COMP == COMP_W) ? GS_WARPS : 1][2][KMAX_LEVELS];
    const int w = threadIdx.x >> 5;
    float (*S)[KMAX_LEVELS] = sm[w];
    double (*SD)[KMAX_LEVELS] = smd[(MODEL == 0 && COMP == COMP_W) ? w : 0];
    constexpr int PH = COMP == COMP_U ? PH_U : (COMP == COMP_V ? PH_V : PH_W);
    constexpr bool REV = (MODEL == 1 && COMP == COMP_V);     // model-1 V sweeps with (-IS,-JS)
    gs_tasks<PH, REV, false>(a, g, [&](int s, int i, int j, int, int, bool) {
        plain_mom_column<MODEL, COMP>(a, s, i, j, S, SD);
    });
}

__global__ void __launch_bounds__(GS_WARPS * 32) k_tke(KArgs a, SweepGeom g) {
    __shared__ float sm[GS_WARPS][9][KMAX_LEVELS];
    float (*S)[KMAX_LEVELS] = sm[threadIdx.x >> 5];
    gs_tasks<PH_TKE, false, false>(a, g, [&](int s, int i, int j, int, int, bool) {
        plain_tke_column(a, s, i, j, S);
    });
}

// ---------------------------- plain family, split tasks ------------------------------------
// Model-1 momentum and the pressure correction run each column task in two halves around the
// wait: `pre` does everything that does not read values the column's Gauss-Seidel predecessors
// write (coefficients, sources, the Thomas forward elimination of the momentum equations), `post`
// reads the predecessors' results and finishes the column.  Only `post` sits on the wavefront's
// critical path; `pre` overlaps the predecessors' work.  Results are bit-identical to the unsplit
// evaluation (the operations and their order are the same).

// Sweep orders of the diagnostic pressure solve by IterationLoops % 4 (DiagnosticFlowfield.cs:94-
// 315): 0 rows and columns ascending, 1 rows descending, 2 both descending, 3 columns descending.
__device__ __forceinline__ void diag_dir(int it, int &IS, int &JS) {
    const int m = it % 4;
    IS = (m == 2 || m == 3) ? -1 : 1;
    JS = (m == 1 || m == 2) ? -1 : 1;
}

template <int PHASE, bool REVERSE, class Job>
__device__ __forceinline__ void gs_tasks_split(const KArgs &a, const SweepGeom &g, Job &job) {
    const int lane = threadIdx.x & 31;
    const unsigned units = (unsigned)*a.nact;
    const unsigned total = (unsigned)g.diag_start[g.ndiag] * units;
    unsigned int *ctr = a.counters + PHASE;
    const int it = (PHASE == PH_DIAG) ? a.diag_iter : *a.it_global;
    int IS, JS;
    if (PHASE == PH_DIAG) diag_dir(it, IS, JS);
    else sweep_dir(it, IS, JS);
    if (REVERSE) { IS = -IS; JS = -JS; }
    const int stamp = it * 8 + PHASE;
    job.stamp = stamp;
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
            u = a.act[u];
            const int i = (IS == 1) ? i1 : a.nii - i1 + 1;
            const int j = (JS == 1) ? j1 : a.njj - j1 + 1;
            int *fl = a.flags + (size_t)u * a.ncols;
            job.pre(u, i, j, IS, JS, i1 == g.ia);
            int ok = 1;
            if (lane == 0)      // spins without sleeping: these waits sit on the sweep's critical path
                ok = wait_stamps((i1 > g.ia) ? fl + (i - IS) * a.nj2 + j : nullptr,
                                 (j1 > g.ja) ? fl + i * a.nj2 + (j - JS) : nullptr, stamp, a.err, a.wait_limit_ns,
                                 0);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            __syncwarp();
            if (ok) job.post(u, IS, JS);
            __syncwarp();
            if (lane == 0) st_release(fl + i * a.nj2 + j, stamp);
        }
    }
    job.finish();
}

// Model-1 Thomas recurrence split at the wait (U-prognostic-microscale_1.cs:485-524).  Each level's
// operands are one 16-byte record L[k] = {A -> T, C, D -> Q, B -> P} in shared memory (the level's
// old value phi in a row of its own), so lane 0 reads a level with one load.  Before the wait, A, B
// become T = 1/(A - C*P) and P; after it, D becomes Q and the relaxed back-substitution updates
// phi.  Lane 0 runs the recurrences eight levels at a time: the eight levels' records are loaded
// together, so only the arithmetic chain is serial.
constexpr int TCH = 8;

__device__ __forceinline__ void ml_forward(float4 *L, int K0, int KK, int VI) {
    float P = 0.0f;
    int k = K0;
    for (; k + TCH - 1 <= VI; k += TCH) {
        float4 r[TCH];
#pragma unroll
        for (int q = 0; q < TCH; ++q) r[q] = L[k + q];
#pragma unroll
        for (int q = 0; q < TCH; ++q) {
            const float T = (k + q > KK + 1) ? 1.0f / (r[q].x - r[q].y * P) : 1.0f / r[q].x;
            P = r[q].w * T;
            r[q].x = T;
            r[q].w = P;
        }
#pragma unroll
        for (int q = 0; q < TCH; ++q) L[k + q] = r[q];
    }
    for (; k <= VI; ++k) {
        float4 r = L[k];
        const float T = (k > KK + 1) ? 1.0f / (r.x - r.y * P) : 1.0f / r.x;
        P = r.w * T;
        r.x = T;
        r.w = P;
        L[k] = r;
    }
}

__device__ __forceinline__ void ml_backward(float4 *L, float *U0, int K0, int KK, int VI, int kkm, float relax,
                                            float top) {
    // Q_k = D_k*T_k up to KKART+1 (K0 <= KKART+1 always), then Q_k = (D_k + C_k*Q_{k-1})*T_k;
    // the level ranges are split instead of selecting per level, which keeps the chain short
    const int kq = min(KK + 1, VI);
    for (int k = K0; k <= kq; ++k) L[k].z = L[k].z * L[k].x;
    float Q = L[kq].z;
    int k = kq + 1;
    for (; k + TCH - 1 <= VI; k += TCH) {
        float4 r[TCH];
#pragma unroll
        for (int q = 0; q < TCH; ++q) r[q] = L[k + q];
#pragma unroll
        for (int q = 0; q < TCH; ++q) {
            Q = (r[q].z + r[q].y * Q) * r[q].x;
            r[q].z = Q;
        }
#pragma unroll
        for (int q = 0; q < TCH; ++q) L[k + q].z = r[q].z;
    }
    for (; k <= VI; ++k) {
        Q = (L[k].z + L[k].y * Q) * L[k].x;
        L[k].z = Q;
    }
    // relaxed back-substitution downwards over the levels above kkm (the others keep their value
    // and lie below every updated level)
    const int kb = max(K0, kkm + 1);
    float up = top;
    k = VI;
    for (; k - (TCH - 1) >= kb; k -= TCH) {
        float4 r[TCH];
        float U[TCH];
#pragma unroll
        for (int q = 0; q < TCH; ++q) { r[q] = L[k - q]; U[q] = U0[k - q]; }
#pragma unroll
        for (int q = 0; q < TCH; ++q) {
            const float u = U[q] + relax * (r[q].w * up + r[q].z - U[q]);
            U[q] = u;
            up = u;
        }
#pragma unroll
        for (int q = 0; q < TCH; ++q) U0[k - q] = U[q];
    }
    for (; k >= kb; --k) {
        const float u = U0[k] + relax * (L[k].w * up + L[k].z - U0[k]);
        U0[k] = u;
        up = u;
    }
}

template <int COMP>
struct Mom1Job {
    const KArgs &a;
    float (*S)[KMAX_LEVELS];
    int stamp;
    ColCtx c;
    Acc<false> x;
    bool act;
    float top;          // the column's value at VerticalIndex+1 (not swept)
    MomPre p[2];
    float own[2];       // strip schedule: the swept field's column at levels lane, lane+32 (final after post)
    float suc[2][2];    // strip schedule: the sweep successors (i+IS, j), (i, j+JS) at the task's levels
    static constexpr bool kAllFlags = false;   // no task of another column waits on this phase's flags

    // the level records of the recurrences: rows 0-3 of the warp's shared memory, 16-byte aligned
    __device__ __forceinline__ float4 *lev() const { return reinterpret_cast<float4 *>(S[0]); }

    __device__ void pre(int s, int i, int j, int, int, bool) {
        const int lane = threadIdx.x & 31;
        c = make_col(a, i, j);
        act = (c.fl & F_ADV) && a.sit[s].active;
        if (!act) return;
        const SitCtx sc = make_sit(a, s);
        x = make_acc<false>(a, s, c.col);
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (k < c.K0 || k > c.VI) continue;
            if (COMP == COMP_U) p[r] = u1_pre<false>(a, x, c, sc, k);
            else if (COMP == COMP_V) p[r] = v1_pre<false>(a, x, c, sc, k);
            else p[r] = w1_pre<false>(a, x, c, sc, k);
            lev()[k] = make_float4(p[r].A, p[r].C, 0.0f, p[r].B);
            S[4][k] = p[r].phi;
        }
        __syncwarp();
        if (lane == 0) {
            top = __ldcg(comp_field<COMP>(a) + x.at(0, c.VI + 1));
            ml_forward(lev(), c.K0, c.KK, c.VI);
        }
    }

    // Strip schedule: besides pre(), the column's values at every level (for the shared-memory copy
    // the next tasks of the strip read) and the successors' old values, so that after the wait only
    // the predecessors' values are read.  Neither changes before this task finishes.
    __device__ void pre_strip(int s, int i, int j, int IS, int JS, bool first) {
        pre(s, i, j, IS, JS, first);
        const int lane = threadIdx.x & 31;
        const float *F = comp_field<COMP>(a);
        const size_t base = ((size_t)s * a.ncols + (size_t)(i * a.nj2 + j)) * a.ks;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            own[r] = (k < a.ks) ? __ldcg(F + base + k) : 0.0f;
            if (act && k >= c.K0 && k <= c.VI) {
                suc[r][0] = __ldcg(F + x.at((long long)IS * c.nj2, k));
                suc[r][1] = __ldcg(F + x.at((long long)JS, k));
            }
        }
    }

    // pI, pJ (strip schedule): this sweep's values of the predecessors (i-IS, j), (i, j-JS) in
    // shared memory, or null to read them from the field.
    __device__ void post(int, int IS, int JS, bool strip = false, const float *pI = nullptr, const float *pJ = nullptr) {
        if (!act) return;
        const int lane = threadIdx.x & 31;
        float *F = comp_field<COMP>(a);
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (k < c.K0 || k > c.VI) continue;
            float nW, nS, nE, nN;
            if (strip) {
                const float vI = pI ? pI[k] : __ldcg(F + x.at(-(long long)IS * c.nj2, k));
                const float vJ = pJ ? pJ[k] : __ldcg(F + x.at(-(long long)JS, k));
                nW = (IS == 1) ? vI : suc[r][0];
                nE = (IS == 1) ? suc[r][0] : vI;
                nS = (JS == 1) ? vJ : suc[r][1];
                nN = (JS == 1) ? suc[r][1] : vJ;
            } else {
                nbr4(F, x, c, k, nW, nS, nE, nN);
            }
            if (COMP == COMP_U) lev()[k].z = u1_post(p[r], c, k, nW, nS, nE, nN, a.simd == 16);
            else if (COMP == COMP_V) lev()[k].z = v1_post(p[r], c, k, nW, nS, nE, nN, a.simd == 16);
            else lev()[k].z = w1_post(p[r], c, k, nW, nS, nE, nN, a.simd == 16);
        }
        __syncwarp();
        const int kkm = back_limit<COMP>(c);
        if (lane == 0) ml_backward(lev(), S[4], c.K0, c.KK, c.VI, kkm, a.relax, top);
        __syncwarp();
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (k < c.K0 || k > c.VI) continue;
            const float v = S[4][k];
            own[r] = v;
            if (kkm < k) __stcg(F + x.at(0, k), v);
        }
    }

    __device__ void finish() {}
};

template <int COMP>
__global__ void __launch_bounds__(GS_WARPS * 32) k_mom1s(KArgs a, SweepGeom g) {
    __shared__ __align__(16) float sm[GS_WARPS][SM_ROWS][KMAX_LEVELS];
    Mom1Job<COMP> job{a, sm[threadIdx.x >> 5], 0};
    constexpr int PH = COMP == COMP_U ? PH_U : (COMP == COMP_V ? PH_V : PH_W);
    gs_tasks_split<PH, COMP == COMP_V>(a, g, job);     // model-1 V sweeps with (-IS,-JS)
}

// Pressure correction (PrognosticFlowfield.cs:804-901).  The reference's PIMP/QIMP buffer lives per
// sweep row and is not cleared between columns, so the top level reads P/Q at VerticalIndex+1 left
// by an earlier column of the same row (:865-868); the row carry buffer [s][j][2][KS] reproduces
// that, zeroed by the first column of each row.
// Split at the wait.  Before it: the divergence terms and the downward Thomas elimination, which
// starts from the carry's P at VerticalIndex+1: zero when no earlier column of the row writes that
// level (a host-built table names the last writer), else read after waiting for that writer --
// an ancestor of this column in the wavefront, usually finished long before; the carry's Q at that
// level comes from the same writer and is read there too.  After the wait: the swept neighbours'
// DPM, Q from that start, the back-substitution, the residual and the stores.
struct PressJob {
    const KArgs &a;
    float (*S)[KMAX_LEVELS];
    int stamp;
    ColCtx c;
    Acc<false> x;
    SitCtx sc;
    float *rc;
    bool act;
    float t0[2];
    float dn[2];        // DPMNEW of the column (only this task updates it)
    unsigned run_max;   // residual key maximum of this warp's tasks of situation run_s so far
    int run_s;
    float own[2];       // strip schedule: the column's DPM at levels lane, lane+32 (final after post)
    float q0;           // lane 0: the row carry's Q at VerticalIndex+1
    static constexpr bool kAllFlags = true;    // the row carry's readers wait on its writer's flag

    // The residual maximum is only read after the phase (k_bookkeeping), so each warp keeps a
    // running maximum and publishes it once per situation instead of once per column.
    __device__ void flush() {
        if ((threadIdx.x & 31) == 0 && run_s >= 0 && run_max > 0) atomicMax(&a.sit[run_s].dumax_bits, run_max);
        run_max = 0;
    }
    __device__ void finish() { flush(); }

    // the level records of the recurrences, 16 bytes each in rows 0-3 of the warp's shared memory:
    // {T, P, DIM -> Q, ATP}; row 4 holds the new DPM
    __device__ __forceinline__ float4 *lev() const { return reinterpret_cast<float4 *>(S[0]); }

    // T = 1/(APP - ATP*P), P = ABP*T from level VI down to KKART+1, eight levels per step.
    __device__ void forward(float P) {
        float4 *L = lev();
        int k = c.VI;
        for (; k - (TCH - 1) > c.KK; k -= TCH) {
            float ap[TCH], at[TCH], ab[TCH];
#pragma unroll
            for (int q = 0; q < TCH; ++q) { ap[q] = a.app[k - q]; at[q] = a.atp[k - q]; ab[q] = a.abp[k - q]; }
#pragma unroll
            for (int q = 0; q < TCH; ++q) {
                const float T = 1.0f / (ap[q] - at[q] * P);
                P = ab[q] * T;
                ap[q] = T;
                ab[q] = P;
            }
#pragma unroll
            for (int q = 0; q < TCH; ++q) L[k - q] = make_float4(ap[q], ab[q], 0.0f, at[q]);
        }
        for (; k > c.KK; --k) {
            const float T = 1.0f / (a.app[k] - a.atp[k] * P);
            P = a.abp[k] * T;
            L[k] = make_float4(T, P, 0.0f, a.atp[k]);
        }
    }

    __device__ void pre(int s, int i, int j, int IS, int, bool first) {
        const int lane = threadIdx.x & 31;
        const int ks = a.ks;
        rc = a.rowcarry + ((size_t)s * a.nj2 + j) * 2 * ks;
        if (first) {
            for (int k = lane; k < 2 * ks; k += 32) __stcg(rc + k, 0.0f);
            __threadfence_block();
            __syncwarp();
        }
        c = make_col(a, i, j);
        act = (c.fl & F_ADV) && a.sit[s].active;
        if (!act) return;
        sc = make_sit(a, s);
        x = make_acc<false>(a, s, c.col);
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (k <= c.KK || k > c.VI) continue;
            t0[r] = pressure_pre<false>(a, x, c, sc, k);
            dn[r] = a.dpmnew[x.at(0, k)];
        }
        if (lane == 0) {
            const short2 w = a.rcw[c.col];
            const int wi = (IS == 1) ? w.x : w.y;
            // the carry's P and Q at VerticalIndex+1 are final once their writer, the last column
            // before this one in its row that writes that level, has finished (zero without one)
            float P0 = 0.0f;
            q0 = 0.0f;
            if (wi >= 0) {
                const int *fl = a.flags + (size_t)s * a.ncols;
                if (wait_stamp(fl + wi * a.nj2 + j, stamp, a.err, a.wait_limit_ns)) {
                    P0 = __ldcg(rc + c.VI + 1);
                    q0 = __ldcg(rc + a.ks + c.VI + 1);
                }
            }
            forward(P0);
        }
    }

    // Strip schedule: besides pre(), the column's DPM at every level for the shared-memory copy
    // the next tasks of the strip read (unchanged before this task finishes).
    __device__ void pre_strip(int s, int i, int j, int IS, int JS, bool first) {
        pre(s, i, j, IS, JS, first);
        const int lane = threadIdx.x & 31;
        const size_t base = ((size_t)s * a.ncols + (size_t)(i * a.nj2 + j)) * a.ks;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            own[r] = (k < a.ks) ? __ldcg(a.dpm + base + k) : 0.0f;
        }
    }

    // pI, pJ (strip schedule): this sweep's DPM of the predecessors (i-IS, j), (i, j-JS) in shared
    // memory, or null to read them from the field.
    __device__ void post(int s, int IS, int JS, bool strip = false, const float *pI = nullptr, const float *pJ = nullptr) {
        if (!act) return;
        const int lane = threadIdx.x & 31;
        const int ks = a.ks;
        float Q = 0.0f;
        if (lane == 0) Q = q0;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (k <= c.KK || k > c.VI) continue;
            const float vI = (strip && pI) ? pI[k] : __ldcg(a.dpm + x.at(-(long long)IS * c.nj2, k));
            const float vJ = (strip && pJ) ? pJ[k] : __ldcg(a.dpm + x.at(-(long long)JS, k));
            lev()[k].z = pressure_post_v(a, t0[r], k, IS, JS, vI, vJ);
        }
        __syncwarp();
        if (lane == 0) {
            float4 *L = lev();
            int k = c.VI;
            for (; k - (TCH - 1) > c.KK; k -= TCH) {
                float4 r[TCH];
#pragma unroll
                for (int q = 0; q < TCH; ++q) r[q] = L[k - q];
#pragma unroll
                for (int q = 0; q < TCH; ++q) {
                    Q = (r[q].w * Q + r[q].z) * r[q].x;
                    r[q].z = Q;
                }
#pragma unroll
                for (int q = 0; q < TCH; ++q) L[k - q].z = r[q].z;
            }
            for (; k > c.KK; --k) {
                Q = (L[k].w * Q + L[k].z) * L[k].x;
                L[k].z = Q;
            }
            float prev = 0.0f;                                     // DPM[KKART] is always 0
            k = c.KK + 1;
            for (; k + TCH - 1 <= c.VI; k += TCH) {
                float4 r[TCH];
                float qq[TCH];
#pragma unroll
                for (int q = 0; q < TCH; ++q) r[q] = L[k + q];
#pragma unroll
                for (int q = 0; q < TCH; ++q) {
                    prev = r[q].y * prev + r[q].z;
                    qq[q] = prev;
                }
#pragma unroll
                for (int q = 0; q < TCH; ++q) S[4][k + q] = qq[q];
            }
            for (; k <= c.VI; ++k) {
                prev = L[k].y * prev + L[k].z;
                S[4][k] = prev;
            }
        }
        __syncwarp();
        unsigned dmax = 0;
        const int klo = max(c.KK, a.vi_min);
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (k <= c.KK || k > c.VI) continue;
            const float temp = S[4][k];
            own[r] = temp;
            dmax = max(dmax, residual_key(temp, sc));
            __stcg(a.dpm + x.at(0, k), temp);
            a.dpmnew[x.at(0, k)] = dn[r] + a.relaxp * temp;
            if (k > klo) {
                const float4 r = lev()[k];
                __stcg(rc + k, r.y);
                __stcg(rc + ks + k, r.z);
            }
        }
        for (int d = 16; d > 0; d >>= 1) dmax = max(dmax, __shfl_xor_sync(0xffffffffu, dmax, d));
        if (s != run_s) {
            flush();
            run_s = s;
        }
        run_max = max(run_max, dmax);
    }
};

__global__ void __launch_bounds__(GS_WARPS * 32) k_pressure_s(KArgs a, SweepGeom g) {
    __shared__ __align__(16) float sm[GS_WARPS][SM_ROWS][KMAX_LEVELS];
    PressJob job{a, sm[threadIdx.x >> 5], 0};
    job.run_max = 0;
    job.run_s = -1;
    gs_tasks_split<PH_PRESSURE, false>(a, g, job);
}

// ---------------------------- strip schedule, slab family -------------------------------------
// The same split tasks, scheduled by strips of sweep rows.  A block claims a strip (one situation,
// SR consecutive rows i1) from an atomic counter, in order, and runs it column by column: warp
// (r, m) takes row r's columns j1 = ja+m, ja+m+SMW, ...  A task's row predecessor (i1, j1-1) is
// then another warp of the block, and so is its column predecessor (i1-1, j1) unless r = 0.  Those
// hand-offs go through per-row progress counters in shared memory (CTA-scope release/acquire)
// instead of a global flag's round trips through L2; only a strip's first row waits on a global
// flag, published by the previous strip's last row.  Every task still publishes its global flag,
// after the shared counter, for the waits of other tasks on it (the pressure row carry's writer).
// Strips are claimed in order and a strip only waits on earlier ones, so no co-residency is
// assumed.  While one warp of a row waits and solves, the row's other warps evaluate the pre-wait
// parts of its next columns.

__device__ __forceinline__ int ld_acquire_cta(const int *p) {
    int v;
    asm volatile("ld.acquire.cta.shared::cta.s32 %0, [%1];"
                 : "=r"(v)
                 : "r"((unsigned)__cvta_generic_to_shared(p))
                 : "memory");
    return v;
}
__device__ __forceinline__ void st_release_cta(int *p, int v) {
    asm volatile("st.release.cta.shared::cta.s32 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(p)), "r"(v)
                 : "memory");
}

// Spin (one thread) until the shared progress counter *cnt reaches `need`.  Bounded like
// wait_stamps: gives up after limit_ns or on another warp's error and returns false then.
__device__ inline bool wait_count(const int *cnt, int need, int *err, unsigned long long limit_ns) {
    if (ld_acquire_cta(cnt) >= need) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (unsigned n = 1;; ++n) {
        if (ld_acquire_cta(cnt) >= need) return true;
        if ((n & 15) == 0) {
            if (*(volatile int *)err != ERR_NONE) return false;
            if (globaltimer_ns() - t0 > limit_ns) {
                atomicCAS(err, ERR_NONE, ERR_TIMEOUT);
                return false;
            }
        }
    }
}

// Shared-memory copies of finished columns: a ring of SDEPTH slots per row of the strip, slot
// c % SDEPTH holding the swept field of the row's column c at every level.  A task reads its row
// predecessor's slot and, for r > 0, its column predecessor's slot of the row above; before it
// overwrites a slot, the row below must have finished the column that slot held.
constexpr int SDEPTH = 4;

// Lanes 0..n-1 each wait on one flag (relaxed polls, all in flight together), then every lane
// issues the acquire fence that completes the acquire pattern; true if all flags reached their
// stamp.
__device__ __forceinline__ bool wait_lanes(const KArgs &a, const int *flag, int stamp, bool mine) {
    bool ok = true;
    if (mine) ok = wait_stamps(flag, nullptr, stamp, a.err, a.wait_limit_ns);
    return __all_sync(0xffffffffu, ok);
}

// The sweep rows i1_first + r (r = 0..SR-1; rows outside the geometry are skipped) of one strip,
// run by warps w = r*SMW + m of a group of SR*SMW warps.  With AVW, a column first waits until the
// averages of its 3x3 neighbourhood are done (the U part of the fused strip kernel).
template <int SR, int SMW, bool AVW, class Job>
__device__ __forceinline__ void strip_run(const KArgs &a, const SweepGeom &g, Job &job, int w, int u, int i1_first,
                                          int IS, int JS, int stamp, int *s_done, float (*s_col)[KMAX_LEVELS]) {
    const int lane = threadIdx.x & 31;
    const int r = w / SMW, m = w % SMW;
    const int i1 = i1_first + r;
    if (i1 < g.ia || i1 >= g.ia + g.ni) return;
    const int i = (IS == 1) ? i1 : a.nii - i1 + 1;
    int *fl = a.flags + (size_t)u * a.ncols;
    const bool above = i1 > g.ia;                            // a predecessor row exists
    const bool above_here = above && r > 0;                  // ... and runs in this block
    const bool below = r + 1 < SR && i1 + 1 < g.ia + g.ni;   // the row below runs in this block
    const bool last = r == SR - 1 || i1 + 1 == g.ia + g.ni;  // the next strip's first row reads this one
    const int sAV = stamp - PH_U + PH_AV;
    for (int c = m; c < g.nj; c += SMW) {
        const int j1 = g.ja + c;
        const int j = (JS == 1) ? j1 : a.njj - j1 + 1;
        bool okav = true;
        if (AVW) {
            const int wi = i + (lane % 3) - 1, wj = j + (lane / 3) - 1;
            const bool mine = lane < 9 && wi >= 2 && wi <= a.nii - 1 && wj >= 2 && wj <= a.njj - 1;
            okav = wait_lanes(a, fl + wi * a.nj2 + wj, sAV, mine);
            __syncwarp();
        }
        job.pre_strip(u, i, j, IS, JS, i1 == g.ia);
        int ok = okav;
        if (lane == 0 && ok) {
            ok = wait_count(s_done + r, c, a.err, a.wait_limit_ns);
            if (ok && above_here) ok = wait_count(s_done + r - 1, c + 1, a.err, a.wait_limit_ns);
            else if (ok && above)
                ok = wait_stamps(fl + (i - IS) * a.nj2 + j, nullptr, stamp, a.err, a.wait_limit_ns, 0);
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        __syncwarp();
        if (ok)
            job.post(u, IS, JS, true, above_here ? s_col[(r - 1) * SDEPTH + c % SDEPTH] : nullptr,
                     (c > 0) ? s_col[r * SDEPTH + (c - 1) % SDEPTH] : nullptr);
        if (lane == 0 && below && c >= SDEPTH) wait_count(s_done + r + 1, c - SDEPTH + 1, a.err, a.wait_limit_ns);
        __syncwarp();
        float *slot = s_col[r * SDEPTH + c % SDEPTH];
        slot[lane] = job.own[0];
        if (lane + 32 < KMAX_LEVELS) slot[lane + 32] = job.own[1];
        __syncwarp();
        if (lane == 0) {
            st_release_cta(s_done + r, c + 1);
            if (Job::kAllFlags || last) st_release(fl + i * a.nj2 + j, stamp);
        }
    }
}

template <int PHASE, bool REVERSE, int SR, int SMW, class Job>
__device__ __forceinline__ void gs_tasks_strip(const KArgs &a, const SweepGeom &g, Job &job, int *s_done,
                                               unsigned *s_claim, float (*s_col)[KMAX_LEVELS]) {
    const unsigned units = (unsigned)*a.nact;
    const unsigned total = (unsigned)((g.ni + SR - 1) / SR) * units;
    unsigned int *ctr = a.counters + PHASE;
    const int it = *a.it_global;
    int IS, JS;
    sweep_dir(it, IS, JS);
    if (REVERSE) { IS = -IS; JS = -JS; }
    const int stamp = it * 8 + PHASE;
    job.stamp = stamp;
    for (;;) {
        if (threadIdx.x == 0) *s_claim = (*(volatile int *)a.err != ERR_NONE) ? 0xffffffffu : atomicAdd(ctr, 1u);
        if (threadIdx.x < SR) s_done[threadIdx.x] = 0;
        __syncthreads();
        const unsigned t = *s_claim;
        if (t >= total) break;
        strip_run<SR, SMW, false>(a, g, job, threadIdx.x >> 5, a.act[t % units], g.ia + (int)(t / units) * SR, IS, JS,
                                  stamp, s_done, s_col);
        __syncthreads();
    }
    job.finish();
}

// ------------------------ fused strips: pressure -> velocity correction -> averages -> U --------
// One launch claims, in order, pressure strip 0, U strip 0, pressure strip 1, U strip 1, ...,
// and a last U strip.  Pressure strip s (16 warps) runs sweep rows ia + 4s .. ia + 4s + 3 as
// k_pressure_strip.  U strip s runs the velocity corrections of the rows one behind (ia + 4s - 1
// ...), the averages of the rows two behind and the U sweep of the rows three behind: warps 0-3
// take one velocity-correction row and one averages row each, in column order (the averages two
// columns behind), and warps 4-15 the U rows on the strip schedule (3 warps per row), each U column
// first waiting until the averages of its 3x3 neighbourhood are done.  The dependencies across
// cells are those of k_fused_pvau and go through the global flags (stamps it*8 + kind): velocity
// correction (i,j) after pressure at (i,j), (i-1,j), (i,j-1); averages (i,j) after the velocity
// corrections at (i,j), (i+1,j), (i,j+1); U (i,j) after the averages of its 3x3 neighbourhood.  With
// those row offsets every wait is on a strip claimed earlier: a velocity correction reads the
// pressure of at most the next row, an average the velocity correction of at most the next row,
// and U the averages of at most the next row.
constexpr int FSR = 4;     // rows per strip

__global__ void __launch_bounds__(16 * 32, 1) k_fused_strip(KArgs a, FusedGeom fg) {
    __shared__ __align__(16) float sm[16][SM_ROWS][KMAX_LEVELS];
    __shared__ float s_col[FSR * SDEPTH][KMAX_LEVELS];
    __shared__ int s_done[FSR];
    __shared__ unsigned s_claim;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const SweepGeom &gp = fg.gp, &gu = fg.gu;
    const int it = *a.it_global;
    int IS, JS;
    sweep_dir(it, IS, JS);
    const int sP = it * 8 + PH_PRESSURE, sVC = it * 8 + PH_VC, sAV = it * 8 + PH_AV, sU = it * 8 + PH_U;
    PressJob pj{a, sm[warp], sP};
    pj.run_max = 0;
    pj.run_s = -1;
    Mom1Job<COMP_U> uj{a, sm[warp], sU};
    const unsigned units = (unsigned)*a.nact;
    const int np = (gp.ni + FSR - 1) / FSR;
    const unsigned total = (unsigned)(2 * np + 1) * units;
    unsigned int *ctr = a.counters + PH_PRESSURE;
    const int ilo = 2, ihi = a.nii - 1, jlo = 2, jhi = a.njj - 1;   // velocity correction / averages range
    for (;;) {
        if (threadIdx.x == 0) s_claim = (*(volatile int *)a.err != ERR_NONE) ? 0xffffffffu : atomicAdd(ctr, 1u);
        if (threadIdx.x < FSR) s_done[threadIdx.x] = 0;
        __syncthreads();
        const unsigned t = s_claim;
        if (t >= total) break;
        const int item = (int)(t / units), u = a.act[t % units];
        const bool pstrip = item < 2 * np && (item & 1) == 0;
        const int s = pstrip ? item / 2 : (item < 2 * np ? item / 2 : np);
        const int base = gp.ia + s * FSR;
        if (pstrip) {
            strip_run<FSR, 4, false>(a, gp, pj, warp, u, base, IS, JS, sP, s_done, s_col);
        } else if (warp >= 4) {
            strip_run<FSR, 3, true>(a, gu, uj, warp - 4, u, base - 3, IS, JS, sU, s_done, s_col);
        } else {
            int *fl = a.flags + (size_t)u * a.ncols;
            const bool act = a.sit[u].active != 0;
            const int iv1 = base - 1 + warp, ia1 = base - 2 + warp;   // sweep rows of this warp
            const bool vrow = iv1 >= gp.ia && iv1 < gp.ia + gp.ni, arow = ia1 >= gp.ia && ia1 < gp.ia + gp.ni;
            const int iv = (IS == 1) ? iv1 : a.nii - iv1 + 1, ia = (IS == 1) ? ia1 : a.nii - ia1 + 1;
            // columns in chunks of VCH: the chunk's three dependency flags per column are polled by
            // lanes 3q..3q+2 together, the columns run one after the other, and lanes q publish
            // their column's flag; the averages trail the velocity corrections by one chunk
            constexpr int VCH = 4;
            const int q = lane / 3, k3 = lane % 3;
            for (int c0 = 0; c0 < gp.nj + VCH; c0 += VCH) {
                if (vrow && c0 < gp.nj) {
                    const int nc = min(VCH, gp.nj - c0);
                    bool mine = false;
                    const int *fp = fl;
                    if (q < nc) {
                        const int j1 = gp.ja + c0 + q, j = (JS == 1) ? j1 : a.njj - j1 + 1;
                        const int wi = (k3 == 1) ? iv - 1 : iv, wj = (k3 == 2) ? j - 1 : j;
                        mine = wi >= ilo && wj >= jlo;
                        fp = fl + wi * a.nj2 + wj;
                    }
                    const bool ok = wait_lanes(a, fp, sP, mine);
                    __syncwarp();
                    for (int qq = 0; qq < nc; ++qq) {
                        const int j1 = gp.ja + c0 + qq, j = (JS == 1) ? j1 : a.njj - j1 + 1;
                        const int col = iv * a.nj2 + j;
                        if (ok && act) velcorr_col<false>(a, u, col, iv, j, make_acc<false>(a, u, col), lane, 32);
                    }
                    __syncwarp();
                    if (lane < nc) {
                        const int j1 = gp.ja + c0 + lane, j = (JS == 1) ? j1 : a.njj - j1 + 1;
                        st_release(fl + iv * a.nj2 + j, sVC);
                    }
                }
                const int ca = c0 - VCH;
                if (arow && ca >= 0 && ca < gp.nj) {
                    const int nc = min(VCH, gp.nj - ca);
                    bool mine = false;
                    const int *fp = fl;
                    if (q < nc) {
                        const int j1 = gp.ja + ca + q, j = (JS == 1) ? j1 : a.njj - j1 + 1;
                        const int wi = (k3 == 1) ? ia + 1 : ia, wj = (k3 == 2) ? j + 1 : j;
                        mine = wi <= ihi && wj <= jhi;
                        fp = fl + wi * a.nj2 + wj;
                    }
                    const bool ok = wait_lanes(a, fp, sVC, mine);
                    __syncwarp();
                    for (int qq = 0; qq < nc; ++qq) {
                        const int j1 = gp.ja + ca + qq, j = (JS == 1) ? j1 : a.njj - j1 + 1;
                        const int col = ia * a.nj2 + j;
                        if (ok && act) average_col<false>(a, col, ia, j, make_acc<false>(a, u, col), lane, 32);
                    }
                    __syncwarp();
                    if (lane < nc) {
                        const int j1 = gp.ja + ca + lane, j = (JS == 1) ? j1 : a.njj - j1 + 1;
                        st_release(fl + ia * a.nj2 + j, sAV);
                    }
                }
            }
        }
        __syncthreads();
    }
    pj.finish();
}

template <int SR, int SMW>
__global__ void __launch_bounds__(SR * SMW * 32, 1) k_pressure_strip(KArgs a, SweepGeom g) {
    __shared__ __align__(16) float sm[SR * SMW][SM_ROWS][KMAX_LEVELS];
    __shared__ float s_col[SR * SDEPTH][KMAX_LEVELS];
    __shared__ int s_done[SR];
    __shared__ unsigned s_claim;
    PressJob job{a, sm[threadIdx.x >> 5], 0};
    job.run_max = 0;
    job.run_s = -1;
    gs_tasks_strip<PH_PRESSURE, false, SR, SMW>(a, g, job, s_done, &s_claim, s_col);
}

template <int COMP, int SR, int SMW>
__global__ void __launch_bounds__(SR * SMW * 32, 1) k_mom1_strip(KArgs a, SweepGeom g) {
    __shared__ __align__(16) float sm[SR * SMW][SM_ROWS][KMAX_LEVELS];
    __shared__ float s_col[SR * SDEPTH][KMAX_LEVELS];
    __shared__ int s_done[SR];
    __shared__ unsigned s_claim;
    Mom1Job<COMP> job{a, sm[threadIdx.x >> 5], 0};
    constexpr int PH = COMP == COMP_U ? PH_U : (COMP == COMP_V ? PH_V : PH_W);
    gs_tasks_strip<PH, COMP == COMP_V, SR, SMW>(a, g, job, s_done, &s_claim, s_col);   // model-1 V sweeps with (-IS,-JS)
}

// ---------------------------- fused wavefront, slab family --------------------------------
// Pressure, velocity correction, averages and the model-1 U sweep of one iteration in one launch.
// U sweeps in the pressure's direction and reads only the averages of its 3x3 neighbourhood, so
// its front can trail the pressure front by a few diagonals instead of a whole phase.  Step s of
// the task list holds the pressure tasks of diagonal s, the velocity corrections of diagonal s-1,
// the averages of s-2 and the U tasks of U-diagonal s-5 (P-diagonal s-4): every dependency of a
// task lies in an earlier step or an earlier segment of its step, so claiming in list order stays
// deadlock-free.  Dependencies (actual coordinates, stamps it*8 + kind):
//   velocity correction (i,j) after pressure at (i,j), (i-1,j), (i,j-1)  -- it reads their DPM and
//                         overwrites U/V/W that pressure tasks (i-1,j), (i,j-1) read for DIV;
//   averages (i,j) after the velocity corrections at (i,j), (i+1,j), (i,j+1);
//   U (i,j) after the averages of the 3x3 neighbourhood (which also covers the corrected U/V/W and
//   final DPMNEW it reads) and its two U sweep predecessors.

__global__ void __launch_bounds__(GS_WARPS * 32) k_fused_pvau(KArgs a, FusedGeom fg) {
    __shared__ __align__(16) float sm[GS_WARPS][SM_ROWS][KMAX_LEVELS];
    float (*S)[KMAX_LEVELS] = sm[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int it = *a.it_global;
    int IS, JS;
    sweep_dir(it, IS, JS);
    const int sP = it * 8 + PH_PRESSURE, sVC = it * 8 + PH_VC, sAV = it * 8 + PH_AV, sU = it * 8 + PH_U;
    PressJob pj{a, S, sP};
    pj.run_max = 0;
    pj.run_s = -1;
    Mom1Job<COMP_U> uj{a, S, sU};
    const unsigned units = (unsigned)*a.nact;
    const unsigned total = (unsigned)fg.seg_start[fg.nseg] * units;
    unsigned int *ctr = a.counters + PH_PRESSURE;
    const int ilo = 2, ihi = a.nii - 1, jlo = 2, jhi = a.njj - 1;   // velocity correction / averages range
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(ctr, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= total) break;
        if (*(volatile int *)a.err != ERR_NONE) break;
        int kind, uu, i1, j1;
        {   // segment by binary search over the starts (in columns, times the number of units)
            int lo = 0, hi = fg.nseg;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if ((unsigned)fg.seg_start[mid] * units <= t) lo = mid; else hi = mid;
            }
            const int code = fg.seg_code[lo];
            kind = code & 7;
            const int d = code >> 3;
            const SweepGeom &g = (kind == PH_U) ? fg.gu : fg.gp;
            const unsigned len = (unsigned)(g.diag_start[d + 1] - g.diag_start[d]);
            const unsigned r = t - (unsigned)fg.seg_start[lo] * units;
            uu = (int)(r / len);
            const int pos = (int)(r % len);
            const int ioff = max(0, d - (g.nj - 1)) + pos;
            i1 = g.ia + ioff;
            j1 = g.ja + d - ioff;
        }
        const int s = a.act[uu];
        const int i = (IS == 1) ? i1 : a.nii - i1 + 1;
        const int j = (JS == 1) ? j1 : a.njj - j1 + 1;
        int *fl = a.flags + (size_t)s * a.ncols;
        const int col = i * a.nj2 + j;
        int stamp;
        if (kind == PH_PRESSURE) {
            stamp = sP;
            pj.pre(s, i, j, IS, JS, i1 == fg.gp.ia);
            bool ok = true;
            if (lane == 0)
                ok = wait_stamps((i1 > fg.gp.ia) ? fl + (i - IS) * a.nj2 + j : nullptr,
                                 (j1 > fg.gp.ja) ? fl + i * a.nj2 + (j - JS) : nullptr, sP, a.err, a.wait_limit_ns);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            __syncwarp();
            if (ok) pj.post(s, IS, JS);
        } else if (kind == PH_VC) {
            stamp = sVC;
            const int wi = (lane == 1) ? i - 1 : i, wj = (lane == 2) ? j - 1 : j;
            const bool mine = lane < 3 && wi >= ilo && wj >= jlo;
            const bool ok = wait_lanes(a, fl + wi * a.nj2 + wj, sP, mine);
            __syncwarp();
            if (ok && a.sit[s].active) velcorr_col<false>(a, s, col, i, j, make_acc<false>(a, s, col), lane, 32);
        } else if (kind == PH_AV) {
            stamp = sAV;
            const int wi = (lane == 1) ? i + 1 : i, wj = (lane == 2) ? j + 1 : j;
            const bool mine = lane < 3 && wi <= ihi && wj <= jhi;
            const bool ok = wait_lanes(a, fl + wi * a.nj2 + wj, sVC, mine);
            __syncwarp();
            if (ok && a.sit[s].active) average_col<false>(a, col, i, j, make_acc<false>(a, s, col), lane, 32);
        } else {
            stamp = sU;
            const int wi = i + (lane % 3) - 1, wj = j + (lane / 3) - 1;
            const bool mine = lane < 9 && wi >= ilo && wi <= ihi && wj >= jlo && wj <= jhi;
            bool ok = wait_lanes(a, fl + wi * a.nj2 + wj, sAV, mine);
            __syncwarp();
            if (ok) {
                uj.pre(s, i, j, IS, JS, false);
                if (lane == 0)
                    ok = wait_stamps((i1 > fg.gu.ia) ? fl + (i - IS) * a.nj2 + j : nullptr,
                                     (j1 > fg.gu.ja) ? fl + i * a.nj2 + (j - JS) : nullptr, sU, a.err,
                                     a.wait_limit_ns);
                ok = __shfl_sync(0xffffffffu, ok, 0);
                __syncwarp();
                if (ok) uj.post(s, IS, JS);
            }
        }
        __syncwarp();
        if (lane == 0) st_release(fl + col, stamp);
    }
    pj.finish();
}

// DiagnosticFlowfield.Calculate's pressure sweep (DiagnosticFlowfield.cs:86-315) on the full-height
// fields after a prognostic solve: every column of the sweep range, levels KKART+1..NKK-1, the four
// neighbours' DPM of this sweep or the last one (plain Gauss-Seidel, DPM zeroed once before the
// first iteration), PIMP/QIMP at NKK zero, no quantisation and no residual.  Split at the wait
// like the prognostic pressure: divergence and forward elimination before it, the neighbours'
// DPM, Q and the back-substitution after.  Rows per warp (dynamic shared memory, KS = NKK+2):
// T, P, Q, D, DPM, DIV/DTIME.
struct DiagJob {
    const KArgs &a;
    float *R;
    int stamp;
    const DiagTabs &t;
    int col, KK, top;
    Acc<false> x;
    float DT;

    __device__ float &row(int r, int k) { return R[r * a.ks + k]; }

    __device__ void pre(int s, int i, int j, int, int, bool) {
        const int lane = threadIdx.x & 31;
        const long long E = a.nj2, N = 1;
        const float DXK = a.dxk, DYK = a.dyk;
        col = i * a.nj2 + j;
        KK = a.meta[col].kkart;
        top = a.nkk - 1;
        x = make_acc<false>(a, s, col);
        DT = t.dtime[s];
        for (int k = KK + 1 + lane; k <= top; k += 32) {
            const float u0 = a.uk[x.at(0, k)], uE = a.uk[x.at(E, k)], v0 = a.vk[x.at(0, k)], vN = a.vk[x.at(N, k)];
            const float w0 = a.wk[x.at(0, k)], wT = a.wk[x.at(0, k + 1)];
            const float dz = t.dzk[k];
            const float DIV = (k > KK + 1) ? (u0 - uE) * DYK * dz + (v0 - vN) * DXK * dz + (w0 - wT) * DXK * DYK
                                           : (u0 - uE) * DYK * dz + (v0 - vN) * DXK * dz - wT * DXK * DYK;
            row(5, k) = DIV / DT;
        }
        if (lane == 0) {
            float P = 0.0f;
            for (int k = top; k > KK; --k) {
                const float T = 1.0f / (t.app[k] - t.atp[k] * P);
                P = ((k > KK + 1) ? t.abp1[k] : t.abp0[k]) * T;
                row(0, k) = T;
                row(1, k) = P;
            }
        }
    }

    __device__ void post(int, int, int) {
        const int lane = threadIdx.x & 31;
        const float DXK = a.dxk, DYK = a.dyk;
        const long long E = a.nj2, N = 1;
        for (int k = KK + 1 + lane; k <= top; k += 32) {
            const float dz = t.dzk[k];
            const float im = __ldcg(a.dpm + x.at(-E, k)), ip = __ldcg(a.dpm + x.at(E, k));
            const float jm = __ldcg(a.dpm + x.at(-N, k)), jp = __ldcg(a.dpm + x.at(N, k));
            row(3, k) = row(5, k) + (im + ip) / DXK * DYK * dz + (jm - jp) / DYK * DXK * dz;
        }
        __syncwarp();
        if (lane == 0) {
            float Q = 0.0f;
            for (int k = top; k > KK; --k) {
                Q = (t.atp[k] * Q + row(3, k)) * row(0, k);
                row(2, k) = Q;
            }
            float prev = 0.0f;                                     // DPM[KKART] = 0
            for (int k = KK + 1; k <= top; ++k) {
                prev = row(1, k) * prev + row(2, k);
                row(4, k) = prev;
            }
        }
        __syncwarp();
        for (int k = 1 + lane; k <= top; k += 32) __stcg(a.dpm + x.at(0, k), (k > KK) ? row(4, k) : 0.0f);
    }

    __device__ void finish() {}
};

__global__ void __launch_bounds__(GS_WARPS * 32) k_diag_pressure(KArgs a, SweepGeom g, DiagTabs t) {
    extern __shared__ float dsm[];
    DiagJob job{a, dsm + (size_t)(threadIdx.x >> 5) * 6 * a.ks, 0, t};
    gs_tasks_split<PH_DIAG, false>(a, g, job);
}

// ---------------------------- batched family -----------------------------------------------
// One block per task = (group of 32 situations, column).  The block's warps split the levels for
// the coefficient assembly (lane = situation, contiguous 128-byte loads in the interleaved layout)
// and write rows [k][32] to shared memory; warp 0 then runs the 32 situations' Thomas
// recurrences and back-substitutions side by side.

// L2 prefetch of one contiguous run (the interleaved layout keeps a (field, column) block of a
// group contiguous over levels); 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void l2_prefetch(const float *p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Operand blocks of a batched task, prefetched into L2 while the block still works on the task
// before it: for each field the columns (offsets in columns) the phase's level function reads,
// levels KSTART-1..VerticalIndex+1 (pressure: KKART..VerticalIndex+1).
template <int PHASE>
__device__ void prefetch_task(const KArgs &a, const SweepGeom &g, unsigned t, unsigned units, int IS, int JS) {
    int grp, i1, j1;
    decode_task(t, g, units, grp, i1, j1);
    grp += a.group_lo;
    const int i = (IS == 1) ? i1 : a.nii - i1 + 1;
    const int j = (JS == 1) ? j1 : a.njj - j1 + 1;
    const int col = i * a.nj2 + j;
    if (!(a.cflags[col] & F_ADV)) return;
    const ColMeta m = a.meta[col];
    const int klo = (PHASE == PH_PRESSURE) ? (int)m.kkart : max(0, (int)m.kstart - 1);
    const int khi = m.vi + 1;
    const unsigned bytes = (unsigned)(khi - klo + 1) * 32u * sizeof(float);
    const long long W = -(long long)a.nj2, E = a.nj2, S = -1, N = 1;
    auto pf = [&](const float *F, long long dc) {
        l2_prefetch(F + (((size_t)grp * a.ncols + (size_t)((long long)col + dc)) * a.ks + klo) * 32, bytes);
    };
    if (PHASE == PH_U) {
        pf(a.uk, 0); pf(a.uk, W); pf(a.uk, S); pf(a.uk, E); pf(a.uk, N); pf(a.vk, 0);
        pf(a.uks, 0); pf(a.uks, W); pf(a.wks, 0); pf(a.wks, W); pf(a.wk, E); pf(a.dpmnew, 0); pf(a.dpmnew, W);
        pf(a.vks, 0); pf(a.vks, W); pf(a.vks, W + S); pf(a.vks, S); pf(a.vks, W + N); pf(a.vks, N);
        pf(a.vks, E + N); pf(a.vks, E + S);
    } else if (PHASE == PH_V) {
        pf(a.vk, 0); pf(a.vk, W); pf(a.vk, S); pf(a.vk, E); pf(a.vk, N); pf(a.uk, 0);
        pf(a.vks, 0); pf(a.vks, W); pf(a.vks, S); pf(a.wks, 0); pf(a.wks, S); pf(a.wk, N); pf(a.dpmnew, 0);
        pf(a.dpmnew, S); pf(a.uks, 0); pf(a.uks, E); pf(a.uks, S); pf(a.uks, E + S); pf(a.uks, W);
        pf(a.uks, W + S); pf(a.uks, E + N); pf(a.uks, W + N);
    } else if (PHASE == PH_W) {
        pf(a.wk, 0); pf(a.wk, W); pf(a.wk, S); pf(a.wk, E); pf(a.wk, N); pf(a.uk, 0); pf(a.vk, 0);
        pf(a.uks, 0); pf(a.uks, W); pf(a.uks, E); pf(a.vks, 0); pf(a.vks, S); pf(a.vks, N); pf(a.wks, 0);
        pf(a.dpmnew, 0);
    } else if (PHASE == PH_PRESSURE) {
        pf(a.uk, 0); pf(a.uk, E); pf(a.vk, 0); pf(a.vk, N); pf(a.wk, 0); pf(a.dpmnew, 0);
        pf(a.dpm, -(long long)IS * a.nj2); pf(a.dpm, -(long long)JS);
    }
}

// Block-wide variant of gs_tasks: thread 0 claims and waits, the block works, thread 0 publishes.
// While warp 0 runs the serial recurrences, the body calls `ahead` from one idle thread, which
// prefetches into L2 the operands of the task one round of blocks further in claim order (task
// t + gridDim.x): some block claims it about one task duration later.
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
            if (threadIdx.x == 0)
                s_ok = wait_stamps((i1 > g.ia) ? fl + (i - IS) * a.nj2 + j : nullptr,
                                   (j1 > g.ja) ? fl + i * a.nj2 + (j - JS) : nullptr, stamp, a.err, a.wait_limit_ns);
            __syncthreads();
            auto ahead = [&]() {
                const unsigned pt = t + gridDim.x;
                if (pt < total) prefetch_task<PHASE>(a, g, pt, units, IS, JS);
            };
            if (s_ok) body(grp, i, j, IS, JS, i1 == g.ia, ahead);
            __syncthreads();
            if (threadIdx.x == 0) st_release(fl + i * a.nj2 + j, stamp);
        }
    }
}

// Rows [row][k][32] of one lane (= situation) in dynamic shared memory; the model-0 W rows P/Q
// in double follow the float rows.
struct BLane {
    float *base;
    double *dbase;
    int ks, lane;
    __device__ __forceinline__ float &row(int r, int k) { return base[((size_t)r * ks + k) * 32 + lane]; }
    __device__ __forceinline__ float &a(int k) { return row(0, k); }
    __device__ __forceinline__ float &b(int k) { return row(1, k); }
    __device__ __forceinline__ float &c(int k) { return row(2, k); }
    __device__ __forceinline__ float &d(int k) { return row(3, k); }
    __device__ __forceinline__ float &p(int k) { return row(4, k); }
    __device__ __forceinline__ double &pd(int k) { return dbase[((size_t)0 * ks + k) * 32 + lane]; }
    __device__ __forceinline__ double &qd(int k) { return dbase[((size_t)1 * ks + k) * 32 + lane]; }
    __device__ __forceinline__ float &b1(int k) { return row(1, k); }
    __device__ __forceinline__ float &c1(int k) { return row(2, k); }
    __device__ __forceinline__ float &d1(int k) { return row(3, k); }
    __device__ __forceinline__ float &k1(int k) { return row(4, k); }
    __device__ __forceinline__ float &b2(int k) { return row(5, k); }
    __device__ __forceinline__ float &c2(int k) { return row(6, k); }
    __device__ __forceinline__ float &d2(int k) { return row(7, k); }
    __device__ __forceinline__ float &e1(int k) { return row(8, k); }
};

__device__ __forceinline__ BLane blane(float *smem, int ks, int slot = -1) {
    BLane R;
    R.base = smem;
    R.dbase = reinterpret_cast<double *>(smem + (size_t)9 * ks * 32);
    R.ks = ks;
    R.lane = slot >= 0 ? slot : (threadIdx.x & 31);
    return R;
}

// Lanes of a batched task in its level loops.  A group that holds at most 16 situations (the
// last group of a batch such as 144 = 4 x 32 + 16) runs them two levels per warp instruction:
// lanes 16-31 take the odd levels of the situations of lanes 0-15.  slot = the situation's lane
// in the group, k = k0 + ofs, k0 + ofs + step, ...  The serial recurrences keep lane = slot.
struct BLoop {
    int slot, ofs, step;
    bool half;
};

template <int NW>
__device__ __forceinline__ BLoop bloop(const KArgs &a, int grp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    BLoop L;
    L.half = a.nb - grp * 32 <= 16;
    L.slot = L.half ? (lane & 15) : lane;
    L.ofs = L.half ? 2 * warp + (lane >> 4) : warp;
    L.step = L.half ? 2 * NW : NW;
    return L;
}

template <int MODEL, int COMP, int NW, int SW, class Ahead>
__device__ void batch_mom_column(const KArgs &a, int grp, int i, int j, float *smem, Ahead &&ahead) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const ColCtx c = make_col(a, i, j);
    if (!(c.fl & F_ADV)) return;
    const BLoop L = bloop<NW>(a, grp);
    const int s = grp * 32 + L.slot;
    const bool act = (s < a.nb) && a.sit[s].active;
    BLane R = blane(smem, a.ks, L.slot);
    const Acc<true> x = make_acc<true>(a, act ? s : grp * 32, c.col);
    if (act) {
        const SitCtx sc = make_sit(a, s);
        // one level per step: within the register budget of four resident blocks a second level's
        // operands did not overlap the first's (each level cost the same either way)
        for (int k = c.K0 + L.ofs; k <= c.VI; k += L.step) {
            const Coef q = mom_level<MODEL, COMP, true, SW>(a, x, c, sc, k);
            R.a(k) = q.A; R.b(k) = q.B; R.c(k) = q.C; R.d(k) = q.D; R.p(k) = q.phi;
        }
    }
    __syncthreads();
    if (threadIdx.x == 32) ahead();
    float *F = comp_field<COMP>(a);
    const int kkm = back_limit<COMP>(c);
    if (warp == 0) {     // the recurrences: lane = situation slot
        const int s0 = grp * 32 + lane;
        if (!L.half ? act : (s0 < a.nb && a.sit[s0].active)) {
            BLane R0 = blane(smem, a.ks);
            const Acc<true> x0 = L.half ? make_acc<true>(a, s0, c.col) : x;
            mom_sweep<MODEL, COMP>(R0, c.K0, c.KK, c.VI, kkm, a.relax, __ldcg(F + x0.at(0, c.VI + 1)));
        }
    }
    __syncthreads();
    if (!act) return;
    for (int k = max(c.K0, kkm + 1) + L.ofs; k <= c.VI; k += L.step) __stcg(F + x.at(0, k), R.p(k));
}

template <int NW, class Ahead>
__device__ void batch_tke_column(const KArgs &a, int grp, int i, int j, float *smem, Ahead &&ahead) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = grp * 32 + lane;
    const ColCtx c = make_col(a, i, j);
    if (!(c.fl & F_ADV)) return;
    const bool act = (s < a.nb) && a.sit[s].active;
    BLane R = blane(smem, a.ks);
    const Acc<true> x = make_acc<true>(a, act ? s : grp * 32, c.col);
    if (act) {
        const SitCtx sc = make_sit(a, s);
        for (int k = c.K0 + warp; k <= c.VI; k += NW) {
            const CoefKE q = tke_level<true>(a, x, c, sc, k);
            R.a(k) = q.A; R.b1(k) = q.B1; R.c1(k) = q.C1; R.d1(k) = q.D1; R.k1(k) = q.k1;
            R.b2(k) = q.B2; R.c2(k) = q.C2; R.d2(k) = q.D2; R.e1(k) = q.e1;
        }
    }
    __syncthreads();
    if (threadIdx.x == 32) ahead();
    if (warp != 0 || !act) return;
    const ColKE ke = a.colke[c.col];
    const float *vf[3] = {a.uk, a.vk, a.wk};
    tke_sweep(R, a, c, ke, __ldcg(a.turb + x.at(0, c.VI + 1)), __ldcg(a.tdiss + x.at(0, c.VI + 1)),
              [&](int f, long long dc, int k) { return vf[f][x.at(dc, k)]; });
    for (int k = c.K0; k <= c.VI; ++k)
        if (c.KK < k) {
            __stcg(a.turb + x.at(0, k), R.k1(k));
            __stcg(a.tdiss + x.at(0, k), R.e1(k));
        }
}

// Row carry of the batched family: [group][j][2][KS][32].
template <int NW, class Ahead>
__device__ void batch_pressure_column(const KArgs &a, int grp, int i, int j, int IS, int JS, bool first,
                                      float *smem, unsigned &nmax_acc, Ahead &&ahead) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = grp * 32 + lane;
    const int ks = a.ks;
    float *rc = a.rowcarry + (((size_t)grp * a.nj2 + j) * 2 * ks) * 32 + lane;
    if (first && warp == 0)
        for (int k = 0; k < 2 * ks; ++k) __stcg(rc + (size_t)k * 32, 0.0f);
    const ColCtx c = make_col(a, i, j);
    if (!(c.fl & F_ADV)) return;
    const bool act = (s < a.nb) && a.sit[s].active;
    BLane R = blane(smem, ks);
    const Acc<true> x = make_acc<true>(a, act ? s : grp * 32, c.col);
    const SitCtx sc = make_sit(a, act ? s : grp * 32);
    // Row a holds DPMNEW of the level, loaded here for the update after the recurrences (only
    // this task writes DPMNEW of its column, and no pressure task reads it).
    if (act) {
#pragma unroll 2
        for (int k = c.KK + 1 + warp; k <= c.VI; k += NW) {
            R.d(k) = pressure_dim<true>(a, x, c, sc, k, IS, JS);
            R.a(k) = a.dpmnew[x.at(0, k)];
        }
    }
    float P = 0.0f, Q = 0.0f;
    if (warp == 0 && act) {      // the row carry of the predecessor (published before our wait)
        P = __ldcg(rc + (size_t)(c.VI + 1) * 32);
        Q = __ldcg(rc + (size_t)(ks + c.VI + 1) * 32);
    }
    __syncthreads();
    if (threadIdx.x == 32) ahead();
    if (warp == 0 && act) {
        // eight levels per step: their table and row loads are issued together, the chain is serial
        constexpr int CH = 8;
        int k = c.VI;
        for (; k - (CH - 1) > c.KK; k -= CH) {
            float ap[CH], at[CH], ab[CH], d[CH];
#pragma unroll
            for (int q = 0; q < CH; ++q) {
                ap[q] = a.app[k - q]; at[q] = a.atp[k - q]; ab[q] = a.abp[k - q]; d[q] = R.d(k - q);
            }
#pragma unroll
            for (int q = 0; q < CH; ++q) {
                const float T = 1.0f / (ap[q] - at[q] * P);
                P = ab[q] * T;
                Q = (at[q] * Q + d[q]) * T;
                R.b(k - q) = P;
                R.c(k - q) = Q;
            }
        }
        for (; k > c.KK; --k) {
            const float T = 1.0f / (a.app[k] - a.atp[k] * P);
            P = a.abp[k] * T;
            Q = (a.atp[k] * Q + R.d(k)) * T;
            R.b(k) = P;
            R.c(k) = Q;
        }
        float prev = 0.0f;                                         // DPM[KKART] is always 0
        for (int k = c.KK + 1; k <= c.VI; ++k) {
            prev = R.b(k) * prev + R.c(k);
            R.p(k) = prev;
        }
    }
    __syncthreads();
    if (!act) return;
    const int klo = max(c.KK, a.vi_min);
    unsigned nmax = 0;
    for (int k = c.KK + 1 + warp; k <= c.VI; k += NW) {
        const float temp = R.p(k);
        nmax = max(nmax, residual_key(temp, sc));
        __stcg(a.dpm + x.at(0, k), temp);
        a.dpmnew[x.at(0, k)] = R.a(k) + a.relaxp * temp;
        if (k > klo) {
            __stcg(rc + (size_t)k * 32, R.b(k));
            __stcg(rc + (size_t)(ks + k) * 32, R.c(k));
        }
    }
    nmax_acc = max(nmax_acc, nmax);
}

template <int NW, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB) k_pressure_b(KArgs a, SweepGeom g) {
    extern __shared__ float smem[];
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
    gs_tasks_block<PH_PRESSURE, false>(a, g, [&](int grp, int i, int j, int IS, int JS, bool first, auto &&ahead) {
        if (grp != cur) { flush(); cur = grp; }
        batch_pressure_column<NW>(a, grp, i, j, IS, JS, first, smem, nmax, ahead);
    });
    flush();
}

// SW: parity width of model 1 fixed at compile time (8 or 16; 0 for the other models).
template <int MODEL, int COMP, int NW, int MINB, int SW>
__global__ void __launch_bounds__(NW * 32, MINB) k_mom_b(KArgs a, SweepGeom g) {
    extern __shared__ float smem[];
    constexpr int PH = COMP == COMP_U ? PH_U : (COMP == COMP_V ? PH_V : PH_W);
    constexpr bool REV = (MODEL == 1 && COMP == COMP_V);
    gs_tasks_block<PH, REV>(a, g, [&](int grp, int i, int j, int, int, bool, auto &&ahead) {
        batch_mom_column<MODEL, COMP, NW, SW>(a, grp, i, j, smem, ahead);
    });
}

template <int NW, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB) k_tke_b(KArgs a, SweepGeom g) {
    extern __shared__ float smem[];
    gs_tasks_block<PH_TKE, false>(a, g, [&](int grp, int i, int j, int, int, bool, auto &&ahead) {
        batch_tke_column<NW>(a, grp, i, j, smem, ahead);
    });
}

using KFn = void (*)(KArgs, SweepGeom);

// Launch variants of the batched family: (warps per block, minimum resident blocks per SM).
struct BVariant {
    int nw, minb;
    KFn pressure;
    KFn mom[3][3];   // [model][comp]; model 1 at parity width 8
    KFn mom16[3];    // model 1 at parity width 16, [comp]
    KFn tke;
};

#define GRAL_BV(NW, MB)                                                                              \
    BVariant{NW, MB, k_pressure_b<NW, MB>,                                                                 \
             {{k_mom_b<0, COMP_U, NW, MB, 0>, k_mom_b<0, COMP_V, NW, MB, 0>, k_mom_b<0, COMP_W, NW, MB, 0>},  \
              {k_mom_b<1, COMP_U, NW, MB, 8>, k_mom_b<1, COMP_V, NW, MB, 8>, k_mom_b<1, COMP_W, NW, MB, 8>},  \
              {k_mom_b<2, COMP_U, NW, MB, 0>, k_mom_b<2, COMP_V, NW, MB, 0>, k_mom_b<2, COMP_W, NW, MB, 0>}}, \
             {k_mom_b<1, COMP_U, NW, MB, 16>, k_mom_b<1, COMP_V, NW, MB, 16>, k_mom_b<1, COMP_W, NW, MB, 16>}, \
             k_tke_b<NW, MB>}

const BVariant kVariants[] = {GRAL_BV(8, 2), GRAL_BV(4, 4), GRAL_BV(4, 6), GRAL_BV(6, 4),
                              GRAL_BV(5, 5), GRAL_BV(6, 5), GRAL_BV(5, 6)};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

// Strip variants of the slab family's model-1 sweeps: (rows per strip, warps per row).
struct SVariant {
    int sr, smw;
    KFn pressure;
    KFn mom[3];   // [comp]
};

#define GRAL_SV(SR, SMW)                                                                           \
    SVariant{SR, SMW, k_pressure_strip<SR, SMW>,                                                   \
             {k_mom1_strip<COMP_U, SR, SMW>, k_mom1_strip<COMP_V, SR, SMW>, k_mom1_strip<COMP_W, SR, SMW>}}

const SVariant kStrips[] = {GRAL_SV(4, 4), GRAL_SV(2, 8), GRAL_SV(3, 5), GRAL_SV(2, 6)};
constexpr int kNumStrips = sizeof(kStrips) / sizeof(kStrips[0]);

KFn strip_kernel(int v, int kind) {
    const SVariant &S = kStrips[v];
    switch (kind) {
        case PH_PRESSURE: return S.pressure;
        case PH_U: return S.mom[0];
        case PH_V: return S.mom[1];
        default: return S.mom[2];
    }
}

const KFn kPlainMom[3][3] = {{k_mom<0, COMP_U>, k_mom<0, COMP_V>, k_mom<0, COMP_W>},
                             {k_mom1s<COMP_U>, k_mom1s<COMP_V>, k_mom1s<COMP_W>},
                             {k_mom<2, COMP_U>, k_mom<2, COMP_V>, k_mom<2, COMP_W>}};

// Dynamic shared memory of a batched kernel: 5 float rows (momentum, pressure), 9 float rows
// (TKE), 9 float rows + 2 double rows (model-0 W, whose P/Q are double).
size_t bsmem(int kind, int model, int ks) {
    const size_t row = (size_t)ks * 32 * sizeof(float);
    if (kind == PH_TKE) return 9 * row;
    if (kind == PH_W && model == 0) return 9 * row + 4 * row;
    return 5 * row;
}

// simd: the loaded parity width (16 selects the model-1 kernels compiled for Vector512).
KFn batch_kernel(const BVariant &V, int kind, int model, int simd) {
    const bool w16 = (model == 1 && simd == 16);
    switch (kind) {
        case PH_PRESSURE: return V.pressure;
        case PH_U: return w16 ? V.mom16[0] : V.mom[model][0];
        case PH_V: return w16 ? V.mom16[1] : V.mom[model][1];
        case PH_W: return w16 ? V.mom16[2] : V.mom[model][2];
        default: return V.tke;
    }
}

KFn plain_kernel(int kind, int model) {
    switch (kind) {
        case PH_PRESSURE: return k_pressure_s;
        case PH_U: return kPlainMom[model][0];
        case PH_V: return kPlainMom[model][1];
        case PH_W: return kPlainMom[model][2];
        default: return k_tke;
    }
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

}  // namespace

int gs_num_variants() { return kNumVariants; }

int gs_block_threads(bool il, int variant) { return il ? kVariants[variant].nw * 32 : GS_WARPS * 32; }

cudaError_t gs_prepare(bool il, int ks, int model) {
    if (!il) return cudaSuccess;
    const int kinds[5] = {PH_PRESSURE, PH_U, PH_V, PH_W, PH_TKE};
    for (int v = 0; v < kNumVariants; ++v)
        for (int q = 0; q < 5; ++q) {
            const int bytes = (int)bsmem(kinds[q], model, ks);
            for (int simd : {8, 16}) {
                cudaError_t e = cudaFuncSetAttribute(batch_kernel(kVariants[v], kinds[q], model, simd),
                                                     cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
                if (e != cudaSuccess) return e;
            }
        }
    return cudaSuccess;
}

cudaError_t gs_occupancy(bool il, int kind, int model, int simd, int ks, int variant, int *blocks_per_sm) {
    const int th = gs_block_threads(il, variant);
    if (!il) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, plain_kernel(kind, model), th, 0);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        blocks_per_sm, batch_kernel(kVariants[variant], kind, model, simd), th, bsmem(kind, model, ks));
}

void launch_gs(int kind, const KArgs &a, const SweepGeom &g, int grid, cudaStream_t st) {
    if (a.il) {
        const BVariant &V = kVariants[a.variant];
        KFn f = batch_kernel(V, kind, a.model, a.simd);
        const size_t sm = bsmem(kind, a.model, a.ks);
        for_group_sets(a, [&](const KArgs &b) { f<<<grid, V.nw * 32, sm, st>>>(b, g); });
    } else {
        plain_kernel(kind, a.model)<<<grid, GS_WARPS * 32, 0, st>>>(a, g);
    }
}

int strip_num_variants() { return kNumStrips; }

int strip_rows(int variant) { return kStrips[variant].sr; }

int strip_block_threads(int variant) { return kStrips[variant].sr * kStrips[variant].smw * 32; }

cudaError_t strip_occupancy(int kind, int variant, int *blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, strip_kernel(variant, kind),
                                                         strip_block_threads(variant), 0);
}

void launch_strip(int kind, const KArgs &a, const SweepGeom &g, int variant, int grid, cudaStream_t st) {
    strip_kernel(variant, kind)<<<grid, strip_block_threads(variant), 0, st>>>(a, g);
}

cudaError_t fused_strip_occupancy(int *blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_fused_strip, 16 * 32, 0);
}

int fused_strip_claims(const SweepGeom &gp) { return 2 * ((gp.ni + FSR - 1) / FSR) + 1; }

void launch_fused_strip(const KArgs &a, const FusedGeom &fg, int grid, cudaStream_t st) {
    k_fused_strip<<<grid, 16 * 32, 0, st>>>(a, fg);
}

size_t diag_smem(int ks) { return (size_t)GS_WARPS * 6 * ks * sizeof(float); }

cudaError_t diag_prepare(int ks) {
    return cudaFuncSetAttribute(k_diag_pressure, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)diag_smem(ks));
}

cudaError_t diag_occupancy(int ks, int *blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_diag_pressure, GS_WARPS * 32, diag_smem(ks));
}

void launch_diag_pressure(const KArgs &a, const SweepGeom &g, const DiagTabs &t, int grid, cudaStream_t st) {
    k_diag_pressure<<<grid, GS_WARPS * 32, diag_smem(a.ks), st>>>(a, g, t);
}

cudaError_t fused_occupancy(int *blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_fused_pvau, GS_WARPS * 32, 0);
}

void launch_fused_pvau(const KArgs &a, const FusedGeom &fg, int grid, cudaStream_t st) {
    k_fused_pvau<<<grid, GS_WARPS * 32, 0, st>>>(a, fg);
}

}  // namespace gral
