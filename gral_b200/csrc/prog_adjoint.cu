// prog_adjoint.cu -- discrete adjoint (vector-Jacobian product) of the unrolled SIMPLE iterations
// of one situation: gral_prog_vjp_forward and gral_prog_vjp.
//
// Differentiated configuration: turbulence model 1, Vector<float> parity width 8, no Frund
// rounding (its derivative is zero almost everywhere), a fixed number of iterations.  The set-up's
// scalars (topwind, DTIME, AP0, UG, VG, the wall-law help terms, Frund) are constants of the map.
// Inputs of the map: the initial U, V, W fields and the vegetation density VEG; output: the final
// U, V, W fields.
//
// The forward run keeps the state (UK, VK, WK, UKS, VKS, WKS, DPMNEW and the situation's loop
// state) every `checkpoint_every` iterations.  The reverse pass walks the checkpoint segments from
// the last: it restores the segment's checkpoint, recomputes its iterations with the solver's own
// kernels while keeping, per iteration, the state after the staggered averages ("mid") and after
// the W sweep ("end") and the branch taken by every lateral boundary copy, then reverses the
// segment's iterations one by one.  Reversing one iteration (PrognosticFlowfield.cs:584-1137):
//
//   W, V, U momentum sweeps   reverse Gauss-Seidel wavefronts: a column receives the cotangents
//                             of its new values from its two sweep successors (stamped 8-byte
//                             words), reverses the relaxed back-substitution and the Thomas
//                             recurrence (U-prognostic-microscale_1.cs:485-524) on lane 0, sends
//                             its two predecessors the cotangents of their new values the same
//                             way, and then adds the per-level vector-Jacobian products of the
//                             coefficient assembly (adj_level.cuh) to every other input;
//   staggered averages        gathers (PrognosticFlowfield.cs:958-1039);
//   velocity correction       a gather into DPM (PrognosticFlowfield.cs:904-949);
//   pressure correction       a reverse wavefront of the transposed tridiagonal solves
//                             (PrognosticFlowfield.cs:804-901), the row carry of Q included;
//   divergence                a gather (PrognosticFlowfield.cs:723-758);
//   boundary conditions       the copies reversed in reverse order (PrognosticFlowfield.cs:595-714).
//
// After the first iteration the set-up's staggered averages, border copies and zeroing inside
// buildings (PrognosticFlowfield.cs:295-329, 410-432, 518-575) are reversed as well.  Cotangents
// are accumulated with float atomics, so their summation order varies from run to run at the
// level of float rounding.  Every wait is bounded like the forward's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include <cstdlib>

#include "adj_level.cuh"
#include "prog_ctx.cuh"
#include "prog_level.cuh"

namespace gral {

namespace {

using namespace adj;

constexpr int AW = 4;               // warps per block of the reverse sweeps
constexpr int WL = 99;              // level marker of the wall-law inputs
enum : int { FU = 0, FV, FW, FUS, FVS, FWS, FDP, FVEG, NLAM_IN };
// cotangent fields: the eight input kinds above, then DPM, DIV and the pressure row-carry Q
enum : int { L_DPM = NLAM_IN, L_DIV, L_QC, NLAM };
constexpr int NKEEP = 10;           // per iteration: mid UK VK WK UKS VKS WKS DPMNEW, end UK VK WK
constexpr int NCKPT = 7;            // checkpoint: UK VK WK UKS VKS WKS DPMNEW

struct InDesc {
    int8_t f, di, dj, dk;
};

// Input tables of the level functions of adj_level.cuh: field, column offset (i, j), level offset.
// They are constexpr and read with compile-time indices (InTab<COMP>::at inside for_inputs), so the
// choice of field, the cell offset and the wall-law level of every input fold into the code.
template <int COMP> struct InTab;
template <> struct InTab<0> {
    static constexpr int N = U_COUNT;
    static constexpr __host__ __device__ InDesc at(int q) {
        constexpr InDesc t[U_COUNT] = {
            {FU, 0, 0, 0}, {FU, 0, 0, 1}, {FU, 0, 0, -1}, {FV, 0, 0, 1}, {FV, 0, 0, -1},
            {FUS, 0, 0, 0}, {FVS, 0, 0, 0}, {FWS, 0, 0, 0},
            {FUS, -1, 0, 0}, {FVS, -1, 0, 0}, {FVS, -1, -1, 0}, {FVS, 0, -1, 0}, {FVS, -1, 1, 0}, {FVS, 0, 1, 0},
            {FWS, -1, 0, 0}, {FWS, -1, 0, 1}, {FWS, 0, 0, 1}, {FWS, 0, 0, -1}, {FWS, -1, 0, -1},
            {FDP, -1, 0, 0}, {FDP, 0, 0, 0},
            {FVS, 1, 1, 0}, {FVS, 1, -1, 0}, {FW, 1, 0, 0}, {FW, 1, 0, -1},
            {FVEG, 0, 0, -1},
            {FUS, -1, 0, WL}, {FUS, 0, 0, WL}, {FVS, -1, 0, WL}, {FVS, 0, 0, WL},
            {FU, -1, 0, 0}, {FU, 0, -1, 0}, {FU, 1, 0, 0}, {FU, 0, 1, 0}};
        return t[q];
    }
};
template <> struct InTab<1> {
    static constexpr int N = V_COUNT;
    static constexpr __host__ __device__ InDesc at(int q) {
        constexpr InDesc t[V_COUNT] = {
            {FV, 0, 0, 0}, {FU, 0, 0, 1}, {FU, 0, 0, -1}, {FV, 0, 0, 1}, {FV, 0, 0, -1},
            {FUS, 0, 0, 0}, {FVS, 0, 0, 0}, {FWS, 0, 0, 0},
            {FUS, 1, 0, 0}, {FUS, 0, -1, 0}, {FUS, 1, -1, 0}, {FUS, -1, 0, 0}, {FVS, -1, 0, 0}, {FUS, -1, -1, 0},
            {FVS, 0, -1, 0}, {FWS, 0, -1, 0}, {FWS, 0, 0, -1}, {FWS, 0, -1, 1}, {FWS, 0, 0, 1}, {FWS, 0, -1, -1},
            {FDP, 0, -1, 0}, {FDP, 0, 0, 0},
            {FUS, 1, 1, 0}, {FUS, -1, 1, 0}, {FW, 0, 1, 0}, {FW, 0, 1, -1},
            {FVEG, 0, 0, -1},
            {FUS, -1, 0, WL}, {FUS, 0, 0, WL}, {FVS, -1, 0, WL}, {FVS, 0, 0, WL},
            {FV, -1, 0, 0}, {FV, 0, -1, 0}, {FV, 1, 0, 0}, {FV, 0, 1, 0}};
        return t[q];
    }
};
template <> struct InTab<2> {
    static constexpr int N = W_COUNT;
    static constexpr __host__ __device__ InDesc at(int q) {
        constexpr InDesc t[W_COUNT] = {
            {FW, 0, 0, 0}, {FU, 0, 0, 1}, {FU, 0, 0, -1}, {FV, 0, 0, 1}, {FV, 0, 0, -1},
            {FUS, 0, 0, 0}, {FVS, 0, 0, 0}, {FWS, 0, 0, 0}, {FUS, 0, 0, -1}, {FVS, 0, 0, -1},
            {FUS, -1, 0, 0}, {FUS, -1, 0, -1}, {FVS, 0, -1, 0}, {FVS, 0, -1, -1}, {FUS, 1, 0, 0}, {FUS, 1, 0, -1},
            {FVS, 0, 1, 0}, {FVS, 0, 1, -1},
            {FWS, 0, 0, -1}, {FDP, 0, 0, -1}, {FDP, 0, 0, 0},
            {FUS, 0, 0, 1}, {FUS, -1, 0, 1}, {FVS, 0, 0, 1}, {FVS, 0, -1, 1},
            {FW, 0, 0, 1}, {FW, 0, 0, -1},
            {FVEG, 0, 0, -1},
            {FW, -1, 0, 0}, {FW, 0, -1, 0}, {FW, 1, 0, 0}, {FW, 0, 1, 0}};
        return t[q];
    }
};

// f(std::integral_constant<int, q>) for q = 0 .. N-1, unrolled at compile time
template <class F, int... Q>
__device__ __forceinline__ void for_inputs_(F &&f, std::integer_sequence<int, Q...>) {
    (f(std::integral_constant<int, Q>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void for_inputs(F &&f) {
    for_inputs_(f, std::make_integer_sequence<int, N>{});
}

// Everything the adjoint kernels read besides the solver's KArgs (all device pointers, slab
// layout [ncols][KS] of the one situation).
struct AdjArgs {
    const float *mid[7];     // UK VK WK UKS VKS WKS DPMNEW after the averages of the iteration
    const float *end[3];     // UK VK WK after the W sweep
    float *lam[NLAM];        // cotangents: FU..FVEG, then DPM, DIV, row-carry Q
    const float *ptab;       // [2][2][ncols][KS]: pressure P and TERMP per i-direction (IS = +1, -1)
    // per column and level, the cotangent sent by the sweep successor in i (slot 0) and in j
    // (slot 1), as 8-byte words (float bits, launch stamp): [2][ncols][KS]
    unsigned long long *slot;
    const int *rcr;          // per column: bit 0 (IS = +1) / bit 1 (IS = -1) set where a column reads its row carry
    unsigned int *ctr;       // task counter of the launch
    int stamp;               // stamp of the launch's words
    int it;                  // IterationLoops of the reversed iteration
    const uint8_t *bits;     // boundary-copy branches of the iteration: [we events + sn events][KS]
    int nwe;                 // W/E events (the S/N events follow)
};

__device__ __forceinline__ size_t cell(const KArgs &a, int col, int k) { return (size_t)col * a.ks + k; }

__device__ __forceinline__ void sweep_dir_of(int it, int &IS, int &JS) {
    const int m = it % 4;   // PrognosticFlowfield.cs:770-802
    if (m == 0) { IS = -1; JS = 1; }
    else if (m == 1) { IS = -1; JS = -1; }
    else if (m == 2) { IS = 1; JS = -1; }
    else { IS = 1; JS = 1; }
}

// The words of this launch sent to column col by its successors in i (s1) and in j (s2), summed per
// level k = lane + 32*r (v[r], zero above KS).  Bounded like every wait: 0 after the time limit
// (the error word set) or on another warp's error.
__device__ __forceinline__ int poll_words(const KArgs &a, const AdjArgs &d, int col, bool s1, bool s2, float v[2]) {
    const int lane = threadIdx.x & 31;
    const unsigned long long *w1 = d.slot + (size_t)col * a.ks;
    const unsigned long long *w2 = d.slot + ((size_t)a.ncols + col) * a.ks;
    const int stamp = d.stamp;
    bool need[2][2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        v[r] = 0.0f;
        need[r][0] = s1 && k < a.ks;
        need[r][1] = s2 && k < a.ks;
    }
    unsigned long long t0 = 0;
    for (unsigned n = 0;; ++n) {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (need[r][0]) {
                const unsigned long long x = ld_word(w1 + k);
                if ((int)(x >> 32) >= stamp) { v[r] += __uint_as_float((unsigned)x); need[r][0] = false; }
            }
            if (need[r][1]) {
                const unsigned long long x = ld_word(w2 + k);
                if ((int)(x >> 32) >= stamp) { v[r] += __uint_as_float((unsigned)x); need[r][1] = false; }
            }
        }
        const bool pending = need[0][0] || need[0][1] || need[1][0] || need[1][1];
        if (!__any_sync(0xffffffffu, pending)) break;
        if (n == 0) t0 = globaltimer_ns();
        if ((n & 15) == 15) {
            int bad = *(volatile int *)a.err != ERR_NONE;
            if (!bad && globaltimer_ns() - t0 > a.wait_limit_ns) {
                if (lane == 0) atomicCAS(a.err, ERR_NONE, ERR_TIMEOUT);
                bad = 1;
            }
            if (__any_sync(0xffffffffu, bad)) return 0;
        }
    }
    asm volatile("fence.acquire.gpu;" ::: "memory");
    return 1;
}

// task t -> (i1, j1): diagonal-major, then position (one situation)
__device__ __forceinline__ void decode(unsigned t, const SweepGeom &g, int &i1, int &j1) {
    int lo = 0, hi = g.ndiag;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if ((unsigned)g.diag_start[mid] <= t) lo = mid; else hi = mid;
    }
    const int d = lo;
    const int pos = (int)(t - (unsigned)g.diag_start[d]);
    const int ioff = max(0, d - (g.nj - 1)) + pos;
    i1 = g.ia + ioff;
    j1 = g.ja + d - ioff;
}

// The reverse wavefront task loop: tasks in reverse diagonal order; a column receives the
// cotangents its two sweep successors (i1+1, j1) and (i1, j1+1) send it as stamped words
// (job.receive), runs job.critical, which sends its two predecessors theirs the same way, then
// runs job.after.  A word carries its own value, so no flag, release or fence sits between a
// column's recurrence and its predecessors'.  Successors are claimed earlier, so no task waits on
// one that is not running or done.
template <class Job>
__device__ __forceinline__ void rev_tasks(const KArgs &a, const AdjArgs &d, const SweepGeom &g, int IS, int JS,
                                          Job &job) {
    const int lane = threadIdx.x & 31;
    const unsigned total = (unsigned)g.diag_start[g.ndiag];
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(d.ctr, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= total) break;
        if (*(volatile int *)a.err != ERR_NONE) break;
        int i1, j1;
        decode(total - 1 - t, g, i1, j1);
        const int i = (IS == 1) ? i1 : a.nii - i1 + 1;
        const int j = (JS == 1) ? j1 : a.njj - j1 + 1;
        job.pre(i, j, IS, JS);
        const bool s1 = i1 < g.ia + g.ni - 1, s2 = j1 < g.ja + g.nj - 1;   // successors in the sweep
        // the successors' cotangents arrive as stamped words: no flag, no fence on the chain
        const int ok = job.receive(s1, s2);
        __syncwarp();
        if (ok) job.critical(IS, JS, i1 > g.ia, j1 > g.ja);
        if (ok) job.after(IS, JS);
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------------------------
// momentum sweeps
// ------------------------------------------------------------------------------------------------
template <int COMP> struct CompTraits;
template <> struct CompTraits<0> {
    static constexpr int N = U_COUNT;
    template <class T> static __device__ void row(const LevelConst &c, const T *x, T *o) { u_row(c, x, o); }
    template <class T> static __device__ void vjp(const LevelConst &c, const T *x, const T *l, T *g) {
        u_row_vjp(c, x, l, g);
    }
};
template <> struct CompTraits<1> {
    static constexpr int N = V_COUNT;
    template <class T> static __device__ void row(const LevelConst &c, const T *x, T *o) { v_row(c, x, o); }
    template <class T> static __device__ void vjp(const LevelConst &c, const T *x, const T *l, T *g) {
        v_row_vjp(c, x, l, g);
    }
};
template <> struct CompTraits<2> {
    static constexpr int N = W_COUNT;
    template <class T> static __device__ void row(const LevelConst &c, const T *x, T *o) { w_row(c, x, o); }
    template <class T> static __device__ void vjp(const LevelConst &c, const T *x, const T *l, T *g) {
        w_row_vjp(c, x, l, g);
    }
};

// shared rows per warp: A B C D (then their cotangents), the forward T P Q, the new value above
// (`up` of the back-substitution), the coefficients of the two predecessors in D, the cotangent
// of the new value (then of the old value, LO), and per-level products of the reversed
// recurrence: -T*T, Q_{k-1}*T, P_{k-1} (zero where the level has no predecessor in the recurrence)
enum : int { R_A, R_B, R_C, R_D, R_T, R_P, R_Q, R_UP, R_C1, R_C2, R_LO, R_NT2, R_QPT, R_PP, NROW };

// The two reversed recurrences run on lane 0 over level records packed so that one shared-memory
// load brings a level's coefficients, prefetched four levels ahead; the records are offset by RPAD
// levels so that the prefetch past either end of the column stays inside the arrays.
constexpr int RPAD = 8;
struct __align__(16) MomShared {
    float4 bect[KMAX_LEVELS + 2 * RPAD];   // B, D + C*Q_{k-1}, C*T, T*T*C (the last two zero without predecessor)
    float2 lrp[KMAX_LEVELS + 2 * RPAD];    // cotangent L0 of the new value, relax*P
    float2 lpq[KMAX_LEVELS + 2 * RPAD];    // relax*UP*mu, relax*mu; then the cotangents of P and Q
    float rows[NROW][KMAX_LEVELS];
};

template <int COMP>
struct MomRev {
    const KArgs &a;
    const AdjArgs &d;
    MomShared &M;
    float (*S)[KMAX_LEVELS];
    ColCtx c;
    bool act;
    int kkm, kwl;
    float top_carry;

    __device__ LevelConst level_const(int k) const {
        LevelConst L;
        const float dz = a.dzk[k];
        L.dz = dz; L.dxdz = a.dxk * dz; L.dydz = a.dyk * dz;
        L.dxk = a.dxk; L.dyk = a.dyk; L.area = a.areaxy;
        L.ap0 = a.ap0[k]; L.vishmin = a.vishmin; L.cor = a.coriolis;
        L.geo = (COMP == 0) ? a.sit[0].ug : a.sit[0].vg;
        L.hok = a.hokart[k]; L.hokK = c.hokK; L.cov = c.cf.cov;
        L.help_t = c.cf.help_t; L.help_o = c.cf.help_o;
        L.k = k; L.KK = c.KK; L.kad = c.kad; L.wlo = c.wlo; L.whi = c.whi;
        L.fl = c.fl;
        return L;
    }

    // input q of the level at k: the swept field's predecessors hold their new values, U is final
    // in the V and W sweeps and V in the W sweep; every other input is the state after the averages
    template <int Q> __device__ __forceinline__ float input(int k, int IS, int JS) const {
        constexpr InDesc e = InTab<COMP>::at(Q);
        const int kk = (e.dk == WL) ? kwl : k + e.dk;
        const size_t at = (size_t)(c.col + e.di * a.nj2 + e.dj) * a.ks + kk;
        if constexpr (e.f == FVEG) {
            return a.veg ? __ldcg(a.veg + at) : 0.0f;
        } else if constexpr (e.f >= FUS) {
            return __ldcg(d.mid[e.f] + at);
        } else if constexpr (e.f == COMP) {
            const bool pred = (e.di != 0 && e.dj == 0 && e.di == -IS) || (e.di == 0 && e.dj != 0 && e.dj == -JS);
            return __ldcg((pred ? d.end[e.f] : d.mid[e.f]) + at);
        } else {
            return __ldcg((e.f < COMP ? d.end[e.f] : d.mid[e.f]) + at);
        }
    }

    __device__ __forceinline__ void load(int k, int IS, int JS, float *x) const {
        for_inputs<InTab<COMP>::N>([&](auto q) { x[q.value] = input<q.value>(k, IS, JS); });
    }

    // before the wait: the forward rows of the column from the kept states and its Thomas
    // recurrence (U-prognostic-microscale_1.cs:485-504)
    __device__ void pre(int i, int j, int IS, int JS) {
        const int lane = threadIdx.x & 31;
        c = make_col(a, i, j);
        act = (c.fl & F_ADV) != 0;
        kkm = (COMP == 0) ? c.kkm_u : (COMP == 1 ? c.kkm_v : -32768);
        kwl = ((c.fl & F_CUTKLT1) && (c.fl & F_Z0GE)) ? c.KK + 2 : c.KK + 1;
        top_carry = 0.0f;
        if (!act) return;
#pragma unroll 1
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (k < c.K0 || k > c.VI) continue;
            float x[CompTraits<COMP>::N];
            load(k, IS, JS, x);
            const LevelConst LC = level_const(k);
            float o[8];
            CompTraits<COMP>::row(LC, x, o);
            S[R_A][k] = o[0]; S[R_B][k] = o[1]; S[R_C][k] = o[2]; S[R_D][k] = o[3];
            // predecessor 1 is (i - IS, j): W (o[4]) or E (o[6]); predecessor 2 is (i, j - JS): S or N
            S[R_C1][k] = (IS == 1) ? o[4] : o[6];
            S[R_C2][k] = (JS == 1) ? o[5] : o[7];
            S[R_UP][k] = __ldcg(d.end[COMP] + cell(a, c.col, k + 1));
        }
        __syncwarp();
        if (lane == 0) {
            float P = 0.0f, Q = 0.0f;
            for (int k = c.K0; k <= c.VI; ++k) {
                const float A = S[R_A][k], B = S[R_B][k], C = S[R_C][k], D = S[R_D][k];
                const bool ch = k > c.KK + 1;
                const float T = ch ? 1.0f / (A - C * P) : 1.0f / A;
                Q = ch ? (D + C * Q) * T : D * T;
                P = B * T;
                S[R_T][k] = T; S[R_P][k] = P; S[R_Q][k] = Q;
            }
        }
        __syncwarp();
        // the products the reversed recurrence needs, off its critical path
        float *L = d.lam[COMP];
        for (int k = c.K0 + lane; k <= c.VI; k += 32) {
            const bool ch = k > c.KK + 1;
            const float B = S[R_B][k], C = S[R_C][k], D = S[R_D][k], T = S[R_T][k];
            const float Qp = ch ? S[R_Q][k - 1] : 0.0f;
            M.bect[RPAD + k] = make_float4(B, ch ? D + C * Qp : D, ch ? C * T : 0.0f, ch ? T * T * C : 0.0f);
            // an updated level's cotangent is handed over from its new to its old value: what the
            // later phases left is taken now, the successors' parts arrive as words
            float l0 = 0.0f;
            if (kkm < k) {
                const size_t e = cell(a, c.col, k);
                l0 = __ldcg(L + e);
                L[e] = 0.0f;
            }
            M.lrp[RPAD + k] = make_float2(l0, a.relax * S[R_P][k]);
            S[R_NT2][k] = -(T * T);
            S[R_QPT][k] = Qp * T;
            S[R_PP][k] = ch ? S[R_P][k - 1] : 0.0f;
        }
        // the cleared cells are seen cleared before any word this column sends, hence before the
        // predecessors add the cotangents of the old values to them
        __threadfence();
        __syncwarp();
    }

    // the successors' words of this launch for every level: added to L0 at the updated levels,
    // to the cotangent field everywhere else (levels outside the column's solve, inactive columns)
    __device__ int receive(bool s1, bool s2) {
        const int lane = threadIdx.x & 31;
        float v[2];
        if (!poll_words(a, d, c.col, s1, s2, v)) return 0;
        float *L = d.lam[COMP];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (k >= a.ks || v[r] == 0.0f) continue;
            if (act && k >= c.K0 && k <= c.VI && kkm < k) M.lrp[RPAD + k].x += v[r];
            else atomicAdd(L + cell(a, c.col, k), v[r]);
        }
        return 1;
    }

    // after the wait: the cotangents of the column's new values are complete (later phases and
    // both successors have added theirs); reverse the back-substitution and the recurrence and
    // send the predecessors their cotangents
    __device__ void critical(int IS, int JS, bool p1, bool p2) {
        const int lane = threadIdx.x & 31;
        if (!act) {
            send(IS, JS, p1, p2);
            return;
        }
        float2 *lrp = M.lrp + RPAD, *lpq = M.lpq + RPAD;
        const float4 *bect = M.bect + RPAD;
        __syncwarp();
        const int K0 = c.K0, VI = c.VI;
        const float relax = a.relax, r1 = 1.0f - relax;
        // relaxed back-substitution (:513-524) reversed, bottom up: phi'_k = phi_k +
        // relax*(P_k*up + Q_k - phi_k) with up = phi'_{k+1}, so the cotangent of the new value at k
        // is mu_k = L0_k + carry with carry = relax*P_{k-1}*mu_{k-1}; the levels up to kkm are not
        // updated, have L0 = 0 and carry nothing.  Lane 0 runs only the chain (one add, one multiply
        // per level) and keeps mu in the LO row.
        if (lane == 0) {
            float carry = 0.0f, topc = 0.0f;
            float2 x0 = lrp[K0], x1 = lrp[K0 + 1], x2 = lrp[K0 + 2], x3 = lrp[K0 + 3];
            for (int k = K0; k <= VI; k += 4) {
                const float2 y0 = lrp[k + 4], y1 = lrp[k + 5], y2 = lrp[k + 6], y3 = lrp[k + 7];
                float mu = x0.x + carry;
                carry = x0.y * mu;
                S[R_LO][k] = mu;
                if (k == VI) topc = carry;
                mu = x1.x + carry;
                carry = x1.y * mu;
                if (k + 1 <= VI) S[R_LO][k + 1] = mu;
                if (k + 1 == VI) topc = carry;
                mu = x2.x + carry;
                carry = x2.y * mu;
                if (k + 2 <= VI) S[R_LO][k + 2] = mu;
                if (k + 2 == VI) topc = carry;
                mu = x3.x + carry;
                carry = x3.y * mu;
                if (k + 3 <= VI) S[R_LO][k + 3] = mu;
                if (k + 3 == VI) topc = carry;
                x0 = y0; x1 = y1; x2 = y2; x3 = y3;
            }
            top_carry = topc;
        }
        __syncwarp();
        for (int k = K0 + lane; k <= VI; k += 32) {
            const float mu = S[R_LO][k];
            S[R_LO][k] = r1 * mu;
            lpq[k] = make_float2(relax * S[R_UP][k] * mu, relax * mu);
        }
        __syncwarp();
        // Thomas recurrence reversed, top down, on the products made before the wait (zero at
        // the levels without predecessor, which ends the carried cotangents there):
        //   lP_k = LP_k + TTC_{k+1}*lT_{k+1},  lQ_k = LQ_k + CT_{k+1}*lQ_{k+1},  lT_k = lP_k*B_k + lQ_k*E_k
        if (lane == 0) {
            float lPn = 0.0f, lQn = 0.0f;
            float2 q0 = lpq[VI], q1 = lpq[VI - 1], q2 = lpq[VI - 2], q3 = lpq[VI - 3];
            float4 e0 = bect[VI], e1 = bect[VI - 1], e2 = bect[VI - 2], e3 = bect[VI - 3];
            for (int k = VI; k >= K0; k -= 4) {
                const float2 p0 = lpq[k - 4], p1 = lpq[k - 5], p2 = lpq[k - 6], p3 = lpq[k - 7];
                const float4 f0 = bect[k - 4], f1 = bect[k - 5], f2 = bect[k - 6], f3 = bect[k - 7];
                float lP = q0.x + lPn, lQ = q0.y + lQn;
                float lT = fmaf(lP, e0.x, lQ * e0.y);
                lQn = lQ * e0.z;
                lPn = lT * e0.w;
                lpq[k] = make_float2(lP, lQ);
                lP = q1.x + lPn; lQ = q1.y + lQn;
                lT = fmaf(lP, e1.x, lQ * e1.y);
                lQn = lQ * e1.z;
                lPn = lT * e1.w;
                if (k - 1 >= K0) lpq[k - 1] = make_float2(lP, lQ);
                lP = q2.x + lPn; lQ = q2.y + lQn;
                lT = fmaf(lP, e2.x, lQ * e2.y);
                lQn = lQ * e2.z;
                lPn = lT * e2.w;
                if (k - 2 >= K0) lpq[k - 2] = make_float2(lP, lQ);
                lP = q3.x + lPn; lQ = q3.y + lQn;
                lT = fmaf(lP, e3.x, lQ * e3.y);
                lQn = lQ * e3.z;
                lPn = lT * e3.w;
                if (k - 3 >= K0) lpq[k - 3] = make_float2(lP, lQ);
                q0 = p0; q1 = p1; q2 = p2; q3 = p3;
                e0 = f0; e1 = f1; e2 = f2; e3 = f3;
            }
        }
        __syncwarp();
        // the cotangents of the row (A, B, C, D) on all lanes
        for (int k = K0 + lane; k <= VI; k += 32) {
            const float2 pq = lpq[k];
            const float4 e = bect[k];
            const float lP = pq.x, lQ = pq.y, T = S[R_T][k];
            const float lT = fmaf(lP, e.x, lQ * e.y);
            const float lden = lT * S[R_NT2][k];
            S[R_A][k] = lden;
            S[R_B][k] = lP * T;
            S[R_C][k] = lQ * S[R_QPT][k] - lden * S[R_PP][k];
            S[R_D][k] = lQ * T;
        }
        __syncwarp();
        send(IS, JS, p1, p2);
    }

    // the cotangents of the predecessors' new values (they run after this column), for every level
    // (zero outside the column's solve): as words to a predecessor inside the sweep, added to the
    // cotangent field of one outside it
    __device__ void send(int IS, int JS, bool p1, bool p2) {
        const int lane = threadIdx.x & 31;
        const int c1 = c.col - IS * a.nj2, c2 = c.col - JS;
        unsigned long long *w1 = d.slot + (size_t)c1 * a.ks;
        unsigned long long *w2 = d.slot + ((size_t)a.ncols + c2) * a.ks;
        float *L = d.lam[COMP];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (k >= a.ks) continue;
            const float lD = (act && k >= c.K0 && k <= c.VI) ? S[R_D][k] : 0.0f;
            const float g1 = lD != 0.0f ? lD * S[R_C1][k] : 0.0f, g2 = lD != 0.0f ? lD * S[R_C2][k] : 0.0f;
            if (p1) st_word(w1 + k, g1, d.stamp);
            else if (g1 != 0.0f) atomicAdd(L + cell(a, c1, k), g1);
            if (p2) st_word(w2 + k, g2, d.stamp);
            else if (g2 != 0.0f) atomicAdd(L + cell(a, c2, k), g2);
        }
    }

    __device__ void after(int IS, int JS) {
        if (!act) return;
        const int lane = threadIdx.x & 31;
        constexpr int N = CompTraits<COMP>::N;
        if (lane == 0 && top_carry != 0.0f) atomicAdd(d.lam[COMP] + cell(a, c.col, c.VI + 1), top_carry);
#pragma unroll 1
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (k < c.K0 || k > c.VI) continue;
            float x[N], g[N];
            load(k, IS, JS, x);
#pragma unroll
            for (int q = 0; q < N; ++q) g[q] = 0.0f;
            const float l4[4] = {S[R_A][k], S[R_B][k], S[R_C][k], S[R_D][k]};
            const LevelConst LC = level_const(k);
            CompTraits<COMP>::vjp(LC, x, l4, g);
            g[0] += S[R_LO][k];
            for_inputs<N>([&](auto q) {
                constexpr InDesc e = InTab<COMP>::at(q.value);
                const float v = g[q.value];
                if constexpr (e.f == COMP) {
                    // the predecessors' cotangents were sent as words
                    if ((e.di != 0 && e.dj == 0 && e.di == -IS) || (e.di == 0 && e.dj != 0 && e.dj == -JS)) return;
                }
                if constexpr (e.f == FVEG) {
                    if (!a.veg) return;
                }
                if (v == 0.0f) return;
                const int kk = (e.dk == WL) ? kwl : k + e.dk;
                atomicAdd(d.lam[e.f] + (size_t)(c.col + e.di * a.nj2 + e.dj) * a.ks + kk, v);
            });
        }
    }
};

template <int COMP>
__global__ void __launch_bounds__(AW * 32) k_adj_mom(KArgs a, AdjArgs d, SweepGeom g) {
    __shared__ MomShared sm[AW];
    MomShared &M = sm[threadIdx.x >> 5];
    MomRev<COMP> job{a, d, M, M.rows};
    int IS, JS;
    sweep_dir_of(d.it, IS, JS);
    if (COMP == 1) { IS = -IS; JS = -JS; }   // model-1 V sweeps with (-IS, -JS)
    rev_tasks(a, d, g, IS, JS, job);
}

// ------------------------------------------------------------------------------------------------
// pressure correction (PrognosticFlowfield.cs:804-901): per column, for k = VI..KK+1
//   DIM_k = DIV_k/DTIME + (DPM_im + DPM_ip)/DXK*DYK*DZK + (DPM_jm - DPM_jp)/DYK*DXK*DZK
//   Q_k = (ATP_k*Q_{k+1} + DIM_k)*TERMP_k   (Q_{VI+1} from the row carry)
// then DPM_k = P_k*DPM_{k-1} + Q_k and DPMNEW_k += relaxp*DPM_k for k = KK+1..VI.  The neighbours
// not yet swept hold 0 (DPM is zeroed before the sweep), so only the two predecessors carry
// cotangents; P and TERMP do not depend on the state.
// ------------------------------------------------------------------------------------------------
struct __align__(16) PresShared {
    float4 rec[KMAX_LEVELS + 2 * RPAD];   // cotangent of Q (mu), carry cotangent, ATP*TERMP, TERMP
    float2 sp[KMAX_LEVELS + 2 * RPAD];    // cotangent of DPM (relaxp * that of DPMNEW before the wait), P
    float ldim[KMAX_LEVELS];              // cotangent of DIM
};

struct PresRev {
    const KArgs &a;
    const AdjArgs &d;
    PresShared &M;
    ColCtx c;
    bool act;
    bool reader;                 // some later column of the row read this column's row carry
    int dirx;                    // 0: IS = +1, 1: IS = -1

    // before the wait: the state-independent level records, and the cotangents of DPMNEW and of
    // DPM as the later phases left them (the successors' parts arrive as words)
    __device__ void pre(int i, int j, int IS, int) {
        const int lane = threadIdx.x & 31;
        c = make_col(a, i, j);
        act = (c.fl & F_ADV) != 0;
        dirx = (IS == 1) ? 0 : 1;
        reader = act && ((d.rcr[c.col] >> dirx) & 1);
        if (!act) return;
        const size_t fsz = (size_t)a.ncols * a.ks;
        const float *P = d.ptab + (size_t)(2 * dirx) * fsz, *TM = d.ptab + (size_t)(2 * dirx + 1) * fsz;
        const float *LN = d.lam[FDP], *LD = d.lam[L_DPM];
        for (int k = lane; k <= c.VI + 1 && k < KMAX_LEVELS; k += 32) {
            const size_t e = cell(a, c.col, k);
            const float tm = TM[e];
            const float ld = (k > c.KK && k <= c.VI) ? __ldcg(LD + e) : 0.0f;
            M.sp[RPAD + k] = make_float2(ld + a.relaxp * __ldcg(LN + e), P[e]);
            M.rec[RPAD + k] = make_float4(0.0f, 0.0f, a.atp[k] * tm, tm);
        }
        __syncwarp();
    }

    // the successors' words: added to the cotangent of DPM at the solved levels, to the field at
    // every other level (and everywhere in an inactive column)
    __device__ int receive(bool s1, bool s2) {
        const int lane = threadIdx.x & 31;
        float v[2];
        if (!poll_words(a, d, c.col, s1, s2, v)) return 0;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (k >= a.ks || v[r] == 0.0f) continue;
            if (act && k > c.KK && k <= c.VI) M.sp[RPAD + k].x += v[r];
            else atomicAdd(d.lam[L_DPM] + cell(a, c.col, k), v[r]);
        }
        return 1;
    }

    // after the wait: the two reversed recurrences on lane 0, then the predecessors' cotangents
    __device__ void critical(int IS, int JS, bool p1, bool p2) {
        const int lane = threadIdx.x & 31;
        if (!act) {
            send(IS, JS, p1, p2);
            return;
        }
        float *LQ = d.lam[L_QC];
        float4 *rec = M.rec + RPAD;
        const float2 *sp = M.sp + RPAD;
        const int K1 = c.KK + 1, VI = c.VI;
        // carry cotangents left by the columns that read this one's row carry: every one of them
        // fenced its add before the words that led here
        if (reader)
            for (int k = K1 + lane; k <= VI; k += 32) rec[k].y = __ldcg(LQ + cell(a, c.col, k));
        __syncwarp();
        if (lane == 0) {
            // back-substitution reversed, top down: mu_k = S0_k + P_{k+1}*mu_{k+1} (cotangent of Q_k)
            float next = 0.0f;
            float2 x0 = sp[VI], x1 = sp[VI - 1], x2 = sp[VI - 2], x3 = sp[VI - 3];
            for (int k = VI; k >= K1; k -= 4) {
                const float2 y0 = sp[k - 4], y1 = sp[k - 5], y2 = sp[k - 6], y3 = sp[k - 7];
                float mu = x0.x + next;
                next = x0.y * mu;
                rec[k].x = mu;
                mu = x1.x + next;
                next = x1.y * mu;
                if (k - 1 >= K1) rec[k - 1].x = mu;
                mu = x2.x + next;
                next = x2.y * mu;
                if (k - 2 >= K1) rec[k - 2].x = mu;
                mu = x3.x + next;
                next = x3.y * mu;
                if (k - 3 >= K1) rec[k - 3].x = mu;
                x0 = y0; x1 = y1; x2 = y2; x3 = y3;
            }
            // elimination reversed, bottom up: lam_k = mu_k + S1_k + ATP_{k-1}*TERMP_{k-1}*lam_{k-1};
            // the cotangent of DIM_k is lam_k*TERMP_k
            float prev = 0.0f, topp = 0.0f;
            float4 r0 = rec[K1], r1 = rec[K1 + 1], r2 = rec[K1 + 2], r3 = rec[K1 + 3];
            for (int k = K1; k <= VI; k += 4) {
                const float4 t0 = rec[k + 4], t1 = rec[k + 5], t2 = rec[k + 6], t3 = rec[k + 7];
                float lam = r0.x + r0.y + prev;
                M.ldim[k] = lam * r0.w;
                prev = r0.z * lam;
                if (k == VI) topp = prev;
                lam = r1.x + r1.y + prev;
                if (k + 1 <= VI) M.ldim[k + 1] = lam * r1.w;
                prev = r1.z * lam;
                if (k + 1 == VI) topp = prev;
                lam = r2.x + r2.y + prev;
                if (k + 2 <= VI) M.ldim[k + 2] = lam * r2.w;
                prev = r2.z * lam;
                if (k + 2 == VI) topp = prev;
                lam = r3.x + r3.y + prev;
                if (k + 3 <= VI) M.ldim[k + 3] = lam * r3.w;
                prev = r3.z * lam;
                if (k + 3 == VI) topp = prev;
                r0 = t0; r1 = t1; r2 = t2; r3 = t3;
            }
            // the top level read Q_{VI+1} of the row carry: its writer runs after this column and
            // reads the add once the words that follow have reached it, so the add is fenced first
            const short2 w = a.rcw[c.col];
            const int wi = dirx == 0 ? w.x : w.y;
            if (wi >= 0 && topp != 0.0f) {
                atomicAdd(LQ + cell(a, wi * a.nj2 + c.j, VI + 1), topp);
                __threadfence();
            }
        }
        __syncwarp();
        send(IS, JS, p1, p2);
    }

    // the cotangents of the predecessors' DPM for every level (zero outside the column's solve):
    // as words to a predecessor inside the sweep, added to the field of one outside it
    __device__ void send(int IS, int JS, bool p1, bool p2) {
        const int lane = threadIdx.x & 31;
        const int c1 = c.col - IS * a.nj2, c2 = c.col - JS;
        unsigned long long *w1 = d.slot + (size_t)c1 * a.ks;
        unsigned long long *w2 = d.slot + ((size_t)a.ncols + c2) * a.ks;
        float *LD = d.lam[L_DPM];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int k = lane + 32 * r;
            if (k >= a.ks) continue;
            float g1 = 0.0f, g2 = 0.0f;
            if (act && k > c.KK && k <= c.VI) {
                const float lD = M.ldim[k];
                if (lD != 0.0f) {
                    const float dz = a.dzk[k];
                    g1 = lD * (a.dyk * dz / a.dxk);
                    // DPM_jm enters with +, DPM_jp with - (the reference's sign, :853-854)
                    g2 = (JS == 1 ? 1.0f : -1.0f) * lD * (a.dxk * dz / a.dyk);
                }
            }
            if (p1) st_word(w1 + k, g1, d.stamp);
            else if (g1 != 0.0f) atomicAdd(LD + cell(a, c1, k), g1);
            if (p2) st_word(w2 + k, g2, d.stamp);
            else if (g2 != 0.0f) atomicAdd(LD + cell(a, c2, k), g2);
        }
    }

    __device__ void after(int, int) {
        if (!act) return;
        const int lane = threadIdx.x & 31;
        const float dt = a.sit[0].dtime;
        float *LQ = d.lam[L_QC];
        for (int k = c.KK + 1 + lane; k <= c.VI; k += 32) {
            const size_t e = cell(a, c.col, k);
            d.lam[L_DIV][e] = M.ldim[k] / dt;
            if (reader) LQ[e] = 0.0f;   // the carry cotangents were consumed
        }
    }
};

__global__ void __launch_bounds__(AW * 32) k_adj_pressure(KArgs a, AdjArgs d, SweepGeom g) {
    __shared__ PresShared sm[AW];
    PresRev job{a, d, sm[threadIdx.x >> 5]};
    int IS, JS;
    sweep_dir_of(d.it, IS, JS);
    rev_tasks(a, d, g, IS, JS, job);
}

// which columns' row carry some column reads (bit 0: IS = +1, bit 1: IS = -1); rcr zeroed before
__global__ void k_adj_readers(KArgs a, int *rcr) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= a.ncols) return;
    const short2 w = a.rcw[col];
    const int j = col % a.nj2;
    if (w.x >= 0) atomicOr(rcr + w.x * a.nj2 + j, 1);
    if (w.y >= 0) atomicOr(rcr + w.y * a.nj2 + j, 2);
}

// ------------------------------------------------------------------------------------------------
// pointwise phases: one warp per column, lanes over levels
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ bool warp_col(const KArgs &a, int &col, int &i, int &j) {
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (gw >= a.ncols) return false;
    col = (int)gw;
    i = col / a.nj2;
    j = col - i * a.nj2;
    return true;
}

// velocity correction (:904-949) reversed: cotangent of DPM gathered from the corrected U, V, W
// (DPM is only read), and the cotangent of a W the correction sets to 0 cleared
__device__ __forceinline__ bool vc_u(const KArgs &a, int i, int j, int k) {
    if (i < 3 || i > a.nii - 1 || j < 2 || j > a.njj - 1) return false;   // du: i > 2
    const int col = i * a.nj2 + j;
    if (!(a.cflags[col] & F_VC)) return false;
    const ColMeta m = a.meta[col];
    return k >= 1 && k <= m.vi && m.kkm_u < k;
}
__device__ __forceinline__ bool vc_v(const KArgs &a, int i, int j, int k) {
    if (i < 2 || i > a.nii - 1 || j < 3 || j > a.njj - 1) return false;   // dv: j > 2
    const int col = i * a.nj2 + j;
    if (!(a.cflags[col] & F_VC)) return false;
    const ColMeta m = a.meta[col];
    return k >= 1 && k <= m.vi && m.kkm_v < k;
}
// 1: W corrected, 0: W set to 0, -1: not touched
__device__ __forceinline__ int vc_w(const KArgs &a, int i, int j, int k) {
    if (i < 2 || i > a.nii - 1 || j < 2 || j > a.njj - 1) return -1;
    const int col = i * a.nj2 + j;
    if (!(a.cflags[col] & F_VC)) return -1;
    const ColMeta m = a.meta[col];
    if (k < 1 || k > m.vi) return -1;
    return (m.kkart + 1 < k) ? 1 : 0;
}

__global__ void k_adj_velcorr(KArgs a, AdjArgs d) {
    int col, i, j;
    if (!warp_col(a, col, i, j)) return;
    const int lane = threadIdx.x & 31;
    const float DT = a.sit[0].dtime;
    const float *LU = d.lam[FU], *LV = d.lam[FV];
    float *LW = d.lam[FW];
    const int nj2 = a.nj2;
    for (int k = lane; k < a.ks; k += 32) {
        float g = 0.0f;
        if (k >= 1) {
            if (vc_u(a, i, j, k)) g -= LU[cell(a, col, k)] / a.dxk * DT;
            if (vc_u(a, i + 1, j, k)) g += LU[cell(a, col + nj2, k)] / a.dxk * DT;
            if (vc_v(a, i, j, k)) g -= LV[cell(a, col, k)] / a.dyk * DT;
            if (vc_v(a, i, j + 1, k)) g += LV[cell(a, col + 1, k)] / a.dyk * DT;
            if (vc_w(a, i, j, k) == 1) g -= LW[cell(a, col, k)] / (a.dzk[k] + a.dzk[k - 1]) * 2.0f * DT;
            if (k + 1 < a.ks && vc_w(a, i, j, k + 1) == 1)
                g += LW[cell(a, col, k + 1)] / (a.dzk[k + 1] + a.dzk[k]) * 2.0f * DT;
        }
        d.lam[L_DPM][cell(a, col, k)] = g;
    }
    __syncwarp();
    for (int k = lane; k < a.ks; k += 32)
        if (vc_w(a, i, j, k) == 0) LW[cell(a, col, k)] = 0.0f;
}

// staggered averages (:958-1039) reversed in three passes: the border copies, the gathers into
// U, V, W, the clearing of the overwritten averages' cotangents
__device__ __forceinline__ bool av_col(const KArgs &a, int i, int j) {
    if (i < 2 || i > a.nii - 1 || j < 2 || j > a.njj - 1) return false;
    return (a.cflags[i * a.nj2 + j] & F_VC) != 0;
}

__global__ void k_adj_avg_copies(KArgs a, AdjArgs d) {
    int col, i, j;
    if (!warp_col(a, col, i, j)) return;
    if (!av_col(a, i, j)) return;
    const int lane = threadIdx.x & 31;
    const int nj2 = a.nj2;
    float *LUS = d.lam[FUS], *LVS = d.lam[FVS];
    // VKS[1][j] = VKS[2][j], VKS[NII][j] = VKS[NII-1][j] on every level (after the level loop)
    const bool west = (i == 2) && (a.cflags[1 * nj2 + j] & F_ADV);
    const bool east = (i == a.nii - 1) && (a.cflags[col] & F_ADV);
    if (west || east) {
        const long long dd = west ? -(long long)nj2 : nj2;
        for (int k = lane; k < a.ks; k += 32) {
            const size_t e = cell(a, (int)(col + dd), k);
            LVS[cell(a, col, k)] += LVS[e];
            LVS[e] = 0.0f;
        }
    }
    // UKS[i][1] = UKS[i][2] and UKS[i][NJJ] = UKS[i][NJJ-1] on KSTART..VI
    const ColMeta m = a.meta[col];
    const bool cpS = (j == 2);
    const bool cpN = (j == a.njj - 1) && (a.cflags[i * nj2 + a.njj] & F_ADV);
    if (cpS || cpN) {
        for (int k = lane; k < a.ks; k += 32) {
            if (k < m.kstart || k > m.vi) continue;
            float add = 0.0f;
            if (cpS) { const size_t e = cell(a, col - 1, k); add += LUS[e]; LUS[e] = 0.0f; }
            if (cpN) { const size_t e = cell(a, col + 1, k); add += LUS[e]; LUS[e] = 0.0f; }
            LUS[cell(a, col, k)] += add;
        }
    }
}

// level k of column (i, j) gets a new UKS/VKS (kind 0) or WKS (kind 1) from the averages
__device__ __forceinline__ bool av_new(const KArgs &a, int i, int j, int k, int kind) {
    if (!av_col(a, i, j)) return false;
    const ColMeta m = a.meta[i * a.nj2 + j];
    if (k < m.kstart || k > m.vi) return false;
    return kind == 0 ? (m.kkart < k) : (m.kkart + 1 < k);
}

__global__ void k_adj_avg_gather(KArgs a, AdjArgs d) {
    int col, i, j;
    if (!warp_col(a, col, i, j)) return;
    const int lane = threadIdx.x & 31;
    const int nj2 = a.nj2;
    const float *LUS = d.lam[FUS], *LVS = d.lam[FVS], *LWS = d.lam[FWS];
    for (int k = lane; k < a.ks; k += 32) {
        float gu = 0.0f, gv = 0.0f, gw = 0.0f;
        if (av_new(a, i, j, k, 0)) { gu += 0.5f * LUS[cell(a, col, k)]; gv += 0.5f * LVS[cell(a, col, k)]; }
        if (av_new(a, i - 1, j, k, 0)) gu += 0.5f * LUS[cell(a, col - nj2, k)];
        if (av_new(a, i, j - 1, k, 0)) gv += 0.5f * LVS[cell(a, col - 1, k)];
        if (av_new(a, i, j, k, 1)) gw += 0.5f * LWS[cell(a, col, k)];
        if (k >= 1 && av_new(a, i, j, k - 1, 1)) gw += 0.5f * LWS[cell(a, col, k - 1)];
        if (gu != 0.0f) d.lam[FU][cell(a, col, k)] += gu;
        if (gv != 0.0f) d.lam[FV][cell(a, col, k)] += gv;
        if (gw != 0.0f) d.lam[FW][cell(a, col, k)] += gw;
    }
}

__global__ void k_adj_avg_clear(KArgs a, AdjArgs d) {
    int col, i, j;
    if (!warp_col(a, col, i, j)) return;
    const int lane = threadIdx.x & 31;
    for (int k = lane; k < a.ks; k += 32) {
        if (av_new(a, i, j, k, 0)) { d.lam[FUS][cell(a, col, k)] = 0.0f; d.lam[FVS][cell(a, col, k)] = 0.0f; }
        if (av_new(a, i, j, k, 1)) d.lam[FWS][cell(a, col, k)] = 0.0f;
    }
}

// divergence (:723-758) reversed: a gather of the cotangent of DIV into U, V, W
__device__ __forceinline__ bool div_at(const KArgs &a, int i, int j, int k) {
    if (i < 2 || i > a.nii - 1 || j < 2 || j > a.njj - 1) return false;
    const int col = i * a.nj2 + j;
    if (!(a.cflags[col] & F_ADV)) return false;
    const ColMeta m = a.meta[col];
    return k > m.kkart && k <= m.vi;
}

__global__ void k_adj_div(KArgs a, AdjArgs d) {
    int col, i, j;
    if (!warp_col(a, col, i, j)) return;
    const int lane = threadIdx.x & 31;
    const int nj2 = a.nj2;
    const float *LDV = d.lam[L_DIV];
    const float AREA = a.areaxy;
    for (int k = lane; k < a.ks; k += 32) {
        if (k < 1) continue;
        const float dz = a.dzk[k];
        float gu = 0.0f, gv = 0.0f, gw = 0.0f;
        if (div_at(a, i, j, k)) {
            const float l = LDV[cell(a, col, k)];
            gu += l * a.dyk * dz;
            gv += l * a.dxk * dz;
            if (k > a.meta[col].kkart + 1) gw += l * AREA;
        }
        if (div_at(a, i - 1, j, k)) gu -= LDV[cell(a, col - nj2, k)] * a.dyk * dz;
        if (div_at(a, i, j - 1, k)) gv -= LDV[cell(a, col - 1, k)] * a.dxk * dz;
        if (div_at(a, i, j, k - 1)) gw -= LDV[cell(a, col, k - 1)] * AREA;
        if (gu != 0.0f) d.lam[FU][cell(a, col, k)] += gu;
        if (gv != 0.0f) d.lam[FV][cell(a, col, k)] += gv;
        if (gw != 0.0f) d.lam[FW][cell(a, col, k)] += gw;
    }
}

// ------------------------------------------------------------------------------------------------
// lateral and top boundary conditions (:595-714).  The recompute runs the forward copies itself
// (the same operations as the solver's boundary kernels) and keeps the branch of every
// sign-conditioned copy; the reverse undoes the copies in reverse order.
// ------------------------------------------------------------------------------------------------
__global__ void k_adj_bc_we_fwd(KArgs a, BcLists bc, uint8_t *bits) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 2 + (int)(t / a.ks);
    const int k = (int)(t % a.ks);
    if (j > a.njj || k < 1) return;
    const int nj2 = a.nj2;
    for (int e = bc.we_ptr[j]; e < bc.we_ptr[j + 1]; ++e) {
        const int ev = bc.we_ev[e];
        const int i = ev & 0xffff;
        const int c = i * nj2 + j;
        if (k > a.meta[c].vi) continue;
        uint8_t b = 0;
        if (ev & (1 << 16)) {
            const float u = a.uk[cell(a, c - 2 * nj2, k)];
            if (u >= 0) { a.uk[cell(a, c - nj2, k)] = u; b |= 1; }
            a.vk[cell(a, c - 2 * nj2, k)] = a.vk[cell(a, c - nj2, k)];
            a.wk[cell(a, c - 2 * nj2, k)] = a.wk[cell(a, c - nj2, k)];
        }
        if (ev & (1 << 17)) {
            const float u = a.uk[cell(a, c + 2 * nj2, k)];
            if (u <= 0) { a.uk[cell(a, c + nj2, k)] = u; b |= 2; }
            a.vk[cell(a, c + nj2, k)] = a.vk[cell(a, c, k)];
            a.wk[cell(a, c + nj2, k)] = a.wk[cell(a, c, k)];
        }
        bits[(size_t)e * a.ks + k] = b;
    }
}

__global__ void k_adj_bc_sn_fwd(KArgs a, BcLists bc, uint8_t *bits, int nwe) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = 2 + (int)(t / a.ks);
    const int k = (int)(t % a.ks);
    if (i > a.nii || k < 1) return;
    const int nj2 = a.nj2;
    for (int e = bc.sn_ptr[i]; e < bc.sn_ptr[i + 1]; ++e) {
        const int ev = bc.sn_ev[e];
        const int j = ev & 0xffff;
        const int c = i * nj2 + j;
        if (k > a.meta[c].vi) continue;
        uint8_t b = 0;
        if (ev & (1 << 16)) {
            const float v = a.vk[cell(a, c - 2, k)];
            if (v >= 0) { a.vk[cell(a, c - 1, k)] = v; b |= 1; }
            a.uk[cell(a, c - 2, k)] = a.uk[cell(a, c - 1, k)];
            a.wk[cell(a, c - 2, k)] = a.wk[cell(a, c - 1, k)];
        }
        if (ev & (1 << 17)) {
            const float v = a.vk[cell(a, c + 2, k)];
            if (v <= 0) { a.vk[cell(a, c + 1, k)] = v; b |= 2; }
            a.uk[cell(a, c + 1, k)] = a.uk[cell(a, c, k)];
            a.wk[cell(a, c + 1, k)] = a.wk[cell(a, c, k)];
        }
        bits[(size_t)(nwe + e) * a.ks + k] = b;
    }
}

__global__ void k_adj_bc_top_fwd(KArgs a) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.ncols) return;
    const int col = (int)t, i = col / a.nj2, j = col - i * a.nj2;
    if (i < 2 || i > a.nii - 1 || j < 2 || j > a.njj - 1) return;
    if (!(a.cflags[col] & F_ADV)) return;
    const int k = a.meta[col].vi;
    a.wk[cell(a, col, k + 1)] = a.wk[cell(a, col, k)];
    a.uk[cell(a, col, k + 1)] = a.uk[cell(a, col, k)];
    a.vk[cell(a, col, k + 1)] = a.vk[cell(a, col, k)];
}

// a = b reversed: the cotangent of a moves to b
__device__ __forceinline__ void rev_copy(float *L, size_t dst, size_t src) {
    L[src] += L[dst];
    L[dst] = 0.0f;
}

__global__ void k_adj_bc_top_rev(KArgs a, AdjArgs d) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.ncols) return;
    const int col = (int)t, i = col / a.nj2, j = col - i * a.nj2;
    if (i < 2 || i > a.nii - 1 || j < 2 || j > a.njj - 1) return;
    if (!(a.cflags[col] & F_ADV)) return;
    const int k = a.meta[col].vi;
    rev_copy(d.lam[FV], cell(a, col, k + 1), cell(a, col, k));
    rev_copy(d.lam[FU], cell(a, col, k + 1), cell(a, col, k));
    rev_copy(d.lam[FW], cell(a, col, k + 1), cell(a, col, k));
}

__global__ void k_adj_bc_sn_rev(KArgs a, BcLists bc, AdjArgs d) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = 2 + (int)(t / a.ks);
    const int k = (int)(t % a.ks);
    if (i > a.nii || k < 1) return;
    float *LU = d.lam[FU], *LV = d.lam[FV], *LW = d.lam[FW];
    for (int e = bc.sn_ptr[i + 1] - 1; e >= bc.sn_ptr[i]; --e) {
        const int ev = bc.sn_ev[e];
        const int j = ev & 0xffff;
        const int c = i * a.nj2 + j;
        if (k > a.meta[c].vi) continue;
        const uint8_t b = d.bits[(size_t)(d.nwe + e) * a.ks + k];
        if (ev & (1 << 17)) {
            rev_copy(LW, cell(a, c + 1, k), cell(a, c, k));
            rev_copy(LU, cell(a, c + 1, k), cell(a, c, k));
            if (b & 2) rev_copy(LV, cell(a, c + 1, k), cell(a, c + 2, k));
        }
        if (ev & (1 << 16)) {
            rev_copy(LW, cell(a, c - 2, k), cell(a, c - 1, k));
            rev_copy(LU, cell(a, c - 2, k), cell(a, c - 1, k));
            if (b & 1) rev_copy(LV, cell(a, c - 1, k), cell(a, c - 2, k));
        }
    }
}

__global__ void k_adj_bc_we_rev(KArgs a, BcLists bc, AdjArgs d) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 2 + (int)(t / a.ks);
    const int k = (int)(t % a.ks);
    if (j > a.njj || k < 1) return;
    const int nj2 = a.nj2;
    float *LU = d.lam[FU], *LV = d.lam[FV], *LW = d.lam[FW];
    for (int e = bc.we_ptr[j + 1] - 1; e >= bc.we_ptr[j]; --e) {
        const int ev = bc.we_ev[e];
        const int i = ev & 0xffff;
        const int c = i * nj2 + j;
        if (k > a.meta[c].vi) continue;
        const uint8_t b = d.bits[(size_t)e * a.ks + k];
        if (ev & (1 << 17)) {
            rev_copy(LW, cell(a, c + nj2, k), cell(a, c, k));
            rev_copy(LV, cell(a, c + nj2, k), cell(a, c, k));
            if (b & 2) rev_copy(LU, cell(a, c + nj2, k), cell(a, c + 2 * nj2, k));
        }
        if (ev & (1 << 16)) {
            rev_copy(LW, cell(a, c - 2 * nj2, k), cell(a, c - nj2, k));
            rev_copy(LV, cell(a, c - 2 * nj2, k), cell(a, c - nj2, k));
            if (b & 1) rev_copy(LU, cell(a, c - nj2, k), cell(a, c - 2 * nj2, k));
        }
    }
}

// ------------------------------------------------------------------------------------------------
// set-up (:295-329, 410-432, 518-575) reversed, on the full-height staging layout of the initial
// fields: gather of the device layout, zeroing inside buildings, border copies, staggered averages
// ------------------------------------------------------------------------------------------------
struct StageLam {
    float *u, *v, *w;   // [NII+2][NJJ+2][NKK+2]
};

__device__ __forceinline__ size_t sx(const KArgs &a, int i, int j, int k) {
    return ((size_t)i * a.nj2 + j) * (a.nkk + 2) + k;
}

// levels below KS come from the device-layout cotangents (the levels above pass through)
__global__ void k_adj_setup_scatter(KArgs a, AdjArgs d, StageLam L) {
    int col, i, j;
    if (!warp_col(a, col, i, j)) return;
    const int lane = threadIdx.x & 31;
    const int nk2 = a.nkk + 2;
    for (int k = lane; k < a.ks && k < nk2; k += 32) {
        const size_t s = (size_t)col * nk2 + k;
        L.u[s] = d.lam[FU][cell(a, col, k)];
        L.v[s] = d.lam[FV][cell(a, col, k)];
        L.w[s] = d.lam[FW][cell(a, col, k)];
    }
}

__global__ void k_adj_setup_zero(KArgs a, AdjArgs d, StageLam L) {
    int col, i, j;
    if (!warp_col(a, col, i, j)) return;
    if (i < 1 || i > a.nii || j < 1 || j > a.njj) return;
    if (!(a.cflags[col] & F_ADV)) return;
    const int lane = threadIdx.x & 31;
    const ColMeta m = a.meta[col];
    for (int k = 1 + lane; k <= m.vi; k += 32) {
        if (m.kkart < k) continue;
        L.u[sx(a, i, j, k)] = 0.0f;
        if (i == a.nii) L.u[sx(a, i + 1, j, k)] = 0.0f;
        L.v[sx(a, i, j, k)] = 0.0f;
        if (j == a.njj) L.v[sx(a, i, j + 1, k)] = 0.0f;
        L.w[sx(a, i, j, k)] = 0.0f;
        if (k == m.vi) L.w[sx(a, i, j, k + 1)] = 0.0f;
        d.lam[FUS][cell(a, col, k)] = 0.0f;
        d.lam[FVS][cell(a, col, k)] = 0.0f;
        d.lam[FWS][cell(a, col, k)] = 0.0f;
    }
}

// UK[NII+1] = UK[NII], VK[.][NJJ+1] = VK[.][NJJ] on levels 1..NKK-1, reversed
__global__ void k_adj_setup_border(KArgs a, StageLam L) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nk = a.nkk - 1;
    const long long per = (long long)(a.njj + a.nii) * nk;
    if (t >= per) return;
    const int k = 1 + (int)(t % nk);
    const int q = (int)(t / nk);
    if (q < a.njj) {
        const int j = 1 + q;
        L.u[sx(a, a.nii, j, k)] += L.u[sx(a, a.nii + 1, j, k)];
        L.u[sx(a, a.nii + 1, j, k)] = 0.0f;
    } else {
        const int i = 1 + (q - a.njj);
        L.v[sx(a, i, a.njj, k)] += L.v[sx(a, i, a.njj + 1, k)];
        L.v[sx(a, i, a.njj + 1, k)] = 0.0f;
    }
}

// initial staggered averages UKS = (UK_i + UK_i+1)/2 etc. on the columns with ADVDOM in their 3x3
// neighbourhood, levels 1..NKK-1 (those below KS are kept), reversed as a gather
__device__ __forceinline__ bool uks0(const KArgs &a, int i, int j, int k) {
    if (i < 1 || i > a.nii || j < 1 || j > a.njj) return false;
    if (!(a.cflags[i * a.nj2 + j] & F_ALLOC3)) return false;
    return k >= 1 && k <= a.nkk - 1 && k < a.ks;
}

__global__ void k_adj_setup_avg(KArgs a, AdjArgs d, StageLam L) {
    int col, i, j;
    if (!warp_col(a, col, i, j)) return;
    const int lane = threadIdx.x & 31;
    const int nj2 = a.nj2;
    for (int k = lane; k < a.ks && k <= a.nkk; k += 32) {
        float gu = 0.0f, gv = 0.0f, gw = 0.0f;
        if (uks0(a, i, j, k)) {
            gu += 0.5f * d.lam[FUS][cell(a, col, k)];
            gv += 0.5f * d.lam[FVS][cell(a, col, k)];
            gw += 0.5f * d.lam[FWS][cell(a, col, k)];
        }
        if (uks0(a, i - 1, j, k)) gu += 0.5f * d.lam[FUS][cell(a, col - nj2, k)];
        if (uks0(a, i, j - 1, k)) gv += 0.5f * d.lam[FVS][cell(a, col - 1, k)];
        if (k >= 1 && uks0(a, i, j, k - 1)) gw += 0.5f * d.lam[FWS][cell(a, col, k - 1)];
        const size_t s = (size_t)col * (a.nkk + 2) + k;
        L.u[s] += gu;
        L.v[s] += gv;
        L.w[s] += gw;
    }
}

// VEG cotangent in the host layout [NII+2][NJJ+2][NKK+2] (device layout index k-1 -> level k-1)
__global__ void k_adj_veg_out(KArgs a, AdjArgs d, float *out) {
    int col, i, j;
    if (!warp_col(a, col, i, j)) return;
    const int lane = threadIdx.x & 31;
    const int nk2 = a.nkk + 2;
    for (int k = lane; k < nk2; k += 32)
        out[(size_t)col * nk2 + k] = (k < a.ks) ? d.lam[FVEG][cell(a, col, k)] : 0.0f;
}

// host-layout cotangents of the final fields -> device layout (levels below KS)
__global__ void k_adj_gather_in(KArgs a, AdjArgs d, StageLam L) {
    int col, i, j;
    if (!warp_col(a, col, i, j)) return;
    const int lane = threadIdx.x & 31;
    const int nk2 = a.nkk + 2;
    for (int k = lane; k < a.ks; k += 32) {
        const bool in = k < nk2;
        const size_t s = (size_t)col * nk2 + k;
        d.lam[FU][cell(a, col, k)] = in ? L.u[s] : 0.0f;
        d.lam[FV][cell(a, col, k)] = in ? L.v[s] : 0.0f;
        d.lam[FW][cell(a, col, k)] = in ? L.w[s] : 0.0f;
    }
}

}  // namespace

// ================================================================================================
// host side
// ================================================================================================

namespace {

int col_blocks(const KArgs &a) { return (a.ncols * 32 + 255) / 256; }

// one Gauss-Seidel phase of the forward on the loaded schedule (strips or diagonal claims)
void forward_phase(gral_ctx *ctx, int kind, const SweepGeom &g, cudaStream_t st) {
    if (ctx->pmode > 0) launch_strip(kind, ctx->ka, g, strip_variant_of(ctx), ctx->strip_grid[kind], st);
    else launch_gs(kind, ctx->ka, g, ctx->grid_gs[kind], st);
}

// one forward SIMPLE iteration with separate phase launches on stream st; when `keep` is given,
// the mid and end states go there and the boundary copies' branches to `bits`
int forward_iteration(gral_ctx *ctx, float *keep, uint8_t *bits, cudaStream_t st) {
    const KArgs &a = ctx->ka;
    CK(cudaMemsetAsync(ctx->counters.p, 0, 8 * kCounterSlots * sizeof(unsigned int), st));
    if (bits) {
        const long long nw = (long long)(a.njj - 1) * a.ks, ns = (long long)(a.nii - 1) * a.ks;
        k_adj_bc_we_fwd<<<(int)((nw + 127) / 128), 128, 0, st>>>(a, ctx->bc, bits);
        k_adj_bc_sn_fwd<<<(int)((ns + 127) / 128), 128, 0, st>>>(a, ctx->bc, bits, ctx->adj_nwe);
        k_adj_bc_top_fwd<<<(a.ncols + 127) / 128, 128, 0, st>>>(a);
    } else {
        launch_bc(a, ctx->bc, st);
    }
    forward_phase(ctx, PH_PRESSURE, ctx->geo_p.g, st);
    launch_velcorr(a, st);
    launch_average(a, st);
    const size_t fsz = (size_t)a.ncols * a.ks;
    if (keep) {
        const float *src[7] = {a.uk, a.vk, a.wk, a.uks, a.vks, a.wks, a.dpmnew};
        for (int q = 0; q < 7; ++q)
            CK(cudaMemcpyAsync(keep + q * fsz, src[q], fsz * sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
    forward_phase(ctx, PH_U, ctx->geo_u.g, st);
    forward_phase(ctx, PH_V, ctx->geo_v.g, st);
    forward_phase(ctx, PH_W, ctx->geo_p.g, st);
    launch_bookkeeping(a, st);
    if (keep) {
        const float *src[3] = {a.uk, a.vk, a.wk};
        for (int q = 0; q < 3; ++q)
            CK(cudaMemcpyAsync(keep + (7 + q) * fsz, src[q], fsz * sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
    return GRAL_OK;
}

// the state of a checkpoint: fields, loop state, IterationLoops; wavefront flags cleared
int save_checkpoint(gral_ctx *ctx, int q) {
    const KArgs &a = ctx->ka;
    cudaStream_t st = ctx->stream;
    const size_t fsz = (size_t)a.ncols * a.ks;
    const float *src[NCKPT] = {a.uk, a.vk, a.wk, a.uks, a.vks, a.wks, a.dpmnew};
    float *dst = ctx->adj_ckpt.p + (size_t)q * NCKPT * fsz;
    for (int f = 0; f < NCKPT; ++f)
        CK(cudaMemcpyAsync(dst + f * fsz, src[f], fsz * sizeof(float), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(ctx->adj_cksit.p + q, a.sit, sizeof(SitDev), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(ctx->adj_ckit.p + q, a.it_global, sizeof(int), cudaMemcpyDeviceToDevice, st));
    return GRAL_OK;
}

int restore_checkpoint(gral_ctx *ctx, int q, cudaStream_t st) {
    const KArgs &a = ctx->ka;
    const size_t fsz = (size_t)a.ncols * a.ks;
    float *dst[NCKPT] = {a.uk, a.vk, a.wk, a.uks, a.vks, a.wks, a.dpmnew};
    const float *src = ctx->adj_ckpt.p + (size_t)q * NCKPT * fsz;
    for (int f = 0; f < NCKPT; ++f)
        CK(cudaMemcpyAsync(dst[f], src + f * fsz, fsz * sizeof(float), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(a.sit, ctx->adj_cksit.p + q, sizeof(SitDev), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(a.it_global, ctx->adj_ckit.p + q, sizeof(int), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemsetAsync(a.flags, 0, (size_t)a.ncols * sizeof(int), st));
    return GRAL_OK;
}

// P and TERMP of the pressure elimination per column, level and i-direction (they depend on the
// grid and on the row carry of P, not on the state): the forward's row loop replayed on the host
int pressure_tables(gral_ctx *ctx) {
    const KArgs &a = ctx->ka;
    const int ks = a.ks, nj2 = a.nj2, NII = a.nii, NJJ = a.njj;
    std::vector<ColMeta> meta(a.ncols);
    std::vector<uint32_t> fl(a.ncols);
    std::vector<float> tab(5 * (size_t)ks);
    CK(cudaMemcpy(meta.data(), a.meta, meta.size() * sizeof(ColMeta), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(fl.data(), a.cflags, fl.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(tab.data(), ctx->tables.p, tab.size() * sizeof(float), cudaMemcpyDeviceToHost));
    const float *APP = tab.data() + 2 * ks, *ABP = tab.data() + 3 * ks, *ATP = tab.data() + 4 * ks;
    const size_t fsz = (size_t)a.ncols * ks;
    std::vector<float> pt(4 * fsz, 0.0f);
    std::vector<float> PIMP(ks + 1);
    for (int dir = 0; dir < 2; ++dir) {
        float *P = pt.data() + (size_t)(2 * dir) * fsz, *TM = pt.data() + (size_t)(2 * dir + 1) * fsz;
        for (int j = 2; j <= NJJ - 1; ++j) {
            std::fill(PIMP.begin(), PIMP.end(), 0.0f);
            for (int q = 2; q <= NII - 1; ++q) {
                const int i = (dir == 0) ? q : NII + 1 - q;
                const int c = i * nj2 + j;
                if (!(fl[c] & F_ADV)) continue;
                for (int k = meta[c].vi; k > meta[c].kkart; --k) {
                    const float termp = 1 / (APP[k] - ATP[k] * PIMP[k + 1]);
                    PIMP[k] = ABP[k] * termp;
                    P[(size_t)c * ks + k] = PIMP[k];
                    TM[(size_t)c * ks + k] = termp;
                }
            }
        }
    }
    CK(ctx->adj_ptab.ensure(pt.size()));
    CK(cudaMemcpy(ctx->adj_ptab.p, pt.data(), pt.size() * sizeof(float), cudaMemcpyHostToDevice));
    return GRAL_OK;
}

int rev_grid(gral_ctx *ctx, const SweepGeom &g) {
    const double width = (double)g.ni * g.nj / std::max(1, g.ni + g.nj - 1);
    double la = 12.0;   // diagonals of wavefront width the reverse sweeps keep warps for (6: 12 % slower)
    if (const char *v = std::getenv("GRAL_PROG_ADJ_LOOKAHEAD")) la = std::max(1.0, std::atof(v));
    const long long want = (long long)std::ceil(la * width / AW);
    return (int)std::max<long long>(ctx->num_sms, std::min<long long>(4LL * ctx->num_sms, want));
}

}  // namespace

}  // namespace gral

using namespace gral;

extern "C" {

int gral_prog_vjp_forward(gral_ctx *ctx, const gral_params *p, const gral_static *s, gral_fields *f,
                          int32_t iterations, int32_t checkpoint_every) {
    if (!ctx) return GRAL_EINVAL;
    if (!p || !s || !f) return fail(ctx, GRAL_EINVAL, "null argument");
    if (p->turbulence_model != 1 || p->simd_width != 8 || p->quantise != 0)
        return fail(ctx, GRAL_EINVAL, "the adjoint differentiates turbulence model 1, parity width 8, quantise 0");
    if (iterations < 1 || checkpoint_every < 0)
        return fail(ctx, GRAL_EINVAL, "iterations must be >= 1 and checkpoint_every >= 0");
    ctx->adj_ready = false;
    gral_params q = *p;
    q.iteration_steps_min = iterations;
    q.iteration_steps_max = iterations;
    q.post_diagnostic = 0;
    CK(cudaSetDevice(ctx->device));
    CK_RC(gral_prog_load(ctx, 1, &q, s, f));
    if (ctx->il) return fail(ctx, GRAL_EINVAL, "the adjoint runs the slab layout (unset GRAL_PROG_LAYOUT)");
    ctx->fused = false;
    CK_RC(plain_schedule_default(ctx));
    const KArgs &a = ctx->ka;
    const size_t fsz = (size_t)a.ncols * a.ks;
    cudaStream_t st = ctx->stream;
    int nev[2] = {0, 0};
    CK(cudaMemcpy(&nev[0], ctx->bc.we_ptr + a.nj2, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&nev[1], ctx->bc.sn_ptr + a.nii + 2, sizeof(int), cudaMemcpyDeviceToHost));
    ctx->adj_nwe = nev[0];
    ctx->adj_nsn = nev[1];
    if (checkpoint_every == 0) {
        // every iteration's kept states (and boundary branches) stay on the device: gral_prog_vjp
        // reverses them without recomputing anything
        const size_t nevk = (size_t)std::max(nev[0] + nev[1], 1) * a.ks;
        CK(ctx->adj_keep.ensure((size_t)iterations * NKEEP * fsz));
        CK(ctx->adj_bits.ensure((size_t)iterations * nevk));
        CK(cudaMemsetAsync(ctx->adj_bits.p, 0, (size_t)iterations * nevk, st));
        CK(cudaEventRecord(ctx->ev[0], st));
        for (int it = 0; it < iterations; ++it)
            CK_RC(forward_iteration(ctx, ctx->adj_keep.p + (size_t)it * NKEEP * fsz, ctx->adj_bits.p + (size_t)it * nevk,
                                    st));
    } else {
        const int nck = (iterations + checkpoint_every - 1) / checkpoint_every;
        CK(ctx->adj_ckpt.ensure((size_t)nck * NCKPT * fsz));
        CK(ctx->adj_cksit.ensure(nck));
        CK(ctx->adj_ckit.ensure(nck));
        CK(cudaEventRecord(ctx->ev[0], st));
        for (int it = 0; it < iterations; ++it) {
            if (it % checkpoint_every == 0) CK_RC(save_checkpoint(ctx, it / checkpoint_every));
            CK_RC(forward_iteration(ctx, nullptr, nullptr, st));
        }
    }
    CK(cudaEventRecord(ctx->ev[1], st));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    ctx->adj_ms_forward = ms;
    int herr = 0;
    CK(cudaMemcpy(&herr, ctx->misc.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr == ERR_TIMEOUT) return fail(ctx, GRAL_ETIMEDOUT, "a wavefront wait exceeded its time limit");
    ctx->it_host = iterations + 1;
    CK_RC(gral_prog_store(ctx, f, nullptr));
    CK_RC(pressure_tables(ctx));
    ctx->adj_iters = iterations;
    ctx->adj_every = checkpoint_every;
    ctx->adj_ready = true;
    return GRAL_OK;
}

int gral_prog_vjp(gral_ctx *ctx, const float *dj_duk, const float *dj_dvk, const float *dj_dwk, float *dj_dveg,
                  float *dj_duk0, float *dj_dvk0, float *dj_dwk0, gral_vjp_stats *stats) {
    if (!ctx) return GRAL_EINVAL;
    if (!ctx->adj_ready) return fail(ctx, GRAL_ESTATE, "gral_prog_vjp before gral_prog_vjp_forward");
    CK(cudaSetDevice(ctx->device));
    KArgs &a = ctx->ka;
    cudaStream_t st = ctx->stream;
    const int N = ctx->adj_iters;
    const bool all = ctx->adj_every == 0;            // every iteration's states kept by the forward
    const int K = all ? N : ctx->adj_every;
    const size_t fsz = (size_t)a.ncols * a.ks, ssz = (size_t)a.ncols * (a.nkk + 2);
    const int nev = ctx->adj_nwe + ctx->adj_nsn;
    const int nseg = (N + K - 1) / K;
    const int nbuf = nseg > 1 ? 2 : 1;     // the next segment is recomputed while this one is reversed
    // (with all states kept there is one segment, and nothing to recompute)
    const size_t nevk = (size_t)std::max(nev, 1) * a.ks;
    CK(ctx->adj_keep.ensure((size_t)nbuf * K * NKEEP * fsz));
    CK(ctx->adj_lam.ensure((size_t)NLAM * fsz));
    CK(ctx->adj_stg.ensure(3 * ssz));
    CK(ctx->adj_slot.ensure(2 * (size_t)a.ncols * a.ks));
    CK(ctx->adj_rcr.ensure(a.ncols));
    CK(ctx->adj_ctr.ensure(4));
    CK(ctx->adj_bits.ensure((size_t)nbuf * K * nevk));
    CK(cudaMemsetAsync(ctx->adj_lam.p, 0, (size_t)NLAM * fsz * sizeof(float), st));
    CK(cudaMemsetAsync(ctx->adj_slot.p, 0, 2 * (size_t)a.ncols * a.ks * sizeof(unsigned long long), st));
    if (!all) CK(cudaMemsetAsync(ctx->adj_bits.p, 0, (size_t)nbuf * K * nevk, st));
    if (!ctx->adj_stream) CK(cudaStreamCreateWithFlags(&ctx->adj_stream, cudaStreamNonBlocking));
    cudaStream_t st2 = ctx->adj_stream;
    StageLam L{ctx->adj_stg.p, ctx->adj_stg.p + ssz, ctx->adj_stg.p + 2 * ssz};
    const float *gin[3] = {dj_duk, dj_dvk, dj_dwk};
    float *stg[3] = {L.u, L.v, L.w};
    for (int q = 0; q < 3; ++q) {
        if (gin[q]) CK(cudaMemcpyAsync(stg[q], gin[q], ssz * sizeof(float), cudaMemcpyHostToDevice, st));
        else CK(cudaMemsetAsync(stg[q], 0, ssz * sizeof(float), st));
    }
    AdjArgs d{};
    for (int q = 0; q < NLAM; ++q) d.lam[q] = ctx->adj_lam.p + (size_t)q * fsz;
    d.ptab = ctx->adj_ptab.p;
    d.slot = ctx->adj_slot.p;
    d.rcr = ctx->adj_rcr.p;
    CK(cudaMemsetAsync(ctx->adj_rcr.p, 0, a.ncols * sizeof(int), st));
    k_adj_readers<<<(a.ncols + 255) / 256, 256, 0, st>>>(a, ctx->adj_rcr.p);
    d.ctr = ctx->adj_ctr.p;
    d.nwe = ctx->adj_nwe;
    const int cb = col_blocks(a);
    k_adj_gather_in<<<cb, 256, 0, st>>>(a, d, L);
    CK(cudaEventRecord(ctx->ev[0], st));
    const int g_p = rev_grid(ctx, ctx->geo_p.g), g_u = rev_grid(ctx, ctx->geo_u.g), g_v = rev_grid(ctx, ctx->geo_v.g);
    int stamp = 0;
    // Segments are reversed from the last one down.  The recomputation of segment sg-1 (restore its
    // checkpoint, run its iterations keeping the states) runs on a second stream into the other
    // keep buffer while segment sg is reversed: the reverse sweeps read only the kept states, the
    // cotangents and the static tables, never the solver's fields, so the two only share the GPU.
    // Events order a buffer's recomputation after the reverse that last read it.
    std::vector<cudaEvent_t> ev(4 * (size_t)nseg, nullptr);   // per segment: recompute start/end, reverse start/end
    for (auto &e : ev) CK(cudaEventCreate(&e));
    auto E = [&](int sg, int q) { return ev[4 * (size_t)sg + q]; };
    auto keep_of = [&](int sg, int q) { return ctx->adj_keep.p + ((size_t)(sg % nbuf) * K + q) * NKEEP * fsz; };
    auto bits_of = [&](int sg, int q) { return ctx->adj_bits.p + ((size_t)(sg % nbuf) * K + q) * nevk; };
    auto recompute = [&](int sg) -> int {
        if (sg + nbuf < nseg) CK(cudaStreamWaitEvent(st2, E(sg + nbuf, 3), 0));   // that buffer's last reader
        CK(cudaEventRecord(E(sg, 0), st2));
        if (!all) {
            CK_RC(restore_checkpoint(ctx, sg, st2));
            const int n = std::min(K, N - sg * K);
            for (int q = 0; q < n; ++q) CK_RC(forward_iteration(ctx, keep_of(sg, q), bits_of(sg, q), st2));
        }
        CK(cudaEventRecord(E(sg, 1), st2));
        return GRAL_OK;
    };
    CK(cudaEventRecord(ctx->ev[2], st));
    CK(cudaStreamWaitEvent(st2, ctx->ev[2], 0));
    CK_RC(recompute(nseg - 1));
    for (int sg = nseg - 1; sg >= 0; --sg) {
        if (sg > 0) CK_RC(recompute(sg - 1));
        const int it0 = sg * K, n = std::min(K, N - it0);   // iterations it0+1 .. it0+n
        CK(cudaStreamWaitEvent(st, E(sg, 1), 0));
        CK(cudaEventRecord(E(sg, 2), st));
        for (int q = n - 1; q >= 0; --q) {
            const float *kp = keep_of(sg, q);
            for (int f = 0; f < 7; ++f) d.mid[f] = kp + f * fsz;
            for (int f = 0; f < 3; ++f) d.end[f] = kp + (7 + f) * fsz;
            d.bits = bits_of(sg, q);
            d.it = it0 + q + 1;
            CK(cudaMemsetAsync(d.ctr, 0, 4 * sizeof(unsigned int), st));
            d.stamp = ++stamp;
            k_adj_mom<2><<<g_p, AW * 32, 0, st>>>(a, d, ctx->geo_p.g);
            d.ctr = ctx->adj_ctr.p + 1;
            d.stamp = ++stamp;
            k_adj_mom<1><<<g_v, AW * 32, 0, st>>>(a, d, ctx->geo_v.g);
            d.ctr = ctx->adj_ctr.p + 2;
            d.stamp = ++stamp;
            k_adj_mom<0><<<g_u, AW * 32, 0, st>>>(a, d, ctx->geo_u.g);
            k_adj_avg_copies<<<cb, 256, 0, st>>>(a, d);
            k_adj_avg_gather<<<cb, 256, 0, st>>>(a, d);
            k_adj_avg_clear<<<cb, 256, 0, st>>>(a, d);
            k_adj_velcorr<<<cb, 256, 0, st>>>(a, d);
            d.ctr = ctx->adj_ctr.p + 3;
            d.stamp = ++stamp;
            k_adj_pressure<<<g_p, AW * 32, 0, st>>>(a, d, ctx->geo_p.g);
            d.ctr = ctx->adj_ctr.p;
            k_adj_div<<<cb, 256, 0, st>>>(a, d);
            k_adj_bc_top_rev<<<(a.ncols + 127) / 128, 128, 0, st>>>(a, d);
            const long long ns = (long long)(a.nii - 1) * a.ks, nw = (long long)(a.njj - 1) * a.ks;
            k_adj_bc_sn_rev<<<(int)((ns + 127) / 128), 128, 0, st>>>(a, ctx->bc, d);
            k_adj_bc_we_rev<<<(int)((nw + 127) / 128), 128, 0, st>>>(a, ctx->bc, d);
        }
        CK(cudaEventRecord(E(sg, 3), st));
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(st));
    CK(cudaStreamSynchronize(st2));
    float ms_re = 0.f, ms_rev = 0.f;
    for (int sg = 0; sg < nseg; ++sg) {
        float m1 = 0.f, m2 = 0.f;
        CK(cudaEventElapsedTime(&m1, E(sg, 0), E(sg, 1)));
        CK(cudaEventElapsedTime(&m2, E(sg, 2), E(sg, 3)));
        ms_re += m1;
        ms_rev += m2;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    {
        int herr = 0;
        CK(cudaMemcpy(&herr, ctx->misc.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr == ERR_TIMEOUT) {
            ctx->adj_ready = false;
            return fail(ctx, GRAL_ETIMEDOUT, "an adjoint wavefront wait exceeded its time limit");
        }
    }
    // the set-up, reversed
    k_adj_setup_scatter<<<cb, 256, 0, st>>>(a, d, L);
    k_adj_setup_zero<<<cb, 256, 0, st>>>(a, d, L);
    const long long nbd = (long long)(a.njj + a.nii) * (a.nkk - 1);
    k_adj_setup_border<<<(int)((nbd + 255) / 256), 256, 0, st>>>(a, L);
    k_adj_setup_avg<<<cb, 256, 0, st>>>(a, d, L);
    CK(cudaGetLastError());
    float *out[3] = {dj_duk0, dj_dvk0, dj_dwk0};
    for (int q = 0; q < 3; ++q)
        if (out[q]) CK(cudaMemcpyAsync(out[q], stg[q], ssz * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (dj_dveg) {
        // reuse the first staging block for the VEG cotangent
        k_adj_veg_out<<<cb, 256, 0, st>>>(a, d, L.u);
        CK(cudaMemcpyAsync(dj_dveg, L.u, ssz * sizeof(float), cudaMemcpyDeviceToHost, st));
    }
    CK(cudaEventRecord(ctx->ev[1], st));
    CK(cudaStreamSynchronize(st));
    float ms_all = 0.f;
    CK(cudaEventElapsedTime(&ms_all, ctx->ev[0], ctx->ev[1]));
    int herr = 0;
    CK(cudaMemcpy(&herr, ctx->misc.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr == ERR_TIMEOUT) return fail(ctx, GRAL_ETIMEDOUT, "an adjoint wavefront wait exceeded its time limit");
    if (stats) {
        stats->iterations = N;
        stats->checkpoint_every = K;
        stats->ms_forward = ctx->adj_ms_forward;
        stats->ms_recompute = ms_re;
        stats->ms_reverse = ms_rev;
        stats->ms_total = ms_all;
    }
    return GRAL_OK;
}

}  // extern "C"
