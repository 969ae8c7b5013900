/*
 * oracle_common.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Shared state and scalar helpers of the CPU oracle for GRAL's prognostic microscale flow
 * solver.  The oracle is a from-scratch C++ restatement of the reference's deterministic path
 * (in.dat UseFixedRndSeedVal=1, ReadInDat.cs:270-287, which serialises every Gauss-Seidel phase,
 * PrognosticFlowfield.cs:806-811, 1060-1065, 1085-1090, 1106-1111, 1129-1135).  Only tests/,
 * the smoke check and the CPU-baseline leg of bench.py may load it; the product never does.
 *
 * Parity status: unpinned.  The reference is C#/.NET 8 and cannot be built or run in this
 * environment, and it ships no tests or golden vectors for this path.  The oracle follows the
 * reference's source operation by operation (float vs double promotion, association order, .NET 8
 * Math.Max/Min and Vector.Max/Min semantics), and is built without floating-point contraction.
 */
#ifndef GRAL_ORACLE_COMMON_H
#define GRAL_ORACLE_COMMON_H

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <type_traits>
#include <vector>
#ifdef ORACLE_THREADS
#include <atomic>
#include <thread>
#endif

#include "gral_prog.h"

namespace oracle {

/* ---- racy-order throughput build ----
 * Built with ORACLE_THREADS (liboracle_mt.so), the outer loops of the sweeps run over host threads
 * the way the reference's default (non-deterministic) mode runs them: momentum and k-eps sweeps
 * over i-slabs of min(max(4, NII/threads), 64) columns handed out dynamically (Parallel.ForEach
 * over Partitioner.Create(3, NII, ...), U-prognostic-microscale_1.cs:59-61), the pressure sweep
 * over rows j (Parallel.For(2, NJJ), PrognosticFlowfield.cs:812), the divergence, velocity
 * correction and averages over i.  Neighbouring slabs then read each other's cells while they are
 * written, so results depend on thread timing as in the reference's default mode: that build is a
 * throughput analogue only, never a parity reference.  Without ORACLE_THREADS, for_chunks calls
 * its body once over the whole range and every loop runs in the deterministic order. */
int worker_threads();
inline int slab_chunk(int n) { return std::min(std::max(4, n / worker_threads()), 64); }
#ifdef ORACLE_THREADS
template <class F> void for_chunks(int lo, int hi, int chunk, F &&body) {
    std::atomic<int> next(lo);
    auto work = [&]() {
        for (;;) {
            const int a = next.fetch_add(chunk);
            if (a >= hi) break;
            body(a, std::min(a + chunk, hi));
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < worker_threads(); ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
}
#else
template <class F> void for_chunks(int lo, int hi, int, F &&body) { body(lo, hi); }
#endif
template <class F> void for_slabs(int lo, int hi, F &&body) { for_chunks(lo, hi, slab_chunk(hi), body); }

/* ---- .NET 8 scalar semantics (ProgramFunctions.cs:768-849 and System.Math) ---- */

/* Math.Max(float, float) / MathF.Max: IEEE 754:2019 maximum (NaN propagates, +0 > -0). */
static inline float net_max(float a, float b) {
    if (a != b) {
        if (!std::isnan(a)) return (b < a) ? a : b;
        return a;
    }
    return std::signbit(b) ? a : b;
}
static inline float net_min(float a, float b) {
    if (a != b) {
        if (!std::isnan(a)) return (a < b) ? a : b;
        return a;
    }
    return std::signbit(a) ? a : b;
}
static inline double net_maxd(double a, double b) {
    if (a != b) {
        if (!std::isnan(a)) return (b < a) ? a : b;
        return a;
    }
    return std::signbit(b) ? a : b;
}
/* Program.FloatMax (ProgramFunctions.cs:768): val1 > val2 ? val1 : val2. */
static inline float float_max(float a, float b) { return (a > b) ? a : b; }
/* Vector.Max / Vector.Min on .NET 8 x64 (maxps / minps): left > right ? left : right.  The double
 * overloads serve the FP64 twin of the model-1 path (the same operations in double). */
static inline float vmax(float a, float b) { return (a > b) ? a : b; }
static inline float vmin(float a, float b) { return (a < b) ? a : b; }
static inline double vmax(double a, double b) { return (a > b) ? a : b; }
static inline double vmin(double a, double b) { return (a < b) ? a : b; }
static inline double vmax(double a, float b) { return vmax(a, (double)b); }
static inline double vmax(float a, double b) { return vmax((double)a, b); }
static inline double vmin(double a, float b) { return vmin(a, (double)b); }
static inline double vmin(float a, double b) { return vmin((double)a, b); }
static inline float osqrt(float x) { return std::sqrt(x); }
static inline double osqrt(double x) { return std::sqrt(x); }
static inline float ofabs(float x) { return std::fabs(x); }
static inline double ofabs(double x) { return std::fabs(x); }
static inline float ofma(float a, float b, float c) { return std::fma(a, b, c); }
template <class A, class B, class C,
          class = typename std::enable_if<std::is_arithmetic<A>::value && std::is_arithmetic<B>::value &&
                                          std::is_arithmetic<C>::value>::type>
static inline double ofma(A a, B b, C c) { return std::fma((double)a, (double)b, (double)c); }

/* Program.ConvToInt(double) (ProgramFunctions.cs:798): round half away from zero through a
 * truncating (int) cast.  An out-of-range or NaN operand converts to int.MinValue, as the x64
 * cvttsd2si conversion of .NET 8 does. */
static inline int conv_to_int(double v) {
    double t = (v < 0) ? (v - 0.5) : (v + 0.5);
    if (!(t > -2147483649.0 && t < 2147483648.0)) return INT_MIN;
    return (int)t;
}

static inline float pow2f(float x) { return x * x; }
static inline double pow2d(double x) { return x * x; }
static inline float pow3f(float x) { return x * x * x; }
static inline float pow5f(float x) { return x * x * x * x * x; }
static inline double pow5d(double x) { return x * x * x * x * x; }

/* ---- solver state: every 3-D array is [NII+2][NJJ+2][NKK+2], k fastest ----
 * T is the type of the flow fields: float for the oracle proper; double for the FP64 twin of the
 * model-1 path and the tape type of its reverse-mode differentiation (oracle/adjoint.cpp), which
 * run the same operations on the same grid constants (float). */
template <class T>
struct StateT {
    int nii, njj, nkk, kadvmax, vcff;
    int ni2, nj2, nk2;
    float dxk, dyk;
    const gral_params *p;
    const gral_static *s;
    T *uk, *vk, *wk;                               /* flow fields */
    float *turb, *tdiss;                           /* k-eps fields (model 2, float only) */
    std::vector<T> uks, vks, wks, dpm, dpmnew, div;
    std::vector<float> turb_own, tdiss_own;        /* used when model == 1 (never read) */
    std::vector<int> vert_index;                   /* Program.VerticalIndex [NII+2][NJJ+2] */
    std::vector<float> ustern_terrain, ustern_obst;/* UsternTerrain/ObstaclesHelpterm */
    std::vector<float> ap0;                        /* PrognosticFlowfield.AP0 */
    const T *veg_t = nullptr;                      /* VEG as T (null: s->veg, float only) */

    size_t i3(int i, int j, int k) const { return ((size_t)i * nj2 + j) * nk2 + k; }
    size_t i2(int i, int j) const { return (size_t)i * nj2 + j; }
    int kkart(int i, int j) const { return s->kkart[i2(i, j)]; }
    int advdom(int i, int j) const { return s->advdom[i2(i, j)]; }
    float cutk(int i, int j) const { return s->cutk[i2(i, j)]; }
    float cov(int i, int j) const { return s->cov ? s->cov[i2(i, j)] : 0.0f; }
    float z0(int i, int j) const { return s->z0[i2(i, j)]; }
    bool has_veg(int i, int j) const { return s->veg && s->veg_mask && s->veg_mask[i2(i, j)]; }
    float *col(float *a, int i, int j) const { return a + i3(i, j, 0); }
    float *col(std::vector<float> &a, int i, int j) { return a.data() + i3(i, j, 0); }
    template <class U, class = typename std::enable_if<!std::is_same<U, float>::value>::type>
    U *col(U *a, int i, int j) const { return a + i3(i, j, 0); }
    template <class U, class = typename std::enable_if<!std::is_same<U, float>::value>::type>
    U *col(std::vector<U> &a, int i, int j) { return a.data() + i3(i, j, 0); }
    const T *vegcol(int i, int j) const {
        if constexpr (std::is_same<T, float>::value) return veg_t ? veg_t + i3(i, j, 0) : s->veg + i3(i, j, 0);
        else return veg_t + i3(i, j, 0);   /* the twin always supplies VEG as T */
    }
    const float *dzk() const { return s->dzk; }
    const float *hokart() const { return s->hokart; }
};
using State = StateT<float>;

/* Momentum routines (one translation unit each model family).  The model-1 routines are
 * instantiated for float (the oracle), double and the tape type (oracle/adjoint.cpp). */
template <class T>
void u_mom_ml(StateT<T> &st, int simd, int IS, int JS, float VISHMIN, float AREAxy, float UG, float relax);
template <class T>
void v_mom_ml(StateT<T> &st, int simd, int IS, int JS, float VISHMIN, float AREAxy, float VG, float relax);
template <class T>
void w_mom_ml(StateT<T> &st, int simd, int IS, int JS, float VISHMIN, float AREAxy, float relax);
void u_mom_ke(State &st, int IS, int JS, float Cmueh, float VISHMIN, float AREAxy, float UG, float relax);
void v_mom_ke(State &st, int IS, int JS, float Cmueh, float VISHMIN, float AREAxy, float VG, float relax);
void w_mom_ke(State &st, int IS, int JS, float Cmueh, float VISHMIN, float AREAxy, float relax);
void tke_ke(State &st, int IS, int JS, float Cmueh, float Ceps, float Ceps1, float Ceps2,
            float VISHMIN, float VISVMIN, float AREAxy, float building_Z0, float relax,
            float Ustern_factorX);
void u_mom_nd(State &st, int IS, int JS, float AREAxy, float UG, float relax);
void v_mom_nd(State &st, int IS, int JS, float AREAxy, float VG, float relax);
void w_mom_nd(State &st, int IS, int JS, float AREAxy, float relax);

}  // namespace oracle

#endif
