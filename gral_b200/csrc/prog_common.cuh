// prog_common.cuh -- device-side data structures and helpers of the B200 prognostic solver.
//
// Device layout (private to the library): every 3-D field of one situation is a slab
// [col][KS] float, col = i*(NJJ+2) + j, k fastest, holding levels 0..KS-1 with
// KS >= KADVMAX+2 (every level the SIMPLE loop reads or writes, PrognosticFlowfield.cs:584-1182).
// Situations of a batch are consecutive slabs.  Per-column constants live in ColMeta/ColF,
// per-situation scalars in SitDev.
//
// Arithmetic follows the reference's float/double evaluation exactly: the library is built with
// --fmad=false (no contraction, like .NET RyuJIT), IEEE division and square root, and the
// max/min helpers below reproduce .NET 8 semantics.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gral {

constexpr int KMAX_LEVELS = 64;   // largest KS the column kernels handle (two rounds of 32 lanes)
constexpr int MAX_HIST = 64;

// ---- per-column flag bits (ColMeta::flags) ----
enum : uint32_t {
    F_ADV = 1u << 0,      // ADVDOM[i][j] == 1
    F_ALLOC3 = 1u << 1,   // ADVDOM set in the 3x3 neighbourhood (staggered arrays exist), :64-86
    F_VEG = 1u << 2,      // VEG[i][j] != null
    F_CUTK0 = 1u << 3,    // CUTK == 0   (KSTART = KKART+1)
    F_CUTKLT1 = 1u << 4,  // CUTK < 1    (terrain wall law instead of building law)
    F_CUTKGT0 = 1u << 5,  // CUTK > 0
    F_VC = 1u << 6,       // ADVDOM(i,j) | ADVDOM(i-1,j) | ADVDOM(i,j-1): velocity correction, :965
    F_BS = 1u << 7,       // ADVDOM[i][j-1] < 1 || j == 2     (diffusion boundary, U-...1.cs:145-148)
    F_BN = 1u << 8,       // ADVDOM[i][j+1] < 1 || j == NJJ-1
    F_BW = 1u << 9,       // ADVDOM[i-1][j] < 1 || i == 2
    F_BE = 1u << 10,      // ADVDOM[i+1][j] < 1 || i == NII-1
    F_Z0GE = 1u << 11,    // Z0 >= DZK[KKART+1]*0.1F (float test of the model-1 wall law)
    F_Z0GED = 1u << 12,   // Z0 >= DZK[KKART+1]*0.1 (double test of the model-0/2 wall law)
};

struct ColMeta {          // 16 bytes
    int16_t kkart, vi, kstart, kad;   // KKART, VerticalIndex, KSTART, first level with ADD_DIFF
    int16_t wc_lo, wc_hi;             // levels whose SIMD chunk holds KKART+1 (wall chunk)
    int16_t kkm_u, kkm_v;             // max(KKART, KKART[i-1][j]), max(KKART, KKART[i][j-1])
};

struct ColF {             // 16 bytes
    float cov, z0, help_t, help_o;    // COV, roughness, UsternTerrain/ObstaclesHelpterm
};

// k-eps wall functions of the TKE back-substitution (TKE-prognostic-microscale.cs:272-343):
// gfac = 0.4/ln(z/Z0) of the ground law in double (gmode 1: z = DZK[k]+DZK[k+1]/2, 0: DZK[k]/2);
// kw_e/w/n/s = KKART+1 of the east/west/north/south neighbour when it is a building, else -1.
struct ColKE {            // 16 bytes
    double gfac;
    int16_t kw_e, kw_w, kw_n, kw_s;
};

// Per-situation scalars and convergence state (PrognosticFlowfield.cs:146-163, 231-240, 1144-1170).
struct SitDev {
    double frund;
    double rfrund;           // 1/Frund correctly rounded (host), for rcp_ok
    double delta_mean;
    double conv_threshold;
    double hist[MAX_HIST];
    unsigned long long geschw_bits;   // GESCHW_MAX as non-negative double bits (atomicMax)
    float dtime, topwind, ug, vg;
    float potdtdz;           // Program.PotdTdz of the situation (k-eps buoyancy)
    float std_dev_v, v0_1;   // TURB initialisation (PrognosticFlowfield.cs:477-486)
    int32_t turb_init;       // 0: initialise TURB/TDISS as the reference, 1: keep the caller's
    float delta_first, delta_finish, last_dumax;
    uint32_t dumax_bits;     // running max of the residual keys of this iteration (see residual_key)
    int32_t it;              // IterationLoops
    int32_t active;          // 1 while the SIMPLE loop runs for this situation
    int32_t iters_done;
    int32_t converged;
    int32_t n_hist;
    int32_t it_min, it_max, cadence;
    int32_t quantise;
    int32_t rcp_ok;          // ConvToInt(x*Frund)/Frund by the reciprocal (verified at the load)
};

// Everything a kernel needs, passed by value (all pointers are device pointers).
struct KArgs {
    // geometry
    int nii, njj, nkk, ks, nj2, ncols, nb;
    int il;                              // 1: interleaved layout (batched family), 0: slab layout
    int ngroups;                         // groups of 32 situations (interleaved layout)
    int variant;                         // launch variant of the batched wavefront kernels
    int group_lo, group_n;               // groups swept by one wavefront launch (batched family)
    int ctr_slot;                        // task-counter slot of the launch
    int group_set;                       // groups per wavefront launch (0 = all)
    float dxk, dyk, areaxy;
    float relax, relaxp, coriolis, vishmin;
    int simd;
    // static tables (device)
    const ColMeta *meta;
    const uint32_t *cflags;              // F_* bits per column
    const ColF *colf;
    const ColKE *colke;                  // per column, model 2 only (else null)
    float ustern_fx, building_z0;        // Ustern_factorX, building roughness (k-eps wall laws)
    int model;                           // TurbulenceModel 0, 1, 2
    const float *dzk, *hokart;           // [ks]
    const float *app, *abp, *atp;        // pressure coefficients per level [ks]
    const float *veg;                    // [ncols][ks] or null
    // per-situation state
    SitDev *sit;                         // [nb]
    const float *ap0;                    // [nb][ks]
    // fields [nb][ncols][ks]
    float *uk, *vk, *wk, *dpm, *dpmnew, *uks, *vks, *wks, *turb, *tdiss;
    // scheduling
    int *flags;                          // [nb][ncols] stamps
    unsigned int *counters;              // task counters, one per GS phase kind
    float *rowcarry;                     // [nb][nj2][2][ks] pressure row carry (P, Q)
    const short2 *rcw;                   // per column: i of the last column before it in its sweep row
                                         // that writes the row carry at VerticalIndex+1 (x: IS=+1,
                                         // y: IS=-1), -1 if none
    int *err;                            // device error word (0 = ok)
    const int *act;                      // active situation list (slab layout)
    const int *nact;                     // number of active situations
    int *it_global;                      // IterationLoops of the batch (all situations in lockstep)
    unsigned long long wait_limit_ns;    // bound of every spin wait
    int chunk;                           // tasks claimed per atomic
    float *trace;                        // [nb][trace_cap] DeltaUMax per iteration, or null
    int trace_cap;
    int vi_min;                          // smallest VerticalIndex of an active column
    int diag_iter;                       // iteration (1..10) of a DiagnosticFlowfield sweep launch
};

// Geometry of a Gauss-Seidel sweep: sweep coordinates i1 in [ia, ia+ni), j1 in [ja, ja+nj);
// tasks are numbered diagonal by diagonal (d = (i1-ia) + (j1-ja)), then situation, then position.
struct SweepGeom {
    int ia, ni, ja, nj, ndiag;
    const int *diag_start;   // [ndiag+1] cells on diagonals < d (device)
};

// Task list of the fused pressure -> velocity correction -> averages -> U wavefront (slab family,
// model 1): steps of segments (kind, diagonal); segment q holds seg_start[q+1]-seg_start[q] tasks,
// its code = kind | diagonal << 3.  Pressure, velocity correction and averages use geometry gp
// (the pressure sweep range), U uses gu.
struct FusedGeom {
    const int *seg_start;     // [nseg+1]
    const int *seg_code;      // [nseg]
    int nseg;
    SweepGeom gp, gu;
};

enum : int { ERR_NONE = 0, ERR_TIMEOUT = 1, ERR_NONFINITE = 2 };

// Gauss-Seidel task kinds.  A column's flag carries stamp = IterationLoops*8 + kind; within an
// iteration a column completes its kinds in increasing order (pressure, velocity correction,
// averages, U, V, W, TKE), so one monotonic flag per column serves every kind.  The value also
// indexes the task counters.  The diagnostic sweep has flags of its own.
enum : int { PH_DIAG = 0, PH_PRESSURE = 1, PH_VC = 2, PH_AV = 3, PH_U = 4, PH_V = 5, PH_W = 6, PH_TKE = 7 };
enum : int { F_GMODE1 = 1 << 13 };   // ColKE ground law uses level k+1 (Z0 >= DZK/2)

__host__ __device__ inline size_t fidx(int s, int col, int ncols, int ks) {
    return ((size_t)s * ncols + col) * ks;
}

// ---- .NET 8 semantics ----
// Vector.Max / Vector.Min / Program.FloatMax: left > right ? left : right.
__device__ __forceinline__ float vmaxf(float a, float b) { return (a > b) ? a : b; }
__device__ __forceinline__ float vminf(float a, float b) { return (a < b) ? a : b; }
// Math.Max(float,float) / Math.Min (IEEE 754:2019 maximum/minimum).
__device__ __forceinline__ float net_maxf(float a, float b) {
    if (a != b) { if (!isnan(a)) return (b < a) ? a : b; return a; }
    return signbit(b) ? a : b;
}
__device__ __forceinline__ float net_minf(float a, float b) {
    if (a != b) { if (!isnan(a)) return (a < b) ? a : b; return a; }
    return signbit(a) ? a : b;
}
__device__ __forceinline__ double net_maxd(double a, double b) {
    if (a != b) { if (!isnan(a)) return (b < a) ? a : b; return a; }
    return signbit(b) ? a : b;
}
// Program.ConvToInt(double): round half away from zero through a truncating cast; out of
// range or NaN gives int.MinValue as .NET 8 on x64.
__device__ __forceinline__ int conv_to_int(double v) {
    double t = (v < 0) ? (v - 0.5) : (v + 0.5);
    if (!(t > -2147483649.0 && t < 2147483648.0)) return INT32_MIN;
    return (int)t;
}
__device__ __forceinline__ double quantd(double x, double frund, int on) {
    return on ? (double)conv_to_int(x * frund) / frund : x;
}
// The same with the division n/Frund (n = ConvToInt(x*Frund), an integer) done as Markstein's
// correction step on the precomputed y = RN(1/Frund): q0 = RN(n*y), r = n - q0*Frund (exact by
// FMA), q = RN(q0 + r*y).  rok says that the load-time check (k_rcp_check) found q equal to the
// IEEE quotient n/Frund for every integer n of magnitude up to 2^31 with this Frund; without it
// the IEEE division is used.
__device__ __forceinline__ double quantd_r(double x, double frund, double rfrund, bool rok, int on) {
    if (!on) return x;
    const double n = (double)conv_to_int(x * frund);
    if (rok) {
        const double q0 = n * rfrund;
        return fma(fma(-q0, frund, n), rfrund, q0);
    }
    return n / frund;
}

// ---- inter-warp ordering of the Gauss-Seidel wavefront ----
__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Spin (lane 0 only) until *flag >= stamp.  The first polls follow each other directly (the
// predecessor is usually about to publish), later ones back off with __nanosleep up to 32 ns
// (a longer back-off delayed the wake-up on the single-situation wavefront's critical path).
// Gives up after limit_ns, or as soon as another warp reported an error; returns false then.
// Never waits unboundedly.
__device__ inline bool wait_stamp(const int *flag, int stamp, int *err, unsigned long long limit_ns) {
    if (ld_acquire(flag) >= stamp) return true;
    const unsigned long long t0 = globaltimer_ns();
    unsigned ns = 16;
    for (unsigned n = 1;; ++n) {
        if (n > 4) {
            __nanosleep(ns);
            if (ns < 32) ns += ns;
        }
        if (ld_acquire(flag) >= stamp) return true;
        if ((n & 7) == 0) {
            if (*(volatile int *)err != ERR_NONE) return false;
            if (globaltimer_ns() - t0 > limit_ns) {
                atomicCAS(err, ERR_NONE, ERR_TIMEOUT);
                return false;
            }
        }
    }
}

__device__ __forceinline__ int ld_relaxed(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// 8-byte words of a value and a stamp: float bits in the low half, the stamp in the high half.
// One aligned 8-byte access is single-copy atomic, so a word that shows the stamp carries its
// value, with no flag, release or fence between the writer's store and the reader's use.
__device__ __forceinline__ unsigned long long ld_word(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_word(unsigned long long *p, float v, int stamp) {
    const unsigned long long w = ((unsigned long long)(unsigned)stamp << 32) | __float_as_uint(v);
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}

// Spin (one thread) until both predecessor flags hold at least `stamp` (a null flag has no
// predecessor).  The two flags are polled with relaxed loads, so their round trips overlap, and
// one fence.acquire follows: a strong read followed by an acquire fence is an acquire pattern, so
// it synchronises with the predecessors' st.release as an acquiring load would.  Same bounds as
// wait_stamp: gives up after limit_ns or on another warp's error and returns false then.
// max_sleep_ns caps the back-off between polls (0: poll without sleeping).
__device__ inline bool wait_stamps(const int *f1, const int *f2, int stamp, int *err, unsigned long long limit_ns,
                                   unsigned max_sleep_ns = 32) {
    int v1 = f1 ? ld_relaxed(f1) : stamp;
    int v2 = f2 ? ld_relaxed(f2) : stamp;
    if (v1 < stamp || v2 < stamp) {
        const unsigned long long t0 = globaltimer_ns();
        unsigned ns = 16;
        for (unsigned n = 1;; ++n) {
            if (n > 4 && max_sleep_ns) {
                __nanosleep(ns);
                if (ns < max_sleep_ns) ns += ns;
            }
            if (v1 < stamp) v1 = ld_relaxed(f1);
            if (v2 < stamp) v2 = ld_relaxed(f2);
            if (v1 >= stamp && v2 >= stamp) break;
            if ((n & 7) == 0) {
                if (*(volatile int *)err != ERR_NONE) return false;
                if (globaltimer_ns() - t0 > limit_ns) {
                    atomicCAS(err, ERR_NONE, ERR_TIMEOUT);
                    return false;
                }
            }
        }
    }
    asm volatile("fence.acquire.gpu;" ::: "memory");
    return true;
}

// Full-height level tables of the diagnostic pressure solve (DiagnosticFlowfield.cs:124-138):
// APP, ATP, ABP with KKART < k-1 (abp1) and at KKART+1 (abp0), DZK; and the per-situation DTIME.
struct DiagTabs {
    const float *dzk, *app, *atp, *abp0, *abp1;
    const float *dtime;
};

}  // namespace gral
