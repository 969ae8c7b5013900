/*
 * oracle.cpp -- TEST INFRASTRUCTURE ONLY (CPU oracle, see oracle_common.h).
 *
 * Restates PrognosticFlowfield.Calculate() (PrognosticFlowfield.cs:32-1245) in its deterministic
 * form: set-up (:45-579), the SIMPLE iteration loop (:583-1182) and the post-checks
 * (:1187-1245).  Exported as oracle_solve() with the same argument structs as the product's
 * gral_prog_solve(), so tests feed both the same inputs.
 */
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "oracle_ad.h"
#include "oracle_common.h"

using namespace oracle;

/* Host threads of the racy-order build: ORACLE_THREADS in the environment, else every hardware
 * thread; 1 in the deterministic build. */
extern "C" int oracle_threads(void) { return oracle::worker_threads(); }

int oracle::worker_threads() {
#ifdef ORACLE_THREADS
    static const int n = [] {
        const char *e = std::getenv("ORACLE_THREADS");
        const int v = e ? std::atoi(e) : 0;
        return v > 0 ? v : std::max(1, (int)std::thread::hardware_concurrency());
    }();
    return n;
#else
    return 1;
#endif
}

namespace {

int validate(const gral_params *p, const gral_static *s, const gral_fields *f) {
    if (!p || !s || !f || !f->uk || !f->vk || !f->wk) return GRAL_EINVAL;
    if (p->nii < 4 || p->njj < 4 || p->nkk < 3) return GRAL_EINVAL;
    if (!s->kkart || !s->advdom || !s->cutk || !s->z0 || !s->dzk || !s->hokart) return GRAL_EINVAL;
    if (p->turbulence_model < 0 || p->turbulence_model > 2) return GRAL_EINVAL;
    if (p->turbulence_model == 1 && p->simd_width != 8 && p->simd_width != 16) return GRAL_EINVAL;
    if (p->turbulence_model != 1 && (!f->turb || !f->tdiss)) return GRAL_EINVAL;
    if (p->turbulence_model != 1 && p->turb_init == 0 &&
        (!s->z0_init || !s->ob_init || !s->ust_init)) return GRAL_EINVAL;
    if (p->conv_cadence < 1) return GRAL_EINVAL;
    return GRAL_OK;
}

/* Lateral boundary conditions at the west/east and south/north borders of the prognostic
 * sub-domains (PrognosticFlowfield.cs:595-696) and at the top (:699-714). */
template <class T>
void boundary_conditions(StateT<T> &st) {
    const int NII = st.nii, NJJ = st.njj;
    for (int j = 2; j < NJJ + 1; ++j) {
        for (int i = 3; i < NII; ++i) {
            if (st.advdom(i, j) != 1) continue;
            const int VI = st.vert_index[st.i2(i, j)];
            const bool iM = (st.advdom(i - 1, j) < 1) || (i == 3);
            const bool iP = (st.advdom(i + 1, j) < 1) || (i == NII - 1);
            if (iM) {
                for (int k = 1; k <= VI; ++k) {
                    T u = st.uk[st.i3(i - 2, j, k)];
                    if (u >= 0) st.uk[st.i3(i - 1, j, k)] = u;
                    st.vk[st.i3(i - 2, j, k)] = st.vk[st.i3(i - 1, j, k)];
                    st.wk[st.i3(i - 2, j, k)] = st.wk[st.i3(i - 1, j, k)];
                }
            }
            if (iP) {
                for (int k = 1; k <= VI; ++k) {
                    T u = st.uk[st.i3(i + 2, j, k)];
                    if (u <= 0) st.uk[st.i3(i + 1, j, k)] = u;
                    st.vk[st.i3(i + 1, j, k)] = st.vk[st.i3(i, j, k)];
                    st.wk[st.i3(i + 1, j, k)] = st.wk[st.i3(i, j, k)];
                }
            }
        }
    }
    for (int i = 2; i < NII + 1; ++i) {
        for (int j = 3; j <= NJJ - 1; ++j) {
            if (st.advdom(i, j) != 1) continue;
            const int VI = st.vert_index[st.i2(i, j)];
            const bool jM = (st.advdom(i, j - 1) < 1) || (j == 3);
            const bool jP = (st.advdom(i, j + 1) < 1) || (j == NJJ - 1);
            if (jM) {
                for (int k = 1; k <= VI; ++k) {
                    T v = st.vk[st.i3(i, j - 2, k)];
                    if (v >= 0) st.vk[st.i3(i, j - 1, k)] = v;
                    st.uk[st.i3(i, j - 2, k)] = st.uk[st.i3(i, j - 1, k)];
                    st.wk[st.i3(i, j - 2, k)] = st.wk[st.i3(i, j - 1, k)];
                }
            }
            if (jP) {
                for (int k = 1; k <= VI; ++k) {
                    T v = st.vk[st.i3(i, j + 2, k)];
                    if (v <= 0) st.vk[st.i3(i, j + 1, k)] = v;
                    st.uk[st.i3(i, j + 1, k)] = st.uk[st.i3(i, j, k)];
                    st.wk[st.i3(i, j + 1, k)] = st.wk[st.i3(i, j, k)];
                }
            }
        }
    }
    for (int i = 2; i < NII; ++i) {
        for (int j = 2; j <= NJJ - 1; ++j) {
            if (st.advdom(i, j) != 1) continue;
            const int k = st.vert_index[st.i2(i, j)];
            st.wk[st.i3(i, j, k + 1)] = st.wk[st.i3(i, j, k)];
            st.uk[st.i3(i, j, k + 1)] = st.uk[st.i3(i, j, k)];
            st.vk[st.i3(i, j, k + 1)] = st.vk[st.i3(i, j, k)];
        }
    }
}

/* Round to multiples of 1/Frund in double (PrognosticFlowfield.cs:880, 930-940). */
inline double quant(double x, double Frund, bool on) {
    if (!on) return x;
    return conv_to_int(x * Frund) / Frund;
}

/* Per-solve scalars of the SIMPLE loop, fixed by the set-up (PrognosticFlowfield.cs:146-579). */
struct LoopConsts {
    const gral_params *p;
    float DTIME, AREAxy, UG, VG, relax, relaxp, VISHMIN, VISVMIN, building_Z0, Ustern_factorX;
    float Cmueh, Ceps, Ceps1, Ceps2;
    double Frund;
    bool quantise;
    int model;
};

inline double val(float x) { return (double)x; }
inline double val(double x) { return x; }
inline double val(const AD &x) { return x.v; }
inline double val(const Dual &x) { return x.v; }

/* the velocity-correction rounding of the float oracle; the FP64 twin runs without rounding */
template <class T>
inline T vquant(T x, double Frund, bool on) {
    if constexpr (std::is_same<T, float>::value) return (float)quant((double)x, Frund, on);
    else return x;
}

/* One SIMPLE iteration (PrognosticFlowfield.cs:584-1137): boundary conditions, divergence, the
 * pressure-correction sweep, velocity correction, staggered averages and the momentum sweeps.
 * Returns DeltaUMax of the iteration. */
template <class T>
float simple_iteration(StateT<T> &st, const LoopConsts &c, int IterationLoops) {
    const int NII = st.nii, NJJ = st.njj, NKK = st.nkk;
    const float DXK = st.dxk, DYK = st.dyk;
    const float *DZK = st.s->dzk;
    const gral_params *p = c.p;
    const float DTIME = c.DTIME, AREAxy = c.AREAxy, UG = c.UG, VG = c.VG, relax = c.relax, relaxp = c.relaxp;
    const float VISHMIN = c.VISHMIN, VISVMIN = c.VISVMIN, building_Z0 = c.building_Z0;
    const float Ustern_factorX = c.Ustern_factorX;
    const float Cmueh = c.Cmueh, Ceps = c.Ceps, Ceps1 = c.Ceps1, Ceps2 = c.Ceps2;
    const double Frund = c.Frund;
    const bool quantise = c.quantise;
    const int model = c.model;
    (void)NKK; (void)VISVMIN; (void)building_Z0; (void)Ustern_factorX; (void)Cmueh; (void)Ceps; (void)Ceps1;
    (void)Ceps2; (void)model;
    float DeltaUMax = 0;
    std::mutex delta_mutex;   /* row maxima of the racy-order build's pressure workers */
        boundary_conditions(st);

        /* mass divergence; DPM = 0 on the prognostic levels (:723-758) */
        for_chunks(2, NII, slab_chunk(NII), [&](int i_lo, int i_hi) {
        for (int i = i_lo; i < i_hi; ++i) {
            for (int j = 2; j < NJJ; ++j) {
                if (st.advdom(i, j) != 1) continue;
                const int KK = st.kkart(i, j), VI = st.vert_index[st.i2(i, j)];
                const T *UK_L = st.col(st.uk, i, j), *VK_L = st.col(st.vk, i, j), *WK_L = st.col(st.wk, i, j);
                const T *UKip = st.col(st.uk, i + 1, j), *VKjp = st.col(st.vk, i, j + 1);
                T *DIV_L = st.col(st.div, i, j), *DPM_L = st.col(st.dpm, i, j);
                for (int k = KK + 1; k <= VI; ++k) {
                    if (k > KK + 1)
                        DIV_L[k] = (UK_L[k] - UKip[k]) * DYK * DZK[k] + (VK_L[k] - VKjp[k]) * DXK * DZK[k] +
                                   (WK_L[k] - WK_L[k + 1]) * AREAxy;
                    else
                        DIV_L[k] = (UK_L[k] - UKip[k]) * DYK * DZK[k] + (VK_L[k] - VKjp[k]) * DXK * DZK[k] -
                                   WK_L[k + 1] * AREAxy;
                    DPM_L[k] = 0;
                }
            }
        }
        });

        /* sweep direction (:770-802) */
        int IS = 1, JS = 1;
        if (IterationLoops % 4 == 0) { IS = -1; JS = 1; }
        else if (IterationLoops % 4 == 1) { IS = -1; JS = -1; }
        else if (IterationLoops % 4 == 2) { IS = 1; JS = -1; }

        /* pressure correction, vertical TDMA per column, rows in order (:804-901) */
        for_chunks(2, NJJ, 1, [&](int j1_lo, int j1_hi) {
            std::vector<T> PIMP(st.nk2), QIMP(st.nk2);
            float DeltaUMaxRows = 0;
            for (int j1 = j1_lo; j1 < j1_hi; ++j1) {
                std::fill(PIMP.begin(), PIMP.end(), 0.0f);   /* new float[NKK + 2] per row */
                std::fill(QIMP.begin(), QIMP.end(), 0.0f);
                float DeltaUMaxIntern = 0;
                const int j = (JS == -1) ? NJJ - j1 + 1 : j1;
                for (int i1 = 2; i1 <= NII - 1; ++i1) {
                    const int i = (IS == -1) ? NII - i1 + 1 : i1;
                    if (st.advdom(i, j) != 1) continue;
                    const T *DIV_L = st.col(st.div, i, j);
                    T *DPM_L = st.col(st.dpm, i, j);
                    const T *DPMim = st.col(st.dpm, i - 1, j), *DPMip = st.col(st.dpm, i + 1, j);
                    const T *DPMjm = st.col(st.dpm, i, j - 1), *DPMjp = st.col(st.dpm, i, j + 1);
                    T *DPMNEW_L = st.col(st.dpmnew, i, j);
                    const int KK = st.kkart(i, j), VI = st.vert_index[st.i2(i, j)];
                    for (int k = VI; k > KK; --k) {
                        T DIM = DIV_L[k] / DTIME + (DPMim[k] + DPMip[k]) / DXK * DYK * DZK[k] +
                                    (DPMjm[k] - DPMjp[k]) / DYK * DXK * DZK[k];
                        T APP = 2.0f * (DYK * DZK[k] / DXK + DXK * DZK[k] / DYK + AREAxy / DZK[k]);
                        T ABP = (k > 1) ? AREAxy / (0.5f * (DZK[k - 1] + DZK[k])) : AREAxy / DZK[k];
                        T ATP = AREAxy / (0.5f * (DZK[k + 1] + DZK[k]));
                        T TERMP = 1 / (APP - ATP * PIMP[k + 1]);
                        PIMP[k] = ABP * TERMP;
                        QIMP[k] = (ATP * QIMP[k + 1] + DIM) * TERMP;
                    }
                    for (int k = KK + 1; k <= VI; ++k) {
                        T temp = PIMP[k] * DPM_L[k - 1] + QIMP[k];
                        DeltaUMaxIntern = (float)net_maxd((double)DeltaUMaxIntern,
                            std::fabs(val(DPM_L[k]) - quant(val(temp), Frund, quantise)));
                        DPM_L[k] = temp;
                        DPMNEW_L[k] += relaxp * DPM_L[k];
                    }
                }
                if (DeltaUMaxIntern > DeltaUMaxRows) DeltaUMaxRows = DeltaUMaxIntern;
            }
            std::lock_guard<std::mutex> lk(delta_mutex);
            if (DeltaUMaxRows > DeltaUMax) DeltaUMax = DeltaUMaxRows;
        });

        /* velocity correction with Frund quantisation in double (:904-949) */
        for_chunks(2, NII, slab_chunk(NII), [&](int i_lo, int i_hi) {
        for (int i = i_lo; i < i_hi; ++i) {
            for (int j = 2; j <= NJJ - 1; ++j) {
                if (!(st.advdom(i, j) == 1 || st.advdom(i - 1, j) == 1 || st.advdom(i, j - 1) == 1)) continue;
                const T *DPMim = st.col(st.dpm, i - 1, j), *DPMjm = st.col(st.dpm, i, j - 1);
                const T *DPM_L = st.col(st.dpm, i, j);
                T *UK_L = st.col(st.uk, i, j), *VK_L = st.col(st.vk, i, j), *WK_L = st.col(st.wk, i, j);
                const int KK = st.kkart(i, j), VI = st.vert_index[st.i2(i, j)];
                const int KKim = st.kkart(i - 1, j), KKjm = st.kkart(i, j - 1);
                for (int k = 1; k <= VI; ++k) {
                    const T d = DPM_L[k];
                    if (i > 2 && KK < k && KKim < k)
                        UK_L[k] = vquant<T>(UK_L[k] + (DPMim[k] - d) / DXK * DTIME, Frund, quantise);
                    if (j > 2 && KK < k && KKjm < k)
                        VK_L[k] = vquant<T>(VK_L[k] + (DPMjm[k] - d) / DYK * DTIME, Frund, quantise);
                    if (KK + 1 < k)
                        WK_L[k] = vquant<T>(WK_L[k] + (DPM_L[k - 1] - d) / (DZK[k] + DZK[k - 1]) * 2 * DTIME,
                                            Frund, quantise);
                    else
                        WK_L[k] = 0;
                }
            }
        }
        });

        /* staggered -> cell-centre averages and border copies (:958-1039) */
        for_chunks(2, NII, slab_chunk(NII), [&](int i_lo, int i_hi) {
        for (int i = i_lo; i < i_hi; ++i) {
            for (int j = 2; j <= NJJ - 1; ++j) {
                if (!(st.advdom(i, j) == 1 || st.advdom(i - 1, j) == 1 || st.advdom(i, j - 1) == 1)) continue;
                const T *UK_L = st.col(st.uk, i, j), *UKip = st.col(st.uk, i + 1, j);
                const T *VK_L = st.col(st.vk, i, j), *VKjp = st.col(st.vk, i, j + 1);
                const T *WK_L = st.col(st.wk, i, j);
                T *UKS_L = st.col(st.uks, i, j), *VKS_L = st.col(st.vks, i, j), *WKS_L = st.col(st.wks, i, j);
                const int KK = st.kkart(i, j), VI = st.vert_index[st.i2(i, j)];
                int KSTART = 1;
                if (st.cutk(i, j) == 0) KSTART = KK + 1;
                for (int k = KSTART; k <= VI; ++k) {
                    if (KK < k) {
                        UKS_L[k] = 0.5f * (UK_L[k] + UKip[k]);
                        VKS_L[k] = 0.5f * (VK_L[k] + VKjp[k]);
                    }
                    if (KK + 1 < k) WKS_L[k] = 0.5f * (WK_L[k] + WK_L[k + 1]);
                }
                if (j == 2) {
                    T *UKS1 = st.col(st.uks, i, 1);
                    for (int k = KSTART; k <= VI; ++k) UKS1[k] = UKS_L[k];
                }
                if (j == NJJ - 1 && st.advdom(i, NJJ) == 1) {
                    T *UKSN = st.col(st.uks, i, NJJ);
                    for (int k = KSTART; k <= VI; ++k) UKSN[k] = UKS_L[k];
                }
            }
        }
        });
        for (int j = 2; j < NJJ; ++j) {
            if (st.advdom(1, j) == 1) {
                T *a = st.col(st.vks, 1, j); const T *b = st.col(st.vks, 2, j);
                for (int k = 0; k <= NKK; ++k) a[k] = b[k];
            }
            if (st.advdom(NII - 1, j) == 1) {
                T *a = st.col(st.vks, NII, j); const T *b = st.col(st.vks, NII - 1, j);
                for (int k = 0; k <= NKK; ++k) a[k] = b[k];
            }
        }

        /* momentum equations (:1049-1137), deterministic order; the FP64 twin and the tape type run
         * model 1 only */
        if constexpr (!std::is_same<T, float>::value) {
            u_mom_ml(st, p->simd_width, IS, JS, VISHMIN, AREAxy, UG, relax);
            v_mom_ml(st, p->simd_width, -IS, -JS, VISHMIN, AREAxy, VG, relax);
            w_mom_ml(st, p->simd_width, IS, JS, VISHMIN, AREAxy, relax);
        } else if (model == 0) {
            u_mom_nd(st, IS, JS, AREAxy, UG, relax);
            v_mom_nd(st, IS, JS, AREAxy, VG, relax);
            w_mom_nd(st, IS, JS, AREAxy, relax);
        } else if (model == 1) {
            u_mom_ml(st, p->simd_width, IS, JS, VISHMIN, AREAxy, UG, relax);
            v_mom_ml(st, p->simd_width, -IS, -JS, VISHMIN, AREAxy, VG, relax);
            w_mom_ml(st, p->simd_width, IS, JS, VISHMIN, AREAxy, relax);
        } else {
            u_mom_ke(st, IS, JS, Cmueh, VISHMIN, AREAxy, UG, relax);
            v_mom_ke(st, IS, JS, Cmueh, VISHMIN, AREAxy, VG, relax);
            w_mom_ke(st, IS, JS, Cmueh, VISHMIN, AREAxy, relax);
            tke_ke(st, IS, JS, Cmueh, Ceps, Ceps1, Ceps2, VISHMIN, VISVMIN, AREAxy, building_Z0, relax,
                   Ustern_factorX);
        }
    return DeltaUMax;
}

}  // namespace

/* DiagnosticFlowfield.Calculate after a prognostic solve (DiagnosticFlowfield.cs:24-436), in the
 * deterministic order (UseFixedRndSeedVal: one worker, rows j outer, columns i inner), then the
 * final vertical velocity of the columns outside the prognostic sub-domains
 * (MicroscaleFlat.cs:389-462, FlowFieldLevel = prognostic). */
static void diagnostic_post(State &st) {
    const int NII = st.nii, NJJ = st.njj, NKK = st.nkk;
    const float DXK = st.dxk, DYK = st.dyk;
    const float *DZK = st.dzk();
    const float u11 = st.uk[st.i3(1, 1, st.kadvmax)], v11 = st.vk[st.i3(1, 1, st.kadvmax)];
    float DTIME = (float)(0.5 * (double)net_min(DXK, DYK) / std::sqrt((double)(pow2f(u11) + pow2f(v11))));
    DTIME = net_min(DTIME, 5.0f);
    const int Iterations = 10;
    for (int i = 1; i <= NII; ++i)                                   /* :39-49 */
        for (int j = 1; j <= NJJ; ++j)
            for (int k = 1; k <= NKK + 1; ++k) st.dpm[st.i3(i, j, k)] = 0;
    std::vector<float> PIMP(st.nk2 + 1, 0.0f), QIMP(st.nk2 + 1, 0.0f);
    for (int IterationLoops = 1; IterationLoops <= Iterations; ++IterationLoops) {
        for (int i = 2; i < NII; ++i)                                /* divergence, :54-81 */
            for (int j = 2; j < NJJ; ++j) {
                const int KK = st.kkart(i, j);
                for (int k = 1; k <= NKK - 1; ++k) {
                    if (!(KK < k)) continue;
                    const float u0 = st.uk[st.i3(i, j, k)], uE = st.uk[st.i3(i + 1, j, k)];
                    const float v0 = st.vk[st.i3(i, j, k)], vN = st.vk[st.i3(i, j + 1, k)];
                    if (k > KK + 1)
                        st.div[st.i3(i, j, k)] = (u0 - uE) * DYK * DZK[k] + (v0 - vN) * DXK * DZK[k] +
                                                 (st.wk[st.i3(i, j, k)] - st.wk[st.i3(i, j, k + 1)]) * DXK * DYK;
                    else
                        st.div[st.i3(i, j, k)] = (u0 - uE) * DYK * DZK[k] + (v0 - vN) * DXK * DZK[k] -
                                                 st.wk[st.i3(i, j, k + 1)] * DXK * DYK;
                }
            }
        /* pressure-correction TDMA, :86-315; the four sweep orders of IterationLoops % 4 */
        const int m = IterationLoops % 4;
        const bool jdesc = (m == 1 || m == 2), idesc = (m == 2 || m == 3);
        for (int j1 = 2; j1 < NJJ; ++j1) {
            const int j = jdesc ? NJJ - j1 + 1 : j1;
            for (int i1 = 2; i1 < NII; ++i1) {
                const int i = idesc ? NII - i1 + 1 : i1;
                const int KK = st.kkart(i, j);
                for (int k = NKK - 1; k >= 1; k--) {
                    if (!(KK < k)) continue;
                    const float DIM = st.div[st.i3(i, j, k)] / DTIME +
                                      (st.dpm[st.i3(i - 1, j, k)] + st.dpm[st.i3(i + 1, j, k)]) / DXK * DYK * DZK[k] +
                                      (st.dpm[st.i3(i, j - 1, k)] - st.dpm[st.i3(i, j + 1, k)]) / DYK * DXK * DZK[k];
                    const float APP = 2 * (DYK * DZK[k] / DXK + DXK * DZK[k] / DYK + DXK * DYK / DZK[k]);
                    const float ABP = (k > KK + 1) ? DXK * DYK / (0.5f * (DZK[k - 1] + DZK[k])) : DXK * DYK / DZK[k];
                    const float ATP = (DXK * DYK) / (0.5f * (DZK[k + 1] + DZK[k]));
                    const float TERMP = 1 / (APP - ATP * PIMP[k + 1]);
                    PIMP[k] = ABP * TERMP;
                    QIMP[k] = (ATP * QIMP[k + 1] + DIM) * TERMP;
                }
                float *DPM_L = st.col(st.dpm, i, j);
                DPM_L[0] = 0;
                for (int k = 1; k <= NKK - 1; ++k) DPM_L[k] = (KK < k) ? PIMP[k] * DPM_L[k - 1] + QIMP[k] : 0;
            }
        }
        for (int i = 2; i < NII; ++i)                                /* velocity correction, :320-382 */
            for (int j = 2; j < NJJ; ++j) {
                const int KK = st.kkart(i, j);
                const float *DPM_L = st.col(st.dpm, i, j);
                const float *DPMim = st.col(st.dpm, i - 1, j), *DPMjm = st.col(st.dpm, i, j - 1);
                for (int k = 1; k < NKK; ++k) {
                    const float DDPX = DPMim[k] - DPM_L[k], DDPY = DPMjm[k] - DPM_L[k];
                    const float DDPZ = (k > KK + 1) ? DPM_L[k - 1] - DPM_L[k] : 0.0f;
                    float &u = st.uk[st.i3(i, j, k)], &v = st.vk[st.i3(i, j, k)], &w = st.wk[st.i3(i, j, k)];
                    u = ((KK < k) && (st.kkart(i - 1, j) < k)) ? u + (DDPX / DXK * DTIME) : 0.0f;
                    v = ((KK < k) && (st.kkart(i, j - 1) < k)) ? v + (DDPY / DYK * DTIME) : 0.0f;
                    w = (KK + 1 < k) ? w + (DDPZ * 2 / (DZK[k] + DZK[k - 1]) * DTIME) : 0.0f;
                }
            }
    }
    /* final vertical velocity outside the prognostic sub-domains (MicroscaleFlat.cs:389-462) */
    for (int i = 2; i < NII; ++i)
        for (int j = 2; j < NJJ; ++j) {
            if (st.advdom(i, j) != 0) continue;
            const int KK = st.kkart(i, j);
            for (int k = 1; k < NKK; ++k) {
                if (!(k > KK)) continue;
                const float fwo1 = (k <= st.kkart(i - 1, j)) ? 0.0f : DZK[k] * DYK * st.uk[st.i3(i, j, k)];
                const float fwo2 = (k <= st.kkart(i + 1, j)) ? 0.0f : DZK[k] * DYK * st.uk[st.i3(i + 1, j, k)];
                const float fsn1 = (k <= st.kkart(i, j - 1)) ? 0.0f : DZK[k] * DXK * st.vk[st.i3(i, j, k)];
                const float fsn2 = (k <= st.kkart(i, j + 1)) ? 0.0f : DZK[k] * DXK * st.vk[st.i3(i, j + 1, k)];
                const float fbt1 = ((k <= KK + 1) || (k == 1)) ? 0.0f : DXK * DYK * st.wk[st.i3(i, j, k)];
                st.wk[st.i3(i, j, k + 1)] = (fwo1 - fwo2 + fsn1 - fsn2 + fbt1) / (DXK * DYK);
            }
        }
}

/* UKS/VKS/WKS exist only where ADVDOM is set in the 3x3 neighbourhood (PrognosticFlowfield.cs:64-86). */
template <class T>
bool alloc3x3(const StateT<T> &st, int i, int j) {
    const int NII = st.nii, NJJ = st.njj;
    const int ip = std::min(i + 1, NII + 1), jp = std::min(j + 1, NJJ + 1);
    return st.advdom(i, j) == 1 || st.advdom(i - 1, j) == 1 || st.advdom(ip, j) == 1 ||
           st.advdom(i, j - 1) == 1 || st.advdom(i - 1, j - 1) == 1 || st.advdom(ip, j - 1) == 1 ||
           st.advdom(i, jp) == 1 || st.advdom(i - 1, jp) == 1 || st.advdom(ip, jp) == 1;
}

/* Initial staggered-grid velocities (PrognosticFlowfield.cs:295-329); returns GESCHW_MAX. */
template <class T>
double initial_staggered(StateT<T> &st) {
    const int NII = st.nii, NJJ = st.njj, NKK = st.nkk;
    double GESCHW_MAX = 0;
    for (int i = 1; i < NII + 1; ++i) {
        for (int j = 1; j <= NJJ; ++j) {
            if (!alloc3x3(st, i, j)) continue;
            for (int k = 1; k <= NKK - 1; ++k) {
                T u = 0.5f * (st.uk[st.i3(i, j, k)] + st.uk[st.i3(i + 1, j, k)]);
                T v = 0.5f * (st.vk[st.i3(i, j, k)] + st.vk[st.i3(i, j + 1, k)]);
                T w = 0.5f * (st.wk[st.i3(i, j, k)] + st.wk[st.i3(i, j, k + 1)]);
                st.uks[st.i3(i, j, k)] = u; st.vks[st.i3(i, j, k)] = v; st.wks[st.i3(i, j, k)] = w;
                GESCHW_MAX = net_maxd(GESCHW_MAX, std::sqrt((double)(pow2f((float)val(u)) + pow2f((float)val(v)))));
            }
        }
    }
    return GESCHW_MAX;
}

/* Border copies UK[NII+1] = UK[NII], VK[.][NJJ+1] = VK[.][NJJ] on levels 1..NKK-1 of the set-up
 * (PrognosticFlowfield.cs:410-432); setup_solve makes them in its TURB loop. */
template <class T>
void border_copies(StateT<T> &st) {
    const int NII = st.nii, NJJ = st.njj, NKK = st.nkk;
    for (int j = 1; j <= NJJ; ++j)
        for (int k = 1; k <= NKK - 1; ++k) st.uk[st.i3(NII + 1, j, k)] = st.uk[st.i3(NII, j, k)];
    for (int i = 1; i < NII + 1; ++i)
        for (int k = 1; k <= NKK - 1; ++k) st.vk[st.i3(i, NJJ + 1, k)] = st.vk[st.i3(i, NJJ, k)];
}

/* Velocities (and TKE) inside buildings set to zero (PrognosticFlowfield.cs:518-575). */
template <class T>
void zero_in_buildings(StateT<T> &st, int model) {
    const int NII = st.nii, NJJ = st.njj;
    for (int i = 1; i < NII + 1; ++i) {
        for (int j = 1; j <= NJJ; ++j) {
            if (st.advdom(i, j) != 1) continue;
            const int VI = st.vert_index[st.i2(i, j)];
            const int KK = st.kkart(i, j);
            for (int k = 1; k <= VI; ++k) {
                if (KK >= k) {
                    st.uk[st.i3(i, j, k)] = 0;
                    if (i == NII) st.uk[st.i3(i + 1, j, k)] = 0;
                    st.vk[st.i3(i, j, k)] = 0;
                    if (j == NJJ) st.vk[st.i3(i, j + 1, k)] = 0;
                    st.wk[st.i3(i, j, k)] = 0;
                    if (k == VI) st.wk[st.i3(i, j, k + 1)] = 0;
                    if (model != 1) { st.turb[st.i3(i, j, k)] = 0; st.tdiss[st.i3(i, j, k)] = 0; }
                    st.uks[st.i3(i, j, k)] = 0; st.vks[st.i3(i, j, k)] = 0; st.wks[st.i3(i, j, k)] = 0;
                }
            }
        }
    }
}

struct SetupOut {
    LoopConsts c;
    float topwind;
    double GESCHW_MAX;
};

/* Set-up of one solve (PrognosticFlowfield.cs:45-579) on the float state: allocations, the
 * per-solve scalars and the initial staggered velocities; the fields are zeroed inside buildings. */
static int setup_solve(State &st, const gral_params *p, const gral_static *s, gral_fields *f, SetupOut &o) {
    int rc = validate(p, s, f);
    if (rc != GRAL_OK) return rc;

    st.p = p; st.s = s;
    st.nii = p->nii; st.njj = p->njj; st.nkk = p->nkk;
    st.kadvmax = p->kadvmax; st.vcff = p->vert_cells_ff;
    st.ni2 = p->nii + 2; st.nj2 = p->njj + 2; st.nk2 = p->nkk + 2;
    st.dxk = p->dxk; st.dyk = p->dyk;
    const size_t n3 = (size_t)st.ni2 * st.nj2 * st.nk2, n2 = (size_t)st.ni2 * st.nj2;
    st.uk = f->uk; st.vk = f->vk; st.wk = f->wk;
    st.uks.assign(n3, 0.f); st.vks.assign(n3, 0.f); st.wks.assign(n3, 0.f);
    st.dpm.assign(n3, 0.f); st.dpmnew.assign(n3, 0.f); st.div.assign(n3, 0.f);
    st.vert_index.assign(n2, 0);
    st.ustern_terrain.assign(n2, 0.f); st.ustern_obst.assign(n2, 0.f);
    st.ap0.assign(st.nk2 + 1, 0.f);
    const int model = p->turbulence_model;
    if (model != 1) { st.turb = f->turb; st.tdiss = f->tdiss; }
    else {
        st.turb_own.assign(n3, 0.f); st.tdiss_own.assign(n3, 0.f);
        st.turb = st.turb_own.data(); st.tdiss = st.tdiss_own.data();
    }

    const int NII = st.nii, NJJ = st.njj, NKK = st.nkk;
    const float DXK = st.dxk, DYK = st.dyk;
    const float *DZK = s->dzk;
    const int rx = p->ref_i, ry = p->ref_j;


    /* topwind, DTIME, AP0 (:146-163) */
    float topwind = (float)std::sqrt((double)(pow2f(st.uk[st.i3(rx, ry, NKK - 1)]) +
                                              pow2f(st.vk[st.i3(rx, ry, NKK - 1)])));
    topwind = net_max(topwind, 0.01f);
    float DTIME = 0.5f * net_min(DXK, DZK[1]) /
                  net_max(0.01f, std::sqrt(pow2f(st.uk[st.i3(rx, ry, st.kadvmax)]) +
                                           pow2f(st.vk[st.i3(rx, ry, st.kadvmax)])));
    DTIME = net_min(DTIME, 5);
    const float AREAxy = DXK * DYK;
    for (int k = 1; k <= st.kadvmax; ++k) st.ap0[k] = AREAxy * DZK[k] / DTIME;
    const int MaxProgCellCount = st.vcff;
    const float building_Z0 = p->building_z0;
    const float Cmueh = 0.09f, Ceps = 1, Ceps1 = 1.44f, Ceps2 = 1.92f;

    /* DPM = 0 (:198-209), TURB/TDISS initial constants (:211-227) */
    if (model != 1 && p->turb_init == 0) {
        for (int i = 1; i < NII + 1; ++i)
            for (int j = 1; j <= NJJ; ++j)
                for (int k = 1; k <= NKK + 1; ++k) {
                    st.turb[st.i3(i, j, k)] = 0.001f;
                    st.tdiss[st.i3(i, j, k)] = 0.0000001f;
                }
    }

    /* Frund (:231-240): 8000 / topwind is a float division widened to double */
    double Frund = (double)(8000 / topwind);
    if (model == 2) Frund = (double)(10000 / topwind);
    const bool quantise = p->quantise != 0;

    const float relax = p->relax, relaxp = p->relaxp;

    /* initial staggered-grid velocities and GESCHW_MAX (:295-329) */
    double GESCHW_MAX = initial_staggered(st);

    /* VerticalIndex (:333-344) */
    for (int i = 1; i < NII + 1; ++i)
        for (int j = 1; j <= NJJ; ++j)
            st.vert_index[st.i2(i, j)] = std::min(NKK - 1, st.kkart(i, j) + MaxProgCellCount);

    /* friction-velocity help terms (:347-403) */
    for (int i = 1; i < NII + 1; ++i) {
        for (int j = 1; j <= NJJ; ++j) {
            int KSTART = 1;
            if (st.cutk(i, j) == 0) KSTART = st.kkart(i, j) + 1;
            const int VI = st.vert_index[st.i2(i, j)];
            const int KK = st.kkart(i, j);
            const float CUTK_L = st.cutk(i, j);
            const float rough = st.z0(i, j);
            for (int k = KSTART; k <= VI; ++k) {
                if (k != KK + 1) continue;
                if (CUTK_L < 1) {
                    if ((double)rough >= (double)DZK[k] * 0.1)
                        st.ustern_terrain[st.i2(i, j)] = 0.4f / std::log((DZK[k] + DZK[k + 1] * 0.5f) / DZK[k] * 0.1f);
                    else
                        st.ustern_terrain[st.i2(i, j)] = 0.4f / std::log(DZK[k] * 0.5f / rough);
                } else {
                    st.ustern_obst[st.i2(i, j)] = 0.4f / std::log(DZK[k] * 0.5f / building_Z0);
                }
            }
        }
    }

    /* geostrophic wind at the reference point (:406-407) */
    const float UG = st.uks[st.i3(rx, ry, NKK - 1)];
    const float VG = st.vks[st.i3(rx, ry, NKK - 1)];

    /* border copies and TURB initialisation (:410-510) */
    for (int i = 1; i < NII + 1; ++i) {
        for (int j = 1; j <= NJJ; ++j) {
            const size_t c = st.i2(i, j);
            for (int k = 1; k <= NKK - 1; ++k) {
                if (i == 1) st.uk[st.i3(NII + 1, j, k)] = st.uk[st.i3(NII, j, k)];
                if (j == 1) st.vk[st.i3(i, NJJ + 1, k)] = st.vk[st.i3(i, NJJ, k)];
                if (model != 1 && p->turb_init == 0) {
                    const float ObLength = s->ob_init[c], ust = s->ust_init[c], rough = s->z0_init[c];
                    float V0int = p->v0_1;
                    double windhilf = net_maxd(std::sqrt((double)(pow2f(st.uk[st.i3(i, j, k)]) +
                                                                  pow2f(st.vk[st.i3(i, j, k)]))), 0.01);
                    float U0int = (float)(windhilf * (0.2 * std::pow(windhilf, -0.9) + 0.32 * (double)rough + 0.18));
                    U0int = (float)net_maxd((double)U0int, 0.3) * p->std_dev_v;
                    float varw;
                    if (ObLength < 0)
                        varw = pow2f(ust) * pow2f(1.15f + 0.1f * std::pow(p->bd_lay_height / (-ObLength), 0.67f)) *
                               pow2f(p->std_dev_w);
                    else
                        varw = pow2f(ust * p->std_dev_w * 1.25f);
                    st.turb[st.i3(i, j, k)] = (float)(0.5 * (double)(pow2f(U0int) + pow2f(V0int) + varw));
                }
            }
        }
    }

    float VISHMIN = 0.0f, VISVMIN = 0.0f;
    if (model == 2) { VISHMIN = 0.01f; VISVMIN = 0.01f; }
    const float Ustern_factorX = (float)(0.4 / std::log((double)DXK * 0.5 / (double)building_Z0));

    /* velocities, TKE inside buildings set to zero (:518-575) */
    zero_in_buildings(st, model);

    o.c = LoopConsts{p, DTIME, AREAxy, UG, VG, relax, relaxp, VISHMIN, VISVMIN, building_Z0, Ustern_factorX,
                     Cmueh, Ceps, Ceps1, Ceps2, Frund, quantise, model};
    o.topwind = topwind;
    o.GESCHW_MAX = GESCHW_MAX;
    return GRAL_OK;
}

extern "C" int oracle_solve(const gral_params *p, const gral_static *s, gral_fields *f,
                            gral_stats *stats) {
    State st;
    SetupOut o;
    const int rc = setup_solve(st, p, s, f, o);
    if (rc != GRAL_OK) return rc;
    const LoopConsts &c = o.c;
    const int NII = st.nii, NJJ = st.njj, NKK = st.nkk;
    const float topwind = o.topwind;
    const double GESCHW_MAX = o.GESCHW_MAX;
    const double Frund = c.Frund;
    const float DTIME = c.DTIME;
    const int MaxProgCellCount = st.vcff;
    const int IterationStepsMin = p->iteration_steps_min, IterationStepsMax = p->iteration_steps_max;
    int IterationLoops = 1;
    float DeltaUMax = 0, DeltaFinish = 0, DeltaFirst = 0;
    double DeltaMean = 0;

    int iterations = 0;
    int n_hist = 0;
    bool converged = false;
    /* ------------------------------ SIMPLE loop (:584-1182) ------------------------------ */
    while (IterationLoops <= IterationStepsMax) {
        DeltaUMax = simple_iteration(st, c, IterationLoops);
        iterations++;
        if (stats && stats->trace_delta_umax && iterations <= stats->trace_capacity)
            stats->trace_delta_umax[iterations - 1] = DeltaUMax;

        /* convergence bookkeeping (:1144-1170) */
        if (IterationLoops >= IterationStepsMax) DeltaFinish = (float)(DeltaMean / (double)pow2f(topwind));
        if ((IterationLoops % p->conv_cadence == 0) && (IterationLoops > 1)) {
            double _delta = DeltaMean / (double)pow2f(topwind);
            if (IterationLoops == p->conv_cadence) DeltaFirst = (float)_delta;
            if (stats && n_hist < GRAL_MAX_HISTORY) stats->delta_history[n_hist] = _delta;
            n_hist++;
            if (_delta < p->conv_threshold && (IterationLoops >= IterationStepsMin)) { converged = true; break; }
            DeltaMean = 0;
        } else {
            DeltaMean += DeltaUMax;
        }
        IterationLoops++;
    }

    /* post-checks (:1187-1243) */
    int UKun = 0, VKun = 0, WKun = 0;
    for (int i = 1; i <= NII; ++i) {
        for (int j = 1; j <= NJJ; ++j) {
            if (st.advdom(i, j) != 1) continue;
            const float limit = (float)(10 * GESCHW_MAX);
            const int kmax = std::min(NKK - 1, st.kkart(i, j) + MaxProgCellCount);
            for (int k = 1; k <= kmax; ++k) {
                const float u = std::fabs(st.uk[st.i3(i, j, k)]), v = std::fabs(st.vk[st.i3(i, j, k)]);
                const float w = std::fabs(st.wk[st.i3(i, j, k)]);
                if (u > 55 || u > limit) UKun++;
                if (v > 55 || v > limit) VKun++;
                if (w > 20 || w > limit) WKun++;
            }
        }
    }

    if (p->post_diagnostic) diagnostic_post(st);

    if (stats) {
        stats->iterations = iterations;
        stats->iteration_loops = IterationLoops;
        stats->converged = converged ? 1 : 0;
        stats->convergence_problem = (DeltaFinish > DeltaFirst) ? 1 : 0;
        stats->delta_first = DeltaFirst;
        stats->delta_finish = DeltaFinish;
        stats->n_history = std::min(n_hist, GRAL_MAX_HISTORY);
        stats->uk_unrealistic = UKun; stats->vk_unrealistic = VKun; stats->wk_unrealistic = WKun;
        stats->geschw_max = GESCHW_MAX;
        stats->topwind = topwind; stats->dtime = DTIME; stats->frund = Frund;
        stats->last_delta_umax = DeltaUMax;
    }
    return GRAL_OK;
}

/* ============================================================================================
 * FP64 twin of the model-1 path and its reverse-mode differentiation (TEST INFRASTRUCTURE).
 *
 * The differentiated configuration of the library's adjoint: turbulence model 1, Vector<float>
 * parity width 8, no Frund rounding (its derivative is zero almost everywhere), a fixed number of
 * SIMPLE iterations, and the set-up's scalars (topwind, DTIME, AP0, UG, VG, help terms) held at the
 * values the reference set-up computes from the reference initial fields `f_ref` -- constants of
 * the differentiated map.  The twin runs the oracle's own operations (simple_iteration,
 * initial_staggered, zero_in_buildings, the model-1 sweeps) in double, or on the tape type of
 * oracle_ad.h for the gradient; instantiated for float it is the oracle itself.
 * ============================================================================================ */

thread_local Tape *oracle::g_tape = nullptr;

namespace {

constexpr int kTwinFields = 7;   /* uk, vk, wk, uks, vks, wks, dpmnew: the state between iterations */

int twin_validate(const gral_params *p, int iterations) {
    if (!p || p->turbulence_model != 1 || p->simd_width != 8 || p->quantise != 0 || iterations < 1)
        return GRAL_EINVAL;
    return GRAL_OK;
}

/* The float set-up on a copy of the reference fields: constants and per-column tables. */
int twin_setup(const gral_params *p, const gral_static *s, const gral_fields *f_ref, State &st0, SetupOut &o,
               std::vector<float> &scratch) {
    const size_t n3 = (size_t)(p->nii + 2) * (p->njj + 2) * (p->nkk + 2);
    scratch.assign(3 * n3, 0.f);
    std::memcpy(scratch.data(), f_ref->uk, n3 * sizeof(float));
    std::memcpy(scratch.data() + n3, f_ref->vk, n3 * sizeof(float));
    std::memcpy(scratch.data() + 2 * n3, f_ref->wk, n3 * sizeof(float));
    gral_fields g{scratch.data(), scratch.data() + n3, scratch.data() + 2 * n3, nullptr, nullptr};
    return setup_solve(st0, p, s, &g, o);
}

/* A T state on the grid of st0 with its tables, fields from the given arrays. */
template <class T>
void twin_state(const State &st0, StateT<T> &st, std::vector<T> &fields, const T *veg) {
    st.nii = st0.nii; st.njj = st0.njj; st.nkk = st0.nkk; st.kadvmax = st0.kadvmax; st.vcff = st0.vcff;
    st.ni2 = st0.ni2; st.nj2 = st0.nj2; st.nk2 = st0.nk2; st.dxk = st0.dxk; st.dyk = st0.dyk;
    st.p = st0.p; st.s = st0.s;
    const size_t n3 = (size_t)st.ni2 * st.nj2 * st.nk2;
    st.uk = fields.data(); st.vk = fields.data() + n3; st.wk = fields.data() + 2 * n3;
    st.turb = nullptr; st.tdiss = nullptr;
    st.uks.assign(n3, T(0.0)); st.vks.assign(n3, T(0.0)); st.wks.assign(n3, T(0.0));
    st.dpm.assign(n3, T(0.0)); st.dpmnew.assign(n3, T(0.0)); st.div.assign(n3, T(0.0));
    st.vert_index = st0.vert_index;
    st.ustern_terrain = st0.ustern_terrain; st.ustern_obst = st0.ustern_obst;
    st.ap0 = st0.ap0;
    st.veg_t = veg;
}

template <class T>
T *twin_field(StateT<T> &st, int q) {
    switch (q) {
        case 0: return st.uk;
        case 1: return st.vk;
        case 2: return st.wk;
        case 3: return st.uks.data();
        case 4: return st.vks.data();
        case 5: return st.wks.data();
        default: return st.dpmnew.data();
    }
}

}  // namespace

/* FP64 twin forward: `iterations` SIMPLE iterations from the initial fields uk0/vk0/wk0 (double,
 * host layout) with vegetation density veg (double [NII+2][NJJ+2][NKK+2], or NULL for the static
 * VEG), the set-up's scalars taken from f_ref.  Writes the final fields to uk/vk/wk. */
extern "C" int oracle_twin_forward(const gral_params *p, const gral_static *s, const gral_fields *f_ref,
                                   const double *uk0, const double *vk0, const double *wk0, const double *veg,
                                   int iterations, double *uk, double *vk, double *wk) {
    int rc = twin_validate(p, iterations);
    if (rc != GRAL_OK) return rc;
    State st0;
    SetupOut o;
    std::vector<float> scratch;
    rc = twin_setup(p, s, f_ref, st0, o, scratch);
    if (rc != GRAL_OK) return rc;
    const size_t n3 = (size_t)st0.ni2 * st0.nj2 * st0.nk2;
    std::vector<double> vegd(n3, 0.0);
    if (veg) std::memcpy(vegd.data(), veg, n3 * sizeof(double));
    else if (s->veg) for (size_t q = 0; q < n3; ++q) vegd[q] = s->veg[q];
    std::vector<double> fields(3 * n3);
    std::memcpy(fields.data(), uk0, n3 * sizeof(double));
    std::memcpy(fields.data() + n3, vk0, n3 * sizeof(double));
    std::memcpy(fields.data() + 2 * n3, wk0, n3 * sizeof(double));
    StateT<double> st;
    twin_state(st0, st, fields, vegd.data());
    initial_staggered(st);
    border_copies(st);
    zero_in_buildings(st, 1);
    for (int it = 1; it <= iterations; ++it) simple_iteration(st, o.c, it);
    std::memcpy(uk, st.uk, n3 * sizeof(double));
    std::memcpy(vk, st.vk, n3 * sizeof(double));
    std::memcpy(wk, st.wk, n3 * sizeof(double));
    return GRAL_OK;
}

/* FP64 reverse-mode gradient of the twin: given the cotangents g_uk/g_vk/g_wk of the final fields
 * (dJ/dUK etc.), writes dJ/d(initial fields) to d_uk0/d_vk0/d_wk0 and dJ/dVEG to d_veg (all double,
 * host layout).  The forward is recorded on the tape one iteration at a time from states kept by a
 * double forward pass (one checkpoint per iteration), then differentiated backwards. */
extern "C" int oracle_twin_vjp(const gral_params *p, const gral_static *s, const gral_fields *f_ref,
                               const double *uk0, const double *vk0, const double *wk0, const double *veg,
                               int iterations, const double *g_uk, const double *g_vk, const double *g_wk,
                               double *d_uk0, double *d_vk0, double *d_wk0, double *d_veg) {
    int rc = twin_validate(p, iterations);
    if (rc != GRAL_OK) return rc;
    State st0;
    SetupOut o;
    std::vector<float> scratch;
    rc = twin_setup(p, s, f_ref, st0, o, scratch);
    if (rc != GRAL_OK) return rc;
    const size_t n3 = (size_t)st0.ni2 * st0.nj2 * st0.nk2;
    std::vector<double> vegd(n3, 0.0);
    if (veg) std::memcpy(vegd.data(), veg, n3 * sizeof(double));
    else if (s->veg) for (size_t q = 0; q < n3; ++q) vegd[q] = s->veg[q];

    /* double forward keeping the state at the start of every iteration */
    std::vector<double> fields(3 * n3);
    std::memcpy(fields.data(), uk0, n3 * sizeof(double));
    std::memcpy(fields.data() + n3, vk0, n3 * sizeof(double));
    std::memcpy(fields.data() + 2 * n3, wk0, n3 * sizeof(double));
    StateT<double> st;
    twin_state(st0, st, fields, vegd.data());
    initial_staggered(st);
    border_copies(st);
    zero_in_buildings(st, 1);
    std::vector<std::vector<double>> keep((size_t)iterations, std::vector<double>(kTwinFields * n3));
    for (int it = 1; it <= iterations; ++it) {
        for (int q = 0; q < kTwinFields; ++q)
            std::memcpy(keep[it - 1].data() + q * n3, twin_field(st, q), n3 * sizeof(double));
        simple_iteration(st, o.c, it);
    }

    /* cotangents of the state, seeded with those of the final fields */
    std::vector<double> lam(kTwinFields * n3, 0.0), lveg(n3, 0.0);
    std::memcpy(lam.data(), g_uk, n3 * sizeof(double));
    std::memcpy(lam.data() + n3, g_vk, n3 * sizeof(double));
    std::memcpy(lam.data() + 2 * n3, g_wk, n3 * sizeof(double));

    Tape tape;
    g_tape = &tape;
    std::vector<AD> adf(3 * n3), adveg(n3);
    std::vector<int32_t> leaf(kTwinFields * n3), vleaf(n3);
    std::vector<double> adj;
    for (int it = iterations; it >= 1; --it) {
        tape.clear();
        const double *kp = keep[it - 1].data();
        for (size_t q = 0; q < 3 * n3; ++q) { adf[q] = AD::input(kp[q]); leaf[q] = adf[q].i; }
        for (size_t q = 0; q < n3; ++q) { adveg[q] = AD::input(vegd[q]); vleaf[q] = adveg[q].i; }
        StateT<AD> sa;
        twin_state(st0, sa, adf, adveg.data());
        for (int q = 3; q < kTwinFields; ++q) {
            AD *fld = twin_field(sa, q);
            for (size_t c = 0; c < n3; ++c) { fld[c] = AD::input(kp[q * n3 + c]); leaf[q * n3 + c] = fld[c].i; }
        }
        simple_iteration(sa, o.c, it);
        adj.assign(tape.nodes.size(), 0.0);
        for (int q = 0; q < kTwinFields; ++q) {
            const AD *fld = twin_field(sa, q);
            for (size_t c = 0; c < n3; ++c)
                if (fld[c].i >= 0) adj[(size_t)fld[c].i] += lam[q * n3 + c];
        }
        tape.reverse(adj);
        for (size_t q = 0; q < (size_t)kTwinFields * n3; ++q) lam[q] = adj[(size_t)leaf[q]];
        for (size_t q = 0; q < n3; ++q) lveg[q] += adj[(size_t)vleaf[q]];
    }

    /* the set-up: initial staggered velocities and zeroing inside buildings */
    tape.clear();
    for (size_t q = 0; q < 3 * n3; ++q) {
        const double v = (q < n3) ? uk0[q] : (q < 2 * n3 ? vk0[q - n3] : wk0[q - 2 * n3]);
        adf[q] = AD::input(v);
        leaf[q] = adf[q].i;
    }
    StateT<AD> sa;
    twin_state(st0, sa, adf, adveg.data());
    initial_staggered(sa);
    border_copies(sa);
    zero_in_buildings(sa, 1);
    adj.assign(tape.nodes.size(), 0.0);
    for (int q = 0; q < kTwinFields; ++q) {
        const AD *fld = twin_field(sa, q);
        for (size_t c = 0; c < n3; ++c)
            if (fld[c].i >= 0) adj[(size_t)fld[c].i] += lam[q * n3 + c];
    }
    tape.reverse(adj);
    for (size_t c = 0; c < n3; ++c) {
        d_uk0[c] = adj[(size_t)leaf[c]];
        d_vk0[c] = adj[(size_t)leaf[n3 + c]];
        d_wk0[c] = adj[(size_t)leaf[2 * n3 + c]];
        d_veg[c] = lveg[c];
    }
    g_tape = nullptr;
    return GRAL_OK;
}

/* Forward-mode tangent of the twin: d(final UK, VK, WK) along the direction (duk0, dvk0, dwk0, dveg)
 * of (initial fields, VEG), all double host layout (dveg may be NULL). */
extern "C" int oracle_twin_jvp(const gral_params *p, const gral_static *s, const gral_fields *f_ref,
                               const double *uk0, const double *vk0, const double *wk0, const double *veg,
                               const double *duk0, const double *dvk0, const double *dwk0, const double *dveg,
                               int iterations, double *duk, double *dvk, double *dwk) {
    int rc = twin_validate(p, iterations);
    if (rc != GRAL_OK) return rc;
    State st0;
    SetupOut o;
    std::vector<float> scratch;
    rc = twin_setup(p, s, f_ref, st0, o, scratch);
    if (rc != GRAL_OK) return rc;
    const size_t n3 = (size_t)st0.ni2 * st0.nj2 * st0.nk2;
    std::vector<Dual> vegd(n3), fields(3 * n3);
    for (size_t q = 0; q < n3; ++q) {
        vegd[q] = Dual(veg ? veg[q] : (s->veg ? (double)s->veg[q] : 0.0), dveg ? dveg[q] : 0.0);
        fields[q] = Dual(uk0[q], duk0[q]);
        fields[n3 + q] = Dual(vk0[q], dvk0[q]);
        fields[2 * n3 + q] = Dual(wk0[q], dwk0[q]);
    }
    StateT<Dual> st;
    twin_state(st0, st, fields, vegd.data());
    initial_staggered(st);
    border_copies(st);
    zero_in_buildings(st, 1);
    for (int it = 1; it <= iterations; ++it) simple_iteration(st, o.c, it);
    for (size_t q = 0; q < n3; ++q) { duk[q] = st.uk[q].d; dvk[q] = st.vk[q].d; dwk[q] = st.wk[q].d; }
    return GRAL_OK;
}
