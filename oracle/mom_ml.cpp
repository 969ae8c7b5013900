/*
 * mom_ml.cpp -- TEST INFRASTRUCTURE ONLY (CPU oracle, see oracle_common.h).
 *
 * U, V, W momentum with the algebraic mixing-length model (TurbulenceModel 1, the default),
 * restating U-prognostic-microscale_1.cs:50-529, V-prognostic-microscale_1.cs:50-524 and
 * W-prognostic-microscale_1.cs:51-453.  The reference evaluates each column in chunks of
 * SIMD = Vector<float>.Count lanes along k; chunk-level tests (mask, wall term, extra
 * eddy-viscosity term) use the chunk's base index, and the last chunk is pulled back to
 * KEND-SIMD (U-prognostic-microscale_1.cs:194-202).  This file keeps that chunk structure
 * literally, lane by lane, so the per-lane reformulation of the CUDA kernels is checked against
 * the reference's own loop shape.  SIMD = 8 is the Vector<float> path (.NET 8 x64, AVX2);
 * SIMD = 16 is the Vector512 twins (U/V/W-prognostic-microscale_1_Vec512.cs, chosen with
 * Program.UseVector512Class, PrognosticFlowfield.cs:1072), which keep the same loop but evaluate
 * a few expressions with fused multiply-adds and another association: the height above KKART
 * (zs), the power law, and the neighbour sums of DIM (pairs fma(A, x, B*y)); std::fma restates
 * Avx512F.FusedMultiplyAdd (one rounding).
 */
#include <algorithm>
#include <cmath>
#include <vector>

#include "oracle_ad.h"
#include "oracle_common.h"

namespace oracle {

static const float V0001 = 0.0001f;

/* Patankar power-law coefficient of one face, Vector<float> association order:
 * D * Max(0, i*i*i*i*i) + Max(sign*F, 0) with i = 1 - 0.1*|F/D| (U-prognostic-microscale_1.cs:348-370). */
template <class T>
static inline T pl_coef(T D, T Pe, T Fsigned) {
    T in = 1.0f - 0.1f * Pe;
    return D * vmax(T(0.0f), in * in * in * in * in) + vmax(Fsigned, T(0.0f));
}

/* Vector512 power law: FusedMultiplyAdd(D, Max(0, i*((i*i)*(i*i))), Max(sign*F, 0))
 * (U-prognostic-microscale_1_Vec512.cs:355-377). */
template <class T>
static inline T pl_coef512(T D, T Pe, T Fsigned) {
    T in = 1.0f - 0.1f * Pe;
    return ofma(D, vmax(T(0.0f), in * ((in * in) * (in * in))), vmax(Fsigned, T(0.0f)));
}

template <class T>
static inline T pl(bool v512, T D, T Pe, T Fsigned) {
    return v512 ? pl_coef512(D, Pe, Fsigned) : pl_coef(D, Pe, Fsigned);
}

template <class T>
static inline T opow2(T x) { return x * x; }

/* height of level k above the KKART surface: Vector512 uses HOKART[k] - fma(DZK, 0.5, HOKART[KKART])
 * (U-prognostic-microscale_1_Vec512.cs:218) */
static inline float zs_of(bool v512, float hok, float hokK, float dz) {
    return v512 ? hok - std::fma(dz, 0.5f, hokK) : hok - hokK - dz * 0.5f;
}

/* ------------------------------------------------------------------------------------------ */
/* U component, U-prognostic-microscale_1.cs:50-529                                           */
/* ------------------------------------------------------------------------------------------ */
template <class T>
void u_mom_ml(StateT<T> &st, const int SIMD, int IS, int JS, float VISHMIN, float AREAxy, float UG,
              float relax) {
    const bool v512 = (SIMD == 16);
    const int NII = st.nii, NJJ = st.njj;
    const float DXK = st.dxk, DYK = st.dyk;
    const float *DZK = st.dzk(), *HOKART = st.hokart();
    const float Cor = st.p->coriolis;
    oracle::for_slabs(3, NII, [&](int i1_lo, int i1_hi) {
    std::vector<T> PIMU(st.nk2), QIMU(st.nk2);
    std::vector<T> AIM_A(SIMD), BIM_A(SIMD), CIM_A(SIMD), DIM_A(SIMD), VIS_A(SIMD), MASK(SIMD);

    for (int i1 = i1_lo; i1 < i1_hi; i1++) {                       /* Partitioner.Create(3, NII) :61 */
        int i = (IS == -1) ? NII - i1 + 1 : i1;
        for (int j1 = 2; j1 <= NJJ - 1; ++j1) {
            int j = (JS == -1) ? NJJ - j1 + 1 : j1;
            if (st.advdom(i, j) != 1) continue;
            const int iM1 = i - 1, iP1 = i + 1, jM1 = j - 1, jP1 = j + 1;
            T *UK_L = st.col(st.uk, i, j);
            const T *UKS_L = st.col(st.uks, i, j), *VKS_L = st.col(st.vks, i, j);
            const T *WKS_L = st.col(st.wks, i, j), *DPMNEW_L = st.col(st.dpmnew, i, j);
            const T *UK_W_L = st.col(st.uk, iM1, j), *UK_E_L = st.col(st.uk, iP1, j);
            const T *UK_S_L = st.col(st.uk, i, jM1), *UK_N_L = st.col(st.uk, i, jP1);
            const T *UKS_W_L = st.col(st.uks, iM1, j), *VKS_W_L = st.col(st.vks, iM1, j);
            const T *VKS_WS_L = st.col(st.vks, iM1, jM1), *VKS_S_L = st.col(st.vks, i, jM1);
            const T *VKS_WN_L = st.col(st.vks, iM1, jP1), *VKS_N_L = st.col(st.vks, i, jP1);
            const T *WKS_W_L = st.col(st.wks, iM1, j), *DPMNEW_W_L = st.col(st.dpmnew, iM1, j);
            const T *VKS_EN_L = st.col(st.vks, iP1, jP1), *VKS_ES_L = st.col(st.vks, iP1, jM1);
            const T *WKS_E_L = st.col(st.wk, iP1, j);     /* WK, not WKS (:142) */
            const T *VK_L = st.col(st.vk, i, j);
            const int Vert_Index_LL = st.vert_index[st.i2(i, j)];
            const float Ust_terrain = st.ustern_terrain[st.i2(i, j)];
            const float Ust_obst = st.ustern_obst[st.i2(i, j)];
            const bool ADVDOM_S = (st.advdom(i, jM1) < 1) || (j == 2);
            const bool ADVDOM_N = (st.advdom(i, jP1) < 1) || (j == NJJ - 1);
            const bool ADVDOM_W = (st.advdom(iM1, j) < 1) || (i == 2);
            const bool ADVDOM_E = (st.advdom(iP1, j) < 1) || (i == NII - 1);
            const float CUTK_L = st.cutk(i, j), COV_L = st.cov(i, j), Z0 = st.z0(i, j);
            const bool veg = st.has_veg(i, j);
            const T *VEG_L = veg ? st.vegcol(i, j) : nullptr;
            const int KKART_LL = st.kkart(i, j);
            const float HOKART_KKART = HOKART[KKART_LL];
            int KSTART = 1;
            if (CUTK_L == 0) KSTART = KKART_LL + 1;
            const int KKART_LL_P1 = KKART_LL + 1;
            const int KEND = Vert_Index_LL + 1;

            for (int k = KSTART; k < KEND; k += SIMD) {
                int k_real = k;
                bool end = false;
                if (k > KEND - SIMD) { k = KEND - SIMD; end = true; }
                const bool mask_v_enable = (KKART_LL_P1 >= k && KKART_LL_P1 < (k + SIMD));
                for (int l = 0; l < SIMD; ++l) MASK[l] = ((k + l) > KKART_LL_P1) ? 1.0f : 0.0f;

                for (int l = 0; l < SIMD; ++l) {
                    const int kk = k + l;
                    const float DZK_V = DZK[kk];
                    const float DXKDZK = DXK * DZK_V, DYKDZK = DYK * DZK_V;
                    const float zs = zs_of(v512, HOKART[kk], HOKART_KKART, DZK_V);
                    T VIS = 0.0f;
                    if ((k + SIMD) > KKART_LL_P1) {
                        float mixL = vmin(0.071f * zs, 100.0f);
                        if (COV_L > 0) mixL *= (1.0f - 0.99f * COV_L);
                        T in = (UK_L[kk + 1] - UK_L[kk - 1]) / (2.0f * DZK_V);
                        T DUDZ = in * in;
                        in = (VK_L[kk + 1] - VK_L[kk - 1]) / (2.0f * DZK_V);
                        T DVDZ = in * in;
                        VIS = vmin(mixL * mixL * osqrt(0.5f * (DUDZ + DVDZ)), 15.0f);
                        if (mask_v_enable) VIS = VIS * MASK[l];
                    }
                    VIS_A[l] = VIS;
                    T DE = vmax(VIS, VISHMIN) * DYKDZK / DXK;
                    T DW = DE;
                    T DS = vmax(VIS, VISHMIN) * DXKDZK / DYK;
                    T DN = DS;
                    T DT = vmax(VIS, VISHMIN) * AREAxy / DZK_V;
                    T DB = 0.0f;
                    if (mask_v_enable) DB = DT * MASK[l];
                    else if (k > KKART_LL_P1) DB = DT;
                    if (ADVDOM_S) DS = 0.0f;
                    if (ADVDOM_N) DN = 0.0f;
                    if (ADVDOM_W) DW = 0.0f;
                    if (ADVDOM_E) DE = 0.0f;

                    const T UKS_V = UKS_L[kk], VKS_V = VKS_L[kk], WKS_V = WKS_L[kk];
                    const T VKS_W = VKS_W_L[kk], VKS_WS = VKS_WS_L[kk], VKS_S = VKS_S_L[kk];
                    const T VKS_WN = VKS_WN_L[kk], VKS_E = VKS_N_L[kk];
                    const T WKS_W = WKS_W_L[kk], UKS_W = UKS_W_L[kk];
                    const T FE = UKS_V * DYKDZK;
                    const T FW = UKS_W * DYKDZK;
                    const T FS = 0.25f * (VKS_W + VKS_V + VKS_WS + VKS_S) * DXKDZK;
                    const T FN = 0.25f * (VKS_W + VKS_V + VKS_WN + VKS_E) * DXKDZK;
                    const T FT = 0.25f * (WKS_W + WKS_V + WKS_W_L[kk + 1] + WKS_L[kk + 1]) * AREAxy;
                    const T WKS_B = WKS_L[kk - 1], WKS_WB = WKS_W_L[kk - 1];
                    T FB = 0.0f;
                    if (mask_v_enable) FB = 0.25f * (WKS_W + WKS_V + WKS_WB + WKS_B) * AREAxy * MASK[l];
                    else if (k > KKART_LL_P1) FB = 0.25f * (WKS_W + WKS_V + WKS_WB + WKS_B) * AREAxy;

                    DE = vmax(DE, V0001); DB = vmax(DB, V0001); DW = vmax(DW, V0001);
                    DS = vmax(DS, V0001); DN = vmax(DN, V0001); DT = vmax(DT, V0001);
                    const T PE = ofabs(FE / DE), PB = ofabs(FB / DB);
                    const T PW = ofabs(FW / DW), PS = ofabs(FS / DS);
                    const T PN = ofabs(FN / DN), PT = ofabs(FT / DT);
                    const T BIM = pl(v512, DT, PT, -FT);
                    const T CIM = pl(v512, DB, PB, FB);
                    const T AE1 = pl(v512, DE, PE, -FE);
                    const T AW1 = pl(v512, DW, PW, FW);
                    const T AS1 = pl(v512, DS, PS, FS);
                    const T AN1 = pl(v512, DN, PN, -FN);
                    const float AP0_V = st.ap0[kk];
                    const T AIM = BIM + CIM + AW1 + AS1 + AE1 + AN1 + AP0_V;

                    const T DDPX = DPMNEW_W_L[kk] - DPMNEW_L[kk];
                    const T UK_W = UK_W_L[kk], UK_E = UK_E_L[kk], UK_LV = UK_L[kk];
                    T DIM_U;
                    if (v512) {   /* U-prognostic-microscale_1_Vec512.cs:399-421 */
                        const T S1 = ofma(AW1, UK_W, AS1 * UK_S_L[kk]);
                        const T S2 = ofma(AE1, UK_E, AN1 * UK_N_L[kk]);
                        if (veg) {
                            T in2 = 0.5f * (VKS_W + VKS_V);
                            T in = 0.5f * (UKS_W + UKS_V);
                            T windhilf = vmax(osqrt(in * in + in2 * in2), 0.01f);
                            DIM_U = S1 + S2 + AP0_V * 0.5f * (UKS_W + UKS_V) + DDPX * DYKDZK +
                                    (Cor * (UG - UK_LV) - VEG_L[kk - 1] * UK_LV * windhilf) * AREAxy * DZK_V;
                        } else {
                            DIM_U = S1 + S2 + AP0_V * 0.5f * (UKS_W + UKS_V) +
                                    ofma(DDPX, DYKDZK, Cor * (UG - UK_LV) * AREAxy * DZK_V);
                        }
                    } else if (veg) {
                        T in2 = 0.5f * (VKS_W + VKS_V);
                        T in = 0.5f * (UKS_W + UKS_V);
                        T windhilf = vmax(osqrt(in * in + in2 * in2), 0.01f);
                        DIM_U = AW1 * UK_W + AS1 * UK_S_L[kk] + AE1 * UK_E + AN1 * UK_N_L[kk] +
                                AP0_V * 0.5f * (UKS_W + UKS_V) + DDPX * DYKDZK +
                                (Cor * (UG - UK_LV) - VEG_L[kk - 1] * UK_LV * windhilf) * AREAxy * DZK_V;
                    } else {
                        DIM_U = AW1 * UK_W + AS1 * UK_S_L[kk] + AE1 * UK_E + AN1 * UK_N_L[kk] +
                                AP0_V * 0.5f * (UKS_W + UKS_V) + DDPX * DYKDZK +
                                Cor * (UG - UK_LV) * AREAxy * DZK_V;
                    }
                    AIM_A[l] = AIM; BIM_A[l] = BIM; CIM_A[l] = CIM; DIM_A[l] = DIM_U;
                }

                /* wall function at the chunk holding KKART+1, U-prognostic-microscale_1.cs:419-450 */
                if ((k <= KKART_LL_P1) && ((k + SIMD) > KKART_LL_P1)) {
                    const int ii = KKART_LL_P1 - k;
                    std::vector<T> wh(SIMD);
                    for (int l = 0; l < SIMD; ++l) {
                        const int kk = k + l;
                        T in = 0.5f * (UKS_W_L[kk] + UKS_L[kk]);
                        T in2 = 0.5f * (VKS_W_L[kk] + VKS_L[kk]);
                        wh[l] = vmax(osqrt(in * in + in2 * in2), 0.1f);
                    }
                    T UstB;
                    if (CUTK_L < 1) {
                        UstB = Ust_terrain * wh[ii];
                        if (Z0 >= DZK[k + ii] * 0.1f) {
                            int ind = k + ii + 1;
                            UstB = Ust_terrain * osqrt(opow2(0.5f * ((UKS_W_L[ind]) + UKS_L[ind])) +
                                                           opow2(0.5f * ((VKS_W_L[ind]) + VKS_L[ind])));
                        }
                    } else {
                        UstB = Ust_obst * wh[ii];
                    }
                    const T Ust2 = UstB * UstB;
                    for (int l = 0; l < SIMD; ++l) {
                        const float m2 = (l == ii) ? 1.0f : 0.0f;
                        DIM_A[l] -= UK_L[k + l] / wh[l] * Ust2 * AREAxy * m2;
                    }
                }

                /* additional eddy-viscosity terms, tested on the chunk base, :453-470 */
                if (k > KKART_LL_P1) {
                    for (int l = 0; l < SIMD; ++l) {
                        const int kk = k + l;
                        const float DZK_V = DZK[kk];
                        const float DXKDZK = DXK * DZK_V, DYKDZK = DYK * DZK_V;
                        const T UK_LV = UK_L[kk], UK_E = UK_E_L[kk], UK_W = UK_W_L[kk];
                        const T VKS_E = VKS_N_L[kk], VKS_S = VKS_S_L[kk];
                        const T WKS_V = WKS_L[kk], WKS_W = WKS_W_L[kk];
                        const T WKS_B = WKS_L[kk - 1], WKS_WB = WKS_W_L[kk - 1];
                        T DUDXE = (UK_E - UK_LV) * DYKDZK;
                        T DUDXW = (UK_LV - UK_W) * DYKDZK;
                        T DVDXN = (0.5f * (VKS_EN_L[kk] + VKS_E) - 0.5f * (VKS_E + VKS_WN_L[kk])) * DXKDZK;
                        T DVDXS = (0.5f * (VKS_ES_L[kk] + VKS_S) - 0.5f * (VKS_S + VKS_WS_L[kk])) * DXKDZK;
                        T DWDXT = (0.5f * (WKS_E_L[kk] + WKS_V) - 0.5f * (WKS_V + WKS_W)) * AREAxy;
                        T DWDXB = (0.5f * (WKS_E_L[kk - 1] + WKS_B) - 0.5f * (WKS_B + WKS_WB)) * AREAxy;
                        DIM_A[l] += VIS_A[l] / DXK * (DUDXE - DUDXW + DVDXN - DVDXS + DWDXT - DWDXB);
                    }
                }

                /* recurrence, :473-504 */
                int kint_s = 0;
                if (end) { kint_s = k_real - k; k_real -= kint_s; }
                for (int kint = kint_s; kint < SIMD; ++kint) {
                    int index_i = k_real + kint;
                    if (index_i < KEND) {
                        if (index_i > KKART_LL_P1) {
                            T TERMP = 1 / (AIM_A[kint] - CIM_A[kint] * PIMU[index_i - 1]);
                            PIMU[index_i] = BIM_A[kint] * TERMP;
                            QIMU[index_i] = (DIM_A[kint] + CIM_A[kint] * QIMU[index_i - 1]) * TERMP;
                        } else {
                            T TERMP = 1 / AIM_A[kint];
                            PIMU[index_i] = BIM_A[kint] * TERMP;
                            QIMU[index_i] = DIM_A[kint] * TERMP;
                        }
                    }
                }
                if (end) k = KEND + 1;
            }

            /* relaxed back-substitution, :513-524 */
            const int KKARTm_LL = std::max(KKART_LL, st.kkart(i - 1, j));
            for (int k = Vert_Index_LL; k >= KSTART; --k) {
                if (KKARTm_LL < k) UK_L[k] += relax * (PIMU[k] * UK_L[k + 1] + QIMU[k] - UK_L[k]);
            }
        }
    }
    });
}

/* ------------------------------------------------------------------------------------------ */
/* V component, V-prognostic-microscale_1.cs:50-524 (called with -IS, -JS)                    */
/* ------------------------------------------------------------------------------------------ */
template <class T>
void v_mom_ml(StateT<T> &st, const int SIMD, int IS, int JS, float VISHMIN, float AREAxy, float VG,
              float relax) {
    const bool v512 = (SIMD == 16);
    const int NII = st.nii, NJJ = st.njj;
    const float DXK = st.dxk, DYK = st.dyk;
    const float *DZK = st.dzk(), *HOKART = st.hokart();
    const float Cor = st.p->coriolis;
    oracle::for_slabs(2, NII, [&](int i1_lo, int i1_hi) {
    std::vector<T> PIMV(st.nk2), QIMV(st.nk2);
    std::vector<T> AIM_A(SIMD), BIM_A(SIMD), CIM_A(SIMD), DIM_A(SIMD), VIS_A(SIMD), MASK(SIMD);

    for (int i1 = i1_lo; i1 < i1_hi; i1++) {                       /* Partitioner.Create(2, NII) :61 */
        int i = (IS == -1) ? NII - i1 + 1 : i1;
        for (int j1 = 3; j1 <= NJJ - 1; ++j1) {
            int j = (JS == -1) ? NJJ - j1 + 1 : j1;
            if (st.advdom(i, j) != 1) continue;
            const int iM1 = i - 1, iP1 = i + 1, jM1 = j - 1, jP1 = j + 1;
            T *VK_L = st.col(st.vk, i, j);
            const T *UKS_L = st.col(st.uks, i, j), *VKS_L = st.col(st.vks, i, j);
            const T *WKS_L = st.col(st.wks, i, j), *DPMNEW_L = st.col(st.dpmnew, i, j);
            const T *VK_W_L = st.col(st.vk, iM1, j), *VK_E_L = st.col(st.vk, iP1, j);
            const T *VK_S_L = st.col(st.vk, i, jM1), *VK_N_L = st.col(st.vk, i, jP1);
            const T *UKS_W_L = st.col(st.uks, iM1, j), *UKS_E_L = st.col(st.uks, iP1, j);
            const T *UKS_S_L = st.col(st.uks, i, jM1), *UKS_ES_L = st.col(st.uks, iP1, jM1);
            const T *UKS_WS_L = st.col(st.uks, iM1, jM1), *VKS_S_L = st.col(st.vks, i, jM1);
            const T *VKS_W_L = st.col(st.vks, iM1, j), *WKS_S_L = st.col(st.wks, i, jM1);
            const T *DPMNEW_S_L = st.col(st.dpmnew, i, jM1);
            const T *UKS_EN_L = st.col(st.uks, iP1, jP1), *UKS_WN_L = st.col(st.uks, iM1, jP1);
            const T *WKS_N_L = st.col(st.wk, i, jP1);     /* WK, not WKS (:140) */
            const T *UK_L = st.col(st.uk, i, j);
            const int Vert_Index_LL = st.vert_index[st.i2(i, j)];
            const float Ust_terrain = st.ustern_terrain[st.i2(i, j)];
            const float Ust_obst = st.ustern_obst[st.i2(i, j)];
            const bool ADVDOM_S = (st.advdom(i, jM1) < 1) || (j == 2);
            const bool ADVDOM_N = (st.advdom(i, jP1) < 1) || (j == NJJ - 1);
            const bool ADVDOM_W = (st.advdom(iM1, j) < 1) || (i == 2);
            const bool ADVDOM_E = (st.advdom(iP1, j) < 1) || (i == NII - 1);
            const float CUTK_L = st.cutk(i, j), COV_L = st.cov(i, j), Z0 = st.z0(i, j);
            const bool veg = st.has_veg(i, j);
            const T *VEG_L = veg ? st.vegcol(i, j) : nullptr;
            const int KKART_LL = st.kkart(i, j);
            const float HOKART_KKART = HOKART[KKART_LL];
            int KSTART = 1;
            if (CUTK_L == 0) KSTART = KKART_LL + 1;
            const int KKART_LL_P1 = KKART_LL + 1;
            const int KEND = Vert_Index_LL + 1;

            for (int k = KSTART; k < KEND; k += SIMD) {
                int k_real = k;
                bool end = false;
                if (k > KEND - SIMD) { k = KEND - SIMD; end = true; }
                const bool mask_v_enable = (KKART_LL_P1 >= k && KKART_LL_P1 < (k + SIMD));
                for (int l = 0; l < SIMD; ++l) MASK[l] = ((k + l) > KKART_LL_P1) ? 1.0f : 0.0f;

                for (int l = 0; l < SIMD; ++l) {
                    const int kk = k + l;
                    const float DZK_V = DZK[kk];
                    const float DXKDZK = DXK * DZK_V, DYKDZK = DYK * DZK_V;
                    const T VK_LV = VK_L[kk];
                    const float zs = zs_of(v512, HOKART[kk], HOKART_KKART, DZK_V);
                    T VIS = 0.0f;
                    if ((k + SIMD) > KKART_LL_P1) {
                        float mixL = vmin(0.071f * zs, 100.0f);
                        if (COV_L > 0) mixL *= (1.0f - 0.99f * COV_L);
                        T in = (UK_L[kk + 1] - UK_L[kk - 1]) / (2.0f * DZK_V);
                        T DUDZ = in * in;
                        in = (VK_L[kk + 1] - VK_L[kk - 1]) / (2.0f * DZK_V);
                        T DVDZ = in * in;
                        VIS = vmin(mixL * mixL * osqrt(0.5f * (DUDZ + DVDZ)), 15.0f);
                        if (mask_v_enable) VIS = VIS * MASK[l];
                    }
                    VIS_A[l] = VIS;
                    T DE = vmax(VIS, VISHMIN) * DYKDZK / DXK;
                    T DW = DE;
                    T DS = vmax(VIS, VISHMIN) * DXKDZK / DYK;
                    T DN = DS;
                    T DT = vmax(VIS, VISHMIN) * AREAxy / DZK_V;
                    T DB = 0.0f;
                    if (mask_v_enable) DB = DT * MASK[l];
                    else if (k > KKART_LL_P1) DB = DT;
                    if (ADVDOM_S) DS = 0.0f;
                    if (ADVDOM_N) DN = 0.0f;
                    if (ADVDOM_W) DW = 0.0f;
                    if (ADVDOM_E) DE = 0.0f;

                    const T UKS_V = UKS_L[kk], VKS_V = VKS_L[kk], WKS_V = WKS_L[kk];
                    const T UKS_E = UKS_E_L[kk], UKS_N = UKS_S_L[kk]; /* named N, loads S (:317) */
                    const T UKS_ES = UKS_ES_L[kk], UKS_W = UKS_W_L[kk];
                    const T VKS_W = VKS_W_L[kk], UKS_WS = UKS_WS_L[kk];
                    const T VKS_S = VKS_S_L[kk], WKS_S = WKS_S_L[kk], WKS_B = WKS_L[kk - 1];
                    const T FE = 0.25f * (UKS_V + UKS_E + UKS_N + UKS_ES) * DYKDZK;
                    const T FW = 0.25f * (UKS_V + UKS_W + UKS_N + UKS_WS) * DYKDZK;
                    const T FS = VKS_S * DXKDZK;
                    const T FN = VKS_V * DXKDZK;
                    const T FT = 0.25f * (WKS_S + WKS_V + WKS_S_L[kk + 1] + WKS_L[kk + 1]) * AREAxy;
                    T FB = 0.0f;
                    if (mask_v_enable) FB = 0.25f * (WKS_S + WKS_V + WKS_S_L[kk - 1] + WKS_B) * AREAxy * MASK[l];
                    else if (k > KKART_LL_P1) FB = 0.25f * (WKS_S + WKS_V + WKS_S_L[kk - 1] + WKS_B) * AREAxy;

                    DE = vmax(DE, V0001); DB = vmax(DB, V0001); DW = vmax(DW, V0001);
                    DS = vmax(DS, V0001); DN = vmax(DN, V0001); DT = vmax(DT, V0001);
                    const T PE = ofabs(FE / DE), PB = ofabs(FB / DB);
                    const T PW = ofabs(FW / DW), PS = ofabs(FS / DS);
                    const T PN = ofabs(FN / DN), PT = ofabs(FT / DT);
                    const T BIM = pl(v512, DT, PT, -FT);
                    const T CIM = pl(v512, DB, PB, FB);
                    const T AE1 = pl(v512, DE, PE, -FE);
                    const T AW1 = pl(v512, DW, PW, FW);
                    const T AS1 = pl(v512, DS, PS, FS);
                    const T AN1 = pl(v512, DN, PN, -FN);
                    const float AP0_V = st.ap0[kk];
                    const T AIM = BIM + CIM + AW1 + AS1 + AE1 + AN1 + AP0_V;

                    const T DDPY = DPMNEW_S_L[kk] - DPMNEW_L[kk];
                    const T VK_N = VK_N_L[kk], VK_S = VK_S_L[kk];
                    T DIMV;
                    if (veg) {
                        T in2 = 0.5f * (VKS_W + VKS_V);
                        T in = 0.5f * (UKS_W + UKS_V);
                        T windhilf = vmax(osqrt(in * in + in2 * in2), 0.01f);
                        if (v512)   /* V-prognostic-microscale_1_Vec512.cs:404-410; no vegetation: plain sums */
                            DIMV = ofma(AW1, VK_W_L[kk], AS1 * VK_S) + ofma(AE1, VK_E_L[kk], AN1 * VK_N) +
                                   AP0_V * 0.5f * (VKS_S + VKS_V) + DDPY * DXKDZK +
                                   (Cor * (VG - VK_LV) - VEG_L[kk - 1] * VK_LV * windhilf) * AREAxy * DZK_V;
                        else
                            DIMV = AW1 * VK_W_L[kk] + AS1 * VK_S + AE1 * VK_E_L[kk] + AN1 * VK_N +
                                   AP0_V * 0.5f * (VKS_S + VKS_V) + DDPY * DXKDZK +
                                   (Cor * (VG - VK_LV) - VEG_L[kk - 1] * VK_LV * windhilf) * AREAxy * DZK_V;
                    } else {
                        DIMV = AW1 * VK_W_L[kk] + AS1 * VK_S + AE1 * VK_E_L[kk] + AN1 * VK_N +
                               AP0_V * 0.5f * (VKS_S + VKS_V) + DDPY * DXKDZK +
                               Cor * (VG - VK_LV) * AREAxy * DZK_V;
                    }
                    AIM_A[l] = AIM; BIM_A[l] = BIM; CIM_A[l] = CIM; DIM_A[l] = DIMV;
                }

                if ((k <= KKART_LL_P1) && ((k + SIMD) > KKART_LL_P1)) {   /* :437-467 */
                    const int ii = KKART_LL_P1 - k;
                    std::vector<T> wh(SIMD);
                    for (int l = 0; l < SIMD; ++l) {
                        const int kk = k + l;
                        T in = 0.5f * (UKS_W_L[kk] + UKS_L[kk]);
                        T in2 = 0.5f * (VKS_W_L[kk] + VKS_L[kk]);
                        wh[l] = vmax(osqrt(in * in + in2 * in2), 0.1f);
                    }
                    T UstB;
                    if (CUTK_L < 1) {
                        UstB = Ust_terrain * wh[ii];
                        if (Z0 >= DZK[k + ii] * 0.1f) {
                            int ind = k + ii + 1;
                            UstB = Ust_terrain * osqrt(opow2(0.5f * ((UKS_W_L[ind]) + UKS_L[ind])) +
                                                           opow2(0.5f * ((VKS_W_L[ind]) + VKS_L[ind])));
                        }
                    } else {
                        UstB = Ust_obst * wh[ii];
                    }
                    const T Ust2 = UstB * UstB;
                    for (int l = 0; l < SIMD; ++l) {
                        const float m2 = (l == ii) ? 1.0f : 0.0f;
                        DIM_A[l] -= VK_L[k + l] / wh[l] * Ust2 * AREAxy * m2;
                    }
                }

                if (k > KKART_LL_P1) {                                        /* :470-488 */
                    for (int l = 0; l < SIMD; ++l) {
                        const int kk = k + l;
                        const float DZK_V = DZK[kk];
                        const float DXKDZK = DXK * DZK_V;
                        const T VK_LV = VK_L[kk], VK_N = VK_N_L[kk], VK_S = VK_S_L[kk];
                        const T UKS_E = UKS_E_L[kk], UKS_ES = UKS_ES_L[kk];
                        const T UKS_W = UKS_W_L[kk], UKS_WS = UKS_WS_L[kk];
                        const T WKS_V = WKS_L[kk], WKS_S = WKS_S_L[kk], WKS_B = WKS_L[kk - 1];
                        T DVDYN = (VK_N - VK_LV) * DXKDZK;
                        T DVDYS = (VK_LV - VK_S) * DXKDZK;
                        T DUDYE = (0.5f * (UKS_EN_L[kk] + UKS_E) - 0.5f * (UKS_E + UKS_ES)) * DXKDZK;
                        T DUDYW = (0.5f * (UKS_WN_L[kk] + UKS_W) - 0.5f * (UKS_W + UKS_WS)) * DXKDZK;
                        T DWDYT = (0.5f * (WKS_N_L[kk] + WKS_V) - 0.5f * (WKS_V + WKS_S)) * AREAxy;
                        T DWDYB = (0.5f * (WKS_N_L[kk - 1] + WKS_B) - 0.5f * (WKS_B + WKS_S)) * AREAxy;
                        DIM_A[l] += VIS_A[l] / DXK * (DUDYE - DUDYW + DVDYN - DVDYS + DWDYT - DWDYB);
                    }
                }

                int kint_s = 0;
                if (end) { kint_s = k_real - k; k_real -= kint_s; }
                for (int kint = kint_s; kint < SIMD; ++kint) {
                    int index_i = k_real + kint;
                    if (index_i < KEND) {
                        if (index_i > KKART_LL_P1) {
                            T TERMP = 1 / (AIM_A[kint] - CIM_A[kint] * PIMV[index_i - 1]);
                            PIMV[index_i] = BIM_A[kint] * TERMP;
                            QIMV[index_i] = (DIM_A[kint] + CIM_A[kint] * QIMV[index_i - 1]) * TERMP;
                        } else {
                            T TERMP = 1 / AIM_A[kint];
                            PIMV[index_i] = BIM_A[kint] * TERMP;
                            QIMV[index_i] = DIM_A[kint] * TERMP;
                        }
                    }
                }
                if (end) k = KEND + 1;
            }

            const int KKARTm_LL = std::max(KKART_LL, st.kkart(i, j - 1));   /* :509-519 */
            for (int k = Vert_Index_LL; k >= KSTART; --k) {
                if (KKARTm_LL < k) VK_L[k] += relax * (PIMV[k] * VK_L[k + 1] + QIMV[k] - VK_L[k]);
            }
        }
    }
    });
}

/* ------------------------------------------------------------------------------------------ */
/* W component, W-prognostic-microscale_1.cs:51-453                                           */
/* ------------------------------------------------------------------------------------------ */
template <class T>
void w_mom_ml(StateT<T> &st, const int SIMD, int IS, int JS, float VISHMIN, float AREAxy, float relax) {
    const bool v512 = (SIMD == 16);
    const int NII = st.nii, NJJ = st.njj;
    const float DXK = st.dxk, DYK = st.dyk;
    const float *DZK = st.dzk(), *HOKART = st.hokart();
    oracle::for_slabs(2, NII, [&](int i1_lo, int i1_hi) {
    std::vector<T> PIMW(st.nk2), QIMW(st.nk2);
    std::vector<T> AIM_A(SIMD), BIM_A(SIMD), CIM_A(SIMD), DIM_A(SIMD), VIS_A(SIMD), MASK(SIMD);

    for (int i1 = i1_lo; i1 < i1_hi; i1++) {
        int i = (IS == -1) ? NII - i1 + 1 : i1;
        for (int j1 = 2; j1 < NJJ; ++j1) {
            int j = (JS == -1) ? NJJ - j1 + 1 : j1;
            if (st.advdom(i, j) != 1) continue;
            const int iM1 = i - 1, iP1 = i + 1, jM1 = j - 1, jP1 = j + 1;
            T *WK_L = st.col(st.wk, i, j);
            const T *WK_W_L = st.col(st.wk, iM1, j), *WK_E_L = st.col(st.wk, iP1, j);
            const T *WK_S_L = st.col(st.wk, i, jM1), *WK_N_L = st.col(st.wk, i, jP1);
            const T *UKS_L = st.col(st.uks, i, j), *VKS_L = st.col(st.vks, i, j);
            const T *WKS_L = st.col(st.wks, i, j), *DPMNEW_L = st.col(st.dpmnew, i, j);
            const T *UKS_W_L = st.col(st.uks, iM1, j), *UKS_E_L = st.col(st.uks, iP1, j);
            const T *VKS_S_L = st.col(st.vks, i, jM1), *VKS_N_L = st.col(st.vks, i, jP1);
            const T *UK_L = st.col(st.uk, i, j), *VK_L = st.col(st.vk, i, j);
            const int KKART_LL = st.kkart(i, j);
            const int Vert_Index_LL = st.vert_index[st.i2(i, j)];
            const bool ADVDOM_S = (st.advdom(i, jM1) < 1) || (j == 2);
            const bool ADVDOM_N = (st.advdom(i, jP1) < 1) || (j == NJJ - 1);
            const bool ADVDOM_W = (st.advdom(iM1, j) < 1) || (i == 2);
            const bool ADVDOM_E = (st.advdom(iP1, j) < 1) || (i == NII - 1);
            const bool veg = st.has_veg(i, j);
            const T *VEG_L = veg ? st.vegcol(i, j) : nullptr;
            const float COV_L = st.cov(i, j);
            const float HOKART_KKART = HOKART[KKART_LL];
            int KSTART = 1;
            if (st.cutk(i, j) == 0) KSTART = KKART_LL + 1;
            const int KKART_LL_P1 = KKART_LL + 1;
            const int KEND = Vert_Index_LL + 1;

            for (int k = KSTART; k < KEND; k += SIMD) {
                int k_real = k;
                bool end = false;
                if (k > KEND - SIMD) { k = KEND - SIMD; end = true; }
                const bool mask_v_enable = (KKART_LL_P1 >= k && KKART_LL_P1 < (k + SIMD));
                for (int l = 0; l < SIMD; ++l) MASK[l] = ((k + l) > KKART_LL_P1) ? 1.0f : 0.0f;

                for (int l = 0; l < SIMD; ++l) {
                    const int kk = k + l;
                    const float DZK_V = DZK[kk];
                    const float DXKDZK = DXK * DZK_V, DYKDZK = DYK * DZK_V;
                    const T UKS_V = UKS_L[kk], VKS_V = VKS_L[kk], WKS_V = WKS_L[kk];
                    const T UKS_M = UKS_L[kk - 1], VKS_M = VKS_L[kk - 1];
                    const float zs = zs_of(v512, HOKART[kk], HOKART_KKART, DZK_V);
                    T VIS = 0.0f;
                    if ((k + SIMD) > KKART_LL_P1) {
                        float mixL = vmin(0.071f * zs, 100.0f);
                        if (COV_L > 0) mixL *= (1.0f - 0.99f * COV_L);
                        T in = (UK_L[kk + 1] - UK_L[kk - 1]) / (2.0f * DZK_V);
                        T DUDZ = in * in;
                        in = (VK_L[kk + 1] - VK_L[kk - 1]) / (2.0f * DZK_V);
                        T DVDZ = in * in;
                        VIS = vmin(mixL * mixL * osqrt(0.5f * (DUDZ + DVDZ)), 15.0f);
                        if (mask_v_enable) VIS = VIS * MASK[l];
                    }
                    VIS_A[l] = VIS;
                    T DE = vmax(VIS, VISHMIN) * DYKDZK / DXK;
                    T DW = DE;
                    T DS = vmax(VIS, VISHMIN) * DXKDZK / DYK;
                    T DN = DS;
                    T DT = vmax(VIS, VISHMIN) * AREAxy / DZK_V;
                    T DB = 0.0f;
                    if (mask_v_enable) DB = DT * MASK[l];
                    else if (k > KKART_LL_P1) DB = DT;
                    if (ADVDOM_S) DS = 0.0f;
                    if (ADVDOM_N) DN = 0.0f;
                    if (ADVDOM_W) DW = 0.0f;
                    if (ADVDOM_E) DE = 0.0f;

                    const T UKS_W = UKS_W_L[kk], UKS_WB = UKS_W_L[kk - 1];
                    const T VKS_S = VKS_S_L[kk], VKS_SB = VKS_S_L[kk - 1];
                    const T FE = 0.25f * (UKS_V + UKS_E_L[kk] + UKS_M + UKS_E_L[kk - 1]) * DYKDZK;
                    const T FW = 0.25f * (UKS_V + UKS_W + UKS_M + UKS_WB) * DYKDZK;
                    const T FS = 0.25f * (VKS_V + VKS_S + VKS_M + VKS_SB) * DXKDZK;
                    const T FN = 0.25f * (VKS_V + VKS_N_L[kk] + VKS_M + VKS_N_L[kk - 1]) * DXKDZK;
                    const T FT = WKS_V * AREAxy;
                    T FB = 0.0f;
                    if (mask_v_enable) FB = WKS_L[kk - 1] * AREAxy * MASK[l];
                    else if (k > KKART_LL_P1) FB = WKS_L[kk - 1] * AREAxy;

                    DE = vmax(DE, V0001); DB = vmax(DB, V0001); DW = vmax(DW, V0001);
                    DS = vmax(DS, V0001); DN = vmax(DN, V0001); DT = vmax(DT, V0001);
                    const T PE = ofabs(FE / DE), PB = ofabs(FB / DB);
                    const T PW = ofabs(FW / DW), PS = ofabs(FS / DS);
                    const T PN = ofabs(FN / DN), PT = ofabs(FT / DT);
                    const T BIM = pl(v512, DT, PT, -FT);
                    const T CIM = pl(v512, DB, PB, FB);
                    const T AE1 = pl(v512, DE, PE, -FE);
                    const T AW1 = pl(v512, DW, PW, FW);
                    const T AS1 = pl(v512, DS, PS, FS);
                    const T AN1 = pl(v512, DN, PN, -FN);
                    const float AP0_V = st.ap0[kk];
                    const T AIM = BIM + CIM + AW1 + AS1 + AE1 + AN1 + AP0_V;

                    const T DDPZ = DPMNEW_L[kk - 1] - DPMNEW_L[kk];
                    const T WK_LV = WK_L[kk];
                    T DIMW;
                    if (veg) {
                        T in2 = 0.5f * (VKS_S + VKS_V);
                        T in = 0.5f * (UKS_W + UKS_V);
                        T windhilf = vmax(osqrt(in * in + in2 * in2), 0.01f);
                        if (v512)   /* W-prognostic-microscale_1_Vec512.cs:367-372 */
                            DIMW = ofma(AW1, WK_W_L[kk], AS1 * WK_S_L[kk]) + ofma(AE1, WK_E_L[kk], AN1 * WK_N_L[kk]) +
                                   AP0_V * 0.5f * (WKS_L[kk - 1] + WKS_V) + DDPZ * AREAxy -
                                   VEG_L[kk - 1] * WK_LV * windhilf * AREAxy * DZK_V;
                        else
                            DIMW = AW1 * WK_W_L[kk] + AS1 * WK_S_L[kk] + AE1 * WK_E_L[kk] + AN1 * WK_N_L[kk] +
                                   AP0_V * 0.5f * (WKS_L[kk - 1] + WKS_V) + DDPZ * AREAxy -
                                   VEG_L[kk - 1] * WK_LV * windhilf * AREAxy * DZK_V;
                    } else if (v512) {   /* :377-382 */
                        DIMW = ofma(AW1, WK_W_L[kk], AS1 * WK_S_L[kk]) + ofma(AE1, WK_E_L[kk], AN1 * WK_N_L[kk]) +
                               AP0_V * 0.5f * (WKS_L[kk - 1] + WKS_V) + DDPZ * AREAxy;
                    } else {
                        DIMW = AW1 * WK_W_L[kk] + AS1 * WK_S_L[kk] + AE1 * WK_E_L[kk] + AN1 * WK_N_L[kk] +
                               AP0_V * 0.5f * (WKS_L[kk - 1] + WKS_V) + DDPZ * AREAxy;
                    }
                    AIM_A[l] = AIM; BIM_A[l] = BIM; CIM_A[l] = CIM; DIM_A[l] = DIMW;
                }

                if (k > KKART_LL_P1) {                                        /* :376-402 */
                    for (int l = 0; l < SIMD; ++l) {
                        const int kk = k + l;
                        const float DZK_V = DZK[kk];
                        const float DXKDZK = DXK * DZK_V, DYKDZK = DYK * DZK_V;
                        const T UKS_V = UKS_L[kk], UKS_M = UKS_L[kk - 1];
                        const T VKS_V = VKS_L[kk], VKS_M = VKS_L[kk - 1];
                        const T UKS_W = UKS_W_L[kk], UKS_WB = UKS_W_L[kk - 1];
                        const T VKS_S = VKS_S_L[kk], VKS_SB = VKS_S_L[kk - 1];
                        const T WK_LV = WK_L[kk];
                        T DUDZE = (0.5f * (UKS_L[kk + 1] + UKS_V) - 0.5f * (UKS_V + UKS_M)) * DYKDZK;
                        T DUDZW = (0.5f * (UKS_W_L[kk + 1] + UKS_W) - 0.5f * (UKS_W + UKS_WB)) * DYKDZK;
                        T DVDZN = (0.5f * (VKS_L[kk + 1] + VKS_V) - 0.5f * (VKS_V + VKS_M)) * DXKDZK;
                        T DVDZS = (0.5f * (VKS_S_L[kk + 1] + VKS_S) - 0.5f * (VKS_S + VKS_SB)) * DXKDZK;
                        T DWDZT = (WK_L[kk + 1] - WK_LV) * AREAxy;
                        T DWDZB = (WK_LV - WK_L[kk - 1]) * AREAxy;
                        DIM_A[l] += VIS_A[l] / DZK_V * (DUDZE - DUDZW + DVDZN - DVDZS + DWDZT - DWDZB);
                    }
                }

                int kint_s = 0;
                if (end) { kint_s = k_real - k; k_real -= kint_s; }
                for (int kint = kint_s; kint < SIMD; ++kint) {
                    int index_i = k_real + kint;
                    if (index_i < KEND) {
                        if (index_i > KKART_LL_P1) {
                            T TERMP = 1 / (AIM_A[kint] - CIM_A[kint] * PIMW[index_i - 1]);
                            PIMW[index_i] = BIM_A[kint] * TERMP;
                            QIMW[index_i] = (DIM_A[kint] + CIM_A[kint] * QIMW[index_i - 1]) * TERMP;
                        } else {
                            T TERMP = 1 / AIM_A[kint];
                            PIMW[index_i] = BIM_A[kint] * TERMP;
                            QIMW[index_i] = DIM_A[kint] * TERMP;
                        }
                    }
                }
                if (end) k = KEND + 1;
            }

            for (int k = Vert_Index_LL; k >= KSTART; --k) {               /* :444-448 */
                WK_L[k] += relax * (PIMW[k] * WK_L[k + 1] + QIMW[k] - WK_L[k]);
            }
        }
    }
    });
}

template void u_mom_ml<float>(StateT<float> &, int, int, int, float, float, float, float);
template void v_mom_ml<float>(StateT<float> &, int, int, int, float, float, float, float);
template void w_mom_ml<float>(StateT<float> &, int, int, int, float, float, float);
template void u_mom_ml<double>(StateT<double> &, int, int, int, float, float, float, float);
template void v_mom_ml<double>(StateT<double> &, int, int, int, float, float, float, float);
template void w_mom_ml<double>(StateT<double> &, int, int, int, float, float, float);
template void u_mom_ml<AD>(StateT<AD> &, int, int, int, float, float, float, float);
template void u_mom_ml<Dual>(StateT<Dual> &, int, int, int, float, float, float, float);
template void v_mom_ml<Dual>(StateT<Dual> &, int, int, int, float, float, float, float);
template void w_mom_ml<Dual>(StateT<Dual> &, int, int, int, float, float, float);
template void v_mom_ml<AD>(StateT<AD> &, int, int, int, float, float, float, float);
template void w_mom_ml<AD>(StateT<AD> &, int, int, int, float, float, float);

}  // namespace oracle
