/*
 * mom_ke.cpp -- TEST INFRASTRUCTURE ONLY (CPU oracle, see oracle_common.h).
 *
 * Scalar momentum routines: the k-eps model (TurbulenceModel 2), restating
 * U-prognostic-microscale_2.cs:27-269, V-prognostic-microscale_2.cs:27-269,
 * W-prognostic-microscale_2.cs:27-212 and TKE-prognostic-microscale.cs:25-352; and the
 * no-diffusion upwind model (TurbulenceModel 0), restating U-prognostic-microscale_0.cs:27-190,
 * V-prognostic-microscale_0.cs and W-prognostic-microscale_0.cs:27-140.  These routines mix
 * float and double arithmetic; every promotion below follows the C# expression types.
 */
#include <algorithm>
#include <cmath>
#include <vector>

#include "oracle_common.h"

namespace oracle {

/* Power-law coefficient of the k-eps U/V/W routines, evaluated partly in double:
 * D * FloatMax(0, (float)Pow5(1 - 0.1 * Pe)) + FloatMax(Fs, 0)  (U-prognostic-microscale_2.cs:180-185). */
static inline float pl_ke(float D, float Pe, float Fs) {
    return D * float_max(0.0f, (float)pow5d(1 - 0.1 * (double)Pe)) + float_max(Fs, 0.0f);
}

/* Shared helpers of the wall term (U-prognostic-microscale_2.cs:206-230): windhilf and the
 * friction-velocity estimate, in double with float inputs. */
static inline float wind_half(float a1, float a2, float b1, float b2) {
    return (float)std::sqrt(pow2d(0.5 * (double)(a1 + a2)) + pow2d(0.5 * (double)(b1 + b2)));
}

/* ------------------------------------------------------------------------------------------ */
/* Generic scalar U/V routine (model 2: with diffusion; model 0: without).                    */
/* comp = 0 for U, 1 for V.                                                                   */
/* ------------------------------------------------------------------------------------------ */
static void uv_scalar(State &st, int comp, bool diffusion, int IS, int JS, float Cmueh,
                      float VISHMIN, float AREAxy_L, float UG, float relax) {
    const int NII = st.nii, NJJ = st.njj;
    const float DXK = st.dxk, DYK = st.dyk;
    const float *DZK = st.dzk(), *HOKART = st.hokart();
    const float Cor = st.p->coriolis;
    const int i_lo = (comp == 0) ? 3 : 2;   /* Parallel.For(3, NII) for U, (2, NII) for V */
    const int j_lo = (comp == 0) ? 2 : 3;   /* j1 from 2 for U, from 3 for V */
    oracle::for_slabs(i_lo, NII, [&](int i1_lo, int i1_hi) {
    std::vector<float> PIM(st.nk2), QIM(st.nk2);

    for (int i1 = i1_lo; i1 < i1_hi; i1++) {
        for (int j1 = j_lo; j1 <= NJJ - 1; j1++) {
            int j = (JS == -1) ? NJJ - j1 + 1 : j1;
            int i = (IS == -1) ? NII - i1 + 1 : i1;
            if (st.advdom(i, j) != 1) continue;
            float *PHI = (comp == 0) ? st.col(st.uk, i, j) : st.col(st.vk, i, j);
            const float *TURB_L = st.col(st.turb, i, j);
            const float *UKS_L = st.col(st.uks, i, j), *VKS_L = st.col(st.vks, i, j);
            const float *WKS_L = st.col(st.wks, i, j), *DPMNEW_L = st.col(st.dpmnew, i, j);
            float *const FLD = (comp == 0) ? st.uk : st.vk;
            const float *PHIim = st.col(FLD, i - 1, j), *PHIip = st.col(FLD, i + 1, j);
            const float *PHIjm = st.col(FLD, i, j - 1), *PHIjp = st.col(FLD, i, j + 1);
            const float *UKSim = st.col(st.uks, i - 1, j), *VKSim = st.col(st.vks, i - 1, j);
            const float *VKSimjm = st.col(st.vks, i - 1, j - 1), *VKSjm = st.col(st.vks, i, j - 1);
            const float *VKSimjp = st.col(st.vks, i - 1, j + 1), *VKSjp = st.col(st.vks, i, j + 1);
            const float *WKSim = st.col(st.wks, i - 1, j), *WKSjm = st.col(st.wks, i, j - 1);
            const float *DPMNEWim = st.col(st.dpmnew, i - 1, j), *DPMNEWjm = st.col(st.dpmnew, i, j - 1);
            const float *VKSipjp = st.col(st.vks, i + 1, j + 1), *VKSipjm = st.col(st.vks, i + 1, j - 1);
            const float *UKSip = st.col(st.uks, i + 1, j), *UKSjm = st.col(st.uks, i, j - 1);
            const float *UKSipjm = st.col(st.uks, i + 1, j - 1), *UKSimjm = st.col(st.uks, i - 1, j - 1);
            const float *UKSipjp = st.col(st.uks, i + 1, j + 1), *UKSimjp = st.col(st.uks, i - 1, j + 1);
            const float *WKip = st.col(st.wk, i + 1, j), *WKjp = st.col(st.wk, i, j + 1);
            const int KKART_LL = st.kkart(i, j);
            const int Vert_Index_LL = st.vert_index[st.i2(i, j)];
            const float Ust_terrain = st.ustern_terrain[st.i2(i, j)];
            const float Ust_obst = st.ustern_obst[st.i2(i, j)];
            const float CUTK_L = st.cutk(i, j);
            const float Z0 = st.z0(i, j);
            int KSTART = 1;
            if (CUTK_L == 0) KSTART = KKART_LL + 1;

            for (int k = KSTART; k <= Vert_Index_LL; k++) {
                const float DZK_K = DZK[k];
                const float DXKDZK = DXK * DZK_K, DYKDZK = DYK * DZK_K;
                float VIS = 0, DE = 0, DW = 0, DS = 0, DN = 0, DT = 0, DB = 0;
                if (diffusion) {
                    const float zs = HOKART[k] - HOKART[KKART_LL] - DZK_K * 0.5f;
                    VIS = (float)std::sqrt((double)TURB_L[k]) * zs * Cmueh;
                    DE = float_max(VIS, VISHMIN) * DYKDZK / DXK;
                    DW = DE;
                    DS = float_max(VIS, VISHMIN) * DXKDZK / DYK;
                    DN = DS;
                    DT = float_max(VIS, VISHMIN) * AREAxy_L / DZK_K;
                    DB = 0;
                    if (k > KKART_LL + 1) DB = DT;
                    if ((st.advdom(i, j - 1) < 1) || (j == 2)) DS = 0;
                    if ((st.advdom(i, j + 1) < 1) || (j == NJJ - 1)) DN = 0;
                    if ((st.advdom(i - 1, j) < 1) || (i == 2)) DW = 0;
                    if ((st.advdom(i + 1, j) < 1) || (i == NII - 1)) DE = 0;
                }
                float FE, FW, FS, FN, FT, FB = 0;
                if (comp == 0) {
                    FE = UKS_L[k] * DYKDZK;
                    FW = UKSim[k] * DYKDZK;
                    FS = 0.25f * (VKSim[k] + VKS_L[k] + VKSimjm[k] + VKSjm[k]) * DXKDZK;
                    FN = 0.25f * (VKSim[k] + VKS_L[k] + VKSimjp[k] + VKSjp[k]) * DXKDZK;
                    FT = 0.25f * (WKSim[k] + WKS_L[k] + WKSim[k + 1] + WKS_L[k + 1]) * AREAxy_L;
                    if (k > KKART_LL + 1) FB = 0.25f * (WKSim[k] + WKS_L[k] + WKSim[k - 1] + WKS_L[k - 1]) * AREAxy_L;
                } else {
                    FE = 0.25f * (UKS_L[k] + UKSip[k] + UKSjm[k] + UKSipjm[k]) * DYKDZK;
                    FW = 0.25f * (UKS_L[k] + UKSim[k] + UKSjm[k] + UKSimjm[k]) * DYKDZK;
                    FS = VKSjm[k] * DXKDZK;
                    FN = VKS_L[k] * DXKDZK;
                    FT = 0.25f * (WKSjm[k] + WKS_L[k] + WKSjm[k + 1] + WKS_L[k + 1]) * AREAxy_L;
                    if (k > KKART_LL + 1) FB = 0.25f * (WKSjm[k] + WKS_L[k] + WKSjm[k - 1] + WKS_L[k - 1]) * AREAxy_L;
                }
                float BIM, CIM, AE1, AW1, AS1, AN1;
                if (diffusion) {
                    DE = float_max(DE, 0.0001f); DB = float_max(DB, 0.0001f);
                    DW = float_max(DW, 0.0001f); DS = float_max(DS, 0.0001f);
                    DN = float_max(DN, 0.0001f); DT = float_max(DT, 0.0001f);
                    const float PE = std::fabs(FE / DE), PB = std::fabs(FB / DB);
                    const float PW = std::fabs(FW / DW), PS = std::fabs(FS / DS);
                    const float PN = std::fabs(FN / DN), PT = std::fabs(FT / DT);
                    BIM = pl_ke(DT, PT, -FT);
                    CIM = pl_ke(DB, PB, FB);
                    AE1 = pl_ke(DE, PE, -FE);
                    AW1 = pl_ke(DW, PW, FW);
                    AS1 = pl_ke(DS, PS, FS);
                    AN1 = pl_ke(DN, PN, -FN);
                } else {                       /* upwind, U-prognostic-microscale_0.cs:123-128 */
                    BIM = float_max(-FT, 0.0f);
                    CIM = float_max(FB, 0.0f);
                    AE1 = float_max(-FE, 0.0f);
                    AW1 = float_max(FW, 0.0f);
                    AS1 = float_max(FS, 0.0f);
                    AN1 = float_max(-FN, 0.0f);
                }
                const float AP0 = st.ap0[k];
                const float AIM = BIM + CIM + AW1 + AS1 + AE1 + AN1 + AP0;

                float DIM;
                if (comp == 0) {
                    const float DDPX = DPMNEWim[k] - DPMNEW_L[k];
                    DIM = (float)(AW1 * PHIim[k] + AS1 * PHIjm[k] + AE1 * PHIip[k] + AN1 * PHIjp[k] +
                                  st.ap0[k] * 0.5 * (UKSim[k] + UKS_L[k]) + DDPX * DYKDZK +
                                  Cor * (UG - PHI[k]) * AREAxy_L * DZK_K);
                } else {
                    const float DDPY = DPMNEWjm[k] - DPMNEW_L[k];
                    DIM = (float)(AW1 * PHIim[k] + AS1 * PHIjm[k] + AE1 * PHIip[k] + AN1 * PHIjp[k] +
                                  st.ap0[k] * 0.5 * (VKSjm[k] + VKS_L[k]) + DDPY * DXKDZK +
                                  Cor * (UG - PHI[k]) * AREAxy_L * DZK_K);
                }

                if (k == KKART_LL + 1) {       /* wall function, U-prognostic-microscale_2.cs:205-231 */
                    const float windhilf = float_max(wind_half(UKSim[k], UKS_L[k], VKSim[k], VKS_L[k]), 0.01f);
                    float UstB;
                    if (CUTK_L < 1) {
                        UstB = Ust_terrain * windhilf;
                        if ((double)Z0 >= (double)DZK_K * 0.1) {
                            UstB = Ust_terrain * wind_half(UKSim[k + 1], UKS_L[k + 1], VKSim[k + 1], VKS_L[k + 1]);
                        }
                    } else {
                        UstB = Ust_obst * windhilf;
                    }
                    DIM -= (float)(PHI[k] / windhilf * pow2f(UstB) * AREAxy_L);
                }

                if (diffusion && k > KKART_LL + 1) {   /* :234-245 */
                    float ADD;
                    if (comp == 0) {
                        float DUDXE = (PHIip[k] - PHI[k]) * DYKDZK;
                        float DUDXW = (PHI[k] - PHIim[k]) * DYKDZK;
                        float DVDXN = (0.5f * (VKSipjp[k] + VKSjp[k]) - 0.5f * (VKSjp[k] + VKSimjp[k])) * DXKDZK;
                        float DVDXS = (0.5f * (VKSipjm[k] + VKSjm[k]) - 0.5f * (VKSjm[k] + VKSimjm[k])) * DXKDZK;
                        float DWDXT = (0.5f * (WKip[k] + WKS_L[k]) - 0.5f * (WKS_L[k] + WKSim[k])) * AREAxy_L;
                        float DWDXB = (0.5f * (WKip[k - 1] + WKS_L[k - 1]) - 0.5f * (WKS_L[k - 1] + WKSim[k - 1])) * AREAxy_L;
                        ADD = VIS / DXK * (DUDXE - DUDXW + DVDXN - DVDXS + DWDXT - DWDXB);
                    } else {
                        float DVDYN = (PHIjp[k] - PHI[k]) * DXKDZK;
                        float DVDYS = (PHI[k] - PHIjm[k]) * DXKDZK;
                        float DUDYE = (0.5f * (UKSipjp[k] + UKSip[k]) - 0.5f * (UKSip[k] + UKSipjm[k])) * DXKDZK;
                        float DUDYW = (0.5f * (UKSimjp[k] + UKSim[k]) - 0.5f * (UKSim[k] + UKSimjm[k])) * DXKDZK;
                        float DWDYT = (0.5f * (WKjp[k] + WKS_L[k]) - 0.5f * (WKS_L[k] + WKSjm[k])) * AREAxy_L;
                        float DWDYB = (0.5f * (WKjp[k - 1] + WKS_L[k - 1]) - 0.5f * (WKS_L[k - 1] + WKSjm[k - 1])) * AREAxy_L;
                        ADD = VIS / DXK * (DUDYE - DUDYW + DVDYN - DVDYS + DWDYT - DWDYB);
                    }
                    DIM += ADD;
                }

                if (k > KKART_LL + 1) {            /* recurrence with two divisions, :247-256 */
                    PIM[k] = (BIM / (AIM - CIM * PIM[k - 1]));
                    QIM[k] = ((DIM + CIM * QIM[k - 1]) / (AIM - CIM * PIM[k - 1]));
                } else {
                    PIM[k] = (BIM / AIM);
                    QIM[k] = (DIM / AIM);
                }
            }
            const int KKn = (comp == 0) ? st.kkart(i - 1, j) : st.kkart(i, j - 1);
            for (int k = Vert_Index_LL; k >= KSTART; k--) {
                if ((KKART_LL < k) && (KKn < k)) PHI[k] += (relax * (PIM[k] * PHI[k + 1] + QIM[k] - PHI[k]));
            }
        }
    }
    });
}

void u_mom_ke(State &st, int IS, int JS, float Cmueh, float VISHMIN, float AREAxy, float UG, float relax) {
    uv_scalar(st, 0, true, IS, JS, Cmueh, VISHMIN, AREAxy, UG, relax);
}
void v_mom_ke(State &st, int IS, int JS, float Cmueh, float VISHMIN, float AREAxy, float VG, float relax) {
    uv_scalar(st, 1, true, IS, JS, Cmueh, VISHMIN, AREAxy, VG, relax);
}
void u_mom_nd(State &st, int IS, int JS, float AREAxy, float UG, float relax) {
    uv_scalar(st, 0, false, IS, JS, 0.0f, 0.0f, AREAxy, UG, relax);
}
void v_mom_nd(State &st, int IS, int JS, float AREAxy, float VG, float relax) {
    uv_scalar(st, 1, false, IS, JS, 0.0f, 0.0f, AREAxy, VG, relax);
}

/* ------------------------------------------------------------------------------------------ */
/* W, model 2 (W-prognostic-microscale_2.cs:27-212)                                            */
/* ------------------------------------------------------------------------------------------ */
void w_mom_ke(State &st, int IS, int JS, float Cmueh, float VISHMIN, float AREAxy_L, float relax) {
    const int NII = st.nii, NJJ = st.njj;
    const float DXK = st.dxk, DYK = st.dyk;
    const float *DZK = st.dzk(), *HOKART = st.hokart();
    oracle::for_slabs(2, NII, [&](int i1_lo, int i1_hi) {
    std::vector<float> PIMW(st.nk2), QIMW(st.nk2);
    for (int i1 = i1_lo; i1 < i1_hi; i1++) {
        for (int j1 = 2; j1 <= NJJ - 1; j1++) {
            int j = (JS == -1) ? NJJ - j1 + 1 : j1;
            int i = (IS == -1) ? NII - i1 + 1 : i1;
            if (st.advdom(i, j) != 1) continue;
            const float *TURB_L = st.col(st.turb, i, j);
            float *WK_L = st.col(st.wk, i, j);
            const float *WKim = st.col(st.wk, i - 1, j), *WKip = st.col(st.wk, i + 1, j);
            const float *WKjm = st.col(st.wk, i, j - 1), *WKjp = st.col(st.wk, i, j + 1);
            const float *UKS_L = st.col(st.uks, i, j), *VKS_L = st.col(st.vks, i, j);
            const float *WKS_L = st.col(st.wks, i, j), *DPMNEW_L = st.col(st.dpmnew, i, j);
            const float *UKSim = st.col(st.uks, i - 1, j), *UKSip = st.col(st.uks, i + 1, j);
            const float *VKSjm = st.col(st.vks, i, j - 1), *VKSjp = st.col(st.vks, i, j + 1);
            const int KKART_LL = st.kkart(i, j);
            const int Vert_Index_LL = st.vert_index[st.i2(i, j)];
            int KSTART = 1;
            if (st.cutk(i, j) == 0) KSTART = KKART_LL + 1;
            for (int k = KSTART; k <= Vert_Index_LL; k++) {
                const float DZK_K = DZK[k];
                const float DXKDZK = DXK * DZK_K, DYKDZK = DYK * DZK_K;
                const float UKS_LL = UKS_L[k], UKS_LL_m = UKS_L[k - 1], VKS_LL = VKS_L[k], VKS_LL_m = VKS_L[k - 1];
                const float zs = HOKART[k] - HOKART[KKART_LL] - DZK_K * 0.5f;
                const float VIS = (float)std::sqrt((double)TURB_L[k]) * zs * Cmueh;
                float DE = float_max(VIS, VISHMIN) * DYKDZK / DXK;
                float DW = DE;
                float DS = float_max(VIS, VISHMIN) * DXKDZK / DYK;
                float DN = DS;
                float DT = float_max(VIS, VISHMIN) * AREAxy_L / DZK_K;
                float DB = 0;
                if (k > KKART_LL + 1) DB = DT;
                if ((st.advdom(i, j - 1) < 1) || (j == 2)) DS = 0;
                if ((st.advdom(i, j + 1) < 1) || (j == NJJ - 1)) DN = 0;
                if ((st.advdom(i - 1, j) < 1) || (i == 2)) DW = 0;
                if ((st.advdom(i + 1, j) < 1) || (i == NII - 1)) DE = 0;
                const float FE = 0.25f * (UKS_LL + UKSip[k] + UKS_LL_m + UKSip[k - 1]) * DYKDZK;
                const float FW = 0.25f * (UKS_LL + UKSim[k] + UKS_LL_m + UKSim[k - 1]) * DYKDZK;
                const float FS = 0.25f * (VKS_LL + VKSjm[k] + VKS_LL_m + VKSjm[k - 1]) * DXKDZK;
                const float FN = 0.25f * (VKS_LL + VKSjp[k] + VKS_LL_m + VKSjp[k - 1]) * DXKDZK;
                const float FT = WKS_L[k] * AREAxy_L;
                float FB = 0;
                if (k > KKART_LL + 1) FB = WKS_L[k - 1] * AREAxy_L;
                DE = float_max(DE, 0.0001f); DB = float_max(DB, 0.0001f);
                DW = float_max(DW, 0.0001f); DS = float_max(DS, 0.0001f);
                DN = float_max(DN, 0.0001f); DT = float_max(DT, 0.0001f);
                const float PE = std::fabs(FE / DE), PB = std::fabs(FB / DB);
                const float PW = std::fabs(FW / DW), PS = std::fabs(FS / DS);
                const float PN = std::fabs(FN / DN), PT = std::fabs(FT / DT);
                const float BIM = pl_ke(DT, PT, -FT), CIM = pl_ke(DB, PB, FB);
                const float AE1 = pl_ke(DE, PE, -FE), AW1 = pl_ke(DW, PW, FW);
                const float AS1 = pl_ke(DS, PS, FS), AN1 = pl_ke(DN, PN, -FN);
                const float AIM = BIM + CIM + AW1 + AS1 + AE1 + AN1 + st.ap0[k];
                const float DDPZ = DPMNEW_L[k - 1] - DPMNEW_L[k];
                float DIMW = (float)(AW1 * WKim[k] + AS1 * WKjm[k] + AE1 * WKip[k] + AN1 * WKjp[k] +
                                     st.ap0[k] * 0.5 * (WKS_L[k - 1] + WKS_L[k]) + DDPZ * AREAxy_L);
                if (k > KKART_LL + 1) {
                    float DUDZE = (0.5f * (UKS_L[k + 1] + UKS_LL) - 0.5f * (UKS_LL + UKS_LL_m)) * DYKDZK;
                    float DUDZW = (0.5f * (UKSim[k + 1] + UKSim[k]) - 0.5f * (UKSim[k] + UKSim[k - 1])) * DYKDZK;
                    float DVDZN = (0.5f * (VKS_L[k + 1] + VKS_LL) - 0.5f * (VKS_LL + VKS_LL_m)) * DXKDZK;
                    float DVDZS = (0.5f * (VKSjm[k + 1] + VKSjm[k]) - 0.5f * (VKSjm[k] + VKSjm[k - 1])) * DXKDZK;
                    float DWDZT = (WK_L[k + 1] - WK_L[k]) * AREAxy_L;
                    float DWDZB = (WK_L[k] - WK_L[k - 1]) * AREAxy_L;
                    float ADD = VIS / DZK_K * (DUDZE - DUDZW + DVDZN - DVDZS + DWDZT - DWDZB);
                    DIMW += ADD;
                }
                if (k > KKART_LL + 1) {
                    PIMW[k] = (BIM / (AIM - CIM * PIMW[k - 1]));
                    QIMW[k] = ((DIMW + CIM * QIMW[k - 1]) / (AIM - CIM * PIMW[k - 1]));
                } else {
                    PIMW[k] = (BIM / AIM);
                    QIMW[k] = (DIMW / AIM);
                }
            }
            for (int k = Vert_Index_LL; k >= KSTART; k--) {
                WK_L[k] += (relax * (PIMW[k] * WK_L[k + 1] + QIMW[k] - WK_L[k]));
            }
        }
    }
    });
}

/* ------------------------------------------------------------------------------------------ */
/* W, model 0 (W-prognostic-microscale_0.cs:27-140): recurrence held in double                 */
/* ------------------------------------------------------------------------------------------ */
void w_mom_nd(State &st, int IS, int JS, float AREAxy_L, float relax) {
    const int NII = st.nii, NJJ = st.njj;
    const float DXK = st.dxk, DYK = st.dyk;
    const float *DZK = st.dzk();
    oracle::for_slabs(2, NII, [&](int i1_lo, int i1_hi) {
    std::vector<double> PIMW(st.nk2), QIMW(st.nk2);
    for (int i1 = i1_lo; i1 < i1_hi; i1++) {
        for (int j1 = 2; j1 <= NJJ - 1; j1++) {
            int j = (JS == -1) ? NJJ - j1 + 1 : j1;
            int i = (IS == -1) ? NII - i1 + 1 : i1;
            if (st.advdom(i, j) != 1) continue;
            float *WK_L = st.col(st.wk, i, j);
            const float *WKim = st.col(st.wk, i - 1, j), *WKip = st.col(st.wk, i + 1, j);
            const float *WKjm = st.col(st.wk, i, j - 1), *WKjp = st.col(st.wk, i, j + 1);
            const float *UKS_L = st.col(st.uks, i, j), *VKS_L = st.col(st.vks, i, j);
            const float *WKS_L = st.col(st.wks, i, j), *DPMNEW_L = st.col(st.dpmnew, i, j);
            const float *UKSim = st.col(st.uks, i - 1, j), *UKSip = st.col(st.uks, i + 1, j);
            const float *VKSjm = st.col(st.vks, i, j - 1), *VKSjp = st.col(st.vks, i, j + 1);
            const int KKART_LL = st.kkart(i, j);
            const int Vert_Index_LL = st.vert_index[st.i2(i, j)];
            int KSTART = 1;
            if (st.cutk(i, j) == 0) KSTART = KKART_LL + 1;
            for (int k = KSTART; k <= Vert_Index_LL; k++) {
                const float DZK_K = DZK[k];
                const float DXKDZK = DXK * DZK_K, DYKDZK = DYK * DZK_K;
                const float UKS_LL = UKS_L[k], UKS_LL_m = UKS_L[k - 1], VKS_LL = VKS_L[k], VKS_LL_m = VKS_L[k - 1];
                const float AP0 = st.ap0[k];
                const float FE = 0.25f * (UKS_LL + UKSip[k] + UKS_LL_m + UKSip[k - 1]) * DYKDZK;
                const float FW = 0.25f * (UKS_LL + UKSim[k] + UKS_LL_m + UKSim[k - 1]) * DYKDZK;
                const float FS = 0.25f * (VKS_LL + VKSjm[k] + VKS_LL_m + VKSjm[k - 1]) * DXKDZK;
                const float FN = 0.25f * (VKS_LL + VKSjp[k] + VKS_LL_m + VKSjp[k - 1]) * DXKDZK;
                const float FT = WKS_L[k] * AREAxy_L;
                float FB = 0;
                if (k > KKART_LL + 1) FB = WKS_L[k - 1] * AREAxy_L;
                const float BIM = float_max(-FT, 0), CIM = float_max(FB, 0);
                const float AE1 = float_max(-FE, 0), AW1 = float_max(FW, 0);
                const float AS1 = float_max(FS, 0), AN1 = float_max(-FN, 0);
                const float AIM = BIM + CIM + AW1 + AS1 + AE1 + AN1 + AP0;
                const float DDPZ = DPMNEW_L[k - 1] - DPMNEW_L[k];
                const float DIMW = (float)(AW1 * WKim[k] + AS1 * WKjm[k] + AE1 * WKip[k] + AN1 * WKjp[k] +
                                           AP0 * 0.5 * (WKS_L[k - 1] + WKS_L[k]) + DDPZ * AREAxy_L);
                if (k > KKART_LL + 1) {
                    PIMW[k] = (BIM / (AIM - CIM * PIMW[k - 1]));
                    QIMW[k] = ((DIMW + CIM * QIMW[k - 1]) / (AIM - CIM * PIMW[k - 1]));
                } else {
                    PIMW[k] = (BIM / AIM);
                    QIMW[k] = (DIMW / AIM);
                }
            }
            for (int k = Vert_Index_LL; k >= KSTART; k--) {
                WK_L[k] += (float)(relax * (PIMW[k] * WK_L[k + 1] + QIMW[k] - WK_L[k]));
            }
        }
    }
    });
}

/* ------------------------------------------------------------------------------------------ */
/* TKE and dissipation, k-eps (TKE-prognostic-microscale.cs:25-352)                            */
/* ------------------------------------------------------------------------------------------ */
void tke_ke(State &st, int IS, int JS, float Cmueh, float Ceps, float Ceps1, float Ceps2,
            float VISHMIN, float VISVMIN, float AREAxy, float building_Z0, float relax,
            float Ustern_factorX) {
    (void)relax;
    const int NII = st.nii, NJJ = st.njj;
    const float DXK = st.dxk, DYK = st.dyk;
    const float *DZK = st.dzk(), *HOKART = st.hokart();
    const float DXK_Rez = 1 / DXK, DYK_Rez = 1 / DYK;
    const float PotdTdz = st.p->potdtdz;
    oracle::for_slabs(2, NII, [&](int i1_lo, int i1_hi) {
    std::vector<float> PIMTURB(st.nk2), QIMTURB(st.nk2), PIMTDISS(st.nk2), QIMTDISS(st.nk2);
    for (int i1 = i1_lo; i1 < i1_hi; i1++) {
        for (int j1 = 2; j1 <= NJJ - 1; j1++) {
            int j = (JS == -1) ? NJJ - j1 + 1 : j1;
            int i = (IS == -1) ? NII - i1 + 1 : i1;
            if (st.advdom(i, j) != 1) continue;
            float *TURB_L = st.col(st.turb, i, j), *TDISS_L = st.col(st.tdiss, i, j);
            const float *TURBim = st.col(st.turb, i - 1, j), *TURBip = st.col(st.turb, i + 1, j);
            const float *TURBjm = st.col(st.turb, i, j - 1), *TURBjp = st.col(st.turb, i, j + 1);
            const float *TDISSim = st.col(st.tdiss, i - 1, j), *TDISSip = st.col(st.tdiss, i + 1, j);
            const float *TDISSjm = st.col(st.tdiss, i, j - 1), *TDISSjp = st.col(st.tdiss, i, j + 1);
            const float *UK_L = st.col(st.uk, i, j), *VK_L = st.col(st.vk, i, j), *WK_L = st.col(st.wk, i, j);
            const float *UKip = st.col(st.uk, i + 1, j), *UKjp = st.col(st.uk, i, j + 1);
            const float *UKipjp = st.col(st.uk, i + 1, j + 1), *UKjm = st.col(st.uk, i, j - 1);
            const float *UKipjm = st.col(st.uk, i + 1, j - 1), *VKjp = st.col(st.vk, i, j + 1);
            const float *VKip = st.col(st.vk, i + 1, j), *VKipjp = st.col(st.vk, i + 1, j + 1);
            const float *VKim = st.col(st.vk, i - 1, j), *VKimjp = st.col(st.vk, i - 1, j + 1);
            const float *WKip = st.col(st.wk, i + 1, j), *WKim = st.col(st.wk, i - 1, j);
            const float *WKjp = st.col(st.wk, i, j + 1), *WKjm = st.col(st.wk, i, j - 1);
            const float Z0 = st.z0(i, j);
            const int KKART = st.kkart(i, j);
            const int VI = st.vert_index[st.i2(i, j)];
            int KSTART = 1;
            if (st.cutk(i, j) == 0) KSTART = KKART + 1;

            for (int k = KSTART; k <= VI; k++) {
                const float DXKDZK = DXK * DZK[k], DYKDZK = DYK * DZK[k];
                const float DZK_Rez = 1 / DZK[k];
                const float zs = HOKART[k] - HOKART[KKART] - DZK[k] * 0.5f;
                float VIS = (float)std::sqrt((double)TURB_L[k]) * zs * Cmueh;
                VIS = net_min(VIS, 15);
                float DE = net_max(VIS, VISHMIN) * DYKDZK * DXK_Rez;
                float DW = DE;
                float DS = net_max(VIS, VISHMIN) * DXKDZK * DYK_Rez;
                float DN = DS;
                float DT = net_max(VIS, VISHMIN) * AREAxy * DZK_Rez;
                float DB = 0;
                float DTEPS = net_max(VIS / Ceps, VISVMIN) * AREAxy * DZK_Rez;
                float DBEPS = 0;
                if (k > KKART + 1) { DB = DT; DBEPS = DTEPS; }
                if ((st.advdom(i, j - 1) < 1) || (j == 2)) DS = 0;
                if ((st.advdom(i, j + 1) < 1) || (j == NJJ - 1)) DN = 0;
                if ((st.advdom(i - 1, j) < 1) || (i == 2)) DW = 0;
                if ((st.advdom(i + 1, j) < 1) || (i == NII - 1)) DE = 0;
                const float FE = UKip[k] * DYKDZK;
                const float FW = UK_L[k] * DYKDZK;
                const float FS = VK_L[k] * DXKDZK;
                const float FN = VKjp[k] * DXKDZK;
                const float FT = WK_L[k + 1] * AREAxy;
                float FB = 0;
                if (k > KKART + 1) FB = WK_L[k] * AREAxy;
                DE = net_max(DE, 0.0001f); DB = net_max(DB, 0.0001f);
                DW = net_max(DW, 0.0001f); DS = net_max(DS, 0.0001f);
                DN = net_max(DN, 0.0001f); DT = net_max(DT, 0.0001f);
                DBEPS = net_max(DBEPS, 0.0001f); DTEPS = net_max(DTEPS, 0.0001f);
                const float PE = std::fabs(FE / DE), PB = std::fabs(FB / DB);
                const float PW = std::fabs(FW / DW), PS = std::fabs(FS / DS);
                const float PN = std::fabs(FN / DN), PT = std::fabs(FT / DT);
                const float PBEPS = std::fabs(FN / DBEPS);        /* FN, not FB (:187) */
                const float PTEPS = std::fabs(FT / DTEPS);
                const float BIM = DT * net_max(0, pow5f(1 - 0.1f * PT)) + net_max(-FT, 0);
                const float CIM = DB * net_max(0, pow5f(1 - 0.1f * PB)) + net_max(FB, 0);
                const float AE1 = DE * net_max(0, pow5f(1 - 0.1f * PE)) + net_max(-FE, 0);
                const float AW1 = DW * net_max(0, pow5f(1 - 0.1f * PW)) + net_max(FW, 0);
                const float AS1 = DS * net_max(0, pow5f(1 - 0.1f * PS)) + net_max(FS, 0);
                const float AN1 = DN * net_max(0, pow5f(1 - 0.1f * PN)) + net_max(-FN, 0);
                const float BIMEPS = DT * net_max(0, pow5f(1 - 0.1f * PTEPS)) + net_max(-FT, 0);
                const float CIMEPS = DB * net_max(0, pow5f(1 - 0.1f * PBEPS)) + net_max(FB, 0);
                const float AIM = BIM + CIM + AW1 + AS1 + AE1 + AN1 + st.ap0[k];

                const float UX1 = UKip[k], UX2 = UK_L[k];
                const float VX1 = 0.5f * (VKip[k] + VKipjp[k]);
                const float VX2 = 0.5f * (VKim[k] + VKimjp[k]);
                const float WX1 = 0.5f * (WKip[k] + WKip[k + 1]);
                const float WX2 = 0.5f * (WKim[k] + WKim[k + 1]);
                const float UY1 = 0.5f * (UKjp[k] + UKipjp[k]);
                const float UY2 = 0.5f * (UKjm[k] + UKipjm[k]);
                const float VY1 = VKjp[k], VY2 = VK_L[k];
                const float WY1 = 0.5f * (WKjp[k] + WKjp[k + 1]);
                const float WY2 = 0.5f * (WKjm[k] + WKjm[k + 1]);
                const float DUDX = (UX1 - UX2) * DXK_Rez;
                const float DVDX = (VX1 - VX2) * DXK_Rez * 0.5f;
                const float DWDX = (WX1 - WX2) * DXK_Rez * 0.5f;
                const float DUDY = (UY1 - UY2) * DYK_Rez * 0.5f;
                const float DVDY = (VY1 - VY2) * DYK_Rez;
                const float DWDY = (WY1 - WY2) * DYK_Rez * 0.5f;
                float DUDZ = UK_L[k + 1] * DZK_Rez * 0.5f;
                float DVDZ = VK_L[k + 1] * DZK_Rez * 0.5f;
                float DWDZ = WK_L[k + 1] * DZK_Rez * 0.5f;
                if (k > KKART + 1) {
                    DUDZ = (UK_L[k + 1] - UK_L[k - 1]) * DZK_Rez * 0.5f;
                    DVDZ = (VK_L[k + 1] - VK_L[k - 1]) * DZK_Rez * 0.5f;
                    DWDZ = (WK_L[k + 1] - WK_L[k - 1]) * DZK_Rez * 0.5f;
                }
                const float PROTURB = (float)(VIS * AREAxy * DZK[k] *
                    (2 * pow2f(DUDX) + 2 * pow2f(DVDY) + 2 * pow2f(DWDZ) +
                     pow2f(DUDY + DVDX) + pow2f(DUDZ + DWDX) + pow2f(DVDZ + DWDY) - TDISS_L[k]));
                const float PROBOU = (float)(-PotdTdz * 9.81 / 283 * VIS * 1.35 * AREAxy * DZK[k]);
                const float DIMTURB = AW1 * TURBim[k] + AS1 * TURBjm[k] + AE1 * TURBip[k] + AN1 * TURBjp[k] +
                                      st.ap0[k] * TURB_L[k] + PROTURB + PROBOU;
                const float DIMTDISS = AW1 * TDISSim[k] + AS1 * TDISSjm[k] + AE1 * TDISSip[k] + AN1 * TDISSjp[k] +
                                       st.ap0[k] * TDISS_L[k] + (TDISS_L[k] / TURB_L[k] * (Ceps1 * PROTURB - Ceps2 * TDISS_L[k]));
                if (k > KKART + 1) {
                    PIMTURB[k] = (BIM / (AIM - CIM * PIMTURB[k - 1]));
                    QIMTURB[k] = ((DIMTURB + CIM * QIMTURB[k - 1]) / (AIM - CIM * PIMTURB[k - 1]));
                    PIMTDISS[k] = (BIMEPS / (AIM - CIMEPS * PIMTDISS[k - 1]));
                    QIMTDISS[k] = ((DIMTDISS + CIMEPS * QIMTDISS[k - 1]) / (AIM - CIMEPS * PIMTDISS[k - 1]));
                } else {
                    PIMTURB[k] = (BIM / AIM);
                    QIMTURB[k] = (DIMTURB / AIM);
                    PIMTDISS[k] = (BIMEPS / AIM);
                    QIMTDISS[k] = (DIMTDISS / AIM);
                }
            }

            for (int k = VI; k >= KSTART; k--) {                        /* :272-347 */
                if (KKART < k) {
                    float UstB = 0.01f;
                    if ((k == KKART + 1) && (st.cutk(i, j) == 0)) {
                        if ((double)Z0 >= (double)DZK[k] * 0.5) {
                            UstB = (float)(0.4 / std::log(((double)DZK[k] + (double)DZK[k + 1] * 0.5) / (double)Z0) *
                                           std::sqrt(pow2d(0.5 * (double)(UK_L[k + 1] + UKip[k + 1])) +
                                                     pow2d(0.5 * (double)(VK_L[k + 1] + VKjp[k + 1]))));
                            TURB_L[k] = (float)(3.33 * pow2f(UstB));
                            TDISS_L[k] = (float)(pow3f(UstB) / (((double)DZK[k] + (double)DZK[k + 1] * 0.5) * 0.4));
                        } else {
                            UstB = (float)(0.4 / std::log((double)DZK[k] * 0.5 / (double)Z0) *
                                           std::sqrt(pow2d(0.5 * (double)((UK_L[k + 1]) + UKip[k])) +
                                                     pow2d(0.5 * (double)((VK_L[k]) + VKjp[k]))));
                            TURB_L[k] = (float)(3.33 * pow2f(UstB));
                            TDISS_L[k] = (float)(pow3f(UstB) / ((double)DZK[k] * 0.5 * 0.4));
                        }
                    } else if ((k == KKART + 1) && (st.cutk(i, j) > 0)) {
                        UstB = st.ustern_obst[st.i2(i, j)] *
                               (float)std::sqrt(pow2d(0.5 * (double)(UK_L[k] + UKip[k])) + pow2d(0.5 * (double)(VK_L[k] + VKjp[k])));
                        TURB_L[k] = (float)(3.33 * pow2f(UstB));
                        TDISS_L[k] = (float)(pow3f(UstB) / ((double)DZK[k] * 0.5 * 0.4));
                    } else if ((k == st.kkart(i + 1, j) + 1) && (st.cutk(i + 1, j) > 0)) {
                        UstB = (float)((double)Ustern_factorX *
                                       std::sqrt(pow2d(0.5 * (double)(WK_L[k] + WK_L[k + 1])) + pow2d(0.5 * (double)(VK_L[k] + VKjp[k]))));
                        TURB_L[k] = (float)(3.33 * pow2f(UstB));
                        TDISS_L[k] = (float)(pow3f(UstB) / ((double)building_Z0 * 0.4));
                    } else if ((k == st.kkart(i - 1, j) + 1) && (st.cutk(i - 1, j) > 0)) {
                        UstB = (float)((double)Ustern_factorX *
                                       std::sqrt(pow2d(0.5 * (double)(WK_L[k] + WK_L[k + 1])) + pow2d(0.5 * (double)(VK_L[k] + VKjp[k]))));
                        TURB_L[k] = (float)(3.33 * pow2f(UstB));
                        TDISS_L[k] = (float)(pow3f(UstB) / ((double)building_Z0 * 0.4));
                    } else if ((k == st.kkart(i, j + 1) + 1) && (st.cutk(i, j + 1) > 0)) {
                        UstB = (float)((double)Ustern_factorX *
                                       std::sqrt(pow2d(0.5 * (double)(WK_L[k] + WK_L[k + 1])) + pow2d(0.5 * (double)(UK_L[k] + UKip[k]))));
                        TURB_L[k] = (float)(3.33 * pow2f(UstB));
                        TDISS_L[k] = (float)(pow3f(UstB) / ((double)building_Z0 * 0.4));
                    } else if ((k == st.kkart(i, j - 1) + 1) && (st.cutk(i, j - 1) > 0)) {
                        UstB = (float)((double)Ustern_factorX *
                                       std::sqrt(pow2d(0.5 * (double)(WK_L[k] + WK_L[k + 1])) + pow2d(0.5 * (double)(UK_L[k] + UKip[k]))));
                        TURB_L[k] = (float)(3.33 * pow2f(UstB));
                        TDISS_L[k] = (float)(pow3f(UstB) / ((double)building_Z0 * 0.4));
                    } else {
                        TURB_L[k] = PIMTURB[k] * TURB_L[k + 1] + QIMTURB[k];
                        TDISS_L[k] = PIMTDISS[k] * TDISS_L[k + 1] + QIMTDISS[k];
                    }
                    TURB_L[k] = (float)net_maxd((double)TURB_L[k], 0.001);
                    TDISS_L[k] = (float)net_maxd((double)TDISS_L[k], 0.0000001);
                }
            }
        }
    }
    });
}

}  // namespace oracle
