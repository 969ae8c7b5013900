/*
 * prep.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the flow-field set-up that GRAL runs before each prognostic solve, written
 * as the reference's loops in their sequential order: the prognostic sub-domains
 * (ReadGeometryAndDomains.cs:321-347), the flat-terrain initial field with KKART/AHK/KADVMAX
 * (MicroscaleFlat.cs:29-197) and its near-wall damping (:201-357), and the vegetation
 * rasterisation (ReadVegetation.cs:83-118).  MathF.Pow/Log and Math.Pow are the C library's
 * powf/logf/pow, which .NET calls for them on Linux, evaluated per cell as the reference does.
 * Only tests/ and the CPU legs of bench.py load it.  Parity unpinned (see oracle_common.h).
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "oracle_common.h"

namespace {

using oracle::net_max;

/* MathF.Pow / MathF.Log / Math.Pow: the C library calls */
float (*volatile lib_powf)(float, float) = ::powf;
float (*volatile lib_logf)(float) = ::logf;
double (*volatile lib_pow)(double, double) = ::pow;

}  // namespace

/* ReadGeometryAndDomains.cs:321-347 */
extern "C" void oracle_subdomains(int nii, int njj, float dxk, float dyk, int factor, const float *cutk,
                                  uint8_t *advdom) {
    const int nj2 = njj + 2;
    std::memset(advdom, 0, (size_t)(nii + 2) * nj2);
    for (int i = 1; i <= nii; i++)
        for (int j = 1; j <= njj; j++) {
            const float c = cutk[i * nj2 + j];
            if (c > 0) {
                const int iplus = (int)((float)factor * c / dxk);
                const int jplus = (int)((float)factor * c / dyk);
                for (int i1 = i - iplus; i1 <= i + iplus; i1++)
                    for (int j1 = j - jplus; j1 <= j + jplus; j1++)
                        if ((i1 <= nii) && (i1 >= 1) && (j1 <= njj) && (j1 >= 1)) advdom[i1 * nj2 + j1] = 1;
            }
        }
}

/* MicroscaleFlat.cs:29-197, then :201-357.  The field arrays must be zero on entry (they stand
 * for freshly allocated arrays; the solve keeps the entries this routine does not set at 0). */
extern "C" int oracle_flat_init(const gral_flat_grid *g, const float *CUTK, const float *DZK, const float *HOKART,
                                const uint8_t *ADVDOM, const gral_met *met, int16_t *KKART, float *AHK,
                                int32_t *kadvmax, gral_fields *f) {
    const int NII = g->nii, NJJ = g->njj, NKK = g->nkk, nj2 = NJJ + 2, nk2 = NKK + 2;
    const int inumm = met->n_heights;
    const float *MH = met->measurement_height, *OU = met->obs_u, *OV = met->obs_v;
    float *UK = f->uk, *VK = f->vk, *WK = f->wk;
    auto C2 = [&](int i, int j) { return (size_t)i * nj2 + j; };
    auto I3 = [&](int i, int j, int k) { return ((size_t)i * nj2 + j) * nk2 + k; };
    int KADVMAX = 1;
    for (int i = 1; i <= NII + 1; i++)
        for (int j = 1; j <= NJJ + 1; j++)
            for (int k = 1; k <= NKK; k++) {
                UK[I3(i, j, k)] = 0;
                VK[I3(i, j, k)] = 0;
                WK[I3(i, j, k)] = 0;
            }
    int KADVMAX1 = 1;
    for (int i = 1; i < NII + 1; i++) {
        for (int j = 1; j <= NJJ; j++) {
            AHK[C2(i, j)] = 0;
            KKART[C2(i, j)] = 0;
            float ObLength = met->ob_length;
            if (met->ol_column) ObLength = met->ol_column[C2(i, j)];
            for (int k = NKK; k >= 1; k--) {
                const float vertk = HOKART[k - 1] + DZK[k] * 0.5F;
                if (vertk > CUTK[C2(i, j)]) {
                    double UXint, UYint;
                    float exponent, dumfac;
                    if (vertk <= MH[1]) {
                        if (ObLength <= 0)
                            exponent = net_max(0.35F - 0.4F * lib_powf(std::fabs(ObLength), -0.15F), 0.05F);
                        else
                            exponent = 0.56F * lib_powf(ObLength, -0.15F);
                        dumfac = lib_powf(vertk / MH[1], exponent);
                        UXint = OU[1] * dumfac;
                        UYint = OV[1] * dumfac;
                    } else if (vertk > MH[inumm]) {
                        if (inumm == 1) {
                            if (ObLength <= 0)
                                exponent = net_max(0.35F - 0.4F * lib_powf(std::fabs(ObLength), -0.15F), 0.05F);
                            else
                                exponent = 0.56F * lib_powf(ObLength, -0.15F);
                            dumfac = lib_powf(vertk / MH[inumm], exponent);
                            UXint = OU[inumm] * dumfac;
                            UYint = OV[inumm] * dumfac;
                        } else {
                            UXint = OU[inumm];
                            UYint = OV[inumm];
                        }
                    } else {
                        int ipo = 1;
                        for (int iprof = 1; iprof <= inumm; iprof++)
                            if (vertk > MH[iprof]) ipo = iprof + 1;
                        UXint = OU[ipo - 1] + (OU[ipo] - OU[ipo - 1]) / (MH[ipo] - MH[ipo - 1]) * (vertk - MH[ipo - 1]);
                        UYint = OV[ipo - 1] + (OV[ipo] - OV[ipo - 1]) / (MH[ipo] - MH[ipo - 1]) * (vertk - MH[ipo - 1]);
                    }
                    UK[I3(i, j, k)] = (float)UXint;
                    VK[I3(i, j, k)] = (float)UYint;
                    if (i > 1)
                        if (vertk <= CUTK[C2(i - 1, j)]) UK[I3(i, j, k)] = 0;
                    if (j > 1)
                        if (vertk <= CUTK[C2(i, j - 1)]) VK[I3(i, j, k)] = 0;
                    UK[I3(NII + 1, j, k)] = UK[I3(NII, j, k)];
                    VK[I3(i, NJJ + 1, k)] = VK[I3(i, NJJ, k)];
                } else {
                    UK[I3(i, j, k)] = 0;
                    if (i < NII) UK[I3(i + 1, j, k)] = 0;
                    VK[I3(i, j, k)] = 0;
                    if (j < NJJ) VK[I3(i, j + 1, k)] = 0;
                    AHK[C2(i, j)] = net_max(HOKART[k], AHK[C2(i, j)]);
                    KKART[C2(i, j)] = (int16_t)std::max(k, (int)KKART[C2(i, j)]);
                    if (CUTK[C2(i, j)] > 0) KADVMAX1 = std::max((int)KKART[C2(i, j)], KADVMAX1);
                }
            }
        }
    }
    KADVMAX = std::max(KADVMAX, KADVMAX1);
    KADVMAX = std::min(NKK, KADVMAX + g->vert_cells_ff);
    *kadvmax = KADVMAX;

    if (g->near_wall) {
        const int IGEB = g->igeb;
        const float DXK = g->dxk, DYK = g->dyk;
        auto damp = [&](float entf, float &abmind) {
            if (entf <= 20) abmind *= 0.19F * lib_logf((entf + 0.5F) * 10);
        };
        for (int i = 1 + IGEB; i < NII - IGEB + 1; i++)
            for (int j = 1 + IGEB; j <= NJJ - IGEB; j++) {
                if (!(g->near_wall == 2 || ADVDOM[C2(i, j)] == 0)) continue;
                for (int k = 1; k < NKK; k++) {
                    float abmind = 1;
                    if (k > KKART[C2(i, j)]) {
                        const float vertk = HOKART[k - 1] + DZK[k] * 0.5F;
                        float entf = 21;
                        for (int ig = i - 1; ig >= i - IGEB; ig--)
                            if ((CUTK[C2(ig, j)] > 1) && (vertk <= AHK[C2(ig, j)])) { entf = std::fabs((i - ig) * DXK); break; }
                        damp(entf, abmind);
                        entf = 21;
                        for (int ig = i + 1; ig <= i + IGEB; ig++)
                            if ((CUTK[C2(ig, j)] > 1) && (vertk <= AHK[C2(ig, j)])) { entf = std::fabs((i - ig) * DXK); break; }
                        damp(entf, abmind);
                        entf = 21;
                        for (int jg = j + 1; jg <= j + IGEB; jg++)
                            if ((CUTK[C2(i, jg)] > 1) && (vertk <= AHK[C2(i, jg)])) { entf = std::fabs((j - jg) * DYK); break; }
                        damp(entf, abmind);
                        entf = 21;
                        for (int jg = j - 1; jg >= j - IGEB; jg--)
                            if ((CUTK[C2(i, jg)] > 1) && (vertk <= AHK[C2(i, jg)])) { entf = std::fabs((j - jg) * DYK); break; }
                        damp(entf, abmind);
                        auto diag = [&](int ig, int jg) {
                            const float a = (i - ig) * DXK, b = (j - jg) * DYK;
                            return std::sqrt(a * a + b * b);
                        };
                        entf = 21;
                        for (int ig = i + 1; ig <= i + IGEB; ig++) {
                            const int jg = j + ig - i;
                            if ((CUTK[C2(ig, jg)] > 1) && (vertk <= AHK[C2(ig, jg)])) { entf = diag(ig, jg); break; }
                        }
                        damp(entf, abmind);
                        entf = 21;
                        for (int ig = i - 1; ig >= i - IGEB; ig--) {
                            const int jg = j + ig - i;
                            if ((CUTK[C2(ig, jg)] > 1) && (vertk <= AHK[C2(ig, jg)])) { entf = diag(ig, jg); break; }
                        }
                        damp(entf, abmind);
                        entf = 21;
                        for (int ig = i + 1; ig <= i + IGEB; ig++) {
                            const int jg = j + i - ig;
                            if ((CUTK[C2(ig, jg)] > 1) && (vertk <= AHK[C2(ig, jg)])) { entf = diag(ig, jg); break; }
                        }
                        damp(entf, abmind);
                        entf = 21;
                        for (int ig = i - 1; ig >= i - IGEB; ig--) {
                            const int jg = j + i - ig;
                            if ((CUTK[C2(ig, jg)] > 1) && (vertk <= AHK[C2(ig, jg)])) { entf = diag(ig, jg); break; }
                        }
                        damp(entf, abmind);
                        UK[I3(i, j, k)] *= abmind;
                        VK[I3(i, j, k)] *= abmind;
                    }
                }
            }
    }
    return GRAL_OK;
}

/* ReadVegetation.cs:83-118, one processed coordinate line after the other.  veg and veg_mask must
 * be zero on entry; cov holds the values before reading. */
extern "C" void oracle_vegetation(int nii, int njj, int nkk, const int16_t *KKART, const float *DZK,
                                  const float *HOKART, int n, const gral_veg_point *pts, float *VEG,
                                  uint8_t *mask, float *COV) {
    const int nj2 = njj + 2, nk2 = nkk + 2;
    for (int q = 0; q < n; q++) {
        const gral_veg_point &p = pts[q];
        const int IXCUT = p.i, IYCUT = p.j;
        if ((IXCUT <= nii) && (IXCUT >= 1) && (IYCUT <= njj) && (IYCUT >= 1)) {
            const size_t c = (size_t)IXCUT * nj2 + IYCUT;
            if (p.drag) {
                mask[c] = 1;
                const int kk = KKART[c];
                for (int k = kk - 1; k < nkk; k++) {
                    if (k >= 0) {
                        const float MeanCellHeight = HOKART[k] - HOKART[kk] + DZK[k] * 0.5F;
                        if (MeanCellHeight < p.crown_height) {
                            if (MeanCellHeight >= 0 && MeanCellHeight < p.trunk_height)
                                VEG[c * nk2 + k] = (float)(0.3 * lib_pow(p.cov, 3) * p.trunk_lad);
                            else if (MeanCellHeight >= 0 && MeanCellHeight >= p.trunk_height)
                                VEG[c * nk2 + k] = (float)(0.3 * lib_pow(p.cov, 3) * p.crown_lad);
                        }
                    }
                }
            }
            COV[c] = (float)p.cov;
        }
    }
}
