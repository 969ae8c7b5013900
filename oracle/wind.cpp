/*
 * wind.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of Zeitschleife.IntWindCalculate (Intwind.cs:31-197): the wind at a particle
 * position interpolated from the flow field (terrain: binary level search above AHMIN; flat with
 * buildings: linear level search) or, on flat terrain without buildings, the met profile with
 * MathF.Pow = the C library's powf.  Only tests/ and the CPU legs of bench.py load it.
 */
#include <cmath>
#include <cstdint>

#include "oracle_common.h"

namespace {

float (*volatile lib_powf)(float, float) = ::powf;

/* Intwind.cs:162-197 */
int BinarySearch(const float *hokart, int nkk, float Height) {
    int low = 1;
    int high = nkk;
    const int aQuarter = high >> 3;
    if (hokart[aQuarter] >= Height) high = aQuarter;
    else low = aQuarter;
    int mid = 0;
    while (low <= high) {
        mid = (low + high) >> 1;
        if (hokart[mid] >= Height) high = mid - 1;
        else low = mid + 1;
    }
    if (low > nkk) low = nkk;
    return low;
}

}  // namespace

/* fields: one situation, flat [NII+2][NJJ+2][NKK+2]; one call per particle as the reference */
extern "C" void oracle_wind_at(int nii, int njj, int nkk, const gral_wind_grid *g, const float *DZK,
                               const float *HOKART, const float *UK, const float *VK, const float *WK, int n,
                               const gral_particle *p, float *ux, float *uy, float *uz, int32_t *kidx) {
    const int nj2 = njj + 2, nk2 = nkk + 2;
    auto I3 = [&](int i, int j, int k) { return ((size_t)i * nj2 + j) * nk2 + k; };
    const float DXK = g->dxk, DYK = g->dyk;
    for (int q = 0; q < n; q++) {
        const int IndexI = p[q].i, IndexJ = p[q].j;
        const double xcoord = p[q].x, ycoord = p[q].y;
        const float zcoord = p[q].z, AHint = p[q].ahint;
        float UXint = 0, UYint = 0, UZint = 0;
        int IndexK = 0;
        if (g->terrain) {
            const float f1 = zcoord - g->ahmin;
            IndexK = BinarySearch(HOKART, nkk, f1);
            const float u1 = UK[I3(IndexI, IndexJ, IndexK)], u2 = UK[I3(IndexI + 1, IndexJ, IndexK)];
            UXint = (float)(u1 + (u2 - u1) / DXK * (xcoord - (g->ikooa + (IndexI - 1) * DXK)));
            const float v1 = VK[I3(IndexI, IndexJ, IndexK)], v2 = VK[I3(IndexI, IndexJ + 1, IndexK)];
            UYint = (float)(v1 + (v2 - v1) / DYK * (ycoord - (g->jkooa + (IndexJ - 1) * DYK)));
            const float w1 = WK[I3(IndexI, IndexJ, IndexK)], w2 = WK[I3(IndexI, IndexJ, IndexK + 1)];
            UZint = w1 + (w2 - w1) / DZK[IndexK] * (f1 - HOKART[IndexK - 1]);
        } else if (!g->buildings) {
            const gral_met *m = g->met;
            const int inumm = m->n_heights;
            const float *MH = m->measurement_height, *OU = m->obs_u, *OV = m->obs_v;
            const float ob = m->ob_length;
            float exponent, dumfac;
            if (zcoord <= MH[1]) {
                if (ob <= 0) exponent = oracle::net_max(0.35F - 0.4F * lib_powf(std::fabs(ob), -0.15F), 0.05F);
                else exponent = 0.56F * lib_powf(ob, -0.15F);
                dumfac = lib_powf(zcoord / MH[1], exponent);
                UXint = OU[1] * dumfac;
                UYint = OV[1] * dumfac;
            } else if (zcoord >= MH[inumm]) {
                if (inumm == 1) {
                    if (ob <= 0) exponent = oracle::net_max(0.35F - 0.4F * lib_powf(std::fabs(ob), -0.15F), 0.05F);
                    else exponent = 0.56F * lib_powf(ob, -0.15F);
                    dumfac = lib_powf(zcoord / MH[inumm], exponent);
                    UXint = OU[inumm] * dumfac;
                    UYint = OV[inumm] * dumfac;
                } else {
                    UXint = OU[inumm];
                    UYint = OV[inumm];
                }
            } else {
                int ipo = 1;
                for (int iprof = 1; iprof <= inumm; iprof++)
                    if (zcoord > MH[iprof]) ipo = iprof + 1;
                const float help = 1 / (MH[ipo] - MH[ipo - 1]) * (zcoord - MH[ipo - 1]);
                UXint = OU[ipo - 1] + (OU[ipo] - OU[ipo - 1]) * help;
                UYint = OV[ipo - 1] + (OV[ipo] - OV[ipo - 1]) * help;
            }
        } else {
            for (IndexK = 1; IndexK <= nkk; IndexK++)
                if (zcoord <= HOKART[IndexK]) break;
            if (IndexK > nkk) IndexK = nkk;
            const float u1 = UK[I3(IndexI, IndexJ, IndexK)], u2 = UK[I3(IndexI + 1, IndexJ, IndexK)];
            UXint = (float)(u1 + (u2 - u1) / DXK * (xcoord - (g->ikooa + (IndexI - 1) * DXK)));
            const float v1 = VK[I3(IndexI, IndexJ, IndexK)], v2 = VK[I3(IndexI, IndexJ + 1, IndexK)];
            UYint = (float)(v1 + (v2 - v1) / DYK * (ycoord - (g->jkooa + (IndexJ - 1) * DYK)));
            const float w1 = WK[I3(IndexI, IndexJ, IndexK)], w2 = WK[I3(IndexI, IndexJ, IndexK + 1)];
            UZint = w1 + (w2 - w1) / DZK[IndexK] * (zcoord + AHint - HOKART[IndexK - 1]);
        }
        ux[q] = UXint;
        uy[q] = UYint;
        uz[q] = UZint;
        kidx[q] = IndexK;
    }
}
