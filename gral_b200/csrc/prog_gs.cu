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
// waits with a bounded spin on the predecessors' stamps, solves the column with lanes over k, and
// publishes its own stamp.  Values that another warp may write inside the same kernel (the swept
// field, the pressure row carry) are read with ld.global.cg so no stale L1 line is used.
#include "prog_common.cuh"
#include "prog_kernels.cuh"

namespace gral {

namespace {

constexpr int GS_WARPS = 4;      // warps per block of the wavefront kernels
constexpr int SM_ROWS = 5;       // shared rows per warp: A, B, C, D, phi

__device__ __forceinline__ void sweep_dir(int it, int &IS, int &JS) {
    // PrognosticFlowfield.cs:770-802
    const int m = it % 4;
    if (m == 0) { IS = -1; JS = 1; }
    else if (m == 1) { IS = -1; JS = -1; }
    else if (m == 2) { IS = 1; JS = -1; }
    else { IS = 1; JS = 1; }
}

// Task t -> (situation index, i1, j1): diagonal-major, then situation, then position.
__device__ __forceinline__ void decode_task(unsigned t, const SweepGeom &g, unsigned nact, int &s_idx,
                                            int &i1, int &j1) {
    int lo = 0, hi = g.ndiag;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if ((unsigned)g.diag_start[mid] * nact <= t) lo = mid; else hi = mid;
    }
    const int d = lo;
    const unsigned r = t - (unsigned)g.diag_start[d] * nact;
    const unsigned len = (unsigned)(g.diag_start[d + 1] - g.diag_start[d]);
    s_idx = (int)(r / len);
    const int pos = (int)(r % len);
    const int ioff = max(0, d - (g.nj - 1)) + pos;
    i1 = g.ia + ioff;
    j1 = g.ja + d - ioff;
}

// The wavefront task loop shared by every Gauss-Seidel phase.  body(s, i, j, IS, JS, first) runs
// one column with the whole warp; `first` is true for the first column of a sweep row.
template <int PHASE, bool REVERSE, class Body>
__device__ __forceinline__ void gs_tasks(const KArgs &a, const SweepGeom &g, Body &&body) {
    const int lane = threadIdx.x & 31;
    const unsigned nact = (unsigned)*a.nact;
    const unsigned total = (unsigned)g.diag_start[g.ndiag] * nact;
    unsigned int *ctr = a.counters + PHASE;
    for (;;) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(ctr, (unsigned)a.chunk);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) break;
        if (*(volatile int *)a.err != ERR_NONE) break;
        const unsigned end = min(total, base + (unsigned)a.chunk);
        for (unsigned t = base; t < end; ++t) {
            int s_idx, i1, j1;
            decode_task(t, g, nact, s_idx, i1, j1);
            const int s = a.act[s_idx];
            const int it = a.sit[s].it;
            int IS, JS;
            sweep_dir(it, IS, JS);
            if (REVERSE) { IS = -IS; JS = -JS; }
            const int i = (IS == 1) ? i1 : a.nii - i1 + 1;
            const int j = (JS == 1) ? j1 : a.njj - j1 + 1;
            const int stamp = it * 8 + PHASE;
            int *fl = a.flags + (size_t)s * a.ncols;
            int ok = 1;
            if (lane == 0) {
                if (i1 > g.ia) ok = wait_stamp(fl + (i - IS) * a.nj2 + j, stamp, a.err, a.wait_limit_ns);
                if (ok && j1 > g.ja) ok = wait_stamp(fl + i * a.nj2 + (j - JS), stamp, a.err, a.wait_limit_ns);
            }
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (ok && a.sit[s].active) body(s, i, j, IS, JS, i1 == g.ia);
            __threadfence();
            __syncwarp();
            if (lane == 0) st_release(fl + i * a.nj2 + j, stamp);
        }
    }
}

// Patankar power law of one face, Vector<float> association order (U-prognostic-microscale_1.cs:348-370).
__device__ __forceinline__ float pl_coef(float D, float Pe, float Fs) {
    const float in = 1.0f - 0.1f * Pe;
    return D * vmaxf(0.0f, in * in * in * in * in) + vmaxf(Fs, 0.0f);
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

// ------------------------------------------------------------------------------------------
// Pressure correction (PrognosticFlowfield.cs:723-901): divergence on the fly, downward Thomas
// sweep, upward back-substitution, DeltaUMax, DPMNEW += relaxp*DPM.  The reference zeroes DPM on
// the prognostic levels before the sweep (:755), so a column's not-yet-swept neighbours always
// contribute 0; they are not read.  The reference's PIMP/QIMP buffer lives per sweep row and is
// not cleared between columns, so the top level reads P/Q at VerticalIndex+1 left by an earlier
// column of the same row (:865-868); the row carry buffer reproduces that.
// ------------------------------------------------------------------------------------------
__device__ void pressure_column(const KArgs &a, int s, int i, int j, int IS, int JS, bool first,
                                float (*S)[KMAX_LEVELS]) {
    const int lane = threadIdx.x & 31;
    const int ks = a.ks, nj2 = a.nj2;
    float *rc = a.rowcarry + ((size_t)s * nj2 + j) * 2 * ks;
    if (first) {
        for (int k = lane; k < 2 * ks; k += 32) __stcg(rc + k, 0.0f);
        __threadfence_block();
        __syncwarp();
    }
    const int col = i * nj2 + j;
    const uint32_t fl = a.cflags[col];
    if (!(fl & F_ADV)) return;
    const ColMeta m = a.meta[col];
    const int KK = m.kkart, VI = m.vi;
    const SitDev &sd = a.sit[s];
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy, DT = sd.dtime;
    const size_t o = fidx(s, col, a.ncols, ks);
    const size_t oE = o + (size_t)nj2 * ks, oN = o + ks;
    const size_t oP_i = (IS == 1) ? o - (size_t)nj2 * ks : oE;   // swept neighbour in i
    const size_t oP_j = (JS == 1) ? o - ks : oN;                  // swept neighbour in j
    const float *UK = a.uk, *VK = a.vk, *WK = a.wk;
    const float *DZK = a.dzk;
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k <= KK || k > VI) continue;
        const float dz = DZK[k];
        float DIV;
        if (k > KK + 1)
            DIV = (UK[o + k] - UK[oE + k]) * DYK * dz + (VK[o + k] - VK[oN + k]) * DXK * dz +
                  (WK[o + k] - WK[o + k + 1]) * AREA;
        else
            DIV = (UK[o + k] - UK[oE + k]) * DYK * dz + (VK[o + k] - VK[oN + k]) * DXK * dz -
                  WK[o + k + 1] * AREA;
        const float pi = __ldcg(a.dpm + oP_i + k);
        const float pj = __ldcg(a.dpm + oP_j + k);
        const float si = (IS == 1) ? (pi + 0.0f) : (0.0f + pi);       // DPMim + DPMip
        const float sj = (JS == 1) ? (pj - 0.0f) : (0.0f - pj);       // DPMjm - DPMjp
        S[3][k] = DIV / DT + si / DXK * DYK * dz + sj / DYK * DXK * dz;
    }
    __syncwarp();
    if (lane == 0) {
        float P = __ldcg(rc + VI + 1), Q = __ldcg(rc + ks + VI + 1);
        for (int k = VI; k > KK; --k) {
            const float T = 1.0f / (a.app[k] - a.atp[k] * P);
            P = a.abp[k] * T;
            Q = (a.atp[k] * Q + S[3][k]) * T;
            S[1][k] = P;
            S[2][k] = Q;
        }
        float prev = 0.0f;                                            // DPM[KKART] is always 0
        for (int k = KK + 1; k <= VI; ++k) {
            prev = S[1][k] * prev + S[2][k];
            S[4][k] = prev;
        }
    }
    __syncwarp();
    float dmax = 0.0f;
    const int klo = max(KK, a.vi_min);
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k <= KK || k > VI) continue;
        const float temp = S[4][k];
        const double q = quantd((double)temp, sd.frund, sd.quantise);
        dmax = fmaxf(dmax, (float)fabs(0.0 - q));
        __stcg(a.dpm + o + k, temp);
        a.dpmnew[o + k] += a.relaxp * temp;
        if (k > klo) {
            __stcg(rc + k, S[1][k]);
            __stcg(rc + ks + k, S[2][k]);
        }
    }
    for (int d = 16; d > 0; d >>= 1) dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, d));
    if (lane == 0 && dmax > 0.0f) atomicMax(&a.sit[s].dumax_bits, __float_as_uint(dmax));
}

// ------------------------------------------------------------------------------------------
// U momentum, mixing-length model (U-prognostic-microscale_1.cs:96-529), one column per warp,
// lane = level.  The reference's SIMD chunking shows up only through ColMeta::kad (first level
// whose chunk base lies above KKART+1, where the extra eddy-viscosity terms are added,
// :453-470) and ColMeta::wc_lo..wc_hi (the chunk holding KKART+1, where the wall term is
// subtracted with a lane mask, :419-450).
// ------------------------------------------------------------------------------------------
__device__ void u1_column(const KArgs &a, int s, int i, int j, float (*S)[KMAX_LEVELS]) {
    const int lane = threadIdx.x & 31;
    const int ks = a.ks, nj2 = a.nj2;
    const int col = i * nj2 + j;
    const uint32_t fl = a.cflags[col];
    if (!(fl & F_ADV)) return;
    const ColMeta m = a.meta[col];
    const ColF cf = a.colf[col];
    const int KK = m.kkart, VI = m.vi, K0 = m.kstart;
    const SitDev &sd = a.sit[s];
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy, Cor = a.coriolis, UG = sd.ug;
    const float VISHMIN = a.vishmin;
    const size_t o = fidx(s, col, a.ncols, ks);
    const size_t dI = (size_t)nj2 * ks;
    const size_t oW = o - dI, oE = o + dI, oS = o - ks, oN = o + ks;
    const size_t oWS = oW - ks, oWN = oW + ks, oES = oE - ks, oEN = oE + ks;
    const float *UKS = a.uks, *VKS = a.vks, *WKS = a.wks, *DPMNEW = a.dpmnew, *VK = a.vk, *WK = a.wk;
    const float *UK = a.uk;
    const float *AP0 = a.ap0 + (size_t)s * ks;
    const float *DZK = a.dzk, *HOK = a.hokart;
    const float hokK = HOK[KK];
    const bool veg = (fl & F_VEG) != 0;
    const float *VEG = a.veg + (size_t)col * ks;
    const int kw = KK + 1;

    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k < K0 || k > VI) continue;
        const float dz = DZK[k];
        const float dxdz = DXK * dz, dydz = DYK * dz;
        const float uk = __ldcg(UK + o + k);
        float VIS = 0.0f;
        if (k > kw) {
            const float zs = HOK[k] - hokK - dz * 0.5f;
            float mixL = vminf(0.071f * zs, 100.0f);
            if (cf.cov > 0) mixL *= (1.0f - 0.99f * cf.cov);
            float in = (__ldcg(UK + o + k + 1) - __ldcg(UK + o + k - 1)) / (2.0f * dz);
            const float DUDZ = in * in;
            in = (VK[o + k + 1] - VK[o + k - 1]) / (2.0f * dz);
            const float DVDZ = in * in;
            VIS = vminf(mixL * mixL * sqrtf(0.5f * (DUDZ + DVDZ)), 15.0f);
        }
        float DE = vmaxf(VIS, VISHMIN) * dydz / DXK;
        float DW = DE;
        float DS = vmaxf(VIS, VISHMIN) * dxdz / DYK;
        float DN = DS;
        float DT = vmaxf(VIS, VISHMIN) * AREA / dz;
        float DB = (k > kw) ? DT : 0.0f;
        if (fl & F_BS) DS = 0.0f;
        if (fl & F_BN) DN = 0.0f;
        if (fl & F_BW) DW = 0.0f;
        if (fl & F_BE) DE = 0.0f;
        const float uks = UKS[o + k], vks = VKS[o + k], wks = WKS[o + k];
        const float uksW = UKS[oW + k], vksW = VKS[oW + k], vksWS = VKS[oWS + k];
        const float vksS = VKS[oS + k], vksWN = VKS[oWN + k], vksN = VKS[oN + k], wksW = WKS[oW + k];
        const float FE = uks * dydz;
        const float FW = uksW * dydz;
        const float FS = 0.25f * (vksW + vks + vksWS + vksS) * dxdz;
        const float FN = 0.25f * (vksW + vks + vksWN + vksN) * dxdz;
        const float FT = 0.25f * (wksW + wks + WKS[oW + k + 1] + WKS[o + k + 1]) * AREA;
        const float FB = (k > kw) ? 0.25f * (wksW + wks + WKS[oW + k - 1] + WKS[o + k - 1]) * AREA : 0.0f;
        DE = vmaxf(DE, 0.0001f); DB = vmaxf(DB, 0.0001f); DW = vmaxf(DW, 0.0001f);
        DS = vmaxf(DS, 0.0001f); DN = vmaxf(DN, 0.0001f); DT = vmaxf(DT, 0.0001f);
        const float BIM = pl_coef(DT, fabsf(FT / DT), -FT);
        const float CIM = pl_coef(DB, fabsf(FB / DB), FB);
        const float AE1 = pl_coef(DE, fabsf(FE / DE), -FE);
        const float AW1 = pl_coef(DW, fabsf(FW / DW), FW);
        const float AS1 = pl_coef(DS, fabsf(FS / DS), FS);
        const float AN1 = pl_coef(DN, fabsf(FN / DN), -FN);
        const float ap0 = AP0[k];
        const float AIM = BIM + CIM + AW1 + AS1 + AE1 + AN1 + ap0;
        const float DDPX = DPMNEW[oW + k] - DPMNEW[o + k];
        const float ukW = __ldcg(UK + oW + k), ukE = __ldcg(UK + oE + k);
        const float ukS = __ldcg(UK + oS + k), ukN = __ldcg(UK + oN + k);
        float DIM;
        if (veg) {
            const float in2 = 0.5f * (vksW + vks), in = 0.5f * (uksW + uks);
            const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.01f);
            DIM = AW1 * ukW + AS1 * ukS + AE1 * ukE + AN1 * ukN + ap0 * 0.5f * (uksW + uks) + DDPX * dydz +
                  (Cor * (UG - uk) - VEG[k - 1] * uk * wh) * AREA * dz;
        } else {
            DIM = AW1 * ukW + AS1 * ukS + AE1 * ukE + AN1 * ukN + ap0 * 0.5f * (uksW + uks) + DDPX * dydz +
                  Cor * (UG - uk) * AREA * dz;
        }
        if (k >= m.wc_lo && k <= m.wc_hi) {                       // wall chunk, :419-450
            const float in = 0.5f * (uksW + uks), in2 = 0.5f * (vksW + vks);
            const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.1f);
            float Ust;
            if (fl & F_CUTKLT1) {
                if (fl & F_Z0GE) {
                    const int ind = kw + 1;
                    const float a1 = 0.5f * ((UKS[oW + ind]) + UKS[o + ind]);
                    const float b1 = 0.5f * ((VKS[oW + ind]) + VKS[o + ind]);
                    Ust = cf.help_t * sqrtf(a1 * a1 + b1 * b1);
                } else {
                    const float a1 = 0.5f * (UKS[oW + kw] + UKS[o + kw]), b1 = 0.5f * (VKS[oW + kw] + VKS[o + kw]);
                    Ust = cf.help_t * vmaxf(sqrtf(a1 * a1 + b1 * b1), 0.1f);
                }
            } else {
                const float a1 = 0.5f * (UKS[oW + kw] + UKS[o + kw]), b1 = 0.5f * (VKS[oW + kw] + VKS[o + kw]);
                Ust = cf.help_o * vmaxf(sqrtf(a1 * a1 + b1 * b1), 0.1f);
            }
            const float m2 = (k == kw) ? 1.0f : 0.0f;
            DIM -= uk / wh * (Ust * Ust) * AREA * m2;
        }
        if (k >= m.kad) {                                          // extra eddy-viscosity terms
            const float DUDXE = (ukE - uk) * dydz;
            const float DUDXW = (uk - ukW) * dydz;
            const float DVDXN = (0.5f * (VKS[oEN + k] + vksN) - 0.5f * (vksN + vksWN)) * dxdz;
            const float DVDXS = (0.5f * (VKS[oES + k] + vksS) - 0.5f * (vksS + vksWS)) * dxdz;
            const float DWDXT = (0.5f * (WK[oE + k] + wks) - 0.5f * (wks + wksW)) * AREA;
            const float wksB = WKS[o + k - 1];
            const float DWDXB = (0.5f * (WK[oE + k - 1] + wksB) - 0.5f * (wksB + WKS[oW + k - 1])) * AREA;
            DIM += VIS / DXK * (DUDXE - DUDXW + DVDXN - DVDXS + DWDXT - DWDXB);
        }
        S[0][k] = AIM; S[1][k] = BIM; S[2][k] = CIM; S[3][k] = DIM; S[4][k] = uk;
    }
    if (lane == 0) S[4][VI + 1] = __ldcg(UK + o + VI + 1);
    __syncwarp();
    if (lane == 0) thomas_relax(S, K0, KK, VI, m.kkm_u, a.relax);
    __syncwarp();
    float *UKw = a.uk;
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k >= K0 && k <= VI && m.kkm_u < k) __stcg(UKw + o + k, S[4][k]);
    }
}

// ------------------------------------------------------------------------------------------
// V momentum, mixing-length model (V-prognostic-microscale_1.cs:94-524), swept with (-IS,-JS).
// ------------------------------------------------------------------------------------------
__device__ void v1_column(const KArgs &a, int s, int i, int j, float (*S)[KMAX_LEVELS]) {
    const int lane = threadIdx.x & 31;
    const int ks = a.ks, nj2 = a.nj2;
    const int col = i * nj2 + j;
    const uint32_t fl = a.cflags[col];
    if (!(fl & F_ADV)) return;
    const ColMeta m = a.meta[col];
    const ColF cf = a.colf[col];
    const int KK = m.kkart, VI = m.vi, K0 = m.kstart;
    const SitDev &sd = a.sit[s];
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy, Cor = a.coriolis, VG = sd.vg;
    const float VISHMIN = a.vishmin;
    const size_t o = fidx(s, col, a.ncols, ks);
    const size_t dI = (size_t)nj2 * ks;
    const size_t oW = o - dI, oE = o + dI, oS = o - ks, oN = o + ks;
    const size_t oWS = oW - ks, oWN = oW + ks, oES = oE - ks, oEN = oE + ks;
    const float *UKS = a.uks, *VKS = a.vks, *WKS = a.wks, *DPMNEW = a.dpmnew, *UK = a.uk, *WK = a.wk;
    const float *VK = a.vk;
    const float *AP0 = a.ap0 + (size_t)s * ks;
    const float *DZK = a.dzk, *HOK = a.hokart;
    const float hokK = HOK[KK];
    const bool veg = (fl & F_VEG) != 0;
    const float *VEG = a.veg + (size_t)col * ks;
    const int kw = KK + 1;

    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k < K0 || k > VI) continue;
        const float dz = DZK[k];
        const float dxdz = DXK * dz, dydz = DYK * dz;
        const float vk = __ldcg(VK + o + k);
        float VIS = 0.0f;
        if (k > kw) {
            const float zs = HOK[k] - hokK - dz * 0.5f;
            float mixL = vminf(0.071f * zs, 100.0f);
            if (cf.cov > 0) mixL *= (1.0f - 0.99f * cf.cov);
            float in = (UK[o + k + 1] - UK[o + k - 1]) / (2.0f * dz);
            const float DUDZ = in * in;
            in = (__ldcg(VK + o + k + 1) - __ldcg(VK + o + k - 1)) / (2.0f * dz);
            const float DVDZ = in * in;
            VIS = vminf(mixL * mixL * sqrtf(0.5f * (DUDZ + DVDZ)), 15.0f);
        }
        float DE = vmaxf(VIS, VISHMIN) * dydz / DXK;
        float DW = DE;
        float DS = vmaxf(VIS, VISHMIN) * dxdz / DYK;
        float DN = DS;
        float DT = vmaxf(VIS, VISHMIN) * AREA / dz;
        float DB = (k > kw) ? DT : 0.0f;
        if (fl & F_BS) DS = 0.0f;
        if (fl & F_BN) DN = 0.0f;
        if (fl & F_BW) DW = 0.0f;
        if (fl & F_BE) DE = 0.0f;
        const float uks = UKS[o + k], vks = VKS[o + k], wks = WKS[o + k];
        const float uksE = UKS[oE + k], uksS = UKS[oS + k], uksES = UKS[oES + k];
        const float uksW = UKS[oW + k], vksW = VKS[oW + k], uksWS = UKS[oWS + k];
        const float vksS = VKS[oS + k], wksS = WKS[oS + k], wksB = WKS[o + k - 1];
        const float FE = 0.25f * (uks + uksE + uksS + uksES) * dydz;
        const float FW = 0.25f * (uks + uksW + uksS + uksWS) * dydz;
        const float FS = vksS * dxdz;
        const float FN = vks * dxdz;
        const float FT = 0.25f * (wksS + wks + WKS[oS + k + 1] + WKS[o + k + 1]) * AREA;
        const float FB = (k > kw) ? 0.25f * (wksS + wks + WKS[oS + k - 1] + wksB) * AREA : 0.0f;
        DE = vmaxf(DE, 0.0001f); DB = vmaxf(DB, 0.0001f); DW = vmaxf(DW, 0.0001f);
        DS = vmaxf(DS, 0.0001f); DN = vmaxf(DN, 0.0001f); DT = vmaxf(DT, 0.0001f);
        const float BIM = pl_coef(DT, fabsf(FT / DT), -FT);
        const float CIM = pl_coef(DB, fabsf(FB / DB), FB);
        const float AE1 = pl_coef(DE, fabsf(FE / DE), -FE);
        const float AW1 = pl_coef(DW, fabsf(FW / DW), FW);
        const float AS1 = pl_coef(DS, fabsf(FS / DS), FS);
        const float AN1 = pl_coef(DN, fabsf(FN / DN), -FN);
        const float ap0 = AP0[k];
        const float AIM = BIM + CIM + AW1 + AS1 + AE1 + AN1 + ap0;
        const float DDPY = DPMNEW[oS + k] - DPMNEW[o + k];
        const float vkN = __ldcg(VK + oN + k), vkS = __ldcg(VK + oS + k);
        const float vkW = __ldcg(VK + oW + k), vkE = __ldcg(VK + oE + k);
        float DIM;
        if (veg) {
            const float in2 = 0.5f * (vksW + vks), in = 0.5f * (uksW + uks);
            const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.01f);
            DIM = AW1 * vkW + AS1 * vkS + AE1 * vkE + AN1 * vkN + ap0 * 0.5f * (vksS + vks) + DDPY * dxdz +
                  (Cor * (VG - vk) - VEG[k - 1] * vk * wh) * AREA * dz;
        } else {
            DIM = AW1 * vkW + AS1 * vkS + AE1 * vkE + AN1 * vkN + ap0 * 0.5f * (vksS + vks) + DDPY * dxdz +
                  Cor * (VG - vk) * AREA * dz;
        }
        if (k >= m.wc_lo && k <= m.wc_hi) {                       // wall chunk, :437-467
            const float in = 0.5f * (uksW + uks), in2 = 0.5f * (vksW + vks);
            const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.1f);
            float Ust;
            if (fl & F_CUTKLT1) {
                if (fl & F_Z0GE) {
                    const int ind = kw + 1;
                    const float a1 = 0.5f * ((UKS[oW + ind]) + UKS[o + ind]);
                    const float b1 = 0.5f * ((VKS[oW + ind]) + VKS[o + ind]);
                    Ust = cf.help_t * sqrtf(a1 * a1 + b1 * b1);
                } else {
                    const float a1 = 0.5f * (UKS[oW + kw] + UKS[o + kw]), b1 = 0.5f * (VKS[oW + kw] + VKS[o + kw]);
                    Ust = cf.help_t * vmaxf(sqrtf(a1 * a1 + b1 * b1), 0.1f);
                }
            } else {
                const float a1 = 0.5f * (UKS[oW + kw] + UKS[o + kw]), b1 = 0.5f * (VKS[oW + kw] + VKS[o + kw]);
                Ust = cf.help_o * vmaxf(sqrtf(a1 * a1 + b1 * b1), 0.1f);
            }
            const float m2 = (k == kw) ? 1.0f : 0.0f;
            DIM -= vk / wh * (Ust * Ust) * AREA * m2;
        }
        if (k >= m.kad) {                                          // extra eddy-viscosity terms, :470-488
            const float DVDYN = (vkN - vk) * dxdz;
            const float DVDYS = (vk - vkS) * dxdz;
            const float DUDYE = (0.5f * (UKS[oEN + k] + uksE) - 0.5f * (uksE + uksES)) * dxdz;
            const float DUDYW = (0.5f * (UKS[oWN + k] + uksW) - 0.5f * (uksW + uksWS)) * dxdz;
            const float DWDYT = (0.5f * (WK[oN + k] + wks) - 0.5f * (wks + wksS)) * AREA;
            const float DWDYB = (0.5f * (WK[oN + k - 1] + wksB) - 0.5f * (wksB + wksS)) * AREA;
            DIM += VIS / DXK * (DUDYE - DUDYW + DVDYN - DVDYS + DWDYT - DWDYB);
        }
        S[0][k] = AIM; S[1][k] = BIM; S[2][k] = CIM; S[3][k] = DIM; S[4][k] = vk;
    }
    if (lane == 0) S[4][VI + 1] = __ldcg(VK + o + VI + 1);
    __syncwarp();
    if (lane == 0) thomas_relax(S, K0, KK, VI, m.kkm_v, a.relax);
    __syncwarp();
    float *VKw = a.vk;
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k >= K0 && k <= VI && m.kkm_v < k) __stcg(VKw + o + k, S[4][k]);
    }
}

// ------------------------------------------------------------------------------------------
// W momentum, mixing-length model (W-prognostic-microscale_1.cs:93-453).  No wall term; the
// back-substitution runs over every level from KSTART, buildings included (:444-448).
// ------------------------------------------------------------------------------------------
__device__ void w1_column(const KArgs &a, int s, int i, int j, float (*S)[KMAX_LEVELS]) {
    const int lane = threadIdx.x & 31;
    const int ks = a.ks, nj2 = a.nj2;
    const int col = i * nj2 + j;
    const uint32_t fl = a.cflags[col];
    if (!(fl & F_ADV)) return;
    const ColMeta m = a.meta[col];
    const ColF cf = a.colf[col];
    const int KK = m.kkart, VI = m.vi, K0 = m.kstart;
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy;
    const float VISHMIN = a.vishmin;
    const size_t o = fidx(s, col, a.ncols, ks);
    const size_t dI = (size_t)nj2 * ks;
    const size_t oW = o - dI, oE = o + dI, oS = o - ks, oN = o + ks;
    const float *UKS = a.uks, *VKS = a.vks, *WKS = a.wks, *DPMNEW = a.dpmnew, *UK = a.uk, *VK = a.vk;
    const float *WK = a.wk;
    const float *AP0 = a.ap0 + (size_t)s * ks;
    const float *DZK = a.dzk, *HOK = a.hokart;
    const float hokK = HOK[KK];
    const bool veg = (fl & F_VEG) != 0;
    const float *VEG = a.veg + (size_t)col * ks;
    const int kw = KK + 1;

    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k < K0 || k > VI) continue;
        const float dz = DZK[k];
        const float dxdz = DXK * dz, dydz = DYK * dz;
        const float uks = UKS[o + k], vks = VKS[o + k], wks = WKS[o + k];
        const float uksM = UKS[o + k - 1], vksM = VKS[o + k - 1];
        const float wk = __ldcg(WK + o + k);
        float VIS = 0.0f;
        if (k > kw) {
            const float zs = HOK[k] - hokK - dz * 0.5f;
            float mixL = vminf(0.071f * zs, 100.0f);
            if (cf.cov > 0) mixL *= (1.0f - 0.99f * cf.cov);
            float in = (UK[o + k + 1] - UK[o + k - 1]) / (2.0f * dz);
            const float DUDZ = in * in;
            in = (VK[o + k + 1] - VK[o + k - 1]) / (2.0f * dz);
            const float DVDZ = in * in;
            VIS = vminf(mixL * mixL * sqrtf(0.5f * (DUDZ + DVDZ)), 15.0f);
        }
        float DE = vmaxf(VIS, VISHMIN) * dydz / DXK;
        float DW = DE;
        float DS = vmaxf(VIS, VISHMIN) * dxdz / DYK;
        float DN = DS;
        float DT = vmaxf(VIS, VISHMIN) * AREA / dz;
        float DB = (k > kw) ? DT : 0.0f;
        if (fl & F_BS) DS = 0.0f;
        if (fl & F_BN) DN = 0.0f;
        if (fl & F_BW) DW = 0.0f;
        if (fl & F_BE) DE = 0.0f;
        const float uksW = UKS[oW + k], uksWB = UKS[oW + k - 1];
        const float vksS = VKS[oS + k], vksSB = VKS[oS + k - 1];
        const float FE = 0.25f * (uks + UKS[oE + k] + uksM + UKS[oE + k - 1]) * dydz;
        const float FW = 0.25f * (uks + uksW + uksM + uksWB) * dydz;
        const float FS = 0.25f * (vks + vksS + vksM + vksSB) * dxdz;
        const float FN = 0.25f * (vks + VKS[oN + k] + vksM + VKS[oN + k - 1]) * dxdz;
        const float FT = wks * AREA;
        const float wksB = WKS[o + k - 1];
        const float FB = (k > kw) ? wksB * AREA : 0.0f;
        DE = vmaxf(DE, 0.0001f); DB = vmaxf(DB, 0.0001f); DW = vmaxf(DW, 0.0001f);
        DS = vmaxf(DS, 0.0001f); DN = vmaxf(DN, 0.0001f); DT = vmaxf(DT, 0.0001f);
        const float BIM = pl_coef(DT, fabsf(FT / DT), -FT);
        const float CIM = pl_coef(DB, fabsf(FB / DB), FB);
        const float AE1 = pl_coef(DE, fabsf(FE / DE), -FE);
        const float AW1 = pl_coef(DW, fabsf(FW / DW), FW);
        const float AS1 = pl_coef(DS, fabsf(FS / DS), FS);
        const float AN1 = pl_coef(DN, fabsf(FN / DN), -FN);
        const float ap0 = AP0[k];
        const float AIM = BIM + CIM + AW1 + AS1 + AE1 + AN1 + ap0;
        const float DDPZ = DPMNEW[o + k - 1] - DPMNEW[o + k];
        const float wkW = __ldcg(WK + oW + k), wkS = __ldcg(WK + oS + k);
        const float wkE = __ldcg(WK + oE + k), wkN = __ldcg(WK + oN + k);
        float DIM;
        if (veg) {
            const float in2 = 0.5f * (vksS + vks), in = 0.5f * (uksW + uks);
            const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.01f);
            DIM = AW1 * wkW + AS1 * wkS + AE1 * wkE + AN1 * wkN + ap0 * 0.5f * (wksB + wks) + DDPZ * AREA -
                  VEG[k - 1] * wk * wh * AREA * dz;
        } else {
            DIM = AW1 * wkW + AS1 * wkS + AE1 * wkE + AN1 * wkN + ap0 * 0.5f * (wksB + wks) + DDPZ * AREA;
        }
        if (k >= m.kad) {                                          // extra eddy-viscosity terms, :376-402
            const float DUDZE = (0.5f * (UKS[o + k + 1] + uks) - 0.5f * (uks + uksM)) * dydz;
            const float DUDZW = (0.5f * (UKS[oW + k + 1] + uksW) - 0.5f * (uksW + uksWB)) * dydz;
            const float DVDZN = (0.5f * (VKS[o + k + 1] + vks) - 0.5f * (vks + vksM)) * dxdz;
            const float DVDZS = (0.5f * (VKS[oS + k + 1] + vksS) - 0.5f * (vksS + vksSB)) * dxdz;
            const float DWDZT = (__ldcg(WK + o + k + 1) - wk) * AREA;
            const float DWDZB = (wk - __ldcg(WK + o + k - 1)) * AREA;
            DIM += VIS / dz * (DUDZE - DUDZW + DVDZN - DVDZS + DWDZT - DWDZB);
        }
        S[0][k] = AIM; S[1][k] = BIM; S[2][k] = CIM; S[3][k] = DIM; S[4][k] = wk;
    }
    if (lane == 0) S[4][VI + 1] = __ldcg(WK + o + VI + 1);
    __syncwarp();
    if (lane == 0) thomas_relax(S, K0, KK, VI, -32768, a.relax);
    __syncwarp();
    float *WKw = a.wk;
    for (int r = 0; r < 2; ++r) {
        const int k = lane + 32 * r;
        if (k >= K0 && k <= VI) __stcg(WKw + o + k, S[4][k]);
    }
}

__global__ void __launch_bounds__(GS_WARPS * 32) k_pressure(KArgs a, SweepGeom g) {
    __shared__ float sm[GS_WARPS][SM_ROWS][KMAX_LEVELS];
    float (*S)[KMAX_LEVELS] = sm[threadIdx.x >> 5];
    gs_tasks<PH_PRESSURE, false>(a, g, [&](int s, int i, int j, int IS, int JS, bool first) {
        pressure_column(a, s, i, j, IS, JS, first, S);
    });
}

__global__ void __launch_bounds__(GS_WARPS * 32) k_mom_u1(KArgs a, SweepGeom g) {
    __shared__ float sm[GS_WARPS][SM_ROWS][KMAX_LEVELS];
    float (*S)[KMAX_LEVELS] = sm[threadIdx.x >> 5];
    gs_tasks<PH_U, false>(a, g, [&](int s, int i, int j, int, int, bool) { u1_column(a, s, i, j, S); });
}

__global__ void __launch_bounds__(GS_WARPS * 32) k_mom_v1(KArgs a, SweepGeom g) {
    __shared__ float sm[GS_WARPS][SM_ROWS][KMAX_LEVELS];
    float (*S)[KMAX_LEVELS] = sm[threadIdx.x >> 5];
    gs_tasks<PH_V, true>(a, g, [&](int s, int i, int j, int, int, bool) { v1_column(a, s, i, j, S); });
}

__global__ void __launch_bounds__(GS_WARPS * 32) k_mom_w1(KArgs a, SweepGeom g) {
    __shared__ float sm[GS_WARPS][SM_ROWS][KMAX_LEVELS];
    float (*S)[KMAX_LEVELS] = sm[threadIdx.x >> 5];
    gs_tasks<PH_W, false>(a, g, [&](int s, int i, int j, int, int, bool) { w1_column(a, s, i, j, S); });
}

}  // namespace

int gs_block_threads() { return GS_WARPS * 32; }

cudaError_t gs_occupancy(int kind, int *blocks_per_sm) {
    switch (kind) {
        case PH_PRESSURE: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_pressure, GS_WARPS * 32, 0);
        case PH_U: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_mom_u1, GS_WARPS * 32, 0);
        case PH_V: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_mom_v1, GS_WARPS * 32, 0);
        default: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_mom_w1, GS_WARPS * 32, 0);
    }
}

void launch_pressure(const KArgs &a, const SweepGeom &g, int grid, cudaStream_t st) {
    k_pressure<<<grid, GS_WARPS * 32, 0, st>>>(a, g);
}
void launch_mom_ml(int comp, const KArgs &a, const SweepGeom &g, int grid, cudaStream_t st) {
    if (comp == 0) k_mom_u1<<<grid, GS_WARPS * 32, 0, st>>>(a, g);
    else if (comp == 1) k_mom_v1<<<grid, GS_WARPS * 32, 0, st>>>(a, g);
    else k_mom_w1<<<grid, GS_WARPS * 32, 0, st>>>(a, g);
}

}  // namespace gral
