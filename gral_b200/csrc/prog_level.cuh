// prog_level.cuh -- per-cell arithmetic of the SIMPLE phases, shared by the two kernel families:
//
//   * plain family (few situations): one warp per column, lane = level k, serial Thomas sweep on
//     lane 0 through shared memory;
//   * batched family (32 situations per group): one warp per column of a group, lane = situation,
//     every lane runs its own k loop and Thomas sweep.
//
// The functions below evaluate one (situation, column, level) cell in exactly the reference's
// operation order; an accessor `Acc` hides the two device layouts:
//   slab        element (s, col, k) at ((s*ncols + col)*KS + k)
//   interleaved element (s, col, k) at (((s/32)*ncols + col)*KS + k)*32 + s%32
#pragma once

#include "prog_common.cuh"

namespace gral {

template <bool IL>
struct Acc {
    size_t base;   // element (s, col, 0)
    size_t cs;     // elements between neighbouring columns (KS or KS*32)
    __device__ __forceinline__ size_t at(long long dc, int k) const {
        return (size_t)((long long)base + dc * (long long)cs) + (size_t)k * (IL ? 32u : 1u);
    }
};

template <bool IL>
__device__ __forceinline__ Acc<IL> make_acc(const KArgs &a, int s, int col) {
    Acc<IL> x;
    if (IL) {
        x.base = (((size_t)(s >> 5) * a.ncols + col) * a.ks) * 32 + (s & 31);
        x.cs = (size_t)a.ks * 32;
    } else {
        x.base = ((size_t)s * a.ncols + col) * a.ks;
        x.cs = a.ks;
    }
    return x;
}

struct ColCtx {
    int col, i, j, nj2;
    int KK, VI, K0, kad, wlo, whi, kkm_u, kkm_v;
    uint32_t fl;
    ColF cf;
    float hokK;
};

__device__ __forceinline__ ColCtx make_col(const KArgs &a, int i, int j) {
    ColCtx c;
    c.nj2 = a.nj2;
    c.i = i;
    c.j = j;
    c.col = i * a.nj2 + j;
    const ColMeta m = a.meta[c.col];
    c.KK = m.kkart; c.VI = m.vi; c.K0 = m.kstart; c.kad = m.kad;
    c.wlo = m.wc_lo; c.whi = m.wc_hi; c.kkm_u = m.kkm_u; c.kkm_v = m.kkm_v;
    c.fl = a.cflags[c.col];
    c.cf = a.colf[c.col];
    c.hokK = a.hokart[c.KK];
    return c;
}

struct SitCtx {
    float ug, vg, dtime;
    double frund;
    int quant;
    const float *ap0;
};

__device__ __forceinline__ SitCtx make_sit(const KArgs &a, int s) {
    SitCtx q;
    const SitDev &S = a.sit[s];
    q.ug = S.ug; q.vg = S.vg; q.dtime = S.dtime; q.frund = S.frund; q.quant = S.quantise;
    q.ap0 = a.ap0 + (size_t)s * a.ks;
    return q;
}

// Residual key of one pressure cell.  The reference's DeltaUMax is the float of the maximum over
// cells of |0 - ConvToInt(temp*Frund)/Frund| (PrognosticFlowfield.cs:880); division by the positive
// constant Frund is monotonic, so the maximum is taken over the integers |ConvToInt(temp*Frund)|
// and divided once per iteration (k_bookkeeping).  Without quantisation the key is the bit pattern
// of |temp| (non-negative floats order like their bits).
__device__ __forceinline__ unsigned residual_key(float temp, const SitCtx &sc) {
    if (sc.quant) {
        const long long n = conv_to_int((double)temp * sc.frund);
        return (unsigned)(n < 0 ? -n : n);
    }
    return __float_as_uint(fabsf(temp));
}

struct Coef {
    float A, B, C, D, phi;
};

// Patankar power law of one face, Vector<float> association order (U-prognostic-microscale_1.cs:348-370).
__device__ __forceinline__ float pl_coef(float D, float Pe, float Fs) {
    const float in = 1.0f - 0.1f * Pe;
    return D * vmaxf(0.0f, in * in * in * in * in) + vmaxf(Fs, 0.0f);
}

// Mixing-length eddy viscosity of level k (U-prognostic-microscale_1.cs:239-268); zero at and
// below KKART+1 (the reference masks those lanes).
template <bool IL>
__device__ __forceinline__ float ml_vis(const KArgs &a, const Acc<IL> &x, const ColCtx &c, int k, float dz,
                                        float ukp, float ukm) {
    if (k <= c.KK + 1) return 0.0f;
    const float zs = a.hokart[k] - c.hokK - dz * 0.5f;
    float mixL = vminf(0.071f * zs, 100.0f);
    if (c.cf.cov > 0) mixL *= (1.0f - 0.99f * c.cf.cov);
    float in = (ukp - ukm) / (2.0f * dz);
    const float DUDZ = in * in;
    in = (a.vk[x.at(0, k + 1)] - a.vk[x.at(0, k - 1)]) / (2.0f * dz);
    const float DVDZ = in * in;
    return vminf(mixL * mixL * sqrtf(0.5f * (DUDZ + DVDZ)), 15.0f);
}

// Friction velocity of the model-1 wall law at KKART+1 (U-prognostic-microscale_1.cs:419-450).
template <bool IL>
__device__ __forceinline__ float ml_ustern(const KArgs &a, const Acc<IL> &x, const ColCtx &c) {
    const int kw = c.KK + 1;
    const long long W = -(long long)c.nj2;
    if (c.fl & F_CUTKLT1) {
        if (c.fl & F_Z0GE) {
            const int ind = kw + 1;
            const float a1 = 0.5f * ((a.uks[x.at(W, ind)]) + a.uks[x.at(0, ind)]);
            const float b1 = 0.5f * ((a.vks[x.at(W, ind)]) + a.vks[x.at(0, ind)]);
            return c.cf.help_t * sqrtf(a1 * a1 + b1 * b1);
        }
        const float a1 = 0.5f * (a.uks[x.at(W, kw)] + a.uks[x.at(0, kw)]);
        const float b1 = 0.5f * (a.vks[x.at(W, kw)] + a.vks[x.at(0, kw)]);
        return c.cf.help_t * vmaxf(sqrtf(a1 * a1 + b1 * b1), 0.1f);
    }
    const float a1 = 0.5f * (a.uks[x.at(W, kw)] + a.uks[x.at(0, kw)]);
    const float b1 = 0.5f * (a.vks[x.at(W, kw)] + a.vks[x.at(0, kw)]);
    return c.cf.help_o * vmaxf(sqrtf(a1 * a1 + b1 * b1), 0.1f);
}

// ---------------------------------------------------------------------------------------------
// U momentum, mixing-length model, one level (U-prognostic-microscale_1.cs:205-470).
// ---------------------------------------------------------------------------------------------
template <bool IL>
__device__ __forceinline__ Coef u1_level(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc, int k) {
    const long long W = -(long long)c.nj2, E = c.nj2, S = -1, N = 1;
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy;
    const float dz = a.dzk[k];
    const float dxdz = DXK * dz, dydz = DYK * dz;
    const float uk = __ldcg(a.uk + x.at(0, k));
    const float VIS = ml_vis(a, x, c, k, dz, __ldcg(a.uk + x.at(0, k + 1)), __ldcg(a.uk + x.at(0, k - 1)));
    const float vmx = vmaxf(VIS, a.vishmin);
    float DE = vmx * dydz / DXK;
    float DW = DE;
    float DS = vmx * dxdz / DYK;
    float DN = DS;
    float DT = vmx * AREA / dz;
    float DB = (k > c.KK + 1) ? DT : 0.0f;
    if (c.fl & F_BS) DS = 0.0f;
    if (c.fl & F_BN) DN = 0.0f;
    if (c.fl & F_BW) DW = 0.0f;
    if (c.fl & F_BE) DE = 0.0f;
    const float uks = a.uks[x.at(0, k)], vks = a.vks[x.at(0, k)], wks = a.wks[x.at(0, k)];
    const float uksW = a.uks[x.at(W, k)], vksW = a.vks[x.at(W, k)], vksWS = a.vks[x.at(W + S, k)];
    const float vksS = a.vks[x.at(S, k)], vksWN = a.vks[x.at(W + N, k)], vksN = a.vks[x.at(N, k)];
    const float wksW = a.wks[x.at(W, k)];
    const float FE = uks * dydz;
    const float FW = uksW * dydz;
    const float FS = 0.25f * (vksW + vks + vksWS + vksS) * dxdz;
    const float FN = 0.25f * (vksW + vks + vksWN + vksN) * dxdz;
    const float FT = 0.25f * (wksW + wks + a.wks[x.at(W, k + 1)] + a.wks[x.at(0, k + 1)]) * AREA;
    const float wksB = a.wks[x.at(0, k - 1)], wksWB = a.wks[x.at(W, k - 1)];
    const float FB = (k > c.KK + 1) ? 0.25f * (wksW + wks + wksWB + wksB) * AREA : 0.0f;
    DE = vmaxf(DE, 0.0001f); DB = vmaxf(DB, 0.0001f); DW = vmaxf(DW, 0.0001f);
    DS = vmaxf(DS, 0.0001f); DN = vmaxf(DN, 0.0001f); DT = vmaxf(DT, 0.0001f);
    Coef r;
    r.B = pl_coef(DT, fabsf(FT / DT), -FT);
    r.C = pl_coef(DB, fabsf(FB / DB), FB);
    const float AE1 = pl_coef(DE, fabsf(FE / DE), -FE);
    const float AW1 = pl_coef(DW, fabsf(FW / DW), FW);
    const float AS1 = pl_coef(DS, fabsf(FS / DS), FS);
    const float AN1 = pl_coef(DN, fabsf(FN / DN), -FN);
    const float ap0 = sc.ap0[k];
    r.A = r.B + r.C + AW1 + AS1 + AE1 + AN1 + ap0;
    const float DDPX = a.dpmnew[x.at(W, k)] - a.dpmnew[x.at(0, k)];
    const float ukW = __ldcg(a.uk + x.at(W, k)), ukE = __ldcg(a.uk + x.at(E, k));
    const float ukS = __ldcg(a.uk + x.at(S, k)), ukN = __ldcg(a.uk + x.at(N, k));
    float DIM;
    if (c.fl & F_VEG) {
        const float in2 = 0.5f * (vksW + vks), in = 0.5f * (uksW + uks);
        const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.01f);
        DIM = AW1 * ukW + AS1 * ukS + AE1 * ukE + AN1 * ukN + ap0 * 0.5f * (uksW + uks) + DDPX * dydz +
              (a.coriolis * (sc.ug - uk) - a.veg[(size_t)c.col * a.ks + k - 1] * uk * wh) * AREA * dz;
    } else {
        DIM = AW1 * ukW + AS1 * ukS + AE1 * ukE + AN1 * ukN + ap0 * 0.5f * (uksW + uks) + DDPX * dydz +
              a.coriolis * (sc.ug - uk) * AREA * dz;
    }
    if (k >= c.wlo && k <= c.whi) {                       // masked wall term of the chunk, :419-450
        const float in = 0.5f * (uksW + uks), in2 = 0.5f * (vksW + vks);
        const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.1f);
        const float Ust = ml_ustern(a, x, c);
        const float m2 = (k == c.KK + 1) ? 1.0f : 0.0f;
        DIM -= uk / wh * (Ust * Ust) * AREA * m2;
    }
    if (k >= c.kad) {                                      // extra eddy-viscosity terms, :453-470
        const float DUDXE = (ukE - uk) * dydz;
        const float DUDXW = (uk - ukW) * dydz;
        const float DVDXN = (0.5f * (a.vks[x.at(E + N, k)] + vksN) - 0.5f * (vksN + vksWN)) * dxdz;
        const float DVDXS = (0.5f * (a.vks[x.at(E + S, k)] + vksS) - 0.5f * (vksS + vksWS)) * dxdz;
        const float DWDXT = (0.5f * (a.wk[x.at(E, k)] + wks) - 0.5f * (wks + wksW)) * AREA;
        const float DWDXB = (0.5f * (a.wk[x.at(E, k - 1)] + wksB) - 0.5f * (wksB + wksWB)) * AREA;
        DIM += VIS / DXK * (DUDXE - DUDXW + DVDXN - DVDXS + DWDXT - DWDXB);
    }
    r.D = DIM;
    r.phi = uk;
    return r;
}

// ---------------------------------------------------------------------------------------------
// V momentum, mixing-length model, one level (V-prognostic-microscale_1.cs:205-488).
// ---------------------------------------------------------------------------------------------
template <bool IL>
__device__ __forceinline__ Coef v1_level(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc, int k) {
    const long long W = -(long long)c.nj2, E = c.nj2, S = -1, N = 1;
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy;
    const float dz = a.dzk[k];
    const float dxdz = DXK * dz, dydz = DYK * dz;
    const float vk = __ldcg(a.vk + x.at(0, k));
    float VIS = 0.0f;
    if (k > c.KK + 1) {
        const float zs = a.hokart[k] - c.hokK - dz * 0.5f;
        float mixL = vminf(0.071f * zs, 100.0f);
        if (c.cf.cov > 0) mixL *= (1.0f - 0.99f * c.cf.cov);
        float in = (a.uk[x.at(0, k + 1)] - a.uk[x.at(0, k - 1)]) / (2.0f * dz);
        const float DUDZ = in * in;
        in = (__ldcg(a.vk + x.at(0, k + 1)) - __ldcg(a.vk + x.at(0, k - 1))) / (2.0f * dz);
        const float DVDZ = in * in;
        VIS = vminf(mixL * mixL * sqrtf(0.5f * (DUDZ + DVDZ)), 15.0f);
    }
    const float vmx = vmaxf(VIS, a.vishmin);
    float DE = vmx * dydz / DXK;
    float DW = DE;
    float DS = vmx * dxdz / DYK;
    float DN = DS;
    float DT = vmx * AREA / dz;
    float DB = (k > c.KK + 1) ? DT : 0.0f;
    if (c.fl & F_BS) DS = 0.0f;
    if (c.fl & F_BN) DN = 0.0f;
    if (c.fl & F_BW) DW = 0.0f;
    if (c.fl & F_BE) DE = 0.0f;
    const float uks = a.uks[x.at(0, k)], vks = a.vks[x.at(0, k)], wks = a.wks[x.at(0, k)];
    const float uksE = a.uks[x.at(E, k)], uksS = a.uks[x.at(S, k)], uksES = a.uks[x.at(E + S, k)];
    const float uksW = a.uks[x.at(W, k)], vksW = a.vks[x.at(W, k)], uksWS = a.uks[x.at(W + S, k)];
    const float vksS = a.vks[x.at(S, k)], wksS = a.wks[x.at(S, k)], wksB = a.wks[x.at(0, k - 1)];
    const float FE = 0.25f * (uks + uksE + uksS + uksES) * dydz;
    const float FW = 0.25f * (uks + uksW + uksS + uksWS) * dydz;
    const float FS = vksS * dxdz;
    const float FN = vks * dxdz;
    const float FT = 0.25f * (wksS + wks + a.wks[x.at(S, k + 1)] + a.wks[x.at(0, k + 1)]) * AREA;
    const float FB = (k > c.KK + 1) ? 0.25f * (wksS + wks + a.wks[x.at(S, k - 1)] + wksB) * AREA : 0.0f;
    DE = vmaxf(DE, 0.0001f); DB = vmaxf(DB, 0.0001f); DW = vmaxf(DW, 0.0001f);
    DS = vmaxf(DS, 0.0001f); DN = vmaxf(DN, 0.0001f); DT = vmaxf(DT, 0.0001f);
    Coef r;
    r.B = pl_coef(DT, fabsf(FT / DT), -FT);
    r.C = pl_coef(DB, fabsf(FB / DB), FB);
    const float AE1 = pl_coef(DE, fabsf(FE / DE), -FE);
    const float AW1 = pl_coef(DW, fabsf(FW / DW), FW);
    const float AS1 = pl_coef(DS, fabsf(FS / DS), FS);
    const float AN1 = pl_coef(DN, fabsf(FN / DN), -FN);
    const float ap0 = sc.ap0[k];
    r.A = r.B + r.C + AW1 + AS1 + AE1 + AN1 + ap0;
    const float DDPY = a.dpmnew[x.at(S, k)] - a.dpmnew[x.at(0, k)];
    const float vkN = __ldcg(a.vk + x.at(N, k)), vkS = __ldcg(a.vk + x.at(S, k));
    const float vkW = __ldcg(a.vk + x.at(W, k)), vkE = __ldcg(a.vk + x.at(E, k));
    float DIM;
    if (c.fl & F_VEG) {
        const float in2 = 0.5f * (vksW + vks), in = 0.5f * (uksW + uks);
        const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.01f);
        DIM = AW1 * vkW + AS1 * vkS + AE1 * vkE + AN1 * vkN + ap0 * 0.5f * (vksS + vks) + DDPY * dxdz +
              (a.coriolis * (sc.vg - vk) - a.veg[(size_t)c.col * a.ks + k - 1] * vk * wh) * AREA * dz;
    } else {
        DIM = AW1 * vkW + AS1 * vkS + AE1 * vkE + AN1 * vkN + ap0 * 0.5f * (vksS + vks) + DDPY * dxdz +
              a.coriolis * (sc.vg - vk) * AREA * dz;
    }
    if (k >= c.wlo && k <= c.whi) {                       // :437-467
        const float in = 0.5f * (uksW + uks), in2 = 0.5f * (vksW + vks);
        const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.1f);
        const float Ust = ml_ustern(a, x, c);
        const float m2 = (k == c.KK + 1) ? 1.0f : 0.0f;
        DIM -= vk / wh * (Ust * Ust) * AREA * m2;
    }
    if (k >= c.kad) {                                      // :470-488
        const float DVDYN = (vkN - vk) * dxdz;
        const float DVDYS = (vk - vkS) * dxdz;
        const float DUDYE = (0.5f * (a.uks[x.at(E + N, k)] + uksE) - 0.5f * (uksE + uksES)) * dxdz;
        const float DUDYW = (0.5f * (a.uks[x.at(W + N, k)] + uksW) - 0.5f * (uksW + uksWS)) * dxdz;
        const float DWDYT = (0.5f * (a.wk[x.at(N, k)] + wks) - 0.5f * (wks + wksS)) * AREA;
        const float DWDYB = (0.5f * (a.wk[x.at(N, k - 1)] + wksB) - 0.5f * (wksB + wksS)) * AREA;
        DIM += VIS / DXK * (DUDYE - DUDYW + DVDYN - DVDYS + DWDYT - DWDYB);
    }
    r.D = DIM;
    r.phi = vk;
    return r;
}

// ---------------------------------------------------------------------------------------------
// W momentum, mixing-length model, one level (W-prognostic-microscale_1.cs:205-402).
// ---------------------------------------------------------------------------------------------
template <bool IL>
__device__ __forceinline__ Coef w1_level(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc, int k) {
    const long long W = -(long long)c.nj2, E = c.nj2, S = -1, N = 1;
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy;
    const float dz = a.dzk[k];
    const float dxdz = DXK * dz, dydz = DYK * dz;
    const float uks = a.uks[x.at(0, k)], vks = a.vks[x.at(0, k)], wks = a.wks[x.at(0, k)];
    const float uksM = a.uks[x.at(0, k - 1)], vksM = a.vks[x.at(0, k - 1)];
    const float wk = __ldcg(a.wk + x.at(0, k));
    const float VIS = ml_vis(a, x, c, k, dz, a.uk[x.at(0, k + 1)], a.uk[x.at(0, k - 1)]);
    const float vmx = vmaxf(VIS, a.vishmin);
    float DE = vmx * dydz / DXK;
    float DW = DE;
    float DS = vmx * dxdz / DYK;
    float DN = DS;
    float DT = vmx * AREA / dz;
    float DB = (k > c.KK + 1) ? DT : 0.0f;
    if (c.fl & F_BS) DS = 0.0f;
    if (c.fl & F_BN) DN = 0.0f;
    if (c.fl & F_BW) DW = 0.0f;
    if (c.fl & F_BE) DE = 0.0f;
    const float uksW = a.uks[x.at(W, k)], uksWB = a.uks[x.at(W, k - 1)];
    const float vksS = a.vks[x.at(S, k)], vksSB = a.vks[x.at(S, k - 1)];
    const float FE = 0.25f * (uks + a.uks[x.at(E, k)] + uksM + a.uks[x.at(E, k - 1)]) * dydz;
    const float FW = 0.25f * (uks + uksW + uksM + uksWB) * dydz;
    const float FS = 0.25f * (vks + vksS + vksM + vksSB) * dxdz;
    const float FN = 0.25f * (vks + a.vks[x.at(N, k)] + vksM + a.vks[x.at(N, k - 1)]) * dxdz;
    const float FT = wks * AREA;
    const float wksB = a.wks[x.at(0, k - 1)];
    const float FB = (k > c.KK + 1) ? wksB * AREA : 0.0f;
    DE = vmaxf(DE, 0.0001f); DB = vmaxf(DB, 0.0001f); DW = vmaxf(DW, 0.0001f);
    DS = vmaxf(DS, 0.0001f); DN = vmaxf(DN, 0.0001f); DT = vmaxf(DT, 0.0001f);
    Coef r;
    r.B = pl_coef(DT, fabsf(FT / DT), -FT);
    r.C = pl_coef(DB, fabsf(FB / DB), FB);
    const float AE1 = pl_coef(DE, fabsf(FE / DE), -FE);
    const float AW1 = pl_coef(DW, fabsf(FW / DW), FW);
    const float AS1 = pl_coef(DS, fabsf(FS / DS), FS);
    const float AN1 = pl_coef(DN, fabsf(FN / DN), -FN);
    const float ap0 = sc.ap0[k];
    r.A = r.B + r.C + AW1 + AS1 + AE1 + AN1 + ap0;
    const float DDPZ = a.dpmnew[x.at(0, k - 1)] - a.dpmnew[x.at(0, k)];
    const float wkW = __ldcg(a.wk + x.at(W, k)), wkS = __ldcg(a.wk + x.at(S, k));
    const float wkE = __ldcg(a.wk + x.at(E, k)), wkN = __ldcg(a.wk + x.at(N, k));
    float DIM;
    if (c.fl & F_VEG) {
        const float in2 = 0.5f * (vksS + vks), in = 0.5f * (uksW + uks);
        const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.01f);
        DIM = AW1 * wkW + AS1 * wkS + AE1 * wkE + AN1 * wkN + ap0 * 0.5f * (wksB + wks) + DDPZ * AREA -
              a.veg[(size_t)c.col * a.ks + k - 1] * wk * wh * AREA * dz;
    } else {
        DIM = AW1 * wkW + AS1 * wkS + AE1 * wkE + AN1 * wkN + ap0 * 0.5f * (wksB + wks) + DDPZ * AREA;
    }
    if (k >= c.kad) {                                      // :376-402
        const float DUDZE = (0.5f * (a.uks[x.at(0, k + 1)] + uks) - 0.5f * (uks + uksM)) * dydz;
        const float DUDZW = (0.5f * (a.uks[x.at(W, k + 1)] + uksW) - 0.5f * (uksW + uksWB)) * dydz;
        const float DVDZN = (0.5f * (a.vks[x.at(0, k + 1)] + vks) - 0.5f * (vks + vksM)) * dxdz;
        const float DVDZS = (0.5f * (a.vks[x.at(S, k + 1)] + vksS) - 0.5f * (vksS + vksSB)) * dxdz;
        const float DWDZT = (__ldcg(a.wk + x.at(0, k + 1)) - wk) * AREA;
        const float DWDZB = (wk - __ldcg(a.wk + x.at(0, k - 1))) * AREA;
        DIM += VIS / dz * (DUDZE - DUDZW + DVDZN - DVDZS + DWDZT - DWDZB);
    }
    r.D = DIM;
    r.phi = wk;
    return r;
}

// ---------------------------------------------------------------------------------------------
// Pressure correction, right-hand side of level k (PrognosticFlowfield.cs:739-748, 853-855): the
// divergence on the fly, the already-swept neighbours (i-IS, j) and (i, j-JS); the reference
// zeroed the other two neighbours' DPM before the sweep, so they enter as literal zeros.
// ---------------------------------------------------------------------------------------------
template <bool IL>
__device__ __forceinline__ float pressure_dim(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc,
                                              int k, int IS, int JS) {
    const long long E = c.nj2, N = 1;
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy;
    const float dz = a.dzk[k];
    float DIV;
    if (k > c.KK + 1)
        DIV = (a.uk[x.at(0, k)] - a.uk[x.at(E, k)]) * DYK * dz + (a.vk[x.at(0, k)] - a.vk[x.at(N, k)]) * DXK * dz +
              (a.wk[x.at(0, k)] - a.wk[x.at(0, k + 1)]) * AREA;
    else
        DIV = (a.uk[x.at(0, k)] - a.uk[x.at(E, k)]) * DYK * dz + (a.vk[x.at(0, k)] - a.vk[x.at(N, k)]) * DXK * dz -
              a.wk[x.at(0, k + 1)] * AREA;
    const float pi = __ldcg(a.dpm + x.at(-(long long)IS * c.nj2, k));
    const float pj = __ldcg(a.dpm + x.at(-(long long)JS, k));
    const float si = (IS == 1) ? (pi + 0.0f) : (0.0f + pi);    // DPMim + DPMip
    const float sj = (JS == 1) ? (pj - 0.0f) : (0.0f - pj);    // DPMjm - DPMjp
    return DIV / sc.dtime + si / DXK * DYK * dz + sj / DYK * DXK * dz;
}

}  // namespace gral
