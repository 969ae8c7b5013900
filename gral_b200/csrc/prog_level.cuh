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
    float ug, vg, dtime, potdtdz;
    double frund;
    int quant;
    const float *ap0;
};

__device__ __forceinline__ SitCtx make_sit(const KArgs &a, int s) {
    SitCtx q;
    const SitDev &S = a.sit[s];
    q.ug = S.ug; q.vg = S.vg; q.dtime = S.dtime; q.potdtdz = S.potdtdz; q.frund = S.frund; q.quant = S.quantise;
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

// Patankar power law of one face, Vector<float> association order (U-prognostic-microscale_1.cs:348-370);
// the Vector512 twins fuse the outer multiply-add and square twice
// (U-prognostic-microscale_1_Vec512.cs:355-377).
__device__ __forceinline__ float pl_coef(float D, float Pe, float Fs) {
    const float in = 1.0f - 0.1f * Pe;
    return D * vmaxf(0.0f, in * in * in * in * in) + vmaxf(Fs, 0.0f);
}
__device__ __forceinline__ float pl_coef512(float D, float Pe, float Fs) {
    const float in = 1.0f - 0.1f * Pe;
    return fmaf(D, vmaxf(0.0f, in * ((in * in) * (in * in))), vmaxf(Fs, 0.0f));
}
__device__ __forceinline__ float pl1(bool v512, float D, float Pe, float Fs) {
    return v512 ? pl_coef512(D, Pe, Fs) : pl_coef(D, Pe, Fs);
}

// Parity width of the model-1 routines: SW = 8 or 16 fixes it when the kernel is compiled, SW = 0
// reads the loaded width (a.simd) at run time.
template <int SW>
__device__ __forceinline__ bool simd16(const KArgs &a) {
    return SW == 0 ? a.simd == 16 : SW == 16;
}

// Mixing-length eddy viscosity of level k (U-prognostic-microscale_1.cs:239-268) from the column's
// U and V at k+1 and k-1; zero at and below KKART+1 (the reference masks those lanes).
// The Vector512 twins take the height above KKART as HOKART[k] - fma(DZK, 0.5, HOKART[KKART])
// (U-prognostic-microscale_1_Vec512.cs:218).
template <int SW = 0>
__device__ __forceinline__ float ml_vis(const KArgs &a, const ColCtx &c, int k, float dz, float ukp, float ukm,
                                        float vkp, float vkm) {
    if (k <= c.KK + 1) return 0.0f;
    const float zs = simd16<SW>(a) ? a.hokart[k] - fmaf(dz, 0.5f, c.hokK) : a.hokart[k] - c.hokK - dz * 0.5f;
    float mixL = vminf(0.071f * zs, 100.0f);
    if (c.cf.cov > 0) mixL *= (1.0f - 0.99f * c.cf.cov);
    float in = (ukp - ukm) / (2.0f * dz);
    const float DUDZ = in * in;
    in = (vkp - vkm) / (2.0f * dz);
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
// Model-1 momentum, one level, split in two for the wavefront:
//   *_pre   everything that does not read the swept field's four horizontal neighbours at level k
//           (coefficients, viscosity, source terms, wall law, extra viscous pieces) -- safe to
//           evaluate before the column's Gauss-Seidel predecessors have finished;
//   *_post  reads those four neighbours and completes DIM in the reference's association order.
// pre + post evaluate exactly the operations of the reference expression, so the split changes
// no bit of the result (every product and partial sum is rounded as in the unsplit expression).
// ---------------------------------------------------------------------------------------------
struct MomPre {
    float A, B, C, phi;          // matrix row and the level's old value
    float aw, as, ae, an;        // AW1, AS1, AE1, AN1
    float t1, t2, t3;            // source terms following the neighbour products, in order
    float w;                     // wall term of the wall chunk (U, V)
    float vdx;                   // VIS/DXK (U, V)
    float e0, e1, e2, e3;        // extra viscous pieces (component specific)
    float hz;                    // DYK*DZK (U) or DXK*DZK (V)
};

// U momentum (U-prognostic-microscale_1.cs:205-470).  All operands of the level are loaded first,
// unconditionally (every address lies inside the padded grid and levels 0..KS-1), so a level costs
// one memory round trip; the arithmetic follows in the reference's order.
template <bool IL, int SW = 0>
__device__ __forceinline__ MomPre u1_pre(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc, int k) {
    const long long W = -(long long)c.nj2, E = c.nj2, S = -1, N = 1;
    const bool v512 = simd16<SW>(a);
    const float uk = __ldcg(a.uk + x.at(0, k));
    const float ukp = __ldcg(a.uk + x.at(0, k + 1)), ukm = __ldcg(a.uk + x.at(0, k - 1));
    const float vkp = a.vk[x.at(0, k + 1)], vkm = a.vk[x.at(0, k - 1)];
    const float uks = a.uks[x.at(0, k)], vks = a.vks[x.at(0, k)], wks = a.wks[x.at(0, k)];
    const float uksW = a.uks[x.at(W, k)], vksW = a.vks[x.at(W, k)], vksWS = a.vks[x.at(W + S, k)];
    const float vksS = a.vks[x.at(S, k)], vksWN = a.vks[x.at(W + N, k)], vksN = a.vks[x.at(N, k)];
    const float wksW = a.wks[x.at(W, k)], wksWT = a.wks[x.at(W, k + 1)], wksT = a.wks[x.at(0, k + 1)];
    const float wksB = a.wks[x.at(0, k - 1)], wksWB = a.wks[x.at(W, k - 1)];
    const float dpW = a.dpmnew[x.at(W, k)], dp0 = a.dpmnew[x.at(0, k)];
    const float vksEN = a.vks[x.at(E + N, k)], vksES = a.vks[x.at(E + S, k)];
    const float wkE = a.wk[x.at(E, k)], wkEB = a.wk[x.at(E, k - 1)];
    const float ap0 = sc.ap0[k];
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy;
    const float dz = a.dzk[k];
    const float dxdz = DXK * dz, dydz = DYK * dz;
    const float VIS = ml_vis<SW>(a, c, k, dz, ukp, ukm, vkp, vkm);
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
    const float FE = uks * dydz;
    const float FW = uksW * dydz;
    const float FS = 0.25f * (vksW + vks + vksWS + vksS) * dxdz;
    const float FN = 0.25f * (vksW + vks + vksWN + vksN) * dxdz;
    const float FT = 0.25f * (wksW + wks + wksWT + wksT) * AREA;
    const float FB = (k > c.KK + 1) ? 0.25f * (wksW + wks + wksWB + wksB) * AREA : 0.0f;
    DE = vmaxf(DE, 0.0001f); DB = vmaxf(DB, 0.0001f); DW = vmaxf(DW, 0.0001f);
    DS = vmaxf(DS, 0.0001f); DN = vmaxf(DN, 0.0001f); DT = vmaxf(DT, 0.0001f);
    MomPre r;
    r.B = pl1(v512, DT, fabsf(FT / DT), -FT);
    r.C = pl1(v512, DB, fabsf(FB / DB), FB);
    r.ae = pl1(v512, DE, fabsf(FE / DE), -FE);
    r.aw = pl1(v512, DW, fabsf(FW / DW), FW);
    r.as = pl1(v512, DS, fabsf(FS / DS), FS);
    r.an = pl1(v512, DN, fabsf(FN / DN), -FN);
    r.A = r.B + r.C + r.aw + r.as + r.ae + r.an + ap0;
    const float DDPX = dpW - dp0;
    r.t1 = ap0 * 0.5f * (uksW + uks);
    r.t2 = (v512 && !(c.fl & F_VEG)) ? DDPX : DDPX * dydz;     // Vector512: fma(DDPX, DYKDZK, ...)
    if (c.fl & F_VEG) {
        const float in2 = 0.5f * (vksW + vks), in = 0.5f * (uksW + uks);
        const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.01f);
        r.t3 = (a.coriolis * (sc.ug - uk) - a.veg[(size_t)c.col * a.ks + k - 1] * uk * wh) * AREA * dz;
    } else {
        r.t3 = a.coriolis * (sc.ug - uk) * AREA * dz;
    }
    r.w = 0.0f;
    if (k >= c.wlo && k <= c.whi) {                       // masked wall term of the chunk, :419-450
        const float in = 0.5f * (uksW + uks), in2 = 0.5f * (vksW + vks);
        const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.1f);
        const float Ust = ml_ustern(a, x, c);
        const float m2 = (k == c.KK + 1) ? 1.0f : 0.0f;
        r.w = uk / wh * (Ust * Ust) * AREA * m2;
    }
    r.vdx = VIS / DXK;
    r.hz = dydz;
    if (k >= c.kad) {                                      // extra eddy-viscosity terms, :453-470
        r.e0 = (0.5f * (vksEN + vksN) - 0.5f * (vksN + vksWN)) * dxdz;        // DVDXN
        r.e1 = (0.5f * (vksES + vksS) - 0.5f * (vksS + vksWS)) * dxdz;        // DVDXS
        r.e2 = (0.5f * (wkE + wks) - 0.5f * (wks + wksW)) * AREA;             // DWDXT
        r.e3 = (0.5f * (wkEB + wksB) - 0.5f * (wksB + wksWB)) * AREA;         // DWDXB
    }
    r.phi = uk;
    return r;
}

__device__ __forceinline__ float u1_post(const MomPre &p, const ColCtx &c, int k, float nW, float nS, float nE,
                                         float nN, bool v512) {
    float DIM;
    if (v512) {   // U-prognostic-microscale_1_Vec512.cs:399-421
        const float S1 = fmaf(p.aw, nW, p.as * nS), S2 = fmaf(p.ae, nE, p.an * nN);
        DIM = (c.fl & F_VEG) ? S1 + S2 + p.t1 + p.t2 + p.t3 : S1 + S2 + p.t1 + fmaf(p.t2, p.hz, p.t3);
    } else {
        DIM = p.aw * nW + p.as * nS + p.ae * nE + p.an * nN + p.t1 + p.t2 + p.t3;
    }
    if (k >= c.wlo && k <= c.whi) DIM -= p.w;
    if (k >= c.kad) {
        const float DUDXE = (nE - p.phi) * p.hz;
        const float DUDXW = (p.phi - nW) * p.hz;
        DIM += p.vdx * (DUDXE - DUDXW + p.e0 - p.e1 + p.e2 - p.e3);
    }
    return DIM;
}

// V momentum (V-prognostic-microscale_1.cs:205-488); operands first, as u1_pre.
template <bool IL, int SW = 0>
__device__ __forceinline__ MomPre v1_pre(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc, int k) {
    const long long W = -(long long)c.nj2, E = c.nj2, S = -1, N = 1;
    const bool v512 = simd16<SW>(a);
    const float vk = __ldcg(a.vk + x.at(0, k));
    const float ukp = a.uk[x.at(0, k + 1)], ukm = a.uk[x.at(0, k - 1)];
    const float vkp = __ldcg(a.vk + x.at(0, k + 1)), vkm = __ldcg(a.vk + x.at(0, k - 1));
    const float uks = a.uks[x.at(0, k)], vks = a.vks[x.at(0, k)], wks = a.wks[x.at(0, k)];
    const float uksE = a.uks[x.at(E, k)], uksS = a.uks[x.at(S, k)], uksES = a.uks[x.at(E + S, k)];
    const float uksW = a.uks[x.at(W, k)], vksW = a.vks[x.at(W, k)], uksWS = a.uks[x.at(W + S, k)];
    const float vksS = a.vks[x.at(S, k)], wksS = a.wks[x.at(S, k)], wksB = a.wks[x.at(0, k - 1)];
    const float wksST = a.wks[x.at(S, k + 1)], wksT = a.wks[x.at(0, k + 1)], wksSB = a.wks[x.at(S, k - 1)];
    const float dpS = a.dpmnew[x.at(S, k)], dp0 = a.dpmnew[x.at(0, k)];
    const float uksEN = a.uks[x.at(E + N, k)], uksWN = a.uks[x.at(W + N, k)];
    const float wkN = a.wk[x.at(N, k)], wkNB = a.wk[x.at(N, k - 1)];
    const float ap0 = sc.ap0[k];
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy;
    const float dz = a.dzk[k];
    const float dxdz = DXK * dz, dydz = DYK * dz;
    const float VIS = ml_vis<SW>(a, c, k, dz, ukp, ukm, vkp, vkm);
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
    const float FE = 0.25f * (uks + uksE + uksS + uksES) * dydz;
    const float FW = 0.25f * (uks + uksW + uksS + uksWS) * dydz;
    const float FS = vksS * dxdz;
    const float FN = vks * dxdz;
    const float FT = 0.25f * (wksS + wks + wksST + wksT) * AREA;
    const float FB = (k > c.KK + 1) ? 0.25f * (wksS + wks + wksSB + wksB) * AREA : 0.0f;
    DE = vmaxf(DE, 0.0001f); DB = vmaxf(DB, 0.0001f); DW = vmaxf(DW, 0.0001f);
    DS = vmaxf(DS, 0.0001f); DN = vmaxf(DN, 0.0001f); DT = vmaxf(DT, 0.0001f);
    MomPre r;
    r.B = pl1(v512, DT, fabsf(FT / DT), -FT);
    r.C = pl1(v512, DB, fabsf(FB / DB), FB);
    r.ae = pl1(v512, DE, fabsf(FE / DE), -FE);
    r.aw = pl1(v512, DW, fabsf(FW / DW), FW);
    r.as = pl1(v512, DS, fabsf(FS / DS), FS);
    r.an = pl1(v512, DN, fabsf(FN / DN), -FN);
    r.A = r.B + r.C + r.aw + r.as + r.ae + r.an + ap0;
    const float DDPY = dpS - dp0;
    r.t1 = ap0 * 0.5f * (vksS + vks);
    r.t2 = DDPY * dxdz;
    if (c.fl & F_VEG) {
        const float in2 = 0.5f * (vksW + vks), in = 0.5f * (uksW + uks);
        const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.01f);
        r.t3 = (a.coriolis * (sc.vg - vk) - a.veg[(size_t)c.col * a.ks + k - 1] * vk * wh) * AREA * dz;
    } else {
        r.t3 = a.coriolis * (sc.vg - vk) * AREA * dz;
    }
    r.w = 0.0f;
    if (k >= c.wlo && k <= c.whi) {                       // :437-467
        const float in = 0.5f * (uksW + uks), in2 = 0.5f * (vksW + vks);
        const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.1f);
        const float Ust = ml_ustern(a, x, c);
        const float m2 = (k == c.KK + 1) ? 1.0f : 0.0f;
        r.w = vk / wh * (Ust * Ust) * AREA * m2;
    }
    r.vdx = VIS / DXK;
    r.hz = dxdz;
    if (k >= c.kad) {                                      // :470-488
        const float DUDYE = (0.5f * (uksEN + uksE) - 0.5f * (uksE + uksES)) * dxdz;
        const float DUDYW = (0.5f * (uksWN + uksW) - 0.5f * (uksW + uksWS)) * dxdz;
        r.e0 = DUDYE - DUDYW;
        r.e1 = (0.5f * (wkN + wks) - 0.5f * (wks + wksS)) * AREA;                // DWDYT
        r.e2 = (0.5f * (wkNB + wksB) - 0.5f * (wksB + wksS)) * AREA;             // DWDYB
    }
    r.phi = vk;
    return r;
}

__device__ __forceinline__ float v1_post(const MomPre &p, const ColCtx &c, int k, float nW, float nS, float nE,
                                         float nN, bool v512) {
    float DIM;
    if (v512 && (c.fl & F_VEG))   // V-prognostic-microscale_1_Vec512.cs:404-410 (plain sums without vegetation)
        DIM = fmaf(p.aw, nW, p.as * nS) + fmaf(p.ae, nE, p.an * nN) + p.t1 + p.t2 + p.t3;
    else
        DIM = p.aw * nW + p.as * nS + p.ae * nE + p.an * nN + p.t1 + p.t2 + p.t3;
    if (k >= c.wlo && k <= c.whi) DIM -= p.w;
    if (k >= c.kad) {
        const float DVDYN = (nN - p.phi) * p.hz;
        const float DVDYS = (p.phi - nS) * p.hz;
        DIM += p.vdx * (p.e0 + DVDYN - DVDYS + p.e1 - p.e2);
    }
    return DIM;
}

// W momentum (W-prognostic-microscale_1.cs:205-402); its extra viscous term reads only the own
// column, so it is complete before the wait (e0 = the whole increment).  Operands first.
template <bool IL, int SW = 0>
__device__ __forceinline__ MomPre w1_pre(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc, int k) {
    const long long W = -(long long)c.nj2, E = c.nj2, S = -1, N = 1;
    const bool v512 = simd16<SW>(a);
    const float uks = a.uks[x.at(0, k)], vks = a.vks[x.at(0, k)], wks = a.wks[x.at(0, k)];
    const float uksM = a.uks[x.at(0, k - 1)], vksM = a.vks[x.at(0, k - 1)];
    const float wk = __ldcg(a.wk + x.at(0, k));
    const float ukp = a.uk[x.at(0, k + 1)], ukm = a.uk[x.at(0, k - 1)];
    const float vkp = a.vk[x.at(0, k + 1)], vkm = a.vk[x.at(0, k - 1)];
    const float uksW = a.uks[x.at(W, k)], uksWB = a.uks[x.at(W, k - 1)];
    const float vksS = a.vks[x.at(S, k)], vksSB = a.vks[x.at(S, k - 1)];
    const float uksE = a.uks[x.at(E, k)], uksEB = a.uks[x.at(E, k - 1)];
    const float vksN = a.vks[x.at(N, k)], vksNB = a.vks[x.at(N, k - 1)];
    const float wksB = a.wks[x.at(0, k - 1)];
    const float dpB = a.dpmnew[x.at(0, k - 1)], dp0 = a.dpmnew[x.at(0, k)];
    const float uksT = a.uks[x.at(0, k + 1)], uksWT = a.uks[x.at(W, k + 1)];
    const float vksT = a.vks[x.at(0, k + 1)], vksST = a.vks[x.at(S, k + 1)];
    const float wkT = __ldcg(a.wk + x.at(0, k + 1)), wkB = __ldcg(a.wk + x.at(0, k - 1));
    const float ap0 = sc.ap0[k];
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy;
    const float dz = a.dzk[k];
    const float dxdz = DXK * dz, dydz = DYK * dz;
    const float VIS = ml_vis<SW>(a, c, k, dz, ukp, ukm, vkp, vkm);
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
    const float FE = 0.25f * (uks + uksE + uksM + uksEB) * dydz;
    const float FW = 0.25f * (uks + uksW + uksM + uksWB) * dydz;
    const float FS = 0.25f * (vks + vksS + vksM + vksSB) * dxdz;
    const float FN = 0.25f * (vks + vksN + vksM + vksNB) * dxdz;
    const float FT = wks * AREA;
    const float FB = (k > c.KK + 1) ? wksB * AREA : 0.0f;
    DE = vmaxf(DE, 0.0001f); DB = vmaxf(DB, 0.0001f); DW = vmaxf(DW, 0.0001f);
    DS = vmaxf(DS, 0.0001f); DN = vmaxf(DN, 0.0001f); DT = vmaxf(DT, 0.0001f);
    MomPre r;
    r.B = pl1(v512, DT, fabsf(FT / DT), -FT);
    r.C = pl1(v512, DB, fabsf(FB / DB), FB);
    r.ae = pl1(v512, DE, fabsf(FE / DE), -FE);
    r.aw = pl1(v512, DW, fabsf(FW / DW), FW);
    r.as = pl1(v512, DS, fabsf(FS / DS), FS);
    r.an = pl1(v512, DN, fabsf(FN / DN), -FN);
    r.A = r.B + r.C + r.aw + r.as + r.ae + r.an + ap0;
    const float DDPZ = dpB - dp0;
    r.t1 = ap0 * 0.5f * (wksB + wks);
    r.t2 = DDPZ * AREA;
    r.t3 = 0.0f;
    if (c.fl & F_VEG) {
        const float in2 = 0.5f * (vksS + vks), in = 0.5f * (uksW + uks);
        const float wh = vmaxf(sqrtf(in * in + in2 * in2), 0.01f);
        r.t3 = a.veg[(size_t)c.col * a.ks + k - 1] * wk * wh * AREA * dz;     // subtracted
    }
    if (k >= c.kad) {                                      // :376-402
        const float DUDZE = (0.5f * (uksT + uks) - 0.5f * (uks + uksM)) * dydz;
        const float DUDZW = (0.5f * (uksWT + uksW) - 0.5f * (uksW + uksWB)) * dydz;
        const float DVDZN = (0.5f * (vksT + vks) - 0.5f * (vks + vksM)) * dxdz;
        const float DVDZS = (0.5f * (vksST + vksS) - 0.5f * (vksS + vksSB)) * dxdz;
        const float DWDZT = (wkT - wk) * AREA;
        const float DWDZB = (wk - wkB) * AREA;
        r.e0 = VIS / dz * (DUDZE - DUDZW + DVDZN - DVDZS + DWDZT - DWDZB);
    }
    r.phi = wk;
    return r;
}

__device__ __forceinline__ float w1_post(const MomPre &p, const ColCtx &c, int k, float nW, float nS, float nE,
                                         float nN, bool v512) {
    float DIM = v512 ? fmaf(p.aw, nW, p.as * nS) + fmaf(p.ae, nE, p.an * nN) + p.t1 + p.t2   // W-..._Vec512.cs:367-382
                     : p.aw * nW + p.as * nS + p.ae * nE + p.an * nN + p.t1 + p.t2;
    if (c.fl & F_VEG) DIM = DIM - p.t3;
    if (k >= c.kad) DIM += p.e0;
    return DIM;
}

// The swept field's four horizontal neighbours of level k: W, S, E, N (read through L2: other
// warps of the same launch write them).
template <bool IL>
__device__ __forceinline__ void nbr4(const float *F, const Acc<IL> &x, const ColCtx &c, int k, float &nW, float &nS,
                                     float &nE, float &nN) {
    nW = __ldcg(F + x.at(-(long long)c.nj2, k));
    nS = __ldcg(F + x.at(-1, k));
    nE = __ldcg(F + x.at(c.nj2, k));
    nN = __ldcg(F + x.at(1, k));
}

template <bool IL, int SW = 0>
__device__ __forceinline__ Coef u1_level(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc, int k) {
    const MomPre p = u1_pre<IL, SW>(a, x, c, sc, k);
    float nW, nS, nE, nN;
    nbr4(a.uk, x, c, k, nW, nS, nE, nN);
    return Coef{p.A, p.B, p.C, u1_post(p, c, k, nW, nS, nE, nN, simd16<SW>(a)), p.phi};
}

template <bool IL, int SW = 0>
__device__ __forceinline__ Coef v1_level(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc, int k) {
    const MomPre p = v1_pre<IL, SW>(a, x, c, sc, k);
    float nW, nS, nE, nN;
    nbr4(a.vk, x, c, k, nW, nS, nE, nN);
    return Coef{p.A, p.B, p.C, v1_post(p, c, k, nW, nS, nE, nN, simd16<SW>(a)), p.phi};
}

template <bool IL, int SW = 0>
__device__ __forceinline__ Coef w1_level(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc, int k) {
    const MomPre p = w1_pre<IL, SW>(a, x, c, sc, k);
    float nW, nS, nE, nN;
    nbr4(a.wk, x, c, k, nW, nS, nE, nN);
    return Coef{p.A, p.B, p.C, w1_post(p, c, k, nW, nS, nE, nN, simd16<SW>(a)), p.phi};
}

// ---------------------------------------------------------------------------------------------
// Pressure correction, right-hand side of level k (PrognosticFlowfield.cs:739-748, 853-855): the
// divergence on the fly, the already-swept neighbours (i-IS, j) and (i, j-JS); the reference
// zeroed the other two neighbours' DPM before the sweep, so they enter as literal zeros.
// pressure_pre is the divergence term (no pressure read), pressure_post adds the neighbours.
// ---------------------------------------------------------------------------------------------
template <bool IL>
__device__ __forceinline__ float pressure_pre(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc,
                                              int k) {
    const long long E = c.nj2, N = 1;
    const float u0 = a.uk[x.at(0, k)], uE = a.uk[x.at(E, k)], v0 = a.vk[x.at(0, k)], vN = a.vk[x.at(N, k)];
    const float w0 = a.wk[x.at(0, k)], wT = a.wk[x.at(0, k + 1)];
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy;
    const float dz = a.dzk[k];
    float DIV;
    if (k > c.KK + 1)
        DIV = (u0 - uE) * DYK * dz + (v0 - vN) * DXK * dz + (w0 - wT) * AREA;
    else
        DIV = (u0 - uE) * DYK * dz + (v0 - vN) * DXK * dz - wT * AREA;
    return DIV / sc.dtime;
}

// pi, pj: this sweep's DPM of the predecessors (i-IS, j) and (i, j-JS) at level k
__device__ __forceinline__ float pressure_post_v(const KArgs &a, float t0, int k, int IS, int JS, float pi, float pj) {
    const float DXK = a.dxk, DYK = a.dyk;
    const float dz = a.dzk[k];
    const float si = (IS == 1) ? (pi + 0.0f) : (0.0f + pi);    // DPMim + DPMip
    const float sj = (JS == 1) ? (pj - 0.0f) : (0.0f - pj);    // DPMjm - DPMjp
    return t0 + si / DXK * DYK * dz + sj / DYK * DXK * dz;
}

template <bool IL>
__device__ __forceinline__ float pressure_post(const KArgs &a, const Acc<IL> &x, const ColCtx &c, float t0, int k,
                                               int IS, int JS) {
    const float pi = __ldcg(a.dpm + x.at(-(long long)IS * c.nj2, k));
    const float pj = __ldcg(a.dpm + x.at(-(long long)JS, k));
    return pressure_post_v(a, t0, k, IS, JS, pi, pj);
}

template <bool IL>
__device__ __forceinline__ float pressure_dim(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc,
                                              int k, int IS, int JS) {
    return pressure_post(a, x, c, pressure_pre(a, x, c, sc, k), k, IS, JS);
}


}  // namespace gral

namespace gral {

// =============================================================================================
// k-eps model (TurbulenceModel 2) and no-diffusion model (TurbulenceModel 0): scalar routines of
// the reference, evaluated per level.  Their power law and source sums are partly in double
// (U-prognostic-microscale_2.cs:180-203), their recurrences divide twice per level (:247-256).
// =============================================================================================

// FloatMax(0, (float)Pow5(1 - 0.1*Pe)) * D + FloatMax(F, 0)  (U-prognostic-microscale_2.cs:180-185)
__device__ __forceinline__ float pl_ke(float D, float Pe, float Fs) {
    const double x = 1 - 0.1 * (double)Pe;
    return D * vmaxf(0.0f, (float)(x * x * x * x * x)) + vmaxf(Fs, 0.0f);
}

// (float)Math.Sqrt(Pow2(0.5*(a1+a2)) + Pow2(0.5*(b1+b2))) with float sums (:207-219)
__device__ __forceinline__ float wind_half(float a1, float a2, float b1, float b2) {
    const double x = 0.5 * (double)(a1 + a2), y = 0.5 * (double)(b1 + b2);
    return (float)sqrt(x * x + y * y);
}

// U (COMP 0) or V (COMP 1) of models 2 (DIFF) and 0 (no DIFF), one level
// (U-prognostic-microscale_2.cs:103-257, V-...2.cs, U-...0.cs:103-182, V-...0.cs).
template <bool DIFF, int COMP, bool IL>
__device__ __forceinline__ Coef uv_scalar_level(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc,
                                                int k) {
    const long long W = -(long long)c.nj2, E = c.nj2, S = -1, N = 1;
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy;
    const float dz = a.dzk[k];
    const float dxdz = DXK * dz, dydz = DYK * dz;
    float *PHI = (COMP == 0) ? a.uk : a.vk;
    const float phi = __ldcg(PHI + x.at(0, k));
    float VIS = 0.0f, DE = 0.0f, DW = 0.0f, DS = 0.0f, DN = 0.0f, DT = 0.0f, DB = 0.0f;
    if (DIFF) {
        const float zs = a.hokart[k] - c.hokK - dz * 0.5f;
        VIS = (float)sqrt((double)a.turb[x.at(0, k)]) * zs * 0.09f;
        const float vmx = vmaxf(VIS, a.vishmin);
        DE = vmx * dydz / DXK; DW = DE;
        DS = vmx * dxdz / DYK; DN = DS;
        DT = vmx * AREA / dz;
        DB = (k > c.KK + 1) ? DT : 0.0f;
        if (c.fl & F_BS) DS = 0.0f;
        if (c.fl & F_BN) DN = 0.0f;
        if (c.fl & F_BW) DW = 0.0f;
        if (c.fl & F_BE) DE = 0.0f;
    }
    const float uks = a.uks[x.at(0, k)], vks = a.vks[x.at(0, k)], wks = a.wks[x.at(0, k)];
    const float uksW = a.uks[x.at(W, k)], vksW = a.vks[x.at(W, k)];
    float FE, FW, FS, FN, FT, FB = 0.0f;
    if (COMP == 0) {
        const float vksWS = a.vks[x.at(W + S, k)], vksS = a.vks[x.at(S, k)];
        const float vksWN = a.vks[x.at(W + N, k)], vksN = a.vks[x.at(N, k)];
        const float wksW = a.wks[x.at(W, k)];
        FE = uks * dydz;
        FW = uksW * dydz;
        FS = 0.25f * (vksW + vks + vksWS + vksS) * dxdz;
        FN = 0.25f * (vksW + vks + vksWN + vksN) * dxdz;
        FT = 0.25f * (wksW + wks + a.wks[x.at(W, k + 1)] + a.wks[x.at(0, k + 1)]) * AREA;
        if (k > c.KK + 1) FB = 0.25f * (wksW + wks + a.wks[x.at(W, k - 1)] + a.wks[x.at(0, k - 1)]) * AREA;
    } else {
        const float uksE = a.uks[x.at(E, k)], uksS = a.uks[x.at(S, k)];
        const float uksES = a.uks[x.at(E + S, k)], uksWS = a.uks[x.at(W + S, k)];
        const float wksS = a.wks[x.at(S, k)];
        FE = 0.25f * (uks + uksE + uksS + uksES) * dydz;
        FW = 0.25f * (uks + uksW + uksS + uksWS) * dydz;
        FS = a.vks[x.at(S, k)] * dxdz;
        FN = vks * dxdz;
        FT = 0.25f * (wksS + wks + a.wks[x.at(S, k + 1)] + a.wks[x.at(0, k + 1)]) * AREA;
        if (k > c.KK + 1) FB = 0.25f * (wksS + wks + a.wks[x.at(S, k - 1)] + a.wks[x.at(0, k - 1)]) * AREA;
    }
    Coef r;
    float AE1, AW1, AS1, AN1;
    if (DIFF) {
        DE = vmaxf(DE, 0.0001f); DB = vmaxf(DB, 0.0001f); DW = vmaxf(DW, 0.0001f);
        DS = vmaxf(DS, 0.0001f); DN = vmaxf(DN, 0.0001f); DT = vmaxf(DT, 0.0001f);
        r.B = pl_ke(DT, fabsf(FT / DT), -FT);
        r.C = pl_ke(DB, fabsf(FB / DB), FB);
        AE1 = pl_ke(DE, fabsf(FE / DE), -FE);
        AW1 = pl_ke(DW, fabsf(FW / DW), FW);
        AS1 = pl_ke(DS, fabsf(FS / DS), FS);
        AN1 = pl_ke(DN, fabsf(FN / DN), -FN);
    } else {                                                  // upwind, U-prognostic-microscale_0.cs:123-128
        r.B = vmaxf(-FT, 0.0f);
        r.C = vmaxf(FB, 0.0f);
        AE1 = vmaxf(-FE, 0.0f);
        AW1 = vmaxf(FW, 0.0f);
        AS1 = vmaxf(FS, 0.0f);
        AN1 = vmaxf(-FN, 0.0f);
    }
    const float ap0 = sc.ap0[k];
    r.A = r.B + r.C + AW1 + AS1 + AE1 + AN1 + ap0;
    const float pW = __ldcg(PHI + x.at(W, k)), pE = __ldcg(PHI + x.at(E, k));
    const float pS = __ldcg(PHI + x.at(S, k)), pN = __ldcg(PHI + x.at(N, k));
    float DIM;
    if (COMP == 0) {
        const float DDPX = a.dpmnew[x.at(W, k)] - a.dpmnew[x.at(0, k)];
        DIM = (float)(AW1 * pW + AS1 * pS + AE1 * pE + AN1 * pN + ap0 * 0.5 * (uksW + uks) + DDPX * dydz +
                      a.coriolis * (sc.ug - phi) * AREA * dz);
    } else {
        const float DDPY = a.dpmnew[x.at(S, k)] - a.dpmnew[x.at(0, k)];
        DIM = (float)(AW1 * pW + AS1 * pS + AE1 * pE + AN1 * pN + ap0 * 0.5 * (a.vks[x.at(S, k)] + vks) + DDPY * dxdz +
                      a.coriolis * (sc.vg - phi) * AREA * dz);
    }
    if (k == c.KK + 1) {                                      // wall law, U-prognostic-microscale_2.cs:205-231
        const float windhilf = vmaxf(wind_half(uksW, uks, vksW, vks), 0.01f);
        float Ust;
        if (c.fl & F_CUTKLT1) {
            Ust = c.cf.help_t * windhilf;
            if (c.fl & F_Z0GED)
                Ust = c.cf.help_t * wind_half(a.uks[x.at(W, k + 1)], a.uks[x.at(0, k + 1)], a.vks[x.at(W, k + 1)],
                                              a.vks[x.at(0, k + 1)]);
        } else {
            Ust = c.cf.help_o * windhilf;
        }
        DIM -= (float)(phi / windhilf * (Ust * Ust) * AREA);
    }
    if (DIFF && k > c.KK + 1) {                               // :234-245
        float ADD;
        if (COMP == 0) {
            const float DUDXE = (pE - phi) * dydz;
            const float DUDXW = (phi - pW) * dydz;
            const float vksN = a.vks[x.at(N, k)], vksS = a.vks[x.at(S, k)];
            const float DVDXN = (0.5f * (a.vks[x.at(E + N, k)] + vksN) - 0.5f * (vksN + a.vks[x.at(W + N, k)])) * dxdz;
            const float DVDXS = (0.5f * (a.vks[x.at(E + S, k)] + vksS) - 0.5f * (vksS + a.vks[x.at(W + S, k)])) * dxdz;
            const float wksW = a.wks[x.at(W, k)], wksB = a.wks[x.at(0, k - 1)];
            const float DWDXT = (0.5f * (a.wk[x.at(E, k)] + wks) - 0.5f * (wks + wksW)) * AREA;
            const float DWDXB = (0.5f * (a.wk[x.at(E, k - 1)] + wksB) - 0.5f * (wksB + a.wks[x.at(W, k - 1)])) * AREA;
            ADD = VIS / DXK * (DUDXE - DUDXW + DVDXN - DVDXS + DWDXT - DWDXB);
        } else {
            const float DVDYN = (pN - phi) * dxdz;
            const float DVDYS = (phi - pS) * dxdz;
            const float uksE = a.uks[x.at(E, k)];
            const float DUDYE = (0.5f * (a.uks[x.at(E + N, k)] + uksE) - 0.5f * (uksE + a.uks[x.at(E + S, k)])) * dxdz;
            const float DUDYW = (0.5f * (a.uks[x.at(W + N, k)] + uksW) - 0.5f * (uksW + a.uks[x.at(W + S, k)])) * dxdz;
            const float wksS = a.wks[x.at(S, k)], wksB = a.wks[x.at(0, k - 1)];
            const float DWDYT = (0.5f * (a.wk[x.at(N, k)] + wks) - 0.5f * (wks + wksS)) * AREA;
            const float DWDYB = (0.5f * (a.wk[x.at(N, k - 1)] + wksB) - 0.5f * (wksB + a.wks[x.at(S, k - 1)])) * AREA;
            ADD = VIS / DXK * (DUDYE - DUDYW + DVDYN - DVDYS + DWDYT - DWDYB);
        }
        DIM += ADD;
    }
    r.D = DIM;
    r.phi = phi;
    return r;
}

// W of models 2 (DIFF) and 0, one level (W-prognostic-microscale_2.cs:84-199, W-...0.cs:84-123).
template <bool DIFF, bool IL>
__device__ __forceinline__ Coef w_scalar_level(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc,
                                               int k) {
    const long long W = -(long long)c.nj2, E = c.nj2, S = -1, N = 1;
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy;
    const float dz = a.dzk[k];
    const float dxdz = DXK * dz, dydz = DYK * dz;
    const float uks = a.uks[x.at(0, k)], uksM = a.uks[x.at(0, k - 1)];
    const float vks = a.vks[x.at(0, k)], vksM = a.vks[x.at(0, k - 1)];
    const float wk = __ldcg(a.wk + x.at(0, k));
    float VIS = 0.0f, DE = 0.0f, DW = 0.0f, DS = 0.0f, DN = 0.0f, DT = 0.0f, DB = 0.0f;
    if (DIFF) {
        const float zs = a.hokart[k] - c.hokK - dz * 0.5f;
        VIS = (float)sqrt((double)a.turb[x.at(0, k)]) * zs * 0.09f;
        const float vmx = vmaxf(VIS, a.vishmin);
        DE = vmx * dydz / DXK; DW = DE;
        DS = vmx * dxdz / DYK; DN = DS;
        DT = vmx * AREA / dz;
        DB = (k > c.KK + 1) ? DT : 0.0f;
        if (c.fl & F_BS) DS = 0.0f;
        if (c.fl & F_BN) DN = 0.0f;
        if (c.fl & F_BW) DW = 0.0f;
        if (c.fl & F_BE) DE = 0.0f;
    }
    const float uksE = a.uks[x.at(E, k)], uksW = a.uks[x.at(W, k)];
    const float vksS = a.vks[x.at(S, k)], vksN = a.vks[x.at(N, k)];
    const float FE = 0.25f * (uks + uksE + uksM + a.uks[x.at(E, k - 1)]) * dydz;
    const float FW = 0.25f * (uks + uksW + uksM + a.uks[x.at(W, k - 1)]) * dydz;
    const float FS = 0.25f * (vks + vksS + vksM + a.vks[x.at(S, k - 1)]) * dxdz;
    const float FN = 0.25f * (vks + vksN + vksM + a.vks[x.at(N, k - 1)]) * dxdz;
    const float wks = a.wks[x.at(0, k)], wksB = a.wks[x.at(0, k - 1)];
    const float FT = wks * AREA;
    const float FB = (k > c.KK + 1) ? wksB * AREA : 0.0f;
    Coef r;
    float AE1, AW1, AS1, AN1;
    if (DIFF) {
        DE = vmaxf(DE, 0.0001f); DB = vmaxf(DB, 0.0001f); DW = vmaxf(DW, 0.0001f);
        DS = vmaxf(DS, 0.0001f); DN = vmaxf(DN, 0.0001f); DT = vmaxf(DT, 0.0001f);
        r.B = pl_ke(DT, fabsf(FT / DT), -FT);
        r.C = pl_ke(DB, fabsf(FB / DB), FB);
        AE1 = pl_ke(DE, fabsf(FE / DE), -FE);
        AW1 = pl_ke(DW, fabsf(FW / DW), FW);
        AS1 = pl_ke(DS, fabsf(FS / DS), FS);
        AN1 = pl_ke(DN, fabsf(FN / DN), -FN);
    } else {
        r.B = vmaxf(-FT, 0.0f);
        r.C = vmaxf(FB, 0.0f);
        AE1 = vmaxf(-FE, 0.0f);
        AW1 = vmaxf(FW, 0.0f);
        AS1 = vmaxf(FS, 0.0f);
        AN1 = vmaxf(-FN, 0.0f);
    }
    const float ap0 = sc.ap0[k];
    r.A = r.B + r.C + AW1 + AS1 + AE1 + AN1 + ap0;
    const float DDPZ = a.dpmnew[x.at(0, k - 1)] - a.dpmnew[x.at(0, k)];
    const float wW = __ldcg(a.wk + x.at(W, k)), wS = __ldcg(a.wk + x.at(S, k));
    const float wE = __ldcg(a.wk + x.at(E, k)), wN = __ldcg(a.wk + x.at(N, k));
    float DIM = (float)(AW1 * wW + AS1 * wS + AE1 * wE + AN1 * wN + ap0 * 0.5 * (wksB + wks) + DDPZ * AREA);
    if (DIFF && k > c.KK + 1) {                               // W-prognostic-microscale_2.cs:162-172
        const float DUDZE = (0.5f * (a.uks[x.at(0, k + 1)] + uks) - 0.5f * (uks + uksM)) * dydz;
        const float DUDZW = (0.5f * (a.uks[x.at(W, k + 1)] + uksW) - 0.5f * (uksW + a.uks[x.at(W, k - 1)])) * dydz;
        const float DVDZN = (0.5f * (a.vks[x.at(0, k + 1)] + vks) - 0.5f * (vks + vksM)) * dxdz;
        const float DVDZS = (0.5f * (a.vks[x.at(S, k + 1)] + vksS) - 0.5f * (vksS + a.vks[x.at(S, k - 1)])) * dxdz;
        const float DWDZT = (__ldcg(a.wk + x.at(0, k + 1)) - wk) * AREA;
        const float DWDZB = (wk - __ldcg(a.wk + x.at(0, k - 1))) * AREA;
        DIM += VIS / dz * (DUDZE - DUDZW + DVDZN - DVDZS + DWDZT - DWDZB);
    }
    r.D = DIM;
    r.phi = wk;
    return r;
}

// Coefficients of the turbulent kinetic energy k and its dissipation eps at one level
// (TKE-prognostic-microscale.cs:112-270): shared A, separate (B, C, D) per variable.
struct CoefKE {
    float A, B1, C1, D1, B2, C2, D2, k1, e1;
};

template <bool IL>
__device__ __forceinline__ CoefKE tke_level(const KArgs &a, const Acc<IL> &x, const ColCtx &c, const SitCtx &sc,
                                            int k) {
    const float potdtdz = sc.potdtdz;
    const long long W = -(long long)c.nj2, E = c.nj2, S = -1, N = 1;
    const float DXK = a.dxk, DYK = a.dyk, AREA = a.areaxy;
    const float DXK_Rez = 1 / DXK, DYK_Rez = 1 / DYK;
    const float dz = a.dzk[k];
    const float DXKDZK = DXK * dz, DYKDZK = DYK * dz;
    const float DZK_Rez = 1 / dz;
    const float TURB = __ldcg(a.turb + x.at(0, k)), TDISS = __ldcg(a.tdiss + x.at(0, k));
    const float zs = a.hokart[k] - c.hokK - dz * 0.5f;
    float VIS = (float)sqrt((double)TURB) * zs * 0.09f;
    VIS = net_minf(VIS, 15);
    float DE = net_maxf(VIS, a.vishmin) * DYKDZK * DXK_Rez;
    float DW = DE;
    float DS = net_maxf(VIS, a.vishmin) * DXKDZK * DYK_Rez;
    float DN = DS;
    float DT = net_maxf(VIS, a.vishmin) * AREA * DZK_Rez;
    float DB = 0;
    float DTEPS = net_maxf(VIS / 1.0f, a.vishmin) * AREA * DZK_Rez;   // VIS / Ceps, VISVMIN = VISHMIN
    float DBEPS = 0;
    if (k > c.KK + 1) { DB = DT; DBEPS = DTEPS; }
    if (c.fl & F_BS) DS = 0;
    if (c.fl & F_BN) DN = 0;
    if (c.fl & F_BW) DW = 0;
    if (c.fl & F_BE) DE = 0;
    const float UK = a.uk[x.at(0, k)], UKip = a.uk[x.at(E, k)];
    const float VK = a.vk[x.at(0, k)], VKjp = a.vk[x.at(N, k)];
    const float WK1 = a.wk[x.at(0, k + 1)];
    const float FE = UKip * DYKDZK;
    const float FW = UK * DYKDZK;
    const float FS = VK * DXKDZK;
    const float FN = VKjp * DXKDZK;
    const float FT = WK1 * AREA;
    float FB = 0;
    if (k > c.KK + 1) FB = a.wk[x.at(0, k)] * AREA;
    DE = net_maxf(DE, 0.0001f); DB = net_maxf(DB, 0.0001f); DW = net_maxf(DW, 0.0001f);
    DS = net_maxf(DS, 0.0001f); DN = net_maxf(DN, 0.0001f); DT = net_maxf(DT, 0.0001f);
    DBEPS = net_maxf(DBEPS, 0.0001f); DTEPS = net_maxf(DTEPS, 0.0001f);
    const float PE = fabsf(FE / DE), PB = fabsf(FB / DB), PW = fabsf(FW / DW);
    const float PS = fabsf(FS / DS), PN = fabsf(FN / DN), PT = fabsf(FT / DT);
    const float PBEPS = fabsf(FN / DBEPS);                      // FN, not FB (:187)
    const float PTEPS = fabsf(FT / DTEPS);
    auto p5 = [](float v) { const float q = 1 - 0.1f * v; return q * q * q * q * q; };
    CoefKE r;
    r.B1 = DT * net_maxf(0, p5(PT)) + net_maxf(-FT, 0);
    r.C1 = DB * net_maxf(0, p5(PB)) + net_maxf(FB, 0);
    const float AE1 = DE * net_maxf(0, p5(PE)) + net_maxf(-FE, 0);
    const float AW1 = DW * net_maxf(0, p5(PW)) + net_maxf(FW, 0);
    const float AS1 = DS * net_maxf(0, p5(PS)) + net_maxf(FS, 0);
    const float AN1 = DN * net_maxf(0, p5(PN)) + net_maxf(-FN, 0);
    r.B2 = DT * net_maxf(0, p5(PTEPS)) + net_maxf(-FT, 0);
    r.C2 = DB * net_maxf(0, p5(PBEPS)) + net_maxf(FB, 0);
    const float ap0 = sc.ap0[k];
    r.A = r.B1 + r.C1 + AW1 + AS1 + AE1 + AN1 + ap0;
    // production terms (:213-243)
    const float UX1 = UKip, UX2 = UK;
    const float VX1 = 0.5f * (a.vk[x.at(E, k)] + a.vk[x.at(E + N, k)]);
    const float VX2 = 0.5f * (a.vk[x.at(W, k)] + a.vk[x.at(W + N, k)]);
    const float WX1 = 0.5f * (a.wk[x.at(E, k)] + a.wk[x.at(E, k + 1)]);
    const float WX2 = 0.5f * (a.wk[x.at(W, k)] + a.wk[x.at(W, k + 1)]);
    const float UY1 = 0.5f * (a.uk[x.at(N, k)] + a.uk[x.at(E + N, k)]);
    const float UY2 = 0.5f * (a.uk[x.at(S, k)] + a.uk[x.at(E + S, k)]);
    const float VY1 = VKjp, VY2 = VK;
    const float WY1 = 0.5f * (a.wk[x.at(N, k)] + a.wk[x.at(N, k + 1)]);
    const float WY2 = 0.5f * (a.wk[x.at(S, k)] + a.wk[x.at(S, k + 1)]);
    const float DUDX = (UX1 - UX2) * DXK_Rez;
    const float DVDX = (VX1 - VX2) * DXK_Rez * 0.5f;
    const float DWDX = (WX1 - WX2) * DXK_Rez * 0.5f;
    const float DUDY = (UY1 - UY2) * DYK_Rez * 0.5f;
    const float DVDY = (VY1 - VY2) * DYK_Rez;
    const float DWDY = (WY1 - WY2) * DYK_Rez * 0.5f;
    float DUDZ = a.uk[x.at(0, k + 1)] * DZK_Rez * 0.5f;
    float DVDZ = a.vk[x.at(0, k + 1)] * DZK_Rez * 0.5f;
    float DWDZ = WK1 * DZK_Rez * 0.5f;
    if (k > c.KK + 1) {
        DUDZ = (a.uk[x.at(0, k + 1)] - a.uk[x.at(0, k - 1)]) * DZK_Rez * 0.5f;
        DVDZ = (a.vk[x.at(0, k + 1)] - a.vk[x.at(0, k - 1)]) * DZK_Rez * 0.5f;
        DWDZ = (WK1 - a.wk[x.at(0, k - 1)]) * DZK_Rez * 0.5f;
    }
    auto sq = [](float v) { return v * v; };
    const float PROTURB = VIS * AREA * dz *
        (2 * sq(DUDX) + 2 * sq(DVDY) + 2 * sq(DWDZ) + sq(DUDY + DVDX) + sq(DUDZ + DWDX) + sq(DVDZ + DWDY) - TDISS);
    const float PROBOU = (float)(-potdtdz * 9.81 / 283 * VIS * 1.35 * AREA * dz);
    const float tW = __ldcg(a.turb + x.at(W, k)), tS = __ldcg(a.turb + x.at(S, k));
    const float tE = __ldcg(a.turb + x.at(E, k)), tN = __ldcg(a.turb + x.at(N, k));
    const float eW = __ldcg(a.tdiss + x.at(W, k)), eS = __ldcg(a.tdiss + x.at(S, k));
    const float eE = __ldcg(a.tdiss + x.at(E, k)), eN = __ldcg(a.tdiss + x.at(N, k));
    r.D1 = AW1 * tW + AS1 * tS + AE1 * tE + AN1 * tN + ap0 * TURB + PROTURB + PROBOU;
    r.D2 = AW1 * eW + AS1 * eS + AE1 * eE + AN1 * eN + ap0 * TDISS + (TDISS / TURB * (1.44f * PROTURB - 1.92f * TDISS));
    r.k1 = TURB;
    r.e1 = TDISS;
    return r;
}

// ---------------------------------------------------------------------------------------------
// Column bodies of the velocity correction and the averages, shared by their own kernels and by
// the fused wavefront of the slab family.  Levels kbeg, kbeg+kstep, ... of one (situation, column).
// ---------------------------------------------------------------------------------------------
// velocity correction with Frund quantisation in double (PrognosticFlowfield.cs:904-949)
template <bool IL>
__device__ __forceinline__ void velcorr_col(const KArgs &a, int s, int col, int i, int j, const Acc<IL> &x, int kbeg,
                                            int kstep) {
    if (i < 2 || i > a.nii - 1 || j < 2 || j > a.njj - 1) return;
    if (!(a.cflags[col] & F_VC)) return;
    const ColMeta m = a.meta[col];
    const SitDev &sd = a.sit[s];
    const float DT = sd.dtime, DXK = a.dxk, DYK = a.dyk;
    const double fr = sd.frund, rfr = sd.rfrund;
    const bool rok = sd.rcp_ok != 0;
    const int qz = sd.quantise;
    const long long dW = -(long long)a.nj2;
    const bool du = i > 2, dv = j > 2;
    // Chunks of CH levels: every load of the chunk is issued before its stores.  No level reads
    // what another level writes (DPM is read only; U, V, W are read and written at the same cell),
    // so this only lets the loads overlap instead of queuing behind the previous level's stores.
    constexpr int CH = 4;
    for (int kb = kbeg; kb <= m.vi; kb += CH * kstep) {
        float d[CH], dw[CH], ds[CH], dk[CH], u[CH], v[CH], w[CH];
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int k = kb + q * kstep;
            d[q] = dw[q] = ds[q] = dk[q] = u[q] = v[q] = w[q] = 0.f;
            if (k < 1 || k > m.vi) continue;
            d[q] = a.dpm[x.at(0, k)];
            if (du && m.kkm_u < k) { u[q] = a.uk[x.at(0, k)]; dw[q] = a.dpm[x.at(dW, k)]; }
            if (dv && m.kkm_v < k) { v[q] = a.vk[x.at(0, k)]; ds[q] = a.dpm[x.at(-1, k)]; }
            if (m.kkart + 1 < k) { w[q] = a.wk[x.at(0, k)]; dk[q] = a.dpm[x.at(0, k - 1)]; }
        }
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int k = kb + q * kstep;
            if (k < 1 || k > m.vi) continue;
            if (du && m.kkm_u < k) a.uk[x.at(0, k)] = (float)quantd_r((double)(u[q] + (dw[q] - d[q]) / DXK * DT), fr, rfr, rok, qz);
            if (dv && m.kkm_v < k) a.vk[x.at(0, k)] = (float)quantd_r((double)(v[q] + (ds[q] - d[q]) / DYK * DT), fr, rfr, rok, qz);
            if (m.kkart + 1 < k)
                a.wk[x.at(0, k)] =
                    (float)quantd_r((double)(w[q] + (dk[q] - d[q]) / (a.dzk[k] + a.dzk[k - 1]) * 2 * DT), fr, rfr, rok, qz);
            else
                a.wk[x.at(0, k)] = 0;
        }
    }
}

// staggered -> cell-centre averages and the border copies (PrognosticFlowfield.cs:958-1039)
template <bool IL>
__device__ __forceinline__ void average_col(const KArgs &a, int col, int i, int j, const Acc<IL> &x, int kbeg,
                                            int kstep) {
    if (i < 2 || i > a.nii - 1 || j < 2 || j > a.njj - 1) return;
    if (!(a.cflags[col] & F_VC)) return;
    const ColMeta m = a.meta[col];
    const int nj2 = a.nj2;
    const long long dE = nj2;
    const int KK = m.kkart;
    const bool cpS = (j == 2);
    const bool cpN = (j == a.njj - 1) && (a.cflags[i * nj2 + a.njj] & F_ADV);
    // chunks of CH levels with their loads first, as in velcorr_col (UK, VK, WK are only read
    // here; the border copies take this column's UKS, new or, inside the obstacle, the old value)
    constexpr int CH = 4;
    for (int kb = kbeg; kb <= m.vi; kb += CH * kstep) {
        float u0[CH], u1[CH], v0[CH], v1[CH], w0[CH], w1[CH], uo[CH];
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int k = kb + q * kstep;
            u0[q] = u1[q] = v0[q] = v1[q] = w0[q] = w1[q] = uo[q] = 0.f;
            if (k < m.kstart || k > m.vi) continue;
            if (KK < k) {
                u0[q] = a.uk[x.at(0, k)]; u1[q] = a.uk[x.at(dE, k)];
                v0[q] = a.vk[x.at(0, k)]; v1[q] = a.vk[x.at(1, k)];
            } else if (cpS || cpN) {
                uo[q] = a.uks[x.at(0, k)];
            }
            if (KK + 1 < k) { w0[q] = a.wk[x.at(0, k)]; w1[q] = a.wk[x.at(0, k + 1)]; }
        }
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int k = kb + q * kstep;
            if (k < m.kstart || k > m.vi) continue;
            float us = uo[q];
            if (KK < k) {
                us = 0.5f * (u0[q] + u1[q]);
                a.uks[x.at(0, k)] = us;
                a.vks[x.at(0, k)] = 0.5f * (v0[q] + v1[q]);
            }
            if (KK + 1 < k) a.wks[x.at(0, k)] = 0.5f * (w0[q] + w1[q]);
            if (cpS) a.uks[x.at(-1, k)] = us;
            if (cpN) a.uks[x.at(1, k)] = us;
        }
    }
    // VKS[1][j] = VKS[2][j] and VKS[NII][j] = VKS[NII-1][j] on every level (:1018-1036)
    const bool west = (i == 2) && (a.cflags[1 * nj2 + j] & F_ADV);
    const bool east = (i == a.nii - 1) && (a.cflags[col] & F_ADV);
    if (west || east) {
        const long long dd = west ? -(long long)nj2 : dE;
#pragma unroll 4
        for (int k = kbeg; k < a.ks; k += kstep) a.vks[x.at(dd, k)] = a.vks[x.at(0, k)];
    }
}

}  // namespace gral
