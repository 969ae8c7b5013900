// adj_level.cuh -- one level of the model-1 (mixing-length) momentum equations as a function of
// its inputs, and its hand-derived vector-Jacobian product, for the discrete adjoint.
//
// The forward maps the inputs x[] of one level k of one column (the swept component's own old
// value and its vertical neighbours, the other components of the column, the staggered averages
// of the 3x3 neighbourhood, DPMNEW, VEG and the four horizontal neighbours of the swept field) to
// the row of the vertical tridiagonal system: A (AIM), B (BIM), C (CIM) and D (DIM), exactly as the
// library's solver evaluates them for parity width 8 (U-prognostic-microscale_1.cs:205-470,
// V-prognostic-microscale_1.cs:205-488, W-prognostic-microscale_1.cs:205-402): mixing-length
// viscosity, Patankar power law per face, pressure gradient, Coriolis, vegetation drag, the wall
// law at KKART+1 and the extra eddy-viscosity terms of the SIMD-chunk levels.
//
// The VJP takes the cotangents (lA, lB, lC, lD) of that row and adds d(row)/dx^T * l to gx[].  At
// the kinks of max, min and |.| it follows the branch the forward takes (a subgradient), except at
// a zero face flux, where the power law is smooth and its derivative is used; the square root's
// derivative is taken as zero where its argument is zero.
//
// Both are templates on the arithmetic type: float on the GPU, double in the host-side check of
// the derivatives against central differences of the forward.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define GRAL_HD __host__ __device__ __forceinline__
#else
#define GRAL_HD inline
#endif

namespace gral {
namespace adj {

// column flags used by the level (the F_* bits of prog_common.cuh)
enum : uint32_t {
    LF_VEG = 1u << 2, LF_CUTKLT1 = 1u << 4, LF_BS = 1u << 7, LF_BN = 1u << 8, LF_BW = 1u << 9, LF_BE = 1u << 10,
    LF_Z0GE = 1u << 11,
};

// Constants of one level of one column.
struct LevelConst {
    float dz, dxdz, dydz;      // DZK[k], DXK*DZK[k], DYK*DZK[k]
    float dxk, dyk, area;      // DXK, DYK, DXK*DYK
    float ap0, vishmin, cor, geo;   // AP0[k], VISHMIN, Coriolis, UG (U) or VG (V)
    float hok, hokK, cov;      // HOKART[k], HOKART[KKART], COV
    float help_t, help_o;      // UsternTerrain/ObstaclesHelpterm
    int k, KK, kad, wlo, whi;  // level, KKART, first ADD_DIFF level, wall-chunk levels
    uint32_t fl;               // column flags
};

// Inputs of a U level.  (dc, dk) in the comments: column offset and level offset.
enum UIn {
    U_PHI, U_UKP, U_UKM, U_VKP, U_VKM,                 // UK (0,0) (0,+1) (0,-1); VK (0,+1) (0,-1)
    U_UKS, U_VKS, U_WKS,                               // (0,0)
    U_UKSW, U_VKSW, U_VKSWS, U_VKSS, U_VKSWN, U_VKSN,  // UKS W; VKS W, W+S, S, W+N, N
    U_WKSW, U_WKSWT, U_WKST, U_WKSB, U_WKSWB,          // WKS W, (W,+1), (0,+1), (0,-1), (W,-1)
    U_DPW, U_DP0,                                      // DPMNEW W, (0,0)
    U_VKSEN, U_VKSES, U_WKE, U_WKEB,                   // VKS E+N, E+S; WK E, (E,-1)
    U_VEG,                                             // VEG (0,-1)
    U_AW, U_A0, U_BW, U_B0,                            // wall law: UKS W, UKS 0, VKS W, VKS 0 at its level
    U_NW, U_NS, U_NE, U_NN,                            // UK W, S, E, N
    U_COUNT
};
// Inputs of a V level.
enum VIn {
    V_PHI, V_UKP, V_UKM, V_VKP, V_VKM,                 // VK (0,0); UK (0,+1) (0,-1); VK (0,+1) (0,-1)
    V_UKS, V_VKS, V_WKS,
    V_UKSE, V_UKSS, V_UKSES, V_UKSW, V_VKSW, V_UKSWS,  // UKS E, S, E+S, W; VKS W; UKS W+S
    V_VKSS, V_WKSS, V_WKSB, V_WKSST, V_WKST, V_WKSSB,  // VKS S; WKS S, (0,-1), (S,+1), (0,+1), (S,-1)
    V_DPS, V_DP0,                                      // DPMNEW S, (0,0)
    V_UKSEN, V_UKSWN, V_WKN, V_WKNB,                   // UKS E+N, W+N; WK N, (N,-1)
    V_VEG,
    V_AW, V_A0, V_BW, V_B0,
    V_NW, V_NS, V_NE, V_NN,                            // VK W, S, E, N
    V_COUNT
};
// Inputs of a W level.
enum WIn {
    W_PHI, W_UKP, W_UKM, W_VKP, W_VKM,                 // WK (0,0); UK (0,+1) (0,-1); VK (0,+1) (0,-1)
    W_UKS, W_VKS, W_WKS, W_UKSM, W_VKSM,               // (0,0) and UKS, VKS (0,-1)
    W_UKSW, W_UKSWB, W_VKSS, W_VKSSB, W_UKSE, W_UKSEB, W_VKSN, W_VKSNB,   // (W|S|E|N, 0) and (.., -1)
    W_WKSB, W_DPB, W_DP0,                              // WKS (0,-1); DPMNEW (0,-1), (0,0)
    W_UKST, W_UKSWT, W_VKST, W_VKSST,                  // UKS (0,+1), (W,+1); VKS (0,+1), (S,+1)
    W_WKT, W_WKB,                                      // WK (0,+1), (0,-1)
    W_VEG,
    W_NW, W_NS, W_NE, W_NN,                            // WK W, S, E, N
    W_COUNT
};

template <class T> GRAL_HD T tmax(T a, T b) { return (a > b) ? a : b; }
template <class T> GRAL_HD T tmin(T a, T b) { return (a < b) ? a : b; }
template <class T> GRAL_HD T tsqrt(T x) { return std::sqrt(x); }
#ifdef __CUDA_ARCH__
template <> __device__ __forceinline__ float tsqrt<float>(float x) { return sqrtf(x); }
#endif
template <class T> GRAL_HD T tabs(T x) { return x < T(0) ? -x : x; }

// Power law of one face: a = D*max(0, (1 - 0.1|F/D|)^5) + max(s*F, 0), D = max(D0, 1e-4).
template <class T>
GRAL_HD T face(T D0, T F, int sgn) {
    const T D = tmax(D0, T(0.0001f));
    const T P = tabs(F / D);
    const T in = T(1.0f) - T(0.1f) * P;
    const T Fs = sgn > 0 ? F : -F;
    return D * tmax(T(0.0f), in * in * in * in * in) + tmax(Fs, T(0.0f));
}
// its cotangents: adds da/dD0 * la to gD0 and da/dF * la to gF
template <class T>
GRAL_HD void face_vjp(T D0, T F, int sgn, T la, T &gD0, T &gF) {
    const T D = tmax(D0, T(0.0001f));
    const T q = F / D;
    const T P = tabs(q);
    const T in = T(1.0f) - T(0.1f) * P;
    const T i2 = in * in, i4 = i2 * i2, g5 = i4 * in;
    const T Fs = sgn > 0 ? F : -F;
    T gD = la * tmax(T(0.0f), g5);
    if (!(T(0.0f) > g5)) {                 // max(0, g5) = g5
        const T lP = -T(0.1f) * la * D * T(5.0f) * i4;
        const T lq = (q < T(0.0f)) ? -lP : (q > T(0.0f) ? lP : T(0.0f));
        gF += lq / D;
        gD -= lq * q / D;
    }
    // max(s*F, 0): at F = 0 the mean of the one-sided derivatives, with which the kinks of |F| and
    // max cancel (the coefficient is smooth there: da/dF = s/2)
    if (Fs > T(0.0f)) gF += (sgn > 0) ? la : -la;
    else if (Fs == T(0.0f)) gF += (sgn > 0) ? T(0.5f) * la : -T(0.5f) * la;
    if (D0 > T(0.0001f)) gD0 += gD;
}

// Mixing-length viscosity (zero at and below KKART+1) from the column's U and V at k+1, k-1.
template <class T>
GRAL_HD T vis(const LevelConst &c, T ukp, T ukm, T vkp, T vkm) {
    if (c.k <= c.KK + 1) return T(0.0f);
    const float zs = c.hok - c.hokK - c.dz * 0.5f;
    float mixL = (0.071f * zs < 100.0f) ? 0.071f * zs : 100.0f;
    if (c.cov > 0) mixL *= (1.0f - 0.99f * c.cov);
    const T iu = (ukp - ukm) / T(2.0f * c.dz), iv = (vkp - vkm) / T(2.0f * c.dz);
    return tmin(T(mixL) * T(mixL) * tsqrt(T(0.5f) * (iu * iu + iv * iv)), T(15.0f));
}
template <class T>
GRAL_HD void vis_vjp(const LevelConst &c, T ukp, T ukm, T vkp, T vkm, T lvis, T &gukp, T &gukm, T &gvkp, T &gvkm) {
    if (c.k <= c.KK + 1) return;
    const float zs = c.hok - c.hokK - c.dz * 0.5f;
    float mixL = (0.071f * zs < 100.0f) ? 0.071f * zs : 100.0f;
    if (c.cov > 0) mixL *= (1.0f - 0.99f * c.cov);
    const T iu = (ukp - ukm) / T(2.0f * c.dz), iv = (vkp - vkm) / T(2.0f * c.dz);
    const T s = tsqrt(T(0.5f) * (iu * iu + iv * iv));
    const T m2 = T(mixL) * T(mixL);
    if (!(m2 * s < T(15.0f)) || !(s > T(0.0f))) return;
    const T ls = lvis * m2;
    const T liu = ls * T(0.5f) * iu / s, liv = ls * T(0.5f) * iv / s;
    const T r = T(1.0f) / T(2.0f * c.dz);
    gukp += liu * r; gukm -= liu * r; gvkp += liv * r; gvkm -= liv * r;
}

// The six face diffusions before their 1e-4 floor, from max(VIS, VISHMIN) (zeroed at the
// sub-domain borders); order E, W, S, N, T, B.
template <class T>
GRAL_HD void diffusions(const LevelConst &c, T vmx, T d[6]) {
    d[0] = vmx * T(c.dydz) / T(c.dxk);
    d[1] = d[0];
    d[2] = vmx * T(c.dxdz) / T(c.dyk);
    d[3] = d[2];
    d[4] = vmx * T(c.area) / T(c.dz);
    d[5] = (c.k > c.KK + 1) ? d[4] : T(0.0f);
    if (c.fl & LF_BS) d[2] = T(0.0f);
    if (c.fl & LF_BN) d[3] = T(0.0f);
    if (c.fl & LF_BW) d[1] = T(0.0f);
    if (c.fl & LF_BE) d[0] = T(0.0f);
}
// cotangent of vmx from those of the six diffusions
template <class T>
GRAL_HD T diffusions_vjp(const LevelConst &c, const T ld[6]) {
    T g = T(0.0f);
    if (!(c.fl & LF_BE)) g += ld[0] * T(c.dydz) / T(c.dxk);
    if (!(c.fl & LF_BW)) g += ld[1] * T(c.dydz) / T(c.dxk);
    if (!(c.fl & LF_BS)) g += ld[2] * T(c.dxdz) / T(c.dyk);
    if (!(c.fl & LF_BN)) g += ld[3] * T(c.dxdz) / T(c.dyk);
    g += ld[4] * T(c.area) / T(c.dz);
    if (c.k > c.KK + 1) g += ld[5] * T(c.area) / T(c.dz);
    return g;
}

// |u_h| at the cell from the staggered averages: max(sqrt(in^2 + in2^2), floor)
template <class T>
GRAL_HD T speed(T in, T in2, float floor) { return tmax(tsqrt(in * in + in2 * in2), T(floor)); }
template <class T>
GRAL_HD void speed_vjp(T in, T in2, float floor, T l, T &gin, T &gin2) {
    const T r = tsqrt(in * in + in2 * in2);
    if (!(r > T(floor)) || !(r > T(0.0f))) return;
    gin += l * in / r;
    gin2 += l * in2 / r;
}

// Friction velocity of the wall law from the averages a1 = 0.5(UKS_W + UKS), b1 = 0.5(VKS_W + VKS)
// at the wall law's level (U-prognostic-microscale_1.cs:419-450).
template <class T>
GRAL_HD T ustern(const LevelConst &c, T a1, T b1) {
    if (c.fl & LF_CUTKLT1) {
        if (c.fl & LF_Z0GE) return T(c.help_t) * tsqrt(a1 * a1 + b1 * b1);
        return T(c.help_t) * tmax(tsqrt(a1 * a1 + b1 * b1), T(0.1f));
    }
    return T(c.help_o) * tmax(tsqrt(a1 * a1 + b1 * b1), T(0.1f));
}
template <class T>
GRAL_HD void ustern_vjp(const LevelConst &c, T a1, T b1, T l, T &ga1, T &gb1) {
    const T r = tsqrt(a1 * a1 + b1 * b1);
    if (!(r > T(0.0f))) return;
    const bool clamp = !((c.fl & LF_CUTKLT1) && (c.fl & LF_Z0GE));
    if (clamp && !(r > T(0.1f))) return;
    const T h = T((c.fl & LF_CUTKLT1) ? c.help_t : c.help_o);
    ga1 += l * h * a1 / r;
    gb1 += l * h * b1 / r;
}

// ----------------------------------------------------------------------------------------------
// U
// ----------------------------------------------------------------------------------------------
// out[0..3] = A, B, C, D; out[4..7] = dD/d(nW, nS, nE, nN), the coefficients of the four horizontal
// neighbours of the swept field in D (D is linear in them).
template <class T>
GRAL_HD void u_row(const LevelConst &c, const T *x, T out[8]) {
    const T VIS = vis(c, x[U_UKP], x[U_UKM], x[U_VKP], x[U_VKM]);
    const T vmx = tmax(VIS, T(c.vishmin));
    T d[6];
    diffusions(c, vmx, d);
    const T dydz = T(c.dydz), dxdz = T(c.dxdz), area = T(c.area);
    const T FE = x[U_UKS] * dydz, FW = x[U_UKSW] * dydz;
    const T FS = T(0.25f) * (x[U_VKSW] + x[U_VKS] + x[U_VKSWS] + x[U_VKSS]) * dxdz;
    const T FN = T(0.25f) * (x[U_VKSW] + x[U_VKS] + x[U_VKSWN] + x[U_VKSN]) * dxdz;
    const T FT = T(0.25f) * (x[U_WKSW] + x[U_WKS] + x[U_WKSWT] + x[U_WKST]) * area;
    const T FB = (c.k > c.KK + 1) ? T(0.25f) * (x[U_WKSW] + x[U_WKS] + x[U_WKSWB] + x[U_WKSB]) * area : T(0.0f);
    const T B = face(d[4], FT, -1), C = face(d[5], FB, 1);
    const T ae = face(d[0], FE, -1), aw = face(d[1], FW, 1), as = face(d[2], FS, 1), an = face(d[3], FN, -1);
    const T ap0 = T(c.ap0);
    const T A = B + C + aw + as + ae + an + ap0;
    const T uk = x[U_PHI];
    const T t1 = ap0 * T(0.5f) * (x[U_UKSW] + x[U_UKS]);
    const T t2 = (x[U_DPW] - x[U_DP0]) * dydz;
    const T in = T(0.5f) * (x[U_UKSW] + x[U_UKS]), in2 = T(0.5f) * (x[U_VKSW] + x[U_VKS]);
    T t3;
    if (c.fl & LF_VEG) t3 = (T(c.cor) * (T(c.geo) - uk) - x[U_VEG] * uk * speed(in, in2, 0.01f)) * area * T(c.dz);
    else t3 = T(c.cor) * (T(c.geo) - uk) * area * T(c.dz);
    T D = aw * x[U_NW] + as * x[U_NS] + ae * x[U_NE] + an * x[U_NN] + t1 + t2 + t3;
    if (c.k >= c.wlo && c.k <= c.whi && c.k == c.KK + 1) {
        const T wh = speed(in, in2, 0.1f);
        const T Ust = ustern(c, T(0.5f) * (x[U_AW] + x[U_A0]), T(0.5f) * (x[U_BW] + x[U_B0]));
        D -= uk / wh * (Ust * Ust) * area;
    }
    out[4] = aw; out[5] = as; out[6] = ae; out[7] = an;
    if (c.k >= c.kad) {
        const T hz = dydz;
        const T e0 = (T(0.5f) * (x[U_VKSEN] + x[U_VKSN]) - T(0.5f) * (x[U_VKSN] + x[U_VKSWN])) * dxdz;
        const T e1 = (T(0.5f) * (x[U_VKSES] + x[U_VKSS]) - T(0.5f) * (x[U_VKSS] + x[U_VKSWS])) * dxdz;
        const T e2 = (T(0.5f) * (x[U_WKE] + x[U_WKS]) - T(0.5f) * (x[U_WKS] + x[U_WKSW])) * area;
        const T e3 = (T(0.5f) * (x[U_WKEB] + x[U_WKSB]) - T(0.5f) * (x[U_WKSB] + x[U_WKSWB])) * area;
        D += VIS / T(c.dxk) * ((x[U_NE] - uk) * hz - (uk - x[U_NW]) * hz + e0 - e1 + e2 - e3);
        out[4] += VIS / T(c.dxk) * hz;
        out[6] += VIS / T(c.dxk) * hz;
    }
    out[0] = A; out[1] = B; out[2] = C; out[3] = D;
}

template <class T>
GRAL_HD void u_row_vjp(const LevelConst &c, const T *x, const T l[4], T *g) {
    const T lA = l[0], lD = l[3];
    const T VIS = vis(c, x[U_UKP], x[U_UKM], x[U_VKP], x[U_VKM]);
    const T vmx = tmax(VIS, T(c.vishmin));
    T d[6];
    diffusions(c, vmx, d);
    const T dydz = T(c.dydz), dxdz = T(c.dxdz), area = T(c.area), dz = T(c.dz);
    const T FE = x[U_UKS] * dydz, FW = x[U_UKSW] * dydz;
    const T FS = T(0.25f) * (x[U_VKSW] + x[U_VKS] + x[U_VKSWS] + x[U_VKSS]) * dxdz;
    const T FN = T(0.25f) * (x[U_VKSW] + x[U_VKS] + x[U_VKSWN] + x[U_VKSN]) * dxdz;
    const T FT = T(0.25f) * (x[U_WKSW] + x[U_WKS] + x[U_WKSWT] + x[U_WKST]) * area;
    const bool haveB = c.k > c.KK + 1;
    const T FB = haveB ? T(0.25f) * (x[U_WKSW] + x[U_WKS] + x[U_WKSWB] + x[U_WKSB]) * area : T(0.0f);
    const T ae = face(d[0], FE, -1), aw = face(d[1], FW, 1), as = face(d[2], FS, 1), an = face(d[3], FN, -1);
    const T uk = x[U_PHI];
    // D's neighbour products
    g[U_NW] += lD * aw; g[U_NS] += lD * as; g[U_NE] += lD * ae; g[U_NN] += lD * an;
    const T law = lA + lD * x[U_NW], las = lA + lD * x[U_NS], lae = lA + lD * x[U_NE], lan = lA + lD * x[U_NN];
    const T lB = lA + l[1], lC = lA + l[2];
    // t1, t2
    g[U_UKSW] += lD * T(c.ap0) * T(0.5f);
    g[U_UKS] += lD * T(c.ap0) * T(0.5f);
    g[U_DPW] += lD * dydz;
    g[U_DP0] -= lD * dydz;
    // t3
    const T in = T(0.5f) * (x[U_UKSW] + x[U_UKS]), in2 = T(0.5f) * (x[U_VKSW] + x[U_VKS]);
    T gin = T(0.0f), gin2 = T(0.0f);
    if (c.fl & LF_VEG) {
        const T wv = speed(in, in2, 0.01f);
        g[U_PHI] += lD * (-T(c.cor) - x[U_VEG] * wv) * area * dz;
        g[U_VEG] -= lD * uk * wv * area * dz;
        speed_vjp(in, in2, 0.01f, -lD * x[U_VEG] * uk * area * dz, gin, gin2);
    } else {
        g[U_PHI] -= lD * T(c.cor) * area * dz;
    }
    // wall law
    if (c.k >= c.wlo && c.k <= c.whi && c.k == c.KK + 1) {
        const T wh = speed(in, in2, 0.1f);
        const T a1 = T(0.5f) * (x[U_AW] + x[U_A0]), b1 = T(0.5f) * (x[U_BW] + x[U_B0]);
        const T Ust = ustern(c, a1, b1);
        const T U2 = Ust * Ust;
        const T lw = -lD;
        g[U_PHI] += lw * U2 * area / wh;
        speed_vjp(in, in2, 0.1f, -lw * uk * U2 * area / (wh * wh), gin, gin2);
        T ga1 = T(0.0f), gb1 = T(0.0f);
        ustern_vjp(c, a1, b1, lw * uk / wh * area * T(2.0f) * Ust, ga1, gb1);
        g[U_AW] += T(0.5f) * ga1; g[U_A0] += T(0.5f) * ga1;
        g[U_BW] += T(0.5f) * gb1; g[U_B0] += T(0.5f) * gb1;
    }
    g[U_UKSW] += T(0.5f) * gin; g[U_UKS] += T(0.5f) * gin;
    g[U_VKSW] += T(0.5f) * gin2; g[U_VKS] += T(0.5f) * gin2;
    // extra eddy-viscosity terms
    T lvis = T(0.0f);
    if (c.k >= c.kad) {
        const T hz = dydz;
        const T e0 = (T(0.5f) * (x[U_VKSEN] + x[U_VKSN]) - T(0.5f) * (x[U_VKSN] + x[U_VKSWN])) * dxdz;
        const T e1 = (T(0.5f) * (x[U_VKSES] + x[U_VKSS]) - T(0.5f) * (x[U_VKSS] + x[U_VKSWS])) * dxdz;
        const T e2 = (T(0.5f) * (x[U_WKE] + x[U_WKS]) - T(0.5f) * (x[U_WKS] + x[U_WKSW])) * area;
        const T e3 = (T(0.5f) * (x[U_WKEB] + x[U_WKSB]) - T(0.5f) * (x[U_WKSB] + x[U_WKSWB])) * area;
        const T X = (x[U_NE] - uk) * hz - (uk - x[U_NW]) * hz + e0 - e1 + e2 - e3;
        lvis += lD * X / T(c.dxk);
        const T q = lD * VIS / T(c.dxk);
        g[U_NE] += q * hz; g[U_NW] += q * hz; g[U_PHI] -= T(2.0f) * q * hz;
        g[U_VKSEN] += q * T(0.5f) * dxdz; g[U_VKSWN] -= q * T(0.5f) * dxdz;
        g[U_VKSES] -= q * T(0.5f) * dxdz; g[U_VKSWS] += q * T(0.5f) * dxdz;
        g[U_WKE] += q * T(0.5f) * area; g[U_WKSW] -= q * T(0.5f) * area;
        g[U_WKEB] -= q * T(0.5f) * area; g[U_WKSWB] += q * T(0.5f) * area;
    }
    // faces
    T ld[6] = {T(0.0f), T(0.0f), T(0.0f), T(0.0f), T(0.0f), T(0.0f)};
    T gFE = T(0.0f), gFW = T(0.0f), gFS = T(0.0f), gFN = T(0.0f), gFT = T(0.0f), gFB = T(0.0f);
    face_vjp(d[4], FT, -1, lB, ld[4], gFT);
    face_vjp(d[5], FB, 1, lC, ld[5], gFB);
    face_vjp(d[0], FE, -1, lae, ld[0], gFE);
    face_vjp(d[1], FW, 1, law, ld[1], gFW);
    face_vjp(d[2], FS, 1, las, ld[2], gFS);
    face_vjp(d[3], FN, -1, lan, ld[3], gFN);
    g[U_UKS] += gFE * dydz;
    g[U_UKSW] += gFW * dydz;
    const T s4 = T(0.25f) * dxdz;
    g[U_VKSW] += (gFS + gFN) * s4; g[U_VKS] += (gFS + gFN) * s4;
    g[U_VKSWS] += gFS * s4; g[U_VKSS] += gFS * s4; g[U_VKSWN] += gFN * s4; g[U_VKSN] += gFN * s4;
    const T a4 = T(0.25f) * area;
    g[U_WKSW] += gFT * a4; g[U_WKS] += gFT * a4; g[U_WKSWT] += gFT * a4; g[U_WKST] += gFT * a4;
    if (haveB) { g[U_WKSW] += gFB * a4; g[U_WKS] += gFB * a4; g[U_WKSWB] += gFB * a4; g[U_WKSB] += gFB * a4; }
    const T lvmx = diffusions_vjp(c, ld);
    if (VIS > T(c.vishmin)) lvis += lvmx;
    vis_vjp(c, x[U_UKP], x[U_UKM], x[U_VKP], x[U_VKM], lvis, g[U_UKP], g[U_UKM], g[U_VKP], g[U_VKM]);
}

// ----------------------------------------------------------------------------------------------
// V
// ----------------------------------------------------------------------------------------------
template <class T>
GRAL_HD void v_row(const LevelConst &c, const T *x, T out[8]) {
    const T VIS = vis(c, x[V_UKP], x[V_UKM], x[V_VKP], x[V_VKM]);
    const T vmx = tmax(VIS, T(c.vishmin));
    T d[6];
    diffusions(c, vmx, d);
    const T dydz = T(c.dydz), dxdz = T(c.dxdz), area = T(c.area);
    const T FE = T(0.25f) * (x[V_UKS] + x[V_UKSE] + x[V_UKSS] + x[V_UKSES]) * dydz;
    const T FW = T(0.25f) * (x[V_UKS] + x[V_UKSW] + x[V_UKSS] + x[V_UKSWS]) * dydz;
    const T FS = x[V_VKSS] * dxdz, FN = x[V_VKS] * dxdz;
    const T FT = T(0.25f) * (x[V_WKSS] + x[V_WKS] + x[V_WKSST] + x[V_WKST]) * area;
    const T FB = (c.k > c.KK + 1) ? T(0.25f) * (x[V_WKSS] + x[V_WKS] + x[V_WKSSB] + x[V_WKSB]) * area : T(0.0f);
    const T B = face(d[4], FT, -1), C = face(d[5], FB, 1);
    const T ae = face(d[0], FE, -1), aw = face(d[1], FW, 1), as = face(d[2], FS, 1), an = face(d[3], FN, -1);
    const T ap0 = T(c.ap0);
    const T A = B + C + aw + as + ae + an + ap0;
    const T vk = x[V_PHI];
    const T t1 = ap0 * T(0.5f) * (x[V_VKSS] + x[V_VKS]);
    const T t2 = (x[V_DPS] - x[V_DP0]) * dxdz;
    const T in = T(0.5f) * (x[V_UKSW] + x[V_UKS]), in2 = T(0.5f) * (x[V_VKSW] + x[V_VKS]);
    T t3;
    if (c.fl & LF_VEG) t3 = (T(c.cor) * (T(c.geo) - vk) - x[V_VEG] * vk * speed(in, in2, 0.01f)) * area * T(c.dz);
    else t3 = T(c.cor) * (T(c.geo) - vk) * area * T(c.dz);
    T D = aw * x[V_NW] + as * x[V_NS] + ae * x[V_NE] + an * x[V_NN] + t1 + t2 + t3;
    out[4] = aw; out[5] = as; out[6] = ae; out[7] = an;
    if (c.k >= c.wlo && c.k <= c.whi && c.k == c.KK + 1) {
        const T wh = speed(in, in2, 0.1f);
        const T Ust = ustern(c, T(0.5f) * (x[V_AW] + x[V_A0]), T(0.5f) * (x[V_BW] + x[V_B0]));
        D -= vk / wh * (Ust * Ust) * area;
    }
    if (c.k >= c.kad) {
        const T hz = dxdz;
        const T dudye = (T(0.5f) * (x[V_UKSEN] + x[V_UKSE]) - T(0.5f) * (x[V_UKSE] + x[V_UKSES])) * dxdz;
        const T dudyw = (T(0.5f) * (x[V_UKSWN] + x[V_UKSW]) - T(0.5f) * (x[V_UKSW] + x[V_UKSWS])) * dxdz;
        const T e0 = dudye - dudyw;
        const T e1 = (T(0.5f) * (x[V_WKN] + x[V_WKS]) - T(0.5f) * (x[V_WKS] + x[V_WKSS])) * area;
        const T e2 = (T(0.5f) * (x[V_WKNB] + x[V_WKSB]) - T(0.5f) * (x[V_WKSB] + x[V_WKSS])) * area;
        D += VIS / T(c.dxk) * (e0 + (x[V_NN] - vk) * hz - (vk - x[V_NS]) * hz + e1 - e2);
        out[5] += VIS / T(c.dxk) * hz;
        out[7] += VIS / T(c.dxk) * hz;
    }
    out[0] = A; out[1] = B; out[2] = C; out[3] = D;
}

template <class T>
GRAL_HD void v_row_vjp(const LevelConst &c, const T *x, const T l[4], T *g) {
    const T lA = l[0], lD = l[3];
    const T VIS = vis(c, x[V_UKP], x[V_UKM], x[V_VKP], x[V_VKM]);
    const T vmx = tmax(VIS, T(c.vishmin));
    T d[6];
    diffusions(c, vmx, d);
    const T dydz = T(c.dydz), dxdz = T(c.dxdz), area = T(c.area), dz = T(c.dz);
    const T FE = T(0.25f) * (x[V_UKS] + x[V_UKSE] + x[V_UKSS] + x[V_UKSES]) * dydz;
    const T FW = T(0.25f) * (x[V_UKS] + x[V_UKSW] + x[V_UKSS] + x[V_UKSWS]) * dydz;
    const T FS = x[V_VKSS] * dxdz, FN = x[V_VKS] * dxdz;
    const T FT = T(0.25f) * (x[V_WKSS] + x[V_WKS] + x[V_WKSST] + x[V_WKST]) * area;
    const bool haveB = c.k > c.KK + 1;
    const T FB = haveB ? T(0.25f) * (x[V_WKSS] + x[V_WKS] + x[V_WKSSB] + x[V_WKSB]) * area : T(0.0f);
    const T ae = face(d[0], FE, -1), aw = face(d[1], FW, 1), as = face(d[2], FS, 1), an = face(d[3], FN, -1);
    const T vk = x[V_PHI];
    g[V_NW] += lD * aw; g[V_NS] += lD * as; g[V_NE] += lD * ae; g[V_NN] += lD * an;
    const T law = lA + lD * x[V_NW], las = lA + lD * x[V_NS], lae = lA + lD * x[V_NE], lan = lA + lD * x[V_NN];
    const T lB = lA + l[1], lC = lA + l[2];
    g[V_VKSS] += lD * T(c.ap0) * T(0.5f);
    g[V_VKS] += lD * T(c.ap0) * T(0.5f);
    g[V_DPS] += lD * dxdz;
    g[V_DP0] -= lD * dxdz;
    const T in = T(0.5f) * (x[V_UKSW] + x[V_UKS]), in2 = T(0.5f) * (x[V_VKSW] + x[V_VKS]);
    T gin = T(0.0f), gin2 = T(0.0f);
    if (c.fl & LF_VEG) {
        const T wv = speed(in, in2, 0.01f);
        g[V_PHI] += lD * (-T(c.cor) - x[V_VEG] * wv) * area * dz;
        g[V_VEG] -= lD * vk * wv * area * dz;
        speed_vjp(in, in2, 0.01f, -lD * x[V_VEG] * vk * area * dz, gin, gin2);
    } else {
        g[V_PHI] -= lD * T(c.cor) * area * dz;
    }
    if (c.k >= c.wlo && c.k <= c.whi && c.k == c.KK + 1) {
        const T wh = speed(in, in2, 0.1f);
        const T a1 = T(0.5f) * (x[V_AW] + x[V_A0]), b1 = T(0.5f) * (x[V_BW] + x[V_B0]);
        const T Ust = ustern(c, a1, b1);
        const T U2 = Ust * Ust;
        const T lw = -lD;
        g[V_PHI] += lw * U2 * area / wh;
        speed_vjp(in, in2, 0.1f, -lw * vk * U2 * area / (wh * wh), gin, gin2);
        T ga1 = T(0.0f), gb1 = T(0.0f);
        ustern_vjp(c, a1, b1, lw * vk / wh * area * T(2.0f) * Ust, ga1, gb1);
        g[V_AW] += T(0.5f) * ga1; g[V_A0] += T(0.5f) * ga1;
        g[V_BW] += T(0.5f) * gb1; g[V_B0] += T(0.5f) * gb1;
    }
    g[V_UKSW] += T(0.5f) * gin; g[V_UKS] += T(0.5f) * gin;
    g[V_VKSW] += T(0.5f) * gin2; g[V_VKS] += T(0.5f) * gin2;
    T lvis = T(0.0f);
    if (c.k >= c.kad) {
        const T hz = dxdz;
        const T dudye = (T(0.5f) * (x[V_UKSEN] + x[V_UKSE]) - T(0.5f) * (x[V_UKSE] + x[V_UKSES])) * dxdz;
        const T dudyw = (T(0.5f) * (x[V_UKSWN] + x[V_UKSW]) - T(0.5f) * (x[V_UKSW] + x[V_UKSWS])) * dxdz;
        const T e0 = dudye - dudyw;
        const T e1 = (T(0.5f) * (x[V_WKN] + x[V_WKS]) - T(0.5f) * (x[V_WKS] + x[V_WKSS])) * area;
        const T e2 = (T(0.5f) * (x[V_WKNB] + x[V_WKSB]) - T(0.5f) * (x[V_WKSB] + x[V_WKSS])) * area;
        const T X = e0 + (x[V_NN] - vk) * hz - (vk - x[V_NS]) * hz + e1 - e2;
        lvis += lD * X / T(c.dxk);
        const T q = lD * VIS / T(c.dxk);
        g[V_NN] += q * hz; g[V_NS] += q * hz; g[V_PHI] -= T(2.0f) * q * hz;
        const T h = q * T(0.5f) * dxdz;
        g[V_UKSEN] += h; g[V_UKSES] -= h; g[V_UKSWN] -= h; g[V_UKSWS] += h;
        const T ha = q * T(0.5f) * area;
        g[V_WKN] += ha; g[V_WKSS] -= ha;       // e1
        g[V_WKNB] -= ha; g[V_WKSS] += ha;      // e2 (its second average takes WKS S at level k)
    }
    T ld[6] = {T(0.0f), T(0.0f), T(0.0f), T(0.0f), T(0.0f), T(0.0f)};
    T gFE = T(0.0f), gFW = T(0.0f), gFS = T(0.0f), gFN = T(0.0f), gFT = T(0.0f), gFB = T(0.0f);
    face_vjp(d[4], FT, -1, lB, ld[4], gFT);
    face_vjp(d[5], FB, 1, lC, ld[5], gFB);
    face_vjp(d[0], FE, -1, lae, ld[0], gFE);
    face_vjp(d[1], FW, 1, law, ld[1], gFW);
    face_vjp(d[2], FS, 1, las, ld[2], gFS);
    face_vjp(d[3], FN, -1, lan, ld[3], gFN);
    const T s4 = T(0.25f) * dydz;
    g[V_UKS] += (gFE + gFW) * s4; g[V_UKSS] += (gFE + gFW) * s4;
    g[V_UKSE] += gFE * s4; g[V_UKSES] += gFE * s4; g[V_UKSW] += gFW * s4; g[V_UKSWS] += gFW * s4;
    g[V_VKSS] += gFS * dxdz;
    g[V_VKS] += gFN * dxdz;
    const T a4 = T(0.25f) * area;
    g[V_WKSS] += gFT * a4; g[V_WKS] += gFT * a4; g[V_WKSST] += gFT * a4; g[V_WKST] += gFT * a4;
    if (haveB) { g[V_WKSS] += gFB * a4; g[V_WKS] += gFB * a4; g[V_WKSSB] += gFB * a4; g[V_WKSB] += gFB * a4; }
    const T lvmx = diffusions_vjp(c, ld);
    if (VIS > T(c.vishmin)) lvis += lvmx;
    vis_vjp(c, x[V_UKP], x[V_UKM], x[V_VKP], x[V_VKM], lvis, g[V_UKP], g[V_UKM], g[V_VKP], g[V_VKM]);
}

// ----------------------------------------------------------------------------------------------
// W
// ----------------------------------------------------------------------------------------------
template <class T>
GRAL_HD void w_row(const LevelConst &c, const T *x, T out[8]) {
    const T VIS = vis(c, x[W_UKP], x[W_UKM], x[W_VKP], x[W_VKM]);
    const T vmx = tmax(VIS, T(c.vishmin));
    T d[6];
    diffusions(c, vmx, d);
    const T dydz = T(c.dydz), dxdz = T(c.dxdz), area = T(c.area);
    const T FE = T(0.25f) * (x[W_UKS] + x[W_UKSE] + x[W_UKSM] + x[W_UKSEB]) * dydz;
    const T FW = T(0.25f) * (x[W_UKS] + x[W_UKSW] + x[W_UKSM] + x[W_UKSWB]) * dydz;
    const T FS = T(0.25f) * (x[W_VKS] + x[W_VKSS] + x[W_VKSM] + x[W_VKSSB]) * dxdz;
    const T FN = T(0.25f) * (x[W_VKS] + x[W_VKSN] + x[W_VKSM] + x[W_VKSNB]) * dxdz;
    const T FT = x[W_WKS] * area;
    const T FB = (c.k > c.KK + 1) ? x[W_WKSB] * area : T(0.0f);
    const T B = face(d[4], FT, -1), C = face(d[5], FB, 1);
    const T ae = face(d[0], FE, -1), aw = face(d[1], FW, 1), as = face(d[2], FS, 1), an = face(d[3], FN, -1);
    const T ap0 = T(c.ap0);
    const T A = B + C + aw + as + ae + an + ap0;
    const T wk = x[W_PHI];
    const T t1 = ap0 * T(0.5f) * (x[W_WKSB] + x[W_WKS]);
    const T t2 = (x[W_DPB] - x[W_DP0]) * area;
    T D = aw * x[W_NW] + as * x[W_NS] + ae * x[W_NE] + an * x[W_NN] + t1 + t2;
    out[4] = aw; out[5] = as; out[6] = ae; out[7] = an;
    if (c.fl & LF_VEG) {
        const T in2 = T(0.5f) * (x[W_VKSS] + x[W_VKS]), in = T(0.5f) * (x[W_UKSW] + x[W_UKS]);
        D = D - x[W_VEG] * wk * speed(in, in2, 0.01f) * area * T(c.dz);
    }
    if (c.k >= c.kad) {
        const T dudze = (T(0.5f) * (x[W_UKST] + x[W_UKS]) - T(0.5f) * (x[W_UKS] + x[W_UKSM])) * dydz;
        const T dudzw = (T(0.5f) * (x[W_UKSWT] + x[W_UKSW]) - T(0.5f) * (x[W_UKSW] + x[W_UKSWB])) * dydz;
        const T dvdzn = (T(0.5f) * (x[W_VKST] + x[W_VKS]) - T(0.5f) * (x[W_VKS] + x[W_VKSM])) * dxdz;
        const T dvdzs = (T(0.5f) * (x[W_VKSST] + x[W_VKSS]) - T(0.5f) * (x[W_VKSS] + x[W_VKSSB])) * dxdz;
        const T dwdzt = (x[W_WKT] - wk) * area, dwdzb = (wk - x[W_WKB]) * area;
        D += VIS / T(c.dz) * (dudze - dudzw + dvdzn - dvdzs + dwdzt - dwdzb);
    }
    out[0] = A; out[1] = B; out[2] = C; out[3] = D;
}

template <class T>
GRAL_HD void w_row_vjp(const LevelConst &c, const T *x, const T l[4], T *g) {
    const T lA = l[0], lD = l[3];
    const T VIS = vis(c, x[W_UKP], x[W_UKM], x[W_VKP], x[W_VKM]);
    const T vmx = tmax(VIS, T(c.vishmin));
    T d[6];
    diffusions(c, vmx, d);
    const T dydz = T(c.dydz), dxdz = T(c.dxdz), area = T(c.area), dz = T(c.dz);
    const T FE = T(0.25f) * (x[W_UKS] + x[W_UKSE] + x[W_UKSM] + x[W_UKSEB]) * dydz;
    const T FW = T(0.25f) * (x[W_UKS] + x[W_UKSW] + x[W_UKSM] + x[W_UKSWB]) * dydz;
    const T FS = T(0.25f) * (x[W_VKS] + x[W_VKSS] + x[W_VKSM] + x[W_VKSSB]) * dxdz;
    const T FN = T(0.25f) * (x[W_VKS] + x[W_VKSN] + x[W_VKSM] + x[W_VKSNB]) * dxdz;
    const T FT = x[W_WKS] * area;
    const bool haveB = c.k > c.KK + 1;
    const T FB = haveB ? x[W_WKSB] * area : T(0.0f);
    const T ae = face(d[0], FE, -1), aw = face(d[1], FW, 1), as = face(d[2], FS, 1), an = face(d[3], FN, -1);
    const T wk = x[W_PHI];
    g[W_NW] += lD * aw; g[W_NS] += lD * as; g[W_NE] += lD * ae; g[W_NN] += lD * an;
    const T law = lA + lD * x[W_NW], las = lA + lD * x[W_NS], lae = lA + lD * x[W_NE], lan = lA + lD * x[W_NN];
    const T lB = lA + l[1], lC = lA + l[2];
    g[W_WKSB] += lD * T(c.ap0) * T(0.5f);
    g[W_WKS] += lD * T(c.ap0) * T(0.5f);
    g[W_DPB] += lD * area;
    g[W_DP0] -= lD * area;
    if (c.fl & LF_VEG) {
        const T in2 = T(0.5f) * (x[W_VKSS] + x[W_VKS]), in = T(0.5f) * (x[W_UKSW] + x[W_UKS]);
        const T wv = speed(in, in2, 0.01f);
        g[W_PHI] -= lD * x[W_VEG] * wv * area * dz;
        g[W_VEG] -= lD * wk * wv * area * dz;
        T gin = T(0.0f), gin2 = T(0.0f);
        speed_vjp(in, in2, 0.01f, -lD * x[W_VEG] * wk * area * dz, gin, gin2);
        g[W_UKSW] += T(0.5f) * gin; g[W_UKS] += T(0.5f) * gin;
        g[W_VKSS] += T(0.5f) * gin2; g[W_VKS] += T(0.5f) * gin2;
    }
    T lvis = T(0.0f);
    if (c.k >= c.kad) {
        const T dudze = (T(0.5f) * (x[W_UKST] + x[W_UKS]) - T(0.5f) * (x[W_UKS] + x[W_UKSM])) * dydz;
        const T dudzw = (T(0.5f) * (x[W_UKSWT] + x[W_UKSW]) - T(0.5f) * (x[W_UKSW] + x[W_UKSWB])) * dydz;
        const T dvdzn = (T(0.5f) * (x[W_VKST] + x[W_VKS]) - T(0.5f) * (x[W_VKS] + x[W_VKSM])) * dxdz;
        const T dvdzs = (T(0.5f) * (x[W_VKSST] + x[W_VKSS]) - T(0.5f) * (x[W_VKSS] + x[W_VKSSB])) * dxdz;
        const T dwdzt = (x[W_WKT] - wk) * area, dwdzb = (wk - x[W_WKB]) * area;
        const T X = dudze - dudzw + dvdzn - dvdzs + dwdzt - dwdzb;
        lvis += lD * X / dz;
        const T q = lD * VIS / dz;
        const T hy = q * T(0.5f) * dydz, hx = q * T(0.5f) * dxdz;
        g[W_UKST] += hy; g[W_UKSM] -= hy;          // dudze = 0.5(T - M) dydz
        g[W_UKSWT] -= hy; g[W_UKSWB] += hy;
        g[W_VKST] += hx; g[W_VKSM] -= hx;
        g[W_VKSSB] += hx; g[W_VKSST] -= hx;
        g[W_WKT] += q * area; g[W_WKB] += q * area; g[W_PHI] -= T(2.0f) * q * area;
    }
    T ld[6] = {T(0.0f), T(0.0f), T(0.0f), T(0.0f), T(0.0f), T(0.0f)};
    T gFE = T(0.0f), gFW = T(0.0f), gFS = T(0.0f), gFN = T(0.0f), gFT = T(0.0f), gFB = T(0.0f);
    face_vjp(d[4], FT, -1, lB, ld[4], gFT);
    face_vjp(d[5], FB, 1, lC, ld[5], gFB);
    face_vjp(d[0], FE, -1, lae, ld[0], gFE);
    face_vjp(d[1], FW, 1, law, ld[1], gFW);
    face_vjp(d[2], FS, 1, las, ld[2], gFS);
    face_vjp(d[3], FN, -1, lan, ld[3], gFN);
    const T y4 = T(0.25f) * dydz, x4 = T(0.25f) * dxdz;
    g[W_UKS] += (gFE + gFW) * y4; g[W_UKSM] += (gFE + gFW) * y4;
    g[W_UKSE] += gFE * y4; g[W_UKSEB] += gFE * y4; g[W_UKSW] += gFW * y4; g[W_UKSWB] += gFW * y4;
    g[W_VKS] += (gFS + gFN) * x4; g[W_VKSM] += (gFS + gFN) * x4;
    g[W_VKSS] += gFS * x4; g[W_VKSSB] += gFS * x4; g[W_VKSN] += gFN * x4; g[W_VKSNB] += gFN * x4;
    g[W_WKS] += gFT * area;
    if (haveB) g[W_WKSB] += gFB * area;
    const T lvmx = diffusions_vjp(c, ld);
    if (VIS > T(c.vishmin)) lvis += lvmx;
    vis_vjp(c, x[W_UKP], x[W_UKM], x[W_VKP], x[W_VKM], lvis, g[W_UKP], g[W_UKM], g[W_VKP], g[W_VKM]);
}

}  // namespace adj
}  // namespace gral
