// prog_kernels.cu -- the Jacobi-style passes of one SIMPLE iteration (boundary conditions,
// velocity correction, staggered averages, convergence bookkeeping), the per-situation set-up and
// the post-checks.  Every pass only writes values that no other thread of the same launch reads,
// exactly as the reference's parallel loops do (their results do not depend on thread order).
//
// Thread mapping follows the layout so that a warp's loads are contiguous:
//   slab layout        one warp per (situation, column), lanes over levels;
//   interleaved layout one warp per (group, column), lane = situation, each lane loops over levels.
#include "prog_common.cuh"
#include "prog_kernels.cuh"
#include "prog_level.cuh"

namespace gral {

namespace {

constexpr int COL_WARPS = 8;   // warps per block of the column kernels

// Slab layout: one warp per (situation, column), lanes over levels.  Interleaved layout: one warp
// per (group, column), lane = situation, looping over the levels -- or, with WIDE, one block per
// (group, column) whose warps share the levels (more loads in flight for bandwidth-bound bodies).
template <bool IL, bool WIDE = false>
inline int col_grid(const KArgs &a) {
    if (IL && WIDE) return a.ngroups * a.ncols;
    const long long warps = (long long)(IL ? a.ngroups : a.nb) * a.ncols;
    return (int)((warps + COL_WARPS - 1) / COL_WARPS);
}

// Calls body(s, col, i, j, x, kbeg, kstep) for every active (situation, column): the body loops
// `for (k = kbeg; k <= hi; k += kstep)` over the levels it needs.
template <bool IL, bool WIDE = false, class Body>
__device__ __forceinline__ void col_loop(const KArgs &a, bool need_active, Body &&body) {
    const int lane = threadIdx.x & 31;
    int s, col, kbeg, kstep;
    // A group holding at most 16 situations runs two levels per warp instruction: lanes 16-31
    // take the odd levels of the situations of lanes 0-15 (the body is expanded for both forms,
    // so each keeps a compile-time level step).
    bool half = false;
    if (IL && WIDE) {
        const int unit = blockIdx.x / a.ncols;
        col = blockIdx.x - unit * a.ncols;
        half = a.nb - unit * 32 <= 16;
        s = unit * 32 + (half ? (lane & 15) : lane);
        if (unit >= a.ngroups || s >= a.nb) return;
        kbeg = threadIdx.x >> 5;
        kstep = COL_WARPS;
    } else {
        const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const long long unit = gw / a.ncols;
        col = (int)(gw - unit * a.ncols);
        if (IL) {
            half = a.nb - (int)unit * 32 <= 16;
            s = (int)unit * 32 + (half ? (lane & 15) : lane);
            if (unit >= a.ngroups || s >= a.nb) return;
            kbeg = 0;
            kstep = 1;
        } else {
            if (unit >= *a.nact) return;
            s = a.act[unit];
            kbeg = lane;
            kstep = 32;
        }
    }
    if (need_active && !a.sit[s].active) return;
    const int i = col / a.nj2, j = col - (col / a.nj2) * a.nj2;
    const Acc<IL> x = make_acc<IL>(a, s, col);
    if (IL && half) {
        if (WIDE) body(s, col, i, j, x, 2 * kbeg + (lane >> 4), 2 * COL_WARPS);
        else body(s, col, i, j, x, lane >> 4, 2);
    } else {
        body(s, col, i, j, x, kbeg, kstep);
    }
}

// ---- boundary conditions (PrognosticFlowfield.cs:595-714) ----
// W/E: one thread per (situation, row j, level) walks the row's events in ascending i, which is
// the reference's sequential i loop; rows and levels are independent.
template <bool IL>
__global__ void k_bc_we(KArgs a, BcLists bc) {
    const int j = 2 + blockIdx.x * blockDim.y + threadIdx.y;
    if (j > a.njj) return;
    int s, kbeg, kstep;
    if (IL) {
        s = blockIdx.y * 32 + threadIdx.x;
        if (blockIdx.y >= a.ngroups || s >= a.nb) return;
        kbeg = 0; kstep = 1;
    } else {
        if ((int)blockIdx.y >= *a.nact) return;
        s = a.act[blockIdx.y];
        kbeg = threadIdx.x; kstep = 32;
    }
    if (!a.sit[s].active) return;
    const int nj2 = a.nj2;
    for (int e = bc.we_ptr[j]; e < bc.we_ptr[j + 1]; ++e) {
        const int ev = bc.we_ev[e];
        const int i = ev & 0xffff;
        const int VI = a.meta[i * nj2 + j].vi;
        const Acc<IL> x = make_acc<IL>(a, s, i * nj2 + j);
        const long long dW = -(long long)nj2, dE = nj2;
        for (int k = kbeg; k <= VI; k += kstep) {
            if (k < 1) continue;
            if (ev & (1 << 16)) {
                const float u = a.uk[x.at(2 * dW, k)];
                if (u >= 0) a.uk[x.at(dW, k)] = u;
                a.vk[x.at(2 * dW, k)] = a.vk[x.at(dW, k)];
                a.wk[x.at(2 * dW, k)] = a.wk[x.at(dW, k)];
            }
            if (ev & (1 << 17)) {
                const float u = a.uk[x.at(2 * dE, k)];
                if (u <= 0) a.uk[x.at(dE, k)] = u;
                a.vk[x.at(dE, k)] = a.vk[x.at(0, k)];
                a.wk[x.at(dE, k)] = a.wk[x.at(0, k)];
            }
        }
    }
}

template <bool IL>
__global__ void k_bc_sn(KArgs a, BcLists bc) {
    const int i = 2 + blockIdx.x * blockDim.y + threadIdx.y;
    if (i > a.nii) return;
    int s, kbeg, kstep;
    if (IL) {
        s = blockIdx.y * 32 + threadIdx.x;
        if (blockIdx.y >= a.ngroups || s >= a.nb) return;
        kbeg = 0; kstep = 1;
    } else {
        if ((int)blockIdx.y >= *a.nact) return;
        s = a.act[blockIdx.y];
        kbeg = threadIdx.x; kstep = 32;
    }
    if (!a.sit[s].active) return;
    const int nj2 = a.nj2;
    for (int e = bc.sn_ptr[i]; e < bc.sn_ptr[i + 1]; ++e) {
        const int ev = bc.sn_ev[e];
        const int j = ev & 0xffff;
        const int VI = a.meta[i * nj2 + j].vi;
        const Acc<IL> x = make_acc<IL>(a, s, i * nj2 + j);
        for (int k = kbeg; k <= VI; k += kstep) {
            if (k < 1) continue;
            if (ev & (1 << 16)) {
                const float v = a.vk[x.at(-2, k)];
                if (v >= 0) a.vk[x.at(-1, k)] = v;
                a.uk[x.at(-2, k)] = a.uk[x.at(-1, k)];
                a.wk[x.at(-2, k)] = a.wk[x.at(-1, k)];
            }
            if (ev & (1 << 17)) {
                const float v = a.vk[x.at(2, k)];
                if (v <= 0) a.vk[x.at(1, k)] = v;
                a.uk[x.at(1, k)] = a.uk[x.at(0, k)];
                a.wk[x.at(1, k)] = a.wk[x.at(0, k)];
            }
        }
    }
}

// top: level VerticalIndex copied to VerticalIndex+1 (:699-714)
template <bool IL>
__global__ void k_bc_top(KArgs a) {
    col_loop<IL>(a, true, [&](int, int col, int i, int j, const Acc<IL> &x, int kbeg, int) {
        if (kbeg != 0) return;
        if (i < 2 || i > a.nii - 1 || j < 2 || j > a.njj - 1) return;
        if (!(a.cflags[col] & F_ADV)) return;
        const int k = a.meta[col].vi;
        a.wk[x.at(0, k + 1)] = a.wk[x.at(0, k)];
        a.uk[x.at(0, k + 1)] = a.uk[x.at(0, k)];
        a.vk[x.at(0, k + 1)] = a.vk[x.at(0, k)];
    });
}

// ---- velocity correction with Frund quantisation in double (:904-949) ----
template <bool IL>
__global__ void k_velcorr(KArgs a) {
    col_loop<IL>(a, true, [&](int s, int col, int i, int j, const Acc<IL> &x, int kbeg, int kstep) {
        velcorr_col<IL>(a, s, col, i, j, x, kbeg, kstep);
    });
}

// ---- staggered -> cell-centre averages and the border copies (:958-1039) ----
template <bool IL>
__global__ void k_average(KArgs a) {
    auto body = [&](int, int col, int i, int j, const Acc<IL> &x, int kbeg, int kstep) {
        average_col<IL>(a, col, i, j, x, kbeg, kstep);
    };
    col_loop<IL, true>(a, true, body);
}

// ---- convergence bookkeeping (:1144-1178), one thread per situation ----
__global__ void k_bookkeeping(KArgs a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) *a.it_global += 1;   // kernels of this launch read SitDev::it, never it_global
    if (s >= a.nb) return;
    SitDev &S = a.sit[s];
    if (!S.active) return;
    const float dumax = S.quantise ? (float)((double)S.dumax_bits / S.frund) : __uint_as_float(S.dumax_bits);
    S.dumax_bits = 0;
    S.last_dumax = dumax;
    const int it = S.it;
    if (a.trace && it - 1 < a.trace_cap) a.trace[(size_t)s * a.trace_cap + it - 1] = dumax;
    const double tw2 = (double)(S.topwind * S.topwind);
    if (it >= S.it_max) S.delta_finish = (float)(S.delta_mean / tw2);
    S.iters_done++;
    if ((it % S.cadence == 0) && (it > 1)) {
        const double d = S.delta_mean / tw2;
        if (it == S.cadence) S.delta_first = (float)d;
        if (S.n_hist < MAX_HIST) S.hist[S.n_hist] = d;
        S.n_hist++;
        if (d < S.conv_threshold && it >= S.it_min) {
            S.converged = 1;
            S.active = 0;
            return;
        }
        S.delta_mean = 0;
    } else {
        S.delta_mean += (double)dumax;
    }
    S.it = it + 1;
    if (S.it > S.it_max) S.active = 0;
}

// ---- set-up on the full-height staging copies (:295-329, 410-432, 518-575) ----
__device__ __forceinline__ size_t sidx3(const KArgs &a, int i, int j, int k) {
    return ((size_t)i * a.nj2 + j) * (a.nkk + 2) + k;
}

// staggered-grid initial values and GESCHW_MAX (:295-329)
template <bool IL>
__global__ void k_setup_uks(KArgs a, Staging sg) {
    col_loop<IL>(a, false, [&](int s, int col, int i, int j, const Acc<IL> &x, int kbeg, int kstep) {
        double g = 0.0;
        if (i >= 1 && i <= a.nii && j >= 1 && j <= a.njj && (a.cflags[col] & F_ALLOC3)) {
            const float *U = sg.uk + sg.stride * s, *V = sg.vk + sg.stride * s, *Wf = sg.wk + sg.stride * s;
            for (int k = 1 + kbeg; k <= a.nkk - 1; k += kstep) {
                const float u = 0.5f * (U[sidx3(a, i, j, k)] + U[sidx3(a, i + 1, j, k)]);
                const float v = 0.5f * (V[sidx3(a, i, j, k)] + V[sidx3(a, i, j + 1, k)]);
                const float w = 0.5f * (Wf[sidx3(a, i, j, k)] + Wf[sidx3(a, i, j, k + 1)]);
                if (k < a.ks) { a.uks[x.at(0, k)] = u; a.vks[x.at(0, k)] = v; a.wks[x.at(0, k)] = w; }
                g = net_maxd(g, sqrt((double)(u * u + v * v)));
            }
        }
        if (!IL)
            for (int d = 16; d > 0; d >>= 1) g = fmax(g, __shfl_xor_sync(0xffffffffu, g, d));
        if ((IL || kbeg == 0) && g > 0.0)
            atomicMax(&a.sit[s].geschw_bits, (unsigned long long)__double_as_longlong(g));
    });
}

// border copies UK[NII+1] = UK[NII], VK[.][NJJ+1] = VK[.][NJJ] on levels 1..NKK-1 (:422-429)
__global__ void k_setup_border(KArgs a, Staging sg) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nk = a.nkk - 1;
    const long long per = (long long)(a.njj + a.nii) * nk;
    const long long s = t / per;
    if (s >= a.nb) return;
    const long long r = t - s * per;
    float *U = sg.uk + sg.stride * s, *V = sg.vk + sg.stride * s;
    const int k = 1 + (int)(r % nk);
    const int q = (int)(r / nk);
    if (q < a.njj) {
        const int j = 1 + q;
        U[sidx3(a, a.nii + 1, j, k)] = U[sidx3(a, a.nii, j, k)];
    } else {
        const int i = 1 + (q - a.njj);
        V[sidx3(a, i, a.njj + 1, k)] = V[sidx3(a, i, a.njj, k)];
    }
}

// k and eps initialisation on every level (:211-227, 410-510): TURB = 0.001, TDISS = 1e-7 on
// levels 1..NKK+1, then TURB from the velocity and the variances on levels 1..NKK-1.
__global__ void k_setup_turb(KArgs a, Staging sg, const float *varw, const float *z0_init) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nk2 = a.nkk + 2;
    const long long per = (long long)a.nii * a.njj * nk2;
    const long long s = t / per;
    if (s >= a.nb) return;
    const SitDev &S = a.sit[s];
    if (S.turb_init) return;
    long long r = t - s * per;
    const int k = (int)(r % nk2);
    r /= nk2;
    const int j = 1 + (int)(r % a.njj);
    const int i = 1 + (int)(r / a.njj);
    if (k < 1) return;
    const size_t o = sg.stride * s + sidx3(a, i, j, k);
    float tk = 0.001f;
    sg.tdiss[o] = 0.0000001f;
    if (k <= a.nkk - 1) {
        const float u = sg.uk[o], v = sg.vk[o];
        const double wh = net_maxd(sqrt((double)(u * u + v * v)), 0.01);
        const int col = i * a.nj2 + j;
        float U0int = (float)(wh * (0.2 * pow(wh, -0.9) + 0.32 * (double)z0_init[col] + 0.18));
        U0int = (float)net_maxd((double)U0int, 0.3) * S.std_dev_v;
        const float V0int = S.v0_1;
        tk = (float)(0.5 * (double)(U0int * U0int + V0int * V0int + varw[(size_t)s * a.ncols + col]));
    }
    sg.turb[o] = tk;
}

// velocities (and k, eps) inside buildings set to zero (:518-575)
template <bool IL>
__global__ void k_setup_zero(KArgs a, Staging sg, int model) {
    col_loop<IL>(a, false, [&](int s, int col, int i, int j, const Acc<IL> &x, int kbeg, int kstep) {
        if (i < 1 || i > a.nii || j < 1 || j > a.njj) return;
        if (!(a.cflags[col] & F_ADV)) return;
        const ColMeta m = a.meta[col];
        float *U = sg.uk + sg.stride * s, *V = sg.vk + sg.stride * s, *Wf = sg.wk + sg.stride * s;
        for (int k = 1 + kbeg; k <= m.vi; k += kstep) {
            if (m.kkart < k) continue;
            U[sidx3(a, i, j, k)] = 0;
            if (i == a.nii) U[sidx3(a, i + 1, j, k)] = 0;
            V[sidx3(a, i, j, k)] = 0;
            if (j == a.njj) V[sidx3(a, i, j + 1, k)] = 0;
            Wf[sidx3(a, i, j, k)] = 0;
            if (k == m.vi) Wf[sidx3(a, i, j, k + 1)] = 0;
            if (model != 1) {
                sg.turb[sg.stride * s + sidx3(a, i, j, k)] = 0;
                sg.tdiss[sg.stride * s + sidx3(a, i, j, k)] = 0;
            }
            a.uks[x.at(0, k)] = 0; a.vks[x.at(0, k)] = 0; a.wks[x.at(0, k)] = 0;
        }
    });
}

// staging (full height) <-> device layout (levels 0..KS-1)
template <bool IL>
__global__ void k_gather(KArgs a, Staging sg, int model, int to_dev) {
    col_loop<IL>(a, false, [&](int s, int col, int, int, const Acc<IL> &x, int kbeg, int kstep) {
        const size_t so = sg.stride * s + (size_t)col * (a.nkk + 2);
        const int nk2 = a.nkk + 2;
        const int nf = (model != 1) ? 5 : 3;
        float *dev[5] = {a.uk, a.vk, a.wk, a.turb, a.tdiss};
        float *stag[5] = {sg.uk, sg.vk, sg.wk, sg.turb, sg.tdiss};
        for (int f = 0; f < nf; ++f) {
            for (int k = kbeg; k < a.ks; k += kstep) {
                if (to_dev) dev[f][x.at(0, k)] = (k < nk2) ? stag[f][so + k] : 0.0f;
                else if (k < nk2) stag[f][so + k] = dev[f][x.at(0, k)];
            }
        }
    });
}

// Admission of the reciprocal form of ConvToInt(x*Frund)/Frund (quantd_r): for each situation,
// Markstein's quotient is compared with the IEEE quotient for every integer n in [2^30, 2^31),
// i.e. every 31-bit significand.  Every other dividend of that step is such an integer scaled by a
// power of two (ConvToInt gives magnitudes up to 2^31; 0 and the signs are exact), and scaling by
// a power of two changes no rounding of the three operations while no value leaves the normal
// range, so the comparison covers them all.
__global__ void k_rcp_check(KArgs a, int *bad) {
    const int s = blockIdx.y;
    if (s >= a.nb || !a.sit[s].quantise) return;
    const double b = a.sit[s].frund, y = a.sit[s].rfrund;
    const unsigned long long n0 = 1ull << 30;
    bool fail = false;
    for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < n0;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        const double n = (double)(n0 + t);
        const double q0 = n * y;
        fail |= (fma(fma(-q0, b, n), y, q0) != n / b);
    }
    if (__any_sync(0xffffffffu, fail) && (threadIdx.x & 31) == 0) atomicOr(bad + s, 1);
}

__global__ void k_rcp_set(KArgs a, const int *bad) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < a.nb) a.sit[s].rcp_ok = (a.sit[s].quantise && bad[s] == 0) ? 1 : 0;
}

// unrealistic-speed counts and non-finite values (:1193-1243)
template <bool IL>
__global__ void k_postcheck(KArgs a, int *counts) {
    col_loop<IL>(a, false, [&](int s, int col, int i, int j, const Acc<IL> &x, int kbeg, int kstep) {
        if (i < 1 || i > a.nii || j < 1 || j > a.njj) return;
        if (!(a.cflags[col] & F_ADV)) return;
        const ColMeta m = a.meta[col];
        const float limit = (float)(10 * __longlong_as_double((long long)a.sit[s].geschw_bits));
        int cu = 0, cv = 0, cw = 0, cn = 0;
        for (int k = 1 + kbeg; k <= m.vi; k += kstep) {
            const float u = a.uk[x.at(0, k)], v = a.vk[x.at(0, k)], w = a.wk[x.at(0, k)];
            if (fabsf(u) > 55 || fabsf(u) > limit) cu++;
            if (fabsf(v) > 55 || fabsf(v) > limit) cv++;
            if (fabsf(w) > 20 || fabsf(w) > limit) cw++;
            if (!isfinite(u) || !isfinite(v) || !isfinite(w)) cn++;
        }
        if (cu) atomicAdd(counts + 4 * s + 0, cu);
        if (cv) atomicAdd(counts + 4 * s + 1, cv);
        if (cw) atomicAdd(counts + 4 * s + 2, cw);
        if (cn) atomicAdd(counts + 4 * s + 3, cn);
    });
}

// ---- DiagnosticFlowfield after the prognostic solve (DiagnosticFlowfield.cs:24-436) ----
// time step from the corner column's wind at KADVMAX (:30-31), one thread per situation
__global__ void k_diag_dtime(KArgs a, int kadvmax, float *dtime) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nb) return;
    const Acc<false> x = make_acc<false>(a, s, 1 * a.nj2 + 1);
    const float u = a.uk[x.at(0, kadvmax)], v = a.vk[x.at(0, kadvmax)];
    float DT = (float)(0.5 * (double)net_minf(a.dxk, a.dyk) / sqrt((double)(u * u + v * v)));
    dtime[s] = net_minf(DT, 5.0f);
}

// velocity correction without quantisation on levels 1..NKK-1 (:320-382)
__global__ void k_diag_velcorr(KArgs a, DiagTabs t) {
    col_loop<false>(a, false, [&](int s, int col, int i, int j, const Acc<false> &x, int kbeg, int kstep) {
        if (i < 2 || i > a.nii - 1 || j < 2 || j > a.njj - 1) return;
        const int KK = a.meta[col].kkart, KKW = a.meta[col - a.nj2].kkart, KKS = a.meta[col - 1].kkart;
        const float DXK = a.dxk, DYK = a.dyk, DT = t.dtime[s];
        const long long W = -(long long)a.nj2;
        for (int k = 1 + kbeg; k <= a.nkk - 1; k += kstep) {
            const float d = a.dpm[x.at(0, k)];
            const float DDPX = a.dpm[x.at(W, k)] - d, DDPY = a.dpm[x.at(-1, k)] - d;
            const float DDPZ = (k > KK + 1) ? a.dpm[x.at(0, k - 1)] - d : 0.0f;
            float &u = a.uk[x.at(0, k)], &v = a.vk[x.at(0, k)], &w = a.wk[x.at(0, k)];
            u = ((KK < k) && (KKW < k)) ? u + (DDPX / DXK * DT) : 0.0f;
            v = ((KK < k) && (KKS < k)) ? v + (DDPY / DYK * DT) : 0.0f;
            w = (KK + 1 < k) ? w + (DDPZ * 2 / (t.dzk[k] + t.dzk[k - 1]) * DT) : 0.0f;
        }
    });
}

// final vertical velocity of the columns outside the prognostic sub-domains, bottom-up
// (MicroscaleFlat.cs:389-462); one thread per (situation, column)
__global__ void k_diag_wfinal(KArgs a, DiagTabs t) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long s = g / a.ncols;
    if (s >= a.nb) return;
    const int col = (int)(g - s * a.ncols);
    const int i = col / a.nj2, j = col - i * a.nj2;
    if (i < 2 || i > a.nii - 1 || j < 2 || j > a.njj - 1) return;
    if (a.cflags[col] & F_ADV) return;
    const Acc<false> x = make_acc<false>(a, (int)s, col);
    const long long E = a.nj2, N = 1;
    const int KK = a.meta[col].kkart;
    const int KKW = a.meta[col - a.nj2].kkart, KKE = a.meta[col + a.nj2].kkart;
    const int KKS = a.meta[col - 1].kkart, KKN = a.meta[col + 1].kkart;
    const float DXK = a.dxk, DYK = a.dyk;
    for (int k = 1; k < a.nkk; ++k) {
        if (!(k > KK)) continue;
        const float dz = t.dzk[k];
        const float fwo1 = (k <= KKW) ? 0.0f : dz * DYK * a.uk[x.at(0, k)];
        const float fwo2 = (k <= KKE) ? 0.0f : dz * DYK * a.uk[x.at(E, k)];
        const float fsn1 = (k <= KKS) ? 0.0f : dz * DXK * a.vk[x.at(0, k)];
        const float fsn2 = (k <= KKN) ? 0.0f : dz * DXK * a.vk[x.at(N, k)];
        const float fbt1 = ((k <= KK + 1) || (k == 1)) ? 0.0f : DXK * DYK * a.wk[x.at(0, k)];
        a.wk[x.at(0, k + 1)] = (fwo1 - fwo2 + fsn1 - fsn2 + fbt1) / (DXK * DYK);
    }
}

}  // namespace

#define GRAL_COL_LAUNCH(kern, ...)                                                        \
    do {                                                                                  \
        if (a.il) kern<true><<<col_grid<true>(a), COL_WARPS * 32, 0, st>>>(__VA_ARGS__);  \
        else kern<false><<<col_grid<false>(a), COL_WARPS * 32, 0, st>>>(__VA_ARGS__);     \
    } while (0)

void launch_bc(const KArgs &a, const BcLists &bc, cudaStream_t st) {
    const dim3 blk(32, 8);
    const int units = a.il ? a.ngroups : a.nb;
    if (a.il) {
        k_bc_we<true><<<dim3((a.njj - 1 + 7) / 8, units), blk, 0, st>>>(a, bc);
        k_bc_sn<true><<<dim3((a.nii - 1 + 7) / 8, units), blk, 0, st>>>(a, bc);
    } else {
        k_bc_we<false><<<dim3((a.njj - 1 + 7) / 8, units), blk, 0, st>>>(a, bc);
        k_bc_sn<false><<<dim3((a.nii - 1 + 7) / 8, units), blk, 0, st>>>(a, bc);
    }
    GRAL_COL_LAUNCH(k_bc_top, a);
}

void launch_velcorr(const KArgs &a, cudaStream_t st) { GRAL_COL_LAUNCH(k_velcorr, a); }

void launch_average(const KArgs &a, cudaStream_t st) {
    if (a.il) k_average<true><<<col_grid<true, true>(a), COL_WARPS * 32, 0, st>>>(a);
    else k_average<false><<<col_grid<false>(a), COL_WARPS * 32, 0, st>>>(a);
}

void launch_bookkeeping(const KArgs &a, cudaStream_t st) {
    k_bookkeeping<<<(a.nb + 127) / 128, 128, 0, st>>>(a);
}

void launch_setup(const KArgs &a, const Staging &sg, int model, const float *varw, const float *z0_init,
                  cudaStream_t st) {
    GRAL_COL_LAUNCH(k_setup_uks, a, sg);
    if (model != 1) {
        const long long n = (long long)a.nb * a.nii * a.njj * (a.nkk + 2);
        k_setup_turb<<<(int)((n + 255) / 256), 256, 0, st>>>(a, sg, varw, z0_init);
    }
    const long long nb = (long long)a.nb * (a.njj + a.nii) * (a.nkk - 1);
    k_setup_border<<<(int)((nb + 255) / 256), 256, 0, st>>>(a, sg);
    GRAL_COL_LAUNCH(k_setup_zero, a, sg, model);
}

void launch_gather(const KArgs &a, const Staging &sg, int model, cudaStream_t st) {
    GRAL_COL_LAUNCH(k_gather, a, sg, model, 1);
}

void launch_scatter(const KArgs &a, const Staging &sg, int model, cudaStream_t st) {
    GRAL_COL_LAUNCH(k_gather, a, sg, model, 0);
}

void launch_diag_dtime(const KArgs &a, int kadvmax, float *dtime, cudaStream_t st) {
    k_diag_dtime<<<(a.nb + 127) / 128, 128, 0, st>>>(a, kadvmax, dtime);
}

void launch_diag_velcorr(const KArgs &a, const DiagTabs &t, cudaStream_t st) {
    k_diag_velcorr<<<col_grid<false>(a), COL_WARPS * 32, 0, st>>>(a, t);
}

void launch_diag_wfinal(const KArgs &a, const DiagTabs &t, cudaStream_t st) {
    const long long n = (long long)a.nb * a.ncols;
    k_diag_wfinal<<<(int)((n + 255) / 256), 256, 0, st>>>(a, t);
}

void launch_rcp_check(const KArgs &a, int *bad, cudaStream_t st) {
    k_rcp_check<<<dim3(512, a.nb), 256, 0, st>>>(a, bad);
    k_rcp_set<<<(a.nb + 127) / 128, 128, 0, st>>>(a, bad);
}

void launch_postcheck(const KArgs &a, int *counts, cudaStream_t st) {
    GRAL_COL_LAUNCH(k_postcheck, a, counts);
}

}  // namespace gral
