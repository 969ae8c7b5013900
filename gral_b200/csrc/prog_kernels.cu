// prog_kernels.cu -- the Jacobi-style passes of one SIMPLE iteration (boundary conditions,
// velocity correction, staggered averages, convergence bookkeeping), the per-situation set-up and
// the post-checks.  One warp per column with lanes over k unless stated otherwise; every pass
// only writes values no other thread of the same launch reads, exactly as the reference's
// parallel loops do (their results do not depend on thread order).
#include "prog_common.cuh"
#include "prog_kernels.cuh"

namespace gral {

namespace {

constexpr int COL_WARPS = 8;   // warps per block of the column kernels

struct ColTask {
    int s, col, i, j;
};

// Maps the calling warp to (active situation, column); false when out of range or inactive.
__device__ __forceinline__ bool col_task(const KArgs &a, ColTask &t) {
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nact = *a.nact;
    const long long sidx = gw / a.ncols;
    if (sidx >= nact) return false;
    t.s = a.act[sidx];
    if (!a.sit[t.s].active) return false;
    t.col = (int)(gw - sidx * a.ncols);
    t.i = t.col / a.nj2;
    t.j = t.col - t.i * a.nj2;
    return true;
}

inline int col_grid(const KArgs &a) {
    const long long warps = (long long)a.nb * a.ncols;
    return (int)((warps + COL_WARPS - 1) / COL_WARPS);
}

// ---- boundary conditions (PrognosticFlowfield.cs:595-714) ----
// W/E: one thread per (situation, row j, level k) walks the row's events in ascending i, which is
// the reference's sequential i loop; rows and levels are independent.
__global__ void k_bc_we(KArgs a, BcLists bc) {
    const int j = 2 + blockIdx.x * blockDim.y + threadIdx.y;
    const int sidx = blockIdx.y;
    if (j > a.njj || sidx >= *a.nact) return;
    const int s = a.act[sidx];
    if (!a.sit[s].active) return;
    const size_t sb = (size_t)s * a.ncols;
    const int ks = a.ks, nj2 = a.nj2;
    for (int e = bc.we_ptr[j]; e < bc.we_ptr[j + 1]; ++e) {
        const int ev = bc.we_ev[e];
        const int i = ev & 0xffff;
        const int VI = a.meta[i * nj2 + j].vi;
        for (int k = threadIdx.x; k <= VI; k += 32) {
            if (k < 1) continue;
            auto at = [&](int ii) { return (sb + (size_t)ii * nj2 + j) * ks + k; };
            if (ev & (1 << 16)) {
                const float u = a.uk[at(i - 2)];
                if (u >= 0) a.uk[at(i - 1)] = u;
                a.vk[at(i - 2)] = a.vk[at(i - 1)];
                a.wk[at(i - 2)] = a.wk[at(i - 1)];
            }
            if (ev & (1 << 17)) {
                const float u = a.uk[at(i + 2)];
                if (u <= 0) a.uk[at(i + 1)] = u;
                a.vk[at(i + 1)] = a.vk[at(i)];
                a.wk[at(i + 1)] = a.wk[at(i)];
            }
        }
    }
}

__global__ void k_bc_sn(KArgs a, BcLists bc) {
    const int i = 2 + blockIdx.x * blockDim.y + threadIdx.y;
    const int sidx = blockIdx.y;
    if (i > a.nii || sidx >= *a.nact) return;
    const int s = a.act[sidx];
    if (!a.sit[s].active) return;
    const size_t sb = (size_t)s * a.ncols;
    const int ks = a.ks, nj2 = a.nj2;
    for (int e = bc.sn_ptr[i]; e < bc.sn_ptr[i + 1]; ++e) {
        const int ev = bc.sn_ev[e];
        const int j = ev & 0xffff;
        const int VI = a.meta[i * nj2 + j].vi;
        for (int k = threadIdx.x; k <= VI; k += 32) {
            if (k < 1) continue;
            auto at = [&](int jj) { return (sb + (size_t)i * nj2 + jj) * ks + k; };
            if (ev & (1 << 16)) {
                const float v = a.vk[at(j - 2)];
                if (v >= 0) a.vk[at(j - 1)] = v;
                a.uk[at(j - 2)] = a.uk[at(j - 1)];
                a.wk[at(j - 2)] = a.wk[at(j - 1)];
            }
            if (ev & (1 << 17)) {
                const float v = a.vk[at(j + 2)];
                if (v <= 0) a.vk[at(j + 1)] = v;
                a.uk[at(j + 1)] = a.uk[at(j)];
                a.wk[at(j + 1)] = a.wk[at(j)];
            }
        }
    }
}

// top: level VerticalIndex copied to VerticalIndex+1 (:699-714); one thread per column
__global__ void k_bc_top(KArgs a) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long sidx = t / a.ncols;
    if (sidx >= *a.nact) return;
    const int s = a.act[sidx];
    if (!a.sit[s].active) return;
    const int col = (int)(t - sidx * a.ncols);
    const int i = col / a.nj2, j = col - (col / a.nj2) * a.nj2;
    if (i < 2 || i > a.nii - 1 || j < 2 || j > a.njj - 1) return;
    if (!(a.cflags[col] & F_ADV)) return;
    const int k = a.meta[col].vi;
    const size_t o = fidx(s, col, a.ncols, a.ks);
    a.wk[o + k + 1] = a.wk[o + k];
    a.uk[o + k + 1] = a.uk[o + k];
    a.vk[o + k + 1] = a.vk[o + k];
}

// ---- velocity correction with Frund quantisation in double (:904-949) ----
__global__ void k_velcorr(KArgs a) {
    ColTask t;
    if (!col_task(a, t)) return;
    if (t.i < 2 || t.i > a.nii - 1 || t.j < 2 || t.j > a.njj - 1) return;
    if (!(a.cflags[t.col] & F_VC)) return;
    const int lane = threadIdx.x & 31;
    const ColMeta m = a.meta[t.col];
    const SitDev &sd = a.sit[t.s];
    const float DT = sd.dtime, DXK = a.dxk, DYK = a.dyk;
    const double fr = sd.frund;
    const int q = sd.quantise;
    const size_t o = fidx(t.s, t.col, a.ncols, a.ks);
    const size_t oW = o - (size_t)a.nj2 * a.ks, oS = o - a.ks;
    const float *DPM = a.dpm;
    for (int k = lane; k <= m.vi; k += 32) {
        if (k < 1) continue;
        const float d = DPM[o + k];
        if (t.i > 2 && m.kkm_u < k)
            a.uk[o + k] = (float)quantd((double)(a.uk[o + k] + (DPM[oW + k] - d) / DXK * DT), fr, q);
        if (t.j > 2 && m.kkm_v < k)
            a.vk[o + k] = (float)quantd((double)(a.vk[o + k] + (DPM[oS + k] - d) / DYK * DT), fr, q);
        if (m.kkart + 1 < k)
            a.wk[o + k] = (float)quantd(
                (double)(a.wk[o + k] + (DPM[o + k - 1] - d) / (a.dzk[k] + a.dzk[k - 1]) * 2 * DT), fr, q);
        else
            a.wk[o + k] = 0;
    }
}

// ---- staggered -> cell-centre averages and the border copies (:958-1039) ----
__global__ void k_average(KArgs a) {
    ColTask t;
    if (!col_task(a, t)) return;
    if (t.i < 2 || t.i > a.nii - 1 || t.j < 2 || t.j > a.njj - 1) return;
    if (!(a.cflags[t.col] & F_VC)) return;
    const int lane = threadIdx.x & 31;
    const ColMeta m = a.meta[t.col];
    const int ks = a.ks, nj2 = a.nj2;
    const size_t o = fidx(t.s, t.col, a.ncols, ks);
    const size_t oE = o + (size_t)nj2 * ks, oN = o + ks;
    const int KK = m.kkart;
    for (int k = lane; k <= m.vi; k += 32) {
        if (k < m.kstart) continue;
        if (KK < k) {
            a.uks[o + k] = 0.5f * (a.uk[o + k] + a.uk[oE + k]);
            a.vks[o + k] = 0.5f * (a.vk[o + k] + a.vk[oN + k]);
        }
        if (KK + 1 < k) a.wks[o + k] = 0.5f * (a.wk[o + k] + a.wk[o + k + 1]);
        if (t.j == 2) a.uks[o - ks + k] = a.uks[o + k];
        if (t.j == a.njj - 1 && (a.cflags[t.i * nj2 + a.njj] & F_ADV)) a.uks[o + ks + k] = a.uks[o + k];
    }
    // VKS[1][j] = VKS[2][j] and VKS[NII][j] = VKS[NII-1][j] over all levels (:1018-1036)
    const bool west = (t.i == 2) && (a.cflags[1 * nj2 + t.j] & F_ADV);
    const bool east = (t.i == a.nii - 1) && (a.cflags[t.col] & F_ADV);
    if (west || east) {
        const size_t od = west ? o - (size_t)nj2 * ks : oE;
        for (int k = lane; k < ks; k += 32) a.vks[od + k] = a.vks[o + k];
    }
}

// ---- convergence bookkeeping (:1144-1178), one thread per situation ----
__global__ void k_bookkeeping(KArgs a) {
    const int sidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= *a.nact) return;
    const int s = a.act[sidx];
    SitDev &S = a.sit[s];
    if (!S.active) return;
    const float dumax = __uint_as_float(S.dumax_bits);
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
__global__ void k_setup_uks(KArgs a, Staging sg) {
    ColTask t;
    if (!col_task(a, t)) return;
    if (t.i < 1 || t.i > a.nii || t.j < 1 || t.j > a.njj) return;
    if (!(a.cflags[t.col] & F_ALLOC3)) return;
    const int lane = threadIdx.x & 31;
    const float *U = sg.uk + sg.stride * t.s, *V = sg.vk + sg.stride * t.s, *W = sg.wk + sg.stride * t.s;
    const size_t o = fidx(t.s, t.col, a.ncols, a.ks);
    double g = 0.0;
    for (int k = 1 + lane; k <= a.nkk - 1; k += 32) {
        const float u = 0.5f * (U[sidx3(a, t.i, t.j, k)] + U[sidx3(a, t.i + 1, t.j, k)]);
        const float v = 0.5f * (V[sidx3(a, t.i, t.j, k)] + V[sidx3(a, t.i, t.j + 1, k)]);
        const float w = 0.5f * (W[sidx3(a, t.i, t.j, k)] + W[sidx3(a, t.i, t.j, k + 1)]);
        if (k < a.ks) { a.uks[o + k] = u; a.vks[o + k] = v; a.wks[o + k] = w; }
        g = net_maxd(g, sqrt((double)(u * u + v * v)));
    }
    for (int d = 16; d > 0; d >>= 1) g = fmax(g, __shfl_xor_sync(0xffffffffu, g, d));
    if (lane == 0 && g > 0.0)
        atomicMax(&a.sit[t.s].geschw_bits, (unsigned long long)__double_as_longlong(g));
}

// border copies UK[NII+1] = UK[NII], VK[.][NJJ+1] = VK[.][NJJ] on levels 1..NKK-1 (:422-429)
__global__ void k_setup_border(KArgs a, Staging sg) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nk = a.nkk - 1;
    const long long per = (long long)(a.njj + a.nii) * nk;
    const long long sidx = t / per;
    if (sidx >= *a.nact) return;
    const int s = a.act[sidx];
    const long long r = t - sidx * per;
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

// velocities (and k, eps) inside buildings set to zero (:518-575)
__global__ void k_setup_zero(KArgs a, Staging sg, int model) {
    ColTask t;
    if (!col_task(a, t)) return;
    if (t.i < 1 || t.i > a.nii || t.j < 1 || t.j > a.njj) return;
    if (!(a.cflags[t.col] & F_ADV)) return;
    const int lane = threadIdx.x & 31;
    const ColMeta m = a.meta[t.col];
    float *U = sg.uk + sg.stride * t.s, *V = sg.vk + sg.stride * t.s, *W = sg.wk + sg.stride * t.s;
    const size_t o = fidx(t.s, t.col, a.ncols, a.ks);
    for (int k = 1 + lane; k <= m.vi; k += 32) {
        if (m.kkart < k) continue;
        U[sidx3(a, t.i, t.j, k)] = 0;
        if (t.i == a.nii) U[sidx3(a, t.i + 1, t.j, k)] = 0;
        V[sidx3(a, t.i, t.j, k)] = 0;
        if (t.j == a.njj) V[sidx3(a, t.i, t.j + 1, k)] = 0;
        W[sidx3(a, t.i, t.j, k)] = 0;
        if (k == m.vi) W[sidx3(a, t.i, t.j, k + 1)] = 0;
        if (model != 1) {
            sg.turb[sg.stride * t.s + sidx3(a, t.i, t.j, k)] = 0;
            sg.tdiss[sg.stride * t.s + sidx3(a, t.i, t.j, k)] = 0;
        }
        a.uks[o + k] = 0; a.vks[o + k] = 0; a.wks[o + k] = 0;
    }
}

// staging (full height) <-> slab (levels 0..KS-1)
__global__ void k_gather(KArgs a, Staging sg, int model, int to_slab) {
    ColTask t;
    if (!col_task(a, t)) return;
    const int lane = threadIdx.x & 31;
    const size_t o = fidx(t.s, t.col, a.ncols, a.ks);
    const size_t so = sg.stride * t.s + (size_t)t.col * (a.nkk + 2);
    const int nk2 = a.nkk + 2;
    const int nf = (model != 1) ? 5 : 3;
    float *slab[5] = {a.uk, a.vk, a.wk, a.turb, a.tdiss};
    float *stag[5] = {sg.uk, sg.vk, sg.wk, sg.turb, sg.tdiss};
    for (int f = 0; f < nf; ++f) {
        for (int k = lane; k < a.ks; k += 32) {
            if (to_slab) slab[f][o + k] = (k < nk2) ? stag[f][so + k] : 0.0f;
            else if (k < nk2) stag[f][so + k] = slab[f][o + k];
        }
    }
}

// unrealistic-speed counts and non-finite values (:1193-1243)
__global__ void k_postcheck(KArgs a, int *counts) {
    ColTask t;
    if (!col_task(a, t)) return;
    if (t.i < 1 || t.i > a.nii || t.j < 1 || t.j > a.njj) return;
    if (!(a.cflags[t.col] & F_ADV)) return;
    const int lane = threadIdx.x & 31;
    const ColMeta m = a.meta[t.col];
    const SitDev &sd = a.sit[t.s];
    const float limit = (float)(10 * __longlong_as_double((long long)sd.geschw_bits));
    const size_t o = fidx(t.s, t.col, a.ncols, a.ks);
    int cu = 0, cv = 0, cw = 0, cn = 0;
    for (int k = 1 + lane; k <= m.vi; k += 32) {
        const float u = a.uk[o + k], v = a.vk[o + k], w = a.wk[o + k];
        if (fabsf(u) > 55 || fabsf(u) > limit) cu++;
        if (fabsf(v) > 55 || fabsf(v) > limit) cv++;
        if (fabsf(w) > 20 || fabsf(w) > limit) cw++;
        if (!isfinite(u) || !isfinite(v) || !isfinite(w)) cn++;
    }
    for (int d = 16; d > 0; d >>= 1) {
        cu += __shfl_xor_sync(0xffffffffu, cu, d);
        cv += __shfl_xor_sync(0xffffffffu, cv, d);
        cw += __shfl_xor_sync(0xffffffffu, cw, d);
        cn += __shfl_xor_sync(0xffffffffu, cn, d);
    }
    if (lane == 0 && (cu | cv | cw | cn)) {
        atomicAdd(counts + 4 * t.s + 0, cu);
        atomicAdd(counts + 4 * t.s + 1, cv);
        atomicAdd(counts + 4 * t.s + 2, cw);
        atomicAdd(counts + 4 * t.s + 3, cn);
    }
}

}  // namespace

void launch_bc(const KArgs &a, const BcLists &bc, cudaStream_t st) {
    const dim3 blk(32, 8);
    k_bc_we<<<dim3((a.njj - 1 + 7) / 8, a.nb), blk, 0, st>>>(a, bc);
    k_bc_sn<<<dim3((a.nii - 1 + 7) / 8, a.nb), blk, 0, st>>>(a, bc);
    const long long n = (long long)a.nb * a.ncols;
    k_bc_top<<<(int)((n + 255) / 256), 256, 0, st>>>(a);
}

void launch_velcorr(const KArgs &a, cudaStream_t st) {
    k_velcorr<<<col_grid(a), COL_WARPS * 32, 0, st>>>(a);
}

void launch_average(const KArgs &a, cudaStream_t st) {
    k_average<<<col_grid(a), COL_WARPS * 32, 0, st>>>(a);
}

void launch_bookkeeping(const KArgs &a, cudaStream_t st) {
    k_bookkeeping<<<(a.nb + 127) / 128, 128, 0, st>>>(a);
}

void launch_setup(const KArgs &a, const Staging &sg, int model, cudaStream_t st) {
    k_setup_uks<<<col_grid(a), COL_WARPS * 32, 0, st>>>(a, sg);
    const long long nb = (long long)a.nb * (a.njj + a.nii) * (a.nkk - 1);
    k_setup_border<<<(int)((nb + 255) / 256), 256, 0, st>>>(a, sg);
    k_setup_zero<<<col_grid(a), COL_WARPS * 32, 0, st>>>(a, sg, model);
}

void launch_gather(const KArgs &a, const Staging &sg, int model, cudaStream_t st) {
    k_gather<<<col_grid(a), COL_WARPS * 32, 0, st>>>(a, sg, model, 1);
}

void launch_scatter(const KArgs &a, const Staging &sg, int model, cudaStream_t st) {
    k_gather<<<col_grid(a), COL_WARPS * 32, 0, st>>>(a, sg, model, 0);
}

void launch_postcheck(const KArgs &a, int *counts, cudaStream_t st) {
    k_postcheck<<<col_grid(a), COL_WARPS * 32, 0, st>>>(a, counts);
}

}  // namespace gral
